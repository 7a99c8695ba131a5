/*
 * rt_cuda.h — C ABI of the B200 (sm_100a) wavefront path tracer, librtcuda.so.
 *
 * This is the `cuda` arm of the reference's backend dispatch
 * (src/main.rs:405-453). Each entry point replaces one call of the
 * reference's Metal backend, src/raytracer/metal/renderer.rs; the mapping
 * is given beside each declaration. Plain C types only: a Rust crate binds
 * it with an `extern "C"` block (the reference is Rust).
 *
 * Conventions
 *  - Every function returns an rt_status (0 = RT_OK, negative = error);
 *    rt_last_error() gives the message of the most recent failure on the
 *    calling thread.
 *  - A session owns all of its device memory and one CUDA stream; calls are
 *    synchronous on that stream. One session per host thread (the reference's
 *    PtSession is not Send, renderer.rs:256-259).
 *  - A session lives on the device that was current when it was created.
 *    Every call that takes a session makes that device current for its
 *    duration and restores the caller's current device before returning,
 *    so sessions on several GPUs can be driven from one thread.
 *  - Output buffers are caller-allocated host memory unless the name says
 *    `_device`.
 *  - Seeding is per (pixel, sample) exactly as Pcg32::for_pixel_sample
 *    (src/raytracer/pt/sampler.rs:24-32), so sample ranges rendered in any
 *    split add up to the same image.
 */
#ifndef RT_CUDA_H
#define RT_CUDA_H

#include <stddef.h>
#include <stdint.h>

#include "rt_scene.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef enum rt_status {
    RT_OK = 0,
    RT_ERR_INVALID = -1,   /* bad argument or scene (indices out of range, ...) */
    RT_ERR_CUDA = -2,      /* a CUDA runtime call failed */
    RT_ERR_OOM = -3,       /* device allocation failed */
    RT_ERR_DEVICE = -4,    /* a kernel reported a bounded-loop or capacity overrun */
    RT_ERR_IO = -5,        /* checkpoint file could not be read or written */
    RT_ERR_MISMATCH = -6   /* checkpoint does not match this session */
} rt_status;

typedef struct rt_session rt_session;

/* Flatten the scene (binned-SAH BLAS per mesh + TLAS over instances,
 * collapsed to 8-wide quantised nodes; light BVH; materials) and upload it.
 * Replaces PtSession::new / WfSession::new (renderer.rs:275, 518) and
 * GpuPtScene::build (src/raytracer/metal/gpu_scene.rs:306-753). The
 * descriptor is only read during the call. */
int rt_session_create(const rt_scene_desc* scene, const rt_params* params, rt_session** out);

/* Free the session's device memory and stream. NULL is accepted. */
int rt_session_destroy(rt_session* s);

/* Message of the last failure on this thread ("" if none). */
const char* rt_last_error(void);

/* Render `count` more samples per pixel, sample indices
 * [sample_start, sample_start + count), adding them to the f64
 * accumulator. Replaces PtSession::render_samples / WfSession::render_samples
 * (renderer.rs:410-437, 672-749). */
int rt_render_samples(rt_session* s, uint32_t sample_start, uint32_t count);

/* Zero the accumulators (beauty and AOVs). */
int rt_reset(rt_session* s);

/* Limits of the device's bounded loops for the following calls, as
 * rt_params.max_trav_steps and wait_polls (0 = the defaults, 2^22 traversal
 * steps per ray and 2^24 polls per tensor-core pipeline wait). A loop that
 * reaches its limit ends, sets the session's device error word, and the call
 * returns RT_ERR_DEVICE; the session stays usable (rt_reset, then render
 * again). The reference's counterpart is the GPU watchdog retry of
 * PtSession::render_samples (src/raytracer/metal/renderer.rs:406-437). */
int rt_set_limits(rt_session* s, uint32_t max_trav_steps, uint32_t wait_polls);

/* Copy the f64 accumulator: 4 doubles per pixel (r, g, b sums, sample
 * weight), row-major from the top-left pixel. Replaces
 * PtSession::sum_and_weight (renderer.rs:476-490). */
int rt_read_accum(rt_session* s, double* rgbw);

/* Beauty image: 3 floats per pixel = sum / weight. Replaces
 * PtSession::image (renderer.rs:455-471). */
int rt_read_image(rt_session* s, float* rgb);

/* AOV sums: 12 floats per pixel in the reference's layout
 * (src/raytracer/metal/kernel_pt.metal:1846-1847 and 2435-2452):
 * 0-2 albedo, 3-5 normal, 6 depth, 7 id (first writer), 8-10 diffuse
 * share, 11 hit count. Requires params.aovs = 1. Feeds render_pt_film's
 * decode (renderer.rs:180-217). */
int rt_read_aux(rt_session* s, float* aux12);

/* Checkpoint / resume of the f64 accumulator and completed-sample count.
 * Written to `path`.tmp then renamed (atomic). A load only succeeds when the
 * image size matches. Replaces save_checkpoint / load_checkpoint
 * (renderer.rs:219-254) with an f64 payload (magic "RCU1");
 * rt_checkpoint_save_rckp writes the reference's own f32 format ("RCKP",
 * width, height, passes done, f32 RGBW per pixel; renderer.rs:222-236), and
 * rt_checkpoint_load reads either, so a checkpoint of the Metal backend
 * resumes here and the other way round. */
int rt_checkpoint_save(rt_session* s, const char* path);
int rt_checkpoint_save_rckp(rt_session* s, const char* path);
int rt_checkpoint_load(rt_session* s, const char* path, uint32_t* samples_done);
/* The RCKP file of an RGBW accumulator held by the caller (f64 in, f32 on disk). */
int rt_rckp_write(const char* path, uint32_t width, uint32_t height, uint32_t passes_done, const double* rgbw);

/* Accumulation files of distributed renders (src/output/accum.rs): an
 * OpenEXR image with the f32 channels B, G, R (radiance sums of a sample
 * range) and count (samples per pixel), layer "accum".
 *  - rt_accum_exr_write: writes `rgbw` (4 doubles per pixel: RGB sum, count;
 *    rt_read_accum's layout) as uncompressed scanlines; replaces
 *    write_accum_exr (accum.rs:14-46).
 *  - rt_accum_exr_info / rt_accum_exr_read: size, then the sums and counts of
 *    such a file (scanline or one-level tiled, uncompressed, RLE, ZIPS or
 *    ZIP, FLOAT or HALF channels); replaces read_accum_exr (accum.rs:48-85).
 *  - rt_accum_merge: the mean image of any number of files (sum of sums /
 *    sum of counts, 0 where no samples), 3 floats per pixel; replaces merge
 *    (accum.rs:88-119), the `render merge` subcommand.
 * No GPU is involved; errors are RT_ERR_IO (unreadable or not such a file)
 * and RT_ERR_MISMATCH (resolution). */
int rt_accum_exr_write(const char* path, uint32_t width, uint32_t height, const double* rgbw);
int rt_accum_exr_info(const char* path, uint32_t* width, uint32_t* height);
int rt_accum_exr_read(const char* path, uint32_t width, uint32_t height, double* rgbw);
int rt_accum_merge(const char* const* paths, uint32_t n_paths, uint32_t width, uint32_t height, float* rgb);

/* Ray batch against the session's scene. `rays` holds 8 floats per ray in
 * two planes: [0, 4n) = (ox, oy, oz, unused), [4n, 8n) = (dx, dy, dz, tmax).
 * Directions are used as given; t is parametric along them.
 * Closest hit (any_hit = 0): prim = triangle index within its mesh,
 * inst = instance index, t = hit distance; 0xFFFFFFFF / +inf on a miss.
 * Any hit (any_hit = 1): prim = 1 if anything is hit with t < tmax, else 0;
 * inst and t may be NULL.
 * Host pointers. Replaces intersect_probe (renderer.rs:813-877). */
int rt_intersect_batch(rt_session* s, const float* rays, uint64_t n, int any_hit,
                       uint32_t* prim, uint32_t* inst, float* t);

/* Same, with device pointers, enqueued on the session's stream (or on
 * `stream` when non-NULL, a cudaStream_t) without a host synchronisation. */
int rt_intersect_batch_device(rt_session* s, const float* rays, uint64_t n, int any_hit,
                              uint32_t* prim, uint32_t* inst, float* t, void* stream);

/* Allocation-free ray batch, for callers that must not allocate GPU memory
 * once set up: code that owns a fixed device-memory budget reserved at
 * start-up (a real-time renderer's frame loop, an embedding host that routes
 * all GPU memory through its own allocator and forbids cudaMalloc/cudaFree
 * mid-frame because they synchronise the device and fragment its budget).
 * Same inputs, outputs and semantics as rt_intersect_batch (host pointers),
 * but the device staging for the rays, the results, the work counter and the
 * error word live in a fixed static device array of RT_NOALLOC_MAX_RAYS rays
 * (about 2.9 MB), reserved on every GPU that loads the library until the
 * process exits; nothing is allocated or freed per call. n beyond
 * RT_NOALLOC_MAX_RAYS is rejected with RT_ERR_INVALID. The call runs on the
 * session's device (as every session call does); the first call on a device
 * looks up the array's device address there (cudaGetSymbolAddress). The call
 * is synchronous: it copies the host rays in and the results out on the
 * session's stream and waits for that stream before it returns.
 * All calls share the one array: calls that overlap on the GPU (from several
 * threads or sessions on the same device) race on it and must be serialised
 * by the caller. No counterpart in the reference: its Metal backend has no
 * allocation-free entry point. */
#define RT_NOALLOC_MAX_RAYS 65536u
int rt_intersect_batch_noalloc(rt_session* s, const float* rays, uint64_t n, int any_hit,
                               uint32_t* prim, uint32_t* inst, float* t);

/* Statistics of the session and of its last rt_render_samples call. */
typedef struct rt_stats {
    uint64_t blas_nodes;        /* 8-wide BLAS nodes, all meshes */
    uint64_t tlas_nodes;        /* 8-wide TLAS nodes */
    uint64_t triangles;         /* unique triangles stored */
    uint64_t device_bytes;      /* device memory held by the session */
    uint64_t extension_rays;    /* last render: closest-hit rays traced */
    uint64_t shadow_rays;       /* last render: shadow rays traced */
    uint64_t samples;           /* last render: camera samples */
    uint64_t kernel_launches;   /* last render: kernels launched */
    double   extend_ms;         /* last render: time in the closest-hit kernel */
    double   shadow_ms;         /* last render: time in the shadow kernel */
    double   shade_ms;          /* last render: time in raygen + shade kernels */
    double   total_ms;          /* last render: wall time on the stream */
    uint64_t guide_steps;       /* last render: training iterations of the learned proposal */
    uint64_t guide_records;     /* last render: records in the final training batch */
    double   guide_loss;        /* last render: summed loss of the final training batch */
    uint64_t slabs;             /* last render: wavefront slabs (each: raygen, waves, accumulate) */
    uint64_t waves;             /* last render: waves per slab (extend/shade/shadow launches each) */
} rt_stats;

int rt_get_stats(rt_session* s, rt_stats* out);

/* Diagnostics of the hair BSDF (src/raytracer/pt/hair.rs f, pdf, sample)
 * as the shade kernel evaluates it in f32. params = sigma_a xyz, beta_m,
 * beta_n, eta. rt_hair_eval: per query (wo xyz, wi xyz, h) in the fiber
 * frame, f (3 floats) and pdf. rt_hair_sample: n consecutive samples for
 * one (wo, h) from the PCG32 stream of (pixel, sample): wi xyz, f rgb, pdf
 * (pdf 0 where sampling failed). */
int rt_hair_eval(const double* params, uint64_t n, const float* q, float* f, float* pdf);
int rt_hair_sample(const double* params, const double* wo, double h, uint64_t pixel, uint64_t sample, uint64_t n,
                   float* out);

/* Diagnostic: white-furnace estimate of one material on the GPU, using the
 * shade kernel's f32 BSDF sampling. `wo` is in the local frame (z = shading
 * normal), eta = transmitted / incident IOR. out[0] = mean of
 * lum(f)*|cos|/pdf over n samples, out[1..3] = mean RGB weight. The
 * reference's equivalent is the furnace_estimates unit test
 * (src/raytracer/pt/bxdf.rs:428-453). */
int rt_bsdf_furnace(const rt_material_desc* material, const double* wo, double eta, uint64_t n,
                    uint64_t seed, double* out);

/* Diagnostics: the device functions the render kernels use, run on caller
 * inputs, so tests can compare them one by one with the reference's
 * functions. Host pointers; each call stages through device memory and
 * waits for its result.
 *  - rt_pcg_streams: the first n u32 draws of the generator of (pixel[i],
 *    sample[i]) for i < m, n per row of `out` (Pcg32::for_pixel_sample and
 *    next_u32, src/raytracer/pt/sampler.rs:24-42); runs on the current device.
 *  - rt_light_sample_batch: the light the session's light BVH picks at
 *    points[3i..3i+3) with the uniform u[i], and its pick probability
 *    (LightSampler::sample, src/scene/light_sampler.rs:150-211); light
 *    0xFFFFFFFF and pmf 0 when the scene has no lights.
 *  - rt_light_pmf_batch: the probability of picking light[i] at points[i]
 *    (LightSampler::pmf, light_sampler.rs:213-238).
 *  - rt_transmittance_batch: the shadow kernel's transmittance of rays in
 *    rt_intersect_batch's layout (direction and distance tmax): the product
 *    of (1 - presence) over the cutout surfaces crossed before tmax, 0 when
 *    an opaque surface is crossed or the product falls below 1e-4
 *    (transmittance, src/raytracer/pt/mod.rs:1254-1306). */
int rt_pcg_streams(const uint64_t* pixel, const uint64_t* sample, uint32_t m, uint32_t n, uint32_t* out);
int rt_light_sample_batch(rt_session* s, const float* points, const float* u, uint32_t m,
                          uint32_t* light, float* pmf);
int rt_light_pmf_batch(rt_session* s, const float* points, const uint32_t* light, uint32_t m, float* pmf);
int rt_transmittance_batch(rt_session* s, const float* rays, uint64_t n, float* trans);

/* The session's CUDA stream (a cudaStream_t), for callers that time or
 * order work against it. */
void* rt_session_stream(rt_session* s);

/* Adaptive sampling (WfSession::set_adaptive, src/raytracer/metal/renderer.rs:
 * 580-584; rule of kernel_wf.metal:173-183): with tol > 0, from sample 32 on
 * a pixel with at least 16 samples receives no further samples once the 95%
 * confidence interval of its luminance, 1.96 sqrt(var / n), is below
 * tol * max(mean, 0.05). tol = 0 turns it off (the default). The weight
 * channel of the accumulator counts the samples each pixel actually took. */
int rt_set_adaptive(rt_session* s, double tol);

/* Average samples per pixel actually taken (WfSession::average_spp,
 * renderer.rs:586-591): the mean of the accumulator's weight channel. */
int rt_average_spp(rt_session* s, double* out);

/* The AOV film (src/output/film.rs: Film) of a session created with
 * params.aovs = 1, RT_FILM_FLOATS floats per pixel at the offsets below:
 * beauty, diffuse, specular (max(beauty - diffuse, 0)), albedo, normal (RGB /
 * XYZ), depth (mean over the samples that hit), id and its coverage. Decoded
 * on the device from the accumulator and the AOV sums as render_pt_film
 * (src/raytracer/metal/renderer.rs:180-217), each pixel by its own sample
 * count. */
#define RT_FILM_FLOATS 18
#define RT_FILM_BEAUTY 0
#define RT_FILM_DIFFUSE 3
#define RT_FILM_SPECULAR 6
#define RT_FILM_ALBEDO 9
#define RT_FILM_NORMAL 12
#define RT_FILM_DEPTH 15
#define RT_FILM_ID 16
int rt_read_film(rt_session* s, float* film);

/* The denoised beauty (3 floats per pixel) of a session's film (needs
 * params.aovs = 1) or of a film held by the caller (rt_denoise_film, run on
 * the current device): the reference's edge-avoiding a-trous filter
 * (src/output/denoise.rs:28-139; diffuse demodulated by albedo, 5 passes
 * guided by normal, depth and object id, specular added back). */
int rt_denoise(rt_session* s, float* rgb);
int rt_denoise_film(const float* film, uint32_t width, uint32_t height, float* rgb);

/* A film as the reference's multilayer EXR (src/output/multilayer.rs:
 * channels R G B, diffuse.*, specular.*, albedo.*, N.*, depth.Z, id.x,
 * id.coverage in name order; layer "rgba"; the id manifest "id:name;..." in
 * the render_rs/manifest attribute, NULL for none). Host only. */
int rt_film_exr_write(const char* path, uint32_t width, uint32_t height, const float* film, const char* manifest);

/* The session's learned directional proposal (rt_guide.h) when it renders
 * guided, else NULL. The session owns the handle: callers may pass it to
 * rt_guide_infer / rt_guide_get_params to inspect what the network has
 * learned, and must not destroy it. No counterpart in the reference (path
 * guiding is an unimplemented stretch goal there, ROADMAP.md:34). */
struct rt_guide* rt_session_guide(rt_session* s);

#ifdef __cplusplus
}
#endif

#endif /* RT_CUDA_H */

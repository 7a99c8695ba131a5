/*
 * pt_oracle.h — f64 CPU oracle for the render.rs path tracer.
 *
 * TEST INFRASTRUCTURE ONLY. This library restates the reference's CPU path
 * (anders94/render.rs, Rust, f64) so that tests, smoke() and the bench's
 * cpu_baseline leg can check and time the CUDA backend against it. Nothing in
 * the product links it; the CUDA backend never falls back to it.
 *
 * Sources restated (paths within the reference project):
 *   src/raytracer/pt/sampler.rs      PCG32 + per-(pixel, sample) seeding
 *   src/accel/bvh.rs                 binned-SAH BVH, traverse, any_hit
 *   src/geometry/mesh.rs             Mesh, Möller–Trumbore, Instance
 *   src/scene/mod.rs                 Scene::intersect (TLAS over instances)
 *   src/scene/camera.rs              camera rays, pixel filters
 *   src/scene/light.rs               light records
 *   src/scene/light_sampler.rs       light BVH sample / pmf
 *   src/scene/pbr.rs                 PbrParams, lobe weights
 *   src/raytracer/pt/bxdf.rs         Oren-Nayar, GGX-VNDF, clearcoat, fuzz, glass
 *   src/raytracer/pt/mod.rs          trace_full, sample_light, transmittance
 * Out of scope (no config uses them): media, SSS, hair, textures/patterns,
 * dome/IES lights, motion blur.
 */
#ifndef PT_ORACLE_H
#define PT_ORACLE_H

#include <stdint.h>
#include "rt_scene.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_scene oracle_scene;

/* Traversal work counters (reference binary BVH, both levels). */
typedef struct oracle_counters {
    uint64_t node_pops;      /* nodes popped from the traversal stack */
    uint64_t tri_tests;      /* ray-triangle tests */
    uint64_t inst_tests;     /* instance (TLAS leaf) visits */
    uint64_t rays;
} oracle_counters;

oracle_scene* oracle_scene_create(const rt_scene_desc* desc);
void          oracle_scene_destroy(oracle_scene* s);
/* Binary BVH sizes: total BLAS nodes and TLAS nodes. */
void          oracle_scene_stats(const oracle_scene* s, uint64_t* blas_nodes, uint64_t* tlas_nodes);

/* Ray batch: planes[0..4n) = (ox,oy,oz,-) per ray, planes[4n..8n) =
 * (dx,dy,dz,tmax). Directions are used as given; t is parametric.
 * Closest hit: prim/inst = 0xFFFFFFFF on a miss. Any hit: prim = 1/0. */
int oracle_intersect(const oracle_scene* s, const float* planes, uint64_t n, int any_hit,
                     uint32_t* prim, uint32_t* inst, double* t, oracle_counters* counters,
                     int threads);

/* Render samples [s0, s1) for the listed pixel indices (y*W + x).
 * rgb: 3 doubles per listed pixel (radiance SUM over the samples, each
 * sample firefly-clamped). aux (optional): 12 doubles per listed pixel in
 * the reference's GPU AOV layout (0-2 albedo sum, 3-5 normal sum, 6 depth
 * sum, 7 id, 8-10 diffuse sum, 11 hit count); the id is the majority vote
 * of the CPU film path. ray_counts (optional, 8 x u64): extension rays,
 * shadow rays, then node pops / triangle tests / instance visits of the
 * extension rays, then the same three for the shadow rays. */
int oracle_render(const oracle_scene* s, const rt_params* p, const uint32_t* pixels,
                  uint64_t n_pixels, uint32_t s0, uint32_t s1, double* rgb, double* aux,
                  uint64_t* ray_counts, int threads);

/* First n u32 outputs of Pcg32::for_pixel_sample(pixel, sample). */
void oracle_pcg_stream(uint64_t pixel, uint64_t sample, uint32_t n, uint32_t* out);
/* First n u32 outputs of Pcg32::new(seed, stream). */
void oracle_pcg_new_stream(uint64_t seed, uint64_t stream, uint32_t n, uint32_t* out);

/* BSDF helpers for lobe tests. wo is local (z = shading normal). */
int oracle_bsdf_eval(const rt_material_desc* m, const double* wo, const double* wi,
                     double eta, double* f_out, double* pdf_out);
/* Furnace: mean of lum(f)*|cos|/pdf over n BSDF samples from Pcg32::new(seed, stream). */
double oracle_bsdf_furnace(const rt_material_desc* m, const double* wo, double eta,
                           uint64_t n, uint64_t seed, uint64_t stream, double* rgb_out);

/* Light BVH queries. */
int    oracle_light_sample(const oracle_scene* s, const double* p, double u,
                           uint32_t* light, double* pmf);
double oracle_light_pmf(const oracle_scene* s, const double* p, uint32_t light);
void   oracle_env_eval_pdf(uint32_t w, uint32_t h, const float* rgb, uint64_t n, const double* dirs, double* rad,
                           double* pdf);
void   oracle_env_sample(uint32_t w, uint32_t h, const float* rgb, uint64_t n, const double* uv, double* dirs,
                         double* rad, double* pdf);
// pattern.rs:126-226: node `node` of d's pattern graph at n shading points,
// ctx = (s, t, P xyz, N xyz, footprint, dst_major st, dst_minor st) per
// point (13 doubles); rgb = 3 per point.
void   oracle_pattern_eval(const rt_scene_desc* d, uint32_t node, uint64_t n, const double* ctx, double* rgb);
// Closest hit of n rays (o, d: 6 doubles each): (t or -1, s, t, st density).
/* One analytic quadric against n world rays (6 doubles: origin, direction):
 * 10 doubles per ray (t or -1, point, normal, u, v, st density). */
void   oracle_quadric_intersect(const rt_quadric_desc* q, uint64_t n, const double* rays, double* out);
/* Real roots of coef[0] t^4 + ... + coef[4], ascending; returns the count. */
int    oracle_solve_quartic(const double* coef, double* roots);
/* Shadow-ray transmittance (mod.rs:1254-1306) of rays in the two-plane
 * layout (origin; direction, distance): RGB per ray. */
void   oracle_transmittance(const oracle_scene* s, const float* planes, uint64_t n, double* out, int threads);
void   oracle_intersect_st(const oracle_scene* s, uint64_t n, const double* rays, double* out);
// texture/cache.rs lookups on the mip chain of one w x h RGB texture: per
// query 7 doubles (s, t, footprint, -, -, -, 0) for the trilinear `sample`
// or (s, t, du s, du t, dv s, dv t, 1) for `sample_ewa`; 3 floats out.
void   oracle_texture_sample(uint32_t w, uint32_t h, const float* rgb, int wrap, uint64_t n, const double* q,
                             float* out);
// ies.rs:108-142: raw candela and normalised factor of a profile toward n
// light-local directions (3 doubles each).
void   oracle_ies_eval(uint32_t n_v, uint32_t n_h, const double* v, const double* h, const double* candela,
                       uint64_t n, const double* dirs, double* cd, double* factor);
// camera.rs:36-61: one pixel-filter offset per uniform.
void   oracle_filter_sample(int filter, double width, uint64_t n, const double* u, double* out);
/* Media (src/scene/medium.rs, src/raytracer/pt/volume.rs), for the
 * reference's own unit tests. n draws of sample_distance along the ray
 * (o, d) over [0, t_max] with throughput beta from the PCG32 stream of
 * (pixel, sample): sums of the pass weights and of the scatter weights
 * (3 doubles each); returns the number of scatters. */
uint64_t oracle_medium_sample(const rt_medium_desc* m, const double* o, const double* d, double t_max,
                              const double* beta, uint64_t pixel, uint64_t sample, uint64_t n, double* pass_sum,
                              double* scat_sum);
/* Mean over n estimates of the segment transmittance (3 doubles). */
void   oracle_medium_transmittance(const rt_medium_desc* m, const double* o, const double* d, double dist,
                                   uint64_t pixel, uint64_t sample, uint64_t n, double* mean);
/* Density multiplier at n points (3 doubles each). */
void   oracle_medium_density(const rt_medium_desc* m, uint64_t n, const double* p, double* out);
/* Henyey-Greenstein: phase at n cosines, or n sampled directions around
 * -wo from uniform pairs (u: 2 per draw; out: wi xyz, pdf). */
void   oracle_hg_phase(double g, uint64_t n, const double* cos_theta, double* out);
void   oracle_hg_sample(double g, const double* wo, uint64_t n, const double* u, double* out);
/* sss_medium (volume.rs:259-288): sigma_a, sigma_s (3 doubles each). */
void   oracle_sss_medium(const double* color, const double* dmfp, double* sigma_a, double* sigma_s);
/* Hair (src/raytracer/pt/hair.rs), params = sigma_a xyz, beta_m, beta_n,
 * eta. Per query (wo xyz, wi xyz, h): f rgb and pdf. */
void   oracle_hair_eval(const double* params, uint64_t n, const double* q, double* f, double* pdf);
/* n draws of hair::sample for (wo, h) from the PCG32 stream of (pixel,
 * sample): wi xyz, f rgb, pdf (pdf 0 when the draw failed). */
void   oracle_hair_sample(const double* params, const double* wo, double h, uint64_t pixel, uint64_t sample,
                          uint64_t n, double* out);
/* FiberFrame (hair.rs:378-401): h of (tangent, normal, wo). */
double oracle_fiber_h(const double* tangent, const double* normal, const double* wo);
/* One rounded-cone segment (curves.rs:67-169; p0, p1 = xyz radius) against
 * n rays (origin, direction; 6 doubles): t or -1, normal xyz, tangent xyz, v. */
void   oracle_curve_segment(const double* p0, const double* p1, double v0, double v1, uint64_t n,
                            const double* rays, double* out);

#ifdef __cplusplus
}
#endif

#endif

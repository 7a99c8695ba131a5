// session.cu — the C ABI of librtcuda.so (include/rt_cuda.h).
//
// A session flattens the scene once (flatten.cpp), uploads it, and owns the
// wavefront path state, queues and the f64 accumulator on one CUDA stream.
// All device waits in the kernels are bounded (traversal step cap, stack
// capacity); overruns set bits in a device error word that every call
// checks and reports as RT_ERR_DEVICE instead of hanging or faulting.

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "bvh_build.h"
#include "devmem.h"
#include "flatten.h"
#include "guide_internal.h"
#include "pt_kernels.cuh"
#include "rt_cuda.h"

using namespace rt;

namespace rt {

cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t st) {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    cudaMemPool_t pool;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (!pools[dev]) {
            cudaMemPoolProps props = {};
            props.allocType = cudaMemAllocationTypePinned;
            props.handleTypes = cudaMemHandleTypeNone;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            e = cudaMemPoolCreate(&pools[dev], &props);
            if (e != cudaSuccess) {
                pools[dev] = nullptr;
                return e;
            }
            uint64_t keep = ~0ull;
            cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
        }
        pool = pools[dev];
    }
    return cudaMallocFromPoolAsync(p, bytes, pool, st);
}

cudaError_t pool_free(void* p, cudaStream_t st) { return cudaFreeAsync(p, st); }

}  // namespace rt

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define CUDA_TRY(expr)                                                                         \
    do {                                                                                       \
        cudaError_t e_ = (expr);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            return fail(e_ == cudaErrorMemoryAllocation ? RT_ERR_OOM : RT_ERR_CUDA,            \
                        std::string(#expr) + ": " + cudaGetErrorString(e_));                  \
        }                                                                                      \
    } while (0)

// The text of a device error word (RT_DEVERR_* bits), shared by every
// entry point that reads one.
std::string device_error_text(uint32_t e) {
    std::string t = "device reported";
    if (e & RT_DEVERR_STACK) t += " traversal stack overflow";
    if (e & RT_DEVERR_ITER) t += " traversal step limit";
    if (e & ~(RT_DEVERR_STACK | RT_DEVERR_ITER)) t += " error bits " + std::to_string(e);
    return t;
}

// Makes a session's device current for the duration of an entry point and
// restores the caller's device afterwards, so a session created on one GPU
// runs there whatever device the calling thread has current.
struct DeviceScope {
    int prev = -1;
    cudaError_t status = cudaSuccess;
    explicit DeviceScope(int dev) {
        status = cudaGetDevice(&prev);
        if (status == cudaSuccess && prev != dev) status = cudaSetDevice(dev);
        else prev = -1;
    }
    ~DeviceScope() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

#define SESSION_DEVICE(s)                                                                      \
    DeviceScope dev_scope_((s)->device);                                                       \
    if (dev_scope_.status != cudaSuccess)                                                      \
        return fail(RT_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(dev_scope_.status))

#ifndef RT_TRAV_BLOCK
#define RT_TRAV_BLOCK 128
#endif
constexpr int TRAV_BLOCK = RT_TRAV_BLOCK;

// Adam steps per sample pass of a guided render: 0 selects the default of 3
// (on the two-room scene at 1280x720 and a 1024-pass budget, equal-time
// relMSE ratios to plain were 1.53 / 1.59 / 1.56 for 2 / 3 / 4 steps; a step
// costs ~0.5 ms per pass there).
uint32_t guide_steps_per_pass(uint32_t requested) { return requested ? std::min(16u, requested) : 3u; }
// Sample passes that train the proposal before it is kept fixed: 0 selects
// the default of 512. On the two-room scene at 1280x720 (2048 guided passes
// against plain path tracing at equal device time), budgets of 256 / 512 /
// 1024 / unlimited gave relMSE ratios of 2.00 / 2.06 / 1.91 / 1.73: after a
// few hundred passes the proposal barely improves while training still
// costs ~2.4 ms per pass.
uint64_t guide_train_budget(uint32_t requested) { return requested ? requested : 512u; }
constexpr int SHADE_BLOCK = 128;

}  // namespace

namespace rt {
std::string& accum_error() { return g_err; }
int film_decode_device(const double* accum, const float* aux, uint32_t npix, float* film, cudaStream_t st);
int denoise_device(const float* film, uint32_t w, uint32_t h, float* rgb, cudaStream_t st);
}  // namespace rt

struct rt_session {
    HostScene host;
    DevScene S{};
    rt_params params{};
    cudaStream_t stream = nullptr;
    int device = 0;                // the device the session was created on; every call runs there
    int sm_count = 148;
    std::vector<void*> allocs;
    uint64_t device_bytes = 0;
    // path state
    Paths paths{};
    uint32_t slab_samples = 1;     // sample passes per slab
    double* lum_stats = nullptr;   // per pixel: luminance sum, sum of squares, count, pad
    float adaptive_tol = 0.0f;     // rt_set_adaptive
    double* accum = nullptr;       // 4 doubles per pixel
    float* aux = nullptr;          // 12 floats per pixel
    uint32_t* err = nullptr;       // device error word
    unsigned long long* stats = nullptr;
    uint32_t* fetch = nullptr;     // ray-batch work counter
    uint32_t npix = 0;
    uint32_t samples_done = 0;
    // learned proposal (params.guided)
    rt_guide* guide = nullptr;
    uint64_t guide_slabs = 0;    // slabs rendered with the guide (drives the slab growth)
    uint64_t guide_trained_passes = 0;  // sample passes whose vertices trained the network
    uint32_t guide_prev_k = 0;   // sample passes of the previous guided slab
    uint64_t guide_records = 0;
    double guide_loss = 0.0;
    // ray-batch staging for host-pointer calls
    void* batch_buf = nullptr;
    size_t batch_cap = 0;
    rt_stats last{};
    cudaEvent_t ev[8] = {};
    std::vector<cudaEvent_t> evpool;
    int trav_grid = 148 * 4;      // resident blocks of the traversal kernels

    template <class T>
    int alloc(T** p, size_t count) {
        size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
        void* v = nullptr;
        cudaError_t e = pool_alloc(&v, bytes, stream);
        if (e != cudaSuccess)
            return fail(e == cudaErrorMemoryAllocation ? RT_ERR_OOM : RT_ERR_CUDA,
                        std::string("device allocation (") + std::to_string(bytes) + " B): " + cudaGetErrorString(e));
        allocs.push_back(v);
        device_bytes += bytes;
        *p = (T*)v;
        return RT_OK;
    }
    template <class T>
    int upload(const T** dst, const std::vector<T>& src) {
        T* d = nullptr;
        int rc = alloc(&d, src.size());
        if (rc) return rc;
        if (!src.empty()) CUDA_TRY(cudaMemcpyAsync(d, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
        *dst = d;
        return RT_OK;
    }
    int check_device_error() {
        uint32_t e = 0;
        CUDA_TRY(cudaMemcpyAsync(&e, err, 4, cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        if (e) {
            cudaMemsetAsync(err, 0, 4, stream);
            cudaStreamSynchronize(stream);
            return fail(RT_ERR_DEVICE, device_error_text(e));
        }
        return RT_OK;
    }
    ~rt_session() {
        DeviceScope scope(device);
        if (stream) cudaStreamSynchronize(stream);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        for (auto& e : evpool) cudaEventDestroy(e);
        for (void* p : allocs) pool_free(p, stream);
        if (batch_buf) cudaFree(batch_buf);
        if (guide) rt_guide_destroy(guide);
        if (stream) {
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
    }
};

// Scenes with analytic quadrics or curve sets run the kernel variants that
// test them (the others keep their registers for the BVH walk).
// Quadrics or curve sets: the traversal kernels' extra-geometry variants
// (quadrics first, segment leaves); scenes with motion blur run them too,
// with rays placed at their shutter time.
static bool extra_geometry(const rt_session* s) { return s->S.n_quadrics > 0 || s->S.any_curves; }

// The ray-batch kernel variant for the query and the scene.
static void launch_intersect(rt_session* s, int any_hit, int grid, cudaStream_t st, const float4* o, const float4* d,
                             uint64_t n, uint32_t* prim, uint32_t* inst, float* t, uint32_t* fetch, uint32_t* err) {
    const bool quad = extra_geometry(s);
    if (any_hit && quad)
        k_intersect<TRAV_BLOCK, true, true><<<grid, TRAV_BLOCK, 0, st>>>(s->S, o, d, n, prim, inst, t, fetch, err);
    else if (any_hit)
        k_intersect<TRAV_BLOCK, true><<<grid, TRAV_BLOCK, 0, st>>>(s->S, o, d, n, prim, inst, t, fetch, err);
    else if (quad)
        k_intersect<TRAV_BLOCK, false, true><<<grid, TRAV_BLOCK, 0, st>>>(s->S, o, d, n, prim, inst, t, fetch, err);
    else
        k_intersect<TRAV_BLOCK, false><<<grid, TRAV_BLOCK, 0, st>>>(s->S, o, d, n, prim, inst, t, fetch, err);
}

extern "C" {

const char* rt_last_error(void) { return g_err.c_str(); }

int rt_session_create(const rt_scene_desc* scene, const rt_params* params, rt_session** out) {
    if (!out) return fail(RT_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!scene || !params) return fail(RT_ERR_INVALID, "scene or params is NULL");
    if (params->max_depth == 0 || params->max_depth > 255) return fail(RT_ERR_INVALID, "max_depth must be in 1..255");
    auto* s = new rt_session();
    s->params = *params;
    std::string err;
    // The device builder covers static triangle meshes; scenes with curve
    // sets or motion blur are built on the host (the same SAH rules and wide
    // layout).
    const bool device_bvh = params->bvh_build == 0 &&
                            !(scene && (scene->n_curves || scene->n_mesh_motion || scene->n_instance_motion));
    if (!flatten_scene(scene, &s->host, &err, !device_bvh)) {
        delete s;
        return fail(RT_ERR_INVALID, err);
    }
    int dev = 0;
    cudaError_t de = cudaGetDevice(&dev);
    if (de != cudaSuccess) {
        delete s;
        return fail(RT_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(de));
    }
    s->device = dev;
    cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, dev);
    {
        // Persistent traversal grids: every resident block slot on every SM.
        int nb = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_extend<TRAV_BLOCK, false>, TRAV_BLOCK, 0);
        s->trav_grid = s->sm_count * std::max(nb, 1);
    }
    cudaError_t ce = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (ce != cudaSuccess) {
        delete s;
        return fail(RT_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(ce));
    }
    for (auto& e : s->ev) cudaEventCreate(&e);
    HostScene& H = s->host;
    DevScene& S = s->S;
    int rc = 0;
    if (device_bvh) {
        DeviceBvh b;
        rc = device_build_scene(scene, &H, &b, s->stream, &err);
        for (void* p : b.allocations) s->allocs.push_back(p);
        if (rc) {
            delete s;
            return fail(rc, err);
        }
        s->device_bytes += b.n_nodes * WIDE_NODE_WORDS * 16 + H.n_tris * 48 + (uint64_t)scene->n_instances * 64;
        S = H.scalars;
        S.nodes = b.nodes;
        S.tris = b.tris;
        S.inst_xf = b.inst_xf;
        S.inst = b.inst;
        S.items = b.items;
    } else {
        S = H.scalars;
        rc = rc ? rc : s->upload((const uint4**)&S.nodes, H.nodes);
        rc = rc ? rc : s->upload((const float4**)&S.tris, H.tris);
        rc = rc ? rc : s->upload((const float4**)&S.inst_xf, H.inst_xf);
        rc = rc ? rc : s->upload((const uint4**)&S.inst, H.inst);
        rc = rc ? rc : s->upload((const uint2**)&S.items, H.items);
    }
    S.max_steps = params->max_trav_steps ? params->max_trav_steps : RT_MAX_TRAV_STEPS;
    rc = rc ? rc : s->upload(&S.meshes, H.meshes);
    rc = rc ? rc : s->upload(&S.orig_idx, H.orig_idx);
    rc = rc ? rc : s->upload(&S.normals, H.normals);
    // Texture coordinates and the pattern graph: null pointers when absent.
    if (!H.st.empty()) rc = rc ? rc : s->upload(&S.st, H.st);
    if (!H.mat_pat.empty()) {
        rc = rc ? rc : s->upload(&S.inst_scale, H.inst_scale);
        rc = rc ? rc : s->upload(&S.patterns, H.patterns);
        rc = rc ? rc : s->upload(&S.ramp, H.ramp);
        rc = rc ? rc : s->upload(&S.mat_pat, H.mat_pat);
        rc = rc ? rc : s->upload(&S.binds, H.binds);
        rc = rc ? rc : s->upload(&S.pbr, H.pbr);
        if (!H.textures.empty()) {
            rc = rc ? rc : s->upload(&S.textures, H.textures);
            rc = rc ? rc : s->upload(&S.tex_mips, H.tex_mips);
            rc = rc ? rc : s->upload(&S.texels, H.texels);
        }
        if (!H.udim.empty()) rc = rc ? rc : s->upload(&S.udim, H.udim);
    }
    if (!H.ies.empty()) {
        rc = rc ? rc : s->upload(&S.ies, H.ies);
        rc = rc ? rc : s->upload(&S.ies_data, H.ies_data);
    }
    if (!H.quadrics.empty()) rc = rc ? rc : s->upload(&S.quadrics, H.quadrics);
    if (!H.media.empty()) rc = rc ? rc : s->upload(&S.media, H.media);
    if (!H.hair.empty()) rc = rc ? rc : s->upload(&S.hair, H.hair);
    if (!H.tris1.empty()) rc = rc ? rc : s->upload((const float4**)&S.tris1, H.tris1);
    if (!H.inst_motion.empty()) {
        rc = rc ? rc : s->upload(&S.inst_motion, H.inst_motion);
        rc = rc ? rc : s->upload(&S.inst_mot, H.inst_mot);
    }
    rc = rc ? rc : s->upload(&S.materials, H.materials);
    rc = rc ? rc : s->upload(&S.lights, H.lights);
    rc = rc ? rc : s->upload(&S.lbvh, H.lbvh);
    rc = rc ? rc : s->upload(&S.light_leaf, H.light_leaf);
    rc = rc ? rc : s->upload(&S.inf_lights, H.inf_lights);
    rc = rc ? rc : s->upload(&S.inf_power, H.inf_power);
    rc = rc ? rc : s->upload((const float4**)&S.env, H.env);
    rc = rc ? rc : s->upload(&S.env_marg, H.env_marg);
    rc = rc ? rc : s->upload(&S.env_cond, H.env_cond);
    if (rc) {
        delete s;
        return rc;
    }
    // Path state: slabs of whole sample passes (see pt_kernels.cuh).
    s->npix = scene->camera.width * scene->camera.height;
    // Guided renders train between slabs: their slabs grow 1, 2, 4, ... sample
    // passes up to about 4M paths (16 passes at most), with guide_steps
    // network updates per sample pass.
    const bool guided = params->guided != 0;
    if (guided && S.n_media) {
        delete s;
        return fail(RT_ERR_INVALID, "the learned proposal does not guide scenes with participating media");
    }
    uint64_t guided_k = std::max<uint64_t>(1, std::min<uint64_t>(16, (4ull << 20) / s->npix));
    // Plain renders: slabs of up to 32M paths and 16 passes. A wave lasts as
    // long as its longest rays, so more passes per slab spread those tails
    // over more samples: on the forest at 3840x2160, 1 / 2 / 4 passes per
    // slab took 415 / 388 / 376 ms per pass.
    uint64_t cap = params->max_paths ? params->max_paths : guided ? guided_k * s->npix : (32ull << 20);
    uint64_t k = std::max<uint64_t>(1, cap / s->npix);
    if (!params->max_paths && !guided) k = std::min<uint64_t>(k, 16);
    if (k * s->npix > 0xFFFFFFFFull / 8) k = std::max<uint64_t>(1, (0xFFFFFFFFull / 8) / s->npix);
    s->slab_samples = (uint32_t)k;
    uint64_t P = k * s->npix;
    Paths& Pp = s->paths;
    Pp.P = (uint32_t)P;
    bool aov = params->aovs != 0;
    rc = rc ? rc : s->alloc(&Pp.ray_o, P);
    rc = rc ? rc : s->alloc(&Pp.ray_d, P);
    rc = rc ? rc : s->alloc(&Pp.hit, P);
    rc = rc ? rc : s->alloc(&Pp.beta, P);
    rc = rc ? rc : s->alloc(&Pp.L, P);
    rc = rc ? rc : s->alloc(&Pp.prev, P);
    rc = rc ? rc : s->alloc(&Pp.rng, P);
    rc = rc ? rc : s->alloc(&Pp.sh_o, P);
    rc = rc ? rc : s->alloc(&Pp.sh_d, P);
    rc = rc ? rc : s->alloc(&Pp.sh_c, P);
    rc = rc ? rc : s->alloc(&Pp.aux_a, aov ? P : 1);
    rc = rc ? rc : s->alloc(&Pp.aux_n, aov ? P : 1);
    rc = rc ? rc : s->alloc(&Pp.aux_d, aov ? P : 1);
    Pp.cone = nullptr;
    if (S.mat_pat) rc = rc ? rc : s->alloc(&Pp.cone, P);
    Pp.time = nullptr;
    if (S.motion) rc = rc ? rc : s->alloc(&Pp.time, P);
    // Media: nested-medium stacks and the equiangular shadow slot; walks:
    // their queue.
    Pp.med = nullptr;
    Pp.sh2_o = Pp.sh2_d = Pp.sh2_c = nullptr;
    Pp.q_sss = nullptr;
    if (S.n_media) {
        rc = rc ? rc : s->alloc(&Pp.med, P);
        rc = rc ? rc : s->alloc(&Pp.sh2_o, P);
        rc = rc ? rc : s->alloc(&Pp.sh2_d, P);
        rc = rc ? rc : s->alloc(&Pp.sh2_c, P);
    }
    if (S.any_sss) rc = rc ? rc : s->alloc(&Pp.q_sss, P);
    rc = rc ? rc : s->alloc(&Pp.q_ext[0], P);
    rc = rc ? rc : s->alloc(&Pp.q_ext[1], P);
    rc = rc ? rc : s->alloc(&Pp.q_cls, P * N_QUEUES);
    rc = rc ? rc : s->alloc(&Pp.q_sh, P);
    rc = rc ? rc : s->alloc(&Pp.cnt, CNT_WORDS);
    rc = rc ? rc : s->alloc(&s->stats, 4);
    rc = rc ? rc : s->alloc(&s->err, 1);
    rc = rc ? rc : s->alloc(&s->fetch, 1);
    rc = rc ? rc : s->alloc(&s->accum, 4ull * s->npix);
    rc = rc ? rc : s->alloc(&s->lum_stats, 4ull * s->npix);
    rc = rc ? rc : s->alloc(&s->aux, aov ? 12ull * s->npix : 1);
    // Guiding: inference records per slot, training vertices of every path
    // of the slab, and the slab's training batches (2^16 records per Adam
    // step) subsampled from them.
    const uint32_t steps_per_pass = guide_steps_per_pass(params->guide_steps);
    Pp.tr_tag = 0;
    Pp.tb_cap = guided ? (1u << 16) * (uint32_t)k * steps_per_pass : 0u;
    const size_t tr_floats = guided ? P * params->max_depth * TR_FLOATS : 1;
    float* keep = nullptr;
    rc = rc ? rc : s->alloc(&Pp.g_rec, guided ? P * 16 : 1);
    rc = rc ? rc : s->alloc(&Pp.g_idx, guided ? P : 1);
    rc = rc ? rc : s->alloc(&Pp.g_cnt, 1);
    rc = rc ? rc : s->alloc(&Pp.tr_rec, tr_floats);
    rc = rc ? rc : s->alloc(&Pp.tb_rec, guided ? (size_t)Pp.tb_cap * 16 : 1);
    rc = rc ? rc : s->alloc(&Pp.tb_cnt, 4);
    rc = rc ? rc : s->alloc(&Pp.tb_blk, guided ? (P * params->max_depth + COLLECT_BLOCK - 1) / COLLECT_BLOCK : 1);
    rc = rc ? rc : s->alloc(&keep, 1);
    if (!rc) {
        const float one = 1.0f;
        Pp.tr_keep = keep;
        if (cudaMemsetAsync(Pp.tr_rec, 0, tr_floats * 4, s->stream) != cudaSuccess ||
            cudaMemsetAsync(Pp.tb_cnt, 0, 16, s->stream) != cudaSuccess ||
            cudaMemcpyAsync(keep, &one, 4, cudaMemcpyHostToDevice, s->stream) != cudaSuccess ||
            cudaStreamSynchronize(s->stream) != cudaSuccess)
            rc = fail(RT_ERR_CUDA, "guide buffers: initialisation failed");
    }
    if (!rc && guided) {
        float lo[3], hi[3];
        for (int a = 0; a < 3; a++) {
            double wlo = s->host.world_lo[a], whi = s->host.world_hi[a];
            if (s->host.quad_lo[a] <= s->host.quad_hi[a]) {
                const bool meshes = scene->n_instances > 0;
                wlo = meshes ? std::min(wlo, s->host.quad_lo[a]) : s->host.quad_lo[a];
                whi = meshes ? std::max(whi, s->host.quad_hi[a]) : s->host.quad_hi[a];
            }
            double pad = 1e-3 * (whi - wlo) + 1e-6;
            lo[a] = (float)(wlo - pad);
            hi[a] = (float)(whi + pad);
        }
        const float lr = params->guide_lr > 0.0 ? (float)params->guide_lr : 1e-2f;
        if (rt_guide_create(lo, hi, 0x5eed, lr, &s->guide) != 0 || guide_reserve(s->guide, (uint32_t)P) != 0)
            rc = fail(RT_ERR_CUDA, rt_guide_last_error());
        else
            guide_set_wait_polls(s->guide, params->wait_polls);
    }
    if (rc) {
        delete s;
        return rc;
    }
    Pp.stats = s->stats;
    Pp.err = s->err;
    cudaMemsetAsync(s->err, 0, 4, s->stream);
    cudaMemsetAsync(s->accum, 0, 32ull * s->npix, s->stream);
    cudaMemsetAsync(s->lum_stats, 0, 32ull * s->npix, s->stream);
    if (aov) cudaMemsetAsync(s->aux, 0, 48ull * s->npix, s->stream);
    ce = cudaStreamSynchronize(s->stream);
    if (ce != cudaSuccess) {
        delete s;
        return fail(RT_ERR_CUDA, std::string("upload: ") + cudaGetErrorString(ce));
    }
    *out = s;
    return RT_OK;
}

int rt_session_destroy(rt_session* s) {
    delete s;
    return RT_OK;
}

void* rt_session_stream(rt_session* s) { return s ? (void*)s->stream : nullptr; }

rt_guide* rt_session_guide(rt_session* s) { return s ? s->guide : nullptr; }

int rt_set_adaptive(rt_session* s, double tol) {
    if (!s) return fail(RT_ERR_INVALID, "session is NULL");
    if (!(tol >= 0.0) || tol > 1e30) return fail(RT_ERR_INVALID, "adaptive tolerance must be >= 0");
    s->adaptive_tol = (float)tol;
    return RT_OK;
}

int rt_average_spp(rt_session* s, double* out) {
    if (!s || !out) return fail(RT_ERR_INVALID, "NULL argument");
    SESSION_DEVICE(s);
    std::vector<double> a(4ull * s->npix);
    int rc = rt_read_accum(s, a.data());
    if (rc) return rc;
    double sum = 0.0;
    for (size_t p = 0; p < s->npix; p++) sum += a[4 * p + 3];
    *out = sum / (double)s->npix;
    return RT_OK;
}

int rt_set_limits(rt_session* s, uint32_t max_trav_steps, uint32_t wait_polls) {
    if (!s) return fail(RT_ERR_INVALID, "session is NULL");
    s->params.max_trav_steps = max_trav_steps;
    s->params.wait_polls = wait_polls;
    s->S.max_steps = max_trav_steps ? max_trav_steps : RT_MAX_TRAV_STEPS;
    if (s->guide) guide_set_wait_polls(s->guide, wait_polls);
    return RT_OK;
}

int rt_reset(rt_session* s) {
    if (!s) return fail(RT_ERR_INVALID, "session is NULL");
    SESSION_DEVICE(s);
    CUDA_TRY(cudaMemsetAsync(s->accum, 0, 32ull * s->npix, s->stream));
    CUDA_TRY(cudaMemsetAsync(s->lum_stats, 0, 32ull * s->npix, s->stream));
    if (s->params.aovs) CUDA_TRY(cudaMemsetAsync(s->aux, 0, 48ull * s->npix, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->samples_done = 0;
    return RT_OK;
}

int rt_render_samples(rt_session* s, uint32_t sample_start, uint32_t count) {
    if (!s) return fail(RT_ERR_INVALID, "session is NULL");
    SESSION_DEVICE(s);
    if (count == 0) return RT_OK;
    cudaStream_t st = s->stream;
    Paths& P = s->paths;
    PtConsts C;
    C.npix = s->npix;
    C.width = s->S.width;
    // Multiple scattering needs a deeper budget: 64 bounces in scenes with
    // media (pt/mod.rs:483-484, gpu_scene.rs:671).
    C.max_depth = s->S.n_media ? 64u : s->params.max_depth;
    C.rr_start = s->params.rr_start;
    C.aovs = s->params.aovs;
    C.clamp = (float)s->params.firefly_clamp;
    C.guided = s->guide ? 1u : 0u;
    C.alpha = (float)std::min(std::max(s->params.guide_fraction, 0.0), 1.0);
    if (s->guide) C.G = guide_dev(s->guide);
    C.adaptive_tol = s->adaptive_tol;
    C.lum_stats = s->lum_stats;
    int guide_trainings = 0;
    // Cutouts: decided inside the extension traversal, except when AOVs are
    // kept, whose first-hit values come from the first surface a camera ray
    // meets even when it passes through it (pt/mod.rs:690-700); then the
    // shade kernel skips surfaces as the reference does, in extra waves.
    // Cutouts decided in the extension traversal, unless AOVs want the first
    // surface met or the cutouts are pattern-driven (decided in shading).
    C.pres_in_trav = (s->S.any_presence && !s->params.aovs && !s->S.presence_pat) ? 1u : 0u;
    // Waves: one per bounce, plus the surfaces a path may pass without a
    // bounce (cutouts skipped in shade waves, volume-hull crossings).
    const bool skip_waves = (s->S.any_presence && !C.pres_in_trav) || s->S.n_media;
    uint32_t waves = C.max_depth + (skip_waves ? RT_MAX_PRESENCE_SKIPS : 0u);
    const int trav_grid = s->trav_grid, shade_grid = s->sm_count * 8;
    const uint32_t batch = 1u << 16;  // training records per Adam step
    CUDA_TRY(cudaMemsetAsync(s->stats, 0, 32, st));
    float ms_ext = 0, ms_sh = 0, ms_shade = 0;
    uint64_t launches = 0;
    uint32_t last_records_slab = 0;
    uint64_t slabs = 0;
    // Per-wave timing events are recorded without host waits and read once
    // at the end, so the waves of a slab run back to back.
    auto events = [&](size_t need) -> int {
        while (s->evpool.size() < need) {
            cudaEvent_t e;
            CUDA_TRY(cudaEventCreate(&e));
            s->evpool.push_back(e);
        }
        return RT_OK;
    };
    int erc = events(2);
    if (erc) return erc;
    size_t ei = 2;
    CUDA_TRY(cudaEventRecord(s->evpool[0], st));
    for (uint32_t done = 0; done < count;) {
        uint32_t k = std::min(s->slab_samples, count - done);
        // Adaptive sampling decides per sample pass, so every decision sees
        // all earlier samples of the pixel (as the reference's per-sample
        // dispatches do): one pass per slab.
        if (s->adaptive_tol > 0.0f) k = 1;
        if (s->guide) {
            // Slabs grow while the network is young, so it is updated often early on.
            k = std::min(k, 1u << std::min<uint64_t>(s->guide_slabs, 31));
        }
        erc = events(ei + 4 * (size_t)waves);
        if (erc) return erc;
        uint32_t slab_paths = k * s->npix;
        P.P = slab_paths;
        C.sample0 = (uint64_t)sample_start + done;
        // Training stops once the budget of trained passes is spent; later
        // slabs only sample the fixed proposal (no training vertices, no
        // collection, no Adam steps).
        const bool train = s->guide && s->guide_trained_passes < guide_train_budget(s->params.guide_train_passes);
        if (train) k = (uint32_t)std::min<uint64_t>(k, guide_train_budget(s->params.guide_train_passes) - s->guide_trained_passes);
        C.train = train ? 1u : 0u;
        if (train) P.tr_tag++;  // new tag: the training records of this slab
        CUDA_TRY(cudaMemsetAsync(P.cnt, 0, CNT_WORDS * 4, st));
        k_raygen<<<(slab_paths + 255) / 256, 256, 0, st>>>(s->S, P, C);
        launches++;
        for (uint32_t w = 0; w < waves; w++) {
            uint32_t qin = w & 1u, qout = qin ^ 1u;
            CUDA_TRY(cudaEventRecord(s->evpool[ei], st));
            const bool quad = extra_geometry(s), mot = s->S.motion != 0;
            if (C.pres_in_trav && mot) k_extend<TRAV_BLOCK, true, true, true><<<trav_grid, TRAV_BLOCK, 0, st>>>(s->S, P, qin);
            else if (mot) k_extend<TRAV_BLOCK, false, true, true><<<trav_grid, TRAV_BLOCK, 0, st>>>(s->S, P, qin);
            else if (C.pres_in_trav && quad) k_extend<TRAV_BLOCK, true, true><<<trav_grid, TRAV_BLOCK, 0, st>>>(s->S, P, qin);
            else if (C.pres_in_trav) k_extend<TRAV_BLOCK, true><<<trav_grid, TRAV_BLOCK, 0, st>>>(s->S, P, qin);
            else if (quad) k_extend<TRAV_BLOCK, false, true><<<trav_grid, TRAV_BLOCK, 0, st>>>(s->S, P, qin);
            else k_extend<TRAV_BLOCK, false><<<trav_grid, TRAV_BLOCK, 0, st>>>(s->S, P, qin);
            CUDA_TRY(cudaEventRecord(s->evpool[ei + 1], st));
            if (s->guide) {
                // Network inputs for this wave's guided vertices, then inference.
                CUDA_TRY(cudaMemsetAsync(P.g_cnt, 0, 4, st));
                k_guide_gather<<<shade_grid, 128, 0, st>>>(s->S, P, s->params.guide_depth);
                float* raw = nullptr;
                int grc = guide_infer_counted(s->guide, P.g_rec, P.g_cnt, P.P, &raw, st);
                if (grc) return fail(grc, rt_guide_last_error());
                P.g_raw = raw;
                launches += 3;
            }
            const bool med = s->S.n_media > 0;
            if (P.cone && med) k_shade<true, true><<<shade_grid, SHADE_BLOCK, 0, st>>>(s->S, P, C, qout);
            else if (P.cone) k_shade<true><<<shade_grid, SHADE_BLOCK, 0, st>>>(s->S, P, C, qout);
            else if (med) k_shade<false, true><<<shade_grid, SHADE_BLOCK, 0, st>>>(s->S, P, C, qout);
            else k_shade<false><<<shade_grid, SHADE_BLOCK, 0, st>>>(s->S, P, C, qout);
            if (s->S.any_sss) {
                // Subsurface walks started by this wave's shading.
                const bool mt = s->S.motion != 0;
                if (med && mt) k_sss<TRAV_BLOCK, true, true><<<trav_grid, TRAV_BLOCK, 0, st>>>(s->S, P, C, qout);
                else if (med) k_sss<TRAV_BLOCK, true><<<trav_grid, TRAV_BLOCK, 0, st>>>(s->S, P, C, qout);
                else if (mt) k_sss<TRAV_BLOCK, false, true><<<trav_grid, TRAV_BLOCK, 0, st>>>(s->S, P, C, qout);
                else k_sss<TRAV_BLOCK, false><<<trav_grid, TRAV_BLOCK, 0, st>>>(s->S, P, C, qout);
                launches++;
            }
            CUDA_TRY(cudaEventRecord(s->evpool[ei + 2], st));
            const bool walk_extra = s->S.motion || s->S.presence_pat;
            if (med && walk_extra) k_shadow_walk<TRAV_BLOCK, true, true><<<trav_grid, TRAV_BLOCK, 0, st>>>(s->S, P, C);
            else if (med) k_shadow_walk<TRAV_BLOCK><<<trav_grid, TRAV_BLOCK, 0, st>>>(s->S, P, C);
            else if (s->S.presence_pat)
                k_shadow_walk<TRAV_BLOCK, false, true><<<trav_grid, TRAV_BLOCK, 0, st>>>(s->S, P, C);
            else if (mot) k_shadow<TRAV_BLOCK, true, true><<<trav_grid, TRAV_BLOCK, 0, st>>>(s->S, P, C);
            else if (quad) k_shadow<TRAV_BLOCK, true><<<trav_grid, TRAV_BLOCK, 0, st>>>(s->S, P, C);
            else k_shadow<TRAV_BLOCK><<<trav_grid, TRAV_BLOCK, 0, st>>>(s->S, P, C);
            CUDA_TRY(cudaEventRecord(s->evpool[ei + 3], st));
            k_wave_prep<<<1, 32, 0, st>>>(P.cnt);
            launches += 4;
            ei += 4;
        }
        k_accumulate<<<(s->npix + 255) / 256, 256, 0, st>>>(P, C, k, s->accum, s->aux);
        launches++;
        if (s->guide) s->guide_slabs++;
        if (train) {
            // Adam steps (guide_steps per sample pass) on this slab's closed
            // vertices: a subsample of about steps * 2^16 records (keep
            // probability from the previous slab's candidate count), split
            // into consecutive batches.
            const uint32_t steps = k * guide_steps_per_pass(s->params.guide_steps);
            const float scale = s->guide_prev_k ? (float)k / (float)s->guide_prev_k : 1.0f;
            k_guide_keep<<<1, 1, 0, st>>>(P.tb_cnt, scale, steps * batch, P.tr_keep);
            CUDA_TRY(cudaMemsetAsync(P.tb_cnt, 0, 8, st));
            Paths Pc = P;
            Pc.tb_cap = steps * batch;
            const uint64_t collect_threads = (uint64_t)P.P * C.max_depth;
            const uint32_t nb = (uint32_t)((collect_threads + COLLECT_BLOCK - 1) / COLLECT_BLOCK);
            k_guide_collect_count<<<nb, COLLECT_BLOCK, 0, st>>>(Pc, C);
            k_guide_collect_scan<<<1, 1024, 0, st>>>(Pc.tb_blk, nb, Pc.tb_cnt);
            k_guide_collect_write<<<nb, COLLECT_BLOCK, 0, st>>>(Pc, C);
            int grc = guide_train_slices(s->guide, P.tb_rec, P.tb_cnt, batch, steps, st);
            if (grc) return fail(grc, rt_guide_last_error());
            guide_trainings += (int)steps;
            launches += 4 + 8 * (uint64_t)steps;
            s->guide_prev_k = k;
            s->guide_trained_passes += k;
            last_records_slab = steps * batch;
        }
        done += k;
        slabs++;
    }
    CUDA_TRY(cudaEventRecord(s->evpool[1], st));
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(st));
    for (size_t e = 2; e < ei; e += 4) {
        float a, b, c;
        cudaEventElapsedTime(&a, s->evpool[e], s->evpool[e + 1]);
        cudaEventElapsedTime(&b, s->evpool[e + 1], s->evpool[e + 2]);
        cudaEventElapsedTime(&c, s->evpool[e + 2], s->evpool[e + 3]);
        ms_ext += a;
        ms_shade += b;
        ms_sh += c;
    }
    int rc = s->check_device_error();
    if (rc) return rc;
    unsigned long long stats[2];
    CUDA_TRY(cudaMemcpy(stats, s->stats, 16, cudaMemcpyDeviceToHost));
    float total = 0;
    cudaEventElapsedTime(&total, s->evpool[0], s->evpool[1]);
    s->last.extension_rays = stats[0];
    s->last.shadow_rays = stats[1];
    s->last.samples = (uint64_t)count * s->npix;
    s->last.kernel_launches = launches;
    s->last.extend_ms = ms_ext;
    s->last.shadow_ms = ms_sh;
    s->last.shade_ms = ms_shade;
    s->last.total_ms = total;
    s->last.guide_steps = (uint64_t)guide_trainings;
    s->last.slabs = slabs;
    s->last.waves = waves;
    s->last.guide_records = 0;
    s->last.guide_loss = 0.0;
    if (s->guide) {
        uint32_t gerr = 0, nrec = 0;
        float loss = 0.f;
        CUDA_TRY(cudaMemcpy(&gerr, guide_err_ptr(s->guide), 4, cudaMemcpyDeviceToHost));
        if (gerr) {
            cudaMemsetAsync((void*)guide_err_ptr(s->guide), 0, 4, st);
            cudaStreamSynchronize(st);
            return fail(RT_ERR_DEVICE, "guide network: tensor-core pipeline wait timed out");
        }
        CUDA_TRY(cudaMemcpy(&nrec, P.tb_cnt, 4, cudaMemcpyDeviceToHost));
        CUDA_TRY(cudaMemcpy(&loss, guide_loss_ptr(s->guide), 4, cudaMemcpyDeviceToHost));
        s->last.guide_records = std::min(nrec, last_records_slab);
        s->last.guide_loss = loss;
    }
    s->samples_done += count;
    return RT_OK;
}

int rt_read_accum(rt_session* s, double* rgbw) {
    if (!s || !rgbw) return fail(RT_ERR_INVALID, "NULL argument");
    SESSION_DEVICE(s);
    CUDA_TRY(cudaMemcpyAsync(rgbw, s->accum, 32ull * s->npix, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return RT_OK;
}

int rt_read_image(rt_session* s, float* rgb) {
    if (!s || !rgb) return fail(RT_ERR_INVALID, "NULL argument");
    SESSION_DEVICE(s);
    // Resolve on the device into the shadow-ray origin buffer (free between
    // renders; at least 16 B per pixel), then copy 12 B per pixel.
    float* img = reinterpret_cast<float*>(s->paths.sh_o);
    k_resolve<<<(s->npix + 255) / 256, 256, 0, s->stream>>>(s->accum, img, s->npix);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(rgb, img, 12ull * s->npix, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return RT_OK;
}

int rt_read_aux(rt_session* s, float* aux12) {
    if (!s || !aux12) return fail(RT_ERR_INVALID, "NULL argument");
    SESSION_DEVICE(s);
    if (!s->params.aovs) return fail(RT_ERR_INVALID, "session was created with aovs = 0");
    CUDA_TRY(cudaMemcpyAsync(aux12, s->aux, 48ull * s->npix, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return RT_OK;
}

int rt_checkpoint_save(rt_session* s, const char* path) {
    if (!s || !path) return fail(RT_ERR_INVALID, "NULL argument");
    SESSION_DEVICE(s);
    std::vector<double> a(4ull * s->npix);
    int rc = rt_read_accum(s, a.data());
    if (rc) return rc;
    std::string tmp = std::string(path) + ".tmp";
    FILE* f = fopen(tmp.c_str(), "wb");
    if (!f) return fail(RT_ERR_IO, "cannot open " + tmp);
    uint32_t hdr[4] = {0x31554352u /* "RCU1" */, s->S.width, s->S.height, s->samples_done};
    bool ok = fwrite(hdr, 4, 4, f) == 4 && fwrite(a.data(), 8, a.size(), f) == a.size();
    ok = (fclose(f) == 0) && ok;
    if (!ok || rename(tmp.c_str(), path) != 0) {
        remove(tmp.c_str());
        return fail(RT_ERR_IO, std::string("cannot write checkpoint ") + path);
    }
    return RT_OK;
}

int rt_read_film(rt_session* s, float* film) {
    if (!s || !film) return fail(RT_ERR_INVALID, "NULL argument");
    SESSION_DEVICE(s);
    if (!s->params.aovs) return fail(RT_ERR_INVALID, "the session was created without AOVs (params.aovs = 0)");
    float* d = nullptr;
    CUDA_TRY(pool_alloc((void**)&d, 4ull * RT_FILM_FLOATS * s->npix, s->stream));
    int rc = film_decode_device(s->accum, s->aux, s->npix, d, s->stream);
    cudaError_t e = rc ? cudaSuccess
                       : cudaMemcpyAsync(film, d, 4ull * RT_FILM_FLOATS * s->npix, cudaMemcpyDeviceToHost, s->stream);
    pool_free(d, s->stream);
    cudaStreamSynchronize(s->stream);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(RT_ERR_CUDA, std::string("film read-back: ") + cudaGetErrorString(e));
    return RT_OK;
}

int rt_denoise(rt_session* s, float* rgb) {
    if (!s || !rgb) return fail(RT_ERR_INVALID, "NULL argument");
    SESSION_DEVICE(s);
    if (!s->params.aovs) return fail(RT_ERR_INVALID, "the session was created without AOVs (params.aovs = 0)");
    float *d = nullptr, *o = nullptr;
    CUDA_TRY(pool_alloc((void**)&d, 4ull * RT_FILM_FLOATS * s->npix, s->stream));
    cudaError_t e = pool_alloc((void**)&o, 12ull * s->npix, s->stream);
    int rc = e != cudaSuccess ? fail(RT_ERR_OOM, "denoise buffers") : RT_OK;
    rc = rc ? rc : film_decode_device(s->accum, s->aux, s->npix, d, s->stream);
    rc = rc ? rc : denoise_device(d, s->S.width, s->S.height, o, s->stream);
    if (!rc && cudaMemcpyAsync(rgb, o, 12ull * s->npix, cudaMemcpyDeviceToHost, s->stream) != cudaSuccess)
        rc = fail(RT_ERR_CUDA, "denoise read-back failed");
    pool_free(d, s->stream);
    if (o) pool_free(o, s->stream);
    cudaStreamSynchronize(s->stream);
    return rc;
}

int rt_checkpoint_save_rckp(rt_session* s, const char* path) {
    if (!s || !path) return fail(RT_ERR_INVALID, "NULL argument");
    SESSION_DEVICE(s);
    std::vector<double> a(4ull * s->npix);
    int rc = rt_read_accum(s, a.data());
    if (rc) return rc;
    return rt_rckp_write(path, s->S.width, s->S.height, s->samples_done, a.data());
}

int rt_checkpoint_load(rt_session* s, const char* path, uint32_t* samples_done) {
    if (!s || !path) return fail(RT_ERR_INVALID, "NULL argument");
    SESSION_DEVICE(s);
    FILE* f = fopen(path, "rb");
    if (!f) return fail(RT_ERR_IO, std::string("cannot open ") + path);
    uint32_t hdr[4];
    std::vector<double> a(4ull * s->npix);
    bool ok = fread(hdr, 4, 4, f) == 4;
    // This library's f64 checkpoint ("RCU1") or the Metal backend's f32 one
    // ("RCKP", src/raytracer/metal/renderer.rs:219-254).
    const bool rckp = ok && hdr[0] == 0x504B4352u;
    if (ok && ((hdr[0] != 0x31554352u && !rckp) || hdr[1] != s->S.width || hdr[2] != s->S.height)) {
        fclose(f);
        return fail(RT_ERR_MISMATCH, "checkpoint does not match this session");
    }
    if (rckp) {
        std::vector<float> a32(a.size());
        ok = ok && fread(a32.data(), 4, a32.size(), f) == a32.size();
        for (size_t i = 0; i < a.size(); i++) a[i] = a32[i];
    } else {
        ok = ok && fread(a.data(), 8, a.size(), f) == a.size();
    }
    char extra;
    ok = ok && fread(&extra, 1, 1, f) == 0;
    fclose(f);
    if (!ok) return fail(RT_ERR_IO, std::string("truncated checkpoint ") + path);
    CUDA_TRY(cudaMemcpyAsync(s->accum, a.data(), 32ull * s->npix, cudaMemcpyHostToDevice, s->stream));
    // The file holds no luminance statistics: adaptive stopping restarts its
    // count from the samples rendered after the load.
    CUDA_TRY(cudaMemsetAsync(s->lum_stats, 0, 32ull * s->npix, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->samples_done = hdr[3];
    if (samples_done) *samples_done = hdr[3];
    return RT_OK;
}

int rt_intersect_batch_device(rt_session* s, const float* rays, uint64_t n, int any_hit, uint32_t* prim,
                              uint32_t* inst, float* t, void* stream) {
    if (!s || (!rays && n) || (!prim && n)) return fail(RT_ERR_INVALID, "NULL argument");
    SESSION_DEVICE(s);
    if (n >= 0xFFFFFFFFull - 64) return fail(RT_ERR_INVALID, "batch larger than 2^32 rays");
    if (((uintptr_t)rays & 15u) != 0) return fail(RT_ERR_INVALID, "rays must be 16-byte aligned");
    if (n == 0) return RT_OK;
    cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
    CUDA_TRY(cudaMemsetAsync(s->fetch, 0, 4, st));
    const float4* o = (const float4*)rays;
    const float4* d = o + n;
    int grid = s->trav_grid;
    launch_intersect(s, any_hit, grid, st, o, d, n, prim, inst, t, s->fetch, s->err);
    CUDA_TRY(cudaGetLastError());
    return RT_OK;
}

int rt_intersect_batch(rt_session* s, const float* rays, uint64_t n, int any_hit, uint32_t* prim, uint32_t* inst,
                       float* t) {
    if (!s || (!rays && n) || (!prim && n)) return fail(RT_ERR_INVALID, "NULL argument");
    SESSION_DEVICE(s);
    if (n == 0) return RT_OK;
    size_t need = n * (32 + 12);
    if (need > s->batch_cap) {
        if (s->batch_buf) cudaFree(s->batch_buf);
        s->batch_buf = nullptr;
        s->batch_cap = 0;
        CUDA_TRY(cudaMalloc(&s->batch_buf, need));
        s->batch_cap = need;
    }
    char* b = (char*)s->batch_buf;
    float* d_rays = (float*)b;
    uint32_t* d_prim = (uint32_t*)(b + 32 * n);
    uint32_t* d_inst = (uint32_t*)(b + 36 * n);
    float* d_t = (float*)(b + 40 * n);
    CUDA_TRY(cudaMemcpyAsync(d_rays, rays, 32 * n, cudaMemcpyHostToDevice, s->stream));
    int rc = rt_intersect_batch_device(s, d_rays, n, any_hit, d_prim, d_inst, d_t, nullptr);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpyAsync(prim, d_prim, 4 * n, cudaMemcpyDeviceToHost, s->stream));
    if (!any_hit && inst) CUDA_TRY(cudaMemcpyAsync(inst, d_inst, 4 * n, cudaMemcpyDeviceToHost, s->stream));
    if (!any_hit && t) CUDA_TRY(cudaMemcpyAsync(t, d_t, 4 * n, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return s->check_device_error();
}

}  // extern "C"

// ---- ray batch without allocation ------------------------------------------------------
// rt_intersect_batch stages the caller's host rays and results in a device
// buffer it grows with cudaMalloc, plus a work counter and an error word.
// rt_intersect_batch_noalloc keeps all of that in this file-scope array
// instead: RT_NOALLOC_MAX_RAYS rays of staging (32 B in, 12 B out each) and
// two counter words (padded to 64), 2,883,840 bytes in all, held by every GPU
// that loads the library until the process exits.
namespace {
constexpr uint64_t NOALLOC_IN = 8ull * RT_NOALLOC_MAX_RAYS;       // floats: two planes of float4
constexpr uint64_t NOALLOC_OUT = 3ull * RT_NOALLOC_MAX_RAYS;      // prim, inst, t (32-bit each)
constexpr uint64_t NOALLOC_WORDS = NOALLOC_IN + NOALLOC_OUT + 64; // + fetch counter, error word (padded)
}  // namespace
static __device__ __align__(256) uint32_t g_noalloc_scratch[NOALLOC_WORDS];

namespace {
// Device address of g_noalloc_scratch per device. Host code cannot use the
// array's name as a device address; cudaGetSymbolAddress gives it, once per
// device, with that device current.
// Threads that make their first call on a device at the same time may both
// look the address up; the atomic store makes that benign.
constexpr int NOALLOC_MAX_DEVICES = 64;
std::atomic<uint32_t*> g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};

int noalloc_scratch(uint32_t** out) {
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return fail(RT_ERR_INVALID, "device index beyond the no-alloc table");
    uint32_t* p = g_noalloc_ptr[dev].load(std::memory_order_acquire);
    if (!p) {
        void* v = nullptr;
        CUDA_TRY(cudaGetSymbolAddress(&v, g_noalloc_scratch));
        p = (uint32_t*)v;
        g_noalloc_ptr[dev].store(p, std::memory_order_release);
    }
    *out = p;
    return RT_OK;
}
}  // namespace

extern "C" int rt_intersect_batch_noalloc(rt_session* s, const float* rays, uint64_t n, int any_hit, uint32_t* prim,
                                          uint32_t* inst, float* t) {
    if (!s || (!rays && n) || (!prim && n)) return fail(RT_ERR_INVALID, "NULL argument");
    SESSION_DEVICE(s);
    if (n > RT_NOALLOC_MAX_RAYS)
        return fail(RT_ERR_INVALID, "rt_intersect_batch_noalloc: " + std::to_string(n) + " rays exceed its fixed " +
                                        std::to_string(RT_NOALLOC_MAX_RAYS) + "-ray staging area");
    if (n == 0) return RT_OK;
    uint32_t* base = nullptr;
    int rc = noalloc_scratch(&base);
    if (rc) return rc;
    float* d_rays = (float*)base;                          // two planes, 16-byte aligned
    uint32_t* d_prim = base + NOALLOC_IN;
    uint32_t* d_inst = d_prim + RT_NOALLOC_MAX_RAYS;
    float* d_t = (float*)(d_inst + RT_NOALLOC_MAX_RAYS);
    uint32_t* d_fetch = base + NOALLOC_IN + NOALLOC_OUT;   // must start at zero
    uint32_t* d_err = d_fetch + 32;                        // must start at zero
    cudaStream_t st = s->stream;
    // The planes are packed for n rays: origins [0, 4n), directions [4n, 8n).
    CUDA_TRY(cudaMemcpyAsync(d_rays, rays, 32 * n, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemsetAsync(d_fetch, 0, 4, st));
    CUDA_TRY(cudaMemsetAsync(d_err, 0, 4, st));
    const float4* o = (const float4*)d_rays;
    const float4* d = o + n;
    launch_intersect(s, any_hit, s->trav_grid, st, o, d, n, d_prim, d_inst, d_t, d_fetch, d_err);
    CUDA_TRY(cudaGetLastError());
    uint32_t e = 0;
    CUDA_TRY(cudaMemcpyAsync(prim, d_prim, 4 * n, cudaMemcpyDeviceToHost, st));
    if (!any_hit && inst) CUDA_TRY(cudaMemcpyAsync(inst, d_inst, 4 * n, cudaMemcpyDeviceToHost, st));
    if (!any_hit && t) CUDA_TRY(cudaMemcpyAsync(t, d_t, 4 * n, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaMemcpyAsync(&e, d_err, 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    if (e) return fail(RT_ERR_DEVICE, device_error_text(e));
    return RT_OK;
}

extern "C" {

int rt_bsdf_furnace(const rt_material_desc* material, const double* wo, double eta, uint64_t n, uint64_t seed,
                    double* out) {
    if (!material || !wo || !out) return fail(RT_ERR_INVALID, "NULL argument");
    DevMaterial m = fold_material_public(*material);
    const int threads = 256, blocks = 148 * 8;
    const uint64_t nt = (uint64_t)threads * blocks;
    uint64_t per = (n + nt - 1) / nt;
    double* d = nullptr;
    CUDA_TRY(cudaMalloc(&d, nt * 4 * sizeof(double)));
    float3 w = make_float3((float)wo[0], (float)wo[1], (float)wo[2]);
    k_furnace<<<blocks, threads>>>(m, w, (float)eta, per, seed, d);
    cudaError_t e = cudaDeviceSynchronize();
    std::vector<double> h(nt * 4);
    if (e == cudaSuccess) e = cudaMemcpy(h.data(), d, nt * 4 * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(RT_ERR_CUDA, std::string("furnace: ") + cudaGetErrorString(e));
    double acc[4] = {0, 0, 0, 0};
    for (uint64_t i = 0; i < nt; i++)
        for (int c = 0; c < 4; c++) acc[c] += h[4 * i + c];
    double total = (double)(per * nt);
    for (int c = 0; c < 4; c++) out[c] = acc[c] / total;
    return RT_OK;
}

// HairParams::new (hair.rs:40-55) in f32, as flatten_scene folds a hair material.
static DevHair hair_params(const double* p) {
    rt_material_desc md{};
    md.hair = 1;
    for (int c = 0; c < 3; c++) md.hair_sigma_a[c] = p[c];
    md.hair_beta_m = p[3];
    md.hair_beta_n = p[4];
    md.hair_eta = p[5];
    return hair_dev_public(md);
}

int rt_hair_eval(const double* params, uint64_t n, const float* q, float* f, float* pdf) {
    if ((!params || !q || !f || !pdf) && n) return fail(RT_ERR_INVALID, "NULL argument");
    if (!n) return RT_OK;
    if (n > (1ull << 26)) return fail(RT_ERR_INVALID, "rt_hair_eval: more than 2^26 queries");
    const DevHair hp = hair_params(params);
    float* d = nullptr;
    CUDA_TRY(cudaMalloc(&d, 4ull * 11 * n));
    cudaError_t e = cudaMemcpy(d, q, 4ull * 7 * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_hair_eval_batch<<<(uint32_t)((n + 127) / 128), 128>>>(hp, d, (uint32_t)n, d + 7 * n, d + 10 * n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(f, d + 7 * n, 12ull * n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(pdf, d + 10 * n, 4ull * n, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(RT_ERR_CUDA, std::string("rt_hair_eval: ") + cudaGetErrorString(e));
    return RT_OK;
}

int rt_hair_sample(const double* params, const double* wo, double h, uint64_t pixel, uint64_t sample, uint64_t n,
                   float* out) {
    if ((!params || !wo || !out) && n) return fail(RT_ERR_INVALID, "NULL argument");
    if (!n) return RT_OK;
    if (n > (1ull << 24)) return fail(RT_ERR_INVALID, "rt_hair_sample: more than 2^24 samples");
    const DevHair hp = hair_params(params);
    float* d = nullptr;
    CUDA_TRY(cudaMalloc(&d, 28ull * n));
    k_hair_sample_batch<<<1, 32>>>(hp, make_float3((float)wo[0], (float)wo[1], (float)wo[2]), (float)h, pixel, sample,
                                   (uint32_t)n, d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(out, d, 28ull * n, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(RT_ERR_CUDA, std::string("rt_hair_sample: ") + cudaGetErrorString(e));
    return RT_OK;
}

int rt_pcg_streams(const uint64_t* pixel, const uint64_t* sample, uint32_t m, uint32_t n, uint32_t* out) {
    if ((!pixel || !sample || !out) && m && n) return fail(RT_ERR_INVALID, "NULL argument");
    if (!m || !n) return RT_OK;
    if ((uint64_t)m * n > (1ull << 31)) return fail(RT_ERR_INVALID, "rt_pcg_streams: more than 2^31 draws");
    void* d = nullptr;
    const size_t bytes = 16ull * m + 4ull * m * n;
    CUDA_TRY(cudaMalloc(&d, bytes));
    uint64_t* dp = (uint64_t*)d;
    uint64_t* ds = dp + m;
    uint32_t* dout = (uint32_t*)(ds + m);
    cudaError_t e = cudaMemcpy(dp, pixel, 8ull * m, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(ds, sample, 8ull * m, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_pcg_streams<<<(m + 127) / 128, 128>>>(dp, ds, m, n, dout);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, dout, 4ull * m * n, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(RT_ERR_CUDA, std::string("rt_pcg_streams: ") + cudaGetErrorString(e));
    return RT_OK;
}

// Staging for the session diagnostics below: one pool block on the
// session's stream, freed before returning.
namespace {
struct Staging {
    rt_session* s;
    void* p = nullptr;
    explicit Staging(rt_session* s_) : s(s_) {}
    cudaError_t get(size_t bytes) { return pool_alloc(&p, bytes, s->stream); }
    ~Staging() {
        if (p) {
            pool_free(p, s->stream);
            cudaStreamSynchronize(s->stream);
        }
    }
};
}  // namespace

int rt_light_sample_batch(rt_session* s, const float* points, const float* u, uint32_t m, uint32_t* light,
                          float* pmf) {
    if (!s || ((!points || !u || !light || !pmf) && m)) return fail(RT_ERR_INVALID, "NULL argument");
    SESSION_DEVICE(s);
    if (!m) return RT_OK;
    Staging g(s);
    CUDA_TRY(g.get(24ull * m));
    float* dp = (float*)g.p;
    float* du = dp + 3ull * m;
    uint32_t* dl = (uint32_t*)(du + m);
    float* dm = (float*)(dl + m);
    CUDA_TRY(cudaMemcpyAsync(dp, points, 12ull * m, cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemcpyAsync(du, u, 4ull * m, cudaMemcpyHostToDevice, s->stream));
    k_light_sample_batch<<<(m + 127) / 128, 128, 0, s->stream>>>(s->S, dp, du, m, dl, dm);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(light, dl, 4ull * m, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaMemcpyAsync(pmf, dm, 4ull * m, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return RT_OK;
}

int rt_light_pmf_batch(rt_session* s, const float* points, const uint32_t* light, uint32_t m, float* pmf) {
    if (!s || ((!points || !light || !pmf) && m)) return fail(RT_ERR_INVALID, "NULL argument");
    SESSION_DEVICE(s);
    if (!m) return RT_OK;
    Staging g(s);
    CUDA_TRY(g.get(20ull * m));
    float* dp = (float*)g.p;
    uint32_t* dl = (uint32_t*)(dp + 3ull * m);
    float* dm = (float*)(dl + m);
    CUDA_TRY(cudaMemcpyAsync(dp, points, 12ull * m, cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemcpyAsync(dl, light, 4ull * m, cudaMemcpyHostToDevice, s->stream));
    k_light_pmf_batch<<<(m + 127) / 128, 128, 0, s->stream>>>(s->S, dp, dl, m, dm);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(pmf, dm, 4ull * m, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return RT_OK;
}

int rt_transmittance_batch(rt_session* s, const float* rays, uint64_t n, float* trans) {
    if (!s || ((!rays || !trans) && n)) return fail(RT_ERR_INVALID, "NULL argument");
    if (n >= 0xFFFFFFFFull - 64) return fail(RT_ERR_INVALID, "batch larger than 2^32 rays");
    SESSION_DEVICE(s);
    if (!n) return RT_OK;
    Staging g(s);
    CUDA_TRY(g.get(36ull * n + 16));
    float* d_rays = (float*)g.p;
    float* d_out = d_rays + 8 * n;
    CUDA_TRY(cudaMemcpyAsync(d_rays, rays, 32 * n, cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemsetAsync(s->fetch, 0, 4, s->stream));
    const float4* o = (const float4*)d_rays;
    if (extra_geometry(s))
        k_transmit_batch<TRAV_BLOCK, true><<<s->trav_grid, TRAV_BLOCK, 0, s->stream>>>(s->S, o, o + n, n, d_out,
                                                                                       s->fetch, s->err);
    else
        k_transmit_batch<TRAV_BLOCK><<<s->trav_grid, TRAV_BLOCK, 0, s->stream>>>(s->S, o, o + n, n, d_out, s->fetch,
                                                                                 s->err);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(trans, d_out, 4 * n, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return s->check_device_error();
}

int rt_get_stats(rt_session* s, rt_stats* out) {
    if (!s || !out) return fail(RT_ERR_INVALID, "NULL argument");
    *out = s->last;
    out->blas_nodes = s->host.blas_nodes;
    out->tlas_nodes = s->host.tlas_nodes;
    out->triangles = s->host.n_tris;
    out->device_bytes = s->device_bytes;
    return RT_OK;
}

}  // extern "C"

// bvh_build.cu — BVH construction on the device.
//
// The trees are the host builder's (flatten.cpp): binned SAH with the
// reference's rules (src/accel/bvh.rs:256-345: 16 bins on the widest
// centroid axis, leaves of <= 4 primitives or <= 16 when SAH prefers a
// leaf, median split otherwise), then the 8-wide collapse (open the child
// of largest surface area until 8 children) and the per-node 8-bit
// quantisation. Every decision is taken in f64 with explicitly rounded
// operations (no contraction into FMA) on the same f32 boxes, so each node
// gets the same box, split and children as on the host, and the wide-node
// words come out byte-identical; the only freedom is the order of the
// primitives inside a leaf (the host's swap partition vs the stable
// partition here).
//
// Binary build, level-synchronous for nodes of more than SMALL primitives
// (one pass each for bounds, bins, left counts and the stable scatter, over
// CHUNK-primitive blocks of every node of the level), then one warp per
// remaining subtree of <= SMALL primitives. Primitives ping-pong between two
// buffers; leaves end in buffer 0. The wide tree is laid out in the host
// collapser's depth-first preorder: structure top-down, subtree sizes
// bottom-up, indices top-down, then every node quantised independently.

#include "bvh_build.h"
#include "devmem.h"
#include "rt_cuda.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <functional>
#include <thread>

namespace rt {
namespace {

constexpr int BINS = 16;
constexpr uint32_t MAX_LEAF = 4;       // always a leaf at or below this count
constexpr uint32_t SAH_LEAF_MAX = 16;  // a leaf when SAH prefers one
constexpr uint32_t SMALL = 256;        // subtrees of at most this many primitives: one warp each
constexpr uint32_t CHUNK = 2048;       // primitives per block in the level passes
constexpr int LB = 256;                // level-pass block size
constexpr int SMALL_WARPS = 4;         // warps per block of the subtree kernel
constexpr int STACK = 16;              // subtree stack (log2(SMALL) + 1 entries suffice)
constexpr int JB = 128;                // per-job kernels' block size
constexpr uint32_t NONE = 0xFFFFFFFFu;

enum : uint32_t { MODE_MEDIAN = 0, MODE_SAH = 1, MODE_LEAF = 2 };
enum : uint32_t {
    BERR_CAP = 1u,        // a fixed-capacity array would have overflowed
    BERR_STACK = 2u,      // subtree stack overflow
    BERR_INDEX = 4u,      // vertex index out of range
    BERR_VERTEX = 8u,     // non-finite vertex
    BERR_DECODE = 16u,    // a quantised box failed its conservativeness check
    BERR_GRID = 32u,      // no quantisation grid found
    BERR_LARGE_LEAF = 64u,
};

// Primitive record: (lo.xyz, original index bits), (hi.xyz, 0).
struct BPrim {
    float4 a, b;
};
// Binary node: interior nodes have count 0 and children first, first + 1.
struct BNode {
    float lo[3], hi[3];
    uint32_t first, count;
};
static_assert(sizeof(BNode) == 32, "BNode layout");
struct Job {
    uint32_t node, start, count, parity;
};
struct JobInfo {
    uint32_t mode, axis, chunk_first, nchunks;
    double amin, scale, boundary;
    uint32_t m, pad;
};
// One wide node under construction: its binary root, children (binary node
// ids) and, for interior children, the slot of the child's record.
struct WideS {
    uint32_t root, nk, size, idx;
    uint32_t kids[8];
    uint32_t child[8];
};

// Order-preserving keys for atomic min / max of floats and doubles.
__device__ __forceinline__ uint32_t fkey(float f) {
    uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float fval(uint32_t k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}
__device__ __forceinline__ unsigned long long dkey(double d) {
    unsigned long long b = (unsigned long long)__double_as_longlong(d);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double dval(unsigned long long k) {
    return __longlong_as_double((long long)((k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k));
}
constexpr uint32_t KEY_F_POS_INF = 0xFF800000u;  // fkey(+inf)
constexpr uint32_t KEY_F_NEG_INF = 0x007FFFFFu;  // fkey(-inf)
constexpr unsigned long long KEY_D_POS_INF = 0xFFF0000000000000ull;
constexpr unsigned long long KEY_D_NEG_INF = 0x000FFFFFFFFFFFFFull;

__device__ __forceinline__ float lo_of(const BPrim& p, int a) { return a == 0 ? p.a.x : a == 1 ? p.a.y : p.a.z; }
__device__ __forceinline__ float hi_of(const BPrim& p, int a) { return a == 0 ? p.b.x : a == 1 ? p.b.y : p.b.z; }
// Centroid along an axis, as the host builder computes it: (lo + hi) * 0.5 in f64.
__device__ __forceinline__ double centroid(const BPrim& p, int a) {
    return __dmul_rn(__dadd_rn((double)lo_of(p, a), (double)hi_of(p, a)), 0.5);
}
__device__ __forceinline__ double centroid_at(const BPrim* P, uint32_t i, int a) {
    const float* f = reinterpret_cast<const float*>(P + i);
    return __dmul_rn(__dadd_rn((double)f[a], (double)f[4 + a]), 0.5);
}
// Surface area in f64 of an f32 box, with the host's operation order.
__device__ __forceinline__ double area_d(const float* lo, const float* hi) {
    double d0 = __dsub_rn((double)hi[0], (double)lo[0]);
    double d1 = __dsub_rn((double)hi[1], (double)lo[1]);
    double d2 = __dsub_rn((double)hi[2], (double)lo[2]);
    if (d0 < 0 || d1 < 0 || d2 < 0) return 0.0;
    return __dmul_rn(2.0, __dadd_rn(__dadd_rn(__dmul_rn(d0, d1), __dmul_rn(d1, d2)), __dmul_rn(d2, d0)));
}
__device__ __forceinline__ uint32_t bin_of(double c, double amin, double scale) {
    double f = __dmul_rn(__dsub_rn(c, amin), scale);
    uint32_t k = f > 0.0 ? (uint32_t)f : 0u;
    return k > (uint32_t)BINS - 1 ? (uint32_t)BINS - 1 : k;
}
__device__ __forceinline__ int widest_axis(const double* ext) {
    return (ext[0] >= ext[1] && ext[0] >= ext[2]) ? 0 : (ext[1] >= ext[2] ? 1 : 2);
}
__device__ __forceinline__ double split_boundary(double amin, double aext, int best_bin) {
    return __dadd_rn(amin, __ddiv_rn(__dmul_rn(aext, (double)(best_bin + 1)), (double)BINS));
}

// SAH over 16 bins (7 words each: lo keys, hi keys, count), the host
// builder's sweep: (cost, bin after which to split).
__device__ double sah_sweep(const uint32_t* bins, uint32_t count, int* best_bin_out) {
    float rlo[BINS][3], rhi[BINS][3];
    float alo[3] = {INFINITY, INFINITY, INFINITY}, ahi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = BINS - 1; i >= 1; i--) {
        for (int a = 0; a < 3; a++) {
            float l = fval(bins[i * 7 + a]), h = fval(bins[i * 7 + 3 + a]);
            alo[a] = l < alo[a] ? l : alo[a];
            ahi[a] = h > ahi[a] ? h : ahi[a];
            rlo[i][a] = alo[a];
            rhi[i][a] = ahi[a];
        }
    }
    double best = INFINITY;
    int best_bin = 0;
    float llo[3] = {INFINITY, INFINITY, INFINITY}, lhi[3] = {-INFINITY, -INFINITY, -INFINITY};
    uint32_t lc = 0;
    for (int i = 0; i < BINS - 1; i++) {
        for (int a = 0; a < 3; a++) {
            float l = fval(bins[i * 7 + a]), h = fval(bins[i * 7 + 3 + a]);
            llo[a] = l < llo[a] ? l : llo[a];
            lhi[a] = h > lhi[a] ? h : lhi[a];
        }
        lc += bins[i * 7 + 6];
        uint32_t rc = count - lc;
        if (lc == 0 || rc == 0) continue;
        double cost = __dadd_rn(__dmul_rn(area_d(llo, lhi), (double)lc), __dmul_rn(area_d(rlo[i + 1], rhi[i + 1]), (double)rc));
        if (cost < best) {
            best = cost;
            best_bin = i;
        }
    }
    *best_bin_out = best_bin;
    return best;
}

__device__ __forceinline__ void init_bins(uint32_t* bins, uint32_t k) {
    uint32_t r = k % 7;
    bins[k] = r < 3 ? KEY_F_POS_INF : r < 6 ? KEY_F_NEG_INF : 0u;
}

// ---- primitives ---------------------------------------------------------------

// Mesh of global triangle g: the last mesh whose first triangle is <= g.
__device__ __forceinline__ uint32_t mesh_of(const uint32_t* tri_base, uint32_t n_meshes, uint32_t g) {
    uint32_t lo = 0, hi = n_meshes;  // answer in [lo, hi)
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (tri_base[mid] <= g) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Triangle boxes from f32 vertices (exact), with -0 folded into +0 so that
// min / max by key and by comparison agree.
__global__ void k_tri_prims(const float* __restrict__ pos, const uint32_t* __restrict__ idx,
                            const uint32_t* __restrict__ tri_base, const uint32_t* __restrict__ vbase,
                            const uint32_t* __restrict__ nverts, uint32_t n_meshes, uint32_t n_tris,
                            BPrim* __restrict__ out, uint32_t* err) {
    uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_tris) return;
    uint32_t m = mesh_of(tri_base, n_meshes, g);
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    uint32_t bad = 0;
    for (int k = 0; k < 3; k++) {
        uint32_t vi = idx[3ull * g + k];
        if (vi >= nverts[m]) {
            bad |= BERR_INDEX;
            continue;
        }
        const float* p = pos + 3ull * (vbase[m] + (uint64_t)vi);
        float x = p[0], y = p[1], z = p[2];
        if (!isfinite(x) || !isfinite(y) || !isfinite(z)) {
            bad |= BERR_VERTEX;
            continue;
        }
        float v[3] = {x + 0.0f, y + 0.0f, z + 0.0f};
        for (int a = 0; a < 3; a++) {
            lo[a] = v[a] < lo[a] ? v[a] : lo[a];
            hi[a] = v[a] > hi[a] ? v[a] : hi[a];
        }
    }
    if (bad) atomicOr(err, bad);
    BPrim r;
    r.a = make_float4(lo[0], lo[1], lo[2], __uint_as_float(g));
    r.b = make_float4(hi[0], hi[1], hi[2], 0.0f);
    out[g] = r;
}

// Leaf-order triangles: (v0, original triangle id within its mesh) (v1, 0) (v2, 0).
__global__ void k_tri_gather(const BPrim* __restrict__ P0, const float* __restrict__ pos,
                             const uint32_t* __restrict__ idx, const uint32_t* __restrict__ tri_base,
                             const uint32_t* __restrict__ vbase, uint32_t n_meshes, uint32_t n_tris,
                             float4* __restrict__ tris) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_tris) return;
    uint32_t g = __float_as_uint(P0[k].a.w);
    if (g >= n_tris) return;  // unreachable: P0 is a permutation of 0..n_tris-1
    uint32_t m = mesh_of(tri_base, n_meshes, g);
    for (int c = 0; c < 3; c++) {
        const float* p = pos + 3ull * (vbase[m] + (uint64_t)idx[3ull * g + c]);
        float w = c == 0 ? __uint_as_float(g - tri_base[m]) : 0.0f;
        tris[3ull * k + c] = make_float4(p[0], p[1], p[2], w);
    }
}

// Leaf-order TLAS items.
__global__ void k_item_gather(const BPrim* __restrict__ P0, const uint2* __restrict__ in, uint32_t n,
                              uint2* __restrict__ out) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    uint32_t i = __float_as_uint(P0[k].a.w);
    if (i < n) out[k] = in[i];
}

// ---- binary build: level passes over nodes of more than SMALL primitives ------------
//
// Per level: k_bounds (node box and centroid box), k_bin (16 bins on the
// widest centroid axis), k_decide (SAH sweep: split, median or leaf),
// k_count (left side per chunk), k_scatter (stable partition into the other
// buffer), k_children (child nodes; children of <= SMALL primitives go to
// the subtree list, larger ones to the next level). Chunk c of the level
// belongs to job chunk_job[c]; accumulators are per job slot.

struct LevelArgs {
    const Job* jobs;
    JobInfo* info;
    const uint32_t* chunk_job;
    uint32_t* chunk_left;
    uint32_t* acc_box;             // 6 keys per job: lo xyz, hi xyz
    unsigned long long* acc_cb;    // 6 keys per job: centroid lo xyz, hi xyz
    uint32_t* acc_bin;             // BINS * 7 words per job
    BPrim* P[2];
};

__device__ __forceinline__ void chunk_range(const Job& J, const JobInfo& I, uint32_t c, uint32_t* b, uint32_t* e) {
    uint32_t base = J.start + (c - I.chunk_first) * CHUNK;
    uint32_t end = J.start + J.count;
    *b = base;
    *e = min(end, base + CHUNK);
}

template <class T, class Op>
__device__ __forceinline__ T warp_reduce(T v, Op op) {
    for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
    return v;
}
struct MinOp {
    template <class T>
    __device__ T operator()(T a, T b) const { return b < a ? b : a; }
};
struct MaxOp {
    template <class T>
    __device__ T operator()(T a, T b) const { return b > a ? b : a; }
};
struct AddOp {
    template <class T>
    __device__ T operator()(T a, T b) const { return a + b; }
};

__global__ void __launch_bounds__(LB) k_bounds(LevelArgs A) {
    const uint32_t c = blockIdx.x;
    const uint32_t j = A.chunk_job[c];
    const Job J = A.jobs[j];
    const JobInfo I = A.info[j];
    uint32_t b, e;
    chunk_range(J, I, c, &b, &e);
    const BPrim* src = A.P[J.parity];
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    double clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = b + threadIdx.x; i < e; i += LB) {
        BPrim p = src[i];
        for (int a = 0; a < 3; a++) {
            float l = lo_of(p, a), h = hi_of(p, a);
            lo[a] = l < lo[a] ? l : lo[a];
            hi[a] = h > hi[a] ? h : hi[a];
            double cc = centroid(p, a);
            clo[a] = cc < clo[a] ? cc : clo[a];
            chi[a] = cc > chi[a] ? cc : chi[a];
        }
    }
    __shared__ float sf[LB / 32][6];
    __shared__ double sd[LB / 32][6];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int a = 0; a < 3; a++) {
        lo[a] = warp_reduce(lo[a], MinOp());
        hi[a] = warp_reduce(hi[a], MaxOp());
        clo[a] = warp_reduce(clo[a], MinOp());
        chi[a] = warp_reduce(chi[a], MaxOp());
    }
    if (lane == 0)
        for (int a = 0; a < 3; a++) {
            sf[w][a] = lo[a];
            sf[w][3 + a] = hi[a];
            sd[w][a] = clo[a];
            sd[w][3 + a] = chi[a];
        }
    __syncthreads();
    if (threadIdx.x < 12) {
        const int q = threadIdx.x % 6;
        const bool is_d = threadIdx.x >= 6;
        if (!is_d) {
            float v = sf[0][q];
            for (int k = 1; k < LB / 32; k++) v = q < 3 ? (sf[k][q] < v ? sf[k][q] : v) : (sf[k][q] > v ? sf[k][q] : v);
            if (q < 3) atomicMin(&A.acc_box[6ull * j + q], fkey(v));
            else atomicMax(&A.acc_box[6ull * j + q], fkey(v));
        } else {
            double v = sd[0][q];
            for (int k = 1; k < LB / 32; k++) v = q < 3 ? (sd[k][q] < v ? sd[k][q] : v) : (sd[k][q] > v ? sd[k][q] : v);
            if (q < 3) atomicMin(&A.acc_cb[6ull * j + q], dkey(v));
            else atomicMax(&A.acc_cb[6ull * j + q], dkey(v));
        }
    }
}

// Centroid box of job j -> extent, widest axis, bin origin and scale.
struct AxisSetup {
    double ext[3], amin, scale;
    int axis;
};
__device__ __forceinline__ AxisSetup axis_setup(const unsigned long long* cbk) {
    AxisSetup s;
    double lo[3], hi[3];
    for (int a = 0; a < 3; a++) {
        lo[a] = dval(cbk[a]);
        hi[a] = dval(cbk[3 + a]);
        s.ext[a] = __dsub_rn(hi[a], lo[a]);
    }
    s.axis = widest_axis(s.ext);
    s.amin = lo[s.axis];
    s.scale = s.ext[s.axis] > 1e-12 ? __ddiv_rn((double)BINS, s.ext[s.axis]) : 0.0;
    return s;
}

__global__ void __launch_bounds__(LB) k_bin(LevelArgs A) {
    const uint32_t c = blockIdx.x;
    const uint32_t j = A.chunk_job[c];
    const Job J = A.jobs[j];
    const JobInfo I = A.info[j];
    const AxisSetup s = axis_setup(&A.acc_cb[6ull * j]);
    if (!(s.ext[s.axis] > 1e-12)) return;  // all centroids coincide: median split, no bins
    uint32_t b, e;
    chunk_range(J, I, c, &b, &e);
    __shared__ uint32_t bins[BINS * 7];
    for (uint32_t k = threadIdx.x; k < BINS * 7; k += LB) init_bins(bins, k);
    __syncthreads();
    const BPrim* src = A.P[J.parity];
    for (uint32_t i = b + threadIdx.x; i < e; i += LB) {
        BPrim p = src[i];
        uint32_t k = bin_of(centroid(p, s.axis), s.amin, s.scale);
        atomicAdd(&bins[k * 7 + 6], 1u);
        for (int a = 0; a < 3; a++) {
            atomicMin(&bins[k * 7 + a], fkey(lo_of(p, a)));
            atomicMax(&bins[k * 7 + 3 + a], fkey(hi_of(p, a)));
        }
    }
    __syncthreads();
    if (threadIdx.x < BINS * 7) {
        const uint32_t k = threadIdx.x, bin = k / 7, r = k % 7;
        if (bins[bin * 7 + 6] != 0) {
            uint32_t* g = &A.acc_bin[(size_t)BINS * 7 * j + k];
            if (r < 3) atomicMin(g, bins[k]);
            else if (r < 6) atomicMax(g, bins[k]);
            else atomicAdd(g, bins[k]);
        }
    }
}

// Split decision per job (the host builder's split_node rules).
__global__ void k_decide(LevelArgs A, uint32_t n_jobs) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_jobs) return;
    const Job J = A.jobs[j];
    JobInfo I = A.info[j];
    I.m = 0;
    I.mode = MODE_MEDIAN;
    if (J.count <= MAX_LEAF) {
        I.mode = MODE_LEAF;
    } else {
        const AxisSetup s = axis_setup(&A.acc_cb[6ull * j]);
        I.axis = (uint32_t)s.axis;
        if (s.ext[s.axis] > 1e-12) {
            int best_bin = 0;
            double best = sah_sweep(&A.acc_bin[(size_t)BINS * 7 * j], J.count, &best_bin);
            float lo[3], hi[3];
            for (int a = 0; a < 3; a++) {
                lo[a] = fval(A.acc_box[6ull * j + a]);
                hi[a] = fval(A.acc_box[6ull * j + 3 + a]);
            }
            double leaf_cost = __dmul_rn(area_d(lo, hi), (double)J.count);
            if (isfinite(best) && best < leaf_cost) {
                I.mode = MODE_SAH;
                I.amin = s.amin;
                I.boundary = split_boundary(s.amin, s.ext[s.axis], best_bin);
            } else if (J.count <= SAH_LEAF_MAX) {
                I.mode = MODE_LEAF;
            }
        }
    }
    A.info[j] = I;
}

__device__ __forceinline__ uint32_t block_sum(uint32_t v, uint32_t* sh) {
    v = warp_reduce(v, AddOp());
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    uint32_t t = 0;
    for (int k = 0; k < LB / 32; k++) t += sh[k];
    return t;
}

__global__ void __launch_bounds__(LB) k_count(LevelArgs A) {
    const uint32_t c = blockIdx.x;
    const uint32_t j = A.chunk_job[c];
    const JobInfo I = A.info[j];
    if (I.mode != MODE_SAH) return;
    const Job J = A.jobs[j];
    uint32_t b, e;
    chunk_range(J, I, c, &b, &e);
    const BPrim* src = A.P[J.parity];
    uint32_t n = 0;
    for (uint32_t i = b + threadIdx.x; i < e; i += LB) n += centroid_at(src, i, (int)I.axis) < I.boundary;
    __shared__ uint32_t sh[LB / 32];
    n = block_sum(n, sh);
    if (threadIdx.x == 0) {
        A.chunk_left[c] = n;
        atomicAdd(&A.info[j].m, n);
    }
}

// Stable partition of one chunk into the other buffer: left side at
// start + (left count of earlier chunks) + rank, right side after all m
// left primitives. Each thread owns 8 consecutive primitives.
__global__ void __launch_bounds__(LB) k_scatter(LevelArgs A) {
    const uint32_t c = blockIdx.x;
    const uint32_t j = A.chunk_job[c];
    const JobInfo I = A.info[j];
    if (I.mode != MODE_SAH) return;
    const Job J = A.jobs[j];
    uint32_t b, e;
    chunk_range(J, I, c, &b, &e);
    __shared__ uint32_t sh[LB / 32];
    uint32_t before = 0;
    for (uint32_t q = I.chunk_first + threadIdx.x; q < c; q += LB) before += A.chunk_left[q];
    before = block_sum(before, sh);
    const BPrim* src = A.P[J.parity];
    BPrim* dst = A.P[J.parity ^ 1u];
    const uint32_t i0 = b + threadIdx.x * (CHUNK / LB);
    uint32_t nv = i0 < e ? min(CHUNK / LB, e - i0) : 0u;
    uint32_t flags = 0;
    for (uint32_t q = 0; q < nv; q++) flags |= (uint32_t)(centroid_at(src, i0 + q, (int)I.axis) < I.boundary) << q;
    // exclusive scan of the per-thread left counts across the block
    const uint32_t cnt = __popc(flags);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
    }
    __shared__ uint32_t wsum[LB / 32];
    __syncthreads();
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    uint32_t wbase = 0;
    for (int k = 0; k < w; k++) wbase += wsum[k];
    const uint32_t left_before = before + wbase + incl - cnt;
    const uint32_t right_before = (i0 - J.start) - left_before;  // used only when nv > 0 (i0 < e)
    uint32_t lp = J.start + left_before, rp = J.start + I.m + right_before;
    for (uint32_t q = 0; q < nv; q++) {
        BPrim p = src[i0 + q];
        if ((flags >> q) & 1u) dst[lp++] = p;
        else dst[rp++] = p;
    }
}

struct ChildArgs {
    const Job* jobs;
    const JobInfo* info;
    const uint32_t* acc_box;
    BNode* nodes;
    uint32_t* node_counter;
    uint32_t node_cap;
    Job* next;
    JobInfo* next_info;
    uint32_t* next_count;
    uint32_t next_cap;
    uint32_t* chunk_job;     // next level's chunk table
    uint32_t* chunk_count;
    uint32_t chunk_cap;
    uint32_t* next_acc_box;
    unsigned long long* next_acc_cb;
    uint32_t* next_acc_bin;
    Job* small;
    uint32_t* small_count;
    uint32_t small_cap;
    uint32_t* err;
};

__device__ void clear_acc(const ChildArgs& C, uint32_t k) {
    for (int a = 0; a < 3; a++) {
        C.next_acc_box[6ull * k + a] = KEY_F_POS_INF;
        C.next_acc_box[6ull * k + 3 + a] = KEY_F_NEG_INF;
        C.next_acc_cb[6ull * k + a] = KEY_D_POS_INF;
        C.next_acc_cb[6ull * k + 3 + a] = KEY_D_NEG_INF;
    }
    for (uint32_t q = 0; q < BINS * 7; q++) init_bins(&C.next_acc_bin[(size_t)BINS * 7 * k], q);
}

__device__ void push_child(const ChildArgs& C, const Job& cj) {
    if (cj.count <= SMALL) {
        uint32_t k = atomicAdd(C.small_count, 1u);
        if (k < C.small_cap) C.small[k] = cj;
        else atomicOr(C.err, BERR_CAP);
        return;
    }
    uint32_t k = atomicAdd(C.next_count, 1u);
    if (k >= C.next_cap) {
        atomicOr(C.err, BERR_CAP);
        return;
    }
    uint32_t nch = (cj.count + CHUNK - 1) / CHUNK;
    uint32_t f = atomicAdd(C.chunk_count, nch);
    if (f + nch > C.chunk_cap) {
        atomicOr(C.err, BERR_CAP);
        return;
    }
    for (uint32_t q = 0; q < nch; q++) C.chunk_job[f + q] = k;
    C.next[k] = cj;
    JobInfo ni{};
    ni.chunk_first = f;
    ni.nchunks = nch;
    C.next_info[k] = ni;
    clear_acc(C, k);
}

__global__ void k_children(ChildArgs C, uint32_t n_jobs) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_jobs) return;
    const Job J = C.jobs[j];
    const JobInfo I = C.info[j];
    BNode nd;
    for (int a = 0; a < 3; a++) {
        nd.lo[a] = fval(C.acc_box[6ull * j + a]);
        nd.hi[a] = fval(C.acc_box[6ull * j + 3 + a]);
    }
    if (I.mode == MODE_LEAF) {
        // Level jobs hold more than SMALL >= SAH_LEAF_MAX primitives.
        atomicOr(C.err, BERR_LARGE_LEAF);
        return;
    }
    uint32_t split = J.start + J.count / 2, par = J.parity;
    if (I.mode == MODE_SAH) {
        par ^= 1u;
        if (I.m > 0 && I.m < J.count) split = J.start + I.m;
    }
    uint32_t l = atomicAdd(C.node_counter, 2u);
    if (l + 2 > C.node_cap) {
        atomicOr(C.err, BERR_CAP);
        return;
    }
    nd.first = l;
    nd.count = 0;
    C.nodes[J.node] = nd;
    push_child(C, Job{l, J.start, split - J.start, par});
    push_child(C, Job{l + 1, split, J.start + J.count - split, par});
}

__global__ void k_clear_acc(ChildArgs C, uint32_t n) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) clear_acc(C, k);
}

// ---- binary build: one warp per subtree of <= SMALL primitives -----------------------
//
// The same decisions as the level passes, with the node's primitives spread
// over the lanes: bounds by warp reduction, bins in shared memory, the
// stable partition by ballots. The smaller child is built next and the
// larger one stacked, so the stack never holds more than log2(SMALL) + 1
// entries.
__global__ void __launch_bounds__(32 * SMALL_WARPS)
    k_subtrees(const Job* __restrict__ small, const uint32_t* n_small_p, BPrim* P0, BPrim* P1, BNode* nodes,
               uint32_t* node_counter, uint32_t node_cap, uint32_t* err) {
    __shared__ uint32_t bins_sh[SMALL_WARPS][BINS * 7];
    const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const uint32_t w = blockIdx.x * SMALL_WARPS + wib;
    if (w >= *n_small_p) return;  // the whole warp leaves together
    uint32_t* bins = bins_sh[wib];
    const uint32_t lt_mask = (1u << lane) - 1u;
    Job stack[STACK];
    int sp = 0;
    stack[sp++] = small[w];
    while (sp > 0) {
        const Job J = stack[--sp];
        const BPrim* src = J.parity ? P1 : P0;
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        double clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (uint32_t i = lane; i < J.count; i += 32) {
            BPrim p = src[J.start + i];
            for (int a = 0; a < 3; a++) {
                float l = lo_of(p, a), h = hi_of(p, a);
                lo[a] = l < lo[a] ? l : lo[a];
                hi[a] = h > hi[a] ? h : hi[a];
                double cc = centroid(p, a);
                clo[a] = cc < clo[a] ? cc : clo[a];
                chi[a] = cc > chi[a] ? cc : chi[a];
            }
        }
        for (int a = 0; a < 3; a++) {
            lo[a] = warp_reduce(lo[a], MinOp());
            hi[a] = warp_reduce(hi[a], MaxOp());
            clo[a] = warp_reduce(clo[a], MinOp());
            chi[a] = warp_reduce(chi[a], MaxOp());
        }
        BNode nd;
        for (int a = 0; a < 3; a++) {
            nd.lo[a] = lo[a];
            nd.hi[a] = hi[a];
        }
        bool leaf = J.count <= MAX_LEAF;
        uint32_t split = J.start + J.count / 2, par = J.parity;
        if (!leaf) {
            double ext[3];
            for (int a = 0; a < 3; a++) ext[a] = __dsub_rn(chi[a], clo[a]);
            const int axis = widest_axis(ext);
            if (ext[axis] > 1e-12) {
                const double amin = clo[axis], scale = __ddiv_rn((double)BINS, ext[axis]);
                for (uint32_t k = lane; k < BINS * 7; k += 32) init_bins(bins, k);
                __syncwarp();
                for (uint32_t i = lane; i < J.count; i += 32) {
                    BPrim p = src[J.start + i];
                    uint32_t k = bin_of(centroid(p, axis), amin, scale);
                    atomicAdd(&bins[k * 7 + 6], 1u);
                    for (int a = 0; a < 3; a++) {
                        atomicMin(&bins[k * 7 + a], fkey(lo_of(p, a)));
                        atomicMax(&bins[k * 7 + 3 + a], fkey(hi_of(p, a)));
                    }
                }
                __syncwarp();
                int best_bin = 0;
                const double best = sah_sweep(bins, J.count, &best_bin);
                __syncwarp();  // every lane has read the bins before the next node clears them
                const double leaf_cost = __dmul_rn(area_d(nd.lo, nd.hi), (double)J.count);
                if (isfinite(best) && best < leaf_cost) {
                    const double boundary = split_boundary(amin, ext[axis], best_bin);
                    BPrim* dst = J.parity ? P0 : P1;
                    uint32_t m = 0;
                    for (uint32_t base = 0; base < J.count; base += 32) {
                        const uint32_t i = base + lane;
                        const bool f = i < J.count && centroid_at(src, J.start + i, axis) < boundary;
                        m += __popc(__ballot_sync(0xFFFFFFFFu, f));
                    }
                    uint32_t lw = 0, rw = 0;
                    for (uint32_t base = 0; base < J.count; base += 32) {
                        const uint32_t i = base + lane;
                        const bool v = i < J.count;
                        BPrim p;
                        bool f = false;
                        if (v) {
                            p = src[J.start + i];
                            f = centroid(p, axis) < boundary;
                        }
                        const uint32_t bl = __ballot_sync(0xFFFFFFFFu, v && f);
                        const uint32_t br = __ballot_sync(0xFFFFFFFFu, v && !f);
                        if (v) {
                            const uint32_t pos = f ? J.start + lw + __popc(bl & lt_mask)
                                                   : J.start + m + rw + __popc(br & lt_mask);
                            dst[pos] = p;
                        }
                        lw += __popc(bl);
                        rw += __popc(br);
                    }
                    __syncwarp();  // the children read what other lanes wrote
                    par ^= 1u;
                    if (m > 0 && m < J.count) split = J.start + m;
                } else if (J.count <= SAH_LEAF_MAX) {
                    leaf = true;
                }
            }
        }
        if (leaf) {
            nd.first = J.start;
            nd.count = J.count;
            if (lane == 0) nodes[J.node] = nd;
            if (J.parity && lane < J.count) P0[J.start + lane] = P1[J.start + lane];
            continue;
        }
        uint32_t l = 0;
        if (lane == 0) l = atomicAdd(node_counter, 2u);
        l = __shfl_sync(0xFFFFFFFFu, l, 0);
        if (l + 2 > node_cap || sp + 2 > STACK) {
            if (lane == 0) atomicOr(err, l + 2 > node_cap ? BERR_CAP : BERR_STACK);
            break;
        }
        nd.first = l;
        nd.count = 0;
        if (lane == 0) nodes[J.node] = nd;
        const Job a{l, J.start, split - J.start, par}, b{l + 1, split, J.start + J.count - split, par};
        if (a.count >= b.count) {
            stack[sp++] = a;
            stack[sp++] = b;
        } else {
            stack[sp++] = b;
            stack[sp++] = a;
        }
    }
}

// ---- 8-wide collapse -------------------------------------------------------------------

// Children of the wide node rooted at binary node W[s].root: open the
// interior child of largest area until 8 (the host collapser's rule);
// interior children get the next level's records.
__global__ void k_wide_level(WideS* W, uint32_t a, uint32_t b, const BNode* __restrict__ nodes, uint32_t* counter,
                             uint32_t cap, uint32_t* err) {
    const uint32_t s = a + blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= b) return;
    const uint32_t root = W[s].root;
    uint32_t kids[8];
    double ar[8];
    uint32_t nk = 0;
    const BNode r = nodes[root];
    if (r.count > 0) {
        kids[nk++] = root;  // a lone leaf becomes a one-child wide node
    } else {
        for (uint32_t q = 0; q < 2; q++) {
            const BNode c = nodes[r.first + q];
            kids[nk] = r.first + q;
            ar[nk++] = area_d(c.lo, c.hi);
        }
        while (nk < 8) {
            int best = -1;
            double best_a = -1.0;
            for (uint32_t k = 0; k < nk; k++)
                if (nodes[kids[k]].count == 0 && ar[k] > best_a) {
                    best_a = ar[k];
                    best = (int)k;
                }
            if (best < 0) break;
            const uint32_t f = nodes[kids[best]].first;
            const BNode c0 = nodes[f], c1 = nodes[f + 1];
            kids[best] = f;
            ar[best] = area_d(c0.lo, c0.hi);
            kids[nk] = f + 1;
            ar[nk++] = area_d(c1.lo, c1.hi);
        }
    }
    WideS& o = W[s];
    o.nk = nk;
    for (uint32_t k = 0; k < 8; k++) {
        uint32_t ch = NONE;
        if (k < nk) {
            o.kids[k] = kids[k];
            if (nodes[kids[k]].count == 0) {
                ch = atomicAdd(counter, 1u);
                if (ch < cap) {
                    W[ch].root = kids[k];
                } else {
                    atomicOr(err, BERR_CAP);
                    ch = NONE;
                }
            }
        } else {
            o.kids[k] = NONE;
        }
        o.child[k] = ch;
    }
}

// Subtree sizes, deepest level first.
__global__ void k_wide_size(WideS* W, uint32_t a, uint32_t b) {
    const uint32_t s = a + blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= b) return;
    uint32_t size = 1;
    for (int k = 0; k < 8; k++)
        if (W[s].child[k] != NONE) size += W[W[s].child[k]].size;
    W[s].size = size;
}

// Depth-first preorder indices, root level first: a node's interior
// children follow it in child order, each followed by its own subtree.
__global__ void k_wide_index(WideS* W, uint32_t a, uint32_t b) {
    const uint32_t s = a + blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= b) return;
    uint32_t run = W[s].idx + 1;
    for (int k = 0; k < 8; k++) {
        const uint32_t ch = W[s].child[k];
        if (ch != NONE) {
            W[ch].idx = run;
            run += W[ch].size;
        }
    }
}

__global__ void k_wide_root_index(WideS* W, const uint32_t* root_idx, uint32_t n) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) W[s].idx = root_idx[s];
}

// The children of every BLAS root (boxes and final references) and the
// second-level frontier (each inner child replaced by its children) for the
// TLAS items, in the host builder's order; needs the preorder indices.
__global__ void k_root_children(const WideS* __restrict__ W, uint32_t R, const BNode* __restrict__ nodes,
                                RootChild* __restrict__ out1, uint32_t* __restrict__ nk1,
                                RootChild* __restrict__ out2, uint32_t* __restrict__ nk2) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R) return;
    const WideS w = W[r];
    auto child_of = [&](const BNode& c, uint32_t child) {
        RootChild rc;
        for (int a = 0; a < 3; a++) {
            rc.lo[a] = c.lo[a];
            rc.hi[a] = c.hi[a];
        }
        rc.ref = c.count > 0 ? make_leaf_ref(c.first, c.count) : (child != NONE ? W[child].idx : REF_EMPTY);
        return rc;
    };
    uint32_t n1 = 0, n2 = 0;
    for (uint32_t k = 0; k < w.nk && k < 8; k++) {
        const BNode c = nodes[w.kids[k]];
        const RootChild rc = child_of(c, w.child[k]);
        out1[8ull * r + n1++] = rc;
        if (c.count == 0 && w.child[k] != NONE) {
            const WideS cw = W[w.child[k]];
            for (uint32_t kk = 0; kk < cw.nk && kk < 8; kk++)
                out2[(size_t)RT_TOP_MAX * r + n2++] = child_of(nodes[cw.kids[kk]], cw.child[kk]);
        } else {
            out2[(size_t)RT_TOP_MAX * r + n2++] = rc;
        }
    }
    nk1[r] = n1;
    nk2[r] = n2;
}

// ---- TLAS items on the device (flatten.cpp tlas_items, the same numbers) ----------------
// A mesh's BLAS frontiers for the items: its root's children (off1, n1) and
// its second-level frontier (off2, n2) in one RootChild table.
struct MeshFrontier {
    uint32_t off1, n1, off2, n2;
    uint32_t blas_root, n_tris, pad_[2];
};
// world_box in f64 with every product and sum rounded on its own, as the
// host computes it (no contraction into fused multiply-adds), so both
// builders make the same boxes and the same trees.
__device__ __forceinline__ void world_box_d(const double* m, const RootChild& rc, double* lo, double* hi) {
#pragma unroll
    for (int r = 0; r < 3; r++) {
        double c = m[r * 4 + 3], e = 0.0;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const double ck = __dmul_rn(0.5, __dadd_rn((double)rc.lo[k], (double)rc.hi[k]));
            const double hk = __dmul_rn(0.5, __dsub_rn((double)rc.hi[k], (double)rc.lo[k]));
            c = __dadd_rn(c, __dmul_rn(m[r * 4 + k], ck));
            e = __dadd_rn(e, __dmul_rn(fabs(m[r * 4 + k]), hk));
        }
        lo[r] = __dsub_rn(c, e);
        hi[r] = __dadd_rn(c, e);
    }
}
__device__ __forceinline__ double area_d(const double* lo, const double* hi) {
    const double d0 = __dsub_rn(hi[0], lo[0]), d1 = __dsub_rn(hi[1], lo[1]), d2 = __dsub_rn(hi[2], lo[2]);
    if (d0 < 0 || d1 < 0 || d2 < 0) return 0.0;
    return __dmul_rn(2.0, __dadd_rn(__dadd_rn(__dmul_rn(d0, d1), __dmul_rn(d1, d2)), __dmul_rn(d2, d0)));
}
__device__ __forceinline__ void grow_d(double* lo, double* hi, const double* blo, const double* bhi) {
#pragma unroll
    for (int a = 0; a < 3; a++) {
        lo[a] = blo[a] < lo[a] ? blo[a] : lo[a];
        hi[a] = bhi[a] > hi[a] ? bhi[a] : hi[a];
    }
}
// An instance's frontier (the root's children, or the second level) under
// its transform: the union of the children's world boxes and how many items
// it becomes (flatten.cpp child_boxes); boxes of the children into cb when
// given.
__device__ uint32_t child_boxes_d(const rt_instance_desc& id, const MeshFrontier& f, const RootChild* fr, bool second,
                                  bool split_all, double* ulo, double* uhi, double* cb) {
    for (int a = 0; a < 3; a++) {
        ulo[a] = HUGE_VAL;
        uhi[a] = -HUGE_VAL;
    }
    if (!f.n_tris) return 0;
    const uint32_t n = second ? f.n2 : f.n1, off = second ? f.off2 : f.off1;
    double sum = 0.0;
    for (uint32_t k = 0; k < n; k++) {
        double lo[3], hi[3];
        world_box_d(id.object_to_world, fr[off + k], lo, hi);
        if (cb)
            for (int a = 0; a < 3; a++) {
                cb[6 * k + a] = lo[a];
                cb[6 * k + 3 + a] = hi[a];
            }
        grow_d(ulo, uhi, lo, hi);
        sum = __dadd_rn(sum, area_d(lo, hi));
    }
    if (n <= 1) return 1u;
    return split_all || sum < __dmul_rn(RT_BRAID_RATIO, area_d(ulo, uhi)) ? n : 1u;
}
// Pass 1: per instance the union of its root children's world boxes and
// the number of items it becomes in a scene that is not dense.
__global__ void k_items_density(const rt_instance_desc* __restrict__ inst, uint32_t n, const MeshFrontier* __restrict__ mf,
                                const RootChild* __restrict__ fr, double* __restrict__ ubox, uint32_t* __restrict__ cnt) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const rt_instance_desc id = inst[i];
    double lo[3], hi[3];
    cnt[i] = child_boxes_d(id, mf[id.mesh_id], fr, false, false, lo, hi, nullptr);
    for (int a = 0; a < 3; a++) {
        ubox[6ull * i + a] = lo[a];
        ubox[6ull * i + 3 + a] = hi[a];
    }
}
// f32_box (flatten.cpp): rounded outward, -0 folded into +0.
__device__ __forceinline__ float f32_down(double x) { return __double2float_rd(x) + 0.0f; }
__device__ __forceinline__ float f32_up(double x) { return __double2float_ru(x) + 0.0f; }
// Pass 2: each instance's items at its offset: builder records (f32 box,
// item index) and (instance, BLAS reference); the union of the item boxes
// per instance for the world box.
__global__ void k_items_write(const rt_instance_desc* __restrict__ inst, uint32_t n, const MeshFrontier* __restrict__ mf,
                              const RootChild* __restrict__ fr, bool dense, const uint64_t* __restrict__ off,
                              BPrim* __restrict__ prims, uint2* __restrict__ items, double* __restrict__ ubox) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const rt_instance_desc id = inst[i];
    const MeshFrontier f = mf[id.mesh_id];
    double cb[6 * RT_TOP_MAX], lo[3], hi[3];
    const uint32_t k_items = child_boxes_d(id, f, fr, dense, dense, lo, hi, cb);
    for (uint32_t k = 0; k < k_items; k++) {
        const uint64_t j = off[i] + k;
        const double* b = cb + 6 * k;
        const double blo[3] = {k_items == 1 ? lo[0] : b[0], k_items == 1 ? lo[1] : b[1], k_items == 1 ? lo[2] : b[2]};
        const double bhi[3] = {k_items == 1 ? hi[0] : b[3], k_items == 1 ? hi[1] : b[4], k_items == 1 ? hi[2] : b[5]};
        BPrim p;
        p.a = make_float4(f32_down(blo[0]), f32_down(blo[1]), f32_down(blo[2]), __uint_as_float((uint32_t)j));
        p.b = make_float4(f32_up(bhi[0]), f32_up(bhi[1]), f32_up(bhi[2]), 0.0f);
        prims[j] = p;
        const uint32_t ref = k_items == 1 ? f.blas_root : fr[(dense ? f.off2 : f.off1) + k].ref;
        items[j] = make_uint2(i, ref);
    }
    for (int a = 0; a < 3; a++) {
        ubox[6ull * i + a] = k_items ? lo[a] : HUGE_VAL;
        ubox[6ull * i + 3 + a] = k_items ? hi[a] : -HUGE_VAL;
    }
}

// Quantisation grid of one axis (the host's choose_grid): origin p, a
// multiple of s = 2^e, with every p + q*s (q in 0..255) an exact f32 and
// p + 255*s >= hi. floor(log2) and ceil(log2) are taken exactly from the
// binary exponent.
__device__ bool choose_grid_d(double lo, double hi, float* p_out, int* e_out) {
    if (!(hi >= lo)) hi = lo;
    const double maxabs = fmax(fabs(lo), fabs(hi));
    int e_ulp = -149;
    if (maxabs > 0) e_ulp = ilogb(maxabs) - 23 + 4;
    const double extent = __dsub_rn(hi, lo);
    int e = -126;
    if (extent > 0) {
        int q;
        const double mant = frexp(__ddiv_rn(extent, 255.0), &q);
        e = mant == 0.5 ? q - 1 : q;
    }
    e = max(max(e, e_ulp), -126);
    for (int it = 0; it < 400; it++, e++) {
        const double s = ldexp(1.0, e);
        const double p = __dmul_rn(floor(__ddiv_rn(lo, s)), s);
        if (__ddiv_rn(__dsub_rn(hi, p), s) <= 255.0 && (double)(float)p == p) {
            *p_out = (float)p;
            *e_out = e;
            return true;
        }
    }
    return false;
}

__device__ __forceinline__ uint32_t pack4(const uint8_t* b) {
    return (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) | ((uint32_t)b[3] << 24);
}

// One wide node's 6 words (the host collapser's write()).
__global__ void k_wide_write(const WideS* __restrict__ W, uint32_t n, const BNode* __restrict__ nodes,
                             uint32_t prim_base, uint4* __restrict__ out, uint64_t out_nodes, uint32_t* err) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const WideS wn = W[s];
    if (wn.idx >= out_nodes) {
        atomicOr(err, BERR_CAP);
        return;
    }
    float nlo[3] = {INFINITY, INFINITY, INFINITY}, nhi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t k = 0; k < wn.nk; k++) {
        const BNode c = nodes[wn.kids[k]];
        for (int a = 0; a < 3; a++) {
            nlo[a] = c.lo[a] < nlo[a] ? c.lo[a] : nlo[a];
            nhi[a] = c.hi[a] > nhi[a] ? c.hi[a] : nhi[a];
        }
    }
    float p[3];
    int e[3];
    double sc[3];
    for (int a = 0; a < 3; a++) {
        if (!choose_grid_d((double)nlo[a], (double)nhi[a], &p[a], &e[a])) {
            atomicOr(err, BERR_GRID);
            return;
        }
        sc[a] = ldexp(1.0, e[a]);
    }
    uint8_t qlo[3][8], qhi[3][8];
    for (int k = 0; k < 8; k++)
        for (int a = 0; a < 3; a++) {
            qlo[a][k] = 255;
            qhi[a][k] = 0;
        }
    uint32_t refs[8];
    bool bad = false;
    for (uint32_t k = 0; k < 8; k++) {
        refs[k] = REF_EMPTY;
        if (k >= wn.nk) continue;
        const BNode c = nodes[wn.kids[k]];
        if (c.count == 0 && wn.child[k] == NONE) {  // unreachable: the structure pass reports overflow first
            bad = true;
            continue;
        }
        refs[k] = c.count > 0 ? make_leaf_ref(prim_base + c.first, c.count) : W[wn.child[k]].idx;
        for (int a = 0; a < 3; a++) {
            const double s = sc[a], pa = (double)p[a], clo = (double)c.lo[a], chi = (double)c.hi[a];
            double ql = floor(__ddiv_rn(__dsub_rn(clo, pa), s));
            double qh = ceil(__ddiv_rn(__dsub_rn(chi, pa), s));
            ql = fmin(fmax(ql, 0.0), 255.0);
            qh = fmin(fmax(qh, 0.0), 255.0);
            while (ql > 0 && __dadd_rn(pa, __dmul_rn(ql, s)) > clo) ql -= 1;
            while (qh < 255 && __dadd_rn(pa, __dmul_rn(qh, s)) < chi) qh += 1;
            qlo[a][k] = (uint8_t)ql;
            qhi[a][k] = (uint8_t)qh;
            const float sf = (float)s, p2 = __fsub_rn(p[a], __fmul_rn(8388608.0f, sf));
            const float dlo = __fmaf_rn(__fadd_rn(8388608.0f, (float)ql), sf, p2);
            const float dhi = __fmaf_rn(__fadd_rn(8388608.0f, (float)qh), sf, p2);
            if ((double)dlo != __dadd_rn(pa, __dmul_rn(ql, s)) || (double)dhi != __dadd_rn(pa, __dmul_rn(qh, s)) ||
                (double)dlo > clo || (double)dhi < chi)
                bad = true;
        }
    }
    if (bad) atomicOr(err, BERR_DECODE);
    uint4* o = out + (size_t)wn.idx * WIDE_NODE_WORDS;
    o[0] = make_uint4(__float_as_uint(p[0]), __float_as_uint(p[1]), __float_as_uint(p[2]),
                      (uint32_t)(e[0] + 127) | ((uint32_t)(e[1] + 127) << 8) | ((uint32_t)(e[2] + 127) << 16) |
                          (wn.nk << 24));
    o[1] = make_uint4(pack4(qlo[0]), pack4(qlo[0] + 4), pack4(qlo[1]), pack4(qlo[1] + 4));
    o[2] = make_uint4(pack4(qlo[2]), pack4(qlo[2] + 4), pack4(qhi[0]), pack4(qhi[0] + 4));
    o[3] = make_uint4(pack4(qhi[1]), pack4(qhi[1] + 4), pack4(qhi[2]), pack4(qhi[2] + 4));
    o[4] = make_uint4(refs[0], refs[1], refs[2], refs[3]);
    o[5] = make_uint4(refs[4], refs[5], refs[6], refs[7]);
}

// ---- host side ---------------------------------------------------------------------------

struct Fail {
    int code;
};

// Device allocations of one build; returned to the pool when the build
// returns (after the work queued on the build's stream).
struct Scratch {
    cudaStream_t st;
    std::vector<void*> ptrs;
    explicit Scratch(cudaStream_t s) : st(s) {}
    ~Scratch() {
        for (void* p : ptrs) pool_free(p, st);
    }
};

#define BV_TRY(expr)                                                                                 \
    do {                                                                                             \
        cudaError_t e_ = (expr);                                                                     \
        if (e_ != cudaSuccess) {                                                                     \
            *err = std::string(#expr) + ": " + cudaGetErrorString(e_);                              \
            return e_ == cudaErrorMemoryAllocation ? RT_ERR_OOM : RT_ERR_CUDA;                       \
        }                                                                                            \
    } while (0)

template <class T>
int dev_alloc(std::vector<void*>& owner, T** p, size_t count, cudaStream_t st, std::string* err) {
    void* v = nullptr;
    BV_TRY(pool_alloc(&v, std::max<size_t>(count, 1) * sizeof(T), st));
    owner.push_back(v);
    *p = (T*)v;
    return RT_OK;
}

inline uint32_t blocks_for(uint64_t n, int bs) { return (uint32_t)((n + bs - 1) / bs); }

std::string berr_text(uint32_t e) {
    std::string s = "device BVH build:";
    if (e & BERR_CAP) s += " capacity exceeded";
    if (e & BERR_STACK) s += " subtree stack overflow";
    if (e & BERR_DECODE) s += " quantised boxes not conservative";
    if (e & BERR_GRID) s += " no quantisation grid";
    if (e & BERR_LARGE_LEAF) s += " leaf above 16 primitives";
    return s;
}

// Binary trees over P0[0..n): root r (node r) covers roots[r] = (start, count).
// On return P0 holds the primitives in leaf order.
int build_binary_device(Scratch& D, BPrim* P0, BPrim* P1, uint32_t n,
                        const std::vector<std::pair<uint32_t, uint32_t>>& roots, uint32_t* d_err, BNode** nodes_out,
                        uint32_t* n_nodes_out, cudaStream_t st, std::string* err) {
    const uint32_t R = (uint32_t)roots.size();
    const uint64_t node_cap = 2ull * n + R + 2;
    const uint32_t J_cap = n / (SMALL + 1) + 2;
    const uint32_t C_cap = n / CHUNK + J_cap + 2;
    const uint32_t S_cap = n + R + 2;
    BNode* nodes;
    Job *jobs[2], *small;
    JobInfo* info[2];
    uint32_t *chunk_job, *chunk_left, *acc_box[2], *acc_bin[2], *counters;
    unsigned long long* acc_cb[2];
    int rc = 0;
    rc = rc ? rc : dev_alloc(D.ptrs, &nodes, node_cap, st, err);
    for (int b = 0; b < 2; b++) {
        rc = rc ? rc : dev_alloc(D.ptrs, &jobs[b], J_cap, st, err);
        rc = rc ? rc : dev_alloc(D.ptrs, &info[b], J_cap, st, err);
        rc = rc ? rc : dev_alloc(D.ptrs, &acc_box[b], 6ull * J_cap, st, err);
        rc = rc ? rc : dev_alloc(D.ptrs, &acc_cb[b], 6ull * J_cap, st, err);
        rc = rc ? rc : dev_alloc(D.ptrs, &acc_bin[b], (size_t)BINS * 7 * J_cap, st, err);
    }
    rc = rc ? rc : dev_alloc(D.ptrs, &chunk_job, C_cap, st, err);
    rc = rc ? rc : dev_alloc(D.ptrs, &chunk_left, C_cap, st, err);
    rc = rc ? rc : dev_alloc(D.ptrs, &small, S_cap, st, err);
    rc = rc ? rc : dev_alloc(D.ptrs, &counters, 4, st, err);  // nodes, next jobs, next chunks, small jobs
    if (rc) return rc;

    // Level 0: roots above SMALL are level jobs, the rest subtree jobs.
    std::vector<Job> lj, sj;
    std::vector<JobInfo> li;
    std::vector<uint32_t> cj;
    for (uint32_t r = 0; r < R; r++) {
        Job J{r, roots[r].first, roots[r].second, 0};
        if (J.count <= SMALL) {
            sj.push_back(J);
            continue;
        }
        JobInfo I{};
        I.chunk_first = (uint32_t)cj.size();
        I.nchunks = (J.count + CHUNK - 1) / CHUNK;
        for (uint32_t q = 0; q < I.nchunks; q++) cj.push_back((uint32_t)lj.size());
        lj.push_back(J);
        li.push_back(I);
    }
    uint32_t host_ctr[4] = {R, 0, 0, (uint32_t)sj.size()};
    if (!lj.empty()) {
        BV_TRY(cudaMemcpyAsync(jobs[0], lj.data(), lj.size() * sizeof(Job), cudaMemcpyHostToDevice, st));
        BV_TRY(cudaMemcpyAsync(info[0], li.data(), li.size() * sizeof(JobInfo), cudaMemcpyHostToDevice, st));
        BV_TRY(cudaMemcpyAsync(chunk_job, cj.data(), cj.size() * 4, cudaMemcpyHostToDevice, st));
    }
    if (!sj.empty()) BV_TRY(cudaMemcpyAsync(small, sj.data(), sj.size() * sizeof(Job), cudaMemcpyHostToDevice, st));
    BV_TRY(cudaMemcpyAsync(counters, host_ctr, sizeof(host_ctr), cudaMemcpyHostToDevice, st));

    ChildArgs C{};
    C.nodes = nodes;
    C.node_counter = &counters[0];
    C.node_cap = (uint32_t)std::min<uint64_t>(node_cap, 0xFFFFFFF0ull);
    C.next_count = &counters[1];
    C.next_cap = J_cap;
    C.chunk_job = chunk_job;
    C.chunk_count = &counters[2];
    C.chunk_cap = C_cap;
    C.small = small;
    C.small_count = &counters[3];
    C.small_cap = S_cap;
    C.err = d_err;
    uint32_t J = (uint32_t)lj.size(), nch = (uint32_t)cj.size();
    int cur = 0;
    if (J) {
        C.next_acc_box = acc_box[0];
        C.next_acc_cb = acc_cb[0];
        C.next_acc_bin = acc_bin[0];
        k_clear_acc<<<blocks_for(J, JB), JB, 0, st>>>(C, J);
    }
    for (uint64_t level = 0; J > 0; level++) {
        if (level > n) {
            *err = "device BVH build: level loop did not finish";
            return RT_ERR_DEVICE;
        }
        LevelArgs A{jobs[cur], info[cur], chunk_job, chunk_left, acc_box[cur], acc_cb[cur], acc_bin[cur], {P0, P1}};
        k_bounds<<<nch, LB, 0, st>>>(A);
        k_bin<<<nch, LB, 0, st>>>(A);
        k_decide<<<blocks_for(J, JB), JB, 0, st>>>(A, J);
        k_count<<<nch, LB, 0, st>>>(A);
        k_scatter<<<nch, LB, 0, st>>>(A);
        BV_TRY(cudaMemsetAsync(&counters[1], 0, 8, st));
        C.jobs = jobs[cur];
        C.info = info[cur];
        C.acc_box = acc_box[cur];
        C.next = jobs[cur ^ 1];
        C.next_info = info[cur ^ 1];
        C.next_acc_box = acc_box[cur ^ 1];
        C.next_acc_cb = acc_cb[cur ^ 1];
        C.next_acc_bin = acc_bin[cur ^ 1];
        k_children<<<blocks_for(J, JB), JB, 0, st>>>(C, J);
        uint32_t e = 0;
        BV_TRY(cudaMemcpyAsync(host_ctr, counters, sizeof(host_ctr), cudaMemcpyDeviceToHost, st));
        BV_TRY(cudaMemcpyAsync(&e, d_err, 4, cudaMemcpyDeviceToHost, st));
        BV_TRY(cudaStreamSynchronize(st));
        if (e & (BERR_CAP | BERR_LARGE_LEAF)) {
            *err = berr_text(e);
            return RT_ERR_DEVICE;
        }
        J = host_ctr[1];
        nch = host_ctr[2];
        cur ^= 1;
    }
    if (host_ctr[3]) {
        k_subtrees<<<blocks_for(host_ctr[3], SMALL_WARPS), 32 * SMALL_WARPS, 0, st>>>(
            small, &counters[3], P0, P1, nodes, &counters[0], C.node_cap, d_err);
    }
    uint32_t e = 0;
    BV_TRY(cudaMemcpyAsync(host_ctr, counters, sizeof(host_ctr), cudaMemcpyDeviceToHost, st));
    BV_TRY(cudaMemcpyAsync(&e, d_err, 4, cudaMemcpyDeviceToHost, st));
    BV_TRY(cudaStreamSynchronize(st));
    if (e & (BERR_CAP | BERR_STACK)) {
        *err = berr_text(e);
        return RT_ERR_DEVICE;
    }
    *nodes_out = nodes;
    *n_nodes_out = host_ctr[0];
    return RT_OK;
}

// Wide-tree structure and subtree sizes over binary trees whose roots are
// nodes 0..R-1; root_sizes[r] = wide nodes of tree r.
struct WideTree {
    WideS* W = nullptr;
    uint32_t n = 0;
    std::vector<uint32_t> level_off;  // level l = [level_off[l], level_off[l+1])
    std::vector<uint32_t> root_sizes;
};

int wide_structure(Scratch& D, const BNode* nodes, uint32_t n_nodes, uint32_t R, uint32_t* d_err, WideTree* T,
                   cudaStream_t st, std::string* err) {
    const uint32_t cap = n_nodes + 1;
    uint32_t* counter;
    int rc = dev_alloc(D.ptrs, &T->W, cap, st, err);
    rc = rc ? rc : dev_alloc(D.ptrs, &counter, 1, st, err);
    if (rc) return rc;
    std::vector<WideS> roots(R);
    for (uint32_t r = 0; r < R; r++) {
        memset(&roots[r], 0, sizeof(WideS));
        roots[r].root = r;
    }
    BV_TRY(cudaMemcpyAsync(T->W, roots.data(), R * sizeof(WideS), cudaMemcpyHostToDevice, st));
    BV_TRY(cudaMemcpyAsync(counter, &R, 4, cudaMemcpyHostToDevice, st));
    T->level_off = {0, R};
    uint32_t a = 0, b = R;
    while (a < b) {
        k_wide_level<<<blocks_for(b - a, JB), JB, 0, st>>>(T->W, a, b, nodes, counter, cap, d_err);
        uint32_t c = 0;
        BV_TRY(cudaMemcpyAsync(&c, counter, 4, cudaMemcpyDeviceToHost, st));
        BV_TRY(cudaStreamSynchronize(st));
        if (c > cap || T->level_off.size() > 4096) {
            *err = "device BVH build: wide structure overflow";
            return RT_ERR_DEVICE;
        }
        a = b;
        b = c;
        T->level_off.push_back(b);
    }
    T->n = b;
    const size_t L = T->level_off.size() - 1;
    for (size_t l = L; l-- > 0;) {
        uint32_t lo = T->level_off[l], hi = T->level_off[l + 1];
        if (hi > lo) k_wide_size<<<blocks_for(hi - lo, JB), JB, 0, st>>>(T->W, lo, hi);
    }
    T->root_sizes.resize(R);
    if (R)
        BV_TRY(cudaMemcpy2DAsync(T->root_sizes.data(), 4, &T->W[0].size, sizeof(WideS), 4, R, cudaMemcpyDeviceToHost, st));
    BV_TRY(cudaStreamSynchronize(st));
    return RT_OK;
}

// Preorder indices from the roots' indices.
int wide_index(Scratch& D, WideTree& T, const std::vector<uint32_t>& root_idx, cudaStream_t st, std::string* err) {
    const uint32_t R = (uint32_t)root_idx.size();
    if (T.n == 0) return RT_OK;
    uint32_t* d_root;
    int rc = dev_alloc(D.ptrs, &d_root, R, st, err);
    if (rc) return rc;
    BV_TRY(cudaMemcpyAsync(d_root, root_idx.data(), R * 4, cudaMemcpyHostToDevice, st));
    k_wide_root_index<<<blocks_for(R, JB), JB, 0, st>>>(T.W, d_root, R);
    for (size_t l = 0; l + 1 < T.level_off.size(); l++) {
        uint32_t lo = T.level_off[l], hi = T.level_off[l + 1];
        if (hi > lo) k_wide_index<<<blocks_for(hi - lo, JB), JB, 0, st>>>(T.W, lo, hi);
    }
    BV_TRY(cudaGetLastError());
    return RT_OK;
}

// Every node's 6 words (after wide_index).
int wide_words(WideTree& T, const BNode* nodes, uint4* out, uint64_t out_nodes, uint32_t* d_err, cudaStream_t st,
               std::string* err) {
    if (T.n == 0) return RT_OK;
    k_wide_write<<<blocks_for(T.n, JB), JB, 0, st>>>(T.W, T.n, nodes, 0, out, out_nodes, d_err);
    BV_TRY(cudaGetLastError());
    return RT_OK;
}

}  // namespace

int device_build_scene(const rt_scene_desc* d, HostScene* H, DeviceBvh* out, cudaStream_t st, std::string* err) {
    Scratch D(st);
    const uint32_t M = d->n_meshes;
    std::vector<uint32_t> tri_base(M), vbase(M), nverts(M);
    uint64_t N = 0, V = 0;
    for (uint32_t m = 0; m < M; m++) {
        tri_base[m] = (uint32_t)N;
        vbase[m] = (uint32_t)V;
        nverts[m] = d->meshes[m].n_triangles ? d->meshes[m].n_vertices : 0;
        N += d->meshes[m].n_triangles;
        V += nverts[m];
    }
    if (V >= (1ull << 32)) {
        *err = "more than 2^32 vertices";
        return RT_ERR_INVALID;
    }
    uint32_t* d_err;
    int rc = dev_alloc(D.ptrs, &d_err, 1, st, err);
    if (rc) return rc;
    BV_TRY(cudaMemsetAsync(d_err, 0, 4, st));

    // ---- BLAS: every mesh's triangles in one primitive array ----------------------
    uint32_t blas_total = 0;
    std::vector<uint32_t> blas_root(M, 0xFFFFFFFFu);
    std::vector<std::vector<RootChild>> root_children(M), grand_children(M);
    BNode* bnodes = nullptr;
    WideTree bw;
    BPrim *P0 = nullptr, *P1 = nullptr;
    float *d_pos = nullptr;
    uint32_t *d_idx = nullptr, *d_tri_base = nullptr, *d_vbase = nullptr, *d_nverts = nullptr;
    std::vector<std::pair<uint32_t, uint32_t>> roots;
    std::vector<uint32_t> root_mesh;
    for (uint32_t m = 0; m < M; m++)
        if (d->meshes[m].n_triangles) {
            roots.push_back({tri_base[m], d->meshes[m].n_triangles});
            root_mesh.push_back(m);
        }
    if (N) {
        rc = rc ? rc : dev_alloc(D.ptrs, &d_pos, 3 * V, st, err);
        rc = rc ? rc : dev_alloc(D.ptrs, &d_idx, 3 * N, st, err);
        rc = rc ? rc : dev_alloc(D.ptrs, &d_tri_base, M, st, err);
        rc = rc ? rc : dev_alloc(D.ptrs, &d_vbase, M, st, err);
        rc = rc ? rc : dev_alloc(D.ptrs, &d_nverts, M, st, err);
        rc = rc ? rc : dev_alloc(D.ptrs, &P0, N, st, err);
        rc = rc ? rc : dev_alloc(D.ptrs, &P1, N, st, err);
        if (rc) return rc;
        for (uint32_t m = 0; m < M; m++) {
            const rt_mesh_desc& md = d->meshes[m];
            if (!md.n_triangles) continue;
            BV_TRY(cudaMemcpyAsync(d_pos + 3ull * vbase[m], md.positions, 12ull * md.n_vertices, cudaMemcpyHostToDevice, st));
            BV_TRY(cudaMemcpyAsync(d_idx + 3ull * tri_base[m], md.indices, 12ull * md.n_triangles, cudaMemcpyHostToDevice, st));
        }
        BV_TRY(cudaMemcpyAsync(d_tri_base, tri_base.data(), 4ull * M, cudaMemcpyHostToDevice, st));
        BV_TRY(cudaMemcpyAsync(d_vbase, vbase.data(), 4ull * M, cudaMemcpyHostToDevice, st));
        BV_TRY(cudaMemcpyAsync(d_nverts, nverts.data(), 4ull * M, cudaMemcpyHostToDevice, st));
        k_tri_prims<<<blocks_for(N, 256), 256, 0, st>>>(d_pos, d_idx, d_tri_base, d_vbase, d_nverts, M, (uint32_t)N,
                                                         P0, d_err);
        uint32_t e = 0;
        BV_TRY(cudaMemcpyAsync(&e, d_err, 4, cudaMemcpyDeviceToHost, st));
        BV_TRY(cudaStreamSynchronize(st));
        if (e & (BERR_INDEX | BERR_VERTEX)) {
            // Name the first bad mesh as the host builder does.
            for (uint32_t m = 0; m < M; m++) {
                const rt_mesh_desc& md = d->meshes[m];
                bool bad_index = false, bad_vertex = false;
                for (uint64_t k = 0; k < 3ull * md.n_triangles; k++) {
                    uint32_t vi = md.indices[k];
                    if (vi >= md.n_vertices) {
                        bad_index = true;
                        continue;
                    }
                    for (int a = 0; a < 3; a++)
                        if (!std::isfinite(md.positions[3ull * vi + a])) bad_vertex = true;
                }
                if (bad_index) *err = "mesh " + std::to_string(m) + " index out of range";
                else if (bad_vertex) *err = "mesh " + std::to_string(m) + " has a non-finite vertex";
                if (bad_index || bad_vertex) return RT_ERR_INVALID;
            }
            *err = "invalid mesh data";
            return RT_ERR_INVALID;
        }
        uint32_t n_bnodes = 0;
        rc = build_binary_device(D, P0, P1, (uint32_t)N, roots, d_err, &bnodes, &n_bnodes, st, err);
        if (rc) return rc;
        H->binary_blas_nodes = n_bnodes;
        rc = wide_structure(D, bnodes, n_bnodes, (uint32_t)roots.size(), d_err, &bw, st, err);
        if (rc) return rc;
        std::vector<uint32_t> ridx(roots.size());
        for (size_t r = 0; r < roots.size(); r++) {
            const uint32_t m = root_mesh[r];
            blas_root[m] = blas_total;
            ridx[r] = blas_total;
            blas_total += bw.root_sizes[r];
        }
        rc = wide_index(D, bw, ridx, st, err);
        if (rc) return rc;
        // The BLAS roots' children (and their children) become the TLAS items.
        const uint32_t R = (uint32_t)roots.size();
        RootChild *d_rc1, *d_rc2;
        uint32_t *d_nk1, *d_nk2;
        rc = rc ? rc : dev_alloc(D.ptrs, &d_rc1, 8ull * R, st, err);
        rc = rc ? rc : dev_alloc(D.ptrs, &d_rc2, (size_t)RT_TOP_MAX * R, st, err);
        rc = rc ? rc : dev_alloc(D.ptrs, &d_nk1, R, st, err);
        rc = rc ? rc : dev_alloc(D.ptrs, &d_nk2, R, st, err);
        if (rc) return rc;
        k_root_children<<<blocks_for(R, JB), JB, 0, st>>>(bw.W, R, bnodes, d_rc1, d_nk1, d_rc2, d_nk2);
        std::vector<RootChild> hrc1(8ull * R), hrc2((size_t)RT_TOP_MAX * R);
        std::vector<uint32_t> hnk1(R), hnk2(R);
        BV_TRY(cudaMemcpyAsync(hrc1.data(), d_rc1, hrc1.size() * sizeof(RootChild), cudaMemcpyDeviceToHost, st));
        BV_TRY(cudaMemcpyAsync(hrc2.data(), d_rc2, hrc2.size() * sizeof(RootChild), cudaMemcpyDeviceToHost, st));
        BV_TRY(cudaMemcpyAsync(hnk1.data(), d_nk1, 4ull * R, cudaMemcpyDeviceToHost, st));
        BV_TRY(cudaMemcpyAsync(hnk2.data(), d_nk2, 4ull * R, cudaMemcpyDeviceToHost, st));
        BV_TRY(cudaStreamSynchronize(st));
        for (uint32_t r = 0; r < R; r++) {
            root_children[root_mesh[r]].assign(hrc1.begin() + 8ull * r, hrc1.begin() + 8ull * r + std::min(hnk1[r], 8u));
            grand_children[root_mesh[r]].assign(hrc2.begin() + (size_t)RT_TOP_MAX * r,
                                                hrc2.begin() + (size_t)RT_TOP_MAX * r + std::min(hnk2[r], RT_TOP_MAX));
        }
    }
    for (uint32_t m = 0; m < M; m++) H->meshes[m].blas_root = blas_root[m];
    H->blas_nodes = blas_total;

    // ---- TLAS over instance subtrees ------------------------------------------------------
    const uint32_t NI = d->n_instances;
    BNode* tnodes = nullptr;
    WideTree tw;
    BPrim* Q0 = nullptr;
    uint32_t tlas_total = 0, NIT = 0;
    std::vector<float4> xf;
    std::vector<uint4> rec;
    uint2* d_items = nullptr;
    if (NI) {
        // TLAS items on the device: the host's tlas_items rules and numbers
        // (flatten.cpp), with the density decision and the offsets on the host.
        std::vector<MeshFrontier> mf(M);
        std::vector<RootChild> fr;
        for (uint32_t m = 0; m < M; m++) {
            MeshFrontier& f = mf[m];
            f.off1 = (uint32_t)fr.size();
            f.n1 = (uint32_t)root_children[m].size();
            fr.insert(fr.end(), root_children[m].begin(), root_children[m].end());
            f.off2 = (uint32_t)fr.size();
            f.n2 = (uint32_t)grand_children[m].size();
            fr.insert(fr.end(), grand_children[m].begin(), grand_children[m].end());
            f.blas_root = blas_root[m];
            f.n_tris = H->meshes[m].n_tris;
        }
        rt_instance_desc* d_inst;
        MeshFrontier* d_mf;
        RootChild* d_fr;
        double* d_ubox;
        uint32_t* d_cnt;
        uint64_t* d_off;
        rc = rc ? rc : dev_alloc(D.ptrs, &d_inst, NI, st, err);
        rc = rc ? rc : dev_alloc(D.ptrs, &d_mf, M, st, err);
        rc = rc ? rc : dev_alloc(D.ptrs, &d_fr, std::max<size_t>(fr.size(), 1), st, err);
        rc = rc ? rc : dev_alloc(D.ptrs, &d_ubox, 6ull * NI, st, err);
        rc = rc ? rc : dev_alloc(D.ptrs, &d_cnt, NI, st, err);
        rc = rc ? rc : dev_alloc(D.ptrs, &d_off, NI, st, err);
        if (rc) return rc;
        BV_TRY(cudaMemcpyAsync(d_inst, d->instances, sizeof(rt_instance_desc) * NI, cudaMemcpyHostToDevice, st));
        BV_TRY(cudaMemcpyAsync(d_mf, mf.data(), sizeof(MeshFrontier) * M, cudaMemcpyHostToDevice, st));
        if (!fr.empty()) BV_TRY(cudaMemcpyAsync(d_fr, fr.data(), sizeof(RootChild) * fr.size(), cudaMemcpyHostToDevice, st));
        k_items_density<<<blocks_for(NI, JB), JB, 0, st>>>(d_inst, NI, d_mf, d_fr, d_ubox, d_cnt);
        std::vector<double> ubox(6ull * NI);
        std::vector<uint32_t> cnt(NI);
        BV_TRY(cudaMemcpyAsync(ubox.data(), d_ubox, 48ull * NI, cudaMemcpyDeviceToHost, st));
        BV_TRY(cudaMemcpyAsync(cnt.data(), d_cnt, 4ull * NI, cudaMemcpyDeviceToHost, st));
        BV_TRY(cudaStreamSynchronize(st));
        // Density: the instances' union boxes against their union.
        double total_area = 0.0, alo[3] = {HUGE_VAL, HUGE_VAL, HUGE_VAL}, ahi[3] = {-HUGE_VAL, -HUGE_VAL, -HUGE_VAL};
        auto area = [](const double* lo, const double* hi) {
            const double d0 = hi[0] - lo[0], d1 = hi[1] - lo[1], d2 = hi[2] - lo[2];
            if (d0 < 0 || d1 < 0 || d2 < 0) return 0.0;
            return 2.0 * (d0 * d1 + d1 * d2 + d2 * d0);
        };
        for (uint32_t i = 0; i < NI; i++) {
            if (!cnt[i]) continue;
            const double* u = ubox.data() + 6ull * i;
            total_area += area(u, u + 3);
            for (int a = 0; a < 3; a++) {
                alo[a] = u[a] < alo[a] ? u[a] : alo[a];
                ahi[a] = u[3 + a] > ahi[a] ? u[3 + a] : ahi[a];
            }
        }
        const double wa = area(alo, ahi);
        const bool dense = wa > 0.0 && total_area > RT_BRAID_DENSE * wa;
        H->scalars.refill_at = dense ? RT_REFILL_DENSE : RT_REFILL_SPARSE;
        std::vector<uint64_t> off(NI);
        uint64_t total = 0;
        for (uint32_t i = 0; i < NI; i++) {
            off[i] = total;
            const MeshFrontier& f = mf[d->instances[i].mesh_id];
            total += dense ? (f.n_tris ? std::max<uint32_t>(f.n2, 1u) : 0u) : cnt[i];
        }
        if (total >= (1ull << 27)) {
            *err = "more than 2^27 instance subtrees";
            return RT_ERR_INVALID;
        }
        NIT = (uint32_t)total;
        instance_records(d, *H, &xf, &rec);
        BPrim* Q1 = nullptr;
        rc = rc ? rc : dev_alloc(D.ptrs, &Q0, std::max<uint32_t>(NIT, 1), st, err);
        rc = rc ? rc : dev_alloc(D.ptrs, &Q1, std::max<uint32_t>(NIT, 1), st, err);
        rc = rc ? rc : dev_alloc(D.ptrs, &d_items, std::max<uint32_t>(NIT, 1), st, err);
        if (rc) return rc;
        BV_TRY(cudaMemcpyAsync(d_off, off.data(), 8ull * NI, cudaMemcpyHostToDevice, st));
        k_items_write<<<blocks_for(NI, JB), JB, 0, st>>>(d_inst, NI, d_mf, d_fr, dense, d_off, Q0, d_items, d_ubox);
        BV_TRY(cudaMemcpyAsync(ubox.data(), d_ubox, 48ull * NI, cudaMemcpyDeviceToHost, st));
        BV_TRY(cudaStreamSynchronize(st));
        double wlo[3] = {HUGE_VAL, HUGE_VAL, HUGE_VAL}, whi[3] = {-HUGE_VAL, -HUGE_VAL, -HUGE_VAL};
        for (uint32_t i = 0; i < NI; i++)
            for (int a = 0; a < 3; a++) {
                const double* u = ubox.data() + 6ull * i;
                wlo[a] = u[a] < wlo[a] ? u[a] : wlo[a];
                whi[a] = u[3 + a] > whi[a] ? u[3 + a] : whi[a];
            }
        for (int a = 0; a < 3; a++) {
            H->world_lo[a] = wlo[a] <= whi[a] ? wlo[a] : 0.0;
            H->world_hi[a] = wlo[a] <= whi[a] ? whi[a] : 0.0;
        }
        if (NIT) {
            uint32_t n_tnodes = 0;
            rc = build_binary_device(D, Q0, Q1, NIT, {{0u, NIT}}, d_err, &tnodes, &n_tnodes, st, err);
            if (rc) return rc;
            rc = wide_structure(D, tnodes, n_tnodes, 1, d_err, &tw, st, err);
            if (rc) return rc;
            tlas_total = tw.root_sizes[0];
            H->scalars.tlas_root = blas_total;
            rc = wide_index(D, tw, {blas_total}, st, err);
            if (rc) return rc;
        }
    }
    H->tlas_nodes = tlas_total;

    // ---- outputs ------------------------------------------------------------------------
    const uint64_t total = (uint64_t)blas_total + tlas_total;
    out->n_nodes = total;
    rc = rc ? rc : dev_alloc(out->allocations, &out->nodes, WIDE_NODE_WORDS * total, st, err);
    rc = rc ? rc : dev_alloc(out->allocations, &out->tris, 3 * N, st, err);
    rc = rc ? rc : dev_alloc(out->allocations, &out->inst_xf, 3ull * NI, st, err);
    rc = rc ? rc : dev_alloc(out->allocations, &out->inst, NI, st, err);
    rc = rc ? rc : dev_alloc(out->allocations, &out->items, NIT, st, err);
    if (rc) return rc;
    if (N) {
        rc = wide_words(bw, bnodes, out->nodes, total, d_err, st, err);
        if (rc) return rc;
        k_tri_gather<<<blocks_for(N, 256), 256, 0, st>>>(P0, d_pos, d_idx, d_tri_base, d_vbase, M, (uint32_t)N, out->tris);
    }
    if (NI) {
        BV_TRY(cudaMemcpyAsync(out->inst_xf, xf.data(), xf.size() * sizeof(float4), cudaMemcpyHostToDevice, st));
        BV_TRY(cudaMemcpyAsync(out->inst, rec.data(), rec.size() * sizeof(uint4), cudaMemcpyHostToDevice, st));
    }
    if (NIT) {
        rc = wide_words(tw, tnodes, out->nodes, total, d_err, st, err);
        if (rc) return rc;
        k_item_gather<<<blocks_for(NIT, 256), 256, 0, st>>>(Q0, d_items, NIT, out->items);
    }
    BV_TRY(cudaGetLastError());
    uint32_t e = 0;
    BV_TRY(cudaMemcpyAsync(&e, d_err, 4, cudaMemcpyDeviceToHost, st));
    BV_TRY(cudaStreamSynchronize(st));
    if (e) {
        *err = berr_text(e);
        return RT_ERR_DEVICE;
    }
    return RT_OK;
}

}  // namespace rt

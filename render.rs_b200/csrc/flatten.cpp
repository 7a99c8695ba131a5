// flatten.cpp — scene flattening for the CUDA backend (host, C++17).
//
// 1. Binary BVHs are built with the reference's binned-SAH rules
//    (src/accel/bvh.rs:96-108, 256-345: 16 bins on the widest centroid axis,
//    leaves of <= 4 primitives or <= 16 when SAH prefers a leaf, median
//    fallback, the same in-place partition), so the GPU sees the same tree
//    the reference's CPU path traverses.
// 2. Each binary tree is collapsed into 8-wide nodes (the child with the
//    largest surface area is opened until 8 children), and the child boxes
//    are quantised to 8 bits per plane against a per-node power-of-two grid
//    chosen so every decoded plane p + q * 2^e is exactly representable in
//    f32 and never inside the true box (conservative).
// 3. The light BVH follows src/scene/light_sampler.rs:97-141, 242-312.
// 4. Materials are folded to f32 constants as src/raytracer/pt/bxdf.rs and
//    src/scene/pbr.rs evaluate them.

#include "flatten.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <atomic>
#include <functional>
#include <limits>
#include <condition_variable>
#include <mutex>
#include <thread>

namespace rt {

namespace {

const double PI = 3.14159265358979323846;
const double INF = std::numeric_limits<double>::infinity();

struct Box {
    double lo[3] = {INF, INF, INF};
    double hi[3] = {-INF, -INF, -INF};
    // Plain comparisons (inputs are finite: flatten_scene rejects NaN/inf
    // vertices), which compile to minsd / maxsd. grow() takes the union of
    // two boxes, so an empty box leaves the other unchanged; the reference's
    // Aabb::grow (src/accel/bvh.rs:36-39) grows by the other's corner points,
    // which makes a union with an empty SAH bin infinite and rules out every
    // split with an empty bin on either side. Here those splits stay open.
    void grow_pt(const double* p) {
        for (int a = 0; a < 3; a++) {
            lo[a] = p[a] < lo[a] ? p[a] : lo[a];
            hi[a] = p[a] > hi[a] ? p[a] : hi[a];
        }
    }
    void grow(const Box& b) {
        for (int a = 0; a < 3; a++) {
            lo[a] = b.lo[a] < lo[a] ? b.lo[a] : lo[a];
            hi[a] = b.hi[a] > hi[a] ? b.hi[a] : hi[a];
        }
    }
    double area() const {
        double d0 = hi[0] - lo[0], d1 = hi[1] - lo[1], d2 = hi[2] - lo[2];
        if (d0 < 0 || d1 < 0 || d2 < 0) return 0.0;
        return 2.0 * (d0 * d1 + d1 * d2 + d2 * d0);
    }
};

// Run fn(begin, end) over [0, n) in contiguous chunks on all host threads
// (one thread when n is below two chunks of min_chunk items).
void parallel_for(size_t n, const std::function<void(size_t, size_t)>& fn, size_t min_chunk = 65536) {
    size_t threads = std::max<size_t>(1, std::min<size_t>(16, std::thread::hardware_concurrency()));
    threads = std::min(threads, std::max<size_t>(1, n / min_chunk));
    if (threads <= 1) {
        fn(0, n);
        return;
    }
    std::vector<std::thread> pool;
    for (size_t t = 0; t < threads; t++)
        pool.emplace_back([&, t] { fn(n * t / threads, n * (t + 1) / threads); });
    for (auto& th : pool) th.join();
}

// A box in f32 for the builders: rounded outward (exact for boxes of f32
// vertices), with -0 folded into +0 so every comparison-based and key-based
// min / max agrees.
void f32_box(const Box& b, float* lo, float* hi) {
    for (int a = 0; a < 3; a++) {
        float l = (float)b.lo[a], h = (float)b.hi[a];
        if ((double)l > b.lo[a]) l = std::nextafter(l, -INFINITY);
        if ((double)h < b.hi[a]) h = std::nextafter(h, INFINITY);
        lo[a] = l + 0.0f;
        hi[a] = h + 0.0f;
    }
}

struct BinNode {
    Box b;
    uint32_t first = 0, count = 0;  // interior: first = left child index, count = 0
};

struct BinBvh {
    std::vector<BinNode> nodes;
    std::vector<uint32_t> order;
};

// Binned SAH with the reference's split rules. Subtrees are independent
// (each partitions only its own primitive range), so large ones are built on
// their own threads; the tree is the same as a sequential build, only the
// node numbering differs, and nothing downstream depends on it. The
// primitives' boxes and centroids are partitioned in place with their
// indices (the reference's swap partition, same order), so every pass over a
// node's range reads memory sequentially.
BinBvh build_binary(const std::vector<Box>& bounds) {
// Build-time options. 32 bins, or SAH over all three axes, traced the
// 1M-triangle cloud within 2% of the reference's rule (16 bins, widest axis)
// and took 6-28% longer to build, so the reference's rule is the default.
#ifndef RT_SAH_BINS
#define RT_SAH_BINS 16      // the reference's bin count
#endif
#ifndef RT_SAH_ALL_AXES
#define RT_SAH_ALL_AXES 0   // 0: the widest centroid axis only (the reference's rule)
#endif
    const int BINS = RT_SAH_BINS, MAX_LEAF = 4;
    BinBvh t;
    size_t n = bounds.size();
    t.order.resize(n);
    if (n == 0) return t;
    // Primitive boxes are kept in f32 (28-byte records: the passes are
    // memory-bound). Triangle bounds come from f32 vertices, so they are
    // exact and every SAH decision (made in f64 from these values) is the
    // one an f64 record would give; other boxes (instances) are rounded
    // outward, which keeps them conservative.
    struct Prim {
        float lo[3], hi[3];
        uint32_t idx;
        double c(int a) const { return ((double)lo[a] + (double)hi[a]) * 0.5; }  // centroid, as the reference
        Box box() const {
            Box b;
            for (int a = 0; a < 3; a++) {
                b.lo[a] = lo[a];
                b.hi[a] = hi[a];
            }
            return b;
        }
    };
    std::vector<Prim> prims(n);
    for (size_t i = 0; i < n; i++) {
        f32_box(bounds[i], prims[i].lo, prims[i].hi);
        prims[i].idx = (uint32_t)i;
    }
    t.nodes.resize(2 * n + 1);
    std::atomic<size_t> next{1};
    Prim* P = prims.data();
    BinNode* nodes = t.nodes.data();
    struct Job { size_t node, start, count; };
    const size_t PAR_MIN = 32768;
    const int max_threads = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));

    // Nodes of at least PAR_SPLIT primitives (the top levels, which are the
    // build's critical path) run their passes on all threads: chunked bounds
    // and bins merged afterwards, and a stable two-pass partition through a
    // scratch buffer (same left / right sets as the swap partition; the order
    // within each side differs, which only permutes leaf contents).
    const size_t PAR_SPLIT = 262144;
    const size_t CHUNKS = (size_t)max_threads;
    auto chunked = [&](size_t count, const std::function<void(size_t, size_t, size_t)>& fn) {
        std::vector<std::thread> pool;
        for (size_t c = 1; c < CHUNKS; c++) pool.emplace_back([&, c] { fn(c, count * c / CHUNKS, count * (c + 1) / CHUNKS); });
        fn(0, 0, count / CHUNKS);
        for (auto& th : pool) th.join();
    };
    std::vector<Prim> scratch;

    // One level: bounds, split choice, partition. Returns false for a leaf.
    auto split_node = [&](const Job& j, size_t* split_out) -> bool {
        Prim* r = P + j.start;
        const bool wide_node = j.count >= PAR_SPLIT && CHUNKS > 1;
        Box b, cb;
        if (wide_node) {
            std::vector<Box> pb(CHUNKS), pcb(CHUNKS);
            chunked(j.count, [&](size_t c, size_t i0, size_t i1) {
                for (size_t i = i0; i < i1; i++) {
                    pb[c].grow(r[i].box());
                    const double cc[3] = {r[i].c(0), r[i].c(1), r[i].c(2)};
                    pcb[c].grow_pt(cc);
                }
            });
            for (size_t c = 0; c < CHUNKS; c++) {
                b.grow(pb[c]);
                cb.grow(pcb[c]);
            }
        } else {
            for (size_t i = 0; i < j.count; i++) {
                b.grow(r[i].box());
                const double c[3] = {r[i].c(0), r[i].c(1), r[i].c(2)};
                cb.grow_pt(c);
            }
        }
        nodes[j.node].b = b;
        auto make_leaf = [&]() {
            nodes[j.node].first = (uint32_t)j.start;
            nodes[j.node].count = (uint32_t)j.count;
        };
        if (j.count <= (size_t)MAX_LEAF) {
            make_leaf();
            return false;
        }
        double ext[3] = {cb.hi[0] - cb.lo[0], cb.hi[1] - cb.lo[1], cb.hi[2] - cb.lo[2]};
        const int widest = (ext[0] >= ext[1] && ext[0] >= ext[2]) ? 0 : (ext[1] >= ext[2] ? 1 : 2);
        size_t split = j.start + j.count / 2;
        // SAH over the bins of one axis: (cost, bin after which to split).
        auto eval_axis = [&](int axis, int* best_bin_out) -> double {
            const double amin = cb.lo[axis], aext = ext[axis];
            Box bb[BINS];
            size_t bc[BINS] = {0};
            double scale = (double)BINS / aext;
            auto bin_range = [&](size_t i0, size_t i1, Box* obb, size_t* obc) {
                for (size_t i = i0; i < i1; i++) {
                    double f = (r[i].c(axis) - amin) * scale;
                    size_t k = f > 0.0 ? (size_t)f : 0;
                    if (k > (size_t)BINS - 1) k = BINS - 1;
                    obc[k]++;
                    obb[k].grow(r[i].box());
                }
            };
            if (wide_node) {
                std::vector<Box> pbb(CHUNKS * BINS);
                std::vector<size_t> pbc(CHUNKS * BINS, 0);
                chunked(j.count, [&](size_t c, size_t i0, size_t i1) { bin_range(i0, i1, &pbb[c * BINS], &pbc[c * BINS]); });
                for (size_t c = 0; c < CHUNKS; c++)
                    for (int k = 0; k < BINS; k++) {
                        bb[k].grow(pbb[c * BINS + k]);
                        bc[k] += pbc[c * BINS + k];
                    }
            } else {
                bin_range(0, j.count, bb, bc);
            }
            Box racc[BINS], acc;
            for (int i = BINS - 1; i >= 1; i--) {
                acc.grow(bb[i]);
                racc[i] = acc;
            }
            double best = INF;
            int best_bin = 0;
            Box left;
            size_t lc = 0;
            for (int i = 0; i < BINS - 1; i++) {
                left.grow(bb[i]);
                lc += bc[i];
                size_t rc = j.count - lc;
                if (lc == 0 || rc == 0) continue;
                double cost = left.area() * (double)lc + racc[i + 1].area() * (double)rc;
                if (cost < best) {
                    best = cost;
                    best_bin = i;
                }
            }
            *best_bin_out = best_bin;
            return best;
        };
        int axis = widest;
        if (ext[widest] > 1e-12) {
            int best_bin = 0;
            double best = eval_axis(widest, &best_bin);
            if (RT_SAH_ALL_AXES) {
                for (int a = 0; a < 3; a++) {
                    if (a == widest || !(ext[a] > 1e-12)) continue;
                    int bb_a = 0;
                    double c = eval_axis(a, &bb_a);
                    if (c < best) {
                        best = c;
                        best_bin = bb_a;
                        axis = a;
                    }
                }
            }
            const double amin = cb.lo[axis], aext = ext[axis];
            double leaf_cost = b.area() * (double)j.count;
            if (std::isfinite(best) && best < leaf_cost) {
                double boundary = amin + aext * (double)(best_bin + 1) / (double)BINS;
                size_t m = 0;
                if (wide_node) {
                    std::vector<size_t> nleft(CHUNKS, 0);
                    chunked(j.count, [&](size_t c, size_t i0, size_t i1) {
                        size_t cnt = 0;
                        for (size_t i = i0; i < i1; i++) cnt += r[i].c(axis) < boundary;
                        nleft[c] = cnt;
                    });
                    for (size_t c = 0; c < CHUNKS; c++) m += nleft[c];
                    std::vector<size_t> lo_at(CHUNKS), hi_at(CHUNKS);
                    size_t lacc = 0, racc_n = m;
                    for (size_t c = 0; c < CHUNKS; c++) {
                        lo_at[c] = lacc;
                        hi_at[c] = racc_n;
                        size_t len = j.count * (c + 1) / CHUNKS - j.count * c / CHUNKS;
                        lacc += nleft[c];
                        racc_n += len - nleft[c];
                    }
                    Prim* tmp = scratch.data() + j.start;  // this node's own range of the scratch buffer
                    chunked(j.count, [&](size_t c, size_t i0, size_t i1) {
                        size_t lw = lo_at[c], rw = hi_at[c];
                        for (size_t i = i0; i < i1; i++) {
                            if (r[i].c(axis) < boundary) tmp[lw++] = r[i];
                            else tmp[rw++] = r[i];
                        }
                    });
                    chunked(j.count, [&](size_t, size_t i0, size_t i1) {
                        std::copy(tmp + i0, tmp + i1, r + i0);
                    });
                } else {
                    for (size_t q = 0; q < j.count; q++) {
                        if (r[q].c(axis) < boundary) {
                            if (q != m) std::swap(r[m], r[q]);
                            m++;
                        }
                    }
                }
                if (m > 0 && m < j.count) split = j.start + m;
            } else if (j.count <= (size_t)MAX_LEAF * 4) {
                make_leaf();
                return false;
            }
        }
        *split_out = split;
        return true;
    };

    // Worker pool: subtrees of at least PAR_MIN primitives go to a shared
    // queue that idle workers take from; smaller ones are finished by the
    // worker that split them.
    std::mutex mu;
    std::condition_variable cv;
    std::vector<Job> shared{Job{0, 0, n}};
    int busy = 0;
    auto worker = [&]() {
        for (;;) {
            Job root;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return !shared.empty() || busy == 0; });
                if (shared.empty()) return;  // nothing queued and nobody can add more
                root = shared.back();
                shared.pop_back();
                busy++;
            }
            std::vector<Job> stack{root};
            while (!stack.empty()) {
                Job j = stack.back();
                stack.pop_back();
                size_t split;
                if (!split_node(j, &split)) continue;
                size_t l = next.fetch_add(2);
                nodes[j.node].first = (uint32_t)l;
                nodes[j.node].count = 0;
                Job left{l, j.start, split - j.start}, right{l + 1, split, j.start + j.count - split};
                if (left.count >= PAR_MIN) {
                    {
                        std::lock_guard<std::mutex> lk(mu);
                        shared.push_back(left);
                    }
                    cv.notify_one();
                    stack.push_back(right);
                } else {
                    stack.push_back(right);
                    stack.push_back(left);
                }
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                busy--;
            }
            cv.notify_all();
        }
    };
    if (n >= PAR_SPLIT && CHUNKS > 1) scratch.resize(n);
    const int workers = n >= PAR_MIN ? max_threads : 1;
    std::vector<std::thread> pool;
    for (int w = 1; w < workers; w++) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    t.nodes.resize(next.load());
    for (size_t i = 0; i < n; i++) t.order[i] = P[i].idx;
    return t;
}

// Per-node quantisation grid: origin p (multiple of s = 2^e) and e such that
// every p + q*s (q in 0..255) is an exact f32 and p + 255*s >= box hi.
void choose_grid(double lo, double hi, float* p_out, int* e_out) {
    if (!(hi >= lo)) hi = lo;
    double maxabs = std::fmax(std::fabs(lo), std::fabs(hi));
    int e_ulp = -149;
    if (maxabs > 0) e_ulp = std::ilogb(maxabs) - 23 + 4;  // floor(log2), exact
    double extent = hi - lo;
    int e = -126;
    if (extent > 0) {  // ceil(log2(extent / 255)), exact
        int q;
        double mant = std::frexp(extent / 255.0, &q);
        e = mant == 0.5 ? q - 1 : q;
    }
    e = std::max(std::max(e, e_ulp), -126);
    for (;;) {
        double s = std::ldexp(1.0, e);
        double p = std::floor(lo / s) * s;
        if ((hi - p) / s <= 255.0 && (float)p == p) {
            *p_out = (float)p;
            *e_out = e;
            return;
        }
        e++;
    }
}

struct Collapser {
    const BinBvh& bin;
    std::vector<uint4>& out;
    uint32_t prim_base;
    uint64_t emitted = 0;
    uint64_t decode_errors = 0;
    // Structure first (sequential recursion: which binary nodes become the
    // children of each wide node), then quantisation of all wide nodes in
    // parallel (finish()).
    struct Wide {
        uint32_t idx, nk;
        uint32_t kids[8], refs[8];
    };
    std::vector<Wide> wide;

    uint32_t leaf_ref(const BinNode& nd) const { return make_leaf_ref(prim_base + nd.first, nd.count); }

    // Reserve the wide node covering binary node `bi` (and, recursively, its
    // descendants); returns its index. finish() writes the words.
    uint32_t emit(uint32_t bi) {
        const BinNode& root = bin.nodes[bi];
        Wide w{};
        uint32_t nk = 0;
        if (root.count > 0) {
            w.kids[nk++] = bi;  // a lone leaf becomes a one-child wide node
        } else {
            w.kids[nk++] = root.first;
            w.kids[nk++] = root.first + 1;
            while (nk < 8) {
                int best = -1;
                double best_a = -1.0;
                for (uint32_t k = 0; k < nk; k++) {
                    const BinNode& c = bin.nodes[w.kids[k]];
                    if (c.count == 0 && c.b.area() > best_a) {
                        best_a = c.b.area();
                        best = (int)k;
                    }
                }
                if (best < 0) break;
                uint32_t open = w.kids[best];
                w.kids[best] = bin.nodes[open].first;
                w.kids[nk++] = bin.nodes[open].first + 1;
            }
        }
        w.nk = nk;
        w.idx = (uint32_t)(out.size() / WIDE_NODE_WORDS);
        out.resize(out.size() + WIDE_NODE_WORDS);
        emitted++;
        const size_t slot = wide.size();
        wide.push_back(w);
        for (int k = 0; k < 8; k++) wide[slot].refs[k] = REF_EMPTY;
        for (uint32_t k = 0; k < nk; k++) {
            const BinNode& c = bin.nodes[wide[slot].kids[k]];
            uint32_t r = c.count > 0 ? leaf_ref(c) : emit(wide[slot].kids[k]);
            wide[slot].refs[k] = r;
        }
        return w.idx;
    }

    void finish() {
        std::atomic<uint64_t> errors{0};
        parallel_for(wide.size(), [&](size_t w0, size_t w1) {
            uint64_t local_errors = 0;
            for (size_t wi = w0; wi < w1; wi++) local_errors += write(wide[wi]);
            errors += local_errors;
        }, 2048);
        decode_errors += errors.load();
    }

    // Quantise one wide node's child boxes and write its 6 words; returns the
    // number of decode checks that failed.
    uint64_t write(const Wide& wn) {
        const uint32_t nk = wn.nk;
        uint64_t errors = 0;
        // Node box = union of children boxes.
        Box nb;
        for (uint32_t k = 0; k < nk; k++) nb.grow(bin.nodes[wn.kids[k]].b);
        float p[3];
        int e[3];
        double sc[3];
        for (int a = 0; a < 3; a++) {
            choose_grid(nb.lo[a], nb.hi[a], &p[a], &e[a]);
            sc[a] = std::ldexp(1.0, e[a]);
        }
        uint8_t qlo[3][8], qhi[3][8];
        for (int k = 0; k < 8; k++)
            for (int a = 0; a < 3; a++) {
                qlo[a][k] = 255;
                qhi[a][k] = 0;
            }
        for (uint32_t k = 0; k < nk; k++) {
            const Box& cbx = bin.nodes[wn.kids[k]].b;
            for (int a = 0; a < 3; a++) {
                const double s = sc[a];
                double ql = std::floor((cbx.lo[a] - (double)p[a]) / s);
                double qh = std::ceil((cbx.hi[a] - (double)p[a]) / s);
                ql = std::min(std::max(ql, 0.0), 255.0);
                qh = std::min(std::max(qh, 0.0), 255.0);
                // Conservative by construction; widen if rounding ever bit.
                while (ql > 0 && (double)p[a] + ql * s > cbx.lo[a]) ql -= 1;
                while (qh < 255 && (double)p[a] + qh * s < cbx.hi[a]) qh += 1;
                qlo[a][k] = (uint8_t)ql;
                qhi[a][k] = (uint8_t)qh;
                // The traversal decodes fma(2^23 + q, s, p - 2^23 s) in f32;
                // it must reproduce p + q s exactly and enclose the child.
                float sf = (float)s, p2 = p[a] - 8388608.0f * sf;
                float dlo = std::fmaf(8388608.0f + (float)ql, sf, p2);
                float dhi = std::fmaf(8388608.0f + (float)qh, sf, p2);
                if ((double)dlo != (double)p[a] + ql * s || (double)dhi != (double)p[a] + qh * s ||
                    (double)dlo > cbx.lo[a] || (double)dhi < cbx.hi[a])
                    errors++;
            }
        }
        uint4* w = &out[(size_t)wn.idx * WIDE_NODE_WORDS];
        uint32_t pb[3];
        memcpy(pb, p, sizeof(pb));
        w[0] = make_uint4(pb[0], pb[1], pb[2],
                          (uint32_t)(e[0] + 127) | ((uint32_t)(e[1] + 127) << 8) | ((uint32_t)(e[2] + 127) << 16) |
                              ((uint32_t)nk << 24));
        auto pack4 = [](const uint8_t* b) {
            return (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) | ((uint32_t)b[3] << 24);
        };
        w[1] = make_uint4(pack4(qlo[0]), pack4(qlo[0] + 4), pack4(qlo[1]), pack4(qlo[1] + 4));
        w[2] = make_uint4(pack4(qlo[2]), pack4(qlo[2] + 4), pack4(qhi[0]), pack4(qhi[0] + 4));
        w[3] = make_uint4(pack4(qhi[1]), pack4(qhi[1] + 4), pack4(qhi[2]), pack4(qhi[2] + 4));
        w[4] = make_uint4(wn.refs[0], wn.refs[1], wn.refs[2], wn.refs[3]);
        w[5] = make_uint4(wn.refs[4], wn.refs[5], wn.refs[6], wn.refs[7]);
        return errors;
    }
};

inline double lum(const double* c) { return 0.2126 * c[0] + 0.7152 * c[1] + 0.0722 * c[2]; }

// Affine 3x4 inverse in f64; identity when |det| < 1e-6 as the reference's
// Matrix4::inverse().unwrap_or(identity) (src/geometry/mesh.rs:282).
void affine_inverse(const double* m, double* inv) {
    double a = m[0], b = m[1], c = m[2], d = m[4], e = m[5], f = m[6], g = m[8], h = m[9], i = m[10];
    double A = e * i - f * h, B = -(d * i - f * g), Cc = d * h - e * g;
    double det = a * A + b * B + c * Cc;
    if (std::fabs(det) < 1e-6) {
        static const double id[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};
        memcpy(inv, id, sizeof(id));
        return;
    }
    double r[9] = {A, -(b * i - c * h), b * f - c * e, B, a * i - c * g, -(a * f - c * d), Cc, -(a * h - b * g),
                   a * e - b * d};
    for (int k = 0; k < 9; k++) r[k] /= det;
    double t[3] = {m[3], m[7], m[11]};
    for (int row = 0; row < 3; row++) {
        inv[row * 4 + 0] = r[row * 3 + 0];
        inv[row * 4 + 1] = r[row * 3 + 1];
        inv[row * 4 + 2] = r[row * 3 + 2];
        inv[row * 4 + 3] = -(r[row * 3 + 0] * t[0] + r[row * 3 + 1] * t[1] + r[row * 3 + 2] * t[2]);
    }
}

void xf_point(const double* m, const double* p, double* o) {
    for (int r = 0; r < 3; r++) o[r] = m[r * 4] * p[0] + m[r * 4 + 1] * p[1] + m[r * 4 + 2] * p[2] + m[r * 4 + 3];
}

DevMaterial fold_material(const rt_material_desc& m) {
    DevMaterial d;
    memset(&d, 0, sizeof(d));
    // PbrParams::specular_f0 (pbr.rs:86-96)
    double f0[3] = {0, 0, 0};
    if (lum(m.specular_face_color) > 1e-6) {
        for (int k = 0; k < 3; k++) f0[k] = m.specular_face_color[k];
    } else if (m.specular_ior > 1.0) {
        double r = (m.specular_ior - 1.0) / (m.specular_ior + 1.0);
        for (int k = 0; k < 3; k++) f0[k] = r * r;
    }
    bool has_spec = lum(f0) > 1e-6;
    // lobe_weights (pbr.rs:188-201)
    double wd = m.diffuse_gain * lum(m.diffuse_color);
    double ws = std::sqrt(lum(f0));
    double wc = m.clearcoat_gain * 0.2;
    double wf = m.fuzz_gain * lum(m.fuzz_color) * 0.3;
    double wg = m.glass_gain;
    double total = wd + ws + wc + wf + wg;
    bool lobes = total > 1e-9;
    if (lobes) {
        d.w_diff = (float)(wd / total);
        d.w_spec = (float)(ws / total);
        d.w_coat = (float)(wc / total);
        d.w_fuzz = (float)(wf / total);
        d.w_glass = (float)(wg / total);
    }
    d.has_lobes = lobes ? 1.0f : 0.0f;
    // under_layer_scale (bxdf.rs:137-143)
    double uls = std::min(std::max((1.0 - lum(f0)) * (1.0 - 0.04 * m.clearcoat_gain), 0.0), 1.0);
    double sigma2 = m.diffuse_roughness * m.diffuse_roughness;
    d.on_a = (float)(1.0 - sigma2 / (2.0 * (sigma2 + 0.33)));
    d.on_b = (float)(0.45 * sigma2 / (sigma2 + 0.09));
    auto alpha_of = [](double r) { return std::min(std::max(r * r, 2.5e-5), 1.0); };
    d.alpha_spec = (float)alpha_of(m.specular_roughness);
    d.alpha_coat = (float)alpha_of(m.clearcoat_roughness);
    d.alpha_glass = (float)alpha_of(m.glass_roughness);
    d.coat_gain = (float)m.clearcoat_gain;
    d.glass_scale = (float)(m.glass_gain * uls);
    d.ior = (float)m.glass_ior;
    d.presence = (float)std::min(std::max(m.presence, 0.0), 1.0);
    double alb[3];
    for (int k = 0; k < 3; k++) {
        d.kd[k] = (float)(m.diffuse_color[k] * m.diffuse_gain * uls / PI);
        d.f0[k] = (float)f0[k];
        d.f90[k] = (float)m.specular_edge_color[k];
        d.kfuzz[k] = (float)(m.fuzz_color[k] * m.fuzz_gain / PI);
        d.refr[k] = (float)m.refraction_color[k];
        d.emission[k] = (float)(m.emission[k] + m.glow[k]);
        alb[k] = m.diffuse_color[k] * m.diffuse_gain + f0[k] * (has_spec ? 1.0 : 0.0) +
                 m.subsurface_color[k] * m.subsurface_gain + m.refraction_color[k] * m.glass_gain;
        d.albedo[k] = (float)std::fmin(alb[k], 1.0);
    }
    d.area_light = m.area_light;
    d.id = m.id;
    // Interior medium (validated by the caller) and volume hulls
    // (pt/mod.rs:662-667): no lobes and no emission; a hull is never a
    // cutout, the reference testing it before presence.
    d.interior = m.interior >= 0 ? (uint32_t)m.interior : 0xFFFFFFFFu;
    const bool emits = std::max({m.emission[0] + m.glow[0], m.emission[1] + m.glow[1], m.emission[2] + m.glow[2]}) > 0.0;
    d.hull = (m.interior >= 0 && !m.hair && !lobes && !emits) ? 1.0f : 0.0f;
    if (d.hull != 0.0f) d.presence = 1.0f;
    // Subsurface walk: probability and the Burley-fit medium (volume.rs:259-288).
    d.sss_gain = m.hair ? 0.0f : (float)std::min(std::max(m.subsurface_gain, 0.0), 1.0);
    d.hair = 0xFFFFFFFFu;  // set by the caller with the hair table
    for (int k = 0; k < 3; k++) {
        const double a = std::min(std::max(m.subsurface_color[k], 0.0), 1.0);
        const double st = (1.85 - a + 7.0 * std::pow(std::fabs(a - 0.8), 3)) / std::max(m.subsurface_dmfp[k], 1e-5);
        const double alpha = 1.0 - std::exp(-a * (11.43 - 15.38 * a + 13.91 * a * a));
        d.sss_st[k] = (float)st;
        d.sss_ss[k] = (float)(alpha * st);
    }
    if (!lobes) d.mclass = MAT_EMITTER;
    else if (wd > 0 && ws == 0 && wc == 0 && wf == 0 && wg == 0) d.mclass = MAT_DIFFUSE;
    else if (ws > 0 && wd == 0 && wc == 0 && wf == 0 && wg == 0) d.mclass = MAT_CONDUCTOR;
    else if (wg > 0 && wd == 0 && ws == 0 && wc == 0 && wf == 0) d.mclass = MAT_GLASS;
    else d.mclass = MAT_MIXED;
    return d;
}

// HairParams::new (hair.rs:40-55): clamped roughnesses, the longitudinal
// variance per lobe, the azimuthal logistic scale.
DevHair hair_dev(const rt_material_desc& md) {
    DevHair hp{};
    const double bm = std::min(std::max(md.hair_beta_m, 0.01), 1.0);
    const double bn = std::min(std::max(md.hair_beta_n, 0.01), 1.0);
    double v0 = 0.726 * bm + 0.812 * bm * bm + 3.7 * std::pow(bm, 20);
    v0 *= v0;
    const double v[4] = {v0, 0.25 * v0, 4.0 * v0, 4.0 * v0};
    for (int k = 0; k < 4; k++) hp.v[k] = (float)v[k];
    for (int c = 0; c < 3; c++) hp.sigma_a[c] = (float)md.hair_sigma_a[c];
    hp.eta = (float)md.hair_eta;
    hp.s = (float)(0.626657069 * (0.265 * bn + 1.194 * bn * bn + 5.372 * std::pow(bn, 22)));
    return hp;
}

// Light BVH (light_sampler.rs:242-312): median split on the widest axis of
// the light-extent box, stable sort by centre along that axis.
struct LEntry {
    uint32_t light;
    double c[3], radius, power;
};

uint32_t lbvh_build(std::vector<LightNode>& nodes, std::vector<uint32_t>& leaf_of, const std::vector<LEntry>& e,
                    std::vector<size_t>& order, size_t s, size_t t, uint32_t parent) {
    uint32_t index = (uint32_t)nodes.size();
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    double power = 0;
    for (size_t k = s; k < t; k++) {
        const LEntry& en = e[order[k]];
        for (int a = 0; a < 3; a++) {
            mn[a] = std::fmin(mn[a], (float)(en.c[a] - en.radius));
            mx[a] = std::fmax(mx[a], (float)(en.c[a] + en.radius));
        }
        power += en.power;
    }
    LightNode nd;
    memset(&nd, 0, sizeof(nd));
    for (int a = 0; a < 3; a++) {
        nd.mn[a] = mn[a];
        nd.mx[a] = mx[a];
    }
    nd.power = (float)power;
    nd.parent = parent;
    nd.b = 0xFFFFFFFFu;
    nodes.push_back(nd);
    if (t - s == 1) {
        uint32_t l = e[order[s]].light;
        nodes[index].a = l;
        leaf_of[l] = index;
        return index;
    }
    int axis = 0;
    float widest = -1.0f;
    for (int a = 0; a < 3; a++)
        if (mx[a] - mn[a] > widest) {
            widest = mx[a] - mn[a];
            axis = a;
        }
    size_t mid = (s + t) / 2;
    std::stable_sort(order.begin() + s, order.begin() + t,
                     [&](size_t x, size_t y) { return e[x].c[axis] < e[y].c[axis]; });
    uint32_t a = lbvh_build(nodes, leaf_of, e, order, s, mid, index);
    uint32_t b = lbvh_build(nodes, leaf_of, e, order, mid, t, index);
    nodes[index].a = a;
    nodes[index].b = b;
    return index;
}

// Pattern graph and bindings (src/texture/pattern.rs, material.rs:29-30,
// 95-101) in device form. Nodes may read only lower-indexed nodes, so the
// graph is evaluated in index order; a material's bindings may reach at
// most RT_MAX_PATTERN_NODES consecutive nodes. A presence binding makes the
// scene's cutouts pattern-driven (DevScene::presence_pat).
bool flatten_patterns(const rt_scene_desc* d, HostScene& H, std::string* err) {
    if (!d->n_patterns && !d->n_bindings) return true;
    if ((d->n_patterns && !d->patterns) || (d->n_bindings && !d->bindings) || (d->n_textures && !d->textures)) {
        *err = "patterns, bindings or textures pointer is NULL";
        return false;
    }
    // Texture mip chains (texture/tex.rs:89-130): 2x2 f32 box averages,
    // odd sizes clamping the second tap, down to 1x1.
    for (uint32_t k = 0; k < d->n_textures; k++) {
        const rt_texture_desc& td = d->textures[k];
        if (!td.rgb || !td.width || !td.height) {
            *err = "texture " + std::to_string(k) + " has no pixels";
            return false;
        }
        DevTexture t{(uint32_t)H.tex_mips.size(), 0, (float)std::max(td.width, td.height), 0};
        std::vector<float> cur(td.rgb, td.rgb + 3ull * td.width * td.height), next;
        uint32_t w = td.width, h = td.height;
        for (;;) {
            if (H.texels.size() + (size_t)w * h >= (1ull << 32)) {
                *err = "textures hold more than 2^32 texels";
                return false;
            }
            H.tex_mips.push_back(DevMip{(uint32_t)H.texels.size(), w, h, 0});
            for (size_t p = 0; p < (size_t)w * h; p++)
                H.texels.push_back(make_float4(cur[3 * p], cur[3 * p + 1], cur[3 * p + 2], 0.0f));
            t.n_mips++;
            if (w == 1 && h == 1) break;
            const uint32_t nw = std::max(w / 2, 1u), nh = std::max(h / 2, 1u);
            next.assign(3ull * nw * nh, 0.0f);
            for (uint32_t y = 0; y < nh; y++) {
                const uint32_t y0 = std::min(2 * y, h - 1), y1 = std::min(2 * y + 1, h - 1);
                for (uint32_t x = 0; x < nw; x++) {
                    const uint32_t x0 = std::min(2 * x, w - 1), x1 = std::min(2 * x + 1, w - 1);
                    for (int c = 0; c < 3; c++) {
                        float sum = cur[3 * ((size_t)y0 * w + x0) + c] + cur[3 * ((size_t)y0 * w + x1) + c];
                        sum = sum + cur[3 * ((size_t)y1 * w + x0) + c];
                        sum = sum + cur[3 * ((size_t)y1 * w + x1) + c];
                        next[3 * ((size_t)y * nw + x) + c] = sum * 0.25f;
                    }
                }
            }
            cur.swap(next);
            w = nw;
            h = nh;
        }
        H.textures.push_back(t);
    }
    const uint32_t np = d->n_patterns;
    H.patterns.resize(np);
    for (uint32_t i = 0; i < np; i++) {
        const rt_pattern_desc& pd = d->patterns[i];
        DevPattern& g = H.patterns[i];
        memset(&g, 0, sizeof(g));
        if (pd.type < RT_PATTERN_CHECKER || pd.type > RT_PATTERN_TRIPLANAR) {
            *err = "pattern node " + std::to_string(i) + " has an unknown type";
            return false;
        }
        g.type = (uint32_t)pd.type;
        for (int k = 0; k < 3; k++) {
            const bool used = (pd.type == RT_PATTERN_MIX) || (pd.type == RT_PATTERN_COLOR_CORRECT && k == 0);
            g.in[k] = 0xFFFFFFFFu;
            if (used && pd.in[k].node >= 0) {
                if ((uint32_t)pd.in[k].node >= i) {
                    *err = "pattern node " + std::to_string(i) + " reads node " + std::to_string(pd.in[k].node) +
                           " (a node may read only nodes of lower index)";
                    return false;
                }
                g.in[k] = (uint32_t)pd.in[k].node;
            }
            for (int c = 0; c < 3; c++) g.c[k][c] = (float)pd.in[k].value[c];
        }
        switch (pd.type) {
            case RT_PATTERN_CHECKER:
                for (int c = 0; c < 3; c++) {
                    g.c[0][c] = (float)pd.color_a[c];
                    g.c[1][c] = (float)pd.color_b[c];
                }
                g.s0 = (float)pd.scale[0];
                g.s1 = (float)pd.scale[1];
                break;
            case RT_PATTERN_FRACTAL:
                g.s0 = (float)pd.frequency;
                g.s1 = (float)pd.gain;
                g.s2 = (float)pd.lacunarity;
                g.u0 = std::max(pd.octaves, 1u);
                if (g.u0 > 32) {
                    *err = "pattern node " + std::to_string(i) + " asks for more than 32 octaves";
                    return false;
                }
                break;
            case RT_PATTERN_COLOR_CORRECT:
                for (int c = 0; c < 3; c++) {
                    g.c[1][c] = (float)pd.color_a[c];
                    g.c[2][c] = (float)pd.color_b[c];
                }
                g.s0 = (float)pd.gamma;
                g.s1 = (float)pd.saturation;
                break;
            case RT_PATTERN_TEXTURE:
            case RT_PATTERN_TRIPLANAR:
                // A texture index outside the table is the reference's
                // missing texture (magenta), as is -1.
                g.u0 = (pd.texture >= 0 && (uint32_t)pd.texture < d->n_textures) ? (uint32_t)pd.texture : 0xFFFFFFFFu;
                if (pd.wrap > RT_WRAP_BLACK) {
                    *err = "pattern node " + std::to_string(i) + " has an unknown wrap mode";
                    return false;
                }
                g.u1 = pd.wrap;
                if (pd.n_udim) {
                    if (!pd.udim_tiles || !pd.udim_textures) {
                        *err = "pattern node " + std::to_string(i) + " has a UDIM set without tiles";
                        return false;
                    }
                    g.u2 = pd.n_udim;
                    g.udim_off = (uint32_t)H.udim.size();
                    for (uint32_t k = 0; k < pd.n_udim; k++) {
                        const int32_t t = pd.udim_textures[k];
                        H.udim.push_back(make_uint2(pd.udim_tiles[k], (t >= 0 && (uint32_t)t < d->n_textures)
                                                                          ? (uint32_t)t
                                                                          : 0xFFFFFFFFu));
                    }
                }
                if (pd.type == RT_PATTERN_TEXTURE) {
                    g.s0 = (float)pd.scale[0];
                    g.s1 = (float)pd.scale[1];
                } else {
                    g.s0 = (float)pd.frequency;
                }
                break;
            case RT_PATTERN_RAMP:
                if (pd.n_ramp && (!pd.ramp_positions || !pd.ramp_colors)) {
                    *err = "pattern node " + std::to_string(i) + " has a ramp without positions or colours";
                    return false;
                }
                g.u0 = (uint32_t)H.ramp.size();
                g.u1 = pd.n_ramp;
                g.u2 = pd.use_t ? 1u : 0u;
                for (uint32_t r = 0; r < pd.n_ramp; r++)
                    H.ramp.push_back(make_float4((float)pd.ramp_positions[r], (float)pd.ramp_colors[3 * r],
                                                 (float)pd.ramp_colors[3 * r + 1], (float)pd.ramp_colors[3 * r + 2]));
                break;
            default: break;
        }
    }
    std::vector<std::vector<uint2>> per_mat(d->n_materials);
    for (uint32_t b = 0; b < d->n_bindings; b++) {
        const rt_pattern_binding& pb = d->bindings[b];
        if (pb.material >= d->n_materials || pb.node >= np || pb.field > RT_FIELD_PRESENCE) {
            *err = "pattern binding " + std::to_string(b) + " names a missing material, node or field";
            return false;
        }
        if (pb.field == RT_FIELD_PRESENCE) {
            // Pattern-driven cutouts (texture alpha): decided where the
            // pattern is evaluated, at shading and per shadow-ray blocker.
            H.scalars.presence_pat = 1;
            H.scalars.any_presence = 1;
        }
        per_mat[pb.material].push_back(make_uint2(pb.field, pb.node));
    }
    H.mat_pat.assign(d->n_materials, DevMatPat{});
    for (uint32_t m = 0; m < d->n_materials; m++) {
        DevMatPat& mp = H.mat_pat[m];
        if (per_mat[m].empty()) continue;
        // Nodes reached from the bindings (inputs always point lower).
        std::vector<uint8_t> reach(np, 0);
        for (const uint2& b : per_mat[m]) reach[b.y] = 1;
        uint32_t lo = np, hi = 0;
        for (uint32_t i = np; i-- > 0;) {
            if (!reach[i]) continue;
            lo = std::min(lo, i);
            hi = std::max(hi, i);
            for (int k = 0; k < 3; k++)
                if (H.patterns[i].in[k] != 0xFFFFFFFFu) reach[H.patterns[i].in[k]] = 1;
        }
        if (hi - lo >= RT_MAX_PATTERN_NODES) {
            *err = "material " + std::to_string(m) + " reaches pattern nodes " + std::to_string(lo) + ".." +
                   std::to_string(hi) + " (at most 16 consecutive nodes per material)";
            return false;
        }
        mp.bind_off = (uint32_t)H.binds.size();
        mp.bind_n = (uint32_t)per_mat[m].size();
        mp.node_lo = lo;
        for (uint32_t i = lo; i <= hi; i++)
            if (reach[i]) mp.node_mask |= 1u << (i - lo);
        H.binds.insert(H.binds.end(), per_mat[m].begin(), per_mat[m].end());
        mp.pbr_index = (uint32_t)H.pbr.size();
        const rt_material_desc& md = d->materials[m];
        DevPbr p;
        p.diffuse_gain = (float)md.diffuse_gain;
        p.diffuse_roughness = (float)md.diffuse_roughness;
        p.spec_rough = (float)md.specular_roughness;
        p.spec_ior = (float)md.specular_ior;
        p.cc_gain = (float)md.clearcoat_gain;
        p.cc_rough = (float)md.clearcoat_roughness;
        p.fuzz_gain = (float)md.fuzz_gain;
        p.glass_gain = (float)md.glass_gain;
        p.glass_ior = (float)md.glass_ior;
        p.glass_rough = (float)md.glass_roughness;
        p.presence = (float)md.presence;
        for (int c = 0; c < 3; c++) {
            p.diffuse_color[c] = (float)md.diffuse_color[c];
            p.spec_face[c] = (float)md.specular_face_color[c];
            p.spec_edge[c] = (float)md.specular_edge_color[c];
            p.fuzz_color[c] = (float)md.fuzz_color[c];
            p.refraction[c] = (float)md.refraction_color[c];
            p.glow[c] = (float)md.glow[c];
            p.emission[c] = (float)md.emission[c];
            p.sss_albedo[c] = (float)(md.subsurface_color[c] * md.subsurface_gain);
        }
        p.pad_ = 0.0f;
        H.pbr.push_back(p);
        // The lobe set varies per hit: shade through the general class.
        H.materials[m].mclass = MAT_MIXED;
    }
    // Matrix4::approx_scale (math/matrix.rs:246-251): st density per world unit.
    H.inst_scale.resize(d->n_instances);
    for (uint32_t i = 0; i < d->n_instances; i++) {
        const double* x = d->instances[i].object_to_world;
        double l[3];
        for (int c = 0; c < 3; c++) l[c] = std::sqrt(x[c] * x[c] + x[4 + c] * x[4 + c] + x[8 + c] * x[8 + c]);
        H.inst_scale[i] = (float)std::max(std::cbrt(l[0] * l[1] * l[2]), 1e-12);
    }
    return true;
}

}  // namespace

DevMaterial fold_material_public(const rt_material_desc& m) { return fold_material(m); }
DevHair hair_dev_public(const rt_material_desc& m) { return hair_dev(m); }

// An instance is split into its BLAS root's children (one TLAS item each)
// when their world boxes' summed surface area is below RT_BRAID_RATIO times
// the area of their union: a ray crossing the instance's box then enters
// much less box area, which pays for the extra instance entries. Otherwise
// the instance is one item whose box is that union (tighter than the
// transformed root box for rotated instances). A volumetric mesh split in
// 8 has children of ~2x its surface area, so those stay whole. Measured
// (B200): the 1280x720 forest frame 239 -> 211 ms at 1.75 (-6% at 0 with
// union boxes alone, -16% at 1.9); at 2.2 and above the 1M-triangle cloud's
// single instance splits and its frame slows by 40%, the instanced scene by
// 18%. (RT_BRAID_RATIO in flatten.h.)
// In a dense scene, where the instances' boxes add up to more than
// RT_BRAID_DENSE times the world box's area (the forest: 385; the instanced
// scene: 5; one instance: 1), every instance with several root children is
// split: a ray there crosses hundreds of instance boxes, and the children's
// boxes overlap far less (forest frame 211 -> 182 ms). (RT_BRAID_DENSE in
// flatten.h.)

// World box of a local box under an affine 3x4: centre mapped, half
// extents through |M| (the exact box of the 8 transformed corners).
static Box world_box(const double* m, const float* lo, const float* hi) {
    Box wb;
    for (int r = 0; r < 3; r++) {
        double c = m[r * 4 + 3], e = 0.0;
        for (int k = 0; k < 3; k++) {
            const double ck = 0.5 * ((double)lo[k] + (double)hi[k]), hk = 0.5 * ((double)hi[k] - (double)lo[k]);
            c += m[r * 4 + k] * ck;
            e += std::fabs(m[r * 4 + k]) * hk;
        }
        wb.lo[r] = c - e;
        wb.hi[r] = c + e;
    }
    return wb;
}

void tlas_items(const rt_scene_desc* d, const std::vector<std::vector<RootChild>>& root_children,
                const std::vector<std::vector<RootChild>>& grand_children, std::vector<double>* boxes,
                std::vector<uint2>* items, HostScene* H) {
    const uint32_t n = d->n_instances;
    bool dense = false;
    // Shutter-close transforms of moving instances (mesh.rs:276-290: their
    // world boxes cover both endpoints; a corner moves on a segment under
    // the lerped transform, so the union of the two boxes bounds it).
    std::vector<const double*> xf1(n, nullptr);
    for (uint32_t k = 0; k < d->n_instance_motion; k++) xf1[d->instance_motion[k].instance] = d->instance_motion[k].object_to_world1;
    // World boxes of one instance's frontier (`list` per mesh), their union,
    // and how many items it becomes: every child in a dense scene, else the
    // children when their summed area is below RT_BRAID_RATIO x the union's.
    auto child_boxes = [&](uint32_t i, const std::vector<std::vector<RootChild>>& list, bool split_all, Box* cb,
                           Box* u) -> uint32_t {
        const rt_instance_desc& id = d->instances[i];
        if (!H->meshes[id.mesh_id].n_tris) return 0;
        const auto& rc = list[id.mesh_id];
        double sum = 0.0;
        for (size_t k = 0; k < rc.size(); k++) {
            Box wb = world_box(id.object_to_world, rc[k].lo, rc[k].hi);
            if (xf1[i]) wb.grow(world_box(xf1[i], rc[k].lo, rc[k].hi));
            if (cb) cb[k] = wb;
            u->grow(wb);
            sum += wb.area();
        }
        if (rc.size() <= 1) return 1u;
        return split_all || sum < RT_BRAID_RATIO * u->area() ? (uint32_t)rc.size() : 1u;
    };
    // Density: the instances' union boxes against the world box.
    {
        std::mutex mu_d;
        double total_area = 0.0;
        Box all;
        parallel_for(n, [&](size_t i0, size_t i1) {
            Box local;
            double a = 0.0;
            for (size_t i = i0; i < i1; i++) {
                Box u;
                if (child_boxes((uint32_t)i, root_children, false, nullptr, &u)) {
                    a += u.area();
                    local.grow(u);
                }
            }
            std::lock_guard<std::mutex> lk(mu_d);
            total_area += a;
            all.grow(local);
        }, 4096);
        dense = all.area() > 0.0 && total_area > RT_BRAID_DENSE * all.area();
        H->scalars.refill_at = dense ? RT_REFILL_DENSE : RT_REFILL_SPARSE;
    }
    // A dense scene splits every instance into its BLAS's second-level
    // frontier; others split an instance into its root's children when
    // they overlap little.
    const auto& list = dense ? grand_children : root_children;
    std::vector<uint64_t> off(n + 1, 0);
    parallel_for(n, [&](size_t i0, size_t i1) {
        Box cb[RT_TOP_MAX];
        for (size_t i = i0; i < i1; i++) {
            const rt_instance_desc& id = d->instances[i];
            if (dense) {
                const size_t k = list[id.mesh_id].size();
                off[i + 1] = d->meshes[id.mesh_id].n_triangles ? (k > 1 ? k : 1) : 0;
                continue;
            }
            Box u;
            off[i + 1] = child_boxes((uint32_t)i, list, false, cb, &u);
        }
    }, 4096);
    for (uint32_t i = 0; i < n; i++) off[i + 1] += off[i];
    const uint64_t total = off[n];
    boxes->assign(6 * total, 0.0);
    items->resize(total);
    std::mutex mu;
    Box world;
    parallel_for(n, [&](size_t i0, size_t i1) {
        Box local, cb[RT_TOP_MAX];
        for (size_t i = i0; i < i1; i++) {
            Box u;
            const uint32_t k_items = child_boxes((uint32_t)i, list, dense, cb, &u);
            const rt_instance_desc& id = d->instances[i];
            const auto& rc = list[id.mesh_id];
            for (uint32_t k = 0; k < k_items; k++) {
                const uint64_t j = off[i] + k;
                const Box& b = k_items == 1 ? u : cb[k];
                for (int a = 0; a < 3; a++) {
                    (*boxes)[6 * j + a] = b.lo[a];
                    (*boxes)[6 * j + 3 + a] = b.hi[a];
                }
                (*items)[j] = make_uint2((uint32_t)i, k_items == 1 ? H->meshes[id.mesh_id].blas_root : rc[k].ref);
            }
            if (k_items) local.grow(u);
        }
        std::lock_guard<std::mutex> lk(mu);
        world.grow(local);
    }, 4096);
    for (int a = 0; a < 3; a++) {
        H->world_lo[a] = world.lo[a] <= world.hi[a] ? world.lo[a] : 0.0;
        H->world_hi[a] = world.lo[a] <= world.hi[a] ? world.hi[a] : 0.0;
    }
}

void instance_records(const rt_scene_desc* d, const HostScene& H, std::vector<float4>* xf, std::vector<uint4>* rec) {
    const uint32_t n = d->n_instances;
    xf->resize(3ull * n);
    rec->resize(n);
    parallel_for(n, [&](size_t i0, size_t i1) {
        for (size_t i = i0; i < i1; i++) {
            const rt_instance_desc& id = d->instances[i];
            double v[12];
            affine_inverse(id.object_to_world, v);
            for (int r = 0; r < 3; r++)
                (*xf)[3 * i + r] = make_float4((float)v[r * 4], (float)v[r * 4 + 1], (float)v[r * 4 + 2], (float)v[r * 4 + 3]);
            (*rec)[i] = make_uint4(H.meshes[id.mesh_id].blas_root, (uint32_t)i, id.material_id, id.mesh_id);
        }
    }, 4096);
}

void prim_records(const std::vector<double>& boxes, float* out) {
    const size_t n = boxes.size() / 6;
    parallel_for(n, [&](size_t i0, size_t i1) {
        for (size_t i = i0; i < i1; i++) {
            Box b;
            for (int a = 0; a < 3; a++) {
                b.lo[a] = boxes[6 * i + a];
                b.hi[a] = boxes[6 * i + 3 + a];
            }
            float* o = out + 8 * i;
            f32_box(b, o, o + 4);
            uint32_t idx = (uint32_t)i;
            memcpy(&o[3], &idx, 4);
            o[7] = 0.0f;
        }
    });
}

// Analytic quadrics (rt_quadric_desc): f32 transforms both ways (the
// inverse in f64, identity when singular as Matrix4::inverse().unwrap_or),
// Matrix4::approx_scale, and the union of the world boxes of the shapes'
// local bounds (the learned proposal's position bounds include it).
bool flatten_quadrics(const rt_scene_desc* d, HostScene& H, std::string* err) {
    H.scalars.n_quadrics = 0;
    if (!d->n_quadrics) return true;
    if (!d->quadrics) {
        *err = "quadrics pointer is NULL";
        return false;
    }
    for (uint32_t k = 0; k < d->n_quadrics; k++) {
        const rt_quadric_desc& q = d->quadrics[k];
        if (q.type > RT_QUADRIC_HYPERBOLOID) {
            *err = "quadric " + std::to_string(k) + " has an unknown type";
            return false;
        }
        if (q.material_id >= d->n_materials) {
            *err = "quadric " + std::to_string(k) + " names a missing material";
            return false;
        }
        for (int j = 0; j < 12; j++)
            if (!std::isfinite(q.object_to_world[j])) {
                *err = "quadric " + std::to_string(k) + " has a non-finite transform";
                return false;
            }
        DevQuadric dq{};
        double inv[12];
        affine_inverse(q.object_to_world, inv);
        for (int r = 0; r < 3; r++) {
            dq.w2o[r] = make_float4((float)inv[r * 4], (float)inv[r * 4 + 1], (float)inv[r * 4 + 2], (float)inv[r * 4 + 3]);
            const double* m = q.object_to_world + r * 4;
            dq.o2w[r] = make_float4((float)m[0], (float)m[1], (float)m[2], (float)m[3]);
        }
        for (int j = 0; j < 8; j++) dq.prm[j] = (float)q.params[j];
        dq.type = q.type;
        dq.material = q.material_id;
        double len[3];
        for (int c = 0; c < 3; c++) {
            const double* m = q.object_to_world;
            len[c] = std::sqrt(m[c] * m[c] + m[4 + c] * m[4 + c] + m[8 + c] * m[8 + c]);
        }
        dq.scale = (float)std::fmax(std::cbrt(len[0] * len[1] * len[2]), 1e-12);
        H.quadrics.push_back(dq);
        // Local bounds of the shape, then the world box of its corners.
        const double* p = q.params;
        double lo[3], hi[3];
        auto box = [&](double rx, double z0, double z1) {
            lo[0] = lo[1] = -rx;
            hi[0] = hi[1] = rx;
            lo[2] = std::fmin(z0, z1);
            hi[2] = std::fmax(z0, z1);
        };
        switch (q.type) {
            case RT_QUADRIC_SPHERE: box(p[0], std::fmax(p[1], -p[0]), std::fmin(p[2], p[0])); break;
            case RT_QUADRIC_CYLINDER: box(p[0], p[1], p[2]); break;
            case RT_QUADRIC_CONE: box(p[1], 0.0, p[0]); break;
            case RT_QUADRIC_TORUS: box(p[0] + p[1], -p[1], p[1]); break;
            case RT_QUADRIC_DISK: box(p[1], p[0], p[0]); break;
            case RT_QUADRIC_PARABOLOID: box(p[0], p[1], p[2]); break;
            default:
                box(std::sqrt(std::fmax(p[0] * p[0] + p[1] * p[1], p[3] * p[3] + p[4] * p[4])), p[2], p[5]);
                break;
        }
        for (int c = 0; c < 8; c++) {
            const double pt[3] = {(c & 1) ? hi[0] : lo[0], (c & 2) ? hi[1] : lo[1], (c & 4) ? hi[2] : lo[2]};
            double w[3];
            xf_point(q.object_to_world, pt, w);
            for (int a = 0; a < 3; a++) {
                if (!std::isfinite(w[a])) continue;
                H.quad_lo[a] = std::fmin(H.quad_lo[a], w[a]);
                H.quad_hi[a] = std::fmax(H.quad_hi[a], w[a]);
            }
        }
    }
    H.scalars.n_quadrics = d->n_quadrics;
    return true;
}

bool flatten_scene(const rt_scene_desc* d, HostScene* out, std::string* err, bool build_bvh) {
    HostScene& H = *out;
    if (!d) {
        *err = "null scene descriptor";
        return false;
    }
    if (d->camera.width == 0 || d->camera.height == 0) {
        *err = "camera has zero width or height";
        return false;
    }
    if (d->n_meshes && !d->meshes) {
        *err = "meshes pointer is NULL";
        return false;
    }
    if (d->n_curves && !d->curves) {
        *err = "curves pointer is NULL";
        return false;
    }
    // ---- motion blur endpoints (mesh.rs:29-31, 230-235) -------------------------
    std::vector<const float*> pos1(d->n_meshes, nullptr);
    if (d->n_mesh_motion && !d->mesh_motion) {
        *err = "mesh_motion pointer is NULL";
        return false;
    }
    if (d->n_instance_motion && !d->instance_motion) {
        *err = "instance_motion pointer is NULL";
        return false;
    }
    for (uint32_t k = 0; k < d->n_mesh_motion; k++) {
        const rt_mesh_motion& mm = d->mesh_motion[k];
        if (mm.mesh >= d->n_meshes || !mm.positions1 || pos1[mm.mesh]) {
            *err = "mesh motion " + std::to_string(k) + " names a missing or repeated mesh, or has no positions";
            return false;
        }
        const rt_mesh_desc& md = d->meshes[mm.mesh];
        for (size_t v = 0; v < 3ull * md.n_vertices; v++)
            if (!std::isfinite(mm.positions1[v])) {
                *err = "mesh motion " + std::to_string(k) + " has a non-finite position";
                return false;
            }
        pos1[mm.mesh] = mm.positions1;
    }
    std::vector<const double*> xf1(d->n_instances, nullptr);
    for (uint32_t k = 0; k < d->n_instance_motion; k++) {
        const rt_instance_motion& im = d->instance_motion[k];
        if (im.instance >= d->n_instances || xf1[im.instance]) {
            *err = "instance motion " + std::to_string(k) + " names a missing or repeated instance";
            return false;
        }
        for (int j = 0; j < 12; j++)
            if (!std::isfinite(im.object_to_world1[j])) {
                *err = "instance motion " + std::to_string(k) + " has a non-finite transform";
                return false;
            }
        xf1[im.instance] = im.object_to_world1;
    }
    if (d->camera_motion_inv)
        for (int j = 0; j < 12; j++)
            if (!std::isfinite(d->camera_motion_inv[j])) {
                *err = "camera motion has a non-finite entry";
                return false;
            }
    const bool motion = d->n_mesh_motion || d->n_instance_motion || d->camera_motion_inv;
    if ((d->n_mesh_motion || d->n_instance_motion) && !build_bvh) {
        *err = "internal: scenes with moving geometry are built by the host BVH builder";
        return false;
    }
    // ---- BLAS per mesh, then per curve set (geometry n_meshes + k) ------------
    const uint32_t n_geom = d->n_meshes + d->n_curves;
    std::vector<std::vector<RootChild>> root_children(n_geom), grand_children(n_geom);
    H.meshes.resize(n_geom);
    uint64_t tri_total = 0;
    for (uint32_t m = 0; m < d->n_meshes; m++) tri_total += d->meshes[m].n_triangles;
    for (uint32_t k = 0; k < d->n_curves; k++) tri_total += d->curves[k].n_segments;
    if (tri_total >= (1ull << 27)) {
        *err = "more than 2^27 unique triangles";
        return false;
    }
    H.n_tris = tri_total;
    if (build_bvh) H.tris.reserve(3 * tri_total);
    if (d->n_curves && !build_bvh) {
        *err = "internal: curve sets are built by the host BVH builder";
        return false;
    }
    // A geometry's collapsed BLAS (its primitives already in `tris` in the
    // leaf order of `bin`), its root's children and second-level frontier.
    auto emit_blas = [&](uint32_t g, const BinBvh& bin) -> bool {
        MeshInfo& mi = H.meshes[g];
        Collapser col{bin, H.nodes, mi.tri_base};
        H.nodes.reserve(H.nodes.size() + WIDE_NODE_WORDS * (bin.nodes.size() / 4 + 1));
        mi.blas_root = col.emit(0);
        col.finish();
        H.blas_nodes += col.emitted;
        if (col.decode_errors) {
            *err = "internal: quantised BLAS boxes not conservative";
            return false;
        }
        // The root's children, and the second-level frontier (each inner
        // child replaced by its own children; the wide nodes were emitted in
        // preorder, one `wide` entry per node index).
        const auto& root = col.wide[0];
        for (uint32_t k = 0; k < root.nk; k++) {
            const BinNode& kn = bin.nodes[root.kids[k]];
            RootChild c;
            f32_box(kn.b, c.lo, c.hi);
            c.ref = root.refs[k];
            root_children[g].push_back(c);
            if (kn.count == 0) {
                const auto& cw = col.wide[root.refs[k] - root.idx];
                for (uint32_t kk = 0; kk < cw.nk; kk++) {
                    RootChild gc;
                    f32_box(bin.nodes[cw.kids[kk]].b, gc.lo, gc.hi);
                    gc.ref = cw.refs[kk];
                    grand_children[g].push_back(gc);
                }
            } else {
                grand_children[g].push_back(c);
            }
        }
        return true;
    };
    uint64_t tri_base = 0;
    for (uint32_t m = 0; m < d->n_meshes; m++) {
        const rt_mesh_desc& md = d->meshes[m];
        if (md.n_triangles && (!md.positions || !md.indices)) {
            *err = "mesh " + std::to_string(m) + " has NULL positions or indices";
            return false;
        }
        MeshInfo& mi = H.meshes[m];
        mi.n_tris = md.n_triangles;
        mi.tri_base = (uint32_t)tri_base;
        mi.blas_root = 0xFFFFFFFFu;
        mi.idx_base = 0xFFFFFFFFu;
        tri_base += md.n_triangles;
        mi.attrs = (md.normals ? MESH_NORMALS : 0u) | (md.st ? MESH_ST : 0u);
        if (mi.attrs) {
            // Vertex attributes (normals and/or st) share one vertex
            // numbering; a mesh without one of them stores zeros there.
            mi.idx_base = (uint32_t)H.orig_idx.size();
            uint32_t vbase = (uint32_t)(H.normals.size() / 3);
            const size_t o = H.orig_idx.size();
            H.orig_idx.resize(o + 3ull * md.n_triangles);
            uint32_t* oi = H.orig_idx.data() + o;
            parallel_for(3ull * md.n_triangles, [&](size_t k0, size_t k1) {
                for (size_t k = k0; k < k1; k++) oi[k] = vbase + md.indices[k];
            });
            if (md.normals) H.normals.insert(H.normals.end(), md.normals, md.normals + 3ull * md.n_vertices);
            else H.normals.resize(H.normals.size() + 3ull * md.n_vertices, 0.0f);
            if (md.st) {
                H.st.resize(2ull * vbase, 0.0f);
                H.st.insert(H.st.end(), md.st, md.st + 2ull * md.n_vertices);
            }
        }
        if (!build_bvh) continue;  // the device builder validates, bounds and builds
        std::vector<Box> tb(md.n_triangles);
        std::atomic<int> bad_index{0}, bad_vertex{0};
        parallel_for(md.n_triangles, [&](size_t t0, size_t t1) {
            for (size_t t = t0; t < t1; t++) {
                Box b;
                for (int k = 0; k < 3; k++) {
                    uint32_t vi = md.indices[3ull * t + k];
                    if (vi >= md.n_vertices) {
                        bad_index = 1;
                        continue;
                    }
                    double p[3] = {md.positions[3ull * vi], md.positions[3ull * vi + 1], md.positions[3ull * vi + 2]};
                    if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2])) {
                        bad_vertex = 1;
                        continue;
                    }
                    b.grow_pt(p);
                    if (pos1[m]) {  // mesh.rs:62-77: the box covers both endpoints
                        const double q[3] = {pos1[m][3ull * vi], pos1[m][3ull * vi + 1], pos1[m][3ull * vi + 2]};
                        b.grow_pt(q);
                    }
                }
                tb[t] = b;
            }
        });
        if (bad_index) {
            *err = "mesh " + std::to_string(m) + " index out of range";
            return false;
        }
        if (bad_vertex) {
            *err = "mesh " + std::to_string(m) + " has a non-finite vertex";
            return false;
        }
        BinBvh bin = build_binary(tb);
        H.binary_blas_nodes += bin.nodes.size();
        const size_t tri_off = H.tris.size();
        H.tris.resize(tri_off + 3ull * md.n_triangles);
        float4* dst = H.tris.data() + tri_off;
        const float* p1 = pos1[m];
        if (p1) H.tris1.resize(tri_off + 3ull * md.n_triangles);  // entries of static meshes stay unused
        float4* dst1 = p1 ? H.tris1.data() + tri_off : nullptr;
        parallel_for(md.n_triangles, [&](size_t k0, size_t k1) {
            for (size_t k = k0; k < k1; k++) {
                uint32_t t = bin.order[k];
                float4 v[3];
                for (int c = 0; c < 3; c++) {
                    uint32_t vi = md.indices[3ull * t + c];
                    v[c] = make_float4(md.positions[3ull * vi], md.positions[3ull * vi + 1],
                                       md.positions[3ull * vi + 2], 0.0f);
                    if (p1) dst1[3 * k + c] = make_float4(p1[3ull * vi], p1[3ull * vi + 1], p1[3ull * vi + 2], 0.0f);
                }
                uint32_t tid = t;
                memcpy(&v[0].w, &tid, 4);
                if (p1) {
                    const uint32_t mark = RT_DEFORM_MARK;
                    memcpy(&v[1].w, &mark, 4);
                }
                dst[3 * k] = v[0];
                dst[3 * k + 1] = v[1];
                dst[3 * k + 2] = v[2];
            }
        });
        if (md.n_triangles == 0) continue;
        if (!emit_blas(m, bin)) return false;
    }
    // Curve sets (curves.rs:29-62): BLASes over the boxes of each segment's
    // two end spheres; segments stored in the triangles' records.
    for (uint32_t k = 0; k < d->n_curves; k++) {
        const rt_curves_desc& cd = d->curves[k];
        const uint32_t g = d->n_meshes + k;
        if (cd.n_segments && (!cd.p0 || !cd.p1 || !cd.v0 || !cd.v1)) {
            *err = "curve set " + std::to_string(k) + " has NULL arrays";
            return false;
        }
        MeshInfo& mi = H.meshes[g];
        mi.n_tris = cd.n_segments;
        mi.tri_base = (uint32_t)tri_base;
        mi.blas_root = 0xFFFFFFFFu;
        mi.idx_base = 0xFFFFFFFFu;
        mi.attrs = MESH_CURVES;
        tri_base += cd.n_segments;
        std::vector<Box> sb(cd.n_segments);
        for (uint32_t t = 0; t < cd.n_segments; t++) {
            Box b;
            for (const float* e : {cd.p0 + 4ull * t, cd.p1 + 4ull * t}) {
                if (!std::isfinite(e[0] + e[1] + e[2] + e[3]) || e[3] < 0.0f) {
                    *err = "curve set " + std::to_string(k) + " has a non-finite point or a negative radius";
                    return false;
                }
                const double r = e[3];
                const double lo[3] = {(double)e[0] - r, (double)e[1] - r, (double)e[2] - r};
                const double hi[3] = {(double)e[0] + r, (double)e[1] + r, (double)e[2] + r};
                b.grow_pt(lo);
                b.grow_pt(hi);
            }
            sb[t] = b;
        }
        BinBvh bin = build_binary(sb);
        H.binary_blas_nodes += bin.nodes.size();
        for (uint32_t j = 0; j < cd.n_segments; j++) {
            const uint32_t t = bin.order[j];
            const float* a = cd.p0 + 4ull * t;
            const float* b = cd.p1 + 4ull * t;
            float4 r0 = make_float4(a[0], a[1], a[2], 0.0f), r1 = make_float4(b[0], b[1], b[2], a[3]);
            float4 r2 = make_float4(b[3], cd.v0[t], cd.v1[t], 0.0f);
            const uint32_t mark = RT_SEG_MARK;
            memcpy(&r0.w, &t, 4);
            memcpy(&r2.w, &mark, 4);
            H.tris.push_back(r0);
            H.tris.push_back(r1);
            H.tris.push_back(r2);
        }
        if (cd.n_segments && !emit_blas(g, bin)) return false;
    }
    if (!H.st.empty()) H.st.resize(2 * (H.normals.size() / 3), 0.0f);
    // ---- instances + TLAS ------------------------------------------------
    if (d->n_instances && !d->instances) {
        *err = "instances pointer is NULL";
        return false;
    }
    for (uint32_t i = 0; i < d->n_instances; i++) {
        const rt_instance_desc& id = d->instances[i];
        if (id.mesh_id >= n_geom || id.material_id >= d->n_materials) {
            *err = "instance " + std::to_string(i) + " references a missing mesh or material";
            return false;
        }
    }
    H.tlas_nodes = 0;
    H.scalars.tlas_root = 0xFFFFFFFFu;
    H.scalars.refill_at = RT_REFILL_SPARSE;
    if (build_bvh && d->n_instances) {
        std::vector<double> boxes;
        std::vector<uint2> items;
        tlas_items(d, root_children, grand_children, &boxes, &items, &H);
        if (items.size() >= (1ull << 27)) {
            *err = "more than 2^27 instance subtrees";
            return false;
        }
        instance_records(d, H, &H.inst_xf, &H.inst);
        if (!items.empty()) {
            std::vector<Box> ib(items.size());
            parallel_for(items.size(), [&](size_t i0, size_t i1) {
                for (size_t i = i0; i < i1; i++)
                    for (int a = 0; a < 3; a++) {
                        ib[i].lo[a] = boxes[6 * i + a];
                        ib[i].hi[a] = boxes[6 * i + 3 + a];
                    }
            });
            BinBvh tl = build_binary(ib);
            Collapser col{tl, H.nodes, 0};
            H.scalars.tlas_root = col.emit(0);
            col.finish();
            H.tlas_nodes = col.emitted;
            if (col.decode_errors) {
                *err = "internal: quantised TLAS boxes not conservative";
                return false;
            }
            H.items.resize(items.size());
            for (size_t k = 0; k < items.size(); k++) H.items[k] = items[tl.order[k]];
        }
    }
    H.scalars.n_instances = d->n_instances;
    H.scalars.any_curves = d->n_curves ? 1u : 0u;
    // ---- motion blur tables ---------------------------------------------------
    if (!H.tris1.empty()) H.tris1.resize(H.tris.size(), make_float4(0.0f, 0.0f, 0.0f, 0.0f));
    H.inst_motion.clear();
    H.inst_mot.clear();
    if (d->n_instance_motion) {
        H.inst_mot.assign(d->n_instances, 0xFFFFFFFFu);
        for (uint32_t i = 0; i < d->n_instances; i++) {
            if (!xf1[i]) continue;
            DevInstMotion im;
            for (int r = 0; r < 3; r++) {
                const double* a = d->instances[i].object_to_world + 4 * r;
                const double* b = xf1[i] + 4 * r;
                im.o2w0[r] = make_float4((float)a[0], (float)a[1], (float)a[2], (float)a[3]);
                im.o2w1[r] = make_float4((float)b[0], (float)b[1], (float)b[2], (float)b[3]);
            }
            H.inst_mot[i] = (uint32_t)H.inst_motion.size();
            H.inst_motion.push_back(im);
        }
    }
    H.scalars.motion = motion ? 1u : 0u;
    H.scalars.cam_moving = d->camera_motion_inv ? 1u : 0u;
    for (int k = 0; k < 12; k++)
        H.scalars.cam_mot[k] = d->camera_motion_inv ? (float)d->camera_motion_inv[k] : 0.0f;
    // ---- materials ---------------------------------------------------------
    if (d->n_materials && !d->materials) {
        *err = "materials pointer is NULL";
        return false;
    }
    // ---- participating media (medium.rs:28-66) ------------------------------
    // Indices are read only when the scene has media: an interior or
    // atmosphere of -1 means none, anything else must name a medium.
    if (d->n_media && !d->media) {
        *err = "media pointer is NULL";
        return false;
    }
    if (d->n_media > RT_MAX_MEDIA) {
        *err = "at most " + std::to_string(RT_MAX_MEDIA) + " media";
        return false;
    }
    H.scalars.n_media = d->n_media;
    H.scalars.atmosphere = 0xFFFFFFFFu;
    if (d->n_media) {
        if (d->atmosphere >= (int32_t)d->n_media || d->atmosphere < -1) {
            *err = "the atmosphere names a missing medium";
            return false;
        }
        if (d->atmosphere >= 0) H.scalars.atmosphere = (uint32_t)d->atmosphere;
    }
    for (uint32_t k = 0; k < d->n_media; k++) {
        const rt_medium_desc& md = d->media[k];
        DevMedium m{};
        double maj = 0.0;
        for (int c = 0; c < 3; c++) {
            if (!(md.sigma_a[c] >= 0.0) || !(md.sigma_s[c] >= 0.0) || !std::isfinite(md.sigma_a[c] + md.sigma_s[c])) {
                *err = "medium " + std::to_string(k) + " has a negative or non-finite coefficient";
                return false;
            }
            m.sigma_a[c] = (float)md.sigma_a[c];
            m.sigma_s[c] = (float)md.sigma_s[c];
            m.emission[c] = (float)md.emission[c];
            maj = std::max(maj, md.sigma_a[c] + md.sigma_s[c]);
        }
        if (md.density > RT_DENSITY_FBM || !(md.max_distance >= 0.0)) {
            *err = "medium " + std::to_string(k) + " has an unknown density or a negative extent";
            return false;
        }
        m.g = (float)md.g;
        m.max_distance = (float)std::min(md.max_distance, 3.0e38);
        m.majorant = (float)maj;
        m.frequency = (float)md.frequency;
        m.gain = (float)md.gain;
        m.lacunarity = (float)md.lacunarity;
        m.coverage = (float)md.coverage;
        m.sharpness = (float)md.sharpness;
        m.octaves = md.octaves;
        m.density = md.density;
        H.media.push_back(m);
    }
    H.scalars.any_presence = 0;
    H.scalars.any_sss = 0;
    for (uint32_t m = 0; m < d->n_materials; m++) {
        rt_material_desc md = d->materials[m];
        if (md.area_light >= (int32_t)d->n_lights) {
            *err = "material " + std::to_string(m) + " names a missing area light";
            return false;
        }
        if (!d->n_media) md.interior = -1;
        if (md.interior >= (int32_t)d->n_media || md.interior < -1) {
            *err = "material " + std::to_string(m) + " names a missing medium";
            return false;
        }
        H.materials.push_back(fold_material(md));
        if (md.hair) {
            H.materials.back().hair = (uint32_t)H.hair.size();
            H.hair.push_back(hair_dev(md));
        }
        if (H.materials.back().presence < 1.0f) H.scalars.any_presence = 1;
        if (H.materials.back().sss_gain > 0.0f) H.scalars.any_sss = 1;
    }
    if (!flatten_patterns(d, H, err)) return false;
    if (!flatten_quadrics(d, H, err)) return false;
    // ---- lights + light BVH --------------------------------------------------
    if (d->n_lights && !d->lights) {
        *err = "lights pointer is NULL";
        return false;
    }
    // Environment map of a dome light (envmap.rs:36-55): CDFs over the
    // sin-weighted luminance, accumulated in f64, stored in f32 as the
    // reference's GPU export does (envmap.rs:64-71).
    H.scalars.env_light = 0xFFFFFFFFu;
    H.scalars.env_w = H.scalars.env_h = 0;
    H.scalars.env_total = 0.0f;
    double env_mean_lum = 0.0;
    if (d->env_rgb) {
        if (!d->env_width || !d->env_height || d->env_light >= d->n_lights ||
            d->lights[d->env_light].type != RT_LIGHT_DOME) {
            *err = "environment map without a size or a dome light";
            return false;
        }
        const uint32_t w = d->env_width, h = d->env_height;
        H.env.resize((size_t)w * h);
        H.env_marg.assign(h + 1, 0.0f);
        H.env_cond.assign((size_t)(w + 1) * h, 0.0f);
        std::vector<double> marg(h + 1, 0.0);
        for (uint32_t y = 0; y < h; y++) {
            const double sin_t = std::sin(PI * (y + 0.5) / h);
            double acc = 0.0;
            for (uint32_t x = 0; x < w; x++) {
                const float* c = d->env_rgb + 3 * ((size_t)y * w + x);
                if (!std::isfinite(c[0]) || !std::isfinite(c[1]) || !std::isfinite(c[2])) {
                    *err = "environment map has a non-finite texel";
                    return false;
                }
                H.env[(size_t)y * w + x] = make_float4(c[0], c[1], c[2], 0.0f);
                acc += (0.2126 * c[0] + 0.7152 * c[1] + 0.0722 * c[2]) * sin_t;
                H.env_cond[(size_t)y * (w + 1) + x + 1] = (float)acc;
            }
            marg[y + 1] = marg[y] + acc;
            H.env_marg[y + 1] = (float)marg[y + 1];
        }
        const double total = std::max(marg[h], 1e-12);
        H.scalars.env_total = (float)total;
        H.scalars.env_w = w;
        H.scalars.env_h = h;
        H.scalars.env_light = d->env_light;
        env_mean_lum = total / std::max((double)w * h * (2.0 / PI), 1e-12);
    }
    std::vector<LEntry> finite;
    H.light_leaf.assign(d->n_lights, 0xFFFFFFFFu);
    H.scalars.dome = 0xFFFFFFFFu;
    double inf_total = 0;
    for (uint32_t l = 0; l < d->n_lights; l++) {
        const rt_light_desc& ld = d->lights[l];
        DevLight dl;
        memset(&dl, 0, sizeof(dl));
        dl.type = (uint32_t)ld.type;
        dl.ies = 0xFFFFFFFFu;
        double rad[3];
        for (int k = 0; k < 3; k++) {
            rad[k] = ld.color[k] * ld.intensity;
            dl.radiance[k] = (float)rad[k];
            dl.p[k] = (float)ld.p[k];
            dl.e1[k] = (float)ld.e1[k];
            dl.e2[k] = (float)ld.e2[k];
        }
        dl.radius = (float)ld.radius;
        double pw = std::fmax(lum(rad), 1e-9);
        double cx[3] = {ld.e1[1] * ld.e2[2] - ld.e1[2] * ld.e2[1], ld.e1[2] * ld.e2[0] - ld.e1[0] * ld.e2[2],
                        ld.e1[0] * ld.e2[1] - ld.e1[1] * ld.e2[0]};
        double cl = std::sqrt(cx[0] * cx[0] + cx[1] * cx[1] + cx[2] * cx[2]);
        double l1 = std::sqrt(ld.e1[0] * ld.e1[0] + ld.e1[1] * ld.e1[1] + ld.e1[2] * ld.e1[2]);
        double l2 = std::sqrt(ld.e2[0] * ld.e2[0] + ld.e2[1] * ld.e2[1] + ld.e2[2] * ld.e2[2]);
        LEntry en{l, {ld.p[0], ld.p[1], ld.p[2]}, 0.0, 0.0};
        switch (ld.type) {
            case RT_LIGHT_POINT: en.power = pw * 4.0 * PI; finite.push_back(en); break;
            case RT_LIGHT_RECT:
                dl.area = (float)cl;
                for (int k = 0; k < 3; k++) {
                    dl.n[k] = (float)(cl > 1e-6 ? cx[k] / cl : cx[k]);
                    en.c[k] = ld.p[k] + ld.e1[k] * 0.5 + ld.e2[k] * 0.5;
                }
                en.radius = (l1 + l2) * 0.5;
                en.power = pw * cl * PI;
                finite.push_back(en);
                break;
            case RT_LIGHT_SPHERE:
                en.radius = ld.radius;
                en.power = pw * 4.0 * PI * ld.radius * ld.radius * PI;
                finite.push_back(en);
                break;
            case RT_LIGHT_DISK: {
                double area = PI * l1 * l2;
                dl.area = (float)area;
                for (int k = 0; k < 3; k++) dl.n[k] = (float)(cl > 1e-6 ? cx[k] / cl : cx[k]);
                en.radius = l1;
                en.power = pw * area * PI;
                finite.push_back(en);
                break;
            }
            case RT_LIGHT_DOME: {  // light_sampler.rs:104-118: infinite group
                if (H.scalars.dome == 0xFFFFFFFFu) H.scalars.dome = l;
                // power: lum(radiance) * 4 pi, or with a map its mean luminance * intensity * 4 pi
                const double base = l == H.scalars.env_light ? env_mean_lum * ld.intensity : pw;
                H.inf_lights.push_back(l);
                H.inf_power.push_back((float)(base * 4.0 * PI));
                inf_total += base * 4.0 * PI;
                break;
            }
            case RT_LIGHT_DISTANT: {
                double dn = l1 > 1e-6 ? l1 : 1.0;
                for (int k = 0; k < 3; k++) dl.e1[k] = (float)(ld.e1[k] / dn);
                dl.cos_max = (float)std::cos(ld.radius);
                H.inf_lights.push_back(l);
                H.inf_power.push_back((float)(pw * 4.0 * PI));
                inf_total += pw * 4.0 * PI;
                break;
            }
            default: *err = "light " + std::to_string(l) + " has an unknown type"; return false;
        }
        H.lights.push_back(dl);
    }
    // IES profiles of point lights (ies.rs): f32 angles and candela, the
    // sin-weighted mean candela in f64 as ies.rs:67-80 takes it.
    if (d->n_ies && !d->ies) {
        *err = "ies pointer is NULL";
        return false;
    }
    for (uint32_t k = 0; k < d->n_ies; k++) {
        const rt_ies_desc& e = d->ies[k];
        if (e.light >= d->n_lights || d->lights[e.light].type != RT_LIGHT_POINT || !e.n_v || !e.n_h ||
            e.n_v > 4096 || e.n_h > 4096 || !e.v_angles || !e.h_angles || !e.candela) {
            *err = "IES profile " + std::to_string(k) + " is empty or not on a point light";
            return false;
        }
        if (H.lights[e.light].ies != 0xFFFFFFFFu) {
            *err = "light " + std::to_string(e.light) + " has two IES profiles";
            return false;
        }
        DevIes g;
        memset(&g, 0, sizeof(g));
        g.off = (uint32_t)H.ies_data.size();
        g.n_v = e.n_v;
        g.n_h = e.n_h;
        double num = 0.0, den = 0.0;
        for (uint32_t vi = 0; vi < e.n_v; vi++) {
            double w = std::fmax(std::sin(e.v_angles[vi] * PI / 180.0), 1e-4), mean = 0.0;
            for (uint32_t hi = 0; hi < e.n_h; hi++) mean += e.candela[(size_t)hi * e.n_v + vi];
            num += mean / (double)e.n_h * w;
            den += w;
        }
        g.average = (float)std::fmax(num / std::fmax(den, 1e-9), 1e-9);
        for (int j = 0; j < 9; j++) g.m[j] = (float)e.world_to_local[j];
        for (uint32_t vi = 0; vi < e.n_v; vi++) H.ies_data.push_back((float)e.v_angles[vi]);
        for (uint32_t hi = 0; hi < e.n_h; hi++) H.ies_data.push_back((float)e.h_angles[hi]);
        for (size_t c = 0; c < (size_t)e.n_v * e.n_h; c++) H.ies_data.push_back((float)e.candela[c]);
        H.lights[e.light].ies = (uint32_t)H.ies.size();
        H.ies.push_back(g);
    }
    double finite_total = 0;
    for (auto& e : finite) finite_total += e.power;
    if (!finite.empty()) {
        std::vector<size_t> order(finite.size());
        for (size_t k = 0; k < order.size(); k++) order[k] = k;
        lbvh_build(H.lbvh, H.light_leaf, finite, order, 0, finite.size(), 0xFFFFFFFFu);
    }
    H.scalars.n_lights = d->n_lights;
    H.scalars.n_lbvh = (uint32_t)H.lbvh.size();
    H.scalars.n_inf = (uint32_t)H.inf_lights.size();
    H.scalars.inf_total = (float)inf_total;
    H.scalars.p_infinite = H.inf_lights.empty() ? 0.0f
                           : finite.empty()     ? 1.0f
                                                : (float)std::min(std::max(inf_total / (inf_total + finite_total), 0.1), 0.9);
    // ---- camera (camera.rs:150-179) ------------------------------------------
    const rt_camera_desc& c = d->camera;
    for (int k = 0; k < 3; k++) {
        H.scalars.eye[k] = (float)c.eye[k];
        H.scalars.fwd[k] = (float)c.forward[k];
        H.scalars.right[k] = (float)c.right[k];
        H.scalars.up[k] = (float)c.up[k];
        H.scalars.background[k] = (float)d->background[k];
    }
    double half_h = std::tan(c.fov_deg * PI / 180.0 / 2.0);
    H.scalars.half_h = (float)half_h;
    H.scalars.half_w = (float)((double)c.width / (double)c.height * half_h);
    H.scalars.lens_radius = (float)c.lens_radius;
    H.scalars.focal_distance = (float)c.focal_distance;
    H.scalars.filter = (uint32_t)c.filter;
    H.scalars.filter_width = (float)c.filter_width;
    if (c.projection != RT_PROJECTION_PERSPECTIVE && c.projection != RT_PROJECTION_ORTHOGRAPHIC) {
        *err = "unknown camera projection";
        return false;
    }
    H.scalars.projection = (uint32_t)c.projection;
    H.scalars.ortho_hw = (float)c.ortho_half[0];
    H.scalars.ortho_hh = (float)c.ortho_half[1];
    H.scalars.width = c.width;
    H.scalars.height = c.height;
    return true;
}

}  // namespace rt

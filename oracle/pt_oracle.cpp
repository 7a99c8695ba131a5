// pt_oracle.cpp — f64 CPU oracle for the render.rs path tracer.
//
// TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
// bench's cpu_baseline leg as the checker and the timed CPU baseline. The
// CUDA backend never calls it.
//
// Every function cites the reference source (path:line within
// anders94/render.rs) whose behaviour it restates. Arithmetic is f64 as in
// the reference; the choices that decide tree shape or random-number use
// (partition order, stable sort, bin index, draw order) follow it exactly.

#include "pt_oracle.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <thread>
#include <vector>

namespace orc {

static const double PI = 3.14159265358979323846;
static const double INF = std::numeric_limits<double>::infinity();
static const double EPSILON = 1e-6;          // src/math/mod.rs:9
static const double RAY_OFFSET = 1e-4;       // src/raytracer/pt/mod.rs:30
static const int MAX_PRESENCE_SKIPS = 16;    // src/raytracer/pt/mod.rs:32

// ---- math (src/math/vector.rs, point.rs, matrix.rs) ----------------------

struct V3 {
    double x = 0, y = 0, z = 0;
    V3() = default;
    V3(double a, double b, double c) : x(a), y(b), z(c) {}
};
static inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
static inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
static inline V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
static inline V3 operator/(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
static inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
static inline double length_sq(V3 a) { return dot(a, a); }
static inline double length(V3 a) { return std::sqrt(length_sq(a)); }
// vector.rs:31-38 — normalise only when the length exceeds EPSILON.
static inline V3 normalize(V3 a) {
    double l = length(a);
    return l > EPSILON ? a / l : a;
}
// vector.rs:52-54
static inline V3 reflect(V3 v, V3 n) { return v - n * 2.0 * dot(v, n); }
static inline double max_comp(V3 c) { return std::fmax(std::fmax(c.x, c.y), c.z); }
static inline double lum(V3 c) { return 0.2126 * c.x + 0.7152 * c.y + 0.0722 * c.z; }
static inline double axis_of(V3 v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }
static inline V3 v3(const double* p) { return {p[0], p[1], p[2]}; }

struct M4 {
    double m[4][4];
};
static M4 identity() {
    M4 r{};
    for (int i = 0; i < 4; i++) r.m[i][i] = 1.0;
    return r;
}
// matrix.rs:228-240 component-wise interpolation toward b.
static M4 lerp(const M4& a, const M4& b, double t) {
    M4 r;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) r.m[i][j] = a.m[i][j] + (b.m[i][j] - a.m[i][j]) * t;
    return r;
}
// matrix.rs: inverse via cofactors; None when |det| < EPSILON.
static bool inverse(const M4& a, M4& out) {
    const double(*m)[4] = a.m;
    double inv[4][4];
    inv[0][0] = m[1][1] * m[2][2] * m[3][3] - m[1][1] * m[2][3] * m[3][2] - m[2][1] * m[1][2] * m[3][3] +
                m[2][1] * m[1][3] * m[3][2] + m[3][1] * m[1][2] * m[2][3] - m[3][1] * m[1][3] * m[2][2];
    inv[1][0] = -m[1][0] * m[2][2] * m[3][3] + m[1][0] * m[2][3] * m[3][2] + m[2][0] * m[1][2] * m[3][3] -
                m[2][0] * m[1][3] * m[3][2] - m[3][0] * m[1][2] * m[2][3] + m[3][0] * m[1][3] * m[2][2];
    inv[2][0] = m[1][0] * m[2][1] * m[3][3] - m[1][0] * m[2][3] * m[3][1] - m[2][0] * m[1][1] * m[3][3] +
                m[2][0] * m[1][3] * m[3][1] + m[3][0] * m[1][1] * m[2][3] - m[3][0] * m[1][3] * m[2][1];
    inv[3][0] = -m[1][0] * m[2][1] * m[3][2] + m[1][0] * m[2][2] * m[3][1] + m[2][0] * m[1][1] * m[3][2] -
                m[2][0] * m[1][2] * m[3][1] - m[3][0] * m[1][1] * m[2][2] + m[3][0] * m[1][2] * m[2][1];
    double det = m[0][0] * inv[0][0] + m[0][1] * inv[1][0] + m[0][2] * inv[2][0] + m[0][3] * inv[3][0];
    if (std::fabs(det) < EPSILON) return false;
    inv[0][1] = -m[0][1] * m[2][2] * m[3][3] + m[0][1] * m[2][3] * m[3][2] + m[2][1] * m[0][2] * m[3][3] -
                m[2][1] * m[0][3] * m[3][2] - m[3][1] * m[0][2] * m[2][3] + m[3][1] * m[0][3] * m[2][2];
    inv[1][1] = m[0][0] * m[2][2] * m[3][3] - m[0][0] * m[2][3] * m[3][2] - m[2][0] * m[0][2] * m[3][3] +
                m[2][0] * m[0][3] * m[3][2] + m[3][0] * m[0][2] * m[2][3] - m[3][0] * m[0][3] * m[2][2];
    inv[2][1] = -m[0][0] * m[2][1] * m[3][3] + m[0][0] * m[2][3] * m[3][1] + m[2][0] * m[0][1] * m[3][3] -
                m[2][0] * m[0][3] * m[3][1] - m[3][0] * m[0][1] * m[2][3] + m[3][0] * m[0][3] * m[2][1];
    inv[3][1] = m[0][0] * m[2][1] * m[3][2] - m[0][0] * m[2][2] * m[3][1] - m[2][0] * m[0][1] * m[3][2] +
                m[2][0] * m[0][2] * m[3][1] + m[3][0] * m[0][1] * m[2][2] - m[3][0] * m[0][2] * m[2][1];
    inv[0][2] = m[0][1] * m[1][2] * m[3][3] - m[0][1] * m[1][3] * m[3][2] - m[1][1] * m[0][2] * m[3][3] +
                m[1][1] * m[0][3] * m[3][2] + m[3][1] * m[0][2] * m[1][3] - m[3][1] * m[0][3] * m[1][2];
    inv[1][2] = -m[0][0] * m[1][2] * m[3][3] + m[0][0] * m[1][3] * m[3][2] + m[1][0] * m[0][2] * m[3][3] -
                m[1][0] * m[0][3] * m[3][2] - m[3][0] * m[0][2] * m[1][3] + m[3][0] * m[0][3] * m[1][2];
    inv[2][2] = m[0][0] * m[1][1] * m[3][3] - m[0][0] * m[1][3] * m[3][1] - m[1][0] * m[0][1] * m[3][3] +
                m[1][0] * m[0][3] * m[3][1] + m[3][0] * m[0][1] * m[1][3] - m[3][0] * m[0][3] * m[1][1];
    inv[3][2] = -m[0][0] * m[1][1] * m[3][2] + m[0][0] * m[1][2] * m[3][1] + m[1][0] * m[0][1] * m[3][2] -
                m[1][0] * m[0][2] * m[3][1] - m[3][0] * m[0][1] * m[1][2] + m[3][0] * m[0][2] * m[1][1];
    inv[0][3] = -m[0][1] * m[1][2] * m[2][3] + m[0][1] * m[1][3] * m[2][2] + m[1][1] * m[0][2] * m[2][3] -
                m[1][1] * m[0][3] * m[2][2] - m[2][1] * m[0][2] * m[1][3] + m[2][1] * m[0][3] * m[1][2];
    inv[1][3] = m[0][0] * m[1][2] * m[2][3] - m[0][0] * m[1][3] * m[2][2] - m[1][0] * m[0][2] * m[2][3] +
                m[1][0] * m[0][3] * m[2][2] + m[2][0] * m[0][2] * m[1][3] - m[2][0] * m[0][3] * m[1][2];
    inv[2][3] = -m[0][0] * m[1][1] * m[2][3] + m[0][0] * m[1][3] * m[2][1] + m[1][0] * m[0][1] * m[2][3] -
                m[1][0] * m[0][3] * m[2][1] - m[2][0] * m[0][1] * m[1][3] + m[2][0] * m[0][3] * m[1][1];
    inv[3][3] = m[0][0] * m[1][1] * m[2][2] - m[0][0] * m[1][2] * m[2][1] - m[1][0] * m[0][1] * m[2][2] +
                m[1][0] * m[0][2] * m[2][1] + m[2][0] * m[0][1] * m[1][2] - m[2][0] * m[0][2] * m[1][1];
    double det_inv = 1.0 / det;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) out.m[i][j] = inv[i][j] * det_inv;
    return true;
}
// matrix.rs transform_point: divides by w only when w differs from 1.
static V3 xf_point(const M4& a, V3 p) {
    const double(*m)[4] = a.m;
    double x = m[0][0] * p.x + m[0][1] * p.y + m[0][2] * p.z + m[0][3];
    double y = m[1][0] * p.x + m[1][1] * p.y + m[1][2] * p.z + m[1][3];
    double z = m[2][0] * p.x + m[2][1] * p.y + m[2][2] * p.z + m[2][3];
    double w = m[3][0] * p.x + m[3][1] * p.y + m[3][2] * p.z + m[3][3];
    if (std::fabs(w - 1.0) < EPSILON) return {x, y, z};
    return {x / w, y / w, z / w};
}
static V3 xf_vec(const M4& a, V3 v) {
    const double(*m)[4] = a.m;
    return {m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z, m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z,
            m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z};
}
// transform_normal: multiplies by the transpose (callers pass the inverse).
static V3 xf_normal(const M4& a, V3 n) {
    const double(*m)[4] = a.m;
    return {m[0][0] * n.x + m[1][0] * n.y + m[2][0] * n.z, m[0][1] * n.x + m[1][1] * n.y + m[2][1] * n.z,
            m[0][2] * n.x + m[1][2] * n.y + m[2][2] * n.z};
}

// ---- sampler (src/raytracer/pt/sampler.rs:6-60) ---------------------------

struct Pcg32 {
    uint64_t state, inc;
    Pcg32(uint64_t seed, uint64_t stream) : state(0), inc((stream << 1) | 1u) {  // :12-21
        next_u32();
        state += seed;
        next_u32();
    }
    static uint64_t mix(uint64_t z) {  // :26-30
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return z ^ (z >> 31);
    }
    static Pcg32 for_pixel_sample(uint64_t pixel, uint64_t sample) {  // :24-32
        return Pcg32(mix((pixel * 0x9e3779b97f4a7c15ull) ^ sample), mix(sample) | 1u);
    }
    uint32_t next_u32() {  // :34-42
        uint64_t old = state;
        state = old * 6364136223846793005ull + inc;
        uint32_t xorshifted = (uint32_t)(((old >> 18) ^ old) >> 27);
        uint32_t rot = (uint32_t)(old >> 59);
        return (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
    }
    double next_f64() { return (double)next_u32() * (1.0 / 4294967296.0); }  // :45-47
};

// ---- BVH (src/accel/bvh.rs) -----------------------------------------------

struct Aabb {
    V3 mn{INF, INF, INF}, mx{-INF, -INF, -INF};
    // Rust f64::min/max ignore a NaN operand, as fmin/fmax do.
    void grow_point(V3 p) {
        mn = {std::fmin(mn.x, p.x), std::fmin(mn.y, p.y), std::fmin(mn.z, p.z)};
        mx = {std::fmax(mx.x, p.x), std::fmax(mx.y, p.y), std::fmax(mx.z, p.z)};
    }
    void grow(const Aabb& o) {
        grow_point(o.mn);
        grow_point(o.mx);
    }
    V3 centroid() const { return (mn + mx) * 0.5; }
    double surface_area() const {  // bvh.rs:45-51
        V3 d = mx - mn;
        if (d.x < 0.0 || d.y < 0.0 || d.z < 0.0) return 0.0;
        return 2.0 * (d.x * d.y + d.y * d.z + d.z * d.x);
    }
    // bvh.rs:55-72 slab test.
    bool hit(V3 o, V3 inv, double t_max, double* t_entry) const {
        double t0x = (mn.x - o.x) * inv.x, t1x = (mx.x - o.x) * inv.x;
        double t_near = std::fmin(t0x, t1x), t_far = std::fmax(t0x, t1x);
        double t0y = (mn.y - o.y) * inv.y, t1y = (mx.y - o.y) * inv.y;
        t_near = std::fmax(t_near, std::fmin(t0y, t1y));
        t_far = std::fmin(t_far, std::fmax(t0y, t1y));
        double t0z = (mn.z - o.z) * inv.z, t1z = (mx.z - o.z) * inv.z;
        t_near = std::fmax(t_near, std::fmin(t0z, t1z));
        t_far = std::fmin(t_far, std::fmax(t0z, t1z));
        if (t_near <= t_far && t_far > 0.0 && t_near < t_max) {
            if (t_entry) *t_entry = std::fmax(t_near, 0.0);
            return true;
        }
        return false;
    }
};

// `time`: the shutter time in [0, 1) the ray samples (0 in static scenes);
// every ray of a path carries the camera ray's (`Ray::with_time`).
struct Ray {
    V3 o, d;
    double time = 0.0;
};
// raytracer/ray.rs:13-19 — Ray::new normalises the direction.
static inline Ray make_ray(V3 o, V3 d, double time = 0.0) { return {o, normalize(d), time}; }

struct Counters {
    uint64_t pops = 0, tris = 0, insts = 0;
};

struct Bvh {
    struct Node {
        Aabb bounds;
        uint32_t first = 0, count = 0;
    };
    std::vector<Node> nodes;
    std::vector<uint32_t> prim_order;
    static const int BINS = 16;     // bvh.rs:91
    static const int MAX_LEAF = 4;  // bvh.rs:92

    // bvh.rs:96-108
    void build(const std::vector<Aabb>& bounds) {
        prim_order.resize(bounds.size());
        for (size_t i = 0; i < bounds.size(); i++) prim_order[i] = (uint32_t)i;
        nodes.clear();
        if (bounds.empty()) return;
        nodes.reserve(bounds.size() * 2);
        std::vector<V3> centroids(bounds.size());
        for (size_t i = 0; i < bounds.size(); i++) centroids[i] = bounds[i].centroid();
        nodes.push_back(Node{});
        // Explicit stack keeps the reference's recursion order (left subtree
        // fully before right) without deep native recursion.
        struct Job { size_t node, start, count; };
        std::vector<Job> stack{{0, 0, bounds.size()}};
        while (!stack.empty()) {
            Job j = stack.back();
            stack.pop_back();
            size_t split_at;
            if (!subdivide(bounds, centroids, j.node, j.start, j.count, &split_at)) continue;
            size_t left = nodes.size();
            nodes.push_back(Node{});
            nodes.push_back(Node{});
            nodes[j.node].first = (uint32_t)left;
            nodes[j.node].count = 0;
            // Children are appended in pre-order: the left subtree's nodes
            // must all be created before the right child's descendants.
            stack.push_back({left + 1, split_at, j.start + j.count - split_at});
            stack.push_back({left, j.start, split_at - j.start});
        }
    }

    // bvh.rs:256-345 (one level). Returns false when the node became a leaf.
    bool subdivide(const std::vector<Aabb>& bounds, const std::vector<V3>& centroids, size_t node_idx,
                   size_t start, size_t count, size_t* split_out) {
        Aabb b, cb;
        for (size_t i = start; i < start + count; i++) {
            uint32_t p = prim_order[i];
            b.grow(bounds[p]);
            cb.grow_point(centroids[p]);
        }
        nodes[node_idx].bounds = b;
        if (count <= (size_t)MAX_LEAF) {
            nodes[node_idx].first = (uint32_t)start;
            nodes[node_idx].count = (uint32_t)count;
            return false;
        }
        V3 ext = cb.mx - cb.mn;
        int axis = (ext.x >= ext.y && ext.x >= ext.z) ? 0 : (ext.y >= ext.z ? 1 : 2);
        double axis_min = axis_of(cb.mn, axis), axis_extent = axis_of(ext, axis);
        size_t split_at = start + count / 2;  // median fallback
        if (axis_extent > 1e-12) {
            Aabb bin_bounds[BINS];
            size_t bin_counts[BINS] = {0};
            double scale = (double)BINS / axis_extent;
            for (size_t i = start; i < start + count; i++) {
                uint32_t p = prim_order[i];
                double f = (axis_of(centroids[p], axis) - axis_min) * scale;
                size_t bi = f > 0.0 ? (size_t)f : 0;  // Rust `as usize` saturates at 0
                if (bi > (size_t)BINS - 1) bi = BINS - 1;
                bin_counts[bi]++;
                bin_bounds[bi].grow(bounds[p]);
            }
            Aabb right_acc[BINS], acc;
            for (int i = BINS - 1; i >= 1; i--) {
                acc.grow(bin_bounds[i]);
                right_acc[i] = acc;
            }
            double best_cost = INF;
            int best_bin = 0;
            Aabb left;
            size_t left_count = 0;
            for (int i = 0; i < BINS - 1; i++) {
                left.grow(bin_bounds[i]);
                left_count += bin_counts[i];
                size_t right_count = count - left_count;
                if (left_count == 0 || right_count == 0) continue;
                double cost = left.surface_area() * (double)left_count +
                              right_acc[i + 1].surface_area() * (double)right_count;
                if (cost < best_cost) {
                    best_cost = cost;
                    best_bin = i;
                }
            }
            double leaf_cost = b.surface_area() * (double)count;
            if (std::isfinite(best_cost) && best_cost < leaf_cost) {
                double boundary = axis_min + axis_extent * (double)(best_bin + 1) / (double)BINS;
                // bvh.rs:362-371 in-place swap partition.
                size_t i = 0;
                for (size_t j = 0; j < count; j++) {
                    if (axis_of(centroids[prim_order[start + j]], axis) < boundary) {
                        std::swap(prim_order[start + i], prim_order[start + j]);
                        i++;
                    }
                }
                if (i > 0 && i < count) split_at = start + i;
            } else if (count <= (size_t)MAX_LEAF * 4) {
                nodes[node_idx].first = (uint32_t)start;
                nodes[node_idx].count = (uint32_t)count;
                return false;
            }
        }
        *split_out = split_at;
        return true;
    }

    // bvh.rs:141-204. `isect(prim, t_max, &t)` must report hits < t_max.
    template <class F>
    bool traverse(V3 o, V3 d, double t_max, F&& isect, uint32_t* best_prim, double* best_t,
                  Counters* c) const {
        if (nodes.empty()) return false;
        V3 inv{1.0 / d.x, 1.0 / d.y, 1.0 / d.z};
        bool found = false;
        uint32_t stack[64];
        int sp = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            const Node& node = nodes[stack[--sp]];
            if (c) c->pops++;
            if (!node.bounds.hit(o, inv, t_max, nullptr)) continue;
            if (node.count > 0) {
                for (uint32_t i = node.first; i < node.first + node.count; i++) {
                    uint32_t prim = prim_order[i];
                    double t;
                    if (isect(prim, t_max, &t) && t < t_max) {
                        t_max = t;
                        *best_prim = prim;
                        *best_t = t;
                        found = true;
                    }
                }
            } else {
                uint32_t l = node.first, r = l + 1;
                double a, b;
                bool hl = nodes[l].bounds.hit(o, inv, t_max, &a);
                bool hr = nodes[r].bounds.hit(o, inv, t_max, &b);
                if (hl && hr) {
                    uint32_t nr = a <= b ? l : r, fr = a <= b ? r : l;
                    stack[sp++] = fr;
                    stack[sp++] = nr;
                } else if (hl) {
                    stack[sp++] = l;
                } else if (hr) {
                    stack[sp++] = r;
                }
            }
        }
        return found;
    }

    // bvh.rs:208-245
    template <class F>
    bool any_hit(V3 o, V3 d, double t_limit, F&& hitp, Counters* c) const {
        if (nodes.empty()) return false;
        V3 inv{1.0 / d.x, 1.0 / d.y, 1.0 / d.z};
        uint32_t stack[64];
        int sp = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            const Node& node = nodes[stack[--sp]];
            if (c) c->pops++;
            if (!node.bounds.hit(o, inv, t_limit, nullptr)) continue;
            if (node.count > 0) {
                for (uint32_t i = node.first; i < node.first + node.count; i++)
                    if (hitp(prim_order[i], t_limit)) return true;
            } else {
                stack[sp++] = node.first;
                stack[sp++] = node.first + 1;
            }
        }
        return false;
    }
};

// ---- meshes and instances (src/geometry/mesh.rs) --------------------------

struct Mesh {
    std::vector<float> pos;
    std::vector<uint32_t> idx;
    std::vector<float> nrm;  // empty when absent
    std::vector<float> st;   // 2 per vertex; empty when absent
    std::vector<float> pos1; // positions at shutter close (deformation blur); empty when static
    Bvh blas;
    Aabb local_bounds;

    V3 vertex(uint32_t i) const { return {(double)pos[3 * i], (double)pos[3 * i + 1], (double)pos[3 * i + 2]}; }
    // mesh.rs:96-111 vertex at shutter time (lerped toward the endpoint).
    V3 vertex_at(uint32_t i, double time) const {
        if (pos1.empty() || !(time > 0.0)) return vertex(i);
        V3 a = vertex(i), b{(double)pos1[3 * i], (double)pos1[3 * i + 1], (double)pos1[3 * i + 2]};
        return {a.x + (b.x - a.x) * time, a.y + (b.y - a.y) * time, a.z + (b.z - a.z) * time};
    }

    void build() {  // mesh.rs:45-86: triangle boxes cover both endpoints when deforming
        size_t n = idx.size() / 3;
        std::vector<Aabb> bounds(n);
        for (size_t t = 0; t < n; t++) {
            Aabb b;
            b.grow_point(vertex(idx[3 * t]));
            b.grow_point(vertex(idx[3 * t + 1]));
            b.grow_point(vertex(idx[3 * t + 2]));
            if (!pos1.empty())
                for (int k = 0; k < 3; k++) b.grow_point(vertex_at(idx[3 * t + k], 1.0));
            bounds[t] = b;
            local_bounds.grow(b);
        }
        blas.build(bounds);
    }

    // mesh.rs:117-142 Möller–Trumbore (parametric t along the local ray),
    // against the triangle at the ray's shutter time.
    bool intersect_triangle(const Ray& r, uint32_t tri, double t_max, double* t_out, double* u_out,
                            double* v_out) const {
        V3 v0 = vertex_at(idx[3 * tri], r.time);
        V3 e1 = vertex_at(idx[3 * tri + 1], r.time) - v0;
        V3 e2 = vertex_at(idx[3 * tri + 2], r.time) - v0;
        V3 p = cross(r.d, e2);
        double det = dot(e1, p);
        if (std::fabs(det) < 1e-14) return false;
        double inv = 1.0 / det;
        V3 tv = r.o - v0;
        double u = dot(tv, p) * inv;
        if (!(u >= 0.0 && u <= 1.0)) return false;
        V3 q = cross(tv, e1);
        double v = dot(r.d, q) * inv;
        if (v < 0.0 || u + v > 1.0) return false;
        double t = dot(e2, q) * inv;
        if (!(t > 1e-9 && t < t_max)) return false;
        *t_out = t;
        *u_out = u;
        *v_out = v;
        return true;
    }

    // mesh.rs:200-220 interpolated or geometric local normal; a deforming
    // mesh takes the geometric normal at the shutter time (vertex normals
    // are authored for the rest pose).
    V3 local_normal(uint32_t tri, double u, double v, double time = 0.0) const {
        uint32_t i0 = idx[3 * tri], i1 = idx[3 * tri + 1], i2 = idx[3 * tri + 2];
        if (!nrm.empty() && pos1.empty()) {
            auto n = [&](uint32_t i) { return V3{nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]}; };
            double w = 1.0 - u - v;
            return normalize(n(i0) * w + n(i1) * u + n(i2) * v);
        }
        V3 v0 = vertex_at(i0, time);
        return normalize(cross(vertex_at(i1, time) - v0, vertex_at(i2, time) - v0));
    }

    // mesh.rs:147-173 local gradients of s and t within the triangle's
    // plane (dual basis of its edges); false without st or when degenerate.
    bool st_gradients(uint32_t tri, V3* gs, V3* gt) const {
        if (st.empty()) return false;
        uint32_t i0 = idx[3 * tri], i1 = idx[3 * tri + 1], i2 = idx[3 * tri + 2];
        V3 p0 = vertex(i0);
        V3 e1 = vertex(i1) - p0, e2 = vertex(i2) - p0;
        double ds1 = (double)(st[2 * i1] - st[2 * i0]), dt1 = (double)(st[2 * i1 + 1] - st[2 * i0 + 1]);
        double ds2 = (double)(st[2 * i2] - st[2 * i0]), dt2 = (double)(st[2 * i2 + 1] - st[2 * i0 + 1]);
        V3 n = cross(e1, e2);
        double n2 = length_sq(n);
        if (n2 < 1e-24) return false;
        V3 dual1 = cross(e2, n) / n2, dual2 = cross(e1, n) / -n2;
        *gs = dual1 * ds1 + dual2 * ds2;
        *gt = dual1 * dt1 + dual2 * dt2;
        return true;
    }

    // mesh.rs:177-197 interpolated st and st density (sqrt of st area over
    // local geometric area); false without st.
    bool st_at(uint32_t tri, double u, double v, double st_out[2], double* density) const {
        if (st.empty()) return false;
        uint32_t i0 = idx[3 * tri], i1 = idx[3 * tri + 1], i2 = idx[3 * tri + 2];
        const float *s0 = &st[2 * i0], *s1 = &st[2 * i1], *s2 = &st[2 * i2];
        double w = 1.0 - u - v;
        st_out[0] = (double)s0[0] * w + (double)s1[0] * u + (double)s2[0] * v;
        st_out[1] = (double)s0[1] * w + (double)s1[1] * u + (double)s2[1] * v;
        double st_area = 0.5 * std::fabs((double)(s1[0] - s0[0]) * (double)(s2[1] - s0[1]) -
                                         (double)(s2[0] - s0[0]) * (double)(s1[1] - s0[1]));
        V3 v0 = vertex(i0);
        double geo_area = 0.5 * length(cross(vertex(i1) - v0, vertex(i2) - v0));
        *density = geo_area > 1e-18 ? std::sqrt(st_area / geo_area) : 0.0;
        return true;
    }
};

// ---- curve sets (src/geometry/curves.rs) ------------------------------------
// Rounded-cone segments: a sphere swept from p0 to p1 with its radius going
// linearly from r0 to r1 (curves.rs:15-26).
struct CurveSet {
    std::vector<float> p0, p1;  // xyz + radius per segment
    std::vector<float> v0, v1;  // curve parameter at each end
    Bvh blas;
    Aabb local_bounds;

    size_t segments() const { return v0.size(); }
    void build() {  // curves.rs:29-62: boxes of the two end spheres
        std::vector<Aabb> bounds(segments());
        for (size_t k = 0; k < segments(); k++) {
            Aabb b;
            for (const float* e : {&p0[4 * k], &p1[4 * k]}) {
                const double r = e[3];
                b.grow_point(V3{(double)e[0] - r, (double)e[1] - r, (double)e[2] - r});
                b.grow_point(V3{(double)e[0] + r, (double)e[1] + r, (double)e[2] + r});
            }
            bounds[k] = b;
            local_bounds.grow(b);
        }
        blas.build(bounds);
    }

    // curves.rs:171-188
    static bool sphere_hit(const Ray& r, V3 c, double radius, double t_max, double* t_out, V3* n_out) {
        V3 oc = r.o - c;
        double a = dot(r.d, r.d), b = dot(oc, r.d), cc = dot(oc, oc) - radius * radius;
        double disc = b * b - a * cc;
        if (disc < 0.0) return false;
        double sq = std::sqrt(disc);
        double t = (-b - sq) / a;
        if (t <= 1e-9) t = (-b + sq) / a;
        if (t <= 1e-9 || t >= t_max) return false;
        *t_out = t;
        *n_out = normalize(r.o + r.d * t - c);
        return true;
    }

    // curves.rs:107-169: Quilez's rounded cone, parametric t along the
    // (unnormalised) local ray, outward normal.
    static bool rounded_cone(const Ray& r, V3 pa, double ra, V3 pb, double rb, double t_max, double* t_out,
                             V3* n_out) {
        V3 ba = pb - pa, oa = r.o - pa;
        double rr = ra - rb;
        double m0 = dot(ba, ba), m1 = dot(ba, oa), m2 = dot(ba, r.d), m3 = dot(r.d, oa), m5 = dot(oa, oa);
        double dd = dot(r.d, r.d);
        if (m0 < 1e-24) return sphere_hit(r, pa, std::fmax(ra, rb), t_max, t_out, n_out);
        double d2 = m0 - rr * rr;
        double k2 = d2 * dd - m2 * m2;
        double k1 = d2 * m3 - m1 * m2 + m2 * rr * ra;
        double k0 = d2 * m5 - m1 * m1 + m1 * rr * ra * 2.0 - m0 * ra * ra;
        if (std::fabs(k2) > 1e-24) {
            double h = k1 * k1 - k0 * k2;
            if (h >= 0.0) {
                double t = (-k1 - std::sqrt(h)) / k2;
                double y = m1 + t * m2;
                if (t > 1e-9 && t < t_max && y > 0.0 && y < d2) {
                    *t_out = t;
                    *n_out = normalize((oa + r.d * t) * d2 - ba * y);
                    return true;
                }
            }
        }
        // Caps: the start sphere owns y <= 0, the end sphere y >= d2.
        bool any = false;
        double tb = t_max, t;
        V3 n;
        if (sphere_hit(r, pa, ra, t_max, &t, &n) && m1 + t * m2 <= 0.0) {
            any = true;
            tb = t;
            *t_out = t;
            *n_out = n;
        }
        if (sphere_hit(r, pb, rb, tb, &t, &n) && m1 + t * m2 >= d2) {
            any = true;
            *t_out = t;
            *n_out = n;
        }
        return any;
    }

    // curves.rs:67-101: hit t, outward normal, tangent, curve parameter v.
    bool intersect_segment(const Ray& r, uint32_t k, double t_max, double* t, V3* n, V3* tang, double* v) const {
        const float *a = &p0[4 * k], *b = &p1[4 * k];
        V3 pa{a[0], a[1], a[2]}, pb{b[0], b[1], b[2]};
        if (!rounded_cone(r, pa, a[3], pb, b[3], t_max, t, n)) return false;
        V3 axis = pb - pa;
        double len2 = length_sq(axis);
        double along = len2 > 1e-24 ? std::min(std::max(dot(r.o + r.d * *t - pa, axis) / len2, 0.0), 1.0) : 0.5;
        *v = (double)v0[k] + (double)(v1[k] - v0[k]) * along;
        *tang = len2 > 1e-24 ? normalize(axis) : V3{0, 0, 1};
        return true;
    }
};

struct Instance {
    uint32_t mesh_id = 0, material_id = 0;
    bool curves = false;  // GeomKind::Curves: mesh_id indexes the curve sets
    M4 transform, inv;
    bool moving = false;  // transform1 holds the shutter-close endpoint
    M4 transform1;
    Aabb world_bounds;
    double scale = 1.0;  // Matrix4::approx_scale (math/matrix.rs:246-251)

    // mesh.rs:295-304 Instance::transforms_at: the inverse at shutter time
    // (the lerped transform inverted, identity when singular).
    M4 inv_at(double time) const {
        if (!moving || !(time > 0.0)) return inv;
        M4 r;
        if (!inverse(lerp(transform, transform1, time), r)) r = identity();
        return r;
    }
};

// ---- analytic quadrics (src/geometry/sphere.rs, cylinder.rs, cone.rs, extra.rs) ----
// The reference's legacy RiSpec primitives: the ray goes to object space
// with its direction normalised there, the local root is tested against the
// shape's cuts, and t is the world distance of the hit point from the ray
// origin. Each function returns the local hit point and local normal.
struct QuadricHit {
    V3 p, n;          // object space
    double u, v;      // RiSpec parameterisation
    double dpdu, dpdv;
    bool front_set;   // the shape decides the front face from the world normal (sphere)
};

// extra.rs:44-54 (phi in [0, 360) from x, y; accepted when <= thetamax).
static bool q_theta_ok(double x, double y, double thetamax) {
    if (thetamax >= 360.0) return true;
    double phi = std::atan2(y, x) * 180.0 / PI;
    if (phi < 0.0) phi += 360.0;
    return phi <= thetamax;
}
// extra.rs:35-42.
static double q_phi_u(double x, double y, double thetamax) {
    double phi = std::atan2(y, x) * 180.0 / PI;
    if (phi < 0.0) phi += 360.0;
    return std::min(std::max(phi / std::fmax(thetamax, 1e-9), 0.0), 1.0);
}

// Real roots of a3 t^3 + a2 t^2 + a1 t + a0, ascending: Cardano with the
// trigonometric form for three real roots (extra.rs:195-241 solves it the
// same way).
static std::vector<double> q_cubic(double a3, double a2, double a1, double a0) {
    if (std::fabs(a3) < 1e-12) {
        if (std::fabs(a2) < 1e-12) {
            if (std::fabs(a1) < 1e-12) return {};
            return {-a0 / a1};
        }
        double disc = a1 * a1 - 4.0 * a2 * a0;
        if (disc < 0.0) return {};
        double r = std::sqrt(disc);
        std::vector<double> v{(-a1 - r) / (2.0 * a2), (-a1 + r) / (2.0 * a2)};
        std::sort(v.begin(), v.end());
        return v;
    }
    const double a = a2 / a3, b = a1 / a3, c = a0 / a3;
    const double p = b - a * a / 3.0, q = 2.0 * a * a * a / 27.0 - a * b / 3.0 + c, shift = -a / 3.0;
    const double disc = q * q / 4.0 + p * p * p / 27.0;
    std::vector<double> out;
    if (disc > 0.0) {
        double r = std::sqrt(disc);
        out.push_back(std::cbrt(-q / 2.0 + r) + std::cbrt(-q / 2.0 - r) + shift);
    } else {
        double m = 2.0 * std::sqrt(std::fmax(-p / 3.0, 0.0));
        if (m < 1e-30) {
            out.push_back(shift);
        } else {
            double th = std::acos(std::min(std::max(3.0 * q / (p * m), -1.0), 1.0)) / 3.0;
            for (int k = 0; k < 3; k++) out.push_back(m * std::cos(th - 2.0 * PI * k / 3.0) + shift);
        }
    }
    std::sort(out.begin(), out.end());
    return out;
}

// Real roots of a4 t^4 + ... + a0, ascending (extra.rs:112-193): Ferrari's
// reduction to the resolvent cubic (biquadratic when the depressed quartic
// has no linear term), each root polished by Newton on the original
// polynomial, spurious roots and duplicates dropped.
static std::vector<double> q_quartic(double a4, double a3, double a2, double a1, double a0) {
    if (std::fabs(a4) < 1e-12) return q_cubic(a3, a2, a1, a0);
    const double b = a3 / a4, c = a2 / a4, d = a1 / a4, e = a0 / a4;
    const double p = c - 3.0 * b * b / 8.0;
    const double q = d - b * c / 2.0 + b * b * b / 8.0;
    const double r = e - b * d / 4.0 + b * b * c / 16.0 - 3.0 * b * b * b * b / 256.0;
    const double shift = -b / 4.0;
    auto f = [&](double t) { return (((a4 * t + a3) * t + a2) * t + a1) * t + a0; };
    auto df = [&](double t) { return ((4.0 * a4 * t + 3.0 * a3) * t + 2.0 * a2) * t + a1; };
    auto polish = [&](double t) {
        for (int it = 0; it < 8; it++) {
            double g = df(t);
            if (std::fabs(g) < 1e-30) break;
            double step = f(t) / g;
            t -= step;
            if (std::fabs(step) < 1e-12 * std::fmax(std::fabs(t), 1.0)) break;
        }
        return t;
    };
    std::vector<double> roots;
    if (std::fabs(q) < 1e-12) {
        double disc = p * p - 4.0 * r;
        if (disc >= 0.0) {
            double sq = std::sqrt(disc);
            for (double y2 : {(-p - sq) / 2.0, (-p + sq) / 2.0})
                if (y2 >= 0.0) {
                    double y = std::sqrt(y2);
                    roots.push_back(polish(y + shift));
                    roots.push_back(polish(-y + shift));
                }
        }
    } else {
        double z = NAN;
        for (double zz : q_cubic(1.0, 2.0 * p, p * p - 4.0 * r, -q * q))
            if (zz > 1e-12 && !(zz <= z)) z = zz;   // the largest positive root
        if (std::isfinite(z)) {
            double m = std::sqrt(z), n = q / (2.0 * m);
            for (int sgn : {1, -1}) {
                double bq = sgn * m, cq = (p + z) / 2.0 - sgn * n;
                double disc = bq * bq - 4.0 * cq;
                if (disc >= 0.0) {
                    double sq = std::sqrt(disc);
                    roots.push_back(polish((-bq - sq) / 2.0 + shift));
                    roots.push_back(polish((-bq + sq) / 2.0 + shift));
                }
            }
        }
    }
    std::vector<double> keep;
    for (double t : roots)
        if (std::isfinite(t) && std::fabs(f(t)) < 1e-6 * (1.0 + std::pow(std::fabs(t), 4) * std::fabs(a4)))
            keep.push_back(t);
    std::sort(keep.begin(), keep.end());
    std::vector<double> out;
    for (double t : keep)
        if (out.empty() || std::fabs(t - out.back()) >= 1e-9) out.push_back(t);
    return out;
}

struct Quadric {
    uint32_t type = 0, material_id = 0;
    double prm[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    M4 transform, inv;
    double scale = 1.0;  // Matrix4::approx_scale

    // Local intersection; false on a miss.
    bool local_hit(V3 lo, V3 ld, QuadricHit* h) const {
        h->front_set = false;
        switch (type) {
            case RT_QUADRIC_SPHERE: return sphere(lo, ld, h);
            case RT_QUADRIC_CYLINDER: return cylinder(lo, ld, h);
            case RT_QUADRIC_CONE: return cone(lo, ld, h);
            case RT_QUADRIC_TORUS: return torus(lo, ld, h);
            case RT_QUADRIC_DISK: return disk(lo, ld, h);
            case RT_QUADRIC_PARABOLOID: return paraboloid(lo, ld, h);
            case RT_QUADRIC_HYPERBOLOID: return hyperboloid(lo, ld, h);
        }
        return false;
    }
    // sphere.rs:39-103: near root, else far root; the z cut and the theta
    // cut reject without trying the other root.
    bool sphere(V3 o, V3 d, QuadricHit* h) const {
        const double radius = prm[0], zmin = prm[1], zmax = prm[2], thetamax = prm[3];
        double a = dot(d, d), b = 2.0 * dot(o, d), c = dot(o, o) - radius * radius;
        double disc = b * b - 4.0 * a * c;
        if (disc < 0.0) return false;
        double sq = std::sqrt(disc), t1 = (-b - sq) / (2.0 * a), t2 = (-b + sq) / (2.0 * a);
        double t = t1 > EPSILON ? t1 : t2;
        if (!(t > EPSILON)) return false;
        V3 p = o + d * t;
        if (p.z < zmin || p.z > zmax) return false;
        if (thetamax < 360.0 && !q_theta_ok(p.x, p.y, thetamax)) return false;
        h->p = p;
        h->n = normalize(p);
        h->u = q_phi_u(p.x, p.y, thetamax);
        double zr = std::fmax(zmax - zmin, 1e-12);
        h->v = std::min(std::max((p.z - zmin) / zr, 0.0), 1.0);
        double ring = std::fmax(std::sqrt(p.x * p.x + p.y * p.y), 1e-6 * std::fmax(radius, 1e-12));
        h->dpdu = ring * thetamax * PI / 180.0;
        h->dpdv = zr * radius / ring;
        h->front_set = true;
        return true;
    }
    // cylinder.rs:37-120: a z-cut miss on the near root retries the far root.
    bool cylinder(V3 o, V3 d, QuadricHit* h) const {
        const double radius = prm[0], zmin = prm[1], zmax = prm[2], thetamax = prm[3];
        double a = d.x * d.x + d.y * d.y, b = 2.0 * (o.x * d.x + o.y * d.y), c = o.x * o.x + o.y * o.y - radius * radius;
        if (std::fabs(a) < EPSILON) return false;
        double disc = b * b - 4.0 * a * c;
        if (disc < 0.0) return false;
        double sq = std::sqrt(disc), t1 = (-b - sq) / (2.0 * a), t2 = (-b + sq) / (2.0 * a);
        double t = t1 > EPSILON ? t1 : t2;
        if (t <= EPSILON) return false;
        V3 p = o + d * t;
        if (p.z < zmin || p.z > zmax) {
            if (t == t1 && t2 > EPSILON) {
                t = t2;
                p = o + d * t;
                if (p.z < zmin || p.z > zmax) return false;
            } else {
                return false;
            }
        }
        if (thetamax < 360.0 && !q_theta_ok(p.x, p.y, thetamax)) return false;
        h->p = p;
        h->n = normalize(V3{p.x, p.y, 0.0});
        h->u = q_phi_u(p.x, p.y, thetamax);
        double zr = std::fmax(zmax - zmin, 1e-12);
        h->v = std::min(std::max((p.z - zmin) / zr, 0.0), 1.0);
        h->dpdu = std::fmax(radius, 1e-12) * thetamax * PI / 180.0;
        h->dpdv = zr;
        return true;
    }
    // cone.rs:36-142: the cone x^2 + y^2 = k z^2, k = (radius / height)^2,
    // apex at the origin, 0 <= z <= height.
    bool cone_finish(V3 p, QuadricHit* h) const {
        const double height = prm[0], radius = prm[1], thetamax = prm[2];
        double r = std::sqrt(p.x * p.x + p.y * p.y);
        double k = radius / height;
        h->p = p;
        h->n = normalize(V3{p.x / r, p.y / r, -k});
        h->u = q_phi_u(p.x, p.y, thetamax);
        h->v = std::min(std::max(p.z / std::fmax(height, 1e-12), 0.0), 1.0);
        h->dpdu = std::fmax(r, 1e-6 * std::fmax(radius, 1e-12)) * thetamax * PI / 180.0;
        h->dpdv = std::sqrt(height * height + radius * radius);
        return true;
    }
    bool cone(V3 o, V3 d, QuadricHit* h) const {
        const double height = prm[0], radius = prm[1], thetamax = prm[2];
        double k = (radius / height) * (radius / height);
        double a = d.x * d.x + d.y * d.y - k * d.z * d.z;
        double b = 2.0 * (o.x * d.x + o.y * d.y - k * o.z * d.z);
        double c = o.x * o.x + o.y * o.y - k * o.z * o.z;
        if (std::fabs(a) < EPSILON) {
            if (std::fabs(b) < EPSILON) return false;
            double t = -c / b;
            if (t > EPSILON) {
                V3 p = o + d * t;
                if (p.z >= 0.0 && p.z <= height) return cone_finish(p, h);
            }
            return false;
        }
        double disc = b * b - 4.0 * a * c;
        if (disc < 0.0) return false;
        double sq = std::sqrt(disc);
        for (double t : {(-b - sq) / (2.0 * a), (-b + sq) / (2.0 * a)}) {
            if (!(t > EPSILON)) continue;
            V3 p = o + d * t;
            if (!(p.z >= 0.0 && p.z <= height)) continue;
            if (thetamax < 360.0 && !q_theta_ok(p.x, p.y, thetamax)) continue;
            return cone_finish(p, h);
        }
        return false;
    }
    // extra.rs:92-109 (the tube angle phi in [phimin, phimin + 360)).
    bool torus_phi(V3 p, double* vphi) const {
        const double R = prm[0], phimin = prm[2];
        double rxy = std::sqrt(p.x * p.x + p.y * p.y);
        double phi = std::atan2(p.z, rxy - R) * 180.0 / PI;
        while (phi < phimin) phi += 360.0;
        while (phi >= phimin + 360.0) phi -= 360.0;
        *vphi = phi;
        return true;
    }
    // extra.rs:243-303: roots ascending, the first past EPSILON inside both cuts.
    bool torus(V3 o, V3 d, QuadricHit* h) const {
        const double R = prm[0], r = prm[1], phimin = prm[2], phimax = prm[3], thetamax = prm[4];
        double g = dot(d, d), hh = 2.0 * dot(o, d), i = dot(o, o) + R * R - r * r;
        double j = d.x * d.x + d.y * d.y, k = 2.0 * (o.x * d.x + o.y * d.y), l = o.x * o.x + o.y * o.y;
        double fr = 4.0 * R * R;
        for (double t : q_quartic(g * g, 2.0 * g * hh, hh * hh + 2.0 * g * i - fr * j, 2.0 * hh * i - fr * k,
                                  i * i - fr * l)) {
            if (t <= EPSILON) continue;
            V3 p = o + d * t;
            double vphi;
            torus_phi(p, &vphi);
            if (phimax - phimin < 360.0 && !(vphi <= phimax)) continue;
            if (!q_theta_ok(p.x, p.y, thetamax)) continue;
            double rxy = std::fmax(std::sqrt(p.x * p.x + p.y * p.y), 1e-12);
            double sc = 1.0 - R / rxy;
            h->p = p;
            h->n = normalize(V3{p.x * sc, p.y * sc, p.z});
            h->u = q_phi_u(p.x, p.y, thetamax);
            double vr = std::fmax(phimax - phimin, 1e-9);
            h->v = std::min(std::max((vphi - phimin) / vr, 0.0), 1.0);
            h->dpdu = rxy * thetamax * PI / 180.0;
            h->dpdv = std::fmax(r, 1e-12) * vr * PI / 180.0;
            return true;
        }
        return false;
    }
    // extra.rs:347-381.
    bool disk(V3 o, V3 d, QuadricHit* h) const {
        const double height = prm[0], radius = prm[1], thetamax = prm[2];
        if (std::fabs(d.z) < EPSILON) return false;
        double t = (height - o.z) / d.z;
        if (t <= EPSILON) return false;
        V3 p = o + d * t;
        if (p.x * p.x + p.y * p.y > radius * radius) return false;
        if (!q_theta_ok(p.x, p.y, thetamax)) return false;
        double rh = std::sqrt(p.x * p.x + p.y * p.y);
        h->p = p;
        h->n = V3{0, 0, 1};
        h->u = q_phi_u(p.x, p.y, thetamax);
        h->v = std::min(std::max((radius - rh) / std::fmax(radius, 1e-12), 0.0), 1.0);
        h->dpdu = std::fmax(rh, 1e-6 * std::fmax(radius, 1e-12)) * thetamax * PI / 180.0;
        h->dpdv = radius;
        return true;
    }
    // extra.rs:425-484: candidates in order, the first inside both cuts.
    bool paraboloid(V3 o, V3 d, QuadricHit* h) const {
        const double rmax = prm[0], zmin = prm[1], zmax = prm[2], thetamax = prm[3];
        if (std::fabs(zmax) < EPSILON) return false;
        double k = rmax * rmax / zmax;
        double a = d.x * d.x + d.y * d.y, b = 2.0 * (o.x * d.x + o.y * d.y) - k * d.z;
        double c = o.x * o.x + o.y * o.y - k * o.z;
        double cand[2];
        int nc = 0;
        if (std::fabs(a) < EPSILON) {
            if (std::fabs(b) < EPSILON) return false;
            cand[nc++] = -c / b;
        } else {
            double disc = b * b - 4.0 * a * c;
            if (disc < 0.0) return false;
            double sq = std::sqrt(disc);
            cand[nc++] = (-b - sq) / (2.0 * a);
            cand[nc++] = (-b + sq) / (2.0 * a);
        }
        for (int i = 0; i < nc; i++) {
            double t = cand[i];
            if (t <= EPSILON) continue;
            V3 p = o + d * t;
            if (p.z < zmin || p.z > zmax) continue;
            if (!q_theta_ok(p.x, p.y, thetamax)) continue;
            h->p = p;
            h->n = normalize(V3{2.0 * p.x, 2.0 * p.y, -k});
            h->u = q_phi_u(p.x, p.y, thetamax);
            double zr = std::fmax(zmax - zmin, 1e-12);
            h->v = std::min(std::max((p.z - zmin) / zr, 0.0), 1.0);
            double ring = std::fmax(std::sqrt(p.x * p.x + p.y * p.y), 1e-6 * std::fmax(rmax, 1e-12));
            h->dpdu = ring * thetamax * PI / 180.0;
            h->dpdv = zr;
            return true;
        }
        return false;
    }
    // extra.rs:526-632: a flat annulus when p1 and p2 share z, else the
    // hyperboloid of revolution swept by the line p1 -> p2.
    bool hyperboloid(V3 o, V3 d, QuadricHit* h) const {
        const double p1[3] = {prm[0], prm[1], prm[2]}, p2[3] = {prm[3], prm[4], prm[5]};
        const double thetamax = prm[6];
        const double zlo = std::fmin(p1[2], p2[2]), zhi = std::fmax(p1[2], p2[2]);
        if (std::fabs(p2[2] - p1[2]) < EPSILON) {
            if (std::fabs(d.z) < EPSILON) return false;
            double t = (p1[2] - o.z) / d.z;
            if (t <= EPSILON) return false;
            V3 p = o + d * t;
            double r2 = p.x * p.x + p.y * p.y;
            double ra = p1[0] * p1[0] + p1[1] * p1[1], rb = p2[0] * p2[0] + p2[1] * p2[1];
            if (r2 < std::fmin(ra, rb) || r2 > std::fmax(ra, rb)) return false;
            if (!q_theta_ok(p.x, p.y, thetamax)) return false;
            h->p = p;
            h->n = V3{0, 0, 1};
            h->u = h->v = 0.0;
            h->dpdu = h->dpdv = 0.0;   // no st on the flat case (extra.rs:560-567)
            return true;
        }
        const double dz = p2[2] - p1[2], iu = 1.0 / dz;
        const double sx = (p2[0] - p1[0]) * iu, sy = (p2[1] - p1[1]) * iu;
        const double cx = p1[0] - p1[2] * sx, cy = p1[1] - p1[2] * sy;
        const double pa = sx * sx + sy * sy, pb = 2.0 * (cx * sx + cy * sy), pc = cx * cx + cy * cy;
        double a = d.x * d.x + d.y * d.y - pa * d.z * d.z;
        double b = 2.0 * (o.x * d.x + o.y * d.y - pa * o.z * d.z) - pb * d.z;
        double c = o.x * o.x + o.y * o.y - pa * o.z * o.z - pb * o.z - pc;
        double cand[2];
        int nc = 0;
        if (std::fabs(a) < EPSILON) {
            if (std::fabs(b) < EPSILON) return false;
            cand[nc++] = -c / b;
        } else {
            double disc = b * b - 4.0 * a * c;
            if (disc < 0.0) return false;
            double sq = std::sqrt(disc);
            cand[nc++] = (-b - sq) / (2.0 * a);
            cand[nc++] = (-b + sq) / (2.0 * a);
        }
        for (int i = 0; i < nc; i++) {
            double t = cand[i];
            if (t <= EPSILON) continue;
            V3 p = o + d * t;
            if (p.z < zlo || p.z > zhi) continue;
            if (!q_theta_ok(p.x, p.y, thetamax)) continue;
            h->p = p;
            h->n = normalize(V3{2.0 * p.x, 2.0 * p.y, -(2.0 * pa * p.z + pb)});
            h->u = q_phi_u(p.x, p.y, thetamax);
            h->v = std::min(std::max((p.z - p1[2]) / dz, 0.0), 1.0);
            double ring = std::fmax(std::sqrt(p.x * p.x + p.y * p.y), 1e-12);
            h->dpdu = ring * thetamax * PI / 180.0;
            double sw[3] = {p2[0] - p1[0], p2[1] - p1[1], p2[2] - p1[2]};
            h->dpdv = std::fmax(std::sqrt(sw[0] * sw[0] + sw[1] * sw[1] + sw[2] * sw[2]), 1e-12);
            return true;
        }
        return false;
    }
};

struct Hit {
    double t;        // euclidean distance from the ray origin
    V3 point, normal;
    uint32_t material_id, inst, prim;
    bool front_face;
    double st[2] = {0.0, 0.0};
    double st_density = 0.0;  // st units per world unit (0 without st)
    V3 st_grad[2] = {{0, 0, 0}, {0, 0, 0}};  // world-space gradients of s and t
    V3 tangent{0, 0, 0};                        // curve tangent (zero for surfaces)
};

// ---- patterns (src/texture/pattern.rs, src/geometry/displace.rs) -------------

// displace.rs:36-80: classic Perlin gradient noise over a hashed lattice.
static uint32_t lattice_hash(int64_t x) {
    uint64_t u = (uint64_t)x * 0x9e3779b97f4a7c15ull;
    x = (int64_t)u;
    x ^= x >> 29;  // arithmetic shift, as on the reference's i64
    u = (uint64_t)x * 0xbf58476d1ce4e5b9ull;
    x = (int64_t)u;
    x ^= x >> 32;
    return (uint32_t)(uint64_t)x;
}
static double perlin(double px, double py, double pz) {
    double cx = std::floor(px), cy = std::floor(py), cz = std::floor(pz);
    double f[3] = {px - cx, py - cy, pz - cz};
    int64_t ix = (int64_t)cx, iy = (int64_t)cy, iz = (int64_t)cz;
    double corner[8];
    for (int k = 0; k < 8; k++) {
        int64_t dx = k & 1, dy = (k >> 1) & 1, dz = (k >> 2) & 1;
        uint64_t key = (uint64_t)(ix + dx) * 73856093ull ^ (uint64_t)(iy + dy) * 19349663ull ^
                       (uint64_t)(iz + dz) * 83492791ull;
        uint32_t h = lattice_hash((int64_t)key) % 12u;
        // The 12 cube-edge gradients, in the reference's order.
        double g0 = (h < 8) ? ((h & 1) ? -1.0 : 1.0) : 0.0;
        double g1 = (h < 4) ? ((h & 2) ? -1.0 : 1.0) : (h < 8 ? 0.0 : ((h & 1) ? -1.0 : 1.0));
        double g2 = (h < 4) ? 0.0 : (h < 8 ? ((h & 2) ? -1.0 : 1.0) : ((h & 2) ? -1.0 : 1.0));
        corner[k] = g0 * (f[0] - (double)dx) + g1 * (f[1] - (double)dy) + g2 * (f[2] - (double)dz);
    }
    auto fade = [](double t) { return t * t * t * (t * (t * 6.0 - 15.0) + 10.0); };
    auto lerp = [](double a, double b, double t) { return a + (b - a) * t; };
    double u = fade(f[0]), v = fade(f[1]), w = fade(f[2]);
    double y0 = lerp(lerp(corner[0], corner[1], u), lerp(corner[2], corner[3], u), v);
    double y1 = lerp(lerp(corner[4], corner[5], u), lerp(corner[6], corner[7], u), v);
    return lerp(y0, y1, w);
}
// displace.rs:82-97 (offset 0, as PatternNode::Fractal passes it).
static double fbm(V3 p, double frequency, uint32_t octaves, double gain, double lacunarity) {
    double sum = 0.0, amp = 1.0, freq = frequency;
    for (uint32_t o = 0; o < std::max(octaves, 1u); o++) {
        sum += amp * perlin(p.x * freq, p.y * freq, p.z * freq);
        amp *= gain;
        freq *= lacunarity;
    }
    return sum;
}

// ---- participating media (src/scene/medium.rs, src/raytracer/pt/volume.rs) ----

struct Medium {  // medium.rs:28-43
    V3 sigma_a, sigma_s, emission;
    double g = 0.0, max_distance = INF;
    bool fbm_density = false;
    uint32_t octaves = 5;
    double frequency = 0.3, gain = 0.55, lacunarity = 2.0, coverage = 0.5, sharpness = 4.0;
    V3 sigma_t() const { return sigma_a + sigma_s; }
    double majorant() const { return max_comp(sigma_t()); }  // medium.rs:50-55
    double density_at(V3 p) const {                           // medium.rs:57-66
        if (!fbm_density) return 1.0;
        double n = fbm(p, frequency, octaves, gain, lacunarity) * 0.5 + 0.5;
        return std::min(std::max((n - (1.0 - coverage)) * sharpness, 0.0), 1.0);
    }
};

// medium.rs:73-76
static double hg_phase(double g, double cos_theta) {
    double denom = 1.0 + g * g + 2.0 * g * cos_theta;
    return (1.0 - g * g) / (4.0 * PI * denom * std::sqrt(std::fmax(denom, 1e-9)));
}

// medium.rs:80-103: direction around the propagation direction -wo; pdf = phase.
static V3 hg_sample(double g, V3 wo, double u1, double u2, double* pdf) {
    double cos_theta;
    if (std::fabs(g) < 1e-3) {
        cos_theta = 1.0 - 2.0 * u1;
    } else {
        double sq = (1.0 - g * g) / (1.0 + g - 2.0 * g * u1);
        cos_theta = -(1.0 + g * g - sq * sq) / (2.0 * g);
    }
    double sin_theta = std::sqrt(std::fmax(1.0 - cos_theta * cos_theta, 0.0));
    double phi = 2.0 * PI * u2;
    V3 w = -wo;
    V3 a = std::fabs(w.x) > 0.9 ? V3{0, 1, 0} : V3{1, 0, 0};
    V3 t = normalize(cross(w, a));
    V3 b = cross(w, t);
    V3 wi = normalize(t * (sin_theta * std::cos(phi)) + b * (sin_theta * std::sin(phi)) + w * cos_theta);
    *pdf = hg_phase(g, dot(wo, wi) * -1.0);
    return wi;
}

static V3 exp3(V3 v, double t) { return {std::exp(-v.x * t), std::exp(-v.y * t), std::exp(-v.z * t)}; }

// volume.rs:11-20: scatter at t (scatter = true) or pass the segment; the
// weight folds transmittance, sigma_s and the sampling pdf.
struct MediumEvent {
    bool scatter = false;
    double t = 0.0;
    V3 weight{1, 1, 1};
};

template <class R>
static MediumEvent sample_homogeneous(const Medium& m, double t_max, V3 beta, R& rng) {  // volume.rs:62-105
    MediumEvent ev;
    V3 st = m.sigma_t();
    if ((st.x + st.y + st.z) / 3.0 <= 1e-9) return ev;
    V3 b{std::fmax(beta.x, 0.0), std::fmax(beta.y, 0.0), std::fmax(beta.z, 0.0)};  // volume.rs:51-59
    double total = b.x + b.y + b.z;
    double w[3] = {1.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0};
    if (total > 1e-12) {
        w[0] = b.x / total;
        w[1] = b.y / total;
        w[2] = b.z / total;
    }
    double u = rng.next_f64();
    int c = u < w[0] ? 0 : (u < w[0] + w[1] ? 1 : 2);
    double sigma_c = std::fmax(axis_of(st, c), 1e-9);
    double t = -std::log(std::fmax(1.0 - rng.next_f64(), 1e-12)) / sigma_c;
    if (t < t_max) {
        V3 tr = exp3(st, t);
        double pdf = w[0] * st.x * tr.x + w[1] * st.y * tr.y + w[2] * st.z * tr.z;
        if (pdf <= 1e-300) {
            ev.weight = {0, 0, 0};
            return ev;
        }
        ev.scatter = true;
        ev.t = t;
        ev.weight = m.sigma_s * tr / pdf;
        return ev;
    }
    V3 tr = exp3(st, t_max);
    double pdf = w[0] * tr.x + w[1] * tr.y + w[2] * tr.z;
    ev.weight = pdf <= 1e-300 ? V3{0, 0, 0} : tr / pdf;
    return ev;
}

// volume.rs:109-156: weighted delta tracking against the channel-max majorant.
template <class R>
static MediumEvent sample_delta_tracked(const Medium& m, V3 o, V3 d, double t_max, R& rng) {
    MediumEvent ev;
    double maj = m.majorant();
    if (maj <= 1e-9) return ev;
    V3 st = m.sigma_t();
    double t = 0.0;
    V3 weight{1, 1, 1};
    for (int i = 0; i < 10000; i++) {
        t -= std::log(std::fmax(1.0 - rng.next_f64(), 1e-12)) / maj;
        if (t >= t_max) {
            ev.weight = weight;
            return ev;
        }
        double rho = m.density_at(o + d * t);
        V3 sh = st * rho;
        double p_real = std::min(std::max((sh.x + sh.y + sh.z) / 3.0 / maj, 0.0), 1.0);
        if (rng.next_f64() < p_real) {
            ev.scatter = true;
            ev.t = t;
            ev.weight = weight * (m.sigma_s * rho) / (maj * p_real);
            return ev;
        }
        double p_null = std::fmax(1.0 - p_real, 1e-9);
        weight = weight * V3{(1.0 - sh.x / maj) / p_null, (1.0 - sh.y / maj) / p_null, (1.0 - sh.z / maj) / p_null};
        if (max_comp(weight) < 1e-6) {
            ev.weight = {0, 0, 0};
            return ev;
        }
    }
    ev.weight = weight;
    return ev;
}

// volume.rs:35-49 (o, d: the ray; d normalised as Ray::new keeps it).
template <class R>
static MediumEvent sample_distance(const Medium& m, V3 o, V3 d, double t_max, V3 beta, R& rng) {
    t_max = std::fmin(t_max, m.max_distance);
    if (!m.fbm_density) return sample_homogeneous(m, t_max, beta, rng);
    return sample_delta_tracked(m, o, d, t_max, rng);
}

// volume.rs:160-193: closed form, or ratio tracking.
template <class R>
static V3 medium_transmittance(const Medium& m, V3 o, V3 d, double dist, R& rng) {
    dist = std::fmin(dist, m.max_distance);
    V3 st = m.sigma_t();
    if (!m.fbm_density) return exp3(st, dist);
    double maj = m.majorant();
    if (maj <= 1e-9) return {1, 1, 1};
    double t = 0.0;
    V3 tr{1, 1, 1};
    for (int i = 0; i < 10000; i++) {
        t -= std::log(std::fmax(1.0 - rng.next_f64(), 1e-12)) / maj;
        if (t >= dist) break;
        double rho = m.density_at(o + d * t);
        tr = tr * V3{1.0 - st.x * rho / maj, 1.0 - st.y * rho / maj, 1.0 - st.z * rho / maj};
        if (max_comp(tr) < 1e-5) return {0, 0, 0};
    }
    return tr;
}

// volume.rs:199-235: equiangular sampling toward a point light and its pdf.
static double equiangular_pdf(V3 o, V3 d, double t_max, V3 lp, double t) {
    double delta = dot(lp - o, d);
    double h = std::fmax(length(lp - (o + d * delta)), 1e-6);
    double ta = std::atan(-delta / h), tb = std::atan((t_max - delta) / h);
    double span = std::fmax(tb - ta, 1e-9);
    return h / (span * (h * h + (t - delta) * (t - delta)));
}
static double equiangular_sample(V3 o, V3 d, double t_max, V3 lp, double u, double* pdf) {
    double delta = dot(lp - o, d);
    double h = std::fmax(length(lp - (o + d * delta)), 1e-6);
    double ta = std::atan(-delta / h), tb = std::atan((t_max - delta) / h);
    double span = std::fmax(tb - ta, 1e-9);
    double t = delta + h * std::tan(ta + u * span);
    t = std::min(std::max(t, 0.0), t_max);
    *pdf = h / (span * (h * h + (t - delta) * (t - delta)));
    return t;
}

// volume.rs:240-249
static double distance_pdf_approx(const Medium& m, double t, double t_max) {
    V3 st = m.sigma_t();
    double s = std::fmax((st.x + st.y + st.z) / 3.0, 1e-9);
    return t < t_max ? s * std::exp(-s * t) : std::exp(-s * t_max);
}

// volume.rs:259-288: the random-walk medium of a PxrSurface subsurface
// colour and mean free path (Kulla-Conty albedo inversion, Christensen-Burley
// scaling).
static Medium sss_medium(V3 color, V3 dmfp) {
    auto alpha_fit = [](double a) {
        a = std::min(std::max(a, 0.0), 1.0);
        return 1.0 - std::exp(-a * (11.43 - 15.38 * a + 13.91 * a * a));
    };
    auto s_fit = [](double a) { return 1.85 - a + 7.0 * std::pow(std::fabs(a - 0.8), 3); };
    auto cl = [](double v) { return std::min(std::max(v, 0.0), 1.0); };
    V3 a{cl(color.x), cl(color.y), cl(color.z)};
    V3 st{s_fit(a.x) / std::fmax(dmfp.x, 1e-5), s_fit(a.y) / std::fmax(dmfp.y, 1e-5), s_fit(a.z) / std::fmax(dmfp.z, 1e-5)};
    V3 alpha{alpha_fit(a.x), alpha_fit(a.y), alpha_fit(a.z)};
    Medium m;
    m.sigma_s = alpha * st;
    m.sigma_a = st - m.sigma_s;
    m.emission = {0, 0, 0};
    return m;
}

struct PatInput {
    int32_t node;  // -1: constant
    V3 value;
};
struct PatNode {
    int32_t type;
    uint32_t octaves;
    V3 a, b;
    double scale[2], frequency, gain, lacunarity, gamma, saturation;
    PatInput in[3];
    std::vector<double> ramp_pos;
    std::vector<V3> ramp_col;
    bool use_t;
    int32_t texture;  // texture / triplanar: index, -1 = missing
    int wrap;
    std::vector<std::pair<uint32_t, int32_t>> udim;  // (tile, texture) when a UDIM set
};
struct ShadeCtx {  // pattern.rs:69-82
    double st[2];
    V3 p, n;
    double footprint;
    double dst_major[2], dst_minor[2];
};

// A file texture as the reference's cache serves it (texture/cache.rs,
// texture/tex.rs): the box mip chain down to 1x1 (f32 2x2 averages, odd
// sizes clamping the second tap), texels read with wrap, bilinear,
// trilinear and EWA lookups. Sums are f32 where the reference's are.
struct Texture {
    struct Mip {
        uint32_t w, h;
        std::vector<float> rgb;
    };
    std::vector<Mip> mips;

    void build(const float* rgb, uint32_t w, uint32_t h) {  // tex.rs:89-130
        mips.clear();
        mips.push_back({w, h, std::vector<float>(rgb, rgb + 3ull * w * h)});
        while (mips.back().w > 1 || mips.back().h > 1) {
            const Mip& a = mips.back();
            Mip b{std::max(a.w / 2, 1u), std::max(a.h / 2, 1u), {}};
            b.rgb.resize(3ull * b.w * b.h);
            for (uint32_t y = 0; y < b.h; y++) {
                uint32_t y0 = std::min(2 * y, a.h - 1), y1 = std::min(2 * y + 1, a.h - 1);
                for (uint32_t x = 0; x < b.w; x++) {
                    uint32_t x0 = std::min(2 * x, a.w - 1), x1 = std::min(2 * x + 1, a.w - 1);
                    for (int c = 0; c < 3; c++) {
                        float sum = a.rgb[3 * ((size_t)y0 * a.w + x0) + c] + a.rgb[3 * ((size_t)y0 * a.w + x1) + c];
                        sum = sum + a.rgb[3 * ((size_t)y1 * a.w + x0) + c];
                        sum = sum + a.rgb[3 * ((size_t)y1 * a.w + x1) + c];
                        b.rgb[3 * ((size_t)y * b.w + x) + c] = sum * 0.25f;
                    }
                }
            }
            mips.push_back(std::move(b));
        }
    }
    // cache.rs:186-203
    void texel(size_t mip, int64_t x, int64_t y, int wrap, float out[3]) const {
        const Mip& m = mips[mip];
        const int64_t w = m.w, h = m.h;
        if (wrap == RT_WRAP_PERIODIC) {
            x = ((x % w) + w) % w;
            y = ((y % h) + h) % h;
        } else if (wrap == RT_WRAP_CLAMP) {
            x = std::min(std::max(x, (int64_t)0), w - 1);
            y = std::min(std::max(y, (int64_t)0), h - 1);
        } else if (x < 0 || x >= w || y < 0 || y >= h) {
            out[0] = out[1] = out[2] = 0.0f;
            return;
        }
        for (int c = 0; c < 3; c++) out[c] = m.rgb[3 * ((size_t)y * m.w + (size_t)x) + c];
    }
    // cache.rs:205-229
    void bilinear(size_t mip, double s, double t, int wrap, float out[3]) const {
        const Mip& m = mips[mip];
        double fx = s * m.w - 0.5, fy = t * m.h - 0.5;
        double x0 = std::floor(fx), y0 = std::floor(fy);
        double ax = fx - x0, ay = fy - y0;
        const int64_t ix = (int64_t)x0, iy = (int64_t)y0;
        out[0] = out[1] = out[2] = 0.0f;
        const int64_t dx[4] = {0, 1, 0, 1}, dy[4] = {0, 0, 1, 1};
        const double wt[4] = {(1.0 - ax) * (1.0 - ay), ax * (1.0 - ay), (1.0 - ax) * ay, ax * ay};
        for (int k = 0; k < 4; k++) {
            float px[3];
            texel(mip, ix + dx[k], iy + dy[k], wrap, px);
            for (int c = 0; c < 3; c++) out[c] += px[c] * (float)wt[k];
        }
    }
    // cache.rs:230-252
    void sample(double s, double t, double footprint, int wrap, float out[3]) const {
        const double base = std::max(mips[0].w, mips[0].h);
        const double texels = std::fmax(footprint * base, 1e-9);
        const double mip_f = std::min(std::max(std::log2(texels), 0.0), (double)(mips.size() - 1));
        const size_t m0 = (size_t)std::floor(mip_f), m1 = std::min(m0 + 1, mips.size() - 1);
        const double a = mip_f - (double)m0;
        bilinear(m0, s, t, wrap, out);
        if (a < 1e-6 || m1 == m0) return;
        float hi[3];
        bilinear(m1, s, t, wrap, hi);
        for (int c = 0; c < 3; c++) out[c] = out[c] * (float)(1.0 - a) + hi[c] * (float)a;
    }
    // cache.rs:283-377 (Heckbert's EWA with a Gaussian falloff)
    void sample_ewa(double s, double t, const double du[2], const double dv[2], int wrap, float out[3]) const {
        double major = std::sqrt(du[0] * du[0] + du[1] * du[1]), minor = std::sqrt(dv[0] * dv[0] + dv[1] * dv[1]);
        const double *axm = du, *axn = dv;
        if (minor > major) {
            std::swap(major, minor);
            std::swap(axm, axn);
        }
        if (major <= 1e-9) return sample(s, t, 0.0, wrap, out);
        if (minor < major / 16.0) minor = major / 16.0;
        const double base = std::max(mips[0].w, mips[0].h);
        const double level = std::min(std::max(std::log2(std::fmax(minor * base, 1e-9)), 0.0), (double)(mips.size() - 1));
        const size_t mip = (size_t)std::floor(level);
        const double mw = mips[mip].w, mh = mips[mip].h;
        const double px = s * mw - 0.5, py = t * mh - 0.5;
        const double dux = axm[0] * mw, duy = axm[1] * mh, dvx = axn[0] * mw, dvy = axn[1] * mh;
        double a = duy * duy + dvy * dvy + 1.0, b = -2.0 * (dux * duy + dvx * dvy), c = dux * dux + dvx * dvx + 1.0;
        const double f = a * c - 0.25 * b * b;
        if (f <= 1e-12) return sample(s, t, minor, wrap, out);
        a /= f;
        b /= f;
        c /= f;
        const double det = -b * b + 4.0 * a * c;
        if (det <= 0.0) return sample(s, t, minor, wrap, out);
        const double ur = std::sqrt(4.0 * c * det) / det, vr = std::sqrt(4.0 * a * det) / det;
        const int64_t x0 = (int64_t)std::floor(px - ur), x1 = (int64_t)std::ceil(px + ur);
        const int64_t y0 = (int64_t)std::floor(py - vr), y1 = (int64_t)std::ceil(py + vr);
        if ((x1 - x0) * (y1 - y0) > 4096) return sample(s, t, minor, wrap, out);
        float sum[3] = {0, 0, 0}, wsum = 0.0f;
        for (int64_t y = y0; y <= y1; y++) {
            const double ddy = (double)y - py;
            for (int64_t x = x0; x <= x1; x++) {
                const double ddx = (double)x - px;
                const double r2 = a * ddx * ddx + b * ddx * ddy + c * ddy * ddy;
                if (r2 < 1.0) {
                    const float w = (float)std::exp(-2.0 * r2);
                    float p3[3];
                    texel(mip, x, y, wrap, p3);
                    for (int k = 0; k < 3; k++) sum[k] += p3[k] * w;
                    wsum += w;
                }
            }
        }
        if (wsum <= 1e-9f) return sample(s, t, minor, wrap, out);
        for (int k = 0; k < 3; k++) out[k] = sum[k] / wsum;
    }
};
static const V3 MISSING_COLOR{1.0, 0.0, 1.0};

// pattern.rs:126-226 eval_at.
// TextureRef::resolve (pattern.rs:25-38): the texture of (s, t) and the
// st within it; a UDIM set picks tile 1001 + s cell + 10 t cell (s cells
// clamped to 0..9, t cells from 0) at the cell-local st. -1: missing.
static int32_t tex_resolve(const PatNode& n, double* s, double* t) {
    if (n.udim.empty()) return n.texture;
    const double sc = std::min(std::max(std::floor(*s), 0.0), 9.0), tc = std::fmax(std::floor(*t), 0.0);
    const uint32_t tile = 1001u + (uint32_t)sc + 10u * (uint32_t)tc;
    for (const auto& e : n.udim)
        if (e.first == tile) {
            *s -= sc;
            *t -= tc;
            return e.second;
        }
    return -1;
}

// pattern.rs:93-124: a texture lookup with t flipped into image rows; a
// missing texture reads magenta.
static V3 sample_tex(const std::vector<Texture>& tex, const PatNode& n, double s, double t, double footprint) {
    const int32_t id = tex_resolve(n, &s, &t);
    if (id < 0 || (size_t)id >= tex.size()) return MISSING_COLOR;
    float c[3];
    tex[(size_t)id].sample(s, 1.0 - t, footprint, n.wrap, c);
    return {c[0], c[1], c[2]};
}
static V3 sample_tex_ewa(const std::vector<Texture>& tex, const PatNode& n, double s, double t, const double du[2],
                         const double dv[2]) {
    const int32_t id = tex_resolve(n, &s, &t);
    if (id < 0 || (size_t)id >= tex.size()) return MISSING_COLOR;
    const double u[2] = {du[0], -du[1]}, v[2] = {dv[0], -dv[1]};
    float c[3];
    tex[(size_t)id].sample_ewa(s, 1.0 - t, u, v, n.wrap, c);
    return {c[0], c[1], c[2]};
}

static V3 pattern_eval(const std::vector<PatNode>& nodes, const std::vector<Texture>& tex, int64_t index,
                       const ShadeCtx& c, uint32_t depth) {
    if (depth > 16) return MISSING_COLOR;
    if (index < 0 || (size_t)index >= nodes.size()) return MISSING_COLOR;
    const PatNode& n = nodes[(size_t)index];
    auto input = [&](int k) {
        return n.in[k].node < 0 ? n.in[k].value : pattern_eval(nodes, tex, n.in[k].node, c, depth + 1);
    };
    switch (n.type) {
        case RT_PATTERN_TEXTURE: {  // pattern.rs:134-149
            const double s = c.st[0] * n.scale[0], t = c.st[1] * n.scale[1];
            const double aniso = std::fabs(c.dst_major[0]) + std::fabs(c.dst_major[1]) + std::fabs(c.dst_minor[0]) +
                                 std::fabs(c.dst_minor[1]);
            if (aniso > 1e-12) {
                const double du[2] = {c.dst_major[0] * n.scale[0], c.dst_major[1] * n.scale[1]};
                const double dv[2] = {c.dst_minor[0] * n.scale[0], c.dst_minor[1] * n.scale[1]};
                return sample_tex_ewa(tex, n, s, t, du, dv);
            }
            return sample_tex(tex, n, s, t, c.footprint * std::fmax(std::fabs(n.scale[0]), std::fabs(n.scale[1])));
        }
        case RT_PATTERN_TRIPLANAR: {  // pattern.rs:200-214
            const V3 a{std::fabs(c.n.x), std::fabs(c.n.y), std::fabs(c.n.z)};
            const double total = std::fmax(a.x + a.y + a.z, 1e-9);
            const double f = n.frequency;
            const V3 cx = sample_tex(tex, n, c.p.y * f, c.p.z * f, c.footprint);
            const V3 cy = sample_tex(tex, n, c.p.z * f, c.p.x * f, c.footprint);
            const V3 cz = sample_tex(tex, n, c.p.x * f, c.p.y * f, c.footprint);
            return cx * (a.x / total) + cy * (a.y / total) + cz * (a.z / total);
        }
        case RT_PATTERN_CHECKER: {
            double fs = c.st[0] * n.scale[0], ft = c.st[1] * n.scale[1];
            int64_t cell = (int64_t)(std::floor(fs) + std::floor(ft));
            cell = ((cell % 2) + 2) % 2;
            V3 sharp = cell == 0 ? n.a : n.b;
            V3 mean = (n.a + n.b) * 0.5;
            double w = std::fmin(c.footprint * std::fmax(std::fabs(n.scale[0]), std::fabs(n.scale[1])), 1.0);
            return sharp * (1.0 - w) + mean * w;
        }
        case RT_PATTERN_FRACTAL: {
            double v = std::min(std::max(fbm(c.p, n.frequency, n.octaves, n.gain, n.lacunarity) * 0.5 + 0.5, 0.0), 1.0);
            return {v, v, v};
        }
        case RT_PATTERN_MIX: {
            V3 a = input(0), b = input(1);
            double m = std::min(std::max(input(2).x, 0.0), 1.0);
            return a * (1.0 - m) + b * m;
        }
        case RT_PATTERN_COLOR_CORRECT: {
            V3 in = input(0);
            double g = 1.0 / std::fmax(n.gamma, 1e-6);
            V3 out{std::pow(std::fmax(in.x * n.a.x + n.b.x, 0.0), g), std::pow(std::fmax(in.y * n.a.y + n.b.y, 0.0), g),
                   std::pow(std::fmax(in.z * n.a.z + n.b.z, 0.0), g)};
            if (std::fabs(n.saturation - 1.0) > 1e-9) {
                double l = 0.2126 * out.x + 0.7152 * out.y + 0.0722 * out.z;
                V3 grey{l, l, l};
                out = grey + (out - grey) * n.saturation;
            }
            return out;
        }
        case RT_PATTERN_RAMP: {
            double x = std::min(std::max(n.use_t ? c.st[1] : c.st[0], 0.0), 1.0);
            if (n.ramp_col.empty()) return MISSING_COLOR;
            if (x <= n.ramp_pos[0]) return n.ramp_col[0];
            for (size_t i = 1; i < n.ramp_pos.size(); i++)
                if (x <= n.ramp_pos[i]) {
                    double span = std::fmax(n.ramp_pos[i] - n.ramp_pos[i - 1], 1e-9);
                    double a = (x - n.ramp_pos[i - 1]) / span;
                    return n.ramp_col[i - 1] * (1.0 - a) + n.ramp_col[i] * a;
                }
            return n.ramp_col.back();
        }
        default: return MISSING_COLOR;
    }
}

// ---- lights (src/scene/light.rs) and the light BVH (light_sampler.rs) ----

// envmap.rs: lat-long environment map of a dome light with 2D-CDF
// importance sampling (f64 CDFs, nearest texel).
struct EnvMap {
    uint32_t w = 0, h = 0;
    std::vector<float> rgb;  // 3 per texel, row-major, row 0 at the zenith
    std::vector<double> marginal, conditional;
    double total = 0.0;
    V3 texel(size_t x, size_t y) const {
        const float* c = &rgb[3 * (std::min<size_t>(y, h - 1) * w + std::min<size_t>(x, w - 1))];
        return V3{c[0], c[1], c[2]};
    }
    void build() {  // envmap.rs:36-55
        marginal.assign(h + 1, 0.0);
        conditional.assign((size_t)(w + 1) * h, 0.0);
        for (uint32_t y = 0; y < h; y++) {
            const double sin_t = std::sin(PI * (y + 0.5) / h);
            double acc = 0.0;
            for (uint32_t x = 0; x < w; x++) {
                acc += lum(texel(x, y)) * sin_t;
                conditional[(size_t)y * (w + 1) + x + 1] = acc;
            }
            marginal[y + 1] = marginal[y] + acc;
        }
        total = std::fmax(marginal[h], 1e-12);
    }
    double mean_luminance() const { return total / std::fmax((double)w * h * (2.0 / PI), 1e-12); }  // :62-67
    void texel_of(V3 dir, size_t* x, size_t* y) const {
        V3 d = normalize(dir);
        double u = std::atan2(d.x, -d.z) / (2.0 * PI);
        u -= std::floor(u);
        double v = std::fmin(std::fmax(std::acos(std::fmin(std::fmax(d.y, -1.0), 1.0)) / PI, 0.0), 1.0);
        *x = std::min((size_t)(u * w), (size_t)w - 1);
        *y = std::min((size_t)(v * h), (size_t)h - 1);
    }
    V3 eval(V3 dir) const {  // :83-91
        size_t x, y;
        texel_of(dir, &x, &y);
        return texel(x, y);
    }
    double pdf(V3 dir) const {  // :129-144
        size_t x, y;
        texel_of(dir, &x, &y);
        const double sin_t = std::sin(PI * (y + 0.5) / h);
        if (sin_t < 1e-9) return 0.0;
        return lum(texel(x, y)) * sin_t * w * h / (total * 2.0 * PI * PI * sin_t);
    }
    static size_t find(const double* cdf, size_t n, double target) {  // binary_search, then clamp
        const double* it = std::lower_bound(cdf, cdf + n + 1, target);
        size_t i = (size_t)(it - cdf);
        size_t r = (i <= n && cdf[i] == target) ? i : (i > 0 ? i - 1 : 0);
        return std::min(r, n - 1);
    }
    V3 sample(double u1, double u2, V3* rad, double* pdf_out) const {  // :100-126
        size_t y = find(marginal.data(), h, u1 * total);
        double row = std::fmax(marginal[y + 1] - marginal[y], 1e-12);
        size_t x = find(&conditional[y * (w + 1)], w, u2 * row);
        double u = (x + 0.5) / w, v = (y + 0.5) / h;
        double phi = u * 2.0 * PI, theta = v * PI, st = std::sin(theta);
        V3 dir{st * std::sin(phi), std::cos(theta), -st * std::cos(phi)};
        *rad = texel(x, y);
        *pdf_out = pdf(dir);
        return dir;
    }
};

// ies.rs: an LM-63 candela grid and its sin-weighted mean candela.
struct Ies {
    std::vector<double> v, h;   // angles in degrees, ascending
    std::vector<double> cd;     // cd[hi * n_v + vi]
    double average = 1.0;
    M4 to_local;                // world -> light (upper 3x3 used)

    void finish() {  // ies.rs:67-80
        double num = 0.0, den = 0.0;
        for (size_t vi = 0; vi < v.size(); vi++) {
            double w = std::fmax(std::sin(v[vi] * PI / 180.0), 1e-4), mean = 0.0;
            for (size_t hi = 0; hi < h.size(); hi++) mean += cd[hi * v.size() + vi];
            num += mean / (double)h.size() * w;
            den += w;
        }
        average = std::fmax(num / std::fmax(den, 1e-9), 1e-9);
    }
    static void axis(const std::vector<double>& a, double x, size_t* i0, size_t* i1, double* t) {  // ies.rs:89-106
        *t = 0.0;
        if (x <= a[0]) {
            *i0 = *i1 = 0;
            return;
        }
        if (x >= a.back()) {
            *i0 = *i1 = a.size() - 1;
            return;
        }
        for (size_t i = 0; i + 1 < a.size(); i++)
            if (x <= a[i + 1]) {
                *i0 = i;
                *i1 = i + 1;
                *t = (x - a[i]) / std::fmax(a[i + 1] - a[i], 1e-9);
                return;
            }
        *i0 = *i1 = a.size() - 1;
    }
    double candela(V3 dir_local) const {  // ies.rs:108-137
        V3 d = normalize(dir_local);
        double theta = std::acos(std::min(std::max(-d.y, -1.0), 1.0)) * 180.0 / PI;
        double phi = std::atan2(d.z, d.x) * 180.0 / PI;
        if (phi < 0.0) phi += 360.0;
        const double hmax = h.back();
        if (hmax <= 0.0) {
            phi = 0.0;
        } else if (hmax <= 90.0) {
            double q = std::fmod(phi, 180.0);
            phi = q > 90.0 ? 180.0 - q : q;
        } else if (hmax <= 180.0) {
            double q = std::fmod(phi, 360.0);
            phi = q > 180.0 ? 360.0 - q : q;
        }
        size_t v0, v1, h0, h1;
        double tv, th;
        axis(v, theta, &v0, &v1, &tv);
        axis(h, phi, &h0, &h1, &th);
        const size_t nv = v.size();
        const double c00 = cd[h0 * nv + v0], c01 = cd[h0 * nv + v1], c10 = cd[h1 * nv + v0], c11 = cd[h1 * nv + v1];
        return (c00 * (1.0 - tv) + c01 * tv) * (1.0 - th) + (c10 * (1.0 - tv) + c11 * tv) * th;
    }
    double factor(V3 dir_local) const { return candela(dir_local) / average; }
};

struct Light {
    int type;
    double intensity;
    V3 color, p, e1, e2, normal;
    double radius = 0, area = 0;
    std::shared_ptr<EnvMap> env;  // dome lights only
    std::shared_ptr<Ies> ies;     // point lights only
    V3 radiance() const { return color * intensity; }  // light.rs:151-153
    // light.rs:155-167: point lights with a profile reshape their output
    // toward the emission direction -wi.
    V3 radiance_toward(V3 wi) const {
        if (!ies) return radiance();
        return radiance() * ies->factor(xf_vec(ies->to_local, -wi));
    }
};

struct LightNode {  // light_sampler.rs:19-31 (f32 storage, 48 B)
    float mn[3];
    float power;
    float mx[3];
    uint32_t parent, a, b;
};

struct LightSampler {
    std::vector<LightNode> nodes;
    std::vector<uint32_t> light_leaf, infinite;
    std::vector<double> infinite_power;
    double infinite_total = 0, p_infinite = 0;

    static double lum_floor(V3 c) { return std::fmax(lum(c), 1e-9); }  // light_sampler.rs:45-47

    // light_sampler.rs:74-87
    static double importance(const LightNode& n, V3 p) {
        double cx = ((double)n.mn[0] + (double)n.mx[0]) * 0.5;
        double cy = ((double)n.mn[1] + (double)n.mx[1]) * 0.5;
        double cz = ((double)n.mn[2] + (double)n.mx[2]) * 0.5;
        double dx = p.x - cx, dy = p.y - cy, dz = p.z - cz;
        double d2 = dx * dx + dy * dy + dz * dz;
        double rx = (double)(n.mx[0] - n.mn[0]) * 0.5;
        double ry = (double)(n.mx[1] - n.mn[1]) * 0.5;
        double rz = (double)(n.mx[2] - n.mn[2]) * 0.5;
        double r2 = rx * rx + ry * ry + rz * rz;
        return (double)n.power / std::fmax(std::fmax(d2, r2), 1e-6);
    }

    struct Entry {
        uint32_t light;
        V3 center;
        double radius, power;
    };

    // light_sampler.rs:242-312 median split; stable sort as Rust's sort_by.
    uint32_t build_rec(const std::vector<Entry>& e, std::vector<size_t>& order, size_t start, size_t end,
                       uint32_t parent) {
        uint32_t index = (uint32_t)nodes.size();
        float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
        double power = 0;
        for (size_t k = start; k < end; k++) {
            const Entry& en = e[order[k]];
            double c[3] = {en.center.x, en.center.y, en.center.z};
            for (int a = 0; a < 3; a++) {
                mn[a] = std::fmin(mn[a], (float)(c[a] - en.radius));
                mx[a] = std::fmax(mx[a], (float)(c[a] + en.radius));
            }
            power += en.power;
        }
        LightNode nd{};
        for (int a = 0; a < 3; a++) {
            nd.mn[a] = mn[a];
            nd.mx[a] = mx[a];
        }
        nd.power = (float)power;
        nd.parent = parent;
        nd.a = 0;
        nd.b = 0xFFFFFFFFu;
        nodes.push_back(nd);
        if (end - start == 1) {
            uint32_t light = e[order[start]].light;
            nodes[index].a = light;
            light_leaf[light] = index;
            return index;
        }
        int axis = 0;
        float widest = -1.0f;
        for (int a = 0; a < 3; a++) {
            float w = mx[a] - mn[a];
            if (w > widest) {
                widest = w;
                axis = a;
            }
        }
        size_t mid = (start + end) / 2;
        std::stable_sort(order.begin() + start, order.begin() + end, [&](size_t x, size_t y) {
            return axis_of(e[x].center, axis) < axis_of(e[y].center, axis);
        });
        uint32_t a = build_rec(e, order, start, mid, index);
        uint32_t b = build_rec(e, order, mid, end, index);
        nodes[index].a = a;
        nodes[index].b = b;
        return index;
    }

    // light_sampler.rs:97-141
    void build(const std::vector<Light>& lights) {
        std::vector<Entry> finite;
        light_leaf.assign(lights.size(), 0xFFFFFFFFu);
        for (size_t i = 0; i < lights.size(); i++) {
            const Light& l = lights[i];
            double pw = lum_floor(l.radiance());
            switch (l.type) {
                case RT_LIGHT_POINT: finite.push_back({(uint32_t)i, l.p, 0.0, pw * 4.0 * PI}); break;
                case RT_LIGHT_RECT: {
                    V3 c = l.p + l.e1 * 0.5 + l.e2 * 0.5;
                    finite.push_back({(uint32_t)i, c, (length(l.e1) + length(l.e2)) * 0.5, pw * l.area * PI});
                    break;
                }
                case RT_LIGHT_SPHERE:
                    finite.push_back({(uint32_t)i, l.p, l.radius, pw * 4.0 * PI * l.radius * l.radius * PI});
                    break;
                case RT_LIGHT_DISK: finite.push_back({(uint32_t)i, l.p, length(l.e1), pw * l.area * PI}); break;
                default: {
                    // light_sampler.rs:104-118: env maps fold in their mean luminance
                    double base = l.env ? l.env->mean_luminance() * l.intensity : pw;
                    infinite.push_back((uint32_t)i);
                    infinite_power.push_back(base * 4.0 * PI);
                }
            }
        }
        infinite_total = 0;
        for (double w : infinite_power) infinite_total += w;
        if (!finite.empty()) {
            std::vector<size_t> order(finite.size());
            for (size_t i = 0; i < order.size(); i++) order[i] = i;
            build_rec(finite, order, 0, finite.size(), 0xFFFFFFFFu);
        }
        double finite_total = 0;
        for (auto& e : finite) finite_total += e.power;
        if (infinite.empty()) p_infinite = 0.0;
        else if (finite.empty()) p_infinite = 1.0;
        else p_infinite = std::min(std::max(infinite_total / (infinite_total + finite_total), 0.1), 0.9);
    }

    // light_sampler.rs:150-208
    bool sample(V3 p, double u, uint32_t* light, double* pmf_out) const {
        bool has_f = !nodes.empty(), has_i = !infinite.empty();
        if (!has_f && !has_i) return false;
        double pmf = 1.0;
        bool inf;
        if (has_f && has_i) {
            if (u < p_infinite) {
                u /= p_infinite;
                pmf *= p_infinite;
                inf = true;
            } else {
                u = (u - p_infinite) / (1.0 - p_infinite);
                pmf *= 1.0 - p_infinite;
                inf = false;
            }
        } else {
            inf = has_i;
        }
        if (inf) {
            double acc = 0.0, target = u * infinite_total;
            for (size_t k = 0; k < infinite_power.size(); k++) {
                acc += infinite_power[k];
                if (target <= acc || k == infinite.size() - 1) {
                    *light = infinite[k];
                    *pmf_out = pmf * infinite_power[k] / std::fmax(infinite_total, 1e-12);
                    return true;
                }
            }
            return false;
        }
        size_t node = 0;
        for (;;) {
            const LightNode& nd = nodes[node];
            if (nd.b == 0xFFFFFFFFu) {
                *light = nd.a;
                *pmf_out = pmf;
                return true;
            }
            double ia = importance(nodes[nd.a], p), ib = importance(nodes[nd.b], p);
            double total = ia + ib;
            double pa = total > 1e-30 ? ia / total : 0.5;
            if (u < pa) {
                u = std::fmin(u / pa, 1.0 - 1e-12);
                pmf *= pa;
                node = nd.a;
            } else {
                u = std::fmin((u - pa) / (1.0 - pa), 1.0 - 1e-12);
                pmf *= 1.0 - pa;
                node = nd.b;
            }
        }
    }

    // light_sampler.rs:212-238
    double pmf(V3 p, uint32_t light) const {
        bool has_f = !nodes.empty(), has_i = !infinite.empty();
        for (size_t k = 0; k < infinite.size(); k++)
            if (infinite[k] == light) {
                double group = has_f ? p_infinite : 1.0;
                return group * infinite_power[k] / std::fmax(infinite_total, 1e-12);
            }
        uint32_t leaf = light < light_leaf.size() ? light_leaf[light] : 0xFFFFFFFFu;
        if (leaf == 0xFFFFFFFFu) return 0.0;
        double pmf = has_i ? 1.0 - p_infinite : 1.0;
        uint32_t node = leaf;
        while (nodes[node].parent != 0xFFFFFFFFu) {
            uint32_t parent = nodes[node].parent;
            const LightNode& pn = nodes[parent];
            double ia = importance(nodes[pn.a], p), ib = importance(nodes[pn.b], p);
            double total = ia + ib;
            double mine = node == pn.a ? ia : ib;
            pmf *= total > 1e-30 ? mine / total : 0.5;
            node = parent;
        }
        return pmf;
    }
};

// ---- materials (src/scene/pbr.rs, material.rs) ----------------------------

struct Pbr {
    double diffuse_gain;
    V3 diffuse_color;
    double diffuse_roughness;
    V3 spec_face, spec_edge;
    double spec_rough, spec_ior;
    double cc_gain, cc_rough;
    double fuzz_gain;
    V3 fuzz_color;
    double glass_gain, glass_ior, glass_rough;
    V3 refraction_color, glow;
    double presence;
    double subsurface_gain = 0.0;
    V3 subsurface_color, subsurface_dmfp;
    V3 hair_sigma_a;
    double hair_beta_m = 0.3, hair_beta_n = 0.3, hair_eta = 1.55;
    // Material fields
    V3 emission;
    int32_t area_light;
    uint32_t id;
    int32_t interior = -1;  // Material::interior (material.rs:35-37), -1 for none
    bool hair = false;      // Material::hair (Marschner on curve hits)

    static Pbr from(const rt_material_desc& m) {
        Pbr p;
        p.diffuse_gain = m.diffuse_gain;
        p.diffuse_color = v3(m.diffuse_color);
        p.diffuse_roughness = m.diffuse_roughness;
        p.spec_face = v3(m.specular_face_color);
        p.spec_edge = v3(m.specular_edge_color);
        p.spec_rough = m.specular_roughness;
        p.spec_ior = m.specular_ior;
        p.cc_gain = m.clearcoat_gain;
        p.cc_rough = m.clearcoat_roughness;
        p.fuzz_gain = m.fuzz_gain;
        p.fuzz_color = v3(m.fuzz_color);
        p.glass_gain = m.glass_gain;
        p.glass_ior = m.glass_ior;
        p.glass_rough = m.glass_roughness;
        p.refraction_color = v3(m.refraction_color);
        p.glow = v3(m.glow);
        p.presence = m.presence;
        p.emission = v3(m.emission);
        p.area_light = m.area_light;
        p.id = m.id;
        p.subsurface_gain = m.subsurface_gain;
        p.subsurface_color = v3(m.subsurface_color);
        p.subsurface_dmfp = v3(m.subsurface_dmfp);
        p.interior = m.interior;
        p.hair = m.hair != 0;
        p.hair_sigma_a = v3(m.hair_sigma_a);
        p.hair_beta_m = m.hair_beta_m;
        p.hair_beta_n = m.hair_beta_n;
        p.hair_eta = m.hair_eta;
        return p;
    }
    // pbr.rs:86-96
    V3 specular_f0() const {
        if (lum(spec_face) > 1e-6) return spec_face;
        if (spec_ior > 1.0) {
            double r = (spec_ior - 1.0) / (spec_ior + 1.0);
            return V3{1, 1, 1} * (r * r);
        }
        return {0, 0, 0};
    }
    bool has_specular() const { return lum(specular_f0()) > 1e-6; }  // pbr.rs:100-102
    // BoundField::apply (pattern.rs:278-296): scalars take channel 0.
    void apply(uint32_t field, V3 v) {
        switch (field) {
            case RT_FIELD_DIFFUSE_COLOR: diffuse_color = v; break;
            case RT_FIELD_DIFFUSE_GAIN: diffuse_gain = v.x; break;
            case RT_FIELD_DIFFUSE_ROUGHNESS: diffuse_roughness = v.x; break;
            case RT_FIELD_SPECULAR_FACE_COLOR: spec_face = v; break;
            case RT_FIELD_SPECULAR_EDGE_COLOR: spec_edge = v; break;
            case RT_FIELD_SPECULAR_ROUGHNESS: spec_rough = std::min(std::max(v.x, 0.005), 1.0); break;
            case RT_FIELD_CLEARCOAT_GAIN: cc_gain = v.x; break;
            case RT_FIELD_FUZZ_GAIN: fuzz_gain = v.x; break;
            case RT_FIELD_FUZZ_COLOR: fuzz_color = v; break;
            case RT_FIELD_GLASS_GAIN: glass_gain = v.x; break;
            case RT_FIELD_GLASS_ROUGHNESS: glass_rough = std::min(std::max(v.x, 0.005), 1.0); break;
            case RT_FIELD_REFRACTION_COLOR: refraction_color = v; break;
            case RT_FIELD_GLOW: glow = v; break;
            case RT_FIELD_PRESENCE: presence = std::min(std::max(v.x, 0.0), 1.0); break;
            default: break;
        }
    }
    // pbr.rs:188-201
    bool lobe_weights(double w[5]) const {
        double wd = diffuse_gain * lum(diffuse_color);
        double ws = std::sqrt(lum(specular_f0()));
        double wc = cc_gain * 0.2;
        double wf = fuzz_gain * lum(fuzz_color) * 0.3;
        double wg = glass_gain;
        double total = wd + ws + wc + wf + wg;
        if (total <= 1e-9) return false;
        w[0] = wd / total;
        w[1] = ws / total;
        w[2] = wc / total;
        w[3] = wf / total;
        w[4] = wg / total;
        return true;
    }
};

// ---- BSDF (src/raytracer/pt/bxdf.rs) ---------------------------------------

struct Frame {  // bxdf.rs:16-39
    V3 t, b, n;
    explicit Frame(V3 nn) : n(nn) {
        V3 t0 = std::fabs(n.x) > 0.9 ? V3{0, 1, 0} : V3{1, 0, 0};
        t = normalize(cross(n, t0));
        b = cross(n, t);
    }
    V3 to_local(V3 w) const { return {dot(w, t), dot(w, b), dot(w, n)}; }
    V3 to_world(V3 w) const { return t * w.x + b * w.y + n * w.z; }
};

static V3 schlick(V3 f0, V3 f90, double c) {  // bxdf.rs:57-60
    double m = std::pow(std::min(std::max(1.0 - c, 0.0), 1.0), 5);
    return f0 + (f90 - f0) * m;
}
double fresnel_dielectric(double cos_i, double eta) {  // bxdf.rs:63-73
    cos_i = std::min(std::max(cos_i, 0.0), 1.0);
    double sin2_t = (1.0 - cos_i * cos_i) / (eta * eta);
    if (sin2_t >= 1.0) return 1.0;
    double cos_t = std::sqrt(1.0 - sin2_t);
    double r_par = (eta * cos_i - cos_t) / (eta * cos_i + cos_t);
    double r_perp = (cos_i - eta * cos_t) / (cos_i + eta * cos_t);
    return 0.5 * (r_par * r_par + r_perp * r_perp);
}
static double ggx_d(V3 h, double alpha) {  // bxdf.rs:77-84
    if (h.z <= 0.0) return 0.0;
    double a2 = alpha * alpha;
    double d = h.z * h.z * (a2 - 1.0) + 1.0;
    return a2 / (PI * d * d);
}
static double ggx_lambda(V3 w, double alpha) {  // bxdf.rs:86-93
    double cos2 = w.z * w.z;
    if (cos2 <= 0.0) return 0.0;
    double tan2 = std::fmax(1.0 - cos2, 0.0) / cos2;
    return (std::sqrt(1.0 + alpha * alpha * tan2) - 1.0) * 0.5;
}
static double ggx_g1(V3 w, double a) { return 1.0 / (1.0 + ggx_lambda(w, a)); }
static double ggx_g2(V3 wo, V3 wi, double a) { return 1.0 / (1.0 + ggx_lambda(wo, a) + ggx_lambda(wi, a)); }
// bxdf.rs:104-123 Heitz 2018 VNDF sampling.
static V3 ggx_sample_vndf(V3 wo, double alpha, double u1, double u2) {
    V3 v = normalize(V3{alpha * wo.x, alpha * wo.y, wo.z});
    double lensq = v.x * v.x + v.y * v.y;
    V3 t1 = lensq > 1e-12 ? V3{-v.y, v.x, 0.0} / std::sqrt(lensq) : V3{1, 0, 0};
    V3 t2 = cross(v, t1);
    double r = std::sqrt(u1), phi = 2.0 * PI * u2;
    double p1 = r * std::cos(phi), p2 = r * std::sin(phi);
    double s = 0.5 * (1.0 + v.z);
    p2 = (1.0 - s) * std::sqrt(std::fmax(1.0 - p1 * p1, 0.0)) + s * p2;
    V3 nh = t1 * p1 + t2 * p2 + v * std::sqrt(std::fmax(1.0 - p1 * p1 - p2 * p2, 0.0));
    return normalize(V3{alpha * nh.x, alpha * nh.y, std::fmax(nh.z, 1e-9)});
}
static double ggx_pdf_h(V3 wo, V3 h, double alpha) {  // bxdf.rs:126-132
    double odh = dot(wo, h);
    if (odh <= 0.0 || wo.z <= 0.0) return 0.0;
    return ggx_g1(wo, alpha) * odh * ggx_d(h, alpha) / wo.z;
}
static double under_layer_scale(const Pbr& p) {  // bxdf.rs:137-143
    V3 f0 = p.specular_f0();
    double spec_take = 0.2126 * f0.x + 0.7152 * f0.y + 0.0722 * f0.z;
    double coat_take = 0.04 * p.cc_gain;
    return std::min(std::max((1.0 - spec_take) * (1.0 - coat_take), 0.0), 1.0);
}
static V3 eval_diffuse(const Pbr& p, V3 wo, V3 wi) {  // bxdf.rs:145-165
    double sigma2 = p.diffuse_roughness * p.diffuse_roughness;
    double a = 1.0 - sigma2 / (2.0 * (sigma2 + 0.33));
    double b = 0.45 * sigma2 / (sigma2 + 0.09);
    double sin_o = std::sqrt(std::fmax(1.0 - wo.z * wo.z, 0.0));
    double sin_i = std::sqrt(std::fmax(1.0 - wi.z * wi.z, 0.0));
    double cos_dphi = 0.0;
    if (sin_o > 1e-6 && sin_i > 1e-6)
        cos_dphi = std::min(std::max((wo.x * wi.x + wo.y * wi.y) / (sin_o * sin_i), -1.0), 1.0);
    double sin_a, tan_b;
    if (wo.z < wi.z) {
        sin_a = sin_o;
        tan_b = sin_i / std::fmax(wi.z, 1e-6);
    } else {
        sin_a = sin_i;
        tan_b = sin_o / std::fmax(wo.z, 1e-6);
    }
    return p.diffuse_color * (p.diffuse_gain * under_layer_scale(p) / PI) *
           (a + b * std::fmax(cos_dphi, 0.0) * sin_a * tan_b);
}
static V3 eval_fuzz(const Pbr& p, V3 wo, V3 wi) {  // bxdf.rs:167-171
    double rim = 0.5 * (std::pow(1.0 - wi.z, 4) + std::pow(1.0 - wo.z, 4));
    return p.fuzz_color * (p.fuzz_gain / PI) * rim;
}
static V3 eval_spec(V3 f0, V3 f90, double alpha, V3 wo, V3 wi) {  // bxdf.rs:173-179
    V3 h = normalize(wo + wi);
    double d = ggx_d(h, alpha), g = ggx_g2(wo, wi, alpha);
    V3 f = schlick(f0, f90, std::fmax(dot(wo, h), 0.0));
    return f * (d * g / std::fmax(4.0 * wo.z * wi.z, 1e-9));
}
static double spec_pdf(V3 wo, V3 wi, double alpha) {  // bxdf.rs:181-185
    V3 h = normalize(wo + wi);
    double odh = std::fmax(dot(wo, h), 1e-9);
    return ggx_pdf_h(wo, h, alpha) / (4.0 * odh);
}
static double alpha_of(double r) { return std::min(std::max(r * r, 2.5e-5), 1.0); }  // bxdf.rs:187-189

// bxdf.rs:193-232
static V3 glass_transmit(const Pbr& p, V3 wo, V3 wi, double eta, double* pdf) {
    double alpha = alpha_of(p.glass_rough);
    V3 h = normalize(wo + wi * eta);
    if (h.z < 0.0) h = -h;
    double odh = dot(wo, h), idh = dot(wi, h);
    *pdf = 0.0;
    if (odh <= 0.0 || idh >= 0.0) return {0, 0, 0};
    double fres = fresnel_dielectric(odh, eta);
    double d = ggx_d(h, alpha);
    double g = ggx_g2(wo, V3{wi.x, wi.y, -wi.z}, alpha);
    double sqrt_denom = odh + eta * idh;
    if (std::fabs(sqrt_denom) < 1e-9) return {0, 0, 0};
    double factor = 1.0 / (eta * eta);
    V3 f = p.refraction_color * (p.glass_gain * under_layer_scale(p) * (1.0 - fres) * d * g * factor *
                                 std::fabs(idh * odh / (wi.z * wo.z)) * (eta * eta) / (sqrt_denom * sqrt_denom));
    double dwh_dwi = std::fabs(eta * eta * idh) / (sqrt_denom * sqrt_denom);
    *pdf = ggx_pdf_h(wo, h, alpha) * dwh_dwi;
    return f;
}

// bxdf.rs:241-299
static void eval_pdf(const Pbr& p, V3 wo, V3 wi, double eta, V3* f_out, double* pdf_out) {
    double w[5];
    *f_out = {0, 0, 0};
    *pdf_out = 0.0;
    if (!p.lobe_weights(w)) return;
    double wd = w[0], ws = w[1], wc = w[2], wf = w[3], wg = w[4];
    if (wi.z > 0.0) {
        V3 f{0, 0, 0};
        double pdf = 0.0, cos_pdf = wi.z / PI;
        if (wd > 0.0) {
            f = f + eval_diffuse(p, wo, wi);
            pdf += wd * cos_pdf;
        }
        if (wf > 0.0) {
            f = f + eval_fuzz(p, wo, wi);
            pdf += wf * cos_pdf;
        }
        if (ws > 0.0) {
            double a = alpha_of(p.spec_rough);
            f = f + eval_spec(p.specular_f0(), p.spec_edge, a, wo, wi);
            pdf += ws * spec_pdf(wo, wi, a);
        }
        if (wc > 0.0) {
            double a = alpha_of(p.cc_rough);
            V3 f0 = V3{0.04, 0.04, 0.04} * p.cc_gain;
            f = f + eval_spec(f0, V3{1, 1, 1} * p.cc_gain, a, wo, wi);
            pdf += wc * spec_pdf(wo, wi, a);
        }
        if (wg > 0.0) {
            double a = alpha_of(p.glass_rough);
            V3 h = normalize(wo + wi);
            double fres = fresnel_dielectric(std::fmax(dot(wo, h), 0.0), eta);
            double d = ggx_d(h, a), g = ggx_g2(wo, wi, a);
            f = f + V3{1, 1, 1} * (p.glass_gain * under_layer_scale(p) * fres * d * g /
                                   std::fmax(4.0 * wo.z * wi.z, 1e-9));
            pdf += wg * fres * spec_pdf(wo, wi, a);
        }
        *f_out = f;
        *pdf_out = pdf;
    } else {
        if (wg <= 0.0) return;
        double pdf_lobe;
        V3 f = glass_transmit(p, wo, wi, eta, &pdf_lobe);
        V3 h = normalize(wo + wi * eta);
        if (h.z < 0.0) h = -h;
        double fres = fresnel_dielectric(std::fmax(dot(wo, h), 0.0), eta);
        *f_out = f;
        *pdf_out = wg * (1.0 - fres) * pdf_lobe;
    }
}

struct BsdfSample {
    bool specular_lobe, transmitted;
    V3 wi, f;
    double pdf;
};

static V3 cosine_sample(Pcg32& rng) {  // bxdf.rs:301-306
    double u = rng.next_f64(), v = rng.next_f64();
    double r = std::sqrt(u), phi = 2.0 * PI * v;
    return {r * std::cos(phi), r * std::sin(phi), std::sqrt(std::fmax(1.0 - u, 0.0))};
}

// bxdf.rs:309-374
static bool sample_bsdf(const Pbr& p, V3 wo, double eta, Pcg32& rng, BsdfSample* s) {
    double w[5];
    if (!p.lobe_weights(w)) return false;
    double wd = w[0], ws = w[1], wc = w[2], wf = w[3], wg = w[4];
    double pick = rng.next_f64();
    bool transmitted = false;
    bool specular_lobe = pick >= wd + wf;
    V3 wi;
    if (pick < wd + wf) {
        wi = cosine_sample(rng);
    } else if (pick < wd + wf + ws) {
        double a = alpha_of(p.spec_rough);
        double u1 = rng.next_f64(), u2 = rng.next_f64();
        V3 h = ggx_sample_vndf(wo, a, u1, u2);
        wi = reflect(-wo, h);
        if (wi.z <= 0.0) return false;
    } else if (pick < wd + wf + ws + wc) {
        double a = alpha_of(p.cc_rough);
        double u1 = rng.next_f64(), u2 = rng.next_f64();
        V3 h = ggx_sample_vndf(wo, a, u1, u2);
        wi = reflect(-wo, h);
        if (wi.z <= 0.0) return false;
    } else if (wg > 0.0) {
        double a = alpha_of(p.glass_rough);
        double u1 = rng.next_f64(), u2 = rng.next_f64();
        V3 h = ggx_sample_vndf(wo, a, u1, u2);
        double fres = fresnel_dielectric(std::fmax(dot(wo, h), 0.0), eta);
        if (rng.next_f64() < fres) {
            wi = reflect(-wo, h);
            if (wi.z <= 0.0) return false;
        } else {
            double cos_i = dot(wo, h);
            double sin2_t = (1.0 - cos_i * cos_i) / (eta * eta);
            if (sin2_t >= 1.0) return false;
            double cos_t = std::sqrt(1.0 - sin2_t);
            wi = normalize((-wo) / eta + h * (cos_i / eta - cos_t));
            if (wi.z >= 0.0) return false;
            transmitted = true;
        }
    } else {
        return false;
    }
    V3 f;
    double pdf;
    eval_pdf(p, wo, wi, eta, &f, &pdf);
    if (pdf <= 0.0) return false;
    s->wi = wi;
    s->f = f;
    s->pdf = pdf;
    s->transmitted = transmitted;
    s->specular_lobe = specular_lobe;
    return true;
}

// ---- hair (src/raytracer/pt/hair.rs) --------------------------------------
// Marschner / d'Eon / pbrt-v3 hair: R, TT, TRT lobes and a residual, in the
// fiber frame (x along the fiber); f is per solid angle with no cosine.
static const int HAIR_PMAX = 3;

struct HairParams {  // hair.rs:24-55
    V3 sigma_a;
    double beta_m = 0.3, beta_n = 0.3, eta = 1.55;
    double v[HAIR_PMAX + 1] = {0, 0, 0, 0};
    double s = 0.0;
    void init(V3 sa, double bm, double bn, double e) {
        sigma_a = sa;
        beta_m = std::min(std::max(bm, 0.01), 1.0);
        beta_n = std::min(std::max(bn, 0.01), 1.0);
        eta = e;
        double v0 = 0.726 * beta_m + 0.812 * beta_m * beta_m + 3.7 * std::pow(beta_m, 20);
        v0 *= v0;
        v[0] = v0;
        v[1] = 0.25 * v0;
        v[2] = 4.0 * v0;
        v[3] = 4.0 * v0;
        s = 0.626657069 * (0.265 * beta_n + 1.194 * beta_n * beta_n + 5.372 * std::pow(beta_n, 22));
    }
};

static double hair_i0(double x) {  // hair.rs:104-118 (series to 10 terms)
    double val = 0.0, x2i = 1.0, ifact = 1.0, i4 = 1.0;
    for (int i = 0; i < 10; i++) {
        if (i > 1) ifact *= i;
        val += x2i / (i4 * ifact * ifact);
        x2i *= x * x;
        i4 *= 4.0;
    }
    return val;
}
static double hair_log_i0(double x) {  // hair.rs:120-126
    if (x > 12.0) return x + 0.5 * (-std::log(2.0 * PI * x) + 1.0 / (8.0 * x));
    return std::log(hair_i0(x));
}
// hair.rs:129-137: energy-conserving longitudinal lobe.
static double hair_mp(double cos_ti, double cos_to, double sin_ti, double sin_to, double v) {
    double a = cos_ti * cos_to / v, b = sin_ti * sin_to / v;
    if (v <= 0.1) return std::exp(hair_log_i0(a) - b - 1.0 / v + 0.6931 + std::log(1.0 / (2.0 * v)));
    return std::exp(-b) * hair_i0(a) / (std::sinh(1.0 / v) * 2.0 * v);
}
static double hair_fr(double cos_i, double eta_i, double eta_t) {  // hair.rs:139-157
    cos_i = std::min(std::max(cos_i, -1.0), 1.0);
    if (cos_i <= 0.0) {
        std::swap(eta_i, eta_t);
        cos_i = -cos_i;
    }
    double sin_i = std::sqrt(std::fmax(1.0 - cos_i * cos_i, 0.0));
    double sin_t = eta_i / eta_t * sin_i;
    if (sin_t >= 1.0) return 1.0;
    double cos_t = std::sqrt(std::fmax(1.0 - sin_t * sin_t, 0.0));
    double rpa = (eta_t * cos_i - eta_i * cos_t) / (eta_t * cos_i + eta_i * cos_t);
    double rpe = (eta_i * cos_i - eta_t * cos_t) / (eta_i * cos_i + eta_t * cos_t);
    return (rpa * rpa + rpe * rpe) / 2.0;
}
// hair.rs:160-183: attenuation per lobe, then the residual's geometric series.
static void hair_ap(double cos_to, double eta, double h, V3 t, V3 out[HAIR_PMAX + 1]) {
    double cos_gamma_o = std::sqrt(std::fmax(1.0 - h * h, 0.0));
    double f = hair_fr(cos_to * cos_gamma_o, 1.0, eta);
    out[0] = V3{f, f, f};
    out[1] = t * ((1.0 - f) * (1.0 - f));
    for (int p = 2; p < HAIR_PMAX; p++) out[p] = out[p - 1] * t * f;
    V3 last = out[HAIR_PMAX - 1];
    out[HAIR_PMAX] = V3{last.x * f * t.x / std::fmax(1.0 - t.x * f, 1e-6), last.y * f * t.y / std::fmax(1.0 - t.y * f, 1e-6),
                        last.z * f * t.z / std::fmax(1.0 - t.z * f, 1e-6)};
}
static double hair_logistic(double x, double s) {  // hair.rs:185-189
    x = std::fabs(x);
    double e = std::exp(-x / s);
    return e / (s * (1.0 + e) * (1.0 + e));
}
static double hair_logistic_cdf(double x, double s) { return 1.0 / (1.0 + std::exp(-x / s)); }
static double hair_trimmed_logistic(double x, double s, double a, double b) {
    return hair_logistic(x, s) / (hair_logistic_cdf(b, s) - hair_logistic_cdf(a, s));
}
static double hair_sample_trimmed_logistic(double u, double s, double a, double b) {  // hair.rs:199-203
    double k = hair_logistic_cdf(b, s) - hair_logistic_cdf(a, s);
    double x = -s * std::log(1.0 / std::min(std::max(u * k + hair_logistic_cdf(a, s), 1e-9), 1.0 - 1e-9) - 1.0);
    return std::min(std::max(x, a), b);
}
static double hair_phi(int p, double gamma_o, double gamma_t) { return 2.0 * p * gamma_t - 2.0 * gamma_o + p * PI; }
static double hair_np(double phi, int p, double s, double gamma_o, double gamma_t) {  // hair.rs:211-220
    double dphi = phi - hair_phi(p, gamma_o, gamma_t);
    while (dphi > PI) dphi -= 2.0 * PI;
    while (dphi < -PI) dphi += 2.0 * PI;
    return hair_trimmed_logistic(dphi, s, -PI, PI);
}
struct HairGeom {  // hair.rs:224-258
    double sin_to, cos_to, phi_o, gamma_o, gamma_t;
    V3 t;
};
static HairGeom hair_geom(const HairParams& hp, V3 wo, double h) {
    HairGeom g;
    g.sin_to = std::min(std::max(wo.x, -1.0), 1.0);
    g.cos_to = std::sqrt(std::fmax(1.0 - g.sin_to * g.sin_to, 0.0));
    g.phi_o = std::atan2(wo.z, wo.y);
    g.gamma_o = std::asin(std::min(std::max(h, -1.0), 1.0));
    double sin_tt = g.sin_to / hp.eta;
    double cos_tt = std::sqrt(std::fmax(1.0 - sin_tt * sin_tt, 0.0));
    double etap = std::sqrt(std::fmax(hp.eta * hp.eta - g.sin_to * g.sin_to, 0.0)) / std::fmax(g.cos_to, 1e-9);
    double sin_gt = std::min(std::max(h / etap, -1.0), 1.0);
    double cos_gt = std::sqrt(std::fmax(1.0 - sin_gt * sin_gt, 0.0));
    g.gamma_t = std::asin(sin_gt);
    double l = 2.0 * cos_gt / std::fmax(cos_tt, 1e-9);
    g.t = exp3(hp.sigma_a, l);
    return g;
}
static V3 hair_f(const HairParams& hp, V3 wo, V3 wi, double h) {  // hair.rs:262-281
    HairGeom g = hair_geom(hp, wo, h);
    double sin_ti = std::min(std::max(wi.x, -1.0), 1.0);
    double cos_ti = std::sqrt(std::fmax(1.0 - sin_ti * sin_ti, 0.0));
    double phi = std::atan2(wi.z, wi.y) - g.phi_o;
    V3 a[HAIR_PMAX + 1];
    hair_ap(g.cos_to, hp.eta, h, g.t, a);
    V3 out{0, 0, 0};
    for (int p = 0; p <= HAIR_PMAX; p++) {
        double m = hair_mp(cos_ti, g.cos_to, sin_ti, g.sin_to, hp.v[p]);
        double n = p < HAIR_PMAX ? hair_np(phi, p, hp.s, g.gamma_o, g.gamma_t) : 1.0 / (2.0 * PI);
        out = out + a[p] * (m * n);
    }
    return out;
}
static void hair_ap_pdf(const HairParams& hp, const HairGeom& g, double h, double w[HAIR_PMAX + 1]) {  // :284-302
    V3 a[HAIR_PMAX + 1];
    hair_ap(g.cos_to, hp.eta, h, g.t, a);
    double total = 0.0;
    for (int p = 0; p <= HAIR_PMAX; p++) total += (w[p] = lum(a[p]));
    if (total > 1e-12) {
        for (int p = 0; p <= HAIR_PMAX; p++) w[p] /= total;
    } else {
        for (int p = 0; p <= HAIR_PMAX; p++) w[p] = p == 0 ? 1.0 : 0.0;
    }
}
static double hair_pdf(const HairParams& hp, V3 wo, V3 wi, double h) {  // hair.rs:305-324
    HairGeom g = hair_geom(hp, wo, h);
    double sin_ti = std::min(std::max(wi.x, -1.0), 1.0);
    double cos_ti = std::sqrt(std::fmax(1.0 - sin_ti * sin_ti, 0.0));
    double phi = std::atan2(wi.z, wi.y) - g.phi_o;
    double w[HAIR_PMAX + 1];
    hair_ap_pdf(hp, g, h, w);
    double out = 0.0;
    for (int p = 0; p <= HAIR_PMAX; p++) {
        double m = hair_mp(cos_ti, g.cos_to, sin_ti, g.sin_to, hp.v[p]);
        double n = p < HAIR_PMAX ? hair_np(phi, p, hp.s, g.gamma_o, g.gamma_t) : 1.0 / (2.0 * PI);
        out += w[p] * m * n;
    }
    return std::fmax(out, 0.0);
}
// hair.rs:327-374: lobe by attenuation energy, d'Eon's longitudinal
// inverse, trimmed-logistic azimuth; false when the pdf vanishes.
template <class R>
static bool hair_sample(const HairParams& hp, V3 wo, double h, R& rng, V3* wi_out, V3* f_out, double* pdf_out) {
    HairGeom g = hair_geom(hp, wo, h);
    double w[HAIR_PMAX + 1];
    hair_ap_pdf(hp, g, h, w);
    double u = rng.next_f64();
    int p = HAIR_PMAX;
    for (int i = 0; i <= HAIR_PMAX; i++) {
        if (u < w[i]) {
            p = i;
            break;
        }
        u -= w[i];
    }
    double v = hp.v[p];
    double u1 = std::fmax(rng.next_f64(), 1e-9);
    double u2 = rng.next_f64();
    double cos_theta = 1.0 + v * std::log(u1 + (1.0 - u1) * std::exp(-2.0 / v));
    double sin_theta = std::sqrt(std::fmax(1.0 - cos_theta * cos_theta, 0.0));
    double cos_phi_l = std::cos(2.0 * PI * u2);
    double sin_ti = -cos_theta * g.sin_to + sin_theta * cos_phi_l * g.cos_to;
    double cos_ti = std::sqrt(std::fmax(1.0 - sin_ti * sin_ti, 0.0));
    double u3 = rng.next_f64();
    double dphi = p < HAIR_PMAX ? hair_phi(p, g.gamma_o, g.gamma_t) + hair_sample_trimmed_logistic(u3, hp.s, -PI, PI)
                                : 2.0 * PI * u3;
    double phi_i = g.phi_o + dphi;
    V3 wi{sin_ti, cos_ti * std::cos(phi_i), cos_ti * std::sin(phi_i)};
    double pdf = hair_pdf(hp, wo, wi, h);
    if (pdf <= 1e-12) return false;
    *wi_out = wi;
    *f_out = hair_f(hp, wo, wi, h);
    *pdf_out = pdf;
    return true;
}
struct FiberFrame {  // hair.rs:378-411
    V3 x, y, z;
    double h;
    FiberFrame(V3 tangent, V3 n, V3 wo) {
        x = normalize(tangent);
        V3 zz = wo - x * dot(wo, x);
        if (length_sq(zz) < 1e-12) zz = n - x * dot(n, x);
        z = normalize(zz);
        y = normalize(cross(z, x));
        V3 n_perp = normalize(n - x * dot(n, x));
        h = std::min(std::max(dot(n_perp, y), -1.0), 1.0);
    }
    V3 to_local(V3 w) const { return {dot(w, x), dot(w, y), dot(w, z)}; }
    V3 to_world(V3 w) const { return x * w.x + y * w.y + z * w.z; }
};

// ---- scene ------------------------------------------------------------------

struct Camera {
    uint32_t width, height;
    double fov;
    V3 eye, forward, up, right;
    double lens_radius, focal_distance;
    int filter;
    double filter_width;
    int projection = RT_PROJECTION_PERSPECTIVE;  // camera.rs:5-9
    double ortho_half[2] = {1.0, 1.0};           // camera.rs:82-83
    bool moving = false;  // camera.rs:87-92 motion_inv present
    M4 motion_inv;

    // camera.rs:134-146 Camera::apply_motion: lerp(I, motion_inv, t) applied
    // to the ray, direction renormalised.
    Ray apply_motion(Ray r) const {
        if (!moving || !(r.time > 0.0)) return r;
        const M4 m = lerp(identity(), motion_inv, r.time);
        return {xf_point(m, r.o), normalize(xf_vec(m, r.d)), r.time};
    }

    double sample_1d(double u) const {  // camera.rs:36-61
        switch (filter) {
            case RT_FILTER_TRIANGLE: {
                double half = filter_width * 0.5;
                return u < 0.5 ? (std::sqrt(2.0 * u) - 1.0) * half : (1.0 - std::sqrt(2.0 * (1.0 - u))) * half;
            }
            case RT_FILTER_GAUSSIAN: {
                double u1 = std::fmax(u, 1e-12);
                double x = u * 2654435761.0;
                double u2 = x - std::trunc(x);
                double sigma = filter_width / 4.0;
                double g = std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * PI * u2);
                return std::min(std::max(g * sigma, -filter_width * 0.5), filter_width * 0.5);
            }
            default: return (u - 0.5) * filter_width;
        }
    }
    // camera.rs:150-179: orthographic rays start on the screen window and
    // ignore the lens; perspective rays through the thin lens.
    Ray generate(double px, double py, double lu, double lv) const {
        double u = (px / (double)width) * 2.0 - 1.0;
        double v = 1.0 - (py / (double)height) * 2.0;
        if (projection == RT_PROJECTION_ORTHOGRAPHIC)
            return make_ray(eye + right * (u * ortho_half[0]) + up * (v * ortho_half[1]), forward);
        double aspect = (double)width / (double)height;
        double half_h = std::tan(fov * PI / 180.0 / 2.0);
        double half_w = aspect * half_h;
        V3 dir = forward + right * (u * half_w) + up * (v * half_h);
        if (lens_radius <= 0.0) return make_ray(eye, dir);
        double r = lens_radius * std::sqrt(lu), phi = 2.0 * PI * lv;
        V3 off = right * (r * std::cos(phi)) + up * (r * std::sin(phi));
        V3 focus = eye + dir * focal_distance;
        V3 origin = eye + off;
        return make_ray(origin, focus - origin);
    }
};

struct Scene {
    std::vector<Mesh> meshes;
    std::vector<CurveSet> curve_sets;
    std::vector<Instance> instances;
    std::vector<Quadric> quadrics;
    std::vector<Pbr> materials;
    std::vector<Light> lights;
    LightSampler ls;
    Bvh tlas;
    Camera cam;
    V3 background;
    bool any_presence = false;
    std::vector<PatNode> patterns;
    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> bindings;  // per material: (field, node)
    std::vector<Texture> textures;
    std::vector<Medium> media;  // Scene::media
    int32_t atmosphere = -1;     // Scene::atmosphere
    bool has_motion = false;     // scene/mod.rs:42-44: rays draw a shutter time

    // A volume hull (pt/mod.rs:662-667, 1280-1284): an interior medium, no
    // lobes, no emission -- the surface only bounds the medium.
    bool is_hull(uint32_t material_id) const {
        const Pbr& m = materials[material_id];
        double w[5];
        return m.interior >= 0 && !m.hair && !m.lobe_weights(w) && max_comp(m.emission + m.glow) <= 0.0;
    }

    // shade_params (pt/mod.rs:389-439): the material with its pattern
    // outputs substituted; footprint = cone width x st density, and the ray
    // cone's ellipse on the surface carried into st by the st gradients.
    Pbr shade_params(const Hit& h, V3 ray_dir, double cone_width) const {
        const Pbr& base = materials[h.material_id];
        if (h.material_id >= bindings.size() || bindings[h.material_id].empty()) return base;
        ShadeCtx c{{h.st[0], h.st[1]}, h.point, h.normal, cone_width * h.st_density, {0, 0}, {0, 0}};
        const V3 gs = h.st_grad[0], gt = h.st_grad[1];
        if (length_sq(gs) + length_sq(gt) > 1e-18 && cone_width > 0.0) {
            const V3 n = h.normal, d = normalize(ray_dir);
            const double cs = std::fmax(std::fabs(dot(d, n)), 1.0 / 16.0);
            V3 t1 = d - n * dot(d, n);
            if (length_sq(t1) < 1e-12) t1 = std::fabs(n.x) < 0.9 ? cross(V3{1, 0, 0}, n) : cross(V3{0, 1, 0}, n);
            t1 = normalize(t1) * (cone_width / cs);
            const V3 t2 = normalize(cross(n, t1)) * cone_width;
            c.dst_major[0] = dot(gs, t1);
            c.dst_major[1] = dot(gt, t1);
            c.dst_minor[0] = dot(gs, t2);
            c.dst_minor[1] = dot(gt, t2);
        }
        Pbr p = base;
        for (const auto& b : bindings[h.material_id])
            p.apply(b.first, pattern_eval(patterns, textures, b.second, c, 0));
        return p;
    }

    const Bvh& blas_of(const Instance& in) const {
        return in.curves ? curve_sets[in.mesh_id].blas : meshes[in.mesh_id].blas;
    }
    // One primitive of an instance against the local ray (mesh.rs:311-333):
    // a triangle (u, v its barycentrics) or a curve segment.
    bool prim_isect(const Instance& in, const Ray& lr, uint32_t p, double t_max, double* t, double* u,
                    double* v) const {
        if (in.curves) {
            V3 n, tg;
            return curve_sets[in.mesh_id].intersect_segment(lr, p, t_max, t, &n, &tg, v);
        }
        return meshes[in.mesh_id].intersect_triangle(lr, p, t_max, t, u, v);
    }

    // scene/mod.rs:105-146, the scan of `objects`: the closest quadric hit
    // (world distance) below t_limit.
    bool quadric_closest(const Ray& ray, double t_limit, Hit* out) const {
        bool any = false;
        double best = t_limit;
        for (size_t k = 0; k < quadrics.size(); k++) {
            const Quadric& q = quadrics[k];
            QuadricHit qh;
            V3 lo = xf_point(q.inv, ray.o), ld = normalize(xf_vec(q.inv, ray.d));
            if (!q.local_hit(lo, ld, &qh)) continue;
            V3 wp = xf_point(q.transform, qh.p);
            double t = length(wp - ray.o);
            if (!(t < best)) continue;
            best = t;
            any = true;
            V3 wn = normalize(xf_normal(q.inv, qh.n));
            out->t = t;
            out->point = wp;
            out->normal = wn;
            out->material_id = q.material_id;
            out->inst = RT_HIT_QUADRIC | (uint32_t)k;
            out->prim = 0;
            out->front_face = qh.front_set ? dot(ray.d, wn) < 0.0 : true;
            out->st[0] = qh.u;
            out->st[1] = qh.v;
            out->st_density = (qh.dpdu > 0.0 || qh.dpdv > 0.0)
                                  ? 1.0 / std::sqrt(std::fmax(qh.dpdu * qh.dpdv, 1e-24)) / q.scale : 0.0;
            out->st_grad[0] = out->st_grad[1] = V3{0, 0, 0};
        }
        return any;
    }

    // mesh.rs:308-381 Instance::intersect + scene/mod.rs:105-146.
    bool intersect(const Ray& ray, Hit* out, Counters* c) const {
        bool have_q = !quadrics.empty() && quadric_closest(ray, INF, out);
        if (instances.empty()) return have_q;
        double dir_len = std::fmax(length(ray.d), 1e-300);
        double t_budget = (have_q ? out->t : INF) / dir_len;
        struct Best {
            uint32_t inst, tri;
            double u, v;
        } best{0, 0, 0, 0};
        auto inst_isect = [&](uint32_t ii, double t_max, double* t_out) -> bool {
            const Instance& in = instances[ii];
            if (c) c->insts++;
            const M4 iv = in.inv_at(ray.time);
            Ray lr{xf_point(iv, ray.o), xf_vec(iv, ray.d), ray.time};
            double hu = 0, hv = 0;
            uint32_t tri;
            double t;
            auto tri_isect = [&](uint32_t tr, double tmax, double* to) -> bool {
                if (c) c->tris++;
                double tt, uu = 0, vv = 0;
                if (prim_isect(in, lr, tr, tmax, &tt, &uu, &vv)) {
                    hu = uu;
                    hv = vv;
                    *to = tt;
                    return true;
                }
                return false;
            };
            if (!blas_of(in).traverse(lr.o, lr.d, t_max, tri_isect, &tri, &t, c)) return false;
            best = {ii, tri, hu, hv};
            *t_out = t;
            return true;
        };
        uint32_t winner;
        double tw;
        if (!tlas.traverse(ray.o, ray.d, t_budget, inst_isect, &winner, &tw, c)) return have_q;
        if (have_q && !(length(ray.d * tw) < out->t)) return true;
        const Instance& in = instances[best.inst];
        const M4 iv = in.inv_at(ray.time);  // mesh.rs:315: normals through the inverse at shutter time
        if (in.curves) {
            // mesh.rs:323-344: the segment's normal and tangent, st = (0.5, v).
            const CurveSet& cs = curve_sets[in.mesh_id];
            Ray lr{xf_point(iv, ray.o), xf_vec(iv, ray.d), ray.time};
            double t, v;
            V3 n, tg;
            cs.intersect_segment(lr, best.tri, INF, &t, &n, &tg, &v);
            V3 wn = normalize(xf_normal(iv, n));
            V3 point = ray.o + ray.d * tw;
            bool front = dot(wn, ray.d) < 0.0;
            if (!front) wn = -wn;
            out->t = length(point - ray.o);
            out->point = point;
            out->normal = normalize(wn);
            out->material_id = in.material_id;
            out->inst = best.inst;
            out->prim = best.tri;
            out->front_face = front;
            out->st[0] = 0.5;
            out->st[1] = v;
            out->st_density = 0.0;
            out->st_grad[0] = out->st_grad[1] = V3{0, 0, 0};
            out->tangent = normalize(xf_vec(in.transform, tg));
            return true;
        }
        const Mesh& m = meshes[in.mesh_id];
        V3 ln = m.local_normal(best.tri, best.u, best.v, ray.time);
        V3 wn = normalize(xf_normal(iv, ln));
        // mesh.rs:427-439 to_intersection.
        V3 point = ray.o + ray.d * tw;
        bool front = dot(wn, ray.d) < 0.0;
        if (!front) wn = -wn;
        out->t = length(point - ray.o);
        out->point = point;
        out->normal = normalize(wn);
        out->material_id = in.material_id;
        out->inst = best.inst;
        out->prim = best.tri;
        out->front_face = front;
        // mesh.rs:357-360: st and its density, transferred to world scale.
        double dens;
        if (m.st_at(best.tri, best.u, best.v, out->st, &dens)) out->st_density = dens / in.scale;
        V3 gs, gt;  // mesh.rs:361-371: gradients pulled back through the inverse
        if (m.st_gradients(best.tri, &gs, &gt)) {
            out->st_grad[0] = xf_normal(in.inv, gs);
            out->st_grad[1] = xf_normal(in.inv, gt);
        }
        return true;
    }

    bool intersect_param(V3 o, V3 d, double t_max, uint32_t* inst, uint32_t* prim, double* t_out,
                         Counters* c) const {
        Ray ray{o, d};
        const double dl = std::fmax(length(d), 1e-300);
        if (!quadrics.empty()) {
            Hit qh;
            if (quadric_closest(ray, t_max * dl, &qh)) {
                t_max = qh.t / dl;
                *inst = qh.inst;
                *prim = 0;
                *t_out = t_max;
                if (instances.empty()) return true;
                uint32_t ii, pp;
                double tt;
                if (intersect_param_meshes(o, d, t_max, &ii, &pp, &tt, c) && tt * dl < qh.t) {
                    *inst = ii;
                    *prim = pp;
                    *t_out = tt;
                }
                return true;
            }
        }
        return intersect_param_meshes(o, d, t_max, inst, prim, t_out, c);
    }

    bool intersect_param_meshes(V3 o, V3 d, double t_max, uint32_t* inst, uint32_t* prim, double* t_out,
                                Counters* c) const {
        if (instances.empty()) return false;
        Ray ray{o, d};
        uint32_t bi = 0, bt = 0;
        auto inst_isect = [&](uint32_t ii, double tmax, double* to) -> bool {
            const Instance& in = instances[ii];
            if (c) c->insts++;
            Ray lr{xf_point(in.inv, ray.o), xf_vec(in.inv, ray.d)};
            uint32_t tri;
            double t;
            auto tri_isect = [&](uint32_t tr, double tm, double* tt) -> bool {
                if (c) c->tris++;
                double uu, vv;
                return prim_isect(in, lr, tr, tm, tt, &uu, &vv);
            };
            if (!blas_of(in).traverse(lr.o, lr.d, tmax, tri_isect, &tri, &t, c)) return false;
            bi = ii;
            bt = tri;
            *to = t;
            return true;
        };
        uint32_t w;
        double tw;
        if (!tlas.traverse(o, d, t_max, inst_isect, &w, &tw, c)) return false;
        *inst = bi;
        *prim = bt;
        *t_out = tw;
        return true;
    }

    // mesh.rs:384-407 Instance::occludes under Bvh::any_hit on the TLAS.
    bool occluded_param(V3 o, V3 d, double t_limit, Counters* c) const {
        if (!quadrics.empty()) {
            Hit qh;
            if (quadric_closest(Ray{o, d}, t_limit * std::fmax(length(d), 1e-300), &qh)) return true;
        }
        if (instances.empty()) return false;
        auto inst_hit = [&](uint32_t ii, double lim) -> bool {
            const Instance& in = instances[ii];
            if (c) c->insts++;
            Ray lr{xf_point(in.inv, o), xf_vec(in.inv, d)};
            return blas_of(in).any_hit(lr.o, lr.d, lim, [&](uint32_t tr, double l2) -> bool {
                if (c) c->tris++;
                double t, u, v;
                return prim_isect(in, lr, tr, l2, &t, &u, &v);
            }, c);
        };
        return tlas.any_hit(o, d, t_limit, inst_hit, c);
    }
};

// ---- integrator (src/raytracer/pt/mod.rs) -----------------------------------

struct Aux {
    V3 albedo, normal, diffuse;
    double depth = 0;
    uint32_t id = 0;
};

static double power_heuristic(double a, double b) {  // mod.rs:992-996
    double a2 = a * a, b2 = b * b;
    return a2 + b2 <= 0.0 ? 0.0 : a2 / (a2 + b2);
}

// mod.rs:34-67: nested media, the top is the medium the ray travels in and
// the atmosphere the implicit bottom.
struct MedStack {
    uint32_t s[8];
    int depth = 0;
    int32_t atmosphere;
    explicit MedStack(int32_t a) : atmosphere(a) {}
    int32_t current() const { return depth > 0 ? (int32_t)s[depth - 1] : atmosphere; }
    void push(uint32_t m) {
        if (depth < 8) s[depth++] = m;
    }
    void pop() {
        if (depth > 0) depth--;
    }
};

struct Tracer {
    const Scene& sc;
    const rt_params& prm;
    uint64_t ext_rays = 0, shadow_rays = 0;
    Counters cext, cshadow;  // traversal work of extension / shadow rays
    double time_ = 0.0;      // the current path's shutter time: every ray it traces carries it
    // Angular size of one pixel, the initial ray-cone spread (pt/mod.rs:73-76).
    double pixel_spread() const { return std::tan(sc.cam.fov * PI / 180.0 / 2.0) * 2.0 / (double)sc.cam.height; }

    // mod.rs:1244-1306 transmittance: opaque surfaces block, cutouts
    // attenuate, volume hulls push and pop the medium (the shadow ray starts
    // in the shading point's medium), and every segment takes its medium's
    // transmittance.
    V3 transmittance(V3 origin, V3 dir, double remaining, int32_t medium, Pcg32& rng) {
        MedStack ms(sc.atmosphere);
        if (medium >= 0 && medium != sc.atmosphere) ms.push((uint32_t)medium);
        V3 vis{1, 1, 1};
        for (int k = 0; k < MAX_PRESENCE_SKIPS; k++) {
            shadow_rays++;
            Hit h;
            Ray r = make_ray(origin, dir, time_);
            const bool found = sc.intersect(r, &h, &cshadow);
            const double seg = std::fmin(found ? h.t : remaining, remaining);
            const int32_t cur = ms.current();
            if (cur >= 0) {
                vis = vis * medium_transmittance(sc.media[cur], origin, dir, seg, rng);
                if (max_comp(vis) < 1e-4) return {0, 0, 0};
            }
            if (!found || h.t >= remaining) return vis;
            if (sc.is_hull(h.material_id)) {
                if (h.front_face) ms.push((uint32_t)sc.materials[h.material_id].interior);
                else ms.pop();
                origin = h.point + dir * RAY_OFFSET;
                remaining -= h.t + RAY_OFFSET;
                continue;
            }
            double presence = std::min(std::max(sc.shade_params(h, dir, 0.0).presence, 0.0), 1.0);
            if (presence >= 1.0) return {0, 0, 0};
            vis = vis * (1.0 - presence);
            if (max_comp(vis) < 1e-4) return {0, 0, 0};
            origin = h.point + dir * RAY_OFFSET;
            remaining -= h.t + RAY_OFFSET;
        }
        return vis;
    }
    // mod.rs:1212-1237
    V3 visibility_to(V3 p, V3 n, V3 target, int32_t medium, Pcg32& rng) {
        V3 dir = target - p;
        double dist = length(dir);
        return transmittance(p + n * RAY_OFFSET, normalize(dir), dist - 1e-3, medium, rng);
    }
    V3 visibility_toward(V3 p, V3 n, V3 wi, int32_t medium, Pcg32& rng) {
        return transmittance(p + n * RAY_OFFSET, wi, 1e8, medium, rng);
    }

    // mod.rs:1000-1023 (rect/disk/sphere).
    static double light_pdf_sa(const Light& l, V3 origin, const Hit& h) {
        if (l.type == RT_LIGHT_RECT || l.type == RT_LIGHT_DISK) {
            V3 d = h.point - origin;
            double dist2 = length_sq(d);
            double cos_l = std::fabs(dot(normalize(d), l.normal));
            if (cos_l < 1e-9 || l.area <= 0.0) return 0.0;
            return dist2 / (cos_l * l.area);
        }
        if (l.type == RT_LIGHT_SPHERE) {
            double dist2 = length_sq(l.p - origin);
            double sin2 = std::fmin(l.radius * l.radius / dist2, 1.0);
            double cos_max = std::sqrt(std::fmax(1.0 - sin2, 0.0));
            double sa = 2.0 * PI * (1.0 - cos_max);
            return sa < 1e-12 ? 0.0 : 1.0 / sa;
        }
        return 0.0;
    }

    // mod.rs:1177-1209
    template <class E>
    V3 area_contrib(V3 p, V3 n, V3 sp, const Light& l, E& eval, double pick, int32_t medium, Pcg32& rng) {
        V3 to = sp - p;
        double dist2 = std::fmax(length_sq(to), 1e-12);
        V3 wi = normalize(to);
        double cos_l = std::fabs(dot(wi, l.normal));
        if (cos_l < 1e-9 || l.area <= 0.0) return {0, 0, 0};
        double bpdf;
        V3 f = eval(wi, &bpdf);
        if (max_comp(f) <= 0.0) return {0, 0, 0};
        V3 vis = visibility_to(p, n, sp, medium, rng);
        if (max_comp(vis) <= 0.0) return {0, 0, 0};
        double pdf_sa = pick * dist2 / (cos_l * l.area);
        double w = power_heuristic(pdf_sa, bpdf);
        return f * l.radiance() * vis * (w / pdf_sa);
    }

    // mod.rs:1032-1174 (point, distant, rect, disk, sphere).
    template <class E>
    V3 sample_light(const Light& l, V3 p, V3 n, E& eval, double pick, int32_t medium, Pcg32& rng) {
        switch (l.type) {
            case RT_LIGHT_POINT: {
                V3 to = l.p - p;
                double dist2 = std::fmax(length_sq(to), 1e-12);
                V3 wi = normalize(to);
                double bp;
                V3 f = eval(wi, &bp);
                if (max_comp(f) <= 0.0) return {0, 0, 0};
                V3 vis = visibility_to(p, n, l.p, medium, rng);
                if (max_comp(vis) <= 0.0) return {0, 0, 0};
                return f * l.radiance_toward(wi) * vis / (dist2 * pick);
            }
            case RT_LIGHT_DISTANT: {
                V3 base = -l.e1;
                V3 wi = base;
                if (l.radius > 1e-5) {
                    double cos_max = std::cos(l.radius);
                    double u = rng.next_f64(), v = rng.next_f64();
                    double cos_t = 1.0 - u * (1.0 - cos_max);
                    double sin_t = std::sqrt(std::fmax(1.0 - cos_t * cos_t, 0.0));
                    double phi = 2.0 * PI * v;
                    Frame lf(base);
                    wi = lf.to_world(V3{sin_t * std::cos(phi), sin_t * std::sin(phi), cos_t});
                }
                double bp;
                V3 f = eval(wi, &bp);
                if (max_comp(f) <= 0.0) return {0, 0, 0};
                V3 vis = visibility_toward(p, n, wi, medium, rng);
                if (max_comp(vis) <= 0.0) return {0, 0, 0};
                return f * l.radiance() * vis / pick;
            }
            case RT_LIGHT_RECT: {
                double u = rng.next_f64(), v = rng.next_f64();
                V3 sp = l.p + l.e1 * u + l.e2 * v;
                return area_contrib(p, n, sp, l, eval, pick, medium, rng);
            }
            case RT_LIGHT_DISK: {
                double u = rng.next_f64(), v = rng.next_f64();
                double r = std::sqrt(u), phi = 2.0 * PI * v;
                V3 sp = l.p + l.e1 * (r * std::cos(phi)) + l.e2 * (r * std::sin(phi));
                return area_contrib(p, n, sp, l, eval, pick, medium, rng);
            }
            case RT_LIGHT_DOME: {  // mod.rs:1139-1172: the map's importance sampling, or a uniform sphere
                double u = rng.next_f64(), v = rng.next_f64();
                V3 wi, rad = l.radiance();
                double pdf_dir = 1.0 / (4.0 * PI);
                if (l.env) {
                    V3 tex;
                    wi = l.env->sample(u, v, &tex, &pdf_dir);
                    rad = tex * l.radiance();
                } else {
                    double z = 1.0 - 2.0 * u;
                    double r = std::sqrt(std::fmax(1.0 - z * z, 0.0));
                    double phi = 2.0 * PI * v;
                    wi = V3{r * std::cos(phi), r * std::sin(phi), z};
                }
                if (pdf_dir <= 0.0) return {0, 0, 0};
                double pdf_sa = pdf_dir * pick;
                double bp;
                V3 f = eval(wi, &bp);
                if (max_comp(f) <= 0.0) return {0, 0, 0};
                V3 vis = visibility_toward(p, n, wi, medium, rng);
                if (max_comp(vis) <= 0.0) return {0, 0, 0};
                return f * rad * vis * (power_heuristic(pdf_sa, bp) / pdf_sa);
            }
            case RT_LIGHT_SPHERE: {
                V3 tc = l.p - p;
                double dist2 = length_sq(tc);
                if (dist2 <= l.radius * l.radius * 1.0001) return {0, 0, 0};
                double sin2 = std::fmin(l.radius * l.radius / dist2, 1.0);
                double cos_max = std::sqrt(std::fmax(1.0 - sin2, 0.0));
                double u = rng.next_f64(), v = rng.next_f64();
                double cos_t = 1.0 - u * (1.0 - cos_max);
                double sin_t = std::sqrt(std::fmax(1.0 - cos_t * cos_t, 0.0));
                double phi = 2.0 * PI * v;
                Frame lf(normalize(tc));
                V3 wi = lf.to_world(V3{sin_t * std::cos(phi), sin_t * std::sin(phi), cos_t});
                double bp;
                V3 f = eval(wi, &bp);
                if (max_comp(f) <= 0.0) return {0, 0, 0};
                double dist = std::sqrt(dist2) * cos_t -
                              std::sqrt(std::fmax(l.radius * l.radius - dist2 * sin_t * sin_t, 0.0));
                V3 target = p + wi * dist;
                V3 vis = visibility_to(p, n, target, medium, rng);
                if (max_comp(vis) <= 0.0) return {0, 0, 0};
                double pdf_sa = pick / std::fmax(2.0 * PI * (1.0 - cos_max), 1e-12);
                double w = power_heuristic(pdf_sa, bp);
                return f * l.radiance() * vis * (w / pdf_sa);
            }
        }
        return {0, 0, 0};
    }

    // mod.rs:449-990 trace_full.
    V3 trace(Ray ray, Pcg32& rng, Aux& aux) {
        time_ = ray.time;
        V3 L{0, 0, 0};
        int first_specular = -1;  // -1 None, 0 false, 1 true
        bool aux_set = false;
        double travel = 0.0;
        auto emit = [&](V3 c) {
            L = L + c;
            if (first_specular != 1) aux.diffuse = aux.diffuse + c;
        };
        V3 beta{1, 1, 1};
        double prev_pdf = 0.0;
        V3 prev_origin = ray.o;
        bool from_camera = true;
        int presence_skips = 0;
        double cone_width = 0.0, cone_spread = pixel_spread();
        MedStack med_stack(sc.atmosphere);
        // Multiple scattering needs a deeper budget (mod.rs:483-484).
        const uint32_t max_bounces = sc.media.empty() ? prm.max_depth : 64u;
        uint32_t depth = 0;
        auto roulette = [&]() {
            if (depth >= prm.rr_start) {
                double q = std::fmin(max_comp(beta), 0.95);
                if (q <= 0.0 || rng.next_f64() > q) return false;
                beta = beta / q;
            }
            return true;
        };
        while (depth < max_bounces) {
            Hit hit;
            ext_rays++;
            const bool found = sc.intersect(ray, &hit, &cext);
            // Medium interaction along this segment, before any surface
            // (mod.rs:490-640).
            const int32_t medium = med_stack.current();
            if (medium >= 0) {
                const Medium& med = sc.media[medium];
                const double t_limit = found ? hit.t : 1e8;
                // One light pick per segment, shared by equiangular and
                // collision NEE so their MIS weights cancel the pick pmf.
                uint32_t pli = 0;
                double ppmf = 0.0;
                const V3 mid = ray.o + ray.d * std::fmin(std::fmin(t_limit, med.max_distance) * 0.5, 50.0);
                const bool seg_pick = sc.ls.sample(mid, rng.next_f64(), &pli, &ppmf);
                const bool point = seg_pick && sc.lights[pli].type == RT_LIGHT_POINT;
                const double t_seg = std::fmin(t_limit, med.max_distance);
                if (point && t_seg > 1e-6) {
                    // Equiangular single-scatter NEE toward the point light.
                    const V3 lp = sc.lights[pli].p;
                    double pdf_eq;
                    const double t_eq = equiangular_sample(ray.o, ray.d, t_seg, lp, rng.next_f64(), &pdf_eq);
                    if (pdf_eq > 1e-12) {
                        const V3 p = ray.o + ray.d * t_eq;
                        const double rho = med.density_at(p);
                        if (rho > 0.0) {
                            const V3 tr = medium_transmittance(med, ray.o, ray.d, t_eq, rng);
                            const V3 sig_s = med.sigma_s * rho;
                            const V3 to_l = lp - p;
                            const double dist2 = std::fmax(length_sq(to_l), 1e-12);
                            const V3 wi = normalize(to_l), wo = -normalize(ray.d);
                            const double ph = hg_phase(med.g, -dot(wo, wi));
                            const V3 vis = transmittance(p, wi, std::sqrt(dist2) - 1e-3, medium, rng);
                            if (max_comp(vis) > 0.0) {
                                const double pdf_d = distance_pdf_approx(med, t_eq, t_seg);
                                const double w_eq = pdf_eq / (pdf_eq + pdf_d);
                                emit(beta * (sig_s * tr * vis * sc.lights[pli].radiance_toward(wi) *
                                             (ph * w_eq / (dist2 * pdf_eq * ppmf))));
                            }
                        }
                    }
                }
                const MediumEvent ev = sample_distance(med, ray.o, ray.d, t_limit, beta, rng);
                beta = beta * ev.weight;
                if (ev.scatter) {
                    const V3 p = ray.o + ray.d * ev.t;
                    if (!aux_set) {
                        aux_set = true;
                        const V3 st = med.sigma_t();
                        aux.albedo = {med.sigma_s.x / std::fmax(st.x, 1e-9), med.sigma_s.y / std::fmax(st.y, 1e-9),
                                      med.sigma_s.z / std::fmax(st.z, 1e-9)};
                        aux.normal = -normalize(ray.d);
                        aux.depth = travel + ev.t;
                        aux.id = 0;
                    }
                    if (first_specular < 0) first_specular = 0;
                    if (max_comp(med.emission) > 0.0) emit(beta * med.emission);
                    const V3 wo = -normalize(ray.d);
                    const double g = med.g;
                    if (seg_pick) {
                        double w_dist = 1.0;
                        if (point) {
                            const double pdf_d = distance_pdf_approx(med, ev.t, t_seg);
                            const double pdf_e = equiangular_pdf(ray.o, ray.d, t_seg, sc.lights[pli].p, ev.t);
                            w_dist = pdf_d / (pdf_d + pdf_e);
                        }
                        auto eval = [&](V3 wi, double* pdf) -> V3 {
                            const double ph = hg_phase(g, -dot(wo, wi));
                            *pdf = ph;
                            return {ph, ph, ph};
                        };
                        const V3 c = sample_light(sc.lights[pli], p, V3{0, 0, 0}, eval, ppmf, medium, rng);
                        emit(beta * c * w_dist);
                    }
                    const double u1 = rng.next_f64(), u2 = rng.next_f64();
                    double pdf;
                    const V3 wi = hg_sample(g, wo, u1, u2, &pdf);
                    prev_pdf = pdf;
                    prev_origin = p;
                    from_camera = false;
                    cone_spread += 0.4;
                    ray = make_ray(p, wi, time_);
                    depth++;
                    if (!roulette()) break;
                    continue;
                }
                if (max_comp(beta) <= 0.0) break;
            }
            if (!found) {
                // mod.rs:643-656: the first dome light (MIS against its NEE
                // sampling unless seen from the camera), else the background.
                int dome = -1;
                for (size_t k = 0; k < sc.lights.size(); k++)
                    if (sc.lights[k].type == RT_LIGHT_DOME) {
                        dome = (int)k;
                        break;
                    }
                if (dome >= 0) {
                    const Light& dl = sc.lights[dome];
                    V3 dir = normalize(ray.d);
                    double w = 1.0;
                    if (!from_camera)
                        w = power_heuristic(prev_pdf, sc.ls.pmf(prev_origin, (uint32_t)dome) *
                                                          (dl.env ? dl.env->pdf(dir) : 1.0 / (4.0 * PI)));
                    emit(beta * (dl.env ? dl.env->eval(dir) * dl.radiance() : dl.radiance()) * w);
                } else {
                    emit(beta * sc.background);
                }
                break;
            }
            // Volume hull: the crossing only toggles the medium (mod.rs:662-680).
            if (sc.is_hull(hit.material_id) && presence_skips < MAX_PRESENCE_SKIPS) {
                presence_skips++;
                travel += hit.t;
                if (hit.front_face) med_stack.push((uint32_t)sc.materials[hit.material_id].interior);
                else med_stack.pop();
                ray = make_ray(hit.point + normalize(ray.d) * RAY_OFFSET, ray.d, time_);
                continue;
            }
            V3 wo = -normalize(ray.d);
            cone_width += hit.t * cone_spread;
            travel += hit.t;
            const Pbr pbr = sc.shade_params(hit, ray.d, cone_width);
            if (!aux_set) {
                aux_set = true;
                V3 a = pbr.diffuse_color * pbr.diffuse_gain + pbr.specular_f0() * (pbr.has_specular() ? 1.0 : 0.0) +
                       pbr.subsurface_color * pbr.subsurface_gain + pbr.refraction_color * pbr.glass_gain;
                aux.albedo = {std::fmin(a.x, 1.0), std::fmin(a.y, 1.0), std::fmin(a.z, 1.0)};
                aux.normal = dot(hit.normal, wo) >= 0.0 ? hit.normal : -hit.normal;
                aux.depth = travel;
                aux.id = pbr.id;
            }
            double presence = std::min(std::max(pbr.presence, 0.0), 1.0);
            if (presence < 1.0 && rng.next_f64() >= presence && presence_skips < MAX_PRESENCE_SKIPS) {
                presence_skips++;
                travel += hit.t;
                ray = make_ray(hit.point + normalize(ray.d) * RAY_OFFSET, ray.d, time_);
                continue;
            }
            bool entering = hit.front_face;
            V3 n = dot(hit.normal, wo) >= 0.0 ? hit.normal : -hit.normal;
            double eta_rel = entering ? pbr.glass_ior : 1.0 / pbr.glass_ior;
            V3 emission = pbr.emission + pbr.glow;
            if (max_comp(emission) > 0.0) {
                double weight = 1.0;
                if (!from_camera && pbr.area_light >= 0) {
                    const Light& l = sc.lights[pbr.area_light];
                    double pick = sc.ls.pmf(prev_origin, (uint32_t)pbr.area_light);
                    double pdf_light = light_pdf_sa(l, prev_origin, hit) * pick;
                    weight = power_heuristic(prev_pdf, pdf_light);
                }
                emit(beta * emission * weight);
            }
            // Subsurface scattering (mod.rs:794-892): with probability
            // subsurfaceGain an isotropic random walk inside the object through
            // the Burley-fit homogeneous medium, leaving diffusely where the
            // walk first reaches a surface.
            // Hair fibers scatter over the whole sphere with their own BSDF
            // (mod.rs:737-781), on curve hits only.
            if (pbr.hair && length_sq(hit.tangent) > 0.5) {
                HairParams hp;
                hp.init(pbr.hair_sigma_a, pbr.hair_beta_m, pbr.hair_beta_n, pbr.hair_eta);
                const FiberFrame ff(hit.tangent, hit.normal, wo);
                const V3 wo_f = ff.to_local(wo);
                const double hh = ff.h;
                if (!sc.lights.empty()) {
                    auto eval = [&](V3 wi, double* pdf) -> V3 {
                        const V3 wf = ff.to_local(wi);
                        *pdf = hair_pdf(hp, wo_f, wf, hh);
                        return hair_f(hp, wo_f, wf, hh);
                    };
                    uint32_t li;
                    double pmf;
                    if (sc.ls.sample(hit.point, rng.next_f64(), &li, &pmf))
                        emit(beta * sample_light(sc.lights[li], hit.point, n, eval, pmf, medium, rng));
                }
                V3 wi_f, fv;
                double pv;
                if (!hair_sample(hp, wo_f, hh, rng, &wi_f, &fv, &pv)) break;
                const V3 wi = ff.to_world(wi_f);
                beta = beta * fv / pv;  // f is per solid angle: no cosine
                if (first_specular < 0) first_specular = 0;
                prev_pdf = pv;
                prev_origin = hit.point;
                from_camera = false;
                cone_spread += 0.4;
                const V3 side = dot(wi, hit.normal) >= 0.0 ? hit.normal : -hit.normal;
                ray = make_ray(hit.point + side * RAY_OFFSET, wi, time_);
                depth++;
                if (!roulette()) break;
                continue;
            }
            if (pbr.subsurface_gain > 0.0 && !pbr.hair &&
                rng.next_f64() < std::min(std::max(pbr.subsurface_gain, 0.0), 1.0)) {
                if (first_specular < 0) first_specular = 0;
                const Medium sss = sss_medium(pbr.subsurface_color, pbr.subsurface_dmfp);
                const Frame entry(-n);
                const double e1 = rng.next_f64(), e2 = rng.next_f64();
                const double er = std::sqrt(e1), ephi = 2.0 * PI * e2;
                Ray walk = make_ray(hit.point - n * RAY_OFFSET,
                                    entry.to_world(V3{er * std::cos(ephi), er * std::sin(ephi), std::sqrt(std::fmax(1.0 - e1, 0.0))}), time_);
                bool exited = false;
                for (int step = 0; step < 256; step++) {
                    Hit wh;
                    ext_rays++;
                    if (!sc.intersect(walk, &wh, &cext)) break;  // escaped through a crack
                    const MediumEvent ev = sample_distance(sss, walk.o, walk.d, wh.t, beta, rng);
                    beta = beta * ev.weight;
                    if (ev.scatter) {
                        const V3 p = walk.o + walk.d * ev.t;
                        const double u = rng.next_f64(), v = rng.next_f64();
                        const double z = 1.0 - 2.0 * u, rr = std::sqrt(std::fmax(1.0 - z * z, 0.0)), ph = 2.0 * PI * v;
                        walk = make_ray(p, V3{rr * std::cos(ph), rr * std::sin(ph), z}, time_);
                        const double q = std::fmin(max_comp(beta), 0.95);
                        if (q <= 0.0 || (step > 8 && rng.next_f64() > q)) break;
                        if (step > 8) beta = beta / q;
                        continue;
                    }
                    const V3 out_n = dot(wh.normal, walk.d) > 0.0 ? wh.normal : -wh.normal;
                    const Frame xf(out_n);
                    const V3 exit_p = walk.o + walk.d * wh.t;
                    uint32_t xli;
                    double xpmf;
                    if (sc.ls.sample(exit_p, rng.next_f64(), &xli, &xpmf)) {
                        auto eval = [&](V3 wi, double* pdf) -> V3 {
                            const V3 wl = xf.to_local(wi);
                            if (wl.z <= 0.0) {
                                *pdf = 0.0;
                                return {0, 0, 0};
                            }
                            *pdf = wl.z / PI;
                            return V3{1, 1, 1} * (wl.z / PI);
                        };
                        emit(beta * sample_light(sc.lights[xli], exit_p, out_n, eval, xpmf, medium, rng));
                    }
                    const double x1 = rng.next_f64(), x2 = rng.next_f64();
                    const double xr = std::sqrt(x1), xphi = 2.0 * PI * x2;
                    const V3 local{xr * std::cos(xphi), xr * std::sin(xphi), std::sqrt(std::fmax(1.0 - x1, 0.0))};
                    prev_pdf = std::fmax(local.z, 1e-9) / PI;
                    prev_origin = exit_p;
                    from_camera = false;
                    cone_spread += 0.4;
                    ray = make_ray(exit_p + out_n * RAY_OFFSET, xf.to_world(local), time_);
                    exited = true;
                    break;
                }
                if (!exited) break;
                depth++;
                if (!roulette()) break;
                continue;
            }
            Frame frame(n);
            V3 wo_l = frame.to_local(wo);
            double lw[5];
            if (!sc.lights.empty() && pbr.lobe_weights(lw)) {
                auto eval = [&](V3 wi_world, double* pdf) -> V3 {
                    V3 wi_l = frame.to_local(wi_world);
                    if (wi_l.z <= 0.0) {
                        *pdf = 0.0;
                        return {0, 0, 0};
                    }
                    V3 f;
                    eval_pdf(pbr, wo_l, wi_l, eta_rel, &f, pdf);
                    return f * wi_l.z;
                };
                uint32_t li;
                double pmf;
                if (sc.ls.sample(hit.point, rng.next_f64(), &li, &pmf)) {
                    V3 c = sample_light(sc.lights[li], hit.point, n, eval, pmf, medium, rng);
                    emit(beta * c);
                }
            }
            BsdfSample s;
            if (!sample_bsdf(pbr, wo_l, eta_rel, rng, &s)) break;
            V3 wi_world = frame.to_world(s.wi);
            beta = beta * s.f * (std::fabs(s.wi.z) / s.pdf);
            if (first_specular < 0) first_specular = s.specular_lobe ? 1 : 0;
            prev_pdf = s.pdf;
            prev_origin = hit.point;
            from_camera = false;
            cone_spread += std::fmin(1.0 / (1.0 + s.pdf), 0.4);  // pt/mod.rs:965-967
            if (s.transmitted && pbr.interior >= 0) {  // mod.rs:969-975
                if (entering) med_stack.push((uint32_t)pbr.interior);
                else med_stack.pop();
            }
            double off = s.transmitted ? -RAY_OFFSET : RAY_OFFSET;
            ray = make_ray(hit.point + n * off, wi_world, time_);
            depth++;
            if (!roulette()) break;
        }
        return L;
    }
};

}  // namespace orc

using namespace orc;

static void load_textures(const rt_scene_desc* d, std::vector<Texture>& out) {
    out.resize(d->textures ? d->n_textures : 0);
    for (size_t i = 0; i < out.size(); i++) out[i].build(d->textures[i].rgb, d->textures[i].width, d->textures[i].height);
}

static void load_patterns(const rt_scene_desc* d, std::vector<PatNode>& out) {
    for (uint32_t i = 0; i < d->n_patterns && d->patterns; i++) {
        const rt_pattern_desc& pd = d->patterns[i];
        PatNode n;
        n.type = pd.type;
        n.octaves = pd.octaves;
        n.a = v3(pd.color_a);
        n.b = v3(pd.color_b);
        n.scale[0] = pd.scale[0];
        n.scale[1] = pd.scale[1];
        n.frequency = pd.frequency;
        n.gain = pd.gain;
        n.lacunarity = pd.lacunarity;
        n.gamma = pd.gamma;
        n.saturation = pd.saturation;
        for (int k = 0; k < 3; k++) n.in[k] = {pd.in[k].node, v3(pd.in[k].value)};
        for (uint32_t r = 0; r < pd.n_ramp && pd.ramp_positions && pd.ramp_colors; r++) {
            n.ramp_pos.push_back(pd.ramp_positions[r]);
            n.ramp_col.push_back(v3(pd.ramp_colors + 3 * r));
        }
        n.use_t = pd.use_t != 0;
        n.texture = pd.texture;
        n.wrap = (int)pd.wrap;
        for (uint32_t k = 0; k < pd.n_udim && pd.udim_tiles && pd.udim_textures; k++)
            n.udim.push_back({pd.udim_tiles[k], pd.udim_textures[k]});
        out.push_back(n);
    }
}

struct oracle_scene {
    Scene s;
};

static Light make_light(const rt_light_desc& d) {
    Light l;
    l.type = d.type;
    l.intensity = d.intensity;
    l.color = v3(d.color);
    l.p = v3(d.p);
    l.e1 = v3(d.e1);
    l.e2 = v3(d.e2);
    l.radius = d.radius;
    if (d.type == RT_LIGHT_DISTANT) l.e1 = normalize(l.e1);  // light.rs:68-80
    if (d.type == RT_LIGHT_RECT) {                            // light.rs:95-110
        V3 c = cross(l.e1, l.e2);
        l.area = length(c);
        l.normal = normalize(c);
    }
    if (d.type == RT_LIGHT_DISK) {  // light.rs:124-135
        l.normal = normalize(cross(l.e1, l.e2));
        l.area = PI * length(l.e1) * length(l.e2);
    }
    return l;
}

template <class F>
static void parallel_for(uint64_t n, int threads, F&& f) {
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    if (threads == 1 || n < 64) {
        f(0, n, 0);
        return;
    }
    std::atomic<uint64_t> next{0};
    // Chunks of up to 64 items, smaller when there are few items per thread
    // (a few hundred pixels of an expensive scene still use every thread).
    const uint64_t chunk = std::max<uint64_t>(1, std::min<uint64_t>(64, n / ((uint64_t)threads * 16)));
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++)
        pool.emplace_back([&, t] {
            for (;;) {
                uint64_t b = next.fetch_add(chunk);
                if (b >= n) break;
                f(b, std::min(n, b + chunk), t);
            }
        });
    for (auto& th : pool) th.join();
}

extern "C" {

static Medium medium_from(const rt_medium_desc& md) {
    Medium m;
    m.sigma_a = v3(md.sigma_a);
    m.sigma_s = v3(md.sigma_s);
    m.emission = v3(md.emission);
    m.g = md.g;
    m.max_distance = md.max_distance;
    m.fbm_density = md.density == RT_DENSITY_FBM;
    m.octaves = md.octaves;
    m.frequency = md.frequency;
    m.gain = md.gain;
    m.lacunarity = md.lacunarity;
    m.coverage = md.coverage;
    m.sharpness = md.sharpness;
    return m;
}

oracle_scene* oracle_scene_create(const rt_scene_desc* d) {
    if (!d) return nullptr;
    auto* os = new oracle_scene();
    Scene& s = os->s;
    s.meshes.resize(d->n_meshes);
    for (uint32_t i = 0; i < d->n_meshes; i++) {
        const rt_mesh_desc& md = d->meshes[i];
        Mesh& m = s.meshes[i];
        m.pos.assign(md.positions, md.positions + 3ull * md.n_vertices);
        m.idx.assign(md.indices, md.indices + 3ull * md.n_triangles);
        if (md.normals) m.nrm.assign(md.normals, md.normals + 3ull * md.n_vertices);
        if (md.st) m.st.assign(md.st, md.st + 2ull * md.n_vertices);
        for (uint32_t k = 0; k < d->n_mesh_motion && d->mesh_motion; k++)
            if (d->mesh_motion[k].mesh == i && d->mesh_motion[k].positions1)
                m.pos1.assign(d->mesh_motion[k].positions1, d->mesh_motion[k].positions1 + 3ull * md.n_vertices);
        m.build();
        s.has_motion |= !m.pos1.empty();
    }
    s.curve_sets.resize(d->curves ? d->n_curves : 0);
    for (uint32_t k = 0; k < s.curve_sets.size(); k++) {
        const rt_curves_desc& cd = d->curves[k];
        CurveSet& cs = s.curve_sets[k];
        cs.p0.assign(cd.p0, cd.p0 + 4ull * cd.n_segments);
        cs.p1.assign(cd.p1, cd.p1 + 4ull * cd.n_segments);
        cs.v0.assign(cd.v0, cd.v0 + cd.n_segments);
        cs.v1.assign(cd.v1, cd.v1 + cd.n_segments);
        cs.build();
    }
    s.instances.resize(d->n_instances);
    std::vector<Aabb> ib(d->n_instances);
    for (uint32_t i = 0; i < d->n_instances; i++) {
        const rt_instance_desc& id = d->instances[i];
        Instance& in = s.instances[i];
        in.curves = id.mesh_id >= d->n_meshes;
        in.mesh_id = in.curves ? id.mesh_id - d->n_meshes : id.mesh_id;
        in.material_id = id.material_id;
        in.transform = identity();
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 4; c++) in.transform.m[r][c] = id.object_to_world[r * 4 + c];
        if (!inverse(in.transform, in.inv)) in.inv = identity();  // mesh.rs:282
        double lx = length(xf_vec(in.transform, V3{1, 0, 0})), ly = length(xf_vec(in.transform, V3{0, 1, 0})),
               lz = length(xf_vec(in.transform, V3{0, 0, 1}));
        in.scale = std::fmax(std::cbrt(lx * ly * lz), 1e-12);
        ib[i] = Aabb{};
    }
    for (uint32_t k = 0; k < d->n_instance_motion && d->instance_motion; k++) {
        const rt_instance_motion& im = d->instance_motion[k];
        if (im.instance >= d->n_instances) continue;
        Instance& in = s.instances[im.instance];
        in.moving = true;
        in.transform1 = identity();
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 4; c++) in.transform1.m[r][c] = im.object_to_world1[r * 4 + c];
        s.has_motion = true;
    }
    for (uint32_t i = 0; i < d->n_instances; i++) {
        Instance& in = s.instances[i];
        // mesh.rs:276-290 world bounds from the 8 transformed corners, at
        // both shutter endpoints when moving.
        const Aabb& lb = in.curves ? s.curve_sets[in.mesh_id].local_bounds : s.meshes[in.mesh_id].local_bounds;
        for (const M4* xf : {&in.transform, in.moving ? &in.transform1 : nullptr}) {
            if (!xf) continue;
            for (int k = 0; k < 8; k++) {
                V3 corner{(k & 1) ? lb.mx.x : lb.mn.x, (k & 2) ? lb.mx.y : lb.mn.y, (k & 4) ? lb.mx.z : lb.mn.z};
                in.world_bounds.grow_point(xf_point(*xf, corner));
            }
        }
        ib[i] = in.world_bounds;
    }
    s.tlas.build(ib);  // scene/mod.rs:82-86
    for (uint32_t k = 0; k < d->n_quadrics && d->quadrics; k++) {
        const rt_quadric_desc& qd = d->quadrics[k];
        Quadric q;
        q.type = qd.type;
        q.material_id = qd.material_id;
        for (int j = 0; j < 8; j++) q.prm[j] = qd.params[j];
        q.transform = identity();
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 4; c++) q.transform.m[r][c] = qd.object_to_world[r * 4 + c];
        if (!inverse(q.transform, q.inv)) q.inv = identity();
        double lx = length(xf_vec(q.transform, V3{1, 0, 0})), ly = length(xf_vec(q.transform, V3{0, 1, 0})),
               lz = length(xf_vec(q.transform, V3{0, 0, 1}));
        q.scale = std::fmax(std::cbrt(lx * ly * lz), 1e-12);
        s.quadrics.push_back(q);
    }
    for (uint32_t k = 0; k < d->n_media && d->media; k++) s.media.push_back(medium_from(d->media[k]));
    s.atmosphere = (d->atmosphere >= 0 && (uint32_t)d->atmosphere < s.media.size()) ? d->atmosphere : -1;
    for (uint32_t i = 0; i < d->n_materials; i++) {
        s.materials.push_back(Pbr::from(d->materials[i]));
        if (s.materials.back().interior >= (int32_t)s.media.size()) s.materials.back().interior = -1;
        if (d->materials[i].presence < 1.0) s.any_presence = true;
    }
    load_patterns(d, s.patterns);
    load_textures(d, s.textures);
    s.bindings.resize(d->n_materials);
    for (uint32_t i = 0; i < d->n_bindings && d->bindings; i++) {
        const rt_pattern_binding& b = d->bindings[i];
        if (b.material < d->n_materials) {
            s.bindings[b.material].push_back({b.field, b.node});
            if (b.field == RT_FIELD_PRESENCE) s.any_presence = true;
        }
    }
    for (uint32_t i = 0; i < d->n_lights; i++) s.lights.push_back(make_light(d->lights[i]));
    for (uint32_t k = 0; k < d->n_ies && d->ies; k++) {
        const rt_ies_desc& e = d->ies[k];
        if (e.light >= d->n_lights || !e.n_v || !e.n_h) continue;
        auto ies = std::make_shared<Ies>();
        ies->v.assign(e.v_angles, e.v_angles + e.n_v);
        ies->h.assign(e.h_angles, e.h_angles + e.n_h);
        ies->cd.assign(e.candela, e.candela + (size_t)e.n_v * e.n_h);
        ies->to_local = identity();
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) ies->to_local.m[r][c] = e.world_to_local[3 * r + c];
        ies->finish();
        s.lights[e.light].ies = ies;
    }
    if (d->env_rgb && d->env_width && d->env_height && d->env_light < d->n_lights) {
        auto env = std::make_shared<EnvMap>();
        env->w = d->env_width;
        env->h = d->env_height;
        env->rgb.assign(d->env_rgb, d->env_rgb + 3ull * env->w * env->h);
        env->build();
        s.lights[d->env_light].env = env;
    }
    s.ls.build(s.lights);
    const rt_camera_desc& c = d->camera;
    s.cam.width = c.width;
    s.cam.height = c.height;
    s.cam.fov = c.fov_deg;
    s.cam.eye = v3(c.eye);
    s.cam.forward = v3(c.forward);
    s.cam.up = v3(c.up);
    s.cam.right = v3(c.right);
    s.cam.lens_radius = c.lens_radius;
    s.cam.focal_distance = c.focal_distance;
    s.cam.filter = c.filter;
    s.cam.filter_width = c.filter_width;
    s.cam.projection = c.projection;
    s.cam.ortho_half[0] = c.ortho_half[0];
    s.cam.ortho_half[1] = c.ortho_half[1];
    if (d->camera_motion_inv) {
        s.cam.moving = true;
        s.cam.motion_inv = identity();
        for (int r = 0; r < 3; r++)
            for (int k = 0; k < 4; k++) s.cam.motion_inv.m[r][k] = d->camera_motion_inv[r * 4 + k];
        s.has_motion = true;  // scene_builder.rs:239-241
    }
    s.background = v3(d->background);
    return os;
}

void oracle_scene_destroy(oracle_scene* s) { delete s; }

void oracle_scene_stats(const oracle_scene* os, uint64_t* blas_nodes, uint64_t* tlas_nodes) {
    uint64_t b = 0;
    for (auto& m : os->s.meshes) b += m.blas.nodes.size();
    if (blas_nodes) *blas_nodes = b;
    if (tlas_nodes) *tlas_nodes = os->s.tlas.nodes.size();
}

int oracle_intersect(const oracle_scene* os, const float* planes, uint64_t n, int any_hit, uint32_t* prim,
                     uint32_t* inst, double* t, oracle_counters* counters, int threads) {
    if (!os || !planes) return -1;
    const Scene& s = os->s;
    int nt = threads <= 0 ? (int)std::max(1u, std::thread::hardware_concurrency()) : threads;
    std::vector<Counters> per(nt);
    parallel_for(n, nt, [&](uint64_t b, uint64_t e, int tid) {
        Counters& c = per[tid];
        for (uint64_t i = b; i < e; i++) {
            const float* po = planes + 4 * i;
            const float* pd = planes + 4 * n + 4 * i;
            V3 o{po[0], po[1], po[2]}, d{pd[0], pd[1], pd[2]};
            double tmax = pd[3];
            if (any_hit) {
                bool h = s.occluded_param(o, d, tmax, &c);
                if (prim) prim[i] = h ? 1u : 0u;
            } else {
                uint32_t ii = 0xFFFFFFFFu, pp = 0xFFFFFFFFu;
                double tt = INF;
                if (!s.intersect_param(o, d, tmax, &ii, &pp, &tt, &c)) {
                    ii = pp = 0xFFFFFFFFu;
                    tt = INF;
                }
                if (prim) prim[i] = pp;
                if (inst) inst[i] = ii;
                if (t) t[i] = tt;
            }
        }
    });
    if (counters) {
        memset(counters, 0, sizeof(*counters));
        for (auto& c : per) {
            counters->node_pops += c.pops;
            counters->tri_tests += c.tris;
            counters->inst_tests += c.insts;
        }
        counters->rays = n;
    }
    return 0;
}

int oracle_render(const oracle_scene* os, const rt_params* p, const uint32_t* pixels, uint64_t n_pixels, uint32_t s0,
                  uint32_t s1, double* rgb, double* aux_out, uint64_t* ray_counts, int threads) {
    if (!os || !p || !pixels || !rgb) return -1;
    const Scene& s = os->s;
    int nt = threads <= 0 ? (int)std::max(1u, std::thread::hardware_concurrency()) : threads;
    std::vector<uint64_t> ext(nt, 0), shd(nt, 0);
    std::vector<std::array<uint64_t, 6>> work(nt, std::array<uint64_t, 6>{});
    const double clampv = p->firefly_clamp;
    parallel_for(n_pixels, nt, [&](uint64_t b, uint64_t e, int tid) {
        Tracer tr{s, *p, 0, 0, Counters{}, Counters{}};
        for (uint64_t k = b; k < e; k++) {
            uint32_t pix = pixels[k];
            uint32_t x = pix % s.cam.width, y = pix / s.cam.width;
            V3 sum{0, 0, 0}, alb{0, 0, 0}, nrm{0, 0, 0}, dif{0, 0, 0};
            double depth_sum = 0;
            uint32_t hits = 0;
            std::map<uint32_t, uint32_t> votes;
            for (uint32_t smp = s0; smp < s1; smp++) {
                // mod.rs:84-93 per-sample seeding, camera ray, clamp.
                Pcg32 rng = Pcg32::for_pixel_sample(pix, smp);
                double u1 = rng.next_f64(), u2 = rng.next_f64();
                double px = x + 0.5 + s.cam.sample_1d(u1), py = y + 0.5 + s.cam.sample_1d(u2);
                double lu = 0.5, lv = 0.5;
                if (s.cam.lens_radius > 0.0) {
                    lu = rng.next_f64();
                    lv = rng.next_f64();
                }
                Ray ray = s.cam.generate(px, py, lu, lv);
                if (s.has_motion) {  // mod.rs:350-353 shutter time, camera motion
                    ray.time = rng.next_f64();
                    ray = s.cam.apply_motion(ray);
                }
                Aux aux;
                V3 l = tr.trace(ray, rng, aux);
                double lm = lum(l);
                if (lm > clampv) {
                    double kk = clampv / lm;
                    l = l * kk;
                    aux.diffuse = aux.diffuse * kk;
                }
                sum = sum + l;
                dif = dif + aux.diffuse;
                alb = alb + aux.albedo;
                nrm = nrm + aux.normal;
                if (aux.depth > 0.0) {
                    depth_sum += aux.depth;
                    hits++;
                }
                votes[aux.id]++;
            }
            rgb[3 * k] = sum.x;
            rgb[3 * k + 1] = sum.y;
            rgb[3 * k + 2] = sum.z;
            if (aux_out) {
                double* a = aux_out + 12 * k;
                uint32_t best_id = 0, best_n = 0;
                for (auto& kv : votes)
                    if (kv.second > best_n) {
                        best_n = kv.second;
                        best_id = kv.first;
                    }
                a[0] = alb.x; a[1] = alb.y; a[2] = alb.z;
                a[3] = nrm.x; a[4] = nrm.y; a[5] = nrm.z;
                a[6] = depth_sum;
                a[7] = best_id;
                a[8] = dif.x; a[9] = dif.y; a[10] = dif.z;
                a[11] = hits;
            }
        }
        ext[tid] += tr.ext_rays;
        shd[tid] += tr.shadow_rays;
        work[tid][0] += tr.cext.pops;
        work[tid][1] += tr.cext.tris;
        work[tid][2] += tr.cext.insts;
        work[tid][3] += tr.cshadow.pops;
        work[tid][4] += tr.cshadow.tris;
        work[tid][5] += tr.cshadow.insts;
    });
    if (ray_counts) {
        for (int k = 0; k < 8; k++) ray_counts[k] = 0;
        for (int t = 0; t < nt; t++) {
            ray_counts[0] += ext[t];
            ray_counts[1] += shd[t];
            for (int k = 0; k < 6; k++) ray_counts[2 + k] += work[t][k];
        }
    }
    return 0;
}

void oracle_pcg_stream(uint64_t pixel, uint64_t sample, uint32_t n, uint32_t* out) {
    Pcg32 r = Pcg32::for_pixel_sample(pixel, sample);
    for (uint32_t i = 0; i < n; i++) out[i] = r.next_u32();
}

void oracle_pcg_new_stream(uint64_t seed, uint64_t stream, uint32_t n, uint32_t* out) {
    Pcg32 r(seed, stream);
    for (uint32_t i = 0; i < n; i++) out[i] = r.next_u32();
}

int oracle_bsdf_eval(const rt_material_desc* m, const double* wo, const double* wi, double eta, double* f_out,
                     double* pdf_out) {
    Pbr p = Pbr::from(*m);
    V3 f;
    double pdf;
    eval_pdf(p, v3(wo), v3(wi), eta, &f, &pdf);
    f_out[0] = f.x;
    f_out[1] = f.y;
    f_out[2] = f.z;
    *pdf_out = pdf;
    return 0;
}

double oracle_bsdf_furnace(const rt_material_desc* m, const double* wo, double eta, uint64_t n, uint64_t seed,
                           uint64_t stream, double* rgb_out) {
    Pbr p = Pbr::from(*m);
    Pcg32 rng(seed, stream);
    V3 w = v3(wo);
    double acc = 0.0;
    V3 acc3{0, 0, 0};
    for (uint64_t i = 0; i < n; i++) {
        BsdfSample s;
        if (sample_bsdf(p, w, eta, rng, &s)) {
            double k = std::fabs(s.wi.z) / s.pdf;
            acc += lum(s.f) * k;
            acc3 = acc3 + s.f * k;
        }
    }
    if (rgb_out) {
        rgb_out[0] = acc3.x / (double)n;
        rgb_out[1] = acc3.y / (double)n;
        rgb_out[2] = acc3.z / (double)n;
    }
    return acc / (double)n;
}

int oracle_light_sample(const oracle_scene* os, const double* p, double u, uint32_t* light, double* pmf) {
    return os->s.ls.sample(v3(p), u, light, pmf) ? 1 : 0;
}

double oracle_light_pmf(const oracle_scene* os, const double* p, uint32_t light) { return os->s.ls.pmf(v3(p), light); }

// Environment map functions (envmap.rs) on a w x h RGB map: per direction
// eval (3 doubles) and pdf; per (u1, u2) the sampled direction, radiance
// and pdf.
void oracle_env_eval_pdf(uint32_t w, uint32_t h, const float* rgb, uint64_t n, const double* dirs, double* rad,
                         double* pdf) {
    EnvMap e;
    e.w = w;
    e.h = h;
    e.rgb.assign(rgb, rgb + 3ull * w * h);
    e.build();
    for (uint64_t i = 0; i < n; i++) {
        V3 d{dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]};
        V3 c = e.eval(d);
        rad[3 * i] = c.x;
        rad[3 * i + 1] = c.y;
        rad[3 * i + 2] = c.z;
        pdf[i] = e.pdf(d);
    }
}

void oracle_env_sample(uint32_t w, uint32_t h, const float* rgb, uint64_t n, const double* uv, double* dirs,
                       double* rad, double* pdf) {
    EnvMap e;
    e.w = w;
    e.h = h;
    e.rgb.assign(rgb, rgb + 3ull * w * h);
    e.build();
    for (uint64_t i = 0; i < n; i++) {
        V3 c;
        V3 d = e.sample(uv[2 * i], uv[2 * i + 1], &c, &pdf[i]);
        dirs[3 * i] = d.x;
        dirs[3 * i + 1] = d.y;
        dirs[3 * i + 2] = d.z;
        rad[3 * i] = c.x;
        rad[3 * i + 1] = c.y;
        rad[3 * i + 2] = c.z;
    }
}

void oracle_pattern_eval(const rt_scene_desc* d, uint32_t node, uint64_t n, const double* ctx, double* rgb) {
    std::vector<PatNode> nodes;
    std::vector<Texture> tex;
    load_patterns(d, nodes);
    load_textures(d, tex);
    for (uint64_t i = 0; i < n; i++) {
        const double* c = ctx + 13 * i;
        ShadeCtx sc{{c[0], c[1]}, V3{c[2], c[3], c[4]}, V3{c[5], c[6], c[7]}, c[8], {c[9], c[10]}, {c[11], c[12]}};
        V3 v = pattern_eval(nodes, tex, node, sc, 0);
        rgb[3 * i] = v.x;
        rgb[3 * i + 1] = v.y;
        rgb[3 * i + 2] = v.z;
    }
}

// One quadric against world rays (origin, direction: 6 doubles each): per
// ray t (world distance, -1 on a miss), hit point, world normal, u, v, st
// density, front face (10 doubles).
void oracle_quadric_intersect(const rt_quadric_desc* qd, uint64_t n, const double* rays, double* out) {
    Quadric q;
    q.type = qd->type;
    q.material_id = qd->material_id;
    for (int j = 0; j < 8; j++) q.prm[j] = qd->params[j];
    q.transform = identity();
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 4; c++) q.transform.m[r][c] = qd->object_to_world[r * 4 + c];
    if (!inverse(q.transform, q.inv)) q.inv = identity();
    double lx = length(xf_vec(q.transform, V3{1, 0, 0})), ly = length(xf_vec(q.transform, V3{0, 1, 0})),
           lz = length(xf_vec(q.transform, V3{0, 0, 1}));
    q.scale = std::fmax(std::cbrt(lx * ly * lz), 1e-12);
    Scene one;
    one.quadrics.push_back(q);
    for (uint64_t i = 0; i < n; i++) {
        const double* r = rays + 6 * i;
        double* o = out + 10 * i;
        Hit h;
        if (!one.quadric_closest(Ray{V3{r[0], r[1], r[2]}, V3{r[3], r[4], r[5]}}, INF, &h)) {
            for (int k = 0; k < 10; k++) o[k] = k == 0 ? -1.0 : 0.0;
            continue;
        }
        o[0] = h.t;
        o[1] = h.point.x;
        o[2] = h.point.y;
        o[3] = h.point.z;
        o[4] = h.normal.x;
        o[5] = h.normal.y;
        o[6] = h.normal.z;
        o[7] = h.st[0];
        o[8] = h.st[1];
        o[9] = h.st_density;
        (void)h.front_face;
    }
}

// Real roots of a quartic (extra.rs:112-193), ascending; returns the count.
int oracle_solve_quartic(const double* coef, double* roots) {
    std::vector<double> r = q_quartic(coef[0], coef[1], coef[2], coef[3], coef[4]);
    for (size_t k = 0; k < r.size() && k < 4; k++) roots[k] = r[k];
    return (int)std::min<size_t>(r.size(), 4);
}

// Shadow-ray transmittance (mod.rs:1254-1306, Tracer::transmittance) of
// rays in rt_intersect_batch's two-plane layout: from each origin along the
// normalised direction for the distance tmax; one RGB transmittance each.
void oracle_transmittance(const oracle_scene* os, const float* planes, uint64_t n, double* out, int threads) {
    const Scene& s = os->s;
    rt_params prm{};
    int nt = threads <= 0 ? (int)std::max(1u, std::thread::hardware_concurrency()) : threads;
    parallel_for(n, nt, [&](uint64_t b, uint64_t e, int) {
        Tracer tr{s, prm, 0, 0, Counters{}, Counters{}};
        for (uint64_t i = b; i < e; i++) {
            const float* po = planes + 4 * i;
            const float* pd = planes + 4 * n + 4 * i;
            V3 o{po[0], po[1], po[2]}, d{pd[0], pd[1], pd[2]};
            Pcg32 rng = Pcg32::for_pixel_sample(i, 0);
            V3 v = tr.transmittance(o, normalize(d), pd[3], s.atmosphere, rng);
            out[3 * i] = v.x;
            out[3 * i + 1] = v.y;
            out[3 * i + 2] = v.z;
        }
    });
}

void oracle_intersect_st(const oracle_scene* os, uint64_t n, const double* rays, double* out) {
    for (uint64_t i = 0; i < n; i++) {
        const double* r = rays + 6 * i;
        Hit h;
        bool hit = os->s.intersect(make_ray(V3{r[0], r[1], r[2]}, V3{r[3], r[4], r[5]}), &h, nullptr);
        out[4 * i] = hit ? h.t : -1.0;
        out[4 * i + 1] = hit ? h.st[0] : 0.0;
        out[4 * i + 2] = hit ? h.st[1] : 0.0;
        out[4 * i + 3] = hit ? h.st_density : 0.0;
    }
}

void oracle_texture_sample(uint32_t w, uint32_t h, const float* rgb, int wrap, uint64_t n, const double* q,
                           float* out) {
    Texture t;
    t.build(rgb, w, h);
    for (uint64_t i = 0; i < n; i++) {
        const double* c = q + 7 * i;
        if (c[6] != 0.0) {
            const double du[2] = {c[2], c[3]}, dv[2] = {c[4], c[5]};
            t.sample_ewa(c[0], c[1], du, dv, wrap, out + 3 * i);
        } else {
            t.sample(c[0], c[1], c[2], wrap, out + 3 * i);
        }
    }
}

void oracle_ies_eval(uint32_t n_v, uint32_t n_h, const double* v, const double* h, const double* candela,
                     uint64_t n, const double* dirs, double* cd, double* factor) {
    Ies p;
    p.v.assign(v, v + n_v);
    p.h.assign(h, h + n_h);
    p.cd.assign(candela, candela + (size_t)n_v * n_h);
    p.finish();
    for (uint64_t i = 0; i < n; i++) {
        V3 d{dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]};
        cd[i] = p.candela(d);
        factor[i] = p.factor(d);
    }
}

void oracle_filter_sample(int filter, double width, uint64_t n, const double* u, double* out) {
    Camera c{};
    c.filter = filter;
    c.filter_width = width;
    for (uint64_t i = 0; i < n; i++) out[i] = c.sample_1d(u[i]);
}

}  // extern "C"

uint64_t oracle_medium_sample(const rt_medium_desc* md, const double* o, const double* d, double t_max,
                              const double* beta, uint64_t pixel, uint64_t sample, uint64_t n, double* pass_sum,
                              double* scat_sum) {
    const Medium m = medium_from(*md);
    Pcg32 rng = Pcg32::for_pixel_sample(pixel, sample);
    V3 ps{0, 0, 0}, ss{0, 0, 0};
    uint64_t scatters = 0;
    for (uint64_t i = 0; i < n; i++) {
        MediumEvent ev = sample_distance(m, v3(o), v3(d), t_max, v3(beta), rng);
        if (ev.scatter) {
            ss = ss + ev.weight;
            scatters++;
        } else {
            ps = ps + ev.weight;
        }
    }
    pass_sum[0] = ps.x, pass_sum[1] = ps.y, pass_sum[2] = ps.z;
    scat_sum[0] = ss.x, scat_sum[1] = ss.y, scat_sum[2] = ss.z;
    return scatters;
}

void oracle_medium_transmittance(const rt_medium_desc* md, const double* o, const double* d, double dist,
                                 uint64_t pixel, uint64_t sample, uint64_t n, double* mean) {
    const Medium m = medium_from(*md);
    Pcg32 rng = Pcg32::for_pixel_sample(pixel, sample);
    V3 sum{0, 0, 0};
    for (uint64_t i = 0; i < n; i++) sum = sum + medium_transmittance(m, v3(o), v3(d), dist, rng);
    mean[0] = sum.x / (double)n, mean[1] = sum.y / (double)n, mean[2] = sum.z / (double)n;
}

void oracle_medium_density(const rt_medium_desc* md, uint64_t n, const double* p, double* out) {
    const Medium m = medium_from(*md);
    for (uint64_t i = 0; i < n; i++) out[i] = m.density_at(v3(p + 3 * i));
}

void oracle_hg_phase(double g, uint64_t n, const double* c, double* out) {
    for (uint64_t i = 0; i < n; i++) out[i] = hg_phase(g, c[i]);
}

void oracle_hg_sample(double g, const double* wo, uint64_t n, const double* u, double* out) {
    for (uint64_t i = 0; i < n; i++) {
        double pdf;
        V3 wi = hg_sample(g, v3(wo), u[2 * i], u[2 * i + 1], &pdf);
        out[4 * i] = wi.x, out[4 * i + 1] = wi.y, out[4 * i + 2] = wi.z, out[4 * i + 3] = pdf;
    }
}

void oracle_sss_medium(const double* color, const double* dmfp, double* sigma_a, double* sigma_s) {
    Medium m = sss_medium(v3(color), v3(dmfp));
    sigma_a[0] = m.sigma_a.x, sigma_a[1] = m.sigma_a.y, sigma_a[2] = m.sigma_a.z;
    sigma_s[0] = m.sigma_s.x, sigma_s[1] = m.sigma_s.y, sigma_s[2] = m.sigma_s.z;
}

static HairParams hair_params(const double* p) {
    HairParams hp;
    hp.init(v3(p), p[3], p[4], p[5]);
    return hp;
}

void oracle_hair_eval(const double* params, uint64_t n, const double* q, double* f, double* pdf) {
    const HairParams hp = hair_params(params);
    for (uint64_t i = 0; i < n; i++) {
        const double* r = q + 7 * i;
        V3 v = hair_f(hp, v3(r), v3(r + 3), r[6]);
        f[3 * i] = v.x, f[3 * i + 1] = v.y, f[3 * i + 2] = v.z;
        pdf[i] = hair_pdf(hp, v3(r), v3(r + 3), r[6]);
    }
}

void oracle_hair_sample(const double* params, const double* wo, double h, uint64_t pixel, uint64_t sample,
                        uint64_t n, double* out) {
    const HairParams hp = hair_params(params);
    Pcg32 rng = Pcg32::for_pixel_sample(pixel, sample);
    for (uint64_t i = 0; i < n; i++) {
        V3 wi{0, 0, 0}, fv{0, 0, 0};
        double pdf = 0.0;
        if (!hair_sample(hp, v3(wo), h, rng, &wi, &fv, &pdf)) pdf = 0.0;
        double* o = out + 7 * i;
        o[0] = wi.x, o[1] = wi.y, o[2] = wi.z, o[3] = fv.x, o[4] = fv.y, o[5] = fv.z, o[6] = pdf;
    }
}

double oracle_fiber_h(const double* tangent, const double* normal, const double* wo) {
    return FiberFrame(v3(tangent), v3(normal), v3(wo)).h;
}

void oracle_curve_segment(const double* p0, const double* p1, double v0, double v1, uint64_t n, const double* rays,
                          double* out) {
    CurveSet cs;
    for (int k = 0; k < 4; k++) {
        cs.p0.push_back((float)p0[k]);
        cs.p1.push_back((float)p1[k]);
    }
    cs.v0.push_back((float)v0);
    cs.v1.push_back((float)v1);
    for (uint64_t i = 0; i < n; i++) {
        Ray r{v3(rays + 6 * i), v3(rays + 6 * i + 3)};
        double t, v;
        V3 nn, tg;
        double* o = out + 8 * i;
        if (cs.intersect_segment(r, 0, INF, &t, &nn, &tg, &v)) {
            o[0] = t, o[1] = nn.x, o[2] = nn.y, o[3] = nn.z, o[4] = tg.x, o[5] = tg.y, o[6] = tg.z, o[7] = v;
        } else {
            for (int k = 0; k < 8; k++) o[k] = k == 0 ? -1.0 : 0.0;
        }
    }
}


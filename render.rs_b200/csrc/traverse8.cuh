// traverse8.cuh — group traversal: one ray per 8 lanes.
//
// The 8-wide BVH has one child per lane: lane c of a group decodes and tests
// child c of the current node, and tests triangle c (and c + 8) of a leaf.
// Group-wide shuffles then choose the nearest child (continue), rank the
// other hit children far-to-near for the group's shared-memory stack, and
// reduce triangle hits to the closest. Every lane of a group executes the
// same instruction stream, so the warp's only divergence is between its
// four groups (which also alternate node and leaf phases together).
//
// Same answers as the per-lane traversal in traverse.cuh: the same child
// boxes and the same watertight triangle test, closest hit with ties broken
// by the lower leaf-order triangle index.
#pragma once

#include "traverse.cuh"

namespace rt {

#define G8_STACK 192  // entries per group (shared memory, 8 B each)

struct GroupRay {
    RayPre r;
    float3 o, d;          // world ray
    TraceHit hit;
    uint32_t cur;         // node reference being processed
    uint32_t pending;     // parked leaf (bit 31 set), 0 = none
    uint32_t cur_inst;
    uint32_t steps;
    int sp, inst_sp;
    bool in_inst, found, need_pop;
};

__device__ __forceinline__ bool g8_begin(const DevScene& S, GroupRay& g, float3 o, float3 d, float t_max) {
    g.hit.t = t_max;
    g.hit.tri = 0xFFFFFFFFu;
    g.hit.inst = 0xFFFFFFFFu;
    g.hit.b1 = g.hit.b2 = 0.0f;
    g.o = o;
    g.d = d;
    g.in_inst = false;
    g.found = false;
    g.need_pop = false;
    g.pending = 0;
    g.inst_sp = 0;
    g.cur_inst = 0;
    g.steps = 0;
    g.sp = 0;
    if (S.n_instances == 0) return false;
    ray_pre(g.r, o, d);
    g.cur = S.tlas_root;
    return true;
}

// Next stack entry that can still hold a closer hit. False: stack empty.
__device__ __forceinline__ bool g8_pop(GroupRay& g, const uint2* stk) {
    for (;;) {
        if (g.in_inst && g.sp == g.inst_sp) {
            g.in_inst = false;
            ray_pre(g.r, g.o, g.d);
        }
        if (g.sp == 0) return false;
        uint2 e = stk[--g.sp];
        if (__uint_as_float(e.y) < g.hit.t) {
            g.need_pop = false;
            if (e.x & REF_LEAF) {
                g.pending = e.x;
                g.need_pop = true;
            } else {
                g.cur = e.x;
            }
            return true;
        }
    }
}

// Test the 8 children of g.cur, one per lane. Returns true on a stack overflow.
template <bool ANY>
__device__ __forceinline__ bool g8_node(const DevScene& S, GroupRay& g, uint2* stk, uint32_t c, uint32_t gmask,
                                        uint32_t gshift) {
    const uint4* n = S.nodes + (size_t)g.cur * WIDE_NODE_WORDS;
    uint4 w0 = __ldg(n), w1 = __ldg(n + 1), w2 = __ldg(n + 2), w3 = __ldg(n + 3);
    uint32_t ref = __ldg(reinterpret_cast<const uint32_t*>(n + 4) + c);
    float sx = __uint_as_float((w0.w & 0xFFu) << 23);
    float sy = __uint_as_float(((w0.w >> 8) & 0xFFu) << 23);
    float sz = __uint_as_float(((w0.w >> 16) & 0xFFu) << 23);
    float px = __uint_as_float(w0.x) - 8388608.0f * sx;
    float py = __uint_as_float(w0.y) - 8388608.0f * sy;
    float pz = __uint_as_float(w0.z) - 8388608.0f * sz;
    const bool hi4 = c >= 4;
    const uint32_t sel = 0x7440u | (c & 3u);
    auto qf = [&](uint32_t w) { return __uint_as_float(__byte_perm(w, 0x4B000000u, sel)); };
    float lox = fmaf(qf(hi4 ? w1.y : w1.x), sx, px), hix = fmaf(qf(hi4 ? w2.w : w2.z), sx, px);
    float loy = fmaf(qf(hi4 ? w1.w : w1.z), sy, py), hiy = fmaf(qf(hi4 ? w3.y : w3.x), sy, py);
    float loz = fmaf(qf(hi4 ? w2.y : w2.x), sz, pz), hiz = fmaf(qf(hi4 ? w3.w : w3.z), sz, pz);
    const RayPre& r = g.r;
    float t0x = (lox - r.o.x) * r.inv.x, t1x = (hix - r.o.x) * r.inv.x;
    float t0y = (loy - r.o.y) * r.inv.y, t1y = (hiy - r.o.y) * r.inv.y;
    float t0z = (loz - r.o.z) * r.inv.z, t1z = (hiz - r.o.z) * r.inv.z;
    float tnear = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fmaxf(fminf(t0z, t1z), 0.0f));
    float tfar = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fminf(fmaxf(t0z, t1z), g.hit.t));
    tfar *= RT_ROBUST_SCALE;
    const bool hit = c < (w0.w >> 24) && ref != REF_EMPTY && tnear <= tfar;
    const uint32_t hm = (__ballot_sync(gmask, hit) >> gshift) & 0xFFu;
    if (!hm) {
        g.need_pop = true;
        return false;
    }
    const float key = hit ? tnear : INFINITY;
    uint32_t keep;  // child the group continues with
    if (ANY) {
        keep = __ffs(hm) - 1;
    } else {
        // Nearest hit child: min over (t, lane), 3 butterfly steps.
        float bt = key;
        uint32_t bi = c;
#pragma unroll
        for (int off = 4; off > 0; off >>= 1) {
            float ot = __shfl_xor_sync(gmask, bt, off, 8);
            uint32_t oi = __shfl_xor_sync(gmask, bi, off, 8);
            if (ot < bt || (ot == bt && oi < bi)) {
                bt = ot;
                bi = oi;
            }
        }
        keep = bi;
    }
    const uint32_t next = __shfl_sync(gmask, ref, keep, 8);
    const uint32_t others = hm & ~(1u << keep);
    const int npush = __popc(others);
    if (g.sp + npush > G8_STACK) return true;
    if (npush) {
        // Far-to-near: an entry sits above every entry that is farther
        // (ties: the higher lane index lies deeper).
        int rank = 0;
        bool mine = (others >> c) & 1u;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            float tj = __shfl_sync(gmask, key, j, 8);
            if (((others >> j) & 1u) && (tj > key || (tj == key && (uint32_t)j > c))) rank++;
        }
        if (mine) stk[g.sp + rank] = make_uint2(ref, __float_as_uint(ANY ? 0.0f : tnear));
        g.sp += npush;
    }
    if (next & REF_LEAF) {
        g.pending = next;
        g.need_pop = true;
    } else {
        g.cur = next;
    }
    return false;
}

// Process the parked leaf. Returns true when the query is over (any-hit
// found, or a stack overflow).
template <bool ANY>
__device__ __forceinline__ bool g8_leaf(const DevScene& S, GroupRay& g, uint2* stk, uint32_t c, uint32_t gmask,
                                        uint32_t gshift) {
    const uint32_t leaf = g.pending;
    g.pending = 0;
    const uint32_t first = leaf & LEAF_FIRST_MASK;
    const uint32_t count = ((leaf >> 27) & 15u) + 1u;
    if (!g.in_inst) {
        // TLAS leaf: defer the extra instances, enter the first.
        if (g.sp + (int)count - 1 > G8_STACK) return true;
        // Entry k holds instance first + count - 1 - k, so first + 1 ends on top.
#pragma unroll
        for (uint32_t k = c; k < 16; k += 8)
            if (k + 1 < count) stk[g.sp + (int)k] = make_uint2(make_leaf_ref(first + count - 1 - k, 1), 0u);
        g.sp += (int)count - 1;
        g.cur_inst = first;
        float4 x0 = __ldg(S.inst_xf + 3 * (size_t)first), x1 = __ldg(S.inst_xf + 3 * (size_t)first + 1),
               x2 = __ldg(S.inst_xf + 3 * (size_t)first + 2);
        uint32_t root = __ldg(&S.inst[first].x);
        ray_pre(g.r, xf_point(x0, x1, x2, g.o), xf_vec(x0, x1, x2, g.d));
        g.in_inst = true;
        g.inst_sp = g.sp;
        if (root == 0xFFFFFFFFu) {
            g.need_pop = true;
        } else {
            g.cur = root;
            g.need_pop = false;
        }
        return false;
    }
    // BLAS leaf: lane c tests triangles c and c + 8.
    float bt = g.hit.t, b1 = 0.f, b2 = 0.f;
    uint32_t bi = 0xFFFFFFFFu;
#pragma unroll
    for (uint32_t k = 0; k < 2; k++) {
        uint32_t i = c + 8 * k;
        if (i < count) {
            const float4* tp = S.tris + 3 * (size_t)(first + i);
            float4 a = __ldg(tp), b = __ldg(tp + 1), cc = __ldg(tp + 2);
            float t, u, v;
            if (tri_watertight(g.r, xyz(a), xyz(b), xyz(cc), bt, t, u, v)) {
                bt = t;
                bi = i;
                b1 = u;
                b2 = v;
            }
        }
    }
    if (ANY) {
        const uint32_t any = (__ballot_sync(gmask, bi != 0xFFFFFFFFu) >> gshift) & 0xFFu;
        if (any) {
            g.found = true;
            return true;
        }
        g.need_pop = true;
        return false;
    }
    // Closest over the group: min over (t, leaf index).
#pragma unroll
    for (int off = 4; off > 0; off >>= 1) {
        float ot = __shfl_xor_sync(gmask, bt, off, 8);
        uint32_t oi = __shfl_xor_sync(gmask, bi, off, 8);
        float o1 = __shfl_xor_sync(gmask, b1, off, 8);
        float o2 = __shfl_xor_sync(gmask, b2, off, 8);
        if (oi != 0xFFFFFFFFu && (bi == 0xFFFFFFFFu || ot < bt || (ot == bt && oi < bi))) {
            bt = ot;
            bi = oi;
            b1 = o1;
            b2 = o2;
        }
    }
    if (bi != 0xFFFFFFFFu) {
        g.hit.t = bt;
        g.hit.tri = first + bi;
        g.hit.inst = g.cur_inst;
        g.hit.b1 = b1;
        g.hit.b2 = b2;
        g.found = true;
    }
    g.need_pop = true;
    return false;
}

// Persistent pump at group granularity: 4 rays per warp in flight; idle
// groups are refilled (one warp-aggregated atomic) whenever two or more
// groups are idle. load(j, o, d, tmax) reads work item j (all 8 lanes of the
// group call it with the same j); finish(done, j, g) is called by the whole
// warp whenever a group finished, with `done` true on lane 0 of each
// finished group only.
template <bool ANY, class Load, class Finish>
__device__ __forceinline__ void g8_pump(const DevScene& S, uint32_t n, uint32_t* fetch, uint32_t* err, uint2* stk,
                                        Load load, Finish finish) {
    const uint32_t lane = threadIdx.x & 31u, c = lane & 7u, grp = lane >> 3, gshift = grp * 8;
    const uint32_t gmask = 0xFFu << gshift;
    GroupRay g;
    bool active = false, exhausted = false;
    uint32_t item = 0;
    for (;;) {
        uint32_t act = __ballot_sync(0xFFFFFFFFu, active);
        uint32_t idle_groups = 0;
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (((act >> (8 * k)) & 0xFFu) == 0) idle_groups |= 1u << k;
        if (!exhausted && __popc(idle_groups) >= 2) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(fetch, (uint32_t)__popc(idle_groups));
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if (base >= n || n - base <= (uint32_t)__popc(idle_groups)) exhausted = true;
            bool fresh = false;
            if ((idle_groups >> grp) & 1u) {
                uint32_t j = base + __popc(idle_groups & ((1u << grp) - 1u));
                if (base < n && j < n) {
                    item = j;
                    float3 o, d;
                    float tmax;
                    load(j, o, d, tmax);
                    active = g8_begin(S, g, o, d, tmax);
                    fresh = !active;  // empty scene: a miss, finished at once
                }
            }
            if (__any_sync(0xFFFFFFFFu, fresh)) finish(fresh && c == 0, item, g);
            act = __ballot_sync(0xFFFFFFFFu, active);
        }
        if (act == 0) {
            if (exhausted) break;
            continue;
        }
        // Node phase: groups without a parked leaf test nodes / pop.
        for (;;) {
            const bool want = active && g.pending == 0;
            if (!__any_sync(0xFFFFFFFFu, want)) break;
            bool done_now = false;
            if (want) {
                if (++g.steps > RT_MAX_TRAV_STEPS) {
                    if (c == 0) atomicOr(err, RT_DEVERR_ITER);
                    done_now = true;
                } else if (g.need_pop) {
                    done_now = !g8_pop(g, stk);
                } else if (g8_node<ANY>(S, g, stk, c, gmask, gshift)) {
                    if (c == 0) atomicOr(err, RT_DEVERR_STACK);
                    done_now = true;
                }
            }
            if (__any_sync(0xFFFFFFFFu, done_now)) finish(done_now && c == 0, item, g);
            if (done_now) active = false;
        }
        // Leaf phase: every group with a parked leaf processes it.
        bool done_now = false;
        if (active && g.pending) {
            if (g8_leaf<ANY>(S, g, stk, c, gmask, gshift)) {
                done_now = true;
                if (!g.found && c == 0) atomicOr(err, RT_DEVERR_STACK);
            }
        }
        if (__any_sync(0xFFFFFFFFu, done_now)) finish(done_now && c == 0, item, g);
        if (done_now) active = false;
    }
}

}  // namespace rt

// Ray traversal of the compressed 8-wide BVH: closest hit and any hit.
//
// Semantics follow meshAccelTraceRay (PathTracerLib/src/MeshAccel/
// MeshAccelIntersectCore.h:110-221):
//   * the direction is normalised first (zero length -> (0, 0, -1));
//   * triangles are intersected with the reference's Moller-Trumbore
//     (:52-108), rounded exactly like the reference (no FMA contraction), and
//     accepted when tMin <= t <= closest; of several hits at exactly the same t
//     the one with the highest original triangle index wins (the reference
//     keeps the last one its own traversal order meets).  The rule depends
//     neither on the visiting order nor on the BVH's layout -- the parallel
//     top-down collapse places nodes and leaves in an order that differs
//     between builds -- so every kernel, and every build of the same scene,
//     picks the same triangle;
//   * a hit is reported only if the final t < tMax;
//   * quirk Q1: a direction component with |d| <= 1e-8 gets a zero reciprocal
//     in the reference, which turns every slab test into "does the box contain
//     the origin in the other axes" and fails all boxes when tMin > 0.  The
//     reference's leaves are single triangles with exact bounds, so this is
//     reproduced independently of the tree by testing only triangles whose
//     exact bounds contain the origin in the non-degenerate axes (traceQ1).
// Child boxes are quantised outward, so the tree is conservative; the slab
// test widens tExit by 2^-21 relative to absorb its own rounding.
#pragma once

#include "pt_common.cuh"

namespace pt {

// Tuning knobs (compile-time; the defaults are the measured best).
#ifndef PT_SHARED_STACK
#define PT_SHARED_STACK 20
#endif
#ifndef PT_POSTPONE_LANES
#define PT_POSTPONE_LANES 8
#endif
constexpr int kTraversalStack = 32;                 // entries of the local-memory stack (fallback / Q1 path)
constexpr int kSharedStack = PT_SHARED_STACK;       // entries per thread of the shared-memory stack
constexpr int kPostponeLanes = PT_POSTPONE_LANES;   // postpone triangle tests when fewer lanes want them
constexpr float kSlabWiden = 1.0000005f;

// Original triangle index of the triangle at leaf position k.
__device__ __forceinline__ uint32_t leafId(const TriVerts* __restrict__ tris, uint32_t k)
{
    return __float_as_uint(__ldg(&tris[k].v0.w));
}

struct HitRec {
    float t;
    float u;
    float v;
    uint32_t tri;  // original triangle index (instanced scene: shading-record index), 0xFFFFFFFF = miss
    uint32_t inst; // instance of the hit in an instanced scene, else 0xFFFFFFFF
};

// Moller-Trumbore, MeshAccelIntersectCore.h:52-93, exact rounding.
__device__ __forceinline__ bool intersectTriExact(
    float3 o, float3 d, float3 v0, float3 v1, float3 v2, float tMin, float tMax, float& t, float& u, float& v)
{
    const float3 e1 = xsub(v1, v0);
    const float3 e2 = xsub(v2, v0);
    const float3 p = xcross(d, e2);
    const float det = xdot(e1, p);
    if (fabsf(det) < 1.0e-8f) {
        return false;
    }
    const float invDet = __fdiv_rn(1.0f, det);
    const float3 tv = xsub(o, v0);
    const float bu = __fmul_rn(xdot(tv, p), invDet);
    if (bu < 0.0f || bu > 1.0f) {
        return false;
    }
    const float3 q = xcross(tv, e1);
    const float bv = __fmul_rn(xdot(d, q), invDet);
    if (bv < 0.0f || __fadd_rn(bu, bv) > 1.0f) {
        return false;
    }
    const float tt = __fmul_rn(xdot(e2, q), invDet);
    if (tt < tMin || tt > tMax) {
        return false;
    }
    t = tt;
    u = bu;
    v = bv;
    return true;
}

// Shading normal and uv at a hit (MeshAccelIntersectCore.h:95-106 and the
// final renormalisation at :215), exact rounding.
__device__ __forceinline__ void hitShading(const TriShade& s, float3 dn, float bu, float bv, float3& n, float& tu, float& tv)
{
    const float bw = __fsub_rn(__fsub_rn(1.0f, bu), bv);
    const float3 n0 = f3(s.a.x, s.a.y, s.a.z), n1 = f3(s.b.x, s.b.y, s.b.z), n2 = f3(s.c.x, s.c.y, s.c.z);
    float3 m = xnormalize(xadd(xadd(xscl(n0, bw), xscl(n1, bu)), xscl(n2, bv)));
    if (xdot(m, dn) > 0.0f) {
        m = xscl(m, -1.0f);
    }
    n = xnormalize(m);
    tu = __fadd_rn(__fadd_rn(__fmul_rn(s.a.w, bw), __fmul_rn(s.c.w, bu)), __fmul_rn(s.d.y, bv));
    tv = __fadd_rn(__fadd_rn(__fmul_rn(s.b.w, bw), __fmul_rn(s.d.x, bu)), __fmul_rn(s.d.z, bv));
}

// Affine transforms of an instance (rows r[0..2]: linear part, translation in w).
__device__ __forceinline__ float3 xformPoint(const float4* r, float3 p)
{
    return f3(fmaf(r[0].x, p.x, fmaf(r[0].y, p.y, fmaf(r[0].z, p.z, r[0].w))),
        fmaf(r[1].x, p.x, fmaf(r[1].y, p.y, fmaf(r[1].z, p.z, r[1].w))),
        fmaf(r[2].x, p.x, fmaf(r[2].y, p.y, fmaf(r[2].z, p.z, r[2].w))));
}
__device__ __forceinline__ float3 xformVector(const float4* r, float3 v)
{
    return f3(fmaf(r[0].x, v.x, fmaf(r[0].y, v.y, r[0].z * v.z)), fmaf(r[1].x, v.x, fmaf(r[1].y, v.y, r[1].z * v.z)),
        fmaf(r[2].x, v.x, fmaf(r[2].y, v.y, r[2].z * v.z)));
}
// Normal to world space: the transpose of the world -> object linear part.
__device__ __forceinline__ float3 xformNormal(const float4* w2o, float3 n)
{
    return f3(fmaf(w2o[0].x, n.x, fmaf(w2o[1].x, n.y, w2o[2].x * n.z)),
        fmaf(w2o[0].y, n.x, fmaf(w2o[1].y, n.y, w2o[2].y * n.z)),
        fmaf(w2o[0].z, n.x, fmaf(w2o[1].z, n.y, w2o[2].z * n.z)));
}

// Shading normal (facing the world ray dn) and uv of a hit in any scene: for
// an instanced scene the interpolated object-space normal is carried to world
// space before the flip.
__device__ __forceinline__ void hitShadingAt(const DevScene& S, const TriShade& sh, uint32_t inst, float3 dn, float bu,
    float bv, float3& n, float& tu, float& tv)
{
    if (inst == 0xFFFFFFFFu || S.instanceCount == 0) {
        hitShading(sh, dn, bu, bv, n, tu, tv);
        return;
    }
    const float bw = __fsub_rn(__fsub_rn(1.0f, bu), bv);
    const float3 n0 = f3(sh.a.x, sh.a.y, sh.a.z), n1 = f3(sh.b.x, sh.b.y, sh.b.z), n2 = f3(sh.c.x, sh.c.y, sh.c.z);
    const float3 mo = xadd(xadd(xscl(n0, bw), xscl(n1, bu)), xscl(n2, bv));
    float3 m = xnormalize(xformNormal(S.instances[inst].w2o, mo));
    if (xdot(m, dn) > 0.0f) {
        m = xscl(m, -1.0f);
    }
    n = m;
    tu = __fadd_rn(__fadd_rn(__fmul_rn(sh.a.w, bw), __fmul_rn(sh.c.w, bu)), __fmul_rn(sh.d.y, bv));
    tv = __fadd_rn(__fadd_rn(__fmul_rn(sh.b.w, bw), __fmul_rn(sh.d.x, bu)), __fmul_rn(sh.d.z, bv));
}

__device__ __forceinline__ bool isDegenerateDir(float3 dn)
{
    return !(fabsf(dn.x) > 1.0e-8f) || !(fabsf(dn.y) > 1.0e-8f) || !(fabsf(dn.z) > 1.0e-8f);
}

// Intersects the ray with the eight quantised child boxes of a node.
// Returns the hit mask: bits 24..31 internal children (slot ^ octinv), bits
// 0..23 leaf triangles (node-local offsets).
__device__ __forceinline__ uint32_t intersectChildren(const CwNode* __restrict__ nodes, uint32_t idx, float3 o,
    float3 idir, uint32_t octinv, float tMin, float tMax, uint32_t& childBase, uint32_t& triBase, uint32_t& imask)
{
    const uint4* np = reinterpret_cast<const uint4*>(nodes + idx);
    const uint4 w0 = __ldg(np + 0);
    const uint4 w1 = __ldg(np + 1);
    const uint4 w2 = __ldg(np + 2);
    const uint4 w3 = __ldg(np + 3);
    const uint4 w4 = __ldg(np + 4);
    const float px = __uint_as_float(w0.x), py = __uint_as_float(w0.y), pz = __uint_as_float(w0.z);
    const uint32_t ex = w0.w & 0xffu, ey = (w0.w >> 8) & 0xffu, ez = (w0.w >> 16) & 0xffu;
    imask = w0.w >> 24;
    childBase = w1.x;
    triBase = w1.y;
    const float ax = __uint_as_float(ex << 23) * idir.x;
    const float ay = __uint_as_float(ey << 23) * idir.y;
    const float az = __uint_as_float(ez << 23) * idir.z;
    const float bx = (px - o.x) * idir.x;
    const float by = (py - o.y) * idir.y;
    const float bz = (pz - o.z) * idir.z;
    // near/far plane words per axis (quantised lo/hi swapped for negative directions)
    const bool sx = idir.x < 0.0f, sy = idir.y < 0.0f, sz = idir.z < 0.0f;
    const uint32_t nearX[2] = {sx ? w3.z : w2.x, sx ? w3.w : w2.y};
    const uint32_t farX[2] = {sx ? w2.x : w3.z, sx ? w2.y : w3.w};
    const uint32_t nearY[2] = {sy ? w4.x : w2.z, sy ? w4.y : w2.w};
    const uint32_t farY[2] = {sy ? w2.z : w4.x, sy ? w2.w : w4.y};
    const uint32_t nearZ[2] = {sz ? w4.z : w3.x, sz ? w4.w : w3.y};
    const uint32_t farZ[2] = {sz ? w3.x : w4.z, sz ? w3.y : w4.w};
    const uint32_t meta[2] = {w1.z, w1.w};
    uint32_t hitmask = 0;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int sh = 8 * j;
            const float t0x = fmaf(static_cast<float>((nearX[h] >> sh) & 0xffu), ax, bx);
            const float t0y = fmaf(static_cast<float>((nearY[h] >> sh) & 0xffu), ay, by);
            const float t0z = fmaf(static_cast<float>((nearZ[h] >> sh) & 0xffu), az, bz);
            const float t1x = fmaf(static_cast<float>((farX[h] >> sh) & 0xffu), ax, bx);
            const float t1y = fmaf(static_cast<float>((farY[h] >> sh) & 0xffu), ay, by);
            const float t1z = fmaf(static_cast<float>((farZ[h] >> sh) & 0xffu), az, bz);
            const float tEnter = fmaxf(fmaxf(t0x, t0y), fmaxf(t0z, tMin));
            const float tExit = fminf(fminf(t1x, t1y), fminf(t1z, tMax)) * kSlabWiden;
            const uint32_t m = (meta[h] >> sh) & 0xffu;
            if (tEnter <= tExit) {
                const uint32_t inner = ((m & 0x18u) == 0x18u) ? octinv : 0u;
                hitmask |= (m >> 5) << ((m ^ inner) & 0x1fu);
            }
        }
    }
    return hitmask;
}

// Slow path for quirk Q1 (degenerate direction components); see the file comment.
static __device__ __noinline__ bool traceQ1(const DevScene& S, float3 o, float3 dn, float tMin, float tMax, bool anyHit,
    HitRec& out, unsigned int* overflowCounter)
{
    out.tri = 0xFFFFFFFFu;
    out.inst = 0xFFFFFFFFu;
    if (tMin > 0.0f || S.nodeCount == 0) {
        return false;
    }
    const bool useX = fabsf(dn.x) > 1.0e-8f, useY = fabsf(dn.y) > 1.0e-8f, useZ = fabsf(dn.z) > 1.0e-8f;
    uint32_t stack[kTraversalStack * 2];
    int sp = 0;
    bool dropped = false;
    stack[sp++] = 0;
    float closest = tMax;
    uint32_t best = 0xFFFFFFFFu;
    float bu = 0.0f, bv = 0.0f;
    while (sp > 0) {
        const uint32_t idx = stack[--sp];
        const uint4* np = reinterpret_cast<const uint4*>(S.nodes + idx);
        const uint4 w0 = np[0], w1 = np[1], w2 = np[2], w3 = np[3], w4 = np[4];
        const float p[3] = {__uint_as_float(w0.x), __uint_as_float(w0.y), __uint_as_float(w0.z)};
        const float sc[3] = {__uint_as_float((w0.w & 0xffu) << 23), __uint_as_float(((w0.w >> 8) & 0xffu) << 23),
            __uint_as_float(((w0.w >> 16) & 0xffu) << 23)};
        const uint32_t imask = w0.w >> 24;
        const uint64_t qlo[3] = {w2.x | (uint64_t(w2.y) << 32), w2.z | (uint64_t(w2.w) << 32),
            w3.x | (uint64_t(w3.y) << 32)};
        const uint64_t qhi[3] = {w3.z | (uint64_t(w3.w) << 32), w4.x | (uint64_t(w4.y) << 32),
            w4.z | (uint64_t(w4.w) << 32)};
        const uint64_t meta = w1.z | (uint64_t(w1.w) << 32);
        const float oo[3] = {o.x, o.y, o.z};
        const bool use[3] = {useX, useY, useZ};
        int rank = 0;
        for (int s = 0; s < 8; ++s) {
            const uint32_t m = static_cast<uint32_t>(meta >> (8 * s)) & 0xffu;
            const bool inner = (imask >> s) & 1u;
            bool pass = m != 0u;
            for (int a = 0; a < 3 && pass; ++a) {
                if (!use[a]) {
                    continue;
                }
                const float lo = fmaf(static_cast<float>((qlo[a] >> (8 * s)) & 0xffu), sc[a], p[a]);
                const float hi = fmaf(static_cast<float>((qhi[a] >> (8 * s)) & 0xffu), sc[a], p[a]);
                pass = lo <= oo[a] && oo[a] <= hi;
            }
            if (inner) {
                if (pass) {
                    if (sp < kTraversalStack * 2) {
                        stack[sp++] = w1.x + rank;
                    } else {
                        dropped = true; // a full stack drops the child, like the reference's 64-entry stack
                    }
                }
                ++rank;
                continue;
            }
            if (!pass) {
                continue;
            }
            const int cnt = __popc(m >> 5);
            const int off = m & 0x1f;
            for (int k = 0; k < cnt; ++k) {
                const TriVerts tv = S.tris[w1.y + off + k];
                const float3 v0 = f3(tv.v0.x, tv.v0.y, tv.v0.z), v1 = f3(tv.v1.x, tv.v1.y, tv.v1.z),
                             v2 = f3(tv.v2.x, tv.v2.y, tv.v2.z);
                const float lo3[3] = {fminf(fminf(v0.x, v1.x), v2.x), fminf(fminf(v0.y, v1.y), v2.y),
                    fminf(fminf(v0.z, v1.z), v2.z)};
                const float hi3[3] = {fmaxf(fmaxf(v0.x, v1.x), v2.x), fmaxf(fmaxf(v0.y, v1.y), v2.y),
                    fmaxf(fmaxf(v0.z, v1.z), v2.z)};
                bool inside = true;
                for (int a = 0; a < 3; ++a) {
                    if (use[a] && !(lo3[a] <= oo[a] && oo[a] <= hi3[a])) {
                        inside = false;
                    }
                }
                float t, u, v;
                const uint32_t id = __float_as_uint(tv.v0.w);
                if (inside && intersectTriExact(o, dn, v0, v1, v2, tMin, closest, t, u, v)) {
                    if (anyHit && t < tMax) {
                        out.t = t;
                        out.u = u;
                        out.v = v;
                        out.tri = id;
                        return true;
                    }
                    if (t < closest || id > best || best == 0xFFFFFFFFu) {
                        closest = t;
                        best = id; // (original index; see the tie rule above)
                        bu = u;
                        bv = v;
                    }
                }
            }
        }
    }
    if (dropped && overflowCounter != nullptr) {
        atomicAdd(overflowCounter, 1u);
    }
    if (best != 0xFFFFFFFFu && closest < tMax) {
        out.t = closest;
        out.u = bu;
        out.v = bv;
        out.tri = best;
        return true;
    }
    return false;
}

// Two-level traversal of an instanced scene: the top-level BVH's leaves are
// instances; on reaching one, the ray goes to the object's space
// (o' = W2O o, d' = W2O d, unnormalised, so t is the same parameter) and the
// object's BVH is traversed on the same stack above the top level's entries;
// when those are used up the world ray is restored.  Exact-t ties go to the
// larger (instance, original triangle index) pair.
template <bool AnyHit, bool Count>
__device__ __noinline__ bool traceInstanced(const DevScene& S, float3 o, float3 dn, float tMin, float tMax, HitRec& out,
    unsigned int* overflowCounter, unsigned long long* visits, uint2* sstack, int sstride)
{
    out.tri = 0xFFFFFFFFu;
    out.inst = 0xFFFFFFFFu;
    float3 ro = o, idir;
    uint32_t oct = 0, octinv = 7;
    auto setRay = [&](float3 a, float3 d) {
        ro = a;
        const float dx = fabsf(d.x) < 1.0e-20f ? copysignf(1.0e-20f, d.x) : d.x;
        const float dy = fabsf(d.y) < 1.0e-20f ? copysignf(1.0e-20f, d.y) : d.y;
        const float dz = fabsf(d.z) < 1.0e-20f ? copysignf(1.0e-20f, d.z) : d.z;
        idir = f3(__frcp_rn(dx), __frcp_rn(dy), __frcp_rn(dz));
        oct = (d.x < 0.0f ? 4u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 1u : 0u);
        octinv = 7u - oct;
    };
    setRay(o, dn);
    float3 rd = dn;
    const CwNode* nodes = S.tlasNodes;
    const TriVerts* leaves = S.tlasLeaves;
    int level = 0, base = 0;
    uint32_t curInst = 0, curTriBase = 0;
    uint2 stack[kTraversalStack];
    int sp = 0;
    uint2 ngroup = make_uint2(0u, 0x80000000u | (1u << oct));
    uint2 tgroup = make_uint2(0u, 0u);
    float closest = tMax;
    unsigned long long bestKey = ~0ull;
    uint32_t bestTri = 0xFFFFFFFFu, bestInst = 0xFFFFFFFFu;
    float bu = 0.0f, bv = 0.0f;
    bool overflow = false;
    uint32_t nodeVisits = 0, triVisits = 0;
    auto push = [&](uint2 g) -> bool {
        if (sstack != nullptr && sp < kSharedStack) {
            sstack[sp * sstride] = g;
        } else if (sp < (sstack != nullptr ? kSharedStack : 0) + kTraversalStack) {
            stack[sp - (sstack != nullptr ? kSharedStack : 0)] = g;
        } else {
            return false;
        }
        ++sp;
        return true;
    };
    while (true) {
        if (ngroup.y > 0x00FFFFFFu) {
            const uint32_t bit = 31u - __clz(ngroup.y);
            ngroup.y &= ~(1u << bit);
            const uint32_t slot = (bit - 24u) ^ octinv;
            const uint32_t child = ngroup.x + __popc(ngroup.y & 0xffu & ((1u << slot) - 1u));
            if (ngroup.y > 0x00FFFFFFu && !push(ngroup)) {
                overflow = true;
            }
            uint32_t childBase, triBase, imask;
            const uint32_t hits = intersectChildren(nodes, child, ro, idir, octinv, tMin, closest, childBase, triBase,
                imask);
            if (Count) {
                ++nodeVisits;
            }
            ngroup = make_uint2(childBase, (hits & 0xFF000000u) | imask);
            tgroup = make_uint2(triBase, hits & 0x00FFFFFFu);
        } else {
            tgroup = ngroup;
            ngroup = make_uint2(0u, 0u);
        }
        while (tgroup.y != 0u) {
            if (level == 0) {
                // an instance: descend into its object
                const int k = __ffs(tgroup.y) - 1;
                tgroup.y &= tgroup.y - 1u;
                const uint32_t inst = __float_as_uint(__ldg(&leaves[tgroup.x + k].v0.w));
                bool saved = true;
                if (ngroup.y > 0x00FFFFFFu) {
                    saved = push(ngroup);
                }
                if (saved && tgroup.y != 0u) {
                    saved = push(tgroup);
                }
                if (!saved) {
                    overflow = true; // the rest of this top-level group is dropped
                }
                const DevInstance& I = S.instances[inst];
                const DevBlas B = S.blases[I.meta.x];
                curInst = inst;
                curTriBase = B.triBase;
                nodes = B.nodes;
                leaves = B.tris;
                rd = xformVector(I.w2o, dn);
                setRay(xformPoint(I.w2o, o), rd);
                level = 1;
                base = sp;
                ngroup = make_uint2(0u, B.nodeCount > 0 ? (0x80000000u | (1u << oct)) : 0u);
                tgroup = make_uint2(0u, 0u);
                break;
            }
            if (ngroup.y > 0x00FFFFFFu && __popc(__activemask()) < kPostponeLanes && push(tgroup)) {
                break;
            }
            const int k = __ffs(tgroup.y) - 1;
            tgroup.y &= tgroup.y - 1u;
            const TriVerts tv = leaves[tgroup.x + k];
            float t, u, v;
            if (Count) {
                ++triVisits;
            }
            if (intersectTriExact(ro, rd, f3(tv.v0.x, tv.v0.y, tv.v0.z), f3(tv.v1.x, tv.v1.y, tv.v1.z),
                    f3(tv.v2.x, tv.v2.y, tv.v2.z), tMin, closest, t, u, v)) {
                const unsigned long long key = (static_cast<unsigned long long>(curInst) << 32) |
                    static_cast<unsigned long long>(__float_as_uint(tv.v0.w));
                if (AnyHit) {
                    if (t < tMax) {
                        if (Count) {
                            atomicAdd(&visits[0], static_cast<unsigned long long>(nodeVisits));
                            atomicAdd(&visits[1], static_cast<unsigned long long>(triVisits));
                        }
                        out.t = t;
                        out.u = u;
                        out.v = v;
                        out.tri = curTriBase + __float_as_uint(tv.v0.w);
                        out.inst = curInst;
                        return true;
                    }
                } else if (t < closest || key > bestKey || bestKey == ~0ull) {
                    closest = t;
                    bestKey = key;
                    bestTri = curTriBase + __float_as_uint(tv.v0.w);
                    bestInst = curInst;
                    bu = u;
                    bv = v;
                }
            }
        }
        if (ngroup.y <= 0x00FFFFFFu) {
            if (level == 1 && sp == base) {
                // the object is done: back to the top level in world space
                level = 0;
                nodes = S.tlasNodes;
                leaves = S.tlasLeaves;
                rd = dn;
                setRay(o, dn);
            }
            if (ngroup.y <= 0x00FFFFFFu) {
                if (sp == 0) {
                    break;
                }
                --sp;
                if (sstack != nullptr && sp < kSharedStack) {
                    ngroup = sstack[sp * sstride];
                } else {
                    ngroup = stack[sp - (sstack != nullptr ? kSharedStack : 0)];
                }
            }
        }
    }
    if (overflow && overflowCounter != nullptr) {
        atomicAdd(overflowCounter, 1u);
    }
    if (Count) {
        atomicAdd(&visits[0], static_cast<unsigned long long>(nodeVisits));
        atomicAdd(&visits[1], static_cast<unsigned long long>(triVisits));
    }
    if (!AnyHit && bestTri != 0xFFFFFFFFu && closest < tMax) {
        out.t = closest;
        out.u = bu;
        out.v = bv;
        out.tri = bestTri;
        out.inst = bestInst;
        return true;
    }
    return false;
}

// Closest hit (AnyHit = false) or occlusion (AnyHit = true) for a normalised
// direction dn. Returns true on a hit; out.tri is the ORIGINAL triangle index.
// Count = true adds the nodes and triangles visited to visits[0] / visits[1].
// The traversal stack lives in shared memory when `sstack` is given (this
// thread's column of a [kSharedStack][blockDim] array, so that consecutive
// threads hit consecutive banks), spilling to a local array beyond that.
// Inst = true compiles the instanced-scene branch in (kernels launched for
// scenes without instances use Inst = false and keep their register budget).
template <bool AnyHit, bool Count = false, bool Inst = false>
__device__ __forceinline__ bool traceRay(const DevScene& S, float3 o, float3 dn, float tMin, float tMax, HitRec& out,
    unsigned int* overflowCounter = nullptr, unsigned long long* visits = nullptr, uint2* sstack = nullptr,
    int sstride = 0)
{
    out.tri = 0xFFFFFFFFu;
    out.inst = 0xFFFFFFFFu;
    if constexpr (Inst) {
        if (S.instanceCount > 0) {
            return traceInstanced<AnyHit, Count>(S, o, dn, tMin, tMax, out, overflowCounter, visits, sstack, sstride);
        }
    }
    if (S.nodeCount == 0) {
        return false;
    }
    if (isDegenerateDir(dn)) {
        return traceQ1(S, o, dn, tMin, tMax, AnyHit, out, overflowCounter);
    }
    const float3 idir = f3(__frcp_rn(dn.x), __frcp_rn(dn.y), __frcp_rn(dn.z));
    const uint32_t oct = (dn.x < 0.0f ? 4u : 0u) | (dn.y < 0.0f ? 2u : 0u) | (dn.z < 0.0f ? 1u : 0u);
    const uint32_t octinv = 7u - oct;
    uint2 stack[kTraversalStack];
    int sp = 0;
    uint2 ngroup = make_uint2(0u, 0x80000000u | (1u << oct));
    float closest = tMax;
    uint32_t best = 0xFFFFFFFFu;
    float bu = 0.0f, bv = 0.0f;
    bool overflow = false;
    uint32_t nodeVisits = 0, triVisits = 0;
    uint2 tgroup = make_uint2(0u, 0u);
    auto push = [&](uint2 g) -> bool {
        if (sstack != nullptr && sp < kSharedStack) {
            sstack[sp * sstride] = g;
        } else if (sp < (sstack != nullptr ? kSharedStack : 0) + kTraversalStack) {
            stack[sp - (sstack != nullptr ? kSharedStack : 0)] = g;
        } else {
            return false;
        }
        ++sp;
        return true;
    };
    while (true) {
        if (ngroup.y > 0x00FFFFFFu) {
            // descend into the nearest remaining child of the current node group
            const uint32_t bit = 31u - __clz(ngroup.y);
            ngroup.y &= ~(1u << bit);
            const uint32_t slot = (bit - 24u) ^ octinv;
            const uint32_t child = ngroup.x + __popc(ngroup.y & 0xffu & ((1u << slot) - 1u));
            if (ngroup.y > 0x00FFFFFFu && !push(ngroup)) {
                overflow = true;
            }
            uint32_t childBase, triBase, imask;
            const uint32_t hits = intersectChildren(S.nodes, child, o, idir, octinv, tMin, closest, childBase, triBase,
                imask);
            if (Count) {
                ++nodeVisits;
            }
            ngroup = make_uint2(childBase, (hits & 0xFF000000u) | imask);
            tgroup = make_uint2(triBase, hits & 0x00FFFFFFu);
        } else {
            // a group popped without node hits holds postponed triangles
            tgroup = ngroup;
            ngroup = make_uint2(0u, 0u);
        }
        while (tgroup.y != 0u) {
            // Postpone the triangle tests while few lanes of the warp have any and this
            // lane can keep descending (Ylitie, Karras & Laine 2017); they are retried
            // from the stack, so SIMT lanes test triangles together.
            if (ngroup.y > 0x00FFFFFFu && __popc(__activemask()) < kPostponeLanes && push(tgroup)) {
                break;
            }
            const int k = __ffs(tgroup.y) - 1;
            tgroup.y &= tgroup.y - 1u;
            const TriVerts tv = S.tris[tgroup.x + k];
            float t, u, v;
            if (Count) {
                ++triVisits;
            }
            if (intersectTriExact(o, dn, f3(tv.v0.x, tv.v0.y, tv.v0.z), f3(tv.v1.x, tv.v1.y, tv.v1.z),
                    f3(tv.v2.x, tv.v2.y, tv.v2.z), tMin, closest, t, u, v)) {
                if (AnyHit) {
                    if (t < tMax) {
                        if (Count) {
                            atomicAdd(&visits[0], static_cast<unsigned long long>(nodeVisits));
                            atomicAdd(&visits[1], static_cast<unsigned long long>(triVisits));
                        }
                        out.t = t;
                        out.u = u;
                        out.v = v;
                        out.tri = __float_as_uint(tv.v0.w);
                        return true;
                    }
                } else if (t < closest || best == 0xFFFFFFFFu ||
                           leafId(S.tris, tgroup.x + k) > leafId(S.tris, best)) {
                    // an exact tie in t goes to the higher original triangle index,
                    // whatever the visiting order and the BVH's layout (both ids are
                    // read again only on a tie, which keeps no register live)
                    closest = t;
                    best = tgroup.x + k;
                    bu = u;
                    bv = v;
                }
            }
        }
        if (ngroup.y <= 0x00FFFFFFu) {
            if (sp == 0) {
                break;
            }
            --sp;
            if (sstack != nullptr && sp < kSharedStack) {
                ngroup = sstack[sp * sstride];
            } else {
                ngroup = stack[sp - (sstack != nullptr ? kSharedStack : 0)];
            }
        }
    }
    if (overflow && overflowCounter != nullptr) {
        atomicAdd(overflowCounter, 1u);
    }
    if (Count) {
        atomicAdd(&visits[0], static_cast<unsigned long long>(nodeVisits));
        atomicAdd(&visits[1], static_cast<unsigned long long>(triVisits));
    }
    if (!AnyHit && best != 0xFFFFFFFFu && closest < tMax) {
        out.t = closest;
        out.u = bu;
        out.v = bv;
        out.tri = leafId(S.tris, best);
        return true;
    }
    return false;
}

} // namespace pt

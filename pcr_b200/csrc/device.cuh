// Device functions of the wavefront path tracer.
//
// Intersection arithmetic uses explicit round-to-nearest intrinsics
// (__fmul_rn/__fadd_rn/__fsub_rn/__fdiv_rn/__fsqrt_rn), which nvcc never
// fuses into FMA, so every hit test performs the reference's float
// operations in the reference's order (x86-64 g++ -O2 issues no FMA).  That is
// what makes hit primitive ids bit-exact against the reference BVH.  Shading
// arithmetic is free to contract.
#pragma once

#include <cfloat>
#include <cstdint>

#include "layout.h"

namespace pcr {

// ----------------------------------------------------------------- exact ops
namespace ex {
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return make_float3(sub(a.x, b.x), sub(a.y, b.y), sub(a.z, b.z)); }
__device__ __forceinline__ float3 add3(float3 a, float3 b) { return make_float3(add(a.x, b.x), add(a.y, b.y), add(a.z, b.z)); }
__device__ __forceinline__ float3 scale3(float3 a, float s) { return make_float3(mul(a.x, s), mul(a.y, s), mul(a.z, s)); }
// Vec3f::dot (Vec3f.h:16-19): (a0*b0 + a1*b1) + a2*b2
__device__ __forceinline__ float dot(float3 a, float3 b) { return add(add(mul(a.x, b.x), mul(a.y, b.y)), mul(a.z, b.z)); }
// Vec3f::cross (Vec3f.h:21-28)
__device__ __forceinline__ float3 cross(float3 a, float3 b)
{
    return make_float3(sub(mul(a.y, b.z), mul(a.z, b.y)), sub(mul(a.z, b.x), mul(a.x, b.z)),
                       sub(mul(a.x, b.y), mul(a.y, b.x)));
}
__device__ __forceinline__ float3 normalize(float3 a)
{
    float m = __fsqrt_rn(dot(a, a));
    return make_float3(div(a.x, m), div(a.y, m), div(a.z, m));
}
}  // namespace ex

__device__ __forceinline__ float3 xyz(float4 v) { return make_float3(v.x, v.y, v.z); }
__device__ __forceinline__ float3 f3add(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 f3sub(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 f3mul(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float f3dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 f3neg(float3 a) { return make_float3(-a.x, -a.y, -a.z); }

// ----------------------------------------------------------------- primitives
// Sphere::intersect (code/Includes/Sphere.h:20-40)
__device__ __forceinline__ bool sphere_hit(const DSphere& s, float3 o, float3 d, float& t0)
{
    using namespace ex;
    float4 cr = s.c_r;
    float3 cp = sub3(make_float3(cr.x, cr.y, cr.z), o);
    float rayLen = dot(d, cp);
    float tSq = sub(dot(cp, cp), mul(rayLen, rayLen));
    float r2 = mul(cr.w, cr.w);
    if (tSq > r2) return false;
    float tDist = __fsqrt_rn(sub(r2, tSq));
    t0 = sub(rayLen, tDist);
    float t1 = add(rayLen, tDist);
    if (t0 < 0) t0 = t1;
    if (t0 < 0) return false;
    return true;
}

// One-instruction reciprocal (PTX rcp.approx.ftz.f32) for conservative
// pre-filters only; never for a value the reference computes.
__device__ __forceinline__ float rcp_approx(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Plane::intersect (code/Includes/Plane.h:33-54); uu, vv precomputed with
// the same dot the reference evaluates per call.
//
// The three IEEE divides are first decided by a reciprocal product: for
// x > 0, y > 0 normal, x * rcp_approx(y) is within 2^-21 relative of x / y
// (the instruction's reciprocal is within 2 ulp, the product adds half an
// ulp), so a product beyond a bound by 2^-20 fixes the comparison the
// correctly rounded quotient would make.  Only the t of planes that survive, and quotients near
// a bound, are divided exactly; the accept/reject decisions and t are the
// same as dividing every time.  t0 is only meaningful when true is returned.
__device__ __forceinline__ bool plane_hit(const DPlane& p, float3 o, float3 d, float closest, float& t0)
{
    using namespace ex;
    const float kUp = 1.f + 9.5367431640625e-07f, kDown = 1.f - 9.5367431640625e-07f;  // 1 +- 2^-20
    float4 nA = p.n_emit;
    float3 N = make_float3(nA.x, nA.y, nA.z);
    float denom = dot(d, N);
    if (fabsf(denom) <= 1e-6f) return false;
    float4 oM = p.o_mat;
    float3 po = make_float3(oM.x, oM.y, oM.z);
    float num = dot(sub3(po, o), N);
    // t = num / denom is <= 0 when the signs differ (or num is zero)
    const float an = denom > 0.f ? num : -num;
    if (an <= 0.f) return false;
    const float tq = an * rcp_approx(fabsf(denom));
    if (tq > closest * kUp || tq < 1e-6f * kDown) return false;
    float t = div(num, denom);
    t0 = t;
    // every caller keeps a hit only when t < closest (first tested wins a
    // tie), so t == closest is rejected here already
    if (t <= 1e-6f || t >= closest) return false;
    float3 lh = sub3(add3(o, scale3(d, t)), po);
    float4 u = p.u_uu, v = p.v_vv;
    float a = dot(lh, make_float3(u.x, u.y, u.z));
    float b = dot(lh, make_float3(v.x, v.y, v.z));
    // s = a / uu, q = b / vv must lie in [0, 1]; uu, vv > 0.  a < -1e-20
    // makes s negative (|a / uu| stays far above the smallest subnormal for
    // any |u| < 1e12).
    if (a < -1e-20f || b < -1e-20f) return false;
    const float sa = a * rcp_approx(u.w), qa = b * rcp_approx(v.w);
    if (sa > kUp || qa > kUp) return false;
    // s and q only feed the range test: an estimate inside (0, 1) by more
    // than its error margin (a, b > 1e-30, far from underflow) decides it
    // as the correctly rounded quotient would, so only estimates near 0 or
    // 1 are divided exactly
    const bool s_in = a > 1e-30f && sa < kDown, q_in = b > 1e-30f && qa < kDown;
    if (!s_in) {
        const float sx = div(a, u.w);
        if (sx > 1.f || sx < 0.f) return false;
    }
    if (!q_in) {
        const float qx = div(b, v.w);
        if (qx > 1.f || qx < 0.f) return false;
    }
    return true;
}

// Triangle::intersect (code/Includes/Triangle.h:53-92), Moller-Trumbore.
__device__ __forceinline__ bool tri_hit(float4 a, float4 b, float4 c, float3 o, float3 d, float closest,
                                        float& t_out, float& u_out, float& v_out)
{
    using namespace ex;
    float3 v0 = make_float3(a.x, a.y, a.z), e1 = make_float3(b.x, b.y, b.z), e2 = make_float3(c.x, c.y, c.z);
    float3 pvec = cross(d, e2);
    float det = dot(e1, pvec);
    if (fabsf(det) < 1e-6f) return false;
    // Clear rejections are decided before the exact reciprocal: with
    // r = rcp_approx(det), x * r is within 2^-21 relative of x * (1 / det),
    // so a product below -1e-30 (far from underflow) is negative in the
    // exact arithmetic too, and one beyond a bound by 2^-20 (2^-19 for the
    // sum of two) is beyond it there.  Triangles that pass run the
    // reference's arithmetic unchanged.
    const float kUp = 1.f + 9.5367431640625e-07f, kUp2 = 1.f + 1.9073486328125e-06f;
    const float kDown = 1.f - 9.5367431640625e-07f;
    const float r = rcp_approx(det);
    float3 tvec = sub3(o, v0);
    const float U = dot(tvec, pvec);
    const float ua = U * r;
    if (ua < -1e-30f || ua > kUp) return false;
    float3 qvec = cross(tvec, e1);
    const float V = dot(d, qvec);
    const float va = V * r;
    if (va < -1e-30f || ua + va > kUp2) return false;
    const float T = dot(e2, qvec);
    const float ta = T * r;
    if (ta < 1e-6f * kDown || ta > closest * kUp) return false;
    float invDet = div(1.f, det);
    float u = mul(U, invDet);
    if (u < 0.f || u > 1.f) return false;
    float v = mul(V, invDet);
    if (v < 0.f || add(u, v) > 1.f) return false;
    float t = mul(T, invDet);
    if (t <= 1e-6f || t >= closest) return false;
    t_out = t;
    u_out = u;
    v_out = v;
    return true;
}

// The shadow test's distance check (code/Renderer.cpp:852-860): a hit at t
// blocks when lightDist2 - 1e-3 > |hit - origin|^2, the hit point and its
// squared distance taken with the reference's float operations and the
// comparison in double (`lim` = lightDist2 - 1e-3 in double).
__device__ __forceinline__ bool blocks_at(float3 o, float3 d, float t, double lim)
{
    const float3 sh = make_float3(__fadd_rn(o.x, __fmul_rn(d.x, t)), __fadd_rn(o.y, __fmul_rn(d.y, t)),
                                  __fadd_rn(o.z, __fmul_rn(d.z, t)));
    const float3 dd = ex::sub3(sh, o);
    return lim > (double)ex::dot(dd, dd);
}

// One child box of a 4-wide node with the reference's slab arithmetic
// (code/Bvh/Bvh.cpp:294-311), branch-free: the reference returns at the
// first axis where tmin > tmax, and since tmin only grows and tmax only
// shrinks, testing once after all three axes gives the same answer.  NaN
// lanes are ignored the way std::max/std::min ignore a NaN second argument.
// Returns tNear, or +inf for a miss.
__device__ __forceinline__ float slab4(float lx, float hx, float ly, float hy, float lz, float hz, float3 o, float3 inv,
                                       float segMax)
{
    using namespace ex;
    float tmin = 0.f, tmax = segMax;
    float t1 = mul(sub(lx, o.x), inv.x), t2 = mul(sub(hx, o.x), inv.x);
    float a = t1 > t2 ? t2 : t1, b = t1 > t2 ? t1 : t2;
    tmin = (tmin < a) ? a : tmin;
    tmax = (b < tmax) ? b : tmax;
    t1 = mul(sub(ly, o.y), inv.y); t2 = mul(sub(hy, o.y), inv.y);
    a = t1 > t2 ? t2 : t1; b = t1 > t2 ? t1 : t2;
    tmin = (tmin < a) ? a : tmin;
    tmax = (b < tmax) ? b : tmax;
    t1 = mul(sub(lz, o.z), inv.z); t2 = mul(sub(hz, o.z), inv.z);
    a = t1 > t2 ? t2 : t1; b = t1 > t2 ? t1 : t2;
    tmin = (tmin < a) ? a : tmin;
    tmax = (b < tmax) ? b : tmax;
    return tmin > tmax ? __int_as_float(0x7f800000) : tmin;
}

__device__ __forceinline__ void cas(float& ta, int& ca, float& tb, int& cb)
{
    if (tb < ta) {
        const float t = ta; ta = tb; tb = t;
        const int c = ca; ca = cb; cb = c;
    }
}

struct TraceCounts { int nodes, tris; };

// Closest hit over the 4-wide BVH: ordered traversal with the stack in
// local memory; the nearest hit child is visited next without a push, the
// others are pushed far-to-near.  `closest` comes in as the best t from
// spheres/planes.  Returns the leaf-order triangle index or -1; t/u/v of the
// hit.  With kAny (shadow rays over a mesh without emissive triangles) it
// returns -2 as soon as a hit closer than `closest` blocks (blocks_at with
// `lim`).  Empty child slots carry the code 0x80000000 (a leaf of no
// triangles).
template <bool kCount, bool kAny = false>
__device__ __forceinline__ int bvh4_closest(const DScene& S, float3 o, float3 d, float& closest, float& hu, float& hv,
                                            TraceCounts* cnt, double lim = 0.0)
{
    if (S.n_nodes <= 0) return -1;
    const float inf = __int_as_float(0x7f800000);
    const float3 inv = make_float3(__fdiv_rn(1.f, d.x), __fdiv_rn(1.f, d.y), __fdiv_rn(1.f, d.z));
    int stk[kStackSize];
    float stt[kStackSize];
    int top = 0;
    int best = -1;
    int code = 0;        // the root
    float tcode = 0.f;
    while (true) {
        if (!(tcode > closest)) {
            if (code >= 0) {
                const DNode4* n = S.nodes + code;
                const float4 lx = __ldg(&n->lox), hx = __ldg(&n->hix), ly = __ldg(&n->loy), hy = __ldg(&n->hiy);
                const float4 lz = __ldg(&n->loz), hz = __ldg(&n->hiz);
                const int4 ch = __ldg(&n->child);
                if (kCount) cnt->nodes++;
                const int kEmpty = (int)0x80000000u;
                float t0 = ch.x != kEmpty ? slab4(lx.x, hx.x, ly.x, hy.x, lz.x, hz.x, o, inv, closest) : inf;
                float t1 = ch.y != kEmpty ? slab4(lx.y, hx.y, ly.y, hy.y, lz.y, hz.y, o, inv, closest) : inf;
                float t2 = ch.z != kEmpty ? slab4(lx.z, hx.z, ly.z, hy.z, lz.z, hz.z, o, inv, closest) : inf;
                float t3 = ch.w != kEmpty ? slab4(lx.w, hx.w, ly.w, hy.w, lz.w, hz.w, o, inv, closest) : inf;
                int c0 = ch.x, c1 = ch.y, c2 = ch.z, c3 = ch.w;
                const int k = (t0 < inf) + (t1 < inf) + (t2 < inf) + (t3 < inf);
                // the reference skips all children when they would overflow its stack
                if (k > 0 && top + k - 1 <= kStackSize) {
                    if constexpr (kAny) {
                        // A shadow query's answer does not depend on the
                        // visit order (blocked iff some hit in front of the
                        // bound blocks, and blocking is monotone in t): the
                        // first hit child in slot order is visited next, the
                        // others are pushed unsorted.
                        bool have = false;
                        auto take = [&](int c, float t) {
                            if (!(t < inf)) return;
                            if (!have) {
                                code = c;
                                tcode = t;
                                have = true;
                            } else {
                                stk[top] = c;
                                stt[top] = t;
                                top++;
                            }
                        };
                        take(c0, t0);
                        take(c1, t1);
                        take(c2, t2);
                        take(c3, t3);
                    } else {
                        // ascending by tNear; misses (+inf) last
                        cas(t0, c0, t1, c1);
                        cas(t2, c2, t3, c3);
                        cas(t0, c0, t2, c2);
                        cas(t1, c1, t3, c3);
                        cas(t1, c1, t2, c2);
                        if (k > 3) { stk[top] = c3; stt[top] = t3; top++; }
                        if (k > 2) { stk[top] = c2; stt[top] = t2; top++; }
                        if (k > 1) { stk[top] = c1; stt[top] = t1; top++; }
                        code = c0;
                        tcode = t0;
                    }
                    continue;
                }
            } else {
                const int first = code & 0x00FFFFFF;
                const int count = (code >> 24) & 0x7F;
                for (int i = 0; i < count; i++) {
                    const DTri* tr = S.tris + first + i;
                    float4 a = __ldg(&tr->v0_id), b = __ldg(&tr->e1_mat), c = __ldg(&tr->e2_flags);
                    if (kCount) cnt->tris++;
                    float t, u, v;
                    if (tri_hit(a, b, c, o, d, closest, t, u, v)) {
                        if (kAny && blocks_at(o, d, t, lim)) return -2;
                        closest = t;
                        hu = u;
                        hv = v;
                        best = first + i;
                    }
                }
            }
        }
        if (top == 0) break;
        --top;
        code = stk[top];
        tcode = stt[top];
    }
    return best;
}

// Conservative ray-box test for a plane group.  The box is padded on the
// host by well over the rounding error of a hit point, the segment end by
// 1e-4 relative; direction components below 1e-30 count as zero (the ray
// then moves less than the padding along that axis), the others enter as
// their 1-ulp rcp_approx, whose error the padding also covers.  A false
// answer means no plane of the group can be hit in (0, closest].
__device__ __forceinline__ bool group_axis(float lo, float hi, float o, float d, float r, float& tmin, float& tmax)
{
    if (fabsf(d) < 1e-30f) return o >= lo && o <= hi;
    const float t1 = (lo - o) * r, t2 = (hi - o) * r;
    tmin = fmaxf(tmin, fminf(t1, t2));
    tmax = fminf(tmax, fmaxf(t1, t2));
    return true;
}
__device__ __forceinline__ bool group_may_hit(float4 lo, float4 hi, float3 o, float3 d, float3 rd, float closest)
{
    float tmin = 0.f, tmax = closest * 1.0001f + 1e-4f;
    if (!group_axis(lo.x, hi.x, o.x, d.x, rd.x, tmin, tmax)) return false;
    if (!group_axis(lo.y, hi.y, o.y, d.y, rd.y, tmin, tmax)) return false;
    if (!group_axis(lo.z, hi.z, o.z, d.z, rd.z, tmin, tmax)) return false;
    return tmin <= tmax;
}

// The analytic part of Renderer::sceneIntersect (code/Renderer.cpp:891-949):
// spheres, then planes (light planes first); first-tested wins ties.
// Returns the primitive code (kPrimNone on a miss) with `closest` lowered to
// its t.
__device__ __forceinline__ uint32_t scene_analytic(const DScene& S, float3 o, float3 d, float& closest)
{
    uint32_t prim = kPrimNone;
    for (int i = 0; i < S.n_spheres; i++) {
        float t0;
        if (sphere_hit(S.spheres[i], o, d, t0) && t0 < closest) {
            closest = t0;
            prim = kPrimSphere | (uint32_t)i;
        }
    }
    // planes in order, a group's planes skipped together when the ray cannot
    // reach the group's (padded) box before `closest`; skipping planes that
    // cannot be hit leaves the closest hit and its tie order unchanged
    const float3 rd = make_float3(rcp_approx(d.x), rcp_approx(d.y), rcp_approx(d.z));
    for (int g = 0; g < S.n_pgroups; g++) {
        const float4 lo = S.pgroups[2 * g], hi = S.pgroups[2 * g + 1];
        const int first = __float_as_int(lo.w), count = __float_as_int(hi.w);
        if (count > 1 && !group_may_hit(lo, hi, o, d, rd, closest)) continue;
        for (int i = first; i < first + count; i++) {
            float t0;
            if (plane_hit(S.planes[i], o, d, closest, t0) && t0 < closest) {
                closest = t0;
                prim = kPrimPlane | (uint32_t)i;
            }
        }
    }
    return prim;
}

// Renderer::sceneIntersect: the analytic primitives, then the triangle BVH.
// Returns the primitive code; t and barycentrics through refs.
__device__ __forceinline__ uint32_t scene_closest(const DScene& S, float3 o, float3 d, float tmax, float& t, float& hu,
                                                  float& hv)
{
    float closest = tmax;
    uint32_t prim = scene_analytic(S, o, d, closest);
    int tri = bvh4_closest<false>(S, o, d, closest, hu, hv, nullptr);
    if (tri >= 0) prim = kPrimTri | (uint32_t)tri;
    t = closest;
    return prim;
}

// Shadow query with early exit: true when the closest hit of the segment
// would block (non-emissive and closer than the light, code/Renderer.cpp:852-
// 860).  The closest emissive sphere or plane is found first; nothing behind
// it can block.  Then the other spheres, the non-emissive planes (their own
// grouped copy) and the BVH are tested against that bound; a hit strictly in
// front of the bound is non-emissive, so it either blocks (return at once) or
// lies at the light and becomes the new bound.  A blocking hit found
// this way implies the closest hit blocks as well (the squared distance grows
// with t), so the answer is the closest-hit test's.  Scenes with emissive
// triangles, or with more emissive spheres or planes than the scene record
// lists, take the closest-hit route.
// The part of the shadow query before the triangle BVH: kShadowBlocked or
// kShadowLit when that already decides it (the closest-hit route of scenes
// with emissive triangles is decided here in full), else kShadowWalk with
// `bound` set for an any-hit walk of the BVH.
constexpr int kShadowLit = 0, kShadowBlocked = 1, kShadowWalk = 2;
__device__ __forceinline__ int scene_blocked_analytic(const DScene& S, const DMaterial* mats, float3 o, float3 d,
                                                      float tmax, double lim, float& bound)
{
    if (S.emissive_tris || S.n_emit_spheres < 0 || S.n_emit_planes < 0) {
        float t = FLT_MAX, hu, hv;
        const uint32_t prim = scene_closest(S, o, d, tmax, t, hu, hv);
        if ((prim & kPrimKindMask) == kPrimNone) return kShadowLit;
        const uint32_t kind = prim & kPrimKindMask, pidx = prim & kPrimIndexMask;
        int mi;
        if (kind == kPrimSphere) mi = S.spheres[pidx].mat.x;
        else if (kind == kPrimPlane) mi = __float_as_int(S.planes[pidx].o_mat.w);
        else mi = __float_as_int(S.tris[pidx].e1_mat.w);
        if (mats[S.mat_base + mi].flags & kMatEmissive) return kShadowLit;
        return blocks_at(o, d, t, lim) ? kShadowBlocked : kShadowLit;
    }
    bound = tmax;
    for (int k = 0; k < S.n_emit_spheres; k++) {
        float t0;
        if (sphere_hit(S.spheres[S.emit_spheres[k]], o, d, t0) && t0 < bound) bound = t0;
    }
    for (int k = 0; k < S.n_emit_planes; k++) {
        float t0;
        if (plane_hit(S.planes[S.emit_planes[k]], o, d, bound, t0) && t0 < bound) bound = t0;
    }
    for (int i = 0; i < S.n_spheres; i++) {
        float t0;
        if (sphere_hit(S.spheres[i], o, d, t0) && t0 < bound) {
            if (blocks_at(o, d, t0, lim)) return kShadowBlocked;
            bound = t0;
        }
    }
    const float3 rd = make_float3(rcp_approx(d.x), rcp_approx(d.y), rcp_approx(d.z));
    for (int g = 0; g < S.n_sgroups; g++) {
        const float4 lo = S.sgroups[2 * g], hi = S.sgroups[2 * g + 1];
        const int first = __float_as_int(lo.w), count = __float_as_int(hi.w);
        if (count > 1 && !group_may_hit(lo, hi, o, d, rd, bound)) continue;
        for (int i = first; i < first + count; i++) {
            float t0;
            if (plane_hit(S.splanes[i], o, d, bound, t0) && t0 < bound) {
                if (blocks_at(o, d, t0, lim)) return kShadowBlocked;
                bound = t0;
            }
        }
    }
    return S.n_nodes > 0 ? kShadowWalk : kShadowLit;
}

__device__ __forceinline__ bool scene_blocked(const DScene& S, const DMaterial* mats, float3 o, float3 d, float tmax,
                                              double lim)
{
    float bound = tmax, hu, hv;
    const int r = scene_blocked_analytic(S, mats, o, d, tmax, lim, bound);
    if (r != kShadowWalk) return r == kShadowBlocked;
    return bvh4_closest<false, true>(S, o, d, bound, hu, hv, nullptr, lim) == -2;
}

// ----------------------------------------------------------------- spectra
// The stage functions below use the exact (never-contracted) ops: the
// sigmoid 0.5 + p / (2 sqrt(1 + p^2)) cancels for strongly negative p, where
// a fused multiply-add would move the result by more than 1e-5 relative.
__device__ __forceinline__ float sigmoid_fit(float4 f, float lambda)
{
    // RGBToSpectrum::evalSigmoidFit (code/Includes/RGBToSpectrum.h:118-125)
    using namespace ex;
    float L = div(sub(lambda, 550.f), 150.f);
    float p = add(f.x, mul(L, add(f.y, mul(L, f.z))));
    return mul(add(0.5f, div(p, mul(2.f, __fsqrt_rn(add(1.f, mul(p, p)))))), f.w);
}

__device__ __forceinline__ float spectrum_lerp(const float* s, float lambda)
{
    // Spectrum::operator() (code/Includes/Spectrum.h:82-90)
    using namespace ex;
    if (lambda < 400.f || lambda > 700.f) return 0.f;
    float t = div(sub(lambda, 400.f), 5.0f);
    int i = (int)t;
    if (i >= kSpecN - 1) return s[kSpecN - 1];
    float f = sub(t, (float)i);
    return add(mul(s[i], sub(1.f, f)), mul(s[i + 1], f));
}

// Material::albedoAt / emissiveAt (code/Includes/Material.h:92-101)
__device__ __forceinline__ float albedo_at(const DMaterial& m, float lambda)
{
    if (m.flags & kMatTabA) return spectrum_lerp(m.tabA, lambda);
    float v = sigmoid_fit(m.afit, lambda);
    return v > 1.f ? 1.f : v;
}
__device__ __forceinline__ float emissive_at(const DMaterial& m, float lambda)
{
    if (m.flags & kMatTabE) return spectrum_lerp(m.tabE, lambda);
    return sigmoid_fit(m.efit, lambda);
}

// Wyman-Sloan-Shirley piecewise Gaussians (code/Includes/CIE.h:27-53)
__device__ __forceinline__ float wyman(float l, float mu, float s1, float s2)
{
    using namespace ex;
    float t = (l < mu) ? mul(sub(l, mu), s1) : mul(sub(l, mu), s2);
    // the exponential is taken in double and rounded once, which gives the
    // correctly rounded float result; x-bar's negative lobe cancels against
    // the other two near 500 nm, so a float exp's last-bit error would be
    // amplified past 1e-5 there
    return (float)exp((double)mul(mul(-0.5f, t), t));
}
// x-bar with the reference's float operations: its negative lobe cancels the
// other two near 501 nm, where the float evaluation's own rounding is a
// sizeable part of the (small) result
__device__ __forceinline__ float cmf_x(float l)
{
    using namespace ex;
    return sub(add(mul(0.362f, wyman(l, 442.0f, 0.0624f, 0.0374f)), mul(1.056f, wyman(l, 599.8f, 0.0264f, 0.0323f))),
               mul(0.065f, wyman(l, 501.1f, 0.0490f, 0.0382f)));
}
__device__ __forceinline__ float3 cmf(float l)
{
    using namespace ex;
    float x = cmf_x(l);
    float y = add(mul(0.821f, wyman(l, 568.8f, 0.0213f, 0.0247f)), mul(0.286f, wyman(l, 530.9f, 0.0613f, 0.0322f)));
    float z = add(mul(1.217f, wyman(l, 437.0f, 0.0845f, 0.0278f)), mul(0.681f, wyman(l, 459.0f, 0.0385f, 0.0725f)));
    return make_float3(x, y, z);
}

// XYZ -> linear sRGB, D65 (code/Includes/CIE.h:115-123)
__device__ __forceinline__ float3 xyz_to_srgb(float3 c)
{
    using namespace ex;
    return make_float3(sub(sub(mul(3.2404542f, c.x), mul(1.5371385f, c.y)), mul(0.4985314f, c.z)),
                       add(add(mul(-0.9692660f, c.x), mul(1.8760108f, c.y)), mul(0.0415560f, c.z)),
                       add(sub(mul(0.0556434f, c.x), mul(0.2040259f, c.y)), mul(1.0572252f, c.z)));
}

// ToneMap::reinhard / aces (code/Includes/ToneMap.h:14-39)
__device__ __forceinline__ float reinhard(float x) { return __fdiv_rn(x, __fadd_rn(x, 1.f)); }
__device__ __forceinline__ float aces(float x)
{
    using namespace ex;
    float v = div(mul(x, add(mul(2.51f, x), 0.03f)), add(mul(x, add(mul(2.43f, x), 0.59f)), 0.14f));
    return v < 0.f ? 0.f : (v > 1.f ? 1.f : v);
}
// (unsigned char)(255*c + 0.5f) as x86-64 lowers it: truncate to int32, keep
// the low byte (code/Renderer.cpp:379-381).
__device__ __forceinline__ unsigned char quantize(float c)
{
    float v = __fadd_rn(__fmul_rn(255.f, c), 0.5f);
    if (!(v > -2147483648.0f && v < 2147483648.0f)) return 0;
    return (unsigned char)(__float2int_rz(v) & 0xFF);
}

// ----------------------------------------------------------------- RNG
// Counter-based: pcg4d (Jarzynski & Olano, "Hash Functions for GPU
// Rendering", JCGT 2020) keyed on (pixel, sample|fork, seed^bounce, seed^dim).
// A path's random numbers depend only on its request seed, pixel, sample,
// fork channel, bounce and dimension, never on its queue slot, so a render
// is the same alone or batched with others.
__device__ __forceinline__ uint4 pcg4d(uint4 v)
{
    v.x = v.x * 1664525u + 1013904223u;
    v.y = v.y * 1664525u + 1013904223u;
    v.z = v.z * 1664525u + 1013904223u;
    v.w = v.w * 1664525u + 1013904223u;
    v.x += v.y * v.w; v.y += v.z * v.x; v.z += v.x * v.y; v.w += v.y * v.z;
    v.x ^= v.x >> 16; v.y ^= v.y >> 16; v.z ^= v.z >> 16; v.w ^= v.w >> 16;
    v.x += v.y * v.w; v.y += v.z * v.x; v.z += v.x * v.y; v.w += v.y * v.z;
    return v;
}
__device__ __forceinline__ float u01(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }
__device__ __forceinline__ float4 rand4(const DRequest& R, uint32_t pixel, uint32_t sample, uint32_t fork, uint32_t bounce,
                                        uint32_t dim)
{
    uint4 v = make_uint4(pixel, sample ^ (fork << 27), R.seed_lo ^ (bounce * 0x9E3779B9u),
                         R.seed_hi + dim * 0x85EBCA6Bu);
    v = pcg4d(v);
    return make_float4(u01(v.x), u01(v.y), u01(v.z), u01(v.w));
}

// Cosine hemisphere (code/Includes/Ray.h:37-53): disk sample, helper axis,
// T = normalize(N x helper), B = N x T.  The direction is not renormalised.
__device__ __forceinline__ float3 hemisphere(float3 N, float r1, float r2)
{
    float3 helper = fabsf(N.x) <= fabsf(N.y) ? make_float3(1.f, 0.f, 0.f) : make_float3(0.f, 1.f, 0.f);
    float3 T = make_float3(N.y * helper.z - N.z * helper.y, N.z * helper.x - N.x * helper.z,
                           N.x * helper.y - N.y * helper.x);
    float tl = rsqrtf(f3dot(T, T));
    T = f3mul(T, tl);
    float3 B = make_float3(N.y * T.z - N.z * T.y, N.z * T.x - N.x * T.z, N.x * T.y - N.y * T.x);
    float r = sqrtf(r1);
    float s, c;
    // hardware sine/cosine: |error| < 1e-6 on [0, 2pi), far below the
    // sample's own randomness
    __sincosf(6.28318548f * r2, &s, &c);
    float x = r * c, y = r * s;
    float z = sqrtf(fmaxf(0.f, 1.f - x * x - y * y));
    return make_float3(T.x * x + B.x * y + N.x * z, T.y * x + B.y * y + N.y * z, T.z * x + B.z * y + N.z * z);
}

}  // namespace pcr

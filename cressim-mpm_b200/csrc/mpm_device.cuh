// Device-side math, SDF geometry, rigid contact and slicer predicates of the B200 MPM engine.
//
// The formulas restate CRESSim-MPM's L1 functions (paths are inside the reference project):
//   quaternion rotation          include/math/quat.h:117-150
//   analytic / grid SDFs         include/geometry_utils/sdf.h:67-662
//   rigid contact and friction   src/solver/mpm_rigid_contact.h:101-399
//   slicer side test (cutting)   src/solver/mpm_rigid_contact.h:401-478
// Everything that feeds an integer or boolean result compared bit for bit (cell keys, slicer
// masks) is evaluated with explicitly rounded operations (__fmul_rn / __fadd_rn / ...), i.e. with
// no fused multiply-add, so that it equals the reference's host arithmetic on identical inputs.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/crmpm_b200.h"

namespace crb200
{
    constexpr float kEps = 1.1920928955078125e-07f; // FLT_EPSILON, the reference's CR_EPS
    constexpr float kMaxF32 = 3.4028234663852885981170418348452e+38F;
    constexpr int kMaxShapes = 64;

    enum GeomType : int
    {
        G_BOX = 0, G_SPHERE, G_PLANE, G_CAPSULE, G_TRIMESH, G_QUAD_SLICER, G_TRIMESH_SLICER, G_LINES, G_ARC
    };
    enum ShapeKind : int { S_STATIC = 0, S_KINEMATIC = 1, S_DYNAMIC = 2 };

    enum ShapeFlags : int
    {
        SF_SLICER = 1,  // at least one slicer geometry: P2G/G2P must test node sides
        SF_DYNAMIC = 2, // at least one dynamic shape: grid contact accumulates coupling force
    };

    // One rigid shape of a scene, gathered once per substep from the bound struct-of-arrays.
    // cull.x / cull.y: a node / particle whose local SDF lower bound (sdfLowerBound) is at least
    // this value cannot be in contact with the shape (+inf disables the test).
    struct __align__(16) ShapeRec
    {
        float4 pos, rot, invScale, linVel, angVel, params0, gparams, comInvMass, inertia0, inertia1, cull;
        int kind, gtype, id;
        int dynSlot; // rank among the scene's dynamic shapes (deterministic coupling), -1 otherwise
    };

    struct SdfPtrs
    {
        const int4 *dim;
        const float4 *lbcs;
        const float4 *data;
    };

    // ---------------------------------------------------------------------------------------
    // small vector helpers (fused multiply-add allowed)
    struct V3
    {
        float x, y, z;
    };
    __device__ __forceinline__ V3 v3(float a, float b, float c) { return V3{a, b, c}; }
    __device__ __forceinline__ V3 v3(const float4 &f) { return V3{f.x, f.y, f.z}; }
    __device__ __forceinline__ V3 v3(const float3 &f) { return V3{f.x, f.y, f.z}; }
    __device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
    __device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
    __device__ __forceinline__ V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
    __device__ __forceinline__ V3 operator/(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
    __device__ __forceinline__ V3 mul(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
    __device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
    __device__ __forceinline__ V3 cross(V3 a, V3 b)
    {
        return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
    }
    __device__ __forceinline__ float sq(V3 a) { return dot(a, a); }
    __device__ __forceinline__ V3 normalized(V3 v)
    {
        float s = sq(v);
        return s > 0.f ? v * rsqrtf(s) : v;
    }
    __device__ __forceinline__ float comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

    // sm_100's paired FP32 arithmetic: one instruction computes two lanes, each rounded as the
    // scalar fused multiply-add or multiply, so results equal the scalar code's bit for bit.
    // v + a * s
    __device__ __forceinline__ V3 fma3(V3 a, float s, V3 v)
    {
        const float2 lo = __ffma2_rn(make_float2(a.x, a.y), make_float2(s, s), make_float2(v.x, v.y));
        return v3(lo.x, lo.y, fmaf(a.z, s, v.z));
    }
    // a * s
    __device__ __forceinline__ V3 mul3(V3 a, float s)
    {
        const float2 lo = __fmul2_rn(make_float2(a.x, a.y), make_float2(s, s));
        return v3(lo.x, lo.y, a.z * s);
    }
    // acc[0..3] += (v.x, v.y, v.z, m) * s: a node's momentum and mass sums
    __device__ __forceinline__ void fma4acc(float acc[4], V3 v, float m, float s)
    {
        const float2 s2 = make_float2(s, s);
        const float2 lo = __ffma2_rn(make_float2(v.x, v.y), s2, make_float2(acc[0], acc[1]));
        const float2 hi = __ffma2_rn(make_float2(v.z, m), s2, make_float2(acc[2], acc[3]));
        acc[0] = lo.x;
        acc[1] = lo.y;
        acc[2] = hi.x;
        acc[3] = hi.y;
    }

    // Quaternion rotation (quat.h:117-150).
    __device__ __forceinline__ V3 qrot(const float4 &q, V3 v)
    {
        const float vx = 2.f * v.x, vy = 2.f * v.y, vz = 2.f * v.z;
        const float w2 = q.w * q.w - 0.5f;
        const float d2 = q.x * vx + q.y * vy + q.z * vz;
        return v3(vx * w2 + (q.y * vz - q.z * vy) * q.w + q.x * d2, vy * w2 + (q.z * vx - q.x * vz) * q.w + q.y * d2,
                  vz * w2 + (q.x * vy - q.y * vx) * q.w + q.z * d2);
    }
    __device__ __forceinline__ V3 qrotInv(const float4 &q, V3 v)
    {
        const float vx = 2.f * v.x, vy = 2.f * v.y, vz = 2.f * v.z;
        const float w2 = q.w * q.w - 0.5f;
        const float d2 = q.x * vx + q.y * vy + q.z * vz;
        return v3(vx * w2 - (q.y * vz - q.z * vy) * q.w + q.x * d2, vy * w2 - (q.z * vx - q.x * vz) * q.w + q.y * d2,
                  vz * w2 - (q.x * vy - q.y * vx) * q.w + q.z * d2);
    }

    // ---------------------------------------------------------------------------------------
    // Exactly rounded arithmetic (no contraction) for bit-exact integer and side outputs.
    namespace ex
    {
        __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
        __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
        __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
        __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
        __device__ __forceinline__ V3 add(V3 a, V3 b) { return v3(add(a.x, b.x), add(a.y, b.y), add(a.z, b.z)); }
        __device__ __forceinline__ V3 sub(V3 a, V3 b) { return v3(sub(a.x, b.x), sub(a.y, b.y), sub(a.z, b.z)); }
        __device__ __forceinline__ V3 mul(V3 a, V3 b) { return v3(mul(a.x, b.x), mul(a.y, b.y), mul(a.z, b.z)); }
        __device__ __forceinline__ V3 muls(V3 a, float s) { return v3(mul(a.x, s), mul(a.y, s), mul(a.z, s)); }
        __device__ __forceinline__ float dot(V3 a, V3 b) { return add(add(mul(a.x, b.x), mul(a.y, b.y)), mul(a.z, b.z)); }

        // quat.h:137-150, evaluated left to right as the host compiles it.
        __device__ __forceinline__ V3 qrotInv(const float4 &q, V3 v)
        {
            const float vx = mul(2.f, v.x), vy = mul(2.f, v.y), vz = mul(2.f, v.z);
            const float w2 = sub(mul(q.w, q.w), 0.5f);
            const float d2 = add(add(mul(q.x, vx), mul(q.y, vy)), mul(q.z, vz));
            return v3(add(sub(mul(vx, w2), mul(sub(mul(q.y, vz), mul(q.z, vy)), q.w)), mul(q.x, d2)),
                      add(sub(mul(vy, w2), mul(sub(mul(q.z, vx), mul(q.x, vz)), q.w)), mul(q.y, d2)),
                      add(sub(mul(vz, w2), mul(sub(mul(q.x, vy), mul(q.y, vx)), q.w)), mul(q.z, d2)));
        }

        // Trilinear SDF distance with the reference's value/weight pairing (sdf.h:243-276).
        __device__ __forceinline__ float trilinear(const SdfPtrs &s, int4 dim, int off, int bx, int by, int bz, V3 fr)
        {
            float vals[8];
#pragma unroll
            for (int dx = 0; dx <= 1; ++dx)
#pragma unroll
                for (int dy = 0; dy <= 1; ++dy)
#pragma unroll
                    for (int dz = 0; dz <= 1; ++dz)
                        vals[(dx << 2) | (dy << 1) | dz] =
                            __ldg(&s.data[off + ((bz + dz) * dim.x * dim.y) + ((by + dy) * dim.x) + (bx + dx)].w);
            const float ox = sub(1.f, fr.x), oy = sub(1.f, fr.y), oz = sub(1.f, fr.z);
            const float w[8] = {mul(mul(ox, oy), oz), mul(mul(fr.x, oy), oz), mul(mul(ox, fr.y), oz),
                                mul(mul(fr.x, fr.y), oz), mul(mul(ox, oy), fr.z), mul(mul(fr.x, oy), fr.z),
                                mul(mul(ox, fr.y), fr.z), mul(mul(fr.x, fr.y), fr.z)};
            float acc = 0.f;
#pragma unroll
            for (int i = 0; i < 8; ++i)
                acc = add(acc, mul(vals[i], w[i]));
            return acc;
        }

        // getGeometryModSdf (sdf.h:504-662): does the point project onto the slicer surface, and
        // on which side (signed distance in *d, gradient in *g).
        __device__ __forceinline__ bool modSdf(V3 lp, int gtype, const float4 &p0, const SdfPtrs &s, float *d, V3 *g)
        {
            if (gtype == G_QUAD_SLICER)
            {
                if (lp.x < -p0.x || lp.x > p0.x || lp.z < -p0.y || lp.z > p0.y)
                    return false;
                *g = v3(0.f, copysignf(1.f, lp.y), 0.f);
                *d = lp.y;
                return true;
            }
            if (gtype == G_TRIMESH_SLICER)
            {
                int off = __float_as_int(p0.x);
                const float4 spine = __ldg(&s.data[off]);
                if (isnan(spine.x))
                    return false;
                if (add(ex::dot(lp, v3(spine)), spine.w) > 0.f)
                    return false;
                off++;
                const int id = __float_as_int(p0.y);
                const float4 lb = __ldg(&s.lbcs[id]);
                const int4 dim = __ldg(&s.dim[id]);
                const V3 sp = v3(div(sub(lp.x, lb.x), lb.w), div(sub(lp.y, lb.y), lb.w), div(sub(lp.z, lb.z), lb.w));
                const int qx = __float2int_rz(add(sp.x, 0.5f)), qy = __float2int_rz(add(sp.y, 0.5f)),
                          qz = __float2int_rz(add(sp.z, 0.5f));
                if (qx < 1 || qx >= dim.x - 1 || qy < 1 || qy >= dim.y - 1 || qz < 1 || qz >= dim.z - 1)
                    return false;
                const float4 qv = __ldg(&s.data[off + (qz * dim.x * dim.y) + (qy * dim.x) + qx]);
                if (isnan(qv.w))
                    return false;
                const int bx = __float2int_rz(sp.x), by = __float2int_rz(sp.y), bz = __float2int_rz(sp.z);
                const V3 fr = v3(sub(sp.x, (float)bx), sub(sp.y, (float)by), sub(sp.z, (float)bz));
                const float iv = trilinear(s, dim, off, bx, by, bz, fr);
                if (isnan(iv))
                    return false;
                *d = iv;
                *g = (mul(qv.w, iv) < 0.f) ? v3(-qv.x, -qv.y, -qv.z) : v3(qv);
                return true;
            }
            return false;
        }
    } // namespace ex

    // checkOnDifferentSides (mpm_rigid_contact.h:401-478) for particle p1 and node position p2,
    // both given exactly as the reference forms them.  *normal (optional) is the side gradient at
    // p2 in the shape's local frame, as the reference returns it.
    __device__ __forceinline__ bool differentSides(V3 p1, V3 p2, const ShapeRec *sh, int num, const SdfPtrs &sdf,
                                                   V3 *normal)
    {
        for (int s = 0; s < num; ++s)
        {
            const ShapeRec &r = sh[s];
            if (r.gtype != G_QUAD_SLICER && r.gtype != G_TRIMESH_SLICER)
                continue;
            const V3 pos = v3(r.pos), isc = v3(r.invScale);
            const V3 r1 = ex::mul(ex::qrotInv(r.rot, ex::sub(p1, pos)), isc);
            float d1, d2;
            V3 g1, g2;
            if (!ex::modSdf(r1, r.gtype, r.gparams, sdf, &d1, &g1))
                continue;
            const V3 r2 = ex::mul(ex::qrotInv(r.rot, ex::sub(p2, pos)), isc);
            if (ex::modSdf(r2, r.gtype, r.gparams, sdf, &d2, &g2) && (signbit(d1) != signbit(d2)))
            {
                if (normal)
                {
                    V3 g = mul(g2, isc);
                    *normal = g * rsqrtf(sq(g));
                }
                return true;
            }
        }
        return false;
    }

    // ---------------------------------------------------------------------------------------
    // getGeometrySdf (sdf.h:67-496): gradient/distance in the shape's local (unscaled) frame.
    // Returns the slicer-spine flag; *tangent is written for lines and arcs.
    __device__ __forceinline__ float trilinearF(const SdfPtrs &s, int4 dim, int off, int bx, int by, int bz, V3 fr)
    {
        float vals[8];
#pragma unroll
        for (int dx = 0; dx <= 1; ++dx)
#pragma unroll
            for (int dy = 0; dy <= 1; ++dy)
#pragma unroll
                for (int dz = 0; dz <= 1; ++dz)
                    vals[(dx << 2) | (dy << 1) | dz] =
                        __ldg(&s.data[off + ((bz + dz) * dim.x * dim.y) + ((by + dy) * dim.x) + (bx + dx)].w);
        const float ox = 1.f - fr.x, oy = 1.f - fr.y, oz = 1.f - fr.z;
        const float w[8] = {ox * oy * oz, fr.x * oy * oz, ox * fr.y * oz, fr.x * fr.y * oz,
                            ox * oy * fr.z, fr.x * oy * fr.z, ox * fr.y * fr.z, fr.x * fr.y * fr.z};
        float acc = 0.f;
#pragma unroll
        for (int i = 0; i < 8; ++i)
            acc += vals[i] * w[i];
        return acc;
    }

    static __device__ __noinline__ bool geometrySdf(V3 lp, int gtype, const float4 &p0, const SdfPtrs &s, V3 &grad, float &dist,
                                             V3 &tangent)
    {
        bool inSpine = false;
        switch (gtype)
        {
        case G_BOX:
        {
            const V3 pen = v3(fabsf(lp.x) - p0.x, fabsf(lp.y) - p0.y, fabsf(lp.z) - p0.z);
            const V3 sg = v3(lp.x < 0.f ? -1.f : 1.f, lp.y < 0.f ? -1.f : 1.f, lp.z < 0.f ? -1.f : 1.f);
            const float g = fmaxf(pen.x, fmaxf(pen.y, pen.z));
            const V3 q = v3(fmaxf(pen.x, 0.f), fmaxf(pen.y, 0.f), fmaxf(pen.z, 0.f));
            const float l = sqrtf(sq(q));
            V3 dir;
            if (g > 0.f)
                dir = q / l;
            else if (pen.x > pen.y)
                dir = (pen.x > pen.z) ? v3(1.f, 0.f, 0.f) : v3(0.f, 0.f, 1.f);
            else
                dir = (pen.y > pen.z) ? v3(0.f, 1.f, 0.f) : v3(0.f, 0.f, 1.f);
            grad = mul(sg, dir);
            dist = l + fminf(g, 0.f);
            break;
        }
        case G_SPHERE:
        {
            const float len = sqrtf(sq(lp));
            grad = lp / fmaxf(len, kEps);
            dist = len - p0.x;
            break;
        }
        case G_PLANE:
            grad = v3(0.f, 1.f, 0.f);
            dist = lp.y;
            break;
        case G_CAPSULE:
        {
            const float h2 = p0.y * 2.f;
            V3 pa = lp;
            pa.y -= p0.y;
            const float h = fminf(fmaxf(-pa.y / h2, 0.f), 1.f);
            pa.y += h2 * h;
            const float d = sqrtf(sq(pa));
            grad = pa / fmaxf(d, kEps);
            dist = d - p0.x;
            break;
        }
        case G_ARC:
        {
            const float ang = atan2f(lp.z, lp.x);
            if (ang < p0.x || ang > p0.y)
            {
                grad = v3(0.f, 1.f, 0.f);
                dist = __int_as_float(0x7fc00000);
                break;
            }
            float sn, cs;
            sincosf(ang, &sn, &cs);
            const V3 ptp = lp - v3(cs, 0.f, sn);
            const float d = sqrtf(sq(ptp));
            grad = ptp / fmaxf(d, kEps);
            dist = d;
            tangent = v3(-sn, 0.f, cs);
            break;
        }
        case G_TRIMESH:
        {
            const int off = __float_as_int(p0.x), id = __float_as_int(p0.y);
            const float4 lb = __ldg(&s.lbcs[id]);
            const int4 dim = __ldg(&s.dim[id]);
            const V3 sp = (lp - v3(lb)) / lb.w;
            const int qx = __float2int_rz(sp.x + 0.5f), qy = __float2int_rz(sp.y + 0.5f), qz = __float2int_rz(sp.z + 0.5f);
            if (qx < 0 || qx >= dim.x || qy < 0 || qy >= dim.y || qz < 0 || qz >= dim.z)
            {
                grad = v3(0.f, 1.f, 0.f);
                dist = kMaxF32;
                break;
            }
            const float4 qv = __ldg(&s.data[off + (qz * dim.x * dim.y) + (qy * dim.x) + qx]);
            grad = v3(qv);
            const int bx = __float2int_rz(sp.x), by = __float2int_rz(sp.y), bz = __float2int_rz(sp.z);
            if (bx < 0 || bx >= dim.x - 1 || by < 0 || by >= dim.y - 1 || bz < 0 || bz >= dim.z - 1)
            {
                dist = qv.w;
                break;
            }
            dist = trilinearF(s, dim, off, bx, by, bz, v3(sp.x - (float)bx, sp.y - (float)by, sp.z - (float)bz));
            break;
        }
        case G_QUAD_SLICER:
        {
            if (lp.x < -p0.x || lp.x > p0.x || lp.z < -p0.y || lp.z > p0.y)
            {
                grad = v3(0.f, 0.f, 0.f);
                dist = kMaxF32;
            }
            else
            {
                grad = v3(0.f, copysignf(1.f, lp.y), 0.f);
                dist = fabsf(lp.y);
            }
            break;
        }
        case G_TRIMESH_SLICER:
        {
            grad = v3(0.f, 1.f, 0.f);
            dist = __int_as_float(0x7fc00000);
            const int off = __float_as_int(p0.x) + 1, id = __float_as_int(p0.y);
            const float4 lb = __ldg(&s.lbcs[id]);
            const int4 dim = __ldg(&s.dim[id]);
            const V3 sp = (lp - v3(lb)) / lb.w;
            const int qx = __float2int_rz(sp.x + 0.5f), qy = __float2int_rz(sp.y + 0.5f), qz = __float2int_rz(sp.z + 0.5f);
            if (qx < 1 || qx >= dim.x - 1 || qy < 1 || qy >= dim.y - 1 || qz < 1 || qz >= dim.z - 1)
                break;
            const float4 qv = __ldg(&s.data[off + (qz * dim.x * dim.y) + (qy * dim.x) + qx]);
            if (isnan(qv.w))
                break;
            grad = v3(qv);
            const int bx = __float2int_rz(sp.x), by = __float2int_rz(sp.y), bz = __float2int_rz(sp.z);
            const float iv = trilinearF(s, dim, off, bx, by, bz, v3(sp.x - (float)bx, sp.y - (float)by, sp.z - (float)bz));
            if (isnan(iv))
                break;
            dist = fabsf(iv);
            if (qv.w * iv < 0.f)
                grad = v3(-grad.x, -grad.y, -grad.z);
            const float4 spine = __ldg(&s.data[off - 1]);
            if (isnan(spine.x))
                break;
            const V3 sn = v3(spine);
            const float len = sqrtf(sq(sn));
            if (dot(lp, sn / len) + spine.w > 0.f)
            {
                dist -= len - 1.f;
                inSpine = true;
            }
            break;
        }
        case G_LINES:
        {
            grad = v3(0.f, 1.f, 0.f);
            dist = __int_as_float(0x7fc00000);
            const int off = __float_as_int(p0.x), id = __float_as_int(p0.y), size = __float_as_int(p0.z);
            const float4 bmin = __ldg(&s.lbcs[id]), bmax = __ldg(&s.data[off]);
            if (lp.x < bmin.x || lp.x > bmax.x || lp.y < bmin.y || lp.y > bmax.y || lp.z < bmin.z || lp.z > bmax.z)
                break;
            int closestIdx = 0;
            V3 closest = v3(0.f, 0.f, 0.f), pt1 = v3(0.f, 0.f, 0.f);
            float closestD = kMaxF32;
            for (int p = off + 1; p < off + size - 1; ++p)
            {
                const V3 a = v3(__ldg(&s.data[p]));
                pt1 = v3(__ldg(&s.data[p + 1]));
                const V3 line = pt1 - a;
                float t = dot(lp - a, line) / sq(line);
                t = fmaxf(0.f, fminf(1.f, t));
                const V3 proj = a + line * t;
                const float d = sqrtf(sq(lp - proj));
                if (d < closestD)
                {
                    closestD = d;
                    closest = proj;
                    closestIdx = p;
                }
            }
            const V3 pt0 = v3(__ldg(&s.data[off + 1]));
            if (sq(closest - pt0) < kEps || sq(closest - pt1) < kEps)
                break;
            grad = normalized(lp - closest);
            tangent = normalized(v3(__ldg(&s.data[closestIdx])) - v3(__ldg(&s.data[closestIdx + 1])));
            dist = closestD;
            break;
        }
        default:
            break;
        }
        return inSpine;
    }

    // Conservative lower bound of the local SDF of the analytic geometries (box, sphere, plane,
    // capsule; sdf.h:77-150).  For a unit-gradient SDF the scaled distance is at least
    // bound / max(invScale), so a point whose bound reaches (smooth + fatten) * max(invScale) is
    // outside the contact band and the full evaluation can be skipped.
    __device__ __forceinline__ float sdfLowerBound(V3 lp, int gtype, const float4 &p0)
    {
        switch (gtype)
        {
        case G_BOX:
            return fmaxf(fabsf(lp.x) - p0.x, fmaxf(fabsf(lp.y) - p0.y, fabsf(lp.z) - p0.z));
        case G_SPHERE:
            return sqrtf(sq(lp)) - p0.x;
        case G_PLANE:
            return lp.y;
        case G_CAPSULE:
            return fmaxf(sqrtf(lp.x * lp.x + lp.z * lp.z), fabsf(lp.y) - p0.y) - p0.x;
        default:
            return -kMaxF32;
        }
    }

    // Gathers shape `id` of the bound struct-of-arrays into one record, with the culling
    // thresholds of sdfLowerBound (a small safety margin keeps the test conservative).
    __device__ __forceinline__ ShapeRec makeShapeRec(int id, const CrB200ShapeData &sh, const CrB200GeometryData &ge)
    {
        const int gid = sh.geometryIdx[id];
        ShapeRec r;
        r.pos = reinterpret_cast<const float4 *>(sh.position)[id];
        r.rot = reinterpret_cast<const float4 *>(sh.rotation)[id];
        r.invScale = reinterpret_cast<const float4 *>(sh.invScale)[id];
        r.linVel = reinterpret_cast<const float4 *>(sh.linearVelocity)[id];
        r.angVel = reinterpret_cast<const float4 *>(sh.angularVelocity)[id];
        r.params0 = reinterpret_cast<const float4 *>(sh.params0)[id];
        r.gparams = reinterpret_cast<const float4 *>(ge.params0)[gid];
        r.comInvMass = sh.comInvMass ? reinterpret_cast<const float4 *>(sh.comInvMass)[id] : make_float4(0, 0, 0, 0);
        r.inertia0 = sh.inertiaInv0 ? reinterpret_cast<const float4 *>(sh.inertiaInv0)[id] : make_float4(0, 0, 0, 0);
        r.inertia1 = sh.inertiaInv1 ? reinterpret_cast<const float4 *>(sh.inertiaInv1)[id] : make_float4(0, 0, 0, 0);
        r.kind = sh.type[id];
        r.gtype = ge.type[gid];
        r.id = id;
        r.dynSlot = -1;
        const float maxIsc = fmaxf(fabsf(r.invScale.x), fmaxf(fabsf(r.invScale.y), fabsf(r.invScale.z)));
        const bool analytic = r.gtype == G_BOX || r.gtype == G_SPHERE || r.gtype == G_PLANE || r.gtype == G_CAPSULE;
        const float band = r.params0.x + r.params0.w, pband = r.params0.w;
        r.cull.x = (analytic && band >= 0.f && isfinite(band * maxIsc)) ? band * maxIsc * 1.0001f + 1e-6f : kMaxF32;
        r.cull.y = (analytic && pband >= 0.f && isfinite(pband * maxIsc)) ? pband * maxIsc * 1.0001f + 1e-6f : kMaxF32;
        r.cull.z = 0.f;
        r.cull.w = 0.f;
        return r;
    }

    __device__ __forceinline__ int shapeFlagsOf(const ShapeRec &r)
    {
        int f = 0;
        if (r.gtype == G_QUAD_SLICER || r.gtype == G_TRIMESH_SLICER)
            f |= SF_SLICER;
        if (r.kind == S_DYNAMIC)
            f |= SF_DYNAMIC;
        return f;
    }

    constexpr int kDetSlots = 4; // dynamic shapes whose coupling is reduced deterministically

    // Where the grid contact puts the momentum it exchanges with a dynamic shape.
    // CoupleAtomic: float atomics into the shape's force / torque, in arrival order, as the
    // reference does (mpm_rigid_contact.h:59-82, 380-389).
    struct CoupleAtomic
    {
        float4 *force, *torque;
        __device__ __forceinline__ void add(const ShapeRec &r, V3 mom, V3 tq)
        {
            atomicAdd(&force[r.id].x, mom.x);
            atomicAdd(&force[r.id].y, mom.y);
            atomicAdd(&force[r.id].z, mom.z);
            atomicAdd(&torque[r.id].x, tq.x);
            atomicAdd(&torque[r.id].y, tq.y);
            atomicAdd(&torque[r.id].z, tq.z);
        }
    };

    // CoupleRow: this thread's row of per-slot sums (force xyz, torque xyz for each of the first
    // kDetSlots dynamic shapes) in shared memory, reduced later in a fixed order; further dynamic
    // shapes fall back to atomics.
    struct CoupleRow
    {
        float *row; // kDetSlots * 6 floats
        CoupleAtomic spill;
        bool any; // some momentum went into the row
        __device__ __forceinline__ void add(const ShapeRec &r, V3 mom, V3 tq)
        {
            if (r.dynSlot < 0 || r.dynSlot >= kDetSlots)
            {
                spill.add(r, mom, tq);
                return;
            }
            any = true;
            float *q = row + 6 * r.dynSlot;
            q[0] += mom.x;
            q[1] += mom.y;
            q[2] += mom.z;
            q[3] += tq.x;
            q[4] += tq.y;
            q[5] += tq.z;
        }
    };

    // resolveRigidCollision (mpm_rigid_contact.h:101-399).
    //   isParticle = false: grid node with velocity vel (mass m) evaluated at pos; contact inside
    //       the smooth distance, separating nodes skipped, Coulomb-like friction, drag, rigid
    //       velocity, line/arc tangent restriction, dynamic coupling (kinematic or effective mass).
    //   isParticle = true: positional push-out only (lines and arcs skipped).
    //   mask: shapes to consider (bit s = shape s); shapes outside it are known not to reach pos.
    template <bool IsParticle, class Couple = CoupleAtomic>
    __device__ __forceinline__ void rigidContact(V3 &vel, float m, V3 &pos, const ShapeRec *sh, int num, const SdfPtrs &sdf,
                                                 bool effMass, Couple &couple, unsigned long long mask = ~0ull)
    {
        unsigned long long left = mask & (num >= 64 ? ~0ull : ((1ull << num) - 1ull));
        while (left)
        {
            const int s = __ffsll((long long)left) - 1;
            left &= left - 1ull;
            const ShapeRec &r = sh[s];
            if (IsParticle && (r.gtype == G_LINES || r.gtype == G_ARC))
                continue;
            const V3 isc = v3(r.invScale);
            const V3 wrel = pos - v3(r.pos);
            const V3 lp = mul(qrotInv(r.rot, wrel), isc);
            const float cull = IsParticle ? r.cull.y : r.cull.x;
            if (cull < kMaxF32 && sdfLowerBound(lp, r.gtype, r.gparams) >= cull)
                continue;
            V3 grad, tangent = v3(0.f, 0.f, 0.f);
            float dist;
            const bool onSpine = geometrySdf(lp, r.gtype, r.gparams, sdf, grad, dist, tangent);
            if (isnan(dist))
                continue;
            grad = mul(grad, isc);
            const float is = rsqrtf(sq(grad));
            dist = dist * is - r.params0.w;
            grad = grad * is;
            const float smooth = IsParticle ? 0.f : r.params0.x;
            if (!(dist < smooth))
                continue;
            const V3 normal = qrot(r.rot, grad);
            const V3 rigidVel = r.kind == S_STATIC ? v3(0.f, 0.f, 0.f) : v3(r.linVel) + cross(v3(r.angVel), wrel);
            const V3 relVel = vel - rigidVel;
            const float vn = dot(relVel, normal);
            if (IsParticle)
            {
                pos = pos - normal * fminf(dist, 0.f);
                continue;
            }
            if (vn >= 0.f)
                continue;
            const float friction = onSpine ? 100.f : r.params0.z;
            const float sticky = r.params0.y;
            V3 resp;
            if (effMass && r.kind == S_DYNAMIC)
            {
                resp = v3(0.f, 0.f, 0.f); // zero unless the impulse below is defined (:231)
                const float invMassRigid = r.comInvMass.w;
                if (invMassRigid > 0.f)
                {
                    const V3 rr = wrel - qrot(r.rot, v3(r.comInvMass));
                    const V3 rxnl = qrotInv(r.rot, cross(rr, normal));
                    const V3 wl = v3(r.inertia0.x * rxnl.x + r.inertia1.x * rxnl.y + r.inertia1.y * rxnl.z,
                                     r.inertia1.x * rxnl.x + r.inertia0.y * rxnl.y + r.inertia1.z * rxnl.z,
                                     r.inertia1.y * rxnl.x + r.inertia1.z * rxnl.y + r.inertia0.z * rxnl.z);
                    const V3 tt = cross(qrot(r.rot, wl), rr);
                    const float invMassGrid = 1.f / m;
                    const float invMassComb = invMassGrid + (invMassRigid + dot(normal, tt));
                    if (invMassComb > 0.f)
                    {
                        const float Jn = -1.f * vn / invMassComb;
                        const V3 vt = relVel - normal * vn;
                        const float vtn = sqrtf(sq(vt));
                        V3 impT = v3(0.f, 0.f, 0.f);
                        if (vtn > kEps)
                        {
                            const float fJt = fminf(friction * Jn, vtn / invMassComb);
                            const float fin = (vtn - fJt * invMassComb) * sticky;
                            impT = (vt * -1.f / vtn) * ((vtn - fin) / invMassComb);
                        }
                        const V3 tot = normal * Jn + impT;
                        resp = vel + tot * invMassGrid;
                        const V3 mom = tot * -1.f;
                        couple.add(r, mom, cross(rr, mom));
                    }
                }
            }
            else
            {
                V3 tang = relVel - normal * vn;
                if (r.gtype == G_LINES || r.gtype == G_ARC)
                {
                    const V3 td = qrot(r.rot, normalized(mul(tangent, isc)));
                    tang = td * dot(tang, td);
                }
                const float tn = sqrtf(sq(tang));
                const float fc = fmaxf(friction * vn / (tn + kEps), -1.f);
                resp = (tang + tang * fc) * sticky + rigidVel;
                if (!effMass && r.kind == S_DYNAMIC)
                {
                    const V3 mom = (vel - resp) * m;
                    couple.add(r, mom, cross(pos - v3(r.pos), mom));
                }
            }
            vel = resp;
        }
    }

    // Shapes that may reach some point within R of c, decided by the calling warp (lane s tests
    // shape s, 32 at a time).  The local SDF is 1-Lipschitz in local coordinates, which stretch by
    // at most max(invScale): a lower bound at c minus max(invScale) R at or above the culling
    // threshold (cull.x for grid nodes, cull.y for particles) rules the shape out for the whole
    // ball.  Every lane of the warp must call it.
    __device__ __forceinline__ void regionShapeMasks(const ShapeRec *sh, int num, V3 c, float R,
                                                     unsigned long long &nodeMask, unsigned long long &partMask)
    {
        nodeMask = 0ull;
        partMask = 0ull;
        const int lane = (int)(threadIdx.x & 31);
        for (int base = 0; base < num; base += 32)
        {
            const int s = base + lane;
            bool keepNode = false, keepPart = false;
            if (s < num)
            {
                const ShapeRec &r = sh[s];
                keepNode = keepPart = true;
                if (r.cull.x < kMaxF32 || r.cull.y < kMaxF32)
                {
                    const V3 isc = v3(r.invScale);
                    const V3 lp = mul(qrotInv(r.rot, c - v3(r.pos)), isc);
                    const float mx = fmaxf(isc.x, fmaxf(isc.y, isc.z));
                    const float lb = sdfLowerBound(lp, r.gtype, r.gparams) - mx * R;
                    keepNode = !(r.cull.x < kMaxF32 && lb >= r.cull.x);
                    keepPart = !(r.cull.y < kMaxF32 && lb >= r.cull.y);
                }
            }
            nodeMask |= (unsigned long long)__ballot_sync(0xffffffffu, keepNode) << base;
            partMask |= (unsigned long long)__ballot_sync(0xffffffffu, keepPart) << base;
        }
    }

    // ---------------------------------------------------------------------------------------
    // 3x3 matrices, column-major in registers: m[c*3 + r].
    struct M3
    {
        float m[9];
    };
    __device__ __forceinline__ float det3(const M3 &a)
    {
        const float A = a.m[0], B = a.m[3], Cc = a.m[6], D = a.m[1], E = a.m[4], F = a.m[7], G = a.m[2], H = a.m[5],
                    I = a.m[8];
        return A * (E * I - F * H) - B * (D * I - F * G) + Cc * (D * H - E * G);
    }
    __device__ __forceinline__ M3 matmul(const M3 &a, const M3 &b)
    {
        M3 r;
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int rr = 0; rr < 3; ++rr)
                r.m[c * 3 + rr] = a.m[rr] * b.m[c * 3] + a.m[3 + rr] * b.m[c * 3 + 1] + a.m[6 + rr] * b.m[c * 3 + 2];
        return r;
    }
    __device__ __forceinline__ M3 transpose(const M3 &a)
    {
        M3 r;
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int rr = 0; rr < 3; ++rr)
                r.m[c * 3 + rr] = a.m[rr * 3 + c];
        return r;
    }
    // inverse with the reference's singular cutoff (mat33.h:256-283)
    __device__ __forceinline__ M3 inverse3(const M3 &a)
    {
        const float A = a.m[0], B = a.m[3], Cc = a.m[6], D = a.m[1], E = a.m[4], F = a.m[7], G = a.m[2], H = a.m[5],
                    I = a.m[8];
        const float dt = A * (E * I - F * H) - B * (D * I - F * G) + Cc * (D * H - E * G);
        M3 r;
        if (fabsf(dt) < 1e-6f)
        {
#pragma unroll
            for (int i = 0; i < 9; ++i)
                r.m[i] = 0.f;
            return r;
        }
        const float inv = 1.f / dt;
        r.m[0] = (E * I - F * H) * inv;
        r.m[1] = -(B * I - Cc * H) * inv;
        r.m[2] = (B * F - Cc * E) * inv;
        r.m[3] = -(D * I - F * G) * inv;
        r.m[4] = (A * I - Cc * G) * inv;
        r.m[5] = -(A * F - Cc * D) * inv;
        r.m[6] = (D * H - E * G) * inv;
        r.m[7] = -(A * H - B * G) * inv;
        r.m[8] = (A * E - B * D) * inv;
        return r;
    }

    // Kirchhoff stress (constitutive_models.h:49-118).  eCoRotational falls through to the
    // linear (St. Venant-Kirchhoff) model in the reference, so it is computed as such here.
    __device__ __forceinline__ M3 kirchhoffStress(const M3 &F, float lambda, float mu, int type)
    {
        M3 s;
        if (type == 1) // Neo-Hookean
        {
            float J = det3(F);
            J = J < 1e-6f ? 1e-6f : J;
            const float l = lambda * logf(J);
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int r = 0; r < 3; ++r)
                {
                    const float b = F.m[r] * F.m[c] + F.m[3 + r] * F.m[3 + c] + F.m[6 + r] * F.m[6 + c];
                    s.m[c * 3 + r] = mu * (b - (r == c ? 1.f : 0.f)) + (r == c ? l : 0.f);
                }
        }
        else if (type == 0 || type == 2) // co-rotational (falls through) and linear
        {
            M3 E;
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int r = 0; r < 3; ++r)
                {
                    const float ftf = F.m[r * 3] * F.m[c * 3] + F.m[r * 3 + 1] * F.m[c * 3 + 1] + F.m[r * 3 + 2] * F.m[c * 3 + 2];
                    E.m[c * 3 + r] = 0.5f * (ftf - (r == c ? 1.f : 0.f));
                }
            const float tr = E.m[0] + E.m[4] + E.m[8];
            M3 S;
#pragma unroll
            for (int i = 0; i < 9; ++i)
                S.m[i] = 2.f * mu * E.m[i];
            S.m[0] += tr * lambda;
            S.m[4] += tr * lambda;
            S.m[8] += tr * lambda;
            s = matmul(matmul(F, S), transpose(F));
        }
        else
        {
#pragma unroll
            for (int i = 0; i < 9; ++i)
                s.m[i] = 0.f;
        }
        return s;
    }

    // ---------------------------------------------------------------------------------------
    // Polar rotation via SVD: A = U diag(s) V^T with U, V proper rotations and sign(det A) on s[2]
    // (the convention of the reference's svd3: McAdams et al., UW-Madison TR1690, 2011).
    // Jacobi eigen-analysis of A^T A with exact rotations, column sort of B = A V, Givens QR of B.
    template <typename T>
    __device__ __forceinline__ void svdRotations(const T A[9], T U[9], T V[9], T s[3], int sweeps)
    {
        T S[6]; // symmetric A^T A: s00 s11 s22 s01 s02 s12
        auto a = [&](int r, int c) { return A[c * 3 + r]; };
        S[0] = a(0, 0) * a(0, 0) + a(1, 0) * a(1, 0) + a(2, 0) * a(2, 0);
        S[1] = a(0, 1) * a(0, 1) + a(1, 1) * a(1, 1) + a(2, 1) * a(2, 1);
        S[2] = a(0, 2) * a(0, 2) + a(1, 2) * a(1, 2) + a(2, 2) * a(2, 2);
        S[3] = a(0, 0) * a(0, 1) + a(1, 0) * a(1, 1) + a(2, 0) * a(2, 1);
        S[4] = a(0, 0) * a(0, 2) + a(1, 0) * a(1, 2) + a(2, 0) * a(2, 2);
        S[5] = a(0, 1) * a(0, 2) + a(1, 1) * a(1, 2) + a(2, 1) * a(2, 2);
        T Vm[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        for (int sw = 0; sw < sweeps; ++sw)
        {
#pragma unroll
            for (int pq = 0; pq < 3; ++pq)
            {
                const int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
                const int ipq = pq == 0 ? 3 : (pq == 1 ? 4 : 5);
                const T apq = S[ipq];
                if (apq == T(0))
                    continue;
                const T app = S[p], aqq = S[q];
                T theta, t, c;
                if constexpr (sizeof(T) == 4)
                {
                    // single precision: hardware reciprocal, reciprocal square root and approximate
                    // division; the sweeps converge all the same and the ill-conditioned cases are
                    // redone in double precision
                    theta = __fdividef(aqq - app, 2.f * apq);
                    const float h = theta * theta + 1.f;
                    // |theta| beyond 1e18: theta^2 overflows; t -> 1 / (2 theta)
                    t = fabsf(theta) > 1e18f ? 0.5f / theta
                                             : __fdividef(theta >= 0.f ? 1.f : -1.f, fabsf(theta) + h * rsqrtf(h));
                    c = rsqrtf(t * t + 1.f);
                }
                else
                {
                    theta = (aqq - app) / (T(2) * apq);
                    t = (theta >= T(0) ? T(1) : T(-1)) / (fabs(theta) + sqrt(theta * theta + T(1)));
                    c = T(1) / sqrt(t * t + T(1));
                }
                const T sn = t * c;
                // rotate S in the (p, q) plane: new diagonal and the off-diagonals with the third index
                const int o = 3 - p - q;
                const int ipo = (p == 0 && o == 1) || (p == 1 && o == 0) ? 3 : ((p == 0 && o == 2) || (p == 2 && o == 0) ? 4 : 5);
                const int iqo = (q == 0 && o == 1) || (q == 1 && o == 0) ? 3 : ((q == 0 && o == 2) || (q == 2 && o == 0) ? 4 : 5);
                const T spo = S[ipo], sqo = S[iqo];
                S[p] = app - t * apq;
                S[q] = aqq + t * apq;
                S[ipq] = T(0);
                S[ipo] = c * spo - sn * sqo;
                S[iqo] = sn * spo + c * sqo;
#pragma unroll
                for (int k = 0; k < 3; ++k)
                {
                    const T vkp = Vm[k][p], vkq = Vm[k][q];
                    Vm[k][p] = c * vkp - sn * vkq;
                    Vm[k][q] = sn * vkp + c * vkq;
                }
            }
        }
        T B[3][3];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                B[r][c] = a(r, 0) * Vm[0][c] + a(r, 1) * Vm[1][c] + a(r, 2) * Vm[2][c];
        auto n2 = [&](int c) { return B[0][c] * B[0][c] + B[1][c] * B[1][c] + B[2][c] * B[2][c]; };
        auto swapc = [&](int x, int y) {
#pragma unroll
            for (int r = 0; r < 3; ++r)
            {
                T tb = B[r][x];
                B[r][x] = B[r][y];
                B[r][y] = -tb;
                T tv = Vm[r][x];
                Vm[r][x] = Vm[r][y];
                Vm[r][y] = -tv;
            }
        };
        T c0 = n2(0), c1 = n2(1), c2 = n2(2);
        if (c0 < c1) { swapc(0, 1); T t = c0; c0 = c1; c1 = t; }
        if (c0 < c2) { swapc(0, 2); T t = c0; c0 = c2; c2 = t; }
        if (c1 < c2) { swapc(1, 2); }
        T Um[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
#pragma unroll
        for (int gi = 0; gi < 3; ++gi)
        {
            const int p = gi == 2 ? 1 : 0, q = gi == 0 ? 1 : 2, col = gi == 2 ? 1 : 0;
            const T x = B[p][col], y = B[q][col];
            const T r2 = x * x + y * y;
            T c = T(1), sn = T(0);
            if (r2 > T(0))
            {
                if constexpr (sizeof(T) == 4)
                {
                    const float inv = rsqrtf(r2); // r2 is a normal float here or the matrix is degenerate
                    c = x * inv;
                    sn = y * inv;
                }
                else
                {
                    const T rr = sqrt(r2);
                    c = x / rr;
                    sn = y / rr;
                }
            }
#pragma unroll
            for (int k = 0; k < 3; ++k)
            {
                const T bp = B[p][k], bq = B[q][k];
                B[p][k] = c * bp + sn * bq;
                B[q][k] = -sn * bp + c * bq;
                const T up = Um[k][p], uq = Um[k][q];
                Um[k][p] = c * up + sn * uq;
                Um[k][q] = -sn * up + c * uq;
            }
        }
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c)
            {
                U[c * 3 + r] = Um[r][c];
                V[c * 3 + r] = Vm[r][c];
            }
        s[0] = B[0][0];
        s[1] = B[1][1];
        s[2] = B[2][2];
    }

    // Rotation the reference's PB-MPM constraint blends toward: `u * vt` of svd3(targetF), which
    // factors targetF^T (svd3.h:1271-1274) and therefore equals R^T = V U^T for targetF = U S V^T.
    // V U^T is the polar factor (A (A^T A)^(-1/2))^T: it does not depend on how U and V are chosen
    // inside a near-degenerate singular subspace, so nearly equal positive singular values need no
    // care.  Float first; the ill-conditioned cases are redone in double precision: a tiny smallest
    // singular value, or an inverted matrix (negative smallest singular value) whose two smallest
    // magnitudes nearly tie (the closest rotation is then ambiguous).
    // The cases the single-precision SVD leaves to double precision (see pbRotationTarget).
    __device__ __forceinline__ bool pbNeedsFp64(const float s[3])
    {
        const float smax = fabsf(s[0]);
        return !(fabsf(s[2]) > 1e-3f * smax) || (s[2] < 0.f && s[1] - fabsf(s[2]) < 1e-4f * smax);
    }

    __device__ __forceinline__ M3 pbRotationTarget(const M3 &A, unsigned *fp64Count)
    {
        float U[9], V[9], s[3];
        svdRotations<float>(A.m, U, V, s, 5);
        const bool degenerate = pbNeedsFp64(s);
        M3 R;
        if (degenerate)
        {
            double Ad[9], Ud[9], Vd[9], sd[3];
#pragma unroll
            for (int i = 0; i < 9; ++i)
                Ad[i] = (double)A.m[i];
            svdRotations<double>(Ad, Ud, Vd, sd, 12);
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int r = 0; r < 3; ++r)
                    R.m[c * 3 + r] = (float)(Vd[r] * Ud[c] + Vd[3 + r] * Ud[3 + c] + Vd[6 + r] * Ud[6 + c]);
            if (fp64Count)
            {
                // one atomic per warp: the lanes taking this branch
                const unsigned am = __activemask();
                if ((threadIdx.x & 31) == (unsigned)(__ffs(am) - 1))
                    atomicAdd(fp64Count, (unsigned)__popc(am));
            }
        }
        else
        {
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int r = 0; r < 3; ++r)
                    R.m[c * 3 + r] = V[r] * U[c] + V[3 + r] * U[3 + c] + V[6 + r] * U[6 + c];
        }
        return R;
    }
} // namespace crb200

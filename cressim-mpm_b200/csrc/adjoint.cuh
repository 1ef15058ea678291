// Adjoint of the MLS-MPM substep (no counterpart in the reference, which has no gradient path).
//
// Forward map of one substep, state (x, v, F, C) per particle, parameters (lambda, mu) per particle:
//   P2G          P_n += w_n (m (v + g dt) + A d_n),  M_n += w_n m,  A = -dt 4/dx^2 V0 tau(F) + m C
//                (mls_mpm_algorithm.h:147-241; tau Neo-Hookean, constitutive_models.h:62-75)
//   grid update  V_n = P_n / M_n, rigid contact at x_n + V_n dt, two-node boundary band; nodes below
//                the 1e-4 mass cutoff keep their momentum (mls_mpm_algorithm.h:243-294)
//   G2P          v' = sum w_n V_n, C' = 4/dx sum w_n d_n V_n^T, x' = clamp(x + v' dt) then the
//                particle push-out, F' = (I + dt C') F (mls_mpm_algorithm.h:296-390)
// The reverse substep runs three kernels in the opposite order, after replaying the forward P2G and
// grid update of that substep from its recomputed input state:
//   k_adjG2P         per particle: adjoint of G2P; scatters dL/dV_n to the adjoint grid
//   k_adjGridUpdate  per touched node: adjoint of the division and of the contact chain -> dL/dP_n, dL/dM_n
//   k_adjP2G         per particle: gathers dL/dP_n, dL/dM_n; adjoint of P2G and of the stress
// Branch decisions (contact on/off, friction clamp, position clamp, mass cutoff) are those of the
// replayed forward and are held fixed.  Scope: MLS-MPM, Neo-Hookean particles, the kinematic contact
// model, analytic shapes (box, sphere, plane, capsule) of uniform scale, no slicers.
#pragma once

namespace crb200
{
    constexpr int kAdjMaxHits = 8; // contacts per particle / node that one reverse step can undo
    constexpr int kAdjThreads = 128; // threads per CTA of the per-particle reverse kernels

    // Signed distance, unit normal and the local frame quantities of shape r at world point pos,
    // exactly as rigidContact evaluates them (mpm_rigid_contact.h:129-148).
    __device__ __forceinline__ bool adjShapeEval(const ShapeRec &r, V3 pos, const SdfPtrs &sdf, float &dist, V3 &n,
                                                 V3 &lp, V3 &gl)
    {
        const V3 isc = v3(r.invScale);
        const V3 wrel = pos - v3(r.pos);
        lp = mul(qrotInv(r.rot, wrel), isc);
        V3 grad, tangent = v3(0.f, 0.f, 0.f);
        float d;
        geometrySdf(lp, r.gtype, r.gparams, sdf, grad, d, tangent);
        if (isnan(d))
            return false;
        gl = grad;
        grad = mul(grad, isc);
        const float is = rsqrtf(sq(grad));
        dist = d * is - r.params0.w;
        n = qrot(r.rot, grad * is);
        return true;
    }

    // d(normal)/d(pos) in world space, row-major J[3 i + j] = dn_i / dpos_j, for the analytic
    // geometries of uniform scale s: J = s R J_local R^T.
    __device__ __forceinline__ void adjNormalJacobian(const ShapeRec &r, V3 lp, V3 gl, float J[9])
    {
        float L[9];
#pragma unroll
        for (int e = 0; e < 9; ++e)
            L[e] = 0.f;
        const float4 p0 = r.gparams;
        if (r.gtype == G_SPHERE || r.gtype == G_CAPSULE)
        {
            V3 pa = lp;
            bool slide = false;
            if (r.gtype == G_CAPSULE)
            {
                const float h2 = p0.y * 2.f;
                pa.y -= p0.y;
                const float h = fminf(fmaxf(-pa.y / h2, 0.f), 1.f);
                slide = h > 0.f && h < 1.f;
                pa.y += h2 * h;
            }
            const float ln = fmaxf(sqrtf(sq(pa)), kEps);
            const float g[3] = {gl.x, gl.y, gl.z};
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j)
                    L[3 * i + j] = (slide && j == 1) ? 0.f : ((i == j ? 1.f : 0.f) - g[i] * g[j]) / ln;
        }
        else if (r.gtype == G_BOX)
        {
            const float pen[3] = {fabsf(lp.x) - p0.x, fabsf(lp.y) - p0.y, fabsf(lp.z) - p0.z};
            const float sg[3] = {lp.x < 0.f ? -1.f : 1.f, lp.y < 0.f ? -1.f : 1.f, lp.z < 0.f ? -1.f : 1.f};
            const float gm = fmaxf(pen[0], fmaxf(pen[1], pen[2]));
            if (gm > 0.f)
            {
                const float q[3] = {fmaxf(pen[0], 0.f), fmaxf(pen[1], 0.f), fmaxf(pen[2], 0.f)};
                const float l = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
                const float dir[3] = {q[0] / l, q[1] / l, q[2] / l};
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j)
                        L[3 * i + j] = sg[i] * (((i == j ? 1.f : 0.f) - dir[i] * dir[j]) / l) * (pen[j] > 0.f ? sg[j] : 0.f);
            }
        }
        // R columns
        const V3 c0 = qrot(r.rot, v3(1.f, 0.f, 0.f)), c1 = qrot(r.rot, v3(0.f, 1.f, 0.f)), c2 = qrot(r.rot, v3(0.f, 0.f, 1.f));
        const float R[9] = {c0.x, c1.x, c2.x, c0.y, c1.y, c2.y, c0.z, c1.z, c2.z}; // row-major
        float T[9];                                                              // L R^T
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                T[3 * i + j] = L[3 * i] * R[3 * j] + L[3 * i + 1] * R[3 * j + 1] + L[3 * i + 2] * R[3 * j + 2];
        const float s = r.invScale.x;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                J[3 * i + j] = s * (R[3 * i] * T[j] + R[3 * i + 1] * T[3 + j] + R[3 * i + 2] * T[6 + j]);
    }

    // J^T g for a row-major 3x3 J
    __device__ __forceinline__ V3 adjJtG(const float J[9], V3 g)
    {
        return v3(J[0] * g.x + J[3] * g.y + J[6] * g.z, J[1] * g.x + J[4] * g.y + J[7] * g.z,
                  J[2] * g.x + J[5] * g.y + J[8] * g.z);
    }

    // Separable node addresses of a stencil (addr = AX[a] + AY[b] + AZ[c]) and the in-grid bits of
    // each axis offset (x: bits 0-2, y: 3-5, z: 6-8).
    struct StencilAddrs
    {
        unsigned AX[3], AY[3], AZ[3];
        unsigned valid;
        __device__ __forceinline__ bool ok(int a, int b, int c) const
        {
            return ((valid >> a) & (valid >> (3 + b)) & (valid >> (6 + c)) & 1u) != 0u;
        }
        __device__ __forceinline__ unsigned addr(int a, int b, int c) const { return AX[a] + AY[b] + AZ[c]; }
    };
    __device__ __forceinline__ StencilAddrs stencilAddrs(const GridGeom &g, const Stencil &st)
    {
        StencilAddrs s;
        s.valid = 0u;
#pragma unroll
        for (int e = 0; e < 3; ++e)
        {
            const int xi = st.b[0] + e, yi = st.b[1] + e, zi = st.b[2] + e;
            s.AX[e] = g.blockBase * 64u + (unsigned)(((xi >> 2) << 6) + (xi & 3));
            s.AY[e] = (unsigned)(((g.nb.x * (yi >> 2)) << 6) + 4 * (yi & 3));
            s.AZ[e] = (unsigned)(((g.nb.x * g.nb.y * (zi >> 2)) << 6) + 16 * (zi & 3));
            s.valid |= ((xi >= 0 && xi < g.n.x) ? 1u : 0u) << e;
            s.valid |= ((yi >= 0 && yi < g.n.y) ? 1u : 0u) << (3 + e);
            s.valid |= ((zi >= 0 && zi < g.n.z) ? 1u : 0u) << (6 + e);
        }
        return s;
    }

    // ---------------------------------------------------------------------------------------
    // Reverse of G2P (per particle).  In: adjoint of the substep's output state in aX, aV, aF, aC.
    // Out: aX, aF hold the G2P part of the adjoint of the input x and F.  dL/dV_n =
    // w_n (g_v + 4/dx g_C^T d_n) is affine in the node offset like a P2G contribution, so it is
    // written as a P2G record (base g_v, matrix 4/dx g_C^T, no mass) that k_accumulate sums into
    // gridG in cell order; stencils outside the grid are added here with atomics.
    template <bool Multi>
    __global__ void __launch_bounds__(kAdjThreads, 4) k_adjG2P(const __grid_constant__ StepParams p0, SceneTable sc,
                                                   const float4 *__restrict__ xm, const unsigned char *__restrict__ mask,
                                                   const float *__restrict__ F, unsigned stride,
                                                   const ShapeRec *__restrict__ shapeTable, SdfPtrs sdf,
                                                   const float4 *__restrict__ gridV, float4 *__restrict__ aX,
                                                   const float4 *__restrict__ aV, float *__restrict__ aF,
                                                   const float *__restrict__ aC, float4 *__restrict__ gridG,
                                                   float4 *__restrict__ records)
    {
        __shared__ ShapeRec sh[Multi ? 1 : kMaxShapes];
        // the particle's streams, staged at entry (launched with kAdjThreads threads)
        __shared__ float4 sX[kAdjThreads], sAx[kAdjThreads], sAv[kAdjThreads];
        __shared__ float sF[9][kAdjThreads], sAF[9][kAdjThreads], sAC[9][kAdjThreads];
        const unsigned t = threadIdx.x;
        const unsigned i = blockIdx.x * blockDim.x + t;
        const bool inRange = i < (Multi ? sc.numParticles : p0.numActive);
        if (inRange)
        {
            stage16(&sX[t], &xm[i]);
            stage16(&sAx[t], &aX[i]);
            stage16(&sAv[t], &aV[i]);
#pragma unroll
            for (int k = 0; k < 9; ++k)
            {
                stage4(&sF[k][t], &F[k * stride + i]);
                stage4(&sAF[k][t], &aF[k * stride + i]);
                stage4(&sAC[k][t], &aC[k * stride + i]);
            }
        }
        if (!Multi && p0.numShapes > 0)
            loadShapes(sh, shapeTable, p0.numShapes);
        const bool active = inRange && mask[i] != 0;
        const unsigned si = (Multi && inRange) ? sc.particleScene[i] : 0u;
        stageWait();
        __syncthreads();
        if (!active || (Multi && si == 0xFFFFu))
            return;
        const StepParams &p = Multi ? sc.params[si] : p0;
        const GridGeom &g = p.g;
        const ShapeRec *shp = Multi ? shapeTable + p.shapeBegin : sh;
        const V3 x = v3(sX[t]);
        const Stencil st = stencilOf(g, x);
        if (!st.finite)
            return;
        float w[3][3], dw[3][3];
        weights(st.fx, w);
        weightGrads(st.fx, dw);
        // adjoint inputs; g_C' + dt g_F' F^T depends on them only, so the x-gradient moments can be
        // gathered in the same pass as the forward replay of v' and C'
        const float4 gx4 = sAx[t], gv4 = sAv[t];
        float gFo[9], gCt[9], Fp[9];
#pragma unroll
        for (int k = 0; k < 9; ++k)
        {
            gFo[k] = sAF[k][t];
            gCt[k] = sAC[k][t];
            Fp[k] = sF[k][t];
        }
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c)
            {
                float acc = 0.f;
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    acc += gFo[3 * k + r] * Fp[3 * k + c]; // (gF' F^T)(r,c)
                gCt[3 * c + r] += p.dt * acc;
            }
        // one pass over the stencil:
        //   S = sum w V, T[3r + c] = sum o_r w V_c                  (forward v', C')
        //   G[3k + c] = sum dw/dfx_k V_c, A2_k = sum dw/dfx_k d.(g_C V)  (x-gradient moments)
        V3 S = v3(0.f, 0.f, 0.f), A2 = v3(0.f, 0.f, 0.f);
        float T[9], G[9];
#pragma unroll
        for (int e = 0; e < 9; ++e)
        {
            T[e] = 0.f;
            G[e] = 0.f;
        }
        const StencilAddrs sa = stencilAddrs(g, st);
        const float dfx[3] = {-st.fx.x * g.dx, -st.fx.y * g.dx, -st.fx.z * g.dx};
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b)
#pragma unroll
                for (int c = 0; c < 3; ++c)
                {
                    if (!sa.ok(a, b, c))
                        continue;
                    const V3 Vn = v3(__ldg(&gridV[sa.addr(a, b, c)]));
                    const float wab = w[a][0] * w[b][1];
                    const float W = wab * w[c][2];
                    const V3 gWd = v3(dw[a][0] * w[b][1] * w[c][2], w[a][0] * dw[b][1] * w[c][2], wab * dw[c][2]);
                    const V3 wv = Vn * W;
                    S = S + wv;
                    const float o[3] = {(float)a, (float)b, (float)c};
#pragma unroll
                    for (int r = 0; r < 3; ++r)
                    {
                        T[3 * r + 0] += o[r] * wv.x;
                        T[3 * r + 1] += o[r] * wv.y;
                        T[3 * r + 2] += o[r] * wv.z;
                    }
                    G[0] += gWd.x * Vn.x; G[1] += gWd.x * Vn.y; G[2] += gWd.x * Vn.z;
                    G[3] += gWd.y * Vn.x; G[4] += gWd.y * Vn.y; G[5] += gWd.y * Vn.z;
                    G[6] += gWd.z * Vn.x; G[7] += gWd.z * Vn.y; G[8] += gWd.z * Vn.z;
                    const V3 q = v3(gCt[0] * Vn.x + gCt[3] * Vn.y + gCt[6] * Vn.z, gCt[1] * Vn.x + gCt[4] * Vn.y + gCt[7] * Vn.z,
                                    gCt[2] * Vn.x + gCt[5] * Vn.y + gCt[8] * Vn.z);
                    const float e = (o[0] * g.dx + dfx[0]) * q.x + (o[1] * g.dx + dfx[1]) * q.y + (o[2] * g.dx + dfx[2]) * q.z;
                    A2 = A2 + gWd * e;
                }
        const float s4 = 4.f * g.invDx * g.dx;
        const float fxa[3] = {st.fx.x, st.fx.y, st.fx.z};
        const float Sv[3] = {S.x, S.y, S.z};
        M3 Cn;
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                Cn.m[3 * c + r] = s4 * (T[3 * r + c] - fxa[r] * Sv[c]);
        const V3 xpre = x + S * p.dt;
        V3 xc = v3(fminf(fmaxf(xpre.x, g.gmin.x), g.gmax.x), fminf(fmaxf(xpre.y, g.gmin.y), g.gmax.y),
                   fminf(fmaxf(xpre.z, g.gmin.z), g.gmax.z));
        // particle push-out, positions before each contact kept for the reverse
        V3 hitPos[kAdjMaxHits];
        int hitShape[kAdjMaxHits];
        int nh = 0;
        for (int s = 0; s < p.numShapes; ++s)
        {
            const ShapeRec &r = shp[s];
            if (r.gtype == G_LINES || r.gtype == G_ARC)
                continue;
            float dist;
            V3 nrm, lp, gl;
            if (!adjShapeEval(r, xc, sdf, dist, nrm, lp, gl))
                continue;
            if (!(dist < 0.f))
                continue;
            if (nh < kAdjMaxHits)
            {
                hitPos[nh] = xc;
                hitShape[nh] = s;
                ++nh;
            }
            xc = xc - nrm * fminf(dist, 0.f);
        }
        // ---- reverse
        // F' = (I + dt C') F: dL/dF = (I + dt C')^T gF'   (column-major m[3c + r])
        float gFn[9];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c)
            {
                float acf = 0.f;
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    acf += (((k == r) ? 1.f : 0.f) + p.dt * Cn.m[3 * r + k]) * gFo[3 * c + k];
                gFn[3 * c + r] = acf;
            }
        V3 gxp = v3(gx4.x, gx4.y, gx4.z);
        for (int h = nh - 1; h >= 0; --h)
        {
            const ShapeRec &r = shp[hitShape[h]];
            float dist, J[9];
            V3 nrm, lp, gl;
            adjShapeEval(r, hitPos[h], sdf, dist, nrm, lp, gl);
            adjNormalJacobian(r, lp, gl, J);
            gxp = gxp - nrm * dot(nrm, gxp) - adjJtG(J, gxp) * dist;
        }
        if (xpre.x < g.gmin.x || xpre.x > g.gmax.x)
            gxp.x = 0.f;
        if (xpre.y < g.gmin.y || xpre.y > g.gmax.y)
            gxp.y = 0.f;
        if (xpre.z < g.gmin.z || xpre.z > g.gmax.z)
            gxp.z = 0.f;
        const V3 gvt = v3(gv4.x, gv4.y, gv4.z) + gxp * p.dt;
        const float k4 = 4.f * g.invDx;
        const float ddx = g.invDx * g.dx;
        // dL/dx = gxp + 1/dx sum_n dw_n (V_n.g_v + 4/dx d_n.(g_C V_n)) - 4/dx (dx/dx) g_C S
        const V3 Gg = v3(G[0] * gvt.x + G[1] * gvt.y + G[2] * gvt.z, G[3] * gvt.x + G[4] * gvt.y + G[5] * gvt.z,
                         G[6] * gvt.x + G[7] * gvt.y + G[8] * gvt.z);
        const V3 gCS = v3(gCt[0] * S.x + gCt[3] * S.y + gCt[6] * S.z, gCt[1] * S.x + gCt[4] * S.y + gCt[7] * S.z,
                          gCt[2] * S.x + gCt[5] * S.y + gCt[8] * S.z);
        const V3 gx = gxp + (Gg + A2 * k4) * g.invDx - gCS * (k4 * ddx);
        const bool inside = st.b[0] >= 0 && st.b[0] <= g.n.x - 2 && st.b[1] >= 0 && st.b[1] <= g.n.y - 2 &&
                            st.b[2] >= 0 && st.b[2] <= g.n.z - 2;
        {
            // record: u = g_v - A' (fx dx), a_c = dx A'(:, c), A'(r, c) = 4/dx g_C(c, r)
            float rec[kRec];
            if (inside)
            {
                const float fd[3] = {st.fx.x * g.dx, st.fx.y * g.dx, st.fx.z * g.dx};
                const float gvv[3] = {gvt.x, gvt.y, gvt.z};
#pragma unroll
                for (int r = 0; r < 3; ++r)
                {
                    float sacc = 0.f;
#pragma unroll
                    for (int c = 0; c < 3; ++c)
                    {
                        const float Ap = k4 * gCt[3 * r + c];
                        sacc += Ap * fd[c];
                        rec[4 + 3 * c + r] = Ap * g.dx;
                    }
                    rec[r] = gvv[r] - sacc;
                }
                rec[3] = 0.f;
                rec[13] = st.fx.x;
                rec[14] = st.fx.y;
                rec[15] = st.fx.z;
            }
            else
            {
#pragma unroll
                for (int e = 0; e < kRec; ++e)
                    rec[e] = 0.f;
                // stencil crossing the grid edge: its dL/dV_n goes to the grid directly
#pragma unroll 1
                for (int n = 0; n < 27; ++n)
                {
                    const int a = n / 9, b = (n / 3) % 3, c = n % 3;
                    if (!sa.ok(a, b, c))
                        continue;
                    const float W = w[a][0] * w[b][1] * w[c][2];
                    const float d[3] = {((float)a - st.fx.x) * g.dx, ((float)b - st.fx.y) * g.dx, ((float)c - st.fx.z) * g.dx};
                    const V3 gCd = v3(gCt[0] * d[0] + gCt[1] * d[1] + gCt[2] * d[2], gCt[3] * d[0] + gCt[4] * d[1] + gCt[5] * d[2],
                                      gCt[6] * d[0] + gCt[7] * d[1] + gCt[8] * d[2]);
                    const V3 gVn = (gvt + gCd * k4) * W;
                    atomicAdd(&gridG[sa.addr(a, b, c)], make_float4(gVn.x, gVn.y, gVn.z, 0.f));
                }
            }
            float4 *out = records + 4ull * i;
            out[0] = make_float4(rec[0], rec[1], rec[2], rec[3]);
            out[1] = make_float4(rec[4], rec[5], rec[6], rec[7]);
            out[2] = make_float4(rec[8], rec[9], rec[10], rec[11]);
            out[3] = make_float4(rec[12], rec[13], rec[14], rec[15]);
        }
        aX[i] = make_float4(gx.x, gx.y, gx.z, 0.f);
#pragma unroll
        for (int k = 0; k < 9; ++k)
            aF[k * stride + i] = gFn[k];
    }

    // ---------------------------------------------------------------------------------------
    // The effective-mass response of a dynamic shape to one grid node (mpm_rigid_contact.h:219-320,
    // as rigidContact computes it) and what its reverse needs.  ok = false: the impulse is
    // undefined (non-positive inverse masses) and the node velocity becomes zero (:231).
    struct EffMassHit
    {
        bool ok, hasT, caseA;
        V3 rr, w, vt, e, tot;
        float imc, Jn, vtn, fJt, fin, totJt;
    };
    __device__ __forceinline__ V3 effMassResponse(const ShapeRec &r, V3 v, float m, V3 wrel, V3 nrm, V3 rel, float vn,
                                                  EffMassHit &h)
    {
        h.ok = false;
        const float imR = r.comInvMass.w;
        if (!(imR > 0.f))
            return v3(0.f, 0.f, 0.f);
        h.rr = wrel - qrot(r.rot, v3(r.comInvMass));
        const V3 rxnl = qrotInv(r.rot, cross(h.rr, nrm));
        const V3 wl = v3(r.inertia0.x * rxnl.x + r.inertia1.x * rxnl.y + r.inertia1.y * rxnl.z,
                         r.inertia1.x * rxnl.x + r.inertia0.y * rxnl.y + r.inertia1.z * rxnl.z,
                         r.inertia1.y * rxnl.x + r.inertia1.z * rxnl.y + r.inertia0.z * rxnl.z);
        h.w = qrot(r.rot, wl); // world inverse inertia times (r x n)
        const V3 tt = cross(h.w, h.rr);
        const float invMassGrid = 1.f / m;
        h.imc = invMassGrid + (imR + dot(nrm, tt));
        if (!(h.imc > 0.f))
            return v3(0.f, 0.f, 0.f);
        h.ok = true;
        h.Jn = -1.f * vn / h.imc;
        h.vt = rel - nrm * vn;
        h.vtn = sqrtf(sq(h.vt));
        h.hasT = h.vtn > kEps;
        V3 impT = v3(0.f, 0.f, 0.f);
        h.totJt = 0.f;
        h.e = v3(0.f, 0.f, 0.f);
        h.fJt = 0.f;
        h.fin = 0.f;
        h.caseA = false;
        if (h.hasT)
        {
            const float capA = r.params0.z * h.Jn, capB = h.vtn / h.imc;
            h.caseA = capA <= capB;
            h.fJt = fminf(capA, capB);
            h.fin = (h.vtn - h.fJt * h.imc) * r.params0.y;
            h.totJt = (h.vtn - h.fin) / h.imc;
            h.e = h.vt * (1.f / h.vtn);
            impT = (h.vt * -1.f / h.vtn) * h.totJt;
        }
        h.tot = nrm * h.Jn + impT;
        return v + h.tot * invMassGrid;
    }

    // Reverse of effMassResponse for g = dL/dresp: returns dL/dv (input velocity) and adds
    // dL/dn, dL/drel's rigid part (through gvr), dL/dr and dL/dm.
    __device__ __forceinline__ V3 effMassReverse(const ShapeRec &r, const EffMassHit &h, V3 g, float m, V3 nrm, V3 rel,
                                                 float vn, V3 &gn, V3 &grr, V3 &gvr, float &gm)
    {
        gn = v3(0.f, 0.f, 0.f);
        grr = v3(0.f, 0.f, 0.f);
        gvr = v3(0.f, 0.f, 0.f);
        if (!h.ok)
            return v3(0.f, 0.f, 0.f); // resp = 0 whatever the input
        const float im = 1.f / m, imc = h.imc, s = r.params0.y, mu = r.params0.z;
        V3 gvin = g;                                       // resp = v + tot / m
        const V3 gtot = g * im;
        gm += -dot(g, h.tot) * im * im;
        float gJn = dot(gtot, nrm);                        // tot = n Jn + impT
        gn = gtot * h.Jn;
        V3 ge = v3(0.f, 0.f, 0.f);
        float gtotJt = 0.f;
        if (h.hasT)
        {
            ge = gtot * (-h.totJt);                        // impT = -e totJt
            gtotJt = -dot(gtot, h.e);
        }
        float gvtn = gtotJt / imc;                         // totJt = (vtn - fin) / imc
        const float gfin = -gtotJt / imc;
        float gimc = -gtotJt * (h.vtn - h.fin) / (imc * imc);
        gvtn += gfin * s;                                  // fin = (vtn - fJt imc) s
        const float gfJt = -gfin * s * imc;
        gimc += -gfin * s * h.fJt;
        if (h.caseA)                                       // fJt = min(mu Jn, vtn / imc)
            gJn += gfJt * mu;
        else
        {
            gvtn += gfJt / imc;
            gimc += -gfJt * h.vtn / (imc * imc);
        }
        V3 gvt = v3(0.f, 0.f, 0.f);
        if (h.hasT)
            gvt = (ge - h.e * dot(h.e, ge)) * (1.f / h.vtn) + h.e * gvtn; // e = vt / vtn, vtn = |vt|
        float gvn = -gJn / imc;                            // Jn = -vn / imc
        gimc += gJn * vn / (imc * imc);
        V3 grel = gvt;                                     // vt = rel - n vn
        gn = gn - gvt * vn;
        gvn -= dot(gvt, nrm);
        grel = grel + nrm * gvn;                           // vn = rel . n
        gn = gn + rel * gvn;
        gm += -gimc * im * im;                             // imc = 1 / m + imr
        const V3 gu = h.w * (2.f * gimc);                  // imr = m_R^-1 + u^T Iw u, Iw u = w
        grr = cross(nrm, gu);                              // u = rr x n
        gn = gn + cross(gu, h.rr);
        gvin = gvin + grel;                                // rel = v - vr
        gvr = grel * -1.f;
        return gvin;
    }

    // Reverse of the grid update (per touched node): gridG (dL/dV_n) -> (dL/dP_n, dL/dM_n).
    // Clears gridA for the next replayed P2G.
    template <bool Multi>
    __global__ void __launch_bounds__(256) k_adjGridUpdate(const __grid_constant__ StepParams p0, SceneTable sc,
                                                          const SortHeader *__restrict__ hdr,
                                                          const unsigned *__restrict__ touchedList,
                                                          const ShapeRec *__restrict__ shapeTable, SdfPtrs sdf,
                                                          float4 *__restrict__ gridA, float4 *__restrict__ gridG)
    {
        __shared__ ShapeRec sh[Multi ? 1 : kMaxShapes];
        if (!Multi && p0.numShapes > 0)
            loadShapes(sh, shapeTable, p0.numShapes);
        __syncthreads();
        const unsigned nT = hdr->numTouchedBlocks;
        const unsigned perCta = blockDim.x / 64;
        for (unsigned base = blockIdx.x * perCta; base < nT; base += gridDim.x * perCta)
        {
            const unsigned bi = base + threadIdx.x / 64;
            if (bi >= nT)
                continue;
            const unsigned b = touchedList[bi];
            const StepParams &p = Multi ? sc.params[sceneOfBlock(sc, b)] : p0;
            const GridGeom &g = p.g;
            const ShapeRec *shp = Multi ? shapeTable + p.shapeBegin : sh;
            const unsigned l = threadIdx.x & 63;
            const unsigned lb = b - g.blockBase;
            const int bx = lb % g.nb.x, by = (lb / g.nb.x) % g.nb.y, bz = lb / (g.nb.x * g.nb.y);
            const int i = 4 * bx + (l & 3), j = 4 * by + ((l >> 2) & 3), k = 4 * bz + (l >> 4);
            if (!inGrid(g, i, j, k))
                continue;
            const unsigned a = b * 64u + l;
            const float4 acc = gridA[a];
            gridA[a] = make_float4(0.f, 0.f, 0.f, 0.f);
            const float4 gg = gridG[a];
            V3 gv = v3(gg.x, gg.y, gg.z);
            if (acc.w < p.cutoff)
            {
                gridG[a] = make_float4(gv.x, gv.y, gv.z, 0.f); // light node: V = P
                continue;
            }
            const V3 v0 = v3(acc.x / acc.w, acc.y / acc.w, acc.z / acc.w);
            const V3 pos = v3((float)i * g.dx, (float)j * g.dx, (float)k * g.dx) + v3(g.gmin.x, g.gmin.y, g.gmin.z) +
                           v0 * p.dt;
            // forward contact chain: velocity before each active contact
            const bool effMass = p.contactModel == CRB200_CONTACT_EFFECTIVE_MASS;
            V3 vin[kAdjMaxHits];
            int hs[kAdjMaxHits];
            int nh = 0;
            V3 v = v0;
            for (int s = 0; s < p.numShapes; ++s)
            {
                const ShapeRec &r = shp[s];
                float dist;
                V3 nrm, lp, gl;
                if (!adjShapeEval(r, pos, sdf, dist, nrm, lp, gl))
                    continue;
                if (!(dist < r.params0.x))
                    continue;
                const V3 wrel = pos - v3(r.pos);
                const V3 rv = r.kind == S_STATIC ? v3(0.f, 0.f, 0.f) : v3(r.linVel) + cross(v3(r.angVel), wrel);
                const V3 rel = v - rv;
                const float vn = dot(rel, nrm);
                if (vn >= 0.f)
                    continue;
                if (nh < kAdjMaxHits)
                {
                    vin[nh] = v;
                    hs[nh] = s;
                    ++nh;
                }
                if (effMass && r.kind == S_DYNAMIC)
                {
                    EffMassHit h;
                    v = effMassResponse(r, v, acc.w, wrel, nrm, rel, vn, h);
                    continue;
                }
                const V3 tang = rel - nrm * vn;
                const float tn = sqrtf(sq(tang));
                const float fc = fmaxf(r.params0.z * vn / (tn + kEps), -1.f);
                v = (tang + tang * fc) * r.params0.y + rv;
            }
            // boundary band
            if (i < 2 || i > g.n.x - 3)
                gv.x = 0.f;
            if (j < 2 || j > g.n.y - 3)
                gv.y = 0.f;
            if (k < 2 || k > g.n.z - 3)
                gv.z = 0.f;
            V3 gpos = v3(0.f, 0.f, 0.f);
            float gmEff = 0.f; // dL/dm through the effective-mass responses
            for (int h = nh - 1; h >= 0; --h)
            {
                const ShapeRec &r = shp[hs[h]];
                float dist, J[9];
                V3 nrm, lp, gl;
                adjShapeEval(r, pos, sdf, dist, nrm, lp, gl);
                const V3 wrel = pos - v3(r.pos);
                const V3 rv = r.kind == S_STATIC ? v3(0.f, 0.f, 0.f) : v3(r.linVel) + cross(v3(r.angVel), wrel);
                const V3 rel = vin[h] - rv;
                const float vn = dot(rel, nrm);
                if (effMass && r.kind == S_DYNAMIC)
                {
                    EffMassHit eh;
                    (void)effMassResponse(r, vin[h], acc.w, wrel, nrm, rel, vn, eh);
                    V3 gn, grr, gvr;
                    gv = effMassReverse(r, eh, gv, acc.w, nrm, rel, vn, gn, grr, gvr, gmEff);
                    if (eh.ok)
                    {
                        adjNormalJacobian(r, lp, gl, J);
                        gpos = gpos + adjJtG(J, gn) + grr + cross(gvr, v3(r.angVel));
                    }
                    continue;
                }
                const V3 tang = rel - nrm * vn;
                const float tn = sqrtf(sq(tang));
                const float fr = r.params0.z, sticky = r.params0.y;
                const float arg = fr * vn / (tn + kEps);
                V3 grel = v3(0.f, 0.f, 0.f), gn = v3(0.f, 0.f, 0.f);
                if (arg > -1.f)
                {
                    const float fc = arg;
                    V3 gt = gv * (sticky * (1.f + fc));
                    const float gfc = sticky * dot(tang, gv);
                    const float den = tn + kEps;
                    float gvn = gfc * fr / den;
                    const float gtn = -gfc * fr * vn / (den * den);
                    if (tn > 0.f)
                        gt = gt + tang * (gtn / tn);
                    grel = gt;
                    gn = gt * (-vn);
                    gvn -= dot(nrm, gt);
                    grel = grel + nrm * gvn;
                    gn = gn + rel * gvn;
                }
                const V3 gvr = gv - grel;
                adjNormalJacobian(r, lp, gl, J);
                gpos = gpos + adjJtG(J, gn);
                if (r.kind != S_STATIC)
                    gpos = gpos + cross(gvr, v3(r.angVel));
                gv = grel;
            }
            const V3 gv0 = gv + gpos * p.dt;
            const float im = 1.f / acc.w;
            gridG[a] = make_float4(gv0.x * im, gv0.y * im, gv0.z * im, -dot(gv0, v0) * im + gmEff);
        }
    }

    // ---------------------------------------------------------------------------------------
    // Reverse of P2G and of the stress (per particle); completes the adjoint of the substep's input
    // state and accumulates dL/dlambda, dL/dmu.
    template <bool Multi>
    __global__ void __launch_bounds__(kAdjThreads, 5) k_adjP2G(const __grid_constant__ StepParams p0, SceneTable sc,
                                                   const float4 *__restrict__ xm, const float4 *__restrict__ vel,
                                                   const unsigned char *__restrict__ mask,
                                                   const float4 *__restrict__ matParams, const float *__restrict__ F,
                                                   const float *__restrict__ Cm, const float *__restrict__ V0,
                                                   unsigned stride, const float4 *__restrict__ gridG,
                                                   float4 *__restrict__ aX, float4 *__restrict__ aV,
                                                   float *__restrict__ aF, float *__restrict__ aC,
                                                   float4 *__restrict__ aMat)
    {
        // the particle's streams, staged at entry (launched with kAdjThreads threads)
        __shared__ float4 sX[kAdjThreads], sVel[kAdjThreads], sMp[kAdjThreads], sAx[kAdjThreads], sAm[kAdjThreads];
        __shared__ float sF[9][kAdjThreads], sC[9][kAdjThreads], sAF[9][kAdjThreads], sV0[kAdjThreads];
        const unsigned t = threadIdx.x;
        const unsigned i = blockIdx.x * blockDim.x + t;
        if (i >= (Multi ? sc.numParticles : p0.numActive))
            return;
        stage16(&sX[t], &xm[i]);
        stage16(&sVel[t], &vel[i]);
        stage16(&sMp[t], &matParams[i]);
        stage16(&sAx[t], &aX[i]);
        stage16(&sAm[t], &aMat[i]);
#pragma unroll
        for (int k = 0; k < 9; ++k)
        {
            stage4(&sF[k][t], &F[k * stride + i]);
            stage4(&sC[k][t], &Cm[k * stride + i]);
            stage4(&sAF[k][t], &aF[k * stride + i]);
        }
        stage4(&sV0[t], &V0[i]);
        const bool active = mask[i] != 0;
        const unsigned si = Multi ? sc.particleScene[i] : 0u;
        stageWait();
        if (!active || (Multi && si == 0xFFFFu))
            return;
        const StepParams &p = Multi ? sc.params[si] : p0;
        const GridGeom &g = p.g;
        const float4 x4 = sX[t];
        const float m = x4.w;
        const Stencil st = stencilOf(g, v3(x4));
        if (!st.finite)
            return;
        float w[3][3], dw[3][3];
        weights(st.fx, w);
        weightGrads(st.fx, dw);
        M3 Fp, Cp;
#pragma unroll
        for (int k = 0; k < 9; ++k)
        {
            Fp.m[k] = sF[k][t];
            Cp.m[k] = sC[k][t];
        }
        const float4 mp = sMp[t];
        const float lam = mp.x, mu = mp.y;
        const float J = det3(Fp);
        const float Jc = J < 1e-6f ? 1e-6f : J;
        const M3 tau = kirchhoffStress(Fp, lam, mu, 1);
        const float coef = -p.dt * 4.f * g.invDx * g.invDx * sV0[t];
        M3 A;
#pragma unroll
        for (int e = 0; e < 9; ++e)
            A.m[e] = tau.m[e] * coef + Cp.m[e] * m;
        const V3 u = (v3(sVel[t]) + v3(p.gravity) * p.dt) * m;
        // node value u + A d_n = u' + sum_c a_c o_c with u' = u - A (fx dx), a_c = dx A(:, c)
        const V3 fd = v3(st.fx.x * g.dx, st.fx.y * g.dx, st.fx.z * g.dx);
        const V3 up = u - v3(A.m[0] * fd.x + A.m[3] * fd.y + A.m[6] * fd.z, A.m[1] * fd.x + A.m[4] * fd.y + A.m[7] * fd.z,
                             A.m[2] * fd.x + A.m[5] * fd.y + A.m[8] * fd.z);
        const V3 a0 = v3(A.m[0], A.m[1], A.m[2]) * g.dx, a1 = v3(A.m[3], A.m[4], A.m[5]) * g.dx,
                 a2 = v3(A.m[6], A.m[7], A.m[8]) * g.dx;
        // one pass: gu = sum w gP, M[3c + r] = sum w gP_r o_c, gs = sum dw/dfx (gP.(u + A d) + gM m)
        V3 gu = v3(0.f, 0.f, 0.f), gs = v3(0.f, 0.f, 0.f);
        float Mo[9];
#pragma unroll
        for (int e = 0; e < 9; ++e)
            Mo[e] = 0.f;
        const StencilAddrs sa = stencilAddrs(g, st);
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b)
#pragma unroll
                for (int c = 0; c < 3; ++c)
                {
                    if (!sa.ok(a, b, c))
                        continue;
                    const float4 gg = __ldg(&gridG[sa.addr(a, b, c)]);
                    const V3 gP = v3(gg.x, gg.y, gg.z);
                    const float wab = w[a][0] * w[b][1];
                    const float W = wab * w[c][2];
                    const V3 gWd = v3(dw[a][0] * w[b][1] * w[c][2], w[a][0] * dw[b][1] * w[c][2], wab * dw[c][2]);
                    const V3 wgP = gP * W;
                    gu = gu + wgP;
                    if (a) { Mo[0] += (float)a * wgP.x; Mo[1] += (float)a * wgP.y; Mo[2] += (float)a * wgP.z; }
                    if (b) { Mo[3] += (float)b * wgP.x; Mo[4] += (float)b * wgP.y; Mo[5] += (float)b * wgP.z; }
                    if (c) { Mo[6] += (float)c * wgP.x; Mo[7] += (float)c * wgP.y; Mo[8] += (float)c * wgP.z; }
                    const V3 val = up + a0 * (float)a + a1 * (float)b + a2 * (float)c;
                    gs = gs + gWd * (dot(gP, val) + gg.w * m);
                }
        // gA(r, c) = sum w gP_r d_c = dx (M(r, c) - gu_r fx_c);  sum_n w A^T gP = A^T gu
        const float ddx = g.invDx * g.dx;
        float gA[9];
        const float fxv[3] = {st.fx.x, st.fx.y, st.fx.z};
        const float guv[3] = {gu.x, gu.y, gu.z};
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int r = 0; r < 3; ++r)
                gA[3 * c + r] = g.dx * (Mo[3 * c + r] - guv[r] * fxv[c]);
        const V3 AtG = v3(A.m[0] * gu.x + A.m[1] * gu.y + A.m[2] * gu.z, A.m[3] * gu.x + A.m[4] * gu.y + A.m[5] * gu.z,
                          A.m[6] * gu.x + A.m[7] * gu.y + A.m[8] * gu.z);
        const V3 gx = gs * g.invDx - AtG * ddx;
        // stress: tau = mu (F F^T - I) + lam log(J) I
        float gtau[9];
#pragma unroll
        for (int e = 0; e < 9; ++e)
            gtau[e] = coef * gA[e];
        float dmu = 0.f;
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int r = 0; r < 3; ++r)
            {
                const float bb = Fp.m[r] * Fp.m[c] + Fp.m[3 + r] * Fp.m[3 + c] + Fp.m[6 + r] * Fp.m[6 + c];
                dmu += gtau[3 * c + r] * (bb - (r == c ? 1.f : 0.f));
            }
        const float trg = gtau[0] + gtau[4] + gtau[8];
        const float dlam = logf(Jc) * trg;
        // gF = mu (gtau + gtau^T) F + lam tr(gtau) F^-T
        float gF[9];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int r = 0; r < 3; ++r)
            {
                float s = 0.f;
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    s += (gtau[3 * k + r] + gtau[3 * r + k]) * Fp.m[3 * c + k];
                gF[3 * c + r] = mu * s;
            }
        if (J >= 1e-6f)
        {
            const M3 Fi = inverse3(Fp);
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int r = 0; r < 3; ++r)
                    gF[3 * c + r] += lam * trg * Fi.m[3 * r + c];
        }
        const float4 ax = sAx[t];
        aX[i] = make_float4(ax.x + gx.x, ax.y + gx.y, ax.z + gx.z, 0.f);
        aV[i] = make_float4(gu.x * m, gu.y * m, gu.z * m, 0.f);
#pragma unroll
        for (int e = 0; e < 9; ++e)
        {
            aF[e * stride + i] = sAF[e][t] + gF[e];
            aC[e * stride + i] = gA[e] * m;
        }
        const float4 am = sAm[t];
        aMat[i] = make_float4(am.x + dlam, am.y + dmu, 0.f, 0.f);
    }

    __global__ void k_adjAddSeeds(unsigned n, const float4 *__restrict__ seed, float4 *__restrict__ aX)
    {
        const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= n)
            return;
        const float4 s = seed[i], a = aX[i];
        aX[i] = make_float4(a.x + s.x, a.y + s.y, a.z + s.z, 0.f);
    }

    // ---------------------------------------------------------------------------------------
    // Host side
    void Solver::releaseAdjoint()
    {
        releaseAdjointGraphs();
        void *bufs[] = {adjCkpt, adjSeg, aX, aV, aMat, aF, aC, gridG, adjForce, adjTorque, adjTape};
        for (void *b : bufs)
            if (b)
                cudaFree(b);
        adjCkpt = adjSeg = nullptr;
        aX = aV = aMat = nullptr;
        aF = aC = nullptr;
        gridG = adjForce = adjTorque = nullptr;
        adjCkptCap = adjSegCap = adjTapeCap = 0;
        adjTape = nullptr;
        adjRecorded = false;
    }

    // State blob: x|m (float4 n), v (float4 n), F (9 planes of n), C (9 planes of n).
    // One kernel moves a particle state between the solver's arrays and a blob (x|m and v as
    // float4, then F and C as 9 planes of n floats each); loading also clears the bin counters and
    // the carried-records flag (what invalidateRecords does), so a replayed state costs one graph
    // node instead of seven.
    __global__ void k_stateCopy(unsigned n, unsigned stride, bool load, float4 *__restrict__ x, float4 *__restrict__ v,
                                float *__restrict__ F, float *__restrict__ C, unsigned char *__restrict__ blob,
                                unsigned *__restrict__ blockCount, unsigned numBlockCounts,
                                unsigned *__restrict__ cellCount, unsigned numCellCounts, unsigned *__restrict__ flag)
    {
        // the blob has the live arrays' layout (x, v, then the F and C planes, `stride` apart), so
        // the reverse kernels can read a saved state in place
        float4 *bx = reinterpret_cast<float4 *>(blob);
        float4 *bv = bx + stride;
        float *bF = reinterpret_cast<float *>(bv + stride);
        float *bC = bF + 9ull * stride;
        const unsigned stepN = gridDim.x * blockDim.x, t0 = blockIdx.x * blockDim.x + threadIdx.x;
        // x and v (float4 items), then the 18 planes of F and C (float items): independent
        // elements, so every thread has loads in flight
        for (unsigned t = t0; t < 2u * n; t += stepN)
        {
            const unsigned i = t < n ? t : t - n;
            float4 *a = t < n ? x : v;
            float4 *b = t < n ? bx : bv;
            if (load)
                a[i] = b[i];
            else
                b[i] = a[i];
        }
#pragma unroll 1
        for (int plane = 0; plane < 18; ++plane)
        {
            float *a = plane < 9 ? F + (size_t)plane * stride : C + (size_t)(plane - 9) * stride;
            float *b = plane < 9 ? bF + (size_t)plane * stride : bC + (size_t)(plane - 9) * stride;
            for (unsigned i = t0; i < n; i += stepN)
            {
                if (load)
                    a[i] = b[i];
                else
                    b[i] = a[i];
            }
        }
        if (load)
        {
            for (unsigned j = blockIdx.x * blockDim.x + threadIdx.x; j < numBlockCounts; j += stepN)
                blockCount[j] = 0u;
            for (unsigned j = blockIdx.x * blockDim.x + threadIdx.x; j < numCellCounts; j += stepN)
                cellCount[j] = 0u;
            if (blockIdx.x == 0 && threadIdx.x == 0)
            {
                flag[0] = 0u; // recordsValid
                flag[1] = 0u; // pbRecordsValid
            }
        }
    }

    int Solver::saveState(unsigned char *dst)
    {
        const unsigned n = totalParticles();
        if (!n)
            return CRB200_OK;
        if (int r = residentSyncPlanes()) // F and C of the resident path into the particle-id planes
            return r;
        k_stateCopy<<<std::min((n + 255) / 256, 2u * (unsigned)strideCtas), 256, 0, stream>>>(
            n, (unsigned)numMaxParticles, false, positionMass, velocity, F, Cm, dst, nullptr, 0u, nullptr, 0u, nullptr);
        CRB_LAUNCHED(1);
        return CRB200_OK;
    }

    int Solver::loadState(const unsigned char *src)
    {
        // the loaded state replaces the resident one (the next resident call re-sorts from it), and
        // the substeps that follow (the adjoint's replays among them) sort their particles
        resValid = false;
        resPlanesStale = false;
        CRB_CHECK(cudaMemsetAsync(&header->sortSkip, 0, sizeof(unsigned), stream));
        const unsigned n = totalParticles();
        const unsigned nodes = totalBlocks * 64u;
        k_stateCopy<<<std::max(1u, std::min((std::max(n, nodes) + 255) / 256, 2u * (unsigned)strideCtas)), 256, 0, stream>>>(
            n, (unsigned)numMaxParticles, true, positionMass, velocity, F, Cm, const_cast<unsigned char *>(src),
            blockCount, totalBlocks + 1, cellCount, nodes, &header->recordsValid);
        CRB_LAUNCHED(1);
        return CRB200_OK;
    }

    // What the adjoint differentiates: MLS-MPM, the kinematic and effective-mass contact models,
    // Neo-Hookean active particles, analytic shapes of uniform scale.  Reads the (small) shape table and the particle
    // material types / mask back to the host once per recording.
    int Solver::adjointCheck()
    {
        if (solverType != CRB200_SOLVER_GPU_MLS)
        {
            setLastError("adjoint: only the MLS-MPM solver has an adjoint");
            return CRB200_ERR_UNSUPPORTED;
        }
        for (const StepParams &sp : allParams())
            if (sp.contactModel != CRB200_CONTACT_KINEMATIC && sp.contactModel != CRB200_CONTACT_EFFECTIVE_MASS)
            {
                setLastError("adjoint: unknown contact model");
                return CRB200_ERR_UNSUPPORTED;
            }
        const unsigned n = totalParticles();
        if (n == 0 || !matType || !activeMask || !matParams)
        {
            setLastError("adjoint: no particles, or materials / active mask not bound");
            return CRB200_ERR_NOT_INITIALIZED;
        }
        std::vector<int> types(n);
        std::vector<unsigned char> msk(n);
        CRB_CHECK(cudaMemcpyAsync(types.data(), matType, n * sizeof(int), cudaMemcpyDeviceToHost, stream));
        CRB_CHECK(cudaMemcpyAsync(msk.data(), activeMask, n, cudaMemcpyDeviceToHost, stream));
        const int nsh = isBatch() ? totalShapes() : numShapes;
        std::vector<ShapeRec> recs(nsh > 0 ? nsh : 1);
        if (nsh > 0)
        {
            gatherShapes(stream);
            CRB_LAUNCHED(1);
            CRB_CHECK(cudaMemcpyAsync(recs.data(), shapeTable, nsh * sizeof(ShapeRec), cudaMemcpyDeviceToHost, stream));
        }
        CRB_CHECK(cudaStreamSynchronize(stream));
        std::vector<unsigned short> owner;
        if (isBatch())
        {
            owner.resize(n);
            CRB_CHECK(cudaMemcpy(owner.data(), dParticleScene, n * sizeof(unsigned short), cudaMemcpyDeviceToHost));
        }
        for (unsigned q = 0; q < n; ++q)
        {
            if (isBatch() && owner[q] == 0xFFFF)
                continue;
            if (!msk[q] || types[q] != CRB200_MATERIAL_NEOHOOKEAN)
            {
                setLastError("adjoint: every particle must be active and Neo-Hookean");
                return CRB200_ERR_UNSUPPORTED;
            }
        }
        for (int q = 0; q < nsh; ++q)
        {
            const ShapeRec &r = recs[q];
            if (r.gtype != G_BOX && r.gtype != G_SPHERE && r.gtype != G_PLANE && r.gtype != G_CAPSULE)
            {
                setLastError("adjoint: only box, sphere, plane and capsule shapes are differentiated");
                return CRB200_ERR_UNSUPPORTED;
            }
            if (!(r.invScale.x == r.invScale.y && r.invScale.y == r.invScale.z))
            {
                setLastError("adjoint: shapes must have uniform scale");
                return CRB200_ERR_UNSUPPORTED;
            }
        }
        return CRB200_OK;
    }

    int Solver::adjointRecord(int T, int K, const int *caps, int nc, float4 *capturedX)
    {
        if (!initialized)
        {
            setLastError("adjoint: solver not initialized");
            return CRB200_ERR_NOT_INITIALIZED;
        }
        int r = adjointCheck();
        if (r != CRB200_OK)
            return r;
        const unsigned n = totalParticles();
        const size_t sb = stateBytes();
        const int nck = T / K + 2; // checkpoints at 0, K, 2K, ... and the final state
        if ((size_t)nck * sb > adjCkptCap)
        {
            if (adjCkpt)
                cudaFree(adjCkpt);
            adjCkpt = nullptr;
            adjCkptCap = 0;
            CRB_CHECK(cudaMalloc(&adjCkpt, (size_t)nck * sb));
            adjCkptCap = (size_t)nck * sb;
        }
        adjSubsteps = T;
        adjInterval = K;
        adjCaptures.assign(caps, caps + nc);
        adjRecorded = false;
        if ((r = saveState(adjCkpt)) != CRB200_OK)
            return r;
        int t = 0, c = 0;
        while (t < T)
        {
            int next = std::min(T, (t / K + 1) * K);
            if (c < nc)
                next = std::min(next, adjCaptures[c]);
            if ((r = stepMany(next - t)) != CRB200_OK)
                return r;
            t = next;
            if (c < nc && adjCaptures[c] == t)
            {
                CRB_CHECK(cudaMemcpyAsync(capturedX + (size_t)c * n, positionMass, n * sizeof(float4),
                                          cudaMemcpyDeviceToDevice, stream));
                ++c;
            }
            if (t % K == 0 && t < T)
                if ((r = saveState(adjCkpt + (size_t)(t / K) * sb)) != CRB200_OK)
                    return r;
        }
        if ((r = saveState(adjCkpt + (size_t)(nck - 1) * sb)) != CRB200_OK)
            return r;
        adjRecorded = true;
        return CRB200_OK;
    }

    // Tape layout of one slot (each part 256-byte aligned).
    size_t Solver::tapeSlotBytes() const
    {
        auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
        const size_t nodes = (size_t)totalBlocks * 64;
        return 2 * al(nodes * sizeof(float4)) + al((size_t)numMaxParticles * 4) + al(nodes * 4) +
               3 * al(((size_t)totalBlocks + 1) * 4) + al(sizeof(SortHeader));
    }

    Solver::TapeSlot Solver::tapeSlot(int k) const
    {
        auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
        const size_t nodes = (size_t)totalBlocks * 64;
        unsigned char *p = adjTape + (size_t)k * tapeSlotBytes();
        TapeSlot t;
        t.gridA = reinterpret_cast<float4 *>(p);
        p += al(nodes * sizeof(float4));
        t.gridV = reinterpret_cast<float4 *>(p);
        p += al(nodes * sizeof(float4));
        t.sortedIds = reinterpret_cast<unsigned *>(p);
        p += al((size_t)numMaxParticles * 4);
        t.cellStart = reinterpret_cast<unsigned *>(p);
        p += al(nodes * 4);
        t.blockStart = reinterpret_cast<unsigned *>(p);
        p += al(((size_t)totalBlocks + 1) * 4);
        t.activeList = reinterpret_cast<unsigned *>(p);
        p += al(((size_t)totalBlocks + 1) * 4);
        t.touchedList = reinterpret_cast<unsigned *>(p);
        p += al(((size_t)totalBlocks + 1) * 4);
        t.hdr = reinterpret_cast<SortHeader *>(p);
        return t;
    }

    // One reverse substep from the tape of slot k (the replayed forward of the same input state
    // wrote its P2G grid, grid velocities and sort there); the input state itself is loaded.
    template <bool Multi>
    int Solver::adjointSubstepTape(int k, const unsigned char *state)
    {
        const TapeSlot ts = tapeSlot(k);
        // the substep's input state, saved by its replay in the layout of the live arrays
        const size_t nm = (size_t)numMaxParticles;
        const float4 *sx = reinterpret_cast<const float4 *>(state), *sv = sx + nm;
        const float *sF = reinterpret_cast<const float *>(sv + nm), *sC = sF + 9 * nm;
        const StepParams p = params();
        const SceneTable sc = sceneTable();
        const unsigned pg = (sc.numParticles + kAdjThreads - 1) / kAdjThreads;
        const SdfPtrs sp{reinterpret_cast<const int4 *>(sdf.dimension), reinterpret_cast<const float4 *>(sdf.lowerBoundCellSize),
                         reinterpret_cast<const float4 *>(sdf.gradientSignedDistance)};
        const unsigned stride = (unsigned)numMaxParticles;
        CRB_CHECK(cudaMemsetAsync(gridG, 0, (size_t)totalBlocks * 64 * sizeof(float4), stream));
        k_adjG2P<Multi><<<pg, kAdjThreads, 0, stream>>>(p, sc, sx, activeMask, sF, stride, shapeTable, sp, ts.gridV, aX, aV, aF,
                                                aC, gridG, records);
        k_accumulate<0, Multi><<<p2gCtas, 64, 0, stream>>>(p, sc, ts.hdr, ts.activeList, ts.blockStart, ts.sortedIds,
                                                            ts.cellStart, records, cutMasks, gridG, gridF);
        k_adjGridUpdate<Multi><<<updCtas, 256, 0, stream>>>(p, sc, ts.hdr, ts.touchedList, shapeTable, sp, ts.gridA, gridG);
        k_adjP2G<Multi><<<pg, kAdjThreads, 0, stream>>>(p, sc, sx, sv, activeMask, matParams, sF, sC, V0, stride, gridG, aX, aV,
                                                aF, aC, aMat);
        CRB_LAUNCHED(4);
        return CRB200_OK;
    }

    int Solver::adjointBackward(const float4 *gradX, float4 *gradV0, float4 *gradMat, float4 *gradX0)
    {
        if (!adjRecorded)
        {
            setLastError("adjoint: no recorded trajectory (call AdjointRecord first)");
            return CRB200_ERR_NOT_INITIALIZED;
        }
        const unsigned n = totalParticles();
        const size_t sb = stateBytes();
        const int T = adjSubsteps, K = adjInterval;
        const int nck = T / K + 2;
        const size_t nodes = (size_t)totalBlocks * 64;
        if (!aX)
        {
            const size_t nm = (size_t)numMaxParticles;
            CRB_CHECK(cudaMalloc(&aX, nm * sizeof(float4)));
            CRB_CHECK(cudaMalloc(&aV, nm * sizeof(float4)));
            CRB_CHECK(cudaMalloc(&aMat, nm * sizeof(float4)));
            CRB_CHECK(cudaMalloc(&aF, 9 * nm * sizeof(float)));
            CRB_CHECK(cudaMalloc(&aC, 9 * nm * sizeof(float)));
            CRB_CHECK(cudaMalloc(&gridG, nodes * sizeof(float4)));
            const int ns = std::max(shapes.size, 1);
            CRB_CHECK(cudaMalloc(&adjForce, ns * sizeof(float4)));
            CRB_CHECK(cudaMalloc(&adjTorque, ns * sizeof(float4)));
        }
        if ((size_t)K * tapeSlotBytes() > adjTapeCap)
        {
            if (adjTape)
                cudaFree(adjTape);
            adjTape = nullptr;
            adjTapeCap = 0;
            CRB_CHECK(cudaMalloc(&adjTape, (size_t)K * tapeSlotBytes()));
            adjTapeCap = (size_t)K * tapeSlotBytes();
        }
        if ((size_t)K * sb > adjSegCap)
        {
            if (adjSeg)
                cudaFree(adjSeg);
            adjSeg = nullptr;
            adjSegCap = 0;
            CRB_CHECK(cudaMalloc(&adjSeg, (size_t)K * sb));
            adjSegCap = (size_t)K * sb;
        }
        const size_t nm = (size_t)numMaxParticles;
        CRB_CHECK(cudaMemsetAsync(aX, 0, nm * sizeof(float4), stream));
        CRB_CHECK(cudaMemsetAsync(aV, 0, nm * sizeof(float4), stream));
        CRB_CHECK(cudaMemsetAsync(aMat, 0, nm * sizeof(float4), stream));
        CRB_CHECK(cudaMemsetAsync(aF, 0, 9 * nm * sizeof(float), stream));
        CRB_CHECK(cudaMemsetAsync(aC, 0, 9 * nm * sizeof(float), stream));
        const unsigned pg = (n + 127) / 128;
        int c = (int)adjCaptures.size() - 1;
        int r = runBackward(gradX, n, pg, sb, T, K, c);
        adjReplay = false;
        if (r != CRB200_OK)
            return r;
        // leave the solver in the recorded final state
        if ((r = loadState(adjCkpt + (size_t)(nck - 1) * sb)) != CRB200_OK)
            return r;
        if (gradV0)
            CRB_CHECK(cudaMemcpyAsync(gradV0, aV, n * sizeof(float4), cudaMemcpyDeviceToDevice, stream));
        if (gradMat)
            CRB_CHECK(cudaMemcpyAsync(gradMat, aMat, n * sizeof(float4), cudaMemcpyDeviceToDevice, stream));
        if (gradX0)
            CRB_CHECK(cudaMemcpyAsync(gradX0, aX, n * sizeof(float4), cudaMemcpyDeviceToDevice, stream));
        return CRB200_OK;
    }

    // One CUDA graph per segment slot k: replay[k] = save the state into slot k and run one forward
    // substep, reverse[k] = one reverse substep on slot k's saved state.  Built once per configuration
    // (pointers, parameters, K) and replayed for every segment of every backward pass.
    int Solver::captureGraph(int which, int k, cudaGraphExec_t *out, int *kernels)
    {
        const size_t sb = stateBytes();
        const uint64_t before = launchCount();
        CRB_CHECK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        const int r = which == 1 ? reverseBody(k, sb) : replayBody(k, sb, which == 2);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(stream, &g);
        const uint64_t captured = launchCount() - before;
        noteLaunches((uint64_t)0 - captured);
        if (r != CRB200_OK)
        {
            if (g)
                cudaGraphDestroy(g);
            return r;
        }
        if (e != cudaSuccess)
            return cudaFail(e, "adjoint graph capture");
        e = cudaGraphInstantiate(out, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess)
            return cudaFail(e, "adjoint graph instantiate");
        *kernels = (int)captured;
        return CRB200_OK;
    }

    // The state blob of segment slot k, in the layout of the live arrays.
    Solver::StateView Solver::slotState(int k, size_t sb) const
    {
        const size_t nm = (size_t)numMaxParticles;
        StateView v;
        v.x = reinterpret_cast<float4 *>(adjSeg + (size_t)k * sb);
        v.v = v.x + nm;
        v.F = reinterpret_cast<float *>(v.v + nm);
        v.C = v.F + 9 * nm;
        return v;
    }

    // Points the solver's particle state at `v` (the live arrays again for v = {}), returning what
    // it pointed at.
    Solver::StateView Solver::bindState(const StateView &v)
    {
        const StateView old{positionMass, velocity, F, Cm};
        positionMass = v.x;
        velocity = v.v;
        F = v.F;
        Cm = v.C;
        return old;
    }

    // replay slot k: the forward substep runs on slot k as its state and writes slot k's tape; its
    // G2P writes the updated state into slot k + 1, so slot k keeps the substep's input for the
    // reverse pass without a copy (the segment's last slot: only up to the grid update)
    int Solver::replayBody(int k, size_t sb, bool last)
    {
        const StateView live = bindState(slotState(k, sb));
        if (!last)
        {
            const StateView next = slotState(k + 1, sb);
            outX = next.x;
            outV = next.v;
            outF = next.F;
            outC = next.C;
        }
        tapeActive = k;
        const int r = last ? (isBatch() ? launchStepT<true>(true) : launchStepT<false>(true)) : launchStep();
        tapeActive = -1;
        outX = outV = nullptr;
        outF = outC = nullptr;
        bindState(live);
        return r;
    }

    // reverse slot k: the reverse kernels read the slot's saved input state in place
    int Solver::reverseBody(int k, size_t sb)
    {
        const unsigned char *slot = adjSeg + (size_t)k * sb;
        return isBatch() ? adjointSubstepTape<true>(k, slot) : adjointSubstepTape<false>(k, slot);
    }

    void Solver::releaseAdjointGraphs()
    {
        for (auto &v : {&adjReplayG, &adjReverseG, &adjReplayLastG})
            for (cudaGraphExec_t gx : *v)
                if (gx)
                    cudaGraphExecDestroy(gx);
        adjReplayG.clear();
        adjReverseG.clear();
        adjReplayLastG.clear();
        adjGraphKernels[0] = adjGraphKernels[1] = adjGraphKernels[2] = 0;
    }

    int Solver::adjointGraphs(int K)
    {
        if ((int)adjReplayG.size() == K && adjGraphVersion == configVersion && adjGraphSeg == adjSeg &&
            adjGraphTape == adjTape)
            return CRB200_OK;
        releaseAdjointGraphs();
        adjReplayG.assign(K, nullptr);
        adjReverseG.assign(K, nullptr);
        adjReplayLastG.assign(K, nullptr);
        for (int k = 0; k < K; ++k)
        {
            // slot K-1 is always a segment's last substep: it has no full replay (which would write
            // slot K)
            int r = k + 1 < K ? captureGraph(0, k, &adjReplayG[k], &adjGraphKernels[0]) : CRB200_OK;
            if (r == CRB200_OK)
                r = captureGraph(1, k, &adjReverseG[k], &adjGraphKernels[1]);
            if (r == CRB200_OK)
                r = captureGraph(2, k, &adjReplayLastG[k], &adjGraphKernels[2]);
            if (r != CRB200_OK)
            {
                releaseAdjointGraphs();
                return r;
            }
        }
        adjGraphVersion = configVersion;
        adjGraphSeg = adjSeg;
        adjGraphTape = adjTape;
        return CRB200_OK;
    }

    int Solver::runBackward(const float4 *gradX, unsigned n, unsigned pg, size_t sb, int T, int K, int c)
    {
        int r;
        adjReplay = true;
        const bool graphs = stream != nullptr && !phaseTiming;
        if (graphs && (r = adjointGraphs(K)) != CRB200_OK)
            return r;
        for (int seg = (T - 1) / K; seg >= 0; --seg)
        {
            const int t0 = seg * K, t1 = std::min(T, t0 + K);
            // replay the segment's inputs s_t0 .. s_(t1-1) in slots 0 .. t1-t0-1, each substep
            // writing its slot's tape; the checkpoint is loaded into slot 0
            {
                const StateView live = bindState(slotState(0, sb));
                r = loadState(adjCkpt + (size_t)seg * sb);
                bindState(live);
                if (r != CRB200_OK)
                    return r;
            }
            for (int t = t0; t < t1; ++t)
            {
                const int k = t - t0;
                const bool last = t + 1 == t1;
                if (graphs)
                {
                    CRB_CHECK(cudaGraphLaunch(last ? adjReplayLastG[k] : adjReplayG[k], stream));
                    noteLaunches(adjGraphKernels[last ? 2 : 0]);
                }
                else if ((r = replayBody(k, sb, last)) != CRB200_OK)
                    return r;
            }
            for (int t = t1; t > t0; --t)
            {
                while (c >= 0 && adjCaptures[c] == t)
                {
                    k_adjAddSeeds<<<pg, 128, 0, stream>>>(n, gradX + (size_t)c * n, aX);
                    CRB_LAUNCHED(1);
                    --c;
                }
                const int k = t - 1 - t0;
                if (graphs)
                {
                    CRB_CHECK(cudaGraphLaunch(adjReverseG[k], stream));
                    noteLaunches(adjGraphKernels[1]);
                }
                else if ((r = reverseBody(k, sb)) != CRB200_OK)
                    return r;
            }
        }
        return CRB200_OK;
    }
} // namespace crb200

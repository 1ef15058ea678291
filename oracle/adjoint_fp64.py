"""ORACLE / TEST INFRASTRUCTURE ONLY: FP64 host adjoint of the MLS-MPM substep.

The reference has no gradient path, so the GPU adjoint kernels are checked against this module,
and this module is pinned two ways in the CPU tests: (1) its forward substep reproduces the FP64
restatement of the reference (oracle/mpm_oracle.cpp, ``PortOracle(scene, 64)``) to rounding, and
(2) its gradients match central finite differences of its own FP64 forward.

Forward arithmetic followed (reference file:line):
  * stencil, quadratic B-spline weights       mls_mpm_algorithm.h:170-175, shape_functions.h:44-57
  * Neo-Hookean Kirchhoff stress, J >= 1e-6   constitutive_models.h:62-75
  * P2G momentum / mass with the affine term  mls_mpm_algorithm.h:147-241
  * grid update: 1e-4 mass cutoff (light nodes keep momentum), contact at x_n + v dt, two-node
    boundary band                             mls_mpm_algorithm.h:243-294
  * rigid contact (kinematic contact model: friction, drag, rigid velocity) and the particle
    push-out                                  mpm_rigid_contact.h:101-399
  * G2P: v, C = 4/dx sum w d v^T (the reference's transposed outer product), x += v dt clamped to
    the grid bounds, F <- (I + dt C) F        mls_mpm_algorithm.h:296-390

Scope (the same as the GPU adjoint): MLS-MPM, Neo-Hookean particles, the kinematic and the
effective-mass contact models (mpm_rigid_contact.h:219-320: two-body normal and friction impulses
against dynamic shapes), static / kinematic / dynamic shapes of analytic geometry (box, sphere,
plane, capsule) with uniform scale, no slicers.  Branch decisions (contact on/off, friction clamp, position clamp, grid mass
cutoff) are held fixed when differentiating.

State layout: x, v (N, 3); F, C (N, 3, 3) with F[p, r, c] = F(r, c).
"""
from __future__ import annotations

import numpy as np

GEOM_BOX, GEOM_SPHERE, GEOM_PLANE, GEOM_CAPSULE = 0, 1, 2, 3
EPS = float(np.float32(1.1920928955078125e-07))
OFFS = np.array([(a, b, c) for a in range(3) for b in range(3) for c in range(3)], np.int64)  # n = 9a + 3b + c


def quat_matrix(q):
    """Rotation matrix of quaternion (x, y, z, w): qrot(q, v) = R v."""
    x, y, z, w = (float(t) for t in q)
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def _skew(w):
    return np.array([[0.0, -w[2], w[1]], [w[2], 0.0, -w[0]], [-w[1], w[0], 0.0]])


class _Shape:
    def __init__(self, st, sid: int):
        self.kind = int(st.shape_type[sid])
        gid = int(st.geom_idx[sid])
        self.gtype = int(st.geom_type[gid])
        if self.gtype not in (GEOM_BOX, GEOM_SPHERE, GEOM_PLANE, GEOM_CAPSULE):
            raise NotImplementedError("adjoint: only box / sphere / plane / capsule shapes")
        self.gp = st.geom_params[gid].astype(np.float64)
        self.p = st.position[sid, :3].astype(np.float64)
        self.R = quat_matrix(st.rotation[sid])
        isc = st.inv_scale[sid, :3].astype(np.float64)
        if not (isc[0] == isc[1] == isc[2]):
            raise NotImplementedError("adjoint: shapes must have uniform scale")
        self.s = float(isc[0])
        self.lin = st.lin_vel[sid, :3].astype(np.float64)
        self.ang = st.ang_vel[sid, :3].astype(np.float64)
        smooth, drag, friction, fatten = (float(t) for t in st.params0[sid])
        self.smooth, self.drag, self.friction, self.fatten = smooth, drag, friction, fatten
        # dynamic shapes under the effective-mass model: centre of mass (local), inverse mass and
        # the world inverse inertia R I^-1 R^T (inertiaInv0 = diagonal, inertiaInv1 = xy, xz, yz;
        # mpm_rigid_contact.h:84-94)
        self.com = st.com_inv_mass[sid, :3].astype(np.float64)
        self.inv_mass = float(st.com_inv_mass[sid, 3])
        d0, d1 = st.inertia0[sid].astype(np.float64), st.inertia1[sid].astype(np.float64)
        Iloc = np.array([[d0[0], d1[0], d1[1]], [d1[0], d0[1], d1[2]], [d1[1], d1[2], d0[2]]])
        self.Iw = self.R @ Iloc @ self.R.T

    def eval(self, pos):
        """dist (K,), unit normal n (K,3) and dn/dpos (K,3,3) at world points (mpm_rigid_contact.h:129-148)."""
        s, R = self.s, self.R
        lp = ((pos - self.p) @ R) * s
        K = pos.shape[0]
        Jl = np.zeros((K, 3, 3))
        g = self.gp
        if self.gtype == GEOM_PLANE:
            grad = np.tile([0.0, 1.0, 0.0], (K, 1))
            dr = lp[:, 1].copy()
        elif self.gtype == GEOM_SPHERE:
            ln = np.sqrt((lp * lp).sum(1))
            lc = np.maximum(ln, EPS)
            grad = lp / lc[:, None]
            dr = ln - g[0]
            Jl = (np.eye(3)[None] - grad[:, :, None] * grad[:, None, :]) / lc[:, None, None]
        elif self.gtype == GEOM_CAPSULE:
            h2 = g[1] * 2.0
            pa = lp.copy()
            pa[:, 1] -= g[1]
            h = np.clip(-pa[:, 1] / h2, 0.0, 1.0)
            inner = (h > 0.0) & (h < 1.0)
            pa[:, 1] += h2 * h
            d = np.sqrt((pa * pa).sum(1))
            dc = np.maximum(d, EPS)
            grad = pa / dc[:, None]
            dr = d - g[0]
            P = np.tile(np.eye(3), (K, 1, 1))
            P[inner, 1, 1] = 0.0  # the closest point slides along the axis
            Jl = ((np.eye(3)[None] - grad[:, :, None] * grad[:, None, :]) / dc[:, None, None]) @ P
        else:  # box
            pen = np.abs(lp) - g[None, :3]
            sg = np.where(lp < 0.0, -1.0, 1.0)
            gm = pen.max(1)
            q = np.maximum(pen, 0.0)
            ln = np.sqrt((q * q).sum(1))
            out = gm > 0.0
            dirv = np.zeros((K, 3))
            dirv[out] = q[out] / ln[out, None]
            ins = ~out
            ax = np.where(pen[:, 0] > pen[:, 1], np.where(pen[:, 0] > pen[:, 2], 0, 2),
                          np.where(pen[:, 1] > pen[:, 2], 1, 2))
            dirv[ins, ax[ins]] = 1.0
            grad = sg * dirv
            dr = ln + np.minimum(gm, 0.0)
            if out.any():
                do = dirv[out]
                Dq = sg[out] * (pen[out] > 0.0)
                Jo = (np.eye(3)[None] - do[:, :, None] * do[:, None, :]) / ln[out, None, None]
                Jl[out] = sg[out][:, :, None] * Jo * Dq[:, None, :]
        # uniform scale: |grad * s| = s, so dist = dr / s - fatten and the normal is R grad
        dist = dr / s - self.fatten
        n = grad @ R.T
        Jn = np.einsum("ij,kjl,lm->kim", R, Jl, R.T) * s
        return dist, n, Jn

    def rigid_vel(self, pos):
        if self.kind == 0:
            return np.zeros_like(pos)
        return self.lin[None] + np.cross(self.ang[None], pos - self.p[None])


class Fp64Adjoint:
    """FP64 MLS-MPM forward with a tape of every substep's state, and its reverse pass."""

    def __init__(self, scene):
        from crmpm_b200 import scenes as S

        if scene.solver_type != S.SOLVER_MLS:
            raise NotImplementedError("adjoint: MLS-MPM only")
        if scene.contact_model not in (0, 1):
            raise NotImplementedError("adjoint: kinematic or effective-mass contact model only")
        self.eff_mass = scene.contact_model == 1
        if not np.all(scene.mat_type == S.MAT_NEOHOOKEAN):
            raise NotImplementedError("adjoint: Neo-Hookean particles only")
        self.sc = scene
        self.gmin = scene.grid_min.astype(np.float64)
        self.gmax = scene.grid_max.astype(np.float64)
        # the solver's inputs are float32: round them as the solver receives them
        self.dx = float(np.float32(scene.cell_size))
        self.invDx = 1.0 / self.dx
        self.n = np.array(scene.grid_dims(), np.int64)
        self.dt = float(np.float32(scene.dt))
        self.grav = scene.gravity.astype(np.float64)
        self.m = scene.pos_mass[:, 3].astype(np.float64)
        self.shapes = [_Shape(scene.shapes, int(i)) for i in scene.shapes.shape_ids]
        self.mask = scene.mask.astype(bool)
        if not self.mask.all():
            raise NotImplementedError("adjoint: every particle must be active")
        nn = self.n
        ii = np.arange(nn[0] * nn[1] * nn[2])
        self.node_ijk = np.stack([ii % nn[0], (ii // nn[0]) % nn[1], ii // (nn[0] * nn[1])], 1)
        self.V0 = self._initial_volume(scene.pos_mass[:, :3].astype(np.float64))

    # ------------------------------------------------------------------ stencil helpers
    def _stencil(self, x):
        sp = (x - self.gmin) * self.invDx
        base = np.trunc(sp - 0.5).astype(np.int64)
        fx = sp - base
        w = np.stack([0.5 * (1.5 - fx) ** 2, 0.75 - (fx - 1.0) ** 2, 0.5 * (fx - 0.5) ** 2], 1)  # (N, 3a, 3d)
        dw = np.stack([fx - 1.5, -2.0 * (fx - 1.0), fx - 0.5], 1)
        a, b, c = OFFS[:, 0], OFFS[:, 1], OFFS[:, 2]
        W = w[:, a, 0] * w[:, b, 1] * w[:, c, 2]  # (N, 27)
        gW = np.stack([dw[:, a, 0] * w[:, b, 1] * w[:, c, 2], w[:, a, 0] * dw[:, b, 1] * w[:, c, 2],
                       w[:, a, 0] * w[:, b, 1] * dw[:, c, 2]], 2)  # dW/dfx (N, 27, 3)
        ijk = base[:, None, :] + OFFS[None]
        nn = self.n
        valid = np.all((ijk >= 0) & (ijk < nn[None, None]), 2) & self.mask[:, None]
        flat = ijk[..., 0] + nn[0] * (ijk[..., 1] + nn[1] * ijk[..., 2])
        flat = np.where(valid, flat, 0)
        d = (OFFS[None].astype(np.float64) - fx[:, None, :]) * self.dx  # (N, 27, 3)
        return flat, valid, W * valid, gW * valid[..., None], d

    def _scatter(self, flat, valid, vals):
        size = int(np.prod(self.n))
        out = np.zeros((size,) + vals.shape[2:])
        f = flat[valid]
        v = vals[valid]
        if v.ndim == 1:
            return np.bincount(f, weights=v, minlength=size)
        for k in range(v.shape[1]):
            out[:, k] = np.bincount(f, weights=v[:, k], minlength=size)
        return out

    def _initial_volume(self, x):
        flat, valid, W, _, _ = self._stencil(x)
        M = self._scatter(flat, valid, W * self.m[:, None])
        dens = ((M[flat] / (self.dx ** 3)) * W).sum(1)
        return np.where(dens > float(np.float32(1e-8)), self.m / np.maximum(dens, 1e-300), float(np.float32(1e-8)))

    # ------------------------------------------------------------------ forward pieces
    def _stress(self, F, lam, mu):
        J = np.linalg.det(F)
        Jc = np.maximum(J, 1e-6)
        b = F @ F.transpose(0, 2, 1)
        tau = mu[:, None, None] * (b - np.eye(3)[None]) + (lam * np.log(Jc))[:, None, None] * np.eye(3)[None]
        return tau, J, Jc, b

    def _p2g(self, x, v, F, C, lam, mu):
        flat, valid, W, gW, d = self._stencil(x)
        tau, J, Jc, b = self._stress(F, lam, mu)
        coef = -self.dt * 4.0 * self.invDx * self.invDx * self.V0
        A = coef[:, None, None] * tau + self.m[:, None, None] * C
        u = self.m[:, None] * (v + self.grav[None] * self.dt)
        val = u[:, None, :] + np.einsum("prc,pnc->pnr", A, d)
        P = self._scatter(flat, valid, W[..., None] * val)
        M = self._scatter(flat, valid, W * self.m[:, None])
        return dict(flat=flat, valid=valid, W=W, gW=gW, d=d, tau=tau, J=J, Jc=Jc, b=b, coef=coef, A=A, u=u,
                    val=val, P=P, M=M)

    def _grid_update(self, P, M, tape: bool = False):
        V = P.copy()
        heavy = M >= float(np.float32(1e-4))
        idx = np.nonzero(heavy)[0]
        v0 = P[idx] / M[idx, None]
        pos = self.node_ijk[idx] * self.dx + self.gmin[None] + v0 * self.dt
        v = v0.copy()
        steps = []
        Mh = M[idx]
        for sh in self.shapes:
            dist, n, Jn = sh.eval(pos)
            vr = sh.rigid_vel(pos)
            rel = v - vr
            vn = (rel * n).sum(1)
            act = (dist < sh.smooth) & (vn < 0.0)
            t = rel - n * vn[:, None]
            tn = np.sqrt((t * t).sum(1))
            if self.eff_mass and sh.kind == 2:
                em = self._eff_mass_forward(sh, pos, n, v, rel, vn, t, tn, Mh)
                resp = em["resp"]
                if tape:
                    steps.append(dict(sh=sh, n=n, Jn=Jn, rel=rel, vn=vn, act=act, t=t, tn=tn, em=em, v=v))
            else:
                arg = sh.friction * vn / (tn + EPS)
                fc = np.maximum(arg, -1.0)
                resp = (t + t * fc[:, None]) * sh.drag + vr
                if tape:
                    steps.append(dict(sh=sh, n=n, Jn=Jn, rel=rel, vn=vn, act=act, t=t, tn=tn, fc=fc,
                                      clamped=arg <= -1.0))
            v = np.where(act[:, None], resp, v)
        ijk = self.node_ijk[idx]
        bc = np.stack([(ijk[:, k] < 2) | (ijk[:, k] > self.n[k] - 3) for k in range(3)], 1)
        v = np.where(bc, 0.0, v)
        V[idx] = v
        if tape:
            return V, dict(idx=idx, v0=v0, M=M[idx], P=P[idx], steps=steps, bc=bc)
        return V

    def _eff_mass_forward(self, sh, pos, n, v, rel, vn, vt, vtn, M):
        """Effective-mass response of a dynamic shape (mpm_rigid_contact.h:219-320): the normal and
        friction impulses of a two-body contact between the node (mass M) and the rigid body; the
        node velocity is zero where the impulse is undefined (non-positive inverse masses, :231)."""
        K = pos.shape[0]
        out = dict(ok=np.zeros(K, bool), resp=np.zeros((K, 3)))
        if sh.inv_mass <= 0.0:
            return out
        rr = (pos - sh.p[None]) - (sh.R @ sh.com)[None]
        u = np.cross(rr, n)
        imr = sh.inv_mass + np.einsum("ki,ij,kj->k", u, sh.Iw, u)
        imc = 1.0 / M + imr
        ok = imc > 0.0
        imc_s = np.where(ok, imc, 1.0)
        Jn = -vn / imc_s
        has_t = vtn > EPS
        vtn_s = np.where(has_t, vtn, 1.0)
        capA = sh.friction * Jn
        capB = vtn / imc_s
        caseA = capA <= capB
        fJt = np.where(caseA, capA, capB)
        fin = (vtn - fJt * imc_s) * sh.drag
        totJt = (vtn - fin) / imc_s
        e = vt / vtn_s[:, None]
        impT = np.where(has_t[:, None], -e * totJt[:, None], 0.0)
        tot = n * Jn[:, None] + impT
        resp = v + tot / M[:, None]
        out.update(ok=ok, resp=np.where(ok[:, None], resp, 0.0), rr=rr, u=u, imr=imr, imc=imc_s, Jn=Jn,
                   has_t=has_t, vtn=vtn_s, caseA=caseA, fJt=fJt, fin=fin, totJt=totJt, e=e, tot=tot, M=M)
        return out

    def _eff_mass_reverse(self, sh, st, g):
        """Reverse of _eff_mass_forward for gradient g = dL/dresp: (dL/dv_in, dL/dpos, dL/dM)."""
        em = st["em"]
        K = g.shape[0]
        gv_in = np.zeros((K, 3))
        gpos = np.zeros((K, 3))
        gM = np.zeros(K)
        if sh.inv_mass <= 0.0:
            return gv_in, gpos, gM
        ok = em["ok"][:, None]
        g = np.where(ok, g, 0.0)
        n, rel, vn, vt, M = st["n"], st["rel"], st["vn"], st["t"], em["M"]
        imc, Jn, vtn, e, totJt, fJt, fin = em["imc"], em["Jn"], em["vtn"], em["e"], em["totJt"], em["fJt"], em["fin"]
        has_t = em["has_t"]
        s_, mu = sh.drag, sh.friction
        gv_in += g                                   # resp = v + tot / M
        gtot = g / M[:, None]
        gM += -(g * em["tot"]).sum(1) / M ** 2
        gJn = (gtot * n).sum(1)                      # tot = n Jn + impT
        gn = gtot * Jn[:, None]
        ge = np.where(has_t[:, None], -gtot * totJt[:, None], 0.0)   # impT = -e totJt
        gtotJt = np.where(has_t, -(gtot * e).sum(1), 0.0)
        gvtn = gtotJt / imc                          # totJt = (vtn - fin) / imc
        gfin = -gtotJt / imc
        gimc = -gtotJt * (vtn - fin) / imc ** 2
        gvtn += gfin * s_                            # fin = (vtn - fJt imc) s
        gfJt = -gfin * s_ * imc
        gimc += -gfin * s_ * fJt
        caseA = em["caseA"]                          # fJt = min(mu Jn, vtn / imc)
        gJn += np.where(caseA, gfJt * mu, 0.0)
        gvtn += np.where(caseA, 0.0, gfJt / imc)
        gimc += np.where(caseA, 0.0, -gfJt * vtn / imc ** 2)
        gvt = (ge - e * (e * ge).sum(1, keepdims=True)) / vtn[:, None]   # e = vt / vtn
        gvt += gvtn[:, None] * e                     # vtn = |vt|
        gvt = np.where(has_t[:, None], gvt, 0.0)
        gvn = -gJn / imc                             # Jn = -vn / imc
        gimc += gJn * vn / imc ** 2
        grel = gvt.copy()                            # vt = rel - n vn
        gn += -gvt * vn[:, None]
        gvn += -(gvt * n).sum(1)
        grel += gvn[:, None] * n                     # vn = rel . n
        gn += gvn[:, None] * rel
        gM += -gimc / M ** 2                         # imc = 1 / M + imr
        gimr = gimc
        gu = 2.0 * (em["u"] @ sh.Iw.T) * gimr[:, None]   # imr = m^-1 + u^T Iw u (Iw symmetric)
        rr = em["rr"]
        grr = np.cross(n, gu)                        # u = rr x n
        gn += np.cross(gu, rr)
        gpos += grr                                  # rr = pos - p - R com
        gv_in += grel                                # rel = v - vr
        gvr = -grel
        gpos += np.einsum("kji,kj->ki", st["Jn"], gn)
        if sh.kind != 0:
            gpos += np.cross(gvr, sh.ang[None])
        return gv_in, gpos, gM

    def _push_out(self, xs, tape: bool = False):
        steps = []
        for sh in self.shapes:
            dist, n, Jn = sh.eval(xs)
            hit = dist < 0.0
            if tape:
                steps.append(dict(n=n, Jn=Jn, dist=dist, hit=hit))
            xs = np.where(hit[:, None], xs - n * dist[:, None], xs)
        return xs, steps

    def step(self, x, v, F, C, lam, mu):
        f = self._p2g(x, v, F, C, lam, mu)
        V = self._grid_update(f["P"], f["M"])
        Vn = V[f["flat"]] * f["valid"][..., None]
        W, d = f["W"], f["d"]
        vn = (W[..., None] * Vn).sum(1)
        Cn = 4.0 * self.invDx * np.einsum("pn,pnr,pnc->prc", W, d, Vn)
        xn = np.clip(x + vn * self.dt, self.gmin, self.gmax)
        xn, _ = self._push_out(xn)
        Fn = (np.eye(3)[None] + Cn * self.dt) @ F
        keep = self.mask
        return (np.where(keep[:, None], xn, x), np.where(keep[:, None], vn, v),
                np.where(keep[:, None, None], Fn, F), np.where(keep[:, None, None], Cn, C))

    # ------------------------------------------------------------------ trajectory and reverse pass
    def forward(self, lam, mu, v0, num_substeps: int, x0=None, F0=None, C0=None):
        """Run num_substeps from (x0, v0, F0 = I, C0 = 0); keeps every state.  Returns x after each substep."""
        N = self.m.shape[0]
        x = self.sc.pos_mass[:, :3].astype(np.float64) if x0 is None else np.asarray(x0, np.float64)
        v = np.asarray(v0, np.float64).reshape(N, 3)
        F = np.tile(np.eye(3), (N, 1, 1)) if F0 is None else np.asarray(F0, np.float64)
        C = np.zeros((N, 3, 3)) if C0 is None else np.asarray(C0, np.float64)
        self.lam = np.asarray(lam, np.float64).reshape(N)
        self.mu = np.asarray(mu, np.float64).reshape(N)
        self.tape = [(x, v, F, C)]
        for _ in range(num_substeps):
            x, v, F, C = self.step(x, v, F, C, self.lam, self.mu)
            self.tape.append((x, v, F, C))
        return np.stack([t[0] for t in self.tape[1:]])

    def backward(self, gx_seeds: dict):
        """Reverse pass.  gx_seeds maps substep t (1-based: the state after substep t) to dL/dx (N, 3).

        Returns dict with g_lam, g_mu (N,), g_v0 (N, 3), g_x0 (N, 3), g_F0, g_C0 (N, 3, 3)."""
        T = len(self.tape) - 1
        N = self.m.shape[0]
        gx = np.zeros((N, 3))
        gv = np.zeros((N, 3))
        gF = np.zeros((N, 3, 3))
        gC = np.zeros((N, 3, 3))
        glam = np.zeros(N)
        gmu = np.zeros(N)
        mk = self.mask.astype(np.float64)
        for t in range(T, 0, -1):
            if t in gx_seeds:
                gx = gx + np.asarray(gx_seeds[t], np.float64)
            x, v, F, C = self.tape[t - 1]
            gx, gv, gF, gC, dl, dm = self._reverse_substep(x, v, F, C, gx * mk[:, None], gv * mk[:, None],
                                                           gF * mk[:, None, None], gC * mk[:, None, None])
            glam += dl
            gmu += dm
        if 0 in gx_seeds:
            gx = gx + np.asarray(gx_seeds[0], np.float64)
        return dict(g_lam=glam, g_mu=gmu, g_v0=gv, g_x0=gx, g_F0=gF, g_C0=gC)

    def _reverse_substep(self, x, v, F, C, gxo, gvo, gFo, gCo):
        lam, mu = self.lam, self.mu
        f = self._p2g(x, v, F, C, lam, mu)
        V, gt = self._grid_update(f["P"], f["M"], tape=True)
        flat, valid, W, gW, d = f["flat"], f["valid"], f["W"], f["gW"], f["d"]
        Vn = V[flat] * valid[..., None]
        vn = (W[..., None] * Vn).sum(1)
        Cn = 4.0 * self.invDx * np.einsum("pn,pnr,pnc->prc", W, d, Vn)
        xpre = x + vn * self.dt
        xc = np.clip(xpre, self.gmin, self.gmax)
        _, psteps = self._push_out(xc, tape=True)
        inv, dt, k4 = self.invDx, self.dt, 4.0 * self.invDx
        # ---- G2P reverse
        gCt = gCo + dt * gFo @ F.transpose(0, 2, 1)
        gF = (np.eye(3)[None] + dt * Cn).transpose(0, 2, 1) @ gFo
        g = gxo.copy()
        for st in reversed(psteps):
            h = st["hit"]
            n, Jn, dist = st["n"], st["Jn"], st["dist"]
            gin = g - n * (n * g).sum(1, keepdims=True) - dist[:, None] * np.einsum("kji,kj->ki", Jn, g)
            g = np.where(h[:, None], gin, g)
        inside = (xpre >= self.gmin) & (xpre <= self.gmax)
        g = g * inside
        gx = g.copy()
        gvt = gvo + dt * g
        gCd = np.einsum("prc,pnr->pnc", gCt, d)  # (gC^T d)_c
        gVn = W[..., None] * (gvt[:, None, :] + k4 * gCd)
        gWn = (Vn * gvt[:, None, :]).sum(2) + k4 * (gCd * Vn).sum(2)
        gdn = k4 * W[..., None] * np.einsum("prc,pnc->pnr", gCt, Vn)
        gx += inv * (gWn[..., None] * gW).sum(1) - inv * self.dx * gdn.sum(1)
        gV = self._scatter(flat, valid, gVn)
        # ---- grid update reverse
        gP = gV.copy()  # light nodes: V = P
        gM = np.zeros(gV.shape[0])
        idx = gt["idx"]
        gv_ = np.where(gt["bc"], 0.0, gV[idx])
        gpos = np.zeros_like(gv_)
        gM_eff = np.zeros(gv_.shape[0])
        for st in reversed(gt["steps"]):
            sh = st["sh"]
            act = st["act"]
            if "em" in st:
                gvi, gpi, gmi = self._eff_mass_reverse(sh, st, gv_)
                gv_ = np.where(act[:, None], gvi, gv_)
                gpos = gpos + np.where(act[:, None], gpi, 0.0)
                gM_eff += np.where(act, gmi, 0.0)
                continue
            n, rel, vn_, tt, tn, fc = st["n"], st["rel"], st["vn"], st["t"], st["tn"], st["fc"]
            gr = gv_
            free = ~st["clamped"]
            g_t = sh.drag * (1.0 + fc)[:, None] * gr
            g_fc = sh.drag * (tt * gr).sum(1)
            den = tn + EPS
            g_vn = np.where(free, g_fc * sh.friction / den, 0.0)
            g_tn = np.where(free, -g_fc * sh.friction * vn_ / den ** 2, 0.0)
            g_t = np.where(free[:, None], g_t + (g_tn / np.maximum(tn, 1e-300))[:, None] * tt * (tn > 0)[:, None],
                           0.0)
            g_rel = g_t.copy()
            g_n = -vn_[:, None] * g_t
            g_vn = g_vn - (n * g_t).sum(1)
            g_rel += g_vn[:, None] * n
            g_n += g_vn[:, None] * rel
            g_vr = gr - g_rel
            gp_add = np.einsum("kji,kj->ki", st["Jn"], g_n)
            if sh.kind != 0:
                gp_add = gp_add + np.cross(g_vr, sh.ang[None])
            gv_ = np.where(act[:, None], g_rel, gv_)
            gpos = gpos + np.where(act[:, None], gp_add, 0.0)
        gv0 = gv_ + dt * gpos
        Mi = gt["M"]
        gP[idx] = gv0 / Mi[:, None]
        gM[idx] = -(gv0 * gt["v0"]).sum(1) / Mi + gM_eff
        # ---- P2G reverse
        gPn = gP[flat] * valid[..., None]
        gMn = gM[flat] * valid
        A, u, val = f["A"], f["u"], f["val"]
        gu = (W[..., None] * gPn).sum(1)
        gA = np.einsum("pn,pnr,pnc->prc", W, gPn, d)
        gdn2 = W[..., None] * np.einsum("prc,pnr->pnc", A, gPn)
        gWn2 = (gPn * val).sum(2) + gMn * self.m[:, None]
        gx += inv * (gWn2[..., None] * gW).sum(1) - inv * self.dx * gdn2.sum(1)
        gv = self.m[:, None] * gu
        gC = self.m[:, None, None] * gA
        gtau = f["coef"][:, None, None] * gA
        b, J, Jc = f["b"], f["J"], f["Jc"]
        dmu = (gtau * (b - np.eye(3)[None])).sum((1, 2))
        trg = np.trace(gtau, axis1=1, axis2=2)
        dlam = np.log(Jc) * trg
        gF += mu[:, None, None] * (gtau + gtau.transpose(0, 2, 1)) @ F
        Finv_T = np.linalg.inv(F).transpose(0, 2, 1)
        gF += np.where((J >= 1e-6)[:, None, None], (lam * trg)[:, None, None] * Finv_T, 0.0)
        return gx, gv, gF, gC, dlam, dmu


def lame(E, nu):
    """Lamé parameters from Young's modulus and Poisson ratio (the reference's benchmark formula)."""
    return E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), E / (2.0 * (1.0 + nu))


def lame_grad(E, nu):
    """d(lambda, mu)/d(E, nu) as ((dl/dE, dl/dnu), (dm/dE, dm/dnu))."""
    den = (1.0 + nu) * (1.0 - 2.0 * nu)
    dl_dE = nu / den
    dl_dnu = E * (den - nu * (1.0 - 2.0 * nu - 2.0 * (1.0 + nu))) / den ** 2
    dm_dE = 1.0 / (2.0 * (1.0 + nu))
    dm_dnu = -E / (2.0 * (1.0 + nu) ** 2)
    return (dl_dE, dl_dnu), (dm_dE, dm_dnu)

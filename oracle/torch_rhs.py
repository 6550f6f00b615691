"""Differentiable CPU restatement of the DGSEM right-hand side (torch, float64).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the reference gradient of
the adjoint (vector-Jacobian product) kernels, never by the product path.

It restates the same operator as ``dgsem_oracle.cpp`` in its ``fixed``
(compat = 0) form — the reference's algorithm without its value-changing
quirks — written with vectorised torch operations so that
``torch.autograd`` yields exact (to rounding) Jacobian-vector and
vector-Jacobian products.  The reference has no adjoint, so this gradient is
pinned only through its forward values, which the tests check against the C
oracle (itself checked against the reference's own sources).

Reference functions followed (file:line in the Prandtl tree):
  ComputeLogMean            src/BasicOperations/BasicOperations.cpp:6-12
  ComputeVolumeFlux         src/RiemannSolvers/ChandrashekarFlux.cpp:11-83
  ComputeFaceFlux           src/RiemannSolvers/ChandrashekarFlux.cpp:85-161
  ComputeViscousFlux        src/Fluxes/NavierStokesFlux.cpp:12-90
  Conserv2Entropy           src/BasicOperations/BasicOperations.cpp:81-104
  EntropyGrad2PrimGrad      src/BasicOperations/BasicOperations.cpp:126-170
  ComputeBlendingCoefficient src/Operators/DGSEMOperator.cpp:60-80
  CheckSmoothness           src/Indicators/PerssonPeraireIndicator.cpp:21-58
  AssembleElementVector     src/Integrators/DGSEMIntegrator/DGSEMIntegrator.cpp:224-433, 601-864
  ComputeFVFluxes           DGSEMIntegrator.cpp:972-1196
  AssembleFaceVector        DGSEMIntegrator.cpp:151-222, 435-549
  LiftingBR1                src/Integrators/Lifting/LiftingBR1/LiftingBR1.cpp:10-272
"""
from __future__ import annotations

import numpy as np
import torch

from prandtl_b200.mesh import CartesianMesh, gll_nodes

SHARPNESS = 9.21024


def _derivative_matrices(x, w):
    Np = len(x)
    wb = np.ones(Np)
    for i in range(Np):
        for j in range(Np):
            if i != j:
                wb[i] *= x[i] - x[j]
    wb = 1.0 / wb
    D = np.zeros((Np, Np))
    for i in range(Np):
        for l in range(Np):
            if l != i:
                D[i, l] = wb[l] / wb[i] / (x[i] - x[l])
                D[i, i] -= D[i, l]
    Dhat = D.copy()
    Dhat[0, 0] += 1.0 / w[0]
    Dhat[-1, -1] -= 1.0 / w[-1]
    Dhat2 = 2.0 * D
    Dhat2[0, 0] += 1.0 / w[0]
    Dhat2[-1, -1] -= 1.0 / w[-1]
    return D, Dhat, Dhat2


def _legendre01(N, x):
    z = 2.0 * x - 1.0
    L = np.zeros((len(x), N + 1))
    L[:, 0] = 1.0
    if N >= 1:
        L[:, 1] = z
    for n in range(1, N):
        L[:, n + 1] = ((2 * n + 1) * z * L[:, n] - n * L[:, n - 1]) / (n + 1)
    return L


def logmean(x, y):
    """(y - x) / ln(y / x) with the reference's series branch for u < 1e-4."""
    s = x + y
    f = (y - x) / s
    u = f * f
    small = u < 1e-4
    series = s * 52.5 / (105.0 + u * (35.0 + u * (21.0 + 15.0 * u)))
    # keep the unused branch finite so that its (masked) gradient is too
    ys = torch.where(small, 2.0 * x, y)
    direct = (ys - x) / torch.log(ys / x)
    return torch.where(small, series, direct)


def _norm(vsq):
    """sqrt(vsq) with a zero (not NaN) derivative at vsq = 0."""
    pos = vsq > 0
    return torch.where(pos, torch.sqrt(torch.where(pos, vsq, torch.ones_like(vsq))), torch.zeros_like(vsq))


class TorchDGSEM:
    """RHS of the fixed DGSEM operator on a Cartesian mesh: periodic, or with
    the boundary conditions 1-5 of mesh.boundaries (Euler)."""

    def __init__(self, mesh: CartesianMesh, parabolic=False, blending=True, gamma=1.4, Pr=0.72, mu=0.0,
                 alpha_max=0.5, alpha_min=0.001, face_dissipation=1.0):
        self.m = mesh
        self.dim, self.N = mesh.dim, mesh.order
        self.Np = self.N + 1
        self.nv = self.dim + 2
        self.ne = mesh.num_elements
        self.parabolic, self.blending = parabolic, blending
        self.gamma, self.Pr, self.mu = gamma, Pr, mu
        self.gm1 = gamma - 1.0
        self.alpha_max, self.alpha_min, self.diss = alpha_max, alpha_min, face_dissipation
        x, w = gll_nodes(self.Np)
        self.x, self.w = np.asarray(x), np.asarray(w)
        D, Dh, Dh2 = _derivative_matrices(self.x, self.w)
        self.D, self.Dhat, self.Dhat2 = (torch.tensor(a) for a in (D, Dh, Dh2))
        h = list(mesh.h)
        J = float(np.prod(h))
        self.J = J
        self.adj = [J / hd for hd in h]
        self.area = list(self.adj)
        self.face_scale = 1.0 / (self.w[0] * J)
        # subcell interface normals (affine element): adj + sum_{l<i} w_l sum_m D(l,m) adj
        self.snor = []
        for d in range(self.dim):
            a = self.adj[d]
            nor = [a + sum(self.w[l] * sum(a * D[l, m] for m in range(self.Np)) for l in range(i))
                   for i in range(self.Np + 1)]
            self.snor.append(torch.tensor(nor))
        V1 = _legendre01(self.N, self.x)
        self.Vinv = torch.tensor(np.linalg.inv(V1))
        deg = np.arange(self.Np)
        if self.dim == 2:
            md = np.maximum.outer(deg, deg)  # [j, i]
        else:
            md = np.maximum(np.maximum.outer(deg, deg)[None, :, :], deg[:, None, None])  # [k, j, i]
        self.maxdeg = torch.tensor(md)
        self.T = 0.5 * 10 ** (-1.8 * self.N ** 0.25)
        self.nbr = torch.tensor(np.asarray(mesh.nbr, dtype=np.int64).reshape(self.ne, 2 * self.dim))
        self.bcs = dict(getattr(mesh, "boundaries", None) or {})
        if self.bcs and parabolic:
            raise ValueError("boundary faces: Euler only")
        for b, (typ, _) in self.bcs.items():
            if typ not in range(1, 12):
                raise ValueError(f"boundary condition {b}: unknown type {typ}")
            if typ == 8 and self.dim != 2:
                raise ValueError("the total-pressure inflow is 2D only")

    # ---- layout ----
    def shape(self, u):
        return u.reshape((self.nv, self.ne) + (self.Np,) * self.dim)

    # ---- pointwise physics ----
    def prims(self, s):
        rho = s[0]
        vel = [s[1 + d] / rho for d in range(self.dim)]
        vsq = sum(v * v for v in vel)
        p = self.gm1 * (s[self.dim + 1] - 0.5 * rho * vsq)
        return rho, vel, p

    def volume_flux(self, sa, sb, d, metric):
        ra, va, pa = self.prims(sa)
        rb, vb, pb = self.prims(sb)
        ba, bb = 0.5 * ra / pa, 0.5 * rb / pb
        rho_ln = logmean(ra, rb)
        beta_ln = logmean(ba, bb)
        p_hat = 0.5 * (ra + rb) / (ba + bb)
        vm = [0.5 * (va[k] + vb[k]) for k in range(self.dim)]
        h = sum(-0.25 * (va[k] ** 2 + vb[k] ** 2) + vm[k] ** 2 for k in range(self.dim))
        h = h + 0.5 / (beta_ln * self.gm1) + p_hat / rho_ln
        fm = rho_ln * vm[d] * metric
        F = [fm] + [fm * vm[k] + (p_hat * metric if k == d else 0.0) for k in range(self.dim)] + [fm * h]
        return F

    def face_flux(self, sa, sb, d, nrm):
        """Chandrashekar flux + local Lax-Friedrichs along axis d with signed
        normal magnitude nrm (fixed form of the 3D energy term)."""
        ra, va, pa = self.prims(sa)
        rb, vb, pb = self.prims(sb)
        ba, bb = 0.5 * ra / pa, 0.5 * rb / pb
        rho_ln = logmean(ra, rb)
        beta_ln = logmean(ba, bb)
        p_hat = 0.5 * (ra + rb) / (ba + bb)
        rho_mean = 0.5 * (ra + rb)
        drho = rb - ra
        vm = [0.5 * (va[k] + vb[k]) for k in range(self.dim)]
        h = sum(-0.25 * (va[k] ** 2 + vb[k] ** 2) + vm[k] ** 2 for k in range(self.dim))
        h = h + 0.5 / (beta_ln * self.gm1) + p_hat / rho_ln
        diss = sum(0.5 * drho * va[k] * vb[k] + rho_mean * (vb[k] - va[k]) * vm[k] for k in range(self.dim))
        diss = diss + 0.5 * drho / (self.gm1 * beta_ln) + 0.5 * rho_mean / self.gm1 * (1.0 / bb - 1.0 / ba)
        la = _norm(sum(v * v for v in va)) + torch.sqrt(self.gamma * pa / ra)
        lb = _norm(sum(v * v for v in vb)) + torch.sqrt(self.gamma * pb / rb)
        lam = 0.5 * torch.maximum(la, lb) * self.diss * abs(nrm)
        fm = rho_ln * vm[d] * nrm
        F = [fm - lam * drho]
        for k in range(self.dim):
            F.append(fm * vm[k] + (p_hat * nrm if k == d else 0.0) - lam * (sb[1 + k] - sa[1 + k]))
        F.append(fm * h - lam * diss)
        return F

    def boundary_flux(self, s1, d, sgn, typ, state):
        """Normal flux of a boundary face (src/Integrators/BoundaryConditions):
        interior trace s1, outward normal sgn |n_d| e_d."""
        nrm = sgn * self.area[d]
        if typ in (4, 10, 11):  # slip wall (SlipWallBdrFaceIntegrator.cpp:15-58); no-slip walls derive from it
            rho, vel, p = self.prims(s1)
            vn = sgn * vel[d]
            an = torch.sqrt(self.gamma * p / rho)
            gp1 = 1.0 + self.gamma
            K = self.gm1 / gp1 + 1.0
            S = torch.sqrt(vn * vn + 8.0 / gp1 / rho * p * K)
            ps_pos = p + 0.25 * vn * gp1 * rho * (vn + S)
            X = torch.clamp(1.0 + 0.5 * self.gm1 * vn / an, min=0.0001)
            ps_neg = p * X ** (2.0 * self.gamma / self.gm1)
            ps = torch.where(vn > 0, ps_pos, ps_neg)
            z = torch.zeros_like(ps)
            return [z] + [ps * nrm if k == d else z for k in range(self.dim)] + [z]
        if typ >= 6:
            s2 = self.subsonic_outer_state(s1, d, sgn, typ, [float(x) for x in state])
        elif typ in (1, 3):
            s2 = [torch.full_like(s1[0], float(state[v])) for v in range(self.nv)]
        else:
            s2 = list(s1)
            if typ == 5:
                s2[1 + d] = -s1[1 + d]
        return self.face_flux(s1, s2, d, torch.full_like(s1[0], nrm))

    def subsonic_outer_state(self, s1, d, sgn, typ, prm):
        """Outer states of the subsonic and Riemann-invariant conditions as
        the fixed operator takes them (the interior state as it is)."""
        g, gm1 = self.gamma, self.gm1
        rho = s1[0]
        V = [s1[1 + q] / rho for q in range(self.dim)]
        vv = sum(v * v for v in V)
        msq = sum(s1[1 + q] * s1[1 + q] for q in range(self.dim))
        if typ == 6:   # SubsonicOutflowPBdrFaceIntegrator.cpp:17-31
            return list(s1[:-1]) + [prm[0] / gm1 + 0.5 * rho * vv]
        if typ == 7:   # SubsonicInflowRVBdrFaceIntegrator.cpp:20-50
            r = prm[0]
            uu = sum(prm[1 + q] ** 2 for q in range(self.dim))
            z = torch.zeros_like(rho)
            return ([z + r] + [z + r * prm[1 + q] for q in range(self.dim)]
                    + [s1[-1] - 0.5 * msq / rho + 0.5 * uu * r])
        p = gm1 * (s1[-1] - 0.5 * rho * vv)
        if typ == 8:   # SubsonicInflowPtTtAngBdrFaceIntegrator.cpp:52-80 (2D)
            cp, p0, T0, th = prm[0], prm[1], prm[2], prm[3] * np.pi / 180.0
            dirs = [np.cos(th), np.sin(th)]
            V_sq = torch.clamp(2.0 * cp * T0 * (1.0 - (p / p0) ** (gm1 / g)), min=0.0)
            r2 = g / gm1 * p / (cp * T0 - 0.5 * V_sq)
            return [r2] + [r2 * torch.sqrt(V_sq) * dirs[q] for q in range(self.dim)] + [p / gm1 + 0.5 * r2 * V_sq]
        # typ 9, RiemannInvariantBdrFaceIntegrator.cpp:43-112: prm = rho, v, p
        rho_o, p_o, V_o = prm[0], prm[-1], prm[1:1 + self.dim]
        nq = [sgn if q == d else 0.0 for q in range(self.dim)]
        Vn_i, Vn_o = sgn * V[d], sgn * V_o[d]
        a_o = float(np.sqrt(g * p_o / rho_o))
        a_i = torch.sqrt(g * p / rho)
        sup = abs(Vn_o) >= a_o
        R_minus = torch.where(sup & (Vn_i >= 0), Vn_i - 2.0 * a_i / gm1, Vn_o - 2.0 * a_o / gm1)
        R_plus = torch.where(sup & (Vn_i < 0), Vn_o + 2.0 * a_o / gm1, Vn_i + 2.0 * a_i / gm1)
        Vn_b = 0.5 * (R_plus + R_minus)
        a_b = 0.25 * gm1 * (R_plus - R_minus)
        r2 = torch.where(Vn_i < 0, (a_b * a_b / g * rho_o / p_o) ** (1.0 / gm1) * rho_o,
                         (a_b * a_b / g * rho / p) ** (1.0 / gm1) * rho)
        m2 = [torch.where(Vn_i >= 0, r2 * (V[q] + (Vn_b - Vn_i) * nq[q]), r2 * (V_o[q] + (Vn_b - Vn_o) * nq[q]))
              for q in range(self.dim)]
        p_b = a_b * a_b * r2 / g
        return [r2] + m2 + [0.5 * sum(m * m for m in m2) / r2 + p_b / gm1]

    def entropy_vars(self, s):
        rho, vel, p = self.prims(s)
        v_sq = 0.5 * sum(v * v for v in vel)
        beta = rho / p
        sent = torch.log(p) - self.gamma * torch.log(rho)
        w0 = (self.gamma - sent) / self.gm1 - beta * v_sq
        return [w0] + [beta * v for v in vel] + [-beta]

    def entgrad_to_primgrad(self, s, g):
        rho = s[0]
        vel = [s[1 + k] / rho for k in range(self.dim)]
        v_sq = 0.5 * sum(v * v for v in vel)
        p = self.gm1 * (s[self.dim + 1] - rho * v_sq)
        KE = v_sq * rho
        gl = g[self.dim + 1]
        o = [None] * self.nv
        acc = 0.0
        for k in range(self.dim):
            o[1 + k] = p / rho * (g[1 + k] + vel[k] * gl)
            acc = acc + s[1 + k] * o[1 + k]
        o[0] = rho * g[0] - gl * (KE - p / self.gm1) + rho / p * acc
        o[self.dim + 1] = p / rho * (o[0] + p * gl)
        return o

    def viscous_cols(self, s, dq):
        """Viscous flux columns: cols[d][i], i = 0..dim (momentum rows, energy).
        dq[d][v] = primitive gradient of variable v along x_d."""
        rho, vel, p = self.prims(s)
        mu, lk = self.mu, self.mu * self.gamma / self.Pr
        div = sum(dq[k][1 + k] for k in range(self.dim))
        cols = []
        for d in range(self.dim):
            tau = []
            for i in range(self.dim):
                if i == d:
                    tau.append(mu * (2.0 * dq[d][1 + i] - (2.0 / 3.0) * div))
                else:
                    tau.append(mu * (dq[d][1 + i] + dq[i][1 + d]))
            e = sum(vel[i] * tau[i] for i in range(self.dim))
            cv_dT = (dq[d][self.dim + 1] - p / rho * dq[d][0]) / (self.gm1 * rho)
            cols.append(tau + [e + lk * cv_dT])
        return cols

    # ---- helpers on element fields ----
    def line_apply(self, M, f, d):
        """(M f) along direction d of a field [.., ne, (k,) j, i]: out[..p..] = sum_l M[p, l] f[..l..]."""
        ax = f.dim() - 1 - d
        f2 = f.movedim(ax, -1)
        out = torch.einsum("pl,...l->...p", M, f2)
        return out.movedim(-1, ax)

    def trace(self, f, d, side):
        """Face trace of field f ([..., ne, (k,) j, i]) at position 0 / N along d."""
        ax = f.dim() - 1 - d
        return f.select(ax, self.N if side else 0)

    def add_trace(self, f, d, side, val):
        ax = f.dim() - 1 - d
        idx = [slice(None)] * f.dim()
        idx[ax] = self.N if side else 0
        add = torch.zeros_like(f)
        add[tuple(idx)] = val
        return f + add

    # ---- operator ----
    def alpha(self, s):
        if not self.blending:
            return torch.zeros(self.ne, dtype=s[0].dtype)
        rho, vel, p = self.prims(s)
        q = rho * p  # [ne, ...]
        m = q
        for d in range(self.dim):
            ax = m.dim() - 1 - d
            m = torch.einsum("kl,...l->...k", self.Vinv, m.movedim(ax, -1)).movedim(-1, ax)
        m2 = m * m
        red = tuple(range(1, m.dim()))
        mm = m2.sum(red)
        m1 = (m2 * (self.maxdeg <= self.N - 1)).sum(red)
        mz = (m2 * (self.maxdeg <= self.N - 2)).sum(red)
        eta = torch.maximum(1.0 - m1 / mm, 1.0 - mz / m1)
        a = 1.0 / (1.0 + torch.exp(-SHARPNESS * (eta - self.T) / self.T))
        a = torch.where(a < self.alpha_min, torch.zeros_like(a), a)
        a = torch.where(a > 1.0 - self.alpha_min, torch.ones_like(a), a)
        return torch.minimum(a, torch.full_like(a, self.alpha_max))

    def ec_volume(self, s):
        """sum_d sum_m Dhat2(pos, m) F#_d(u_pos, u_m), diagonal excluded: [nv, ne, ...]."""
        out = torch.zeros_like(s)
        eye = torch.eye(self.Np, dtype=torch.bool)
        for d in range(self.dim):
            ax = s.dim() - 1 - d
            sl = s.movedim(ax, -1)  # [nv, ne, ..., Np]
            sa = [sl[v].unsqueeze(-1) for v in range(self.nv)]  # [..., Np(i), 1]
            sb = [sl[v].unsqueeze(-2) for v in range(self.nv)]  # [..., 1, Np(m)]
            sa = [x.expand(*x.shape[:-1], self.Np) for x in sa]
            sb = [x.expand(*x.shape[:-2], self.Np, self.Np) for x in sb]
            F = self.volume_flux(sa, sb, d, self.adj[d])
            res = []
            for v in range(self.nv):
                Fv = torch.where(eye, torch.zeros_like(F[v]), F[v])
                res.append(torch.einsum("im,...im->...i", self.Dhat2, Fv))
            out = out + torch.stack(res).movedim(-1, ax)
        return out

    def fv_volume(self, s):
        """Subcell finite-volume update (before the alpha factor)."""
        out = torch.zeros_like(s)
        w = torch.tensor(self.w)
        for d in range(self.dim):
            ax = s.dim() - 1 - d
            sl = s.movedim(ax, -1)
            sa = [sl[v][..., :-1] for v in range(self.nv)]
            sb = [sl[v][..., 1:] for v in range(self.nv)]
            F = self.face_flux(sa, sb, d, self.snor[d][1:-1])
            res = []
            for v in range(self.nv):
                z = torch.zeros_like(F[v][..., :1])
                Fl = torch.cat([z, F[v]], -1)
                Fr = torch.cat([F[v], z], -1)
                res.append((Fl - Fr) / (self.J * w))
            out = out + torch.stack(res).movedim(-1, ax)
        return out

    def lifting(self, s):
        """Primitive gradients dq[d][v] as fields [ne, ...]."""
        W = torch.stack(self.entropy_vars(s))  # [nv, ne, ...]
        g = [self.line_apply(self.D, W, d) * (self.adj[d] / self.J) for d in range(self.dim)]
        for d in range(self.dim):
            wa = self.trace(W, d, 1)  # a's +d face
            nb = self.nbr[:, 2 * d + 1]
            wb = self.trace(W, d, 0)[:, nb]  # neighbour's -d face
            a_is_1 = (torch.arange(self.ne) <= nb).to(W.dtype)
            sign = 2.0 * a_is_1 - 1.0
            sh = (self.ne,) + (1,) * (self.dim - 1)
            nrm = sign.reshape(sh) * self.area[d]
            w1 = torch.where(a_is_1.reshape(sh).bool(), wa, wb)
            w2 = torch.where(a_is_1.reshape(sh).bool(), wb, wa)
            fval = self.face_scale * ((0.5 * (w2 - w1)) * nrm)  # [nv, ne, face nodes]
            # added to the a side (pos N) and to the neighbour b (pos 0)
            g[d] = self.add_trace(g[d], d, 1, fval)
            add_b = torch.zeros_like(fval).index_add(1, nb, fval)
            g[d] = self.add_trace(g[d], d, 0, add_b)
        dq = []
        for d in range(self.dim):
            dq.append(self.entgrad_to_primgrad(s, [g[d][v] for v in range(self.nv)]))
        return dq  # dq[d][v]: [ne, ...]

    def rhs(self, u):
        s = self.shape(u)
        sl = [s[v] for v in range(self.nv)]
        alpha = self.alpha(sl)
        ash = (self.ne,) + (1,) * self.dim
        a = alpha.reshape(ash)
        out = -(1.0 - a) * self.ec_volume(s) if self.blending else -self.ec_volume(s)
        if self.parabolic:
            dq = self.lifting(sl)
            cols = self.viscous_cols(sl, dq)  # cols[d][i]: [ne, ...]
            dv = []
            for i in range(self.dim + 1):
                acc = 0.0
                for d in range(self.dim):
                    acc = acc + self.line_apply(self.Dhat, (cols[d][i] * self.adj[d]).unsqueeze(0), d)[0]
                dv.append(acc)
            out = out + torch.stack([torch.zeros_like(dv[0])] + dv)
        out = out / self.J
        if self.blending:
            out = out + a * self.fv_volume(s)
        # faces (boundary faces: a negative neighbour entry -1 - b)
        for d in range(self.dim):
            nb_raw = self.nbr[:, 2 * d + 1]
            inner = nb_raw >= 0
            nb = torch.where(inner, nb_raw, torch.arange(self.ne))
            sa = self.trace(s, d, 1)
            sb = self.trace(s, d, 0)[:, nb]
            a1 = (torch.arange(self.ne) <= nb)
            sh = (self.ne,) + (1,) * (self.dim - 1)
            m1 = a1.reshape(sh)
            s1 = [torch.where(m1, sa[v], sb[v]) for v in range(self.nv)]
            s2 = [torch.where(m1, sb[v], sa[v]) for v in range(self.nv)]
            nrm = (2.0 * a1.to(u.dtype) - 1.0).reshape(sh) * self.area[d]
            F = self.face_flux(s1, s2, d, nrm)
            dU1 = [-f for f in F]
            dU2 = list(F)
            if self.parabolic:
                ca = [self.trace(cols[d][i], d - 0, 1) for i in range(self.dim + 1)]
                cb = [self.trace(cols[d][i], d, 0)[nb] for i in range(self.dim + 1)]
                for i in range(self.dim + 1):
                    c1 = torch.where(m1, ca[i], cb[i])
                    c2 = torch.where(m1, cb[i], ca[i])
                    fn = (0.5 * (c1 + c2)) * nrm
                    dU1[1 + i] = dU1[1 + i] + fn
                    dU2[1 + i] = dU2[1 + i] - fn
            # element a (= e) gets dU1 when it is element 1, else dU2
            mi = inner.reshape(sh)
            ca_ = torch.stack([torch.where(m1, dU1[v], dU2[v]) for v in range(self.nv)]) * self.face_scale
            cb_ = torch.stack([torch.where(m1, dU2[v], dU1[v]) for v in range(self.nv)]) * self.face_scale
            ca_ = torch.where(mi, ca_, torch.zeros_like(ca_))
            cb_ = torch.where(mi, cb_, torch.zeros_like(cb_))
            out = self.add_trace(out, d, 1, ca_)
            add_b = torch.zeros_like(cb_).index_add(1, nb, cb_)
            out = self.add_trace(out, d, 0, add_b)
            for side in (0, 1):
                nbs = self.nbr[:, 2 * d + side]
                for b, (typ, state) in self.bcs.items():
                    mb = (nbs == -1 - b).reshape(sh)
                    if not bool(mb.any()):
                        continue
                    s1 = [self.trace(s[v], d, side) for v in range(self.nv)]
                    F = self.boundary_flux(s1, d, 1.0 if side else -1.0, typ, state)
                    add = torch.stack([torch.where(mb, -F[v], torch.zeros_like(F[v])) for v in range(self.nv)])
                    out = self.add_trace(out, d, side, add * self.face_scale)
        return out.reshape(-1)

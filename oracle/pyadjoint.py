"""TEST INFRASTRUCTURE ONLY: a numpy restatement of the PLRC step in the plane
layout of include/mpulse_b200.h (interior x/y with periodic wraps, z planes
0..nz+1) and of its discrete adjoint, used to check mp_adjoint.

MPulse has no adjoint; what is restated here is the transpose of its step as
the oracle computes it (fdtd_plrc.t:127-168; plrcStepD fdtd_plrc.cpp:94-261,
:304-427; plrcStepB :263-293; CPML cpml_border.cpp:398-425, :499-527), with the
per-cell design parameters of mp_config.design_box.  The coefficients (kappa
lines, CPML b/c lines, PLRC recursion constants) are taken from the C oracle so
that both use the same numbers.

State of one step: E[3], B[3], psi[pole][3] (complex), psiE[layer][2],
psiH[layer][2], all full plane-layout arrays (zero outside their support).
"""
from __future__ import annotations

import numpy as np

from mpulse_b200 import abi
from oracle.pyoracle import OracleSim

# component fed by psi0 / psi1 of a CPML layer along dim (cpml_border.cpp:357-386)
_COMP = {0: (1, 2), 1: (2, 0), 2: (0, 1)}


def _up(a):
    """a[k + 1] at k (zero at the top plane)."""
    out = np.zeros_like(a)
    out[:-1] = a[1:]
    return out


def _down(a):
    """a[k - 1] at k (zero at plane 0)."""
    out = np.zeros_like(a)
    out[1:] = a[:-1]
    return out


def _xm(a):
    return np.roll(a, 1, axis=2)   # a[i - 1]


def _xp(a):
    return np.roll(a, -1, axis=2)  # a[i + 1]


def _ym(a):
    return np.roll(a, 1, axis=1)


def _yp(a):
    return np.roll(a, -1, axis=1)


class Model:
    def __init__(self, cfg: abi.Config):
        if cfg.solver not in (abi.MP_SOLVER_PLRC_LIN, abi.MP_SOLVER_PLRC_NONLIN):
            raise ValueError("PLRC solvers only")
        if cfg.boundary != abi.MP_BOUNDARY_XY_PERIODIC:
            raise ValueError("xy-periodic boundary only")
        self.cfg = cfg
        o = OracleSim(cfg)
        nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
        self.shape = (nz + 2, ny, nx)
        self.dt = cfg.dt
        self.nonlin = cfg.solver == abi.MP_SOLVER_PLRC_NONLIN
        kE = [o.kappa(0, d) for d in range(3)]
        kH = [o.kappa(1, d) for d in range(3)]
        sp = (cfg.dx, cfg.dy, cfg.dz)
        # 1 / (kappa delta) broadcast over the plane layout
        self.ikE = (1 / (kE[0][1:nx + 1] * sp[0]))[None, None, :], (1 / (kE[1][1:ny + 1] * sp[1]))[None, :, None], \
            (1 / (kE[2] * sp[2]))[:, None, None]
        self.ikH = (1 / (kH[0][1:nx + 1] * sp[0]))[None, None, :], (1 / (kH[1][1:ny + 1] * sp[1]))[None, :, None], \
            (1 / (kH[2] * sp[2]))[:, None, None]
        self.layers = {0: self._layers(o, 0), 1: self._layers(o, 1)}
        pc = o.plrc_coefficients()
        active = [n for n in range(3) if cfg.poles[n].eps != 0]
        self.D = [pc["dchi0"][n] - pc["dxi0"][n] for n in active]
        self.Xi = [pc["dxi0"][n] for n in active]
        self.Cr = [pc["crec"][n] for n in active]
        self.sumChi0, self.sumXi0 = pc["sumChi0"], pc["sumXi0"]
        o.close()
        # masks: E cells (planes 1..nz), medium, B cells (planes 0..nz)
        k = np.arange(nz + 2)[:, None, None]
        self.ecell = np.broadcast_to((k >= 1) & (k <= nz), self.shape)
        self.bcell = np.broadcast_to(k <= nz, self.shape)
        self.med = np.broadcast_to((k >= cfg.medium_z0) & (k <= cfg.medium_z1), self.shape) & self.ecell
        # per-cell parameters (eps, Delta-eps factor, chi factor)
        self.eps = np.where(self.med, cfg.eps, cfg.eps_bg)
        self.s = np.ones(self.shape)
        self.u = np.ones(self.shape)
        b = cfg.design_box
        self.dsl = None
        if b[0] <= b[1]:
            self.dsl = (slice(b[4], b[5] + 1), slice(b[2] - 1, b[3]), slice(b[0] - 1, b[1]))

    def _layers(self, o, isH):
        nx, ny, nz = self.cfg.nx, self.cfg.ny, self.cfg.nz
        out = []
        for (_dir, dim, lo, hi, b, c, delta) in o.cpml_layers(isH):
            bf = np.zeros(self.shape)
            cf = np.zeros(self.shape)
            mask = np.zeros(self.shape, dtype=bool)
            # plane-layout ranges of the layer box (x, y ghosts dropped)
            xs = [i - 1 for i in range(lo[0], hi[0] + 1) if 1 <= i <= nx]
            ys = [j - 1 for j in range(lo[1], hi[1] + 1) if 1 <= j <= ny]
            zs = [k for k in range(lo[2], hi[2] + 1) if 0 <= k <= nz + 1]
            for k in zs:
                for j in ys:
                    for i in xs:
                        pos = (i + 1, j + 1, k)[dim]
                        mask[k, j, i] = True
                        bf[k, j, i] = b[pos - lo[dim]]
                        cf[k, j, i] = c[pos - lo[dim]] / delta
            out.append((dim, mask, bf, cf))
        return out

    def set_design(self, eps=None, dscale=None, chiscale=None):
        if self.dsl is None:
            raise ValueError("no design box")
        for arr, val in ((self.eps, eps), (self.s, dscale), (self.u, chiscale)):
            if val is not None:
                arr[self.dsl] = np.asarray(val).reshape(arr[self.dsl].shape)

    # ------------------------------------------------------------------
    def zero_state(self):
        z = lambda: np.zeros(self.shape)  # noqa: E731
        return {
            "E": [z() for _ in range(3)], "B": [z() for _ in range(3)],
            "psi": [[np.zeros(self.shape, complex) for _ in range(3)] for _ in self.D],
            "psiE": [[z(), z()] for _ in self.layers[0]], "psiH": [[z(), z()] for _ in self.layers[1]],
        }

    def _coeffs(self):
        s = self.s * self.med
        numer = self.eps - s * self.sumXi0
        denom = self.eps + s * (self.sumChi0 - self.sumXi0)
        A = np.where(self.med, self.u * self.cfg.chi, 0.0) / denom if self.nonlin else np.zeros(self.shape)
        return s, numer, denom, A

    def step(self, st, J=None, M=None):
        """One forward step in place (sources as given full-array J / M, or none)."""
        dt = self.dt
        E, B = st["E"], st["B"]
        ikx, iky, ikz = self.ikE
        # E side
        cur = [np.zeros(self.shape) for _ in range(3)] if J is None else [j.copy() for j in J]
        for l, (dim, mask, bf, cf) in enumerate(self.layers[0]):
            c0, c1 = _COMP[dim]
            if dim == 2:
                d0, d1 = -(B[1] - _down(B[1])), B[0] - _down(B[0])
            elif dim == 0:
                d0, d1 = -(B[2] - _xm(B[2])), B[1] - _xm(B[1])
            else:
                d0, d1 = -(B[0] - _ym(B[0])), B[2] - _ym(B[2])
            p = st["psiE"][l]
            p[0] = np.where(mask, bf * p[0] + cf * d0, 0.0)
            p[1] = np.where(mask, bf * p[1] + cf * d1, 0.0)
            cur[c0] = cur[c0] + p[0]
            cur[c1] = cur[c1] + p[1]
        cb = [(B[2] - _ym(B[2])) * iky - (B[1] - _down(B[1])) * ikz,
              (B[0] - _down(B[0])) * ikz - (B[2] - _xm(B[2])) * ikx,
              (B[1] - _xm(B[1])) * ikx - (B[0] - _ym(B[0])) * iky]
        s, numer, denom, A = self._coeffs()
        P = [np.zeros(self.shape) for _ in range(3)]
        for n in range(len(self.D)):
            for c in range(3):
                pt = s * self.D[n] * E[c] + st["psi"][n][c]
                P[c] = P[c] + np.where(self.med, pt.real, 0.0)
                st["psi"][n][c] = np.where(self.med, s * self.Xi[n] * E[c] + self.Cr[n] * pt, 0.0)
        E2 = E[0] ** 2 + E[1] ** 2 + E[2] ** 2
        chi = np.where(self.med, self.u * self.cfg.chi, 0.0) if self.nonlin else 0.0
        X = [(numer + chi * E2) * E[c] + dt * (cb[c] + cur[c]) + P[c] for c in range(3)]
        cvec = [X[c] / denom for c in range(3)]
        if self.nonlin:
            C = np.sqrt(cvec[0] ** 2 + cvec[1] ** 2 + cvec[2] ** 2)
            r = np.sqrt(E2)
            for _ in range(200):
                r = (2 * A * r ** 3 + C) / (3 * A * r ** 2 + 1)
            scale = np.where(C > 0, r / np.where(C > 0, C, 1), 0.0)
            new = [cvec[c] * scale for c in range(3)]
        else:
            new = cvec
        for c in range(3):
            E[c] = np.where(self.ecell, new[c], E[c])
        # H side
        ikx, iky, ikz = self.ikH
        mag = [np.zeros(self.shape) for _ in range(3)] if M is None else [m.copy() for m in M]
        for l, (dim, mask, bf, cf) in enumerate(self.layers[1]):
            c0, c1 = _COMP[dim]
            if dim == 2:
                d0, d1 = _up(E[1]) - E[1], -(_up(E[0]) - E[0])
            elif dim == 0:
                d0, d1 = _xp(E[2]) - E[2], -(_xp(E[1]) - E[1])
            else:
                d0, d1 = _yp(E[0]) - E[0], -(_yp(E[2]) - E[2])
            p = st["psiH"][l]
            p[0] = np.where(mask, bf * p[0] + cf * d0, 0.0)
            p[1] = np.where(mask, bf * p[1] + cf * d1, 0.0)
            mag[c0] = mag[c0] + p[0]
            mag[c1] = mag[c1] + p[1]
        cE = [(_up(E[1]) - E[1]) * ikz - (_yp(E[2]) - E[2]) * iky,
              (_xp(E[2]) - E[2]) * ikx - (_up(E[0]) - E[0]) * ikz,
              (_yp(E[0]) - E[0]) * iky - (_xp(E[1]) - E[1]) * ikx]
        for c in range(3):
            B[c] = np.where(self.bcell, B[c] + dt * (cE[c] + mag[c]), B[c])
        return st

    # ------------------------------------------------------------------
    def reverse_step(self, En, En1, lam, grads=None):
        """Adjoint of one step.  En, En1: E before / after the step.  lam holds
        the adjoint of the state after the step (keys of zero_state) and is
        replaced by the adjoint of the state before it.  grads (dict of
        full-size arrays eps, s, u) accumulates dJ/d parameters."""
        dt = self.dt
        Eb, Bb = lam["E"], lam["B"]
        # ---- B half: B' = B + dt (curl_H E' + M), psiH' = b psiH + c d(E')
        Q = [np.where(self.bcell, dt * Bb[c], 0.0) for c in range(3)]
        ikx, iky, ikz = self.ikH
        Et = [Eb[c].copy() for c in range(3)]
        # curl_H transposed
        w = Q[0]  # Bx: +ey(k+1) ikz, -ez(j+1) iky
        Et[1] += _down(ikz * w) - ikz * w
        Et[2] += -_ym(iky * w) + iky * w
        w = Q[1]  # By: +ez(i+1) ikx, -ex(k+1) ikz
        Et[2] += _xm(ikx * w) - ikx * w
        Et[0] += -_down(ikz * w) + ikz * w
        w = Q[2]  # Bz: +ex(j+1) iky, -ey(i+1) ikx
        Et[0] += _ym(iky * w) - iky * w
        Et[1] += -_xm(ikx * w) + ikx * w
        for l, (dim, mask, bf, cf) in enumerate(self.layers[1]):
            c0, c1 = _COMP[dim]
            U0 = np.where(mask, lam["psiH"][l][0] + Q[c0], 0.0)
            U1 = np.where(mask, lam["psiH"][l][1] + Q[c1], 0.0)
            W0, W1 = cf * U0, cf * U1
            if dim == 2:
                Et[1] += _down(W0) - W0
                Et[0] += W1 - _down(W1)
            elif dim == 0:
                Et[2] += _xm(W0) - W0
                Et[1] += W1 - _xm(W1)
            else:
                Et[0] += _ym(W0) - W0
                Et[2] += W1 - _ym(W1)
            lam["psiH"][l] = [bf * U0, bf * U1]
        # ---- E half
        s, numer, denom, A = self._coeffs()
        E2 = En[0] ** 2 + En[1] ** 2 + En[2] ** 2
        if self.nonlin:
            r2 = En1[0] ** 2 + En1[1] ** 2 + En1[2] ** 2
            r = np.sqrt(r2)
            safe = np.where(r > 0, r, 1.0)
            ehat = [np.where(r > 0, En1[c] / safe, 0.0) for c in range(3)]
            alpha = 1 / (1 + A * r2)
            beta = 1 / (1 + 3 * A * r2)
            ea = ehat[0] * Et[0] + ehat[1] * Et[1] + ehat[2] * Et[2]
            cbar = [alpha * (Et[c] - ehat[c] * ea) + beta * ehat[c] * ea for c in range(3)]
            Abar = -ea * r * r2 * beta
            cvec = [En1[c] * (1 + A * r2) for c in range(3)]
            chi = np.where(self.med, self.u * self.cfg.chi, 0.0)
        else:
            cbar = Et
            Abar = np.zeros(self.shape)
            cvec = En1
            chi = np.zeros(self.shape)
        g = [np.where(self.ecell, cbar[c] / denom, 0.0) for c in range(3)]
        newE = [np.zeros(self.shape) for _ in range(3)]
        Eg = En[0] * g[0] + En[1] * g[1] + En[2] * g[2]
        for c in range(3):
            newE[c] = (numer + chi * E2) * g[c] + 2 * chi * En[c] * Eg
        gs = np.zeros(self.shape)
        SD = sum(d.real for d in self.D) if self.D else 0.0
        for n in range(len(self.D)):
            for c in range(3):
                pb = lam["psi"][n][c]
                pt_bar = np.conj(self.Cr[n]) * pb + g[c]
                a1 = s * self.D[n]
                a2 = s * self.Xi[n]
                newE[c] += np.where(self.med, (np.conj(a1) * pt_bar).real + (np.conj(a2) * pb).real, 0.0)
                gs += np.where(self.med, (np.conj(pb) * (self.Xi[n] * En[c] + self.Cr[n] * self.D[n] * En[c])).real,
                               0.0)
                lam["psi"][n][c] = np.where(self.med, pt_bar, 0.0)
        if grads is not None:
            dD = self.sumChi0 - self.sumXi0
            dXs = [(-self.sumXi0 + SD) * En[c] for c in range(3)]
            ge = sum(g[c] * (En[c] - cvec[c]) for c in range(3)) - Abar * A / denom
            gs += sum(g[c] * (dXs[c] - cvec[c] * dD) for c in range(3)) - Abar * A * dD / denom
            gu = (sum(g[c] * self.cfg.chi * E2 * En[c] for c in range(3)) + Abar * self.cfg.chi / denom
                  if self.nonlin else np.zeros(self.shape))
            grads["eps"] += np.where(self.med, ge, 0.0)
            grads["s"] += np.where(self.med, gs, 0.0)
            grads["u"] += np.where(self.med, gu, 0.0)
        # background cells: E' = (eps_bg E + dt(...)) / eps_bg
        for c in range(3):
            newE[c] = np.where(self.med, newE[c], np.where(self.ecell, self.eps * g[c], 0.0))
        # curl_E transposed into B
        G = [dt * g[c] for c in range(3)]
        ikx, iky, ikz = self.ikE
        Bn = [Bb[c].copy() for c in range(3)]
        w = G[0]  # cbx = (bz - bz[j-1]) iky - (by - by[k-1]) ikz
        Bn[2] += iky * w - _yp(iky * w)
        Bn[1] += -ikz * w + _up(ikz * w)
        w = G[1]  # cby = (bx - bx[k-1]) ikz - (bz - bz[i-1]) ikx
        Bn[0] += ikz * w - _up(ikz * w)
        Bn[2] += -ikx * w + _xp(ikx * w)
        w = G[2]  # cbz = (by - by[i-1]) ikx - (bx - bx[j-1]) iky
        Bn[1] += ikx * w - _xp(ikx * w)
        Bn[0] += -iky * w + _yp(iky * w)
        for l, (dim, mask, bf, cf) in enumerate(self.layers[0]):
            c0, c1 = _COMP[dim]
            V0 = np.where(mask & self.ecell, lam["psiE"][l][0] + G[c0], 0.0)
            V1 = np.where(mask & self.ecell, lam["psiE"][l][1] + G[c1], 0.0)
            W0, W1 = cf * V0, cf * V1
            if dim == 2:
                Bn[1] += -W0 + _up(W0)
                Bn[0] += W1 - _up(W1)
            elif dim == 0:
                Bn[2] += -W0 + _xp(W0)
                Bn[1] += W1 - _xp(W1)
            else:
                Bn[0] += -W0 + _yp(W0)
                Bn[2] += W1 - _yp(W1)
            lam["psiE"][l] = [np.where(mask, bf * V0, 0.0), np.where(mask, bf * V1, 0.0)]
        for c in range(3):
            Eb[c] = np.where(self.ecell, newE[c], 0.0)
            Bb[c] = np.where(self.bcell, Bn[c], 0.0)
        return lam


def objective_grad(cfg: abi.Config, adj: abi.AdjointConfig, E, B):
    """dJ/dE, dJ/dB of one step's term of mp_objective (plane layout)."""
    gE = [np.zeros(cfg.field_shape()) for _ in range(3)]
    gB = [np.zeros(cfg.field_shape()) for _ in range(3)]
    b = adj.box
    if adj.kind == abi.MP_OBJ_E2_BOX:
        sl = (slice(b[4], b[5] + 1), slice(b[2] - 1, b[3]), slice(b[0] - 1, b[1]))
        for c in range(3):
            gE[c][sl] = 2 * cfg.dt * E[c][sl]
    else:
        sl = (b[4], slice(b[2] - 1, b[3]), slice(b[0] - 1, b[1]))
        f = cfg.dt * cfg.dx * cfg.dy
        gE[0][sl] = f * B[1][sl]
        gE[1][sl] = -f * B[0][sl]
        gB[0][sl] = -f * E[1][sl]
        gB[1][sl] = f * E[0][sl]
    return gE, gB


def adjoint_gradient(cfg: abi.Config, adj: abi.AdjointConfig, init: dict, design: dict):
    """J and dJ/d(DesignEps, DesignDepsScale, DesignChiScale) with the C oracle
    as the forward (sources included) and Model.reverse_step backwards."""
    o = OracleSim(cfg)
    for n, v in init.items():
        o.upload(n, v)
    for n, v in design.items():
        o.upload_design(n, v)
    names = abi.FIELD_NAMES
    hist = [[o.download(n) for n in names]]
    J = 0.0
    for _ in range(adj.steps):
        assert o.step(1) == abi.MP_OK
        f = [o.download(n) for n in names]
        hist.append(f)
    o.close()
    m = Model(cfg)
    m.set_design(design.get("DesignEps"), design.get("DesignDepsScale"), design.get("DesignChiScale"))
    for n in range(1, adj.steps + 1):
        gE, _ = objective_grad(cfg, adj, hist[n][:3], hist[n][3:])
        if adj.kind == abi.MP_OBJ_E2_BOX:
            J += 0.5 * sum(float(np.sum(gE[c] * hist[n][c])) for c in range(3))
        else:
            b = adj.box
            sl = (b[4], slice(b[2] - 1, b[3]), slice(b[0] - 1, b[1]))
            E, B = hist[n][:3], hist[n][3:]
            J += cfg.dt * cfg.dx * cfg.dy * float(np.sum(E[0][sl] * B[1][sl] - E[1][sl] * B[0][sl]))
    lam = m.zero_state()
    grads = {k: np.zeros(m.shape) for k in ("eps", "s", "u")}
    for n in range(adj.steps - 1, -1, -1):
        gE, gB = objective_grad(cfg, adj, hist[n + 1][:3], hist[n + 1][3:])
        for c in range(3):
            lam["E"][c] += gE[c]
            lam["B"][c] += gB[c]
        m.reverse_step(hist[n][:3], hist[n + 1][:3], lam, grads)
    out = {k: grads[k][m.dsl].copy() for k in grads}
    return J, out

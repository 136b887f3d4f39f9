"""Line-by-line Python transliteration of the reference's hot path, for golden vectors.

Written directly from the Fortran sources (paths relative to the reference project), separately
from oracle/oracle.c, with Python floats (IEEE binary64, no contraction) and the reference's
library calls through scipy: LAPACK dgeev (utility/SMOD_eigenvalue_problem.f90:53-66, workspace
query first) and BLAS dgemv (utility/SMOD_matrix_operations.f90:108-113).  It is slow and only
meant for tiny grids: make_golden.py runs it once and commits the results.

Arrays keep the reference's index ranges through the helper class FArr (lower bound -1).
"""
from __future__ import annotations

import math

import numpy as np
from scipy.linalg import blas, lapack

UD = 1e-10  # constant/MOD_constants.f90:18


class FArr:
    """Fortran-style array with arbitrary lower bounds (column-major index order kept)."""

    def __init__(self, *bounds):
        self.lo = [b[0] for b in bounds]
        self.a = np.zeros([b[1] - b[0] + 1 for b in bounds], dtype=np.float64)

    def _k(self, idx):
        return tuple(i - l for i, l in zip(idx, self.lo))

    def __getitem__(self, idx):
        return float(self.a[self._k(idx)])

    def __setitem__(self, idx, v):
        self.a[self._k(idx)] = v


def getjakobi(ixy, q, g):
    """examples/2D_dam_break/cartesian/SMOD_jakobian.f90:43-53 (jakobi(row, col))."""
    h, hu, hv = q
    J = np.zeros((3, 3), dtype=np.float64, order="F")
    if ixy == 1:
        J[0, :] = [0.0, 1.0, 0.0]
        J[1, :] = [-(hu * hu / (h * h)) + g * h, 2.0 * hu / h, 0.0]
        J[2, :] = [-(hu * hv / (h * h)), hv / h, hu / h]
    else:
        J[0, :] = [0.0, 0.0, 1.0]
        J[1, :] = [-(hu * hv / (h * h)), hv / h, hu / h]
        J[2, :] = [-(hv * hv / (h * h)) + g * h, 0.0, 2.0 * hv / h]
    if np.isnan(J).any():
        raise FloatingPointError("isnan in jakobi")
    return J


def eigen_real(J):
    """calculateEigenSolution: dgeev('N', 'V') after a workspace query."""
    lw = lapack.dgeev_lwork(3, compute_vl=0, compute_vr=1)
    lwork = int(lw[0])
    wr, wi, vl, vr, info = lapack.dgeev(np.asfortranarray(J.copy()), compute_vl=0, compute_vr=1, lwork=lwork)
    if (wi > UD).any():
        raise FloatingPointError("complex eigenvalue")
    return [float(x) for x in wr]


def matvec(J, v):
    """matrix_vector_product: dgemv('N', 3, 3, 1.0, J, 3, v, 1, 0.0, b, 1)."""
    return [float(x) for x in blas.dgemv(1.0, np.asfortranarray(J), np.asarray(v, dtype=np.float64), beta=0.0)]


def hll(ixy, qL, qR, g):
    """solver/SMOD_approximate_Riemann_solvers.f90:169-224 for one interface."""
    JL = getjakobi(ixy, qL, g)
    JR = getjakobi(ixy, qR, g)
    lL = eigen_real(JL)
    lR = eigen_real(JR)
    s2 = max([abs(x) for x in lL] + [abs(x) for x in lR])
    s1 = -s2
    lam = [s1, s2]
    if abs(lam[0]) > UD and abs(lam[1]) > UD:
        fL = matvec(JL, qL)
        fR = matvec(JR, qR)
        qi = [(fR[k] - fL[k] - s2 * qR[k] + s1 * qL[k]) / (UD + s1 - s2) for k in range(3)]
        W1 = [qi[k] - qL[k] for k in range(3)]
        W2 = [qR[k] - qi[k] for k in range(3)]
    else:
        lam = [0.0, 0.0]
        W1 = [0.0, 0.0, 0.0]
        W2 = [0.0, 0.0, 0.0]
    return lam, W1, W2


def phi(method, r):
    """solver/MOD_flux_correction.f90:101-112."""
    if method == 1:
        return max(0.0, min(1.0, r))
    if method == 2:
        return max(0.0, min(1.0, 2.0 * r), min(2.0, r))
    if method == 3:
        return (r + abs(r)) / (1.0 + abs(r))
    if method == 4:
        return max(0.0, min((1.0 + r) / 2.0, 2.0, 2.0 * r))
    raise ValueError("invalid limiter choice")


class Solver:
    """Single-rank main loop of main.f90 with the dam-break equation module."""

    def __init__(self, p):
        self.p = dict(p)
        mx, my = p["m_xi"], p["m_eta"]
        self.mx, self.my = mx, my
        B = ((-1, mx + 2), (-1, my + 2))
        self.vars = FArr((1, 3), *B)
        self.lam = FArr((1, 2), *B)
        self.waves = FArr((1, 3), (1, 2), *B)
        self.Am = FArr((1, 3), *B)
        self.Ap = FArr((1, 3), *B)
        self.f = FArr((1, 3), *B)
        self.wnl = FArr((1, 2), *B)
        self.wnr = FArr((1, 2), *B)
        self.kappa = FArr(*B)
        self.lrx = FArr(*B)
        self.lre = FArr(*B)
        self.xi = FArr(*B)
        self.eta = FArr(*B)
        self.mesh()
        self.tinit()

    # domain/SMOD_mesh_manipulation.f90
    def mesh(self):
        p = self.p
        self.dxi = (p["xi_max"] - p["xi_min"]) / self.mx
        self.deta = (p["eta_max"] - p["eta_min"]) / self.my
        for j in range(-1, self.my + 3):
            for i in range(-1, self.mx + 3):
                xc = [0.0] * 6
                yc = [0.0] * 6
                xc[1] = p["xi_min"] + (i - 1) * self.dxi
                xc[2] = xc[1] + self.dxi
                xc[3] = xc[2]
                xc[4] = xc[1]
                xc[5] = xc[1]
                yc[1] = p["eta_min"] + (j - 1) * self.deta
                yc[2] = yc[1]
                yc[3] = yc[2] + self.deta
                yc[4] = yc[3]
                yc[5] = yc[1]
                self.xi[i, j] = p["xi_min"] + (i - 1) * self.dxi + self.dxi / 2
                self.eta[i, j] = p["eta_min"] + (j - 1) * self.deta + self.deta / 2
                fdx, fdy = xc[4] - xc[1], yc[4] - yc[1]
                self.lrx[i, j] = math.hypot(fdx, fdy) / self.deta
                fdx, fdy = xc[2] - xc[1], yc[2] - yc[1]
                self.lre[i, j] = math.hypot(fdx, fdy) / self.dxi
                area = 0.0
                for m in range(1, 5):
                    area = area + 0.5 * (yc[m] + yc[m + 1]) * (xc[m] - xc[m + 1])
                self.kappa[i, j] = area / (self.dxi * self.deta)

    # time_control/MOD_time_control.f90
    def tinit(self):
        p = self.p
        self.time = p["t_start"]
        self.tf = p["t_final"]
        self.dt = p["dt_initial"]
        self.dt_prev = p["dt_initial"]
        n = max(p["n_snapshots"], 1)
        si = (self.tf - self.time) / n
        self.snaps = [p["t_start"] + i * si for i in range(1, n + 1)]
        self.snaps[-1] = self.tf
        self.snap_idx = 1
        self.CFL = 0.0
        self.cfl_target = p["cfl"]
        self.shrink = p["shrink"]
        self.growth = p["growth"]
        self.dt_max = p["dt_max"]
        self.dt_min = p["dt_min"]
        self.snap_exc = False

    def update_time(self, valid):
        self.dt_prev = self.dt
        dt_step = self.dt
        if valid:
            cf = self.cfl_target / self.CFL if self.CFL > 0.0 else 1.0
            if cf >= self.growth:
                cf = self.growth
            elif abs(cf - 1.0) <= 0.01:
                cf = 1.0
            dt_step = self.dt_prev * cf
            ts = self.snaps[min(self.snap_idx, len(self.snaps)) - 1]
            if self.time + dt_step > ts:
                dt_step = ts - self.time
                self.snap_exc = True
            else:
                self.snap_exc = False
        else:
            dt_step = 0.25 * self.dt
        if dt_step > self.dt_max:
            dt_step = self.dt_max
        if dt_step < self.dt_min:
            dt_step = self.dt_min
        if valid:
            self.time = self.time + dt_step
        self.dt = dt_step

    def valid(self):
        return self.cfl_target / self.CFL >= self.shrink

    def zero_work(self):
        for a in (self.lam, self.waves, self.Am, self.Ap, self.f, self.wnl, self.wnr):
            a.a[...] = 0.0

    # solver/MOD_solve.f90
    def sweep(self, ixy):
        mx, my, g = self.mx, self.my, self.p["grav"]
        cfl = 0.0
        d = self.dxi if ixy == 1 else self.deta
        if ixy == 1:
            pairs = [(i, j) for j in range(1, my + 1) for i in range(0, mx + 2)]
        else:
            pairs = [(i, j) for i in range(1, mx + 1) for j in range(0, my + 2)]
        for (i, j) in pairs:
            il, jl = (i - 1, j) if ixy == 1 else (i, j - 1)
            qL = [self.vars[me, il, jl] for me in (1, 2, 3)]
            qR = [self.vars[me, i, j] for me in (1, 2, 3)]
            lam, W1, W2 = hll(ixy, qL, qR, g)
            self.lam[1, i, j], self.lam[2, i, j] = lam
            for me in range(3):
                self.waves[me + 1, 1, i, j] = W1[me]
                self.waves[me + 1, 2, i, j] = W2[me]
            for mw in (1, 2):
                cfl = max(cfl, self.lam[mw, i, j] * self.dt / d)
        # split_flux
        for j in range(0, my + 2):
            for i in range(0, mx + 2):
                for mw in (1, 2):
                    s = self.lam[mw, i, j]
                    for me in (1, 2, 3):
                        w = self.waves[me, mw, i, j]
                        mask = 1.0 if s < 0.0 else 0.0
                        self.Am[me, i, j] = self.Am[me, i, j] + mask * s * w
                        self.Ap[me, i, j] = self.Ap[me, i, j] + (1.0 - mask) * s * w
        dtod = self.dt / d
        # integrate_flux_difference
        for j in range(1, my + 1):
            for i in range(1, mx + 1):
                if ixy == 1:
                    ll, lr = self.lrx[i, j], self.lrx[i + 1, j]
                else:
                    ll, lr = self.lre[i, j], self.lre[i, j + 1]
                for me in (1, 2, 3):
                    amr = self.Am[me, i + 1, j] if ixy == 1 else self.Am[me, i, j + 1]
                    self.vars[me, i, j] = self.vars[me, i, j] - dtod / self.kappa[i, j] * (
                        ll * self.Ap[me, i, j] + lr * amr)
        if self.p["higher_order"]:
            self.limiter(ixy)
            # second_order_flux_correction
            if ixy == 1:
                rng = [(i, j) for j in range(1, my + 1) for i in range(0, mx + 2)]
            else:
                rng = [(i, j) for j in range(0, my + 2) for i in range(1, mx + 1)]
            for (i, j) in rng:
                kb = 0.5 * (self.kappa[i - 1, j] + self.kappa[i, j]) if ixy == 1 else \
                    0.5 * (self.kappa[i, j - 1] + self.kappa[i, j])
                for mw in (1, 2):
                    al = abs(self.lam[mw, i, j])
                    for me in (1, 2, 3):
                        self.f[me, i, j] = self.f[me, i, j] + 0.5 * al * (1.0 - al * dtod / kb) * self.waves[me, mw, i, j]
            # integrator_flux_correction_increment
            for j in range(1, my + 1):
                for i in range(1, mx + 1):
                    for me in (1, 2, 3):
                        fr = self.f[me, i + 1, j] if ixy == 1 else self.f[me, i, j + 1]
                        self.vars[me, i, j] = self.vars[me, i, j] - dtod / self.kappa[i, j] * (fr - self.f[me, i, j])
        return cfl

    def limiter(self, ixy):
        if not self.p["use_limiter"]:
            return
        mx, my = self.mx, self.my
        if ixy == 1:
            i = 0
            for j in range(1, my + 1):
                for mw in (1, 2):
                    for me in (1, 2, 3):
                        self.wnr[mw, i, j] = self.wnr[mw, i, j] + self.waves[me, mw, i, j] * self.waves[me, mw, i + 1, j]
        else:
            j = 0
            for i in range(1, mx + 1):
                for mw in (1, 2):
                    for me in (1, 2, 3):
                        self.wnr[mw, i, j] = self.wnr[mw, i, j] + self.waves[me, mw, i, j] * self.waves[me, mw, i, j + 1]
        for j in range(1, my + 1):
            for i in range(1, mx + 1):
                for mw in (1, 2):
                    wn2 = 0.0
                    self.wnl[mw, i, j] = self.wnr[mw, i - 1, j] if ixy == 1 else self.wnr[mw, i, j - 1]
                    self.wnr[mw, i, j] = 0.0
                    ir, jr = (i + 1, j) if ixy == 1 else (i, j + 1)
                    for me in (1, 2, 3):
                        w = self.waves[me, mw, i, j]
                        wn2 = wn2 + w * w  # Fortran expands **2 to a product
                        self.wnr[mw, i, j] = self.wnr[mw, i, j] + self.waves[me, mw, i, j] * self.waves[me, mw, ir, jr]
                    up = self.wnl[mw, i, j] if self.lam[mw, i, j] > 0.0 else self.wnr[mw, i, j]
                    r = up / wn2 if wn2 != 0.0 else math.nan
                    ph = phi(self.p["limiter"], r) if not math.isnan(r) else 0.0
                    if not (abs(wn2) <= UD):
                        for me in (1, 2, 3):
                            self.waves[me, mw, i, j] = ph * self.waves[me, mw, i, j]

    def solve(self):
        cfl = self.sweep(1)
        self.CFL = max(self.CFL, cfl)
        self.zero_work()
        if not self.valid():
            return -1
        cfl = max(cfl, self.sweep(2))
        self.CFL = max(self.CFL, cfl)
        self.zero_work()
        return 1 if self.valid() else -1

    # user_subroutines/SMOD_boundary_conditions.f90 (codes 2 and 3)
    def bc(self):
        mx, my = self.mx, self.my
        b = self.p["bc"]
        for j in range(1, my + 1):
            for i in (-1, 0):
                for me in (1, 2, 3):
                    if b == 2:
                        self.vars[me, i, j] = self.vars[me, 1, j]
                    else:
                        d = (self.vars[me, 2, j] - self.vars[me, 1, j]) / (self.xi[2, j] - self.xi[1, j])
                        self.vars[me, i, j] = self.vars[me, 1, j] + d * (self.xi[i, j] - self.xi[1, j])
            for i in (mx + 1, mx + 2):
                for me in (1, 2, 3):
                    if b == 2:
                        self.vars[me, i, j] = self.vars[me, mx, j]
                    else:
                        d = (self.vars[me, mx, j] - self.vars[me, mx - 1, j]) / (self.xi[mx, j] - self.xi[mx - 1, j])
                        self.vars[me, i, j] = self.vars[me, mx, j] + d * (self.xi[i, j] - self.xi[mx, j])
        for j in (-1, 0):
            for i in range(1, mx + 1):
                for me in (1, 2, 3):
                    if b == 2:
                        self.vars[me, i, j] = self.vars[me, i, 1]
                    else:
                        d = (self.vars[me, i, 2] - self.vars[me, i, 1]) / (self.eta[i, 2] - self.eta[i, 1])
                        self.vars[me, i, j] = self.vars[me, i, 1] + d * (self.eta[i, j] - self.eta[i, 1])
        for j in (my + 1, my + 2):
            for i in range(1, mx + 1):
                for me in (1, 2, 3):
                    if b == 2:
                        self.vars[me, i, j] = self.vars[me, i, my]
                    else:
                        d = (self.vars[me, i, my] - self.vars[me, i, my - 1]) / (self.eta[i, my] - self.eta[i, my - 1])
                        self.vars[me, i, j] = self.vars[me, i, my] + d * (self.eta[i, j] - self.eta[i, my])

    def run(self, max_attempts):
        """main.f90:193-283; returns (dt used, ierr) per attempt."""
        log = []
        while self.time < self.tf and len(log) < max_attempts:
            old = self.vars.a.copy()
            dt_used = self.dt
            ierr = self.solve()
            if ierr < 0:
                self.update_time(False)
                self.vars.a[...] = old
                self.CFL = 0.0
            else:
                self.bc()
                self.update_time(True)
                if self.time >= self.snaps[min(self.snap_idx, len(self.snaps)) - 1]:
                    self.snap_idx += 1
                self.CFL = 0.0
            log.append((dt_used, ierr))
        return log

    def state(self):
        """Padded state as a (m_eta+4, m_xi+4, 3) array, the layout of vars(3, i, j)."""
        return np.ascontiguousarray(np.transpose(self.vars.a, (2, 1, 0)))

    def set_state(self, q):
        self.vars.a[...] = np.transpose(q, (2, 1, 0))

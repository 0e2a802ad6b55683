"""Fast FCM of the reference restated in FP64 with numpy (test infrastructure only).

Follows racksa/CUFCM_FIL src/cufcm/:
  FCM_solver::init_config / init_fcm_var   CUFCM_SOLVER.cu:37-125 (derived parameters)
  box / images                             CUFCM_DATA.cu:427-460   (wrap into the box)
  spread (modified Gaussian, ROTATION 0)   CUFCM_FCM.cu:16-184
  cufcm_flow_solve                         CUFCM_FCM.cu:187-246
  gather                                   CUFCM_FCM.cu:249-423
  cufcm_pair_correction / self_correction  CUFCM_CORRECTION.cu:43-352
The near-field correction visits all pairs directly (equivalent to the
reference's cell list, which only prunes pairs beyond Rc).  Sizes are meant for
small grids (tests).
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import erf


class FcmParams:
    def __init__(self, rh=1.0, alpha=1.0, beta=10.0, eta=6.0, nx=64, ny=64, nz=64, boxsize=128.0):
        self.rh, self.alpha, self.beta, self.eta = rh, alpha, beta, eta
        self.nx, self.ny, self.nz = nx, ny, nz
        self.Lx = boxsize
        self.Ly = boxsize / nx * ny
        self.Lz = boxsize / nx * nz
        self.dx = self.Lx / nx
        self.ngd = int(round(alpha * beta))
        self.sigma = rh / math.sqrt(math.pi)
        self.Sigma = self.dx * alpha
        self.pdmag = self.sigma ** 2 - self.Sigma ** 2
        self.Rc = eta * alpha * self.dx
        pi = math.pi
        self.self_mob = (1.0 / (6 * pi * rh) - 1.0 / (6 * pi * self.Sigma * math.sqrt(pi))
                         + self.pdmag / (12.0 * (math.sqrt(pi) * self.Sigma) ** 3)
                         - self.pdmag ** 2 / (32.0 * pi ** 1.5 * self.Sigma ** 5))


def _wrap(x, L):
    x = x - np.floor(x / L) * L
    return np.where(x == L, 0.0, x)


def _tables(p: FcmParams, y):
    """1-D Gaussian factors, offsets and grid indices of one particle along x, y, z."""
    ngdh = p.ngd // 2
    anorm = 1.0 / math.sqrt(2 * math.pi * p.Sigma ** 2)
    out = []
    for c, n in enumerate((p.nx, p.ny, p.nz)):
        xg = np.rint(y[c] / p.dx) - ngdh + np.arange(p.ngd)
        xx = xg * p.dx - y[c]
        g = anorm * np.exp(-xx * xx / (2 * p.Sigma ** 2))
        ind = (xg - n * np.floor(xg / n)).astype(np.int64)
        out.append((g, xx, ind))
    return out


def _weights(p: FcmParams, tabs):
    (gx, dx_, ix), (gy, dy_, iy), (gz, dz_, iz) = tabs
    S2 = p.Sigma ** 2
    r2 = dx_[None, None, :] ** 2 + dy_[None, :, None] ** 2 + dz_[:, None, None] ** 2   # [k, j, i]
    w = gz[:, None, None] * gy[None, :, None] * gx[None, None, :] * (1.0 + 0.5 * p.pdmag / S2 ** 2 * r2
                                                                      - 1.5 * p.pdmag / S2)
    return w, iz, iy, ix


def fcm_apply(Y, F, p: FcmParams):
    """V = M_FCM F for positions Y [N,3] and forces F [N,3], FP64."""
    Y = np.asarray(Y, float).reshape(-1, 3)
    F = np.asarray(F, float).reshape(-1, 3)
    N = Y.shape[0]
    Y = np.stack([_wrap(Y[:, 0], p.Lx), _wrap(Y[:, 1], p.Ly), _wrap(Y[:, 2], p.Lz)], axis=1)
    grid = np.zeros((3, p.nz, p.ny, p.nx))
    tabs_all = []
    for n in range(N):
        tabs = _tables(p, Y[n])
        w, iz, iy, ix = _weights(p, tabs)
        tabs_all.append((w, iz, iy, ix))
        K, J, I = np.meshgrid(iz, iy, ix, indexing="ij")
        for c in range(3):
            np.add.at(grid[c], (K, J, I), F[n, c] * w)
    spec = np.fft.rfftn(grid, axes=(1, 2, 3))
    q1 = 2 * math.pi / p.Lx * np.arange(p.nx // 2 + 1)
    q2 = 2 * math.pi / p.Ly * np.fft.fftfreq(p.ny, 1.0 / p.ny)
    q3 = 2 * math.pi / p.Lz * np.fft.fftfreq(p.nz, 1.0 / p.nz)
    Q3, Q2, Q1 = np.meshgrid(q3, q2, q1, indexing="ij")
    qq = Q1 ** 2 + Q2 ** 2 + Q3 ** 2
    qq[0, 0, 0] = 1.0
    kdotf = (Q1 * spec[0] + Q2 * spec[1] + Q3 * spec[2]) / qq
    u = np.stack([(spec[0] - Q1 * kdotf) / qq, (spec[1] - Q2 * kdotf) / qq, (spec[2] - Q3 * kdotf) / qq])
    u[:, 0, 0, 0] = 0.0
    ugrid = np.fft.irfftn(u, s=(p.nz, p.ny, p.nx), axes=(1, 2, 3))
    V = np.zeros((N, 3))
    vol = p.dx ** 3
    for n in range(N):
        w, iz, iy, ix = tabs_all[n]
        K, J, I = np.meshgrid(iz, iy, ix, indexing="ij")
        for c in range(3):
            V[n, c] = np.sum(ugrid[c][K, J, I] * w) * vol
    V += pair_correction(Y, F, p) + F * p.self_mob
    return V


def _blob_pair(r, rsq, sg, sgsq, gauss, erfS):
    SI = 1.0 / (8 * math.pi * r) * ((1.0 + sgsq / rsq) * erfS) - 0.5 * sgsq * sgsq / rsq * gauss
    Sxx = 1.0 / (8 * math.pi * r ** 3) * ((1.0 - 3.0 * sgsq / rsq) * erfS) + 1.5 * sgsq * sgsq / rsq / rsq * gauss
    return SI, Sxx


def pair_correction(Y, F, p: FcmParams):
    """Near-field replacement of the grid interaction within Rc (CUFCM_CORRECTION.cu:103-331)."""
    N = Y.shape[0]
    d = Y[:, None, :] - Y[None, :, :]
    for c, L in enumerate((p.Lx, p.Ly, p.Lz)):
        d[..., c] -= L * np.trunc(d[..., c] / (0.5 * L))
    rsq = np.sum(d * d, axis=-1)
    mask = (rsq < p.Rc ** 2) & ~np.eye(N, dtype=bool)
    V = np.zeros((N, 3))
    ii, jj = np.nonzero(mask)
    if ii.size == 0:
        return V
    x = d[ii, jj]
    rs = rsq[ii, jj]
    r = np.sqrt(rs)
    gam = math.sqrt(2.0) * p.Sigma
    gsq = gam * gam
    gvf = math.sqrt(2.0) * p.sigma
    gvfsq = gvf * gvf
    erfS = erf(0.5 * r / p.Sigma)
    gg = np.exp(-0.5 * rs / gsq) / (2 * math.pi * gsq) ** 1.5
    erfV = erf(r / (math.sqrt(2.0) * gvf))
    ggV = np.exp(-0.5 * rs / gvfsq) / (2 * math.pi * gvfsq) ** 1.5
    A_vf, B_vf = _blob_pair(r, rs, gvf, gvfsq, ggV, erfV)
    A, B = _blob_pair(r, rs, gam, gsq, gg, erfS)
    QI = erfS / (4 * math.pi * r ** 3) - (1.0 + gsq / rs) * gg
    Qxx = -3.0 * erfS / (4 * math.pi * r ** 5) + (1.0 + 3.0 * gsq / rs) / rs * gg
    TI = (2.0 - rs / gsq) / gsq * gg
    Txx = gg / gsq ** 2
    pd = p.pdmag
    t1 = A_vf - A - QI * pd - TI * 0.25 * pd * pd
    t2 = B_vf - B - Qxx * pd - Txx * 0.25 * pd * pd
    Fj = F[jj]
    xf = np.sum(x * Fj, axis=1)
    contrib = t1[:, None] * Fj + t2[:, None] * x * xf[:, None]
    np.add.at(V, ii, contrib)
    return V

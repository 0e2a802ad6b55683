"""Flow-field velocities of the reference's post-processing tool, restated in FP64 (test infrastructure only).

Follows racksa/CUFCM_FIL src/flow_field/flow_field_evaluator.cu:13-217
(flow_velocities) and :545-557 (the 1/(8 pi mu) prefactor): the velocity at
each flow point is the sum over segments of a Stokeslet, with the Blake image
system of a no-slip wall at z = 0 when the simulation has no blobs (a Stokeslet
at the image point subtracted, plus the higher-order image terms), and a rotlet
from each segment torque (no image); plus a Stokeslet per blob; and, with
remove_net_force, minus a Stokeslet of each source's force placed at its body's
position.  Same sign and term order as the kernel; no guard at r = 0 (the
kernel has none either).
"""
from __future__ import annotations

import numpy as np


def flow_velocities(x_flow, x_segs, f_segs, x_blobs=None, f_blobs=None, x_bodies=None, *, n_seg_per_body,
                    n_blob_per_body=0, mu=1.0, remove_net_force=False):
    """x_flow [Nf,3]; x_segs [S,3]; f_segs [S,6] (force, torque); x_blobs [B,3]; f_blobs [B,3];
    x_bodies [Nbods,3].  Returns [Nf,3]."""
    xf = np.asarray(x_flow, float).reshape(-1, 3)
    xs = np.asarray(x_segs, float).reshape(-1, 3)
    fs = np.asarray(f_segs, float).reshape(-1, 6)
    nb_total = 0 if x_blobs is None else np.asarray(x_blobs).size // 3
    v = np.zeros_like(xf)
    for i, (xi, yi, zi) in enumerate(xf):
        dx, dy, dz = xi - xs[:, 0], yi - xs[:, 1], zi - xs[:, 2]
        f, t = fs[:, :3], fs[:, 3:]
        rm2 = 1.0 / (dx * dx + dy * dy + dz * dz)
        rm1 = np.sqrt(rm2)
        rdf = rm2 * (dx * f[:, 0] + dy * f[:, 1] + dz * f[:, 2])
        vx = rm1 * (f[:, 0] + dx * rdf)
        vy = rm1 * (f[:, 1] + dy * rdf)
        vz = rm1 * (f[:, 2] + dz * rdf)
        if n_blob_per_body == 0:
            Rz = zi + xs[:, 2]
            R2 = dx * dx + dy * dy + Rz * Rz
            Rm1 = np.sqrt(1.0 / R2)
            Rdf = (dx * f[:, 0] + dy * f[:, 1] + Rz * f[:, 2]) * Rm1 * Rm1
            vx -= Rm1 * (f[:, 0] + dx * Rdf)
            vy -= Rm1 * (f[:, 1] + dy * Rdf)
            vz -= Rm1 * (f[:, 2] + Rz * Rdf)
            Dxx = (3.0 * dx * dx - R2) * zi
            Dxy = 3.0 * dx * dy * zi
            Dxz = (R2 - 3.0 * Rz * zi) * dx
            Dyy = (3.0 * dy * dy - R2) * zi
            Dyz = (R2 - 3.0 * Rz * zi) * dy
            Dzx = (3.0 * Rz * zi + R2) * dx
            Dzy = (3.0 * Rz * zi + R2) * dy
            Dzz = (R2 - 3.0 * Rz * Rz) * zi
            Dfac = 2.0 * xs[:, 2] * Rm1 ** 5
            vx += Dfac * (Dxx * f[:, 0] + Dxy * f[:, 1] + Dxz * f[:, 2])
            vy += Dfac * (Dxy * f[:, 0] + Dyy * f[:, 1] + Dyz * f[:, 2])
            vz += Dfac * (Dzx * f[:, 0] + Dzy * f[:, 1] + Dzz * f[:, 2])
        rm3 = rm1 * rm2
        vx += rm3 * (t[:, 1] * dz - t[:, 2] * dy)
        vy += rm3 * (t[:, 2] * dx - t[:, 0] * dz)
        vz += rm3 * (t[:, 0] * dy - t[:, 1] * dx)
        if remove_net_force:
            body = np.arange(xs.shape[0]) // n_seg_per_body
            xb = np.asarray(x_bodies, float).reshape(-1, 3)[body]
            vx, vy, vz = _minus_stokeslet(vx, vy, vz, xi - xb[:, 0], yi - xb[:, 1], zi - xb[:, 2], f)
        acc = np.array([vx.sum(), vy.sum(), vz.sum()])
        if nb_total:
            xb_ = np.asarray(x_blobs, float).reshape(-1, 3)
            fb = np.asarray(f_blobs, float).reshape(-1, 3)
            dx, dy, dz = xi - xb_[:, 0], yi - xb_[:, 1], zi - xb_[:, 2]
            rm2 = 1.0 / (dx * dx + dy * dy + dz * dz)
            rm1 = np.sqrt(rm2)
            rdf = rm2 * (dx * fb[:, 0] + dy * fb[:, 1] + dz * fb[:, 2])
            bx = rm1 * (fb[:, 0] + dx * rdf)
            by = rm1 * (fb[:, 1] + dy * rdf)
            bz = rm1 * (fb[:, 2] + dz * rdf)
            if remove_net_force:
                body = np.arange(nb_total) // n_blob_per_body
                xbd = np.asarray(x_bodies, float).reshape(-1, 3)[body]
                bx, by, bz = _minus_stokeslet(bx, by, bz, xi - xbd[:, 0], yi - xbd[:, 1], zi - xbd[:, 2], fb)
            acc += np.array([bx.sum(), by.sum(), bz.sum()])
        v[i] = acc / (8.0 * np.pi * mu)
    return v


def _minus_stokeslet(vx, vy, vz, dx, dy, dz, f):
    rm2 = 1.0 / (dx * dx + dy * dy + dz * dz)
    rm1 = np.sqrt(rm2)
    rdf = rm2 * (dx * f[:, 0] + dy * f[:, 1] + dz * f[:, 2])
    return (vx - rm1 * (f[:, 0] + dx * rdf), vy - rm1 * (f[:, 1] + dy * rdf), vz - rm1 * (f[:, 2] + dz * rdf))

// learned_kernels.cuh -- the per-filament network inside flexible GMRES
// (CF_PRECOND_LEARNED).  No counterpart in the reference.
//
// For a residual vector r and filament m the network sees, scaled by
// s_m = |(r_m, rbar_m)|:
//   r_m      the filament's 3*nseg constraint-force rows and its two rate rows
//            (zero where the rate block is absent),
//   rbar_m   the mean force rows of its neighbours along the lattice line
//            (the beat direction, where the hydrodynamic coupling is strongest),
// and, unscaled, its segment positions relative to its base divided by the
// filament length.  Its output delta_m (3*nseg + 2 values) corrects the
// block-diagonal preconditioner (CF_PRECOND_LEARNED) or the line-patch
// preconditioner (CF_PRECOND_LEARNED_LINE):  z_m = P(r)_m + s_m delta_m.
// Training pairs come from the plain solver itself: after each Arnoldi
// product w = A z (z = P_bd(q)) the features of w and the target
// (z_m - P_bd(w)_m) / s_m are stored, so that the network learns the part of
// A^-1 that the block-diagonal preconditioner misses.
#pragma once

#include "sim_kernels.cuh"

namespace cufil {

// Features of v (and the scale of each filament) into d.lx / d.lscale; one block per filament.
__global__ void learned_features_kernel(SimDev d, const double *v, float *X, float *scale) {
    __shared__ double sm32[32];
    __shared__ double s_inv;
    const int m = blockIdx.x;
    const FilRows fr = fil_rows(d, m);
    const int nl = 3 * d.nseg;
    const int n0 = d.nbr[2 * m], n1 = d.nbr[2 * m + 1];
    const int nn = (n0 >= 0) + (n1 >= 0);
    const FilRows f0 = fil_rows(d, n0 >= 0 ? n0 : m), f1 = fil_rows(d, n1 >= 0 ? n1 : m);
    double ss = 0.0;
    for (int j = threadIdx.x; j < nl; j += blockDim.x) {
        const double a = v[fr.lam + j];
        double b = 0.0;
        if (n0 >= 0) b += v[f0.lam + j];
        if (n1 >= 0) b += v[f1.lam + j];
        if (nn) b /= nn;
        ss += a * a + b * b;
    }
    if (threadIdx.x == 0) {
        if (fr.pr >= 0) ss += v[fr.pr] * v[fr.pr];
        if (fr.ar >= 0) ss += v[fr.ar] * v[fr.ar];
    }
    ss = block_sum(ss, sm32);
    if (threadIdx.x == 0) {
        const double s = sqrt(ss);
        scale[m] = static_cast<float>(s);
        s_inv = s > 0.0 ? 1.0 / s : 0.0;
    }
    __syncthreads();
    const double si = s_inv;
    float *x = X + static_cast<size_t>(m) * d.lin;
    for (int j = threadIdx.x; j < nl; j += blockDim.x) {
        double b = 0.0;
        if (n0 >= 0) b += v[f0.lam + j];
        if (n1 >= 0) b += v[f1.lam + j];
        if (nn) b /= nn;
        x[j] = static_cast<float>(v[fr.lam + j] * si);
        x[nl + 2 + j] = static_cast<float>(b * si);
        const int k = j / 3, c = j - 3 * k;
        x[2 * nl + 2 + j] = static_cast<float>((d.xd[3 * (m * d.nseg + k) + c] - d.base[3 * m + c]) / d.L);
    }
    if (threadIdx.x == 0) {
        x[nl] = fr.pr >= 0 ? static_cast<float>(v[fr.pr] * si) : 0.0f;
        x[nl + 1] = fr.ar >= 0 ? static_cast<float>(v[fr.ar] * si) : 0.0f;
    }
}

// Z_k = P(Q_k) + s_m delta_m (the current basis index k), copied to z; P(Q_k) is Z_k itself (block-diagonal
// base) or z (line-patch base, base_z).  One block per filament.
__global__ void learned_correct_kernel(SimDev d, const float *Y, const float *scale, int base_z) {
    const int m = blockIdx.x;
    const FilRows fr = fil_rows(d, m);
    if (!d.active[fr.b]) return;
    const int k = d.lc->k;
    if (k >= d.arr[fr.b].max_iter) return;
    double *zk = d.Z + static_cast<size_t>(k) * d.ldq;
    const int nl = 3 * d.nseg;
    const double s = d.lalpha * scale[m];
    const float *y = Y + static_cast<size_t>(m) * d.lout;
    const double *base = base_z ? d.z : zk;
    for (int j = threadIdx.x; j < nl; j += blockDim.x) {
        const double val = base[fr.lam + j] + s * y[j];
        zk[fr.lam + j] = val;
        d.z[fr.lam + j] = val;
    }
    if (threadIdx.x == 0) {
        if (fr.pr >= 0) {
            const double val = base[fr.pr] + s * y[nl];
            zk[fr.pr] = val;
            d.z[fr.pr] = val;
        }
        if (fr.ar >= 0) {
            const double val = base[fr.ar] + s * y[nl + 1];
            zk[fr.ar] = val;
            d.z[fr.ar] = val;
        }
    }
}

// Training target of one Arnoldi pair: T_m = (z_m - P_bd(w)_m) / s_m with the
// scale of w's features; pbd = P_bd(w).  One block per filament.
__global__ void learned_target_kernel(SimDev d, const double *z, const double *pbd, const float *scale, float *T) {
    const int m = blockIdx.x;
    const FilRows fr = fil_rows(d, m);
    const int nl = 3 * d.nseg;
    const double s = scale[m];
    const double si = s > 0.0 ? 1.0 / s : 0.0;
    float *t = T + static_cast<size_t>(m) * d.lout;
    for (int j = threadIdx.x; j < nl; j += blockDim.x) t[j] = static_cast<float>((z[fr.lam + j] - pbd[fr.lam + j]) * si);
    if (threadIdx.x == 0) {
        t[nl] = fr.pr >= 0 ? static_cast<float>((z[fr.pr] - pbd[fr.pr]) * si) : 0.0f;
        t[nl + 1] = fr.ar >= 0 ? static_cast<float>((z[fr.ar] - pbd[fr.ar]) * si) : 0.0f;
    }
}

}  // namespace cufil

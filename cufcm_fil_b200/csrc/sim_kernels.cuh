// sim_kernels.cuh -- device side of the implicit prescribed-cilia step.
//
// Everything here runs in FP64 except the pairwise mobility (rpy_kernels.cu),
// which is FP32 with compensated sums:
//   kinematics_kernel   filament::initial_guess for prescribed cilia
//                       (src/cilia/filament.cpp:1336-1500): phase/angle update,
//                       arclength parameters (table or bisection,
//                       filament.cpp:1096-1230), positions and the velocity
//                       directions K_phase, K_angle
//   rhs_kernel          mobility_solver::assemble_rhs (mobility_solver.cpp:284-420)
//   precond             apply_preconditioner_new (mobility_solver.cpp:1102-1243)
//   saddle_epilogue     system_matrix_mult_new (mobility_solver.cpp:1887-2105):
//                       reduces the mobility partials and adds the K terms
//   GMRES kernels       solve_linear_system (mobility_solver.cpp:2187-2669) with
//                       classical Gram-Schmidt applied twice (CGS2) in place of
//                       modified Gram-Schmidt: the same Krylov basis and
//                       Hessenberg matrix up to rounding, with two reductions
//                       per iteration instead of one per basis vector.
// One thread block per filament for all per-filament work; reductions that span
// blocks write per-block partials and the last block to finish combines them in
// a fixed order (deterministic, no spin waits).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace cufil {

constexpr int kBeatModes = 4;    // Fourier modes of the fitted beat (mode 0 = constant)
constexpr int kBeatDegrees = 3;  // polynomial degree in the arclength parameter

struct BeatCoeffs {
    double Ax[kBeatModes][kBeatDegrees], Ay[kBeatModes][kBeatDegrees];
    double Bx[kBeatModes - 1][kBeatDegrees], By[kBeatModes - 1][kBeatDegrees];
    double c0;  // weight of the constant mode (1, or 1/2 for the original table)
};

enum GmresStatus : int {
    kGmresRunning = 0,
    kGmresConverged = 1,
    kGmresMaxIter = 2,
    kGmresNonFinite = 3,
    kGmresGuessGood = 4,
    kGmresZeroRhs = 5,
};

struct GmresCtl {
    int nt;           // time-step index of the step being solved
    int k;            // index of the newest basis vector
    int iters;        // Arnoldi iterations done
    int status;       // GmresStatus
    int zero_guess;   // initial guess discarded (start from 0)
    int cond;         // loop condition (mirrors the graph conditional)
    unsigned int counter;  // last-block ticket
    int pad;
    double norm_rhs, beta0, relres;
    double inv_scale; // normalisation pending for the newest basis vector
};

struct SimDev {
    int F, nseg, N, n;       // filaments, segments per filament, segments, system size
    int po, ao;              // offsets of the phase / angle rate blocks (-1 if absent)
    int ldq, ldh, max_iter;  // basis stride, Hessenberg leading dimension, iteration cap
    int flexible;            // keep Z = P^{-1} Q (nonlinear preconditioner)
    int precond;             // 0: none, 1: block-diagonal
    int nsplit;              // mobility partial splits
    int s_rows, s_cols;      // arclength table (0 rows: bisection)
    int n_phase_refs, n_angle_refs;
    double dt, L, spring, tol, s_tol;
    double R[9];             // filament frame (row-major)
    BeatCoeffs beat;
    const double *s_table, *phase_refs, *angle_refs, *omega0, *base;
    double *phase, *angle, *phase_dot, *angle_dot;
    float4 *x4;              // segment centres for the pair kernel
    double *xd, *kp, *ka;    // centres and velocity directions [3N]
    double *s_cur;           // arclength parameters of the current step [N]
    double *gram;            // per filament (c11, c22, c12)
    double *rhs, *sol, *w, *z, *t, *y;
    double *Q, *Z, *H, *cs, *sn, *beta, *h1, *h2;
    double *dots_partial, *norm_partial;
    float4 *f4;              // forces for the pair kernel
    const float4 *partial;   // mobility partials [nsplit][N]
    GmresCtl *ctl;
    int *iter_log;           // GMRES iterations of each step, [iter_log_cap] ring
    int iter_log_cap;
    int dots_chunk, dots_nchunk;
};

constexpr double kSegMobInv = 6.0 * 3.14159265358979323846;  // 6 pi mu a, mu = a = 1

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum (blockDim.x a multiple of 32, <= 1024); result valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double *sm32) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sm32[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        r = lane < nw ? sm32[lane] : 0.0;
        r = warp_sum(r);
    }
    return r;
}

// Returns true in every thread of the last block to pass this point (after
// the block's global writes were fenced); that block must reset the ticket.
__device__ __forceinline__ bool last_block_ticket(unsigned int *counter, int *sm_flag) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) *sm_flag = (atomicAdd(counter, 1u) == gridDim.x - 1) ? 1 : 0;
    __syncthreads();
    return *sm_flag != 0;
}

__device__ __forceinline__ void set_loop(cudaGraphConditionalHandle h, GmresCtl *ctl, int cond) {
    ctl->cond = cond;
    if (h) cudaGraphSetConditional(h, cond ? 1u : 0u);
}

// Wall self-mobility block in FP64 (cuda_functions.cu:24-38).
__device__ __forceinline__ void wall_self_f64(double z, const double *f, double *v) {
    const double c = 1.0 / (6.0 * 3.14159265358979323846);
    const double h1 = 1.0 / z, h3 = h1 * h1 * h1, h5 = h3 * h1 * h1;
    v[0] += (c - (9.0 * h1 - 2.0 * h3 + h5) * (c / 16.0)) * f[0];
    v[1] += (c - (9.0 * h1 - 2.0 * h3 + h5) * (c / 16.0)) * f[1];
    v[2] += (c - (9.0 * h1 - 4.0 * h3 + h5) * (c / 8.0)) * f[2];
}

// Filament rows of the saddle product, out[po+m] = -K_phase^T lambda_m and
// out[ao+m] = -K_angle^T lambda_m (mobility_solver.cpp:2000-2060), for block m.
// Called by the kernels that produce the vector v (all threads of the block).
__device__ void filament_rows(const SimDev &d, int m, const double *v, double *out, double *sm32) {
    if (d.po < 0 && d.ao < 0) return;
    const int nb = 3 * d.nseg, off = nb * m;
    double dp = 0.0, da = 0.0;
    for (int j = threadIdx.x; j < nb; j += blockDim.x) {
        dp += d.kp[off + j] * v[off + j];
        da += d.ka[off + j] * v[off + j];
    }
    dp = block_sum(dp, sm32);
    da = block_sum(da, sm32);
    if (threadIdx.x == 0) {
        if (d.po >= 0) out[d.po + m] = -dp;
        if (d.ao >= 0) out[d.ao + m] = -da;
    }
}

// ------------------------------------------------------------- beat shape
struct BeatRow {  // coefficient vectors of one phase
    double cx[kBeatDegrees], cy[kBeatDegrees];  // shape
    double dx[kBeatDegrees], dy[kBeatDegrees];  // d/dpsi
};

__device__ inline void beat_row(const BeatCoeffs &b, double psi, BeatRow &r) {
    double c[kBeatModes], s[kBeatModes];
    c[0] = b.c0;
    s[0] = 0.0;
    for (int n = 1; n < kBeatModes; ++n) sincos(n * psi, &s[n], &c[n]);
    for (int d = 0; d < kBeatDegrees; ++d) {
        double cx = 0, cy = 0, dx = 0, dy = 0;
        for (int n = 0; n < kBeatModes; ++n) {
            cx += c[n] * b.Ax[n][d];
            cy += c[n] * b.Ay[n][d];
            dx += -n * s[n] * b.Ax[n][d];
            dy += -n * s[n] * b.Ay[n][d];
        }
        for (int n = 1; n < kBeatModes; ++n) {
            cx += s[n] * b.Bx[n - 1][d];
            cy += s[n] * b.By[n - 1][d];
            dx += n * c[n] * b.Bx[n - 1][d];
            dy += n * c[n] * b.By[n - 1][d];
        }
        r.cx[d] = cx;
        r.cy[d] = cy;
        r.dx[d] = dx;
        r.dy[d] = dy;
    }
}

// |d(shape)/ds| at s (filament.cpp:962-990 + the norm in fitted_curve_length).
__device__ __forceinline__ double beat_speed(const BeatRow &r, double s) {
    double tx = 0, ty = 0, sp = 1.0;
    for (int d = 0; d < kBeatDegrees; ++d) {
        tx += (d + 1) * r.cx[d] * sp;
        ty += (d + 1) * r.cy[d] * sp;
        sp *= s;
    }
    return sqrt(tx * tx + ty * ty);
}

// --------------------------------------------------------------- kernels

// One block per filament.  Dynamic shared memory: doubles for the trapezoid
// table (2*(10*nseg+1)) and the arclength parameters (nseg).
__global__ void kinematics_kernel(SimDev d) {
    extern __shared__ double smk[];
    __shared__ double sm32[32];
    __shared__ double sh_psi, sh_ang;
    __shared__ BeatRow row;
    const int m = blockIdx.x;
    const int nseg = d.nseg;
    const int ntraps = 10 * nseg;
    double *f = smk;                 // [ntraps+1]
    double *cum = smk + ntraps + 1;  // [ntraps+1]
    double *s = cum + ntraps + 1;    // [nseg]

    if (threadIdx.x == 0) {
        double psi = d.phase[m], ang = d.angle[m];
        if (d.ctl->nt > 0) {
            psi += d.phase_dot[m] * d.dt;
            ang += d.angle_dot[m] * d.dt;
            d.phase[m] = psi;
            d.angle[m] = ang;
        }
        sh_psi = psi;
        sh_ang = ang;
        beat_row(d.beat, psi, row);
    }
    __syncthreads();
    const double psi = sh_psi;

    if (d.s_rows > 0) {
        // bilinear interpolation in the reference table (filament.cpp:1186-1224)
        double idx = 0.5 * psi / 3.14159265358979323846;
        idx -= floor(idx);
        idx *= d.s_rows;
        const int lo = static_cast<int>(idx);
        for (int k = threadIdx.x; k < nseg; k += blockDim.x) {
            double val;
            if (k == 0) {
                val = 0.0;
            } else if (k == nseg - 1) {
                val = 1.0;
            } else {
                const double si = (d.s_cols - 1) * static_cast<double>(k) / (nseg - 1);
                const int sl = static_cast<int>(si);
                auto row_at = [&](int r, int c) { return d.s_table[r * d.s_cols + c]; };
                double a0, a1;
                if (lo >= d.s_rows) {
                    a0 = row_at(0, sl);
                    a1 = row_at(0, sl + 1);
                } else {
                    const int up = (lo == d.s_rows - 1) ? 0 : lo + 1;
                    const double t = idx - lo;
                    a0 = row_at(lo, sl) + (row_at(up, sl) - row_at(lo, sl)) * t;
                    a1 = row_at(lo, sl + 1) + (row_at(up, sl + 1) - row_at(lo, sl + 1)) * t;
                }
                val = a0 + (si - sl) * (a1 - a0);
            }
            s[k] = val;
        }
    } else {
        // bisection on the trapezoid-rule arclength (filament.cpp:1054-1180)
        const double dl = 1.0 / ntraps;
        for (int p = threadIdx.x; p <= ntraps; p += blockDim.x) f[p] = beat_speed(row, p * dl);
        __syncthreads();
        if (threadIdx.x == 0) {
            cum[0] = 0.0;
            for (int p = 1; p <= ntraps; ++p) cum[p] = cum[p - 1] + 0.5 * dl * (f[p - 1] + f[p]);
            auto length = [&](double sv) {
                if (sv <= 0.0) return 0.0;
                const double fl = floor(sv / dl);
                const int ifl = static_cast<int>(fl);
                double len = cum[ifl];
                const double ce = ceil(sv / dl);
                if (ce > fl) len += ((sv / dl - fl) / (ce - fl)) * 0.5 * dl * (f[ifl] + f[static_cast<int>(ce)]);
                return len;
            };
            const double total = length(1.0);
            s[0] = 0.0;
            s[nseg - 1] = 1.0;
            for (int k = 1; k < nseg - 1; ++k) {
                const double target = static_cast<double>(k) / (nseg - 1);
                double lo = s[k - 1], hi = 1.0;
                double est = 0.5 * (lo + hi);
                double frac = length(est) / total;
                // The interval halves each pass; 200 passes exhaust FP64 resolution.
                for (int it = 0; it < 200 && fabs(frac - target) > d.s_tol; ++it) {
                    if (frac > target) hi = est;
                    else lo = est;
                    est = 0.5 * (lo + hi);
                    frac = length(est) / total;
                }
                s[k] = est;
            }
        }
    }
    __syncthreads();

    for (int k = threadIdx.x; k < nseg; k += blockDim.x) d.s_cur[m * nseg + k] = s[k];

    // positions and velocity directions (filament.cpp:1425-1500)
    const double ca = cos(sh_ang), sa = sin(sh_ang);
    const double *R = d.R;
    const double bx = d.base[3 * m], by = d.base[3 * m + 1], bz = d.base[3 * m + 2];
    double g11 = 0, g22 = 0, g12 = 0;
    for (int k = threadIdx.x; k < nseg; k += blockDim.x) {
        const int i = m * nseg + k;
        double x[3] = {bx, by, bz}, kpv[3] = {0, 0, 0}, kav[3] = {0, 0, 0};
        if (k > 0) {
            const double sv = s[k];
            double sx = 0, sy = 0, vx = 0, vy = 0, sp = sv;
            for (int dd = 0; dd < kBeatDegrees; ++dd) {
                sx += row.cx[dd] * sp;
                sy += row.cy[dd] * sp;
                vx += row.dx[dd] * sp;
                vy += row.dy[dd] * sp;
                sp *= sv;
            }
            // ref = L * Rshape * (sx, sy, 0); Rshape rotates about the reference z axis
            const double rx = d.L * (ca * sx - sa * sy), ry = d.L * (sa * sx + ca * sy);
            const double qx = d.L * (ca * vx - sa * vy), qy = d.L * (sa * vx + ca * vy);
            for (int c = 0; c < 3; ++c) {
                x[c] += R[3 * c + 0] * rx + R[3 * c + 1] * ry;
                kav[c] = R[3 * c + 0] * (-ry) + R[3 * c + 1] * rx;  // R (e_z x ref)
                kpv[c] = R[3 * c + 0] * qx + R[3 * c + 1] * qy;
            }
        }
        d.x4[i] = make_float4(static_cast<float>(x[0]), static_cast<float>(x[1]), static_cast<float>(x[2]), 0.0f);
        for (int c = 0; c < 3; ++c) {
            d.xd[3 * i + c] = x[c];
            d.kp[3 * i + c] = kpv[c];
            d.ka[3 * i + c] = kav[c];
            g11 += kpv[c] * kpv[c];
            g22 += kav[c] * kav[c];
            g12 += kav[c] * kpv[c];
        }
    }
    g11 = block_sum(g11, sm32);
    if (threadIdx.x == 0) d.gram[3 * m + 0] = g11;
    g22 = block_sum(g22, sm32);
    if (threadIdx.x == 0) d.gram[3 * m + 1] = g22;
    g12 = block_sum(g12, sm32);
    if (threadIdx.x == 0) d.gram[3 * m + 2] = g12;
}

// Cyclic cubic Hermite interpolation over one beat (mobility_solver.cpp:242-282).
__device__ inline double cyclic_spline(double phase, const double *tab, int n) {
    double x = 0.5 * phase / 3.14159265358979323846;
    x -= floor(x);
    x *= n;
    const int lo = static_cast<int>(x);
    if (lo >= n) return tab[0];
    const int up = (lo == n - 1) ? 0 : lo + 1;
    const double qlo = tab[lo];
    const double dqlo = (lo == 0) ? (tab[1] - tab[0]) : 0.5 * (tab[up] - tab[lo - 1]);
    const double qup = tab[up];
    const double dqup = (up == 0) ? (tab[0] - tab[n - 1]) : 0.5 * (tab[(up == n - 1) ? 0 : up + 1] - tab[lo]);
    const double t = x - lo, t2 = t * t, t3 = t2 * t;
    return qlo * (2 * t3 - 3 * t2 + 1) + dqlo * (t3 - 2 * t2 + t) + qup * (3 * t2 - 2 * t3) + dqup * (t3 - t2);
}

// RHS (one block per filament) + packing of the current solution's forces for
// the initial residual; ||rhs|| into ctl->norm_rhs by the last block.
__global__ void rhs_kernel(SimDev d) {
    __shared__ double sm32[32];
    __shared__ int last;
    const int m = blockIdx.x;
    const int nb = 3 * d.nseg, off = nb * m;
    double ss = 0.0;
    const bool lam_rows_zero = d.po >= 0;
    for (int j = threadIdx.x; j < nb; j += blockDim.x) {
        const double v = lam_rows_zero ? 0.0 : d.phase_dot[m] * d.kp[off + j];
        d.rhs[off + j] = v;
        ss += v * v;
    }
    for (int k = threadIdx.x; k < d.nseg; k += blockDim.x) {
        const int i = m * d.nseg + k;
        d.f4[i] = make_float4(static_cast<float>(d.sol[3 * i]), static_cast<float>(d.sol[3 * i + 1]),
                              static_cast<float>(d.sol[3 * i + 2]), 0.0f);
    }
    if (threadIdx.x == 0) {
        const double w0 = d.omega0[m] * 0.5 / 3.14159265358979323846;
        double q_angle = 0.0;
        if (d.ao >= 0) {
            q_angle = cyclic_spline(d.phase[m], d.angle_refs, d.n_angle_refs) * w0;
            q_angle -= d.spring * d.omega0[m] * d.L * d.L * d.L * d.angle[m];
            d.rhs[d.ao + m] = -q_angle;
            ss += q_angle * q_angle;
        }
        if (d.po >= 0) {
            const double q_phase = cyclic_spline(d.phase[m], d.phase_refs, d.n_phase_refs) * w0;
            d.rhs[d.po + m] = -q_phase;
            ss += q_phase * q_phase;
        }
    }
    ss = block_sum(ss, sm32);
    if (threadIdx.x == 0) d.norm_partial[m] = ss;
    filament_rows(d, m, d.sol, d.w, sm32);  // filament rows of A x0 for the initial residual
    if (last_block_ticket(&d.ctl->counter, &last)) {
        if (threadIdx.x == 0) {
            double acc = 0.0;
            for (int b = 0; b < gridDim.x; ++b) acc += __ldcg(&d.norm_partial[b]);
            d.ctl->norm_rhs = sqrt(acc);
            d.ctl->counter = 0;
        }
    }
}

// Block-diagonal preconditioner of one filament (apply_preconditioner_new,
// PRESCRIBED_BODY_VELOCITIES branch): in -> out, may alias.  sm holds 3*nseg doubles.
__device__ void precond_block(const SimDev &d, int m, const double *in, double *out, double *sm, double *sm32) {
    __shared__ double coef[2];
    const int nb = 3 * d.nseg, off = nb * m;
    const double *kp = d.kp + off, *ka = d.ka + off;
    double dp = 0.0, da = 0.0;
    for (int j = threadIdx.x; j < nb; j += blockDim.x) {
        const double r = (d.precond ? kSegMobInv : 1.0) * in[off + j];
        sm[j] = r;
        dp += kp[j] * r;
        da += ka[j] * r;
    }
    if (!d.precond) {
        __syncthreads();
        for (int j = threadIdx.x; j < nb; j += blockDim.x) out[off + j] = sm[j];
        if (threadIdx.x == 0) {
            if (d.po >= 0) out[d.po + m] = in[d.po + m];
            if (d.ao >= 0) out[d.ao + m] = in[d.ao + m];
        }
        return;
    }
    if (d.po < 0 && d.ao < 0) {
        __syncthreads();
        for (int j = threadIdx.x; j < nb; j += blockDim.x) out[off + j] = sm[j];
        return;
    }
    dp = block_sum(dp, sm32);
    da = block_sum(da, sm32);
    if (threadIdx.x == 0) {
        const double c11 = d.gram[3 * m], c22 = d.gram[3 * m + 1], c12 = d.gram[3 * m + 2];
        double ph = 0.0, an = 0.0;
        if (d.po >= 0 && d.ao >= 0) {
            const double p = -in[d.po + m] - dp;
            const double a = -in[d.ao + m] - da;
            const double det = c11 * c22 - c12 * c12;
            ph = (p * (c22 / det) + a * (-c12 / det)) / kSegMobInv;
            an = (p * (-c12 / det) + a * (c11 / det)) / kSegMobInv;
        } else if (d.po >= 0) {
            ph = (-in[d.po + m] - dp) / (c11 * kSegMobInv);
        } else {
            an = (-in[d.ao + m] - da) / (c22 * kSegMobInv);
        }
        coef[0] = ph;
        coef[1] = an;
        if (d.po >= 0) out[d.po + m] = ph;
        if (d.ao >= 0) out[d.ao + m] = an;
    }
    __syncthreads();
    const double ph = coef[0], an = coef[1];
    for (int j = threadIdx.x; j < nb; j += blockDim.x)
        out[off + j] = sm[j] + kSegMobInv * (ph * kp[j] + an * ka[j]);
    __syncthreads();
}

// Standalone preconditioner application (host API and final update).
__global__ void precond_kernel(SimDev d, const double *in, double *out) {
    extern __shared__ double smp[];
    __shared__ double sm32[32];
    precond_block(d, blockIdx.x, in, out, smp, sm32);
}

// First kernel of a GMRES iteration: stores the normalised basis vector
// Q_k = src * inv_scale, applies P^{-1} into z (and Z_k when flexible) and
// packs the force part of z for the pair kernel.
//
// It also clears the loop condition: only a completed Givens step of this
// iteration (update_kernel, final pass) re-arms it, so the loop cannot outlive
// a kernel that failed to run its bookkeeping, and never passes max_iter.
__global__ void arnoldi_precond_kernel(SimDev d, cudaGraphConditionalHandle h) {
    extern __shared__ double smp[];
    __shared__ double sm32[32];
    const int m = blockIdx.x;
    GmresCtl *ctl = d.ctl;
    const int k = ctl->k;
    if (m == 0 && threadIdx.x == 0) set_loop(h, ctl, 0);
    if (k >= d.max_iter) return;  // defensive: the cap was reached (uniform over the grid)
    const double sc = ctl->inv_scale;
    const double *src = (k == 0) ? (ctl->zero_guess ? d.rhs : d.Q) : d.w;
    double *q = d.Q + static_cast<size_t>(k) * d.ldq;
    const int nb = 3 * d.nseg, off = nb * m;
    for (int j = threadIdx.x; j < nb; j += blockDim.x) q[off + j] = src[off + j] * sc;
    if (threadIdx.x == 0) {
        if (d.po >= 0) q[d.po + m] = src[d.po + m] * sc;
        if (d.ao >= 0) q[d.ao + m] = src[d.ao + m] * sc;
    }
    __syncthreads();
    double *zout = d.flexible ? d.Z + static_cast<size_t>(k) * d.ldq : d.z;
    precond_block(d, m, q, zout, smp, sm32);
    for (int kk = threadIdx.x; kk < d.nseg; kk += blockDim.x) {
        const int i = m * d.nseg + kk;
        d.f4[i] = make_float4(static_cast<float>(zout[3 * i]), static_cast<float>(zout[3 * i + 1]),
                              static_cast<float>(zout[3 * i + 2]), 0.0f);
    }
    if (d.flexible) {
        for (int j = threadIdx.x; j < nb; j += blockDim.x) d.z[off + j] = zout[off + j];
        if (threadIdx.x == 0) {
            if (d.po >= 0) d.z[d.po + m] = zout[d.po + m];
            if (d.ao >= 0) d.z[d.ao + m] = zout[d.ao + m];
        }
    }
    // Block m read w only in its own rows (above), so it may now write the
    // filament rows of the new product A z.
    __syncthreads();
    filament_rows(d, m, zout, d.w, sm32);
}

__global__ void filament_rows_kernel(SimDev d, const double *v, double *out) {
    __shared__ double sm32[32];
    filament_rows(d, blockIdx.x, v, out, sm32);
}

// Segment rows of out = A v (system_matrix_mult_new): reduces the mobility
// partials of v's force part (one warp per segment, splits strided over the
// lanes), adds the FP64 wall self block and the -K rate terms.  The filament
// rows are written by the kernel that produced v.
__global__ void saddle_epilogue_kernel(SimDev d, const double *v, double *out) {
    const int lane = threadIdx.x & 31;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= d.N) return;
    const float4 *pt = d.partial + static_cast<size_t>(i) * d.nsplit;
    double u0 = 0.0, u1 = 0.0, u2 = 0.0;
    for (int s = lane; s < d.nsplit; s += 32) {
        const float4 q = pt[s];
        u0 += q.x;
        u1 += q.y;
        u2 += q.z;
    }
    u0 = warp_sum(u0);
    u1 = warp_sum(u1);
    u2 = warp_sum(u2);
    if (lane == 0) {
        const int m = i / d.nseg;
        const double vp = d.po >= 0 ? v[d.po + m] : 0.0;
        const double va = d.ao >= 0 ? v[d.ao + m] : 0.0;
        double u[3] = {u0, u1, u2};
        const double f[3] = {v[3 * i], v[3 * i + 1], v[3 * i + 2]};
        wall_self_f64(d.xd[3 * i + 2], f, u);
        for (int c = 0; c < 3; ++c) out[3 * i + c] = u[c] - vp * d.kp[3 * i + c] - va * d.ka[3 * i + c];
    }
}

// r = rhs - A sol into Q_0 (unnormalised); the last block decides how GMRES
// starts (mobility_solver.cpp:2216-2424): zero RHS, good initial guess,
// discard a poor guess, or iterate.
__global__ void residual_decide_kernel(SimDev d, cudaGraphConditionalHandle h) {
    __shared__ double sm32[32];
    __shared__ int last;
    const int m = blockIdx.x;
    const int nb = 3 * d.nseg, off = nb * m;
    double ss = 0.0;
    for (int j = threadIdx.x; j < nb; j += blockDim.x) {
        const double r = d.rhs[off + j] - d.w[off + j];
        d.Q[off + j] = r;
        ss += r * r;
    }
    if (threadIdx.x == 0) {
        if (d.po >= 0) {
            const double r = d.rhs[d.po + m] - d.w[d.po + m];
            d.Q[d.po + m] = r;
            ss += r * r;
        }
        if (d.ao >= 0) {
            const double r = d.rhs[d.ao + m] - d.w[d.ao + m];
            d.Q[d.ao + m] = r;
            ss += r * r;
        }
    }
    ss = block_sum(ss, sm32);
    if (threadIdx.x == 0) d.norm_partial[m] = ss;
    if (last_block_ticket(&d.ctl->counter, &last) && threadIdx.x == 0) {
        GmresCtl *ctl = d.ctl;
        double acc = 0.0;
        for (int b = 0; b < gridDim.x; ++b) acc += __ldcg(&d.norm_partial[b]);
        ctl->counter = 0;
        const double nr = ctl->norm_rhs;
        double b0 = sqrt(acc);
        ctl->k = 0;
        ctl->iters = 0;
        ctl->zero_guess = 0;
        int cond = 1;
        if (!(nr == nr) || !(b0 == b0) || nr > 1.0e300 || b0 > 1.0e300) {
            ctl->status = kGmresNonFinite;
            ctl->relres = b0 / nr;
            cond = 0;
        } else if (nr == 0.0) {
            ctl->status = kGmresZeroRhs;
            ctl->relres = 0.0;
            cond = 0;
        } else if (b0 <= d.tol * nr) {
            ctl->status = kGmresGuessGood;
            ctl->relres = b0 / nr;
            cond = 0;
        } else {
            if (b0 > nr) {  // the initial guess is worse than zero
                ctl->zero_guess = 1;
                b0 = nr;
            }
            ctl->status = kGmresRunning;
            ctl->relres = b0 / nr;
        }
        ctl->beta0 = b0;
        d.beta[0] = b0;
        ctl->inv_scale = (b0 > 0.0) ? 1.0 / b0 : 0.0;
        set_loop(h, ctl, cond);
    }
}

// Partial dot products <Q_j, w>, j <= k, over row chunks; the last block sums
// the chunks of each j in order into h.  Loads are issued four at a time into
// independent accumulators so that each thread keeps several in flight.
__global__ void __launch_bounds__(256) dots_kernel(SimDev d, double *h) {
    __shared__ double sm32[32];
    __shared__ int last;
    const int k = d.ctl->k;
    if (k >= d.max_iter) return;  // defensive, uniform over the grid
    const int C = d.dots_nchunk;
    const int items = (k + 1) * C;
    const double *__restrict__ w = d.w;
    for (int it = blockIdx.x; it < items; it += gridDim.x) {
        const int j = it / C, c = it - j * C;
        const int r0 = c * d.dots_chunk, r1 = min(d.n, r0 + d.dots_chunk);
        const double *__restrict__ q = d.Q + static_cast<size_t>(j) * d.ldq;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
        int i = r0 + threadIdx.x;
        for (; i + 3 * 256 < r1; i += 4 * 256) {
            a0 += q[i] * w[i];
            a1 += q[i + 256] * w[i + 256];
            a2 += q[i + 512] * w[i + 512];
            a3 += q[i + 768] * w[i + 768];
        }
        for (; i < r1; i += 256) a0 += q[i] * w[i];
        double sum = block_sum((a0 + a1) + (a2 + a3), sm32);
        if (threadIdx.x == 0) d.dots_partial[static_cast<size_t>(j) * C + c] = sum;
    }
    if (last_block_ticket(&d.ctl->counter, &last)) {
        for (int j = threadIdx.x; j <= k; j += blockDim.x) {
            double acc = 0.0;
            for (int c = 0; c < C; ++c) acc += __ldcg(&d.dots_partial[static_cast<size_t>(j) * C + c]);
            h[j] = acc;
        }
        __syncthreads();
        if (threadIdx.x == 0) d.ctl->counter = 0;
    }
}

// Givens update of the least-squares problem for column k (mobility_solver.cpp:2462-2515).
// Called by every thread of one block: the column, the previous rotations and
// beta are staged in shared memory (gs: 3*(max_iter+2) doubles), thread 0 runs
// the sequential recurrence there, and the block writes the results back.
__device__ void givens_step(const SimDev &d, double qn, cudaGraphConditionalHandle hcond, double *gs) {
    GmresCtl *ctl = d.ctl;
    const int k = ctl->k;
    double *Hs = gs, *cs = gs + (d.max_iter + 2), *sn = cs + (d.max_iter + 2);
    double *Hc = d.H + static_cast<size_t>(k) * d.ldh;
    for (int j = threadIdx.x; j <= k; j += blockDim.x) Hs[j] = d.h1[j] + d.h2[j];
    for (int j = threadIdx.x; j < k; j += blockDim.x) {
        cs[j] = d.cs[j];
        sn[j] = d.sn[j];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        Hs[k + 1] = qn;
        for (int i = 1; i <= k; ++i) {
            const double t = cs[i - 1] * Hs[i - 1] + sn[i - 1] * Hs[i];
            Hs[i] = cs[i - 1] * Hs[i] - sn[i - 1] * Hs[i - 1];
            Hs[i - 1] = t;
        }
        const double a = Hs[k], b = Hs[k + 1];
        double c, s;
        if (b == 0.0) {
            c = 1.0;
            s = 0.0;
        } else if (fabs(b) > fabs(a)) {
            const double t = a / b;
            s = (b > 0 ? 1.0 : -1.0) / sqrt(1.0 + t * t);
            c = t * s;
        } else {
            const double t = b / a;
            c = (a > 0 ? 1.0 : -1.0) / sqrt(1.0 + t * t);
            s = t * c;
        }
        d.cs[k] = c;
        d.sn[k] = s;
        Hs[k] = c * a + s * b;
        Hs[k + 1] = 0.0;
        const double bk = d.beta[k];
        d.beta[k + 1] = -s * bk;
        d.beta[k] = c * bk;
        const int it = k + 1;
        const double rel = fabs(-s * bk) / ctl->norm_rhs;
        ctl->iters = it;
        ctl->relres = rel;
        int cond = 1;
        if (!(rel == rel) || !(qn == qn) || qn > 1.0e300) {
            ctl->status = kGmresNonFinite;
            cond = 0;
        } else if (rel <= d.tol) {
            ctl->status = kGmresConverged;
            cond = 0;
        } else if (it >= d.max_iter) {
            ctl->status = kGmresMaxIter;
            cond = 0;
        }
        ctl->inv_scale = qn > 0.0 ? 1.0 / qn : 0.0;
        ctl->k = k + 1;
        if (k + 1 >= d.max_iter) cond = 0;
        set_loop(hcond, ctl, cond);
    }
    __syncthreads();
    for (int j = threadIdx.x; j <= k + 1; j += blockDim.x) Hc[j] = Hs[j];
}

// w -= sum_j h_j Q_j; in the final pass also ||w|| and the Givens step.
// Block = 32 rows x 8 basis-vector groups: each thread sums every 8th basis
// vector for one row with loads unrolled 4 deep, and the 8 groups are combined
// in shared memory in a fixed order.
constexpr int kUpdRows = 32, kUpdGroups = 8;
__global__ void __launch_bounds__(kUpdRows * kUpdGroups) update_kernel(SimDev d, const double *h, int final_pass,
                                                                      cudaGraphConditionalHandle hcond) {
    extern __shared__ double gsm[];  // Givens staging, 3*(max_iter+2) doubles (final pass)
    __shared__ double sm32[32];
    __shared__ double part[kUpdGroups][kUpdRows];
    __shared__ int last;
    const int k = d.ctl->k;
    if (k >= d.max_iter) return;  // defensive, uniform over the grid
    const int r = threadIdx.x % kUpdRows, g = threadIdx.x / kUpdRows;
    double ss = 0.0;
    for (int base = blockIdx.x * kUpdRows; base < d.n; base += gridDim.x * kUpdRows) {
        const int i = base + r;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
        if (i < d.n) {
            int j = g;
            for (; j + 3 * kUpdGroups <= k; j += 4 * kUpdGroups) {
                a0 += h[j] * d.Q[static_cast<size_t>(j) * d.ldq + i];
                a1 += h[j + kUpdGroups] * d.Q[static_cast<size_t>(j + kUpdGroups) * d.ldq + i];
                a2 += h[j + 2 * kUpdGroups] * d.Q[static_cast<size_t>(j + 2 * kUpdGroups) * d.ldq + i];
                a3 += h[j + 3 * kUpdGroups] * d.Q[static_cast<size_t>(j + 3 * kUpdGroups) * d.ldq + i];
            }
            for (; j <= k; j += kUpdGroups) a0 += h[j] * d.Q[static_cast<size_t>(j) * d.ldq + i];
        }
        part[g][r] = (a0 + a1) + (a2 + a3);
        __syncthreads();
        if (g == 0 && i < d.n) {
            double acc = 0.0;
            for (int gg = 0; gg < kUpdGroups; ++gg) acc += part[gg][r];
            const double wn = d.w[i] - acc;
            d.w[i] = wn;
            ss += wn * wn;
        }
        __syncthreads();
    }
    if (!final_pass) return;
    ss = block_sum(ss, sm32);
    if (threadIdx.x == 0) d.norm_partial[blockIdx.x] = ss;
    if (last_block_ticket(&d.ctl->counter, &last)) {
        __shared__ double qn;
        if (threadIdx.x == 0) {
            double acc = 0.0;
            for (int b = 0; b < gridDim.x; ++b) acc += __ldcg(&d.norm_partial[b]);
            d.ctl->counter = 0;
            qn = sqrt(acc);
        }
        __syncthreads();
        givens_step(d, qn, hcond, gsm);
    }
}

// Back-substitution H y = beta for the iterations done (mobility_solver.cpp:2520-2537),
// column oriented: after y_i is known every thread updates its own right-hand
// side entry with column i of H (contiguous), so each step is one coalesced sweep.
__global__ void __launch_bounds__(1024) backsub_kernel(SimDev d) {
    extern __shared__ double bsm[];  // [max_iter + 1]
    const GmresCtl *ctl = d.ctl;
    const bool iterated = ctl->status == kGmresConverged || ctl->status == kGmresMaxIter;
    const int it = iterated ? ctl->iters : 0;
    for (int r = threadIdx.x; r < it; r += blockDim.x) bsm[r] = d.beta[r];
    __syncthreads();
    for (int i = it - 1; i >= 0; --i) {
        const double *col = d.H + static_cast<size_t>(i) * d.ldh;
        const double yi = bsm[i] / col[i];
        __syncthreads();
        for (int r = threadIdx.x; r < i; r += blockDim.x) bsm[r] -= col[r] * yi;
        if (threadIdx.x == 0) d.y[i] = yi;
        __syncthreads();
    }
    for (int i = it + threadIdx.x; i < d.max_iter; i += blockDim.x) d.y[i] = 0.0;
    if (threadIdx.x == 0 && d.iter_log_cap > 0) d.iter_log[ctl->nt % d.iter_log_cap] = it;
}

// t = sum_{j < it} y_j V_j with V = Z (flexible) or Q; same 2-D layout as update_kernel.
__global__ void __launch_bounds__(kUpdRows * kUpdGroups) combine_kernel(SimDev d) {
    __shared__ double part[kUpdGroups][kUpdRows];
    const GmresCtl *ctl = d.ctl;
    const bool iterated = ctl->status == kGmresConverged || ctl->status == kGmresMaxIter;
    const int it = iterated ? ctl->iters : 0;
    const double *V = d.flexible ? d.Z : d.Q;
    const int r = threadIdx.x % kUpdRows, g = threadIdx.x / kUpdRows;
    for (int base = blockIdx.x * kUpdRows; base < d.n; base += gridDim.x * kUpdRows) {
        const int i = base + r;
        double a0 = 0.0, a1 = 0.0;
        if (i < d.n) {
            int j = g;
            for (; j + kUpdGroups < it; j += 2 * kUpdGroups) {
                a0 += d.y[j] * V[static_cast<size_t>(j) * d.ldq + i];
                a1 += d.y[j + kUpdGroups] * V[static_cast<size_t>(j + kUpdGroups) * d.ldq + i];
            }
            for (; j < it; j += kUpdGroups) a0 += d.y[j] * V[static_cast<size_t>(j) * d.ldq + i];
        }
        part[g][r] = a0 + a1;
        __syncthreads();
        if (g == 0 && i < d.n) {
            double acc = 0.0;
            for (int gg = 0; gg < kUpdGroups; ++gg) acc += part[gg][r];
            d.t[i] = acc;
        }
        __syncthreads();
    }
}

// sol = (guess or 0) + P^{-1} t (or t when flexible); unpack the rates into the
// filament state (mobility_solver.cpp:2550-2644).  One block per filament.
__global__ void finish_kernel(SimDev d) {
    extern __shared__ double smp[];
    __shared__ double sm32[32];
    const int m = blockIdx.x;
    const GmresCtl *ctl = d.ctl;
    const int st = ctl->status;
    const int nb = 3 * d.nseg, off = nb * m;
    const bool iterated = st == kGmresConverged || st == kGmresMaxIter;
    if (iterated && !d.flexible) precond_block(d, m, d.t, d.t, smp, sm32);
    __syncthreads();
    const bool reset = st == kGmresZeroRhs || (iterated && ctl->zero_guess);
    const bool add = iterated;
    for (int j = threadIdx.x; j < nb; j += blockDim.x) {
        const double base = reset ? 0.0 : d.sol[off + j];
        d.sol[off + j] = base + (add ? d.t[off + j] : 0.0);
    }
    if (threadIdx.x == 0) {
        if (d.po >= 0) {
            const double base = reset ? 0.0 : d.sol[d.po + m];
            d.sol[d.po + m] = base + (add ? d.t[d.po + m] : 0.0);
            d.phase_dot[m] = d.sol[d.po + m];
        }
        if (d.ao >= 0) {
            const double base = reset ? 0.0 : d.sol[d.ao + m];
            d.sol[d.ao + m] = base + (add ? d.t[d.ao + m] : 0.0);
            d.angle_dot[m] = d.sol[d.ao + m];
        }
    }
}

__global__ void set_nt_kernel(GmresCtl *ctl, int nt) {
    if (threadIdx.x == 0 && blockIdx.x == 0) ctl->nt = nt;
}

// f4 = float(v[0:3N]) for the pair kernel.
__global__ void pack_forces_kernel(SimDev d, const double *v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < d.N)
        d.f4[i] = make_float4(static_cast<float>(v[3 * i]), static_cast<float>(v[3 * i + 1]),
                              static_cast<float>(v[3 * i + 2]), 0.0f);
}

}  // namespace cufil

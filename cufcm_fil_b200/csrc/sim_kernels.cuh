// sim_kernels.cuh -- device side of the implicit prescribed-cilia step, for a
// batch of independent filament arrays (one array is a batch of one).
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
//
// Batch layout.  Filaments and segments are numbered across the batch (array
// by array); per-filament and per-segment state is indexed by those global
// numbers.  Saddle-point vectors of all arrays are concatenated, each array
// starting on a 256-row boundary (ArrayInfo::voff), so one batch vector holds
// every array's [3N lambda | F phase rates | F angle rates] block, and the
// Krylov basis stores basis vector j of every array in row j of Q
// (Q[j * ldq + row]).  Each array has its own GMRES control record,
// Hessenberg matrix, rotations and right-hand side.  Every GMRES iteration of
// the batch advances all running arrays together (they share the basis index
// k); arrays that stopped are masked out (active[b] = 0) of every kernel.
//
// One thread block per filament for all per-filament work.  Reductions that
// span blocks write partials; the block that makes the last arrival on an
// array's ticket combines that array's partials in a fixed order
// (deterministic, no spin waits), and the last array to finish a pass updates
// the loop state and the graph's loop condition.
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

// GMRES state of one array.
struct GmresCtl {
    int iters;        // Arnoldi iterations done
    int status;       // GmresStatus
    int zero_guess;   // initial guess discarded (start from 0)
    unsigned int counter;  // arrivals on this array's ticket
    double norm_rhs, beta0, relres;
    double inv_scale; // normalisation pending for the newest basis vector
};

// Loop state shared by the batch.
struct LoopCtl {
    int nt;           // time-step index of the step being solved
    int k;            // index of the newest basis vector (shared by every running array)
    int cond;         // loop condition (mirrors the graph conditional)
    int running;      // arrays still iterating
    unsigned int counter;  // arrays that finished the current pass
    int pad[3];
};

// Placement of one array in the batch.
struct ArrayInfo {
    int F, N, n;          // filaments, segments, system size
    int fil0, seg0;       // first filament / segment in the batch numbering
    int po, ao;           // local rows of the phase / angle rate blocks (-1 if absent)
    int max_iter;         // GMRES iteration cap
    int nb;               // 32-segment tiles = mobility partials per segment
    int chunk0, nchunk;   // dot-product row chunks: first (batch numbering), count
    long long voff;       // first row in the batch vectors (a multiple of kRowPad)
    long long vlen;       // rows reserved for the array (n rounded up to kRowPad)
    long long poff;       // first mobility partial
};

struct SimDev {
    int B, F, nseg, N;        // arrays, filaments, segments per filament, segments (batch totals)
    long long nrows;          // rows of a batch vector (padded)
    long long ldq;            // basis stride (>= nrows)
    int mi_max;               // largest iteration cap in the batch
    int ldh;                  // Hessenberg leading dimension (mi_max + 1)
    long long hstride;        // Hessenberg block per array
    int sstride;              // small per-array vectors (cs, sn, beta, h1, h2, y)
    int flexible;             // keep Z = P^{-1} Q (nonlinear preconditioner)
    int precond;              // 0: none, 1: block-diagonal (also the fallback of the patch preconditioner)
    int line;                 // line-patch preconditioner (patch_kernels.cuh) applied between kernels
    int learned;              // block-diagonal + network correction (learned_kernels.cuh), flexible GMRES
    const int *nbr;           // [F][2] neighbours of each filament along its lattice line (-1: none)
    float *lx, *ly, *lscale;  // network input [F][lin], output [F][lout], residual scale [F]
    int lin, lout;            // feature and correction widths
    double lalpha;            // weight of the network correction (chosen by validation; 1 by default)
    int dyn_phase, dyn_angle; // rate blocks present
    int rhs_given;            // solve of a caller's RHS (already in rhs): no RHS assembly, no iteration log
    int epi_fil_rows;         // the saddle epilogue also writes the filament rows of A v (line patches)
    int s_rows, s_cols;       // arclength table (0 rows: bisection)
    int n_phase_refs, n_angle_refs;
    int dots_chunk, C_tot;
    double dt, L, spring, tol, s_tol;
    double R[9];              // filament frame (row-major)
    const double *Rfil;       // per-filament frames [F][9] (a body's cilia); null: every filament uses R
    BeatCoeffs beat;
    const ArrayInfo *arr;     // [B]
    const int *fil_arr;       // array of each filament [F]
    const int *chunk_arr;     // array of each dot-product chunk [C_tot]
    const int *rb_arr;        // array of each 32-row unit of a batch vector [nrows / 32]
    int *active;              // [B] array still iterating
    const double *s_table, *phase_refs, *angle_refs, *omega0, *base;
    double *phase, *angle, *phase_dot, *angle_dot;
    float4 *x4;               // segment centres for the pair kernel
    double *xd, *kp, *ka;     // centres and velocity directions [3N]
    double *s_cur;            // arclength parameters of the current step [N]
    double *gram;             // per filament (c11, c22, c12)
    double *rhs, *sol, *w, *z, *t;   // batch vectors [nrows]
    double *Q, *Z;            // bases [(mi_max + 1) * ldq]
    double *H, *cs, *sn, *beta, *h1, *h2, *y;   // per array, strides hstride / sstride
    double *dots_partial, *norm_partial;
    float4 *f4;               // forces for the pair kernel
    const float4 *partial;    // mobility partials, per array [N][nb]
    GmresCtl *ctl;            // [B]
    LoopCtl *lc;
    int *iter_log;            // GMRES iterations of each step, [B][iter_log_cap] rings
    int iter_log_cap;
};

constexpr double kSegMobInv = 6.0 * 3.14159265358979323846;  // 6 pi mu a, mu = a = 1
constexpr int kRowUnit = 32;   // granularity of the row -> array table
constexpr int kRowPad = 256;   // every array's rows start on a multiple of this (largest update tile)

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

// Called by every thread of a block after the block's partial was written:
// returns true in every thread of the block whose arrival is number `total`
// on `counter` (global writes of all arrivals fenced before).  That block must
// reset the counter.  Safe to call repeatedly in one kernel.
__device__ __forceinline__ bool arrive_last(unsigned int *counter, unsigned int total, int *sm_flag) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) *sm_flag = (atomicAdd(counter, 1u) == total - 1u) ? 1 : 0;
    __syncthreads();
    const bool last = *sm_flag != 0;
    if (last) __threadfence();
    return last;
}

__device__ __forceinline__ void set_loop(cudaGraphConditionalHandle h, LoopCtl *lc, int cond) {
    lc->cond = cond;
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

// Rows of filament m in the batch vectors.
struct FilRows {
    int b;            // array
    int lm;           // filament index within the array
    long long lam;    // first lambda row (batch numbering)
    long long pr, ar; // phase / angle rate rows (batch numbering, -1 if absent)
    int ks;           // first entry in the per-segment [3N] arrays (xd, kp, ka)
};

__device__ __forceinline__ FilRows fil_rows(const SimDev &d, int m) {
    FilRows r;
    r.b = d.fil_arr[m];
    const ArrayInfo &a = d.arr[r.b];
    r.lm = m - a.fil0;
    r.lam = a.voff + 3LL * d.nseg * r.lm;
    r.pr = a.po >= 0 ? a.voff + a.po + r.lm : -1;
    r.ar = a.ao >= 0 ? a.voff + a.ao + r.lm : -1;
    r.ks = 3 * d.nseg * m;
    return r;
}

// Filament rows of the saddle product, out[pr] = -K_phase^T lambda_m and
// out[ar] = -K_angle^T lambda_m (mobility_solver.cpp:2000-2060), for filament m.
// Called by the kernels that produce the vector v (all threads of the block).
__device__ void filament_rows(const SimDev &d, const FilRows &fr, const double *v, double *out, double *sm32) {
    if (!d.dyn_phase && !d.dyn_angle) return;
    const int nb = 3 * d.nseg;
    double dp = 0.0, da = 0.0;
    for (int j = threadIdx.x; j < nb; j += blockDim.x) {
        dp += d.kp[fr.ks + j] * v[fr.lam + j];
        da += d.ka[fr.ks + j] * v[fr.lam + j];
    }
    dp = block_sum(dp, sm32);
    da = block_sum(da, sm32);
    if (threadIdx.x == 0) {
        if (fr.pr >= 0) out[fr.pr] = -dp;
        if (fr.ar >= 0) out[fr.ar] = -da;
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

// Start of a step: records the step index (nt >= 0) and marks every array
// active (the prologue works on all arrays; residual_decide then masks the
// finished ones).  Also clears every ticket.
__global__ void step_begin_kernel(SimDev d, int nt) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (nt >= 0) d.lc->nt = nt;
        d.lc->running = d.B;
        d.lc->counter = 0;
    }
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < d.B; b += gridDim.x * blockDim.x) {
        d.active[b] = 1;
        d.ctl[b].counter = 0;
    }
}

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
        if (d.lc->nt > 0) {
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
        if (!isfinite(idx)) idx = 0.0;  // non-finite phase: the shape is NaN anyway; keep the index in range
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
    const double *R = d.Rfil ? d.Rfil + 9 * m : d.R;
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
    if (!isfinite(x)) return x - x;  // non-finite phase: NaN, and no table index is formed
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
// the initial residual; ||rhs|| of each array into its ctl by the block that
// arrives last for that array.
__global__ void rhs_kernel(SimDev d) {
    __shared__ double sm32[32];
    __shared__ int last;
    const int m = blockIdx.x;
    const FilRows fr = fil_rows(d, m);
    const int nb = 3 * d.nseg;
    double ss = 0.0;
    const bool lam_rows_zero = d.dyn_phase;
    for (int j = threadIdx.x; j < nb; j += blockDim.x) {
        double v;
        if (d.rhs_given) {
            v = d.rhs[fr.lam + j];
        } else {
            v = lam_rows_zero ? 0.0 : d.phase_dot[m] * d.kp[fr.ks + j];
            d.rhs[fr.lam + j] = v;
        }
        ss += v * v;
    }
    for (int k = threadIdx.x; k < d.nseg; k += blockDim.x) {
        const long long r = fr.lam + 3 * k;
        d.f4[m * d.nseg + k] = make_float4(static_cast<float>(d.sol[r]), static_cast<float>(d.sol[r + 1]),
                                           static_cast<float>(d.sol[r + 2]), 0.0f);
    }
    if (threadIdx.x == 0 && d.rhs_given) {
        if (fr.ar >= 0) ss += d.rhs[fr.ar] * d.rhs[fr.ar];
        if (fr.pr >= 0) ss += d.rhs[fr.pr] * d.rhs[fr.pr];
    } else if (threadIdx.x == 0) {
        const double w0 = d.omega0[m] * 0.5 / 3.14159265358979323846;
        if (fr.ar >= 0) {
            double q_angle = cyclic_spline(d.phase[m], d.angle_refs, d.n_angle_refs) * w0;
            q_angle -= d.spring * d.omega0[m] * d.L * d.L * d.L * d.angle[m];
            d.rhs[fr.ar] = -q_angle;
            ss += q_angle * q_angle;
        }
        if (fr.pr >= 0) {
            const double q_phase = cyclic_spline(d.phase[m], d.phase_refs, d.n_phase_refs) * w0;
            d.rhs[fr.pr] = -q_phase;
            ss += q_phase * q_phase;
        }
    }
    ss = block_sum(ss, sm32);
    if (threadIdx.x == 0) d.norm_partial[m] = ss;
    filament_rows(d, fr, d.sol, d.w, sm32);  // filament rows of A x0 for the initial residual
    const ArrayInfo &a = d.arr[fr.b];
    if (arrive_last(&d.ctl[fr.b].counter, a.F, &last)) {
        double acc = 0.0;  // the filaments' partials, summed by the whole block in a fixed order
        for (int q = threadIdx.x; q < a.F; q += blockDim.x) acc += __ldcg(&d.norm_partial[a.fil0 + q]);
        acc = block_sum(acc, sm32);
        if (threadIdx.x == 0) {
            d.ctl[fr.b].norm_rhs = sqrt(acc);
            d.ctl[fr.b].counter = 0;
        }
    }
}

// Block-diagonal preconditioner of one filament (apply_preconditioner_new,
// PRESCRIBED_BODY_VELOCITIES branch): in -> out, may alias.  sm holds 3*nseg doubles.
__device__ void precond_block(const SimDev &d, int m, const FilRows &fr, const double *in, double *out, double *sm,
                              double *sm32) {
    __shared__ double coef[2];
    const int nb = 3 * d.nseg;
    const double *kp = d.kp + fr.ks, *ka = d.ka + fr.ks;
    double dp = 0.0, da = 0.0;
    for (int j = threadIdx.x; j < nb; j += blockDim.x) {
        const double r = (d.precond ? kSegMobInv : 1.0) * in[fr.lam + j];
        sm[j] = r;
        dp += kp[j] * r;
        da += ka[j] * r;
    }
    if (!d.precond) {
        __syncthreads();
        for (int j = threadIdx.x; j < nb; j += blockDim.x) out[fr.lam + j] = sm[j];
        if (threadIdx.x == 0) {
            if (fr.pr >= 0) out[fr.pr] = in[fr.pr];
            if (fr.ar >= 0) out[fr.ar] = in[fr.ar];
        }
        return;
    }
    if (fr.pr < 0 && fr.ar < 0) {
        __syncthreads();
        for (int j = threadIdx.x; j < nb; j += blockDim.x) out[fr.lam + j] = sm[j];
        return;
    }
    dp = block_sum(dp, sm32);
    da = block_sum(da, sm32);
    if (threadIdx.x == 0) {
        const double c11 = d.gram[3 * m], c22 = d.gram[3 * m + 1], c12 = d.gram[3 * m + 2];
        double ph = 0.0, an = 0.0;
        if (fr.pr >= 0 && fr.ar >= 0) {
            const double p = -in[fr.pr] - dp;
            const double a = -in[fr.ar] - da;
            const double det = c11 * c22 - c12 * c12;
            ph = (p * (c22 / det) + a * (-c12 / det)) / kSegMobInv;
            an = (p * (-c12 / det) + a * (c11 / det)) / kSegMobInv;
        } else if (fr.pr >= 0) {
            ph = (-in[fr.pr] - dp) / (c11 * kSegMobInv);
        } else {
            an = (-in[fr.ar] - da) / (c22 * kSegMobInv);
        }
        coef[0] = ph;
        coef[1] = an;
        if (fr.pr >= 0) out[fr.pr] = ph;
        if (fr.ar >= 0) out[fr.ar] = an;
    }
    __syncthreads();
    const double ph = coef[0], an = coef[1];
    for (int j = threadIdx.x; j < nb; j += blockDim.x) out[fr.lam + j] = sm[j] + kSegMobInv * (ph * kp[j] + an * ka[j]);
    __syncthreads();
}

// Standalone preconditioner application (host API and final update).
__global__ void precond_kernel(SimDev d, const double *in, double *out) {
    extern __shared__ double smp[];
    __shared__ double sm32[32];
    const int m = blockIdx.x;
    precond_block(d, m, fil_rows(d, m), in, out, smp, sm32);
}

// First kernel of a GMRES iteration: stores the normalised basis vector
// Q_k = src * inv_scale, applies P^{-1} into z (and Z_k when flexible) and
// packs the force part of z for the pair kernel.
//
// It also clears the loop condition: only a completed pass of the Givens
// bookkeeping of this iteration (update_kernel, final pass) re-arms it, so the
// loop cannot outlive a kernel that failed to run, and never passes max_iter.
__global__ void arnoldi_precond_kernel(SimDev d, cudaGraphConditionalHandle h) {
    extern __shared__ double smp[];
    __shared__ double sm32[32];
    const int m = blockIdx.x;
    if (m == 0 && threadIdx.x == 0) set_loop(h, d.lc, 0);
    const FilRows fr = fil_rows(d, m);
    if (!d.active[fr.b]) return;  // uniform over the block
    const int k = d.lc->k;
    if (k >= d.arr[fr.b].max_iter) return;  // defensive: the cap was reached
    const GmresCtl &c = d.ctl[fr.b];
    const double sc = c.inv_scale;
    const double *src = (k == 0 && c.zero_guess) ? d.rhs : d.w;  // r0 (residual kernel) or A z
    double *q = d.Q + static_cast<size_t>(k) * d.ldq;
    const int nb = 3 * d.nseg;
    for (int j = threadIdx.x; j < nb; j += blockDim.x) q[fr.lam + j] = src[fr.lam + j] * sc;
    if (threadIdx.x == 0) {
        if (fr.pr >= 0) q[fr.pr] = src[fr.pr] * sc;
        if (fr.ar >= 0) q[fr.ar] = src[fr.ar] * sc;
    }
    if (d.line || d.learned) {  // the next kernels read a fixed copy of Q_k
        for (int j = threadIdx.x; j < nb; j += blockDim.x) d.t[fr.lam + j] = q[fr.lam + j];
        if (threadIdx.x == 0) {
            if (fr.pr >= 0) d.t[fr.pr] = q[fr.pr];
            if (fr.ar >= 0) d.t[fr.ar] = q[fr.ar];
        }
        if (d.line) return;
    }
    __syncthreads();
    double *zout = d.flexible ? d.Z + static_cast<size_t>(k) * d.ldq : d.z;
    precond_block(d, m, fr, q, zout, smp, sm32);
    if (d.learned) return;  // the network's correction and the packing follow
    for (int kk = threadIdx.x; kk < d.nseg; kk += blockDim.x) {
        const long long r = fr.lam + 3 * kk;
        d.f4[m * d.nseg + kk] = make_float4(static_cast<float>(zout[r]), static_cast<float>(zout[r + 1]),
                                            static_cast<float>(zout[r + 2]), 0.0f);
    }
    if (d.flexible) {
        for (int j = threadIdx.x; j < nb; j += blockDim.x) d.z[fr.lam + j] = zout[fr.lam + j];
        if (threadIdx.x == 0) {
            if (fr.pr >= 0) d.z[fr.pr] = zout[fr.pr];
            if (fr.ar >= 0) d.z[fr.ar] = zout[fr.ar];
        }
    }
    // Block m read w only in its own rows (above), so it may now write the
    // filament rows of the new product A z.
    __syncthreads();
    filament_rows(d, fr, zout, d.w, sm32);
}

__global__ void filament_rows_kernel(SimDev d, const double *v, double *out) {
    __shared__ double sm32[32];
    filament_rows(d, fil_rows(d, blockIdx.x), v, out, sm32);
}

// Segment rows of out = A v (system_matrix_mult_new): reduces the mobility
// partials of v's force part, adds the FP64 wall self block and the -K rate
// terms.  A block of 8 warps takes 32 consecutive segments: lane l of every
// warp serves segment 32*blockIdx.x + l, warp w sums the partial slots
// s = w, w + 8, ... (the slot-major layout makes every warp load one
// contiguous run), and warp 0 combines the 8 sums in a fixed order.  The
// filament rows are written by the kernel that produced v.
constexpr int kEpiWarps = 8;
__global__ void __launch_bounds__(32 * kEpiWarps) saddle_epilogue_kernel(SimDev d, const double *v, double *out) {
    __shared__ double red[kEpiWarps][3][32];
    chain_wait();
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const int i = blockIdx.x * 32 + lane;
    int b = -1;
    if (i < d.N) {
        b = d.fil_arr[i / d.nseg];
        if (!d.active[b]) b = -1;
    }
    double u0 = 0.0, u1 = 0.0, u2 = 0.0;
    if (b >= 0) {
        const ArrayInfo &a = d.arr[b];
        const size_t n = a.N;
        const float4 *pt = d.partial + a.poff + (i - a.seg0);
        for (int s = wp; s < a.nb; s += kEpiWarps) {
            const float4 q = __ldcs(pt + s * n);
            u0 += q.x;
            u1 += q.y;
            u2 += q.z;
        }
    }
    red[wp][0][lane] = u0;
    red[wp][1][lane] = u1;
    red[wp][2][lane] = u2;
    if (d.epi_fil_rows && (d.dyn_phase || d.dyn_angle)) {
        // Filament rows out[pr] = -K_phase^T v_m, out[ar] = -K_angle^T v_m of the filaments whose first
        // segment lies in this block's 32 segments (each filament in exactly one block), one warp each.
        const int s0 = blockIdx.x * 32;
        const int m_end = min(d.F, (s0 + 32 + d.nseg - 1) / d.nseg);
        for (int m = (s0 + d.nseg - 1) / d.nseg + wp; m < m_end; m += kEpiWarps) {
            const FilRows fr = fil_rows(d, m);
            if (!d.active[fr.b]) continue;
            double dp = 0.0, da = 0.0;
            for (int j = lane; j < 3 * d.nseg; j += 32) {
                dp += d.kp[fr.ks + j] * v[fr.lam + j];
                da += d.ka[fr.ks + j] * v[fr.lam + j];
            }
            dp = warp_sum(dp);
            da = warp_sum(da);
            if (lane == 0) {
                if (fr.pr >= 0) out[fr.pr] = -dp;
                if (fr.ar >= 0) out[fr.ar] = -da;
            }
        }
    }
    __syncthreads();
    if (wp != 0 || b < 0) return;
    double u[3] = {0.0, 0.0, 0.0};
    for (int w = 0; w < kEpiWarps; ++w)
        for (int c = 0; c < 3; ++c) u[c] += red[w][c][lane];
    const ArrayInfo &a = d.arr[b];
    const int m = i / d.nseg;
    const int lm = m - a.fil0;
    const long long row = a.voff + 3LL * (i - a.seg0);
    const double vp = a.po >= 0 ? v[a.voff + a.po + lm] : 0.0;
    const double va = a.ao >= 0 ? v[a.voff + a.ao + lm] : 0.0;
    const double f[3] = {v[row], v[row + 1], v[row + 2]};
    wall_self_f64(d.xd[3 * i + 2], f, u);
    for (int c = 0; c < 3; ++c) out[row + c] = u[c] - vp * d.kp[3 * i + c] - va * d.ka[3 * i + c];
}

// End of a bookkeeping pass (one block, after every array of the pass
// arrived): refreshes the active mask from the arrays' status, sets the basis
// index for the next iteration and the loop condition.
__device__ void loop_pass_done(const SimDev &d, int next_k, cudaGraphConditionalHandle h, double *sm32) {
    double run = 0.0;
    for (int b = threadIdx.x; b < d.B; b += blockDim.x) {
        const int r = __ldcg(&d.ctl[b].status) == kGmresRunning ? 1 : 0;
        d.active[b] = r;
        run += r;
    }
    run = block_sum(run, sm32);
    if (threadIdx.x == 0) {
        const int nrun = static_cast<int>(run + 0.5);
        LoopCtl *lc = d.lc;
        lc->running = nrun;
        lc->counter = 0;
        lc->k = next_k;
        set_loop(h, lc, (nrun > 0 && next_k < d.mi_max) ? 1 : 0);
    }
}

// r = rhs - A sol into Q_0 (unnormalised); for each array the block arriving
// last decides how GMRES starts (mobility_solver.cpp:2216-2424): zero RHS,
// good initial guess, discard a poor guess, or iterate.
__global__ void residual_decide_kernel(SimDev d, cudaGraphConditionalHandle h) {
    __shared__ double sm32[32];
    __shared__ int last, last_all;
    const int m = blockIdx.x;
    const FilRows fr = fil_rows(d, m);
    const int nb = 3 * d.nseg;
    double ss = 0.0;
    // r0 = rhs - A x0 in place of A x0 in w (each entry read and written by the same thread):
    // the first basis vector is r0 / |r0|, stored into Q_0 by the next kernel.
    for (int j = threadIdx.x; j < nb; j += blockDim.x) {
        const double r = d.rhs[fr.lam + j] - d.w[fr.lam + j];
        d.w[fr.lam + j] = r;
        ss += r * r;
    }
    if (threadIdx.x == 0) {
        if (fr.pr >= 0) {
            const double r = d.rhs[fr.pr] - d.w[fr.pr];
            d.w[fr.pr] = r;
            ss += r * r;
        }
        if (fr.ar >= 0) {
            const double r = d.rhs[fr.ar] - d.w[fr.ar];
            d.w[fr.ar] = r;
            ss += r * r;
        }
    }
    ss = block_sum(ss, sm32);
    if (threadIdx.x == 0) d.norm_partial[m] = ss;
    const ArrayInfo &a = d.arr[fr.b];
    if (!arrive_last(&d.ctl[fr.b].counter, a.F, &last)) return;
    double acc = 0.0;  // the filaments' partials, summed by the whole block in a fixed order
    for (int q = threadIdx.x; q < a.F; q += blockDim.x) acc += __ldcg(&d.norm_partial[a.fil0 + q]);
    acc = block_sum(acc, sm32);
    if (threadIdx.x == 0) {
        GmresCtl *ctl = d.ctl + fr.b;
        ctl->counter = 0;
        const double nr = ctl->norm_rhs;
        double b0 = sqrt(acc);
        ctl->iters = 0;
        ctl->zero_guess = 0;
        if (!(nr == nr) || !(b0 == b0) || nr > 1.0e300 || b0 > 1.0e300) {
            ctl->status = kGmresNonFinite;
            ctl->relres = b0 / nr;
        } else if (nr == 0.0) {
            ctl->status = kGmresZeroRhs;
            ctl->relres = 0.0;
        } else if (b0 <= d.tol * nr) {
            ctl->status = kGmresGuessGood;
            ctl->relres = b0 / nr;
        } else {
            if (b0 > nr) {  // the initial guess is worse than zero
                ctl->zero_guess = 1;
                b0 = nr;
            }
            ctl->status = kGmresRunning;
            ctl->relres = b0 / nr;
        }
        ctl->beta0 = b0;
        d.beta[static_cast<size_t>(fr.b) * d.sstride] = b0;
        ctl->inv_scale = (b0 > 0.0) ? 1.0 / b0 : 0.0;
    }
    if (arrive_last(&d.lc->counter, d.B, &last_all)) loop_pass_done(d, 0, h, sm32);
}

// Work split used by the multi-array sweeps: the items [0, total) are cut
// into gridDim.x contiguous ranges of `per` items; a block arrives once on an
// array's ticket for each array its range meets, so the arrivals an array
// needs are the number of ranges that meet its items [i0, i1).
__device__ __forceinline__ unsigned int ranges_meeting(long long i0, long long i1, long long per) {
    return static_cast<unsigned int>((i1 - 1) / per - i0 / per + 1);
}

// Partial dot products <Q_j, w>, j <= k, over row chunks of the running
// arrays.  Items are ordered array by array (array b owns items
// (k+1)*[chunk0, chunk0 + nchunk), j-major inside), each block takes a
// contiguous range of them, and the block arriving last for an array sums its
// chunks of each j into h (one warp per j, a fixed order).  Loads are issued four at a time into
// independent accumulators so that each thread keeps several in flight.
__global__ void __launch_bounds__(256) dots_kernel(SimDev d, double *h) {
    __shared__ double sm32[32];
    __shared__ int last;
    chain_wait();
    const int k = d.lc->k;
    if (k >= d.mi_max) return;  // defensive, uniform over the grid
    const int C = d.C_tot;
    const long long K1 = k + 1;
    const long long items = K1 * C;
    const long long per = (items + gridDim.x - 1) / gridDim.x;
    const long long lo = static_cast<long long>(blockIdx.x) * per, hi = min(items, lo + per);
    const double *__restrict__ w = d.w;
    int cur = -1;
    bool cur_active = false;
    for (long long it = lo;; ++it) {
        const bool done = it >= hi;
        const int b = done ? -1 : d.chunk_arr[it / K1];
        if (done || b != cur) {
            if (cur >= 0 && cur_active) {  // close this block's share of array cur
                const ArrayInfo &a = d.arr[cur];
                const unsigned int need = ranges_meeting(K1 * a.chunk0, K1 * (a.chunk0 + a.nchunk), per);
                if (arrive_last(&d.ctl[cur].counter, need, &last)) {
                    // one warp per basis vector sums its chunks' partials in a fixed order
                    double *hb = h + static_cast<size_t>(cur) * d.sstride;
                    const int lane = threadIdx.x & 31;
                    for (int jj = threadIdx.x >> 5; jj <= k; jj += blockDim.x >> 5) {
                        double acc = 0.0;
                        for (int cc = lane; cc < a.nchunk; cc += 32)
                            acc += __ldcg(&d.dots_partial[static_cast<size_t>(jj) * C + a.chunk0 + cc]);
                        acc = warp_sum(acc);
                        if (lane == 0) hb[jj] = acc;
                    }
                    __syncthreads();
                    if (threadIdx.x == 0) d.ctl[cur].counter = 0;
                }
            }
            if (done) break;
            cur = b;
            cur_active = d.active[b] != 0;
        }
        if (!cur_active) continue;  // uniform over the block
        const ArrayInfo &a = d.arr[b];
        const long long tl = it - K1 * a.chunk0;
        const int j = static_cast<int>(tl / a.nchunk), c = static_cast<int>(tl - static_cast<long long>(j) * a.nchunk);
        const long long r0 = a.voff + static_cast<long long>(c) * d.dots_chunk;
        const long long r1 = a.voff + min(static_cast<long long>(a.n), static_cast<long long>(c + 1) * d.dots_chunk);
        const double *__restrict__ q = d.Q + static_cast<size_t>(j) * d.ldq;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
        long long i = r0 + threadIdx.x;
        for (; i + 3 * 256 < r1; i += 4 * 256) {
            a0 += q[i] * w[i];
            a1 += q[i + 256] * w[i + 256];
            a2 += q[i + 512] * w[i + 512];
            a3 += q[i + 768] * w[i + 768];
        }
        for (; i < r1; i += 256) a0 += q[i] * w[i];
        const double sum = block_sum((a0 + a1) + (a2 + a3), sm32);
        if (threadIdx.x == 0) d.dots_partial[static_cast<size_t>(j) * C + a.chunk0 + c] = sum;
    }
}

// Givens update of the least-squares problem of array b for column k
// (mobility_solver.cpp:2462-2515).  Called by every thread of one block: the
// column, the previous rotations and beta are staged in shared memory (gs:
// 3*(mi_max+2) doubles), thread 0 runs the sequential recurrence there, and
// the block writes the results back.
__device__ void givens_step(const SimDev &d, int b, int k, double qn, double *gs) {
    GmresCtl *ctl = d.ctl + b;
    const int max_iter = d.arr[b].max_iter;
    const size_t so = static_cast<size_t>(b) * d.sstride;
    double *Hs = gs, *cs = gs + (d.mi_max + 2), *sn = cs + (d.mi_max + 2);
    double *Hc = d.H + static_cast<size_t>(b) * d.hstride + static_cast<size_t>(k) * d.ldh;
    const double *h1 = d.h1 + so, *h2 = d.h2 + so;
    double *gcs = d.cs + so, *gsn = d.sn + so, *beta = d.beta + so;
    for (int j = threadIdx.x; j <= k; j += blockDim.x) Hs[j] = h1[j] + h2[j];
    for (int j = threadIdx.x; j < k; j += blockDim.x) {
        cs[j] = gcs[j];
        sn[j] = gsn[j];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        Hs[k + 1] = qn;
        for (int i = 1; i <= k; ++i) {
            const double t = cs[i - 1] * Hs[i - 1] + sn[i - 1] * Hs[i];
            Hs[i] = cs[i - 1] * Hs[i] - sn[i - 1] * Hs[i - 1];
            Hs[i - 1] = t;
        }
        const double a = Hs[k], bb = Hs[k + 1];
        double c, s;
        if (bb == 0.0) {
            c = 1.0;
            s = 0.0;
        } else if (fabs(bb) > fabs(a)) {
            const double t = a / bb;
            s = (bb > 0 ? 1.0 : -1.0) / sqrt(1.0 + t * t);
            c = t * s;
        } else {
            const double t = bb / a;
            c = (a > 0 ? 1.0 : -1.0) / sqrt(1.0 + t * t);
            s = t * c;
        }
        gcs[k] = c;
        gsn[k] = s;
        Hs[k] = c * a + s * bb;
        Hs[k + 1] = 0.0;
        const double bk = beta[k];
        beta[k + 1] = -s * bk;
        beta[k] = c * bk;
        const int it = k + 1;
        const double rel = fabs(-s * bk) / ctl->norm_rhs;
        ctl->iters = it;
        ctl->relres = rel;
        if (!(rel == rel) || !(qn == qn) || qn > 1.0e300) {
            ctl->status = kGmresNonFinite;
        } else if (rel <= d.tol) {
            ctl->status = kGmresConverged;
        } else if (it >= max_iter) {
            ctl->status = kGmresMaxIter;
        }
        ctl->inv_scale = qn > 0.0 ? 1.0 / qn : 0.0;
    }
    __syncthreads();
    for (int j = threadIdx.x; j <= k + 1; j += blockDim.x) Hc[j] = Hs[j];
}

// w -= sum_j h_j Q_j over the rows of the running arrays; in the final pass
// also ||w|| and, by the block arriving last for an array, that array's
// Givens step; the last array to finish closes the iteration.
// Tile = ROWS rows x (256/ROWS) basis-vector groups: each thread sums every
// G-th basis vector for one row with loads unrolled 4 deep, and the groups are
// combined in shared memory in a fixed order.  Each block takes a contiguous
// range of tiles (tiles never straddle arrays: arrays start on kRowPad rows).
template <int ROWS>
__global__ void __launch_bounds__(256) update_kernel(SimDev d, const double *h, int final_pass,
                                                     cudaGraphConditionalHandle hcond) {
    constexpr int G = 256 / ROWS;
    extern __shared__ double gsm[];  // Givens staging, 3*(mi_max+2) doubles (final pass)
    __shared__ double sm32[32];
    __shared__ double part[G][ROWS];
    __shared__ int last, last_all;
    __shared__ double qn;
    chain_wait();
    const int k = d.lc->k;
    if (k >= d.mi_max) return;  // defensive, uniform over the grid
    const int r = threadIdx.x % ROWS, g = threadIdx.x / ROWS;
    const long long ntiles = d.nrows / ROWS;
    const long long per = (ntiles + gridDim.x - 1) / gridDim.x;
    const long long lo = static_cast<long long>(blockIdx.x) * per, hi = min(ntiles, lo + per);
    int cur = -1;
    bool cur_active = false;
    double ss = 0.0;
    for (long long tile = lo;; ++tile) {
        const bool done = tile >= hi;
        const int b = done ? -1 : d.rb_arr[tile * (ROWS / kRowUnit)];
        if (done || b != cur) {
            if (final_pass && cur >= 0 && cur_active) {  // close this block's share of array cur
                const ArrayInfo &a = d.arr[cur];
                const long long t0 = a.voff / ROWS, t1 = (a.voff + a.vlen) / ROWS;
                const double tot = block_sum(ss, sm32);
                if (threadIdx.x == 0) d.norm_partial[max(lo, t0)] = tot;
                if (arrive_last(&d.ctl[cur].counter, ranges_meeting(t0, t1, per), &last)) {
                    double acc = 0.0;  // the blocks' partials, summed by the whole block in a fixed order
                    for (long long c = t0 / per + threadIdx.x; c <= (t1 - 1) / per; c += blockDim.x)
                        acc += __ldcg(&d.norm_partial[max(c * per, t0)]);
                    acc = block_sum(acc, sm32);
                    if (threadIdx.x == 0) {
                        d.ctl[cur].counter = 0;
                        qn = sqrt(acc);
                    }
                    __syncthreads();
                    givens_step(d, cur, k, qn, gsm);
                    if (arrive_last(&d.lc->counter, static_cast<unsigned int>(d.lc->running), &last_all))
                        loop_pass_done(d, k + 1, hcond, sm32);
                }
            }
            if (done) break;
            cur = b;
            cur_active = d.active[b] != 0;
            ss = 0.0;
        }
        if (!cur_active) continue;  // uniform over the block
        const ArrayInfo &a = d.arr[b];
        const long long i = tile * ROWS + r;
        const bool valid = i - a.voff < a.n;
        const double *hb = h + static_cast<size_t>(b) * d.sstride;
        const double wi = (valid && g == 0) ? d.w[i] : 0.0;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
        if (valid) {
            int j = g;
            for (; j + 3 * G <= k; j += 4 * G) {
                a0 += hb[j] * d.Q[static_cast<size_t>(j) * d.ldq + i];
                a1 += hb[j + G] * d.Q[static_cast<size_t>(j + G) * d.ldq + i];
                a2 += hb[j + 2 * G] * d.Q[static_cast<size_t>(j + 2 * G) * d.ldq + i];
                a3 += hb[j + 3 * G] * d.Q[static_cast<size_t>(j + 3 * G) * d.ldq + i];
            }
            for (; j <= k; j += G) a0 += hb[j] * d.Q[static_cast<size_t>(j) * d.ldq + i];
        }
        double acc = (a0 + a1) + (a2 + a3);
        if (G > 1) {
            part[g][r] = acc;
            __syncthreads();
            if (g == 0) {
                acc = 0.0;
                for (int gg = 0; gg < G; ++gg) acc += part[gg][r];
            }
            __syncthreads();
        }
        if (g == 0 && valid) {
            const double wn = wi - acc;
            d.w[i] = wn;
            ss += wn * wn;
        }
    }
}

// Back-substitution H y = beta for the iterations done (mobility_solver.cpp:2520-2537),
// one block per array, column oriented: after y_i is known every thread
// updates its own right-hand side entry with column i of H (contiguous), so
// each step is one coalesced sweep.
__global__ void __launch_bounds__(1024) backsub_kernel(SimDev d) {
    extern __shared__ double bsm[];  // [mi_max + 1]
    const int b = blockIdx.x;
    const GmresCtl *ctl = d.ctl + b;
    const size_t so = static_cast<size_t>(b) * d.sstride;
    const double *H = d.H + static_cast<size_t>(b) * d.hstride;
    double *y = d.y + so;
    const bool iterated = ctl->status == kGmresConverged || ctl->status == kGmresMaxIter;
    const int it = iterated ? ctl->iters : 0;
    for (int r = threadIdx.x; r < it; r += blockDim.x) bsm[r] = d.beta[so + r];
    __syncthreads();
    for (int i = it - 1; i >= 0; --i) {
        const double *col = H + static_cast<size_t>(i) * d.ldh;
        const double yi = bsm[i] / col[i];
        __syncthreads();
        for (int r = threadIdx.x; r < i; r += blockDim.x) bsm[r] -= col[r] * yi;
        if (threadIdx.x == 0) y[i] = yi;
        __syncthreads();
    }
    for (int i = it + threadIdx.x; i < d.mi_max; i += blockDim.x) y[i] = 0.0;
    if (threadIdx.x == 0 && d.iter_log_cap > 0 && !d.rhs_given)
        d.iter_log[static_cast<size_t>(b) * d.iter_log_cap + d.lc->nt % d.iter_log_cap] = it;
}

// t = sum_{j < it} y_j V_j with V = Z (flexible) or Q, for every array that
// iterated; same tiles and ranges as update_kernel.
template <int ROWS>
__global__ void __launch_bounds__(256) combine_kernel(SimDev d) {
    constexpr int G = 256 / ROWS;
    __shared__ double part[G][ROWS];
    const double *V = d.flexible ? d.Z : d.Q;
    const int r = threadIdx.x % ROWS, g = threadIdx.x / ROWS;
    const long long ntiles = d.nrows / ROWS;
    const long long per = (ntiles + gridDim.x - 1) / gridDim.x;
    const long long lo = static_cast<long long>(blockIdx.x) * per, hi = min(ntiles, lo + per);
    for (long long tile = lo; tile < hi; ++tile) {
        const int b = d.rb_arr[tile * (ROWS / kRowUnit)];
        const GmresCtl *ctl = d.ctl + b;
        const bool iterated = ctl->status == kGmresConverged || ctl->status == kGmresMaxIter;
        const int it = iterated ? ctl->iters : 0;
        if (it == 0) continue;  // uniform over the block; t is not read for this array
        const ArrayInfo &a = d.arr[b];
        const long long i = tile * ROWS + r;
        const bool valid = i - a.voff < a.n;
        const double *y = d.y + static_cast<size_t>(b) * d.sstride;
        double a0 = 0.0, a1 = 0.0;
        if (valid) {
            int j = g;
            for (; j + G < it; j += 2 * G) {
                a0 += y[j] * V[static_cast<size_t>(j) * d.ldq + i];
                a1 += y[j + G] * V[static_cast<size_t>(j + G) * d.ldq + i];
            }
            for (; j < it; j += G) a0 += y[j] * V[static_cast<size_t>(j) * d.ldq + i];
        }
        double acc = a0 + a1;
        if (G > 1) {
            part[g][r] = acc;
            __syncthreads();
            if (g == 0) {
                acc = 0.0;
                for (int gg = 0; gg < G; ++gg) acc += part[gg][r];
            }
            __syncthreads();
        }
        if (g == 0 && valid) d.t[i] = acc;
    }
}

// sol = (guess or 0) + P^{-1} t (or t when flexible); unpack the rates into the
// filament state (mobility_solver.cpp:2550-2644).  One block per filament.
__global__ void finish_kernel(SimDev d) {
    extern __shared__ double smp[];
    __shared__ double sm32[32];
    const int m = blockIdx.x;
    const FilRows fr = fil_rows(d, m);
    const GmresCtl *ctl = d.ctl + fr.b;
    const int st = ctl->status;
    const int nb = 3 * d.nseg;
    const bool iterated = st == kGmresConverged || st == kGmresMaxIter;
    if (iterated && !d.flexible && !d.line) precond_block(d, m, fr, d.t, d.t, smp, sm32);
    __syncthreads();
    const double *dx = (d.line && !d.flexible) ? d.z : d.t;  // the patch preconditioner left P^-1 t in z
    const bool reset = st == kGmresZeroRhs || (iterated && ctl->zero_guess);
    const bool add = iterated;
    for (int j = threadIdx.x; j < nb; j += blockDim.x) {
        const double base = reset ? 0.0 : d.sol[fr.lam + j];
        d.sol[fr.lam + j] = base + (add ? dx[fr.lam + j] : 0.0);
    }
    if (threadIdx.x == 0) {
        if (fr.pr >= 0) {
            const double base = reset ? 0.0 : d.sol[fr.pr];
            d.sol[fr.pr] = base + (add ? dx[fr.pr] : 0.0);
            d.phase_dot[m] = d.sol[fr.pr];
        }
        if (fr.ar >= 0) {
            const double base = reset ? 0.0 : d.sol[fr.ar];
            d.sol[fr.ar] = base + (add ? dx[fr.ar] : 0.0);
            d.angle_dot[m] = d.sol[fr.ar];
        }
    }
}

// Segment positions and constraint forces of the batch's first array in the
// reference's host layouts (x_segs [3N], f_segs [6N] with zero torques), FP32.
__global__ void segments_out_kernel(SimDev d, float *x, float *f) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const ArrayInfo &a = d.arr[0];
    if (i >= a.N) return;
    const int g = a.seg0 + i;
    const long long row = a.voff + 3LL * i;
    for (int c = 0; c < 3; ++c) {
        x[3 * i + c] = static_cast<float>(d.xd[3 * g + c]);
        f[6 * i + c] = static_cast<float>(d.sol[row + c]);
        f[6 * i + 3 + c] = 0.0f;
    }
}

// f4 = float(force rows of v) for the pair kernel, one thread per segment.
__global__ void pack_forces_kernel(SimDev d, const double *v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.N) return;
    const int m = i / d.nseg;
    const ArrayInfo &a = d.arr[d.fil_arr[m]];
    const long long row = a.voff + 3LL * (i - a.seg0);
    d.f4[i] = make_float4(static_cast<float>(v[row]), static_cast<float>(v[row + 1]), static_cast<float>(v[row + 2]),
                          0.0f);
}

}  // namespace cufil

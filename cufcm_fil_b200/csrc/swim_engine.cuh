// swim_engine.cuh -- cf_swim: one free rigid body carrying prescribed cilia,
// the reference's swimmer path (PRESCRIBED_CILIA with a body whose motion is
// solved for: BODY_VELOCITY_TYPE 0, BODY_OR_SURFACE_TYPE 2).  Included by sim.cu,
// whose beat kinematics it shares.
//
// Per step (cilia_sim_main.cu:405-716 with swimmer::initial_guess, swimmer.cpp:433-466):
//   body frame      filament frames q_body * q_ref (the filaments' own quaternions follow
//                   the body's rotation increments, filament.cpp:653-666), bases and blob
//                   positions from the body-frame references (swimmer.cpp:440-458);
//   kinematics      the Fulford-Blake beat in each filament's frame (kinematics_kernel);
//   precon matrix   swimmer::make_precon_mat (swimmer.cpp:1175-1349), the 6x6 body Schur
//                   matrix, on the host in FP64 and inverted there;
//   RHS             -q_phase, -q_angle rows (mobility_solver.cpp:284-420), zero elsewhere;
//   solve           right-preconditioned GMRES on the saddle system
//                   [3N lambda | 3B blob forces | V, Omega | N_fil phase rates | N_fil angle rates]
//                   (mobility_solver.cpp:2187-2669) with
//                     A: system_matrix_mult_new's body branch (:1887-2105): unbounded RPY over
//                        segments and blobs together, minus K V for every particle, the body's
//                        force and torque balance rows, and the filament rate rows;
//                     P: apply_preconditioner_new's body branch (:1244-1475);
//   body update     x += dt V, q = lie_exp(dt Omega) q (cilia_sim_main.cu:700-716).
// The Krylov vectors live on the device in FP64; the Hessenberg and Givens
// bookkeeping runs on the host (classical Gram-Schmidt with one
// re-orthogonalisation, one synchronisation per iteration).  The pair products
// are the FP32 tile kernel with compensated sums (rpy_kernels.cu).
#pragma once

struct cf_swim {
    cf_swim_config cfg{};
    int device = 0, num_sms = CF_B200_SMS;
    cudaStream_t stream = nullptr;
    int F = 0, nseg = 0, N = 0, B = 0, n = 0, o_blob = 0, o_body = 0, o_phase = 0, o_angle = 0, max_iter = 0;
    cufil::SimDev d{};  // kinematics state (phases, frames, positions, velocity directions)
    std::vector<double> qref;    // [F][4] filament frames in the body frame (scalar first)
    std::vector<double> fil_ref;  // [3F] filament bases in the body frame
    std::vector<double> blob_ref; // [3B] blobs in the body frame
    double bx[3] = {0, 0, 0}, bq[4] = {1, 0, 0, 0}, bv[6] = {0, 0, 0, 0, 0, 0};
    double *Rfil = nullptr, *xb = nullptr, *body = nullptr, *aux = nullptr, *kinv = nullptr, *gram_h = nullptr;
    float4 *x4all = nullptr, *f4all = nullptr, *scratch = nullptr;
    float *u = nullptr;
    size_t scratch_cap = 0;
    int *err = nullptr;
    double *rhs = nullptr, *sol = nullptr, *w = nullptr, *z = nullptr, *t = nullptr, *Q = nullptr, *hb = nullptr;
    double *dpart = nullptr;          // chunk partials of swim_dots_kernel [(max_iter + 1) * kSwimChunks]
    unsigned int *dcount = nullptr;   // its arrival counter (zero between launches)
    int last_iters = 0, last_status = CF_OK;
    double last_relres = 0.0;
    bool stepped = false;
    std::vector<void *> allocations;
};

namespace cufil {
namespace swim {

// ------------------------------------------------------------ quaternions
// Host FP64 quaternions (scalar first), as src/general/quaternion.cpp defines them.
struct Quat {
    double s, v[3];
};

Quat qmul(const Quat &a, const Quat &b) {  // operator*= (quaternion.cpp:104-118)
    Quat r;
    r.s = a.s * b.s - (a.v[0] * b.v[0] + a.v[1] * b.v[1] + a.v[2] * b.v[2]);
    r.v[0] = a.s * b.v[0] + b.s * a.v[0] + a.v[1] * b.v[2] - a.v[2] * b.v[1];
    r.v[1] = a.s * b.v[1] + b.s * a.v[1] + a.v[2] * b.v[0] - a.v[0] * b.v[2];
    r.v[2] = a.s * b.v[2] + b.s * a.v[2] + a.v[0] * b.v[1] - a.v[1] * b.v[0];
    return r;
}

void qnormalise(Quat &q) {  // normalise_in_place (:183-187)
    const double nrm = std::sqrt(q.s * q.s + q.v[0] * q.v[0] + q.v[1] * q.v[1] + q.v[2] * q.v[2]);
    q.s /= nrm;
    for (double &c : q.v) c /= nrm;
}

void qsqrt_ortho(Quat &q) {  // sqrt_in_place_ortho (:197-223), including its guard near -1
    if (q.s < -0.999999) {
        q.s = -0.9999999;
        q.s = std::sqrt(0.5 * (1.0 + q.s));
        const double temp = 2.0 * q.s;
        for (double &c : q.v) c /= temp;
        const double qn = std::sqrt(q.s * q.s + q.v[0] * q.v[0] + q.v[1] * q.v[1] + q.v[2] * q.v[2]);
        q.s *= qn;
        for (double &c : q.v) c /= qn;
    } else {
        q.s = std::sqrt(0.5 * (1.0 + q.s));
        const double temp = 2.0 * q.s;
        for (double &c : q.v) c /= temp;
    }
    qnormalise(q);
}

void qnormal(const Quat &q, double n[3]) {  // normal (:271-277)
    n[0] = 2.0 * (q.v[0] * q.v[1] - q.s * q.v[2]);
    n[1] = 1.0 - 2.0 * (q.v[0] * q.v[0] + q.v[2] * q.v[2]);
    n[2] = 2.0 * (q.v[1] * q.v[2] + q.s * q.v[0]);
}

void qrot(const Quat &q, double R[9]) {  // rot_mat (:305-345), row-major
    const double x = q.v[0], y = q.v[1], zc = q.v[2], s = q.s;
    R[0] = 1.0 - 2.0 * y * y - 2.0 * zc * zc;
    R[4] = 1.0 - 2.0 * x * x - 2.0 * zc * zc;
    R[8] = 1.0 - 2.0 * x * x - 2.0 * y * y;
    R[3] = 2.0 * x * y + 2.0 * s * zc;
    R[1] = 2.0 * x * y - 2.0 * s * zc;
    R[6] = 2.0 * x * zc - 2.0 * s * y;
    R[2] = 2.0 * x * zc + 2.0 * s * y;
    R[5] = 2.0 * y * zc - 2.0 * s * x;
    R[7] = 2.0 * y * zc + 2.0 * s * x;
}

Quat qlie_exp(const double u[3]) {  // lie_exp (:500-523)
    const double th = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    if (th < 1e-6) return Quat{1.0, {0.0, 0.0, 0.0}};
    const double cs = std::cos(0.5 * th), sn = std::sin(0.5 * th) / th;
    return Quat{cs, {sn * u[0], sn * u[1], sn * u[2]}};
}

// The frame of a filament whose base direction is dir in the body frame
// (filament.cpp:224-236, 368-400, 422-430 with TILT_ANGLE = 0): the rotation
// taking the reference x axis to dir, followed by the one that aligns the
// reference y axis with the polar direction (the projection of -e_z).
Quat filament_frame(const double *dir_in) {
    const double dn = std::sqrt(dir_in[0] * dir_in[0] + dir_in[1] * dir_in[1] + dir_in[2] * dir_in[2]);
    const double dir[3] = {dir_in[0] / dn, dir_in[1] / dn, dir_in[2] / dn};
    Quat qtemp{dir[0], {0.0, -dir[2], dir[1]}};
    qsqrt_ortho(qtemp);
    double bn[3];
    qnormal(qtemp, bn);
    double pol[3] = {0.0, 0.0, -1.0};
    const double dp = dir[0] * pol[0] + dir[1] * pol[1] + dir[2] * pol[2];
    for (int c = 0; c < 3; ++c) pol[c] -= dp * dir[c];
    const double np = std::sqrt(pol[0] * pol[0] + pol[1] * pol[1] + pol[2] * pol[2]);
    Quat q2{1.0, {0.0, 0.0, 0.0}};
    if (np > 0.0) {
        for (double &c : pol) c /= np;
        q2.s = pol[0] * bn[0] + pol[1] * bn[1] + pol[2] * bn[2];
        q2.v[0] = bn[1] * pol[2] - bn[2] * pol[1];
        q2.v[1] = bn[2] * pol[0] - bn[0] * pol[2];
        q2.v[2] = bn[0] * pol[1] - bn[1] * pol[0];
        qsqrt_ortho(q2);
    }
    return qmul(q2, qtemp);
}

// 6x6 inverse by Gauss-Jordan with partial pivoting (row-major, FP64); false if singular.
bool invert6(double *A) {
    double M[6][12];
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 12; ++j) M[i][j] = j < 6 ? A[6 * i + j] : (j - 6 == i ? 1.0 : 0.0);
    for (int c = 0; c < 6; ++c) {
        int p = c;
        for (int r = c + 1; r < 6; ++r)
            if (std::fabs(M[r][c]) > std::fabs(M[p][c])) p = r;
        if (M[p][c] == 0.0 || !std::isfinite(M[p][c])) return false;
        if (p != c)
            for (int j = 0; j < 12; ++j) std::swap(M[p][j], M[c][j]);
        const double inv = 1.0 / M[c][c];
        for (int j = 0; j < 12; ++j) M[c][j] *= inv;
        for (int r = 0; r < 6; ++r)
            if (r != c) {
                const double f = M[r][c];
                if (f != 0.0)
                    for (int j = 0; j < 12; ++j) M[r][j] -= f * M[c][j];
            }
    }
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) A[6 * i + j] = M[i][j + 6];
    return true;
}

// ------------------------------------------------------------ device side
constexpr double kSwimMobInv = 6.0 * 3.14159265358979323846;  // 6 pi mu a, mu = a = 1 (segments and blobs)

struct SwimParams {
    int F, nseg, N, B, o_blob, o_body, o_phase, o_angle;
    const double *xd, *kp, *ka, *gram;  // segment positions and velocity directions, per-filament (c11, c22, c12)
    const double *xb;                   // blob positions [3B]
    const double *body;                 // body centre [3]
    const double *aux;                  // per filament: v_phi, u_phi, v_theta, u_theta (12)
    const double *kinv;                 // inverse of the 6x6 body Schur matrix (row-major)
};

__device__ __forceinline__ void swim_diff(const SwimParams &p, int i, double r[3]) {
    const double *x = i < p.N ? p.xd + 3 * i : p.xb + 3 * (i - p.N);
    for (int c = 0; c < 3; ++c) r[c] = x[c] - p.body[c];
}

__device__ __forceinline__ long long swim_row(const SwimParams &p, int i) {
    return i < p.N ? 3LL * i : p.o_blob + 3LL * (i - p.N);
}

__global__ void swim_pack_positions_kernel(const float4 *seg, const double *xb, int N, int B, float4 *all) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) all[i] = seg[i];
    else if (i < N + B)
        all[i] = make_float4(static_cast<float>(xb[3 * (i - N)]), static_cast<float>(xb[3 * (i - N) + 1]),
                             static_cast<float>(xb[3 * (i - N) + 2]), 0.0f);
}

__global__ void swim_pack_forces_kernel(SwimParams p, const double *v, float4 *f4) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.N + p.B) return;
    const long long r = swim_row(p, i);
    f4[i] = make_float4(static_cast<float>(v[r]), static_cast<float>(v[r + 1]), static_cast<float>(v[r + 2]), 0.0f);
}

// Particle rows of A v: u - V - Omega x r, and for segments - phi_dot k_phi - theta_dot k_theta.
__global__ void swim_rows_kernel(SwimParams p, const double *v, const float *u, double *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.N + p.B) return;
    double r[3];
    swim_diff(p, i, r);
    const double *V = v + p.o_body, *W = v + p.o_body + 3;
    const double wr[3] = {W[1] * r[2] - W[2] * r[1], W[2] * r[0] - W[0] * r[2], W[0] * r[1] - W[1] * r[0]};
    const long long row = swim_row(p, i);
    double o[3];
    for (int c = 0; c < 3; ++c) o[c] = static_cast<double>(u[3 * i + c]) - V[c] - wr[c];
    if (i < p.N) {
        const int m = i / p.nseg;
        const double ph = v[p.o_phase + m], an = v[p.o_angle + m];
        for (int c = 0; c < 3; ++c) o[c] -= ph * p.kp[3 * i + c] + an * p.ka[3 * i + c];
    }
    for (int c = 0; c < 3; ++c) out[row + c] = o[c];
}

// Filament rows of A v: -K_phi^T lambda_m, -K_theta^T lambda_m (one block per filament).
__global__ void swim_fil_rows_kernel(SwimParams p, const double *v, double *out) {
    __shared__ double sm32[32];
    const int m = blockIdx.x;
    const int nb = 3 * p.nseg;
    double dp = 0.0, da = 0.0;
    for (int j = threadIdx.x; j < nb; j += blockDim.x) {
        const long long r = 3LL * m * p.nseg + j;
        dp += p.kp[r] * v[r];
        da += p.ka[r] * v[r];
    }
    dp = block_sum(dp, sm32);
    da = block_sum(da, sm32);
    if (threadIdx.x == 0) {
        out[p.o_phase + m] = -dp;
        out[p.o_angle + m] = -da;
    }
}

// Body rows of A v: minus the total force and torque (about the body centre) of every segment and blob (one block).
__global__ void swim_body_rows_kernel(SwimParams p, const double *v, double *out) {
    __shared__ double sm32[32];
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < p.N + p.B; i += blockDim.x) {
        double r[3];
        swim_diff(p, i, r);
        const double *f = v + swim_row(p, i);
        acc[0] += f[0];
        acc[1] += f[1];
        acc[2] += f[2];
        acc[3] += r[1] * f[2] - r[2] * f[1];
        acc[4] += r[2] * f[0] - r[0] * f[2];
        acc[5] += r[0] * f[1] - r[1] * f[0];
    }
    for (int c = 0; c < 6; ++c) {
        const double s = block_sum(acc[c], sm32);
        if (threadIdx.x == 0) out[p.o_body + c] = -s;
        __syncthreads();
    }
}

// The driving rows: -q_phase, -(q_angle - spring term) per filament (one thread each).
__global__ void swim_rhs_kernel(SwimParams p, SimDev d, double *rhs) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= p.F) return;
    const double w0 = d.omega0[m] * 0.5 / 3.14159265358979323846;
    double q_angle = cyclic_spline(d.phase[m], d.angle_refs, d.n_angle_refs) * w0;
    q_angle -= d.spring * d.omega0[m] * d.L * d.L * d.L * d.angle[m];
    const double q_phase = cyclic_spline(d.phase[m], d.phase_refs, d.n_phase_refs) * w0;
    rhs[p.o_phase + m] = -q_phase;
    rhs[p.o_angle + m] = -q_angle;
}

// ---- preconditioner (apply_preconditioner_new, body branch, mobility_solver.cpp:1244-1475)
// (1) M^-1 r_1 on the particle rows.
__global__ void swim_pc_scale_kernel(SwimParams p, const double *r, double *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.N + p.B) return;
    const long long row = swim_row(p, i);
    for (int c = 0; c < 3; ++c) out[row + c] = kSwimMobInv * r[row + c];
}

// (2) per filament: (-r_rate - K^T M^-1 r_1), through the filament's 2x2 C^-1 (one block per filament).
__global__ void swim_pc_fil1_kernel(SwimParams p, const double *r, double *out) {
    __shared__ double sm32[32];
    const int m = blockIdx.x;
    const int nb = 3 * p.nseg;
    double dp = 0.0, da = 0.0;
    for (int j = threadIdx.x; j < nb; j += blockDim.x) {
        const long long k = 3LL * m * p.nseg + j;
        dp += p.kp[k] * out[k];
        da += p.ka[k] * out[k];
    }
    dp = block_sum(dp, sm32);
    da = block_sum(da, sm32);
    if (threadIdx.x == 0) {
        const double ph = -r[p.o_phase + m] - dp, an = -r[p.o_angle + m] - da;
        const double c11 = p.gram[3 * m], c22 = p.gram[3 * m + 1], c12 = p.gram[3 * m + 2];
        const double det = c11 * c22 - c12 * c12;
        const double i11 = c22 / det, i22 = c11 / det, i12 = -c12 / det;
        out[p.o_phase + m] = i11 * ph + i12 * an;
        out[p.o_angle + m] = i12 * ph + i22 * an;
    }
}

// (3) the body: -r_2 - K^T M^-1 r_1 - the filaments' B terms, then the 6x6 solve (one block).
__global__ void swim_pc_body_kernel(SwimParams p, const double *r, double *out) {
    __shared__ double sm32[32];
    __shared__ double bsum[6];
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < p.N + p.B; i += blockDim.x) {
        double d3[3];
        swim_diff(p, i, d3);
        const double *f = out + swim_row(p, i);
        acc[0] += f[0];
        acc[1] += f[1];
        acc[2] += f[2];
        acc[3] += d3[1] * f[2] - d3[2] * f[1];
        acc[4] += d3[2] * f[0] - d3[0] * f[2];
        acc[5] += d3[0] * f[1] - d3[1] * f[0];
    }
    for (int m = threadIdx.x; m < p.F; m += blockDim.x) {
        const double ph = out[p.o_phase + m], an = out[p.o_angle + m];
        const double *a = p.aux + 12 * m;  // v_phi, u_phi, v_theta, u_theta
        for (int c = 0; c < 3; ++c) {
            acc[c] += ph * a[c] + an * a[6 + c];
            acc[3 + c] += ph * a[3 + c] + an * a[9 + c];
        }
    }
    for (int c = 0; c < 6; ++c) {
        const double s = block_sum(acc[c], sm32);
        if (threadIdx.x == 0) bsum[c] = -r[p.o_body + c] - s;
        __syncthreads();
    }
    if (threadIdx.x < 6) {
        double v = 0.0;
        for (int c = 0; c < 6; ++c) v += p.kinv[6 * threadIdx.x + c] * bsum[c];
        out[p.o_body + threadIdx.x] = v;
    }
}

// (4) the rates: divided by 6 pi mu a, minus C^-1 B^T of the body solution (one thread per filament).
__global__ void swim_pc_fil2_kernel(SwimParams p, double *out) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= p.F) return;
    const double c11 = p.gram[3 * m], c22 = p.gram[3 * m + 1], c12 = p.gram[3 * m + 2];
    const double det = c11 * c22 - c12 * c12;
    const double i11 = c22 / det, i22 = c11 / det, i12 = -c12 / det;
    const double *a = p.aux + 12 * m;
    const double *V = out + p.o_body, *W = out + p.o_body + 3;
    double vpV = 0, vtV = 0, upW = 0, utW = 0;
    for (int c = 0; c < 3; ++c) {
        vpV += a[c] * V[c];
        upW += a[3 + c] * W[c];
        vtV += a[6 + c] * V[c];
        utW += a[9 + c] * W[c];
    }
    const double ph = out[p.o_phase + m] / kSwimMobInv, an = out[p.o_angle + m] / kSwimMobInv;
    out[p.o_phase + m] = ph - (i11 * vpV + i12 * vtV + i11 * upW + i12 * utW);
    out[p.o_angle + m] = an - (i12 * vpV + i22 * vtV + i12 * upW + i22 * utW);
}

// (5) s1 = M^-1 (r_1 + K s_2) on the particle rows.
__global__ void swim_pc_add_kernel(SwimParams p, double *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.N + p.B) return;
    double r[3];
    swim_diff(p, i, r);
    const double *V = out + p.o_body, *W = out + p.o_body + 3;
    double k[3] = {V[0] + W[1] * r[2] - W[2] * r[1], V[1] + W[2] * r[0] - W[0] * r[2],
                   V[2] + W[0] * r[1] - W[1] * r[0]};
    if (i < p.N) {
        const int m = i / p.nseg;
        const double ph = out[p.o_phase + m], an = out[p.o_angle + m];
        for (int c = 0; c < 3; ++c) k[c] += ph * p.kp[3 * i + c] + an * p.ka[3 * i + c];
    }
    const long long row = swim_row(p, i);
    for (int c = 0; c < 3; ++c) out[row + c] += kSwimMobInv * k[c];
}

// ---- Krylov vector kernels (rows [0, n))
// h[j] = <Q_j, w> for j < k1 (with `root`, h[0] = sqrt(<w, w>) for Q = w, k1 = 1).  Block (c, j) sums the
// rows of chunk c with four independent accumulators; the block arriving last sums every j's chunks in a
// fixed order (part: k1 x kSwimChunks partials, counter: zero on entry, reset by that block).
constexpr int kSwimChunks = 16;
__global__ void __launch_bounds__(256) swim_dots_kernel(const double *Q, long long ldq, const double *w, int n,
                                                        double *part, unsigned int *counter, double *h, int root) {
    __shared__ double sm32[32];
    __shared__ int last;
    const int c = blockIdx.x, j = blockIdx.y;
    const int chunk = (n + kSwimChunks - 1) / kSwimChunks;
    const int r0 = c * chunk, r1 = min(n, r0 + chunk);
    const double *q = Q + static_cast<long long>(j) * ldq;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    int i = r0 + threadIdx.x;
    for (; i + 3 * 256 < r1; i += 4 * 256) {
        a0 += q[i] * w[i];
        a1 += q[i + 256] * w[i + 256];
        a2 += q[i + 512] * w[i + 512];
        a3 += q[i + 768] * w[i + 768];
    }
    for (; i < r1; i += 256) a0 += q[i] * w[i];
    const double sum = block_sum((a0 + a1) + (a2 + a3), sm32);
    if (threadIdx.x == 0) part[j * kSwimChunks + c] = sum;
    if (!arrive_last(counter, gridDim.x * gridDim.y, &last)) return;
    for (int jj = threadIdx.x; jj < static_cast<int>(gridDim.y); jj += blockDim.x) {
        double t = 0.0;
        for (int cc = 0; cc < kSwimChunks; ++cc) t += __ldcg(&part[jj * kSwimChunks + cc]);
        h[jj] = root ? sqrt(t) : t;
    }
    if (threadIdx.x == 0) *counter = 0;
}

// w -= sum_j h[j] Q_j (j < k1)
__global__ void swim_sub_basis_kernel(double *w, const double *Q, long long ldq, const double *h, int k1, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    for (int j = 0; j < k1; ++j) s += h[j] * Q[static_cast<long long>(j) * ldq + i];
    w[i] -= s;
}

// dst = a * src + b * dst2 (dst2 may alias dst; b = 0 ignores it)
__global__ void swim_axpby_kernel(double *dst, double a, const double *src, double b, const double *dst2, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    dst[i] = a * src[i] + (b != 0.0 ? b * dst2[i] : 0.0);
}

// t = sum_j y[j] Q_j (j < k)
__global__ void swim_combine_kernel(double *t, const double *Q, long long ldq, const double *y, int k, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    for (int j = 0; j < k; ++j) s += y[j] * Q[static_cast<long long>(j) * ldq + i];
    t[i] = s;
}

// ------------------------------------------------------------ host side
template <typename T>
int swim_alloc(cf_swim *h, T **p, size_t n) {
    *p = nullptr;
    void *q = nullptr;
    CF_CUDA(cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)));
    h->allocations.push_back(q);
    *p = static_cast<T *>(q);
    return CF_OK;
}

template <typename T>
int swim_upload(cf_swim *h, T **p, const T *host, size_t n) {
    CF_TRY(swim_alloc(h, p, n));
    if (host && n) CF_CUDA(cudaMemcpy(*p, host, n * sizeof(T), cudaMemcpyHostToDevice));
    return CF_OK;
}

SwimParams swim_params(const cf_swim *h) {
    SwimParams p{};
    p.F = h->F;
    p.nseg = h->nseg;
    p.N = h->N;
    p.B = h->B;
    p.o_blob = h->o_blob;
    p.o_body = h->o_body;
    p.o_phase = h->o_phase;
    p.o_angle = h->o_angle;
    p.xd = h->d.xd;
    p.kp = h->d.kp;
    p.ka = h->d.ka;
    p.gram = h->d.gram;
    p.xb = h->xb;
    p.body = h->body;
    p.aux = h->aux;
    p.kinv = h->kinv;
    return p;
}

int swim_grid(int n) { return std::max(1, (n + 255) / 256); }

// out = A v (system_matrix_mult_new, body branch)
int swim_matvec(cf_swim *h, const double *v, double *out) {
    cudaStream_t st = h->stream;
    const SwimParams p = swim_params(h);
    const int np = h->N + h->B;
    swim_pack_forces_kernel<<<swim_grid(np), 256, 0, st>>>(p, v, h->f4all);
    CF_CHECK_LAUNCH("swim_pack_forces_kernel");
    RpyBlockDesc d{};
    d.wall = 0;
    d.vd = 3;
    d.fd = 3;
    d.self_set = 0;
    d.xt = h->x4all;
    d.nt = np;
    d.at = 1.0f;
    d.xs = h->x4all;
    d.fs = h->f4all;
    d.ts = nullptr;
    d.ns = np;
    d.as = 1.0f;
    d.mu = 1.0f;
    CF_TRY(rpy_block_product(d, h->scratch, h->scratch_cap, h->err, h->u, 3, kOutWrite, h->num_sms, st));
    swim_rows_kernel<<<swim_grid(np), 256, 0, st>>>(p, v, h->u, out);
    CF_CHECK_LAUNCH("swim_rows_kernel");
    swim_fil_rows_kernel<<<h->F, 64, 0, st>>>(p, v, out);
    CF_CHECK_LAUNCH("swim_fil_rows_kernel");
    swim_body_rows_kernel<<<1, 1024, 0, st>>>(p, v, out);
    CF_CHECK_LAUNCH("swim_body_rows_kernel");
    return CF_OK;
}

// out = P r (apply_preconditioner_new, body branch)
int swim_precond(cf_swim *h, const double *r, double *out) {
    cudaStream_t st = h->stream;
    const SwimParams p = swim_params(h);
    const int np = h->N + h->B;
    swim_pc_scale_kernel<<<swim_grid(np), 256, 0, st>>>(p, r, out);
    CF_CHECK_LAUNCH("swim_pc_scale_kernel");
    swim_pc_fil1_kernel<<<h->F, 64, 0, st>>>(p, r, out);
    CF_CHECK_LAUNCH("swim_pc_fil1_kernel");
    swim_pc_body_kernel<<<1, 1024, 0, st>>>(p, r, out);
    CF_CHECK_LAUNCH("swim_pc_body_kernel");
    swim_pc_fil2_kernel<<<swim_grid(h->F), 256, 0, st>>>(p, out);
    CF_CHECK_LAUNCH("swim_pc_fil2_kernel");
    swim_pc_add_kernel<<<swim_grid(np), 256, 0, st>>>(p, out);
    CF_CHECK_LAUNCH("swim_pc_add_kernel");
    return CF_OK;
}

int swim_sync(cf_swim *h) {
    CF_CUDA(cudaStreamSynchronize(h->stream));
    int flags = 0;
    CF_CUDA(cudaMemcpy(&flags, h->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (flags) {
        CF_CUDA(cudaMemset(h->err, 0, sizeof(int)));
        return set_error(CF_TIMEOUT, "swim: a bounded device wait gave up (flags 0x%x)", flags);
    }
    return CF_OK;
}

// Body frame of the current body state: filament frames, bases and blob positions to the device
// (swimmer::initial_guess, swimmer.cpp:433-466; the filaments' quaternions follow the body's).
int swim_frames(cf_swim *h) {
    const int F = h->F, B = h->B;
    double Rb[9];
    const Quat qb{h->bq[0], {h->bq[1], h->bq[2], h->bq[3]}};
    qrot(qb, Rb);
    std::vector<double> R(9 * static_cast<size_t>(F)), base(3 * static_cast<size_t>(F)), xb(3 * static_cast<size_t>(B));
    for (int m = 0; m < F; ++m) {
        const Quat qr{h->qref[4 * m], {h->qref[4 * m + 1], h->qref[4 * m + 2], h->qref[4 * m + 3]}};
        qrot(qmul(qb, qr), &R[9 * m]);
        for (int c = 0; c < 3; ++c)
            base[3 * m + c] = h->bx[c] + Rb[3 * c] * h->fil_ref[3 * m] + Rb[3 * c + 1] * h->fil_ref[3 * m + 1] +
                              Rb[3 * c + 2] * h->fil_ref[3 * m + 2];
    }
    for (int k = 0; k < B; ++k)
        for (int c = 0; c < 3; ++c)
            xb[3 * k + c] = h->bx[c] + Rb[3 * c] * h->blob_ref[3 * k] + Rb[3 * c + 1] * h->blob_ref[3 * k + 1] +
                            Rb[3 * c + 2] * h->blob_ref[3 * k + 2];
    cudaStream_t st = h->stream;
    CF_CUDA(cudaMemcpyAsync(h->Rfil, R.data(), R.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    CF_CUDA(cudaMemcpyAsync(const_cast<double *>(h->d.base), base.data(), base.size() * sizeof(double),
                            cudaMemcpyHostToDevice, st));
    if (B) CF_CUDA(cudaMemcpyAsync(h->xb, xb.data(), xb.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    CF_CUDA(cudaMemcpyAsync(h->body, h->bx, 3 * sizeof(double), cudaMemcpyHostToDevice, st));
    CF_CUDA(cudaStreamSynchronize(st));  // the host vectors go out of scope
    return CF_OK;
}

// swimmer::make_precon_mat (swimmer.cpp:1175-1349, dynamic phase and angle) on the host in FP64, with the
// per-filament sums v_phi, u_phi, v_theta, u_theta that the preconditioner reuses.
int swim_precon_matrix(cf_swim *h) {
    const int F = h->F, nseg = h->nseg, N = h->N, B = h->B;
    std::vector<double> x(3 * static_cast<size_t>(N)), kp(3 * static_cast<size_t>(N)), ka(3 * static_cast<size_t>(N));
    cudaStream_t st = h->stream;
    CF_CUDA(cudaMemcpyAsync(x.data(), h->d.xd, x.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CF_CUDA(cudaMemcpyAsync(kp.data(), h->d.kp, kp.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CF_CUDA(cudaMemcpyAsync(ka.data(), h->d.ka, ka.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CF_CUDA(cudaStreamSynchronize(st));
    const double mob = kSwimMobInv;
    double K[36] = {0};
    const double eye = static_cast<double>(N) * mob + static_cast<double>(B) * mob;
    K[0] = K[7] = K[14] = eye;
    auto add_r = [&](const double *d3) {
        // rcross(d) (matrix.cpp:665-679): rcross(d) w = w x d
        const double rc[9] = {0.0, d3[2], -d3[1], -d3[2], 0.0, d3[0], d3[1], -d3[0], 0.0};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                K[6 * i + 3 + j] += mob * rc[3 * i + j];
                double rr = 0.0;
                for (int q = 0; q < 3; ++q) rr += rc[3 * i + q] * rc[3 * q + j];
                K[6 * (3 + i) + 3 + j] -= mob * rr;
            }
    };
    for (int i = 0; i < N; ++i) {
        const double d3[3] = {x[3 * i] - h->bx[0], x[3 * i + 1] - h->bx[1], x[3 * i + 2] - h->bx[2]};
        add_r(d3);
    }
    double Rb[9];
    qrot(Quat{h->bq[0], {h->bq[1], h->bq[2], h->bq[3]}}, Rb);
    for (int k = 0; k < B; ++k) {
        double d3[3];
        for (int c = 0; c < 3; ++c)
            d3[c] = Rb[3 * c] * h->blob_ref[3 * k] + Rb[3 * c + 1] * h->blob_ref[3 * k + 1] +
                    Rb[3 * c + 2] * h->blob_ref[3 * k + 2];
        add_r(d3);
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) K[6 * (3 + i) + j] = -K[6 * i + 3 + j];
    double C[36] = {0};
    std::vector<double> aux(12 * static_cast<size_t>(F));
    std::vector<double> gram(3 * static_cast<size_t>(F));
    for (int m = 0; m < F; ++m) {
        double c11 = 0, c22 = 0, c12 = 0, vp[3] = {0, 0, 0}, up[3] = {0, 0, 0}, vt[3] = {0, 0, 0}, ut[3] = {0, 0, 0};
        for (int k = 0; k < nseg; ++k) {
            const int i = m * nseg + k;
            const double *a = &kp[3 * i], *b = &ka[3 * i];
            const double d3[3] = {x[3 * i] - h->bx[0], x[3 * i + 1] - h->bx[1], x[3 * i + 2] - h->bx[2]};
            for (int c = 0; c < 3; ++c) {
                vp[c] += a[c];
                vt[c] += b[c];
            }
            up[0] += d3[1] * a[2] - d3[2] * a[1];
            up[1] += d3[2] * a[0] - d3[0] * a[2];
            up[2] += d3[0] * a[1] - d3[1] * a[0];
            ut[0] += d3[1] * b[2] - d3[2] * b[1];
            ut[1] += d3[2] * b[0] - d3[0] * b[2];
            ut[2] += d3[0] * b[1] - d3[1] * b[0];
            c11 += a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
            c22 += b[0] * b[0] + b[1] * b[1] + b[2] * b[2];
            c12 += a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
        }
        const double det = c11 * c22 - c12 * c12;
        const double i11 = c22 / det, i22 = c11 / det, i12 = -c12 / det;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                C[6 * i + j] += vp[i] * vp[j] * i11 + vp[i] * vt[j] * i12 + vt[i] * vp[j] * i12 + vt[i] * vt[j] * i22;
                C[6 * (3 + i) + j] +=
                    up[i] * vp[j] * i11 + up[i] * vt[j] * i12 + ut[i] * vp[j] * i12 + ut[i] * vt[j] * i22;
                C[6 * (3 + i) + 3 + j] +=
                    up[i] * up[j] * i11 + up[i] * ut[j] * i12 + ut[i] * up[j] * i12 + ut[i] * ut[j] * i22;
            }
        for (int c = 0; c < 3; ++c) {
            aux[12 * m + c] = vp[c];
            aux[12 * m + 3 + c] = up[c];
            aux[12 * m + 6 + c] = vt[c];
            aux[12 * m + 9 + c] = ut[c];
        }
        gram[3 * m] = c11;
        gram[3 * m + 1] = c22;
        gram[3 * m + 2] = c12;
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C[6 * i + 3 + j] = C[6 * (3 + j) + i];
    for (int q = 0; q < 36; ++q) K[q] -= mob * C[q];
    if (!invert6(K)) return set_error(CF_NONFINITE, "cf_swim: the body's 6x6 preconditioner matrix is singular");
    CF_CUDA(cudaMemcpyAsync(h->kinv, K, sizeof(K), cudaMemcpyHostToDevice, st));
    CF_CUDA(cudaMemcpyAsync(h->aux, aux.data(), aux.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    CF_CUDA(cudaMemcpyAsync(h->d.gram, gram.data(), gram.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    CF_CUDA(cudaStreamSynchronize(st));
    return CF_OK;
}

// out[j] = <Q_j, w> for j < k1 (Q rows n apart), or with `root` out[0] = |w| for Q = w, k1 = 1.
int swim_dots(cf_swim *h, const double *Q, const double *w, int k1, double *out, int root) {
    swim_dots_kernel<<<dim3(kSwimChunks, k1), 256, 0, h->stream>>>(Q, h->n, w, h->n, h->dpart, h->dcount, out, root);
    CF_CHECK_LAUNCH("swim_dots_kernel");
    return CF_OK;
}

// Right-preconditioned GMRES on A sol = rhs with the warm start in sol (mobility_solver.cpp:2187-2669):
// zero RHS -> zero solution; a good guess is kept; a guess worse than zero is discarded.
int swim_gmres(cf_swim *h) {
    const int n = h->n;
    cudaStream_t st = h->stream;
    const long long ldq = n;
    const int g = swim_grid(n);
    // hb layout: [0, M+1) h1, [M+1, 2M+2) h2, [2M+2] norm, [2M+3] |rhs|, [2M+4..) y
    const int M = h->max_iter;
    double *h1 = h->hb, *h2 = h->hb + (M + 1), *nrm = h->hb + 2 * (M + 1), *nrhs = nrm + 1, *yd = nrm + 2;
    CF_TRY(swim_dots(h, h->rhs, h->rhs, 1, nrhs, 1));
    CF_TRY(swim_matvec(h, h->sol, h->w));
    swim_axpby_kernel<<<g, 256, 0, st>>>(h->w, 1.0, h->rhs, -1.0, h->w, n);  // r0 = rhs - A x0
    CF_CHECK_LAUNCH("swim_axpby_kernel");
    CF_TRY(swim_dots(h, h->w, h->w, 1, nrm, 1));
    double nb[2];
    CF_CUDA(cudaMemcpyAsync(nb, nrm, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CF_TRY(swim_sync(h));
    double beta0 = nb[0];
    const double nr = nb[1];
    h->last_iters = 0;
    if (!std::isfinite(nr) || !std::isfinite(beta0)) {
        h->last_status = CF_NONFINITE;
        h->last_relres = beta0 / nr;
        return CF_OK;
    }
    if (nr == 0.0) {
        CF_CUDA(cudaMemsetAsync(h->sol, 0, sizeof(double) * n, st));
        h->last_status = CF_OK;
        h->last_relres = 0.0;
        return CF_OK;
    }
    if (beta0 <= h->cfg.gmres_tol * nr) {
        h->last_status = CF_OK;
        h->last_relres = beta0 / nr;
        return CF_OK;
    }
    if (beta0 > nr) {  // the initial guess is worse than zero
        CF_CUDA(cudaMemsetAsync(h->sol, 0, sizeof(double) * n, st));
        CF_CUDA(cudaMemcpyAsync(h->w, h->rhs, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        beta0 = nr;
    }
    swim_axpby_kernel<<<g, 256, 0, st>>>(h->Q, 1.0 / beta0, h->w, 0.0, nullptr, n);
    CF_CHECK_LAUNCH("swim_axpby_kernel");
    std::vector<double> H(static_cast<size_t>(M + 1) * (M + 1), 0.0), cs(M), sn(M), beta(M + 1, 0.0);
    beta[0] = beta0;
    std::vector<double> hh(2 * (M + 1) + 1);
    int it = 0;
    double rel = 1.0;
    for (it = 1; it <= M; ++it) {
        const int k1 = it;  // basis vectors Q_0 .. Q_{it-1}
        CF_TRY(swim_precond(h, h->Q + static_cast<long long>(it - 1) * ldq, h->z));
        CF_TRY(swim_matvec(h, h->z, h->w));
        CF_TRY(swim_dots(h, h->Q, h->w, k1, h1, 0));
        swim_sub_basis_kernel<<<g, 256, 0, st>>>(h->w, h->Q, ldq, h1, k1, n);
        CF_CHECK_LAUNCH("swim_sub_basis_kernel");
        CF_TRY(swim_dots(h, h->Q, h->w, k1, h2, 0));
        swim_sub_basis_kernel<<<g, 256, 0, st>>>(h->w, h->Q, ldq, h2, k1, n);
        CF_CHECK_LAUNCH("swim_sub_basis_kernel");
        CF_TRY(swim_dots(h, h->w, h->w, 1, nrm, 1));
        CF_CUDA(cudaMemcpyAsync(hh.data(), h->hb, hh.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        CF_TRY(swim_sync(h));
        const double qn = hh[2 * (M + 1)];
        double *col = &H[static_cast<size_t>(it - 1) * (M + 1)];  // column it-1, rows 0..it
        for (int i = 0; i < it; ++i) col[i] = hh[i] + hh[(M + 1) + i];
        col[it] = qn;
        if (!std::isfinite(qn)) {
            h->last_iters = it;
            h->last_status = CF_NONFINITE;
            h->last_relres = qn;
            return CF_OK;
        }
        swim_axpby_kernel<<<g, 256, 0, st>>>(h->Q + static_cast<long long>(it) * ldq, qn != 0.0 ? 1.0 / qn : 1.0,
                                             h->w, 0.0, nullptr, n);
        CF_CHECK_LAUNCH("swim_axpby_kernel");
        // previous rotations, then the new one (the oracle's and the reference's Givens recurrence)
        for (int i = 1; i < it; ++i) {
            const double tmp = cs[i - 1] * col[i - 1] + sn[i - 1] * col[i];
            col[i] = cs[i - 1] * col[i] - sn[i - 1] * col[i - 1];
            col[i - 1] = tmp;
        }
        const double a = col[it - 1], b = col[it];
        if (b == 0.0) {
            cs[it - 1] = 1.0;
            sn[it - 1] = 0.0;
        } else if (std::fabs(b) > std::fabs(a)) {
            const double tt = a / b;
            sn[it - 1] = (b > 0 ? 1.0 : -1.0) / std::sqrt(1.0 + tt * tt);
            cs[it - 1] = tt * sn[it - 1];
        } else {
            const double tt = b / a;
            cs[it - 1] = (a > 0 ? 1.0 : -1.0) / std::sqrt(1.0 + tt * tt);
            sn[it - 1] = tt * cs[it - 1];
        }
        col[it - 1] = cs[it - 1] * a + sn[it - 1] * b;
        col[it] = 0.0;
        beta[it] = -sn[it - 1] * beta[it - 1];
        beta[it - 1] = cs[it - 1] * beta[it - 1];
        rel = std::fabs(beta[it]) / nr;
        if (rel <= h->cfg.gmres_tol || it == M) break;
    }
    if (it > M) it = M;
    std::vector<double> y(it, 0.0);
    for (int i = it - 1; i >= 0; --i) {
        double s = beta[i];
        for (int j = i + 1; j < it; ++j) s -= H[static_cast<size_t>(j) * (M + 1) + i] * y[j];
        y[i] = s / H[static_cast<size_t>(i) * (M + 1) + i];
    }
    CF_CUDA(cudaMemcpyAsync(yd, y.data(), it * sizeof(double), cudaMemcpyHostToDevice, st));
    swim_combine_kernel<<<g, 256, 0, st>>>(h->t, h->Q, ldq, yd, it, n);
    CF_CHECK_LAUNCH("swim_combine_kernel");
    CF_TRY(swim_precond(h, h->t, h->z));
    swim_axpby_kernel<<<g, 256, 0, st>>>(h->sol, 1.0, h->z, 1.0, h->sol, n);
    CF_CHECK_LAUNCH("swim_axpby_kernel");
    CF_TRY(swim_sync(h));
    h->last_iters = it;
    h->last_relres = rel;
    h->last_status = rel <= h->cfg.gmres_tol ? CF_OK : CF_NOT_CONVERGED;
    return CF_OK;
}

void swim_release(cf_swim *h) {
    cudaSetDevice(h->device);
    for (void *p : h->allocations) cudaFree(p);
    h->allocations.clear();
    if (h->stream) cudaStreamDestroy(h->stream);
    h->stream = nullptr;
}

}  // namespace swim
}  // namespace cufil

using namespace cufil;
using namespace cufil::swim;

extern "C" int cf_swim_destroy(cf_swim *h) {
    if (!h) return CF_OK;
    swim_release(h);
    delete h;
    return CF_OK;
}

extern "C" int cf_swim_create(const cf_swim_config *cfg, cf_swim **out) {
    clear_error();
    CF_REQUIRE(cfg && out, "cf_swim_create: null argument");
    *out = nullptr;
    CF_REQUIRE(cfg->n_fil > 0 && cfg->n_seg >= 2 && cfg->n_seg <= 256 && cfg->n_blob >= 0,
               "cf_swim_create: need n_fil > 0, 2 <= n_seg <= 256, n_blob >= 0 (got %d, %d, %d)", cfg->n_fil,
               cfg->n_seg, cfg->n_blob);
    CF_REQUIRE(cfg->beat == CF_BEAT_FULFORD_BLAKE || cfg->beat == CF_BEAT_FULFORD_BLAKE_ORIGINAL,
               "cf_swim_create: unknown beat %d", cfg->beat);
    CF_REQUIRE(cfg->dt > 0 && cfg->seg_sep > 0 && cfg->gmres_tol > 0 && cfg->gmres_max_iter > 0,
               "cf_swim_create: dt, seg_sep, gmres_tol and gmres_max_iter must be positive");
    CF_REQUIRE(cfg->fil_refs && cfg->fil_dirs && (cfg->n_blob == 0 || cfg->blob_refs),
               "cf_swim_create: fil_refs, fil_dirs (and blob_refs when n_blob > 0) are required");
    CF_REQUIRE(cfg->gen_phase_force_refs && cfg->n_gen_phase_refs > 1 && cfg->gen_angle_force_refs &&
                   cfg->n_gen_angle_refs > 1,
               "cf_swim_create: the generalised-force tables are required (dynamic phase and angle)");
    const long long nsys = 3LL * cfg->n_fil * cfg->n_seg + 3LL * cfg->n_blob + 6 + 2LL * cfg->n_fil;
    CF_REQUIRE(nsys < (1LL << 28), "cf_swim_create: system too large");
    CF_CUDA(cudaSetDevice(cfg->device));
    cf_swim *h = new (std::nothrow) cf_swim();
    if (!h) return set_error(CF_ENOMEM, "cf_swim_create: host allocation failed");
    h->cfg = *cfg;
    h->device = cfg->device;
    h->F = cfg->n_fil;
    h->nseg = cfg->n_seg;
    h->N = cfg->n_fil * cfg->n_seg;
    h->B = cfg->n_blob;
    h->o_blob = 3 * h->N;
    h->o_body = h->o_blob + 3 * h->B;
    h->o_phase = h->o_body + 6;
    h->o_angle = h->o_phase + h->F;
    h->n = static_cast<int>(nsys);
    h->max_iter = std::min(h->n, cfg->gmres_max_iter);
    h->fil_ref.assign(cfg->fil_refs, cfg->fil_refs + 3 * static_cast<size_t>(h->F));
    if (h->B) h->blob_ref.assign(cfg->blob_refs, cfg->blob_refs + 3 * static_cast<size_t>(h->B));
    if (cfg->body_x0)
        for (int c = 0; c < 3; ++c) h->bx[c] = cfg->body_x0[c];
    if (cfg->body_q0) {
        Quat q{cfg->body_q0[0], {cfg->body_q0[1], cfg->body_q0[2], cfg->body_q0[3]}};
        qnormalise(q);
        h->bq[0] = q.s;
        for (int c = 0; c < 3; ++c) h->bq[1 + c] = q.v[c];
    }
    h->qref.resize(4 * static_cast<size_t>(h->F));
    for (int m = 0; m < h->F; ++m) {
        const Quat q = filament_frame(cfg->fil_dirs + 3 * m);
        h->qref[4 * m] = q.s;
        for (int c = 0; c < 3; ++c) h->qref[4 * m + 1 + c] = q.v[c];
    }
    int rc = CF_OK;
    do {
        if ((rc = cuda_status(cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, cfg->device),
                              "cudaDeviceGetAttribute", __FILE__, __LINE__)))
            break;
        if ((rc = cuda_status(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate",
                              __FILE__, __LINE__)))
            break;
        SimDev &d = h->d;
        const int F = h->F, ns = h->nseg;
        d.B = 1;
        d.F = F;
        d.nseg = ns;
        d.N = h->N;
        d.dt = cfg->dt;
        d.L = cfg->seg_sep * (ns - 1);
        d.spring = cfg->spring_factor;
        d.s_tol = (cfg->s_tol_factor > 0 ? cfg->s_tol_factor : 0.1) / ns;
        d.beat = beat_table(cfg->beat);
        d.s_rows = cfg->s_values_ref ? cfg->s_ref_rows : 0;
        d.s_cols = cfg->s_values_ref ? cfg->s_ref_cols : 0;
        d.n_phase_refs = cfg->n_gen_phase_refs;
        d.n_angle_refs = cfg->n_gen_angle_refs;
        d.dyn_phase = d.dyn_angle = 1;
        std::vector<double> omega(F), ph(F, 0.0), an(F, 0.0), zeros(F, 0.0);
        for (int m = 0; m < F; ++m) {
            omega[m] = cfg->omega0 ? cfg->omega0[m] : 2.0 * 3.14159265358979323846;
            if (cfg->phase0) ph[m] = cfg->phase0[m];
            if (cfg->angle0) an[m] = cfg->angle0[m];
        }
        const size_t N = h->N, np = h->N + h->B, nv = h->n;
        if ((rc = swim_upload(h, const_cast<double **>(&d.s_table), cfg->s_values_ref,
                              static_cast<size_t>(d.s_rows) * d.s_cols)) ||
            (rc = swim_upload(h, const_cast<double **>(&d.phase_refs), cfg->gen_phase_force_refs, d.n_phase_refs)) ||
            (rc = swim_upload(h, const_cast<double **>(&d.angle_refs), cfg->gen_angle_force_refs, d.n_angle_refs)) ||
            (rc = swim_upload(h, const_cast<double **>(&d.omega0), omega.data(), F)) ||
            (rc = swim_alloc(h, const_cast<double **>(&d.base), 3 * static_cast<size_t>(F))) ||
            (rc = swim_upload(h, &d.phase, ph.data(), F)) || (rc = swim_upload(h, &d.angle, an.data(), F)) ||
            (rc = swim_upload(h, &d.phase_dot, omega.data(), F)) ||
            (rc = swim_upload(h, &d.angle_dot, zeros.data(), F)) || (rc = swim_alloc(h, &d.x4, N)) ||
            (rc = swim_alloc(h, &d.xd, 3 * N)) || (rc = swim_alloc(h, &d.s_cur, N)) ||
            (rc = swim_alloc(h, &d.kp, 3 * N)) || (rc = swim_alloc(h, &d.ka, 3 * N)) ||
            (rc = swim_alloc(h, &d.gram, 3 * static_cast<size_t>(F))) || (rc = swim_alloc(h, &d.lc, 1)) ||
            (rc = swim_alloc(h, &h->Rfil, 9 * static_cast<size_t>(F))) ||
            (rc = swim_alloc(h, &h->xb, 3 * static_cast<size_t>(h->B))) || (rc = swim_alloc(h, &h->body, 3)) ||
            (rc = swim_alloc(h, &h->aux, 12 * static_cast<size_t>(F))) || (rc = swim_alloc(h, &h->kinv, 36)) ||
            (rc = swim_alloc(h, &h->x4all, np)) || (rc = swim_alloc(h, &h->f4all, np)) ||
            (rc = swim_alloc(h, &h->u, 3 * np)) || (rc = swim_alloc(h, &h->err, 1)) ||
            (rc = swim_alloc(h, &h->rhs, nv)) || (rc = swim_alloc(h, &h->sol, nv)) || (rc = swim_alloc(h, &h->w, nv)) ||
            (rc = swim_alloc(h, &h->z, nv)) || (rc = swim_alloc(h, &h->t, nv)) ||
            (rc = swim_alloc(h, &h->Q, static_cast<size_t>(h->max_iter + 1) * nv)) ||
            (rc = swim_alloc(h, &h->hb, 3 * static_cast<size_t>(h->max_iter + 1) + 4)) ||
            (rc = swim_alloc(h, &h->dpart, static_cast<size_t>(h->max_iter + 1) * kSwimChunks)) ||
            (rc = swim_alloc(h, &h->dcount, 1)))
            break;
        if ((rc = cuda_status(cudaMemset(h->dcount, 0, sizeof(unsigned int)), "cudaMemset", __FILE__, __LINE__))) break;
        d.Rfil = h->Rfil;
        RpyBlockDesc bd{};
        bd.wall = 0;
        bd.vd = 3;
        bd.fd = 3;
        bd.nt = bd.ns = static_cast<int>(np);
        h->scratch_cap = rpy_plan_for(bd, h->num_sms).scratch_float4;
        if ((rc = swim_alloc(h, &h->scratch, h->scratch_cap))) break;
        if ((rc = cuda_status(cudaMemset(h->err, 0, sizeof(int)), "cudaMemset", __FILE__, __LINE__))) break;
        if ((rc = cuda_status(cudaMemset(h->sol, 0, sizeof(double) * nv), "cudaMemset", __FILE__, __LINE__))) break;
        LoopCtl lc{};
        if ((rc = cuda_status(cudaMemcpy(d.lc, &lc, sizeof(lc), cudaMemcpyHostToDevice), "cudaMemcpy", __FILE__,
                              __LINE__)))
            break;
        const size_t kin_smem = sizeof(double) * (2 * (10 * ns + 1) + ns);
        if (kin_smem > 48 * 1024 &&
            (rc = cuda_status(cudaFuncSetAttribute(kinematics_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   static_cast<int>(kin_smem)),
                              "cudaFuncSetAttribute", __FILE__, __LINE__)))
            break;
    } while (0);
    if (rc != CF_OK) {
        const std::string msg = cf_last_error();
        cf_swim_destroy(h);
        return set_error(rc, "%s", msg.c_str());
    }
    *out = h;
    return CF_OK;
}

// One implicit step of the swimmer (filament and swimmer initial_guess, compute_velocities, the body update).
extern "C" int cf_swim_step(cf_swim *h, int nt, int *iters, double *relres) {
    clear_error();
    CF_REQUIRE(h && nt >= 0, "cf_swim_step: bad arguments");
    CF_CUDA(cudaSetDevice(h->device));
    cudaStream_t st = h->stream;
    SimDev &d = h->d;
    CF_TRY(swim_frames(h));
    LoopCtl lc{};
    lc.nt = nt;
    CF_CUDA(cudaMemcpyAsync(d.lc, &lc, sizeof(lc), cudaMemcpyHostToDevice, st));
    const int ns = h->nseg;
    const int threads = std::min(256, std::max(64, (3 * ns + 31) / 32 * 32));
    const size_t kin_smem = sizeof(double) * (2 * (10 * ns + 1) + ns);
    kinematics_kernel<<<h->F, threads, kin_smem, st>>>(d);
    CF_CHECK_LAUNCH("kinematics_kernel");
    swim_pack_positions_kernel<<<swim_grid(h->N + h->B), 256, 0, st>>>(d.x4, h->xb, h->N, h->B, h->x4all);
    CF_CHECK_LAUNCH("swim_pack_positions_kernel");
    CF_TRY(swim_precon_matrix(h));  // synchronises
    const SwimParams p = swim_params(h);
    CF_CUDA(cudaMemsetAsync(h->rhs, 0, sizeof(double) * h->n, st));
    swim_rhs_kernel<<<swim_grid(h->F), 256, 0, st>>>(p, d, h->rhs);
    CF_CHECK_LAUNCH("swim_rhs_kernel");
    CF_TRY(swim_gmres(h));
    h->stepped = true;
    // the rates the next step advances with, and the body's velocity for its update
    const size_t fb = sizeof(double) * h->F;
    CF_CUDA(cudaMemcpyAsync(d.phase_dot, h->sol + h->o_phase, fb, cudaMemcpyDeviceToDevice, st));
    CF_CUDA(cudaMemcpyAsync(d.angle_dot, h->sol + h->o_angle, fb, cudaMemcpyDeviceToDevice, st));
    CF_CUDA(cudaMemcpyAsync(h->bv, h->sol + h->o_body, 6 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CF_CUDA(cudaStreamSynchronize(st));
    if (iters) *iters = h->last_iters;
    if (relres) *relres = h->last_relres;
    if (h->last_status == CF_NONFINITE)
        return set_error(CF_NONFINITE, "cf_swim: GMRES met a non-finite value (relative residual %.3e)",
                         h->last_relres);
    // explicit body update (cilia_sim_main.cu:700-716): x += dt V, q = lie_exp(dt Omega) q
    const double dt = h->cfg.dt;
    for (int c = 0; c < 3; ++c) h->bx[c] += dt * h->bv[c];
    const double uu[3] = {dt * h->bv[3], dt * h->bv[4], dt * h->bv[5]};
    const Quat q = qmul(qlie_exp(uu), Quat{h->bq[0], {h->bq[1], h->bq[2], h->bq[3]}});
    h->bq[0] = q.s;
    for (int c = 0; c < 3; ++c) h->bq[1 + c] = q.v[c];
    if (h->last_status == CF_NOT_CONVERGED)
        return set_error(CF_NOT_CONVERGED, "cf_swim: GMRES stopped at its cap: %d iterations, relative residual %.3e",
                         h->last_iters, h->last_relres);
    return CF_OK;
}

// State after the last step: per filament phase, angle and their rates [F] each; the body's
// position [3] and orientation [4] for the next step, and the velocity [6] (V, Omega) solved in the last step.
extern "C" int cf_swim_get_state(cf_swim *h, double *phase, double *angle, double *phase_dot, double *angle_dot,
                                 double *body_x, double *body_q, double *body_v) {
    clear_error();
    CF_REQUIRE(h, "null handle");
    CF_CUDA(cudaSetDevice(h->device));
    const size_t fb = sizeof(double) * h->F;
    cudaStream_t st = h->stream;
    if (phase) CF_CUDA(cudaMemcpyAsync(phase, h->d.phase, fb, cudaMemcpyDeviceToHost, st));
    if (angle) CF_CUDA(cudaMemcpyAsync(angle, h->d.angle, fb, cudaMemcpyDeviceToHost, st));
    if (phase_dot) CF_CUDA(cudaMemcpyAsync(phase_dot, h->d.phase_dot, fb, cudaMemcpyDeviceToHost, st));
    if (angle_dot) CF_CUDA(cudaMemcpyAsync(angle_dot, h->d.angle_dot, fb, cudaMemcpyDeviceToHost, st));
    CF_CUDA(cudaStreamSynchronize(st));
    if (body_x) std::memcpy(body_x, h->bx, sizeof(h->bx));
    if (body_q) std::memcpy(body_q, h->bq, sizeof(h->bq));
    if (body_v) std::memcpy(body_v, h->bv, sizeof(h->bv));
    return CF_OK;
}

// Segment positions [3N] and blob positions [3B] of the last step (FP64), and the solution's
// segment and blob forces [3N], [3B]; any pointer may be NULL.
extern "C" int cf_swim_get_particles(cf_swim *h, double *x_segs, double *x_blobs, double *f_segs, double *f_blobs) {
    clear_error();
    CF_REQUIRE(h, "null handle");
    CF_CUDA(cudaSetDevice(h->device));
    cudaStream_t st = h->stream;
    if (x_segs) CF_CUDA(cudaMemcpyAsync(x_segs, h->d.xd, sizeof(double) * 3 * h->N, cudaMemcpyDeviceToHost, st));
    if (x_blobs && h->B)
        CF_CUDA(cudaMemcpyAsync(x_blobs, h->xb, sizeof(double) * 3 * h->B, cudaMemcpyDeviceToHost, st));
    if (f_segs) CF_CUDA(cudaMemcpyAsync(f_segs, h->sol, sizeof(double) * 3 * h->N, cudaMemcpyDeviceToHost, st));
    if (f_blobs && h->B)
        CF_CUDA(cudaMemcpyAsync(f_blobs, h->sol + h->o_blob, sizeof(double) * 3 * h->B, cudaMemcpyDeviceToHost, st));
    CF_CUDA(cudaStreamSynchronize(st));
    return CF_OK;
}

// Velocity directions of the last step's kinematics (vel_dir_phase, vel_dir_angle) [3N] each.
extern "C" int cf_swim_get_directions(cf_swim *h, double *k_phase, double *k_angle) {
    clear_error();
    CF_REQUIRE(h && h->stepped, "cf_swim_get_directions: bad handle or no step yet");
    CF_CUDA(cudaSetDevice(h->device));
    const size_t b = sizeof(double) * 3 * h->N;
    if (k_phase) CF_CUDA(cudaMemcpyAsync(k_phase, h->d.kp, b, cudaMemcpyDeviceToHost, h->stream));
    if (k_angle) CF_CUDA(cudaMemcpyAsync(k_angle, h->d.ka, b, cudaMemcpyDeviceToHost, h->stream));
    CF_CUDA(cudaStreamSynchronize(h->stream));
    return CF_OK;
}

// A x and P x on host vectors of the system size, for the current geometry (after a step).
extern "C" int cf_swim_system_matvec(cf_swim *h, const double *in, double *out) {
    clear_error();
    CF_REQUIRE(h && in && out && h->stepped, "cf_swim_system_matvec: bad arguments or no step yet");
    CF_CUDA(cudaSetDevice(h->device));
    CF_CUDA(cudaMemcpyAsync(h->z, in, sizeof(double) * h->n, cudaMemcpyHostToDevice, h->stream));
    CF_TRY(swim_matvec(h, h->z, h->w));
    CF_CUDA(cudaMemcpyAsync(out, h->w, sizeof(double) * h->n, cudaMemcpyDeviceToHost, h->stream));
    return swim_sync(h);
}

extern "C" int cf_swim_apply_preconditioner(cf_swim *h, const double *in, double *out) {
    clear_error();
    CF_REQUIRE(h && in && out && h->stepped, "cf_swim_apply_preconditioner: bad arguments or no step yet");
    CF_CUDA(cudaSetDevice(h->device));
    CF_CUDA(cudaMemcpyAsync(h->t, in, sizeof(double) * h->n, cudaMemcpyHostToDevice, h->stream));
    CF_TRY(swim_precond(h, h->t, h->z));
    CF_CUDA(cudaMemcpyAsync(out, h->z, sizeof(double) * h->n, cudaMemcpyDeviceToHost, h->stream));
    return swim_sync(h);
}

extern "C" int cf_swim_system_size(cf_swim *h) { return h ? h->n : -1; }

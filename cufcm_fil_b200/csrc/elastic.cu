// elastic.cu -- cf_elastic: instability-driven elastic cilia on a no-slip wall,
// one implicit step solved by Broyden's method (the reference's CILIA_TYPE 0
// path: cilia_sim_main.cu:405-560).
//
// Model (filament.cpp, segment.cpp): each filament is a chain of S segments
// with positions x_k, orientations q_k and Lie-algebra increments u_k
// (q_k = exp(u_k) q_k^{n-1}); positions follow the orientations (robot arm,
// filament.cpp:629-651).  Internal forces and torques
// (internal_forces_and_torques, filament.cpp:1745-1853): the inextensibility
// multipliers lambda (S-1 links), the tethering multiplier of segment 0, the
// elastic moments diag(KT, KB, KB) (body-frame strain), the follower force
// -F_end t at the tip, a one-off perturbation at step 0 and the clamping torque
// of segment 0.  Velocities: V = M (F + barrier forces), M the 6x6 wall RPY
// matrix (Mss_mult, tile kernel of rpy_kernels.cu).  Residual: backward Euler
// at step 0, BDF2 afterwards, on positions and Lie-algebra elements
// (compute_errors, mobility_solver.cpp:2760-2860).
//
// Unknowns per filament, in the reference's order (filament::update,
// filament.cpp:2174-2206): [tether | lambda_1..lambda_{S-1} | clamp |
// u_1..u_{S-1}], 6S values; residual rows [positions of segments 0..S-1 |
// Lie algebra of segments 0..S-1].  Broyden's method (broyden_solver.cpp:26-131)
// keeps the approximate inverse Jacobian as the per-filament block inverse of
// invert_approx_jacobian (filament.cpp:1855-2172) plus rank-one corrections
// C_i D_i^T; everything is FP64 on the device except the pair mobility.
#include "common.cuh"
#include "rpy_kernels.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

struct cf_elastic {
    cf_elastic_config cfg{};
    int device = 0, num_sms = CF_B200_SMS;
    cudaStream_t stream = nullptr;
    int F = 0, S = 0, N = 0, NB = 0, maxb = 0;
    double DL = 0, dt = 0, kb = 0, kt = 0, fend = 0, frep = 0, tol = 0, conf = 0;
    // segment state [N] (FP64)
    double *x = nullptr, *xm1 = nullptr, *xm2 = nullptr, *q = nullptr, *qm1 = nullptr, *u = nullptr, *um1 = nullptr;
    // multipliers: lambda [F][S-1][3], tether/clamp [F][3], two back values each
    double *lam = nullptr, *lamm1 = nullptr, *lamm2 = nullptr;
    double *tet = nullptr, *tetm1 = nullptr, *tetm2 = nullptr, *clp = nullptr, *clpm1 = nullptr, *clpm2 = nullptr;
    double *pert = nullptr;  // [F][2][3] perturbations at segments 4 and 12 (step 0)
    double *base = nullptr;  // [F][3]
    double *f = nullptr;     // internal forces and torques [6N]
    float4 *x4 = nullptr, *f4 = nullptr, *t4 = nullptr, *scratch = nullptr;
    size_t scratch_cap = 0;
    float *v = nullptr;  // [6N]
    double *jinv = nullptr;  // [F][6S][6S]
    double *err = nullptr, *nerr = nullptr, *upd = nullptr, *C = nullptr, *D = nullptr, *dots = nullptr,
           *scal = nullptr;
    int *flags = nullptr, *h_flags = nullptr;
    int last_iters = 0, total_iters = 0, max_iters = 0, steps = 0;
    bool stepped = false;
    std::vector<void *> allocations;
};

namespace cufil {
namespace elastic {

constexpr double kPi = 3.14159265358979323846;
constexpr int kTooLarge = 1, kNonFinite = 2;
constexpr int kMaxSeg = 24;  // the inverse Jacobian block (6S)^2 FP64 is held in shared memory

struct ElDev {
    int F, S, N, NB;
    double DL, dt, kb, kt, fend, frep;
    double *x, *xm1, *xm2, *q, *qm1, *u, *um1;
    double *lam, *lamm1, *lamm2, *tet, *tetm1, *tetm2, *clp, *clpm1, *clpm2, *pert, *base, *f;
    float4 *x4, *f4, *t4;
    const float *v;
    double *jinv;
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum (blockDim.x a multiple of 32); the result is valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double *sm32) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sm32[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (wid == 0) {
        r = lane < static_cast<int>(blockDim.x >> 5) ? sm32[lane] : 0.0;
        r = warp_sum(r);
    }
    return r;
}

// ------------------------------------------------------------ FP64 rotations
// Quaternions (scalar first) and the Lie-group maps of src/general/quaternion.cpp,
// written from their definitions.
struct Q4 {
    double s, a, b, c;
};

__host__ __device__ inline Q4 qload(const double *p) { return Q4{p[0], p[1], p[2], p[3]}; }
__host__ __device__ inline void qstore(double *p, const Q4 &q) {
    p[0] = q.s;
    p[1] = q.a;
    p[2] = q.b;
    p[3] = q.c;
}
__host__ __device__ inline Q4 qmul(const Q4 &p, const Q4 &q) {
    return Q4{p.s * q.s - (p.a * q.a + p.b * q.b + p.c * q.c), p.s * q.a + q.s * p.a + p.b * q.c - p.c * q.b,
              p.s * q.b + q.s * p.b + p.c * q.a - p.a * q.c, p.s * q.c + q.s * p.c + p.a * q.b - p.b * q.a};
}
__host__ __device__ inline Q4 qconj(const Q4 &q) { return Q4{q.s, -q.a, -q.b, -q.c}; }
__device__ inline Q4 qexp(const double *u) {  // lie_exp: identity below a rotation of 1e-6
    const double th = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    if (th < 1e-6) return Q4{1.0, 0.0, 0.0, 0.0};
    const double sn = sin(0.5 * th) / th;
    return Q4{cos(0.5 * th), sn * u[0], sn * u[1], sn * u[2]};
}
// Principal square root of a unit quaternion (quaternion::sqrt_in_place: the rotation by half the
// angle; a rotation by pi about an unspecified axis is sent to the z axis).
__device__ inline Q4 qsqrt(Q4 q) {
    if (q.s < -0.999999999) return Q4{0.0, 0.0, 0.0, 1.0};
    q.s = sqrt(0.5 * (1.0 + q.s));
    const double t = 2.0 * q.s;
    q.a /= t;
    q.b /= t;
    q.c /= t;
    return q;
}
// The rotation half-way between q1 and q2: (q2 q1*)^(1/2) q1.
__device__ inline Q4 qmid(const Q4 &q1, const Q4 &q2) { return qmul(qsqrt(qmul(q2, qconj(q1))), q1); }
// Images of the reference x, y, z axes (tangent, normal, binormal).
__device__ inline void qtan(const Q4 &q, double *t) {
    t[0] = 1.0 - 2.0 * (q.b * q.b + q.c * q.c);
    t[1] = 2.0 * (q.a * q.b + q.s * q.c);
    t[2] = 2.0 * (q.a * q.c - q.s * q.b);
}
__device__ inline void qnor(const Q4 &q, double *n) {
    n[0] = 2.0 * (q.a * q.b - q.s * q.c);
    n[1] = 1.0 - 2.0 * (q.a * q.a + q.c * q.c);
    n[2] = 2.0 * (q.b * q.c + q.s * q.a);
}
__device__ inline void qbin(const Q4 &q, double *b) {
    b[0] = 2.0 * (q.a * q.c + q.s * q.b);
    b[1] = 2.0 * (q.b * q.c - q.s * q.a);
    b[2] = 1.0 - 2.0 * (q.a * q.a + q.b * q.b);
}
__device__ inline void qrot(const Q4 &q, double *R) {  // row-major; columns t, n, b
    double t[3], n[3], b[3];
    qtan(q, t);
    qnor(q, n);
    qbin(q, b);
    for (int i = 0; i < 3; ++i) {
        R[3 * i] = t[i];
        R[3 * i + 1] = n[i];
        R[3 * i + 2] = b[i];
    }
}

// 3x3 helpers (row-major).  cross(v) is the matrix of w -> w x v, the reference's rcross.
__device__ inline void rx(const double *v, double *M) {
    M[0] = 0.0;
    M[1] = v[2];
    M[2] = -v[1];
    M[3] = -v[2];
    M[4] = 0.0;
    M[5] = v[0];
    M[6] = v[1];
    M[7] = -v[0];
    M[8] = 0.0;
}
__device__ inline void mm3(const double *A, const double *B, double *C) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
}
__device__ inline void mv3(const double *A, const double *v, double *o) {
    for (int i = 0; i < 3; ++i) o[i] = A[3 * i] * v[0] + A[3 * i + 1] * v[1] + A[3 * i + 2] * v[2];
}
__device__ inline void cross3(const double *a, const double *b, double *o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

// dexp_u^{-1} v and its transpose (Lie algebra of SO(3)): v -+ u x v / 2 - c u x (u x v),
// c = (theta/2 cot(theta/2) - 1)/theta^2, -1/12 below a rotation of 1e-5.
__device__ inline double dexpinv_coef(const double *u) {
    const double th2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    const double th = sqrt(th2);
    if (th < 1e-5) return -1.0 / 12.0;
    return (0.5 * th * cos(0.5 * th) / sin(0.5 * th) - 1.0) / th2;
}
__device__ inline void dexpinv(const double *u, const double *v, double *o, double sign) {
    const double c = dexpinv_coef(u);
    double uv[3], uuv[3];
    cross3(u, v, uv);
    cross3(u, uv, uuv);
    for (int i = 0; i < 3; ++i) o[i] = v[i] - sign * 0.5 * uv[i] - c * uuv[i];
}

// Body-frame moment of link k (filament::body_frame_moment): diag(KT, KB, KB) times the vector
// part of 2 qmid* (q_{k+1} - q_k)/DL (the intrinsic strain is zero).
__device__ inline void link_moment(const ElDev &d, const Q4 &q1, const Q4 &q2, double *M) {
    const Q4 m = qconj(qmid(q1, q2));
    const Q4 dq{(q2.s - q1.s) / d.DL, (q2.a - q1.a) / d.DL, (q2.b - q1.b) / d.DL, (q2.c - q1.c) / d.DL};
    const Q4 r = qmul(m, dq);
    M[0] = d.kt * 2.0 * r.a;
    M[1] = d.kb * 2.0 * r.b;
    M[2] = d.kb * 2.0 * r.c;
}

// 4x3 matrix Psi(q) with dq/dt = Psi Omega, and the 4x4 matrix of p -> q p.
__device__ inline void psi_mat(const Q4 &q, double *P) {  // row-major 4x3
    P[0] = -0.5 * q.a;
    P[1] = -0.5 * q.b;
    P[2] = -0.5 * q.c;
    const double v[3] = {q.a, q.b, q.c};
    double X[9];
    rx(v, X);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) P[3 + 3 * i + j] = 0.5 * (X[3 * i + j] + (i == j ? q.s : 0.0));
}
__device__ inline void left_mat(const Q4 &q, double *L) {  // row-major 4x4
    const double v[3] = {q.a, q.b, q.c};
    double X[9];
    rx(v, X);
    L[0] = q.s;
    L[1] = -q.a;
    L[2] = -q.b;
    L[3] = -q.c;
    for (int i = 0; i < 3; ++i) {
        L[4 * (i + 1)] = v[i];
        for (int j = 0; j < 3; ++j) L[4 * (i + 1) + 1 + j] = -X[3 * i + j] + (i == j ? q.s : 0.0);
    }
}

// Derivative of the link moment with respect to the Lie-algebra element of the
// upper (q2) or lower (q1) segment of the link (body_frame_moment_lie_derivative).
__device__ inline void moment_derivative(const ElDev &d, const Q4 &q1, const Q4 &q2, bool upper, double *out) {
    double A[12];
    psi_mat(upper ? q2 : q1, A);
    const double sA = upper ? 1.0 / d.DL : -1.0 / d.DL;
    for (double &a : A) a *= sA;
    const Q4 m = qconj(qmid(q1, q2));
    double L[16], dM[12];
    left_mat(m, L);
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 3; ++j)
            dM[3 * i + j] = L[4 * i] * A[j] + L[4 * i + 1] * A[3 + j] + L[4 * i + 2] * A[6 + j] + L[4 * i + 3] * A[9 + j];
    const Q4 dq{(q2.s - q1.s) / d.DL, (q2.a - q1.a) / d.DL, (q2.b - q1.b) / d.DL, (q2.c - q1.c) / d.DL};
    left_mat(dq, L);
    const double sB = upper ? 0.5 * d.DL : -0.5 * d.DL;
    for (double &a : A) a *= sB;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 3; ++j)
            dM[3 * i + j] += L[4 * i] * A[j] + L[4 * i + 1] * A[3 + j] + L[4 * i + 2] * A[6 + j] + L[4 * i + 3] * A[9 + j];
    for (int i = 0; i < 3; ++i) {
        const double k = i == 0 ? d.kt : d.kb;
        for (int j = 0; j < 3; ++j) out[3 * i + j] = 2.0 * k * dM[3 * (i + 1) + j];
    }
}

// Robot arm: x_k = x_{k-1} + DL/2 (t_{k-1} + t_k) from the base (one thread).
__device__ inline void robot_arm(const ElDev &d, int m) {
    const int S = d.S;
    double *x = d.x + 3 * m * S;
    const double *q = d.q + 4 * m * S;
    double t1[3], t2[3];
    qtan(qload(q), t1);
    for (int k = 1; k < S; ++k) {
        qtan(qload(q + 4 * k), t2);
        for (int c = 0; c < 3; ++c) x[3 * k + c] = x[3 * (k - 1) + c] + 0.5 * d.DL * (t1[c] + t2[c]);
        for (int c = 0; c < 3; ++c) t1[c] = t2[c];
    }
}

// ------------------------------------------------------------ kernels
// filament::initial_guess for elastic filaments on a fixed wall (filament.cpp:1336-1376, 1553-1660):
// back values shift, u is extrapolated (from step 2 on), q = exp(u) q^{n-1}; segment 0 is held at its
// base with u = 0 (accept_state_from_rigid_body); positions by the robot arm; the multipliers are
// extrapolated linearly (step 2) or quadratically (step 3 on).  One block of 32 threads per filament.
__global__ void el_initial_guess_kernel(ElDev d, int nt) {
    const int m = blockIdx.x, S = d.S;
    for (int k = threadIdx.x; k < S; k += blockDim.x) {
        const int i = m * S + k;
        for (int c = 0; c < 3; ++c) {
            d.xm2[3 * i + c] = d.xm1[3 * i + c];
            d.xm1[3 * i + c] = d.x[3 * i + c];
        }
        double *u = d.u + 3 * i, *um1 = d.um1 + 3 * i;
        if (nt <= 1) {
            for (int c = 0; c < 3; ++c) um1[c] = u[c];
        } else {
            for (int c = 0; c < 3; ++c) {
                const double t = 2.0 * u[c] - um1[c];
                um1[c] = u[c];
                u[c] = t;
            }
        }
        const Q4 qo = qload(d.q + 4 * i);
        qstore(d.qm1 + 4 * i, qo);
        if (k == 0) {  // held by the wall: u = 0, q = q^{n-1}, x = base
            for (int c = 0; c < 3; ++c) u[c] = 0.0;
            const double zero[3] = {0.0, 0.0, 0.0};
            qstore(d.q + 4 * i, qmul(qexp(zero), qo));
            for (int c = 0; c < 3; ++c) d.x[3 * i + c] = d.base[3 * m + c];
        } else {
            qstore(d.q + 4 * i, qmul(qexp(u), qo));
        }
    }
    const int nl = 3 * (S - 1);
    auto extrap = [&](double *a, double *a1, double *a2, int j) {
        if (nt == 1) {
            a1[j] = a[j];
        } else if (nt == 2) {
            a2[j] = a1[j];
            a1[j] = a[j];
            a[j] = 2.0 * a1[j] - a2[j];
        } else if (nt > 2) {
            const double t = 3.0 * (a[j] - a1[j]) + a2[j];
            a2[j] = a1[j];
            a1[j] = a[j];
            a[j] = t;
        }
    };
    for (int j = threadIdx.x; j < nl; j += blockDim.x) extrap(d.lam, d.lamm1, d.lamm2, m * nl + j);
    if (threadIdx.x < 3) {
        extrap(d.tet, d.tetm1, d.tetm2, 3 * m + threadIdx.x);
        extrap(d.clp, d.clpm1, d.clpm2, 3 * m + threadIdx.x);
    }
    __syncthreads();
    if (threadIdx.x == 0) robot_arm(d, m);
}

// filament::update (filament.cpp:2174-2206): multipliers += their updates, u_k += update and
// q_k = exp(u_k) q_k^{n-1} for k >= 1, then the robot arm.  One block of 32 threads per filament.
__global__ void el_update_kernel(ElDev d, const double *du) {
    const int m = blockIdx.x, S = d.S;
    const double *w = du + static_cast<size_t>(6) * S * m;
    for (int k = threadIdx.x; k < S; k += blockDim.x) {
        if (k == 0) {
            for (int c = 0; c < 3; ++c) {
                d.tet[3 * m + c] += w[c];
                d.clp[3 * m + c] += w[3 * S + c];
            }
        } else {
            const int i = m * S + k;
            for (int c = 0; c < 3; ++c) d.lam[3 * (m * (S - 1) + k - 1) + c] += w[3 * k + c];
            double *u = d.u + 3 * i;
            for (int c = 0; c < 3; ++c) u[c] += w[3 * (S + k) + c];
            qstore(d.q + 4 * i, qmul(qexp(u), qload(d.qm1 + 4 * i)));
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) robot_arm(d, m);
}

// internal_forces_and_torques (filament.cpp:1745-1853) for instability cilia: FP64 forces and
// torques f [6N], then their FP32 copy (with the barrier forces added by el_barrier_kernel) for the
// pair kernel.  One block per filament, one thread per link; the link terms are collected in
// shared memory and added segment by segment in the reference's order.
__global__ void el_forces_kernel(ElDev d, int nt) {
    __shared__ double lk[kMaxSeg][12];  // per link: force on k, torque on k, force on k+1, torque on k+1
    const int m = blockIdx.x, S = d.S;
    const int i0 = m * S;
    for (int k = threadIdx.x; k < S - 1; k += blockDim.x) {
        const double *lam = d.lam + 3 * (m * (S - 1) + k);
        const Q4 qa = qload(d.q + 4 * (i0 + k)), qb = qload(d.q + 4 * (i0 + k + 1));
        double ta[3], tb[3], tq[3], R[9], M[3], RM[3];
        qtan(qa, ta);
        qtan(qb, tb);
        double *o = lk[k];
        for (int c = 0; c < 3; ++c) {
            o[c] = -lam[c];
            o[6 + c] = lam[c];
        }
        cross3(ta, lam, tq);
        for (int c = 0; c < 3; ++c) o[3 + c] = -0.5 * d.DL * tq[c];
        cross3(tb, lam, tq);
        for (int c = 0; c < 3; ++c) o[9 + c] = -0.5 * d.DL * tq[c];
        qrot(qmid(qa, qb), R);
        link_moment(d, qa, qb, M);
        mv3(R, M, RM);
        for (int c = 0; c < 3; ++c) {
            o[3 + c] += RM[c];
            o[9 + c] -= RM[c];
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < S; k += blockDim.x) {
        double fk[6] = {0, 0, 0, 0, 0, 0};
        if (k > 0)
            for (int c = 0; c < 6; ++c) fk[c] += lk[k - 1][6 + c];
        if (k < S - 1)
            for (int c = 0; c < 6; ++c) fk[c] += lk[k][c];
        if (k == 0) {
            for (int c = 0; c < 3; ++c) fk[c] += d.tet[3 * m + c];
            double ct[3];
            dexpinv(d.u + 3 * i0, d.clp + 3 * m, ct, -1.0);  // dexpinv^T(u_0) clamp
            for (int c = 0; c < 3; ++c) fk[3 + c] += ct[c];
        }
        if (k == S - 1) {
            double t[3];
            qtan(qload(d.q + 4 * (i0 + k)), t);
            for (int c = 0; c < 3; ++c) fk[c] -= d.fend * t[c];
        }
        if (nt == 0 && k == 4)
            for (int c = 0; c < 3; ++c) fk[c] += d.pert[6 * m + c];
        if (nt == 0 && k == 12)
            for (int c = 0; c < 3; ++c) fk[c] += d.pert[6 * m + 3 + c];
        const int i = i0 + k;
        for (int c = 0; c < 6; ++c) d.f[6 * i + c] = fk[c];
        d.x4[i] = make_float4(static_cast<float>(d.x[3 * i]), static_cast<float>(d.x[3 * i + 1]),
                              static_cast<float>(d.x[3 * i + 2]), 0.0f);
        d.t4[i] = make_float4(static_cast<float>(fk[3]), static_cast<float>(fk[4]), static_cast<float>(fk[5]), 0.0f);
    }
}

// Barrier forces (barrier_forces, cuda_functions.cu:1825-1919, wall and segment-segment terms):
// a repulsion growing as the fourth power of the overlap within 1.1 (a_i + a_j) of another segment
// (not the segment itself nor its neighbours in the same filament) and within DL/2 of the wall;
// added in FP64 to the internal forces and packed as FP32 for the pair kernel.  A block takes 16
// targets; its threads split the sources sixteen ways (split c takes every sixteenth of each
// 1024-source tile staged in shared memory), screen the pairs on the FP32 positions with a margin and
// evaluate the few within reach in FP64; the sixteen partial sums are added in a fixed order.
constexpr int kBarTargets = 16, kBarSplit = 16, kBarThreads = kBarTargets * kBarSplit, kBarTile = 1024;
__global__ void __launch_bounds__(kBarThreads) el_barrier_kernel(ElDev d) {
    __shared__ float4 sx[kBarTile];
    __shared__ double part[kBarSplit][kBarTargets][3];
    const int t = threadIdx.x % kBarTargets, c = threadIdx.x / kBarTargets;
    const int i = blockIdx.x * kBarTargets + t;
    const bool live = i < d.N;
    double xi[3] = {0.0, 0.0, 0.0}, fb[3] = {0.0, 0.0, 0.0};
    float4 xf = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (live) {
        for (int q = 0; q < 3; ++q) xi[q] = d.x[3 * i + q];
        xf = d.x4[i];
        if (c == 0 && xi[2] < 0.5 * d.DL) {
            const double w = fmin(1.0, 1.0 - (xi[2] - 1.0) / (0.5 * d.DL - 1.0));
            fb[2] = d.frep * w * w * w * w;
        }
    }
    const int fi = live ? i / d.S : -1;
    for (int j0 = 0; j0 < d.N; j0 += kBarTile) {
        const int nj = min(kBarTile, d.N - j0);
        __syncthreads();
        for (int q = threadIdx.x; q < nj; q += kBarThreads) sx[q] = d.x4[j0 + q];
        __syncthreads();
        if (!live) continue;
        for (int jj = c; jj < nj; jj += kBarSplit) {
            const float4 sj = sx[jj];
            const float ex = xf.x - sj.x, ey = xf.y - sj.y, ez = xf.z - sj.z;
            if (ex * ex + ey * ey + ez * ez >= 4.9f) continue;  // screen: (1.1 * 2a)^2 = 4.84, with margin
            const int js = j0 + jj;
            const double dx = xi[0] - d.x[3 * js], dy = xi[1] - d.x[3 * js + 1], dz = xi[2] - d.x[3 * js + 2];
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 >= 4.84) continue;
            if (fi == js / d.S && abs(i - js) <= 1) continue;
            const double r = sqrt(r2);
            double w = fmin(1.0, 1.0 - 5.0 * (r - 2.0));
            w = d.frep * w * w * w * w;
            fb[0] += w * dx / r;
            fb[1] += w * dy / r;
            fb[2] += w * dz / r;
        }
    }
    for (int q = 0; q < 3; ++q) part[c][t][q] = fb[q];
    __syncthreads();
    if (c == 0 && live) {
        double tot[3] = {0.0, 0.0, 0.0};
        for (int cc = 0; cc < kBarSplit; ++cc)
            for (int q = 0; q < 3; ++q) tot[q] += part[cc][t][q];
        d.f4[i] = make_float4(static_cast<float>(d.f[6 * i] + tot[0]), static_cast<float>(d.f[6 * i + 1] + tot[1]),
                              static_cast<float>(d.f[6 * i + 2] + tot[2]), 0.0f);
    }
}

// compute_errors (mobility_solver.cpp:2760-2860, wall): backward Euler at step 0, BDF2 afterwards,
// on positions (test |e| > DL tol) and Lie-algebra elements (test |e| > tol, with dexp^{-1}_u Omega);
// flags: too large, non-finite.
__global__ void el_errors_kernel(ElDev d, int nt, double tol, double *e, int *flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int fl = 0;
    if (i < d.N) {
        const int m = i / d.S, k = i - m * d.S;
        const float *v = d.v + 6 * static_cast<size_t>(i);
        double vel[3], om[3], W[3];
        for (int c = 0; c < 3; ++c) {
            vel[c] = v[c];
            om[c] = v[3 + c];
        }
        const size_t id = static_cast<size_t>(6) * d.S * m + 3 * k;
        const double *u = d.u + 3 * i;
        dexpinv(u, om, W, 1.0);
        for (int c = 0; c < 3; ++c) {
            double ep, eu;
            if (nt < 1) {
                ep = d.x[3 * i + c] - d.xm1[3 * i + c] - d.dt * vel[c];
                eu = u[c] - d.dt * W[c];
            } else {
                ep = d.x[3 * i + c] - (4.0 / 3.0) * d.xm1[3 * i + c] + (1.0 / 3.0) * d.xm2[3 * i + c] -
                     (2.0 / 3.0) * d.dt * vel[c];
                eu = u[c] - (1.0 / 3.0) * d.um1[3 * i + c] - (2.0 / 3.0) * d.dt * W[c];
            }
            e[id + c] = ep;
            e[id + 3 * d.S + c] = eu;
            if (fabs(ep) > d.DL * tol || fabs(eu) > tol) fl |= kTooLarge;
            if (!isfinite(ep) || !isfinite(eu)) fl |= kNonFinite;
        }
    }
    fl = __reduce_or_sync(0xffffffffu, fl);
    if ((threadIdx.x & 31) == 0 && fl) atomicOr(flags, fl);
}

// invert_approx_jacobian (filament.cpp:1855-2172), assembled row-major into J [6S][6S] of filament m;
// one block per filament: the position rows by the first threads, the Lie-algebra block
// (jacobian_lie_algebra_block) one segment per thread.
__global__ void el_jacobian_kernel(ElDev d, int nt) {
    const int m = blockIdx.x, S = d.S, n = 6 * S;
    double *J = d.jinv + static_cast<size_t>(m) * n * n;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) J[e] = 0.0;
    __syncthreads();
    const int i0 = m * S;
    const bool euler = nt < 1;
    auto set3 = [&](int r, int c, const double *B) {
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) J[static_cast<size_t>(r + a) * n + c + b] = B[3 * a + b];
    };
    auto seg_q = [&](int k) { return qload(d.q + 4 * (i0 + k)); };
    const double fac = euler ? -d.dt / (6.0 * kPi) : -d.dt / (9.0 * kPi);
    // positions on the tether / inextensibility multipliers
    for (int r = threadIdx.x; r < 3 * S; r += blockDim.x) {
        J[static_cast<size_t>(r) * n + r] = fac;
        if (r < 3 * S - 3) J[static_cast<size_t>(r) * n + r + 3] = -fac;
    }
    __syncthreads();
    // positions on the Lie-algebra elements: segment j >= 1 moves segments j.. by DL/2 t_j x (.) and DL t_j x (.)
    for (int j = 1 + threadIdx.x; j < S; j += blockDim.x) {
        double t[3], X[9], H[9];
        qtan(seg_q(j), t);
        rx(t, X);
        for (int e = 0; e < 9; ++e) {
            H[e] = 0.5 * d.DL * X[e];
            X[e] *= d.DL;
        }
        const int jpos = 3 * (S + j);
        set3(3 * j, jpos, H);
        for (int i = j + 1; i < S; ++i) set3(3 * i, jpos, X);
    }
    __syncthreads();
    if (threadIdx.x == 0) {  // the follower force at the tip
        double t[3], X[9];
        qtan(seg_q(S - 1), t);
        rx(t, X);
        const size_t r = 3 * (S - 1), c = 3 * (2 * S - 1);
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) J[(r + a) * n + c + b] -= fac * d.fend * X[3 * a + b];
    }
    // Lie-algebra rows on the multipliers
    const double fac2 = euler ? d.DL * d.dt / (16.0 * kPi) : d.DL * d.dt / (24.0 * kPi);
    for (int j = 1 + threadIdx.x; j < S; j += blockDim.x) {
        for (int side = 0; side < 2; ++side) {
            const int k = j - 1 + side;
            double t[3], T[9], U[9], UT[9], UUT[9], B[9];
            qtan(seg_q(k), t);
            rx(t, T);
            for (double &a : T) a = -a;
            rx(d.u + 3 * (i0 + k), U);
            mm3(U, T, UT);
            mm3(U, UT, UUT);
            for (int e = 0; e < 9; ++e) B[e] = fac2 * (T[e] + 0.5 * UT[e] + UUT[e] / 12.0);
            set3(3 * (S + j - 1 + side), 3 * j, B);
        }
    }
    __syncthreads();
    // Lie-algebra rows on the Lie-algebra elements (jacobian_lie_algebra_block), segment k per thread
    const double tsf = euler ? d.dt : 2.0 * d.dt / 3.0;
    const double Tf = 1.0 / (8.0 * kPi);
    for (int k = threadIdx.x; k < S; k += blockDim.x) {
        const Q4 qk = seg_q(k);
        double t[3], nn[3], b[3], Lie[9], Om[9], dO[9], tmp[9], tmp2[9], B[9];
        qtan(qk, t);
        qnor(qk, nn);
        qbin(qk, b);
        const double *uk = d.u + 3 * (i0 + k);
        rx(uk, Lie);
        for (double &a : Lie) a = -a;
        double aom[3];
        for (int c = 0; c < 3; ++c) aom[c] = Tf * d.f[6 * (i0 + k) + 3 + c];
        rx(aom, Om);
        // elastic part of the diagonal block from the link above (k < S-1) and below (k > 0)
        double El[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        auto tnb_part = [&](const double *K, double sgn, const double *ta, const double *na, const double *ba) {
            double Xa[9], Xb[9], Xc[9];
            rx(ta, Xa);
            rx(na, Xb);
            rx(ba, Xc);
            for (int e = 0; e < 9; ++e) El[e] += sgn * 0.5 * (K[0] * Xa[e] + K[1] * Xb[e] + K[2] * Xc[e]);
        };
        double lamv[3] = {0.0, 0.0, 0.0};
        if (k < S - 1) {
            const Q4 qp = seg_q(k + 1);
            double K[3], R[9], LD[9], RLD[9];
            link_moment(d, qk, qp, K);
            tnb_part(K, 1.0, t, nn, b);
            qrot(qmid(qk, qp), R);
            moment_derivative(d, qk, qp, false, LD);
            mm3(R, LD, RLD);
            for (int e = 0; e < 9; ++e) El[e] += RLD[e];
            for (int c = 0; c < 3; ++c) lamv[c] += d.lam[3 * (m * (S - 1) + k) + c];
        }
        if (k > 0) {
            const Q4 qm = seg_q(k - 1);
            double K[3], R[9], LD[9], RLD[9];
            link_moment(d, qm, qk, K);
            tnb_part(K, -1.0, t, nn, b);
            qrot(qmid(qm, qk), R);
            moment_derivative(d, qm, qk, true, LD);
            mm3(R, LD, RLD);
            for (int e = 0; e < 9; ++e) El[e] -= RLD[e];
            for (int c = 0; c < 3; ++c) lamv[c] += d.lam[3 * (m * (S - 1) + k - 1) + c];
        }
        // constraint part -DL/2 cross(lambda) cross(t)
        double Xl[9], Xt[9], Cp[9];
        rx(lamv, Xl);
        rx(t, Xt);
        mm3(Xl, Xt, Cp);
        for (int e = 0; e < 9; ++e) dO[e] = Tf * (El[e] - 0.5 * d.DL * Cp[e]);
        // diagonal block: -tsf (dO - (Om + Lie dO)/2 + (cross(Om u) + Lie Om + Lie Lie dO)/12) + I
        double LdO[9], LOm[9], LLdO[9], Omu[3], XOmu[9];
        mm3(Lie, dO, LdO);
        mm3(Lie, Om, LOm);
        mm3(Lie, LdO, LLdO);
        mv3(Om, uk, Omu);
        rx(Omu, XOmu);
        for (int e = 0; e < 9; ++e)
            B[e] = -tsf * (dO[e] - 0.5 * (Om[e] + LdO[e]) + (XOmu[e] + LOm[e] + LLdO[e]) / 12.0) + (e % 4 == 0 ? 1.0 : 0.0);
        set3(3 * (S + k), 3 * (S + k), B);
        // off-diagonal blocks: -tsf (dO - Lie dO/2 + Lie Lie dO/12) with dO from the neighbour's frame
        for (int side = 0; side < 2; ++side) {
            const int kn = side == 0 ? k - 1 : k + 1;
            if (kn < 0 || kn >= S) continue;
            const Q4 qn = seg_q(kn);
            double tn[3], nnb[3], bn[3], K[3], R[9], LD[9], RLD[9];
            qtan(qn, tn);
            qnor(qn, nnb);
            qbin(qn, bn);
            for (double &a : El) a = 0.0;
            if (side == 0) {  // left: link (k-1, k), derivative in the lower segment
                link_moment(d, qn, qk, K);
                tnb_part(K, -1.0, tn, nnb, bn);
                qrot(qmid(qn, qk), R);
                moment_derivative(d, qn, qk, false, LD);
                mm3(R, LD, RLD);
                for (int e = 0; e < 9; ++e) El[e] -= RLD[e];
            } else {  // right: link (k, k+1), derivative in the upper segment
                link_moment(d, qk, qn, K);
                tnb_part(K, 1.0, tn, nnb, bn);
                qrot(qmid(qk, qn), R);
                moment_derivative(d, qk, qn, true, LD);
                mm3(R, LD, RLD);
                for (int e = 0; e < 9; ++e) El[e] += RLD[e];
            }
            for (int e = 0; e < 9; ++e) dO[e] = Tf * El[e];
            mm3(Lie, dO, tmp);
            mm3(Lie, tmp, tmp2);
            for (int e = 0; e < 9; ++e) B[e] = -tsf * (dO[e] - 0.5 * tmp[e] + tmp2[e] / 12.0);
            set3(3 * (S + k), 3 * (S + kn), B);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {  // the clamped frame: the first three columns of the Lie block
        const double fac3 = euler ? -d.dt / (8.0 * kPi) : -d.dt / (12.0 * kPi);
        double U[9], UU[9], P[9], Pt[9], B[9];
        rx(d.u + 3 * i0, U);
        mm3(U, U, UU);
        for (int e = 0; e < 9; ++e) {
            const double id = e % 4 == 0 ? 1.0 : 0.0;
            P[e] = id + 0.5 * U[e] + UU[e] / 12.0;
            Pt[e] = id - 0.5 * U[e] + UU[e] / 12.0;
        }
        mm3(P, Pt, B);
        for (double &a : B) a *= fac3;
        set3(3 * S, 3 * S, B);
        const double Z[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        set3(3 * S + 3, 3 * S, Z);
    }
}

// In-place Gauss-Jordan inversion with partial pivoting of each filament's 6S x 6S block (FP64,
// held in shared memory); a zero pivot column sets the non-finite flag.  Per pivot, three barriers:
// warp 0 finds the pivot row; the pivot row, row k and the pivot column are saved; then the row
// interchange, the scaling of the pivot row and the rank-one update are one pass in which every element
// is written from its own old value and the saved vectors, over a 2-D split of the matrix (warp w takes
// rows w, w + 16, ..., its lanes consecutive columns).
constexpr int kInvThreads = 512;
__global__ void __launch_bounds__(kInvThreads) el_invert_kernel(ElDev d, int *flags) {
    extern __shared__ double A[];
    __shared__ int piv_row[6 * kMaxSeg];
    __shared__ double colk[6 * kMaxSeg], prow_s[6 * kMaxSeg], rowk_s[6 * kMaxSeg];
    __shared__ int sp;
    const int m = blockIdx.x, n = 6 * d.S;
    double *J = d.jinv + static_cast<size_t>(m) * n * n;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) A[e] = J[e];
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    bool singular = false;
    for (int k = 0; k < n; ++k) {
        if (w == 0) {  // pivot: the largest |A[r][k]|, r >= k (lowest index among ties)
            double best = -1.0;
            int bi = k;
            for (int r = k + lane; r < n; r += 32) {
                const double a = fabs(A[r * n + k]);
                if (a > best) {
                    best = a;
                    bi = r;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_down_sync(0xffffffffu, best, o);
                const int oi = __shfl_down_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) {
                    best = ob;
                    bi = oi;
                }
            }
            if (lane == 0) {
                sp = (best > 0.0) ? bi : -1;
                piv_row[k] = sp < 0 ? k : sp;
            }
        }
        __syncthreads();
        const int p = sp;
        if (p < 0) {
            singular = true;
            break;
        }
        // save the scaled pivot row (old row p times 1/pivot, 1/pivot in column k), old row k and the pivot
        // column with rows k and p interchanged
        const double inv = 1.0 / A[p * n + k];
        for (int c = threadIdx.x; c < n; c += blockDim.x) {
            prow_s[c] = (c == k) ? inv : A[p * n + c] * inv;
            rowk_s[c] = A[k * n + c];
        }
        for (int r = threadIdx.x; r < n; r += blockDim.x) colk[r] = A[(r == k ? p : (r == p ? k : r)) * n + k];
        __syncthreads();
        // every element from its own old value and the saved vectors: row k becomes the scaled pivot row, every
        // other row (row p holding old row k after the interchange) loses its pivot-column entry times it; the
        // lane that wrote a row's column-k entry then replaces it by -entry / pivot
        for (int r = w; r < n; r += nw) {
            double *Ar = A + r * n;
            if (r == k) {
                for (int c = lane; c < n; c += 32) Ar[c] = prow_s[c];
                continue;
            }
            const double fr = colk[r];
            const double *src = (r == p) ? rowk_s : Ar;
            for (int c = lane; c < n; c += 32) Ar[c] = fma(-fr, prow_s[c], src[c]);
            if (lane == (k & 31)) Ar[k] = -fr * inv;
        }
        __syncthreads();
    }
    if (singular) {
        if (threadIdx.x == 0) atomicOr(flags, kNonFinite);
        return;
    }
    // undo the row interchanges as column interchanges, last first
    for (int k = n - 1; k >= 0; --k) {
        const int p = piv_row[k];
        if (p != k)
            for (int r = threadIdx.x; r < n; r += blockDim.x) {
                const double t = A[r * n + k];
                A[r * n + k] = A[r * n + p];
                A[r * n + p] = t;
            }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) J[e] = A[e];
}

// out_m = s * Jinv_m in_m per filament (swimmer::jacobian_inv_mult); one warp per row.
__global__ void el_jinv_mult_kernel(ElDev d, const double *in, double *out, double s) {
    const int m = blockIdx.x, n = 6 * d.S;
    const double *J = d.jinv + static_cast<size_t>(m) * n * n;
    const double *x = in + static_cast<size_t>(m) * n;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int r = w; r < n; r += nw) {
        double a = 0.0;
        for (int c = lane; c < n; c += 32) a += J[static_cast<size_t>(r) * n + c] * x[c];
        a = warp_sum(a);
        if (lane == 0) out[static_cast<size_t>(m) * n + r] = s * a;
    }
}

// dots[i] = <vec, D_i>, i < k (one block per column, fixed-order block sum).
__global__ void el_dots_kernel(const double *vec, const double *D, size_t ld, int len, double *dots) {
    __shared__ double sm32[32];
    const double *col = D + static_cast<size_t>(blockIdx.x) * ld;
    double a = 0.0;
    for (int i = threadIdx.x; i < len; i += blockDim.x) a += vec[i] * col[i];
    a = block_sum(a, sm32);
    if (threadIdx.x == 0) dots[blockIdx.x] = a;
}

// out -= sum_i dots[i] C_i, i = 0..k-1 in order (the reference's sequential column updates).
__global__ void el_sub_cols_kernel(double *out, const double *C, size_t ld, const double *dots, int k, int len) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= len) return;
    double a = out[i];
    for (int j = 0; j < k; ++j) a -= dots[j] * C[static_cast<size_t>(j) * ld + i];
    out[i] = a;
}

// D_k = nerr - err and its norm into scal[0] (one block).
__global__ void el_diff_norm_kernel(const double *nerr, const double *err, double *Dk, int len, double *scal) {
    __shared__ double sm32[32];
    double a = 0.0;
    for (int i = threadIdx.x; i < len; i += blockDim.x) {
        const double t = nerr[i] - err[i];
        Dk[i] = t;
        a += t * t;
    }
    a = block_sum(a, sm32);
    if (threadIdx.x == 0) scal[0] = sqrt(a);
}

__global__ void el_scale2_kernel(double *a, double *b, int len, const double *scal) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= len) return;
    const double s = scal[0];
    a[i] /= s;
    b[i] /= s;
}

// ------------------------------------------------------------ host side
template <typename T>
int el_alloc(cf_elastic *h, T **p, size_t n) {
    *p = nullptr;
    void *q = nullptr;
    CF_CUDA(cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)));
    h->allocations.push_back(q);
    *p = static_cast<T *>(q);
    return CF_OK;
}

ElDev dev(const cf_elastic *h) {
    ElDev d{};
    d.F = h->F;
    d.S = h->S;
    d.N = h->N;
    d.NB = h->NB;
    d.DL = h->DL;
    d.dt = h->dt;
    d.kb = h->kb;
    d.kt = h->kt;
    d.fend = h->fend;
    d.frep = h->frep;
    d.x = h->x;
    d.xm1 = h->xm1;
    d.xm2 = h->xm2;
    d.q = h->q;
    d.qm1 = h->qm1;
    d.u = h->u;
    d.um1 = h->um1;
    d.lam = h->lam;
    d.lamm1 = h->lamm1;
    d.lamm2 = h->lamm2;
    d.tet = h->tet;
    d.tetm1 = h->tetm1;
    d.tetm2 = h->tetm2;
    d.clp = h->clp;
    d.clpm1 = h->clpm1;
    d.clpm2 = h->clpm2;
    d.pert = h->pert;
    d.base = h->base;
    d.f = h->f;
    d.x4 = h->x4;
    d.f4 = h->f4;
    d.t4 = h->t4;
    d.v = h->v;
    d.jinv = h->jinv;
    return d;
}

int grid_for(int n, int t) { return std::max(1, (n + t - 1) / t); }

// forces, barrier forces, the 6x6 wall mobility and the residual into e; the flags word is
// cleared first and left on the device.
int evaluate(cf_elastic *h, int nt, double *e) {
    cudaStream_t st = h->stream;
    const ElDev d = dev(h);
    el_forces_kernel<<<h->F, 32, 0, st>>>(d, nt);
    CF_CHECK_LAUNCH("el_forces_kernel");
    el_barrier_kernel<<<grid_for(h->N, kBarTargets), kBarThreads, 0, st>>>(d);
    CF_CHECK_LAUNCH("el_barrier_kernel");
    RpyBlockDesc bd{};
    bd.wall = 1;
    bd.vd = 6;
    bd.fd = 6;
    bd.self_set = 1;
    bd.xt = h->x4;
    bd.nt = h->N;
    bd.at = 1.0f;
    bd.xs = h->x4;
    bd.fs = h->f4;
    bd.ts = h->t4;
    bd.ns = h->N;
    bd.as = 1.0f;
    bd.mu = 1.0f;
    CF_TRY(rpy_block_product(bd, h->scratch, h->scratch_cap, h->flags + 1, h->v, 6, kOutWrite, h->num_sms, st));
    CF_CUDA(cudaMemsetAsync(h->flags, 0, sizeof(int), st));
    el_errors_kernel<<<grid_for(h->N, 256), 256, 0, st>>>(d, nt, h->tol, e, h->flags);
    CF_CHECK_LAUNCH("el_errors_kernel");
    return CF_OK;
}

// Reads the flags word (and the pair kernel's wait flag); one synchronisation.
int read_flags(cf_elastic *h, int *fl) {
    CF_CUDA(cudaMemcpyAsync(h->h_flags, h->flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CF_CUDA(cudaStreamSynchronize(h->stream));
    *fl = h->h_flags[0];
    if (h->h_flags[1]) {
        CF_CUDA(cudaMemset(h->flags + 1, 0, sizeof(int)));
        return set_error(CF_TIMEOUT, "cf_elastic: a bounded device wait of the pair kernel gave up");
    }
    return CF_OK;
}

int prepare_jacobian(cf_elastic *h, int nt) {
    const ElDev d = dev(h);
    el_jacobian_kernel<<<h->F, 64, 0, h->stream>>>(d, nt);
    CF_CHECK_LAUNCH("el_jacobian_kernel");
    const size_t smem = sizeof(double) * 36 * h->S * h->S;
    el_invert_kernel<<<h->F, kInvThreads, smem, h->stream>>>(d, h->flags);
    CF_CHECK_LAUNCH("el_invert_kernel");
    return CF_OK;
}

// update = -conf Jinv err - sum_i <err, D_i> C_i (broyden_solver::find_update)
int find_update(cf_elastic *h, int iter) {
    cudaStream_t st = h->stream;
    const ElDev d = dev(h);
    el_jinv_mult_kernel<<<h->F, 256, 0, st>>>(d, h->err, h->upd, -h->conf);
    CF_CHECK_LAUNCH("el_jinv_mult_kernel");
    if (iter > 0) {
        el_dots_kernel<<<iter, 512, 0, st>>>(h->err, h->D, h->NB, h->NB, h->dots);
        CF_CHECK_LAUNCH("el_dots_kernel");
        el_sub_cols_kernel<<<grid_for(h->NB, 256), 256, 0, st>>>(h->upd, h->C, h->NB, h->dots, iter, h->NB);
        CF_CHECK_LAUNCH("el_sub_cols_kernel");
    }
    return CF_OK;
}

// The new rank-one pair (broyden_solver::end_of_iter): C_k = (-conf Jinv nerr - sum_i <nerr, D_i> C_i)/|D_k|,
// D_k = (nerr - err)/|D_k|; then err <-> nerr.
int end_of_iter(cf_elastic *h, int iter) {
    cudaStream_t st = h->stream;
    const ElDev d = dev(h);
    double *Ck = h->C + static_cast<size_t>(iter) * h->NB, *Dk = h->D + static_cast<size_t>(iter) * h->NB;
    el_jinv_mult_kernel<<<h->F, 256, 0, st>>>(d, h->nerr, Ck, -h->conf);
    CF_CHECK_LAUNCH("el_jinv_mult_kernel");
    if (iter > 0) {
        el_dots_kernel<<<iter, 512, 0, st>>>(h->nerr, h->D, h->NB, h->NB, h->dots);
        CF_CHECK_LAUNCH("el_dots_kernel");
        el_sub_cols_kernel<<<grid_for(h->NB, 256), 256, 0, st>>>(Ck, h->C, h->NB, h->dots, iter, h->NB);
        CF_CHECK_LAUNCH("el_sub_cols_kernel");
    }
    el_diff_norm_kernel<<<1, 1024, 0, st>>>(h->nerr, h->err, Dk, h->NB, h->scal);
    CF_CHECK_LAUNCH("el_diff_norm_kernel");
    el_scale2_kernel<<<grid_for(h->NB, 256), 256, 0, st>>>(Ck, Dk, h->NB, h->scal);
    CF_CHECK_LAUNCH("el_scale2_kernel");
    std::swap(h->err, h->nerr);
    return CF_OK;
}

void release(cf_elastic *h) {
    cudaSetDevice(h->device);
    for (void *p : h->allocations) cudaFree(p);
    h->allocations.clear();
    if (h->h_flags) cudaFreeHost(h->h_flags);
    h->h_flags = nullptr;
    if (h->stream) cudaStreamDestroy(h->stream);
    h->stream = nullptr;
}

// The reference's initial frame of a filament along +z (filament.cpp:221-236): the square root of
// the rotation taking e_x to e_z, (1/sqrt2, 0, -1/sqrt2, 0).
void initial_frame(double *q) {
    q[0] = std::sqrt(0.5);
    q[1] = 0.0;
    q[2] = -std::sqrt(0.5);
    q[3] = 0.0;
}

}  // namespace elastic
}  // namespace cufil

using namespace cufil;
using namespace cufil::elastic;

extern "C" int cf_elastic_destroy(cf_elastic *h) {
    if (!h) return CF_OK;
    release(h);
    delete h;
    return CF_OK;
}

extern "C" int cf_elastic_create(const cf_elastic_config *cfg, cf_elastic **out) {
    clear_error();
    CF_REQUIRE(cfg && out && cfg->base_pos, "cf_elastic_create: null argument");
    *out = nullptr;
    CF_REQUIRE(cfg->n_fil > 0 && cfg->n_seg >= 13 && cfg->n_seg <= kMaxSeg,
               "cf_elastic_create: need n_fil > 0 and 13 <= n_seg <= %d (the step-0 perturbations act on "
               "segments 4 and 12), got %d, %d",
               kMaxSeg, cfg->n_fil, cfg->n_seg);
    CF_REQUIRE(cfg->seg_sep > 2.0 && cfg->dt > 0.0,
               "cf_elastic_create: seg_sep must exceed 2 (the barrier's wall zone) and dt be positive");
    CF_REQUIRE(cfg->ic_type >= 0 && cfg->ic_type <= 2, "cf_elastic_create: ic_type must be 0, 1 or 2");
    CF_REQUIRE(cfg->ic_type != 2 || cfg->perturbations, "cf_elastic_create: ic_type 2 needs perturbations");
    CF_REQUIRE(static_cast<long long>(cfg->n_fil) * cfg->n_seg < (1LL << 22), "cf_elastic_create: too many segments");
    CF_CUDA(cudaSetDevice(cfg->device));
    cf_elastic *h = new (std::nothrow) cf_elastic();
    if (!h) return set_error(CF_ENOMEM, "cf_elastic_create: host allocation failed");
    h->cfg = *cfg;
    h->device = cfg->device;
    h->F = cfg->n_fil;
    h->S = cfg->n_seg;
    h->N = h->F * h->S;
    h->NB = 6 * h->N;
    h->DL = cfg->seg_sep;
    h->dt = cfg->dt;
    h->kb = cfg->kb > 0 ? cfg->kb : 1800.0;
    h->kt = cfg->kt > 0 ? cfg->kt : 1800.0;
    const double df = cfg->dimensionless_force > 0 ? cfg->dimensionless_force : 220.0;
    h->fend = df * h->kb / (h->DL * h->DL * h->S * h->S);
    h->frep = (cfg->repulsion_factor > 0 ? cfg->repulsion_factor : 2.0) * h->fend;
    h->tol = cfg->broyden_tol > 0 ? cfg->broyden_tol : 1e-4;
    h->conf = cfg->jacobian_confidence > 0 ? cfg->jacobian_confidence : 0.1;
    h->maxb = cfg->max_broyden_iter > 0 ? cfg->max_broyden_iter : 400;
    const int F = h->F, S = h->S;
    const size_t N = h->N, NB = h->NB;
    int rc = CF_OK;
    do {
        if ((rc = cuda_status(cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, cfg->device),
                              "cudaDeviceGetAttribute", __FILE__, __LINE__)))
            break;
        if ((rc = cuda_status(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate",
                              __FILE__, __LINE__)))
            break;
        if ((rc = cuda_status(cudaMallocHost(&h->h_flags, 2 * sizeof(int)), "cudaMallocHost", __FILE__, __LINE__)))
            break;
        const size_t nl = 3 * static_cast<size_t>(F) * (S - 1);
        if ((rc = el_alloc(h, &h->x, 3 * N)) || (rc = el_alloc(h, &h->xm1, 3 * N)) ||
            (rc = el_alloc(h, &h->xm2, 3 * N)) || (rc = el_alloc(h, &h->q, 4 * N)) ||
            (rc = el_alloc(h, &h->qm1, 4 * N)) || (rc = el_alloc(h, &h->u, 3 * N)) ||
            (rc = el_alloc(h, &h->um1, 3 * N)) || (rc = el_alloc(h, &h->lam, nl)) ||
            (rc = el_alloc(h, &h->lamm1, nl)) || (rc = el_alloc(h, &h->lamm2, nl)) ||
            (rc = el_alloc(h, &h->tet, 3 * static_cast<size_t>(F))) ||
            (rc = el_alloc(h, &h->tetm1, 3 * static_cast<size_t>(F))) ||
            (rc = el_alloc(h, &h->tetm2, 3 * static_cast<size_t>(F))) ||
            (rc = el_alloc(h, &h->clp, 3 * static_cast<size_t>(F))) ||
            (rc = el_alloc(h, &h->clpm1, 3 * static_cast<size_t>(F))) ||
            (rc = el_alloc(h, &h->clpm2, 3 * static_cast<size_t>(F))) ||
            (rc = el_alloc(h, &h->pert, 6 * static_cast<size_t>(F))) ||
            (rc = el_alloc(h, &h->base, 3 * static_cast<size_t>(F))) || (rc = el_alloc(h, &h->f, 6 * N)) ||
            (rc = el_alloc(h, &h->x4, N)) || (rc = el_alloc(h, &h->f4, N)) || (rc = el_alloc(h, &h->t4, N)) ||
            (rc = el_alloc(h, &h->v, 6 * N)) ||
            (rc = el_alloc(h, &h->jinv, static_cast<size_t>(F) * 36 * S * S)) || (rc = el_alloc(h, &h->err, NB)) ||
            (rc = el_alloc(h, &h->nerr, NB)) || (rc = el_alloc(h, &h->upd, NB)) ||
            (rc = el_alloc(h, &h->C, NB * h->maxb)) || (rc = el_alloc(h, &h->D, NB * h->maxb)) ||
            (rc = el_alloc(h, &h->dots, static_cast<size_t>(h->maxb))) || (rc = el_alloc(h, &h->scal, 1)) ||
            (rc = el_alloc(h, &h->flags, 2)))
            break;
        RpyBlockDesc bd{};
        bd.wall = 1;
        bd.vd = 6;
        bd.fd = 6;
        bd.self_set = 1;
        bd.nt = bd.ns = h->N;
        bd.xt = bd.xs = h->x4;
        h->scratch_cap = rpy_plan_for(bd, h->num_sms).scratch_float4;
        if ((rc = el_alloc(h, &h->scratch, h->scratch_cap))) break;
        const size_t inv_smem = sizeof(double) * 36 * S * S;
        if ((rc = cuda_status(cudaFuncSetAttribute(el_invert_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   static_cast<int>(inv_smem)),
                              "cudaFuncSetAttribute", __FILE__, __LINE__)))
            break;
        // initial state (filament.cpp:468-520): straight filaments along +z from their bases, all
        // multipliers zero, the step-0 perturbations of the chosen kind
        std::vector<double> x(3 * N), q(4 * N), zeros(std::max<size_t>(nl, 6 * N), 0.0), pert(6 * F, 0.0);
        for (int m = 0; m < F; ++m)
            for (int k = 0; k < S; ++k) {
                const size_t i = static_cast<size_t>(m) * S + k;
                x[3 * i] = cfg->base_pos[3 * m];
                x[3 * i + 1] = cfg->base_pos[3 * m + 1];
                x[3 * i + 2] = cfg->base_pos[3 * m + 2] + k * h->DL;
                initial_frame(&q[4 * i]);
            }
        const double pmag = 0.01 * h->fend;
        for (int m = 0; m < F; ++m) {
            if (cfg->ic_type == 2) {
                for (int c = 0; c < 6; ++c) pert[6 * m + c] = cfg->perturbations[6 * m + c];
            } else {
                pert[6 * m] = pmag;
                if (cfg->ic_type == 1) pert[6 * m + 4] = pmag;
            }
        }
        auto up = [&](double *dst, const double *src, size_t n) {
            return cuda_status(cudaMemcpy(dst, src, n * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy",
                               __FILE__, __LINE__);
        };
        if ((rc = up(h->x, x.data(), 3 * N)) || (rc = up(h->xm1, x.data(), 3 * N)) ||
            (rc = up(h->xm2, x.data(), 3 * N)) || (rc = up(h->q, q.data(), 4 * N)) ||
            (rc = up(h->qm1, q.data(), 4 * N)) || (rc = up(h->u, zeros.data(), 3 * N)) ||
            (rc = up(h->um1, zeros.data(), 3 * N)) || (rc = up(h->lam, zeros.data(), nl)) ||
            (rc = up(h->lamm1, zeros.data(), nl)) || (rc = up(h->lamm2, zeros.data(), nl)) ||
            (rc = up(h->tet, zeros.data(), 3 * F)) || (rc = up(h->tetm1, zeros.data(), 3 * F)) ||
            (rc = up(h->tetm2, zeros.data(), 3 * F)) || (rc = up(h->clp, zeros.data(), 3 * F)) ||
            (rc = up(h->clpm1, zeros.data(), 3 * F)) || (rc = up(h->clpm2, zeros.data(), 3 * F)) ||
            (rc = up(h->pert, pert.data(), 6 * F)) || (rc = up(h->base, cfg->base_pos, 3 * F)) ||
            (rc = up(h->f, zeros.data(), 6 * N)))
            break;
        if ((rc = cuda_status(cudaMemset(h->flags, 0, 2 * sizeof(int)), "cudaMemset", __FILE__, __LINE__))) break;
    } while (0);
    if (rc != CF_OK) {
        const std::string msg = cf_last_error();
        cf_elastic_destroy(h);
        return set_error(rc, "%s", msg.c_str());
    }
    *out = h;
    return CF_OK;
}

// One implicit step nt (cilia_sim_main.cu:405-560 for elastic filaments on a wall).
extern "C" int cf_elastic_step(cf_elastic *h, int nt, int *broyden_iters) {
    clear_error();
    CF_REQUIRE(h && nt >= 0, "cf_elastic_step: bad arguments");
    CF_CUDA(cudaSetDevice(h->device));
    cudaStream_t st = h->stream;
    el_initial_guess_kernel<<<h->F, 32, 0, st>>>(dev(h), nt);
    CF_CHECK_LAUNCH("el_initial_guess_kernel");
    CF_TRY(evaluate(h, nt, h->err));
    int fl = 0;
    CF_TRY(read_flags(h, &fl));
    if (fl & kNonFinite) return set_error(CF_NONFINITE, "cf_elastic: non-finite residual at step %d", nt);
    bool too_large = (fl & kTooLarge) != 0;
    if (too_large) {
        CF_TRY(prepare_jacobian(h, nt));
        CF_TRY(read_flags(h, &fl));
        if (fl & kNonFinite) return set_error(CF_NONFINITE, "cf_elastic: singular approximate Jacobian at step %d", nt);
    }
    int iter = 0;
    while (too_large && iter < h->maxb) {
        CF_TRY(find_update(h, iter));
        el_update_kernel<<<h->F, 32, 0, st>>>(dev(h), h->upd);
        CF_CHECK_LAUNCH("el_update_kernel");
        CF_TRY(evaluate(h, nt, h->nerr));
        CF_TRY(read_flags(h, &fl));
        if (fl & kNonFinite) {
            h->last_iters = iter + 1;
            return set_error(CF_NONFINITE, "cf_elastic: Broyden's method diverged after %d iterations at step %d",
                             iter + 1, nt);
        }
        too_large = (fl & kTooLarge) != 0;
        if (too_large && iter < h->maxb - 1) CF_TRY(end_of_iter(h, iter));
        ++iter;
    }
    h->last_iters = iter;
    h->total_iters += iter;
    h->max_iters = std::max(h->max_iters, iter);
    h->steps += 1;
    h->stepped = true;
    if (broyden_iters) *broyden_iters = iter;
    if (too_large)
        return set_error(CF_NOT_CONVERGED, "cf_elastic: Broyden's method did not converge within %d iterations at step %d",
                         h->maxb, nt);
    return CF_OK;
}

// Segment positions [3N] and orientations [4N] (FP64), the internal forces and torques [6N] of the
// last evaluation; any pointer may be NULL.
extern "C" int cf_elastic_get_segments(cf_elastic *h, double *x, double *q, double *f) {
    clear_error();
    CF_REQUIRE(h, "null handle");
    CF_CUDA(cudaSetDevice(h->device));
    const size_t N = h->N;
    if (x) CF_CUDA(cudaMemcpyAsync(x, h->x, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (q) CF_CUDA(cudaMemcpyAsync(q, h->q, 4 * N * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (f) CF_CUDA(cudaMemcpyAsync(f, h->f, 6 * N * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CF_CUDA(cudaStreamSynchronize(h->stream));
    return CF_OK;
}

// The approximate inverse Jacobian block [6S x 6S, row-major] of filament m as last prepared, and the
// residual vector [6 N] of the start of the last step's solve (err) -- both for checking.
extern "C" int cf_elastic_get_jacobian_inverse(cf_elastic *h, int m, double *jinv) {
    clear_error();
    CF_REQUIRE(h && jinv && m >= 0 && m < h->F, "cf_elastic_get_jacobian_inverse: bad arguments");
    CF_CUDA(cudaSetDevice(h->device));
    const size_t n = 6 * static_cast<size_t>(h->S);
    CF_CUDA(cudaMemcpyAsync(jinv, h->jinv + n * n * m, n * n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CF_CUDA(cudaStreamSynchronize(h->stream));
    return CF_OK;
}

// Broyden statistics: iterations of the last step, the largest and the total over the steps taken.
extern "C" int cf_elastic_stats(cf_elastic *h, int *last, int *max_iters, long long *total, int *steps) {
    clear_error();
    CF_REQUIRE(h, "null handle");
    if (last) *last = h->last_iters;
    if (max_iters) *max_iters = h->max_iters;
    if (total) *total = h->total_iters;
    if (steps) *steps = h->steps;
    return CF_OK;
}

// Prepares the approximate Jacobian for the current state as the step's first evaluation would,
// without iterating (runs the initial guess and one evaluation of step nt); for checking.
extern "C" int cf_elastic_first_evaluation(cf_elastic *h, int nt, double *err_out) {
    clear_error();
    CF_REQUIRE(h && nt >= 0, "cf_elastic_first_evaluation: bad arguments");
    CF_CUDA(cudaSetDevice(h->device));
    el_initial_guess_kernel<<<h->F, 32, 0, h->stream>>>(dev(h), nt);
    CF_CHECK_LAUNCH("el_initial_guess_kernel");
    CF_TRY(evaluate(h, nt, h->err));
    CF_TRY(prepare_jacobian(h, nt));
    int fl = 0;
    CF_TRY(read_flags(h, &fl));
    if (err_out) {
        CF_CUDA(cudaMemcpy(err_out, h->err, sizeof(double) * h->NB, cudaMemcpyDeviceToHost));
    }
    if (fl & kNonFinite) return set_error(CF_NONFINITE, "cf_elastic: non-finite residual or singular Jacobian");
    return CF_OK;
}

extern "C" int cf_elastic_system_size(cf_elastic *h) { return h ? h->NB : -1; }

// rpy_pairs.cuh -- FP32 device blocks of the RPY grand mobility matrix.
//
// Same mathematics as the reference's rpy_interaction<vel_dof, force_dof>
// (src/cilia/cuda_functions.cu:9-358), rearranged for the FP32 pipe:
//   * the wall blocks (Swan & Brady 2007, reference sign convention for the
//     rotation-translation couplings, cuda_functions.cu:12-203) assume a = 1,
//     mu = 1 as the reference does (cuda_functions.cu:22);
//   * the unbounded blocks carry radii and viscosity (cuda_functions.cu:205-356).
// Forces f[0..2], torques f[3..5]; velocities v[0..2], angular velocities v[3..5].
// Pair functions take d = x_i - x_j and the two heights separately so that the
// tile loops keep only differences in registers.
#pragma once

#include <cuda_runtime.h>

namespace cufil {

struct RpyConst {
    static constexpr float inv6pi = 0.053051647697298445f;   // 1/(6 pi)
    static constexpr float inv8pi = 0.039788735772973836f;   // 1/(8 pi)
};

// Self block of one unit sphere at height z above the wall
// (cuda_functions.cu:24-61).  Evaluated once per target, outside the tiles.
template <int VD, int FD>
__device__ __forceinline__ void wall_self_f32(float z, const float *f, float *v) {
    const float h1 = 1.0f / z;
    const float h3 = h1 * h1 * h1;
    const float h4 = h3 * h1;
    const float h5 = h4 * h1;
    const float c = RpyConst::inv6pi;
    const float m_par = c - (9.0f * h1 - 2.0f * h3 + h5) * (c * 0.0625f);
    const float m_perp = c - (9.0f * h1 - 4.0f * h3 + h5) * (c * 0.125f);
    const float c_tr = (3.0f / 32.0f) * c * h4;
    v[0] += m_par * f[0];
    v[1] += m_par * f[1];
    v[2] += m_perp * f[2];
    if constexpr (FD > 3) {
        v[0] += c_tr * f[4];
        v[1] -= c_tr * f[3];
    }
    if constexpr (VD > 3) {
        v[3] -= c_tr * f[1];
        v[4] += c_tr * f[0];
        if constexpr (FD > 3) {
            const float r_par = RpyConst::inv8pi - (15.0f / 64.0f) * c * h3;
            const float r_perp = RpyConst::inv8pi - (3.0f / 32.0f) * c * h3;
            v[3] += r_par * f[3];
            v[4] += r_par * f[4];
            v[5] += r_perp * f[5];
        }
    }
}

// Pair block i <- j above the wall (cuda_functions.cu:63-200).
//   dx, dy, dz = x_i - x_j;  zi, zj heights;  f = source force (+ torque).
// Constants 1/(6 pi), 1/(8 pi) are folded into the coefficients.
template <int VD, int FD>
__device__ __forceinline__ void wall_pair_f32(float dx, float dy, float dz, float zi, float zj,
                                              const float *f, float *v) {
    const float c6 = RpyConst::inv6pi;
    const float c8 = RpyConst::inv8pi;
    const float q2 = dx * dx + dy * dy;

    // ---- free-space RPY of two unit spheres ----
    const float s = rsqrtf(fmaf(dz, dz, q2));
    const float s2 = s * s;
    const float df = dx * f[0] + dy * f[1] + dz * f[2];     // d . F
    const float g = c8 * s;
    const float a_iso = g * fmaf(2.0f / 3.0f, s2, 1.0f);   // (1 + 2/(3 r^2)) / (8 pi r)
    const float a_dir = g * fmaf(-2.0f, s2, 1.0f) * df * s2; // coefficient of d
    v[0] += a_iso * f[0] + a_dir * dx;
    v[1] += a_iso * f[1] + a_dir * dy;
    v[2] += a_iso * f[2] + a_dir * dz;
    if constexpr (FD > 3 || VD > 3) {
        const float g2 = g * s2;  // 1/(8 pi r^3): multiplies d (not the unit vector)
        if constexpr (FD > 3) {
            v[0] += g2 * (f[4] * dz - f[5] * dy);
            v[1] += g2 * (f[5] * dx - f[3] * dz);
            v[2] += g2 * (f[3] * dy - f[4] * dx);
        }
        if constexpr (VD > 3) {
            v[3] += g2 * (f[1] * dz - f[2] * dy);
            v[4] += g2 * (f[2] * dx - f[0] * dz);
            v[5] += g2 * (f[0] * dy - f[1] * dx);
            if constexpr (FD > 3) {
                const float dt = dx * f[3] + dy * f[4] + dz * f[5];
                const float q = 0.5f * g * s2;  // 1/(16 pi r^3)
                const float qd = 3.0f * q * dt * s2;
                v[3] += qd * dx - q * f[3];
                v[4] += qd * dy - q * f[4];
                v[5] += qd * dz - q * f[5];
            }
        }
    }

    // ---- image system ----
    const float hz = zi + zj;
    const float w = rsqrtf(fmaf(hz, hz, q2));
    const float w2 = w * w, w3 = w2 * w, w4 = w2 * w2, w5 = w4 * w;
    const float ex = dx * w, ey = dy * w, ez = hz * w;
    const float h = __fdividef(zj, hz);
    const float ez2 = ez * ez;
    const float ef = ex * f[0] + ey * f[1] + ez * f[2];
    const float hh = h * (1.0f - h);
    const float t5 = fmaf(-5.0f, ez2, 1.0f);
    {
        const float k0 = -(0.75f * w * fmaf(2.0f * hh, ez2, 1.0f)
                           + 0.5f * (w3 * fmaf(-3.0f, ez2, 1.0f) - w5 * t5));
        const float k1 = -(0.75f * w * fmaf(-6.0f * hh, ez2, 1.0f) - 1.5f * w3 * t5
                           + 2.5f * w5 * fmaf(-7.0f, ez2, 1.0f)) * ef;
        const float k2 = ez * f[2] * (1.5f * h * w * fmaf(-6.0f * (1.0f - h), ez2, 1.0f)
                                      - 3.0f * w3 * t5 + 5.0f * w5 * fmaf(-7.0f, ez2, 2.0f));
        const float k3 = (1.5f * h * w - 5.0f * w5) * ef;
        const float k4 = -((3.0f * h * h * w + 3.0f * w3) * ez2 + fmaf(-15.0f, ez2, 2.0f) * w5) * f[2];
        const float k12 = c6 * (k1 + k2);
        const float k0c = c6 * k0;
        v[0] += k0c * f[0] + k12 * ex;
        v[1] += k0c * f[1] + k12 * ey;
        v[2] += k0c * f[2] + (k12 + c6 * k3) * ez + c6 * k4;
    }
    if constexpr (VD > 3) {
        const float b0 = 0.75f * w2;
        const float b1 = f[2] * (9.0f * h * ez2 * w2 + fmaf(-15.0f, ez2, 1.5f) * w4);
        const float b2 = -ez * ef * (4.5f * h * w2 - 7.5f * w4);
        const float b3 = -1.5f * ez * (h * w2 - w4);
        v[3] -= c6 * (b0 * (f[1] * ez - f[2] * ey) - (b1 + b2) * ey + b3 * f[1]);
        v[4] -= c6 * (b0 * (f[2] * ex - f[0] * ez) + (b1 + b2) * ex - b3 * f[0]);
        v[5] -= c6 * b0 * (f[0] * ey - f[1] * ex);
        if constexpr (FD > 3) {
            const float et = ex * f[3] + ey * f[4] + ez * f[5];
            const float d0 = w3 * fmaf(-2.25f, ez2, 0.375f);
            const float d1 = -1.125f * w3 * et;
            const float d2 = 2.25f * ez * w3 * et;
            const float d3 = 2.25f * w3 * (ex * f[4] - ey * f[3]);
            v[3] += c6 * (d0 * f[3] + d1 * ex - d3 * ey);
            v[4] += c6 * (d0 * f[4] + d1 * ey + d3 * ex);
            v[5] += c6 * (d0 * f[5] + d1 * ez + d2);
        }
    }
    if constexpr (FD > 3) {
        // translation from torque: transpose of the rotation-from-force block
        // with i and j swapped (h -> 1-h, in-plane e flips sign).
        const float hs = 1.0f - h;
        const float fx = -ex, fy = -ey;
        const float ext = fx * f[4] - fy * f[3];
        const float g0 = 0.75f * w2;
        const float g1 = (9.0f * hs * ez2 * w2 + fmaf(-15.0f, ez2, 1.5f) * w4) * ext;
        const float g2 = -ez * (4.5f * hs * w2 - 7.5f * w4) * ext;
        const float g3 = -1.5f * ez * (hs * w2 - w4);
        v[0] -= c6 * (g0 * (f[5] * fy - f[4] * ez) + g2 * fx - g3 * f[4]);
        v[1] -= c6 * (g0 * (f[3] * ez - f[5] * fx) + g2 * fy + g3 * f[3]);
        v[2] -= c6 * (g0 * (f[4] * fx - f[3] * fy) + g2 * ez + g1);
    }
}

// Unbounded RPY pair with radii ai, aj and viscosity mu (cuda_functions.cu:205-356),
// including the overlap (r < ai + aj) and containment (r < |ai - aj|) branches.
// Coincident centres are not special-cased (1/(r + 1e-20)), which yields the
// self-mobility through the containment branch exactly as in the reference.
template <int VD, int FD>
__device__ __forceinline__ void free_pair_f32(float dx, float dy, float dz, float ai, float aj,
                                              float inv_mu, const float *f, float *v) {
    const float pi = 3.14159265358979f;
    const float r2 = dx * dx + dy * dy + dz * dz;
    const float r = sqrtf(r2);
    const float s = 1.0f / (r + 1e-20f);
    const float dmin = fabsf(ai - aj);
    const float asum = ai + aj;
    const float ux = dx * s, uy = dy * s, uz = dz * s;
    const float uf = ux * f[0] + uy * f[1] + uz * f[2];
    const bool far = r > asum;
    const bool overlap = !far && (r > dmin);
    float A, B;
    if (far) {
        const float q = s * s * (ai * ai + aj * aj) * (1.0f / 3.0f);
        const float c = s * inv_mu * (1.0f / (8.0f * pi));
        A = (1.0f + q) * c;
        B = (1.0f - 3.0f * q) * c * uf;
    } else if (overlap) {
        const float den = 1.0f / (32.0f * r2 * r);
        const float t1 = dmin * dmin + 3.0f * r2;
        const float t2 = dmin * dmin - r2;
        const float c = inv_mu / (6.0f * pi * ai * aj);
        A = (0.5f * asum - t1 * t1 * den) * c;
        B = 3.0f * t2 * t2 * den * c * uf;
    } else {
        A = inv_mu / (6.0f * pi * fmaxf(ai, aj));
        B = 0.0f;
    }
    v[0] += A * f[0] + B * ux;
    v[1] += A * f[1] + B * uy;
    v[2] += A * f[2] + B * uz;
    if constexpr (FD > 3) {
        if (far) {
            A = s * s * inv_mu * (1.0f / (8.0f * pi));
        } else if (overlap) {
            const float wv = aj - ai + r;
            A = wv * wv * s * s * (ai * ai + 2.0f * ai * (r + aj) - 3.0f * (aj - r) * (aj - r)) * inv_mu
                / (128.0f * pi * ai * aj * aj * aj);
        } else {
            A = (aj > ai ? r : 0.0f) * inv_mu / (8.0f * pi * aj * aj * aj);
        }
        v[0] += A * (f[4] * uz - f[5] * uy);
        v[1] += A * (f[5] * ux - f[3] * uz);
        v[2] += A * (f[3] * uy - f[4] * ux);
    }
    if constexpr (VD > 3) {
        if (far) {
            A = s * s * inv_mu * (1.0f / (8.0f * pi));
        } else if (overlap) {
            const float wv = ai - aj + r;
            A = wv * wv * s * s * (aj * aj + 2.0f * aj * (r + ai) - 3.0f * (ai - r) * (ai - r)) * inv_mu
                / (128.0f * pi * aj * ai * ai * ai);
        } else {
            A = (ai > aj ? r : 0.0f) * inv_mu / (8.0f * pi * ai * ai * ai);
        }
        v[3] += A * (f[1] * uz - f[2] * uy);
        v[4] += A * (f[2] * ux - f[0] * uz);
        v[5] += A * (f[0] * uy - f[1] * ux);
        if constexpr (FD > 3) {
            const float ut = ux * f[3] + uy * f[4] + uz * f[5];
            if (far) {
                A = -s * s * s * inv_mu * (1.0f / (16.0f * pi));
                B = -3.0f * ut * A;
            } else if (overlap) {
                const float r3 = r2 * r;
                const float ai2 = ai * ai, aj2 = aj * aj;
                const float dd = dmin * dmin;
                A = 5.0f * r3 * r3 - 27.0f * r2 * r2 * (ai2 + aj2) + 32.0f * r3 * (ai2 * ai + aj2 * aj)
                    - 9.0f * r2 * (ai2 - aj2) * (ai2 - aj2) - dd * dd * (ai2 + aj2 + 4.0f * ai * aj);
                const float t = (ai - aj) * (ai - aj) - r2;
                B = 3.0f * t * t * (ai2 + aj2 + 4.0f * ai * aj - r2);
                const float c = inv_mu / (512.0f * pi * r3 * ai2 * ai * aj2 * aj);
                A *= c;
                B *= c * ut;
            } else {
                const float am = fmaxf(ai, aj);
                A = inv_mu / (8.0f * pi * am * am * am);
                B = 0.0f;
            }
            v[3] += A * f[3] + B * ux;
            v[4] += A * f[4] + B * uy;
            v[5] += A * f[5] + B * uz;
        }
    }
}

}  // namespace cufil

namespace cufil {

// Both directions of one wall pair from a single block evaluation.
//   d = x_i - x_j, hz = z_i + z_j; fj, fi: source forces of j and i.
//   vi += M(i <- j) fj,  vj += M(j <- i) fi = M(i <- j)^T fi.
// The grand mobility is symmetric, so the image block is written as
//   M = c6 [k0 I + a d' d'^T + b d' z^T + c z d'^T + k4 z z^T],  d' = (dx, dy, hz),
// with the coefficients of the reference's wall branch (cuda_functions.cu:118-150)
// regrouped: a = alpha w^2, b = beta w, c = gamma w^2 hz (w = 1/|d'|).
__device__ __forceinline__ void wall_pair_sym_f32(float dx, float dy, float dz, float zi, float zj, const float *fj,
                                                  const float *fi, float *vi, float *vj) {
    const float c6 = RpyConst::inv6pi;
    const float c8 = RpyConst::inv8pi;
    const float q2 = dx * dx + dy * dy;
    // free space: M = A I + B d d^T (even in d)
    const float s = rsqrtf(fmaf(dz, dz, q2));
    const float s2 = s * s;
    const float g = c8 * s;
    const float A = g * fmaf(2.0f / 3.0f, s2, 1.0f);
    const float B = g * fmaf(-2.0f, s2, 1.0f) * s2;
    // image system
    const float hz = zi + zj;
    const float hz2 = hz * hz;
    const float w = rsqrtf(q2 + hz2);
    const float w2 = w * w, w3 = w2 * w, w5 = w3 * w2;
    const float h = __fdividef(zj, hz);
    const float hm = 1.0f - h;
    const float ez2 = w2 * hz2;
    const float hh = h * hm;
    const float t5 = fmaf(-5.0f, ez2, 1.0f);
    const float w075 = 0.75f * w;
    const float hw15 = 1.5f * h * w;
    const float k0 = -(w075 * fmaf(2.0f * hh, ez2, 1.0f) + 0.5f * (w3 * fmaf(-3.0f, ez2, 1.0f) - w5 * t5));
    const float al = -(w075 * fmaf(-6.0f * hh, ez2, 1.0f) - 1.5f * w3 * t5 + 2.5f * w5 * fmaf(-7.0f, ez2, 1.0f));
    const float be = (hz * w) * (hw15 * fmaf(-6.0f * hm, ez2, 1.0f) - 3.0f * w3 * t5 + 5.0f * w5 * fmaf(-7.0f, ez2, 2.0f));
    const float ga = hw15 - 5.0f * w5;
    const float de = -((3.0f * h * h * w + 3.0f * w3) * ez2 + fmaf(-15.0f, ez2, 2.0f) * w5);
    const float K0 = c6 * k0;
    const float a = c6 * al * w2;
    const float b = c6 * be * w;
    const float c = c6 * ga * w2 * hz;
    const float e = c6 * de;
    // i <- j
    {
        const float dF = dx * fj[0] + dy * fj[1] + dz * fj[2];
        const float dpF = dx * fj[0] + dy * fj[1] + hz * fj[2];
        const float t0 = B * dF;
        const float t1 = a * dpF + b * fj[2];
        const float t2 = c * dpF + e * fj[2];
        const float AK = A + K0;
        vi[0] += AK * fj[0] + t0 * dx + t1 * dx;
        vi[1] += AK * fj[1] + t0 * dy + t1 * dy;
        vi[2] += AK * fj[2] + t0 * dz + t1 * hz + t2;
    }
    // j <- i (transpose)
    {
        const float dF = dx * fi[0] + dy * fi[1] + dz * fi[2];
        const float dpF = dx * fi[0] + dy * fi[1] + hz * fi[2];
        const float t0 = B * dF;
        const float t1 = a * dpF + c * fi[2];
        const float t2 = b * dpF + e * fi[2];
        const float AK = A + K0;
        vj[0] += AK * fi[0] + t0 * dx + t1 * dx;
        vj[1] += AK * fi[1] + t0 * dy + t1 * dy;
        vj[2] += AK * fi[2] + t0 * dz + t1 * hz + t2;
    }
}

// Unbounded RPY pair of two equal spheres (radius a) in both directions: the block M = A I + B u u^T is the
// same for i <- j and j <- i (u changes sign, u u^T does not), so one evaluation serves both.  Branches as in
// free_pair_f32 with ai = aj = a (far; overlapping, with dmin = 0; coincident: the self mobility).
__device__ __forceinline__ void free_pair_sym_f32(float dx, float dy, float dz, float a, float inv_mu, const float *fj,
                                                  const float *fi, float *vi, float *vj) {
    const float pi = 3.14159265358979f;
    const float r2 = dx * dx + dy * dy + dz * dz;
    const float r = sqrtf(r2);
    const float s = 1.0f / (r + 1e-20f);
    const float ux = dx * s, uy = dy * s, uz = dz * s;
    float A, Bc;
    if (r > 2.0f * a) {
        const float q = s * s * (2.0f * a * a) * (1.0f / 3.0f);
        const float c = s * inv_mu * (1.0f / (8.0f * pi));
        A = (1.0f + q) * c;
        Bc = (1.0f - 3.0f * q) * c;
    } else if (r > 0.0f) {
        const float c = inv_mu / (6.0f * pi * a * a);
        A = (a - (9.0f / 32.0f) * r) * c;
        Bc = (3.0f / 32.0f) * r * c;
    } else {
        A = inv_mu / (6.0f * pi * a);
        Bc = 0.0f;
    }
    const float tj = Bc * (ux * fj[0] + uy * fj[1] + uz * fj[2]);
    const float ti = Bc * (ux * fi[0] + uy * fi[1] + uz * fi[2]);
    vi[0] += A * fj[0] + tj * ux;
    vi[1] += A * fj[1] + tj * uy;
    vi[2] += A * fj[2] + tj * uz;
    vj[0] += A * fi[0] + ti * ux;
    vj[1] += A * fi[1] + ti * uy;
    vj[2] += A * fi[2] + ti * uz;
}

}  // namespace cufil

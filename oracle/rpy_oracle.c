/*
 * rpy_oracle.c -- CPU restatement of the reference's Rotne-Prager-Yamakawa pair
 * mobility, used ONLY as test infrastructure (the parity checker and the timed
 * CPU baseline).  Nothing in the product links or calls this file.
 *
 * Follows racksa/CUFCM_FIL  src/cilia/cuda_functions.cu:
 *   - rpy_interaction<vel_dof,force_dof>, wall branch (Swan & Brady 2007 with the
 *     reference's sign convention for the rot-trans terms)   :12-203
 *       self block                                             :24-61
 *       free-space part of a pair                              :63-116
 *       wall image part of a pair                              :118-200
 *     The wall branch assumes mu = 1 and a = 1 exactly as the reference does
 *     (cuda_functions.cu:22); radii passed in are ignored there.
 *   - rpy_interaction unbounded branch (Zuk et al. 2014, unequal radii,
 *     overlap and containment branches)                        :205-356
 *   - the block products Mss/Mbb/Msb/Mbs                        :362-757
 *     are expressed by oracle_rpy_apply_*: V_t += M(t <- s) F_s.
 *
 * The arithmetic type is selected at compile time (ORACLE_REAL = double or
 * float); the build compiles this file twice, exporting *_f64 and *_f32.
 * Parity status: pinned against the reference's own generalised-force tables
 * (single filament above a wall) and against the reference's CUDA kernels run
 * on the same inputs (see the tests).
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef ORACLE_REAL
#define ORACLE_REAL double
#define ORACLE_SUFFIX f64
#endif

typedef ORACLE_REAL R;

#define CAT2(a, b) a##_##b
#define CAT(a, b) CAT2(a, b)
#define EXPORT(name) CAT(name, ORACLE_SUFFIX)

static const R kPi = (R)3.14159265358979323846264338327950288;

/* ------------------------------------------------------------------------- */
/* Wall-bounded (z = 0 no-slip plane) blocks, unit radius, unit viscosity.    */
/* ------------------------------------------------------------------------- */

/* Self-mobility of one sphere at height z (cuda_functions.cu:24-61). */
static void wall_self(int vdof, int fdof, R z, const R *f, R *v)
{
    const R inv6pi = (R)1 / ((R)6 * kPi);
    const R inv8pi = (R)1 / ((R)8 * kPi);
    const R h1 = (R)1 / z;
    const R h3 = h1 * h1 * h1;
    const R h4 = h3 * h1;
    const R h5 = h4 * h1;

    /* parallel and normal translational self-mobility */
    const R m_par = inv6pi - ((R)9 * h1 - (R)2 * h3 + h5) * inv6pi / (R)16;
    const R m_perp = inv6pi - ((R)9 * h1 - (R)4 * h3 + h5) * inv6pi / (R)8;
    /* translation-rotation coupling magnitude, 3/(6 pi 32) h^-4 */
    const R c_tr = (R)3 * inv6pi / (R)32 * h4;

    v[0] += m_par * f[0];
    v[1] += m_par * f[1];
    v[2] += m_perp * f[2];
    if (fdof > 3) {
        v[0] += c_tr * f[4];
        v[1] -= c_tr * f[3];
    }
    if (vdof > 3) {
        v[3] -= c_tr * f[1];
        v[4] += c_tr * f[0];
        if (fdof > 3) {
            const R r_par = inv8pi - (R)15 * inv6pi / (R)64 * h3;
            const R r_perp = inv8pi - (R)3 * inv6pi / (R)32 * h3;
            v[3] += r_par * f[3];
            v[4] += r_par * f[4];
            v[5] += r_perp * f[5];
        }
    }
}

/* Pair block i <- j for two distinct spheres above the wall
 * (cuda_functions.cu:63-200).  d = x_i - x_j. */
static void wall_pair(int vdof, int fdof, const R *xi, const R *xj, const R *f, R *v)
{
    const R inv6pi = (R)1 / ((R)6 * kPi);
    const R inv8pi = (R)1 / ((R)8 * kPi);
    const R dx = xi[0] - xj[0], dy = xi[1] - xj[1], dz = xi[2] - xj[2];

    /* ---- free-space RPY for non-overlapping unit spheres ---- */
    R s = (R)1 / sqrt(dx * dx + dy * dy + dz * dz);
    const R ux = dx * s, uy = dy * s, uz = dz * s;
    const R uf = ux * f[0] + uy * f[1] + uz * f[2];
    R g = inv8pi * s;
    {
        const R iso = (R)1 + (R)2 / (R)3 * s * s;
        const R aniso = ((R)1 - (R)2 * s * s) * uf;
        v[0] += g * (iso * f[0] + aniso * ux);
        v[1] += g * (iso * f[1] + aniso * uy);
        v[2] += g * (iso * f[2] + aniso * uz);
    }
    g *= s; /* 1/(8 pi r^2) */
    if (fdof > 3) { /* translation from torque: (T x u)/(8 pi r^2) */
        v[0] += g * (f[4] * uz - f[5] * uy);
        v[1] += g * (f[5] * ux - f[3] * uz);
        v[2] += g * (f[3] * uy - f[4] * ux);
    }
    if (vdof > 3) { /* rotation from force: (F x u)/(8 pi r^2) */
        v[3] += g * (f[1] * uz - f[2] * uy);
        v[4] += g * (f[2] * ux - f[0] * uz);
        v[5] += g * (f[0] * uy - f[1] * ux);
        if (fdof > 3) { /* rotation from torque: (3 (u.T) u - T)/(16 pi r^3) */
            const R ut = ux * f[3] + uy * f[4] + uz * f[5];
            const R q = g * (R)0.5 * s;
            v[3] += q * ((R)3 * ut * ux - f[3]);
            v[4] += q * ((R)3 * ut * uy - f[4]);
            v[5] += q * ((R)3 * ut * uz - f[5]);
        }
    }

    /* ---- image system: e is the unit vector from the image of j to i ---- */
    const R hz = xi[2] + xj[2];
    s = (R)1 / sqrt(dx * dx + dy * dy + hz * hz);
    const R s2 = s * s, s3 = s2 * s, s4 = s3 * s, s5 = s4 * s;
    const R ex = dx * s, ey = dy * s, ez = hz * s;
    const R h = xj[2] / hz;
    const R ez2 = ez * ez;
    const R ef = ex * f[0] + ey * f[1] + ez * f[2];

    {
        const R k0 = -((R)0.75 * s * ((R)1 + (R)2 * h * ((R)1 - h) * ez2)
                       + (R)0.5 * (s3 * ((R)1 - (R)3 * ez2) - s5 * ((R)1 - (R)5 * ez2)));
        const R k1 = -((R)0.75 * s * ((R)1 - (R)6 * h * ((R)1 - h) * ez2)
                       - (R)1.5 * s3 * ((R)1 - (R)5 * ez2)
                       + (R)2.5 * s5 * ((R)1 - (R)7 * ez2)) * ef;
        const R k2 = ez * f[2] * ((R)1.5 * h * s * ((R)1 - (R)6 * ((R)1 - h) * ez2)
                                  - (R)3 * s3 * ((R)1 - (R)5 * ez2)
                                  + (R)5 * s5 * ((R)2 - (R)7 * ez2));
        const R k3 = ((R)1.5 * h * s - (R)5 * s5) * ef;
        const R k4 = -(((R)3 * h * h * s + (R)3 * s3) * ez2 + ((R)2 - (R)15 * ez2) * s5) * f[2];
        v[0] += inv6pi * (k0 * f[0] + (k1 + k2) * ex);
        v[1] += inv6pi * (k0 * f[1] + (k1 + k2) * ey);
        v[2] += inv6pi * (k0 * f[2] + (k1 + k2 + k3) * ez + k4);
    }

    if (vdof > 3) {
        /* rotation of i due to force on j (reference sign convention) */
        const R b0 = (R)0.75 * s2;
        const R b1 = f[2] * ((R)9 * h * ez2 * s2 + ((R)1.5 - (R)15 * ez2) * s4);
        const R b2 = -ez * ef * ((R)4.5 * h * s2 - (R)7.5 * s4);
        const R b3 = -(R)1.5 * ez * (h * s2 - s4);
        v[3] -= inv6pi * (b0 * (f[1] * ez - f[2] * ey) - (b1 + b2) * ey + b3 * f[1]);
        v[4] -= inv6pi * (b0 * (f[2] * ex - f[0] * ez) + (b1 + b2) * ex - b3 * f[0]);
        v[5] -= inv6pi * b0 * (f[0] * ey - f[1] * ex);
        if (fdof > 3) {
            const R et = ex * f[3] + ey * f[4] + ez * f[5];
            const R d0 = s3 * ((R)0.375 - (R)2.25 * ez2);
            const R d1 = -(R)1.125 * s3 * et;
            const R d2 = (R)2.25 * ez * s3 * et;
            const R d3 = (R)2.25 * s3 * (ex * f[4] - ey * f[3]);
            v[3] += inv6pi * (d0 * f[3] + d1 * ex - d3 * ey);
            v[4] += inv6pi * (d0 * f[4] + d1 * ey + d3 * ex);
            v[5] += inv6pi * (d0 * f[5] + d1 * ez + d2);
        }
    }

    if (fdof > 3) {
        /* translation of i due to torque on j, from the transpose of the
         * rotation-from-force block with the roles of i and j swapped:
         * h -> 1 - h and the in-plane components of e flip sign. */
        const R hs = (R)1 - h;
        const R fx = -ex, fy = -ey;
        const R ext = fx * f[4] - fy * f[3];
        const R g0 = (R)0.75 * s2;
        const R g1 = ((R)9 * hs * ez2 * s2 + ((R)1.5 - (R)15 * ez2) * s4) * ext;
        const R g2 = -ez * ((R)4.5 * hs * s2 - (R)7.5 * s4) * ext;
        const R g3 = -(R)1.5 * ez * (hs * s2 - s4);
        v[0] -= inv6pi * (g0 * (f[5] * fy - f[4] * ez) + g2 * fx - g3 * f[4]);
        v[1] -= inv6pi * (g0 * (f[3] * ez - f[5] * fx) + g2 * fy + g3 * f[3]);
        v[2] -= inv6pi * (g0 * (f[4] * fx - f[3] * fy) + g2 * ez + g1);
    }
}

/* ------------------------------------------------------------------------- */
/* Unbounded RPY with unequal radii (cuda_functions.cu:205-356).             */
/* ------------------------------------------------------------------------- */
static void free_pair(int vdof, int fdof, const R *xi, R ai, const R *xj, R aj, R mu,
                      const R *f, R *v)
{
    R dx = xi[0] - xj[0], dy = xi[1] - xj[1], dz = xi[2] - xj[2];
    const R r = sqrt(dx * dx + dy * dy + dz * dz);
    const R s = (R)1 / (r + (R)1e-20); /* coincident centres are not special-cased */
    const R dmin = fabs(ai - aj);
    const R asum = ai + aj;
    dx *= s; dy *= s; dz *= s;

    R A, B;
    R uf = dx * f[0] + dy * f[1] + dz * f[2];
    if (r > asum) {
        const R q = s * s * (ai * ai + aj * aj) / (R)3;
        const R c = s / ((R)8 * kPi * mu);
        A = ((R)1 + q) * c;
        B = ((R)1 - (R)3 * q) * c * uf;
    } else if (r > dmin) {
        const R den = (R)32 * r * r * r;
        const R t1 = dmin * dmin + (R)3 * r * r;
        const R t2 = dmin * dmin - r * r;
        const R c = (R)1 / ((R)6 * kPi * mu * ai * aj);
        A = ((R)0.5 * asum - t1 * t1 / den) * c;
        B = (R)3 * t2 * t2 / den * c * uf;
    } else {
        A = (R)1 / ((R)6 * kPi * mu * (ai > aj ? ai : aj));
        B = (R)0;
    }
    v[0] += A * f[0] + B * dx;
    v[1] += A * f[1] + B * dy;
    v[2] += A * f[2] + B * dz;

    if (fdof > 3) { /* translation from torque */
        if (r > asum) {
            A = s * s / ((R)8 * kPi * mu);
        } else if (r > dmin) {
            const R w = aj - ai + r;
            A = w * w * s * s * (ai * ai + (R)2 * ai * (r + aj) - (R)3 * (aj - r) * (aj - r))
                / ((R)128 * kPi * mu * ai * aj * aj * aj);
        } else {
            A = (aj > ai ? (R)1 : (R)0) * r / ((R)8 * kPi * mu * aj * aj * aj);
        }
        v[0] += A * (f[4] * dz - f[5] * dy);
        v[1] += A * (f[5] * dx - f[3] * dz);
        v[2] += A * (f[3] * dy - f[4] * dx);
    }
    if (vdof > 3) { /* rotation from force: translation-from-torque with ai <-> aj */
        if (r > asum) {
            A = s * s / ((R)8 * kPi * mu);
        } else if (r > dmin) {
            const R w = ai - aj + r;
            A = w * w * s * s * (aj * aj + (R)2 * aj * (r + ai) - (R)3 * (ai - r) * (ai - r))
                / ((R)128 * kPi * mu * aj * ai * ai * ai);
        } else {
            A = (ai > aj ? (R)1 : (R)0) * r / ((R)8 * kPi * mu * ai * ai * ai);
        }
        v[3] += A * (f[1] * dz - f[2] * dy);
        v[4] += A * (f[2] * dx - f[0] * dz);
        v[5] += A * (f[0] * dy - f[1] * dx);

        if (fdof > 3) { /* rotation from torque */
            const R ut = dx * f[3] + dy * f[4] + dz * f[5];
            if (r > asum) {
                A = -s * s * s / ((R)16 * kPi * mu);
                B = -(R)3 * ut * A;
            } else if (r > dmin) {
                const R r2 = r * r, r3 = r2 * r;
                const R ai2 = ai * ai, aj2 = aj * aj;
                const R dd = dmin * dmin;
                A = (R)5 * r3 * r3 - (R)27 * r2 * r2 * (ai2 + aj2) + (R)32 * r3 * (ai2 * ai + aj2 * aj)
                    - (R)9 * r2 * (ai2 - aj2) * (ai2 - aj2) - dd * dd * (ai2 + aj2 + (R)4 * ai * aj);
                const R t = (ai - aj) * (ai - aj) - r2;
                B = (R)3 * t * t * (ai2 + aj2 + (R)4 * ai * aj - r2);
                const R c = (R)1 / ((R)512 * kPi * mu * r3 * ai2 * ai * aj2 * aj);
                A *= c;
                B *= c * ut;
            } else {
                const R am = ai > aj ? ai : aj;
                A = (R)1 / ((R)8 * kPi * mu * am * am * am);
                B = (R)0;
            }
            v[3] += A * f[3] + B * dx;
            v[4] += A * f[4] + B * dy;
            v[5] += A * f[5] + B * dz;
        }
    }
}

/* ------------------------------------------------------------------------- */
/* Block products.                                                           */
/* ------------------------------------------------------------------------- */

/*
 * V_t[i] += sum_j M(t_i <- s_j) F_s[j]
 *
 *   wall          1: Swan-Brady wall-bounded blocks (unit radius, unit mu)
 *                 0: unbounded RPY with radii at/as and viscosity mu
 *   vdof, fdof    3 or 6: per-particle velocity / force component counts;
 *                 xt, xs are [n*3], fs is [ns*fdof], vt is [nt*vdof]
 *   t_ids         global ids of the targets (NULL: t_off + i)
 *   s_off         global id of source 0
 *   self_by_index 1: in wall mode a pair whose global ids agree uses the
 *                 self-mobility block (the reference's i == j test,
 *                 cuda_functions.cu:24); 0: never.
 *   nthreads      OpenMP threads (<= 0: runtime default)
 */
void EXPORT(oracle_rpy_apply)(int wall, int vdof, int fdof, int self_by_index,
                              int64_t nt, const R *xt, R at, const int64_t *t_ids, int64_t t_off,
                              int64_t ns, const R *xs, const R *fs, R as, int64_t s_off,
                              R mu, R *vt, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 8)
#endif
    for (int64_t i = 0; i < nt; ++i) {
        R acc[6] = {0, 0, 0, 0, 0, 0};
        const int64_t gi = t_ids ? t_ids[i] : t_off + i;
        const R *xi = xt + 3 * i;
        for (int64_t j = 0; j < ns; ++j) {
            const R *xj = xs + 3 * j;
            const R *fj = fs + fdof * j;
            if (wall) {
                if (self_by_index && gi == s_off + j)
                    wall_self(vdof, fdof, xi[2], fj, acc);
                else
                    wall_pair(vdof, fdof, xi, xj, fj, acc);
            } else {
                free_pair(vdof, fdof, xi, at, xj, as, mu, fj, acc);
            }
        }
        for (int c = 0; c < vdof; ++c) vt[vdof * i + c] += acc[c];
    }
}

/* Number of OpenMP threads the runtime would use (1 without OpenMP). */
int EXPORT(oracle_num_threads)(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// fcm.cu -- cf_fcm: fast force-coupling method in a triply periodic box.
//
// Replaces the reference's FCM_solver (src/cufcm/CUFCM_SOLVER.cu:20-727) for
// translation-only particles (ROTATION 0, src/cufcm/config.hpp:23):
//   wrap + cell hash + sort   box / create_hash_gpu / sort_index_by_key
//                             (CUFCM_DATA.cu:427-460, CUFCM_CELLLIST.cu:57-132)
//   spread                    cufcm_mono_dipole_distribution_bpp_shared_dynamic (CUFCM_FCM.cu:16-184)
//   FFT, Stokes solve, iFFT   cufftExec*, cufcm_flow_solve (CUFCM_SOLVER.cu:538-577, CUFCM_FCM.cu:187-246)
//   gather                    cufcm_particle_velocities_bpp_shared_dynamic (CUFCM_FCM.cu:249-423)
//   pair + self correction    cufcm_pair_correction, cufcm_self_correction (CUFCM_CORRECTION.cu:103-352)
//   sort back                 sortback (CUFCM_SOLVER.cu:493-515)
// Differences in the execution, not the mathematics: one warp per particle for
// spread and gather with the particle's 1-D Gaussian tables in that warp's
// shared memory (no block barriers); the three components' FFTs batched in one
// cuFFT plan each way; the Stokes projector applied in place to the spectra;
// the near-field correction one-sided over all 27 neighbour cells (every pair
// is visited from both ends, so no atomics and a deterministic result); and
// results scattered straight back to input order instead of a second sort.
#include "common.cuh"

#include <cub/cub.cuh>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

struct cf_fcm {
    cf_fcm_config cfg{};
    cudaStream_t stream = nullptr;
    // derived parameters (FCM_solver::init_config / init_fcm_var)
    int N = 0, nx = 0, ny = 0, nz = 0, ngd = 0, Mx = 0, My = 0, Mz = 0, ncell = 0, hash_bits = 1;
    double Lx = 0, Ly = 0, Lz = 0, dx = 0, sigma = 0, Sigma = 0, pdmag = 0, Rc = 0, self_mob = 0;
    size_t grid_size = 0, fft_size = 0;
    // buffers
    float *grid = nullptr;         // 3 real grids, component-major
    cufftComplex *spec = nullptr;  // 3 spectra
    float4 *x4 = nullptr, *xs = nullptr, *fs = nullptr;
    float *ys = nullptr;           // caller-layout staging [3N] (host path)
    float *fsrc = nullptr;         // [3N]
    float *vout = nullptr;         // [3N]
    float4 *vgs = nullptr;         // gathered velocities, sorted order
    int *keys = nullptr, *keys_sorted = nullptr, *vals = nullptr, *perm = nullptr;
    int *cell_start = nullptr, *cell_end = nullptr;
    void *sort_tmp = nullptr;
    size_t sort_tmp_bytes = 0;
    cufftHandle plan_fwd = 0, plan_inv = 0;
    bool have_fwd = false, have_inv = false;
    // optional per-stage timing: events between stages of the last apply
    bool timing = false;
    cudaEvent_t ev[7] = {};
};

namespace cufil {
namespace fcmk {

struct Params {
    int N, nx, ny, nz, ngd, Mx, My, Mz;
    float Lx, Ly, Lz, dx;
    float Sigma, sigma, pdmag, Rcsq, self_mob;
    size_t grid_size, fft_size;
};

__device__ __forceinline__ float wrap_box(float x, float L) {
    // images() of the reference (CUFCM_DATA.cu:448-460)
    x -= floorf(x / L) * L;
    if (x == L) x = 0.0f;
    return x;
}

__global__ void prep_kernel(Params p, const float *__restrict__ Y, float4 *x4, int *keys, int *vals) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.N) return;
    const float x = wrap_box(Y[3 * i], p.Lx), y = wrap_box(Y[3 * i + 1], p.Ly), z = wrap_box(Y[3 * i + 2], p.Lz);
    x4[i] = make_float4(x, y, z, 0.0f);
    int cx = static_cast<int>(x / p.Lx * p.Mx), cy = static_cast<int>(y / p.Ly * p.My),
        cz = static_cast<int>(z / p.Lz * p.Mz);
    cx = min(max(cx, 0), p.Mx - 1);
    cy = min(max(cy, 0), p.My - 1);
    cz = min(max(cz, 0), p.Mz - 1);
    keys[i] = cx + (cy + cz * p.My) * p.Mx;
    vals[i] = i;
}

__global__ void permute_kernel(Params p, const int *__restrict__ perm, const float4 *__restrict__ x4,
                               const float *__restrict__ F, float4 *xs, float4 *fs) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= p.N) return;
    const int i = perm[k];
    xs[k] = x4[i];
    fs[k] = make_float4(F[3 * i], F[3 * i + 1], F[3 * i + 2], 0.0f);
}

__global__ void cell_bounds_kernel(Params p, const int *__restrict__ keys, int *start, int *end) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= p.N) return;
    const int h = keys[k];
    if (k == 0 || keys[k - 1] != h) start[h] = k;
    if (k == p.N - 1 || keys[k + 1] != h) end[h] = k + 1;
}

// Per-warp tables of the particle's 1-D kernels (ngd <= 32).
struct WarpTables {
    float g[3][32];   // Gaussian factors along x, y, z
    float d2[3][32];  // squared distance of the grid point to the particle along x, y, z
    int ind[3][32];   // periodic grid offsets: i, j*nx, k*nx*ny
};

// Walks the ngd^3 points of a particle's support, lane L taking the flattened
// points L, L+32, ...: (ii, jj, kk) advance by the fixed strides of 32 with one
// carry each instead of being divided out of the flat index.
struct SupportWalk {
    int ii, jj, kk, di, dj, dk, ngd;
    __device__ __forceinline__ SupportWalk(int lane, int n) : ngd(n) {
        const int n2 = n * n;
        kk = lane / n2;
        jj = (lane - kk * n2) / n;
        ii = lane - kk * n2 - jj * n;
        dk = 32 / n2;
        dj = (32 - dk * n2) / n;
        di = 32 - dk * n2 - dj * n;
    }
    __device__ __forceinline__ void next() {
        ii += di;
        jj += dj;
        kk += dk;
        if (ii >= ngd) { ii -= ngd; ++jj; }
        if (jj >= ngd) { jj -= ngd; ++kk; }
    }
};

__device__ __forceinline__ void build_tables(const Params &p, float4 y, WarpTables &t, int lane) {
    if (lane < p.ngd) {
        const int ngdh = p.ngd / 2;
        const float anorm = rsqrtf(2.0f * 3.14159265358979f * p.Sigma * p.Sigma);
        const float inv2s2 = 1.0f / (2.0f * p.Sigma * p.Sigma);
        const float pos[3] = {y.x, y.y, y.z};
        const int n[3] = {p.nx, p.ny, p.nz};
        for (int c = 0; c < 3; ++c) {
            const float xg = rintf(pos[c] / p.dx) - ngdh + lane;
            const float xx = xg * p.dx - pos[c];
            t.g[c][lane] = anorm * expf(-xx * xx * inv2s2);
            t.d2[c][lane] = xx * xx;
            const int stride = c == 0 ? 1 : (c == 1 ? p.nx : p.nx * p.ny);
            t.ind[c][lane] = static_cast<int>(xg - n[c] * floorf(xg / n[c])) * stride;
        }
    }
    __syncwarp();
}

// Spreading: F * (modified Gaussian) onto the three grids, one warp per particle
// (sorted order, so neighbouring warps touch neighbouring grid lines).
__global__ void __launch_bounds__(128) spread_kernel(Params p, const float4 *__restrict__ xs,
                                                     const float4 *__restrict__ fs, float *grid) {
    __shared__ WarpTables tabs[4];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int k = blockIdx.x * 4 + w;
    if (k >= p.N) return;
    WarpTables &t = tabs[w];
    build_tables(p, xs[k], t, lane);
    const float4 f = fs[k];
    const float S2 = p.Sigma * p.Sigma;
    const float c_r2 = 0.5f * p.pdmag / (S2 * S2);
    const float c_0 = 1.0f - 1.5f * p.pdmag / S2;
    const int ngd = p.ngd, ngd2 = ngd * ngd;
    float *gx = grid, *gy = grid + p.grid_size, *gz = grid + 2 * p.grid_size;
    SupportWalk sw(lane, ngd);
    for (int tt = lane; tt < ngd2 * ngd; tt += 32, sw.next()) {
        const int ii = sw.ii, jj = sw.jj, kk = sw.kk;
        const float r2 = t.d2[0][ii] + t.d2[1][jj] + t.d2[2][kk];
        const float wgt = t.g[0][ii] * t.g[1][jj] * t.g[2][kk] * (c_0 + c_r2 * r2);
        const int ind = t.ind[0][ii] + t.ind[1][jj] + t.ind[2][kk];
        atomicAdd(gx + ind, f.x * wgt);
        atomicAdd(gy + ind, f.y * wgt);
        atomicAdd(gz + ind, f.z * wgt);
    }
}

// Spectral Stokes solve, in place: u = (f - q (q.f)/q^2) / (q^2 n), q = 0 removed
// (cufcm_flow_solve, CUFCM_FCM.cu:187-246).
__global__ void stokes_kernel(Params p, cufftComplex *spec) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i >= p.fft_size) return;
    const int fnx = p.nx / 2 + 1;
    const int ik = static_cast<int>(i / (static_cast<size_t>(p.ny) * fnx));
    const int ij = static_cast<int>((i - static_cast<size_t>(ik) * p.ny * fnx) / fnx);
    const int ii = static_cast<int>(i - (static_cast<size_t>(ij) + static_cast<size_t>(ik) * p.ny) * fnx);
    const float two_pi = 6.28318530717959f;
    const float q1 = ((ii <= p.nx / 2) ? ii : ii - p.nx) * (two_pi / p.Lx);
    const float q2 = ((ij <= p.ny / 2) ? ij : ij - p.ny) * (two_pi / p.Ly);
    const float q3 = ((ik <= p.nz / 2) ? ik : ik - p.nz) * (two_pi / p.Lz);
    cufftComplex *fx = spec, *fy = spec + p.fft_size, *fz = spec + 2 * p.fft_size;
    if (i == 0) {
        fx[0] = fy[0] = fz[0] = make_cuComplex(0.0f, 0.0f);
        return;
    }
    const float qq = q1 * q1 + q2 * q2 + q3 * q3;
    const float qq_inv = 1.0f / qq;
    const float norm = qq_inv / static_cast<float>(p.grid_size);
    const cufftComplex a = fx[i], b = fy[i], c = fz[i];
    const float kf_re = (q1 * a.x + q2 * b.x + q3 * c.x) * qq_inv;
    const float kf_im = (q1 * a.y + q2 * b.y + q3 * c.y) * qq_inv;
    fx[i] = make_cuComplex(norm * (a.x - q1 * kf_re), norm * (a.y - q1 * kf_im));
    fy[i] = make_cuComplex(norm * (b.x - q2 * kf_re), norm * (b.y - q2 * kf_im));
    fz[i] = make_cuComplex(norm * (c.x - q3 * kf_re), norm * (c.y - q3 * kf_im));
}

// Gathering: V = dx^3 sum u(grid) * (modified Gaussian), one warp per particle.
__global__ void __launch_bounds__(128) gather_kernel(Params p, const float4 *__restrict__ xs,
                                                     const float *__restrict__ grid, float4 *vgs) {
    __shared__ WarpTables tabs[4];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int k = blockIdx.x * 4 + w;
    if (k >= p.N) return;
    WarpTables &t = tabs[w];
    build_tables(p, xs[k], t, lane);
    const float S2 = p.Sigma * p.Sigma;
    const float c_r2 = 0.5f * p.pdmag / (S2 * S2);
    const float c_0 = 1.0f - 1.5f * p.pdmag / S2;
    const float vol = p.dx * p.dx * p.dx;
    const int ngd = p.ngd, ngd2 = ngd * ngd;
    const float *gx = grid, *gy = grid + p.grid_size, *gz = grid + 2 * p.grid_size;
    float vx = 0.0f, vy = 0.0f, vz = 0.0f;
    SupportWalk sw(lane, ngd);
    for (int tt = lane; tt < ngd2 * ngd; tt += 32, sw.next()) {
        const int ii = sw.ii, jj = sw.jj, kk = sw.kk;
        const float r2 = t.d2[0][ii] + t.d2[1][jj] + t.d2[2][kk];
        const float wgt = t.g[0][ii] * t.g[1][jj] * t.g[2][kk] * (c_0 + c_r2 * r2) * vol;
        const int ind = t.ind[0][ii] + t.ind[1][jj] + t.ind[2][kk];
        vx += __ldg(gx + ind) * wgt;
        vy += __ldg(gy + ind) * wgt;
        vz += __ldg(gz + ind) * wgt;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        vx += __shfl_down_sync(0xffffffffu, vx, o);
        vy += __shfl_down_sync(0xffffffffu, vy, o);
        vz += __shfl_down_sync(0xffffffffu, vz, o);
    }
    if (lane == 0) vgs[k] = make_float4(vx, vy, vz, 0.0f);
}

// Gaussian-blob pair functions (CUFCM_CORRECTION.cu:43-100): S = S_I I + S_xx x x^T etc.
struct PairFns {
    float SI, Sxx;
};

__device__ __forceinline__ void blob_pair(float r, float rsq, float sg, float sgsq, float gauss, float erfS,
                                          float &SI, float &Sxx) {
    const float inv8pi = 0.0397887357729738f;
    SI = inv8pi / r * ((1.0f + sgsq / rsq) * erfS) - 0.5f * sgsq * sgsq / rsq * gauss;
    Sxx = inv8pi / (r * rsq) * ((1.0f - 3.0f * sgsq / rsq) * erfS) + 1.5f * sgsq * sgsq / (rsq * rsq) * gauss;
}

// Near-field correction + self correction, then the scatter to input order.
// One thread per sorted particle, all 27 neighbour cells, pairs within Rc.
__global__ void __launch_bounds__(128) correction_kernel(Params p, const float4 *__restrict__ xs,
                                                         const float4 *__restrict__ fs, const int *__restrict__ keys,
                                                         const int *__restrict__ cstart, const int *__restrict__ cend,
                                                         const float4 *__restrict__ vgs, const int *__restrict__ perm,
                                                         float *vout) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= p.N) return;
    const float4 xi = xs[k];
    const int h = keys[k];
    const int cx = h % p.Mx, cy = (h / p.Mx) % p.My, cz = h / (p.Mx * p.My);
    const float pi = 3.14159265358979f;
    const float gam = 1.41421356237310f * p.Sigma, gamsq = gam * gam;
    const float gvf = 1.41421356237310f * p.sigma, gvfsq = gvf * gvf;
    const float gnorm = 1.0f / powf(2.0f * pi * gamsq, 1.5f);
    const float gnorm_vf = 1.0f / powf(2.0f * pi * gvfsq, 1.5f);
    const float pd = p.pdmag, pdq = 0.25f * pd * pd;
    float vx = 0.0f, vy = 0.0f, vz = 0.0f;
    for (int dz = -1; dz <= 1; ++dz) {
        const int zc = (cz + dz + p.Mz) % p.Mz;
        for (int dy = -1; dy <= 1; ++dy) {
            const int yc = (cy + dy + p.My) % p.My;
            for (int dxc = -1; dxc <= 1; ++dxc) {
                const int xc = (cx + dxc + p.Mx) % p.Mx;
                const int c = xc + (yc + zc * p.My) * p.Mx;
                const int j1 = cend[c];
                for (int j = cstart[c]; j < j1; ++j) {
                    if (j == k) continue;
                    const float4 xj = xs[j];
                    float xij = xi.x - xj.x, yij = xi.y - xj.y, zij = xi.z - xj.z;
                    // minimum image as the reference writes it (CUFCM_CORRECTION.cu:149-151)
                    xij -= p.Lx * static_cast<float>(static_cast<int>(xij / (0.5f * p.Lx)));
                    yij -= p.Ly * static_cast<float>(static_cast<int>(yij / (0.5f * p.Ly)));
                    zij -= p.Lz * static_cast<float>(static_cast<int>(zij / (0.5f * p.Lz)));
                    const float rsq = xij * xij + yij * yij + zij * zij;
                    if (rsq >= p.Rcsq) continue;
                    const float r = sqrtf(rsq);
                    const float erfS = erff(0.5f * r / p.Sigma);
                    const float gg = expf(-0.5f * rsq / gamsq) * gnorm;
                    const float erfS_vf = erff(r / (1.41421356237310f * gvf));
                    const float gg_vf = expf(-0.5f * rsq / gvfsq) * gnorm_vf;
                    float A_vf, B_vf, A, B;
                    blob_pair(r, rsq, gvf, gvfsq, gg_vf, erfS_vf, A_vf, B_vf);
                    blob_pair(r, rsq, gam, gamsq, gg, erfS, A, B);
                    const float r3 = r * rsq;
                    const float QI = erfS / (4.0f * pi * r3) - (1.0f + gamsq / rsq) * gg;
                    const float Qxx = -3.0f * erfS / (4.0f * pi * r3 * rsq) + (1.0f + 3.0f * gamsq / rsq) / rsq * gg;
                    const float TI = (2.0f - rsq / gamsq) / gamsq * gg;
                    const float Txx = gg / (gamsq * gamsq);
                    const float t1 = A_vf - A - QI * pd - TI * pdq;
                    const float t2 = B_vf - B - Qxx * pd - Txx * pdq;
                    const float4 fj = fs[j];
                    const float xf = xij * fj.x + yij * fj.y + zij * fj.z;
                    vx += t1 * fj.x + t2 * xij * xf;
                    vy += t1 * fj.y + t2 * yij * xf;
                    vz += t1 * fj.z + t2 * zij * xf;
                }
            }
        }
    }
    const float4 fi = fs[k];
    const float4 vg = vgs[k];
    const int o = perm[k];
    vout[3 * o + 0] = vg.x + vx + fi.x * p.self_mob;
    vout[3 * o + 1] = vg.y + vy + fi.y * p.self_mob;
    vout[3 * o + 2] = vg.z + vz + fi.z * p.self_mob;
}

}  // namespace fcmk
}  // namespace cufil

using namespace cufil;

namespace {

fcmk::Params params_of(const cf_fcm *h) {
    fcmk::Params p;
    p.N = h->N;
    p.nx = h->nx;
    p.ny = h->ny;
    p.nz = h->nz;
    p.ngd = h->ngd;
    p.Mx = h->Mx;
    p.My = h->My;
    p.Mz = h->Mz;
    p.Lx = static_cast<float>(h->Lx);
    p.Ly = static_cast<float>(h->Ly);
    p.Lz = static_cast<float>(h->Lz);
    p.dx = static_cast<float>(h->dx);
    p.Sigma = static_cast<float>(h->Sigma);
    p.sigma = static_cast<float>(h->sigma);
    p.pdmag = static_cast<float>(h->pdmag);
    p.Rcsq = static_cast<float>(h->Rc * h->Rc);
    p.self_mob = static_cast<float>(h->self_mob);
    p.grid_size = h->grid_size;
    p.fft_size = h->fft_size;
    return p;
}

int cufft_status(cufftResult r, const char *what) {
    if (r == CUFFT_SUCCESS) return CF_OK;
    return set_error(r == CUFFT_ALLOC_FAILED ? CF_ENOMEM : CF_ECUDA, "%s failed: cuFFT error %d", what,
                     static_cast<int>(r));
}

template <typename T>
int falloc(T **p, size_t n) {
    *p = nullptr;
    CF_CUDA(cudaMalloc(reinterpret_cast<void **>(p), std::max<size_t>(n, 1) * sizeof(T)));
    return CF_OK;
}

// The pipeline on device buffers: Y, F in the caller's [3N] layout, V out [3N].
int fcm_run(cf_fcm *h, const float *dY, const float *dF, float *dV, cudaStream_t st) {
    const fcmk::Params p = params_of(h);
    const int N = h->N;
    const int tb = 128, nb = (N + tb - 1) / tb, wb = (N + 3) / 4;
    auto mark = [&](int i) -> int {
        if (h->timing) CF_CUDA(cudaEventRecord(h->ev[i], st));
        return CF_OK;
    };
    CF_TRY(mark(0));
    CF_CUDA(cudaMemsetAsync(h->grid, 0, sizeof(float) * 3 * h->grid_size, st));
    CF_TRY(mark(1));
    fcmk::prep_kernel<<<nb, tb, 0, st>>>(p, dY, h->x4, h->keys, h->vals);
    CF_CHECK_LAUNCH("fcm prep_kernel");
    size_t tmp = h->sort_tmp_bytes;
    CF_CUDA(cub::DeviceRadixSort::SortPairs(h->sort_tmp, tmp, h->keys, h->keys_sorted, h->vals, h->perm, N, 0,
                                            h->hash_bits, st));
    fcmk::permute_kernel<<<nb, tb, 0, st>>>(p, h->perm, h->x4, dF, h->xs, h->fs);
    CF_CHECK_LAUNCH("fcm permute_kernel");
    CF_CUDA(cudaMemsetAsync(h->cell_start, 0, sizeof(int) * h->ncell, st));
    CF_CUDA(cudaMemsetAsync(h->cell_end, 0, sizeof(int) * h->ncell, st));
    fcmk::cell_bounds_kernel<<<nb, tb, 0, st>>>(p, h->keys_sorted, h->cell_start, h->cell_end);
    CF_CHECK_LAUNCH("fcm cell_bounds_kernel");
    CF_TRY(mark(2));
    fcmk::spread_kernel<<<wb, 128, 0, st>>>(p, h->xs, h->fs, h->grid);
    CF_CHECK_LAUNCH("fcm spread_kernel");
    CF_TRY(mark(3));
    CF_TRY(cufft_status(cufftExecR2C(h->plan_fwd, h->grid, h->spec), "cufftExecR2C"));
    const size_t sb = (h->fft_size + 255) / 256;
    fcmk::stokes_kernel<<<static_cast<unsigned>(sb), 256, 0, st>>>(p, h->spec);
    CF_CHECK_LAUNCH("fcm stokes_kernel");
    CF_TRY(cufft_status(cufftExecC2R(h->plan_inv, h->spec, h->grid), "cufftExecC2R"));
    CF_TRY(mark(4));
    fcmk::gather_kernel<<<wb, 128, 0, st>>>(p, h->xs, h->grid, h->vgs);
    CF_CHECK_LAUNCH("fcm gather_kernel");
    CF_TRY(mark(5));
    fcmk::correction_kernel<<<nb, tb, 0, st>>>(p, h->xs, h->fs, h->keys_sorted, h->cell_start, h->cell_end, h->vgs,
                                               h->perm, dV);
    CF_CHECK_LAUNCH("fcm correction_kernel");
    CF_TRY(mark(6));
    return CF_OK;
}

}  // namespace

extern "C" int cf_fcm_create(const cf_fcm_config *cfg, cf_fcm **out) {
    clear_error();
    CF_REQUIRE(cfg && out, "cf_fcm_create: null argument");
    *out = nullptr;
    CF_REQUIRE(cfg->n >= 1, "cf_fcm_create: need n >= 1");
    CF_REQUIRE(cfg->nx >= 8 && cfg->ny >= 8 && cfg->nz >= 8 && cfg->nx % 2 == 0, "cf_fcm_create: bad grid %dx%dx%d",
               cfg->nx, cfg->ny, cfg->nz);
    CF_REQUIRE(cfg->rh > 0 && cfg->alpha > 0 && cfg->beta > 0 && cfg->eta > 0 && cfg->boxsize > 0,
               "cf_fcm_create: parameters must be positive");
    const int ngd = static_cast<int>(std::lround(cfg->alpha * cfg->beta));
    CF_REQUIRE(ngd >= 1 && ngd <= 32, "cf_fcm_create: kernel support round(alpha*beta) = %d must lie in [1, 32]", ngd);
    CF_REQUIRE(static_cast<double>(cfg->nx) * cfg->ny * cfg->nz < 2147483647.0,
               "cf_fcm_create: grid too large (at most 2^31 - 1 points: the kernels index it with 32-bit offsets)");
    CF_CUDA(cudaSetDevice(cfg->device));
    cf_fcm *h = new (std::nothrow) cf_fcm();
    if (!h) return set_error(CF_ENOMEM, "cf_fcm_create: host allocation failed");
    h->cfg = *cfg;
    // FCM_solver::init_config / init_fcm_var (CUFCM_SOLVER.cu:37-125), in FP64 on the host
    h->N = cfg->n;
    h->nx = cfg->nx;
    h->ny = cfg->ny;
    h->nz = cfg->nz;
    h->ngd = ngd;
    h->Lx = cfg->boxsize;
    h->Ly = cfg->boxsize / cfg->nx * cfg->ny;
    h->Lz = cfg->boxsize / cfg->nx * cfg->nz;
    h->dx = h->Lx / cfg->nx;
    const double pi = 3.14159265358979323846;
    h->sigma = cfg->rh / std::sqrt(pi);
    h->Sigma = h->dx * cfg->alpha;
    h->pdmag = h->sigma * h->sigma - h->Sigma * h->Sigma;
    h->Rc = cfg->eta * cfg->alpha * h->dx;
    h->Mx = static_cast<int>(std::max(h->Lx / h->Rc, 3.0));
    h->My = static_cast<int>(std::max(h->Ly / h->Rc, 3.0));
    h->Mz = static_cast<int>(std::max(h->Lz / h->Rc, 3.0));
    h->ncell = h->Mx * h->My * h->Mz;
    while ((1LL << h->hash_bits) < h->ncell) ++h->hash_bits;
    const double stokes = 1.0 / (6.0 * pi * cfg->rh);
    const double mod_stokes = 1.0 / (6.0 * pi * h->Sigma * std::sqrt(pi));
    const double pd_stokes = h->pdmag / (12.0 * std::pow(std::sqrt(pi) * h->Sigma, 3.0));
    const double bilap = h->pdmag * h->pdmag / (32.0 * std::pow(pi, 1.5) * std::pow(h->Sigma, 5.0));
    h->self_mob = stokes - mod_stokes + pd_stokes - bilap;  // cufcm_self_correction (CUFCM_CORRECTION.cu:333-352)
    h->grid_size = static_cast<size_t>(h->nx) * h->ny * h->nz;
    h->fft_size = static_cast<size_t>(h->nx / 2 + 1) * h->ny * h->nz;
    int rc = CF_OK;
    do {
        if ((rc = cuda_status(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate",
                              __FILE__, __LINE__)))
            break;
        const size_t N = h->N;
        if ((rc = falloc(&h->grid, 3 * h->grid_size)) || (rc = falloc(&h->spec, 3 * h->fft_size)) ||
            (rc = falloc(&h->x4, N)) || (rc = falloc(&h->xs, N)) || (rc = falloc(&h->fs, N)) ||
            (rc = falloc(&h->ys, 3 * N)) || (rc = falloc(&h->fsrc, 3 * N)) || (rc = falloc(&h->vout, 3 * N)) ||
            (rc = falloc(&h->vgs, N)) || (rc = falloc(&h->keys, N)) || (rc = falloc(&h->keys_sorted, N)) ||
            (rc = falloc(&h->vals, N)) || (rc = falloc(&h->perm, N)) || (rc = falloc(&h->cell_start, h->ncell)) ||
            (rc = falloc(&h->cell_end, h->ncell)))
            break;
        size_t tmp = 0;
        if ((rc = cuda_status(cub::DeviceRadixSort::SortPairs(nullptr, tmp, h->keys, h->keys_sorted, h->vals, h->perm,
                                                              h->N, 0, h->hash_bits, h->stream),
                              "cub sort sizing", __FILE__, __LINE__)))
            break;
        h->sort_tmp_bytes = tmp;
        if ((rc = cuda_status(cudaMalloc(&h->sort_tmp, std::max<size_t>(tmp, 1)), "cudaMalloc", __FILE__, __LINE__)))
            break;
        // batched 3-D transforms of the three components, x fastest (cufftPlan3d(nz, ny, nx) in the reference)
        int n3[3] = {h->nz, h->ny, h->nx};
        if ((rc = cufft_status(cufftPlanMany(&h->plan_fwd, 3, n3, nullptr, 1, static_cast<int>(h->grid_size), nullptr,
                                             1, static_cast<int>(h->fft_size), CUFFT_R2C, 3),
                               "cufftPlanMany(R2C)")))
            break;
        h->have_fwd = true;
        if ((rc = cufft_status(cufftPlanMany(&h->plan_inv, 3, n3, nullptr, 1, static_cast<int>(h->fft_size), nullptr,
                                             1, static_cast<int>(h->grid_size), CUFFT_C2R, 3),
                               "cufftPlanMany(C2R)")))
            break;
        h->have_inv = true;
        if ((rc = cufft_status(cufftSetStream(h->plan_fwd, h->stream), "cufftSetStream")) ||
            (rc = cufft_status(cufftSetStream(h->plan_inv, h->stream), "cufftSetStream")))
            break;
    } while (0);
    if (rc != CF_OK) {
        std::string msg = cf_last_error();
        cf_fcm_destroy(h);
        set_error(rc, "%s", msg.c_str());
        return rc;
    }
    *out = h;
    return CF_OK;
}

extern "C" int cf_fcm_destroy(cf_fcm *h) {
    if (!h) return CF_OK;
    cudaSetDevice(h->cfg.device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (cudaEvent_t e : h->ev)
        if (e) cudaEventDestroy(e);
    if (h->have_fwd) cufftDestroy(h->plan_fwd);
    if (h->have_inv) cufftDestroy(h->plan_inv);
    for (void *p : {(void *)h->grid, (void *)h->spec, (void *)h->x4, (void *)h->xs, (void *)h->fs, (void *)h->ys,
                    (void *)h->fsrc, (void *)h->vout, (void *)h->vgs, (void *)h->keys, (void *)h->keys_sorted,
                    (void *)h->vals, (void *)h->perm, (void *)h->cell_start, (void *)h->cell_end, h->sort_tmp})
        if (p) cudaFree(p);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return CF_OK;
}

extern "C" int cf_fcm_apply_device(cf_fcm *h, const float *d_Y, const float *d_F, float *d_V, void *stream) {
    clear_error();
    CF_REQUIRE(h && d_Y && d_F && d_V, "cf_fcm_apply_device: null argument");
    CF_CUDA(cudaSetDevice(h->cfg.device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // cuFFT runs on the handle's stream: order it after the caller's stream and back.
    cudaEvent_t ev;
    CF_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    int rc = CF_OK;
    do {
        if ((rc = cuda_status(cudaEventRecord(ev, st), "cudaEventRecord", __FILE__, __LINE__))) break;
        if ((rc = cuda_status(cudaStreamWaitEvent(h->stream, ev, 0), "cudaStreamWaitEvent", __FILE__, __LINE__)))
            break;
        if ((rc = fcm_run(h, d_Y, d_F, d_V, h->stream))) break;
        if ((rc = cuda_status(cudaEventRecord(ev, h->stream), "cudaEventRecord", __FILE__, __LINE__))) break;
        rc = cuda_status(cudaStreamWaitEvent(st, ev, 0), "cudaStreamWaitEvent", __FILE__, __LINE__);
    } while (0);
    cudaEventDestroy(ev);
    return rc;
}

extern "C" int cf_fcm_apply(cf_fcm *h, const float *Y, const float *F, float *V) {
    clear_error();
    CF_REQUIRE(h && Y && F && V, "cf_fcm_apply: null argument");
    CF_CUDA(cudaSetDevice(h->cfg.device));
    const size_t b = sizeof(float) * 3 * h->N;
    CF_CUDA(cudaMemcpyAsync(h->ys, Y, b, cudaMemcpyHostToDevice, h->stream));
    CF_CUDA(cudaMemcpyAsync(h->fsrc, F, b, cudaMemcpyHostToDevice, h->stream));
    CF_TRY(fcm_run(h, h->ys, h->fsrc, h->vout, h->stream));
    CF_CUDA(cudaMemcpyAsync(V, h->vout, b, cudaMemcpyDeviceToHost, h->stream));
    CF_CUDA(cudaStreamSynchronize(h->stream));
    return CF_OK;
}

extern "C" int cf_fcm_apply_segments_blobs(cf_fcm *h, int n_seg, const float *x_segs, const float *x_blobs,
                                           const float *f_segs, const float *f_blobs, float *v_segs,
                                           float *v_blobs) {
    clear_error();
    CF_REQUIRE(h, "cf_fcm_apply_segments_blobs: null handle");
    const int n_blob = h->N - n_seg;
    CF_REQUIRE(n_seg >= 0 && n_blob >= 0, "cf_fcm_apply_segments_blobs: n_seg = %d out of [0, %d]", n_seg, h->N);
    CF_REQUIRE((!n_seg || (x_segs && f_segs && v_segs)) && (!n_blob || (x_blobs && f_blobs && v_blobs)),
               "cf_fcm_apply_segments_blobs: missing buffer");
    // fcm_mobility_solver::evaluate_full_mobility (fcm_mobility_solver.cu:463-502): segments then blobs,
    // forces taken from the 6-dof segment records, torques ignored (ROTATION 0).
    std::vector<float> Y(3 * static_cast<size_t>(h->N)), F(Y.size()), V(Y.size());
    for (int i = 0; i < n_seg; ++i)
        for (int c = 0; c < 3; ++c) {
            Y[3 * i + c] = x_segs[3 * i + c];
            F[3 * i + c] = f_segs[6 * i + c];
        }
    for (int i = 0; i < n_blob; ++i)
        for (int c = 0; c < 3; ++c) {
            Y[3 * (n_seg + i) + c] = x_blobs[3 * i + c];
            F[3 * (n_seg + i) + c] = f_blobs[3 * i + c];
        }
    CF_TRY(cf_fcm_apply(h, Y.data(), F.data(), V.data()));
    for (int i = 0; i < n_seg; ++i)
        for (int c = 0; c < 6; ++c) v_segs[6 * i + c] = c < 3 ? V[3 * i + c] : 0.0f;
    for (int i = 0; i < n_blob; ++i)
        for (int c = 0; c < 3; ++c) v_blobs[3 * i + c] = V[3 * (n_seg + i) + c];
    return CF_OK;
}

extern "C" int cf_fcm_info(cf_fcm *h, double *info) {
    clear_error();
    CF_REQUIRE(h && info, "cf_fcm_info: null argument");
    info[0] = h->ngd;
    info[1] = h->dx;
    info[2] = h->sigma;
    info[3] = h->Sigma;
    info[4] = h->Rc;
    info[5] = h->Mx;
    info[6] = h->My;
    info[7] = h->Mz;
    info[8] = h->self_mob;
    return CF_OK;
}

extern "C" int cf_fcm_set_timing(cf_fcm *h, int enable) {
    clear_error();
    CF_REQUIRE(h, "cf_fcm_set_timing: null handle");
    CF_CUDA(cudaSetDevice(h->cfg.device));
    if (enable && !h->ev[0])
        for (cudaEvent_t &e : h->ev) CF_CUDA(cudaEventCreate(&e));
    h->timing = enable != 0;
    return CF_OK;
}

extern "C" int cf_fcm_stage_times(cf_fcm *h, float *ms) {
    clear_error();
    CF_REQUIRE(h && ms, "cf_fcm_stage_times: null argument");
    CF_REQUIRE(h->timing, "cf_fcm_stage_times: timing is off (cf_fcm_set_timing)");
    CF_CUDA(cudaSetDevice(h->cfg.device));
    CF_CUDA(cudaEventSynchronize(h->ev[6]));
    for (int i = 0; i < 6; ++i) CF_CUDA(cudaEventElapsedTime(&ms[i], h->ev[i], h->ev[i + 1]));
    return CF_OK;
}

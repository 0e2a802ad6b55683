// rpy_kernels.cu -- pairwise RPY block products on the FP32 pipe.
//
// Replaces the reference kernels Mss_mult / Mbb_mult / Msb_mult / Mbs_mult
// (src/cilia/cuda_functions.cu:362-757).  Those use one thread per target,
// 64-thread blocks and AoS global loads; here a CTA of 128 threads owns
// 128*TI targets and one split of the sources, staged by a single bulk async
// copy per array into shared memory, so that the grid covers every SM even
// for a few thousand particles.  Partial sums are reduced in FP64 by a second
// small kernel in a fixed order.
#include "common.cuh"
#include "rpy_kernels.cuh"
#include "rpy_pairs.cuh"
#include "tma.cuh"

#include <algorithm>

namespace cufil {

namespace {

constexpr int kThreads = 128;
constexpr int kMaxSplit = 2048;   // sources staged per CTA (<= 96 KB with torques)
constexpr int kMinSplit = 64;     // keep each split long enough to amortise staging
constexpr int kBlockSum = 64;     // sources per FP32 block sum before TwoSum

struct TileParams {
    const float4 *xt;
    const float4 *xs;
    const float4 *fs;
    const float4 *ts;
    float4 *partial;
    int nt, ns, split, ntp;
    float at, as, inv_mu;
    int *err;
};

template <int VD>
__device__ __forceinline__ void two_sum_add(float *hi, float *lo, const float *a) {
#pragma unroll
    for (int c = 0; c < VD; ++c) {
        const float t = hi[c] + a[c];
        const float bp = t - hi[c];
        lo[c] += (hi[c] - (t - bp)) + (a[c] - bp);
        hi[c] = t;
    }
}

template <bool WALL, int VD, int FD, int TI, bool MASK>
__device__ __forceinline__ void tile_sum(const float4 *__restrict__ xs_s, const float4 *__restrict__ fs_s,
                                         const float4 *__restrict__ ts_s, int nsrc, int j0, const int *gi,
                                         const float (*xi)[3], float at, float as, float inv_mu,
                                         float (*hi)[VD], float (*lo)[VD]) {
    for (int jb = 0; jb < nsrc; jb += kBlockSum) {
        const int je = min(nsrc, jb + kBlockSum);
        float acc[TI][VD];
#pragma unroll
        for (int k = 0; k < TI; ++k)
#pragma unroll
            for (int c = 0; c < VD; ++c) acc[k][c] = 0.0f;
#pragma unroll 2
        for (int j = jb; j < je; ++j) {
            const float4 p = xs_s[j];
            const float4 f4 = fs_s[j];
            float f[6] = {f4.x, f4.y, f4.z, 0.f, 0.f, 0.f};
            if constexpr (FD > 3) {
                const float4 t4 = ts_s[j];
                f[3] = t4.x;
                f[4] = t4.y;
                f[5] = t4.z;
            }
#pragma unroll
            for (int k = 0; k < TI; ++k) {
                if constexpr (MASK) {
                    if (gi[k] == j0 + j) continue;  // the self block is added by the reduction
                }
                const float dx = xi[k][0] - p.x, dy = xi[k][1] - p.y, dz = xi[k][2] - p.z;
                if constexpr (WALL)
                    wall_pair_f32<VD, FD>(dx, dy, dz, xi[k][2], p.z, f, acc[k]);
                else
                    free_pair_f32<VD, FD>(dx, dy, dz, at, as, inv_mu, f, acc[k]);
            }
        }
#pragma unroll
        for (int k = 0; k < TI; ++k) two_sum_add<VD>(hi[k], lo[k], acc[k]);
    }
}

// grid: (tiles, nsplit); block: 128.  SELF: targets and sources are the same
// particle set (wall mode skips j == i here; the reduction adds the self block).
template <bool WALL, int VD, int FD, int TI, bool SELF>
__global__ void __launch_bounds__(kThreads) rpy_tile_kernel(TileParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw);
    float4 *xs_s = reinterpret_cast<float4 *>(smem_raw + 16);
    float4 *fs_s = xs_s + p.split;
    float4 *ts_s = fs_s + p.split;

    const int j0 = blockIdx.y * p.split;
    const int nsrc = max(0, min(p.ns, j0 + p.split) - j0);
    const int t0 = blockIdx.x * (kThreads * TI);

    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0 && nsrc > 0) {
        const uint32_t bytes = static_cast<uint32_t>(nsrc) * sizeof(float4);
        mbar_arrive_expect_tx(bar, bytes * (FD > 3 ? 3u : 2u));
        bulk_g2s(xs_s, p.xs + j0, bytes, bar);
        bulk_g2s(fs_s, p.fs + j0, bytes, bar);
        if constexpr (FD > 3) bulk_g2s(ts_s, p.ts + j0, bytes, bar);
    }

    // Targets of this thread (tail threads duplicate the last target and do not store).
    int gi[TI];
    float xi[TI][3];
#pragma unroll
    for (int k = 0; k < TI; ++k) {
        const int i = t0 + k * kThreads + threadIdx.x;
        gi[k] = i;
        const float4 q = p.xt[min(i, p.nt - 1)];
        xi[k][0] = q.x;
        xi[k][1] = q.y;
        xi[k][2] = q.z;
    }
    float hi[TI][VD], lo[TI][VD];
#pragma unroll
    for (int k = 0; k < TI; ++k)
#pragma unroll
        for (int c = 0; c < VD; ++c) hi[k][c] = lo[k][c] = 0.0f;

    if (nsrc > 0) {
        if (!mbar_wait_bounded(bar, 0)) {
            if (threadIdx.x == 0) {
                atomicOr(p.err, kErrTmaTimeout);
                mbar_wait_bounded(bar, 0);  // give the copies in flight a second bounded chance
            }
            return;
        }
        bool diag = false;
        if constexpr (WALL && SELF) diag = (j0 < t0 + kThreads * TI) && (t0 < j0 + nsrc);
        if (diag)
            tile_sum<WALL, VD, FD, TI, true>(xs_s, fs_s, ts_s, nsrc, j0, gi, xi, p.at, p.as, p.inv_mu, hi, lo);
        else
            tile_sum<WALL, VD, FD, TI, false>(xs_s, fs_s, ts_s, nsrc, j0, gi, xi, p.at, p.as, p.inv_mu, hi, lo);
    }

    constexpr int W = VD / 3;
#pragma unroll
    for (int k = 0; k < TI; ++k) {
        const int i = gi[k];
        if (i >= p.nt) continue;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            float4 o;
            o.x = hi[k][3 * w + 0] + lo[k][3 * w + 0];
            o.y = hi[k][3 * w + 1] + lo[k][3 * w + 1];
            o.z = hi[k][3 * w + 2] + lo[k][3 * w + 2];
            o.w = 0.0f;
            p.partial[(static_cast<size_t>(blockIdx.y) * W + w) * p.ntp + i] = o;
        }
    }
}

struct ReduceParams {
    const float4 *partial;
    const float4 *xt, *ft, *tt;  // self block inputs (wall, self set)
    float *out;
    int nsplit, nt, ntp, stride, mode;
};

template <bool WALL_SELF, int VD, int FD>
__global__ void rpy_reduce_kernel(ReduceParams p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.nt) return;
    constexpr int W = VD / 3;
    double v[VD];
#pragma unroll
    for (int c = 0; c < VD; ++c) v[c] = 0.0;
    for (int s = 0; s < p.nsplit; ++s) {
#pragma unroll
        for (int w = 0; w < W; ++w) {
            const float4 q = p.partial[(static_cast<size_t>(s) * W + w) * p.ntp + i];
            v[3 * w + 0] += q.x;
            v[3 * w + 1] += q.y;
            v[3 * w + 2] += q.z;
        }
    }
    if constexpr (WALL_SELF) {
        const float4 f4 = p.ft[i];
        float f[6] = {f4.x, f4.y, f4.z, 0.f, 0.f, 0.f};
        if constexpr (FD > 3) {
            const float4 t4 = p.tt[i];
            f[3] = t4.x;
            f[4] = t4.y;
            f[5] = t4.z;
        }
        float vs[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        wall_self_f32<VD, FD>(p.xt[i].z, f, vs);
#pragma unroll
        for (int c = 0; c < VD; ++c) v[c] += vs[c];
    }
    float *o = p.out + static_cast<size_t>(i) * p.stride;
    if (p.mode == kOutAdd) {
#pragma unroll
        for (int c = 0; c < VD; ++c) o[c] = static_cast<float>(static_cast<double>(o[c]) + v[c]);
    } else {
#pragma unroll
        for (int c = 0; c < VD; ++c) o[c] = static_cast<float>(v[c]);
        for (int c = VD; c < p.stride; ++c) o[c] = 0.0f;
    }
}

__global__ void pack_xyz_kernel(const float *__restrict__ a, float4 *__restrict__ o, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) o[i] = make_float4(a[3 * i], a[3 * i + 1], a[3 * i + 2], 0.0f);
}

__global__ void pack_ft6_kernel(const float *__restrict__ a, float4 *__restrict__ f, float4 *__restrict__ t,
                                int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        f[i] = make_float4(a[6 * i], a[6 * i + 1], a[6 * i + 2], 0.0f);
        if (t) t[i] = make_float4(a[6 * i + 3], a[6 * i + 4], a[6 * i + 5], 0.0f);
    }
}

// Raises the dynamic shared-memory cap of one instantiation once per device.
// Called before any launch (and therefore before any stream capture).
template <bool WALL, int VD, int FD, int TI, bool SELF>
int configure_tiles_t() {
    auto kern = rpy_tile_kernel<WALL, VD, FD, TI, SELF>;
    static bool configured[64] = {};
    int dev = 0;
    CF_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64 || !configured[dev]) {
        CF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 16 + 3 * kMaxSplit * 16));
        if (dev >= 0 && dev < 64) configured[dev] = true;
    }
    return CF_OK;
}

template <bool WALL, int VD, int FD, int TI, bool SELF>
int launch_tiles_t(const RpyBlockDesc &d, const RpyPlan &plan, float4 *scratch, int *dev_err,
                   cudaStream_t st) {
    auto kern = rpy_tile_kernel<WALL, VD, FD, TI, SELF>;
    CF_TRY((configure_tiles_t<WALL, VD, FD, TI, SELF>()));
    TileParams p;
    p.xt = d.xt;
    p.xs = d.xs;
    p.fs = d.fs;
    p.ts = d.ts;
    p.partial = scratch;
    p.nt = d.nt;
    p.ns = d.ns;
    p.split = plan.split;
    p.ntp = d.nt;
    p.at = d.at;
    p.as = d.as;
    p.inv_mu = 1.0f / d.mu;
    p.err = dev_err;
    dim3 grid(plan.tiles, plan.nsplit);
    kern<<<grid, kThreads, plan.smem, st>>>(p);
    CF_CHECK_LAUNCH("rpy_tile_kernel");
    return CF_OK;
}

template <bool WALL, int VD, int FD, bool SELF>
int dispatch_ti(const RpyBlockDesc &d, const RpyPlan &plan, float4 *scratch, int *dev_err, cudaStream_t st) {
    if (plan.ti == 2) return launch_tiles_t<WALL, VD, FD, 2, SELF>(d, plan, scratch, dev_err, st);
    return launch_tiles_t<WALL, VD, FD, 1, SELF>(d, plan, scratch, dev_err, st);
}

template <bool WALL, bool SELF>
int dispatch_dof(const RpyBlockDesc &d, const RpyPlan &plan, float4 *scratch, int *dev_err, cudaStream_t st) {
    if (d.vd == 3 && d.fd == 3) return dispatch_ti<WALL, 3, 3, SELF>(d, plan, scratch, dev_err, st);
    if (d.vd == 6 && d.fd == 6) return dispatch_ti<WALL, 6, 6, SELF>(d, plan, scratch, dev_err, st);
    if (d.vd == 6 && d.fd == 3) return dispatch_ti<WALL, 6, 3, SELF>(d, plan, scratch, dev_err, st);
    if (d.vd == 3 && d.fd == 6) return dispatch_ti<WALL, 3, 6, SELF>(d, plan, scratch, dev_err, st);
    return set_error(CF_EINVAL, "rpy: unsupported dof pair %d/%d", d.vd, d.fd);
}

template <bool WS, int VD, int FD>
int launch_reduce_t(const ReduceParams &p, cudaStream_t st) {
    const int threads = 128;
    const int blocks = (p.nt + threads - 1) / threads;
    rpy_reduce_kernel<WS, VD, FD><<<blocks, threads, 0, st>>>(p);
    CF_CHECK_LAUNCH("rpy_reduce_kernel");
    return CF_OK;
}

}  // namespace

RpyPlan rpy_plan(int nt, int ns, int vd, int fd, int num_sms) {
    RpyPlan pl;
    pl.ti = (vd == 3) ? 2 : 1;
    const int per_cta = kThreads * pl.ti;
    pl.tiles = std::max(1, (nt + per_cta - 1) / per_cta);
    // Aim for ~8 resident CTAs per SM in one wave.
    const int want_ctas = std::max(1, num_sms) * 8;
    int nsplit = std::max(1, (want_ctas + pl.tiles - 1) / pl.tiles);
    nsplit = std::min(nsplit, std::max(1, ns / kMinSplit));
    nsplit = std::max(nsplit, (ns + kMaxSplit - 1) / kMaxSplit);
    nsplit = std::max(nsplit, 1);
    int split = (ns + nsplit - 1) / nsplit;
    split = std::max(split, 1);
    nsplit = std::max(1, (ns + split - 1) / split);
    pl.nsplit = nsplit;
    pl.split = split;
    pl.smem = 16 + static_cast<size_t>(split) * sizeof(float4) * (fd > 3 ? 3 : 2);
    pl.scratch_float4 = static_cast<size_t>(nsplit) * (vd / 3) * std::max(nt, 1);
    return pl;
}

size_t rpy_scratch_float4(int nt_max, int ns_max, int vd, int num_sms) {
    // The partial count is nsplit*nt; nsplit*tiles is bounded by the CTA target
    // or by the split caps, so take the maximum over both regimes.
    size_t best = 0;
    for (int fd : {3, 6}) {
        RpyPlan pl = rpy_plan(nt_max, ns_max, vd, fd, num_sms);
        best = std::max(best, pl.scratch_float4);
    }
    return best;
}

int rpy_launch_tiles(const RpyBlockDesc &d, const RpyPlan &plan, float4 *scratch, int *dev_err,
                     cudaStream_t st) {
    if (d.nt <= 0) return CF_OK;
    const bool self = d.self_set != 0;
    if (d.wall) return self ? dispatch_dof<true, true>(d, plan, scratch, dev_err, st)
                            : dispatch_dof<true, false>(d, plan, scratch, dev_err, st);
    // Unbounded blocks need no mask: r = 0 is handled by the containment branch.
    return dispatch_dof<false, false>(d, plan, scratch, dev_err, st);
}

int rpy_prepare(const RpyBlockDesc &d, const RpyPlan &plan) {
    const bool self = d.self_set != 0;
    if (d.wall && self) {
        if (d.vd == 3 && d.fd == 3) return plan.ti == 2 ? configure_tiles_t<true, 3, 3, 2, true>() : configure_tiles_t<true, 3, 3, 1, true>();
        if (d.vd == 6 && d.fd == 6) return plan.ti == 2 ? configure_tiles_t<true, 6, 6, 2, true>() : configure_tiles_t<true, 6, 6, 1, true>();
    }
    return CF_OK;  // other instantiations configure themselves on first launch
}

int rpy_launch_reduce_f32(const RpyBlockDesc &d, const RpyPlan &plan, const float4 *scratch, float *out_f,
                          int stride, int mode, cudaStream_t st) {
    if (d.nt <= 0) return CF_OK;
    ReduceParams p;
    p.partial = scratch;
    p.xt = d.xt;
    p.ft = d.fs;
    p.tt = d.ts;
    p.out = out_f;
    p.nsplit = d.ns > 0 ? plan.nsplit : 0;
    p.nt = d.nt;
    p.ntp = d.nt;
    p.stride = stride;
    p.mode = mode;
    const bool ws = d.wall && d.self_set;
    if (d.vd == 3 && d.fd == 3) return ws ? launch_reduce_t<true, 3, 3>(p, st) : launch_reduce_t<false, 3, 3>(p, st);
    if (d.vd == 6 && d.fd == 6) return ws ? launch_reduce_t<true, 6, 6>(p, st) : launch_reduce_t<false, 6, 6>(p, st);
    if (d.vd == 6 && d.fd == 3) return ws ? launch_reduce_t<true, 6, 3>(p, st) : launch_reduce_t<false, 6, 3>(p, st);
    if (d.vd == 3 && d.fd == 6) return ws ? launch_reduce_t<true, 3, 6>(p, st) : launch_reduce_t<false, 3, 6>(p, st);
    return set_error(CF_EINVAL, "rpy: unsupported dof pair %d/%d", d.vd, d.fd);
}

int pack_xyz_to_float4(const float *aos3, float4 *out, int n, cudaStream_t st) {
    if (n <= 0) return CF_OK;
    pack_xyz_kernel<<<(n + 255) / 256, 256, 0, st>>>(aos3, out, n);
    CF_CHECK_LAUNCH("pack_xyz_kernel");
    return CF_OK;
}

int pack_ft6_to_float4(const float *aos6, float4 *force, float4 *torque, int n, cudaStream_t st) {
    if (n <= 0) return CF_OK;
    pack_ft6_kernel<<<(n + 255) / 256, 256, 0, st>>>(aos6, force, torque, n);
    CF_CHECK_LAUNCH("pack_ft6_kernel");
    return CF_OK;
}

int rpy_block_product(const RpyBlockDesc &d, float4 *scratch, size_t scratch_cap, int *dev_err, float *out_f,
                      int stride, int mode, int num_sms, cudaStream_t st) {
    if (d.nt <= 0) return CF_OK;
    RpyPlan plan = rpy_plan(d.nt, d.ns, d.vd, d.fd, num_sms);
    if (plan.scratch_float4 > scratch_cap)
        return set_error(CF_EINVAL, "rpy: scratch too small (%zu < %zu float4)", scratch_cap, plan.scratch_float4);
    if (d.ns > 0) CF_TRY(rpy_launch_tiles(d, plan, scratch, dev_err, st));
    return rpy_launch_reduce_f32(d, plan, scratch, out_f, stride, mode, st);
}

}  // namespace cufil

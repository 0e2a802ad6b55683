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
#include <atomic>

namespace cufil {

namespace {

constexpr int kThreads = 128;
constexpr int kMaxSplit = 2048;   // sources staged per CTA (<= 96 KB with torques)
constexpr int kMinSplit = 64;     // keep each split long enough to amortise staging
constexpr int kBlockSum = 64;     // sources per FP32 block sum before TwoSum
constexpr int kCtasPerSm = 8;     // launch bound: 8 x 128 threads x 64 registers = one SM's file
constexpr int kStageCost = 24;    // per-CTA staging/epilogue cost in units of one source

struct TileParams {
    const float4 *xt;
    const float4 *xs;
    const float4 *fs;
    const float4 *ts;
    float4 *partial;
    int nt, ns, split, ntp;
    float at, as, inv_mu;
    int *err;
    unsigned wait_limit;  // tries of the first wait for the staged sources
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
__global__ void __launch_bounds__(kThreads, kCtasPerSm) rpy_tile_kernel(TileParams p) {
    chain_wait();  // launched as a programmatic dependent of the packing launch
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
        if (!mbar_wait_bounded(bar, 0, p.wait_limit)) {
            // Gave up: flag it, skip the sum and the stores, and let every
            // thread drain the copies already issued (one more bounded wait
            // with the full limit) before it exits, so that no copy lands in
            // shared memory that another block has been given.  A copy still
            // in flight after that second limit is not handled.
            if (threadIdx.x == 0) atomicOr(p.err, kErrTmaTimeout);
            mbar_wait_bounded(bar, 0);
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
            p.partial[(static_cast<size_t>(i) * gridDim.y + blockIdx.y) * W + w] = o;
        }
    }
}

// ---------------------------------------------------------------------------
// Symmetric wall kernel for the segment-segment block (targets == sources, 3x3).
// The grand mobility is symmetric, so each unordered pair is evaluated once and
// applied in both directions (wall_pair_sym_f32).  Work unit: one warp and one
// pair of 32-particle tiles (I <= J) of the upper triangle.  The warp's lanes
// own the 32 targets of tile I; the 32 sources of tile J, with the accumulators
// of their own velocities, rotate around the warp by one lane per step, so after
// 32 steps every lane has met every source and every source accumulator is back
// in its home lane.  Diagonal tiles are evaluated one-sided (j != i).  Each
// target receives exactly one partial per tile, written to
// partial[i * nb + tile] -- no atomics, deterministic.
struct SymParams {
    const float4 *x;
    const float4 *f;
    float4 *partial;
    int n, nb;
    long long items;
    float a, inv_mu;  // unbounded form: the common radius and 1 / viscosity
};

__device__ __forceinline__ void sym_item(long long t, int nb, int &I, int &J) {
    // t enumerates the upper triangle row by row: row I holds nb - I tiles.
    const double b = 2.0 * nb + 1.0;
    int r = static_cast<int>(floor(0.5 * (b - sqrt(fmax(0.0, b * b - 8.0 * static_cast<double>(t))))));
    r = max(0, min(r, nb - 1));
    auto start = [nb](long long row) { return row * nb - row * (row - 1) / 2; };
    while (r + 1 < nb && start(r + 1) <= t) ++r;
    while (r > 0 && start(r) > t) --r;
    I = r;
    J = r + static_cast<int>(t - start(r));
}

__device__ __forceinline__ void sym_load(const SymParams &p, int idx, int lane, float4 &x, float4 &f) {
    if (idx < p.n) {
        x = p.x[idx];
        f = p.f[idx];
    } else {
        // inert padding: far from everything (and from each other), zero force
        x = make_float4(1.0e5f * static_cast<float>(lane + 1), 0.0f, 1.0e4f, 0.0f);
        f = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}

// WALL false: the same scheme for the unbounded product of equal spheres (free_pair_sym_f32); the diagonal
// tiles then add each target's own self mobility, which the one-sided loop (j != i) leaves out.
template <bool WALL>
__global__ void __launch_bounds__(kThreads, kCtasPerSm) rpy_sym_kernel(SymParams p) {
    chain_wait();  // launched as a programmatic dependent of the packing launch
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int src_lane = (lane + 1) & 31;
    const long long nwarps = static_cast<long long>(gridDim.x) * (kThreads / 32);
    for (long long t = static_cast<long long>(blockIdx.x) * (kThreads / 32) + (threadIdx.x >> 5); t < p.items;
         t += nwarps) {
        int I, J;
        sym_item(t, p.nb, I, J);
        const int i = I * 32 + lane;
        const int j = J * 32 + lane;
        float4 xi, fi, xs, fs;
        sym_load(p, i, lane, xi, fi);
        sym_load(p, j, lane, xs, fs);
        const float fiv[3] = {fi.x, fi.y, fi.z};
        float vi[3] = {0.0f, 0.0f, 0.0f};
        if (I == J) {
#pragma unroll 1
            for (int step = 1; step < 32; ++step) {
                xs.x = __shfl_sync(full, xs.x, src_lane);
                xs.y = __shfl_sync(full, xs.y, src_lane);
                xs.z = __shfl_sync(full, xs.z, src_lane);
                fs.x = __shfl_sync(full, fs.x, src_lane);
                fs.y = __shfl_sync(full, fs.y, src_lane);
                fs.z = __shfl_sync(full, fs.z, src_lane);
                const float fsv[3] = {fs.x, fs.y, fs.z};
                if constexpr (WALL)
                    wall_pair_f32<3, 3>(xi.x - xs.x, xi.y - xs.y, xi.z - xs.z, xi.z, xs.z, fsv, vi);
                else
                    free_pair_f32<3, 3>(xi.x - xs.x, xi.y - xs.y, xi.z - xs.z, p.a, p.a, p.inv_mu, fsv, vi);
            }
            if constexpr (!WALL) {  // the self mobility of the target
                const float self = p.inv_mu / (6.0f * 3.14159265358979f * p.a);
                vi[0] += self * fi.x;
                vi[1] += self * fi.y;
                vi[2] += self * fi.z;
            }
            if (i < p.n) p.partial[static_cast<size_t>(i) * p.nb + I] = make_float4(vi[0], vi[1], vi[2], 0.0f);
        } else {
            float vs[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll 2
            for (int step = 0; step < 32; ++step) {
                const float fsv[3] = {fs.x, fs.y, fs.z};
                if constexpr (WALL)
                    wall_pair_sym_f32(xi.x - xs.x, xi.y - xs.y, xi.z - xs.z, xi.z, xs.z, fsv, fiv, vi, vs);
                else
                    free_pair_sym_f32(xi.x - xs.x, xi.y - xs.y, xi.z - xs.z, p.a, p.inv_mu, fsv, fiv, vi, vs);
                xs.x = __shfl_sync(full, xs.x, src_lane);
                xs.y = __shfl_sync(full, xs.y, src_lane);
                xs.z = __shfl_sync(full, xs.z, src_lane);
                fs.x = __shfl_sync(full, fs.x, src_lane);
                fs.y = __shfl_sync(full, fs.y, src_lane);
                fs.z = __shfl_sync(full, fs.z, src_lane);
                vs[0] = __shfl_sync(full, vs[0], src_lane);
                vs[1] = __shfl_sync(full, vs[1], src_lane);
                vs[2] = __shfl_sync(full, vs[2], src_lane);
            }
            if (i < p.n) p.partial[static_cast<size_t>(i) * p.nb + J] = make_float4(vi[0], vi[1], vi[2], 0.0f);
            if (j < p.n) p.partial[static_cast<size_t>(j) * p.nb + I] = make_float4(vs[0], vs[1], vs[2], 0.0f);
        }
    }
}

// ---------------------------------------------------------------------------
// Batched form of the symmetric wall kernel: many independent particle sets
// (arrays) in one launch.  Work items of all arrays are concatenated; a warp
// finds its array by binary search over the arrays' first items.  Arrays whose
// `active` flag is 0 are skipped (converged GMRES systems).  Partials are
// stored slot-major per array, partial[poff + slot * n + i] (slot = the other
// tile of the pair), so that both these writes and the per-segment reduction
// that reads them are coalesced.
__global__ void __launch_bounds__(kThreads, kCtasPerSm) rpy_wall_sym_batch_kernel(SymBatchParams p) {
    chain_wait();
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int src_lane = (lane + 1) & 31;
    const long long nwarps = static_cast<long long>(gridDim.x) * (kThreads / 32);
    for (long long t = static_cast<long long>(blockIdx.x) * (kThreads / 32) + (threadIdx.x >> 5); t < p.items;
         t += nwarps) {
        int lo = 0, hi = p.B - 1;  // last array whose first item <= t
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (p.item0[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        const int b = lo;
        if (p.active && !p.active[b]) continue;
        const int nb = p.nb[b];
        SymParams q;
        q.x = p.x + p.seg0[b];
        q.f = p.f + p.seg0[b];
        q.partial = p.partial + p.poff[b];
        q.n = p.n[b];
        q.nb = nb;
        int I, J;
        sym_item(t - p.item0[b], nb, I, J);
        const int i = I * 32 + lane;
        const int j = J * 32 + lane;
        float4 xi, fi, xs, fs;
        sym_load(q, i, lane, xi, fi);
        sym_load(q, j, lane, xs, fs);
        const float fiv[3] = {fi.x, fi.y, fi.z};
        float vi[3] = {0.0f, 0.0f, 0.0f};
        if (I == J) {
#pragma unroll 1
            for (int step = 1; step < 32; ++step) {
                xs.x = __shfl_sync(full, xs.x, src_lane);
                xs.y = __shfl_sync(full, xs.y, src_lane);
                xs.z = __shfl_sync(full, xs.z, src_lane);
                fs.x = __shfl_sync(full, fs.x, src_lane);
                fs.y = __shfl_sync(full, fs.y, src_lane);
                fs.z = __shfl_sync(full, fs.z, src_lane);
                const float fsv[3] = {fs.x, fs.y, fs.z};
                wall_pair_f32<3, 3>(xi.x - xs.x, xi.y - xs.y, xi.z - xs.z, xi.z, xs.z, fsv, vi);
            }
            if (i < q.n) q.partial[static_cast<size_t>(I) * q.n + i] = make_float4(vi[0], vi[1], vi[2], 0.0f);
        } else {
            float vs[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll 2
            for (int step = 0; step < 32; ++step) {
                const float fsv[3] = {fs.x, fs.y, fs.z};
                wall_pair_sym_f32(xi.x - xs.x, xi.y - xs.y, xi.z - xs.z, xi.z, xs.z, fsv, fiv, vi, vs);
                xs.x = __shfl_sync(full, xs.x, src_lane);
                xs.y = __shfl_sync(full, xs.y, src_lane);
                xs.z = __shfl_sync(full, xs.z, src_lane);
                fs.x = __shfl_sync(full, fs.x, src_lane);
                fs.y = __shfl_sync(full, fs.y, src_lane);
                fs.z = __shfl_sync(full, fs.z, src_lane);
                vs[0] = __shfl_sync(full, vs[0], src_lane);
                vs[1] = __shfl_sync(full, vs[1], src_lane);
                vs[2] = __shfl_sync(full, vs[2], src_lane);
            }
            if (i < q.n) q.partial[static_cast<size_t>(J) * q.n + i] = make_float4(vi[0], vi[1], vi[2], 0.0f);
            if (j < q.n) q.partial[static_cast<size_t>(I) * q.n + j] = make_float4(vs[0], vs[1], vs[2], 0.0f);
        }
    }
}

struct ReduceParams {
    const float4 *partial;
    const float4 *xt, *ft, *tt;  // self block inputs (wall, self set)
    float *out;
    const int *err;  // may be null; when the word is non-zero every output is a quiet NaN
    int nsplit, nt, ntp, stride, mode;
};

// One warp per target: the lanes stride over the target's partials, FP64
// shuffle reduction (fixed order, deterministic), lane 0 adds the wall self
// block and writes or accumulates the result.
template <bool WALL_SELF, int VD, int FD>
__global__ void rpy_reduce_kernel(ReduceParams p) {
    chain_wait();  // launched as a programmatic dependent of the tile launch
    const int lane = threadIdx.x & 31;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= p.nt) return;
    constexpr int W = VD / 3;
    double v[VD];
#pragma unroll
    for (int c = 0; c < VD; ++c) v[c] = 0.0;
    const float4 *pt = p.partial + static_cast<size_t>(i) * p.nsplit * W;
    for (int s = lane; s < p.nsplit; s += 32) {
#pragma unroll
        for (int w = 0; w < W; ++w) {
            const float4 q = pt[s * W + w];
            v[3 * w + 0] += q.x;
            v[3 * w + 1] += q.y;
            v[3 * w + 2] += q.z;
        }
    }
#pragma unroll
    for (int c = 0; c < VD; ++c)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_down_sync(0xffffffffu, v[c], o);
    if (lane != 0) return;
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
    if (p.err && *p.err) {
        // A tile block gave up waiting and left its partials unwritten: poison
        // the result instead of summing stale partials.
        for (int c = 0; c < p.stride; ++c) o[c] = __int_as_float(0x7fc00000);
        return;
    }
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

// Positions and forces (+ torques) of one particle set in one launch.
__global__ void pack_set_kernel(const float *__restrict__ x, const float *__restrict__ ft, float4 *__restrict__ xo,
                                float4 *__restrict__ fo, float4 *__restrict__ to, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        xo[i] = make_float4(x[3 * i], x[3 * i + 1], x[3 * i + 2], 0.0f);
        fo[i] = make_float4(ft[6 * i], ft[6 * i + 1], ft[6 * i + 2], 0.0f);
        if (to) to[i] = make_float4(ft[6 * i + 3], ft[6 * i + 4], ft[6 * i + 5], 0.0f);
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
    p.wait_limit = rpy_wait_limit();
    dim3 grid(plan.tiles, plan.nsplit);
    CF_CUDA(launch_chained(kern, grid, dim3(kThreads), plan.smem, st, p));
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
    const int threads = 256;  // 8 targets per block
    const int blocks = (p.nt + 7) / 8;
    CF_CUDA(launch_chained(rpy_reduce_kernel<WS, VD, FD>, dim3(blocks), dim3(threads), 0, st, p));
    CF_CHECK_LAUNCH("rpy_reduce_kernel");
    return CF_OK;
}

}  // namespace

RpyPlan rpy_plan_sym(int n, int num_sms) {
    RpyPlan pl{};
    pl.sym = 1;
    pl.ti = 1;
    const int nb = std::max(1, (n + 31) / 32);
    pl.nb = nb;
    pl.items = static_cast<long long>(nb) * (nb + 1) / 2;
    const long long max_warps = static_cast<long long>(std::max(1, num_sms)) * kCtasPerSm * (kThreads / 32);
    const long long per_warp = (pl.items + max_warps - 1) / max_warps;  // balanced: every warp does per_warp items
    const long long warps = (pl.items + per_warp - 1) / per_warp;
    pl.grid = static_cast<int>((warps + (kThreads / 32) - 1) / (kThreads / 32));
    pl.tiles = pl.grid;
    pl.nsplit = nb;  // partials per target
    pl.split = 32;
    pl.smem = 0;
    pl.scratch_float4 = static_cast<size_t>(nb) * std::max(n, 1);
    return pl;
}

RpyPlan rpy_plan(int nt, int ns, int vd, int fd, int num_sms) {
    return rpy_plan_capped(nt, ns, vd, fd, num_sms, 1 << 30);
}

RpyPlan rpy_plan_capped(int nt, int ns, int vd, int fd, int num_sms, int max_nsplit) {
    // Every CTA does the same work (128*TI targets x `split` sources), so the
    // kernel time is (waves) x (time of one CTA).  Choose the split count that
    // minimises waves * (split + staging overhead), with the resident CTA count
    // per SM bounded by the launch bounds (8) and by shared memory.
    RpyPlan pl{};
    pl.ti = (vd == 3) ? 2 : 1;
    const int per_cta = kThreads * pl.ti;
    pl.tiles = std::max(1, (nt + per_cta - 1) / per_cta);
    const int sms = std::max(1, num_sms);
    const size_t src_bytes = sizeof(float4) * (fd > 3 ? 3 : 2);
    const int nmin = std::max(1, (ns + kMaxSplit - 1) / kMaxSplit);
    const int nmax = std::max(nmin, std::min(std::min(ns / kMinSplit, 8 * sms), max_nsplit));
    int best_nsplit = nmin;
    double best_cost = 1e300;
    for (int cand = nmin; cand <= nmax; ++cand) {
        const int split = std::max(1, (ns + cand - 1) / cand);
        const int nsplit = std::max(1, (ns + split - 1) / split);
        const size_t smem = 16 + static_cast<size_t>(split) * src_bytes;
        const int cap = std::min<int>(kCtasPerSm, static_cast<int>((227u * 1024u) / (smem + 1024u)));
        if (cap < 1) continue;
        const long long slots = static_cast<long long>(sms) * cap;
        const long long ctas = static_cast<long long>(pl.tiles) * nsplit;
        const long long waves = (ctas + slots - 1) / slots;
        // fewer than 4 resident CTAs (16 warps) per SM issues poorly: penalise
        const double occ = cap >= 4 ? 1.0 : 4.0 / cap;
        const double cost = static_cast<double>(waves) * (split + kStageCost) * occ;
        if (cost < best_cost - 1e-9) {
            best_cost = cost;
            best_nsplit = nsplit;
        }
    }
    pl.split = std::max(1, (ns + best_nsplit - 1) / best_nsplit);
    pl.nsplit = std::max(1, (ns + pl.split - 1) / pl.split);
    pl.smem = 16 + static_cast<size_t>(pl.split) * src_bytes;
    pl.scratch_float4 = static_cast<size_t>(pl.nsplit) * (vd / 3) * std::max(nt, 1);
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
    if (plan.sym) {
        SymParams p;
        p.x = d.xs;
        p.f = d.fs;
        p.partial = scratch;
        p.n = d.nt;
        p.nb = plan.nb;
        p.items = plan.items;
        p.a = d.at;
        p.inv_mu = 1.0f / d.mu;
        if (d.wall) CF_CUDA(launch_chained(rpy_sym_kernel<true>, dim3(plan.grid), dim3(kThreads), 0, st, p));
        else CF_CUDA(launch_chained(rpy_sym_kernel<false>, dim3(plan.grid), dim3(kThreads), 0, st, p));
        CF_CHECK_LAUNCH("rpy_sym_kernel");
        return CF_OK;
    }
    const bool self = d.self_set != 0;
    if (d.wall) return self ? dispatch_dof<true, true>(d, plan, scratch, dev_err, st)
                            : dispatch_dof<true, false>(d, plan, scratch, dev_err, st);
    // Unbounded blocks need no mask: r = 0 is handled by the containment branch.
    return dispatch_dof<false, false>(d, plan, scratch, dev_err, st);
}

int rpy_prepare(const RpyBlockDesc &d, const RpyPlan &plan) {
    if (plan.sym) return CF_OK;  // no dynamic shared memory
    const bool self = d.self_set != 0;
    if (d.wall && self) {
        if (d.vd == 3 && d.fd == 3) return plan.ti == 2 ? configure_tiles_t<true, 3, 3, 2, true>() : configure_tiles_t<true, 3, 3, 1, true>();
        if (d.vd == 6 && d.fd == 6) return plan.ti == 2 ? configure_tiles_t<true, 6, 6, 2, true>() : configure_tiles_t<true, 6, 6, 1, true>();
    }
    return CF_OK;  // other instantiations configure themselves on first launch
}

int rpy_launch_reduce_f32(const RpyBlockDesc &d, const RpyPlan &plan, const float4 *scratch, float *out_f,
                          int stride, int mode, cudaStream_t st, const int *dev_err) {
    if (d.nt <= 0) return CF_OK;
    ReduceParams p;
    p.partial = scratch;
    p.err = dev_err;
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

int pack_set_to_float4(const float *aos3, const float *aos6, float4 *x, float4 *force, float4 *torque, int n,
                       cudaStream_t st) {
    if (n <= 0) return CF_OK;
    pack_set_kernel<<<(n + 255) / 256, 256, 0, st>>>(aos3, aos6, x, force, torque, n);
    CF_CHECK_LAUNCH("pack_set_kernel");
    return CF_OK;
}

int pack_ft6_to_float4(const float *aos6, float4 *force, float4 *torque, int n, cudaStream_t st) {
    if (n <= 0) return CF_OK;
    pack_ft6_kernel<<<(n + 255) / 256, 256, 0, st>>>(aos6, force, torque, n);
    CF_CHECK_LAUNCH("pack_ft6_kernel");
    return CF_OK;
}

RpyPlan rpy_plan_for(const RpyBlockDesc &d, int num_sms) {
    if (d.wall && d.self_set && d.vd == 3 && d.fd == 3 && d.nt == d.ns && d.xt == d.xs)
        return rpy_plan_sym(d.nt, num_sms);
    if (!d.wall && d.vd == 3 && d.fd == 3 && d.nt == d.ns && d.xt == d.xs && d.at == d.as)  // equal spheres
        return rpy_plan_sym(d.nt, num_sms);
    return rpy_plan(d.nt, d.ns, d.vd, d.fd, num_sms);
}

int rpy_block_product(const RpyBlockDesc &d, float4 *scratch, size_t scratch_cap, int *dev_err, float *out_f,
                      int stride, int mode, int num_sms, cudaStream_t st) {
    if (d.nt <= 0) return CF_OK;
    RpyPlan plan = rpy_plan_for(d, num_sms);
    if (plan.scratch_float4 > scratch_cap)
        return set_error(CF_EINVAL, "rpy: scratch too small (%zu < %zu float4)", scratch_cap, plan.scratch_float4);
    if (d.ns > 0) CF_TRY(rpy_launch_tiles(d, plan, scratch, dev_err, st));
    return rpy_launch_reduce_f32(d, plan, scratch, out_f, stride, mode, st, plan.sym ? nullptr : dev_err);
}

}  // namespace cufil

namespace {
std::atomic<unsigned> g_wait_limit{cufil::kMbarSpinLimit};
}

namespace cufil {

unsigned rpy_wait_limit() { return g_wait_limit.load(std::memory_order_relaxed); }

}  // namespace cufil

// Test hook: sets the tries of the first bounded wait of later tile launches
// (0: give up at once); a value above the default is clamped to it.
extern "C" int cf_set_wait_limit(unsigned limit) {
    cufil::clear_error();
    g_wait_limit.store(limit < cufil::kMbarSpinLimit ? limit : cufil::kMbarSpinLimit, std::memory_order_relaxed);
    return CF_OK;
}

namespace cufil {

int rpy_launch_sym_batch(const SymBatchParams &p, int grid, cudaStream_t st) {
    if (p.items <= 0) return CF_OK;
    CF_CUDA(launch_chained(rpy_wall_sym_batch_kernel, dim3(grid), dim3(kThreads), 0, st, p));
    return CF_OK;
}

int rpy_sym_batch_max_grid(int num_sms) { return std::max(1, num_sms) * kCtasPerSm; }

}  // namespace cufil

// patch_kernels.cuh -- line-patch block-Jacobi preconditioner of the implicit step.
//
// Filaments are grouped into patches of up to P neighbours along a lattice
// line in the beat direction (the beat plane of the wall frame is y-z, so a
// patch is a run of filaments with equal x, consecutive in y).  Each patch's
// saddle-point block
//     [ M_pp   -K_p ]      M_pp : wall RPY mobility of all segments of the patch
//     [ -K_p^T   0  ]      K_p  : velocity directions (K_phase, K_angle) per filament
// -- the same operator as system_matrix_mult_new (mobility_solver.cpp:1887-2105)
// restricted to the patch -- is assembled in FP32 and inverted in place by a
// blocked Gauss-Jordan elimination without pivoting, in per-filament order
// ([3*nseg lambda | phase rate | angle rate] per filament): every 62-unknown
// filament block is eliminated lambda-first, so the rate pivots are Schur
// complements -k^T M^-1 k and stay away from zero.  The elimination is the
// symmetric sweep (every intermediate matrix stays symmetric), so only the upper
// block triangle is updated and the result is -A_pp^-1.  The preconditioner is
// P^-1 r = blockdiag(A_pp^-1) r; it replaces apply_preconditioner_new
// (mobility_solver.cpp:1102-1243), whose block-diagonal form (6 pi a on the
// forces, a 2x2 Schur solve for the rates) remains the fallback of any patch
// whose inverse is not finite.  The GMRES residual is always formed with the
// exact operator, so the patch inverses change only the iteration count.
//
// Cost: one refresh is sum_p n_p^3 FP32 FMAs (n_p = 62 * filaments), done as
// ceil(n/64) rounds of (a) inverting the 64x64 pivot block (one block per
// patch), (b) scaling the pivot rows and saving the pivot columns (one thread
// per column) and (c) a rank-64 update of the matrix in 64x64 tiles.  One application is a dense n_p x n_p product per
// patch, reading the FP32 inverses once.
#pragma once

#include "rpy_pairs.cuh"
#include "sim_kernels.cuh"
#include "tc_tf32.cuh"

namespace cufil {

constexpr int kGjBlock = 64;  // pivot block of the Gauss-Jordan rounds
constexpr int kGjTile = 64;   // tile of the rank-64 updates

struct PatchDev {
    int np;                  // patches
    int nbf;                 // unknowns per filament (3*nseg + rate rows)
    int max_n;               // largest patch system
    int T;                   // 64-wide tiles per side of the largest patch
    const int *fil0;         // first entry of each patch in `fils` [np]
    const int *nf;           // filaments per patch [np]
    const int *fils;         // filament ids (batch numbering), patch by patch
    const long long *moff;   // first float of each patch matrix [np]
    const long long *roff;   // first entry of each patch in `rows` [np]
    const long long *rows;   // batch-vector row of each local unknown
    float *A;                // patch matrices, then their inverses (row-major n x n, row stride patch_ld(n))
    // Round operands of the tile update, per patch and 64-column tile, split for the tensor cores
    // (tc_tf32.cuh: a TF32 high part and an FP32 remainder, 4096 floats each, canonical K-major
    // layout with k the pivot row s and m or n the tile column c):
    float *csplit;           // the pivot-row copies U[s][c], [np][T][2][4096]
    float *rsplit;           // the scaled pivot rows (D^-1 U)[s][c] (-D^-1 in the pivot columns), same shape
    float *dinv;             // inverted pivot blocks, [np][kGjBlock][kGjBlock]
    int *ok;                 // [np] 1 when the inverse is finite
    int *counter;            // per-round tile counters of the update [rounds]
};

// Row stride of a patch system of n unknowns: rows start on 16 bytes, so tiles
// move in 16-byte copies.  The padding columns [n, ld) are never part of a result.
__host__ __device__ __forceinline__ int patch_ld(int n) { return (n + 3) & ~3; }

// Mobility entries: one thread per (target segment, source segment) pair of a
// patch; writes the 3x3 block into the lambda rows / columns.
__global__ void patch_mobility_kernel(SimDev d, PatchDev P) {
    const int p = blockIdx.y;
    const int nfp = P.nf[p];
    const int ns = nfp * d.nseg;
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<long long>(ns) * ns) return;
    const int si = static_cast<int>(t / ns), sj = static_cast<int>(t - static_cast<long long>(si) * ns);
    const int ai = si / d.nseg, ki = si - ai * d.nseg;
    const int aj = sj / d.nseg, kj = sj - aj * d.nseg;
    const int gi = P.fils[P.fil0[p] + ai] * d.nseg + ki;
    const int gj = P.fils[P.fil0[p] + aj] * d.nseg + kj;
    const int ld = patch_ld(nfp * P.nbf);
    float *A = P.A + P.moff[p];
    const long long r0 = static_cast<long long>(ai) * P.nbf + 3 * ki;
    const long long c0 = static_cast<long long>(aj) * P.nbf + 3 * kj;
    if (r0 / kGjTile > (c0 + 2) / kGjTile) return;  // wholly in the lower block triangle, which the sweep never reads
    const float zi = static_cast<float>(d.xd[3 * gi + 2]);
    for (int c = 0; c < 3; ++c) {
        float f[3] = {0.0f, 0.0f, 0.0f}, v[3] = {0.0f, 0.0f, 0.0f};
        f[c] = 1.0f;
        if (gi == gj) {
            wall_self_f32<3, 3>(zi, f, v);
        } else {
            const float dx = static_cast<float>(d.xd[3 * gi] - d.xd[3 * gj]);
            const float dy = static_cast<float>(d.xd[3 * gi + 1] - d.xd[3 * gj + 1]);
            const float dz = static_cast<float>(d.xd[3 * gi + 2] - d.xd[3 * gj + 2]);
            wall_pair_f32<3, 3>(dx, dy, dz, zi, static_cast<float>(d.xd[3 * gj + 2]), f, v);
        }
        for (int q = 0; q < 3; ++q)  // the sweep reads the upper block triangle only
            if ((r0 + q) / kGjTile <= (c0 + c) / kGjTile) A[(r0 + q) * ld + c0 + c] = v[q];
    }
}

// Rate rows and columns of a patch: -K / -K^T of each filament, zero between
// filaments and between rates.  grid = (entry chunks, patches).
__global__ void patch_rates_kernel(SimDev d, PatchDev P) {
    const int p = blockIdx.y;
    const int nfp = P.nf[p];
    const int n = nfp * P.nbf, ld = patch_ld(n);
    const int nl = 3 * d.nseg, nr = P.nbf - nl;  // lambda rows and rate rows per filament
    float *A = P.A + P.moff[p];
    // every (row, rate column) entry and its transpose: -k of the row's own filament, zero elsewhere (the
    // matrix is not cleared between rebuilds: the lambda block is assembled in full, and this covers the rest)
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n * nfp * nr; e += gridDim.x * blockDim.x) {
        const int rc = e / n, r = e - rc * n;
        const int a = rc / nr, q = rc - a * nr;  // rate column: filament a, rate q (phase first)
        const int c = a * P.nbf + nl + q;
        const int ar = r / P.nbf, li = r - ar * P.nbf;
        float v = 0.0f;
        if (ar == a && li < nl) {
            const int g3 = 3 * P.fils[P.fil0[p] + a] * d.nseg + li;  // entry of kp / ka
            v = -static_cast<float>((d.dyn_phase && q == 0) ? d.kp[g3] : d.ka[g3]);
        }
        A[static_cast<size_t>(r) * ld + c] = v;
        A[static_cast<size_t>(c) * ld + r] = v;
    }
}

// acc = L R for 64x64 blocks in shared memory (leading dimension kInvLd, 16-byte
// rows); each of the 256 threads owns rows 4*(tid/16) + u and columns
// 4*(tid%16) + v, the R operand read as one float4 per step.
constexpr int kInvLd = kGjBlock + 4;
__device__ __forceinline__ void block_gemm64(const float *L, const float *R, float (&acc)[4][4]) {
    const int r0 = 4 * (threadIdx.x >> 4), c0 = 4 * (threadIdx.x & 15);
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = 0.0f;
#pragma unroll 8
    for (int k = 0; k < kGjBlock; ++k) {
        float l[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) l[u] = L[(r0 + u) * kInvLd + k];
        const float4 r4 = *reinterpret_cast<const float4 *>(&R[k * kInvLd + c0]);
        const float r[4] = {r4.x, r4.y, r4.z, r4.w};
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[u][v] = fmaf(l[u], r[v], acc[u][v]);
    }
}

// The pivot block D (rows and columns [k0, k0 + b) of A, padded with the identity to 64 x 64) into M.
__device__ __forceinline__ void load_pivot_block(const float *A, int n, int k0, int b, float *M) {
    for (int e = threadIdx.x; e < kGjBlock * kGjBlock; e += blockDim.x) {
        const int r = e >> 6, c = e & 63;
        M[r * kInvLd + c] = (r < b && c < b) ? A[static_cast<size_t>(k0 + r) * patch_ld(n) + k0 + c] : (r == c ? 1.0f : 0.0f);
    }
}

// Part (a) of a round: inverts pivot block K of patch p (rows and columns
// [64K, 64K + b)) into its dinv block, zero-padded to 64 x 64; called by all
// 256 threads of a block.  The 64x64 block D (padded with the identity beyond
// b) is inverted in place by Gauss-Jordan elimination without pivoting in
// registers: thread (row r = tid / 4, quarter g = tid % 4) holds D[r][16g ..
// 16g + 15], so warp w holds rows 8w .. 8w + 7.  The pivots are taken in eight
// panels of eight (block Gauss-Jordan, two barriers per panel instead of one
// per pivot; the loop below says how).  Forming the inverse explicitly loses accuracy
// when D is ill conditioned, so the result X is refined by one Newton step,
// X <- X + X (I - D X), which squares its residual.  A zero or non-finite
// pivot clears the patch's ok flag.
// A: the patch matrix (n x n), dv: its dinv block, ok: its flag, ws: shared
// memory of at least kInvWs floats.
constexpr int kInvWs = 2 * kGjBlock * kInvLd;
__device__ __noinline__ void pivot_invert(const float *A, int n, float *dv, int *ok, int K, float *ws) {
    static_assert(kGjBlock == 64, "four threads of 16 columns per row, eight rows per warp");
    const int k0 = K * kGjBlock;
    const int b = min(kGjBlock, n - k0);
    float *X = ws, *W = ws + kGjBlock * kInvLd;  // X: the inverse; W: D, then I - D X
    const int r = threadIdx.x >> 2, g = threadIdx.x & 3;
    const size_t ld = patch_ld(n);
    float v[16];
    {
        const float *Ar = A + (k0 + r) * ld + k0 + 16 * g;
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int c = 16 * g + q;
            v[q] = (r < b && c < b) ? Ar[q] : (r == c ? 1.0f : 0.0f);
        }
    }
    // Eight panels of eight pivots, panel m held by warp m (rows 8m .. 8m + 7): the warp eliminates the
    // panel's pivots inside its own rows (pivot rows and column entries by shuffles, no block barrier),
    // publishes its rows and every other row its entries in the panel's columns, and after one barrier every
    // other row takes the rank-8 update  x <- [x outside the panel columns] - a_G panel  (block Gauss-Jordan).
    __shared__ __align__(16) float panel[8][kGjBlock];
    __shared__ __align__(16) float colg[kGjBlock][8];
    __shared__ int sbad;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, rl = lane >> 2;
    if (threadIdx.x == 0) sbad = 0;
#pragma unroll 1
    for (int m = 0; m < 8; ++m) {
        const int cg = m >> 1, half = m & 1;  // the panel's columns 8m + t: chunk cg, element 8 half + t
        if (w == m) {
            bool bad = false;
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                float p[16];
#pragma unroll
                for (int q = 0; q < 16; ++q) p[q] = __shfl_sync(0xffffffffu, v[q], 4 * t + g);  // pivot row
                const float mine = half ? v[8 + t] : v[t];
                const float f = __shfl_sync(0xffffffffu, mine, (lane & ~3) | cg);  // this row's entry, column k
                const float piv = __shfl_sync(0xffffffffu, mine, 4 * t + cg);
                bad |= !(fabsf(piv) > 0.0f) || !isfinite(piv);
                const float ip = __frcp_rn(piv);
                // v <- a v + b p with (a, b) = (0, 1/piv) in the pivot row, (1, -f/piv) elsewhere; the pivot
                // column takes b itself
                const bool own = rl == t;
                const float a = own ? 0.0f : 1.0f, bq = own ? ip : -f * ip;
#pragma unroll
                for (int q = 0; q < 16; ++q) v[q] = fmaf(bq, p[q], a * v[q]);
                if (g == cg) {
                    if (half) v[8 + t] = bq;
                    else v[t] = bq;
                }
            }
            if (bad) sbad = 1;
#pragma unroll
            for (int q = 0; q < 16; q += 4)
                *reinterpret_cast<float4 *>(&panel[rl][16 * g + q]) = make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]);
        } else if (g == cg) {
            const float4 a0 = half ? make_float4(v[8], v[9], v[10], v[11]) : make_float4(v[0], v[1], v[2], v[3]);
            const float4 a1 = half ? make_float4(v[12], v[13], v[14], v[15]) : make_float4(v[4], v[5], v[6], v[7]);
            *reinterpret_cast<float4 *>(&colg[r][0]) = a0;
            *reinterpret_cast<float4 *>(&colg[r][4]) = a1;
        }
        __syncthreads();
        if (w != m) {
            const float4 a0 = *reinterpret_cast<const float4 *>(&colg[r][0]);
            const float4 a1 = *reinterpret_cast<const float4 *>(&colg[r][4]);
            const float ag[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            if (g == cg) {  // the panel's columns are replaced, not updated
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    if (half) v[8 + q] = 0.0f;
                    else v[q] = 0.0f;
                }
            }
#pragma unroll
            for (int t = 0; t < 8; ++t) {
#pragma unroll
                for (int q = 0; q < 16; q += 4) {
                    const float4 pp = *reinterpret_cast<const float4 *>(&panel[t][16 * g + q]);
                    v[q] = fmaf(-ag[t], pp.x, v[q]);
                    v[q + 1] = fmaf(-ag[t], pp.y, v[q + 1]);
                    v[q + 2] = fmaf(-ag[t], pp.z, v[q + 2]);
                    v[q + 3] = fmaf(-ag[t], pp.w, v[q + 3]);
                }
            }
        }
        __syncthreads();  // panel and colg are rewritten by the next panel
    }
    const bool bad = sbad != 0;
#pragma unroll
    for (int q = 0; q < 16; q += 4)
        *reinterpret_cast<float4 *>(X + r * kInvLd + 16 * g + q) = make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]);
    // Newton step: W = D, then W = I - D X, then X + X W straight to dv
    load_pivot_block(A, n, k0, b, W);
    __syncthreads();
    float acc[4][4];
    block_gemm64(W, X, acc);
    __syncthreads();
    const int r0 = 4 * (threadIdx.x >> 4), c0 = 4 * (threadIdx.x & 15);
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int w = 0; w < 4; ++w) W[(r0 + u) * kInvLd + c0 + w] = (r0 + u == c0 + w ? 1.0f : 0.0f) - acc[u][w];
    __syncthreads();
    block_gemm64(X, W, acc);
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int w = 0; w < 4; ++w) {
            const int rr = r0 + u, c = c0 + w;
            dv[rr * kGjBlock + c] = (rr < b && c < b) ? X[rr * kInvLd + c] + acc[u][w] : 0.0f;
        }
    if (threadIdx.x == 0) {
        if (bad) *ok = 0;
        else if (K == 0) *ok = 1;
    }
}

__device__ __forceinline__ void pivot_invert_patch(const PatchDev &P, int p, int K, float *ws) {
    pivot_invert(P.A + P.moff[p], P.nf[p] * P.nbf, P.dinv + static_cast<size_t>(p) * kGjBlock * kGjBlock, P.ok + p, K,
                 ws);
}

// Round 0, part (a): the first pivot block of every patch (later pivot blocks
// are inverted by the previous round's update, see gj_update_kernel).
__global__ void __launch_bounds__(256) gj_pivot_kernel(PatchDev P, int K) {
    __shared__ __align__(16) float ws[kInvWs];
    const int p = blockIdx.x;
    const int n = P.nf[p] * P.nbf;
    if (K * kGjBlock >= n) return;
    pivot_invert_patch(P, p, K, ws);
}

// Round K, part (b), one 64-column tile [j0, j0 + 64) of a patch per block.
// The matrix is kept symmetric and only its upper block triangle is
// maintained, so the pivot rows' entries are
//   U[s][j] = A[k0 + s][j] for j >= k0,   A[j][k0 + s] for j < k0  (by symmetry);
// both are read as 64 contiguous floats per row of A and staged in shared
// memory as U[s][c].  The pass writes, for the tile's columns c (j = j0 + c),
//   rsplit: (D^-1 U)[s][c] outside the pivot columns, -D^-1[s][c] inside,
//   csplit: U[s][c]         outside the pivot columns (zero inside),
// each split into its TF32 high part and FP32 remainder in the canonical layout of
// the tensor-core operands (element (c, s) at tc::canon(c, s)), the form in which
// the update pass multiplies them.  Tiles and pivot blocks are both 64 wide, so a tile is either the pivot
// block's or disjoint from it.  Each thread owns 4 rows x 4 columns of
// D^-1 U (rows 4ty + u, columns 4tx + v); the loads and stores of the
// product's operands and results move 16 bytes each.  grid = (tiles, patches).
__global__ void __launch_bounds__(256) gj_prep_kernel(PatchDev P, int K) {
    static_assert(kGjTile == kGjBlock, "column tiles are pivot-block wide");
    constexpr int LD = kGjTile + 4;  // 16-byte rows
    __shared__ __align__(16) float DvT[kGjBlock][LD];  // DvT[s][r] = D^-1[r][s]
    __shared__ __align__(16) float Us[kGjBlock][LD];
    chain_wait();
    const int p = blockIdx.y;
    const int n = P.nf[p] * P.nbf;
    const int k0 = K * kGjBlock;
    const int j0 = blockIdx.x * kGjTile;
    if (k0 >= n || j0 >= n) return;
    const int b = min(kGjBlock, n - k0);
    const int w = min(kGjTile, n - j0);  // columns in this tile
    const size_t ld = patch_ld(n);
    const float *A = P.A + P.moff[p];
    float *rs = P.rsplit + (static_cast<size_t>(p) * P.T + blockIdx.x) * 2 * tc::kOperandFloats;
    float *cs = P.csplit + (static_cast<size_t>(p) * P.T + blockIdx.x) * 2 * tc::kOperandFloats;
    const float *dv = P.dinv + static_cast<size_t>(p) * kGjBlock * kGjBlock;
    if (j0 == k0) {  // the pivot columns: -D^-1, and no pivot-row copies
        for (int e = threadIdx.x; e < kGjBlock * kGjTile; e += blockDim.x) {
            const int r = e / kGjTile, c = e - r * kGjTile;
            float h, l;
            tc::split_tf32(c < w ? -dv[r * kGjBlock + c] : 0.0f, h, l);  // zero-padded rows
            rs[tc::canon(c, r)] = h;
            rs[tc::kOperandFloats + tc::canon(c, r)] = l;
            cs[tc::canon(c, r)] = 0.0f;
            cs[tc::kOperandFloats + tc::canon(c, r)] = 0.0f;
        }
        return;
    }
    // D^-1, 16-byte loads, stored transposed
    for (int e4 = threadIdx.x; e4 < kGjBlock * kGjBlock / 4; e4 += blockDim.x) {
        const int r = e4 >> 4, c4 = 4 * (e4 & 15);
        const float4 v = *reinterpret_cast<const float4 *>(dv + r * kGjBlock + c4);
        DvT[c4][r] = v.x;
        DvT[c4 + 1][r] = v.y;
        DvT[c4 + 2][r] = v.z;
        DvT[c4 + 3][r] = v.w;
    }
    // U, 16-byte chunks of rows of A; chunks at or beyond the row stride are zeros, and so are the padding
    // columns [n, ld) inside it, so U[s][c] is zero for s >= b or c >= w as the product needs
    if (j0 > k0) {  // U[s][c] = A[k0 + s][j0 + c]
        for (int e4 = threadIdx.x; e4 < kGjBlock * kGjTile / 4; e4 += blockDim.x) {
            const int s_ = e4 >> 4, c4 = 4 * (e4 & 15);
            float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if (s_ < b && j0 + c4 < static_cast<int>(ld)) v = *reinterpret_cast<const float4 *>(A + (k0 + s_) * ld + j0 + c4);
            *reinterpret_cast<float4 *>(&Us[s_][c4]) = v;
        }
    } else {  // j0 + 64 <= k0: U[s][c] = A[j0 + c][k0 + s], rows of A read contiguously, stored transposed
        for (int e4 = threadIdx.x; e4 < kGjTile * kGjBlock / 4; e4 += blockDim.x) {
            const int c = e4 >> 4, s4 = 4 * (e4 & 15);
            float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if (k0 + s4 < static_cast<int>(ld)) v = *reinterpret_cast<const float4 *>(A + (j0 + c) * ld + k0 + s4);
            Us[s4][c] = v.x;
            Us[s4 + 1][c] = v.y;
            Us[s4 + 2][c] = v.z;
            Us[s4 + 3][c] = v.w;
        }
    }
    __syncthreads();
    // rows 4ty + u, columns 4tx + v of D^-1 U: one float4 of each operand per step
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    float acc[4][4] = {};
#pragma unroll 8
    for (int s_ = 0; s_ < kGjBlock; ++s_) {
        const float4 d4 = *reinterpret_cast<const float4 *>(&DvT[s_][4 * ty]);
        const float4 u4 = *reinterpret_cast<const float4 *>(&Us[s_][4 * tx]);
        const float dr[4] = {d4.x, d4.y, d4.z, d4.w}, uc[4] = {u4.x, u4.y, u4.z, u4.w};
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[u][v] = fmaf(dr[u], uc[v], acc[u][v]);
    }
    const int c0 = 4 * tx;
    __syncthreads();  // DvT is free: it holds the product tile while it is written out
    float(*Pt)[LD] = DvT;
#pragma unroll
    for (int u = 0; u < 4; ++u)  // rows >= b: zeros (D^-1 is zero-padded); columns >= w: zeros
        *reinterpret_cast<float4 *>(&Pt[4 * ty + u][c0]) =
            make_float4(c0 < w ? acc[u][0] : 0.0f, c0 + 1 < w ? acc[u][1] : 0.0f, c0 + 2 < w ? acc[u][2] : 0.0f,
                        c0 + 3 < w ? acc[u][3] : 0.0f);
    __syncthreads();
    // both operands written in the canonical order (consecutive threads, consecutive addresses): element q of
    // the layout is (c, s) = tc::canon_inverse(q); the pivot-row entries are U itself (zero beyond w, as U is)
    for (int q = threadIdx.x; q < tc::kOperandFloats; q += blockDim.x) {
        const int c = tc::canon_mn(q), s_ = tc::canon_k(q);
        float h, l;
        tc::split_tf32(Pt[s_][c], h, l);
        rs[q] = h;
        rs[tc::kOperandFloats + q] = l;
        tc::split_tf32(Us[s_][c], h, l);
        cs[q] = h;
        cs[tc::kOperandFloats + q] = l;
    }
}

// 16-byte asynchronous copy global -> shared (zero-filled when !valid; src is
// then not read but must still be a mapped address).  Both addresses 16-byte aligned.
__device__ __forceinline__ void cp_async16(float *dst, const float *src, bool valid) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// One tile of round K's update: which tile of which patch, and its kind.
struct GjTile {
    int p, n, row0, col0;
    bool valid, prow, pcol, diag;
};

// Work item -> tile.  Items run patch-fastest over a triangle enumeration of
// the upper block triangle (T = the largest patch's tiles per side) in which
// index 0 is the next round's diagonal tile (K + 1, K + 1), so the first np
// items are the patches' diagonal tiles and are taken first.
__device__ __forceinline__ GjTile gj_tile(const PatchDev &P, int K, int T, int item) {
    GjTile t{};
    t.p = item % P.np;
    int q = item / P.np;
    t.n = P.nf[t.p] * P.nbf;
    const int Tp = (t.n + kGjTile - 1) / kGjTile;
    const int d = K + 1;
    if (d < T) {
        const int qd = d * T - d * (d - 1) / 2;  // triangle index of (d, d)
        q = (q == 0) ? qd : (q <= qd ? q - 1 : q);
    }
    int ti = 0;
    while (ti < T && q >= T - ti) {
        q -= T - ti;
        ++ti;
    }
    const int tj = ti + q;
    t.valid = K * kGjBlock < t.n && ti < Tp && tj < Tp;
    t.row0 = ti * kGjTile;
    t.col0 = tj * kGjTile;
    t.prow = ti == K;
    t.pcol = tj == K;
    t.diag = ti == d && tj == d;
    return t;
}

// Stage of the update: the tile's split operands as the prep pass left them
// (A = the pivot-row copies of its row tile, B = the scaled pivot rows of its
// column tile, each a TF32 high part and an FP32 remainder in the canonical
// layout, 4 x 16 KB).  The old values are read from global memory by the
// epilogue.  One stage per block and two blocks per SM: one block's copies
// overlap the other's products and stores.
constexpr int kUpStage = 4 * tc::kOperandFloats;
constexpr size_t kUpdateSmem = kUpStage * sizeof(float);

// Issues the 16-byte copies of a tile's operands into `stage` (contiguous blocks: 8 + 8 chunks per thread;
// the pivot rows need B only).
__device__ __forceinline__ void gj_issue_tile(const PatchDev &P, const GjTile &t, float *stage) {
    float *Ab = stage, *Bb = stage + 2 * tc::kOperandFloats;
    const float *csrc = P.csplit + (static_cast<size_t>(t.p) * P.T + t.row0 / kGjTile) * 2 * tc::kOperandFloats;
    const float *rsrc = P.rsplit + (static_cast<size_t>(t.p) * P.T + t.col0 / kGjTile) * 2 * tc::kOperandFloats;
    for (int c = threadIdx.x; c < 2 * tc::kOperandFloats / 4; c += blockDim.x) {
        cp_async16(Bb + 4 * c, rsrc + 4 * c, true);
        if (!t.prow) cp_async16(Ab + 4 * c, csrc + 4 * c, true);
    }
}

// Round K, part (c), the 64x64 tiles of the upper block triangle:
//   pivot rows       A[i, j] = rbuf[i - k0][j]      (-D^-1 in the pivot block)
//   other rows       A[i, j] -= C_i . rbuf[:, j]   (j outside the pivot columns)
//                    A[i, j]  = -C_i . rbuf[:, j]  (pivot columns: C_i D^-1)
// with C_i = cbuf[:][i] (the pivot-row copies) and rbuf the scaled pivot rows
// -- the symmetric sweep, which leaves -A^-1 after the last round.  Tiles and
// pivot blocks are both 64 wide, so a tile lies in the pivot rows (ti == K, a
// copy), in the pivot columns (tj == K) or in neither.  Persistent blocks (two
// per SM) take tiles from a per-round counter.  The tile product C^T rbuf runs
// on the tensor cores (tc_tf32.cuh: the operands as the prep pass split them,
// three TF32 products accumulated in FP32 in tensor memory, issued by one
// thread and committed to an mbarrier).  Read-back: warp w holds tile rows
// 16 (w % 4) .. + 15 in lanes 0-15 and columns 32 (w / 4) .. + 31; each lane
// pair (l, l + 16) then splits the 32 columns, so every thread writes 16
// columns of one row.  The block that takes a patch's diagonal tile
// (K + 1, K + 1) inverts it for the next round right after its update, while
// the other blocks go on with the rest.  A wait for the products that gives up
// (bounded) marks the tile's patch unusable -- it falls back to the
// block-diagonal preconditioner -- and the block computes no further products.
// Dynamic shared memory: kUpdateSmem.
__global__ void __launch_bounds__(256, 2) gj_update_kernel(PatchDev P, int K, int T, int *counter) {
    static_assert(kGjTile == 64 && kGjBlock == 64 && tc::kTileMN == 64 && tc::kTileK == 64, "64-wide tiles");
    static_assert(kUpStage >= kInvWs, "the inversion reuses the stage");
    extern __shared__ __align__(128) float usm[];
    __shared__ int next_item;
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tbase;
    __shared__ int tc_ok, dead;
    chain_wait();
    const int total = P.np * (T * (T + 1) / 2);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) next_item = atomicAdd(counter, 1);
    __syncthreads();
    int item = next_item;
    if (item >= total) return;
    if (warp == 0) tc::tmem_alloc(&tbase, tc::kTmemCols);
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
        dead = 0;
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tbase;
    uint32_t products = 0;  // completed phases of `bar`
    const float *Ab = usm, *Bb = usm + 2 * tc::kOperandFloats;
    // this thread's output: tile row tr, columns tc0 .. tc0 + 15
    const int tr = 16 * (warp & 3) + (lane & 15), tc0 = 32 * (warp >> 2) + 16 * (lane >> 4);
    while (item < total) {
        const GjTile cur = gj_tile(P, K, T, item);
        if (cur.valid) {
            gj_issue_tile(P, cur, usm);
            cp_async_commit();
            const int n = cur.n, ld = patch_ld(n);
            const int i = cur.row0 + tr, j = cur.col0 + tc0;
            float *Arow = P.A + P.moff[cur.p] + static_cast<size_t>(i) * ld + j;
            // the old values, while the operands land (the pivot columns and rows are overwritten)
            float res[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) res[q] = 0.0f;
            if (!cur.prow && !cur.pcol && i < n) {
#pragma unroll
                for (int q = 0; q < 16; q += 4) {
                    if (j + q < ld) {
                        const float4 o4 = *reinterpret_cast<const float4 *>(Arow + q);
                        res[q] = o4.x;
                        res[q + 1] = o4.y;
                        res[q + 2] = o4.z;
                        res[q + 3] = o4.w;
                    }
                }
            }
            cp_async_wait<0>();
            tc::fence_proxy_async();  // the operands are visible to the tensor cores
            tc::fence_before_sync();
            __syncthreads();
            tc::fence_after_sync();
            bool have = true;
            if (cur.prow) {  // the pivot rows: the scaled pivot rows themselves (row0 == k0), high + low parts
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    const int e = tc::canon(tc0 + q, tr);
                    res[q] = Bb[e] + Bb[tc::kOperandFloats + e];
                }
            } else if (dead) {
                have = false;
            } else {
                if (threadIdx.x == 0) {
                    tc::issue_tile_products(tmem, Ab, Ab + tc::kOperandFloats, Bb, Bb + tc::kOperandFloats);
                    tc::commit(&bar);
                    bool ok = mbar_wait_bounded(&bar, products & 1u);
                    if (!ok) ok = mbar_wait_bounded(&bar, products & 1u);  // drain before going on
                    tc_ok = ok ? 1 : 0;
                    if (!ok) {
                        dead = 1;
                        P.ok[cur.p] = 0;
                    }
                }
                ++products;
                __syncthreads();
                tc::fence_after_sync();
                have = tc_ok != 0;
                if (have) {
                    float v[32];
                    tc::tmem_ld32(tc::tmem_addr(tmem, warp, 32 * (warp >> 2)), v);
                    // lanes l and l + 16 share row l's 32 columns: l keeps 0..15, l + 16 takes 16..31
#pragma unroll
                    for (int q = 0; q < 16; ++q) {
                        const float hi16 = __shfl_sync(0xffffffffu, v[16 + q], lane & 15);
                        res[q] -= (lane < 16) ? v[q] : hi16;
                    }
                    tc::fence_before_sync();
                }
            }
            if (have) {
                // the patch's last round writes its final values: a non-finite one marks the inverse unusable
                const bool last = (K + 1) * kGjBlock >= n;
                bool bad = false;
                if (i < n) {
#pragma unroll
                    for (int q = 0; q < 16; q += 4) {
                        if (j + q + 3 < n) {
                            *reinterpret_cast<float4 *>(Arow + q) = make_float4(res[q], res[q + 1], res[q + 2], res[q + 3]);
                        } else {  // the row's last, partial chunk: nothing beyond column n - 1
#pragma unroll
                            for (int u = 0; u < 4; ++u)
                                if (j + q + u < n) Arow[q + u] = res[q + u];
                        }
                    }
                    if (last)
#pragma unroll
                        for (int q = 0; q < 16; ++q) bad |= (j + q < n) && !isfinite(res[q]);
                }
                if (bad) P.ok[cur.p] = 0;
                if (last && cur.row0 < cur.col0 && i < n) {
                    // final values: also the transposed tile of the lower block triangle (A^-1 is symmetric)
                    float *At = P.A + P.moff[cur.p] + i;
#pragma unroll
                    for (int q = 0; q < 16; ++q)
                        if (j + q < n) At[static_cast<size_t>(j + q) * ld] = res[q];
                }
            } else if (threadIdx.x == 0) {
                P.ok[cur.p] = 0;
            }
            if (cur.diag) {  // the tile is final for round K + 1: invert it now (its writes are the block's own)
                __syncthreads();
                pivot_invert_patch(P, cur.p, K + 1, usm);
            }
        }
        __syncthreads();  // every thread is done with the stage and with next_item
        if (threadIdx.x == 0) next_item = atomicAdd(counter, 1);
        __syncthreads();
        item = next_item;
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, tc::kTmemCols);
}

// out = blockdiag(A_pp^-1) in over the patches (in and out must differ).
// grid = (row chunks of kApplyRows, patches), kApplyThreads threads; the block
// gathers the patch's rows of `in` into shared memory, each warp forms two
// output rows with the lanes striding the (coalesced, 16-byte) matrix rows,
// four loads per row in flight.  A patch without a finite inverse uses the
// block-diagonal preconditioner instead (first row chunk only).
// Dynamic shared memory: max(patch_ld(max_n), 3*nseg) doubles.
// With `masked`, patches of arrays whose GMRES stopped are skipped.
constexpr int kApplyRows = 32, kApplyThreads = 16 * 32;  // two rows per warp
__global__ void __launch_bounds__(kApplyThreads) patch_apply_kernel(SimDev d, PatchDev P, const double *in,
                                                                   double *out, int masked) {
    extern __shared__ __align__(16) double xs[];
    __shared__ double sm32[32];
    const int p = blockIdx.y;
    const int n = P.nf[p] * P.nbf;
    const int r0 = blockIdx.x * kApplyRows;
    if (r0 >= n) return;
    if (masked && !d.active[d.fil_arr[P.fils[P.fil0[p]]]]) return;
    if (!P.ok[p]) {
        if (blockIdx.x != 0) return;
        for (int a = 0; a < P.nf[p]; ++a) {
            const int m = P.fils[P.fil0[p] + a];
            precond_block(d, m, fil_rows(d, m), in, out, xs, sm32);
            __syncthreads();
        }
        return;
    }
    const long long *rows = P.rows + P.roff[p];
    const int ld = patch_ld(n), n4 = ld >> 2;
    for (int c = threadIdx.x; c < ld; c += blockDim.x) xs[c] = c < n ? in[rows[c]] : 0.0;  // padding: zeros
    __syncthreads();
    const float *A = P.A + P.moff[p];
    const double2 *x2 = reinterpret_cast<const double2 *>(xs);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    {
        const int r = r0 + 2 * warp;  // this warp's two rows
        if (r >= n) return;
        const bool two = r + 1 < n;
        const float4 *a0 = reinterpret_cast<const float4 *>(A + static_cast<size_t>(r) * ld);
        const float4 *a1 = a0 + n4;
        double s0 = 0.0, s1 = 0.0;
#pragma unroll 4
        for (int c4 = lane; c4 < n4; c4 += 32) {
            const float4 v0 = __ldg(a0 + c4);
            const float4 v1 = two ? __ldg(a1 + c4) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            const double2 xa = x2[2 * c4], xb = x2[2 * c4 + 1];
            s0 = fma(static_cast<double>(v0.x), xa.x, s0);
            s0 = fma(static_cast<double>(v0.y), xa.y, s0);
            s0 = fma(static_cast<double>(v0.z), xb.x, s0);
            s0 = fma(static_cast<double>(v0.w), xb.y, s0);
            s1 = fma(static_cast<double>(v1.x), xa.x, s1);
            s1 = fma(static_cast<double>(v1.y), xa.y, s1);
            s1 = fma(static_cast<double>(v1.z), xb.x, s1);
            s1 = fma(static_cast<double>(v1.w), xb.y, s1);
        }
        s0 = warp_sum(s0);
        s1 = warp_sum(s1);
        if (lane == 0) {  // the refresh leaves -A_pp^-1
            out[rows[r]] = -s0;
            if (two) out[rows[r + 1]] = -s1;
        }
    }
}

// The preconditioning step of one GMRES iteration with the line patches in a
// single launch (in place of arnoldi_precond_kernel + patch_apply_kernel +
// pack_rows_kernel).  Block (a, p) serves filament a of patch p: it clears the
// loop condition (block (0, 0)), gathers the patch's rows of the new basis
// vector Q_k = src * inv_scale (src = r0 or A z in w, or rhs after a discarded
// guess), stores its own filament's rows of Q_k (and of the copy t that the
// network's features read), forms its filament's rows of z = P^-1 Q_k (the
// refresh leaves -A_pp^-1: each warp two rows, lanes striding the 16-byte
// matrix rows) and packs their forces for the pair kernel.  The filament rows
// of A z are written by the saddle epilogue (epi_fil_rows): other blocks of
// the patch still read w here.  A patch without a finite inverse falls back to
// the block-diagonal preconditioner for the filament.
// Dynamic shared memory: patch_ld(max_n) + max(nbf, 3*nseg) doubles.
constexpr int kArnThreads = 256;
constexpr int kArnParts = 2;  // blocks per filament: the rows of segments [0, ceil(nseg/2)) and the rest
__global__ void __launch_bounds__(kArnThreads, 4) patch_arnoldi_kernel(SimDev d, PatchDev P,
                                                                       cudaGraphConditionalHandle h) {
    extern __shared__ __align__(16) double xs[];
    __shared__ double sm32[32];
    chain_wait();
    const int p = blockIdx.y, a = blockIdx.x / kArnParts, part = blockIdx.x % kArnParts;
    if (p == 0 && blockIdx.x == 0 && threadIdx.x == 0) set_loop(h, d.lc, 0);
    if (a >= P.nf[p]) return;
    const int m = P.fils[P.fil0[p] + a];
    const FilRows fr = fil_rows(d, m);
    if (!d.active[fr.b]) return;  // uniform over the block
    const int k = d.lc->k;
    if (k >= d.arr[fr.b].max_iter) return;  // defensive: the cap was reached
    const GmresCtl &c = d.ctl[fr.b];
    const double sc = c.inv_scale;
    const double *src = (k == 0 && c.zero_guess) ? d.rhs : d.w;
    double *q = d.Q + static_cast<size_t>(k) * d.ldq;
    const int n = P.nf[p] * P.nbf, nbf = P.nbf, r_lo = a * nbf;
    // this block's rows of the filament: whole segments (3 rows each), the rate rows with the second part
    const int split = 3 * ((d.nseg + 1) / 2);
    const int r_beg = part == 0 ? 0 : split, r_end = part == 0 ? split : nbf;
    const long long *rows = P.rows + P.roff[p];
    const int ld = patch_ld(n), n4 = ld >> 2;
    double *zs = xs + ld;
    for (int cc = threadIdx.x; cc < ld; cc += blockDim.x) xs[cc] = cc < n ? src[rows[cc]] * sc : 0.0;
    __syncthreads();
    if (!P.ok[p]) {  // the first part alone: the whole filament through the block-diagonal preconditioner
        if (part != 0) return;
        for (int r = threadIdx.x; r < nbf; r += blockDim.x) q[rows[r_lo + r]] = xs[r_lo + r];
        if (d.learned)
            for (int r = threadIdx.x; r < nbf; r += blockDim.x) d.t[rows[r_lo + r]] = xs[r_lo + r];
        __syncthreads();  // this block's rows of Q_k are in global memory
        precond_block(d, m, fr, q, d.z, zs, sm32);
        __syncthreads();
        for (int kk = threadIdx.x; kk < d.nseg; kk += blockDim.x) {
            const long long r = fr.lam + 3 * kk;
            d.f4[m * d.nseg + kk] = make_float4(static_cast<float>(d.z[r]), static_cast<float>(d.z[r + 1]),
                                                static_cast<float>(d.z[r + 2]), 0.0f);
        }
        return;
    }
    for (int r = r_beg + threadIdx.x; r < r_end; r += blockDim.x) q[rows[r_lo + r]] = xs[r_lo + r];
    if (d.learned)
        for (int r = r_beg + threadIdx.x; r < r_end; r += blockDim.x) d.t[rows[r_lo + r]] = xs[r_lo + r];
    const float *A = P.A + P.moff[p];
    const double2 *x2 = reinterpret_cast<const double2 *>(xs);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int r = r_beg + 2 * warp; r < r_end; r += 2 * (kArnThreads / 32)) {
        const bool two = r + 1 < r_end;
        const float4 *a0 = reinterpret_cast<const float4 *>(A + static_cast<size_t>(r_lo + r) * ld);
        const float4 *a1 = a0 + n4;
        double s0 = 0.0, s1 = 0.0;
#pragma unroll 4
        for (int c4 = lane; c4 < n4; c4 += 32) {
            const float4 v0 = __ldg(a0 + c4);
            const float4 v1 = two ? __ldg(a1 + c4) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            const double2 xa = x2[2 * c4], xb = x2[2 * c4 + 1];
            s0 = fma(static_cast<double>(v0.x), xa.x, s0);
            s0 = fma(static_cast<double>(v0.y), xa.y, s0);
            s0 = fma(static_cast<double>(v0.z), xb.x, s0);
            s0 = fma(static_cast<double>(v0.w), xb.y, s0);
            s1 = fma(static_cast<double>(v1.x), xa.x, s1);
            s1 = fma(static_cast<double>(v1.y), xa.y, s1);
            s1 = fma(static_cast<double>(v1.z), xb.x, s1);
            s1 = fma(static_cast<double>(v1.w), xb.y, s1);
        }
        s0 = warp_sum(s0);
        s1 = warp_sum(s1);
        if (lane == 0) {
            d.z[rows[r_lo + r]] = -s0;
            zs[r] = -s0;
            if (two) {
                d.z[rows[r_lo + r + 1]] = -s1;
                zs[r + 1] = -s1;
            }
        }
    }
    __syncthreads();
    const int kk_end = min(d.nseg, r_end / 3);
    for (int kk = r_beg / 3 + threadIdx.x; kk < kk_end; kk += blockDim.x)
        d.f4[m * d.nseg + kk] = make_float4(static_cast<float>(zs[3 * kk]), static_cast<float>(zs[3 * kk + 1]),
                                            static_cast<float>(zs[3 * kk + 2]), 0.0f);
}

// After a patch application: packs the force rows of z for the pair kernel
// and writes the filament rows of A z (one block per filament), the work that
// arnoldi_precond_kernel does itself with the block-diagonal preconditioner.
__global__ void pack_rows_kernel(SimDev d, const double *z, double *w) {
    __shared__ double sm32[32];
    const int m = blockIdx.x;
    const FilRows fr = fil_rows(d, m);
    if (!d.active[fr.b]) return;
    for (int kk = threadIdx.x; kk < d.nseg; kk += blockDim.x) {
        const long long r = fr.lam + 3 * kk;
        d.f4[m * d.nseg + kk] = make_float4(static_cast<float>(z[r]), static_cast<float>(z[r + 1]),
                                            static_cast<float>(z[r + 2]), 0.0f);
    }
    filament_rows(d, fr, z, w, sm32);
}

}  // namespace cufil

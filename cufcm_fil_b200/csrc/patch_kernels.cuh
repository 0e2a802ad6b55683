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

namespace cufil {

constexpr int kGjBlock = 64;  // pivot block of the Gauss-Jordan rounds
constexpr int kGjTile = 64;   // tile of the rank-64 updates

struct PatchDev {
    int np;                  // patches
    int nbf;                 // unknowns per filament (3*nseg + rate rows)
    int max_n;               // largest patch system
    const int *fil0;         // first entry of each patch in `fils` [np]
    const int *nf;           // filaments per patch [np]
    const int *fils;         // filament ids (batch numbering), patch by patch
    const long long *moff;   // first float of each patch matrix [np]
    const long long *roff;   // first entry of each patch in `rows` [np]
    const long long *rows;   // batch-vector row of each local unknown
    float *A;                // patch matrices, then their inverses (row-major n x n)
    float *cbuf;             // pivot-column copies, [np][max_n][kGjBlock]
    float *rbuf;             // scaled pivot rows, [np][kGjBlock][max_n]
    float *dinv;             // inverted pivot blocks, [np][kGjBlock][kGjBlock]
    int *ok;                 // [np] 1 when the inverse is finite
};

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
    const int n = nfp * P.nbf;
    float *A = P.A + P.moff[p];
    const long long r0 = static_cast<long long>(ai) * P.nbf + 3 * ki;
    const long long c0 = static_cast<long long>(aj) * P.nbf + 3 * kj;
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
        for (int q = 0; q < 3; ++q) A[(r0 + q) * n + c0 + c] = v[q];
    }
}

// Rate entries -K / -K^T of each filament of a patch (one block per patch).
__global__ void patch_rates_kernel(SimDev d, PatchDev P) {
    const int p = blockIdx.x;
    const int nfp = P.nf[p];
    const int n = nfp * P.nbf;
    const int nl = 3 * d.nseg;
    float *A = P.A + P.moff[p];
    for (int e = threadIdx.x; e < nfp * nl; e += blockDim.x) {
        const int a = e / nl, li = e - a * nl;
        const int g3 = 3 * P.fils[P.fil0[p] + a] * d.nseg + li;  // entry of kp / ka
        const long long r = static_cast<long long>(a) * P.nbf + li;
        long long c = static_cast<long long>(a) * P.nbf + nl;
        if (d.dyn_phase) {
            const float v = -static_cast<float>(d.kp[g3]);
            A[r * n + c] = v;
            A[c * n + r] = v;
            ++c;
        }
        if (d.dyn_angle) {
            const float v = -static_cast<float>(d.ka[g3]);
            A[r * n + c] = v;
            A[c * n + r] = v;
        }
    }
}

// Part (a) of a round: inverts pivot block K of patch p (rows and columns [64K, 64K + b)) in
// place of dinv; called by all 256 threads of a block.  Each thread keeps 16
// entries of the 64x64 block in registers (row tid/4, columns tid%4 + 4q); per
// elimination step the pivot row is published through a double-buffered
// shared row (one barrier per step) and each row's pivot-column entry comes
// from a shuffle among the row's 4 threads.  A non-finite or zero pivot clears
// the patch's ok flag.
// A: the patch matrix (n x n), dv: its dinv block, ok: its flag.
__device__ __noinline__ void pivot_invert(const float *A, int n, float *dv, int *ok, int K, float (*rowbuf)[kGjBlock]) {
    static_assert(kGjBlock * 4 == 256, "one row per 4 threads");
    constexpr int Q = kGjBlock / 4;
    const int k0 = K * kGjBlock;
    const int b = min(kGjBlock, n - k0);
    const int r = threadIdx.x >> 2, cq = threadIdx.x & 3;
    const int lane = threadIdx.x & 31;
    if (K == 0 && threadIdx.x == 0) *ok = 1;
    float reg[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int c = cq + 4 * q;
        reg[q] = (r < b && c < b) ? A[static_cast<size_t>(k0 + r) * n + k0 + c] : 0.0f;
    }
    for (int t = 0; t < b; ++t) {
        float own = 0.0f;
#pragma unroll
        for (int q = 0; q < Q; ++q)
            if (q == (t >> 2)) own = reg[q];
        const float colr = __shfl_sync(0xffffffffu, own, (lane & ~3) | (t & 3));
        float *rb = rowbuf[t & 1];
        if (r == t) {  // scale the pivot row and publish it
            const float ip = 1.0f / colr;  // colr is the pivot here
            if (cq == (t & 3) && (!(fabsf(colr) > 0.0f) || !isfinite(colr))) *ok = 0;
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const int c = cq + 4 * q;
                reg[q] = (c == t) ? ip : reg[q] * ip;
                rb[c] = reg[q];
            }
        }
        __syncthreads();
        if (r != t && r < b) {  // eliminate column t from the other rows
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const int c = cq + 4 * q;
                reg[q] = ((c == t) ? 0.0f : reg[q]) - colr * rb[c];
            }
        }
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) dv[r * kGjBlock + cq + 4 * q] = (r < b) ? reg[q] : 0.0f;
}

__device__ __forceinline__ void pivot_invert_patch(const PatchDev &P, int p, int K, float (*rowbuf)[kGjBlock]) {
    pivot_invert(P.A + P.moff[p], P.nf[p] * P.nbf, P.dinv + static_cast<size_t>(p) * kGjBlock * kGjBlock, P.ok + p, K,
                 rowbuf);
}

// Round 0, part (a): the first pivot block of every patch (later pivot blocks
// are inverted by the previous round's update, see gj_update_kernel).
__global__ void __launch_bounds__(256) gj_pivot_kernel(PatchDev P, int K) {
    __shared__ float rowbuf[2][kGjBlock];
    const int p = blockIdx.x;
    const int n = P.nf[p] * P.nbf;
    if (K * kGjBlock >= n) return;
    pivot_invert_patch(P, p, K, rowbuf);
}

// Round K, part (b), one 64-column tile [j0, j0 + 64) of a patch per block.
// The matrix is kept symmetric and only its upper block triangle is
// maintained, so the pivot rows' entries are
//   U[s][j] = A[k0 + s][j] for j >= k0,   A[j][k0 + s] for j < k0  (by symmetry);
// both are read as 64 contiguous floats per row of A and staged in shared
// memory as U[s][c].  The pass writes
//   rbuf[s][j] = (D^-1 U)[s][j] outside the pivot columns, -D^-1[s][j - k0] inside,
//   cbuf[j][s] = U[s][j]         for j outside the pivot rows (zero inside).
// Tiles and pivot blocks are both 64 wide, so a tile is either the pivot
// block's or disjoint from it.  Each thread owns 4 rows x 4 columns of
// D^-1 U (rows ty + 16u, columns tx + 16v).  grid = (tiles, patches).
__global__ void __launch_bounds__(256) gj_prep_kernel(PatchDev P, int K) {
    static_assert(kGjTile == kGjBlock, "column tiles are pivot-block wide");
    __shared__ float Dv[kGjBlock][kGjBlock + 1];
    __shared__ float Us[kGjBlock][kGjTile + 1];
    const int p = blockIdx.y;
    const int n = P.nf[p] * P.nbf;
    const int k0 = K * kGjBlock;
    const int j0 = blockIdx.x * kGjTile;
    if (k0 >= n || j0 >= n) return;
    const int b = min(kGjBlock, n - k0);
    const int w = min(kGjTile, n - j0);  // columns in this tile
    const float *A = P.A + P.moff[p];
    float *rb = P.rbuf + static_cast<size_t>(p) * kGjBlock * P.max_n;
    float *cb = P.cbuf + static_cast<size_t>(p) * P.max_n * kGjBlock;
    const float *dv = P.dinv + static_cast<size_t>(p) * kGjBlock * kGjBlock;
    if (j0 == k0) {  // the pivot columns: -D^-1, and no pivot-row copies
        for (int e = threadIdx.x; e < kGjBlock * kGjTile; e += blockDim.x) {
            const int r = e / kGjTile, c = e - r * kGjTile;
            if (c < w) rb[static_cast<size_t>(r) * n + j0 + c] = -dv[r * kGjBlock + c];  // zero-padded rows
        }
        for (int e = threadIdx.x; e < w * kGjBlock; e += blockDim.x) cb[static_cast<size_t>(j0) * kGjBlock + e] = 0.0f;
        return;
    }
    for (int e = threadIdx.x; e < kGjBlock * kGjBlock; e += blockDim.x) Dv[e / kGjBlock][e % kGjBlock] = dv[e];
    if (j0 > k0) {  // U[s][c] = A[k0 + s][j0 + c]
        for (int e = threadIdx.x; e < kGjBlock * kGjTile; e += blockDim.x) {
            const int s_ = e / kGjTile, c = e - s_ * kGjTile;
            Us[s_][c] = (s_ < b && c < w) ? A[static_cast<size_t>(k0 + s_) * n + j0 + c] : 0.0f;
        }
    } else {  // j0 + 64 <= k0: U[s][c] = A[j0 + c][k0 + s], rows of A read contiguously
        for (int e = threadIdx.x; e < kGjTile * kGjBlock; e += blockDim.x) {
            const int c = e / kGjBlock, s_ = e - c * kGjBlock;
            Us[s_][c] = (s_ < b) ? A[static_cast<size_t>(j0 + c) * n + k0 + s_] : 0.0f;
        }
    }
    __syncthreads();
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    float acc[4][4] = {};
#pragma unroll 8
    for (int s_ = 0; s_ < kGjBlock; ++s_) {
        float dr[4], uc[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) dr[u] = Dv[ty + 16 * u][s_];
#pragma unroll
        for (int v = 0; v < 4; ++v) uc[v] = Us[s_][tx + 16 * v];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[u][v] = fmaf(dr[u], uc[v], acc[u][v]);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int c = tx + 16 * v;
            if (c < w) rb[static_cast<size_t>(ty + 16 * u) * n + j0 + c] = acc[u][v];  // rows >= b: zeros
        }
    // the pivot-row entries of the tile's columns, transposed: rows j0 .. j0 + w of cbuf
    for (int e = threadIdx.x; e < w * kGjBlock; e += blockDim.x) {
        const int c = e / kGjBlock, s_ = e - c * kGjBlock;
        cb[static_cast<size_t>(j0 + c) * kGjBlock + s_] = Us[s_][c];
    }
}

// Round K, part (c), the 64x64 tiles of the upper block triangle:
//   pivot rows       A[i, j] = rbuf[i - k0][j]      (-D^-1 in the pivot block)
//   other rows       A[i, j] -= C_i . rbuf[:, j]   (j outside the pivot columns)
//                    A[i, j]  = -C_i . rbuf[:, j]  (pivot columns: C_i D^-1)
// with C_i = cbuf[i][:] -- the symmetric sweep, which leaves -A^-1 after the
// last round.  Each thread owns 4 rows x 4 columns of the tile
// (columns interleaved by 16, so every load and store of a half-warp is one
// contiguous run) and loads each of its rows of A in one batch.
// grid = (patches, tiles): patches run fastest, so every patch's first block
// (the diagonal tile below) is issued in the first wave.
__global__ void __launch_bounds__(256, 4) gj_update_kernel(PatchDev P, int K) {
    __shared__ float Cs[kGjTile][kGjBlock + 1];
    __shared__ float Rs[kGjBlock][kGjTile + 1];
    const int p = blockIdx.x;
    const int n = P.nf[p] * P.nbf;
    const int k0 = K * kGjBlock;
    if (k0 >= n) return;
    const int b = min(kGjBlock, n - k0);
    const int T = (n + kGjTile - 1) / kGjTile;
    const int bid = blockIdx.y;
    if (bid >= T * T) return;
    // Block 0 takes the next round's diagonal tile, so that it starts first and, after its update,
    // inverts that pivot block for the next round while the other blocks finish theirs.
    const int diag = (K + 1 < T) ? (K + 1) * T + (K + 1) : -1;
    int tile = bid;
    if (diag >= 0) tile = (bid == 0) ? diag : (bid <= diag ? bid - 1 : bid);
    const int ti = tile / T, tj = tile - ti * T;
    if (ti > tj) return;  // the lower block triangle is filled in once, after the last round
    const int row0 = ti * kGjTile, col0 = tj * kGjTile;
    float *__restrict__ A = P.A + P.moff[p];
    const float *__restrict__ cb = P.cbuf + static_cast<size_t>(p) * P.max_n * kGjBlock;
    const float *__restrict__ rb = P.rbuf + static_cast<size_t>(p) * kGjBlock * P.max_n;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    for (int e = threadIdx.x; e < kGjTile * kGjBlock; e += blockDim.x) {
        const int r = e / kGjBlock, s = e - r * kGjBlock;
        const int i = row0 + r;
        Cs[r][s] = (i < n) ? cb[static_cast<size_t>(i) * kGjBlock + s] : 0.0f;
    }
    for (int e = threadIdx.x; e < kGjBlock * kGjTile; e += blockDim.x) {
        const int s = e / kGjTile, c = e - s * kGjTile;
        const int j = col0 + c;
        Rs[s][c] = (j < n) ? rb[static_cast<size_t>(s) * n + j] : 0.0f;
    }
    __syncthreads();
    float acc[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = 0.0f;
#pragma unroll 8
    for (int s = 0; s < kGjBlock; ++s) {
        float cr[4], rr[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) cr[u] = Cs[ty * 4 + u][s];
#pragma unroll
        for (int v = 0; v < 4; ++v) rr[v] = Rs[s][v * 16 + tx];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[u][v] += cr[u] * rr[v];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int i = row0 + ty * 4 + u;
        if (i >= n) continue;
        const bool pivot_row = i >= k0 && i < k0 + b;
        float *__restrict__ ar = A + static_cast<size_t>(i) * n;
        float old[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int j = col0 + v * 16 + tx;
            old[v] = (!pivot_row && j < n) ? ar[j] : 0.0f;
        }
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int j = col0 + v * 16 + tx;
            if (j >= n) continue;
            ar[j] = pivot_row ? Rs[i - k0][v * 16 + tx]
                              : ((j >= k0 && j < k0 + b) ? -acc[u][v] : old[v] - acc[u][v]);
        }
    }
    if (tile == diag) {  // the tile is final for round K + 1: invert it now (its writes are the block's own)
        __shared__ float rowbuf[2][kGjBlock];
        __syncthreads();
        pivot_invert_patch(P, p, K + 1, rowbuf);
    }
}

// After the last round: fills the lower block triangle from the upper one
// (tile (ti, tj), ti > tj, from the transpose of tile (tj, ti)); the matrix is
// then -A_pp^-1 in full.  grid = (tiles, patches).
__global__ void __launch_bounds__(256) gj_mirror_kernel(PatchDev P) {
    __shared__ float tile[kGjTile][kGjTile + 1];
    const int p = blockIdx.y;
    const int n = P.nf[p] * P.nbf;
    const int T = (n + kGjTile - 1) / kGjTile;
    if (static_cast<int>(blockIdx.x) >= T * T) return;
    const int ti = blockIdx.x / T, tj = blockIdx.x - ti * T;
    if (ti <= tj) return;
    float *A = P.A + P.moff[p];
    const int r0 = tj * kGjTile, c0 = ti * kGjTile;  // the source tile, upper triangle
    for (int e = threadIdx.x; e < kGjTile * kGjTile; e += blockDim.x) {
        const int r = e / kGjTile, c = e - r * kGjTile;
        tile[r][c] = (r0 + r < n && c0 + c < n) ? A[static_cast<size_t>(r0 + r) * n + c0 + c] : 0.0f;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kGjTile * kGjTile; e += blockDim.x) {
        const int r = e / kGjTile, c = e - r * kGjTile;  // destination (c0 + r, r0 + c)
        if (c0 + r < n && r0 + c < n) A[static_cast<size_t>(c0 + r) * n + r0 + c] = tile[c][r];
    }
}

// Clears a patch's ok flag if its inverse holds a non-finite entry.
__global__ void patch_check_kernel(PatchDev P) {
    const int p = blockIdx.y;
    const int n = P.nf[p] * P.nbf;
    const long long nn = static_cast<long long>(n) * n;
    const float *A = P.A + P.moff[p];
    bool bad = false;
    for (long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; e < nn;
         e += static_cast<long long>(gridDim.x) * blockDim.x)
        bad |= !isfinite(A[e]);
    if (__syncthreads_or(bad) && threadIdx.x == 0) P.ok[p] = 0;
}

// out = blockdiag(A_pp^-1) in over the patches (in and out must differ).
// grid = (row chunks of 64, patches); the block gathers the patch's rows of
// `in` into shared memory, each warp forms 8 output rows with the lanes
// striding the (coalesced) matrix row.  A patch without a finite inverse uses
// the block-diagonal preconditioner instead (first row chunk only).
// Dynamic shared memory: max(max_n, 3*nseg) doubles.
// With `masked`, patches of arrays whose GMRES stopped are skipped.
__global__ void __launch_bounds__(256) patch_apply_kernel(SimDev d, PatchDev P, const double *in, double *out,
                                                          int masked) {
    extern __shared__ double xs[];
    __shared__ double sm32[32];
    const int p = blockIdx.y;
    const int n = P.nf[p] * P.nbf;
    const int r0 = blockIdx.x * 64;
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
    for (int c = threadIdx.x; c < n; c += blockDim.x) xs[c] = in[rows[c]];
    __syncthreads();
    const float *A = P.A + P.moff[p];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int rr = 0; rr < 8; ++rr) {
        const int r = r0 + warp * 8 + rr;
        if (r >= n) break;
        const float *ar = A + static_cast<size_t>(r) * n;
        double acc = 0.0;
        for (int c = lane; c < n; c += 32) acc += static_cast<double>(__ldg(ar + c)) * xs[c];
        acc = warp_sum(acc);
        if (lane == 0) out[rows[r]] = -acc;  // the refresh leaves -A_pp^-1
    }
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

// mlp.cu -- cf_mlp: a small fully connected network (in -> H -> H -> out, ReLU)
// with its own forward, backward and Adam kernels, used as a learned
// per-filament correction inside flexible GMRES (CF_PRECOND_LEARNED).
// No counterpart in the reference.
//
// Every product is one GEMM kernel: C[M x N] = op(A)[M x K] op(B)[K x N] with
// FP32 operands in memory, rounded to BF16 while they are staged in shared
// memory in the canonical K-major layout, multiplied on the 5th-generation
// tensor cores (tcgen05.mma kind::f16, BF16 x BF16, FP32 accumulation in
// tensor memory, 128 x 32 tiles, K in chunks of 64), and an FP32 epilogue
// (bias, ReLU, or the ReLU mask of the backward pass) after tcgen05.ld.  Forward:  A1 = relu(X W1 + b1), A2 = relu(A1 W2 + b2),
// Y = A2 W3 + b3.  Backward of the mean squared error:
//   dY = 2 (Y - T) / (n out)      dW3 = A2^T dY    db3 = colsum dY
//   dZ2 = (dY W3^T) o [A2 > 0]    dW2 = A1^T dZ2   db2 = colsum dZ2
//   dZ1 = (dZ2 W2^T) o [A1 > 0]   dW1 = X^T dZ1    db1 = colsum dZ1
// then one Adam step on FP32 master weights.  Reductions (loss, bias
// gradients) are fixed-order: results do not depend on the launch.
#include "common.cuh"
#include "tc_tf32.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <random>
#include <string>
#include <vector>

namespace cufil {
namespace {

constexpr int kTcM = 128, kTcN = 32, kTcK = 64;  // C tile and K chunk
constexpr int kTcA = kTcM * kTcK, kTcB = kTcN * kTcK;  // BF16 elements of the staged operands
// 20 KB of operands, requested as 32 KB so that at most 7 blocks share an SM: their 7 x 64 allocated
// accumulator columns stay within the 512 of tensor memory, so no allocation ever waits for another block.
constexpr size_t kTcSmem = 32 * 1024;
static_assert(sizeof(__nv_bfloat16) * (kTcA + kTcB) <= kTcSmem, "operands fit the request");

enum Epi : int { kEpiStore = 0, kEpiBias = 1, kEpiBiasRelu = 2, kEpiReluMask = 3 };

struct GemmArgs {
    const float *A, *B;
    float *C;
    const float *bias;  // [N] (kEpiBias, kEpiBiasRelu)
    const float *mask;  // [M x N], ldc (kEpiReluMask): keep where mask > 0
    int lda, ldb, ldc;
    int M, N, K;
    int ta, tb, epi;
};

// One 128 x 32 tile of C per block of 4 warps.  Per K chunk of 64 the block stages op(A) [128 x 64] and
// op(B)^T [32 x 64] as BF16 in the canonical layout (consecutive threads read consecutive addresses of the
// operand as it lies in memory), one thread issues four tcgen05.mma (K = 16 each) and commits them to an
// mbarrier (bounded wait), and the next chunk is staged once they are done.  Row m of the accumulator lives
// in TMEM lane m: warp w reads rows 32 w + lane, 32 columns.  A wait that gives up fills the tile with quiet
// NaNs (the caller's residual then reports a non-finite value).
__global__ void __launch_bounds__(128) gemm_bf16_kernel(GemmArgs g) {
    extern __shared__ __align__(128) __nv_bfloat16 tsm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tbase;
    __shared__ int ok_all;
    __nv_bfloat16 *As = tsm, *Bs = tsm + kTcA;
    const int m0 = blockIdx.y * kTcM, n0 = blockIdx.x * kTcN;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) tc::tmem_alloc(&tbase, tc::kTmemCols);
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
        ok_all = 1;
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tbase;
    uint32_t phase = 0;
    for (int k0 = 0; k0 < g.K; k0 += kTcK) {
        // eight independent loads in flight per thread, then the conversions and stores
        for (int e0 = threadIdx.x; e0 < kTcA; e0 += 8 * blockDim.x) {  // op(A)(m, k): A[m lda + k] or A[k lda + m]
            float v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int e = e0 + u * blockDim.x;
                int m, k;
                if (g.ta) { k = e / kTcM; m = e - k * kTcM; } else { m = e / kTcK; k = e - m * kTcK; }
                const int gm = m0 + m, gk = k0 + k;
                v[u] = (gm < g.M && gk < g.K) ? (g.ta ? g.A[static_cast<size_t>(gk) * g.lda + gm] : g.A[static_cast<size_t>(gm) * g.lda + gk]) : 0.0f;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int e = e0 + u * blockDim.x;
                int m, k;
                if (g.ta) { k = e / kTcM; m = e - k * kTcM; } else { m = e / kTcK; k = e - m * kTcK; }
                As[tc::canon16(m, k)] = __float2bfloat16_rn(v[u]);
            }
        }
        for (int e0 = threadIdx.x; e0 < kTcB; e0 += 8 * blockDim.x) {  // op(B)(k, n): B[k ldb + n] or B[n ldb + k]
            float v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int e = e0 + u * blockDim.x;
                int n, k;
                if (g.tb) { n = e / kTcK; k = e - n * kTcK; } else { k = e / kTcN; n = e - k * kTcN; }
                const int gn = n0 + n, gk = k0 + k;
                v[u] = (gn < g.N && gk < g.K) ? (g.tb ? g.B[static_cast<size_t>(gn) * g.ldb + gk] : g.B[static_cast<size_t>(gk) * g.ldb + gn]) : 0.0f;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int e = e0 + u * blockDim.x;
                int n, k;
                if (g.tb) { n = e / kTcK; k = e - n * kTcK; } else { k = e / kTcN; n = e - k * kTcN; }
                Bs[tc::canon16(n, k)] = __float2bfloat16_rn(v[u]);
            }
        }
        tc::fence_proxy_async();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (threadIdx.x == 0 && ok_all) {
            const uint64_t da = tc::smem_desc16(As), db = tc::smem_desc16(Bs);
#pragma unroll
            for (int s = 0; s < kTcK / 16; ++s)
                tc::mma_bf16(tmem, da + s * (256 >> 4), db + s * (256 >> 4), (k0 > 0 || s > 0) ? 1u : 0u);
            tc::commit(&bar);
            bool ok = mbar_wait_bounded(&bar, phase & 1u);
            if (!ok) ok = mbar_wait_bounded(&bar, phase & 1u);  // drain before the operands are restaged
            if (!ok) ok_all = 0;
        }
        ++phase;
        tc::fence_before_sync();
        __syncthreads();  // the products are done with the staged operands
        tc::fence_after_sync();
    }
    const int row = m0 + 32 * warp + lane;
    if (ok_all) {
        float v[32];
        tc::tmem_ld32(tc::tmem_addr(tmem, warp, 0), v);
        if (row < g.M) {
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                const int col = n0 + j;
                if (col >= g.N) continue;
                float x = v[j];
                const size_t o = static_cast<size_t>(row) * g.ldc + col;
                if (g.epi == kEpiBias || g.epi == kEpiBiasRelu) x += g.bias[col];
                if (g.epi == kEpiBiasRelu) x = fmaxf(x, 0.0f);
                if (g.epi == kEpiReluMask && !(g.mask[o] > 0.0f)) x = 0.0f;
                g.C[o] = x;
            }
        }
    } else if (row < g.M) {
        for (int j = 0; j < kTcN && n0 + j < g.N; ++j) g.C[static_cast<size_t>(row) * g.ldc + n0 + j] = __int_as_float(0x7fc00000);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, tc::kTmemCols);
}

// dY = 2 (Y - T) / (n * out) and per-block partial sums of (Y - T)^2.
__global__ void __launch_bounds__(256) mse_kernel(const float *Y, const float *T, float *dY, long long count,
                                                  float scale, double *partial) {
    __shared__ double sm[8];
    double s = 0.0;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const float d = Y[i] - T[i];
        dY[i] = 2.0f * d * scale;
        s += static_cast<double>(d) * d;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += sm[w];
        partial[blockIdx.x] = t;
    }
}

// db[j] = sum_i dZ[i][j], rows summed in order by one thread per column.
__global__ void colsum_kernel(const float *dZ, int n, int cols, float *db) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= cols) return;
    float s = 0.0f;
    for (int i = 0; i < n; ++i) s += dZ[static_cast<size_t>(i) * cols + j];
    db[j] = s;
}

__global__ void adam_kernel(float *p, const float *gr, float *m, float *v, long long count, float lr, float b1,
                            float b2, float c1, float c2, float eps) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const float gi = gr[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

}  // namespace

int gemm_bf16(const float *A, int lda, int ta, const float *B, int ldb, int tb, float *C, int ldc, int M, int N, int K,
              const float *bias, const float *mask, int epi, cudaStream_t st) {
    if (M <= 0 || N <= 0) return CF_OK;
    if (K <= 0) return set_error(CF_EINVAL, "gemm_bf16: empty inner dimension");
    GemmArgs g{A, B, C, bias, mask, lda, ldb, ldc, M, N, K, ta, tb, epi};
    dim3 grid((N + kTcN - 1) / kTcN, (M + kTcM - 1) / kTcM);
    gemm_bf16_kernel<<<grid, 128, kTcSmem, st>>>(g);
    CF_CHECK_LAUNCH("gemm_bf16_kernel");
    return CF_OK;
}

}  // namespace cufil

using namespace cufil;

struct cf_mlp {
    int in = 0, hid = 0, out = 0, max_batch = 0, device = 0;
    long long nparam = 0;
    float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    float *W1, *b1, *W2, *b2, *W3, *b3;      // views into params
    float *gW1, *gb1, *gW2, *gb2, *gW3, *gb3; // views into grads
    float *A1 = nullptr, *A2 = nullptr, *Y = nullptr, *dY = nullptr, *dZ2 = nullptr, *dZ1 = nullptr;
    double *partial = nullptr;
    int loss_blocks = 256;
    long long step = 0;
    cudaStream_t stream = nullptr;
    std::vector<void *> allocations;
};

namespace {

template <typename T>
int mlp_alloc(cf_mlp *h, T **p, size_t n) {
    void *q = nullptr;
    CF_CUDA(cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)));
    h->allocations.push_back(q);
    *p = static_cast<T *>(q);
    return CF_OK;
}

void set_views(cf_mlp *h) {
    const long long in = h->in, hd = h->hid, out = h->out;
    float *p = h->params, *g = h->grads;
    const long long off[6] = {0, in * hd, in * hd + hd, in * hd + hd + hd * hd, in * hd + 2 * hd + hd * hd,
                              in * hd + 2 * hd + hd * hd + hd * out};
    h->W1 = p + off[0]; h->b1 = p + off[1]; h->W2 = p + off[2]; h->b2 = p + off[3]; h->W3 = p + off[4]; h->b3 = p + off[5];
    h->gW1 = g + off[0]; h->gb1 = g + off[1]; h->gW2 = g + off[2]; h->gb2 = g + off[3]; h->gW3 = g + off[4];
    h->gb3 = g + off[5];
}

int forward(cf_mlp *h, const float *x, int n, float *y, cudaStream_t st) {
    CF_TRY(gemm_bf16(x, h->in, 0, h->W1, h->hid, 0, h->A1, h->hid, n, h->hid, h->in, h->b1, nullptr, kEpiBiasRelu, st));
    CF_TRY(gemm_bf16(h->A1, h->hid, 0, h->W2, h->hid, 0, h->A2, h->hid, n, h->hid, h->hid, h->b2, nullptr,
                     kEpiBiasRelu, st));
    return gemm_bf16(h->A2, h->hid, 0, h->W3, h->out, 0, y, h->out, n, h->out, h->hid, h->b3, nullptr, kEpiBias, st);
}

// Forward + backward into h->grads; the loss (mean squared error) into *loss when asked (synchronises).
int backward(cf_mlp *h, const float *x, const float *t, int n, double *loss) {
    cudaStream_t st = h->stream;
    CF_TRY(forward(h, x, n, h->Y, st));
    const long long cnt = static_cast<long long>(n) * h->out;
    mse_kernel<<<h->loss_blocks, 256, 0, st>>>(h->Y, t, h->dY, cnt, 1.0f / static_cast<float>(cnt), h->partial);
    CF_CHECK_LAUNCH("mse_kernel");
    // layer 3
    CF_TRY(gemm_bf16(h->A2, h->hid, 1, h->dY, h->out, 0, h->gW3, h->out, h->hid, h->out, n, nullptr, nullptr,
                     kEpiStore, st));
    colsum_kernel<<<(h->out + 127) / 128, 128, 0, st>>>(h->dY, n, h->out, h->gb3);
    CF_CHECK_LAUNCH("colsum_kernel");
    CF_TRY(gemm_bf16(h->dY, h->out, 0, h->W3, h->out, 1, h->dZ2, h->hid, n, h->hid, h->out, nullptr, h->A2,
                     kEpiReluMask, st));
    // layer 2
    CF_TRY(gemm_bf16(h->A1, h->hid, 1, h->dZ2, h->hid, 0, h->gW2, h->hid, h->hid, h->hid, n, nullptr, nullptr,
                     kEpiStore, st));
    colsum_kernel<<<(h->hid + 127) / 128, 128, 0, st>>>(h->dZ2, n, h->hid, h->gb2);
    CF_CHECK_LAUNCH("colsum_kernel");
    CF_TRY(gemm_bf16(h->dZ2, h->hid, 0, h->W2, h->hid, 1, h->dZ1, h->hid, n, h->hid, h->hid, nullptr, h->A1,
                     kEpiReluMask, st));
    // layer 1
    CF_TRY(gemm_bf16(x, h->in, 1, h->dZ1, h->hid, 0, h->gW1, h->hid, h->in, h->hid, n, nullptr, nullptr, kEpiStore,
                     st));
    colsum_kernel<<<(h->hid + 127) / 128, 128, 0, st>>>(h->dZ1, n, h->hid, h->gb1);
    CF_CHECK_LAUNCH("colsum_kernel");
    if (loss) {
        std::vector<double> part(h->loss_blocks);
        CF_CUDA(cudaMemcpyAsync(part.data(), h->partial, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, st));
        CF_CUDA(cudaStreamSynchronize(st));
        double s = 0.0;
        for (double v : part) s += v;
        *loss = s / static_cast<double>(cnt);
    }
    return CF_OK;
}

}  // namespace

namespace cufil {
// Forward pass on a caller's stream for the implicit step (checked sizes).
int mlp_forward_dev(cf_mlp *h, const float *x, int n, float *y, cudaStream_t st) {
    if (n > h->max_batch) return set_error(CF_EINVAL, "network batch %d above its capacity %d", n, h->max_batch);
    return forward(h, x, n, y, st);
}
int mlp_dims(const cf_mlp *h, int *in, int *out, int *max_batch) {
    *in = h->in;
    *out = h->out;
    *max_batch = h->max_batch;
    return CF_OK;
}
}  // namespace cufil

extern "C" int cf_mlp_create(int in_dim, int hidden, int out_dim, int max_batch, unsigned long long seed, int device,
                             cf_mlp **out) {
    clear_error();
    CF_REQUIRE(out, "cf_mlp_create: null handle pointer");
    *out = nullptr;
    CF_REQUIRE(in_dim > 0 && hidden > 0 && out_dim > 0 && max_batch > 0 && in_dim <= 4096 && hidden <= 4096 &&
                   out_dim <= 4096,
               "cf_mlp_create: bad sizes (%d, %d, %d, batch %d)", in_dim, hidden, out_dim, max_batch);
    CF_CUDA(cudaSetDevice(device));
    cf_mlp *h = new (std::nothrow) cf_mlp();
    if (!h) return set_error(CF_ENOMEM, "cf_mlp_create: host allocation failed");
    h->in = in_dim;
    h->hid = hidden;
    h->out = out_dim;
    h->max_batch = max_batch;
    h->device = device;
    h->nparam = static_cast<long long>(in_dim) * hidden + hidden + static_cast<long long>(hidden) * hidden + hidden +
                static_cast<long long>(hidden) * out_dim + out_dim;
    int rc = CF_OK;
    do {
        if ((rc = cuda_status(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate",
                              __FILE__, __LINE__)))
            break;
        const size_t np = h->nparam, act = static_cast<size_t>(max_batch) * hidden;
        if ((rc = mlp_alloc(h, &h->params, np)) || (rc = mlp_alloc(h, &h->grads, np)) ||
            (rc = mlp_alloc(h, &h->adam_m, np)) || (rc = mlp_alloc(h, &h->adam_v, np)) ||
            (rc = mlp_alloc(h, &h->A1, act)) || (rc = mlp_alloc(h, &h->A2, act)) || (rc = mlp_alloc(h, &h->dZ1, act)) ||
            (rc = mlp_alloc(h, &h->dZ2, act)) || (rc = mlp_alloc(h, &h->Y, static_cast<size_t>(max_batch) * out_dim)) ||
            (rc = mlp_alloc(h, &h->dY, static_cast<size_t>(max_batch) * out_dim)) ||
            (rc = mlp_alloc(h, &h->partial, h->loss_blocks)))
            break;
        set_views(h);
        // He-uniform weights from the seed, zero biases
        std::vector<float> p(np, 0.0f);
        std::mt19937_64 rng(seed);
        auto fill = [&](long long off, int fan_in, long long count) {
            std::uniform_real_distribution<float> u(-std::sqrt(6.0f / fan_in), std::sqrt(6.0f / fan_in));
            for (long long i = 0; i < count; ++i) p[off + i] = u(rng);
        };
        fill(h->W1 - h->params, in_dim, static_cast<long long>(in_dim) * hidden);
        fill(h->W2 - h->params, hidden, static_cast<long long>(hidden) * hidden);
        fill(h->W3 - h->params, hidden, static_cast<long long>(hidden) * out_dim);
        if ((rc = cuda_status(cudaMemcpy(h->params, p.data(), np * sizeof(float), cudaMemcpyHostToDevice),
                              "cudaMemcpy", __FILE__, __LINE__)) ||
            (rc = cuda_status(cudaMemset(h->adam_m, 0, np * sizeof(float)), "cudaMemset", __FILE__, __LINE__)) ||
            (rc = cuda_status(cudaMemset(h->adam_v, 0, np * sizeof(float)), "cudaMemset", __FILE__, __LINE__)))
            break;
    } while (0);
    if (rc != CF_OK) {
        std::string msg = cf_last_error();
        for (void *q : h->allocations) cudaFree(q);
        if (h->stream) cudaStreamDestroy(h->stream);
        delete h;
        return set_error(rc, "%s", msg.c_str());
    }
    *out = h;
    return CF_OK;
}

extern "C" int cf_mlp_destroy(cf_mlp *h) {
    if (!h) return CF_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (void *q : h->allocations) cudaFree(q);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return CF_OK;
}

extern "C" long long cf_mlp_num_params(cf_mlp *h) { return h ? h->nparam : -1; }

extern "C" int cf_mlp_forward(cf_mlp *h, const float *x, int n, float *y, void *stream) {
    clear_error();
    CF_REQUIRE(h && x && y, "cf_mlp_forward: null argument");
    CF_REQUIRE(n >= 0 && n <= h->max_batch, "cf_mlp_forward: batch %d outside [0, %d]", n, h->max_batch);
    CF_CUDA(cudaSetDevice(h->device));
    return forward(h, x, n, y, stream ? static_cast<cudaStream_t>(stream) : h->stream);
}

extern "C" int cf_mlp_gradients(cf_mlp *h, const float *x, const float *t, int n, float *grads, double *loss) {
    clear_error();
    CF_REQUIRE(h && x && t, "cf_mlp_gradients: null argument");
    CF_REQUIRE(n > 0 && n <= h->max_batch, "cf_mlp_gradients: batch %d outside [1, %d]", n, h->max_batch);
    CF_CUDA(cudaSetDevice(h->device));
    double l = 0.0;
    CF_TRY(backward(h, x, t, n, &l));
    if (loss) *loss = l;
    if (grads) {
        CF_CUDA(cudaMemcpyAsync(grads, h->grads, sizeof(float) * h->nparam, cudaMemcpyDeviceToHost, h->stream));
        CF_CUDA(cudaStreamSynchronize(h->stream));
    }
    return CF_OK;
}

extern "C" int cf_mlp_train_step(cf_mlp *h, const float *x, const float *t, int n, float lr, double *loss) {
    clear_error();
    CF_REQUIRE(h && x && t, "cf_mlp_train_step: null argument");
    CF_REQUIRE(n > 0 && n <= h->max_batch, "cf_mlp_train_step: batch %d outside [1, %d]", n, h->max_batch);
    CF_REQUIRE(lr > 0.0f, "cf_mlp_train_step: learning rate must be positive");
    CF_CUDA(cudaSetDevice(h->device));
    CF_TRY(backward(h, x, t, n, loss));
    h->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, static_cast<float>(h->step));
    const float c2 = 1.0f - std::pow(b2, static_cast<float>(h->step));
    adam_kernel<<<256, 256, 0, h->stream>>>(h->params, h->grads, h->adam_m, h->adam_v, h->nparam, lr, b1, b2, c1, c2,
                                            1e-8f);
    CF_CHECK_LAUNCH("adam_kernel");
    return CF_OK;
}

extern "C" int cf_mlp_get_params(cf_mlp *h, float *params) {
    clear_error();
    CF_REQUIRE(h && params, "cf_mlp_get_params: null argument");
    CF_CUDA(cudaSetDevice(h->device));
    CF_CUDA(cudaStreamSynchronize(h->stream));
    CF_CUDA(cudaMemcpy(params, h->params, sizeof(float) * h->nparam, cudaMemcpyDeviceToHost));
    return CF_OK;
}

extern "C" int cf_mlp_set_params(cf_mlp *h, const float *params) {
    clear_error();
    CF_REQUIRE(h && params, "cf_mlp_set_params: null argument");
    CF_CUDA(cudaSetDevice(h->device));
    CF_CUDA(cudaStreamSynchronize(h->stream));
    CF_CUDA(cudaMemcpy(h->params, params, sizeof(float) * h->nparam, cudaMemcpyHostToDevice));
    return CF_OK;
}

// ------------------------------------------------------------ checkpoints
// Versioned file of a trained network: the reference keeps no learned state,
// so the layout is this library's own (little-endian):
//   char magic[8] = "CFPRECN\0"; uint32 version = 1; uint32 kind = 1 (three
//   layers, ReLU); int32 in, hidden, out; float64 weight (the correction weight
//   alpha); int64 nparam; uint64 FNV-1a hash of the parameter bytes;
//   float32 params[nparam] (W1, b1, W2, b2, W3, b3 as cf_mlp_get_params).
namespace {
constexpr char kPrecondMagic[8] = {'C', 'F', 'P', 'R', 'E', 'C', 'N', '\0'};
constexpr uint32_t kPrecondVersion = 1, kPrecondKind = 1;

uint64_t fnv1a(const void *data, size_t n) {
    const unsigned char *p = static_cast<const unsigned char *>(data);
    uint64_t h = 1469598103934665603ull;
    for (size_t i = 0; i < n; ++i) {
        h ^= p[i];
        h *= 1099511628211ull;
    }
    return h;
}

struct PrecondHeader {
    char magic[8];
    uint32_t version, kind;
    int32_t in, hidden, out, pad;
    double weight;
    int64_t nparam;
    uint64_t hash;
};
static_assert(sizeof(PrecondHeader) == 56, "checkpoint header layout");
}  // namespace

extern "C" int cf_precond_save(cf_mlp *h, double weight, const char *path) {
    clear_error();
    CF_REQUIRE(h && path, "cf_precond_save: null argument");
    CF_REQUIRE(weight == weight, "cf_precond_save: weight is NaN");
    std::vector<float> params(static_cast<size_t>(h->nparam));
    CF_TRY(cf_mlp_get_params(h, params.data()));
    PrecondHeader hd{};
    std::memcpy(hd.magic, kPrecondMagic, sizeof(hd.magic));
    hd.version = kPrecondVersion;
    hd.kind = kPrecondKind;
    hd.in = h->in;
    hd.hidden = h->hid;
    hd.out = h->out;
    hd.weight = weight;
    hd.nparam = h->nparam;
    hd.hash = fnv1a(params.data(), params.size() * sizeof(float));
    std::FILE *f = std::fopen(path, "wb");
    if (!f) return set_error(CF_EINVAL, "cf_precond_save: cannot open %s for writing", path);
    const bool ok = std::fwrite(&hd, sizeof(hd), 1, f) == 1 &&
                    std::fwrite(params.data(), sizeof(float), params.size(), f) == params.size();
    const bool closed = std::fclose(f) == 0;
    if (!ok || !closed) return set_error(CF_EINVAL, "cf_precond_save: write to %s failed", path);
    return CF_OK;
}

extern "C" int cf_precond_load(const char *path, int max_batch, int device, cf_mlp **out, double *weight) {
    clear_error();
    CF_REQUIRE(path && out, "cf_precond_load: null argument");
    *out = nullptr;
    std::FILE *f = std::fopen(path, "rb");
    if (!f) return set_error(CF_EINVAL, "cf_precond_load: cannot open %s", path);
    PrecondHeader hd{};
    std::vector<float> params;
    const char *bad = nullptr;
    if (std::fread(&hd, sizeof(hd), 1, f) != 1) bad = "truncated header";
    else if (std::memcmp(hd.magic, kPrecondMagic, sizeof(hd.magic)) != 0) bad = "not a preconditioner checkpoint";
    else if (hd.version != kPrecondVersion) bad = "unsupported version";
    else if (hd.kind != kPrecondKind) bad = "unsupported network kind";
    else if (hd.in <= 0 || hd.hidden <= 0 || hd.out <= 0 || hd.in > 4096 || hd.hidden > 4096 || hd.out > 4096)
        bad = "bad layer widths";
    else if (hd.nparam != static_cast<int64_t>(hd.in) * hd.hidden + hd.hidden +
                              static_cast<int64_t>(hd.hidden) * hd.hidden + hd.hidden +
                              static_cast<int64_t>(hd.hidden) * hd.out + hd.out)
        bad = "parameter count does not match the widths";
    if (!bad) {
        params.resize(static_cast<size_t>(hd.nparam));
        if (std::fread(params.data(), sizeof(float), params.size(), f) != params.size()) bad = "truncated parameters";
        else if (fnv1a(params.data(), params.size() * sizeof(float)) != hd.hash) bad = "parameter hash mismatch";
    }
    std::fclose(f);
    if (bad) return set_error(CF_EINVAL, "cf_precond_load: %s: %s", path, bad);
    cf_mlp *h = nullptr;
    CF_TRY(cf_mlp_create(hd.in, hd.hidden, hd.out, max_batch, 0ull, device, &h));
    const int rc = cf_mlp_set_params(h, params.data());
    if (rc != CF_OK) {
        cf_mlp_destroy(h);
        return rc;
    }
    *out = h;
    if (weight) *weight = hd.weight;
    return CF_OK;
}

extern "C" int cf_mlp_stream(cf_mlp *h, void **stream) {
    clear_error();
    CF_REQUIRE(h && stream, "null argument");
    *stream = static_cast<void *>(h->stream);
    return CF_OK;
}

// tc_selftest.cu -- cf_tc_tile_product: one 64 x 64 x 64 tile product D = A^T B on
// the tensor cores through the building blocks of tc_tf32.cuh (operand split and
// canonical layout, descriptors, tcgen05.mma, commit, TMEM read-back), for
// checking those blocks against an FP64 product.
#include "common.cuh"
#include "tc_tf32.cuh"

namespace cufil {
namespace {

// One CTA of 256 threads: A [K][M], B [K][N] (FP32, row-major), D [M][N].
__global__ void __launch_bounds__(256, 1) tc_tile_kernel(const float *A, const float *B, float *D, int *status,
                                                         uint32_t wait_limit) {
    extern __shared__ __align__(128) float sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tbase;
    float *ahi = sm, *alo = sm + tc::kOperandFloats, *bhi = sm + 2 * tc::kOperandFloats,
          *blo = sm + 3 * tc::kOperandFloats;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) tc::tmem_alloc(&tbase, tc::kTmemCols);
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
    }
    for (int e = threadIdx.x; e < tc::kTileK * tc::kTileMN; e += blockDim.x) {
        const int k = e / tc::kTileMN, mn = e - k * tc::kTileMN;
        float h, l;
        tc::split_tf32(A[e], h, l);
        ahi[tc::canon(mn, k)] = h;
        alo[tc::canon(mn, k)] = l;
        tc::split_tf32(B[e], h, l);
        bhi[tc::canon(mn, k)] = h;
        blo[tc::canon(mn, k)] = l;
    }
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t base = tbase;
    if (threadIdx.x == 0) {
        tc::issue_tile_products(base, ahi, alo, bhi, blo);
        tc::commit(&bar);
    }
    bool done = mbar_wait_bounded(&bar, 0, wait_limit);
    if (!done) done = mbar_wait_bounded(&bar, 0);  // drain before the tensor memory is given back
    tc::fence_after_sync();
    if (done) {
        float v[32];
        tc::tmem_ld32(tc::tmem_addr(base, warp, (warp >> 2) * 32), v);
        if (lane < 16) {
            const int row = 16 * (warp & 3) + lane;
#pragma unroll
            for (int j = 0; j < 32; ++j) D[row * tc::kTileMN + (warp >> 2) * 32 + j] = v[j];
        }
    } else if (threadIdx.x == 0) {
        *status = 1;
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(base, tc::kTmemCols);
}

}  // namespace
}  // namespace cufil

using namespace cufil;

// D [64][64] = A^T B for A, B [64][64] (host arrays, row-major [k][m], [k][n]).  CF_TIMEOUT when the
// wait for the products gave up (`wait_limit` tries; 0 selects the default limit).
extern "C" int cf_tc_tile_product(const float *A, const float *B, float *D, unsigned wait_limit) {
    clear_error();
    CF_REQUIRE(A && B && D, "cf_tc_tile_product: null argument");
    const size_t bytes = sizeof(float) * tc::kTileK * tc::kTileMN;
    float *dA = nullptr, *dB = nullptr, *dD = nullptr;
    int *dst = nullptr;
    int rc = CF_OK, st = 0;
    const size_t smem = 4 * sizeof(float) * tc::kOperandFloats;
    do {
        if ((rc = cuda_status(cudaMalloc(&dA, bytes), "cudaMalloc", __FILE__, __LINE__))) break;
        if ((rc = cuda_status(cudaMalloc(&dB, bytes), "cudaMalloc", __FILE__, __LINE__))) break;
        if ((rc = cuda_status(cudaMalloc(&dD, bytes), "cudaMalloc", __FILE__, __LINE__))) break;
        if ((rc = cuda_status(cudaMalloc(&dst, sizeof(int)), "cudaMalloc", __FILE__, __LINE__))) break;
        if ((rc = cuda_status(cudaMemcpy(dA, A, bytes, cudaMemcpyHostToDevice), "cudaMemcpy", __FILE__, __LINE__))) break;
        if ((rc = cuda_status(cudaMemcpy(dB, B, bytes, cudaMemcpyHostToDevice), "cudaMemcpy", __FILE__, __LINE__))) break;
        if ((rc = cuda_status(cudaMemset(dD, 0, bytes), "cudaMemset", __FILE__, __LINE__))) break;
        if ((rc = cuda_status(cudaMemset(dst, 0, sizeof(int)), "cudaMemset", __FILE__, __LINE__))) break;
        if ((rc = cuda_status(cudaFuncSetAttribute(tc_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   static_cast<int>(smem)),
                              "cudaFuncSetAttribute", __FILE__, __LINE__)))
            break;
        tc_tile_kernel<<<1, 256, smem>>>(dA, dB, dD, dst, wait_limit ? wait_limit : kMbarSpinLimit);
        if ((rc = cuda_status(cudaGetLastError(), "tc_tile_kernel", __FILE__, __LINE__))) break;
        if ((rc = cuda_status(cudaMemcpy(D, dD, bytes, cudaMemcpyDeviceToHost), "cudaMemcpy", __FILE__, __LINE__))) break;
        if ((rc = cuda_status(cudaMemcpy(&st, dst, sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy", __FILE__,
                              __LINE__)))
            break;
    } while (0);
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dD);
    cudaFree(dst);
    if (rc != CF_OK) return rc;
    if (st) return set_error(CF_TIMEOUT, "cf_tc_tile_product: the wait for the tensor-core products gave up");
    return CF_OK;
}

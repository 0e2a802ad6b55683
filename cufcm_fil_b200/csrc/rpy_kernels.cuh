// rpy_kernels.cuh -- launch interface of the pairwise RPY block products.
//
// A block product V_t = M(t <- s) F_s is computed in two launches:
//   1. rpy_tile: grid (target tiles x source splits); each CTA stages its
//      source split (positions, forces, torques as float4) into shared memory
//      with one bulk async copy per array, then every thread sums the pair
//      blocks of its TI targets over the split in FP32 with blockwise
//      compensated (TwoSum) accumulation, and writes one partial per target.
//   2. rpy_reduce: sums the partials of each target over the splits in FP64
//      in a fixed order (deterministic), adds the wall self block, and writes
//      or accumulates the result in the caller's layout.
// The split count is chosen so that the grid fills every SM; the partials
// buffer (`scratch`) holds nt * nsplit * (VD/3) float4, target-major:
// partial[(i * nsplit + s) * (VD/3) + w], so the splits of one target are
// contiguous for the reduction.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>

namespace cufil {

struct RpyBlockDesc {
    int wall;             // 1: Swan-Brady wall blocks, 0: unbounded
    int vd, fd;           // 3 or 6
    int self_set;         // targets and sources are the same particles
    const float4 *xt;     // target centres [nt] (w ignored)
    int nt;
    float at;             // target radius (unbounded only)
    const float4 *xs;     // source centres [ns]
    const float4 *fs;     // source forces [ns]
    const float4 *ts;     // source torques [ns] (fd == 6)
    int ns;
    float as;             // source radius (unbounded only)
    float mu;             // viscosity (unbounded only)
};

struct RpyPlan {
    int sym;       // 1: symmetric warp-tile kernel (wall, segments on segments, 3x3)
    int nb;        // symmetric: 32-particle tiles
    long long items;  // symmetric: tile pairs of the upper triangle
    int grid;      // symmetric: CTAs
    int ti;        // targets per thread
    int tiles;     // target tiles (gridDim.x)
    int nsplit;    // source splits (gridDim.y)
    int split;     // sources per split
    size_t smem;   // dynamic shared memory bytes of the tile kernel
    size_t scratch_float4;  // float4 entries of the partials buffer
};

// Number of float4 entries needed in the partials buffer for any product with
// at most nt_max targets (sizing helper for allocators).
size_t rpy_scratch_float4(int nt_max, int ns_max, int vd, int num_sms);

RpyPlan rpy_plan(int nt, int ns, int vd, int fd, int num_sms);
// Same with at most max_nsplit source splits (bounded partials buffer); the
// split count never drops below ceil(ns / 2048).
RpyPlan rpy_plan_capped(int nt, int ns, int vd, int fd, int num_sms, int max_nsplit);
// Plan of the symmetric kernel for n particles acting on themselves.
RpyPlan rpy_plan_sym(int n, int num_sms);
// The plan rpy_block_product uses for d (symmetric when d allows it).
RpyPlan rpy_plan_for(const RpyBlockDesc &d, int num_sms);

// Configures the tile-kernel instantiation used by (d, plan) so that later
// launches may be captured into a CUDA graph.
int rpy_prepare(const RpyBlockDesc &d, const RpyPlan &plan);

// Launches the tile kernel; partials land in `scratch`.
int rpy_launch_tiles(const RpyBlockDesc &d, const RpyPlan &plan, float4 *scratch, int *dev_err,
                     cudaStream_t st);

// Batched symmetric wall products (segments on segments, 3x3) of B independent
// particle sets stored back to back.  Per array b: particles [seg0[b], seg0[b]+n[b])
// of x/f, nb[b] = ceil(n[b]/32) tiles, partials at partial + poff[b] laid out
// slot-major, [tile * n[b] + i], and work items [item0[b], item0[b+1]) (item0[B] == items).
struct SymBatchParams {
    const float4 *x;
    const float4 *f;
    float4 *partial;
    const int *seg0, *n, *nb;
    const long long *poff, *item0;
    const int *active;  // may be null: every array active
    int B;
    long long items;
};
int rpy_launch_sym_batch(const SymBatchParams &p, int grid, cudaStream_t st);
// Largest useful grid of the batched kernel (one resident wave).
int rpy_sym_batch_max_grid(int num_sms);

// Output modes of the reduction.
enum RpyOut : int { kOutWrite = 0, kOutAdd = 1 };

// Reduces partials into out_f[i*stride + c] (float) for c < vd; components
// vd..stride-1 are zeroed in write mode (the reference writes all six
// entries of a segment velocity, cuda_functions.cu:460-469).
// With dev_err given, every output of the launch is a quiet NaN when that
// word is non-zero (a tile block gave up waiting for its sources).
int rpy_launch_reduce_f32(const RpyBlockDesc &d, const RpyPlan &plan, const float4 *scratch, float *out_f,
                          int stride, int mode, cudaStream_t st, const int *dev_err = nullptr);

// Tries of the tile kernel's first bounded wait for its staged sources
// (cf_set_wait_limit); the default is the full limit.
unsigned rpy_wait_limit();

// Packing helpers between the reference's AoS host layouts and float4 arrays.
int pack_xyz_to_float4(const float *aos3, float4 *out, int n, cudaStream_t st);
int pack_ft6_to_float4(const float *aos6, float4 *force, float4 *torque, int n, cudaStream_t st);
// Both of the above for one particle set (positions [3n], forces + torques [6n]) in one launch.
int pack_set_to_float4(const float *aos3, const float *aos6, float4 *x, float4 *force, float4 *torque, int n,
                       cudaStream_t st);

// Full product V_t (=|+=) M F_s with the right staging; convenience wrapper.
int rpy_block_product(const RpyBlockDesc &d, float4 *scratch, size_t scratch_cap, int *dev_err, float *out_f,
                      int stride, int mode, int num_sms, cudaStream_t st);

}  // namespace cufil

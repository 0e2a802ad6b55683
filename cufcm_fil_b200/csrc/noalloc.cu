// noalloc.cu -- the wall segment-segment mobility product without any allocation.
//
// Some callers cannot allocate device memory at the moment they need a
// mobility product: code that runs while a CUDA stream is being captured into
// a graph (cudaMalloc is not permitted during capture), and hosts that own all
// of the device memory through their own pool or caching allocator and forbid
// or cannot afford a foreign cudaMalloc/cudaFree (which also synchronises the
// device) in their hot loop.  cf_rpy_wall_segments_noalloc serves them: the
// caller passes inputs and outputs, and the only scratch -- the float4 copies
// of positions and forces and the per-split partial sums of the split-source
// tile kernel (rpy_kernels.cu) -- lives in the file-scope array below, which
// every GPU that loads this library holds until the process exits.
#include "common.cuh"
#include "rpy_kernels.cuh"

#include <mutex>

namespace {

constexpr int kNoAllocMaxSegments = 8192;   // largest n_seg accepted
constexpr int kNoAllocMaxSplits = 16;       // source splits (partials per segment)
constexpr size_t kNoAllocHeader = 256;      // device flag word, padded to keep alignment
constexpr size_t kNoAllocBytes =
    kNoAllocHeader + sizeof(float4) * (2 * static_cast<size_t>(kNoAllocMaxSegments) +
                                       static_cast<size_t>(kNoAllocMaxSegments) * kNoAllocMaxSplits);

// Shared by every call on a device; contents persist from the previous call.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

struct DeviceSlot {
    bool ready = false;
    unsigned char *base = nullptr;  // device address of g_noalloc_scratch on this device
    int num_sms = CF_B200_SMS;
};
static DeviceSlot g_slots[64];
static std::mutex g_slots_mutex;

// Once per device, with that device current: resolve the array's device
// address (the host-side symbol is only a stand-in) and the SM count.
int device_slot(int dev, DeviceSlot **out) {
    CF_REQUIRE(dev >= 0 && dev < 64, "cf_rpy_wall_segments_noalloc: device %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_slots_mutex);
    DeviceSlot &s = g_slots[dev];
    if (!s.ready) {
        void *ptr = nullptr;
        CF_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
        CF_CUDA(cudaDeviceGetAttribute(&s.num_sms, cudaDevAttrMultiProcessorCount, dev));
        s.base = static_cast<unsigned char *>(ptr);
        s.ready = true;
    }
    *out = &s;
    return CF_OK;
}

}  // namespace

using namespace cufil;

extern "C" int cf_rpy_wall_segments_noalloc(const float *d_x_segs, const float *d_f_segs, float *d_v_segs, int n_seg,
                                            void *stream) {
    clear_error();
    CF_REQUIRE(n_seg >= 1, "cf_rpy_wall_segments_noalloc: n_seg must be >= 1 (got %d)", n_seg);
    CF_REQUIRE(n_seg <= kNoAllocMaxSegments,
               "cf_rpy_wall_segments_noalloc: n_seg = %d exceeds the fixed scratch limit of %d segments", n_seg,
               kNoAllocMaxSegments);
    CF_REQUIRE(d_x_segs && d_f_segs && d_v_segs, "cf_rpy_wall_segments_noalloc: null buffer");
    int dev = 0;
    CF_CUDA(cudaGetDevice(&dev));
    DeviceSlot *slot = nullptr;
    CF_TRY(device_slot(dev, &slot));
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    int *err = reinterpret_cast<int *>(slot->base);
    float4 *x4 = reinterpret_cast<float4 *>(slot->base + kNoAllocHeader);
    float4 *f4 = x4 + n_seg;
    float4 *partial = f4 + n_seg;

    RpyBlockDesc d{};
    d.wall = 1;
    d.vd = 3;
    d.fd = 3;
    d.self_set = 1;
    d.xt = x4;
    d.nt = n_seg;
    d.at = 1.0f;
    d.xs = x4;
    d.fs = f4;
    d.ts = nullptr;
    d.ns = n_seg;
    d.as = 1.0f;
    d.mu = 1.0f;
    const RpyPlan plan = rpy_plan_capped(n_seg, n_seg, 3, 3, slot->num_sms, kNoAllocMaxSplits);
    if (plan.scratch_float4 > static_cast<size_t>(kNoAllocMaxSegments) * kNoAllocMaxSplits)
        return set_error(CF_EINVAL, "cf_rpy_wall_segments_noalloc: plan needs %zu partials", plan.scratch_float4);

    // The flag word must start at zero; x4, f4 and every partial slot are
    // written before they are read, so nothing else needs clearing.  If a tile
    // block gives up waiting for its staged sources it leaves its partials
    // unwritten (stale from an earlier call) and sets the flag; the reduction
    // reads the flag and then writes NaN to every output instead of a sum.
    CF_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
    CF_TRY(pack_set_to_float4(d_x_segs, d_f_segs, x4, f4, nullptr, n_seg, st));
    CF_TRY(rpy_launch_tiles(d, plan, partial, err, st));
    return rpy_launch_reduce_f32(d, plan, partial, d_v_segs, 6, kOutWrite, st, err);
}

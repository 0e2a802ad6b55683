// mobility.cu -- cf_mobility: the RPY back-end of the mobility-solver contract.
//
// Mirrors rpy_mobility_solver (src/cilia/mobility/rpy_mobility_solver.{hpp,cu}):
// the same AoS host layouts and the same evaluate_* write/accumulate semantics,
// but one device, one stream per handle, no device-wide synchronisation, and
// float4 particle records repacked once per copy.
#include "common.cuh"
#include "rpy_kernels.cuh"

#include <algorithm>
#include <new>

struct cf_mobility {
    cf_mobility_config cfg{};
    int num_sms = CF_B200_SMS;
    cudaStream_t stream = nullptr;
    // Device copies of the reference host layouts.
    float *x_segs = nullptr, *f_segs = nullptr, *v_segs = nullptr;
    float *x_blobs = nullptr, *f_blobs = nullptr, *v_blobs = nullptr;
    // float4 particle records used by the kernels.
    float4 *xs4 = nullptr, *fs4 = nullptr, *ts4 = nullptr;
    float4 *xb4 = nullptr, *fb4 = nullptr;
    // Partial sums of the split-source products.
    float4 *scratch = nullptr;
    size_t scratch_cap = 0;
    int *err = nullptr;  // device error flags (bulk-copy timeouts)
};

namespace cufil {
namespace {

template <typename T>
int dalloc(T **p, size_t n) {
    *p = nullptr;
    if (n == 0) return CF_OK;
    CF_CUDA(cudaMalloc(reinterpret_cast<void **>(p), n * sizeof(T)));
    return CF_OK;
}

int check_device_flags(cf_mobility *h) {
    int flags = 0;
    CF_CUDA(cudaMemcpyAsync(&flags, h->err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CF_CUDA(cudaStreamSynchronize(h->stream));
    if (flags) {
        CF_CUDA(cudaMemsetAsync(h->err, 0, sizeof(int), h->stream));
        return set_error(CF_TIMEOUT, "mobility: a bounded device wait gave up (flags 0x%x)", flags);
    }
    return CF_OK;
}

RpyBlockDesc desc_ss(cf_mobility *h) {
    RpyBlockDesc d{};
    d.wall = h->cfg.wall;
    d.vd = h->cfg.seg_dof;
    d.fd = h->cfg.seg_dof;
    d.self_set = 1;
    d.xt = h->xs4;
    d.nt = h->cfg.n_seg;
    d.at = static_cast<float>(h->cfg.seg_radius);
    d.xs = h->xs4;
    d.fs = h->fs4;
    d.ts = h->ts4;
    d.ns = h->cfg.n_seg;
    d.as = static_cast<float>(h->cfg.seg_radius);
    d.mu = static_cast<float>(h->cfg.mu);
    return d;
}

RpyBlockDesc desc_sb(cf_mobility *h) {
    RpyBlockDesc d{};
    d.wall = h->cfg.wall;
    d.vd = h->cfg.seg_dof;
    d.fd = 3;
    d.self_set = 0;
    d.xt = h->xs4;
    d.nt = h->cfg.n_seg;
    d.at = static_cast<float>(h->cfg.seg_radius);
    d.xs = h->xb4;
    d.fs = h->fb4;
    d.ts = nullptr;
    d.ns = h->cfg.n_blob;
    d.as = static_cast<float>(h->cfg.blob_radius);
    d.mu = static_cast<float>(h->cfg.mu);
    return d;
}

RpyBlockDesc desc_bb(cf_mobility *h) {
    RpyBlockDesc d{};
    d.wall = h->cfg.wall;
    d.vd = 3;
    d.fd = 3;
    d.self_set = 1;
    d.xt = h->xb4;
    d.nt = h->cfg.n_blob;
    d.at = static_cast<float>(h->cfg.blob_radius);
    d.xs = h->xb4;
    d.fs = h->fb4;
    d.ts = nullptr;
    d.ns = h->cfg.n_blob;
    d.as = static_cast<float>(h->cfg.blob_radius);
    d.mu = static_cast<float>(h->cfg.mu);
    return d;
}

RpyBlockDesc desc_bs(cf_mobility *h) {
    RpyBlockDesc d{};
    d.wall = h->cfg.wall;
    d.vd = 3;
    d.fd = h->cfg.seg_dof;
    d.self_set = 0;
    d.xt = h->xb4;
    d.nt = h->cfg.n_blob;
    d.at = static_cast<float>(h->cfg.blob_radius);
    d.xs = h->xs4;
    d.fs = h->fs4;
    d.ts = h->ts4;
    d.ns = h->cfg.n_seg;
    d.as = static_cast<float>(h->cfg.seg_radius);
    d.mu = static_cast<float>(h->cfg.mu);
    return d;
}

int product(cf_mobility *h, const RpyBlockDesc &d, float *out, int stride, int mode, cudaStream_t st) {
    return rpy_block_product(d, h->scratch, h->scratch_cap, h->err, out, stride, mode, h->num_sms, st);
}

int eval_ss(cf_mobility *h, float *v_segs, cudaStream_t st) {
    if (h->cfg.n_seg == 0) return CF_OK;
    return product(h, desc_ss(h), v_segs, 6, kOutWrite, st);
}
int eval_sb(cf_mobility *h, float *v_segs, cudaStream_t st) {
    if (h->cfg.n_seg == 0 || h->cfg.n_blob == 0) return CF_OK;
    return product(h, desc_sb(h), v_segs, 6, kOutAdd, st);
}
int eval_bb(cf_mobility *h, float *v_blobs, cudaStream_t st) {
    if (h->cfg.n_blob == 0) return CF_OK;
    return product(h, desc_bb(h), v_blobs, 3, kOutWrite, st);
}
int eval_bs(cf_mobility *h, float *v_blobs, cudaStream_t st) {
    if (h->cfg.n_blob == 0) return CF_OK;
    if (h->cfg.n_seg == 0) {
        if (h->cfg.seg_dof == 6) CF_CUDA(cudaMemsetAsync(v_blobs, 0, 3 * sizeof(float) * h->cfg.n_blob, st));
        return CF_OK;
    }
    // Mbs_mult accumulates for prescribed cilia and overwrites otherwise
    // (cuda_functions.cu:740-752, SOLVER_TYPE 1).
    return product(h, desc_bs(h), v_blobs, 3, h->cfg.seg_dof == 3 ? kOutAdd : kOutWrite, st);
}

int eval_full(cf_mobility *h, float *v_segs, float *v_blobs, cudaStream_t st) {
    CF_TRY(eval_ss(h, v_segs, st));
    CF_TRY(eval_sb(h, v_segs, st));
    CF_TRY(eval_bb(h, v_blobs, st));
    if (h->cfg.n_blob > 0 && h->cfg.n_seg > 0)
        CF_TRY(product(h, desc_bs(h), v_blobs, 3, kOutAdd, st));
    return CF_OK;
}

}  // namespace
}  // namespace cufil

using namespace cufil;

extern "C" int cf_mobility_create(const cf_mobility_config *cfg, cf_mobility **out) {
    clear_error();
    CF_REQUIRE(cfg && out, "cf_mobility_create: null argument");
    *out = nullptr;
    CF_REQUIRE(cfg->n_seg >= 0 && cfg->n_blob >= 0 && cfg->n_seg + cfg->n_blob > 0,
               "cf_mobility_create: need n_seg + n_blob > 0 (got %d, %d)", cfg->n_seg, cfg->n_blob);
    CF_REQUIRE(cfg->seg_dof == 3 || cfg->seg_dof == 6, "cf_mobility_create: seg_dof must be 3 or 6 (got %d)",
               cfg->seg_dof);
    CF_REQUIRE(cfg->wall == 0 || cfg->wall == 1, "cf_mobility_create: wall must be 0 or 1");
    CF_REQUIRE(cfg->wall || (cfg->seg_radius > 0 && cfg->blob_radius > 0 && cfg->mu > 0),
               "cf_mobility_create: radii and viscosity must be positive");
    CF_REQUIRE(cfg->n_seg < (1 << 28) && cfg->n_blob < (1 << 28), "cf_mobility_create: particle count too large");
    CF_CUDA(cudaSetDevice(cfg->device));
    cf_mobility *h = new (std::nothrow) cf_mobility();
    if (!h) return set_error(CF_ENOMEM, "cf_mobility_create: host allocation failed");
    h->cfg = *cfg;
    int rc = CF_OK;
    do {
        cudaDeviceProp prop;
        if ((rc = cuda_status(cudaGetDeviceProperties(&prop, cfg->device), "cudaGetDeviceProperties", __FILE__,
                              __LINE__)) != CF_OK)
            break;
        h->num_sms = prop.multiProcessorCount;
        if ((rc = cuda_status(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate",
                              __FILE__, __LINE__)) != CF_OK)
            break;
        const size_t ns = cfg->n_seg, nb = cfg->n_blob;
        if ((rc = dalloc(&h->x_segs, 3 * ns)) || (rc = dalloc(&h->f_segs, 6 * ns)) || (rc = dalloc(&h->v_segs, 6 * ns)) ||
            (rc = dalloc(&h->x_blobs, 3 * nb)) || (rc = dalloc(&h->f_blobs, 3 * nb)) ||
            (rc = dalloc(&h->v_blobs, 3 * nb)) || (rc = dalloc(&h->xs4, ns)) || (rc = dalloc(&h->fs4, ns)) ||
            (rc = dalloc(&h->ts4, ns)) || (rc = dalloc(&h->xb4, nb)) || (rc = dalloc(&h->fb4, nb)) ||
            (rc = dalloc(&h->err, 1)))
            break;
        // Partials buffer: the largest of the four block products' plans.
        const int sd = cfg->seg_dof, n_s = cfg->n_seg, n_b = cfg->n_blob;
        const RpyPlan plans[6] = {rpy_plan(n_s, n_s, sd, sd, h->num_sms), rpy_plan(n_s, n_b, sd, 3, h->num_sms),
                                  rpy_plan(n_b, n_b, 3, 3, h->num_sms), rpy_plan(n_b, n_s, 3, sd, h->num_sms),
                                  rpy_plan_sym(n_s, h->num_sms), rpy_plan_sym(n_b, h->num_sms)};
        h->scratch_cap = 1;
        for (const RpyPlan &pl : plans) h->scratch_cap = std::max(h->scratch_cap, pl.scratch_float4);
        if ((rc = dalloc(&h->scratch, h->scratch_cap))) break;
        if ((rc = cuda_status(cudaMemsetAsync(h->err, 0, sizeof(int), h->stream), "cudaMemsetAsync", __FILE__,
                              __LINE__)))
            break;
        if (ns && (rc = cuda_status(cudaMemsetAsync(h->ts4, 0, ns * sizeof(float4), h->stream), "cudaMemsetAsync",
                                    __FILE__, __LINE__)))
            break;
        if ((rc = cuda_status(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize", __FILE__, __LINE__)))
            break;
    } while (0);
    if (rc != CF_OK) {
        std::string msg = cf_last_error();
        cf_mobility_destroy(h);
        set_error(rc, "%s", msg.c_str());
        return rc;
    }
    *out = h;
    return CF_OK;
}

extern "C" int cf_mobility_destroy(cf_mobility *h) {
    if (!h) return CF_OK;
    cudaSetDevice(h->cfg.device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (void *p : {(void *)h->x_segs, (void *)h->f_segs, (void *)h->v_segs, (void *)h->x_blobs, (void *)h->f_blobs,
                    (void *)h->v_blobs, (void *)h->xs4, (void *)h->fs4, (void *)h->ts4, (void *)h->xb4,
                    (void *)h->fb4, (void *)h->scratch, (void *)h->err})
        if (p) cudaFree(p);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return CF_OK;
}

extern "C" int cf_copy_segment_positions_to_device(cf_mobility *h, const float *x_segs) {
    clear_error();
    CF_REQUIRE(h && (x_segs || h->cfg.n_seg == 0), "cf_copy_segment_positions_to_device: null argument");
    const int n = h->cfg.n_seg;
    if (!n) return CF_OK;
    CF_CUDA(cudaSetDevice(h->cfg.device));
    CF_CUDA(cudaMemcpyAsync(h->x_segs, x_segs, 3 * sizeof(float) * n, cudaMemcpyHostToDevice, h->stream));
    return pack_xyz_to_float4(h->x_segs, h->xs4, n, h->stream);
}

extern "C" int cf_copy_segment_forces_to_device(cf_mobility *h, const float *f_segs) {
    clear_error();
    CF_REQUIRE(h && (f_segs || h->cfg.n_seg == 0), "cf_copy_segment_forces_to_device: null argument");
    const int n = h->cfg.n_seg;
    if (!n) return CF_OK;
    CF_CUDA(cudaSetDevice(h->cfg.device));
    CF_CUDA(cudaMemcpyAsync(h->f_segs, f_segs, 6 * sizeof(float) * n, cudaMemcpyHostToDevice, h->stream));
    return pack_ft6_to_float4(h->f_segs, h->fs4, h->ts4, n, h->stream);
}

extern "C" int cf_copy_blob_positions_to_device(cf_mobility *h, const float *x_blobs) {
    clear_error();
    CF_REQUIRE(h && (x_blobs || h->cfg.n_blob == 0), "cf_copy_blob_positions_to_device: null argument");
    const int n = h->cfg.n_blob;
    if (!n) return CF_OK;
    CF_CUDA(cudaSetDevice(h->cfg.device));
    CF_CUDA(cudaMemcpyAsync(h->x_blobs, x_blobs, 3 * sizeof(float) * n, cudaMemcpyHostToDevice, h->stream));
    return pack_xyz_to_float4(h->x_blobs, h->xb4, n, h->stream);
}

extern "C" int cf_copy_blob_forces_to_device(cf_mobility *h, const float *f_blobs) {
    clear_error();
    CF_REQUIRE(h && (f_blobs || h->cfg.n_blob == 0), "cf_copy_blob_forces_to_device: null argument");
    const int n = h->cfg.n_blob;
    if (!n) return CF_OK;
    CF_CUDA(cudaSetDevice(h->cfg.device));
    CF_CUDA(cudaMemcpyAsync(h->f_blobs, f_blobs, 3 * sizeof(float) * n, cudaMemcpyHostToDevice, h->stream));
    return pack_xyz_to_float4(h->f_blobs, h->fb4, n, h->stream);
}

extern "C" int cf_copy_segment_velocities_to_host(cf_mobility *h, float *v_segs) {
    clear_error();
    CF_REQUIRE(h && (v_segs || h->cfg.n_seg == 0), "cf_copy_segment_velocities_to_host: null argument");
    if (!h->cfg.n_seg) return CF_OK;
    CF_CUDA(cudaSetDevice(h->cfg.device));
    CF_CUDA(cudaMemcpyAsync(v_segs, h->v_segs, 6 * sizeof(float) * h->cfg.n_seg, cudaMemcpyDeviceToHost, h->stream));
    return check_device_flags(h);
}

extern "C" int cf_copy_blob_velocities_to_host(cf_mobility *h, float *v_blobs) {
    clear_error();
    CF_REQUIRE(h && (v_blobs || h->cfg.n_blob == 0), "cf_copy_blob_velocities_to_host: null argument");
    if (!h->cfg.n_blob) return CF_OK;
    CF_CUDA(cudaSetDevice(h->cfg.device));
    CF_CUDA(cudaMemcpyAsync(v_blobs, h->v_blobs, 3 * sizeof(float) * h->cfg.n_blob, cudaMemcpyDeviceToHost,
                            h->stream));
    return check_device_flags(h);
}

extern "C" int cf_wait_for_device(cf_mobility *h) {
    clear_error();
    CF_REQUIRE(h, "cf_wait_for_device: null handle");
    CF_CUDA(cudaSetDevice(h->cfg.device));
    return check_device_flags(h);
}

extern "C" int cf_evaluate_segment_segment_mobility(cf_mobility *h) {
    clear_error();
    CF_REQUIRE(h, "null handle");
    CF_CUDA(cudaSetDevice(h->cfg.device));
    return eval_ss(h, h->v_segs, h->stream);
}

extern "C" int cf_evaluate_segment_blob_mobility(cf_mobility *h) {
    clear_error();
    CF_REQUIRE(h, "null handle");
    CF_CUDA(cudaSetDevice(h->cfg.device));
    return eval_sb(h, h->v_segs, h->stream);
}

extern "C" int cf_evaluate_blob_blob_mobility(cf_mobility *h) {
    clear_error();
    CF_REQUIRE(h, "null handle");
    CF_CUDA(cudaSetDevice(h->cfg.device));
    return eval_bb(h, h->v_blobs, h->stream);
}

extern "C" int cf_evaluate_blob_segment_mobility(cf_mobility *h) {
    clear_error();
    CF_REQUIRE(h, "null handle");
    CF_CUDA(cudaSetDevice(h->cfg.device));
    return eval_bs(h, h->v_blobs, h->stream);
}

extern "C" int cf_evaluate_full_mobility(cf_mobility *h) {
    clear_error();
    CF_REQUIRE(h, "null handle");
    CF_CUDA(cudaSetDevice(h->cfg.device));
    return eval_full(h, h->v_segs, h->v_blobs, h->stream);
}

extern "C" int cf_apply_mobility(cf_mobility *h, const float *x_segs, const float *x_blobs, const float *f_segs,
                                 const float *f_blobs, float *v_segs, float *v_blobs) {
    clear_error();
    CF_REQUIRE(h, "cf_apply_mobility: null handle");
    CF_TRY(cf_copy_segment_positions_to_device(h, x_segs));
    CF_TRY(cf_copy_blob_positions_to_device(h, x_blobs));
    CF_TRY(cf_copy_segment_forces_to_device(h, f_segs));
    CF_TRY(cf_copy_blob_forces_to_device(h, f_blobs));
    CF_TRY(cf_evaluate_full_mobility(h));
    CF_TRY(cf_copy_segment_velocities_to_host(h, v_segs));
    CF_TRY(cf_copy_blob_velocities_to_host(h, v_blobs));
    return cf_wait_for_device(h);
}

extern "C" int cf_apply_mobility_device(cf_mobility *h, const float *d_x_segs, const float *d_x_blobs,
                                        const float *d_f_segs, const float *d_f_blobs, float *d_v_segs,
                                        float *d_v_blobs, void *stream) {
    clear_error();
    CF_REQUIRE(h, "cf_apply_mobility_device: null handle");
    const int ns = h->cfg.n_seg, nb = h->cfg.n_blob;
    CF_REQUIRE(!ns || (d_x_segs && d_f_segs && d_v_segs), "cf_apply_mobility_device: missing segment buffers");
    CF_REQUIRE(!nb || (d_x_blobs && d_f_blobs && d_v_blobs), "cf_apply_mobility_device: missing blob buffers");
    CF_CUDA(cudaSetDevice(h->cfg.device));
    // A null stream is CUDA's legacy default stream, as for any runtime call.
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    CF_TRY(pack_set_to_float4(d_x_segs, d_f_segs, h->xs4, h->fs4, h->ts4, ns, st));
    CF_TRY(pack_xyz_to_float4(d_x_blobs, h->xb4, nb, st));
    CF_TRY(pack_xyz_to_float4(d_f_blobs, h->fb4, nb, st));
    return eval_full(h, d_v_segs, d_v_blobs, st);
}

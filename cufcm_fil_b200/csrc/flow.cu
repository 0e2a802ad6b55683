// flow.cu -- cf_flow: flow velocities at field points from saved segment and
// blob forces, the reference's flow-field post-processor
// (src/flow_field/flow_field_evaluator.cu:13-217, flow_velocities; host side
// :222-557).  Per flow point i:
//   v_i = 1/(8 pi mu) * ( sum over segments j of  S(x_i - x_j) f_j
//                           [+ Blake image terms of a wall at z = 0 when the data has no blobs]
//                           + rotlet of the segment torque
//                           [- S(x_i - X_body(j)) f_j with remove_net_force]
//                       + sum over blobs k of  S(x_i - x_k) f_k  [- S(x_i - X_body(k)) f_k] )
// with S(r) f = f/|r| + r (r.f)/|r|^3, the kernel's expressions term by term.
//
// The reference runs one thread per flow point over 64-wide shared-memory
// tiles.  Here: float4 source records packed once per call, 256-source tiles
// in shared memory, two flow points per thread, the source range split over
// gridDim.y so that a small set of flow points still fills every SM, FP32
// blockwise TwoSum accumulation, and an FP64 reduction of the split partials
// in a fixed order (deterministic, no atomics).
#include "common.cuh"

#include <algorithm>
#include <new>

struct cf_flow {
    cf_flow_config cfg{};
    int num_sms = CF_B200_SMS;
    cudaStream_t stream = nullptr;
    float4 *sx = nullptr, *sf = nullptr, *st = nullptr, *sb = nullptr;  // sources: centre, force, torque, body
    float4 *partial = nullptr;
    size_t partial_cap = 0;
    float *hx_flow = nullptr, *hx_segs = nullptr, *hf_segs = nullptr, *hx_blobs = nullptr, *hf_blobs = nullptr,
          *hx_bodies = nullptr, *hv_flow = nullptr;  // device staging of the host entry point
    int max_bodies = 0;
};

namespace cufil {
namespace {

constexpr int kFlowThreads = 128;
constexpr int kFlowTI = 2;      // flow points per thread
constexpr int kFlowTile = 256;  // sources per shared-memory tile
constexpr int kFlowTargets = kFlowThreads * kFlowTI;

struct FlowParams {
    const float *xf;                  // [3 Nf]
    const float4 *sx, *sf, *st, *sb;  // sources
    float4 *partial;                  // [Nf][nsplit]
    int nf, ns, split, nsplit;
};

template <bool SEG, bool WALL, bool NET>
__device__ __forceinline__ void flow_pair(float xi, float yi, float zi, const float4 &xs, const float4 &f,
                                          const float4 &t, const float4 &xb, float &vx, float &vy, float &vz) {
    const float dx = xi - xs.x, dy = yi - xs.y, dz = zi - xs.z;
    const float rm2 = 1.0f / (dx * dx + dy * dy + dz * dz);
    const float rm1 = sqrtf(rm2);
    const float rdf = rm2 * (dx * f.x + dy * f.y + dz * f.z);
    vx += rm1 * (f.x + dx * rdf);
    vy += rm1 * (f.y + dy * rdf);
    vz += rm1 * (f.z + dz * rdf);
    if constexpr (SEG && WALL) {  // Blake's image system (no blobs: half-space data)
        const float Rz = zi + xs.z;
        const float R2 = dx * dx + dy * dy + Rz * Rz;
        const float Rm1 = sqrtf(1.0f / R2);
        const float Rdf = (dx * f.x + dy * f.y + Rz * f.z) * Rm1 * Rm1;
        vx -= Rm1 * (f.x + dx * Rdf);
        vy -= Rm1 * (f.y + dy * Rdf);
        vz -= Rm1 * (f.z + Rz * Rdf);
        const float Dxx = (3.0f * dx * dx - R2) * zi;
        const float Dxy = 3.0f * dx * dy * zi;
        const float Dxz = (R2 - 3.0f * Rz * zi) * dx;
        const float Dyy = (3.0f * dy * dy - R2) * zi;
        const float Dyz = (R2 - 3.0f * Rz * zi) * dy;
        const float Dzx = (3.0f * Rz * zi + R2) * dx;
        const float Dzy = (3.0f * Rz * zi + R2) * dy;
        const float Dzz = (R2 - 3.0f * Rz * Rz) * zi;
        const float Rm2 = Rm1 * Rm1;
        const float Dfac = 2.0f * xs.z * Rm2 * Rm2 * Rm1;
        vx += Dfac * (Dxx * f.x + Dxy * f.y + Dxz * f.z);
        vy += Dfac * (Dxy * f.x + Dyy * f.y + Dyz * f.z);
        vz += Dfac * (Dzx * f.x + Dzy * f.y + Dzz * f.z);
    }
    if constexpr (SEG) {  // rotlet of the segment torque
        const float rm3 = rm1 * rm2;
        vx += rm3 * (t.y * dz - t.z * dy);
        vy += rm3 * (t.z * dx - t.x * dz);
        vz += rm3 * (t.x * dy - t.y * dx);
    }
    if constexpr (NET) {  // minus a Stokeslet of the same force at the source's body
        const float ex = xi - xb.x, ey = yi - xb.y, ez = zi - xb.z;
        const float qm2 = 1.0f / (ex * ex + ey * ey + ez * ez);
        const float qm1 = sqrtf(qm2);
        const float qdf = qm2 * (ex * f.x + ey * f.y + ez * f.z);
        vx -= qm1 * (f.x + ex * qdf);
        vy -= qm1 * (f.y + ey * qdf);
        vz -= qm1 * (f.z + ez * qdf);
    }
}

__device__ __forceinline__ void two_sum3(float *hi, float *lo, float ax, float ay, float az) {
    const float a[3] = {ax, ay, az};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float s = hi[c] + a[c];
        const float bp = s - hi[c];
        lo[c] += (hi[c] - (s - bp)) + (a[c] - bp);
        hi[c] = s;
    }
}

// grid (ceil(nf / 256), nsplit): block (x, y) sums sources [y*split, (y+1)*split)
// of its 256 flow points.  Sources [0, nseg_src) are segments, the rest blobs.
template <bool WALL, bool NET>
__global__ void __launch_bounds__(kFlowThreads) flow_tile_kernel(FlowParams p, int nseg_src) {
    __shared__ float4 s_x[kFlowTile], s_f[kFlowTile], s_t[kFlowTile], s_b[kFlowTile];
    const int j0 = blockIdx.y * p.split;
    const int j1 = min(p.ns, j0 + p.split);
    float xi[kFlowTI], yi[kFlowTI], zi[kFlowTI];
    float hi[kFlowTI][3], lo[kFlowTI][3];
#pragma unroll
    for (int k = 0; k < kFlowTI; ++k) {
        const int i = min(static_cast<int>(blockIdx.x * kFlowTargets + k * kFlowThreads + threadIdx.x), p.nf - 1);
        xi[k] = p.xf[3 * i];
        yi[k] = p.xf[3 * i + 1];
        zi[k] = p.xf[3 * i + 2];
#pragma unroll
        for (int c = 0; c < 3; ++c) hi[k][c] = lo[k][c] = 0.0f;
    }
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int t0 = j0; t0 < j1; t0 += kFlowTile) {
        const int nt = min(kFlowTile, j1 - t0);
        __syncthreads();
        for (int q = threadIdx.x; q < nt; q += kFlowThreads) {
            s_x[q] = p.sx[t0 + q];
            s_f[q] = p.sf[t0 + q];
            s_t[q] = (t0 + q < nseg_src) ? p.st[t0 + q] : zero4;
            s_b[q] = NET ? p.sb[t0 + q] : zero4;
        }
        __syncthreads();
        // Segments and blobs of this tile: two branch-free loops.
        const int nsg = max(0, min(nt, nseg_src - t0));
        float vx[kFlowTI], vy[kFlowTI], vz[kFlowTI];
#pragma unroll
        for (int k = 0; k < kFlowTI; ++k) vx[k] = vy[k] = vz[k] = 0.0f;
        for (int q = 0; q < nsg; ++q) {
            const float4 xs = s_x[q], f = s_f[q], tq = s_t[q], xb = s_b[q];
#pragma unroll
            for (int k = 0; k < kFlowTI; ++k)
                flow_pair<true, WALL, NET>(xi[k], yi[k], zi[k], xs, f, tq, xb, vx[k], vy[k], vz[k]);
        }
        for (int q = nsg; q < nt; ++q) {
            const float4 xs = s_x[q], f = s_f[q], xb = s_b[q];
#pragma unroll
            for (int k = 0; k < kFlowTI; ++k)
                flow_pair<false, false, NET>(xi[k], yi[k], zi[k], xs, f, zero4, xb, vx[k], vy[k], vz[k]);
        }
#pragma unroll
        for (int k = 0; k < kFlowTI; ++k) two_sum3(hi[k], lo[k], vx[k], vy[k], vz[k]);
    }
#pragma unroll
    for (int k = 0; k < kFlowTI; ++k) {
        const int i = static_cast<int>(blockIdx.x * kFlowTargets + k * kFlowThreads + threadIdx.x);
        if (i < p.nf)
            p.partial[static_cast<size_t>(i) * p.nsplit + blockIdx.y] =
                make_float4(hi[k][0] + lo[k][0], hi[k][1] + lo[k][1], hi[k][2] + lo[k][2], 0.0f);
    }
}

// One warp per flow point: FP64 sum of its partials in a fixed order, times 1/(8 pi mu).
__global__ void flow_reduce_kernel(const float4 *__restrict__ partial, int nf, int nsplit, double prefac,
                                   float *__restrict__ v) {
    const int lane = threadIdx.x & 31;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= nf) return;
    double a[3] = {0.0, 0.0, 0.0};
    for (int s = lane; s < nsplit; s += 32) {
        const float4 q = partial[static_cast<size_t>(i) * nsplit + s];
        a[0] += q.x;
        a[1] += q.y;
        a[2] += q.z;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a[c] += __shfl_down_sync(0xffffffffu, a[c], o);
    if (lane == 0)
        for (int c = 0; c < 3; ++c) v[3 * i + c] = static_cast<float>(prefac * a[c]);
}

// Source records: segments [0, ns) from x [3ns] and f [6ns] (force, torque),
// then blobs [ns, ns + nb) from x [3nb] and f [3nb]; with bodies, the position
// of each source's body (segment j: body j / ns_per_body; blob k: k / nb_per_body).
__global__ void flow_pack_kernel(const float *xs, const float *fs, int ns, int ns_pb, const float *xb,
                                 const float *fb, int nb, int nb_pb, const float *xbod, float4 *sx, float4 *sf,
                                 float4 *st, float4 *sbod) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ns + nb) return;
    int body = 0;
    if (j < ns) {
        sx[j] = make_float4(xs[3 * j], xs[3 * j + 1], xs[3 * j + 2], 0.0f);
        sf[j] = make_float4(fs[6 * j], fs[6 * j + 1], fs[6 * j + 2], 0.0f);
        st[j] = make_float4(fs[6 * j + 3], fs[6 * j + 4], fs[6 * j + 5], 0.0f);
        body = ns_pb > 0 ? j / ns_pb : 0;
    } else {
        const int k = j - ns;
        sx[j] = make_float4(xb[3 * k], xb[3 * k + 1], xb[3 * k + 2], 0.0f);
        sf[j] = make_float4(fb[3 * k], fb[3 * k + 1], fb[3 * k + 2], 0.0f);
        body = nb_pb > 0 ? k / nb_pb : 0;
    }
    if (xbod) sbod[j] = make_float4(xbod[3 * body], xbod[3 * body + 1], xbod[3 * body + 2], 0.0f);
}

struct FlowPlan {
    int tiles, nsplit, split;
};

// Splits the sources so that about two waves of 256-point blocks (4 resident per
// SM) cover the SMs, keeping at least one tile of sources per split.
FlowPlan flow_plan(int nf, int nsrc, int num_sms) {
    FlowPlan p{};
    p.tiles = std::max(1, (nf + kFlowTargets - 1) / kFlowTargets);
    const int want = std::max(1, (2 * 4 * num_sms + p.tiles - 1) / p.tiles);
    const int max_split = std::max(1, (nsrc + kFlowTile - 1) / kFlowTile);
    p.nsplit = std::min(want, max_split);
    p.split = (nsrc + p.nsplit - 1) / p.nsplit;
    p.split = ((p.split + kFlowTile - 1) / kFlowTile) * kFlowTile;
    p.nsplit = std::max(1, (nsrc + p.split - 1) / p.split);
    return p;
}

template <typename T>
int falloc(T **p, size_t n) {
    *p = nullptr;
    CF_CUDA(cudaMalloc(reinterpret_cast<void **>(p), std::max<size_t>(n, 1) * sizeof(T)));
    return CF_OK;
}

int flow_run(cf_flow *h, const float *xf, int nf, const float *xs, const float *fs, int ns, int ns_pb,
             const float *xb, const float *fb, int nb, int nb_pb, const float *xbod, float *v, cudaStream_t st) {
    const int nsrc = ns + nb;
    if (nf == 0) return CF_OK;
    if (nsrc == 0) {
        CF_CUDA(cudaMemsetAsync(v, 0, sizeof(float) * 3 * nf, st));
        return CF_OK;
    }
    const bool net = h->cfg.remove_net_force != 0;
    flow_pack_kernel<<<(nsrc + 255) / 256, 256, 0, st>>>(xs, fs, ns, ns_pb, xb, fb, nb, nb_pb, net ? xbod : nullptr,
                                                         h->sx, h->sf, h->st, h->sb);
    CF_CHECK_LAUNCH("flow_pack_kernel");
    const FlowPlan pl = flow_plan(nf, nsrc, h->num_sms);
    CF_REQUIRE(static_cast<size_t>(nf) * pl.nsplit <= h->partial_cap, "cf_flow: scratch too small");
    FlowParams p{xf, h->sx, h->sf, h->st, h->sb, h->partial, nf, nsrc, pl.split, pl.nsplit};
    const dim3 grid(pl.tiles, pl.nsplit);
    const bool wall = nb_pb == 0;  // no blobs: half-space data (flow_field_evaluator.cu:75-78)
    if (wall && net) flow_tile_kernel<true, true><<<grid, kFlowThreads, 0, st>>>(p, ns);
    else if (wall) flow_tile_kernel<true, false><<<grid, kFlowThreads, 0, st>>>(p, ns);
    else if (net) flow_tile_kernel<false, true><<<grid, kFlowThreads, 0, st>>>(p, ns);
    else flow_tile_kernel<false, false><<<grid, kFlowThreads, 0, st>>>(p, ns);
    CF_CHECK_LAUNCH("flow_tile_kernel");
    const double prefac = 1.0 / (8.0 * 3.14159265358979323846 * h->cfg.mu);
    flow_reduce_kernel<<<(nf + 7) / 8, 256, 0, st>>>(h->partial, nf, pl.nsplit, prefac, v);
    CF_CHECK_LAUNCH("flow_reduce_kernel");
    return CF_OK;
}

int flow_check(cf_flow *h, int nf, int ns, int ns_pb, int nb, int nb_pb, const char *who) {
    CF_REQUIRE(h, "%s: null handle", who);
    CF_REQUIRE(nf >= 0 && nf <= h->cfg.max_flow, "%s: n_flow %d outside [0, %d]", who, nf, h->cfg.max_flow);
    CF_REQUIRE(ns >= 0 && ns <= h->cfg.max_seg, "%s: n_seg %d outside [0, %d]", who, ns, h->cfg.max_seg);
    CF_REQUIRE(nb >= 0 && nb <= h->cfg.max_blob, "%s: n_blob %d outside [0, %d]", who, nb, h->cfg.max_blob);
    CF_REQUIRE(ns == 0 || (ns_pb >= 1 && ns % ns_pb == 0), "%s: n_seg must be a multiple of n_seg_per_body", who);
    CF_REQUIRE(nb == 0 || (nb_pb >= 1 && nb % nb_pb == 0), "%s: n_blob must be a multiple of n_blob_per_body", who);
    const int bodies = std::max(ns ? ns / ns_pb : 0, nb ? nb / nb_pb : 0);
    CF_REQUIRE(bodies <= h->max_bodies, "%s: %d bodies exceed max_bodies %d", who, bodies, h->max_bodies);
    return CF_OK;
}

}  // namespace
}  // namespace cufil

using namespace cufil;

extern "C" int cf_flow_destroy(cf_flow *h) {
    if (!h) return CF_OK;
    cudaSetDevice(h->cfg.device);
    for (void *p : {(void *)h->sx, (void *)h->sf, (void *)h->st, (void *)h->sb, (void *)h->partial,
                    (void *)h->hx_flow, (void *)h->hv_flow, (void *)h->hx_segs, (void *)h->hf_segs,
                    (void *)h->hx_blobs, (void *)h->hf_blobs, (void *)h->hx_bodies})
        if (p) cudaFree(p);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return CF_OK;
}

extern "C" int cf_flow_create(const cf_flow_config *cfg, cf_flow **out) {
    clear_error();
    CF_REQUIRE(cfg && out, "cf_flow_create: null argument");
    *out = nullptr;
    CF_REQUIRE(cfg->max_flow >= 1 && cfg->max_seg >= 0 && cfg->max_blob >= 0 && cfg->max_bodies >= 1,
               "cf_flow_create: bad sizes (max_flow %d, max_seg %d, max_blob %d, max_bodies %d)", cfg->max_flow,
               cfg->max_seg, cfg->max_blob, cfg->max_bodies);
    CF_REQUIRE(cfg->mu > 0.0, "cf_flow_create: mu must be positive");
    CF_CUDA(cudaSetDevice(cfg->device));
    cf_flow *h = new (std::nothrow) cf_flow();
    if (!h) return set_error(CF_ENOMEM, "cf_flow_create: host allocation failed");
    h->cfg = *cfg;
    h->max_bodies = cfg->max_bodies;
    int rc = CF_OK;
    do {
        if ((rc = cuda_status(cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, cfg->device),
                              "cudaDeviceGetAttribute", __FILE__, __LINE__)))
            break;
        if ((rc = cuda_status(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate",
                              __FILE__, __LINE__)))
            break;
        const size_t nsrc = static_cast<size_t>(cfg->max_seg) + cfg->max_blob;
        // flow_plan keeps tiles * nsplit near 8 blocks per SM, so nf * nsplit stays below this bound
        h->partial_cap =
            static_cast<size_t>(2 * 4 * h->num_sms + 1) * kFlowTargets + 2 * static_cast<size_t>(cfg->max_flow);
        if ((rc = falloc(&h->sx, nsrc)) || (rc = falloc(&h->sf, nsrc)) || (rc = falloc(&h->st, nsrc)) ||
            (rc = falloc(&h->sb, nsrc)) || (rc = falloc(&h->partial, h->partial_cap)) ||
            (rc = falloc(&h->hx_flow, 3 * static_cast<size_t>(cfg->max_flow))) ||
            (rc = falloc(&h->hv_flow, 3 * static_cast<size_t>(cfg->max_flow))) ||
            (rc = falloc(&h->hx_segs, 3 * static_cast<size_t>(cfg->max_seg))) ||
            (rc = falloc(&h->hf_segs, 6 * static_cast<size_t>(cfg->max_seg))) ||
            (rc = falloc(&h->hx_blobs, 3 * static_cast<size_t>(cfg->max_blob))) ||
            (rc = falloc(&h->hf_blobs, 3 * static_cast<size_t>(cfg->max_blob))) ||
            (rc = falloc(&h->hx_bodies, 3 * static_cast<size_t>(cfg->max_bodies))))
            break;
    } while (0);
    if (rc != CF_OK) {
        cf_flow_destroy(h);
        return rc;
    }
    *out = h;
    return CF_OK;
}

extern "C" int cf_flow_velocities_device(cf_flow *h, const float *d_x_flow, int n_flow, const float *d_x_segs,
                                         const float *d_f_segs, int n_seg, int n_seg_per_body, const float *d_x_blobs,
                                         const float *d_f_blobs, int n_blob, int n_blob_per_body,
                                         const float *d_x_bodies, float *d_v_flow, void *stream) {
    clear_error();
    CF_TRY(flow_check(h, n_flow, n_seg, n_seg_per_body, n_blob, n_blob_per_body, "cf_flow_velocities_device"));
    CF_REQUIRE(!n_flow || (d_x_flow && d_v_flow), "cf_flow_velocities_device: missing flow-point buffers");
    CF_REQUIRE(!n_seg || (d_x_segs && d_f_segs), "cf_flow_velocities_device: missing segment buffers");
    CF_REQUIRE(!n_blob || (d_x_blobs && d_f_blobs), "cf_flow_velocities_device: missing blob buffers");
    CF_REQUIRE(!h->cfg.remove_net_force || d_x_bodies, "cf_flow_velocities_device: remove_net_force needs bodies");
    CF_CUDA(cudaSetDevice(h->cfg.device));
    return flow_run(h, d_x_flow, n_flow, d_x_segs, d_f_segs, n_seg, n_seg_per_body, d_x_blobs, d_f_blobs, n_blob,
                    n_blob_per_body, d_x_bodies, d_v_flow, static_cast<cudaStream_t>(stream));
}

extern "C" int cf_flow_velocities(cf_flow *h, const float *x_flow, int n_flow, const float *x_segs,
                                  const float *f_segs, int n_seg, int n_seg_per_body, const float *x_blobs,
                                  const float *f_blobs, int n_blob, int n_blob_per_body, const float *x_bodies,
                                  float *v_flow) {
    clear_error();
    CF_TRY(flow_check(h, n_flow, n_seg, n_seg_per_body, n_blob, n_blob_per_body, "cf_flow_velocities"));
    CF_REQUIRE(!n_flow || (x_flow && v_flow), "cf_flow_velocities: missing flow-point arrays");
    CF_REQUIRE(!n_seg || (x_segs && f_segs), "cf_flow_velocities: missing segment arrays");
    CF_REQUIRE(!n_blob || (x_blobs && f_blobs), "cf_flow_velocities: missing blob arrays");
    CF_REQUIRE(!h->cfg.remove_net_force || x_bodies, "cf_flow_velocities: remove_net_force needs bodies");
    CF_CUDA(cudaSetDevice(h->cfg.device));
    cudaStream_t st = h->stream;
    const int bodies = std::max(n_seg ? n_seg / n_seg_per_body : 0, n_blob ? n_blob / n_blob_per_body : 0);
    if (n_flow) CF_CUDA(cudaMemcpyAsync(h->hx_flow, x_flow, sizeof(float) * 3 * n_flow, cudaMemcpyHostToDevice, st));
    if (n_seg) {
        CF_CUDA(cudaMemcpyAsync(h->hx_segs, x_segs, sizeof(float) * 3 * n_seg, cudaMemcpyHostToDevice, st));
        CF_CUDA(cudaMemcpyAsync(h->hf_segs, f_segs, sizeof(float) * 6 * n_seg, cudaMemcpyHostToDevice, st));
    }
    if (n_blob) {
        CF_CUDA(cudaMemcpyAsync(h->hx_blobs, x_blobs, sizeof(float) * 3 * n_blob, cudaMemcpyHostToDevice, st));
        CF_CUDA(cudaMemcpyAsync(h->hf_blobs, f_blobs, sizeof(float) * 3 * n_blob, cudaMemcpyHostToDevice, st));
    }
    if (x_bodies && bodies)
        CF_CUDA(cudaMemcpyAsync(h->hx_bodies, x_bodies, sizeof(float) * 3 * bodies, cudaMemcpyHostToDevice, st));
    CF_TRY(flow_run(h, h->hx_flow, n_flow, h->hx_segs, h->hf_segs, n_seg, n_seg_per_body, h->hx_blobs, h->hf_blobs,
                    n_blob, n_blob_per_body, x_bodies ? h->hx_bodies : nullptr, h->hv_flow, st));
    if (n_flow) CF_CUDA(cudaMemcpyAsync(v_flow, h->hv_flow, sizeof(float) * 3 * n_flow, cudaMemcpyDeviceToHost, st));
    CF_CUDA(cudaStreamSynchronize(st));
    return CF_OK;
}

// sim.cu -- cf_sim / cf_batch: the device-resident implicit step for
// prescribed cilia on a wall, for one array or a batch of independent arrays.
//
// Host side of the generic mobility_solver layer
// (src/cilia/mobility/mobility_solver.{hpp,cpp}) for CILIA_TYPE 3 on an
// INFINITE_PLANE_WALL with SOLVER_TYPE 1: one step is
//   kinematics -> RHS -> r0 = b - A x0 -> GMRES loop -> x = x0 + P^{-1} Q y
// and is captured once as a CUDA graph whose GMRES loop is a conditional
// WHILE node driven from the device, so a time step costs one graph launch
// and no host synchronisation.  The reference instead runs GMRES on the host
// with one H2D copy, one kernel and one D2H copy per iteration
// (mobility_solver.cpp:1910-1913, 2102).
//
// A batch runs many independent arrays (periodic-orbit / bisection sweeps)
// through the same graph: every stage is one kernel over all arrays, the pair
// product is one grid-stride launch over the (array, target tile, source tile)
// work list of every array, and arrays whose GMRES stopped are masked out of
// the remaining iterations.  A single array (cf_sim) is a batch of one.
#include "common.cuh"
#include "rpy_kernels.cuh"
#include "sim_kernels.cuh"
#include "patch_kernels.cuh"
#include "learned_kernels.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

using namespace cufil;

namespace cufil {
int mlp_forward_dev(cf_mlp *h, const float *x, int n, float *y, cudaStream_t st);
int mlp_dims(const cf_mlp *h, int *in, int *out, int *max_batch);
}  // namespace cufil

namespace {
constexpr int kIterLogCap = 4096;  // steps remembered by the iteration log (per array)
constexpr int kMinDotsChunk = 1024;

// Launch shapes chosen by the autotuner (or the defaults).
struct Tuning {
    int pair_ctas_per_sm = 8;   // pair kernel residency target
    int dots_chunk = 4096;      // rows per dot-product item
    int dots_blocks_per_sm = 2;
    int update_blocks_per_sm = 8;
    int update_rows = 32;       // rows per update / combine tile (32, 64, 128 or 256)
};
}  // namespace

struct Engine {
    int device = 0;
    int num_sms = CF_B200_SMS;
    int B = 0;
    cf_sim_config common{};
    std::vector<ArrayInfo> arr;  // host copy of the placement table
    cudaStream_t stream = nullptr;
    cudaStream_t cap_stream = nullptr;  // captures the loop body
    SimDev d{};
    SymBatchParams pair{};
    int pair_grid = 1, dots_grid = 1, update_grid = 1, epi_grid = 1;
    Tuning tune;
    ArrayInfo *d_arr = nullptr;
    int *d_chunk_arr = nullptr;
    int *err = nullptr;
    int fil_threads = 64;
    size_t kin_smem = 0, pre_smem = 0, givens_smem = 0;
    bool use_graph = true;
    bool stepped = false;
    long long geometry = 0;         // kinematics launches so far (the geometry's version)
    long long refresh_geometry = -1; // geometry version of the current patch inverses
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphConditionalHandle handle = 0;
    // line-patch preconditioner
    bool line = false;
    PatchDev P{};
    long long patch_floats = 0;
    int refresh_every = 1, last_refresh_nt = -1, mob_grid = 1, gj_rounds = 0, gj_cols = 1;
    int apply_chunks = 1, gj_update_grid = 1, rates_grid = 1;
    int arn_fils = 1;  // blocks per patch of patch_arnoldi_kernel (largest filament count)
    size_t arn_smem = 0;
    bool refreshed_last = false;
    size_t apply_smem = 0;
    cudaGraph_t rgraph = nullptr;
    cudaGraphExec_t rexec = nullptr;
    // learned correction
    bool learned = false;
    cf_mlp *net = nullptr;
    float *seg_out = nullptr;  // staging of cf_sim_step_io's segment outputs [9N]
    // training-pair collection (host-driven steps only)
    float *cx = nullptr, *ct = nullptr;
    int c_max = 0, c_pairs = 0;
    std::vector<void *> allocations;
};

struct cf_sim : Engine {};
struct cf_batch : Engine {};

namespace {

template <typename T>
int eng_alloc(Engine *e, T **p, size_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    void *q = nullptr;
    CF_CUDA(cudaMalloc(&q, n * sizeof(T)));
    e->allocations.push_back(q);
    *p = static_cast<T *>(q);
    return CF_OK;
}

template <typename T>
int eng_upload(Engine *e, T **p, const T *host, size_t n) {
    CF_TRY(eng_alloc(e, p, n));
    if (host && n) CF_CUDA(cudaMemcpy(*p, host, n * sizeof(T), cudaMemcpyHostToDevice));
    return CF_OK;
}

// Fulford & Blake beat tables as used by the reference (filament.cpp:686-747
// for SHAPE_SEQUENCE 1, :893-958 for SHAPE_SEQUENCE 4), laid out [mode][degree].
BeatCoeffs beat_table(int beat) {
    BeatCoeffs b{};
    if (beat == CF_BEAT_FULFORD_BLAKE) {
        const double Ax[4][3] = {{9.7204e-01, -2.8315e-01, 4.9243e-02}, {-1.8466e-02, -1.2926e-01, 2.6981e-01},
                                 {1.6209e-01, -3.4983e-01, 1.9082e-01}, {1.0259e-02, 3.5907e-02, -6.8736e-02}};
        const double Ay[4][3] = {{-3.3547e-01, 4.0369e-01, 1.0362e-01}, {4.0318e-01, -1.5553e+00, 7.3455e-01},
                                 {-9.9513e-02, 3.2829e-02, -1.2106e-01}, {8.1046e-02, -3.0982e-01, 1.4568e-01}};
        const double Bx[3][3] = {{1.9697e-01, -5.1193e-01, 3.4778e-01}, {-5.1295e-02, 4.3396e-01, -3.3547e-01},
                                 {1.2311e-02, 1.4157e-01, -1.1695e-01}};
        const double By[3][3] = {{2.9136e-01, 1.0721e+00, -1.0433e+00}, {6.1554e-03, 3.2521e-01, -2.8315e-01},
                                 {-6.0528e-02, 2.3185e-01, -2.0108e-01}};
        std::memcpy(b.Ax, Ax, sizeof(Ax));
        std::memcpy(b.Ay, Ay, sizeof(Ay));
        std::memcpy(b.Bx, Bx, sizeof(Bx));
        std::memcpy(b.By, By, sizeof(By));
        b.c0 = 1.0;
    } else {
        const double Ax[4][3] = {{1.895, -0.552, 0.096}, {-0.018, -0.126, 0.263}, {0.158, -0.341, 0.186},
                                 {0.010, 0.035, -0.067}};
        const double Ay[4][3] = {{-0.654, 0.787, 0.202}, {0.393, -1.516, 0.716}, {-0.097, 0.032, -0.118},
                                 {0.079, -0.302, 0.142}};
        const double Bx[3][3] = {{0.192, -0.499, 0.339}, {-0.050, 0.423, -0.327}, {0.012, 0.138, -0.114}};
        const double By[3][3] = {{0.284, 1.045, -1.017}, {0.006, 0.317, -0.276}, {-0.059, 0.226, -0.196}};
        std::memcpy(b.Ax, Ax, sizeof(Ax));
        std::memcpy(b.Ay, Ay, sizeof(Ay));
        std::memcpy(b.Bx, Bx, sizeof(Bx));
        std::memcpy(b.By, By, sizeof(By));
        b.c0 = 0.5;
    }
    return b;
}

// Pair-kernel grid: every warp gets the same number of (array, tile, tile) items.
int pair_grid_for(long long items, int num_sms, int ctas_per_sm) {
    const long long max_warps = static_cast<long long>(std::max(1, num_sms)) * std::max(1, ctas_per_sm) * 4;
    const long long per_warp = std::max(1LL, (items + max_warps - 1) / max_warps);
    const long long warps = (items + per_warp - 1) / per_warp;
    return static_cast<int>(std::max(1LL, (warps + 3) / 4));
}

// Re-derives the chunk tables and launch grids from the tuning and uploads
// the placement table; drops the captured graph (it holds the old values).
int apply_tuning(Engine *e, const Tuning &t) {
    SimDev &d = e->d;
    e->tune = t;
    d.dots_chunk = t.dots_chunk;
    int c = 0;
    std::vector<int> chunk_arr;
    for (int b = 0; b < e->B; ++b) {
        ArrayInfo &a = e->arr[b];
        a.chunk0 = c;
        a.nchunk = (a.n + t.dots_chunk - 1) / t.dots_chunk;
        for (int q = 0; q < a.nchunk; ++q) chunk_arr.push_back(b);
        c += a.nchunk;
    }
    d.C_tot = c;
    CF_CUDA(cudaMemcpy(e->d_arr, e->arr.data(), sizeof(ArrayInfo) * e->B, cudaMemcpyHostToDevice));
    CF_CUDA(cudaMemcpy(e->d_chunk_arr, chunk_arr.data(), sizeof(int) * c, cudaMemcpyHostToDevice));
    e->pair_grid = pair_grid_for(e->pair.items, e->num_sms, t.pair_ctas_per_sm);
    e->dots_grid = std::max(1, e->num_sms * t.dots_blocks_per_sm);
    const long long ntiles = d.nrows / t.update_rows;
    e->update_grid = static_cast<int>(std::max(1LL, std::min(ntiles, 1LL * e->num_sms * t.update_blocks_per_sm)));
    if (e->exec) cudaGraphExecDestroy(e->exec);
    if (e->graph) cudaGraphDestroy(e->graph);
    e->exec = nullptr;
    e->graph = nullptr;
    return CF_OK;
}

int launch_kinematics(Engine *e, cudaStream_t st) {
    kinematics_kernel<<<e->d.F, e->fil_threads, e->kin_smem, st>>>(e->d);
    CF_CHECK_LAUNCH("kinematics_kernel");
    e->geometry += 1;
    return CF_OK;
}

int launch_step_begin(Engine *e, int nt, cudaStream_t st) {
    step_begin_kernel<<<1, 256, 0, st>>>(e->d, nt);
    CF_CHECK_LAUNCH("step_begin_kernel");
    return CF_OK;
}

int launch_matvec_tail(Engine *e, const double *v, double *out, cudaStream_t st) {
    CF_TRY(rpy_launch_sym_batch(e->pair, e->pair_grid, st));
    CF_CUDA(launch_chained(saddle_epilogue_kernel, dim3(e->epi_grid), dim3(32 * kEpiWarps), 0, st, e->d, v, out));
    return CF_OK;
}

template <int ROWS>
int launch_update_t(Engine *e, const double *h, int final_pass, cudaGraphConditionalHandle hc, int grid,
                    cudaStream_t st) {
    CF_CUDA(launch_chained(update_kernel<ROWS>, dim3(grid), dim3(256), final_pass ? e->givens_smem : 0, st, e->d, h,
                           final_pass, hc));
    return CF_OK;
}

int launch_update(Engine *e, const double *h, int final_pass, cudaGraphConditionalHandle hc, cudaStream_t st,
                  int rows, int grid) {
    switch (rows) {
        case 32: return launch_update_t<32>(e, h, final_pass, hc, grid, st);
        case 64: return launch_update_t<64>(e, h, final_pass, hc, grid, st);
        case 128: return launch_update_t<128>(e, h, final_pass, hc, grid, st);
        case 256: return launch_update_t<256>(e, h, final_pass, hc, grid, st);
        default: return set_error(CF_EINVAL, "update tile of %d rows not built", rows);
    }
}

int launch_combine(Engine *e, cudaStream_t st) {
    const int grid = e->update_grid;
    switch (e->tune.update_rows) {
        case 32: combine_kernel<32><<<grid, 256, 0, st>>>(e->d); break;
        case 64: combine_kernel<64><<<grid, 256, 0, st>>>(e->d); break;
        case 128: combine_kernel<128><<<grid, 256, 0, st>>>(e->d); break;
        case 256: combine_kernel<256><<<grid, 256, 0, st>>>(e->d); break;
        default: return set_error(CF_EINVAL, "combine tile of %d rows not built", e->tune.update_rows);
    }
    CF_CHECK_LAUNCH("combine_kernel");
    return CF_OK;
}

// Assembles and inverts every patch block for the current kinematics.
int launch_refresh(Engine *e, cudaStream_t st) {
    const PatchDev &P = e->P;
    e->refresh_geometry = e->geometry;
    CF_CUDA(cudaMemsetAsync(P.counter, 0, sizeof(int) * e->gj_rounds, st));
    patch_mobility_kernel<<<dim3(e->mob_grid, P.np), 256, 0, st>>>(e->d, P);
    CF_CHECK_LAUNCH("patch_mobility_kernel");
    patch_rates_kernel<<<dim3(e->rates_grid, P.np), 256, 0, st>>>(e->d, P);
    CF_CHECK_LAUNCH("patch_rates_kernel");
    gj_pivot_kernel<<<P.np, 256, 0, st>>>(P, 0);  // later pivot blocks: inverted inside the previous update
    CF_CHECK_LAUNCH("gj_pivot_kernel");
    for (int K = 0; K < e->gj_rounds; ++K) {
        CF_CUDA(launch_chained(gj_prep_kernel, dim3(e->gj_cols, P.np), dim3(256), 0, st, P, K));
        CF_CUDA(launch_chained(gj_update_kernel, dim3(e->gj_update_grid), dim3(256), kUpdateSmem, st, P, K, e->gj_cols,
                               P.counter + K));
    }
    return CF_OK;
}

int refresh_launches(const Engine *e) { return e->line ? 3 + 2 * e->gj_rounds : 0; }

int launch_patch_apply(Engine *e, const double *in, double *out, int masked, cudaStream_t st) {
    patch_apply_kernel<<<dim3(e->apply_chunks, e->P.np), kApplyThreads, e->apply_smem, st>>>(e->d, e->P, in, out,
                                                                                            masked);
    CF_CHECK_LAUNCH("patch_apply_kernel");
    return CF_OK;
}

// Refreshes the patch inverses when the step calls for it (graph-captured once).
int maybe_refresh(Engine *e, int nt) {
    e->refreshed_last = false;
    if (!e->line) return CF_OK;
    const bool due = e->last_refresh_nt < 0 || nt < e->last_refresh_nt || nt - e->last_refresh_nt >= e->refresh_every;
    if (!due) return CF_OK;
    if (e->use_graph && !e->rexec) {
        CF_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
        const int rc = launch_refresh(e, e->stream);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
        if (rc != CF_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        CF_TRY(cuda_status(ce, "cudaStreamEndCapture(refresh)", __FILE__, __LINE__));
        e->rgraph = g;
        CF_CUDA(cudaGraphInstantiate(&e->rexec, e->rgraph, 0));
    }
    if (e->rexec) CF_CUDA(cudaGraphLaunch(e->rexec, e->stream));
    else CF_TRY(launch_refresh(e, e->stream));
    e->refresh_geometry = e->geometry;
    e->last_refresh_nt = nt;
    e->refreshed_last = true;
    return CF_OK;
}

int launch_prologue(Engine *e, cudaGraphConditionalHandle h, cudaStream_t st) {
    rhs_kernel<<<e->d.F, e->fil_threads, 0, st>>>(e->d);
    CF_CHECK_LAUNCH("rhs_kernel");
    CF_TRY(launch_matvec_tail(e, e->d.sol, e->d.w, st));
    residual_decide_kernel<<<e->d.F, e->fil_threads, 0, st>>>(e->d, h);
    CF_CHECK_LAUNCH("residual_decide_kernel");
    return CF_OK;
}

int launch_body(Engine *e, cudaGraphConditionalHandle h, cudaStream_t st) {
    if (e->line) {  // Q_k, z = P^-1 Q_k and the packed forces in one launch
        CF_CUDA(launch_chained(patch_arnoldi_kernel, dim3(kArnParts * e->arn_fils, e->P.np), dim3(kArnThreads),
                               e->arn_smem, st, e->d, e->P, h));
    } else {
        arnoldi_precond_kernel<<<e->d.F, e->fil_threads, e->pre_smem, st>>>(e->d, h);
        CF_CHECK_LAUNCH("arnoldi_precond_kernel");
    }
    if (e->learned) {  // z = P(q) + s * net(features(q)), P block-diagonal or the line patches, then the rows
                       // the previous kernel left to us
        learned_features_kernel<<<e->d.F, e->fil_threads, 0, st>>>(e->d, e->d.t, e->d.lx, e->d.lscale);
        CF_CHECK_LAUNCH("learned_features_kernel");
        CF_TRY(mlp_forward_dev(e->net, e->d.lx, e->d.F, e->d.ly, st));
        learned_correct_kernel<<<e->d.F, e->fil_threads, 0, st>>>(e->d, e->d.ly, e->d.lscale, e->line ? 1 : 0);
        CF_CHECK_LAUNCH("learned_correct_kernel");
        pack_rows_kernel<<<e->d.F, e->fil_threads, 0, st>>>(e->d, e->d.z, e->d.w);
        CF_CHECK_LAUNCH("pack_rows_kernel");
    }
    CF_TRY(launch_matvec_tail(e, e->d.z, e->d.w, st));
    if (e->cx && e->c_pairs < e->c_max) {  // one training pair (w = A z, z) of the plain solver
        const size_t F = e->d.F;
        learned_features_kernel<<<e->d.F, e->fil_threads, 0, st>>>(e->d, e->d.w,
                                                                   e->cx + e->c_pairs * F * e->d.lin, e->d.lscale);
        CF_CHECK_LAUNCH("learned_features_kernel");
        if (e->line) {
            CF_TRY(launch_patch_apply(e, e->d.w, e->d.t, 0, st));
        } else {
            precond_kernel<<<e->d.F, e->fil_threads, e->pre_smem, st>>>(e->d, e->d.w, e->d.t);
            CF_CHECK_LAUNCH("precond_kernel");
        }
        learned_target_kernel<<<e->d.F, e->fil_threads, 0, st>>>(e->d, e->d.z, e->d.t, e->d.lscale,
                                                                 e->ct + e->c_pairs * F * e->d.lout);
        CF_CHECK_LAUNCH("learned_target_kernel");
        e->c_pairs += 1;
    }
    CF_CUDA(launch_chained(dots_kernel, dim3(e->dots_grid), dim3(256), 0, st, e->d, e->d.h1));
    CF_TRY(launch_update(e, e->d.h1, 0, h, st, e->tune.update_rows, e->update_grid));
    CF_CUDA(launch_chained(dots_kernel, dim3(e->dots_grid), dim3(256), 0, st, e->d, e->d.h2));
    return launch_update(e, e->d.h2, 1, h, st, e->tune.update_rows, e->update_grid);
}

int launch_finish(Engine *e, cudaStream_t st) {
    backsub_kernel<<<e->B, 256, sizeof(double) * (e->d.mi_max + 1), st>>>(e->d);
    CF_CHECK_LAUNCH("backsub_kernel");
    CF_TRY(launch_combine(e, st));
    if (e->line && !e->d.flexible) CF_TRY(launch_patch_apply(e, e->d.t, e->d.z, 0, st));
    finish_kernel<<<e->d.F, e->fil_threads, e->pre_smem, st>>>(e->d);
    CF_CHECK_LAUNCH("finish_kernel");
    return CF_OK;
}

// Captures prologue -> WHILE(body) -> finish into one executable graph.
int build_graph(Engine *e) {
    cudaStream_t st = e->stream;
    CF_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = CF_OK;
    cudaGraph_t g = nullptr;
    do {
        cudaStreamCaptureStatus cs;
        const cudaGraphNode_t *deps = nullptr;
        size_t ndeps = 0;
        if ((rc = cuda_status(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &ndeps),
                              "cudaStreamGetCaptureInfo", __FILE__, __LINE__)))
            break;
        if ((rc = cuda_status(cudaGraphConditionalHandleCreate(&e->handle, g, 0, cudaGraphCondAssignDefault),
                              "cudaGraphConditionalHandleCreate", __FILE__, __LINE__)))
            break;
        if ((rc = launch_prologue(e, e->handle, st))) break;
        if ((rc = cuda_status(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &ndeps),
                              "cudaStreamGetCaptureInfo", __FILE__, __LINE__)))
            break;
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = e->handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t wnode;
        if ((rc = cuda_status(cudaGraphAddNode(&wnode, g, deps, ndeps, &cp), "cudaGraphAddNode", __FILE__,
                              __LINE__)))
            break;
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        if ((rc = cuda_status(cudaStreamUpdateCaptureDependencies(st, &wnode, 1, cudaStreamSetCaptureDependencies),
                              "cudaStreamUpdateCaptureDependencies", __FILE__, __LINE__)))
            break;
        if ((rc = cuda_status(cudaStreamBeginCaptureToGraph(e->cap_stream, body, nullptr, nullptr, 0,
                                                            cudaStreamCaptureModeThreadLocal),
                              "cudaStreamBeginCaptureToGraph", __FILE__, __LINE__)))
            break;
        rc = launch_body(e, e->handle, e->cap_stream);
        cudaGraph_t body_out = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(e->cap_stream, &body_out);
        if (rc) break;
        if ((rc = cuda_status(e2, "cudaStreamEndCapture(body)", __FILE__, __LINE__))) break;
        if ((rc = launch_finish(e, st))) break;
    } while (0);
    cudaGraph_t full = nullptr;
    cudaError_t ce = cudaStreamEndCapture(st, &full);
    if (rc) {
        if (full) cudaGraphDestroy(full);
        return rc;
    }
    CF_TRY(cuda_status(ce, "cudaStreamEndCapture", __FILE__, __LINE__));
    e->graph = full;
    CF_CUDA(cudaGraphInstantiate(&e->exec, e->graph, 0));
    return CF_OK;
}

int check_err_flag(Engine *e) {
    int flags = 0;
    CF_CUDA(cudaMemcpy(&flags, e->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (flags) {
        CF_CUDA(cudaMemset(e->err, 0, sizeof(int)));
        return set_error(CF_TIMEOUT, "sim: a bounded device wait gave up (flags 0x%x)", flags);
    }
    return CF_OK;
}

int read_loop(Engine *e, LoopCtl *out) {
    CF_CUDA(cudaMemcpyAsync(out, e->d.lc, sizeof(LoopCtl), cudaMemcpyDeviceToHost, e->stream));
    CF_CUDA(cudaStreamSynchronize(e->stream));
    return check_err_flag(e);
}

int read_ctls(Engine *e, std::vector<GmresCtl> &out) {
    out.resize(e->B);
    CF_CUDA(cudaMemcpyAsync(out.data(), e->d.ctl, sizeof(GmresCtl) * e->B, cudaMemcpyDeviceToHost, e->stream));
    CF_CUDA(cudaStreamSynchronize(e->stream));
    return check_err_flag(e);
}

int iters_of(const GmresCtl &c) {
    return (c.status == kGmresConverged || c.status == kGmresMaxIter) ? c.iters : 0;
}

int status_of(const GmresCtl &c, int b, int B) {
    char where[48] = "";
    if (B > 1) std::snprintf(where, sizeof(where), " (array %d)", b);
    switch (c.status) {
        case kGmresMaxIter:
            return set_error(CF_NOT_CONVERGED, "GMRES stopped at its cap%s: %d iterations, relative residual %.3e",
                             where, c.iters, c.relres);
        case kGmresNonFinite:
            return set_error(CF_NONFINITE, "GMRES met a non-finite value%s (relative residual %.3e)", where,
                             c.relres);
        default:
            return CF_OK;
    }
}

// Worst status over the arrays: a non-finite array outranks a capped one.
int batch_status(const std::vector<GmresCtl> &c) {
    int rc = CF_OK;
    for (size_t b = 0; b < c.size(); ++b) {
        if (c[b].status == kGmresNonFinite) return status_of(c[b], static_cast<int>(b), static_cast<int>(c.size()));
        if (c[b].status == kGmresMaxIter && rc == CF_OK)
            rc = status_of(c[b], static_cast<int>(b), static_cast<int>(c.size()));
    }
    return rc;
}

int run_step(Engine *e, int nt) {
    CF_REQUIRE(!e->learned || e->net, "CF_PRECOND_LEARNED: no network attached (cf_sim_set_network)");
    CF_TRY(launch_step_begin(e, nt, e->stream));
    CF_TRY(launch_kinematics(e, e->stream));
    CF_TRY(maybe_refresh(e, nt));
    e->stepped = true;
    if (e->use_graph && !e->cx) {
        if (!e->exec) {
            int rc = build_graph(e);
            if (rc != CF_OK) {
                // Conditional graph nodes unavailable: fall back to the host-driven loop.
                cudaGetLastError();
                e->use_graph = false;
            }
        }
        if (e->use_graph) {
            CF_CUDA(cudaGraphLaunch(e->exec, e->stream));
            return CF_OK;
        }
    }
    CF_TRY(launch_prologue(e, 0, e->stream));
    LoopCtl lc;
    CF_TRY(read_loop(e, &lc));
    int guard = 0;
    while (lc.cond && guard++ <= e->d.mi_max) {
        CF_TRY(launch_body(e, 0, e->stream));
        CF_TRY(read_loop(e, &lc));
    }
    return launch_finish(e, e->stream);
}

bool same_table(const double *a, const double *b, int n) {
    if (a == b) return true;
    if (!a || !b) return false;
    return std::memcmp(a, b, sizeof(double) * n) == 0;
}

int validate(const cf_sim_config *cfg, const char *who) {
    CF_REQUIRE(cfg->n_fil > 0 && cfg->n_seg >= 2 && cfg->n_seg <= 256,
               "%s: need n_fil > 0 and 2 <= n_seg <= 256 (got %d, %d)", who, cfg->n_fil, cfg->n_seg);
    CF_REQUIRE(static_cast<long long>(cfg->n_fil) * cfg->n_seg < (1LL << 26), "%s: too many segments", who);
    CF_REQUIRE(cfg->beat == CF_BEAT_FULFORD_BLAKE || cfg->beat == CF_BEAT_FULFORD_BLAKE_ORIGINAL,
               "%s: unknown beat %d", who, cfg->beat);
    CF_REQUIRE(cfg->precond == CF_PRECOND_NONE || cfg->precond == CF_PRECOND_BLOCK_DIAG ||
                   cfg->precond == CF_PRECOND_LINE || cfg->precond == CF_PRECOND_LEARNED ||
                   cfg->precond == CF_PRECOND_LEARNED_LINE,
               "%s: preconditioner %d not available in this entry point", who, cfg->precond);
    CF_REQUIRE(cfg->line_patch >= 0 && cfg->line_patch <= 32, "%s: line_patch must be 0..32 (got %d)", who,
               cfg->line_patch);
    CF_REQUIRE(cfg->precond_refresh >= 0, "%s: precond_refresh must be >= 0", who);
    CF_REQUIRE(cfg->dt > 0 && cfg->seg_sep > 0, "%s: dt and seg_sep must be positive", who);
    CF_REQUIRE(cfg->gmres_tol > 0 && cfg->gmres_max_iter > 0, "%s: bad GMRES tolerance / cap", who);
    CF_REQUIRE(cfg->base_pos, "%s: base_pos is required", who);
    CF_REQUIRE(!cfg->dynamic_phase || (cfg->gen_phase_force_refs && cfg->n_gen_phase_refs >= 2),
               "%s: dynamic phase needs the reference generalised phase forces", who);
    CF_REQUIRE(!cfg->dynamic_angle || (cfg->gen_angle_force_refs && cfg->n_gen_angle_refs >= 2),
               "%s: dynamic angle needs the reference generalised angle forces", who);
    CF_REQUIRE(!cfg->s_values_ref || (cfg->s_ref_rows >= 1 && cfg->s_ref_cols >= 2),
               "%s: bad arclength table shape", who);
    return CF_OK;
}

// Fields every array of a batch shares with the first.
int validate_shared(const cf_sim_config &a, const cf_sim_config &c, int b) {
    const bool same = a.n_seg == c.n_seg && a.seg_sep == c.seg_sep && a.beat == c.beat &&
                      a.dynamic_phase == c.dynamic_phase && a.dynamic_angle == c.dynamic_angle && a.dt == c.dt &&
                      a.spring_factor == c.spring_factor && a.gmres_tol == c.gmres_tol &&
                      a.gmres_max_iter == c.gmres_max_iter && a.precond == c.precond &&
                      a.s_tol_factor == c.s_tol_factor && a.device == c.device &&
                      a.line_patch == c.line_patch && a.precond_refresh == c.precond_refresh &&
                      a.n_gen_phase_refs == c.n_gen_phase_refs && a.n_gen_angle_refs == c.n_gen_angle_refs &&
                      a.s_ref_rows == c.s_ref_rows && a.s_ref_cols == c.s_ref_cols &&
                      (a.s_values_ref == nullptr) == (c.s_values_ref == nullptr);
    CF_REQUIRE(same, "cf_batch_create: array %d differs from array 0 in a shared setting "
               "(segments, beat, dt, tolerance, preconditioner, tables)", b);
    CF_REQUIRE(!a.dynamic_phase || same_table(a.gen_phase_force_refs, c.gen_phase_force_refs, a.n_gen_phase_refs),
               "cf_batch_create: array %d has different generalised phase forces", b);
    CF_REQUIRE(!a.dynamic_angle || same_table(a.gen_angle_force_refs, c.gen_angle_force_refs, a.n_gen_angle_refs),
               "cf_batch_create: array %d has different generalised angle forces", b);
    CF_REQUIRE(!a.s_values_ref || same_table(a.s_values_ref, c.s_values_ref, a.s_ref_rows * a.s_ref_cols),
               "cf_batch_create: array %d has a different arclength table", b);
    return CF_OK;
}

// Line patches: within each array, filaments with equal base x (a lattice line
// along y, the beat direction of the wall frame) sorted by y and cut into
// runs of at most line_patch filaments of near-equal length.
int build_patches(Engine *e, const cf_sim_config *cfgs) {
    SimDev &d = e->d;
    const int Pmax = cfgs[0].line_patch > 0 ? cfgs[0].line_patch : 32;
    const int nl = 3 * d.nseg;
    const int nbf = nl + d.dyn_phase + d.dyn_angle;
    std::vector<int> fil0, nf, fils;
    std::vector<long long> moff, roff, rows;
    long long mo = 0, ro = 0;
    int max_n = 0, max_nf = 0;
    for (int b = 0; b < e->B; ++b) {
        const ArrayInfo &a = e->arr[b];
        const double *bp = cfgs[b].base_pos;
        std::vector<int> idx(a.F);
        for (int q = 0; q < a.F; ++q) idx[q] = q;
        std::sort(idx.begin(), idx.end(), [&](int u, int v) {
            if (bp[3 * u] != bp[3 * v]) return bp[3 * u] < bp[3 * v];
            return bp[3 * u + 1] < bp[3 * v + 1];
        });
        size_t s0 = 0;
        while (s0 < idx.size()) {
            const double x0 = bp[3 * idx[s0]];
            size_t s1 = s0 + 1;
            while (s1 < idx.size() && std::fabs(bp[3 * idx[s1]] - x0) <= 1e-6 * (1.0 + std::fabs(x0))) ++s1;
            const int L = static_cast<int>(s1 - s0);
            const int c = (L + Pmax - 1) / Pmax, base = L / c, extra = L % c;
            size_t pos = s0;
            for (int q = 0; q < c; ++q) {
                const int sz = base + (q < extra ? 1 : 0);
                fil0.push_back(static_cast<int>(fils.size()));
                nf.push_back(sz);
                const int n = sz * nbf;
                moff.push_back(mo);
                roff.push_back(ro);
                mo += static_cast<long long>(patch_ld(n)) * patch_ld(n);
                ro += n;
                max_n = std::max(max_n, n);
                max_nf = std::max(max_nf, sz);
                for (int u = 0; u < sz; ++u) {
                    const int lm = idx[pos + u];
                    fils.push_back(a.fil0 + lm);
                    const long long lam = a.voff + static_cast<long long>(nl) * lm;
                    for (int li = 0; li < nl; ++li) rows.push_back(lam + li);
                    if (a.po >= 0) rows.push_back(a.voff + a.po + lm);
                    if (a.ao >= 0) rows.push_back(a.voff + a.ao + lm);
                }
                pos += sz;
            }
            s0 = s1;
        }
    }
    PatchDev &P = e->P;
    P.np = static_cast<int>(nf.size());
    P.nbf = nbf;
    P.max_n = max_n;
    CF_TRY(eng_upload(e, const_cast<int **>(&P.fil0), fil0.data(), fil0.size()));
    CF_TRY(eng_upload(e, const_cast<int **>(&P.nf), nf.data(), nf.size()));
    CF_TRY(eng_upload(e, const_cast<int **>(&P.fils), fils.data(), fils.size()));
    CF_TRY(eng_upload(e, const_cast<long long **>(&P.moff), moff.data(), moff.size()));
    CF_TRY(eng_upload(e, const_cast<long long **>(&P.roff), roff.data(), roff.size()));
    CF_TRY(eng_upload(e, const_cast<long long **>(&P.rows), rows.data(), rows.size()));
    CF_TRY(eng_alloc(e, &P.A, static_cast<size_t>(mo)));
    CF_CUDA(cudaMemset(P.A, 0, sizeof(float) * static_cast<size_t>(mo)));  // the padding columns stay zero
    P.T = (max_n + kGjTile - 1) / kGjTile;
    const size_t split_floats = static_cast<size_t>(P.np) * P.T * 2 * tc::kOperandFloats;
    CF_TRY(eng_alloc(e, &P.csplit, split_floats));
    CF_TRY(eng_alloc(e, &P.rsplit, split_floats));
    CF_CUDA(cudaMemset(P.csplit, 0, sizeof(float) * split_floats));
    CF_CUDA(cudaMemset(P.rsplit, 0, sizeof(float) * split_floats));
    CF_TRY(eng_alloc(e, &P.dinv, static_cast<size_t>(P.np) * kGjBlock * kGjBlock));
    CF_TRY(eng_alloc(e, &P.ok, P.np));
    CF_TRY(eng_alloc(e, &P.counter, std::max(1, (max_n + kGjBlock - 1) / kGjBlock)));
    e->patch_floats = mo;
    const long long ns = static_cast<long long>(max_nf) * d.nseg;
    e->mob_grid = static_cast<int>((ns * ns + 255) / 256);
    e->gj_rounds = (max_n + kGjBlock - 1) / kGjBlock;
    const int T = (max_n + kGjTile - 1) / kGjTile;
    e->rates_grid = std::max(1, (max_n * max_nf * (nbf - nl) + 255) / 256);
    e->gj_cols = T;
    e->gj_update_grid = static_cast<int>(std::min<long long>(1LL * P.np * (T * (T + 1) / 2), 2LL * e->num_sms));
    CF_CUDA(cudaFuncSetAttribute(gj_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kUpdateSmem)));
    e->apply_chunks = (max_n + kApplyRows - 1) / kApplyRows;
    e->apply_smem = sizeof(double) * std::max(patch_ld(max_n), 3 * d.nseg);
    e->arn_fils = max_nf;
    e->arn_smem = sizeof(double) * (patch_ld(max_n) + std::max(nbf, 3 * d.nseg));
    CF_REQUIRE(e->arn_smem <= 227 * 1024, "line patches of %d unknowns exceed the shared memory of one block", max_n);
    if (e->arn_smem > 48 * 1024)
        CF_CUDA(cudaFuncSetAttribute(patch_arnoldi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(e->arn_smem)));
    if (e->apply_smem > 48 * 1024)
        CF_CUDA(cudaFuncSetAttribute(patch_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(e->apply_smem)));
    d.epi_fil_rows = 1;
    e->refresh_every = cfgs[0].precond_refresh > 0 ? cfgs[0].precond_refresh : 1;
    return CF_OK;
}

// Neighbours of each filament along its lattice line (equal base x, consecutive
// in y, the beat direction): [F][2], -1 where the line ends.
int build_neighbours(Engine *e, const cf_sim_config *cfgs) {
    std::vector<int> nbr(2 * static_cast<size_t>(e->d.F), -1);
    for (int b = 0; b < e->B; ++b) {
        const ArrayInfo &a = e->arr[b];
        const double *bp = cfgs[b].base_pos;
        std::vector<int> idx(a.F);
        for (int q = 0; q < a.F; ++q) idx[q] = q;
        std::sort(idx.begin(), idx.end(), [&](int u, int v) {
            if (bp[3 * u] != bp[3 * v]) return bp[3 * u] < bp[3 * v];
            return bp[3 * u + 1] < bp[3 * v + 1];
        });
        for (size_t q = 0; q < idx.size(); ++q) {
            const double x0 = bp[3 * idx[q]];
            const int g = a.fil0 + idx[q];
            if (q > 0 && std::fabs(bp[3 * idx[q - 1]] - x0) <= 1e-6 * (1.0 + std::fabs(x0)))
                nbr[2 * g] = a.fil0 + idx[q - 1];
            if (q + 1 < idx.size() && std::fabs(bp[3 * idx[q + 1]] - x0) <= 1e-6 * (1.0 + std::fabs(x0)))
                nbr[2 * g + 1] = a.fil0 + idx[q + 1];
        }
    }
    return eng_upload(e, const_cast<int **>(&e->d.nbr), nbr.data(), nbr.size());
}

int engine_init(Engine *e, const cf_sim_config *cfgs, int B) {
    const cf_sim_config &c0 = cfgs[0];
    e->common = c0;
    e->device = c0.device;
    e->B = B;
    cudaDeviceProp prop;
    CF_CUDA(cudaGetDeviceProperties(&prop, e->device));
    e->num_sms = prop.multiProcessorCount;
    CF_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    CF_CUDA(cudaStreamCreateWithFlags(&e->cap_stream, cudaStreamNonBlocking));

    SimDev &d = e->d;
    const int ns = c0.n_seg;
    const int dp = c0.dynamic_phase ? 1 : 0, da = c0.dynamic_angle ? 1 : 0;
    // placement of every array in the batch
    e->arr.resize(B);
    int fil = 0, seg = 0, mi_max = 1;
    long long voff = 0, poff = 0, item0 = 0;
    std::vector<int> fil_arr, rb_arr, h_seg0(B), h_n(B), h_nb(B);
    std::vector<long long> h_poff(B), h_item0(B);
    for (int b = 0; b < B; ++b) {
        ArrayInfo &a = e->arr[b];
        a.F = cfgs[b].n_fil;
        a.N = a.F * ns;
        a.n = 3 * a.N + a.F * (dp + da);
        a.fil0 = fil;
        a.seg0 = seg;
        a.po = dp ? 3 * a.N : -1;
        a.ao = da ? 3 * a.N + (dp ? a.F : 0) : -1;
        a.max_iter = std::min(a.n, c0.gmres_max_iter);
        a.nb = (a.N + 31) / 32;
        a.voff = voff;
        a.vlen = (static_cast<long long>(a.n) + kRowPad - 1) / kRowPad * kRowPad;
        a.poff = poff;
        a.chunk0 = 0;
        a.nchunk = 0;
        for (int q = 0; q < a.F; ++q) fil_arr.push_back(b);
        for (long long q = 0; q < a.vlen / kRowUnit; ++q) rb_arr.push_back(b);
        h_seg0[b] = a.seg0;
        h_n[b] = a.N;
        h_nb[b] = a.nb;
        h_poff[b] = a.poff;
        h_item0[b] = item0;
        fil += a.F;
        seg += a.N;
        voff += a.vlen;
        poff += static_cast<long long>(a.N) * a.nb;
        item0 += static_cast<long long>(a.nb) * (a.nb + 1) / 2;
        mi_max = std::max(mi_max, a.max_iter);
    }
    CF_REQUIRE(voff < (1LL << 31), "cf_batch_create: the batch vectors exceed 2^31 rows");
    d.B = B;
    d.F = fil;
    d.nseg = ns;
    d.N = seg;
    d.nrows = voff;
    d.ldq = voff;
    d.mi_max = mi_max;
    d.ldh = mi_max + 1;
    d.hstride = static_cast<long long>(mi_max + 2) * (mi_max + 1);
    d.sstride = mi_max + 2;
    d.precond = (c0.precond == CF_PRECOND_NONE) ? 0 : 1;
    d.line = (c0.precond == CF_PRECOND_LINE || c0.precond == CF_PRECOND_LEARNED_LINE) ? 1 : 0;
    e->line = d.line != 0;
    d.learned = (c0.precond == CF_PRECOND_LEARNED || c0.precond == CF_PRECOND_LEARNED_LINE) ? 1 : 0;
    e->learned = d.learned != 0;
    d.flexible = d.learned;
    d.lin = 9 * ns + 2;   // own force rows, 2 rate rows, neighbour-mean force rows, shape
    d.lalpha = 1.0;
    d.lout = 3 * ns + 2;
    d.dyn_phase = dp;
    d.dyn_angle = da;
    d.dt = c0.dt;
    d.L = c0.seg_sep * (ns - 1);  // FIL_LENGTH = DL*(NSEG_PER_CILIA-1), RSEG = 1
    d.spring = c0.spring_factor;
    d.tol = c0.gmres_tol;
    d.s_tol = (c0.s_tol_factor > 0 ? c0.s_tol_factor : 0.1) / ns;
    // Wall frame: rot_mat of (1/sqrt2, 0, -1/sqrt2, 0) maps the reference x axis to e_z.
    const double R[9] = {0, 0, -1, 0, 1, 0, 1, 0, 0};
    std::memcpy(d.R, R, sizeof(R));
    d.beat = beat_table(c0.beat);
    d.s_rows = c0.s_values_ref ? c0.s_ref_rows : 0;
    d.s_cols = c0.s_values_ref ? c0.s_ref_cols : 0;
    d.n_phase_refs = dp ? c0.n_gen_phase_refs : 0;
    d.n_angle_refs = da ? c0.n_gen_angle_refs : 0;

    // per-filament state, array by array
    const int F = fil;
    std::vector<double> omega(F), ph(F, 0.0), an(F, 0.0), base(3 * static_cast<size_t>(F)), zeros(F, 0.0);
    for (int b = 0; b < B; ++b) {
        const ArrayInfo &a = e->arr[b];
        const cf_sim_config &c = cfgs[b];
        for (int q = 0; q < a.F; ++q) {
            omega[a.fil0 + q] = c.omega0 ? c.omega0[q] : 2.0 * 3.14159265358979323846;
            if (c.phase0) ph[a.fil0 + q] = c.phase0[q];
            if (c.angle0) an[a.fil0 + q] = c.angle0[q];
        }
        std::copy(c.base_pos, c.base_pos + 3 * static_cast<size_t>(a.F), base.begin() + 3 * static_cast<size_t>(a.fil0));
    }
    CF_TRY(eng_upload(e, const_cast<double **>(&d.s_table), c0.s_values_ref, static_cast<size_t>(d.s_rows) * d.s_cols));
    CF_TRY(eng_upload(e, const_cast<double **>(&d.phase_refs), c0.gen_phase_force_refs, d.n_phase_refs));
    CF_TRY(eng_upload(e, const_cast<double **>(&d.angle_refs), c0.gen_angle_force_refs, d.n_angle_refs));
    CF_TRY(eng_upload(e, const_cast<double **>(&d.omega0), omega.data(), F));
    CF_TRY(eng_upload(e, const_cast<double **>(&d.base), base.data(), base.size()));
    CF_TRY(eng_upload(e, &d.phase, ph.data(), F));
    CF_TRY(eng_upload(e, &d.angle, an.data(), F));
    CF_TRY(eng_upload(e, &d.phase_dot, omega.data(), F));  // phase_dot = omega0 (filament.cpp:472)
    CF_TRY(eng_upload(e, &d.angle_dot, zeros.data(), F));

    const size_t N = seg, nr = voff, mi = mi_max, ldq = voff;
    CF_TRY(eng_alloc(e, &d.x4, N));
    CF_TRY(eng_alloc(e, &d.f4, N));
    CF_TRY(eng_alloc(e, &d.xd, 3 * N));
    CF_TRY(eng_alloc(e, &d.s_cur, N));
    CF_TRY(eng_alloc(e, &d.kp, 3 * N));
    CF_TRY(eng_alloc(e, &d.ka, 3 * N));
    CF_TRY(eng_alloc(e, &d.gram, 3 * static_cast<size_t>(F)));
    CF_TRY(eng_alloc(e, &d.rhs, nr));
    CF_TRY(eng_alloc(e, &d.sol, nr));
    CF_TRY(eng_alloc(e, &d.w, nr));
    CF_TRY(eng_alloc(e, &d.z, nr));
    CF_TRY(eng_alloc(e, &d.t, nr));
    CF_TRY(eng_alloc(e, &d.Q, (mi + 1) * ldq));
    d.Z = nullptr;
    if (d.flexible) CF_TRY(eng_alloc(e, &d.Z, (mi + 1) * ldq));
    CF_TRY(eng_alloc(e, &d.lx, static_cast<size_t>(F) * d.lin));
    CF_TRY(eng_alloc(e, &d.ly, static_cast<size_t>(F) * d.lout));
    CF_TRY(eng_alloc(e, &d.lscale, F));
    CF_TRY(build_neighbours(e, cfgs));
    const size_t sm = static_cast<size_t>(B) * d.sstride;
    CF_TRY(eng_alloc(e, &d.H, static_cast<size_t>(B) * d.hstride));
    CF_TRY(eng_alloc(e, &d.cs, sm));
    CF_TRY(eng_alloc(e, &d.sn, sm));
    CF_TRY(eng_alloc(e, &d.beta, sm));
    CF_TRY(eng_alloc(e, &d.h1, sm));
    CF_TRY(eng_alloc(e, &d.h2, sm));
    CF_TRY(eng_alloc(e, &d.y, sm));
    CF_TRY(eng_alloc(e, &d.ctl, B));
    CF_TRY(eng_alloc(e, &d.lc, 1));
    CF_TRY(eng_alloc(e, &d.active, B));
    CF_TRY(eng_alloc(e, &d.iter_log, static_cast<size_t>(B) * kIterLogCap));
    CF_TRY(eng_alloc(e, &e->err, 1));
    d.iter_log_cap = kIterLogCap;
    // placement tables
    CF_TRY(eng_alloc(e, &e->d_arr, B));
    d.arr = e->d_arr;
    CF_TRY(eng_upload(e, const_cast<int **>(&d.fil_arr), fil_arr.data(), fil_arr.size()));
    CF_TRY(eng_upload(e, const_cast<int **>(&d.rb_arr), rb_arr.data(), rb_arr.size()));
    size_t max_chunks = 0;
    for (const ArrayInfo &a : e->arr) max_chunks += (a.n + kMinDotsChunk - 1) / kMinDotsChunk;
    CF_TRY(eng_alloc(e, &e->d_chunk_arr, max_chunks));
    d.chunk_arr = e->d_chunk_arr;
    CF_TRY(eng_alloc(e, &d.dots_partial, (mi + 1) * max_chunks));
    CF_TRY(eng_alloc(e, &d.norm_partial, std::max<size_t>(F, nr / kRowUnit)));
    // pair kernel work list
    int *p_seg0, *p_n, *p_nb;
    long long *p_poff, *p_item0;
    CF_TRY(eng_upload(e, &p_seg0, h_seg0.data(), B));
    CF_TRY(eng_upload(e, &p_n, h_n.data(), B));
    CF_TRY(eng_upload(e, &p_nb, h_nb.data(), B));
    CF_TRY(eng_upload(e, &p_poff, h_poff.data(), B));
    CF_TRY(eng_upload(e, &p_item0, h_item0.data(), B));
    float4 *partial;
    CF_TRY(eng_alloc(e, &partial, static_cast<size_t>(poff)));
    d.partial = partial;
    SymBatchParams &p = e->pair;
    p.x = d.x4;
    p.f = d.f4;
    p.partial = partial;
    p.seg0 = p_seg0;
    p.n = p_n;
    p.nb = p_nb;
    p.poff = p_poff;
    p.item0 = p_item0;
    p.active = d.active;
    p.B = B;
    p.items = item0;

    CF_CUDA(cudaMemset(d.iter_log, 0, sizeof(int) * static_cast<size_t>(B) * kIterLogCap));
    CF_CUDA(cudaMemset(d.ctl, 0, sizeof(GmresCtl) * B));
    CF_CUDA(cudaMemset(d.lc, 0, sizeof(LoopCtl)));
    CF_CUDA(cudaMemset(e->err, 0, sizeof(int)));
    CF_CUDA(cudaMemset(d.H, 0, sizeof(double) * static_cast<size_t>(B) * d.hstride));
    // initial solution: lambda = 0, phase rate = omega0, angle rate = 0
    std::vector<double> sol(nr, 0.0);
    if (dp)
        for (int b = 0; b < B; ++b)
            for (int q = 0; q < e->arr[b].F; ++q) sol[e->arr[b].voff + e->arr[b].po + q] = omega[e->arr[b].fil0 + q];
    CF_CUDA(cudaMemcpy(d.sol, sol.data(), nr * sizeof(double), cudaMemcpyHostToDevice));
    CF_CUDA(cudaMemset(d.rhs, 0, nr * sizeof(double)));
    CF_CUDA(cudaMemset(d.w, 0, nr * sizeof(double)));

    // launch shapes
    e->fil_threads = std::min(256, std::max(64, (3 * ns + 31) / 32 * 32));
    e->kin_smem = sizeof(double) * (2 * (10 * ns + 1) + ns);
    e->pre_smem = sizeof(double) * 3 * ns;
    e->givens_smem = sizeof(double) * 3 * (d.mi_max + 2);
    e->epi_grid = (seg + 31) / 32;
    if (e->givens_smem > 48 * 1024) {
        const int gs = static_cast<int>(e->givens_smem);
        CF_CUDA(cudaFuncSetAttribute(update_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, gs));
        CF_CUDA(cudaFuncSetAttribute(update_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, gs));
        CF_CUDA(cudaFuncSetAttribute(update_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, gs));
        CF_CUDA(cudaFuncSetAttribute(update_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, gs));
    }
    if (e->kin_smem > 48 * 1024)
        CF_CUDA(cudaFuncSetAttribute(kinematics_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(e->kin_smem)));
    if (e->line) CF_TRY(build_patches(e, cfgs));
    // default dot-product chunk: about 16 chunks of the largest array, so that the (k + 1) x chunks
    // items of the first iterations already cover the SMs (1024..4096 rows)
    Tuning t0;
    long long nmax = 1;
    for (const ArrayInfo &a : e->arr) nmax = std::max<long long>(nmax, a.n);
    t0.dots_chunk = static_cast<int>(std::min<long long>(4096, std::max<long long>(kMinDotsChunk, (nmax / 16 + 255) / 256 * 256)));
    CF_TRY(apply_tuning(e, t0));
    const char *ng = std::getenv("CUFIL_NO_GRAPH");
    e->use_graph = !(ng && ng[0] == '1');
    return CF_OK;
}

void engine_release(Engine *e) {
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    if (e->exec) cudaGraphExecDestroy(e->exec);
    if (e->graph) cudaGraphDestroy(e->graph);
    if (e->rexec) cudaGraphExecDestroy(e->rexec);
    if (e->rgraph) cudaGraphDestroy(e->rgraph);
    for (void *p : e->allocations) cudaFree(p);
    if (e->cap_stream) cudaStreamDestroy(e->cap_stream);
    if (e->stream) cudaStreamDestroy(e->stream);
    e->allocations.clear();
}

template <typename H>
int create_handle(const cf_sim_config *cfgs, int B, H **out, const char *who) {
    clear_error();
    CF_REQUIRE(cfgs && out && B > 0, "%s: bad arguments", who);
    *out = nullptr;
    for (int b = 0; b < B; ++b) {
        CF_TRY(validate(&cfgs[b], who));
        if (b) CF_TRY(validate_shared(cfgs[0], cfgs[b], b));
    }
    CF_CUDA(cudaSetDevice(cfgs[0].device));
    H *h = new (std::nothrow) H();
    if (!h) return set_error(CF_ENOMEM, "%s: host allocation failed", who);
    const int rc = engine_init(h, cfgs, B);
    if (rc != CF_OK) {
        std::string msg = cf_last_error();
        engine_release(h);
        delete h;
        set_error(rc, "%s", msg.c_str());
        return rc;
    }
    *out = h;
    return CF_OK;
}

// --------------------------------------------------------------- autotuner
// Times one kernel configuration: `launch` issued `reps` times between two
// events on the engine's stream, after two untimed launches.
template <typename Fn>
int time_launches(Engine *e, Fn launch, int reps, float *ms) {
    for (int r = 0; r < 2; ++r) CF_TRY(launch());
    cudaEvent_t a, b;
    CF_CUDA(cudaEventCreate(&a));
    CF_CUDA(cudaEventCreate(&b));
    CF_CUDA(cudaEventRecord(a, e->stream));
    int rc = CF_OK;
    for (int r = 0; r < reps && rc == CF_OK; ++r) rc = launch();
    cudaEventRecord(b, e->stream);
    cudaEventSynchronize(b);
    float t = 0.0f;
    cudaEventElapsedTime(&t, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    CF_TRY(rc);
    *ms = t / reps;
    return CF_OK;
}

__global__ void set_k_kernel(LoopCtl *lc, int k) {
    if (threadIdx.x == 0 && blockIdx.x == 0) lc->k = k;
}

// Picks the launch shapes of the iteration kernels by timing them on the
// batch as it stands (every array active, basis index k_rep): the pair
// kernel's residency target, the dot-product row chunk and grid, and the
// grid of the row-block updates.  Only scratch buffers are written (the
// mobility partials, w with a zero update, h1, the dot partials); the filament
// state and the solution are untouched.
int engine_autotune(Engine *e, int k_hint, int *choice) {
    SimDev &d = e->d;
    CF_CUDA(cudaStreamSynchronize(e->stream));
    int k_rep = k_hint;
    if (k_rep <= 0) {
        k_rep = 100;
        if (e->stepped) {
            std::vector<GmresCtl> c;
            CF_TRY(read_ctls(e, c));
            int mx = 0;
            for (const GmresCtl &g : c) mx = std::max(mx, iters_of(g));
            if (mx > 0) k_rep = (mx + 1) / 2;
        }
    }
    k_rep = std::max(0, std::min(k_rep, d.mi_max - 1));
    CF_TRY(launch_step_begin(e, -1, e->stream));
    set_k_kernel<<<1, 1, 0, e->stream>>>(d.lc, k_rep);
    CF_CHECK_LAUNCH("set_k_kernel");
    CF_CUDA(cudaMemsetAsync(d.h1, 0, sizeof(double) * static_cast<size_t>(e->B) * d.sstride, e->stream));
    const int reps = 5;
    Tuning best = e->tune;
    float t;
    // pair kernel
    {
        float bt = 1e30f;
        for (int c : {2, 4, 6, 8}) {
            const int grid = pair_grid_for(e->pair.items, e->num_sms, c);
            CF_TRY(time_launches(e, [&] { return rpy_launch_sym_batch(e->pair, grid, e->stream); }, reps, &t));
            if (t < bt * 0.98f) {
                bt = t;
                best.pair_ctas_per_sm = c;
            }
        }
    }
    // dot products: the chunk tables change with the chunk size
    {
        float bt = 1e30f;
        Tuning trial = best;
        for (int chunk : {1024, 2048, 4096, 8192}) {
            for (int bps : {1, 2, 4}) {
                trial.dots_chunk = chunk;
                trial.dots_blocks_per_sm = bps;
                CF_TRY(apply_tuning(e, trial));
                CF_TRY(time_launches(
                    e,
                    [&] {
                        dots_kernel<<<e->dots_grid, 256, 0, e->stream>>>(e->d, e->d.h1);
                        CF_CHECK_LAUNCH("dots_kernel");
                        return CF_OK;
                    },
                    reps, &t));
                if (t < bt * 0.98f) {
                    bt = t;
                    best.dots_chunk = chunk;
                    best.dots_blocks_per_sm = bps;
                }
            }
        }
        CF_TRY(apply_tuning(e, best));
        CF_CUDA(cudaMemsetAsync(d.h1, 0, sizeof(double) * static_cast<size_t>(e->B) * d.sstride, e->stream));
    }
    // row-tile updates (w -= Q h with h = 0: the timing of the real update, w unchanged):
    // tile height and grid
    {
        float bt = 1e30f;
        for (int rows : {32, 64, 128, 256}) {
            for (int bps : {2, 4, 8, 16}) {
                const long long ntiles = d.nrows / rows;
                const int grid = static_cast<int>(std::max(1LL, std::min(ntiles, 1LL * e->num_sms * bps)));
                CF_TRY(time_launches(
                    e, [&] { return launch_update(e, e->d.h1, 0, 0, e->stream, rows, grid); }, reps, &t));
                if (t < bt * 0.98f) {
                    bt = t;
                    best.update_rows = rows;
                    best.update_blocks_per_sm = bps;
                }
            }
        }
    }
    CF_TRY(apply_tuning(e, best));
    CF_CUDA(cudaStreamSynchronize(e->stream));
    if (choice) {
        choice[0] = best.pair_ctas_per_sm;
        choice[1] = best.dots_chunk;
        choice[2] = best.dots_blocks_per_sm;
        choice[3] = best.update_blocks_per_sm;
        choice[4] = best.update_rows;
    }
    return CF_OK;
}

int engine_set_tuning(Engine *e, const int *choice) {
    CF_REQUIRE(choice, "null tuning");
    Tuning t;
    t.pair_ctas_per_sm = choice[0];
    t.dots_chunk = choice[1];
    t.dots_blocks_per_sm = choice[2];
    t.update_blocks_per_sm = choice[3];
    t.update_rows = choice[4];
    CF_REQUIRE(t.pair_ctas_per_sm >= 1 && t.pair_ctas_per_sm <= 8, "tuning: pair CTAs per SM must be 1..8");
    CF_REQUIRE(t.dots_chunk >= kMinDotsChunk && t.dots_chunk % 256 == 0 && t.dots_chunk <= (1 << 20),
               "tuning: dot chunk must be a multiple of 256 in [%d, 2^20]", kMinDotsChunk);
    CF_REQUIRE(t.dots_blocks_per_sm >= 1 && t.dots_blocks_per_sm <= 16, "tuning: dot blocks per SM must be 1..16");
    CF_REQUIRE(t.update_blocks_per_sm >= 1 && t.update_blocks_per_sm <= 32,
               "tuning: update blocks per SM must be 1..32");
    CF_REQUIRE(t.update_rows == 32 || t.update_rows == 64 || t.update_rows == 128 || t.update_rows == 256,
               "tuning: update tile rows must be 32, 64, 128 or 256");
    CF_CUDA(cudaStreamSynchronize(e->stream));
    return apply_tuning(e, t);
}

void engine_get_tuning(const Engine *e, int *choice) {
    choice[0] = e->tune.pair_ctas_per_sm;
    choice[1] = e->tune.dots_chunk;
    choice[2] = e->tune.dots_blocks_per_sm;
    choice[3] = e->tune.update_blocks_per_sm;
    choice[4] = e->tune.update_rows;
}

// Filament-state copies for arrays [b0, b1) (all filaments of those arrays).
int copy_state_out(Engine *e, double *phase, double *angle, double *phase_dot, double *angle_dot) {
    const size_t bytes = sizeof(double) * e->d.F;
    if (phase) CF_CUDA(cudaMemcpyAsync(phase, e->d.phase, bytes, cudaMemcpyDeviceToHost, e->stream));
    if (angle) CF_CUDA(cudaMemcpyAsync(angle, e->d.angle, bytes, cudaMemcpyDeviceToHost, e->stream));
    if (phase_dot) CF_CUDA(cudaMemcpyAsync(phase_dot, e->d.phase_dot, bytes, cudaMemcpyDeviceToHost, e->stream));
    if (angle_dot) CF_CUDA(cudaMemcpyAsync(angle_dot, e->d.angle_dot, bytes, cudaMemcpyDeviceToHost, e->stream));
    CF_CUDA(cudaStreamSynchronize(e->stream));
    return CF_OK;
}

int copy_state_in(Engine *e, const double *phase, const double *angle, const double *phase_dot,
                  const double *angle_dot) {
    SimDev &d = e->d;
    const size_t bytes = sizeof(double) * d.F;
    if (phase) CF_CUDA(cudaMemcpyAsync(d.phase, phase, bytes, cudaMemcpyHostToDevice, e->stream));
    if (angle) CF_CUDA(cudaMemcpyAsync(d.angle, angle, bytes, cudaMemcpyHostToDevice, e->stream));
    // the rates are both filament state and the GMRES warm start (mobility_solver.cpp:2298-2388)
    for (int b = 0; b < e->B; ++b) {
        const ArrayInfo &a = e->arr[b];
        const size_t fb = sizeof(double) * a.F;
        if (phase_dot) {
            CF_CUDA(cudaMemcpyAsync(d.phase_dot + a.fil0, phase_dot + a.fil0, fb, cudaMemcpyHostToDevice, e->stream));
            if (a.po >= 0)
                CF_CUDA(cudaMemcpyAsync(d.sol + a.voff + a.po, phase_dot + a.fil0, fb, cudaMemcpyHostToDevice,
                                        e->stream));
        }
        if (angle_dot) {
            CF_CUDA(cudaMemcpyAsync(d.angle_dot + a.fil0, angle_dot + a.fil0, fb, cudaMemcpyHostToDevice, e->stream));
            if (a.ao >= 0)
                CF_CUDA(cudaMemcpyAsync(d.sol + a.voff + a.ao, angle_dot + a.fil0, fb, cudaMemcpyHostToDevice,
                                        e->stream));
        }
    }
    return CF_OK;
}

}  // namespace

// ===================================================================== cf_sim
extern "C" int cf_sim_create(const cf_sim_config *cfg, cf_sim **out) {
    return create_handle<cf_sim>(cfg, 1, out, "cf_sim_create");
}

extern "C" int cf_sim_destroy(cf_sim *s) {
    if (!s) return CF_OK;
    engine_release(s);
    delete s;
    return CF_OK;
}

extern "C" int cf_sim_step_async(cf_sim *s, int nt) {
    clear_error();
    CF_REQUIRE(s, "null handle");
    CF_REQUIRE(nt >= 0, "cf_sim_step: nt must be >= 0");
    CF_CUDA(cudaSetDevice(s->device));
    return run_step(s, nt);
}

extern "C" int cf_sim_last_solve(cf_sim *s, int *iters, double *relres) {
    clear_error();
    CF_REQUIRE(s, "null handle");
    CF_CUDA(cudaSetDevice(s->device));
    std::vector<GmresCtl> c;
    CF_TRY(read_ctls(s, c));
    if (iters) *iters = iters_of(c[0]);
    if (relres) *relres = c[0].relres;
    return status_of(c[0], 0, 1);
}

extern "C" int cf_sim_step(cf_sim *s, int nt, int *iters, double *relres) {
    CF_TRY(cf_sim_step_async(s, nt));
    return cf_sim_last_solve(s, iters, relres);
}

extern "C" int cf_sim_get_state(cf_sim *s, double *phase, double *angle, double *phase_dot, double *angle_dot) {
    clear_error();
    CF_REQUIRE(s, "null handle");
    CF_CUDA(cudaSetDevice(s->device));
    return copy_state_out(s, phase, angle, phase_dot, angle_dot);
}

extern "C" int cf_sim_get_segments(cf_sim *s, float *x_segs, float *f_segs) {
    clear_error();
    CF_REQUIRE(s, "null handle");
    CF_CUDA(cudaSetDevice(s->device));
    const int N = s->d.N;
    std::vector<double> buf(3 * static_cast<size_t>(N));
    if (x_segs) {
        CF_CUDA(cudaMemcpyAsync(buf.data(), s->d.xd, buf.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
        CF_CUDA(cudaStreamSynchronize(s->stream));
        for (size_t i = 0; i < buf.size(); ++i) x_segs[i] = static_cast<float>(buf[i]);
    }
    if (f_segs) {
        CF_CUDA(cudaMemcpyAsync(buf.data(), s->d.sol, buf.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
        CF_CUDA(cudaStreamSynchronize(s->stream));
        for (int i = 0; i < N; ++i)
            for (int c = 0; c < 6; ++c) f_segs[6 * i + c] = c < 3 ? static_cast<float>(buf[3 * i + c]) : 0.0f;
    }
    return CF_OK;
}

extern "C" int cf_sim_step_io(cf_sim *s, int nt, const double *phase_in, const double *angle_in,
                              const double *phase_dot_in, const double *angle_dot_in, double *phase_out,
                              double *angle_out, double *phase_dot_out, double *angle_dot_out, float *x_segs,
                              float *f_segs, int *iters, double *relres) {
    clear_error();
    CF_REQUIRE(s, "null handle");
    CF_REQUIRE(nt >= 0, "cf_sim_step_io: nt must be >= 0");
    CF_CUDA(cudaSetDevice(s->device));
    const int N = s->d.N;
    if ((x_segs || f_segs) && !s->seg_out) CF_TRY(eng_alloc(s, &s->seg_out, 9 * static_cast<size_t>(N)));
    CF_TRY(copy_state_in(s, phase_in, angle_in, phase_dot_in, angle_dot_in));
    CF_TRY(run_step(s, nt));
    const size_t fb = sizeof(double) * s->d.F;
    cudaStream_t st = s->stream;
    if (phase_out) CF_CUDA(cudaMemcpyAsync(phase_out, s->d.phase, fb, cudaMemcpyDeviceToHost, st));
    if (angle_out) CF_CUDA(cudaMemcpyAsync(angle_out, s->d.angle, fb, cudaMemcpyDeviceToHost, st));
    if (phase_dot_out) CF_CUDA(cudaMemcpyAsync(phase_dot_out, s->d.phase_dot, fb, cudaMemcpyDeviceToHost, st));
    if (angle_dot_out) CF_CUDA(cudaMemcpyAsync(angle_dot_out, s->d.angle_dot, fb, cudaMemcpyDeviceToHost, st));
    if (x_segs || f_segs) {
        segments_out_kernel<<<(N + 255) / 256, 256, 0, st>>>(s->d, s->seg_out, s->seg_out + 3 * static_cast<size_t>(N));
        CF_CHECK_LAUNCH("segments_out_kernel");
        if (x_segs) CF_CUDA(cudaMemcpyAsync(x_segs, s->seg_out, sizeof(float) * 3 * N, cudaMemcpyDeviceToHost, st));
        if (f_segs)
            CF_CUDA(cudaMemcpyAsync(f_segs, s->seg_out + 3 * static_cast<size_t>(N), sizeof(float) * 6 * N,
                                    cudaMemcpyDeviceToHost, st));
    }
    std::vector<GmresCtl> c;
    CF_TRY(read_ctls(s, c));  // the one synchronisation
    if (iters) *iters = iters_of(c[0]);
    if (relres) *relres = c[0].relres;
    return status_of(c[0], 0, 1);
}

extern "C" int cf_sim_get_directions(cf_sim *s, double *k_phase, double *k_angle) {
    clear_error();
    CF_REQUIRE(s, "null handle");
    CF_CUDA(cudaSetDevice(s->device));
    const size_t b = sizeof(double) * 3 * s->d.N;
    if (k_phase) CF_CUDA(cudaMemcpyAsync(k_phase, s->d.kp, b, cudaMemcpyDeviceToHost, s->stream));
    if (k_angle) CF_CUDA(cudaMemcpyAsync(k_angle, s->d.ka, b, cudaMemcpyDeviceToHost, s->stream));
    CF_CUDA(cudaStreamSynchronize(s->stream));
    return CF_OK;
}

extern "C" int cf_sim_get_arclengths(cf_sim *s, double *s_values) {
    clear_error();
    CF_REQUIRE(s && s_values, "null argument");
    CF_CUDA(cudaSetDevice(s->device));
    CF_CUDA(cudaMemcpyAsync(s_values, s->d.s_cur, sizeof(double) * s->d.N, cudaMemcpyDeviceToHost, s->stream));
    CF_CUDA(cudaStreamSynchronize(s->stream));
    return CF_OK;
}

extern "C" int cf_sim_system_size(cf_sim *s) { return s ? s->arr[0].n : -1; }

extern "C" int cf_sim_stream(cf_sim *s, void **stream) {
    clear_error();
    CF_REQUIRE(s && stream, "null argument");
    *stream = static_cast<void *>(s->stream);
    return CF_OK;
}

extern "C" int cf_sim_set_state(cf_sim *s, const double *phase, const double *angle, const double *phase_dot,
                                const double *angle_dot) {
    clear_error();
    CF_REQUIRE(s, "null handle");
    CF_CUDA(cudaSetDevice(s->device));
    return copy_state_in(s, phase, angle, phase_dot, angle_dot);
}

extern "C" int cf_sim_get_solution(cf_sim *s, double *sol) {
    clear_error();
    CF_REQUIRE(s && sol, "cf_sim_get_solution: bad arguments");
    CF_CUDA(cudaSetDevice(s->device));
    CF_CUDA(cudaMemcpyAsync(sol, s->d.sol, sizeof(double) * s->arr[0].n, cudaMemcpyDeviceToHost, s->stream));
    CF_CUDA(cudaStreamSynchronize(s->stream));
    return CF_OK;
}

extern "C" int cf_sim_set_solution(cf_sim *s, const double *sol) {
    clear_error();
    CF_REQUIRE(s && sol, "cf_sim_set_solution: bad arguments");
    CF_CUDA(cudaSetDevice(s->device));
    const ArrayInfo &a = s->arr[0];
    CF_CUDA(cudaMemcpyAsync(s->d.sol, sol, sizeof(double) * a.n, cudaMemcpyHostToDevice, s->stream));
    // the rate rows are the filament rates too
    const size_t fb = sizeof(double) * a.F;
    if (a.po >= 0) CF_CUDA(cudaMemcpyAsync(s->d.phase_dot, s->d.sol + a.po, fb, cudaMemcpyDeviceToDevice, s->stream));
    if (a.ao >= 0) CF_CUDA(cudaMemcpyAsync(s->d.angle_dot, s->d.sol + a.ao, fb, cudaMemcpyDeviceToDevice, s->stream));
    CF_CUDA(cudaStreamSynchronize(s->stream));  // the host buffer may be reused on return
    return CF_OK;
}

extern "C" int cf_sim_iteration_log(cf_sim *s, int *iters, int n) {
    clear_error();
    CF_REQUIRE(s && iters && n >= 0 && n <= kIterLogCap, "cf_sim_iteration_log: bad arguments");
    CF_CUDA(cudaSetDevice(s->device));
    CF_CUDA(cudaMemcpyAsync(iters, s->d.iter_log, sizeof(int) * n, cudaMemcpyDeviceToHost, s->stream));
    CF_CUDA(cudaStreamSynchronize(s->stream));
    return CF_OK;
}

namespace {
// step_begin + kinematics, rhs, pair, epilogue, residual + 7 per iteration + backsub, combine, finish;
// the line-patch preconditioner adds 2 per iteration, 1 in the finish and the refresh when it ran.
int launches_for(const Engine *e, int iters) {
    int n = 1 + 5 + 7 * iters + 3;  // with the line patches, patch_arnoldi_kernel takes arnoldi_precond's place
    if (e && e->line) n += (e->d.flexible ? 0 : 1) + (e->refreshed_last ? refresh_launches(e) : 0);
    if (e && e->learned) n += 6 * iters;  // features, 3 GEMMs, correction, packing
    return n;
}
}  // namespace

extern "C" int cf_sim_launches_per_step(cf_sim *s, int iters) { return launches_for(s, iters); }

extern "C" int cf_sim_initial_guess(cf_sim *s, int nt) {
    clear_error();
    CF_REQUIRE(s, "null handle");
    CF_CUDA(cudaSetDevice(s->device));
    CF_TRY(launch_step_begin(s, nt, s->stream));
    CF_TRY(launch_kinematics(s, s->stream));
    CF_CUDA(cudaStreamSynchronize(s->stream));
    return CF_OK;
}

extern "C" int cf_sim_assemble_rhs(cf_sim *s, int nt, double *rhs) {
    clear_error();
    CF_REQUIRE(s && rhs, "null argument");
    CF_CUDA(cudaSetDevice(s->device));
    CF_TRY(launch_step_begin(s, nt, s->stream));
    rhs_kernel<<<s->d.F, s->fil_threads, 0, s->stream>>>(s->d);
    CF_CHECK_LAUNCH("rhs_kernel");
    CF_CUDA(cudaMemcpyAsync(rhs, s->d.rhs, sizeof(double) * s->arr[0].n, cudaMemcpyDeviceToHost, s->stream));
    CF_CUDA(cudaStreamSynchronize(s->stream));
    return CF_OK;
}

extern "C" int cf_sim_apply_preconditioner(cf_sim *s, const double *in, double *out) {
    clear_error();
    CF_REQUIRE(s && in && out, "null argument");
    CF_CUDA(cudaSetDevice(s->device));
    const size_t b = sizeof(double) * s->arr[0].n;
    CF_CUDA(cudaMemcpyAsync(s->d.t, in, b, cudaMemcpyHostToDevice, s->stream));
    if (s->line) {  // patch inverses of the current kinematics
        CF_TRY(launch_refresh(s, s->stream));
        s->last_refresh_nt = -1;
        CF_TRY(launch_patch_apply(s, s->d.t, s->d.z, 0, s->stream));
        CF_CUDA(cudaMemcpyAsync(out, s->d.z, b, cudaMemcpyDeviceToHost, s->stream));
        CF_CUDA(cudaStreamSynchronize(s->stream));
        return CF_OK;
    }
    precond_kernel<<<s->d.F, s->fil_threads, s->pre_smem, s->stream>>>(s->d, s->d.t, s->d.t);
    CF_CHECK_LAUNCH("precond_kernel");
    CF_CUDA(cudaMemcpyAsync(out, s->d.t, b, cudaMemcpyDeviceToHost, s->stream));
    CF_CUDA(cudaStreamSynchronize(s->stream));
    return CF_OK;
}

extern "C" int cf_sim_system_matvec(cf_sim *s, const double *in, double *out) {
    clear_error();
    CF_REQUIRE(s && in && out, "null argument");
    CF_CUDA(cudaSetDevice(s->device));
    const size_t b = sizeof(double) * s->arr[0].n;
    CF_TRY(launch_step_begin(s, -1, s->stream));  // every array active for the product
    CF_CUDA(cudaMemcpyAsync(s->d.z, in, b, cudaMemcpyHostToDevice, s->stream));
    pack_forces_kernel<<<(s->d.N + 255) / 256, 256, 0, s->stream>>>(s->d, s->d.z);
    CF_CHECK_LAUNCH("pack_forces_kernel");
    filament_rows_kernel<<<s->d.F, s->fil_threads, 0, s->stream>>>(s->d, s->d.z, s->d.w);
    CF_CHECK_LAUNCH("filament_rows_kernel");
    CF_TRY(launch_matvec_tail(s, s->d.z, s->d.w, s->stream));
    CF_CUDA(cudaMemcpyAsync(out, s->d.w, b, cudaMemcpyDeviceToHost, s->stream));
    LoopCtl lc;
    return read_loop(s, &lc);
}

namespace {
// The host-driven GMRES loop on the caller's RHS (already in d.rhs) and
// initial guess (in d.sol); tolerance and iteration cap of this solve only.
int solve_given(cf_sim *s, double tol, int max_iter) {
    const int cap = s->arr[0].max_iter;
    CF_CUDA(cudaMemcpyAsync(&s->d_arr[0].max_iter, &max_iter, sizeof(int), cudaMemcpyHostToDevice, s->stream));
    const SimDev saved = s->d;
    s->d.tol = tol;
    s->d.rhs_given = 1;
    int rc = launch_prologue(s, 0, s->stream);
    LoopCtl lc{};
    if (rc == CF_OK) rc = read_loop(s, &lc);
    int guard = 0;
    while (rc == CF_OK && lc.cond && guard++ <= s->d.mi_max) {
        rc = launch_body(s, 0, s->stream);
        if (rc == CF_OK) rc = read_loop(s, &lc);
    }
    if (rc == CF_OK) rc = launch_finish(s, s->stream);
    s->d = saved;
    const cudaError_t ce = cudaMemcpyAsync(&s->d_arr[0].max_iter, &cap, sizeof(int), cudaMemcpyHostToDevice,
                                           s->stream);
    if (rc != CF_OK) return rc;
    return cuda_status(ce, "cudaMemcpyAsync", __FILE__, __LINE__);
}
}  // namespace

extern "C" int cf_sim_solve(cf_sim *s, const double *rhs, double *x_inout, double tol, int max_iter, int *iters,
                            double *relres) {
    clear_error();
    CF_REQUIRE(s && rhs && x_inout, "cf_sim_solve: null argument");
    CF_REQUIRE(tol > 0.0 && tol < 1.0, "cf_sim_solve: tol must lie in (0, 1) (got %g)", tol);
    CF_REQUIRE(max_iter >= 1 && max_iter <= s->d.mi_max,
               "cf_sim_solve: max_iter must lie in [1, %d] (the handle's gmres_max_iter), got %d", s->d.mi_max,
               max_iter);
    CF_REQUIRE(s->geometry > 0, "cf_sim_solve: no geometry yet (call cf_sim_initial_guess or cf_sim_step first)");
    CF_REQUIRE(!s->learned || s->net, "CF_PRECOND_LEARNED: no network attached (cf_sim_set_network)");
    CF_CUDA(cudaSetDevice(s->device));
    const size_t b = sizeof(double) * s->arr[0].n;
    CF_TRY(launch_step_begin(s, -1, s->stream));
    CF_CUDA(cudaMemcpyAsync(s->d.rhs, rhs, b, cudaMemcpyHostToDevice, s->stream));
    CF_CUDA(cudaMemcpyAsync(s->d.sol, x_inout, b, cudaMemcpyHostToDevice, s->stream));
    if (s->line && s->refresh_geometry != s->geometry) {  // patch inverses of the current geometry
        CF_TRY(launch_refresh(s, s->stream));
        s->last_refresh_nt = -1;
    }
    CF_TRY(solve_given(s, tol, max_iter));
    CF_CUDA(cudaMemcpyAsync(x_inout, s->d.sol, b, cudaMemcpyDeviceToHost, s->stream));
    return cf_sim_last_solve(s, iters, relres);
}

extern "C" int cf_sim_refresh_preconditioner(cf_sim *s) {
    clear_error();
    CF_REQUIRE(s, "null handle");
    CF_REQUIRE(s->line, "cf_sim_refresh_preconditioner: the handle does not use CF_PRECOND_LINE");
    CF_CUDA(cudaSetDevice(s->device));
    CF_TRY(launch_refresh(s, s->stream));
    s->last_refresh_nt = -1;  // the next step refreshes again for its own kinematics
    return CF_OK;
}

extern "C" int cf_sim_precond_info(cf_sim *s, int *n_patches, int *max_n, double *refresh_flops,
                                   double *apply_bytes) {
    clear_error();
    CF_REQUIRE(s, "null handle");
    double fl = 0.0, by = 0.0;
    if (s->line) {
        std::vector<int> nf(s->P.np);
        CF_CUDA(cudaMemcpy(nf.data(), s->P.nf, sizeof(int) * nf.size(), cudaMemcpyDeviceToHost));
        for (int f : nf) {
            const double n = static_cast<double>(f) * s->P.nbf;
            fl += 2.0 * n * n * n;        // Gauss-Jordan inversion: n^3 multiply-adds
            by += 4.0 * n * n + 16.0 * n; // FP32 inverse read once, FP64 vector gathered and scattered
        }
    }
    if (n_patches) *n_patches = s->line ? s->P.np : 0;
    if (max_n) *max_n = s->line ? s->P.max_n : 0;
    if (refresh_flops) *refresh_flops = fl;
    if (apply_bytes) *apply_bytes = by;
    return CF_OK;
}

extern "C" int cf_sim_learned_dims(cf_sim *s, int *n_in, int *n_out) {
    clear_error();
    CF_REQUIRE(s, "null handle");
    if (n_in) *n_in = s->d.lin;
    if (n_out) *n_out = s->d.lout;
    return CF_OK;
}

extern "C" int cf_sim_set_network(cf_sim *s, cf_mlp *net) {
    clear_error();
    CF_REQUIRE(s && net, "null argument");
    CF_REQUIRE(s->learned, "cf_sim_set_network: the handle does not use CF_PRECOND_LEARNED");
    int in = 0, out = 0, mb = 0;
    mlp_dims(net, &in, &out, &mb);
    CF_REQUIRE(in == s->d.lin && out == s->d.lout && mb >= s->d.F,
               "cf_sim_set_network: network %d -> %d (batch %d) does not fit %d -> %d for %d filaments", in, out, mb,
               s->d.lin, s->d.lout, s->d.F);
    CF_CUDA(cudaSetDevice(s->device));
    CF_CUDA(cudaStreamSynchronize(s->stream));
    s->net = net;
    if (s->exec) cudaGraphExecDestroy(s->exec);
    if (s->graph) cudaGraphDestroy(s->graph);
    s->exec = nullptr;
    s->graph = nullptr;
    return CF_OK;
}

extern "C" int cf_sim_set_network_weight(cf_sim *s, double alpha) {
    clear_error();
    CF_REQUIRE(s, "null handle");
    CF_REQUIRE(alpha >= 0.0 && alpha <= 4.0, "cf_sim_set_network_weight: weight %g outside [0, 4]", alpha);
    CF_CUDA(cudaSetDevice(s->device));
    CF_CUDA(cudaStreamSynchronize(s->stream));
    s->d.lalpha = alpha;
    if (s->exec) cudaGraphExecDestroy(s->exec);
    if (s->graph) cudaGraphDestroy(s->graph);
    s->exec = nullptr;
    s->graph = nullptr;
    return CF_OK;
}

extern "C" int cf_sim_collect_pairs(cf_sim *s, int nt, int max_pairs, float *x, float *t, int *rows) {
    clear_error();
    CF_REQUIRE(s && x && t && max_pairs > 0, "cf_sim_collect_pairs: bad arguments");
    CF_REQUIRE(!s->learned && s->d.precond == 1,
               "cf_sim_collect_pairs: pairs come from the plain solver (CF_PRECOND_BLOCK_DIAG or CF_PRECOND_LINE)");
    CF_REQUIRE(nt >= 0, "cf_sim_collect_pairs: nt must be >= 0");
    CF_CUDA(cudaSetDevice(s->device));
    s->cx = x;
    s->ct = t;
    s->c_max = max_pairs;
    s->c_pairs = 0;
    const int rc = run_step(s, nt);
    const int pairs = s->c_pairs;
    s->cx = s->ct = nullptr;
    s->c_max = s->c_pairs = 0;
    CF_TRY(rc);
    CF_CUDA(cudaStreamSynchronize(s->stream));
    if (rows) *rows = pairs * s->d.F;
    return CF_OK;
}

extern "C" int cf_sim_features(cf_sim *s, const double *v, float *x) {
    clear_error();
    CF_REQUIRE(s && v && x, "null argument");
    CF_CUDA(cudaSetDevice(s->device));
    CF_CUDA(cudaMemcpyAsync(s->d.t, v, sizeof(double) * s->arr[0].n, cudaMemcpyHostToDevice, s->stream));
    learned_features_kernel<<<s->d.F, s->fil_threads, 0, s->stream>>>(s->d, s->d.t, s->d.lx, s->d.lscale);
    CF_CHECK_LAUNCH("learned_features_kernel");
    CF_CUDA(cudaMemcpyAsync(x, s->d.lx, sizeof(float) * s->d.F * s->d.lin, cudaMemcpyDeviceToHost, s->stream));
    CF_CUDA(cudaStreamSynchronize(s->stream));
    return CF_OK;
}

extern "C" int cf_sim_autotune(cf_sim *s, int k_hint, int *choice) {
    clear_error();
    CF_REQUIRE(s, "null handle");
    CF_CUDA(cudaSetDevice(s->device));
    return engine_autotune(s, k_hint, choice);
}

extern "C" int cf_sim_set_tuning(cf_sim *s, const int *choice) {
    clear_error();
    CF_REQUIRE(s, "null handle");
    CF_CUDA(cudaSetDevice(s->device));
    return engine_set_tuning(s, choice);
}

extern "C" int cf_sim_get_tuning(cf_sim *s, int *choice) {
    clear_error();
    CF_REQUIRE(s && choice, "null argument");
    engine_get_tuning(s, choice);
    return CF_OK;
}

// =================================================================== cf_batch
extern "C" int cf_batch_create(const cf_sim_config *cfgs, int n_arrays, cf_batch **out) {
    return create_handle<cf_batch>(cfgs, n_arrays, out, "cf_batch_create");
}

extern "C" int cf_batch_destroy(cf_batch *bt) {
    if (!bt) return CF_OK;
    engine_release(bt);
    delete bt;
    return CF_OK;
}

extern "C" int cf_batch_shape(cf_batch *bt, int *n_arrays, int *n_fil, int *n_seg, int *sizes) {
    clear_error();
    CF_REQUIRE(bt, "null handle");
    if (n_arrays) *n_arrays = bt->B;
    if (n_fil) *n_fil = bt->d.F;
    if (n_seg) *n_seg = bt->d.N;
    if (sizes)
        for (int b = 0; b < bt->B; ++b) sizes[b] = bt->arr[b].n;
    return CF_OK;
}

extern "C" int cf_batch_step_async(cf_batch *bt, int nt) {
    clear_error();
    CF_REQUIRE(bt, "null handle");
    CF_REQUIRE(nt >= 0, "cf_batch_step: nt must be >= 0");
    CF_CUDA(cudaSetDevice(bt->device));
    return run_step(bt, nt);
}

extern "C" int cf_batch_last_solve(cf_batch *bt, int *iters, double *relres, int *status) {
    clear_error();
    CF_REQUIRE(bt, "null handle");
    CF_CUDA(cudaSetDevice(bt->device));
    std::vector<GmresCtl> c;
    CF_TRY(read_ctls(bt, c));
    for (int b = 0; b < bt->B; ++b) {
        if (iters) iters[b] = iters_of(c[b]);
        if (relres) relres[b] = c[b].relres;
        if (status) status[b] = c[b].status;
    }
    return batch_status(c);
}

extern "C" int cf_batch_step(cf_batch *bt, int nt, int *iters, double *relres) {
    CF_TRY(cf_batch_step_async(bt, nt));
    return cf_batch_last_solve(bt, iters, relres, nullptr);
}

extern "C" int cf_batch_get_state(cf_batch *bt, double *phase, double *angle, double *phase_dot, double *angle_dot) {
    clear_error();
    CF_REQUIRE(bt, "null handle");
    CF_CUDA(cudaSetDevice(bt->device));
    return copy_state_out(bt, phase, angle, phase_dot, angle_dot);
}

extern "C" int cf_batch_set_state(cf_batch *bt, const double *phase, const double *angle, const double *phase_dot,
                                  const double *angle_dot) {
    clear_error();
    CF_REQUIRE(bt, "null handle");
    CF_CUDA(cudaSetDevice(bt->device));
    return copy_state_in(bt, phase, angle, phase_dot, angle_dot);
}

extern "C" int cf_batch_get_segments(cf_batch *bt, double *x_segs) {
    clear_error();
    CF_REQUIRE(bt && x_segs, "null argument");
    CF_CUDA(cudaSetDevice(bt->device));
    CF_CUDA(cudaMemcpyAsync(x_segs, bt->d.xd, sizeof(double) * 3 * bt->d.N, cudaMemcpyDeviceToHost, bt->stream));
    CF_CUDA(cudaStreamSynchronize(bt->stream));
    return CF_OK;
}

extern "C" int cf_batch_get_solution(cf_batch *bt, int array, double *sol) {
    clear_error();
    CF_REQUIRE(bt && sol && array >= 0 && array < bt->B, "cf_batch_get_solution: bad arguments");
    CF_CUDA(cudaSetDevice(bt->device));
    const ArrayInfo &a = bt->arr[array];
    CF_CUDA(cudaMemcpyAsync(sol, bt->d.sol + a.voff, sizeof(double) * a.n, cudaMemcpyDeviceToHost, bt->stream));
    CF_CUDA(cudaStreamSynchronize(bt->stream));
    return CF_OK;
}

extern "C" int cf_batch_iteration_log(cf_batch *bt, int array, int *iters, int n) {
    clear_error();
    CF_REQUIRE(bt && iters && array >= 0 && array < bt->B && n >= 0 && n <= kIterLogCap,
               "cf_batch_iteration_log: bad arguments");
    CF_CUDA(cudaSetDevice(bt->device));
    CF_CUDA(cudaMemcpyAsync(iters, bt->d.iter_log + static_cast<size_t>(array) * kIterLogCap, sizeof(int) * n,
                            cudaMemcpyDeviceToHost, bt->stream));
    CF_CUDA(cudaStreamSynchronize(bt->stream));
    return CF_OK;
}

extern "C" int cf_batch_stream(cf_batch *bt, void **stream) {
    clear_error();
    CF_REQUIRE(bt && stream, "null argument");
    *stream = static_cast<void *>(bt->stream);
    return CF_OK;
}

extern "C" int cf_batch_launches_per_step(cf_batch *bt, int loop_iters) { return launches_for(bt, loop_iters); }

extern "C" int cf_batch_autotune(cf_batch *bt, int k_hint, int *choice) {
    clear_error();
    CF_REQUIRE(bt, "null handle");
    CF_CUDA(cudaSetDevice(bt->device));
    return engine_autotune(bt, k_hint, choice);
}

extern "C" int cf_batch_set_tuning(cf_batch *bt, const int *choice) {
    clear_error();
    CF_REQUIRE(bt, "null handle");
    CF_CUDA(cudaSetDevice(bt->device));
    return engine_set_tuning(bt, choice);
}

extern "C" int cf_batch_get_tuning(cf_batch *bt, int *choice) {
    clear_error();
    CF_REQUIRE(bt && choice, "null argument");
    engine_get_tuning(bt, choice);
    return CF_OK;
}

// =================================================================== files
// The reference's data files for a wall of prescribed cilia, so that its
// sweep drivers (pyfile/find_periodic, pyfile/bisection) read this engine's
// output as they read the reference's.  Line formats follow
// cilia_sim_main.cu:624-718, swimmer.cpp:1144-1158, filament.cpp:2210-2226,
// rigid_body.cpp:565-569 and mobility_solver.cpp:3150-3279; the initial
// condition file is read as filament.cpp:310-340 reads it.  States are FP64
// here, so they are written with 15 significant digits (the reference's
// OUTPUT_DIGIT of its FP64 build); velocities and forces with 10, as there.
namespace {

struct LineFile {
    std::FILE *f = nullptr;
    explicit LineFile(const std::string &path) { f = std::fopen(path.c_str(), "a"); }
    ~LineFile() {
        if (f) std::fclose(f);
    }
    void lead(long long k) { std::fprintf(f, "%lld ", k); }
    void num(double v, int digits) { std::fprintf(f, "%.*e ", digits, v); }
    bool end() {
        std::fputc('\n', f);
        return std::ferror(f) == 0;
    }
};

int open_all(const std::string &prefix, const char *const *suffixes, int n, std::vector<LineFile *> &out) {
    for (int i = 0; i < n; ++i) {
        auto *lf = new LineFile(prefix + suffixes[i]);
        out.push_back(lf);
        if (!lf->f) return set_error(CF_EINVAL, "cf_sim_write_data: cannot open %s%s", prefix.c_str(), suffixes[i]);
    }
    return CF_OK;
}

}  // namespace

extern "C" int cf_sim_write_data(cf_sim *s, int save_step, double period, const char *prefix) {
    clear_error();
    CF_REQUIRE(s && prefix, "cf_sim_write_data: null argument");
    CF_REQUIRE(s->B == 1, "cf_sim_write_data: one array per handle");
    CF_REQUIRE(s->geometry > 0, "cf_sim_write_data: no step has run yet");
    CF_CUDA(cudaSetDevice(s->device));
    const ArrayInfo a = s->arr[0];
    const int F = a.F, N = a.N, nseg = s->d.nseg;
    std::vector<double> phase(F), angle(F), pd(F), ad(F), x(3 * static_cast<size_t>(N)), sol(a.n), av(a.n);
    std::vector<double> kp(3 * static_cast<size_t>(N)), ka(3 * static_cast<size_t>(N));
    CF_TRY(copy_state_out(s, phase.data(), angle.data(), pd.data(), ad.data()));
    CF_CUDA(cudaMemcpyAsync(x.data(), s->d.xd, x.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CF_CUDA(cudaMemcpyAsync(sol.data(), s->d.sol, sol.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CF_CUDA(cudaMemcpyAsync(kp.data(), s->d.kp, kp.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CF_CUDA(cudaMemcpyAsync(ka.data(), s->d.ka, ka.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CF_CUDA(cudaStreamSynchronize(s->stream));
    // Segment velocities as the reference writes them: M applied to the solution's
    // constraint forces (mobility_solver.cpp:3154-3156 recomputes the product
    // before writing), i.e. the lambda rows of A sol plus the rate terms.
    CF_TRY(cf_sim_system_matvec(s, sol.data(), av.data()));
    const char *suffixes[] = {"_seg_states.dat", "_body_states.dat", "_true_states.dat", "_seg_vels.dat",
                              "_seg_forces.dat"};
    std::vector<LineFile *> files;
    int rc = open_all(prefix, suffixes, 5, files);
    if (rc == CF_OK) {
        LineFile &seg = *files[0], &body = *files[1], &tru = *files[2], &vel = *files[3], &frc = *files[4];
        seg.lead(save_step);
        for (size_t i = 0; i < x.size(); ++i) seg.num(x[i], 15);
        body.lead(save_step);  // the wall case has no moving body: at the origin, identity orientation
        for (double v : {0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0}) body.num(v, 15);
        tru.lead(save_step);
        tru.num(period, 15);
        for (int m = 0; m < F; ++m) tru.num(phase[m], 15);
        if (s->d.dyn_angle)
            for (int m = 0; m < F; ++m) tru.num(angle[m], 15);
        vel.lead(save_step);
        frc.lead(save_step);
        for (int i = 0; i < N; ++i) {
            const int m = i / nseg;
            for (int c = 0; c < 3; ++c) {
                double v = av[3 * i + c];
                if (a.po >= 0) v += kp[3 * i + c] * sol[a.po + m];
                if (a.ao >= 0) v += ka[3 * i + c] * sol[a.ao + m];
                vel.num(v, 10);
            }
            for (int c = 0; c < 3; ++c) vel.num(0.0, 10);
            for (int c = 0; c < 3; ++c) frc.num(sol[3 * i + c], 10);
            for (int c = 0; c < 3; ++c) frc.num(0.0, 10);
        }
        for (LineFile *lf : files)
            if (!lf->end()) rc = set_error(CF_EINVAL, "cf_sim_write_data: write under %s failed", prefix);
    }
    for (LineFile *lf : files) delete lf;
    return rc;
}

extern "C" int cf_sim_write_config(cf_sim *s, const char *prefix, int total_steps) {
    clear_error();
    CF_REQUIRE(s && prefix, "cf_sim_write_config: null argument");
    CF_REQUIRE(s->B == 1, "cf_sim_write_config: one array per handle");
    CF_CUDA(cudaSetDevice(s->device));
    const cf_sim_config &c = s->common;
    const int F = s->arr[0].F, nseg = s->d.nseg;
    std::vector<double> base(3 * static_cast<size_t>(F));
    CF_CUDA(cudaMemcpy(base.data(), s->d.base, base.size() * sizeof(double), cudaMemcpyDeviceToHost));
    const std::string p(prefix);
    // swimmer::write_reference_positions (swimmer.cpp:1114-1127): the filament base positions on one line
    std::FILE *f = std::fopen((p + "_fil_references.dat").c_str(), "w");
    if (!f) return set_error(CF_EINVAL, "cf_sim_write_config: cannot open %s_fil_references.dat", prefix);
    for (double v : base) std::fprintf(f, "%.15g ", v);
    std::fputc('\n', f);
    const bool ok1 = std::fclose(f) == 0;
    // The .par summary of cilia_sim_main.cu:178-232 (prescribed cilia)
    f = std::fopen((p + ".par").c_str(), "w");
    if (!f) return set_error(CF_EINVAL, "cf_sim_write_config: cannot open %s.par", prefix);
    const double dl = c.seg_sep, L = dl * (nseg - 1);
    std::fprintf(f, "%d %%%% NFIL\n%d %%%% NSEG\n%d %%%% NSWIM\n%d %%%% NBLOB\n", F, nseg, 1, 0);
    std::fprintf(f, "%.15g %%%% MU\n%.15g %%%% RSEG\n%.15g %%%% DL\n%.15g %%%% FIL_LENGTH\n", 1.0, 1.0, dl, L);
    std::fprintf(f, "%.15g %%%% RBLOB\n%.15g %%%% KB\n%.15g %%%% KT\n", 1.0, 1800.0, 1800.0);
    std::fprintf(f, "%.15g %%%% TOL\n%d %%%% TOTAL_TIME_STEPS\n%.15g %%%% DT\n", c.gmres_tol, total_steps, c.dt);
    std::fprintf(f, "%d %%%% PLOT_FREQUENCY_IN_STEPS\n%d %%%% STEPS_PER_PERIOD\n", 10, 300);
    std::fprintf(f, "%d %%%% PRESCRIBED_CILIA\n", 1);
    if (s->d.dyn_angle) std::fprintf(f, "%.15g %%%% TORSIONAL_SPRING_MAGNITUDE_FACTOR\n", c.spring_factor);
    const bool ok2 = std::fclose(f) == 0;
    if (!ok1 || !ok2) return set_error(CF_EINVAL, "cf_sim_write_config: write under %s failed", prefix);
    return CF_OK;
}

extern "C" int cf_read_ic(const char *path, int n_fil, double *header, double *phase, double *angle) {
    clear_error();
    CF_REQUIRE(path && n_fil > 0 && phase && angle, "cf_read_ic: bad arguments");
    std::FILE *f = std::fopen(path, "r");
    if (!f) return set_error(CF_EINVAL, "cf_read_ic: cannot open %s", path);
    double h[2] = {0.0, 0.0};
    std::vector<double> v(2 * static_cast<size_t>(n_fil));
    int got = 0;
    for (int i = 0; i < 2 && std::fscanf(f, "%lf", &h[i]) == 1; ++i) ++got;
    size_t nv = 0;
    while (got == 2 && nv < v.size() && std::fscanf(f, "%lf", &v[nv]) == 1) ++nv;
    std::fclose(f);
    if (got < 2 || nv < v.size())
        return set_error(CF_EINVAL,
                         "cf_read_ic: %s holds %zu of the 2 + %d values (2 header values, %d phases, %d angles)",
                         path, got + nv, 2 * n_fil, n_fil, n_fil);
    if (header) {
        header[0] = h[0];
        header[1] = h[1];
    }
    std::memcpy(phase, v.data(), sizeof(double) * n_fil);
    std::memcpy(angle, v.data() + n_fil, sizeof(double) * n_fil);
    return CF_OK;
}

// The free swimmer (cf_swim): shares the beat kinematics above.
#include "swim_engine.cuh"

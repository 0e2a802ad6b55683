// sim.cu -- cf_sim: the device-resident implicit step for prescribed cilia on a wall.
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
#include "common.cuh"
#include "rpy_kernels.cuh"
#include "sim_kernels.cuh"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

using namespace cufil;

namespace {
constexpr int kIterLogCap = 4096;  // steps remembered by cf_sim_iteration_log
}

struct cf_sim {
    cf_sim_config cfg{};
    int num_sms = CF_B200_SMS;
    cudaStream_t stream = nullptr;
    cudaStream_t cap_stream = nullptr;  // captures the loop body
    SimDev d{};
    RpyBlockDesc desc{};
    RpyPlan plan{};
    float4 *partial = nullptr;
    int *err = nullptr;
    int fil_threads = 64;
    size_t kin_smem = 0, pre_smem = 0, givens_smem = 0;
    int dots_grid = 0, update_grid = 0;
    bool use_graph = true;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphConditionalHandle handle = 0;
    std::vector<void *> allocations;
};

namespace {

template <typename T>
int sim_alloc(cf_sim *s, T **p, size_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    void *q = nullptr;
    CF_CUDA(cudaMalloc(&q, n * sizeof(T)));
    s->allocations.push_back(q);
    *p = static_cast<T *>(q);
    return CF_OK;
}

template <typename T>
int sim_upload(cf_sim *s, T **p, const T *host, size_t n) {
    CF_TRY(sim_alloc(s, p, n));
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

int launch_kinematics(cf_sim *s, cudaStream_t st) {
    kinematics_kernel<<<s->d.F, s->fil_threads, s->kin_smem, st>>>(s->d);
    CF_CHECK_LAUNCH("kinematics_kernel");
    return CF_OK;
}

int launch_matvec_tail(cf_sim *s, const double *v, double *out, cudaStream_t st) {
    CF_TRY(rpy_launch_tiles(s->desc, s->plan, s->partial, s->err, st));
    const int warps_per_block = 8;
    saddle_epilogue_kernel<<<(s->d.N + warps_per_block - 1) / warps_per_block, 32 * warps_per_block, 0, st>>>(
        s->d, v, out);
    CF_CHECK_LAUNCH("saddle_epilogue_kernel");
    return CF_OK;
}

int launch_prologue(cf_sim *s, cudaGraphConditionalHandle h, cudaStream_t st) {
    CF_TRY(launch_kinematics(s, st));
    rhs_kernel<<<s->d.F, s->fil_threads, 0, st>>>(s->d);
    CF_CHECK_LAUNCH("rhs_kernel");
    CF_TRY(launch_matvec_tail(s, s->d.sol, s->d.w, st));
    residual_decide_kernel<<<s->d.F, s->fil_threads, 0, st>>>(s->d, h);
    CF_CHECK_LAUNCH("residual_decide_kernel");
    return CF_OK;
}

int launch_body(cf_sim *s, cudaGraphConditionalHandle h, cudaStream_t st) {
    arnoldi_precond_kernel<<<s->d.F, s->fil_threads, s->pre_smem, st>>>(s->d, h);
    CF_CHECK_LAUNCH("arnoldi_precond_kernel");
    CF_TRY(launch_matvec_tail(s, s->d.z, s->d.w, st));
    dots_kernel<<<s->dots_grid, 256, 0, st>>>(s->d, s->d.h1);
    CF_CHECK_LAUNCH("dots_kernel");
    update_kernel<<<s->update_grid, 256, 0, st>>>(s->d, s->d.h1, 0, h);
    CF_CHECK_LAUNCH("update_kernel");
    dots_kernel<<<s->dots_grid, 256, 0, st>>>(s->d, s->d.h2);
    CF_CHECK_LAUNCH("dots_kernel");
    update_kernel<<<s->update_grid, 256, s->givens_smem, st>>>(s->d, s->d.h2, 1, h);
    CF_CHECK_LAUNCH("update_kernel");
    return CF_OK;
}

int launch_finish(cf_sim *s, cudaStream_t st) {
    backsub_kernel<<<1, 256, sizeof(double) * (s->d.max_iter + 1), st>>>(s->d);
    CF_CHECK_LAUNCH("backsub_kernel");
    combine_kernel<<<s->update_grid, 256, 0, st>>>(s->d);
    CF_CHECK_LAUNCH("combine_kernel");
    finish_kernel<<<s->d.F, s->fil_threads, s->pre_smem, st>>>(s->d);
    CF_CHECK_LAUNCH("finish_kernel");
    return CF_OK;
}

// Captures prologue -> WHILE(body) -> finish into one executable graph.
int build_graph(cf_sim *s) {
    CF_TRY(rpy_prepare(s->desc, s->plan));
    cudaStream_t st = s->stream;
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
        if ((rc = cuda_status(cudaGraphConditionalHandleCreate(&s->handle, g, 0, cudaGraphCondAssignDefault),
                              "cudaGraphConditionalHandleCreate", __FILE__, __LINE__)))
            break;
        if ((rc = launch_prologue(s, s->handle, st))) break;
        if ((rc = cuda_status(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &ndeps),
                              "cudaStreamGetCaptureInfo", __FILE__, __LINE__)))
            break;
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = s->handle;
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
        if ((rc = cuda_status(cudaStreamBeginCaptureToGraph(s->cap_stream, body, nullptr, nullptr, 0,
                                                            cudaStreamCaptureModeThreadLocal),
                              "cudaStreamBeginCaptureToGraph", __FILE__, __LINE__)))
            break;
        rc = launch_body(s, s->handle, s->cap_stream);
        cudaGraph_t body_out = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(s->cap_stream, &body_out);
        if (rc) break;
        if ((rc = cuda_status(e2, "cudaStreamEndCapture(body)", __FILE__, __LINE__))) break;
        if ((rc = launch_finish(s, st))) break;
    } while (0);
    cudaGraph_t full = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &full);
    if (rc) {
        if (full) cudaGraphDestroy(full);
        return rc;
    }
    CF_TRY(cuda_status(e, "cudaStreamEndCapture", __FILE__, __LINE__));
    s->graph = full;
    CF_CUDA(cudaGraphInstantiate(&s->exec, s->graph, 0));
    return CF_OK;
}

int read_ctl(cf_sim *s, GmresCtl *out) {
    CF_CUDA(cudaMemcpyAsync(out, s->d.ctl, sizeof(GmresCtl), cudaMemcpyDeviceToHost, s->stream));
    CF_CUDA(cudaStreamSynchronize(s->stream));
    int flags = 0;
    CF_CUDA(cudaMemcpy(&flags, s->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (flags) {
        CF_CUDA(cudaMemset(s->err, 0, sizeof(int)));
        return set_error(CF_TIMEOUT, "sim: a bounded device wait gave up (flags 0x%x)", flags);
    }
    return CF_OK;
}

int status_of(const GmresCtl &c) {
    switch (c.status) {
        case kGmresMaxIter:
            return set_error(CF_NOT_CONVERGED, "GMRES stopped at its cap: %d iterations, relative residual %.3e",
                             c.iters, c.relres);
        case kGmresNonFinite:
            return set_error(CF_NONFINITE, "GMRES met a non-finite value (relative residual %.3e)", c.relres);
        default:
            return CF_OK;
    }
}

int run_step(cf_sim *s, int nt) {
    set_nt_kernel<<<1, 1, 0, s->stream>>>(s->d.ctl, nt);
    CF_CHECK_LAUNCH("set_nt_kernel");
    if (s->use_graph) {
        if (!s->exec) {
            int rc = build_graph(s);
            if (rc != CF_OK) {
                // Conditional graph nodes unavailable: fall back to the host-driven loop.
                cudaGetLastError();
                s->use_graph = false;
            }
        }
        if (s->use_graph) {
            CF_CUDA(cudaGraphLaunch(s->exec, s->stream));
            return CF_OK;
        }
    }
    CF_TRY(launch_prologue(s, 0, s->stream));
    GmresCtl c;
    CF_TRY(read_ctl(s, &c));
    int guard = 0;
    while (c.cond && guard++ <= s->d.max_iter) {
        CF_TRY(launch_body(s, 0, s->stream));
        CF_TRY(read_ctl(s, &c));
    }
    return launch_finish(s, s->stream);
}

}  // namespace

extern "C" int cf_sim_create(const cf_sim_config *cfg, cf_sim **out) {
    clear_error();
    CF_REQUIRE(cfg && out, "cf_sim_create: null argument");
    *out = nullptr;
    CF_REQUIRE(cfg->n_fil > 0 && cfg->n_seg >= 2 && cfg->n_seg <= 256,
               "cf_sim_create: need n_fil > 0 and 2 <= n_seg <= 256 (got %d, %d)", cfg->n_fil, cfg->n_seg);
    CF_REQUIRE(static_cast<long long>(cfg->n_fil) * cfg->n_seg < (1LL << 26), "cf_sim_create: too many segments");
    CF_REQUIRE(cfg->beat == CF_BEAT_FULFORD_BLAKE || cfg->beat == CF_BEAT_FULFORD_BLAKE_ORIGINAL,
               "cf_sim_create: unknown beat %d", cfg->beat);
    CF_REQUIRE(cfg->precond == CF_PRECOND_NONE || cfg->precond == CF_PRECOND_BLOCK_DIAG,
               "cf_sim_create: preconditioner %d not available in this entry point", cfg->precond);
    CF_REQUIRE(cfg->dt > 0 && cfg->seg_sep > 0, "cf_sim_create: dt and seg_sep must be positive");
    CF_REQUIRE(cfg->gmres_tol > 0 && cfg->gmres_max_iter > 0, "cf_sim_create: bad GMRES tolerance / cap");
    CF_REQUIRE(cfg->base_pos, "cf_sim_create: base_pos is required");
    CF_REQUIRE(!cfg->dynamic_phase || (cfg->gen_phase_force_refs && cfg->n_gen_phase_refs >= 2),
               "cf_sim_create: dynamic phase needs the reference generalised phase forces");
    CF_REQUIRE(!cfg->dynamic_angle || (cfg->gen_angle_force_refs && cfg->n_gen_angle_refs >= 2),
               "cf_sim_create: dynamic angle needs the reference generalised angle forces");
    CF_REQUIRE(!cfg->s_values_ref || (cfg->s_ref_rows >= 1 && cfg->s_ref_cols >= 2),
               "cf_sim_create: bad arclength table shape");
    CF_CUDA(cudaSetDevice(cfg->device));
    cf_sim *s = new (std::nothrow) cf_sim();
    if (!s) return set_error(CF_ENOMEM, "cf_sim_create: host allocation failed");
    s->cfg = *cfg;
    int rc = CF_OK;
    do {
        cudaDeviceProp prop;
        if ((rc = cuda_status(cudaGetDeviceProperties(&prop, cfg->device), "cudaGetDeviceProperties", __FILE__,
                              __LINE__)))
            break;
        s->num_sms = prop.multiProcessorCount;
        if ((rc = cuda_status(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "cudaStreamCreate",
                              __FILE__, __LINE__)))
            break;
        if ((rc = cuda_status(cudaStreamCreateWithFlags(&s->cap_stream, cudaStreamNonBlocking), "cudaStreamCreate",
                              __FILE__, __LINE__)))
            break;
        SimDev &d = s->d;
        const int F = cfg->n_fil, ns = cfg->n_seg, N = F * ns;
        d.F = F;
        d.nseg = ns;
        d.N = N;
        d.po = cfg->dynamic_phase ? 3 * N : -1;
        d.ao = cfg->dynamic_angle ? 3 * N + (cfg->dynamic_phase ? F : 0) : -1;
        d.n = 3 * N + F * ((cfg->dynamic_phase ? 1 : 0) + (cfg->dynamic_angle ? 1 : 0));
        d.ldq = (d.n + 31) / 32 * 32;
        d.max_iter = std::min(d.n, cfg->gmres_max_iter);
        d.ldh = d.max_iter + 1;
        d.flexible = 0;
        d.precond = cfg->precond == CF_PRECOND_BLOCK_DIAG ? 1 : 0;
        d.dt = cfg->dt;
        d.L = cfg->seg_sep * (ns - 1);  // FIL_LENGTH = DL*(NSEG_PER_CILIA-1), RSEG = 1
        d.spring = cfg->spring_factor;
        d.tol = cfg->gmres_tol;
        d.s_tol = (cfg->s_tol_factor > 0 ? cfg->s_tol_factor : 0.1) / ns;
        // Wall frame: rot_mat of (1/sqrt2, 0, -1/sqrt2, 0) maps the reference x axis to e_z.
        const double R[9] = {0, 0, -1, 0, 1, 0, 1, 0, 0};
        std::memcpy(d.R, R, sizeof(R));
        d.beat = beat_table(cfg->beat);
        d.s_rows = cfg->s_values_ref ? cfg->s_ref_rows : 0;
        d.s_cols = cfg->s_values_ref ? cfg->s_ref_cols : 0;
        d.n_phase_refs = cfg->dynamic_phase ? cfg->n_gen_phase_refs : 0;
        d.n_angle_refs = cfg->dynamic_angle ? cfg->n_gen_angle_refs : 0;

        std::vector<double> omega(F, 2.0 * 3.14159265358979323846), ph(F, 0.0), an(F, 0.0);
        if (cfg->omega0) std::copy(cfg->omega0, cfg->omega0 + F, omega.begin());
        if (cfg->phase0) std::copy(cfg->phase0, cfg->phase0 + F, ph.begin());
        if (cfg->angle0) std::copy(cfg->angle0, cfg->angle0 + F, an.begin());
        std::vector<double> zeros(F, 0.0);
        const double *cst;
        if ((rc = sim_upload(s, const_cast<double **>(&d.s_table), cfg->s_values_ref,
                             static_cast<size_t>(d.s_rows) * d.s_cols)) ||
            (rc = sim_upload(s, const_cast<double **>(&d.phase_refs), cfg->gen_phase_force_refs, d.n_phase_refs)) ||
            (rc = sim_upload(s, const_cast<double **>(&d.angle_refs), cfg->gen_angle_force_refs, d.n_angle_refs)) ||
            (rc = sim_upload(s, const_cast<double **>(&d.omega0), omega.data(), F)) ||
            (rc = sim_upload(s, const_cast<double **>(&d.base), cfg->base_pos, 3 * static_cast<size_t>(F))) ||
            (rc = sim_upload(s, &d.phase, ph.data(), F)) || (rc = sim_upload(s, &d.angle, an.data(), F)) ||
            (rc = sim_upload(s, &d.phase_dot, omega.data(), F)) ||  // phase_dot = omega0 (filament.cpp:472)
            (rc = sim_upload(s, &d.angle_dot, zeros.data(), F)))
            break;
        (void)cst;
        const size_t n = d.n, ldq = d.ldq, mi = d.max_iter;
        if ((rc = sim_alloc(s, &d.x4, N)) || (rc = sim_alloc(s, &d.xd, 3 * N)) || (rc = sim_alloc(s, &d.s_cur, N)) || (rc = sim_alloc(s, &d.kp, 3 * N)) ||
            (rc = sim_alloc(s, &d.ka, 3 * N)) || (rc = sim_alloc(s, &d.gram, 3 * F)) ||
            (rc = sim_alloc(s, &d.rhs, n)) || (rc = sim_alloc(s, &d.sol, n)) || (rc = sim_alloc(s, &d.w, n)) ||
            (rc = sim_alloc(s, &d.z, n)) || (rc = sim_alloc(s, &d.t, n)) || (rc = sim_alloc(s, &d.y, mi + 1)) ||
            (rc = sim_alloc(s, &d.Q, (mi + 1) * ldq)) || (rc = sim_alloc(s, &d.H, (mi + 2) * (mi + 1))) ||
            (rc = sim_alloc(s, &d.cs, mi + 1)) || (rc = sim_alloc(s, &d.sn, mi + 1)) ||
            (rc = sim_alloc(s, &d.beta, mi + 2)) || (rc = sim_alloc(s, &d.h1, mi + 2)) ||
            (rc = sim_alloc(s, &d.h2, mi + 2)) || (rc = sim_alloc(s, &d.f4, N)) || (rc = sim_alloc(s, &d.ctl, 1)) ||
            (rc = sim_alloc(s, &d.iter_log, kIterLogCap)) ||
            (rc = sim_alloc(s, &s->err, 1)))
            break;
        d.Z = nullptr;
        d.iter_log_cap = kIterLogCap;
        if ((rc = cuda_status(cudaMemset(d.iter_log, 0, sizeof(int) * kIterLogCap), "cudaMemset", __FILE__, __LINE__)))
            break;
        // initial solution: lambda = 0, phase rate = omega0, angle rate = 0
        std::vector<double> sol(n, 0.0);
        if (d.po >= 0)
            for (int m = 0; m < F; ++m) sol[d.po + m] = omega[m];
        if ((rc = cuda_status(cudaMemcpy(d.sol, sol.data(), n * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy",
                              __FILE__, __LINE__)))
            break;
        // pair-kernel plan (wall, 3x3, segments on segments)
        RpyBlockDesc &desc = s->desc;
        desc.wall = 1;
        desc.vd = 3;
        desc.fd = 3;
        desc.self_set = 1;
        desc.xt = d.x4;
        desc.nt = N;
        desc.at = 1.0f;
        desc.xs = d.x4;
        desc.fs = d.f4;
        desc.ts = nullptr;
        desc.ns = N;
        desc.as = 1.0f;
        desc.mu = 1.0f;
        s->plan = rpy_plan_for(desc, s->num_sms);
        if ((rc = sim_alloc(s, &s->partial, s->plan.scratch_float4))) break;
        d.partial = s->partial;
        d.nsplit = s->plan.nsplit;
        // launch shapes
        s->fil_threads = std::min(256, std::max(64, (3 * ns + 31) / 32 * 32));
        s->kin_smem = sizeof(double) * (2 * (10 * ns + 1) + ns);
        s->pre_smem = sizeof(double) * 3 * ns;
        s->givens_smem = sizeof(double) * 3 * (d.max_iter + 2);
        d.dots_chunk = 4096;
        d.dots_nchunk = (d.n + d.dots_chunk - 1) / d.dots_chunk;
        s->dots_grid = 2 * s->num_sms;
        s->update_grid = std::min(8 * s->num_sms, (d.n + 31) / 32);
        if ((rc = sim_alloc(s, &d.dots_partial, (mi + 1) * d.dots_nchunk)) ||
            (rc = sim_alloc(s, &d.norm_partial, std::max(F, std::max(s->update_grid, s->dots_grid)))))
            break;
        if ((rc = cuda_status(cudaMemset(d.ctl, 0, sizeof(GmresCtl)), "cudaMemset", __FILE__, __LINE__)) ||
            (rc = cuda_status(cudaMemset(s->err, 0, sizeof(int)), "cudaMemset", __FILE__, __LINE__)) ||
            (rc = cuda_status(cudaMemset(d.H, 0, sizeof(double) * (mi + 2) * (mi + 1)), "cudaMemset", __FILE__,
                              __LINE__)))
            break;
        if (s->givens_smem > 48 * 1024) {
            if ((rc = cuda_status(cudaFuncSetAttribute(update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       static_cast<int>(s->givens_smem)),
                                  "cudaFuncSetAttribute", __FILE__, __LINE__)))
                break;
        }
        if (s->kin_smem > 48 * 1024) {
            if ((rc = cuda_status(cudaFuncSetAttribute(kinematics_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       static_cast<int>(s->kin_smem)),
                                  "cudaFuncSetAttribute", __FILE__, __LINE__)))
                break;
        }
        const char *ng = std::getenv("CUFIL_NO_GRAPH");
        s->use_graph = !(ng && ng[0] == '1');
    } while (0);
    if (rc != CF_OK) {
        std::string msg = cf_last_error();
        cf_sim_destroy(s);
        set_error(rc, "%s", msg.c_str());
        return rc;
    }
    *out = s;
    return CF_OK;
}

extern "C" int cf_sim_destroy(cf_sim *s) {
    if (!s) return CF_OK;
    cudaSetDevice(s->cfg.device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->exec) cudaGraphExecDestroy(s->exec);
    if (s->graph) cudaGraphDestroy(s->graph);
    for (void *p : s->allocations) cudaFree(p);
    if (s->cap_stream) cudaStreamDestroy(s->cap_stream);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return CF_OK;
}

extern "C" int cf_sim_step_async(cf_sim *s, int nt) {
    clear_error();
    CF_REQUIRE(s, "null handle");
    CF_REQUIRE(nt >= 0, "cf_sim_step: nt must be >= 0");
    CF_CUDA(cudaSetDevice(s->cfg.device));
    return run_step(s, nt);
}

extern "C" int cf_sim_last_solve(cf_sim *s, int *iters, double *relres) {
    clear_error();
    CF_REQUIRE(s, "null handle");
    CF_CUDA(cudaSetDevice(s->cfg.device));
    GmresCtl c;
    CF_TRY(read_ctl(s, &c));
    if (iters) *iters = (c.status == kGmresConverged || c.status == kGmresMaxIter) ? c.iters : 0;
    if (relres) *relres = c.relres;
    return status_of(c);
}

extern "C" int cf_sim_step(cf_sim *s, int nt, int *iters, double *relres) {
    CF_TRY(cf_sim_step_async(s, nt));
    return cf_sim_last_solve(s, iters, relres);
}

extern "C" int cf_sim_get_state(cf_sim *s, double *phase, double *angle, double *phase_dot, double *angle_dot) {
    clear_error();
    CF_REQUIRE(s, "null handle");
    CF_CUDA(cudaSetDevice(s->cfg.device));
    const size_t b = sizeof(double) * s->d.F;
    if (phase) CF_CUDA(cudaMemcpyAsync(phase, s->d.phase, b, cudaMemcpyDeviceToHost, s->stream));
    if (angle) CF_CUDA(cudaMemcpyAsync(angle, s->d.angle, b, cudaMemcpyDeviceToHost, s->stream));
    if (phase_dot) CF_CUDA(cudaMemcpyAsync(phase_dot, s->d.phase_dot, b, cudaMemcpyDeviceToHost, s->stream));
    if (angle_dot) CF_CUDA(cudaMemcpyAsync(angle_dot, s->d.angle_dot, b, cudaMemcpyDeviceToHost, s->stream));
    CF_CUDA(cudaStreamSynchronize(s->stream));
    return CF_OK;
}

extern "C" int cf_sim_get_segments(cf_sim *s, float *x_segs, float *f_segs) {
    clear_error();
    CF_REQUIRE(s, "null handle");
    CF_CUDA(cudaSetDevice(s->cfg.device));
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

extern "C" int cf_sim_get_directions(cf_sim *s, double *k_phase, double *k_angle) {
    clear_error();
    CF_REQUIRE(s, "null handle");
    CF_CUDA(cudaSetDevice(s->cfg.device));
    const size_t b = sizeof(double) * 3 * s->d.N;
    if (k_phase) CF_CUDA(cudaMemcpyAsync(k_phase, s->d.kp, b, cudaMemcpyDeviceToHost, s->stream));
    if (k_angle) CF_CUDA(cudaMemcpyAsync(k_angle, s->d.ka, b, cudaMemcpyDeviceToHost, s->stream));
    CF_CUDA(cudaStreamSynchronize(s->stream));
    return CF_OK;
}

extern "C" int cf_sim_get_arclengths(cf_sim *s, double *s_values) {
    clear_error();
    CF_REQUIRE(s && s_values, "null argument");
    CF_CUDA(cudaSetDevice(s->cfg.device));
    CF_CUDA(cudaMemcpyAsync(s_values, s->d.s_cur, sizeof(double) * s->d.N, cudaMemcpyDeviceToHost, s->stream));
    CF_CUDA(cudaStreamSynchronize(s->stream));
    return CF_OK;
}

extern "C" int cf_sim_system_size(cf_sim *s) { return s ? s->d.n : -1; }

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
    CF_CUDA(cudaSetDevice(s->cfg.device));
    const size_t b = sizeof(double) * s->d.F;
    if (phase) CF_CUDA(cudaMemcpyAsync(s->d.phase, phase, b, cudaMemcpyHostToDevice, s->stream));
    if (angle) CF_CUDA(cudaMemcpyAsync(s->d.angle, angle, b, cudaMemcpyHostToDevice, s->stream));
    // the rates are both filament state and the GMRES warm start (mobility_solver.cpp:2298-2388)
    if (phase_dot) {
        CF_CUDA(cudaMemcpyAsync(s->d.phase_dot, phase_dot, b, cudaMemcpyHostToDevice, s->stream));
        if (s->d.po >= 0)
            CF_CUDA(cudaMemcpyAsync(s->d.sol + s->d.po, phase_dot, b, cudaMemcpyHostToDevice, s->stream));
    }
    if (angle_dot) {
        CF_CUDA(cudaMemcpyAsync(s->d.angle_dot, angle_dot, b, cudaMemcpyHostToDevice, s->stream));
        if (s->d.ao >= 0)
            CF_CUDA(cudaMemcpyAsync(s->d.sol + s->d.ao, angle_dot, b, cudaMemcpyHostToDevice, s->stream));
    }
    return CF_OK;
}

extern "C" int cf_sim_iteration_log(cf_sim *s, int *iters, int n) {
    clear_error();
    CF_REQUIRE(s && iters && n >= 0 && n <= kIterLogCap, "cf_sim_iteration_log: bad arguments");
    CF_CUDA(cudaSetDevice(s->cfg.device));
    CF_CUDA(cudaMemcpyAsync(iters, s->d.iter_log, sizeof(int) * n, cudaMemcpyDeviceToHost, s->stream));
    CF_CUDA(cudaStreamSynchronize(s->stream));
    return CF_OK;
}

extern "C" int cf_sim_launches_per_step(cf_sim *s, int iters) {
    // set_nt + kinematics, rhs, tiles, epilogue, residual + 7 per iteration + backsub, combine, finish
    (void)s;
    return 1 + 5 + 7 * iters + 3;
}

extern "C" int cf_sim_initial_guess(cf_sim *s, int nt) {
    clear_error();
    CF_REQUIRE(s, "null handle");
    CF_CUDA(cudaSetDevice(s->cfg.device));
    set_nt_kernel<<<1, 1, 0, s->stream>>>(s->d.ctl, nt);
    CF_CHECK_LAUNCH("set_nt_kernel");
    CF_TRY(launch_kinematics(s, s->stream));
    CF_CUDA(cudaStreamSynchronize(s->stream));
    return CF_OK;
}

extern "C" int cf_sim_assemble_rhs(cf_sim *s, int nt, double *rhs) {
    clear_error();
    CF_REQUIRE(s && rhs, "null argument");
    CF_CUDA(cudaSetDevice(s->cfg.device));
    set_nt_kernel<<<1, 1, 0, s->stream>>>(s->d.ctl, nt);
    rhs_kernel<<<s->d.F, s->fil_threads, 0, s->stream>>>(s->d);
    CF_CHECK_LAUNCH("rhs_kernel");
    CF_CUDA(cudaMemcpyAsync(rhs, s->d.rhs, sizeof(double) * s->d.n, cudaMemcpyDeviceToHost, s->stream));
    CF_CUDA(cudaStreamSynchronize(s->stream));
    return CF_OK;
}

extern "C" int cf_sim_apply_preconditioner(cf_sim *s, const double *in, double *out) {
    clear_error();
    CF_REQUIRE(s && in && out, "null argument");
    CF_CUDA(cudaSetDevice(s->cfg.device));
    const size_t b = sizeof(double) * s->d.n;
    CF_CUDA(cudaMemcpyAsync(s->d.t, in, b, cudaMemcpyHostToDevice, s->stream));
    precond_kernel<<<s->d.F, s->fil_threads, s->pre_smem, s->stream>>>(s->d, s->d.t, s->d.t);
    CF_CHECK_LAUNCH("precond_kernel");
    CF_CUDA(cudaMemcpyAsync(out, s->d.t, b, cudaMemcpyDeviceToHost, s->stream));
    CF_CUDA(cudaStreamSynchronize(s->stream));
    return CF_OK;
}

extern "C" int cf_sim_system_matvec(cf_sim *s, const double *in, double *out) {
    clear_error();
    CF_REQUIRE(s && in && out, "null argument");
    CF_CUDA(cudaSetDevice(s->cfg.device));
    const size_t b = sizeof(double) * s->d.n;
    CF_CUDA(cudaMemcpyAsync(s->d.z, in, b, cudaMemcpyHostToDevice, s->stream));
    pack_forces_kernel<<<(s->d.N + 255) / 256, 256, 0, s->stream>>>(s->d, s->d.z);
    CF_CHECK_LAUNCH("pack_forces_kernel");
    filament_rows_kernel<<<s->d.F, s->fil_threads, 0, s->stream>>>(s->d, s->d.z, s->d.w);
    CF_CHECK_LAUNCH("filament_rows_kernel");
    CF_TRY(launch_matvec_tail(s, s->d.z, s->d.w, s->stream));
    CF_CUDA(cudaMemcpyAsync(out, s->d.w, b, cudaMemcpyDeviceToHost, s->stream));
    GmresCtl c;
    return read_ctl(s, &c);
}

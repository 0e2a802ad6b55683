// ref_fcm_wrapper.cu -- C entry points around the reference's OWN cuFCM solver
// (test infrastructure only).  Compiled by oracle/ref_build.py together with
// the reference's src/cufcm/*.cu read in place (never copied); FCM_solver is
// constructed from a Pars record exactly as the reference's drivers do
// (CUFCM_SOLVER.cu:20-34) and run through FCM_solver::hydrodynamic_solver
// (:363-436), which leaves its results in the caller's V array, input order.
// Same header order as the reference's CUFCM_SOLVER.cu (CUFCM_DATA.cuh brings in cuRAND).
#include "config.hpp"
#include "CUFCM_FCM.cuh"
#include "CUFCM_CORRECTION.cuh"
#include "CUFCM_DATA.cuh"
#include "CUFCM_SOLVER.cuh"

extern "C" {

void *ref_fcm_create(int n, float rh, float alpha, float beta, float eta, int nx, int ny, int nz, float boxsize) {
    Pars p;
    p.N = n;
    p.rh = rh;
    p.alpha = alpha;
    p.beta = beta;
    p.eta = eta;
    p.nx = nx;
    p.ny = ny;
    p.nz = nz;
    p.repeat = 1 << 16;  // the solver keeps per-call timing slots; plenty for a test session
    p.prompt = -1;       // silent
    p.boxsize = boxsize;
    p.checkerror = 0;
    return new FCM_solver(p);
}

// Device arrays [3n]; Y and F are permuted in place during the call and
// restored by the solver's own sort-back.
int ref_fcm_apply(void *s, float *Y, float *F, float *T, float *V, float *W) {
    static_cast<FCM_solver *>(s)->hydrodynamic_solver(Y, F, T, V, W);
    return static_cast<int>(cudaDeviceSynchronize());
}

}  // extern "C"

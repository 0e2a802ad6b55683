// ref_flow_wrapper.cu -- a C entry point around the reference's OWN flow-field
// kernel (test infrastructure only).  Compiled by oracle/ref_build.py together
// with src/flow_field/flow_field_evaluator.cu, read in place from the
// reference tree (#included below, never copied), in FP64 (the reference's
// flow_field_main reads its inputs with "%lf", so only its FP64 build is
// usable).  The kernel is launched as flow_field_evaluator::velocities
// launches it (flow_field_evaluator.cu:545-557): one thread per flow point,
// THREADS_PER_BLOCK-wide blocks, prefactor 1/(8 pi MU).
//
// config.hpp defines MU and RSEG as macros, which collide with the data members
// of the same names in flow_field_evaluator.hpp:21-22; the reference's flow-field
// target does not compile against the current config.hpp for that reason, so
// the macros are dropped here before the reference's sources are included.
#include "config.hpp"
#undef MU
#undef RSEG
#include "flow_field_evaluator.cu"

extern "C" {

int ref_flow_real_size(void) { return (int)sizeof(Real); }

// Device arrays in the reference's layouts.
int ref_flow_velocities(Real *Vf, const Real *Xf, const Real *Fs, const Real *Fb, const Real *Xs, const Real *Xbody,
                        const Real *Xb, int Nf, int Ns, int Nbods, int Nb, double mu, int remove_net_force) {
    const Real prefac = 1.0 / (8.0 * PI * mu);
    const int blocks = (Nf + THREADS_PER_BLOCK - 1) / THREADS_PER_BLOCK;
    if (Nf > 0)
        flow_velocities<<<blocks, THREADS_PER_BLOCK>>>(Vf, Xf, Fs, Fb, Xs, Xbody, Xb, Nf, Ns, Nbods, Nb, prefac,
                                                       remove_net_force);
    return (int)cudaDeviceSynchronize();
}

}  // extern "C"

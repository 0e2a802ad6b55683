// ref_rpy_wrapper.cu -- C entry points around the reference's OWN RPY kernels
// (test infrastructure only).
//
// This file is compiled by oracle/ref_build.py together with the reference's
// src/cilia/cuda_functions.cu, read in place from the reference tree (it is
// #included below, never copied).  A generated configuration header selects the
// variant (wall / unbounded, 3- or 6-dof segments) and is pre-included so that
// the reference's own config.hpp include guard makes it a no-op.  The kernels
// are launched exactly as rpy_mobility_solver.cu:258-328 launches them: one
// thread per target, THREADS_PER_BLOCK-wide blocks, globals set by sync_var.
#include "cuda_functions.cu"

extern "C" {

// sync_var launch of cilia_sim_main.cu:154 (sizes only; the other globals are
// not read by the RPY kernels).
int ref_set_sizes(int nswim, int nseg, int nfil, int nblob) {
    sync_var<<<1, 1>>>(nswim, nseg, nfil, nblob, 0, (Real)1.0, (Real)1.0);
    return (int)cudaDeviceSynchronize();
}

int ref_real_size(void) { return (int)sizeof(Real); }
int ref_prescribed(void) { return (int)PRESCRIBED_CILIA; }
int ref_wall(void) { return (int)INFINITE_PLANE_WALL; }

static int blocks_for(int n) { return (n + THREADS_PER_BLOCK - 1) / THREADS_PER_BLOCK; }

// Device pointers in the reference's layouts (rpy_mobility_solver.cu:105-115).
int ref_mss(Real *v_segs, const Real *f_segs, const Real *x_segs, int start_seg, int num_segs) {
    if (num_segs > 0) Mss_mult<<<blocks_for(num_segs), THREADS_PER_BLOCK>>>(v_segs, f_segs, x_segs, start_seg, num_segs);
    return (int)cudaDeviceSynchronize();
}

int ref_msb(Real *v_segs, const Real *f_blobs, const Real *x_segs, const Real *x_blobs, int start_seg, int num_segs) {
    if (num_segs > 0)
        Msb_mult<<<blocks_for(num_segs), THREADS_PER_BLOCK>>>(v_segs, f_blobs, x_segs, x_blobs, start_seg, num_segs);
    return (int)cudaDeviceSynchronize();
}

int ref_mbb(Real *v_blobs, const Real *f_blobs, const Real *x_blobs, int start_blob, int num_blobs) {
    if (num_blobs > 0)
        Mbb_mult<<<blocks_for(num_blobs), THREADS_PER_BLOCK>>>(v_blobs, f_blobs, x_blobs, start_blob, num_blobs);
    return (int)cudaDeviceSynchronize();
}

int ref_mbs(Real *v_blobs, const Real *f_segs, const Real *x_blobs, const Real *x_segs, int start_blob, int num_blobs) {
    if (num_blobs > 0)
        Mbs_mult<<<blocks_for(num_blobs), THREADS_PER_BLOCK>>>(v_blobs, f_segs, x_blobs, x_segs, start_blob, num_blobs);
    return (int)cudaDeviceSynchronize();
}

// Asynchronous Mss launch for timing (no synchronisation), on the legacy stream.
int ref_mss_async(Real *v_segs, const Real *f_segs, const Real *x_segs, int start_seg, int num_segs) {
    if (num_segs > 0) Mss_mult<<<blocks_for(num_segs), THREADS_PER_BLOCK>>>(v_segs, f_segs, x_segs, start_seg, num_segs);
    return (int)cudaGetLastError();
}

}  // extern "C"

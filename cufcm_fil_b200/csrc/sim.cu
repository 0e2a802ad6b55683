// sim.cu -- implicit prescribed-cilia step (placeholder entry points until the device solver lands).
#include "common.cuh"

using namespace cufil;

#define CF_STUB(sig) extern "C" sig { return set_error(CF_ENOTSUP, "not implemented yet"); }
CF_STUB(int cf_sim_create(const cf_sim_config *, cf_sim **))
CF_STUB(int cf_sim_destroy(cf_sim *))
CF_STUB(int cf_sim_step(cf_sim *, int, int *, double *))
CF_STUB(int cf_sim_step_async(cf_sim *, int))
CF_STUB(int cf_sim_last_solve(cf_sim *, int *, double *))
CF_STUB(int cf_sim_get_state(cf_sim *, double *, double *, double *, double *))
CF_STUB(int cf_sim_get_segments(cf_sim *, float *, float *))
CF_STUB(int cf_sim_get_directions(cf_sim *, double *, double *))
CF_STUB(int cf_sim_system_size(cf_sim *))
CF_STUB(int cf_sim_initial_guess(cf_sim *, int))
CF_STUB(int cf_sim_assemble_rhs(cf_sim *, int, double *))
CF_STUB(int cf_sim_apply_preconditioner(cf_sim *, const double *, double *))
CF_STUB(int cf_sim_system_matvec(cf_sim *, const double *, double *))

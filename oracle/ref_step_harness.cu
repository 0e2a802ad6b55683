// ref_step_harness.cu -- runs the reference's own prescribed-cilia time step
// (test infrastructure only: a checker and a timed baseline, never product).
//
// The reference's host code is compiled in place, unmodified, from its own
// sources by oracle/ref_build.py (mobility_solver.cpp, filament.cpp,
// swimmer.cpp, segment.cpp, rigid_body.cpp, broyden_solver.cpp, matrix.cpp,
// quaternion.cpp, seeding.cu, util.cu, globals.cu) against a generated
// config.hpp variant, and linked with this driver.  So the RHS
// (mobility_solver.cpp:284-634), the block-diagonal preconditioner
// (:1102-1594), the saddle product (:1887-2185), the right-preconditioned
// GMRES (:2187-2669), the Fulford-Blake beat and its arclength bisection
// (filament.cpp:962-1500) and the time stepping are the reference's own.
//
// Mobility back-ends (mobility_solver.hpp:26-46):
//   REF_HARNESS_GPU defined: the reference's rpy_mobility_solver with its
//     Mss_mult kernel (rpy_mobility_solver.cu, cuda_functions.cu), i.e. the
//     reference's whole GPU path, FP32 as the reference ships it;
//   otherwise: host_rpy_solver below, which evaluates V = M F with the
//     oracle's FP64 restatement of the wall RPY pair (rpy_oracle.c), so the
//     whole step runs in FP64 on the CPU.
//
// The driver follows the order of cilia_sim_main.cu:56-575: globals from the
// command line instead of globals.ini (:59-146), mobility.initialise() (reads
// the generalised-force tables, :248-249), swimmer set-up (:260-266), the
// s-value table (:318-375), then per step initial_guess, forces_and_torques,
// compute_velocities, [generalised forces], end_of_step (:405-575).
//
// Usage (run in a directory holding input/forcing/ and the IC file):
//   ref_step_* wgf  <nseg> <seg_sep> <out.bin>
//       the WRITE_GENERALISED_FORCES pre-run (binary built with that switch):
//       writes input/forcing/..._{phase,angle}_generalised_forces_... and
//       ..._s_values_... exactly as the reference does.
//   ref_step_* run  <nseg> <nfil> <fil_x_dim> <spacing> <seg_sep> <spring> <steps> <ic_file> <out.bin> [write]
//       (a body variant reads <nblob> <ar> in place of <fil_x_dim> <spacing>, the seeding files
//       input/fourier_modes/sphere<N>.{seed,polar_dir,azi_dir,normal} of swimmer.cpp:310-345 and
//       rigid_body.cpp:330-380 from the run directory, and appends the body's position,
//       orientation and velocity to each record)
//       the dynamic run.  out.bin: per step, doubles
//       [iterations, seconds, phase[F], angle[F], phase_dot[F], angle_dot[F], x_tip[3F]].
//       With "write", the reference's data files (ref_step_seg_states.dat, _body_states.dat,
//       _true_states.dat, _seg_vels.dat, _seg_forces.dat) are appended every
//       PLOT_FREQUENCY_IN_STEPS steps by the reference's own writers, as its main loop does
//       (cilia_sim_main.cu:624-718).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <string>
#include <vector>

#include "swimmer.hpp"
#include "mobility_solver.hpp"
#include "util.hpp"

#ifdef REF_HARNESS_GPU
#include "rpy_mobility_solver.hpp"
#include "cuda_functions.hpp"
typedef rpy_mobility_solver harness_mobility_solver;
#else
#include <cstdint>
extern "C" void oracle_rpy_apply_f64(int wall, int vdof, int fdof, int self_by_index, int64_t nt, const double *xt,
                                     double at, const int64_t *t_ids, int64_t t_off, int64_t ns, const double *xs,
                                     const double *fs, double as, int64_t s_off, double mu, double *vt, int nthreads);

// A CPU back-end of the reference's mobility_solver: host arrays only, and
// the segment-segment product of Mss_mult (cuda_functions.cu:362-474: all
// sources, 3-dof forces read from the 6-strided force array, the six velocity
// slots written) evaluated by the oracle's FP64 wall RPY sum.
class host_rpy_solver : public mobility_solver {
  public:
    std::vector<double> xs, fs, vs;

    void allocate_host_memory() override {
        const int ns = NSWIM * NFIL * NSEG, nb = NSWIM * NBLOB;
        v_segs_host = new Real[6 * ns];
        x_segs_host = new Real[3 * ns];
        f_segs_host = new Real[6 * ns];
        v_blobs_host = new Real[3 * nb + 1];
        x_blobs_host = new Real[3 * nb + 1];
        f_blobs_host = new Real[3 * nb + 1];
        f_blobs_repulsion_host = new Real[3 * nb + 1];
        std::memset(f_segs_host, 0, 6 * ns * sizeof(Real));
        xs.resize(3 * ns);
        fs.resize(3 * ns);
        vs.resize(3 * ns);
    }
    void free_host_memory() override {
        delete[] v_segs_host;
        delete[] x_segs_host;
        delete[] f_segs_host;
        delete[] v_blobs_host;
        delete[] x_blobs_host;
        delete[] f_blobs_host;
        delete[] f_blobs_repulsion_host;
    }
    void allocate_device_memory() override {}
    void free_device_memory() override {}
    void copy_segment_positions_to_device() override {}
    void copy_segment_forces_to_device() override {}
    void copy_blob_positions_to_device() override {}
    void copy_blob_forces_to_device() override {}
    void copy_interparticle_blob_forces_to_host() override {}
    void copy_blob_velocities_to_host() override {}
    void copy_segment_velocities_to_host() override {}
    void apply_interparticle_forces() override {}
    void wait_for_device() override {}
#if !INFINITE_PLANE_WALL
    // Bodies: unbounded RPY over the segments and blobs together (all radii 1; a particle's own block
    // is the coincident-sphere branch), V_seg = M_ss F_seg + M_sb F_blob, V_blob = M_bs F_seg + M_bb F_blob.
    std::vector<double> xa, fa, va;
    void evaluate_full_mobility() override {
        const int ns = NSWIM * NFIL * NSEG, nb = NSWIM * NBLOB, n = ns + nb;
        xa.assign(3 * n, 0.0);
        fa.assign(3 * n, 0.0);
        va.assign(3 * n, 0.0);
        for (int i = 0; i < ns; ++i)
            for (int c = 0; c < 3; ++c) {
                xa[3 * i + c] = x_segs_host[3 * i + c];
                fa[3 * i + c] = f_segs_host[6 * i + c];
            }
        for (int i = 0; i < nb; ++i)
            for (int c = 0; c < 3; ++c) {
                xa[3 * (ns + i) + c] = x_blobs_host[3 * i + c];
                fa[3 * (ns + i) + c] = f_blobs_host[3 * i + c];
            }
        oracle_rpy_apply_f64(0, 3, 3, 0, n, xa.data(), 1.0, nullptr, 0, n, xa.data(), fa.data(), 1.0, 0, 1.0,
                             va.data(), 0);
        for (int i = 0; i < ns; ++i) {
            for (int c = 0; c < 3; ++c) v_segs_host[6 * i + c] = static_cast<Real>(va[3 * i + c]);
            for (int c = 3; c < 6; ++c) v_segs_host[6 * i + c] = 0;
        }
        for (int i = 0; i < nb; ++i)
            for (int c = 0; c < 3; ++c) v_blobs_host[3 * i + c] = static_cast<Real>(va[3 * (ns + i) + c]);
    }
    void evaluate_segment_segment_mobility() override { evaluate_full_mobility(); }
    void evaluate_segment_blob_mobility() override {}
    void evaluate_blob_blob_mobility() override {}
    void evaluate_blob_segment_mobility() override {}
};
#else
    void evaluate_segment_segment_mobility() override {
        const int ns = NSWIM * NFIL * NSEG;
        for (int i = 0; i < ns; ++i)
            for (int c = 0; c < 3; ++c) {
                xs[3 * i + c] = x_segs_host[3 * i + c];
                fs[3 * i + c] = f_segs_host[6 * i + c];
            }
        std::fill(vs.begin(), vs.end(), 0.0);
        oracle_rpy_apply_f64(1, 3, 3, 1, ns, xs.data(), 1.0, nullptr, 0, ns, xs.data(), fs.data(), 1.0, 0, 1.0,
                             vs.data(), 0);
        for (int i = 0; i < ns; ++i) {
            for (int c = 0; c < 3; ++c) v_segs_host[6 * i + c] = static_cast<Real>(vs[3 * i + c]);
            for (int c = 3; c < 6; ++c) v_segs_host[6 * i + c] = 0;
        }
    }
    // No blobs on the wall (cilia_sim_main.cu:96-99 forces NBLOB = 0).
    void evaluate_segment_blob_mobility() override {}
    void evaluate_blob_blob_mobility() override {}
    void evaluate_blob_segment_mobility() override {}
    void evaluate_full_mobility() override { evaluate_segment_segment_mobility(); }
};
#endif
typedef host_rpy_solver harness_mobility_solver;
#endif

namespace {

void usage() {
    std::fprintf(stderr,
                 "usage: ref_step wgf <nseg> <seg_sep> <out.bin>\n"
                 "       ref_step run <nseg> <nfil> <fil_x_dim> <spacing> <seg_sep> <spring> <steps> <ic_file> "
                 "<out.bin>\n");
    std::exit(2);
}

// The globals cilia_sim_main.cu reads from globals.ini (:59-91) and derives (:93-146).
void set_globals(int nseg, int nfil, double fil_x_dim, double spacing, double seg_sep, double spring, int steps,
                 const std::string &ic_file) {
    NSWIM = 1;
    NSEG = nseg;
    NFIL = nfil;
    NBLOB = 0;
    AR = 1;
#if !INFINITE_PLANE_WALL
    // A rigid body: the run line's lattice fields carry the blob count and the aspect ratio AR
    // (AXIS_DIR_BODY_LENGTH = AR * FIL_LENGTH, the diameter of a spherical body).
    NBLOB = static_cast<int>(fil_x_dim);
    AR = static_cast<Real>(spacing);
#endif
    SEG_SEP = static_cast<Real>(seg_sep);
    PERIOD = 1;
    SIM_LENGTH = 1;
    TORSIONAL_SPRING_MAGNITUDE_FACTOR = static_cast<Real>(spring);
    TILT_ANGLE = 0;
    PAIR_DP = 0;
    WAVNUM = 0;
    WAVNUM_DIA = 0;
    DIMENSIONLESS_FORCE = 220;
    FENE_MODEL = 0;
    FORCE_NOISE_MAG = 0;
    OMEGA_SPREAD = 0;
    INDEX = 0;
    FIL_X_DIM = static_cast<Real>(fil_x_dim);
    FIL_SPACING = static_cast<Real>(spacing);
    BLOB_X_DIM = 1;
    BLOB_SPACING = static_cast<Real>(spacing);
    HEX_NUM = 1;
    REV_RATIO = 0;
    TWOFIL_ANGLE = 0;
    GEN_FORCE_MAGNITUDE_FACTOR = 1;
    SIMULATION_DIR = "./";
    SIMULATION_FILE = "ref_step";
    SIMULATION_ICSTATE_NAME = ic_file;
    SIMULATION_NAME = SIMULATION_DIR + SIMULATION_FILE;
    SIMULATION_SEG_STATE_NAME = SIMULATION_NAME + "_seg_states.dat";
    SIMULATION_BODY_STATE_NAME = SIMULATION_NAME + "_body_states.dat";
    SIMULATION_SEG_VEL_NAME = SIMULATION_NAME + "_seg_vels.dat";
    SIMULATION_SEG_FORCES_NAME = SIMULATION_NAME + "_seg_forces.dat";
    SIMULATION_TRUESTATE_NAME = SIMULATION_NAME + "_true_states.dat";
#if WRITE_GENERALISED_FORCES
    NSWIM = 1;
    NFIL = 1;
    NBLOB = 0;
#endif
    NSEG_PER_CILIA = NSEG;
    NPAIR = NFIL;
    NTOTAL = NSWIM * (NFIL * NSEG + NBLOB);
    DL = SEG_SEP * RSEG;
    AXIS_DIR_BODY_LENGTH = AR * FIL_LENGTH;
    END_FORCE_MAGNITUDE = DIMENSIONLESS_FORCE * KB / (DL * DL * NSEG_PER_CILIA * NSEG_PER_CILIA);
    DT = PERIOD / STEPS_PER_PERIOD;
    TOTAL_TIME_STEPS = steps;
#if WRITE_GENERALISED_FORCES
    PERIOD = 1.0;
    DT = 1.0 / STEPS_PER_PERIOD;
    TOTAL_TIME_STEPS = STEPS_PER_PERIOD;
#endif
#ifdef REF_HARNESS_GPU
    sync_var<<<1, 1>>>(NSWIM, NSEG, NFIL, NBLOB, END_FORCE_MAGNITUDE, SEG_SEP, DL);
    cudaDeviceSynchronize();
#endif
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 2) usage();
    const std::string mode = argv[1];
    std::string out_name;
#if WRITE_GENERALISED_FORCES
    if (mode != "wgf" || argc != 5) usage();
    set_globals(std::atoi(argv[2]), 1, 1, 1, std::atof(argv[3]), 0, STEPS_PER_PERIOD, "none");
    out_name = argv[4];
#else
    if (mode != "run" || (argc != 11 && argc != 12)) usage();
    const bool write_files = argc == 12 && std::string(argv[11]) == "write";
    set_globals(std::atoi(argv[2]), std::atoi(argv[3]), std::atof(argv[4]), std::atof(argv[5]), std::atof(argv[6]),
                std::atof(argv[7]), std::atoi(argv[8]), argv[9]);
    out_name = argv[10];
#endif

    harness_mobility_solver mobility;
    mobility.initialise();

    std::vector<swimmer> swimmers(NSWIM);
    for (int n = 0; n < NSWIM; n++)
        swimmers[n].initial_setup(n, nullptr, &mobility.x_segs_host[3 * n * NFIL * NSEG],
                                  &mobility.f_segs_host[6 * n * NFIL * NSEG], &mobility.f_blobs_host[3 * n * NBLOB]);

#if WRITE_GENERALISED_FORCES
    // The reference's pre-run writes the two force tables and the s-value table (cilia_sim_main.cu:322-336).
    std::ofstream phase_file(reference_phase_generalised_force_file_name());
    phase_file << TOTAL_TIME_STEPS << " " << std::scientific << std::setprecision(15);
    std::ofstream angle_file(reference_angle_generalised_force_file_name());
    angle_file << TOTAL_TIME_STEPS << " " << std::scientific << std::setprecision(15);
    {
        std::ofstream s_file(reference_s_values_file_name());
        s_file << TOTAL_TIME_STEPS << " " << NSEG_PER_CILIA << " " << std::scientific << std::setprecision(15);
    }
#else
    // The s-value table of the pre-run (cilia_sim_main.cu:340-375).
    std::ifstream s_file(reference_s_values_file_name());
    if (!s_file.good()) {
        std::fprintf(stderr, "missing s-value table %s\n", reference_s_values_file_name().c_str());
        return 3;
    }
    int ref_steps = 0, ref_segs = 0;
    s_file >> ref_steps >> ref_segs;
    matrix s_values_ref(ref_steps, ref_segs);
    for (int i = 0; i < ref_steps; i++)
        for (int j = 0; j < ref_segs; j++) s_file >> s_values_ref(i, j);
    for (int i = 0; i < NSWIM; i++)
        for (int j = 0; j < NFIL; j++) swimmers[i].filaments[j].s_to_use_ref_ptr = &s_values_ref;
#endif

    std::FILE *out = std::fopen(out_name.c_str(), "wb");
    if (!out) {
        std::fprintf(stderr, "cannot open %s\n", out_name.c_str());
        return 3;
    }
    const int F = NFIL;
#if INFINITE_PLANE_WALL
    std::vector<double> rec(2 + 7 * F);
#else
    std::vector<double> rec(2 + 7 * F + 13);  // + body position, orientation, velocity and angular velocity
#endif
    for (int nt = 0; nt < TOTAL_TIME_STEPS; nt++) {
        const auto t0 = std::chrono::steady_clock::now();
        for (int i = 0; i < NSWIM; i++) {
            swimmers[i].initial_guess(nt);
            swimmers[i].forces_and_torques(nt, i);
        }
        int iters = 0;
        mobility.compute_velocities(swimmers, iters, nt);
#if WRITE_GENERALISED_FORCES
        Real qp = 0, qa = 0;  // cilia_sim_main.cu:420-440
        for (int n = 0; n < NSEG; n++)
            for (int c = 0; c < 3; c++) {
                qp += swimmers[0].filaments[0].vel_dir_phase[3 * n + c] * mobility.f_segs_host[6 * n + c];
                qa += swimmers[0].filaments[0].vel_dir_angle[3 * n + c] * mobility.f_segs_host[6 * n + c];
            }
        phase_file << qp << " ";
        angle_file << qa << " ";
#endif
        // The state of this step, before end_of_step (filament.cpp:1665) and the next initial_guess move it on.
        rec[0] = iters;
        for (int m = 0; m < F; m++) {
            const filament &fil = swimmers[0].filaments[m];
            rec[2 + m] = fil.phase;
            rec[2 + F + m] = fil.shape_rotation_angle;
            rec[2 + 2 * F + m] = fil.phase_dot;
            rec[2 + 3 * F + m] = fil.shape_rotation_angle_dot;
            for (int c = 0; c < 3; c++)
                rec[2 + 4 * F + 3 * m + c] = mobility.x_segs_host[3 * (m * NSEG + NSEG - 1) + c];
        }
#if !WRITE_GENERALISED_FORCES
        if (write_files && nt % PLOT_FREQUENCY_IN_STEPS == 0) {
            // The reference's writers in its main loop's order (cilia_sim_main.cu:628-700); prescribed
            // cilia save the step index itself (explicit description).
            std::ofstream seg_state_file(SIMULATION_SEG_STATE_NAME, std::ios::app);
            seg_state_file << nt << " " << std::scientific << std::setprecision(OUTPUT_DIGIT);
            std::ofstream body_state_file(SIMULATION_BODY_STATE_NAME, std::ios::app);
            body_state_file << nt << " " << std::scientific << std::setprecision(OUTPUT_DIGIT);
            for (int n = 0; n < NSWIM; n++) swimmers[n].write_data(seg_state_file, body_state_file);
            seg_state_file << std::endl;
            body_state_file << std::endl;
            mobility.write_data(nt, swimmers);
            std::ofstream true_states_file(SIMULATION_TRUESTATE_NAME, std::ios::app);
            true_states_file << std::scientific << std::setprecision(OUTPUT_DIGIT) << nt << " " << PERIOD << " ";
            for (int n = 0; n < NSWIM; n++)
                for (int m = 0; m < NFIL; m++) true_states_file << swimmers[n].filaments[m].phase << " ";
            for (int n = 0; n < NSWIM; n++)
                for (int m = 0; m < NFIL; m++) true_states_file << swimmers[n].filaments[m].shape_rotation_angle << " ";
            true_states_file << std::endl;
        }
#endif
#if !INFINITE_PLANE_WALL
        for (int c = 0; c < 3; c++) rec[2 + 7 * F + c] = swimmers[0].body.x[c];
        rec[2 + 7 * F + 3] = swimmers[0].body.q.scalar_part;
        for (int c = 0; c < 3; c++) rec[2 + 7 * F + 4 + c] = swimmers[0].body.q.vector_part[c];
        for (int c = 0; c < 6; c++) rec[2 + 7 * F + 7 + c] = mobility.v_bodies(c);
#endif
        for (int i = 0; i < NSWIM; i++) swimmers[i].end_of_step(nt);
#if !INFINITE_PLANE_WALL && !WRITE_GENERALISED_FORCES
        // The explicit body update of cilia_sim_main.cu:700-716 (after the step's data are written).
        for (int n = 0; n < NSWIM; n++) {
            for (int c = 0; c < 3; c++) swimmers[n].body.x[c] += DT * mobility.v_bodies(6 * n + c);
            for (int c = 0; c < 3; c++) swimmers[n].body.u[c] = DT * mobility.v_bodies(6 * n + 3 + c);
            swimmers[n].body.q = lie_exp(swimmers[n].body.u) * swimmers[n].body.qm1;
        }
#endif
        rec[1] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::fwrite(rec.data(), sizeof(double), rec.size(), out);
        std::fflush(out);
    }
    std::fclose(out);
#if WRITE_GENERALISED_FORCES
    phase_file.close();
    angle_file.close();
#endif
    mobility.finalise();
    return 0;
}

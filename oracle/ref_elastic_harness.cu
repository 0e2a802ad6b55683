// ref_elastic_harness.cu -- TEST INFRASTRUCTURE ONLY: runs the reference's own
// host step code for instability-driven elastic cilia on a wall (CILIA_TYPE 0,
// INFINITE_PLANE_WALL) on the CPU, as the oracle of the engine's elastic step.
//
// Built by oracle/ref_build.py against the reference's unmodified sources
// (mobility_solver.cpp, filament.cpp, swimmer.cpp, segment.cpp, rigid_body.cpp,
// broyden_solver.cpp, matrix.cpp, quaternion.cpp, seeding.cu, util.cu,
// globals.cu) with a generated config (CILIA_TYPE 0, CILIA_IC_TYPE 0,
// FIL_USE_DOUBLE_PRECISION true).  The mobility back-end below is the only part
// written here: the 6x6 wall RPY product of Mss_mult (cuda_functions.cu:362-474)
// by the FP64 oracle sum, and the barrier forces of barrier_forces
// (cuda_functions.cu:1825-1919, wall and segment-segment terms) added to a copy
// of the segment forces, as the reference adds them to its device copy only.
// The time loop follows cilia_sim_main.cu:405-560 (Broyden's method around the
// mobility evaluation, compute_errors and end_of_iter).
//
//   ref_elastic run <nseg> <nfil> <fil_x_dim> <spacing> <seg_sep> <period> <steps> <out.bin>
//       out.bin: per step, doubles [broyden_iterations, seconds, x_segs[3 N]] with
//       N = nfil * nseg, the positions after the step's last Broyden update.
//   ref_elastic jac <nseg> <seg_sep> <period> <out.bin>
//       one filament: the approximate Jacobian inverse of step 0 (after the first
//       error evaluation), [6 nseg * 6 nseg] row-major, then the error vector [6 nseg].
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "swimmer.hpp"
#include "mobility_solver.hpp"
#include "broyden_solver.hpp"
#include "util.hpp"

extern "C" void oracle_rpy_apply_f64(int wall, int vdof, int fdof, int self_by_index, int64_t nt, const double *xt,
                                     double at, const int64_t *t_ids, int64_t t_off, int64_t ns, const double *xs,
                                     const double *fs, double as, int64_t s_off, double mu, double *vt, int nthreads);

class host_elastic_solver : public mobility_solver {
  public:
    std::vector<double> xs, fs, vs;

    void allocate_host_memory() override {
        const int ns = NSWIM * NFIL * NSEG;
        v_segs_host = new Real[6 * ns];
        x_segs_host = new Real[3 * ns];
        f_segs_host = new Real[6 * ns];
        v_blobs_host = new Real[1];
        x_blobs_host = new Real[1];
        f_blobs_host = new Real[1];
        f_blobs_repulsion_host = new Real[1];
        std::memset(f_segs_host, 0, 6 * ns * sizeof(Real));
        xs.resize(3 * ns);
        fs.resize(6 * ns);
        vs.resize(6 * ns);
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
    // The "device" copies: positions and forces as the mobility product reads them.
    void copy_segment_positions_to_device() override {
        const int ns = NSWIM * NFIL * NSEG;
        for (int i = 0; i < 3 * ns; ++i) xs[i] = x_segs_host[i];
    }
    void copy_segment_forces_to_device() override {
        const int ns = NSWIM * NFIL * NSEG;
        for (int i = 0; i < 6 * ns; ++i) fs[i] = f_segs_host[i];
    }
    void copy_blob_positions_to_device() override {}
    void copy_blob_forces_to_device() override {}
    void copy_interparticle_blob_forces_to_host() override {}
    void copy_blob_velocities_to_host() override {}
    void copy_segment_velocities_to_host() override {
        const int ns = NSWIM * NFIL * NSEG;
        for (int i = 0; i < 6 * ns; ++i) v_segs_host[i] = static_cast<Real>(vs[i]);
    }
    void wait_for_device() override {}
    // Barrier forces on the segment forces' copy (the wall term and the segment-segment term of
    // barrier_forces; no blobs on a wall).
    void apply_interparticle_forces() override {
        const int ns = NSWIM * NFIL * NSEG;
        const double fmag = REPULSIVE_FORCE_FACTOR * END_FORCE_MAGNITUDE;
        for (int i = 0; i < ns; ++i) {
            const double xi = xs[3 * i], yi = xs[3 * i + 1], zi = xs[3 * i + 2];
            double fx = 0.0, fy = 0.0, fz = 0.0;
            if (zi < BASE_HEIGHT_ABOVE_SURFACE) {
                double w = std::fmin(1.0, 1.0 - (zi - RSEG) / (0.5 * DL - RSEG));
                fz = fmag * w * w * w * w;
            }
            const int fi = i / NSEG;
            const double a_sum = 2.0 * RSEG, chi = 10.0 / a_sum;
            for (int j = 0; j < ns; ++j) {
                const double dx = xi - xs[3 * j], dy = yi - xs[3 * j + 1], dz = zi - xs[3 * j + 2];
                const double dist = std::sqrt(dx * dx + dy * dy + dz * dz);
                if (!(fi == j / NSEG && std::abs(i - j) <= 1) && dist < 1.1 * a_sum) {
                    double w = std::fmin(1.0, 1.0 - chi * (dist - a_sum));
                    w = fmag * w * w * w * w;
                    fx += w * dx / dist;
                    fy += w * dy / dist;
                    fz += w * dz / dist;
                }
            }
            fs[6 * i] += fx;
            fs[6 * i + 1] += fy;
            fs[6 * i + 2] += fz;
        }
    }
    void evaluate_segment_segment_mobility() override {
        const int ns = NSWIM * NFIL * NSEG;
        std::fill(vs.begin(), vs.end(), 0.0);
        oracle_rpy_apply_f64(1, 6, 6, 1, ns, xs.data(), 1.0, nullptr, 0, ns, xs.data(), fs.data(), 1.0, 0, 1.0,
                             vs.data(), 0);
    }
    void evaluate_segment_blob_mobility() override {}
    void evaluate_blob_blob_mobility() override {}
    void evaluate_blob_segment_mobility() override {}
    void evaluate_full_mobility() override { evaluate_segment_segment_mobility(); }
};

namespace {

void usage() {
    std::fprintf(stderr,
                 "usage: ref_elastic run <nseg> <nfil> <fil_x_dim> <spacing> <seg_sep> <period> <steps> <out.bin>\n"
                 "       ref_elastic jac <nseg> <seg_sep> <period> <out.bin>\n");
    std::exit(2);
}

// The globals cilia_sim_main.cu reads from globals.ini (:59-91) and derives (:93-146).
void set_globals(int nseg, int nfil, double fil_x_dim, double spacing, double seg_sep, double period, int steps) {
    NSWIM = 1;
    NSEG = nseg;
    NFIL = nfil;
    NBLOB = 0;
    AR = 1;
    SEG_SEP = static_cast<Real>(seg_sep);
    PERIOD = static_cast<Real>(period);
    SIM_LENGTH = 1;
    TORSIONAL_SPRING_MAGNITUDE_FACTOR = 0;
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
    SIMULATION_FILE = "ref_elastic";
    SIMULATION_ICSTATE_NAME = "none";
    SIMULATION_NAME = SIMULATION_DIR + SIMULATION_FILE;
    SIMULATION_SEG_STATE_NAME = SIMULATION_NAME + "_seg_states.dat";
    SIMULATION_BODY_STATE_NAME = SIMULATION_NAME + "_body_states.dat";
    NSEG_PER_CILIA = NSEG;
    NPAIR = NFIL;
    NTOTAL = NSWIM * (NFIL * NSEG + NBLOB);
    DL = SEG_SEP * RSEG;
    AXIS_DIR_BODY_LENGTH = AR * FIL_LENGTH;
    END_FORCE_MAGNITUDE = DIMENSIONLESS_FORCE * KB / (DL * DL * NSEG_PER_CILIA * NSEG_PER_CILIA);
    DT = PERIOD / STEPS_PER_PERIOD;
    TOTAL_TIME_STEPS = steps;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 2) usage();
    const std::string mode = argv[1];
    const bool jac = mode == "jac";
    if (jac ? argc != 6 : (mode != "run" || argc != 10)) usage();
    if (jac)
        set_globals(std::atoi(argv[2]), 1, 1, 1.0, std::atof(argv[3]), std::atof(argv[4]), 1);
    else
        set_globals(std::atoi(argv[2]), std::atoi(argv[3]), std::atof(argv[4]), std::atof(argv[5]), std::atof(argv[6]),
                    std::atof(argv[7]), std::atoi(argv[8]));
    const std::string out_name = jac ? argv[5] : argv[9];

    host_elastic_solver mobility;
    mobility.initialise();
    std::vector<swimmer> swimmers(NSWIM);
    for (int n = 0; n < NSWIM; n++)
        swimmers[n].initial_setup(n, nullptr, &mobility.x_segs_host[3 * n * NFIL * NSEG],
                                  &mobility.f_segs_host[6 * n * NFIL * NSEG], &mobility.f_blobs_host[3 * n * NBLOB]);
    broyden_solver broyden;

    std::FILE *out = std::fopen(out_name.c_str(), "wb");
    if (!out) {
        std::fprintf(stderr, "cannot open %s\n", out_name.c_str());
        return 3;
    }
    const int N = NSWIM * NFIL * NSEG;
    std::vector<double> rec(2 + 3 * N);
    int rc = 0;
    for (int nt = 0; nt < TOTAL_TIME_STEPS; nt++) {
        const auto t0 = std::chrono::steady_clock::now();
        for (int i = 0; i < NSWIM; i++) {
            swimmers[i].initial_guess(nt);
            swimmers[i].forces_and_torques(nt, i);
        }
        int gmres_iters = 0;
        mobility.compute_velocities(swimmers, gmres_iters, nt);
        bool error_is_too_large = mobility.compute_errors(broyden.error, swimmers, nt);
        if (error_is_too_large)
            for (int i = 0; i < NSWIM; i++) swimmers[i].prepare_jacobian_inv(nt);
        if (jac) {
            const filament &fil = swimmers[0].filaments[0];
            const int n6 = 6 * NSEG;
            std::vector<double> buf(n6 * n6 + n6);
            for (int r = 0; r < n6; r++)
                for (int c = 0; c < n6; c++) buf[r * n6 + c] = fil.inverse_jacobian(r, c);
            for (int r = 0; r < n6; r++) buf[n6 * n6 + r] = broyden.error(r);
            std::fwrite(buf.data(), sizeof(double), buf.size(), out);
            break;
        }
        broyden.iter = 0;
        while (error_is_too_large && (broyden.iter < MAX_BROYDEN_ITER)) {
            broyden.find_update(swimmers, nt);
            for (int i = 0; i < NSWIM; i++) {
                swimmers[i].update(&broyden.update.data[i * 6 * NFIL * NSEG]);
                swimmers[i].forces_and_torques(nt, i);
            }
            mobility.compute_velocities(swimmers, gmres_iters, nt);
            error_is_too_large = mobility.compute_errors(broyden.new_error, swimmers, nt);
            if (!broyden.new_error.is_finite()) {
                std::fprintf(stderr, "Broyden's method diverged at step %d\n", nt);
                rc = 4;
                break;
            }
            broyden.end_of_iter(swimmers, nt, 0, error_is_too_large);
        }
        if (rc) break;
        if (error_is_too_large) {
            std::fprintf(stderr, "Broyden's method did not converge within %d iterations at step %d\n",
                         MAX_BROYDEN_ITER, nt);
            rc = 5;
            break;
        }
        for (int i = 0; i < NSWIM; i++) swimmers[i].end_of_step(nt);
        rec[0] = broyden.iter;
        for (int i = 0; i < 3 * N; i++) rec[2 + i] = mobility.x_segs_host[i];
        rec[1] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::fwrite(rec.data(), sizeof(double), rec.size(), out);
        std::fflush(out);
    }
    std::fclose(out);
    mobility.finalise();
    return rc;
}

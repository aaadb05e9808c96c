// CrankNicolsonModes.hpp -- drop-in of the reference class over the B200 C ABI.
//
// Same constructor, public members, methods and output folder as the reference's
// CrankNicolsonModes (include/CrankNicolsonModes.hpp:60-455), with Eigen-free types:
// vectors are std::vector<double> / std::vector<std::complex<double>> and the sparse
// operator members (H, V, dVdt, A, B, ...) are replaced by apply(op, x), since the
// B200 path never assembles them.  The numerics run on the GPU through
// include/cnm_gpu.h; this class keeps the host side of the reference: the public
// scalar members, the Simulation_* folder, the 14 diagnostic files, snapshots,
// checkpoints and resume.  Files are written by a background thread in the order the
// synchronous code would write them (cnm_output_queue.hpp); snapshots are copied off
// the device into page-locked buffers and formatted there.
#pragma once

#include <complex>
#include <fstream>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "cnm_gpu.h"
#include "cnm_output_queue.hpp"

using dcomplex = std::complex<double>;

/// A spherical-harmonic mode (l, m) (include/Definitions.hpp:8-17).
struct mode {
    int l;
    int m;
    bool operator==(const mode &o) const { return l == o.l && m == o.m; }
};

class CrankNicolsonModes {
public:
    // The reference's constructor (include/CrankNicolsonModes.hpp:84); `precision` (CNM_FP64, the
    // default, or CNM_MIXED) selects the solver path of the device handle.
    CrankNicolsonModes(int Nx, double L, double dt, double epsilon, int l_max, double mu, double M_c, double q,
                       double a, double R, bool counter, bool absorption, int save_every, double ramp_periods,
                       double epsilon_smear, std::string config_file, int precision = CNM_FP64);
    ~CrankNicolsonModes();
    CrankNicolsonModes(const CrankNicolsonModes &) = delete;
    CrankNicolsonModes &operator=(const CrankNicolsonModes &) = delete;

    // public members of the reference (include/CrankNicolsonModes.hpp:88-110)
    int Nr, save_every, l_max, n_modes;
    double epsilon, mu, q, R, theta, phase, Omega, Omega_0, P, R1, R2, M1, M2, a, L, dr, dt;
    bool counter;
    double M_c;

    void step(int step_id);
    void run(int n_steps, double r_ex);
    void resume(const std::string &folder, int n_steps, double r_ex);

    bool evolve_orbit = true;
    bool ramp_secondary_potential = true;
    double steps_per_period = 50.0;
    void set_power_average_orbits(double n_orbits);
    bool use_block_preconditioner = true;
    double last_solver_residual = 0.0;
    int last_solver_iterations = 0;

    std::vector<double> t;
    std::vector<double> r;
    std::vector<dcomplex> psi;  ///< host mirror of the device state (see sync_every_step)
    bool mask = false;
    bool cap = false;

    void set_initial_state_full(const std::vector<dcomplex> &psi_0);
    std::vector<mode> modes;
    void initialize();
    void configure_isolated_black_hole(double x);

    /// Replacement of the operator members: y = op x (enum cnm_operator).
    std::vector<dcomplex> apply(int op, const std::vector<dcomplex> &x);
    std::vector<dcomplex> apply_sink(const std::vector<dcomplex> &state);
    std::vector<dcomplex> schrodinger_rhs(const std::vector<dcomplex> &state);
    double sink_strength(int body);
    bool absorption_sink_active();

    void build_damping_mask(double mask_L_factor, double mask_W, int mask_n);
    void build_cap(double cap_L_factor, double cap_W, int cap_n);

    /// Refresh the host mirror psi after every step (the reference's tests read psi
    /// between steps); off, it is refreshed at snapshots and by sync_state().
    bool sync_every_step = true;
    void sync_state();
    /// Print the per-step progress line as the reference does.
    bool verbose = true;
    /// BiCGSTAB tolerance (the reference hard-codes 1e-10).
    double tolerance = 1e-10;
    /// Write diagnostics, snapshots and checkpoints on the background thread (the bytes
    /// are the same either way); off, they are written before step() returns.
    bool async_output = true;
    /// Wait until every file write queued so far is done.
    void wait_output();
    const std::string &output_folder() const { return output_folder_; }

private:
    cnm_handle *h_ = nullptr;
    std::string config_file_;
    std::string output_folder_;
    double t_i_ = 0.0, p_bin_ = 0.0, r_ex_ = 0.0;
    int idx_ex_ = 0;
    bool isolated_ = false;
    double orbits_average_ = 2.0;
    double ramp_periods_;
    double initial_period_;

    OutputQueue out_;
    std::mutex pool_m_;
    std::vector<void *> pool_free_;                  // snapshot buffers of Nr * n_modes values
    std::vector<std::pair<void *, bool>> pool_all_;  // (buffer, page-locked)

    // A snapshot buffer filled with the device state (the public mirror psi is refreshed
    // from it); it returns to the pool when the last holder drops it.
    std::shared_ptr<dcomplex> state_to_buffer();
    void post_snapshot(int step_id, std::shared_ptr<const dcomplex> data, const std::string &name);
    OutputQueue &output();

    void check(int rc) const;
    void push();  // public scalars -> device solver
    void pull();  // device solver -> public scalars
    double ramp_end_time() const { return ramp_periods_ * initial_period_; }

    void evolve(int first_step, int n_steps);
    void set_extraction_radius(double r_ex, int n_steps);
    void save_snapshot(int step_id, const std::vector<dcomplex> &state, const std::string &name);
    void save_run_info();
    void flush_diagnostics();
    void open_diagnostics(std::ios::openmode mode);
    std::vector<std::pair<std::ofstream *, std::string>> diagnostic_files();
    void save_checkpoint(int step_id);
    bool load_checkpoint(int step_id);
    void reconstruct_state_from_diagnostics(int step_id);

    std::ofstream flux_file, energy_flux_file, energy_file, norms_file, time_file, energy_modes_file, R_file,
        theta_file, Omega_file, p_bin_file, p_bin_inst_file, d_V_bin_dt_file, M_1_file, q_file;
    void write_quantity_line(double quantity, std::ofstream &file);
    void write_quantity_line_modes(const std::vector<double> &quantity, std::ofstream &file);
};

/// create_output_folder (src/Utils.cpp:11-27): Simulation_YYYY_MM_DD_HH_MM_SS with psi/ and psi_dt/.
std::string create_output_folder();

/// load_initial_modes_binary (src/InitialData.cpp:7-79): MODESBIN reader; stored modes
/// not in `modes` are ignored, missing ones are zero.
std::vector<dcomplex> load_initial_modes_binary(const std::string &filename, const std::vector<mode> &modes);

/// displaced_100_state (src/DisplacedAtom.cpp:12-76), computed on the device: the mode
/// projection of a hydrogenic 1s state centred at x_bh on the x axis.
std::vector<dcomplex> displaced_100_state(const std::vector<double> &r, const std::vector<mode> &modes, double mu,
                                          double x_bh);

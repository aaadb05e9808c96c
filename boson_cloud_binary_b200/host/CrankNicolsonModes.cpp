// CrankNicolsonModes.cpp -- host side of the drop-in class: scalars, writers, run,
// checkpoints and resume, over the C ABI of include/cnm_gpu.h.
#include "CrankNicolsonModes.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <filesystem>
#include <iomanip>
#include <iostream>
#include <limits>
#include <map>
#include <regex>
#include <sstream>
#include <stdexcept>

namespace fs = std::filesystem;

namespace {

[[noreturn]] void raise(int rc, const std::string &msg)
{
    if (rc == CNM_EINVAL) throw std::invalid_argument(msg);
    if (rc == CNM_ELOGIC) throw std::logic_error(msg);
    throw std::runtime_error(msg);
}

// Byte offsets just past each '\n' of a file; a trailing partial line is not counted
// (src/CrankNicolsonModes_restart.cpp:39-58).
std::vector<std::uintmax_t> line_ends(const std::string &path)
{
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("Cannot open " + path);
    std::vector<std::uintmax_t> ends;
    std::vector<char> buf(1 << 20);
    std::uintmax_t off = 0;
    while (in) {
        in.read(buf.data(), (std::streamsize)buf.size());
        const std::streamsize got = in.gcount();
        for (std::streamsize i = 0; i < got; ++i)
            if (buf[(size_t)i] == '\n') ends.push_back(off + (std::uintmax_t)i + 1);
        off += (std::uintmax_t)got;
    }
    return ends;
}

// First n_rows values of a one-column diagnostic file (_restart.cpp:61-76).
std::vector<double> read_column(const std::string &path, int n_rows)
{
    std::ifstream in(path);
    if (!in) throw std::runtime_error("Cannot open " + path);
    std::vector<double> v;
    v.reserve((size_t)std::max(n_rows, 0));
    std::string line;
    while ((int)v.size() < n_rows && std::getline(in, line)) v.push_back(std::strtod(line.c_str(), nullptr));
    if ((int)v.size() != n_rows) throw std::runtime_error("Too few rows in " + path);
    return v;
}

// A text snapshot "re im" per line, exactly `size` rows (_restart.cpp:78-104).
bool load_snapshot(const std::string &path, std::vector<dcomplex> &state, size_t size)
{
    std::ifstream in(path);
    if (!in) return false;
    std::vector<dcomplex> values(size);
    std::string line;
    size_t k = 0;
    while (std::getline(in, line)) {
        if (line.empty()) continue;
        if (k == size) return false;
        char *end = nullptr, *end_im = nullptr;
        const double re = std::strtod(line.c_str(), &end);
        const double im = std::strtod(end, &end_im);
        if (end == line.c_str() || end_im == end) return false;
        values[k++] = dcomplex(re, im);
    }
    if (k != size) return false;
    state.swap(values);
    return true;
}

}  // namespace

// ------------------------------------------------------------------ construction

CrankNicolsonModes::CrankNicolsonModes(int Nx, double L_, double dt_i, double epsilon_, int l_max_, double mu_,
                                       double M_c_, double q_, double a_, double R_, bool counter_, bool absorption,
                                       int save_every_, double ramp_periods, double epsilon_smear,
                                       std::string config_file)
    : Nr(Nx), save_every(save_every_), l_max(l_max_), n_modes(0), epsilon(epsilon_), mu(mu_), q(q_), R(R_),
      theta(0), phase(0), Omega(0), Omega_0(0), P(0), R1(0), R2(0), M1(1), M2(q_), a(a_), L(L_), dr(0), dt(dt_i),
      counter(counter_), M_c(M_c_), config_file_(std::move(config_file)), ramp_periods_(ramp_periods),
      initial_period_(2.0 * M_PI / std::sqrt((1 + q_) / std::pow(R_, 3)))
{
    cnm_params p{Nx, L_, dt_i, epsilon_, l_max_, mu_, M_c_, q_, a_, R_, counter_ ? 1 : 0, absorption ? 1 : 0,
                 save_every_, ramp_periods, epsilon_smear, CNM_FP64};
    const int rc = cnm_create(&p, &h_);
    if (rc != CNM_OK) raise(rc, cnm_create_error());
    int32_t n = 0;
    check(cnm_n_modes(h_, &n));
    n_modes = n;
    std::vector<int32_t> ls(n), ms(n);
    check(cnm_modes(h_, ls.data(), ms.data()));
    for (int j = 0; j < n; ++j) modes.push_back({ls[j], ms[j]});
    r.resize(Nr);
    check(cnm_grid(h_, r.data()));
    dr = L / (Nr - 1);
    pull();
    if (verbose && q > 0.0) std::cout << "Orbital period = " << P << std::endl;
}

CrankNicolsonModes::~CrankNicolsonModes()
{
    flush_diagnostics();
    if (h_) cnm_destroy(h_);
}

void CrankNicolsonModes::check(int rc) const
{
    if (rc != CNM_OK) raise(rc, h_ ? cnm_last_error(h_) : "invalid handle");
}

void CrankNicolsonModes::pull()
{
    cnm_scalars s;
    check(cnm_get_scalars(h_, &s));
    t_i_ = s.t;
    theta = s.theta;
    phase = s.phase;
    Omega = s.Omega;
    Omega_0 = s.Omega_0;
    P = s.P;
    R = s.R;
    R1 = s.R1;
    R2 = s.R2;
    M1 = s.M1;
    M2 = s.M2;
    q = s.q;
    dt = s.dt;
    p_bin_ = s.p_bin;
    steps_per_period = s.steps_per_period;
    evolve_orbit = s.evolve_orbit != 0;
    ramp_secondary_potential = s.ramp_secondary_potential != 0;
    use_block_preconditioner = s.use_block_preconditioner != 0;
    last_solver_iterations = s.last_solver_iterations;
    last_solver_residual = s.last_solver_residual;
    tolerance = s.tolerance;
}

void CrankNicolsonModes::push()
{
    cnm_scalars s;
    check(cnm_get_scalars(h_, &s));
    s.t = t_i_;
    s.theta = theta;
    s.phase = phase;
    s.Omega = Omega;
    s.Omega_0 = Omega_0;
    s.P = P;
    s.R = R;
    s.R1 = R1;
    s.R2 = R2;
    s.M1 = M1;
    s.M2 = M2;
    s.q = q;
    s.dt = dt;
    s.p_bin = p_bin_;
    s.steps_per_period = steps_per_period;
    s.evolve_orbit = evolve_orbit ? 1 : 0;
    s.ramp_secondary_potential = ramp_secondary_potential ? 1 : 0;
    s.use_block_preconditioner = use_block_preconditioner ? 1 : 0;
    s.tolerance = tolerance;
    check(cnm_set_scalars(h_, &s));
}

void CrankNicolsonModes::sync_state()
{
    psi.resize((size_t)Nr * n_modes);
    check(cnm_get_state(h_, reinterpret_cast<double *>(psi.data()), (int64_t)psi.size()));
}

// ------------------------------------------------------------------ set-up

void CrankNicolsonModes::set_power_average_orbits(double n_orbits)
{
    check(cnm_set_power_average_orbits(h_, n_orbits));
    orbits_average_ = n_orbits;
}

void CrankNicolsonModes::configure_isolated_black_hole(double x)
{
    check(cnm_configure_isolated_black_hole(h_, x));
    isolated_ = true;
    ramp_periods_ = 0.0;
    pull();
}

void CrankNicolsonModes::set_initial_state_full(const std::vector<dcomplex> &psi_0)
{
    check(cnm_set_initial_state_full(h_, reinterpret_cast<const double *>(psi_0.data()), (int64_t)psi_0.size()));
    sync_state();
}

void CrankNicolsonModes::initialize()
{
    push();
    check(cnm_initialize(h_));
    pull();
}

void CrankNicolsonModes::build_damping_mask(double f, double W, int n)
{
    check(cnm_build_damping_mask(h_, f, W, n));
    mask = true;
}

void CrankNicolsonModes::build_cap(double f, double W, int n)
{
    check(cnm_build_cap(h_, f, W, n));
    cap = true;
}

// ------------------------------------------------------------------ operators

std::vector<dcomplex> CrankNicolsonModes::apply(int op, const std::vector<dcomplex> &x)
{
    if (x.size() != (size_t)Nr * n_modes) throw std::invalid_argument("Vector size does not match Nr * n_modes");
    push();
    std::vector<dcomplex> y(x.size());
    check(cnm_apply(h_, op, reinterpret_cast<const double *>(x.data()), reinterpret_cast<double *>(y.data())));
    return y;
}

std::vector<dcomplex> CrankNicolsonModes::apply_sink(const std::vector<dcomplex> &state)
{
    return apply(CNM_OP_SINK, state);
}

std::vector<dcomplex> CrankNicolsonModes::schrodinger_rhs(const std::vector<dcomplex> &state)
{
    return apply(CNM_OP_RHS, state);
}

double CrankNicolsonModes::sink_strength(int body)
{
    double v = 0.0;
    check(cnm_sink_strength(h_, body, &v));
    return v;
}

bool CrankNicolsonModes::absorption_sink_active()
{
    int32_t a = 0;
    check(cnm_sink_active(h_, &a));
    return a != 0;
}

// ------------------------------------------------------------------ stepping

// src/CrankNicolsonModes.cpp:145-234: the GPU runs the step; the host writes the 14
// diagnostic rows in the reference's order and the snapshot / checkpoint.
void CrankNicolsonModes::step(int step_id)
{
    push();
    cnm_diag d;
    std::vector<double> ef(n_modes), fl(n_modes), nm(n_modes), en(n_modes);
    check(cnm_step(h_, step_id, &d, ef.data(), fl.data(), nm.data(), en.data()));
    pull();
    if (step_id >= 0 && (size_t)step_id < t.size()) t[(size_t)step_id] = d.t;
    if (verbose) {
        std::cout << "\rStep: " << step_id << "/" << t.size() << " | Time " << d.t;
        if (evolve_orbit) std::cout << " | R = " << d.R;
        std::cout << std::flush;
    }
    write_quantity_line(d.R, R_file);
    write_quantity_line(d.theta, theta_file);
    write_quantity_line(d.Omega, Omega_file);
    write_quantity_line(d.M1, M_1_file);
    write_quantity_line(d.q, q_file);
    write_quantity_line(d.t, time_file);
    write_quantity_line_modes(ef, energy_flux_file);
    write_quantity_line_modes(fl, flux_file);
    write_quantity_line(d.energy, energy_file);
    write_quantity_line(d.p_bin, p_bin_file);
    write_quantity_line(d.p_bin_inst, p_bin_inst_file);
    write_quantity_line(d.dV_bin_dt, d_V_bin_dt_file);
    write_quantity_line_modes(nm, norms_file);
    write_quantity_line_modes(en, energy_modes_file);
    const bool snapshot = step_id % save_every == 0;
    if (sync_every_step || snapshot) sync_state();
    if (snapshot) {
        save_snapshot(step_id, psi, "psi");
        flush_diagnostics();
        save_checkpoint(step_id);
    }
}

void CrankNicolsonModes::set_extraction_radius(double r_ex, int n_steps)
{
    r_ex_ = r_ex;
    idx_ex_ = (int)std::floor(r_ex / dr);
    if (verbose) std::cout << "Computing fluxes at: " << r_ex << " [Index: " << idx_ex_ << "]" << std::endl;
    check(cnm_prepare_run(h_, n_steps, r_ex));  // validates like the reference
}

// src/CrankNicolsonModes.cpp:236-259.
void CrankNicolsonModes::run(int n_steps, double r_ex)
{
    if (verbose) std::cout << "Running simulation..." << std::endl;
    push();
    set_extraction_radius(r_ex, n_steps);  // t = 0 and the t = 0 operator
    pull();
    t.assign((size_t)n_steps, 0.0);
    t[0] = t_i_;
    output_folder_ = create_output_folder();
    if (verbose) std::cout << "Output folder: " << output_folder_ << std::endl;
    open_diagnostics(std::ios::out);
    save_run_info();
    sync_state();
    save_snapshot(0, psi, "psi");
    save_snapshot(0, schrodinger_rhs(psi), "psi_dt");
    save_checkpoint(0);
    evolve(1, n_steps);
}

// src/CrankNicolsonModes.cpp:272-289.
void CrankNicolsonModes::evolve(int first_step, int n_steps)
{
    for (int n = first_step; n < n_steps; ++n) {
        int32_t stop = 0;
        check(cnm_should_stop(h_, &stop));
        if (stop) break;
        step(n);
    }
    if (verbose) std::cout << std::endl;
    flush_diagnostics();
    sync_state();
    if (verbose) std::cout << "Simulation completed!" << std::endl;
}

// ------------------------------------------------------------------ output

std::string create_output_folder()
{
    const auto now = std::chrono::system_clock::now();
    const std::time_t tt = std::chrono::system_clock::to_time_t(now);
    std::stringstream ss;
    ss << std::put_time(std::localtime(&tt), "Simulation_%Y_%m_%d_%H_%M_%S");
    const std::string folder = ss.str();
    fs::create_directory(folder);
    fs::create_directory(folder + "/psi");
    fs::create_directory(folder + "/psi_dt");
    return folder;
}

// src/CrankNicolsonModes_utils.cpp:11-46.
void CrankNicolsonModes::save_run_info()
{
    if (!config_file_.empty() && fs::exists(config_file_))
        fs::copy_file(config_file_, output_folder_ + "/config.toml", fs::copy_options::overwrite_existing);
    std::ofstream out(output_folder_ + "/r.txt");
    for (int i = 0; i < Nr; ++i) out << r[i] << "\n";
    std::ofstream mo(output_folder_ + "/modes.txt");
    for (int n = 0; n < n_modes; ++n) mo << modes[n].l << "," << modes[n].m << std::endl;
}

// src/CrankNicolsonModes_utils.cpp:48-64.
void CrankNicolsonModes::save_snapshot(int step_id, const std::vector<dcomplex> &state, const std::string &name)
{
    std::stringstream fn;
    fn << output_folder_ << "/" << name << "/snapshot_" << std::setw(6) << std::setfill('0') << step_id << ".txt";
    std::ofstream out(fn.str());
    if (!out) {
        std::cerr << "Could not open file: " << fn.str() << "\n";
        return;
    }
    for (const dcomplex &v : state) out << v.real() << " " << v.imag() << "\n";
}

void CrankNicolsonModes::write_quantity_line_modes(const std::vector<double> &quantity, std::ofstream &file)
{
    for (size_t i = 0; i < quantity.size(); ++i) {
        file << std::scientific << std::setprecision(12) << quantity[i];
        if (i + 1 < quantity.size()) file << " ";
    }
    file << '\n';
}

void CrankNicolsonModes::write_quantity_line(double quantity, std::ofstream &file)
{
    file << std::scientific << std::setprecision(12) << quantity << '\n';
}

void CrankNicolsonModes::flush_diagnostics()
{
    for (auto &[stream, name] : diagnostic_files())
        if (stream->is_open()) stream->flush();
}

// src/CrankNicolsonModes_restart.cpp:107-137.
std::vector<std::pair<std::ofstream *, std::string>> CrankNicolsonModes::diagnostic_files()
{
    return {
        {&flux_file, "flux.txt"},         {&energy_flux_file, "energy_flux.txt"},
        {&energy_file, "energy.txt"},     {&energy_modes_file, "energy_modes.txt"},
        {&norms_file, "norms.txt"},       {&time_file, "t.txt"},
        {&p_bin_file, "p_bin.txt"},       {&p_bin_inst_file, "p_bin_inst.txt"},
        {&d_V_bin_dt_file, "dV_bin_dt.txt"}, {&R_file, "R_orb.txt"},
        {&Omega_file, "Omega_orb.txt"},   {&M_1_file, "M_1.txt"},
        {&q_file, "q.txt"},               {&theta_file, "theta_orb.txt"},
    };
}

void CrankNicolsonModes::open_diagnostics(std::ios::openmode mode)
{
    for (auto &[stream, name] : diagnostic_files()) {
        if (stream->is_open()) stream->close();
        stream->open(output_folder_ + "/" + name, mode);
        if (!*stream) throw std::runtime_error("Cannot open " + output_folder_ + "/" + name);
    }
}

// ------------------------------------------------------------------ checkpoints

// src/CrankNicolsonModes_restart.cpp:139-177: the bytes come from the device state
// (cnm_save_checkpoint); the file is replaced atomically through a .tmp file.
void CrankNicolsonModes::save_checkpoint(int step_id)
{
    push();
    int64_t size = 0;
    check(cnm_save_checkpoint(h_, step_id, nullptr, 0, &size));
    std::vector<char> bytes((size_t)size);
    check(cnm_save_checkpoint(h_, step_id, bytes.data(), size, &size));
    const std::string final_path = output_folder_ + "/checkpoint.bin", tmp_path = final_path + ".tmp";
    {
        std::ofstream out(tmp_path, std::ios::binary | std::ios::trunc);
        if (!out) {
            std::cerr << "Could not write checkpoint " << tmp_path << "\n";
            return;
        }
        out.write(bytes.data(), (std::streamsize)bytes.size());
        if (!out) {
            std::cerr << "Could not write checkpoint " << tmp_path << "\n";
            return;
        }
    }
    std::error_code err;
    fs::rename(tmp_path, final_path, err);
    if (err) std::cerr << "Could not replace checkpoint: " << err.message() << "\n";
}

// src/CrankNicolsonModes_restart.cpp:179-233.
bool CrankNicolsonModes::load_checkpoint(int step_id)
{
    std::ifstream in(output_folder_ + "/checkpoint.bin", std::ios::binary);
    if (!in) return false;
    std::vector<char> bytes((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    int32_t loaded = 0;
    check(cnm_load_checkpoint(h_, step_id, bytes.data(), (int64_t)bytes.size(), &loaded));
    if (!loaded) return false;
    pull();
    sync_state();
    return true;
}

// src/CrankNicolsonModes_restart.cpp:235-286: the evolving scalars from the diagnostic
// rows 0..step_id-1 (12 significant digits: accurate, not bitwise).
void CrankNicolsonModes::reconstruct_state_from_diagnostics(int step_id)
{
    const std::string f = output_folder_ + "/";
    const std::vector<double> times = read_column(f + "t.txt", step_id);
    const std::vector<double> Rs = read_column(f + "R_orb.txt", step_id);
    const std::vector<double> thetas = read_column(f + "theta_orb.txt", step_id);
    const std::vector<double> Omegas = read_column(f + "Omega_orb.txt", step_id);
    const std::vector<double> M1s = read_column(f + "M_1.txt", step_id);
    const std::vector<double> qs = read_column(f + "q.txt", step_id);
    const std::vector<double> p_bins = read_column(f + "p_bin.txt", step_id);
    const std::vector<double> p_insts = read_column(f + "p_bin_inst.txt", step_id);
    double Omega_prev = isolated_ ? 0.0 : (ramp_end_time() > 0.0 ? 0.0 : Omega_0);
    double t_prev = 0.0;
    std::vector<double> phases((size_t)step_id);
    double ph = 0.0;
    for (int k = 0; k < step_id; ++k) {
        ph += Omega_prev * (times[k] - t_prev);
        phases[(size_t)k] = ph;
        Omega_prev = Omegas[k];
        t_prev = times[k];
    }
    phase = ph;
    if (isolated_) check(cnm_replay_power_average(h_, nullptr, nullptr, nullptr, 0));
    else check(cnm_replay_power_average(h_, times.data(), phases.data(), p_insts.data(), step_id));
    if (step_id == 0) {
        push();
        return;
    }
    const int last = step_id - 1;
    t_i_ = times[last];
    R = Rs[last];
    theta = thetas[last];
    M1 = M1s[last];
    q = qs[last];
    M2 = q * M1;
    R1 = M2 / (M1 + M2) * R;
    R2 = M1 / (M1 + M2) * R;
    Omega = Omegas[last];
    p_bin_ = p_bins[last];
    if (!isolated_ && evolve_orbit && t_i_ > ramp_end_time()) {
        P = 2.0 * M_PI / Omega;
        dt = P / steps_per_period;
    }
    push();
}

// src/CrankNicolsonModes_restart.cpp:288-399.
void CrankNicolsonModes::resume(const std::string &folder, int n_steps, double r_ex)
{
    if (verbose) std::cout << "Resuming simulation in " << folder << std::endl;
    push();
    set_extraction_radius(r_ex, n_steps);
    pull();
    output_folder_ = folder;
    {
        std::ifstream modes_in(folder + "/modes.txt");
        std::string line;
        int count = 0;
        while (std::getline(modes_in, line)) {
            if (line.empty()) continue;
            int l = 0, m = 0;
            char comma = 0;
            std::istringstream row(line);
            row >> l >> comma >> m;
            if (count >= n_modes || modes[count].l != l || modes[count].m != m)
                throw std::runtime_error("modes.txt does not match the modes built from config.toml");
            ++count;
        }
        if (modes_in.is_open() && count != n_modes)
            throw std::runtime_error("modes.txt does not match the modes built from config.toml");
    }
    size_t complete_rows = std::numeric_limits<size_t>::max();
    std::vector<std::vector<std::uintmax_t>> ends;
    for (auto &[stream, name] : diagnostic_files()) {
        ends.push_back(line_ends(folder + "/" + name));
        complete_rows = std::min(complete_rows, ends.back().size());
    }
    std::vector<int> steps;
    const std::regex pattern(R"(snapshot_(\d+)\.txt)");
    for (const auto &entry : fs::directory_iterator(folder + "/psi")) {
        std::smatch m;
        const std::string name = entry.path().filename().string();
        if (std::regex_match(name, m, pattern)) steps.push_back(std::stoi(m[1].str()));
    }
    std::sort(steps.rbegin(), steps.rend());
    int start = -1;
    std::vector<dcomplex> state;
    for (const int c : steps) {
        if ((size_t)c > complete_rows) continue;
        std::ostringstream path;
        path << folder << "/psi/snapshot_" << std::setw(6) << std::setfill('0') << c << ".txt";
        if (load_snapshot(path.str(), state, (size_t)Nr * n_modes)) {
            start = c;
            break;
        }
        if (verbose) std::cout << "Skipping incomplete snapshot " << path.str() << std::endl;
    }
    if (start < 0) throw std::runtime_error("No usable snapshot found in " + folder + "/psi");
    if (verbose) std::cout << "Restarting from snapshot " << start << std::endl;
    check(cnm_set_state(h_, reinterpret_cast<const double *>(state.data()), (int64_t)state.size()));
    if (!load_checkpoint(start)) {
        if (verbose) std::cout << "No checkpoint for this snapshot: rebuilding the orbit state from the diagnostics."
                               << std::endl;
        reconstruct_state_from_diagnostics(start);
        sync_state();
    }
    int fi = 0;
    for (auto &[stream, name] : diagnostic_files()) {
        const auto &fe = ends[(size_t)fi++];
        const std::uintmax_t keep = start == 0 ? 0 : fe[(size_t)(start - 1)];
        if (stream->is_open()) stream->close();
        fs::resize_file(folder + "/" + name, keep);
    }
    open_diagnostics(std::ios::out | std::ios::app);
    t.assign((size_t)n_steps, 0.0);
    if (start < n_steps) t[(size_t)start] = t_i_;
    // H(t_n) with the restored orbit; keep the stored Omega (the refresh recomputes it)
    const double restored_Omega = Omega;
    check(cnm_refresh(h_, t_i_));
    pull();
    Omega = restored_Omega;
    push();
    if (start + 1 >= n_steps) {
        if (verbose) std::cout << "The run had already reached its last step (" << n_steps - 1 << ")." << std::endl;
        return;
    }
    evolve(start + 1, n_steps);
}

// ------------------------------------------------------------------ initial data

// src/InitialData.cpp:7-79.
std::vector<dcomplex> load_initial_modes_binary(const std::string &filename, const std::vector<mode> &modes)
{
    std::ifstream in(filename, std::ios::binary);
    if (!in) throw std::runtime_error("Cannot open initial-state file " + filename);
    char magic[8];
    in.read(magic, 8);
    if (std::string(magic, 8) != "MODESBIN") throw std::runtime_error(filename + " is not a MODESBIN file");
    int32_t version = 0;
    in.read(reinterpret_cast<char *>(&version), sizeof(version));
    if (version != 1) throw std::runtime_error("Unsupported MODESBIN version in " + filename);
    int64_t Nr = 0, Nm = 0;
    in.read(reinterpret_cast<char *>(&Nr), sizeof(Nr));
    in.read(reinterpret_cast<char *>(&Nm), sizeof(Nm));
    std::map<std::pair<int, int>, std::vector<dcomplex>> stored;
    for (int64_t k = 0; k < Nm; ++k) {
        int32_t l = 0, m = 0;
        in.read(reinterpret_cast<char *>(&l), sizeof(l));
        in.read(reinterpret_cast<char *>(&m), sizeof(m));
        std::vector<double> re((size_t)Nr), im((size_t)Nr);
        in.read(reinterpret_cast<char *>(re.data()), Nr * (int64_t)sizeof(double));
        in.read(reinterpret_cast<char *>(im.data()), Nr * (int64_t)sizeof(double));
        std::vector<dcomplex> prof((size_t)Nr);
        for (int64_t i = 0; i < Nr; ++i) prof[(size_t)i] = dcomplex(re[(size_t)i], im[(size_t)i]);
        stored[{l, m}] = std::move(prof);
    }
    if (!in) throw std::runtime_error("Truncated MODESBIN file " + filename);
    std::vector<dcomplex> psi((size_t)Nr * modes.size(), dcomplex(0.0, 0.0));
    for (size_t j = 0; j < modes.size(); ++j) {
        auto it = stored.find({modes[j].l, modes[j].m});
        if (it != stored.end()) std::copy(it->second.begin(), it->second.end(), psi.begin() + (int64_t)(j * Nr));
    }
    return psi;
}

std::vector<dcomplex> displaced_100_state(const std::vector<double> &r, const std::vector<mode> &modes, double mu,
                                          double x_bh)
{
    std::vector<int32_t> l(modes.size()), m(modes.size());
    for (size_t j = 0; j < modes.size(); ++j) {
        l[j] = modes[j].l;
        m[j] = modes[j].m;
    }
    std::vector<dcomplex> psi(r.size() * modes.size());
    const int rc = cnm_displaced_100_state(r.data(), (int32_t)r.size(), l.data(), m.data(), (int32_t)modes.size(), mu,
                                           x_bh, reinterpret_cast<double *>(psi.data()));
    if (rc != CNM_OK) raise(rc, cnm_create_error());
    return psi;
}

// CrankNicolsonModes.cpp -- host side of the drop-in class: scalars, writers, run,
// checkpoints and resume, over the C ABI of include/cnm_gpu.h.
#include "CrankNicolsonModes.hpp"
#include "cnm_snapshot_text.hpp"

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
#include <thread>

namespace fs = std::filesystem;

namespace {

[[noreturn]] void raise(int rc, const std::string &msg)
{
    if (rc == CNM_EINVAL) throw std::invalid_argument(msg);
    if (rc == CNM_ELOGIC) throw std::logic_error(msg);
    throw std::runtime_error(msg);
}

// A file's bytes, or nothing when it cannot be opened.
bool slurp(const std::string &path, std::string &out)
{
    std::ifstream in(path, std::ios::binary | std::ios::ate);
    if (!in) return false;
    const std::streamoff n = in.tellg();
    out.assign(n > 0 ? (size_t)n : 0, '\0');
    in.seekg(0);
    if (n > 0) in.read(&out[0], n);
    return (bool)in || n == 0;
}

// What a run folder holds, read in one pass per file: for every diagnostic file its text
// and the byte offset just past each complete row (a row is complete once its '\n' is
// written), and the steps of the state snapshots psi/snapshot_NNNNNN.txt, newest first.
// A resume restarts from the newest snapshot whose diagnostic rows are complete in every
// file (src/CrankNicolsonModes_restart.cpp:288-399 defines that behaviour).
struct RunIndex {
    struct File {
        std::string name, text;
        std::vector<size_t> row_end;
    };
    std::vector<File> files;
    std::vector<int> snapshots;

    size_t complete_rows() const
    {
        size_t n = std::numeric_limits<size_t>::max();
        for (const File &f : files) n = std::min(n, f.row_end.size());
        return files.empty() ? 0 : n;
    }

    const File &file(const std::string &name) const
    {
        for (const File &f : files)
            if (f.name == name) return f;
        throw std::runtime_error("Diagnostic file " + name + " is not part of the run index");
    }

    // First value of row k of a diagnostic file.
    double value(const std::string &name, size_t k) const
    {
        const File &f = file(name);
        if (k >= f.row_end.size()) throw std::runtime_error("Row " + std::to_string(k) + " missing from " + name);
        return std::strtod(f.text.c_str() + (k == 0 ? 0 : f.row_end[k - 1]), nullptr);
    }
};

RunIndex index_run(const std::string &folder, const std::vector<std::string> &names)
{
    RunIndex ix;
    for (const std::string &name : names) {
        RunIndex::File f;
        f.name = name;
        if (!slurp(folder + "/" + name, f.text)) throw std::runtime_error("Cannot read " + folder + "/" + name);
        for (size_t i = 0; i < f.text.size(); ++i)
            if (f.text[i] == '\n') f.row_end.push_back(i + 1);
        ix.files.push_back(std::move(f));
    }
    // snapshot_ + digits + .txt
    const std::string head = "snapshot_", tail = ".txt";
    for (const auto &entry : fs::directory_iterator(folder + "/psi")) {
        const std::string nm = entry.path().filename().string();
        if (nm.size() <= head.size() + tail.size() || nm.compare(0, head.size(), head) != 0 ||
            nm.compare(nm.size() - tail.size(), tail.size(), tail) != 0)
            continue;
        const std::string digits = nm.substr(head.size(), nm.size() - head.size() - tail.size());
        if (!std::all_of(digits.begin(), digits.end(), [](char ch) { return ch >= '0' && ch <= '9'; })) continue;
        ix.snapshots.push_back(std::stoi(digits));
    }
    std::sort(ix.snapshots.begin(), ix.snapshots.end(), std::greater<int>());
    return ix;
}

// A text snapshot: one "re im" pair per non-empty line, exactly `size` of them; anything
// else (a short, over-long or garbled file) is not a usable snapshot.
bool parse_snapshot(const std::string &path, size_t size, std::vector<dcomplex> &state)
{
    std::string text;
    if (!slurp(path, text)) return false;
    std::vector<dcomplex> values;
    values.reserve(size);
    size_t pos = 0;
    while (pos < text.size()) {
        size_t eol = text.find('\n', pos);
        if (eol == std::string::npos) eol = text.size();
        if (eol > pos) {
            const std::string line = text.substr(pos, eol - pos);
            const char *p0 = line.c_str();
            char *p1 = nullptr, *p2 = nullptr;
            const double re = std::strtod(p0, &p1);
            const double im = std::strtod(p1, &p2);
            if (p1 == p0 || p2 == p1 || values.size() == size) return false;
            values.emplace_back(re, im);
        }
        pos = eol + 1;
    }
    if (values.size() != size) return false;
    state.swap(values);
    return true;
}

// One state snapshot as text: "re im" per value in the default stream format (the bytes
// of src/CrankNicolsonModes_utils.cpp:48-64), formatted on up to 8 threads.
void write_snapshot_file(const std::string &path, const dcomplex *v, size_t n)
{
    std::ofstream out(path, std::ios::binary);
    if (!out) {
        std::cerr << "Could not open file: " << path << "\n";
        return;
    }
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    for (const std::string &piece : snapshot_text(v, n, std::min(8u, hw)))
        out.write(piece.data(), (std::streamsize)piece.size());
}

// The (l, m) list of a run's modes.txt ("l,m" per line); false when there is no file.
bool read_mode_list(const std::string &path, std::vector<mode> &out)
{
    std::string text;
    if (!slurp(path, text)) return false;
    std::istringstream in(text);
    std::string line;
    while (std::getline(in, line)) {
        const size_t comma = line.find(',');
        if (line.empty() || comma == std::string::npos) continue;
        out.push_back(mode{std::stoi(line.substr(0, comma)), std::stoi(line.substr(comma + 1))});
    }
    return true;
}

}  // namespace

// ------------------------------------------------------------------ construction

CrankNicolsonModes::CrankNicolsonModes(int Nx, double L_, double dt_i, double epsilon_, int l_max_, double mu_,
                                       double M_c_, double q_, double a_, double R_, bool counter_, bool absorption,
                                       int save_every_, double ramp_periods, double epsilon_smear,
                                       std::string config_file, int precision)
    : Nr(Nx), save_every(save_every_), l_max(l_max_), n_modes(0), epsilon(epsilon_), mu(mu_), q(q_), R(R_),
      theta(0), phase(0), Omega(0), Omega_0(0), P(0), R1(0), R2(0), M1(1), M2(q_), a(a_), L(L_), dr(0), dt(dt_i),
      counter(counter_), M_c(M_c_), config_file_(std::move(config_file)), ramp_periods_(ramp_periods),
      initial_period_(2.0 * M_PI / std::sqrt((1 + q_) / std::pow(R_, 3)))
{
    cnm_params p{Nx, L_, dt_i, epsilon_, l_max_, mu_, M_c_, q_, a_, R_, counter_ ? 1 : 0, absorption ? 1 : 0,
                 save_every_, ramp_periods, epsilon_smear, precision};
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
    out_.stop();  // every queued write has run
    for (auto &[stream, name] : diagnostic_files())
        if (stream->is_open()) stream->flush();
    for (auto &[ptr, pinned] : pool_all_) {
        if (pinned) cnm_host_free(ptr);
        else std::free(ptr);
    }
    if (h_) cnm_destroy(h_);
}

OutputQueue &CrankNicolsonModes::output()
{
    if (out_.inline_mode == async_output) {
        out_.drain();  // writes queued under the previous setting go first
        out_.inline_mode = !async_output;
    }
    return out_;
}

void CrankNicolsonModes::wait_output() { out_.drain(); }

std::shared_ptr<dcomplex> CrankNicolsonModes::state_to_buffer()
{
    const size_t n = (size_t)Nr * n_modes;
    void *p = nullptr;
    {
        std::lock_guard<std::mutex> lk(pool_m_);
        if (!pool_free_.empty()) {
            p = pool_free_.back();
            pool_free_.pop_back();
        }
    }
    if (!p) {
        const bool pinned = cnm_host_alloc((int64_t)(n * sizeof(dcomplex)), &p) == CNM_OK;
        if (!pinned && !(p = std::malloc(n * sizeof(dcomplex)))) throw std::bad_alloc();
        std::lock_guard<std::mutex> lk(pool_m_);
        pool_all_.emplace_back(p, pinned);
    }
    std::shared_ptr<dcomplex> buf(static_cast<dcomplex *>(p), [this](dcomplex *q) {
        std::lock_guard<std::mutex> lk(pool_m_);
        pool_free_.push_back(q);
    });
    check(cnm_get_state(h_, reinterpret_cast<double *>(buf.get()), (int64_t)n));
    psi.assign(buf.get(), buf.get() + n);
    return buf;
}

void CrankNicolsonModes::post_snapshot(int step_id, std::shared_ptr<const dcomplex> data, const std::string &name)
{
    std::stringstream fn;
    fn << output_folder_ << "/" << name << "/snapshot_" << std::setw(6) << std::setfill('0') << step_id << ".txt";
    const size_t n = (size_t)Nr * n_modes;
    output().post([path = fn.str(), data = std::move(data), n]() { write_snapshot_file(path, data.get(), n); }, true);
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
    output().post([this, d, ef = std::move(ef), fl = std::move(fl), nm = std::move(nm), en = std::move(en)]() {
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
    });
    if (step_id % save_every == 0) {
        post_snapshot(step_id, state_to_buffer(), "psi");
        flush_diagnostics();
        save_checkpoint(step_id);
    } else if (sync_every_step) {
        sync_state();
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
    post_snapshot(0, state_to_buffer(), "psi");
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
    wait_output();  // the run's files are complete when it returns
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
    auto keep = std::make_shared<std::vector<dcomplex>>(state);
    post_snapshot(step_id, std::shared_ptr<const dcomplex>(keep, keep->data()), name);
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
    output().post([this] {
        for (auto &[stream, name] : diagnostic_files())
            if (stream->is_open()) stream->flush();
    });
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
    wait_output();
    for (auto &[stream, name] : diagnostic_files()) {
        if (stream->is_open()) stream->close();
        stream->open(output_folder_ + "/" + name, mode);
        if (!*stream) throw std::runtime_error("Cannot open " + output_folder_ + "/" + name);
    }
}

// ------------------------------------------------------------------ checkpoints

// src/CrankNicolsonModes_restart.cpp:139-177: the bytes come from the device state
// (cnm_save_checkpoint) now; the file, replaced atomically through a .tmp file, is written
// after the snapshot and the diagnostic rows queued before it.
void CrankNicolsonModes::save_checkpoint(int step_id)
{
    push();
    int64_t size = 0;
    check(cnm_save_checkpoint(h_, step_id, nullptr, 0, &size));
    auto bytes = std::make_shared<std::vector<char>>((size_t)size);
    check(cnm_save_checkpoint(h_, step_id, bytes->data(), size, &size));
    const std::string final_path = output_folder_ + "/checkpoint.bin";
    output().post([final_path, bytes]() {
        const std::string tmp_path = final_path + ".tmp";
        {
            std::ofstream out(tmp_path, std::ios::binary | std::ios::trunc);
            if (!out) {
                std::cerr << "Could not write checkpoint " << tmp_path << "\n";
                return;
            }
            out.write(bytes->data(), (std::streamsize)bytes->size());
            if (!out) {
                std::cerr << "Could not write checkpoint " << tmp_path << "\n";
                return;
            }
        }
        std::error_code err;
        fs::rename(tmp_path, final_path, err);
        if (err) std::cerr << "Could not replace checkpoint: " << err.message() << "\n";
    });
}

// src/CrankNicolsonModes_restart.cpp:179-233.
bool CrankNicolsonModes::load_checkpoint(int step_id)
{
    wait_output();
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

std::vector<std::string> CrankNicolsonModes_diagnostic_names(
    const std::vector<std::pair<std::ofstream *, std::string>> &files)
{
    std::vector<std::string> names;
    for (const auto &f : files) names.push_back(f.second);
    return names;
}

// Without a checkpoint for the restart step, the evolving scalars come from the
// diagnostic rows 0 .. step_id-1 (row k is written by step k+1; 12 significant digits, so
// the restart is close, not bitwise): the orbit of the last row, and the rolling average of
// p_bin replayed over the phases the rows imply.  The rules -- phase advancing with the
// previous row's Omega from t = 0 (Omega = 0 during a start-up ramp, Omega_0 otherwise),
// P and dt following Omega once an evolving orbit is past its ramp -- are those of
// src/CrankNicolsonModes_restart.cpp:236-286.
void CrankNicolsonModes::reconstruct_state_from_diagnostics(int step_id)
{
    const RunIndex ix = index_run(output_folder_, CrankNicolsonModes_diagnostic_names(diagnostic_files()));
    const size_t n = (size_t)step_id;
    if (ix.complete_rows() < n) throw std::runtime_error("The diagnostics end before step " + std::to_string(step_id));
    std::vector<double> times(n), phases(n), p_inst(n);
    double omega_before = isolated_ || ramp_end_time() > 0.0 ? 0.0 : Omega_0;
    double t_before = 0.0, ph = 0.0;
    for (size_t k = 0; k < n; ++k) {
        times[k] = ix.value("t.txt", k);
        p_inst[k] = ix.value("p_bin_inst.txt", k);
        ph += omega_before * (times[k] - t_before);
        phases[k] = ph;
        omega_before = ix.value("Omega_orb.txt", k);
        t_before = times[k];
    }
    phase = ph;
    check(cnm_replay_power_average(h_, isolated_ ? nullptr : times.data(), isolated_ ? nullptr : phases.data(),
                                   isolated_ ? nullptr : p_inst.data(), isolated_ ? 0 : step_id));
    if (n > 0) {
        const size_t last = n - 1;
        t_i_ = times[last];
        R = ix.value("R_orb.txt", last);
        theta = ix.value("theta_orb.txt", last);
        M1 = ix.value("M_1.txt", last);
        q = ix.value("q.txt", last);
        Omega = ix.value("Omega_orb.txt", last);
        p_bin_ = ix.value("p_bin.txt", last);
        M2 = q * M1;
        R1 = M2 / (M1 + M2) * R;
        R2 = M1 / (M1 + M2) * R;
        if (!isolated_ && evolve_orbit && t_i_ > ramp_end_time()) {
            P = 2.0 * M_PI / Omega;
            dt = P / steps_per_period;
        }
    }
    push();
}

// resume (behaviour of src/CrankNicolsonModes_restart.cpp:288-399): the run folder is
// indexed once; the restart step is the newest snapshot that parses completely and whose
// diagnostic rows are complete in every file; the state comes from that snapshot, the
// scalars from checkpoint.bin when it holds that step (bitwise) or else from the
// diagnostics; every diagnostic file is cut back to the restart step's rows and the run
// continues by appending.
void CrankNicolsonModes::resume(const std::string &folder, int n_steps, double r_ex)
{
    if (verbose) std::cout << "Resuming the run in " << folder << std::endl;
    wait_output();
    push();
    set_extraction_radius(r_ex, n_steps);
    pull();
    output_folder_ = folder;
    std::vector<mode> stored;
    if (read_mode_list(folder + "/modes.txt", stored) && stored != modes)
        throw std::runtime_error("The mode list of " + folder + "/modes.txt differs from this configuration's");
    const RunIndex ix = index_run(folder, CrankNicolsonModes_diagnostic_names(diagnostic_files()));
    const size_t rows = ix.complete_rows();
    int start = -1;
    std::vector<dcomplex> state;
    for (const int s : ix.snapshots) {
        if ((size_t)s > rows) continue;  // its diagnostic rows were not all written
        std::ostringstream path;
        path << folder << "/psi/snapshot_" << std::setw(6) << std::setfill('0') << s << ".txt";
        if (parse_snapshot(path.str(), (size_t)Nr * n_modes, state)) {
            start = s;
            break;
        }
        if (verbose) std::cout << "Snapshot " << path.str() << " is incomplete; trying an earlier one" << std::endl;
    }
    if (start < 0) throw std::runtime_error("No complete snapshot to resume from in " + folder + "/psi");
    if (verbose) std::cout << "Restart step: " << start << std::endl;
    check(cnm_set_state(h_, reinterpret_cast<const double *>(state.data()), (int64_t)state.size()));
    if (!load_checkpoint(start)) {
        if (verbose) std::cout << "checkpoint.bin does not hold this step: orbit state from the diagnostics" << std::endl;
        reconstruct_state_from_diagnostics(start);
        sync_state();
    }
    for (auto &[stream, name] : diagnostic_files()) {
        if (stream->is_open()) stream->close();
        const RunIndex::File &f = ix.file(name);
        fs::resize_file(folder + "/" + name, start == 0 ? 0 : f.row_end[(size_t)start - 1]);
    }
    open_diagnostics(std::ios::out | std::ios::app);
    t.assign((size_t)n_steps, 0.0);
    if (start < n_steps) t[(size_t)start] = t_i_;
    // rebuild H(t_start) from the restored orbit; the refresh derives Omega from R and the
    // masses, while the next step must start from the stored Omega
    const double stored_Omega = Omega;
    check(cnm_refresh(h_, t_i_));
    pull();
    Omega = stored_Omega;
    push();
    if (start + 1 >= n_steps) {
        if (verbose) std::cout << "Nothing to do: the run already reached step " << n_steps - 1 << std::endl;
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

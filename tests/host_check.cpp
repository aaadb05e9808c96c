// host_check.cpp -- exercises the C++ drop-in class (boson_cloud_binary_b200/host) on
// the scenarios of the reference's tests/restart.cpp:
//   * a run stopped early and resumed from its checkpoint reproduces the uninterrupted
//     run's folder byte for byte (state snapshots, 14 diagnostic files, checkpoint);
//   * the same after a crash mid-write (a partial diagnostic row and a snapshot written
//     ahead of its rows);
//   * resuming without checkpoint.bin rebuilds the orbit state from the diagnostics
//     (6-digit snapshots: every diagnostic within 2e-4 of the uninterrupted run);
//   * a truncated last snapshot is skipped for the previous one;
//   * a folder with another mode list, or without snapshots, is refused;
//   * the background writer leaves the same bytes as writing before step() returns;
// plus the MODESBIN reader.
//
//   host_check <work_dir>        exit status 0 on success
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "../boson_cloud_binary_b200/host/CrankNicolsonModes.hpp"

namespace fs = std::filesystem;

namespace {

int failures = 0;

void require(bool ok, const std::string &msg)
{
    if (!ok) {
        std::cerr << "FAIL: " << msg << "\n";
        ++failures;
    }
}

// the fixture of the reference's tests/restart.cpp: a coarse evolving binary with
// both sinks, a phase average over one orbit and one Gaussian shell per mode
std::unique_ptr<CrankNicolsonModes> make_solver(int l_max = 2)
{
    // Nx, L, dt, eps, l_max, mu, M_c, q, a, R, counter, absorption, save_every,
    // ramp_periods, epsilon_smear
    auto cn = std::make_unique<CrankNicolsonModes>(65, 64.0, 2.0, 0.0, l_max, 0.2, 0.05, 0.5, 0.0, 20.0, false, true,
                                                   10, 0.5, 4.0, "");
    cn->verbose = false;
    cn->evolve_orbit = true;
    cn->steps_per_period = 32;
    cn->set_power_average_orbits(1.0);
    std::vector<dcomplex> psi0((size_t)cn->Nr * cn->n_modes, dcomplex(0, 0));
    double nrm = 0;
    for (int j = 0; j < cn->n_modes; ++j)
        for (int i = 1; i < cn->Nr - 1; ++i) {
            const double g = std::exp(-std::pow((cn->r[i] - 12.0 - 3 * j) / 6.0, 2));
            psi0[(size_t)j * cn->Nr + i] = std::polar(g, 0.3 * j);
            nrm += g * g;
        }
    for (auto &v : psi0) v /= std::sqrt(nrm * cn->dr);
    cn->set_initial_state_full(psi0);
    cn->initialize();
    return cn;
}

constexpr double kREx = 40.0;

// A fresh run of n_steps in work/name; returns its folder.
fs::path new_run(const fs::path &work, const std::string &name, int n_steps, bool async_output = true)
{
    fs::create_directories(work / name);
    fs::current_path(work / name);
    auto cn = make_solver();
    cn->async_output = async_output;
    cn->run(n_steps, kREx);
    return fs::absolute(cn->output_folder());
}

void resume_run(const fs::path &folder, int n_steps)
{
    auto cn = make_solver();
    cn->resume(folder.string(), n_steps, kREx);
}

std::string contents(const fs::path &p)
{
    std::ifstream in(p, std::ios::binary);
    std::stringstream ss;
    ss << in.rdbuf();
    return ss.str();
}

void require_identical(const fs::path &expected, const fs::path &actual, const std::string &what)
{
    int compared = 0;
    for (const auto &entry : fs::recursive_directory_iterator(expected)) {
        if (!entry.is_regular_file()) continue;
        const fs::path rel = fs::relative(entry.path(), expected);
        require(fs::exists(actual / rel), what + ": missing " + rel.string());
        require(contents(entry.path()) == contents(actual / rel), what + ": " + rel.string() + " differs");
        ++compared;
    }
    require(compared > 20, what + ": too few files compared");
}

std::vector<std::vector<double>> read_rows(const fs::path &p)
{
    std::ifstream in(p);
    std::vector<std::vector<double>> rows;
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream s(line);
        std::vector<double> row;
        double v;
        while (s >> v) row.push_back(v);
        rows.push_back(row);
    }
    return rows;
}

// Largest difference of two numeric files relative to the largest magnitude of the first.
double max_difference(const fs::path &a, const fs::path &b)
{
    const auto x = read_rows(a), y = read_rows(b);
    if (x.size() != y.size()) return 1e300;
    double scale = 0, worst = 0;
    for (const auto &row : x)
        for (double v : row) scale = std::max(scale, std::abs(v));
    for (size_t i = 0; i < x.size(); ++i) {
        if (x[i].size() != y[i].size()) return 1e300;
        for (size_t k = 0; k < x[i].size(); ++k) worst = std::max(worst, std::abs(x[i][k] - y[i][k]) / scale);
    }
    return worst;
}

const char *kDiagnostics[] = {"t.txt",    "R_orb.txt",  "theta_orb.txt", "Omega_orb.txt", "M_1.txt",      "q.txt",
                              "energy.txt", "p_bin.txt", "norms.txt",     "flux.txt",      "energy_flux.txt"};

void check_close(const fs::path &reference, const fs::path &run, const std::string &what)
{
    double worst = 0;
    for (const char *name : kDiagnostics) {
        const double d = max_difference(reference / name, run / name);
        worst = std::max(worst, d);
        require(d < 2e-4, what + ": " + name + " deviates by " + std::to_string(d));
    }
    std::printf("%s: largest diagnostic deviation %.3e\n", what.c_str(), worst);
}

void modesbin_reader(const fs::path &work)
{
    const std::string path = (work / "state.modesbin").string();
    std::ofstream out(path, std::ios::binary);
    out.write("MODESBIN", 8);
    const int32_t version = 1;
    const int64_t Nr = 5, Nm = 2;
    out.write(reinterpret_cast<const char *>(&version), 4);
    out.write(reinterpret_cast<const char *>(&Nr), 8);
    out.write(reinterpret_cast<const char *>(&Nm), 8);
    for (int k = 0; k < 2; ++k) {
        const int32_t lm[2] = {k == 0 ? 1 : 7, 1};  // (1,1) and (7,1): the second is not in the list
        out.write(reinterpret_cast<const char *>(lm), 8);
        for (int part = 0; part < 2; ++part)
            for (int i = 0; i < 5; ++i) {
                const double v = (k + 1) * 10 + i + 0.5 * part;
                out.write(reinterpret_cast<const char *>(&v), 8);
            }
    }
    out.close();
    const std::vector<mode> modes = {{0, 0}, {1, -1}, {1, 1}};
    const std::vector<dcomplex> psi = load_initial_modes_binary(path, modes);
    bool ok = psi.size() == 15;
    for (int i = 0; ok && i < 5; ++i)
        ok = psi[i] == dcomplex(0, 0) && psi[5 + i] == dcomplex(0, 0) && psi[10 + i] == dcomplex(10 + i, 10.5 + i);
    require(ok, "MODESBIN reader");
}

}  // namespace

int main(int argc, char **argv)
{
    if (argc != 2) {
        std::fprintf(stderr, "usage: %s work_dir\n", argv[0]);
        return 2;
    }
    const fs::path work = fs::absolute(argv[1]);
    const int n_full = 41, n_cut = 25;  // snapshots every 10 steps: the cut run ends 4 rows past snapshot 20
    const fs::path reference = new_run(work, "reference", n_full);

    {  // synchronous writing: the same folder
        const fs::path run = new_run(work, "synchronous", n_full, false);
        require_identical(reference, run, "synchronous writer");
        std::printf("background writer: folder identical to synchronous writing\n");
    }
    {  // exact resume from the checkpoint
        const fs::path run = new_run(work, "interrupted", n_cut);
        require(read_rows(run / "t.txt").size() == (size_t)(n_cut - 1), "interrupted run has the wrong row count");
        resume_run(run, n_full);
        require_identical(reference, run, "checkpoint resume");
        std::printf("checkpoint resume: folder identical to the uninterrupted run\n");
    }
    {  // crash mid-write: partial row and a snapshot ahead of the rows
        const fs::path run = new_run(work, "crashed", n_cut);
        std::ofstream(run / "flux.txt", std::ios::app) << "0.123 0.4";
        fs::copy_file(run / "psi" / "snapshot_000020.txt", run / "psi" / "snapshot_000030.txt");
        resume_run(run, n_full);
        require_identical(reference, run, "crash resume");
    }
    {  // no checkpoint: orbit state from the diagnostics
        const fs::path run = new_run(work, "reconstruct", n_cut);
        fs::remove(run / "checkpoint.bin");
        resume_run(run, n_full);
        check_close(reference, run, "diagnostics resume");
    }
    {  // truncated last snapshot: restart from the one before
        const fs::path run = new_run(work, "incomplete", 31);
        const fs::path last = run / "psi" / "snapshot_000030.txt";
        const std::string text = contents(last);
        std::ofstream(last, std::ios::trunc) << text.substr(0, text.size() / 2);
        resume_run(run, n_full);
        check_close(reference, run, "earlier-snapshot resume");
    }
    {  // refusals
        bool threw = false;
        try {
            auto cn = make_solver(3);
            cn->resume(reference.string(), n_full, kREx);
        } catch (const std::runtime_error &) {
            threw = true;
        }
        require(threw, "resume accepted a folder with a different mode list");
        const fs::path empty = work / "empty" / "Simulation_x";
        fs::create_directories(empty / "psi");
        for (const char *name : {"flux.txt", "energy_flux.txt", "energy.txt", "energy_modes.txt", "norms.txt", "t.txt",
                                 "p_bin.txt", "p_bin_inst.txt", "dV_bin_dt.txt", "R_orb.txt", "Omega_orb.txt",
                                 "M_1.txt", "q.txt", "theta_orb.txt"})
            std::ofstream(empty / name);
        threw = false;
        try {
            resume_run(empty, n_full);
        } catch (const std::runtime_error &) {
            threw = true;
        }
        require(threw, "resume without any snapshot did not fail");
    }
    modesbin_reader(work);
    {  // displaced_100_state: the centred state is the analytic 1s radial function
        std::vector<double> r(257);
        for (int i = 0; i < 257; ++i) r[i] = 40.0 * i / 256;
        std::vector<mode> modes;
        for (int l = 0; l <= 4; ++l)
            for (int m = -l; m <= l; m += 2) modes.push_back({l, m});
        const std::vector<dcomplex> psi = displaced_100_state(r, modes, 0.5, 0.0);
        double worst = 0.0;
        for (int i = 1; i < 256; ++i)
            worst = std::max(worst, std::abs(psi[i] - 2 * r[i] * std::exp(-r[i] / 4.0) / 8.0));
        require(worst < 1e-13, "displaced_100_state: centred state differs from 2 r e^{-r/a0} / a0^{3/2}");
    }
    std::printf(failures ? "host_check: %d failure(s)\n" : "host_check: OK\n", failures);
    return failures ? 1 : 0;
}

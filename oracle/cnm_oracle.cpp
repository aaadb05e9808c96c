/*
 * cnm_oracle.cpp -- CPU FP64 restatement of the Crank-Nicolson step of the
 * reference solver (rdellamonica/boson-cloud-binary, class CrankNicolsonModes).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle: the parity tests, the
 * smoke check and the benchmark's CPU-baseline leg load it as the checker.
 * The product (boson_cloud_binary_b200) never links or calls it.
 *
 * Parity status: the reference itself cannot be built here (its Eigen 3 and
 * GSL dependencies are absent), so this restatement is pinned by the
 * reference's own known-answer tests, ported to tests/test_oracle_*.py:
 * the dense formula matrices and dense-LU CN solve of
 * tests/parallel_correctness.cpp:53-107,150-193, the addition-theorem sink of
 * tests/SphericalAbsorptionReference.hpp:19-89, the analytic hydrogen
 * energies / CN phase / Peters law / balance laws of tests/physics.cpp, and
 * golden special-function tables made with sympy/scipy/numpy
 * (tests/golden/make_golden.py).
 *
 * Data structures follow the reference one to one: row-major CSR operators
 * H0, V1, V2, V, dVdt, H, A, B with the reference's union sparsity pattern
 * (src/CrankNicolsonModes_hamiltonian.cpp:111-174), assembled every step,
 * a Thomas block-Jacobi preconditioner that reads its coefficients through
 * binary searches (include/RadialBlockPreconditioner.hpp:44-98), and the
 * right-preconditioned BiCGSTAB recurrences of
 * src/CrankNicolsonModes_matrices.cpp:47-91 (sink path) and of Eigen's
 * BiCGSTAB (no-sink path; Eigen 3.4 IterativeLinearSolvers/BiCGSTAB.h,
 * restated from its published algorithm).  OpenMP parallelism sits on the
 * same loops as in the reference, so the timing of this file stands in for
 * the reference's own CPU cost.
 *
 * Third-party arithmetic restated here (neither library is vendored in the
 * reference; no version is pinned, CMakeLists.txt:8-9):
 *   GSL gsl_sf_coupling_3j      -> wigner3j()   (Racah formula, binary128)
 *   GSL gsl_sf_legendre_sphPlm  -> sph_plm_equator() (closed form at x = 0)
 *   GSL gsl_integration_glfixed -> gauss_legendre() (Newton on P_n)
 *   Eigen row-major SpMV, dot (conjugate-linear in the first argument),
 *   squaredNorm, 2x2 inverse.
 */
#include <quadmath.h>
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <deque>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

using cd = std::complex<double>;
using cvec = std::vector<cd>;
const cd I(0.0, 1.0);

// ---------------------------------------------------------------- special functions

__float128 qfact(int n)
{
    static std::vector<__float128> table;
    if (table.empty()) {
        table.resize(301);
        table[0] = 1;
        for (int k = 1; k <= 300; ++k) table[k] = table[k - 1] * k;
    }
    if (n < 0 || n > 300) throw std::invalid_argument("factorial argument out of range");
    return table[n];
}

// Wigner 3j symbol with doubled arguments, as gsl_sf_coupling_3j takes them.
// Racah's single-sum formula evaluated in binary128 so that the alternating sum
// keeps full double precision for every l <= 64.
double wigner3j(int tj1, int tj2, int tj3, int tm1, int tm2, int tm3)
{
    if (tm1 + tm2 + tm3 != 0) return 0.0;
    if (((tj1 + tm1) & 1) || ((tj2 + tm2) & 1) || ((tj3 + tm3) & 1)) return 0.0;
    if (std::abs(tm1) > tj1 || std::abs(tm2) > tj2 || std::abs(tm3) > tj3) return 0.0;
    if (tj3 < std::abs(tj1 - tj2) || tj3 > tj1 + tj2 || ((tj1 + tj2 + tj3) & 1)) return 0.0;
    // The reference only uses integer angular momenta.
    if ((tj1 & 1) || (tj2 & 1) || (tj3 & 1)) throw std::invalid_argument("half-integer 3j");
    const int j1 = tj1 / 2, j2 = tj2 / 2, j3 = tj3 / 2;
    const int m1 = tm1 / 2, m2 = tm2 / 2, m3 = tm3 / 2;
    const int kmin = std::max({0, j2 - j3 - m1, j1 - j3 + m2});
    const int kmax = std::min({j1 + j2 - j3, j1 - m1, j2 + m2});
    if (m1 == 0 && m2 == 0 && ((j1 + j2 + j3) & 1)) return 0.0;
    __float128 sum = 0, largest = 0;
    for (int k = kmin; k <= kmax; ++k) {
        const __float128 den = qfact(k) * qfact(j3 - j2 + k + m1) * qfact(j3 - j1 + k - m2) *
                               qfact(j1 + j2 - j3 - k) * qfact(j1 - k - m1) * qfact(j2 - k + m2);
        sum += ((k & 1) ? -1 : 1) / den;
        largest = fmaxq(largest, 1 / den);
    }
    // An exact (accidental) zero leaves only binary128 rounding residue behind.
    if (fabsq(sum) <= 1e-26Q * largest) return 0.0;
    const __float128 delta = qfact(j1 + j2 - j3) * qfact(j1 - j2 + j3) * qfact(-j1 + j2 + j3) /
                             qfact(j1 + j2 + j3 + 1);
    const __float128 pre = sqrtq(delta * qfact(j1 + m1) * qfact(j1 - m1) * qfact(j2 + m2) *
                                 qfact(j2 - m2) * qfact(j3 + m3) * qfact(j3 - m3));
    const int phase = j1 - j2 - m3;
    return static_cast<double>(((phase & 1) ? -1 : 1) * pre * sum);
}

// Normalised associated Legendre function with the Condon-Shortley phase at
// x = cos(pi/2) = 0, i.e. gsl_sf_legendre_sphPlm(l, m, 0.0) for 0 <= m <= l:
// sqrt((2l+1)/(4pi) (l-m)!/(l+m)!) P_l^m(0), P_l^m(0) = (-1)^((l+m)/2) (l+m-1)!!/(l-m)!!.
double sph_plm_equator(int l, int m)
{
    if (m < 0 || m > l) throw std::invalid_argument("sph_plm_equator needs 0 <= m <= l");
    if ((l + m) & 1) return 0.0;
    __float128 dfn = 1, dfd = 1;  // (l+m-1)!! and (l-m)!!
    for (int k = l + m - 1; k > 1; k -= 2) dfn *= k;
    for (int k = l - m; k > 1; k -= 2) dfd *= k;
    const __float128 plm = ((((l + m) / 2) & 1) ? -1 : 1) * dfn / dfd;
    const __float128 norm = sqrtq((2 * l + 1) / (4 * M_PIq) * qfact(l - m) / qfact(l + m));
    return static_cast<double>(norm * plm);
}

// n-point Gauss-Legendre rule on [a, b], nodes in increasing order.
void gauss_legendre(int n, double a, double b, std::vector<double> &x, std::vector<double> &w)
{
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int k = 0; k < n; ++k) {
        // k-th root counted from the right end, refined by Newton in binary128.
        __float128 z = cosq(M_PIq * (k + 0.75Q) / (n + 0.5Q));
        __float128 dp = 0;
        for (int it = 0; it < 100; ++it) {
            __float128 p0 = 1, p1 = z;
            for (int j = 2; j <= n; ++j) {
                const __float128 p2 = ((2 * j - 1) * z * p1 - (j - 1) * p0) / j;
                p0 = p1;
                p1 = p2;
            }
            if (n == 1) p0 = 1;
            dp = n * (z * p1 - p0) / (z * z - 1);
            const __float128 dz = p1 / dp;
            z -= dz;
            if (fabsq(dz) < 1e-32Q) break;
        }
        {
            __float128 p0 = 1, p1 = z;
            for (int j = 2; j <= n; ++j) {
                const __float128 p2 = ((2 * j - 1) * z * p1 - (j - 1) * p0) / j;
                p0 = p1;
                p1 = p2;
            }
            if (n == 1) p0 = 1;
            dp = n * (z * p1 - p0) / (z * z - 1);
        }
        const __float128 wz = 2 / ((1 - z * z) * dp * dp);
        const int idx = n - 1 - k;  // increasing order
        x[idx] = static_cast<double>((b - a) / 2.0Q * z + (a + b) / 2.0Q);
        w[idx] = static_cast<double>((b - a) / 2.0Q * wz);
    }
}

// ---------------------------------------------------------------- vector helpers (Eigen semantics)

// Reductions are summed in fixed chunks, then over the chunks in order, so the
// result does not depend on the number of OpenMP threads.
constexpr int64_t kChunk = 16384;

template <class T, class F>
T chunked_sum(int64_t n, F f)
{
    const int64_t nc = (n + kChunk - 1) / kChunk;
    std::vector<T> part(nc, T(0));
#pragma omp parallel for schedule(static) if (nc > 1)
    for (int64_t c = 0; c < nc; ++c) {
        T s(0);
        const int64_t e = std::min(n, (c + 1) * kChunk);
        for (int64_t i = c * kChunk; i < e; ++i) s += f(i);
        part[c] = s;
    }
    T s(0);
    for (const T &v : part) s += v;
    return s;
}

cd dot(const cvec &a, const cvec &b)  // sum conj(a_i) b_i, like Eigen's a.dot(b)
{
    return chunked_sum<cd>((int64_t)a.size(), [&](int64_t i) { return std::conj(a[i]) * b[i]; });
}

double sqnorm(const cvec &a)
{
    return chunked_sum<double>((int64_t)a.size(), [&](int64_t i) { return std::norm(a[i]); });
}

bool all_finite(const cvec &a)
{
    for (const cd &v : a)
        if (!std::isfinite(v.real()) || !std::isfinite(v.imag())) return false;
    return true;
}

// ---------------------------------------------------------------- CSR matrix (row-major)

struct Csr {
    int64_t n = 0;
    std::vector<int64_t> outer;
    std::vector<int32_t> inner;
    cvec val;

    cd coeff(int64_t r, int64_t c) const
    {
        const int32_t *b = inner.data() + outer[r], *e = inner.data() + outer[r + 1];
        const int32_t *f = std::lower_bound(b, e, (int32_t)c);
        return (f != e && *f == c) ? val[f - inner.data()] : cd(0.0);
    }

    // y = M x, each row summed in storage order (Eigen's row-major product).
    void apply(const cvec &x, cvec &y) const
    {
        y.assign(n, cd(0.0));
#pragma omp parallel for schedule(static)
        for (int64_t r = 0; r < n; ++r) {
            cd t(0.0);
            for (int64_t s = outer[r]; s < outer[r + 1]; ++s) t += val[s] * x[inner[s]];
            y[r] = t;
        }
    }
};

// ---------------------------------------------------------------- rolling phase average

// Restatement of src/RollingPhase.cpp:24-129.
class RollingPhaseAverage {
public:
    explicit RollingPhaseAverage(double n_orbits = 2.0) : window_phase_(2.0 * M_PI * n_orbits)
    {
        if (n_orbits <= 0.0) throw std::invalid_argument("RollingPhaseAverage: n_orbits must be positive");
    }
    double update(double time, double phase, double value)
    {
        if (!has_previous_) {
            previous_ = {time, phase, value};
            initial_phase_ = phase;
            has_previous_ = true;
            average_ = value;
            return average_;
        }
        if (time <= previous_.time) throw std::runtime_error("RollingPhaseAverage: time must increase");
        if (phase <= previous_.phase) throw std::runtime_error("RollingPhaseAverage: phase must increase");
        Segment seg{previous_.time, time, previous_.phase, phase, previous_.value, value, 0.0};
        seg.integral = 0.5 * (seg.value0 + seg.value1) * (seg.time1 - seg.time0);
        segments_.push_back(seg);
        integral_ += seg.integral;
        duration_ += seg.time1 - seg.time0;
        if (phase - initial_phase_ >= window_phase_) ready_ = true;
        const double cut = phase - window_phase_;
        while (!segments_.empty() && segments_.front().phase1 <= cut) {
            integral_ -= segments_.front().integral;
            duration_ -= segments_.front().time1 - segments_.front().time0;
            segments_.pop_front();
        }
        if (!segments_.empty()) {
            Segment &f = segments_.front();
            if (f.phase0 < cut && cut < f.phase1) {
                const double frac = (cut - f.phase0) / (f.phase1 - f.phase0);
                const double tc = f.time0 + frac * (f.time1 - f.time0);
                const double vc = f.value0 + frac * (f.value1 - f.value0);
                integral_ -= 0.5 * (f.value0 + vc) * (tc - f.time0);
                duration_ -= tc - f.time0;
                f.time0 = tc;
                f.phase0 = cut;
                f.value0 = vc;
                f.integral = 0.5 * (f.value0 + f.value1) * (f.time1 - f.time0);
            }
        }
        duration_ = std::max(duration_, 0.0);
        average_ = duration_ > 0.0 ? integral_ / duration_ : value;
        previous_ = {time, phase, value};
        return average_;
    }

private:
    struct Sample { double time, phase, value; };
    struct Segment { double time0, time1, phase0, phase1, value0, value1, integral; };
    double window_phase_;
    std::deque<Segment> segments_;
    Sample previous_{};
    bool has_previous_ = false, ready_ = false;
    double initial_phase_ = 0, integral_ = 0, duration_ = 0, average_ = 0;
};

// ---------------------------------------------------------------- the solver

struct Mode { int l, m; };
struct Term { int l_star; cd angular; };
struct ModePair {
    int row_mode, col_mode, m_star;
    std::vector<Term> terms;
    std::vector<int64_t> offsets;
};
struct Profile { double radius = -1.0, width = -1.0; std::vector<double> multipoles; };
struct Sink { cvec v; double strength = 0.0; };

struct Oracle {
    // public state of the reference class (include/CrankNicolsonModes.hpp:88-164)
    int Nr, save_every, l_max, n_modes = 0;
    double epsilon, mu, q, R, theta, phase, Omega, Omega_0, P, R1, R2, M1, M2, a, L, dr, dt;
    bool counter;
    double M_c;
    bool evolve_orbit = true, ramp_secondary_potential = true;
    double steps_per_period = 50.0;
    bool use_block_preconditioner = true;
    double last_solver_residual = 0.0;
    int last_solver_iterations = 0;
    std::vector<double> t, r;
    cvec psi;
    bool mask = false, cap = false;
    std::vector<Mode> modes;
    Csr H, H0, A, B, V1, V2, V, dVdt, CAP;

    // private state
    bool isolated_black_hole = false;
    double ramp_periods, initial_period;
    cvec psi_last, damping_mask;
    double ramp_factor = 0.0, potential_ramp_factor = 0.0;
    double r_ex = 0.0;
    int idx_ex = 0;
    double t_i = 0.0;
    double orbits_average = 2.0;
    RollingPhaseAverage power_average{2.0};
    std::vector<ModePair> mode_pairs;
    std::vector<double> radial_f1, radial_f2;
    cvec stationary_values;
    std::vector<int64_t> potential_offsets;
    bool absorption;
    Profile profile1, profile2;
    double Ah1 = 0.0, Ah2 = 0.0, epsilon_smear;
    Sink sink1, sink2;
    bool sink_active = false;
    int mode00 = -1;
    double p_bin = 0.0;
    bool initialized = false;

    // solver knobs (the reference hard-codes 1e-10 / 500, _matrices.cpp:19-20)
    double tolerance = 1e-10;
    int max_iterations = 500;
    double accept_residual = 1e-9;

    double ramp_end_time() const { return ramp_periods * initial_period; }

    // src/CrankNicolsonModes.cpp:11-50
    Oracle(int Nr_, double L_, double dt_i, double eps, int lmax, double mu_, double Mc, double q_, double a_,
           double R_, bool counter_, bool absorption_, int save_every_, double ramp_periods_, double smear)
        : Nr(Nr_), save_every(save_every_), l_max(lmax), epsilon(eps), mu(mu_), q(q_), R(R_), a(a_), L(L_),
          dr(L_ / (Nr_ - 1)), dt(dt_i), counter(counter_), M_c(Mc), ramp_periods(ramp_periods_),
          initial_period(2.0 * M_PI / std::sqrt((1 + q_) / std::pow(R_, 3))), absorption(absorption_),
          epsilon_smear(smear)
    {
        if (Nr < 3 || l_max < 0 || L <= 0.0 || dt <= 0.0 || save_every <= 0)
            throw std::invalid_argument("Require Nr >= 3, l_max >= 0, and positive L, dt, save_every");
        Omega = 0.0;
        Omega_0 = std::sqrt((1.0 + q) / std::pow(R, 3));
        P = initial_period;
        R1 = q / (1 + q) * R;
        R2 = 1 / (1 + q) * R;
        theta = 0.0;
        phase = 0.0;
        M1 = 1.0;
        M2 = q;
        r.resize(Nr);
        for (int i = 0; i < Nr; i++) r[i] = epsilon + i * dr;
        for (int l = 0; l <= l_max; ++l)
            for (int m = -l; m <= l; ++m)
                if (std::abs(l - m) % 2 == 0) { modes.push_back({l, m}); ++n_modes; }
        build_stationary_hamiltonian();
    }

    int64_t size() const { return (int64_t)Nr * n_modes; }

    // src/CrankNicolsonModes_hamiltonian.cpp:44-66, as a directly built CSR.
    void build_stationary_hamiltonian()
    {
        H0.n = size();
        H0.outer.assign(H0.n + 1, 0);
        for (int j = 0; j < n_modes; ++j)
            for (int i = 1; i < Nr - 1; ++i) H0.outer[(int64_t)j * Nr + i + 1] = 3;
        for (int64_t k = 0; k < H0.n; ++k) H0.outer[k + 1] += H0.outer[k];
        H0.inner.resize(H0.outer.back());
        H0.val.resize(H0.outer.back());
        const cd alpha = 1.0 / (dr * dr);
        for (int j = 0; j < n_modes; ++j)
            for (int i = 1; i < Nr - 1; ++i) {
                const int64_t row = (int64_t)j * Nr + i, s = H0.outer[row];
                H0.inner[s] = (int32_t)(row - 1);
                H0.inner[s + 1] = (int32_t)row;
                H0.inner[s + 2] = (int32_t)(row + 1);
                H0.val[s + 1] = -(-2.0 * alpha - modes[j].l * (modes[j].l + 1) / (r[i] * r[i])) / (2 * mu);
                H0.val[s] = -alpha / (2 * mu);
                H0.val[s + 2] = -alpha / (2 * mu);
            }
    }

    // src/CrankNicolsonModes.cpp:130-143
    void set_initial_state_full(const cvec &psi0)
    {
        if ((int64_t)psi0.size() != size())
            throw std::invalid_argument("Initial state size does not match the radial grid and modes");
        psi = psi0;
        const double s = std::sqrt(M_c / mu);
        for (cd &v : psi) v *= s;
        psi_last.assign(size(), cd(0.0));
    }

    // src/CrankNicolsonModes.cpp:58-74
    void configure_isolated_black_hole(double x)
    {
        if (!std::isfinite(x) || std::abs(x) >= L)
            throw std::invalid_argument("The isolated BH must lie inside the radial domain");
        if (initialized) throw std::logic_error("Configure the isolated BH before initialize()");
        isolated_black_hole = true;
        evolve_orbit = false;
        M1 = 1.0;
        M2 = q = 0.0;
        R = R1 = std::abs(x);
        R2 = 0.0;
        theta = x < 0.0 ? M_PI : 0.0;
        phase = 0.0;
        Omega = Omega_0 = 0.0;
        ramp_periods = 0.0;
    }

    // src/CrankNicolsonModes.cpp:76-98
    void initialize()
    {
        build_coupling_cache();
        build_sparse_element_caches();
        t_i = 0.0;
        build_time_dependent_perturbation(0.0);
        A = H;
        B = H;
        update_CN_values();
        initialized = true;
    }

    void set_power_average_orbits(double n)
    {
        power_average = RollingPhaseAverage(n);
        orbits_average = n;
    }

    // src/CrankNicolsonModes_hamiltonian.cpp:12-42
    double F1(double rr, int ls) const
    {
        if (rr >= R1) return 1 / (1 + q) * std::pow(R1, ls) / std::pow(rr, ls + 1);
        return 1 / (1 + q) * std::pow(rr, ls) / std::pow(R1, ls + 1);
    }
    double F2(double rr, int ls) const
    {
        if (rr >= R2) return 1.0 * q / (1 + q) * std::pow(R2, ls) / std::pow(rr, ls + 1);
        return 1.0 * q / (1 + q) * std::pow(rr, ls) / std::pow(R2, ls + 1);
    }

    // src/CrankNicolsonModes_hamiltonian.cpp:68-104
    void build_coupling_cache()
    {
        mode_pairs.clear();
        for (int j = 0; j < n_modes; ++j)
            for (int k = 0; k < n_modes; ++k) {
                const int l = modes[j].l, m = modes[j].m, l1 = modes[k].l, m1 = modes[k].m;
                const int ms = m1 - m;
                ModePair pair{j, k, ms, {}, {}};
                for (int ls = std::abs(l1 - l); ls <= l1 + l; ++ls) {
                    if (std::abs(ms) > ls || (l + l1 + ls) % 2 != 0) continue;
                    const double w1 = wigner3j(2 * ls, 2 * l1, 2 * l, 0, 0, 0);
                    const double w2 = wigner3j(2 * ls, 2 * l1, 2 * l, -2 * ms, 2 * m1, -2 * m);
                    double y = sph_plm_equator(ls, std::abs(ms));
                    if (ms < 0 && std::abs(ms) % 2 != 0) y = -y;
                    const double pref = (m1 % 2 == 0 ? 1.0 : -1.0) *
                                        std::sqrt((2.0 * l + 1) * (2.0 * l1 + 1) * (2.0 * ls + 1) / (4.0 * M_PI));
                    const cd ang = cd(pref) * cd(w1) * cd(w2) * cd(y);
                    if (std::abs(ang) != 0.0) pair.terms.push_back({ls, ang});
                }
                if (!pair.terms.empty()) mode_pairs.push_back(std::move(pair));
            }
    }

    cd orbital_phase(int ms) const { return std::exp(I * static_cast<double>(ms) * theta); }

    // src/CrankNicolsonModes_hamiltonian.cpp:111-174: fixed union patterns and offset caches.
    void build_sparse_element_caches()
    {
        const int64_t n = size();
        // V pattern: row (j, i) holds (k, i) for every pair (j, k), i = 1..Nr-2, columns increasing.
        std::vector<int> pairs_in_row(n_modes, 0);
        for (const auto &p : mode_pairs) pairs_in_row[p.row_mode]++;
        V1.n = n;
        V1.outer.assign(n + 1, 0);
        for (int j = 0; j < n_modes; ++j)
            for (int i = 1; i < Nr - 1; ++i) V1.outer[(int64_t)j * Nr + i + 1] = pairs_in_row[j];
        for (int64_t k = 0; k < n; ++k) V1.outer[k + 1] += V1.outer[k];
        V1.inner.assign(V1.outer.back(), 0);
        V1.val.assign(V1.outer.back(), cd(0.0));
        std::vector<int> cursor(n_modes, 0);
        for (auto &p : mode_pairs) {
            p.offsets.resize(Nr - 2);
            const int c = cursor[p.row_mode]++;
            for (int i = 1; i < Nr - 1; ++i) {
                const int64_t row = (int64_t)p.row_mode * Nr + i;
                const int64_t slot = V1.outer[row] + c;
                V1.inner[slot] = (int32_t)((int64_t)p.col_mode * Nr + i);
                p.offsets[i - 1] = slot;
            }
        }
        V2 = V1;
        V = V1;
        dVdt = V1;
        if (absorption) {
            profile1 = {};
            profile2 = {};
            mode00 = -1;
            for (int j = 0; j < n_modes; ++j)
                if (modes[j].l == 0 && modes[j].m == 0) mode00 = j;
            sink1 = {};
            sink2 = {};
        }
        // H = H0 + V + Id pattern (sorted union per row).
        H.n = n;
        H.outer.assign(n + 1, 0);
        std::vector<std::vector<int32_t>> cols(n);
#pragma omp parallel for schedule(static)
        for (int64_t row = 0; row < n; ++row) {
            std::vector<int32_t> c;
            for (int64_t s = H0.outer[row]; s < H0.outer[row + 1]; ++s) c.push_back(H0.inner[s]);
            for (int64_t s = V1.outer[row]; s < V1.outer[row + 1]; ++s) c.push_back(V1.inner[s]);
            c.push_back((int32_t)row);
            std::sort(c.begin(), c.end());
            c.erase(std::unique(c.begin(), c.end()), c.end());
            cols[row] = std::move(c);
        }
        for (int64_t row = 0; row < n; ++row) H.outer[row + 1] = H.outer[row] + (int64_t)cols[row].size();
        H.inner.resize(H.outer.back());
        H.val.assign(H.outer.back(), cd(0.0));
        for (int64_t row = 0; row < n; ++row)
            std::copy(cols[row].begin(), cols[row].end(), H.inner.begin() + H.outer[row]);
        stationary_values.assign(H.outer.back(), cd(0.0));
        potential_offsets.assign(H.outer.back(), -1);
#pragma omp parallel for schedule(static)
        for (int64_t row = 0; row < n; ++row)
            for (int64_t s = H.outer[row]; s < H.outer[row + 1]; ++s) {
                stationary_values[s] = H0.coeff(row, H.inner[s]);
                const int32_t *b = V.inner.data() + V.outer[row], *e = V.inner.data() + V.outer[row + 1];
                const int32_t *f = std::lower_bound(b, e, H.inner[s]);
                if (f != e && *f == H.inner[s]) potential_offsets[s] = f - V.inner.data();
            }
        radial_f1.assign((size_t)(2 * l_max + 1) * Nr, 0.0);
        radial_f2.assign(radial_f1.size(), 0.0);
    }

    // src/CrankNicolsonModes_hamiltonian.cpp:176-222
    void build_static_perturbation()
    {
#pragma omp parallel for schedule(static)
        for (int l = 0; l <= 2 * l_max; ++l)
            for (int i = 1; i < Nr - 1; ++i) {
                radial_f1[(size_t)l * Nr + i] = F1(r[i], l);
                radial_f2[(size_t)l * Nr + i] = F2(r[i], l);
            }
        std::vector<cd> phases(4 * l_max + 1);
        for (int m = -2 * l_max; m <= 2 * l_max; ++m) phases[m + 2 * l_max] = orbital_phase(m);
        const double phase_sign = counter ? -1.0 : 1.0;
#pragma omp parallel for schedule(static)
        for (size_t p = 0; p < mode_pairs.size(); ++p) {
            const auto &pair = mode_pairs[p];
            const cd ph = phases[pair.m_star + 2 * l_max];
            const double parity = pair.m_star % 2 == 0 ? 1.0 : -1.0;
            for (int i = 1; i < Nr - 1; ++i) {
                cd v1 = 0.0, v2 = 0.0, der = 0.0;
                for (const auto &term : pair.terms) {
                    const cd common = -mu * (M1 + M2) * 4.0 * M_PI / (2.0 * term.l_star + 1.0) * term.angular * ph;
                    const cd value1 = common * radial_f1[(size_t)term.l_star * Nr + i];
                    const cd value2 = common * (parity * radial_f2[(size_t)term.l_star * Nr + i]);
                    v1 += value1;
                    v2 += value2;
                    der += (value1 + potential_ramp_factor * value2) * phase_sign * I *
                           static_cast<double>(pair.m_star) * Omega;
                }
                const int64_t off = pair.offsets[i - 1];
                V1.val[off] = v1;
                V2.val[off] = v2;
                V.val[off] = v1 + v2 * potential_ramp_factor;
                dVdt.val[off] = der;
            }
        }
    }

    // src/CrankNicolsonModes_hamiltonian.cpp:224-243
    void assemble_hamiltonian(bool include_absorption)
    {
        sink_active = include_absorption;
#pragma omp parallel for schedule(static)
        for (int64_t row = 0; row < H.n; ++row)
            for (int64_t s = H.outer[row]; s < H.outer[row + 1]; ++s) {
                cd value = stationary_values[s];
                if (potential_offsets[s] >= 0) value += V.val[potential_offsets[s]];
                if (cap && H.inner[s] == row) value += CAP.coeff(row, row);
                H.val[s] = value;
            }
    }

    // src/CrankNicolsonModes_hamiltonian.cpp:245-268
    void build_time_dependent_perturbation(double time)
    {
        ramp_factor = 1.0;
        if (isolated_black_hole) {
            Omega = 0.0;
        } else if (time < ramp_end_time()) {
            const double x = time / ramp_end_time();
            ramp_factor = 3.0 * x * x - 2.0 * x * x * x;
            Omega = Omega_0 * ramp_factor;
        } else {
            Omega = std::sqrt((M1 + M2) / std::pow(R, 3));
        }
        potential_ramp_factor = ramp_secondary_potential ? ramp_factor : 1.0;
        build_static_perturbation();
        if (absorption) build_spherical_absorption();
        assemble_hamiltonian(absorption && time >= ramp_end_time());
    }

    // src/CrankNicolsonModes_matrices.cpp:27-40
    void update_CN_values()
    {
        const cd scale = I * (dt * 0.5);
#pragma omp parallel for schedule(static)
        for (int64_t row = 0; row < H.n; ++row)
            for (int64_t s = H.outer[row]; s < H.outer[row + 1]; ++s) {
                const cd diag = H.inner[s] == row ? 1.0 : 0.0;
                A.val[s] = diag + scale * H.val[s];
                B.val[s] = diag - scale * H.val[s];
            }
    }

    // ------------------------------------------------------------ absorption (_absorption.cpp)

    // src/CrankNicolsonModes_absorption.cpp:12-81
    void update_absorption_profile(Profile &profile, double radius, double width)
    {
        const int degree = 2 * l_max;
        const size_t sz = (size_t)(degree + 1) * Nr;
        if (profile.radius == radius && profile.width == width && profile.multipoles.size() == sz) return;
        profile.radius = radius;
        profile.width = width;
        profile.multipoles.assign(sz, 0.0);
        if (width < dr || width <= 0.0 || radius < 0.0) return;
        const int nq = std::max(128, degree + 16);
        std::vector<double> nodes, weights;
        gauss_legendre(nq, 0.0, 1.0, nodes, weights);
#pragma omp parallel for schedule(static)
        for (int i = 1; i < Nr - 1; ++i) {
            const double delta = r[i] - radius;
            if (std::abs(delta) >= width) continue;
            if (radius == 0.0) {
                const double x = r[i] / width;
                profile.multipoles[i] = 4.0 * M_PI * std::exp(-1.0 / (1.0 - x * x));
                continue;
            }
            const double product = 2.0 * r[i] * radius;
            const double capv = std::min(2.0, (width * width - delta * delta) / product);
            for (int k = 0; k < nq; ++k) {
                const double z = capv * nodes[k];
                const double u = 1.0 - z;
                const double d2 = delta * delta + product * z;
                const double weight = 2.0 * M_PI * capv * weights[k] * std::exp(-1.0 / (1.0 - d2 / (width * width)));
                double prev = 1.0, cur = u;
                profile.multipoles[i] += weight;
                if (degree > 0) profile.multipoles[(size_t)Nr + i] += weight * cur;
                for (int l = 2; l <= degree; ++l) {
                    const double next = ((2 * l - 1) * u * cur - (l - 1) * prev) / l;
                    profile.multipoles[(size_t)l * Nr + i] += weight * next;
                    prev = cur;
                    cur = next;
                }
            }
        }
        double norm = 0.0;
        for (int i = 1; i < Nr - 1; ++i) norm += dr * r[i] * r[i] * profile.multipoles[i];
        if (norm > 0.0)
            for (double &v : profile.multipoles) v /= norm;
    }

    double absorption_rate(const Sink &s, const cvec &state) const
    {
        if (s.strength == 0.0 || (int64_t)s.v.size() != (int64_t)state.size()) return 0.0;
        return mu * dr * s.strength * std::norm(dot(s.v, state));
    }

    // src/CrankNicolsonModes_absorption.cpp:100-117
    cvec apply_sink(const cvec &state) const
    {
        cvec res(state.size(), cd(0.0));
        if (!sink_active) return res;
        for (const Sink *s : {&sink1, &sink2})
            if (s->strength != 0.0 && s->v.size() == state.size()) {
                const cd c = s->strength * dot(s->v, state);
                for (size_t i = 0; i < res.size(); ++i) res[i] += c * s->v[i];
            }
        return res;
    }

    cvec schrodinger_rhs(const cvec &state) const
    {
        cvec hs;
        H.apply(state, hs);
        cvec res(state.size());
        for (size_t i = 0; i < res.size(); ++i) res[i] = -I * hs[i];
        if (sink_active) {
            const cvec g = apply_sink(state);
            for (size_t i = 0; i < res.size(); ++i) res[i] -= 0.5 * g[i];
        }
        return res;
    }

    double sink_strength(int body) const
    {
        const Sink &s = body == 1 ? sink1 : sink2;
        if (!sink_active || s.strength == 0.0) return 0.0;
        return s.strength * sqnorm(s.v);
    }

    // src/CrankNicolsonModes_absorption.cpp:127-151
    void build_swave_projector(const Profile &profile, bool secondary, cvec &v) const
    {
        v.assign(size(), cd(0.0));
        if (mode00 < 0) return;
        const double sqrt4pi = std::sqrt(4.0 * M_PI);
        for (const auto &pair : mode_pairs) {
            if (pair.col_mode != mode00) continue;
            const cd ph = orbital_phase(pair.m_star);
            const double parity = secondary && pair.m_star % 2 != 0 ? -1.0 : 1.0;
            for (int i = 1; i < Nr - 1; ++i) {
                cd kappa = 0.0;
                for (const auto &term : pair.terms)
                    kappa += profile.multipoles[(size_t)term.l_star * Nr + i] * term.angular * ph;
                v[(size_t)pair.row_mode * Nr + i] = r[i] * sqrt4pi * parity * kappa;
            }
        }
    }

    // src/CrankNicolsonModes_absorption.cpp:153-182
    void build_spherical_absorption()
    {
        update_absorption_profile(profile1, R1, epsilon_smear * M1);
        update_absorption_profile(profile2, R2, epsilon_smear * M2);
        double ramp = 1.0;
        if (!isolated_black_hole && t_i < ramp_end_time()) {
            ramp = 0.0;
        } else if (!isolated_black_hole && t_i < ramp_end_time() + initial_period) {
            const double x = (t_i - ramp_end_time()) / initial_period;
            ramp = 3.0 * x * x - 2.0 * x * x * x;
        }
        Ah1 = 16.0 * M_PI * M1 * M1 * ramp;
        Ah2 = 16.0 * M_PI * M2 * M2 * ramp;
        build_swave_projector(profile1, false, sink1.v);
        sink1.strength = Ah1 * dr;
        build_swave_projector(profile2, true, sink2.v);
        sink2.strength = Ah2 * dr;
    }

    // ------------------------------------------------------------ outer boundary (_outgoing.cpp)

    void build_damping_mask(double fL, double W, int n)
    {
        damping_mask.assign(size(), cd(1.0));
        mask = true;
        const int idx = (int)std::floor(L * fL / dr);
        const double rm = fL * L, Lm = (1 - fL) * L;
        for (int i = 0; i < Nr; i++)
            for (int j = 0; j < n_modes; j++)
                damping_mask[i + (size_t)j * Nr] = i >= idx ? std::exp(-W * std::pow((r[i] - rm) / Lm, n)) : 1.0;
    }

    void build_cap(double fL, double W, int n)
    {
        CAP.n = size();
        CAP.outer.assign(CAP.n + 1, 0);
        cap = true;
        const int idx = (int)std::floor(L * fL / dr);
        const double rc = fL * L, Lc = (1 - fL) * L;
        for (int j = 0; j < n_modes; ++j)
            for (int i = idx < 0 ? 0 : idx; i < Nr; ++i) CAP.outer[(int64_t)j * Nr + i + 1] = 1;
        for (int64_t k = 0; k < CAP.n; ++k) CAP.outer[k + 1] += CAP.outer[k];
        CAP.inner.resize(CAP.outer.back());
        CAP.val.resize(CAP.outer.back());
        for (int j = 0; j < n_modes; ++j)
            for (int i = idx < 0 ? 0 : idx; i < Nr; ++i) {
                const int64_t row = (int64_t)j * Nr + i;
                CAP.inner[CAP.outer[row]] = (int32_t)row;
                CAP.val[CAP.outer[row]] = -I * W * std::pow((r[i] - rc) / (r[i] - Lc), n);
            }
    }

    // ------------------------------------------------------------ preconditioner

    // include/RadialBlockPreconditioner.hpp:44-98
    struct BlockPrecond {
        int block = 0;
        cvec inv_diag, lower, upper;
        bool ok = false;
        void factorize(const Csr &M, int bs)
        {
            block = bs;
            const int64_t n = M.n;
            inv_diag.resize(n);
            lower.resize(n);
            upper.resize(n);
            const int64_t blocks = n / bs;
            int failed = 0;
#pragma omp parallel for schedule(static) reduction(| : failed)
            for (int64_t b = 0; b < blocks; ++b) {
                const int64_t start = b * bs;
                for (int i = 0; i < bs; ++i) {
                    const int64_t row = start + i;
                    lower[row] = i > 0 ? M.coeff(row, row - 1) : cd(0);
                    upper[row] = i + 1 < bs ? M.coeff(row, row + 1) : cd(0);
                    cd pivot = M.coeff(row, row);
                    if (i > 0) pivot -= lower[row] * inv_diag[row - 1] * upper[row - 1];
                    if (std::abs(pivot) == 0.0 || !std::isfinite(std::abs(pivot))) {
                        failed = 1;
                        inv_diag[row] = 0.0;
                    } else {
                        inv_diag[row] = cd(1) / pivot;
                    }
                }
            }
            ok = !failed;
        }
        cvec solve(const cvec &rhs) const
        {
            cvec x(rhs.size());
            const int64_t blocks = (int64_t)rhs.size() / block;
#pragma omp parallel for schedule(static)
            for (int64_t b = 0; b < blocks; ++b) {
                const int64_t start = b * block, end = start + block;
                x[start] = rhs[start] * inv_diag[start];
                for (int64_t row = start + 1; row < end; ++row)
                    x[row] = (rhs[row] - lower[row] * x[row - 1]) * inv_diag[row];
                for (int64_t row = end - 2; row >= start; --row) x[row] -= upper[row] * inv_diag[row] * x[row + 1];
            }
            return x;
        }
    };
    BlockPrecond block;

    // ------------------------------------------------------------ Krylov

    // src/CrankNicolsonModes_matrices.cpp:47-91 (restart at |rho| < 1e-32 |r0|^2)
    template <class AF, class MF>
    static bool bicgstab_ref(const AF &apply_A, const MF &apply_M, const cvec &b, cvec &x, double tol, int maxit,
                             int &iterations)
    {
        const double b2 = sqnorm(b), thr = tol * tol * b2;
        cvec r = apply_A(x);
        for (size_t i = 0; i < r.size(); ++i) r[i] = b[i] - r[i];
        cvec r0 = r;
        double r0n2 = sqnorm(r0);
        const double restart_thr = r0n2 * 1e-32;
        cd rho = 1.0, alpha = 1.0, w = 1.0;
        cvec v(b.size(), cd(0.0)), p = v, y, z, s(b.size()), tt;
        iterations = 0;
        if (b2 == 0.0) {
            std::fill(x.begin(), x.end(), cd(0.0));
            return true;
        }
        while (sqnorm(r) > thr && iterations < maxit) {
            const cd rho_old = rho;
            rho = dot(r0, r);
            if (std::abs(rho) < restart_thr) {
                r = apply_A(x);
                for (size_t i = 0; i < r.size(); ++i) r[i] = b[i] - r[i];
                r0 = r;
                rho = r0n2 = sqnorm(r);
            }
            const cd beta = (rho / rho_old) * (alpha / w);
            for (size_t i = 0; i < p.size(); ++i) p[i] = r[i] + beta * (p[i] - w * v[i]);
            y = apply_M(p);
            v = apply_A(y);
            alpha = rho / dot(r0, v);
            for (size_t i = 0; i < s.size(); ++i) s[i] = r[i] - alpha * v[i];
            z = apply_M(s);
            tt = apply_A(z);
            const double tn2 = sqnorm(tt);
            w = tn2 > 0.0 ? dot(tt, s) / tn2 : cd(0.0);
            for (size_t i = 0; i < x.size(); ++i) x[i] += alpha * y[i] + w * z[i];
            for (size_t i = 0; i < r.size(); ++i) r[i] = s[i] - w * tt[i];
            ++iterations;
        }
        return sqnorm(r) <= thr;
    }

    // Eigen's BiCGSTAB (Eigen 3.4 IterativeLinearSolvers/BiCGSTAB.h): same recurrence,
    // restart when |rho| < eps^2 |r0|^2 with eps the double epsilon, and the iteration
    // counter reset on the first restart.
    template <class AF, class MF>
    static bool bicgstab_eigen(const AF &apply_A, const MF &apply_M, const cvec &b, cvec &x, double tol, int maxit,
                               int &iterations)
    {
        cvec r = apply_A(x);
        for (size_t i = 0; i < r.size(); ++i) r[i] = b[i] - r[i];
        cvec r0 = r;
        double r0n2 = sqnorm(r0);
        const double b2 = sqnorm(b);
        if (b2 == 0.0) {
            std::fill(x.begin(), x.end(), cd(0.0));
            iterations = 0;
            return true;
        }
        cd rho = 1.0, alpha = 1.0, w = 1.0;
        cvec v(b.size(), cd(0.0)), p = v, y, z, s(b.size()), tt;
        const double tol2 = tol * tol * b2;
        const double eps = std::numeric_limits<double>::epsilon(), eps2 = eps * eps;
        int i = 0, restarts = 0;
        while (sqnorm(r) > tol2 && i < maxit) {
            const cd rho_old = rho;
            rho = dot(r0, r);
            if (std::abs(rho) < eps2 * r0n2) {
                r = apply_A(x);
                for (size_t k = 0; k < r.size(); ++k) r[k] = b[k] - r[k];
                r0 = r;
                rho = r0n2 = sqnorm(r);
                if (restarts++ == 0) i = 0;
            }
            const cd beta = (rho / rho_old) * (alpha / w);
            for (size_t k = 0; k < p.size(); ++k) p[k] = r[k] + beta * (p[k] - w * v[k]);
            y = apply_M(p);
            v = apply_A(y);
            alpha = rho / dot(r0, v);
            for (size_t k = 0; k < s.size(); ++k) s[k] = r[k] - alpha * v[k];
            z = apply_M(s);
            tt = apply_A(z);
            const double tn2 = sqnorm(tt);
            w = tn2 > 0.0 ? dot(tt, s) / tn2 : cd(0.0);
            for (size_t k = 0; k < x.size(); ++k) x[k] += alpha * y[k] + w * z[k];
            for (size_t k = 0; k < r.size(); ++k) r[k] = s[k] - w * tt[k];
            ++i;
        }
        iterations = i;
        return true;
    }

    // src/CrankNicolsonModes_matrices.cpp:94-215 (radial preconditioner branch; the
    // ILUT fallback of :173-186 and :203-214 is not restated: a failure raises).
    void solve_CN(const cvec &rhs)
    {
        const double rhs_norm = std::sqrt(sqnorm(rhs));
        if (rhs_norm == 0.0) {
            std::fill(psi.begin(), psi.end(), cd(0.0));
            last_solver_residual = 0.0;
            last_solver_iterations = 0;
            return;
        }
        std::vector<const Sink *> sinks;
        if (sink_active)
            for (const Sink *s : {&sink1, &sink2})
                if (s->strength != 0.0 && s->v.size() == rhs.size() && sqnorm(s->v) > 0.0) sinks.push_back(s);
        auto apply_A = [&](const cvec &x) {
            cvec y;
            A.apply(x, y);
            for (const Sink *s : sinks) {
                const cd c = 0.25 * dt * s->strength * dot(s->v, x);
                for (size_t i = 0; i < y.size(); ++i) y[i] += c * s->v[i];
            }
            return y;
        };
        auto residual = [&](const cvec &cand) {
            if (!all_finite(cand)) return std::numeric_limits<double>::infinity();
            cvec ax = apply_A(cand);
            double s = 0;
            for (size_t i = 0; i < ax.size(); ++i) s += std::norm(ax[i] - rhs[i]);
            return std::sqrt(s) / rhs_norm;
        };
        cvec nrhs(rhs.size()), guess(rhs.size());
        for (size_t i = 0; i < rhs.size(); ++i) {
            nrhs[i] = rhs[i] / rhs_norm;
            guess[i] = psi[i] / rhs_norm;
        }
        if (!use_block_preconditioner) throw std::runtime_error("ILUT preconditioner is not part of the oracle");
        block.factorize(A, Nr);
        if (!block.ok) throw std::runtime_error("Radial preconditioner factorization failed (ILUT fallback not restated)");
        cvec x = guess;
        if (!sinks.empty()) {
            const int k = (int)sinks.size();
            std::vector<cvec> W(k);
            for (int a2 = 0; a2 < k; ++a2) W[a2] = block.solve(sinks[a2]->v);
            cd G[2][2] = {{0, 0}, {0, 0}};
            for (int a2 = 0; a2 < k; ++a2) {
                G[a2][a2] += 1.0 / (0.25 * dt * sinks[a2]->strength);
                for (int b2 = 0; b2 < k; ++b2) G[a2][b2] += dot(sinks[a2]->v, W[b2]);
            }
            cd Gi[2][2];
            if (k == 1) {
                Gi[0][0] = 1.0 / G[0][0];
            } else {
                const cd det = G[0][0] * G[1][1] - G[0][1] * G[1][0];
                Gi[0][0] = G[1][1] / det;
                Gi[0][1] = -G[0][1] / det;
                Gi[1][0] = -G[1][0] / det;
                Gi[1][1] = G[0][0] / det;
            }
            auto apply_M = [&](const cvec &xx) {
                cvec y = block.solve(xx);
                cd proj[2];
                for (int a2 = 0; a2 < k; ++a2) proj[a2] = dot(sinks[a2]->v, y);
                cd c[2] = {0, 0};
                for (int a2 = 0; a2 < k; ++a2)
                    for (int b2 = 0; b2 < k; ++b2) c[a2] += Gi[a2][b2] * proj[b2];
                for (size_t i = 0; i < y.size(); ++i) {
                    cd corr = 0.0;
                    for (int a2 = 0; a2 < k; ++a2) corr += W[a2][i] * c[a2];
                    y[i] -= corr;
                }
                return y;
            };
            bicgstab_ref(apply_A, apply_M, nrhs, x, tolerance, max_iterations, last_solver_iterations);
        } else {
            auto apply_M = [&](const cvec &xx) { return block.solve(xx); };
            bicgstab_eigen(apply_A, apply_M, nrhs, x, tolerance, max_iterations, last_solver_iterations);
        }
        for (cd &v : x) v *= rhs_norm;
        last_solver_residual = residual(x);
        if (!(last_solver_residual <= accept_residual))
            throw std::runtime_error("Crank-Nicolson solve failed the relative residual check");
        psi.swap(x);
    }

    // ------------------------------------------------------------ orbit (_evolution.cpp)

    void update_time_dependent_increment(double orbit_dt)
    {
        cvec mid(psi.size());
        for (size_t i = 0; i < mid.size(); ++i) {
            mid[i] = psi[i] + psi_last[i];
            mid[i] *= 0.5;
        }
        double Md1 = 0.0, Md2 = 0.0;
        if (absorption) {
            Md1 = absorption_rate(sink1, mid);
            Md2 = absorption_rate(sink2, mid);
        }
        double ramp = 1.0;
        if (t_i < ramp_end_time()) ramp = 0.0;
        else if (t_i < ramp_end_time() + initial_period) {
            const double x = (t_i - ramp_end_time()) / initial_period;
            ramp = 3.0 * x * x - 2.0 * x * x * x;
        }
        const double dR_gw = -(64.0 / 5.0) * M1 * M2 * (M1 + M2) / std::pow(R, 3);
        const double dR_cloud = -2.0 * R * R * p_bin / (M1 * M2);
        const double dR = (dR_gw + dR_cloud) * ramp;
        R += dR * orbit_dt;
        M1 += Md1 * orbit_dt;
        M2 += Md2 * orbit_dt;
        q = M2 / M1;
        const double Mt = M1 + M2;
        R1 = M2 / Mt * R;
        R2 = M1 / Mt * R;
        Omega = std::sqrt(Mt / std::pow(R, 3));
        P = 2.0 * M_PI / Omega;
        if (ramp_factor == 1.0) dt = P / steps_per_period;
    }

    // ------------------------------------------------------------ diagnostics (_extraction.cpp)

    double restricted_expectation(const cvec &ps, const Csr &M, int cut) const
    {
        cvec ap;
        M.apply(ps, ap);
        cd res = 0.0;
        for (int j = 0; j < n_modes; ++j)
            for (int i = 0; i <= cut; ++i) {
                const size_t k = (size_t)j * Nr + i;
                res += std::conj(ps[k]) * ap[k];
            }
        return res.real() * dr;
    }

    // ------------------------------------------------------------ run / step

    void set_extraction_radius(double rex, int n_steps)
    {
        r_ex = rex;
        idx_ex = (int)std::floor(r_ex / dr);
        if (n_steps < 1 || idx_ex < 1 || idx_ex >= Nr - 1)
            throw std::invalid_argument("Require at least one time sample and an interior extraction radius");
    }

    // The computational part of run() (src/CrankNicolsonModes.cpp:236-259): no files.
    void prepare_run(int n_steps, double rex)
    {
        set_extraction_radius(rex, n_steps);
        t_i = 0.0;
        t.assign(n_steps, 0.0);
        build_time_dependent_perturbation(t_i);
    }

    // Diagnostic record of one step, in the order step() writes them
    // (src/CrankNicolsonModes.cpp:209-226).
    struct Diag {
        double R, theta, Omega, M1, q, t, energy, p_bin, p_bin_inst, dV_bin_dt;
        std::vector<double> energy_flux, flux, norms, energies;
    };

    // src/CrankNicolsonModes.cpp:145-234 without the text writes.
    Diag step(int step_id)
    {
        psi_last = psi;
        const double step_start = t_i;
        t_i += dt;
        theta += (counter ? -1.0 : 1.0) * Omega * dt;
        phase += Omega * dt;
        if ((int)t.size() <= step_id) t.resize(step_id + 1, 0.0);
        t[step_id] = t_i;
        build_time_dependent_perturbation(t_i);
        update_CN_values();
        cvec rhs;
        B.apply(psi, rhs);
        if (sink_active) {
            const cvec g = apply_sink(psi);
            for (size_t i = 0; i < rhs.size(); ++i) rhs[i] -= (0.25 * dt) * g[i];
        }
        solve_CN(rhs);
        if (mask)
            for (size_t i = 0; i < psi.size(); ++i) psi[i] *= damping_mask[i];
        const cvec dpsi_dt = schrodinger_rhs(psi);
        if (!isolated_black_hole && evolve_orbit && t_i > ramp_end_time()) {
            const double orbit_dt = t_i - std::max(step_start, ramp_end_time());
            update_time_dependent_increment(orbit_dt);
        }
        Diag d;
        d.flux.resize(n_modes);
        d.energy_flux.resize(n_modes);
        for (int j = 0; j < n_modes; ++j) {
            const size_t c = (size_t)j * Nr + idx_ex;
            const cd dU = (psi[c + 1] - psi[c - 1]) / (2.0 * dr) - psi[c] / r[idx_ex];
            d.flux[j] = (std::conj(psi[c]) * dU).imag();
            d.energy_flux[j] = (std::conj(dpsi_dt[c]) * dU).real() / mu;
        }
        d.energy = restricted_expectation(psi, H, idx_ex);
        d.p_bin_inst = restricted_expectation(psi, dVdt, idx_ex);
        p_bin = isolated_black_hole ? 0.0 : power_average.update(t_i, phase, d.p_bin_inst);
        {
            cvec vp;
            V.apply(psi, vp);
            cd res = 0.0;
            for (int j = 0; j < n_modes; ++j)
                for (int i = 0; i <= idx_ex; ++i) {
                    const size_t k = (size_t)j * Nr + i;
                    res += std::conj(dpsi_dt[k]) * vp[k];
                }
            d.dV_bin_dt = res.real() * dr;
        }
        d.norms.resize(n_modes);
        d.energies.resize(n_modes);
        cvec hp;
        H.apply(psi, hp);
        for (int j = 0; j < n_modes; ++j) {
            double nsum = 0.0;
            cd e = 0.0;
            for (int i = 0; i < idx_ex; ++i) {
                const size_t k = (size_t)j * Nr + i;
                nsum += std::norm(psi[k]);
                e += std::conj(psi[k]) * hp[k];
            }
            d.norms[j] = nsum * dr;
            d.energies[j] = e.real() * dr;
        }
        d.R = R;
        d.theta = theta;
        d.Omega = Omega;
        d.M1 = M1;
        d.q = q;
        d.t = t_i;
        d.p_bin = p_bin;
        return d;
    }

    bool evolve_should_stop() const { return !isolated_black_hole && evolve_orbit && R <= 6.0; }
};

thread_local std::string g_error;

template <class F>
int guarded(F &&f)
{
    try {
        f();
        return 0;
    } catch (const std::invalid_argument &e) {
        g_error = e.what();
        return 1;
    } catch (const std::logic_error &e) {
        g_error = e.what();
        return 2;
    } catch (const std::runtime_error &e) {
        g_error = e.what();
        return 3;
    } catch (const std::exception &e) {
        g_error = e.what();
        return 4;
    }
}

cvec from_interleaved(const double *x, int64_t n)
{
    cvec v(n);
    for (int64_t i = 0; i < n; ++i) v[i] = cd(x[2 * i], x[2 * i + 1]);
    return v;
}

void to_interleaved(const cvec &v, double *y)
{
    for (size_t i = 0; i < v.size(); ++i) {
        y[2 * i] = v[i].real();
        y[2 * i + 1] = v[i].imag();
    }
}

double *scalar_slot(Oracle *o, const std::string &name)
{
    if (name == "R") return &o->R;
    if (name == "R1") return &o->R1;
    if (name == "R2") return &o->R2;
    if (name == "M1") return &o->M1;
    if (name == "M2") return &o->M2;
    if (name == "q") return &o->q;
    if (name == "theta") return &o->theta;
    if (name == "phase") return &o->phase;
    if (name == "Omega") return &o->Omega;
    if (name == "Omega_0") return &o->Omega_0;
    if (name == "P") return &o->P;
    if (name == "dt") return &o->dt;
    if (name == "dr") return &o->dr;
    if (name == "L") return &o->L;
    if (name == "mu") return &o->mu;
    if (name == "M_c") return &o->M_c;
    if (name == "epsilon") return &o->epsilon;
    if (name == "t_i") return &o->t_i;
    if (name == "p_bin") return &o->p_bin;
    if (name == "steps_per_period") return &o->steps_per_period;
    if (name == "last_solver_residual") return &o->last_solver_residual;
    if (name == "tolerance") return &o->tolerance;
    if (name == "accept_residual") return &o->accept_residual;
    if (name == "initial_period") return &o->initial_period;
    if (name == "ramp_factor") return &o->ramp_factor;
    return nullptr;
}

}  // namespace

// ---------------------------------------------------------------- C interface (ctypes)

extern "C" {

const char *orc_last_error() { return g_error.c_str(); }

void *orc_create(int Nr, double L, double dt, double eps, int lmax, double mu, double Mc, double q, double a,
                 double R, int counter, int absorption, int save_every, double ramp_periods, double smear)
{
    Oracle *o = nullptr;
    const int rc = guarded([&] {
        o = new Oracle(Nr, L, dt, eps, lmax, mu, Mc, q, a, R, counter != 0, absorption != 0, save_every,
                       ramp_periods, smear);
    });
    return rc == 0 ? o : nullptr;
}

void orc_destroy(void *h) { delete static_cast<Oracle *>(h); }

int orc_set_threads(int n)
{
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
}

int orc_n_modes(void *h) { return static_cast<Oracle *>(h)->n_modes; }

void orc_modes(void *h, int *l, int *m)
{
    const Oracle *o = static_cast<Oracle *>(h);
    for (int j = 0; j < o->n_modes; ++j) {
        l[j] = o->modes[j].l;
        m[j] = o->modes[j].m;
    }
}

void orc_grid(void *h, double *r)
{
    const Oracle *o = static_cast<Oracle *>(h);
    std::copy(o->r.begin(), o->r.end(), r);
}

int orc_set_initial_state_full(void *h, const double *psi, int64_t n)
{
    return guarded([&] { static_cast<Oracle *>(h)->set_initial_state_full(from_interleaved(psi, n)); });
}

int orc_set_psi(void *h, const double *psi, int64_t n)
{
    return guarded([&] {
        Oracle *o = static_cast<Oracle *>(h);
        if (n != o->size()) throw std::invalid_argument("state size");
        o->psi = from_interleaved(psi, n);
    });
}

void orc_get_psi(void *h, double *out) { to_interleaved(static_cast<Oracle *>(h)->psi, out); }

int orc_initialize(void *h) { return guarded([&] { static_cast<Oracle *>(h)->initialize(); }); }

int orc_configure_isolated_black_hole(void *h, double x)
{
    return guarded([&] { static_cast<Oracle *>(h)->configure_isolated_black_hole(x); });
}

int orc_build_damping_mask(void *h, double f, double W, int n)
{
    return guarded([&] { static_cast<Oracle *>(h)->build_damping_mask(f, W, n); });
}

int orc_build_cap(void *h, double f, double W, int n)
{
    return guarded([&] { static_cast<Oracle *>(h)->build_cap(f, W, n); });
}

int orc_set_power_average_orbits(void *h, double n)
{
    return guarded([&] { static_cast<Oracle *>(h)->set_power_average_orbits(n); });
}

int orc_set_flag(void *h, const char *name, int value)
{
    return guarded([&] {
        Oracle *o = static_cast<Oracle *>(h);
        const std::string s(name);
        if (s == "evolve_orbit") o->evolve_orbit = value != 0;
        else if (s == "ramp_secondary_potential") o->ramp_secondary_potential = value != 0;
        else if (s == "use_block_preconditioner") o->use_block_preconditioner = value != 0;
        else if (s == "max_iterations") o->max_iterations = value;
        else throw std::invalid_argument("unknown flag " + s);
    });
}

int orc_get_int(void *h, const char *name)
{
    const Oracle *o = static_cast<Oracle *>(h);
    const std::string s(name);
    if (s == "last_solver_iterations") return o->last_solver_iterations;
    if (s == "idx_ex") return o->idx_ex;
    if (s == "sink_active") return o->sink_active ? 1 : 0;
    if (s == "n_pairs") return (int)o->mode_pairs.size();
    if (s == "mode00") return o->mode00;
    if (s == "evolve_orbit") return o->evolve_orbit ? 1 : 0;
    if (s == "should_stop") return o->evolve_should_stop() ? 1 : 0;
    return -1;
}

int orc_get_scalar(void *h, const char *name, double *out)
{
    return guarded([&] {
        double *p = scalar_slot(static_cast<Oracle *>(h), name);
        if (!p) throw std::invalid_argument(std::string("unknown scalar ") + name);
        *out = *p;
    });
}

int orc_set_scalar(void *h, const char *name, double value)
{
    return guarded([&] {
        double *p = scalar_slot(static_cast<Oracle *>(h), name);
        if (!p) throw std::invalid_argument(std::string("unknown scalar ") + name);
        *p = value;
    });
}

int orc_prepare_run(void *h, int n_steps, double r_ex)
{
    return guarded([&] { static_cast<Oracle *>(h)->prepare_run(n_steps, r_ex); });
}

int orc_refresh(void *h, double time)
{
    return guarded([&] {
        Oracle *o = static_cast<Oracle *>(h);
        o->build_time_dependent_perturbation(time);
        o->update_CN_values();
    });
}

// diag layout: [R, theta, Omega, M1, q, t, energy, p_bin, p_bin_inst, dV_bin_dt,
//               residual, iterations, energy_flux[n], flux[n], norms[n], energies[n]]
int orc_step(void *h, int step_id, double *diag)
{
    return guarded([&] {
        Oracle *o = static_cast<Oracle *>(h);
        const Oracle::Diag d = o->step(step_id);
        const double head[12] = {d.R,      d.theta,  d.Omega,      d.M1,        d.q,
                                 d.t,      d.energy, d.p_bin,      d.p_bin_inst, d.dV_bin_dt,
                                 o->last_solver_residual, (double)o->last_solver_iterations};
        std::copy(head, head + 12, diag);
        const int n = o->n_modes;
        std::copy(d.energy_flux.begin(), d.energy_flux.end(), diag + 12);
        std::copy(d.flux.begin(), d.flux.end(), diag + 12 + n);
        std::copy(d.norms.begin(), d.norms.end(), diag + 12 + 2 * n);
        std::copy(d.energies.begin(), d.energies.end(), diag + 12 + 3 * n);
    });
}

// which: 0 H, 1 H0, 2 V, 3 V1, 4 V2, 5 dVdt, 6 A (sparse part), 7 B (sparse part),
//        8 apply_sink, 9 schrodinger_rhs, 10 A_full = A + dt/4 Gamma, 11 CAP
int orc_apply(void *h, int which, const double *x, double *y)
{
    return guarded([&] {
        Oracle *o = static_cast<Oracle *>(h);
        const cvec xv = from_interleaved(x, o->size());
        cvec yv;
        switch (which) {
        case 0: o->H.apply(xv, yv); break;
        case 1: o->H0.apply(xv, yv); break;
        case 2: o->V.apply(xv, yv); break;
        case 3: o->V1.apply(xv, yv); break;
        case 4: o->V2.apply(xv, yv); break;
        case 5: o->dVdt.apply(xv, yv); break;
        case 6: o->A.apply(xv, yv); break;
        case 7: o->B.apply(xv, yv); break;
        case 8: yv = o->apply_sink(xv); break;
        case 9: yv = o->schrodinger_rhs(xv); break;
        case 10: {
            o->A.apply(xv, yv);
            if (o->sink_active) {
                const cvec g = o->apply_sink(xv);
                for (size_t i = 0; i < yv.size(); ++i) yv[i] += (0.25 * o->dt) * g[i];
            }
            break;
        }
        case 11:
            if (o->cap) o->CAP.apply(xv, yv);
            else yv.assign(xv.size(), cd(0.0));
            break;
        default: throw std::invalid_argument("unknown operator");
        }
        to_interleaved(yv, y);
    });
}

double orc_sink_strength(void *h, int body) { return static_cast<Oracle *>(h)->sink_strength(body); }

void orc_sink_vector(void *h, int body, double *out)
{
    const Oracle *o = static_cast<Oracle *>(h);
    const Sink &s = body == 1 ? o->sink1 : o->sink2;
    if ((int64_t)s.v.size() == o->size()) to_interleaved(s.v, out);
    else std::fill(out, out + 2 * o->size(), 0.0);
}

// Dense export of one sparse operator (small grids only), for matrix-level tests.
int orc_dense(void *h, int which, double *out)
{
    return guarded([&] {
        Oracle *o = static_cast<Oracle *>(h);
        const Csr *m = nullptr;
        switch (which) {
        case 0: m = &o->H; break;
        case 1: m = &o->H0; break;
        case 2: m = &o->V; break;
        case 3: m = &o->V1; break;
        case 4: m = &o->V2; break;
        case 5: m = &o->dVdt; break;
        case 6: m = &o->A; break;
        case 7: m = &o->B; break;
        case 11: m = &o->CAP; break;
        default: throw std::invalid_argument("unknown operator");
        }
        const int64_t n = o->size();
        std::fill(out, out + 2 * n * n, 0.0);
        if (m->n == 0) return;
        for (int64_t r = 0; r < n; ++r)
            for (int64_t s = m->outer[r]; s < m->outer[r + 1]; ++s) {
                out[2 * (r * n + m->inner[s])] = m->val[s].real();
                out[2 * (r * n + m->inner[s]) + 1] = m->val[s].imag();
            }
    });
}

// Coupling cache export: per term (row, col, m_star, l_star, angular).
int orc_coupling_terms(void *h, int *rows, int *cols, int *lstar, double *angular)
{
    const Oracle *o = static_cast<Oracle *>(h);
    int n = 0;
    for (const auto &p : o->mode_pairs)
        for (const auto &t : p.terms) {
            if (rows) {
                rows[n] = p.row_mode;
                cols[n] = p.col_mode;
                lstar[n] = t.l_star;
                angular[n] = t.angular.real();
            }
            ++n;
        }
    return n;
}

void orc_multipoles(void *h, int body, double *out)
{
    const Oracle *o = static_cast<Oracle *>(h);
    const Profile &p = body == 1 ? o->profile1 : o->profile2;
    std::copy(p.multipoles.begin(), p.multipoles.end(), out);
}

double orc_wigner3j(int a, int b, int c, int d, int e, int f) { return wigner3j(a, b, c, d, e, f); }
double orc_sph_plm_equator(int l, int m) { return sph_plm_equator(l, m); }
void orc_gauss_legendre(int n, double a, double b, double *x, double *w)
{
    std::vector<double> xv, wv;
    gauss_legendre(n, a, b, xv, wv);
    std::copy(xv.begin(), xv.end(), x);
    std::copy(wv.begin(), wv.end(), w);
}

// displaced_100_state (src/DisplacedAtom.cpp:12-76): the mode projection of a
// hydrogenic 1s state centred at x_bh on the x axis.  For every interior node the
// Legendre moments of the displaced density about the origin, by Gauss-Legendre
// quadrature in the body-centred distance s (tail beyond 40 a0 dropped), times r and
// Y*_lm(pi/2, phi_BH).  out: interleaved complex, n_modes x Nr.
int orc_displaced_100_state(const double *r, int Nr, const int *l, const int *m, int n_modes, double mu, double x_bh,
                            double *out)
{
    return guarded([&] {
        if (!std::isfinite(mu) || mu <= 0 || !std::isfinite(x_bh) || Nr < 3 || n_modes < 1)
            throw std::invalid_argument("Invalid displaced 100 state parameters");
        for (int i = 0; i < Nr; ++i)
            if (!std::isfinite(r[i]) || r[0] < 0) throw std::invalid_argument("Radial coordinates must be finite and nonnegative");
        for (int i = 1; i < Nr; ++i)
            if (r[i] <= r[i - 1]) throw std::invalid_argument("Radial coordinates must increase");
        int lmax = 0;
        for (int j = 0; j < n_modes; ++j) {
            if (l[j] < 0 || std::abs(m[j]) > l[j]) throw std::invalid_argument("Invalid spherical harmonic mode");
            lmax = std::max(lmax, l[j]);
        }
        const double a0 = 1.0 / (mu * mu), distance = std::abs(x_bh);
        const double amplitude = 1.0 / std::sqrt(M_PI * a0 * a0 * a0);
        const int nq = std::max(128, 2 * lmax + 32);
        std::vector<double> nodes, weights;
        gauss_legendre(nq, 0.0, 1.0, nodes, weights);
        std::vector<double> direction(n_modes);
        for (int j = 0; j < n_modes; ++j) {
            double y = sph_plm_equator(l[j], std::abs(m[j]));
            if (m[j] < 0 && (std::abs(m[j]) & 1)) y = -y;
            if (x_bh < 0 && (std::abs(m[j]) & 1)) y = -y;
            direction[j] = y;
        }
        std::fill(out, out + 2 * (int64_t)Nr * n_modes, 0.0);
#pragma omp parallel for schedule(static)
        for (int i = 1; i < Nr - 1; ++i) {
            std::vector<double> mom(lmax + 1, 0.0);
            if (distance == 0.0) {
                mom[0] = 4 * M_PI * amplitude * std::exp(-r[i] / a0);
            } else {
                const double low = std::abs(r[i] - distance);
                const double high = std::min(r[i] + distance, low + 40 * a0);
                for (int k = 0; k < nq; ++k) {
                    const double sv = low + (high - low) * nodes[k];
                    const double u =
                        std::clamp((r[i] * r[i] + distance * distance - sv * sv) / (2 * r[i] * distance), -1.0, 1.0);
                    const double wgt =
                        2 * M_PI * (high - low) * weights[k] * sv / (r[i] * distance) * amplitude * std::exp(-sv / a0);
                    double prev = 1.0, cur = u;
                    mom[0] += wgt;
                    if (lmax > 0) mom[1] += wgt * cur;
                    for (int q = 2; q <= lmax; ++q) {
                        const double next = ((2 * q - 1) * u * cur - (q - 1) * prev) / q;
                        mom[q] += wgt * next;
                        prev = cur;
                        cur = next;
                    }
                }
            }
            for (int j = 0; j < n_modes; ++j) out[2 * ((int64_t)j * Nr + i)] = r[i] * mom[l[j]] * direction[j];
        }
    });
}

}  // extern "C"

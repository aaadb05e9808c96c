// cnm_initial.cu -- initial states of the sweeps on the device: the mode projection of a
// hydrogenic (n, l, m) state centred off the origin on the x axis,
//     U_j(r) = r * int conj(Y_j(Omega)) psi_nlm(r Omega - x_c e_x) dOmega,
// by Gauss-Legendre quadrature in cos(theta) and the trapezoidal rule in phi (the state the
// reference's initial_states/get_initial_state_COM_fast.py writes to a MODESBIN file, there
// through translation matrices).  The angular integral is a product of an (n_modes x n_ang)
// table of conj(Y_j) times the weights with the state on the angular grid, node by node.
#include "../../include/cnm_gpu.h"
#include "cnm_coupling.h"
#include "cnm_device.cuh"
#include "cnm_initial.h"

#include <cuda_runtime.h>

#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

namespace cnm {

namespace {

constexpr int HP_THREADS = 256, HP_TILE = 32, HP_CH = 64, HP_MAXK = 20;  // modes per thread: up to 160 modes

struct HydroArgs {
    double xc;      // centre of the state on the x axis
    double na0;     // n a0 (a0 = 1 / (mu^2 M1))
    double rnorm;   // normalisation of R_nl
    double ynorm;   // N_l|m| (-1)^|m| (2|m| - 1)!! of Y_l|m|
    int n, l, m;
};

// R_nl(d) Y_lm(p / d) at the point p, with Y_l|m| = ynorm Q(cos t) ((p_x + i p_y) / d)^|m|
// (Q the polynomial part of P_l^|m|) and Y_l,-|m| = (-1)^|m| conj(Y_l|m|).
__device__ __host__ inline double2 hydro_psi(double px, double py, double pz, const HydroArgs &h)
{
    const double d = sqrt(px * px + py * py + pz * pz);
    const int am = h.m < 0 ? -h.m : h.m;
    if (d == 0.0) {
        if (h.l > 0) return make_double2(0.0, 0.0);
        return make_double2(h.rnorm * h.ynorm * h.n, 0.0);  // L^1_{n-1}(0) = n
    }
    // radial: rnorm e^{-rho/2} rho^l L^{2l+1}_{n-l-1}(rho), rho = 2 d / (n a0)
    const double rho = 2.0 * d / h.na0;
    const int kmax = h.n - h.l - 1;
    const double alpha = 2.0 * h.l + 1.0;
    double lag0 = 1.0, lag1 = 1.0 + alpha - rho;
    double lag = kmax == 0 ? lag0 : lag1;
    for (int k = 1; k < kmax; ++k) {
        const double lag2 = ((2.0 * k + 1.0 + alpha - rho) * lag1 - (k + alpha) * lag0) / (k + 1.0);
        lag0 = lag1;
        lag1 = lag2;
        lag = lag2;
    }
    double rl = 1.0;
    for (int q = 0; q < h.l; ++q) rl *= rho;
    const double rad = h.rnorm * exp(-0.5 * rho) * rl * lag;
    // angular: Q_l^|m|(x) by the three-term recurrence from Q_|m|^|m| = 1
    const double x = pz / d;
    double q0 = 1.0, q1 = x * (2.0 * am + 1.0);
    double qv = h.l == am ? q0 : q1;
    for (int ll = am + 2; ll <= h.l; ++ll) {
        const double q2 = ((2.0 * ll - 1.0) * x * q1 - (ll + am - 1.0) * q0) / (ll - am);
        q0 = q1;
        q1 = q2;
        qv = q2;
    }
    // ((p_x + i p_y) / d)^|m|
    double er = 1.0, ei = 0.0;
    const double ur = px / d, ui = py / d;
    for (int q = 0; q < am; ++q) {
        const double t = er * ur - ei * ui;
        ei = er * ui + ei * ur;
        er = t;
    }
    double yr = h.ynorm * qv * er, yi = h.ynorm * qv * ei;
    if (h.m < 0) {
        const double s = (am & 1) ? -1.0 : 1.0;
        yr *= s;
        yi *= -s;
    }
    return make_double2(rad * yr, rad * yi);
}

// CTA = HP_TILE radial nodes; the angular points in chunks of HP_CH: the state at
// (node, point) into shared memory, then every thread accumulates its node's projections
// onto modes warp, warp + 8, ... (the table entries are warp-uniform loads).
__global__ void __launch_bounds__(HP_THREADS) k_hydrogenic_proj(const double *r, int Nr, int n_modes, int n_ang,
                                                                const double *ang, const double2 *yw, HydroArgs h,
                                                                double2 *out)
{
    __shared__ double2 ps[HP_TILE][HP_CH + 1];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int i0 = blockIdx.x * HP_TILE;
    double2 acc[HP_MAXK];
#pragma unroll
    for (int k = 0; k < HP_MAXK; ++k) acc[k] = make_double2(0.0, 0.0);
    for (int a0 = 0; a0 < n_ang; a0 += HP_CH) {
        __syncthreads();
        for (int e = tid; e < HP_TILE * HP_CH; e += HP_THREADS) {
            const int node = e / HP_CH, a = e % HP_CH;
            const int i = i0 + node, ag = a0 + a;
            double2 v = make_double2(0.0, 0.0);
            if (i < Nr && ag < n_ang) {
                const double ri = r[i];
                v = hydro_psi(ri * ang[3 * ag] - h.xc, ri * ang[3 * ag + 1], ri * ang[3 * ag + 2], h);
            }
            ps[node][a] = v;
        }
        __syncthreads();
        const int na = min(HP_CH, n_ang - a0);
        for (int a = 0; a < na; ++a) {
            const double2 pv = ps[lane][a];
#pragma unroll
            for (int k = 0; k < HP_MAXK; ++k) {
                const int j = warp + 8 * k;
                if (j < n_modes) {
                    const double2 y = yw[(int64_t)j * n_ang + a0 + a];
                    acc[k].x = fma(y.x, pv.x, fma(-y.y, pv.y, acc[k].x));
                    acc[k].y = fma(y.x, pv.y, fma(y.y, pv.x, acc[k].y));
                }
            }
        }
    }
    const int i = i0 + lane;
    if (i >= Nr) return;
    const double ri = (i >= 1 && i <= Nr - 2) ? r[i] : 0.0;
#pragma unroll
    for (int k = 0; k < HP_MAXK; ++k) {
        const int j = warp + 8 * k;
        if (j < n_modes) out[(int64_t)j * Nr + i] = make_double2(ri * acc[k].x, ri * acc[k].y);
    }
}

double factorial(int n)
{
    double f = 1.0;
    for (int k = 2; k <= n; ++k) f *= k;
    return f;
}

// N_l|m| (-1)^|m| (2|m| - 1)!!, the constant of Y_l|m| = c Q(cos t) (sin t e^{i phi})^|m|
double ylm_const(int l, int m)
{
    const int am = std::abs(m);
    double dfact = 1.0;
    for (int k = 2 * am - 1; k > 1; k -= 2) dfact *= k;
    const double nlm = std::sqrt((2.0 * l + 1.0) / (4.0 * M_PI) * factorial(l - am) / factorial(l + am));
    return nlm * ((am & 1) ? -1.0 : 1.0) * dfact;
}

// Y_lm(theta, phi) with the Condon-Shortley phase (host; the same recurrence as the device)
void ylm(int l, int m, double ct, double st, double phi, double &yr, double &yi)
{
    const int am = std::abs(m);
    double q0 = 1.0, q1 = ct * (2.0 * am + 1.0);
    double qv = l == am ? q0 : q1;
    for (int ll = am + 2; ll <= l; ++ll) {
        const double q2 = ((2.0 * ll - 1.0) * ct * q1 - (ll + am - 1.0) * q0) / (ll - am);
        q0 = q1;
        q1 = q2;
        qv = q2;
    }
    const double s = std::pow(st, am) * ylm_const(l, am) * qv;
    yr = s * std::cos(am * phi);
    yi = s * std::sin(am * phi);
    if (m < 0) {
        const double sg = (am & 1) ? -1.0 : 1.0;
        yr *= sg;
        yi *= -sg;
    }
}

// Device buffer owned for the duration of one call.
template <class T>
struct Scratch {
    T *p = nullptr;
    cudaError_t alloc(size_t n) { return cudaMalloc(&p, n * sizeof(T)); }
    ~Scratch()
    {
        if (p) cudaFree(p);
    }
};

}  // namespace

int hydrogenic_state(const double *r, int Nr, const int *l, const int *m, int n_modes, double mu, double M1,
                     double x_center, int n, int la, int ma, int n_theta, int n_phi, double *state, std::string &err)
{
    if (!r || !l || !m || !state || Nr < 3 || n_modes < 1 || n_modes > 8 * HP_MAXK || !std::isfinite(mu) || mu <= 0 ||
        !std::isfinite(M1) || M1 <= 0 || !std::isfinite(x_center) || n < 1 || la < 0 || la >= n || std::abs(ma) > la ||
        n_theta < 2 || n_phi < 1) {
        err = "Invalid hydrogenic state parameters";
        return CNM_EINVAL;
    }
    for (int i = 1; i < Nr; ++i)
        if (!(r[i] > r[i - 1]) || r[0] < 0) {
            err = "Radial coordinates must increase from r >= 0";
            return CNM_EINVAL;
        }
    for (int j = 0; j < n_modes; ++j)
        if (l[j] < 0 || std::abs(m[j]) > l[j]) {
            err = "Invalid spherical harmonic mode";
            return CNM_EINVAL;
        }
    // angular grid: Gauss-Legendre in cos(theta), uniform in phi
    std::vector<double> gx, gw;
    gauss_legendre01(n_theta, gx, gw);
    const int n_ang = n_theta * n_phi;
    std::vector<double> ang((size_t)3 * n_ang);
    std::vector<double2> yw((size_t)n_modes * n_ang);
    for (int t = 0; t < n_theta; ++t) {
        const double ct = 2.0 * gx[t] - 1.0, st = std::sqrt(std::max(0.0, 1.0 - ct * ct));
        const double wt = 2.0 * gw[t] * (2.0 * M_PI / n_phi);
        for (int p = 0; p < n_phi; ++p) {
            const double phi = 2.0 * M_PI * p / n_phi;
            const int a = t * n_phi + p;
            ang[3 * a] = st * std::cos(phi);
            ang[3 * a + 1] = st * std::sin(phi);
            ang[3 * a + 2] = ct;
            for (int j = 0; j < n_modes; ++j) {
                double yr, yi;
                ylm(l[j], m[j], ct, st, phi, yr, yi);
                yw[(size_t)j * n_ang + a] = make_double2(wt * yr, -wt * yi);  // conj(Y_j) w
            }
        }
    }
    HydroArgs h;
    h.xc = x_center;
    const double a0 = 1.0 / (mu * mu * M1);
    h.na0 = n * a0;
    h.rnorm = std::sqrt(std::pow(2.0 / (n * a0), 3) * factorial(n - la - 1) / (2.0 * n * factorial(n + la)));
    h.ynorm = ylm_const(la, ma);
    h.n = n;
    h.l = la;
    h.m = ma;
    Scratch<double> d_r, d_ang;
    Scratch<double2> d_yw, d_out;
    cudaError_t e = d_r.alloc(Nr);
    if (e == cudaSuccess) e = d_ang.alloc(ang.size());
    if (e == cudaSuccess) e = d_yw.alloc(yw.size());
    if (e == cudaSuccess) e = d_out.alloc((size_t)n_modes * Nr);
    if (e == cudaSuccess) e = cudaMemcpy(d_r.p, r, Nr * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_ang.p, ang.data(), ang.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_yw.p, yw.data(), yw.size() * sizeof(double2), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_hydrogenic_proj<<<(Nr + HP_TILE - 1) / HP_TILE, HP_THREADS>>>(d_r.p, Nr, n_modes, n_ang, d_ang.p, d_yw.p, h,
                                                                        d_out.p);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(state, d_out.p, (size_t)n_modes * Nr * sizeof(double2), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        err = std::string("hydrogenic state: ") + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? CNM_ENOMEM : CNM_ECUDA;
    }
    // normalised to sum |U|^2 dr = 1 on the (uniform) grid
    double s2 = 0.0;
    for (int64_t q = 0; q < 2 * (int64_t)n_modes * Nr; ++q) s2 += state[q] * state[q];
    if (!(s2 > 0.0)) {
        err = "The state has no weight on the grid";
        return CNM_EINVAL;
    }
    const double sc = 1.0 / std::sqrt(s2 * (r[1] - r[0]));
    for (int64_t q = 0; q < 2 * (int64_t)n_modes * Nr; ++q) state[q] *= sc;
    return CNM_OK;
}

}  // namespace cnm

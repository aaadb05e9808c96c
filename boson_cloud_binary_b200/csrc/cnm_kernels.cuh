// cnm_kernels.cuh -- kernel declarations and launch constants.
#pragma once

#include "cnm_common.cuh"

namespace cnm {

constexpr int APPLY_THREADS = 256;  // 8 warps share the rows of a tile
constexpr int SCAN_THREADS = 256;   // preconditioner scan CTAs (per-thread chunk kernels)
constexpr int SCAN2_THREADS = 512;  // staged preconditioner scan CTAs
constexpr int PCL_THREADS = 256;    // cluster preconditioner scan CTAs
constexpr int VEC_THREADS = 256;    // streaming vector kernels

// Device-resident scalars of one BiCGSTAB solve (src/CrankNicolsonModes_matrices.cpp:47-91)
// and of its Woodbury correction (:133-157).
struct Krylov {
    double2 rho, rho_old, alpha, omega, beta;
    double2 r0r;          // r0 . r of the current residual
    double r2;            // |r|^2
    double thr;           // tol^2 |b|^2
    double restart_thr;   // 1e-32 |r0|^2 (sink path) or eps^2 |r0|^2 (Eigen path)
    int iterations, max_iterations, done, restart;
    int n_sinks;
    double2 Gi[2][2];     // G^{-1}
    double2 vW[2][2];     // v_a . W_b
    double2 wc[2][2];     // c = G^{-1} proj for the two preconditioner calls of an iteration
    double2 sdots[2][2];  // sink projections of the corrected vectors y and z
    double tol;           // relative tolerance
    int eigen_path;       // 1: Eigen's restart rule (no sinks), 0: the sink path's
    int zero_rhs;
    double rhs_norm;
    int pturn;            // which of the two search-direction buffers the next PI_P solve writes
    int accepted;         // KS_RESID: the candidate passed the residual (and pivot) check
    double residual;      // KS_RESID: | |rhs| A x - rhs | / |rhs|
    double accept;        // acceptance bound of the true relative residual
    const int *status;    // pivot-failure word of the factorisation (device)
};

// Right-hand side of a preconditioner solve: b itself, or a BiCGSTAB combination
// formed while staging (PI_P: p = r + beta (p_old - omega v); PI_S: s = r - alpha v),
// which is also written to `out`.
enum PrecondMode : int { PI_PLAIN = 0, PI_P = 1, PI_S = 2 };
struct PrecondInput {
    int mode;
    const struct Krylov *kr;
    const double2 *r, *p_old, *v;
    double2 *out;
    // PI_P with p_alt set: the search directions alternate between p_old and p_alt by
    // kr->pturn (out = pturn ? p_alt : p_old, the previous direction the other one);
    // `first`: no previous direction (p = r)
    double2 *p_alt;
    int first;
    int gate;  // GateMode of the launch (GATE_ITER for the iteration's solves)
    int *fault = nullptr;  // set (bit 1) when a staging copy did not complete in time
};

// Launches queued ahead of the host's convergence test skip themselves on the device:
// GATE_ITER while the solve is done or must restart, GATE_DONE until it is done,
// GATE_ACCEPTED until its candidate passed the residual check.
enum GateMode : int { GATE_NONE = 0, GATE_ITER = 1, GATE_DONE = 2, GATE_ACCEPTED = 3 };

enum KrylovStage : int { KS_BETA = 0, KS_ALPHA = 1, KS_OMEGA = 2, KS_UPDATE = 3, KS_INIT = 4, KS_NONE = 5, KS_RESID = 6 };
// Completion tickets (one counter per kind of launch that finishes a stage).
enum Ticket : int { TK_APPLY_T = 0, TK_UPDATE_T = 1, TK_START_T = 2, TK_WOOD_T = 3, TK_DIAG_T = 4, TK_COUNT_T = 8 };

__global__ void k_hh_table(double *hh, const double *r, int Nr, int K, double R1, double R2, double q,
                           double scale, double a1, double a2);
// Two-nodes-per-thread operator kernel on 64-node tiles with a two-row blocked table
// (templated on the widest Gaunt block), launched through these host functions.
constexpr int APPLY3_TILE = 64;
cudaError_t set_apply3_smem(int bytes);
const void *apply3_kernel(int l_max, int vpart, bool gsm);
void launch_apply3(int l_max, bool gsm, dim3 blocks, size_t smem, cudaStream_t st, const Grid &g,
                   const CouplingTable &ct, const BlockTable &bt, const ApplyPlan &pl, const ApplyArgs &a);
// Arguments of the diagnostics pass (k_diag3, and k_diag5 for l_max <= 8): H psi,
// V psi, dV/dt psi and dpsi/dt on nodes <= idx_ex, reduced into per-CTA partials
// [slot][block]: slots 0..n-1 norms, n..2n-1 energies, 2n edge energy, 2n+1 p_bin,
// 2n+2 dV; dpsi/dt and psi around idx_ex stored for the fluxes).
struct DiagArgs {
    const double *hh;
    double theta, domega;
    const double2 *psi;
    int idx_ex;
    int n_sinks;
    const double2 *sv0, *sv1, *sink_dots;
    double sink_coef0, sink_coef1;
    int slo0, shi0, slo1, shi1;
    double *partials;
    double2 *dpsi_edge, *psi_edge;
    const struct Krylov *gate;  // skip until the step's candidate is accepted (null: always run)
};

// The diagnostics pass on the operator kernel's tiles and work plan (grid: tiles up to
// idx_ex x row groups; the partials' stride is the grid's size).
cudaError_t set_diag3_smem(int bytes);
const void *diag3_kernel(int l_max);
void launch_diag3(int l_max, dim3 blocks, size_t smem, cudaStream_t st, const Grid &g, const CouplingTable &ct,
                  const BlockTable &bt, const ApplyPlan &pl, const DiagArgs &d);
__global__ void k_sink_dots(const double2 *x, int Nr, int n_modes, int n_sinks, const double2 *v0,
                            const double2 *v1, int lo0, int hi0, int lo1, int hi1, double2 *dots, const Krylov *gate,
                            int gate_mode);
__global__ void k_precond_factor_diag(const double2 *diag, int Nr, double2 off, int chunk, int window, double rho_max,
                                      double2 *dinv, int *status);
__global__ void k_precond_solve(int Nr, int chunk, int window, double2 off, const double2 *dinv,
                                const double2 *b, double2 *x);
__global__ void k_dots(int64_t n, int nq, const double2 *a0, const double2 *b0, const double2 *a1,
                       const double2 *b1, const double2 *a2, const double2 *b2, double *partials);
__global__ void k_sum_partials(const double *partials, int nblocks, int nslots, double *out);
__global__ void k_axpby(int64_t n, double2 a, const double2 *x, double2 b, const double2 *w, double2 *y);
__global__ void k_scale_mask(int64_t n, int Nr, double s, const double *mask, const double2 *x, double2 *y,
                             const Krylov *kr);
__global__ void k_bicg_update(int64_t n, Krylov *kr, double2 *x, const double2 *y, const double2 *z, double2 *r,
                              const double2 *s, const double2 *t, const double2 *r0, double *partials, double *red,
                              unsigned *ticket);
__global__ void k_wood_scalar(Krylov *kr, int which, const double2 *proj);
__global__ void k_wood_setup(Krylov *kr, const double2 *vw, double c0, double c1);
__global__ void k_krylov_start(int64_t n, Krylov *kr, const double *red_in, const double2 *rhs, const double2 *psi,
                               double2 *x, double2 *r, double2 *r0, double *partials, double *red, unsigned *ticket);
__global__ void k_precond_solve2(int Nr, int chunk, int window, double2 off, const double2 *dinv, const double2 *b,
                                 double2 *x, PrecondInput in);
__global__ void k_precond_factor2(Grid g, CouplingTable ct, const double *hh, double half_dt, double2 off, int chunk,
                                  int window, double2 *dinv, int *status);
// Woodbury scalars finished by the cluster solve (last CTA): WD_SETUP after solving
// W_b = P^{-1} v_b (b = 0 in the first half of the grid, 1 in the second), WD_PROJ
// after y = P^{-1} b (c = G^{-1} v^dag y into kr->wc[which], kr->sdots[which]).
enum WoodMode : int { WD_NONE = 0, WD_SETUP = 1, WD_PROJ = 2 };
struct WoodArgs {
    int mode, which, n_sinks;
    const double2 *v0, *v1;
    int lo0, hi0, lo1, hi1;
    double c0, c1;       // dt/4 g_a (WD_SETUP)
    double *partials;    // [8][grid blocks]
    unsigned *ticket;
    Krylov *kr;
};
__global__ void k_precond_solve_cl(int Nr, int n_modes, int per, double2 off, const double2 *dinv, const double2 *b,
                                   double2 *x, const double2 *b2, double2 *x2, PrecondInput in, WoodArgs wd);
// Woodbury set-up restricted to the band of nodes where W_a = P^{-1} v_a is not
// negligible (one CTA of WSB_THREADS per radial block and sink, 32 bytes of dynamic
// shared memory per band node); see k_wood_setup_band.
struct WoodBand {
    int n_sinks;
    const double2 *v0, *v1;  // sink projectors (zero outside their supports)
    double2 *W0, *W1;        // W_a on the band (not written elsewhere)
    int slo0, shi0, slo1, shi1;
    double c0, c1;           // dt/4 g_a
    double *partials;        // [8][n_modes]
    unsigned *ticket;
    Krylov *kr;
};
constexpr int WSB_THREADS = 512;
__global__ void k_wood_setup_band(int Nr, int n_modes, int blo, int bhi, double2 off, const double2 *dinv,
                                  WoodBand wb);
__global__ void k_precond_factor_cl(Grid g, CouplingTable ct, const double *hh, double half_dt, double2 off, int per,
                                    double2 *dinv, float2 *dinv32, int *status);
// One or two absorbers: support [lo, hi), projector range [wlo, whi) (the support and
// the previous one), moments and projector buffers, the parity flag of the second body.
struct AbsorberPair {
    int count;
    int lo[2], hi[2], wlo[2], whi[2];
    double radius[2], width[2];
    double *mom[2];
    double2 *v[2];
    int secondary[2];
};
__global__ void k_abs_moments(const double *r, int Nr, int nq, const double *gl_x, const double *gl_w, int degree,
                              AbsorberPair ap);
__global__ void k_swave_projector(const double *r, int Nr, int n_modes, double dr, const double *ang00,
                                  const int *mode_l, const int *mode_m, double theta, AbsorberPair ap);
__global__ void k_sum_slots(const double *partials, int nblocks, int nslots, double *out, const Krylov *gate);

__global__ void k_fp64_peak(double *out, int iters, double b, double c);

__global__ void k_jacobi_diag(Grid g, CouplingTable ct, const double *hh, double half_dt, double2 *dj);
__global__ void k_jacobi_apply(int64_t n, const double2 *dj, const double2 *b, double2 *out, PrecondInput in);

__global__ void k_woodbury_band(int Nr, int n_modes, int lo, int hi, const Krylov *kr, int which, const double2 *W0,
                                const double2 *W1, double2 *y);

__global__ void k_displaced_100(const double *r, int Nr, int lmax, double a0, double distance, double amplitude,
                                int nq, const double *gl_x, const double *gl_w, double *mom);

}  // namespace cnm

/*
 * cnm_gpu.h -- C ABI of the B200 Crank-Nicolson step of CrankNicolsonModes.
 *
 * The reference (rdellamonica/boson-cloud-binary) exposes its solver as the C++
 * class CrankNicolsonModes (include/CrankNicolsonModes.hpp:60-455).  This header
 * is the flat interface underneath a drop-in replacement of that class: plain
 * pointers and sizes, no Eigen or torch types.  Every entry point names the
 * reference member it replaces.
 *
 * Conventions
 *  - A handle owns all device memory of one binary; host buffers belong to the
 *    caller.  A handle must not be used from two threads at once.
 *  - States are complex128, stored as interleaved (re, im) doubles, mode-major:
 *    entry j*Nr+i is mode j at radial node i, exactly the reference's layout
 *    (include/CrankNicolsonModes.hpp:10-12).
 *  - Every function returns CNM_OK (0) or an error code; cnm_last_error()
 *    gives the message.  The codes map one to one onto the exceptions the
 *    reference throws: CNM_EINVAL <-> std::invalid_argument,
 *    CNM_ELOGIC <-> std::logic_error, CNM_ESOLVE <-> std::runtime_error.
 *  - Calls are synchronous with respect to the host.
 */
#ifndef CNM_GPU_H
#define CNM_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum cnm_status {
    CNM_OK = 0,
    CNM_EINVAL = 1,   /* std::invalid_argument in the reference */
    CNM_ELOGIC = 2,   /* std::logic_error */
    CNM_ESOLVE = 3,   /* std::runtime_error: the CN solve failed its residual check */
    CNM_ECUDA = 4,    /* CUDA runtime error, or the CUDA kernels are unavailable */
    CNM_ENOMEM = 5,   /* device allocation failed */
    CNM_EDEVICE = 6   /* a device-side check failed (non-finite pivot, scan window) */
};

enum cnm_precision {
    CNM_FP64 = 0,     /* complex128 everywhere: the drop-in path */
    CNM_MIXED = 1     /* complex64 inner iterations on a tensor-core coupling apply, fp64
                         residuals, refinement, dots, diagnostics and orbit (no counterpart
                         in the reference, which is fp64 only) */
};

/* Operators for cnm_apply (all of size Nr*n_modes). */
enum cnm_operator {
    CNM_OP_H = 0,      /* conservative Hamiltonian H = H0 + V (+ CAP)               */
    CNM_OP_H0 = 1,     /* free radial Hamiltonian with the centrifugal term         */
    CNM_OP_V = 2,      /* active potential V1 + ramp * V2                           */
    CNM_OP_V1 = 3,     /* primary's potential                                      */
    CNM_OP_V2 = 4,     /* companion's potential                                    */
    CNM_OP_DVDT = 5,   /* dV/dt from the orbital rotation                          */
    CNM_OP_A = 6,      /* sparse CN operator 1 + i dt H / 2                        */
    CNM_OP_B = 7,      /* sparse CN operator 1 - i dt H / 2                        */
    CNM_OP_SINK = 8,   /* Gamma = sum_a g_a v_a v_a^dagger (zero when inactive)    */
    CNM_OP_RHS = 9,    /* schrodinger_rhs: -i H x - Gamma x / 2                    */
    CNM_OP_AFULL = 10, /* A + (dt/4) Gamma, the operator BiCGSTAB inverts          */
    CNM_OP_CAP = 11,   /* diagonal complex absorbing potential (zero if not built) */
    CNM_OP_PRECOND = 12 /* inverse of the per-mode radial blocks of A              */
};

typedef struct cnm_handle cnm_handle;

/* Constructor arguments, in the order of CrankNicolsonModes::CrankNicolsonModes
 * (include/CrankNicolsonModes.hpp:84; src/CrankNicolsonModes.cpp:11-50). */
typedef struct cnm_params {
    int32_t Nr;
    double L;
    double dt;
    double epsilon;
    int32_t l_max;
    double mu;
    double M_c;
    double q;
    double a;
    double R;
    int32_t counter;
    int32_t absorption;
    int32_t save_every;
    double ramp_periods;
    double epsilon_smear;
    int32_t precision;   /* enum cnm_precision */
} cnm_params;

/* The evolving public scalars of the class (include/CrankNicolsonModes.hpp:88-158)
 * plus the private time t_i, the phase-averaged p_bin and the solver knobs that
 * the reference hard-codes (src/CrankNicolsonModes_matrices.cpp:19-20). */
typedef struct cnm_scalars {
    double t;              /* t_i, time of the current state                    */
    double theta, phase, Omega, Omega_0, P;
    double R, R1, R2, M1, M2, q;
    double dt;
    double p_bin;
    double steps_per_period;
    int32_t evolve_orbit;
    int32_t ramp_secondary_potential;
    int32_t use_block_preconditioner;
    int32_t last_solver_iterations;
    double last_solver_residual;
    double tolerance;      /* BiCGSTAB relative tolerance, reference 1e-10       */
    int32_t max_iterations;/* reference 500                                      */
    double accept_residual;/* acceptance of the true residual, reference 1e-9    */
} cnm_scalars;

/* One step's diagnostics: the rows step() appends to R.txt ... energy_modes.txt
 * (src/CrankNicolsonModes.cpp:197-226).  The four per-mode arrays are written to
 * caller buffers of n_modes doubles each (any of them may be NULL). */
typedef struct cnm_diag {
    double R, theta, Omega, M1, q, t;
    double energy, p_bin, p_bin_inst, dV_bin_dt;
    double residual;
    int32_t iterations;
} cnm_diag;

/* --- lifetime ---------------------------------------------------------------- */

/* CrankNicolsonModes::CrankNicolsonModes (src/CrankNicolsonModes.cpp:11-50):
 * builds the grid, the (l, m) list with even l-m, and the free Hamiltonian. */
int cnm_create(const cnm_params *params, cnm_handle **out);
/* Make `device` current for the calling thread before cnm_create (one process per
 * GPU; the handle stays on the device that was current when it was created). */
int cnm_select_device(int32_t device);
int cnm_destroy(cnm_handle *h);
const char *cnm_last_error(const cnm_handle *h);
/* Message of the last failed cnm_create (no handle exists then). */
const char *cnm_create_error(void);

/* --- geometry ---------------------------------------------------------------- */

int cnm_n_modes(const cnm_handle *h, int32_t *n_modes);       /* member n_modes */
int cnm_modes(const cnm_handle *h, int32_t *l, int32_t *m);   /* member modes   */
int cnm_grid(const cnm_handle *h, double *r);                 /* member r       */
/* Size of the coupling cache (mode_pairs and their Gaunt terms,
 * src/CrankNicolsonModes_hamiltonian.cpp:68-104). */
int cnm_coupling_info(const cnm_handle *h, int32_t *n_pairs, int32_t *n_terms);

/* --- scalar members ---------------------------------------------------------- */

int cnm_get_scalars(const cnm_handle *h, cnm_scalars *out);
int cnm_set_scalars(cnm_handle *h, const cnm_scalars *in);

/* --- state -------------------------------------------------------------------- */

/* set_initial_state_full (src/CrankNicolsonModes.cpp:130-143): copies psi_0 and
 * scales it by sqrt(M_c / mu).  CNM_EINVAL if n != Nr * n_modes. */
int cnm_set_initial_state_full(cnm_handle *h, const double *psi0, int64_t n);
/* Raw access to member psi (no scaling). */
int cnm_set_state(cnm_handle *h, const double *psi, int64_t n);
int cnm_get_state(const cnm_handle *h, double *psi, int64_t n);
/* Page-locked host memory for state copies (cnm_get_state into it runs at the full
 * device-to-host rate): cnm_host_alloc returns *ptr = NULL and CNM_ECUDA when the
 * allocation fails (cnm_create_error() says why); cnm_host_free(NULL) does nothing.
 * No counterpart in the reference, whose state lives in host memory. */
int cnm_host_alloc(int64_t bytes, void **ptr);
int cnm_host_free(void *ptr);

/* --- set-up ------------------------------------------------------------------- */

/* configure_isolated_black_hole (src/CrankNicolsonModes.cpp:58-74). */
int cnm_configure_isolated_black_hole(cnm_handle *h, double x);
/* initialize (src/CrankNicolsonModes.cpp:76-98): coupling tables, t = 0 operator. */
int cnm_initialize(cnm_handle *h);
/* set_power_average_orbits (src/CrankNicolsonModes.cpp:52-56). */
int cnm_set_power_average_orbits(cnm_handle *h, double n_orbits);
/* build_damping_mask / build_cap (src/CrankNicolsonModes_outgoing.cpp:10-62). */
int cnm_build_damping_mask(cnm_handle *h, double L_factor, double W, int32_t n);
int cnm_build_cap(cnm_handle *h, double L_factor, double W, int32_t n);

/* --- evolution ---------------------------------------------------------------- */

/* The computational part of run() (src/CrankNicolsonModes.cpp:236-259,261-270):
 * validates r_ex against the grid, sets t = 0 and refreshes the operator. */
int cnm_prepare_run(cnm_handle *h, int32_t n_steps, double r_ex);
/* build_time_dependent_perturbation(time) (_hamiltonian.cpp:245-268). */
int cnm_refresh(cnm_handle *h, double time);
/* step(step_id) (src/CrankNicolsonModes.cpp:145-234) without the text writes:
 * the CN solve, mask, orbit update and all diagnostics of the step. */
int cnm_step(cnm_handle *h, int32_t step_id, cnm_diag *diag, double *energy_flux,
             double *flux, double *norms, double *energies);
/* The stop test of evolve() (src/CrankNicolsonModes.cpp:276-282): 1 when R <= 6
 * on an evolving binary orbit. */
int cnm_should_stop(const cnm_handle *h, int32_t *stop);

/* --- initial states ----------------------------------------------------------------
 * displaced_100_state (src/DisplacedAtom.cpp:12-76) on the device: the mode projection
 * of a hydrogenic 1s state of reduced mass mu centred at x_bh on the x axis, on the
 * radial nodes r[Nr] and modes (l[j], m[j]); state: interleaved complex, n_modes x Nr
 * (host buffer).  CNM_EINVAL for the reference's invalid_argument cases. */
int cnm_displaced_100_state(const double *r, int32_t Nr, const int32_t *l, const int32_t *m, int32_t n_modes,
                            double mu, double x_bh, double *state);

/* The initial states of the sweeps (initial_states/get_initial_state_COM_fast.py of the
 * reference, which writes them to MODESBIN files): the mode projection of the hydrogenic
 * (n, la, ma) state of reduced mass mu about a body of mass M1 at x = x_center on the x axis,
 *     U_j(r) = r int conj(Y_j) psi_nlm(r Omega - x_center e_x) dOmega,
 * on the device, with n_theta Gauss-Legendre nodes in cos(theta) and n_phi uniform angles;
 * normalised to sum |U|^2 dr = 1 on the (uniform) grid; U vanishes on the two end nodes.
 * state: interleaved complex, n_modes x Nr (host buffer); at most 160 modes. */
int cnm_hydrogenic_state(const double *r, int32_t Nr, const int32_t *l, const int32_t *m, int32_t n_modes, double mu,
                         double M1, double x_center, int32_t n, int32_t la, int32_t ma, int32_t n_theta, int32_t n_phi,
                         double *state);

/* --- batched sweep (independent binaries) ------------------------------------------
 * A batch owns one handle per binary, each with its own stream.  cnm_batch_step
 * advances every binary by one step: it queues the device work of all binaries
 * before it waits on any, so binaries too small to fill the device run side by side.
 * The per-binary handles are set up and read through the single-binary calls
 * (cnm_set_initial_state_full, cnm_initialize, cnm_prepare_run, cnm_get_state, ...). */
typedef struct cnm_batch cnm_batch;
/* params[count]: one binary each.  On failure no batch is created. */
int cnm_batch_create(const cnm_params *params, int32_t count, cnm_batch **out);
int cnm_batch_size(const cnm_batch *b, int32_t *count);
int cnm_batch_handle(cnm_batch *b, int32_t index, cnm_handle **h);
/* diags[count] may be NULL; the per-mode diagnostics of a binary are not returned here
 * (step it alone with cnm_step for those).  Every binary's step is completed even when
 * another one fails; the first failure's status is returned. */
int cnm_batch_step(cnm_batch *b, int32_t step_id, cnm_diag *diags);
int cnm_batch_destroy(cnm_batch *b);

/* --- checkpoints --------------------------------------------------------------- */

/* save_checkpoint (src/CrankNicolsonModes_restart.cpp:139-177): the exact bytes of
 * checkpoint.bin -- "GMCKPT01", int32 {step_id, Nr, n_modes}, 13 doubles {t, theta,
 * phase, R, M1, M2, q, R1, R2, Omega, P, dt, p_bin}, uint64 size, psi as complex128,
 * then the rolling-average state of src/RollingPhase.cpp:169-184.  Writes *size; the
 * bytes go to buf when buf is non-NULL and capacity >= *size.  The caller writes the
 * file (the reference replaces it atomically through a .tmp file). */
int cnm_save_checkpoint(const cnm_handle *h, int32_t step_id, void *buf, int64_t capacity, int64_t *size);
/* load_checkpoint (src/CrankNicolsonModes_restart.cpp:179-233): restores psi, the
 * evolving scalars and the rolling average when buf is a complete checkpoint of
 * step_id for this grid; *loaded = 1 then, else 0 and nothing changes. */
int cnm_load_checkpoint(cnm_handle *h, int32_t step_id, const void *buf, int64_t size, int32_t *loaded);

/* reconstruct_state_from_diagnostics (src/CrankNicolsonModes_restart.cpp:238-286): reset
 * the rolling phase average of p_bin and feed it the n stored samples (time, phase,
 * p_bin_inst) of the diagnostic rows. */
int cnm_replay_power_average(cnm_handle *h, const double *times, const double *phases, const double *values,
                             int32_t n);

/* --- operators ------------------------------------------------------------------ */

/* y = op x for an interleaved complex128 vector of length Nr * n_modes, with
 * the operators of the current time (H, V, dVdt, A, B, apply_sink and
 * schrodinger_rhs of include/CrankNicolsonModes.hpp:197-213). */
int cnm_apply(cnm_handle *h, int32_t op, const double *x, double *y);
/* The low-precision operator of the mixed path (CNM_MIXED handles only): y = op x with
 * x rounded to complex64 and the coupling on the tensor cores (bf16 operands, fp32
 * accumulation), for op in {CNM_OP_H, CNM_OP_V, CNM_OP_A, CNM_OP_AFULL}; the result is
 * widened to complex128.  No counterpart in the reference (used by the parity tests). */
int cnm_apply_lowp(cnm_handle *h, int32_t op, const double *x, double *y);
/* Counters of the mixed solve's last step: defect-correction passes, fp64 operator
 * applications, and the final relative residual (fp64 or from the tensor-core check). */
int cnm_mixed_info(const cnm_handle *h, int32_t *passes, int32_t *fp64_applies, double *residual);
/* The last residual check of the mixed solve, six doubles relative to |rhs|: the
 * tensor-core residual, its error estimate, the last fp64 residual, the calibration
 * correction's norm, the last correction's norm, and the calibrated error ratio
 * |A_fp64 d - A_tc d| / |d|.  Measurement hook (no counterpart in the reference). */
int cnm_mixed_trace(const cnm_handle *h, double *out);
/* sink_strength(body) (_absorption.cpp:119-125). */
int cnm_sink_strength(const cnm_handle *h, int32_t body, double *out);
/* absorption_sink_active(). */
int cnm_sink_active(const cnm_handle *h, int32_t *active);
/* The projector v_a of one body's sink (interleaved, Nr * n_modes). */
int cnm_sink_vector(const cnm_handle *h, int32_t body, double *out);

/* --- measurement hooks (no counterpart in the reference) -------------------------
 * Device-event timing of the handle's stream, used by the benchmark: whole regions
 * (start/stop) and, while profiling is on, every launch of the hot kernel classes:
 * 0 fp64 operator apply, 1 fp64 preconditioner solve, 2 pivot factorisation, 3 fused
 * diagnostics, 4 tensor-core operator apply, 5 fp32 preconditioner solve. */
int cnm_set_profiling(cnm_handle *h, int32_t on);
int cnm_kernel_times(cnm_handle *h, int32_t which, double *total_ms, int64_t *launches);
int cnm_timer_start(cnm_handle *h);
/* Tensor-core operator layout of a CNM_MIXED handle: the padded mode count, for each of
 * the 2 l_max + 1 multipoles the number of non-zero 16-column slices of its Gaunt matrix
 * (one M128 x N(2 nt) x K16 MMA per slice and tile), the highest multipole every tile runs
 * whatever its radial cut, and the nodes per tile nt (any pointer may be NULL). */
int cnm_tc_blocks(const cnm_handle *h, int32_t *kp, int32_t *nblk, int32_t *lc_min, int32_t *nt);
/* Kernels the handle has launched since its creation (every launch site counts). */
int cnm_launch_count(const cnm_handle *h, int64_t *count);
int cnm_timer_stop(cnm_handle *h, double *ms);
/* Operator kernel selection (testing and measurement): 1 (default) uses the kernel
 * specialised at compile time for l_max <= 8 where it exists, 0 the generic
 * plan-driven kernel. */
int cnm_set_operator_kernel(cnm_handle *h, int32_t specialised);
/* FP64 FMA throughput of the current device in TFLOP/s (2 flops per FMA), from a
 * register-resident chain microbenchmark timed with device events: the denominator of
 * the FP64 roofline of the operator kernels. */
int cnm_measure_fp64_peak(double *tflops);
/* Autotuner (no counterpart in the reference, which has no device plans): times every
 * row-group count of the operator kernel that has a resident configuration (five
 * applications of A to the current state each, device events on the handle's stream) and,
 * on a CNM_MIXED handle, every Gaunt-stage count of the tensor-core apply from 3 to the most
 * that fit; keeps the fastest of each and reports them.  Needs an initialized handle.
 * cnm_set_tuning applies choices found earlier (0 = the creation-time plan: the cost
 * model's row groups, as many stages as fit), e.g. from a cache keyed by device and shape. */
int cnm_autotune(cnm_handle *h, int32_t *apply_groups, int32_t *tc_stages);
/* The current device's name (the autotuner cache's key), NUL-terminated in name[size]. */
int cnm_device_name(char *name, int32_t size);
int cnm_set_tuning(cnm_handle *h, int32_t apply_groups, int32_t tc_stages);
/* Launch plan chosen at creation for this device: nodes per thread and CTAs per cluster
 * of the exact preconditioner scans (0, 0 when the windowed scans are used), row groups
 * of the operator kernel in use (the kernel specialised for l_max <= 8 when it is
 * enabled, else CTA groups per node tile of the generic kernel) and whether a group's
 * weights sit in shared memory (1) or are read through L1 (0). */
int cnm_plan_info(const cnm_handle *h, int32_t *scan_per, int32_t *scan_cluster, int32_t *apply_groups,
                  int32_t *apply_weights_in_smem);

/* --- radial block solve without allocation (no counterpart in the reference) -----
 * For callers that cannot call cudaMalloc -- a host code that gives the solver a
 * fixed, pre-reserved device arena and allows no other allocation, a driver that
 * launches from a region where allocation is forbidden, a plug-in that only
 * receives device pointers -- and so cannot create a handle.  Solves, for every
 * mode j, the tridiagonal system
 *     diag[j,i] x[j,i] + off (x[j,i-1] + x[j,i+1]) = b[j,i]   for 1 <= i <= Nr-2,
 *     diag[j,i] x[j,i] = b[j,i]                                for i = 0, Nr-1,
 * by chunked parallel Thomas sweeps (2048 nodes per chunk, each chunk started from a
 * warm-up window).  The windows are sized for a diagonally dominant system: the
 * sweeps must contract by |off / p_i| < rho per node (p_i the Thomas pivots), with rho
 * the rate of the diagonal 1 + 1.98 i |off| (the CN radial blocks satisfy this).  With
 * Nr <= 2048 there is one chunk per mode and the solve is exact for any non-singular
 * system; beyond that a system that contracts more slowly is refused (CNM_EDEVICE),
 * never solved inexactly.
 *   diag, b, x  device pointers to Nr * n_modes interleaved complex128 values,
 *               mode-major (x may not alias diag or b);
 *   off         the constant off-diagonal (re, im);
 *   stream      a cudaStream_t (NULL: the legacy default stream); the call returns
 *               after the solve has finished on it.
 * It allocates nothing: the inverse pivots live in one file-scope device array
 * of CNM_NOALLOC_MAX_UNKNOWNS complex values (16 MiB per GPU, held from the
 * library's load until the process exits).  Larger problems (Nr * n_modes above
 * the maximum) are rejected with CNM_EINVAL before any GPU work.  The first call on
 * a device looks up the array's device address (and sets the solve kernel's
 * shared-memory limit); make that first call before any stream capture.  Every call
 * shares the one array, so calls that overlap on the GPU (concurrent streams or
 * threads) race and must be serialised by the caller.  Returns CNM_EDEVICE if a
 * pivot is zero or not finite or the system is not dominant enough for the chunked
 * sweeps, CNM_ECUDA on a CUDA error. */
#define CNM_NOALLOC_MAX_UNKNOWNS (1 << 20)
int cnm_radial_solve_noalloc(const double *diag, double off_re, double off_im, int32_t Nr, int32_t n_modes,
                             const double *b, double *x, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CNM_GPU_H */

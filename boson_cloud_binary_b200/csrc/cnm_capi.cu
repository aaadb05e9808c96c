// cnm_capi.cu -- the handle behind include/cnm_gpu.h: state, one CN step on the
// device, and the host-side FP64 orbit bookkeeping of the reference class.
//
// Call sequence of one step (src/CrankNicolsonModes.cpp:145-234):
//   host:   t += dt, theta += s Omega dt, phase += Omega dt; ramps and Omega
//           (build_time_dependent_perturbation, _hamiltonian.cpp:245-268)
//   device: hh table, absorber moments and projectors, sink projections of the
//           old state, rhs = B psi - dt/4 Gamma psi, pivots, Woodbury set-up,
//           BiCGSTAB (device-resident scalars), residual check, mask,
//           fused diagnostics (one pass for H psi, V psi, dV/dt psi and dpsi/dt)
//   host:   orbit ODE (_evolution.cpp:17-72), rolling phase average, diagnostics.
#include "../../include/cnm_gpu.h"
#include "cnm_coupling.h"
#include "cnm_kernels.cuh"
#include "cnm_apply5.cuh"
#include "cnm_mixed.cuh"
#include "cnm_initial.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cmath>
#include <complex>
#include <cstring>
#include <deque>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

namespace cnm {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

void cuda_check(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) throw Error(e == cudaErrorMemoryAllocation ? CNM_ENOMEM : CNM_ECUDA,
                                      std::string(what) + ": " + cudaGetErrorString(e));
}
#define CK(x) ::cnm::cuda_check((x), #x)

template <class T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    void alloc(size_t count)
    {
        release();
        if (count == 0) return;
        CK(cudaMalloc(&p, count * sizeof(T)));
        n = count;
        CK(cudaMemset(p, 0, count * sizeof(T)));
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    ~DevBuf() { release(); }
};

// Fused reductions of an operator launch: up to two inner products of its output
// (ApplyArgs::dot_kind), optionally finished by the last CTA into `red` with a scalar
// stage (KS_*; KS_NONE only stores the sums).
struct DotSpec {
    int n = 0;
    int kind[2] = {0, 0};
    const double2 *ext[2] = {nullptr, nullptr};
    double scale = 1.0;
    int stage = -1;
    double *red = nullptr;
    int gate_mode = 0;         // GateMode of the launch
    bool scale_from_kr = false;  // kind 4 scale = the solve's |rhs| (device)
};

// Rolling time average over a window of orbital phase (src/RollingPhase.cpp:24-129).
class RollingPhaseAverage {
public:
    explicit RollingPhaseAverage(double n_orbits = 2.0) : window_(2.0 * M_PI * n_orbits)
    {
        if (n_orbits <= 0.0) throw Error(CNM_EINVAL, "RollingPhaseAverage: n_orbits must be positive");
    }
    double update(double time, double phase, double value)
    {
        if (!has_prev_) {
            prev_ = {time, phase, value};
            initial_phase_ = phase;
            has_prev_ = true;
            average_ = value;
            return average_;
        }
        if (time <= prev_.time) throw Error(CNM_ESOLVE, "RollingPhaseAverage: time must increase");
        if (phase <= prev_.phase) throw Error(CNM_ESOLVE, "RollingPhaseAverage: phase must increase");
        Seg s{prev_.time, time, prev_.phase, phase, prev_.value, value, 0.0};
        s.integral = 0.5 * (s.v0 + s.v1) * (s.t1 - s.t0);
        segs_.push_back(s);
        integral_ += s.integral;
        duration_ += s.t1 - s.t0;
        if (phase - initial_phase_ >= window_) ready_ = true;
        const double cut = phase - window_;
        while (!segs_.empty() && segs_.front().p1 <= cut) {
            integral_ -= segs_.front().integral;
            duration_ -= segs_.front().t1 - segs_.front().t0;
            segs_.pop_front();
        }
        if (!segs_.empty()) {
            Seg &f = segs_.front();
            if (f.p0 < cut && cut < f.p1) {
                const double fr = (cut - f.p0) / (f.p1 - f.p0);
                const double tc = f.t0 + fr * (f.t1 - f.t0), vc = f.v0 + fr * (f.v1 - f.v0);
                integral_ -= 0.5 * (f.v0 + vc) * (tc - f.t0);
                duration_ -= tc - f.t0;
                f.t0 = tc;
                f.p0 = cut;
                f.v0 = vc;
                f.integral = 0.5 * (f.v0 + f.v1) * (f.t1 - f.t0);
            }
        }
        duration_ = std::max(duration_, 0.0);
        average_ = duration_ > 0.0 ? integral_ / duration_ : value;
        prev_ = {time, phase, value};
        return average_;
    }

    // Exact state in the byte layout of the reference's RollingPhaseAverage::save
    // (src/RollingPhase.cpp:169-184): window, previous sample (3 doubles), two bools,
    // initial phase, integral, duration, average, u64 count, then 7 doubles per segment.
    size_t blob_size() const { return 8 + 24 + 1 + 1 + 4 * 8 + 8 + 56 * segs_.size(); }
    void save(std::vector<char> &out) const
    {
        auto put = [&](const void *p, size_t n) {
            const char *c = static_cast<const char *>(p);
            out.insert(out.end(), c, c + n);
        };
        put(&window_, 8);
        put(&prev_, 24);
        put(&has_prev_, 1);
        put(&ready_, 1);
        put(&initial_phase_, 8);
        put(&integral_, 8);
        put(&duration_, 8);
        put(&average_, 8);
        const uint64_t n = segs_.size();
        put(&n, 8);
        for (const Seg &sg : segs_) put(&sg, 56);
    }
    // Returns false on a truncated blob (the reference throws there and the caller
    // treats the checkpoint as unusable).
    bool load(const char *p, size_t size, size_t &used)
    {
        size_t o = 0;
        auto get = [&](void *dst, size_t n) {
            if (o + n > size) return false;
            std::memcpy(dst, p + o, n);
            o += n;
            return true;
        };
        RollingPhaseAverage r(1.0);
        uint64_t n = 0;
        if (!(get(&r.window_, 8) && get(&r.prev_, 24) && get(&r.has_prev_, 1) && get(&r.ready_, 1) &&
              get(&r.initial_phase_, 8) && get(&r.integral_, 8) && get(&r.duration_, 8) && get(&r.average_, 8) &&
              get(&n, 8)))
            return false;
        for (uint64_t i = 0; i < n; ++i) {
            Seg sg;
            if (!get(&sg, 56)) return false;
            r.segs_.push_back(sg);
        }
        *this = r;
        used = o;
        return true;
    }

private:
    struct Sample { double time, phase, value; };
    struct Seg { double t0, t1, p0, p1, v0, v1, integral; };
    static_assert(sizeof(Sample) == 24 && sizeof(Seg) == 56, "checkpoint layout");
    double window_;
    std::deque<Seg> segs_;
    Sample prev_{};
    bool has_prev_ = false, ready_ = false;
    double initial_phase_ = 0, integral_ = 0, duration_ = 0, average_ = 0;
};

// One body's absorber: kernel moments on the device, support on the host.
struct Absorber {
    double radius = -1.0, width = -1.0;
    bool valid = false;
    int lo = 0, hi = 0;            // node support [lo, hi) of the projector
    int wlo = 0, whi = 0;          // nodes the projector kernel must (re)write
    double strength = 0.0;         // g = A_h dr
    DevBuf<double> mom;            // (2 l_max + 1) x Nr
    DevBuf<double2> v;             // projector, Nr * n_modes
};

// Operator parameters frozen at the last build_time_dependent_perturbation; the
// reference's assembled matrices keep these values until the next rebuild.
struct OpState {
    bool built = false;
    double theta = 0, domega = 0, dt = 0;
    double R1 = 0, R2 = 0, q = 0, Mtot = 0, w = 0;  // geometry of the hh table
    bool cap = false;
    bool sink_active = false;
};

// Device-event timing of one class of kernel launches (profiling hook).
struct KernelTimer {
    std::vector<cudaEvent_t> a, b;
    int used = 0;
    double ms = 0.0;
    int64_t launches = 0;
    ~KernelTimer()
    {
        for (cudaEvent_t e : a) cudaEventDestroy(e);
        for (cudaEvent_t e : b) cudaEventDestroy(e);
    }
};

enum TimedKernel : int { TK_APPLY = 0, TK_PSOLVE = 1, TK_PFACTOR = 2, TK_DIAG = 3, TK_TC = 4, TK_PSOLVE32 = 5, TK_COUNT = 6 };

struct Solver {
    // constructor arguments and derived constants
    int Nr, l_max, n_modes, save_every;
    double L, dr, epsilon, mu, M_c, a_spin, epsilon_smear, ramp_periods, initial_period;
    bool counter, absorption;
    // evolving scalars (public members of the reference class)
    double t_i = 0, theta = 0, phase = 0, Omega = 0, Omega_0, P, R, R1, R2, M1, M2, q, dt, p_bin = 0;
    double steps_per_period = 50.0;
    bool evolve_orbit = true, ramp_secondary_potential = true, use_block = true;
    double last_residual = 0.0;
    int last_iterations = 0;
    double tolerance = 1e-10, accept_residual = 1e-9;
    int max_iterations = 500;
    // private state
    bool isolated = false, initialized = false, sink_active = false, mask = false, cap = false;
    double ramp_factor = 0.0, potential_ramp_factor = 0.0;
    int idx_ex = 0;
    double r_ex = 0.0;
    double orbits_average = 2.0;
    RollingPhaseAverage power_average{2.0};
    OpState op;
    std::vector<double> r;
    Coupling cpl;
    std::vector<double> capw_h, mask_h;

    // device
    cudaStream_t stream = nullptr;
    int64_t nN;
    int K;
    DevBuf<double> d_r, d_hh, d_hh_aux, d_capw, d_mask, d_glx, d_glw, d_partials, d_red, d_ang00;
    DevBuf<int> d_pair_row_ptr, d_pair_col, d_pair_term_ptr, d_term_l, d_diag_pair, d_mode_l, d_mode_m, d_status;
    DevBuf<double> d_term_g;
    CouplingPlan plan3;           // operator kernel work plan (its blocks: 1-2 row chunks in list order)
    bool apply3_gsm = false;      // group weights staged in shared memory
    DevBuf<int> d3_list_ptr, d3_group_goff;
    DevBuf<double> d_ir2;
    DevBuf<int> d2_chunk_l, d2_chunk_nrows, d2_chunk_rows, d2_chunk_goff, d2_l_off;
    DevBuf<double> d2_block_g;
    size_t apply3_smem = 0;
    DevBuf<double2> psi, rhs, x, rr, r0, p, p2, v, s, t, y, z, yP, W0, W1, tmp, cand, dinv;
    DevBuf<double2> d_dots;   // [0..1] psi, [2..3] psi_last, [4..5] scratch, [6..7] G set-up
    DevBuf<double2> d_edge;   // dpsi at idx_ex (n) + psi at idx_ex-1..idx_ex+1 (3n)
    DevBuf<Krylov> d_kr;
    Absorber abs1, abs2;
    int gl_n = 0;
    int vec_blocks = 0;
    int precond_chunk = 2048, precond_window = 256;
    // exact cluster scans: nodes per thread (odd) and CTAs per radial block; 0 = the
    // windowed scans are used instead
    int pcl_per = 0, pcl_cs = 0;
    bool jacobi = false;  // fallback solve: point-Jacobi preconditioner in place of the radial blocks
    int wband_lo = 0, wband_hi = 0;  // nodes where the Woodbury vectors W_a are applied
    int iter_hint = 2;               // iterations of the previous solve (first batch size)
    Krylov h_kr_init;                // host source of the Krylov struct's asynchronous upload
    // The reference's A and B are refreshed only by initialize() and step()
    // (update_CN_values), not by the operator rebuild of run(); a CAP built after
    // initialize() reaches H at run() but A and B only at the next step.
    bool ab_cap = false;
    // operator kernel specialised for this l_max (0 groups: the generic plan-driven kernel)
    int a5_groups = 0;
    bool a5_enabled = true;
    DevBuf<double> d_a5tab, d_d5tab;  // weights of the specialised operator and diagnostics layouts
    DevBuf<unsigned> d_tickets;  // completion tickets (zero between launches)
    DevBuf<double> d_wpart;      // partials of the Woodbury projections
    // red slots past the diagnostics' 2 n + 3 sums: |rhs|^2 and the candidate's residual^2
    int RED_RHS = 0, RED_RES = 0;
    size_t diag3_smem = 0;       // the diagnostics pass on the operator kernel's tiles
    int n_sm = 0;
    int tc_amax = 0;             // bytes of the largest multipole's Gaunt image (tensor-core stages)
    // pinned host staging
    double *h_stage = nullptr;
    size_t h_stage_n = 0;
    // mixed precision (CNM_MIXED): tensor-core Gaunt image and plan, complex64 work
    // vectors, fp32 pivots, the fp64 residual and the inner scalars
    bool mixed = false;
    TcGaunt tg;
    TcPlan tcp;
    int64_t tc_replica_bytes = 0;
    DevBuf<uint8_t> d_tcblob;
    DevBuf<int> d_tc_loff, d_tc_lbytes, d_tc_slices, d_tc_lnblk;
    DevBuf<int> d_tc_ctr;           // tile counter of the tensor-core apply (zero between launches)
    DevBuf<unsigned> d_mx_ticket;   // finished blocks of a mixed-solve vector kernel (zero between launches)
    bool pivots32 = false;          // the last factorisation also wrote the fp32 pivots dinv32
    DevBuf<float2> m_r, m_y, m_v, m_s, m_z, m_t, m_d, m_xa, dinv32, m_r1, m_q;
    DevBuf<double2> m_r64, m_dots;  // m_dots: [0..1] sink projections, [2..3] corrected ones
    DevBuf<MixScalars> d_msc;
    DevBuf<double> m_part;
    int ps_per = 0, ps_cs = 0;      // fp32 cluster solve: nodes per thread, CTAs per cluster
    int mx_passes = 0, mx_fp64 = 0; // counters of the last mixed step
    double mx_residual = 0.0;
    double mx_trace[6] = {0, 0, 0, 0, 0, 0};  // last check: see cnm_mixed_trace
    double mixed_tol = 1e-12;       // fp64 relative residual the mixed solve stops at
    int mixed_max_passes = 8;
    // profiling
    bool profiling = false;
    KernelTimer ktime[TK_COUNT];
    cudaEvent_t region_a = nullptr, region_b = nullptr;

    void kt_begin(int k)
    {
        if (!profiling) return;
        KernelTimer &t = ktime[k];
        if (t.used == (int)t.a.size()) {
            if (t.a.size() >= 4096) kt_flush();
            else {
                cudaEvent_t e1, e2;
                CK(cudaEventCreate(&e1));
                CK(cudaEventCreate(&e2));
                t.a.push_back(e1);
                t.b.push_back(e2);
            }
        }
        CK(cudaEventRecord(t.a[t.used], stream));
    }
    void kt_end(int k)
    {
        if (!profiling) return;
        KernelTimer &t = ktime[k];
        CK(cudaEventRecord(t.b[t.used], stream));
        ++t.used;
        ++t.launches;
    }
    void kt_flush()
    {
        if (!profiling) return;
        CK(cudaStreamSynchronize(stream));
        for (KernelTimer &t : ktime) {
            for (int i = 0; i < t.used; ++i) {
                float ms = 0.f;
                CK(cudaEventElapsedTime(&ms, t.a[i], t.b[i]));
                t.ms += ms;
            }
            t.used = 0;
        }
    }

    Solver(const cnm_params &pr)
        : Nr(pr.Nr), l_max(pr.l_max), save_every(pr.save_every), L(pr.L), dr(pr.L / (pr.Nr - 1)),
          epsilon(pr.epsilon), mu(pr.mu), M_c(pr.M_c), a_spin(pr.a), epsilon_smear(pr.epsilon_smear),
          ramp_periods(pr.ramp_periods), initial_period(2.0 * M_PI / std::sqrt((1 + pr.q) / std::pow(pr.R, 3))),
          counter(pr.counter != 0), absorption(pr.absorption != 0), R(pr.R), q(pr.q), dt(pr.dt)
    {
        if (Nr < 3 || l_max < 0 || L <= 0.0 || dt <= 0.0 || save_every <= 0)
            throw Error(CNM_EINVAL, "Require Nr >= 3, l_max >= 0, and positive L, dt, save_every");
        if (pr.precision != CNM_FP64 && pr.precision != CNM_MIXED) throw Error(CNM_EINVAL, "unknown precision");
        mixed = pr.precision == CNM_MIXED;
        Omega = 0.0;
        Omega_0 = std::sqrt((1.0 + q) / std::pow(R, 3));
        P = initial_period;
        R1 = q / (1 + q) * R;
        R2 = 1 / (1 + q) * R;
        M1 = 1.0;
        M2 = q;
        r.resize(Nr);
        for (int i = 0; i < Nr; i++) r[i] = epsilon + i * dr;
        cpl = build_coupling(l_max);
        n_modes = cpl.n_modes;
        K = 2 * l_max + 1;
        nN = (int64_t)Nr * n_modes;
        setup_device();
    }

    ~Solver()
    {
        if (region_a) cudaEventDestroy(region_a);
        if (region_b) cudaEventDestroy(region_b);
        if (h_stage) cudaFreeHost(h_stage);
        if (stream) cudaStreamDestroy(stream);
    }

    template <class T>
    void upload(DevBuf<T> &d, const std::vector<T> &h)
    {
        d.alloc(std::max<size_t>(h.size(), 1));
        if (!h.empty()) CK(cudaMemcpy(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    }

    double *stage(size_t n)
    {
        if (n > h_stage_n) {
            if (h_stage) cudaFreeHost(h_stage);
            CK(cudaMallocHost(&h_stage, n * sizeof(double)));
            h_stage_n = n;
        }
        return h_stage;
    }

    void setup_device()
    {
        int dev = 0;
        CK(cudaGetDevice(&dev));
        int nsm = 0;
        CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        n_sm = nsm;
        CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        vec_blocks = (int)std::max<int64_t>(1, std::min<int64_t>((nN + VEC_THREADS - 1) / VEC_THREADS, (int64_t)nsm * 4));
        upload(d_r, r);
        upload(d_pair_row_ptr, cpl.pair_row_ptr);
        upload(d_pair_col, cpl.pair_col);
        upload(d_pair_term_ptr, cpl.pair_term_ptr);
        upload(d_term_l, cpl.term_l);
        upload(d_term_g, cpl.term_g);
        upload(d_diag_pair, cpl.diag_pair);
        upload(d_mode_l, cpl.mode_l);
        upload(d_mode_m, cpl.mode_m);
        upload(d_ang00, cpl.ang00);
        {
            std::vector<double> ir2(Nr, 0.0);
            for (int i = 0; i < Nr; ++i) ir2[i] = r[i] > 0.0 ? 1.0 / (r[i] * r[i]) : 0.0;
            upload(d_ir2, ir2);
        }
        d_hh.alloc((size_t)K * Nr);
        d_hh_aux.alloc((size_t)K * Nr);
        for (DevBuf<double2> *bptr : {&psi, &rhs, &x, &rr, &r0, &p, &p2, &v, &s, &t, &y, &z, &yP, &W0, &W1, &tmp,
                                      &cand, &dinv})
            bptr->alloc(nN);
        d_dots.alloc(8);
        d_edge.alloc(4 * (size_t)n_modes);
        d_kr.alloc(1);
        d_status.alloc(1);
        RED_RHS = 2 * n_modes + 8;
        RED_RES = 2 * n_modes + 12;
        d_red.alloc(std::max(64, 2 * n_modes + 16));
        d_tickets.alloc(TK_COUNT_T);
        plan_operator(nsm);
        // partials: the vector kernels' slots, the diagnostics pass's 2n + 3 slots per CTA
        // (64-node tiles x row groups) and the operator kernel's fused reductions
        const size_t tiles3 = (size_t)(Nr + APPLY3_TILE - 1) / APPLY3_TILE;
        // (for any row-group count the autotuner may choose: up to 8 per tile)
        const size_t diag_blocks = std::max<size_t>(tiles3 * 8, diag5_blocks(l_max, Nr));
        d_partials.alloc(std::max<size_t>({(size_t)6 * vec_blocks, (size_t)(2 * n_modes + 3) * diag_blocks,
                                           (size_t)4 * 8 * tiles3}));
        a5_groups = apply5_groups(l_max);
        if (a5_groups > 0) {
            upload(d_a5tab, apply5_table(l_max, apply5_groups(l_max), cpl));
            upload(d_d5tab, apply5_table(l_max, diag5_groups(l_max), cpl));
            CK(set_apply5_smem());
            CK(set_diag5_smem());
        }
        CK(cudaFuncSetAttribute(k_precond_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        CK(cudaFuncSetAttribute(k_wood_setup_band, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(2 * WOOD_BAND_MAX * sizeof(double2))));
        CK(cudaFuncSetAttribute(k_precond_solve2, cudaFuncAttributeMaxDynamicSharedMemorySize, 210 * 1024));
        CK(cudaFuncSetAttribute(k_precond_factor2, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
        plan_cluster_scans();
        d_wpart.alloc((size_t)8 * std::max(1, pcl_cs) * 2 * n_modes);
        if (mixed) setup_mixed(nsm);
    }

    // Tensor-core image of the Gaunt matrices, the tensor-core apply's plan, the fp32
    // cluster solve's plan and the complex64 work vectors of the mixed solve.
    void setup_mixed(int nsm)
    {
        if (pcl_per <= 0) throw Error(CNM_EINVAL, "The mixed solve needs the cluster preconditioner scans");
        tg = build_tc_gaunt(cpl);
        int amax = 0;
        for (int b : tg.l_bytes) amax = std::max(amax, b);
        tc_amax = amax;
        if (!tc_plan(n_modes, K, Nr, amax, nsm, tcp))
            throw Error(CNM_EINVAL, "The mixed solve supports at most 112 modes (l_max <= 13)");
        // TC_REPLICAS copies of the image (each 256-byte aligned); CTA b reads copy b % TC_REPLICAS
        tc_replica_bytes = (int64_t)((tg.blob.size() * 2 + 255) / 256 * 256);
        std::vector<uint8_t> bytes((size_t)tc_replica_bytes * TC_REPLICAS, 0);
        for (int rcp = 0; rcp < TC_REPLICAS; ++rcp)
            std::memcpy(bytes.data() + (size_t)rcp * tc_replica_bytes, tg.blob.data(), tg.blob.size() * 2);
        upload(d_tcblob, bytes);
        upload(d_tc_loff, tg.l_off);
        upload(d_tc_lbytes, tg.l_bytes);
        upload(d_tc_slices, tg.slices);
        upload(d_tc_lnblk, tg.l_nblk);
        d_tc_ctr.alloc(2);
        d_mx_ticket.alloc(1);
        CK(tc_prepare(tcp));
        for (DevBuf<float2> *b : {&m_r, &m_y, &m_v, &m_s, &m_z, &m_t, &m_d, &m_xa, &dinv32, &m_r1, &m_q}) b->alloc(nN);
        m_r64.alloc(nN);
        m_dots.alloc(8);
        d_msc.alloc(1);
        m_part.alloc((size_t)8 * std::max(vec_blocks, tcp.tiles));
        // fp32 cluster solve: the fp64 solve's CTAs per cluster, nodes per thread from it
        ps_cs = pcl_cs;
        ps_per = pcl_per;
        int optin = 0, dev = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        cudaFuncAttributes fa;
        CK(cudaFuncGetAttributes(&fa, k_psolve32_cl));
        CK(cudaFuncSetAttribute(k_psolve32_cl, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                optin - (int)fa.sharedSizeBytes));
        if (ps_cs > 8) CK(cudaFuncSetAttribute(k_psolve32_cl, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    }

    // Work plan of the operator kernel: for 1..8 CTA groups per 64-node tile, the LPT
    // warp lists (cnm::plan_coupling) and the resident CTAs per SM give an estimated
    // time  waves x heaviest warp list; the cheapest plan is kept.  A group's weights
    // are staged in shared memory when they fit beside the tile.
    void plan_operator(int nsm, int force_ng = 0)
    {
        int optin = 0, dev = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        cudaFuncAttributes fa;
        CK(cudaFuncGetAttributes(&fa, apply3_kernel(l_max, V_POT, true)));
        const int dyn_max = optin - (int)fa.sharedSizeBytes;
        CK(set_apply3_smem(dyn_max));
        const size_t base = (size_t)n_modes * (APPLY3_TILE + 1) * sizeof(double2) +
                            (size_t)std::max(K, 4) * APPLY3_TILE * sizeof(double);
        if (base > (size_t)dyn_max) throw Error(CNM_EINVAL, "Too many modes for the operator kernel's shared tile");
        const int tiles = (Nr + APPLY3_TILE - 1) / APPLY3_TILE;
        double best = 0.0;
        plan3 = CouplingPlan();
        for (int ng = 1; ng <= 8; ++ng) {
            if (force_ng > 0 && ng != force_ng) continue;
            CouplingPlan pl = plan_coupling(cpl, ng, APPLY_THREADS / 32);
            const size_t with_g = base + (size_t)pl.max_group_g * sizeof(double);
            const bool gsm = with_g <= (size_t)dyn_max;
            const size_t smem = gsm ? with_g : base;
            int occ = 0;
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, apply3_kernel(l_max, V_POT, gsm), APPLY_THREADS,
                                                             smem));
            if (occ < 1) continue;
            const int waves = (tiles * ng + occ * nsm - 1) / (occ * nsm);
            const double est = waves * pl.max_list_cost * (gsm ? 1.0 : 1.25);
            if (plan3.list_ptr.empty() || est < best) {
                best = est;
                plan3 = std::move(pl);
                apply3_gsm = gsm;
                apply3_smem = smem;
            }
        }
        if (plan3.list_ptr.empty()) throw Error(CNM_EINVAL, "No resident configuration of the operator kernel");
        // the diagnostics pass: the same tile (weights read through L1) and the per-row and
        // per-warp sums of its reductions
        diag3_smem = base + (size_t)(2 * n_modes + 3 * (APPLY_THREADS / 32)) * sizeof(double);
        if (diag3_smem > (size_t)dyn_max) throw Error(CNM_EINVAL, "Too many modes for the diagnostics pass's shared tile");
        // the attribute is shared by every handle of the process: the device's limit, not
        // this handle's size (a smaller value set by another handle would fail this one's launch)
        CK(set_diag3_smem(dyn_max));
        const BlockedCoupling &b = plan3.blocks;
        upload(d2_chunk_l, b.chunk_l);
        upload(d2_chunk_nrows, b.chunk_nrows);
        upload(d2_chunk_rows, b.chunk_rows);
        upload(d2_chunk_goff, b.chunk_goff);
        upload(d2_l_off, b.l_off);
        upload(d2_block_g, b.g);
        upload(d3_list_ptr, plan3.list_ptr);
        upload(d3_group_goff, plan3.group_goff);
    }

    // ------------------------------------------------------------ autotuner
    // Device-event time (ms per launch) of `reps` operator applications A x (no sinks, no
    // reductions) with the current plan, after one untimed launch.
    double time_operator(int reps)
    {
        ApplyArgs a = base_args(psi.p, tmp.p);
        a.alpha = cmake(1.0, 0.0);
        a.beta = cmake(0.0, 0.5 * op.dt);
        a.use_h0 = 1;
        a.use_cap = 1;
        a.vpart = V_POT;
        launch_apply(a);
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        CK(cudaEventRecord(e0, stream));
        for (int q = 0; q < reps; ++q) launch_apply(a);
        CK(cudaEventRecord(e1, stream));
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return ms / reps;
    }

    // The same for the tensor-core apply on the complex64 copy of psi.
    double time_tc(int reps)
    {
        k_to_f32<<<vec_blocks, VEC_THREADS, 0, stream>>>(nN, psi.p, m_xa.p);
        launch_check();
        TcArgs a = tc_a_args(m_xa.p, m_t.p, nullptr, 0, nullptr, op.dt);
        launch_tc(a);
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        CK(cudaEventRecord(e0, stream));
        for (int q = 0; q < reps; ++q) launch_tc(a);
        CK(cudaEventRecord(e1, stream));
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return ms / reps;
    }

    // Re-plans with the given choices (0 keeps the cost model's / the largest that fits).
    void set_tuning(int apply_groups, int tc_stages)
    {
        if (apply_groups < 0 || apply_groups > 8 || tc_stages < 0 || tc_stages > TC_MAX_STAGES)
            throw Error(CNM_EINVAL, "tuning choices out of range (row groups 0..8, stages 0..8)");
        plan_operator(n_sm, apply_groups);
        if (mixed) {
            TcPlan p;
            if (!tc_plan(n_modes, K, Nr, tc_amax, n_sm, p, tc_stages))
                throw Error(CNM_EINVAL, "no tensor-core plan with that many stages");
            tcp = p;
        }
    }

    // Timed search: every row-group count of the operator kernel that has a resident
    // configuration, then (mixed handles) every Gaunt-stage count of the tensor-core apply
    // from TC_MIN_STAGES to the most that fit; the fastest of each is kept.
    void autotune(int *apply_groups, int *tc_stages)
    {
        if (!initialized) throw Error(CNM_ELOGIC, "autotune needs an initialized solver (its operators and state)");
        sync();
        double best = 1e30;
        int best_ng = 0;
        for (int ng = 1; ng <= 8; ++ng) {
            try {
                plan_operator(n_sm, ng);
            } catch (const Error &) {
                continue;
            }
            const double ms = time_operator(5);
            if (ms < best) {
                best = ms;
                best_ng = ng;
            }
        }
        if (best_ng == 0) throw Error(CNM_EINVAL, "No resident configuration of the operator kernel");
        plan_operator(n_sm, best_ng);
        *apply_groups = best_ng;
        *tc_stages = 0;
        if (mixed) {
            TcPlan full;
            tc_plan(n_modes, K, Nr, tc_amax, n_sm, full);
            double bt = 1e30;
            int best_g = full.gst;
            for (int g = TC_MIN_STAGES; g <= full.gst; ++g) {
                TcPlan p;
                if (!tc_plan(n_modes, K, Nr, tc_amax, n_sm, p, g)) continue;
                tcp = p;
                const double ms = time_tc(5);
                if (ms < bt) {
                    bt = ms;
                    best_g = g;
                }
            }
            tc_plan(n_modes, K, Nr, tc_amax, n_sm, tcp, best_g);
            *tc_stages = best_g;
        }
        sync();
    }

    // Cluster plan of the exact preconditioner scans.  Candidates: every odd count of
    // nodes per thread whose cluster (CTAs per radial block) has at most 16 CTAs (more
    // than 8 only where the device allows non-portable clusters) and whose two staged
    // vectors fit the opt-in shared memory.  The plan minimises the estimated time
    //   rounds x per,  rounds = ceil(blocks / clusters resident at once),
    // so that, where possible, every radial block's cluster is resident in one round.
    void plan_cluster_scans()
    {
        pcl_per = pcl_cs = 0;
        int optin = 0, dev = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        bool nonportable = true;
        for (const void *kern : {(const void *)k_precond_solve_cl, (const void *)k_precond_factor_cl})
            if (cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
                cudaGetLastError();
                nonportable = false;
            }
        // dynamic shared memory may use what the kernels' static arrays leave of the opt-in limit
        cudaFuncAttributes fs, ff;
        CK(cudaFuncGetAttributes(&fs, k_precond_solve_cl));
        CK(cudaFuncGetAttributes(&ff, k_precond_factor_cl));
        const int dyn_max = optin - (int)std::max(fs.sharedSizeBytes, ff.sharedSizeBytes);
        CK(cudaFuncSetAttribute(k_precond_solve_cl, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_max));
        CK(cudaFuncSetAttribute(k_precond_factor_cl, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_max));
        const int cs_max = nonportable ? 16 : 8;
        double best = 0.0;
        for (int per = ((Nr + cs_max * PCL_THREADS - 1) / (cs_max * PCL_THREADS)) | 1;; per += 2) {
            const int cs = (Nr + PCL_THREADS * per - 1) / (PCL_THREADS * per);
            const size_t smem = (size_t)2 * PCL_THREADS * per * sizeof(double2);
            if (smem > (size_t)dyn_max) break;
            cudaLaunchConfig_t cfg = cluster_config(cs, n_modes, smem);
            cudaLaunchAttribute at;
            cluster_attr(at, cs);
            cfg.attrs = &at;
            int nclusters = 0;
            if (cudaOccupancyMaxActiveClusters(&nclusters, (const void *)k_precond_solve_cl, &cfg) != cudaSuccess ||
                nclusters < 1) {
                cudaGetLastError();
            } else {
                const double est = (double)((n_modes + nclusters - 1) / nclusters) * per;
                if (pcl_per == 0 || est < best) {
                    best = est;
                    pcl_per = per;
                    pcl_cs = cs;
                }
            }
            if (cs == 1) break;
        }
    }

    cudaLaunchConfig_t cluster_config(int cs, int blocks_y, size_t smem) const
    {
        cudaLaunchConfig_t cfg;
        std::memset(&cfg, 0, sizeof(cfg));
        cfg.gridDim = dim3((unsigned)cs, (unsigned)blocks_y, 1);
        cfg.blockDim = dim3(PCL_THREADS, 1, 1);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = stream;
        cfg.numAttrs = 1;
        return cfg;
    }

    // programmatic stream serialization (see launch_pdl)
    static void pdl_attr(cudaLaunchAttribute &at)
    {
        std::memset(&at, 0, sizeof(at));
        at.id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at.val.programmaticStreamSerializationAllowed = 1;
    }

    static void cluster_attr(cudaLaunchAttribute &at, int cs)
    {
        std::memset(&at, 0, sizeof(at));
        at.id = cudaLaunchAttributeClusterDimension;
        at.val.clusterDim.x = (unsigned)cs;
        at.val.clusterDim.y = 1;
        at.val.clusterDim.z = 1;
    }

    Grid grid() const
    {
        Grid g;
        g.Nr = Nr;
        g.n_modes = n_modes;
        g.dr = dr;
        g.mu = mu;
        g.r = d_r.p;
        g.capw = op.cap ? d_capw.p : nullptr;
        g.ir2 = d_ir2.p;
        return g;
    }

    CouplingTable table() const
    {
        CouplingTable c;
        c.n_modes = n_modes;
        c.l_max = l_max;
        c.n_pairs = (int)cpl.pair_col.size();
        c.n_terms = (int)cpl.term_l.size();
        c.pair_row_ptr = d_pair_row_ptr.p;
        c.pair_col = d_pair_col.p;
        c.pair_term_ptr = d_pair_term_ptr.p;
        c.term_l = d_term_l.p;
        c.term_g = d_term_g.p;
        c.diag_pair = d_diag_pair.p;
        c.mode_l = d_mode_l.p;
        c.mode_m = d_mode_m.p;
        return c;
    }

    BlockTable btable2() const
    {
        BlockTable b;
        b.n_chunks = plan3.blocks.n_chunks;
        b.chunk_l = d2_chunk_l.p;
        b.chunk_nrows = d2_chunk_nrows.p;
        b.chunk_rows = d2_chunk_rows.p;
        b.chunk_goff = d2_chunk_goff.p;
        b.l_off = d2_l_off.p;
        b.g = d2_block_g.p;
        return b;
    }

    ApplyPlan aplan() const
    {
        ApplyPlan p;
        p.list_ptr = d3_list_ptr.p;
        p.group_goff = d3_group_goff.p;
        return p;
    }

    void sync() { CK(cudaStreamSynchronize(stream)); }
    // kernels this handle has launched (counted at every launch site)
    int64_t n_launches = 0;
    void launch_check()
    {
        CK(cudaGetLastError());
        ++n_launches;
    }

    double ramp_end_time() const { return ramp_periods * initial_period; }

    // -------------------------------------------------------------- set-up API

    void set_initial_state_full(const double *h, int64_t n)
    {
        if (n != nN) throw Error(CNM_EINVAL, "Initial state size does not match the radial grid and modes");
        std::vector<double> tmp_h(h, h + 2 * n);
        const double sc = std::sqrt(M_c / mu);
        for (double &e : tmp_h) e *= sc;
        CK(cudaMemcpy(psi.p, tmp_h.data(), 2 * n * sizeof(double), cudaMemcpyHostToDevice));
    }

    void set_state(const double *h, int64_t n)
    {
        if (n != nN) throw Error(CNM_EINVAL, "state size does not match the radial grid and modes");
        CK(cudaMemcpy(psi.p, h, 2 * n * sizeof(double), cudaMemcpyHostToDevice));
    }

    void get_state(double *h, int64_t n) const
    {
        if (n != nN) throw Error(CNM_EINVAL, "state size does not match the radial grid and modes");
        CK(cudaMemcpy(h, psi.p, 2 * n * sizeof(double), cudaMemcpyDeviceToHost));
    }

    void configure_isolated_black_hole(double xbh)
    {
        if (!std::isfinite(xbh) || std::abs(xbh) >= L)
            throw Error(CNM_EINVAL, "The isolated BH must lie inside the radial domain");
        if (initialized) throw Error(CNM_ELOGIC, "Configure the isolated BH before initialize()");
        isolated = true;
        evolve_orbit = false;
        M1 = 1.0;
        M2 = q = 0.0;
        R = R1 = std::abs(xbh);
        R2 = 0.0;
        theta = xbh < 0.0 ? M_PI : 0.0;
        phase = 0.0;
        Omega = Omega_0 = 0.0;
        ramp_periods = 0.0;
    }

    void initialize()
    {
        abs1.valid = abs2.valid = false;
        t_i = 0.0;
        build_time_dependent_perturbation(0.0);
        ab_cap = op.cap;
        initialized = true;
    }

    void build_damping_mask(double fL, double W, int n)
    {
        mask = true;
        mask_h.assign(Nr, 1.0);
        const int idx = (int)std::floor(L * fL / dr);
        const double rm = fL * L, Lm = (1 - fL) * L;
        for (int i = 0; i < Nr; i++)
            if (i >= idx) mask_h[i] = std::exp(-W * std::pow((r[i] - rm) / Lm, n));
        upload(d_mask, mask_h);
    }

    void build_cap(double fL, double W, int n)
    {
        cap = true;
        capw_h.assign(Nr, 0.0);
        const int idx = (int)std::floor(L * fL / dr);
        const double rc = fL * L, Lc = (1 - fL) * L;
        for (int i = std::max(idx, 0); i < Nr; i++) capw_h[i] = W * std::pow((r[i] - rc) / (r[i] - Lc), n);
        upload(d_capw, capw_h);
    }

    // -------------------------------------------------------------- operators

    // hh table of the geometry frozen in `op` (set by build_time_dependent_perturbation).
    void build_hh(double *dst, double a1, double a2)
    {
        CK(launch_pdl(k_hh_table, (unsigned)((Nr + 255) / 256), 256, 0, stream, dst, d_r.p, Nr, K, op.R1, op.R2, op.q,
                                                                     -mu * op.Mtot, a1, a2));
        launch_check();
    }

    // src/CrankNicolsonModes_hamiltonian.cpp:245-268
    void build_time_dependent_perturbation(double time)
    {
        ramp_factor = 1.0;
        if (isolated) {
            Omega = 0.0;
        } else if (time < ramp_end_time()) {
            const double xr = time / ramp_end_time();
            ramp_factor = 3.0 * xr * xr - 2.0 * xr * xr * xr;
            Omega = Omega_0 * ramp_factor;
        } else {
            Omega = std::sqrt((M1 + M2) / std::pow(R, 3));
        }
        potential_ramp_factor = ramp_secondary_potential ? ramp_factor : 1.0;
        op.R1 = R1;
        op.R2 = R2;
        op.q = q;
        op.Mtot = M1 + M2;
        op.w = potential_ramp_factor;
        build_hh(d_hh.p, 1.0, potential_ramp_factor);
        if (absorption) build_spherical_absorption();
        sink_active = absorption && time >= ramp_end_time();
        op.built = true;
        op.theta = theta;
        op.domega = (counter ? -1.0 : 1.0) * Omega;
        op.dt = dt;
        op.cap = cap;
        op.sink_active = sink_active;
    }

    // src/CrankNicolsonModes_absorption.cpp:12-81: the support of a changed profile; true
    // when its moments must be computed (launch_moments)
    bool prepare_profile(Absorber &ab, double radius, double width)
    {
        if (ab.valid && ab.radius == radius && ab.width == width) return false;
        const int old_lo = ab.lo, old_hi = ab.hi;
        ab.radius = radius;
        ab.width = width;
        ab.valid = true;
        if (!ab.mom.p) {
            ab.mom.alloc((size_t)K * Nr);
            ab.v.alloc(nN);
        }
        ab.lo = ab.hi = 0;
        if (!(width < dr || width <= 0.0 || radius < 0.0)) {
            int lo = Nr, hi = 0;
            for (int i = 1; i < Nr - 1; ++i)
                if (std::abs(r[i] - radius) < width) {
                    lo = std::min(lo, i);
                    hi = std::max(hi, i + 1);
                }
            if (hi > lo) {
                ab.lo = lo;
                ab.hi = hi;
            }
        }
        ab.wlo = std::min(old_lo, ab.lo);
        ab.whi = std::max(old_hi, ab.hi);
        if (old_hi <= old_lo) {
            ab.wlo = ab.lo;
            ab.whi = ab.hi;
        } else if (ab.hi <= ab.lo) {
            ab.wlo = old_lo;
            ab.whi = old_hi;
        }
        if (ab.hi <= ab.lo) return false;
        const int nq = abs_nodes();
        if (gl_n != nq) {
            std::vector<double> gx, gw;
            gauss_legendre01(nq, gx, gw);
            upload(d_glx, gx);
            upload(d_glw, gw);
            gl_n = nq;
        }
        return true;
    }

    // Gauss-Legendre nodes of the angular quadrature and the moment kernels' CTA size
    // (one quadrature node per thread)
    int abs_nodes() const { return std::max(128, 2 * l_max + 16); }
    int abs_threads() const { return std::max(128, (abs_nodes() + 31) / 32 * 32); }

    static void add_absorber(AbsorberPair &ap, Absorber &ab, bool secondary)
    {
        const int c = ap.count++;
        ap.lo[c] = ab.lo;
        ap.hi[c] = ab.hi;
        ap.wlo[c] = ab.wlo;
        ap.whi[c] = ab.whi;
        ap.radius[c] = ab.radius;
        ap.width[c] = ab.width;
        ap.mom[c] = ab.mom.p;
        ap.v[c] = ab.v.p;
        ap.secondary[c] = secondary ? 1 : 0;
    }

    // moments of the changed profiles, one launch
    void launch_moments(bool m1, bool m2)
    {
        AbsorberPair ap;
        std::memset(&ap, 0, sizeof(ap));
        if (m1) add_absorber(ap, abs1, false);
        if (m2) add_absorber(ap, abs2, true);
        if (ap.count == 0) return;
        const int degree = 2 * l_max, threads = abs_threads();
        const unsigned blocks = (unsigned)((ap.hi[0] - ap.lo[0]) + (ap.count > 1 ? ap.hi[1] - ap.lo[1] : 0));
        CK(launch_pdl(k_abs_moments, blocks, threads, (size_t)(degree + 1) * (threads / 32) * sizeof(double), stream, 
            d_r.p, Nr, abs_nodes(), d_glx.p, d_glw.p, degree, ap));
        launch_check();
    }

    // both projectors, one launch; nodes of a previous support are rewritten (as zero)
    void build_projectors()
    {
        AbsorberPair ap;
        std::memset(&ap, 0, sizeof(ap));
        int64_t work = 0;
        for (int a = 0; a < 2; ++a) {
            Absorber &ab = a == 0 ? abs1 : abs2;
            const int lo = ab.wlo, hi = ab.whi;
            if (hi <= lo) continue;
            if (ab.hi > ab.lo) {
                add_absorber(ap, ab, a == 1);
                work += (int64_t)(hi - lo) * n_modes;
            } else {
                for (int j = 0; j < n_modes; ++j)
                    CK(cudaMemsetAsync(ab.v.p + (int64_t)j * Nr + lo, 0, (size_t)(hi - lo) * sizeof(double2), stream));
            }
            ab.wlo = ab.lo;
            ab.whi = ab.hi;
        }
        if (ap.count == 0) return;
        const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(1024, (work + 255) / 256));
        CK(launch_pdl(k_swave_projector, blocks, 256, 0, stream, d_r.p, Nr, n_modes, dr, d_ang00.p, d_mode_l.p, d_mode_m.p, theta,
                                                       ap));
        launch_check();
    }

    // src/CrankNicolsonModes_absorption.cpp:153-182
    void build_spherical_absorption()
    {
        const bool m1 = prepare_profile(abs1, R1, epsilon_smear * M1);
        const bool m2 = prepare_profile(abs2, R2, epsilon_smear * M2);
        launch_moments(m1, m2);
        double ramp = 1.0;
        if (!isolated && t_i < ramp_end_time()) {
            ramp = 0.0;
        } else if (!isolated && t_i < ramp_end_time() + initial_period) {
            const double xr = (t_i - ramp_end_time()) / initial_period;
            ramp = 3.0 * xr * xr - 2.0 * xr * xr * xr;
        }
        const double Ah1 = 16.0 * M_PI * M1 * M1 * ramp;
        const double Ah2 = 16.0 * M_PI * M2 * M2 * ramp;
        if (cpl.mode00 >= 0) build_projectors();
        abs1.strength = Ah1 * dr;
        abs2.strength = Ah2 * dr;
    }

    // Sinks that enter the CN operator: active, non-zero strength, non-empty projector
    // (src/CrankNicolsonModes_matrices.cpp:106-110).
    int active_sinks(const Absorber *out[2]) const
    {
        int k = 0;
        if (!op.sink_active || cpl.mode00 < 0) return 0;
        for (const Absorber *ab : {&abs1, &abs2})
            if (ab->strength != 0.0 && ab->hi > ab->lo) out[k++] = ab;
        return k;
    }

    int sink_slot(const Absorber *ab) const { return ab == &abs1 ? 0 : 1; }

    void sink_dots(const double2 *xv, double2 *dots, const Absorber *const *sk, int k, int gate_mode = GATE_NONE)
    {
        CK(launch_pdl(k_sink_dots, 1, 1024, 0, stream, xv, Nr, n_modes, k, k > 0 ? sk[0]->v.p : nullptr,
                                           k > 1 ? sk[1]->v.p : nullptr, k > 0 ? sk[0]->lo : 0,
                                           k > 0 ? sk[0]->hi : 0, k > 1 ? sk[1]->lo : 0, k > 1 ? sk[1]->hi : 0, dots,
                                           gate_mode == GATE_NONE ? nullptr : d_kr.p, gate_mode));
        launch_check();
    }

    // The same for a complex64 vector (the mixed solve's inner iterations; k >= 1).
    void sink_dots32(const float2 *xv, double2 *dots, const Absorber *const *sk, int k)
    {
        k_sink_dots32<<<1, 1024, 0, stream>>>(xv, Nr, n_modes, k, sk[0]->v.p, k > 1 ? sk[1]->v.p : nullptr, sk[0]->lo,
                                             sk[0]->hi, k > 1 ? sk[1]->lo : 0, k > 1 ? sk[1]->hi : 0, dots);
        launch_check();
    }

    ApplyArgs base_args(const double2 *xv, double2 *yv) const
    {
        ApplyArgs a;
        std::memset(&a, 0, sizeof(a));
        a.x = xv;
        a.y = yv;
        a.hh = d_hh.p;
        a.theta = op.theta;
        a.domega = op.domega;
        a.stage = -1;
        a.dot_scale = 1.0;
        a.gate = nullptr;
        a.gate_mode = GATE_NONE;
        a.scale_kr = nullptr;
        return a;
    }

    // Operator kernel grid: 64-node tiles x the plan's CTA groups.
    dim3 apply3_grid() const
    {
        return dim3((unsigned)((Nr + APPLY3_TILE - 1) / APPLY3_TILE), (unsigned)plan3.n_groups);
    }

    bool use_apply5(const ApplyArgs &a) const { return a5_groups > 0 && a5_enabled && a.vpart == V_POT; }

    void launch_apply(const ApplyArgs &a)
    {
        if (use_apply5(a)) {
            kt_begin(TK_APPLY);
            ::cnm::launch_apply5(l_max, stream, grid(), d_a5tab.p, a);
            launch_check();
            kt_end(TK_APPLY);
            return;
        }
        const dim3 blocks3 = apply3_grid();
        kt_begin(TK_APPLY);
        ::cnm::launch_apply3(l_max, apply3_gsm, blocks3, apply3_smem, stream, grid(), table(), btable2(), aplan(), a);
        launch_check();
        kt_end(TK_APPLY);
    }

    // y = A_full x (sparse CN operator plus dt/4 Gamma) with the sink projections of x at `dots`;
    // optionally with up to two inner products of y (ApplyArgs::dot_kind) reduced into
    // per-CTA partials.
    void apply_A(const double2 *xv, double2 *yv, const Absorber *const *sk, int k, const double2 *dots, double dtv,
                 const DotSpec &ds = DotSpec())
    {
        ApplyArgs a = base_args(xv, yv);
        a.n_dots = ds.n;
        a.dot_kind[0] = ds.kind[0];
        a.dot_kind[1] = ds.kind[1];
        a.dot_ext[0] = ds.ext[0];
        a.dot_ext[1] = ds.ext[1];
        a.dot_scale = ds.scale;
        a.dot_partials = d_partials.p;
        set_finish(a, ds);
        a.alpha = cmake(1.0, 0.0);
        a.beta = cmake(0.0, 0.5 * dtv);
        a.use_h0 = 1;
        a.use_cap = 1;
        a.vpart = V_POT;
        a.n_sinks = k;
        a.sink_dots = dots;
        for (int i = 0; i < k; ++i) {
            a.sink_v[i] = sk[i]->v.p;
            a.sink_coef[i] = 0.25 * dtv * sk[i]->strength;
            a.sink_lo[i] = sk[i]->lo;
            a.sink_hi[i] = sk[i]->hi;
        }
        launch_apply(a);
    }

    void set_finish(ApplyArgs &a, const DotSpec &ds)
    {
        a.stage = ds.n > 0 ? ds.stage : -1;
        a.kr = d_kr.p;
        a.ticket = ticket(TK_APPLY_T);
        a.red = ds.red ? ds.red : d_red.p;
        a.gate = ds.gate_mode != GATE_NONE ? d_kr.p : nullptr;
        a.gate_mode = ds.gate_mode;
        a.scale_kr = ds.scale_from_kr ? d_kr.p : nullptr;
    }

    unsigned *ticket(int which) const { return d_tickets.p + which; }

    // -------------------------------------------------------------- preconditioner

    double2 offdiag(double dtv) const
    {
        // A's radial off-diagonal: i dt/2 * (-1/(2 mu dr^2))
        const double alpha_d = 1.0 / (dr * dr);
        return cmake(0.0, 0.5 * dtv * (-alpha_d / (2 * mu)));
    }

    // Warm-up window of the chunked scans: the recurrences contract by rho = |off| / |p+|
    // per node, p+ the attracting pivot of a block whose diagonal sits 1% below the
    // free one.  The window forgets the chunk's start value to exp(-40).
    // Largest |Ahat_jj(r)| over modes and interior nodes for the frozen geometry:
    // |h_l*(r)| <= mu (M1+M2) [1/((1+q) max(r,R1)) + |w| q/((1+q) max(r,R2))] and
    // |Ahat_jj| <= (sum_l* |g_jjl*|) max_l* |h_l*|.
    double diag_potential_bound() const
    {
        double gsum = 0.0;
        for (int j = 0; j < n_modes; ++j) {
            const int p = cpl.diag_pair[j];
            double s2 = 0.0;
            if (p >= 0)
                for (int t = cpl.pair_term_ptr[p]; t < cpl.pair_term_ptr[p + 1]; ++t) s2 += std::abs(cpl.term_g[t]);
            gsum = std::max(gsum, s2);
        }
        const double r1 = std::max(r[1], 1e-300);
        const double h = mu * op.Mtot * (1.0 / ((1 + op.q) * std::max(r1, op.R1)) +
                                         std::abs(op.w) * op.q / ((1 + op.q) * std::max(r1, op.R2)));
        return gsum * h;
    }

    void choose_window(double dtv)
    {
        const double kappa = std::abs(offdiag(dtv).y);
        // the potential can only lower the imaginary part of the diagonal 2 kappa (1 + ...)
        // by (dt/2) |Ahat_jj|; CAP and centrifugal terms only strengthen the decay
        const double depress = std::min(0.5, 0.5 * dtv * diag_potential_bound() / (2.0 * kappa));
        const std::complex<double> a(1.0, 2.0 * kappa * (1.0 - depress)), c(-kappa * kappa, 0.0);
        const std::complex<double> sq = std::sqrt(a * a - 4.0 * c);
        const double pp = std::max(std::abs((a + sq) * 0.5), std::abs((a - sq) * 0.5));
        const double rho = kappa / pp;
        int w = rho < 1.0 ? (int)std::ceil(40.0 / -std::log(rho)) + 16 : 4096;
        precond_chunk = 2048;
        // two staged solve CTAs per SM: (chunk + 2 window) * 32 bytes <= 96 KiB where possible
        precond_window = std::max(32, std::min((6720 - precond_chunk) / 2, w));
    }

    void factorize(double dtv)
    {
        pivots32 = false;
        CK(cudaMemsetAsync(d_status.p, 0, sizeof(int), stream));
        if (jacobi) {
            k_jacobi_diag<<<vec_blocks, VEC_THREADS, 0, stream>>>(grid(), table(), d_hh.p, 0.5 * dtv, dinv.p);
            launch_check();
            return;
        }
        if (pcl_per > 0) {
            const size_t smem = (size_t)PCL_THREADS * pcl_per * sizeof(double2);
            cudaLaunchConfig_t cfg = cluster_config(pcl_cs, n_modes, smem);
            cudaLaunchAttribute at[2];
            cluster_attr(at[0], pcl_cs);
            pdl_attr(at[1]);
            cfg.attrs = at;
            cfg.numAttrs = 2;
            kt_begin(TK_PFACTOR);
            ++n_launches;
            float2 *const d32 = mixed ? dinv32.p : nullptr;
            CK(cudaLaunchKernelEx(&cfg, k_precond_factor_cl, grid(), table(), (const double *)d_hh.p, 0.5 * dtv,
                                  offdiag(dtv), pcl_per, dinv.p, d32, d_status.p));
            kt_end(TK_PFACTOR);
            pivots32 = d32 != nullptr;
            return;
        }
        choose_window(dtv);
        const int chunks = (Nr + precond_chunk - 1) / precond_chunk;
        const int fwin = precond_window / 2 + 16;
        const size_t smem = (size_t)std::min(Nr, precond_chunk + fwin) * sizeof(double2);
        kt_begin(TK_PFACTOR);
        k_precond_factor2<<<dim3(chunks, n_modes), SCAN2_THREADS, smem, stream>>>(
            grid(), table(), d_hh.p, 0.5 * dtv, offdiag(dtv), precond_chunk, fwin, dinv.p, d_status.p);
        launch_check();
        kt_end(TK_PFACTOR);
    }

    unsigned apply_blocks() const { return apply3_grid().x * apply3_grid().y; }

    void precond(const double2 *bv, double2 *xv, double dtv, PrecondInput in = PrecondInput{PI_PLAIN, nullptr,
                                                                                             nullptr, nullptr,
                                                                                             nullptr, nullptr})
    {
        if (jacobi) {
            k_jacobi_apply<<<vec_blocks, VEC_THREADS, 0, stream>>>(nN, dinv.p, bv, xv, in);
            launch_check();
            return;
        }
        if (pcl_per > 0) {
            precond_cl(bv, xv, nullptr, nullptr, dtv, in);
            return;
        }
        const int chunks = (Nr + precond_chunk - 1) / precond_chunk;
        const size_t smem = (size_t)2 * std::min(Nr, precond_chunk + 2 * precond_window) * sizeof(double2);
        kt_begin(TK_PSOLVE);
        k_precond_solve2<<<dim3(chunks, n_modes), SCAN2_THREADS, smem, stream>>>(Nr, precond_chunk, precond_window,
                                                                                offdiag(dtv), dinv.p, bv, xv, in);
        launch_check();
        kt_end(TK_PSOLVE);
    }

    // Exact cluster solve; with b2/x2 set the launch solves both right-hand sides.
    void precond_cl(const double2 *bv, double2 *xv, const double2 *b2, double2 *x2, double dtv, PrecondInput in,
                    WoodArgs wd = WoodArgs{WD_NONE, 0, 0, nullptr, nullptr, 0, 0, 0, 0, 0.0, 0.0, nullptr, nullptr,
                                           nullptr})
    {
        const size_t smem = (size_t)2 * PCL_THREADS * pcl_per * sizeof(double2);
        in.fault = d_status.p;
        cudaLaunchConfig_t cfg = cluster_config(pcl_cs, b2 ? 2 * n_modes : n_modes, smem);
        cudaLaunchAttribute at[2];
        cluster_attr(at[0], pcl_cs);
        pdl_attr(at[1]);
        cfg.attrs = at;
        cfg.numAttrs = 2;
        kt_begin(TK_PSOLVE);
        ++n_launches;
        CK(cudaLaunchKernelEx(&cfg, k_precond_solve_cl, Nr, n_modes, pcl_per, offdiag(dtv), (const double2 *)dinv.p,
                              bv, xv, b2, x2, in, wd));
        kt_end(TK_PSOLVE);
    }

    // -------------------------------------------------------------- reductions

    // red[0..2*nq-1] = sum conj(a_q) b_q (re, im pairs), synchronous read if `host`.
    void dots(int nq, const double2 *a0, const double2 *b0, const double2 *a1 = nullptr, const double2 *b1 = nullptr,
              const double2 *a2 = nullptr, const double2 *b2 = nullptr)
    {
        k_dots<<<vec_blocks, VEC_THREADS, 0, stream>>>(nN, nq, a0, b0, a1, b1, a2, b2, d_partials.p);
        launch_check();
        k_sum_partials<<<1, 512, 0, stream>>>(d_partials.p, vec_blocks, 2 * nq, d_red.p);
        launch_check();
    }

    double read_red(int idx)
    {
        double vv = 0;
        CK(cudaMemcpyAsync(&vv, d_red.p + idx, sizeof(double), cudaMemcpyDeviceToHost, stream));
        sync();
        return vv;
    }

    void axpby(double2 al, const double2 *xv, double2 be, const double2 *wv, double2 *yv)
    {
        k_axpby<<<vec_blocks, VEC_THREADS, 0, stream>>>(nN, al, xv, be, wv, yv);
        launch_check();
    }

    // -------------------------------------------------------------- CN solve

    // src/CrankNicolsonModes_matrices.cpp:94-215 with the radial block preconditioner.
    // Scalars live on the device (Krylov): every launch that produces a reduction
    // finishes the matching scalar stage in its last CTA, so an iteration is seven
    // launches (five without sinks) and one host synchronisation (convergence and
    // restart test).  |rhs|^2 is left in red[RED_RHS] by the right-hand-side apply.
    // The diagnostics pass of the accepted end-of-step state with the step's operators
    // (src/CrankNicolsonModes_extraction.cpp), gated on the candidate's acceptance:
    // the sink projections of the new state, the fused pass and the sums of its slots.
    void enqueue_diagnostics(const Absorber *const *sk, int k, const double2 *state = nullptr)
    {
        const double2 *st = state ? state : psi.p;
        const Absorber *all[2] = {&abs1, &abs2};
        const bool have_sinks = absorption && cpl.mode00 >= 0;
        if (have_sinks) sink_dots(st, d_dots.p + 4, all, 2, GATE_ACCEPTED);
        unsigned dblocks = 0;
        kt_begin(TK_DIAG);
        DiagArgs da;
        da.hh = d_hh.p;
        da.theta = op.theta;
        da.domega = op.domega;
        da.psi = st;
        da.idx_ex = idx_ex;
        da.n_sinks = k;
        da.sv0 = k > 0 ? sk[0]->v.p : nullptr;
        da.sv1 = k > 1 ? sk[1]->v.p : nullptr;
        da.sink_dots = k > 0 ? d_dots.p + 4 + sink_slot(sk[0]) : d_dots.p;
        da.sink_coef0 = k > 0 ? -0.5 * sk[0]->strength : 0.0;
        da.sink_coef1 = k > 1 ? -0.5 * sk[1]->strength : 0.0;
        da.slo0 = k > 0 ? sk[0]->lo : 0;
        da.shi0 = k > 0 ? sk[0]->hi : 0;
        da.slo1 = k > 1 ? sk[1]->lo : 0;
        da.shi1 = k > 1 ? sk[1]->hi : 0;
        da.partials = d_partials.p;
        da.dpsi_edge = d_edge.p;
        da.psi_edge = d_edge.p + n_modes;
        da.gate = d_kr.p;
        if (a5_groups > 0 && a5_enabled) {
            dblocks = ::cnm::launch_diag5(l_max, stream, grid(), d_d5tab.p, da);
        } else {
            const dim3 dgrid((unsigned)(std::min(idx_ex, Nr - 1) / APPLY3_TILE + 1), (unsigned)plan3.n_groups);
            ::cnm::launch_diag3(l_max, dgrid, diag3_smem, stream, grid(), table(), btable2(), aplan(), da);
            dblocks = dgrid.x * dgrid.y;
        }
        launch_check();
        kt_end(TK_DIAG);
        const int nslots = 2 * n_modes + 3;
        CK(launch_pdl(k_sum_slots, nslots, 256, 0, stream, d_partials.p, (int)dblocks, nslots, d_red.p, d_kr.p));
        launch_check();
    }

    // One BiCGSTAB iteration (src/CrankNicolsonModes_matrices.cpp:47-91), every launch
    // gated on the device (skipped once the solve is done or must restart), so several
    // can be queued ahead of the host's convergence test.
    void enqueue_iteration(const Absorber *const *sk, int k, double dtv, bool first)
    {
        Krylov *dk = d_kr.p;
        // p = r + beta (p - omega v) formed inside the preconditioner pass; y = M p
        precond_M(PrecondInput{PI_P, dk, rr.p, p.p, v.p, nullptr, p2.p, first ? 1 : 0, GATE_ITER}, 0, sk, k, dtv,
                  y.p);
        // v = A y with r0 . v reduced in the same pass; alpha = rho / r0.v
        {
            DotSpec ds;
            ds.n = 1;
            ds.kind[0] = 1;
            ds.ext[0] = r0.p;
            ds.stage = KS_ALPHA;
            ds.gate_mode = GATE_ITER;
            apply_A(y.p, v.p, sk, k, reinterpret_cast<const double2 *>(&dk->sdots[0][0]), dtv, ds);
        }
        // s = r - alpha v formed inside the preconditioner pass; z = M s
        precond_M(PrecondInput{PI_S, dk, rr.p, nullptr, v.p, s.p, nullptr, 0, GATE_ITER}, 1, sk, k, dtv, z.p);
        // t = A z with t . s and |t|^2 reduced in the same pass; omega = t.s / |t|^2
        {
            DotSpec ds;
            ds.n = 2;
            ds.kind[0] = 2;
            ds.ext[0] = s.p;
            ds.kind[1] = 3;
            ds.stage = KS_OMEGA;
            ds.gate_mode = GATE_ITER;
            apply_A(z.p, t.p, sk, k, reinterpret_cast<const double2 *>(&dk->sdots[1][0]), dtv, ds);
        }
        // x += alpha y + omega z; r = s - omega t; then KS_UPDATE and the next beta
        CK(launch_pdl(k_bicg_update, vec_blocks, VEC_THREADS, 0, stream, nN, dk, x.p, y.p, z.p, rr.p, s.p, t.p, r0.p,
                                                               d_partials.p, d_red.p, ticket(TK_UPDATE_T)));
        launch_check();
    }

    // Read-backs of a step, in the pinned stage: the Krylov scalars, the diagnostics'
    // 2 n + 3 sums, psi and dpsi/dt around the extraction node, the sink projections.
    size_t readback_doubles() const
    {
        return (sizeof(Krylov) + 7) / 8 + (size_t)(2 * n_modes + 3) + 8 * (size_t)n_modes + 16 +
               (sizeof(MixScalars) + 7) / 8;
    }

    // -------------------------------------------------------------- mixed precision

    TcTable tc_table() const
    {
        TcTable t;
        t.blob = d_tcblob.p;
        t.l_off = d_tc_loff.p;
        t.l_bytes = d_tc_lbytes.p;
        t.slices = d_tc_slices.p;
        t.l_nblk = d_tc_lnblk.p;
        t.g_exp = tg.g_exp;
        t.replicas = TC_REPLICAS;
        t.replica_bytes = tc_replica_bytes;
        return t;
    }

    // y = A_full x on complex64 vectors (tensor-core coupling): alpha = 1, beta = i dt/2,
    // the sinks with their projections at `dots`; up to three fused reductions.
    TcArgs tc_a_args(const float2 *xv, float2 *yv, const Absorber *const *sk, int k, const double2 *dots, double dtv)
    {
        TcArgs a;
        std::memset(&a, 0, sizeof(a));
        a.x = xv;
        a.y = yv;
        a.alpha = make_float2(1.f, 0.f);
        a.beta = make_float2(0.f, (float)(0.5 * dtv));
        a.use_h0 = 1;
        a.use_cap = 1;
        a.use_v = 1;
        a.hh = d_hh.p;
        a.theta = (float)op.theta;
        a.n_sinks = k;
        a.sink_dots = dots;
        for (int i = 0; i < k; ++i) {
            a.sink_v[i] = sk[i]->v.p;
            a.sink_coef[i] = (float)(0.25 * dtv * sk[i]->strength);
            a.sink_lo[i] = sk[i]->lo;
            a.sink_hi[i] = sk[i]->hi;
        }
        a.partials = m_part.p;
        a.status = d_status.p;
        a.tile_ctr = d_tc_ctr.p;
        a.mx_stage = -1;
        a.msc = d_msc.p;
        return a;
    }

    void launch_tc(const TcArgs &a)
    {
        kt_begin(TK_TC);
        ++n_launches;
        CK(launch_tc_apply(tcp, stream, grid(), d_mode_l.p, d_mode_m.p, K, tc_table(), a));
        kt_end(TK_TC);
    }

    // the last-block scalar stage of a mixed-solve vector kernel
    MxFinish mxf(int stage)
    {
        MxFinish f;
        f.sc = d_msc.p;
        f.stage = stage;
        f.ticket = d_mx_ticket.p;
        return f;
    }


    // out = P32^{-1} in (mode 0); mode 1: s = r - alpha v formed and stored to s_out,
    // out = P32^{-1} s; mode 2: out = P32^{-1} (r + beta (r0 - omega v)) with r0 = m_r
    void psolve32(int mode, const float2 *in, float2 *out, const float2 *r = nullptr, float2 *s_out = nullptr)
    {
        Ps32Args a;
        std::memset(&a, 0, sizeof(a));
        a.mode = mode;
        a.b = in;
        a.r = r ? r : m_r.p;
        a.v = m_v.p;
        a.r0 = m_r.p;
        a.s_out = s_out ? s_out : m_s.p;
        a.sc = d_msc.p;
        a.status = d_status.p;
        cudaLaunchConfig_t cfg;
        std::memset(&cfg, 0, sizeof(cfg));
        cfg.gridDim = dim3((unsigned)ps_cs, (unsigned)n_modes, 1);
        cfg.blockDim = dim3(PS32_THREADS, 1, 1);
        cfg.dynamicSmemBytes = (size_t)2 * PS32_THREADS * ps_per * sizeof(float2);
        cfg.stream = stream;
        cudaLaunchAttribute at[1];
        cluster_attr(at[0], ps_cs);
        cfg.attrs = at;
        cfg.numAttrs = 1;
        const double2 o = offdiag(op.dt);
        kt_begin(TK_PSOLVE32);
        ++n_launches;
        CK(cudaLaunchKernelEx(&cfg, k_psolve32_cl, Nr, ps_per, make_float2((float)o.x, (float)o.y),
                              (const float2 *)dinv32.p, out, a));
        kt_end(TK_PSOLVE32);
    }

    // One defect-correction pass on the current residual m_r (complex64): `iters`
    // right-preconditioned BiCGSTAB iterations from d = 0 (_matrices.cpp:47-91 with the
    // shadow residual r0 = r, rho0 = |r|^2, p = r):
    //   y = M p, v = A y, alpha = rho / r0.v, s = r - alpha v, z = M s, t = A z,
    //   omega = t.s / |t|^2, d += alpha y + omega z,
    // then r1 = s - omega t, rho1 = r0.r1, beta = (rho1 / rho0)(alpha / omega) and
    // p = r1 + beta (r0 - omega v) for the second iteration; x += d (exactly) at the end.
    void mixed_pass(const Absorber *const *sk, int k, double dtv, int iters)
    {
        for (int q = 0; q < iters; ++q) {
            const bool first = q == 0, last = q + 1 == iters;
            if (first) psolve32(0, m_r.p, m_y.p);
            else psolve32(2, nullptr, m_y.p, m_r1.p);
            wood32(sk, k, m_y.p);
            {
                TcArgs a = tc_a_args(m_y.p, m_v.p, sk, k, m_dots.p + 2, dtv);
                a.n_dots = 1;
                a.dot_kind[0] = 1;
                a.dot_ext[0] = m_r.p;  // r0
                a.mx_stage = first ? MX_ALPHA : MX_ALPHA2;
                launch_tc(a);
            }
            psolve32(1, nullptr, m_z.p, first ? m_r.p : m_r1.p, first ? m_s.p : m_q.p);
            wood32(sk, k, m_z.p);
            {
                TcArgs a = tc_a_args(m_z.p, m_t.p, sk, k, m_dots.p + 2, dtv);
                a.n_dots = 2;
                a.dot_kind[0] = 2;
                a.dot_ext[0] = first ? m_s.p : m_q.p;
                a.dot_kind[1] = 3;
                a.mx_stage = MX_OMEGA;
                launch_tc(a);
            }
            k_mx_update<<<vec_blocks, VEC_THREADS, 0, stream>>>(nN, d_msc.p, x.p, m_y.p, m_z.p, m_d.p, first ? 1 : 0,
                                                                last ? 1 : 0, m_part.p, mxf(last ? MX_D2 : -1));
            launch_check();
            if (!last) {
                k_mx_next<<<vec_blocks, VEC_THREADS, 0, stream>>>(nN, d_msc.p, m_s.p, m_t.p, m_r.p, m_r1.p, m_part.p,
                                                                  mxf(MX_BETA));
                launch_check();
            }
        }
        ++mx_passes;
    }

    // fp64 residual of x: r64 = rhs - A_full x (fp64 operator), r = r64 in complex64.
    void mixed_resid64(const Absorber *const *sk, int k, double dtv, double2 *diff = nullptr)
    {
        sink_dots(x.p, d_dots.p, sk, k);
        apply_A(x.p, tmp.p, sk, k, d_dots.p, dtv);
        k_mx_resid<<<vec_blocks, VEC_THREADS, 0, stream>>>(nN, rhs.p, tmp.p, m_r64.p, diff, m_r.p, m_part.p,
                                                           mxf(MX_R64));
        launch_check();
        ++mx_fp64;
    }

    // Residual of x = x_prev + d from the tensor-core operator: |r64 - A_full d|^2, where
    // r64 is the fp64 residual of x_prev (valid when |d| is small, see mixed_check_bound).
    void mixed_resid_tc(const Absorber *const *sk, int k, double dtv)
    {
        if (k > 0) {
            sink_dots32(m_d.p, m_dots.p + 4, sk, k);
        }
        TcArgs a = tc_a_args(m_d.p, m_t.p, sk, k, m_dots.p + 4, dtv);
        a.n_dots = 1;
        a.dot_kind[0] = 4;
        a.dot_ext64 = m_r64.p;
        a.mx_stage = MX_TCRES;
        launch_tc(a);
    }

    // Calibration of the tensor-core residual check on the pass just verified in fp64:
    // |(r_before - r_after) - A_tc d|^2 with d the pass's correction (m_d) and the fp64
    // change of the residual in cand.
    void mixed_calibrate(const Absorber *const *sk, int k, double dtv)
    {
        if (k > 0) {
            sink_dots32(m_d.p, m_dots.p + 4, sk, k);
        }
        TcArgs a = tc_a_args(m_d.p, m_t.p, sk, k, m_dots.p + 4, dtv);
        a.n_dots = 1;
        a.dot_kind[0] = 4;
        a.dot_ext64 = cand.p;
        a.mx_stage = MX_ECAL;
        launch_tc(a);
    }

    // psi candidate = mask x into cand, the diagnostics pass on it, the read-backs (the
    // Krylov struct's slot, the diagnostics sums, the edge values, the sink projections,
    // then the inner scalars).
    void mixed_tail(const Absorber *const *sk, int k, double *hs)
    {
        CK(launch_pdl(k_scale_mask, vec_blocks, VEC_THREADS, 0, stream, nN, Nr, 1.0, mask ? d_mask.p : nullptr,
                      (const double2 *)x.p, cand.p, (const Krylov *)nullptr));
        launch_check();
        enqueue_diagnostics(sk, k, cand.p);
        const size_t kd = (sizeof(Krylov) + 7) / 8;
        const int nslots = 2 * n_modes + 3;
        CK(cudaMemcpyAsync(hs, d_kr.p, sizeof(Krylov), cudaMemcpyDeviceToHost, stream));
        CK(cudaMemcpyAsync(hs + kd, d_red.p, nslots * sizeof(double), cudaMemcpyDeviceToHost, stream));
        CK(cudaMemcpyAsync(hs + kd + nslots, d_edge.p, 4 * n_modes * sizeof(double2), cudaMemcpyDeviceToHost,
                           stream));
        CK(cudaMemcpyAsync(hs + kd + nslots + 8 * n_modes, d_dots.p, 8 * sizeof(double2), cudaMemcpyDeviceToHost,
                           stream));
        CK(cudaMemcpyAsync(hs + kd + nslots + 8 * n_modes + 16, d_msc.p, sizeof(MixScalars), cudaMemcpyDeviceToHost,
                           stream));
    }

    MixScalars mixed_scalars(const double *hs) const
    {
        MixScalars m;
        const size_t kd = (sizeof(Krylov) + 7) / 8;
        std::memcpy(&m, hs + kd + (2 * n_modes + 3) + 8 * n_modes + 16, sizeof(m));
        return m;
    }

    // The mixed solve of one step, queued without waiting: rhs is in place (fp64 rhs
    // apply); pivots (fp64, then fp32 copies), Woodbury set-up, r0 = 2 (rhs - psi), pass 1,
    // the fp64 residual and the calibration of the tensor-core check, pass 2, the
    // tensor-core residual check, and the tail.
    void begin_mixed(const Absorber *const *sk, int k, double *hs)
    {
        const double dtv = op.dt;
        mx_passes = 0;
        mx_fp64 = 1;  // the right-hand side
        Krylov kr;
        std::memset(&kr, 0, sizeof(kr));
        kr.n_sinks = k;
        kr.accepted = 1;  // gates of the diagnostics pass: the host decides acceptance
        kr.rhs_norm = 1.0;
        kr.status = d_status.p;
        h_kr_init = kr;
        CK(cudaMemcpyAsync(d_kr.p, &h_kr_init, sizeof(kr), cudaMemcpyHostToDevice, stream));
        jacobi = false;
        factorize(dtv);
        if (!pivots32) {
            k_to_f32<<<vec_blocks, VEC_THREADS, 0, stream>>>(nN, dinv.p, dinv32.p);
            launch_check();
        }
        if (k > 0) wood_setup(sk, k, dtv);
        k_mx_start<<<vec_blocks, VEC_THREADS, 0, stream>>>(nN, rhs.p, psi.p, x.p, m_r64.p, m_r.p, m_part.p,
                                                           mxf(MX_B2R0));
        launch_check();
        mixed_pass(sk, k, dtv, 1);
        mixed_resid64(sk, k, dtv, cand.p);
        mixed_calibrate(sk, k, dtv);
        mixed_pass(sk, k, dtv, 2);
        mixed_resid_tc(sk, k, dtv);
        mixed_tail(sk, k, hs);
    }

    // Waits for the queued mixed solve and decides: accepted when the tensor-core residual
    // plus four times its calibrated error is within `tolerance`; when only the error
    // estimate is too large, an fp64 residual decides; otherwise further passes (fp64
    // residual, pass, tensor-core check) up to mixed_max_passes.  A solve that still misses
    // `tolerance` is accepted at accept_residual, else the step is redone by the fp64 solve.
    void finish_mixed(const Absorber *const *sk, int k, double *hs)
    {
        const double dtv = op.dt;
        for (;;) {
            sync();
            int st = 0;
            CK(cudaMemcpy(&st, d_status.p, sizeof(int), cudaMemcpyDeviceToHost));
            const MixScalars m = mixed_scalars(hs);
            const double bn = std::sqrt(std::max(m.b2, 1e-300));
            const double res_tc = std::sqrt(m.tc_res2) / bn;
            const double ratio = m.d2_cal > 0.0 ? std::sqrt(m.e2_cal / m.d2_cal) : 0.0;
            const double est = 4.0 * ratio * std::sqrt(m.d2) / bn;
            const bool finite = std::isfinite(res_tc) && std::isfinite(est) && st == 0;
            mx_trace[0] = res_tc;
            mx_trace[1] = est;
            mx_trace[2] = std::sqrt(m.r64) / bn;
            mx_trace[3] = std::sqrt(m.d2_cal) / bn;
            mx_trace[4] = std::sqrt(m.d2) / bn;
            mx_trace[5] = ratio;
            bool ok = finite && res_tc + est <= tolerance;
            double res = res_tc + est;
            if (finite && !ok && res_tc <= tolerance) {
                // the estimate alone is too large: the fp64 residual decides
                mixed_resid64(sk, k, dtv);
                MixScalars m2;
                CK(cudaMemcpyAsync(&m2, d_msc.p, sizeof(m2), cudaMemcpyDeviceToHost, stream));
                sync();
                res = std::sqrt(m2.r64) / bn;
                ok = std::isfinite(res) && res <= tolerance;
                if (!ok) {
                    // continue from this fp64 residual
                    if (mx_passes >= mixed_max_passes) break;
                    mixed_pass(sk, k, dtv, 2);
                    mixed_resid_tc(sk, k, dtv);
                    mixed_tail(sk, k, hs);
                    continue;
                }
            }
            if (ok) {
                std::swap(psi.p, cand.p);
                last_iterations = mx_passes;
                last_residual = res;
                mx_residual = res;
                return;
            }
            if (!finite || mx_passes >= mixed_max_passes) break;
            mixed_resid64(sk, k, dtv, cand.p);
            mixed_calibrate(sk, k, dtv);
            mixed_pass(sk, k, dtv, 2);
            mixed_resid_tc(sk, k, dtv);
            mixed_tail(sk, k, hs);
        }
        // not converged in low precision: the fp64 solve from the step's psi and rhs
        std::fprintf(stderr, "\nMixed solve did not reach the tolerance; redoing the step with the fp64 solve.\n");
        begin_solve(sk, k, hs);
        finish_solve(sk, k, hs);
        mx_residual = last_residual;
    }

    // Woodbury correction of a preconditioner output y; the corrected sink projections
    // land in m_dots[2..3]
    void wood32(const Absorber *const *sk, int k, float2 *yv)
    {
        if (k == 0) return;
        sink_dots32(yv, m_dots.p, sk, k);
        const int64_t nb = (int64_t)std::max(1, wband_hi - wband_lo) * n_modes;
        const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((nb + 255) / 256, vec_blocks));
        k_wood32<<<blocks, 256, 0, stream>>>(Nr, n_modes, wband_lo, wband_hi, d_kr.p, m_dots.p, W0.p, W1.p, yv,
                                            m_dots.p + 2);
        launch_check();
    }

    // Launches that follow the solve, queued behind every batch of iterations and gated
    // on the device: the true residual of the candidate once the solve is done (its
    // last CTA decides acceptance, KS_RESID), then psi = mask (|rhs| x), the
    // diagnostics pass of the new state and the read-backs, once accepted.
    void enqueue_tail(const Absorber *const *sk, int k, double dtv, double *hs)
    {
        sink_dots(x.p, d_dots.p, sk, k, GATE_DONE);
        {
            DotSpec ds;
            ds.n = 1;
            ds.kind[0] = 4;
            ds.ext[0] = rhs.p;
            ds.scale_from_kr = true;
            ds.stage = KS_RESID;
            ds.red = d_red.p + RED_RES;
            ds.gate_mode = GATE_DONE;
            apply_A(x.p, tmp.p, sk, k, d_dots.p, dtv, ds);
        }
        CK(launch_pdl(k_scale_mask, vec_blocks, VEC_THREADS, 0, stream, nN, Nr, 0.0, mask ? d_mask.p : nullptr, x.p, psi.p,
                                                              d_kr.p));
        launch_check();
        enqueue_diagnostics(sk, k);
        const size_t kd = (sizeof(Krylov) + 7) / 8;
        const int nslots = 2 * n_modes + 3;
        CK(cudaMemcpyAsync(hs, d_kr.p, sizeof(Krylov), cudaMemcpyDeviceToHost, stream));
        CK(cudaMemcpyAsync(hs + kd, d_red.p, nslots * sizeof(double), cudaMemcpyDeviceToHost, stream));
        CK(cudaMemcpyAsync(hs + kd + nslots, d_edge.p, 4 * n_modes * sizeof(double2), cudaMemcpyDeviceToHost,
                           stream));
        CK(cudaMemcpyAsync(hs + kd + nslots + 8 * n_modes, d_dots.p, 8 * sizeof(double2), cudaMemcpyDeviceToHost,
                           stream));
    }

    // One preconditioned BiCGSTAB attempt from the initial guess psi / |rhs| with the
    // radial-block preconditioner or, when `jacobi` is set, the point-Jacobi one.  The
    // iterations go out in batches (as many as the previous step needed) followed by
    // the gated tail, with one host synchronisation per batch for the convergence and
    // restart test.  begin_attempt queues the set-up and the first batch; finish_attempt
    // waits, queues further batches (and restarts) until the solve is done, and tells
    // whether the candidate was accepted (pivots finite and true residual <=
    // accept_residual); the tail's read-backs are then in hs.
    struct AttemptState {
        int restarts = 0;
        int max_it = 0;
    } att;

    void begin_attempt(int max_it, const Absorber *const *sk, int k, double *hs)
    {
        const double dtv = op.dt;
        Krylov *dk = d_kr.p;
        Krylov kr;
        std::memset(&kr, 0, sizeof(kr));
        kr.n_sinks = k;
        kr.tol = tolerance;
        kr.max_iterations = max_it;
        kr.eigen_path = k == 0;
        kr.accept = accept_residual;
        kr.status = d_status.p;
        h_kr_init = kr;
        CK(cudaMemcpyAsync(dk, &h_kr_init, sizeof(kr), cudaMemcpyHostToDevice, stream));
        // with b = rhs / |rhs| (never stored): x = psi / |rhs|, r = r0 = b - A_full x in one
        // pass; its last CTA runs KS_INIT (and the first beta) on |r0|^2 and |b|^2
        CK(launch_pdl(k_krylov_start, vec_blocks, VEC_THREADS, 0, stream, nN, dk, d_red.p + RED_RHS, rhs.p, psi.p, x.p, rr.p,
                                                                r0.p, d_partials.p, d_red.p + 8, ticket(TK_START_T)));
        launch_check();
        factorize(dtv);
        if (k > 0) wood_setup(sk, k, dtv);
        att = AttemptState();
        att.max_it = max_it;
        const int batch = std::max(1, std::min(4, iter_hint));
        for (int q = 0; q < batch; ++q) enqueue_iteration(sk, k, dtv, q == 0);
        enqueue_tail(sk, k, dtv, hs);
    }

    bool finish_attempt(const Absorber *const *sk, int k, double *hs)
    {
        const double dtv = op.dt;
        Krylov *dk = d_kr.p;
        Krylov kr;
        const bool eigen_path = k == 0;
        const double eps = std::numeric_limits<double>::epsilon();
        for (;;) {
            sync();
            std::memcpy(&kr, hs, sizeof(kr));
            if (kr.done) break;
            if (kr.restart) {
                // Lost biorthogonality: restart from the current residual (_matrices.cpp:69-75).
                const double2 rho_old = kr.rho;
                sink_dots(x.p, d_dots.p, sk, k);
                apply_A(x.p, tmp.p, sk, k, d_dots.p, dtv);
                // r = rhs / |rhs| - A_full x
                axpby(cmake(kr.rhs_norm > 0.0 ? 1.0 / kr.rhs_norm : 0.0, 0.0), rhs.p, cmake(-1, 0), tmp.p, rr.p);
                CK(cudaMemcpyAsync(r0.p, rr.p, nN * sizeof(double2), cudaMemcpyDeviceToDevice, stream));
                dots(1, rr.p, rr.p);
                const double nr2 = read_red(0);
                kr.rho_old = rho_old;
                kr.rho = cmake(nr2, 0.0);
                if (eigen_path) {
                    kr.restart_thr = eps * eps * nr2;
                    if (att.restarts++ == 0) kr.iterations = 0;
                }
                kr.beta = cmul(cdiv(kr.rho, rho_old), cdiv(kr.alpha, kr.omega));
                kr.restart = 0;
                h_kr_init = kr;
                CK(cudaMemcpyAsync(dk, &h_kr_init, sizeof(kr), cudaMemcpyHostToDevice, stream));
            }
            for (int q = 0; q < 2; ++q) enqueue_iteration(sk, k, dtv, false);
            enqueue_tail(sk, k, dtv, hs);
        }
        last_iterations = kr.iterations;
        last_residual = kr.residual;
        iter_hint = std::max(1, kr.iterations);
        return kr.accepted != 0;
    }

    // solve_CN (src/CrankNicolsonModes_matrices.cpp:94-215): the radial-block attempt;
    // if its factorisation fails or its result misses the 1e-9 residual, the reference
    // retries with a full ILUT preconditioner and 5000 iterations -- here the retry is a
    // point-Jacobi BiCGSTAB on the device with the same iteration budget.  With
    // use_block_preconditioner off the retry path is the only one, as in the reference.
    // begin_solve queues the first attempt; finish_solve completes it (and the retry)
    // and leaves psi holding the accepted state and hs the step's read-backs.
    void begin_solve(const Absorber *const *sk, int k, double *hs)
    {
        jacobi = !use_block;
        begin_attempt(use_block ? max_iterations : 5000, sk, k, hs);
    }

    void finish_solve(const Absorber *const *sk, int k, double *hs)
    {
        bool ok = false;
        try {
            ok = finish_attempt(sk, k, hs);
            if (!ok && !jacobi) {
                std::fprintf(stderr,
                             "\nRadial preconditioner did not converge; retrying with the point-Jacobi fallback.\n");
                jacobi = true;
                begin_attempt(5000, sk, k, hs);
                ok = finish_attempt(sk, k, hs);
            }
        } catch (...) {
            jacobi = false;
            throw;
        }
        jacobi = false;
        if (!ok) throw Error(CNM_ESOLVE, "Crank-Nicolson solve failed the relative residual check");
    }

    // Woodbury set-up (src/CrankNicolsonModes_matrices.cpp:133-145): W_a = P^{-1} v_a and
    // G = diag(1 / (dt/4 g_a)) + v_a^dag W_b with its inverse, into the Krylov struct.
    void wood_setup(const Absorber *const *sk, int k, double dtv)
    {
        const double c0 = 0.25 * dtv * sk[0]->strength, c1 = k > 1 ? 0.25 * dtv * sk[1]->strength : 1.0;
        set_wood_band(sk, k, dtv);
        if (pcl_per > 0 && !jacobi && wband_hi - wband_lo <= WOOD_BAND_MAX) {
            // W_a only on the band, one warp per (radial block, sink)
            WoodBand wb;
            wb.n_sinks = k;
            wb.v0 = sk[0]->v.p;
            wb.v1 = k > 1 ? sk[1]->v.p : nullptr;
            wb.W0 = W0.p;
            wb.W1 = W1.p;
            wb.slo0 = sk[0]->lo;
            wb.shi0 = sk[0]->hi;
            wb.slo1 = k > 1 ? sk[1]->lo : 0;
            wb.shi1 = k > 1 ? sk[1]->hi : 0;
            wb.c0 = c0;
            wb.c1 = c1;
            wb.partials = d_wpart.p;
            wb.ticket = ticket(TK_WOOD_T);
            wb.kr = d_kr.p;
            const size_t smem = (size_t)2 * (wband_hi - wband_lo) * sizeof(double2);
            CK(launch_pdl(k_wood_setup_band, n_modes * k, WSB_THREADS, smem, stream, Nr, n_modes, wband_lo, wband_hi,
                                                                          offdiag(dtv), dinv.p, wb));
            launch_check();
            return;
        }
        if (pcl_per > 0 && !jacobi) {
            WoodArgs wd = wood_args(WD_SETUP, 0, sk, k);
            wd.c0 = c0;
            wd.c1 = c1;
            const PrecondInput plain{PI_PLAIN, nullptr, nullptr, nullptr, nullptr, nullptr};
            if (k > 1) precond_cl(sk[0]->v.p, W0.p, sk[1]->v.p, W1.p, dtv, plain, wd);
            else precond_cl(sk[0]->v.p, W0.p, nullptr, nullptr, dtv, plain, wd);
            return;
        }
        precond(sk[0]->v.p, W0.p, dtv);
        if (k > 1) precond(sk[1]->v.p, W1.p, dtv);
        sink_dots(W0.p, d_dots.p + 4, sk, k);
        if (k > 1) sink_dots(W1.p, d_dots.p + 6, sk, k);
        k_wood_setup<<<1, 32, 0, stream>>>(d_kr.p, d_dots.p + 4, c0, c1);
        launch_check();
    }

    WoodArgs wood_args(int mode, int which, const Absorber *const *sk, int k)
    {
        WoodArgs wd;
        std::memset(&wd, 0, sizeof(wd));
        wd.mode = k > 0 ? mode : WD_NONE;
        wd.which = which;
        wd.n_sinks = k;
        wd.v0 = k > 0 ? sk[0]->v.p : nullptr;
        wd.v1 = k > 1 ? sk[1]->v.p : nullptr;
        wd.lo0 = k > 0 ? sk[0]->lo : 0;
        wd.hi0 = k > 0 ? sk[0]->hi : 0;
        wd.lo1 = k > 1 ? sk[1]->lo : 0;
        wd.hi1 = k > 1 ? sk[1]->hi : 0;
        wd.partials = d_wpart.p;
        wd.ticket = ticket(TK_WOOD_T);
        wd.kr = d_kr.p;
        return wd;
    }

    // out = M b (src/CrankNicolsonModes_matrices.cpp:146-153): out = P^{-1} b without sinks;
    // with sinks yP = P^{-1} b, c = G^{-1} v^dag yP (in the solve's last CTA) and
    // out = yP - W c.  `in` forms b inside the solve (PI_P / PI_S).
    void precond_M(const PrecondInput &in, int which, const Absorber *const *sk, int k, double dtv, double2 *out)
    {
        if (k == 0) {
            precond(nullptr, out, dtv, in);
            return;
        }
        if (pcl_per > 0 && !jacobi) {
            precond_cl(nullptr, out, nullptr, nullptr, dtv, in, wood_args(WD_PROJ, which, sk, k));
        } else {
            precond(nullptr, out, dtv, in);
            sink_dots(out, d_dots.p + 4, sk, k);
            k_wood_scalar<<<1, 32, 0, stream>>>(d_kr.p, which, d_dots.p + 4);
            launch_check();
        }
        // out -= sum_a W_a c_a where the W_a live
        const int64_t nb = (int64_t)(wband_hi - wband_lo) * n_modes;
        const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((nb + 255) / 256, vec_blocks));
        CK(launch_pdl(k_woodbury_band, blocks, 256, 0, stream, Nr, n_modes, wband_lo, wband_hi, d_kr.p, which, W0.p, W1.p, out));
        launch_check();
    }

    // Widest band the CTA-per-block Woodbury set-up takes (its shared memory holds the
    // band's pivots and values); wider bands use the cluster solve.
    static constexpr int WOOD_BAND_MAX = 4096;

    // Band of nodes outside which every W_a = P^{-1} v_a is below 1e-40 of its largest
    // value: the entries of the inverse of a radial block decay by the contraction
    // rho = |off| / |p+| per node (with the potential's deepest depression of the
    // diagonal, as choose_window bounds it), so 92 / -ln(rho) nodes past the sinks'
    // support suffice; the point-Jacobi W_a vanish outside the support itself.
    void set_wood_band(const Absorber *const *sk, int k, double dtv)
    {
        int lo = Nr, hi = 0;
        for (int a = 0; a < k; ++a) {
            lo = std::min(lo, sk[a]->lo);
            hi = std::max(hi, sk[a]->hi);
        }
        if (hi <= lo) {
            wband_lo = wband_hi = 0;
            return;
        }
        int w = 0;
        if (!jacobi) {
            const double kappa = std::abs(offdiag(dtv).y);
            const double depress = std::min(0.5, 0.5 * dtv * diag_potential_bound() / (2.0 * kappa));
            const std::complex<double> a(1.0, 2.0 * kappa * (1.0 - depress)), c(-kappa * kappa, 0.0);
            const std::complex<double> sq = std::sqrt(a * a - 4.0 * c);
            const double pp = std::max(std::abs((a + sq) * 0.5), std::abs((a - sq) * 0.5));
            const double rho = kappa / pp;
            w = rho < 1.0 ? (int)std::min<double>(Nr, std::ceil(92.2 / -std::log(rho)) + 16) : Nr;
        }
        wband_lo = std::max(0, lo - w);
        wband_hi = std::min(Nr, hi + w);
    }

    // -------------------------------------------------------------- step

    void set_extraction_radius(double rex, int n_steps)
    {
        r_ex = rex;
        idx_ex = (int)std::floor(r_ex / dr);
        if (n_steps < 1 || idx_ex < 1 || idx_ex >= Nr - 1)
            throw Error(CNM_EINVAL, "Require at least one time sample and an interior extraction radius");
    }

    void prepare_run(int n_steps, double rex)
    {
        set_extraction_radius(rex, n_steps);
        t_i = 0.0;
        build_time_dependent_perturbation(t_i);
        sync();
    }

    // step (src/CrankNicolsonModes.cpp:145-234) in two halves: step_begin queues the
    // operator rebuild, the right-hand side and the first batch of the solve (with its
    // gated tail) without waiting; step_end waits, completes the solve and runs the
    // host side (orbit, diagnostics).  step() is both; batches of binaries call all the
    // begins before the ends so that their launches share the device.
    double step_start_t = 0.0;
    double *step_hs = nullptr;

    void step(int step_id, cnm_diag *dg, double *ef, double *fl, double *nm, double *en)
    {
        step_begin(step_id);
        step_end(step_id, dg, ef, fl, nm, en);
    }

    void step_begin(int step_id)
    {
        (void)step_id;
        if (!initialized) throw Error(CNM_ELOGIC, "initialize() must be called before step()");
        if (idx_ex < 1) throw Error(CNM_ELOGIC, "run() (cnm_prepare_run) must set the extraction radius first");
        step_start_t = t_i;
        t_i += dt;
        theta += (counter ? -1.0 : 1.0) * Omega * dt;
        phase += Omega * dt;
        build_time_dependent_perturbation(t_i);
        ab_cap = op.cap;
        // projections of the old state on the new sinks (for the midpoint accretion rate)
        const Absorber *all[2] = {&abs1, &abs2};
        const bool have_sinks = absorption && cpl.mode00 >= 0;
        // v_a^dag psi on both sinks (d_dots[2..3]); the active sinks are a contiguous
        // subsequence of (abs1, abs2), so their projections are read in place
        if (have_sinks) sink_dots(psi.p, d_dots.p + 2, all, 2);
        // rhs = B psi - dt/4 Gamma psi, with |rhs|^2 into red[RED_RHS]
        const Absorber *sk[2];
        const int k = active_sinks(sk);
        {
            ApplyArgs a = base_args(psi.p, rhs.p);
            DotSpec ds;
            ds.n = 1;
            ds.kind[0] = 3;
            ds.stage = KS_NONE;
            ds.red = d_red.p + RED_RHS;
            a.n_dots = 1;
            a.dot_kind[0] = 3;
            a.dot_partials = d_partials.p;
            set_finish(a, ds);
            a.alpha = cmake(1.0, 0.0);
            a.beta = cmake(0.0, -0.5 * op.dt);
            a.use_h0 = 1;
            a.use_cap = 1;
            a.vpart = V_POT;
            a.n_sinks = k;
            a.sink_dots = k > 0 ? d_dots.p + 2 + sink_slot(sk[0]) : d_dots.p;
            for (int i = 0; i < k; ++i) {
                a.sink_v[i] = sk[i]->v.p;
                a.sink_coef[i] = -0.25 * op.dt * sk[i]->strength;
                a.sink_lo[i] = sk[i]->lo;
                a.sink_hi[i] = sk[i]->hi;
            }
            launch_apply(a);
        }
        step_hs = stage(readback_doubles());
        if (mixed && use_block) begin_mixed(sk, k, step_hs);
        else begin_solve(sk, k, step_hs);
    }

    void step_end(int step_id, cnm_diag *dg, double *ef, double *fl, double *nm, double *en)
    {
        const double step_start = step_start_t;
        const Absorber *all[2] = {&abs1, &abs2};
        const bool have_sinks = absorption && cpl.mode00 >= 0;
        const Absorber *sk[2];
        const int k = active_sinks(sk);
        double *hs = step_hs;
        if (mixed && use_block) finish_mixed(sk, k, hs);
        else finish_solve(sk, k, hs);
        const int nslots = 2 * n_modes + 3;
        const size_t kd = (sizeof(Krylov) + 7) / 8;
        hs += kd;
        const double *redh = hs;
        const double2 *edge = reinterpret_cast<const double2 *>(hs + nslots);
        const double2 *dh = reinterpret_cast<const double2 *>(hs + nslots + 8 * n_modes);
        // orbit (src/CrankNicolsonModes.cpp:189-195)
        if (!isolated && evolve_orbit && t_i > ramp_end_time()) {
            const double orbit_dt = t_i - std::max(step_start, ramp_end_time());
            double md[2] = {0.0, 0.0};
            if (have_sinks)
                for (int a2 = 0; a2 < 2; ++a2) {
                    const Absorber *ab = all[a2];
                    if (ab->strength == 0.0) continue;
                    // v^dag psi_mid = (v^dag psi + v^dag psi_last) / 2
                    const std::complex<double> pm(0.5 * (dh[4 + a2].x + dh[2 + a2].x),
                                                  0.5 * (dh[4 + a2].y + dh[2 + a2].y));
                    md[a2] = mu * dr * ab->strength * std::norm(pm);
                }
            update_time_dependent_increment(orbit_dt, md[0], md[1]);
        }
        // diagnostics (src/CrankNicolsonModes_extraction.cpp)
        const int n = n_modes;
        const double rx = r[idx_ex];
        double energy_sum = 0.0;
        for (int j = 0; j < n; ++j) {
            const std::complex<double> pl(edge[n + 3 * j].x, edge[n + 3 * j].y);
            const std::complex<double> pc(edge[n + 3 * j + 1].x, edge[n + 3 * j + 1].y);
            const std::complex<double> pr(edge[n + 3 * j + 2].x, edge[n + 3 * j + 2].y);
            const std::complex<double> dpsi(edge[j].x, edge[j].y);
            const std::complex<double> dU = (pr - pl) / (2.0 * dr) - pc / rx;
            if (fl) fl[j] = (std::conj(pc) * dU).imag();
            if (ef) ef[j] = (std::conj(dpsi) * dU).real() / mu;
            if (nm) nm[j] = redh[j] * dr;
            if (en) en[j] = redh[n + j] * dr;
            energy_sum += redh[n + j];
        }
        const double energy = (energy_sum + redh[2 * n]) * dr;
        const double p_bin_inst = redh[2 * n + 1] * dr;
        const double dV = redh[2 * n + 2] * dr;
        p_bin = isolated ? 0.0 : power_average.update(t_i, phase, p_bin_inst);
        kt_flush();
        if (dg) {
            dg->R = R;
            dg->theta = theta;
            dg->Omega = Omega;
            dg->M1 = M1;
            dg->q = q;
            dg->t = t_i;
            dg->energy = energy;
            dg->p_bin = p_bin;
            dg->p_bin_inst = p_bin_inst;
            dg->dV_bin_dt = dV;
            dg->residual = last_residual;
            dg->iterations = last_iterations;
        }
        (void)step_id;
    }

    // src/CrankNicolsonModes_evolution.cpp:17-72
    void update_time_dependent_increment(double orbit_dt, double Mdot1, double Mdot2)
    {
        double ramp = 1.0;
        if (t_i < ramp_end_time()) ramp = 0.0;
        else if (t_i < ramp_end_time() + initial_period) {
            const double xr = (t_i - ramp_end_time()) / initial_period;
            ramp = 3.0 * xr * xr - 2.0 * xr * xr * xr;
        }
        const double dR_gw = -(64.0 / 5.0) * M1 * M2 * (M1 + M2) / std::pow(R, 3);
        const double dR_cloud = -2.0 * R * R * p_bin / (M1 * M2);
        const double dRdt = (dR_gw + dR_cloud) * ramp;
        R += dRdt * orbit_dt;
        M1 += Mdot1 * orbit_dt;
        M2 += Mdot2 * orbit_dt;
        q = M2 / M1;
        const double Mt = M1 + M2;
        R1 = M2 / Mt * R;
        R2 = M1 / Mt * R;
        Omega = std::sqrt(Mt / std::pow(R, 3));
        P = 2.0 * M_PI / Omega;
        if (ramp_factor == 1.0) dt = P / steps_per_period;
    }

    // -------------------------------------------------------------- checkpoint

    // src/CrankNicolsonModes_restart.cpp:139-177: "GMCKPT01", int32 {step, Nr, n_modes},
    // 13 f64 {t, theta, phase, R, M1, M2, q, R1, R2, Omega, P, dt, p_bin}, u64 size,
    // psi as complex128, the rolling-average blob.
    std::vector<char> checkpoint(int step_id) const
    {
        std::vector<char> out;
        auto put = [&](const void *p, size_t n) {
            const char *c = static_cast<const char *>(p);
            out.insert(out.end(), c, c + n);
        };
        put("GMCKPT01", 8);
        const int32_t header[3] = {step_id, Nr, n_modes};
        put(header, sizeof(header));
        const double values[13] = {t_i, theta, phase, R, M1, M2, q, R1, R2, Omega, P, dt, p_bin};
        put(values, sizeof(values));
        const uint64_t size = (uint64_t)nN;
        put(&size, 8);
        const size_t at = out.size();
        out.resize(at + (size_t)nN * sizeof(double2));
        CK(cudaMemcpy(out.data() + at, psi.p, (size_t)nN * sizeof(double2), cudaMemcpyDeviceToHost));
        power_average.save(out);
        return out;
    }

    // src/CrankNicolsonModes_restart.cpp:179-233: false (state untouched) unless the blob
    // is a complete checkpoint of this step and geometry.
    bool restore(int step_id, const char *p, size_t size)
    {
        const size_t head = 8 + 12 + 13 * 8 + 8;
        if (size < head || std::memcmp(p, "GMCKPT01", 8) != 0) return false;
        int32_t header[3];
        std::memcpy(header, p + 8, sizeof(header));
        if (header[0] != step_id || header[1] != Nr || header[2] != n_modes) return false;
        double values[13];
        std::memcpy(values, p + 20, sizeof(values));
        uint64_t n = 0;
        std::memcpy(&n, p + 20 + 104, 8);
        if (n != (uint64_t)nN || size < head + n * sizeof(double2)) return false;
        RollingPhaseAverage avg(orbits_average);
        size_t used = 0;
        if (!avg.load(p + head + n * sizeof(double2), size - head - n * sizeof(double2), used)) return false;
        CK(cudaMemcpy(psi.p, p + head, (size_t)n * sizeof(double2), cudaMemcpyHostToDevice));
        t_i = values[0];
        theta = values[1];
        phase = values[2];
        R = values[3];
        M1 = values[4];
        M2 = values[5];
        q = values[6];
        R1 = values[7];
        R2 = values[8];
        Omega = values[9];
        P = values[10];
        dt = values[11];
        p_bin = values[12];
        power_average = avg;
        return true;
    }

    // -------------------------------------------------------------- cnm_apply

    void apply_op(int opc, const double *xh, double *yh)
    {
        if (!op.built) throw Error(CNM_ELOGIC, "operators exist only after initialize()");
        CK(cudaMemcpyAsync(tmp.p, xh, nN * sizeof(double2), cudaMemcpyHostToDevice, stream));
        const Absorber *sk[2];
        const int k = active_sinks(sk);
        ApplyArgs a = base_args(tmp.p, cand.p);
        a.alpha = cmake(0, 0);
        a.beta = cmake(1, 0);
        auto with_sinks = [&](double coef) {
            sink_dots(tmp.p, d_dots.p + 6, sk, k);
            a.n_sinks = k;
            a.sink_dots = d_dots.p + 6;
            for (int i = 0; i < k; ++i) {
                a.sink_v[i] = sk[i]->v.p;
                a.sink_coef[i] = coef * sk[i]->strength;
                a.sink_lo[i] = sk[i]->lo;
                a.sink_hi[i] = sk[i]->hi;
            }
        };
        switch (opc) {
        case CNM_OP_H: a.use_h0 = 1; a.use_cap = 1; a.vpart = V_POT; break;
        case CNM_OP_H0: a.use_h0 = 1; break;
        case CNM_OP_V: a.vpart = V_POT; break;
        case CNM_OP_V1: build_hh(d_hh_aux.p, 1.0, 0.0); a.vpart = V_POT; a.hh = d_hh_aux.p; break;
        case CNM_OP_V2: build_hh(d_hh_aux.p, 0.0, 1.0); a.vpart = V_POT; a.hh = d_hh_aux.p; break;
        case CNM_OP_DVDT: a.vpart = V_DVDT; break;
        case CNM_OP_A:
        case CNM_OP_B:
        case CNM_OP_AFULL:
            a.alpha = cmake(1, 0);
            a.beta = cmake(0, (opc == CNM_OP_B ? -0.5 : 0.5) * op.dt);
            a.use_h0 = 1;
            a.use_cap = ab_cap ? 1 : 0;
            a.vpart = V_POT;
            if (opc == CNM_OP_AFULL) with_sinks(0.25 * op.dt);
            break;
        case CNM_OP_SINK: a.beta = cmake(0, 0); with_sinks(1.0); break;
        case CNM_OP_RHS:
            a.beta = cmake(0, -1);
            a.use_h0 = 1;
            a.use_cap = 1;
            a.vpart = V_POT;
            with_sinks(-0.5);
            break;
        case CNM_OP_CAP: a.use_cap = 1; break;
        case CNM_OP_PRECOND: {
            // the radial blocks of the member A (whose CAP term follows ab_cap)
            const bool cap_now = op.cap;
            op.cap = ab_cap;
            factorize(op.dt);
            precond(tmp.p, cand.p, op.dt);
            op.cap = cap_now;
            break;
        }
        default: throw Error(CNM_EINVAL, "unknown operator");
        }
        if (opc != CNM_OP_PRECOND) launch_apply(a);
        CK(cudaMemcpyAsync(yh, cand.p, nN * sizeof(double2), cudaMemcpyDeviceToHost, stream));
        sync();
    }

    // cnm_apply_lowp: the mixed path's complex64 tensor-core operator on a host vector.
    void apply_lowp(int opc, const double *xh, double *yh)
    {
        if (!mixed) throw Error(CNM_ELOGIC, "the low-precision operator exists only on a CNM_MIXED handle");
        if (!op.built) throw Error(CNM_ELOGIC, "operators exist only after initialize()");
        CK(cudaMemcpyAsync(tmp.p, xh, nN * sizeof(double2), cudaMemcpyHostToDevice, stream));
        k_to_f32<<<vec_blocks, VEC_THREADS, 0, stream>>>(nN, tmp.p, m_xa.p);
        launch_check();
        const Absorber *sk[2];
        int k = 0;
        TcArgs a = tc_a_args(m_xa.p, m_t.p, sk, 0, nullptr, op.dt);
        switch (opc) {
        case CNM_OP_H: a.alpha = make_float2(0.f, 0.f); a.beta = make_float2(1.f, 0.f); break;
        case CNM_OP_V: a.alpha = make_float2(0.f, 0.f); a.beta = make_float2(1.f, 0.f); a.use_h0 = 0; a.use_cap = 0; break;
        case CNM_OP_A: a.use_cap = ab_cap ? 1 : 0; break;
        case CNM_OP_AFULL:
            a.use_cap = ab_cap ? 1 : 0;
            k = active_sinks(sk);
            if (k > 0) {
                sink_dots32(m_xa.p, m_dots.p + 6, sk, k);
            }
            {
                TcArgs b = tc_a_args(m_xa.p, m_t.p, sk, k, m_dots.p + 6, op.dt);
                b.use_cap = a.use_cap;
                a = b;
            }
            break;
        default: throw Error(CNM_EINVAL, "operator not available in low precision");
        }
        CK(cudaMemsetAsync(d_status.p, 0, sizeof(int), stream));
        launch_tc(a);
        k_to_f64<<<vec_blocks, VEC_THREADS, 0, stream>>>(nN, m_t.p, cand.p);
        launch_check();
        CK(cudaMemcpyAsync(yh, cand.p, nN * sizeof(double2), cudaMemcpyDeviceToHost, stream));
        sync();
        int st = 0;
        CK(cudaMemcpy(&st, d_status.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (st) throw Error(CNM_EDEVICE, "tensor-core apply: a pipeline wait gave up");
    }

    double sink_strength(int body)
    {
        const Absorber &ab = body == 1 ? abs1 : abs2;
        if (!op.sink_active || ab.strength == 0.0 || ab.hi <= ab.lo || cpl.mode00 < 0) return 0.0;
        const Absorber *one[1] = {&ab};
        sink_dots(ab.v.p, d_dots.p + 6, one, 1);
        double2 vv;
        CK(cudaMemcpyAsync(&vv, d_dots.p + 6, sizeof(vv), cudaMemcpyDeviceToHost, stream));
        sync();
        return ab.strength * vv.x;
    }
};

}  // namespace cnm

// ==================================================================== C ABI

struct cnm_handle {
    cnm::Solver *s = nullptr;
    std::string err;
};

static thread_local std::string g_create_error;

template <class F>
static int guarded(cnm_handle *h, F &&f)
{
    if (!h || !h->s) return CNM_EINVAL;
    try {
        f(*h->s);
        return CNM_OK;
    } catch (const cnm::Error &e) {
        h->err = e.what();
        return e.code;
    } catch (const std::exception &e) {
        h->err = e.what();
        return CNM_ECUDA;
    }
}

extern "C" {

int cnm_select_device(int32_t device)
{
    const cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        g_create_error = std::string("cudaSetDevice: ") + cudaGetErrorString(e);
        return CNM_ECUDA;
    }
    return CNM_OK;
}

int cnm_create(const cnm_params *params, cnm_handle **out)
{
    if (!params || !out) return CNM_EINVAL;
    *out = nullptr;
    try {
        cnm_handle *h = new cnm_handle;
        h->s = new cnm::Solver(*params);
        *out = h;
        return CNM_OK;
    } catch (const cnm::Error &e) {
        g_create_error = e.what();
        return e.code;
    } catch (const std::exception &e) {
        g_create_error = e.what();
        return CNM_ECUDA;
    }
}

int cnm_destroy(cnm_handle *h)
{
    if (!h) return CNM_OK;
    delete h->s;
    delete h;
    return CNM_OK;
}

const char *cnm_last_error(const cnm_handle *h) { return h ? h->err.c_str() : g_create_error.c_str(); }
const char *cnm_create_error(void) { return g_create_error.c_str(); }

int cnm_n_modes(const cnm_handle *h, int32_t *n)
{
    if (!h || !n) return CNM_EINVAL;
    *n = h->s->n_modes;
    return CNM_OK;
}

int cnm_modes(const cnm_handle *h, int32_t *l, int32_t *m)
{
    if (!h || !l || !m) return CNM_EINVAL;
    for (int j = 0; j < h->s->n_modes; ++j) {
        l[j] = h->s->cpl.mode_l[j];
        m[j] = h->s->cpl.mode_m[j];
    }
    return CNM_OK;
}

int cnm_coupling_info(const cnm_handle *h, int32_t *n_pairs, int32_t *n_terms)
{
    if (!h || !n_pairs || !n_terms) return CNM_EINVAL;
    *n_pairs = (int32_t)h->s->cpl.pair_col.size();
    *n_terms = (int32_t)h->s->cpl.term_l.size();
    return CNM_OK;
}

int cnm_grid(const cnm_handle *h, double *r)
{
    if (!h || !r) return CNM_EINVAL;
    std::copy(h->s->r.begin(), h->s->r.end(), r);
    return CNM_OK;
}

int cnm_get_scalars(const cnm_handle *h, cnm_scalars *o)
{
    if (!h || !o) return CNM_EINVAL;
    const cnm::Solver &s = *h->s;
    o->t = s.t_i;
    o->theta = s.theta;
    o->phase = s.phase;
    o->Omega = s.Omega;
    o->Omega_0 = s.Omega_0;
    o->P = s.P;
    o->R = s.R;
    o->R1 = s.R1;
    o->R2 = s.R2;
    o->M1 = s.M1;
    o->M2 = s.M2;
    o->q = s.q;
    o->dt = s.dt;
    o->p_bin = s.p_bin;
    o->steps_per_period = s.steps_per_period;
    o->evolve_orbit = s.evolve_orbit;
    o->ramp_secondary_potential = s.ramp_secondary_potential;
    o->use_block_preconditioner = s.use_block;
    o->last_solver_iterations = s.last_iterations;
    o->last_solver_residual = s.last_residual;
    o->tolerance = s.tolerance;
    o->max_iterations = s.max_iterations;
    o->accept_residual = s.accept_residual;
    return CNM_OK;
}

int cnm_set_scalars(cnm_handle *h, const cnm_scalars *i)
{
    if (!h || !i) return CNM_EINVAL;
    cnm::Solver &s = *h->s;
    s.t_i = i->t;
    s.theta = i->theta;
    s.phase = i->phase;
    s.Omega = i->Omega;
    s.Omega_0 = i->Omega_0;
    s.P = i->P;
    s.R = i->R;
    s.R1 = i->R1;
    s.R2 = i->R2;
    s.M1 = i->M1;
    s.M2 = i->M2;
    s.q = i->q;
    s.dt = i->dt;
    s.p_bin = i->p_bin;
    s.steps_per_period = i->steps_per_period;
    s.evolve_orbit = i->evolve_orbit != 0;
    s.ramp_secondary_potential = i->ramp_secondary_potential != 0;
    s.use_block = i->use_block_preconditioner != 0;
    s.last_iterations = i->last_solver_iterations;
    s.last_residual = i->last_solver_residual;
    s.tolerance = i->tolerance;
    s.max_iterations = i->max_iterations;
    s.accept_residual = i->accept_residual;
    return CNM_OK;
}

int cnm_set_initial_state_full(cnm_handle *h, const double *psi0, int64_t n)
{
    return guarded(h, [&](cnm::Solver &s) { s.set_initial_state_full(psi0, n); });
}

int cnm_set_state(cnm_handle *h, const double *psi, int64_t n)
{
    return guarded(h, [&](cnm::Solver &s) { s.set_state(psi, n); });
}

int cnm_get_state(const cnm_handle *h, double *psi, int64_t n)
{
    return guarded(const_cast<cnm_handle *>(h), [&](cnm::Solver &s) { s.get_state(psi, n); });
}

int cnm_configure_isolated_black_hole(cnm_handle *h, double x)
{
    return guarded(h, [&](cnm::Solver &s) { s.configure_isolated_black_hole(x); });
}

int cnm_initialize(cnm_handle *h)
{
    return guarded(h, [&](cnm::Solver &s) {
        s.initialize();
        s.sync();
    });
}

int cnm_set_power_average_orbits(cnm_handle *h, double n_orbits)
{
    return guarded(h, [&](cnm::Solver &s) {
        s.power_average = cnm::RollingPhaseAverage(n_orbits);
        s.orbits_average = n_orbits;
    });
}

int cnm_build_damping_mask(cnm_handle *h, double f, double W, int32_t n)
{
    return guarded(h, [&](cnm::Solver &s) { s.build_damping_mask(f, W, n); });
}

int cnm_build_cap(cnm_handle *h, double f, double W, int32_t n)
{
    return guarded(h, [&](cnm::Solver &s) { s.build_cap(f, W, n); });
}

int cnm_prepare_run(cnm_handle *h, int32_t n_steps, double r_ex)
{
    return guarded(h, [&](cnm::Solver &s) { s.prepare_run(n_steps, r_ex); });
}

int cnm_refresh(cnm_handle *h, double time)
{
    return guarded(h, [&](cnm::Solver &s) {
        s.build_time_dependent_perturbation(time);
        s.sync();
    });
}

int cnm_step(cnm_handle *h, int32_t step_id, cnm_diag *d, double *ef, double *fl, double *nm, double *en)
{
    return guarded(h, [&](cnm::Solver &s) { s.step(step_id, d, ef, fl, nm, en); });
}

int cnm_should_stop(const cnm_handle *h, int32_t *stop)
{
    if (!h || !stop) return CNM_EINVAL;
    const cnm::Solver &s = *h->s;
    *stop = (!s.isolated && s.evolve_orbit && s.R <= 6.0) ? 1 : 0;
    return CNM_OK;
}

int cnm_apply(cnm_handle *h, int32_t op, const double *x, double *y)
{
    return guarded(h, [&](cnm::Solver &s) { s.apply_op(op, x, y); });
}

int cnm_apply_lowp(cnm_handle *h, int32_t op, const double *x, double *y)
{
    return guarded(h, [&](cnm::Solver &s) { s.apply_lowp(op, x, y); });
}

int cnm_mixed_info(const cnm_handle *h, int32_t *passes, int32_t *fp64_applies, double *residual)
{
    return guarded(const_cast<cnm_handle *>(h), [&](cnm::Solver &s) {
        if (passes) *passes = s.mx_passes;
        if (fp64_applies) *fp64_applies = s.mx_fp64;
        if (residual) *residual = s.mx_residual;
    });
}

int cnm_tc_blocks(const cnm_handle *h, int32_t *kp, int32_t *nblk, int32_t *lc_min, int32_t *nt)
{
    return guarded(const_cast<cnm_handle *>(h), [&](cnm::Solver &s) {
        if (!s.mixed) throw cnm::Error(CNM_ELOGIC, "no tensor-core operator on an fp64 handle");
        if (kp) *kp = s.tg.kp;
        if (nblk)
            for (int l = 0; l < s.K; ++l) nblk[l] = s.tg.l_nblk[l];
        if (lc_min) *lc_min = std::max(1, s.tcp.gst - 2);
        if (nt) *nt = s.tcp.nt;
    });
}

int cnm_launch_count(const cnm_handle *h, int64_t *count)
{
    return guarded(const_cast<cnm_handle *>(h), [&](cnm::Solver &s) { *count = s.n_launches; });
}

int cnm_mixed_trace(const cnm_handle *h, double *out)
{
    return guarded(const_cast<cnm_handle *>(h), [&](cnm::Solver &s) {
        for (int q = 0; q < 6; ++q) out[q] = s.mx_trace[q];
    });
}

int cnm_sink_strength(const cnm_handle *h, int32_t body, double *out)
{
    return guarded(const_cast<cnm_handle *>(h), [&](cnm::Solver &s) { *out = s.sink_strength(body); });
}

int cnm_sink_active(const cnm_handle *h, int32_t *active)
{
    if (!h || !active) return CNM_EINVAL;
    *active = h->s->sink_active ? 1 : 0;
    return CNM_OK;
}

int cnm_sink_vector(const cnm_handle *h, int32_t body, double *out)
{
    return guarded(const_cast<cnm_handle *>(h), [&](cnm::Solver &s) {
        const cnm::Absorber &ab = body == 1 ? s.abs1 : s.abs2;
        if (ab.v.p) cnm::cuda_check(cudaMemcpy(out, ab.v.p, s.nN * sizeof(double2), cudaMemcpyDeviceToHost), "cudaMemcpy");
        else std::fill(out, out + 2 * s.nN, 0.0);
    });
}

int cnm_save_checkpoint(const cnm_handle *h, int32_t step_id, void *buf, int64_t capacity, int64_t *size)
{
    return guarded(const_cast<cnm_handle *>(h), [&](cnm::Solver &s) {
        const std::vector<char> blob = s.checkpoint(step_id);
        *size = (int64_t)blob.size();
        if (buf) {
            if (capacity < (int64_t)blob.size()) throw cnm::Error(CNM_EINVAL, "checkpoint buffer too small");
            std::memcpy(buf, blob.data(), blob.size());
        }
    });
}

int cnm_load_checkpoint(cnm_handle *h, int32_t step_id, const void *buf, int64_t size, int32_t *loaded)
{
    return guarded(h, [&](cnm::Solver &s) {
        *loaded = (buf && size > 0 && s.restore(step_id, static_cast<const char *>(buf), (size_t)size)) ? 1 : 0;
    });
}

int cnm_replay_power_average(cnm_handle *h, const double *times, const double *phases, const double *values,
                             int32_t n)
{
    return guarded(h, [&](cnm::Solver &s) {
        if (n < 0 || (n > 0 && (!times || !phases || !values))) throw cnm::Error(CNM_EINVAL, "bad samples");
        s.power_average = cnm::RollingPhaseAverage(s.orbits_average);
        for (int32_t k = 0; k < n; ++k) s.power_average.update(times[k], phases[k], values[k]);
    });
}

int cnm_set_profiling(cnm_handle *h, int32_t on)
{
    return guarded(h, [&](cnm::Solver &s) {
        s.kt_flush();
        s.profiling = on != 0;
        for (cnm::KernelTimer &t : s.ktime) {
            t.ms = 0.0;
            t.launches = 0;
            t.used = 0;
        }
    });
}

int cnm_kernel_times(cnm_handle *h, int32_t which, double *total_ms, int64_t *launches)
{
    return guarded(h, [&](cnm::Solver &s) {
        if (which < 0 || which >= cnm::TK_COUNT) throw cnm::Error(CNM_EINVAL, "unknown kernel class");
        s.kt_flush();
        *total_ms = s.ktime[which].ms;
        *launches = s.ktime[which].launches;
    });
}

int cnm_timer_start(cnm_handle *h)
{
    return guarded(h, [&](cnm::Solver &s) {
        if (!s.region_a) {
            CK(cudaEventCreate(&s.region_a));
            CK(cudaEventCreate(&s.region_b));
        }
        CK(cudaEventRecord(s.region_a, s.stream));
    });
}

int cnm_timer_stop(cnm_handle *h, double *ms)
{
    return guarded(h, [&](cnm::Solver &s) {
        if (!s.region_a) throw cnm::Error(CNM_ELOGIC, "cnm_timer_start was not called");
        CK(cudaEventRecord(s.region_b, s.stream));
        CK(cudaEventSynchronize(s.region_b));
        float f = 0.f;
        CK(cudaEventElapsedTime(&f, s.region_a, s.region_b));
        *ms = f;
    });
}

int cnm_hydrogenic_state(const double *r, int32_t Nr, const int32_t *l, const int32_t *m, int32_t n_modes, double mu,
                         double M1, double x_center, int32_t n, int32_t la, int32_t ma, int32_t n_theta, int32_t n_phi,
                         double *state)
{
    std::string err;
    const int rc = cnm::hydrogenic_state(r, Nr, l, m, n_modes, mu, M1, x_center, n, la, ma, n_theta, n_phi, state, err);
    if (rc != CNM_OK) g_create_error = err;
    return rc;
}

int cnm_displaced_100_state(const double *r, int32_t Nr, const int32_t *l, const int32_t *m, int32_t n_modes,
                            double mu, double x_bh, double *state)
{
    try {
        if (!r || !l || !m || !state || !std::isfinite(mu) || mu <= 0 || !std::isfinite(x_bh) || Nr < 3 || n_modes < 1)
            throw cnm::Error(CNM_EINVAL, "Invalid displaced 100 state parameters");
        for (int i = 0; i < Nr; ++i)
            if (!std::isfinite(r[i]) || r[0] < 0)
                throw cnm::Error(CNM_EINVAL, "Radial coordinates must be finite and nonnegative");
        for (int i = 1; i < Nr; ++i)
            if (r[i] <= r[i - 1]) throw cnm::Error(CNM_EINVAL, "Radial coordinates must increase");
        int lmax = 0;
        for (int j = 0; j < n_modes; ++j) {
            if (l[j] < 0 || std::abs(m[j]) > l[j]) throw cnm::Error(CNM_EINVAL, "Invalid spherical harmonic mode");
            lmax = std::max(lmax, (int)l[j]);
        }
        const double a0 = 1.0 / (mu * mu), distance = std::abs(x_bh);
        const double amplitude = 1.0 / std::sqrt(M_PI * a0 * a0 * a0);
        const int nq = std::max(128, 2 * lmax + 32);
        std::vector<double> gx, gw;
        cnm::gauss_legendre01(nq, gx, gw);
        cnm::DevBuf<double> d_r, d_gx, d_gw, d_mom;
        d_r.alloc(Nr);
        d_gx.alloc(nq);
        d_gw.alloc(nq);
        d_mom.alloc((size_t)(lmax + 1) * Nr);
        CK(cudaMemcpy(d_r.p, r, Nr * sizeof(double), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d_gx.p, gx.data(), nq * sizeof(double), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d_gw.p, gw.data(), nq * sizeof(double), cudaMemcpyHostToDevice));
        const int threads = (nq + 31) / 32 * 32;
        const size_t smem = (size_t)(lmax + 1) * (threads / 32) * sizeof(double);
        cnm::k_displaced_100<<<Nr - 2, threads, smem>>>(d_r.p, Nr, lmax, a0, distance, amplitude, nq, d_gx.p, d_gw.p,
                                                        d_mom.p);
        CK(cudaGetLastError());
        std::vector<double> mom((size_t)(lmax + 1) * Nr);
        CK(cudaMemcpy(mom.data(), d_mom.p, mom.size() * sizeof(double), cudaMemcpyDeviceToHost));
        std::fill(state, state + 2 * (int64_t)Nr * n_modes, 0.0);
        for (int j = 0; j < n_modes; ++j) {
            // Y*_lm(pi/2, phi_BH) with phi_BH = 0 or pi (real, exact parity)
            double y = cnm::sph_plm_equator(l[j], std::abs(m[j]));
            if (m[j] < 0 && (std::abs(m[j]) & 1)) y = -y;
            if (x_bh < 0 && (std::abs(m[j]) & 1)) y = -y;
            for (int i = 1; i < Nr - 1; ++i)
                state[2 * ((int64_t)j * Nr + i)] = r[i] * mom[(size_t)l[j] * Nr + i] * y;
        }
        return CNM_OK;
    } catch (const cnm::Error &e) {
        g_create_error = e.what();
        return e.code;
    } catch (const std::exception &e) {
        g_create_error = e.what();
        return CNM_ECUDA;
    }
}

struct cnm_batch {
    std::vector<cnm_handle *> hs;
};

int cnm_batch_create(const cnm_params *params, int32_t count, cnm_batch **out)
{
    if (!params || !out || count < 1) {
        g_create_error = "cnm_batch_create: need params[count >= 1] and an output pointer";
        return CNM_EINVAL;
    }
    cnm_batch *b = new cnm_batch();
    for (int32_t i = 0; i < count; ++i) {
        cnm_handle *h = nullptr;
        const int rc = cnm_create(&params[i], &h);
        if (rc != CNM_OK) {
            for (cnm_handle *q : b->hs) cnm_destroy(q);
            delete b;
            g_create_error = "binary " + std::to_string(i) + ": " + g_create_error;
            return rc;
        }
        b->hs.push_back(h);
    }
    *out = b;
    return CNM_OK;
}

int cnm_batch_size(const cnm_batch *b, int32_t *count)
{
    if (!b || !count) return CNM_EINVAL;
    *count = (int32_t)b->hs.size();
    return CNM_OK;
}

int cnm_batch_handle(cnm_batch *b, int32_t index, cnm_handle **h)
{
    if (!b || !h || index < 0 || index >= (int32_t)b->hs.size()) return CNM_EINVAL;
    *h = b->hs[(size_t)index];
    return CNM_OK;
}

int cnm_batch_step(cnm_batch *b, int32_t step_id, cnm_diag *diags)
{
    if (!b) return CNM_EINVAL;
    const size_t n = b->hs.size();
    std::vector<int> rc(n, CNM_OK);
    for (size_t i = 0; i < n; ++i)
        rc[i] = guarded(b->hs[i], [&](cnm::Solver &s) { s.step_begin(step_id); });
    for (size_t i = 0; i < n; ++i)
        if (rc[i] == CNM_OK)
            rc[i] = guarded(b->hs[i], [&](cnm::Solver &s) {
                s.step_end(step_id, diags ? &diags[i] : nullptr, nullptr, nullptr, nullptr, nullptr);
            });
    for (size_t i = 0; i < n; ++i)
        if (rc[i] != CNM_OK) return rc[i];
    return CNM_OK;
}

int cnm_batch_destroy(cnm_batch *b)
{
    if (!b) return CNM_EINVAL;
    for (cnm_handle *h : b->hs) cnm_destroy(h);
    delete b;
    return CNM_OK;
}

int cnm_set_operator_kernel(cnm_handle *h, int32_t specialised)
{
    return guarded(h, [&](cnm::Solver &s) { s.a5_enabled = specialised != 0; });
}

int cnm_measure_fp64_peak(double *tflops)
{
    if (!tflops) return CNM_EINVAL;
    try {
        int dev = 0, nsm = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        double *buf = nullptr;
        CK(cudaMalloc(&buf, sizeof(double) * 4 * nsm));
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        const int blocks = 4 * nsm, threads = 512, iters = 1 << 14;
        cnm::k_fp64_peak<<<blocks, threads>>>(buf, 256, 1.0000001, 1e-12);  // warm-up
        CK(cudaGetLastError());
        float best = 1e30f;
        for (int rep = 0; rep < 5; ++rep) {
            CK(cudaEventRecord(e0));
            cnm::k_fp64_peak<<<blocks, threads>>>(buf, iters, 1.0000001, 1e-12);
            CK(cudaEventRecord(e1));
            CK(cudaEventSynchronize(e1));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            best = std::min(best, ms);
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaFree(buf);
        const double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
        *tflops = flops / (best * 1e-3) / 1e12;
        return CNM_OK;
    } catch (const cnm::Error &e) {
        g_create_error = e.what();
        return e.code;
    } catch (const std::exception &e) {
        g_create_error = e.what();
        return CNM_ECUDA;
    }
}

int cnm_host_alloc(int64_t bytes, void **ptr)
{
    if (!ptr) return CNM_EINVAL;
    *ptr = nullptr;
    if (bytes <= 0) return CNM_EINVAL;
    const cudaError_t e = cudaMallocHost(ptr, (size_t)bytes);
    if (e != cudaSuccess) {
        *ptr = nullptr;
        cudaGetLastError();
        g_create_error = std::string("cudaMallocHost failed: ") + cudaGetErrorString(e);
        return CNM_ECUDA;
    }
    return CNM_OK;
}

int cnm_host_free(void *ptr)
{
    if (!ptr) return CNM_OK;
    return cudaFreeHost(ptr) == cudaSuccess ? CNM_OK : CNM_ECUDA;
}

int cnm_device_name(char *name, int32_t size)
{
    if (!name || size < 1) return CNM_EINVAL;
    int dev = 0;
    cudaDeviceProp prop;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
        g_create_error = "cudaGetDeviceProperties failed";
        return CNM_ECUDA;
    }
    std::snprintf(name, (size_t)size, "%s", prop.name);
    return CNM_OK;
}

int cnm_autotune(cnm_handle *h, int32_t *apply_groups, int32_t *tc_stages)
{
    return guarded(h, [&](cnm::Solver &s) {
        int g = 0, st = 0;
        s.autotune(&g, &st);
        if (apply_groups) *apply_groups = g;
        if (tc_stages) *tc_stages = st;
    });
}

int cnm_set_tuning(cnm_handle *h, int32_t apply_groups, int32_t tc_stages)
{
    return guarded(h, [&](cnm::Solver &s) { s.set_tuning(apply_groups, tc_stages); });
}

int cnm_plan_info(const cnm_handle *h, int32_t *scan_per, int32_t *scan_cluster, int32_t *apply_groups,
                  int32_t *apply_weights_in_smem)
{
    if (!h || !h->s) return CNM_EINVAL;
    const cnm::Solver &s = *h->s;
    if (scan_per) *scan_per = s.pcl_per;
    if (scan_cluster) *scan_cluster = s.pcl_cs;
    const bool a5 = s.a5_groups > 0 && s.a5_enabled;
    if (apply_groups) *apply_groups = a5 ? s.a5_groups : s.plan3.n_groups;
    if (apply_weights_in_smem) *apply_weights_in_smem = a5 || s.apply3_gsm ? 1 : 0;
    return CNM_OK;
}

}  // extern "C"

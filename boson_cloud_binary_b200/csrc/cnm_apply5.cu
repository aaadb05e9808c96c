// cnm_apply5.cu -- the CN operator kernel specialised at compile time for l_max <= 8.
//
// One node per thread.  The rows (modes) are split into G contiguous groups of about
// equal cost; CTA (node tile, group) keeps the accumulators of its group's rows for its
// nodes in registers and streams over the columns: for column k it loads
// z_k = e^{i m_k theta} x_k once and, for every row j of the group,
//     a   = sum_s g[j, k, s] h_{|l_j - l_k| + 2 s}(r)      (Ahat_jk at this node)
//     acc += a z_k.
// Row degrees, term counts and table offsets are compile-time constants, so the row
// loop and the term loops unroll completely: the instruction stream is the FP64 FMAs
// plus one broadcast shared-memory load per two Gaunt weights.  The group's weights are
// staged in shared memory ([column degree l1][column][row][s], s padded to even).
// The epilogue (stencil, centrifugal term, CAP, sinks, fused inner products and their
// completion) follows the generic kernel k_apply3 node for node.
#include "cnm_device.cuh"
#include "cnm_apply5.cuh"

#include <cuda_runtime.h>

namespace cnm {

namespace {

constexpr int A5_THREADS = 128;

// This thread's column values x_k(r_i), consumed in mode order k = 0, 1, ..., n-1 across
// the degree blocks; every load is issued three columns ahead of its use, so the column
// stream does not wait on L2 latency.
struct XQueue {
    double2 q0, q1, q2;
    const double2 *__restrict__ xp;  // x + i
    int Nr, nm;
    bool active;
    __device__ __forceinline__ double2 ld(int k) const
    {
        return (active && k < nm) ? xp[(int64_t)k * Nr] : cmake(0.0, 0.0);
    }
    __device__ __forceinline__ void init(const double2 *x, int i, int Nr_, int nm_, bool active_)
    {
        xp = x + i;
        Nr = Nr_;
        nm = nm_;
        active = active_;
        q0 = ld(0);
        q1 = ld(1);
        q2 = ld(2);
    }
    __device__ __forceinline__ double2 pop(int k)
    {
        const double2 v = q0;
        q0 = q1;
        q1 = q2;
        q2 = ld(k + 3);
        return v;
    }
};

template <int L, int G, int GR, int J, int J1>
struct Rows {
    // acc[j - J0] += (sum_s g h) z for rows J .. J1-1 of one column of degree L1
    template <int L1, int J0>
    static __device__ __forceinline__ void column(const double *__restrict__ gc, const double (&h)[2 * L + 1],
                                                  double2 z, double2 (&acc)[A5Layout<L, G>::nrows(GR)])
    {
        if constexpr (J < J1) {
            constexpr int lj = A5Layout<L, G>::l_of(J);
            constexpr int L0 = lj > L1 ? lj - L1 : L1 - lj;
            constexpr int S = A5Layout<L, G>::spad(lj, L1);
            constexpr int RO = A5Layout<L, G>::rowoff(GR, L1, J);
            double a0, a1 = 0.0;
            {
                const double2 g01 = *reinterpret_cast<const double2 *>(gc + RO);
                a0 = g01.x * h[L0];
                if constexpr (S > 1) a1 = g01.y * h[L0 + 2];
            }
#pragma unroll
            for (int s = 2; s < S; s += 2) {
                const double2 gg = *reinterpret_cast<const double2 *>(gc + RO + s);
                a0 = fma(gg.x, h[L0 + 2 * s], a0);
                if (s + 1 < S) a1 = fma(gg.y, h[L0 + 2 * s + 2], a1);
            }
            const double av = a0 + a1;
            acc[J - J0].x = fma(av, z.x, acc[J - J0].x);
            acc[J - J0].y = fma(av, z.y, acc[J - J0].y);
            Rows<L, G, GR, J + 1, J1>::template column<L1, J0>(gc, h, z, acc);
        }
    }
};

template <int L, int G, int GR, int L1>
struct Cols {
    static __device__ __forceinline__ void run(const double *gs, const double2 *ph, XQueue &xq,
                                               const double (&h)[2 * L + 1],
                                               double2 (&acc)[A5Layout<L, G>::nrows(GR)])
    {
        if constexpr (L1 <= L) {
            using Lay = A5Layout<L, G>;
            constexpr int J0 = Lay::first(GR), J1 = Lay::first(GR + 1);
            constexpr int CB = Lay::colbase(GR, L1), CS = Lay::colsize(GR, L1), K0 = Lay::loff(L1);
#pragma unroll 1
            for (int c = 0; c <= L1; ++c) {
                const int k = K0 + c;
                const double2 xv = xq.pop(k);
                const double2 z = cmul(ph[k], xv);
                Rows<L, G, GR, J0, J1>::template column<L1, J0>(gs + CB + c * CS, h, z, acc);
            }
            Cols<L, G, GR, L1 + 1>::run(gs, ph, xq, h, acc);
        }
    }
};

template <int L, int G, int GR, int J, int J1>
struct Epi {
    static __device__ __forceinline__ void run(const Grid &g, const ApplyArgs &a, const double2 *ph, int i,
                                               bool active, bool interior, double alpha_d, double inv2mu,
                                               const double2 (&acc)[A5Layout<L, G>::nrows(GR)], double (&dacc)[4])
    {
        if constexpr (J < J1) {
            using Lay = A5Layout<L, G>;
            constexpr int J0 = Lay::first(GR);
            constexpr int lj = Lay::l_of(J);
            const int Nr = g.Nr;
            if (active) {
                const double2 *xr = a.x + (int64_t)J * Nr;
                const double2 xv = xr[i];
                double2 hv = cmake(0.0, 0.0);
                if (a.use_h0 && interior) {
                    const double diag = (2.0 * alpha_d + (double)(lj * (lj + 1)) * g.ir2[i]) * inv2mu;
                    const double off = -alpha_d * inv2mu;
                    hv = cadd(cscale(xv, diag), cscale(cadd(xr[i - 1], xr[i + 1]), off));
                }
                if (interior) hv = cadd(hv, cmul(cconj(ph[J]), acc[J - J0]));
                if (a.use_cap && g.capw) hv = cadd(hv, cmake(g.capw[i] * xv.y, -g.capw[i] * xv.x));
                double2 y = cadd(cmul(a.alpha, xv), cmul(a.beta, hv));
                for (int s2 = 0; s2 < a.n_sinks; ++s2)
                    if (i >= a.sink_lo[s2] && i < a.sink_hi[s2])
                        y = cadd(y, cmul(cscale(a.sink_dots[s2], a.sink_coef[s2]), a.sink_v[s2][(int64_t)J * Nr + i]));
                a.y[(int64_t)J * Nr + i] = y;
                for (int q = 0; q < a.n_dots; ++q) {
                    double2 d;
                    const int64_t e = (int64_t)J * Nr + i;
                    if (a.dot_kind[q] == 1) d = cconjmul(a.dot_ext[q][e], y);
                    else if (a.dot_kind[q] == 2) d = cconjmul(y, a.dot_ext[q][e]);
                    else if (a.dot_kind[q] == 4)
                        d = cmake(cabs2(csub(cscale(y, a.scale_kr ? a.scale_kr->rhs_norm : a.dot_scale), a.dot_ext[q][e])),
                                  0.0);
                    else d = cmake(cabs2(y), 0.0);
                    dacc[2 * q] += d.x;
                    dacc[2 * q + 1] += d.y;
                }
            }
            Epi<L, G, GR, J + 1, J1>::run(g, a, ph, i, active, interior, alpha_d, inv2mu, acc, dacc);
        }
    }
};

// ---- diagnostics pass: the same column stream with a second accumulator for dV/dt

template <int L, int G, int GR, int J, int J1>
struct RowsD {
    template <int L1, int J0>
    static __device__ __forceinline__ void column(const double *__restrict__ gc, const double (&h)[2 * L + 1],
                                                  double2 z, double2 zm,
                                                  double2 (&acc)[A5Layout<L, G>::nrows(GR)],
                                                  double2 (&accm)[A5Layout<L, G>::nrows(GR)])
    {
        if constexpr (J < J1) {
            constexpr int lj = A5Layout<L, G>::l_of(J);
            constexpr int L0 = lj > L1 ? lj - L1 : L1 - lj;
            constexpr int S = A5Layout<L, G>::spad(lj, L1);
            constexpr int RO = A5Layout<L, G>::rowoff(GR, L1, J);
            double a0, a1 = 0.0;
            {
                const double2 g01 = *reinterpret_cast<const double2 *>(gc + RO);
                a0 = g01.x * h[L0];
                if constexpr (S > 1) a1 = g01.y * h[L0 + 2];
            }
#pragma unroll
            for (int s = 2; s < S; s += 2) {
                const double2 gg = *reinterpret_cast<const double2 *>(gc + RO + s);
                a0 = fma(gg.x, h[L0 + 2 * s], a0);
                if (s + 1 < S) a1 = fma(gg.y, h[L0 + 2 * s + 2], a1);
            }
            const double av = a0 + a1;
            acc[J - J0].x = fma(av, z.x, acc[J - J0].x);
            acc[J - J0].y = fma(av, z.y, acc[J - J0].y);
            accm[J - J0].x = fma(av, zm.x, accm[J - J0].x);
            accm[J - J0].y = fma(av, zm.y, accm[J - J0].y);
            RowsD<L, G, GR, J + 1, J1>::template column<L1, J0>(gc, h, z, zm, acc, accm);
        }
    }
};

template <int L, int G, int GR, int L1>
struct ColsD {
    static __device__ __forceinline__ void run(const double *gs, const double2 *ph, XQueue &xq,
                                               const double (&h)[2 * L + 1],
                                               double2 (&acc)[A5Layout<L, G>::nrows(GR)],
                                               double2 (&accm)[A5Layout<L, G>::nrows(GR)])
    {
        if constexpr (L1 <= L) {
            using Lay = A5Layout<L, G>;
            constexpr int J0 = Lay::first(GR), J1 = Lay::first(GR + 1);
            constexpr int CB = Lay::colbase(GR, L1), CS = Lay::colsize(GR, L1), K0 = Lay::loff(L1);
#pragma unroll 1
            for (int c = 0; c <= L1; ++c) {
                const int k = K0 + c;
                const double2 xv = xq.pop(k);
                const double2 z = cmul(ph[k], xv);
                const double mk = (double)(2 * c - L1);
                RowsD<L, G, GR, J0, J1>::template column<L1, J0>(gs + CB + c * CS, h, z, cscale(z, mk), acc, accm);
            }
            ColsD<L, G, GR, L1 + 1>::run(gs, ph, xq, h, acc, accm);
        }
    }
};

template <int L, int G, int GR, int J, int J1>
struct EpiD {
    static __device__ __forceinline__ void run(const Grid &g, const DiagArgs &d, const double2 *ph, int i,
                                               bool active, bool interior, double alpha_d, double inv2mu,
                                               const double2 (&acc)[A5Layout<L, G>::nrows(GR)],
                                               const double2 (&accm)[A5Layout<L, G>::nrows(GR)], double *red,
                                               int lane, int warp, int nw, double &e_edge, double &pb, double &dv)
    {
        if constexpr (J < J1) {
            using Lay = A5Layout<L, G>;
            constexpr int J0 = Lay::first(GR);
            constexpr int lj = Lay::l_of(J), mj = Lay::m_of(J);
            constexpr int NM = Lay::nm();
            const int Nr = g.Nr;
            double nrm = 0.0, en = 0.0;
            if (active) {
                const double2 *xr = d.psi + (int64_t)J * Nr;
                const double2 xv = xr[i];
                double2 hx = cmake(0.0, 0.0), vx = cmake(0.0, 0.0), dx = cmake(0.0, 0.0);
                if (interior) {
                    const double diag = (2.0 * alpha_d + (double)(lj * (lj + 1)) * g.ir2[i]) * inv2mu;
                    const double off = -alpha_d * inv2mu;
                    hx = cadd(cscale(xv, diag), cscale(cadd(xr[i - 1], xr[i + 1]), off));
                    const double2 a = acc[J - J0], am = accm[J - J0];
                    vx = cmul(cconj(ph[J]), a);
                    dx = cmul(cconj(ph[J]), cmuli(cscale(cmake(am.x - mj * a.x, am.y - mj * a.y), d.domega)));
                    hx = cadd(hx, vx);
                }
                if (g.capw) hx = cadd(hx, cmake(g.capw[i] * xv.y, -g.capw[i] * xv.x));
                double2 dp = cmake(hx.y, -hx.x);  // -i H psi
                if (d.n_sinks > 0 && i >= d.slo0 && i < d.shi0)
                    dp = cadd(dp, cmul(cscale(d.sink_dots[0], d.sink_coef0), d.sv0[(int64_t)J * Nr + i]));
                if (d.n_sinks > 1 && i >= d.slo1 && i < d.shi1)
                    dp = cadd(dp, cmul(cscale(d.sink_dots[1], d.sink_coef1), d.sv1[(int64_t)J * Nr + i]));
                const double ce = cconjmul(xv, hx).x;
                if (i < d.idx_ex) {
                    nrm = cabs2(xv);
                    en = ce;
                } else {
                    e_edge += ce;
                    d.dpsi_edge[J] = dp;
                    d.psi_edge[3 * J] = xr[i - 1];
                    d.psi_edge[3 * J + 1] = xv;
                    d.psi_edge[3 * J + 2] = xr[i + 1];
                }
                pb += cconjmul(xv, dx).x;
                dv += cconjmul(dp, vx).x;
            }
            nrm = warp_sum(nrm);
            en = warp_sum(en);
            if (lane == 0) {
                red[J * nw + warp] = nrm;
                red[(NM + J) * nw + warp] = en;
            }
            EpiD<L, G, GR, J + 1, J1>::run(g, d, ph, i, active, interior, alpha_d, inv2mu, acc, accm, red, lane, warp,
                                           nw, e_edge, pb, dv);
        }
    }
};

template <int L, int G, int GR>
__device__ __forceinline__ void diag_body(const Grid &g, const double *gtab, const DiagArgs &d, double *gs,
                                          double2 *ph, double *red)
{
    using Lay = A5Layout<L, G>;
    constexpr int J0 = Lay::first(GR), J1 = Lay::first(GR + 1), NR = J1 - J0;
    constexpr int GS = Lay::gsize(GR), GB = Lay::gbase(GR);
    constexpr int NM = Lay::nm(), K = 2 * L + 1;
    const int Nr = g.Nr, lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    {
        const double2 *src = reinterpret_cast<const double2 *>(gtab + GB);
        for (int e = threadIdx.x; e < GS / 2; e += blockDim.x) reinterpret_cast<double2 *>(gs)[e] = src[e];
    }
    for (int k = threadIdx.x; k < NM; k += blockDim.x) {
        double sn, cs;
        sincos((double)Lay::m_of(k) * d.theta, &sn, &cs);
        ph[k] = cmake(cs, sn);
    }
    for (int e = threadIdx.x; e < (2 * NM + 3) * nw; e += blockDim.x) red[e] = 0.0;
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < Nr && i <= d.idx_ex, interior = i >= 1 && i <= Nr - 2;
    double h[K];
#pragma unroll
    for (int l = 0; l < K; ++l) h[l] = active ? d.hh[(int64_t)l * Nr + i] : 0.0;
    double2 acc[NR], accm[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) acc[r] = accm[r] = cmake(0.0, 0.0);
    XQueue xq;
    xq.init(d.psi, i, Nr, NM, active);
    ColsD<L, G, GR, 0>::run(gs, ph, xq, h, acc, accm);
    const double alpha_d = 1.0 / (g.dr * g.dr), inv2mu = 1.0 / (2 * g.mu);
    double e_edge = 0.0, pb = 0.0, dv = 0.0;
    EpiD<L, G, GR, J0, J1>::run(g, d, ph, i, active, interior, alpha_d, inv2mu, acc, accm, red, lane, warp, nw,
                                e_edge, pb, dv);
    e_edge = warp_sum(e_edge);
    pb = warp_sum(pb);
    dv = warp_sum(dv);
    if (lane == 0) {
        red[(2 * NM) * nw + warp] = e_edge;
        red[(2 * NM + 1) * nw + warp] = pb;
        red[(2 * NM + 2) * nw + warp] = dv;
    }
    __syncthreads();
    const int nblocks = gridDim.x * gridDim.y, blk = blockIdx.y * gridDim.x + blockIdx.x;
    for (int q = threadIdx.x; q < 2 * NM + 3; q += blockDim.x) {
        double sm = 0.0;
        for (int w = 0; w < nw; ++w) sm += red[q * nw + w];
        d.partials[(int64_t)q * nblocks + blk] = sm;
    }
}

template <int L, int G, int GR>
__device__ __forceinline__ void diag_dispatch(int grp, const Grid &g, const double *gtab, const DiagArgs &d,
                                              double *gs, double2 *ph, double *red)
{
    if constexpr (GR < G) {
        if (grp == GR) diag_body<L, G, GR>(g, gtab, d, gs, ph, red);
        else diag_dispatch<L, G, GR + 1>(grp, g, gtab, d, gs, ph, red);
    }
}

template <int L>
__global__ void __launch_bounds__(A5_THREADS) k_diag5(Grid g, const double *gtab, DiagArgs d)
{
    pdl_wait();
    if (d.gate && gate_closed(d.gate, GATE_ACCEPTED)) return;
    constexpr int G = D5Groups<L>::value;
    using Lay = A5Layout<L, G>;
    extern __shared__ double smem5[];
    double *gs = smem5;
    double2 *ph = reinterpret_cast<double2 *>(smem5 + Lay::gsize_max());
    double *red = reinterpret_cast<double *>(ph + Lay::nm());
    diag_dispatch<L, G, 0>(blockIdx.y, g, gtab, d, gs, ph, red);
}

template <int L, int G, int GR>
__device__ __forceinline__ void group_body(const Grid &g, const double *gtab, const ApplyArgs &a, double *gs,
                                           double2 *ph, double *red)
{
    using Lay = A5Layout<L, G>;
    constexpr int J0 = Lay::first(GR), J1 = Lay::first(GR + 1), NR = J1 - J0;
    constexpr int GS = Lay::gsize(GR), GB = Lay::gbase(GR);
    constexpr int NM = Lay::nm(), K = 2 * L + 1;
    const int Nr = g.Nr;
    {
        const double2 *src = reinterpret_cast<const double2 *>(gtab + GB);
        for (int e = threadIdx.x; e < GS / 2; e += blockDim.x) reinterpret_cast<double2 *>(gs)[e] = src[e];
    }
    for (int k = threadIdx.x; k < NM; k += blockDim.x) {
        double sn, cs;
        sincos((double)Lay::m_of(k) * a.theta, &sn, &cs);
        ph[k] = cmake(cs, sn);
    }
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < Nr, interior = i >= 1 && i <= Nr - 2;
    double h[K];
#pragma unroll
    for (int l = 0; l < K; ++l) h[l] = active ? a.hh[(int64_t)l * Nr + i] : 0.0;
    double2 acc[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) acc[r] = cmake(0.0, 0.0);
    XQueue xq;
    xq.init(a.x, i, Nr, NM, active);
    Cols<L, G, GR, 0>::run(gs, ph, xq, h, acc);
    double dacc[4] = {0.0, 0.0, 0.0, 0.0};
    const double alpha_d = 1.0 / (g.dr * g.dr), inv2mu = 1.0 / (2 * g.mu);
    Epi<L, G, GR, J0, J1>::run(g, a, ph, i, active, interior, alpha_d, inv2mu, acc, dacc);
    if (a.n_dots > 0) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
        for (int q = 0; q < 4; ++q) dacc[q] = warp_sum(dacc[q]);
        if (lane == 0)
#pragma unroll
            for (int q = 0; q < 4; ++q) red[q * 32 + warp] = dacc[q];
        __syncthreads();
        const int nblocks = gridDim.x * gridDim.y, blk = blockIdx.y * gridDim.x + blockIdx.x;
        if (threadIdx.x < 2 * a.n_dots) {
            double sm = 0.0;
            for (int w = 0; w < nw; ++w) sm += red[threadIdx.x * 32 + w];
            a.dot_partials[(int64_t)threadIdx.x * nblocks + blk] = sm;
            if (a.stage >= 0) __threadfence();
        }
        if (a.stage >= 0) {
            __syncthreads();
            finish_stage(a.dot_partials, nblocks, 2 * a.n_dots, a.red, a.kr, a.stage, a.ticket, red + 4 * 32);
        }
    }
}

template <int L, int G, int GR>
__device__ __forceinline__ void dispatch(int grp, const Grid &g, const double *gtab, const ApplyArgs &a, double *gs,
                                         double2 *ph, double *red)
{
    if constexpr (GR < G) {
        if (grp == GR) group_body<L, G, GR>(g, gtab, a, gs, ph, red);
        else dispatch<L, G, GR + 1>(grp, g, gtab, a, gs, ph, red);
    }
}

template <int L>
__global__ void __launch_bounds__(A5_THREADS) k_apply5(Grid g, const double *gtab, ApplyArgs a)
{
    pdl_wait();
    if (a.gate && gate_closed(a.gate, a.gate_mode)) return;
    constexpr int G = A5Groups<L>::value;
    using Lay = A5Layout<L, G>;
    extern __shared__ double smem5[];
    __shared__ double red[10 * 32];
    double *gs = smem5;
    double2 *ph = reinterpret_cast<double2 *>(smem5 + Lay::gsize_max());
    dispatch<L, G, 0>(blockIdx.y, g, gtab, a, gs, ph, red);
}

}  // namespace

int apply5_groups(int l_max)
{
    switch (l_max) {
#define CNM_A5G(L) \
    case L: return A5Groups<L>::value;
        CNM_A5G(1) CNM_A5G(2) CNM_A5G(3) CNM_A5G(4) CNM_A5G(5) CNM_A5G(6) CNM_A5G(7) CNM_A5G(8)
#undef CNM_A5G
    default: return 0;
    }
}

int diag5_groups(int l_max)
{
    switch (l_max) {
#define CNM_D5G(L) \
    case L: return D5Groups<L>::value;
        CNM_D5G(1) CNM_D5G(2) CNM_D5G(3) CNM_D5G(4) CNM_D5G(5) CNM_D5G(6) CNM_D5G(7) CNM_D5G(8)
#undef CNM_D5G
    default: return 0;
    }
}

size_t apply5_smem(int l_max)
{
    switch (l_max) {
#define CNM_A5S(L) \
    case L: return (size_t)A5Layout<L, A5Groups<L>::value>::gsize_max() * sizeof(double) + (size_t)A5Layout<L, A5Groups<L>::value>::nm() * sizeof(double2);
        CNM_A5S(1) CNM_A5S(2) CNM_A5S(3) CNM_A5S(4) CNM_A5S(5) CNM_A5S(6) CNM_A5S(7) CNM_A5S(8)
#undef CNM_A5S
    default: return 0;
    }
}

std::vector<double> apply5_table(int l_max, int G, const Coupling &c)
{
    std::vector<double> t;
    if (G == 0) return t;
    const int n = c.n_modes, Lm = c.l_max;
    // dense (j, k) -> term vector over l*
    std::vector<std::vector<double>> dense((size_t)n * n);
    for (int j = 0; j < n; ++j)
        for (int p = c.pair_row_ptr[j]; p < c.pair_row_ptr[j + 1]; ++p) {
            std::vector<double> &v = dense[(size_t)j * n + c.pair_col[p]];
            v.assign(2 * Lm + 1, 0.0);
            for (int tt = c.pair_term_ptr[p]; tt < c.pair_term_ptr[p + 1]; ++tt) v[c.term_l[tt]] = c.term_g[tt];
        }
    const A5Host lay(l_max, G);
    t.assign((size_t)lay.gbase(G), 0.0);
    for (int gr = 0; gr < G; ++gr)
        for (int l1 = 0; l1 <= l_max; ++l1)
            for (int cc = 0; cc <= l1; ++cc) {
                const int k = l1 * (l1 + 1) / 2 + cc;
                const size_t base = (size_t)lay.gbase(gr) + lay.colbase(gr, l1) + (size_t)cc * lay.colsize(gr, l1);
                for (int j = lay.first(gr); j < lay.first(gr + 1); ++j) {
                    const int lj = lay.l_of(j);
                    const int L0 = lj > l1 ? lj - l1 : l1 - lj, S = lay.spad(lj, l1);
                    const std::vector<double> &v = dense[(size_t)j * n + k];
                    for (int s = 0; s < S; ++s)
                        t[base + lay.rowoff(gr, l1, j) + s] = v.empty() ? 0.0 : v[L0 + 2 * s];
                }
            }
    return t;
}

cudaError_t set_apply5_smem()
{
    cudaError_t e = cudaSuccess;
#define CNM_A5A(L) \
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_apply5<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)apply5_smem(L));
    CNM_A5A(1) CNM_A5A(2) CNM_A5A(3) CNM_A5A(4) CNM_A5A(5) CNM_A5A(6) CNM_A5A(7) CNM_A5A(8)
#undef CNM_A5A
    return e;
}

void launch_apply5(int l_max, cudaStream_t st, const Grid &g, const double *gtab, const ApplyArgs &a)
{
    const dim3 blocks((unsigned)((g.Nr + A5_THREADS - 1) / A5_THREADS), (unsigned)apply5_groups(l_max));
    const size_t smem = apply5_smem(l_max);
    switch (l_max) {
#define CNM_A5L(L) \
    case L: (void)launch_pdl(k_apply5<L>, blocks, dim3(A5_THREADS), smem, st, g, gtab, a); break;
        CNM_A5L(1) CNM_A5L(2) CNM_A5L(3) CNM_A5L(4) CNM_A5L(5) CNM_A5L(6) CNM_A5L(7) CNM_A5L(8)
#undef CNM_A5L
    default: break;
    }
}

size_t diag5_smem(int l_max)
{
    const int n = (l_max + 1) * (l_max + 2) / 2;
    size_t g = 0;
    switch (l_max) {
#define CNM_D5S(L) \
    case L: g = (size_t)A5Layout<L, D5Groups<L>::value>::gsize_max(); break;
        CNM_D5S(1) CNM_D5S(2) CNM_D5S(3) CNM_D5S(4) CNM_D5S(5) CNM_D5S(6) CNM_D5S(7) CNM_D5S(8)
#undef CNM_D5S
    default: return 0;
    }
    return g * sizeof(double) + (size_t)n * sizeof(double2) + (size_t)(2 * n + 3) * (A5_THREADS / 32) * sizeof(double);
}

cudaError_t set_diag5_smem()
{
    cudaError_t e = cudaSuccess;
#define CNM_D5A(L) \
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_diag5<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)diag5_smem(L));
    CNM_D5A(1) CNM_D5A(2) CNM_D5A(3) CNM_D5A(4) CNM_D5A(5) CNM_D5A(6) CNM_D5A(7) CNM_D5A(8)
#undef CNM_D5A
    return e;
}

unsigned launch_diag5(int l_max, cudaStream_t st, const Grid &g, const double *gtab, const DiagArgs &d)
{
    const int nodes = d.idx_ex + 1;
    const dim3 blocks((unsigned)((nodes + A5_THREADS - 1) / A5_THREADS), (unsigned)diag5_groups(l_max));
    const size_t smem = diag5_smem(l_max);
    switch (l_max) {
#define CNM_D5L(L) \
    case L: (void)launch_pdl(k_diag5<L>, blocks, dim3(A5_THREADS), smem, st, g, gtab, d); break;
        CNM_D5L(1) CNM_D5L(2) CNM_D5L(3) CNM_D5L(4) CNM_D5L(5) CNM_D5L(6) CNM_D5L(7) CNM_D5L(8)
#undef CNM_D5L
    default: return 0;
    }
    return blocks.x * blocks.y;
}

unsigned diag5_blocks(int l_max, int Nr)
{
    return diag5_groups(l_max) > 0 ? (unsigned)((Nr + A5_THREADS - 1) / A5_THREADS) * (unsigned)diag5_groups(l_max) : 0u;
}

unsigned apply5_blocks(int l_max, int Nr)
{
    return (unsigned)((Nr + A5_THREADS - 1) / A5_THREADS) * (unsigned)apply5_groups(l_max);
}

}  // namespace cnm

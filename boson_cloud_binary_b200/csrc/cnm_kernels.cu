// cnm_kernels.cu -- sm_100a kernels of the Crank-Nicolson step (FP64 drop-in path).
//
// Every kernel here is memory-streaming or FMA work on complex128 vectors in the
// reference's mode-major layout; see cnm_common.cuh for the data layout.
#include "cnm_kernels.cuh"
#include "cnm_device.cuh"

#include <cooperative_groups.h>
#include <cuda_runtime.h>

namespace cnm {

// ------------------------------------------------------------------ radial weights

__device__ void wood_setup_dev(Krylov *kr, const double2 *vw, double c0, double c1);
__device__ void wood_scalar_dev(Krylov *kr, int which, const double2 *proj);


// hh[l][i] = scale * (a1 F1_l(r_i) + a2 (-1)^l F2_l(r_i)) on interior nodes, zero on the
// two boundary nodes (the reference fills radial_f1/f2 for i = 1..Nr-2 only,
// src/CrankNicolsonModes_hamiltonian.cpp:178-185).
__global__ void k_hh_table(double *hh, const double *r, int Nr, int K, double R1, double R2, double q,
                           double scale, double a1, double a2)
{
    pdl_wait();
    // one node per thread; the radial factors r_<^l / r_>^(l+1) of both bodies
    // (_hamiltonian.cpp:12-42) by repeated multiplication with r_< / r_> over l
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Nr) return;
    if (i == 0 || i == Nr - 1) {
        for (int l = 0; l < K; ++l) hh[(int64_t)l * Nr + i] = 0.0;
        return;
    }
    const double ri = r[i];
    const double big1 = ri >= R1 ? ri : R1, small1 = ri >= R1 ? R1 : ri;
    const double big2 = ri >= R2 ? ri : R2, small2 = ri >= R2 ? R2 : ri;
    const double x1 = small1 / big1, x2 = small2 / big2;
    double f1 = 1 / (1 + q) / big1, f2 = 1.0 * q / (1 + q) / big2;
    for (int l = 0; l < K; ++l) {
        const double par = (l & 1) ? -1.0 : 1.0;
        hh[(int64_t)l * Nr + i] = scale * (a1 * f1 + a2 * par * f2);
        f1 *= x1;
        f2 *= x2;
    }
}

// ------------------------------------------------------------------ operator application

// ------------------------------------------------------------------ operator kernel, two nodes per thread

// Tiles of TILE3 = 64 nodes: lane l of every warp owns nodes l and l + 32, so each
// warp-uniform Gaunt weight loaded for a chunk of at most two rows feeds the FMA
// chains of both nodes.  z = D^dag x and the hh tile sit in shared memory; x itself
// is read through L1 where the stencil and the output need it.
constexpr int TILE3 = 64;

template <int S_EFF, int RB, bool DVDT, bool GSM>
__device__ __forceinline__ void coupling_block3(const double *__restrict__ g, int stride, int ncols, int col0,
                                                const double2 *zs, const double *hs_l0, const int *mode_m, int lane,
                                                double2 (&acc)[RB][2], double2 (&accm)[RB][2])
{
    double h0[S_EFF], h1[S_EFF];
#pragma unroll
    for (int s2 = 0; s2 < S_EFF; ++s2) {
        h0[s2] = hs_l0[2 * s2 * TILE3 + lane];
        h1[s2] = hs_l0[2 * s2 * TILE3 + lane + 32];
    }
    for (int kk = 0; kk < ncols; ++kk) {
        const double2 z0 = zs[(col0 + kk) * TILE3 + lane];
        const double2 z1 = zs[(col0 + kk) * TILE3 + lane + 32];
        const double *gk = g + kk * RB * stride;
        const double mk = DVDT ? (double)mode_m[col0 + kk] : 0.0;
#pragma unroll
        for (int rr = 0; rr < RB; ++rr) {
            const double *gr = gk + rr * stride;
            double a0 = 0.0, a1 = 0.0, b0 = 0.0, b1 = 0.0;
#pragma unroll
            for (int s2 = 0; s2 + 1 < S_EFF; s2 += 2) {
                const double2 gg = GSM ? *reinterpret_cast<const double2 *>(gr + s2)
                                       : __ldg(reinterpret_cast<const double2 *>(gr + s2));
                a0 = fma(gg.x, h0[s2], a0);
                a1 = fma(gg.y, h0[s2 + 1], a1);
                b0 = fma(gg.x, h1[s2], b0);
                b1 = fma(gg.y, h1[s2 + 1], b1);
            }
            if (S_EFF & 1) {
                const double gl = GSM ? gr[S_EFF - 1] : __ldg(gr + S_EFF - 1);
                a0 = fma(gl, h0[S_EFF - 1], a0);
                b0 = fma(gl, h1[S_EFF - 1], b0);
            }
            const double a = a0 + a1, b = b0 + b1;
            acc[rr][0].x = fma(a, z0.x, acc[rr][0].x);
            acc[rr][0].y = fma(a, z0.y, acc[rr][0].y);
            acc[rr][1].x = fma(b, z1.x, acc[rr][1].x);
            acc[rr][1].y = fma(b, z1.y, acc[rr][1].y);
            if (DVDT) {
                const double am = a * mk, bm = b * mk;
                accm[rr][0].x = fma(am, z0.x, accm[rr][0].x);
                accm[rr][0].y = fma(am, z0.y, accm[rr][0].y);
                accm[rr][1].x = fma(bm, z1.x, accm[rr][1].x);
                accm[rr][1].y = fma(bm, z1.y, accm[rr][1].y);
            }
        }
    }
}

// One (chunk, l1) block with its leading s_eff multipoles (dispatched to the compile-time width).
template <int SMAX, int RB, bool DVDT, bool GSM>
__device__ __forceinline__ void coupling_block_dispatch3(int s_eff, const double *g, int stride, int ncols, int col0,
                                                         const double2 *zs, const double *hs_l0, const int *mode_m,
                                                         int lane, double2 (&acc)[RB][2], double2 (&accm)[RB][2])
{
#define CNM_CASE3(S2)                                                                                            \
    case S2:                                                                                                     \
        if (S2 <= SMAX)                                                                                          \
            coupling_block3<(S2 <= SMAX ? S2 : 1), RB, DVDT, GSM>(g, stride, ncols, col0, zs, hs_l0, mode_m,    \
                                                                  lane, acc, accm);                              \
        break;
    switch (s_eff) {
        CNM_CASE3(1) CNM_CASE3(2) CNM_CASE3(3) CNM_CASE3(4) CNM_CASE3(5) CNM_CASE3(6) CNM_CASE3(7)
        CNM_CASE3(8) CNM_CASE3(9) CNM_CASE3(10) CNM_CASE3(11) CNM_CASE3(12) CNM_CASE3(13) CNM_CASE3(14)
        CNM_CASE3(15) CNM_CASE3(16) CNM_CASE3(17) CNM_CASE3(18) CNM_CASE3(19) CNM_CASE3(20) CNM_CASE3(21)
        CNM_CASE3(22) CNM_CASE3(23) CNM_CASE3(24) CNM_CASE3(25)
    default: break;
    }
#undef CNM_CASE3
}

template <int SMAX, int RB, bool DVDT, bool GSM>
__device__ __forceinline__ void coupling_chunk3(const BlockTable &bt, const double *gbase, int goff0, int l_max, int ci,
                                                int lcut, const double2 *zs, const double *hs, const int *mode_m,
                                                int lane, double2 (&acc)[RB][2], double2 (&accm)[RB][2])
{
#pragma unroll
    for (int rr = 0; rr < RB; ++rr) acc[rr][0] = acc[rr][1] = accm[rr][0] = accm[rr][1] = cmake(0.0, 0.0);
    if (lcut < 0) return;
    const int l = bt.chunk_l[ci];
    for (int l1 = 0; l1 <= l_max; ++l1) {
        const int L0 = abs(l - l1), S = min(l, l1) + 1;
        if (lcut < L0) continue;
        const int s_eff = min(S, (lcut - L0) / 2 + 1);
        const double *g = gbase + (bt.chunk_goff[ci * (l_max + 1) + l1] - goff0);
        const int stride = (S + 1) & ~1, col0 = bt.l_off[l1];
        coupling_block_dispatch3<SMAX, RB, DVDT, GSM>(s_eff, g, stride, l1 + 1, col0, zs, hs + L0 * TILE3, mode_m,
                                                      lane, acc, accm);
    }
}

// The output rows of one chunk at the lane's two nodes from the coupling sums acc (accm for
// dV/dt): stencil, centrifugal term, CAP, sinks, the store and the fused inner products.
template <int RB, int VP>
__device__ __forceinline__ void apply_epilogue3(const Grid &g, const CouplingTable &ct, const BlockTable &bt,
                                                const ApplyArgs &a, const double2 *ph, int lane, int i0, int ci,
                                                const double2 (&acc)[RB][2], const double2 (&accm)[RB][2],
                                                double (&dacc)[4])
{
    const int Nr = g.Nr;
    const double alpha_d = 1.0 / (g.dr * g.dr), inv2mu = 1.0 / (2 * g.mu);
#pragma unroll
    for (int rr = 0; rr < RB; ++rr) {
        const int j = bt.chunk_rows[ci * 2 + rr];
        const double2 *xr = a.x + (int64_t)j * Nr;
#pragma unroll
        for (int nb = 0; nb < 2; ++nb) {
            const int i = i0 + lane + 32 * nb;
            if (i >= Nr) continue;
            const bool interior = i >= 1 && i <= Nr - 2;
            const double2 xv = xr[i];
            double2 h = cmake(0.0, 0.0);
            if (a.use_h0 && interior) {
                const int l = ct.mode_l[j];
                const double diag = (2.0 * alpha_d + (double)(l * (l + 1)) * g.ir2[i]) * inv2mu;
                const double off = -alpha_d * inv2mu;
                h = cadd(cscale(xv, diag), cscale(cadd(xr[i - 1], xr[i + 1]), off));
            }
            if (VP != V_NONE && interior) {
                double2 vj;
                if (VP == V_DVDT) {
                    const double mj = (double)ct.mode_m[j];
                    vj = cmuli(cscale(cmake(accm[rr][nb].x - mj * acc[rr][nb].x, accm[rr][nb].y - mj * acc[rr][nb].y),
                                      a.domega));
                } else {
                    vj = acc[rr][nb];
                }
                h = cadd(h, cmul(cconj(ph[j]), vj));
            }
            if (a.use_cap && g.capw) h = cadd(h, cmake(g.capw[i] * xv.y, -g.capw[i] * xv.x));
            double2 y = cadd(cmul(a.alpha, xv), cmul(a.beta, h));
            for (int s2 = 0; s2 < a.n_sinks; ++s2)
                if (i >= a.sink_lo[s2] && i < a.sink_hi[s2])
                    y = cadd(y, cmul(cscale(a.sink_dots[s2], a.sink_coef[s2]), a.sink_v[s2][(int64_t)j * Nr + i]));
            a.y[(int64_t)j * Nr + i] = y;
            for (int q = 0; q < a.n_dots; ++q) {
                double2 d;
                if (a.dot_kind[q] == 1) d = cconjmul(a.dot_ext[q][(int64_t)j * Nr + i], y);
                else if (a.dot_kind[q] == 2) d = cconjmul(y, a.dot_ext[q][(int64_t)j * Nr + i]);
                else if (a.dot_kind[q] == 4)
                    d = cmake(cabs2(csub(cscale(y, a.scale_kr ? a.scale_kr->rhs_norm : a.dot_scale),
                                         a.dot_ext[q][(int64_t)j * Nr + i])),
                              0.0);
                else d = cmake(cabs2(y), 0.0);
                dacc[2 * q] += d.x;
                dacc[2 * q + 1] += d.y;
            }
        }
    }
}

template <int SMAX, int RB, int VP, bool GSM>
__device__ __forceinline__ void apply_chunk3(const Grid &g, const CouplingTable &ct, const BlockTable &bt,
                                             const double *gbase, int goff0, const ApplyArgs &a, const double2 *zs,
                                             const double2 *ph, const double *hs, int lane, int i0, int lcut, int ci,
                                             double (&dacc)[4])
{
    double2 acc[RB][2], accm[RB][2];
#pragma unroll
    for (int rr = 0; rr < RB; ++rr) acc[rr][0] = acc[rr][1] = accm[rr][0] = accm[rr][1] = cmake(0.0, 0.0);
    if (VP != V_NONE)
        coupling_chunk3<SMAX, RB, VP == V_DVDT, GSM>(bt, gbase, goff0, ct.l_max, ci, lcut, zs, hs, ct.mode_m, lane,
                                                     acc, accm);
    apply_epilogue3<RB, VP>(g, ct, bt, a, ph, lane, i0, ci, acc, accm, dacc);
}

// CTA (tile, group): the group's warp lists (ApplyPlan), one per warp; the group's
// Gaunt weights are staged in shared memory when GSM is set.
template <int SMAX, int VP, bool GSM>
__global__ void __launch_bounds__(APPLY_THREADS, 2) k_apply3(Grid g, CouplingTable ct, BlockTable bt, ApplyPlan pl,
                                                             ApplyArgs a)
{
    if (a.gate && gate_closed(a.gate, a.gate_mode)) return;
    extern __shared__ double2 smem3[];
    __shared__ int s_lcut;
    const int n = g.n_modes, Nr = g.Nr;
    const int K = 2 * ct.l_max + 1;
    const int i0 = blockIdx.x * TILE3;
    double2 *zs = smem3;                              // n * TILE3
    double2 *ph = zs + n * TILE3;                     // n
    double *hs = reinterpret_cast<double *>(ph + n);  // max(K, 4) * TILE3
    double *gs = hs + max(K, 4) * TILE3;              // group weights (GSM)
    constexpr bool vp = VP != V_NONE;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int grp = blockIdx.y;
    const int goff0 = pl.group_goff[grp];
    if (GSM && vp) {
        const int ng2 = (pl.group_goff[grp + 1] - goff0) >> 1;
        const double2 *src = reinterpret_cast<const double2 *>(bt.g + goff0);
        for (int e = threadIdx.x; e < ng2; e += blockDim.x) reinterpret_cast<double2 *>(gs)[e] = src[e];
    }
    const double *gbase = GSM ? gs : bt.g + goff0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        double sn, cs;
        sincos((double)ct.mode_m[k] * a.theta, &sn, &cs);
        ph[k] = cmake(cs, sn);
    }
    if (vp)
        for (int e = threadIdx.x; e < K * TILE3; e += blockDim.x) {
            const int l = e / TILE3, c = e % TILE3;
            const int i = i0 + c;
            hs[e] = i < Nr ? a.hh[(int64_t)l * Nr + i] : 0.0;
        }
    __syncthreads();
    if (vp) {
        for (int e = threadIdx.x; e < n * TILE3; e += blockDim.x) {
            const int k = e / TILE3, c = e % TILE3;
            const int i = i0 + c;
            zs[e] = i < Nr ? cmul(ph[k], a.x[(int64_t)k * Nr + i]) : cmake(0.0, 0.0);
        }
        if (warp == 0) {
            // multipole cut over both halves of the tile
            int lc = -1;
            for (int half = 0; half < 2; ++half) {
                const int c = lane + 32 * half;
                const double h0 = fabs(hs[c]);
                if (h0 > 0.0) {
                    int lcc = 0;
                    for (int l = K - 1; l > 0; --l)
                        if (fabs(hs[l * TILE3 + c]) > 1e-18 * h0) {
                            lcc = l;
                            break;
                        }
                    lc = max(lc, lcc);
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) lc = max(lc, __shfl_xor_sync(0xffffffffu, lc, o));
            if (lane == 0) s_lcut = lc;
        }
    }
    __syncthreads();
    const int lcut = vp ? s_lcut : -1;
    double dacc[4] = {0.0, 0.0, 0.0, 0.0};
    const int list = grp * nw + warp;
    for (int ci = pl.list_ptr[list]; ci < pl.list_ptr[list + 1]; ++ci) {
        if (bt.chunk_nrows[ci] == 1)
            apply_chunk3<SMAX, 1, VP, GSM>(g, ct, bt, gbase, goff0, a, zs, ph, hs, lane, i0, lcut, ci, dacc);
        else
            apply_chunk3<SMAX, 2, VP, GSM>(g, ct, bt, gbase, goff0, a, zs, ph, hs, lane, i0, lcut, ci, dacc);
    }
    if (a.n_dots > 0) {
        __syncthreads();
        double *red = hs;
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
            finish_stage(a.dot_partials, nblocks, 2 * a.n_dots, a.red, a.kr, a.stage, a.ticket,
                         reinterpret_cast<double *>(smem3));
        }
    }
}

// ------------------------------------------------------------------ diagnostics pass, two nodes per thread

// The diagnostics of one row chunk (src/CrankNicolsonModes_extraction.cpp:8-129) at the
// lane's two nodes: H psi, V psi, dV/dt psi and dpsi/dt = -i H psi - Gamma psi / 2, the
// mode's norm and energy sums (nodes < idx_ex, one value per row and tile in `rowred`),
// the edge values at idx_ex, and the lane's p_bin and dV/dt sums.
template <int SMAX, int RB>
__device__ __forceinline__ void diag_chunk3(const Grid &g, const CouplingTable &ct, const BlockTable &bt,
                                            const double *gbase, int goff0, const DiagArgs &d, const double2 *zs,
                                            const double2 *ph, const double *hs, int lane, int i0, int lcut, int ci,
                                            double *rowred, double &e_edge, double &pb, double &dv)
{
    double2 acc[RB][2], accm[RB][2];
    coupling_chunk3<SMAX, RB, true, false>(bt, gbase, goff0, ct.l_max, ci, lcut, zs, hs, ct.mode_m, lane, acc, accm);
    const int Nr = g.Nr, n = g.n_modes;
    const double alpha_d = 1.0 / (g.dr * g.dr), inv2mu = 1.0 / (2 * g.mu);
#pragma unroll
    for (int rr = 0; rr < RB; ++rr) {
        const int j = bt.chunk_rows[ci * 2 + rr];
        const double2 *xr = d.psi + (int64_t)j * Nr;
        double nrm = 0.0, en = 0.0;
#pragma unroll
        for (int nb = 0; nb < 2; ++nb) {
            const int i = i0 + lane + 32 * nb;
            if (i >= Nr || i > d.idx_ex) continue;
            const bool interior = i >= 1 && i <= Nr - 2;
            const double2 xv = xr[i];
            double2 hx = cmake(0.0, 0.0), vx = cmake(0.0, 0.0), dx = cmake(0.0, 0.0);
            if (interior) {
                const int l = ct.mode_l[j];
                const double diag = (2.0 * alpha_d + (double)(l * (l + 1)) * g.ir2[i]) * inv2mu;
                const double off = -alpha_d * inv2mu;
                hx = cadd(cscale(xv, diag), cscale(cadd(xr[i - 1], xr[i + 1]), off));
                const double mj = (double)ct.mode_m[j];
                vx = cmul(cconj(ph[j]), acc[rr][nb]);
                dx = cmul(cconj(ph[j]), cmuli(cscale(cmake(accm[rr][nb].x - mj * acc[rr][nb].x,
                                                           accm[rr][nb].y - mj * acc[rr][nb].y),
                                                     d.domega)));
                hx = cadd(hx, vx);
            }
            if (g.capw) hx = cadd(hx, cmake(g.capw[i] * xv.y, -g.capw[i] * xv.x));
            double2 dp = cmake(hx.y, -hx.x);  // -i H psi
            if (d.n_sinks > 0 && i >= d.slo0 && i < d.shi0)
                dp = cadd(dp, cmul(cscale(d.sink_dots[0], d.sink_coef0), d.sv0[(int64_t)j * Nr + i]));
            if (d.n_sinks > 1 && i >= d.slo1 && i < d.shi1)
                dp = cadd(dp, cmul(cscale(d.sink_dots[1], d.sink_coef1), d.sv1[(int64_t)j * Nr + i]));
            const double ce = cconjmul(xv, hx).x;
            if (i < d.idx_ex) {
                nrm += cabs2(xv);
                en += ce;
            } else {
                e_edge += ce;
                d.dpsi_edge[j] = dp;
                d.psi_edge[3 * j] = i >= 1 ? xr[i - 1] : cmake(0.0, 0.0);
                d.psi_edge[3 * j + 1] = xv;
                d.psi_edge[3 * j + 2] = i + 1 < Nr ? xr[i + 1] : cmake(0.0, 0.0);
            }
            pb += cconjmul(xv, dx).x;
            dv += cconjmul(dp, vx).x;
        }
        nrm = warp_sum(nrm);
        en = warp_sum(en);
        if (lane == 0) {
            rowred[j] = nrm;
            rowred[n + j] = en;
        }
    }
}

// The diagnostics pass on the operator kernel's tiles and work plan: CTA (64-node tile,
// row group) over the tiles up to idx_ex; the group's warp lists of 1-2-row chunks, every
// row in exactly one list.  Per-CTA partials [slot][block] (block = group x tiles +
// tile): slots 0..n-1 norms, n..2n-1 energies (written by the row's group, zero in the
// others), 2n edge energy, 2n+1 p_bin, 2n+2 dV.
template <int SMAX>
__global__ void __launch_bounds__(APPLY_THREADS, 2) k_diag3(Grid g, CouplingTable ct, BlockTable bt, ApplyPlan pl,
                                                            DiagArgs d)
{
    if (d.gate && gate_closed(d.gate, GATE_ACCEPTED)) return;
    extern __shared__ double2 smemd3[];
    __shared__ int s_lcut;
    const int n = g.n_modes, Nr = g.Nr;
    const int K = 2 * ct.l_max + 1;
    const int i0 = blockIdx.x * TILE3;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double2 *zs = smemd3;                             // n * TILE3
    double2 *ph = zs + n * TILE3;                     // n
    double *hs = reinterpret_cast<double *>(ph + n);  // max(K, 4) * TILE3
    double *rowred = hs + max(K, 4) * TILE3;          // 2n per-row sums + 3 x nw lane sums
    const int grp = blockIdx.y;
    const int goff0 = pl.group_goff[grp];
    const double *gbase = bt.g + goff0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        double sn, cs;
        sincos((double)ct.mode_m[k] * d.theta, &sn, &cs);
        ph[k] = cmake(cs, sn);
    }
    for (int e = threadIdx.x; e < K * TILE3; e += blockDim.x) {
        const int l = e / TILE3, c = e % TILE3;
        const int i = i0 + c;
        hs[e] = i < Nr ? d.hh[(int64_t)l * Nr + i] : 0.0;
    }
    for (int e = threadIdx.x; e < 2 * n + 3 * nw; e += blockDim.x) rowred[e] = 0.0;
    __syncthreads();
    for (int e = threadIdx.x; e < n * TILE3; e += blockDim.x) {
        const int k = e / TILE3, c = e % TILE3;
        const int i = i0 + c;
        zs[e] = i < Nr ? cmul(ph[k], d.psi[(int64_t)k * Nr + i]) : cmake(0.0, 0.0);
    }
    if (warp == 0) {
        // multipole cut over both halves of the tile (as in k_apply3)
        int lc = -1;
        for (int half = 0; half < 2; ++half) {
            const int c = lane + 32 * half;
            const double h0 = fabs(hs[c]);
            if (h0 > 0.0) {
                int lcc = 0;
                for (int l = K - 1; l > 0; --l)
                    if (fabs(hs[l * TILE3 + c]) > 1e-18 * h0) {
                        lcc = l;
                        break;
                    }
                lc = max(lc, lcc);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) lc = max(lc, __shfl_xor_sync(0xffffffffu, lc, o));
        if (lane == 0) s_lcut = lc;
    }
    __syncthreads();
    const int lcut = s_lcut;
    double e_edge = 0.0, pb = 0.0, dv = 0.0;
    const int list = grp * nw + warp;
    for (int ci = pl.list_ptr[list]; ci < pl.list_ptr[list + 1]; ++ci) {
        if (bt.chunk_nrows[ci] == 1)
            diag_chunk3<SMAX, 1>(g, ct, bt, gbase, goff0, d, zs, ph, hs, lane, i0, lcut, ci, rowred, e_edge, pb, dv);
        else
            diag_chunk3<SMAX, 2>(g, ct, bt, gbase, goff0, d, zs, ph, hs, lane, i0, lcut, ci, rowred, e_edge, pb, dv);
    }
    e_edge = warp_sum(e_edge);
    pb = warp_sum(pb);
    dv = warp_sum(dv);
    double *lred = rowred + 2 * n;
    if (lane == 0) {
        lred[warp] = e_edge;
        lred[nw + warp] = pb;
        lred[2 * nw + warp] = dv;
    }
    __syncthreads();
    const int nblocks = gridDim.x * gridDim.y, blk = blockIdx.y * gridDim.x + blockIdx.x;
    for (int q = threadIdx.x; q < 2 * n + 3; q += blockDim.x) {
        double sm = 0.0;
        if (q < 2 * n) {
            sm = rowred[q];
        } else {
            for (int w = 0; w < nw; ++w) sm += lred[(q - 2 * n) * nw + w];
        }
        d.partials[(int64_t)q * nblocks + blk] = sm;
    }
}

// ---- launchers of the templated operator kernels

static int smax_for(int l_max)
{
    const int need = l_max + 1;
    return need <= 5 ? 5 : need <= 9 ? 9 : need <= 13 ? 13 : need <= 17 ? 17 : 25;
}

#define CNM_FOR_SMAX(MACRO) MACRO(5) MACRO(9) MACRO(13) MACRO(17) MACRO(25)

cudaError_t set_diag3_smem(int bytes)
{
    cudaError_t e = cudaSuccess;
#define CNM_ATTRD(S) \
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_diag3<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    CNM_FOR_SMAX(CNM_ATTRD)
#undef CNM_ATTRD
    return e;
}

const void *diag3_kernel(int l_max)
{
    const int smax = smax_for(l_max);
#define CNM_PICKD(S) \
    if (smax == S) return (const void *)k_diag3<S>;
    CNM_FOR_SMAX(CNM_PICKD)
#undef CNM_PICKD
    return nullptr;
}

cudaError_t set_apply3_smem(int bytes)
{
    cudaError_t e = cudaSuccess;
#define CNM_ATTR3V(S, V, G) \
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_apply3<S, V, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
#define CNM_ATTR3(S) \
    CNM_ATTR3V(S, V_NONE, false) CNM_ATTR3V(S, V_POT, false) CNM_ATTR3V(S, V_DVDT, false) \
    CNM_ATTR3V(S, V_NONE, true) CNM_ATTR3V(S, V_POT, true) CNM_ATTR3V(S, V_DVDT, true)
    CNM_FOR_SMAX(CNM_ATTR3)
#undef CNM_ATTR3
#undef CNM_ATTR3V
    return e;
}

const void *apply3_kernel(int l_max, int vpart, bool gsm)
{
    const int smax = smax_for(l_max);
#define CNM_PICK3(S)                                                                            \
    if (smax == S) {                                                                            \
        if (gsm) return vpart == V_POT ? (const void *)k_apply3<S, V_POT, true>                 \
                      : vpart == V_DVDT ? (const void *)k_apply3<S, V_DVDT, true>               \
                                         : (const void *)k_apply3<S, V_NONE, true>;             \
        return vpart == V_POT ? (const void *)k_apply3<S, V_POT, false>                          \
             : vpart == V_DVDT ? (const void *)k_apply3<S, V_DVDT, false>                        \
                                : (const void *)k_apply3<S, V_NONE, false>;                      \
    }
    CNM_FOR_SMAX(CNM_PICK3)
#undef CNM_PICK3
    return nullptr;
}

void launch_apply3(int l_max, bool gsm, dim3 blocks, size_t smem, cudaStream_t st, const Grid &g,
                   const CouplingTable &ct, const BlockTable &bt, const ApplyPlan &pl, const ApplyArgs &a)
{
    const int smax = smax_for(l_max);
#define CNM_LAUNCH3G(S, G)                                                                                      \
    if (a.vpart == V_POT) k_apply3<S, V_POT, G><<<blocks, APPLY_THREADS, smem, st>>>(g, ct, bt, pl, a);        \
    else if (a.vpart == V_DVDT) k_apply3<S, V_DVDT, G><<<blocks, APPLY_THREADS, smem, st>>>(g, ct, bt, pl, a); \
    else k_apply3<S, V_NONE, G><<<blocks, APPLY_THREADS, smem, st>>>(g, ct, bt, pl, a);
#define CNM_LAUNCH3(S)              \
    if (smax == S) {                \
        if (gsm) {                  \
            CNM_LAUNCH3G(S, true)   \
        } else {                    \
            CNM_LAUNCH3G(S, false)  \
        }                           \
        return;                     \
    }
    CNM_FOR_SMAX(CNM_LAUNCH3)
#undef CNM_LAUNCH3
#undef CNM_LAUNCH3G
}
void launch_diag3(int l_max, dim3 blocks, size_t smem, cudaStream_t st, const Grid &g, const CouplingTable &ct,
                  const BlockTable &bt, const ApplyPlan &pl, const DiagArgs &d)
{
    const int smax = smax_for(l_max);
#define CNM_LAUNCHD(S)                                                           \
    if (smax == S) {                                                             \
        k_diag3<S><<<blocks, APPLY_THREADS, smem, st>>>(g, ct, bt, pl, d);       \
        return;                                                                  \
    }
    CNM_FOR_SMAX(CNM_LAUNCHD)
#undef CNM_LAUNCHD
}

// ------------------------------------------------------------------ sink projections

// dots[s] = v_s^dagger x over the support of v_s (v_s vanishes elsewhere), one CTA,
// fixed summation order.
__global__ void k_sink_dots(const double2 *x, int Nr, int n_modes, int n_sinks, const double2 *v0,
                            const double2 *v1, int lo0, int hi0, int lo1, int hi1, double2 *dots, const Krylov *gate,
                            int gate_mode)
{
    pdl_wait();
    if (gate && gate_closed(gate, gate_mode)) return;
    // the (sink, mode, support node) terms are dealt to the threads in a fixed order, a
    // few per thread with independent loads (deterministic: fixed per-thread order, then
    // a fixed block reduction)
    __shared__ double scratch[4 * 32];
    const int n0 = n_sinks > 0 ? max(0, hi0 - lo0) : 0, n1 = n_sinks > 1 ? max(0, hi1 - lo1) : 0;
    const int64_t tot0 = (int64_t)n0 * n_modes, tot = tot0 + (int64_t)n1 * n_modes;
    double acc[4] = {0, 0, 0, 0};
#pragma unroll 4
    for (int64_t e = threadIdx.x; e < tot; e += blockDim.x) {
        const bool first = e < tot0;
        const int64_t f = first ? e : e - tot0;
        const int w = first ? n0 : n1;
        const int j = (int)(f / w), i = (first ? lo0 : lo1) + (int)(f - (int64_t)j * w);
        const int64_t q = (int64_t)j * Nr + i;
        const double2 d = cconjmul((first ? v0 : v1)[q], x[q]);
        if (first) {
            acc[0] += d.x;
            acc[1] += d.y;
        } else {
            acc[2] += d.x;
            acc[3] += d.y;
        }
    }
    block_sum<4>(acc, scratch);
    if (threadIdx.x == 0) {
        dots[0] = cmake(acc[0], acc[1]);
        dots[1] = cmake(acc[2], acc[3]);
    }
}

// ------------------------------------------------------------------ preconditioner

// Diagonal of the sparse CN operator A = 1 + i dt/2 (H0 + V + CAP) at (j, i)
// (src/CrankNicolsonModes_matrices.cpp:27-40).
__device__ __forceinline__ double2 a_diag(const Grid &g, const CouplingTable &ct, const double *hh, double half_dt,
                                          int j, int i)
{
    double hre = 0.0, him = 0.0;
    if (i >= 1 && i <= g.Nr - 2) {
        const int l = ct.mode_l[j];
        const double alpha_d = 1.0 / (g.dr * g.dr);
        const double ri = g.r[i];
        hre = (2.0 * alpha_d + (double)(l * (l + 1)) / (ri * ri)) / (2 * g.mu);
        const int p = ct.diag_pair[j];
        if (p >= 0)
            for (int t = ct.pair_term_ptr[p]; t < ct.pair_term_ptr[p + 1]; ++t)
                hre += ct.term_g[t] * hh[(int64_t)ct.term_l[t] * g.Nr + i];
    }
    if (g.capw) him = -g.capw[i];
    // 1 + i (dt/2) (hre + i him) = (1 - dt/2 him) + i dt/2 hre
    return cmake(1.0 - half_dt * him, half_dt * hre);
}

// 2x2 complex matrix (Moebius map p -> (m00 p + m01) / (m10 p + m11)).
struct Mob {
    double2 m00, m01, m10, m11;
};

__device__ __forceinline__ Mob mob_mul(const Mob &A, const Mob &B)  // A after B
{
    Mob C;
    C.m00 = cadd(cmul(A.m00, B.m00), cmul(A.m01, B.m10));
    C.m01 = cadd(cmul(A.m00, B.m01), cmul(A.m01, B.m11));
    C.m10 = cadd(cmul(A.m10, B.m00), cmul(A.m11, B.m10));
    C.m11 = cadd(cmul(A.m10, B.m01), cmul(A.m11, B.m11));
    return C;
}

__device__ __forceinline__ void mob_normalize(Mob &A)
{
    double s = fmax(fmax(fabs(A.m00.x), fabs(A.m00.y)), fmax(fabs(A.m01.x), fabs(A.m01.y)));
    s = fmax(s, fmax(fmax(fabs(A.m10.x), fabs(A.m10.y)), fmax(fabs(A.m11.x), fabs(A.m11.y))));
    if (s > 0.0 && isfinite(s)) {
        // scale by a power of two: exact, and the map is scale invariant
        int e;
        frexp(s, &e);
        const double f = ldexp(1.0, -e);
        A.m00 = cscale(A.m00, f);
        A.m01 = cscale(A.m01, f);
        A.m10 = cscale(A.m10, f);
        A.m11 = cscale(A.m11, f);
    }
}

// Pivot map of node i of one radial block (include/RadialBlockPreconditioner.hpp:59-76):
// p_i = a_i - l_i d_{i-1} u_{i-1}; with l_i = u_{i-1} = off for 2 <= i <= Nr-2 and zero
// couplings to the two boundary nodes, p_i = a_i - c / p_{i-1} (c = off^2) in the
// interior and p_i = a_i at i = 0, 1 and Nr-1.
__device__ __forceinline__ Mob pivot_map(double2 ai, int i, int Nr, double2 c)
{
    Mob M;
    if (i >= 2 && i <= Nr - 2) {
        M.m00 = ai;
        M.m01 = cmake(-c.x, -c.y);
        M.m10 = cmake(1.0, 0.0);
        M.m11 = cmake(0.0, 0.0);
    } else {
        M.m00 = cmake(0.0, 0.0);
        M.m01 = ai;
        M.m10 = cmake(0.0, 0.0);
        M.m11 = cmake(1.0, 0.0);
    }
    return M;
}

__device__ __forceinline__ double2 mob_apply(const Mob &M, double2 p)
{
    return cdiv(cadd(cmul(M.m00, p), M.m01), cadd(cmul(M.m10, p), M.m11));
}

// The pivot kernel above for a caller-supplied diagonal: a_i = diag[j * Nr + i] instead
// of the diagonal rebuilt from the Hamiltonian.  Same chunking, window and scan.
// With rho_max finite the pivots are also checked against the contraction the warm-up
// windows were sized for: |off d_i| <= rho_max on every interior node, else bit 2 of
// status (the windows would not forget their start values, and the solve would be
// inexact).
__global__ void __launch_bounds__(SCAN_THREADS) k_precond_factor_diag(const double2 *diag, int Nr, double2 off,
                                                                       int chunk, int window, double rho_max,
                                                                       double2 *dinv, int *status)
{
    const double off_abs = sqrt(cabs2(off));
    __shared__ Mob tmat[SCAN_THREADS];
    const int j = blockIdx.y;
    const int64_t base = (int64_t)j * Nr;
    const int c0 = blockIdx.x * chunk, c1 = min(Nr, c0 + chunk);
    const int lo = max(0, c0 - window), hi = c1;
    const int len = hi - lo;
    const int per = (len + blockDim.x - 1) / blockDim.x;
    const int s0 = lo + threadIdx.x * per, s1 = min(hi, s0 + per);
    const double2 c = cmul(off, off);
    Mob acc;
    acc.m00 = cmake(1, 0);
    acc.m01 = cmake(0, 0);
    acc.m10 = cmake(0, 0);
    acc.m11 = cmake(1, 0);
    for (int i = s0; i < s1; ++i) {
        acc = mob_mul(pivot_map(diag[base + i], i, Nr, c), acc);
        mob_normalize(acc);
    }
    tmat[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 1; o < (int)blockDim.x; o <<= 1) {
        Mob mine = tmat[threadIdx.x];
        Mob prev;
        const bool has = threadIdx.x >= (unsigned)o;
        if (has) prev = tmat[threadIdx.x - o];
        __syncthreads();
        if (has) {
            mine = mob_mul(mine, prev);
            mob_normalize(mine);
            tmat[threadIdx.x] = mine;
        }
        __syncthreads();
    }
    double2 p = diag[base + lo];
    if (threadIdx.x > 0) p = mob_apply(tmat[threadIdx.x - 1], p);
    for (int i = s0; i < s1; ++i) {
        p = mob_apply(pivot_map(diag[base + i], i, Nr, c), p);
        if (i >= c0) {
            const double m = cabs2(p);
            if (!(m > 0.0) || !isfinite(m)) {
                atomicOr(status, 1);
                dinv[base + i] = cmake(0.0, 0.0);
            } else {
                dinv[base + i] = crcp(p);
                if (i >= 1 && i <= Nr - 2 && off_abs / sqrt(m) > rho_max) atomicOr(status, 2);
            }
        }
    }
}

// Affine map y -> A y + B.
struct Aff {
    double2 A, B;
};

__device__ __forceinline__ Aff aff_then(const Aff &first, const Aff &second)  // second(first(y))
{
    Aff r;
    r.A = cmul(second.A, first.A);
    r.B = cadd(cmul(second.A, first.B), second.B);
    return r;
}

// x = P^{-1} b for the per-mode tridiagonal blocks (include/RadialBlockPreconditioner.hpp:80-98):
// forward y_i = d_i (b_i - l_i y_{i-1}), backward x_i = y_i - u_i d_i x_{i+1}.  Both sweeps
// are linear recurrences solved by an in-CTA scan of affine maps over the chunk and
// its warm-up windows (the recurrences contract, |l_i d_i| < 1).  If `fuse` is set
// the input is b = r + beta (p - omega v) and b is also stored to `bout` (the
// BiCGSTAB search direction), or b = r - alpha v (fuse == 2).
__global__ void __launch_bounds__(SCAN_THREADS) k_precond_solve(int Nr, int chunk, int window, double2 off,
                                                                 const double2 *dinv, const double2 *b, double2 *x)
{
    extern __shared__ double2 ys[];
    __shared__ Aff tf[SCAN_THREADS];
    const int j = blockIdx.y;
    const int c0 = blockIdx.x * chunk, c1 = min(Nr, c0 + chunk);
    const int lo = max(0, c0 - window), hi = min(Nr, c1 + window);
    const int len = hi - lo;
    int per = (len + blockDim.x - 1) / blockDim.x;
    per |= 1;  // odd stride: conflict-free 16-byte shared-memory accesses
    const int s0 = lo + threadIdx.x * per, s1 = min(hi, s0 + per);
    const int64_t base = (int64_t)j * Nr;

    // forward sweep
    Aff acc{cmake(1, 0), cmake(0, 0)};
    for (int i = s0; i < s1; ++i) {
        const double2 d = dinv[base + i];
        const double2 l = (i >= 1 && i <= Nr - 2) ? off : cmake(0, 0);
        const Aff m{cmake(-(l.x * d.x - l.y * d.y), -(l.x * d.y + l.y * d.x)), cmul(d, b[base + i])};
        acc = aff_then(acc, m);
    }
    tf[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 1; o < (int)blockDim.x; o <<= 1) {
        Aff mine = tf[threadIdx.x], prev;
        const bool has = threadIdx.x >= (unsigned)o;
        if (has) prev = tf[threadIdx.x - o];
        __syncthreads();
        if (has) tf[threadIdx.x] = aff_then(prev, mine);
        __syncthreads();
    }
    double2 y = threadIdx.x > 0 ? tf[threadIdx.x - 1].B : cmake(0, 0);
    for (int i = s0; i < s1; ++i) {
        const double2 d = dinv[base + i];
        const double2 l = (i >= 1 && i <= Nr - 2) ? off : cmake(0, 0);
        y = cmul(d, csub(b[base + i], cmul(l, y)));
        ys[i - lo] = y;
    }
    __syncthreads();
    // backward sweep, right to left
    Aff bcc{cmake(1, 0), cmake(0, 0)};
    for (int i = s1 - 1; i >= s0; --i) {
        const double2 d = dinv[base + i];
        const double2 u = (i >= 1 && i <= Nr - 2) ? off : cmake(0, 0);
        const Aff m{cmake(-(u.x * d.x - u.y * d.y), -(u.x * d.y + u.y * d.x)), ys[i - lo]};
        bcc = aff_then(bcc, m);
    }
    tf[threadIdx.x] = bcc;
    __syncthreads();
    const int T = blockDim.x;
    for (int o = 1; o < T; o <<= 1) {
        Aff mine = tf[threadIdx.x], prev;
        const bool has = (int)threadIdx.x + o < T;
        if (has) prev = tf[threadIdx.x + o];
        __syncthreads();
        if (has) tf[threadIdx.x] = aff_then(prev, mine);
        __syncthreads();
    }
    double2 xv = (int)threadIdx.x + 1 < T ? tf[threadIdx.x + 1].B : cmake(0, 0);
    for (int i = s1 - 1; i >= s0; --i) {
        const double2 d = dinv[base + i];
        const double2 u = (i >= 1 && i <= Nr - 2) ? off : cmake(0, 0);
        xv = csub(ys[i - lo], cmul(cmul(u, d), xv));
        if (i >= c0 && i < c1) x[base + i] = xv;
    }
}

// x = P^{-1} b with the chunk, its windows, the pivots and the right-hand side staged in
// shared memory by coalesced loads; the sweeps run in place in shared memory.
__global__ void __launch_bounds__(SCAN2_THREADS) k_precond_solve2(int Nr, int chunk, int window, double2 off,
                                                                  const double2 *dinv, const double2 *b, double2 *x,
                                                                  PrecondInput in)
{
    if (!resolve_input(in)) return;
    extern __shared__ double2 sm2[];
    __shared__ Aff tf[SCAN2_THREADS];
    const int j = blockIdx.y;
    const int c0 = blockIdx.x * chunk, c1 = min(Nr, c0 + chunk);
    const int lo = max(0, c0 - window), hi = min(Nr, c1 + window);
    const int len = hi - lo;
    const int cap = min(Nr, chunk + 2 * window);
    double2 *D = sm2, *Y = sm2 + cap;
    const int64_t base = (int64_t)j * Nr + lo;
    if (in.mode == PI_PLAIN) {
        for (int e = threadIdx.x; e < len; e += blockDim.x) {
            D[e] = dinv[base + e];
            Y[e] = b[base + e];
        }
    } else {
        // the right-hand side is a BiCGSTAB combination formed here and also stored
        // (own chunk only) as the search direction p or the vector s
        const double2 beta = in.kr->beta, omega = in.kr->omega, alpha = in.kr->alpha;
        for (int e = threadIdx.x; e < len; e += blockDim.x) {
            D[e] = dinv[base + e];
            const int64_t k = base + e;
            double2 rhsv;
            if (in.mode == PI_P)
                rhsv = in.p_old ? cadd(in.r[k], cmul(beta, csub(in.p_old[k], cmul(omega, in.v[k])))) : in.r[k];
            else rhsv = csub(in.r[k], cmul(alpha, in.v[k]));
            Y[e] = rhsv;
            const int i = lo + e;
            if (i >= c0 && i < c1) in.out[k] = rhsv;
        }
    }
    __syncthreads();
    int per = (len + blockDim.x - 1) / blockDim.x;
    per |= 1;
    const int s0 = threadIdx.x * per, s1 = min(len, s0 + per);
    // forward: y_i = d_i (b_i - l_i y_{i-1})
    Aff acc{cmake(1, 0), cmake(0, 0)};
    for (int e = s0; e < s1; ++e) {
        const int i = lo + e;
        const double2 d = D[e];
        const double2 l = (i >= 1 && i <= Nr - 2) ? off : cmake(0, 0);
        const Aff m{cmake(-(l.x * d.x - l.y * d.y), -(l.x * d.y + l.y * d.x)), cmul(d, Y[e])};
        acc = aff_then(acc, m);
    }
    tf[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 1; o < (int)blockDim.x; o <<= 1) {
        Aff mine = tf[threadIdx.x], prev;
        const bool has = threadIdx.x >= (unsigned)o;
        if (has) prev = tf[threadIdx.x - o];
        __syncthreads();
        if (has) tf[threadIdx.x] = aff_then(prev, mine);
        __syncthreads();
    }
    double2 y = threadIdx.x > 0 ? tf[threadIdx.x - 1].B : cmake(0, 0);
    for (int e = s0; e < s1; ++e) {
        const int i = lo + e;
        const double2 l = (i >= 1 && i <= Nr - 2) ? off : cmake(0, 0);
        y = cmul(D[e], csub(Y[e], cmul(l, y)));
        Y[e] = y;
    }
    __syncthreads();
    // backward: x_i = y_i - u_i d_i x_{i+1}
    Aff bcc{cmake(1, 0), cmake(0, 0)};
    for (int e = s1 - 1; e >= s0; --e) {
        const int i = lo + e;
        const double2 d = D[e];
        const double2 u = (i >= 1 && i <= Nr - 2) ? off : cmake(0, 0);
        const Aff m{cmake(-(u.x * d.x - u.y * d.y), -(u.x * d.y + u.y * d.x)), Y[e]};
        bcc = aff_then(bcc, m);
    }
    tf[threadIdx.x] = bcc;
    __syncthreads();
    const int T = blockDim.x;
    for (int o = 1; o < T; o <<= 1) {
        Aff mine = tf[threadIdx.x], prev;
        const bool has = (int)threadIdx.x + o < T;
        if (has) prev = tf[threadIdx.x + o];
        __syncthreads();
        if (has) tf[threadIdx.x] = aff_then(prev, mine);
        __syncthreads();
    }
    double2 xv = (int)threadIdx.x + 1 < T ? tf[threadIdx.x + 1].B : cmake(0, 0);
    for (int e = s1 - 1; e >= s0; --e) {
        const int i = lo + e;
        const double2 u = (i >= 1 && i <= Nr - 2) ? off : cmake(0, 0);
        xv = csub(Y[e], cmul(cmul(u, D[e]), xv));
        Y[e] = xv;
    }
    __syncthreads();
    for (int e = (c0 - lo) + threadIdx.x; e < (c1 - lo); e += blockDim.x) x[base + e] = Y[e];
}

// Pivots with the chunk's diagonal staged in shared memory by coalesced passes over
// the hh table; the recurrence then runs from shared memory and the inverse pivots
// leave through one coalesced store.
__global__ void __launch_bounds__(SCAN2_THREADS) k_precond_factor2(Grid g, CouplingTable ct, const double *hh,
                                                                   double half_dt, double2 off, int chunk, int window,
                                                                   double2 *dinv, int *status)
{
    extern __shared__ double2 sm2[];
    __shared__ Mob tmat[SCAN2_THREADS];
    const int Nr = g.Nr, j = blockIdx.y;
    const int c0 = blockIdx.x * chunk, c1 = min(Nr, c0 + chunk);
    const int lo = max(0, c0 - window), hi = c1;
    const int len = hi - lo;
    double2 *A = sm2;
    // diagonal of A = 1 + i dt/2 (H0 + V + CAP) staged term by term: every pass over the
    // nodes reads one row of the hh table with coalesced, independent loads
    {
        const int l = ct.mode_l[j];
        const double alpha_d = 1.0 / (g.dr * g.dr);
        for (int e = threadIdx.x; e < len; e += blockDim.x) {
            const int i = lo + e;
            double hre = 0.0;
            if (i >= 1 && i <= Nr - 2) {
                const double ri = g.r[i];
                hre = (2.0 * alpha_d + (double)(l * (l + 1)) / (ri * ri)) / (2 * g.mu);
            }
            A[e] = cmake(0.0, hre);
        }
        const int p = ct.diag_pair[j];
        if (p >= 0)
            for (int t = ct.pair_term_ptr[p]; t < ct.pair_term_ptr[p + 1]; ++t) {
                const double gt = ct.term_g[t];
                const double *row = hh + (int64_t)ct.term_l[t] * Nr + lo;
                for (int e = threadIdx.x; e < len; e += blockDim.x) {
                    const int i = lo + e;
                    if (i >= 1 && i <= Nr - 2) A[e].y += gt * row[e];
                }
            }
        for (int e = threadIdx.x; e < len; e += blockDim.x) {
            const double him = g.capw ? -g.capw[lo + e] : 0.0;
            // 1 + i (dt/2) (hre + i him) = (1 - dt/2 him) + i dt/2 hre
            A[e] = cmake(1.0 - half_dt * him, half_dt * A[e].y);
        }
    }
    __syncthreads();
    const double2 pstart = A[0];  // start value before node lo (exact when lo == 0)
    int per = (len + blockDim.x - 1) / blockDim.x;
    per |= 1;
    const int s0 = threadIdx.x * per, s1 = min(len, s0 + per);
    const double2 c = cmul(off, off);
    Mob acc;
    acc.m00 = cmake(1, 0);
    acc.m01 = cmake(0, 0);
    acc.m10 = cmake(0, 0);
    acc.m11 = cmake(1, 0);
    for (int e = s0; e < s1; ++e) {
        acc = mob_mul(pivot_map(A[e], lo + e, Nr, c), acc);
        mob_normalize(acc);
    }
    tmat[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 1; o < (int)blockDim.x; o <<= 1) {
        Mob mine = tmat[threadIdx.x];
        Mob prev;
        const bool has = threadIdx.x >= (unsigned)o;
        if (has) prev = tmat[threadIdx.x - o];
        __syncthreads();
        if (has) {
            mine = mob_mul(mine, prev);
            mob_normalize(mine);
            tmat[threadIdx.x] = mine;
        }
        __syncthreads();
    }
    double2 p = pstart;
    if (threadIdx.x > 0 && s0 < len) p = mob_apply(tmat[threadIdx.x - 1], p);
    int bad = 0;
    for (int e = s0; e < s1; ++e) {
        p = mob_apply(pivot_map(A[e], lo + e, Nr, c), p);
        const double m = cabs2(p);
        if (!(m > 0.0) || !isfinite(m)) {
            if (lo + e >= c0) bad = 1;
            A[e] = cmake(0.0, 0.0);
        } else {
            A[e] = crcp(p);
        }
    }
    if (bad) atomicOr(status, 1);
    __syncthreads();
    const int64_t base = (int64_t)j * Nr + lo;
    for (int e = (c0 - lo) + threadIdx.x; e < len; e += blockDim.x) dinv[base + e] = A[e];
}

// ------------------------------------------------------------------ exact cluster scans

// One thread-block cluster per radial block (mode): the cluster's CTAs split the Nr
// nodes into consecutive chunks of PCL_THREADS * per nodes, every thread owns `per`
// consecutive nodes (odd, so the threads' 16-byte shared-memory accesses are
// conflict-free).  A recurrence is solved exactly, without warm-up windows:
//   thread:  compose the maps of its nodes,
//   warp:    shuffle scan of the thread maps,
//   CTA:     composition of the warp totals,
//   cluster: every CTA reads the totals of the CTAs before it (after it, for a
//            backward sweep) from their shared memory and folds them into its start
//            value; then each thread replays its nodes from its exact start value.

__device__ __forceinline__ Aff aff_identity() { return Aff{cmake(1.0, 0.0), cmake(0.0, 0.0)}; }
__device__ __forceinline__ double2 aff_apply(const Aff &m, double2 y) { return cadd(cmul(m.A, y), m.B); }

__device__ __forceinline__ Aff shfl_up_aff(const Aff &a, int o)
{
    Aff r;
    r.A.x = __shfl_up_sync(0xffffffffu, a.A.x, o);
    r.A.y = __shfl_up_sync(0xffffffffu, a.A.y, o);
    r.B.x = __shfl_up_sync(0xffffffffu, a.B.x, o);
    r.B.y = __shfl_up_sync(0xffffffffu, a.B.y, o);
    return r;
}

__device__ __forceinline__ Aff shfl_down_aff(const Aff &a, int o)
{
    Aff r;
    r.A.x = __shfl_down_sync(0xffffffffu, a.A.x, o);
    r.A.y = __shfl_down_sync(0xffffffffu, a.A.y, o);
    r.B.x = __shfl_down_sync(0xffffffffu, a.B.x, o);
    r.B.y = __shfl_down_sync(0xffffffffu, a.B.y, o);
    return r;
}

__device__ __forceinline__ Mob shfl_up_mob(const Mob &a, int o)
{
    Mob r;
    r.m00 = cmake(__shfl_up_sync(0xffffffffu, a.m00.x, o), __shfl_up_sync(0xffffffffu, a.m00.y, o));
    r.m01 = cmake(__shfl_up_sync(0xffffffffu, a.m01.x, o), __shfl_up_sync(0xffffffffu, a.m01.y, o));
    r.m10 = cmake(__shfl_up_sync(0xffffffffu, a.m10.x, o), __shfl_up_sync(0xffffffffu, a.m10.y, o));
    r.m11 = cmake(__shfl_up_sync(0xffffffffu, a.m11.x, o), __shfl_up_sync(0xffffffffu, a.m11.y, o));
    return r;
}

__device__ __forceinline__ Mob mob_identity()
{
    Mob m;
    m.m00 = cmake(1, 0);
    m.m01 = cmake(0, 0);
    m.m10 = cmake(0, 0);
    m.m11 = cmake(1, 0);
    return m;
}

// Bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) from global to
// this CTA's shared memory, completing on the mbarrier at shared address `bar`.
__device__ __forceinline__ void bulk_load_s(void *dst, const void *src, unsigned bytes, unsigned bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     (unsigned)__cvta_generic_to_shared(dst)),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// Wait for phase `parity` of the mbarrier at `bar`, giving up after a bounded number of
// polls (each try_wait suspends for a hardware-chosen interval); false if it gave up.
__device__ __forceinline__ bool mbar_wait_parity(unsigned bar, unsigned parity)
{
    for (int it = 0; it < (1 << 22); ++it) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// x = P^{-1} b for every radial block, exact (see the scan scheme above).  Grid
// (cluster size, blocks): blockIdx.y selects the mode j = blockIdx.y % n_modes and,
// for blockIdx.y >= n_modes, the second right-hand side / output pair (b2, x2), so
// one launch can carry two independent solves.  PrecondInput fuses the BiCGSTAB
// combinations as in k_precond_solve2.
__global__ void __launch_bounds__(PCL_THREADS, 3) k_precond_solve_cl(int Nr, int n_modes, int per, double2 off,
                                                                   const double2 *dinv, const double2 *b, double2 *x,
                                                                   const double2 *b2, double2 *x2, PrecondInput in,
                                                                   WoodArgs wd)
{
    pdl_wait();
    if (!resolve_input(in)) return;
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ double2 smc[];
    __shared__ Aff wagg[PCL_THREADS / 32];
    __shared__ Aff wex_s[PCL_THREADS / 32];  // exclusive prefix (forward) / suffix (backward) of wagg
    __shared__ Aff cagg_f, cagg_b;
    const int rank = (int)cl.block_rank(), cs = (int)cl.num_blocks();
    const int second = blockIdx.y >= (unsigned)n_modes;
    const int j = blockIdx.y - (second ? n_modes : 0);
    const double2 *bv = second ? b2 : b;
    double2 *xv = second ? x2 : x;
    const int T = PCL_THREADS, NW = PCL_THREADS / 32;
    const int Lc = T * per;
    const int c0 = rank * Lc, c1 = min(Nr, c0 + Lc), len = max(0, c1 - c0);
    double2 *D = smc, *Y = smc + Lc;
    const int64_t base = (int64_t)j * Nr + c0;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // staging: two elements per thread in flight (every load of a batch issues
    // before its stores)
    // staging: the pivots and b (or r) arrive by bulk copies into shared memory that
    // complete on an mbarrier; the threads load the other inputs of a BiCGSTAB combination
    __shared__ __align__(8) unsigned long long stage_bar;
    const unsigned bar = (unsigned)__cvta_generic_to_shared(&stage_bar);
    bool staged = true;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (len > 0) {
        if (tid == 0) {
            const unsigned bytes = (unsigned)len * (unsigned)sizeof(double2);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(2u * bytes)
                         : "memory");
            bulk_load_s(D, dinv + base, bytes, bar);
            bulk_load_s(Y, (in.mode == PI_PLAIN ? bv : in.r) + base, bytes, bar);
        }
        if (!mbar_wait_parity(bar, 0u)) {
            // the copies did not complete in time: flag the solve as failed (the attempt
            // is then not accepted) and wait once more for them before going on; if that
            // wait gives up too, this CTA still takes part in every cluster barrier but
            // stores nothing (a copy's completion is then left unobserved)
            if (tid == 0 && in.fault) atomicOr(in.fault, 2);
            staged = mbar_wait_parity(bar, 0u);
        }
    }
    if (in.mode != PI_PLAIN && staged) {
        const double2 beta = in.kr->beta, omega = in.kr->omega, alpha = in.kr->alpha;
        // PI_P without p_old (first iteration: p_old = v = 0) is p = r
        const bool first = in.mode == PI_P && in.p_old == nullptr;
        const double2 *__restrict__ vsrc = first ? nullptr : in.v + base;
        const double2 *__restrict__ psrc = (in.mode == PI_P && !first) ? in.p_old + base : nullptr;
        double2 *__restrict__ odst = in.out + base;
        constexpr int SB = 4;
        for (int e0 = tid; e0 < len; e0 += SB * T) {
            double2 vv[SB], pv[SB];
#pragma unroll
            for (int u = 0; u < SB; ++u) {
                const int e = e0 + u * T;
                if (e < len) {
                    vv[u] = vsrc ? vsrc[e] : cmake(0.0, 0.0);
                    pv[u] = psrc ? psrc[e] : cmake(0.0, 0.0);
                }
            }
#pragma unroll
            for (int u = 0; u < SB; ++u) {
                const int e = e0 + u * T;
                if (e < len) {
                    const double2 rv = Y[e];
                    const double2 rhsv = first ? rv
                                         : psrc ? cadd(rv, cmul(beta, csub(pv[u], cmul(omega, vv[u]))))
                                                : csub(rv, cmul(alpha, vv[u]));
                    Y[e] = rhsv;
                    odst[e] = rhsv;
                }
            }
        }
    }
    __syncthreads();
    const int s0 = tid * per, s1 = min(len, s0 + per);

    // ---- forward: y_i = d_i (b_i - l_i y_{i-1})
    Aff acc = aff_identity();
    for (int e = s0; e < s1; ++e) {
        const int i = c0 + e;
        const double2 d = D[e];
        const double2 l = (i >= 1 && i <= Nr - 2) ? off : cmake(0, 0);
        const Aff m{cmake(-(l.x * d.x - l.y * d.y), -(l.x * d.y + l.y * d.x)), cmul(d, Y[e])};
        acc = aff_then(acc, m);
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const Aff prev = shfl_up_aff(acc, o);
        if (lane >= o) acc = aff_then(prev, acc);
    }
    Aff excl = shfl_up_aff(acc, 1);
    if (lane == 0) excl = aff_identity();
    if (lane == 31) wagg[warp] = acc;
    __syncthreads();
    if (warp == 0) {
        // CTA total: ordered scan of the warp totals in lanes 0..NW-1; each warp's exclusive
        // prefix is kept for the apply pass
        Aff c = lane < NW ? wagg[lane] : aff_identity();
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const Aff prev = shfl_up_aff(c, o);
            if (lane >= o) c = aff_then(prev, c);
        }
        Aff ex = shfl_up_aff(c, 1);
        if (lane == 0) ex = aff_identity();
        if (lane < NW) wex_s[lane] = ex;
        if (lane == 31) cagg_f = c;
    }
    cl.sync();
    // Every warp derives its own start value (the same scans in each warp): a single
    // warp doing this while the others wait at a barrier ran about six times slower.
    double2 ywarp;
    {
        // start value of the CTA: lane q < rank holds CTA q's total; their ordered
        // composition applied to y = 0 is its B part
        Aff c = lane < rank ? *cl.map_shared_rank(&cagg_f, lane) : aff_identity();
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const Aff prev = shfl_up_aff(c, o);
            if (lane >= o) c = aff_then(prev, c);
        }
        const double2 ycta = cmake(__shfl_sync(0xffffffffu, c.B.x, 31), __shfl_sync(0xffffffffu, c.B.y, 31));
        ywarp = aff_apply(wex_s[warp], ycta);
    }
    // ---- forward apply and, composed as it goes, the thread's backward map
    // bcc = f_s0 o ... o f_s1-1 with f_e(x) = y_e - u_e d_e x (x_i = y_i - u_i d_i x_{i+1})
    Aff bcc = aff_identity();
    {
        double2 y = aff_apply(excl, ywarp);
        for (int e = s0; e < s1; ++e) {
            const int i = c0 + e;
            const double2 l = (i >= 1 && i <= Nr - 2) ? off : cmake(0, 0);
            const double2 d = D[e];
            y = cmul(d, csub(Y[e], cmul(l, y)));
            Y[e] = y;
            const Aff m{cmake(-(l.x * d.x - l.y * d.y), -(l.x * d.y + l.y * d.x)), y};
            bcc = aff_then(m, bcc);
        }
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const Aff nxt = shfl_down_aff(bcc, o);
        if (lane + o < 32) bcc = aff_then(nxt, bcc);
    }
    Aff bexcl = shfl_down_aff(bcc, 1);
    if (lane == 31) bexcl = aff_identity();
    __syncthreads();  // every thread has read wex_s[] of the forward sweep
    if (lane == 0) wagg[warp] = bcc;
    __syncthreads();
    if (warp == 0) {
        // CTA total of the backward maps: ordered suffix scan of the warp totals; each
        // warp's exclusive suffix is kept for the apply pass
        Aff c = lane < NW ? wagg[lane] : aff_identity();
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const Aff nxt = shfl_down_aff(c, o);
            if (lane + o < 32) c = aff_then(nxt, c);
        }
        Aff ex = shfl_down_aff(c, 1);
        if (lane == 31) ex = aff_identity();
        if (lane < NW) wex_s[lane] = ex;
        if (lane == 0) cagg_b = c;
    }
    cl.sync();
    double2 xwarp;
    {
        // start value of the CTA from the CTAs after it (applied last to first)
        Aff c = (lane > rank && lane < cs) ? *cl.map_shared_rank(&cagg_b, lane) : aff_identity();
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const Aff nxt = shfl_down_aff(c, o);
            if (lane + o < 32) c = aff_then(nxt, c);
        }
        const double2 xcta = cmake(__shfl_sync(0xffffffffu, c.B.x, 0), __shfl_sync(0xffffffffu, c.B.y, 0));
        xwarp = aff_apply(wex_s[warp], xcta);
    }
    // the other CTAs read cagg_b only before this arrive; the matching wait is the
    // last statement, so a CTA's shared memory outlives every remote read of it
    cl.barrier_arrive();
    {
        double2 xr = aff_apply(bexcl, xwarp);
        for (int e = s1 - 1; e >= s0; --e) {
            const int i = c0 + e;
            const double2 u = (i >= 1 && i <= Nr - 2) ? off : cmake(0, 0);
            xr = csub(Y[e], cmul(cmul(u, D[e]), xr));
            Y[e] = xr;
        }
    }
    __syncthreads();
    if (staged)
        for (int e = tid; e < len; e += T) xv[base + e] = Y[e];
    if (wd.mode != WD_NONE) {
        // sink projections v_a^dag x of this CTA's nodes; the last CTA finishes the
        // Woodbury scalars
        __shared__ double wscr[8 * 32];
        double acc[4] = {0, 0, 0, 0};
        for (int a = 0; a < wd.n_sinks; ++a) {
            const double2 *va = a == 0 ? wd.v0 : wd.v1;
            const int lo = max((a == 0 ? wd.lo0 : wd.lo1) - c0, 0), hi = min((a == 0 ? wd.hi0 : wd.hi1) - c0, len);
            for (int e = lo + tid; e < hi; e += T) {
                const double2 d = cconjmul(va[base + e], Y[e]);
                acc[2 * a] += d.x;
                acc[2 * a + 1] += d.y;
            }
        }
        block_sum<4>(acc, wscr);
        const int nblk = gridDim.x * gridDim.y, blk = blockIdx.y * gridDim.x + blockIdx.x;
        const int nslots = wd.mode == WD_SETUP ? 8 : 4;
        if (tid == 0) {
            for (int q = 0; q < nslots; ++q) {
                // setup: slots 4 b + (2 a + re/im) hold v_a^dag W_b
                const int own = wd.mode == WD_SETUP ? q - 4 * second : q;
                wd.partials[(int64_t)q * nblk + blk] = (own >= 0 && own < 4) ? acc[own] : 0.0;
            }
            __threadfence();
        }
        __shared__ unsigned s_last;
        __syncthreads();
        if (tid == 0) s_last = atomicAdd(wd.ticket, 1u) == (unsigned)nblk - 1u ? 1u : 0u;
        __syncthreads();
        if (s_last) {
            __threadfence();
            double sm[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) sm[q] = 0.0;
            for (int bb = tid; bb < nblk; bb += T) {
                double v[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) v[q] = q < nslots ? __ldcg(wd.partials + (int64_t)q * nblk + bb) : 0.0;
#pragma unroll
                for (int q = 0; q < 8; ++q) sm[q] += v[q];
            }
            block_sum<8>(sm, wscr);
            if (tid == 0) {
                if (wd.mode == WD_SETUP) {
                    // vw[2 b + a] = v_a^dag W_b
                    double2 vw[4] = {cmake(sm[0], sm[1]), cmake(sm[2], sm[3]), cmake(sm[4], sm[5]),
                                     cmake(sm[6], sm[7])};
                    wood_setup_dev(wd.kr, vw, wd.c0, wd.c1);
                } else {
                    const double2 proj[2] = {cmake(sm[0], sm[1]), cmake(sm[2], sm[3])};
                    wood_scalar_dev(wd.kr, wd.which, proj);
                }
                *wd.ticket = 0u;
            }
        }
    }
    cl.barrier_wait();
}

// Woodbury set-up (src/CrankNicolsonModes_matrices.cpp:133-145) on the band [blo, bhi)
// outside which every W_a = P^{-1} v_a is below 1e-40 of its largest value: one CTA per
// (radial block j, sink a) stages the band's pivots and v_a in shared memory and runs the
// block's forward and backward Thomas sweeps over it as affine scans (thread: its run of
// nodes, an odd count so 16-byte shared accesses do not conflict; warp: shuffles; CTA:
// every warp composes the warp totals before it).  Left of the band y vanishes exactly
// (v_a does), right of it x is taken as zero; the pivots are the full block's, so the band
// values are those of the full solve.  Each CTA reduces v_b^dag W_a over the sinks'
// supports into partials[slot][j] (slot 4 a + 2 b + re/im); the last CTA sums them over j
// in order and forms G = diag(1 / (dt/4 g)) + v^dag W and its inverse.
__global__ void __launch_bounds__(WSB_THREADS) k_wood_setup_band(int Nr, int n_modes, int blo, int bhi, double2 off,
                                                                 const double2 *dinv, WoodBand wb)
{
    pdl_wait();
    extern __shared__ double2 wsb[];
    __shared__ Aff wagg[WSB_THREADS / 32];
    __shared__ double wscr[4 * 32];
    constexpr int T = WSB_THREADS, NW = WSB_THREADS / 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int j = blockIdx.x / wb.n_sinks, a = blockIdx.x - j * wb.n_sinks;
    const int Lb = bhi - blo;
    double2 *D = wsb, *Y = wsb + Lb;
    const int64_t base = (int64_t)j * Nr + blo;
    {
        const double2 *__restrict__ v = (a == 0 ? wb.v0 : wb.v1) + base;
        const double2 *__restrict__ d = dinv + base;
        for (int e0 = tid; e0 < Lb; e0 += 4 * T) {
            double2 dv[4], vv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int e = e0 + T * u;
                if (e < Lb) {
                    dv[u] = d[e];
                    vv[u] = v[e];
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int e = e0 + T * u;
                if (e < Lb) {
                    D[e] = dv[u];
                    Y[e] = vv[u];
                }
            }
        }
    }
    __syncthreads();
    const int cnt = ((Lb + T - 1) / T) | 1;
    const int s0 = min(Lb, tid * cnt), s1 = min(Lb, s0 + cnt);
    // forward: y_i = d_i (v_i - l y_{i-1}), y = 0 left of the band
    Aff acc = aff_identity();
    for (int e = s0; e < s1; ++e) {
        const int i = blo + e;
        const double2 di = D[e];
        const double2 l = (i >= 1 && i <= Nr - 2) ? off : cmake(0.0, 0.0);
        const Aff m{cmake(-(l.x * di.x - l.y * di.y), -(l.x * di.y + l.y * di.x)), cmul(di, Y[e])};
        acc = aff_then(acc, m);
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const Aff prev = shfl_up_aff(acc, o);
        if (lane >= o) acc = aff_then(prev, acc);
    }
    Aff excl = shfl_up_aff(acc, 1);
    if (lane == 0) excl = aff_identity();
    if (lane == 31) wagg[warp] = acc;
    __syncthreads();
    double2 y;
    {
        // start of this warp: the warp totals before it, applied to y = 0
        Aff w = lane < NW ? wagg[lane] : aff_identity();
#pragma unroll
        for (int o = 1; o < NW; o <<= 1) {
            const Aff prev = shfl_up_aff(w, o);
            if (lane >= o) w = aff_then(prev, w);
        }
        const Aff wex = shfl_up_aff(w, 1);
        const double2 ys = lane == 0 ? cmake(0.0, 0.0) : wex.B;
        y = aff_apply(excl, cmake(__shfl_sync(0xffffffffu, ys.x, warp), __shfl_sync(0xffffffffu, ys.y, warp)));
    }
    for (int e = s0; e < s1; ++e) {
        const int i = blo + e;
        const double2 l = (i >= 1 && i <= Nr - 2) ? off : cmake(0.0, 0.0);
        y = cmul(D[e], csub(Y[e], cmul(l, y)));
        Y[e] = y;
    }
    // backward: x_i = y_i - u d_i x_{i+1}, x = 0 right of the band
    Aff bcc = aff_identity();
    for (int e = s1 - 1; e >= s0; --e) {
        const int i = blo + e;
        const double2 di = D[e];
        const double2 u = (i >= 1 && i <= Nr - 2) ? off : cmake(0.0, 0.0);
        const Aff m{cmake(-(u.x * di.x - u.y * di.y), -(u.x * di.y + u.y * di.x)), Y[e]};
        bcc = aff_then(bcc, m);
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const Aff nxt = shfl_down_aff(bcc, o);
        if (lane + o < 32) bcc = aff_then(nxt, bcc);
    }
    Aff bexcl = shfl_down_aff(bcc, 1);
    if (lane == 31) bexcl = aff_identity();
    __syncthreads();  // every warp has read wagg[] of the forward sweep
    if (lane == 0) wagg[warp] = bcc;
    __syncthreads();
    double2 x;
    {
        // start of this warp: the warp totals after it (applied last to first), x = 0 past the band
        Aff w = lane < NW ? wagg[lane] : aff_identity();
#pragma unroll
        for (int o = 1; o < NW; o <<= 1) {
            const Aff nxt = shfl_down_aff(w, o);
            if (lane + o < 32) w = aff_then(nxt, w);
        }
        const Aff wex = shfl_down_aff(w, 1);
        const double2 xs = lane >= NW - 1 ? cmake(0.0, 0.0) : wex.B;
        x = aff_apply(bexcl, cmake(__shfl_sync(0xffffffffu, xs.x, warp), __shfl_sync(0xffffffffu, xs.y, warp)));
    }
    for (int e = s1 - 1; e >= s0; --e) {
        const int i = blo + e;
        const double2 u = (i >= 1 && i <= Nr - 2) ? off : cmake(0.0, 0.0);
        x = csub(Y[e], cmul(cmul(u, D[e]), x));
        Y[e] = x;
    }
    __syncthreads();
    // W_a on the band and the projections v_b^dag W_a (b = 0, 1) over the supports
    double pr[4] = {0.0, 0.0, 0.0, 0.0};
    {
        double2 *__restrict__ W = (a == 0 ? wb.W0 : wb.W1) + base;
        for (int e = tid; e < Lb; e += T) {
            const double2 xv = Y[e];
            W[e] = xv;
            const int i = blo + e;
            if (i >= wb.slo0 && i < wb.shi0) {
                const double2 q = cconjmul(wb.v0[base + e], xv);
                pr[0] += q.x;
                pr[1] += q.y;
            }
            if (wb.n_sinks > 1 && i >= wb.slo1 && i < wb.shi1) {
                const double2 q = cconjmul(wb.v1[base + e], xv);
                pr[2] += q.x;
                pr[3] += q.y;
            }
        }
    }
    block_sum<4>(pr, wscr);
    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < 4; ++q) wb.partials[(int64_t)(4 * a + q) * n_modes + j] = pr[q];
        __threadfence();
    }
    __shared__ unsigned s_last;
    __syncthreads();
    if (tid == 0) s_last = atomicAdd(wb.ticket, 1u) == gridDim.x - 1u ? 1u : 0u;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // the partials of up to T / 8 blocks at a time are loaded together, then slot q's are
    // added in block order by thread q
    __shared__ double fin[8][WSB_THREADS / 8];
    const int nq = 4 * wb.n_sinks, per = T / 8;
    double sm = 0.0;
    for (int j0 = 0; j0 < n_modes; j0 += per) {
        {
            const int q = tid / per, jj = j0 + tid % per;
            if (q < nq && jj < n_modes) fin[q][tid % per] = __ldcg(wb.partials + (int64_t)q * n_modes + jj);
        }
        __syncthreads();
        if (tid < nq)
            for (int u = 0; u < per && j0 + u < n_modes; ++u) sm += fin[tid][u];
        __syncthreads();
    }
    __shared__ double sums[8];
    if (tid < 8) sums[tid] = (tid < nq && (tid & 3) < 2 * wb.n_sinks) ? sm : 0.0;
    __syncthreads();
    if (tid == 0) {
        // vw[2 a + b] = v_b^dag W_a
        const double2 vw[4] = {cmake(sums[0], sums[1]), cmake(sums[2], sums[3]), cmake(sums[4], sums[5]),
                               cmake(sums[6], sums[7])};
        wood_setup_dev(wb.kr, vw, wb.c0, wb.c1);
        *wb.ticket = 0u;
    }
}

// Inverse Thomas pivots d_i = 1 / p_i, exact: the pivot recurrence p_i = a_i - c / p_{i-1}
// is a chain of Moebius maps composed by the cluster scan above (2x2 complex matrices,
// rescaled by powers of two as they grow).  Grid (cluster size, modes).
__global__ void __launch_bounds__(PCL_THREADS) k_precond_factor_cl(Grid g, CouplingTable ct, const double *hh,
                                                                    double half_dt, double2 off, int per,
                                                                    double2 *dinv, float2 *dinv32, int *status)
{
    pdl_wait();
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ double2 smc[];
    __shared__ Mob wmob[PCL_THREADS / 32];
    __shared__ Mob wex_s[PCL_THREADS / 32];  // each warp's exclusive prefix of wmob
    __shared__ Mob cmob;
    const int rank = (int)cl.block_rank();
    const int Nr = g.Nr, j = blockIdx.y;
    const int T = PCL_THREADS, NW = PCL_THREADS / 32;
    const int Lc = T * per;
    const int c0 = rank * Lc, c1 = min(Nr, c0 + Lc), len = max(0, c1 - c0);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double2 *A = smc;
    // diagonal of A = 1 + i dt/2 (H0 + V + CAP): the diagonal pair's terms go to shared
    // memory first, then every node's loads (r, CAP, one hh row per term) are
    // independent and issue together
    __shared__ double tg[64];
    __shared__ int tl[64];
    const int pd = ct.diag_pair[j];
    const int t0 = pd >= 0 ? ct.pair_term_ptr[pd] : 0, nt = pd >= 0 ? min(64, ct.pair_term_ptr[pd + 1] - t0) : 0;
    if (tid < nt) {
        tg[tid] = ct.term_g[t0 + tid];
        tl[tid] = ct.term_l[t0 + tid];
    }
    __syncthreads();
    {
        const int l = ct.mode_l[j];
        const double alpha_d = 1.0 / (g.dr * g.dr), ll = (double)(l * (l + 1)), inv2mu = 1.0 / (2 * g.mu);
#pragma unroll 2
        for (int e = tid; e < len; e += T) {
            const int i = c0 + e;
            double hre = 0.0;
            if (i >= 1 && i <= Nr - 2) {
                hre = (2.0 * alpha_d + ll * g.ir2[i]) * inv2mu;
                for (int t = 0; t < nt; ++t) hre += tg[t] * hh[(int64_t)tl[t] * Nr + i];
            }
            const double him = g.capw ? -g.capw[i] : 0.0;
            A[e] = cmake(1.0 - half_dt * him, half_dt * hre);
        }
    }
    __syncthreads();
    const int s0 = tid * per, s1 = min(len, s0 + per);
    const double2 c = cmul(off, off);
    Mob acc = mob_identity();
    for (int e = s0; e < s1; ++e) {
        acc = mob_mul(pivot_map(A[e], c0 + e, Nr, c), acc);
        if (((e - s0) & 3) == 3) mob_normalize(acc);
    }
    mob_normalize(acc);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const Mob prev = shfl_up_mob(acc, o);
        if (lane >= o) {
            acc = mob_mul(acc, prev);
            mob_normalize(acc);
        }
    }
    const Mob excl = shfl_up_mob(acc, 1);
    if (lane == 31) wmob[warp] = acc;
    __syncthreads();
    if (warp == 0) {
        // the CTA total, and each warp's exclusive prefix for its start pivot below
        Mob m = lane < NW ? wmob[lane] : mob_identity();
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const Mob prev = shfl_up_mob(m, o);
            if (lane >= o) {
                m = mob_mul(m, prev);
                mob_normalize(m);
            }
        }
        Mob ex = shfl_up_mob(m, 1);
        if (lane == 0) ex = mob_identity();
        if (lane < NW) wex_s[lane] = ex;
        if (lane == 31) cmob = m;
    }
    cl.sync();
    // every warp derives its own start pivot (see the solve: a lone warp here is slow)
    double2 p;
    {
        // node 0's map is constant (p_0 = a_0), so any finite start value is exact
        Mob m = lane < rank ? *cl.map_shared_rank(&cmob, lane) : mob_identity();
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const Mob prev = shfl_up_mob(m, o);
            if (lane >= o) {
                m = mob_mul(m, prev);
                mob_normalize(m);
            }
        }
        double2 pc = lane == 31 ? mob_apply(m, cmake(1.0, 0.0)) : cmake(0.0, 0.0);
        pc = cmake(__shfl_sync(0xffffffffu, pc.x, 31), __shfl_sync(0xffffffffu, pc.y, 31));
        p = mob_apply(wex_s[warp], pc);
    }
    cl.barrier_arrive();
    if (lane > 0) p = mob_apply(excl, p);
    int bad = 0;
    double2 dprev = crcp(p);
    for (int e = s0; e < s1; ++e) {
        const int i = c0 + e;
        const double2 a = A[e];
        p = (i >= 2 && i <= Nr - 2) ? csub(a, cmul(c, dprev)) : a;
        const double m = cabs2(p);
        if (!(m > 0.0) || !isfinite(m)) {
            bad = 1;
            dprev = cmake(0.0, 0.0);
        } else {
            dprev = crcp(p);
        }
        A[e] = dprev;
    }
    if (bad) atomicOr(status, 1);
    __syncthreads();
    const int64_t base = (int64_t)j * Nr + c0;
    for (int e = tid; e < len; e += T) dinv[base + e] = A[e];
    if (dinv32)  // the mixed solve's fp32 copy of the pivots
        for (int e = tid; e < len; e += T) dinv32[base + e] = make_float2((float)A[e].x, (float)A[e].y);
    cl.barrier_wait();
}

// ------------------------------------------------------------------ vector kernels

// Per-CTA partial sums of up to three complex inner products conj(a_q) . b_q over n
// elements (grid-stride, fixed assignment, deterministic).
__global__ void __launch_bounds__(VEC_THREADS) k_dots(int64_t n, int nq, const double2 *a0, const double2 *b0,
                                                       const double2 *a1, const double2 *b1, const double2 *a2,
                                                       const double2 *b2, double *partials)
{
    __shared__ double scratch[6 * 32];
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        double2 d = cconjmul(a0[e], b0[e]);
        acc[0] += d.x;
        acc[1] += d.y;
        if (nq > 1) {
            d = cconjmul(a1[e], b1[e]);
            acc[2] += d.x;
            acc[3] += d.y;
        }
        if (nq > 2) {
            d = cconjmul(a2[e], b2[e]);
            acc[4] += d.x;
            acc[5] += d.y;
        }
    }
    block_sum<6>(acc, scratch);
    if (threadIdx.x == 0)
        for (int q = 0; q < 6; ++q) partials[(int64_t)q * gridDim.x + blockIdx.x] = acc[q];
}

// out[q] = sum over `nblocks` partials of slot q (fixed order), q < nslots.
__global__ void k_sum_partials(const double *partials, int nblocks, int nslots, double *out)
{
    __shared__ double scratch[6 * 32];
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
        for (int q = 0; q < nslots; ++q) acc[q] += partials[(int64_t)q * nblocks + b];
    block_sum<6>(acc, scratch);
    if (threadIdx.x == 0)
        for (int q = 0; q < nslots; ++q) out[q] = acc[q];
}

// y = a x (+ b w): scaled copies and combinations with host-side scalars.
__global__ void k_axpby(int64_t n, double2 a, const double2 *x, double2 b, const double2 *w, double2 *y)
{
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        double2 v = cmul(a, x[e]);
        if (w) v = cadd(v, cmul(b, w[e]));
        y[e] = v;
    }
}

// y *= mask(i) (the damping mask is one profile shared by every mode).
__global__ void k_scale_mask(int64_t n, int Nr, double s, const double *mask, const double2 *x, double2 *y,
                             const Krylov *kr)
{
    pdl_wait();
    // with kr: s = kr->rhs_norm, and only once the candidate is accepted
    if (kr) {
        if (!kr->accepted) return;
        s = kr->rhs_norm;
    }
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const double f = mask ? s * mask[e % Nr] : s;
        y[e] = cscale(x[e], f);
    }
}

// ---- BiCGSTAB (src/CrankNicolsonModes_matrices.cpp:47-91), device-resident scalars

// x += alpha y + omega z; r = s - omega t; per-CTA partials of |r|^2 and r0 . r.
__global__ void __launch_bounds__(VEC_THREADS) k_bicg_update(int64_t n, Krylov *kr, double2 *x, const double2 *y,
                                                              const double2 *z, double2 *r, const double2 *s,
                                                              const double2 *t, const double2 *r0, double *partials,
                                                              double *red, unsigned *ticket)
{
    pdl_wait();
    if (kr->done || kr->restart) return;  // queued ahead of the convergence test
    __shared__ double scratch[6 * 32];
    const double2 al = kr->alpha, w = kr->omega;
    double acc[3] = {0, 0, 0};
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        x[e] = cadd(x[e], cadd(cmul(al, y[e]), cmul(w, z[e])));
        const double2 rv = csub(s[e], cmul(w, t[e]));
        r[e] = rv;
        acc[0] += cabs2(rv);
        const double2 d = cconjmul(r0[e], rv);
        acc[1] += d.x;
        acc[2] += d.y;
    }
    block_sum<3>(acc, scratch);
    if (threadIdx.x == 0) {
        for (int q = 0; q < 3; ++q) partials[(int64_t)q * gridDim.x + blockIdx.x] = acc[q];
        __threadfence();
    }
    if (ticket) finish_stage(partials, gridDim.x, 3, red, kr, KS_UPDATE, ticket, scratch);
}

// Woodbury correction in place on the band of nodes [lo, hi) of every mode where the
// W_a = P^{-1} v_a can be non-negligible: y -= sum_a W_a c_a (c from kr->wc[which]).
__global__ void k_woodbury_band(int Nr, int n_modes, int lo, int hi, const Krylov *kr, int which, const double2 *W0,
                                const double2 *W1, double2 *y)
{
    pdl_wait();
    if (kr->done || kr->restart) return;  // queued ahead of the convergence test
    const double2 c0 = kr->wc[which][0], c1 = kr->wc[which][1];
    const int k = kr->n_sinks, w = hi - lo;
    const int64_t n = (int64_t)w * n_modes;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int j = (int)(e / w), i = lo + (int)(e % w);
        const int64_t q = (int64_t)j * Nr + i;
        double2 corr = cmul(W0[q], c0);
        if (k > 1) corr = cadd(corr, cmul(W1[q], c1));
        y[q] = csub(y[q], corr);
    }
}

// Woodbury set-up on the device (src/CrankNicolsonModes_matrices.cpp:133-145):
// G = diag(1 / (dt/4 g_a)) + v_a^dag W_b from vw[2 b + a] = v_a^dag W_b, and G^{-1}.
__device__ void wood_setup_dev(Krylov *kr, const double2 *vw, double c0, double c1)
{
    const int k = kr->n_sinks;
    double2 G[2][2];
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
            const double2 v = (a < k && b < k) ? vw[2 * b + a] : cmake(0.0, 0.0);
            kr->vW[a][b] = v;
            G[a][b] = v;
        }
    G[0][0].x += 1.0 / c0;
    if (k > 1) G[1][1].x += 1.0 / c1;
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) kr->Gi[a][b] = cmake(0.0, 0.0);
    if (k == 1) {
        kr->Gi[0][0] = crcp(G[0][0]);
    } else if (k == 2) {
        const double2 det = csub(cmul(G[0][0], G[1][1]), cmul(G[0][1], G[1][0]));
        const double2 id = crcp(det);
        kr->Gi[0][0] = cmul(G[1][1], id);
        kr->Gi[0][1] = cmul(cmake(-G[0][1].x, -G[0][1].y), id);
        kr->Gi[1][0] = cmul(cmake(-G[1][0].x, -G[1][0].y), id);
        kr->Gi[1][1] = cmul(G[0][0], id);
    }
}

__global__ void k_wood_setup(Krylov *kr, const double2 *vw, double c0, double c1)
{
    if (threadIdx.x == 0) wood_setup_dev(kr, vw, c0, c1);
}

// Start of the solve in one pass: with s = 1/|rhs| (|rhs|^2 = red[0]),
//   b = s rhs, x = s psi, r = r0 = b - A_full x = 2 s (rhs - psi)
// because A_full + B_full = 2 I and rhs = B_full psi (src/CrankNicolsonModes.cpp:170-172,
// _matrices.cpp:36-37); per-CTA partials of |r|^2 and |b|^2 for KS_INIT.
__global__ void __launch_bounds__(VEC_THREADS) k_krylov_start(int64_t n, Krylov *kr, const double *red_in,
                                                               const double2 *rhs, const double2 *psi, double2 *x,
                                                               double2 *r, double2 *r0, double *partials, double *red,
                                                               unsigned *ticket)
{
    pdl_wait();
    __shared__ double scratch[6 * 32];
    const double nrm = sqrt(red_in[0]);
    const double sc = nrm > 0.0 ? 1.0 / nrm : 0.0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        kr->rhs_norm = nrm;
        kr->zero_rhs = nrm == 0.0;
    }
    double acc[4] = {0, 0, 0, 0};
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const double2 hv = rhs[e], pv = psi[e];
        const double2 bv = cscale(hv, sc);
        const double2 rv = cscale(csub(hv, pv), 2.0 * sc);
        x[e] = cscale(pv, sc);
        r[e] = rv;
        r0[e] = rv;
        acc[0] += cabs2(rv);
        acc[2] += cabs2(bv);
    }
    block_sum<4>(acc, scratch);
    if (threadIdx.x == 0) {
        for (int q = 0; q < 4; ++q) partials[(int64_t)q * gridDim.x + blockIdx.x] = acc[q];
        __threadfence();
    }
    if (ticket) finish_stage(partials, gridDim.x, 4, red, kr, KS_INIT, ticket, scratch);
}

// Woodbury projections: with proj_a = v_a^dag yP (dots), c = G^{-1} proj and the sink
// dots of the corrected vector, v_a^dag y = proj_a - sum_b (v_a^dag W_b) c_b.
__device__ void wood_scalar_dev(Krylov *kr, int which, const double2 *proj)
{
    const int k = kr->n_sinks;
    double2 c[2] = {cmake(0, 0), cmake(0, 0)};
    for (int a = 0; a < k; ++a)
        for (int b = 0; b < k; ++b) c[a] = cadd(c[a], cmul(kr->Gi[a][b], proj[b]));
    for (int a = 0; a < 2; ++a) kr->wc[which][a] = c[a];
    for (int a = 0; a < k; ++a) {
        double2 d = proj[a];
        for (int b = 0; b < k; ++b) d = csub(d, cmul(kr->vW[a][b], c[b]));
        kr->sdots[which][a] = d;
    }
}

__global__ void k_wood_scalar(Krylov *kr, int which, const double2 *proj)
{
    if (threadIdx.x == 0 && !(kr->done || kr->restart)) wood_scalar_dev(kr, which, proj);
}

// ------------------------------------------------------------------ absorbers

// Legendre moments 2 pi int K(s) P_l(cos gamma) d cos gamma of one body's kernel at one
// radial node per CTA (src/CrankNicolsonModes_absorption.cpp:35-70): Gauss-Legendre
// quadrature over the angular cap z = 1 - cos(gamma) in [0, cap], one quadrature node
// per thread, Legendre recurrence to degree 2 l_max.
// Legendre moments of an absorber profile at node i into mom[l][i], l <= degree
// (src/CrankNicolsonModes_absorption.cpp:12-81), unnormalised; sh: (degree + 1) x warps doubles.
__device__ void abs_moments_node(const double *r, int Nr, int i, double radius, double width, int nq,
                                 const double *gl_x, const double *gl_w, int degree, double *mom, double *sh)
{
    if (i < 1 || i > Nr - 2) return;
    const double delta = r[i] - radius;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (fabs(delta) >= width) {
        for (int l = threadIdx.x; l <= degree; l += blockDim.x) mom[(int64_t)l * Nr + i] = 0.0;
        return;
    }
    if (radius == 0.0) {
        if (threadIdx.x == 0) {
            const double x = r[i] / width;
            mom[i] = 4.0 * M_PI * exp(-1.0 / (1.0 - x * x));
            for (int l = 1; l <= degree; ++l) mom[(int64_t)l * Nr + i] = 0.0;
        }
        return;
    }
    const double product = 2.0 * r[i] * radius;
    const double cap = fmin(2.0, (width * width - delta * delta) / product);
    // one quadrature node per thread (blockDim.x >= nq): its weight and u = cos(gamma)
    // once, then the Legendre recurrence advanced degree by degree
    const int k = threadIdx.x;
    double weight = 0.0, u = 0.0;
    if (k < nq) {
        const double z = cap * gl_x[k];
        u = 1.0 - z;
        const double d2 = delta * delta + product * z;
        weight = 2.0 * M_PI * cap * gl_w[k] * exp(-1.0 / (1.0 - d2 / (width * width)));
    }
    double prev = 1.0, cur = u;
    for (int l = 0; l <= degree; ++l) {
        double pl;
        if (l == 0) {
            pl = 1.0;
        } else if (l == 1) {
            pl = u;
        } else {
            const double next = ((2 * l - 1) * u * cur - (l - 1) * prev) / l;
            prev = cur;
            cur = next;
            pl = cur;
        }
        double part = k < nq ? 0.0 + weight * pl : 0.0;
        part = warp_sum(part);
        if (lane == 0) sh[l * nw + warp] = part;
    }
    __syncthreads();
    for (int l = threadIdx.x; l <= degree; l += blockDim.x) {
        double s = 0.0;
        for (int w = 0; w < nw; ++w) s += sh[l * nw + w];
        mom[(int64_t)l * Nr + i] = s;
    }
}

// Moments of one or two absorbers in one launch: CTA b < hi[0] - lo[0] takes node lo[0] + b
// of the first entry, the others the nodes of the second.  The moments stay unnormalised;
// the projector kernel divides by the profile's norm.
__global__ void k_abs_moments(const double *r, int Nr, int nq, const double *gl_x, const double *gl_w, int degree,
                              AbsorberPair ap)
{
    pdl_wait();
    extern __shared__ double sh[];  // (degree + 1) * nwarps
    const int n0 = ap.hi[0] - ap.lo[0];
    const int a = (int)blockIdx.x < n0 ? 0 : 1;
    abs_moments_node(r, Nr, ap.lo[a] + (int)blockIdx.x - (a == 0 ? 0 : n0), ap.radius[a], ap.width[a], nq, gl_x,
                     gl_w, degree, ap.mom[a], sh);
}

// s-wave projectors of one or two absorbers (src/CrankNicolsonModes_absorption.cpp:
// 153-182): every CTA first forms each profile's norm sum_support dr r^2 mom_0 (the same
// fixed-order sum in every CTA), then the threads write v_a on [wlo_a, whi_a), zero
// outside the support [lo_a, hi_a); blockDim.x = 256.
__global__ void __launch_bounds__(256) k_swave_projector(const double *r, int Nr, int n_modes, double dr,
                                                         const double *ang00, const int *mode_l, const int *mode_m,
                                                         double theta, AbsorberPair ap)
{
    pdl_wait();
    __shared__ double scratch[32];
    __shared__ double norm_s[2];
    for (int a = 0; a < ap.count; ++a) {
        double acc[1] = {0.0};
        for (int i = ap.lo[a] + threadIdx.x; i < ap.hi[a]; i += blockDim.x)
            if (i >= 1 && i <= Nr - 2) acc[0] += dr * r[i] * r[i] * ap.mom[a][i];
        block_sum<1>(acc, scratch);
        if (threadIdx.x == 0) norm_s[a] = acc[0];
    }
    __syncthreads();
    const int w0 = ap.whi[0] - ap.wlo[0];
    const int64_t t0 = (int64_t)w0 * n_modes;
    const int64_t tot = t0 + (ap.count > 1 ? (int64_t)(ap.whi[1] - ap.wlo[1]) * n_modes : 0);
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int a = e < t0 ? 0 : 1;
        const int64_t f = a == 0 ? e : e - t0;
        const int w = ap.whi[a] - ap.wlo[a];
        const int j = (int)(f / w), i = ap.wlo[a] + (int)(f - (int64_t)j * w);
        double2 val = cmake(0.0, 0.0);
        if (i >= 1 && i <= Nr - 2 && ang00[j] != 0.0 && i >= ap.lo[a] && i < ap.hi[a]) {
            const int ms = -mode_m[j];
            double sn, cs;
            sincos((double)ms * theta, &sn, &cs);
            const double parity = (ap.secondary[a] && (ms & 1)) ? -1.0 : 1.0;
            const double norm = norm_s[a];
            double m = ap.mom[a][(int64_t)mode_l[j] * Nr + i];
            if (norm > 0.0) m /= norm;
            const double2 kappa = cscale(cmake(cs, sn), m * ang00[j]);
            val = cscale(kappa, r[i] * sqrt(4.0 * M_PI) * parity);
        }
        ap.v[a][(int64_t)j * Nr + i] = val;
    }
}

// ------------------------------------------------------------------ diagnostics

// out[q] = sum_b partials[q][b]: one CTA per slot, coalesced loads, fixed-order tree.
__global__ void k_sum_slots(const double *partials, int nblocks, int nslots, double *out, const Krylov *gate)
{
    pdl_wait();
    if (gate && gate_closed(gate, GATE_ACCEPTED)) return;
    __shared__ double scratch[32];
    const int q = blockIdx.x;
    if (q >= nslots) return;
    double acc[1] = {0.0};
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) acc[0] += partials[(int64_t)q * nblocks + b];
    block_sum<1>(acc, scratch);
    if (threadIdx.x == 0) out[q] = acc[0];
}

// ------------------------------------------------------------------ initial states

// Legendre moments of a hydrogenic 1s density centred at distance `distance` from the
// origin (src/DisplacedAtom.cpp:45-70): one CTA per interior node, one Gauss-Legendre
// node of the body-centred distance s per thread (blockDim.x >= nq), the Legendre
// recurrence advanced degree by degree, fixed-order sums.  mom: (lmax + 1) x Nr.
__global__ void k_displaced_100(const double *r, int Nr, int lmax, double a0, double distance, double amplitude,
                                int nq, const double *gl_x, const double *gl_w, double *mom)
{
    extern __shared__ double shd[];  // (lmax + 1) * nwarps
    const int i = blockIdx.x + 1;
    if (i > Nr - 2) return;
    const double ri = r[i];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (distance == 0.0) {
        if (threadIdx.x == 0) {
            mom[i] = 4.0 * M_PI * amplitude * exp(-ri / a0);
            for (int l = 1; l <= lmax; ++l) mom[(int64_t)l * Nr + i] = 0.0;
        }
        return;
    }
    const double low = fabs(ri - distance), high = fmin(ri + distance, low + 40.0 * a0);
    const int k = threadIdx.x;
    double weight = 0.0, u = 0.0;
    if (k < nq) {
        const double sv = low + (high - low) * gl_x[k];
        u = fmin(1.0, fmax(-1.0, (ri * ri + distance * distance - sv * sv) / (2.0 * ri * distance)));
        weight = 2.0 * M_PI * (high - low) * gl_w[k] * sv / (ri * distance) * amplitude * exp(-sv / a0);
    }
    double prev = 1.0, cur = u;
    for (int l = 0; l <= lmax; ++l) {
        double pl;
        if (l == 0) {
            pl = 1.0;
        } else if (l == 1) {
            pl = u;
        } else {
            const double next = ((2 * l - 1) * u * cur - (l - 1) * prev) / l;
            prev = cur;
            cur = next;
            pl = cur;
        }
        double part = k < nq ? weight * pl : 0.0;
        part = warp_sum(part);
        if (lane == 0) shd[l * nw + warp] = part;
    }
    __syncthreads();
    for (int l = threadIdx.x; l <= lmax; l += blockDim.x) {
        double sm = 0.0;
        for (int w = 0; w < nw; ++w) sm += shd[l * nw + w];
        mom[(int64_t)l * Nr + i] = sm;
    }
}

// ------------------------------------------------------------------ fallback preconditioner

// Inverse diagonal of A = 1 + i dt/2 (H0 + V + CAP): the point-Jacobi preconditioner of
// the fallback solve that replaces the reference's ILUT retry
// (src/CrankNicolsonModes_matrices.cpp:175-186,203-214).
__global__ void k_jacobi_diag(Grid g, CouplingTable ct, const double *hh, double half_dt, double2 *dj)
{
    const int64_t n = (int64_t)g.n_modes * g.Nr;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int j = (int)(e / g.Nr), i = (int)(e % g.Nr);
        dj[e] = crcp(a_diag(g, ct, hh, half_dt, j, i));
    }
}

// out = diag(A)^{-1} b, with b = the PrecondInput combination formed on the fly (and
// stored to in.out) as in the block solves.
__global__ void k_jacobi_apply(int64_t n, const double2 *dj, const double2 *b, double2 *out, PrecondInput in)
{
    if (!resolve_input(in)) return;
    double2 beta = cmake(0, 0), omega = cmake(0, 0), alpha = cmake(0, 0);
    if (in.mode != PI_PLAIN) {
        beta = in.kr->beta;
        omega = in.kr->omega;
        alpha = in.kr->alpha;
    }
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        double2 rhsv;
        if (in.mode == PI_PLAIN) {
            rhsv = b[e];
        } else {
            if (in.mode == PI_P)
                rhsv = in.p_old ? cadd(in.r[e], cmul(beta, csub(in.p_old[e], cmul(omega, in.v[e])))) : in.r[e];
            else
                rhsv = csub(in.r[e], cmul(alpha, in.v[e]));
            in.out[e] = rhsv;
        }
        out[e] = cmul(dj[e], rhsv);
    }
}

// ------------------------------------------------------------------ FP64 FMA peak

// Microbenchmark of the FP64 pipe: eight independent FMA chains per thread (enough
// to cover the FMA latency with two or more warps per scheduler); the sum is stored
// only under a condition that never holds, so the chains stay live.
__global__ void __launch_bounds__(512) k_fp64_peak(double *out, int iters, double b, double c)
{
    double a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = 1.0 + 1e-3 * (threadIdx.x + 32 * k);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = fma(a[k], b, c);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == -1.0) out[blockIdx.x] = s;
}

}  // namespace cnm

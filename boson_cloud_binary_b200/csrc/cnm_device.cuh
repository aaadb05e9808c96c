// cnm_device.cuh -- device helpers shared by the kernel translation units:
// deterministic warp/block sums, the scalar steps of the BiCGSTAB recurrence and the
// last-CTA completion of a reduction.
#pragma once

#include "cnm_kernels.cuh"

namespace cnm {

// ------------------------------------------------------------------ reductions

// Programmatic dependent launch: a kernel launched with programmatic stream serialization
// may be scheduled before the kernel ahead of it on the stream has finished; it waits here,
// before its first access to global memory, until that kernel has completed and its
// writes are visible.  A no-op for an ordinary launch.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block sum of NV doubles per thread; result valid in thread 0.
template <int NV>
__device__ inline void block_sum(double (&v)[NV], double *scratch /* NV * 32 */)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = warp_sum(v[q]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) scratch[q * 32 + warp] = v[q];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double s = lane < nw ? scratch[q * 32 + lane] : 0.0;
            v[q] = warp_sum(s);
        }
    }
    __syncthreads();
}

// Scalar steps of the recurrence.
__device__ inline void bicg_stage(Krylov *kr, int stage, const double *red)
{
    switch (stage) {
    case KS_BETA: {  // rho_old = rho; rho = r0 . r; restart check; beta
        const double2 rho_old = kr->rho;
        kr->rho = kr->r0r;
        kr->restart = sqrt(cabs2(kr->rho)) < kr->restart_thr ? 1 : 0;
        kr->rho_old = rho_old;
        kr->beta = cmul(cdiv(kr->rho, rho_old), cdiv(kr->alpha, kr->omega));
        break;
    }
    case KS_ALPHA:  // alpha = rho / (r0 . v); red = {re, im}
        kr->alpha = cdiv(kr->rho, cmake(red[0], red[1]));
        break;
    case KS_OMEGA: {  // red = {ts.re, ts.im, tt}
        const double tt = red[2];
        kr->omega = tt > 0.0 ? cscale(cmake(red[0], red[1]), 1.0 / tt) : cmake(0.0, 0.0);
        break;
    }
    case KS_UPDATE:  // red = {|r|^2, r0.r re, im}; also flags the next iteration's restart
        kr->r2 = red[0];
        kr->r0r = cmake(red[1], red[2]);
        kr->iterations += 1;
        kr->pturn ^= 1;
        kr->done = !(kr->r2 > kr->thr) || kr->iterations >= kr->max_iterations;
        kr->restart = sqrt(cabs2(kr->r0r)) < kr->restart_thr ? 1 : 0;
        break;
    case KS_INIT: {  // red = {|r0|^2, 0, |b|^2, 0}
        const double r0n2 = red[0], b2 = red[2];
        kr->rho = kr->alpha = kr->omega = cmake(1.0, 0.0);
        kr->thr = kr->tol * kr->tol * b2;
        const double eps = 2.220446049250313e-16;
        kr->restart_thr = kr->eigen_path ? eps * eps * r0n2 : 1e-32 * r0n2;
        kr->r2 = r0n2;
        kr->r0r = cmake(r0n2, 0.0);
        kr->iterations = 0;
        kr->done = !(r0n2 > kr->thr) || kr->max_iterations <= 0;
        kr->restart = 0;
        break;
    }
    case KS_RESID: {  // red = {| |rhs| A x - rhs |^2}
        const double r2 = red[0];
        double res;
        if (!isfinite(r2)) res = INFINITY;
        else if (kr->rhs_norm > 0.0) res = sqrt(r2) / kr->rhs_norm;
        else res = r2 == 0.0 ? 0.0 : INFINITY;
        kr->residual = res;
        kr->accepted = (res <= kr->accept) && !(kr->status && *kr->status != 0);
        break;
    }
    default: break;
    }
}

__device__ __forceinline__ bool gate_closed(const Krylov *kr, int mode)
{
    if (!kr || mode == GATE_NONE) return false;
    if (mode == GATE_ITER) return kr->done || kr->restart;
    if (mode == GATE_DONE) return !kr->done;
    return !kr->accepted;
}

// Resolve a solve's input at launch: false when the gate is closed; otherwise picks the
// search-direction buffers of a ping-pong PI_P input.
__device__ __forceinline__ bool resolve_input(PrecondInput &in)
{
    if (in.gate != GATE_NONE && gate_closed(in.kr, in.gate)) return false;
    if (in.mode == PI_P && in.p_alt) {
        const int turn = in.kr->pturn;
        double2 *a = const_cast<double2 *>(in.p_old), *b = in.p_alt;
        in.out = turn ? b : a;
        in.p_old = in.first ? nullptr : (turn ? a : b);
    } else if (in.mode == PI_P && in.first) {
        in.p_old = nullptr;
    }
    return true;
}

// Completion of a launch whose CTAs each left `nslots` partial sums in
// partials[slot * nblocks + block]: every CTA calls this after its partial store (the
// threads that stored a partial issue __threadfence() right after it; no other
// thread waits on a fence, so the CTA's bulk stores stay in flight); the CTA that
// takes the last ticket sums the partials in a fixed order, independent of which CTA
// finishes last, stores red[0..nslots) and runs the scalar stage; after KS_INIT and
// KS_UPDATE it also forms the next beta unless the solve is done or must restart.
// The ticket is re-armed for the next launch.  `scratch` is 6 * 32 doubles of shared
// memory; blockDim.x must be a multiple of 32.
__device__ inline void finish_stage(const double *partials, int nblocks, int nslots, double *red, Krylov *kr, int stage,
                             unsigned *ticket, double *scratch)
{
    __shared__ unsigned s_last;
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(ticket, 1u) == (unsigned)nblocks - 1u ? 1u : 0u;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // four partials of every slot in flight per thread; each thread still adds its
    // partials in increasing block order
    double acc[6] = {0, 0, 0, 0, 0, 0};
    const int ns = min(nslots, 6);
    for (int b0 = threadIdx.x; b0 < nblocks; b0 += 4 * blockDim.x) {
        double v[4][6];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int b = b0 + u * blockDim.x;
#pragma unroll
            for (int q = 0; q < 6; ++q)
                v[u][q] = (b < nblocks && q < ns) ? __ldcg(partials + (int64_t)q * nblocks + b) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int q = 0; q < 6; ++q) acc[q] += v[u][q];
    }
    block_sum<6>(acc, scratch);
    if (threadIdx.x == 0) {
        for (int q = 0; q < nslots && q < 6; ++q) red[q] = acc[q];
        if (kr && stage != KS_NONE) {
            bicg_stage(kr, stage, red);
            if ((stage == KS_INIT || stage == KS_UPDATE) && !kr->done && !kr->restart) bicg_stage(kr, KS_BETA, red);
        }
        *ticket = 0u;
    }
}

}  // namespace cnm

// cnm_common.cuh -- shared types of the B200 Crank-Nicolson step.
//
// Layout in HBM (one binary):
//   states      complex128 (double2), mode-major: element j*Nr + i is mode j at
//               radial node i, as in the reference (include/CrankNicolsonModes.hpp:10-12).
//   hh table    (2 l_max + 1) x Nr doubles: the radial multipole weights
//               h_l*(r_i) = -mu (M1+M2) [F1_l*(r_i) + w (-1)^l* F2_l*(r_i)]
//               (F1, F2 of src/CrankNicolsonModes_hamiltonian.cpp:12-42).
//   coupling    per row mode j a list of pairs (j, k); per pair a list of terms
//               (l*, g) with g = angular * 4 pi / (2 l* + 1): the reference's
//               coupling cache (src/CrankNicolsonModes_hamiltonian.cpp:68-104)
//               with the l*-dependent prefactor folded in.
//   pivots      complex128 inverse Thomas pivots, mode-major, rebuilt whenever
//               the diagonal of A changes (include/RadialBlockPreconditioner.hpp:44-77).
//
// The coupling is never materialised.  At node r the potential block is
//   V(r) = D(theta) Ahat(r) D(theta)^dagger,  D = diag(exp(-i m_j theta)),
//   Ahat_jk(r) = sum_l* g_jkl* h_l*(r)   (real and symmetric),
// because the orbital phase of a pair is exp(i (m_k - m_j) theta)
// (_hamiltonian.cpp:106-109,186-188) and (-1)^(m_k-m_j) = (-1)^l* for every
// non-zero Gaunt term.  Kernels rebuild Ahat(r) on chip from the term list and
// the hh table.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <utility>

namespace cnm {

// ------------------------------------------------------------------ complex helpers

__host__ __device__ __forceinline__ double2 cmake(double re, double im) { return make_double2(re, im); }
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
// conj(a) * b
__host__ __device__ __forceinline__ double2 cconjmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }
__host__ __device__ __forceinline__ double2 crcp(double2 a)
{
    const double n = a.x * a.x + a.y * a.y;
    return make_double2(a.x / n, -a.y / n);
}
__host__ __device__ __forceinline__ double2 cdiv(double2 a, double2 b) { return cmul(a, crcp(b)); }
// i * a
__host__ __device__ __forceinline__ double2 cmuli(double2 a) { return make_double2(-a.y, a.x); }

// ------------------------------------------------------------------ device tables

struct CouplingTable {
    int n_modes;
    int l_max;
    int n_pairs;
    int n_terms;
    const int *pair_row_ptr;   // [n_modes + 1]
    const int *pair_col;       // [n_pairs]
    const int *pair_term_ptr;  // [n_pairs + 1]
    const int *term_l;         // [n_terms]
    const double *term_g;      // [n_terms]
    const int *diag_pair;      // [n_modes]: the pair (j, j), or -1
    const int *mode_l;         // [n_modes]
    const int *mode_m;         // [n_modes]
};

// Register-blocked layout of the same coupling (see BlockedCoupling in cnm_coupling.h).
constexpr int ROW_BLOCK = 4;
struct BlockTable {
    int n_chunks;
    const int *chunk_l;     // [n_chunks]
    const int *chunk_nrows; // [n_chunks]
    const int *chunk_rows;  // [n_chunks * ROW_BLOCK]
    const int *chunk_goff;  // [n_chunks * (l_max + 1)]
    const int *l_off;       // [l_max + 2]
    const double *g;
};

// Grid description shared by all kernels.
struct Grid {
    int Nr;
    int n_modes;
    double dr;
    double mu;
    const double *r;     // [Nr]
    const double *capw;  // [Nr] or null: CAP = -i capw(r) (all modes)
    const double *ir2;   // [Nr] 1 / r^2 (0 at r = 0)
};

// Work plan of the operator kernel (host side: cnm::CouplingPlan): warp list b of
// the CTA group y = b / warps is the chunk range [list_ptr[b], list_ptr[b + 1]); the
// group's Gaunt weights are g[group_goff[y] .. group_goff[y + 1]).
struct ApplyPlan {
    const int *list_ptr;
    const int *group_goff;
};

// Components of a generic operator application
//   y = alpha x + beta (c_h0 H0 x + Vop x + c_cap CAP x) + sum_a coef_a (v_a^dag x_a) v_a.
enum VPart : int { V_NONE = 0, V_POT = 1, V_DVDT = 2 };

struct ApplyArgs {
    const double2 *x;
    double2 *y;
    double2 alpha;
    double2 beta;
    int use_h0;
    int use_cap;
    int vpart;                  // VPart
    const double *hh;           // (2 l_max + 1) x Nr table for the potential part
    double theta;               // orbital angle for D(theta)
    double domega;              // s * Omega for dV/dt
    // rank-one sinks (up to two): y += sink_coef[a] * dots[a] * v_a on the support
    int n_sinks;
    const double2 *sink_v[2];
    const double2 *sink_dots;   // device: v_a^dag x for each sink
    double sink_coef[2];
    int sink_lo[2], sink_hi[2]; // node support [lo, hi) of each v_a
    // fused inner products of the output y with itself or another vector, as per-CTA
    // partials [slot][block]: kind 1 conj(ext) . y, 2 conj(y) . ext, 3 |y|^2 (real)
    // (kind 4: |dot_scale y - ext|^2, real)
    int n_dots;
    int dot_kind[2];
    const double2 *dot_ext[2];
    double *dot_partials;
    double dot_scale;
    // completion (stage >= 0): the CTA that finishes last sums the partials into red
    // and runs that scalar stage of the Krylov recurrence (see finish_stage)
    int stage;
    struct Krylov *kr;
    unsigned *ticket;
    double *red;
    // device-side gate of a launch queued ahead of the host's test (GateMode), and the
    // source of dot_scale (kr->rhs_norm) when set
    const struct Krylov *gate;
    int gate_mode;
    const struct Krylov *scale_kr;
};

#ifdef __CUDACC__
// Launch with programmatic stream serialization: the kernel may be scheduled while the
// kernel ahead of it on the stream is still running, so its launch overlaps that kernel's
// tail.  Every kernel launched this way calls pdl_wait() (cnm_device.cuh) before its first
// access to global memory.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                              Args &&...args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}
#endif

}  // namespace cnm

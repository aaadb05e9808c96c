// cnm_mixed.cuh -- the mixed-precision Crank-Nicolson solve: complex64 work vectors, a
// tensor-core coupling apply (tcgen05, fp16 operands, fp32 accumulators in TMEM), an
// fp32 radial-block preconditioner, and fp64 residuals, dots and refinement.
//
// The CN system A_full x = b (src/CrankNicolsonModes_matrices.cpp:94-215) is solved by
// defect correction: x0 = psi, r0 = b - A_full psi (fp64); each pass runs one
// right-preconditioned BiCGSTAB iteration (the reference's recurrence,
// src/CrankNicolsonModes_matrices.cpp:47-91, from a zero guess) on A_full d = r with the
// low-precision operator, adds d to x in fp64 and forms the next residual.  The
// residual after the first pass is an fp64 operator application; the last correction
// is small enough (|d| ~ 1e-8 |x|) that A_full d from the tensor-core apply, subtracted
// from the fp64 residual, gives the fp64 residual of the sum to well below the
// 1e-12 stopping bound (the host checks an error bound before trusting it).
//
// Tensor-core coupling.  At node r the potential block is D(theta) Ahat(r) D^dag with
// Ahat(r) = sum_l* h_l*(r) G_l*, G_l* the real Gaunt matrix of multipole l* (rows j,
// columns k).  For a tile of 128 nodes the kernel forms, per l*, the fp16 operand
//   Z_l*[m, k] = h_l*(r_node) z_k(r_node)_(Re|Im),   m = 2 node + (0 | 1),
// and accumulates  D[j, m] += sum_k G_l*[j, k] Z_l*[m, k]  in one fp32 TMEM accumulator
// (M = 128 modes, N = 256 node components, K = 16 per instruction); G_l*
// arrives in shared memory by bulk copy from a pre-formatted fp16 image (scaled by a power
// of two, as the operand is per tile, to sit near the top of the fp16 range).  Multipoles
// whose radial weight is below 1e-9 of the monopole at every node of the tile are
// skipped, and so are 16-column slices of G_l* that are zero.
#pragma once

#include <cstdint>
#include <vector>

#include "cnm_kernels.cuh"

namespace cnm {

// Shared-memory image of the Gaunt matrices for the tensor-core apply (host built).
// Per multipole l* the blob holds its non-zero K slices (16 columns k each) as 4096-byte
// blocks in the canonical K-major, no-swizzle layout of tcgen05 (rows j padded to 128):
//   byte (k % 16 / 8) * 2048 + (j / 8) * 128 + (j % 8) * 16 + (k % 8) * 2,  j < 128.
struct TcGaunt {
    int n_modes = 0, kp = 0, K = 0;           // rows, padded columns (multiple of 16), multipoles
    std::vector<uint16_t> blob;               // fp16 bits, all multipoles back to back
    std::vector<int> l_off, l_bytes;          // [K] byte offset / size of each multipole's blob
    std::vector<int> slices;                  // [K * 16]: K-slice index of each block (-1 pads)
    std::vector<int> l_nblk;                  // [K] blocks per multipole
    double fro_sum = 0.0;                     // sum_l* |G_l*|_F (error bound of the apply)
    int g_exp = 0;                            // the blob holds G 2^g_exp (fp16)
};
TcGaunt build_tc_gaunt(const struct Coupling &c);

// Device view of the image.
struct TcTable {
    const uint8_t *blob;       // `replicas` copies of the image, replica_bytes apart
    const int *l_off, *l_bytes, *slices, *l_nblk;
    int g_exp;
    int replicas;
    int64_t replica_bytes;
};
constexpr int TC_REPLICAS = 16;

// Arguments of one tensor-core operator application on complex64 vectors:
//   y = alpha x + beta (c_h0 H0 x + V x + CAP x) + sum_a coef_a (v_a^dag x) v_a,
// with up to three fused fp64 reductions of y (per-CTA partials, [slot][block]):
//   kind 1 conj(e) . y,  2 conj(y) . e,  3 |y|^2,  4 |e64 - y|^2 (e64 complex128);
// a launch's reductions read at most one external operand (kinds 1 and 2 the same e,
// and kind 4 not beside them).
struct TcArgs {
    const float2 *x;
    float2 *y;
    float2 alpha, beta;
    int use_h0, use_cap, use_v;
    const double *hh;         // (2 l_max + 1) x Nr radial weights
    float theta;
    int n_sinks;
    const double2 *sink_v[2];
    const double2 *sink_dots; // device, v_a^dag x (fp64)
    float sink_coef[2];
    int sink_lo[2], sink_hi[2];
    int n_dots;
    int dot_kind[3];
    const float2 *dot_ext[3];
    const double2 *dot_ext64;
    double *partials;         // [slot][tile]: per-tile sums, independent of the CTA that ran the tile
    int *status;              // bit 4: an mbarrier wait gave up
    int *tile_ctr;            // [2]: next tile, finished CTAs (zero between launches)
    int mx_stage;             // scalar stage run by the last CTA on the reductions (-1: none)
    struct MixScalars *msc;
};

// Host entry points (cnm_mixed.cu).
struct TcPlan {
    int kp = 0, nt = 0;       // padded mode count, nodes per tile
    int tiles = 0, grid = 0;
    size_t smem = 0;
    int a_stage = 0;          // bytes of one Gaunt stage (largest multipole blob)
    int gst = 3;              // Gaunt stages (copies run gst - 1 multipoles ahead)
};
// max_gst > 0 caps the Gaunt stages (the autotuner's candidates); 0 takes as many as fit.
bool tc_plan(int n_modes, int K, int Nr, int g_stage_bytes, int n_sm, TcPlan &p, int max_gst = 0);
constexpr int TC_MAX_STAGES = 8, TC_MIN_STAGES = 2;
cudaError_t tc_prepare(const TcPlan &p);
cudaError_t launch_tc_apply(const TcPlan &p, cudaStream_t st, const Grid &g, const int *mode_l, const int *mode_m,
                            int K, const TcTable &tt, const TcArgs &a);

// Scalars of the low-precision inner iterations (device).
struct MixScalars {
    double rr;            // |r|^2 of the pass residual (fp32 copy)
    double2 rv;           // conj(r) . v
    double2 alpha;        // rr / rv
    double2 ts;           // conj(t) . s
    double tt;            // |t|^2
    double2 omega;        // ts / tt
    double2 rho1;         // conj(r0) . r1 of the second inner iteration
    double2 beta;         // (rho1 / rho0) (alpha / omega)
    double r64;           // |r|^2 of the fp64 residual
    double b2;            // |b|^2
    double d2;            // |d|^2 of the last correction
    double tc_res2;       // |r - A d|^2 of the tensor-core residual check
    double d2_cal, e2_cal;// |d|^2 and |(r_prev - r) - A_tc d|^2 of the calibration pass
    double2 wc[2];        // Woodbury coefficients c = G^{-1} v^dag y of the last M application
    int fault;
};

// fp32 radial-block solve over thread-block clusters (one cluster per mode):
//   mode 0: x = P^{-1} b;  mode 1: s = r - alpha v (alpha from sc) is formed, stored to
//   s_out and solved;  mode 2: p = r + beta (r0 - omega v) (the second iteration's search
//   direction, with the first one's p = r0) is formed and solved.
struct Ps32Args {
    int mode;
    const float2 *b, *r, *v, *r0;
    float2 *s_out;
    const MixScalars *sc;
    int *status;
};
constexpr int PS32_THREADS = 256;
__global__ void k_psolve32_cl(int Nr, int per, float2 off, const float2 *dinv, float2 *x, Ps32Args in);

// The scalar stage a vector kernel's last block runs on its reductions (stage -1: none; the
// ticket counts finished blocks and is zero between launches).
struct MxFinish {
    MixScalars *sc;
    int stage;
    unsigned *ticket;
};
// Vector kernels of the mixed solve (fp64 accumulations into per-CTA partials).
__global__ void k_mx_start(int64_t n, const double2 *b, const double2 *psi, double2 *x, double2 *r64, float2 *r32,
                           double *partials, MxFinish f);
__global__ void k_mx_resid(int64_t n, const double2 *b, const double2 *ax, double2 *r64, double2 *diff, float2 *r32,
                           double *partials, MxFinish f);
__global__ void k_mx_update(int64_t n, const MixScalars *sc, double2 *x, const float2 *y, const float2 *z, float2 *d,
                            int first, int apply, double *partials, MxFinish f);
__global__ void k_mx_next(int64_t n, const MixScalars *sc, const float2 *s, const float2 *t, const float2 *r0,
                          float2 *r1, double *partials, MxFinish f);
__global__ void k_to_f32(int64_t n, const double2 *a, float2 *b);
__global__ void k_to_f64(int64_t n, const float2 *a, double2 *b);
__global__ void k_sink_dots32(const float2 *x, int Nr, int n_modes, int n_sinks, const double2 *v0,
                              const double2 *v1, int lo0, int hi0, int lo1, int hi1, double2 *dots);
__global__ void k_wood32(int Nr, int n_modes, int lo, int hi, const Krylov *kr, const double2 *proj,
                         const double2 *W0, const double2 *W1, float2 *y, double2 *dots_out);

enum MixStage : int { MX_RR = 0, MX_ALPHA = 1, MX_OMEGA = 2, MX_R64 = 3, MX_D2 = 4, MX_TCRES = 5, MX_B2R0 = 6, MX_ECAL = 7, MX_BETA = 8, MX_ALPHA2 = 9 };

}  // namespace cnm

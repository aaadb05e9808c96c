// cnm_mixed.cu -- kernels of the mixed-precision CN solve (see cnm_mixed.cuh): the
// tcgen05 tensor-core operator apply, the fp32 cluster radial-block solve and the
// vector kernels of the defect correction.
#include <cooperative_groups.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "cnm_coupling.h"
#include "cnm_device.cuh"
#include "cnm_mixed.cuh"

namespace cnm {

// ==================================================================== host: Gaunt image

static uint16_t f16_bits(double v)
{
    const __half h = __float2half_rn((float)v);
    uint16_t u;
    std::memcpy(&u, &h, 2);
    return u;
}

TcGaunt build_tc_gaunt(const Coupling &c)
{
    TcGaunt t;
    const int n = c.n_modes;
    t.n_modes = n;
    t.kp = (n + 15) / 16 * 16;
    t.K = 2 * c.l_max + 1;
    const int nsl = t.kp / 16;
    std::vector<double> G((size_t)t.K * n * n, 0.0);
    for (int j = 0; j < n; ++j)
        for (int p = c.pair_row_ptr[j]; p < c.pair_row_ptr[j + 1]; ++p) {
            const int k = c.pair_col[p];
            for (int e = c.pair_term_ptr[p]; e < c.pair_term_ptr[p + 1]; ++e)
                G[((size_t)c.term_l[e] * n + j) * n + k] += c.term_g[e];
        }
    // a power-of-two scale that puts the largest |G| just below 2^14, well inside fp16
    double gmax = 0.0;
    for (double v : G) gmax = std::max(gmax, std::abs(v));
    int e2 = 0;
    std::frexp(gmax > 0.0 ? gmax : 1.0, &e2);  // gmax < 2^e2
    t.g_exp = 14 - e2;
    t.l_off.assign(t.K, 0);
    t.l_bytes.assign(t.K, 0);
    t.l_nblk.assign(t.K, 0);
    t.slices.assign((size_t)t.K * 16, -1);
    for (int l = 0; l < t.K; ++l) {
        double fro = 0.0;
        t.l_off[l] = (int)(t.blob.size() * sizeof(uint16_t));
        for (int s = 0; s < nsl; ++s) {
            bool nz = false;
            for (int j = 0; j < n && !nz; ++j)
                for (int k = 16 * s; k < std::min(n, 16 * s + 16); ++k)
                    if (G[((size_t)l * n + j) * n + k] != 0.0) {
                        nz = true;
                        break;
                    }
            if (!nz) continue;
            const size_t at = t.blob.size();
            t.blob.resize(at + 2048, 0);  // 4096 bytes: 128 rows j x 16 columns k
            for (int j = 0; j < n; ++j)
                for (int k = 16 * s; k < std::min(n, 16 * s + 16); ++k) {
                    const double g = G[((size_t)l * n + j) * n + k];
                    fro += g * g;
                    const int kk = k - 16 * s;
                    const size_t byte = (size_t)(kk / 8) * 2048 + (size_t)(j / 8) * 128 + (size_t)(j % 8) * 16 +
                                        (size_t)(kk % 8) * 2;
                    t.blob[at + byte / 2] = f16_bits(std::ldexp(g, t.g_exp));
                }
            t.slices[(size_t)l * 16 + t.l_nblk[l]] = s;
            t.l_nblk[l] += 1;
        }
        t.l_bytes[l] = t.l_nblk[l] * 4096;
        t.fro_sum += std::sqrt(fro);
    }
    return t;
}

// ==================================================================== device helpers

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait on phase `parity`.  Once any wait of the CTA has given up (*abort set),
// later waits return at once, so a failed launch ends quickly; `force` waits (bounded)
// even then -- the drains of copies and MMAs in flight before the CTA exits.
__device__ __forceinline__ void mbar_wait(uint32_t bar, uint32_t parity, volatile int *abort, bool force = false)
{
    for (int it = 0; it < (1 << 22); ++it) {
        if (mbar_try(bar, parity)) return;
        if (!force && *abort) return;
    }
    *abort = 1;
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// 8-byte asynchronous global -> shared copy (zero fill when `valid` is false: nothing is read)
__device__ __forceinline__ void cp_async8(uint32_t dst, const void *src, bool valid)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(valid ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor, K-major, no swizzle: start address, leading (K)
// byte offset, stride (M/N) byte offset, descriptor version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3fffu) | ((uint64_t)((lbo >> 4) & 0x3fffu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3fffu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: fp16 A and B, fp32 D, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N)
{
    return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t dtmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
        "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

// 32 consecutive fp32 columns of this warp's 32 TMEM lanes.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 32; ++q) v[q] = __uint_as_float(r[q]);
}

// Named barrier 1 over the W worker threads (the copy / MMA warp does not take part).
template <int W>
__device__ __forceinline__ void workers_sync()
{
    asm volatile("bar.sync 1, %0;" ::"n"(W) : "memory");
}

__device__ __forceinline__ uint32_t pack_f16(float lo, float hi)
{
    const __half2 v = __floats2half2_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}

__device__ void mx_stage(const double *acc, MixScalars *sc, int stage);

// ==================================================================== tensor-core apply

constexpr int TC_GMAX = 8, TC_BSTAGES = 2;  // at most 8 Gaunt stages (the plan sets how many)
constexpr int TC_KMAX = 32;                  // multipoles (2 l_max + 1) the kernel handles
constexpr float TC_HCUT = 1e-9f;             // multipoles below this fraction of the monopole are skipped

// The launch shape by padded mode count KP.  Nodes per tile NT (2 NT node-component rows,
// the MMA's N) and CTAs per SM: 128 nodes and one CTA per SM.  The kernel also runs 64-node
// tiles with two CTAs per SM (one CTA's loads and epilogue beside the other's multipole
// loop; KP <= 96, where two CTAs' shared memory fits): on 91 modes x 40000 nodes that
// measured the same per launch (103.9 against 104.0 us), since both leave 2.1 tiles per CTA
// and the launch ends with the CTAs that run a third.  One worker thread per operand row and
// half of the columns k (4 NT workers, operand producers and epilogue), plus the copy / MMA
// warp.
__host__ __device__ constexpr int tc_nt(int) { return 128; }
__host__ __device__ constexpr int tc_ctas(int kp) { return tc_nt(kp) == 64 ? 2 : 1; }
__host__ __device__ constexpr int tc_workers(int kp) { return 4 * tc_nt(kp); }
__host__ __device__ constexpr int tc_threads(int kp) { return tc_workers(kp) + 32; }
// Row stride (floats) of the accumulator image W[j][m]: 2 NT + 4, so that 16-byte stores of
// 8 consecutive rows hit distinct banks.
__host__ __device__ constexpr int tc_ws(int kp) { return 2 * tc_nt(kp) + 4; }
// Dynamic shared memory of a plan: with two CTAs per SM each stays below half of the SM's
// 228 KiB less the per-CTA reservation and the ~3.2 KiB of static shared memory.
__host__ __device__ constexpr int tc_smem_max(int kp) { return tc_ctas(kp) == 2 ? 108 * 1024 : 220 * 1024; }
constexpr int TC_SMEM_MAX = 220 * 1024;  // the kernels' shared-memory attribute (every plan stays within it)

// Bytes of the region that holds the Z stages and, in the epilogue, the accumulator image.
__host__ __device__ constexpr size_t tc_zregion(int kp)
{
    return (size_t)TC_BSTAGES * kp * 2 * tc_nt(kp) * 2 > (size_t)kp * tc_ws(kp) * 4
               ? (size_t)TC_BSTAGES * kp * 2 * tc_nt(kp) * 2
               : (size_t)kp * tc_ws(kp) * 4;
}

struct TcShared {
    unsigned long long gfull[TC_GMAX], gfree[TC_GMAX], zfull[TC_BSTAGES], zfree[TC_BSTAGES];
    unsigned long long accfull, accfree, tinfo, drain;
    uint32_t tmem_base;
    int lcut[2];        // multipole cut of the tile in flight (-1: no further tile)
    int tile[2];        // tile index drawn from the launch's counter
    int lcut_red;
    int pmax_bits;      // largest |h z| of the tile (float bits, non-negative)
    int abort;
    int l_off[TC_KMAX], l_bytes[TC_KMAX], l_nblk[TC_KMAX];
    int slices[TC_KMAX * 16];
    double red[4 * 16];  // warp sums of a tile's fused reductions (at most 16 worker warps)
    int last;            // this CTA finished last (runs the launch's scalar stage)
};

// Bulk copy of multipole lv's Gaunt blocks into the G stage of use v (v % gst).
__device__ __forceinline__ void tc_issue_g(TcShared &sh, uint8_t *Gst, int g_stage, int gst, const uint8_t *blob, int v,
                                           int lv)
{
    const int s = v % gst;
    const uint32_t bar = smem_addr(&sh.gfull[s]);
    if (sh.l_bytes[lv] == 0) {  // no non-zero block: complete the phase without a copy
        mbar_arrive(bar);
        return;
    }
    mbar_expect_tx(bar, (uint32_t)sh.l_bytes[lv]);
    bulk_g2s(smem_addr(Gst + (size_t)s * g_stage), blob + sh.l_off[lv], (uint32_t)sh.l_bytes[lv], bar);
}

// y = alpha x + beta (H0 x + V x + CAP x) + sinks on complex64 vectors, the coupling on the
// tensor cores.  A tile is NT nodes; its 2 NT node-component rows m = 2 node + (0: Re,
// 1: Im) of Z_l*[m, k] = h_l*(r_node) z_k(r_node)_(Re|Im) form the MMA's B operand (N = 2 NT,
// K-major), the Gaunt matrix G_l* (M = 128 rows j, K-major) its A operand, and
// D[j, m] = sum_l* sum_k G_l*[j, k] Z_l*[m, k] accumulates in one fp32 TMEM accumulator
// (lane j, column m).  Worker thread w produces operand row m = w % 2 NT for half of the
// columns k (w / 2 NT); in the epilogue warp w reads TMEM lanes 32 (w % 4) .. (its quarter of
// the modes j) and its share of the columns, writes them to shared memory, and the workers
// then form one complex output per (mode, node), consecutive threads on consecutive nodes.
// Warp 16 copies Gaunt stages and issues the MMAs (one thread).  Tiles are drawn from a
// per-handle counter (tile_ctr[0]; the last CTA to finish resets it), so a CTA that got
// light tiles (few multipoles above the cut, far from the bodies) takes more of them.
// DK fixes the launch's fused reductions at compile time: 0 none, 1 conj(e) . y,
// 23 conj(y) . e and |y|^2, 4 |e64 - y|^2.
template <int KP, int DK>
__global__ void __launch_bounds__(tc_threads(KP), tc_ctas(KP))
    k_tc_apply(Grid g, const int *mode_l, const int *mode_m, int K, TcTable tt, TcArgs a, int tiles, int g_stage,
               int gst)
{
    constexpr int TC_NT = tc_nt(KP), TC_WORKERS = tc_workers(KP), TC_THREADS = tc_threads(KP);
    constexpr int TC_CTRL = TC_WORKERS / 32;   // the copy / MMA warp
    constexpr int TC_WS = tc_ws(KP);
    constexpr int LBO_Z = 2 * TC_NT / 8 * 128;   // bytes between 8-column groups of k in a Z stage
    constexpr int Z_STAGE = KP * 2 * TC_NT * 2;  // bytes of one Z stage (2 NT rows x KP fp16)
    constexpr int G_LBO = 2048;                // bytes between the two 8-column halves of a G block
    constexpr int G_BLK = 4096;                // bytes of one G block (128 rows j x 16 columns k)
    constexpr uint32_t IDESC = idesc_f16(128, 2 * TC_NT);
    constexpr uint32_t NCOLS = 2 * TC_NT;      // one fp32 accumulator: 128 lanes (modes) x 2 NT columns
    constexpr int NDOT = DK == 0 ? 0 : DK == 23 ? 2 : 1;  // fused reductions (complex slots)
    extern __shared__ __align__(128) uint8_t tc_smem[];
    __shared__ TcShared sh;
    const int n = g.n_modes, Nr = g.Nr;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // this CTA's replica of the Gaunt image: CTAs that start together would otherwise all
    // read the same lines of L2 at once
    const uint8_t *gblob = tt.blob + (size_t)(blockIdx.x % tt.replicas) * tt.replica_bytes;
    uint8_t *Gst = tc_smem;                                              // gst x g_stage
    uint8_t *Zst = Gst + (size_t)gst * g_stage;                          // Z stages / accumulator image
    // copies run gst - 1 uses ahead; a tile's first gst - 1 uses are copied before its cut is
    // known, so every tile runs at least multipoles 0 .. gst - 2
    const int lc_min = max(1, gst - 2);
    float *hs = reinterpret_cast<float *>(Zst + tc_zregion(KP));        // K x TC_NT
    float2 *ph = reinterpret_cast<float2 *>(hs + (size_t)K * TC_NT);    // KP phases e^{i m_k theta}
    float *cent = reinterpret_cast<float *>(ph + KP);                   // KP: l (l + 1) / (2 mu)
    float *ir2s = cent + KP;                                             // TC_NT: 1 / r^2 of the tile
    float *caps = ir2s + TC_NT;                                          // TC_NT: CAP weights of the tile
    volatile int *abort = &sh.abort;

    if (tid == 0) {
        for (int s = 0; s < gst; ++s) {
            mbar_init(smem_addr(&sh.gfull[s]), 1);
            mbar_init(smem_addr(&sh.gfree[s]), 1);
        }
        for (int s = 0; s < TC_BSTAGES; ++s) {
            mbar_init(smem_addr(&sh.zfull[s]), TC_WORKERS / 32);
            mbar_init(smem_addr(&sh.zfree[s]), 1);
        }
        mbar_init(smem_addr(&sh.accfull), 1);
        mbar_init(smem_addr(&sh.accfree), TC_WORKERS / 32);
        mbar_init(smem_addr(&sh.tinfo), 1);
        mbar_init(smem_addr(&sh.drain), 1);
        sh.abort = 0;
        sh.lcut_red = 0;
        sh.pmax_bits = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int l = tid; l < K; l += TC_THREADS) {
        sh.l_off[l] = tt.l_off[l];
        sh.l_bytes[l] = tt.l_bytes[l];
        sh.l_nblk[l] = tt.l_nblk[l];
    }
    for (int e = tid; e < K * 16; e += TC_THREADS) sh.slices[e] = tt.slices[e];
    for (int k = tid; k < KP; k += TC_THREADS) {
        float s = 0.f, c = 0.f;
        if (k < n) sincosf((float)mode_m[k] * a.theta, &s, &c);
        ph[k] = k < n ? make_float2(c, s) : make_float2(0.f, 0.f);
        const int l = k < n ? mode_l[k] : 0;
        cent[k] = (float)((double)(l * (l + 1)) / (2.0 * g.mu));
    }
    if (warp == TC_CTRL) {
        // TMEM accumulator: 128 lanes x 2 NT fp32 columns
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&sh.tmem_base)),
                     "r"(NCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        tc_fence_before();
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = sh.tmem_base;

    if (warp == TC_CTRL) {
        // ---------------------------------------------------------- copies and MMAs
        if (lane == 0) {
            int u = 0;       // multipole uses issued so far (all tiles)
            int copies = 0;
            // the first tile's first gst - 1 multipoles (copied even if this CTA draws no
            // tile: the drain below waits for them)
            for (; copies < gst - 1; ++copies) tc_issue_g(sh, Gst, g_stage, gst, gblob, copies, copies);
            // a CTA runs at most `tiles` tiles; the bound only matters after a wait gave up
            for (int it = 0; it < tiles; ++it) {
                mbar_wait(smem_addr(&sh.tinfo), it & 1, abort);
                const int lc = sh.lcut[it & 1];
                if (lc < 0) break;
                if (it > 0) mbar_wait(smem_addr(&sh.accfree), (it - 1) & 1, abort);
                tc_fence_after();
                bool firstmma = true;
                for (int l = 0; l <= lc; ++l, ++u) {
                    const int sg = u % gst, sz = u % TC_BSTAGES;
                    mbar_wait(smem_addr(&sh.gfull[sg]), (u / gst) & 1, abort);
                    mbar_wait(smem_addr(&sh.zfull[sz]), (u / TC_BSTAGES) & 1, abort);
                    tc_fence_after();
                    const uint32_t gbase = smem_addr(Gst + (size_t)sg * g_stage);
                    const uint32_t zbase = smem_addr(Zst + (size_t)sz * Z_STAGE);
                    const int nb = sh.l_nblk[l];
                    // one M = 128 (modes j), N = 2 NT (the tile's node-component rows), K = 16
                    // MMA per non-zero slice of G_l*: every tcgen05.mma of K = 16 costs about the
                    // same whatever its N, so N is kept at its maximum
                    for (int q = 0; q < nb; ++q) {
                        const int s16 = sh.slices[l * 16 + q];
                        const uint64_t ad = sdesc(gbase + (uint32_t)(q * G_BLK), (uint32_t)G_LBO, 128u);
                        const uint64_t bd = sdesc(zbase + (uint32_t)(s16 * 2 * LBO_Z), (uint32_t)LBO_Z, 128u);
                        tc_mma(tmem, ad, bd, IDESC, firstmma ? 0u : 1u);
                        firstmma = false;
                    }
                    tc_commit(smem_addr(&sh.gfree[sg]));
                    tc_commit(smem_addr(&sh.zfree[sz]));
                    // refill: use u + gst - 1 goes into the G stage of use u - 1; past this
                    // tile's cut it is one of the next tile's multipoles 0 .. gst - 2, which
                    // every tile runs (copied whether or not a next tile comes)
                    const int ahead = gst - 1;
                    const int lnext = l + ahead <= lc ? l + ahead : l + ahead - (lc + 1);
                    if (u >= 1) mbar_wait(smem_addr(&sh.gfree[(u - 1) % gst]), ((u - 1) / gst) & 1, abort);
                    tc_issue_g(sh, Gst, g_stage, gst, gblob, u + ahead, lnext);
                    ++copies;
                }
                tc_commit(smem_addr(&sh.accfull));
            }
            // drain: every MMA issued has completed, every copy issued has landed
            tc_commit(smem_addr(&sh.drain));
            mbar_wait(smem_addr(&sh.drain), 0, abort, true);
            for (int v = u; v < copies; ++v)
                mbar_wait(smem_addr(&sh.gfull[v % gst]), (v / gst) & 1, abort, true);
        }
        __syncwarp();
    } else {
        // ---------------------------------------------------------- workers
        // operand row m = 2 node + (Re | Im) and half of its columns k
        constexpr int KH = KP / 2;
        const int m = tid & (2 * TC_NT - 1), khalf = tid / (2 * TC_NT), zc_node = m >> 1, zc_comp = m & 1;
        const float ad = (float)(1.0 / (2.0 * g.mu * g.dr * g.dr));
        // epilogue phase 1: TMEM lane quarter (warp % 4: modes j) and a share of the columns
        // (one share per group of four warps)
        const int q4 = warp & 3, cq = warp >> 2;
        constexpr int CQ_SPAN = 2 * TC_NT / (TC_WORKERS / 128);
        const float2 al = a.alpha, be = a.beta;
        // the sinks' coefficients coef_a (v_a^dag x), fp64
        double2 sk_c[2];
#pragma unroll
        for (int s2 = 0; s2 < 2; ++s2) {
            sk_c[s2] = make_double2(0.0, 0.0);
            if (s2 < a.n_sinks) {
                const double2 dd = a.sink_dots[s2];
                sk_c[s2] = make_double2(a.sink_coef[s2] * dd.x, a.sink_coef[s2] * dd.y);
            }
        }
        // the launch's reduction operand: complex64 (kinds 1, 2) or complex128 (kind 4)
        const float2 *__restrict__ ext32 = (DK == 1 || DK == 23) ? a.dot_ext[0] : nullptr;
        const double2 *__restrict__ ext64 = DK == 4 ? a.dot_ext64 : nullptr;
        const float2 *__restrict__ xg = a.x;
        int u = 0;
        for (int it = 0;; ++it) {
            // the next tile (the barrier first: every worker has finished the previous
            // epilogue and read the previous tile index)
            if (tid == 0) sh.tile[it & 1] = atomicAdd(a.tile_ctr, 1);
            workers_sync<TC_WORKERS>();
            const int tile = sh.tile[it & 1];
            if (tile >= tiles) {
                if (tid == 0) {
                    sh.lcut[it & 1] = -1;
                    mbar_arrive(smem_addr(&sh.tinfo));
                }
                break;
            }
            const int i0 = tile * TC_NT;
            // the epilogue's reduction operand of this tile into L2 while the tile's multipole
            // loop runs (one bulk prefetch per mode row, within the vector)
            if constexpr (DK != 0) {
                if (tid < n) {
                    constexpr size_t es = DK == 4 ? sizeof(double2) : sizeof(float2);
                    const char *base = DK == 4 ? (const char *)ext64 : (const char *)ext32;
                    const size_t end = (size_t)n * Nr * es;
                    size_t b0 = ((size_t)tid * Nr + i0) * es, b1 = b0 + (size_t)min(TC_NT, Nr - i0) * es;
                    b0 &= ~(size_t)15;
                    b1 = min((b1 + 15) & ~(size_t)15, end & ~(size_t)15);
                    if (b1 > b0)
                        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(base + b0), "r"((uint32_t)(b1 - b0))
                                     : "memory");
                }
            }
            // radial weights of the tile (K x TC_NT, independent loads spread over the
            // workers), 1/r^2 and the CAP weights of its nodes
            constexpr int HPT = TC_KMAX * TC_NT / TC_WORKERS;
            double hv[HPT];
            {
#pragma unroll
                for (int q = 0; q < HPT; ++q) {
                    const int e = tid + q * TC_WORKERS;
                    const int l = e / TC_NT, i = i0 + (e % TC_NT);
                    hv[q] = (l < K && a.use_v && i >= 1 && i <= Nr - 2) ? a.hh[(int64_t)l * Nr + i] : 0.0;
                }
                if (tid < TC_NT) {
                    const int i = i0 + tid;
                    ir2s[tid] = i < Nr ? (float)g.ir2[i] : 0.f;
                } else if (tid < 2 * TC_NT) {
                    const int i = i0 + tid - TC_NT;
                    caps[tid - TC_NT] = (g.capw && i < Nr) ? (float)g.capw[i] : 0.f;
                }
            }
            // z_k of this row's node and component (e^{i m_k theta} x_k), k in this thread's half,
            // from the tile's x staged in the (idle) Z region by asynchronous copies: xs[k][c]
            float zc[KH];
            {
                float2 *xs = reinterpret_cast<float2 *>(Zst);
                constexpr int XPT = KP * TC_NT / TC_WORKERS;
#pragma unroll
                for (int q = 0; q < XPT; ++q) {
                    const int e = tid + q * TC_WORKERS;
                    const int k = e / TC_NT, i = i0 + (e % TC_NT);
                    const bool valid = k < n && i < Nr;
                    cp_async8(smem_addr(xs + e), valid ? (const void *)(xg + (int64_t)k * Nr + i) : (const void *)xg,
                              valid);
                }
                // the radial weights land while the copies are in flight
#pragma unroll
                for (int q = 0; q < HPT; ++q) {
                    const int e = tid + q * TC_WORKERS;
                    if (e < K * TC_NT) hs[e] = (float)hv[q];
                }
                cp_async_wait_all();
                workers_sync<TC_WORKERS>();
#pragma unroll
                for (int kk = 0; kk < KH; ++kk) {
                    const int k = khalf * KH + kk;
                    const float2 xv = xs[k * TC_NT + zc_node];
                    const float2 p = ph[k];
                    zc[kk] = zc_comp ? p.x * xv.y + p.y * xv.x : p.x * xv.x - p.y * xv.y;
                }
            }
            {
                // the multipole cut (the highest l* above TC_HCUT of the monopole at some node
                // of the tile) and the operand scale S = 2^se with max |S h z| < 2^14: every
                // thread evaluates its own node, a warp reduction, one atomic per warp
                const float h0 = fabsf(hs[zc_node]);
                int lcl = 0;
                float hm = h0;
                for (int l = 1; l < K; ++l) {
                    const float h = fabsf(hs[l * TC_NT + zc_node]);
                    if (h > TC_HCUT * h0) lcl = l;
                    hm = fmaxf(hm, h);
                }
                float zm = 0.f;
#pragma unroll
                for (int k = 0; k < KH; ++k) zm = fmaxf(zm, fabsf(zc[k]));
                const int lw = __reduce_max_sync(0xffffffffu, lcl);
                const int pw = __reduce_max_sync(0xffffffffu, __float_as_int(zm * hm));  // non-negative floats
                if (lane == 0) {
                    if (lw > 0) atomicMax(&sh.lcut_red, lw);
                    atomicMax(&sh.pmax_bits, pw);
                }
            }
            workers_sync<TC_WORKERS>();
            const int lc = max(lc_min, sh.lcut_red);
            int se = 0;
            {
                const float pm = __int_as_float(sh.pmax_bits);
                int e2 = 0;
                frexpf(pm > 0.f ? pm : 1.f, &e2);  // pm < 2^e2
                // clamped so that 2^se and 2^-(se + g_exp) are normal floats; a tile of values
                // below 2^-86 only loses scale, not range
                se = min(100, max(-100, 14 - e2));
                const float sz = ldexpf(1.f, se);
#pragma unroll
                for (int k = 0; k < KH; ++k) zc[k] *= sz;
            }
            const float wscale = ldexpf(1.f, -(se + tt.g_exp));  // undoes both operand scales
            workers_sync<TC_WORKERS>();
            if (tid == 0) {
                sh.lcut[it & 1] = lc;
                sh.lcut_red = 0;
                sh.pmax_bits = 0;
                mbar_arrive(smem_addr(&sh.tinfo));
            }
            // B operand rows, one multipole per stage
            for (int l = 0; l <= lc; ++l, ++u) {
                const int sz = u % TC_BSTAGES;
                if (u >= TC_BSTAGES) mbar_wait(smem_addr(&sh.zfree[sz]), ((u / TC_BSTAGES) - 1) & 1, abort);
                uint8_t *Z = Zst + (size_t)sz * Z_STAGE + (size_t)khalf * (KH / 8) * LBO_Z + (m >> 3) * 128 + (m & 7) * 16;
                const float h = hs[l * TC_NT + zc_node];
#pragma unroll
                for (int gq = 0; gq < KH / 8; ++gq) {
                    uint4 v;
                    v.x = pack_f16(h * zc[8 * gq + 0], h * zc[8 * gq + 1]);
                    v.y = pack_f16(h * zc[8 * gq + 2], h * zc[8 * gq + 3]);
                    v.z = pack_f16(h * zc[8 * gq + 4], h * zc[8 * gq + 5]);
                    v.w = pack_f16(h * zc[8 * gq + 6], h * zc[8 * gq + 7]);
                    *reinterpret_cast<uint4 *>(Z + (size_t)gq * LBO_Z) = v;
                }
                fence_proxy_async();
                __syncwarp();
                if (lane == 0) mbar_arrive(smem_addr(&sh.zfull[sz]));
            }
            // epilogue, phase 1: the accumulator to shared memory, W[j][m] with row stride
            // TC_WS (the Z stages are idle until the next tile's operand rows)
            mbar_wait(smem_addr(&sh.accfull), it & 1, abort);
            tc_fence_after();
            float *W = reinterpret_cast<float *>(Zst);
            {
                const uint32_t taddr = tmem + ((uint32_t)(32 * q4) << 16);
                const int j = 32 * q4 + lane;
                float *wrow = W + (size_t)j * TC_WS;
#pragma unroll 1
                for (int col = cq * CQ_SPAN; col < (cq + 1) * CQ_SPAN; col += 32) {
                    float wv[32];
                    tmem_ld32(taddr + (uint32_t)col, wv);
                    if (j < n)
#pragma unroll
                        for (int q = 0; q < 32; q += 4)
                            *reinterpret_cast<float4 *>(wrow + col + q) = make_float4(wv[q], wv[q + 1], wv[q + 2], wv[q + 3]);
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_addr(&sh.accfree));
            workers_sync<TC_WORKERS>();
            // phase 2: one complex output per (mode j, node) and thread, consecutive threads
            // on consecutive nodes of one mode (coalesced loads and stores); a warp's lanes
            // hold 32 consecutive nodes, so the stencil's neighbours come by shuffles and
            // only the first lane's left and the last lane's right neighbour are loaded.  The
            // products of the fused reductions are formed in fp32 (their operands are fp32
            // values; the residual check's difference in fp64) and summed per tile in fp32,
            // then in fp64 across tiles.
            {
                const int tile_nodes = min(TC_NT, Nr - i0);
                constexpr int EB = 6;  // elements in flight per thread
                using Ext = typename std::conditional<DK == 4, double2, float2>::type;
                float2 *__restrict__ yg = a.y;
                float tacc[3] = {0.f, 0.f, 0.f};
#pragma unroll 1
                for (int e0 = tid; e0 < n * TC_NT; e0 += EB * TC_WORKERS) {
                    float2 x0[EB], xh[EB];
                    Ext ev[EB];
#pragma unroll
                    for (int q = 0; q < EB; ++q) {
                        const int e = e0 + q * TC_WORKERS;
                        const int j = e / TC_NT, c = e - j * TC_NT;
                        const bool ok = e < n * TC_NT && c < tile_nodes;
                        const int i = i0 + c;
                        const int64_t o = (int64_t)j * Nr + i;
                        const float2 zero = make_float2(0.f, 0.f);
                        x0[q] = ok ? __ldg(xg + o) : zero;
                        xh[q] = zero;
                        if (ok && lane == 0 && i >= 1) xh[q] = __ldg(xg + o - 1);
                        if (ok && lane == 31 && i + 1 < Nr) xh[q] = __ldg(xg + o + 1);
                        if constexpr (DK == 1 || DK == 23) ev[q] = ok ? __ldg(ext32 + o) : zero;
                        else if constexpr (DK == 4) ev[q] = ok ? __ldg(ext64 + o) : make_double2(0.0, 0.0);
                    }
#pragma unroll
                    for (int q = 0; q < EB; ++q) {
                        float2 xm, xp;
                        xm.x = __shfl_up_sync(0xffffffffu, x0[q].x, 1);
                        xm.y = __shfl_up_sync(0xffffffffu, x0[q].y, 1);
                        xp.x = __shfl_down_sync(0xffffffffu, x0[q].x, 1);
                        xp.y = __shfl_down_sync(0xffffffffu, x0[q].y, 1);
                        if (lane == 0) xm = xh[q];
                        if (lane == 31) xp = xh[q];
                        const int e = e0 + q * TC_WORKERS;
                        const int j = e / TC_NT, c = e - j * TC_NT;
                        if (!(e < n * TC_NT && c < tile_nodes)) continue;
                        const int i = i0 + c;
                        const int64_t o = (int64_t)j * Nr + i;
                        const float2 w = *reinterpret_cast<const float2 *>(W + j * TC_WS + 2 * c);
                        const float wr_ = w.x * wscale, wi_ = w.y * wscale;
                        float hr = 0.f, hi = 0.f;
                        if (i >= 1 && i <= Nr - 2) {
                            if (a.use_h0) {
                                // H0 x = ad ((x - x_-) + (x - x_+)) + l (l + 1) / (2 mu r^2) x: the
                                // differences of neighbours are exact for a smooth x
                                const float cen = cent[j] * ir2s[c];
                                hr = ad * ((x0[q].x - xm.x) + (x0[q].x - xp.x)) + cen * x0[q].x;
                                hi = ad * ((x0[q].y - xm.y) + (x0[q].y - xp.y)) + cen * x0[q].y;
                            }
                            if (a.use_v) {  // conj(ph_j) w
                                const float2 p = ph[j];
                                hr += p.x * wr_ + p.y * wi_;
                                hi += p.x * wi_ - p.y * wr_;
                            }
                        }
                        if (a.use_cap) {
                            const float cw = caps[c];
                            hr += cw * x0[q].y;
                            hi -= cw * x0[q].x;
                        }
                        float yr = al.x * x0[q].x - al.y * x0[q].y + be.x * hr - be.y * hi;
                        float yi = al.x * x0[q].y + al.y * x0[q].x + be.x * hi + be.y * hr;
#pragma unroll
                        for (int s2 = 0; s2 < 2; ++s2)
                            if (s2 < a.n_sinks && i >= a.sink_lo[s2] && i < a.sink_hi[s2]) {
                                const double2 vv = a.sink_v[s2][o];
                                yr += (float)(sk_c[s2].x * vv.x - sk_c[s2].y * vv.y);
                                yi += (float)(sk_c[s2].x * vv.y + sk_c[s2].y * vv.x);
                            }
                        yg[o] = make_float2(yr, yi);
                        if constexpr (DK == 1) {  // conj(e) y
                            tacc[0] = fmaf(ev[q].x, yr, fmaf(ev[q].y, yi, tacc[0]));
                            tacc[1] = fmaf(ev[q].x, yi, fmaf(-ev[q].y, yr, tacc[1]));
                        } else if constexpr (DK == 23) {  // conj(y) e, |y|^2
                            tacc[0] = fmaf(yr, ev[q].x, fmaf(yi, ev[q].y, tacc[0]));
                            tacc[1] = fmaf(yr, ev[q].y, fmaf(-yi, ev[q].x, tacc[1]));
                            tacc[2] = fmaf(yr, yr, fmaf(yi, yi, tacc[2]));
                        } else if constexpr (DK == 4) {  // |e64 - y|^2
                            const float ddr = (float)(ev[q].x - (double)yr), ddi = (float)(ev[q].y - (double)yi);
                            tacc[0] = fmaf(ddr, ddr, fmaf(ddi, ddi, tacc[0]));
                        }
                    }
                }
                // the tile's partials [slot][tile] (warps, then the warp sums in order): the
                // sums do not depend on which CTA ran the tile
                if constexpr (NDOT > 0) {
                    double v[4] = {(double)tacc[0], DK == 4 ? 0.0 : (double)tacc[1], DK == 23 ? (double)tacc[2] : 0.0,
                                   0.0};
#pragma unroll
                    for (int q = 0; q < 2 * NDOT; ++q) v[q] = warp_sum(v[q]);
                    if (lane == 0)
#pragma unroll
                        for (int q = 0; q < 2 * NDOT; ++q) sh.red[q * 16 + warp] = v[q];
                    workers_sync<TC_WORKERS>();
                    if (tid < 2 * NDOT) {
                        double sum = 0.0;
                        for (int w = 0; w < TC_CTRL; ++w) sum += sh.red[tid * 16 + w];
                        a.partials[(int64_t)tid * tiles + tile] = sum;
                        __threadfence();  // before this CTA's finish ticket
                    }
                }
            }
        }
    }
    __syncthreads();
    if (tid == 0) {
        if (sh.abort && a.status) atomicOr(a.status, 16);
        // the last CTA to finish resets the tile counter for the next launch on the stream
        __threadfence();
        sh.last = atomicAdd(a.tile_ctr + 1, 1) == (int)gridDim.x - 1;
        if (sh.last) {
            atomicExch(a.tile_ctr, 0);
            atomicExch(a.tile_ctr + 1, 0);
        }
    }
    __syncthreads();
    if constexpr (NDOT > 0) {
        // the launch's scalar stage of the inner iteration (a.mx_stage), by the last CTA: the
        // per-tile partials summed in tile order, one warp per slot
        if (sh.last && a.mx_stage >= 0) {
            if (warp < 2 * NDOT) {
                double v = 0.0;
                for (int t = lane; t < tiles; t += 32) v += __ldcg(a.partials + (int64_t)warp * tiles + t);
                v = warp_sum(v);
                if (lane == 0) sh.red[warp] = v;
            }
            __syncthreads();
            if (tid == 0) {
                double acc[6] = {0, 0, 0, 0, 0, 0};
                for (int q = 0; q < 2 * NDOT; ++q) acc[q] = sh.red[q];
                mx_stage(acc, a.msc, a.mx_stage);
            }
        }
    }
    if (warp == TC_CTRL) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NCOLS) : "memory");
    }
}

// Kernels by padded mode count KP (the worker thread keeps KP z values in registers).
#define CNM_TC_PLANS(X) X(16) X(32) X(48) X(64) X(80) X(96) X(112)

bool tc_plan(int n_modes, int K, int Nr, int g_stage_bytes, int n_sm, TcPlan &p, int max_gst)
{
    p.kp = (n_modes + 15) / 16 * 16;
    if (p.kp > 112 || K > TC_KMAX) return false;
    p.nt = tc_nt(p.kp);
    p.a_stage = (g_stage_bytes + 127) / 128 * 128;
    const size_t fixed = tc_zregion(p.kp) + (size_t)K * p.nt * 4 + (size_t)p.kp * 12 + (size_t)2 * p.nt * 4 + 128;
    // as many Gaunt stages as fit (2 to 8, at most K: every tile runs gst - 1 multipoles)
    const size_t budget = tc_smem_max(p.kp);
    p.gst = (int)std::min<size_t>(TC_GMAX, budget > fixed ? (budget - fixed) / std::max(p.a_stage, 128) : 0);
    p.gst = std::min(p.gst, K);
    if (max_gst > 0) p.gst = std::min(p.gst, max_gst);
    if (p.gst < TC_MIN_STAGES) return false;
    p.smem = (size_t)p.gst * p.a_stage + fixed;
    // one CTA per SM (KP 112): at least 120 KiB, so that no second CTA shares the SM and no
    // tcgen05.alloc waits for another CTA's columns; two per SM (2 x 2 NT = 256 TMEM columns)
    // never wait either
    if (tc_ctas(p.kp) == 1) p.smem = std::max<size_t>(p.smem, 120 * 1024);
    p.tiles = (Nr + p.nt - 1) / p.nt;
    p.grid = std::min(p.tiles, tc_ctas(p.kp) * n_sm);
    return p.smem <= (size_t)tc_smem_max(p.kp);
}

cudaError_t tc_prepare(const TcPlan &p)
{
    // the kernels' attribute is shared by every handle of the process: set it to the plan
    // limit TC_SMEM_MAX, which every plan's shared memory stays within
    cudaError_t e = cudaSuccess;
#define CNM_TC_ATTR1(KP_, DK_)                                                                                 \
    if (e == cudaSuccess)                                                                                      \
        e = cudaFuncSetAttribute(k_tc_apply<KP_, DK_>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM_MAX);
#define CNM_TC_ATTR(KP_) \
    if (p.kp == KP_) { CNM_TC_ATTR1(KP_, 0) CNM_TC_ATTR1(KP_, 1) CNM_TC_ATTR1(KP_, 23) CNM_TC_ATTR1(KP_, 4) }
    CNM_TC_PLANS(CNM_TC_ATTR)
#undef CNM_TC_ATTR1
#undef CNM_TC_ATTR
    return e;
}

cudaError_t launch_tc_apply(const TcPlan &p, cudaStream_t st, const Grid &g, const int *mode_l, const int *mode_m,
                            int K, const TcTable &tt, const TcArgs &a)
{
    // the launch's reduction set (the combinations the mixed solve uses)
    int dk = -1;
    if (a.n_dots == 0) dk = 0;
    else if (a.n_dots == 1 && a.dot_kind[0] == 1) dk = 1;
    else if (a.n_dots == 2 && a.dot_kind[0] == 2 && a.dot_kind[1] == 3) dk = 23;
    else if (a.n_dots == 1 && a.dot_kind[0] == 4) dk = 4;
    if (dk < 0) return cudaErrorInvalidValue;
#define CNM_TC_LAUNCH1(KP_, DK_)                                                                                  \
    if (dk == DK_) {                                                                                              \
        k_tc_apply<KP_, DK_><<<p.grid, tc_threads(KP_), p.smem, st>>>(g, mode_l, mode_m, K, tt, a, p.tiles,       \
                                                                     p.a_stage, p.gst);                            \
        return cudaGetLastError();                                                                                \
    }
#define CNM_TC_LAUNCH(KP_)                                                                          \
    if (p.kp == KP_) {                                                                              \
        CNM_TC_LAUNCH1(KP_, 0) CNM_TC_LAUNCH1(KP_, 1) CNM_TC_LAUNCH1(KP_, 23) CNM_TC_LAUNCH1(KP_, 4) \
    }
    CNM_TC_PLANS(CNM_TC_LAUNCH)
#undef CNM_TC_LAUNCH
#undef CNM_TC_LAUNCH1
    return cudaErrorInvalidConfiguration;
}

// ==================================================================== fp32 radial solve

struct Aff32 {
    float2 A, B;  // y -> A y + B
};

__device__ __forceinline__ float2 fmul2(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ float2 fadd2(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 fsub2(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ Aff32 aff32_id() { return Aff32{make_float2(1.f, 0.f), make_float2(0.f, 0.f)}; }
// first f, then g
__device__ __forceinline__ Aff32 aff32_then(const Aff32 &f, const Aff32 &g)
{
    return Aff32{fmul2(g.A, f.A), fadd2(fmul2(g.A, f.B), g.B)};
}
__device__ __forceinline__ float2 aff32_apply(const Aff32 &m, float2 y) { return fadd2(fmul2(m.A, y), m.B); }
__device__ __forceinline__ Aff32 shfl_aff32(const Aff32 &a, int src_delta, bool up)
{
    Aff32 r;
    if (up) {
        r.A.x = __shfl_up_sync(0xffffffffu, a.A.x, src_delta);
        r.A.y = __shfl_up_sync(0xffffffffu, a.A.y, src_delta);
        r.B.x = __shfl_up_sync(0xffffffffu, a.B.x, src_delta);
        r.B.y = __shfl_up_sync(0xffffffffu, a.B.y, src_delta);
    } else {
        r.A.x = __shfl_down_sync(0xffffffffu, a.A.x, src_delta);
        r.A.y = __shfl_down_sync(0xffffffffu, a.A.y, src_delta);
        r.B.x = __shfl_down_sync(0xffffffffu, a.B.x, src_delta);
        r.B.y = __shfl_down_sync(0xffffffffu, a.B.y, src_delta);
    }
    return r;
}

// x = P^{-1} rhs for radial block j = blockIdx.y, exactly (forward and backward Thomas
// sweeps as affine-map scans: thread -> warp shuffles -> CTA -> cluster through
// distributed shared memory; the same scheme as the fp64 cluster solve, in fp32).
__global__ void __launch_bounds__(PS32_THREADS) k_psolve32_cl(int Nr, int per, float2 off, const float2 *dinv,
                                                              float2 *x, Ps32Args in)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ float2 ps32[];
    __shared__ Aff32 wagg[PS32_THREADS / 32];
    __shared__ Aff32 wex_s[PS32_THREADS / 32];  // exclusive prefix (forward) / suffix (backward) of wagg
    __shared__ Aff32 cagg_f, cagg_b;
    constexpr int T = PS32_THREADS, NW = PS32_THREADS / 32;
    const int rank = (int)cl.block_rank(), cs = (int)cl.num_blocks();
    const int j = blockIdx.y;
    const int Lc = T * per;
    const int c0 = rank * Lc, c1 = min(Nr, c0 + Lc), len = max(0, c1 - c0);
    float2 *D = ps32, *Y = ps32 + Lc;
    const int64_t base = (int64_t)j * Nr + c0;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (in.mode == 0) {
        for (int e = tid; e < len; e += T) {
            D[e] = dinv[base + e];
            Y[e] = in.b[base + e];
        }
    } else if (in.mode == 2) {
        const float2 be = make_float2((float)in.sc->beta.x, (float)in.sc->beta.y);
        const float2 om = make_float2((float)in.sc->omega.x, (float)in.sc->omega.y);
        for (int e = tid; e < len; e += T) {
            D[e] = dinv[base + e];
            Y[e] = fadd2(in.r[base + e], fmul2(be, fsub2(in.r0[base + e], fmul2(om, in.v[base + e]))));
        }
    } else {
        const float2 al = make_float2((float)in.sc->alpha.x, (float)in.sc->alpha.y);
        for (int e = tid; e < len; e += T) {
            D[e] = dinv[base + e];
            const float2 s = fsub2(in.r[base + e], fmul2(al, in.v[base + e]));
            Y[e] = s;
            in.s_out[base + e] = s;
        }
    }
    __syncthreads();
    const int s0 = tid * per, s1 = min(len, s0 + per);
    // forward: y_i = d_i (b_i - l_i y_{i-1})
    Aff32 acc = aff32_id();
    for (int e = s0; e < s1; ++e) {
        const int i = c0 + e;
        const float2 d = D[e];
        const float2 l = (i >= 1 && i <= Nr - 2) ? off : make_float2(0.f, 0.f);
        const float2 ld = fmul2(l, d);
        acc = aff32_then(acc, Aff32{make_float2(-ld.x, -ld.y), fmul2(d, Y[e])});
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const Aff32 prev = shfl_aff32(acc, o, true);
        if (lane >= o) acc = aff32_then(prev, acc);
    }
    Aff32 excl = shfl_aff32(acc, 1, true);
    if (lane == 0) excl = aff32_id();
    if (lane == 31) wagg[warp] = acc;
    __syncthreads();
    if (warp == 0) {
        // the CTA total, and every warp's exclusive prefix for the apply pass below
        Aff32 cc = lane < NW ? wagg[lane] : aff32_id();
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const Aff32 prev = shfl_aff32(cc, o, true);
            if (lane >= o) cc = aff32_then(prev, cc);
        }
        Aff32 ex = shfl_aff32(cc, 1, true);
        if (lane == 0) ex = aff32_id();
        if (lane < NW) wex_s[lane] = ex;
        if (lane == 31) cagg_f = cc;
    }
    cl.sync();
    float2 ywarp;
    {
        Aff32 cc = lane < rank ? *cl.map_shared_rank(&cagg_f, lane) : aff32_id();
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const Aff32 prev = shfl_aff32(cc, o, true);
            if (lane >= o) cc = aff32_then(prev, cc);
        }
        const float2 ycta = make_float2(__shfl_sync(0xffffffffu, cc.B.x, 31), __shfl_sync(0xffffffffu, cc.B.y, 31));
        ywarp = aff32_apply(wex_s[warp], ycta);
    }
    // forward apply, and with it (ascending) the thread's backward map
    // bcc = f_s0 o ... o f_s1-1, f_e(x) = y_e - u_e d_e x: x_i = y_i - u_i d_i x_{i+1}
    Aff32 bcc = aff32_id();
    {
        float2 y = aff32_apply(excl, ywarp);
        for (int e = s0; e < s1; ++e) {
            const int i = c0 + e;
            const float2 l = (i >= 1 && i <= Nr - 2) ? off : make_float2(0.f, 0.f);
            const float2 d = D[e];
            y = fmul2(d, fsub2(Y[e], fmul2(l, y)));
            Y[e] = y;
            const float2 ud = fmul2(l, d);
            bcc = aff32_then(Aff32{make_float2(-ud.x, -ud.y), y}, bcc);
        }
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const Aff32 nxt = shfl_aff32(bcc, o, false);
        if (lane + o < 32) bcc = aff32_then(nxt, bcc);
    }
    Aff32 bexcl = shfl_aff32(bcc, 1, false);
    if (lane == 31) bexcl = aff32_id();
    __syncthreads();
    if (lane == 0) wagg[warp] = bcc;
    __syncthreads();
    if (warp == 0) {
        // the CTA total, and every warp's exclusive suffix for the apply pass below
        Aff32 cc = lane < NW ? wagg[lane] : aff32_id();
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const Aff32 nxt = shfl_aff32(cc, o, false);
            if (lane + o < 32) cc = aff32_then(nxt, cc);
        }
        Aff32 ex = shfl_aff32(cc, 1, false);
        if (lane == 31) ex = aff32_id();
        if (lane < NW) wex_s[lane] = ex;
        if (lane == 0) cagg_b = cc;
    }
    cl.sync();
    float2 xwarp;
    {
        Aff32 cc = (lane > rank && lane < cs) ? *cl.map_shared_rank(&cagg_b, lane) : aff32_id();
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const Aff32 nxt = shfl_aff32(cc, o, false);
            if (lane + o < 32) cc = aff32_then(nxt, cc);
        }
        const float2 xcta = make_float2(__shfl_sync(0xffffffffu, cc.B.x, 0), __shfl_sync(0xffffffffu, cc.B.y, 0));
        xwarp = aff32_apply(wex_s[warp], xcta);
    }
    // remote reads of cagg_b happen before this arrive; the wait is the last statement
    cl.barrier_arrive();
    {
        float2 xr = aff32_apply(bexcl, xwarp);
        for (int e = s1 - 1; e >= s0; --e) {
            const int i = c0 + e;
            const float2 ud = fmul2((i >= 1 && i <= Nr - 2) ? off : make_float2(0.f, 0.f), D[e]);
            xr = fsub2(Y[e], fmul2(ud, xr));
            Y[e] = xr;
        }
    }
    __syncthreads();
    for (int e = tid; e < len; e += T) x[base + e] = Y[e];
    cl.barrier_wait();
}

// ==================================================================== vector kernels

template <int NV>
__device__ __forceinline__ void partials_out(double (&v)[NV], double *partials)
{
    __shared__ double scr[NV * 32];
    block_sum<NV>(v, scr);
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) partials[(int64_t)q * gridDim.x + blockIdx.x] = v[q];
}

// partials_out, then (f.stage >= 0) the scalar stage by the last block to finish: the
// blocks' partials summed in block order, and the ticket reset for the next launch.
template <int NV>
__device__ __forceinline__ void partials_finish(double (&v)[NV], double *partials, const MxFinish &f)
{
    __shared__ double scr[NV * 32];
    __shared__ double scr6[6 * 32];
    __shared__ int last;
    block_sum<NV>(v, scr);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) partials[(int64_t)q * gridDim.x + blockIdx.x] = v[q];
        last = 0;
        if (f.stage >= 0) {
            __threadfence();
            last = atomicAdd(f.ticket, 1u) == gridDim.x - 1;
        }
    }
    __syncthreads();
    if (!last) return;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
#pragma unroll
        for (int q = 0; q < NV; ++q) acc[q] += __ldcg(partials + (int64_t)q * gridDim.x + b);
    block_sum<6>(acc, scr6);
    if (threadIdx.x == 0) {
        mx_stage(acc, f.sc, f.stage);
        *f.ticket = 0u;
    }
}

// x = psi, r = b - A_full psi = 2 (b - psi) (A_full psi = 2 psi - b by construction of b);
// partials: |r|^2, |b|^2.
__global__ void __launch_bounds__(VEC_THREADS) k_mx_start(int64_t n, const double2 *b, const double2 *psi,
                                                          double2 *x, double2 *r64, float2 *r32, double *partials,
                                                          MxFinish f)
{
    double acc[2] = {0.0, 0.0};
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const double2 bv = b[e], pv = psi[e];
        x[e] = pv;
        const double rr = 2.0 * (bv.x - pv.x), ri = 2.0 * (bv.y - pv.y);
        r64[e] = make_double2(rr, ri);
        r32[e] = make_float2((float)rr, (float)ri);
        acc[0] += rr * rr + ri * ri;
        acc[1] += bv.x * bv.x + bv.y * bv.y;
    }
    partials_finish<2>(acc, partials, f);
}

// r64 = b - A_full x, r32 = r64; with diff set, diff = r64_before - r64_after (the change
// the last correction made, against which its tensor-core image is calibrated); partial
// |r64|^2.
__global__ void __launch_bounds__(VEC_THREADS) k_mx_resid(int64_t n, const double2 *b, const double2 *ax,
                                                          double2 *r64, double2 *diff, float2 *r32, double *partials,
                                                          MxFinish f)
{
    double acc[1] = {0.0};
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const double2 bv = b[e], av = ax[e];
        const double rr = bv.x - av.x, ri = bv.y - av.y;
        if (diff) {
            const double2 old = r64[e];
            diff[e] = make_double2(old.x - rr, old.y - ri);
        }
        r64[e] = make_double2(rr, ri);
        r32[e] = make_float2((float)rr, (float)ri);
        acc[0] += rr * rr + ri * ri;
    }
    partials_finish<1>(acc, partials, f);
}

// The pass's correction d (complex64): d = alpha y + omega z (first iteration) or
// d += alpha y + omega z, formed in fp64 and rounded once; with `apply`, x += d, so x
// receives exactly the complex64 vector a later tensor-core check applies the operator to.
// Partial |d|^2.
__global__ void __launch_bounds__(VEC_THREADS) k_mx_update(int64_t n, const MixScalars *sc, double2 *x,
                                                           const float2 *y, const float2 *z, float2 *d, int first,
                                                           int apply, double *partials, MxFinish f)
{
    const double2 al = sc->alpha, om = sc->omega;
    double acc[1] = {0.0};
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const float2 yv = y[e], zv = z[e];
        double dr = al.x * yv.x - al.y * yv.y + om.x * zv.x - om.y * zv.y;
        double di = al.x * yv.y + al.y * yv.x + om.x * zv.y + om.y * zv.x;
        if (!first) {
            const float2 dv = d[e];
            dr += dv.x;
            di += dv.y;
        }
        const float2 df = make_float2((float)dr, (float)di);
        d[e] = df;
        if (apply) {
            double2 xv = x[e];
            xv.x += (double)df.x;
            xv.y += (double)df.y;
            x[e] = xv;
        }
        acc[0] += (double)df.x * df.x + (double)df.y * df.y;
    }
    partials_finish<1>(acc, partials, f);
}

// Inner residual after an iteration, r1 = s - omega t, and the partial conj(r0) . r1 of the
// next iteration's rho.
__global__ void __launch_bounds__(VEC_THREADS) k_mx_next(int64_t n, const MixScalars *sc, const float2 *s,
                                                         const float2 *t, const float2 *r0, float2 *r1,
                                                         double *partials, MxFinish f)
{
    const double2 om = sc->omega;
    const float2 omf = make_float2((float)om.x, (float)om.y);
    double acc[2] = {0.0, 0.0};
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const float2 sv = s[e], tv = t[e], rv = r0[e];
        const float2 r = make_float2(sv.x - (omf.x * tv.x - omf.y * tv.y), sv.y - (omf.x * tv.y + omf.y * tv.x));
        r1[e] = r;
        acc[0] += (double)rv.x * r.x + (double)rv.y * r.y;
        acc[1] += (double)rv.x * r.y - (double)rv.y * r.x;
    }
    partials_finish<2>(acc, partials, f);
}

// Sum the partials in a fixed order and run one scalar step of the inner iteration.

// One scalar step of the inner iteration from the summed reductions acc (run by the last
// CTA of the launch whose reductions they are).
__device__ void mx_stage(const double *acc, MixScalars *sc, int stage)
{
    switch (stage) {
    case MX_B2R0:
        sc->rr = acc[0];
        sc->r64 = acc[0];
        sc->b2 = acc[1];
        break;
    case MX_R64:
        sc->rr = acc[0];
        sc->r64 = acc[0];
        break;
    case MX_ALPHA: {
        sc->rv = make_double2(acc[0], acc[1]);
        const double2 rv = sc->rv;
        const double den = rv.x * rv.x + rv.y * rv.y;
        // alpha = rr / rv
        sc->alpha = den > 0.0 ? make_double2(sc->rr * rv.x / den, -sc->rr * rv.y / den) : make_double2(0.0, 0.0);
        break;
    }
    case MX_BETA: {  // rho1 = r0 . r1, beta = (rho1 / rho0) (alpha / omega), rho0 = |r0|^2
        const double2 rho1 = make_double2(acc[0], acc[1]);
        sc->rho1 = rho1;
        const double2 al = sc->alpha, om = sc->omega;
        const double omn = om.x * om.x + om.y * om.y;
        // alpha / omega
        const double2 ao = omn > 0.0 ? make_double2((al.x * om.x + al.y * om.y) / omn, (al.y * om.x - al.x * om.y) / omn)
                                     : make_double2(0.0, 0.0);
        const double r0n = sc->rr > 0.0 ? 1.0 / sc->rr : 0.0;
        sc->beta = make_double2(r0n * (rho1.x * ao.x - rho1.y * ao.y), r0n * (rho1.x * ao.y + rho1.y * ao.x));
        break;
    }
    case MX_ALPHA2: {  // alpha = rho1 / (r0 . v)
        sc->rv = make_double2(acc[0], acc[1]);
        const double2 rv = sc->rv, rho = sc->rho1;
        const double den = rv.x * rv.x + rv.y * rv.y;
        sc->alpha = den > 0.0 ? make_double2((rho.x * rv.x + rho.y * rv.y) / den, (rho.y * rv.x - rho.x * rv.y) / den)
                              : make_double2(0.0, 0.0);
        break;
    }
    case MX_OMEGA:
        sc->ts = make_double2(acc[0], acc[1]);
        sc->tt = acc[2];
        sc->omega = acc[2] > 0.0 ? make_double2(acc[0] / acc[2], acc[1] / acc[2]) : make_double2(0.0, 0.0);
        break;
    case MX_D2: sc->d2 = acc[0]; break;
    case MX_TCRES: sc->tc_res2 = acc[0]; break;
    case MX_ECAL:
        sc->e2_cal = acc[0];
        sc->d2_cal = sc->d2;
        break;
    default: break;
    }
}

__global__ void k_to_f64(int64_t n, const float2 *a, double2 *b)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const float2 v = a[e];
        b[e] = make_double2(v.x, v.y);
    }
}

__global__ void k_to_f32(int64_t n, const double2 *a, float2 *b)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const double2 v = a[e];
        b[e] = make_float2((float)v.x, (float)v.y);
    }
}

// dots[s] = v_s^dag x over the support of v_s (fp64 sums, one CTA, fixed order: the
// (sink, mode, node) terms are dealt to the threads, then a fixed block reduction).
__global__ void k_sink_dots32(const float2 *x, int Nr, int n_modes, int n_sinks, const double2 *v0,
                              const double2 *v1, int lo0, int hi0, int lo1, int hi1, double2 *dots)
{
    __shared__ double scr[4 * 32];
    const int n0 = n_sinks > 0 ? max(0, hi0 - lo0) : 0, n1 = n_sinks > 1 ? max(0, hi1 - lo1) : 0;
    const int64_t tot0 = (int64_t)n0 * n_modes, tot = tot0 + (int64_t)n1 * n_modes;
    double acc[4] = {0, 0, 0, 0};
    for (int64_t e = threadIdx.x; e < tot; e += blockDim.x) {
        const bool first = e < tot0;
        const int64_t f = first ? e : e - tot0;
        const int w = first ? n0 : n1;
        const int j = (int)(f / w), i = (first ? lo0 : lo1) + (int)(f - (int64_t)j * w);
        const int64_t q = (int64_t)j * Nr + i;
        const double2 v = (first ? v0 : v1)[q];
        const float2 xv = x[q];
        const double dr = v.x * xv.x + v.y * xv.y, di = v.x * xv.y - v.y * xv.x;
        if (first) {
            acc[0] += dr;
            acc[1] += di;
        } else {
            acc[2] += dr;
            acc[3] += di;
        }
    }
    block_sum<4>(acc, scr);
    if (threadIdx.x == 0) {
        dots[0] = make_double2(acc[0], acc[1]);
        dots[1] = make_double2(acc[2], acc[3]);
    }
}

// Woodbury correction of a preconditioner output (src/CrankNicolsonModes_matrices.cpp:146-153)
// in the inner iterations: c = G^{-1} proj (proj = v^dag y, G^{-1} and v_a^dag W_b from the
// step's fp64 set-up), y -= sum_a W_a c_a on the band [lo, hi) where the W_a live, and
// dots_out = v^dag y of the corrected y = proj - (v^dag W) c.
__global__ void k_wood32(int Nr, int n_modes, int lo, int hi, const Krylov *kr, const double2 *proj,
                         const double2 *W0, const double2 *W1, float2 *y, double2 *dots_out)
{
    const int k = kr->n_sinks;
    double2 c[2] = {make_double2(0, 0), make_double2(0, 0)};
    for (int a = 0; a < k; ++a)
        for (int b = 0; b < k; ++b) c[a] = cadd(c[a], cmul(kr->Gi[a][b], proj[b]));
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        for (int a = 0; a < 2; ++a) {
            double2 d = a < k ? proj[a] : make_double2(0, 0);
            for (int b = 0; b < k && a < k; ++b) d = csub(d, cmul(kr->vW[a][b], c[b]));
            dots_out[a] = d;
        }
    }
    const int w = hi - lo;
    const int64_t n = (int64_t)w * n_modes;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int j = (int)(e / w), i = lo + (int)(e % w);
        const int64_t q = (int64_t)j * Nr + i;
        double2 corr = cmul(W0[q], c[0]);
        if (k > 1) corr = cadd(corr, cmul(W1[q], c[1]));
        const float2 yv = y[q];
        y[q] = make_float2((float)((double)yv.x - corr.x), (float)((double)yv.y - corr.y));
    }
}

}  // namespace cnm

// cnm_apply5.cuh -- compile-time layout of the specialised operator kernel (l_max <= 8).
//
// Modes are ordered by degree l (l + 1 modes per degree, m = -l, -l+2, ..., l), as the
// reference's build_modes does.  The rows are cut into G contiguous groups of about
// equal cost; group gr's Gaunt weights are stored as
//     [column degree l1][column c = 0..l1][row j of the group][s = 0..stride)
// with stride = S rounded up to even, S = min(l_j, l1) + 1 the terms l* = |l_j - l1| + 2s
// (zero where a pair has no term at that l*).  The same formulas serve the kernel
// (template constants) and the host (table builder).
#pragma once

#include <cstddef>
#include <vector>

#include <cuda_runtime.h>

#include "cnm_common.cuh"
#include "cnm_kernels.cuh"
#include "cnm_coupling.h"

namespace cnm {

namespace a5f {
__host__ __device__ constexpr int nm(int L) { return (L + 1) * (L + 2) / 2; }
__host__ __device__ constexpr int loff(int l) { return l * (l + 1) / 2; }
__host__ __device__ constexpr int l_of(int j)
{
    int l = 0;
    while ((l + 1) * (l + 2) / 2 <= j) ++l;
    return l;
}
__host__ __device__ constexpr int m_of(int k) { return -l_of(k) + 2 * (k - loff(l_of(k))); }
__host__ __device__ constexpr int spad(int l, int l1) { return (l < l1 ? l : l1) + 1; }
__host__ __device__ constexpr int stride(int l, int l1) { return (spad(l, l1) + 1) & ~1; }
__host__ __device__ constexpr int row_cost(int l, int L)
{
    int c = 0;
    for (int l1 = 0; l1 <= L; ++l1) c += (l1 + 1) * (spad(l, l1) + 2);
    return c;
}
__host__ __device__ constexpr int first(int L, int G, int g)
{
    if (g <= 0) return 0;
    if (g >= G) return nm(L);
    // rows come in degree blocks of l + 1 rows of equal cost
    long total = 0;
    for (int l = 0; l <= L; ++l) total += (long)(l + 1) * row_cost(l, L);
    const long target = total * g / G;
    long cum = 0;
    int j = 0;
    for (int l = 0; l <= L; ++l) {
        const long c = row_cost(l, L);
        for (int r = 0; r <= l; ++r, ++j) {
            if (cum >= target) return j;
            cum += c;
        }
    }
    return nm(L);
}
__host__ __device__ constexpr int colsize(int L, int G, int g, int l1)
{
    int s = 0;
    const int j0 = first(L, G, g), j1 = first(L, G, g + 1);
    for (int j = j0; j < j1; ++j) s += stride(l_of(j), l1);
    return s;
}
__host__ __device__ constexpr int colbase(int L, int G, int g, int l1)
{
    int b = 0;
    for (int q = 0; q < l1; ++q) b += (q + 1) * colsize(L, G, g, q);
    return b;
}
__host__ __device__ constexpr int gsize(int L, int G, int g) { return colbase(L, G, g, L + 1); }
__host__ __device__ constexpr int gbase(int L, int G, int g)
{
    int b = 0;
    for (int q = 0; q < g; ++q) b += gsize(L, G, q);
    return b;
}
__host__ __device__ constexpr int rowoff(int L, int G, int g, int l1, int j)
{
    int o = 0;
    const int q0 = first(L, G, g);
    for (int q = q0; q < j; ++q) o += stride(l_of(q), l1);
    return o;
}
}  // namespace a5f

// Row groups per degree: the groups multiply the CTAs of a grid (one node per thread)
// and divide the accumulators each thread keeps; at l_max 7-8 seven groups keep about
// six rows per thread, so a thread needs few enough registers for 32 warps per SM and a
// 20000-node grid fills one wave.
template <int L>
struct A5Groups {
    static constexpr int value = L <= 2 ? 1 : (L <= 4 ? 2 : (L <= 6 ? 4 : 9));
};
// The diagnostics pass keeps a second accumulator per row, so it takes fewer groups.
template <int L>
struct D5Groups {
    static constexpr int value = L <= 2 ? 1 : (L <= 4 ? 2 : (L <= 6 ? 4 : 7));
};

template <int L, int G>
struct A5Layout {
    static __host__ __device__ constexpr int nm() { return a5f::nm(L); }
    static __host__ __device__ constexpr int loff(int l) { return a5f::loff(l); }
    static __host__ __device__ constexpr int l_of(int j) { return a5f::l_of(j); }
    static __host__ __device__ constexpr int m_of(int k) { return a5f::m_of(k); }
    static __host__ __device__ constexpr int spad(int l, int l1) { return a5f::spad(l, l1); }
    static __host__ __device__ constexpr int first(int g) { return a5f::first(L, G, g); }
    static __host__ __device__ constexpr int nrows(int g) { return first(g + 1) - first(g); }
    static __host__ __device__ constexpr int colsize(int g, int l1) { return a5f::colsize(L, G, g, l1); }
    static __host__ __device__ constexpr int colbase(int g, int l1) { return a5f::colbase(L, G, g, l1); }
    static __host__ __device__ constexpr int gsize(int g) { return a5f::gsize(L, G, g); }
    static __host__ __device__ constexpr int gbase(int g) { return a5f::gbase(L, G, g); }
    static __host__ __device__ constexpr int rowoff(int g, int l1, int j) { return a5f::rowoff(L, G, g, l1, j); }
    static __host__ __device__ constexpr int gsize_max()
    {
        int m = 0;
        for (int g = 0; g < G; ++g) m = gsize(g) > m ? gsize(g) : m;
        return m;
    }
};

// The same layout with run-time degree and group count (host table builder).
struct A5Host {
    int L, G;
    A5Host(int L_, int G_) : L(L_), G(G_) {}
    int first(int g) const { return a5f::first(L, G, g); }
    int l_of(int j) const { return a5f::l_of(j); }
    int spad(int l, int l1) const { return a5f::spad(l, l1); }
    int colsize(int g, int l1) const { return a5f::colsize(L, G, g, l1); }
    int colbase(int g, int l1) const { return a5f::colbase(L, G, g, l1); }
    int gbase(int g) const { return a5f::gbase(L, G, g); }
    int rowoff(int g, int l1, int j) const { return a5f::rowoff(L, G, g, l1, j); }
};

// Host side of the specialised kernels (0 groups: l_max not specialised).
int apply5_groups(int l_max);
size_t apply5_smem(int l_max);
unsigned apply5_blocks(int l_max, int Nr);
unsigned diag5_blocks(int l_max, int Nr);  // the diagnostics pass over every node (an upper bound)
int diag5_groups(int l_max);
// the weight table of a layout with G row groups (apply5_groups or diag5_groups)
std::vector<double> apply5_table(int l_max, int G, const Coupling &c);
cudaError_t set_apply5_smem();
void launch_apply5(int l_max, cudaStream_t st, const Grid &g, const double *gtab, const ApplyArgs &a);
size_t diag5_smem(int l_max);
cudaError_t set_diag5_smem();
// launches the diagnostics pass and returns its number of CTAs (the partials' stride)
unsigned launch_diag5(int l_max, cudaStream_t st, const Grid &g, const double *gtab, const DiagArgs &d);

}  // namespace cnm

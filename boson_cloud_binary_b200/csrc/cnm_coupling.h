// cnm_coupling.h -- host-side Gaunt coupling cache and special functions.
#pragma once

#include <vector>

namespace cnm {

// Wigner 3j symbol for integer angular momenta (the reference calls
// gsl_sf_coupling_3j with doubled arguments; these are the plain values).
double wigner3j_int(int j1, int j2, int j3, int m1, int m2, int m3);
// gsl_sf_legendre_sphPlm(l, m, 0): normalised associated Legendre function with the
// Condon-Shortley phase at the equator, 0 <= m <= l.
double sph_plm_equator(int l, int m);
// n-point Gauss-Legendre rule on [0, 1], nodes increasing (gsl_integration_glfixed_point).
void gauss_legendre01(int n, std::vector<double> &x, std::vector<double> &w);

// The coupling cache in the flat layout the kernels read (see cnm_common.cuh).
struct Coupling {
    int n_modes = 0, l_max = 0, mode00 = -1;
    std::vector<int> mode_l, mode_m;
    std::vector<int> pair_row_ptr, pair_col, pair_term_ptr, diag_pair;
    std::vector<int> term_l;
    std::vector<double> term_angular;  // the reference's angular coefficient
    std::vector<double> term_g;        // angular * 4 pi / (2 l* + 1)
    std::vector<double> ang00;         // angular of the pair (j, (0,0)), used by the s-wave sinks
};

Coupling build_coupling(int l_max);

// The coupling cache regrouped for the register-blocked kernels: rows with the same
// l are taken `rb` at a time ("row chunks"); for every chunk and every column
// degree l1 the Gaunt weights of the (l, l1) block are stored densely as
// [column m1][row][s] with l* = |l - l1| + 2 s, s < min(l, l1) + 1 (zero where a
// pair has no term at that l*; the s stride is rounded up to an even count so
// pairs of weights load as one 16-byte word), so the kernel's inner loops have
// compile-time trip counts.  The l + 1 rows of a degree are split into chunks of
// near-equal size, at most rb each, so no chunk carries empty rows.
struct BlockedCoupling {
    int rb = 4;                    // most rows per chunk
    int n_chunks = 0;
    std::vector<int> chunk_l;      // [n_chunks]
    std::vector<int> chunk_nrows;  // [n_chunks] rows in the chunk (1..rb)
    std::vector<int> chunk_rows;   // [n_chunks * rb], -1 pads
    std::vector<int> chunk_goff;   // [n_chunks * (l_max + 1)] offset of block (chunk, l1) in g
    std::vector<int> l_off;        // [l_max + 2] first mode index of each l
    std::vector<double> g;
};

BlockedCoupling block_coupling(const Coupling &c, int rb);

// Work plan of the operator kernel: the rows are cut into chunks of one or two rows
// of one degree l (two only where the pair costs at most the mean warp load), and
// the chunks are dealt to n_groups x warps warp lists, longest first, each to the
// least loaded list.  CTA (tile, group) runs the `warps` lists of its group, one per
// warp.  Chunks are stored list by list, so list b is the chunk range
// [list_ptr[b], list_ptr[b + 1]) and the Gaunt weights of group y are the contiguous
// range [group_goff[y], group_goff[y + 1]) of g, which the kernel stages in shared
// memory where it fits.  Costs follow the kernel's inner loops: a row of degree l
// costs sum_l1 (l1 + 1) (min(l, l1) + 3).
struct CouplingPlan {
    BlockedCoupling blocks;     // rb = 2, chunks in list order
    int n_groups = 1, warps = 8;
    std::vector<int> list_ptr;  // [n_groups * warps + 1]
    std::vector<int> group_goff;  // [n_groups + 1]
    double max_list_cost = 0, total_cost = 0;
    int max_group_g = 0;        // doubles of the largest group's weights
};

CouplingPlan plan_coupling(const Coupling &c, int n_groups, int warps);

}  // namespace cnm

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

}  // namespace cnm

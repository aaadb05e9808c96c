// cnm_coupling.cpp -- host-side special functions and the Gaunt coupling cache.
//
// Builds, once per l_max, the coupling cache of the reference
// (src/CrankNicolsonModes_hamiltonian.cpp:68-104): for every ordered mode pair
// (j, k) in row-major order the multipoles l* = |l-l1| .. l+l1 with
//   angular = (-1)^m1 sqrt((2l+1)(2l1+1)(2l*+1)/4pi) (l* l1 l; 0 0 0) (l* l1 l; -m* m1 -m) Y_{l*,|m*|}(pi/2)
// (sign of Y flipped for odd negative m*).  The reference evaluates the symbols
// with GSL; here they come from Racah's formula in extended precision.
#include "cnm_coupling.h"

#include <algorithm>
#include <cmath>
#include <stdexcept>

namespace cnm {

namespace {

long double lfact(int n)
{
    static std::vector<long double> t;
    if (t.empty()) {
        t.resize(400);
        t[0] = 1.0L;
        for (int k = 1; k < 400; ++k) t[k] = t[k - 1] * k;
    }
    if (n < 0 || n >= 400) throw std::invalid_argument("factorial out of range");
    return t[n];
}

}  // namespace

double wigner3j_int(int j1, int j2, int j3, int m1, int m2, int m3)
{
    if (m1 + m2 + m3 != 0) return 0.0;
    if (std::abs(m1) > j1 || std::abs(m2) > j2 || std::abs(m3) > j3) return 0.0;
    if (j3 < std::abs(j1 - j2) || j3 > j1 + j2) return 0.0;
    if (m1 == 0 && m2 == 0 && ((j1 + j2 + j3) & 1)) return 0.0;
    const int kmin = std::max({0, j2 - j3 - m1, j1 - j3 + m2});
    const int kmax = std::min({j1 + j2 - j3, j1 - m1, j2 + m2});
    // Sum the alternating series from its largest terms outwards with a
    // compensated (Kahan) accumulator.
    long double sum = 0.0L, comp = 0.0L, largest = 0.0L;
    for (int k = kmin; k <= kmax; ++k) {
        const long double den = lfact(k) * lfact(j3 - j2 + k + m1) * lfact(j3 - j1 + k - m2) *
                                lfact(j1 + j2 - j3 - k) * lfact(j1 - k - m1) * lfact(j2 - k + m2);
        const long double term = ((k & 1) ? -1.0L : 1.0L) / den;
        largest = std::max(largest, std::fabs(term));
        const long double y = term - comp;
        const long double t = sum + y;
        comp = (t - sum) - y;
        sum = t;
    }
    if (std::fabs(sum) <= 1e-17L * largest) return 0.0;  // exact (accidental) zero
    const long double tri = lfact(j1 + j2 - j3) * lfact(j1 - j2 + j3) * lfact(-j1 + j2 + j3) / lfact(j1 + j2 + j3 + 1);
    const long double pre = std::sqrt(tri * lfact(j1 + m1) * lfact(j1 - m1) * lfact(j2 + m2) * lfact(j2 - m2) *
                                      lfact(j3 + m3) * lfact(j3 - m3));
    const int phase = j1 - j2 - m3;
    return (double)(((phase & 1) ? -1.0L : 1.0L) * pre * sum);
}

double sph_plm_equator(int l, int m)
{
    if (m < 0 || m > l) throw std::invalid_argument("sph_plm_equator: need 0 <= m <= l");
    if ((l + m) & 1) return 0.0;
    // P_l^m(0) = (-1)^((l+m)/2) (l+m-1)!! / (l-m)!!, normalised by sqrt((2l+1)/4pi (l-m)!/(l+m)!).
    long double v = std::sqrt((2.0L * l + 1.0L) / (4.0L * 3.14159265358979323846264338327950288L));
    // multiply in the ratio (l+m-1)!!/(l-m)!! * sqrt((l-m)!/(l+m)!) as one product
    long double ratio = 1.0L;
    for (int k = l + m - 1; k > 1; k -= 2) ratio *= k;
    for (int k = l - m; k > 1; k -= 2) ratio /= k;
    ratio *= std::sqrt(lfact(l - m) / lfact(l + m));
    v *= ratio;
    return (double)((((l + m) / 2) & 1) ? -v : v);
}

void gauss_legendre01(int n, std::vector<double> &x, std::vector<double> &w)
{
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    const long double pi = 3.14159265358979323846264338327950288L;
    for (int k = 0; k < n; ++k) {
        long double z = std::cos(pi * (k + 0.75L) / (n + 0.5L));
        long double dp = 1.0L;
        for (int it = 0; it < 60; ++it) {
            long double p0 = 1.0L, p1 = z;
            for (int j = 2; j <= n; ++j) {
                const long double p2 = ((2 * j - 1) * z * p1 - (j - 1) * p0) / j;
                p0 = p1;
                p1 = p2;
            }
            if (n == 1) p0 = 1.0L;
            dp = n * (z * p1 - p0) / (z * z - 1.0L);
            const long double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-19L) {
                long double q0 = 1.0L, q1 = z;
                for (int j = 2; j <= n; ++j) {
                    const long double q2 = ((2 * j - 1) * z * q1 - (j - 1) * q0) / j;
                    q0 = q1;
                    q1 = q2;
                }
                if (n == 1) q0 = 1.0L;
                dp = n * (z * q1 - q0) / (z * z - 1.0L);
                break;
            }
        }
        const int idx = n - 1 - k;  // increasing order on [0, 1]
        x[idx] = (double)(0.5L * z + 0.5L);
        w[idx] = (double)(0.5L * 2.0L / ((1.0L - z * z) * dp * dp));
    }
}

Coupling build_coupling(int l_max)
{
    Coupling c;
    for (int l = 0; l <= l_max; ++l)
        for (int m = -l; m <= l; ++m)
            if (std::abs(l - m) % 2 == 0) {
                c.mode_l.push_back(l);
                c.mode_m.push_back(m);
            }
    const int n = (int)c.mode_l.size();
    c.n_modes = n;
    c.l_max = l_max;
    c.pair_row_ptr.assign(n + 1, 0);
    c.diag_pair.assign(n, -1);
    c.ang00.assign(n, 0.0);
    c.pair_term_ptr.push_back(0);
    const double four_pi = 4.0 * M_PI;
    int mode00 = -1;
    for (int j = 0; j < n; ++j)
        if (c.mode_l[j] == 0 && c.mode_m[j] == 0) mode00 = j;
    c.mode00 = mode00;
    for (int j = 0; j < n; ++j) {
        for (int k = 0; k < n; ++k) {
            const int l = c.mode_l[j], m = c.mode_m[j], l1 = c.mode_l[k], m1 = c.mode_m[k];
            const int ms = m1 - m;
            int count = 0;
            for (int ls = std::abs(l1 - l); ls <= l1 + l; ++ls) {
                if (std::abs(ms) > ls || (l + l1 + ls) % 2 != 0) continue;
                const double w1 = wigner3j_int(ls, l1, l, 0, 0, 0);
                const double w2 = wigner3j_int(ls, l1, l, -ms, m1, -m);
                double y = sph_plm_equator(ls, std::abs(ms));
                if (ms < 0 && std::abs(ms) % 2 != 0) y = -y;
                const double pref = (m1 % 2 == 0 ? 1.0 : -1.0) *
                                    std::sqrt((2.0 * l + 1) * (2.0 * l1 + 1) * (2.0 * ls + 1) / (4.0 * M_PI));
                const double ang = pref * w1 * w2 * y;
                if (ang == 0.0) continue;
                c.term_l.push_back(ls);
                c.term_angular.push_back(ang);
                c.term_g.push_back(ang * four_pi / (2.0 * ls + 1.0));
                ++count;
                if (k == mode00) c.ang00[j] = ang;
            }
            if (count > 0) {
                if (j == k) c.diag_pair[j] = (int)c.pair_col.size();
                c.pair_col.push_back(k);
                c.pair_term_ptr.push_back((int)c.term_l.size());
            }
        }
        c.pair_row_ptr[j + 1] = (int)c.pair_col.size();
    }
    return c;
}

BlockedCoupling block_coupling(const Coupling &c, int rb)
{
    BlockedCoupling b;
    b.rb = rb;
    const int L = c.l_max;
    b.l_off.assign(L + 2, 0);
    for (int j = 0; j < c.n_modes; ++j) b.l_off[c.mode_l[j] + 1] = j + 1;
    for (int l = 1; l <= L + 1; ++l) b.l_off[l] = std::max(b.l_off[l], b.l_off[l - 1]);
    // term lookup: (j, k, l*) -> g
    std::vector<std::vector<double>> dense(c.n_modes * (size_t)c.n_modes);
    for (int j = 0; j < c.n_modes; ++j)
        for (int p = c.pair_row_ptr[j]; p < c.pair_row_ptr[j + 1]; ++p) {
            std::vector<double> &v = dense[(size_t)j * c.n_modes + c.pair_col[p]];
            v.assign(2 * L + 1, 0.0);
            for (int t = c.pair_term_ptr[p]; t < c.pair_term_ptr[p + 1]; ++t) v[c.term_l[t]] = c.term_g[t];
        }
    // chunks, heaviest first so warps that take chunks round-robin stay balanced
    struct Ch { int l, first, count; double cost; };
    std::vector<Ch> chunks;
    for (int l = 0; l <= L; ++l) {
        const int first = b.l_off[l], count = b.l_off[l + 1] - b.l_off[l];
        const int nch = (count + rb - 1) / rb;
        int r0 = 0;
        for (int c2 = 0; c2 < nch; ++c2) {
            const int size = count / nch + (c2 < count % nch ? 1 : 0);
            double cost = 0;
            for (int l1 = 0; l1 <= L; ++l1) cost += (l1 + 1) * size * (std::min(l, l1) + 3);
            chunks.push_back({l, first + r0, size, cost});
            r0 += size;
        }
    }
    std::stable_sort(chunks.begin(), chunks.end(), [](const Ch &a, const Ch &b2) { return a.cost > b2.cost; });
    b.n_chunks = (int)chunks.size();
    for (const Ch &ch : chunks) {
        b.chunk_l.push_back(ch.l);
        b.chunk_nrows.push_back(ch.count);
        for (int rr = 0; rr < rb; ++rr) b.chunk_rows.push_back(rr < ch.count ? ch.first + rr : -1);
        for (int l1 = 0; l1 <= L; ++l1) {
            b.chunk_goff.push_back((int)b.g.size());
            const int L0 = std::abs(ch.l - l1), S = std::min(ch.l, l1) + 1;
            const int stride = (S + 1) & ~1;
            for (int k = b.l_off[l1]; k < b.l_off[l1 + 1]; ++k)
                for (int rr = 0; rr < ch.count; ++rr)
                    for (int s2 = 0; s2 < stride; ++s2) {
                        double gv = 0.0;
                        const std::vector<double> &v = dense[(size_t)(ch.first + rr) * c.n_modes + k];
                        if (s2 < S && !v.empty()) gv = v[L0 + 2 * s2];
                        b.g.push_back(gv);
                    }
        }
    }
    return b;
}

CouplingPlan plan_coupling(const Coupling &c, int n_groups, int warps)
{
    CouplingPlan pl;
    pl.n_groups = n_groups;
    pl.warps = warps;
    BlockedCoupling &b = pl.blocks;
    b.rb = 2;
    const int L = c.l_max;
    b.l_off.assign(L + 2, 0);
    for (int j = 0; j < c.n_modes; ++j) b.l_off[c.mode_l[j] + 1] = j + 1;
    for (int l = 1; l <= L + 1; ++l) b.l_off[l] = std::max(b.l_off[l], b.l_off[l - 1]);
    std::vector<std::vector<double>> dense(c.n_modes * (size_t)c.n_modes);
    for (int j = 0; j < c.n_modes; ++j)
        for (int p = c.pair_row_ptr[j]; p < c.pair_row_ptr[j + 1]; ++p) {
            std::vector<double> &v = dense[(size_t)j * c.n_modes + c.pair_col[p]];
            v.assign(2 * L + 1, 0.0);
            for (int t = c.pair_term_ptr[p]; t < c.pair_term_ptr[p + 1]; ++t) v[c.term_l[t]] = c.term_g[t];
        }
    std::vector<double> row_cost(L + 1, 0.0);
    for (int l = 0; l <= L; ++l)
        for (int l1 = 0; l1 <= L; ++l1) row_cost[l] += (l1 + 1) * (std::min(l, l1) + 3);
    for (int l = 0; l <= L; ++l) pl.total_cost += (b.l_off[l + 1] - b.l_off[l]) * row_cost[l];
    const int n_lists = n_groups * warps;
    const double target = pl.total_cost / n_lists;
    struct Ch { int l, first, count; double cost; };
    std::vector<Ch> chunks;
    for (int l = 0; l <= L; ++l) {
        const int first = b.l_off[l], count = b.l_off[l + 1] - b.l_off[l];
        const int size = 2 * row_cost[l] <= target ? 2 : 1;
        for (int r0 = 0; r0 < count; r0 += size) {
            const int sz = std::min(size, count - r0);
            chunks.push_back({l, first + r0, sz, sz * row_cost[l]});
        }
    }
    std::stable_sort(chunks.begin(), chunks.end(), [](const Ch &a, const Ch &b2) { return a.cost > b2.cost; });
    std::vector<double> load(n_lists, 0.0);
    std::vector<std::vector<int>> lists(n_lists);
    for (int ci = 0; ci < (int)chunks.size(); ++ci) {
        int best = 0;
        for (int q = 1; q < n_lists; ++q)
            if (load[q] < load[best]) best = q;
        load[best] += chunks[ci].cost;
        lists[best].push_back(ci);
    }
    pl.max_list_cost = *std::max_element(load.begin(), load.end());
    pl.list_ptr.assign(1, 0);
    pl.group_goff.assign(1, 0);
    for (int q = 0; q < n_lists; ++q) {
        for (int ci : lists[q]) {
            const Ch &ch = chunks[ci];
            b.chunk_l.push_back(ch.l);
            b.chunk_nrows.push_back(ch.count);
            for (int rr = 0; rr < 2; ++rr) b.chunk_rows.push_back(rr < ch.count ? ch.first + rr : -1);
            for (int l1 = 0; l1 <= L; ++l1) {
                b.chunk_goff.push_back((int)b.g.size());
                const int L0 = std::abs(ch.l - l1), S = std::min(ch.l, l1) + 1;
                const int stride = (S + 1) & ~1;
                for (int k = b.l_off[l1]; k < b.l_off[l1 + 1]; ++k)
                    for (int rr = 0; rr < ch.count; ++rr)
                        for (int s2 = 0; s2 < stride; ++s2) {
                            double gv = 0.0;
                            const std::vector<double> &v = dense[(size_t)(ch.first + rr) * c.n_modes + k];
                            if (s2 < S && !v.empty()) gv = v[L0 + 2 * s2];
                            b.g.push_back(gv);
                        }
            }
        }
        pl.list_ptr.push_back((int)b.chunk_l.size());
        if ((q + 1) % warps == 0) {
            pl.group_goff.push_back((int)b.g.size());
            const int gsz = pl.group_goff.back() - pl.group_goff[pl.group_goff.size() - 2];
            pl.max_group_g = std::max(pl.max_group_g, gsz);
        }
    }
    b.n_chunks = (int)b.chunk_l.size();
    return pl;
}

}  // namespace cnm

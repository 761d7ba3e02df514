// ORACLE — test infrastructure only (see oracle.hpp). FP64 restatement of the reference's AMR
// refinement (src/amr/refinement.cpp) on hexahedral LGL elements of one order N, dof
// i + np (j + np k):
//  * GradientErrorEstimator::estimate (:44-68) and estimate_element (:70-93): the element's
//    value is (max - min of its nodal values) times its characteristic length
//    h = cbrt(volume) (supplied per element), normalised by the maximum over all elements when
//    that maximum exceeds 1e-14 (and only then are the refine / coarsen flags set:
//    value > refine_threshold, value < coarsen_threshold);
//  * compute_directional_mask (:95-160) with the basis of the solution's own order: per axis
//    the largest (max - min) along the element's node lines of that axis; NONE below 1e-14,
//    else the axes above smoothness_factor x the largest of the three (X = 1, Y = 2, Z = 4,
//    include/mesh/refine_mask.hpp:13);
//  * SolutionProjection::project_to_children (:217-276): each child's nodes mapped into its
//    sub-box of the parent, [-1 + c, c] along a refined axis, and the parent's interpolant
//    evaluated there (interpolate_3d, :345-378: the Lagrange product formula, summed in dof
//    order); children in the order cx fastest, then cy, then cz;
//  * SolutionProjection::project_from_children (:278-343): each parent node takes the child on
//    its side of 0 along every refined axis (0 itself goes to the upper child), mapped into
//    that child's reference coordinates (clamped to [-1, 1]), and interpolates the child there.
// The column-wise remap orc_amr_transfer generalises both to a change of per-column levels
// (k levels up or down per axis, k = 1 being the reference's projections): every new node takes
// the old solution's value at its position, from the old element on its side (a node on a
// cell boundary takes the upper cell, as project_from_children's x >= 0 does).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <vector>

#include "oracle.hpp"

namespace orc {
namespace {

// interpolate_3d: the Lagrange basis by the product formula, then the sum in dof order
double interp3(const Basis1D &b, const double *U, double xi, double eta, double zeta) {
    const int n = b.order + 1;
    std::vector<double> Lx(n), Ly(n), Lz(n);
    for (int i = 0; i < n; ++i) {
        Lx[i] = Ly[i] = Lz[i] = 1.0;
        for (int j = 0; j < n; ++j)
            if (j != i) {
                const double d = b.nodes[i] - b.nodes[j];
                Lx[i] *= (xi - b.nodes[j]) / d;
                Ly[i] *= (eta - b.nodes[j]) / d;
                Lz[i] *= (zeta - b.nodes[j]) / d;
            }
    }
    double r = 0.0;
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) r += U[i + n * (j + n * k)] * Lx[i] * Ly[j] * Lz[k];
    return r;
}

// the parent coordinate of child coordinate x on a refined axis (child c of [-1, 1])
double to_parent(double x, int c) {
    const double lo = -1.0 + c, hi = c;
    return lo + 0.5 * (x + 1.0) * (hi - lo);
}
// the child on the side of parent coordinate x, and x in that child's coordinates
int child_of(double x) { return x >= 0 ? 1 : 0; }
double to_child(double x, int c) {
    const double lo = -1.0 + c, hi = c;
    return std::clamp(2.0 * (x - lo) / (hi - lo) - 1.0, -1.0, 1.0);
}

// element order of a column-wise refined mesh: columns sorted by (lx, ly, lz, column), each
// column's cells sx + nxc (sy + nyc sz)
std::vector<long> column_offsets(int ncol, const int *lv) {
    std::vector<int> ord(ncol);
    std::iota(ord.begin(), ord.end(), 0);
    std::sort(ord.begin(), ord.end(), [&](int a, int b) {
        for (int d = 0; d < 3; ++d)
            if (lv[3 * a + d] != lv[3 * b + d]) return lv[3 * a + d] < lv[3 * b + d];
        return a < b;
    });
    std::vector<long> off(ncol + 1, 0);
    long acc = 0;
    for (int c : ord) {
        off[c] = acc;
        acc += 1L << (lv[3 * c] + lv[3 * c + 1] + lv[3 * c + 2]);
    }
    off[ncol] = acc;
    return off;
}

}  // namespace
}  // namespace orc

using namespace orc;

extern "C" {

// value, mask (RefineMask bits) and flags (1 refine, 2 coarsen) of every element.
int orc_amr_estimate(int order, long n_elem, const double *U, const double *hchar, double refine_threshold,
                     double coarsen_threshold, double smoothness_factor, double *value, int *mask, int *flags) {
    if (order < 1 || n_elem < 0) return -1;
    const int n = order + 1, nd = n * n * n;
    for (long e = 0; e < n_elem; ++e) {
        const double *u = U + e * nd;
        double mx = u[0], mn = u[0];
        for (int q = 1; q < nd; ++q) {
            mx = std::max(mx, u[q]);
            mn = std::min(mn, u[q]);
        }
        value[e] = (mx - mn) * hchar[e];
        double var[3] = {0.0, 0.0, 0.0};
        for (int a = 0; a < n; ++a)
            for (int b = 0; b < n; ++b) {
                // lines along x (j = a, k = b), y (i = a, k = b), z (i = a, j = b)
                const int base[3] = {n * (a + n * b), a + n * n * b, a + n * b};
                const int step[3] = {1, n, n * n};
                for (int d = 0; d < 3; ++d) {
                    double lo = u[base[d]], hi = lo;
                    for (int m = 1; m < n; ++m) {
                        const double v = u[base[d] + step[d] * m];
                        lo = std::min(lo, v);
                        hi = std::max(hi, v);
                    }
                    var[d] = std::max(var[d], hi - lo);
                }
            }
        const double mv = std::max({var[0], var[1], var[2]});
        int m = 0;
        if (mv >= 1e-14) {
            const double thr = smoothness_factor * mv;
            for (int d = 0; d < 3; ++d)
                if (var[d] > thr) m |= 1 << d;
        }
        mask[e] = m;
        flags[e] = 0;
    }
    double vmax = 0.0;
    for (long e = 0; e < n_elem; ++e) vmax = std::max(vmax, value[e]);
    if (vmax > 1e-14)
        for (long e = 0; e < n_elem; ++e) {
            value[e] /= vmax;
            flags[e] = (value[e] > refine_threshold ? 1 : 0) | (value[e] < coarsen_threshold ? 2 : 0);
        }
    return 0;
}

// project_to_children: U_children holds num_children(mask) elements.
int orc_amr_project_children(int order, const double *U_parent, int mask, double *U_children) {
    if (order < 1) return -1;
    const Basis1D b = make_lgl(order);
    const int n = order + 1, nd = n * n * n;
    const int cxn = (mask & 1) ? 2 : 1, cyn = (mask & 2) ? 2 : 1, czn = (mask & 4) ? 2 : 1;
    int child = 0;
    for (int cz = 0; cz < czn; ++cz)
        for (int cy = 0; cy < cyn; ++cy)
            for (int cx = 0; cx < cxn; ++cx, ++child)
                for (int k = 0; k < n; ++k)
                    for (int j = 0; j < n; ++j)
                        for (int i = 0; i < n; ++i) {
                            const double xi = (mask & 1) ? to_parent(b.nodes[i], cx) : b.nodes[i];
                            const double eta = (mask & 2) ? to_parent(b.nodes[j], cy) : b.nodes[j];
                            const double zeta = (mask & 4) ? to_parent(b.nodes[k], cz) : b.nodes[k];
                            U_children[(long)child * nd + i + n * (j + n * k)] = interp3(b, U_parent, xi, eta, zeta);
                        }
    return 0;
}

// project_from_children
int orc_amr_project_parent(int order, const double *U_children, int mask, double *U_parent) {
    if (order < 1) return -1;
    const Basis1D b = make_lgl(order);
    const int n = order + 1, nd = n * n * n;
    const int cxn = (mask & 1) ? 2 : 1, cyn = (mask & 2) ? 2 : 1;
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const int cx = (mask & 1) ? child_of(b.nodes[i]) : 0;
                const int cy = (mask & 2) ? child_of(b.nodes[j]) : 0;
                const int cz = (mask & 4) ? child_of(b.nodes[k]) : 0;
                const int child = cx + cxn * (cy + cyn * cz);
                const double xi = (mask & 1) ? to_child(b.nodes[i], cx) : b.nodes[i];
                const double eta = (mask & 2) ? to_child(b.nodes[j], cy) : b.nodes[j];
                const double zeta = (mask & 4) ? to_child(b.nodes[k], cz) : b.nodes[k];
                U_parent[i + n * (j + n * k)] = interp3(b, U_children + (long)child * nd, xi, eta, zeta);
            }
    return 0;
}

// The solution of a column-wise refined mesh (nx x ny columns, levels old_lv[3 c + d]) carried to
// new levels (new_lv): each new node takes, per axis, the old cell on its side
// (project_to_children on a refined axis, project_from_children on a coarsened one, k levels at
// a time) and the old cell's interpolant at its position.
int orc_amr_transfer(int order, int nx, int ny, const int *old_lv, const int *new_lv, const double *U_old,
                     double *U_new) {
    if (order < 1 || nx < 1 || ny < 1) return -1;
    const int ncol = nx * ny;
    const Basis1D b = make_lgl(order);
    const int n = order + 1, nd = n * n * n;
    const std::vector<long> offo = column_offsets(ncol, old_lv), offn = column_offsets(ncol, new_lv);
    for (int c = 0; c < ncol; ++c) {
        const int *lo = old_lv + 3 * c, *ln = new_lv + 3 * c;
        const int nxn = 1 << ln[0], nyn = 1 << ln[1], nzn = 1 << ln[2];
        const int nxo = 1 << lo[0], nyo = 1 << lo[1];
        for (int sz = 0; sz < nzn; ++sz)
            for (int sy = 0; sy < nyn; ++sy)
                for (int sx = 0; sx < nxn; ++sx) {
                    const long e = offn[c] + sx + (long)nxn * (sy + (long)nyn * sz);
                    const int s[3] = {sx, sy, sz};
                    for (int k = 0; k < n; ++k)
                        for (int j = 0; j < n; ++j)
                            for (int i = 0; i < n; ++i) {
                                const int m[3] = {i, j, k};
                                int so[3];
                                double xo[3];
                                for (int d = 0; d < 3; ++d) {
                                    const double x = b.nodes[m[d]];
                                    if (ln[d] == lo[d]) {
                                        so[d] = s[d];
                                        xo[d] = x;
                                    } else if (ln[d] > lo[d]) {
                                        // refined k levels: sub-cell r of old cell s >> k
                                        // (k = 1: to_parent, child r)
                                        const int k = ln[d] - lo[d], r = s[d] & ((1 << k) - 1);
                                        const double cl = -1.0 + 2.0 * r / (1 << k), chh = cl + 2.0 / (1 << k);
                                        so[d] = s[d] >> k;
                                        xo[d] = cl + 0.5 * (x + 1.0) * (chh - cl);
                                    } else {
                                        // coarsened k levels: the old cell on the node's side
                                        // (k = 1: child_of and to_child)
                                        const int k = lo[d] - ln[d];
                                        const int ch = k == 1 ? child_of(x)
                                                              : std::min((1 << k) - 1, (int)std::floor((x + 1.0) * (1 << (k - 1))));
                                        const double cl = -1.0 + 2.0 * ch / (1 << k), chh = cl + 2.0 / (1 << k);
                                        so[d] = (s[d] << k) + ch;
                                        xo[d] = std::clamp(2.0 * (x - cl) / (chh - cl) - 1.0, -1.0, 1.0);
                                    }
                                }
                                const long eo = offo[c] + so[0] + (long)nxo * (so[1] + (long)nyo * so[2]);
                                U_new[e * nd + i + n * (j + n * k)] = interp3(b, U_old + eo * nd, xo[0], xo[1], xo[2]);
                            }
                }
    }
    return 0;
}

}  // extern "C"

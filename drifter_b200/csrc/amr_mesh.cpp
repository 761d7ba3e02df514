// Face connections of a column-wise directionally refined hexahedral mesh (host C++).
//
// The producer of the tables the AMR right-hand side consumes: the reference builds them per
// element and face with OctreeAdapter::build_face_connections (src/mesh/octree_adapter.cpp:369),
// typed by get_connection_type (include/dg/face_connection.hpp:110) as SameLevel, Fine2x1,
// Fine1x2, Fine2x2 or Boundary. Here the mesh is a base grid of nx x ny columns; column c
// (= ix + nx iy) is split into 2^lx x 2^ly x 2^lz cells (directional levels per column, 2:1
// balanced between neighbouring columns). The output is the face list itself:
//  * elements grouped by level tuple (columns sorted by (lx, ly, lz, c)), each column's cells
//    numbered sx + nxc (sy + nyc sz); per element its levels and its box;
//  * conforming pairs (e1, f1, e2, f2) and boundary faces (e, f), in column order: the faces
//    inside a column, its bed, surface and basin sides, then its faces with the next column in
//    x and in y;
//  * non-conforming interfaces (type, coarse element and face, fine elements and faces in the
//    sub-face order of MortarSpace::compute_subface_bounds, src/dg/mortar.cpp:27), grouped by
//    type (stable).
// Face f has its normal along axis f / 2, positive when f is odd.
// The refinement of these meshes (new levels per column from the error indicators, with the
// same 2:1 balance) is drf_amr_refine_levels, below the builder.
#include <algorithm>
#include <array>
#include <cstdint>
#include <numeric>
#include <vector>

#include "amr_layout.hpp"
#include "common.cuh"

namespace {

struct Iface {
    int type;
    int64_t ce;
    int cf;
    std::array<int64_t, 4> fe;
    std::array<int, 4> ff;
};

// MortarSpace connection types (include/dg/face_connection.hpp:15): Fine2x1 = 1 (two halves
// along the first tangent), Fine1x2 = 2 (along the second), Fine2x2 = 5; 0 = SameLevel
int fine_type(int d1, int d2) { return d1 == 0 && d2 == 0 ? 0 : (d1 == 1 && d2 == 0 ? 1 : (d1 == 0 ? 2 : 5)); }

struct Mesh {
    int nx = 0, ny = 0;
    std::vector<std::array<int, 3>> lv;
    std::vector<int64_t> off;
    int64_t n_elem = 0;
    std::vector<std::array<int, 3>> elevel;
    std::vector<std::array<double, 6>> ebox;
    std::vector<std::array<int64_t, 4>> conf;
    std::vector<std::array<int64_t, 2>> bnd;
    std::vector<Iface> ifs;

    int64_t eid(int c, int sx, int sy, int sz) const {
        const int nxc = 1 << lv[c][0], nyc = 1 << lv[c][1];
        return off[c] + sx + (int64_t)nxc * (sy + (int64_t)nyc * sz);
    }

    void build(int nx_, int ny_, const int *lx, const int *ly, const int *lz, double L) {
        nx = nx_;
        ny = ny_;
        const int ncol = nx * ny;
        lv.resize(ncol);
        for (int c = 0; c < ncol; ++c) {
            lv[c] = {lx[c], ly[c], lz[c]};
            for (int d = 0; d < 3; ++d)
                DRF_CHECK(lv[c][d] >= 0 && lv[c][d] <= 10, DRF_E_INVALID, "refinement level out of range (0..10)");
        }
        static_assert(sizeof(std::array<int, 3>) == 3 * sizeof(int), "levels must be packed");
        off = drf::amr_column_offsets(ncol, reinterpret_cast<const int *>(lv.data()));
        n_elem = off[ncol];
        off.resize(ncol);
        elevel.assign(n_elem, {0, 0, 0});
        ebox.assign(n_elem, {0, 0, 0, 0, 0, 0});
        const double dxb = L / nx;
        for (int c = 0; c < ncol; ++c) {
            const int ix = c % nx, iy = c / nx;
            const int nxc = 1 << lv[c][0], nyc = 1 << lv[c][1], nzc = 1 << lv[c][2];
            for (int sz = 0; sz < nzc; ++sz)
                for (int sy = 0; sy < nyc; ++sy)
                    for (int sx = 0; sx < nxc; ++sx) {
                        const int64_t e = eid(c, sx, sy, sz);
                        elevel[e] = lv[c];
                        ebox[e] = {(ix + (double)sx / nxc) * dxb, (iy + (double)sy / nyc) * dxb, (double)sz / nzc,
                                   (ix + (double)(sx + 1) / nxc) * dxb, (iy + (double)(sy + 1) / nyc) * dxb,
                                   (double)(sz + 1) / nzc};
                        if (sx + 1 < nxc) conf.push_back({e, 1, eid(c, sx + 1, sy, sz), 0});
                        if (sy + 1 < nyc) conf.push_back({e, 3, eid(c, sx, sy + 1, sz), 2});
                        if (sz + 1 < nzc) conf.push_back({e, 5, eid(c, sx, sy, sz + 1), 4});
                        if (sz == 0) bnd.push_back({e, 4});
                        if (sz == nzc - 1) bnd.push_back({e, 5});
                        if (sx == 0 && ix == 0) bnd.push_back({e, 0});
                        if (sx == nxc - 1 && ix == nx - 1) bnd.push_back({e, 1});
                        if (sy == 0 && iy == 0) bnd.push_back({e, 2});
                        if (sy == nyc - 1 && iy == ny - 1) bnd.push_back({e, 3});
                    }
            // faces with the next column in x (normal axis 0, tangents y, z) and in y (axis 1: x, z)
            for (int axis = 0; axis < 2; ++axis) {
                const int nbc = axis == 0 ? (ix + 1 < nx ? c + 1 : -1) : (iy + 1 < ny ? c + nx : -1);
                if (nbc < 0) continue;
                const int t1 = axis == 0 ? 1 : 0;
                const int da0 = lv[c][t1] - lv[nbc][t1], da1 = lv[c][2] - lv[nbc][2];
                const int fa = 2 * axis + 1, fb = 2 * axis;  // face of this column / of the neighbour
                int coarse, fine, cf, ff, d0, d1;
                if (da0 >= 0 && da1 >= 0) {
                    coarse = nbc; fine = c; cf = fb; ff = fa; d0 = da0; d1 = da1;
                } else {
                    coarse = c; fine = nbc; cf = fa; ff = fb; d0 = -da0; d1 = -da1;
                }
                DRF_CHECK(d0 >= 0 && d0 <= 1 && d1 >= 0 && d1 <= 1, DRF_E_INVALID,
                          "neighbouring columns violate the 2:1 balance");
                const auto &lc = lv[coarse], &lf = lv[fine];
                const int n1c = 1 << lc[t1], nzc_ = 1 << lc[2];
                const bool coarse_is_low = coarse == c;  // the lower column holds the +normal face
                auto cell = [&](int col, const std::array<int, 3> &lvl, int a1, int a2, bool at_max) {
                    const int nxcc = 1 << lvl[0], nycc = 1 << lvl[1];
                    const int s_norm = at_max ? (axis == 0 ? nxcc : nycc) - 1 : 0;
                    return axis == 0 ? eid(col, s_norm, a1, a2) : eid(col, a1, s_norm, a2);
                };
                const int t = fine_type(d0, d1);
                for (int p2 = 0; p2 < nzc_; ++p2)
                    for (int p1 = 0; p1 < n1c; ++p1) {
                        const int64_t ce = cell(coarse, lc, p1, p2, coarse_is_low);
                        Iface r{t, ce, cf, {-1, -1, -1, -1}, {-1, -1, -1, -1}};
                        int nf = 0;
                        for (int b2 = 0; b2 < 1 + d1; ++b2)
                            for (int b1 = 0; b1 < 1 + d0; ++b1) {
                                r.fe[nf] = cell(fine, lf, p1 * (1 + d0) + b1, p2 * (1 + d1) + b2, !coarse_is_low);
                                r.ff[nf] = ff;
                                ++nf;
                            }
                        if (t == 0) conf.push_back({ce, cf, r.fe[0], ff});
                        else ifs.push_back(r);
                    }
            }
        }
        std::stable_sort(ifs.begin(), ifs.end(), [](const Iface &a, const Iface &b) { return a.type < b.type; });
    }
};

}  // namespace

extern "C" {

int drf_amr_build_mesh(int nx, int ny, const int *lx, const int *ly, const int *lz, double L, int64_t *n_elem,
                       int64_t *n_conf, int64_t *n_bnd, int64_t *n_if, int *elem_level, double *elem_box,
                       int64_t *conf, int64_t *bnd, int *if_type, int64_t *if_coarse_elem, int *if_coarse_face,
                       int64_t *if_fine_elem, int *if_fine_face) {
    return drf::guard([&] {
        DRF_CHECK(nx >= 1 && ny >= 1 && lx && ly && lz && n_elem && n_conf && n_bnd && n_if, DRF_E_INVALID,
                  "bad arguments");
        DRF_CHECK(L > 0, DRF_E_INVALID, "basin extent must be positive");
        Mesh m;
        m.build(nx, ny, lx, ly, lz, L);
        *n_elem = m.n_elem;
        *n_conf = (int64_t)m.conf.size();
        *n_bnd = (int64_t)m.bnd.size();
        *n_if = (int64_t)m.ifs.size();
        if (elem_level)
            for (int64_t e = 0; e < m.n_elem; ++e)
                for (int d = 0; d < 3; ++d) elem_level[3 * e + d] = m.elevel[e][d];
        if (elem_box)
            for (int64_t e = 0; e < m.n_elem; ++e)
                for (int d = 0; d < 6; ++d) elem_box[6 * e + d] = m.ebox[e][d];
        if (conf)
            for (size_t i = 0; i < m.conf.size(); ++i)
                for (int d = 0; d < 4; ++d) conf[4 * i + d] = m.conf[i][d];
        if (bnd)
            for (size_t i = 0; i < m.bnd.size(); ++i) {
                bnd[2 * i] = m.bnd[i][0];
                bnd[2 * i + 1] = m.bnd[i][1];
            }
        for (size_t i = 0; i < m.ifs.size(); ++i) {
            const Iface &r = m.ifs[i];
            if (if_type) if_type[i] = r.type;
            if (if_coarse_elem) if_coarse_elem[i] = r.ce;
            if (if_coarse_face) if_coarse_face[i] = r.cf;
            for (int k = 0; k < 4; ++k) {
                if (if_fine_elem) if_fine_elem[4 * i + k] = r.fe[k];
                if (if_fine_face) if_fine_face[4 * i + k] = r.ff[k];
            }
        }
    });
}

// AdaptiveMeshRefinement::mark_elements / refine / coarsen (src/amr/refinement.cpp:488-530) and
// OctreeAdapter::balance (src/mesh/octree_adapter.cpp:138) on column-wise levels. An element is
// marked Refine when its refine flag is set and every level of its column is below max_level
// (can_refine, :597), with its suggested mask or XYZ when that is NONE; Coarsen when its
// coarsen flag is set and some level is above min_level (can_coarsen, :602). Elements share
// their column's levels, so a column is refined along the union of its Refine masks; else,
// when any of its elements is marked Coarsen, its last refinement is undone along every axis
// above min_level (the reference merges all siblings of a marked child). Then the balance
// the builder needs is restored by raising the coarser side, as balance() refines the coarser
// neighbour: across every face between columns the tangential and vertical levels differ by at
// most one, and one side is at least as fine as the other along both (a face split in one
// axis from one side and in the other from the other side has no sub-face order).
int drf_amr_refine_levels(int nx, int ny, const int *lx, const int *ly, const int *lz, int64_t n_elem,
                          const int32_t *mask, const int32_t *flags, int max_level, int min_level, int *new_lx,
                          int *new_ly, int *new_lz, int *changed) {
    return drf::guard([&] {
        DRF_CHECK(nx >= 1 && ny >= 1 && lx && ly && lz && mask && flags && new_lx && new_ly && new_lz && changed,
                  DRF_E_INVALID, "bad arguments");
        DRF_CHECK(min_level >= 0 && max_level >= min_level && max_level <= 10, DRF_E_INVALID,
                  "levels must satisfy 0 <= min_level <= max_level <= 10");
        const int ncol = nx * ny;
        std::vector<int> lv(3 * ncol);
        for (int c = 0; c < ncol; ++c) {
            lv[3 * c] = lx[c];
            lv[3 * c + 1] = ly[c];
            lv[3 * c + 2] = lz[c];
            for (int d = 0; d < 3; ++d)
                DRF_CHECK(lv[3 * c + d] >= 0 && lv[3 * c + d] <= 10, DRF_E_INVALID,
                          "refinement level out of range (0..10)");
        }
        const std::vector<int64_t> off = drf::amr_column_offsets(ncol, lv.data());
        DRF_CHECK(off[ncol] == n_elem, DRF_E_INVALID, "element count does not match the levels");
        std::vector<int> nl(lv);
        for (int c = 0; c < ncol; ++c) {
            const int *l = &lv[3 * c];
            const bool can_refine = l[0] < max_level && l[1] < max_level && l[2] < max_level;
            const bool can_coarsen = l[0] > min_level || l[1] > min_level || l[2] > min_level;
            int rmask = 0;
            bool coarsen = false;
            for (int64_t e = off[c]; e < off[c] + ((int64_t)1 << (l[0] + l[1] + l[2])); ++e) {
                if ((flags[e] & 1) && can_refine) rmask |= mask[e] != 0 ? mask[e] : 7;
                else if ((flags[e] & 2) && can_coarsen) coarsen = true;
            }
            for (int d = 0; d < 3; ++d) {
                if (rmask) nl[3 * c + d] = l[d] + ((rmask >> d) & 1);
                else if (coarsen && l[d] > min_level) nl[3 * c + d] = l[d] - 1;
            }
        }
        // 2:1 balance across the faces between columns (raise the coarser side until stable)
        for (bool moved = true; moved;) {
            moved = false;
            for (int c = 0; c < ncol; ++c) {
                const int ix = c % nx, iy = c / nx;
                const int nb[4] = {ix > 0 ? c - 1 : -1, ix + 1 < nx ? c + 1 : -1, iy > 0 ? c - nx : -1,
                                   iy + 1 < ny ? c + nx : -1};
                for (int s = 0; s < 4; ++s) {
                    if (nb[s] < 0) continue;
                    const int t1 = s < 2 ? 1 : 0;  // the face's horizontal tangent
                    const int ax[2] = {t1, 2};
                    int dif[2];
                    for (int q = 0; q < 2; ++q) dif[q] = nl[3 * nb[s] + ax[q]] - nl[3 * c + ax[q]];
                    // one side finer along one face axis and coarser along the other has no
                    // sub-face split: the column that is coarser along an axis takes the level
                    const bool crossed = (dif[0] > 0 && dif[1] < 0) || (dif[0] < 0 && dif[1] > 0);
                    for (int q = 0; q < 2; ++q) {
                        const int want = dif[q] > 1 ? nl[3 * nb[s] + ax[q]] - 1
                                                    : (crossed && dif[q] > 0 ? nl[3 * nb[s] + ax[q]] : -1);
                        if (want > nl[3 * c + ax[q]]) {
                            nl[3 * c + ax[q]] = want;
                            moved = true;
                        }
                    }
                }
            }
        }
        int nch = 0;
        for (int c = 0; c < ncol; ++c) {
            new_lx[c] = nl[3 * c];
            new_ly[c] = nl[3 * c + 1];
            new_lz[c] = nl[3 * c + 2];
            nch += (nl[3 * c] != lv[3 * c]) || (nl[3 * c + 1] != lv[3 * c + 1]) || (nl[3 * c + 2] != lv[3 * c + 2]);
        }
        *changed = nch;
    });
}

}  // extern "C"

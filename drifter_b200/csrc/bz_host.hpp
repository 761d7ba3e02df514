// Host-side setup of the GPU Bezier smoother: element operators, normalisation, multigrid
// hierarchy. All FP64.
#pragma once
#include <vector>

#include "../../include/drifter_b200.h"

namespace drf {

struct BzLevelHost {
    int n = 0, nd = 0;        // elements and control points per direction
    double K[256];            // element operator (row-major 16x16)
    std::vector<double> rho;  // separable ridge factor per control-point index
    std::vector<double> binv; // 9 element-block inverses, class cx + 3 cy
};

struct BzSetup {
    drf_bz_grid_desc g{};
    double dx = 0, dy = 0;
    double He[256], Be[256];
    double alpha = 0, lam_eps = 0;
    std::vector<double> Bq;           // 16 x 16: W_q B_a(q) for the right-hand side
    std::vector<BzLevelHost> levels;  // [0] coarsest .. back() finest
    std::vector<double> coarse_inv;
    int pre = 1, post = 1;
};

void bz_subdivision_1d(double S[2][16]);
void bz_setup_fine(BzSetup &s, const drf_bz_grid_desc &g);
// Finest-level element operator K = alpha H + lambda B and alpha, without heap allocation.
void bz_fine_operator(const drf_bz_grid_desc &g, double K[256], double *alpha);
void bz_setup_levels(BzSetup &s, int coarsest_n, int pre, int post);

}  // namespace drf

// ORACLE — test infrastructure only (see oracle.hpp). FP64 CPU restatement of the cubic
// Bezier bathymetry smoother on a uniform grid: basis (src/bathymetry/cubic_bezier_basis_2d.cpp),
// thin-plate Hessian (src/bathymetry/cubic_thin_plate_hessian.cpp:131), data-fitting assembly and
// Q = alpha H + lambda (B^T W B + eps I) (src/bathymetry/cg_bezier_smoother_base.cpp:260-405),
// C1 edge constraints (src/bathymetry/cg_cubic_bezier_dof_manager.cpp:319,
// src/bathymetry/cg_cubic_bezier_bathymetry_smoother.cpp:798), CG/PCG and the geometric
// multigrid V-cycle (src/bathymetry/bezier_multigrid_preconditioner.cpp:740).
#pragma once
#include <vector>

namespace orc {

using BVec = std::vector<double>;

struct CSR {
    long n = 0, m = 0;
    std::vector<long> rp;
    std::vector<long> ci;
    BVec v;
    void matvec(const double *x, double *y) const;
    double frob2() const;
};

struct BzGrid {
    int nx = 1, ny = 1;
    double x0 = 0, y0 = 0, Lx = 1, Ly = 1;
    double lambda = 1.0, eps = 1e-4;
    int ngauss_energy = 4, ngauss_data = 4;
};

// Bernstein cubic values / derivatives, dof = i + 4 j (cubic_bezier_basis_2d.cpp:42,259)
void bernstein3(double t, int deriv, double out[4]);
void gauss01(int n, BVec &pts, BVec &wts);  // CGBezierSmootherBase::gauss_legendre_01
void element_hessian(double dx, double dy, int ngauss, double H[256]);
void element_mass(double dx, double dy, int ngauss, double B[256]);
// de Casteljau halves (cubic_bezier_basis_2d.cpp:397): child points = S[c] * parent points
void subdivision_1d(double S[2][16]);

struct BzSystem {
    BzGrid g;
    int nxd = 0, nyd = 0;  // control points per direction (3n + 1)
    long ndof = 0;
    double dx = 0, dy = 0;
    double He[256], Be[256];
    double alpha = 0, dTWd = 0;
    CSR H, BtWB, Q;
    BVec BtWd, b;
    long dof(int ex, int ey, int k) const { return (3L * ex + k % 4) + (long)nxd * (3L * ey + k / 4); }
};
// dgauss: data at the ngauss_data^2 Gauss points of every element, [ey][ex][qj][qi]
void bz_build(BzSystem &S, const BzGrid &g, const double *dgauss);
void bz_constraints(const BzSystem &S, int edge_ngauss, CSR &A);
double bz_objective(const BzSystem &S, const double *x, double parts[2]);

// Multigrid (uniform-grid composite of this build): Bezier subdivision prolongation P,
// restriction P^T, exact Galerkin element matrices per level, separable Galerkin ridge,
// symmetric colored multiplicative Schwarz (colors 0..3 pre, 3..0 post), dense coarse solve.
struct BzLevel {
    int n = 0, nd = 0;  // elements and control points per direction
    double K[256];
    BVec rho;           // 1D ridge factor per control point index (ridge = lambda eps rho_i rho_j)
    BVec binv;          // 9 element-block inverses (class cx + 3 cy), 256 each
};
struct BzMG {
    std::vector<BzLevel> lv;  // lv[0] coarsest
    BVec coarse_inv;          // dense inverse of the coarsest operator
    double lam_eps = 0;
    int pre = 1, post = 1;
};
void bz_mg_setup(const BzSystem &S, BzMG &M, int coarsest_n);
void bz_level_apply(const BzMG &M, int l, const double *x, double *y);
void bz_mg_vcycle(const BzMG &M, const double *r, double *z);
// BezierMultigridPreconditioner::apply with the reference's V-cycle (row-normalised R, same
// colour order before and after the coarse correction), repeated to tol; returns the cycles.
int bz_mg_apply_ref(const BzMG &M, const double *b, double *x, double tol, int max_cycles);
// PCG on Q x = b; precond 0 none, 1 Jacobi, 2 MG V-cycle. Returns iterations.
int bz_pcg(const BzSystem &S, const BzMG *M, int precond, const double *b, double *x, double tol,
           int maxit, double *relres);

}  // namespace orc

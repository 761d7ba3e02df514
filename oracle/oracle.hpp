// ORACLE — test infrastructure only. Nothing in the product library links, calls or
// ships this code. It is an FP64 CPU restatement of the reference algorithms of
// olelindberg/drifter (file:line citations on each function), used by tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker.
//
// Parity status: pinned against the reference's own unit-test assertions
// (basis exactness, flux consistency/symmetry/conservation, mode-split element
// properties, RK convergence orders, Bezier DOF counts and transfer properties);
// the reference itself cannot be compiled here (needs Eigen, Boost, GDAL, MPI),
// so no reference-produced vectors exist. The coupled physical DG step and the
// learned preconditioner have no reference counterpart: "parity unpinned" there,
// this oracle is the judge.
#pragma once
#include <cstdint>
#include <functional>
#include <vector>

namespace orc {

using Vec = std::vector<double>;

// ---------------------------------------------------------------- basis (a1, a2)
// Restates src/dg/basis_hexahedron.cpp:70 (LGL), :14 (GL), :152 (barycentric),
// :190 (derivative matrix), :218 (interpolation matrix).
struct Basis1D {
    int order = 0;
    Vec nodes, weights, bary, D;  // D row-major (np x np): D[i*np+j] = l'_j(x_i)
    Vec S;                        // S[k*np+m] = int_{-1}^{x_k} l_m(x) dx (exact)
    // inverse of the strong-form derivative with the value at x = -1 lifted in:
    // A = D + e_0 e_0^T / w_0, Ainv row-major; a0 = Ainv e_0 / w_0
    Vec Ainv, a0;
    int np() const { return order + 1; }
};
void legendre(int n, double x, double &L, double &dL);
void gauss_legendre(int n, Vec &x, Vec &w);
void gauss_lobatto(int n, Vec &x, Vec &w);
Vec barycentric_weights(const Vec &x);
Vec derivative_matrix(const Vec &x);
Vec interpolation_matrix(const Vec &from, const Vec &to);
Basis1D make_lgl(int order);
Basis1D make_gl(int order);

// Dense Kronecker 3D derivative matrices exactly as the reference builds them
// (src/dg/basis_hexahedron.cpp:321), dof = i + np*(j + np*k).
void build_dense_3d(const Basis1D &b, Vec &Dxi, Vec &Deta, Vec &Dzeta);

// ---------------------------------------------------------------- fluxes (a6)
// include/flux/numerical_flux.hpp:222 (LF), :272 (HLLC), src/flux/numerical_flux.cpp:13 (Roe),
// factory LF speed :165-180. State (h, hu, hv), n = (nx, ny).
enum FluxKind { FLUX_LF = 0, FLUX_HLLC = 1, FLUX_ROE = 2 };
void sw_physical_flux(const double U[3], double nx, double ny, double g, double F[3]);
void sw_flux(int kind, const double UL[3], const double UR[3], double nx, double ny, double g,
             double F[3]);

// ---------------------------------------------------------------- compat mode (a3, a4, a8, a9)
struct CompatParams {
    double g = 9.81, rho0 = 1025.0, alpha = 2e-4, beta = 7.6e-4;
    double nu_h = 1.0, nu_v = 1e-4, kappa_v_T = 1e-5, kappa_v_S = 1e-5;
};
// PrimitiveEquationsSolver::compute_rhs (src/physics/primitive_equations.cpp:428) on nel
// independent elements. in: 6 fields [Hu,Hv,eta,HT,HS,omega] x nel*ndof; h, f: nel*ndof.
// out: 5 fields [dHu,dHv,deta,dHT,dHS] x nel*ndof.
void compat_compute_rhs(int order, int nel, const double *const in[6], const double *h,
                        const double *f, const CompatParams &p, double *const out[5]);
// ModeSplittingSolver::step (src/physics/mode_splitting.cpp:434): state = 12 fields
// [Hu,Hv,eta,HT,HS,H,u,v,T,S,omega,rho] x nel*ndof, updated in place.
void compat_modesplit_step(int order, int nel, double dt, int nsub, double *const st[12],
                           const double *h, const double *f, const CompatParams &p);

// SimulationDriver::step without mode splitting (src/solver/simulation_driver.cpp:108-131):
// pack [Hu, Hv, eta, HT, HS] per element (:199), SSPRK3 (src/solver/time_stepper.cpp:64) over
// compute_rhs (:170: unpack_state + update_derived, PrimitiveEquationsSolver::compute_rhs).
// The element loop runs on nthreads host threads (the reference's inert `omp parallel for`).
// st6 = {Hu, Hv, eta, HT, HS, omega} x nel*ndof, updated in place.
void compat_ssprk3_step(int order, int nel, double dt, double *const st6[6], const double *h,
                        const double *f, const CompatParams &p, int nthreads);

// ---------------------------------------------------------------- physical mode
struct PhysParams {
    int nx = 1, ny = 1, nz = 1, order = 3;
    double Lx = 1.0, Ly = 1.0;
    double g = 9.81, rho0 = 1025.0;
    double nu_h = 1.0, nu_v = 1e-4, kappa_v_T = 1e-5, kappa_v_S = 1e-5;
    double cd = 2.5e-3;
    int flux2d = FLUX_LF;
    int bc[4] = {0, 0, 0, 0};  // W, E, S, N: 0 wall, 1 tidal elevation
    double tide_amp = 0.0, tide_period = 44714.0;
    // linear equation of state rho = rho0 (1 - alpha (T - T0) + beta (S - S0))
    // (include/physics/equation_of_state.hpp:35-40,161); alpha = beta = 0 switches the
    // baroclinic pressure gradient off
    double alpha = 2e-4, beta = 7.6e-4, T0 = 10.0, S0 = 35.0;
    // horizontally uniform reference stratification T_ref(z) = Tref_s + Tref_dz z (S_ref = S0)
    // whose hydrostatic pressure has no horizontal gradient at constant z: the force is formed
    // from the anomaly b - b_ref(z). The default (T0, 0) subtracts nothing.
    double Tref_s = 10.0, Tref_dz = 0.0;
};

struct PhysModel {
    PhysParams p;
    Basis1D b;
    int np = 0, np2 = 0, np3 = 0, ncol = 0;
    long n3 = 0, n2 = 0;
    double dx = 0, dy = 0, dsig = 0;
    Vec h, f, taux, tauy;      // 2D: ncol*np2
    // state
    Vec Q[4];                  // 3D: Hu, Hv, HT, HS
    Vec eta, HU, HV;           // 2D barotropic state (FP64)
    Vec eta_avg;               // 2D, time mean of eta over the last subcycle loop
    double t = 0.0;

    void init(const PhysParams &pp, const double *h2, const double *f2, const double *tx,
              const double *ty);
    void set_state(const double *const q[4], const double *eta2);
    double tide(double time) const;
    // 3D right-hand side with eta frozen, tidal ghost at time tb. omega3 optional out.
    // etab (optional, default etaf): the surface elevation the baroclinic pressure gradient
    // uses (in a mode-split step the stage elevation, advanced with the 3D stages)
    void rhs3d(const Vec *Qin, const Vec &etaf, double tb, Vec *R, Vec *omega3,
               Vec *deta2, const Vec *etab = nullptr) const;
    // 2D barotropic operator Phi + forcing (F may be null).
    void rhs2d(const Vec &e, const Vec &hu, const Vec &hv, const Vec *Fx, const Vec *Fy,
               double time, Vec &ke, Vec &khu, Vec &khv) const;
    void column_integral(const Vec &g3, Vec &out2) const;  // int_{-1}^{0} g dsigma per 2D node
    // buoyancy anomaly b = (rho - rho0) / rho0 at every 3D node and its integral from the node
    // up to the surface, B(sigma) = int_sigma^0 b dsigma' (hydrostatic pressure p' = rho0 g H B)
    void baroclinic_B(const Vec *Qin, const Vec &etaf, Vec &b3, Vec &B3) const;
    void split_step(double dt, int nsub);                  // one baroclinic step
    void rk_step(int scheme, double dt);                   // non-split RK of (Q, eta)
    void diagnostics(double out[10]) const;
};

// LSRK45 coefficients, include/solver/time_stepper.hpp:56-61
extern const double LSRK_A[5], LSRK_B[5], LSRK_C[5];

// Generic RK schemes on a vector, src/solver/time_stepper.cpp:13-240.
enum RKScheme { RK_EULER = 0, RK_MIDPOINT = 1, RK_SSP3 = 2, RK_RK4 = 3, RK_LSRK45 = 4, RK_DOPRI = 5 };
using RHSFn = std::function<void(double, const Vec &, Vec &)>;
void rk_step(int scheme, double t, double dt, Vec &U, const RHSFn &rhs);

}  // namespace orc

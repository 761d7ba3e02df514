/* drifter_b200 — C++20 adapters with the reference's class names and call shapes over the C ABI
 * of libdrifter_b200.so (drifter_b200.h). Header-only; link with -ldrifter_b200.
 *
 * Errors come back as exceptions, as the reference throws them: std::invalid_argument for a bad
 * argument (DRF_E_INVALID), drifter_b200::Error (a std::runtime_error carrying the status code)
 * otherwise. VecX is a small std::vector-backed stand-in for Eigen::VectorXd with the members
 * these adapters use; define DRIFTER_B200_USE_EIGEN before including this header to use
 * Eigen::VectorXd itself.
 *
 * Adapter                              replaces (reference)
 * PrimitiveEquationsSolver             PrimitiveEquationsSolver::compute_rhs
 *                                      (include/physics/primitive_equations.hpp:240)
 * ModeSplittingSolver                  ModeSplittingSolver::initialize/step
 *                                      (include/physics/mode_splitting.hpp:211,241)
 * CoupledOceanModel                    SimulationDriver::initialize/step with mode splitting
 *                                      (include/solver/simulation_driver.hpp:92-127), the coupled
 *                                      model the reference declares
 * shallow_water_flux                   NumericalFluxFactory::shallow_water_* (NumericalFluxFunc,
 *                                      include/flux/numerical_flux.hpp:25), batched
 * CGCubicBezierBathymetrySmoother      CGCubicBezierBathymetrySmoother::solve
 *                                      (include/bathymetry/cg_cubic_bezier_bathymetry_smoother.hpp:214)
 * BezierMultigridPreconditioner        BezierMultigridPreconditioner::setup/apply
 *                                      (include/bathymetry/bezier_multigrid_preconditioner.hpp:240,246)
 *                                      as an ISchurPreconditioner-shaped variable preconditioner
 *                                      (include/bathymetry/schur_preconditioner.hpp:36-46)
 */
#ifndef DRIFTER_B200_HPP
#define DRIFTER_B200_HPP

#include <array>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "drifter_b200.h"

#ifdef DRIFTER_B200_USE_EIGEN
#include <Eigen/Dense>
#endif

namespace drifter_b200 {

using Real = double;
using Index = std::int64_t;

#ifdef DRIFTER_B200_USE_EIGEN
using VecX = Eigen::VectorXd;
#else
class VecX {
public:
    VecX() = default;
    explicit VecX(Index n) : v_(static_cast<size_t>(n), 0.0) {}
    VecX(std::initializer_list<double> l) : v_(l) {}
    static VecX Zero(Index n) { return VecX(n); }
    Index size() const { return static_cast<Index>(v_.size()); }
    void resize(Index n) { v_.assign(static_cast<size_t>(n), 0.0); }
    void setZero() { std::fill(v_.begin(), v_.end(), 0.0); }
    double *data() { return v_.data(); }
    const double *data() const { return v_.data(); }
    double &operator()(Index i) { return v_[static_cast<size_t>(i)]; }
    double operator()(Index i) const { return v_[static_cast<size_t>(i)]; }
    double &operator[](Index i) { return v_[static_cast<size_t>(i)]; }
    double operator[](Index i) const { return v_[static_cast<size_t>(i)]; }
    double dot(const VecX &o) const {
        double s = 0.0;
        for (size_t i = 0; i < v_.size(); ++i) s += v_[i] * o.v_[i];
        return s;
    }
    double squaredNorm() const { return dot(*this); }
    double norm() const { return std::sqrt(squaredNorm()); }

private:
    std::vector<double> v_;
};
#endif

/* ------------------------------------------------------------------------------ errors */
class Error : public std::runtime_error {
public:
    Error(int code, const std::string &msg) : std::runtime_error(msg), code_(code) {}
    int code() const { return code_; }

private:
    int code_;
};

inline void check(int rc) {
    if (rc == DRF_OK) return;
    char buf[1024];
    drf_last_error(buf, sizeof(buf));
    const std::string msg = std::string("drifter_b200: ") + buf;
    if (rc == DRF_E_INVALID) throw std::invalid_argument(msg);
    throw Error(rc, msg);
}

namespace detail {
inline void need(bool ok, const char *what) {
    if (!ok) throw std::invalid_argument(std::string("drifter_b200: ") + what);
}
// concatenates per-element vectors of ndof values into one contiguous array
template <class Get>
std::vector<double> gather(size_t nel, Index ndof, Get get) {
    std::vector<double> out(nel * static_cast<size_t>(ndof));
    for (size_t e = 0; e < nel; ++e) {
        const VecX &v = get(e);
        need(v.size() == ndof, "element vector of the wrong size");
        for (Index i = 0; i < ndof; ++i) out[e * ndof + i] = v(i);
    }
    return out;
}
}  // namespace detail

/* ------------------------------------------------------------------- reference-semantics DG
 * OceanConstants / DiffusivityParams (include/physics/primitive_equations.hpp:41,106) */
struct OceanConstants {
    Real g = 9.81, rho_0 = 1025.0, alpha = 2e-4, beta = 7.6e-4;
    Real nu_h = 1.0, nu_v = 1e-4, kappa_v_T = 1e-5, kappa_v_S = 1e-5;
    std::array<double, 8> packed() const { return {g, rho_0, alpha, beta, nu_h, nu_v, kappa_v_T, kappa_v_S}; }
};

/* PrimitiveState / PrimitiveTendencies (include/physics/primitive_equations.hpp:82), per element,
 * dof = i + (N+1) (j + (N+1) k) */
struct PrimitiveState {
    VecX Hu, Hv, eta, HT, HS, omega;  // prognostic + sigma velocity
    VecX H, u, v, T, S, rho;          // derived (ModeSplittingSolver::step updates them)
};
struct PrimitiveTendencies {
    VecX dHu_dt, dHv_dt, deta_dt, dHT_dt, dHS_dt;
};

/* PrimitiveEquationsSolver::compute_rhs (include/physics/primitive_equations.hpp:240): the
 * element-local tendencies exactly as the reference computes them (its quirks included). */
class PrimitiveEquationsSolver {
public:
    explicit PrimitiveEquationsSolver(int order, const OceanConstants &c = {}) : order_(order), c_(c) {}
    void initialize(const std::vector<VecX> &bathymetry, const std::vector<VecX> &coriolis) {
        detail::need(bathymetry.size() == coriolis.size(), "bathymetry and coriolis sizes differ");
        const Index nd = ndof();
        h_ = detail::gather(bathymetry.size(), nd, [&](size_t e) -> const VecX & { return bathymetry[e]; });
        f_ = detail::gather(coriolis.size(), nd, [&](size_t e) -> const VecX & { return coriolis[e]; });
        nel_ = bathymetry.size();
    }
    void compute_rhs(const std::vector<PrimitiveState> &states, std::vector<PrimitiveTendencies> &tend) const {
        detail::need(states.size() == nel_, "state count differs from the initialised elements");
        const Index nd = ndof();
        std::array<std::vector<double>, 6> in;
        const VecX PrimitiveState::*fields[6] = {&PrimitiveState::Hu, &PrimitiveState::Hv, &PrimitiveState::eta,
                                                  &PrimitiveState::HT, &PrimitiveState::HS, &PrimitiveState::omega};
        for (int k = 0; k < 6; ++k)
            in[k] = detail::gather(nel_, nd, [&](size_t e) -> const VecX & { return states[e].*fields[k]; });
        std::array<std::vector<double>, 5> out;
        for (auto &o : out) o.assign(nel_ * nd, 0.0);
        const double *ip[6];
        double *op[5];
        for (int k = 0; k < 6; ++k) ip[k] = in[k].data();
        for (int k = 0; k < 5; ++k) op[k] = out[k].data();
        const auto p8 = c_.packed();
        check(drf_compat_compute_rhs(order_, static_cast<int>(nel_), ip, h_.data(), f_.data(), p8.data(), op));
        tend.resize(nel_);
        VecX PrimitiveTendencies::*tf[5] = {&PrimitiveTendencies::dHu_dt, &PrimitiveTendencies::dHv_dt,
                                            &PrimitiveTendencies::deta_dt, &PrimitiveTendencies::dHT_dt,
                                            &PrimitiveTendencies::dHS_dt};
        for (size_t e = 0; e < nel_; ++e)
            for (int k = 0; k < 5; ++k) {
                VecX &v = tend[e].*tf[k];
                v.resize(nd);
                for (Index i = 0; i < nd; ++i) v(i) = out[k][e * nd + i];
            }
    }
    Index ndof() const { return static_cast<Index>(order_ + 1) * (order_ + 1) * (order_ + 1); }

private:
    int order_;
    OceanConstants c_;
    std::vector<double> h_, f_;
    size_t nel_ = 0;
};

/* ModeSplittingSolver::step (include/physics/mode_splitting.hpp:241), per element with the
 * reference's semantics (per-element depth integrals, zero baroclinic forcing). */
class ModeSplittingSolver {
public:
    ModeSplittingSolver(int order, const OceanConstants &c = {}, int subcycles = 30)
        : order_(order), c_(c), nsub_(subcycles) {}
    void initialize(const std::vector<VecX> &bathymetry, const std::vector<VecX> &coriolis) {
        detail::need(bathymetry.size() == coriolis.size(), "bathymetry and coriolis sizes differ");
        const Index nd = ndof();
        h_ = detail::gather(bathymetry.size(), nd, [&](size_t e) -> const VecX & { return bathymetry[e]; });
        f_ = detail::gather(coriolis.size(), nd, [&](size_t e) -> const VecX & { return coriolis[e]; });
        nel_ = bathymetry.size();
    }
    void step(Real dt_3d, std::vector<PrimitiveState> &full_state) const {
        detail::need(full_state.size() == nel_, "state count differs from the initialised elements");
        const Index nd = ndof();
        VecX PrimitiveState::*fields[12] = {&PrimitiveState::Hu, &PrimitiveState::Hv, &PrimitiveState::eta,
                                            &PrimitiveState::HT, &PrimitiveState::HS, &PrimitiveState::H,
                                            &PrimitiveState::u, &PrimitiveState::v, &PrimitiveState::T,
                                            &PrimitiveState::S, &PrimitiveState::omega, &PrimitiveState::rho};
        std::array<std::vector<double>, 12> st;
        for (int k = 0; k < 12; ++k)
            st[k] = detail::gather(nel_, nd, [&](size_t e) -> const VecX & { return full_state[e].*fields[k]; });
        double *sp[12];
        for (int k = 0; k < 12; ++k) sp[k] = st[k].data();
        const auto p8 = c_.packed();
        check(drf_compat_modesplit_step(order_, static_cast<int>(nel_), dt_3d, nsub_, sp, h_.data(), f_.data(),
                                        p8.data()));
        for (size_t e = 0; e < nel_; ++e)
            for (int k = 0; k < 12; ++k) {
                VecX &v = full_state[e].*fields[k];
                for (Index i = 0; i < nd; ++i) v(i) = st[k][e * nd + i];
            }
    }
    Index ndof() const { return static_cast<Index>(order_ + 1) * (order_ + 1) * (order_ + 1); }

private:
    int order_;
    OceanConstants c_;
    int nsub_;
    std::vector<double> h_, f_;
    size_t nel_ = 0;
};

/* ------------------------------------------------------------------- coupled DG model
 * The coupled sigma-coordinate model (face fluxes, full-column omega, baroclinic pressure,
 * FP64 barotropic subcycles), one CUDA graph per baroclinic step. Fields are the C ABI's SoA
 * layouts: 3D [column][layer][k][j][i], 2D [column][j][i]. */
class CoupledOceanModel {
public:
    CoupledOceanModel(const drf_mesh_desc &mesh, const drf_dg_params &params, const std::vector<double> &h,
                      const std::vector<double> &f, const std::vector<double> &taux,
                      const std::vector<double> &tauy)
        : mesh_(mesh) {
        detail::need(h.size() == n2() && f.size() == n2() && taux.size() == n2() && tauy.size() == n2(),
                     "2D field of the wrong size");
        check(drf_dg_create(&mesh, &params, h.data(), f.data(), taux.data(), tauy.data(), &m_));
    }
    ~CoupledOceanModel() {
        if (m_) drf_dg_destroy(m_);
    }
    CoupledOceanModel(const CoupledOceanModel &) = delete;
    CoupledOceanModel &operator=(const CoupledOceanModel &) = delete;

    size_t n2() const {
        const size_t np = static_cast<size_t>(mesh_.order) + 1;
        return static_cast<size_t>(mesh_.nx) * mesh_.ny * np * np;
    }
    size_t n3() const { return n2() * mesh_.nz * (static_cast<size_t>(mesh_.order) + 1); }

    void set_state(const std::array<std::vector<double>, 4> &q, const std::vector<double> &eta, Real t = 0.0) {
        for (const auto &a : q) detail::need(a.size() == n3(), "3D field of the wrong size");
        detail::need(eta.size() == n2(), "eta of the wrong size");
        const double *qp[4] = {q[0].data(), q[1].data(), q[2].data(), q[3].data()};
        check(drf_dg_upload_state(m_, qp, eta.data(), t));
    }
    /* ModeSplittingSolver::step on the coupled model: nsteps baroclinic steps of dt_3d */
    void step(Real dt_3d, int nsub, int nsteps = 1) { check(drf_dg_step_modesplit(m_, dt_3d, nsub, nsteps)); }
    Real get_state(std::array<std::vector<double>, 4> &q, std::vector<double> &eta) const {
        for (auto &a : q) a.resize(n3());
        eta.resize(n2());
        double *qp[4] = {q[0].data(), q[1].data(), q[2].data(), q[3].data()};
        double t = 0.0;
        check(drf_dg_download_state(m_, qp, eta.data(), nullptr, nullptr, nullptr, &t));
        return t;
    }
    /* SimulationDriver::compute_diagnostics: mass_weighted, mass_unweighted, energy, heat, salt,
     * max_speed, max_eta, min_eta, max_T, min_T */
    std::array<double, 10> diagnostics() const {
        std::array<double, 10> d{};
        check(drf_dg_diagnostics(m_, d.data()));
        return d;
    }
    drf_dg *handle() { return m_; }

private:
    drf_mesh_desc mesh_;
    drf_dg *m_ = nullptr;
};

/* NumericalFluxFactory::shallow_water_{lax_friedrichs,hllc,roe}: F*(U_L, U_R, n) for n faces at
 * once (U = (h, hu, hv), n x 3; normals n x 2). */
inline std::vector<double> shallow_water_flux(int kind, const std::vector<double> &UL, const std::vector<double> &UR,
                                              const std::vector<double> &normals, double g = 9.81) {
    detail::need(UL.size() == UR.size() && UL.size() % 3 == 0 && normals.size() == UL.size() / 3 * 2,
                 "flux batch of inconsistent sizes");
    std::vector<double> F(UL.size());
    check(drf_sw_flux_batch(kind, static_cast<int64_t>(UL.size() / 3), UL.data(), UR.data(), normals.data(), g,
                            F.data()));
    return F;
}

/* ----------------------------------------------------------------------- Bezier smoother
 * CGCubicBezierSmootherConfig (lambda, ridge_epsilon) on a uniform nx x nx grid; the data are
 * sampled at the 4 x 4 Gauss points of every element ([ey][ex][qj][qi]). */
class CGCubicBezierBathymetrySmoother {
public:
    CGCubicBezierBathymetrySmoother(int nx, int ny, Real x0, Real y0, Real Lx, Real Ly,
                                    const std::vector<double> &gauss_data, Real lambda = 1.0,
                                    Real ridge_epsilon = 1e-4) {
        const drf_bz_grid_desc g{nx, ny, x0, y0, Lx, Ly, lambda, ridge_epsilon};
        detail::need(gauss_data.size() == static_cast<size_t>(nx) * ny * 16, "data must hold 16 samples per element");
        check(drf_bz_create(&g, gauss_data.data(), &h_));
        int64_t nd = 0;
        double alpha = 0.0;
        int nl = 0;
        check(drf_bz_info(h_, &nd, &alpha, &nl));
        ndof_ = nd;
    }
    ~CGCubicBezierBathymetrySmoother() {
        if (h_) drf_bz_destroy(h_);
    }
    CGCubicBezierBathymetrySmoother(const CGCubicBezierBathymetrySmoother &) = delete;
    CGCubicBezierBathymetrySmoother &operator=(const CGCubicBezierBathymetrySmoother &) = delete;

    Index num_dofs() const { return ndof_; }
    /* y = Q x, matrix-free */
    VecX apply_Q(const VecX &x) const {
        detail::need(x.size() == ndof_, "vector of the wrong size");
        VecX y(ndof_);
        check(drf_bz_apply_Q(h_, x.data(), y.data()));
        return y;
    }
    /* CGCubicBezierBathymetrySmoother::solve (C1 edge constraints, Schur CG with inner PCG on Q):
     * the smoothed control points */
    VecX solve(int edge_ngauss = 4, Real tol = 1e-10, int maxit = 5000, int inner_kind = 2) const {
        VecX x(ndof_);
        int it = 0;
        double rel = 0.0, ms = 0.0;
        check(drf_bz_constrained_solve(h_, edge_ngauss, inner_kind, tol, maxit, 1e-12, x.data(), &it, &rel, &ms));
        return x;
    }
    /* PCG on Q x = b (b empty: the assembled right-hand side); kind as drf_pcg_solve */
    VecX solve_Q(const VecX &b, int kind, Real tol = 1e-10, int maxit = 5000, int *iters = nullptr) const {
        VecX x(ndof_);
        int it = 0;
        double rel = 0.0, ms = 0.0;
        check(drf_pcg_solve(h_, b.size() ? b.data() : nullptr, x.data(), tol, maxit, kind, &it, &rel, &ms));
        if (iters) *iters = it;
        return x;
    }
    drf_bz *handle() const { return h_; }

private:
    drf_bz *h_ = nullptr;
    Index ndof_ = 0;
};

/* ISchurPreconditioner (include/bathymetry/schur_preconditioner.hpp:29) shape */
class ISchurPreconditioner {
public:
    virtual ~ISchurPreconditioner() = default;
    virtual VecX apply(const VecX &r) const = 0;
    virtual bool is_variable() const { return false; }
    virtual Index num_constraints() const = 0;
};

/* MultigridConfig (include/bathymetry/bezier_multigrid_preconditioner.hpp:80-130): the fields
 * the GPU hierarchy uses (coarsest level in elements per direction in place of min_tree_level) */
struct MultigridConfig {
    int coarsest_n = 2;
    int pre_smoothing = 1, post_smoothing = 1;
    int max_vcycles = 100;
    Real vcycle_tolerance = 1e-6;
};

/* BezierMultigridPreconditioner::setup/apply on the GPU: apply() returns what the reference's
 * apply returns (V-cycles with the row-normalised restriction to vcycle_tolerance), a variable
 * preconditioner; apply_symmetric() is this build's single SPD cycle for plain PCG. */
class BezierMultigridPreconditioner : public ISchurPreconditioner {
public:
    explicit BezierMultigridPreconditioner(const MultigridConfig &config = {}) : config_(config) {}
    void setup(const CGCubicBezierBathymetrySmoother &smoother) {
        s_ = &smoother;
        check(drf_mg_setup(smoother.handle(), config_.coarsest_n, config_.pre_smoothing, config_.post_smoothing));
        int64_t nd = 0;
        double alpha = 0.0;
        check(drf_bz_info(smoother.handle(), &nd, &alpha, &levels_));
    }
    VecX apply(const VecX &r) const override {
        detail::need(s_ != nullptr, "BezierMultigridPreconditioner::apply: setup() not called");
        detail::need(r.size() == s_->num_dofs(), "vector of the wrong size");
        VecX z(r.size());
        int cycles = 0;
        double rel = 0.0;
        check(drf_mg_apply_reference(s_->handle(), r.data(), z.data(), config_.vcycle_tolerance,
                                     config_.max_vcycles, &cycles, &rel));
        last_cycles_ = cycles;
        return z;
    }
    VecX apply_symmetric(const VecX &r) const {
        detail::need(s_ != nullptr, "BezierMultigridPreconditioner::apply: setup() not called");
        VecX z(r.size());
        check(drf_mg_apply(s_->handle(), r.data(), z.data()));
        return z;
    }
    bool is_variable() const override { return true; }
    Index num_constraints() const override { return s_ ? s_->num_dofs() : 0; }
    int num_levels() const { return levels_; }
    bool is_setup() const { return s_ != nullptr; }
    int last_vcycles() const { return last_cycles_; }
    const MultigridConfig &config() const { return config_; }

private:
    MultigridConfig config_;
    const CGCubicBezierBathymetrySmoother *s_ = nullptr;
    int levels_ = 0;
    mutable int last_cycles_ = 0;
};

}  // namespace drifter_b200

#endif  // DRIFTER_B200_HPP

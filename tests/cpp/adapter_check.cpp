// Exercises the C++ adapters of include/drifter_b200.hpp the way reference code calls the
// classes they replace, and prints a JSON line of results that tests/test_cpp_adapters.py
// compares with the same computations through the Python mirror. Inputs are closed-form.
#include <cmath>
#include <cstdio>
#include <vector>

#include "drifter_b200.hpp"

using namespace drifter_b200;

int main() {
    std::printf("{");
    // PrimitiveEquationsSolver::compute_rhs and ModeSplittingSolver::step, order 3, 3 elements
    {
        const int order = 3, nel = 3, nd = 64;
        std::vector<VecX> h(nel, VecX(nd)), f(nel, VecX(nd));
        std::vector<PrimitiveState> st(nel);
        for (int e = 0; e < nel; ++e) {
            PrimitiveState &s = st[e];
            for (auto *v : {&s.Hu, &s.Hv, &s.eta, &s.HT, &s.HS, &s.omega, &s.H, &s.u, &s.v, &s.T, &s.S, &s.rho})
                v->resize(nd);
            for (int i = 0; i < nd; ++i) {
                const double x = 0.1 * (i + 7 * e);
                h[e](i) = 50.0 + 10.0 * std::sin(x);
                f[e](i) = 1e-4;
                s.eta(i) = 0.01 * std::cos(x);
                const double H = h[e](i) + s.eta(i);
                s.Hu(i) = 0.1 * H * std::sin(2 * x);
                s.Hv(i) = 0.05 * H * std::cos(3 * x);
                s.HT(i) = (10.0 + std::sin(x)) * H;
                s.HS(i) = 35.0 * H;
                s.omega(i) = 1e-5 * std::sin(x);
                // the derived fields (PrimitiveState::update_derived)
                s.H(i) = H;
                s.u(i) = s.Hu(i) / H;
                s.v(i) = s.Hv(i) / H;
                s.T(i) = s.HT(i) / H;
                s.S(i) = s.HS(i) / H;
                s.rho(i) = 1025.0 * (1.0 - 2e-4 * (s.T(i) - 10.0) + 7.6e-4 * (s.S(i) - 35.0));
            }
        }
        PrimitiveEquationsSolver pe(order);
        pe.initialize(h, f);
        std::vector<PrimitiveTendencies> td;
        pe.compute_rhs(st, td);
        double sums[5] = {0, 0, 0, 0, 0};
        for (const auto &t : td)
            for (int i = 0; i < nd; ++i) {
                sums[0] += t.dHu_dt(i); sums[1] += t.dHv_dt(i); sums[2] += t.deta_dt(i);
                sums[3] += t.dHT_dt(i); sums[4] += t.dHS_dt(i);
            }
        std::printf("\"compat_rhs\": [%.17g, %.17g, %.17g, %.17g, %.17g], ", sums[0], sums[1], sums[2], sums[3],
                    sums[4]);
        ModeSplittingSolver ms(order, OceanConstants{}, 10);
        ms.initialize(h, f);
        ms.step(0.01, st);  // reference coordinates (no metric): a stable step is short
        double se = 0.0, su = 0.0;
        for (const auto &s : st)
            for (int i = 0; i < nd; ++i) { se += s.eta(i); su += s.Hu(i); }
        std::printf("\"compat_step\": [%.17g, %.17g], ", se, su);
        // the reference throws std::invalid_argument for nsub = 0
        bool threw = false;
        try {
            ModeSplittingSolver bad(order, OceanConstants{}, 0);
            bad.initialize(h, f);
            bad.step(0.01, st);
        } catch (const std::invalid_argument &) {
            threw = true;
        }
        std::printf("\"invalid_throws\": %s, ", threw ? "true" : "false");
    }
    // CoupledOceanModel: 3 x 2 x 2 hexes, N = 2, 2 baroclinic steps
    {
        drf_mesh_desc mesh{3, 2, 2, 2, 30e3, 20e3};
        drf_dg_params prm{};
        prm.g = 9.81; prm.rho0 = 1025.0; prm.nu_h = 1.0; prm.nu_v = 1e-4; prm.kappa_v_T = 1e-5;
        prm.kappa_v_S = 1e-5; prm.cd = 2.5e-3; prm.flux2d = DRF_FLUX_LF; prm.precision = DRF_PREC_FP64;
        prm.alpha = 2e-4; prm.beta = 7.6e-4; prm.T0 = 10.0; prm.S0 = 35.0; prm.Tref_s = 10.0; prm.Tref_dz = 0.0;
        const size_t n2 = 3 * 2 * 9, n3 = n2 * 2 * 3;
        std::vector<double> h(n2), f(n2, 1e-4), tx(n2, 0.1), ty(n2, 0.0), eta(n2, 0.0);
        for (size_t i = 0; i < n2; ++i) h[i] = 100.0 + 20.0 * std::sin(0.3 * i);
        std::array<std::vector<double>, 4> q;
        for (auto &a : q) a.assign(n3, 0.0);
        for (size_t n = 0; n < n3; ++n) {
            const size_t c = n / (2 * 27), a2 = n % 9;
            const double H = h[c * 9 + a2];
            q[2][n] = (10.0 + 0.5 * std::sin(0.1 * n)) * H;
            q[3][n] = 35.0 * H;
        }
        CoupledOceanModel m(mesh, prm, h, f, tx, ty);
        m.set_state(q, eta);
        m.step(30.0, 5, 2);
        const auto d = m.diagnostics();
        std::printf("\"coupled_diag\": [%.17g, %.17g, %.17g, %.17g, %.17g], ", d[0], d[2], d[3], d[5], d[6]);
    }
    // Bezier smoother (8 x 8) with the multigrid preconditioner
    {
        const int n = 8;
        std::vector<double> data(n * n * 16);
        for (size_t i = 0; i < data.size(); ++i) data[i] = 500.0 + 100.0 * std::sin(0.05 * i);
        CGCubicBezierBathymetrySmoother sm(n, n, 0.0, 0.0, 2000.0, 2000.0, data, 1.0, 1e-4);
        BezierMultigridPreconditioner mg(MultigridConfig{});
        mg.setup(sm);
        VecX r(sm.num_dofs());
        for (Index i = 0; i < r.size(); ++i) r(i) = std::cos(0.01 * i);
        const VecX z = mg.apply(r);
        int iters = 0;
        const VecX x = sm.solve_Q(VecX(), 2, 1e-10, 500, &iters);
        std::printf("\"mg\": [%d, %.17g, %d, %.17g, %d]", mg.last_vcycles(), z.norm(), iters, x.norm(),
                    mg.num_levels());
    }
    std::printf("}\n");
    return 0;
}

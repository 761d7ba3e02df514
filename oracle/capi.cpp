// ORACLE C API (test infrastructure only): flat extern "C" entry points so the pytest
// suite and bench.py's CPU-baseline leg can drive the FP64 restatement through ctypes.
#include <cmath>
#include <cstring>
#include <exception>
#include <string>

#include "bz_oracle.hpp"
#include "oracle.hpp"

using namespace orc;

static thread_local std::string g_err;

#define ORC_TRY(...)                                   \
    try {                                              \
        __VA_ARGS__;                                   \
        return 0;                                      \
    } catch (const std::exception &e) {                \
        g_err = e.what();                              \
        return -1;                                     \
    }

static PhysParams phys_from(const int *iv, const double *dv) {
    PhysParams p;
    p.nx = iv[0]; p.ny = iv[1]; p.nz = iv[2]; p.order = iv[3]; p.flux2d = iv[4];
    for (int s = 0; s < 4; ++s) p.bc[s] = iv[5 + s];
    p.Lx = dv[0]; p.Ly = dv[1]; p.g = dv[2]; p.rho0 = dv[3]; p.nu_h = dv[4]; p.nu_v = dv[5];
    p.kappa_v_T = dv[6]; p.kappa_v_S = dv[7]; p.cd = dv[8]; p.tide_amp = dv[9];
    p.tide_period = dv[10];
    p.alpha = dv[11]; p.beta = dv[12]; p.T0 = dv[13]; p.S0 = dv[14];
    p.Tref_s = dv[15]; p.Tref_dz = dv[16];
    return p;
}

static CompatParams compat_from(const double *dv) {
    CompatParams p;
    p.g = dv[0]; p.rho0 = dv[1]; p.alpha = dv[2]; p.beta = dv[3];
    p.nu_h = dv[4]; p.nu_v = dv[5]; p.kappa_v_T = dv[6]; p.kappa_v_S = dv[7];
    return p;
}

extern "C" {

const char *orc_last_error() { return g_err.c_str(); }

int orc_basis(int order, int kind, double *nodes, double *weights, double *D, double *S) {
    ORC_TRY({
        Basis1D b = kind == 0 ? make_lgl(order) : make_gl(order);
        const int np = b.np();
        std::memcpy(nodes, b.nodes.data(), sizeof(double) * np);
        std::memcpy(weights, b.weights.data(), sizeof(double) * np);
        std::memcpy(D, b.D.data(), sizeof(double) * np * np);
        std::memcpy(S, b.S.data(), sizeof(double) * np * np);
    })
}

int orc_dense_3d(int order, double *Dxi, double *Deta, double *Dzeta) {
    ORC_TRY({
        Basis1D b = make_lgl(order);
        Vec a, c, d;
        build_dense_3d(b, a, c, d);
        std::memcpy(Dxi, a.data(), sizeof(double) * a.size());
        std::memcpy(Deta, c.data(), sizeof(double) * c.size());
        std::memcpy(Dzeta, d.data(), sizeof(double) * d.size());
    })
}

int orc_sw_flux(int kind, const double *UL, const double *UR, double nx, double ny, double g,
                double *F) {
    ORC_TRY(sw_flux(kind, UL, UR, nx, ny, g, F))
}

int orc_compat_rhs(int order, int nel, const double *const *in6, const double *h, const double *f,
                   const double *params8, double *const *out5) {
    ORC_TRY(compat_compute_rhs(order, nel, in6, h, f, compat_from(params8), out5))
}

int orc_compat_modesplit(int order, int nel, double dt, int nsub, double *const *st12,
                         const double *h, const double *f, const double *params8) {
    ORC_TRY(compat_modesplit_step(order, nel, dt, nsub, st12, h, f, compat_from(params8)))
}

int orc_compat_ssprk3(int order, int nel, double dt, double *const *st6, const double *h,
                      const double *f, const double *params8, int nthreads) {
    ORC_TRY(compat_ssprk3_step(order, nel, dt, st6, h, f, compat_from(params8), nthreads))
}

void *orc_phys_create(const int *iv, const double *dv, const double *h, const double *f,
                      const double *tx, const double *ty) {
    try {
        auto *m = new PhysModel();
        m->init(phys_from(iv, dv), h, f, tx, ty);
        return m;
    } catch (const std::exception &e) {
        g_err = e.what();
        return nullptr;
    }
}
void orc_phys_destroy(void *hd) { delete static_cast<PhysModel *>(hd); }

int orc_phys_set_state(void *hd, const double *const *q4, const double *eta, double t) {
    ORC_TRY({
        auto *m = static_cast<PhysModel *>(hd);
        m->set_state(q4, eta);
        m->t = t;
    })
}

int orc_phys_get_state(void *hd, double *const *q4, double *eta, double *HU, double *HV,
                       double *eta_avg, double *t) {
    ORC_TRY({
        auto *m = static_cast<PhysModel *>(hd);
        for (int v = 0; v < 4; ++v) std::memcpy(q4[v], m->Q[v].data(), sizeof(double) * m->n3);
        std::memcpy(eta, m->eta.data(), sizeof(double) * m->n2);
        std::memcpy(HU, m->HU.data(), sizeof(double) * m->n2);
        std::memcpy(HV, m->HV.data(), sizeof(double) * m->n2);
        std::memcpy(eta_avg, m->eta_avg.data(), sizeof(double) * m->n2);
        *t = m->t;
    })
}

// etab: the baroclinic pressure's surface elevation (null: the model's eta)
int orc_phys_rhs(void *hd, double *const *r4, double *omega, double *deta, const double *etab) {
    ORC_TRY({
        auto *m = static_cast<PhysModel *>(hd);
        Vec R[4], om, de, eb;
        if (etab) eb.assign(etab, etab + m->n2);
        m->rhs3d(m->Q, m->eta, m->t, R, &om, &de, etab ? &eb : nullptr);
        for (int v = 0; v < 4; ++v) std::memcpy(r4[v], R[v].data(), sizeof(double) * m->n3);
        std::memcpy(omega, om.data(), sizeof(double) * m->n3);
        std::memcpy(deta, de.data(), sizeof(double) * m->n2);
    })
}

int orc_phys_rhs2d(void *hd, const double *Fx, const double *Fy, double time, double *ke,
                   double *ku, double *kv) {
    ORC_TRY({
        auto *m = static_cast<PhysModel *>(hd);
        Vec fx(Fx, Fx + m->n2), fy(Fy, Fy + m->n2), a, b, c;
        m->rhs2d(m->eta, m->HU, m->HV, &fx, &fy, time, a, b, c);
        std::memcpy(ke, a.data(), sizeof(double) * m->n2);
        std::memcpy(ku, b.data(), sizeof(double) * m->n2);
        std::memcpy(kv, c.data(), sizeof(double) * m->n2);
    })
}

int orc_phys_split_steps(void *hd, double dt, int nsub, int nsteps) {
    ORC_TRY({
        auto *m = static_cast<PhysModel *>(hd);
        for (int s = 0; s < nsteps; ++s) m->split_step(dt, nsub);
    })
}

int orc_phys_rk_steps(void *hd, int scheme, double dt, int nsteps) {
    ORC_TRY({
        auto *m = static_cast<PhysModel *>(hd);
        for (int s = 0; s < nsteps; ++s) m->rk_step(scheme, dt);
    })
}

int orc_phys_diagnostics(void *hd, double *out10) {
    ORC_TRY(static_cast<PhysModel *>(hd)->diagnostics(out10))
}

// dU/dt = lam * U + sin(t) integrated with a generic scheme (reference time-stepper tests,
// tests/unit/test_time_stepper.cpp).
int orc_rk_ode(int scheme, double lam, double U0, double T, int nsteps, double *out) {
    ORC_TRY({
        Vec U(1, U0);
        const double dt = T / nsteps;
        double t = 0.0;
        for (int s = 0; s < nsteps; ++s) {
            rk_step(scheme, t, dt, U, [lam](double tt, const Vec &x, Vec &dx) {
                dx.resize(1);
                dx[0] = lam * x[0] + std::sin(tt);
            });
            t += dt;
        }
        *out = U[0];
    })
}

// ----------------------------------------------------------------------------- Bezier
struct BzHandle {
    BzSystem S;
    CSR A;
    BzMG M;
};

void *orc_bz_build(int nx, int ny, double x0, double y0, double Lx, double Ly, double lambda,
                   double eps, const double *dgauss) {
    try {
        auto *h = new BzHandle();
        BzGrid g;
        g.nx = nx; g.ny = ny; g.x0 = x0; g.y0 = y0; g.Lx = Lx; g.Ly = Ly;
        g.lambda = lambda; g.eps = eps;
        bz_build(h->S, g, dgauss);
        return h;
    } catch (const std::exception &e) {
        g_err = e.what();
        return nullptr;
    }
}
void orc_bz_destroy(void *h) { delete static_cast<BzHandle *>(h); }

int orc_bz_info(void *hd, long *ndof, double *alpha, double *dTWd) {
    ORC_TRY({
        auto *h = static_cast<BzHandle *>(hd);
        *ndof = h->S.ndof; *alpha = h->S.alpha; *dTWd = h->S.dTWd;
    })
}

int orc_bz_element_mats(double dx, double dy, double *H, double *B) {
    ORC_TRY({
        element_hessian(dx, dy, 4, H);
        element_mass(dx, dy, 4, B);
    })
}

int orc_bz_vec(void *hd, int which, double *out) {
    ORC_TRY({
        auto *h = static_cast<BzHandle *>(hd);
        const BVec &v = which == 0 ? h->S.b : h->S.BtWd;
        std::memcpy(out, v.data(), sizeof(double) * v.size());
    })
}

static const CSR &pick(BzHandle *h, int which) {
    return which == 0 ? h->S.H : which == 1 ? h->S.BtWB : which == 2 ? h->S.Q : h->A;
}

long orc_bz_nnz(void *hd, int which) {
    auto *h = static_cast<BzHandle *>(hd);
    const CSR &M = pick(h, which);
    return M.rp.empty() ? 0 : M.rp.back();
}
long orc_bz_rows(void *hd, int which) { return pick(static_cast<BzHandle *>(hd), which).n; }

int orc_bz_csr(void *hd, int which, long *rp, long *ci, double *v) {
    ORC_TRY({
        const CSR &M = pick(static_cast<BzHandle *>(hd), which);
        std::memcpy(rp, M.rp.data(), sizeof(long) * M.rp.size());
        std::memcpy(ci, M.ci.data(), sizeof(long) * M.ci.size());
        std::memcpy(v, M.v.data(), sizeof(double) * M.v.size());
    })
}

int orc_bz_constraints(void *hd, int edge_ngauss) {
    ORC_TRY({
        auto *h = static_cast<BzHandle *>(hd);
        bz_constraints(h->S, edge_ngauss, h->A);
    })
}

int orc_bz_objective(void *hd, const double *x, double *parts, double *obj) {
    ORC_TRY(*obj = bz_objective(static_cast<BzHandle *>(hd)->S, x, parts))
}

int orc_bz_mg_setup(void *hd, int coarsest_n, int *nlevels) {
    ORC_TRY({
        auto *h = static_cast<BzHandle *>(hd);
        bz_mg_setup(h->S, h->M, coarsest_n);
        *nlevels = (int)h->M.lv.size();
    })
}

int orc_bz_level_info(void *hd, int l, int *n, double *K, double *rho, double *binv) {
    ORC_TRY({
        auto *h = static_cast<BzHandle *>(hd);
        const BzLevel &L = h->M.lv.at(l);
        *n = L.n;
        if (K) std::memcpy(K, L.K, sizeof(L.K));
        if (rho) std::memcpy(rho, L.rho.data(), sizeof(double) * L.rho.size());
        if (binv && !L.binv.empty()) std::memcpy(binv, L.binv.data(), sizeof(double) * L.binv.size());
    })
}

int orc_bz_level_apply(void *hd, int l, const double *x, double *y) {
    ORC_TRY(bz_level_apply(static_cast<BzHandle *>(hd)->M, l, x, y))
}

int orc_bz_mg_vcycle(void *hd, const double *r, double *z) {
    ORC_TRY(bz_mg_vcycle(static_cast<BzHandle *>(hd)->M, r, z))
}

int orc_bz_mg_apply_ref(void *hd, const double *b, double *x, double tol, int max_cycles, int *cycles) {
    ORC_TRY(*cycles = bz_mg_apply_ref(static_cast<BzHandle *>(hd)->M, b, x, tol, max_cycles))
}

int orc_bz_pcg(void *hd, int precond, const double *b, double *x, double tol, int maxit,
               int *iters, double *relres) {
    ORC_TRY({
        auto *h = static_cast<BzHandle *>(hd);
        *iters = bz_pcg(h->S, &h->M, precond, b, x, tol, maxit, relres);
    })
}

}  // extern "C"

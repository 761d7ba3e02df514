/* drifter_b200 — B200-native (sm_100a) matrix-free operator path of DRIFTER.
 *
 * C ABI of libdrifter_b200.so. Plain pointers and sizes only; every call returns an int
 * status (0 = OK, see DRF_E_*); the message of the last failure on the calling thread is
 * available from drf_last_error(). Handles are opaque, own their device memory and one
 * CUDA stream each, and must not be shared between host threads.
 *
 * Array layouts (all host arrays are FP64, caller-owned):
 *   3D nodal field  : [column][layer][k][j][i], column = ex + nx*ey, node = i + np*(j + np*k),
 *                     np = order + 1 (LGL nodes) — size nx*ny*nz*np^3.
 *   2D nodal field  : [column][j][i] — size nx*ny*np^2.
 *   compat fields   : [element][dof], dof = i + np*(j + np*k) (the reference's element
 *                     vectors, include/dg/basis_hexahedron.hpp:255).
 */
#ifndef DRIFTER_B200_H
#define DRIFTER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    DRF_OK = 0,
    DRF_E_INVALID = 1,   /* bad argument (the reference throws std::invalid_argument) */
    DRF_E_CUDA = 2,      /* CUDA runtime failure */
    DRF_E_NOMEM = 3,     /* device allocation failed */
    DRF_E_NONFINITE = 4, /* NaN/Inf found in an input or a result */
    DRF_E_UNSUPPORTED = 5,
    DRF_E_TIMEOUT = 6    /* a bounded device wait gave up */
};

enum { DRF_FLUX_LF = 0, DRF_FLUX_HLLC = 1, DRF_FLUX_ROE = 2 };
enum { DRF_PREC_FP64 = 0, DRF_PREC_MIXED = 1 };
enum { DRF_BC_WALL = 0, DRF_BC_TIDE = 1 };
enum { DRF_RK_EULER = 0, DRF_RK_MIDPOINT = 1, DRF_RK_SSP3 = 2, DRF_RK_RK4 = 3, DRF_RK_LSRK45 = 4,
       DRF_RK_DOPRI = 5 };

/* Copies the last error message of the calling thread into buf (NUL-terminated). */
int drf_last_error(char *buf, size_t n);
/* Library version string and the number of kernels this library has launched (kernels replayed
 * from a CUDA graph count once per replay; queuing them into a graph being captured does not
 * count). No reference counterpart: launch accounting of this library. */
const char *drf_version(void);
uint64_t drf_kernel_launch_count(void);
/* Number of device allocations (cudaMalloc) this library has made since it was loaded. No
 * reference counterpart: lets a caller verify that a call allocated nothing. */
uint64_t drf_device_alloc_count(void);

/* ------------------------------------------------------------------ fluxes
 * Batched shallow-water numerical flux F*(U_L, U_R, n) on the GPU, U = (h, hu, hv).
 * Replaces NumericalFluxFunc (include/flux/numerical_flux.hpp:25) as produced by
 * NumericalFluxFactory::shallow_water_{lax_friedrichs,hllc,roe}
 * (src/flux/numerical_flux.cpp:134-190; LaxFriedrichsFlux::flux
 * include/flux/numerical_flux.hpp:222, ShallowWaterHLLCFlux::flux :272,
 * ShallowWaterRoeFlux::flux src/flux/numerical_flux.cpp:13).
 * UL, UR, F: n x 3; normals: n x 2 (nx, ny). */
int drf_sw_flux_batch(int kind, int64_t n, const double *UL, const double *UR,
                      const double *normals, double g, double *F);

/* ------------------------------------------------------------------ DG, reference semantics
 * compat params (8 doubles): g, rho0, alpha, beta, nu_h, nu_v, kappa_v_T, kappa_v_S
 * (OceanConstants include/physics/primitive_equations.hpp:41, DiffusivityParams :106). */

/* PrimitiveEquationsSolver::compute_rhs (include/physics/primitive_equations.hpp:240,
 * src/physics/primitive_equations.cpp:428): element-local tendencies of nel elements.
 * in6 = {Hu, Hv, eta, HT, HS, omega}, out5 = {dHu, dHv, deta, dHT, dHS}, h/f: per node. */
int drf_compat_compute_rhs(int order, int nel, const double *const *in6, const double *h,
                           const double *f, const double *params8, double *const *out5);

/* Device time of PrimitiveEquationsSolver::compute_rhs (the element-local right-hand side
 * above) on nel elements: the nsrc given elements are repeated to nel on the device, the kernel
 * runs 3 untimed and nrep timed launches, and *ms is the mean per launch (CUDA events). Lets a
 * caller compare the same algorithm on the GPU and on the host. */
int drf_compat_time_rhs(int order, int nsrc, const double *const *in6, const double *h,
                        const double *f, const double *params8, int nel, int nrep, double *ms);

/* ModeSplittingSolver::step (include/physics/mode_splitting.hpp:241,
 * src/physics/mode_splitting.cpp:434) on nel elements, in place.
 * st12 = {Hu, Hv, eta, HT, HS, H, u, v, T, S, omega, rho}. */
int drf_compat_modesplit_step(int order, int nel, double dt, int nsub, double *const *st12,
                              const double *h, const double *f, const double *params8);

/* ------------------------------------------------------------------ DG, coupled model */
typedef struct drf_dg drf_dg;

typedef struct {
    int32_t nx, ny, nz; /* hexes in x, y (columns) and sigma (layers) */
    int32_t order;      /* polynomial order N, np = N + 1 LGL nodes per direction (1..5) */
    double Lx, Ly;      /* basin extent [m] */
} drf_mesh_desc;

typedef struct {
    double g, rho0;                        /* 9.81, 1025 */
    double nu_h, nu_v, kappa_v_T, kappa_v_S; /* DiffusivityParams defaults 1, 1e-4, 1e-5, 1e-5 */
    double cd;                             /* quadratic bottom drag (BottomFriction, 2.5e-3) */
    int32_t flux2d;                        /* DRF_FLUX_* for the barotropic face flux */
    int32_t precision;                     /* DRF_PREC_FP64 or DRF_PREC_MIXED */
    int32_t bc[4];                         /* west, east, south, north: DRF_BC_* */
    double tide_amp, tide_period;          /* tidal elevation on DRF_BC_TIDE sides */
    /* linear equation of state rho = rho0 (1 - alpha (T - T0) + beta (S - S0)) of the
     * baroclinic pressure gradient (EquationOfState include/physics/equation_of_state.hpp:35-40,
     * defaults 2e-4, 7.6e-4, 10, 35); alpha = beta = 0 switches that gradient off */
    double alpha, beta, T0, S0;
    /* horizontally uniform reference stratification T_ref(z) = Tref_s + Tref_dz z (z <= 0 up
     * from the surface, S_ref = S0): the pressure is integrated from the density anomaly
     * against it (its own pressure has no horizontal gradient). Tref_s = T0, Tref_dz = 0
     * subtracts nothing. */
    double Tref_s, Tref_dz;
} drf_dg_params;

/* Creates the model: h (bathymetry > 0), f (Coriolis), taux/tauy (surface stress, N/m^2)
 * are 2D nodal fields. Replaces PrimitiveEquationsSolver/ModeSplittingSolver::initialize
 * (src/physics/primitive_equations.cpp:697, src/physics/mode_splitting.cpp:347) and
 * SimulationDriver::initialize (src/solver/simulation_driver.cpp:29). */
int drf_dg_create(const drf_mesh_desc *mesh, const drf_dg_params *params, const double *h,
                  const double *f, const double *taux, const double *tauy, drf_dg **out);
int drf_dg_destroy(drf_dg *m);
/* Uses the given cudaStream_t for all work of this model (NULL = the model's own stream). */
int drf_dg_set_stream(drf_dg *m, void *cuda_stream);
int drf_dg_sync(drf_dg *m);

/* Host FP64 state in/out. q = {Hu, Hv, HT, HS} 3D fields, eta 2D. On upload the barotropic
 * transports are the depth integrals of Hu, Hv. (SimulationDriver::pack_state/unpack_state,
 * src/solver/simulation_driver.cpp:199,215.) Any output pointer may be NULL. */
int drf_dg_upload_state(drf_dg *m, const double *const *q4, const double *eta, double t);
int drf_dg_download_state(drf_dg *m, double *const *q4, double *eta, double *HU, double *HV,
                          double *eta_avg, double *t);

/* Asynchronous output staging around the time loop (SimulationDriver's output calls,
 * src/io/vtk_writer.cpp, write from host copies of the state): the current state (pending
 * transport correction folded in) is snapshot in FP64 on the model's stream and copied to the
 * given host buffers on a copy stream of its own, so steps enqueued after this call run while
 * the copy is in flight. The buffers (q4 = {Hu, Hv, HT, HS} 3D, eta, HU, HV 2D; any may be NULL)
 * are valid after drf_dg_output_wait, which also returns the snapshot's model time. Pinned
 * (page-locked) host buffers make the copy asynchronous. A new drf_dg_output_stage waits for the
 * previous copy on the device, not on the host. */
int drf_dg_output_stage(drf_dg *m, double *const *q4, double *eta, double *HU, double *HV);
int drf_dg_output_wait(drf_dg *m, double *t);

/* Coupled right-hand side at the current state (eta frozen): R = {dHu, dHv, dHT, dHS},
 * omega (3D sigma velocity), deta (2D, -int div(Hu) dsigma). Maps
 * PrimitiveEquationsSolver::compute_rhs + apply_interface_fluxes + the column diagnosis
 * VerticalVelocityDiagnosis::diagnose_omega (src/physics/vertical_velocity.cpp:55). */
int drf_dg_compute_rhs(drf_dg *m, double *const *r4, double *omega, double *deta);

/* Barotropic operator (2D, FP64) with forcing Fx, Fy at time t on the current state. */
int drf_dg_compute_rhs2d(drf_dg *m, const double *Fx, const double *Fy, double time,
                         double *ke, double *khu, double *khv);

/* nsteps baroclinic steps: LSRK45 3D stages (include/solver/time_stepper.hpp:56-61) plus
 * nsub barotropic predictor-corrector subcycles per step, each step replayed as one CUDA
 * graph. Maps ModeSplittingSolver::step (include/physics/mode_splitting.hpp:241). */
int drf_dg_step_modesplit(drf_dg *m, double dt, int nsub, int nsteps);

/* Non-split RK over (Hu, Hv, HT, HS, eta): TimeStepper::step
 * (include/solver/time_stepper.hpp:18) with the scheme of DRF_RK_*. */
int drf_dg_rk_step(drf_dg *m, int scheme, double dt, int nsteps);

/* FP64 diagnostics (SimulationDriver::compute_diagnostics, src/solver/simulation_driver.cpp:237):
 * out[10] = {mass_weighted, mass_unweighted, energy, heat, salt, max_speed, max_eta,
 *            min_eta, max_T, min_T}. */
int drf_dg_diagnostics(drf_dg *m, double *out10);

/* Device-side timing of the dominant 3D stage kernel: runs nrep stage launches on the
 * model's stream between CUDA events; *ms = mean per launch. Also reports the bytes the
 * stage moves by the algorithmic model (*alg_bytes) and the number of 3D DOFs (*ndof). */
int drf_dg_time_stage(drf_dg *m, int nrep, double *ms, double *alg_bytes, double *ndof);

/* Device time of the stage kernel's memory traffic alone: a copy kernel with the same CTA
 * shape, shared memory and bulk-copy staging that reads the state and the LSRK register and
 * writes 8 arrays back in the stage's store pattern (*bytes moved per launch). It is the
 * bandwidth ceiling of the stage's access structure; the model state is not modified.
 * No counterpart in the reference. */
int drf_dg_time_copy(drf_dg *m, int nrep, double *ms, double *bytes);

/* Replaces the surface stress fields (WindStress::compute, src/physics/primitive_equations.cpp:695)
 * for the following steps; asynchronous on the model's stream (pinned host memory recommended;
 * the caller keeps the buffers alive until the next drf_dg_sync). */
int drf_dg_set_forcing(drf_dg *m, const double *taux, const double *tauy);
/* Copies the 2D surface elevation to the host (synchronous). */
int drf_dg_download_surface(drf_dg *m, double *eta);

/* Autotuned launch shape: the barotropic subcycle kernels' tile (water columns per CTA) chosen
 * by timing the candidates 2, 4, 8, 16 on this model (done at the first step, or here), and
 * the candidates' times in ms (baro_ms4 may be NULL). No counterpart in the reference, which
 * has no kernels; DRIFTER_B200_TUNE=0 keeps the default tile of 8. */
int drf_dg_tuning(drf_dg *m, int *baro_cols_per_cta, double *baro_ms4);
/* Autotuned stage launch: how far ahead (in half waves of resident CTAs, 0..2, and in columns)
 * each stage CTA prefetches a later column into L2, chosen by timing the three on this model (at
 * the first step, or here), and the candidates' times in ms (stage_ms3 may be NULL; zeros when
 * the distance was fixed by DRIFTER_B200_STAGE_PREFETCH or DRIFTER_B200_TUNE=0). No counterpart
 * in the reference. */
int drf_dg_stage_tuning(drf_dg *m, int *prefetch_half_waves, int *prefetch_columns, double *stage_ms3);

/* Size and pointer introspection for the bench (device-resident timing). */
int drf_dg_info(drf_dg *m, int64_t *n3d_nodes, int64_t *n2d_nodes, int *precision);

/* ------------------------------------------------------------------ ensembles
 * An ensemble of independent coupled DG runs with their own meshes (nx, ny, nz), bathymetry,
 * forcing, parameters and step sizes, stepped together: each LSRK stage of all members is ONE
 * kernel launch over every member's water columns (one CTA per column, tallest columns first),
 * each barotropic substep one
 * launch over every member's 2D tiles, and each baroclinic step one CUDA graph. Per member
 * the result is that of ModeSplittingSolver::step (include/physics/mode_splitting.hpp:241)
 * as computed by drf_dg_step_modesplit. The reference runs members one after the other. */
typedef struct drf_ens drf_ens;

/* All members share the order, precision and 2D flux kind; the arrays are indexed by member
 * (h[i], f[i], taux[i], tauy[i] are member i's 2D fields, as for drf_dg_create). */
int drf_ens_create(int nmembers, const drf_mesh_desc *meshes, const drf_dg_params *params,
                   const double *const *h, const double *const *f, const double *const *taux,
                   const double *const *tauy, drf_ens **out);
int drf_ens_destroy(drf_ens *e);
/* Handle of member i for drf_dg_upload_state, drf_dg_download_state, drf_dg_diagnostics,
 * drf_dg_compute_rhs, drf_dg_set_forcing and drf_dg_download_surface. It is owned by the
 * ensemble: drf_dg_destroy, drf_dg_set_stream and drf_dg_step_modesplit reject it. */
int drf_ens_member(drf_ens *e, int i, drf_dg **member);
int drf_ens_set_stream(drf_ens *e, void *cuda_stream);
int drf_ens_sync(drf_ens *e);
/* nsteps baroclinic steps of every member, member i with step dt[i] and nsub subcycles. */
int drf_ens_step(drf_ens *e, const double *dt, int nsub, int nsteps);
/* Totals for the bench: 3D nodes over all members, stage work items (water columns) and the
 * stage grid (one CTA per item). */
int drf_ens_info(drf_ens *e, int64_t *n3d_nodes, int *items, int *grid);

/* ------------------------------------------------------------------ Bezier smoother
 * Uniform-grid cubic Bezier bathymetry smoother: Q = alpha H + lambda (B^T W B + eps I),
 * control points (3 nx + 1) x (3 ny + 1), point (gi, gj) at gi + (3 nx + 1) gj. */
typedef struct drf_bz drf_bz;

typedef struct {
    int32_t nx, ny;               /* elements per direction (the GPU path needs nx == ny) */
    double x0, y0, Lx, Ly;        /* domain */
    double lambda, ridge_epsilon; /* CGCubicBezierSmootherConfig::lambda, ridge_epsilon */
} drf_bz_grid_desc;

/* Builds the operator and assembles b = lambda B^T W d on the GPU from the data sampled at the
 * 4x4 Gauss points of every element (dgauss: [ey][ex][qj][qi]). Replaces
 * CGBezierSmootherBase::assemble_hessian_global / assemble_data_fitting_global / assemble_Q /
 * assemble_b (src/bathymetry/cg_bezier_smoother_base.cpp:260,308,396,405). */
int drf_bz_create(const drf_bz_grid_desc *grid, const double *dgauss, drf_bz **out);
int drf_bz_destroy(drf_bz *h);
int drf_bz_set_stream(drf_bz *h, void *cuda_stream);
int drf_bz_info(drf_bz *h, int64_t *ndof, double *alpha, int *nlevels);
int drf_bz_get_rhs(drf_bz *h, double *b);
/* y = Q x, matrix-free (the SpMV L.Q * x of src/bathymetry/bezier_multigrid_preconditioner.cpp:776). */
int drf_bz_apply_Q(drf_bz *h, const double *x, double *y);
/* Per-element L2 misfit of the smoothed surface x (control points) to the data, for every
 * element: AdaptiveCGCubicBezierSmoother::compute_element_l2_error / estimate_element_error
 * (src/bathymetry/adaptive_cg_cubic_bezier_smoother.cpp:100,142), the error estimate of the
 * adaptive smoother's refinement loop. zdata holds the data sampled at the ngauss x ngauss
 * Gauss-Legendre points of each element ([ey][ex][qj][qi], points on [0,1]^2, the reference's
 * ngauss_error, default 4). l2[e] = sqrt(sum_q w_q (z_data - z_bezier)^2 * dx dy);
 * normalized[e] = l2[e] / sqrt(dx dy) (may be NULL). */
int drf_bz_element_errors(drf_bz *h, const double *x, const double *zdata, int ngauss, double *l2,
                          double *normalized);

/* The same estimate on any quadtree mesh of the adaptive smoother (hanging-node meshes
 * included): n_elem elements, bounds n x (xmin, ymin, xmax, ymax), coeffs n x 16 the element's
 * Bezier control values (i + 4 j, with hanging-node constraints already resolved), zdata
 * n x ngauss^2 ([e][qj][qi]). The Bernstein values follow the reference's recurrence
 * (CubicBezierBasis2D::evaluate_bernstein_1d, src/bathymetry/cubic_bezier_basis_2d.cpp:42) and
 * every product and sum is rounded in the reference's order. Host buffers. */
int drf_bz_mesh_element_errors(int64_t n_elem, const double *bounds, const double *coeffs, const double *zdata,
                               int ngauss, double *l2, double *normalized);
/* The element part of CGBezierSmootherBase::assemble_data_fitting_global
 * (src/bathymetry/cg_bezier_smoother_base.cpp:308-364) on any quadtree mesh: per element the
 * 16 x 16 block BtWB[e][i][j] = sum_q weight B_i B_j, BtWd[e][i] = sum_q weight B_i d and
 * dTWd[e] = sum_q weight d d, weight = w_qi w_qj dx dy relaxation, with gauss_legendre_01
 * (:28-58, which has 4 points at most: ngauss 1..4, a caller of the reference's ngauss_data >= 4
 * passes 4). zdata, relax (NULL: factor 1) n x ngauss^2 ([e][qj][qi]). The scatter into the
 * global system through the DOF map stays with the caller. Host buffers. */
int drf_bz_mesh_data_fitting(int64_t n_elem, const double *bounds, const double *zdata, const double *relax,
                             int ngauss, double *BtWB, double *BtWd, double *dTWd);
/* BezierMultigridPreconditioner::setup (include/bathymetry/bezier_multigrid_preconditioner.hpp:240):
 * levels down to coarsest_n elements per direction, pre/post colored-Schwarz sweeps. */
int drf_mg_setup(drf_bz *h, int coarsest_n, int pre, int post);
/* One V-cycle z = M r of this build's symmetric form (R = P^T, post-smoothing in reverse colour
 * order): a fixed SPD preconditioner for plain PCG (BezierMultigridPreconditioner::apply, :246,
 * repeats V-cycles to a tolerance; drf_mg_apply_reference does that). */
int drf_mg_apply(drf_bz *h, const double *r, double *z);
/* BezierMultigridPreconditioner::apply as the reference computes it
 * (include/bathymetry/bezier_multigrid_preconditioner.hpp:246,
 * src/bathymetry/bezier_multigrid_preconditioner.cpp:690-812): z = 0, then V-cycles with the
 * row-normalised restriction (:209-225) and the same colour order before and after the coarse
 * correction, until ||r - Q z|| < tol ||r|| or max_vcycles (the reference's defaults are 1e-6
 * and 100). *cycles = V-cycles run, *relres = the final relative residual (either may be NULL). */
int drf_mg_apply_reference(drf_bz *h, const double *r, double *z, double tol, int max_vcycles,
                           int *cycles, double *relres);
/* z = M r for preconditioner kind (0 none, 1 Jacobi, 2 multigrid, 3 learned, 4 the reference's
 * multigrid apply with its default tolerance). */
int drf_bz_precondition(drf_bz *h, int kind, const double *r, double *z);
/* PCG on Q x = b to ||r|| <= tol ||b|| (FP64). b NULL = the assembled right-hand side; x holds
 * the initial guess and returns the solution. kind: 0 none, 1 Jacobi, 2 multigrid V-cycle,
 * 3 learned (Jacobi plus the network's correction, flexible CG), 4 the reference's multigrid
 * apply (V-cycles to 1e-6, a variable preconditioner: flexible CG, host-driven iterations).
 * Maps the PCG loop of
 * solve_with_constraints_iterative (src/bathymetry/cg_cubic_bezier_bathymetry_smoother.cpp:479-558)
 * with Q in place of the Schur operator. *ms = device time of the solve. */
int drf_pcg_solve(drf_bz *h, const double *b, double *x, double tol, int maxit, int kind,
                  int *iters, double *relres, double *ms);

/* C1 continuity rows y = A x: the normal derivative matched at edge_ngauss (1..8) Gauss points
 * of every interior edge (CGCubicBezierDofManager::build_edge_derivative_constraints,
 * src/bathymetry/cg_cubic_bezier_dof_manager.cpp:319, scaled by 1/h as assemble_A_edge_free,
 * src/bathymetry/cg_cubic_bezier_bathymetry_smoother.cpp:798). Square grids. y has
 * 2 n (n - 1) edge_ngauss rows: edges between (ex, ey) and (ex + 1, ey) first, row
 * (ey (n - 1) + ex) edge_ngauss + q, then edges between (ex, ey) and (ex, ey + 1), row
 * n (n - 1) edge_ngauss + (ey n + ex) edge_ngauss + q. Host buffers. */
int drf_bz_constraints_apply(drf_bz *h, int edge_ngauss, const double *x, double *y);

/* Constrained minimiser under the C1 rows: CG on the Schur complement S = A Q^-1 A^T with
 * rhs A Q^-1 b, then x = Q^-1 (b - A^T lambda)
 * (CGCubicBezierBathymetrySmoother::solve_with_constraints_iterative,
 * src/bathymetry/cg_cubic_bezier_bathymetry_smoother.cpp:305, Schur preconditioner None:
 * stop when r.r / r0.r0 < tol^2). Every Q^-1 is a PCG solve from zero to inner_tol with
 * preconditioner inner_kind (as drf_pcg_solve). b is the assembled right-hand side. x: host
 * output; *outer_iters, *relres = sqrt(r.r / r0.r0), *ms = device time. */
int drf_bz_constrained_solve(drf_bz *h, int edge_ngauss, int inner_kind, double tol, int maxit,
                             double inner_tol, double *x, int *outer_iters, double *relres, double *ms);

/* ------------------------------------------------------------------ learned preconditioner
 * No counterpart in the reference. A 4-layer conv3x3 network (BF16, FP32 accumulation) on
 * 3x3 superpixels of the control-point grid, trained on the GPU on (residual, error) pairs
 * from the smoother's own multigrid solves; PCG preconditioner kind 3 is z = D^-1 r + the
 * network's correction (flexible CG).
 * Images are NHWC with 16 channels (9 used: control point (3I+di, 3J+dj) -> channel di+3dj). */
typedef struct drf_cnn drf_cnn;
int64_t drf_cnn_nparams(void);
int drf_cnn_create(uint64_t seed, drf_cnn **out);
int drf_cnn_destroy(drf_cnn *h);
/* parameters packed per layer: W [co][tap][ci] (channels 16,32,32,32,16) then bias [co] */
int drf_cnn_get_params(drf_cnn *h, double *p);
int drf_cnn_set_params(drf_cnn *h, const double *p);
/* forward of B images (host FP64 in/out); with T != NULL also the mean-square loss over the 9
 * used channels and its parameter gradient */
int drf_cnn_forward_backward(drf_cnn *h, int B, int H, int W, const double *X, const double *T,
                             double *Y, double *grad, double *loss);
int drf_cnn_set_dataset(drf_cnn *h, int N, int H, int W, const double *X, const double *T);
int drf_cnn_train(drf_cnn *h, int steps, int batch, int crop, double lr, uint64_t seed,
                  double *loss);
/* attaches a trained network to a smoother as preconditioner kind 3 (output scale s:
 * z = D^-1 r + rms(r) s net(r / rms(r))) */
int drf_bz_set_cnn(drf_bz *h, drf_cnn *net, double out_scale);
/* The conv-form autotuning done by drf_bz_set_cnn at the smoother's size: form4[l] = 0 for the
 * warp-level mma.sync conv, 1 for the tcgen05 conv of layer l (bit-identical outputs);
 * ms8[2 l + f] = the timed launch of layer l in form f (0 when not tuned: DRIFTER_B200_TUNE=0 or
 * DRIFTER_B200_CNN_MMA set). No reference counterpart. Either pointer may be NULL. */
int drf_bz_cnn_tuning(drf_bz *h, int *form4, double *ms8);

/* Allocation-free variant of drf_pcg_solve with the Jacobi preconditioner (kind 1), for callers
 * that cannot allocate device memory. No counterpart in the reference (it has no device code).
 * The caller owns d_b (device, (3 nx + 1)^2 doubles) and d_x (device, initial guess in,
 * solution out); stream is a cudaStream_t (NULL = legacy default stream).
 * Scratch: one file-scope device array of 8.5 MB in libdrifter_b200.so, held on every device
 * that loads the library until process exit; grids up to 262,144 control points (nx <= 170),
 * larger sizes return DRF_E_UNSUPPORTED. It calls no cudaMalloc/cudaFree. Every call looks up
 * the array's address in the current device's context (cudaGetSymbolAddress) and waits for its
 * stream between batches of 8 iterations. Every call shares the array: calls that overlap on the
 * GPU (other host threads, other streams) race and must be serialised by the caller. */
int drf_bz_jacobi_pcg_noalloc(const drf_bz_grid_desc *grid, const double *d_b, double *d_x,
                              double tol, int maxit, void *stream, int *iters, double *relres);

/* ------------------------------------------------------------------ mortars (non-conforming faces)
 * MortarSpace (src/dg/mortar.cpp:13; include/dg/mortar.hpp:29) and the non-conforming face flux
 * of DG3DIntegration (compute_interface_flux_nonconforming, src/dg/operators_3d.cpp:345) for
 * hexahedral LGL elements of one order p (1..5): mortar order p, (2p+1)^2 Gauss-Legendre
 * mortar points on the coarse face, P = M^-1 B and L = B^T for the coarse face and each fine
 * face (fine coupling over the mortar points inside the closed sub-face), scalar flux at the
 * mortar nodes, lifts L_c M^-1 F to the coarse face and -L_f M^-1 F to the fine faces.
 * Connection types are FaceConnectionType (include/dg/face_connection.hpp:15); face f has its
 * normal along axis f / 2, positive when f is odd; face node (it, jt) is the volume node with
 * the normal index on the face and the two tangential indices in axis order. */
enum {
    DRF_MORTAR_SAME_LEVEL = 0,
    DRF_MORTAR_FINE_2X1 = 1,
    DRF_MORTAR_FINE_1X2 = 2,
    DRF_MORTAR_FINE_3_2PLUS1 = 3,
    DRF_MORTAR_FINE_3_1PLUS2 = 4,
    DRF_MORTAR_FINE_2X2 = 5
};
/* scalar numerical fluxes for u_t + div(a u) = 0 (include/flux/numerical_flux.hpp):
 * CentralFlux (:244), UpwindFlux (:264), LaxFriedrichsFlux (:222) with speed |a.n| */
enum { DRF_MORTAR_FLUX_CENTRAL = 0, DRF_MORTAR_FLUX_UPWIND = 1, DRF_MORTAR_FLUX_LF = 2 };

typedef struct drf_mortar drf_mortar;

/* Operators of one connection type (MortarSpace::build_projection_operators,
 * src/dg/mortar.cpp:80), row-major, nm = (p+1)^2: M, Minv, Pc (nm x nm), Lc (nm x nm), Pf and Lf
 * (nfine x nm x nm). Any output may be NULL. */
int drf_mortar_ops(int order, int type, double *M, double *Minv, double *Pc, double *Lc, double *Pf,
                   double *Lf, int *nfine);

/* n_if interfaces: type[i], coarse_elem[i], coarse_face[i], and 4 slots per interface of
 * fine_elem / fine_face (the type's first 1..4 are used, in sub-face order of
 * compute_subface_bounds, src/dg/mortar.cpp:27). Elements index a state of n_elem x (p+1)^3
 * values (element-major, node i + (p+1)(j + (p+1)k)). */
int drf_mortar_create(int order, int64_t n_if, const int *type, const int64_t *coarse_elem,
                      const int *coarse_face, const int64_t *fine_elem, const int *fine_face,
                      int64_t n_elem, drf_mortar **out);
int drf_mortar_destroy(drf_mortar *h);
int drf_mortar_set_stream(drf_mortar *h, void *stream);

/* rhs += the mortar flux lifts of every interface, accumulated in interface order (coarse face,
 * then the fine faces), for the scalar field U and advection velocity a[3]. Host buffers. */
int drf_mortar_apply(drf_mortar *h, int flux_kind, const double *a, const double *U, double *rhs);
/* The same on device buffers, enqueued on the handle's stream. */
int drf_mortar_apply_device(drf_mortar *h, int flux_kind, const double *a, const double *d_U,
                            double *d_rhs);

/* ------------------------------------------------------------------ AMR mesh and faces
 * The face tables of a column-wise directionally refined mesh, as
 * OctreeAdapter::build_face_connections (src/mesh/octree_adapter.cpp:369) types them with
 * get_connection_type (include/dg/face_connection.hpp:110): nx x ny base columns over an
 * L x L basin (depth 1), column c = ix + nx iy split into 2^lx[c] x 2^ly[c] x 2^lz[c] cells
 * (levels 0..10, neighbouring columns 2:1 balanced). Outputs, in the order drf_amr_create takes
 * them:
 *  - elements grouped by level tuple; elem_level n_elem x 3, elem_box n_elem x (lo xyz, hi xyz);
 *  - conf n_conf x (e1, f1, e2, f2) conforming pairs and bnd n_bnd x (e, f) boundary faces;
 *  - n_if non-conforming interfaces grouped by type (1 Fine2x1, 2 Fine1x2, 5 Fine2x2): the
 *    coarse element and face, and up to 4 fine elements and faces (-1 padded) in the sub-face
 *    order of MortarSpace::compute_subface_bounds (src/dg/mortar.cpp:27).
 * Face f has its normal along axis f / 2, positive when f is odd. Call with null array outputs
 * to get the counts, then again with arrays of those sizes. Host-only (no device memory). */
int drf_amr_build_mesh(int nx, int ny, const int *lx, const int *ly, const int *lz, double L, int64_t *n_elem,
                       int64_t *n_conf, int64_t *n_bnd, int64_t *n_if, int *elem_level, double *elem_box,
                       int64_t *conf, int64_t *bnd, int *if_type, int64_t *if_coarse_elem, int *if_coarse_face,
                       int64_t *if_fine_elem, int *if_fine_face);

/* ------------------------------------------------------------------ AMR scalar DG
 * DG3DIntegration::compute_rhs (src/dg/operators_3d.cpp:228) for u_t + div(a u) = 0 with a
 * constant velocity a on a directionally refined hexahedral mesh of one order N (1..5), in the
 * reference's reference-coordinate form (identity Jacobian, :249-250): volume_integral (:81)
 * with N Gauss-Legendre points per direction, the mortar flux of every non-conforming face
 * (:345, once per coarse face), then the diagonal LGL mass inverse (:279). mode 0 is exactly
 * that (the reference leaves conforming and boundary faces as TODO, :262-268); mode 1 also
 * applies ConformingInterface::compute_flux (src/dg/mortar.cpp:320) and compute_boundary_flux
 * (:393, Outflow) with the collocated (N+1)-point LGL face weights.
 * conf: n_conf x (elem1, face1, elem2, face2) conforming pairs; bnd: n_bnd x (elem, face);
 * interfaces as drf_mortar_create (FaceConnection, include/dg/face_connection.hpp:51).
 * U, rhs: n_elem x (N+1)^3 element-major host arrays. flux: 0 central, 1 upwind, 2 LF. */
typedef struct drf_amr drf_amr;
int drf_amr_create(int order, int64_t n_elem, int64_t n_conf, const int64_t *conf, int64_t n_bnd,
                   const int64_t *bnd, int64_t n_if, const int *type, const int64_t *coarse_elem,
                   const int *coarse_face, const int64_t *fine_elem, const int *fine_face, drf_amr **out);
int drf_amr_destroy(drf_amr *h);
int drf_amr_set_stream(drf_amr *h, void *cuda_stream);
int drf_amr_sync(drf_amr *h);
/* rhs = compute_rhs(U) (U NULL: the handle's device state). */
int drf_amr_compute_rhs(drf_amr *h, int mode, int flux_kind, const double *a, const double *U, double *rhs);
int drf_amr_upload(drf_amr *h, const double *U);
int drf_amr_download(drf_amr *h, double *U);
/* nsteps of LSRK45 (LSRK45::step, src/solver/time_stepper.cpp:126) on du/dt = -compute_rhs(u)
 * of the device state, each step one CUDA graph (5 x (mortar face kernel; one kernel for the
 * volume, faces, mortar lifts and update)). */
int drf_amr_step(drf_amr *h, int mode, int flux_kind, const double *a, double dt, int nsteps);
/* Device time of one right-hand side (mean of nrep, CUDA events) and its algorithmic bytes. */
int drf_amr_time_rhs(drf_amr *h, int mode, int flux_kind, const double *a, int nrep, double *ms,
                     double *alg_bytes);

/* ------------------------------------------------------------------ AMR refinement
 * AdaptiveMeshRefinement::adapt (src/amr/refinement.cpp:422) on the column-wise refined meshes
 * above: estimate on the device, new levels on the host, the face tables rebuilt by
 * drf_amr_build_mesh, the state carried over on the device.
 *
 * GradientErrorEstimator::estimate (:44-68) with estimate_element (:70) and
 * compute_directional_mask (:95) of the handle's device state: value = (max - min of the
 * element's nodal values) x hchar (its characteristic length, cbrt of its volume, given per
 * element), normalised by the largest value when that exceeds 1e-14; flags bit 0 refine
 * (value > refine_threshold, default 0.1), bit 1 coarsen (value < coarsen_threshold, 0.01),
 * both 0 when not normalised; mask the RefineMask bits (X 1, Y 2, Z 4,
 * include/mesh/refine_mask.hpp:13) of the axes whose largest range along a node line exceeds
 * smoothness_factor (0.5) x the largest of the three, 0 below 1e-14. Host outputs. */
int drf_amr_estimate(drf_amr *h, const double *hchar, double refine_threshold, double coarsen_threshold,
                     double smoothness_factor, double *value, int32_t *mask, int32_t *flags);
/* mark_elements (:488) with can_refine / can_coarsen (:597-605), refine / coarsen, and the 2:1
 * balance of OctreeAdapter::balance (src/mesh/octree_adapter.cpp:138), per base column: a column
 * is refined along the union of its elements' Refine masks (XYZ for a Refine element without
 * one), else one level down along every axis above min_level when any element is marked
 * Coarsen; then neighbouring columns are raised until, across every face between columns, their
 * tangential and vertical levels differ by at most one and one side is at least as fine along
 * both (the meshes drf_amr_build_mesh accepts). Host-only. changed: the number of columns whose
 * levels changed. */
int drf_amr_refine_levels(int nx, int ny, const int *lx, const int *ly, const int *lz, int64_t n_elem,
                          const int32_t *mask, const int32_t *flags, int max_level, int min_level, int *new_lx,
                          int *new_ly, int *new_lz, int *changed);
/* transfer_solution (:532) and SolutionProjection (:217-343): the device state of `from`
 * (levels old_*) carried into `to` (levels new_*, each axis at most one level from the old):
 * per axis a node takes the old cell on its side, the parent's interpolant on a refined axis
 * (project_to_children) and the child on the node's side of 0 on a coarsened one
 * (project_from_children), evaluated by interpolate_3d (:345). Both handles of one order. */
int drf_amr_transfer(drf_amr *from, drf_amr *to, int nx, int ny, const int *old_lx, const int *old_ly,
                     const int *old_lz, const int *new_lx, const int *new_ly, const int *new_lz);

#ifdef __cplusplus
}
#endif
#endif /* DRIFTER_B200_H */

/* zb.h -- C ABI of the B200 DFR residual library (libzefr_b200.so).
 *
 * This is the drop-in boundary for ZEFR's residual hot path: the explicit
 * Direct Flux Reconstruction residual that FRSolver::compute_residual builds
 * (reference include/solver.hpp:152, src/solver.cpp:1494-1645) and the
 * explicit RK stepping around it (include/solver.hpp:158-190,
 * src/solver.cpp:2864-3097).  The reference exposes these as C++ methods
 * (FRSolver, Zefr, namespace zefr:: in include/zefr_interface.hpp:89-159);
 * here they are plain C entry points taking pointers, sizes and strides, so a
 * C++ FRSolver shim, ctypes, cgo or JNI can bind them alike.
 *
 * Conventions
 *  - Every entry point returns zb_status; 0 is success.  No C++ exception
 *    crosses this boundary.  zb_last_error() describes the last failure on the
 *    calling thread (the reference throws std::runtime_error with file:line,
 *    include/macros.hpp:52-54).
 *  - A zb_plan is host-only set-up (mesh connectivity, operators, metrics);
 *    building one needs no GPU.  A zb_ctx owns device memory on the device
 *    current at zb_create time and one CUDA stream.
 *  - Host buffers passed in are borrowed for the duration of the call.
 *  - State and residual arrays are addressed with explicit element, variable
 *    and solution-point strides, the convention of zefr::get_q_spts
 *    (include/zefr_interface.hpp:126-129, src/zefr.cpp:607-645).
 *  - One context per host thread (or per stream); calls on one context are
 *    not thread-safe.
 */
#ifndef ZB_H
#define ZB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int zb_status;

enum {
  ZB_OK = 0,
  ZB_ERR_ARG = -1,          /* invalid argument or size */
  ZB_ERR_CUDA = -2,         /* CUDA runtime error */
  ZB_ERR_MESH = -3,         /* malformed mesh, unpaired periodic face, negative Jacobian */
  ZB_ERR_UNSUPPORTED = -4,  /* element type / order / option not built */
  ZB_ERR_NONFINITE = -5,    /* NaN or Inf found in state or residual */
  ZB_ERR_NOMEM = -6,        /* device or host allocation failed */
  ZB_ERR_INTERNAL = -7
};

/* Boundary conditions: same meaning and numbering as the reference BC_TYPE
 * enum (include/input.hpp:54-70). */
enum {
  ZB_BC_NONE = 0,
  ZB_BC_PERIODIC = 1,
  ZB_BC_CHAR = 2,
  ZB_BC_SUP_IN = 3,
  ZB_BC_SUP_OUT = 4,
  ZB_BC_SLIP_WALL = 5,
  ZB_BC_ISOTHERMAL_NOSLIP = 6,
  ZB_BC_ADIABATIC_NOSLIP = 7,
  ZB_BC_ISOTHERMAL_NOSLIP_MOVING = 8,
  ZB_BC_ADIABATIC_NOSLIP_MOVING = 9,
  ZB_BC_SYMMETRY = 11
};

/* Common convective flux (reference FC_TYPE, include/input.hpp:28-31, plus Roe). */
enum { ZB_FLUX_RUSANOV = 0, ZB_FLUX_ROE = 2 };

/* Arithmetic of the residual.
 *  ZB_FP64:  FP64 storage and arithmetic (the form checked against the
 *            reference).
 *  ZB_MIXED: FP32 state (stored as deviations from its mean), traces, metrics,
 *            residual and pointwise arithmetic, with the inviscid flux
 *            evaluated as a deviation from the reference state; FP64 for the
 *            set-up (metrics, operators) and for the norm and functional
 *            reductions; Kahan-compensated RK accumulation. */
enum { ZB_FP64 = 0, ZB_MIXED = 1 };

/* Where a buffer lives. */
enum { ZB_HOST = 0, ZB_DEVICE = 1 };

/* Kernel ids for zb_profile_read. */
enum {
  ZB_K_EXTRAP = 0,     /* state -> flux points */
  ZB_K_EULER = 1,      /* Euler volume + common flux + divergence (+RK) */
  ZB_K_NS_GRAD = 2,    /* NS common solution, gradient, flux, volume divergence */
  ZB_K_NS_FACE = 3,    /* NS common flux + surface correction (+RK) */
  ZB_K_TO_TILES = 4,   /* state import */
  ZB_K_FROM_TILES = 5, /* state / residual export */
  ZB_K_NORMS = 6,      /* FP64 residual norms */
  ZB_K_ADJ_LIFT = 7,   /* adjoint: residual weight -> surface flux weight */
  ZB_K_ADJ_VOL = 8,    /* adjoint: volume + face fluxes (+ gradient, NS) */
  ZB_K_ADJ_TRACE = 9,  /* adjoint NS: common solution -> traces -> state */
  ZB_K_FUNCTIONALS = 10,
  ZB_NKERNELS = 11
};

typedef struct zb_mesh {
  int ndims;                 /* 2 or 3 */
  int gmsh_type;             /* volume element: 2 tri3, 3 quad4, 10 quad9, 5 hex8 */
  int64_t n_nodes;
  const double *coords;      /* [n_nodes][3] */
  int64_t n_eles;
  int nodes_per_ele;
  const int64_t *ele2nodes;  /* [n_eles][nodes_per_ele], zero-based, gmsh node order */
  int64_t n_bnd_faces;
  int nodes_per_face;        /* nodes listed per boundary face (corner nodes first) */
  const int64_t *face_nodes; /* [n_bnd_faces][nodes_per_face], zero-based */
  const int *face_bc;        /* [n_bnd_faces] ZB_BC_* */
} zb_mesh;

/* Physical and numerical parameters.  Field meanings follow the reference
 * InputStruct after read_input_file / apply_nondim (src/input.cpp:31-539);
 * zb_params_from_deck() performs that computation from deck-style inputs. */
typedef struct zb_params {
  int order;          /* polynomial order P */
  int viscous;        /* 0 Euler, 1 Navier-Stokes (LDG) */
  int fconv;          /* ZB_FLUX_* */
  int precision;      /* ZB_FP64 or ZB_MIXED */
  double gamma, prandtl, mu, rt, c_sth;
  int fix_vis;        /* 1: constant mu; 0: Sutherland */
  double rus_k, ldg_b, ldg_tau;
  double rho_fs, V_fs[3], P_fs;
  double T_wall, R_ref, V_wall[3];
  double dt;          /* RK time step */
  int tri_volume_div; /* triangles: 0 = the reference's operators, whose oppDiv
                         lacks the volume-divergence term (src/elements.cpp:
                         609-623 builds it for quads/hexes only); 1 = include it */
  int tensor_ops;     /* mixed form, triangles, Navier-Stokes: 1 = the gradient
                         kernel's dense operator products on the tensor pipe
                         (tcgen05, TF32x3 split products, FP32 accumulation);
                         0 = on CUDA cores (FP32 FMA).  No reference
                         counterpart (its products are GiMMiK or cuBLAS). */
} zb_params;

/* Deck-style inputs for zb_params_from_deck (reference keys, src/input.cpp). */
typedef struct zb_deck {
  int ndims, order, viscous, fconv, precision;
  int disable_nondim, fix_vis;
  double gamma, prandtl, R, S, T_gas, rho_fs, P_fs, mach_fs, Re_fs, L_fs, T_fs;
  double nx_fs, ny_fs, nz_fs;
  double mach_wall, T_wall, nx_wall, ny_wall, nz_wall;
  double rus_k, ldg_b, ldg_tau, dt;
} zb_deck;

typedef struct zb_info {
  int ndims, nvars, nspts, nfpts, order, etype;  /* etype: 1 tri, 2 quad, 4 hex (reference ELE_TYPE) */
  int64_t n_eles, n_eles_pad, n_gfpts, n_gfpts_int, n_gfpts_bnd;
  int nstages;
  int tile;           /* elements per layout tile */
  int precision;
} zb_info;

typedef struct zb_plan zb_plan;
typedef struct zb_ctx zb_ctx;

/* Error text for the last failing call on this thread. */
const char *zb_last_error(void);

/* Library version string. */
const char *zb_version(void);

/* Fill reference-style parameters (reference src/input.cpp:463-539). */
zb_status zb_params_from_deck(const zb_deck *deck, zb_params *out);

/* Read a gmsh 2.2 ASCII mesh (reference src/geometry.cpp:307-957).
 * names/bcs map boundary physical names (case-insensitive) to ZB_BC_* like the
 * deck's mesh_bound lines.  The returned mesh is freed with zb_mesh_free. */
zb_status zb_mesh_read_gmsh(const char *path, int ndims, int n_map, const char *const *names,
                            const int *bcs, zb_mesh **out);
void zb_mesh_free(zb_mesh *mesh);

/* Host-side set-up: connectivity (reference src/geometry.cpp:1159-1744,
 * src/solver.cpp:312-437), operators (src/elements.cpp:555-810) and metrics
 * (src/elements.cpp:325-407, 845-996).  No GPU needed. */
zb_status zb_plan_create(const zb_mesh *mesh, const zb_params *params, zb_plan **out);
void zb_plan_free(zb_plan *plan);
zb_status zb_plan_info(const zb_plan *plan, zb_info *out);

/* Copy a named set-up array out in the reference's own layout (for checking
 * set-up against the reference).  Names: coord_spts, jaco_det_spts,
 * inv_jaco_spts, oppE, oppD, oppD_fpts, oppDiv, oppDiv_fpts, fpt_partner
 * (partner element*nfpts+fpt per element fpt, -1-bc on boundaries),
 * fpt_slot, fpt_norm (left-element normal per element fpt [fpt][dim][ele]),
 * fpt_dA, coord_fpts, weights_spts, loc_spts, loc_fpts, tnorm ([fpt][dim]
 * reference normals), dshape_spts [dim][spt][node], dshape_fpts
 * [dim][fpt][node], shape_fpts [fpt][node], shape_spts [spt][node] (shape
 * functions, gmsh node order; for geometry derivatives), nodes
 * [node][dim][ele] (element node coordinates, Elements::nodes).  With
 * out == NULL, *n receives the array's length. */
zb_status zb_plan_get(const zb_plan *plan, const char *name, double *out, int64_t *n);

/* Create a device context from a plan on the current device: the device side
 * of FRSolver::setup (src/solver.cpp:55-437, include/solver.hpp:150), which
 * allocates and fills the solver's arrays; zb_destroy releases them. */
zb_status zb_create(const zb_plan *plan, zb_ctx **out);
/* Convenience: mesh + params -> plan -> context. */
zb_status zb_create_from_mesh(const zb_mesh *mesh, const zb_params *params, zb_ctx **out);
void zb_destroy(zb_ctx *ctx);
zb_status zb_info_get(const zb_ctx *ctx, zb_info *out);

/* Use a caller-provided CUDA stream (cudaStream_t) for all later work.  No
 * reference counterpart (the reference launches on its own streams). */
zb_status zb_set_stream(zb_ctx *ctx, void *stream);
/* The fixed time step: the deck's dt (src/input.cpp:74, InputStruct::dt). */
zb_status zb_set_dt(zb_ctx *ctx, double dt);

/* State access with the strides of zefr::get_q_spts / get_q_spts_d
 * (include/zefr_interface.hpp:126-129, src/zefr.cpp:607-645), in doubles.
 * where: ZB_HOST/ZB_DEVICE.  zb_set_state copies and converts into the
 * context's layout and precision. */
zb_status zb_set_state(zb_ctx *ctx, const double *U, int64_t spt_stride, int64_t var_stride,
                       int64_t ele_stride, int where);
zb_status zb_get_state(zb_ctx *ctx, double *U, int64_t spt_stride, int64_t var_stride,
                       int64_t ele_stride, int where);

/* FRSolver::compute_residual(stage) (include/solver.hpp:152,
 * src/solver.cpp:1494-1645): divF_spts(stage) = |J| * div F in reference
 * form (physical residual is -divF/|J|); zb_get_residual reads that register
 * (Elements::divF_spts, include/elements.hpp:91) with caller strides. */
zb_status zb_compute_residual(zb_ctx *ctx, unsigned stage);
zb_status zb_get_residual(zb_ctx *ctx, unsigned stage, double *out, int64_t spt_stride,
                          int64_t var_stride, int64_t ele_stride, int where);

/* divF_spts(stage) for n states held in host memory: for each i,
 * zb_set_state(U[i]) + zb_compute_residual(stage) + zb_get_residual(stage,
 * divF[i]), with U[i] and divF[i] dense in the reference layout
 * [nspts][nvars][n_eles] (the layout of zefr::get_q_spts with its default
 * strides, include/zefr_interface.hpp:126-129, around FRSolver::
 * compute_residual, include/solver.hpp:152).  The copies of state i+1 to the
 * device and of residual i-1 to the host overlap the computation of residual
 * i (one copy engine each way, two staging buffers each way, allocated on the
 * first call and kept by the context); with pinned host buffers the
 * copies run asynchronously, with pageable ones they still complete but
 * overlap less.  Returns once every residual is in host memory; the context
 * then holds state U[n-1] and its residual. */
zb_status zb_compute_residuals_host(zb_ctx *ctx, unsigned stage, int n, const double *const *U, double *const *divF);

/* One RK44 stage of FRSolver::step_RK (src/solver.cpp:2864-3097): residual of
 * stage s, then U = U_ini - a_s dt/|J| divF_s, or on the last stage
 * U = U_ini - sum_s b_s dt/|J| divF_s.  Stage 0 first saves U_ini. */
zb_status zb_rk_stage(zb_ctx *ctx, unsigned stage);
/* The residual and the RK44 stage in three parts, for callers that interleave
 * their own work (the reference's exchange and overset steps) between them:
 * FRSolver::compute_residual_start / _mid / _finish (include/solver.hpp:
 * 153-155, src/solver.cpp:1647-1829) and step_RK_stage_start / _mid /
 * _finish (src/solver.cpp:3696-3760; Zefr::do_rk_stage_start/mid/finish,
 * src/zefr.cpp:372-430).  start extrapolates the state to the flux points;
 * mid (Navier-Stokes) forms the common solution, corrected gradient, fluxes
 * and volume divergence; finish forms the common fluxes and surface
 * correction and, for a stage, applies the RK update.  Called in that order
 * for one stage they equal zb_compute_residual / zb_rk_stage; any other order
 * returns ZB_ERR_ARG and resets the sequence, and zb_set_state,
 * zb_compute_residual and zb_rk_stage reset it too. */
zb_status zb_compute_residual_start(zb_ctx *ctx, unsigned stage);
zb_status zb_compute_residual_mid(zb_ctx *ctx, unsigned stage);
zb_status zb_compute_residual_finish(zb_ctx *ctx, unsigned stage);
zb_status zb_rk_stage_start(zb_ctx *ctx, unsigned stage);
zb_status zb_rk_stage_mid(zb_ctx *ctx, unsigned stage);
zb_status zb_rk_stage_finish(zb_ctx *ctx, unsigned stage);

/* n time steps of FRSolver::update (src/solver.cpp:2600-2660): RK44
 * (step_RK) by default, or the scheme set with zb_set_time_scheme. */
zb_status zb_step(zb_ctx *ctx, int n);

/* Time integration options of the reference deck (dt_scheme, dt_type, CFL,
 * CFL_type, adapt_dt and its controller keys; src/input.cpp:72-127).
 *  - scheme ZB_RK44: step_RK (src/solver.cpp:2864-3097); with dt_type != 0
 *    the time step is the CFL estimate of compute_element_dt
 *    (src/solver.cpp:4105-4272) from the state at the start of the step:
 *    dt_type 1 the global minimum, 2 one step per element.
 *  - scheme ZB_RK54: five-stage low-storage RK (step_LSRK, src/solver.cpp:
 *    3100-3255; coefficients src/solver.cpp:749-777) at the fixed dt, or with
 *    adapt_dt the embedded error estimate and PI controller of
 *    step_adaptive (src/solver.cpp:2663-2757): max over points of
 *    |err| / (atol + rtol max(|U|, |U_ini|)), factor
 *    err^(-pi_alpha/4) prev_err^(pi_beta/4) clamped by safety, min_factor and
 *    max_factor, dt capped at max_dt; a step whose error is >= 1 is redone from
 *    its start state with the new dt.
 * CFL_type 1: dt = 2 CFL c_adv(P) vol / sum_fpt w dA waveSp; CFL_type 2:
 * per direction max over the face points of waveSp / (c_adv h) (+ diffCo /
 * (c_diff h^2) for Navier-Stokes), dt = CFL / sum over directions.  waveSp is
 * max(|Vn| + a) over the two sides of the point (the reference's Rusanov wave
 * speed, also used with the Roe flux), diffCo max(mu/rho, gamma mu/(Pr rho)).
 * Quadrilaterals and hexahedra; dt_type != 0 is refused for triangles. */
enum { ZB_RK44 = 0, ZB_RK54 = 1 };
typedef struct zb_time_scheme {
  int scheme;         /* ZB_RK44 or ZB_RK54 */
  int dt_type;        /* 0 fixed dt (zb_params.dt / zb_set_dt), 1 CFL global, 2 CFL local */
  int cfl_type;       /* 1 or 2 */
  double cfl;
  int adapt_dt;       /* ZB_RK54 only */
  double atol, rtol, pi_alpha, pi_beta, safety, max_factor, min_factor, max_dt;
} zb_time_scheme;
/* Deck defaults (src/input.cpp:72-127): RK44, dt_type 0, CFL 1, CFL_type 1,
 * err_atol = err_rtol = 1e-5, pi_alpha 0.7, pi_beta 0.4, safety_factor 0.8,
 * max_factor 2.5, min_factor 0.3, max_dt 100. */
void zb_time_scheme_defaults(zb_time_scheme *out);
zb_status zb_set_time_scheme(zb_ctx *ctx, const zb_time_scheme *ts);
/* After zb_step: the reference's dt(0) -- the fixed step, the last CFL step
 * (element 0's under dt_type 2) or, with adapt_dt, the step the next step
 * starts from -- the last accepted error estimate, the number of rejected
 * steps so far and the flow time (sum of the steps' dt(0)). */
zb_status zb_time_state(zb_ctx *ctx, double *dt, double *prev_err, int64_t *rejected, double *flow_time);
/* Per-element time step of the last CFL estimate (dt_type != 0), [n_eles]. */
zb_status zb_get_element_dt(zb_ctx *ctx, double *out);

/* Residual norms of report_residuals (src/solver.cpp:6990-7137), FP64 device
 * reduction of divF(stage 0)/|J| per variable, each divided by nspts * n_eles
 * as the reference prints them: out[0..nvars) = max |.| (res_type 0),
 * out[nvars..2 nvars) = sum |.| (res_type 1), out[2 nvars..3 nvars) =
 * sqrt(sum of squares) (res_type 2). */
zb_status zb_residual_norms(zb_ctx *ctx, double *out);

/* Volume integrals of FRSolver::report_turbulent_stats (src/solver.cpp:
 * 7813-7917) in FP64 over the current state: out[0] = integral of
 * 1/2 rho |u|^2, out[1] = integral of 1/2 rho |curl u|^2 (Navier-Stokes only:
 * the gradient is evaluated with the LDG corrected gradient of the residual),
 * out[2] = domain volume.  The reference prints out[0..1] / (out[2] rho_fs
 * |V_fs|^2). */
zb_status zb_functionals(zb_ctx *ctx, double *out);

/* Force and moment on the wall boundaries (slip, isothermal and adiabatic
 * walls) of FRSolver::compute_moments (src/solver.cpp:7600-7811), FP64
 * device reduction over the current state: out[0..2] force, out[3..5]
 * moment about the origin.  Per wall flux point w (P n - tau n) dA with the
 * element's own trace and extrapolated corrected gradient; in 3D each flux
 * point's own state is used where the reference reads flux point 0's
 * (src/solver.cpp:7716-7720). */
zb_status zb_wall_force(zb_ctx *ctx, double *out);

/* Replace the free-stream state the far-field and characteristic boundaries
 * prescribe (input rho_fs, V_fs, P_fs of the reference, src/input.cpp:463-539
 * after non-dimensionalisation); takes effect from the next launch.  Used to
 * differentiate with respect to the free-stream conditions.  No reference
 * counterpart (the reference fixes them at set-up). */
zb_status zb_set_freestream(zb_ctx *ctx, double rho_fs, const double *V_fs, double P_fs);

/* zb_vjp plus the adjoint with respect to the geometry the residual is built
 * on, in the layouts zb_plan_get exports (host arrays, FP64):
 * inv_jaco_bar [D][S][D][E] and jaco_det_bar [S][E] (adjugate and |J| at
 * solution points), norm_bar [Fp][D][E] and dA_bar [Fp][E] (face unit normal
 * and own face area factor at flux points).  A face's normal is the left
 * element's (the right element stores a copy), so its whole adjoint is
 * reported at the left element's flux point and zero at the right one's.
 * For Navier-Stokes the call first evaluates the residual of the current
 * state into register 0.  No reference counterpart. */
zb_status zb_vjp_geometry(zb_ctx *ctx, const double *lam, double *Ubar, int64_t spt_stride, int64_t var_stride,
                          int64_t ele_stride, int where, double *param_bar, double *inv_jaco_bar,
                          double *jaco_det_bar, double *norm_bar, double *dA_bar);

/* zb_vjp that also adds the geometry adjoint to sums kept on the device
 * (for unsteady adjoints, one call per RK stage without host copies);
 * zb_geometry_adjoint_get copies the sums out in the zb_vjp_geometry layouts
 * and, with reset != 0, clears them.  No reference counterpart. */
/* Reverse of one RK44 step U1 = step(U0) of FRSolver::step_RK (plain FP64
 * form), for unsteady adjoints: given the step's start state U0 and the
 * adjoint Ubar1 of its end state, Ubar0 = (d U1 / d U0)^T Ubar1, with the
 * four stage states and residuals recomputed on the device (RK44 tables of
 * src/solver.cpp:722-735).  param_bar (host,
 * 5 values, may be NULL) gets the free-stream adjoint added; with geometry
 * != 0 the metric adjoint of the stage residuals and of the update's 1/|J|
 * is added to the device sums zb_geometry_adjoint_get reads.  Uses the
 * context's fixed dt (zb_set_dt; ZB_ERR_UNSUPPORTED under RK54 or a CFL
 * step); leaves the context's state undefined.  No reference
 * counterpart. */
zb_status zb_rk_step_vjp(zb_ctx *ctx, const double *U0, const double *Ubar1, double *Ubar0, int64_t spt_stride,
                         int64_t var_stride, int64_t ele_stride, int where, double *param_bar, int geometry);

/* Element geometry from element node coordinates, on the device: the set-up's
 * calc_transforms and calc_normals (src/elements.cpp:845-996; GPU forms
 * src/elements_kernels.cu:1649-1737, 1896-1950).  nodes[nNodes][D][E] is the
 * reference's Elements::nodes layout (zb_plan_get "nodes"); outputs in the
 * zb_vjp_geometry layouts: inv_jaco[D][S][D][E] (adjugate), jaco_det[S][E],
 * norm[Fp][D][E] (the left element's unit normal on both sides of a face),
 * dA[Fp][E] (each side's own).  For the context's own nodes the results
 * equal the set-up's bit for bit.  Every pointer is host or device memory as
 * `where` says.  No reference counterpart as an entry point. */
zb_status zb_geometry_eval(zb_ctx *ctx, const double *nodes, double *inv_jaco, double *jaco_det, double *norm,
                           double *dA, int where);
/* Adjoint of zb_geometry_eval at `nodes`: nodes_bar[nNodes][D][E] from the
 * adjoints of the four arrays (as zb_vjp_geometry / zb_geometry_adjoint_get
 * return them; a NULL adjoint counts as zero).  Deterministic. */
zb_status zb_geometry_eval_vjp(zb_ctx *ctx, const double *nodes, const double *inv_jaco_bar,
                               const double *jaco_det_bar, const double *norm_bar, const double *dA_bar,
                               double *nodes_bar, int where);
/* Moves the context's mesh: new element node coordinates (same layout) give
 * new metrics on the device in the context's precision form, with the
 * coordinates, volumes and CFL line lengths that depend on them; the state,
 * the connectivity and the plan handle are unchanged.  The role of the
 * reference's moving-grid metric updates (update_transforms_rigid_wrapper,
 * src/elements_kernels.cu:1840-1895) for arbitrary node motion.
 * ZB_ERR_MESH (context unchanged) if a solution point's |J| turns negative. */
zb_status zb_set_nodes(zb_ctx *ctx, const double *nodes, int where);

zb_status zb_vjp_geometry_accumulate(zb_ctx *ctx, const double *lam, double *Ubar, int64_t spt_stride,
                                     int64_t var_stride, int64_t ele_stride, int where, double *param_bar);
zb_status zb_geometry_adjoint_get(zb_ctx *ctx, double *inv_jaco_bar, double *jaco_det_bar, double *norm_bar,
                                  double *dA_bar, int reset);

/* ---- Batched stepping of independent cases ----
 * Many Euler cases on quadrilaterals (each its own context: mesh, order
 * P1-P5, state, dt) advance together: one persistent launch per RK stage
 * covers every tile of every case, and the four stages of a step replay as
 * one CUDA graph.  The contexts stay owned by the caller and must outlive the
 * batch; do not use them while batched work is queued (zb_batch_synchronize
 * first).  No reference counterpart (the reference steps one mesh). */
typedef struct zb_batch zb_batch;
typedef struct zb_batch_config {
  int threads;        /* threads per CTA: 64, 128 or 256 */
  int blocks_per_sm;  /* persistent CTAs per SM */
  int order;          /* work order: 0 by polynomial order (costliest first), 1 case-major */
  double ms_per_step; /* autotuner: measured time of one RK44 step */
  int group;          /* threads per tile group (64, 128 or 256, dividing threads): a CTA
                         runs threads/group tiles at once */
  int chunk;          /* consecutive work items a group takes at a time; 0: one
                         contiguous run per group */
  int fused;          /* 1: one persistent kernel per stage for all orders (each
                         item dispatches to its order's tile body; registers and
                         shared memory of the largest order present); 0: one
                         kernel per order present, run concurrently */
} zb_batch_config;

zb_status zb_batch_create(zb_ctx *const *ctxs, int n, zb_batch **out);
void zb_batch_destroy(zb_batch *batch);
/* Time every launch shape on `steps` steps from the current states (which are
 * restored afterwards) and keep the fastest; *chosen may be NULL. */
zb_status zb_batch_autotune(zb_batch *batch, int steps, zb_batch_config *chosen);
/* As zb_batch_autotune over the shapes of one form only: form 0 keeps one
 * kernel per order present, form 1 one kernel per stage for all orders, -1
 * either (zb_batch_autotune).  The chosen shape is installed. */
zb_status zb_batch_autotune_form(zb_batch *batch, int steps, int form, zb_batch_config *chosen);
zb_status zb_batch_set_config(zb_batch *batch, const zb_batch_config *cfg);
/* nsteps RK44 steps of every case; use_graph = 1 replays the captured graph,
 * 0 launches the four stages directly.  Returns once queued. */
zb_status zb_batch_step(zb_batch *batch, int nsteps, int use_graph);
/* One RK stage of every case (completes before returning). */
zb_status zb_batch_stage(zb_batch *batch, unsigned stage);
zb_status zb_batch_synchronize(zb_batch *batch);
int64_t zb_batch_launch_count(const zb_batch *batch);

/* Adjoint (vector-Jacobian product) of the residual at the current state:
 * Ubar = (d divF / d U)^T lam, both in the strided layout of zb_set_state,
 * divF as zb_compute_residual computes it.  param_bar, when not NULL,
 * receives d (lam . divF) / d (rho_fs, V_fs[0..2], P_fs), the free-stream
 * state the far-field and characteristic boundaries prescribe (5 doubles).
 * Plain FP64 contexts only; quadrilaterals P1-P5, hexahedra P1-P3 and
 * triangles P1-P8 (the geometry adjoint of zb_vjp_geometry: quadrilaterals
 * and hexahedra).
 * No reference counterpart: the reference has no adjoint. */
zb_status zb_vjp(zb_ctx *ctx, const double *lam, double *Ubar, int64_t spt_stride, int64_t var_stride,
                 int64_t ele_stride, int where, double *param_bar);

/* Wait for all work queued on the context's stream.  No reference
 * counterpart (its calls synchronise internally). */
zb_status zb_synchronize(zb_ctx *ctx);

/* Number of kernels this library launched on the context since creation.
 * No reference counterpart. */
int64_t zb_launch_count(const zb_ctx *ctx);

/* Per-kernel device timing with CUDA events recorded on the context's stream
 * around every launch (no reference counterpart; the reference brackets
 * stages with std::chrono timers, include/inputstruct.hpp:35-95).
 * zb_profile_read synchronises, returns total milliseconds and launch counts
 * per ZB_K_* id accumulated since the last read, and resets them. */
zb_status zb_profile_enable(zb_ctx *ctx, int on);
zb_status zb_profile_read(zb_ctx *ctx, double *ms, int64_t *count);
const char *zb_kernel_name(int id);

/* Operator product on the tensor pipe: C = alpha A B + beta C with A [m][k]
 * (row stride lda) a small constant operator and B [k][n] (row stride ldb),
 * C [m][n] (row stride ldc), all FP32 device arrays; n is the element count
 * times the variables, as in the reference's products (B = U_spts viewed as
 * [nSpts][nVars * nEles]).  Replaces gimmik_mm_gpu (include/gimmik.h:5-22,
 * src/gimmik_gpu.cu:31183-31577), same argument order, in FP32 instead of
 * FP64.  tcgen05 MMAs with the operands split into TF32 parts
 * (A_hi B_hi + A_hi B_lo + A_lo B_hi, FP32 accumulation in tensor memory),
 * about FP32 accuracy.  m <= 256 and the operator (m x k) must fit in shared
 * memory.  Queued on `stream` (NULL: the default stream) without waiting; a
 * product whose tensor-core completion wait timed out (it sets a flag and
 * leaves C unfinished) is reported as ZB_ERR_CUDA by the next call. */
zb_status zb_operator_mm_tf32x3(int m, int n, int k, float alpha, const float *a, int lda, const float *b, int ldb,
                                float beta, float *c, int ldc, void *stream);

/* FP64 residual divF_spts = |J| div F for callers that cannot allocate device
 * memory.  No counterpart in the reference (its residual lives in FRSolver's
 * own allocated arrays).
 *
 * U and divF are device pointers the caller owns, dense in the reference
 * layout [nspts][nvars][n_eles].  Every intermediate lives in one file-scope
 * device array of 32 MiB that each GPU loading this library holds until the
 * process exits; meshes whose geometry and intermediates exceed it are
 * rejected with ZB_ERR_ARG and a message giving the bytes needed.  The call
 * itself allocates nothing: it copies the plan's geometry from host memory
 * into that array, packs it, and runs the same kernels as
 * zb_compute_residual on `stream` (a cudaStream_t, or NULL for the default
 * stream), returning without synchronising.
 * Every call copies the plan's geometry (adjugate, |J|, normals, dA,
 * connectivity) from the plan's pageable host arrays: a few bytes per
 * solution and flux point over PCIe, on top of the residual's own work.
 * The first call on each device looks up the array's device address, with
 * that device current.  Do not record calls into a CUDA graph: the host
 * copies read the plan's host memory at the time of the call.
 * All calls share the array: calls whose work overlaps on the GPU (other
 * streams, other host threads, other plans) race on it. */
zb_status zb_compute_residual_noalloc(const zb_plan *plan, const double *U, double *divF, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* ZB_H */

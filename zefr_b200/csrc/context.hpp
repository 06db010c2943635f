// Device context of the DFR residual (opaque zb_ctx of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <memory>

#include "zb_internal.hpp"

struct zb_plan
{
  zb::Plan plan;
};

namespace zb {

struct Ctx;

Ctx *ctx_create(const Plan &plan);
void ctx_destroy(Ctx *c);
void ctx_info(const Ctx *c, zb_info *out);
void ctx_set_stream(Ctx *c, void *stream);
void ctx_set_dt(Ctx *c, double dt);
void ctx_set_freestream(Ctx *c, double rho_fs, const double *V_fs, double P_fs);
void ctx_set_state(Ctx *c, const double *U, int64_t ss, int64_t vs, int64_t es, int where);
void ctx_get_state(Ctx *c, double *U, int64_t ss, int64_t vs, int64_t es, int where);
void ctx_compute_residual(Ctx *c, unsigned stage);
void ctx_get_residual(Ctx *c, unsigned stage, double *out, int64_t ss, int64_t vs, int64_t es, int where);
void ctx_residuals_host(Ctx *c, unsigned stage, int n, const double *const *U, double *const *R);
void ctx_rk_stage(Ctx *c, unsigned stage);
// C = alpha A B + beta C on the tensor pipe (TF32x3, tc_opmm.cu), queued on st
void opmm_tc(int m, int n, int k, float alpha, const float *a, int lda, const float *b, int ldb, float beta, float *c,
             int ldc, cudaStream_t st, volatile int *err_host, int *err_dev, int max_ctas = 0);
size_t opmm_tc_smem_bytes(int m, int k);
// part 0 start, 1 mid, 2 finish; rk: the RK44 stage rather than the residual alone
void ctx_residual_split(Ctx *c, unsigned stage, int part, int rk);
void ctx_step(Ctx *c, int n);
// time integration (time_scheme.cu)
void ctx_set_time_scheme(Ctx *c, const zb_time_scheme *ts);
void ctx_time_state(Ctx *c, double *dt, double *prev_err, int64_t *rejected, double *flow_time);
void ctx_get_element_dt(Ctx *c, double *out);
void ctx_step_scheme(Ctx *c, int n);  // zb_step with the context's time scheme
void ctx_refresh_cfl_geometry(Ctx *c);  // after the mesh moved
// geometry from element node coordinates (geometry.cu)
void ctx_geometry_eval(Ctx *c, const double *nodes, double *inv_jaco, double *jaco_det, double *norm, double *dA,
                       int where);
void ctx_geometry_eval_vjp(Ctx *c, const double *nodes, const double *inv_jaco_bar, const double *jaco_det_bar,
                           const double *norm_bar, const double *dA_bar, double *nodes_bar, int where);
void ctx_set_nodes(Ctx *c, const double *nodes, int where);
// CFL limits of the upwinded advection and LDG diffusion operators per order
// (reference get_cfl_limit_adv / get_cfl_limit_diff, src/funcs.cpp:435-560)
double cfl_limit_adv(int order);
double cfl_limit_diff(int order, double beta);
void ctx_norms(Ctx *c, double *out);
void ctx_sync(Ctx *c);
int64_t ctx_launches(const Ctx *c);
void ctx_profile_enable(Ctx *c, int on);
void ctx_functionals(Ctx *c, double *out);
void ctx_wall_force(Ctx *c, double *out);
void ctx_vjp(Ctx *c, const double *lam, double *Ubar, int64_t ss, int64_t vs, int64_t es, int where,
             double *param_bar, double *inv_jaco_bar = nullptr, double *jaco_det_bar = nullptr,
             double *norm_bar = nullptr, double *dA_bar = nullptr, bool accumulate = false);
// reverse of one RK44 step with recomputed stages (zb_rk_step_vjp)
void ctx_rk_step_vjp(Ctx *c, const double *U0, const double *Ubar1, double *Ubar0, int64_t ss, int64_t vs,
                     int64_t es, int where, double *param_bar, bool geometry);
void ctx_geometry_adjoint_get(Ctx *c, double *inv_jaco_bar, double *jaco_det_bar, double *norm_bar, double *dA_bar,
                              int reset);
void ctx_profile_read(Ctx *c, double *ms, int64_t *count);
void noalloc_residual(const Plan &p, const double *U, double *divF, cudaStream_t st);

struct Batch;
Batch *batch_create(Ctx *const *ctxs, int n);
void batch_destroy(Batch *b);
void batch_autotune(Batch *b, int steps, int form, zb_batch_config *out);
void batch_config(Batch *b, const zb_batch_config *cfg);
void batch_step(Batch *b, int nsteps, int use_graph);
void batch_stage(Batch *b, unsigned stage);
void batch_sync(Batch *b);
int64_t batch_launches(const Batch *b);

}  // namespace zb

struct zb_ctx
{
  zb::Ctx *impl;
};

struct zb_batch
{
  zb::Batch *impl;
};

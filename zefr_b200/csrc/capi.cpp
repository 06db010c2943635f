// extern "C" boundary of libzefr_b200.so (declarations in include/zb.h).
// Every C++ exception is caught here and turned into a status code plus a
// thread-local message, the C-ABI analogue of the reference's ThrowException
// (include/macros.hpp:52-54).
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <vector>
#include <string>

#include "context.hpp"

namespace zb {

static thread_local std::string g_err;

void set_last_error(const std::string &msg) { g_err = msg; }

}  // namespace zb

#define ZB_GUARD(...)                               \
  try                                               \
  {                                                 \
    __VA_ARGS__;                                    \
    return ZB_OK;                                   \
  }                                                 \
  catch (const zb::Error &e)                        \
  {                                                 \
    zb::set_last_error(e.what());                   \
    return e.code;                                  \
  }                                                 \
  catch (const std::bad_alloc &)                    \
  {                                                 \
    zb::set_last_error("host allocation failed");   \
    return ZB_ERR_NOMEM;                            \
  }                                                 \
  catch (const std::exception &e)                   \
  {                                                 \
    zb::set_last_error(e.what());                   \
    return ZB_ERR_INTERNAL;                         \
  }

#define ZB_REQUIRE(cond, msg) \
  if (!(cond)) ZB_THROW(ZB_ERR_ARG, msg)

// one int of mapped pinned host memory per GPU for the tensor-core product's
// timeout flag (host and device addresses)
struct OpmmFlag
{
  volatile int *host = nullptr;
  int *dev = nullptr;
};

static OpmmFlag opmm_flag_for_current_device()
{
  static std::mutex mu;
  static std::map<int, OpmmFlag> flags;
  int d = 0;
  cudaError_t e = cudaGetDevice(&d);
  if (e != cudaSuccess) ZB_THROW(ZB_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  std::lock_guard<std::mutex> lk(mu);
  auto it = flags.find(d);
  if (it != flags.end()) return it->second;
  void *h = nullptr;
  e = cudaHostAlloc(&h, sizeof(int), cudaHostAllocMapped);
  if (e != cudaSuccess) ZB_THROW(ZB_ERR_NOMEM, std::string("cudaHostAlloc: ") + cudaGetErrorString(e));
  *static_cast<volatile int *>(h) = 0;
  void *dp = nullptr;
  e = cudaHostGetDevicePointer(&dp, h, 0);
  if (e != cudaSuccess) ZB_THROW(ZB_ERR_CUDA, std::string("cudaHostGetDevicePointer: ") + cudaGetErrorString(e));
  OpmmFlag f{static_cast<volatile int *>(h), static_cast<int *>(dp)};
  flags[d] = f;
  return f;
}

extern "C" {

const char *zb_last_error(void) { return zb::g_err.c_str(); }

const char *zb_version(void) { return "zefr_b200 0.1 (sm_100a)"; }

zb_status zb_params_from_deck(const zb_deck *deck, zb_params *out)
{
  ZB_GUARD({
    ZB_REQUIRE(deck && out, "null argument");
    zb::params_from_deck(*deck, *out);
  })
}

zb_status zb_mesh_read_gmsh(const char *path, int ndims, int n_map, const char *const *names, const int *bcs,
                            zb_mesh **out)
{
  ZB_GUARD({
    ZB_REQUIRE(path && out, "null argument");
    ZB_REQUIRE(n_map >= 0 && (n_map == 0 || (names && bcs)), "bad boundary map");
    std::vector<std::string> nm;
    std::vector<int> bc;
    for (int i = 0; i < n_map; i++)
    {
      nm.push_back(names[i]);
      bc.push_back(bcs[i]);
    }
    auto *m = new zb::MeshData();
    try
    {
      zb::read_gmsh(path, ndims, nm, bc, *m);
    }
    catch (...)
    {
      delete m;
      throw;
    }
    // zb_mesh is the first member, so the view pointer doubles as the handle
    static_assert(offsetof(zb::MeshData, view) == 0, "view must be first");
    *out = &m->view;
  })
}

void zb_mesh_free(zb_mesh *mesh)
{
  if (mesh) delete reinterpret_cast<zb::MeshData *>(mesh);
}

zb_status zb_plan_create(const zb_mesh *mesh, const zb_params *params, zb_plan **out)
{
  ZB_GUARD({
    ZB_REQUIRE(mesh && params && out, "null argument");
    auto *p = new zb_plan();
    try
    {
      zb::build_plan(*mesh, *params, p->plan);
    }
    catch (...)
    {
      delete p;
      throw;
    }
    *out = p;
  })
}

void zb_plan_free(zb_plan *plan) { delete plan; }

zb_status zb_plan_info(const zb_plan *plan, zb_info *out)
{
  ZB_GUARD({
    ZB_REQUIRE(plan && out, "null argument");
    const zb::Plan &p = plan->plan;
    std::memset(out, 0, sizeof(*out));
    out->ndims = p.ndims;
    out->nvars = p.nvars;
    out->nspts = p.nspts;
    out->nfpts = p.nfpts;
    out->order = p.order;
    out->etype = p.etype;
    out->n_eles = p.neles;
    out->n_eles_pad = p.neles_pad;
    out->n_gfpts_int = p.n_gfpts_int;
    out->n_gfpts_bnd = p.n_gfpts_bnd;
    out->n_gfpts = p.n_gfpts_int + p.n_gfpts_bnd;
    out->nstages = 4;
    out->tile = p.tile;
    out->precision = p.params.precision;
  })
}

zb_status zb_plan_get(const zb_plan *plan, const char *name, double *out, int64_t *n)
{
  ZB_GUARD({
    ZB_REQUIRE(plan && name && n, "null argument");
    const zb::Plan &p = plan->plan;
    std::string nm(name);
    std::vector<double> tmp;
    auto put = [&](const std::vector<double> &v) {
      if (out == nullptr)
      {
        *n = (int64_t)v.size();
        return;
      }
      ZB_REQUIRE(*n >= (int64_t)v.size(), "output buffer too small");
      std::memcpy(out, v.data(), v.size() * sizeof(double));
      *n = (int64_t)v.size();
    };
    if (nm == "coord_spts") put(p.coord_spts);
    else if (nm == "coord_fpts") put(p.coord_fpts);
    else if (nm == "jaco_det_spts") put(p.jaco_det_spts);
    else if (nm == "inv_jaco_spts") put(p.inv_jaco_spts);
    else if (nm == "fpt_norm") put(p.fnorm);
    else if (nm == "fpt_dA") put(p.fdA);
    else if (nm == "weights_spts") put(p.weights_spts);
    else if (nm == "loc_spts") put(p.loc_spts);
    else if (nm == "loc_fpts") put(p.loc_fpts);
    else if (nm == "tnorm") put(p.tnorm);
    else if (nm == "dshape_spts") put(p.dshape_spts);
    else if (nm == "dshape_fpts") put(p.dshape_fpts);
    else if (nm == "shape_fpts") put(p.shape_fpts);
    else if (nm == "shape_spts") put(p.shape_spts);
    else if (nm == "nodes") put(p.nodes);
    else if (nm == "fpt_partner")
    {
      tmp.assign(p.partner.begin(), p.partner.end());
      put(tmp);
    }
    else if (nm == "fpt_slot")
    {
      tmp.assign(p.slot.begin(), p.slot.end());
      put(tmp);
    }
    else if (nm == "oppE" || nm == "oppD" || nm == "oppD_fpts" || nm == "oppDiv" || nm == "oppDiv_fpts")
    {
      std::vector<double> E, D, Df, Dv, Dvf;
      p.dense_operators(E, D, Df, Dv, Dvf);
      if (nm == "oppE") put(E);
      else if (nm == "oppD") put(D);
      else if (nm == "oppD_fpts") put(Df);
      else if (nm == "oppDiv") put(Dv);
      else put(Dvf);
    }
    else
      ZB_THROW(ZB_ERR_ARG, "unknown plan array " + nm);
  })
}

zb_status zb_create(const zb_plan *plan, zb_ctx **out)
{
  ZB_GUARD({
    ZB_REQUIRE(plan && out, "null argument");
    auto *c = new zb_ctx();
    try
    {
      c->impl = zb::ctx_create(plan->plan);
    }
    catch (...)
    {
      delete c;
      throw;
    }
    *out = c;
  })
}

zb_status zb_create_from_mesh(const zb_mesh *mesh, const zb_params *params, zb_ctx **out)
{
  ZB_GUARD({
    ZB_REQUIRE(mesh && params && out, "null argument");
    zb_plan plan;
    zb::build_plan(*mesh, *params, plan.plan);
    auto *c = new zb_ctx();
    try
    {
      c->impl = zb::ctx_create(plan.plan);
    }
    catch (...)
    {
      delete c;
      throw;
    }
    *out = c;
  })
}

void zb_destroy(zb_ctx *ctx)
{
  if (!ctx) return;
  try
  {
    zb::ctx_destroy(ctx->impl);
  }
  catch (...)
  {
  }
  delete ctx;
}

zb_status zb_info_get(const zb_ctx *ctx, zb_info *out)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx && out, "null argument");
    zb::ctx_info(ctx->impl, out);
  })
}

zb_status zb_set_stream(zb_ctx *ctx, void *stream)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx, "null context");
    zb::ctx_set_stream(ctx->impl, stream);
  })
}

zb_status zb_set_dt(zb_ctx *ctx, double dt)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx, "null context");
    zb::ctx_set_dt(ctx->impl, dt);
  })
}

zb_status zb_set_state(zb_ctx *ctx, const double *U, int64_t ss, int64_t vs, int64_t es, int where)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx, "null context");
    zb::ctx_set_state(ctx->impl, U, ss, vs, es, where);
  })
}

zb_status zb_get_state(zb_ctx *ctx, double *U, int64_t ss, int64_t vs, int64_t es, int where)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx, "null context");
    zb::ctx_get_state(ctx->impl, U, ss, vs, es, where);
  })
}

zb_status zb_compute_residual(zb_ctx *ctx, unsigned stage)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx, "null context");
    zb::ctx_compute_residual(ctx->impl, stage);
  })
}

zb_status zb_get_residual(zb_ctx *ctx, unsigned stage, double *out, int64_t ss, int64_t vs, int64_t es, int where)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx, "null context");
    zb::ctx_get_residual(ctx->impl, stage, out, ss, vs, es, where);
  })
}

zb_status zb_compute_residuals_host(zb_ctx *ctx, unsigned stage, int n, const double *const *U, double *const *divF)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx, "null context");
    zb::ctx_residuals_host(ctx->impl, stage, n, U, divF);
  })
}

zb_status zb_rk_stage(zb_ctx *ctx, unsigned stage)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx, "null context");
    zb::ctx_rk_stage(ctx->impl, stage);
  })
}

#define ZB_SPLIT_ENTRY(fn, part, rk)          \
  zb_status fn(zb_ctx *ctx, unsigned stage)     \
  {                                             \
    ZB_GUARD({                                  \
      ZB_REQUIRE(ctx, "null context");          \
      zb::ctx_residual_split(ctx->impl, stage, part, rk); \
    })                                          \
  }
ZB_SPLIT_ENTRY(zb_compute_residual_start, 0, 0)
ZB_SPLIT_ENTRY(zb_compute_residual_mid, 1, 0)
ZB_SPLIT_ENTRY(zb_compute_residual_finish, 2, 0)
ZB_SPLIT_ENTRY(zb_rk_stage_start, 0, 1)
ZB_SPLIT_ENTRY(zb_rk_stage_mid, 1, 1)
ZB_SPLIT_ENTRY(zb_rk_stage_finish, 2, 1)
#undef ZB_SPLIT_ENTRY

zb_status zb_step(zb_ctx *ctx, int n)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx, "null context");
    zb::ctx_step(ctx->impl, n);
  })
}

void zb_time_scheme_defaults(zb_time_scheme *out)
{
  if (!out) return;
  *out = zb_time_scheme{ZB_RK44, 0, 1, 1.0, 0, 1e-5, 1e-5, 0.7, 0.4, 0.8, 2.5, 0.3, 100.0};
}

zb_status zb_set_time_scheme(zb_ctx *ctx, const zb_time_scheme *ts)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx && ts, "null argument");
    zb::ctx_set_time_scheme(ctx->impl, ts);
  })
}

zb_status zb_time_state(zb_ctx *ctx, double *dt, double *prev_err, int64_t *rejected, double *flow_time)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx, "null context");
    zb::ctx_time_state(ctx->impl, dt, prev_err, rejected, flow_time);
  })
}

zb_status zb_get_element_dt(zb_ctx *ctx, double *out)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx && out, "null argument");
    zb::ctx_get_element_dt(ctx->impl, out);
  })
}

zb_status zb_rk_step_vjp(zb_ctx *ctx, const double *U0, const double *Ubar1, double *Ubar0, int64_t spt_stride,
                         int64_t var_stride, int64_t ele_stride, int where, double *param_bar, int geometry)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx, "null context");
    zb::ctx_rk_step_vjp(ctx->impl, U0, Ubar1, Ubar0, spt_stride, var_stride, ele_stride, where, param_bar,
                        geometry != 0);
  })
}

zb_status zb_geometry_eval(zb_ctx *ctx, const double *nodes, double *inv_jaco, double *jaco_det, double *norm,
                           double *dA, int where)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx, "null context");
    zb::ctx_geometry_eval(ctx->impl, nodes, inv_jaco, jaco_det, norm, dA, where);
  })
}

zb_status zb_geometry_eval_vjp(zb_ctx *ctx, const double *nodes, const double *inv_jaco_bar,
                               const double *jaco_det_bar, const double *norm_bar, const double *dA_bar,
                               double *nodes_bar, int where)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx, "null context");
    zb::ctx_geometry_eval_vjp(ctx->impl, nodes, inv_jaco_bar, jaco_det_bar, norm_bar, dA_bar, nodes_bar, where);
  })
}

zb_status zb_set_nodes(zb_ctx *ctx, const double *nodes, int where)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx, "null context");
    zb::ctx_set_nodes(ctx->impl, nodes, where);
  })
}

zb_status zb_residual_norms(zb_ctx *ctx, double *out)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx && out, "null argument");
    zb::ctx_norms(ctx->impl, out);
  })
}

zb_status zb_functionals(zb_ctx *ctx, double *out)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx && out, "null argument");
    zb::ctx_functionals(ctx->impl, out);
  })
}

zb_status zb_batch_create(zb_ctx *const *ctxs, int n, zb_batch **out)
{
  ZB_GUARD({
    ZB_REQUIRE(ctxs && out && n > 0, "null argument or empty batch");
    std::vector<zb::Ctx *> v((size_t)n);
    for (int i = 0; i < n; i++)
    {
      ZB_REQUIRE(ctxs[i], "null context in batch");
      v[(size_t)i] = ctxs[i]->impl;
    }
    std::unique_ptr<zb_batch> b(new zb_batch{zb::batch_create(v.data(), n)});
    *out = b.release();
  })
}

void zb_batch_destroy(zb_batch *batch)
{
  if (!batch) return;
  try
  {
    zb::batch_destroy(batch->impl);
  }
  catch (...)
  {
  }
  delete batch;
}

zb_status zb_batch_autotune(zb_batch *batch, int steps, zb_batch_config *chosen)
{
  ZB_GUARD({
    ZB_REQUIRE(batch, "null batch");
    zb::batch_autotune(batch->impl, steps, -1, chosen);
  })
}

zb_status zb_batch_autotune_form(zb_batch *batch, int steps, int form, zb_batch_config *chosen)
{
  ZB_GUARD({
    ZB_REQUIRE(batch, "null batch");
    ZB_REQUIRE(form >= -1 && form <= 1, "form must be -1, 0 or 1");
    zb::batch_autotune(batch->impl, steps, form, chosen);
  })
}

zb_status zb_batch_set_config(zb_batch *batch, const zb_batch_config *cfg)
{
  ZB_GUARD({
    ZB_REQUIRE(batch && cfg, "null argument");
    zb::batch_config(batch->impl, cfg);
  })
}

zb_status zb_batch_step(zb_batch *batch, int nsteps, int use_graph)
{
  ZB_GUARD({
    ZB_REQUIRE(batch, "null batch");
    zb::batch_step(batch->impl, nsteps, use_graph);
  })
}

zb_status zb_batch_stage(zb_batch *batch, unsigned stage)
{
  ZB_GUARD({
    ZB_REQUIRE(batch, "null batch");
    zb::batch_stage(batch->impl, stage);
  })
}

zb_status zb_batch_synchronize(zb_batch *batch)
{
  ZB_GUARD({
    ZB_REQUIRE(batch, "null batch");
    zb::batch_sync(batch->impl);
  })
}

int64_t zb_batch_launch_count(const zb_batch *batch) { return batch ? zb::batch_launches(batch->impl) : -1; }

zb_status zb_set_freestream(zb_ctx *ctx, double rho_fs, const double *V_fs, double P_fs)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx && V_fs, "null argument");
    zb::ctx_set_freestream(ctx->impl, rho_fs, V_fs, P_fs);
  })
}

zb_status zb_vjp(zb_ctx *ctx, const double *lam, double *Ubar, int64_t spt_stride, int64_t var_stride,
                 int64_t ele_stride, int where, double *param_bar)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx && lam && Ubar, "null argument");
    ZB_REQUIRE(where == ZB_HOST || where == ZB_DEVICE, "where must be ZB_HOST or ZB_DEVICE");
    zb::ctx_vjp(ctx->impl, lam, Ubar, spt_stride, var_stride, ele_stride, where, param_bar);
  })
}

zb_status zb_wall_force(zb_ctx *ctx, double *out)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx && out, "null argument");
    zb::ctx_wall_force(ctx->impl, out);
  })
}

zb_status zb_vjp_geometry(zb_ctx *ctx, const double *lam, double *Ubar, int64_t spt_stride, int64_t var_stride,
                          int64_t ele_stride, int where, double *param_bar, double *inv_jaco_bar,
                          double *jaco_det_bar, double *norm_bar, double *dA_bar)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx && lam && Ubar && inv_jaco_bar && jaco_det_bar && norm_bar && dA_bar, "null argument");
    ZB_REQUIRE(where == ZB_HOST || where == ZB_DEVICE, "where must be ZB_HOST or ZB_DEVICE");
    zb::ctx_vjp(ctx->impl, lam, Ubar, spt_stride, var_stride, ele_stride, where, param_bar, inv_jaco_bar,
                jaco_det_bar, norm_bar, dA_bar);
  })
}

zb_status zb_vjp_geometry_accumulate(zb_ctx *ctx, const double *lam, double *Ubar, int64_t spt_stride,
                                     int64_t var_stride, int64_t ele_stride, int where, double *param_bar)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx && lam && Ubar, "null argument");
    ZB_REQUIRE(where == ZB_HOST || where == ZB_DEVICE, "where must be ZB_HOST or ZB_DEVICE");
    zb::ctx_vjp(ctx->impl, lam, Ubar, spt_stride, var_stride, ele_stride, where, param_bar, nullptr, nullptr, nullptr,
                nullptr, true);
  })
}

zb_status zb_geometry_adjoint_get(zb_ctx *ctx, double *inv_jaco_bar, double *jaco_det_bar, double *norm_bar,
                                  double *dA_bar, int reset)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx && inv_jaco_bar && jaco_det_bar && norm_bar && dA_bar, "null argument");
    zb::ctx_geometry_adjoint_get(ctx->impl, inv_jaco_bar, jaco_det_bar, norm_bar, dA_bar, reset);
  })
}

zb_status zb_synchronize(zb_ctx *ctx)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx, "null context");
    zb::ctx_sync(ctx->impl);
  })
}

int64_t zb_launch_count(const zb_ctx *ctx) { return ctx ? zb::ctx_launches(ctx->impl) : -1; }

zb_status zb_profile_enable(zb_ctx *ctx, int on)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx, "null context");
    zb::ctx_profile_enable(ctx->impl, on);
  })
}

zb_status zb_profile_read(zb_ctx *ctx, double *ms, int64_t *count)
{
  ZB_GUARD({
    ZB_REQUIRE(ctx, "null context");
    zb::ctx_profile_read(ctx->impl, ms, count);
  })
}

zb_status zb_compute_residual_noalloc(const zb_plan *plan, const double *U, double *divF, void *stream)
{
  ZB_GUARD({
    ZB_REQUIRE(plan, "null plan");
    zb::noalloc_residual(plan->plan, U, divF, (cudaStream_t)stream);
  })
}

const char *zb_kernel_name(int id)
{
  static const char *names[ZB_NKERNELS] = {"k_extrap", "k_euler", "k_ns_grad", "k_ns_face",
                                           "k_to_tiles", "k_from_tiles", "k_norms", "k_adj_lift",
                                           "k_adj_vol", "k_adj_trace", "k_functionals"};
  return (id >= 0 && id < ZB_NKERNELS) ? names[id] : "unknown";
}

zb_status zb_operator_mm_tf32x3(int m, int n, int k, float alpha, const float *a, int lda, const float *b, int ldb,
                                float beta, float *c, int ldc, void *stream)
{
  ZB_GUARD({
    ZB_REQUIRE(a && c && (b || n == 0), "null operand");
    const OpmmFlag f = opmm_flag_for_current_device();
    zb::opmm_tc(m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, static_cast<cudaStream_t>(stream), f.host, f.dev);
  })
}

}  // extern "C"


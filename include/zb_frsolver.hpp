/* zb_frsolver.hpp -- an FRSolver-shaped C++ class over the C ABI of
 * libzefr_b200 (zb.h), for a driver written against the reference's FRSolver
 * (include/solver.hpp:150-190) that swaps its residual and RK stepping for
 * this library's.  Method names follow the reference; errors become
 * std::runtime_error as the reference's ThrowException does
 * (include/macros.hpp:52-54).  Header only; link with -lzefr_b200. */
#ifndef ZB_FRSOLVER_HPP
#define ZB_FRSOLVER_HPP

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "zb.h"

class ZbFRSolver
{
 public:
  /* FRSolver(input) + setup(): mesh and deck-style inputs */
  ZbFRSolver(const zb_mesh &mesh, const zb_deck &deck)
  {
    check(zb_params_from_deck(&deck, &params_));
    init(mesh);
  }
  ZbFRSolver(const zb_mesh &mesh, const zb_params &params) : params_(params) { init(mesh); }
  ~ZbFRSolver()
  {
    if (ctx_) zb_destroy(ctx_);
    if (plan_) zb_plan_free(plan_);
  }
  ZbFRSolver(const ZbFRSolver &) = delete;
  ZbFRSolver &operator=(const ZbFRSolver &) = delete;

  /* FRSolver::compute_residual(stage) (include/solver.hpp:152): divF_spts(stage) */
  void compute_residual(unsigned stage) { check(zb_compute_residual(ctx_, stage)); }
  /* the split form (include/solver.hpp:153-155) */
  void compute_residual_start(unsigned stage) { check(zb_compute_residual_start(ctx_, stage)); }
  void compute_residual_mid(unsigned stage) { check(zb_compute_residual_mid(ctx_, stage)); }
  void compute_residual_finish(unsigned stage) { check(zb_compute_residual_finish(ctx_, stage)); }

  /* FRSolver::update / step_RK / step_RK_stage (include/solver.hpp:158-190) */
  void update() { check(zb_step(ctx_, 1)); }
  void step_RK_stage(unsigned stage) { check(zb_rk_stage(ctx_, stage)); }
  void step_RK_stage_start(unsigned stage) { check(zb_rk_stage_start(ctx_, stage)); }
  void step_RK_stage_mid(unsigned stage) { check(zb_rk_stage_mid(ctx_, stage)); }
  void step_RK_stage_finish(unsigned stage) { check(zb_rk_stage_finish(ctx_, stage)); }

  /* the deck's dt_scheme / dt_type / CFL / adapt_dt keys (step_LSRK,
   * step_adaptive, compute_element_dt); update() follows them afterwards */
  void set_time_scheme(const zb_time_scheme &ts) { check(zb_set_time_scheme(ctx_, &ts)); }
  double dt()
  {
    double dt = 0.0;
    check(zb_time_state(ctx_, &dt, nullptr, nullptr, nullptr));
    return dt;
  }

  /* zefr::get_q_spts-style access (include/zefr_interface.hpp:126-129):
   * U[spt * ss + var * vs + ele * es], host or device memory */
  void set_q(const double *U, int64_t ss, int64_t vs, int64_t es, bool device)
  {
    check(zb_set_state(ctx_, U, ss, vs, es, device ? ZB_DEVICE : ZB_HOST));
  }
  void get_q(double *U, int64_t ss, int64_t vs, int64_t es, bool device)
  {
    check(zb_get_state(ctx_, U, ss, vs, es, device ? ZB_DEVICE : ZB_HOST));
  }
  void get_divF(unsigned stage, double *R, int64_t ss, int64_t vs, int64_t es, bool device)
  {
    check(zb_get_residual(ctx_, stage, R, ss, vs, es, device ? ZB_DEVICE : ZB_HOST));
  }
  /* report_residuals values (src/solver.cpp:6990-7137), per variable:
   * max, sum of |.|, sqrt of the sum of squares of divF/|J| over nSpts*nEles */
  std::vector<double> residual_norms()
  {
    std::vector<double> out((size_t)3 * nVars_);
    check(zb_residual_norms(ctx_, out.data()));
    return out;
  }

  int64_t nEles() const { return nEles_; }
  int nVars() const { return nVars_; }
  int nSpts() const { return nSpts_; }
  zb_ctx *handle() { return ctx_; }

 private:
  void init(const zb_mesh &mesh)
  {
    check(zb_plan_create(&mesh, &params_, &plan_));
    const zb_status s = zb_create(plan_, &ctx_);
    if (s != ZB_OK)
    {
      const std::string msg = zb_last_error();
      zb_plan_free(plan_);
      plan_ = nullptr;
      throw std::runtime_error(msg);
    }
    zb_info info;
    check(zb_info_get(ctx_, &info));
    nEles_ = info.n_eles;
    nVars_ = info.nvars;
    nSpts_ = info.nspts;
  }
  static void check(zb_status s)
  {
    if (s != ZB_OK) throw std::runtime_error(zb_last_error());
  }
  zb_params params_{};
  zb_plan *plan_ = nullptr;
  zb_ctx *ctx_ = nullptr;
  int64_t nEles_ = 0;
  int nVars_ = 0, nSpts_ = 0;
};

#endif /* ZB_FRSOLVER_HPP */

/* C-ABI harness around the reference's own CPU FRSolver (test infrastructure).
 *
 * Built by oracle/Makefile against the unmodified reference sources; the
 * product never links it.  It lets the tests and the golden-fixture script
 * drive the reference exactly as its driver does (src/zefr.cpp:26-152:
 * read_input_file -> FRSolver::setup), overwrite the state, call
 * FRSolver::compute_residual (src/solver.cpp:1494-1645) or FRSolver::update
 * (src/solver.cpp:2598-2644), and read back the residual, state, operators,
 * metrics and face connectivity for comparison.  The diagnostics are the
 * reference's own: report_residuals (src/solver.cpp:6990-7137),
 * report_turbulent_stats (7813-7917) and compute_moments (7600-7811), run on
 * the arrays the last compute_residual left.
 *
 * Layouts returned are the reference's own row-major mdvector layouts
 * (include/mdvector.hpp:189-260) with nElesPad == nEles on the CPU build
 * (src/elements.cpp:71-75).
 */
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <fstream>
#include <cstdio>
#include <cstring>
#include <exception>
#include <iostream>
#include <map>
#include <memory>
#include <set>
#include <sstream>
#include <string>
#include <vector>

/* Reach the reference's private members: the harness reads arrays the
 * reference keeps private (FRSolver::geo, Elements operators). */
#define private public
#define protected public
#include "input.hpp"
#include "geometry.hpp"
#include "elements.hpp"
#include "faces.hpp"
#include "solver.hpp"
#undef private
#undef protected

namespace {

struct RefHandle
{
  InputStruct input;
  std::unique_ptr<FRSolver> solver;
  std::string err;
};

thread_local std::string g_last_error;

int fail(const std::exception &e)
{
  g_last_error = e.what();
  return -1;
}

template <class T>
long copy_out(const mdvector<T> &v, double *out, long n)
{
  long sz = (long)v.size();
  if (out == nullptr) return sz;
  if (n < sz) return -2;
  for (long i = 0; i < sz; i++) out[i] = (double)v.data()[i];
  return sz;
}

}  // namespace

extern "C" {

const char *zr_last_error() { return g_last_error.c_str(); }

void *zr_create(const char *deck)
{
  try
  {
    auto *h = new RefHandle();
    h->input = read_input_file(deck);
    h->input.rank = 0;
    h->input.nRanks = 1;
    std::streambuf *old = std::cout.rdbuf();
    std::ostringstream sink;
    std::cout.rdbuf(sink.rdbuf());
    try
    {
      h->solver.reset(new FRSolver(&h->input));
      h->solver->setup(0);
    }
    catch (...)
    {
      std::cout.rdbuf(old);
      throw;
    }
    std::cout.rdbuf(old);
    return h;
  }
  catch (std::exception &e)
  {
    g_last_error = e.what();
    return nullptr;
  }
}

void zr_destroy(void *p) { delete static_cast<RefHandle *>(p); }

/* out[0..11] = nDims, nVars, nSpts, nFpts, nEles, nElesPad, nStages,
 *              nGfpts, nGfpts_int, nGfpts_bnd, etype, order */
int zr_info(void *p, int *out)
{
  auto *h = static_cast<RefHandle *>(p);
  auto &e = h->solver->eles;
  auto &geo = h->solver->geo;
  out[0] = (int)e->nDims;
  out[1] = (int)e->nVars;
  out[2] = (int)e->nSpts;
  out[3] = (int)e->nFpts;
  out[4] = (int)e->nEles;
  out[5] = (int)e->nElesPad;
  out[6] = (int)h->input.nStages;
  out[7] = (int)geo.nGfpts;
  out[8] = (int)geo.nGfpts_int;
  out[9] = (int)geo.nGfpts_bnd;
  out[10] = (int)e->etype;
  out[11] = (int)e->order;
  return 0;
}

/* Physical parameters after read_input_file / apply_nondim
 * (src/input.cpp:463-539), in a fixed order:
 *  0 gamma 1 prandtl 2 mu 3 rt 4 c_sth 5 fix_vis 6 rus_k 7 ldg_b 8 ldg_tau
 *  9 rho_fs 10-12 V_fs 13 P_fs 14 T_wall 15 R_ref 16-18 V_wall 19 dt
 *  20 viscous 21 T_tot_fs 22 P_tot_fs */
int zr_params(void *p, double *out)
{
  auto *h = static_cast<RefHandle *>(p);
  auto &in = h->input;
  for (int i = 0; i < 23; i++) out[i] = 0.0;
  out[0] = in.gamma;
  out[1] = in.prandtl;
  out[2] = in.mu;
  out[3] = in.rt;
  out[4] = in.c_sth;
  out[5] = in.fix_vis ? 1.0 : 0.0;
  out[6] = in.rus_k;
  out[7] = in.ldg_b;
  out[8] = in.ldg_tau;
  out[9] = in.rho_fs;
  for (unsigned d = 0; d < 3 && d < in.V_fs.size(); d++) out[10 + d] = in.V_fs(d);
  out[13] = in.P_fs;
  out[14] = in.T_wall;
  out[15] = in.R_ref;
  for (unsigned d = 0; d < 3 && d < in.V_wall.size(); d++) out[16 + d] = in.V_wall(d);
  out[19] = in.dt;
  out[20] = in.viscous ? 1.0 : 0.0;
  out[21] = in.T_tot_fs;
  out[22] = in.P_tot_fs;
  return 0;
}

/* U in [nSpts][nVars][nEles] */
int zr_set_state(void *p, const double *U)
{
  auto *h = static_cast<RefHandle *>(p);
  auto &e = h->solver->eles;
  for (unsigned s = 0; s < e->nSpts; s++)
    for (unsigned v = 0; v < e->nVars; v++)
      for (unsigned k = 0; k < e->nEles; k++)
        e->U_spts(s, v, k) = U[((size_t)s * e->nVars + v) * e->nEles + k];
  return 0;
}

int zr_get_state(void *p, double *U)
{
  auto *h = static_cast<RefHandle *>(p);
  auto &e = h->solver->eles;
  for (unsigned s = 0; s < e->nSpts; s++)
    for (unsigned v = 0; v < e->nVars; v++)
      for (unsigned k = 0; k < e->nEles; k++)
        U[((size_t)s * e->nVars + v) * e->nEles + k] = e->U_spts(s, v, k);
  return 0;
}

int zr_compute_residual(void *p, int stage)
{
  try
  {
    static_cast<RefHandle *>(p)->solver->compute_residual((unsigned)stage);
    return 0;
  }
  catch (std::exception &e)
  {
    return fail(e);
  }
}

/* divF_spts(stage) in [nSpts][nVars][nEles] */
int zr_get_residual(void *p, int stage, double *out)
{
  auto *h = static_cast<RefHandle *>(p);
  auto &e = h->solver->eles;
  for (unsigned s = 0; s < e->nSpts; s++)
    for (unsigned v = 0; v < e->nVars; v++)
      for (unsigned k = 0; k < e->nEles; k++)
        out[((size_t)s * e->nVars + v) * e->nEles + k] = e->divF_spts((unsigned)stage, s, v, k);
  return 0;
}

/* nsteps calls of FRSolver::update (one explicit RK step each). */
int zr_update(void *p, int nsteps)
{
  try
  {
    auto *h = static_cast<RefHandle *>(p);
    for (int i = 0; i < nsteps; i++)
    {
      h->solver->update();
      h->input.iter++;
    }
    return 0;
  }
  catch (std::exception &e)
  {
    return fail(e);
  }
}

/* report_residuals (src/solver.cpp:6990-7137) on divF_spts(0) as the last
 * compute_residual left it: out[n] = the value the reference prints for
 * variable n (max, sum of |.| or sqrt of the sum of squares of divF/|J| over
 * solution points, per res_type 0/1/2, divided by nSpts * nEles), read from
 * FRSolver::res_max with res_field = n.  Terminal and history output are
 * dropped. */
int zr_report_residuals(void *p, int res_type, double *out)
{
  try
  {
    auto *h = static_cast<RefHandle *>(p);
    auto &in = h->input;
    const unsigned old_type = in.res_type, old_field = in.res_field;
    std::ofstream hist;  // never opened: the history lines go nowhere
    std::streambuf *old = std::cout.rdbuf();
    std::ostringstream sink;
    std::cout.rdbuf(sink.rdbuf());
    in.res_type = (unsigned)res_type;
    for (unsigned n = 0; n < h->solver->eles->nVars; n++)
    {
      in.res_field = n;
      h->solver->report_residuals(hist, std::chrono::high_resolution_clock::now());
      out[n] = h->solver->res_max;
    }
    std::cout.rdbuf(old);
    in.res_type = old_type;
    in.res_field = old_field;
    return 0;
  }
  catch (std::exception &e)
  {
    return fail(e);
  }
}

/* report_turbulent_stats (src/solver.cpp:7813-7917) on U_spts and the
 * physical gradient dU_spts the last compute_residual left: the reference
 * writes "iter flow_time ke enstrophy" (17 significant digits) to the history
 * file at `path`; out[0] = ke, out[1] = enstrophy as written there, both
 * already divided by vol * rho_fs * |V_fs|^2; out[2] = that divisor. */
int zr_turbulent_stats(void *p, const char *path, double *out)
{
  try
  {
    auto *h = static_cast<RefHandle *>(p);
    std::streambuf *old = std::cout.rdbuf();
    std::ostringstream sink;
    std::cout.rdbuf(sink.rdbuf());
    {
      std::ofstream f(path);
      h->solver->report_turbulent_stats(f);
    }
    std::cout.rdbuf(old);
    std::ifstream g(path);
    double iter = 0, t = 0;
    if (!(g >> iter >> t >> out[0] >> out[1])) throw std::runtime_error("turbulent stats not written");
    double vol = 0;
    for (auto e : h->solver->elesObjs)
      for (unsigned k = 0; k < e->nEles; k++) vol += e->vol(k);
    out[2] = vol * h->input.rho_fs * h->input.v_mag_fs * h->input.v_mag_fs;
    return 0;
  }
  catch (std::exception &e)
  {
    return fail(e);
  }
}

/* compute_moments (src/solver.cpp:7600-7811) on the face arrays (P, U, dU)
 * the last compute_residual left: out[0..2] total force, out[3..5] moment
 * about geo.x_cg. */
int zr_compute_moments(void *p, double *out)
{
  try
  {
    auto *h = static_cast<RefHandle *>(p);
    std::array<double, 3> force, moment;
    h->solver->compute_moments(force, moment, nullptr);
    for (int d = 0; d < 3; d++)
    {
      out[d] = force[d];
      out[3 + d] = moment[d];
    }
    return 0;
  }
  catch (std::exception &e)
  {
    return fail(e);
  }
}

/* Copy a named reference array out as doubles.  Returns the element count
 * (call with out == nullptr to size), -1 for an unknown name, -2 when n is
 * too small. */
long zr_get_array(void *p, const char *cname, double *out, long n)
{
  auto *h = static_cast<RefHandle *>(p);
  auto &e = h->solver->eles;
  auto &f = h->solver->faces;
  auto &geo = h->solver->geo;
  std::string name(cname);
  if (name == "coord_spts") return copy_out(e->coord_spts, out, n);
  if (name == "coord_fpts") return copy_out(e->coord_fpts, out, n);
  if (name == "nodes") return copy_out(e->nodes, out, n);
  if (name == "jaco_det_spts") return copy_out(e->jaco_det_spts, out, n);
  if (name == "inv_jaco_spts") return copy_out(e->inv_jaco_spts, out, n);
  if (name == "weights_spts") return copy_out(e->weights_spts, out, n);
  if (name == "oppE") return copy_out(e->oppE, out, n);
  if (name == "oppD") return copy_out(e->oppD, out, n);
  if (name == "oppD_fpts") return copy_out(e->oppD_fpts, out, n);
  if (name == "oppDiv") return copy_out(e->oppDiv, out, n);
  if (name == "oppDiv_fpts") return copy_out(e->oppDiv_fpts, out, n);
  if (name == "loc_spts") return copy_out(e->loc_spts, out, n);
  if (name == "loc_fpts") return copy_out(e->loc_fpts, out, n);
  if (name == "U_fpts") return copy_out(e->U_fpts, out, n);
  if (name == "F_spts") return copy_out(e->F_spts, out, n);
  if (name == "Fcomm") return copy_out(e->Fcomm, out, n);
  if (name == "Ucomm") return copy_out(e->Ucomm, out, n);
  if (name == "dU_spts") return copy_out(e->dU_spts, out, n);
  if (name == "dU_fpts") return copy_out(e->dU_fpts, out, n);
  if (name == "norm") return copy_out(f->norm, out, n);
  if (name == "dA") return copy_out(f->dA, out, n);
  if (name == "P") return copy_out(f->P, out, n);
  if (name == "waveSp") return copy_out(f->waveSp, out, n);
  if (name == "diffCo") return copy_out(f->diffCo, out, n);
  if (name == "dt") return copy_out(e->dt, out, n);
  if (name == "vol") return copy_out(e->vol, out, n);
  if (name == "h_ref") return copy_out(e->h_ref, out, n);
  if (name == "fpt2gfpt") return copy_out(geo.fpt2gfptBT[e->etype], out, n);
  if (name == "fpt2gfpt_slot") return copy_out(geo.fpt2gfpt_slotBT[e->etype], out, n);
  if (name == "gfpt2bnd")
  {
    long sz = (long)geo.gfpt2bnd.size();
    if (out == nullptr) return sz;
    if (n < sz) return -2;
    for (long i = 0; i < sz; i++) out[i] = (double)geo.gfpt2bnd(i);
    return sz;
  }
  return -1;
}

}  // extern "C"

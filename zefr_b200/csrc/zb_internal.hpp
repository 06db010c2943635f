// Internal declarations shared by the host set-up, the C ABI and the kernels.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/zb.h"

namespace zb {

// Reference ELE_TYPE numbering (include/input.hpp:33-35).
enum EleType { ET_TRI = 1, ET_QUAD = 2, ET_HEX = 4 };

struct Error : std::runtime_error
{
  zb_status code;
  Error(zb_status c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define ZB_THROW(code, msg)                                                                      \
  throw ::zb::Error((code), std::string(__FILE__) + ":" + std::to_string(__LINE__) + ": " + (msg))

// Owned copy of a zb_mesh.
struct MeshData
{
  zb_mesh view{};
  std::vector<double> coords;
  std::vector<int64_t> ele2nodes;
  std::vector<int64_t> face_nodes;
  std::vector<int> face_bc;
  void sync_view();
};

// One-dimensional DFR line operators on N Gauss-Legendre points.
//  Em[m], Ep[m]  : l_m(-1), l_m(+1)          (Lagrange basis on the N points)
//  D[i*N+m]      : l'_{m+1}(x_i) on the extended set [-1, x_0..x_{N-1}, 1]
//  Dbm[i], Dbp[i]: l'_0(x_i), l'_{N+1}(x_i) on the extended set
struct LineOps
{
  int N = 0;
  std::vector<double> x, w, Em, Ep, D, Dbm, Dbp;
};

// Host-side set-up for one mesh of one element type.
struct Plan
{
  zb_params params{};
  int ndims = 0, etype = 0, order = 0, N = 0, nspts = 0, nfpts = 0, nvars = 0;
  int nfaces = 0, nfpts_face = 0, gmsh_type = 0, nnodes_ele = 0;
  int tile = 8;
  int64_t neles = 0, ntiles = 0, neles_pad = 0;
  int64_t n_gfpts_int = 0, n_gfpts_bnd = 0;
  LineOps ops;

  // Point tables (reference orderings, src/quads.cpp:47-158, src/hexas.cpp:52-240)
  std::vector<double> loc_spts;  // [S][D]
  std::vector<double> loc_fpts;  // [Fp][D]
  std::vector<double> tnorm;     // [Fp][D]
  std::vector<int> spt_idx;      // [S][D] line coordinates
  std::vector<int> fpt_dim, fpt_side, fpt_base, fpt_stride;  // per fpt: normal dim, -1/+1, line
  std::vector<int> spt_fm, spt_fp;  // [D][S]: fpt at the -/+ end of the line through spt

  // Geometry in the reference's own layouts (host, FP64)
  std::vector<double> nodes;         // [nNodes][D][E]
  std::vector<double> coord_spts;    // [S][D][E]
  std::vector<double> coord_fpts;    // [Fp][D][E]
  std::vector<double> jaco_det_spts; // [S][E]
  std::vector<double> inv_jaco_spts; // [D][S][D][E]  (adjugate)
  std::vector<double> weights_spts;  // [S]
  std::vector<double> dshape_spts;   // [D][S][nNodes] shape-function derivatives (geometry adjoint)
  std::vector<double> dshape_fpts;   // [D][Fp][nNodes]
  std::vector<double> shape_fpts;    // [Fp][nNodes]
  std::vector<double> shape_spts;    // [S][nNodes]

  // Face connectivity per element flux point
  std::vector<int64_t> partner;  // [Fp][E]: e'*Fp + f' (interior) or -1-bc (boundary)
  std::vector<int8_t> slot;      // [Fp][E]: 0 left, 1 right
  std::vector<double> fnorm;     // [Fp][D][E]: left element's unit normal of the face
  std::vector<double> fdA;       // [Fp][E]: this side's dA

  // Triangles: dense FR operators in the reference layouts
  std::vector<double> tri_oppE;        // [Fp][S]
  std::vector<double> tri_oppD;        // [D][S][S]
  std::vector<double> tri_oppD_fpts;   // [D][S][Fp]
  std::vector<double> tri_oppDiv;      // [S][D][S]
  std::vector<double> tri_oppDiv_fpts; // [S][Fp]

  // Dense operators (assembled from the line operators for quads and hexes)
  void dense_operators(std::vector<double> &oppE, std::vector<double> &oppD,
                       std::vector<double> &oppD_fpts, std::vector<double> &oppDiv,
                       std::vector<double> &oppDiv_fpts) const;
};

// Set-up entry points
LineOps make_line_ops(int N);
void build_plan(const zb_mesh &mesh, const zb_params &params, Plan &plan);
void read_gmsh(const std::string &path, int ndims, const std::vector<std::string> &names,
               const std::vector<int> &bcs, MeshData &out);
void params_from_deck(const zb_deck &deck, zb_params &out);
void tri_tables(Plan &plan);
void tri_shape(int nn, const double *loc, double *val, double *dval);

// Polynomials restated from reference include/polynomials.hpp:16-76
double lagrange(const std::vector<double> &grid, int mode, double x);
double lagrange_d1(const std::vector<double> &grid, int mode, double x);
std::vector<double> gauss_legendre_points(int n);
std::vector<double> gauss_legendre_weights(int n);

void set_last_error(const std::string &msg);

}  // namespace zb

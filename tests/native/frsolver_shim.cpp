// Driver written against include/zb_frsolver.hpp the way the reference's
// driver calls FRSolver: read a gmsh mesh, set the state through the
// get_q_spts-style strides, compute a residual (whole and split), take one
// RK step, write the results.  Test infrastructure for tests/test_frsolver_shim.py.
//
//   frsolver_shim mesh.msh params.bin U.bin out.bin
//
// params.bin holds a zb_params as the Python binding lays it out; U.bin the
// state [nspts][nvars][n_eles] (float64).  out.bin receives divF_spts(0), the
// split residual of stage 1, and the state after one update(), back to back.
// Without a usable GPU the constructor throws; the program then prints
// "no device:" and the library's message and exits 0.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <vector>

#include "zb_frsolver.hpp"

static std::vector<char> slurp(const char *path)
{
  std::ifstream f(path, std::ios::binary);
  return std::vector<char>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

int main(int argc, char **argv)
{
  if (argc != 5)
  {
    std::cerr << "usage: frsolver_shim mesh.msh params.bin U.bin out.bin\n";
    return 2;
  }
  const char *names[] = {"PERIODIC"};
  const int bcs[] = {ZB_BC_PERIODIC};
  zb_mesh *mesh = nullptr;
  if (zb_mesh_read_gmsh(argv[1], 2, 1, names, bcs, &mesh) != ZB_OK)
  {
    std::cerr << "mesh: " << zb_last_error() << "\n";
    return 1;
  }
  const std::vector<char> pb = slurp(argv[2]);
  if (pb.size() != sizeof(zb_params))
  {
    std::cerr << "params: " << pb.size() << " bytes, zb_params is " << sizeof(zb_params) << "\n";
    return 1;
  }
  zb_params params;
  std::memcpy(&params, pb.data(), sizeof(params));
  try
  {
    ZbFRSolver s(*mesh, params);
    const int64_t E = s.nEles(), V = s.nVars(), S = s.nSpts();
    const std::vector<char> ub = slurp(argv[3]);
    if ((int64_t)ub.size() != S * V * E * 8)
    {
      std::cerr << "state size\n";
      return 1;
    }
    std::vector<double> U(S * V * E), R0(S * V * E), R1(S * V * E), U1(S * V * E);
    std::memcpy(U.data(), ub.data(), ub.size());
    // the reference's U_spts strides: ele 1, var nEles, spt nEles * nVars
    s.set_q(U.data(), V * E, E, 1, false);
    s.compute_residual(0);
    s.get_divF(0, R0.data(), V * E, E, 1, false);
    s.compute_residual_start(1);
    s.compute_residual_mid(1);
    s.compute_residual_finish(1);
    s.get_divF(1, R1.data(), V * E, E, 1, false);
    s.update();
    s.get_q(U1.data(), V * E, E, 1, false);
    const std::vector<double> norms = s.residual_norms();
    std::ofstream out(argv[4], std::ios::binary);
    out.write(reinterpret_cast<const char *>(R0.data()), R0.size() * 8);
    out.write(reinterpret_cast<const char *>(R1.data()), R1.size() * 8);
    out.write(reinterpret_cast<const char *>(U1.data()), U1.size() * 8);
    std::printf("ok %lld elements, norms %zu\n", (long long)E, norms.size());
  }
  catch (const std::runtime_error &e)
  {
    std::printf("no device: %s\n", e.what());
  }
  zb_mesh_free(mesh);
  return 0;
}

// Adjoint launches (plain FP64 form): kernel instantiations live in their own
// translation unit so they build in parallel with the forward kernels.
#include "ctx_impl.cuh"
#include "adjoint.cuh"
#include "tri_adjoint.cuh"

namespace zb {

using dev::LineOpsT;
using dev::Shape;
using dev::TW;

// Adjoint of the residual (plain FP64 form): lift, then the volume/face
// pass, then for Navier-Stokes the common-solution pass.
// The volume/face pass and the trace pass, with or without the geometry
// outputs (a separate instantiation, so the state adjoint carries none of
// their registers).
template <int D, int N, bool GEO>
static void launch_adj_kernels(Ctx &c, const dev::AdjArgs &a, const LineOpsT<double, N> &ops)
{
  using G = Shape<D, N>;
  constexpr int S = G::S, Fp = G::Fp, V = G::V, NT = G::NT;
  if (!c.plan.params.viscous)
  {
    const size_t smem = (size_t)(S * V + Fp * V) * TW * sizeof(double);
    set_smem(dev::k_adj_euler<D, N, GEO>, smem);
    ProfScope ps(c, ZB_K_ADJ_VOL);
    dev::k_adj_euler<D, N, GEO><<<(unsigned)c.ntiles, NT, smem, c.stream>>>(a, ops);
    c.launches++;
    CK(cudaGetLastError());
    return;
  }
  // the state adjoint's staged face inputs: [Fp][3V + D][TW]
  const size_t smem1 = (size_t)(GEO ? 2 * S * V + Fp * V + 2 * D * S * V
                                    : S * V + Fp * V + D * S * V + Fp * (3 * V + D)) *
                       TW * sizeof(double);
  set_smem(dev::k_adj_ns1<D, N, GEO>, smem1);
  {
    ProfScope ps(c, ZB_K_ADJ_VOL);
    dev::k_adj_ns1<D, N, GEO><<<(unsigned)c.ntiles, NT, smem1, c.stream>>>(a, ops);
    c.launches++;
    CK(cudaGetLastError());
  }
  const size_t smem2 = (size_t)Fp * V * TW * sizeof(double);
  set_smem(dev::k_adj_ns2<D, N, GEO>, smem2);
  ProfScope ps(c, ZB_K_ADJ_TRACE);
  dev::k_adj_ns2<D, N, GEO><<<(unsigned)c.ntiles, NT, smem2, c.stream>>>(a, ops);
  c.launches++;
  CK(cudaGetLastError());
}

template <int D, int N>
static void launch_vjp_impl(Ctx &c, bool params, bool geo)
{
  using G = Shape<D, N>;
  constexpr int Fp = G::Fp;
  dev::AdjArgs a;
  std::memset(&a, 0, sizeof(a));
  a.U = (const double *)c.U;
  a.Ufp = (const double *)c.Ufp[c.cur];
  a.mets = (const double *)c.mets;
  a.fgeo = (const double *)c.fgeo;
  a.nbr = c.nbr;
  a.lam = c.lam;
  a.Lfp = c.Lfp;
  a.Ubfp = c.Ubfp;
  a.dUbfp = c.dUbfp;
  a.Ubx = c.Ubx;
  a.UCb = c.UCb;
  a.Ubar = c.Ubar;
  a.pbar = params ? c.pbar : nullptr;
  a.mbar = geo ? c.mbar : nullptr;
  a.gbar = geo ? c.gbar : nullptr;
  a.nbx = geo ? c.nbx : nullptr;
  a.Fvn = (const double *)c.Fvn;
  a.ntiles = c.ntiles;
  a.ph = phys_of<double>(c.plan.params, c.uref, D, false);
  const LineOpsT<double, N> ops = line_ops<double, N>(c.plan);
  {
    ProfScope ps(c, ZB_K_ADJ_LIFT);
    dev::k_adj_lift<D, N><<<grid_for(c.ntiles * Fp * TW, 256), 256, 0, c.stream>>>(a, ops);
    c.launches++;
    CK(cudaGetLastError());
  }
  if (geo)
    launch_adj_kernels<D, N, true>(c, a, ops);
  else
    launch_adj_kernels<D, N, false>(c, a, ops);
}

// Triangles: lift, then the Euler pass or the two Navier-Stokes passes
// (tri_adjoint.cuh); the state and free-stream adjoints, no geometry adjoint.
template <int N>
static void launch_vjp_tri(Ctx &c, bool params, bool geo)
{
  if (geo) ZB_THROW(ZB_ERR_UNSUPPORTED, "the geometry adjoint is built for quadrilaterals and hexahedra");
  using G = dev::TriShape<N>;
  dev::AdjArgs a;
  std::memset(&a, 0, sizeof(a));
  a.U = (const double *)c.U;
  a.Ufp = (const double *)c.Ufp[c.cur];
  a.mets = (const double *)c.mets;
  a.fgeo = (const double *)c.fgeo;
  a.nbr = c.nbr;
  a.lam = c.lam;
  a.Lfp = c.Lfp;
  a.Ubfp = c.Ubfp;
  a.dUbfp = c.dUbfp;
  a.Ubx = c.Ubx;
  a.UCb = c.UCb;
  a.Ubar = c.Ubar;
  a.pbar = params ? c.pbar : nullptr;
  a.Fvn = (const double *)c.Fvn;
  a.dops = (const double *)c.dops;
  a.ntiles = c.ntiles;
  a.ph = phys_of<double>(c.plan.params, c.uref, 2, false);
  {
    ProfScope ps(c, ZB_K_ADJ_LIFT);
    dev::k_tri_adj_lift<N><<<grid_for(c.ntiles * G::Fp * TW, 128), 128, 0, c.stream>>>(a);
    c.launches++;
    CK(cudaGetLastError());
  }
  if (!c.plan.params.viscous)
  {
    const size_t smem = dev::tri_adj_euler_smem<N>();
    set_smem(dev::k_tri_adj_euler<N>, smem);
    ProfScope ps(c, ZB_K_ADJ_VOL);
    dev::k_tri_adj_euler<N><<<(unsigned)c.ntiles, 128, smem, c.stream>>>(a);
    c.launches++;
    CK(cudaGetLastError());
    return;
  }
  {
    const size_t smem1 = dev::tri_adj_ns1_smem<N>();
    set_smem(dev::k_tri_adj_ns1<N>, smem1);
    ProfScope ps(c, ZB_K_ADJ_VOL);
    dev::k_tri_adj_ns1<N><<<(unsigned)c.ntiles, 128, smem1, c.stream>>>(a);
    c.launches++;
    CK(cudaGetLastError());
  }
  const size_t smem2 = dev::tri_adj_ns2_smem<N>();
  set_smem(dev::k_tri_adj_ns2<N>, smem2);
  ProfScope ps(c, ZB_K_ADJ_TRACE);
  dev::k_tri_adj_ns2<N><<<(unsigned)c.ntiles, 128, smem2, c.stream>>>(a);
  c.launches++;
  CK(cudaGetLastError());
}

void bind_vjp(Ctx &c)
{
  c.launch_vjp = nullptr;
  if (c.plan.etype == ET_TRI)
  {
#define ZB_BIND_TRI(NN) \
  if (c.N == NN) { c.launch_vjp = &launch_vjp_tri<NN>; return; }
    ZB_BIND_TRI(2) ZB_BIND_TRI(3) ZB_BIND_TRI(4) ZB_BIND_TRI(5) ZB_BIND_TRI(6) ZB_BIND_TRI(7) ZB_BIND_TRI(8)
    ZB_BIND_TRI(9)
#undef ZB_BIND_TRI
    return;
  }
  // the adjoint's shared memory fits hexahedra up to P3
#define ZB_BIND(DD, NN) \
  if (c.D == DD && c.N == NN) { c.launch_vjp = &launch_vjp_impl<DD, NN>; return; }
  ZB_BIND(2, 2) ZB_BIND(2, 3) ZB_BIND(2, 4) ZB_BIND(2, 5) ZB_BIND(2, 6)
  ZB_BIND(3, 2) ZB_BIND(3, 3) ZB_BIND(3, 4)
#undef ZB_BIND
  c.launch_vjp = nullptr;
}

}  // namespace zb

// Residual entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc when they need a residual: a host
// application that owns every device byte through its own allocator, a plugin
// sandbox that forbids device allocation, or a time-critical loop that must not
// enter the driver's allocator.  zb_compute_residual_noalloc serves them: the
// caller passes the input state and the output residual as device pointers it
// already owns, and every intermediate (geometry in the kernels' layout, state
// tiles, flux-point states, viscous normal fluxes, residual tiles) lives in the
// file-scope device array below, which exists on every GPU that loads this
// library until the process exits.
//
// It computes the FP64 residual with the same kernels as zb_compute_residual:
// the column-mapped k_hex_* kernels for hexahedra (with the one-sided common
// flux under beta = +-1/2), the point-mapped kernels for quadrilaterals.
#include <cstring>
#include <mutex>

#include "ctx_impl.cuh"
#include "hex_kernels.cuh"

namespace zb {
namespace {

constexpr size_t kScratchBytes = size_t(32) << 20;  // 32 MiB per device

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void *g_scratch_addr[kMaxDevices] = {};

#define NA_CK(x)                                                                                \
  do                                                                                            \
  {                                                                                             \
    cudaError_t e_ = (x);                                                                       \
    if (e_ != cudaSuccess) ZB_THROW(ZB_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

using dev::TW;

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Per-device address of the scratch array; looked up on the first call made on
// each device, with that device current.
unsigned char *scratch_on_current_device()
{
  int d = 0;
  NA_CK(cudaGetDevice(&d));
  if (d < 0 || d >= kMaxDevices) ZB_THROW(ZB_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_mutex);
  if (!g_scratch_addr[d])
  {
    void *p = nullptr;
    NA_CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_scratch_addr[d] = p;
  }
  return static_cast<unsigned char *>(g_scratch_addr[d]);
}

// reference-layout geometry (staged in scratch) -> kernel layout
__global__ void k_na_pack(const double *__restrict__ inv_jaco, const double *__restrict__ det,
                          const double *__restrict__ fnorm, const double *__restrict__ fdA,
                          const int64_t *__restrict__ partner, const int8_t *__restrict__ slot, double *mets,
                          double *fgeo, int *nbr, int64_t E, int64_t ntiles, int S, int Fp, int D)
{
  const int NM = D * D + 1;
  const int64_t nmet = ntiles * S * TW, nfp = ntiles * Fp * TW;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nmet + nfp; i += (int64_t)gridDim.x * blockDim.x)
  {
    if (i < nmet)
    {
      const int l = (int)(i % TW);
      const int s = (int)((i / TW) % S);
      const int64_t t = i / ((int64_t)TW * S);
      const int64_t e = t * TW + l;
      const int64_t es = e < E ? e : 0;
      for (int d1 = 0; d1 < D; d1++)
        for (int d2 = 0; d2 < D; d2++)
          mets[((t * S + s) * NM + d1 * D + d2) * TW + l] = inv_jaco[(((int64_t)d1 * S + s) * D + d2) * E + es];
      mets[((t * S + s) * NM + D * D) * TW + l] = det[(int64_t)s * E + es];
    }
    else
    {
      const int64_t j = i - nmet;
      const int l = (int)(j % TW);
      const int f = (int)((j / TW) % Fp);
      const int64_t t = j / ((int64_t)TW * Fp);
      const int64_t e = t * TW + l;
      const bool pad = e >= E;
      const int64_t es = pad ? 0 : e;
      for (int d = 0; d < D; d++)
        fgeo[((t * Fp + f) * (D + 1) + d) * TW + l] = fnorm[((int64_t)f * D + d) * E + es];
      fgeo[((t * Fp + f) * (D + 1) + D) * TW + l] = fdA[(int64_t)f * E + es];
      int code;
      if (pad)
        code = (int)(2 * ((t * Fp + f) * TW + l));
      else
      {
        const int64_t pr = partner[(int64_t)f * E + e];
        if (pr < 0)
          code = (int)pr;
        else
        {
          const int64_t e2 = pr / Fp;
          const int f2 = (int)(pr % Fp);
          code = (int)(2 * (((e2 / TW) * Fp + f2) * TW + (e2 % TW)) + slot[(int64_t)f * E + e]);
        }
      }
      nbr[(t * Fp + f) * TW + l] = code;
    }
  }
}

__global__ void k_na_to_tiles(const double *__restrict__ src, double *__restrict__ dst, int64_t E, int64_t ntiles,
                              int S, int V)
{
  const int64_t total = ntiles * S * V * TW;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
  {
    const int l = (int)(i % TW);
    const int v = (int)((i / TW) % V);
    const int s = (int)((i / ((int64_t)TW * V)) % S);
    const int64_t t = i / ((int64_t)TW * V * S);
    int64_t e = t * TW + l;
    if (e >= E) e = 0;
    dst[i] = src[((int64_t)s * V + v) * E + e];
  }
}

__global__ void k_na_from_tiles(const double *__restrict__ src, double *__restrict__ dst, int64_t E, int S, int V)
{
  const int64_t total = E * S * V;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
  {
    const int64_t e = i % E;
    const int v = (int)((i / E) % V);
    const int s = (int)(i / (E * V));
    dst[i] = src[(((e / TW) * S + s) * V + v) * TW + (e % TW)];
  }
}

int blocks_for(int64_t work)
{
  int64_t b = (work + 255) / 256;
  if (b > 148 * 32) b = 148 * 32;
  return (int)(b < 1 ? 1 : b);
}

// hexahedral Navier-Stokes with beta = +-1/2: the gradient kernel forms the
// common flux at the flux points whose side supplies the LDG normal flux
bool one_sided_common_flux(const Plan &p)
{
  return p.ndims == 3 && p.params.viscous && (p.params.ldg_b == 0.5 || p.params.ldg_b == -0.5);
}

struct Regions
{
  size_t inv, det, fnorm, fdA, partner, slot, mets, fgeo, nbr, U, Ufp, divF, divF_vol, Fvn, Fcom, total;
};

Regions layout(const Plan &p)
{
  const size_t E = (size_t)p.neles, S = p.nspts, Fp = p.nfpts, D = p.ndims, V = p.nvars;
  const size_t nt = (size_t)p.ntiles;
  Regions r{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += align256(bytes);
    return o;
  };
  r.inv = take(D * S * D * E * 8);
  r.det = take(S * E * 8);
  r.fnorm = take(Fp * D * E * 8);
  r.fdA = take(Fp * E * 8);
  r.partner = take(Fp * E * 8);
  r.slot = take(Fp * E);
  r.mets = take(nt * S * (D * D + 1) * TW * 8);
  r.fgeo = take(nt * Fp * (D + 1) * TW * 8);
  r.nbr = take(nt * Fp * TW * 4);
  r.U = take(nt * S * V * TW * 8);
  r.Ufp = take(nt * Fp * V * TW * 8);
  r.divF = take(nt * S * V * TW * 8);
  r.divF_vol = p.params.viscous ? take(nt * S * V * TW * 8) : 0;
  r.Fvn = p.params.viscous ? take(nt * Fp * V * TW * 8) : 0;
  r.Fcom = one_sided_common_flux(p) ? take(nt * Fp * V * TW * 8) : 0;
  r.total = off;
  return r;
}

template <int N>
dev::LineOpsT<double, N> line_ops_d(const Plan &p)
{
  dev::LineOpsT<double, N> o;
  for (int i = 0; i < N * N; i++) o.Dm[i] = p.ops.D[i];
  for (int i = 0; i < N; i++)
  {
    o.Em[i] = p.ops.Em[i];
    o.Ep[i] = p.ops.Ep[i];
    o.Dbm[i] = p.ops.Dbm[i];
    o.Dbp[i] = p.ops.Dbp[i];
  }
  return o;
}

template <int D, int N>
void run_kernels(const Plan &p, unsigned char *base, const Regions &r, cudaStream_t st)
{
  using G = dev::Shape<D, N>;
  constexpr int S = G::S, Fp = G::Fp, V = G::V, NT = G::NT;
  const auto ops = line_ops_d<N>(p);
  dev::Args<double, double> a;
  std::memset(&a, 0, sizeof(a));
  a.U = reinterpret_cast<const double *>(base + r.U);
  a.Ufp = reinterpret_cast<const double *>(base + r.Ufp);
  a.mets = reinterpret_cast<const double *>(base + r.mets);
  a.fgeo = reinterpret_cast<const double *>(base + r.fgeo);
  a.nbr = reinterpret_cast<const int *>(base + r.nbr);
  a.divF = reinterpret_cast<double *>(base + r.divF);
  a.divF_vol = p.params.viscous ? reinterpret_cast<double *>(base + r.divF_vol) : nullptr;
  a.Fvn = p.params.viscous ? reinterpret_cast<double *>(base + r.Fvn) : nullptr;
  a.Fcom = one_sided_common_flux(p) ? reinterpret_cast<double *>(base + r.Fcom) : nullptr;
  a.ntiles = p.ntiles;
  const double zero_ref[5] = {0, 0, 0, 0, 0};
  a.ph = phys_of<double>(p.params, zero_ref, p.ndims, false);
  if constexpr (D == 3)
  {
    // hexahedra: column-mapped kernels, TW x N^2 threads per tile (ZS per column)
    constexpr int HT = TW * N * N;
    // with the one-sided common flux the gradient kernel forms the traces
    if (!a.Fcom)
    {
      dev::k_hex_extrap<double, double, N><<<(unsigned)p.ntiles, HT, 0, st>>>(
          a.U, reinterpret_cast<double *>(base + r.Ufp), p.ntiles, ops);
      NA_CK(cudaGetLastError());
    }
    if (!p.params.viscous)
    {
      const size_t smem = (size_t)(S * V + 3 * S * V + Fp * V) * TW * sizeof(double);
      NA_CK(cudaFuncSetAttribute(dev::k_hex_euler<double, double, N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
      dev::k_hex_euler<double, double, N><<<(unsigned)p.ntiles, HT, smem, st>>>(a, ops);
      NA_CK(cudaGetLastError());
    }
    else
    {
      constexpr int ZG = dev::HexNsShape<double, N>::grad_zs, ZF = dev::HexNsShape<double, N>::face_zs;
      const size_t smem1 = (size_t)((S * V + Fp * V + 3 * S * V) * TW + 3 * N * TW) * sizeof(double);
      NA_CK(cudaFuncSetAttribute(dev::k_hex_ns_grad<double, double, N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem1));
      dev::k_hex_ns_grad<double, double, N><<<(unsigned)p.ntiles, HT * ZG, smem1, st>>>(a, ops);
      NA_CK(cudaGetLastError());
      const size_t smem2 = (size_t)(Fp * V + S * V) * TW * sizeof(double);
      NA_CK(cudaFuncSetAttribute(dev::k_hex_ns_face<double, double, N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem2));
      dev::k_hex_ns_face<double, double, N><<<(unsigned)p.ntiles, HT * ZF, smem2, st>>>(a, ops);
      NA_CK(cudaGetLastError());
    }
    return;
  }
  dev::k_extrap<double, double, D, N><<<blocks_for(p.ntiles * Fp * TW), 256, 0, st>>>(
      a.U, reinterpret_cast<double *>(base + r.Ufp), p.ntiles, ops);
  NA_CK(cudaGetLastError());
  const size_t ob = sizeof(dev::LineOpsT<double, N>);
  if (!p.params.viscous)
  {
    const size_t smem = (size_t)(S * V + D * S * V + Fp * V) * TW * sizeof(double) + ob;
    NA_CK(cudaFuncSetAttribute(dev::k_euler<double, double, D, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dev::k_euler<double, double, D, N><<<(unsigned)p.ntiles, NT, smem, st>>>(a, ops);
    NA_CK(cudaGetLastError());
  }
  else
  {
    const size_t smem1 = (size_t)(S * V + Fp * V + D * S * V) * TW * sizeof(double) + ob;
    NA_CK(cudaFuncSetAttribute(dev::k_ns_grad<double, double, D, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem1));
    dev::k_ns_grad<double, double, D, N><<<(unsigned)p.ntiles, NT, smem1, st>>>(a, ops);
    NA_CK(cudaGetLastError());
    const size_t smem2 = (size_t)(Fp * V + S * V) * TW * sizeof(double) + ob;
    NA_CK(cudaFuncSetAttribute(dev::k_ns_face<double, double, D, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2));
    dev::k_ns_face<double, double, D, N><<<(unsigned)p.ntiles, NT, smem2, st>>>(a, ops);
    NA_CK(cudaGetLastError());
  }
}

void dispatch(const Plan &p, unsigned char *base, const Regions &r, cudaStream_t st)
{
  const int D = p.ndims, N = p.N;
  if (p.etype == ET_TRI) ZB_THROW(ZB_ERR_UNSUPPORTED, "the allocation-free residual is built for quads and hexes");
#define NA_CASE(DD, NN) \
  if (D == DD && N == NN) return run_kernels<DD, NN>(p, base, r, st);
  NA_CASE(2, 2) NA_CASE(2, 3) NA_CASE(2, 4) NA_CASE(2, 5) NA_CASE(2, 6)
  NA_CASE(3, 2) NA_CASE(3, 3) NA_CASE(3, 4) NA_CASE(3, 5)
#undef NA_CASE
  ZB_THROW(ZB_ERR_UNSUPPORTED, "no kernels built for this dimension and order");
}

}  // namespace

void noalloc_residual(const Plan &p, const double *U, double *divF, cudaStream_t st)
{
  if (!U || !divF) ZB_THROW(ZB_ERR_ARG, "null state or residual pointer");
  if (p.tile != TW) ZB_THROW(ZB_ERR_INTERNAL, "plan tile width does not match kernels");
  const Regions r = layout(p);
  if (r.total > kScratchBytes)
    ZB_THROW(ZB_ERR_ARG, "mesh needs " + std::to_string(r.total) + " bytes of scratch; the allocation-free residual "
             "holds at most " + std::to_string(kScratchBytes) + " bytes per device (use zb_compute_residual)");
  unsigned char *base = scratch_on_current_device();
  const size_t E = (size_t)p.neles, S = p.nspts, Fp = p.nfpts, D = p.ndims;
  // geometry: the plan's host arrays are copied in and packed on every call
  {
    NA_CK(cudaMemcpyAsync(base + r.inv, p.inv_jaco_spts.data(), D * S * D * E * 8, cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(base + r.det, p.jaco_det_spts.data(), S * E * 8, cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(base + r.fnorm, p.fnorm.data(), Fp * D * E * 8, cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(base + r.fdA, p.fdA.data(), Fp * E * 8, cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(base + r.partner, p.partner.data(), Fp * E * 8, cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(base + r.slot, p.slot.data(), Fp * E, cudaMemcpyHostToDevice, st));
    const int64_t work = p.ntiles * (S + Fp) * TW;
    k_na_pack<<<blocks_for(work), 256, 0, st>>>(
        reinterpret_cast<const double *>(base + r.inv), reinterpret_cast<const double *>(base + r.det),
        reinterpret_cast<const double *>(base + r.fnorm), reinterpret_cast<const double *>(base + r.fdA),
        reinterpret_cast<const int64_t *>(base + r.partner), reinterpret_cast<const int8_t *>(base + r.slot),
        reinterpret_cast<double *>(base + r.mets), reinterpret_cast<double *>(base + r.fgeo),
        reinterpret_cast<int *>(base + r.nbr), p.neles, p.ntiles, (int)S, (int)Fp, (int)D);
    NA_CK(cudaGetLastError());
  }
  // flux points skipped under beta = +-0.5 are never written; start them at zero
  if (p.params.viscous)
    NA_CK(cudaMemsetAsync(base + r.Fvn, 0, (size_t)p.ntiles * Fp * p.nvars * TW * 8, st));
  if (one_sided_common_flux(p))
    NA_CK(cudaMemsetAsync(base + r.Fcom, 0, (size_t)p.ntiles * Fp * p.nvars * TW * 8, st));
  k_na_to_tiles<<<blocks_for(p.ntiles * S * p.nvars * TW), 256, 0, st>>>(
      U, reinterpret_cast<double *>(base + r.U), p.neles, p.ntiles, (int)S, p.nvars);
  NA_CK(cudaGetLastError());
  dispatch(p, base, r, st);
  k_na_from_tiles<<<blocks_for((int64_t)E * S * p.nvars), 256, 0, st>>>(
      reinterpret_cast<const double *>(base + r.divF), divF, p.neles, (int)S, p.nvars);
  NA_CK(cudaGetLastError());
}

}  // namespace zb

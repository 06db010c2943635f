// Hexahedron DFR kernels with a column mapping (sum factorisation).
//
// One CTA processes one tile of TW elements with TW x N^2 threads: thread
// (l, ix, iy) owns the z-column of solution points (ix, iy, 0..N-1) of element
// l and exactly six flux points, one on each face:
//   face 0 (z-) and 1 (z+) at (x=ix, y=iy)    -- the ends of its own column,
//   face 2 (x-) and 3 (x+) at (y=iy, z=ix),
//   face 4 (y-) and 5 (y+) at (x=ix, z=iy),
// so the N^2 threads of an element cover its 6 N^2 flux points once.  z-lines
// live in registers; x- and y-lines are read from shared memory; the line
// operator rows a thread needs are held in registers.  Arithmetic and
// summation order are those of the generic kernels in dfr_kernels.cuh, which
// follow the reference's operator products (src/elements.cpp:1337-1501).
#pragma once

#include "dfr_kernels.cuh"

namespace zb {
namespace dev {

template <int N>
struct HexIdx
{
  static constexpr int N2 = N * N, S = N * N * N, Fp = 6 * N * N;
  // flux point ids of the thread's six flux points
  static __device__ __forceinline__ void fpts(int ix, int iy, int f[6])
  {
    f[0] = iy * N + ix;                        // z-  (x = ix, y = iy)
    f[1] = N2 + iy * N + (N - 1 - ix);         // z+
    f[2] = 2 * N2 + ix * N + iy;               // x-  (y = iy, z = ix)
    f[3] = 3 * N2 + ix * N + (N - 1 - iy);     // x+
    f[4] = 4 * N2 + iy * N + (N - 1 - ix);     // y-  (x = ix, z = iy)
    f[5] = 5 * N2 + iy * N + ix;               // y+
  }
  // id of own flux point q (same order as fpts)
  static __device__ __forceinline__ int fpt(int q, int ix, int iy)
  {
    switch (q)
    {
      case 0: return iy * N + ix;
      case 1: return N2 + iy * N + (N - 1 - ix);
      case 2: return 2 * N2 + ix * N + iy;
      case 3: return 3 * N2 + ix * N + (N - 1 - iy);
      case 4: return 4 * N2 + iy * N + (N - 1 - ix);
      default: return 5 * N2 + iy * N + ix;
    }
  }
  // solution point on the normal line of own flux point q at position m
  static __device__ __forceinline__ int line_spt(int q, int ix, int iy, int m)
  {
    if (q < 2) return ix + N * iy + N2 * m;    // z-line through (ix, iy)
    if (q < 4) return m + N * iy + N2 * ix;    // x-line at (y = iy, z = ix)
    return ix + N * m + N2 * iy;               // y-line at (x = ix, z = iy)
  }
  // x- and y-face flux points at the ends of the lines through spt (ix, iy, iz)
  static __device__ __forceinline__ int fxm(int iy, int iz) { return 2 * N2 + iz * N + iy; }
  static __device__ __forceinline__ int fxp(int iy, int iz) { return 3 * N2 + iz * N + (N - 1 - iy); }
  static __device__ __forceinline__ int fym(int ix, int iz) { return 4 * N2 + iz * N + (N - 1 - ix); }
  static __device__ __forceinline__ int fyp(int ix, int iz) { return 5 * N2 + iz * N + ix; }
};

// The line-operator rows of a thread's x and y coordinates, in registers; the
// z row (uniform across a warp inside a z loop) is read from the kernel
// parameter.
template <typename A, int N>
struct RowOps
{
  A Dx[N], Dy[N], dbxm, dbxp, dbym, dbyp;
  __device__ __forceinline__ void load(const LineOpsT<A, N> &o, int ix, int iy)
  {
#pragma unroll
    for (int m = 0; m < N; m++)
    {
      Dx[m] = o.Dm[ix * N + m];
      Dy[m] = o.Dm[iy * N + m];
    }
    dbxm = o.Dbm[ix];
    dbxp = o.Dbp[ix];
    dbym = o.Dbm[iy];
    dbyp = o.Dbp[iy];
  }
};

// Two variables of a point at once in FP32: the paired FP32 instructions of
// sm_100 (FFMA2, FMUL2, FADD2) take float2 operands and round each lane as
// the scalar instruction does.  Variables v and v + 1 of a point lie TW
// apart in the tile arrays.
struct F2
{
  static __device__ __forceinline__ float2 dup(float x) { return make_float2(x, x); }
  static __device__ __forceinline__ float2 ld(const float *p) { return make_float2(p[0], p[TW]); }
  static __device__ __forceinline__ void st(float *p, float2 x)
  {
    p[0] = x.x;
    p[TW] = x.y;
  }
};

// own flux point q (0..5): side of the face
__device__ __forceinline__ bool q_minus(int q) { return (q & 1) == 0; }

// k-th of the own flux points a thread handles when ZS threads share a column:
// all six for ZS = 1; for ZS = 2 half 0 takes faces z-, x+, y- and half 1
// takes z+, x-, y+, so the work done by only one side of a face (the LDG
// normal flux, usually the side with the + face) is spread over both halves
template <int ZS>
__device__ __forceinline__ int own_face(int zs, int k)
{
  return ZS == 1 ? k : 2 * k + ((zs + k) & 1);
}

template <typename T, typename A, int N>
__device__ __forceinline__ void load_face_geo(const Args<T, A> &a, int64_t tile, int f, int l, A n[3], A &dA, int &code)
{
  using H = HexIdx<N>;
  const T *g = a.fgeo + (tile * H::Fp + f) * (int64_t)4 * TW + l;
  n[0] = g[0];
  n[1] = g[TW];
  n[2] = g[2 * TW];
  dA = g[3 * TW];
  code = a.nbr[(tile * H::Fp + f) * (int64_t)TW + l];
}

// ---------------------------------------------------------------------------
// state -> flux points (src/elements.cpp:1337-1360)
// ---------------------------------------------------------------------------
template <typename T, typename A, int N>
__global__ void __launch_bounds__(TW * N * N) k_hex_extrap(const T *__restrict__ U, T *__restrict__ Ufp, int64_t ntiles,
                                                           const __grid_constant__ LineOpsT<A, N> ops)
{
  using H = HexIdx<N>;
  constexpr int S = H::S, V = 5;
  const int l = threadIdx.x % TW, c = threadIdx.x / TW, ix = c % N, iy = c / N;
  const int64_t tile = blockIdx.x;
  if (tile >= ntiles) return;
  const T *Ut = U + tile * (int64_t)S * V * TW;
  int f[6];
  H::fpts(ix, iy, f);
#pragma unroll
  for (int q = 0; q < 6; q++)
  {
    T *out = Ufp + (tile * H::Fp + f[q]) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      A acc = (q_minus(q) ? ops.Em[0] : ops.Ep[0]) * Ut[(H::line_spt(q, ix, iy, 0) * V + v) * TW + l];
#pragma unroll
      for (int m = 1; m < N; m++)
        acc += (q_minus(q) ? ops.Em[m] : ops.Ep[m]) * Ut[(H::line_spt(q, ix, iy, m) * V + v) * TW + l];
      out[v * TW] = acc;
    }
  }
}

// ---------------------------------------------------------------------------
// common convective (+LDG) flux at the thread's six flux points, dA-scaled and
// signed for this element, into sFc [Fp][V][TW]
// ---------------------------------------------------------------------------
template <typename T, typename A, int N, bool VISC, int ZS = 1>
__device__ __forceinline__ void hex_common_flux(const Args<T, A> &a, int64_t tile, int l, int ix, int iy, A *sFc,
                                                int zs = 0)
{
  using H = HexIdx<N>;
  constexpr int V = 5;
  const A beta = a.ph.ldg_b, tau = a.ph.ldg_tau;
#pragma unroll 1
  for (int k = 0; k < 6 / ZS; k++)
  {
    const int q = own_face<ZS>(zs, k);
    const int fq = H::fpt(q, ix, iy);
    A n[3], dA;
    int code;
    load_face_geo<T, A, N>(a, tile, fq, l, n, dA, code);
    A Uo[V], Un[V], UL[V], UR[V], UB[V], Fc[V];
    const T *uo = a.Ufp + (tile * H::Fp + fq) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++) Uo[v] = uo[v * TW];
    if (code >= 0) gather_fpt<T, A, V>(a.Ufp, code >> 1, Un);
    conv_common<T, A, 3>(a, Uo, Un, code, n, UL, UR, UB, Fc);
    const bool right = (code >= 0) && (code & 1);
    A Fv[V];
    if (VISC)
    {
      const T *fvo = a.Fvn + (tile * H::Fp + fq) * (int64_t)V * TW + l;
      if (code >= 0)
      {
        const int slot = code & 1;
        A FnL[V], FnR[V];
        if (beta == A(0.5))
        {
          if (slot == 0)
          {
#pragma unroll
            for (int v = 0; v < V; v++) FnL[v] = fvo[v * TW];
          }
          else
            gather_fpt<T, A, V>(a.Fvn, code >> 1, FnL);
#pragma unroll
          for (int v = 0; v < V; v++) FnR[v] = A(0);
        }
        else if (beta == A(-0.5))
        {
          if (slot == 1)
          {
#pragma unroll
            for (int v = 0; v < V; v++) FnR[v] = fvo[v * TW];
          }
          else
            gather_fpt<T, A, V>(a.Fvn, code >> 1, FnR);
#pragma unroll
          for (int v = 0; v < V; v++) FnL[v] = A(0);
        }
        else
        {
          A Fo[V], Fx[V];
#pragma unroll
          for (int v = 0; v < V; v++) Fo[v] = fvo[v * TW];
          gather_fpt<T, A, V>(a.Fvn, code >> 1, Fx);
#pragma unroll
          for (int v = 0; v < V; v++)
          {
            FnL[v] = slot ? Fx[v] : Fo[v];
            FnR[v] = slot ? Fo[v] : Fx[v];
          }
        }
#pragma unroll
        for (int v = 0; v < V; v++)
          Fv[v] = A(0.5) * (FnL[v] + FnR[v]) + tau * (UL[v] - UR[v]) + beta * (FnL[v] - FnR[v]);
      }
      else
      {
#pragma unroll
        for (int v = 0; v < V; v++) Fv[v] = fvo[v * TW] + tau * (UL[v] - UB[v]);
      }
    }
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      A acc = right ? -Fc[v] * dA : Fc[v] * dA;
      if (VISC)
      {
        if (right)
          acc -= Fv[v] * dA;
        else
          acc += Fv[v] * dA;
      }
      sFc[(fq * V + v) * TW + l] = acc;
    }
  }
}

// common flux formed by the gradient kernel (Args::Fcom) at the thread's flux
// points: read from this element where it supplied the LDG normal flux, else
// from the partner's flux point; dA-scaled and signed for this element
template <typename T, typename A, int N, int ZS = 1>
__device__ __forceinline__ void hex_gather_common(const Args<T, A> &a, int64_t tile, int l, int ix, int iy, A *sFc,
                                                  int zs = 0)
{
  using H = HexIdx<N>;
  constexpr int V = 5;
  const int supplier = a.ph.ldg_b == A(0.5) ? 0 : 1;  // slot whose normal flux LDG takes
#pragma unroll
  for (int k = 0; k < 6 / ZS; k++)
  {
    const int q = own_face<ZS>(zs, k);
    const int fq = H::fpt(q, ix, iy);
    const int64_t gi = (tile * H::Fp + fq) * (int64_t)TW + l;
    const A dA = a.fgeo[(tile * H::Fp + fq) * (int64_t)4 * TW + 3 * TW + l];
    const int code = a.nbr[gi];
    A F[V];
    if (code < 0 || (code & 1) == supplier)
    {
      const T *fc = a.Fcom + (tile * H::Fp + fq) * (int64_t)V * TW + l;
#pragma unroll
      for (int v = 0; v < V; v++) F[v] = fc[v * TW];
    }
    else
      gather_fpt<T, A, V>(a.Fcom, code >> 1, F);
    const bool right = (code >= 0) && (code & 1);
#pragma unroll
    for (int v = 0; v < V; v++) sFc[(fq * V + v) * TW + l] = right ? -F[v] * dA : F[v] * dA;
  }
}

// surface correction for spt (ix, iy, iz) in flux-point order (faces 0..5)
template <typename A, int N>
__device__ __forceinline__ A hex_surface(const LineOpsT<A, N> &ops, const RowOps<A, N> &o, const A *sFc, int ix, int iy,
                                         int iz, int v, int l)
{
  using H = HexIdx<N>;
  constexpr int V = 5;
  A s = A(0);
  s += -ops.Dbm[iz] * sFc[((iy * N + ix) * V + v) * TW + l];
  s += ops.Dbp[iz] * sFc[((H::N2 + iy * N + (N - 1 - ix)) * V + v) * TW + l];
  s += -o.dbxm * sFc[(H::fxm(iy, iz) * V + v) * TW + l];
  s += o.dbxp * sFc[(H::fxp(iy, iz) * V + v) * TW + l];
  s += -o.dbym * sFc[(H::fym(ix, iz) * V + v) * TW + l];
  s += o.dbyp * sFc[(H::fyp(ix, iz) * V + v) * TW + l];
  return s;
}

// RK update of one spt and optional staging of the new state for extrapolation
// (src/solver.cpp:2916-2937, 3040-3094).  Every load of the point (RK start
// state, earlier residual registers, compensation remainder) is issued before
// the first store: the compiler cannot move a load above a store that may
// alias it, so interleaving them would serialise the point's memory accesses.
template <typename T, typename A, int N>
__device__ __forceinline__ void hex_finish(const Args<T, A> &a, int64_t tile, int s, int l, const A res[5], A *sUnew)
{
  using H = HexIdx<N>;
  constexpr int V = 5, NM = 10, MAXPREV = 3;
  const int64_t base = (tile * H::S + s) * (int64_t)V * TW;
  if (a.rk_mode == 0)
  {
#pragma unroll
    for (int v = 0; v < V; v++) a.divF[base + v * TW + l] = res[v];
    return;
  }
  const A detJ = a.mets[((tile * H::S + s) * NM + 9) * TW + l];
  const A dtv = step_dt(a, tile, l);
  const bool fast = a.rk_mode == 1 || a.nprev <= MAXPREV;
  A u_ini[V], prev[MAXPREV][V], comp[V];
#pragma unroll
  for (int v = 0; v < V; v++)
  {
    const int64_t idx = base + v * TW + l;
    // U_ini (after stage 0) and the earlier residual registers are not
    // written by this kernel: read-only loads, free to move above the stores
    // of the thread's other points
    u_ini[v] = a.save_ini ? (A)a.U[idx] : (A)__ldg(a.U_ini + idx);
    comp[v] = (a.rk_mode == 2 && a.Ucomp) ? (A)a.Ucomp[idx] : A(0);
  }
  if (a.rk_mode == 2 && fast)
  {
#pragma unroll
    for (int st = 0; st < MAXPREV; st++)
      if (st < a.nprev)
      {
#pragma unroll
        for (int v = 0; v < V; v++) prev[st][v] = (A)__ldg(a.divF_prev[st] + base + v * TW + l);
      }
  }
#pragma unroll
  for (int v = 0; v < V; v++) a.divF[base + v * TW + l] = res[v];
#pragma unroll
  for (int v = 0; v < V; v++)
  {
    const int64_t idx = base + v * TW + l;
    if (a.save_ini) a.U_ini[idx] = u_ini[v];
    A unew;
    if (a.rk_mode == 1)
      unew = u_ini[v] - a.rk_coef[0] * dtv / detJ * res[v];
    else if (a.Ucomp)
    {
      // Kahan-compensated step increment; the remainder includes the
      // rounding of the stored state
      A delta = A(0);
      if (fast)
      {
#pragma unroll
        for (int st = 0; st < MAXPREV; st++)
          if (st < a.nprev) delta -= a.rk_coef[st] * dtv / detJ * prev[st][v];
      }
      else
        for (int st = 0; st < a.nprev; st++) delta -= a.rk_coef[st] * dtv / detJ * (A)a.divF_prev[st][idx];
      delta -= a.rk_coef[a.nprev] * dtv / detJ * res[v];
      const A y = delta - comp[v];
      unew = (A)(T)(u_ini[v] + y);
      a.Ucomp[idx] = (T)((unew - u_ini[v]) - y);
    }
    else
    {
      unew = u_ini[v];
      if (fast)
      {
#pragma unroll
        for (int st = 0; st < MAXPREV; st++)
          if (st < a.nprev) unew -= a.rk_coef[st] * dtv / detJ * prev[st][v];
      }
      else
        for (int st = 0; st < a.nprev; st++) unew -= a.rk_coef[st] * dtv / detJ * a.divF_prev[st][idx];
      unew -= a.rk_coef[a.nprev] * dtv / detJ * res[v];
    }
    a.Uout[idx] = unew;
    if (sUnew) sUnew[(s * V + v) * TW + l] = (A)(T)unew;  // the state as stored
  }
}

template <typename T, typename A, int N, int ZS = 1>
__device__ __forceinline__ void hex_extrap_next(const Args<T, A> &a, int64_t tile, int l, int ix, int iy, const int f[6],
                                                const A *sUnew, const LineOpsT<A, N> &o, int zs = 0)
{
  using H = HexIdx<N>;
  constexpr int V = 5;
#pragma unroll
  for (int k = 0; k < 6 / ZS; k++)
  {
    const int q = own_face<ZS>(zs, k);
    T *out = a.Ufp_next + (tile * H::Fp + (ZS == 1 ? f[q] : H::fpt(q, ix, iy))) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      A acc = (q_minus(q) ? o.Em[0] : o.Ep[0]) * sUnew[(H::line_spt(q, ix, iy, 0) * V + v) * TW + l];
#pragma unroll
      for (int m = 1; m < N; m++)
        acc += (q_minus(q) ? o.Em[m] : o.Ep[m]) * sUnew[(H::line_spt(q, ix, iy, m) * V + v) * TW + l];
      out[v * TW] = acc;
    }
  }
}

// Trace of the state at the flux point with tile-layout index pidx
// ((tile * Fp + f) * TW + lane, the partner index of a connectivity code),
// formed from that element's state along the line normal to its face with
// the extrapolation's arithmetic (k_hex_extrap), so the same values.
template <typename T, typename A, int N>
__device__ __forceinline__ void hex_partner_trace(const T *__restrict__ U, const LineOpsT<A, N> &ops, int pidx,
                                                  A out[5])
{
  using H = HexIdx<N>;
  constexpr int V = 5;
  const int lane = pidx % TW, pt = pidx / TW;
  const int64_t ptile = pt / H::Fp;
  const int f = pt % H::Fp, q = f / H::N2, r = f % H::N2;
  // invert H::fpt: the (ix, iy) of the column that owns flux point f on face q
  int ix, iy;
  switch (q)
  {
    case 0: ix = r % N; iy = r / N; break;
    case 1: ix = N - 1 - r % N; iy = r / N; break;
    case 2: ix = r / N; iy = r % N; break;
    case 3: ix = r / N; iy = N - 1 - r % N; break;
    case 4: ix = N - 1 - r % N; iy = r / N; break;
    default: ix = r % N; iy = r / N; break;
  }
  const T *Up = U + ptile * (int64_t)H::S * V * TW + lane;
  const bool minus = q_minus(q);
#pragma unroll
  for (int v = 0; v < V; v++)
  {
    A acc = (minus ? ops.Em[0] : ops.Ep[0]) * Up[(H::line_spt(q, ix, iy, 0) * V + v) * TW];
#pragma unroll
    for (int m = 1; m < N; m++) acc += (minus ? ops.Em[m] : ops.Ep[m]) * Up[(H::line_spt(q, ix, iy, m) * V + v) * TW];
    out[v] = acc;
  }
}

// Own trace at own flux point q of column (ix, iy) from the state tile in
// shared memory ([S][V][TW]), with the extrapolation's arithmetic
template <typename A, int N>
__device__ __forceinline__ void hex_own_trace(const LineOpsT<A, N> &ops, const A *sU, int q, int ix, int iy, int l,
                                              A out[5])
{
  using H = HexIdx<N>;
  constexpr int V = 5;
#pragma unroll
  for (int v = 0; v < V; v++)
  {
    A acc = (q_minus(q) ? ops.Em[0] : ops.Ep[0]) * sU[(H::line_spt(q, ix, iy, 0) * V + v) * TW + l];
#pragma unroll
    for (int m = 1; m < N; m++)
      acc += (q_minus(q) ? ops.Em[m] : ops.Ep[m]) * sU[(H::line_spt(q, ix, iy, m) * V + v) * TW + l];
    out[v] = acc;
  }
}

template <typename T, typename A>
__device__ __forceinline__ void load_adj(const Args<T, A> &a, int64_t tile, int S, int s, int l, A adj[3][3], A &det)
{
  const T *m = a.mets + (tile * S + s) * (int64_t)10 * TW + l;
#pragma unroll
  for (int d1 = 0; d1 < 3; d1++)
#pragma unroll
    for (int d2 = 0; d2 < 3; d2++) adj[d1][d2] = m[(d1 * 3 + d2) * TW];
  det = m[9 * TW];
}

// ---------------------------------------------------------------------------
// Euler: volume flux, common flux, divergence (+RK, +next extrapolation)
// ---------------------------------------------------------------------------
template <typename T, typename A, int N>
__global__ void __launch_bounds__(TW * N * N) k_hex_euler(const __grid_constant__ Args<T, A> a,
                                                          const __grid_constant__ LineOpsT<A, N> ops)
{
  using H = HexIdx<N>;
  constexpr int S = H::S, V = 5;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  A *sU = reinterpret_cast<A *>(smem_raw);   // [S][V][TW] state, then new state
  A *sF = sU + S * V * TW;                   // [3][S][V][TW] transformed flux
  A *sFc = sF + 3 * S * V * TW;              // [Fp][V][TW]
  const int l = threadIdx.x % TW, c = threadIdx.x / TW, ix = c % N, iy = c / N;
  const int64_t tile = blockIdx.x;
  if (tile >= a.ntiles) return;
  RowOps<A, N> o;
  o.load(ops, ix, iy);
  int f[6];
  H::fpts(ix, iy, f);
  const T *Ut = a.U + tile * (int64_t)S * V * TW;
#pragma unroll 1
  for (int iz = 0; iz < N; iz++)
  {
    const int s = ix + N * iy + H::N2 * iz;
    A U[V], F[V][3], P, Pp, adj[3][3], det;
#pragma unroll
    for (int v = 0; v < V; v++) U[v] = Ut[(s * V + v) * TW + l];
    flux_conv_stored<A, 3>(U, F, P, Pp, a.ph);
    load_adj<T, A>(a, tile, S, s, l, adj, det);
#pragma unroll
    for (int v = 0; v < V; v++)
#pragma unroll
      for (int d1 = 0; d1 < 3; d1++)
      {
        A t = F[v][0] * adj[d1][0];
        t += F[v][1] * adj[d1][1];
        t += F[v][2] * adj[d1][2];
        sF[((d1 * S + s) * V + v) * TW + l] = t;
      }
  }
  hex_common_flux<T, A, N, false>(a, tile, l, ix, iy, sFc);
  __syncthreads();
#pragma unroll 1
  for (int iz = 0; iz < N; iz++)
  {
    const int s = ix + N * iy + H::N2 * iz;
    A res[V];
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      A vol = A(0);
#pragma unroll
      for (int m = 0; m < N; m++) vol += o.Dx[m] * sF[((0 * S + m + N * iy + H::N2 * iz) * V + v) * TW + l];
#pragma unroll
      for (int m = 0; m < N; m++) vol += o.Dy[m] * sF[((1 * S + ix + N * m + H::N2 * iz) * V + v) * TW + l];
#pragma unroll
      for (int m = 0; m < N; m++) vol += ops.Dm[iz * N + m] * sF[((2 * S + ix + N * iy + H::N2 * m) * V + v) * TW + l];
      res[v] = vol + hex_surface<A, N>(ops, o, sFc, ix, iy, iz, v, l);
    }
    hex_finish<T, A, N>(a, tile, s, l, res, a.extrap_next ? sU : nullptr);
  }
  if (a.extrap_next)
  {
    __syncthreads();
    hex_extrap_next<T, A, N>(a, tile, l, ix, iy, f, sU, ops);
  }
}

// ---------------------------------------------------------------------------
// Launch shape of the Navier-Stokes kernels.  zs = 2 splits each (element,
// x, y) column between two threads (z-levels and flux points by halves),
// doubling the warps per CTA for the same shared memory; minb is the CTAs per
// SM the register allocation is held to (0: the compiler's choice).  Chosen by
// timing P3 on B200: the split pays for the gradient kernel in both
// precisions and for the face kernel in FP64 only.  The FP64 face kernel is
// held to three CTAs per SM (80 registers; some of the RK update's values
// spill): 0.43 against 0.47 ms per residual at two CTAs, 0.57 at four.
// ---------------------------------------------------------------------------
template <typename A, int N>
struct HexNsShape
{
  static constexpr int grad_zs = (N % 2 == 0) ? 2 : 1;
  static constexpr int grad_minb = grad_zs == 2 ? (sizeof(A) == 4 ? 4 : 2) : 0;
  static constexpr int face_zs = (N % 2 == 0 && sizeof(A) == 8) ? 2 : 1;
  static constexpr int face_minb = face_zs == 2 ? 3 : 0;
};

// ---------------------------------------------------------------------------
// Navier-Stokes kernel 1 (column mapping): common solution, gradient, viscous
// normal flux at own flux points, flux, volume divergence
// ---------------------------------------------------------------------------
template <typename T, typename A, int N>
__global__ void __launch_bounds__(TW * N * N * HexNsShape<A, N>::grad_zs, HexNsShape<A, N>::grad_minb)
    k_hex_ns_grad(const __grid_constant__ Args<T, A> a, const __grid_constant__ LineOpsT<A, N> ops)
{
  using H = HexIdx<N>;
  constexpr int ZS = HexNsShape<A, N>::grad_zs;
  constexpr int S = H::S, Fp = H::Fp, V = 5, NZ = N / ZS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  A *sU = reinterpret_cast<A *>(smem_raw);   // [S][V][TW]
  A *sUC = sU + S * V * TW;                  // [Fp][V][TW] common solution
  A *sX = sUC + Fp * V * TW;                 // [3][S][V][TW] physical gradient, then F~
  // sX is padded by TW words per z-level: the lanes of a warp differ in x, so
  // along an x-line (viscous flux at x-faces) they read points N^2 apart,
  // which would otherwise fall in one bank group
  const auto xo = [](int p) { return p * V * TW + TW * (p / H::N2); };
  const int l = threadIdx.x % TW, c = (threadIdx.x / TW) % H::N2, zs = threadIdx.x / (TW * H::N2);
  const int ix = c % N, iy = c / N, iz0 = zs * NZ;
  const int64_t tile = blockIdx.x;
  if (tile >= a.ntiles) return;
  // the tile's metrics (gradient and flux passes) and face geometry (viscous
  // pass) on their way to L2 while the state and partner traces load; the
  // state and codes of the tile one wave of resident CTAs ahead (2 per SM)
  if (threadIdx.x == 0)
  {
    prefetch_l2(a.mets + tile * (int64_t)S * 10 * TW, S * 10 * TW * sizeof(T));
    prefetch_l2(a.fgeo + tile * (int64_t)Fp * 4 * TW, Fp * 4 * TW * sizeof(T));
    const int64_t ahead = tile + 2 * 148;
    if (ahead < a.ntiles)
    {
      prefetch_l2(a.U + ahead * (int64_t)S * V * TW, S * V * TW * sizeof(T));
      prefetch_l2(a.nbr + ahead * (int64_t)Fp * TW, Fp * TW * sizeof(int));
    }
  }
  RowOps<A, N> o;
  o.load(ops, ix, iy);
  int f[6];
  H::fpts(ix, iy, f);
  const A beta = a.ph.ldg_b;
  // own part of the column of the state -> shared memory
  {
    const T *Ut = a.U + tile * (int64_t)S * V * TW;
#pragma unroll
    for (int k = 0; k < NZ; k++)
#pragma unroll
      for (int v = 0; v < V; v++)
      {
        const int s = ix + N * iy + H::N2 * (iz0 + k);
        sU[(s * V + v) * TW + l] = Ut[(s * V + v) * TW + l];
      }
  }
  // common solution at own flux points (LDG, flip_beta = 1).  The points'
  // connectivity codes stay in registers for the viscous pass.
  int codes[6 / ZS];
  if (a.Fcom)
  {
    // One-sided LDG (beta = +-1/2): no trace buffer.  The side that takes the
    // partner's trace forms it from the partner's state line (all such
    // gathers in flight together, before the barrier that completes the
    // state tile); the other side and boundary points use the own trace,
    // formed from the state tile afterwards.
    const int supplier = beta == A(0.5) ? 0 : 1;
    A Un[6 / ZS][V];
#pragma unroll
    for (int kq = 0; kq < 6 / ZS; kq++)
    {
      const int fq = H::fpt(own_face<ZS>(zs, kq), ix, iy);
      const int code = a.nbr[(tile * Fp + fq) * (int64_t)TW + l];
      codes[kq] = code;
      if (code >= 0 && (code & 1) == supplier) hex_partner_trace<T, A, N>(a.U, ops, code >> 1, Un[kq]);
    }
    __syncthreads();
#pragma unroll
    for (int kq = 0; kq < 6 / ZS; kq++)
    {
      const int q = own_face<ZS>(zs, kq);
      const int fq = H::fpt(q, ix, iy);
      const int code = codes[kq];
      A UC[V];
      if (code >= 0 && (code & 1) == supplier)
      {
#pragma unroll
        for (int v = 0; v < V; v++) UC[v] = Un[kq][v];
      }
      else
      {
        A Uo[V];
        hex_own_trace<A, N>(ops, sU, q, ix, iy, l, Uo);
        if (code >= 0)
        {
#pragma unroll
          for (int v = 0; v < V; v++) UC[v] = Uo[v];
        }
        else
        {
          A n[3], dA;
          int c2;
          load_face_geo<T, A, N>(a, tile, fq, l, n, dA, c2);
          A Ua[V], URa[V], UBa[V];
          to_abs<A, 3>(Uo, Ua, a.ph);
          ghost_state<A, 3>(-code - 1, Ua, n, URa, UBa, a.ph);
          to_stored<A, 3>(UBa, UC, a.ph);
        }
      }
#pragma unroll
      for (int v = 0; v < V; v++) sUC[(fq * V + v) * TW + l] = UC[v];
    }
  }
  else
  {
    // traces from the trace buffer; unrolled so the partner gathers of all
    // points are in flight together
#pragma unroll
    for (int kq = 0; kq < 6 / ZS; kq++)
    {
      const int q = own_face<ZS>(zs, kq);
      const int fq = H::fpt(q, ix, iy);
      A n[3], dA;
      int code;
      load_face_geo<T, A, N>(a, tile, fq, l, n, dA, code);
      codes[kq] = code;
      A Uo[V], UC[V];
      const T *uo = a.Ufp + (tile * Fp + fq) * (int64_t)V * TW + l;
#pragma unroll
      for (int v = 0; v < V; v++) Uo[v] = uo[v * TW];
      if (code >= 0)
      {
        const int slot = code & 1;
        if ((beta == A(0.5) && slot) || (beta == A(-0.5) && !slot))
        {
          // beta = +1/2 (-1/2) takes the right (left) trace: this side's own,
          // no partner gather
#pragma unroll
          for (int v = 0; v < V; v++) UC[v] = Uo[v];
        }
        else
        {
          A Un[V];
          gather_fpt<T, A, V>(a.Ufp, code >> 1, Un);
#pragma unroll
          for (int v = 0; v < V; v++)
          {
            const A ul = slot ? Un[v] : Uo[v];
            const A ur = slot ? Uo[v] : Un[v];
            if (beta == A(0.5))
              UC[v] = ur;
            else if (beta == A(-0.5))
              UC[v] = ul;
            else
              UC[v] = A(0.5) * (ul + ur) - beta * (ul - ur);
          }
        }
      }
      else
      {
        A Ua[V], URa[V], UBa[V];
        to_abs<A, 3>(Uo, Ua, a.ph);
        ghost_state<A, 3>(-code - 1, Ua, n, URa, UBa, a.ph);
        to_stored<A, 3>(UBa, UC, a.ph);
      }
#pragma unroll
      for (int v = 0; v < V; v++) sUC[(fq * V + v) * TW + l] = UC[v];
    }
  }
  __syncthreads();
  // corrected reference gradient -> physical gradient
  const int fzm = H::fpt(0, ix, iy), fzp = H::fpt(1, ix, iy);
#pragma unroll 1
  for (int iz = iz0; iz < iz0 + NZ; iz++)
  {
    const int s = ix + N * iy + H::N2 * iz;
    const int fxm = H::fxm(iy, iz), fxp = H::fxp(iy, iz), fym = H::fym(ix, iz), fyp = H::fyp(ix, iz);
    A adj[3][3], det;
    load_adj<T, A>(a, tile, S, s, l, adj, det);
    const A inv_det = A(1) / det;
    if constexpr (sizeof(A) == 4)
    {
      // FP32: variables 0-3 in pairs on the paired FP32 instructions, the
      // fifth in the loop below
#pragma unroll
      for (int v = 0; v < V - 1; v += 2)
      {
        float2 td[3];
        {
          float2 acc = __fmul2_rn(F2::dup(o.Dx[0]), F2::ld(sU + ((N * iy + H::N2 * iz) * V + v) * TW + l));
#pragma unroll
          for (int m = 1; m < N; m++)
            acc = __ffma2_rn(F2::dup(o.Dx[m]), F2::ld(sU + ((m + N * iy + H::N2 * iz) * V + v) * TW + l), acc);
          const float2 cm = __fmul2_rn(F2::dup(o.dbxm), F2::ld(sUC + (fxm * V + v) * TW + l));
          td[0] = __fadd2_rn(acc, __ffma2_rn(F2::dup(o.dbxp), F2::ld(sUC + (fxp * V + v) * TW + l), cm));
        }
        {
          float2 acc = __fmul2_rn(F2::dup(o.Dy[0]), F2::ld(sU + ((ix + H::N2 * iz) * V + v) * TW + l));
#pragma unroll
          for (int m = 1; m < N; m++)
            acc = __ffma2_rn(F2::dup(o.Dy[m]), F2::ld(sU + ((ix + N * m + H::N2 * iz) * V + v) * TW + l), acc);
          const float2 cm = __fmul2_rn(F2::dup(o.dbym), F2::ld(sUC + (fym * V + v) * TW + l));
          td[1] = __fadd2_rn(acc, __ffma2_rn(F2::dup(o.dbyp), F2::ld(sUC + (fyp * V + v) * TW + l), cm));
        }
        {
          float2 acc = __fmul2_rn(F2::dup(ops.Dm[iz * N]), F2::ld(sU + ((ix + N * iy) * V + v) * TW + l));
#pragma unroll
          for (int m = 1; m < N; m++)
            acc = __ffma2_rn(F2::dup(ops.Dm[iz * N + m]), F2::ld(sU + ((ix + N * iy + H::N2 * m) * V + v) * TW + l),
                             acc);
          const float2 cm = __fmul2_rn(F2::dup(ops.Dbm[iz]), F2::ld(sUC + (fzm * V + v) * TW + l));
          td[2] = __fadd2_rn(acc, __ffma2_rn(F2::dup(ops.Dbp[iz]), F2::ld(sUC + (fzp * V + v) * TW + l), cm));
        }
#pragma unroll
        for (int d1 = 0; d1 < 3; d1++)
        {
          float2 g = __fmul2_rn(td[0], F2::dup(adj[0][d1]));
          g = __ffma2_rn(td[1], F2::dup(adj[1][d1]), g);
          g = __ffma2_rn(td[2], F2::dup(adj[2][d1]), g);
          g = __fmul2_rn(g, F2::dup(inv_det));
          F2::st(sX + xo(d1 * S + s) + v * TW + l, g);
          if (a.dU_out) F2::st(a.dU_out + (((tile * 3 + d1) * S + s) * V + v) * TW + l, g);
        }
      }
    }
#pragma unroll
    for (int v = (sizeof(A) == 4 ? V - 1 : 0); v < V; v++)
    {
      A td[3];
      {
        A acc = A(0);
#pragma unroll
        for (int m = 0; m < N; m++) acc += o.Dx[m] * sU[((m + N * iy + H::N2 * iz) * V + v) * TW + l];
        const A cm = o.dbxm * sUC[(fxm * V + v) * TW + l];
        const A cp = o.dbxp * sUC[(fxp * V + v) * TW + l];
        td[0] = acc + (cm + cp);
      }
      {
        A acc = A(0);
#pragma unroll
        for (int m = 0; m < N; m++) acc += o.Dy[m] * sU[((ix + N * m + H::N2 * iz) * V + v) * TW + l];
        const A cm = o.dbym * sUC[(fym * V + v) * TW + l];
        const A cp = o.dbyp * sUC[(fyp * V + v) * TW + l];
        td[1] = acc + (cm + cp);
      }
      {
        A acc = A(0);
#pragma unroll
        for (int m = 0; m < N; m++) acc += ops.Dm[iz * N + m] * sU[((ix + N * iy + H::N2 * m) * V + v) * TW + l];
        const A cm = ops.Dbm[iz] * sUC[(fzm * V + v) * TW + l];
        const A cp = ops.Dbp[iz] * sUC[(fzp * V + v) * TW + l];
        td[2] = acc + (cm + cp);
      }
#pragma unroll
      for (int d1 = 0; d1 < 3; d1++)
      {
        A g = td[0] * adj[0][d1];
        g += td[1] * adj[1][d1];
        g += td[2] * adj[2][d1];
        sX[xo(d1 * S + s) + v * TW + l] = g * inv_det;
        if (a.dU_out) a.dU_out[(((tile * 3 + d1) * S + s) * V + v) * TW + l] = (T)(g * inv_det);
      }
    }
  }
  __syncthreads();
  // viscous normal flux at own flux points: the points where the partner
  // supplies the LDG normal flux are skipped without a memory access; the own
  // trace is formed from the state in shared memory
#pragma unroll 1
  for (int kq = 0; kq < 6 / ZS; kq++)
  {
    int code = codes[0];
#pragma unroll
    for (int j = 1; j < 6 / ZS; j++) code = kq == j ? codes[j] : code;  // register select
    if (code >= 0 && ((beta == A(0.5) && (code & 1)) || (beta == A(-0.5) && !(code & 1)))) continue;
    const int q = own_face<ZS>(zs, kq);
    const int fq = H::fpt(q, ix, iy);
    A n[3];
    {
      const T *gq = a.fgeo + (tile * Fp + fq) * (int64_t)4 * TW + l;
      n[0] = gq[0];
      n[1] = gq[TW];
      n[2] = gq[2 * TW];
    }
    A Uf[V], dUf[V][3], Fn[V];
    hex_own_trace<A, N>(ops, sU, q, ix, iy, l, Uf);
#pragma unroll
    for (int v = 0; v < V; v++)
    {
#pragma unroll
      for (int d = 0; d < 3; d++)
      {
        A acc = (q_minus(q) ? ops.Em[0] : ops.Ep[0]) * sX[xo(d * S + H::line_spt(q, ix, iy, 0)) + v * TW + l];
#pragma unroll
        for (int m = 1; m < N; m++)
          acc += (q_minus(q) ? ops.Em[m] : ops.Ep[m]) * sX[xo(d * S + H::line_spt(q, ix, iy, m)) + v * TW + l];
        dUf[v][d] = acc;
      }
    }
    A Ua[V];
    to_abs<A, 3>(Uf, Ua, a.ph);
    if (code >= 0)
      visc_normal<A, 3>(Ua, dUf, n, Fn, a.ph);
    else
    {
      A UR[V], UB[V], dUB[V][3];
      ghost_state<A, 3>(-code - 1, Ua, n, UR, UB, a.ph);
      ghost_grad<A, 3>(-code - 1, Ua, dUf, n, dUB);
      visc_normal<A, 3>(UB, dUB, n, Fn, a.ph);
    }
    if (a.Fvn)
    {
      T *out = a.Fvn + (tile * Fp + fq) * (int64_t)V * TW + l;
#pragma unroll
      for (int v = 0; v < V; v++) out[v * TW] = Fn[v];
    }
    if (a.Fcom)
    {
      // this side supplies the LDG normal flux, so it forms the whole common
      // flux of the point once for both elements (same terms as
      // hex_common_flux with the partner's normal flux zero)
      const A tau = a.ph.ldg_tau;
      A Un[V], UL[V], UR[V], UB[V], Fc[V];
      // with beta = +-1/2 the supplying side's common solution is the
      // partner's trace, already in shared memory
      if (code >= 0)
      {
#pragma unroll
        for (int v = 0; v < V; v++) Un[v] = sUC[(fq * V + v) * TW + l];
      }
      conv_common<T, A, 3>(a, Uf, Un, code, n, UL, UR, UB, Fc);
      T *fc = a.Fcom + (tile * Fp + fq) * (int64_t)V * TW + l;
#pragma unroll
      for (int v = 0; v < V; v++)
      {
        A Fv;
        if (code >= 0)
        {
          const A FnL = beta == A(0.5) ? Fn[v] : A(0), FnR = beta == A(0.5) ? A(0) : Fn[v];
          Fv = A(0.5) * (FnL + FnR) + tau * (UL[v] - UR[v]) + beta * (FnL - FnR);
        }
        else
          Fv = Fn[v] + tau * (UL[v] - UB[v]);
        fc[v * TW] = Fc[v] + Fv;
      }
    }
  }
  __syncthreads();
  // flux at own column, transformed F~ = adj F (overwrites the gradient in place)
#pragma unroll 1
  for (int iz = iz0; iz < iz0 + NZ; iz++)
  {
    const int s = ix + N * iy + H::N2 * iz;
    A dU[V][3], F[V][3], P, Pp, Us[V], Ua[V], adj[3][3], det;
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      Us[v] = sU[(s * V + v) * TW + l];
#pragma unroll
      for (int d = 0; d < 3; d++) dU[v][d] = sX[xo(d * S + s) + v * TW + l];
    }
    flux_conv_stored<A, 3>(Us, F, P, Pp, a.ph);
    to_abs<A, 3>(Us, Ua, a.ph);
    flux_visc_add<A, 3>(Ua, dU, F, a.ph);
    load_adj<T, A>(a, tile, S, s, l, adj, det);
#pragma unroll
    for (int v = 0; v < V; v++)
#pragma unroll
      for (int d1 = 0; d1 < 3; d1++)
      {
        A t = F[v][0] * adj[d1][0];
        t += F[v][1] * adj[d1][1];
        t += F[v][2] * adj[d1][2];
        sX[xo(d1 * S + s) + v * TW + l] = t;
      }
  }
  __syncthreads();
  // volume divergence
#pragma unroll 1
  for (int iz = iz0; iz < iz0 + NZ; iz++)
  {
    const int s = ix + N * iy + H::N2 * iz;
    A *out = a.divF_vol + (tile * S + s) * (int64_t)V * TW + l;
    if constexpr (sizeof(A) == 4)
    {
      // FP32: variables 0-3 in pairs, the fifth in the loop below
#pragma unroll
      for (int v = 0; v < V - 1; v += 2)
      {
        float2 vol = __fmul2_rn(F2::dup(o.Dx[0]), F2::ld(sX + xo(N * iy + H::N2 * iz) + v * TW + l));
#pragma unroll
        for (int m = 1; m < N; m++)
          vol = __ffma2_rn(F2::dup(o.Dx[m]), F2::ld(sX + xo(m + N * iy + H::N2 * iz) + v * TW + l), vol);
#pragma unroll
        for (int m = 0; m < N; m++)
          vol = __ffma2_rn(F2::dup(o.Dy[m]), F2::ld(sX + xo(S + ix + N * m + H::N2 * iz) + v * TW + l), vol);
#pragma unroll
        for (int m = 0; m < N; m++)
          vol = __ffma2_rn(F2::dup(ops.Dm[iz * N + m]), F2::ld(sX + xo(2 * S + ix + N * iy + H::N2 * m) + v * TW + l),
                           vol);
        F2::st(out + v * TW, vol);
      }
    }
#pragma unroll
    for (int v = (sizeof(A) == 4 ? V - 1 : 0); v < V; v++)
    {
      A vol = A(0);
#pragma unroll
      for (int m = 0; m < N; m++) vol += o.Dx[m] * sX[xo(0 * S + m + N * iy + H::N2 * iz) + v * TW + l];
#pragma unroll
      for (int m = 0; m < N; m++) vol += o.Dy[m] * sX[xo(1 * S + ix + N * m + H::N2 * iz) + v * TW + l];
#pragma unroll
      for (int m = 0; m < N; m++) vol += ops.Dm[iz * N + m] * sX[xo(2 * S + ix + N * iy + H::N2 * m) + v * TW + l];
      out[v * TW] = vol;
    }
  }
}

// ---------------------------------------------------------------------------
// Navier-Stokes kernel 2 (column mapping): common flux, surface correction,
// RK update, next-stage extrapolation
// ---------------------------------------------------------------------------
template <typename T, typename A, int N>
__global__ void __launch_bounds__(TW * N * N * HexNsShape<A, N>::face_zs, HexNsShape<A, N>::face_minb)
    k_hex_ns_face(const __grid_constant__ Args<T, A> a, const __grid_constant__ LineOpsT<A, N> ops)
{
  using H = HexIdx<N>;
  constexpr int ZS = HexNsShape<A, N>::face_zs;
  constexpr int S = H::S, Fp = H::Fp, V = 5, NZ = N / ZS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  A *sFc = reinterpret_cast<A *>(smem_raw);  // [Fp][V][TW]
  A *sUnew = sFc + Fp * V * TW;              // [S][V][TW]
  const int l = threadIdx.x % TW, c = (threadIdx.x / TW) % H::N2, zs = threadIdx.x / (TW * H::N2);
  const int ix = c % N, iy = c / N;
  const int64_t tile = blockIdx.x;
  if (tile >= a.ntiles) return;
  RowOps<A, N> o;
  o.load(ops, ix, iy);
  int f[6];
  H::fpts(ix, iy, f);
  if (a.Fcom)
    hex_gather_common<T, A, N, ZS>(a, tile, l, ix, iy, sFc, zs);
  else
    hex_common_flux<T, A, N, true, ZS>(a, tile, l, ix, iy, sFc, zs);
  __syncthreads();
  // the volume residual of all of this thread's levels before any store
  // (a load cannot move above a store that may alias it)
  A dvol[NZ][V];
#pragma unroll
  for (int k = 0; k < NZ; k++)
  {
    const int s = ix + N * iy + H::N2 * (zs * NZ + k);
    const A *dv = a.divF_vol + (tile * S + s) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++) dvol[k][v] = dv[v * TW];
  }
#pragma unroll
  for (int k = 0; k < NZ; k++)
  {
    const int iz = zs * NZ + k;
    const int s = ix + N * iy + H::N2 * iz;
    A res[V];
#pragma unroll
    for (int v = 0; v < V; v++) res[v] = dvol[k][v] + hex_surface<A, N>(ops, o, sFc, ix, iy, iz, v, l);
    hex_finish<T, A, N>(a, tile, s, l, res, a.extrap_next ? sUnew : nullptr);
  }
  if (a.extrap_next)
  {
    __syncthreads();
    hex_extrap_next<T, A, N, ZS>(a, tile, l, ix, iy, f, sUnew, ops, zs);
  }
}

}  // namespace dev
}  // namespace zb

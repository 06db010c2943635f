// Batched RK stepping of many independent Euler cases on quadrilaterals:
// per RK stage either one persistent launch per polynomial order present (run
// concurrently) or one persistent launch for all of them, the four stages of
// a step captured once as a CUDA graph, and a small autotuner that picks the
// form and the launch shape.
//
// Each case is an ordinary context (its own mesh, order 1-5, state, time
// step and reference state); the batch only builds per-stage descriptors of
// their buffers.  A work item is one tile (8 elements) of one case; a CTA
// walks the item list with a grid stride and runs the tile with the kernel
// body of its order (euler_tile, the body of the single-case k_euler), so a
// stage of the batch computes exactly what the cases' own stages compute.
// Reference: FRSolver::step_RK (src/solver.cpp:2864-3097) per case.
#include <algorithm>
#include <chrono>

#include "ctx_impl.cuh"

namespace zb {

using dev::Args;
using dev::LineOpsT;
using dev::Shape;
using dev::TW;

constexpr int kBatchMaxN = 6;

template <typename T, typename A>
struct BatchCase
{
  Args<T, A> a;
  int N;
  int pad;
  A ops[kBatchMaxN * kBatchMaxN + 4 * kBatchMaxN];  // LineOpsT<A, N> laid out flat
};

// Shared memory of one tile group: its copy of the case descriptor, then the
// tile body's arrays.
template <typename T, typename A>
constexpr size_t batch_desc_bytes()
{
  return (sizeof(BatchCase<T, A>) + 15) / 16 * 16;
}

// One persistent kernel per order present, each compiled for that order
// (registers, shared memory) and walking that order's work items
// [begin, end).  A CTA holds blockDim.x / gsz independent groups of gsz
// threads (whole warps); each group walks its own share of the items with its
// own named barrier, so low-order tiles do not leave most of a large CTA idle.
template <typename T, typename A, int NN>
__global__ void __launch_bounds__(256) k_batch_euler(const BatchCase<T, A> *__restrict__ cases,
                                                     const int2 *__restrict__ items, int begin, int end, int gsz,
                                                     int gstride, int chunk)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ng = blockDim.x / gsz, g = threadIdx.x / gsz, tid = threadIdx.x % gsz;
  const int bar = (ng == 1) ? 0 : g + 1;
  unsigned char *gbase = smem_raw + (size_t)g * gstride;
  BatchCase<T, A> *sbc = reinterpret_cast<BatchCase<T, A> *>(gbase);
  unsigned char *tsm = gbase + batch_desc_bytes<T, A>();
  constexpr int nwords = (int)(sizeof(BatchCase<T, A>) / sizeof(int));
  const int gid = blockIdx.x * ng + g, ngroups = gridDim.x * ng;
  int have = -1;  // case whose descriptor the group holds
  // a group takes chunks of `chunk` consecutive items; consecutive items of
  // one case reuse the shared descriptor
  for (int c0 = begin + gid * chunk; c0 < end; c0 += ngroups * chunk)
  {
    const int c1 = min(c0 + chunk, end);
    for (int it = c0; it < c1; it++)
    {
      const int2 w = items[it];
      if (w.x != have)
      {
        dev::group_sync(bar, gsz);  // the previous tile is done with the old descriptor
        const int *src = reinterpret_cast<const int *>(&cases[w.x]);
        int *dst = reinterpret_cast<int *>(sbc);
        for (int k = tid; k < nwords; k += gsz) dst[k] = src[k];
        have = w.x;
      }
      dev::group_sync(bar, gsz);
      dev::euler_tile<T, A, 2, NN>(sbc->a, *reinterpret_cast<const LineOpsT<A, NN> *>(sbc->ops), w.y, tsm, tid, gsz,
                                   bar);
    }
  }
}

// The single-launch form: one persistent kernel per stage walks the items of
// every order (costliest order first) and runs each with its order's tile
// body; the group's shared memory fits the largest order present.  In FP32
// the registers are held to four 256-thread CTAs per SM: the kernel carries
// every order's body, and left to itself the compiler sizes it for the
// largest (128 registers, two CTAs per SM: 38 GDOF/s on the 512-case batch
// against 44 at four CTAs per SM, a few bytes of the largest order's
// values spilled).
template <typename T, typename A>
__global__ void __launch_bounds__(256, sizeof(A) == 4 ? 4 : 1) k_batch_euler_fused(const BatchCase<T, A> *__restrict__ cases,
                                                           const int2 *__restrict__ items, int begin, int end, int gsz,
                                                           int gstride, int chunk)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ng = blockDim.x / gsz, g = threadIdx.x / gsz, tid = threadIdx.x % gsz;
  const int bar = (ng == 1) ? 0 : g + 1;
  unsigned char *gbase = smem_raw + (size_t)g * gstride;
  BatchCase<T, A> *sbc = reinterpret_cast<BatchCase<T, A> *>(gbase);
  unsigned char *tsm = gbase + batch_desc_bytes<T, A>();
  constexpr int nwords = (int)(sizeof(BatchCase<T, A>) / sizeof(int));
  const int gid = blockIdx.x * ng + g, ngroups = gridDim.x * ng;
  int have = -1;
  for (int c0 = begin + gid * chunk; c0 < end; c0 += ngroups * chunk)
  {
    const int c1 = min(c0 + chunk, end);
    for (int it = c0; it < c1; it++)
    {
      const int2 w = items[it];
      if (w.x != have)
      {
        dev::group_sync(bar, gsz);
        const int *src = reinterpret_cast<const int *>(&cases[w.x]);
        int *dst = reinterpret_cast<int *>(sbc);
        for (int k = tid; k < nwords; k += gsz) dst[k] = src[k];
        have = w.x;
      }
      dev::group_sync(bar, gsz);
      switch (sbc->N)
      {
#define ZB_TILE(NN)                                                                                              \
  case NN:                                                                                                       \
    dev::euler_tile<T, A, 2, NN>(sbc->a, *reinterpret_cast<const LineOpsT<A, NN> *>(sbc->ops), w.y, tsm, tid, gsz, \
                                 bar);                                                                           \
    break;
        ZB_TILE(2) ZB_TILE(3) ZB_TILE(4) ZB_TILE(5) ZB_TILE(6)
#undef ZB_TILE
        default: break;
      }
    }
  }
}

static size_t euler_smem_bytes(int N, size_t asz)
{
  switch (N)
  {
    case 2: return dev::euler_smem_elems<2, 2>() * asz;
    case 3: return dev::euler_smem_elems<2, 3>() * asz;
    case 4: return dev::euler_smem_elems<2, 4>() * asz;
    case 5: return dev::euler_smem_elems<2, 5>() * asz;
    default: return dev::euler_smem_elems<2, 6>() * asz;
  }
}

struct Batch
{
  std::vector<Ctx *> ctx;
  int prec = ZB_FP64;
  size_t asz = 8;
  cudaStream_t stream = nullptr;
  void *cases[4] = {nullptr, nullptr, nullptr, nullptr};  // BatchCase arrays, one per stage
  int2 *items = nullptr;
  int nitems = 0;
  int obeg[kBatchMaxN + 1] = {0}, oend[kBatchMaxN + 1] = {0};  // items of order N: [obeg[N], oend[N])
  int norders = 0;  // orders present: kernels per stage
  std::vector<int> parity;  // Ufp parity of every case the descriptors assume
  size_t gstride[kBatchMaxN + 1] = {0};  // one group's shared memory per order: descriptor + tile arrays
  cudaStream_t ost[kBatchMaxN + 1] = {nullptr};  // one stream per order, forked from and joined to `stream`
  cudaEvent_t efork = nullptr, ejoin[kBatchMaxN + 1] = {nullptr};
  int sms = 148;
  zb_batch_config cfg{256, 4, 0, 0.0, 64, 1, 0};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t launches = 0;
};

template <typename T, typename A>
static void build_cases(Batch &b)
{
  const size_t n = b.ctx.size();
  std::vector<BatchCase<T, A>> h(n);
  for (unsigned st = 0; st < 4; st++)
  {
    for (size_t i = 0; i < n; i++)
    {
      Ctx &c = *b.ctx[i];
      StageCfg sc;
      sc.stage = st;
      sc.rk_mode = (st + 1 < 4) ? 1 : 2;
      sc.save_ini = (st == 0);
      sc.extrap_next = 1;
      const int cur0 = c.cur;
      c.cur = b.parity[i] ^ (int)(st & 1);
      std::memset(&h[i], 0, sizeof(h[i]));
      h[i].a = make_args<T, A>(c, sc);
      c.cur = cur0;
      h[i].N = c.N;
      const Plan &p = c.plan;
      const int N = c.N;
      A *o = h[i].ops;
      for (int k = 0; k < N * N; k++) o[k] = (A)p.ops.D[k];
      for (int k = 0; k < N; k++)
      {
        o[N * N + k] = (A)p.ops.Em[k];
        o[N * N + N + k] = (A)p.ops.Ep[k];
        o[N * N + 2 * N + k] = (A)p.ops.Dbm[k];
        o[N * N + 3 * N + k] = (A)p.ops.Dbp[k];
      }
    }
    if (!b.cases[st])
    {
      cudaError_t e = cudaMalloc(&b.cases[st], n * sizeof(BatchCase<T, A>));
      if (e != cudaSuccess) ZB_THROW(ZB_ERR_NOMEM, "batch descriptors");
    }
    CK(cudaMemcpy(b.cases[st], h.data(), n * sizeof(BatchCase<T, A>), cudaMemcpyHostToDevice));
  }
}

// Items grouped by order (one kernel each); within an order, work order 0
// interleaves the cases tile by tile, order 1 is case-major.
static void build_items(Batch &b, int order)
{
  std::vector<int2> it;
  const int n = (int)b.ctx.size();
  for (int N = kBatchMaxN; N >= 2; N--)
  {
    b.obeg[N] = (int)it.size();
    if (order == 1)
    {
      for (int i = 0; i < n; i++)
        if (b.ctx[i]->N == N)
          for (int64_t t = 0; t < b.ctx[i]->ntiles; t++) it.push_back(make_int2(i, (int)t));
    }
    else
    {
      int64_t maxt = 0;
      for (int i = 0; i < n; i++)
        if (b.ctx[i]->N == N) maxt = std::max(maxt, b.ctx[i]->ntiles);
      for (int64_t t = 0; t < maxt; t++)
        for (int i = 0; i < n; i++)
          if (b.ctx[i]->N == N && t < b.ctx[i]->ntiles) it.push_back(make_int2(i, (int)t));
    }
    b.oend[N] = (int)it.size();
  }
  b.norders = 0;
  for (int N = 2; N <= kBatchMaxN; N++) b.norders += b.oend[N] > b.obeg[N];
  if (it.size() > (size_t)INT32_MAX) ZB_THROW(ZB_ERR_UNSUPPORTED, "batch too large");
  if (b.items) cudaFree(b.items);
  b.items = nullptr;
  CK(cudaMalloc(&b.items, it.size() * sizeof(int2)));
  CK(cudaMemcpy(b.items, it.data(), it.size() * sizeof(int2), cudaMemcpyHostToDevice));
  b.nitems = (int)it.size();
}

template <typename T, typename A, int NN>
static void launch_order(Batch &b, unsigned st)
{
  const int n = b.oend[NN] - b.obeg[NN];
  if (n == 0) return;
  const int ng = b.cfg.threads / b.cfg.group;
  int chunk = b.cfg.chunk;
  int blocks;
  if (chunk == 0)
  {
    // contiguous: every group takes one run of consecutive items (the items
    // of one order cost the same, so equal runs balance), which keeps a
    // group's descriptor for a whole case
    blocks = std::max(1, std::min((n + ng - 1) / ng, b.cfg.blocks_per_sm * b.sms));
    chunk = (n + blocks * ng - 1) / (blocks * ng);
  }
  else
    blocks = std::max(1, std::min((n + ng * chunk - 1) / (ng * chunk), b.cfg.blocks_per_sm * b.sms));
  CK(cudaStreamWaitEvent(b.ost[NN], b.efork, 0));
  k_batch_euler<T, A, NN><<<blocks, b.cfg.threads, ng * b.gstride[NN], b.ost[NN]>>>(
      (const BatchCase<T, A> *)b.cases[st], b.items, b.obeg[NN], b.oend[NN], b.cfg.group, (int)b.gstride[NN],
      chunk);
  b.launches++;
  CK(cudaGetLastError());
  CK(cudaEventRecord(b.ejoin[NN], b.ost[NN]));
  CK(cudaStreamWaitEvent(b.stream, b.ejoin[NN], 0));
}

// the whole stage in one persistent launch (cfg.fused)
template <typename T, typename A>
static void launch_fused(Batch &b, unsigned st)
{
  size_t gstride = 0;
  for (int N = 2; N <= kBatchMaxN; N++)
    if (b.oend[N] > b.obeg[N]) gstride = std::max(gstride, b.gstride[N]);
  const int n = b.nitems;
  const int ng = b.cfg.threads / b.cfg.group;
  int chunk = b.cfg.chunk, blocks;
  if (chunk == 0)
  {
    blocks = std::max(1, std::min((n + ng - 1) / ng, b.cfg.blocks_per_sm * b.sms));
    chunk = (n + blocks * ng - 1) / (blocks * ng);
  }
  else
    blocks = std::max(1, std::min((n + ng * chunk - 1) / (ng * chunk), b.cfg.blocks_per_sm * b.sms));
  k_batch_euler_fused<T, A><<<blocks, b.cfg.threads, ng * gstride, b.stream>>>(
      (const BatchCase<T, A> *)b.cases[st], b.items, 0, n, b.cfg.group, (int)gstride, chunk);
  b.launches++;
  CK(cudaGetLastError());
}

// one stage: the per-order kernels run concurrently on their own streams,
// forked from and joined back to the batch stream (also under graph capture)
template <typename T, typename A>
static void launch_stage_t(Batch &b, unsigned st)
{
  if (b.cfg.fused) return launch_fused<T, A>(b, st);
  CK(cudaEventRecord(b.efork, b.stream));
  launch_order<T, A, 6>(b, st);
  launch_order<T, A, 5>(b, st);
  launch_order<T, A, 4>(b, st);
  launch_order<T, A, 3>(b, st);
  launch_order<T, A, 2>(b, st);
}

static void launch_stage(Batch &b, unsigned st)
{
  if (b.prec == ZB_FP64)
    launch_stage_t<double, double>(b, st);
  else
    launch_stage_t<float, float>(b, st);
}

static void drop_graph(Batch &b)
{
  if (b.exec) cudaGraphExecDestroy(b.exec);
  if (b.graph) cudaGraphDestroy(b.graph);
  b.exec = nullptr;
  b.graph = nullptr;
}

static void build_graph(Batch &b)
{
  drop_graph(b);
  CK(cudaStreamBeginCapture(b.stream, cudaStreamCaptureModeThreadLocal));
  const int64_t l0 = b.launches;
  for (unsigned st = 0; st < 4; st++) launch_stage(b, st);
  b.launches = l0;  // counted when the graph is replayed
  cudaError_t e = cudaStreamEndCapture(b.stream, &b.graph);
  if (e != cudaSuccess) ZB_THROW(ZB_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  CK(cudaGraphInstantiate(&b.exec, b.graph, 0));
}

// Make every case ready for batched stages from stage `first`: its own
// queued work done, its traces current, and the descriptors built for the
// trace parity its stage 0 had (parity flips once per stage).
static void prepare(Batch &b, unsigned first)
{
  bool stale = b.parity.empty();
  for (size_t i = 0; i < b.ctx.size(); i++)
  {
    Ctx &c = *b.ctx[i];
    if (!c.ufp_valid)
    {
      c.launch_extrap(c);
      c.ufp_valid = true;
    }
    CK(cudaStreamSynchronize(c.stream));
    if (!stale && b.parity[i] != (c.cur ^ (int)(first & 1))) stale = true;
  }
  if (!stale) return;
  b.parity.resize(b.ctx.size());
  for (size_t i = 0; i < b.ctx.size(); i++) b.parity[i] = b.ctx[i]->cur ^ (int)(first & 1);
  if (b.prec == ZB_FP64)
    build_cases<double, double>(b);
  else
    build_cases<float, float>(b);
  drop_graph(b);
}

template <typename T, typename A>
static void set_batch_smem(Batch &b)
{
  size_t gmax = 0;
  for (int N = 2; N <= kBatchMaxN; N++) gmax = std::max(gmax, b.gstride[N]);
  CK(cudaFuncSetAttribute(k_batch_euler_fused<T, A>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(4 * gmax)));
  CK(cudaFuncSetAttribute(k_batch_euler<T, A, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(4 * b.gstride[2])));
  CK(cudaFuncSetAttribute(k_batch_euler<T, A, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(4 * b.gstride[3])));
  CK(cudaFuncSetAttribute(k_batch_euler<T, A, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(4 * b.gstride[4])));
  CK(cudaFuncSetAttribute(k_batch_euler<T, A, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(4 * b.gstride[5])));
  CK(cudaFuncSetAttribute(k_batch_euler<T, A, 6>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(4 * b.gstride[6])));
}

Batch *batch_create(Ctx *const *ctxs, int n)
{
  if (n <= 0 || !ctxs) ZB_THROW(ZB_ERR_ARG, "empty batch");
  std::unique_ptr<Batch> b(new Batch());
  int dev0 = -1;
  for (int i = 0; i < n; i++)
  {
    Ctx *c = ctxs[i];
    if (!c) ZB_THROW(ZB_ERR_ARG, "null context in batch");
    if (c->plan.etype != ET_QUAD || c->plan.params.viscous)
      ZB_THROW(ZB_ERR_UNSUPPORTED, "the batched stage is built for Euler on quadrilaterals");
    if (c->N < 2 || c->N > kBatchMaxN) ZB_THROW(ZB_ERR_UNSUPPORTED, "batched orders are P1-P5");
    if (i == 0)
    {
      b->prec = c->prec;
      dev0 = c->dev;
    }
    else if (c->prec != b->prec || c->dev != dev0)
      ZB_THROW(ZB_ERR_ARG, "batched contexts must share precision and device");
    b->ctx.push_back(c);
  }
  b->asz = (b->prec == ZB_FP64) ? sizeof(double) : sizeof(float);
  const size_t desc = b->prec == ZB_FP64 ? batch_desc_bytes<double, double>() : batch_desc_bytes<float, float>();
  for (int N = 2; N <= kBatchMaxN; N++) b->gstride[N] = desc + (euler_smem_bytes(N, b->asz) + 15) / 16 * 16;
  CK(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev0));
  CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&b->efork, cudaEventDisableTiming));
  for (int N = 2; N <= kBatchMaxN; N++)
  {
    CK(cudaStreamCreateWithFlags(&b->ost[N], cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&b->ejoin[N], cudaEventDisableTiming));
  }
  // up to four groups per CTA
  if (b->prec == ZB_FP64)
    set_batch_smem<double, double>(*b);
  else
    set_batch_smem<float, float>(*b);
  build_items(*b, b->cfg.order);
  return b.release();
}

void batch_destroy(Batch *b)
{
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graph(*b);
  for (void *p : b->cases)
    if (p) cudaFree(p);
  if (b->items) cudaFree(b->items);
  for (int N = 2; N <= kBatchMaxN; N++)
  {
    if (b->ost[N]) cudaStreamDestroy(b->ost[N]);
    if (b->ejoin[N]) cudaEventDestroy(b->ejoin[N]);
  }
  if (b->efork) cudaEventDestroy(b->efork);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

void batch_stage(Batch *b, unsigned stage)
{
  if (stage > 3) ZB_THROW(ZB_ERR_ARG, "stage out of range");
  prepare(*b, stage);
  // a lone stage flips every case's trace parity
  launch_stage(*b, stage);
  CK(cudaStreamSynchronize(b->stream));
  for (Ctx *c : b->ctx) c->cur ^= 1;
}

void batch_step(Batch *b, int nsteps, int use_graph)
{
  if (nsteps < 0) ZB_THROW(ZB_ERR_ARG, "negative step count");
  prepare(*b, 0);
  if (use_graph && !b->exec) build_graph(*b);
  for (int i = 0; i < nsteps; i++)
  {
    if (use_graph)
    {
      CK(cudaGraphLaunch(b->exec, b->stream));
      b->launches += 4 * (b->cfg.fused ? 1 : b->norders);
    }
    else
      for (unsigned st = 0; st < 4; st++) launch_stage(*b, st);
  }
}

void batch_sync(Batch *b) { CK(cudaStreamSynchronize(b->stream)); }

int64_t batch_launches(const Batch *b) { return b->launches; }

// Time each candidate launch shape on a few graph-replayed steps from the
// current state, restore the state, keep the fastest.
void batch_autotune(Batch *b, int steps, int form, zb_batch_config *out)
{
  if (steps < 1) steps = 1;
  prepare(*b, 0);
  // save the states (and compensated remainders) the trials overwrite
  std::vector<void *> saveU(b->ctx.size(), nullptr), saveC(b->ctx.size(), nullptr);
  for (size_t i = 0; i < b->ctx.size(); i++)
  {
    Ctx &c = *b->ctx[i];
    const size_t bytes = (size_t)c.ntiles * c.S * c.V * TW * c.tsz;
    CK(cudaMalloc(&saveU[i], bytes));
    CK(cudaMemcpyAsync(saveU[i], c.U, bytes, cudaMemcpyDeviceToDevice, b->stream));
    if (c.Ucomp)
    {
      CK(cudaMalloc(&saveC[i], bytes));
      CK(cudaMemcpyAsync(saveC[i], c.Ucomp, bytes, cudaMemcpyDeviceToDevice, b->stream));
    }
  }
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const int shapes[][2] = {{64, 64}, {128, 64}, {128, 128}, {256, 64}, {256, 128}, {256, 256}};
  const int bps[] = {2, 4, 8, 16};
  const int orders[] = {0, 1};
  const int chunks[] = {0, 1, 8, 32};  // 0: one contiguous run per group
  zb_batch_config best{0, 0, 0, 1e300, 0, 1, 0};
  for (int fused : {0, 1})
  for (int order : orders)
  {
    if (form >= 0 && fused != form) continue;
    build_items(*b, order);
    for (const auto &sh : shapes)
      for (int bp : bps)
        for (int ch : chunks)
      {
        b->cfg.threads = sh[0];
        b->cfg.group = sh[1];
        b->cfg.blocks_per_sm = bp;
        b->cfg.order = order;
        b->cfg.chunk = ch;
        b->cfg.fused = fused;
        build_graph(*b);
        CK(cudaGraphLaunch(b->exec, b->stream));  // warm-up
        CK(cudaEventRecord(e0, b->stream));
        for (int s = 0; s < steps; s++) CK(cudaGraphLaunch(b->exec, b->stream));
        CK(cudaEventRecord(e1, b->stream));
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        const double per = ms / steps;
        if (per < best.ms_per_step) best = zb_batch_config{sh[0], bp, order, per, sh[1], ch, fused};
      }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  for (size_t i = 0; i < b->ctx.size(); i++)
  {
    Ctx &c = *b->ctx[i];
    const size_t bytes = (size_t)c.ntiles * c.S * c.V * TW * c.tsz;
    CK(cudaMemcpyAsync(c.U, saveU[i], bytes, cudaMemcpyDeviceToDevice, b->stream));
    if (saveC[i]) CK(cudaMemcpyAsync(c.Ucomp, saveC[i], bytes, cudaMemcpyDeviceToDevice, b->stream));
  }
  CK(cudaStreamSynchronize(b->stream));
  for (size_t i = 0; i < b->ctx.size(); i++)
  {
    cudaFree(saveU[i]);
    if (saveC[i]) cudaFree(saveC[i]);
    b->ctx[i]->ufp_valid = false;  // traces of the restored state are recomputed
  }
  b->cfg = best;
  build_items(*b, best.order);
  drop_graph(*b);
  b->parity.clear();
  if (out) *out = best;
}

void batch_config(Batch *b, const zb_batch_config *cfg)
{
  if (cfg->threads != 64 && cfg->threads != 128 && cfg->threads != 256)
    ZB_THROW(ZB_ERR_ARG, "threads must be 64, 128 or 256");
  if (cfg->group < 64 || cfg->group > cfg->threads || cfg->threads % cfg->group != 0 || cfg->group % 32 != 0)
    ZB_THROW(ZB_ERR_ARG, "group must be a multiple of 32, at least 64, dividing threads");
  if (cfg->blocks_per_sm < 1 || cfg->blocks_per_sm > 64) ZB_THROW(ZB_ERR_ARG, "blocks_per_sm out of range");
  if (cfg->order != 0 && cfg->order != 1) ZB_THROW(ZB_ERR_ARG, "order must be 0 or 1");
  if (cfg->chunk < 0) ZB_THROW(ZB_ERR_ARG, "chunk must be 0 (contiguous runs) or positive");
  if (cfg->fused != 0 && cfg->fused != 1) ZB_THROW(ZB_ERR_ARG, "fused must be 0 or 1");
  CK(cudaStreamSynchronize(b->stream));
  b->cfg = *cfg;
  build_items(*b, cfg->order);
  drop_graph(*b);
}

}  // namespace zb

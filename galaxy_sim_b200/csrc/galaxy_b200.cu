// Host runtime and C ABI of the B200 gravity path (declarations and reference
// citations in include/galaxy_b200.h). One gs_ctx owns its device memory and
// one CUDA stream; every operation is stream-ordered like the WebGPU command
// encoder it replaces, and full steps are replayed from captured CUDA graphs.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <thread>
#include <vector>

#include "build.cuh"
#include "common.cuh"
#include "morton.cuh"
#include "particles.cuh"
#include "sort.cuh"
#include "walk.cuh"

using namespace gs;

namespace {

thread_local char g_err[512] = "";

constexpr uint32_t kMaxN = 1u << 27;  // node indices (2N + 4096) fit the walk's 29-bit fields
constexpr int kSortPasses = 4;

inline uint32_t cdiv(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }

// Device workspace of one sort + build over up to N particles.
struct Workspace {
  uint32_t N = 0, cap = 0, tiles = 0, fblocks = 0;
  uint32_t* keys[2] = {nullptr, nullptr};
  uint32_t* vals[2] = {nullptr, nullptr};
  uint32_t* sort_scratch = nullptr;  // hist[4*256] | tile counters[16] | lookback
  size_t sort_scratch_bytes = 0;
  int* bbox_partials = nullptr;
  unsigned* bbox_counter = nullptr;
  MortonFrame* frame = nullptr;
  uint8_t* dl = nullptr;
  uint32_t* blk_counts = nullptr;
  uint32_t* blk_offs = nullptr;
  TreeMeta* meta = nullptr;
  uint32_t* node_start = nullptr;
  uint32_t* child_base = nullptr;
  int32_t* parent = nullptr;
  uint8_t* depth = nullptr;
  uint32_t* arrive = nullptr;
  uint32_t* leaf_node = nullptr;
  uint32_t* leaf_start = nullptr;
  float4* cm = nullptr;
  WalkInfo* info = nullptr;
  std::vector<void*> owned;

  uint32_t* hist() const { return sort_scratch; }
  uint32_t* tile_ctr() const { return sort_scratch + 4 * 256; }
  uint32_t* lookback() const { return sort_scratch + 4 * 256 + 16; }

  BuildBuffers bb(uint32_t max_nodes) const {
    BuildBuffers b;
    b.codes = keys[0];
    b.N = N;
    b.cap = cap;
    b.max_nodes = max_nodes;
    b.dl = dl;
    b.blk_counts = blk_counts;
    b.blk_offs = blk_offs;
    b.meta = meta;
    b.node_start = node_start;
    b.child_base = child_base;
    b.parent = parent;
    b.depth = depth;
    b.arrive = arrive;
    b.leaf_node = leaf_node;
    b.leaf_start = leaf_start;
    b.cm = cm;
    b.info = info;
    return b;
  }

  template <typename T>
  cudaError_t alloc(T** p, size_t count) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, count * sizeof(T) + 16);
    if (e != cudaSuccess) return e;
    owned.push_back(q);
    *p = reinterpret_cast<T*>(q);
    return cudaSuccess;
  }
  cudaError_t init(uint32_t n) {
    N = n;
    cap = 2 * n + 4096;
    tiles = cdiv(n, kSortTile);
    fblocks = cdiv(n, kFlagTile);
    cudaError_t e;
#define A(ptr, cnt)                  \
  if ((e = alloc(&(ptr), (cnt))) != cudaSuccess) return e;
    A(keys[0], n);
    A(keys[1], n);
    A(vals[0], n);
    A(vals[1], n);
    sort_scratch_bytes = sizeof(uint32_t) * (4 * 256 + 16 + (size_t)kSortPasses * tiles * 256);
    A(sort_scratch, sort_scratch_bytes / sizeof(uint32_t));
    A(bbox_partials, kBBoxBlocks * 6);
    A(bbox_counter, 4);
    A(frame, 1);
    A(dl, n + 4);
    A(blk_counts, (size_t)fblocks * kCounters);
    A(blk_offs, (size_t)fblocks * kCounters);
    A(meta, 1);
    A(node_start, cap);
    A(child_base, cap + 1);
    A(parent, cap);
    A(depth, cap);
    A(arrive, cap);
    A(leaf_node, n + 1);
    A(leaf_start, n + 1);
    A(cm, cap);
    A(info, cap);
#undef A
    if ((e = cudaMemset(bbox_counter, 0, 16)) != cudaSuccess) return e;
    if ((e = cudaMemset(arrive, 0, sizeof(uint32_t) * cap)) != cudaSuccess) return e;
    if ((e = cudaMemset(cm, 0, sizeof(float4) * cap)) != cudaSuccess) return e;
    if ((e = cudaMemset(info, 0, sizeof(WalkInfo) * cap)) != cudaSuccess) return e;
    return cudaSuccess;
  }
  void release() {
    for (void* p : owned) cudaFree(p);
    owned.clear();
  }
};

// codes of `pos` (float4 records, stride in float4) into keys[0], sort -> keys[0]
// (sorted codes) and vals[0] (gather permutation).
cudaError_t enqueue_codes_sort(Workspace& w, const float4* pos, uint32_t stride, cudaStream_t s,
                               DevState* st, int advance_time) {
  const uint32_t N = w.N;
  const uint32_t bb = std::min<uint32_t>(kBBoxBlocks, std::max<uint32_t>(1, cdiv(N, kBBoxThreads)));
  bbox_kernel<<<bb, kBBoxThreads, 0, s>>>(pos, stride, N, w.bbox_partials, w.bbox_counter, w.frame,
                                          st, advance_time);
  cudaMemsetAsync(w.sort_scratch, 0, w.sort_scratch_bytes, s);
  const uint32_t cb = std::min<uint32_t>(148 * 8, std::max<uint32_t>(1, cdiv(N, 256)));
  codes_kernel<<<cb, 256, 0, s>>>(pos, stride, N, w.frame, w.keys[0], w.hist(), kSortPasses);
  for (int p = 0; p < kSortPasses; p++) {
    const int src = p & 1, dst = src ^ 1;
    uint32_t* lb = w.lookback() + (size_t)p * w.tiles * 256;
    if (p == 0)
      onesweep_pass<true><<<w.tiles, kSortThreads, 0, s>>>(w.keys[src], nullptr, w.keys[dst],
                                                           w.vals[dst], w.hist() + p * 256, lb,
                                                           w.tile_ctr() + p, N, 8 * p, st);
    else
      onesweep_pass<false><<<w.tiles, kSortThreads, 0, s>>>(w.keys[src], w.vals[src], w.keys[dst],
                                                            w.vals[dst], w.hist() + p * 256, lb,
                                                            w.tile_ctr() + p, N, 8 * p, st);
  }
  return cudaGetLastError();
}

// hist of given keys (stateless radix sort)
__global__ void key_hist_kernel(const uint32_t* __restrict__ keys, uint32_t N, uint32_t* hist,
                                int passes) {
  __shared__ uint32_t s_hist[4 * 256];
  for (int k = threadIdx.x; k < 4 * 256; k += blockDim.x) s_hist[k] = 0;
  __syncthreads();
  for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < N; i0 += gridDim.x * blockDim.x) {
    const uint32_t i = i0 + threadIdx.x;
    const bool valid = i < N;
    hist_add_warp(s_hist, valid ? keys[i] : 0u, valid, passes);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < passes * 256; k += blockDim.x)
    if (s_hist[k]) atomicAdd(&hist[k], s_hist[k]);
}

__global__ void mask30_kernel(uint32_t* keys, uint32_t N) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
    keys[i] &= 0x3fffffffu;
}

// the tree over keys[0] (sorted codes) with COM from pos
// root size: the Morton frame of the preceding sort (frame != NULL) or root_size_host.
cudaError_t enqueue_build(Workspace& w, const float4* pos, uint32_t stride, uint32_t max_nodes,
                          int com_mode, double root_size_host, const MortonFrame* frame,
                          cudaStream_t s, DevState* st, DevState* st_flags) {
  BuildBuffers b = w.bb(max_nodes);
  tree_flags_kernel<<<w.fblocks, kFlagThreads, 0, s>>>(b, st_flags);
  tree_scan_kernel<<<1, kScanThreads, 0, s>>>(b, w.fblocks, root_size_host, frame, st);
  tree_emit_kernel<<<w.fblocks, kFlagThreads, 0, s>>>(b, st);
  const uint32_t lb = std::min<uint32_t>(148 * 16, std::max<uint32_t>(1, cdiv(w.N, 256)));
  if (com_mode == kComJs)
    tree_leaves_kernel<kComJs><<<lb, 256, 0, s>>>(b, pos, stride, st);
  else if (com_mode == kComF64)
    tree_leaves_kernel<kComF64><<<lb, 256, 0, s>>>(b, pos, stride, st);
  else
    tree_leaves_kernel<kComF32><<<lb, 256, 0, s>>>(b, pos, stride, st);
  return cudaGetLastError();
}

void set_err(char* dst, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(dst, 512, fmt, ap);
  va_end(ap);
}

}  // namespace

struct gs_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  uint32_t N = 0;
  Workspace ws;
  float4* part[2] = {nullptr, nullptr};
  float4* stel[2] = {nullptr, nullptr};
  int cur = 0, scur = 0;
  float* energy = nullptr;
  float4* compact = nullptr;
  uint32_t* perm_user = nullptr;
  DevState* st = nullptr;
  gs_params hp{};
  double* partials = nullptr;
  double* diag_out = nullptr;
  uint32_t walk_groups = 0;  // 32-particle groups (diagnostic partials)
  uint32_t walk_grid = 0;    // persistent walk blocks
  unsigned* walk_work = nullptr;
  float4* dbg_acc = nullptr;
  float* dbg_dens = nullptr;
  bool debug = false;
  gs_node* bh = nullptr;  // BHNode staging (upload / materialise)
  uint32_t max_bh = 0;
  enum { kTreeNone, kTreeUploaded, kTreeBuilt } tree = kTreeNone;
  uint32_t up_nodes = 0;
  std::vector<uint32_t> up_lr;
  bool tracking = false;
  int com_mode = kComF32;
  void* host_stage = nullptr;  // pinned, N * 16 bytes
  cudaEvent_t ev = nullptr;
  std::map<int, cudaGraphExec_t> graphs;
  char err[512] = "";

  int fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, sizeof(err), fmt, ap);
    va_end(ap);
    return code;
  }
  int cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return GS_OK;
    return fail(e == cudaErrorMemoryAllocation ? GS_ENOMEM : GS_ECUDA, "%s: %s", what,
                cudaGetErrorString(e));
  }
  void drop_graphs() {
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
    graphs.clear();
  }
};

#define CK(ctx, expr, what)                                    \
  do {                                                         \
    int _rc = (ctx)->cuda((expr), (what));                     \
    if (_rc != GS_OK) return _rc;                              \
  } while (0)

#define CTX_CHECK(ctx)                                         \
  do {                                                         \
    if (!(ctx)) {                                              \
      set_err(g_err, "null context");                          \
      return GS_EINVAL;                                        \
    }                                                          \
    cudaSetDevice((ctx)->device);                              \
  } while (0)

namespace {

uint32_t grid_for(uint32_t N, uint32_t threads, uint32_t cap_blocks) {
  return std::min<uint32_t>(cap_blocks, std::max<uint32_t>(1, cdiv(N, threads)));
}

int wait_stream(gs_ctx* c, uint64_t timeout_ns) {
  CK(c, cudaEventRecord(c->ev, c->stream), "cudaEventRecord");
  if (timeout_ns == 0) {
    CK(c, cudaEventSynchronize(c->ev), "cudaEventSynchronize");
  } else {
    const auto t0 = std::chrono::steady_clock::now();
    while (true) {
      cudaError_t q = cudaEventQuery(c->ev);
      if (q == cudaSuccess) break;
      if (q != cudaErrorNotReady) return c->cuda(q, "cudaEventQuery");
      const auto dt = std::chrono::duration_cast<std::chrono::nanoseconds>(
                          std::chrono::steady_clock::now() - t0)
                          .count();
      if ((uint64_t)dt > timeout_ns)
        return c->fail(GS_ETIMEDOUT, "stream did not drain within %llu ns",
                       (unsigned long long)timeout_ns);
      std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
  }
  unsigned err = 0;
  CK(c, cudaMemcpy(&err, &c->st->err, sizeof(unsigned), cudaMemcpyDeviceToHost), "read error word");
  if (err)
    return c->fail(GS_EDEVICE, "device error word 0x%x (%s%s%s%s)", err,
                   err & GS_DERR_LOOKBACK ? "sort look-back wait limit " : "",
                   err & GS_DERR_STACK ? "walk stack " : "", err & GS_DERR_NODES ? "node pool " : "",
                   err & GS_DERR_TREE ? "uploaded tree not BFS-contiguous" : "");
  return GS_OK;
}

void enqueue_walk(gs_ctx* c, int sf) {
  WalkArgs a;
  a.pin = c->part[c->cur];
  a.pout = c->part[c->cur ^ 1];
  a.stellar = c->stel[c->scur];
  a.cm = c->ws.cm;
  a.info = c->ws.info;
  a.st = c->st;
  a.energy = c->energy;
  a.dbg_acc = c->dbg_acc;
  a.dbg_dens = c->dbg_dens;
  a.partials = c->partials;
  a.N = c->N;
  a.node_cap = c->ws.cap;
  a.work = c->walk_work;
  const uint32_t g = c->walk_grid;
  if (c->debug) {
    if (sf) walk_kernel<true, true><<<g, kWalkThreads, 0, c->stream>>>(a);
    else walk_kernel<false, true><<<g, kWalkThreads, 0, c->stream>>>(a);
  } else {
    if (sf) walk_kernel<true, false><<<g, kWalkThreads, 0, c->stream>>>(a);
    else walk_kernel<false, false><<<g, kWalkThreads, 0, c->stream>>>(a);
  }
  c->cur ^= 1;
}

// codes + sort + gather (+tracking/EMA) + build + refresh; flips cur and scur.
void enqueue_sort_build(gs_ctx* c, int advance_time) {
  Workspace& w = c->ws;
  enqueue_codes_sort(w, c->part[c->cur], 2, c->stream, c->st, advance_time);
  gather_kernel<<<grid_for(c->N, 256, 148 * 16), 256, 0, c->stream>>>(
      w.vals[0], c->part[c->cur], c->part[c->cur ^ 1], c->stel[c->scur], c->stel[c->scur ^ 1],
      c->N, c->st, c->tracking ? 1 : 0);
  c->cur ^= 1;
  c->scur ^= 1;
  enqueue_build(w, c->part[c->cur], 2, w.cap, c->com_mode, 0.0, w.frame, c->stream, c->st, c->st);
  c->tree = gs_ctx::kTreeBuilt;
}

// After a Params upload: sim_time follows Params.time, and tracked halo centres
// keep their device-side smoothed values.
__global__ void params_fixup_kernel(DevState* st, uint32_t N) {
  st->p.N = N;
  st->sim_time = (double)st->p.time;
  for (int h = 0; h < 2; h++) {
    if (st->central[h] < 0) continue;
    float* dst = h == 0 ? st->p.haloC1 : st->p.haloC2;
    for (int k = 0; k < 3; k++) dst[k] = __double2float_rn(st->halo_c[h][k]);
  }
}

__global__ void tracking_init_kernel(DevState* st, const float4* P, long long c0, long long c1,
                                     int have0, double h0x, double h0y, double h0z, int have1,
                                     double h1x, double h1y, double h1z, uint32_t N) {
  const long long c[2] = {c0, c1};
  const int have[2] = {have0, have1};
  const double hv[2][3] = {{h0x, h0y, h0z}, {h1x, h1y, h1z}};
  for (int h = 0; h < 2; h++) {
    st->central[h] = c[h];
    st->central_next[h] = c[h];
    if (have[h]) {
      for (int k = 0; k < 3; k++) st->halo_c[h][k] = hv[h][k];
    } else if (c[h] >= 0 && c[h] < (long long)N) {
      const float4 p = P[2 * (size_t)c[h]];
      st->halo_c[h][0] = p.x;
      st->halo_c[h][1] = p.y;
      st->halo_c[h][2] = p.z;
    }
    if (c[h] >= 0) {
      float* dst = h == 0 ? st->p.haloC1 : st->p.haloC2;
      for (int k = 0; k < 3; k++) dst[k] = __double2float_rn(st->halo_c[h][k]);
    }
  }
}

__global__ void bh_patch_kernel(gs_node* bh, const float4* cm, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 c = cm[i];
    bh[i].com[0] = c.x;
    bh[i].com[1] = c.y;
    bh[i].com[2] = c.z;
    bh[i].mass = c.w;
  }
}

int host_pack4(const float* src, uint32_t N, uint32_t stride, std::vector<float4>& out) {
  out.resize(N);
  for (uint32_t i = 0; i < N; i++)
    out[i] = make_float4(src[(size_t)i * stride], src[(size_t)i * stride + 1],
                         src[(size_t)i * stride + 2], stride >= 4 ? src[(size_t)i * stride + 3] : 0.f);
  return GS_OK;
}

}  // namespace

extern "C" {

const char* gs_last_error(const gs_ctx* ctx) { return ctx ? ctx->err : g_err; }

}  // extern "C"

// Context-free error text for entry points defined in other translation units.
void gs_internal_set_error(const char* msg) { set_err(g_err, "%s", msg); }

extern "C" {
const char* gs_version(void) { return "galaxy_b200 0.1 (sm_100a)"; }

int gs_device_count(int* count) {
  if (!count) return GS_EINVAL;
  cudaError_t e = cudaGetDeviceCount(count);
  if (e != cudaSuccess) {
    *count = 0;
    set_err(g_err, "cudaGetDeviceCount: %s", cudaGetErrorString(e));
    return GS_ECUDA;
  }
  return GS_OK;
}

int gs_create_on(int device, uint32_t N, const float* particles8, const float* stellar4,
                 gs_ctx** out) {
  if (!out) {
    set_err(g_err, "out is NULL");
    return GS_EINVAL;
  }
  *out = nullptr;
  if (N == 0 || N > kMaxN) {
    set_err(g_err, "N must be in [1, %u], got %u", kMaxN, N);
    return GS_EINVAL;
  }
  if (!particles8) {
    set_err(g_err, "particles8 is NULL");
    return GS_EINVAL;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    set_err(g_err, "no CUDA device %d (have %d)", device, ndev);
    return GS_EINVAL;
  }
  gs_ctx* c = new (std::nothrow) gs_ctx();
  if (!c) return GS_ENOMEM;
  c->device = device;
  c->N = N;
  cudaSetDevice(device);
  auto bail = [&](int rc) {
    set_err(g_err, "%s", c->err);
    gs_destroy(c);
    return rc;
  };
  int rc;
  if ((rc = c->cuda(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream")))
    return bail(rc);
  if ((rc = c->cuda(cudaEventCreateWithFlags(&c->ev, cudaEventDisableTiming), "event")))
    return bail(rc);
  if ((rc = c->cuda(c->ws.init(N), "workspace"))) return bail(rc);
  Workspace& w = c->ws;
  if ((rc = c->cuda(w.alloc(&c->part[0], 2 * (size_t)N), "particles"))) return bail(rc);
  if ((rc = c->cuda(w.alloc(&c->part[1], 2 * (size_t)N), "particles"))) return bail(rc);
  if ((rc = c->cuda(w.alloc(&c->stel[0], N), "stellar"))) return bail(rc);
  if ((rc = c->cuda(w.alloc(&c->stel[1], N), "stellar"))) return bail(rc);
  if ((rc = c->cuda(w.alloc(&c->energy, N), "energy"))) return bail(rc);
  if ((rc = c->cuda(w.alloc(&c->compact, N), "compact"))) return bail(rc);
  if ((rc = c->cuda(w.alloc(&c->perm_user, N), "perm"))) return bail(rc);
  if ((rc = c->cuda(w.alloc(&c->st, 1), "state"))) return bail(rc);
  c->walk_groups = cdiv(N, kWalkGroup);
  {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    c->walk_grid = std::min<uint32_t>(cdiv(c->walk_groups, kWalkWarps),
                                      (uint32_t)sms * kWalkBlocksPerSM);
  }
  if ((rc = c->cuda(w.alloc(&c->partials, (size_t)c->walk_groups * kPartials), "partials")))
    return bail(rc);
  if ((rc = c->cuda(w.alloc(&c->walk_work, 4), "walk counters"))) return bail(rc);
  if ((rc = c->cuda(cudaMemset(c->walk_work, 0, 16), "walk counters"))) return bail(rc);
  if ((rc = c->cuda(w.alloc(&c->diag_out, 8), "diag"))) return bail(rc);
  if ((rc = c->cuda(cudaMallocHost(&c->host_stage, (size_t)N * 16 + 256), "pinned stage")))
    return bail(rc);
  const size_t pb = (size_t)N * 32, sb = (size_t)N * 16;
  if ((rc = c->cuda(cudaMemcpy(c->part[0], particles8, pb, cudaMemcpyHostToDevice), "upload")))
    return bail(rc);
  if ((rc = c->cuda(cudaMemcpy(c->part[1], particles8, pb, cudaMemcpyHostToDevice), "upload")))
    return bail(rc);
  for (int k = 0; k < 2; k++) {
    if (stellar4)
      rc = c->cuda(cudaMemcpy(c->stel[k], stellar4, sb, cudaMemcpyHostToDevice), "upload");
    else
      rc = c->cuda(cudaMemset(c->stel[k], 0, sb), "memset");
    if (rc) return bail(rc);
  }
  DevState st0;
  memset(&st0, 0, sizeof(st0));
  st0.p.N = N;
  st0.central[0] = st0.central[1] = -1;
  st0.central_next[0] = st0.central_next[1] = -1;
  c->hp = st0.p;
  if ((rc = c->cuda(cudaMemcpy(c->st, &st0, sizeof(st0), cudaMemcpyHostToDevice), "state")))
    return bail(rc);
  if ((rc = c->cuda(cudaMemset(c->partials, 0, sizeof(double) * c->walk_groups * kPartials), "m")))
    return bail(rc);
  *out = c;
  return GS_OK;
}

int gs_create(uint32_t N, const float* particles8, const float* stellar4, gs_ctx** out) {
  int dev = 0;
  cudaGetDevice(&dev);
  return gs_create_on(dev, N, particles8, stellar4, out);
}

int gs_destroy(gs_ctx* ctx) {
  if (!ctx) return GS_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  ctx->drop_graphs();
  ctx->ws.release();
  if (ctx->host_stage) cudaFreeHost(ctx->host_stage);
  if (ctx->ev) cudaEventDestroy(ctx->ev);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return GS_OK;
}

int gs_update_params(gs_ctx* ctx, const gs_params* params) {
  CTX_CHECK(ctx);
  if (!params) return ctx->fail(GS_EINVAL, "params is NULL");
  ctx->hp = *params;
  ctx->hp.N = ctx->N;
  // the 96-byte uniform goes through pinned memory so the async copy never
  // reads a caller buffer after return
  gs_params* stage = reinterpret_cast<gs_params*>(static_cast<char*>(ctx->host_stage) + (size_t)ctx->N * 16);
  CK(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  *stage = ctx->hp;
  CK(ctx, cudaMemcpyAsync(&ctx->st->p, stage, sizeof(gs_params), cudaMemcpyHostToDevice, ctx->stream),
     "params upload");
  params_fixup_kernel<<<1, 1, 0, ctx->stream>>>(ctx->st, ctx->N);
  CK(ctx, cudaGetLastError(), "params fixup");
  return GS_OK;
}

int gs_set_time(gs_ctx* ctx, double t) {
  CTX_CHECK(ctx);
  CK(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  CK(ctx, cudaMemcpy(&ctx->st->sim_time, &t, sizeof(double), cudaMemcpyHostToDevice), "time");
  return GS_OK;
}

int gs_update_central_mass(gs_ctx* ctx, float mass, uint32_t idx) {
  CTX_CHECK(ctx);
  if (idx >= ctx->N) return ctx->fail(GS_EINVAL, "central index %u >= N %u", idx, ctx->N);
  CK(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  for (int k = 0; k < 2; k++)
    CK(ctx, cudaMemcpy(reinterpret_cast<char*>(ctx->part[k]) + (size_t)idx * 32 + 12, &mass, 4,
                       cudaMemcpyHostToDevice),
       "central mass");
  return GS_OK;
}

int gs_apply_permutation(gs_ctx* ctx, const uint32_t* perm) {
  CTX_CHECK(ctx);
  if (!perm) return ctx->fail(GS_EINVAL, "perm is NULL");
  for (uint32_t i = 0; i < ctx->N; i++)
    if (perm[i] >= ctx->N) return ctx->fail(GS_EINVAL, "perm[%u] = %u out of range", i, perm[i]);
  CK(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  CK(ctx, cudaMemcpyAsync(ctx->perm_user, perm, sizeof(uint32_t) * ctx->N, cudaMemcpyHostToDevice,
                          ctx->stream),
     "perm upload");
  gather_kernel<<<grid_for(ctx->N, 256, 148 * 16), 256, 0, ctx->stream>>>(
      ctx->perm_user, ctx->part[ctx->cur], ctx->part[ctx->cur ^ 1], ctx->stel[ctx->scur],
      ctx->stel[ctx->scur ^ 1], ctx->N, ctx->st, 0);
  CK(ctx, cudaGetLastError(), "gather");
  ctx->cur ^= 1;
  ctx->scur ^= 1;
  CK(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  return GS_OK;
}

int gs_upload_tree(gs_ctx* ctx, const gs_node* nodes, uint32_t num_nodes,
                   const uint32_t* level_ranges, uint32_t n_levels) {
  CTX_CHECK(ctx);
  if (!nodes && num_nodes) return ctx->fail(GS_EINVAL, "nodes is NULL");
  const uint32_t max_bh = 4 * ctx->N + 1024;  // NBodyGPU.js:58
  const uint32_t n = std::min(num_nodes, max_bh);
  if (n > ctx->ws.cap)
    return ctx->fail(GS_EINVAL, "tree of %u nodes exceeds the pool of %u", n, ctx->ws.cap);
  if (!ctx->bh) {
    CK(ctx, ctx->ws.alloc(&ctx->bh, ctx->ws.cap), "bh staging");
    ctx->max_bh = ctx->ws.cap;
  }
  CK(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  if (n) CK(ctx, cudaMemcpy(ctx->bh, nodes, (size_t)n * sizeof(gs_node), cudaMemcpyHostToDevice), "tree");
  if (n)
    upload_convert_kernel<<<grid_for(n, 256, 148 * 8), 256, 0, ctx->stream>>>(
        ctx->bh, n, ctx->N, ctx->ws.cm, ctx->ws.info, ctx->st);
  CK(ctx, cudaGetLastError(), "convert");
  if (level_ranges) {
    ctx->up_lr.assign(level_ranges, level_ranges + 2 * std::min<uint32_t>(n_levels, 16));
  }
  ctx->up_nodes = n;
  ctx->tree = gs_ctx::kTreeUploaded;
  return wait_stream(ctx, 0);
}

int gs_refresh(gs_ctx* ctx) {
  CTX_CHECK(ctx);
  if (ctx->tree == gs_ctx::kTreeUploaded) {
    if (ctx->up_lr.empty()) return GS_OK;  // NBodyGPU.js:309 no-op without levelRanges
    for (int64_t l = (int64_t)ctx->up_lr.size() / 2 - 1; l >= 0; l--) {
      const uint32_t start = ctx->up_lr[2 * l], count = ctx->up_lr[2 * l + 1];
      if (!count) continue;
      if ((uint64_t)start + count > ctx->up_nodes)
        return ctx->fail(GS_EINVAL, "level %lld [%u, +%u) beyond %u nodes", (long long)l, start,
                         count, ctx->up_nodes);
      refresh_level_kernel<<<cdiv(count, 64), 64, 0, ctx->stream>>>(ctx->part[ctx->cur], ctx->ws.cm,
                                                                     ctx->ws.info, start, count);
    }
  } else if (ctx->tree == gs_ctx::kTreeBuilt) {
    BuildBuffers b = ctx->ws.bb(ctx->ws.cap);
    tree_leaves_kernel<kComF32><<<grid_for(ctx->N, 256, 148 * 16), 256, 0, ctx->stream>>>(
        b, ctx->part[ctx->cur], 2, ctx->st);
  }
  CK(ctx, cudaGetLastError(), "refresh");
  return GS_OK;
}

int gs_step(gs_ctx* ctx) {
  CTX_CHECK(ctx);
  enqueue_walk(ctx, 0);
  CK(ctx, cudaGetLastError(), "walk");
  return GS_OK;
}

int gs_star_formation(gs_ctx* ctx) {
  CTX_CHECK(ctx);
  sf_kernel<<<grid_for(ctx->N, 256, 148 * 16), 256, 0, ctx->stream>>>(ctx->part[ctx->cur],
                                                                      ctx->stel[ctx->scur], ctx->N,
                                                                      ctx->st);
  CK(ctx, cudaGetLastError(), "star formation");
  return GS_OK;
}

int gs_read_positions(gs_ctx* ctx, float* out4, uint64_t timeout_ns) {
  CTX_CHECK(ctx);
  if (!out4) return ctx->fail(GS_EINVAL, "out4 is NULL");
  compact_kernel<<<grid_for(ctx->N, 256, 148 * 16), 256, 0, ctx->stream>>>(
      ctx->part[ctx->cur], ctx->energy, ctx->compact, ctx->N);
  CK(ctx, cudaGetLastError(), "compact");
  CK(ctx, cudaMemcpyAsync(ctx->host_stage, ctx->compact, (size_t)ctx->N * 16, cudaMemcpyDeviceToHost,
                          ctx->stream),
     "readback");
  int rc = wait_stream(ctx, timeout_ns);
  if (rc) return rc;
  memcpy(out4, ctx->host_stage, (size_t)ctx->N * 16);
  return GS_OK;
}

int gs_position_buffer(gs_ctx* ctx, void** dptr) {
  CTX_CHECK(ctx);
  if (!dptr) return ctx->fail(GS_EINVAL, "dptr is NULL");
  *dptr = ctx->part[ctx->cur];
  return GS_OK;
}

int gs_stellar_buffer(gs_ctx* ctx, void** dptr) {
  CTX_CHECK(ctx);
  if (!dptr) return ctx->fail(GS_EINVAL, "dptr is NULL");
  *dptr = ctx->stel[ctx->scur];
  return GS_OK;
}

int gs_set_tracking(gs_ctx* ctx, int64_t c1, int64_t c2, const double* h1, const double* h2) {
  CTX_CHECK(ctx);
  if (c1 >= (int64_t)ctx->N || c2 >= (int64_t)ctx->N)
    return ctx->fail(GS_EINVAL, "tracked index out of range");
  ctx->tracking = c1 >= 0 || c2 >= 0;
  tracking_init_kernel<<<1, 1, 0, ctx->stream>>>(
      ctx->st, ctx->part[ctx->cur], c1 < 0 ? -1 : c1, c2 < 0 ? -1 : c2, h1 != nullptr,
      h1 ? h1[0] : 0, h1 ? h1[1] : 0, h1 ? h1[2] : 0, h2 != nullptr, h2 ? h2[0] : 0,
      h2 ? h2[1] : 0, h2 ? h2[2] : 0, ctx->N);
  CK(ctx, cudaGetLastError(), "tracking");
  ctx->drop_graphs();
  return wait_stream(ctx, 0);
}

int gs_get_tracking(gs_ctx* ctx, int64_t* c1, int64_t* c2, double* h1, double* h2) {
  CTX_CHECK(ctx);
  int rc = wait_stream(ctx, 0);
  if (rc) return rc;
  DevState s;
  CK(ctx, cudaMemcpy(&s, ctx->st, sizeof(s), cudaMemcpyDeviceToHost), "state");
  if (c1) *c1 = s.central[0];
  if (c2) *c2 = s.central[1];
  if (h1) memcpy(h1, s.halo_c[0], 3 * sizeof(double));
  if (h2) memcpy(h2, s.halo_c[1], 3 * sizeof(double));
  return GS_OK;
}

int gs_sort_build(gs_ctx* ctx) {
  CTX_CHECK(ctx);
  enqueue_sort_build(ctx, 0);
  CK(ctx, cudaGetLastError(), "sort/build");
  return GS_OK;
}

int gs_set_com_mode(gs_ctx* ctx, int mode) {
  CTX_CHECK(ctx);
  if (mode != kComF32 && mode != kComF64) return ctx->fail(GS_EINVAL, "COM mode %d", mode);
  ctx->com_mode = mode;
  ctx->drop_graphs();
  return GS_OK;
}

int gs_run(gs_ctx* ctx, uint32_t nsteps, int do_sf) {
  CTX_CHECK(ctx);
  for (uint32_t s = 0; s < nsteps; s++) {
    const int key = (ctx->cur) | (ctx->scur << 1) | ((do_sf ? 1 : 0) << 2) | ((ctx->debug ? 1 : 0) << 3);
    auto it = ctx->graphs.find(key);
    if (it == ctx->graphs.end()) {
      const int cur0 = ctx->cur, scur0 = ctx->scur;
      cudaGraph_t g = nullptr;
      CK(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal), "capture");
      enqueue_sort_build(ctx, 1);
      enqueue_walk(ctx, do_sf);
      cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
      ctx->cur = cur0;
      ctx->scur = scur0;
      CK(ctx, e, "end capture");
      cudaGraphExec_t ge = nullptr;
      e = cudaGraphInstantiate(&ge, g, 0);
      cudaGraphDestroy(g);
      CK(ctx, e, "instantiate");
      it = ctx->graphs.emplace(key, ge).first;
    }
    CK(ctx, cudaGraphLaunch(it->second, ctx->stream), "graph launch");
    // a step gathers cur -> cur^1 then walks back: cur unchanged, stellar flipped
    ctx->scur ^= 1;
    ctx->tree = gs_ctx::kTreeBuilt;
  }
  return GS_OK;
}

int gs_stream(gs_ctx* ctx, void** stream) {
  CTX_CHECK(ctx);
  if (!stream) return ctx->fail(GS_EINVAL, "stream is NULL");
  *stream = ctx->stream;
  return GS_OK;
}

int gs_sync(gs_ctx* ctx, uint64_t timeout_ns) {
  CTX_CHECK(ctx);
  return wait_stream(ctx, timeout_ns);
}

int gs_get_tree(gs_ctx* ctx, gs_node* nodes, uint32_t nodes_cap, uint32_t* num_nodes,
                uint32_t* level_ranges, uint32_t lr_cap, uint32_t* n_levels, uint32_t* perm) {
  CTX_CHECK(ctx);
  int rc = wait_stream(ctx, 0);
  if (rc) return rc;
  if (ctx->tree == gs_ctx::kTreeNone) return ctx->fail(GS_ENOTREADY, "no tree yet");
  if (!ctx->bh) {
    CK(ctx, ctx->ws.alloc(&ctx->bh, ctx->ws.cap), "bh staging");
    ctx->max_bh = ctx->ws.cap;
  }
  uint32_t nn = 0, nl = 0;
  std::vector<uint32_t> lr;
  if (ctx->tree == gs_ctx::kTreeBuilt) {
    TreeMeta m;
    CK(ctx, cudaMemcpy(&m, ctx->ws.meta, sizeof(m), cudaMemcpyDeviceToHost), "meta");
    nn = m.num_nodes;
    nl = m.num_levels;
    for (uint32_t l = 0; l < nl; l++) {
      lr.push_back(m.level_start[l]);
      lr.push_back(m.level_count[l]);
    }
    if (nodes) {
      tree_bhnode_kernel<<<grid_for(nn, 256, 148 * 8), 256, 0, ctx->stream>>>(ctx->ws.bb(ctx->ws.cap),
                                                                               ctx->bh);
      CK(ctx, cudaGetLastError(), "materialise");
    }
  } else {
    nn = ctx->up_nodes;
    nl = (uint32_t)ctx->up_lr.size() / 2;
    lr = ctx->up_lr;
    if (nodes && nn) {
      bh_patch_kernel<<<grid_for(nn, 256, 148 * 8), 256, 0, ctx->stream>>>(ctx->bh, ctx->ws.cm, nn);
      CK(ctx, cudaGetLastError(), "patch");
    }
  }
  if (num_nodes) *num_nodes = nn;
  if (n_levels) *n_levels = nl;
  if (level_ranges)
    memcpy(level_ranges, lr.data(), sizeof(uint32_t) * std::min<size_t>(lr.size(), 2 * (size_t)lr_cap));
  if (nodes && nn)
    CK(ctx, cudaMemcpyAsync(nodes, ctx->bh, sizeof(gs_node) * std::min(nn, nodes_cap),
                            cudaMemcpyDeviceToHost, ctx->stream),
       "nodes");
  if (perm) CK(ctx, cudaMemcpyAsync(perm, ctx->ws.vals[0], sizeof(uint32_t) * ctx->N, cudaMemcpyDeviceToHost, ctx->stream), "perm");
  return wait_stream(ctx, 0);
}

int gs_read_state(gs_ctx* ctx, float* particles8, float* stellar4) {
  CTX_CHECK(ctx);
  if (particles8)
    CK(ctx, cudaMemcpyAsync(particles8, ctx->part[ctx->cur], (size_t)ctx->N * 32,
                            cudaMemcpyDeviceToHost, ctx->stream),
       "state");
  if (stellar4)
    CK(ctx, cudaMemcpyAsync(stellar4, ctx->stel[ctx->scur], (size_t)ctx->N * 16,
                            cudaMemcpyDeviceToHost, ctx->stream),
       "stellar");
  return wait_stream(ctx, 0);
}

// Stream-ordered: both ping-pong buffers get the state (like NBodyGPU._init).
int gs_write_state(gs_ctx* ctx, const float* particles8, const float* stellar4) {
  CTX_CHECK(ctx);
  for (int k = 0; k < 2; k++) {
    if (particles8)
      CK(ctx, cudaMemcpyAsync(ctx->part[k], particles8, (size_t)ctx->N * 32, cudaMemcpyHostToDevice,
                              ctx->stream),
         "state");
    if (stellar4)
      CK(ctx, cudaMemcpyAsync(ctx->stel[k], stellar4, (size_t)ctx->N * 16, cudaMemcpyHostToDevice,
                              ctx->stream),
         "stellar");
  }
  return wait_stream(ctx, 0);
}

int gs_set_debug(gs_ctx* ctx, int enable) {
  CTX_CHECK(ctx);
  if (enable && !ctx->dbg_acc) {
    CK(ctx, ctx->ws.alloc(&ctx->dbg_acc, ctx->N), "debug acc");
    CK(ctx, ctx->ws.alloc(&ctx->dbg_dens, ctx->N), "debug density");
  }
  ctx->debug = enable != 0;
  return GS_OK;
}

int gs_read_forces(gs_ctx* ctx, float* acc4, float* density) {
  CTX_CHECK(ctx);
  if (!ctx->dbg_acc) return ctx->fail(GS_ENOTREADY, "gs_set_debug(ctx, 1) first");
  int rc = wait_stream(ctx, 0);
  if (rc) return rc;
  if (acc4) CK(ctx, cudaMemcpy(acc4, ctx->dbg_acc, (size_t)ctx->N * 16, cudaMemcpyDeviceToHost), "acc");
  if (density)
    CK(ctx, cudaMemcpy(density, ctx->dbg_dens, (size_t)ctx->N * 4, cudaMemcpyDeviceToHost), "dens");
  return GS_OK;
}

int gs_energy(gs_ctx* ctx, gs_diag* out) {
  CTX_CHECK(ctx);
  if (!out) return ctx->fail(GS_EINVAL, "out is NULL");
  diag_reduce_kernel<<<1, dim3(32, kPartials), 0, ctx->stream>>>(ctx->partials, ctx->walk_groups,
                                                                  ctx->diag_out);
  CK(ctx, cudaGetLastError(), "diag");
  double h[kPartials];
  CK(ctx, cudaMemcpyAsync(h, ctx->diag_out, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream), "diag");
  int rc = wait_stream(ctx, 0);
  if (rc) return rc;
  out->e_diag = h[0];
  out->e_true = h[1];
  out->momentum[0] = h[2];
  out->momentum[1] = h[3];
  out->momentum[2] = h[4];
  out->mass = h[5];
  return GS_OK;
}

int gs_device_errors(gs_ctx* ctx, uint32_t* bits, int clear) {
  CTX_CHECK(ctx);
  CK(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  unsigned e = 0;
  CK(ctx, cudaMemcpy(&e, &ctx->st->err, 4, cudaMemcpyDeviceToHost), "err");
  if (bits) *bits = e;
  if (clear) CK(ctx, cudaMemset(&ctx->st->err, 0, 4), "clear");
  return GS_OK;
}

int gs_counters(gs_ctx* ctx, uint64_t out[3], int reset) {
  CTX_CHECK(ctx);
  CK(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  unsigned long long c[3];
  CK(ctx, cudaMemcpy(c, ctx->st->counters, sizeof(c), cudaMemcpyDeviceToHost), "counters");
  if (out)
    for (int k = 0; k < 3; k++) out[k] = c[k];
  if (reset) CK(ctx, cudaMemset(ctx->st->counters, 0, sizeof(c)), "reset");
  return GS_OK;
}

// ---- stateless mortonTree.js entry points ----------------------------------------------

namespace {
struct TmpCtx {
  Workspace w;
  cudaStream_t s = nullptr;
  float4* pos = nullptr;
  DevState* st = nullptr;
  ~TmpCtx() {
    if (s) cudaStreamSynchronize(s);
    w.release();
    if (s) cudaStreamDestroy(s);
  }
};

int tmp_fail(cudaError_t e, const char* what) {
  set_err(g_err, "%s: %s", what, cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? GS_ENOMEM : GS_ECUDA;
}

#define TK(expr, what)                                \
  do {                                                \
    cudaError_t _e = (expr);                          \
    if (_e != cudaSuccess) return tmp_fail(_e, what); \
  } while (0)

int tmp_init(TmpCtx& t, uint32_t N) {
  TK(cudaStreamCreateWithFlags(&t.s, cudaStreamNonBlocking), "stream");
  TK(t.w.init(N), "workspace");
  TK(t.w.alloc(&t.pos, N), "positions");
  TK(t.w.alloc(&t.st, 1), "state");
  TK(cudaMemset(t.st, 0, sizeof(DevState)), "state");
  return GS_OK;
}

int tmp_check(TmpCtx& t) {
  TK(cudaStreamSynchronize(t.s), "sync");
  unsigned e = 0;
  TK(cudaMemcpy(&e, &t.st->err, 4, cudaMemcpyDeviceToHost), "err");
  if (e) {
    set_err(g_err, "device error word 0x%x", e);
    return (e & GS_DERR_NODES) ? GS_EINVAL : GS_EDEVICE;
  }
  return GS_OK;
}

// The single empty leaf MortonTree.build makes for N = 0.
void empty_tree(double root, gs_node* nodes, uint32_t* num, uint32_t* lr, uint32_t* nl) {
  if (nodes) {
    memset(nodes, 0, sizeof(gs_node));
    nodes[0].size = (float)root;
    nodes[0].isLeaf = 1;
    for (int k = 0; k < 8; k++) nodes[0].children[k] = -1;
  }
  if (num) *num = 1;
  if (lr) {
    lr[0] = 0;
    lr[1] = 1;
  }
  if (nl) *nl = 1;
}

int tree_outputs(TmpCtx& t, uint32_t max_nodes, gs_node* nodes, uint32_t* num_nodes,
                 uint32_t* level_ranges, uint32_t lr_cap, uint32_t* n_levels) {
  int rc = tmp_check(t);
  if (rc) return rc;
  TreeMeta m;
  TK(cudaMemcpy(&m, t.w.meta, sizeof(m), cudaMemcpyDeviceToHost), "meta");
  if (m.num_nodes > max_nodes) {
    set_err(g_err, "tree needs %u nodes, pool holds %u", m.num_nodes, max_nodes);
    return GS_EINVAL;
  }
  if (num_nodes) *num_nodes = m.num_nodes;
  if (n_levels) *n_levels = m.num_levels;
  if (level_ranges)
    for (uint32_t l = 0; l < m.num_levels && l < lr_cap; l++) {
      level_ranges[2 * l] = m.level_start[l];
      level_ranges[2 * l + 1] = m.level_count[l];
    }
  if (nodes) {
    gs_node* d = nullptr;
    TK(t.w.alloc(&d, std::max<uint32_t>(m.num_nodes, 1)), "nodes");
    tree_bhnode_kernel<<<grid_for(m.num_nodes, 256, 148 * 8), 256, 0, t.s>>>(t.w.bb(max_nodes), d);
    TK(cudaGetLastError(), "materialise");
    TK(cudaMemcpyAsync(nodes, d, sizeof(gs_node) * m.num_nodes, cudaMemcpyDeviceToHost, t.s), "nodes");
    TK(cudaStreamSynchronize(t.s), "sync");
  }
  return GS_OK;
}
}  // namespace

int gs_morton_codes(const float* pos, uint32_t N, uint32_t stride, uint32_t* codes,
                    double* root_size) {
  if ((!pos && N) || (!codes && N) || stride < 3) {
    set_err(g_err, "bad arguments");
    return GS_EINVAL;
  }
  if (N > kMaxN) {
    set_err(g_err, "N too large");
    return GS_EINVAL;
  }
  if (N == 0) {  // mortonTree.js:53 over no particles: -Infinity
    if (root_size) *root_size = -INFINITY;
    return GS_OK;
  }
  TmpCtx t;
  int rc = tmp_init(t, N);
  if (rc) return rc;
  std::vector<float4> h;
  host_pack4(pos, N, stride, h);
  TK(cudaMemcpyAsync(t.pos, h.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, t.s), "upload");
  const uint32_t bb = grid_for(N, kBBoxThreads, kBBoxBlocks);
  bbox_kernel<<<bb, kBBoxThreads, 0, t.s>>>(t.pos, 1, N, t.w.bbox_partials, t.w.bbox_counter,
                                            t.w.frame, t.st, 0);
  codes_kernel<<<grid_for(N, 256, 148 * 8), 256, 0, t.s>>>(t.pos, 1, N, t.w.frame, t.w.keys[0],
                                                            nullptr, 0);
  TK(cudaGetLastError(), "codes");
  MortonFrame f;
  TK(cudaMemcpyAsync(codes, t.w.keys[0], sizeof(uint32_t) * N, cudaMemcpyDeviceToHost, t.s), "codes");
  TK(cudaMemcpyAsync(&f, t.w.frame, sizeof(f), cudaMemcpyDeviceToHost, t.s), "frame");
  rc = tmp_check(t);
  if (rc) return rc;
  if (root_size) *root_size = f.size;
  return GS_OK;
}

int gs_radix_sort_indices(const uint32_t* codes, uint32_t N, uint32_t* perm) {
  if ((!codes || !perm) && N) {
    set_err(g_err, "bad arguments");
    return GS_EINVAL;
  }
  if (N == 0) return GS_OK;
  if (N > kMaxN) {
    set_err(g_err, "N too large");
    return GS_EINVAL;
  }
  TmpCtx t;
  int rc = tmp_init(t, N);
  if (rc) return rc;
  Workspace& w = t.w;
  TK(cudaMemcpyAsync(w.keys[0], codes, sizeof(uint32_t) * N, cudaMemcpyHostToDevice, t.s), "upload");
  // radixSortIndices orders by the low 30 bits only (3 x 10-bit digits)
  mask30_kernel<<<grid_for(N, 256, 148 * 8), 256, 0, t.s>>>(w.keys[0], N);
  cudaMemsetAsync(w.sort_scratch, 0, w.sort_scratch_bytes, t.s);
  key_hist_kernel<<<grid_for(N, 256, 148 * 8), 256, 0, t.s>>>(w.keys[0], N, w.hist(), kSortPasses);
  for (int p = 0; p < kSortPasses; p++) {
    const int src = p & 1, dst = src ^ 1;
    uint32_t* lb = w.lookback() + (size_t)p * w.tiles * 256;
    if (p == 0)
      onesweep_pass<true><<<w.tiles, kSortThreads, 0, t.s>>>(w.keys[src], nullptr, w.keys[dst],
                                                             w.vals[dst], w.hist() + p * 256, lb,
                                                             w.tile_ctr() + p, N, 8 * p, t.st);
    else
      onesweep_pass<false><<<w.tiles, kSortThreads, 0, t.s>>>(w.keys[src], w.vals[src], w.keys[dst],
                                                              w.vals[dst], w.hist() + p * 256, lb,
                                                              w.tile_ctr() + p, N, 8 * p, t.st);
  }
  TK(cudaGetLastError(), "sort");
  TK(cudaMemcpyAsync(perm, w.vals[0], sizeof(uint32_t) * N, cudaMemcpyDeviceToHost, t.s), "perm");
  return tmp_check(t);
}

int gs_tree_build(const uint32_t* sorted_codes, const float* pos3, const float* masses, uint32_t N,
                  double root_size, uint32_t max_nodes, gs_node* nodes, uint32_t* num_nodes,
                  uint32_t* level_ranges, uint32_t lr_cap, uint32_t* n_levels) {
  if (N == 0) {
    empty_tree(root_size, nodes, num_nodes, level_ranges, n_levels);
    return GS_OK;
  }
  if (!sorted_codes || !pos3 || !masses || N > kMaxN) {
    set_err(g_err, "bad arguments");
    return GS_EINVAL;
  }
  TmpCtx t;
  int rc = tmp_init(t, N);
  if (rc) return rc;
  std::vector<float4> h(N);
  std::vector<uint32_t> c(N);
  for (uint32_t i = 0; i < N; i++) {
    h[i] = make_float4(pos3[3 * (size_t)i], pos3[3 * (size_t)i + 1], pos3[3 * (size_t)i + 2], masses[i]);
    c[i] = sorted_codes[i] & 0x3fffffffu;
  }
  TK(cudaMemcpyAsync(t.pos, h.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, t.s), "upload");
  TK(cudaMemcpyAsync(t.w.keys[0], c.data(), sizeof(uint32_t) * N, cudaMemcpyHostToDevice, t.s), "codes");
  if (max_nodes == 0) max_nodes = 2 * N + 4096;
  enqueue_build(t.w, t.pos, 1, max_nodes, kComJs, root_size, nullptr, t.s, t.st, nullptr);
  TK(cudaGetLastError(), "build");
  return tree_outputs(t, max_nodes, nodes, num_nodes, level_ranges, lr_cap, n_levels);
}

int gs_sort_and_build(const float* particles8, const float* stellar4, uint32_t N,
                      int64_t track_idx2, float* sorted8, float* sorted_stellar4, uint32_t* perm,
                      gs_node* nodes, uint32_t max_nodes, uint32_t* num_nodes,
                      uint32_t* level_ranges, uint32_t lr_cap, uint32_t* n_levels,
                      int64_t* central_idx, int64_t* central_idx2, float* sorted_mass) {
  if (N == 0) {
    empty_tree(-INFINITY, nodes, num_nodes, level_ranges, n_levels);
    if (central_idx) *central_idx = 0;
    if (central_idx2) *central_idx2 = -1;
    return GS_OK;
  }
  if (!particles8 || N > kMaxN) {
    set_err(g_err, "bad arguments");
    return GS_EINVAL;
  }
  TmpCtx t;
  int rc = tmp_init(t, N);
  if (rc) return rc;
  float4 *P = nullptr, *P2 = nullptr, *S = nullptr, *S2 = nullptr;
  TK(t.w.alloc(&P, 2 * (size_t)N), "particles");
  TK(t.w.alloc(&P2, 2 * (size_t)N), "particles");
  TK(t.w.alloc(&S, N), "stellar");
  TK(t.w.alloc(&S2, N), "stellar");
  TK(cudaMemcpyAsync(P, particles8, (size_t)N * 32, cudaMemcpyHostToDevice, t.s), "upload");
  if (stellar4) TK(cudaMemcpyAsync(S, stellar4, (size_t)N * 16, cudaMemcpyHostToDevice, t.s), "upload");
  else TK(cudaMemsetAsync(S, 0, (size_t)N * 16, t.s), "memset");
  enqueue_codes_sort(t.w, P, 2, t.s, t.st, 0);
  gather_kernel<<<grid_for(N, 256, 148 * 16), 256, 0, t.s>>>(t.w.vals[0], P, P2, S, S2, N, t.st, 0);
  if (max_nodes == 0) max_nodes = 2 * N + 4096;
  enqueue_build(t.w, P2, 2, max_nodes, kComJs, 0.0, t.w.frame, t.s, t.st, nullptr);
  TK(cudaGetLastError(), "sort and build");
  std::vector<uint32_t> hp(N);
  TK(cudaMemcpyAsync(hp.data(), t.w.vals[0], sizeof(uint32_t) * N, cudaMemcpyDeviceToHost, t.s), "perm");
  if (sorted8) TK(cudaMemcpyAsync(sorted8, P2, (size_t)N * 32, cudaMemcpyDeviceToHost, t.s), "sorted");
  if (sorted_stellar4)
    TK(cudaMemcpyAsync(sorted_stellar4, S2, (size_t)N * 16, cudaMemcpyDeviceToHost, t.s), "stellar");
  rc = tree_outputs(t, max_nodes, nodes, num_nodes, level_ranges, lr_cap, n_levels);
  if (rc) return rc;
  int64_t c1 = 0, c2 = -1;
  for (uint32_t i = 0; i < N; i++) {
    if (hp[i] == 0) c1 = i;
    if ((int64_t)hp[i] == track_idx2) c2 = i;
  }
  if (perm) memcpy(perm, hp.data(), sizeof(uint32_t) * N);
  if (central_idx) *central_idx = c1;
  if (central_idx2) *central_idx2 = c2;
  if (sorted_mass) {
    std::vector<float> s8((size_t)N * 8);
    TK(cudaMemcpy(s8.data(), P2, (size_t)N * 32, cudaMemcpyDeviceToHost), "mass");
    for (uint32_t i = 0; i < N; i++) sorted_mass[i] = s8[(size_t)i * 8 + 3];
  }
  return GS_OK;
}

}  // extern "C"

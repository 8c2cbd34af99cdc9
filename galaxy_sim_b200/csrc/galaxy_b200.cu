// Host runtime and C ABI of the B200 gravity path (declarations and reference
// citations in include/galaxy_b200.h).
//
// A context is a pool of galaxy slots over one set of device buffers and one
// CUDA stream. Every operation is stream-ordered like the WebGPU command encoder
// it replaces; full steps of all resident galaxies are one launch per kernel
// (segmented sort, build and walk), replayed from captured CUDA graphs.
//
// Pool memory: particle records live at [off, off + n) of the particle pool
// (offsets aligned to kAlign), the galaxy's nodes at [2 off, 2 off + 2 n) of
// the node pool. A bucketed octree of n particles has at most n leaves (every
// leaf holds a particle) and at most n / 17 internal nodes per depth 0..9, so
// at most 1.59 n nodes: node ranges never overlap and need no allocator of
// their own. A single-galaxy context gives its galaxy 2 n + 4096 nodes, the
// reference's MortonTree pool, so any uploaded tree of that size fits.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
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
// host-side fault injection (gs_test_fail_alloc): the number of device
// allocations still to succeed before one fails; negative: none fails
std::atomic<long long> g_fail_alloc_in{-1};

constexpr uint64_t kMaxPool = 1ull << 27;  // node indices (2 cap + 4096) fit the walk's 29-bit fields
constexpr uint32_t kMaxSlots = 4096;
constexpr uint32_t kAlign = 256;           // particle offset alignment of a galaxy

inline uint32_t cdiv(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }

void set_err(char* dst, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(dst, 512, fmt, ap);
  va_end(ap);
}

// Launch with programmatic stream serialization: the kernel may be scheduled
// while its predecessor in the stream drains and waits for it in griddep_wait().
template <typename... KArgs, typename... Args>
void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

uint32_t grid_for(uint64_t N, uint32_t threads, uint32_t cap_blocks) {
  return std::min<uint32_t>(cap_blocks, std::max<uint32_t>(1, cdiv(N, threads)));
}

// Sizes of every pool buffer for a particle capacity and slot count.
struct Plan {
  uint64_t cap = 0, nodes = 0;
  uint32_t slots = 0, sort_tiles = 0, flag_tiles = 0, groups = 0, diag_chunks = 0;
  size_t sort_words = 0;  // hist[slots][4][256] | tile counters[16] | look-back[4][tiles][256]
};

Plan make_plan(uint64_t cap, uint32_t slots) {
  Plan p;
  p.cap = cap;
  p.slots = slots;
  p.nodes = 2 * cap + 4096;
  p.sort_tiles = cdiv(cap, kSortTileMin) + slots;  // room for the smallest tile
  p.flag_tiles = cdiv(cap, kFlagTile) + slots;
  p.groups = cdiv(cap, kWalkGroup) + slots;
  p.diag_chunks = cdiv(p.groups, kDiagChunk) + slots;
  p.sort_words = (size_t)slots * kSortPasses * 256 + 16 + (size_t)kSortPasses * p.sort_tiles * 256;
  return p;
}

// Device bytes a pool allocates (the debug force buffers and the BHNode staging
// of gs_get_tree / gs_upload_tree come on demand and are not included).
uint64_t plan_bytes(const Plan& p) {
  const uint64_t c = p.cap, n = p.nodes, s = p.slots;
  uint64_t b = 0;
  b += c * (2 * 32 + 2 * 16 + 4 + 16 + 4 + 4);   // particles x2, stellar x2, energy, compact, perm, inv
  b += c * (4 * 4 + 1 + 2 * 4) + 2 * 4 + 4;     // keys x2, vals x2, dl, leaf lists
  b += p.sort_words * 4;
  b += (uint64_t)p.flag_tiles * (6 * 4 + 2 * kCounters * 4);
  b += n * (16 + 16 + 4 + 4 + 4 + 1 + 4) + 4;   // cm, info, node_start, child_base, parent, depth, arrive
  b += s * (sizeof(DevState) + sizeof(TreeMeta) + sizeof(MortonFrame) + 4 + kPartials * 8 + sizeof(SegDesc));
  b += (uint64_t)(p.sort_tiles + p.flag_tiles + p.groups) * 4;
  b += (uint64_t)p.groups * kWalkParts * kPartials * 8 + 16;
  b += (uint64_t)p.diag_chunks * kPartials * 8 + s * 4;
  return b;
}

// First-fit allocator of particle ranges (free holes keyed by offset).
struct RangeAlloc {
  std::map<uint64_t, uint64_t> free;  // off -> len
  void init(uint64_t cap) {
    free.clear();
    if (cap) free[0] = cap;
  }
  bool alloc(uint64_t len, uint64_t* off) {
    for (auto it = free.begin(); it != free.end(); ++it) {
      if (it->second < len) continue;
      *off = it->first;
      const uint64_t rest = it->second - len;
      free.erase(it);
      if (rest) free[*off + len] = rest;
      return true;
    }
    return false;
  }
  void release(uint64_t off, uint64_t len) {
    auto it = free.emplace(off, len).first;
    auto nx = std::next(it);
    if (nx != free.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free.erase(nx);
    }
    if (it != free.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free.erase(it);
      }
    }
  }
  uint64_t largest() const {
    uint64_t m = 0;
    for (auto& kv : free) m = std::max(m, kv.second);
    return m;
  }
};

struct Slot {
  bool live = false;
  uint32_t off = 0, n = 0, span = 0;  // span: the allocated (aligned) particle range
  uint32_t node_off = 0, node_cap = 0;
  gs_params hp{};
  bool tracking = false;
  enum { kTreeNone, kTreeUploaded, kTreeBuilt } tree = kTreeNone;
  uint32_t up_nodes = 0;
  std::vector<uint32_t> up_lr;
  std::vector<gs_node> up_host;  // the uploaded BHNodes (COM patched on readback)
  uint32_t max_nodes = 0;        // MortonTree pool of the leaf clause (0: 2n + 4096)
  uint32_t rank = 0;             // position in the current layout
};

}  // namespace

struct gs_ctx {
  int device = 0;
  int sms = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev = nullptr;
  Plan plan;
  std::vector<void*> owned;
  // particle pool
  float4* part[2] = {nullptr, nullptr};
  float4* stel[2] = {nullptr, nullptr};
  int cur = 0, scur = 0;
  float* energy = nullptr;
  float4* compact = nullptr;
  uint32_t* perm_user = nullptr;
  uint32_t* inv = nullptr;
  // sort
  uint32_t* keys[2] = {nullptr, nullptr};
  uint32_t* vals[2] = {nullptr, nullptr};
  uint32_t* sort_scratch = nullptr;
  // bbox / frames
  int* bbox_part = nullptr;
  unsigned* seg_ctr = nullptr;
  MortonFrame* frames = nullptr;
  // build
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
  // per slot
  DevState* st = nullptr;
  double* diag_out = nullptr;  // [slots][kPartials]
  double* diag_chunk = nullptr;  // [diag chunks][kPartials]
  unsigned* diag_ctr = nullptr;  // [slots]
  // layout
  SegDesc* segs = nullptr;
  uint32_t* sort_map = nullptr;
  uint32_t* flag_map = nullptr;
  uint32_t* group_map = nullptr;
  Layout lay{};
  std::vector<SegDesc> seg_host;  // the layout's galaxies, host copy
  bool lay_dirty = true;
  uint32_t hist_slots = 0;  // histogram slots cleared per step (max live slot + 1)
  // walk
  double* partials = nullptr;
  unsigned* walk_work = nullptr;
  uint32_t walk_grid = 0;   // persistent walk grid (largest class)
  float4* split_buf = nullptr;       // split walk partial sums (grown on demand)
  unsigned* split_arrive = nullptr;  // split walk arrivals per work item (zero between launches)
  size_t split_buf_cap = 0, split_arrive_cap = 0;
  float4* dbg_acc = nullptr;
  float* dbg_dens = nullptr;
  bool debug = false;
  gs_node* bh = nullptr;  // BHNode staging (upload / materialise)
  uint32_t max_bh = 0;
  // slots
  std::vector<Slot> slots;
  RangeAlloc palloc;
  uint32_t sel = 0;
  bool single = false;  // created by gs_create: one galaxy, node pool 2N + 4096
  int com_mode = kComF32;
  int sort_items = kSortItems;     // tuning: keys per thread of a sort tile (0: by galaxy size; 4, 8 or 16)
  int sort_eff = kSortItems;       // the layout's keys per thread (sort_items, or chosen by size)
  int walk_bps = kWalkBlocksPerSM; // tuning: persistent walk blocks per SM (1..8; < 8: 72-register build)
  int walk_group = 32;             // tuning: walk group size (0: by galaxy size; 4, 8, 16 or 32 particles)
  int walk_split = 1;              // tuning: walk splits per work item of a lone galaxy (0: by its size; 1, 2, 4, 8)
  uint32_t walk_items[4] = {0, 0, 0, 0};  // work items per lanes-per-particle class (1, 2, 4, 8)
  bool walk_comp = false;  // compensated far-field sums in the walk (a Kahan step per round)
  // pinned staging of Params uploads: a ring of entries, each rewritten only after
  // the copy that last read it has run (its event), so an update does not wait
  // for the queued steps (NBodyGPU.updateParams is a queue write too)
  static constexpr int kParamRing = 8;
  void* host_stage = nullptr;  // pinned: [kParamRing] params
  cudaEvent_t param_ev[kParamRing] = {};
  bool param_used[kParamRing] = {};
  int param_next = 0;
  // asynchronous position readback (gs_encode_position_readback), set up on first
  // use: a copy stream, the events ordering it after the compaction, a mapped
  // pinned word block for the diagnostics snapshot and the error word, and the
  // request in flight (at most one per context, like the reference's readbackInFlight)
  cudaStream_t rb_stream = nullptr;
  cudaEvent_t rb_ready = nullptr, rb_done = nullptr;
  double* rb_host = nullptr;       // [kPartials] diagnostics, then the error word
  double* rb_host_dev = nullptr;   // the same block as the device sees it
  gs_diag* rb_diag = nullptr;      // caller's diagnostics destination (may be NULL)
  uint32_t rb_slot = 0;
  bool rb_pending = false;
  std::map<int, cudaGraphExec_t> graphs;
  uint32_t step_kernels = 0;  // kernel nodes of the last captured step graph
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
  template <typename T>
  cudaError_t alloc(T** p, size_t count) {
    void* q = nullptr;
    if (g_fail_alloc_in.load() >= 0 && g_fail_alloc_in.fetch_sub(1) == 0) return cudaErrorMemoryAllocation;
    cudaError_t e = cudaMalloc(&q, count * sizeof(T) + 16);
    if (e != cudaSuccess) return e;
    owned.push_back(q);
    *p = reinterpret_cast<T*>(q);
    return cudaSuccess;
  }
  uint32_t* hist() const { return sort_scratch; }
  uint32_t* tile_ctr() const { return sort_scratch + (size_t)plan.slots * kSortPasses * 256; }
  uint32_t* lookback() const { return tile_ctr() + 16; }
  BuildBuffers bb() const {
    BuildBuffers b;
    b.codes = keys[0];
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
  bool any_tracking() const {
    for (const Slot& s : slots)
      if (s.live && s.tracking) return true;
    return false;
  }
  Slot* selected() { return sel < slots.size() && slots[sel].live ? &slots[sel] : nullptr; }
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

// The selected galaxy, or fail with GS_ENOTREADY.
#define SLOT(ctx, s)                                                                       \
  Slot* s = (ctx)->selected();                                                             \
  if (!s) return (ctx)->fail(GS_ENOTREADY, "no galaxy in selected slot %u", (ctx)->sel);

namespace {

int pool_init(gs_ctx* c, int device, uint64_t cap, uint32_t slots) {
  c->device = device;
  c->plan = make_plan(cap, slots);
  const Plan& p = c->plan;
  cudaSetDevice(device);
  cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
  CK(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream");
  CK(c, cudaEventCreateWithFlags(&c->ev, cudaEventDisableTiming), "event");
#define A(ptr, cnt) CK(c, c->alloc(&(ptr), (cnt)), #ptr)
  A(c->part[0], 2 * p.cap);
  A(c->part[1], 2 * p.cap);
  A(c->stel[0], p.cap);
  A(c->stel[1], p.cap);
  A(c->energy, p.cap);
  A(c->compact, p.cap);
  A(c->perm_user, p.cap);
  A(c->inv, p.cap);
  A(c->keys[0], p.cap);
  A(c->keys[1], p.cap);
  A(c->vals[0], p.cap);
  A(c->vals[1], p.cap);
  A(c->sort_scratch, p.sort_words);
  A(c->bbox_part, (size_t)p.flag_tiles * 6);
  A(c->seg_ctr, p.slots);
  A(c->frames, p.slots);
  A(c->dl, p.cap + 4);
  A(c->blk_counts, (size_t)p.flag_tiles * kCounters);
  A(c->blk_offs, (size_t)p.flag_tiles * kCounters);
  A(c->meta, p.slots);
  A(c->node_start, p.nodes);
  A(c->child_base, p.nodes + 1);
  A(c->parent, p.nodes);
  A(c->depth, p.nodes);
  A(c->arrive, p.nodes);
  A(c->leaf_node, p.cap + 1);
  A(c->leaf_start, p.cap + 1);
  A(c->cm, p.nodes);
  A(c->info, p.nodes);
  A(c->st, p.slots);
  A(c->diag_out, (size_t)p.slots * kPartials);
  A(c->diag_chunk, (size_t)p.diag_chunks * kPartials);
  A(c->diag_ctr, p.slots);
  A(c->segs, p.slots);
  A(c->sort_map, p.sort_tiles);
  A(c->flag_map, p.flag_tiles);
  A(c->group_map, p.groups);
  A(c->partials, (size_t)p.groups * kWalkParts * kPartials);
  A(c->walk_work, 4);
#undef A
  CK(c, cudaMemset(c->seg_ctr, 0, sizeof(unsigned) * p.slots), "memset");
  CK(c, cudaMemset(c->arrive, 0, sizeof(uint32_t) * p.nodes), "memset");
  CK(c, cudaMemset(c->cm, 0, sizeof(float4) * p.nodes), "memset");
  CK(c, cudaMemset(c->info, 0, sizeof(WalkInfo) * p.nodes), "memset");
  CK(c, cudaMemset(c->meta, 0, sizeof(TreeMeta) * p.slots), "memset");
  CK(c, cudaMemset(c->st, 0, sizeof(DevState) * p.slots), "memset");
  CK(c, cudaMemset(c->diag_out, 0, sizeof(double) * kPartials * p.slots), "memset");
  CK(c, cudaMemset(c->diag_ctr, 0, sizeof(unsigned) * p.slots), "memset");
  CK(c, cudaMemset(c->partials, 0, sizeof(double) * kPartials * kWalkParts * p.groups), "memset");
  CK(c, cudaMemset(c->walk_work, 0, 16), "memset");
  CK(c, cudaMallocHost(&c->host_stage, sizeof(gs_params) * (size_t)gs_ctx::kParamRing + 256), "pinned stage");
  for (int k = 0; k < gs_ctx::kParamRing; k++)
    CK(c, cudaEventCreateWithFlags(&c->param_ev[k], cudaEventDisableTiming), "params event");
  c->slots.assign(p.slots, Slot());
  c->palloc.init(p.cap);
  c->lay_dirty = true;
  return GS_OK;
}

void pool_release(gs_ctx* c) {
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->rb_stream) cudaStreamSynchronize(c->rb_stream);  // a readback in flight lands first
  c->drop_graphs();
  for (void* q : c->owned) cudaFree(q);
  c->owned.clear();
  if (c->rb_host) cudaFreeHost(c->rb_host);
  if (c->rb_ready) cudaEventDestroy(c->rb_ready);
  if (c->rb_done) cudaEventDestroy(c->rb_done);
  if (c->rb_stream) cudaStreamDestroy(c->rb_stream);
  c->rb_host = c->rb_host_dev = nullptr;
  c->rb_ready = c->rb_done = nullptr;
  c->rb_stream = nullptr;
  c->rb_pending = false;
  if (c->host_stage) cudaFreeHost(c->host_stage);
  for (int k = 0; k < gs_ctx::kParamRing; k++) {
    if (c->param_ev[k]) cudaEventDestroy(c->param_ev[k]);
    c->param_ev[k] = nullptr;
    c->param_used[k] = false;
  }
  if (c->ev) cudaEventDestroy(c->ev);
  if (c->stream) cudaStreamDestroy(c->stream);
  c->host_stage = nullptr;
  c->ev = nullptr;
  c->stream = nullptr;
}

// Walk lanes per particle of a galaxy of n particles: the context's forced group
// size, or by size (a small galaxy walks in groups of 8 or 16 particles so that
// its walk fills more warps).
uint32_t walk_lpp(const gs_ctx* c, uint32_t n) {
  if (c->walk_group == 4) return 8;
  if (c->walk_group == 8) return 4;
  if (c->walk_group == 16) return 2;
  if (c->walk_group == 32) return 1;
  if (n <= kWalkAuto8) return 4;
  if (n <= kWalkAuto16) return 2;
  return 1;
}

// Walk splits per work item of a lone galaxy of n particles walked in groups of
// lpp > 1 lanes per particle: the context's forced count, or by size (a small
// galaxy's walk is as long as its densest work items; splitting their trees
// shortens them). Groups of 32 (lpp 1) walk unsplit.
uint32_t walk_split_of(const gs_ctx* c, uint32_t n, uint32_t lpp) {
  if (lpp == 1) return 1;
  if (c->walk_split > 0) return (uint32_t)c->walk_split;
  if (n <= kSplitAuto4) return 4;
  if (n <= kSplitAuto2) return 2;
  return 1;
}

// Sort keys per thread of a lone galaxy of n particles with the tile depth chosen
// by size: a small galaxy sorts in more, smaller tiles (measured on a B200: 4
// keys per thread fastest up to 65536 particles, 8 at 262144, 16 at 524288).
int sort_items_of(const gs_ctx* c, uint32_t n) {
  if (c->sort_items > 0) return c->sort_items;
  if (n <= kSortAuto4) return 4;
  if (n <= kSortAuto8) return 8;
  return 16;
}

// Rebuild the device layout (galaxies in offset order, tile/group maps) after
// slots were added or removed. The stream must be idle (no step in flight).
int ensure_layout(gs_ctx* c) {
  if (!c->lay_dirty) return GS_OK;
  std::vector<uint32_t> order;
  for (uint32_t s = 0; s < c->slots.size(); s++)
    if (c->slots[s].live) order.push_back(s);
  std::sort(order.begin(), order.end(),
            [&](uint32_t a, uint32_t b) { return c->slots[a].off < c->slots[b].off; });
  std::vector<SegDesc> h(order.size());
  uint32_t st = 0, ft = 0, gr = 0, dc = 0, hs = 0;
  uint32_t items[4] = {0, 0, 0, 0};
  uint32_t it = 0;  // walk items so far (their diagnostic partials are contiguous per galaxy)
  uint32_t nmax = 0;
  for (uint32_t s : order) nmax = std::max(nmax, c->slots[s].n);
  const int items_eff = sort_items_of(c, nmax);
  for (size_t r = 0; r < order.size(); r++) {
    Slot& s = c->slots[order[r]];
    s.rank = (uint32_t)r;
    SegDesc d;
    memset(&d, 0, sizeof(d));
    d.off = s.off;
    d.n = s.n;
    d.node_off = s.node_off;
    d.node_cap = s.node_cap;
    d.sort_tile0 = st;
    d.flag_tile0 = ft;
    d.group0 = gr;
    d.max_nodes = s.max_nodes ? s.max_nodes : 2 * s.n + 4096;
    d.slot = order[r];
    d.diag_chunk0 = dc;
    d.wlpp = walk_lpp(c, s.n);
    d.item0 = it;
    d.wsplit = order.size() == 1 ? walk_split_of(c, s.n, d.wlpp) : 1;  // a pool of several fills the GPU unsplit
    it += cdiv(s.n, kWalkGroup) * d.wlpp;
    h[r] = d;
    dc += cdiv(cdiv(s.n, kWalkGroup), kDiagChunk);
    st += cdiv(s.n, (uint64_t)kSortThreads * items_eff);
    ft += cdiv(s.n, kFlagTile);
    items[h[r].wlpp == 1 ? 0 : h[r].wlpp == 2 ? 1 : h[r].wlpp == 4 ? 2 : 3] +=
        cdiv(s.n, kWalkGroup) * h[r].wlpp * h[r].wsplit;
    gr += cdiv(s.n, kWalkGroup);
    hs = std::max(hs, order[r] + 1);
  }
  if (st > c->plan.sort_tiles || ft > c->plan.flag_tiles || gr > c->plan.groups ||
      dc > c->plan.diag_chunks)
    return c->fail(GS_EINVAL, "layout exceeds the pool's tile capacity");
  CK(c, cudaStreamSynchronize(c->stream), "sync");
  if (h.size() == 1 && h[0].wsplit > 1) {  // the split walk's sums and arrival counters
    const size_t need = (size_t)3 * h[0].wsplit * h[0].n;
    const size_t arr = (size_t)cdiv(h[0].n, kWalkGroup) * h[0].wlpp;
    if (need > c->split_buf_cap) {
      float4* p = nullptr;
      CK(c, c->alloc(&p, need), "split walk sums");
      c->split_buf = p;  // a smaller one stays owned until the context is destroyed
      c->split_buf_cap = need;
    }
    if (arr > c->split_arrive_cap) {
      unsigned* p = nullptr;
      CK(c, c->alloc(&p, arr), "split walk arrivals");
      CK(c, cudaMemset(p, 0, arr * sizeof(unsigned)), "memset");
      c->split_arrive = p;
      c->split_arrive_cap = arr;
    }
  }
  if (!h.empty()) {
    CK(c, cudaMemcpy(c->segs, h.data(), sizeof(SegDesc) * h.size(), cudaMemcpyHostToDevice), "layout");
    const uint32_t tot = std::max(st, std::max(ft, gr));
    layout_maps_kernel<<<grid_for(tot, 256, 148 * 8), 256, 0, c->stream>>>(
        c->segs, (uint32_t)h.size(), c->sort_map, st, c->flag_map, ft, c->group_map, gr);
    CK(c, cudaGetLastError(), "layout maps");
  }
  Layout& L = c->lay;
  L.segs = c->segs;
  L.seg_of_sort_tile = c->sort_map;
  L.seg_of_flag_tile = c->flag_map;
  L.seg_of_group = c->group_map;
  L.nseg = (uint32_t)h.size();
  L.sort_tiles = st;
  L.flag_tiles = ft;
  L.groups = gr;
  L.diag_chunks = dc;
  c->hist_slots = hs;
  c->seg_host = h;
  c->sort_eff = items_eff;
  const uint32_t most = std::max(std::max(items[0], items[1]), std::max(items[2], items[3]));
  c->walk_grid = std::min<uint32_t>(std::max<uint32_t>(1, cdiv(most, kWalkWarps)), (uint32_t)c->sms * c->walk_bps);
  for (int k = 0; k < 4; k++) c->walk_items[k] = items[k];
  c->drop_graphs();
  c->lay_dirty = false;
  return GS_OK;
}

// bbox, Morton frames and codes of `pos` (float4 records, stride in float4)
// into keys[0], with the digit histograms of the sort.
void enqueue_codes_sort(gs_ctx* c, const float4* pos, uint32_t stride, int advance_time) {
  const Layout& L = c->lay;
  cudaStream_t s = c->stream;
  launch_pdl(bbox_kernel, L.flag_tiles, kTileThreads, s, pos, stride, L, c->bbox_part, c->seg_ctr,
             c->frames, c->st, advance_time, c->sort_scratch,
             (uint32_t)((size_t)c->hist_slots * kSortPasses * 256), c->tile_ctr(),
             (uint32_t)(16 + (size_t)kSortPasses * L.sort_tiles * 256));
  launch_pdl(codes_kernel, L.flag_tiles, kTileThreads, s, pos, stride, L, (const MortonFrame*)c->frames,
             c->keys[0], c->hist(), (int)kSortPasses);
}

template <int ITEMS>
void sort_passes_items(gs_ctx* c, bool inv, uint32_t spin_limit, uint32_t withhold) {
  const Layout& L = c->lay;
  cudaStream_t s = c->stream;
  for (int p = 0; p < kSortPasses; p++) {
    const int src = p & 1, dst = src ^ 1;
    uint32_t* lb = c->lookback() + (size_t)p * L.sort_tiles * 256;
    uint32_t* ctr = c->tile_ctr() + p;
    const uint32_t* kin = c->keys[src];
    const uint32_t* vin = p == 0 ? nullptr : c->vals[src];
    uint32_t* iv = (p == kSortPasses - 1 && inv) ? c->inv : nullptr;
    const uint32_t* h = c->hist();
    if (p == 0)
      launch_pdl(onesweep_pass<true, false, ITEMS>, L.sort_tiles, kSortThreads, s, kin, vin, c->keys[dst],
                 c->vals[dst], iv, h, p, lb, ctr, L, c->st, spin_limit, withhold);
    else if (p < kSortPasses - 1)
      launch_pdl(onesweep_pass<false, false, ITEMS>, L.sort_tiles, kSortThreads, s, kin, vin, c->keys[dst],
                 c->vals[dst], iv, h, p, lb, ctr, L, c->st, spin_limit, withhold);
    else
      launch_pdl(onesweep_pass<false, true, ITEMS>, L.sort_tiles, kSortThreads, s, kin, vin, c->keys[dst],
                 c->vals[dst], iv, h, p, lb, ctr, L, c->st, spin_limit, withhold);
  }
}

// stable segmented sort of keys[0] -> keys[0] (sorted codes), vals[0] (gather
// permutation) and, with inv, the inverse permutation; tile size per the tuning.
// spin_limit / withhold: the look-back wait's failure-detection test settings
// (production: kSpinLimit, no withheld tile).
void enqueue_sort_passes(gs_ctx* c, bool inv, uint32_t spin_limit = kSpinLimit, uint32_t withhold = kNoTile) {
  if (c->sort_eff == 4) sort_passes_items<4>(c, inv, spin_limit, withhold);
  else if (c->sort_eff == 8) sort_passes_items<8>(c, inv, spin_limit, withhold);
  else sort_passes_items<16>(c, inv, spin_limit, withhold);
}

// the trees over keys[0] (sorted codes) with COM from pos; root size from the
// Morton frames of the preceding sort (frames) or root_size.
void enqueue_build(gs_ctx* c, const float4* pos, uint32_t stride, int com_mode, double root_size,
                   const MortonFrame* frames) {
  const Layout& L = c->lay;
  cudaStream_t s = c->stream;
  BuildBuffers b = c->bb();
  launch_pdl(tree_flags_kernel, L.flag_tiles, kFlagThreads, s, b, L);
  launch_pdl(tree_scan_kernel, L.nseg, kScanThreads, s, b, L, root_size, frames, c->st);
  launch_pdl(tree_emit_kernel, L.flag_tiles, kFlagThreads, s, b, L, c->st);
  if (com_mode == kComJs)
    launch_pdl(tree_leaves_kernel<kComJs>, L.flag_tiles, kLeafThreads, s, b, L, pos, stride, c->st);
  else if (com_mode == kComF64)
    launch_pdl(tree_leaves_kernel<kComF64>, L.flag_tiles, kLeafThreads, s, b, L, pos, stride, c->st);
  else
    launch_pdl(tree_leaves_kernel<kComF32>, L.flag_tiles, kLeafThreads, s, b, L, pos, stride, c->st);
}

template <int MINB, int LPP>
void launch_walk(int v, uint32_t g, cudaStream_t s, const WalkArgs& a) {
  switch (v) {
#define GS_WALK_CASE(V, SF, DBG, ONE, COMP) \
  case V: launch_pdl(walk_kernel<SF, DBG, ONE, COMP, MINB, LPP>, g, kWalkThreads, s, a); break;
    GS_WALK_CASE(0, false, false, false, false)
    GS_WALK_CASE(1, true, false, false, false)
    GS_WALK_CASE(2, false, true, false, false)
    GS_WALK_CASE(3, true, true, false, false)
    GS_WALK_CASE(4, false, false, true, false)
    GS_WALK_CASE(5, true, false, true, false)
    GS_WALK_CASE(6, false, true, true, false)
    GS_WALK_CASE(7, true, true, true, false)
    GS_WALK_CASE(8, false, false, false, true)
    GS_WALK_CASE(9, true, false, false, true)
    GS_WALK_CASE(10, false, true, false, true)
    GS_WALK_CASE(11, true, true, false, true)
    GS_WALK_CASE(12, false, false, true, true)
    GS_WALK_CASE(13, true, false, true, true)
    GS_WALK_CASE(14, false, true, true, true)
    GS_WALK_CASE(15, true, true, true, true)
#undef GS_WALK_CASE
  }
}

void enqueue_walk(gs_ctx* c, int sf) {
  WalkArgs a;
  a.pin = c->part[c->cur];
  a.pout = c->part[c->cur ^ 1];
  a.stellar = c->stel[c->scur];
  a.cm = c->cm;
  a.info = c->info;
  a.st = c->st;
  a.energy = c->energy;
  a.dbg_acc = c->dbg_acc;
  a.dbg_dens = c->dbg_dens;
  a.partials = c->partials;
  a.work = c->walk_work;
  a.L = c->lay;
  a.pool_n = (uint32_t)c->plan.cap;
  a.node_pool = (uint32_t)c->plan.nodes;
  const uint32_t g = c->walk_grid;
  cudaStream_t s = c->stream;
  const bool one = c->lay.nseg == 1;
  if (one) a.seg0 = c->seg_host[0];
  else memset(&a.seg0, 0, sizeof(a.seg0));
  a.meta = c->meta;
  a.split_buf = c->split_buf;
  a.split_arrive = c->split_arrive;
  a.split_stride = one ? a.seg0.n : 0u;
  const int v = (sf ? 1 : 0) | (c->debug ? 2 : 0) | (one ? 4 : 0) | (c->walk_comp ? 8 : 0);
  // one launch per walk group size present (a single galaxy: its own); 8 blocks
  // per SM: the 64-register build, fewer: the 72-register build (groups of 32)
  for (int k = 0; k < 4; k++) {
    if (!c->walk_items[k]) continue;
    const uint32_t gk = std::min<uint32_t>(g, std::max<uint32_t>(1, cdiv(c->walk_items[k], kWalkWarps)));
    if (k == 1) launch_walk<kWalkBlocksPerSM, 2>(v, gk, s, a);
    else if (k == 2) launch_walk<kWalkBlocksPerSM, 4>(v, gk, s, a);
    else if (k == 3) launch_walk<kWalkBlocksPerSM, 8>(v, gk, s, a);
    else if (c->walk_bps >= kWalkBlocksPerSM) launch_walk<kWalkBlocksPerSM, 1>(v, gk, s, a);
    else launch_walk<kWalkBlocksWide, 1>(v, gk, s, a);
  }
  // per-galaxy FP64 diagnostics of this walk
  launch_pdl(diag_reduce_kernel, c->lay.diag_chunks, 32 * kPartials, s, (const double*)c->partials, c->lay,
             c->diag_chunk, c->diag_ctr, c->diag_out);
  c->cur ^= 1;
}

// codes + sort + gather (+ tracking/EMA) + build + refresh; flips cur and scur.
void enqueue_sort_build(gs_ctx* c, int advance_time) {
  const bool track = c->any_tracking();
  const Layout& L = c->lay;
  enqueue_codes_sort(c, c->part[c->cur], 2, advance_time);
  enqueue_sort_passes(c, track);
  launch_pdl(gather_kernel, L.flag_tiles, kTileThreads, c->stream, (const uint32_t*)c->vals[0],
             (const float4*)c->part[c->cur], c->part[c->cur ^ 1], (const float4*)c->stel[c->scur],
             c->stel[c->scur ^ 1], L, c->st);
  c->cur ^= 1;
  c->scur ^= 1;
  if (track)
    launch_pdl(track_kernel, cdiv(L.nseg, 128), 128, c->stream, (const uint32_t*)c->inv,
               (const float4*)c->part[c->cur], L, c->st);
  enqueue_build(c, c->part[c->cur], 2, c->com_mode, 0.0, c->frames);
}

// After a Params upload: sim_time follows Params.time, N is the galaxy's, and
// tracked halo centres keep their device-side smoothed values.
__global__ void params_fixup_kernel(DevState* st, uint32_t N) {
  st->p.N = N;
  st->sim_time = (double)st->p.time;
  for (int h = 0; h < 2; h++) {
    if (st->central[h] < 0) continue;
    float* dst = h == 0 ? st->p.haloC1 : st->p.haloC2;
    for (int k = 0; k < 3; k++) dst[k] = __double2float_rn(st->halo_c[h][k]);
  }
}

// c0/c1: pool indices or -1.
__global__ void tracking_init_kernel(DevState* st, const float4* P, long long c0, long long c1,
                                     int have0, double h0x, double h0y, double h0z, int have1,
                                     double h1x, double h1y, double h1z) {
  const long long c[2] = {c0, c1};
  const int have[2] = {have0, have1};
  const double hv[2][3] = {{h0x, h0y, h0z}, {h1x, h1y, h1z}};
  for (int h = 0; h < 2; h++) {
    st->central[h] = c[h];
    if (have[h]) {
      for (int k = 0; k < 3; k++) st->halo_c[h][k] = hv[h][k];
    } else if (c[h] >= 0) {
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

// applyPermutation of one galaxy (pointers at its offset; perm galaxy-local and
// checked on the host): out[i] = in[perm[i]] (nbody_bh.wgsl:322-326, :336-340).
__global__ void gather_range_kernel(const uint32_t* __restrict__ perm, const float4* __restrict__ pin,
                                    float4* __restrict__ pout, const float4* __restrict__ sin,
                                    float4* __restrict__ sout, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t s = perm[i];
    if (s >= n) continue;
    pout[2 * (size_t)i] = pin[2 * (size_t)s];
    pout[2 * (size_t)i + 1] = pin[2 * (size_t)s + 1];
    sout[i] = sin[s];
  }
}

int wait_stream(gs_ctx* c, uint64_t timeout_ns, const Slot* s) {
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
  // error words: the given slot's, or every live slot's (one strided copy)
  unsigned err = 0;
  if (s) {
    const size_t k = (size_t)(s - c->slots.data());
    CK(c, cudaMemcpy(&err, &c->st[k].err, sizeof(unsigned), cudaMemcpyDeviceToHost), "read error word");
  } else if (!c->slots.empty()) {
    std::vector<unsigned> words(c->slots.size());
    CK(c, cudaMemcpy2D(words.data(), sizeof(unsigned), &c->st[0].err, sizeof(DevState), sizeof(unsigned),
                       c->slots.size(), cudaMemcpyDeviceToHost),
       "read error words");
    for (size_t k = 0; k < words.size(); k++)
      if (c->slots[k].live) err |= words[k];
  }
  if (err)
    return c->fail(GS_EDEVICE, "device error word 0x%x (%s%s%s%s)", err,
                   err & GS_DERR_LOOKBACK ? "sort look-back wait limit " : "",
                   err & GS_DERR_STACK ? "walk stack " : "", err & GS_DERR_NODES ? "node pool " : "",
                   err & GS_DERR_TREE ? "uploaded tree not BFS-contiguous" : "");
  return GS_OK;
}

int stage_grow(gs_ctx* c, uint32_t need_nodes) {
  if (c->bh && c->max_bh >= need_nodes) return GS_OK;
  gs_node* p = nullptr;
  CK(c, c->alloc(&p, std::max<uint32_t>(need_nodes, 1)), "bh staging");
  c->bh = p;  // the old staging stays owned until the context is destroyed
  c->max_bh = need_nodes;
  return GS_OK;
}

// Put a galaxy into slot `slot` at pool offset off (both ping-pongs written).
int slot_fill(gs_ctx* c, uint32_t slot, uint32_t off, uint32_t span, uint32_t n, uint32_t node_cap,
              const float* particles8, const float* stellar4, const gs_params* params) {
  Slot& s = c->slots[slot];
  CK(c, cudaStreamSynchronize(c->stream), "sync");
  const size_t pb = (size_t)n * 32, sb = (size_t)n * 16;
  for (int k = 0; k < 2; k++) {
    CK(c, cudaMemcpy(c->part[k] + 2 * (size_t)off, particles8, pb, cudaMemcpyHostToDevice), "upload");
    if (stellar4)
      CK(c, cudaMemcpy(c->stel[k] + off, stellar4, sb, cudaMemcpyHostToDevice), "upload");
    else
      CK(c, cudaMemset(c->stel[k] + off, 0, sb), "memset");
  }
  CK(c, cudaMemset(c->cm + 2 * (size_t)off, 0, sizeof(float4) * node_cap), "memset");
  CK(c, cudaMemset(c->info + 2 * (size_t)off, 0, sizeof(WalkInfo) * node_cap), "memset");
  CK(c, cudaMemset(c->meta + slot, 0, sizeof(TreeMeta)), "memset");
  CK(c, cudaMemset(c->diag_out + (size_t)slot * kPartials, 0, sizeof(double) * kPartials), "memset");
  DevState st0;
  memset(&st0, 0, sizeof(st0));
  if (params) st0.p = *params;
  st0.p.N = n;
  st0.sim_time = (double)st0.p.time;
  st0.central[0] = st0.central[1] = -1;
  CK(c, cudaMemcpy(c->st + slot, &st0, sizeof(st0), cudaMemcpyHostToDevice), "state");
  s = Slot();
  s.live = true;
  s.off = off;
  s.span = span;
  s.n = n;
  s.node_off = 2 * off;
  s.node_cap = node_cap;
  s.hp = st0.p;
  c->lay_dirty = true;
  return GS_OK;
}

int host_pack4(const float* src, uint32_t N, uint32_t stride, std::vector<float4>& out) {
  out.resize(N);
  for (uint32_t i = 0; i < N; i++)
    out[i] = make_float4(src[(size_t)i * stride], src[(size_t)i * stride + 1],
                         src[(size_t)i * stride + 2], stride >= 4 ? src[(size_t)i * stride + 3] : 0.f);
  return GS_OK;
}

}  // namespace

// Context-free error text for entry points defined in other translation units.
void gs_internal_set_error(const char* msg) { set_err(g_err, "%s", msg); }

extern "C" {

const char* gs_last_error(const gs_ctx* ctx) { return ctx ? ctx->err : g_err; }

const char* gs_version(void) { return "galaxy_b200 0.2 (sm_100a)"; }

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

// ---- pools ---------------------------------------------------------------------------

int gs_device_memory(int device, uint64_t* free_bytes, uint64_t* total_bytes) {
  int prev = 0;
  cudaGetDevice(&prev);
  cudaError_t e = cudaSetDevice(device);
  size_t f = 0, t = 0;
  if (e == cudaSuccess) e = cudaMemGetInfo(&f, &t);
  cudaSetDevice(prev);
  if (e != cudaSuccess) {
    set_err(g_err, "cudaMemGetInfo: %s", cudaGetErrorString(e));
    return GS_ECUDA;
  }
  if (free_bytes) *free_bytes = f;
  if (total_bytes) *total_bytes = t;
  return GS_OK;
}

uint64_t gs_pool_bytes(uint64_t particle_capacity, uint32_t max_galaxies) {
  return plan_bytes(make_plan(particle_capacity, max_galaxies));
}

int gs_pool_create(int device, uint64_t particle_capacity, uint32_t max_galaxies, gs_ctx** out) {
  if (!out) {
    set_err(g_err, "out is NULL");
    return GS_EINVAL;
  }
  *out = nullptr;
  if (particle_capacity == 0 || particle_capacity > kMaxPool || max_galaxies == 0 ||
      max_galaxies > kMaxSlots) {
    set_err(g_err, "pool capacity must be in [1, %llu] particles and [1, %u] galaxies",
            (unsigned long long)kMaxPool, kMaxSlots);
    return GS_EINVAL;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    set_err(g_err, "no CUDA device %d (have %d)", device, ndev);
    return GS_EINVAL;
  }
  gs_ctx* c = new (std::nothrow) gs_ctx();
  if (!c) return GS_ENOMEM;
  const int rc = pool_init(c, device, particle_capacity, max_galaxies);
  if (rc) {
    set_err(g_err, "%s", c->err);
    gs_destroy(c);
    return rc;
  }
  *out = c;
  return GS_OK;
}

int gs_pool_add(gs_ctx* ctx, uint32_t N, const float* particles8, const float* stellar4,
                const gs_params* params, uint32_t* slot_out) {
  CTX_CHECK(ctx);
  if (N == 0 || !particles8) return ctx->fail(GS_EINVAL, "N must be >= 1 and particles8 set");
  if (ctx->single) return ctx->fail(GS_EINVAL, "a single-galaxy context takes no more galaxies");
  uint32_t slot = 0;
  while (slot < ctx->slots.size() && ctx->slots[slot].live) slot++;
  if (slot == ctx->slots.size()) return ctx->fail(GS_ENOMEM, "no free galaxy slot");
  const uint64_t span = (uint64_t)cdiv(N, kAlign) * kAlign;
  uint64_t off = 0;
  if (!ctx->palloc.alloc(span, &off))
    return ctx->fail(GS_ENOMEM, "no free particle range of %llu in the pool", (unsigned long long)span);
  int rc = slot_fill(ctx, slot, (uint32_t)off, (uint32_t)span, N, 2 * N, particles8, stellar4, params);
  if (rc) {
    ctx->palloc.release(off, span);
    ctx->slots[slot].live = false;
    return rc;
  }
  if (slot_out) *slot_out = slot;
  return GS_OK;
}

int gs_pool_remove(gs_ctx* ctx, uint32_t slot) {
  CTX_CHECK(ctx);
  if (slot >= ctx->slots.size() || !ctx->slots[slot].live)
    return ctx->fail(GS_EINVAL, "slot %u holds no galaxy", slot);
  CK(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  Slot& s = ctx->slots[slot];
  ctx->palloc.release(s.off, s.span);
  s = Slot();
  ctx->lay_dirty = true;
  return GS_OK;
}

int gs_pool_free(gs_ctx* ctx, uint64_t* largest_range, uint32_t* free_slots) {
  CTX_CHECK(ctx);
  if (largest_range) *largest_range = ctx->palloc.largest();
  if (free_slots) {
    uint32_t f = 0;
    for (const Slot& s : ctx->slots) f += s.live ? 0 : 1;
    *free_slots = f;
  }
  return GS_OK;
}

int gs_select(gs_ctx* ctx, uint32_t slot) {
  CTX_CHECK(ctx);
  if (slot >= ctx->slots.size()) return ctx->fail(GS_EINVAL, "slot %u out of range", slot);
  ctx->sel = slot;
  return GS_OK;
}

int gs_pool_energies(gs_ctx* ctx, gs_diag* out, uint32_t cap) {
  CTX_CHECK(ctx);
  if (!out) return ctx->fail(GS_EINVAL, "out is NULL");
  const uint32_t n = std::min<uint32_t>(cap, (uint32_t)ctx->slots.size());
  std::vector<double> h((size_t)n * kPartials);
  if (n)
    CK(ctx, cudaMemcpyAsync(h.data(), ctx->diag_out, sizeof(double) * h.size(), cudaMemcpyDeviceToHost,
                            ctx->stream),
       "diag");
  int rc = wait_stream(ctx, 0, nullptr);
  if (rc) return rc;
  for (uint32_t k = 0; k < n; k++) {
    const double* v = &h[(size_t)k * kPartials];
    if (!ctx->slots[k].live) {
      memset(&out[k], 0, sizeof(gs_diag));
      continue;
    }
    out[k].e_diag = v[0];
    out[k].e_true = v[1];
    out[k].momentum[0] = v[2];
    out[k].momentum[1] = v[3];
    out[k].momentum[2] = v[4];
    out[k].mass = v[5];
  }
  return GS_OK;
}

// ---- NBodyGPU surface ------------------------------------------------------------------

int gs_create_on(int device, uint32_t N, const float* particles8, const float* stellar4,
                 gs_ctx** out) {
  if (!out) {
    set_err(g_err, "out is NULL");
    return GS_EINVAL;
  }
  *out = nullptr;
  if (N == 0 || N > kMaxPool) {
    set_err(g_err, "N must be in [1, %llu], got %u", (unsigned long long)kMaxPool, N);
    return GS_EINVAL;
  }
  if (!particles8) {
    set_err(g_err, "particles8 is NULL");
    return GS_EINVAL;
  }
  int rc = gs_pool_create(device, N, 1, out);
  if (rc) return rc;
  gs_ctx* c = *out;
  rc = slot_fill(c, 0, 0, N, N, 2 * N + 4096, particles8, stellar4, nullptr);
  if (rc) {
    set_err(g_err, "%s", c->err);
    gs_destroy(c);
    *out = nullptr;
    return rc;
  }
  c->palloc.init(0);
  c->single = true;
  c->walk_bps = kWalkBlocksWide;  // one galaxy: the 72-register walk measured faster
  c->walk_group = 0;              // one galaxy: walk groups by its size (a pool fills the GPU with 32s)
  c->walk_split = 0;              // and walk splits by its size
  c->sort_items = 0;              // and sort tiles by its size
  return GS_OK;
}

int gs_create(uint32_t N, const float* particles8, const float* stellar4, gs_ctx** out) {
  int dev = 0;
  cudaGetDevice(&dev);
  return gs_create_on(dev, N, particles8, stellar4, out);
}

int gs_destroy(gs_ctx* ctx) {
  if (!ctx) return GS_OK;
  pool_release(ctx);
  delete ctx;
  return GS_OK;
}

int gs_update_params(gs_ctx* ctx, const gs_params* params) {
  CTX_CHECK(ctx);
  SLOT(ctx, s);
  if (!params) return ctx->fail(GS_EINVAL, "params is NULL");
  s->hp = *params;
  s->hp.N = s->n;
  // the 96-byte uniform goes through a pinned ring entry, so the async copy never
  // reads the caller's buffer after return and the entry is free once its last
  // copy has run
  const int e = ctx->param_next;
  ctx->param_next = (e + 1) % gs_ctx::kParamRing;
  if (ctx->param_used[e]) CK(ctx, cudaEventSynchronize(ctx->param_ev[e]), "params stage");
  gs_params* stage = reinterpret_cast<gs_params*>(ctx->host_stage) + e;
  *stage = s->hp;
  DevState* st = ctx->st + ctx->sel;
  CK(ctx, cudaMemcpyAsync(&st->p, stage, sizeof(gs_params), cudaMemcpyHostToDevice, ctx->stream),
     "params upload");
  CK(ctx, cudaEventRecord(ctx->param_ev[e], ctx->stream), "params event");
  ctx->param_used[e] = true;
  params_fixup_kernel<<<1, 1, 0, ctx->stream>>>(st, s->n);
  CK(ctx, cudaGetLastError(), "params fixup");
  return GS_OK;
}

int gs_set_time(gs_ctx* ctx, double t) {
  CTX_CHECK(ctx);
  SLOT(ctx, s);
  (void)s;
  CK(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  CK(ctx, cudaMemcpy(&ctx->st[ctx->sel].sim_time, &t, sizeof(double), cudaMemcpyHostToDevice), "time");
  return GS_OK;
}

int gs_set_star_formation(gs_ctx* ctx, int enable) {
  CTX_CHECK(ctx);
  SLOT(ctx, s);
  (void)s;
  CK(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  const unsigned off = enable ? 0u : 1u;
  CK(ctx, cudaMemcpy(&ctx->st[ctx->sel].sf_off, &off, sizeof(off), cudaMemcpyHostToDevice), "sf flag");
  return GS_OK;
}

int gs_update_central_mass(gs_ctx* ctx, float mass, uint32_t idx) {
  CTX_CHECK(ctx);
  SLOT(ctx, s);
  if (idx >= s->n) return ctx->fail(GS_EINVAL, "central index %u >= N %u", idx, s->n);
  CK(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  for (int k = 0; k < 2; k++)
    CK(ctx, cudaMemcpy(reinterpret_cast<char*>(ctx->part[k]) + ((size_t)s->off + idx) * 32 + 12, &mass, 4,
                       cudaMemcpyHostToDevice),
       "central mass");
  return GS_OK;
}

int gs_apply_permutation(gs_ctx* ctx, const uint32_t* perm) {
  CTX_CHECK(ctx);
  SLOT(ctx, s);
  if (!perm) return ctx->fail(GS_EINVAL, "perm is NULL");
  for (uint32_t i = 0; i < s->n; i++)
    if (perm[i] >= s->n) return ctx->fail(GS_EINVAL, "perm[%u] = %u out of range", i, perm[i]);
  CK(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  CK(ctx, cudaMemcpyAsync(ctx->perm_user + s->off, perm, sizeof(uint32_t) * s->n, cudaMemcpyHostToDevice,
                          ctx->stream),
     "perm upload");
  const int c0 = ctx->cur, s0 = ctx->scur;
  gather_range_kernel<<<grid_for(s->n, 256, 148 * 16), 256, 0, ctx->stream>>>(
      ctx->perm_user + s->off, ctx->part[c0] + 2 * (size_t)s->off, ctx->part[c0 ^ 1] + 2 * (size_t)s->off,
      ctx->stel[s0] + s->off, ctx->stel[s0 ^ 1] + s->off, s->n);
  CK(ctx, cudaGetLastError(), "gather");
  int live = 0;
  for (const Slot& q : ctx->slots) live += q.live ? 1 : 0;
  if (live == 1) {
    ctx->cur ^= 1;  // NBodyGPU.js:328 flips the ping-pongs
    ctx->scur ^= 1;
  } else {  // other galaxies share the buffers: copy the result back instead
    CK(ctx, cudaMemcpyAsync(ctx->part[c0] + 2 * (size_t)s->off, ctx->part[c0 ^ 1] + 2 * (size_t)s->off,
                            (size_t)s->n * 32, cudaMemcpyDeviceToDevice, ctx->stream),
       "copy back");
    CK(ctx, cudaMemcpyAsync(ctx->stel[s0] + s->off, ctx->stel[s0 ^ 1] + s->off, (size_t)s->n * 16,
                            cudaMemcpyDeviceToDevice, ctx->stream),
       "copy back");
  }
  CK(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  return GS_OK;
}

int gs_upload_tree(gs_ctx* ctx, const gs_node* nodes, uint32_t num_nodes,
                   const uint32_t* level_ranges, uint32_t n_levels) {
  CTX_CHECK(ctx);
  SLOT(ctx, s);
  if (!nodes && num_nodes) return ctx->fail(GS_EINVAL, "nodes is NULL");
  const uint32_t max_bh = 4 * s->n + 1024;  // NBodyGPU.js:58
  const uint32_t n = std::min(num_nodes, max_bh);
  if (n > s->node_cap)
    return ctx->fail(GS_EINVAL, "tree of %u nodes exceeds the galaxy's pool of %u", n, s->node_cap);
  int rc = stage_grow(ctx, n);
  if (rc) return rc;
  CK(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  if (n) CK(ctx, cudaMemcpy(ctx->bh, nodes, (size_t)n * sizeof(gs_node), cudaMemcpyHostToDevice), "tree");
  // the build's leaves pass skips this galaxy until its next on-device build
  CK(ctx, cudaMemsetAsync(ctx->meta + ctx->sel, 0, sizeof(TreeMeta), ctx->stream), "meta");
  if (n)
    upload_convert_kernel<<<grid_for(n, 256, 148 * 8), 256, 0, ctx->stream>>>(
        ctx->bh, n, s->n, s->node_off, s->off, ctx->cm, ctx->info, ctx->st + ctx->sel);
  CK(ctx, cudaGetLastError(), "convert");
  s->up_lr.clear();
  if (level_ranges) s->up_lr.assign(level_ranges, level_ranges + 2 * std::min<uint32_t>(n_levels, 16));
  s->up_nodes = n;
  s->up_host.assign(nodes, nodes + n);
  s->tree = Slot::kTreeUploaded;
  return wait_stream(ctx, 0, s);
}

int gs_refresh(gs_ctx* ctx) {
  CTX_CHECK(ctx);
  int rc = ensure_layout(ctx);
  if (rc) return rc;
  bool built = false;
  for (Slot& s : ctx->slots) {
    if (!s.live) continue;
    if (s.tree == Slot::kTreeBuilt) built = true;
    if (s.tree != Slot::kTreeUploaded) continue;
    // NBodyGPU.js:309: no-op without levelRanges; deepest level first
    for (int64_t l = (int64_t)s.up_lr.size() / 2 - 1; l >= 0; l--) {
      const uint32_t start = s.up_lr[2 * l], count = s.up_lr[2 * l + 1];
      if (!count) continue;
      if ((uint64_t)start + count > s.up_nodes)
        return ctx->fail(GS_EINVAL, "level %lld [%u, +%u) beyond %u nodes", (long long)l, start, count,
                         s.up_nodes);
      refresh_level_kernel<<<cdiv(count, 64), 64, 0, ctx->stream>>>(ctx->part[ctx->cur], ctx->cm, ctx->info,
                                                                     s.node_off + start, count);
    }
  }
  if (built && ctx->lay.nseg) {
    BuildBuffers b = ctx->bb();
    const Layout& L = ctx->lay;
    if (ctx->com_mode == kComF64)
      tree_leaves_kernel<kComF64><<<L.flag_tiles, kLeafThreads, 0, ctx->stream>>>(b, L, ctx->part[ctx->cur], 2,
                                                                                   ctx->st);
    else
      tree_leaves_kernel<kComF32><<<L.flag_tiles, kLeafThreads, 0, ctx->stream>>>(b, L, ctx->part[ctx->cur], 2,
                                                                                   ctx->st);
  }
  CK(ctx, cudaGetLastError(), "refresh");
  return GS_OK;
}

int gs_step(gs_ctx* ctx) {
  CTX_CHECK(ctx);
  int rc = ensure_layout(ctx);
  if (rc) return rc;
  if (!ctx->lay.nseg) return GS_OK;
  enqueue_walk(ctx, 0);
  CK(ctx, cudaGetLastError(), "walk");
  return GS_OK;
}

int gs_star_formation(gs_ctx* ctx) {
  CTX_CHECK(ctx);
  int rc = ensure_layout(ctx);
  if (rc) return rc;
  if (!ctx->lay.nseg) return GS_OK;
  sf_kernel<<<ctx->lay.flag_tiles, kTileThreads, 0, ctx->stream>>>(ctx->part[ctx->cur], ctx->stel[ctx->scur],
                                                                    ctx->lay, ctx->st);
  CK(ctx, cudaGetLastError(), "star formation");
  return GS_OK;
}

int gs_read_positions(gs_ctx* ctx, float* out4, uint64_t timeout_ns) {
  CTX_CHECK(ctx);
  SLOT(ctx, s);
  if (!out4) return ctx->fail(GS_EINVAL, "out4 is NULL");
  // an asynchronous readback still copying out of the compaction buffer finishes first
  if (ctx->rb_pending) CK(ctx, cudaStreamWaitEvent(ctx->stream, ctx->rb_done, 0), "readback order");
  compact_kernel<<<grid_for(s->n, 256, 148 * 16), 256, 0, ctx->stream>>>(
      ctx->part[ctx->cur] + 2 * (size_t)s->off, ctx->energy + s->off, ctx->compact + s->off, s->n);
  CK(ctx, cudaGetLastError(), "compact");
  int rc = wait_stream(ctx, timeout_ns, s);
  if (rc) return rc;
  CK(ctx, cudaMemcpy(out4, ctx->compact + s->off, (size_t)s->n * 16, cudaMemcpyDeviceToHost), "readback");
  return GS_OK;
}

int gs_encode_position_readback(gs_ctx* ctx, float* out4, gs_diag* diag) {
  CTX_CHECK(ctx);
  SLOT(ctx, s);
  if (!out4) return ctx->fail(GS_EINVAL, "out4 is NULL");
  if (ctx->rb_pending)
    return ctx->fail(GS_ENOTREADY, "a position readback is in flight: await it before encoding another");
  if (!ctx->rb_stream) {  // first use: copy stream, events, mapped pinned words
    CK(ctx, cudaStreamCreateWithFlags(&ctx->rb_stream, cudaStreamNonBlocking), "readback stream");
    CK(ctx, cudaEventCreateWithFlags(&ctx->rb_ready, cudaEventDisableTiming), "readback event");
    CK(ctx, cudaEventCreateWithFlags(&ctx->rb_done, cudaEventDisableTiming), "readback event");
    void* h = nullptr;
    CK(ctx, cudaHostAlloc(&h, (kPartials + 1) * sizeof(double), cudaHostAllocMapped), "readback words");
    ctx->rb_host = static_cast<double*>(h);
    void* d = nullptr;
    CK(ctx, cudaHostGetDevicePointer(&d, h, 0), "readback words");
    ctx->rb_host_dev = static_cast<double*>(d);
  }
  // in stream order: vec4(pos, e_i) into the compaction buffer and the diagnostics
  // snapshot; the copy stream then moves the positions while later steps run
  compact_kernel<<<grid_for(s->n, 256, 148 * 16), 256, 0, ctx->stream>>>(
      ctx->part[ctx->cur] + 2 * (size_t)s->off, ctx->energy + s->off, ctx->compact + s->off, s->n);
  CK(ctx, cudaGetLastError(), "compact");
  readback_snapshot_kernel<<<1, 32, 0, ctx->stream>>>(ctx->diag_out + (size_t)ctx->sel * kPartials,
                                                      &ctx->st[ctx->sel].err, ctx->rb_host_dev);
  CK(ctx, cudaGetLastError(), "readback snapshot");
  CK(ctx, cudaEventRecord(ctx->rb_ready, ctx->stream), "readback event");
  CK(ctx, cudaStreamWaitEvent(ctx->rb_stream, ctx->rb_ready, 0), "readback order");
  CK(ctx, cudaMemcpyAsync(out4, ctx->compact + s->off, (size_t)s->n * 16, cudaMemcpyDeviceToHost, ctx->rb_stream),
     "readback copy");
  CK(ctx, cudaEventRecord(ctx->rb_done, ctx->rb_stream), "readback event");
  ctx->rb_diag = diag;
  ctx->rb_slot = ctx->sel;
  ctx->rb_pending = true;
  return GS_OK;
}

int gs_await_position_readback(gs_ctx* ctx, uint64_t timeout_ns) {
  CTX_CHECK(ctx);
  if (!ctx->rb_pending) return ctx->fail(GS_EINVAL, "no position readback in flight");
  if (timeout_ns == 0) {
    CK(ctx, cudaEventSynchronize(ctx->rb_done), "readback wait");
  } else {
    const auto t0 = std::chrono::steady_clock::now();
    while (true) {
      cudaError_t q = cudaEventQuery(ctx->rb_done);
      if (q == cudaSuccess) break;
      if (q != cudaErrorNotReady) return ctx->cuda(q, "readback wait");
      const auto dt =
          std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count();
      if ((uint64_t)dt > timeout_ns)  // still in flight: a later await can collect it
        return ctx->fail(GS_ETIMEDOUT, "position readback did not land within %llu ns",
                         (unsigned long long)timeout_ns);
      std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
  }
  ctx->rb_pending = false;
  if (ctx->rb_diag) {
    const double* h = ctx->rb_host;
    ctx->rb_diag->e_diag = h[0];
    ctx->rb_diag->e_true = h[1];
    ctx->rb_diag->momentum[0] = h[2];
    ctx->rb_diag->momentum[1] = h[3];
    ctx->rb_diag->momentum[2] = h[4];
    ctx->rb_diag->mass = h[5];
  }
  const unsigned err = reinterpret_cast<const unsigned*>(ctx->rb_host + kPartials)[0];
  if (err)
    return ctx->fail(GS_EDEVICE, "device error word 0x%x of slot %u at the readback", err, ctx->rb_slot);
  return GS_OK;
}

int gs_position_buffer(gs_ctx* ctx, void** dptr) {
  CTX_CHECK(ctx);
  SLOT(ctx, s);
  if (!dptr) return ctx->fail(GS_EINVAL, "dptr is NULL");
  *dptr = ctx->part[ctx->cur] + 2 * (size_t)s->off;
  return GS_OK;
}

int gs_stellar_buffer(gs_ctx* ctx, void** dptr) {
  CTX_CHECK(ctx);
  SLOT(ctx, s);
  if (!dptr) return ctx->fail(GS_EINVAL, "dptr is NULL");
  *dptr = ctx->stel[ctx->scur] + s->off;
  return GS_OK;
}

int gs_set_tracking(gs_ctx* ctx, int64_t c1, int64_t c2, const double* h1, const double* h2) {
  CTX_CHECK(ctx);
  SLOT(ctx, s);
  if (c1 >= (int64_t)s->n || c2 >= (int64_t)s->n) return ctx->fail(GS_EINVAL, "tracked index out of range");
  const bool was = ctx->any_tracking();
  s->tracking = c1 >= 0 || c2 >= 0;
  tracking_init_kernel<<<1, 1, 0, ctx->stream>>>(
      ctx->st + ctx->sel, ctx->part[ctx->cur], c1 < 0 ? -1 : s->off + c1, c2 < 0 ? -1 : s->off + c2,
      h1 != nullptr, h1 ? h1[0] : 0, h1 ? h1[1] : 0, h1 ? h1[2] : 0, h2 != nullptr, h2 ? h2[0] : 0,
      h2 ? h2[1] : 0, h2 ? h2[2] : 0);
  CK(ctx, cudaGetLastError(), "tracking");
  if (was != ctx->any_tracking()) ctx->drop_graphs();
  return wait_stream(ctx, 0, s);
}

int gs_get_tracking(gs_ctx* ctx, int64_t* c1, int64_t* c2, double* h1, double* h2) {
  CTX_CHECK(ctx);
  SLOT(ctx, s);
  int rc = wait_stream(ctx, 0, s);
  if (rc) return rc;
  DevState d;
  CK(ctx, cudaMemcpy(&d, ctx->st + ctx->sel, sizeof(d), cudaMemcpyDeviceToHost), "state");
  if (c1) *c1 = d.central[0] < 0 ? -1 : d.central[0] - s->off;
  if (c2) *c2 = d.central[1] < 0 ? -1 : d.central[1] - s->off;
  if (h1) memcpy(h1, d.halo_c[0], 3 * sizeof(double));
  if (h2) memcpy(h2, d.halo_c[1], 3 * sizeof(double));
  return GS_OK;
}

int gs_sort_build(gs_ctx* ctx) {
  CTX_CHECK(ctx);
  int rc = ensure_layout(ctx);
  if (rc) return rc;
  if (!ctx->lay.nseg) return GS_OK;
  enqueue_sort_build(ctx, 0);
  CK(ctx, cudaGetLastError(), "sort/build");
  for (Slot& s : ctx->slots)
    if (s.live) s.tree = Slot::kTreeBuilt;
  return GS_OK;
}

int gs_set_com_mode(gs_ctx* ctx, int mode) {
  CTX_CHECK(ctx);
  if (mode != kComF32 && mode != kComF64) return ctx->fail(GS_EINVAL, "COM mode %d", mode);
  ctx->com_mode = mode;
  ctx->drop_graphs();
  return GS_OK;
}

int gs_set_tuning(gs_ctx* ctx, int knob, int value) {
  CTX_CHECK(ctx);
  if (knob == GS_TUNE_WALK_BLOCKS_PER_SM) {
    if (value < 1 || value > kWalkBlocksPerSM)
      return ctx->fail(GS_EINVAL, "walk blocks per SM must be in [1, %d]", kWalkBlocksPerSM);
    ctx->walk_bps = value;
  } else if (knob == GS_TUNE_SORT_ITEMS) {
    if (value != 0 && value != 4 && value != 8 && value != 16)
      return ctx->fail(GS_EINVAL, "sort keys per thread must be 0 (by galaxy size), 4, 8 or 16");
    ctx->sort_items = value;
  } else if (knob == GS_TUNE_WALK_GROUP) {
    if (value != 0 && value != 4 && value != 8 && value != 16 && value != 32)
      return ctx->fail(GS_EINVAL, "walk group must be 0 (by galaxy size), 4, 8, 16 or 32 particles");
    ctx->walk_group = value;
  } else if (knob == GS_TUNE_WALK_SPLIT) {
    if (value != 0 && value != 1 && value != 2 && value != 4 && value != 8)
      return ctx->fail(GS_EINVAL, "walk split must be 0 (by galaxy size), 1, 2, 4 or 8");
    ctx->walk_split = value;
  } else {
    return ctx->fail(GS_EINVAL, "unknown tuning knob %d", knob);
  }
  CK(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  ctx->lay_dirty = true;  // tiles and grid follow at the next step
  ctx->drop_graphs();
  return GS_OK;
}

int gs_get_tuning(gs_ctx* ctx, int knob, int* value) {
  CTX_CHECK(ctx);
  if (!value) return ctx->fail(GS_EINVAL, "value is NULL");
  if (knob == GS_TUNE_WALK_BLOCKS_PER_SM) *value = ctx->walk_bps;
  else if (knob == GS_TUNE_SORT_ITEMS) *value = ctx->sort_items;
  else if (knob == GS_TUNE_WALK_GROUP) *value = ctx->walk_group;
  else if (knob == GS_TUNE_WALK_SPLIT) *value = ctx->walk_split;
  else return ctx->fail(GS_EINVAL, "unknown tuning knob %d", knob);
  return GS_OK;
}

int gs_get_launch_setting(gs_ctx* ctx, uint32_t* group, uint32_t* split, uint32_t* sort_items) {
  CTX_CHECK(ctx);
  SLOT(ctx, s);
  int rc = ensure_layout(ctx);
  if (rc) return rc;
  const SegDesc& d = ctx->seg_host[s->rank];
  if (group) *group = kWalkGroup / d.wlpp;
  if (split) *split = d.wsplit;
  if (sort_items) *sort_items = (uint32_t)ctx->sort_eff;
  return GS_OK;
}

int gs_set_walk_mode(gs_ctx* ctx, int compensated) {
  CTX_CHECK(ctx);
  if (compensated != 0 && compensated != 1) return ctx->fail(GS_EINVAL, "walk mode %d", compensated);
  ctx->walk_comp = compensated != 0;
  ctx->drop_graphs();
  return GS_OK;
}

int gs_run(gs_ctx* ctx, uint32_t nsteps, int do_sf) {
  CTX_CHECK(ctx);
  int rc = ensure_layout(ctx);
  if (rc) return rc;
  if (!ctx->lay.nseg) return GS_OK;
  for (uint32_t s = 0; s < nsteps; s++) {
    const int key = (ctx->cur) | (ctx->scur << 1) | ((do_sf ? 1 : 0) << 2) | ((ctx->debug ? 1 : 0) << 3) |
                    ((ctx->walk_comp ? 1 : 0) << 4);
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
      size_t nn = 0;
      if (cudaGraphGetNodes(g, nullptr, &nn) == cudaSuccess) {
        std::vector<cudaGraphNode_t> nodes(nn);
        uint32_t nk = 0;
        if (nn && cudaGraphGetNodes(g, nodes.data(), &nn) == cudaSuccess)
          for (cudaGraphNode_t n : nodes) {
            cudaGraphNodeType t;
            if (cudaGraphNodeGetType(n, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) nk++;
          }
        ctx->step_kernels = nk;
      }
      cudaGraphExec_t ge = nullptr;
      e = cudaGraphInstantiate(&ge, g, 0);
      cudaGraphDestroy(g);
      CK(ctx, e, "instantiate");
      it = ctx->graphs.emplace(key, ge).first;
    }
    CK(ctx, cudaGraphLaunch(it->second, ctx->stream), "graph launch");
    // a step gathers cur -> cur^1 then walks back: cur unchanged, stellar flipped
    ctx->scur ^= 1;
  }
  for (Slot& s : ctx->slots)
    if (s.live && nsteps) s.tree = Slot::kTreeBuilt;
  return GS_OK;
}

int gs_step_kernels(gs_ctx* ctx, uint32_t* n) {
  CTX_CHECK(ctx);
  if (!n) return ctx->fail(GS_EINVAL, "n is NULL");
  *n = ctx->step_kernels;
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
  return wait_stream(ctx, timeout_ns, nullptr);
}

int gs_get_tree(gs_ctx* ctx, gs_node* nodes, uint32_t nodes_cap, uint32_t* num_nodes,
                uint32_t* level_ranges, uint32_t lr_cap, uint32_t* n_levels, uint32_t* perm) {
  CTX_CHECK(ctx);
  SLOT(ctx, s);
  int rc = wait_stream(ctx, 0, s);
  if (rc) return rc;
  if (s->tree == Slot::kTreeNone) return ctx->fail(GS_ENOTREADY, "no tree yet");
  uint32_t nn = 0, nl = 0;
  std::vector<uint32_t> lr;
  if (s->tree == Slot::kTreeBuilt) {
    rc = ensure_layout(ctx);
    if (rc) return rc;
    TreeMeta m;
    CK(ctx, cudaMemcpy(&m, ctx->meta + ctx->sel, sizeof(m), cudaMemcpyDeviceToHost), "meta");
    nn = m.num_nodes;
    nl = m.num_levels;
    for (uint32_t l = 0; l < nl; l++) {
      lr.push_back(m.level_start[l]);
      lr.push_back(m.level_count[l]);
    }
    if (nodes && nn) {
      rc = stage_grow(ctx, nn);
      if (rc) return rc;
      tree_bhnode_kernel<<<grid_for(nn, 256, 148 * 8), 256, 0, ctx->stream>>>(ctx->bb(), ctx->lay, s->rank,
                                                                               ctx->bh);
      CK(ctx, cudaGetLastError(), "materialise");
    }
  } else {
    nn = s->up_nodes;
    nl = (uint32_t)s->up_lr.size() / 2;
    lr = s->up_lr;
    if (nodes && nn) {
      rc = stage_grow(ctx, nn);
      if (rc) return rc;
      CK(ctx, cudaMemcpyAsync(ctx->bh, s->up_host.data(), sizeof(gs_node) * nn, cudaMemcpyHostToDevice,
                              ctx->stream),
         "tree");
      bh_patch_kernel<<<grid_for(nn, 256, 148 * 8), 256, 0, ctx->stream>>>(ctx->bh, ctx->cm + s->node_off, nn);
      CK(ctx, cudaGetLastError(), "patch");
    }
  }
  if (num_nodes) *num_nodes = nn;
  if (n_levels) *n_levels = nl;
  if (level_ranges)
    memcpy(level_ranges, lr.data(), sizeof(uint32_t) * std::min<size_t>(lr.size(), 2 * (size_t)lr_cap));
  if (nodes && nn)
    CK(ctx, cudaMemcpyAsync(nodes, ctx->bh, sizeof(gs_node) * std::min(nn, nodes_cap), cudaMemcpyDeviceToHost,
                            ctx->stream),
       "nodes");
  if (perm)
    CK(ctx, cudaMemcpyAsync(perm, ctx->vals[0] + s->off, sizeof(uint32_t) * s->n, cudaMemcpyDeviceToHost,
                            ctx->stream),
       "perm");
  rc = wait_stream(ctx, 0, s);
  if (rc) return rc;
  if (perm)
    for (uint32_t i = 0; i < s->n; i++) perm[i] -= s->off;  // galaxy-local indices
  return GS_OK;
}

int gs_read_state(gs_ctx* ctx, float* particles8, float* stellar4) {
  CTX_CHECK(ctx);
  SLOT(ctx, s);
  if (particles8)
    CK(ctx, cudaMemcpyAsync(particles8, ctx->part[ctx->cur] + 2 * (size_t)s->off, (size_t)s->n * 32,
                            cudaMemcpyDeviceToHost, ctx->stream),
       "state");
  if (stellar4)
    CK(ctx, cudaMemcpyAsync(stellar4, ctx->stel[ctx->scur] + s->off, (size_t)s->n * 16, cudaMemcpyDeviceToHost,
                            ctx->stream),
       "stellar");
  return wait_stream(ctx, 0, s);
}

// Stream-ordered: both ping-pong buffers get the state (like NBodyGPU._init).
int gs_write_state(gs_ctx* ctx, const float* particles8, const float* stellar4) {
  CTX_CHECK(ctx);
  SLOT(ctx, s);
  // both ping-pong buffers get the records: one upload, then a device copy
  float4* const p0 = ctx->part[0] + 2 * (size_t)s->off;
  float4* const s0 = ctx->stel[0] + s->off;
  if (particles8) {
    CK(ctx, cudaMemcpyAsync(p0, particles8, (size_t)s->n * 32, cudaMemcpyHostToDevice, ctx->stream), "state");
    CK(ctx, cudaMemcpyAsync(ctx->part[1] + 2 * (size_t)s->off, p0, (size_t)s->n * 32, cudaMemcpyDeviceToDevice,
                            ctx->stream),
       "state");
  }
  if (stellar4) {
    CK(ctx, cudaMemcpyAsync(s0, stellar4, (size_t)s->n * 16, cudaMemcpyHostToDevice, ctx->stream), "stellar");
    CK(ctx, cudaMemcpyAsync(ctx->stel[1] + s->off, s0, (size_t)s->n * 16, cudaMemcpyDeviceToDevice, ctx->stream),
       "stellar");
  }
  return wait_stream(ctx, 0, s);
}

int gs_set_debug(gs_ctx* ctx, int enable) {
  CTX_CHECK(ctx);
  if (enable && !ctx->dbg_acc) {
    CK(ctx, ctx->alloc(&ctx->dbg_acc, ctx->plan.cap), "debug acc");
    CK(ctx, ctx->alloc(&ctx->dbg_dens, ctx->plan.cap), "debug density");
  }
  ctx->debug = enable != 0;
  return GS_OK;
}

int gs_read_forces(gs_ctx* ctx, float* acc4, float* density) {
  CTX_CHECK(ctx);
  SLOT(ctx, s);
  if (!ctx->dbg_acc) return ctx->fail(GS_ENOTREADY, "gs_set_debug(ctx, 1) first");
  int rc = wait_stream(ctx, 0, s);
  if (rc) return rc;
  if (acc4)
    CK(ctx, cudaMemcpy(acc4, ctx->dbg_acc + s->off, (size_t)s->n * 16, cudaMemcpyDeviceToHost), "acc");
  if (density)
    CK(ctx, cudaMemcpy(density, ctx->dbg_dens + s->off, (size_t)s->n * 4, cudaMemcpyDeviceToHost), "dens");
  return GS_OK;
}

int gs_energy(gs_ctx* ctx, gs_diag* out) {
  CTX_CHECK(ctx);
  SLOT(ctx, s);
  if (!out) return ctx->fail(GS_EINVAL, "out is NULL");
  double h[kPartials];
  CK(ctx, cudaMemcpyAsync(h, ctx->diag_out + (size_t)ctx->sel * kPartials, sizeof(h), cudaMemcpyDeviceToHost,
                          ctx->stream),
     "diag");
  int rc = wait_stream(ctx, 0, s);
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
  SLOT(ctx, s);
  (void)s;
  CK(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  unsigned e = 0;
  CK(ctx, cudaMemcpy(&e, &ctx->st[ctx->sel].err, 4, cudaMemcpyDeviceToHost), "err");
  if (bits) *bits = e;
  if (clear) CK(ctx, cudaMemset(&ctx->st[ctx->sel].err, 0, 4), "clear");
  return GS_OK;
}

int gs_counters(gs_ctx* ctx, uint64_t out[3], int reset) {
  CTX_CHECK(ctx);
  SLOT(ctx, s);
  (void)s;
  CK(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  unsigned long long c[3];
  CK(ctx, cudaMemcpy(c, ctx->st[ctx->sel].counters, sizeof(c), cudaMemcpyDeviceToHost), "counters");
  if (out)
    for (int k = 0; k < 3; k++) out[k] = c[k];
  if (reset) CK(ctx, cudaMemset(ctx->st[ctx->sel].counters, 0, sizeof(c)), "reset");
  return GS_OK;
}

}  // extern "C"

// ---- stateless mortonTree.js entry points ----------------------------------------------

namespace {

// A one-galaxy pool of N particles whose buffers the stateless calls fill.
struct TmpCtx {
  gs_ctx* c = nullptr;
  ~TmpCtx() { gs_destroy(c); }
};

int tmp_init(TmpCtx& t, uint32_t N, uint32_t max_nodes) {
  int dev = 0;
  cudaGetDevice(&dev);
  int rc = gs_pool_create(dev, N, 1, &t.c);
  if (rc) return rc;
  gs_ctx* c = t.c;
  Slot& s = c->slots[0];
  s.live = true;
  s.off = 0;
  s.n = s.span = N;
  s.node_off = 0;
  s.node_cap = 2 * N + 4096;
  s.max_nodes = max_nodes;
  c->single = true;
  DevState st0;
  memset(&st0, 0, sizeof(st0));
  st0.central[0] = st0.central[1] = -1;
  if (cudaMemcpy(c->st, &st0, sizeof(st0), cudaMemcpyHostToDevice) != cudaSuccess) {
    set_err(g_err, "state upload failed");
    return GS_ECUDA;
  }
  rc = ensure_layout(c);
  if (rc) set_err(g_err, "%s", c->err);
  return rc;
}

int tmp_check(TmpCtx& t) {
  gs_ctx* c = t.c;
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_err(g_err, "%s", cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? GS_ENOMEM : GS_ECUDA;
  }
  unsigned err = 0;
  if ((e = cudaMemcpy(&err, &c->st[0].err, 4, cudaMemcpyDeviceToHost)) != cudaSuccess) {
    set_err(g_err, "%s", cudaGetErrorString(e));
    return GS_ECUDA;
  }
  if (err) {
    set_err(g_err, "device error word 0x%x", err);
    return (err & GS_DERR_NODES) ? GS_EINVAL : GS_EDEVICE;
  }
  return GS_OK;
}

#define TK(expr, what)                                                     \
  do {                                                                     \
    cudaError_t _e = (expr);                                               \
    if (_e != cudaSuccess) {                                               \
      set_err(g_err, "%s: %s", (what), cudaGetErrorString(_e));            \
      return _e == cudaErrorMemoryAllocation ? GS_ENOMEM : GS_ECUDA;       \
    }                                                                      \
  } while (0)

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
  gs_ctx* c = t.c;
  TreeMeta m;
  TK(cudaMemcpy(&m, c->meta, sizeof(m), cudaMemcpyDeviceToHost), "meta");
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
    if (stage_grow(c, m.num_nodes)) {
      set_err(g_err, "%s", c->err);
      return GS_ENOMEM;
    }
    tree_bhnode_kernel<<<grid_for(m.num_nodes, 256, 148 * 8), 256, 0, c->stream>>>(c->bb(), c->lay, 0, c->bh);
    TK(cudaGetLastError(), "materialise");
    TK(cudaMemcpyAsync(nodes, c->bh, sizeof(gs_node) * m.num_nodes, cudaMemcpyDeviceToHost, c->stream), "nodes");
    TK(cudaStreamSynchronize(c->stream), "sync");
  }
  return GS_OK;
}

// Failure-detection settings of the two radix-sort entry points (gs_test_sort_lookback).
std::atomic<uint32_t> g_test_spin_limit{kSpinLimit};
std::atomic<uint32_t> g_test_withhold{kNoTile};

__global__ void mask30_kernel(uint32_t* keys, uint32_t N) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
    keys[i] &= 0x3fffffffu;
}

}  // namespace

extern "C" {

int gs_morton_codes(const float* pos, uint32_t N, uint32_t stride, uint32_t* codes, double* root_size) {
  if ((!pos && N) || (!codes && N) || stride < 3) {
    set_err(g_err, "bad arguments");
    return GS_EINVAL;
  }
  if (N > kMaxPool) {
    set_err(g_err, "N too large");
    return GS_EINVAL;
  }
  if (N == 0) {  // mortonTree.js:53 over no particles: -Infinity
    if (root_size) *root_size = -INFINITY;
    return GS_OK;
  }
  TmpCtx t;
  int rc = tmp_init(t, N, 2 * N + 4096);
  if (rc) return rc;
  gs_ctx* c = t.c;
  std::vector<float4> h;
  host_pack4(pos, N, stride, h);
  TK(cudaMemcpyAsync(c->part[0], h.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, c->stream), "upload");
  const Layout& L = c->lay;
  bbox_kernel<<<L.flag_tiles, kTileThreads, 0, c->stream>>>(c->part[0], 1, L, c->bbox_part, c->seg_ctr,
                                                            c->frames, c->st, 0, nullptr, 0u, nullptr, 0u);
  codes_kernel<<<L.flag_tiles, kTileThreads, 0, c->stream>>>(c->part[0], 1, L, c->frames, c->keys[0], nullptr,
                                                             0);
  TK(cudaGetLastError(), "codes");
  MortonFrame f;
  TK(cudaMemcpyAsync(codes, c->keys[0], sizeof(uint32_t) * N, cudaMemcpyDeviceToHost, c->stream), "codes");
  TK(cudaMemcpyAsync(&f, c->frames, sizeof(f), cudaMemcpyDeviceToHost, c->stream), "frame");
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
  if (N > kMaxPool) {
    set_err(g_err, "N too large");
    return GS_EINVAL;
  }
  TmpCtx t;
  int rc = tmp_init(t, N, 2 * N + 4096);
  if (rc) return rc;
  gs_ctx* c = t.c;
  const Layout& L = c->lay;
  TK(cudaMemcpyAsync(c->keys[0], codes, sizeof(uint32_t) * N, cudaMemcpyHostToDevice, c->stream), "upload");
  // radixSortIndices orders by the low 30 bits only (3 x 10-bit digits)
  mask30_kernel<<<grid_for(N, 256, 148 * 8), 256, 0, c->stream>>>(c->keys[0], N);
  TK(cudaMemsetAsync(c->sort_scratch, 0, sizeof(uint32_t) * c->plan.sort_words, c->stream), "clear");
  key_hist_kernel<<<L.flag_tiles, kTileThreads, 0, c->stream>>>(c->keys[0], L, c->hist(), kSortPasses);
  enqueue_sort_passes(c, false, g_test_spin_limit.load(), g_test_withhold.load());
  TK(cudaGetLastError(), "sort");
  TK(cudaMemcpyAsync(perm, c->vals[0], sizeof(uint32_t) * N, cudaMemcpyDeviceToHost, c->stream), "perm");
  return tmp_check(t);
}

}  // extern "C"

// The failure-detection settings, for the allocation-free sort in noalloc.cu.
void gs_internal_sort_test_settings(uint32_t* spin_limit, uint32_t* withhold) {
  *spin_limit = g_test_spin_limit.load();
  *withhold = g_test_withhold.load();
}

extern "C" {

int gs_test_sort_lookback(uint32_t spin_limit, int64_t withhold_tile) {
  if (spin_limit == 0 || withhold_tile < -1 || withhold_tile >= (int64_t)kNoTile) {
    set_err(g_err, "spin_limit must be positive and withhold_tile a tile index or -1");
    return GS_EINVAL;
  }
  g_test_spin_limit.store(spin_limit);
  g_test_withhold.store(withhold_tile < 0 ? kNoTile : (uint32_t)withhold_tile);
  return GS_OK;
}

int gs_test_fail_alloc(int64_t nth) {
  if (nth < -1) {
    set_err(g_err, "nth must be an allocation count or -1");
    return GS_EINVAL;
  }
  g_fail_alloc_in.store(nth);
  return GS_OK;
}

int gs_tree_build(const uint32_t* sorted_codes, const float* pos3, const float* masses, uint32_t N,
                  double root_size, uint32_t max_nodes, gs_node* nodes, uint32_t* num_nodes,
                  uint32_t* level_ranges, uint32_t lr_cap, uint32_t* n_levels) {
  if (N == 0) {
    empty_tree(root_size, nodes, num_nodes, level_ranges, n_levels);
    return GS_OK;
  }
  if (!sorted_codes || !pos3 || !masses || N > kMaxPool) {
    set_err(g_err, "bad arguments");
    return GS_EINVAL;
  }
  if (max_nodes == 0) max_nodes = 2 * N + 4096;
  TmpCtx t;
  int rc = tmp_init(t, N, max_nodes);
  if (rc) return rc;
  gs_ctx* c = t.c;
  std::vector<float4> h(N);
  std::vector<uint32_t> k(N);
  for (uint32_t i = 0; i < N; i++) {
    h[i] = make_float4(pos3[3 * (size_t)i], pos3[3 * (size_t)i + 1], pos3[3 * (size_t)i + 2], masses[i]);
    k[i] = sorted_codes[i] & 0x3fffffffu;
  }
  TK(cudaMemcpyAsync(c->part[0], h.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, c->stream), "upload");
  TK(cudaMemcpyAsync(c->keys[0], k.data(), sizeof(uint32_t) * N, cudaMemcpyHostToDevice, c->stream), "codes");
  enqueue_build(c, c->part[0], 1, kComJs, root_size, nullptr);
  TK(cudaGetLastError(), "build");
  return tree_outputs(t, max_nodes, nodes, num_nodes, level_ranges, lr_cap, n_levels);
}

int gs_sort_and_build(const float* particles8, const float* stellar4, uint32_t N, int64_t track_idx2,
                      float* sorted8, float* sorted_stellar4, uint32_t* perm, gs_node* nodes,
                      uint32_t max_nodes, uint32_t* num_nodes, uint32_t* level_ranges, uint32_t lr_cap,
                      uint32_t* n_levels, int64_t* central_idx, int64_t* central_idx2, float* sorted_mass) {
  if (N == 0) {
    empty_tree(-INFINITY, nodes, num_nodes, level_ranges, n_levels);
    if (central_idx) *central_idx = 0;
    if (central_idx2) *central_idx2 = -1;
    return GS_OK;
  }
  if (!particles8 || N > kMaxPool) {
    set_err(g_err, "bad arguments");
    return GS_EINVAL;
  }
  if (max_nodes == 0) max_nodes = 2 * N + 4096;
  TmpCtx t;
  int rc = tmp_init(t, N, max_nodes);
  if (rc) return rc;
  gs_ctx* c = t.c;
  float4 *P = c->part[0], *P2 = c->part[1], *S = c->stel[0], *S2 = c->stel[1];
  TK(cudaMemcpyAsync(P, particles8, (size_t)N * 32, cudaMemcpyHostToDevice, c->stream), "upload");
  if (stellar4) TK(cudaMemcpyAsync(S, stellar4, (size_t)N * 16, cudaMemcpyHostToDevice, c->stream), "upload");
  else TK(cudaMemsetAsync(S, 0, (size_t)N * 16, c->stream), "memset");
  enqueue_codes_sort(c, P, 2, 0);
  enqueue_sort_passes(c, false);
  gather_kernel<<<c->lay.flag_tiles, kTileThreads, 0, c->stream>>>(c->vals[0], P, P2, S, S2, c->lay, c->st);
  enqueue_build(c, P2, 2, kComJs, 0.0, c->frames);
  TK(cudaGetLastError(), "sort and build");
  std::vector<uint32_t> hp(N);
  TK(cudaMemcpyAsync(hp.data(), c->vals[0], sizeof(uint32_t) * N, cudaMemcpyDeviceToHost, c->stream), "perm");
  if (sorted8) TK(cudaMemcpyAsync(sorted8, P2, (size_t)N * 32, cudaMemcpyDeviceToHost, c->stream), "sorted");
  if (sorted_stellar4)
    TK(cudaMemcpyAsync(sorted_stellar4, S2, (size_t)N * 16, cudaMemcpyDeviceToHost, c->stream), "stellar");
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

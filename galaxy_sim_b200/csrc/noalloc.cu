// Allocation-free stable radix sort: gs_radix_sort_indices_noalloc.
//
// Some callers may not allocate device memory once they are running: a host
// application's per-frame callback (cudaMalloc and cudaFree can synchronize the
// whole device and stall its other streams mid-frame), or an embedding engine
// that budgets device memory at start-up and forbids allocation afterwards.
// This variant of the sort behind gs_radix_sort_indices allocates nothing. The
// caller passes device pointers for the codes and the permutation, plus the
// stream to run on. Every intermediate buffer lives in one file-scope static
// device array sized for at most kNoAllocMaxN codes. Each GPU that loads the
// library holds that array until the process exits.
//
// The host code never hands the array's name to a kernel. In host code that
// name only stands in for the device object, so a kernel given it would fault
// or, where the GPU can reach host memory, silently use the wrong memory.
// Set-up runs once per device context, with that device current: it looks up
// the array's device address with cudaGetSymbolAddress and caches it, keyed by
// the context's unique id so that a context reset (cudaDeviceReset) is noticed
// and the address looked up again. Under lazy module loading the array and the
// kernels' code are committed when first touched, so set-up also loads every
// kernel of the sort and runs each once over no keys. A call with N == 0 does
// only the set-up; callers make it at start-up, outside any stream capture, so
// that later calls allocate nothing.
//
// Every call is synchronous (it reads the error word back and waits for the
// stream), so it must never run inside a stream capture; a capturing stream is
// rejected before anything is enqueued.
//
// All calls share the one array, and it keeps the contents of the last call.
// Each call therefore clears the histograms, tile counters and look-back
// words it relies on, and rewrites its one-galaxy layout, before using them.
// Calls whose work overlaps on the GPU (two streams, or two host threads) race
// on that shared array: serialize them.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <mutex>

#include "common.cuh"
#include "sort.cuh"

void gs_internal_set_error(const char* msg);
void gs_internal_sort_test_settings(uint32_t* spin_limit, uint32_t* withhold);

namespace {

using namespace gs;

constexpr uint32_t kNoAllocMaxN = 1u << 20;  // 1,048,576 codes
constexpr uint32_t kNoAllocTiles = (kNoAllocMaxN + kSortTile - 1) / kSortTile;
constexpr int kNoAllocPasses = 4;
// two key buffers + one payload buffer, then histograms | tile counters |
// look-back (cleared per call) | the one-galaxy layout (segment, tile map)
constexpr size_t kKeyWords = (size_t)kNoAllocMaxN;
constexpr size_t kHistOff = 3 * kKeyWords;
constexpr size_t kCtrOff = kHistOff + kNoAllocPasses * 256;
constexpr size_t kLbOff = kCtrOff + 16;
constexpr size_t kSegOff = kLbOff + (size_t)kNoAllocPasses * kNoAllocTiles * 256;  // 16-byte aligned
constexpr size_t kMapOff = kSegOff + sizeof(SegDesc) / sizeof(uint32_t);
constexpr size_t kScratchWords = kMapOff + kNoAllocTiles;
constexpr size_t kClearBytes = (kSegOff - kHistOff) * sizeof(uint32_t);
static_assert(kSegOff % 4 == 0 && sizeof(SegDesc) % 16 == 0, "segment descriptor alignment");

static __device__ __align__(256) uint32_t g_noalloc_scratch[kScratchWords];  // about 13 MiB
static __device__ DevState g_noalloc_state;                                   // error word

constexpr int kMaxDevices = 64;
struct DeviceSetup {
  unsigned long long ctx_id = 0;  // the context the addresses belong to (0 = none yet)
  void* scratch = nullptr;
  void* state = nullptr;
};
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mutex;

// radixSortIndices orders by the low 30 bits (mortonTree.js:71-74): copy the
// masked codes into the first key buffer and count every pass's digits.
__global__ void noalloc_mask_hist_kernel(const uint32_t* __restrict__ codes, uint32_t N,
                                         uint32_t* __restrict__ keys, uint32_t* hist) {
  __shared__ uint32_t s_hist[kNoAllocPasses * 256];
  for (int k = threadIdx.x; k < kNoAllocPasses * 256; k += blockDim.x) s_hist[k] = 0;
  __syncthreads();
  for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < N; i0 += gridDim.x * blockDim.x) {
    const uint32_t i = i0 + threadIdx.x;
    const bool valid = i < N;
    uint32_t key = 0;
    if (valid) {
      key = codes[i] & 0x3fffffffu;
      keys[i] = key;
    }
    hist_add_warp(s_hist, key, valid, kNoAllocPasses);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < kNoAllocPasses * 256; k += blockDim.x)
    if (s_hist[k]) atomicAdd(&hist[k], s_hist[k]);
}

// The layout of one galaxy of N codes at offset 0: its descriptor and the
// sort-tile map (every tile belongs to galaxy 0).
__global__ void noalloc_layout_kernel(SegDesc* seg, uint32_t* map, uint32_t N, uint32_t tiles) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    SegDesc d;
    d.off = 0;
    d.n = N;
    d.node_off = 0;
    d.node_cap = 0;
    d.sort_tile0 = 0;
    d.flag_tile0 = 0;
    d.group0 = 0;
    d.max_nodes = 0;
    d.slot = 0;
    d.diag_chunk0 = 0;
    d.wlpp = 1;
    d.item0 = 0;
    d.wsplit = 1;
    d.pad_[0] = d.pad_[1] = d.pad_[2] = 0;
    *seg = d;
  }
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < tiles; t += gridDim.x * blockDim.x) map[t] = 0;
}

int fail(int code, const char* msg) {
  gs_internal_set_error(msg);
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  char buf[256];
  snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
  gs_internal_set_error(buf);
  return e == cudaErrorMemoryAllocation ? GS_ENOMEM : GS_ECUDA;
}

// Unique id of the calling thread's current context (driver entry points,
// resolved once through the runtime, so the library needs no libcuda link).
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;

int current_context_id(unsigned long long* id) {
  if (!g_ctx_get_current || !g_ctx_get_id) {
    void* f0 = nullptr;
    void* f1 = nullptr;
    cudaDriverEntryPointQueryResult q0, q1;
    cudaError_t e = cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f0, 12000, cudaEnableDefault, &q0);
    if (e == cudaSuccess)
      e = cudaGetDriverEntryPointByVersion("cuCtxGetId", &f1, 12000, cudaEnableDefault, &q1);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDriverEntryPointByVersion");
    if (q0 != cudaDriverEntryPointSuccess || q1 != cudaDriverEntryPointSuccess || !f0 || !f1)
      return fail(GS_ECUDA, "the driver lacks cuCtxGetCurrent/cuCtxGetId");
    g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f0);
    g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(f1);
  }
  CUcontext ctx = nullptr;
  if (g_ctx_get_current(&ctx) != CUDA_SUCCESS) return fail(GS_ECUDA, "cuCtxGetCurrent failed");
  *id = 0;
  if (ctx && g_ctx_get_id(ctx, id) != CUDA_SUCCESS) return fail(GS_ECUDA, "cuCtxGetId failed");
  return GS_OK;
}

// Set-up on the current device: load the module's array and kernels and look up
// the array's device address, once per context. Returns the cached addresses.
int setup_device(int dev, uint32_t** base, DevState** st) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  DeviceSetup& d = g_setup[dev];
  unsigned long long id = 0;
  int rc = current_context_id(&id);
  if (rc) return rc;
  if (id == 0 || id != d.ctx_id) {
    void* p = nullptr;
    void* q = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(scratch)");
    e = cudaGetSymbolAddress(&q, g_noalloc_state);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(state)");
    // load the code of every kernel the sort launches (lazy loading would
    // otherwise commit it on the first launch)
    cudaFuncAttributes fa;
    const void* kernels[] = {
        reinterpret_cast<const void*>(noalloc_layout_kernel),
        reinterpret_cast<const void*>(noalloc_mask_hist_kernel),
        reinterpret_cast<const void*>(onesweep_pass<true, false>),
        reinterpret_cast<const void*>(onesweep_pass<false, false>),
    };
    for (const void* k : kernels)
      if ((e = cudaFuncGetAttributes(&fa, k)) != cudaSuccess) return cuda_fail(e, "cudaFuncGetAttributes");
    if ((rc = current_context_id(&id))) return rc;  // the look-up made the context current
    d.scratch = p;
    d.state = q;
    d.ctx_id = id;
  }
  *base = static_cast<uint32_t*>(d.scratch);
  *st = static_cast<DevState*>(d.state);
  return GS_OK;
}

}  // namespace

extern "C" int gs_radix_sort_indices_noalloc(const uint32_t* d_codes, uint32_t N, uint32_t* d_perm,
                                             void* stream) {
  if (N > kNoAllocMaxN)
    return fail(GS_EINVAL, "gs_radix_sort_indices_noalloc: N exceeds its static scratch "
                           "(at most 1048576 codes)");
  if (N && (!d_codes || !d_perm)) return fail(GS_EINVAL, "d_codes and d_perm must be device pointers");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(s, &cap);
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamIsCapturing");
  if (cap != cudaStreamCaptureStatusNone)
    return fail(GS_EINVAL, "gs_radix_sort_indices_noalloc is synchronous and cannot run while its "
                           "stream is capturing");
  int dev = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return fail(GS_EINVAL, "device ordinal out of range");
  uint32_t* base = nullptr;
  DevState* st = nullptr;
  int rc = setup_device(dev, &base, &st);
  if (rc) return rc;
  uint32_t* k0 = base;
  uint32_t* k1 = base + kKeyWords;
  uint32_t* v0 = base + 2 * kKeyWords;
  uint32_t* hist = base + kHistOff;
  uint32_t* ctr = base + kCtrOff;
  uint32_t* lb = base + kLbOff;
  SegDesc* seg = reinterpret_cast<SegDesc*>(base + kSegOff);
  uint32_t* map = base + kMapOff;
  if (N == 0) {
    // the set-up call: every kernel of the sort runs once over no keys, so that
    // its code and local memory are in place before the first real call
    Layout E = {};
    E.segs = seg;
    E.seg_of_sort_tile = map;
    E.nseg = 1;
    noalloc_layout_kernel<<<1, 256, 0, s>>>(seg, map, 0, 0);
    noalloc_mask_hist_kernel<<<1, 256, 0, s>>>(nullptr, 0, k0, hist);
    onesweep_pass<true, false><<<1, kSortThreads, 0, s>>>(nullptr, nullptr, nullptr, nullptr, nullptr, hist, 0,
                                                          lb, ctr, E, st);
    onesweep_pass<false, false><<<1, kSortThreads, 0, s>>>(nullptr, nullptr, nullptr, nullptr, nullptr, hist, 1,
                                                           lb, ctr + 1, E, st);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "set-up launch");
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
    return GS_OK;
  }
  uint32_t spin_limit = kSpinLimit, withhold = kNoTile;
  gs_internal_sort_test_settings(&spin_limit, &withhold);
  const uint32_t tiles = (N + kSortTile - 1) / kSortTile;
  // what must start at zero: histograms, tile counters, look-back words, error word
  if ((e = cudaMemsetAsync(hist, 0, kClearBytes, s)) != cudaSuccess) return cuda_fail(e, "clear");
  if ((e = cudaMemsetAsync(&st->err, 0, sizeof(unsigned), s)) != cudaSuccess)
    return cuda_fail(e, "clear");
  const uint32_t grid = std::min<uint32_t>(148 * 8, (N + 255) / 256);
  noalloc_layout_kernel<<<1, 256, 0, s>>>(seg, map, N, tiles);
  noalloc_mask_hist_kernel<<<grid, 256, 0, s>>>(d_codes, N, k0, hist);
  Layout L;
  L.segs = seg;
  L.seg_of_sort_tile = map;
  L.seg_of_flag_tile = nullptr;
  L.seg_of_group = nullptr;
  L.nseg = 1;
  L.sort_tiles = tiles;
  L.flag_tiles = 0;
  L.groups = 0;
  L.diag_chunks = 0;
  // pass 0: k0 -> k1 (payload = index) -> v0; 1: -> k0, d_perm; 2: -> k1, v0; 3: -> k0, d_perm
  uint32_t* kin[kNoAllocPasses] = {k0, k1, k0, k1};
  uint32_t* kout[kNoAllocPasses] = {k1, k0, k1, k0};
  uint32_t* vin[kNoAllocPasses] = {nullptr, v0, d_perm, v0};
  uint32_t* vout[kNoAllocPasses] = {v0, d_perm, v0, d_perm};
  for (int p = 0; p < kNoAllocPasses; p++) {
    uint32_t* plb = lb + (size_t)p * kNoAllocTiles * 256;
    if (p == 0)
      onesweep_pass<true, false><<<tiles, kSortThreads, 0, s>>>(kin[p], nullptr, kout[p], vout[p], nullptr,
                                                                hist, p, plb, ctr + p, L, st, spin_limit,
                                                                withhold);
    else
      onesweep_pass<false, false><<<tiles, kSortThreads, 0, s>>>(kin[p], vin[p], kout[p], vout[p], nullptr,
                                                                 hist, p, plb, ctr + p, L, st, spin_limit,
                                                                 withhold);
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "sort launch");
  unsigned err = 0;
  if ((e = cudaMemcpyAsync(&err, &st->err, sizeof(unsigned), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return cuda_fail(e, "error word");
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
  if (err) return fail(GS_EDEVICE, "sort look-back wait exceeded its iteration limit");
  return GS_OK;
}

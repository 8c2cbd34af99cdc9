// Per-particle and per-node kernels around the walk: Morton bbox and codes,
// the permutation gather, central tracking with the halo-centre EMA, star
// formation, position compaction, per-level COM refresh, uploaded-tree
// conversion and the FP64 diagnostics reduction.
//
// The per-particle kernels run one 1024-particle tile per block over the tile
// list of a batch layout; a tile lies inside one galaxy.
#pragma once
#include "build.cuh"
#include "common.cuh"
#include "morton.cuh"
#include "sort.cuh"
#include "walk.cuh"

namespace gs {

constexpr int kTileThreads = kFlagThreads;  // 256 threads x 4 particles = one build tile
constexpr int kTilePer = kFlagPer;
constexpr int kTile = kFlagTile;

struct TileRange {
  uint32_t slot;
  uint32_t beg, end;       // pool particles of this tile
  uint32_t seg_beg, seg_end;
  uint32_t lt, ntiles;     // tile index within the galaxy, its tile count
};

__device__ inline TileRange tile_range(const Layout& L, uint32_t tile) {
  const SegDesc sd = L.segs[L.seg_of_flag_tile[tile]];
  TileRange t;
  t.slot = sd.slot;
  t.seg_beg = sd.off;
  t.seg_end = sd.off + sd.n;
  t.lt = tile - sd.flag_tile0;
  t.ntiles = (sd.n + kTile - 1) / kTile;
  t.beg = sd.off + t.lt * kTile;
  t.end = min(t.beg + kTile, t.seg_end);
  return t;
}

// Bounding box over finite particles (mortonTree.js:44-52), per galaxy: each
// tile reduces float min/max as ordered ints into its partial; the galaxy's
// last tile folds its partials, derives the double frame (:53-54) and, with
// advance_time, stamps Params.time = f32(simTime) and advances simTime by dt
// (main.js:422, :476). seg_ctr[slot] counts finished tiles and self-resets.
// It also clears the sort's scratch for this step (zero0[n0], zero1[n1]: digit
// histograms, tile counters, look-back words), which the next kernels fill.
__global__ void __launch_bounds__(kTileThreads)
    bbox_kernel(const float4* __restrict__ pos, uint32_t stride, Layout L, int* partials,
                unsigned* seg_ctr, MortonFrame* frames, DevState* st, int advance_time,
                uint32_t* zero0, uint32_t n0, uint32_t* zero1, uint32_t n1) {
  griddep_wait();  // launched with a programmatic dependency: predecessors' writes first
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n0 + n1; k += gridDim.x * blockDim.x) {
    if (k < n0) zero0[k] = 0u;
    else zero1[k - n0] = 0u;
  }
  __shared__ int s_red[kTileThreads / 32][6];
  __shared__ bool s_last;
  const TileRange t = tile_range(L, blockIdx.x);
  int mn[3] = {float_to_ordered(INFINITY), float_to_ordered(INFINITY), float_to_ordered(INFINITY)};
  int mx[3] = {float_to_ordered(-INFINITY), float_to_ordered(-INFINITY), float_to_ordered(-INFINITY)};
#pragma unroll
  for (int q = 0; q < kTilePer; q++) {
    const uint32_t i = t.beg + q * kTileThreads + threadIdx.x;
    if (i >= t.end) break;
    const float4 p = pos[(size_t)i * stride];
    if (isfinite(p.x) && isfinite(p.y) && isfinite(p.z)) {
      const int e[3] = {float_to_ordered(p.x), float_to_ordered(p.y), float_to_ordered(p.z)};
#pragma unroll
      for (int k = 0; k < 3; k++) {
        mn[k] = min(mn[k], e[k]);
        mx[k] = max(mx[k], e[k]);
      }
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    mn[k] = __reduce_min_sync(0xffffffffu, mn[k]);
    mx[k] = __reduce_max_sync(0xffffffffu, mx[k]);
  }
  if (lane == 0)
    for (int k = 0; k < 3; k++) {
      s_red[warp][k] = mn[k];
      s_red[warp][3 + k] = mx[k];
    }
  __syncthreads();
  if (threadIdx.x < 6) {
    int v = s_red[0][threadIdx.x];
    for (int w = 1; w < kTileThreads / 32; w++)
      v = threadIdx.x < 3 ? min(v, s_red[w][threadIdx.x]) : max(v, s_red[w][threadIdx.x]);
    partials[blockIdx.x * 6 + threadIdx.x] = v;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(&seg_ctr[t.slot], 1u) == t.ntiles - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // fold the galaxy's tile partials with the whole block (independent loads in flight)
#pragma unroll
  for (int k = 0; k < 3; k++) {
    mn[k] = float_to_ordered(INFINITY);
    mx[k] = float_to_ordered(-INFINITY);
  }
  const uint32_t t0 = blockIdx.x - t.lt;
  for (uint32_t b = threadIdx.x; b < t.ntiles; b += blockDim.x) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
      mn[k] = min(mn[k], __ldcg(&partials[(t0 + b) * 6 + k]));
      mx[k] = max(mx[k], __ldcg(&partials[(t0 + b) * 6 + 3 + k]));
    }
  }
#pragma unroll
  for (int k = 0; k < 3; k++) {
    mn[k] = __reduce_min_sync(0xffffffffu, mn[k]);
    mx[k] = __reduce_max_sync(0xffffffffu, mx[k]);
  }
  __syncthreads();
  if (lane == 0)
    for (int k = 0; k < 3; k++) {
      s_red[warp][k] = mn[k];
      s_red[warp][3 + k] = mx[k];
    }
  __syncthreads();
  if (threadIdx.x < 6) {
    int v = s_red[0][threadIdx.x];
    for (int w = 1; w < kTileThreads / 32; w++)
      v = threadIdx.x < 3 ? min(v, s_red[w][threadIdx.x]) : max(v, s_red[w][threadIdx.x]);
    s_red[0][threadIdx.x] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float fmn[3], fmx[3];
    for (int k = 0; k < 3; k++) {
      fmn[k] = ordered_to_float(s_red[0][k]);
      fmx[k] = ordered_to_float(s_red[0][3 + k]);
    }
    frames[t.slot] = frame_from_bbox(fmn, fmx);
    seg_ctr[t.slot] = 0;
    if (advance_time) {
      DevState* s = st + t.slot;
      s->p.time = __double2float_rn(s->sim_time);
      s->sim_time = __dadd_rn(s->sim_time, (double)s->p.dt);
    }
  }
}

// Codes (mortonTree.js:55-60) + the digit histograms of every sort pass, per
// galaxy (hist: [slots][passes][256]).
__global__ void __launch_bounds__(kTileThreads)
    codes_kernel(const float4* __restrict__ pos, uint32_t stride, Layout L,
                 const MortonFrame* __restrict__ frames, uint32_t* __restrict__ codes,
                 uint32_t* hist, int passes) {
  griddep_wait();  // launched with a programmatic dependency: predecessors' writes first
  __shared__ uint32_t s_hist[kSortPasses * 256];
  const TileRange t = tile_range(L, blockIdx.x);
  if (hist)
    for (int k = threadIdx.x; k < passes * 256; k += blockDim.x) s_hist[k] = 0;
  __syncthreads();
  const MortonFrame f = frames[t.slot];
#pragma unroll
  for (int q = 0; q < kTilePer; q++) {
    const uint32_t i = t.beg + q * kTileThreads + threadIdx.x;
    const bool valid = i < t.end;
    uint32_t code = 0;
    if (valid) {
      const float4 p = pos[(size_t)i * stride];
      code = morton_code(f, p.x, p.y, p.z);
      codes[i] = code;
    }
    if (hist && valid)
      for (int p = 0; p < passes; p++) atomicAdd(&s_hist[p * 256 + ((code >> (8 * p)) & 255u)], 1u);
  }
  if (!hist) return;
  __syncthreads();
  uint32_t* h = hist + (size_t)t.slot * kSortPasses * 256;
  for (int k = threadIdx.x; k < passes * 256; k += blockDim.x)
    if (s_hist[k]) atomicAdd(&h[k], s_hist[k]);
}

// Digit histograms of given keys (stateless sort entry points).
__global__ void __launch_bounds__(kTileThreads)
    key_hist_kernel(const uint32_t* __restrict__ keys, Layout L, uint32_t* hist, int passes) {
  __shared__ uint32_t s_hist[kSortPasses * 256];
  const TileRange t = tile_range(L, blockIdx.x);
  for (int k = threadIdx.x; k < passes * 256; k += blockDim.x) s_hist[k] = 0;
  __syncthreads();
#pragma unroll
  for (int q = 0; q < kTilePer; q++) {
    const uint32_t i = t.beg + q * kTileThreads + threadIdx.x;
    const bool valid = i < t.end;
    hist_add_warp(s_hist, valid ? keys[i] : 0u, valid, passes);
  }
  __syncthreads();
  uint32_t* h = hist + (size_t)t.slot * kSortPasses * 256;
  for (int k = threadIdx.x; k < passes * 256; k += blockDim.x)
    if (s_hist[k]) atomicAdd(&h[k], s_hist[k]);
}

// Gather dst[i] = src[perm[i]] of the 32-byte particle and 16-byte stellar
// records (nbody_bh.wgsl:322-326, :336-340). perm holds pool indices of the
// same galaxy; anything else is flagged, never dereferenced.
__global__ void __launch_bounds__(kTileThreads)
    gather_kernel(const uint32_t* __restrict__ perm, const float4* __restrict__ pin,
                  float4* __restrict__ pout, const float4* __restrict__ sin,
                  float4* __restrict__ sout, Layout L, DevState* st) {
  griddep_wait();  // launched with a programmatic dependency: predecessors' writes first
  const TileRange t = tile_range(L, blockIdx.x);
#pragma unroll
  for (int q = 0; q < kTilePer; q++) {
    const uint32_t i = t.beg + q * kTileThreads + threadIdx.x;
    if (i >= t.end) break;
    const uint32_t s = perm[i];
    if (s < t.seg_beg || s >= t.seg_end) {
      raise_err(st + t.slot, GS_DERR_LOOKBACK);
      continue;
    }
    const float4 a = pin[2 * (size_t)s], b = pin[2 * (size_t)s + 1];
    pout[2 * (size_t)i] = a;
    pout[2 * (size_t)i + 1] = b;
    if (sout) sout[i] = sin[s];
  }
}

// Central-particle tracking after a sort (one thread per galaxy): the tracked
// index follows the permutation (bhWorker.js:67-68) through inv[old] = new, and
// the halo centre moves 10% of the way to the particle (main.js:449-457, in
// double like the JS numbers); its f32 copy goes to Params (NBodyGPU.js:272-273).
__global__ void track_kernel(const uint32_t* __restrict__ inv, const float4* __restrict__ P,
                             Layout L, DevState* st) {
  griddep_wait();  // launched with a programmatic dependency: predecessors' writes first
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= L.nseg) return;
  const SegDesc sd = L.segs[r];
  DevState* s = st + sd.slot;
  for (int h = 0; h < 2; h++) {
    const long long c = s->central[h];
    if (c < (long long)sd.off || c >= (long long)sd.off + sd.n) continue;  // -1: not tracked
    const uint32_t ni = inv[c];
    if (ni < sd.off || ni >= sd.off + sd.n) {
      raise_err(s, GS_DERR_LOOKBACK);
      continue;
    }
    s->central[h] = ni;
    if (h < (int)s->p.haloCount) {
      const float4 a = P[2 * (size_t)ni];
      const float q[3] = {a.x, a.y, a.z};
      float* dst = h == 0 ? s->p.haloC1 : s->p.haloC2;
      for (int k = 0; k < 3; k++) {
        const double hc = s->halo_c[h][k];
        const double nv = __dadd_rn(hc, __dmul_rn(__dsub_rn((double)q[k], hc), 0.1));
        s->halo_c[h][k] = nv;
        dst[k] = __double2float_rn(nv);
      }
    }
  }
}

// star_formation as its own pass (NBodyGPU.encodeStarFormation); the RNG
// stream index is the particle's index within its galaxy.
__global__ void __launch_bounds__(kTileThreads)
    sf_kernel(float4* __restrict__ P, float4* __restrict__ S, Layout L,
              const DevState* __restrict__ st) {
  const TileRange t = tile_range(L, blockIdx.x);
  if (st[t.slot].sf_off) return;
  const gs_params prm = st[t.slot].p;
#pragma unroll
  for (int q = 0; q < kTilePer; q++) {
    const uint32_t i = t.beg + q * kTileThreads + threadIdx.x;
    if (i >= t.end) break;
    float4 p1 = P[2 * (size_t)i + 1];
    float4 s = S[i];
    const float4 p1o = p1, so = s;
    star_formation_one(prm, i - t.seg_beg, p1, s);
    if (p1.x != p1o.x || p1.y != p1o.y || p1.z != p1o.z || p1.w != p1o.w) P[2 * (size_t)i + 1] = p1;
    if (s.x != so.x || s.y != so.y || s.z != so.z || s.w != so.w) S[i] = s;
  }
}

// compact_positions (nbody_bh.wgsl:188-195) over one particle range.
__global__ void compact_kernel(const float4* __restrict__ P, const float* __restrict__ energy,
                               float4* __restrict__ out, uint32_t N) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const float4 p = P[2 * (size_t)i];
    out[i] = make_float4(p.x, p.y, p.z, energy[i]);
  }
}

// Snapshot of one galaxy's diagnostics (kPartials doubles) and error word into
// mapped pinned host memory, in stream order: the asynchronous readback delivers
// the values of the step it follows even when later steps overwrite them.
__global__ void readback_snapshot_kernel(const double* __restrict__ diag, const unsigned* __restrict__ err,
                                         double* host) {
  const int t = threadIdx.x;
  if (t < kPartials) host[t] = diag[t];
  if (t == kPartials) reinterpret_cast<unsigned*>(host + kPartials)[0] = *err;
}

// refresh_level (nbody_bh.wgsl:288-313) on one BFS level of the walk layout
// (pool indices).
__global__ void refresh_level_kernel(const float4* __restrict__ P, float4* cm,
                                     const WalkInfo* __restrict__ info, uint32_t start,
                                     uint32_t count) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= count) return;
  const uint32_t n = start + g;
  const WalkInfo w = info[n];
  const uint32_t cnt = w.info & ~kLeafBit;
  float cx = 0, cy = 0, cz = 0, m = 0;
  if (w.info & kLeafBit) {
    for (uint32_t j = w.child; j < w.child + cnt; j++) {
      const float4 p = P[2 * (size_t)j];
      cx = fmaf(p.x, p.w, cx);
      cy = fmaf(p.y, p.w, cy);
      cz = fmaf(p.z, p.w, cz);
      m += p.w;
    }
  } else {
    for (uint32_t k = 0; k < cnt; k++) {
      const float4 q = __ldcg(&cm[w.child + k]);
      cx = fmaf(q.x, q.w, cx);
      cy = fmaf(q.y, q.w, cy);
      cz = fmaf(q.z, q.w, cz);
      m += q.w;
    }
  }
  cm[n] = m > 0.0f ? make_float4(cx / m, cy / m, cz / m, m) : make_float4(0.f, 0.f, 0.f, m);
}

// uploadBHTree: BHNode (64 B) -> walk layout of one galaxy, whose nodes start at
// node_off and particles at off of the pools. Children of an internal node must
// be the contiguous increasing run the BFS build produces (mortonTree.js:146-155).
// A node that breaks the rules (children not after their parent, ranges past
// the node or particle arrays) is flagged and made an empty leaf, so a walk
// over an uploaded tree always terminates and stays in bounds.
__global__ void upload_convert_kernel(const gs_node* __restrict__ nodes, uint32_t num_nodes,
                                      uint32_t N, uint32_t node_off, uint32_t off, float4* cm,
                                      WalkInfo* info, DevState* st) {
  for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < num_nodes; n += gridDim.x * blockDim.x) {
    const gs_node nd = nodes[n];
    float4 c = make_float4(nd.com[0], nd.com[1], nd.com[2], nd.mass);
    WalkInfo w;
    w.s2 = nd.size * nd.size;
    w.size = nd.size;
    bool ok = true;
    if (nd.isLeaf == 1u) {
      ok = nd.count < kLeafBit && (uint64_t)nd.first + nd.count <= N;
      w.child = off + nd.first;
      w.info = kLeafBit | (nd.count & ~kLeafBit);
    } else {
      int32_t first = -1;
      uint32_t nc = 0;
      for (int k = 0; k < 8; k++) {
        const int32_t ch = nd.children[k];
        if (ch < 0) continue;
        if (first < 0) first = ch;
        else if (ch != first + (int32_t)nc) ok = false;
        if ((uint32_t)ch >= num_nodes || (uint32_t)ch <= n) ok = false;
        nc++;
      }
      w.child = node_off + (first < 0 ? 0u : (uint32_t)first);
      w.info = nc;
    }
    if (!ok) {
      raise_err(st, GS_DERR_TREE);
      w.child = off;
      w.info = kLeafBit;  // empty leaf
      c.w = 0.0f;
    }
    cm[node_off + n] = c;
    info[node_off + n] = w;
  }
}

// FP64 diagnostics: fold each galaxy's per-item walk partials into
// out[slot][kPartials]. A block of 32 x kPartials threads sums kDiagChunk groups
// of one galaxy (chunks counted from the galaxy's first group): the chunk's
// partials are one contiguous run of doubles, read coalesced with a stride of
// 32 x kPartials so that thread t always adds component t mod kPartials; the 32
// threads of a component are then added in thread order. The galaxy's last
// block adds the chunk sums in chunk order the same way, so the result does not
// depend on the layout or on block timing. diag_ctr[slot] self-resets.
constexpr uint32_t kDiagChunk = 64;
__global__ void __launch_bounds__(32 * kPartials)
    diag_reduce_kernel(const double* __restrict__ partials, Layout L, double* chunk_part,
                       unsigned* diag_ctr, double* out) {
  griddep_wait();  // launched with a programmatic dependency: predecessors' writes first
  constexpr uint32_t kThreads = 32 * kPartials;
  __shared__ double s_v[kThreads];
  __shared__ bool s_last;
  const uint32_t x = blockIdx.x, t = threadIdx.x;
  uint32_t lo = 0, hi = L.nseg;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (L.segs[mid].diag_chunk0 <= x) lo = mid;
    else hi = mid;
  }
  const SegDesc sd = L.segs[lo];
  const uint32_t ng = (sd.n + kWalkGroup - 1) / kWalkGroup;
  const uint32_t nch = (ng + kDiagChunk - 1) / kDiagChunk;
  const uint32_t g0 = (x - sd.diag_chunk0) * kDiagChunk, g1 = min(ng, g0 + kDiagChunk);
  // the chunk's work items (groups in order, each group's items in order)
  const size_t f0 = ((size_t)sd.item0 + (size_t)g0 * sd.wlpp) * kPartials;
  const size_t f1 = ((size_t)sd.item0 + (size_t)g1 * sd.wlpp) * kPartials;
  double v = 0;
#pragma unroll 4
  for (size_t f = f0 + t; f < f1; f += kThreads) v += partials[f];
  s_v[t] = v;
  __syncthreads();
  if (t < kPartials) {
    double w = 0;
    for (uint32_t j = 0; j < 32; j++) w += s_v[j * kPartials + t];
    chunk_part[(size_t)x * kPartials + t] = w;
  }
  __threadfence();
  __syncthreads();
  if (t == 0) s_last = atomicAdd(&diag_ctr[sd.slot], 1u) == nch - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // component t mod kPartials of chunks j, j + 32, ... (j = t / kPartials)
  double w = 0;
  for (uint32_t c = t / kPartials; c < nch; c += 32)
    w += __ldcg(&chunk_part[(size_t)(sd.diag_chunk0 + c) * kPartials + t % kPartials]);
  __syncthreads();
  s_v[t] = w;
  __syncthreads();
  if (t < kPartials) {
    double u = 0;
    for (uint32_t j = 0; j < 32; j++) u += s_v[j * kPartials + t];
    out[(size_t)sd.slot * kPartials + t] = u;
  }
  if (t == 0) diag_ctr[sd.slot] = 0;
}

// Tile / group -> galaxy maps of a layout (binary search over the galaxies'
// first tiles, which increase with the rank).
__global__ void layout_maps_kernel(const SegDesc* __restrict__ segs, uint32_t nseg,
                                   uint32_t* sort_map, uint32_t sort_tiles, uint32_t* flag_map,
                                   uint32_t flag_tiles, uint32_t* group_map, uint32_t groups) {
  const uint32_t total = max(sort_tiles, max(flag_tiles, groups));
  for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < total; x += gridDim.x * blockDim.x) {
#pragma unroll
    for (int which = 0; which < 3; which++) {
      const uint32_t lim = which == 0 ? sort_tiles : which == 1 ? flag_tiles : groups;
      if (x >= lim) continue;
      uint32_t lo = 0, hi = nseg;
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint32_t f = which == 0 ? segs[mid].sort_tile0
                                      : which == 1 ? segs[mid].flag_tile0 : segs[mid].group0;
        if (f <= x) lo = mid;
        else hi = mid;
      }
      (which == 0 ? sort_map : which == 1 ? flag_map : group_map)[x] = lo;
    }
  }
}

}  // namespace gs

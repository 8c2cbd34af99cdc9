// Stable LSD radix sort of 32-bit keys with a 32-bit payload, one kernel per
// 8-bit digit ("onesweep": per-tile ranking by warp match, decoupled look-back
// for the tile's digit offsets; the passes before the last scatter through
// shared memory so each digit's run is written by consecutive threads). A stable sort of
// (code, original index) gives exactly the permutation of radixSortIndices
// (src/physics/mortonTree.js:68-84): ties keep their original order.
//
// Segmented: every galaxy of a batch is sorted within its own particle range
// by the same four launches. Tiles never cross a galaxy, a galaxy's digit
// offsets start at its first particle, and the look-back stops at its first
// tile, so each galaxy's permutation equals the one a solo sort gives.
#pragma once
#include "common.cuh"

namespace gs {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;                        // default keys per thread
constexpr int kSortTile = kSortThreads * kSortItems;  // default keys per tile (4096)
constexpr int kSortTileMin = kSortThreads * 4;        // smallest tile the runtime selects
// with the tile depth chosen by size, galaxies of at most this many particles
// sort with 4 / 8 keys per thread
constexpr uint32_t kSortAuto4 = 131072;
constexpr uint32_t kSortAuto8 = 393216;
constexpr int kSortPasses = 4;                        // 30-bit codes, 8-bit digits
constexpr uint32_t kLbAgg = 1u << 30;
constexpr uint32_t kLbInc = 2u << 30;
constexpr uint32_t kLbMask = (1u << 30) - 1;

__device__ inline void st_relaxed(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ inline uint32_t ld_relaxed(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Digit histograms of all passes at once, warp-aggregated. hist: [passes][256].
__device__ inline void hist_add_warp(uint32_t* s_hist, uint32_t key, bool valid, int passes) {
  const unsigned lane = threadIdx.x & 31;
  for (int p = 0; p < passes; p++) {
    const uint32_t d = (key >> (8 * p)) & 255u;
    const unsigned peers = __match_any_sync(0xffffffffu, valid ? d : 0x100u + lane);
    if (valid && (__ffs(peers) - 1) == (int)lane) atomicAdd(&s_hist[p * 256 + d], __popc(peers));
  }
}

// One digit pass over every galaxy of the layout, ITEMS keys per thread (tiles of
// 256 x ITEMS keys; the layout's sort tiles must be cut to that size). FIRST:
// payload = source index.
// LAST: also writes the inverse permutation inv[payload] = destination when
// inv_out is given (central-particle tracking).
// hist: [slots][kSortPasses][256] digit counts of each galaxy; lookback: [sort tiles][256];
// st: per-slot states (error word).
// spin_limit: look-back iterations without progress before the tile gives up
// (kSpinLimit in production). withhold: a tile that never publishes its digit
// counts (kNoTile in production); the failure-detection tests set it so that
// the successors' waits run out and raise GS_DERR_LOOKBACK.
constexpr uint32_t kNoTile = 0xffffffffu;
template <bool FIRST, bool LAST, int ITEMS = kSortItems>
__global__ void __launch_bounds__(kSortThreads)
    onesweep_pass(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                  uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out,
                  uint32_t* __restrict__ inv_out, const uint32_t* __restrict__ hist, int pass,
                  uint32_t* lookback, uint32_t* tile_counter, Layout L, DevState* st,
                  uint32_t spin_limit = kSpinLimit, uint32_t withhold = kNoTile) {
  griddep_wait();  // launched with a programmatic dependency: predecessors' writes first
  constexpr int kTileKeys = kSortThreads * ITEMS;
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_warp[kSortWarps][256];
  __shared__ uint32_t s_prefix[256];  // global start of each digit's run, minus its tile-local start
  __shared__ uint32_t s_local[256];   // tile-local start of each digit's run
  __shared__ uint32_t s_scan[kSortWarps], s_tscan[kSortWarps];
  // the tile in output order (passes before the last; the last pass's digit, the
  // code's top six bits, takes few values in a tile, so its runs are long and it
  // scatters directly)
  constexpr int kStage = LAST ? 1 : kTileKeys;
  __shared__ uint32_t s_key[kStage], s_val[kStage];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int shift = 8 * pass;
  if (tid == 0) s_tile = atomicAdd(tile_counter, 1u);
  for (int i = tid; i < kSortWarps * 256; i += kSortThreads) (&s_warp[0][0])[i] = 0;
  __syncthreads();
  const uint32_t tile = s_tile;
  if (tile >= L.sort_tiles) return;  // the grid is sized to the tile count
  const uint32_t seg = L.seg_of_sort_tile[tile];
  const SegDesc sd = L.segs[seg];
  DevState* sst = st + sd.slot;
  const uint32_t lt = tile - sd.sort_tile0;  // tile index within the galaxy
  const uint32_t seg_end = sd.off + sd.n;
  const uint32_t base = sd.off + lt * kTileKeys + warp * (kTileKeys / kSortWarps);

  uint32_t key[ITEMS], val[ITEMS], rank[ITEMS];
#pragma unroll
  for (int k = 0; k < ITEMS; k++) {
    const uint32_t idx = base + k * 32 + lane;
    if (idx < seg_end) {
      key[k] = keys_in[idx];
      val[k] = FIRST ? idx : vals_in[idx];
    } else {
      key[k] = 0xffffffffu;
      val[k] = 0;
    }
  }
  const unsigned lt_mask = (1u << lane) - 1u;
#pragma unroll
  for (int k = 0; k < ITEMS; k++) {
    const bool valid = base + k * 32 + lane < seg_end;
    const uint32_t d = (key[k] >> shift) & 255u;
    const unsigned peers = __match_any_sync(0xffffffffu, valid ? d : 0x100u + lane);
    const uint32_t before = valid ? s_warp[warp][d] : 0u;
    rank[k] = before + __popc(peers & lt_mask);
    __syncwarp();
    if (valid && (__ffs(peers) - 1) == lane) s_warp[warp][d] = before + __popc(peers);
    __syncwarp();
  }
  __syncthreads();

  // Per digit: exclusive scan over warps (stable order warp 0..7) and tile total.
  const uint32_t d = tid;  // kSortThreads == 256 digits
  uint32_t tot = 0;
#pragma unroll
  for (int w = 0; w < kSortWarps; w++) {
    const uint32_t c = s_warp[w][d];
    s_warp[w][d] = tot;
    tot += c;
  }
  // The galaxy's exclusive offset of digit d (block-wide scan of its histogram).
  // Also the tile-local start of digit d (a scan of the tile's own counts).
  const uint32_t h = hist[((size_t)sd.slot * kSortPasses + pass) * 256 + d];
  uint32_t incl = h, tincl = tot;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    const uint32_t u = __shfl_up_sync(0xffffffffu, tincl, o);
    if (lane >= o) {
      incl += t;
      tincl += u;
    }
  }
  if (lane == 31) {
    s_scan[warp] = incl;
    s_tscan[warp] = tincl;
  }
  __syncthreads();
  uint32_t wpre = 0, twpre = 0;
  for (int w = 0; w < warp; w++) {
    wpre += s_scan[w];
    twpre += s_tscan[w];
  }
  const uint32_t gexcl = sd.off + wpre + incl - h;
  const uint32_t tlocal = twpre + tincl - tot;
  s_local[d] = tlocal;

  uint32_t* lb = lookback + (size_t)tile * 256;
  const bool publish = tile != withhold;
  uint32_t excl;
  if (lt == 0) {
    excl = gexcl;
    if (publish) st_relaxed(&lb[d], kLbInc | (gexcl + tot));
  } else {
    if (publish) st_relaxed(&lb[d], kLbAgg | tot);
    excl = 0;
    int64_t t = (int64_t)lt - 1;  // predecessors within the galaxy
    uint32_t spins = 0;
    bool done = false;
    while (t >= 0 && !done) {
      // look at up to 32 predecessors at once (independent loads in flight)
      constexpr int kWin = 32;
      uint32_t v[kWin];
#pragma unroll
      for (int k = 0; k < kWin; k++)
        v[k] = (t - k >= 0) ? ld_relaxed(lookback + (size_t)(sd.sort_tile0 + t - k) * 256 + d)
                            : kLbInc;
      int used = 0;
#pragma unroll
      for (int k = 0; k < kWin; k++) {
        if (used < k) break;  // an earlier entry was not published yet
        const uint32_t flag = v[k] & ~kLbMask;
        if (flag == 0) break;  // not published yet: reload from here
        excl += v[k] & kLbMask;
        used = k + 1;
        if (flag == kLbInc) {
          done = true;
          break;
        }
      }
      t -= used;
      if (!done && used == 0 && ++spins > spin_limit) {
        raise_err(sst, GS_DERR_LOOKBACK);
        break;
      }
    }
    if (publish) st_relaxed(&lb[d], kLbInc | ((excl + tot) & kLbMask));
  }
  s_prefix[d] = excl - tlocal;  // unsigned wrap: global position = local position + this
  __syncthreads();

  if (LAST) {  // direct scatter
#pragma unroll
    for (int k = 0; k < ITEMS; k++) {
      if (base + k * 32 + lane < seg_end) {
        const uint32_t dd = (key[k] >> shift) & 255u;
        const uint32_t pos = s_prefix[dd] + s_local[dd] + s_warp[warp][dd] + rank[k];
        if (pos < sd.off || pos >= seg_end) {  // only after a failed look-back: flag, never write
          raise_err(sst, GS_DERR_LOOKBACK);
          continue;
        }
        keys_out[pos] = key[k];
        vals_out[pos] = val[k];
        if (inv_out) inv_out[val[k]] = pos;
      }
    }
  } else {
    // Scatter through shared memory: each key goes to its tile-local output
    // position first, then consecutive threads write consecutive positions of each
    // digit's run to global memory (the same positions as a direct scatter).
#pragma unroll
    for (int k = 0; k < ITEMS; k++) {
      if (base + k * 32 + lane < seg_end) {
        const uint32_t dd = (key[k] >> shift) & 255u;
        const uint32_t lp = s_local[dd] + s_warp[warp][dd] + rank[k];
        s_key[lp] = key[k];
        s_val[lp] = val[k];
      }
    }
    __syncthreads();
    const uint32_t tile_beg = sd.off + lt * kTileKeys;
    const uint32_t nkeys = min((uint32_t)kTileKeys, seg_end - tile_beg);
    for (uint32_t j = tid; j < nkeys; j += kSortThreads) {
      const uint32_t kk = s_key[j], vv = s_val[j];
      const uint32_t pos = j + s_prefix[(kk >> shift) & 255u];
      if (pos < sd.off || pos >= seg_end) {  // only after a failed look-back: flag, never write
        raise_err(sst, GS_DERR_LOOKBACK);
        continue;
      }
      keys_out[pos] = kk;
      vals_out[pos] = vv;
    }
  }
}

}  // namespace gs

// Breadth-first bucketed octree on the device, bit-exact with MortonTree.build
// (src/physics/mortonTree.js:107-182), without level-synchronous launches.
//
// For sorted 30-bit codes c[0..N), let cpd(a, b) be the number of leading
// 3-bit digits a and b share (10 if equal). The reference's BFS has these
// closed forms, which the kernels below evaluate per particle:
//   * particle i starts a new depth-d group iff d >= D(i), with D(0) = 0 and
//     D(i) = cpd(c[i-1], c[i]) + 1 (11 = never);
//   * the depth-d group of i holds > 16 particles iff some j in [i-16, i] with
//     j + 16 < N has cpd(c[j], c[j+16]) >= d (sorted codes: a run of 17 equal
//     prefixes), so with M(i) = max of those cpd (or -1), the node of i at depth
//     d is internal iff d < min(10, M(i) + 1) =: L(i), its leaf depth
//     (count <= BUCKET || depth >= MAX_LEVEL, mortonTree.js:126);
//   * i therefore starts exactly the nodes at depths D(i)..L(i); BFS numbers
//     the nodes of a level in queue order, which is prefix order, so node
//     (d, i) has index levelStart(d) + #{j < i : D(j) <= d <= L(j)}.
// The third leaf clause of mortonTree.js:127 (numNodes + 8 > maxNodes) cannot
// fire for the reference's pool of 2N + 4096 nodes: a tree has at most N leaves
// and at most 10 * N / 17 internal nodes. The kernels flag a pool where it could.
//
// Every kernel works on a batch of galaxies: a build tile (1024 particles) lies
// inside one galaxy, each galaxy is numbered in its own node pool exactly as a
// solo build would number it, and node/particle indices in the arrays are pool
// indices (the galaxy's node_off / off added).
#pragma once
#include "common.cuh"
#include "morton.cuh"

#include <cuda/atomic>

namespace gs {

constexpr int kFlagThreads = 256;
constexpr int kFlagPer = 4;                          // consecutive particles per thread
constexpr int kFlagTile = kFlagThreads * kFlagPer;   // 1024 particles per block
constexpr int kCounters = 12;                        // depths 0..10 + leaf starts

// cpd of two codes: leading equal 3-bit digits (0..10).
__device__ inline int cpd(uint32_t a, uint32_t b) {
  const uint32_t x = a ^ b;
  if (x == 0) return 10;
  const int msb = 31 - __clz(x);  // 0..29 for 30-bit codes
  return (29 - msb) / 3;
}

struct BuildBuffers {
  const uint32_t* codes;  // sorted codes [pool]
  uint8_t* dl;            // packed D | L << 4 per particle [pool]
  uint32_t* blk_counts;   // [flag tiles][12]
  uint32_t* blk_offs;     // [flag tiles][12]
  TreeMeta* meta;         // [slots]
  uint32_t* node_start;   // [node pool] first particle of the node
  uint32_t* child_base;   // [node pool]
  int32_t* parent;        // [node pool]
  uint8_t* depth;         // [node pool]
  uint32_t* arrive;       // [node pool], zero between builds
  uint32_t* leaf_node;    // [pool] leaf nodes of a galaxy at [off, off + leaves)
  uint32_t* leaf_start;   // [pool]
  float4* cm;             // [node pool] com.xyz, mass
  WalkInfo* info;         // [node pool]
};

// K1: per particle D, L and per-tile start counts.
__global__ void __launch_bounds__(kFlagThreads) tree_flags_kernel(BuildBuffers b, Layout Lo) {
  griddep_wait();  // launched with a programmatic dependency: predecessors' writes first
  __shared__ uint32_t s_code[kFlagTile + 32];
  __shared__ int8_t s_cpd16[kFlagTile + 16];
  __shared__ uint32_t s_red[kFlagThreads / 32][kCounters];
  const int tid = threadIdx.x;
  const uint32_t tile = blockIdx.x;
  const SegDesc sd = Lo.segs[Lo.seg_of_flag_tile[tile]];
  const int64_t seg_beg = sd.off, seg_end = (int64_t)sd.off + sd.n;
  const int64_t base = seg_beg + (int64_t)(tile - sd.flag_tile0) * kFlagTile;
  // codes [base-16, base+tile+16) of this galaxy
  for (int k = tid; k < kFlagTile + 32; k += kFlagThreads) {
    const int64_t g = base - 16 + k;
    s_code[k] = (g >= seg_beg && g < seg_end) ? b.codes[g] : 0u;
  }
  __syncthreads();
  // cpd16(j) for j in [base-16, base+tile): -1 unless j and j + 16 are in the galaxy
  for (int k = tid; k < kFlagTile + 16; k += kFlagThreads) {
    const int64_t j = base - 16 + k;
    s_cpd16[k] = (j >= seg_beg && j + 16 < seg_end) ? (int8_t)cpd(s_code[k], s_code[k + 16])
                                                    : (int8_t)-1;
  }
  __syncthreads();
  uint32_t cnt[kCounters];
#pragma unroll
  for (int k = 0; k < kCounters; k++) cnt[k] = 0;
  uint32_t packed = 0;
#pragma unroll
  for (int q = 0; q < kFlagPer; q++) {
    const int loc = tid * kFlagPer + q;
    const int64_t i = base + loc;
    if (i >= seg_end) break;
    int D;
    if (i == seg_beg) {
      D = 0;
    } else {
      const uint32_t a = s_code[loc + 15], c = s_code[loc + 16];
      D = (a == c) ? 11 : cpd(a, c) + 1;
    }
    int M = -1;
#pragma unroll
    for (int w = 0; w <= 16; w++) M = max(M, (int)s_cpd16[loc + w]);  // j = i-16+w
    const int L = min(kMaxLevel, M + 1);
    packed |= (uint32_t)(D | (L << 4)) << (8 * q);
#pragma unroll
    for (int d = 0; d < kDepths; d++) cnt[d] += (D <= d && d <= L) ? 1u : 0u;
    cnt[11] += (D <= L) ? 1u : 0u;
  }
  // store packed bytes (4 consecutive particles per thread)
  const int64_t i0 = base + tid * kFlagPer;
  if (i0 < seg_end) {
    if (i0 + kFlagPer <= seg_end && (i0 & 3) == 0) {
      reinterpret_cast<uint32_t*>(b.dl)[i0 >> 2] = packed;
    } else {
      for (int q = 0; q < kFlagPer && i0 + q < seg_end; q++) b.dl[i0 + q] = (uint8_t)(packed >> (8 * q));
    }
  }
  const int warp = tid >> 5, lane = tid & 31;
#pragma unroll
  for (int k = 0; k < kCounters; k++) {
    const uint32_t v = __reduce_add_sync(0xffffffffu, cnt[k]);
    if (lane == 0) s_red[warp][k] = v;
  }
  __syncthreads();
  if (tid < kCounters) {
    uint32_t s = 0;
    for (int w = 0; w < kFlagThreads / 32; w++) s += s_red[w][tid];
    b.blk_counts[(size_t)tile * kCounters + tid] = s;
  }
}

// K2: one block per galaxy scans its tiles' counts and fills its TreeMeta.
// root size: the galaxy's Morton frame (frames != NULL) or root_size.
constexpr int kScanThreads = 1024;
__global__ void __launch_bounds__(kScanThreads)
    tree_scan_kernel(BuildBuffers b, Layout Lo, double root_size, const MortonFrame* frames,
                     DevState* st) {
  griddep_wait();  // launched with a programmatic dependency: predecessors' writes first
  __shared__ uint32_t s_warp[kScanThreads / 32][kCounters];
  __shared__ uint32_t s_tot[kCounters];
  const uint32_t seg = blockIdx.x;
  const SegDesc sd = Lo.segs[seg];
  const uint32_t t0 = sd.flag_tile0, ntiles = (sd.n + kFlagTile - 1) / kFlagTile;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t per = (ntiles + kScanThreads - 1) / kScanThreads;
  const uint32_t b0 = t0 + min(ntiles, tid * per), b1 = t0 + min(ntiles, tid * per + per);
  uint32_t sum[kCounters];
#pragma unroll
  for (int k = 0; k < kCounters; k++) sum[k] = 0;
  for (uint32_t x = b0; x < b1; x++)
#pragma unroll
    for (int k = 0; k < kCounters; k++) sum[k] += b.blk_counts[(size_t)x * kCounters + k];
  uint32_t excl[kCounters];
#pragma unroll
  for (int k = 0; k < kCounters; k++) {
    uint32_t inc = sum[k];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    excl[k] = inc - sum[k];
    if (lane == 31) s_warp[warp][k] = inc;
  }
  __syncthreads();
  if (tid < kCounters) {
    uint32_t run = 0;
    for (int w = 0; w < kScanThreads / 32; w++) {
      const uint32_t t = s_warp[w][tid];
      s_warp[w][tid] = run;
      run += t;
    }
    s_tot[tid] = run;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kCounters; k++) excl[k] += s_warp[warp][k];
  for (uint32_t x = b0; x < b1; x++)
#pragma unroll
    for (int k = 0; k < kCounters; k++) {
      const uint32_t c = b.blk_counts[(size_t)x * kCounters + k];
      b.blk_offs[(size_t)x * kCounters + k] = excl[k];
      excl[k] += c;
    }
  if (tid == 0) {
    TreeMeta m;
    uint32_t run = 0, levels = 0;
    for (int d = 0; d < kDepths; d++) {
      m.level_start[d] = run;
      m.level_count[d] = s_tot[d];
      run += s_tot[d];
      if (s_tot[d]) levels = d + 1;
    }
    m.level_start[kDepths] = run;
    m.level_count[kDepths] = 0;
    m.num_nodes = run;
    m.num_levels = levels;
    m.num_leaves = s_tot[11];
    m.overflow = run > sd.node_cap ? 1u : 0u;
    m.root_size = frames ? frames[sd.slot].size : root_size;
    b.meta[sd.slot] = m;
    if (m.overflow) raise_err(st + sd.slot, GS_DERR_NODES);
  }
}

// K3: node indices, parents, child bases, leaf lists.
__global__ void __launch_bounds__(kFlagThreads) tree_emit_kernel(BuildBuffers b, Layout Lo,
                                                                  DevState* st) {
  griddep_wait();  // launched with a programmatic dependency: predecessors' writes first
  __shared__ uint32_t s_warp[kFlagThreads / 32][kCounters];
  __shared__ TreeMeta s_meta;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t tile = blockIdx.x;
  const uint32_t seg = Lo.seg_of_flag_tile[tile];
  const SegDesc sd = Lo.segs[seg];
  const int64_t seg_end = (int64_t)sd.off + sd.n;
  const int64_t base = (int64_t)sd.off + (int64_t)(tile - sd.flag_tile0) * kFlagTile;
  if (tid == 0) s_meta = b.meta[sd.slot];
  uint8_t dl[kFlagPer];
  uint32_t cnt[kCounters];
#pragma unroll
  for (int k = 0; k < kCounters; k++) cnt[k] = 0;
#pragma unroll
  for (int q = 0; q < kFlagPer; q++) {
    const int64_t i = base + tid * kFlagPer + q;
    dl[q] = i < seg_end ? b.dl[i] : (uint8_t)0;
    const int D = dl[q] & 15, L = dl[q] >> 4;
    if (i < seg_end) {
#pragma unroll
      for (int d = 0; d < kDepths; d++) cnt[d] += (D <= d && d <= L) ? 1u : 0u;
      cnt[11] += (D <= L) ? 1u : 0u;
    }
  }
  uint32_t excl[kCounters];
#pragma unroll
  for (int k = 0; k < kCounters; k++) {
    uint32_t inc = cnt[k];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    excl[k] = inc - cnt[k];
    if (lane == 31) s_warp[warp][k] = inc;
  }
  __syncthreads();
  if (tid < kCounters) {
    uint32_t run = b.blk_offs[(size_t)tile * kCounters + tid];
    for (int w = 0; w < kFlagThreads / 32; w++) {
      const uint32_t t = s_warp[w][tid];
      s_warp[w][tid] = run;
      run += t;
    }
  }
  __syncthreads();
  if (s_meta.overflow) return;
#pragma unroll
  for (int k = 0; k < kCounters; k++) excl[k] += s_warp[warp][k];
  const uint32_t* LS = s_meta.level_start;
  const uint32_t no = sd.node_off;
#pragma unroll
  for (int q = 0; q < kFlagPer; q++) {
    const int64_t i = base + tid * kFlagPer + q;
    if (i >= seg_end) break;
    const int D = dl[q] & 15, L = dl[q] >> 4;
    for (int d = D; d <= L; d++) {
      const uint32_t nl = LS[d] + excl[d];  // index within the galaxy's tree
      const uint32_t n = no + nl;
      b.node_start[n] = (uint32_t)i;
      b.depth[n] = (uint8_t)d;
      // first depth-(d+1) node at or after particle i (children of n start here)
      b.child_base[n] = no + (d < kMaxLevel ? LS[d + 1] + excl[d + 1] : LS[kDepths]);
      // parent: the depth-(d-1) node containing i (inclusive count - 1)
      b.parent[n] = d == 0 ? -1
                           : (int32_t)(no + LS[d - 1] + excl[d - 1] +
                                       ((D <= d - 1 && d - 1 <= L) ? 1u : 0u) - 1u);
      if (d == L) {
        b.leaf_node[sd.off + excl[11]] = n;
        b.leaf_start[sd.off + excl[11]] = (uint32_t)i;
      }
      // mortonTree.js:127: an internal node with numNodes + 8 > maxNodes would be a leaf
      if (d < L && nl + 1 + 8 > sd.max_nodes) raise_err(st + sd.slot, GS_DERR_NODES);
    }
#pragma unroll
    for (int d = 0; d < kDepths; d++) excl[d] += (D <= d && d <= L) ? 1u : 0u;
    excl[11] += (D <= L) ? 1u : 0u;
  }
}

// COM precision modes of the leaves-up pass.
enum ComMode : int {
  kComF32 = 0,   // refresh_level arithmetic (nbody_bh.wgsl:289-313), FP32
  kComJs = 1,    // MortonTree.build arithmetic (mortonTree.js:130-137, :166-181), double
  kComF64 = 2,   // FP32 leaves, FP64 internal nodes (large-node reduction in double)
};

// K4: one thread per leaf slot (a block per build tile, kLeafThreads = one
// tile); leaf COM, then carry each finished node to its parent; the last child
// to finish sums the parent (children in slot order).
constexpr int kLeafThreads = kFlagTile;
constexpr int kComChunk = 8;  // leaf particles loaded per round trip
template <int MODE>
__global__ void __launch_bounds__(kLeafThreads)
    tree_leaves_kernel(BuildBuffers b, Layout Lo, const float4* __restrict__ pos,
                       uint32_t pos_stride, DevState* st) {
  griddep_wait();  // launched with a programmatic dependency: predecessors' writes first
  // the galaxy's level table (a block's tile lies in one galaxy), for child counts
  __shared__ uint32_t lvl_start[kDepths + 1], lvl_count[kDepths + 1];
  if (threadIdx.x <= kDepths) {
    const TreeMeta& m0 = b.meta[Lo.segs[Lo.seg_of_flag_tile[blockIdx.x]].slot];
    lvl_start[threadIdx.x] = m0.level_start[threadIdx.x];
    lvl_count[threadIdx.x] = m0.level_count[threadIdx.x];
  }
  __syncthreads();
  do {  // `continue` leaves the block's single iteration
    const uint32_t tile = blockIdx.x;
    const SegDesc sd = Lo.segs[Lo.seg_of_flag_tile[tile]];
    const uint32_t lr = (tile - sd.flag_tile0) * kFlagTile + threadIdx.x;  // leaf slot in the galaxy
    const uint32_t r = sd.off + lr;
    const TreeMeta& m = b.meta[sd.slot];
    if (m.overflow) continue;
    const uint32_t nleaves = m.num_leaves;
    if (lr >= nleaves) continue;
    const uint32_t seg_end = sd.off + sd.n;
    const uint32_t node_end = sd.node_off + m.num_nodes;
    uint32_t n = b.leaf_node[r];
    const uint32_t lo = b.leaf_start[r];
    const uint32_t hi = (lr + 1 < nleaves) ? b.leaf_start[r + 1] : seg_end;
    if (n < sd.node_off || n >= node_end || hi < lo || lo < sd.off || hi > seg_end) {
      raise_err(st + sd.slot, GS_DERR_NODES);  // impossible for a correct emit
      continue;
    }
    const int d = b.depth[n];
    int32_t p = b.parent[n];
    const float size = __double2float_rn(ldexp(m.root_size, -d));
    // particles in index order; each chunk's loads are issued together, so a
    // leaf of <= 16 particles costs two memory round trips instead of one per particle
    float4 c;
    if (MODE == kComJs) {
      double mm = 0, cx = 0, cy = 0, cz = 0;
      for (uint32_t j0 = lo; j0 < hi; j0 += kComChunk) {
        float4 q[kComChunk];
#pragma unroll
        for (int k = 0; k < kComChunk; k++)
          q[k] = j0 + k < hi ? pos[(size_t)(j0 + k) * pos_stride] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int k = 0; k < kComChunk; k++) {
          if (j0 + k >= hi) break;
          const double pm = q[k].w;
          mm = __dadd_rn(mm, pm);
          cx = __dadd_rn(cx, __dmul_rn((double)q[k].x, pm));
          cy = __dadd_rn(cy, __dmul_rn((double)q[k].y, pm));
          cz = __dadd_rn(cz, __dmul_rn((double)q[k].z, pm));
        }
      }
      const double inv = mm > 0 ? __ddiv_rn(1.0, mm) : 0.0;
      c = make_float4(__double2float_rn(__dmul_rn(cx, inv)), __double2float_rn(__dmul_rn(cy, inv)),
                      __double2float_rn(__dmul_rn(cz, inv)), __double2float_rn(mm));
    } else {
      float mm = 0, cx = 0, cy = 0, cz = 0;
      for (uint32_t j0 = lo; j0 < hi; j0 += kComChunk) {
        float4 q[kComChunk];
#pragma unroll
        for (int k = 0; k < kComChunk; k++)
          q[k] = j0 + k < hi ? pos[(size_t)(j0 + k) * pos_stride] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int k = 0; k < kComChunk; k++) {
          if (j0 + k >= hi) break;
          cx = fmaf(q[k].x, q[k].w, cx);
          cy = fmaf(q[k].y, q[k].w, cy);
          cz = fmaf(q[k].z, q[k].w, cz);
          mm += q[k].w;
        }
      }
      c = mm > 0.0f ? make_float4(cx / mm, cy / mm, cz / mm, mm) : make_float4(0.f, 0.f, 0.f, mm);
    }
    b.cm[n] = c;
    WalkInfo w;
    w.s2 = size * size;
    w.child = lo;
    w.info = kLeafBit | (hi - lo);
    w.size = size;
    b.info[n] = w;
    // carry upwards
    while (p >= 0) {
      const uint32_t up = (uint32_t)p;
      if (up >= n || up < sd.node_off) {  // parents precede children in BFS
        raise_err(st + sd.slot, GS_DERR_NODES);
        break;
      }
      // the parent's structure (read-only here), loads issued together; its child
      // range ends where the next node's begins, or at the end of the next level
      const int dp = b.depth[up];
      const uint32_t cb = b.child_base[up];
      const uint32_t cb1 = b.child_base[up + 1];  // up + 1 <= n: inside the galaxy's nodes
      const int32_t pp = b.parent[up];
      if (dp < 0 || dp >= kMaxLevel) {  // internal nodes lie at depths 0..9
        raise_err(st + sd.slot, GS_DERR_NODES);
        break;
      }
      const uint32_t next = (up - sd.node_off + 1 < lvl_start[dp] + lvl_count[dp])
                                ? cb1
                                : sd.node_off + lvl_start[dp + 1] + lvl_count[dp + 1];
      const uint32_t nc = next - cb;
      if (nc == 0 || nc > 8 || (uint64_t)cb + nc > node_end) {
        raise_err(st + sd.slot, GS_DERR_NODES);
        break;
      }
      // release: this node's COM is visible before the count; acquire: the last
      // arriver sees every sibling's COM
      const uint32_t old = cuda::atomic_ref<uint32_t, cuda::thread_scope_device>(b.arrive[up])
                               .fetch_add(1u, cuda::memory_order_acq_rel);
      if (old + 1 != nc) break;
      b.arrive[up] = 0;
      // the (at most 8) children's COMs, loads issued together, summed in slot order
      float4 q[8];
#pragma unroll
      for (int k = 0; k < 8; k++) q[k] = k < (int)nc ? __ldcg(&b.cm[cb + k]) : make_float4(0.f, 0.f, 0.f, 0.f);
      float4 pc;
      if (MODE == kComF32) {
        float mm = 0, cx = 0, cy = 0, cz = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) {
          if (k >= (int)nc) break;
          cx = fmaf(q[k].x, q[k].w, cx);
          cy = fmaf(q[k].y, q[k].w, cy);
          cz = fmaf(q[k].z, q[k].w, cz);
          mm += q[k].w;
        }
        pc = mm > 0.0f ? make_float4(cx / mm, cy / mm, cz / mm, mm) : make_float4(0.f, 0.f, 0.f, mm);
      } else {
        double mm = 0, cx = 0, cy = 0, cz = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) {
          if (k >= (int)nc) break;
          const double qm = q[k].w;
          mm = __dadd_rn(mm, qm);
          cx = __dadd_rn(cx, __dmul_rn((double)q[k].x, qm));
          cy = __dadd_rn(cy, __dmul_rn((double)q[k].y, qm));
          cz = __dadd_rn(cz, __dmul_rn((double)q[k].z, qm));
        }
        if (MODE == kComJs) {
          const double inv = mm > 0 ? __ddiv_rn(1.0, mm) : 0.0;
          pc = make_float4(__double2float_rn(__dmul_rn(cx, inv)),
                           __double2float_rn(__dmul_rn(cy, inv)),
                           __double2float_rn(__dmul_rn(cz, inv)), __double2float_rn(mm));
        } else {
          pc = mm > 0 ? make_float4(__double2float_rn(cx / mm), __double2float_rn(cy / mm),
                                    __double2float_rn(cz / mm), __double2float_rn(mm))
                      : make_float4(0.f, 0.f, 0.f, __double2float_rn(mm));
        }
      }
      const float psize = __double2float_rn(ldexp(m.root_size, -dp));
      b.cm[up] = pc;
      WalkInfo pw;
      pw.s2 = psize * psize;
      pw.child = cb;
      pw.info = nc;
      pw.size = psize;
      b.info[up] = pw;
      n = up;
      p = pp;
    }
  } while (0);
}

// BHNode materialisation of one galaxy (API only): the 64-byte layout of
// mortonTree.js:12-20 with indices local to the galaxy, as a solo build has them.
__global__ void tree_bhnode_kernel(BuildBuffers b, Layout Lo, uint32_t seg, gs_node* out) {
  const SegDesc sd = Lo.segs[seg];
  const TreeMeta m = b.meta[sd.slot];
  for (uint32_t nl = blockIdx.x * blockDim.x + threadIdx.x; nl < m.num_nodes; nl += gridDim.x * blockDim.x) {
    const uint32_t n = sd.node_off + nl;
    const float4 c = b.cm[n];
    const WalkInfo w = b.info[n];
    gs_node o;
    o.com[0] = c.x;
    o.com[1] = c.y;
    o.com[2] = c.z;
    o.mass = c.w;
    o.size = w.size;
    for (int k = 0; k < 8; k++) o.children[k] = -1;
    if (w.info & kLeafBit) {
      o.isLeaf = 1;
      o.first = w.child - sd.off;
      o.count = w.info & ~kLeafBit;
    } else {
      o.isLeaf = 0;
      o.first = 0;
      o.count = 0;
      const int shift = 27 - 3 * min((int)b.depth[n], 9);
      for (uint32_t k = 0; k < w.info && k < 8; k++) {
        const uint32_t ch = w.child + k;
        if (ch < sd.node_off || ch >= sd.node_off + m.num_nodes) break;
        const uint32_t ps = b.node_start[ch];
        if (ps < sd.off || ps >= sd.off + sd.n) break;
        const uint32_t oct = (b.codes[ps] >> shift) & 7u;
        o.children[oct] = (int32_t)(ch - sd.node_off);
      }
    }
    out[nl] = o;
  }
}

}  // namespace gs

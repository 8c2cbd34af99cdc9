// Barnes-Hut walk + Hernquist halo + kick-drift (+ star formation) on sm_100a.
//
// Semantics follow `main` in src/physics/shaders/nbody_bh.wgsl:64-181 per
// particle: own-leaf density, softened opening test
//   accept  <=>  size^2 < theta^2 (r^2 + eps^2)  ||  size^2 < eps^2 / 4,
// monopole G M r / (r^2 + eps^2)^(3/2), leaf direct sum with j != i, halo,
// v += a dt, gas drag, x += v dt, pad and specific-energy writes.
//
// Execution is warp-cooperative: a warp owns 32 Morton-consecutive particles
// (one per lane) and walks the union of their frontiers, but each lane applies
// exactly its own particle's acceptance decisions (a lane is active for a node
// only if it opened every ancestor), so the per-particle interaction set equals
// the reference's thread-per-particle stack walk.
//   * The stack holds child ranges (children of a BFS node are contiguous) with
//     the mask of lanes that opened the parent. Each round pops up to four
//     ranges and stages their children into shared memory by one coalesced load
//     (one child per lane, structure of arrays), so the round's stack, ballot and
//     staging work is shared by up to 32 children.
//   * Children are tested two at a time, and an opened leaf's particles are
//     staged the same way and summed two at a time, with sm_100's packed
//     FP32x2 FMA/ADD/MUL; accumulation is predicated, not branched (a child or
//     source a lane does not take gets r^2 + eps^2 = +inf, so rsqrt gives 0).
//     Walk groups of 16 or fewer stage a round's opened leaves back to back and
//     sum them in batches of 32 source pairs (see the leaf section).
//   * Warps are persistent and take work items from an atomic counter (load
//     balance across the dense core); per-item FP64 partials of the
//     diagnostics replace a block-wide barrier.
//   * Walk group size: a work item is 32, 16, 8 or 4 Morton-consecutive
//     particles (LPP = 1, 2, 4 or 8 lanes per particle). With LPP > 1 the lanes of a
//     particle split the round's slot pairs and each opened leaf's source pairs
//     between them and add their partial sums by shuffles at the end, so a
//     small galaxy keeps more warps busy and each warp walks the union of
//     fewer frontiers. A 32-particle walk group (layout, diagnostics) holds LPP
//     items. The split changes the order of the force sums, so results change
//     at the rounding level (inside the force tolerance) between group sizes;
//     each galaxy carries its own LPP, so it gets the same arithmetic alone or
//     in a pool.
//   * Over a batch, every group belongs to one galaxy and walks that galaxy's
//     tree with its own Params; warps steal groups across all galaxies.
//   * Walk split (one galaxy): a small galaxy's walk is as long as its densest
//     work item. With wsplit = S > 1 each item is walked by S warps over
//     disjoint parts of the tree (the nodes of one level dealt out in turn, with
//     their subtrees; the levels above belong to part 0), and the last of the S
//     to finish adds their sums in part order and integrates. Every interaction
//     happens once, as in the unsplit walk; only the order of the sums changes.
#pragma once
#include "common.cuh"

namespace gs {

constexpr int kWalkThreads = 128;
constexpr int kWalkWarps = kWalkThreads / 32;
constexpr int kPartials = 6;  // e_diag, e_true, px, py, pz, mass
#ifndef GS_WALK_RANGES
#define GS_WALK_RANGES 4
#endif
constexpr int kWalkRanges = GS_WALK_RANGES;  // child ranges popped and tested per round (1..4)
static_assert(kWalkRanges >= 1 && kWalkRanges <= 4, "a round stages at most one child per lane");
// ranges; a round explores kWalkRanges paths, each leaving <= 7 pending ranges per depth
constexpr int kWalkStack = 8 * 11 * kWalkRanges;
// The walk is compiled twice: for 8 resident blocks per SM (64 registers per
// thread) and for 7 (72 registers, fewer spills); the launch tuning picks one.
constexpr int kWalkBlocksPerSM = 8;
constexpr int kWalkBlocksWide = 7;
constexpr uint32_t kWalkGroup = 32;             // particles per walk group (layout, diagnostics)
constexpr uint32_t kWalkParts = 8;              // partial-sum slots per walk group (the largest LPP)
// with the walk group chosen by size, galaxies of at most this many particles
// walk in groups of 8 / 16 particles (measured crossovers of the step time on a
// B200 with the split below: 8 is fastest up to 32768 particles, 16 at 65536,
// 16 and 32 tie at 131072, 32 from 150000 on)
constexpr uint32_t kWalkAuto8 = 45000;
constexpr uint32_t kWalkAuto16 = 100000;
// a split walk splits at the first tree level of at least this many nodes per split
constexpr uint32_t kSplitMinNodes = 4;
// with the walk split chosen by size, a lone galaxy of at most this many
// particles walks each work item in 4 / 2 parts (measured: 4 parts fastest at
// 4096-8192 particles, 2 and 4 tie at 16384, none from 32768 on)
constexpr uint32_t kSplitAuto4 = 12000;
constexpr uint32_t kSplitAuto2 = 24000;

// nbody_bh.wgsl:206-213
__device__ inline uint32_t pcg(uint32_t v0) {
  uint32_t v = v0 * 747796405u + 2891336453u;
  v = ((v >> ((v >> 28u) + 4u)) ^ v) * 277803737u;
  return (v >> 22u) ^ v;
}
__device__ inline float rand01(uint32_t i, uint32_t salt) {
  return __fdiv_rn(__uint2float_rn(pcg(i ^ (salt * 0x9E3779B9u))), 4294967296.0f);
}
// nbody_bh.wgsl:216-227 (Kroupa inverse CDF)
__device__ inline float imf_sample(float u1, float u2) {
  const float a0 = powf(0.08f, -0.3f), b0 = powf(0.5f, -0.3f);
  const float lowInt = __fdiv_rn(__fsub_rn(a0, b0), 0.3f);
  const float a1 = powf(0.5f, -1.3f), b1 = powf(100.0f, -1.3f);
  const float hiInt = __fdiv_rn(__fmul_rn(0.5f, __fsub_rn(a1, b1)), 1.3f);
  if (u1 < __fdiv_rn(lowInt, __fadd_rn(lowInt, hiInt)))
    return powf(__fsub_rn(a0, __fmul_rn(u2, __fsub_rn(a0, b0))), -1.0f / 0.3f);
  return powf(__fsub_rn(a1, __fmul_rn(u2, __fsub_rn(a1, b1))), -1.0f / 1.3f);
}
__device__ inline uint32_t wgsl_u32(float x) {
  if (!(x > 0.0f)) return 0u;
  if (x >= 4294967296.0f) return 0xffffffffu;
  return (uint32_t)x;
}

// star_formation (nbody_bh.wgsl:229-268) on one particle, in registers.
// p1 = (vel, pad), s = stellar record.
__device__ inline void star_formation_one(const gs_params& P, uint32_t i, float4& p1, float4& s) {
  const uint32_t salt = wgsl_u32(__fmul_rn(P.time, 977.0f)) + 1u;
  if (p1.w < -0.5f) {
    const float density = __fsub_rn(-p1.w, 1.0f);
    if (density > P.sfDensity && P.sfEff > 0.0f) {
      const float prob = __fmul_rn(__fmul_rn(P.sfEff, P.sfDt),
                                   fminf(__fsqrt_rn(__fdiv_rn(density, fmaxf(P.sfDensity, 1e-6f))), 3.0f));
      if (rand01(i, salt) < prob) {
        const float m = imf_sample(rand01(i, salt + 7u), rand01(i, salt + 13u));
        s = make_float4(m, __fmul_rn(P.time, P.agingRate), rand01(i, salt + 29u), 0.0f);
        p1.w = 0.0f;
      }
    }
  } else if (s.x >= 8.0f) {
    const float ageMyr = __fsub_rn(__fmul_rn(P.time, P.agingRate), s.y);
    const float tMS = __fmul_rn(10000.0f, powf(s.x, -2.5f));
    const float tGiant = __fadd_rn(__fmul_rn(tMS, 0.12f), 15.0f);
    if (ageMyr > __fadd_rn(__fadd_rn(__fadd_rn(tMS, tGiant), 15.0f), 30.0f)) {
      s = make_float4(-1.0f, 0.0f, s.z, 0.7f);
      p1.w = -1.0f;
      p1.x = __fadd_rn(p1.x, __fmul_rn(__fsub_rn(rand01(i, salt + 41u), 0.5f), 2.0f));
      p1.y = __fadd_rn(p1.y, __fmul_rn(__fsub_rn(rand01(i, salt + 43u), 0.5f), 2.0f));
      p1.z = __fadd_rn(p1.z, __fmul_rn(__fsub_rn(rand01(i, salt + 47u), 0.5f), 2.0f));
    }
  }
}

struct WalkArgs {
  const float4* __restrict__ pin;   // 2 float4 per particle, tree (sorted) order
  float4* __restrict__ pout;
  float4* __restrict__ stellar;     // in place, used when SF is fused
  const float4* __restrict__ cm;    // node com.xyz, mass
  const WalkInfo* __restrict__ info;
  DevState* st;                     // per-slot states
  float* __restrict__ energy;       // e_i
  float4* __restrict__ dbg_acc;     // optional {ax, ay, az, phi} (G applied)
  float* __restrict__ dbg_dens;
  double* __restrict__ partials;    // [walk items][kPartials], a galaxy's from its SegDesc item0
  unsigned* work;                   // [0] next group, [1] finished warps (self-resetting)
  Layout L;                         // galaxies and the group -> galaxy map
  uint32_t pool_n, node_pool;       // particle and node pool sizes (memory-safety bounds)
  SegDesc seg0;                     // the only galaxy, for the one-galaxy instantiation
  // split walks (one galaxy, seg0.wsplit > 1): the tree levels of the split, the
  // per-split partial sums [3][wsplit][split_stride] (float4: ax pair, ay pair;
  // az pair, potential pair; density, self weight) and the arrivals per work item
  const TreeMeta* meta;
  float4* split_buf;
  unsigned* split_arrive;           // zero between launches (the last arrival resets it)
  uint32_t split_stride;
};

// Per-warp shared staging.
struct WalkSmem {
  uint2 stack[kWalkStack];          // {first child | (count-1) << 29, lane mask}
  // staged child ranges, pair-interleaved so a packed test reads two 128-bit
  // words: cxy[4p..4p+3] = {x(2p), x(2p+1), y(2p), y(2p+1)}, czm likewise {z, m}
  __align__(16) float cxy[16 * kWalkRanges];
  __align__(16) float czm[16 * kWalkRanges];
  float cs2[8 * kWalkRanges];
  uint32_t cnode[8 * kWalkRanges];  // node index of each staged child
  uint4 cmeta[8 * kWalkRanges];     // {child, info, own-leaf size bits, massive}
  // staged leaf sources, pair-interleaved the same way (pairs 0..32)
  __align__(16) float lxy[136];
  __align__(16) float lzm[136];
  uint4 bl[32];  // a round's opened leaves: {first particle, count, opening mask, first pair}
};

// Direct sum of a staged leaf segment [off, off + k) for the lanes in `me`
// (nbody_bh.wgsl:117-131), used by walk groups of 32: two sources per packed
// step, up to kmax >= k (staged sources past a leaf's count are massless zeros).
// A particle served by LPP lanes splits the source pairs: lane `sub` takes pairs
// sub, sub + LPP, ... With soft (eps^2 a normal float) the self pair is included (zero
// force at r = 0) and its potential removed once at the end of the walk via
// selfw (counted by the lane whose share holds it); otherwise it is skipped per
// pair.
// Reciprocal square root for the walk's r^2 + eps^2, which is never subnormal
// (eps^2 is zero or at least the smallest normal float, and zero softening adds
// that smallest normal instead): the flush-to-zero form gives the same result as
// rsqrtf there and issues fewer instructions.
__device__ __forceinline__ float rsqrt_walk(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

template <int LPP, typename Smem>
__device__ __forceinline__ void leaf_sum(const Smem& S, uint32_t off, uint32_t k, uint32_t kmax, uint32_t jself,
                                         bool me, bool soft, float2 px, float2 py, float2 pz,
                                         float eps2, float2& ax, float2& ay, float2& az,
                                         float2& pt, float& selfw, unsigned long long& npair,
                                         bool dbg, uint32_t sub) {
  if (soft) {
    // a lane that did not open the leaf gets eps^2 = +inf: its r^2 + eps^2 is
    // +inf, rsqrt gives 0 and every term of the pair vanishes (r is finite)
    const float e2me = me ? eps2 : INFINITY;
    if (me && jself < k && ((jself >> 1) % LPP) == sub) selfw += 1.0f;
    for (uint32_t j = 2 * sub; j < kmax; j += 2 * LPP) {
      const float4 jxy = *reinterpret_cast<const float4*>(&S.lxy[2 * (off + j)]);
      const float4 jzm = *reinterpret_cast<const float4*>(&S.lzm[2 * (off + j)]);
      const float2 jx = make_float2(jxy.x, jxy.y), jy = make_float2(jxy.z, jxy.w);
      const float2 jz = make_float2(jzm.x, jzm.y), jm = make_float2(jzm.z, jzm.w);
      const float2 ex = __fadd2_rn(jx, px), ey = __fadd2_rn(jy, py), ez = __fadd2_rn(jz, pz);
      const float2 e2 = __ffma2_rn(ex, ex, __ffma2_rn(ey, ey, __ffma2_rn(ez, ez, make_float2(e2me, e2me))));
      const float2 ri = make_float2(rsqrt_walk(e2.x), rsqrt_walk(e2.y));
      const float2 mr = __fmul2_rn(jm, ri);
      const float2 ff = __fmul2_rn(__fmul2_rn(mr, ri), ri);
      ax = __ffma2_rn(ex, ff, ax);
      ay = __ffma2_rn(ey, ff, ay);
      az = __ffma2_rn(ez, ff, az);
      pt = __fadd2_rn(pt, mr);
      if (dbg && me) npair += (j < k && j != jself) + (j + 1 < k && j + 1 != jself);
    }
  } else {
    for (uint32_t j = 2 * sub; j < kmax; j += 2 * LPP) {
      const float4 jxy = *reinterpret_cast<const float4*>(&S.lxy[2 * (off + j)]);
      const float4 jzm = *reinterpret_cast<const float4*>(&S.lzm[2 * (off + j)]);
      const float2 jx = make_float2(jxy.x, jxy.y), jy = make_float2(jxy.z, jxy.w);
      const float2 jz = make_float2(jzm.x, jzm.y), jm = make_float2(jzm.z, jzm.w);
      const float2 ex = __fadd2_rn(jx, px), ey = __fadd2_rn(jy, py), ez = __fadd2_rn(jz, pz);
      const float2 e2 = __ffma2_rn(ex, ex, __ffma2_rn(ey, ey, __ffma2_rn(ez, ez, make_float2(eps2, eps2))));
      const bool u0 = me && j < k && j != jself;
      const bool u1 = me && j + 1 < k && j + 1 != jself;
      const float2 ri = make_float2(u0 ? rsqrt_walk(e2.x) : 0.0f, u1 ? rsqrt_walk(e2.y) : 0.0f);
      const float2 mr = __fmul2_rn(jm, ri);
      const float2 ff = __fmul2_rn(__fmul2_rn(mr, ri), ri);
      ax = __ffma2_rn(ex, ff, ax);
      ay = __ffma2_rn(ey, ff, ay);
      az = __ffma2_rn(ez, ff, az);
      pt = __fadd2_rn(pt, mr);
      if (dbg) npair += u0 + u1;
    }
  }
}

// Direct sums of one staged batch of leaf sources for walk groups of 16 or fewer
// (nbody_bh.wgsl:117-131): up to 32 source pairs, pair t pair-interleaved at
// lxy/lzm[4t..4t+3], each pair from one leaf (a leaf of odd count ends in a
// massless zero). A particle served by LPP lanes splits the pairs: lane `sub`
// takes pairs sub, sub + LPP, ... Bit LPP * kk of `pm` tells whether the
// particle opened the leaf of pair sub + LPP * kk.
// With soft (eps^2 a normal float) a pair the lane does not take gets eps^2 = +inf: r^2 +
// eps^2 is then +inf, rsqrt gives 0 and every term vanishes (r is finite); the
// self pair is included (zero force at r = 0) and its potential removed once at
// the end of the walk. Without softening the self pair (batch source `selfloc`)
// is skipped per pair. Pairs past nbp hold massless zeros and are never in pm.
template <int LPP, bool SOFT, typename Smem>
__device__ __forceinline__ void leaf_batch(const Smem& S, uint32_t nbp, uint32_t pm, uint32_t selfloc,
                                           float2 px, float2 py, float2 pz, float eps2, float2& ax,
                                           float2& ay, float2& az, float2& pt, uint32_t sub) {
  constexpr int NB = 32 / LPP;  // steps of a lane over a full batch
  const float* lx = &S.lxy[4 * sub];
  const float* lz = &S.lzm[4 * sub];
#pragma unroll
  for (int kk = 0; kk < NB; kk++) {
    if ((kk * LPP) % 4 == 0 && kk * LPP >= (int)nbp) break;  // one check per four pairs
    const float4 jxy = *reinterpret_cast<const float4*>(lx + 4 * LPP * kk);
    const float4 jzm = *reinterpret_cast<const float4*>(lz + 4 * LPP * kk);
    const float2 jx = make_float2(jxy.x, jxy.y), jy = make_float2(jxy.z, jxy.w);
    const float2 jz = make_float2(jzm.x, jzm.y), jm = make_float2(jzm.z, jzm.w);
    const float2 ex = __fadd2_rn(jx, px), ey = __fadd2_rn(jy, py), ez = __fadd2_rn(jz, pz);
    const bool me = (pm >> (LPP * kk)) & 1u;
    float2 ri;
    if (SOFT) {
      const float e2me = me ? eps2 : INFINITY;
      const float2 e2 = __ffma2_rn(ex, ex, __ffma2_rn(ey, ey, __ffma2_rn(ez, ez, make_float2(e2me, e2me))));
      ri = make_float2(rsqrt_walk(e2.x), rsqrt_walk(e2.y));
    } else {
      const uint32_t j2 = 2 * (sub + LPP * kk);  // the pair's first source in the batch
      const float2 e2 = __ffma2_rn(ex, ex, __ffma2_rn(ey, ey, __ffma2_rn(ez, ez, make_float2(eps2, eps2))));
      ri = make_float2(me && j2 != selfloc ? rsqrt_walk(e2.x) : 0.0f,
                       me && j2 + 1 != selfloc ? rsqrt_walk(e2.y) : 0.0f);
    }
    const float2 mr = __fmul2_rn(jm, ri);
    const float2 ff = __fmul2_rn(__fmul2_rn(mr, ri), ri);
    ax = __ffma2_rn(ex, ff, ax);
    ay = __ffma2_rn(ey, ff, ay);
    az = __ffma2_rn(ez, ff, az);
    pt = __fadd2_rn(pt, mr);
  }
}

__device__ inline float2 f2(float a) { return make_float2(a, a); }

// Kahan step on packed pairs: s + x with the lost low-order part kept in c
// (c holds the negated error; the compensated total is s - c).
__device__ __forceinline__ void kahan_add2(float2& s, float2& c, float2 x) {
  const float2 y = __ffma2_rn(c, f2(-1.0f), x);   // x - c
  const float2 t = __fadd2_rn(s, y);
  c = __ffma2_rn(y, f2(-1.0f), __ffma2_rn(s, f2(-1.0f), t));  // (t - s) - y
  s = t;
}

// All ones if a > b (ordered: NaN gives 0), else 0, as one compare-and-set.
__device__ inline uint32_t set_gt_mask(float a, float b) {
  uint32_t r;
  asm("set.gt.u32.f32 %0, %1, %2;" : "=r"(r) : "f"(a), "f"(b));
  return r;
}

// Transpose of the 32 x 32 bit matrix held one row per lane: afterwards bit j
// of lane i is bit i of lane j (five butterfly stages of 16, 8, 4, 2, 1 bits).
__device__ __forceinline__ uint32_t warp_transpose(uint32_t x, int lane) {
  const uint32_t m16 = 0x0000FFFFu, m8 = 0x00FF00FFu, m4 = 0x0F0F0F0Fu, m2 = 0x33333333u, m1 = 0x55555555u;
#pragma unroll
  for (int j = 16; j >= 1; j >>= 1) {
    const uint32_t m = j == 16 ? m16 : j == 8 ? m8 : j == 4 ? m4 : j == 2 ? m2 : m1;
    const uint32_t y = __shfl_xor_sync(0xffffffffu, x, j);
    x = (lane & j) ? ((x & ~m) | ((y >> j) & m)) : ((x & m) | ((y & m) << j));
  }
  return x;
}

// ONE: the layout holds a single galaxy, whose descriptor comes with the
// kernel parameters instead of a per-group lookup. COMP: far-field (monopole)
// contributions are accumulated with compensation, blocked by round: a round's
// terms (at most 32 per lane) are summed plainly and each round's sum is added to
// the particle's total with a Kahan step; near-field leaf sums add plainly into
// the same totals.
// MINB: resident blocks per SM the register budget is compiled for.
// LPP: lanes per particle (walk group of 32 / LPP particles); a launch walks the
// galaxies whose SegDesc wlpp field equals LPP and skips the others' work items.
template <bool SF, bool DBG, bool ONE, bool COMP, int MINB, int LPP>
__global__ void __launch_bounds__(kWalkThreads, MINB) walk_kernel(WalkArgs a) {
  static_assert(LPP == 1 || LPP == 2 || LPP == 4 || LPP == 8, "lanes per particle");
  constexpr uint32_t G = 32 / LPP;                         // particles per work item
  constexpr int NPP = 16 / LPP;                            // slot pairs a lane tests in a full round
  constexpr unsigned GMASK = G == 32 ? 0xffffffffu : (1u << G) - 1u;
  constexpr uint32_t kStride = LPP;                        // work items per walk group
  griddep_wait();  // launched with a programmatic dependency: predecessors' writes first
  __shared__ WalkSmem smem_all[kWalkWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t pl = lane % G;    // the lane's particle within the item
  const uint32_t sub = lane / G;   // its share of the slot pairs and leaf sources
  // slots whose pairs this lane tests: pairs sub, sub + LPP, ... (bits 2pp, 2pp + 1)
  const uint32_t mine = LPP == 1   ? 0xffffffffu
                        : LPP == 2 ? (0x33333333u << (2 * sub))
                        : LPP == 4 ? (0x03030303u << (2 * sub))
                                   : (0x00030003u << (2 * sub));
  WalkSmem& S = smem_all[warp];
  // splits per work item (1, 2, 4, 8): a lone galaxy walked in groups of 16 or
  // fewer (the 32-particle build, the large galaxies' walk, carries no split code)
  const uint32_t NS = ONE && LPP > 1 ? a.seg0.wsplit : 1u;
  const uint32_t nitems = a.L.groups * kStride * NS;
  const unsigned full = 0xffffffffu;

  while (true) {
    uint32_t c = 0;  // grab the next work item of the schedule
    if (lane == 0) c = atomicAdd(&a.work[0], 1u);
    c = __shfl_sync(full, c, 0);
    if (c >= nitems) break;
    const uint32_t ksp = c % NS, cq = c / NS;  // split ksp of work item cq
    const uint32_t gcur = cq / kStride, part = cq % kStride;
    const SegDesc sd = ONE ? a.seg0 : a.L.segs[a.L.seg_of_group[gcur]];
    if (!ONE && sd.wlpp != LPP) continue;  // a galaxy of another group size
    DevState* const sst = a.st + sd.slot;
    const gs_params& P = sst->p;  // read-only during the walk; fields loaded where used
    const float eps2p = __ldg(&P.epsilon2);
    const float theta2 = __ldg(&P.theta) * __ldg(&P.theta);
    const float qe2 = 0.25f * eps2p;
    // Self pairs may be summed and removed afterwards when softened. Softening below
    // the smallest normal float counts as none, so every r^2 + eps^2 below is a
    // normal number (or +inf, or NaN from non-finite input), for which the
    // flush-to-zero rsqrt gives the same result as the non-flushing one.
    const bool soft = eps2p >= 1.17549435e-38f;
    // Without softening a node test at r = 0 (a particle's own one-particle leaf)
    // would weigh rsqrt(0) = inf by 0 (NaN): the distances add the smallest
    // normal float instead, which moves no r^2 above 1e-30 by more than a
    // rounding step, and such a node is opened as before.
    const float eps2 = soft ? eps2p : 1.17549435e-38f;
    const uint32_t seg_end = sd.off + sd.n;
    const uint32_t gbeg = sd.off + (gcur - sd.group0) * kWalkGroup + part * G, gend = gbeg + G;
    const uint32_t i = gbeg + pl;
    const bool valid = i < seg_end;
    // Walk groups of 32 read the particle's record again for the integration at
    // the end, so only its negated position stays live through the walk (the
    // 64-register build then needs no spills; measured faster for pools, the
    // same for one large galaxy); smaller groups keep it (measured faster there).
    constexpr bool kReload = LPP == 1;
    float4 p0 = make_float4(0.f, 0.f, 0.f, 0.f), p1 = p0;
    if (valid) {
      p0 = a.pin[2 * (size_t)i];
      if (!kReload) p1 = a.pin[2 * (size_t)i + 1];
    }
    const float2 px = f2(-p0.x), py = f2(-p0.y), pz = f2(-p0.z);  // negated: r = q + (-p)
    float2 ax = f2(0.f), ay = f2(0.f), az = f2(0.f), pt = f2(0.f);
    float2 cax = f2(0.f), cay = f2(0.f), caz = f2(0.f), cpt = f2(0.f);  // COMP only
    float dens = 0.f, selfw = 0.f;
    unsigned long long nmono = 0, npair = 0, nvisit = 0;
    const unsigned all = __ballot_sync(full, valid) & GMASK;  // the item's particles (lanes of share 0)

    // Split walk: the first level of at least kSplitMinNodes nodes per split is
    // the split level; split k owns its nodes j with j = k mod NS (counted from
    // the level's start) and their subtrees, and split 0 also every contribution
    // of the levels above, which the other splits test (to reach their own
    // nodes) without adding.
    uint32_t up_end = 0u, win_end = 0u;
    bool idle = false;
    if (NS > 1) {
      const TreeMeta* m = a.meta + sd.slot;
      const uint32_t nl = min(m->num_levels, (uint32_t)kDepths);
      up_end = win_end = 0xffffffffu;
      for (uint32_t l = 1; l < nl; l++) {
        const uint32_t cnt = m->level_count[l];
        if (cnt >= kSplitMinNodes * NS) {
          up_end = sd.node_off + m->level_start[l];
          win_end = up_end + cnt;
          break;
        }
      }
      idle = ksp > 0 && up_end == 0xffffffffu;  // no such level: split 0 walks the whole tree
    }

    int sp = 0;
    if (lane == 0) S.stack[0] = make_uint2(sd.node_off, all);  // the root: range {node_off, 1}
    sp = idle ? 0 : 1;
    uint32_t budget = 4u * sd.node_cap + 1024u;
    while (sp > 0) {
      __syncwarp();
      // pop up to kWalkRanges ranges; their children are staged and tested together
      const int nr = min(sp, kWalkRanges);
      const int sp0 = sp;
      sp -= nr;
      uint32_t masks[kWalkRanges];  // lanes that opened each popped range's parent
#pragma unroll
      for (int r = 0; r < kWalkRanges; r++) masks[r] = r < nr ? S.stack[sp0 - 1 - r].y : 0u;
      if (--budget == 0) {
        if (lane == 0) raise_err(sst, GS_DERR_STACK);
        break;
      }
      // Stage range r in lanes 8r..8r+7: one child per lane; slots past a range's
      // count hold massless dummies. Massless and sub-softening children
      // (size^2 < eps^2/4, always accepted, nbody_bh.wgsl:112) get size^2 = -inf,
      // so the per-lane test is the single compare size^2 < theta^2 (r^2 + eps^2).
      bool own = false, isleaf = false, massive = false, skip = false;
      if (lane < 8 * kWalkRanges) {
        const int r = lane >> 3;
        const uint32_t c = lane & 7;
        const uint2 e = r < nr ? S.stack[sp0 - 1 - r] : make_uint2(0u, 0u);
        const uint32_t rs = e.x & 0x1fffffffu, rc = r < nr ? (e.x >> 29) + 1u : 0u;
        float4 q = make_float4(1e30f, 1e30f, 1e30f, 0.f);
        WalkInfo w;
        w.s2 = 0.f;
        w.child = 0;
        w.info = kLeafBit;
        w.size = 1.f;
        bool real = c < rc, counted = true;
        if (NS > 1 && real) {
          const uint32_t node = rs + c;
          if (node < up_end) counted = ksp == 0;                                    // levels above the split
          else if (node < win_end && ((node - up_end) & (NS - 1)) != ksp) real = false;  // another split's
        }
        if (real) {
          q = __ldg(&a.cm[rs + c]);
          w = a.info[rs + c];
        }
        const uint32_t wc = w.info & ~kLeafBit;
        isleaf = real && (w.info & kLeafBit);
        massive = real && q.w != 0.0f && counted;
        skip = isleaf && !counted;
        own = isleaf && q.w != 0.0f && w.child < gend && w.child + wc > gbeg;
        float s2 = w.s2;
        if (q.w == 0.0f) {  // never opened, contributes nothing (far away, massless)
          s2 = -INFINITY;
          q = make_float4(1e30f, 1e30f, 1e30f, 0.f);
        } else if (s2 < qe2) {
          s2 = -INFINITY;
        }
        const int st = 4 * (lane >> 1) + (lane & 1);
        S.cxy[st] = q.x;
        S.cxy[st + 2] = q.y;
        S.czm[st] = q.z;
        S.czm[st + 2] = counted ? q.w : 0.0f;  // tested for opening, adds nothing
        S.cs2[lane] = s2;
        S.cnode[lane] = rs + c;
        S.cmeta[lane] = make_uint4(w.child, w.info,
                                   own ? __float_as_uint(w.size) : 0u,
                                   massive ? 1u : 0u);
      }
      const unsigned ownmask = __ballot_sync(full, own);  // leaves holding our particles
      const unsigned leafmask = __ballot_sync(full, isleaf);
      const unsigned massmask = DBG ? __ballot_sync(full, massive) : 0u;
      const unsigned skipm = NS > 1 ? __ballot_sync(full, skip) : 0u;  // opened leaves another split sums
      __syncwarp();
      // per range: this lane active; the slots whose open bits this lane keeps (its
      // active ranges' eight slots: a slot past a range's count holds a dummy of
      // size^2 -inf, which every active lane accepts, so it never sets an open bit)
      uint32_t actbits = 0, keep = 0;
#pragma unroll
      for (int r = 0; r < kWalkRanges; r++) {
        const uint32_t a_r = (masks[r] >> pl) & 1u;
        actbits |= a_r << r;
        keep |= a_r ? 0xffu << (8 * r) : 0u;
      }
      keep &= mine;
      // theta^2 per range; a lane inactive for a range tests against -inf, so its
      // td is -inf (or NaN) and it accepts and adds nothing there
      float th2[kWalkRanges];
#pragma unroll
      for (int r = 0; r < kWalkRanges; r++) th2[r] = (actbits >> r) & 1u ? theta2 : -INFINITY;
      uint32_t obits = 0;  // children this lane opens (active, not accepted), bit = slot
      // COMP: the round's far-field terms (at most 32 per lane) are summed plainly,
      // then the round's sum joins the particle's total in one Kahan step
      float2 rax = f2(0.f), ray = f2(0.f), raz = f2(0.f), rpt = f2(0.f);
#pragma unroll
      for (int kk = 0; kk < NPP; kk++) {
        // a range's pairs are tested only if the range was popped (one check per range)
        if ((kk * LPP) % 4 == 0 && kk * LPP >= 4 * nr) break;
        const int pp = (int)sub + kk * LPP;
        const int c = 2 * pp;
        // the pair's range pp >> 2: (kk * LPP) >> 2 for shares below 4, one more above
        const float t2 = LPP < 8 ? th2[(kk * LPP) >> 2] : (sub >= 4 ? th2[2 * kk + 1] : th2[2 * kk]);
        const float4 qxy = *reinterpret_cast<const float4*>(&S.cxy[2 * c]);
        const float4 qzm = *reinterpret_cast<const float4*>(&S.czm[2 * c]);
        const float2 qx = make_float2(qxy.x, qxy.y), qy = make_float2(qxy.z, qxy.w);
        const float2 qz = make_float2(qzm.x, qzm.y), qm = make_float2(qzm.z, qzm.w);
        const float2 s2 = *reinterpret_cast<const float2*>(&S.cs2[c]);
        const float2 rx = __fadd2_rn(qx, px), ry = __fadd2_rn(qy, py), rz = __fadd2_rn(qz, pz);
        const float2 d2 = __ffma2_rn(rx, rx, __ffma2_rn(ry, ry, __ffma2_rn(rz, rz, f2(eps2))));
        const float2 td = __fmul2_rn(f2(t2), d2);
        // all ones where the child is accepted; an accepted child keeps r^2 + eps^2,
        // any other gets +inf, so rsqrt makes its terms exactly 0
        const uint32_t ax_ = set_gt_mask(td.x, s2.x), ay_ = set_gt_mask(td.y, s2.y);
        obits |= (~ax_ & (1u << c)) | (~ay_ & (2u << c));
        const float2 dsel = make_float2(__uint_as_float((__float_as_uint(d2.x) & ax_) | (0x7f800000u & ~ax_)),
                                        __uint_as_float((__float_as_uint(d2.y) & ay_) | (0x7f800000u & ~ay_)));
        const float2 rinv = make_float2(rsqrt_walk(dsel.x), rsqrt_walk(dsel.y));
        const float2 mr = __fmul2_rn(qm, rinv);
        const float2 f = __fmul2_rn(__fmul2_rn(mr, rinv), rinv);
        if (COMP) {
          rax = __ffma2_rn(rx, f, rax);
          ray = __ffma2_rn(ry, f, ray);
          raz = __ffma2_rn(rz, f, raz);
          rpt = __fadd2_rn(rpt, mr);
        } else {
          ax = __ffma2_rn(rx, f, ax);
          ay = __ffma2_rn(ry, f, ay);
          az = __ffma2_rn(rz, f, az);
          pt = __fadd2_rn(pt, mr);  // sum of m/r; potential = -G * sum
        }
      }
      if (COMP) {
        kahan_add2(ax, cax, rax);
        kahan_add2(ay, cay, ray);
        kahan_add2(az, caz, raz);
        kahan_add2(pt, cpt, rpt);
      }
      obits &= keep;
      const uint32_t om = __reduce_or_sync(full, obits);  // children opened by some lane
      if (DBG) {  // keep holds this lane's slots only
        nvisit += __popc(massmask & keep);
        nmono += __popc(massmask & keep & ~obits);
      }
      for (uint32_t bb = ownmask; bb; bb &= bb - 1) {  // own-leaf density (nbody_bh.wgsl:93-95)
        const uint32_t cc = __ffs(bb) - 1;
        const uint4 mt = S.cmeta[cc];
        const uint32_t cnt = mt.y & ~kLeafBit;
        if (((actbits >> (cc >> 3)) & 1u) && (i - mt.x) < cnt) {
          const float sz = __uint_as_float(mt.z);
          dens = (float)cnt / (sz * sz * sz);
        }
      }
      if (!om) continue;
      // Every slot's open mask at once: lane c's col holds the lanes that open
      // slot c (the transpose of the 32 x 32 bit matrix whose rows are the lanes'
      // obits), so each slot's lane can act on its own child in parallel. Only
      // the share that tests slot c has its bits: shifted down, they are the
      // item's particle mask.
      const uint32_t col = (warp_transpose(obits, lane) >> ((((uint32_t)lane >> 1) % LPP) * G)) & GMASK;
      // opened internal children: each slot's lane writes its child range and open
      // mask to the stack, in slot order (prefix positions)
      const uint32_t pushc = om & ~leafmask;
      if (pushc) {
        bool ok = false;
        uint2 ent = make_uint2(0u, 0u);
        if ((pushc >> lane) & 1u) {
          const uint4 mt = S.cmeta[lane];
          const uint32_t cchild = mt.x, ccnt = mt.y & ~kLeafBit;
          // a galaxy's child ranges stay in its node range by construction (build,
          // upload check); the walk itself only guards the pool bounds
          ok = cchild > S.cnode[lane] && (uint64_t)cchild + ccnt <= a.node_pool && ccnt >= 1u && ccnt <= 8u;
          if (!ok) raise_err(sst, GS_DERR_TREE);
          ent = make_uint2(cchild | ((ccnt - 1u) << 29), col);
        }
        const uint32_t okm = __ballot_sync(full, ok);
        const int pos = sp + __popc(okm & ((1u << lane) - 1u));
        if (ok && pos < kWalkStack) S.stack[pos] = ent;
        const int np = __popc(okm);
        if (sp + np > kWalkStack && lane == 0) raise_err(sst, GS_DERR_STACK);  // not for depth <= 10 trees
        sp = min(sp + np, kWalkStack);
      }
      // Opened leaves: direct sums, two sources at a time.
      const uint32_t leafc = om & leafmask & ~skipm;
      // Walk groups of 32: leaves of <= 16 particles get their batch entries from
      // their slots' lanes and are staged four per batch (one load round), each in
      // a block of 16 sources; larger ones go in chunks of 32.
      uint32_t big = 0;
      if (LPP == 1 && leafc) {
        bool sm = false, bg = false;
        uint4 ent = make_uint4(0u, 0u, 0u, 0u);
        if ((leafc >> lane) & 1u) {
          const uint4 mt = S.cmeta[lane];
          const uint32_t ccnt = mt.y & ~kLeafBit;
          if ((uint64_t)mt.x + ccnt > a.pool_n) {
            raise_err(sst, GS_DERR_TREE);
          } else {
            bg = ccnt > 16u;
            sm = !bg;
            ent = make_uint4(mt.x, ccnt, col, 0u);
          }
        }
        const uint32_t smallm = __ballot_sync(full, sm);
        big = __ballot_sync(full, bg);
        __syncwarp();  // earlier leaf sums are done reading the batch entries
        if (sm) S.bl[__popc(smallm & ((1u << lane) - 1u))] = ent;
        const uint32_t nsmall = __popc(smallm);
        for (uint32_t b0 = 0; b0 < nsmall; b0 += 4) {
          const uint32_t nb = min(4u, nsmall - b0);
          __syncwarp();
#pragma unroll
          for (int r = 0; r < 2; r++) {
            const uint32_t e = lane + 32 * r, slot = e >> 4, q = e & 15u;
            if (slot < nb) {
              const uint4 bl = S.bl[b0 + slot];
              float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
              if (q < bl.y) v = __ldg(&a.pin[2 * (size_t)(bl.x + q)]);
              const uint32_t se = 4 * (e >> 1) + (e & 1);
              S.lxy[se] = v.x;
              S.lxy[se + 2] = v.y;
              S.lzm[se] = v.z;
              S.lzm[se + 2] = v.w;
            }
          }
          __syncwarp();
          for (uint32_t sl = 0; sl < nb; sl++) {
            const uint4 bl = S.bl[b0 + sl];
            leaf_sum<LPP>(S, 16 * sl, bl.y, bl.y, i - bl.x, (bl.z >> pl) & 1u, soft, px, py, pz, eps2, ax, ay,
                          az, pt, selfw, npair, DBG, sub);
          }
        }
      }
      for (uint32_t bb = big; bb; bb &= bb - 1) {
        const uint32_t cc = __ffs(bb) - 1;
        const unsigned open = __shfl_sync(full, col, cc);
        const uint4 mt = S.cmeta[cc];
        const uint32_t cchild = mt.x, ccnt = mt.y & ~kLeafBit;
        for (uint32_t b0 = 0; b0 < ccnt; b0 += 32) {
          const uint32_t k = min(32u, ccnt - b0);
          __syncwarp();
          float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
          if (lane < (int)k) v = __ldg(&a.pin[2 * (size_t)(cchild + b0 + lane)]);
          const int se = 4 * (lane >> 1) + (lane & 1);
          S.lxy[se] = v.x;
          S.lxy[se + 2] = v.y;
          S.lzm[se] = v.z;
          S.lzm[se + 2] = v.w;
          if (lane == 0) S.lxy[64] = S.lxy[66] = S.lzm[64] = S.lzm[66] = 0.f;  // source 32
          __syncwarp();
          leaf_sum<LPP>(S, 0, k, k, i - (cchild + b0), (open >> pl) & 1u, soft, px, py, pz, eps2, ax, ay,
                        az, pt, selfw, npair, DBG, sub);
        }
      }
      // Walk groups of 16 or fewer (a particle's pairs split over LPP lanes): the
      // round's opened leaves lie back to back in slot order in a space of source
      // pairs (leaf k at pairs [P_k, P_k + ceil(n_k / 2))), staged and summed in
      // batches of 32 pairs, so every lane's share of a batch is whole pairs of
      // leaf sources and no step is spent on a leaf's unused staging slots.
      if (LPP > 1 && leafc) {
        bool lf = false;
        uint32_t lfirst = 0, lcnt = 0, lnp = 0;
        if ((leafc >> lane) & 1u) {
          const uint4 mt = S.cmeta[lane];
          lfirst = mt.x;
          lcnt = mt.y & ~kLeafBit;
          if ((uint64_t)lfirst + lcnt > a.pool_n) {
            raise_err(sst, GS_DERR_TREE);
          } else {
            lf = lcnt > 0u;  // an empty leaf adds nothing
            lnp = (lcnt + 1u) >> 1;
          }
        }
        uint32_t incl = lnp;  // inclusive prefix of the pair counts over the slots
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t y = __shfl_up_sync(full, incl, o);
          if (lane >= o) incl += y;
        }
        const uint32_t P = incl - lnp, T = __shfl_sync(full, incl, 31);
        const uint32_t lfm = __ballot_sync(full, lf);
        // item particles that opened the leaf holding them (the self pair)
        uint32_t selfm = 0;
        if (lf) {
          const uint32_t lo = max(lfirst, gbeg), hi = min(lfirst + lcnt, gend);
          if (lo < hi) {
            const uint32_t b0 = lo - gbeg, b1 = hi - gbeg;  // item particle positions [b0, b1)
            selfm = col & ((b1 >= 32u ? 0xffffffffu : (1u << b1) - 1u) & ~((1u << b0) - 1u));
          }
        }
        const bool selfhit = (__reduce_or_sync(full, selfm) >> pl) & 1u;
        if (soft && sub == 0 && selfhit) selfw += 1.0f;
        __syncwarp();  // the previous round's batches are done reading the table and staging
        if (lf) S.bl[__popc(lfm & ((1u << lane) - 1u))] = make_uint4(lfirst, lcnt, col, P);
        __syncwarp();
        uint32_t selfsrc = 0xffffffffu;  // without softening: the self source in pair space
        if (DBG || !soft) {
          const uint32_t nl = __popc(lfm);
          for (uint32_t k = 0; k < nl; k++) {
            const uint4 L = S.bl[k];
            if ((L.z >> pl) & 1u) {
              const bool in = i - L.x < L.y;
              if (in) selfsrc = 2 * L.w + (i - L.x);
              if (DBG && sub == 0) npair += L.y - (in ? 1u : 0u);
            }
          }
        }
        for (uint32_t w0 = 0; w0 < T; w0 += 32) {
          // leaves starting in this batch's window of pairs, and those before it
          const uint32_t Wb = __reduce_or_sync(full, lf && P >= w0 && P - w0 < 32u ? 1u << (P - w0) : 0u);
          const uint32_t base = __popc(__ballot_sync(full, lf && P < w0));
          if (w0) __syncwarp();  // the previous batch's sums are done reading the staging
          // stage source e = lane + 32 r of the batch: pair t = e / 2 of leaf k
#pragma unroll
          for (int r = 0; r < 2; r++) {
            const uint32_t e = lane + 32 * r, t = e >> 1;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (w0 + t < T) {
              const uint4 L = S.bl[base + __popc(Wb & (0xffffffffu >> (31 - t))) - 1];
              const uint32_t q = 2 * (w0 + t - L.w) + (e & 1u);  // source within the leaf
              if (q < L.y) v = __ldg(&a.pin[2 * (size_t)(L.x + q)]);
            }
            const uint32_t se = 4 * t + (e & 1u);
            S.lxy[se] = v.x;
            S.lxy[se + 2] = v.y;
            S.lzm[se] = v.z;
            S.lzm[se + 2] = v.w;
          }
          // lane t answers for pair t: the item particles that opened its leaf
          // (copied to every share when LPP > 1); transposed, each lane holds the
          // pairs its particle takes part in
          uint32_t mt = 0;
          if (w0 + lane < T) mt = S.bl[base + __popc(Wb & (0xffffffffu >> (31 - lane))) - 1].z;
          if (LPP == 2) mt *= 0x00010001u;
          if (LPP == 4) mt *= 0x01010101u;
          if (LPP == 8) mt *= 0x11111111u;
          const uint32_t pm = warp_transpose(mt, lane) >> sub;
          const uint32_t nbp = min(32u, T - w0);
          __syncwarp();
          if (soft)
            leaf_batch<LPP, true>(S, nbp, pm, 0u, px, py, pz, eps2, ax, ay, az, pt, sub);
          else
            leaf_batch<LPP, false>(S, nbp, pm, selfsrc - 2 * w0, px, py, pz, eps2, ax, ay, az, pt, sub);
        }
      }
    }
    if (COMP) {  // fold the compensations into the sums
      ax = __ffma2_rn(cax, f2(-1.0f), ax);
      ay = __ffma2_rn(cay, f2(-1.0f), ay);
      az = __ffma2_rn(caz, f2(-1.0f), az);
      pt = __ffma2_rn(cpt, f2(-1.0f), pt);
    }
    if (LPP > 1) {  // add the shares of each particle (lanes pl, pl + G, ...), fixed order
#pragma unroll
      for (uint32_t o = G; o < 32; o <<= 1) {
        ax = __fadd2_rn(ax, make_float2(__shfl_xor_sync(full, ax.x, o), __shfl_xor_sync(full, ax.y, o)));
        ay = __fadd2_rn(ay, make_float2(__shfl_xor_sync(full, ay.x, o), __shfl_xor_sync(full, ay.y, o)));
        az = __fadd2_rn(az, make_float2(__shfl_xor_sync(full, az.x, o), __shfl_xor_sync(full, az.y, o)));
        pt = __fadd2_rn(pt, make_float2(__shfl_xor_sync(full, pt.x, o), __shfl_xor_sync(full, pt.y, o)));
        selfw += __shfl_xor_sync(full, selfw, o);
      }
    }
    if (DBG) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        nmono += __shfl_xor_sync(full, nmono, o);
        npair += __shfl_xor_sync(full, npair, o);
        nvisit += __shfl_xor_sync(full, nvisit, o);
      }
      if (lane == 0) {
        atomicAdd(&sst->counters[0], nmono);
        atomicAdd(&sst->counters[1], npair);
        atomicAdd(&sst->counters[2], nvisit);
      }
    }
    if (NS > 1) {
      // Each split leaves its sums in split_buf; the last split of the item to
      // arrive adds them in split order (the same sums whatever the arrival order)
      // and finishes the item. No split waits for another.
      const uint32_t li = i - sd.off;
      const size_t st = a.split_stride;
      float4* const B = a.split_buf;
      const float4 o0 = make_float4(ax.x, ax.y, ay.x, ay.y), o1 = make_float4(az.x, az.y, pt.x, pt.y);
      const float4 o2 = make_float4(dens, selfw, 0.f, 0.f);
      if (valid && sub == 0) {
        B[(size_t)ksp * st + li] = o0;
        B[(size_t)(NS + ksp) * st + li] = o1;
        B[(size_t)(2 * NS + ksp) * st + li] = o2;
      }
      __threadfence();
      __syncwarp();
      unsigned* const arrive = a.split_arrive + (size_t)(gcur - sd.group0) * kStride + part;
      unsigned prev = 0;
      if (lane == 0) prev = atomicAdd(arrive, 1u);
      prev = __shfl_sync(full, prev, 0);
      if (prev != NS - 1) continue;  // another split finishes this item
      __threadfence();
      if (lane == 0) *arrive = 0u;   // every split of the item has arrived: ready for the next launch
      if (valid && sub == 0) {
        float4 u0 = o0, u1 = o1, u2 = o2;
        for (uint32_t k = 0; k < NS; k++) {
          float4 v0 = o0, v1 = o1, v2 = o2;
          if (k != ksp) {
            v0 = __ldcg(B + (size_t)k * st + li);
            v1 = __ldcg(B + (size_t)(NS + k) * st + li);
            v2 = __ldcg(B + (size_t)(2 * NS + k) * st + li);
          }
          if (k == 0) {
            u0 = v0;
            u1 = v1;
            u2 = v2;
          } else {
            u0 = make_float4(u0.x + v0.x, u0.y + v0.y, u0.z + v0.z, u0.w + v0.w);
            u1 = make_float4(u1.x + v1.x, u1.y + v1.y, u1.z + v1.z, u1.w + v1.w);
            u2 = make_float4(fmaxf(u2.x, v2.x), u2.y + v2.y, 0.f, 0.f);  // the own leaf is found once or equal
          }
        }
        ax = make_float2(u0.x, u0.y);
        ay = make_float2(u0.z, u0.w);
        az = make_float2(u1.x, u1.y);
        pt = make_float2(u1.z, u1.w);
        dens = u2.x;
        selfw = u2.y;
      }
    }
    if (kReload && valid) {
      p0 = a.pin[2 * (size_t)i];
      p1 = a.pin[2 * (size_t)i + 1];
    }
    if (soft && selfw != 0.0f) pt.x -= selfw * p0.w * rsqrtf(eps2);

    double e_diag = 0, e_true = 0, mx = 0, my = 0, mz = 0, ms = 0;
    if (valid && sub == 0) {
      const float G = P.G;
      float fx = (ax.x + ax.y) * G, fy = (ay.x + ay.y) * G, fz = (az.x + az.y) * G;
      const float pot = -(pt.x + pt.y) * G;
      if (DBG) {
        a.dbg_acc[i] = make_float4(fx, fy, fz, pot);
        a.dbg_dens[i] = dens;
      }
      // Hernquist halo(s), nbody_bh.wgsl:147-157
      float potHalo = 0.0f;
      if (P.haloMass > 0.0f) {
        for (uint32_t h = 0; h < P.haloCount && h < 2; h++) {
          const float* cc = h == 0 ? P.haloC1 : P.haloC2;
          const float dx = p0.x - cc[0], dy = p0.y - cc[1], dz = p0.z - cc[2];
          const float rlen = fmaxf(sqrtf(dx * dx + dy * dy + dz * dz), 1e-6f);
          const float ra = rlen + P.haloA;
          const float k = G * P.haloMass / (ra * ra * rlen);
          fx -= dx * k;
          fy -= dy * k;
          fz -= dz * k;
          potHalo -= G * P.haloMass / ra;
        }
      }
      // kick (nbody_bh.wgsl:161), gas drag (:166-171), drift (:173)
      float vx = fmaf(fx, P.dt, p1.x), vy = fmaf(fy, P.dt, p1.y), vz = fmaf(fz, P.dt, p1.z);
      const bool gas = p1.w < -0.5f;
      if (gas && P.gasDrag > 0.0f) {
        const float hx = -p0.y, hy = p0.x, hz = 1e-6f;
        const float il = rsqrtf(hx * hx + hy * hy + hz * hz);
        const float ux = hx * il, uy = hy * il, uz = hz * il;
        const float vp = vx * ux + vy * uy + vz * uz;
        const float damp = expf(-P.gasDrag * P.dt);
        const float qx = vp * ux, qy = vp * uy, qz = vp * uz;
        vx = qx + (vx - qx) * damp;
        vy = qy + (vy - qy) * damp;
        vz = qz + (vz - qz) * damp;
      }
      const float4 o0 = make_float4(fmaf(vx, P.dt, p0.x), fmaf(vy, P.dt, p0.y), fmaf(vz, P.dt, p0.z), p0.w);
      float4 o1 = make_float4(vx, vy, vz, gas ? -(1.0f + dens) : 0.0f);
      const float e = 0.5f * (vx * vx + vy * vy + vz * vz) + 0.5f * pot + potHalo;
      a.energy[i] = e;
      const double m = p0.w;
      e_diag = e;
      e_true = m * (double)e;
      mx = m * vx;
      my = m * vy;
      mz = m * vz;
      ms = m;
      if (SF && !sst->sf_off) {
        float4 s = a.stellar[i];
        const float4 s_old = s;
        star_formation_one(P, i - sd.off, o1, s);
        if (s.x != s_old.x || s.y != s_old.y || s.z != s_old.z || s.w != s_old.w) a.stellar[i] = s;
      }
      a.pout[2 * (size_t)i] = o0;
      a.pout[2 * (size_t)i + 1] = o1;
    }
    // per-group partial sums of the diagnostics (fixed order, no atomics)
    double v[kPartials] = {e_diag, e_true, mx, my, mz, ms};
#pragma unroll
    for (int k = 0; k < kPartials; k++) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(full, v[k], o);
    }
    if (lane < kPartials) {
      double pv = v[0];
#pragma unroll
      for (int k = 1; k < kPartials; k++)
        if (lane == k) pv = v[k];
      a.partials[((size_t)sd.item0 + (gcur - sd.group0) * LPP + part) * kPartials + lane] = pv;
    }
  }
  // the last warp to finish resets the work counters for the next launch
  if (lane == 0) {
    const unsigned total = gridDim.x * kWalkWarps;
    __threadfence();
    if (atomicAdd(&a.work[1], 1u) == total - 1) {
      a.work[0] = 0;
      a.work[1] = 0;
    }
  }
}

}  // namespace gs

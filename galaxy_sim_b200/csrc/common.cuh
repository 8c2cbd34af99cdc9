// Shared device-side definitions of the B200 gravity path.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/galaxy_b200.h"

namespace gs {

constexpr int kBucket = 16;     // max particles per leaf (mortonTree.js:25)
constexpr int kMaxLevel = 10;   // 10 bits per axis (mortonTree.js:26)
constexpr int kDepths = 11;     // node depths 0..10
// iteration cap of every device-side wait: about a second of polling (each
// look-back iteration is one round trip of 32 loads to L2)
constexpr uint32_t kSpinLimit = 1u << 20;

// Walk-layout node (32 B, two 16-byte words), written by the build next to the
// 64-byte BHNode layout of the API. Children of an internal node are the
// contiguous BFS range [child, child + count).
struct __align__(16) WalkInfo {
  float s2;        // size * size (f32, like nbody_bh.wgsl:111)
  uint32_t child;  // leaf: first particle; internal: first child node
  uint32_t info;   // bit 31 = leaf; bits 0..30 = particle count (leaf) or child count
  float size;      // full node width (density = count / size^3, nbody_bh.wgsl:94)
};
constexpr uint32_t kLeafBit = 0x80000000u;

// Per-galaxy copy of the physics state (Params + what main.js keeps).
struct __align__(16) DevState {
  gs_params p;            // 96 B Params, time refreshed from sim_time each step
  double sim_time;        // main.js simTime (JS number)
  double halo_c[2][3];    // smoothed halo centres (main.js haloCenters, doubles)
  long long central[2];   // tracked central particles (particle-pool indices), -1 = none
  unsigned int err;       // GS_DERR_* bits
  unsigned int sf_off;    // nonzero: this galaxy skips star formation
  unsigned long long counters[3];  // monopoles, leaf pairs, node visits
};

// Tree build scalar outputs of one galaxy (node indices local to its pool).
struct __align__(16) TreeMeta {
  uint32_t level_start[kDepths + 1];
  uint32_t level_count[kDepths + 1];
  uint32_t num_nodes;
  uint32_t num_levels;
  uint32_t num_leaves;
  uint32_t overflow;
  double root_size;
};

// One galaxy ("segment") of a batch: a contiguous particle range with its own
// node pool, Morton frame, tree and Params. A single simulation is a batch of one.
struct __align__(16) SegDesc {
  uint32_t off, n;              // particles [off, off + n) of the particle pool
  uint32_t node_off, node_cap;  // nodes [node_off, node_off + node_cap) of the node pool
  uint32_t sort_tile0;          // first sort tile of the batch's tile list
  uint32_t flag_tile0;          // first build tile (also bbox, codes, gather tiles)
  uint32_t group0;              // first walk group
  uint32_t max_nodes;           // pool of MortonTree's third leaf clause (2n + 4096)
  uint32_t slot;                // index of the galaxy's DevState, TreeMeta, frame, histograms
  uint32_t diag_chunk0;         // first block of the diagnostics reduction
  uint32_t wlpp;                 // walk lanes per particle (1, 2, 4, 8: items of 32, 16, 8, 4)
  uint32_t item0;                // first walk item (diagnostic partials: groups x wlpp per galaxy)
  uint32_t wsplit;               // walk splits per work item (1, 2, 4, 8; above 1 for a lone galaxy only)
  uint32_t pad_[3];
};

// Device view of a batch's layout: segments (sorted by particle offset) and the
// maps from each tile / walk group to its segment. Tiles never cross segments;
// the pool between segments holds free holes that no tile covers.
struct Layout {
  const SegDesc* segs;
  const uint32_t* seg_of_sort_tile;
  const uint32_t* seg_of_flag_tile;
  const uint32_t* seg_of_group;
  uint32_t nseg;
  uint32_t sort_tiles, flag_tiles, groups, diag_chunks;
};

__device__ inline int float_to_ordered(float f) {
  int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__device__ inline float ordered_to_float(int i) {
  return __int_as_float(i >= 0 ? i : i ^ 0x7FFFFFFF);
}

__device__ inline void raise_err(DevState* st, unsigned bits) { atomicOr(&st->err, bits); }

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialization may start while its predecessor drains; it waits here, before
// touching any memory, until the predecessor grids have completed and flushed.
// Without such a dependency the wait returns at once.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

}  // namespace gs

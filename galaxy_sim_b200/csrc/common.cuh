// Shared device-side definitions of the B200 gravity path.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/galaxy_b200.h"

namespace gs {

constexpr int kBucket = 16;     // max particles per leaf (mortonTree.js:25)
constexpr int kMaxLevel = 10;   // 10 bits per axis (mortonTree.js:26)
constexpr int kDepths = 11;     // node depths 0..10
constexpr uint32_t kSpinLimit = 1u << 24;  // iteration cap of every device-side wait

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

// Device copy of the per-step physics state (Params + what main.js keeps).
struct __align__(16) DevState {
  gs_params p;            // 96 B Params, time refreshed from sim_time each step
  double sim_time;        // main.js simTime (JS number)
  double halo_c[2][3];    // smoothed halo centres (main.js haloCenters, doubles)
  long long central[2];   // tracked central particle indices, -1 = none
  long long central_next[2];  // written by the gather, published by the next kernel
  unsigned int err;       // GS_DERR_* bits
  unsigned int pad_;
  unsigned long long counters[3];  // monopoles, leaf pairs, node visits
};

// Tree build scalar outputs.
struct __align__(16) TreeMeta {
  uint32_t level_start[kDepths + 1];
  uint32_t level_count[kDepths + 1];
  uint32_t num_nodes;
  uint32_t num_levels;
  uint32_t num_leaves;
  uint32_t overflow;
  double root_size;
};

// Morton bounding box: ordered-int encodings of float min/max (atomics).
struct __align__(16) BBox {
  int mn[3];
  int mx[3];
  int pad_[2];
};

__device__ inline int float_to_ordered(float f) {
  int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__device__ inline float ordered_to_float(int i) {
  return __int_as_float(i >= 0 ? i : i ^ 0x7FFFFFFF);
}

__device__ inline void raise_err(DevState* st, unsigned bits) { atomicOr(&st->err, bits); }

}  // namespace gs

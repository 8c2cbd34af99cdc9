// Per-particle and per-node kernels around the walk: Morton bbox and codes,
// the permutation gather (with central tracking and the halo-centre EMA), star
// formation, position compaction, per-level COM refresh, uploaded-tree
// conversion and the FP64 diagnostics reduction.
#pragma once
#include "common.cuh"
#include "morton.cuh"
#include "sort.cuh"
#include "walk.cuh"

namespace gs {

constexpr int kBBoxThreads = 256;
#ifndef GS_BBOX_BLOCKS
#define GS_BBOX_BLOCKS 1184
#endif
constexpr int kBBoxBlocks = GS_BBOX_BLOCKS;  // blocks of the bbox reduction

// Bounding box over finite particles (mortonTree.js:44-52), float min/max
// as ordered ints; the last block folds the partials, derives the double frame
// (:53-54) and, when advance_time is set, stamps Params.time = f32(simTime) and
// advances simTime by dt (main.js:422, :476).
__global__ void __launch_bounds__(kBBoxThreads)
    bbox_kernel(const float4* __restrict__ pos, uint32_t stride, uint32_t N, int* partials,
                unsigned* counter, MortonFrame* frame, DevState* st, int advance_time) {
  __shared__ int s_red[kBBoxThreads / 32][6];
  __shared__ bool s_last;
  int mn[3] = {float_to_ordered(INFINITY), float_to_ordered(INFINITY), float_to_ordered(INFINITY)};
  int mx[3] = {float_to_ordered(-INFINITY), float_to_ordered(-INFINITY), float_to_ordered(-INFINITY)};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
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
    for (int w = 1; w < kBBoxThreads / 32; w++)
      v = threadIdx.x < 3 ? min(v, s_red[w][threadIdx.x]) : max(v, s_red[w][threadIdx.x]);
    partials[blockIdx.x * 6 + threadIdx.x] = v;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // fold the per-block partials with the whole block (independent loads in flight)
#pragma unroll
  for (int k = 0; k < 3; k++) {
    mn[k] = float_to_ordered(INFINITY);
    mx[k] = float_to_ordered(-INFINITY);
  }
  for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
      mn[k] = min(mn[k], __ldcg(&partials[b * 6 + k]));
      mx[k] = max(mx[k], __ldcg(&partials[b * 6 + 3 + k]));
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
    for (int w = 1; w < kBBoxThreads / 32; w++)
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
    *frame = frame_from_bbox(fmn, fmx);
    *counter = 0;
    if (advance_time && st) {
      st->p.time = __double2float_rn(st->sim_time);
      st->sim_time = __dadd_rn(st->sim_time, (double)st->p.dt);
    }
  }
}

// Codes (mortonTree.js:55-60) + the digit histograms of every sort pass.
__global__ void __launch_bounds__(256)
    codes_kernel(const float4* __restrict__ pos, uint32_t stride, uint32_t N,
                 const MortonFrame* __restrict__ frame, uint32_t* __restrict__ codes,
                 uint32_t* hist, int passes) {
  __shared__ uint32_t s_hist[4 * 256];
  for (int k = threadIdx.x; k < 4 * 256; k += blockDim.x) s_hist[k] = 0;
  __syncthreads();
  const MortonFrame f = *frame;
  const uint32_t stride_all = gridDim.x * blockDim.x;
  for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < N; i0 += stride_all) {
    const uint32_t i = i0 + threadIdx.x;
    const bool valid = i < N;
    uint32_t code = 0;
    if (valid) {
      const float4 p = pos[(size_t)i * stride];
      code = morton_code(f, p.x, p.y, p.z);
      codes[i] = code;
    }
#ifndef GS_HIST_MATCH
    if (hist && valid)
      for (int p = 0; p < passes; p++) atomicAdd(&s_hist[p * 256 + ((code >> (8 * p)) & 255u)], 1u);
#else
    if (hist) hist_add_warp(s_hist, code, valid, passes);
#endif
  }
  if (!hist) return;
  __syncthreads();
  for (int k = threadIdx.x; k < passes * 256; k += blockDim.x)
    if (s_hist[k]) atomicAdd(&hist[k], s_hist[k]);
}

// Gather dst[i] = src[perm[i]] of the 32-byte particle and 16-byte stellar
// records (nbody_bh.wgsl:322-326, :336-340). With tracking, the thread whose
// source is a tracked central particle records its new index
// (bhWorker.js:67-68) and moves that halo centre 10% of the way to the particle
// (main.js:449-457, in double like the JS numbers), then stores the f32 copy
// in Params (NBodyGPU.js:272-273).
__global__ void __launch_bounds__(256)
    gather_kernel(const uint32_t* __restrict__ perm, const float4* __restrict__ pin,
                  float4* __restrict__ pout, const float4* __restrict__ sin,
                  float4* __restrict__ sout, uint32_t N, DevState* st, int track) {
  long long c0 = -1, c1 = -1;
  if (track) {
    c0 = st->central[0];
    c1 = st->central[1];
  }
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const uint32_t s = perm[i];
    if (s >= N) {  // a corrupted permutation is flagged, never dereferenced
      raise_err(st, GS_DERR_LOOKBACK);
      continue;
    }
    const float4 a = pin[2 * (size_t)s], b = pin[2 * (size_t)s + 1];
    pout[2 * (size_t)i] = a;
    pout[2 * (size_t)i + 1] = b;
    if (sout) sout[i] = sin[s];
    if (track) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const long long c = h == 0 ? c0 : c1;
        if (c >= 0 && (long long)s == c) {
          st->central_next[h] = i;
          if (h < (int)st->p.haloCount) {
            const float q[3] = {a.x, a.y, a.z};
            float* dst = h == 0 ? st->p.haloC1 : st->p.haloC2;
            for (int k = 0; k < 3; k++) {
              const double hc = st->halo_c[h][k];
              const double nv = __dadd_rn(hc, __dmul_rn(__dsub_rn((double)q[k], hc), 0.1));
              st->halo_c[h][k] = nv;
              dst[k] = __double2float_rn(nv);
            }
          }
        }
      }
    }
  }
}

// star_formation as its own pass (NBodyGPU.encodeStarFormation).
__global__ void sf_kernel(float4* __restrict__ P, float4* __restrict__ S, uint32_t N,
                          const DevState* __restrict__ st) {
  const gs_params prm = st->p;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    float4 p1 = P[2 * (size_t)i + 1];
    float4 s = S[i];
    const float4 p1o = p1, so = s;
    star_formation_one(prm, i, p1, s);
    if (p1.x != p1o.x || p1.y != p1o.y || p1.z != p1o.z || p1.w != p1o.w) P[2 * (size_t)i + 1] = p1;
    if (s.x != so.x || s.y != so.y || s.z != so.z || s.w != so.w) S[i] = s;
  }
}

// compact_positions (nbody_bh.wgsl:188-195).
__global__ void compact_kernel(const float4* __restrict__ P, const float* __restrict__ energy,
                               float4* __restrict__ out, uint32_t N) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const float4 p = P[2 * (size_t)i];
    out[i] = make_float4(p.x, p.y, p.z, energy[i]);
  }
}

// refresh_level (nbody_bh.wgsl:288-313) on one BFS level of the walk layout.
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

// uploadBHTree: BHNode (64 B) -> walk layout. Children of an internal node must
// be the contiguous increasing run the BFS build produces (mortonTree.js:146-155).
// A node that breaks the rules (children not after their parent, ranges past
// the node or particle arrays) is flagged and made an empty leaf, so a walk
// over an uploaded tree always terminates and stays in bounds.
__global__ void upload_convert_kernel(const gs_node* __restrict__ nodes, uint32_t num_nodes,
                                      uint32_t N, float4* cm, WalkInfo* info, DevState* st) {
  for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < num_nodes; n += gridDim.x * blockDim.x) {
    const gs_node nd = nodes[n];
    cm[n] = make_float4(nd.com[0], nd.com[1], nd.com[2], nd.mass);
    WalkInfo w;
    w.s2 = nd.size * nd.size;
    w.size = nd.size;
    bool ok = true;
    if (nd.isLeaf == 1u) {
      ok = nd.count < kLeafBit && (uint64_t)nd.first + nd.count <= N;
      w.child = nd.first;
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
      w.child = first < 0 ? 0u : (uint32_t)first;
      w.info = nc;
    }
    if (!ok) {
      raise_err(st, GS_DERR_TREE);
      w.child = 0;
      w.info = kLeafBit;  // empty leaf
      cm[n].w = 0.0f;
    }
    info[n] = w;
  }
}

// FP64 diagnostics: fold the walk's per-block partials.
__global__ void diag_reduce_kernel(const double* __restrict__ partials, uint32_t nblocks,
                                   double* out) {
  const int k = threadIdx.y, lane = threadIdx.x;
  double v = 0;
  for (uint32_t b = lane; b < nblocks; b += 32) v += partials[(size_t)b * kPartials + k];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) out[k] = v;
}

}  // namespace gs

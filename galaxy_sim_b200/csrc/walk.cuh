// Barnes-Hut walk + Hernquist halo + kick-drift (+ star formation) on sm_100a.
//
// Semantics follow `main` in src/physics/shaders/nbody_bh.wgsl:64-181 per
// particle: own-leaf density, softened opening test
//   accept  <=>  size^2 < theta^2 (r^2 + eps^2)  ||  size^2 < eps^2 / 4,
// monopole G M r / (r^2 + eps^2)^(3/2), leaf direct sum with j != i, halo,
// v += a dt, gas drag, x += v dt, pad and specific-energy writes.
//
// Execution is warp-cooperative: a warp owns 32 Morton-consecutive particles
// (one per lane) and walks the union of their frontiers with a warp-uniform
// stack of child ranges (children of a BFS node are contiguous), so every node
// and leaf particle is a broadcast load. Each lane still applies exactly its
// own particle's acceptance decisions: a lane is active for a node only if it
// opened every ancestor, so the per-particle interaction set is identical to
// the reference's thread-per-particle stack walk.
#pragma once
#include "common.cuh"

namespace gs {

constexpr int kWalkThreads = 128;
constexpr int kWalkWarps = kWalkThreads / 32;
constexpr int kPartials = 6;  // e_diag, e_true, px, py, pz, mass

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
// p0 = (pos, mass), p1 = (vel, pad), s = stellar record. Returns true if changed.
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
  DevState* st;
  float* __restrict__ energy;       // e_i
  float4* __restrict__ dbg_acc;     // optional {ax, ay, az, phi} (G applied)
  float* __restrict__ dbg_dens;
  double* __restrict__ partials;    // [blocks][kPartials]
  uint32_t N;
  uint32_t node_cap;                // allocated nodes: child ranges must stay below it
};

template <bool SF, bool DBG>
__global__ void __launch_bounds__(kWalkThreads) walk_kernel(WalkArgs a) {
  __shared__ double s_part[kWalkWarps][kPartials];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t i = blockIdx.x * kWalkThreads + threadIdx.x;
  const bool valid = i < a.N;
  const gs_params P = a.st->p;
  const float eps2 = P.epsilon2;
  const float theta2 = P.theta * P.theta;
  const float qe2 = 0.25f * eps2;

  float4 p0 = make_float4(0.f, 0.f, 0.f, 0.f), p1 = p0;
  if (valid) {
    p0 = a.pin[2 * (size_t)i];
    p1 = a.pin[2 * (size_t)i + 1];
  }
  float ax = 0.f, ay = 0.f, az = 0.f, pot = 0.f, dens = 0.f;
  unsigned long long nmono = 0, npair = 0, nvisit = 0;
  const unsigned all = __ballot_sync(0xffffffffu, valid);

  // warp-uniform stack of child ranges; lane k holds entry k
  uint32_t s_start = 0, s_cnt = 0, s_mask = 0;
  int sp = 0;
  if (all) {
    if (lane == 0) {
      s_start = 0;
      s_cnt = 1;
      s_mask = all;
    }
    sp = 1;
  }
  // A well-formed tree is visited at most once per node; the cap only bounds the
  // loop if the node data were ever corrupted.
  uint32_t budget = 4u * a.node_cap + 1024u;
  while (sp > 0) {
    if (--budget == 0) {
      if (lane == 0) raise_err(a.st, GS_DERR_STACK);
      break;
    }
    const int top = sp - 1;
    const uint32_t n = __shfl_sync(0xffffffffu, s_start, top);
    const uint32_t c = __shfl_sync(0xffffffffu, s_cnt, top);
    const uint32_t mask = __shfl_sync(0xffffffffu, s_mask, top);
    if (lane == top) {
      s_start++;
      s_cnt--;
    }
    if (c == 1) sp--;
    const float4 q = __ldg(&a.cm[n]);
    if (q.w == 0.0f) continue;
    const WalkInfo w = a.info[n];
    const bool act = (mask >> lane) & 1u;
    const bool leaf = (w.info & kLeafBit) != 0u;
    const uint32_t cnt = w.info & ~kLeafBit;
    if (DBG) nvisit += act;
    if (leaf && act && (i - w.child) < cnt) dens = (float)cnt / (w.size * w.size * w.size);
    const float rx = q.x - p0.x, ry = q.y - p0.y, rz = q.z - p0.z;
    const float d2 = fmaf(rx, rx, fmaf(ry, ry, fmaf(rz, rz, eps2)));
    const bool ok = (w.s2 < theta2 * d2) || (w.s2 < qe2);
    if (act && ok) {
      const float rinv = rsqrtf(d2);
      const float mr = q.w * rinv;
      const float f = mr * rinv * rinv;
      ax = fmaf(rx, f, ax);
      ay = fmaf(ry, f, ay);
      az = fmaf(rz, f, az);
      pot -= mr;
      if (DBG) nmono++;
    }
    const unsigned open = __ballot_sync(0xffffffffu, act && !ok);
    if (open) {
      // children come after their parent and stay inside the node / particle arrays
      const bool sane = leaf ? ((uint64_t)w.child + cnt <= a.N)
                             : (w.child > n && (uint64_t)w.child + cnt <= a.node_cap && cnt <= 8u);
      if (!sane) {
        if (lane == 0) raise_err(a.st, GS_DERR_TREE);
        continue;
      }
      if (leaf) {
        const bool me = (open >> lane) & 1u;
        const uint32_t end = w.child + cnt;
        for (uint32_t j = w.child; j < end; j++) {
          const float4 pj = __ldg(&a.pin[2 * (size_t)j]);
          if (me) {
            const float jx = pj.x - p0.x, jy = pj.y - p0.y, jz = pj.z - p0.z;
            const float e2 = fmaf(jx, jx, fmaf(jy, jy, fmaf(jz, jz, eps2)));
            const float rinv = rsqrtf(e2);
            const float mj = (j == i) ? 0.0f : pj.w;
            const float mr = mj * rinv;
            const float f = mr * rinv * rinv;
            ax = fmaf(jx, f, ax);
            ay = fmaf(jy, f, ay);
            az = fmaf(jz, f, az);
            pot -= mr;
            if (DBG) npair += (j != i);
          }
        }
      } else {
        if (sp >= 31) {  // cannot happen for depth <= 10 trees; never corrupt the stack
          if (lane == 0) raise_err(a.st, GS_DERR_STACK);
          break;
        }
        if (lane == sp) {
          s_start = w.child;
          s_cnt = cnt;
          s_mask = open;
        }
        sp++;
      }
    }
  }

  double e_diag = 0, e_true = 0, mx = 0, my = 0, mz = 0, ms = 0;
  if (valid) {
    const float G = P.G;
    ax *= G;
    ay *= G;
    az *= G;
    pot *= G;
    if (DBG) {
      a.dbg_acc[i] = make_float4(ax, ay, az, pot);
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
        ax -= dx * k;
        ay -= dy * k;
        az -= dz * k;
        potHalo -= G * P.haloMass / ra;
      }
    }
    // kick (nbody_bh.wgsl:161), gas drag (:166-171), drift (:173)
    float vx = fmaf(ax, P.dt, p1.x), vy = fmaf(ay, P.dt, p1.y), vz = fmaf(az, P.dt, p1.z);
    const bool gas = p1.w < -0.5f;
    if (gas && P.gasDrag > 0.0f) {
      const float hx = -p0.y, hy = p0.x, hz = 1e-6f;
      const float il = rsqrtf(hx * hx + hy * hy + hz * hz);
      const float ux = hx * il, uy = hy * il, uz = hz * il;
      const float vp = vx * ux + vy * uy + vz * uz;
      const float damp = expf(-P.gasDrag * P.dt);
      const float px = vp * ux, py = vp * uy, pz = vp * uz;
      vx = px + (vx - px) * damp;
      vy = py + (vy - py) * damp;
      vz = pz + (vz - pz) * damp;
    }
    float4 o0 = make_float4(fmaf(vx, P.dt, p0.x), fmaf(vy, P.dt, p0.y), fmaf(vz, P.dt, p0.z), p0.w);
    float4 o1 = make_float4(vx, vy, vz, gas ? -(1.0f + dens) : 0.0f);
    const float e = 0.5f * (vx * vx + vy * vy + vz * vz) + 0.5f * pot + potHalo;
    a.energy[i] = e;
    const double m = p0.w;
    e_diag = e;
    e_true = m * ((double)e);
    mx = m * vx;
    my = m * vy;
    mz = m * vz;
    ms = m;
    if (SF) {
      float4 s = a.stellar[i];
      const float4 s_old = s;
      star_formation_one(P, i, o1, s);
      if (s.x != s_old.x || s.y != s_old.y || s.z != s_old.z || s.w != s_old.w) a.stellar[i] = s;
    }
    a.pout[2 * (size_t)i] = o0;
    a.pout[2 * (size_t)i + 1] = o1;
  }
  // block partial sums of the diagnostics (fixed order, no atomics)
  double v[kPartials] = {e_diag, e_true, mx, my, mz, ms};
#pragma unroll
  for (int k = 0; k < kPartials; k++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    if (lane == 0) s_part[warp][k] = v[k];
  }
  if (DBG) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      nmono += __shfl_xor_sync(0xffffffffu, nmono, o);
      npair += __shfl_xor_sync(0xffffffffu, npair, o);
      nvisit += __shfl_xor_sync(0xffffffffu, nvisit, o);
    }
    if (lane == 0) {
      atomicAdd(&a.st->counters[0], nmono);
      atomicAdd(&a.st->counters[1], npair);
      atomicAdd(&a.st->counters[2], nvisit);
    }
  }
  __syncthreads();
  if (threadIdx.x < kPartials) {
    double s = 0;
    for (int w = 0; w < kWalkWarps; w++) s += s_part[w][threadIdx.x];
    a.partials[(size_t)blockIdx.x * kPartials + threadIdx.x] = s;
  }
}

}  // namespace gs

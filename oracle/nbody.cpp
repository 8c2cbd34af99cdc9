// TEST INFRASTRUCTURE ONLY — CPU oracle. Restatement of the compute entry
// points of galaxy-sim's src/physics/shaders/nbody_bh.wgsl (and the dispatch
// order of src/physics/NBodyGPU.js), in FP32 exactly as written (no FMA
// contraction), plus an FP64 walk with the same acceptance rule on the same
// tree, an FP64 direct O(N^2) sum and an FP64 COM refresh used as references.
// Parity unpinned against the reference itself (no WebGPU stack exists here);
// see oracle.h.
#include "oracle.h"

#include <omp.h>

#include <cmath>
#include <cstring>
#include <vector>

namespace {

constexpr int STACK_SIZE = 96;  // nbody_bh.wgsl:62

struct f3 {
  float x, y, z;
};
inline f3 sub(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

inline int set_threads(int nthreads) {
  return nthreads > 0 ? nthreads : omp_get_max_threads();
}

}  // namespace

// nbody_bh.wgsl:319-340 — gather dst[i] = src[perm[i]] of `width`-float records.
extern "C" void or_apply_permutation(const float* in, float* out, const uint32_t* perm,
                                     uint32_t N, uint32_t width) {
  for (uint32_t i = 0; i < N; i++)
    std::memcpy(out + (size_t)i * width, in + (size_t)perm[i] * width, sizeof(float) * width);
}

// nbody_bh.wgsl:289-313 dispatched per level, deepest first (NBodyGPU.js:308-319).
extern "C" void or_refresh_f32(const float* P, or_node* nodes, const uint32_t* lr,
                               uint32_t n_levels) {
  for (int64_t lvl = (int64_t)n_levels - 1; lvl >= 0; lvl--) {
    const uint32_t start = lr[2 * lvl], count = lr[2 * lvl + 1];
    for (uint32_t g = 0; g < count; g++) {
      or_node& nd = nodes[start + g];
      float cx = 0, cy = 0, cz = 0, m = 0;
      if (nd.isLeaf == 1u) {
        for (uint32_t j = nd.first; j < nd.first + nd.count; j++) {
          const float* p = P + (size_t)j * 8;
          cx = cx + p[0] * p[3];
          cy = cy + p[1] * p[3];
          cz = cz + p[2] * p[3];
          m = m + p[3];
        }
      } else {
        for (int c = 0; c < 8; c++) {
          const int32_t ch = nd.children[c];
          if (ch >= 0) {
            const or_node& cn = nodes[ch];
            cx = cx + cn.com[0] * cn.mass;
            cy = cy + cn.com[1] * cn.mass;
            cz = cz + cn.com[2] * cn.mass;
            m = m + cn.mass;
          }
        }
      }
      if (m > 0.0f) {
        nd.com[0] = cx / m;
        nd.com[1] = cy / m;
        nd.com[2] = cz / m;
      } else {
        nd.com[0] = nd.com[1] = nd.com[2] = 0.0f;
      }
      nd.mass = m;
    }
  }
}

// The same refresh in FP64 (reference values for the COM tolerance tests and
// the COM the FP64 walk uses): com4[n] = {cx, cy, cz, m}.
extern "C" void or_refresh_f64(const float* P, const or_node* nodes, uint32_t numNodes,
                               const uint32_t* lr, uint32_t n_levels, double* com4) {
  (void)numNodes;
  for (int64_t lvl = (int64_t)n_levels - 1; lvl >= 0; lvl--) {
    const uint32_t start = lr[2 * lvl], count = lr[2 * lvl + 1];
    for (uint32_t g = 0; g < count; g++) {
      const uint32_t n = start + g;
      const or_node& nd = nodes[n];
      double cx = 0, cy = 0, cz = 0, m = 0;
      if (nd.isLeaf == 1u) {
        for (uint32_t j = nd.first; j < nd.first + nd.count; j++) {
          const float* p = P + (size_t)j * 8;
          cx += (double)p[0] * p[3];
          cy += (double)p[1] * p[3];
          cz += (double)p[2] * p[3];
          m += p[3];
        }
      } else {
        for (int c = 0; c < 8; c++) {
          const int32_t ch = nd.children[c];
          if (ch >= 0) {
            const double* q = com4 + (size_t)ch * 4;
            cx += q[0] * q[3];
            cy += q[1] * q[3];
            cz += q[2] * q[3];
            m += q[3];
          }
        }
      }
      double* o = com4 + (size_t)n * 4;
      if (m > 0) {
        o[0] = cx / m;
        o[1] = cy / m;
        o[2] = cz / m;
      } else {
        o[0] = o[1] = o[2] = 0;
      }
      o[3] = m;
    }
  }
}

// nbody_bh.wgsl:64-181 — BH walk with an explicit 96-entry stack, own-leaf
// density, softened opening test + sub-softening monopole, leaf direct sum with
// j != i, Hernquist halo(s), kick-drift, gas drag, pad/energy writes. FP32.
// acc4 (optional) receives {ax, ay, az, pot} of the pair forces before the halo.
namespace {
// One particle of nbody_bh.wgsl `main` (walk, halo, kick-drift, pad, energy).
inline void step_one(const or_params& p, uint32_t i, const float* pin, float* pout,
                     const or_node* nodes, float* energy, float* acc4, float* dens_out,
                     uint64_t& nMono, uint64_t& nPair, uint64_t& nVisit) {
    const float* pi = pin + (size_t)i * 8;
    const f3 ppos{pi[0], pi[1], pi[2]};
    f3 acc{0, 0, 0};
    float pot = 0.0f, density = 0.0f;
    const float theta2 = p.theta * p.theta;
    int32_t stack[STACK_SIZE];
    int sp = 1;
    stack[0] = 0;
    while (sp > 0) {
      sp -= 1;
      const or_node& node = nodes[stack[sp]];
      const float nodeMass = node.mass;
      nVisit++;
      if (nodeMass == 0.0f) continue;
      const f3 com{node.com[0], node.com[1], node.com[2]};
      const float nodeSize = node.size;
      const bool isLeaf = node.isLeaf == 1u;
      if (isLeaf && i >= node.first && i < node.first + node.count)
        density = (float)node.count / (nodeSize * nodeSize * nodeSize);
      const f3 r = sub(com, ppos);
      const float geomD2 = dot(r, r);
      const float d2 = geomD2 + p.epsilon2;
      const float s2 = nodeSize * nodeSize;
      if (s2 < theta2 * d2 || s2 < 0.25f * p.epsilon2) {
        const float f = p.G * nodeMass / (d2 * std::sqrt(d2));
        acc.x = acc.x + r.x * f;
        acc.y = acc.y + r.y * f;
        acc.z = acc.z + r.z * f;
        pot = pot - f * d2;
        nMono++;
      } else if (isLeaf) {
        const uint32_t first = node.first, count = node.count;
        for (uint32_t j = first; j < first + count; j++) {
          if (j == i) continue;
          const float* pj = pin + (size_t)j * 8;
          const f3 rj = sub(f3{pj[0], pj[1], pj[2]}, ppos);
          const float dj2 = dot(rj, rj) + p.epsilon2;
          const float f = p.G * pj[3] / (dj2 * std::sqrt(dj2));
          acc.x = acc.x + rj.x * f;
          acc.y = acc.y + rj.y * f;
          acc.z = acc.z + rj.z * f;
          pot = pot - f * dj2;
          nPair++;
        }
      } else {
        for (int c = 0; c < 8; c++) {
          const int32_t ch = node.children[c];
          if (ch >= 0 && sp < STACK_SIZE) stack[sp++] = ch;
        }
      }
    }
    if (acc4) {
      acc4[(size_t)i * 4] = acc.x;
      acc4[(size_t)i * 4 + 1] = acc.y;
      acc4[(size_t)i * 4 + 2] = acc.z;
      acc4[(size_t)i * 4 + 3] = pot;
    }
    if (dens_out) dens_out[i] = density;
    float potHalo = 0.0f;
    if (p.haloMass > 0.0f) {
      for (uint32_t h = 0; h < p.haloCount; h++) {
        const float* c = h == 0 ? p.haloC1 : p.haloC2;
        const f3 d = sub(ppos, f3{c[0], c[1], c[2]});
        const float rlen = std::fmax(std::sqrt(dot(d, d)), 1e-6f);
        const float ra = rlen + p.haloA;
        const float k = p.G * p.haloMass / (ra * ra * rlen);
        acc.x = acc.x - d.x * k;
        acc.y = acc.y - d.y * k;
        acc.z = acc.z - d.z * k;
        potHalo = potHalo - p.G * p.haloMass / ra;
      }
    }
    f3 v{pi[4] + acc.x * p.dt, pi[5] + acc.y * p.dt, pi[6] + acc.z * p.dt};
    const bool isGas = pi[7] < -0.5f;
    if (isGas && p.gasDrag > 0.0f) {
      const f3 ph{-ppos.y, ppos.x, 1e-6f};
      const float len = std::sqrt(dot(ph, ph));
      const f3 phiHat{ph.x / len, ph.y / len, ph.z / len};
      const float vp = dot(v, phiHat);
      const f3 vPhi{vp * phiHat.x, vp * phiHat.y, vp * phiHat.z};
      const float damp = std::exp(-p.gasDrag * p.dt);
      v = f3{vPhi.x + (v.x - vPhi.x) * damp, vPhi.y + (v.y - vPhi.y) * damp,
             vPhi.z + (v.z - vPhi.z) * damp};
    }
    float* po = pout + (size_t)i * 8;
    po[0] = ppos.x + v.x * p.dt;
    po[1] = ppos.y + v.y * p.dt;
    po[2] = ppos.z + v.z * p.dt;
    po[3] = pi[3];
    po[4] = v.x;
    po[5] = v.y;
    po[6] = v.z;
    po[7] = isGas ? -(1.0f + density) : 0.0f;
    if (energy) energy[i] = 0.5f * dot(v, v) + 0.5f * pot + potHalo;
  }
}  // namespace

// nbody_bh.wgsl:64-181 — BH walk with an explicit 96-entry stack, own-leaf
// density, softened opening test + sub-softening monopole, leaf direct sum with
// j != i, Hernquist halo(s), kick-drift, gas drag, pad/energy writes. FP32.
// acc4 (optional) receives {ax, ay, az, pot} of the pair forces before the halo.
extern "C" void or_step_f32(const or_params* prm, const float* pin, float* pout,
                            const or_node* nodes, float* energy, float* acc4, float* dens_out,
                            uint64_t* counters, int nthreads) {
  const or_params p = *prm;
  uint64_t nMono = 0, nPair = 0, nVisit = 0;
#pragma omp parallel for schedule(dynamic, 256) num_threads(set_threads(nthreads)) \
    reduction(+ : nMono, nPair, nVisit)
  for (int64_t ii = 0; ii < (int64_t)p.N; ii++)
    step_one(p, (uint32_t)ii, pin, pout, nodes, energy, acc4, dens_out, nMono, nPair, nVisit);
  if (counters) {
    counters[0] = nMono;
    counters[1] = nPair;
    counters[2] = nVisit;
  }
}

// The same step for every `stride`-th particle only (a bounded CPU timing sample).
extern "C" void or_step_f32_sample(const or_params* prm, const float* pin, float* pout,
                                   const or_node* nodes, float* energy, uint32_t stride,
                                   int nthreads) {
  const or_params p = *prm;
  if (stride == 0) stride = 1;
  uint64_t a = 0, b = 0, c = 0;
  const int64_t M = ((int64_t)p.N + stride - 1) / stride;
#pragma omp parallel for schedule(dynamic, 64) num_threads(set_threads(nthreads)) reduction(+ : a, b, c)
  for (int64_t k = 0; k < M; k++)
    step_one(p, (uint32_t)(k * stride), pin, pout, nodes, energy, nullptr, nullptr, a, b, c);
}

// The same walk in FP64 on the same tree (topology, sizes, leaf ranges) with
// FP64 COMs (com4 from or_refresh_f64). Pair forces only (no halo).
extern "C" void or_walk_f64(const or_params* prm, const float* pin, const or_node* nodes,
                            const double* com4, double* acc3, double* pot_out,
                            float* dens_out, uint64_t* counters, int nthreads) {
  const or_params p = *prm;
  const uint32_t N = p.N;
  const double eps2 = p.epsilon2, theta2 = (double)p.theta * p.theta, G = p.G;
  uint64_t nMono = 0, nPair = 0, nVisit = 0;
#pragma omp parallel for schedule(dynamic, 256) num_threads(set_threads(nthreads)) \
    reduction(+ : nMono, nPair, nVisit)
  for (int64_t ii = 0; ii < (int64_t)N; ii++) {
    const uint32_t i = (uint32_t)ii;
    const double px = pin[(size_t)i * 8], py = pin[(size_t)i * 8 + 1],
                 pz = pin[(size_t)i * 8 + 2];
    double ax = 0, ay = 0, az = 0, pot = 0;
    float density = 0;
    int32_t stack[STACK_SIZE];
    int sp = 1;
    stack[0] = 0;
    while (sp > 0) {
      const int32_t n = stack[--sp];
      const or_node& node = nodes[n];
      const double* c = com4 + (size_t)n * 4;
      nVisit++;
      if (c[3] == 0.0) continue;
      const bool isLeaf = node.isLeaf == 1u;
      if (isLeaf && i >= node.first && i < node.first + node.count)
        density = (float)node.count / (node.size * node.size * node.size);
      const double rx = c[0] - px, ry = c[1] - py, rz = c[2] - pz;
      const double d2 = rx * rx + ry * ry + rz * rz + eps2;
      const double s2 = (double)node.size * node.size;
      if (s2 < theta2 * d2 || s2 < 0.25 * eps2) {
        const double f = G * c[3] / (d2 * std::sqrt(d2));
        ax += rx * f;
        ay += ry * f;
        az += rz * f;
        pot -= f * d2;
        nMono++;
      } else if (isLeaf) {
        for (uint32_t j = node.first; j < node.first + node.count; j++) {
          if (j == i) continue;
          const float* pj = pin + (size_t)j * 8;
          const double rjx = pj[0] - px, rjy = pj[1] - py, rjz = pj[2] - pz;
          const double dj2 = rjx * rjx + rjy * rjy + rjz * rjz + eps2;
          const double f = G * pj[3] / (dj2 * std::sqrt(dj2));
          ax += rjx * f;
          ay += rjy * f;
          az += rjz * f;
          pot -= f * dj2;
          nPair++;
        }
      } else {
        for (int ch = 0; ch < 8; ch++) {
          const int32_t cc = node.children[ch];
          if (cc >= 0 && sp < STACK_SIZE) stack[sp++] = cc;
        }
      }
    }
    acc3[(size_t)i * 3] = ax;
    acc3[(size_t)i * 3 + 1] = ay;
    acc3[(size_t)i * 3 + 2] = az;
    if (pot_out) pot_out[i] = pot;
    if (dens_out) dens_out[i] = density;
  }
  if (counters) {
    counters[0] = nMono;
    counters[1] = nPair;
    counters[2] = nVisit;
  }
}

// FP64 direct O(N^2) softened sum for a target subset (pair forces only).
extern "C" void or_direct_f64(const or_params* prm, const float* pin, const uint32_t* targets,
                              uint32_t nT, double* acc3, double* pot_out, int nthreads) {
  const or_params p = *prm;
  const uint32_t N = p.N;
  const double eps2 = p.epsilon2, G = p.G;
#pragma omp parallel for schedule(dynamic, 16) num_threads(set_threads(nthreads))
  for (int64_t t = 0; t < (int64_t)nT; t++) {
    const uint32_t i = targets[t];
    const double px = pin[(size_t)i * 8], py = pin[(size_t)i * 8 + 1],
                 pz = pin[(size_t)i * 8 + 2];
    double ax = 0, ay = 0, az = 0, pot = 0;
    for (uint32_t j = 0; j < N; j++) {
      if (j == i) continue;
      const float* pj = pin + (size_t)j * 8;
      const double rx = pj[0] - px, ry = pj[1] - py, rz = pj[2] - pz;
      const double d2 = rx * rx + ry * ry + rz * rz + eps2;
      const double inv = 1.0 / std::sqrt(d2);
      const double f = G * pj[3] * inv * inv * inv;
      ax += rx * f;
      ay += ry * f;
      az += rz * f;
      pot -= G * pj[3] * inv;
    }
    acc3[(size_t)t * 3] = ax;
    acc3[(size_t)t * 3 + 1] = ay;
    acc3[(size_t)t * 3 + 2] = az;
    if (pot_out) pot_out[t] = pot;
  }
}

// FP64 Hernquist halo term (nbody_bh.wgsl:147-157) for a target subset.
extern "C" void or_halo_f64(const or_params* prm, const float* pin, const uint32_t* targets,
                            uint32_t nT, double* acc3, double* pot_out) {
  const or_params p = *prm;
  for (uint32_t t = 0; t < nT; t++) {
    const uint32_t i = targets[t];
    double ax = 0, ay = 0, az = 0, pot = 0;
    if (p.haloMass > 0.0f) {
      for (uint32_t h = 0; h < p.haloCount; h++) {
        const float* c = h == 0 ? p.haloC1 : p.haloC2;
        const double dx = (double)pin[(size_t)i * 8] - c[0];
        const double dy = (double)pin[(size_t)i * 8 + 1] - c[1];
        const double dz = (double)pin[(size_t)i * 8 + 2] - c[2];
        const double rl = std::fmax(std::sqrt(dx * dx + dy * dy + dz * dz), 1e-6);
        const double ra = rl + p.haloA;
        const double k = (double)p.G * p.haloMass / (ra * ra * rl);
        ax -= dx * k;
        ay -= dy * k;
        az -= dz * k;
        pot -= (double)p.G * p.haloMass / ra;
      }
    }
    acc3[(size_t)t * 3] = ax;
    acc3[(size_t)t * 3 + 1] = ay;
    acc3[(size_t)t * 3 + 2] = az;
    if (pot_out) pot_out[t] = pot;
  }
}

// nbody_bh.wgsl:206-210
extern "C" uint32_t or_pcg(uint32_t v0) {
  uint32_t v = v0 * 747796405u + 2891336453u;
  v = ((v >> ((v >> 28u) + 4u)) ^ v) * 277803737u;
  return (v >> 22u) ^ v;
}

// nbody_bh.wgsl:211-213 — the f32 literal 4294967295.0 rounds to 2^32.
extern "C" float or_rand01(uint32_t i, uint32_t salt) {
  return (float)or_pcg(i ^ (salt * 0x9E3779B9u)) / 4294967295.0f;
}

// nbody_bh.wgsl:216-227 — Kroupa (2001) inverse CDF in f32.
extern "C" float or_imf_sample(float u1, float u2) {
  const float a0 = std::pow(0.08f, -0.3f);
  const float b0 = std::pow(0.5f, -0.3f);
  const float lowInt = (a0 - b0) / 0.3f;
  const float a1 = std::pow(0.5f, -1.3f);
  const float b1 = std::pow(100.0f, -1.3f);
  const float hiInt = 0.5f * (a1 - b1) / 1.3f;
  if (u1 < lowInt / (lowInt + hiInt)) return std::pow(a0 - u2 * (a0 - b0), -1.0f / 0.3f);
  return std::pow(a1 - u2 * (a1 - b1), -1.0f / 1.3f);
}

static inline uint32_t wgsl_u32(float x) {  // WGSL u32(f32): truncate, clamp
  if (!(x > 0.0f)) return 0u;
  if (x >= 4294967296.0f) return 0xFFFFFFFFu;
  return (uint32_t)x;
}

// nbody_bh.wgsl:229-268 — in place on the particle and stellar records.
extern "C" void or_star_formation(const or_params* prm, float* P, float* S) {
  const or_params p = *prm;
  const uint32_t salt = wgsl_u32(p.time * 977.0f) + 1u;
  for (uint32_t i = 0; i < p.N; i++) {
    float* pp = P + (size_t)i * 8;
    float* st = S + (size_t)i * 4;
    if (pp[7] < -0.5f) {
      const float density = -pp[7] - 1.0f;
      if (density > p.sfDensity && p.sfEff > 0.0f) {
        const float prob =
            p.sfEff * p.sfDt * std::fmin(std::sqrt(density / std::fmax(p.sfDensity, 1e-6f)), 3.0f);
        if (or_rand01(i, salt) < prob) {
          const float m = or_imf_sample(or_rand01(i, salt + 7u), or_rand01(i, salt + 13u));
          const float birthMyr = p.time * p.agingRate;
          st[0] = m;
          st[1] = birthMyr;
          st[2] = or_rand01(i, salt + 29u);
          st[3] = 0.0f;
          pp[7] = 0.0f;
        }
      }
    } else if (st[0] >= 8.0f) {
      const float ageMyr = p.time * p.agingRate - st[1];
      const float tMS = 10000.0f * std::pow(st[0], -2.5f);
      const float tGiant = tMS * 0.12f + 15.0f;
      if (ageMyr > tMS + tGiant + 15.0f + 30.0f) {
        const float z = st[2];
        st[0] = -1.0f;
        st[1] = 0.0f;
        st[2] = z;
        st[3] = 0.7f;
        pp[7] = -1.0f;
        const float kx = (or_rand01(i, salt + 41u) - 0.5f) * 2.0f;
        const float ky = (or_rand01(i, salt + 43u) - 0.5f) * 2.0f;
        const float kz = (or_rand01(i, salt + 47u) - 0.5f) * 2.0f;
        pp[4] = pp[4] + kx;
        pp[5] = pp[5] + ky;
        pp[6] = pp[6] + kz;
      }
    }
  }
}

// nbody_bh.wgsl:188-195 — vec4(pos, energy).
extern "C" void or_compact_positions(const float* P, const float* energy, uint32_t N,
                                     float* out4) {
  for (uint32_t i = 0; i < N; i++) {
    out4[(size_t)i * 4] = P[(size_t)i * 8];
    out4[(size_t)i * 4 + 1] = P[(size_t)i * 8 + 1];
    out4[(size_t)i * 4 + 2] = P[(size_t)i * 8 + 2];
    out4[(size_t)i * 4 + 3] = energy[i];
  }
}

// TEST INFRASTRUCTURE ONLY — CPU oracle. Restatement of galaxy-sim's
// src/physics/mortonTree.js and the build half of src/physics/bhWorker.js with
// JavaScript number semantics (IEEE double, ToInt32 for `| 0`, round-to-nearest
// on every Float32Array store). Compiled with -ffp-contract=off -fno-fast-math
// so every double operation rounds exactly as the JS engine's does.
// Parity unpinned against the reference itself (no JS engine exists here);
// see oracle.h.
#include "oracle.h"

#include <cmath>
#include <cstring>
#include <vector>

namespace {

constexpr uint32_t BUCKET = 16;    // mortonTree.js:25
constexpr uint32_t MAX_LEVEL = 10; // mortonTree.js:26

// Math.max(a, b, c): NaN if any argument is NaN (ECMA-262 Math.max).
double js_max3(double a, double b, double c) {
  if (std::isnan(a) || std::isnan(b) || std::isnan(c)) return NAN;
  double m = a;
  if (b > m) m = b;
  if (c > m) m = c;
  return m;
}

}  // namespace

// ECMA-262 ToInt32, the semantics of `x | 0` (mortonTree.js:56-58).
extern "C" int32_t or_js_toint32(double d) {
  if (!std::isfinite(d)) return 0;
  double t = std::trunc(d);
  double m = std::fmod(t, 4294967296.0);
  if (m < 0) m += 4294967296.0;
  uint32_t u = static_cast<uint32_t>(m);
  return static_cast<int32_t>(u);
}

// mortonTree.js:29-36
extern "C" uint32_t or_part1by2(uint32_t v) {
  v &= 0x3ff;
  v = (v | (v << 16)) & 0x30000ff;
  v = (v | (v << 8)) & 0x300f00f;
  v = (v | (v << 4)) & 0x30c30c3;
  v = (v | (v << 2)) & 0x9249249;
  return v;
}

// mortonTree.js:43-62 — cubic bbox over finite particles, 10-bit quantisation
// per axis in double, 30-bit interleave x | y<<1 | z<<2. Returns rootSize.
extern "C" double or_compute_morton_codes(const float* pos, uint32_t N, uint32_t stride,
                                          uint32_t* codes) {
  double minX = INFINITY, minY = INFINITY, minZ = INFINITY;
  double maxX = -INFINITY, maxY = -INFINITY, maxZ = -INFINITY;
  for (uint32_t i = 0; i < N; i++) {
    const double x = pos[(size_t)i * stride], y = pos[(size_t)i * stride + 1],
                 z = pos[(size_t)i * stride + 2];
    if (!std::isfinite(x + y + z)) continue;  // Number.isFinite(x + y + z)
    if (x < minX) minX = x;
    if (x > maxX) maxX = x;
    if (y < minY) minY = y;
    if (y > maxY) maxY = y;
    if (z < minZ) minZ = z;
    if (z > maxZ) maxZ = z;
  }
  const double size = js_max3(maxX - minX, maxY - minY, maxZ - minZ) * 1.0001 + 1e-9;
  const double s = 1024 / size;
  for (uint32_t i = 0; i < N; i++) {
    int32_t x = or_js_toint32(((double)pos[(size_t)i * stride] - minX) * s);
    int32_t y = or_js_toint32(((double)pos[(size_t)i * stride + 1] - minY) * s);
    int32_t z = or_js_toint32(((double)pos[(size_t)i * stride + 2] - minZ) * s);
    if (x > 1023) x = 1023;  // Math.min(…, 1023)
    if (y > 1023) y = 1023;
    if (z > 1023) z = 1023;
    codes[i] = or_part1by2((uint32_t)x) | (or_part1by2((uint32_t)y) << 1) |
               (or_part1by2((uint32_t)z) << 2);
  }
  return size;
}

// mortonTree.js:68-84 — stable LSD sort of the identity permutation by code,
// 3 passes of 10-bit digits, 1024-bin count + exclusive scan + stable scatter.
extern "C" void or_radix_sort_indices(const uint32_t* codes, uint32_t N, uint32_t* perm_out) {
  std::vector<uint32_t> indices(N), scratch(N);
  std::vector<uint32_t> counts(1024);
  for (uint32_t i = 0; i < N; i++) indices[i] = i;
  uint32_t* src = indices.data();
  uint32_t* dst = scratch.data();
  for (int pass = 0; pass < 3; pass++) {
    const uint32_t shift = pass * 10;
    std::fill(counts.begin(), counts.end(), 0u);
    for (uint32_t i = 0; i < N; i++) counts[(codes[src[i]] >> shift) & 1023]++;
    uint32_t sum = 0;
    for (uint32_t b = 0; b < 1024; b++) {
      const uint32_t c = counts[b];
      counts[b] = sum;
      sum += c;
    }
    for (uint32_t i = 0; i < N; i++) {
      const uint32_t v = src[i];
      dst[counts[(codes[v] >> shift) & 1023]++] = v;
    }
    std::swap(src, dst);
  }
  if (N) std::memcpy(perm_out, src, sizeof(uint32_t) * N);
}

// mortonTree.js:107-182 — breadth-first bucketed octree over Morton-sorted
// particles. Node numbering follows the BFS queue; every level's nodes are
// contiguous (level_ranges). COMs are summed in double, stored as f32.
extern "C" int64_t or_tree_build(const uint32_t* codes, const float* pos, const float* masses,
                                 uint32_t N, double rootSize, uint32_t maxNodes, or_node* nodes,
                                 uint32_t* level_ranges, uint32_t level_cap,
                                 uint32_t* n_levels) {
  struct Item {
    uint32_t lo, hi;
    int64_t parent;  // node index of the parent (-1 for the root)
    int slot;        // child slot in the parent
  };
  uint32_t numNodes = 0;
  uint32_t levels = 0;
  std::vector<Item> queue{{0, N, -1, 0}};
  uint32_t depth = 0;
  double size = rootSize;

  while (!queue.empty()) {
    std::vector<Item> next;
    const uint32_t levelStart = numNodes;
    for (const Item& item : queue) {
      const uint32_t idx = numNodes++;
      if (idx >= maxNodes) return -1;  // the JS typed array would drop these writes
      if (item.parent >= 0) nodes[item.parent].children[item.slot] = (int32_t)idx;
      or_node& nd = nodes[idx];
      const uint32_t count = item.hi - item.lo;
      nd.size = (float)size;

      const bool makeLeaf = count <= BUCKET || depth >= MAX_LEVEL || numNodes + 8 > maxNodes;
      if (makeLeaf) {
        double m = 0, cx = 0, cy = 0, cz = 0;
        for (uint32_t p = item.lo; p < item.hi; p++) {
          const double pm = masses[p];
          m += pm;
          cx += pos[(size_t)p * 3] * pm;
          cy += pos[(size_t)p * 3 + 1] * pm;
          cz += pos[(size_t)p * 3 + 2] * pm;
        }
        const double inv = m > 0 ? 1 / m : 0;
        nd.com[0] = (float)(cx * inv);
        nd.com[1] = (float)(cy * inv);
        nd.com[2] = (float)(cz * inv);
        nd.mass = (float)m;
        nd.isLeaf = 1;
        nd.first = item.lo;
        nd.count = count;
        for (int c = 0; c < 8; c++) nd.children[c] = -1;
      } else {
        nd.isLeaf = 0;
        nd.first = 0;
        nd.count = 0;
        const uint32_t shift = 27 - 3 * depth;
        uint32_t start = item.lo;
        for (uint32_t k = 0; k < 8; k++) {
          uint32_t end = start;
          while (end < item.hi && ((codes[end] >> shift) & 7) == k) end++;
          if (end > start) {
            next.push_back({start, end, (int64_t)idx, (int)k});
          } else {
            nd.children[k] = -1;
          }
          start = end;
        }
      }
    }
    if (levels >= level_cap) return -1;
    level_ranges[2 * levels] = levelStart;
    level_ranges[2 * levels + 1] = numNodes - levelStart;
    levels++;
    queue.swap(next);
    depth++;
    size *= 0.5;
  }

  // Bottom-up COM pass for internal nodes (mortonTree.js:166-181).
  for (int64_t n = (int64_t)numNodes - 1; n >= 0; n--) {
    or_node& nd = nodes[n];
    if (nd.isLeaf == 1) continue;
    double m = 0, cx = 0, cy = 0, cz = 0;
    for (int c = 0; c < 8; c++) {
      const int32_t ch = nd.children[c];
      if (ch >= 0) {
        const or_node& cn = nodes[ch];
        const double cm = cn.mass;
        m += cm;
        cx += (double)cn.com[0] * cm;
        cy += (double)cn.com[1] * cm;
        cz += (double)cn.com[2] * cm;
      }
    }
    const double inv = m > 0 ? 1 / m : 0;
    nd.com[0] = (float)(cx * inv);
    nd.com[1] = (float)(cy * inv);
    nd.com[2] = (float)(cz * inv);
    nd.mass = (float)m;
  }
  *n_levels = levels;
  return numNodes;
}

// mortonTree.js:192-224 — bootstrap: codes over the 8-float records, sort,
// gather full particle + stellar records, track the central particles, build.
extern "C" int64_t or_sort_and_build(const float* particles8, const float* stellar4, uint32_t N,
                                     int64_t trackIdx2, float* sorted8, float* sorted_stellar4,
                                     uint32_t* perm, or_node* nodes, uint32_t maxNodes,
                                     uint32_t* level_ranges, uint32_t level_cap,
                                     uint32_t* n_levels, int64_t* centralIdx,
                                     int64_t* centralIdx2, float* sorted_mass,
                                     double* rootSize_out) {
  std::vector<uint32_t> codes(N), sortedCodes(N);
  std::vector<float> sortedPos((size_t)N * 3);
  const double rootSize = or_compute_morton_codes(particles8, N, 8, codes.data());
  or_radix_sort_indices(codes.data(), N, perm);
  int64_t c1 = 0, c2 = -1;
  for (uint32_t i = 0; i < N; i++) {
    const uint32_t s = perm[i];
    if (s == 0) c1 = i;
    if ((int64_t)s == trackIdx2) c2 = i;
    std::memcpy(sorted8 + (size_t)i * 8, particles8 + (size_t)s * 8, 32);
    std::memcpy(sorted_stellar4 + (size_t)i * 4, stellar4 + (size_t)s * 4, 16);
    sortedCodes[i] = codes[s];
    sortedPos[(size_t)i * 3] = particles8[(size_t)s * 8];
    sortedPos[(size_t)i * 3 + 1] = particles8[(size_t)s * 8 + 1];
    sortedPos[(size_t)i * 3 + 2] = particles8[(size_t)s * 8 + 2];
    sorted_mass[i] = particles8[(size_t)s * 8 + 3];
  }
  *centralIdx = c1;
  *centralIdx2 = c2;
  if (rootSize_out) *rootSize_out = rootSize;
  return or_tree_build(sortedCodes.data(), sortedPos.data(), sorted_mass, N, rootSize, maxNodes,
                       nodes, level_ranges, level_cap, n_levels);
}

// bhWorker.js:55-94 — one asynchronous rebuild from a vec4 position readback
// (w = per-particle specific energy). `masses` tracks the current GPU order
// and is re-gathered through the emitted permutation.
extern "C" int64_t or_worker_build(const float* pos4, uint32_t N, float* masses,
                                   int64_t* centralIdx, int64_t* centralIdx2, or_node* nodes,
                                   uint32_t maxNodes, uint32_t* level_ranges, uint32_t level_cap,
                                   uint32_t* n_levels, uint32_t* perm, double* energy_out,
                                   float* bh1, float* bh2) {
  std::vector<uint32_t> codes(N), sortedCodes(N);
  std::vector<float> sortedPos((size_t)N * 3), sortedMass(N);
  const double rootSize = or_compute_morton_codes(pos4, N, 4, codes.data());
  or_radix_sort_indices(codes.data(), N, perm);
  double energy = 0;
  int64_t nc = *centralIdx, nc2 = *centralIdx2;
  for (uint32_t i = 0; i < N; i++) {
    const uint32_t s = perm[i];
    if ((int64_t)s == *centralIdx) nc = i;
    if ((int64_t)s == *centralIdx2) nc2 = i;
    sortedPos[(size_t)i * 3] = pos4[(size_t)s * 4];
    sortedPos[(size_t)i * 3 + 1] = pos4[(size_t)s * 4 + 1];
    sortedPos[(size_t)i * 3 + 2] = pos4[(size_t)s * 4 + 2];
    sortedMass[i] = masses[s];
    sortedCodes[i] = codes[s];
    energy += pos4[(size_t)i * 4 + 3];
  }
  *centralIdx = nc;
  *centralIdx2 = nc2;
  if (N) std::memcpy(masses, sortedMass.data(), sizeof(float) * N);
  const int64_t nn = or_tree_build(sortedCodes.data(), sortedPos.data(), masses, N, rootSize,
                                   maxNodes, nodes, level_ranges, level_cap, n_levels);
  *energy_out = energy;
  if (N && nc >= 0 && nc < (int64_t)N)
    for (int c = 0; c < 3; c++) bh1[c] = sortedPos[(size_t)nc * 3 + c];
  if (N && nc2 >= 0 && nc2 < (int64_t)N)
    for (int c = 0; c < 3; c++) bh2[c] = sortedPos[(size_t)nc2 * 3 + c];
  return nn;
}

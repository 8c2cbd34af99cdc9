// TEST INFRASTRUCTURE ONLY — CPU oracle of one full simulation step as the
// CUDA path runs it: the reference's frame (src/main.js:429-480) with the tree
// rebuilt from the current state every step instead of asynchronously.
//   codes (mortonTree.js:43-62, stride 8) -> sort (:68-84) -> gather particle +
//   stellar records (nbody_bh.wgsl:322-340) with central tracking
//   (bhWorker.js:67-68) -> halo-centre EMA (main.js:449-457) -> build
//   (mortonTree.js:107-182) -> refresh (nbody_bh.wgsl:289-313) -> walk +
//   halo + kick-drift (nbody_bh.wgsl:64-181) -> star formation (:230-268).
// The sort/build half runs on one thread like the reference's Web Worker; the
// refresh/walk half uses `nthreads` OpenMP threads.
#include <omp.h>

#include <cstring>
#include <vector>

#include "oracle.h"

extern "C" int or_full_step(or_params* p, or_pipeline_state* st, float* P, float* S,
                            float* P2, float* S2, float* energy, int do_sf, int nthreads,
                            uint32_t walk_stride, double* t_build, double* t_walk) {
  const uint32_t N = p->N;
  const double t0 = omp_get_wtime();
  std::vector<uint32_t> codes(N), perm(N), sortedCodes(N);
  std::vector<float> pos3((size_t)N * 3), mass(N);
  const double rootSize = or_compute_morton_codes(P, N, 8, codes.data());
  or_radix_sort_indices(codes.data(), N, perm.data());
  int64_t nc[2] = {st->central[0], st->central[1]};
  for (uint32_t i = 0; i < N; i++) {
    const uint32_t s = perm[i];
    for (int h = 0; h < 2; h++)
      if ((int64_t)s == st->central[h]) nc[h] = i;
    std::memcpy(P2 + (size_t)i * 8, P + (size_t)s * 8, 32);
    std::memcpy(S2 + (size_t)i * 4, S + (size_t)s * 4, 16);
    sortedCodes[i] = codes[s];
    pos3[(size_t)i * 3] = P[(size_t)s * 8];
    pos3[(size_t)i * 3 + 1] = P[(size_t)s * 8 + 1];
    pos3[(size_t)i * 3 + 2] = P[(size_t)s * 8 + 2];
    mass[i] = P[(size_t)s * 8 + 3];
  }
  for (int h = 0; h < 2; h++) {
    st->central[h] = nc[h];
    if (nc[h] < 0 || nc[h] >= (int64_t)N) continue;
    for (int c = 0; c < 3; c++)
      st->haloC[h][c] += ((double)P2[(size_t)nc[h] * 8 + c] - st->haloC[h][c]) * 0.1;
  }
  for (int c = 0; c < 3; c++) {
    p->haloC1[c] = (float)st->haloC[0][c];
    p->haloC2[c] = (float)st->haloC[1][c];
  }
  const uint32_t maxNodes = 2 * N + 4096;
  std::vector<or_node> nodes(maxNodes);
  std::vector<uint32_t> lr(64);
  uint32_t nLevels = 0;
  const int64_t nn = or_tree_build(sortedCodes.data(), pos3.data(), mass.data(), N, rootSize,
                                   maxNodes, nodes.data(), lr.data(), 32, &nLevels);
  if (nn < 0) return -1;
  const double t1 = omp_get_wtime();
  or_refresh_f32(P2, nodes.data(), lr.data(), nLevels);
  p->time = (float)st->time;
  if (walk_stride > 1) {
    std::memcpy(P, P2, sizeof(float) * 8 * (size_t)N);
    or_step_f32_sample(p, P2, P, nodes.data(), energy, walk_stride, nthreads);
  } else {
    or_step_f32(p, P2, P, nodes.data(), energy, nullptr, nullptr, nullptr, nthreads);
  }
  if (do_sf) {
    // the stellar records live in S2 (gathered); the step wrote particles to P
    or_star_formation(p, P, S2);
  }
  std::memcpy(S, S2, sizeof(float) * 4 * (size_t)N);
  st->time += p->dt;
  const double t2 = omp_get_wtime();
  if (t_build) *t_build = t1 - t0;
  if (t_walk) *t_walk = t2 - t1;
  return 0;
}

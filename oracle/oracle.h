/*
 * TEST INFRASTRUCTURE ONLY — the CPU oracle for the gravity path.
 *
 * This header declares a plain-C restatement of galaxy-sim's gravity path:
 *   - src/physics/mortonTree.js   (Morton codes, LSD radix sort, BFS bucketed octree)
 *   - src/physics/bhWorker.js     (per-rebuild gather, central tracking, energy sum)
 *   - src/physics/shaders/nbody_bh.wgsl (COM refresh, BH walk, Hernquist halo,
 *     kick-drift, star formation, permutation gather, position compaction)
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * this code, and only as the test reference or the timed CPU baseline. The product
 * path (galaxy_sim_b200) never calls it.
 *
 * Parity pinning: the reference's own tests pin only the gather direction
 * out[i] = in[perm[i]] (test/StarSelection.test.js:51-57). The reference is
 * JavaScript + WGSL and no JS engine or WebGPU stack exists on either machine,
 * so every other result of this restatement is "parity unpinned" against the
 * reference itself: it is a line-by-line restatement checked against hand-
 * derived known answers (tests/test_oracle.py) and committed golden vectors.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 64-byte BHNode, nbody_bh.wgsl:47-54 == mortonTree.js:12-20 */
typedef struct or_node {
  float com[3];
  float mass;
  float size;
  uint32_t isLeaf;
  uint32_t first;
  uint32_t count;
  int32_t children[8];
} or_node;

/* 96-byte Params uniform, nbody_bh.wgsl:19-42, writer NBodyGPU.js:253-275 */
typedef struct or_params {
  float dt, G, epsilon2;
  uint32_t N;
  float theta, haloMass, haloA, gasDrag, time, agingRate, sfDensity, sfEff, sfDt;
  uint32_t haloCount;
  float pad0, pad1;
  float haloC1[4];
  float haloC2[4];
} or_params;

/* ---- mortonTree.js ---- */
uint32_t or_part1by2(uint32_t v);
int32_t or_js_toint32(double d);
double or_compute_morton_codes(const float* pos, uint32_t N, uint32_t stride, uint32_t* codes);
void or_radix_sort_indices(const uint32_t* codes, uint32_t N, uint32_t* perm_out);
/* returns numNodes, or -1 if the node pool (maxNodes) or level table would overflow */
int64_t or_tree_build(const uint32_t* sorted_codes, const float* pos3, const float* masses,
                      uint32_t N, double rootSize, uint32_t maxNodes, or_node* nodes,
                      uint32_t* level_ranges, uint32_t level_cap, uint32_t* n_levels);
int64_t or_sort_and_build(const float* particles8, const float* stellar4, uint32_t N,
                          int64_t trackIdx2, float* sorted8, float* sorted_stellar4,
                          uint32_t* perm, or_node* nodes, uint32_t maxNodes,
                          uint32_t* level_ranges, uint32_t level_cap, uint32_t* n_levels,
                          int64_t* centralIdx, int64_t* centralIdx2, float* sorted_mass,
                          double* rootSize);
/* bhWorker.js:55-94 — masses is updated in place to the new (sorted) order */
int64_t or_worker_build(const float* pos4, uint32_t N, float* masses, int64_t* centralIdx,
                        int64_t* centralIdx2, or_node* nodes, uint32_t maxNodes,
                        uint32_t* level_ranges, uint32_t level_cap, uint32_t* n_levels,
                        uint32_t* perm, double* energy, float* bh1, float* bh2);

/* ---- nbody_bh.wgsl ---- */
void or_apply_permutation(const float* in, float* out, const uint32_t* perm, uint32_t N,
                          uint32_t width);
void or_refresh_f32(const float* particles8, or_node* nodes, const uint32_t* level_ranges,
                    uint32_t n_levels);
void or_refresh_f64(const float* particles8, const or_node* nodes, uint32_t numNodes,
                    const uint32_t* level_ranges, uint32_t n_levels, double* com4);
/* counters: [0] monopole interactions, [1] leaf pair interactions, [2] nodes visited */
void or_step_f32(const or_params* p, const float* pin, float* pout, const or_node* nodes,
                 float* energy, float* acc4, float* density, uint64_t* counters, int nthreads);
void or_walk_f64(const or_params* p, const float* pin, const or_node* nodes, const double* com4,
                 double* acc3, double* pot, float* density, uint64_t* counters, int nthreads);
void or_direct_f64(const or_params* p, const float* pin, const uint32_t* targets, uint32_t nT,
                   double* acc3, double* pot, int nthreads);
void or_halo_f64(const or_params* p, const float* pin, const uint32_t* targets, uint32_t nT,
                 double* acc3, double* pot);
void or_star_formation(const or_params* p, float* particles8, float* stellar4);
void or_compact_positions(const float* particles8, const float* energy, uint32_t N, float* out4);
uint32_t or_pcg(uint32_t v);
float or_rand01(uint32_t i, uint32_t salt);
float or_imf_sample(float u1, float u2);

/* ---- full on-device-style step, the sequence the CUDA step runs ----
 * per step: codes(stride 8) -> sort -> gather particles+stellar -> build ->
 * refresh -> walk/halo/kick-drift -> [star formation] ; the halo centres
 * follow the tracked central particles by the main.js:449-457 EMA (k = 0.1). */
typedef struct or_pipeline_state {
  double haloC[2][3];     /* smoothed halo centres (JS numbers = double) */
  int64_t central[2];     /* tracked particle indices, -1 = none */
  double time;            /* simulation time (JS number) */
} or_pipeline_state;
/* walk_stride > 1 walks only every walk_stride-th particle (a bounded timing
 * sample; the others keep their gathered state). */
int or_full_step(or_params* p, or_pipeline_state* st, float* particles8, float* stellar4,
                 float* scratch8, float* scratch_stellar4, float* energy, int do_sf,
                 int nthreads, uint32_t walk_stride, double* t_build, double* t_walk);
void or_step_f32_sample(const or_params* p, const float* pin, float* pout, const or_node* nodes,
                        float* energy, uint32_t stride, int nthreads);

#ifdef __cplusplus
}
#endif

/*
 * galaxy_b200 — C ABI of the B200 (sm_100a) gravity path of galaxy-sim.
 *
 * This is the drop-in boundary for the reference's compute surface:
 *   - the NBodyGPU class, src/physics/NBodyGPU.js:14-369 (one gs_ctx per
 *     NBodyGPU instance; the WebGPU command encoder maps to the context's
 *     CUDA stream order), and
 *   - the exports of src/physics/mortonTree.js (computeMortonCodes,
 *     radixSortIndices, MortonTree.build, sortAndBuild) and the rebuild of
 *     src/physics/bhWorker.js, which run on the GPU here instead of a Web Worker.
 *
 * Conventions
 *   - Every entry point returns an int status (GS_OK = 0, negative on error)
 *     and never aborts; gs_last_error() describes the last failure of a context
 *     (gs_last_error(NULL) the last context-free failure of the calling thread).
 *   - Host pointers are borrowed for the duration of the call only.
 *   - A context owns all of its device memory; one context = one CUDA stream =
 *     one host thread at a time.
 *   - Particle records keep the reference's 32-byte layout
 *     [x, y, z, m, vx, vy, vz, pad] (nbody_bh.wgsl:10-17) and the 16-byte
 *     stellar layout [stellarMass, birthMyr, seed, dust] (NBodyGPU.js:83-90);
 *     tree nodes the 64-byte BHNode layout (nbody_bh.wgsl:47-54 ==
 *     mortonTree.js:12-20); params the 96-byte Params uniform
 *     (nbody_bh.wgsl:19-42, NBodyGPU.js:253-275).
 *   - The particle buffers ping-pong: step and applyPermutation flip them,
 *     exactly as NBodyGPU.js:236-237, :328 do.
 */
#ifndef GALAXY_B200_H
#define GALAXY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GS_OK 0
#define GS_EINVAL (-1)     /* bad argument (N, pointer, size, layout) */
#define GS_ENOMEM (-2)     /* device or pinned-host allocation failed */
#define GS_ECUDA (-3)      /* a CUDA runtime call failed */
#define GS_ETIMEDOUT (-4)  /* a bounded host wait expired */
#define GS_EDEVICE (-5)    /* a kernel raised its error word (see gs_last_error) */
#define GS_ENOTREADY (-6)  /* the operation needs state that is not there yet */

/* device error-word bits (gs_device_errors) */
#define GS_DERR_LOOKBACK 0x1u   /* sort look-back wait exceeded its iteration limit */
#define GS_DERR_STACK 0x2u      /* walk stack deeper than the tree can be */
#define GS_DERR_NODES 0x4u      /* node pool exhausted */
#define GS_DERR_TREE 0x8u       /* uploaded tree is not a BFS tree with contiguous children */

typedef struct gs_ctx gs_ctx;

/* 96-byte Params uniform (nbody_bh.wgsl:19-42). epsilon2 below the smallest
 * normal float (1.17549435e-38) is walked as no softening: each particle's own
 * pair is then skipped instead of summed. */
typedef struct gs_params {
  float dt, G, epsilon2;
  uint32_t N;
  float theta, haloMass, haloA, gasDrag, time, agingRate, sfDensity, sfEff, sfDt;
  uint32_t haloCount;
  float pad0, pad1;
  float haloC1[4];
  float haloC2[4];
} gs_params;

/* 64-byte BHNode (nbody_bh.wgsl:47-54). */
typedef struct gs_node {
  float com[3];
  float mass;
  float size;
  uint32_t isLeaf;
  uint32_t first;
  uint32_t count;
  int32_t children[8];
} gs_node;

/* Energy and momentum diagnostics (nbody_bh.wgsl:180, bhWorker.js:74). */
typedef struct gs_diag {
  double e_diag;      /* sum of the specific energies e_i the step wrote (the HUD's E) */
  double e_true;      /* sum of m_i (1/2 v_i^2 + 1/2 phi_pair_i + phi_halo_i) */
  double momentum[3]; /* sum of m_i v_i */
  double mass;        /* sum of m_i */
} gs_diag;

const char* gs_last_error(const gs_ctx* ctx);
const char* gs_version(void);
/* Number of CUDA devices visible; returns GS_OK and writes the count. */
int gs_device_count(int* count);

/* ---- NBodyGPU surface (NBodyGPU.js) ---------------------------------------------- */

/* NBodyGPU constructor + _init (NBodyGPU.js:15-203): both ping-pong buffers get
 * the initial particles, both stellar buffers the stellar records. */
int gs_create(uint32_t N, const float* particles8, const float* stellar4, gs_ctx** out);
/* Same on an explicit CUDA device ordinal. */
int gs_create_on(int device, uint32_t N, const float* particles8, const float* stellar4,
                 gs_ctx** out);
/* NBodyGPU.destroy (NBodyGPU.js:358-368). */
int gs_destroy(gs_ctx* ctx);
/* NBodyGPU.updateParams (NBodyGPU.js:253-275); N is forced to the context's N.
 * Queued on the context's stream after the work already queued, without waiting
 * for it (the reference's writeBuffer is a queue write too); params may be reused
 * on return. */
int gs_update_params(gs_ctx* ctx, const gs_params* params);
/* Simulation clock (main.js simTime, a double): full steps stamp
 * Params.time = f32(simTime) and advance it by dt. gs_update_params sets it to
 * Params.time; this sets it exactly. */
int gs_set_time(gs_ctx* ctx, double t);
/* COM arithmetic of the on-device build's refresh: 0 = FP32 like refresh_level
 * (nbody_bh.wgsl:289-313), 2 = FP32 leaves with FP64 internal-node sums. */
int gs_set_com_mode(gs_ctx* ctx, int mode);
/* Whether star formation (gs_star_formation, and gs_run with do_sf) acts on
 * this galaxy; on by default, as the reference encodes it every frame. Off lets
 * galaxies with and without star formation share a pool. */
int gs_set_star_formation(gs_ctx* ctx, int enable);
/* Walk arithmetic: 0 = plain FP32 sums (default), 1 = far-field (monopole)
 * contributions accumulated with compensation: each walk round's terms are
 * summed plainly and the round's sum is added to the total with a Kahan step.
 * Together with gs_set_com_mode this selects the precision variant; no
 * counterpart in the reference. */
int gs_set_walk_mode(gs_ctx* ctx, int compensated);
/* Launch tuning (no counterpart in the reference). Takes effect at the next step;
 * galaxy_sim_b200/autotune.py picks values by timing.
 * GS_TUNE_WALK_BLOCKS_PER_SM = persistent walk blocks per SM (1..8; default 7 for a
 * gs_create context, 8 for a pool; below 8 the walk built for 72 registers per
 * thread runs); never changes results.
 * GS_TUNE_SORT_ITEMS = keys per thread of a sort tile (4, 8 or 16, or 0 = by the
 * largest galaxy's size: 4 up to 131072 particles, 8 up to 393216, else 16;
 * default 0 for a gs_create context, 16 for a pool); never
 * changes results (a stable sort has one answer).
 * GS_TUNE_WALK_GROUP = particles a warp walks together: 32 (one lane per particle),
 * 16, 8 or 4 (two, four or eight lanes per particle, splitting its node tests and
 * leaf sources), or 0 = by each galaxy's size (8 up to 45000 particles, 16 up to
 * 100000, else 32). Default: 0 for a gs_create context (a small galaxy alone needs
 * the smaller groups to fill the GPU), 32 for a pool (many galaxies fill it; 32
 * costs the fewest instructions). The split changes the order of the force sums,
 * so results differ at the rounding level (inside the force tolerance) between
 * group sizes; with the same setting a galaxy gets the same result alone or
 * pooled.
 * GS_TUNE_WALK_SPLIT = parts each work item's walk is split into when the context
 * walks one galaxy in groups of 16 or fewer particles (1, 2, 4 or 8, or 0 = by
 * its size: 4 up to 12000 particles, 2 up to 24000, else 1). The parts walk
 * disjoint subtrees in parallel and the last to finish adds their sums in a
 * fixed order, so a small galaxy's walk is less bound by its densest work
 * items. Default: 0 for a gs_create context, 1 for a pool; groups of 32 and a
 * pool holding more than one galaxy always walk unsplit. Like the group size it
 * changes only the order of the force sums. */
#define GS_TUNE_WALK_BLOCKS_PER_SM 1
#define GS_TUNE_SORT_ITEMS 2
#define GS_TUNE_WALK_GROUP 3
#define GS_TUNE_WALK_SPLIT 4
int gs_set_tuning(gs_ctx* ctx, int knob, int value);
int gs_get_tuning(gs_ctx* ctx, int knob, int* value);
/* The launch setting in effect for the selected galaxy after the knobs' "by size"
 * rules: particles per walk group (4, 8, 16, 32), walk parts per work item (1, 2,
 * 4, 8) and sort keys per thread (4, 8, 16). Any pointer may be NULL. */
int gs_get_launch_setting(gs_ctx* ctx, uint32_t* group, uint32_t* split, uint32_t* sort_items);
/* NBodyGPU.updateCentralMass (NBodyGPU.js:245-251): both ping-pong buffers. */
int gs_update_central_mass(gs_ctx* ctx, float mass, uint32_t idx);
/* NBodyGPU.applyPermutation (NBodyGPU.js:225-238): gather out[i] = in[perm[i]] of
 * particles and stellar records, then flip both ping-pongs. perm is a host array.
 * In a pool holding other galaxies the gathered records are copied back into the
 * current buffers instead of flipping them. */
int gs_apply_permutation(gs_ctx* ctx, const uint32_t* perm);
/* NBodyGPU.uploadBHTree (NBodyGPU.js:288-301): level_ranges holds n_levels
 * [start, count] pairs (at most 16, like the reference's refresh uniform). */
int gs_upload_tree(gs_ctx* ctx, const gs_node* nodes, uint32_t num_nodes,
                   const uint32_t* level_ranges, uint32_t n_levels);
/* NBodyGPU.encodeRefresh (NBodyGPU.js:308-319) → refresh_level deepest first. */
int gs_refresh(gs_ctx* ctx);
/* NBodyGPU.step (NBodyGPU.js:321-329): walk + halo + kick-drift, flip. */
int gs_step(gs_ctx* ctx);
/* NBodyGPU.encodeStarFormation (NBodyGPU.js:278-285). */
int gs_star_formation(gs_ctx* ctx);
/* encodePositionReadback + readPositions (NBodyGPU.js:335-350): vec4(pos, e_i)
 * per particle into out4 (N*4 floats); waits at most timeout_ns (0 = no limit). */
int gs_read_positions(gs_ctx* ctx, float* out4, uint64_t timeout_ns);
/* The same readback without waiting, as the reference drives it: encodePositionReadback
 * (NBodyGPU.js:334-341) queues the compaction and copy behind the work already
 * queued, and the promise of readPositions (NBodyGPU.js:344-348) resolves later while
 * main.js:485-501 keeps stepping with at most one readback in flight.
 * gs_encode_position_readback queues vec4(pos, e_i) of the selected galaxy into out4
 * (N*4 floats) and, if diag is not NULL, that galaxy's energy/momentum diagnostics as
 * of the same point, then returns. The copy runs on a second stream: with out4 in
 * pinned host memory it overlaps the steps queued after it (pageable memory works but
 * the call then returns only when the copy is done). out4 and diag must stay valid
 * until gs_await_position_readback returns GS_OK. A second encode while one is in
 * flight returns GS_ENOTREADY. The first call sets up the copy stream and a small
 * pinned block. gs_await_position_readback waits at most timeout_ns (0 = no limit;
 * GS_ETIMEDOUT leaves the readback in flight), fills diag and returns GS_EDEVICE if
 * the galaxy's device error word was set at that point. */
int gs_encode_position_readback(gs_ctx* ctx, float* out4, gs_diag* diag);
int gs_await_position_readback(gs_ctx* ctx, uint64_t timeout_ns);
/* positionBuffer / stellarBuffer getters (NBodyGPU.js:241-243, :353-356):
 * device pointers of the current buffers (valid until the next flip). */
int gs_position_buffer(gs_ctx* ctx, void** dptr);
int gs_stellar_buffer(gs_ctx* ctx, void** dptr);

/* ---- on-device rebuild (replaces the bhWorker.js round trip) ------------------------ */

/* Track up to two central particles (main.js:272-283) whose smoothed positions
 * centre the halos: c1/c2 are particle indices (-1 = none), halo_c* the
 * initial centres (NULL = the particle's current position). */
int gs_set_tracking(gs_ctx* ctx, int64_t c1, int64_t c2, const double* halo_c1,
                    const double* halo_c2);
int gs_get_tracking(gs_ctx* ctx, int64_t* c1, int64_t* c2, double* halo_c1, double* halo_c2);
/* Morton codes + stable sort + gather (particles, stellar, tracked indices) +
 * halo-centre EMA (main.js:449-457) + BFS bucketed octree + COM refresh, all on
 * the device: one bhWorker.js rebuild plus its application in main.js. */
int gs_sort_build(gs_ctx* ctx);
/* Full steps: nsteps x [gs_sort_build, walk + halo + kick-drift (+ star
 * formation when do_sf)], advancing Params.time by dt each step; replayed from a
 * CUDA graph. */
int gs_run(gs_ctx* ctx, uint32_t nsteps, int do_sf);
/* Kernel launches in one full step: the kernel nodes of the CUDA graph gs_run
 * captured last (0 before the first gs_run). */
int gs_step_kernels(gs_ctx* ctx, uint32_t* n);
/* The context's CUDA stream (cudaStream_t), e.g. to record timing events in
 * its order. */
int gs_stream(gs_ctx* ctx, void** stream);
/* Block until the context's stream is idle (bounded by timeout_ns, 0 = none). */
int gs_sync(gs_ctx* ctx, uint64_t timeout_ns);
/* Read the current tree in BHNode layout (+ level ranges, permutation of the last
 * gs_sort_build). Any output pointer may be NULL. */
int gs_get_tree(gs_ctx* ctx, gs_node* nodes, uint32_t nodes_cap, uint32_t* num_nodes,
                uint32_t* level_ranges, uint32_t lr_cap, uint32_t* n_levels, uint32_t* perm);
/* Raw state read/write (checkpoint): N*8 particle floats, N*4 stellar floats. */
int gs_read_state(gs_ctx* ctx, float* particles8, float* stellar4);
int gs_write_state(gs_ctx* ctx, const float* particles8, const float* stellar4);
/* Per-particle pair acceleration + potential {ax, ay, az, phi} (G applied, halo
 * excluded) and leaf density of the last walk; needs gs_set_debug(ctx, 1) first. */
int gs_set_debug(gs_ctx* ctx, int enable);
int gs_read_forces(gs_ctx* ctx, float* acc4, float* density);
/* FP64 diagnostics of the state the last step wrote. */
int gs_energy(gs_ctx* ctx, gs_diag* out);
/* Device error word (GS_DERR_* bits); clear=1 resets it. */
int gs_device_errors(gs_ctx* ctx, uint32_t* bits, int clear);
/* Interaction counters of the last walk(s): monopoles, leaf pairs, node visits. */
int gs_counters(gs_ctx* ctx, uint64_t out[3], int reset);

/* ---- mortonTree.js exports, stateless (host arrays in and out) ---------------------- */

/* computeMortonCodes (mortonTree.js:43-62): returns rootSize through root_size. */
int gs_morton_codes(const float* pos, uint32_t N, uint32_t stride, uint32_t* codes,
                    double* root_size);
/* radixSortIndices (mortonTree.js:68-84): stable sort -> gather permutation. */
int gs_radix_sort_indices(const uint32_t* codes, uint32_t N, uint32_t* perm);
/* Failure-detection test setting of gs_radix_sort_indices (and of
 * gs_radix_sort_indices_noalloc), no counterpart in the reference. Every later
 * call of those two sorts runs its digit passes with a look-back wait of at
 * most spin_limit polls without progress (production: about a second) and,
 * when withhold_tile >= 0, with that sort tile never publishing its digit
 * counts, so the waits of the tiles after it run out: the call then returns
 * GS_EDEVICE (GS_DERR_LOOKBACK) instead of hanging, its permutation is
 * garbage, and every write stays inside the call's own buffers. The pools'
 * step graphs never use this setting. gs_test_sort_lookback(1u << 20, -1)
 * restores the production setting. */
int gs_test_sort_lookback(uint32_t spin_limit, int64_t withhold_tile);
/* Host-side fault injection for tests (no counterpart in the reference): after
 * nth further device allocations made by the library's contexts, the next one
 * fails as if the device were out of memory (it is reported as GS_ENOMEM and the
 * call unwinds like a real failure); the switch then disarms itself. nth = -1
 * disarms it. Nothing is injected on the device. */
int gs_test_fail_alloc(int64_t nth);
/* MortonTree.build (mortonTree.js:107-182) over sorted codes, stride-3 positions
 * and masses; max_nodes follows the MortonTree pool (2N + 4096 there). */
int gs_tree_build(const uint32_t* sorted_codes, const float* pos3, const float* masses,
                  uint32_t N, double root_size, uint32_t max_nodes, gs_node* nodes,
                  uint32_t* num_nodes, uint32_t* level_ranges, uint32_t lr_cap,
                  uint32_t* n_levels);
/* sortAndBuild (mortonTree.js:192-224). */
int gs_sort_and_build(const float* particles8, const float* stellar4, uint32_t N,
                      int64_t track_idx2, float* sorted8, float* sorted_stellar4,
                      uint32_t* perm, gs_node* nodes, uint32_t max_nodes, uint32_t* num_nodes,
                      uint32_t* level_ranges, uint32_t lr_cap, uint32_t* n_levels,
                      int64_t* central_idx, int64_t* central_idx2, float* sorted_mass);

/* ---- pools: many independent galaxies in one context ---------------------------------- */

/* No counterpart in the reference, which runs one simulation per page. A context
 * is a pool of galaxy slots over one set of device buffers; gs_sort_build,
 * gs_step, gs_refresh, gs_star_formation and gs_run act on every resident galaxy
 * at once, one launch per kernel (segmented sort, build and walk; a CUDA graph per
 * step in gs_run). The per-galaxy entry points above (gs_update_params, gs_set_time,
 * gs_update_central_mass, gs_apply_permutation, gs_upload_tree, gs_read_positions,
 * gs_position_buffer, gs_stellar_buffer, gs_set_tracking, gs_get_tracking,
 * gs_get_tree, gs_read_state, gs_write_state, gs_read_forces, gs_energy,
 * gs_device_errors, gs_counters, gs_set_star_formation) act on the selected slot
 * (gs_select, default 0) and use that galaxy's own indices; gs_set_com_mode,
 * gs_set_walk_mode, gs_set_debug and gs_set_tuning apply to the whole context.
 * gs_create makes a pool holding one galaxy in slot 0. Each galaxy's results equal
 * those of the same galaxy alone. */

/* Free and total device memory of a CUDA device (cudaMemGetInfo). */
int gs_device_memory(int device, uint64_t* free_bytes, uint64_t* total_bytes);
/* Device bytes gs_pool_create allocates for a capacity (admission by free HBM;
 * debug force buffers and BHNode staging come on demand on top). */
uint64_t gs_pool_bytes(uint64_t particle_capacity, uint32_t max_galaxies);
/* An empty pool for up to particle_capacity particles (in total, each galaxy
 * rounded up to a multiple of 256) and max_galaxies galaxies. */
int gs_pool_create(int device, uint64_t particle_capacity, uint32_t max_galaxies, gs_ctx** out);
/* Admit a galaxy: N particles (N*8 floats), optional stellar records (NULL =
 * zeros) and Params (NULL = zeros); its slot index is written to slot. Returns
 * GS_ENOMEM when no slot or no contiguous particle range is free. */
int gs_pool_add(gs_ctx* ctx, uint32_t N, const float* particles8, const float* stellar4,
                const gs_params* params, uint32_t* slot);
/* Release a galaxy's slot and particle range. */
int gs_pool_remove(gs_ctx* ctx, uint32_t slot);
/* Largest free contiguous particle range and number of free slots. */
int gs_pool_free(gs_ctx* ctx, uint64_t* largest_range, uint32_t* free_slots);
/* Select the slot the per-galaxy entry points act on. */
int gs_select(gs_ctx* ctx, uint32_t slot);
/* FP64 diagnostics of every slot's last walk (out[slot], zeros for empty slots),
 * cap entries at most. */
int gs_pool_energies(gs_ctx* ctx, gs_diag* out, uint32_t cap);

/* ---- allocation-free sort ------------------------------------------------------------- */

/* No counterpart in the reference. The stable radix sort of gs_radix_sort_indices
 * (same permutation) for callers that may not allocate device memory while they
 * run, such as a host's per-frame callback (cudaMalloc/cudaFree can synchronize
 * the device and stall the frame) or an engine that budgets device memory at
 * start-up. d_codes (N codes, only the low 30 bits count) and d_perm (N
 * indices) are device buffers the caller owns; stream is a cudaStream_t (NULL =
 * the default stream). The call allocates nothing: its scratch is one static
 * device array for at most 1048576 codes (about 13 MiB), held by every GPU that
 * loads the library until the process exits; larger N is rejected with
 * GS_EINVAL.
 * Set-up: under CUDA's default lazy module loading the array, and the code of
 * the sort's kernels, are committed on the device the first time the library
 * touches them. The first call on a device (and the first after the device's
 * context was reset) therefore does that set-up: it loads the array's module
 * and kernels and looks up the array's device address. A call with N == 0
 * does only this set-up and sorts nothing; make it at start-up, outside any
 * stream capture, so that later calls allocate nothing.
 * The call is synchronous: it reads the sort's error word back and waits for
 * the stream. It must never be made while its stream (or, in global capture
 * mode, any stream) is capturing; a capturing stream is rejected with
 * GS_EINVAL and the capture is left intact. Calls share the array, so calls
 * whose work overlaps on the GPU race: serialize them. Returns after the
 * stream has finished the sort. */
int gs_radix_sort_indices_noalloc(const uint32_t* d_codes, uint32_t N, uint32_t* d_perm,
                                  void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GALAXY_B200_H */

/*
 * Node-API addon: the binding that lets galaxy-sim's JavaScript host
 * (src/main.js) drive the CUDA gravity path through include/galaxy_b200.h.
 *
 *   const { NBodyCUDA, computeMortonCodes, radixSortIndices, buildTree,
 *           sortAndBuild } = require('./galaxy_napi.node');
 *
 * NBodyCUDA mirrors the NBodyGPU class (src/physics/NBodyGPU.js:14-369): the
 * same method names, argument meaning and buffer layouts, with a CUDA device
 * ordinal in place of the GPUDevice and the context's CUDA stream in place of
 * the GPUCommandEncoder (encoder arguments are accepted and ignored). As in
 * the reference, every method returns silently once the simulation is
 * destroyed (`if (!this.ready) return`). CUDA-side failures throw an Error
 * whose code is the status name (GS_EINVAL, GS_ENOMEM, ...) and whose message
 * is gs_last_error(); bad arguments throw TypeError / RangeError before any
 * CUDA call. Beyond the reference's surface: sortBuild() (the worker rebuild on
 * the device), run(steps, starFormation), energy(), setTracking(),
 * getTracking(), sync() and deviceErrors().
 *
 * The module functions mirror the exports of src/physics/mortonTree.js:
 * computeMortonCodes (:43-62), radixSortIndices (:68-84), MortonTree.build
 * (:107-182, as buildTree returning the tree's buffer, node count and level
 * ranges) and sortAndBuild (:192-224).
 *
 * Build (node-gyp, or directly):
 *   cc -shared -fPIC -I<node>/include/node -Iinclude addon/galaxy_napi.c \
 *      -Lgalaxy_sim_b200 -lgalaxy_b200 -o galaxy_napi.node
 */
#include <math.h>
#include <node_api.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "galaxy_b200.h"

typedef struct {
  gs_ctx* ctx;   /* NULL after destroy() */
  uint32_t N;
} Sim;

/* ---- errors ------------------------------------------------------------------------ */

static const char* status_name(int rc) {
  switch (rc) {
    case GS_EINVAL: return "GS_EINVAL";
    case GS_ENOMEM: return "GS_ENOMEM";
    case GS_ECUDA: return "GS_ECUDA";
    case GS_ETIMEDOUT: return "GS_ETIMEDOUT";
    case GS_EDEVICE: return "GS_EDEVICE";
    case GS_ENOTREADY: return "GS_ENOTREADY";
    default: return "GS_ERROR";
  }
}

/* Throw the library's error for status rc (ctx NULL: the thread's context-free error). */
static napi_value throw_gs(napi_env env, const gs_ctx* ctx, int rc) {
  const char* msg = gs_last_error(ctx);
  napi_throw_error(env, status_name(rc), msg && msg[0] ? msg : "gravity-path call failed");
  return NULL;
}

static napi_value throw_type(napi_env env, const char* what) {
  napi_throw_type_error(env, "ERR_INVALID_ARG_TYPE", what);
  return NULL;
}

static napi_value throw_range(napi_env env, const char* what) {
  napi_throw_range_error(env, "ERR_OUT_OF_RANGE", what);
  return NULL;
}

#define NAPI_OK(env, call)                                                   \
  do {                                                                       \
    if ((call) != napi_ok) {                                                 \
      bool _pending = false;                                                 \
      napi_is_exception_pending((env), &_pending);                           \
      if (!_pending) napi_throw_error((env), "ERR_NAPI", "Node-API call failed: " #call); \
      return NULL;                                                           \
    }                                                                        \
  } while (0)

#define GS_OK_OR_THROW(env, ctx, call)      \
  do {                                      \
    int _rc = (call);                       \
    if (_rc != GS_OK) return throw_gs((env), (ctx), _rc); \
  } while (0)

/* ---- argument helpers (each returns 0 and throws on a bad argument) -------------------- */

static napi_value undefined(napi_env env) {
  napi_value u = NULL;
  napi_get_undefined(env, &u);
  return u;
}

static int is_nullish(napi_env env, napi_value v) {
  napi_valuetype t = napi_undefined;
  if (!v || napi_typeof(env, v, &t) != napi_ok) return 1;
  return t == napi_undefined || t == napi_null;
}

static int get_typed(napi_env env, napi_value v, napi_typedarray_type want, const char* what, void** data,
                     size_t* length) {
  bool is = false;
  napi_typedarray_type t;
  napi_value ab;
  size_t off;
  if (!v || napi_is_typedarray(env, v, &is) != napi_ok || !is ||
      napi_get_typedarray_info(env, v, &t, length, data, &ab, &off) != napi_ok || t != want) {
    throw_type(env, what);
    return 0;
  }
  return 1;
}

static int get_f32(napi_env env, napi_value v, const char* what, float** data, size_t* n) {
  return get_typed(env, v, napi_float32_array, what, (void**)data, n);
}

static int get_u32a(napi_env env, napi_value v, const char* what, uint32_t** data, size_t* n) {
  return get_typed(env, v, napi_uint32_array, what, (void**)data, n);
}

static int get_num(napi_env env, napi_value v, const char* what, double* out) {
  napi_valuetype t;
  if (!v || napi_typeof(env, v, &t) != napi_ok || t != napi_number ||
      napi_get_value_double(env, v, out) != napi_ok) {
    throw_type(env, what);
    return 0;
  }
  return 1;
}

/* A JS number used as a count or index: finite, integral, within [lo, hi]. */
static int get_index(napi_env env, napi_value v, const char* what, double lo, double hi, int64_t* out) {
  double d;
  if (!get_num(env, v, what, &d)) return 0;
  if (!isfinite(d) || d != floor(d) || d < lo || d > hi) {
    throw_range(env, what);
    return 0;
  }
  *out = (int64_t)d;
  return 1;
}

/* obj[name] as a number; def when the property is absent or undefined (JS
 * destructuring defaults), NaN when it is present but not a number. */
static double prop_num(napi_env env, napi_value obj, const char* name, double def) {
  bool has = false;
  napi_value v;
  double d = def;
  if (napi_has_named_property(env, obj, name, &has) != napi_ok || !has) return def;
  if (napi_get_named_property(env, obj, name, &v) != napi_ok || is_nullish(env, v)) return def;
  if (napi_get_value_double(env, v, &d) != napi_ok) return NAN;
  return d;
}

/* Numbers of an array or typed array of numbers (up to cap); returns the count. */
static int read_numbers(napi_env env, napi_value v, double* out, uint32_t cap) {
  bool arr = false, ta = false;
  uint32_t n = 0;
  napi_is_array(env, v, &arr);
  napi_is_typedarray(env, v, &ta);
  if (ta) {
    float* f;
    size_t len;
    if (!get_f32(env, v, "halo centres must be arrays or Float32Arrays", &f, &len)) return -1;
    for (size_t i = 0; i < len && i < cap; i++) out[i] = f[i];
    return (int)(len < cap ? len : cap);
  }
  if (!arr || napi_get_array_length(env, v, &n) != napi_ok) {
    throw_type(env, "halo centres must be arrays or Float32Arrays");
    return -1;
  }
  for (uint32_t i = 0; i < n && i < cap; i++) {
    napi_value e;
    if (napi_get_element(env, v, i, &e) != napi_ok || napi_get_value_double(env, e, &out[i]) != napi_ok) {
      throw_type(env, "halo centre coordinates must be numbers");
      return -1;
    }
  }
  return (int)(n < cap ? n : cap);
}

static Sim* this_sim(napi_env env, napi_callback_info info, size_t* argc, napi_value* argv) {
  napi_value self;
  void* p = NULL;
  if (napi_get_cb_info(env, info, argc, argv, &self, NULL) != napi_ok) return NULL;
  if (napi_unwrap(env, self, &p) != napi_ok) return NULL;
  return (Sim*)p;
}

/* ---- NBodyCUDA ---------------------------------------------------------------------- */

static void sim_finalize(napi_env env, void* data, void* hint) {
  (void)env;
  (void)hint;
  Sim* s = (Sim*)data;
  if (s->ctx) gs_destroy(s->ctx);
  free(s);
}

/* new NBodyCUDA(device, particleData: Float32Array, stellarData?: Float32Array)
 * (NBodyGPU.js:15-22 + _init): both ping-pong buffers get the initial records. */
static napi_value Construct(napi_env env, napi_callback_info info) {
  size_t argc = 3;
  napi_value argv[3] = {NULL, NULL, NULL}, self;
  NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, &self, NULL));
  int64_t device = 0;
  if (argc > 0 && !is_nullish(env, argv[0]) && !get_index(env, argv[0], "device must be a CUDA device ordinal",
                                                           0, 1023, &device))
    return NULL;
  float *p = NULL, *st = NULL;
  size_t n8 = 0, n4 = 0;
  if (argc < 2 || !get_f32(env, argv[1], "particleData must be a Float32Array", &p, &n8)) return NULL;
  if (n8 == 0 || n8 % 8) return throw_range(env, "particleData must hold 8 floats per particle");
  const uint32_t N = (uint32_t)(n8 / 8);
  if (argc > 2 && !is_nullish(env, argv[2])) {
    if (!get_f32(env, argv[2], "stellarData must be a Float32Array", &st, &n4)) return NULL;
    if (n4 != 4 * (size_t)N) return throw_range(env, "stellarData must hold 4 floats per particle");
  }
  Sim* s = (Sim*)calloc(1, sizeof(Sim));
  if (!s) return throw_range(env, "out of host memory");
  const int rc = gs_create_on((int)device, N, p, st, &s->ctx);
  if (rc != GS_OK) {
    free(s);
    return throw_gs(env, NULL, rc);
  }
  s->N = N;
  if (napi_wrap(env, self, s, sim_finalize, NULL, NULL) != napi_ok) {
    gs_destroy(s->ctx);
    free(s);
    napi_throw_error(env, "ERR_NAPI", "napi_wrap failed");
    return NULL;
  }
  napi_value nv, t;
  napi_create_uint32(env, N, &nv);
  napi_set_named_property(env, self, "N", nv);
  napi_get_boolean(env, true, &t);
  napi_set_named_property(env, self, "ready", t);
  return self;
}

/* applyPermutation(encoder, perm: Uint32Array) (NBodyGPU.js:225-238): out[i] = in[perm[i]] */
static napi_value ApplyPermutation(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2] = {NULL, NULL};
  Sim* s = this_sim(env, info, &argc, argv);
  if (!s || !s->ctx) return undefined(env);
  uint32_t* perm;
  size_t n;
  if (!get_u32a(env, argc > 1 ? argv[1] : NULL, "perm must be a Uint32Array", &perm, &n)) return NULL;
  if (n < s->N) return throw_range(env, "perm must hold N indices");
  GS_OK_OR_THROW(env, s->ctx, gs_apply_permutation(s->ctx, perm));
  return undefined(env);
}

/* updateCentralMass(mass, idx = 0) (NBodyGPU.js:245-251) */
static napi_value UpdateCentralMass(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2] = {NULL, NULL};
  Sim* s = this_sim(env, info, &argc, argv);
  if (!s || !s->ctx) return undefined(env);
  double mass;
  int64_t idx = 0;
  if (!get_num(env, argc > 0 ? argv[0] : NULL, "mass must be a number", &mass)) return NULL;
  if (argc > 1 && !is_nullish(env, argv[1]) &&
      !get_index(env, argv[1], "idx must be a particle index", 0, (double)s->N - 1, &idx))
    return NULL;
  GS_OK_OR_THROW(env, s->ctx, gs_update_central_mass(s->ctx, (float)mass, (uint32_t)idx));
  return undefined(env);
}

/* updateParams({dt, G, epsilon, theta = 0.5, haloMass = 0, haloA = 1, gasDrag = 0,
 * time = 0, agingRate = 25, sfDensity = 1e9, sfEff = 0, sfDt = 0, haloCenters = []})
 * (NBodyGPU.js:253-275): every field stored as the Float32Array there stores it,
 * epsilon squared in double before the f32 store, at most two halo centres. */
static napi_value UpdateParams(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1] = {NULL};
  Sim* s = this_sim(env, info, &argc, argv);
  if (!s || !s->ctx) return undefined(env);
  napi_valuetype t;
  if (argc < 1 || napi_typeof(env, argv[0], &t) != napi_ok || t != napi_object)
    return throw_type(env, "updateParams takes an object");
  napi_value o = argv[0];
  gs_params p;
  memset(&p, 0, sizeof(p));
  const double eps = prop_num(env, o, "epsilon", NAN);
  p.dt = (float)prop_num(env, o, "dt", NAN);
  p.G = (float)prop_num(env, o, "G", NAN);
  p.epsilon2 = (float)(eps * eps);
  p.N = s->N;
  p.theta = (float)prop_num(env, o, "theta", 0.5);
  p.haloMass = (float)prop_num(env, o, "haloMass", 0.0);
  p.haloA = (float)prop_num(env, o, "haloA", 1.0);
  p.gasDrag = (float)prop_num(env, o, "gasDrag", 0.0);
  p.time = (float)prop_num(env, o, "time", 0.0);
  p.agingRate = (float)prop_num(env, o, "agingRate", 25.0);
  p.sfDensity = (float)prop_num(env, o, "sfDensity", 1e9);
  p.sfEff = (float)prop_num(env, o, "sfEff", 0.0);
  p.sfDt = (float)prop_num(env, o, "sfDt", 0.0);
  bool has = false;
  napi_value hc;
  if (napi_has_named_property(env, o, "haloCenters", &has) == napi_ok && has &&
      napi_get_named_property(env, o, "haloCenters", &hc) == napi_ok && !is_nullish(env, hc)) {
    bool arr = false;
    uint32_t n = 0;
    if (napi_is_array(env, hc, &arr) != napi_ok || !arr || napi_get_array_length(env, hc, &n) != napi_ok)
      return throw_type(env, "haloCenters must be an array");
    p.haloCount = n < 2 ? n : 2;
    for (uint32_t h = 0; h < p.haloCount; h++) {
      napi_value c;
      double v[4];
      if (napi_get_element(env, hc, h, &c) != napi_ok || is_nullish(env, c)) continue;  // `if (haloCenters[h])`
      const int k = read_numbers(env, c, v, 4);
      if (k < 0) return NULL;
      float* dst = h == 0 ? p.haloC1 : p.haloC2;
      for (int i = 0; i < k; i++) dst[i] = (float)v[i];
    }
  }
  GS_OK_OR_THROW(env, s->ctx, gs_update_params(s->ctx, &p));
  return undefined(env);
}

/* encodeStarFormation(encoder) (NBodyGPU.js:278-285) */
static napi_value EncodeStarFormation(napi_env env, napi_callback_info info) {
  size_t argc = 0;
  Sim* s = this_sim(env, info, &argc, NULL);
  if (!s || !s->ctx) return undefined(env);
  GS_OK_OR_THROW(env, s->ctx, gs_star_formation(s->ctx));
  return undefined(env);
}

/* uploadBHTree(treeBuffer: ArrayBuffer | typed array, numNodes, levelRanges?: [start, count][])
 * (NBodyGPU.js:288-301): at most the 16 level slots the refresh keeps. */
static napi_value UploadBHTree(napi_env env, napi_callback_info info) {
  size_t argc = 3;
  napi_value argv[3] = {NULL, NULL, NULL};
  Sim* s = this_sim(env, info, &argc, argv);
  if (!s || !s->ctx) return undefined(env);
  void* buf = NULL;
  size_t bytes = 0;
  bool is_ab = false, is_ta = false;
  if (argc > 0) {
    napi_is_arraybuffer(env, argv[0], &is_ab);
    napi_is_typedarray(env, argv[0], &is_ta);
  }
  if (is_ab) {
    NAPI_OK(env, napi_get_arraybuffer_info(env, argv[0], &buf, &bytes));
  } else if (is_ta) {
    napi_typedarray_type t;
    size_t len, off;
    napi_value ab;
    NAPI_OK(env, napi_get_typedarray_info(env, argv[0], &t, &len, &buf, &ab, &off));
    const size_t esz = (t == napi_float64_array || t == napi_bigint64_array || t == napi_biguint64_array) ? 8
                       : (t == napi_int16_array || t == napi_uint16_array) ? 2
                       : (t == napi_int8_array || t == napi_uint8_array || t == napi_uint8_clamped_array) ? 1 : 4;
    bytes = len * esz;
  } else {
    return throw_type(env, "treeBuffer must be an ArrayBuffer or a typed array");
  }
  int64_t num;
  if (!get_index(env, argc > 1 ? argv[1] : NULL, "numNodes must be a node count", 0, 4294967295.0, &num))
    return NULL;
  if ((uint64_t)num * 64 > bytes) return throw_range(env, "treeBuffer holds fewer than numNodes nodes");
  uint32_t lr[32];
  uint32_t nl = 0;
  int with_levels = argc > 2 && !is_nullish(env, argv[2]);
  if (with_levels) {
    bool arr = false;
    uint32_t n = 0;
    if (napi_is_array(env, argv[2], &arr) != napi_ok || !arr || napi_get_array_length(env, argv[2], &n) != napi_ok)
      return throw_type(env, "levelRanges must be an array of [start, count] pairs");
    nl = n < 16 ? n : 16;
    for (uint32_t l = 0; l < nl; l++) {
      napi_value pair, v;
      double d[2];
      for (int k = 0; k < 2; k++) {
        if (napi_get_element(env, argv[2], l, &pair) != napi_ok || napi_get_element(env, pair, (uint32_t)k, &v) != napi_ok ||
            napi_get_value_double(env, v, &d[k]) != napi_ok || !(d[k] >= 0) || d[k] > 4294967295.0)
          return throw_type(env, "levelRanges must be an array of [start, count] pairs");
        lr[2 * l + k] = (uint32_t)d[k];
      }
    }
  }
  GS_OK_OR_THROW(env, s->ctx, gs_upload_tree(s->ctx, (const gs_node*)buf, (uint32_t)num, with_levels ? lr : NULL,
                                             with_levels ? nl : 0));
  return undefined(env);
}

#define SIMPLE_METHOD(Name, call)                                 \
  static napi_value Name(napi_env env, napi_callback_info info) { \
    size_t argc = 0;                                              \
    Sim* s = this_sim(env, info, &argc, NULL);                    \
    if (!s || !s->ctx) return undefined(env);                     \
    GS_OK_OR_THROW(env, s->ctx, call(s->ctx));                    \
    return undefined(env);                                        \
  }

/* encodeRefresh(encoder) (NBodyGPU.js:308-319), step(encoder) (:321-329),
 * sortBuild(): the bhWorker.js rebuild on the device */
SIMPLE_METHOD(EncodeRefresh, gs_refresh)
SIMPLE_METHOD(Step, gs_step)
SIMPLE_METHOD(SortBuild, gs_sort_build)

/* encodePositionReadback(encoder) (NBodyGPU.js:335-343): the compaction runs
 * inside readPositions, in stream order, so there is nothing to encode. */
static napi_value EncodePositionReadback(napi_env env, napi_callback_info info) {
  size_t argc = 0;
  this_sim(env, info, &argc, NULL);
  return undefined(env);
}

/* readPositions(out: Float32Array) -> Promise (NBodyGPU.js:346-350): vec4(pos, e_i)
 * per particle. The copy completes before the promise is returned (resolved). */
static napi_value ReadPositions(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2] = {NULL, NULL};
  Sim* s = this_sim(env, info, &argc, argv);
  napi_deferred d;
  napi_value promise;
  NAPI_OK(env, napi_create_promise(env, &d, &promise));
  if (!s || !s->ctx) {
    napi_resolve_deferred(env, d, undefined(env));
    return promise;
  }
  float* out;
  size_t n;
  if (!get_f32(env, argc > 0 ? argv[0] : NULL, "out must be a Float32Array", &out, &n)) return NULL;
  if (n < 4 * (size_t)s->N) return throw_range(env, "out must hold 4 floats per particle");
  double timeout_ms = 0;
  if (argc > 1 && !is_nullish(env, argv[1]) && !get_num(env, argv[1], "timeoutMs must be a number", &timeout_ms))
    return NULL;
  const int rc = gs_read_positions(s->ctx, out, timeout_ms > 0 ? (uint64_t)(timeout_ms * 1e6) : 0);
  if (rc != GS_OK) {
    napi_value code, msg, err;
    napi_create_string_utf8(env, status_name(rc), NAPI_AUTO_LENGTH, &code);
    napi_create_string_utf8(env, gs_last_error(s->ctx), NAPI_AUTO_LENGTH, &msg);
    napi_create_error(env, code, msg, &err);
    napi_reject_deferred(env, d, err);
  } else {
    napi_resolve_deferred(env, d, undefined(env));
  }
  return promise;
}

static napi_value device_pointer(napi_env env, napi_callback_info info, int which) {
  size_t argc = 0;
  Sim* s = this_sim(env, info, &argc, NULL);
  if (!s || !s->ctx) return undefined(env);
  void* p = NULL;
  GS_OK_OR_THROW(env, s->ctx, which ? gs_stellar_buffer(s->ctx, &p) : gs_position_buffer(s->ctx, &p));
  napi_value v;
  NAPI_OK(env, napi_create_bigint_uint64(env, (uint64_t)(uintptr_t)p, &v));
  return v;
}

/* positionBuffer / stellarBuffer getters (NBodyGPU.js:241-243, :353-356): the
 * current device address, for a renderer that reads the buffers in place. */
static napi_value GetPositionBuffer(napi_env env, napi_callback_info info) { return device_pointer(env, info, 0); }
static napi_value GetStellarBuffer(napi_env env, napi_callback_info info) { return device_pointer(env, info, 1); }

/* destroy() (NBodyGPU.js:358-368): frees the device memory; later calls are no-ops. */
static napi_value Destroy(napi_env env, napi_callback_info info) {
  size_t argc = 0;
  napi_value self;
  void* p = NULL;
  NAPI_OK(env, napi_get_cb_info(env, info, &argc, NULL, &self, NULL));
  if (napi_unwrap(env, self, &p) == napi_ok && p) {
    Sim* s = (Sim*)p;
    if (s->ctx) gs_destroy(s->ctx);
    s->ctx = NULL;
    napi_value f;
    napi_get_boolean(env, false, &f);
    napi_set_named_property(env, self, "ready", f);
  }
  return undefined(env);
}

/* run(steps, starFormation = false): full steps (rebuild + walk [+ star formation]) */
static napi_value Run(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2] = {NULL, NULL};
  Sim* s = this_sim(env, info, &argc, argv);
  if (!s || !s->ctx) return undefined(env);
  int64_t steps;
  bool sf = false;
  if (!get_index(env, argc > 0 ? argv[0] : NULL, "steps must be a step count", 0, 4294967295.0, &steps))
    return NULL;
  if (argc > 1 && !is_nullish(env, argv[1]) && napi_get_value_bool(env, argv[1], &sf) != napi_ok)
    return throw_type(env, "starFormation must be a boolean");
  GS_OK_OR_THROW(env, s->ctx, gs_run(s->ctx, (uint32_t)steps, sf ? 1 : 0));
  return undefined(env);
}

/* sync(timeoutMs = 0): waits for the queued work (0 = no limit) */
static napi_value Sync(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1] = {NULL};
  Sim* s = this_sim(env, info, &argc, argv);
  if (!s || !s->ctx) return undefined(env);
  double ms = 0;
  if (argc > 0 && !is_nullish(env, argv[0]) && !get_num(env, argv[0], "timeoutMs must be a number", &ms)) return NULL;
  GS_OK_OR_THROW(env, s->ctx, gs_sync(s->ctx, ms > 0 ? (uint64_t)(ms * 1e6) : 0));
  return undefined(env);
}

static napi_value number_array(napi_env env, const double* v, uint32_t n) {
  napi_value a, x;
  if (napi_create_array_with_length(env, n, &a) != napi_ok) return NULL;
  for (uint32_t i = 0; i < n; i++) {
    napi_create_double(env, v[i], &x);
    napi_set_element(env, a, i, x);
  }
  return a;
}

static void set_num(napi_env env, napi_value o, const char* k, double v) {
  napi_value x;
  napi_create_double(env, v, &x);
  napi_set_named_property(env, o, k, x);
}

/* energy() -> {eDiag, eTrue, momentum: [x, y, z], mass}: FP64 diagnostics of the
 * last step (eDiag is the HUD's sum of e_i, bhWorker.js:74) */
static napi_value Energy(napi_env env, napi_callback_info info) {
  size_t argc = 0;
  Sim* s = this_sim(env, info, &argc, NULL);
  if (!s || !s->ctx) return undefined(env);
  gs_diag d;
  GS_OK_OR_THROW(env, s->ctx, gs_energy(s->ctx, &d));
  napi_value o;
  NAPI_OK(env, napi_create_object(env, &o));
  set_num(env, o, "eDiag", d.e_diag);
  set_num(env, o, "eTrue", d.e_true);
  set_num(env, o, "mass", d.mass);
  napi_set_named_property(env, o, "momentum", number_array(env, d.momentum, 3));
  return o;
}

/* setTracking(centralIdx, centralIdx2 = -1, halo1?, halo2?): the halo-centre EMA of
 * main.js:449-457 kept on the device for sortBuild / run */
static napi_value SetTracking(napi_env env, napi_callback_info info) {
  size_t argc = 4;
  napi_value argv[4] = {NULL, NULL, NULL, NULL};
  Sim* s = this_sim(env, info, &argc, argv);
  if (!s || !s->ctx) return undefined(env);
  int64_t c[2] = {-1, -1};
  double h[2][4];
  int have[2] = {0, 0};
  for (int k = 0; k < 2; k++) {
    if (argc > (size_t)k && !is_nullish(env, argv[k]) &&
        !get_index(env, argv[k], "central index must be a particle index or -1", -1, (double)s->N - 1, &c[k]))
      return NULL;
    if (argc > (size_t)(2 + k) && !is_nullish(env, argv[2 + k])) {
      const int n = read_numbers(env, argv[2 + k], h[k], 4);
      if (n < 0) return NULL;
      if (n < 3) return throw_range(env, "a halo centre needs three coordinates");
      have[k] = 1;
    }
  }
  GS_OK_OR_THROW(env, s->ctx, gs_set_tracking(s->ctx, c[0], c[1], have[0] ? h[0] : NULL, have[1] ? h[1] : NULL));
  return undefined(env);
}

/* getTracking() -> {centralIdx, centralIdx2, halo1: [x, y, z], halo2: [x, y, z]} */
static napi_value GetTracking(napi_env env, napi_callback_info info) {
  size_t argc = 0;
  Sim* s = this_sim(env, info, &argc, NULL);
  if (!s || !s->ctx) return undefined(env);
  int64_t c1, c2;
  double h1[3], h2[3];
  GS_OK_OR_THROW(env, s->ctx, gs_get_tracking(s->ctx, &c1, &c2, h1, h2));
  napi_value o;
  NAPI_OK(env, napi_create_object(env, &o));
  set_num(env, o, "centralIdx", (double)c1);
  set_num(env, o, "centralIdx2", (double)c2);
  napi_set_named_property(env, o, "halo1", number_array(env, h1, 3));
  napi_set_named_property(env, o, "halo2", number_array(env, h2, 3));
  return o;
}

/* deviceErrors(clear = false) -> GS_DERR_* bits of the device error word */
static napi_value DeviceErrors(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1] = {NULL};
  Sim* s = this_sim(env, info, &argc, argv);
  if (!s || !s->ctx) return undefined(env);
  bool clear = false;
  if (argc > 0 && !is_nullish(env, argv[0])) napi_get_value_bool(env, argv[0], &clear);
  uint32_t bits = 0;
  GS_OK_OR_THROW(env, s->ctx, gs_device_errors(s->ctx, &bits, clear ? 1 : 0));
  napi_value v;
  napi_create_uint32(env, bits, &v);
  return v;
}

/* ---- mortonTree.js exports ---------------------------------------------------------- */

/* computeMortonCodes(pos: Float32Array, N, stride, codes: Uint32Array) -> rootSize */
static napi_value ComputeMortonCodes(napi_env env, napi_callback_info info) {
  size_t argc = 4;
  napi_value argv[4] = {NULL, NULL, NULL, NULL};
  NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  float* pos;
  uint32_t* codes;
  size_t np, nc;
  int64_t N, stride;
  if (!get_f32(env, argv[0], "pos must be a Float32Array", &pos, &np) ||
      !get_index(env, argv[1], "N must be a particle count", 0, 4294967295.0, &N) ||
      !get_index(env, argv[2], "stride must be 3 or more", 3, 1 << 20, &stride) ||
      !get_u32a(env, argv[3], "codes must be a Uint32Array", &codes, &nc))
    return NULL;
  if (N && ((uint64_t)(N - 1) * stride + 3 > np || (uint64_t)N > nc))
    return throw_range(env, "pos or codes is shorter than N particles");
  double root = 0;
  GS_OK_OR_THROW(env, NULL, gs_morton_codes(pos, (uint32_t)N, (uint32_t)stride, codes, &root));
  napi_value v;
  NAPI_OK(env, napi_create_double(env, root, &v));
  return v;
}

/* radixSortIndices(codes, indices, scratch, counts, N) -> indices, holding the stable
 * gather order by the low 30 bits (scratch and counts are accepted for the signature) */
static napi_value RadixSortIndices(napi_env env, napi_callback_info info) {
  size_t argc = 5;
  napi_value argv[5] = {NULL, NULL, NULL, NULL, NULL};
  NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  uint32_t *codes, *indices;
  size_t nc, ni;
  int64_t N;
  if (!get_u32a(env, argv[0], "codes must be a Uint32Array", &codes, &nc) ||
      !get_u32a(env, argv[1], "indices must be a Uint32Array", &indices, &ni) ||
      !get_index(env, argv[4], "N must be a particle count", 0, 4294967295.0, &N))
    return NULL;
  if ((uint64_t)N > nc || (uint64_t)N > ni) return throw_range(env, "codes or indices is shorter than N");
  GS_OK_OR_THROW(env, NULL, gs_radix_sort_indices(codes, (uint32_t)N, indices));
  return argv[1];
}

/* The MortonTree fields main.js and the worker read: _buf, f32, i32, numNodes,
 * levelRanges, maxNodes, byteLength (mortonTree.js:86-93, :184). */
static napi_value tree_object(napi_env env, const gs_node* nodes, uint32_t num, const uint32_t* lr, uint32_t nl,
                              uint32_t max_nodes) {
  napi_value o, ab, f32, i32, levels, x;
  void* data = NULL;
  if (napi_create_object(env, &o) != napi_ok ||
      napi_create_arraybuffer(env, (size_t)max_nodes * sizeof(gs_node), &data, &ab) != napi_ok)
    return NULL;
  memset(data, 0, (size_t)max_nodes * sizeof(gs_node));
  memcpy(data, nodes, (size_t)num * sizeof(gs_node));
  napi_create_typedarray(env, napi_float32_array, (size_t)max_nodes * 16, ab, 0, &f32);
  napi_create_typedarray(env, napi_int32_array, (size_t)max_nodes * 16, ab, 0, &i32);
  napi_create_array_with_length(env, nl, &levels);
  for (uint32_t l = 0; l < nl; l++) {
    napi_value pair, a, b;
    napi_create_array_with_length(env, 2, &pair);
    napi_create_uint32(env, lr[2 * l], &a);
    napi_create_uint32(env, lr[2 * l + 1], &b);
    napi_set_element(env, pair, 0, a);
    napi_set_element(env, pair, 1, b);
    napi_set_element(env, levels, l, pair);
  }
  napi_set_named_property(env, o, "_buf", ab);
  napi_set_named_property(env, o, "f32", f32);
  napi_set_named_property(env, o, "i32", i32);
  napi_set_named_property(env, o, "levelRanges", levels);
  napi_create_uint32(env, num, &x);
  napi_set_named_property(env, o, "numNodes", x);
  napi_create_uint32(env, max_nodes, &x);
  napi_set_named_property(env, o, "maxNodes", x);
  napi_create_double(env, (double)num * 64.0, &x);
  napi_set_named_property(env, o, "byteLength", x);
  return o;
}

/* buildTree(sortedCodes: Uint32Array, pos: Float32Array (stride 3), masses: Float32Array,
 * N, rootSize, maxParticles = N) -> tree object (MortonTree(maxParticles).build(...)) */
static napi_value BuildTree(napi_env env, napi_callback_info info) {
  size_t argc = 6;
  napi_value argv[6] = {NULL, NULL, NULL, NULL, NULL, NULL};
  NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  uint32_t* codes;
  float *pos, *masses;
  size_t nc, np, nm;
  int64_t N, maxp;
  double root;
  if (!get_u32a(env, argv[0], "sortedCodes must be a Uint32Array", &codes, &nc) ||
      !get_f32(env, argv[1], "pos must be a Float32Array", &pos, &np) ||
      !get_f32(env, argv[2], "masses must be a Float32Array", &masses, &nm) ||
      !get_index(env, argv[3], "N must be a particle count", 0, 4294967295.0, &N) ||
      !get_num(env, argv[4], "rootSize must be a number", &root))
    return NULL;
  maxp = N;
  if (argc > 5 && !is_nullish(env, argv[5]) &&
      !get_index(env, argv[5], "maxParticles must be a count", 0, 4294967295.0, &maxp))
    return NULL;
  if ((uint64_t)N > nc || 3 * (uint64_t)N > np || (uint64_t)N > nm)
    return throw_range(env, "an input is shorter than N particles");
  const uint64_t max_nodes = 2 * (uint64_t)maxp + 4096;   /* mortonTree.js:88 */
  if (max_nodes > 0xffffffffu) return throw_range(env, "maxParticles too large");
  gs_node* nodes = (gs_node*)malloc((size_t)max_nodes * sizeof(gs_node));
  if (!nodes) return throw_range(env, "out of host memory");
  uint32_t num = 0, lr[64], nl = 0;
  const int rc = gs_tree_build(codes, pos, masses, (uint32_t)N, root, (uint32_t)max_nodes, nodes, &num, lr, 32, &nl);
  napi_value o = rc == GS_OK ? tree_object(env, nodes, num, lr, nl, (uint32_t)max_nodes) : NULL;
  free(nodes);
  if (rc != GS_OK) return throw_gs(env, NULL, rc);
  return o;
}

static napi_value f32_array(napi_env env, const float* src, size_t n) {
  napi_value ab, ta;
  void* data;
  if (napi_create_arraybuffer(env, n * 4, &data, &ab) != napi_ok ||
      napi_create_typedarray(env, napi_float32_array, n, ab, 0, &ta) != napi_ok)
    return NULL;
  if (n) memcpy(data, src, n * 4);
  return ta;
}

/* sortAndBuild(particleData, stellarData, N, trackIdx2 = -1) -> {sorted, sortedStellar,
 * tree, perm, centralIdx, centralIdx2, masses} (mortonTree.js:192-224) */
static napi_value SortAndBuild(napi_env env, napi_callback_info info) {
  size_t argc = 4;
  napi_value argv[4] = {NULL, NULL, NULL, NULL};
  NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  float *p, *st;
  size_t n8, n4;
  int64_t N, track2 = -1;
  if (!get_f32(env, argv[0], "particleData must be a Float32Array", &p, &n8) ||
      !get_f32(env, argv[1], "stellarData must be a Float32Array", &st, &n4) ||
      !get_index(env, argv[2], "N must be a particle count", 0, 4294967295.0, &N))
    return NULL;
  if (argc > 3 && !is_nullish(env, argv[3]) &&
      !get_index(env, argv[3], "trackIdx2 must be an index or -1", -1, 9007199254740991.0, &track2))
    return NULL;
  if (8 * (uint64_t)N > n8 || 4 * (uint64_t)N > n4) return throw_range(env, "an input is shorter than N particles");
  const uint32_t n = (uint32_t)N;
  const uint64_t max_nodes = 2 * (uint64_t)n + 4096;
  float* sorted = (float*)malloc((size_t)n * 32 + 32);
  float* sorted4 = (float*)malloc((size_t)n * 16 + 16);
  float* mass = (float*)malloc((size_t)n * 4 + 4);
  uint32_t* perm = (uint32_t*)malloc((size_t)n * 4 + 4);
  gs_node* nodes = (gs_node*)malloc((size_t)max_nodes * sizeof(gs_node));
  napi_value out = NULL;
  if (!sorted || !sorted4 || !mass || !perm || !nodes) {
    throw_range(env, "out of host memory");
  } else {
    uint32_t num = 0, lr[64], nl = 0;
    int64_t c1 = 0, c2 = -1;
    const int rc = gs_sort_and_build(p, st, n, track2, sorted, sorted4, perm, nodes, (uint32_t)max_nodes, &num, lr,
                                     32, &nl, &c1, &c2, mass);
    if (rc != GS_OK) {
      throw_gs(env, NULL, rc);
    } else if (napi_create_object(env, &out) == napi_ok) {
      napi_value ab, pv, x;
      void* data;
      napi_set_named_property(env, out, "sorted", f32_array(env, sorted, (size_t)n * 8));
      napi_set_named_property(env, out, "sortedStellar", f32_array(env, sorted4, (size_t)n * 4));
      napi_set_named_property(env, out, "masses", f32_array(env, mass, n));
      napi_set_named_property(env, out, "tree", tree_object(env, nodes, num, lr, nl, (uint32_t)max_nodes));
      napi_create_arraybuffer(env, (size_t)n * 4, &data, &ab);
      if (n) memcpy(data, perm, (size_t)n * 4);
      napi_create_typedarray(env, napi_uint32_array, n, ab, 0, &pv);
      napi_set_named_property(env, out, "perm", pv);
      napi_create_int64(env, c1, &x);
      napi_set_named_property(env, out, "centralIdx", x);
      napi_create_int64(env, c2, &x);
      napi_set_named_property(env, out, "centralIdx2", x);
    }
  }
  free(sorted);
  free(sorted4);
  free(mass);
  free(perm);
  free(nodes);
  return out;
}

/* ---- module --------------------------------------------------------------------------- */

#define METHOD(name, fn) {name, NULL, fn, NULL, NULL, NULL, napi_default, NULL}
#define GETTER(name, fn) {name, NULL, NULL, fn, NULL, NULL, napi_default, NULL}

NAPI_MODULE_INIT() {
  const napi_property_descriptor methods[] = {
      METHOD("applyPermutation", ApplyPermutation),
      METHOD("updateCentralMass", UpdateCentralMass),
      METHOD("updateParams", UpdateParams),
      METHOD("encodeStarFormation", EncodeStarFormation),
      METHOD("uploadBHTree", UploadBHTree),
      METHOD("encodeRefresh", EncodeRefresh),
      METHOD("step", Step),
      METHOD("encodePositionReadback", EncodePositionReadback),
      METHOD("readPositions", ReadPositions),
      METHOD("destroy", Destroy),
      METHOD("sortBuild", SortBuild),
      METHOD("run", Run),
      METHOD("sync", Sync),
      METHOD("energy", Energy),
      METHOD("setTracking", SetTracking),
      METHOD("getTracking", GetTracking),
      METHOD("deviceErrors", DeviceErrors),
      GETTER("positionBuffer", GetPositionBuffer),
      GETTER("stellarBuffer", GetStellarBuffer),
  };
  napi_value cls;
  if (napi_define_class(env, "NBodyCUDA", NAPI_AUTO_LENGTH, Construct, NULL, sizeof(methods) / sizeof(methods[0]),
                        methods, &cls) != napi_ok)
    return NULL;
  const napi_property_descriptor fns[] = {
      {"NBodyCUDA", NULL, NULL, NULL, NULL, cls, napi_enumerable, NULL},
      METHOD("computeMortonCodes", ComputeMortonCodes),
      METHOD("radixSortIndices", RadixSortIndices),
      METHOD("buildTree", BuildTree),
      METHOD("sortAndBuild", SortAndBuild),
  };
  if (napi_define_properties(env, exports, sizeof(fns) / sizeof(fns[0]), fns) != napi_ok) return NULL;
  return exports;
}

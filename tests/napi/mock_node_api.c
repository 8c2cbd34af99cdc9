/*
 * TEST INFRASTRUCTURE ONLY: a small in-process implementation of the Node-API
 * functions declared in tests/napi/node_api.h, so tests can load
 * addon/galaxy_napi.c without Node.js and call it the way JavaScript would.
 *
 * Values are heap records (numbers, strings, booleans, undefined, null,
 * objects with properties and a prototype, arrays, functions and classes,
 * typed arrays over ArrayBuffers, BigInts, promises, errors); nothing is ever
 * freed (a test process is short). A pending exception is kept on the env, as
 * Node does. The mock_* functions at the end build values, construct objects,
 * call methods and read results for the test driver (ctypes).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "node_api.h"

enum Kind { K_UNDEF, K_NULL, K_BOOL, K_NUM, K_STR, K_OBJ, K_ARR, K_FUNC, K_TA, K_AB, K_BIGINT, K_PROMISE };

typedef struct Val Val;
struct Val {
  int kind;
  double num;
  int b;
  char* str;
  uint64_t big;
  /* properties (objects, functions, arrays, errors): key -> value, or key -> getter */
  int nprops, cprops;
  char** keys;
  Val** vals;
  napi_callback* getters;
  void** getter_data;
  Val* proto;
  /* array elements */
  uint32_t nel, cel;
  Val** el;
  /* function / class */
  napi_callback cb;
  void* cb_data;
  Val* prototype; /* a class's prototype object */
  /* typed array / array buffer */
  int ta_type;
  size_t ta_len, ta_off;
  Val* ab;
  void* ab_data;
  size_t ab_len;
  /* wrapped native object */
  void* wrapped;
  /* promise: 0 pending, 1 resolved, 2 rejected */
  int pstate;
  Val* presult;
};

struct napi_env__ {
  Val* exception;
};

struct napi_callback_info__ {
  Val* thisv;
  size_t argc;
  Val** argv;
  void* data;
};

struct napi_deferred__ {
  Val* promise;
};

static Val* V(napi_value v) { return (Val*)v; }
static napi_value NV(Val* v) { return (napi_value)v; }

static Val* mk(int kind) {
  Val* v = (Val*)calloc(1, sizeof(Val));
  v->kind = kind;
  return v;
}

static char* dupn(const char* s, size_t n) {
  if (n == NAPI_AUTO_LENGTH) n = strlen(s);
  char* d = (char*)malloc(n + 1);
  memcpy(d, s, n);
  d[n] = 0;
  return d;
}

static int find_prop(const Val* o, const char* k) {
  for (int i = 0; i < o->nprops; i++)
    if (!strcmp(o->keys[i], k)) return i;
  return -1;
}

static void put_prop(Val* o, const char* k, Val* v, napi_callback getter, void* gdata) {
  int i = find_prop(o, k);
  if (i < 0) {
    if (o->nprops == o->cprops) {
      o->cprops = o->cprops ? 2 * o->cprops : 8;
      o->keys = (char**)realloc(o->keys, sizeof(char*) * o->cprops);
      o->vals = (Val**)realloc(o->vals, sizeof(Val*) * o->cprops);
      o->getters = (napi_callback*)realloc(o->getters, sizeof(napi_callback) * o->cprops);
      o->getter_data = (void**)realloc(o->getter_data, sizeof(void*) * o->cprops);
    }
    i = o->nprops++;
    o->keys[i] = dupn(k, NAPI_AUTO_LENGTH);
  }
  o->vals[i] = v;
  o->getters[i] = getter;
  o->getter_data[i] = gdata;
}

static napi_status ok(void) { return napi_ok; }

static Val* the_undefined(void) {
  static Val* u = NULL;
  if (!u) u = mk(K_UNDEF);
  return u;
}

/* a call of a native callback: info carries this, the arguments and the data pointer */
static Val* call_cb(napi_env env, napi_callback cb, void* data, Val* thisv, size_t argc, Val** argv) {
  struct napi_callback_info__ info = {thisv, argc, argv, data};
  napi_value r = cb(env, &info);
  return r ? V(r) : the_undefined();
}

static Val* get_chain(napi_env env, Val* o, const char* k) {
  for (Val* p = o; p; p = p->proto) {
    const int i = find_prop(p, k);
    if (i >= 0) {
      if (p->getters[i]) return call_cb(env, p->getters[i], p->getter_data[i], o, 0, NULL);
      return p->vals[i];
    }
  }
  return NULL;
}

/* ---- Node-API ---------------------------------------------------------------------- */

napi_status napi_get_cb_info(napi_env env, napi_callback_info cbinfo, size_t* argc, napi_value* argv,
                             napi_value* this_arg, void** data) {
  (void)env;
  if (argc) {
    for (size_t i = 0; i < *argc; i++)
      if (argv) argv[i] = NV(i < cbinfo->argc ? cbinfo->argv[i] : the_undefined());
    *argc = cbinfo->argc;
  }
  if (this_arg) *this_arg = NV(cbinfo->thisv);
  if (data) *data = cbinfo->data;
  return ok();
}

static void define_on(Val* target, size_t n, const napi_property_descriptor* d) {
  for (size_t i = 0; i < n; i++) {
    if (d[i].method) {
      Val* f = mk(K_FUNC);
      f->cb = d[i].method;
      f->cb_data = d[i].data;
      put_prop(target, d[i].utf8name, f, NULL, NULL);
    } else if (d[i].getter) {
      put_prop(target, d[i].utf8name, NULL, d[i].getter, d[i].data);
    } else {
      put_prop(target, d[i].utf8name, V(d[i].value), NULL, NULL);
    }
  }
}

napi_status napi_define_class(napi_env env, const char* utf8name, size_t length, napi_callback constructor,
                              void* data, size_t property_count, const napi_property_descriptor* properties,
                              napi_value* result) {
  (void)env;
  Val* cls = mk(K_FUNC);
  cls->cb = constructor;
  cls->cb_data = data;
  cls->str = dupn(utf8name, length);
  cls->prototype = mk(K_OBJ);
  for (size_t i = 0; i < property_count; i++) {
    Val* target = (properties[i].attributes & napi_static) ? cls : cls->prototype;
    define_on(target, 1, &properties[i]);
  }
  *result = NV(cls);
  return ok();
}

napi_status napi_define_properties(napi_env env, napi_value object, size_t property_count,
                                   const napi_property_descriptor* properties) {
  (void)env;
  define_on(V(object), property_count, properties);
  return ok();
}

napi_status napi_wrap(napi_env env, napi_value js_object, void* native_object, napi_finalize finalize_cb,
                      void* finalize_hint, napi_ref* result) {
  (void)env;
  (void)finalize_cb;
  (void)finalize_hint;
  if (V(js_object)->wrapped) return napi_invalid_arg;
  V(js_object)->wrapped = native_object;
  if (result) *result = NULL;
  return ok();
}

napi_status napi_unwrap(napi_env env, napi_value js_object, void** result) {
  (void)env;
  if (!V(js_object)->wrapped) return napi_invalid_arg;
  *result = V(js_object)->wrapped;
  return ok();
}

napi_status napi_typeof(napi_env env, napi_value value, napi_valuetype* result) {
  (void)env;
  switch (V(value)->kind) {
    case K_UNDEF: *result = napi_undefined; break;
    case K_NULL: *result = napi_null; break;
    case K_BOOL: *result = napi_boolean; break;
    case K_NUM: *result = napi_number; break;
    case K_STR: *result = napi_string; break;
    case K_FUNC: *result = napi_function; break;
    case K_BIGINT: *result = napi_bigint; break;
    default: *result = napi_object;
  }
  return ok();
}

napi_status napi_is_typedarray(napi_env env, napi_value value, bool* result) {
  (void)env;
  *result = V(value)->kind == K_TA;
  return ok();
}

static size_t elem_size(int t) {
  switch (t) {
    case napi_int8_array: case napi_uint8_array: case napi_uint8_clamped_array: return 1;
    case napi_int16_array: case napi_uint16_array: return 2;
    case napi_float64_array: case napi_bigint64_array: case napi_biguint64_array: return 8;
    default: return 4;
  }
}

napi_status napi_get_typedarray_info(napi_env env, napi_value typedarray, napi_typedarray_type* type,
                                     size_t* length, void** data, napi_value* arraybuffer, size_t* byte_offset) {
  (void)env;
  Val* t = V(typedarray);
  if (t->kind != K_TA) return napi_invalid_arg;
  if (type) *type = (napi_typedarray_type)t->ta_type;
  if (length) *length = t->ta_len;
  if (data) *data = (char*)t->ab->ab_data + t->ta_off;
  if (arraybuffer) *arraybuffer = NV(t->ab);
  if (byte_offset) *byte_offset = t->ta_off;
  return ok();
}

napi_status napi_is_arraybuffer(napi_env env, napi_value value, bool* result) {
  (void)env;
  *result = V(value)->kind == K_AB;
  return ok();
}

napi_status napi_get_arraybuffer_info(napi_env env, napi_value arraybuffer, void** data, size_t* byte_length) {
  (void)env;
  if (V(arraybuffer)->kind != K_AB) return napi_arraybuffer_expected;
  if (data) *data = V(arraybuffer)->ab_data;
  if (byte_length) *byte_length = V(arraybuffer)->ab_len;
  return ok();
}

napi_status napi_create_arraybuffer(napi_env env, size_t byte_length, void** data, napi_value* result) {
  (void)env;
  Val* ab = mk(K_AB);
  ab->ab_data = calloc(1, byte_length ? byte_length : 1);
  ab->ab_len = byte_length;
  if (data) *data = ab->ab_data;
  *result = NV(ab);
  return ok();
}

napi_status napi_create_typedarray(napi_env env, napi_typedarray_type type, size_t length, napi_value arraybuffer,
                                   size_t byte_offset, napi_value* result) {
  (void)env;
  Val* ab = V(arraybuffer);
  if (ab->kind != K_AB || byte_offset + length * elem_size(type) > ab->ab_len) return napi_invalid_arg;
  Val* t = mk(K_TA);
  t->ta_type = type;
  t->ta_len = length;
  t->ta_off = byte_offset;
  t->ab = ab;
  *result = NV(t);
  return ok();
}

napi_status napi_get_value_double(napi_env env, napi_value value, double* result) {
  (void)env;
  if (V(value)->kind != K_NUM) return napi_number_expected;
  *result = V(value)->num;
  return ok();
}

napi_status napi_get_value_uint32(napi_env env, napi_value value, uint32_t* result) {
  (void)env;
  if (V(value)->kind != K_NUM) return napi_number_expected;
  *result = (uint32_t)(int64_t)V(value)->num;
  return ok();
}

napi_status napi_get_value_int64(napi_env env, napi_value value, int64_t* result) {
  (void)env;
  if (V(value)->kind != K_NUM) return napi_number_expected;
  *result = (int64_t)V(value)->num;
  return ok();
}

napi_status napi_get_value_bool(napi_env env, napi_value value, bool* result) {
  (void)env;
  if (V(value)->kind != K_BOOL) return napi_boolean_expected;
  *result = V(value)->b != 0;
  return ok();
}

static napi_value number(double d) {
  Val* v = mk(K_NUM);
  v->num = d;
  return NV(v);
}

napi_status napi_create_double(napi_env env, double value, napi_value* result) {
  (void)env;
  *result = number(value);
  return ok();
}

napi_status napi_create_uint32(napi_env env, uint32_t value, napi_value* result) {
  (void)env;
  *result = number(value);
  return ok();
}

napi_status napi_create_int64(napi_env env, int64_t value, napi_value* result) {
  (void)env;
  *result = number((double)value);
  return ok();
}

napi_status napi_create_bigint_uint64(napi_env env, uint64_t value, napi_value* result) {
  (void)env;
  Val* v = mk(K_BIGINT);
  v->big = value;
  *result = NV(v);
  return ok();
}

napi_status napi_create_string_utf8(napi_env env, const char* str, size_t length, napi_value* result) {
  (void)env;
  Val* v = mk(K_STR);
  v->str = dupn(str ? str : "", str ? length : 0);
  *result = NV(v);
  return ok();
}

napi_status napi_get_boolean(napi_env env, bool value, napi_value* result) {
  (void)env;
  Val* v = mk(K_BOOL);
  v->b = value;
  *result = NV(v);
  return ok();
}

napi_status napi_get_undefined(napi_env env, napi_value* result) {
  (void)env;
  *result = NV(the_undefined());
  return ok();
}

napi_status napi_get_null(napi_env env, napi_value* result) {
  (void)env;
  *result = NV(mk(K_NULL));
  return ok();
}

napi_status napi_create_object(napi_env env, napi_value* result) {
  (void)env;
  *result = NV(mk(K_OBJ));
  return ok();
}

static void arr_set(Val* a, uint32_t i, Val* v) {
  if (i >= a->cel) {
    uint32_t c = a->cel ? a->cel : 4;
    while (c <= i) c *= 2;
    a->el = (Val**)realloc(a->el, sizeof(Val*) * c);
    for (uint32_t k = a->cel; k < c; k++) a->el[k] = the_undefined();
    a->cel = c;
  }
  a->el[i] = v;
  if (i >= a->nel) a->nel = i + 1;
}

napi_status napi_create_array_with_length(napi_env env, size_t length, napi_value* result) {
  (void)env;
  Val* a = mk(K_ARR);
  for (size_t i = 0; i < length; i++) arr_set(a, (uint32_t)i, the_undefined());
  *result = NV(a);
  return ok();
}

napi_status napi_is_array(napi_env env, napi_value value, bool* result) {
  (void)env;
  *result = V(value)->kind == K_ARR;
  return ok();
}

napi_status napi_get_array_length(napi_env env, napi_value value, uint32_t* result) {
  (void)env;
  if (V(value)->kind != K_ARR) return napi_array_expected;
  *result = V(value)->nel;
  return ok();
}

napi_status napi_get_element(napi_env env, napi_value object, uint32_t index, napi_value* result) {
  (void)env;
  Val* o = V(object);
  if (o->kind == K_ARR) {
    *result = NV(index < o->nel ? o->el[index] : the_undefined());
    return ok();
  }
  if (o->kind == K_TA) {
    if (index >= o->ta_len || (o->ta_type != napi_float32_array && o->ta_type != napi_uint32_array &&
                               o->ta_type != napi_int32_array && o->ta_type != napi_float64_array)) {
      *result = NV(the_undefined());
      return ok();
    }
    const char* base = (const char*)o->ab->ab_data + o->ta_off;
    double d = o->ta_type == napi_float32_array ? ((const float*)base)[index]
             : o->ta_type == napi_uint32_array ? ((const uint32_t*)base)[index]
             : o->ta_type == napi_int32_array ? ((const int32_t*)base)[index] : ((const double*)base)[index];
    *result = number(d);
    return ok();
  }
  return napi_object_expected;
}

napi_status napi_set_element(napi_env env, napi_value object, uint32_t index, napi_value value) {
  (void)env;
  if (V(object)->kind != K_ARR) return napi_array_expected;
  arr_set(V(object), index, V(value));
  return ok();
}

napi_status napi_has_named_property(napi_env env, napi_value object, const char* utf8name, bool* result) {
  (void)env;
  *result = false;
  for (Val* p = V(object); p; p = p->proto)
    if (find_prop(p, utf8name) >= 0) *result = true;
  return ok();
}

napi_status napi_get_named_property(napi_env env, napi_value object, const char* utf8name, napi_value* result) {
  Val* v = get_chain(env, V(object), utf8name);
  *result = NV(v ? v : the_undefined());
  return ok();
}

napi_status napi_set_named_property(napi_env env, napi_value object, const char* utf8name, napi_value value) {
  (void)env;
  put_prop(V(object), utf8name, V(value), NULL, NULL);
  return ok();
}

static napi_status throw_named(napi_env env, const char* name, const char* code, const char* msg) {
  Val* e = mk(K_OBJ);
  napi_value s;
  napi_create_string_utf8(env, name, NAPI_AUTO_LENGTH, &s);
  put_prop(e, "name", V(s), NULL, NULL);
  napi_create_string_utf8(env, msg ? msg : "", NAPI_AUTO_LENGTH, &s);
  put_prop(e, "message", V(s), NULL, NULL);
  if (code) {
    napi_create_string_utf8(env, code, NAPI_AUTO_LENGTH, &s);
    put_prop(e, "code", V(s), NULL, NULL);
  }
  if (!env->exception) env->exception = e;
  return ok();
}

napi_status napi_throw_error(napi_env env, const char* code, const char* msg) {
  return throw_named(env, "Error", code, msg);
}

napi_status napi_throw_type_error(napi_env env, const char* code, const char* msg) {
  return throw_named(env, "TypeError", code, msg);
}

napi_status napi_throw_range_error(napi_env env, const char* code, const char* msg) {
  return throw_named(env, "RangeError", code, msg);
}

napi_status napi_is_exception_pending(napi_env env, bool* result) {
  *result = env->exception != NULL;
  return ok();
}

napi_status napi_create_error(napi_env env, napi_value code, napi_value msg, napi_value* result) {
  (void)env;
  Val* e = mk(K_OBJ);
  Val* name = mk(K_STR);
  name->str = dupn("Error", NAPI_AUTO_LENGTH);
  put_prop(e, "name", name, NULL, NULL);
  put_prop(e, "message", V(msg), NULL, NULL);
  if (code) put_prop(e, "code", V(code), NULL, NULL);
  *result = NV(e);
  return ok();
}

napi_status napi_create_promise(napi_env env, napi_deferred* deferred, napi_value* promise) {
  (void)env;
  Val* p = mk(K_PROMISE);
  struct napi_deferred__* d = (struct napi_deferred__*)calloc(1, sizeof(*d));
  d->promise = p;
  *deferred = d;
  *promise = NV(p);
  return ok();
}

napi_status napi_resolve_deferred(napi_env env, napi_deferred deferred, napi_value resolution) {
  (void)env;
  deferred->promise->pstate = 1;
  deferred->promise->presult = V(resolution);
  return ok();
}

napi_status napi_reject_deferred(napi_env env, napi_deferred deferred, napi_value rejection) {
  (void)env;
  deferred->promise->pstate = 2;
  deferred->promise->presult = V(rejection);
  return ok();
}

/* ---- the test driver's side ---------------------------------------------------------- */

napi_value napi_register_module_v1(napi_env env, napi_value exports);

napi_env mock_env(void) { return (napi_env)calloc(1, sizeof(struct napi_env__)); }

napi_value mock_load(napi_env env) {
  napi_value exports = NV(mk(K_OBJ));
  napi_value r = napi_register_module_v1(env, exports);
  return r ? r : exports;
}

napi_value mock_number(double d) { return number(d); }
napi_value mock_bool(int b) {
  Val* v = mk(K_BOOL);
  v->b = b;
  return NV(v);
}
napi_value mock_undefined(void) { return NV(the_undefined()); }
napi_value mock_null(void) { return NV(mk(K_NULL)); }
napi_value mock_string(const char* s) {
  Val* v = mk(K_STR);
  v->str = dupn(s, NAPI_AUTO_LENGTH);
  return NV(v);
}
napi_value mock_object(void) { return NV(mk(K_OBJ)); }
napi_value mock_array(void) { return NV(mk(K_ARR)); }
void mock_array_push(napi_value a, napi_value v) { arr_set(V(a), V(a)->nel, V(v)); }
void mock_set(napi_value o, const char* k, napi_value v) { put_prop(V(o), k, V(v), NULL, NULL); }

/* An ArrayBuffer over caller-owned memory, and a typed array viewing all of it. */
napi_value mock_arraybuffer(void* data, size_t bytes) {
  Val* ab = mk(K_AB);
  ab->ab_data = data;
  ab->ab_len = bytes;
  return NV(ab);
}
napi_value mock_typedarray(int type, void* data, size_t length) {
  Val* t = mk(K_TA);
  t->ta_type = type;
  t->ta_len = length;
  t->ab = V(mock_arraybuffer(data, length * elem_size(type)));
  return NV(t);
}

napi_value mock_get(napi_env env, napi_value o, const char* k) {
  Val* v = get_chain(env, V(o), k);
  return NV(v ? v : the_undefined());
}

napi_value mock_new(napi_env env, napi_value cls, size_t argc, napi_value* argv) {
  Val* obj = mk(K_OBJ);
  obj->proto = V(cls)->prototype;
  Val* r = call_cb(env, V(cls)->cb, V(cls)->cb_data, obj, argc, (Val**)argv);
  (void)r;
  return NV(obj);
}

napi_value mock_call(napi_env env, napi_value fn, napi_value thisv, size_t argc, napi_value* argv) {
  return NV(call_cb(env, V(fn)->cb, V(fn)->cb_data, thisv ? V(thisv) : the_undefined(), argc, (Val**)argv));
}

napi_value mock_call_method(napi_env env, napi_value obj, const char* name, size_t argc, napi_value* argv) {
  Val* f = get_chain(env, V(obj), name);
  if (!f || f->kind != K_FUNC) {
    throw_named(env, "TypeError", NULL, "not a function");
    return NV(the_undefined());
  }
  return NV(call_cb(env, f->cb, f->cb_data, V(obj), argc, (Val**)argv));
}

/* 1 and the error's name / code / message when an exception was pending (then cleared). */
int mock_take_exception(napi_env env, char* name, char* code, char* msg, size_t cap) {
  Val* e = env->exception;
  if (!e) return 0;
  env->exception = NULL;
  const char* parts[3] = {"name", "code", "message"};
  char* outs[3] = {name, code, msg};
  for (int i = 0; i < 3; i++) {
    Val* s = get_chain(env, e, parts[i]);
    snprintf(outs[i], cap, "%s", s && s->kind == K_STR ? s->str : "");
  }
  return 1;
}

int mock_kind(napi_value v) { return V(v)->kind; }
double mock_num(napi_value v) { return V(v)->num; }
int mock_bool_of(napi_value v) { return V(v)->b; }
const char* mock_str(napi_value v) { return V(v)->kind == K_STR ? V(v)->str : ""; }
uint64_t mock_bigint(napi_value v) { return V(v)->big; }
uint32_t mock_array_len(napi_value v) { return V(v)->nel; }
napi_value mock_array_get(napi_value v, uint32_t i) { return NV(i < V(v)->nel ? V(v)->el[i] : the_undefined()); }
int mock_ta_type(napi_value v) { return V(v)->ta_type; }
size_t mock_ta_len(napi_value v) { return V(v)->ta_len; }
void* mock_ta_data(napi_value v) { return (char*)V(v)->ab->ab_data + V(v)->ta_off; }
napi_value mock_ta_buffer(napi_value v) { return NV(V(v)->ab); }
void* mock_ab_data(napi_value v) { return V(v)->ab_data; }
size_t mock_ab_len(napi_value v) { return V(v)->ab_len; }
int mock_promise_state(napi_value v) { return V(v)->pstate; }
napi_value mock_promise_result(napi_value v) { return NV(V(v)->presult ? V(v)->presult : the_undefined()); }
int mock_has_own(napi_value o, const char* k) { return find_prop(V(o), k) >= 0; }
napi_value mock_prototype(napi_value cls) { return NV(V(cls)->prototype); }

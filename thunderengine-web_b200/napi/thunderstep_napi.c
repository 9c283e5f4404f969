/* N-API addon over libthunderstep.so: the JavaScript host's binding of the C-ABI in
 * include/thunderstep.h, one wrapper per call.  Built with node-gyp (binding.gyp beside
 * this file); Node.js is not part of this repository's build image, so the addon is
 * compiled on the JavaScript host.
 *
 * Shape: `new Player(device)` replaces `new Replayer(device, tape, kernels, sources)`
 * (web/replay.js:37-42); the methods keep Replayer's names and argument meaning
 * (plan/build, upload, writeWords, useStep, encodeSteps, encodeDiag, read, readHashes,
 * base, buffersEnd, memWords, hashCount - replay.js:46-396).  A non-zero status throws a
 * JS Error carrying te_last_error, as Replayer throws (replay.js:77, 100, 153, 157, 240,
 * 250).  The blocking calls - plan (Replayer.build), read, readHashes, adjointBackward,
 * ensemble runs with sync - run on the libuv pool and return Promises, as build() and
 * read() are async in replay.js:180, 368.
 *
 * Additions without a reference counterpart: setMode / fusedSegments / runSegment,
 * autotune, the discrete adjoint (adjointForward, adjointBackward, adjointWriteWords,
 * adjointRead, adjointZero, adjointMemory), Ensemble, and wSolveStaticScratch. */
#include <node_api.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "thunderstep.h"

#define NAPI_CALL(env, call)                                   \
  do {                                                         \
    if ((call) != napi_ok) {                                   \
      napi_throw_error((env), NULL, "N-API call failed: " #call); \
      return NULL;                                             \
    }                                                          \
  } while (0)

typedef struct {
  te_ctx *ctx;
} Player;

static napi_value throw_te(napi_env env, te_ctx *ctx, int rc) {
  char msg[512];
  snprintf(msg, sizeof msg, "thunderstep error %d: %s", rc, ctx ? te_last_error(ctx) : "no context");
  napi_throw_error(env, NULL, msg);
  return NULL;
}

static void player_finalize(napi_env env, void *data, void *hint) {
  (void)env;
  (void)hint;
  Player *p = (Player *)data;
  if (p->ctx) te_destroy(p->ctx);
  free(p);
}

/* argument helpers */
static Player *this_player(napi_env env, napi_callback_info info, size_t *argc, napi_value *argv) {
  napi_value self;
  Player *p = NULL;
  if (napi_get_cb_info(env, info, argc, argv, &self, NULL) != napi_ok) return NULL;
  if (napi_unwrap(env, self, (void **)&p) != napi_ok || !p || !p->ctx) {
    napi_throw_error(env, NULL, "not a Player");
    return NULL;
  }
  return p;
}

static char *get_string(napi_env env, napi_value v, size_t *len) {
  size_t n = 0;
  if (napi_get_value_string_utf8(env, v, NULL, 0, &n) != napi_ok) return NULL;
  char *s = (char *)malloc(n + 1);
  napi_get_value_string_utf8(env, v, s, n + 1, &n);
  if (len) *len = n;
  return s;
}

static int64_t get_i64(napi_env env, napi_value v) {
  int64_t x = 0;
  napi_get_value_int64(env, v, &x);
  return x;
}

static int get_bytes(napi_env env, napi_value v, void **data, size_t *len) {
  bool is_typed = false, is_buf = false;
  napi_is_typedarray(env, v, &is_typed);
  if (is_typed) {
    napi_typedarray_type t;
    size_t count, off;
    napi_value ab;
    void *base;
    napi_get_typedarray_info(env, v, &t, &count, &base, &ab, &off);
    size_t esz = (t == napi_int8_array || t == napi_uint8_array || t == napi_uint8_clamped_array) ? 1
                 : (t == napi_int16_array || t == napi_uint16_array) ? 2
                 : (t == napi_float64_array || t == napi_bigint64_array || t == napi_biguint64_array) ? 8 : 4;
    *data = base;
    *len = count * esz;
    return 1;
  }
  napi_is_buffer(env, v, &is_buf);
  if (is_buf) return napi_get_buffer_info(env, v, data, len) == napi_ok;
  return 0;
}

static napi_value make_u32_array(napi_env env, const uint32_t *src, size_t n) {
  void *data;
  napi_value ab, arr;
  napi_create_arraybuffer(env, n * 4, &data, &ab);
  if (n) memcpy(data, src, n * 4);
  napi_create_typedarray(env, napi_uint32_array, n, ab, 0, &arr);
  return arr;
}

/* ---------------------------------------------------------------- Player */

/* new Player(device = 0, flags = 0)  ~ new Replayer(device, tape, kernels, sources) */
static napi_value player_new(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2], self;
  NAPI_CALL(env, napi_get_cb_info(env, info, &argc, argv, &self, NULL));
  te_config cfg;
  memset(&cfg, 0, sizeof cfg);
  if (argc > 0) cfg.device = (int)get_i64(env, argv[0]);
  if (argc > 1) cfg.flags = (int)get_i64(env, argv[1]);
  Player *p = (Player *)calloc(1, sizeof *p);
  int rc = te_create(&cfg, &p->ctx);
  if (rc != TE_OK) {
    napi_value r = throw_te(env, p->ctx, rc);
    if (p->ctx) te_destroy(p->ctx);
    free(p);
    return r;
  }
  NAPI_CALL(env, napi_wrap(env, self, p, player_finalize, NULL, NULL));
  return self;
}

/* async work: a blocking C call on the libuv pool resolving a Promise */
typedef struct {
  napi_async_work work;
  napi_deferred deferred;
  Player *player;
  int kind, rc;
  char *a, *b;
  size_t alen, blen;
  int64_t i0, i1;
  uint32_t *out;
  size_t nout;
} Job;

enum { JOB_PLAN, JOB_READ, JOB_HASHES, JOB_ADJ_BACKWARD, JOB_SYNC };

static void job_execute(napi_env env, void *data) {
  (void)env;
  Job *j = (Job *)data;
  te_ctx *c = j->player->ctx;
  switch (j->kind) {
    case JOB_PLAN: j->rc = te_plan(c, j->a, j->alen, j->b, j->blen, (int)j->i0); break;
    case JOB_READ: j->rc = te_read(c, (uint64_t)j->i1, j->nout, j->out); break;
    case JOB_HASHES: j->rc = te_read_hashes(c, j->out, j->nout); break;
    case JOB_ADJ_BACKWARD: j->rc = te_adjoint_backward(c); if (j->rc == TE_OK) j->rc = te_sync(c); break;
    case JOB_SYNC: j->rc = te_sync(c); break;
  }
}

static void job_complete(napi_env env, napi_status status, void *data) {
  Job *j = (Job *)data;
  if (status != napi_ok || j->rc != TE_OK) {
    char msg[512];
    napi_value err, m;
    snprintf(msg, sizeof msg, "thunderstep error %d: %s", j->rc, te_last_error(j->player->ctx));
    napi_create_string_utf8(env, msg, NAPI_AUTO_LENGTH, &m);
    napi_create_error(env, NULL, m, &err);
    napi_reject_deferred(env, j->deferred, err);
  } else {
    napi_value v;
    if (j->kind == JOB_READ || j->kind == JOB_HASHES) v = make_u32_array(env, j->out, j->nout);
    else napi_get_undefined(env, &v);
    napi_resolve_deferred(env, j->deferred, v);
  }
  napi_delete_async_work(env, j->work);
  free(j->a);
  free(j->b);
  free(j->out);
  free(j);
}

static napi_value queue(napi_env env, Job *j, const char *name) {
  napi_value promise, res;
  NAPI_CALL(env, napi_create_promise(env, &j->deferred, &promise));
  NAPI_CALL(env, napi_create_string_utf8(env, name, NAPI_AUTO_LENGTH, &res));
  NAPI_CALL(env, napi_create_async_work(env, NULL, res, job_execute, job_complete, j, &j->work));
  NAPI_CALL(env, napi_queue_async_work(env, j->work));
  return promise;
}

/* plan(tapeJson, kernelsJson | null, withHashes) -> Promise  ~ plan(withHashes) + build() */
static napi_value player_plan(napi_env env, napi_callback_info info) {
  size_t argc = 3;
  napi_value argv[3];
  Player *p = this_player(env, info, &argc, argv);
  if (!p) return NULL;
  Job *j = (Job *)calloc(1, sizeof *j);
  j->player = p;
  j->kind = JOB_PLAN;
  j->a = get_string(env, argv[0], &j->alen);
  napi_valuetype t;
  napi_typeof(env, argv[1], &t);
  j->b = t == napi_string ? get_string(env, argv[1], &j->blen) : NULL;
  bool h = false;
  if (argc > 2) napi_get_value_bool(env, argv[2], &h);
  j->i0 = h;
  return queue(env, j, "thunderstep.plan");
}

/* info() -> {memWords, buffersEnd, scratchBase, hashCount, numBuffers, numOps, numDispatches} */
static napi_value player_info(napi_env env, napi_callback_info info) {
  size_t argc = 0;
  Player *p = this_player(env, info, &argc, NULL);
  if (!p) return NULL;
  te_info ti;
  int rc = te_get_info(p->ctx, &ti);
  if (rc != TE_OK) return throw_te(env, p->ctx, rc);
  napi_value o, v;
  napi_create_object(env, &o);
#define SETN(name, x)                         \
  napi_create_double(env, (double)(x), &v);   \
  napi_set_named_property(env, o, name, v);
  SETN("memWords", ti.mem_words)
  SETN("buffersEnd", ti.buffers_end)
  SETN("scratchBase", ti.scratch_base)
  SETN("hashCount", ti.hash_count)
  SETN("numBuffers", ti.num_buffers)
  SETN("numOps", ti.num_ops)
  SETN("numDispatches", ti.num_dispatches)
#undef SETN
  return o;
}

/* base(bufId) -> word offset  ~ Replayer.base[id] */
static napi_value player_base(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1], v;
  Player *p = this_player(env, info, &argc, argv);
  if (!p) return NULL;
  uint64_t off;
  int rc = te_buffer_base(p->ctx, (int)get_i64(env, argv[0]), &off);
  if (rc != TE_OK) return throw_te(env, p->ctx, rc);
  napi_create_double(env, (double)off, &v);
  return v;
}

/* upload(bufId, typedArray | Buffer)  ~ Replayer.upload(id, u8) */
static napi_value player_upload(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2];
  Player *p = this_player(env, info, &argc, argv);
  if (!p) return NULL;
  void *d;
  size_t n;
  if (!get_bytes(env, argv[1], &d, &n)) {
    napi_throw_type_error(env, NULL, "upload: expected a TypedArray or Buffer");
    return NULL;
  }
  int rc = te_upload(p->ctx, (int)get_i64(env, argv[0]), d, n);
  return rc == TE_OK ? NULL : throw_te(env, p->ctx, rc);
}

/* writeWords(offWords, typedArray)  ~ Replayer.writeWords(off, words) */
static napi_value player_write_words(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2];
  Player *p = this_player(env, info, &argc, argv);
  if (!p) return NULL;
  void *d;
  size_t n;
  if (!get_bytes(env, argv[1], &d, &n)) {
    napi_throw_type_error(env, NULL, "writeWords: expected a TypedArray or Buffer");
    return NULL;
  }
  int rc = te_write_words(p->ctx, (uint64_t)get_i64(env, argv[0]), d, n);
  return rc == TE_OK ? NULL : throw_te(env, p->ctx, rc);
}

/* useStep(cmdsJson)  ~ Replayer.useStep(cmds) */
static napi_value player_use_step(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  Player *p = this_player(env, info, &argc, argv);
  if (!p) return NULL;
  size_t n;
  char *s = get_string(env, argv[0], &n);
  int rc = te_use_step(p->ctx, s, n);
  free(s);
  return rc == TE_OK ? NULL : throw_te(env, p->ctx, rc);
}

/* encodeSteps(n, withHashes)  ~ Replayer.encodeSteps(enc, n, withHashes) */
static napi_value player_encode_steps(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2];
  Player *p = this_player(env, info, &argc, argv);
  if (!p) return NULL;
  bool h = false;
  if (argc > 1) napi_get_value_bool(env, argv[1], &h);
  int rc = te_run(p->ctx, (int)get_i64(env, argv[0]), h);
  return rc == TE_OK ? NULL : throw_te(env, p->ctx, rc);
}

/* runOps(firstOp, lastOp, withHashes)  ~ encodeSteps(..., lastOp) */
static napi_value player_run_ops(napi_env env, napi_callback_info info) {
  size_t argc = 3;
  napi_value argv[3];
  Player *p = this_player(env, info, &argc, argv);
  if (!p) return NULL;
  bool h = false;
  if (argc > 2) napi_get_value_bool(env, argv[2], &h);
  int rc = te_run_ops(p->ctx, (int)get_i64(env, argv[0]), (int)get_i64(env, argv[1]), h);
  return rc == TE_OK ? NULL : throw_te(env, p->ctx, rc);
}

/* encodeDiag()  ~ Replayer.encodeDiag(enc) */
static napi_value player_encode_diag(napi_env env, napi_callback_info info) {
  size_t argc = 0;
  Player *p = this_player(env, info, &argc, NULL);
  if (!p) return NULL;
  int rc = te_run_diag(p->ctx);
  return rc == TE_OK ? NULL : throw_te(env, p->ctx, rc);
}

/* read(words, offWords) -> Promise<Uint32Array>  ~ Replayer.read(words, offWords) */
static napi_value player_read(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2];
  Player *p = this_player(env, info, &argc, argv);
  if (!p) return NULL;
  Job *j = (Job *)calloc(1, sizeof *j);
  j->player = p;
  j->kind = JOB_READ;
  j->nout = (size_t)get_i64(env, argv[0]);
  j->i1 = argc > 1 ? get_i64(env, argv[1]) : 0;
  j->out = (uint32_t *)malloc(j->nout ? j->nout * 4 : 4);
  return queue(env, j, "thunderstep.read");
}

/* readHashes() -> Promise<Uint32Array>  ~ Replayer.readHashes() */
static napi_value player_read_hashes(napi_env env, napi_callback_info info) {
  size_t argc = 0;
  Player *p = this_player(env, info, &argc, NULL);
  if (!p) return NULL;
  te_info ti;
  int rc = te_get_info(p->ctx, &ti);
  if (rc != TE_OK) return throw_te(env, p->ctx, rc);
  Job *j = (Job *)calloc(1, sizeof *j);
  j->player = p;
  j->kind = JOB_HASHES;
  j->nout = ti.hash_count;
  j->out = (uint32_t *)malloc(j->nout ? j->nout * 4 : 4);
  return queue(env, j, "thunderstep.readHashes");
}

static napi_value player_clear_hashes(napi_env env, napi_callback_info info) {
  size_t argc = 0;
  Player *p = this_player(env, info, &argc, NULL);
  if (!p) return NULL;
  int rc = te_clear_hashes(p->ctx);
  return rc == TE_OK ? NULL : throw_te(env, p->ctx, rc);
}

/* setMode(0 exact | 1 fused) */
static napi_value player_set_mode(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  Player *p = this_player(env, info, &argc, argv);
  if (!p) return NULL;
  int rc = te_set_mode(p->ctx, (int)get_i64(env, argv[0]));
  return rc == TE_OK ? NULL : throw_te(env, p->ctx, rc);
}

/* fusedSegments() -> [[kind, firstOp, lastOp, kernels], ...] */
static napi_value player_fused_segments(napi_env env, napi_callback_info info) {
  size_t argc = 0;
  Player *p = this_player(env, info, &argc, NULL);
  if (!p) return NULL;
  int n = 0;
  int rc = te_fused_segments(p->ctx, NULL, 0, &n);
  if (rc != TE_OK) return throw_te(env, p->ctx, rc);
  te_segment *seg = (te_segment *)calloc(n > 0 ? n : 1, sizeof *seg);
  rc = te_fused_segments(p->ctx, seg, n, &n);
  if (rc != TE_OK) {
    free(seg);
    return throw_te(env, p->ctx, rc);
  }
  napi_value arr;
  napi_create_array_with_length(env, n, &arr);
  for (int i = 0; i < n; i++) {
    napi_value row, v;
    napi_create_array_with_length(env, 4, &row);
    int vals[4] = {seg[i].kind, seg[i].first_op, seg[i].last_op, seg[i].kernels};
    for (int q = 0; q < 4; q++) {
      napi_create_int32(env, vals[q], &v);
      napi_set_element(env, row, q, v);
    }
    napi_set_element(env, arr, i, row);
  }
  free(seg);
  return arr;
}

static napi_value player_run_segment(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2];
  Player *p = this_player(env, info, &argc, argv);
  if (!p) return NULL;
  int rc = te_run_segment(p->ctx, (int)get_i64(env, argv[0]), argc > 1 ? (int)get_i64(env, argv[1]) : -1);
  return rc == TE_OK ? NULL : throw_te(env, p->ctx, rc);
}

/* opName(i) -> string */
static napi_value player_op_name(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1], v;
  Player *p = this_player(env, info, &argc, argv);
  if (!p) return NULL;
  const char *s = te_op_name(p->ctx, (int)get_i64(env, argv[0]));
  if (!s) {
    napi_get_null(env, &v);
    return v;
  }
  napi_create_string_utf8(env, s, NAPI_AUTO_LENGTH, &v);
  return v;
}

/* sync() -> Promise */
static napi_value player_sync(napi_env env, napi_callback_info info) {
  size_t argc = 0;
  Player *p = this_player(env, info, &argc, NULL);
  if (!p) return NULL;
  Job *j = (Job *)calloc(1, sizeof *j);
  j->player = p;
  j->kind = JOB_SYNC;
  return queue(env, j, "thunderstep.sync");
}

/* autotune(reps) -> number of ops whose block shape changed */
static napi_value player_autotune(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1], v;
  Player *p = this_player(env, info, &argc, argv);
  if (!p) return NULL;
  int tuned = 0;
  int rc = te_autotune(p->ctx, argc > 0 ? (int)get_i64(env, argv[0]) : 5, &tuned);
  if (rc != TE_OK) return throw_te(env, p->ctx, rc);
  napi_create_int32(env, tuned, &v);
  return v;
}

/* ---- discrete adjoint: the forward/backward pair of a torch.autograd.Function-shaped
 * host class (forward(): adjointForward + read; backward(): adjointWriteWords +
 * adjointBackward + adjointRead) */
static napi_value player_adjoint_forward(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2];
  Player *p = this_player(env, info, &argc, argv);
  if (!p) return NULL;
  int rc = te_adjoint_forward(p->ctx, (int)get_i64(env, argv[0]), (int)get_i64(env, argv[1]));
  return rc == TE_OK ? NULL : throw_te(env, p->ctx, rc);
}

static napi_value player_adjoint_backward(napi_env env, napi_callback_info info) {
  size_t argc = 0;
  Player *p = this_player(env, info, &argc, NULL);
  if (!p) return NULL;
  Job *j = (Job *)calloc(1, sizeof *j);
  j->player = p;
  j->kind = JOB_ADJ_BACKWARD;
  return queue(env, j, "thunderstep.adjointBackward");
}

static napi_value player_adjoint_write_words(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2];
  Player *p = this_player(env, info, &argc, argv);
  if (!p) return NULL;
  void *d;
  size_t n;
  if (!get_bytes(env, argv[1], &d, &n)) {
    napi_throw_type_error(env, NULL, "adjointWriteWords: expected a Float32Array");
    return NULL;
  }
  int rc = te_adjoint_write_words(p->ctx, (uint64_t)get_i64(env, argv[0]), d, n);
  return rc == TE_OK ? NULL : throw_te(env, p->ctx, rc);
}

/* adjointRead(words, offWords) -> Float32Array (blocking: the adjoint memory is small
 * next to the work that produced it) */
static napi_value player_adjoint_read(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2], ab, arr;
  Player *p = this_player(env, info, &argc, argv);
  if (!p) return NULL;
  size_t n = (size_t)get_i64(env, argv[0]);
  void *data;
  NAPI_CALL(env, napi_create_arraybuffer(env, n * 4, &data, &ab));
  int rc = te_adjoint_read(p->ctx, (uint64_t)(argc > 1 ? get_i64(env, argv[1]) : 0), n, data);
  if (rc != TE_OK) return throw_te(env, p->ctx, rc);
  NAPI_CALL(env, napi_create_typedarray(env, napi_float32_array, n, ab, 0, &arr));
  return arr;
}

static napi_value player_adjoint_zero(napi_env env, napi_callback_info info) {
  size_t argc = 0;
  Player *p = this_player(env, info, &argc, NULL);
  if (!p) return NULL;
  int rc = te_adjoint_zero(p->ctx);
  return rc == TE_OK ? NULL : throw_te(env, p->ctx, rc);
}

static napi_value player_adjoint_memory(napi_env env, napi_callback_info info) {
  size_t argc = 0;
  napi_value v;
  Player *p = this_player(env, info, &argc, NULL);
  if (!p) return NULL;
  uint64_t b = 0;
  int rc = te_adjoint_memory(p->ctx, &b);
  if (rc != TE_OK) return throw_te(env, p->ctx, rc);
  napi_create_double(env, (double)b, &v);
  return v;
}

/* wSolveStaticScratch({pk1, pk2, qk, mm, fpk, wten, pp3d, w}: word offsets in this
 * player's memory, nx, ny, nz, dts, alph, beta): the allocation-free column solve on
 * the player's own fields (device pointers from te_device_ptr), on the default stream */
static napi_value player_w_solve_static(napi_env env, napi_callback_info info) {
  size_t argc = 7;
  napi_value argv[7];
  Player *p = this_player(env, info, &argc, argv);
  if (!p) return NULL;
  static const char *names[8] = {"pk1", "pk2", "qk", "mm", "fpk", "wten", "pp3d", "w"};
  void *ptr[8];
  for (int q = 0; q < 8; q++) {
    napi_value v;
    NAPI_CALL(env, napi_get_named_property(env, argv[0], names[q], &v));
    int rc = te_device_ptr(p->ctx, (uint64_t)get_i64(env, v), &ptr[q]);
    if (rc != TE_OK) return throw_te(env, p->ctx, rc);
  }
  te_wsolve_fields f;
  f.pk1 = (const float *)ptr[0];
  f.pk2 = (const float *)ptr[1];
  f.qk = (const float *)ptr[2];
  f.mm = (const float *)ptr[3];
  f.fpk = (const float *)ptr[4];
  f.wten = (const float *)ptr[5];
  f.pp3d = (const float *)ptr[6];
  f.w = (float *)ptr[7];
  double dts, alph, beta;
  napi_get_value_double(env, argv[4], &dts);
  napi_get_value_double(env, argv[5], &alph);
  napi_get_value_double(env, argv[6], &beta);
  char err[256] = {0};
  int rc = te_w_solve_static_scratch(&f, (int)get_i64(env, argv[1]), (int)get_i64(env, argv[2]),
                                     (int)get_i64(env, argv[3]), (float)dts, (float)alph, (float)beta, NULL, err,
                                     sizeof err);
  if (rc != TE_OK) {
    napi_throw_error(env, NULL, err);
    return NULL;
  }
  return NULL;
}

/* ---------------------------------------------------------------- Ensemble */

typedef struct {
  te_ensemble *ens;
  napi_ref members;  /* keeps the member Players alive */
} Ensemble;

static void ensemble_finalize(napi_env env, void *data, void *hint) {
  (void)hint;
  Ensemble *e = (Ensemble *)data;
  if (e->ens) te_ensemble_destroy(e->ens);
  if (e->members) napi_delete_reference(env, e->members);
  free(e);
}

/* new Ensemble([player, ...]) */
static napi_value ensemble_new(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1], self;
  NAPI_CALL(env, napi_get_cb_info(env, info, &argc, argv, &self, NULL));
  uint32_t n = 0;
  NAPI_CALL(env, napi_get_array_length(env, argv[0], &n));
  te_ctx **ctx = (te_ctx **)calloc(n ? n : 1, sizeof *ctx);
  for (uint32_t i = 0; i < n; i++) {
    napi_value v;
    Player *p = NULL;
    napi_get_element(env, argv[0], i, &v);
    if (napi_unwrap(env, v, (void **)&p) != napi_ok || !p) {
      free(ctx);
      napi_throw_type_error(env, NULL, "Ensemble: every member must be a Player");
      return NULL;
    }
    ctx[i] = p->ctx;
  }
  Ensemble *e = (Ensemble *)calloc(1, sizeof *e);
  int rc = te_ensemble_create(ctx, (int)n, &e->ens);
  free(ctx);
  if (rc != TE_OK) {
    char msg[512];
    snprintf(msg, sizeof msg, "thunderstep error %d: %s", rc, te_ensemble_last_error(e->ens));
    if (e->ens) te_ensemble_destroy(e->ens);
    free(e);
    napi_throw_error(env, NULL, msg);
    return NULL;
  }
  napi_create_reference(env, argv[0], 1, &e->members);
  NAPI_CALL(env, napi_wrap(env, self, e, ensemble_finalize, NULL, NULL));
  return self;
}

static Ensemble *this_ensemble(napi_env env, napi_callback_info info, size_t *argc, napi_value *argv) {
  napi_value self;
  Ensemble *e = NULL;
  if (napi_get_cb_info(env, info, argc, argv, &self, NULL) != napi_ok) return NULL;
  if (napi_unwrap(env, self, (void **)&e) != napi_ok || !e) {
    napi_throw_error(env, NULL, "not an Ensemble");
    return NULL;
  }
  return e;
}

/* run(nsteps): one graph launch per large step, every member advanced */
static napi_value ensemble_run(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  Ensemble *e = this_ensemble(env, info, &argc, argv);
  if (!e) return NULL;
  int rc = te_ensemble_run(e->ens, (int)get_i64(env, argv[0]));
  if (rc != TE_OK) napi_throw_error(env, NULL, te_ensemble_last_error(e->ens));
  return NULL;
}

/* sync(): blocks until the runs queued so far are done */
static napi_value ensemble_sync(napi_env env, napi_callback_info info) {
  size_t argc = 0;
  Ensemble *e = this_ensemble(env, info, &argc, NULL);
  if (!e) return NULL;
  int rc = te_ensemble_sync(e->ens);
  if (rc != TE_OK) napi_throw_error(env, NULL, te_ensemble_last_error(e->ens));
  return NULL;
}

/* ---------------------------------------------------------------- module */

/* kernelTable() -> JSON string of the built-in kernels.json table */
static napi_value kernel_table(napi_env env, napi_callback_info info) {
  (void)info;
  size_t n = te_kernel_table_json(NULL, 0);
  char *s = (char *)malloc(n + 1);
  te_kernel_table_json(s, n + 1);
  napi_value v;
  napi_create_string_utf8(env, s, n, &v);
  free(s);
  return v;
}

/* regionHash(Uint32Array) -> number  (replay.js:407-418) */
static napi_value region_hash(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1], v;
  NAPI_CALL(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  void *d;
  size_t n;
  if (!get_bytes(env, argv[0], &d, &n)) {
    napi_throw_type_error(env, NULL, "regionHash: expected a Uint32Array");
    return NULL;
  }
  napi_create_uint32(env, te_region_hash_host((const uint32_t *)d, n / 4), &v);
  return v;
}

/* checkPow(p, lo, hi) -> {mismatches, firstBad}: the library's self-check of its two
 * routes to x^p over the binary32 patterns [lo, hi) (te_check_pow) */
static napi_value check_pow(napi_env env, napi_callback_info info) {
  size_t argc = 3;
  napi_value argv[3], out, v;
  NAPI_CALL(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  double p = 0;
  uint32_t lo = 0, hi = 0;
  napi_get_value_double(env, argv[0], &p);
  napi_get_value_uint32(env, argv[1], &lo);
  napi_get_value_uint32(env, argv[2], &hi);
  uint64_t bad = 0;
  uint32_t first = 0;
  int rc = te_check_pow((float)p, lo, hi, &bad, &first);
  if (rc != TE_OK) {
    napi_throw_error(env, NULL, "te_check_pow failed");
    return NULL;
  }
  napi_create_object(env, &out);
  napi_create_double(env, (double)bad, &v);
  napi_set_named_property(env, out, "mismatches", v);
  napi_create_uint32(env, first, &v);
  napi_set_named_property(env, out, "firstBad", v);
  return out;
}

static napi_value init(napi_env env, napi_value exports) {
  napi_property_descriptor player_methods[] = {
      {"plan", NULL, player_plan, NULL, NULL, NULL, napi_default, NULL},
      {"info", NULL, player_info, NULL, NULL, NULL, napi_default, NULL},
      {"base", NULL, player_base, NULL, NULL, NULL, napi_default, NULL},
      {"upload", NULL, player_upload, NULL, NULL, NULL, napi_default, NULL},
      {"writeWords", NULL, player_write_words, NULL, NULL, NULL, napi_default, NULL},
      {"useStep", NULL, player_use_step, NULL, NULL, NULL, napi_default, NULL},
      {"encodeSteps", NULL, player_encode_steps, NULL, NULL, NULL, napi_default, NULL},
      {"runOps", NULL, player_run_ops, NULL, NULL, NULL, napi_default, NULL},
      {"encodeDiag", NULL, player_encode_diag, NULL, NULL, NULL, napi_default, NULL},
      {"read", NULL, player_read, NULL, NULL, NULL, napi_default, NULL},
      {"readHashes", NULL, player_read_hashes, NULL, NULL, NULL, napi_default, NULL},
      {"clearHashes", NULL, player_clear_hashes, NULL, NULL, NULL, napi_default, NULL},
      {"setMode", NULL, player_set_mode, NULL, NULL, NULL, napi_default, NULL},
      {"fusedSegments", NULL, player_fused_segments, NULL, NULL, NULL, napi_default, NULL},
      {"runSegment", NULL, player_run_segment, NULL, NULL, NULL, napi_default, NULL},
      {"opName", NULL, player_op_name, NULL, NULL, NULL, napi_default, NULL},
      {"sync", NULL, player_sync, NULL, NULL, NULL, napi_default, NULL},
      {"autotune", NULL, player_autotune, NULL, NULL, NULL, napi_default, NULL},
      {"adjointForward", NULL, player_adjoint_forward, NULL, NULL, NULL, napi_default, NULL},
      {"adjointBackward", NULL, player_adjoint_backward, NULL, NULL, NULL, napi_default, NULL},
      {"adjointWriteWords", NULL, player_adjoint_write_words, NULL, NULL, NULL, napi_default, NULL},
      {"adjointRead", NULL, player_adjoint_read, NULL, NULL, NULL, napi_default, NULL},
      {"adjointZero", NULL, player_adjoint_zero, NULL, NULL, NULL, napi_default, NULL},
      {"adjointMemory", NULL, player_adjoint_memory, NULL, NULL, NULL, napi_default, NULL},
      {"wSolveStaticScratch", NULL, player_w_solve_static, NULL, NULL, NULL, napi_default, NULL},
  };
  napi_value player_class, ensemble_class, v;
  NAPI_CALL(env, napi_define_class(env, "Player", NAPI_AUTO_LENGTH, player_new, NULL,
                                   sizeof player_methods / sizeof player_methods[0], player_methods, &player_class));
  napi_property_descriptor ens_methods[] = {
      {"run", NULL, ensemble_run, NULL, NULL, NULL, napi_default, NULL},
      {"sync", NULL, ensemble_sync, NULL, NULL, NULL, napi_default, NULL},
  };
  NAPI_CALL(env, napi_define_class(env, "Ensemble", NAPI_AUTO_LENGTH, ensemble_new, NULL, 2, ens_methods,
                                   &ensemble_class));
  NAPI_CALL(env, napi_set_named_property(env, exports, "Player", player_class));
  NAPI_CALL(env, napi_set_named_property(env, exports, "Ensemble", ensemble_class));
  NAPI_CALL(env, napi_create_function(env, "kernelTable", NAPI_AUTO_LENGTH, kernel_table, NULL, &v));
  NAPI_CALL(env, napi_set_named_property(env, exports, "kernelTable", v));
  NAPI_CALL(env, napi_create_function(env, "regionHash", NAPI_AUTO_LENGTH, region_hash, NULL, &v));
  NAPI_CALL(env, napi_set_named_property(env, exports, "regionHash", v));
  NAPI_CALL(env, napi_create_function(env, "checkPow", NAPI_AUTO_LENGTH, check_pow, NULL, &v));
  NAPI_CALL(env, napi_set_named_property(env, exports, "checkPow", v));
  return exports;
}

NAPI_MODULE(NODE_GYP_MODULE_NAME, init)

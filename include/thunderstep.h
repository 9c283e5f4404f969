/* thunderstep: B200 (sm_100a) tape player for ThunderEngine's CM1 large-step dynamics.
 *
 * Drop-in for the reference's WebGPU tape player `Replayer` (web/replay.js:36-396).
 * A caller that records tapes with the reference's step encoder (TimeStep.encode,
 * web/core/timestep.js:797; driver.js:53-74) plays them here unchanged: same tape JSON,
 * same kernel ABI (data/kernels/kernels.json), same word-addressed memory layout, same
 * per-dispatch region hashes (replay.js:407-418).  Offsets are 64-bit words (the
 * reference's ARG slots hold u32 word offsets, replay.js:266-268).
 *
 * Conventions: every call returns 0 on success or a negative TE_E* code; the message of
 * the last failure is te_last_error(ctx).  One context = one CUDA device + one stream;
 * a context is not thread-safe.  Device work is stream-ordered; te_read, te_read_hashes
 * and te_sync block until it finishes.
 */
#ifndef THUNDERSTEP_H
#define THUNDERSTEP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TE_OK 0
#define TE_EINVAL -1     /* bad argument or malformed tape / kernels JSON */
#define TE_ENOKERNEL -2  /* the tape names a kernel this library does not implement */
#define TE_ECUDA -3      /* a CUDA runtime call failed */
#define TE_ESTATE -4     /* call out of order (e.g. te_run before te_plan) */
#define TE_ERANGE -5     /* offset / size outside the planned memory */

/* Execution modes of te_run (te_set_mode). */
#define TE_MODE_EXACT 0  /* one CUDA kernel per tape dispatch, reference order */
#define TE_MODE_FUSED 1  /* recognised step phases run as fused kernels (see te_set_mode) */

/* te_config.flags */
#define TE_FLAG_DEFER_MISSING 1  /* te_plan accepts tapes naming kernels this library does
                                    not implement; running such an op fails with
                                    TE_ENOKERNEL (the reference fails at build(),
                                    replay.js:240) */

typedef struct te_ctx te_ctx;

typedef struct te_config {
  int device;          /* CUDA device ordinal */
  int flags;           /* TE_FLAG_* */
  uint64_t reserved[4];
} te_config;

typedef struct te_info {
  uint64_t mem_words;    /* Replayer.memWords (replay.js:65) */
  uint64_t buffers_end;  /* Replayer.buffersEnd (replay.js:51) */
  uint64_t scratch_base; /* word offset of the per-thread scratch area (replay.js:63) */
  uint32_t hash_count;   /* Replayer.hashCount (replay.js:113) */
  uint32_t num_buffers;  /* tape.buffers.length */
  uint32_t num_ops;      /* ops of the active step (kernel dispatches + copies) */
  uint32_t num_dispatches;
} te_info;

/* new Replayer(device, tape, kernels, sources) (replay.js:37-42): create a context. */
int te_create(const te_config *cfg, te_ctx **out);

/* Replayer.plan(withHashes) + Replayer.build() (replay.js:46-66, 180-209): lay out the
 * word memory for `tape_json`, allocate it on the device, write the setBytes payloads
 * and prepare the dispatch list of tape.steps[0].  `kernels_json` is the reference's
 * kernels.json (parameter ABI per kernel; NULL = the built-in table of this library). */
int te_plan(te_ctx *ctx, const char *tape_json, size_t tape_len, const char *kernels_json,
            size_t kernels_len, int with_hashes);

int te_get_info(te_ctx *ctx, te_info *out);

/* Replayer.base[buf_id] (replay.js:49): word offset of a tape buffer in memory. */
int te_buffer_base(te_ctx *ctx, int buf_id, uint64_t *word_off);

/* Replayer.upload(id, u8) (replay.js:301): copy host bytes to the start of a buffer. */
int te_upload(te_ctx *ctx, int buf_id, const void *data, size_t bytes);

/* Replayer.writeWords(off, data) (replay.js:212-225): copy host bytes to word `word_off`. */
int te_write_words(te_ctx *ctx, uint64_t word_off, const void *data, size_t bytes);

/* Replayer.useStep(cmds) (replay.js:127-146): make `cmds_json` (a JSON array of tape
 * commands) the active step.  Same structure as a known step: only changed setBytes
 * payloads are rewritten; a new structure is planned once and cached. */
int te_use_step(te_ctx *ctx, const char *cmds_json, size_t len);

/* Replayer.encodeSteps(enc, n, withHashes) + queue submit (replay.js:335-366): play the
 * active step `nsteps` times.  With hashes, every written binding of every dispatch adds
 * its region hash to its slot (replay.js:102-115, 407-418); slots are not cleared. */
int te_run(te_ctx *ctx, int nsteps, int with_hashes);

/* No counterpart in the reference (its writes and reads are whole-queue operations):
 * te_write_words / te_read queued on the context's stream without waiting, so that a
 * caller driving several contexts overlaps one context's copies with another's step.
 * The host buffer must stay valid and unchanged until te_sync returns (pinned memory
 * lets the copy engine run concurrently); asynchronous writes must lie inside the tape
 * buffers (not the setBytes area, whose host mirror te_write_words keeps). */
int te_write_words_async(te_ctx *ctx, uint64_t word_off, const void *data, size_t bytes);
int te_read_async(te_ctx *ctx, uint64_t word_off, uint64_t words, void *out);

/* encodeSteps(enc, 1, withHashes, lastOp) restricted to ops [first_op, last_op]. */
int te_run_ops(te_ctx *ctx, int first_op, int last_op, int with_hashes);

/* Replayer.encodeDiag(enc) (replay.js:299): play tape.diag once. */
int te_run_diag(te_ctx *ctx);

/* Replayer.read(words, offWords) (replay.js:368-383): copy memory words to the host. */
int te_read(te_ctx *ctx, uint64_t word_off, uint64_t words, void *out);

/* Replayer.readHashes() (replay.js:385-395): copy min(n, hash_count) slots. */
int te_read_hashes(te_ctx *ctx, uint32_t *out, size_t n);
int te_clear_hashes(te_ctx *ctx);

/* Device address of memory word `word_off`, for callers that keep data on the GPU. */
int te_device_ptr(te_ctx *ctx, uint64_t word_off, void **out);

/* TE_MODE_EXACT (default) or TE_MODE_FUSED.  Fused mode replaces recognised phases of
 * the step (acoustic substeps, advection of a variable) by fused kernels; prognostic
 * fields are bit-identical to exact mode, the contents of the step's scratch fields
 * (fx, fy, fz, fpk, cA, cB, ...) are not kept.  Hash runs always use exact mode. */
int te_set_mode(te_ctx *ctx, int mode);

/* Fused-mode plan of the active step (built on first use): segments are runs of exact
 * ops or fused phases.  kind: 0 = exact ops, 1 = acoustic substep (3 kernels),
 * 2 = periodic halo fills, 3 = advection of one variable (1 kernel).  te_run_segment
 * plays one segment (part = -1) or one kernel of it (part >= 0), for profiling. */
typedef struct te_segment {
  int kind;
  int first_op, last_op;
  int kernels;
} te_segment;
int te_fused_segments(te_ctx *ctx, te_segment *out, int max, int *count);
int te_run_segment(te_ctx *ctx, int seg, int part);

/* Name of op `op` of the active step ("copy" for a blit copy), or NULL. */
const char *te_op_name(te_ctx *ctx, int op);

int te_sync(te_ctx *ctx);
void te_destroy(te_ctx *ctx);
const char *te_last_error(te_ctx *ctx);

/* Run on a caller-owned CUDA stream (a cudaStream_t; NULL = the context's own stream),
 * e.g. to time launches with events recorded on that stream. */
int te_set_stream(te_ctx *ctx, void *cuda_stream);

/* The built-in kernel table as kernels.json-shaped JSON ({name: {params: [...]}}),
 * written to buf (NUL-terminated, truncated to n).  Returns the full length. */
size_t te_kernel_table_json(char *buf, size_t n);

/* Region hash of `words` host words with the reference formula (replay.js:407-418). */
uint32_t te_region_hash_host(const uint32_t *words, uint64_t n);

/* Self-check of the library's own arithmetic (no counterpart in the reference): raises
 * every binary32 bit pattern in [lo, hi) to the power p by the short binary64 route that
 * update_rho_prs uses and by the two-float route of the reference's f_rr_pow_cr
 * (update_rho_prs.wgsl), on the current CUDA device, and returns how many results differ
 * and the lowest differing pattern (0xffffffff if none).  Synchronous; allocates 16 bytes
 * of device memory for the counters. */
int te_check_pow(float p, uint32_t lo, uint32_t hi, uint64_t *mismatches, uint32_t *first_bad);

/* ---- Discrete adjoint of a step (no counterpart in the reference; the forward/backward
 * pair behind a torch.autograd.Function-shaped host interface).  The adjoint memory has
 * the layout of the word memory: the adjoint of the value at word w is the float at word
 * w.  Supported steps are those whose every kernel has an adjoint operator: the
 * dynamics-core step (WENO / upwind advection of th', u, v, w, the acoustic substeps and
 * the buoyancy coupling, thermodynamic coefficients held fixed); other kernels fail with
 * TE_ENOKERNEL.
 *
 * te_adjoint_forward: runs `nsteps` steps of the active step from the current memory,
 *   copying the tape buffers every `checkpoint_every` steps (device memory:
 *   ceil(nsteps / checkpoint_every) copies of the tape buffers, plus an undo log of
 *   `checkpoint_every` steps: every region each op writes), and clears the adjoint memory.
 * te_adjoint_backward: with the adjoint memory holding d(cost)/d(state after the last
 *   step) (set with te_adjoint_write_words), replaces it by d(cost)/d(state before the
 *   first step) and returns memory to that first state.  Each block of checkpoint_every
 *   steps is replayed once from its checkpoint with the undo log, then walked in reverse
 *   op by op. */
int te_adjoint_forward(te_ctx *ctx, int nsteps, int checkpoint_every);
int te_adjoint_backward(te_ctx *ctx);
int te_adjoint_write_words(te_ctx *ctx, uint64_t word_off, const void *data, size_t bytes);
int te_adjoint_read(te_ctx *ctx, uint64_t word_off, uint64_t words, void *out);
int te_adjoint_zero(te_ctx *ctx);
int te_adjoint_device_ptr(te_ctx *ctx, uint64_t word_off, void **out);
/* Device bytes held by the adjoint state (adjoint memory, checkpoints, undo log). */
int te_adjoint_memory(te_ctx *ctx, uint64_t *bytes);

/* ---- Launch-shape autotuner (no counterpart in the reference).  Times every candidate
 * thread-block shape of each per-dispatch op of the active step whose launcher takes its
 * block from the op (`reps` launches each, CUDA events on the context's stream), keeps a
 * shape only when it beats the default 32 x 4 by more than 3 %, and restores memory
 * afterwards.  *tuned_ops (may be NULL) receives the number of ops that changed shape. */
int te_autotune(te_ctx *ctx, int reps, int *tuned_ops);

/* ---- Ensembles (no counterpart in the reference): independent planned contexts on one
 * device, of any grid size, time step and substep count, advanced together.  Each
 * member's step (in the member's mode at creation) becomes a child graph of one
 * ensemble graph without edges between members; te_ensemble_run launches it once per
 * large step on the ensemble's own stream, so the members' kernels run concurrently.
 * Members must not be stepped through their own contexts while an ensemble run is in
 * flight; te_ensemble_sync waits for it. */
typedef struct te_ensemble te_ensemble;
int te_ensemble_create(te_ctx *const *members, int n, te_ensemble **out);
int te_ensemble_run(te_ensemble *ens, int nsteps);
int te_ensemble_stream(te_ensemble *ens, void **cuda_stream);
int te_ensemble_sync(te_ensemble *ens);
const char *te_ensemble_last_error(te_ensemble *ens);
void te_ensemble_destroy(te_ensemble *ens);

/* Fields of one vertically implicit w-pi' column solve: device pointers to the start of
 * each field (index 0 = point (i, j, k) = (-3, -3, 0) of the halo-3 layout, strideJ =
 * nx + 7, strideK = ny + 7). */
typedef struct te_wsolve_fields {
  const float *pk1, *pk2, *qk, *mm, *fpk, *wten, *pp3d;
  float *w; /* in: w before the solve; out: w after it */
} te_wsolve_fields;

/* No counterpart in the reference: an addition of this library for callers that cannot
 * allocate device memory where they run the solve (their pool belongs to another
 * allocator, or the host process forbids allocation after start-up).  It computes the
 * same w as the tape kernel acoustic_w_solve (bit for bit) but keeps the Thomas
 * coefficients, which the tape writes to the arena fields cA and cB, in a fixed 64 MiB
 * array inside this library; it allocates nothing.
 *   - Limit: nx * ny * (nz - 2) <= 8,388,608 (256 x 256 columns up to nz = 130) and
 *     ny <= 262,140; larger grids, nz < 3 or a NULL field return TE_ERANGE / TE_EINVAL
 *     with a message in `err` (`err_len` bytes, may be NULL) and launch nothing.
 *   - Every GPU that loads the library holds the 64 MiB until the process exits.
 *   - Runs on the current CUDA device, on `cuda_stream` (NULL = legacy default stream),
 *     asynchronously, in the device's primary context (the CUDA runtime's).  The first
 *     call on a device looks up the array's device address and keeps it for the life of
 *     the process; make that first call before any stream capture, and do not call
 *     again after cudaDeviceReset on that device.
 *   - Nothing in the array has to start at zero: each column's coefficients are written
 *     before they are read.  All calls share the array, so calls that may overlap on the
 *     GPU (different streams, or different host threads) race: order them. */
int te_w_solve_static_scratch(const te_wsolve_fields *f, int nx, int ny, int nz, float dts, float alph,
                              float beta, void *cuda_stream, char *err, size_t err_len);

#ifdef __cplusplus
}
#endif
#endif

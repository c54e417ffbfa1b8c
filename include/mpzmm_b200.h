/*
 * mpzmm_b200 -- exact big-integer matrix product on one B200 (sm_100a).
 *
 * C ABI of libmpzmm_b200.so.  Two layers:
 *
 *  1. Drop-in replacements for the reference's public matmul API
 *     (alexp616/rforest src/include/hwmpz.h), same names and signatures, so
 *     rforest links this library in place of src/lib/hwmpz.c.
 *  2. Status-returning entry points over plain arrays ("packed vectors",
 *     below) for general m x k by k x n shapes, batches of independent
 *     products, device-resident plans, and a serving queue.  They have no
 *     counterpart in the reference, which reports no errors
 *     (src/lib/hwmpz.c:69,146 use assert / exit).
 *
 * Packed vector: entry e has |sizes[e]| 64-bit limbs, least significant
 * first, at limbs[offs[e]], and the sign of sizes[e] -- GMP's own
 * (_mp_size, _mp_d) convention.  Matrices are row-major.
 *
 * All arithmetic is exact integer arithmetic on the GPU; there is no CPU
 * fallback.  Without a usable CUDA device every compute entry point returns
 * MPZMM_ERR_CUDA (the void reference-compatible ones call the fatal hook).
 */
#ifndef MPZMM_B200_H
#define MPZMM_B200_H

#include <stddef.h>
#include <stdint.h>

#include "mpzmm_gmp_abi.h"

#if defined(__GNUC__)
#define MPZMM_API __attribute__((visibility("default")))
#else
#define MPZMM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define MPZMM_OK 0
#define MPZMM_ERR_ARG 1        /* malformed dimensions or pointers        */
#define MPZMM_ERR_TOO_LARGE 2  /* product exceeds the supported size      */
#define MPZMM_ERR_CAPACITY 3   /* an output capacity is too small         */
#define MPZMM_ERR_CUDA 4       /* CUDA runtime failure / no device        */
#define MPZMM_ERR_NOMEM 5      /* host or device allocation failed        */
#define MPZMM_ERR_STATE 6      /* not set up, or object in the wrong state */
#define MPZMM_ERR_TIMEOUT 7    /* a bounded wait gave up                  */
#define MPZMM_ERR_BUSY 8       /* admission refused (queue/memory full)   */
#define MPZMM_ERR_BOUNDS 9     /* debug bounds check: a descriptor outside
                                  the workspace (nothing was launched)     */

/* ======================================================================
 * 1. Reference-compatible API (src/include/hwmpz.h)
 * ====================================================================== */

/* Replaces hw_mpz_setup (src/include/hwmpz.h:74, src/lib/hwmpz.c:51):
   selects the CUDA device (MPZMM_DEVICE env, default 0), builds prime and
   twiddle tables on it.  Idempotent. */
MPZMM_API void hw_mpz_setup(void);
/* Replaces hw_mpz_clear (src/include/hwmpz.h:75, src/lib/hwmpz.c:52). */
MPZMM_API void hw_mpz_clear(void);

/* Replaces mpz_rmatrix_mult_fft (src/include/hwmpz.h:127-129,
   src/lib/hwmpz.c:65-130): C = A * B exactly, A r x d, B d x d, C r x d,
   row-major mpz_t arrays.  C entries must be initialised; they are grown with
   GMP's mpz_realloc (so a caller-installed GMP allocator is honoured).
   w is unused, as in the reference.  No aliasing of C with A or B.
   Errors call mpzmm_fatal (see mpzmm_set_fatal_hook). */
MPZMM_API void mpz_rmatrix_mult_fft(mpz_t *C, mpz_t *A, int r, mpz_t *B, int d, mpz_t w);

/* Replaces cu_mpz_rmatrix_mult_fft (src/include/hwmpz.h:132-134,
   src/lib/hwmpz.c:132-247): the same GPU path (every size, no lgN window). */
MPZMM_API void cu_mpz_rmatrix_mult_fft(mpz_t *C, mpz_t *A, int r, mpz_t *B, int d, mpz_t w);

/* Replaces mpz_rmatrix_gpu_fft_suitable (src/include/hwmpz.h:136-139,
   src/lib/hwmpz.c:249-255): 1 if this library can multiply these operands. */
MPZMM_API int mpz_rmatrix_gpu_fft_suitable(mpz_t *A, int r, mpz_t *B, int d);

/* src/include/hwmpz.h:130 and :134 (header inlines in the reference).  A
   caller that also includes the reference's own hwmpz.h first (whose guard is
   _HWMPZ_INCLUDE_) keeps that header's definitions of these two wrappers;
   the declarations above are then checked against it by the compiler. */
#ifndef _HWMPZ_INCLUDE_
static inline void mpz_matrix_mult_fft(mpz_t *C, mpz_t *A, mpz_t *B, int d, mpz_t w) {
  mpz_rmatrix_mult_fft(C, A, d, B, d, w);
}
static inline void cu_mpz_matrix_mult_fft(mpz_t *C, mpz_t *A, mpz_t *B, int d, mpz_t w) {
  cu_mpz_rmatrix_mult_fft(C, A, d, B, d, w);
}
#endif

/* Fatal-error hook for the void entry points above (default: print the
   error to stderr and abort()).  No counterpart in the reference. */
typedef void (*mpzmm_fatal_fn)(int status, const char *message);
MPZMM_API void mpzmm_set_fatal_hook(mpzmm_fatal_fn fn);

/* ======================================================================
 * 2. Extended API (no counterpart in the reference)
 * ====================================================================== */

/* Explicit set-up on a device; returns a status.  hw_mpz_setup() calls it
   with the default device. */
MPZMM_API int mpzmm_setup(int device);
/* Options (process-wide; a plan keeps the values it was built with).
   MPZMM_OPT_CONTRACT selects the frequency-domain contraction engine:
   0 automatic (per size class, the engine mpzmm_autotune measured faster;
   tensor cores -- tcgen05 kind::i8 -- only for m, n <= 1024 and k <= 64),
   1 CUDA cores only, 2 tensor cores wherever the shape allows.
   The environment variable MPZMM_CONTRACT sets the initial value.
   MPZMM_OPT_CHUNK_LIMBS sets the input limbs per chunk of a pipelined
   one-shot batch (mpzmm_matmul_batch): 0 (default) chooses a 32nd of the
   batch, kept between 2^22 and 2^26 limbs; a batch no larger than one
   chunk runs unchunked.
   MPZMM_OPT_CHECK_BOUNDS (debug, default 0; environment variable
   MPZMM_CHECK_BOUNDS=1): before every execute of a plan (batches, chains,
   server batches included) a kernel checks every descriptor's extents
   against the workspace and writes a status word; on a violation the call
   returns MPZMM_ERR_BOUNDS without launching anything else.  It costs a
   stream synchronisation per execute. */
#define MPZMM_OPT_CONTRACT 1
#define MPZMM_OPT_CHUNK_LIMBS 2
#define MPZMM_OPT_CHECK_BOUNDS 3
/* Failure injection, for tests of a caller's error handling (no counterpart
   in the reference; nothing here faults a GPU).  MPZMM_OPT_TEST_STALL_TC:
   the next `value` tensor-core contraction launches issue no tensor work,
   so each of their CTAs' bounded waits (one second) runs out and the call
   returns MPZMM_ERR_TIMEOUT; the context stays usable.
   MPZMM_OPT_TEST_FAIL_ALLOC: the next `value` device or pinned-host
   allocations of a workspace fail as if out of memory (MPZMM_ERR_NOMEM).
   Reading either option returns the injections still pending. */
#define MPZMM_OPT_TEST_STALL_TC 100
#define MPZMM_OPT_TEST_FAIL_ALLOC 101
MPZMM_API int mpzmm_set_option(int option, int value);
MPZMM_API int mpzmm_get_option(int option);

/* Pinned host memory.  Copies whose host side lies wholly inside memory
   from mpzmm_host_alloc, or inside a range registered with
   mpzmm_host_register (cudaHostRegister), go straight between that memory
   and the device: no staging copy, and the DMA runs at full link speed.
   Other host memory is staged through the library's pinned buffers. */
MPZMM_API int mpzmm_host_alloc(size_t bytes, void **out);
MPZMM_API int mpzmm_host_free(void *p);
MPZMM_API int mpzmm_host_register(void *p, size_t bytes);
MPZMM_API int mpzmm_host_unregister(void *p);

/* Statistics of the last one-shot batch (mpzmm_matmul_batch, mpzmm_matmul,
   mpz_rmatrix_mult_fft), summed over its chunks (any pointer may be NULL):
   host nanoseconds ns4[0] planning, [1] input copies (staging and
   queueing), [2] kernel and output copy queueing, [3] waiting and writing
   results; the chunk count; bytes4[0] host->device and [1] device->host
   bytes, [2] and [3] the parts of those that moved straight between the
   caller's pinned memory and the device. */
MPZMM_API int mpzmm_batch_stats(int64_t *ns4, int64_t *chunks, int64_t *bytes4);

/* Per-chunk timeline of the last one-shot batch: *nchunks gets its chunk
   count and rows (may be NULL) up to max_chunks rows of
   MPZMM_TIMELINE_FIELDS doubles, in ms from the batch's start: [0] planning
   began, [1] planning ended, [2] queueing began, [3] queueing ended (host
   clock); [4] the input copies could start (the copy stream reached them),
   [5] input copies done, [6] kernels done, [7] result copies done (device
   events, -1 where the batch failed before them); [8] bytes host->device,
   [9] bytes device->host. */
#define MPZMM_TIMELINE_FIELDS 10
MPZMM_API int mpzmm_batch_timeline(double *rows, int max_chunks, int *nchunks);

/* How mpzmm_matmul_batch would split a batch whose products have limbs[t]
   input limbs each (A's and B's limbs together), with chunk_limbs as
   MPZMM_OPT_CHUNK_LIMBS (0: automatic): *nchunks gets the chunk count and
   bounds (may be NULL; up to max_bounds values) the product index where
   each chunk starts, then the count.  Host only; no device needed. */
MPZMM_API int mpzmm_batch_chunks(int count, const int64_t *limbs, int64_t chunk_limbs,
                                 int64_t *bounds, int max_bounds, int *nchunks);

/* Autotuner: times a representative batch per size class (m = n = 4, 8,
   16, 32, 64 by k = 8, 16, 32, 64 terms, 2^14-bit entries, copies of one
   product until every SM has several blocks' work) on CUDA cores and on
   tensor cores and makes automatic mode use tensor cores for that class
   where their split + forward + contraction took under 9/10 of the
   CUDA-core time (their operands are written frequency-blocked, which
   costs the forward a little; until the autotuner runs automatic mode uses
   CUDA cores).  ms_out, if not NULL, receives 40 floats: {CUDA, tensor}
   contraction milliseconds per class, k-major. */
MPZMM_API int mpzmm_autotune(void *stream, float *ms_out);

/* Human-readable message for the last error on the calling thread. */
MPZMM_API const char *mpzmm_last_error(void);
/* 1 if a CUDA device is usable, else 0 (never aborts). */
MPZMM_API int mpzmm_device_available(void);

/* Exact C = A * B for A m x k, B k x n, C m x n (packed vectors in host
   memory).  C entry e is written at c_limbs[c_offs[e]] with capacity
   c_caps[e] limbs and its signed size stored in c_sizes[e].  A capacity of
   mpzmm_output_limbs(...) always suffices.  stream: a cudaStream_t, or NULL
   for the library's own stream.  Synchronous: returns after C is written. */
MPZMM_API int mpzmm_matmul(int m, int k, int n,
                 const uint64_t *a_limbs, const int64_t *a_offs, const int32_t *a_sizes,
                 const uint64_t *b_limbs, const int64_t *b_offs, const int32_t *b_sizes,
                 uint64_t *c_limbs, const int64_t *c_offs, const int64_t *c_caps,
                 int32_t *c_sizes, void *stream);

/* Limbs that always suffice for every entry of an m x k by k x n product
   whose A entries have at most a_bits bits and B entries at most b_bits
   bits: ceil((a_bits + b_bits + ceil(log2 k) + 1) / 64).  Host-only. */
MPZMM_API int64_t mpzmm_output_limbs(int k, int64_t a_bits, int64_t b_bits);

/* One product of a batch (host pointers, packed vectors as above). */
typedef struct mpzmm_product {
  int m, k, n;
  const uint64_t *a_limbs;
  const int64_t *a_offs;
  const int32_t *a_sizes;
  const uint64_t *b_limbs;
  const int64_t *b_offs;
  const int32_t *b_sizes;
  uint64_t *c_limbs;
  const int64_t *c_offs;
  const int64_t *c_caps;
  int32_t *c_sizes;
} mpzmm_product;

/* Many independent products of uneven shapes and sizes in one pass: one
   launch per pipeline stage and size class for the batch, or, for a batch
   larger than one chunk (MPZMM_OPT_CHUNK_LIMBS), per chunk of whole
   products, with the chunks pipelined so that copies in both directions
   overlap the kernels.  Operand arrays in pinned memory (mpzmm_host_alloc /
   mpzmm_host_register) are copied without staging, short gaps between
   entries included; an output array takes the device's words directly when
   its entries are evenly spaced with capacity at least
   mpzmm_output_limbs(k, exact operand bit lengths).  Synchronous. */
MPZMM_API int mpzmm_matmul_batch(int count, const mpzmm_product *products, void *stream);

/* ---- device-resident chains (no counterpart in the reference) ----
   M = X_0 X_1 ... X_{count-1} left to right (X_0 r x c_0, X_i c_{i-1} x c_i,
   packed vectors as above), the running product kept in device memory
   between steps: step i copies step i-1's result limbs on the device and
   reads its signs and sizes there, so nothing crosses the host link but the
   X_i and the final result.  Each step is planned for a bound of the
   running product (64 x the previous step's output limbs), so every step is
   exact; mpzmm_chain_output_limbs gives the final entries' capacity (-1 for
   a malformed chain).  Synchronous. */
typedef struct mpzmm_matrix {
  int rows, cols;
  const uint64_t *limbs;
  const int64_t *offs;
  const int32_t *sizes;
} mpzmm_matrix;
MPZMM_API int64_t mpzmm_chain_output_limbs(int count, const mpzmm_matrix *mats);
MPZMM_API int mpzmm_chain(int count, const mpzmm_matrix *mats, uint64_t *c_limbs,
                          const int64_t *c_offs, const int64_t *c_caps, int32_t *c_sizes,
                          void *stream);

/* ---- modular reduction by a fixed modulus ----
   Counterpart of the reference's mpzfft_mod_init / mpzfft_mod_mod /
   mpzfft_mod_clear (src/include/mpzfft.h, src/lib/mpzfft.c:59-100), which
   reduce by one modulus d many times through a precomputed Fermat-transform
   reciprocal.  Here: a Barrett reduction whose two big products run on this
   library's engine, batched over all the x of a call.  mpzmm_mod_create
   takes d > 0 (d_size limbs) and the largest |x| to expect in limbs
   (max_x_limbs; larger x are refused with MPZMM_ERR_TOO_LARGE).
   mpzmm_mod_batch writes r_i = x_i mod d in [0, d) for `count` packed x
   (signed, as above) into packed outputs with capacity r_caps (d's limb count
   always suffices, mpzmm_mod_limbs).  Synchronous. */
typedef struct mpzmm_mod mpzmm_mod;
MPZMM_API int mpzmm_mod_create(mpzmm_mod **mod, const uint64_t *d_limbs, int32_t d_size,
                               int64_t max_x_limbs);
MPZMM_API int64_t mpzmm_mod_limbs(const mpzmm_mod *mod);
MPZMM_API int mpzmm_mod_batch(mpzmm_mod *mod, int count, const uint64_t *x_limbs,
                              const int64_t *x_offs, const int32_t *x_sizes, uint64_t *r_limbs,
                              const int64_t *r_offs, const int64_t *r_caps, int32_t *r_sizes,
                              void *stream);
MPZMM_API void mpzmm_mod_destroy(mpzmm_mod *mod);
/* The same over mpz_t arrays: rop[i] = op[i] mod d for i < count, each rop
   grown with mpz_realloc (the reference's mpzfft_mod_mod, batched; rop may
   alias op). */
MPZMM_API int mpzmm_mod_mpz(mpzmm_mod *mod, mpz_t *rop, mpz_t *op, int count, void *stream);

/* ---- device-resident plans (build once, run many times) ---- */
typedef struct mpzmm_plan mpzmm_plan;

/* Plans a batch and copies its inputs to the device.  The products' host
   input arrays are only read during this call. */
MPZMM_API int mpzmm_plan_create(mpzmm_plan **plan, int count, const mpzmm_product *products,
                      void *stream);
/* Runs every kernel of the plan on the inputs already resident in device
   memory; results stay on the device.  Asynchronous on `stream`. */
MPZMM_API int mpzmm_plan_execute(mpzmm_plan *plan, void *stream);
/* Copies the results of the last execute into the products' host outputs
   (c_limbs / c_sizes given at create time).  Synchronous. */
MPZMM_API int mpzmm_plan_download(mpzmm_plan *plan, void *stream);
/* Re-reads the products' host inputs into the plan (same shapes and sizes)
   and copies them to the device.  Asynchronous on `stream`. */
MPZMM_API int mpzmm_plan_upload(mpzmm_plan *plan, void *stream);
MPZMM_API void mpzmm_plan_destroy(mpzmm_plan *plan);
/* A plan that keeps B's transforms across executes (the same B times many
   A): the first execute after create or mpzmm_plan_upload splits and
   transforms both operands, later executes transform only A.
   mpzmm_plan_upload_a re-reads only the A operands (same shapes and signed
   limb counts),
   so their products with the same B skip B's split and transforms;
   mpzmm_plan_upload re-reads both.  Such a plan does not use graph mode.
   (The reference re-splits and re-transforms B on every call,
   src/lib/hwmpz.c:80-105.) */
MPZMM_API int mpzmm_plan_create_fixed_b(mpzmm_plan **plan, int count,
                                        const mpzmm_product *products, void *stream);
MPZMM_API int mpzmm_plan_upload_a(mpzmm_plan *plan, void *stream);

/* CUDA-graph mode (off by default): the first execute captures every launch
   of the plan into a CUDA graph on its stream; later executes replay it as one
   graph launch.  Ignored while stage timing is on. */
MPZMM_API int mpzmm_plan_set_graph(mpzmm_plan *plan, int enable);

/* Stage timing with CUDA events recorded on the execute stream (off by
   default).  Stages: 0 split + forward NTT, 1 contraction, 2 inverse NTT,
   3 CRT + recompose.  mpzmm_plan_stage_times waits for the last timed
   execute, returns the summed milliseconds per stage over all timed
   executes since the previous call (then resets), the kernel launches per
   stage of one execute, and how many executes were timed. */
MPZMM_API int mpzmm_plan_set_timing(mpzmm_plan *plan, int enable);
MPZMM_API int mpzmm_plan_stage_times(mpzmm_plan *plan, float *ms4, int64_t *launches4,
                                     int64_t *executes);

/* Statistics of a plan: kernels launched per execute, device bytes, and the
   chosen (P, r, lgN) of product `index` (any pointer may be NULL). */
MPZMM_API int mpzmm_plan_info(const mpzmm_plan *plan, int64_t *launches_per_execute,
                    int64_t *device_bytes, int index, int *P, int *r, int *lgN);

/* Exact C = A * B without allocating anything: no counterpart in the
   reference.  For callers that cannot allocate device memory -- a process
   whose GPU memory is all owned by a host framework's pool, where a raw
   cudaMalloc fails or escapes the pool's accounting, or a latency-sensitive
   path that cannot pay for cudaMalloc/cudaFree, which may synchronise the
   whole device.  The caller passes device buffers: d_a_limbs / d_b_limbs
   hold the operands' limbs (entry offsets and signed sizes in the HOST
   arrays a_offs/a_sizes, b_offs/b_sizes); results go to d_c_limbs at the
   HOST offsets c_offs with HOST capacities c_caps, and their signed sizes to
   the DEVICE array d_c_sizes.  Every capacity must be at least
   mpzmm_output_limbs(k, 64 * max |a_sizes|, 64 * max |b_sizes|).
   Scratch is a fixed 16 MiB static device array inside the library (plus
   8 MiB of static transform tables), held on every GPU that loads the
   library until exit; products needing more scratch, or a transform longer
   than 2^15 points, are rejected with MPZMM_ERR_TOO_LARGE.  The first call
   on a device sets up that device's tables.  A call on a stream that is
   capturing a CUDA graph is refused (MPZMM_ERR_ARG): its descriptors come
   from a host buffer the next call overwrites, so a replay would be wrong.
   All calls share the one scratch array and leave their data in
   it: calls whose GPU work overlaps race, so serialise them.  Nothing of
   the caller's is touched when a call is refused.  The kernels run
   asynchronously on `stream` (NULL: the legacy default stream); the call
   itself returns once its descriptors have been copied from the library's
   pageable host buffer, which CUDA stages after the stream's earlier work. */
MPZMM_API int mpzmm_matmul_noalloc(int m, int k, int n,
                                   const uint64_t *d_a_limbs, const int64_t *a_offs,
                                   const int32_t *a_sizes,
                                   const uint64_t *d_b_limbs, const int64_t *b_offs,
                                   const int32_t *b_sizes,
                                   uint64_t *d_c_limbs, const int64_t *c_offs,
                                   const int64_t *c_caps, int32_t *d_c_sizes, void *stream);

/* ---- continuous-batching server (no counterpart in the reference) ----
   Up to `slots` batches are in flight, each slot with its own host thread,
   CUDA stream and workspace.  Whenever a slot is free it admits the oldest
   queued request and then later ones of the same size class (small: at
   most 16 MB of inputs and outputs; large: more), in arrival order, into
   one batch while their estimated device
   footprint fits what the in-flight batches leave of `budget_bytes` (0:
   three quarters of the free device memory), with at most `max_batch`
   products per batch (0: no limit) and at most 256 MB of inputs and outputs
   (a larger request is a batch of its own).  Requests that arrive while
   batches run join the next batch; a request's residues stay on the device
   for the whole pipeline.  Each slot's pinned staging is allocated once at
   creation and its device memory comes from a stream-ordered pool of the
   server's own (a quarter of the budget, at most 32 GB, is taken into it at
   creation), so no batch synchronises the device or waits for the driver
   to map memory.  Each slot has two
   streams: batches of small requests run on one of the device's greatest
   stream priority, batches of large ones on one of its least, so a small
   request waits neither inside a large one's batch nor behind its queued
   GPU work.  A request larger than the budget is refused
   (MPZMM_ERR_TOO_LARGE). */
typedef struct mpzmm_server mpzmm_server;
MPZMM_API int mpzmm_server_create(mpzmm_server **server, int64_t budget_bytes, int slots,
                                  int max_batch);
/* Queues one product (host packed vectors; all arrays must stay valid until
   the request completes) and returns its ticket. */
MPZMM_API int mpzmm_server_submit(mpzmm_server *server, const mpzmm_product *request,
                                  uint64_t *ticket);
/* Waits for a ticket (timeout_ms < 0: no limit); returns the request's status
   (MPZMM_ERR_TIMEOUT if the limit passed first). */
MPZMM_API int mpzmm_server_wait(mpzmm_server *server, uint64_t ticket, int64_t timeout_ms);
MPZMM_API int mpzmm_server_poll(mpzmm_server *server, uint64_t ticket, int *done);
/* Steady-clock nanoseconds: submitted, batch launched, result written. */
MPZMM_API int mpzmm_server_ticket_times(mpzmm_server *server, uint64_t ticket,
                                        int64_t *submit_ns, int64_t *start_ns,
                                        int64_t *done_ns);
/* Forgets a completed ticket. */
MPZMM_API int mpzmm_server_release(mpzmm_server *server, uint64_t ticket);
/* Batches launched, products completed, most batches in flight at once. */
MPZMM_API int mpzmm_server_stats(mpzmm_server *server, int64_t *batches, int64_t *products,
                                 int64_t *max_in_flight);
/* Scheduler-thread nanoseconds spent in: plan building, input gather and
   copy, kernel launches, result copy-back and scatter (4 values). */
MPZMM_API int mpzmm_server_phase_ns(mpzmm_server *server, int64_t *ns4);
/* The longest single batch in each of those phases since the previous call
   (4 values, nanoseconds); reading resets them. */
MPZMM_API int mpzmm_server_phase_max_ns(mpzmm_server *server, int64_t *ns4);
/* Admission window: when a slot frees up while other batches are on the GPU,
   it keeps admitting queued requests for up to this many microseconds
   before launching its batch (default 200; 0 launches at once).  With the
   GPU idle a batch always launches at once.  Larger batches at load, at the
   cost of at most the window in latency. */
MPZMM_API int mpzmm_server_set_admission_window(mpzmm_server *server, int64_t microseconds);
/* Finishes queued and in-flight work, then frees the server. */
MPZMM_API void mpzmm_server_destroy(mpzmm_server *server);

/* Parameters (prime count P, coefficient bits r, transform length 2^lgN)
   that the planner picks for a product with k terms whose A and B entries
   have at most a_bits and b_bits bits.  Host-only; no device needed. */
MPZMM_API int mpzmm_choose_params(int64_t a_bits, int64_t b_bits, int k, int *P, int *r,
                        int *lgN);

#ifdef __cplusplus
}
#endif

#endif /* MPZMM_B200_H */

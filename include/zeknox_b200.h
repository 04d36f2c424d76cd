/*
 * zeknox_b200.h -- entry points this library adds to the zeknox ABI.
 *
 * None of these exist in the reference.  They expose the fused commit path
 * (LDE -> bit-reversed leaf-major rows -> Merkle forest in one call), its
 * batched multi-job form, and diagnostics.  All pointers in a job are device
 * pointers on the job's device; sizes are in 64-bit words.
 */
#ifndef ZEKNOX_B200_H
#define ZEKNOX_B200_H

#include <stddef.h>
#include <stdint.h>

#include "utils/rusterror.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Message of the last failure recorded on this host thread by an entry point
 * that returns void (the fill_digests_* family), or NULL.  The string stays
 * valid until the next call on the same thread. */
const char *zeknox_last_error(void);

/* One polynomial-commitment job (Plonky2 PolynomialBatch::from_coeffs /
 * from_values followed by MerkleTree::new on the LDE rows). */
typedef struct {
    uint32_t lg_n;            /* log2 column length before extension (>= 1) */
    uint32_t rate_bits;       /* blowup 2^rate_bits (>= 1) */
    uint32_t cols;            /* number of polynomials (columns, >= 1) */
    uint32_t cap_height;      /* Merkle cap height, <= lg_n + rate_bits */
    uint32_t hash_type;       /* HashType: 0 Poseidon, 1 Keccak, 3 Poseidon2, 4 Monolith */
    uint32_t input_is_values; /* 0: columns are coefficients; 1: evaluations on H (inverse NTT first) */
    uint64_t coset_gen;       /* coset shift; 0 means 7 */
    const uint64_t *input;    /* cols x 2^lg_n, column-major; device memory, or (zeknox_commit only)
                                 host memory, copied in column chunks that overlap the transform */
    uint64_t *leaves;         /* out: 2^(lg_n+rate_bits) rows x cols; row r = evaluation rev(r) */
    uint64_t *digests;        /* out: 2 * (2^(lg_n+rate_bits) - 2^cap_height) x 4 */
    uint64_t *caps;           /* out: 2^cap_height x 4 */
} zk_commit_job;

/* Run one commit on `device_id`, ordered on `stream` (a cudaStream_t; NULL
 * selects the library's stream for the device).  Returns after queuing the work
 * when stream is non-NULL, after completion otherwise. */
RustError zeknox_commit(size_t device_id, const zk_commit_job *job, void *stream);

/* Run `njobs` commits of any sizes as one batch (see DESIGN: batched path):
 * the whole batch is recorded once as a CUDA graph keyed by its shape and
 * replayed on later calls with the same shapes.  Synchronous. */
RustError zeknox_commit_batch(size_t device_id, const zk_commit_job *jobs, uint32_t njobs);

/* Words of temporary device memory zeknox_commit needs for a job (it
 * allocates them from the stream-ordered pool when called). */
uint64_t zeknox_commit_scratch_words(const zk_commit_job *job);

/* One Merkle forest of fill_digests_buf_linear_gpu_with_gpu_ptr's layout. */
typedef struct {
    const uint64_t *leaves;   /* n_leaves x leaf_size, leaf-major */
    uint64_t *digests;        /* 2 * (n_leaves - 2^cap_height) x 4 */
    uint64_t *caps;           /* 2^cap_height x 4 */
    uint64_t n_leaves;
    uint64_t leaf_size;
    uint32_t cap_height;
    uint32_t hash_type;
} zk_merkle_job;

/* Build `njobs` forests (any mix of hashes and sizes) as one CUDA graph whose
 * branches run concurrently; cached and replayed like zeknox_commit_batch.
 * Synchronous. */
RustError zeknox_merkle_batch(size_t device_id, const zk_merkle_job *jobs, uint32_t njobs);

/* The LDE stage of a commit alone: rows[r * cols + b] = LDE_b(rev(r)), the
 * leaf-major bit-reversed matrix (compute_batched_lde + compute_transpose_rev
 * in one pass structure).  coeffs: cols x 2^lg_n column-major; rows:
 * 2^(lg_n+rate_bits) x cols.  coset_gen 0 means 7.  Stream semantics as
 * zeknox_commit. */
RustError zeknox_lde_rows(size_t device_id, uint64_t *rows, const uint64_t *coeffs, uint32_t lg_n, uint32_t rate_bits,
                          uint32_t cols, uint64_t coset_gen, void *stream);

/* zeknox_lde_rows with the leaf rows spread over n_dst destination buffers
 * (a power of two): row r of the 2^(lg_n + rate_bits) rows goes to
 * dst_ptrs[r / R] (R = rows / n_dst) at row r mod R, columns
 * [col_offset, col_offset + cols) of rows of row_stride words.  The
 * destinations may be other GPUs' memory mapped for peer access: the rows then
 * cross NVLink as stores from the row-writing kernel (the LDE and the row
 * exchange of a multi-GPU commit in one pass).  Queued on `stream` (NULL: the
 * device's stream, and the call waits).  No reference counterpart (zeknox's
 * multi-GPU path copies whole columns between GPUs, native/ntt/ntt.cu:315-471). */
RustError zeknox_lde_rows_scatter(size_t device_id, uint64_t *const *dst_ptrs, uint32_t n_dst, const uint64_t *coeffs,
                                  uint32_t lg_n, uint32_t rate_bits, uint32_t cols, uint32_t col_offset,
                                  uint32_t row_stride, uint64_t coset_gen, void *stream);

/* compute_transpose_rev (native/ntt/ntt.cu:182-226) of device buffers,
 * out[rev(i) * cols + b] = in[b * 2^lg_n + i], queued on `stream` (a
 * cudaStream_t; NULL: the device's stream, and the call waits).  No reference
 * counterpart: the reference call is synchronous. */
RustError zeknox_transpose_rev(size_t device_id, uint64_t *output, const uint64_t *input, uint32_t lg_n,
                               uint32_t cols, void *stream);

/* zeknox_lde_rows for callers that cannot allocate device memory: code whose
 * device memory all belongs to another allocator (a framework's caching
 * allocator, or an arena reserved at start-up) or a thread that must not enter
 * the driver's allocator, which can synchronise the device.  No counterpart
 * in the reference.  It never allocates: its inter-pass scratch (32 MiB) and
 * the tables it reads live in file-scope device arrays that every GPU loading
 * the library holds until exit.  Limit: lg_n + rate_bits <= 18; larger sizes
 * are rejected with cudaErrorInvalidValue.  The first call on a device looks
 * up those arrays' addresses and fills the twiddle tables, and waits for that
 * on `stream`.  Every call rebuilds the coset table for its own shape and
 * generator, ahead of its transform on the same stream.  All calls share the
 * scratch and the coset table, so calls that overlap on the GPU race; stream
 * NULL means the legacy default stream and a synchronous call.  A CUDA error
 * pending from earlier work is reported (and left pending) instead of being
 * taken for this call's. */
RustError zeknox_lde_rows_noalloc(size_t device_id, uint64_t *rows, const uint64_t *coeffs, uint32_t lg_n,
                                  uint32_t rate_bits, uint32_t cols, uint64_t coset_gen, void *stream);

/* ---- Serving: continuous batching of commit requests on one GPU ----
 *
 * A server owns a device-memory budget, reserved as one allocation when it is
 * created (jobs then never call the driver's allocator), and `slots` streams.
 * Requests (zk_serve_request) are queued by any host thread; a server thread
 * admits them in arrival order whenever a slot is free and the job's memory
 * (its leaves, digests, caps and scratch, one contiguous range of the
 * reservation) fits -- while the head waits
 * for memory, up to `slots` small requests (<= budget / 8) behind it that fit
 * may start first -- runs the commit on the slot's stream -- so admitted jobs
 * overlap on the device -- copies the caps to the request's host buffer, and
 * records the latency (submit -> caps on host).  Results stay in server-owned
 * device memory until released: release them as they complete, the budget
 * counts them until then. */
typedef struct {
    uint32_t lg_n, rate_bits, cols, cap_height, hash_type, input_is_values;
    uint64_t coset_gen;       /* 0 means 7 */
    const uint64_t *input;    /* cols x 2^lg_n, column-major, read in place by the server's kernels:
                                 device or pinned host memory (pageable host memory is rejected at
                                 submit unless the GPU can read it); must stay valid until done */
    uint64_t *caps_host;      /* host buffer of 2^cap_height x 4 words, filled on completion (may be NULL) */
} zk_serve_request;

/* zk_serve_result.status of a request cancelled while queued */
#define ZK_SERVE_CANCELLED (-10000)

typedef struct {
    int status;               /* 0 queued, 1 running, 2 done, < 0 failed (negated cudaError, or -1 for a shape
                                 rejected when it started) or ZK_SERVE_CANCELLED */
    double latency_ms;        /* submit -> caps on host (done only) */
    double queue_ms;          /* submit -> admitted */
    const uint64_t *leaves, *digests, *caps;  /* device results (done, until released) */
} zk_serve_result;

RustError zeknox_server_create(size_t device_id, uint64_t budget_bytes, uint32_t slots, void **server);
/* zeknox_server_create with flags.  ZK_SERVE_DEVICE_LOOP: a device-resident
 * request loop runs the admitted requests.  Admission is the same (arrival
 * order, the budget, at most min(slots, 16) requests in flight).  The server
 * thread plans each request's stages, copies the plan to device memory and
 * posts it to a ring in mapped host memory.  Stages estimated above 4 ms are
 * split into pieces (at most 64).  One persistent cooperative kernel takes
 * the ring's entries and runs their stages itself, each stage across the
 * whole GPU, with grid barriers between the stages: the fused LDE's passes,
 * then the forest's leaf, level, fold and tail steps.  At every stage
 * boundary it runs the next stage of the active request with the least
 * estimated work left, so a small request is not held up by all of a large
 * one.  The kernel marks each entry done in host memory, and exits after
 * 20 ms without requests (the next post relaunches it).  Every wait of the
 * kernel is bounded in time.  A request whose wait runs out fails with
 * -cudaErrorLaunchTimeout.  Requests in this mode: coefficients or
 * evaluations (the loop then runs the inverse transform first), any hash
 * type, 2^9 <= 2^lg_n <= 2^22.  No reference counterpart. */
#define ZK_SERVE_DEVICE_LOOP 1u
RustError zeknox_server_create_ex(size_t device_id, uint64_t budget_bytes, uint32_t slots, uint32_t flags,
                                  void **server);
/* Build and keep resident every table a request of lg_n in [lg_n_min,
 * lg_n_max] with this rate and coset generator (0 means 7) reads -- twiddles
 * of every pass, inverse twiddles, the LDE coset tables -- so no request waits
 * for a table build.  Synchronous; call before submitting (optional: a request
 * whose tables are missing has them built on the device context's stream, and
 * its slot stream waits for them on the device). */
RustError zeknox_server_prepare(void *server, uint32_t lg_n_min, uint32_t lg_n_max, uint32_t rate_bits,
                                uint64_t coset_gen);
RustError zeknox_server_submit(void *server, const zk_serve_request *req, uint64_t *ticket);
/* Wait up to timeout_ms (< 0: forever) for the ticket; fills *result. */
RustError zeknox_server_wait(void *server, uint64_t ticket, double timeout_ms, zk_serve_result *result);
/* Take a queued request out of the queue: its status becomes
 * ZK_SERVE_CANCELLED.  A request that has started cannot be cancelled. */
RustError zeknox_server_cancel(void *server, uint64_t ticket);
/* Test hook (failure injection on the host, no GPU fault): the next request
 * the server starts fails at `stage` -- ZK_SERVE_FAIL_ALLOC: as if its device
 * memory were refused (status -cudaErrorMemoryAllocation);
 * ZK_SERVE_FAIL_SHAPE: its shape is rejected when it starts (status -1);
 * ZK_SERVE_FAIL_LAUNCH: queuing its kernels fails after its buffers were
 * placed in the budget (status -cudaErrorLaunchFailure).  The failed
 * request's memory and slot are freed at once; later requests are
 * unaffected.  0 clears. */
#define ZK_SERVE_FAIL_ALLOC 1
#define ZK_SERVE_FAIL_SHAPE 2
#define ZK_SERVE_FAIL_LAUNCH 3
/* Device-loop servers only: the next request is posted with its start gate
 * shut, so the loop's bounded wait for it runs out after 20 ms; the request
 * fails with -cudaErrorLaunchTimeout and the loop goes on with the next. */
#define ZK_SERVE_FAIL_GATE 4
RustError zeknox_server_inject_failure(void *server, int stage);
/* Device-loop servers: the per-stage trace of a finished request (until it is
 * released).  *n = its number of stages; for the first `max` of them kinds[q]
 * = the stage (16 + log2 radix: a transform pass, forward or inverse; 2
 * leaves; 3 leaves, four threads per leaf; 4 a tree level; 5 / 6 the
 * cooperative fold / tail; 7 / 8 the fold / tail with one permutation per
 * thread; 9 the copy of an evaluation-form input; 10 the bit-reversal
 * reorder) and ns[q] = its time on the device, barrier to barrier
 * (%globaltimer).  Either array may
 * be NULL.  Requests of the host-driven mode have no trace (*n = 0). */
RustError zeknox_server_trace(void *server, uint64_t ticket, uint32_t *kinds, uint64_t *ns, uint32_t max, uint32_t *n);
/* Free the ticket's device results (returns their bytes to the budget). */
RustError zeknox_server_release(void *server, uint64_t ticket);
/* Bytes currently admitted against the budget, and the peak so far. */
RustError zeknox_server_stats(void *server, uint64_t *in_use_bytes, uint64_t *peak_bytes, uint64_t *completed);
/* Waits for all admitted work, frees everything. */
RustError zeknox_server_destroy(void *server);

/* ---- Tuning (written by zeknox_b200/autotune.py; no reference counterpart)
 * Knobs, each optionally per log2 size (lg = 0xFFFFFFFF: any size):
 *   "leaf_threads.<hash_type>"  Merkle leaf kernel CTA size, 64/128/256 (lg = log2 leaves)
 *   "lde_chunk_mib"             fused-LDE column chunk budget in MiB (lg = log2 N)
 *   "lde_host_chunk_mib"        the same for inputs in host memory (copies overlap the chunks)
 *   "lde_last_logr"             radix exponent of the fused LDE's row-output pass, 1..8 (lg = log2 n)
 *   "wide_level_nodes.<hash_type>"  Merkle levels at least this wide run node-parallel (lg = log2 leaves)
 *   "coop_leaves.<hash_type>"   forests of at most this many leaves hash them with four threads per
 *                               permutation (Poseidon, Poseidon2; lg = log2 leaves)
 * Unset knobs keep the built-in defaults.  Results never depend on the knobs. */
RustError zeknox_tune_set(const char *name, uint32_t lg, uint64_t value);
RustError zeknox_tune_clear(void);
/* Value a knob has for log2 size lg (the size-free entry, else dflt). */
uint64_t zeknox_tune_get(const char *name, uint32_t lg, uint64_t dflt);
/* Load a table: one knob per line, "<name> <lg or *> <value>". */
RustError zeknox_tune_load(const char *path);

/* ---- Self-tests of the device arithmetic (no reference counterpart; the
 * reference checks its primitives from a test binary, native/tests/tests.cu).
 * The lazily reduced arithmetic of the hashes and the NTT takes its rare
 * carry / borrow / wrap branches only near the field's edges (0, p - 1, 2^32
 * neighbours, 2^64 - 2^32, the non-canonical range [p, 2^64)), which uniform
 * data almost never reaches; these calls run the device primitives on chosen
 * operands.  Device buffers; stream NULL: the device's stream, and the call
 * waits.
 *
 * zeknox_field_selftest: for i < n, with x = a[i], y = b[i], z = c[i] (any
 * 64-bit words; xc, yc = their canonical values), writes the canonical result
 * of operation k to out[k * n + i], k < ZK_SELFTEST_OPS:
 *   0 xc + yc            1 xc - yc           2 xc + yc (the NTT's butterfly sum)
 *   3 x * y              4 x * y (lazy product, multiply-assisted reduction)
 *   5 x * y (lazy product, ALU reduction)    6 x^2 (lazy, multiply-assisted)
 *   7 x^2 (lazy, ALU)    8 x * y + z (lazy, multiply-assisted)   9 the same, ALU
 *  10 x^7 (lazy S-box)  11 x^7 (lazy S-box with the squaring routine)
 *  12 x * 2^(z mod 192) 13 x + yc (lazy sum)
 *  14 4 (x y + y z + z x) through the 128-bit accumulator, multiply-assisted
 *  15 the same, ALU     16 x + 5 y + 6 z (carry-counting sum)
 *  17 4 (41 x + 39 y + 34 z) + yc (small-constant dot product)
 *  18 p0 + 2^22 p1 + 2^44 p2 with p0, p1, p2 the low 28 bits of x, y, z
 *  19 x + 2^64 y        20 x + 2^64 (y mod 2^32)      21 x * 2^(y mod 64)
 *  22 x + y (the NTT's lazy sum)            23 x - y (the NTT's lazy difference)
 *  24..33 x * 2^e (the NTT's lazy power-of-two twiddle), e = 1, 24, 31, 32,
 *         60, 63, 64, 72, 84, 95 */
#define ZK_SELFTEST_OPS 34
RustError zeknox_field_selftest(size_t device_id, const uint64_t *a, const uint64_t *b, const uint64_t *c, uint64_t n,
                                uint64_t *out, void *stream);

/* One permutation of each of n states, in place: 12-word states for Poseidon
 * (0), Poseidon-BN128 (2), Poseidon2 (3) and Monolith (4), lanes any 64-bit
 * words in and canonical out; 25-word Keccak-f[1600] states for Keccak (1).
 * cooperative != 0 runs the four-threads-per-state form the Merkle builder
 * uses for narrow tree levels (Poseidon and Poseidon2 only). */
RustError zeknox_permute(size_t device_id, uint64_t *states, uint64_t n, uint32_t hash_type, uint32_t cooperative,
                         void *stream);

/* The checked build (make -C zeknox_b200 checked -> libzeknox_checked.so)
 * tests every global-memory index of the NTT, reorder, transpose and Merkle
 * kernels against the extent of its buffer and skips an access out of range
 * (no trap: the context stays usable).  This call waits for the device and
 * returns the accesses skipped since the last call: record[0] = count,
 * record[1] = the first one's site (OobSite in csrc/bounds.cuh), record[2]
 * its index, record[3] the extent; and clears them.  In the normal build it
 * returns +cudaErrorNotSupported with a zero record.  No reference
 * counterpart (a sanitizer stand-in). */
RustError zeknox_bounds_report(size_t device_id, uint64_t *record);

/* Bounded device waits.  Kernels that wait on bulk-async copies (the
 * transpose's shared-memory stages) give each wait a limit of 1 s; a CTA whose
 * stage has not completed by then stops and raises a status word, and the
 * call returns -cudaErrorLaunchTimeout (calls queued on a caller's stream:
 * the device's next synchronous call).  This test hook makes the next `count`
 * such transposes on the device declare 16 bytes more than they copy, so one
 * wait runs out (after 20 ms) without any fault; the context stays usable.
 * No reference counterpart. */
RustError zeknox_inject_wait_timeout(size_t device_id, uint32_t count);

/* Number of kernels this library has launched so far in the process. */
uint64_t zeknox_launch_count(void);

/* Measured register-resident Goldilocks multiplies per second on the device
 * (the integer roofline the hash kernels are compared against); < 0 on error. */
double zeknox_measure_mul_rate(size_t device_id);

#ifdef __cplusplus
}
#endif

#endif /* ZEKNOX_B200_H */

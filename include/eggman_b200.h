/*
 * eggman_b200.h -- C ABI of libeggman_b200.so, the B200 (sm_100a) engine behind TheEggman.jl's
 * two hafnian hot paths: the subset DP and the Bjorklund/Glynn sieve.
 *
 * Conventions (all entry points):
 *   - Every function returns an int status: EGG_OK (0) or one of the EGG_ERR_* codes below.
 *     Nothing throws or aborts across the ABI; egg_last_error() gives a message for the calling
 *     thread's last failure.
 *   - Pointers are plain host pointers unless the name ends in _device (then device pointers and
 *     a cudaStream_t passed as void*).  Inputs are borrowed for the call only.
 *   - Matrices are column-major (Julia order); complex values are interleaved (re, im) pairs of
 *     the real type, exactly as Julia lays out Complex{Float64}/Complex{Float32}.
 *   - One device context per process and one internal lock, mirroring the reference's
 *     _DEVICE_PLAN_LOCK (src/dp.jl:542): calls are serialised, and the host-pointer calls are
 *     synchronous to the caller.  The _device calls return once their work is enqueued; it uses
 *     the library's own work buffers, so _device calls whose work could run on the GPU at the
 *     same time (different streams, not ordered by events) race.
 *   - The library never falls back to a CPU implementation.
 */
#ifndef EGGMAN_B200_H
#define EGGMAN_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------------ */
#define EGG_OK 0
#define EGG_ERR_ARGUMENT 1   /* bad argument value (the reference's ArgumentError) */
#define EGG_ERR_DIMENSION 2  /* inconsistent sizes (the reference's DimensionMismatch) */
#define EGG_ERR_TOO_LARGE 3  /* plan or batch cannot be represented / would not fit (src/dp.jl:224-243) */
#define EGG_ERR_NO_PLAN 4    /* no device plan resident for (K, layout): upload or build one first */
#define EGG_ERR_CUDA 5       /* a CUDA runtime call failed */
#define EGG_ERR_TIMEOUT 6    /* a bounded device wait ran out */
#define EGG_ERR_NO_DEVICE 7  /* no usable CUDA device */
#define EGG_ERR_PLAN_INVALID 8 /* an uploaded plan failed the device-side structure check */

/* ---- element types ----------------------------------------------------------------------- */
#define EGG_F64 0   /* Float64 */
#define EGG_C128 1  /* ComplexF64 */
#define EGG_F32 2   /* Float32 */
#define EGG_C64 3   /* ComplexF32 */
#define EGG_I64 4   /* Int64 entries; DP states and results are Int128 (two int64 words, low first) */

/* ---- DP precision modes ------------------------------------------------------------------ */
#define EGG_PREC_EXACT 0  /* DP: one thread per state, plan order, no FMA contraction: bit-identical to
                             the reference's CPU _dp_states! (src/dp.jl:344-363).  Sieve: every
                             term in the reference's loop order and rounding. */
#define EGG_PREC_FMA 1    /* DP: plan order with fused multiply-add (the reference GPU kernel's
                             rounding, ext/TheEggmanKernelAbstractionsExt.jl:47-51).  Sieve: the
                             register-resident fast kernels. */
#define EGG_PREC_MIXED 2  /* FP32 multiplies, FP64 per-state accumulation, FP32 state storage
                             (F64/C128 inputs only) */

/* ---- library ----------------------------------------------------------------------------- */

/* Library version string. */
const char *egg_version(void);

/* Message describing the calling thread's most recent failure ("" if none). */
const char *egg_last_error(void);

/* Kernel launches the library has made since it was loaded, all entry points together (a
 * diagnostic: read it before and after a call to count that call's launches).  No counterpart in
 * the reference. */
int64_t egg_launch_count(void);

/* A diagnostic of the reference-arithmetic sieve's division: for i < n (n <= 2^26, host arrays)
 * writes to q_shared[i] the quotient a[i]/b[i] as the sieve's reference-arithmetic tiles form it
 * (one correctly rounded reciprocal of the divisor, then Markstein's corrections; the full division
 * where operands or quotient leave [2^-1000, 2^1000]) and to q_rn[i] the device's correctly rounded
 * quotient.  The two must agree bit for bit, as the reference's `/` does (src/hafnian.jl:235).
 * Runs synchronously on the calling thread's current device, allocating 32n bytes there for the
 * call.  No counterpart in the reference. */
int egg_selfcheck_division(const double *a, const double *b, int64_t n, double *q_shared, double *q_rn);

/* Bind the library to one CUDA device (idempotent; the first call of any other entry point does
 * this with device 0).  Fails with EGG_ERR_NO_DEVICE if there is none.  The library's streams,
 * plans and work buffers belong to that device: binding another device in the same process fails
 * with EGG_ERR_ARGUMENT, and so does any later call made while the calling thread's current device
 * is a different one.  (egg_sieve_device_noalloc keeps its state per device and is the exception:
 * it runs on the caller's current device.) */
int egg_init(int device);

/* Device bytes held by resident plans and reusable work buffers.
 * Replaces gpu_cache_bytes(), src/dp.jl:552-560. */
int64_t egg_cache_bytes(void);

/* Release every resident plan and work buffer.  Replaces empty_gpu_cache!(), src/dp.jl:567-573. */
int egg_cache_clear(void);

/* Device bytes one DP batch needs besides the shared plan: B x (nstates + npairs) elements of
 * the given type.  Replaces dp_batch_bytes(N, T, B), src/dp.jl:584-587.  Returns -1 on a bad
 * argument. */
int64_t egg_dp_batch_bytes(int N, int dtype, int64_t B);

/* ---- subset DP plans (HafnianDPPlan{I}, src/dp.jl:150-156) -------------------------------- */

/* Closed-form plan size, _dp_counts(K) (src/dp.jl:192-208). */
int egg_dp_counts(int K, int64_t *nstates, int64_t *ntrans);

/* Copy a host-built plan to the device and keep it resident, keyed by (K, idx_bytes).
 * idx_bytes is 4 (Int32 layout, pair bits 9) or 8 (Int64, pair bits 12); arrays are the
 * reference's 1-based starts[nstates+1], trans[ntrans], levels[nlevels].  Idempotent: a
 * resident plan for the key is kept.  The structure is checked on the device (every child in
 * the previous level, every pair index in 1..K(K-1)/2, uniform out-degree per level) and a plan
 * that fails is refused with EGG_ERR_PLAN_INVALID.  A plan equal entry for entry to the layout of
 * _build_dp_plan is then kept in closed form (its array is released and never read again, with
 * identical results); any other valid plan keeps its array and is evaluated in its own order.
 * Replaces _device_plan(backend, plan), ext/TheEggmanKernelAbstractionsExt.jl:31-42. */
int egg_plan_upload(int K, int idx_bytes, const void *starts, const void *trans, const void *levels,
                    int64_t nlevels, int64_t nstates, int64_t ntrans);

/* Make the degree-K plan of _build_dp_plan(K, I) (src/dp.jl:223-304) resident in closed form:
 * its states are the colex-ranked subsets of each level, so the evaluation derives every
 * transition from the state's rank and no transition array is stored.  Same key and caching as
 * egg_plan_upload; refuses what the reference refuses (src/dp.jl:224-234) with
 * EGG_ERR_TOO_LARGE. */
int egg_plan_build(int K, int idx_bytes);

/* Sizes of a resident plan (EGG_ERR_NO_PLAN if absent); device_bytes is 0 for a closed-form
 * plan. */
int egg_plan_info(int K, int idx_bytes, int64_t *nstates, int64_t *ntrans, int64_t *nlevels,
                  int64_t *device_bytes);

/* Copy a resident plan back to the host in the reference layout (starts[nstates+1],
 * trans[ntrans], levels[nlevels], element size idx_bytes).  A closed-form plan is written out
 * through a temporary device array of ntrans * idx_bytes bytes. */
int egg_plan_download(int K, int idx_bytes, void *starts, void *trans, void *levels);

/* Drop one resident plan. */
int egg_plan_release(int K, int idx_bytes);

/* ---- subset DP evaluation ---------------------------------------------------------------- */

/* Hafnians of B instances of degree K on the resident (K, idx_bytes) plan.
 * P is the host B x npairs gathered-pair matrix of _gather_pairs_batch (src/dp.jl:479-512),
 * column-major with the instance index fastest (element (b, q) at b + q*B), npairs = K(K-1)/2;
 * out receives B values (EGG_I64: B Int128 values).  max_batch > 0 evaluates in chunks of at
 * most that many instances (0: one chunk).  prec is an EGG_PREC_* mode.
 * Replaces _haf_dp_backend(backend, P, plan; max_batch),
 * ext/TheEggmanKernelAbstractionsExt.jl:90-146 (hook declared at src/dp.jl:525). */
int egg_dp_batch(int K, int idx_bytes, int dtype, int prec, const void *P, int64_t B, int64_t max_batch,
                 void *out);

/* As egg_dp_batch with P and out in device memory, enqueued on `stream` (a cudaStream_t; NULL
 * for the library's own stream) without a host synchronisation. */
int egg_dp_batch_device(int K, int idx_bytes, int dtype, int prec, const void *P, int64_t B, void *out,
                        void *stream);

/* ---- Bjorklund/Glynn sieve --------------------------------------------------------------- */

/* The sieve of _calc_hafnian(Ax, edge_reps; glynn) (src/hafnian.jl:684-738) for one matrix:
 * Ax is the 2E x 2E matrix already permuted so row i pairs with row i+E (_permuted, :786-792),
 * edge_reps the E multiplicities from matched_reps (:142-188).  glynn selects the Glynn
 * (1) or inclusion-exclusion (0) variant.  FP64 per term, double-double accumulation of the
 * signed terms; out receives one value (EGG_F64 or EGG_C128).
 * prec: EGG_PREC_EXACT evaluates every term in the reference's loop order and rounding (each term
 * bit-identical to _glynn_term!, :528-602); EGG_PREC_FMA keeps each term's matrix in registers
 * and uses fused multiply-adds (terms agree to rounding; the fast path).
 * Replaces _calc_hafnian (src/hafnian.jl:684); the reference has no device sieve. */
int egg_sieve(int dtype, int prec, const void *Ax, int64_t E, const int64_t *edge_reps, int glynn, void *out);

/* Same, Ax and out in device memory (edge_reps on the host), enqueued on `stream`. */
int egg_sieve_device(int dtype, int prec, const void *Ax, int64_t E, const int64_t *edge_reps, int glynn,
                     void *out, void *stream);

/* The same sieve as egg_sieve_device, for callers that cannot let the library allocate device
 * memory: a process whose GPU memory is owned by another allocator (a framework that reserves the
 * device up front), or a loop that must not allocate once running.  Ax and out are the caller's
 * device buffers; the sieve's scratch (its instance tables and per-warp partial sums) lives in a
 * fixed 4 MiB array compiled into the library, present on every GPU that loads it until the
 * process exits.  Nothing is allocated or freed.  A sieve needing more scratch than that (edge
 * counts up to 32 fit on a 148-SM B200: the largest need is about 3.8 MB) is refused with
 * EGG_ERR_TOO_LARGE.  The first call on a device looks up the device addresses of the array and of
 * the library's binomial table (no upload and no stream work), so make it before any stream
 * capture.  The call runs on the calling thread's current device.  All calls share the array:
 * calls whose device work overlaps race on it.  There is no counterpart of this entry point in the
 * reference. */
int egg_sieve_device_noalloc(int dtype, int prec, const void *Ax, int64_t E, const int64_t *edge_reps, int glynn,
                             void *out, void *stream);

/* B independent sieves in one call (the batched form the reference lacks: hafnian_repeated
 * runs its batch as a CPU loop, src/hafnian.jl:1355-1358).  Instance b has E[b] <= Emax edges;
 * its permuted matrix is the leading 2E[b] x 2E[b] block of the 2Emax x 2Emax column-major
 * slab at Ax + b*(2Emax)^2 elements; its multiplicities are edge_reps[b*Emax .. b*Emax+E[b]-1];
 * glynn[b] picks its variant.  out receives B values. */
int egg_sieve_batch(int dtype, int prec, int64_t B, int64_t Emax, const void *Ax, const int64_t *E,
                    const int64_t *edge_reps, const int32_t *glynn, void *out);

/* Same, with the matrix slab Ax and out in device memory (E, edge_reps, glynn on the host),
 * enqueued on `stream`. */
int egg_sieve_batch_device(int dtype, int prec, int64_t B, int64_t Emax, const void *Ax, const int64_t *E,
                           const int64_t *edge_reps, const int32_t *glynn, void *out, void *stream);

/* B instances of hafnian_repeated(A_b, rpt_b; method = :sieve), each with its own matrix and
 * multiplicities, prepared on the device.  A_b is the d x d column-major matrix at mats + b *
 * mat_stride elements (mat_stride 0: one matrix shared by every instance), rpt_b the d entries at
 * rpts + b * d.  Per instance the device forms matched_reps(rpt_b) (src/hafnian.jl:142-188), the
 * sieve variant the reference's cost model picks (:855-884, :974-976; glynn = 0 or 1 forces one,
 * -1 takes the cost model's) and the permuted matrix A_b[x, x] (:786-792), then the batch runs as
 * egg_sieve_batch does; out receives B values.  A zero total gives 1 and an odd one 0.  Instances
 * that match into more than 32 edges, or whose total exceeds 126, are refused with
 * EGG_ERR_TOO_LARGE.  Host pointers.  No counterpart in the reference, whose
 * hafnian_repeated(A, rpts) takes one matrix and runs its batch as a CPU loop (:1317-1359). */
int egg_sieve_repeated_batch(int dtype, int prec, int64_t B, int64_t d, const void *mats, int64_t mat_stride,
                             const int64_t *rpts, int glynn, void *out);

/* Same, with mats, rpts and out in device memory, enqueued on `stream`.  The per-instance edge
 * counts, multiplicities and variants come back to the host, where the sieve's launches are
 * planned, so the call waits for the preparation kernel. */
int egg_sieve_repeated_batch_device(int dtype, int prec, int64_t B, int64_t d, const void *mats, int64_t mat_stride,
                                    const int64_t *rpts, int glynn, void *out, void *stream);

/* One sieve summed exactly as the reference sums it: every term in the reference's arithmetic
 * (as EGG_PREC_EXACT), then plain FP64 `+=` over `nchunks` equal chunks of the term range, each
 * in term order, and the chunk sums left to right, times 2^-(n-1) under Glynn
 * (_sieve_sum, src/hafnian.jl:713-738).  With nchunks = _sieve_chunks(work, steps, nthreads)
 * (src/hafnian.jl:646-647) the result is bit-identical to _calc_hafnian(Ax, edge_reps; nthreads,
 * glynn) run with that thread count.  Host pointers; the terms are kept on the device, so sieves
 * of more than 2^28 terms are refused with EGG_ERR_TOO_LARGE. */
int egg_sieve_reference_sum(int dtype, const void *Ax, int64_t E, const int64_t *edge_reps, int glynn, int64_t nchunks,
                            void *out);

/* ---- mixed-degree batches -------------------------------------------------------------- */

/* Hafnians of B principal submatrices of one parent: instance b is A[r, r] with
 * r = rows[offsets[b] .. offsets[b+1]), 0-based indices into the n x n column-major parent A
 * (dtype EGG_F64, EGG_C128, or EGG_I64 for exact Int128 results; repeated indices act as repeated
 * rows, as in hafnian_repeated).  Degrees may differ from instance to instance: the instances are
 * binned by degree, their pair vectors gathered on the device and each bin runs the subset DP of
 * its degree, so each result equals hafnian(A[r, r]; method = :dp) in the same precision mode.
 * Odd |r| gives 0 and empty r gives 1.  offsets has B + 1 entries, offsets[0] = 0; out receives
 * B values (EGG_I64: B Int128 values).  Row indices outside [0, n) are refused.
 * No counterpart in the reference, whose batch form takes one degree per call
 * (hafnian(As), src/hafnian.jl:1263-1301). */
int egg_dp_mix(int dtype, int prec, const void *A, int64_t n, int64_t B, const int64_t *offsets, const int32_t *rows,
               void *out);

/* Same, with A, rows and out in device memory (offsets on the host, where the binning runs),
 * enqueued on `stream`.  Row indices outside [0, n) are not read; those pairs are NaN (0 for
 * integers).  No counterpart in the reference. */
int egg_dp_mix_device(int dtype, int prec, const void *A, int64_t n, int64_t B, const int64_t *offsets, const int32_t *rows,
                      void *out, void *stream);

/* The engine of the two calls above.  0 (the default): a gather launch, one launch per level of
 * each group of each degree, and a scatter launch, recorded as one CUDA graph on a shape's second
 * call and replayed after that.  1: a mix whose degrees are all at most 32 (Float64, ComplexF64 or
 * Int64 parents, closed-form plans) runs as ONE cooperative kernel launch -- the gather, every
 * degree's levels in lockstep, the scatter -- with grid-wide barriers between phases; other mixes,
 * and calls made while the stream is being captured, use engine 0.  Both engines give identical
 * results; engine 0 is about 10 % faster on B200 (its level kernels are compiled per popcount).
 * Each barrier wait of engine 1 is bounded (2 s); a launch that gave up makes egg_dp_mix return
 * EGG_ERR_TIMEOUT, and for egg_dp_mix_device the next call of either returns it.  The setting is
 * process-wide.  EGG_ERR_ARGUMENT for another value.  No counterpart in the reference. */
int egg_dp_mix_set_engine(int engine);
int egg_dp_mix_engine(void);

/* A diagnostic of engine 1's grid barrier: every block of a cooperative grid on the library's device
 * passes three barriers that each expect `extra` (0..1024) more blocks than the grid has.  With
 * extra = 0 this is the normal barrier and returns EGG_OK; with extra > 0 the first wait runs out
 * after wait_ns (1 ms .. 2 s) and the call returns EGG_ERR_TIMEOUT, having ended every block.
 * *passes (may be null) receives the barriers passed, summed over blocks.  No counterpart in the
 * reference. */
int egg_selfcheck_barrier(int extra, int64_t wait_ns, int64_t *passes);

/* How the mixed-degree batch evaluates degree K in this dtype and precision mode, as chosen by
 * timing the candidates on the first batch that had more than one instance of that degree:
 * batched = 1 runs groups of `group` instances instance-fastest (one thread per state and
 * instance); batched = 0 runs `group` single-instance evaluations side by side.  Degrees up to 22
 * always run as one whole-instance launch per batch and are not tuned.  A choice is made per size
 * class of the degree's bin (fewer than 4, 16, 64, 256 instances, or more); this reports a pinned
 * choice, else the one last tuned in this process, else the file's for the largest class.  Choices
 * are kept in a JSON file per GPU model and SM count ($EGG_TUNE_CACHE, else
 * $XDG_CACHE_HOME/eggman_b200/mix_tuning.json or ~/.cache/eggman_b200/mix_tuning.json; an empty
 * $EGG_TUNE_CACHE turns the file off), which a process reads before its first batch, so a degree
 * tuned once for a size class is not timed again.  EGG_ERR_NO_PLAN if K has not been tuned yet.
 * No counterpart in the reference. */
int egg_dp_mix_tuning(int K, int dtype, int prec, int *batched, int64_t *group);

/* Pin the evaluation of degree K (> 22) for this dtype and mode, for batches of every size, instead
 * of timing candidates: for callers that tuned offline, and for tests that must cover both
 * evaluations.  Process-local.  Results do not depend on the choice.  No counterpart in the
 * reference. */
int egg_dp_mix_set_tuning(int K, int dtype, int prec, int batched, int64_t group);

#ifdef __cplusplus
}
#endif

#endif /* EGGMAN_B200_H */

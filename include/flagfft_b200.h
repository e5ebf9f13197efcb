/*
 * flagfft_b200.h -- entry points the B200 engine adds beside flagfft.h.
 *
 * None of these replaces a public entry point of the reference; each exposes
 * an internal reference behaviour as a C symbol (cited per function) or is an
 * engine extension with no reference counterpart (stated per function).
 */
#ifndef FLAGFFT_B200_H_
#define FLAGFFT_B200_H_

#include "flagfft.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Library version string, e.g. "flagfft-b200 0.1.0 sm_100a".  No reference
 * counterpart. */
FLAGFFT_API const char *flagfftB200Version(void);

/* Plan tree the planner builds for a 1-D complex transform of length n,
 * including the raw-support fallbacks, as JSON in the reference's plan-JSON
 * node shape.  Host only: touches no GPU.  is_double selects complex128;
 * smem_bytes is the per-block shared-memory limit the planner assumes
 * (0 = the B200 opt-in limit, 232448).  Writes at most buflen bytes including
 * the terminating NUL and returns the full JSON length, or -1 on an invalid
 * length / planner error.
 * Exposes PlanBuilder::build (reference src/plan/builder_context.cpp:42-48)
 * with the fallbacks of src/exec/c_api_plan.cpp:9-25,169-194 and the
 * serialiser of src/utils/plan_json.cpp:18-57. */
FLAGFFT_API int flagfftB200PlannerTree(int n, int is_double, long long smem_bytes, char *buf, int buflen);

/* Plan tree of a created plan as JSON (same shape as above); NULL for an
 * invalid or destroyed plan.  The string is owned by the plan.
 * Exposes the reference's plan serialiser (src/utils/plan_json.cpp:18-57). */
FLAGFFT_API const char *flagfftB200PlanJson(flagfftHandle plan);

/* Number of kernel launches one Exec of the plan issues in the given
 * direction (FLAGFFT_FORWARD / FLAGFFT_INVERSE), or -1.  No reference
 * counterpart. */
FLAGFFT_API int flagfftB200LaunchCount(flagfftHandle plan, int direction);

/* Batch plan over transforms of uneven lengths.  No counterpart in the
 * reference.
 *
 * counts[g] transforms of length lengths[g] for g < ngroups, packed group
 * after group: group g's transforms start at element sum_{h<g} counts[h] *
 * lengths[h] of the input and of the output, each transform contiguous.  type
 * is FLAGFFT_C2C or FLAGFFT_Z2Z; execute with flagfftExecC2C / flagfftExecZ2Z
 * (either direction; out-of-place, or in place when idata == odata).
 *
 * Every group is planned as flagfftPlan1d(lengths[g], type, counts[g]) would
 * be, but the passes of all groups run together: pass p of every group forms
 * one phase, and each phase is one persistent launch whose CTAs take work
 * items (tiles of transforms) from a device queue, longest first.  The
 * launches of an Exec are captured into a CUDA graph on the first Exec with a
 * given (idata, odata) pair and replayed afterwards (the plan keeps up to four
 * such bindings; FLAGFFT_BATCH_GRAPH=0 launches them directly).  Like other
 * plans, one batch plan must not run on two streams at once. */
FLAGFFT_API flagfftResult flagfftB200PlanBatch(flagfftHandle *plan, int ngroups, const int *lengths, const int *counts,
                                              flagfftType type);

/* Autotuner: times the planner's alternative trees for a C2C / Z2Z request
 * (batch transforms of length n, one direction) on the current device, and
 * writes the fastest into the tune database as a valid rank-0 row of the
 * reference's table `tuned_measurements` (db_path, or the path plan creation
 * reads: $FLAGFFT_TUNE_DB, else <executable dir>/.flagfft/tuned_plans.sqlite),
 * so later plans of that length, batch bucket, dtype and direction use it.
 * The reference declares this step (flagfft-cli tune) but writes nothing
 * (src/cli_tools/tune/tune.cpp:7-9); its lookup side is
 * src/utils/plan_json.cpp:163-207.  Candidates: the default tree, other
 * orders of its leaf radices, the four most balanced four-step splits, and
 * Bluestein / Rader for primes.  `report` (buflen bytes) receives JSON with
 * every candidate's time; *best_ms the fastest time per Exec. */
FLAGFFT_API flagfftResult flagfftB200Tune(int n, flagfftType type, int batch, int direction, const char *db_path,
                                         char *report, int buflen, double *best_ms);
/* The autotuner's candidate trees for a length, as a JSON array (host only).
 * Returns the full length, or -1. */
FLAGFFT_API int flagfftB200TuneCandidates(int n, int is_double, char *buf, int buflen);

/* Request server: continuous batching of transforms of mixed type, length
 * and batch count.  No counterpart in the reference.
 *
 * A server owns a scheduler thread.  Submit queues a request (batch
 * transforms of length n of any flagfftType, direction for C2C / Z2Z; input
 * and output are device buffers laid out as flagfftPlan1d(n, type, batch)
 * would read and write them) and returns at once with a ticket.  The
 * scheduler admits queued requests in arrival order whenever one of
 * `max_ticks` tick slots is free and the HBM budget allows (a request is
 * charged its input, output and workspace bytes; workspaces come from the
 * stream-ordered memory pool and return to it), and runs each tick's requests
 * together as persistent work-queue launches on the slot's stream, so ticks
 * overlap on the device.  A request's result does not depend on which
 * requests share its tick.  Programs and tables of every (type, n,
 * direction) seen stay resident; Prepare builds one ahead of the first
 * request and runs one transform of it on scratch buffers it allocates, so
 * the kernels the template takes are loaded before requests arrive.  Wait blocks until the request finished and gives its latency
 * from Submit to completion as seen by the scheduler (the caller's buffers
 * may then be reused).  Submit from any thread; a request larger than the
 * budget returns FLAGFFT_INVALID_SIZE. */
typedef struct flagfftB200Server_st *flagfftB200Server;
FLAGFFT_API flagfftResult flagfftB200ServerCreate(flagfftB200Server *srv, long long hbm_budget_bytes, int max_ticks);
FLAGFFT_API flagfftResult flagfftB200ServerPrepare(flagfftB200Server srv, flagfftType type, int n, int direction);
FLAGFFT_API flagfftResult flagfftB200ServerSubmit(flagfftB200Server srv, flagfftType type, int n, int batch,
                                                 int direction, const void *idata, void *odata, long long *ticket);
FLAGFFT_API flagfftResult flagfftB200ServerWait(flagfftB200Server srv, long long ticket, double *latency_ms);
FLAGFFT_API flagfftResult flagfftB200ServerStats(flagfftB200Server srv, long long *completed, long long *ticks,
                                                long long *bytes_in_use);
/* ServerWait with a bound: waits at most timeout_ms.  *done = 1 and the
 * latency as ServerWait when the request finished (the ticket is then
 * released); *done = 0 and FLAGFFT_SUCCESS when it has not finished yet (the
 * ticket stays valid for a later wait).  No reference counterpart. */
FLAGFFT_API flagfftResult flagfftB200ServerWaitFor(flagfftB200Server srv, long long ticket, double timeout_ms,
                                                  double *latency_ms, int *done);
/* Continuous-batching counters: the most ticks the server has had in flight
 * at once, and how many requests it admitted while another tick was still on
 * the GPU.  No reference counterpart. */
FLAGFFT_API flagfftResult flagfftB200ServerOverlap(flagfftB200Server srv, long long *max_ticks_in_flight,
                                                 long long *admitted_while_busy);
FLAGFFT_API flagfftResult flagfftB200ServerDestroy(flagfftB200Server srv);

/* Number of bounded device-side waits that gave up on the current device
 * since the library was loaded: a persistent kernel waits for its own tile
 * copies (TMA) for at most about a second, then records the failure here and
 * ends instead of hanging.  0 in normal operation.  No reference
 * counterpart. */
FLAGFFT_API flagfftResult flagfftB200DeviceWaitFailures(long long *count);

/* Precision-mode prototype: batched complex64 transforms of n = 256 or 4096
 * points whose radix-16 stages run as dense 16-point DFT-matrix products on
 * the tcgen05 tensor cores, split-bf16 operands (terms = 3: the three
 * products of a two-way split; terms = 6: a three-way split, every product
 * down to 2^-24) with fp32 accumulation in tensor memory.  Measurement entry
 * point for the decision whether this mode ships; the plan path does not use
 * it.  No reference counterpart.  idata / odata: batch contiguous rows of n
 * flagfftComplex on the device; direction FLAGFFT_FORWARD / FLAGFFT_INVERSE.
 * Returns FLAGFFT_NOT_SUPPORTED for other n or terms. */
FLAGFFT_API flagfftResult flagfftB200PrecisionC2C(const flagfftComplex *idata, flagfftComplex *odata, int n,
                                                 int batch, int direction, int terms, flagfftStream_t stream);
/* Bounded waits of the precision-mode kernel that gave up on this device. */
FLAGFFT_API flagfftResult flagfftB200PrecisionWaitFailures(long long *count);

/* Batched complex64 FFT of power-of-two length n (8192 <= n <= 2^22) that
 * allocates no memory.  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc when they transform: code running
 * under a memory pool or allocator that must not grow, inside a region that
 * forbids device allocation, or with no spare memory left to carve a plan
 * workspace from.  Transforms of this size need an intermediate buffer of
 * batch * n elements; here it is a fixed 32 MiB array built into the library
 * (every GPU that loads the library holds it until the process exits), so
 * batch * n may not exceed 2^22 elements.  Larger requests return
 * FLAGFFT_INVALID_SIZE with a message on stderr; the entry point never calls
 * cudaMalloc, cudaFree or an allocating library routine.
 *
 * idata / odata are device pointers to batch contiguous rows of n
 * flagfftComplex (odata may equal idata); direction is FLAGFFT_FORWARD or
 * FLAGFFT_INVERSE (unnormalized); work is queued on `stream`.
 *
 * The first call on a device looks up the fixed arrays' device addresses and
 * fills a twiddle table with the device current, then waits for that fill:
 * make the first call on each device before any stream capture.  Every call
 * shares the one workspace and rewrites its twiddle tables, so calls whose
 * work overlaps on the GPU race with each other: serialise them (one stream,
 * or events).  Nothing in the arrays has to start at zero: each call writes
 * every workspace and table element it reads before reading it. */
FLAGFFT_API flagfftResult flagfftB200ExecC2CNoAlloc(const flagfftComplex *idata, flagfftComplex *odata, int n,
                                                    int batch, int direction, flagfftStream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* FLAGFFT_B200_H_ */

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

#ifdef __cplusplus
}
#endif

#endif /* FLAGFFT_B200_H_ */

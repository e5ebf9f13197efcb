/*
 * flagfft.h -- the C ABI of the B200 FFT engine.
 *
 * Drop-in for the reference FlagFFT C API: every declaration below keeps the
 * name, argument meaning, enum value and status behaviour of the reference's
 * include/flagfft.h (the entry points of include/flagfft.h:53-82, the status
 * codes of :10-26, the cuFFT-valued type codes of :28-35, the complex structs
 * of :40-48).  Implemented in flagfft_b200/csrc/api.cpp.
 *
 *   flagfftPlan1d / Plan2d / Plan3d / PlanMany
 *       replace include/flagfft.h:55-68 (src/exec/c_api_plan.cpp:249-336)
 *   flagfftExecC2C / Z2Z / R2C / D2Z / C2R / Z2D
 *       replace include/flagfft.h:70-78 (src/exec/c_api_exec.cpp:5-167)
 *   flagfftSetStream / flagfftDestroy / flagfftGetPlanDescription
 *       replace include/flagfft.h:80-82 (src/exec/c_api_exec.cpp:169-236)
 *
 * Data pointers are device pointers (in-place when idata == odata).  Exec is
 * asynchronous on the plan's stream (a cudaStream_t / CUstream, default the
 * legacy null stream).  The inverse transform is unnormalized.
 */
#ifndef FLAGFFT_H_
#define FLAGFFT_H_

#ifdef __cplusplus
extern "C" {
#endif

/* Exported from libflagfft.so (built with hidden default visibility). */
#if defined(__GNUC__)
#define FLAGFFT_API __attribute__((visibility("default")))
#else
#define FLAGFFT_API
#endif

typedef void *flagfftStream_t;

typedef enum flagfftResult_t {
  FLAGFFT_SUCCESS = 0,
  FLAGFFT_INVALID_PLAN = 1,
  FLAGFFT_ALLOC_FAILED = 2,
  FLAGFFT_INVALID_TYPE = 3,
  FLAGFFT_INVALID_VALUE = 4,
  FLAGFFT_INTERNAL_ERROR = 5,
  FLAGFFT_EXEC_FAILED = 6,
  FLAGFFT_SETUP_FAILED = 7,
  FLAGFFT_INVALID_SIZE = 8,
  FLAGFFT_UNALIGNED_DATA = 9,
  FLAGFFT_INCOMPLETE_PARAMETER_LIST = 10,
  FLAGFFT_INVALID_DEVICE = 11,
  FLAGFFT_PARSE_ERROR = 12,
  FLAGFFT_NO_WORKSPACE = 13,
  FLAGFFT_NOT_SUPPORTED = 14
} flagfftResult;

typedef enum flagfftType_t {
  FLAGFFT_R2C = 0x2a,
  FLAGFFT_C2R = 0x2c,
  FLAGFFT_C2C = 0x29,
  FLAGFFT_D2Z = 0x6a,
  FLAGFFT_Z2D = 0x6c,
  FLAGFFT_Z2Z = 0x69
} flagfftType;

#define FLAGFFT_FORWARD (-1)
#define FLAGFFT_INVERSE 1

typedef struct flagfftComplex_t {
  float x;
  float y;
} flagfftComplex;

typedef struct flagfftDoubleComplex_t {
  double x;
  double y;
} flagfftDoubleComplex;

typedef float flagfftReal;
typedef double flagfftDoubleReal;

typedef struct flagfftPlan_t *flagfftHandle;

FLAGFFT_API flagfftResult flagfftPlan1d(flagfftHandle *plan, int nx, flagfftType type, int batch);
FLAGFFT_API flagfftResult flagfftPlan2d(flagfftHandle *plan, int nx, int ny, flagfftType type);
FLAGFFT_API flagfftResult flagfftPlan3d(flagfftHandle *plan, int nx, int ny, int nz, flagfftType type);
FLAGFFT_API flagfftResult flagfftPlanMany(flagfftHandle *plan, int rank, int *n, int *inembed, int istride, int idist,
                              int *onembed, int ostride, int odist, flagfftType type, int batch);

FLAGFFT_API flagfftResult flagfftExecC2C(flagfftHandle plan, flagfftComplex *idata, flagfftComplex *odata, int direction);
FLAGFFT_API flagfftResult flagfftExecZ2Z(flagfftHandle plan, flagfftDoubleComplex *idata, flagfftDoubleComplex *odata,
                             int direction);
FLAGFFT_API flagfftResult flagfftExecR2C(flagfftHandle plan, flagfftReal *idata, flagfftComplex *odata);
FLAGFFT_API flagfftResult flagfftExecD2Z(flagfftHandle plan, flagfftDoubleReal *idata, flagfftDoubleComplex *odata);
FLAGFFT_API flagfftResult flagfftExecC2R(flagfftHandle plan, flagfftComplex *idata, flagfftReal *odata);
FLAGFFT_API flagfftResult flagfftExecZ2D(flagfftHandle plan, flagfftDoubleComplex *idata, flagfftDoubleReal *odata);

FLAGFFT_API flagfftResult flagfftSetStream(flagfftHandle plan, flagfftStream_t stream);
FLAGFFT_API flagfftResult flagfftDestroy(flagfftHandle plan);
FLAGFFT_API const char *flagfftGetPlanDescription(flagfftHandle plan);

#ifdef __cplusplus
}
#endif

#endif /* FLAGFFT_H_ */

/* Force-included when compiling the reference's own kernels
 * (cuFPM_v3/cuda/kernels.cuh) outside MATLAB: the two MATLAB element types
 * those kernels use, as MATLAB's tmwtypes.h defines them.  TEST INFRASTRUCTURE:
 * only the oracle harness (oracle/ref_harness.cu) is built with it. */
#ifndef FPM_REF_SHIM_H
#define FPM_REF_SHIM_H
typedef float real32_T;
typedef struct { real32_T re, im; } creal32_T;
#endif

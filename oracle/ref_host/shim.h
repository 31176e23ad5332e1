// Pre-include for compiling the reference's host-callable render code here.
// It changes no reference file: it only works around MSVC-isms so that nvcc
// on Linux accepts the sources in place.
//  * 'inline __forceinline__' and '__inline__ inline' (duplicate inline
//    specifiers, rejected by nvcc's front end): __forceinline__ and
//    __inline__ become empty after every system header is included, and the
//    whole reference is built as one translation unit (ref_driver.cu), so no
//    header function is defined twice.
//  * two templates that PrefixScanSum.cuh calls before defining them
//    (MSVC's lookup accepts it, two-phase lookup does not) are declared.
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <map>
#include <vector>
#include <string>
#include <random>
#include <chrono>
#include <unordered_set>
#include <sstream>
#include <fstream>
#include <algorithm>
#include <cuda_runtime.h>
#include <curand_kernel.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <math_constants.h>
#undef __forceinline__
#define __forceinline__
#undef __inline__
#define __inline__
#include "Defines.cuh"
template <typename T> __device__ void prescan_full_threads(T* out_arr, T* in_data, T* sums, idxtype n, bool inclusive);
template <typename T> __device__ void prescan_arbitrary(T* out_arr, T* in_arr, idxtype length, int powerOfTwo);

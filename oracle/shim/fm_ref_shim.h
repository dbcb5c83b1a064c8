/*
 * Host shim for the reference's CUDA kernel bodies (test infrastructure only).
 *
 * The recipe in oracle/build_oracle.py pipes the kernel part of each reference
 * .cu file (everything before its class glue, which uses <<<>>> launches) into
 * g++ with this header force-included.  The execution-space keywords become
 * plain C++, `blockIdx/blockDim/threadIdx` become thread-local structs that the
 * host driver (oracle/ref_driver.cpp) sets before calling a kernel once per
 * "thread", and cudaMemcpyToSymbol becomes a memcpy into the host copy of the
 * __constant__ table, so the reference's own upload functions
 * (src/core/D3Q19Constants.cu:24-31, src/core/D3Q7Constants.cu:24-31) fill the
 * tables the kernels read.
 *
 * Nothing here is product code: only tests/, the smoke check and bench.py's CPU
 * baseline load the library built from it.
 */
#pragma once

#include <cuda_runtime.h>
#include <cstring>

#undef __global__
#undef __device__
#undef __host__
#undef __constant__
#undef __forceinline__
#define __global__
#define __device__
#define __host__
#define __constant__
/* internal linkage: idx3/mapCoord are defined again in several kernel files */
#define __forceinline__ static inline

struct fm_shim_dim3 { unsigned x, y, z; };
extern thread_local fm_shim_dim3 fm_shim_blockIdx;
extern thread_local fm_shim_dim3 fm_shim_blockDim;
extern thread_local fm_shim_dim3 fm_shim_threadIdx;
#define blockIdx  fm_shim_blockIdx
#define blockDim  fm_shim_blockDim
#define threadIdx fm_shim_threadIdx

/* the kernels' `max` helper is only used in class glue, which is cut off */

#define cudaMemcpyToSymbol(sym, src, nbytes) \
    (std::memcpy(static_cast<void*>(&(sym)), (src), (nbytes)), cudaSuccess)

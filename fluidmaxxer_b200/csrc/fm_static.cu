// fm_static.cu -- the allocation-free domain reduction (fm_reduce_static).
//
// Some callers of this library cannot call cudaMalloc: a host application that
// reserved all of its device memory up front in its own pool, or code that
// runs where an allocation would stall the device or break an asynchronous
// pipeline (cudaMalloc may synchronise the device).  fm_reduce_static serves
// them: it sums the same quantities as fm_reduce over buffers the caller
// passes in, and keeps its intermediate sums in a fixed, statically allocated
// device array instead of allocating anything.
#include "../../include/fm.h"

#include <cuda_runtime.h>

#include <mutex>
#include <string>

namespace {

// First pass: one block per kStaticCellsPerBlock cells writes one partial
// (sum rho, sum phi, sum q, unused).  Second pass: one block sums the
// partials in a fixed order into the last slot.
constexpr int kStaticMaxPartials = 4096;
constexpr int kStaticCellsPerBlock = 32768;
constexpr long long kStaticMaxCells = (long long)kStaticMaxPartials * kStaticCellsPerBlock;  // 134,217,728
constexpr int kStaticBlock = 256;
constexpr int kMaxDevices = 64;

// The scratch: (kStaticMaxPartials + 1) slots of 4 doubles = 128 KiB on every
// device that loads this library, held until the process exits.  In host code
// this name is only a host-side stand-in; kernels get its device address from
// cudaGetSymbolAddress.
static __device__ __align__(256) double fm_static_scratch[(kStaticMaxPartials + 1) * 4];

std::mutex g_setup_mutex;
double* g_scratch_addr[kMaxDevices] = {};
void* g_scratch_ctx[kMaxDevices] = {};   // the context each cached address belongs to

}  // namespace

// records the message behind fm_last_error(), and the current context's
// handle (both defined in fm_abi.cu)
namespace fm_internal {
int set_error(int code, const std::string& msg);
void* current_context();
}

namespace {

int static_fail(int code, const std::string& msg) { return fm_internal::set_error(code, msg); }

// Device address of the scratch array for the current device, looked up with
// that device current and cached per device.  The cache is keyed on the
// device's context as well: after cudaDeviceReset the runtime loads this
// module again in a new context, where the array may sit at another address,
// so a changed context triggers a fresh lookup.
int scratch_for_current_device(double** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return static_fail(FM_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return static_fail(FM_ERR_UNSUPPORTED, "device ordinal beyond 63");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    void* ctx = fm_internal::current_context();
    if (!g_scratch_addr[dev] || !ctx || ctx != g_scratch_ctx[dev]) {
        // with no context current yet, the lookup makes the device's primary
        // context current; the context is read again after it
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, fm_static_scratch);
        if (e != cudaSuccess || !p)
            return static_fail(FM_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_scratch_addr[dev] = static_cast<double*>(p);
        g_scratch_ctx[dev] = fm_internal::current_context();
    }
    *out = g_scratch_addr[dev];
    return FM_OK;
}

__device__ __forceinline__ double warp_sum_d(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block sum of three doubles in a fixed order (shuffle tree, then warp 0).
__device__ __forceinline__ void block_sum3(double (&v)[3], double* __restrict__ dst)
{
    __shared__ double part[kStaticBlock / 32][3];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < 3; ++j) v[j] = warp_sum_d(v[j]);
    if (lane == 0) {
#pragma unroll
        for (int j = 0; j < 3; ++j) part[wid][j] = v[j];
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double s = lane < kStaticBlock / 32 ? part[lane][j] : 0.0;
            s = warp_sum_d(s);
            if (lane == 0) dst[j] = s;
        }
    }
}

// Pass 1: block b sums rho (the FP32 sum of the 19 populations of a cell, as
// k_domain_sums forms it), phi and q over its cell range into scratch slot b.
__global__ void __launch_bounds__(kStaticBlock) k_static_partials(const float* __restrict__ f,
                                                                  const float* __restrict__ phi,
                                                                  const float* __restrict__ q, long long ns,
                                                                  long long n, double* __restrict__ scratch)
{
    const long long c0 = (long long)blockIdx.x * kStaticCellsPerBlock;
    const long long c1 = c0 + kStaticCellsPerBlock < n ? c0 + kStaticCellsPerBlock : n;
    double v[3] = {0.0, 0.0, 0.0};
    for (long long c = c0 + threadIdx.x; c < c1; c += kStaticBlock) {
        float r = 0.0f;
#pragma unroll
        for (int k = 0; k < 19; ++k) r += __ldg(f + (long long)k * ns + c);
        v[0] += (double)r;
        v[1] += (double)__ldg(phi + c);
        v[2] += (double)__ldg(q + c);
    }
    block_sum3(v, scratch + 4 * (long long)blockIdx.x);
}

// Pass 2: one block sums the `count` partials into the final slot.
__global__ void __launch_bounds__(kStaticBlock) k_static_final(double* __restrict__ scratch, int count)
{
    double v[3] = {0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < count; b += kStaticBlock) {
#pragma unroll
        for (int j = 0; j < 3; ++j) v[j] += scratch[4 * b + j];
    }
    block_sum3(v, scratch + 4 * kStaticMaxPartials);
}

}  // namespace

extern "C" int fm_reduce_static(const float* d_f, const float* d_phi, const float* d_q, long long plane_stride,
                                long long n_cells, double out[3], void* stream)
{
    if (!out) return static_fail(FM_ERR_ARG, "fm_reduce_static: null output");
    if (n_cells < 0) return static_fail(FM_ERR_ARG, "fm_reduce_static: negative cell count");
    if (n_cells > kStaticMaxCells)
        return static_fail(FM_ERR_ARG, "fm_reduce_static: n_cells exceeds the static scratch limit of "
                                       "134217728 cells");
    if (plane_stride < n_cells) return static_fail(FM_ERR_ARG, "fm_reduce_static: plane_stride < n_cells");
    if (n_cells == 0) {
        out[0] = out[1] = out[2] = 0.0;
        return FM_OK;
    }
    if (!d_f || !d_phi || !d_q) return static_fail(FM_ERR_ARG, "fm_reduce_static: null device pointer");
    double* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const int blocks = (int)((n_cells + kStaticCellsPerBlock - 1) / kStaticCellsPerBlock);
    // every slot the final pass reads is written by this call's first pass,
    // so nothing left from an earlier call is read
    k_static_partials<<<blocks, kStaticBlock, 0, st>>>(d_f, d_phi, d_q, plane_stride, n_cells, scratch);
    k_static_final<<<1, kStaticBlock, 0, st>>>(scratch, blocks);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, scratch + 4 * kStaticMaxPartials, 3 * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return static_fail(FM_ERR_CUDA, std::string("fm_reduce_static: ") + cudaGetErrorString(e));
    return FM_OK;
}

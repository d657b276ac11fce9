// Shared helpers of the B200 IB/MG kernels: error reporting, dtype dispatch,
// exact-order arithmetic and deterministic reductions.
//
// The library is compiled with --fmad=false so that every a*b+c written in
// source rounds twice, as in the reference CPU/Triton arithmetic; kernels
// that want a fused multiply-add say so with fma().
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include "afsi_b200.h"

namespace afsi {

int32_t fail(int32_t code, const char* fmt, ...);
int32_t launched(const char* what);  // AFSI_OK or AFSI_ERR_CUDA after a launch

inline unsigned blocks_for(int64_t n, int threads) {
    return static_cast<unsigned>((n + threads - 1) / threads);
}

template <class T> struct Const;
template <> struct Const<float> { static constexpr int code = AFSI_F32; };
template <> struct Const<double> { static constexpr int code = AFSI_F64; };

__device__ __forceinline__ void flag(int32_t* status, int32_t bit) {
    if (status) atomicOr(status, bit);
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int d = 16; d; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
    return v;
}

// Block-wide deterministic sum of one double per thread (result valid in
// thread 0).  `shared` holds one double per warp.
__device__ __forceinline__ double block_sum(double v, double* shared) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    if (lane == 0) shared[warp] = v;
    __syncthreads();
    const int warps = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < warps) ? shared[threadIdx.x] : 0.0;
    if (warp == 0) v = warp_sum(v);
    __syncthreads();
    return v;
}

// Last-block completion of a grid reduction.  Every block stores its partial
// in partial[blockIdx.x]; the block that arrives last (ticket == gridDim.x-1)
// sums the partials in index order, so the result does not depend on block
// scheduling.  The counter is reset by that block for the next launch.
struct GridReduce {
    double* partial;        // gridDim.x * width doubles
    unsigned int* counter;  // one per reduction site, zero between launches
};

// Returns true in every thread of the last block after all partials are visible.
__device__ __forceinline__ bool grid_reduce_arrive(unsigned int* counter, bool* is_last_smem) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int ticket = atomicAdd(counter, 1u);
        *is_last_smem = (ticket == gridDim.x - 1);
    }
    __syncthreads();
    bool last = *is_last_smem;
    if (last) __threadfence();
    return last;
}

// Sum partial[0..count) (stride `stride`, offset `k`) deterministically in the
// calling block; result in thread 0.
__device__ __forceinline__ double sum_partials(const double* partial, int count, int stride, int k,
                                               double* shared) {
    double v = 0.0;
    // fixed assignment: thread t sums t, t+blockDim, ... in order
    for (int i = threadIdx.x; i < count; i += blockDim.x) v += __ldcg(partial + i * stride + k);
    return block_sum(v, shared);
}

// Programmatic dependent launch (sm_90+): let the next kernel in the stream
// begin launching now, then wait until every kernel this one depends on has
// completed and its writes are visible.  The next kernel is launched only
// after every block of this one has started, so waiting blocks never hold back
// a kernel they depend on.  Both are no-ops for a launch without the
// programmatic-serialization attribute.
// 1/v when v is a positive normal power of two whose reciprocal is normal
// (then x * (1/v) rounds exactly as x / v), else 0.
template <class T>
__device__ __forceinline__ T exact_reciprocal(T v) {
    if constexpr (sizeof(T) == 8) {
        const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(double(v)));
        const unsigned e = unsigned(b >> 52) & 0x7FFu;
        return ((b & 0x800FFFFFFFFFFFFFull) == 0 && e > 0 && e <= 0x7FDu) ? T(1) / v : T(0);
    } else {
        const unsigned b = __float_as_uint(float(v));
        const unsigned e = (b >> 23) & 0xFFu;
        return ((b & 0x807FFFFFu) == 0 && e > 0 && e <= 0xFDu) ? T(1) / v : T(0);
    }
}

__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Launch with programmatic stream serialisation: the kernel may begin
// launching while its predecessor in the stream runs (both sides call
// pdl_enter).  Captured graphs keep this as a programmatic edge.
template <class... Params, class... Args>
int32_t launch_pdl(const char* what, void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem,
                   cudaStream_t stream, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr.val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    const cudaError_t err = cudaLaunchKernelEx(&cfg, kernel, static_cast<Params>(args)...);
    if (err != cudaSuccess) return fail(AFSI_ERR_CUDA, "%s: %s", what, cudaGetErrorString(err));
    return launched(what);
}

}  // namespace afsi

#define AFSI_DISPATCH(dtype, ...)                                              \
    switch (dtype) {                                                           \
    case AFSI_F32: { using T = float; __VA_ARGS__; } break;                    \
    case AFSI_F64: { using T = double; __VA_ARGS__; } break;                   \
    default: return ::afsi::fail(AFSI_ERR_ARG, "unsupported dtype code %d", (int)(dtype)); \
    }

#define AFSI_REQUIRE(cond, ...) \
    do { if (!(cond)) return ::afsi::fail(AFSI_ERR_ARG, __VA_ARGS__); } while (0)

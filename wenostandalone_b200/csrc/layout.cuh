// layout.cuh -- reshape (s_initialize_weno_{x,y,z}, f90:281-330) and order-1
// copy (s_order1_copy_{x,y,z}, f90:332-390) as bandwidth kernels.
//
// Both are index permutations of v_vf.  The x direction keeps the fastest
// axis, so it is a row copy; y and z swap the fastest axis with a strided
// one, done as a 32x32 shared-memory tile transpose so that both the loads
// and the stores are coalesced (the reference's y/z loops over-read HBM
// 3.9x / 7.3x because one side of the copy is strided).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace wsb {

template <typename T>
__device__ __forceinline__ T cvt(double x) { return (T)x; }

// Row copy: out row r (length A, rows contiguous) <- in row (b, p, v).
// Row r = b + B*(p + P*v).  Up to two outputs.
struct RowCopyArgs {
    const double* in;
    long long A, B, P, V;
    long long iB, iP, iV;  // input row strides
};

template <typename T, int NOUT>
__global__ void __launch_bounds__(256) row_copy_kernel(RowCopyArgs g, T* __restrict__ out0,
                                                       T* __restrict__ out1) {
    const long long rows = g.B * g.P * g.V;
    const int lane = threadIdx.x;
    for (long long r = (long long)blockIdx.x * blockDim.y + threadIdx.y; r < rows;
         r += (long long)gridDim.x * blockDim.y) {
        const long long b = r % g.B;
        const long long t = r / g.B;
        const long long p = t % g.P;
        const long long v = t / g.P;
        const double* __restrict__ src = g.in + b * g.iB + p * g.iP + v * g.iV;
        T* __restrict__ d0 = out0 + r * g.A;
        T* __restrict__ d1 = (NOUT > 1) ? out1 + r * g.A : nullptr;
        for (long long a = lane; a < g.A; a += blockDim.x) {
            const T x = cvt<T>(__ldg(src + a));
            d0[a] = x;
            if (NOUT > 1) d1[a] = x;
        }
    }
}

// Tiled transpose: out[a + oB*b + oP*p + oV*v] = in[iA*a + b + iP*p + iV*v]
// for a < A (output-contiguous axis, strided in the input) and b < B
// (input-contiguous axis).  grid = (ceil(A/32), ceil(B/32), P*V chunks).
struct TransposeArgs {
    const double* in;
    long long A, B, P, V;
    long long iA, iP, iV;
    long long oB, oP, oV;
};

template <typename T, int NOUT>
__global__ void __launch_bounds__(256) transpose_kernel(TransposeArgs g, T* __restrict__ out0,
                                                        T* __restrict__ out1) {
    __shared__ double tile[32][33];
    const long long a0 = (long long)blockIdx.x * 32;
    const long long b0 = (long long)blockIdx.y * 32;
    const long long planes = g.P * g.V;
    for (long long pl = blockIdx.z; pl < planes; pl += gridDim.z) {
        const long long p = pl % g.P;
        const long long v = pl / g.P;
        const double* __restrict__ src = g.in + p * g.iP + v * g.iV;
        // load: threadIdx.x runs along b (contiguous in the input)
#pragma unroll
        for (int k = 0; k < 32; k += 8) {
            const long long a = a0 + threadIdx.y + k;
            const long long b = b0 + threadIdx.x;
            if (a < g.A && b < g.B) tile[threadIdx.y + k][threadIdx.x] = __ldg(src + a * g.iA + b);
        }
        __syncthreads();
        // store: threadIdx.x runs along a (contiguous in the output)
        const long long obase = p * g.oP + v * g.oV;
#pragma unroll
        for (int k = 0; k < 32; k += 8) {
            const long long b = b0 + threadIdx.y + k;
            const long long a = a0 + threadIdx.x;
            if (a < g.A && b < g.B) {
                const T x = cvt<T>(tile[threadIdx.x][threadIdx.y + k]);
                out0[obase + a + g.oB * b] = x;
                if (NOUT > 1) out1[obase + a + g.oB * b] = x;
            }
        }
        __syncthreads();
    }
}

// Device-side sum(|x|) (f_checksum, f90:1617-1620): fixed grid, so the
// summation order, and hence the rounding, is the same on every call.
constexpr int kSumBlocks = 592;  // 4 x 148 SMs
constexpr int kSumThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kSumThreads) abs_sum_partial_kernel(const T* __restrict__ a,
                                                                      long long n,
                                                                      double* __restrict__ partial) {
    __shared__ double red[kSumThreads / 32];
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        s += fabs((double)a[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = (threadIdx.x < kSumThreads / 32) ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) partial[blockIdx.x] = s;
    }
}

__global__ void __launch_bounds__(kSumThreads) abs_sum_final_kernel(const double* __restrict__ partial,
                                                                    int np, double* __restrict__ out) {
    __shared__ double red[kSumThreads / 32];
    double s = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) s += partial[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = (threadIdx.x < kSumThreads / 32) ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) *out = s;
    }
}

// FP64 -> FP32 / FP32 -> FP64 element conversion (FP32-bulk handle I/O).
__global__ void f64_to_f32_kernel(const double* __restrict__ a, float* __restrict__ b, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

}  // namespace wsb

// Shared helpers for the oskar_b200 CUDA sources (sm_100a only).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "oskar_b200.h"

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ < 1000)
#error "oskar_b200 is built for sm_100a only"
#endif

namespace oskb {

// Last CUDA error text, kept per thread for oskb_last_error().
void set_last_error(const char* where, cudaError_t err);
void set_last_error_msg(const char* msg);

// Maps a CUDA error after a launch to the OSKAR status convention.
inline int check_launch(const char* where)
{
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess)
    {
        set_last_error(where, err);
        return OSKB_ERR_KERNEL_LAUNCH_FAILURE;
    }
    return 0;
}

inline cudaStream_t as_stream(void* s) { return (cudaStream_t) s; }

// Current device (-1 if none) and its SM count, cached per device
// (scratch.cu); safe to call from several host threads.
int current_device();
int device_sm_count();

// Stream-ordered temporaries from the library's own memory pool, which
// keeps freed blocks across host synchronisations (scratch.cu).
cudaError_t scratch_alloc(void** ptr, size_t bytes, cudaStream_t stream);
cudaError_t scratch_free(void* ptr, cudaStream_t stream);

template <typename T> struct vec2;
template <> struct vec2<float> { typedef float2 type; };
template <> struct vec2<double> { typedef double2 type; };

// 2x2 complex matrix {a, b, c, d}, row-major: [[a, b], [c, d]].
template <typename T> struct Mat2
{
    typename vec2<T>::type a, b, c, d;
};

template <typename T>
__device__ __forceinline__ typename vec2<T>::type cmul(
        typename vec2<T>::type x, typename vec2<T>::type y)
{
    typename vec2<T>::type r;
    r.x = x.x * y.x - x.y * y.y;
    r.y = x.x * y.y + x.y * y.x;
    return r;
}

// Load/store of a 2x2 complex matrix with 16-byte (FP64) or 16-byte
// vector (FP32, two matrices elements per load) accesses.
__device__ __forceinline__ Mat2<double> load_mat(const double* p)
{
    const double2* q = reinterpret_cast<const double2*>(p);
    Mat2<double> m;
    m.a = __ldg(q); m.b = __ldg(q + 1); m.c = __ldg(q + 2); m.d = __ldg(q + 3);
    return m;
}

__device__ __forceinline__ Mat2<float> load_mat(const float* p)
{
    const float4* q = reinterpret_cast<const float4*>(p);
    const float4 u = __ldg(q), v = __ldg(q + 1);
    Mat2<float> m;
    m.a = make_float2(u.x, u.y); m.b = make_float2(u.z, u.w);
    m.c = make_float2(v.x, v.y); m.d = make_float2(v.z, v.w);
    return m;
}

// Baseline index of stations q < p (reference:
// oskar/correlate/define_correlate_utils.h:42).
__host__ __device__ __forceinline__ long long baseline_index(int n, int p,
        int q)
{
    return (long long) q * (n - 1) - (long long) (q - 1) * q / 2 + p - q - 1;
}

constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double kOmegaEarth = 7.272205217e-5;  // rad/s, as the reference

}  // namespace oskb

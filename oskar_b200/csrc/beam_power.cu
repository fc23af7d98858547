// Beam-pattern power terms: auto power J B J^H per station-direction and
// cross power, the average over station pairs p < q of (J_p B) J_q^H per
// direction.
//
// Replace the kernels behind oskar_evaluate_auto_power and
// oskar_evaluate_cross_power (oskar/correlate/src/
// oskar_evaluate_{auto,cross}_power.c; define_evaluate_auto_power.h:3-40,
// define_evaluate_cross_power.h:3-72). The reference forms the cross power
// with a double loop over station pairs, O(N^2) per direction. Here
//
//   sum_{p<q} (J_p B) J_q^H = sum_q P_q J_q^H,  P_q = sum_{p<q} J_p B,
//
// with the running prefix P_q kept in registers: one pass over the
// stations, O(N) per direction, one thread per direction reading each
// station's row of the Jones array coalesced. The kernel is HBM-bound:
// 64 B (FP64 matrix) read per station-direction for ~48 flops.
#include <algorithm>

#include "common.cuh"

namespace oskb {
namespace {

constexpr int kThreads = 256;

template <typename T>
struct C
{
    T re, im;
};

template <typename T>
__device__ __forceinline__ C<T> cmul_(C<T> a, C<T> b)
{
    return C<T>{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}

// a conj(b)
template <typename T>
__device__ __forceinline__ C<T> cmulc_(C<T> a, C<T> b)
{
    return C<T>{a.re * b.re + a.im * b.im, a.im * b.re - a.re * b.im};
}

template <typename T>
__device__ __forceinline__ void load4(const T* p, C<T> m[4])
{
#pragma unroll
    for (int k = 0; k < 4; ++k) m[k] = C<T>{p[2 * k], p[2 * k + 1]};
}

// J B for B = [[I+Q, U+iV], [U-iV, I-Q]] (rows a b / c d).
template <typename T>
__device__ __forceinline__ void mul_b(const C<T> j[4], T I, T Q, T U, T V,
        C<T> r[4])
{
    const C<T> buv{U, V}, buv_c{U, -V};
    const T xx = I + Q, yy = I - Q;
    const C<T> ja_b = cmul_(j[1], buv_c), jc_b = cmul_(j[3], buv_c);
    const C<T> jb_a = cmul_(j[0], buv), jd_c = cmul_(j[2], buv);
    r[0] = C<T>{j[0].re * xx + ja_b.re, j[0].im * xx + ja_b.im};
    r[1] = C<T>{j[1].re * yy + jb_a.re, j[1].im * yy + jb_a.im};
    r[2] = C<T>{j[2].re * xx + jc_b.re, j[2].im * xx + jc_b.im};
    r[3] = C<T>{j[3].re * yy + jd_c.re, j[3].im * yy + jd_c.im};
}

// acc += M N^H
template <typename T>
__device__ __forceinline__ void add_mul_herm(C<T> acc[4], const C<T> m[4],
        const C<T> n[4])
{
    const C<T> t[8] = {cmulc_(m[0], n[0]), cmulc_(m[1], n[1]),
            cmulc_(m[0], n[2]), cmulc_(m[1], n[3]), cmulc_(m[2], n[0]),
            cmulc_(m[3], n[1]), cmulc_(m[2], n[2]), cmulc_(m[3], n[3])};
#pragma unroll
    for (int k = 0; k < 4; ++k)
    {
        acc[k].re += t[2 * k].re + t[2 * k + 1].re;
        acc[k].im += t[2 * k].im + t[2 * k + 1].im;
    }
}

template <typename T, bool MATRIX>
__global__ void __launch_bounds__(kThreads) auto_power_kernel(int n,
        int offset_in, const T* __restrict__ jones, T I, T Q, T U, T V,
        int offset_out, T* __restrict__ out)
{
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n;
            i += gridDim.x * kThreads)
    {
        if constexpr (MATRIX)
        {
            C<T> j[4], jb[4], r[4] = {};
            load4(jones + 8 * ((size_t) i + offset_in), j);
            mul_b(j, I, Q, U, V, jb);
            add_mul_herm(r, jb, j);
            T* o = out + 8 * ((size_t) i + offset_out);
#pragma unroll
            for (int k = 0; k < 4; ++k)
            {
                o[2 * k] = r[k].re;
                o[2 * k + 1] = r[k].im;
            }
        }
        else
        {
            const T* j = jones + 2 * ((size_t) i + offset_in);
            out[2 * ((size_t) i + offset_out)] = j[0] * j[0] + j[1] * j[1];
            out[2 * ((size_t) i + offset_out) + 1] = (T) 0;
        }
    }
}

template <typename T, bool MATRIX>
__global__ void __launch_bounds__(kThreads) cross_power_kernel(
        int num_sources, int num_stations, const T* __restrict__ jones,
        T I, T Q, T U, T V, T norm, int offset_out, T* __restrict__ out)
{
    constexpr int W = MATRIX ? 8 : 2;
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < num_sources;
            i += gridDim.x * kThreads)
    {
        if constexpr (MATRIX)
        {
            C<T> prefix[4] = {}, acc[4] = {};
            for (int q = 0; q < num_stations; ++q)
            {
                C<T> j[4];
                load4(jones + W * ((size_t) q * num_sources + i), j);
                add_mul_herm(acc, prefix, j);
                C<T> jb[4];
                mul_b(j, I, Q, U, V, jb);
#pragma unroll
                for (int k = 0; k < 4; ++k)
                {
                    prefix[k].re += jb[k].re;
                    prefix[k].im += jb[k].im;
                }
            }
            T* o = out + 8 * ((size_t) i + offset_out);
#pragma unroll
            for (int k = 0; k < 4; ++k)
            {
                o[2 * k] = acc[k].re * norm;
                o[2 * k + 1] = acc[k].im * norm;
            }
        }
        else
        {
            C<T> prefix{(T) 0, (T) 0}, acc{(T) 0, (T) 0};
            for (int q = 0; q < num_stations; ++q)
            {
                const T* jq = jones + W * ((size_t) q * num_sources + i);
                const C<T> j{jq[0], jq[1]};
                const C<T> t = cmulc_(prefix, j);
                acc.re += t.re;
                acc.im += t.im;
                prefix.re += j.re;
                prefix.im += j.im;
            }
            out[2 * ((size_t) i + offset_out)] = acc.re * norm;
            out[2 * ((size_t) i + offset_out) + 1] = acc.im * norm;
        }
    }
}

int grid_for(long long n)
{
    return (int) std::max<long long>(1, std::min<long long>(
            (n + kThreads - 1) / kThreads, 1 << 20));
}

template <typename T>
int auto_power(int matrix, int n, int offset_in, const T* jones, T I, T Q,
        T U, T V, int offset_out, T* out, void* stream)
{
    if (n < 0 || offset_in < 0 || offset_out < 0)
        return OSKB_ERR_INVALID_ARGUMENT;
    if (n == 0) return 0;
    if (!jones || !out) return OSKB_ERR_INVALID_ARGUMENT;
    if (matrix)
        auto_power_kernel<T, true><<<grid_for(n), kThreads, 0,
                as_stream(stream)>>>(n, offset_in, jones, I, Q, U, V,
                offset_out, out);
    else
        auto_power_kernel<T, false><<<grid_for(n), kThreads, 0,
                as_stream(stream)>>>(n, offset_in, jones, I, Q, U, V,
                offset_out, out);
    return check_launch("evaluate_auto_power");
}

template <typename T>
int cross_power(int matrix, int num_sources, int num_stations,
        const T* jones, T I, T Q, T U, T V, int offset_out, T* out,
        void* stream)
{
    if (num_sources < 0 || num_stations < 0 || offset_out < 0)
        return OSKB_ERR_INVALID_ARGUMENT;
    if (num_sources == 0) return 0;
    if (!jones || !out) return OSKB_ERR_INVALID_ARGUMENT;
    // oskar_evaluate_cross_power.c:54 (no pairs: the reference divides by
    // zero; here the result is zero)
    const T norm = num_stations > 1 ?
            (T) (2.0 / (num_stations * (double) (num_stations - 1))) : (T) 0;
    if (matrix)
        cross_power_kernel<T, true><<<grid_for(num_sources), kThreads, 0,
                as_stream(stream)>>>(num_sources, num_stations, jones, I, Q,
                U, V, norm, offset_out, out);
    else
        cross_power_kernel<T, false><<<grid_for(num_sources), kThreads, 0,
                as_stream(stream)>>>(num_sources, num_stations, jones, I, Q,
                U, V, norm, offset_out, out);
    return check_launch("evaluate_cross_power");
}

}  // namespace
}  // namespace oskb

extern "C" {

int oskb_evaluate_auto_power_d(int matrix, int n, int offset_in,
        const double* jones, double src_I, double src_Q, double src_U,
        double src_V, int offset_out, double* out, void* stream)
{
    return oskb::auto_power<double>(matrix, n, offset_in, jones, src_I,
            src_Q, src_U, src_V, offset_out, out, stream);
}

int oskb_evaluate_auto_power_f(int matrix, int n, int offset_in,
        const float* jones, float src_I, float src_Q, float src_U,
        float src_V, int offset_out, float* out, void* stream)
{
    return oskb::auto_power<float>(matrix, n, offset_in, jones, src_I,
            src_Q, src_U, src_V, offset_out, out, stream);
}

int oskb_evaluate_cross_power_d(int matrix, int num_sources,
        int num_stations, const double* jones, double src_I, double src_Q,
        double src_U, double src_V, int offset_out, double* out,
        void* stream)
{
    return oskb::cross_power<double>(matrix, num_sources, num_stations,
            jones, src_I, src_Q, src_U, src_V, offset_out, out, stream);
}

int oskb_evaluate_cross_power_f(int matrix, int num_sources,
        int num_stations, const float* jones, float src_I, float src_Q,
        float src_U, float src_V, int offset_out, float* out, void* stream)
{
    return oskb::cross_power<float>(matrix, num_sources, num_stations,
            jones, src_I, src_Q, src_U, src_V, offset_out, out, stream);
}

}  // extern "C"

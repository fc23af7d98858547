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
// station's row of the Jones array coalesced. With few directions the
// stations are split into segments (one CTA row each) whose pair sums,
// J B sums and J sums are combined in segment order by a second launch.
// The kernels are HBM-bound: 64 B (FP64 matrix) read per
// station-direction for ~48 flops.
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

// Station segments: segment g of S covers stations [g L, (g + 1) L). Per
// (direction, segment) the kernel writes the segment's own pair sum
// sum_{p<q in g} (J_p B) J_q^H, its sum of J_p B and its sum of J_q
// (2x2 complex each; scalar: complex, B = 1), to ws[g][term][direction].
template <typename T, bool MATRIX>
__global__ void __launch_bounds__(kThreads) cross_power_segments_kernel(
        int num_sources, int num_stations, int seg_len,
        const T* __restrict__ jones, T I, T Q, T U, T V, T* __restrict__ ws)
{
    constexpr int W = MATRIX ? 8 : 2;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= num_sources) return;
    const int g = blockIdx.y;
    const int q0 = g * seg_len, q1 = min(num_stations, q0 + seg_len);
    T* o = ws + (size_t) g * 3 * W * num_sources;
    if constexpr (MATRIX)
    {
        C<T> prefix[4] = {}, acc[4] = {}, sum_j[4] = {};
        for (int q = q0; q < q1; ++q)
        {
            C<T> j[4], jb[4];
            load4(jones + W * ((size_t) q * num_sources + i), j);
            add_mul_herm(acc, prefix, j);
            mul_b(j, I, Q, U, V, jb);
#pragma unroll
            for (int k = 0; k < 4; ++k)
            {
                prefix[k].re += jb[k].re;
                prefix[k].im += jb[k].im;
                sum_j[k].re += j[k].re;
                sum_j[k].im += j[k].im;
            }
        }
        const C<T>* terms[3] = {acc, prefix, sum_j};
#pragma unroll
        for (int t = 0; t < 3; ++t)
            for (int k = 0; k < 4; ++k)
            {
                o[(size_t) t * W * num_sources + W * (size_t) i + 2 * k] =
                        terms[t][k].re;
                o[(size_t) t * W * num_sources + W * (size_t) i + 2 * k + 1] =
                        terms[t][k].im;
            }
    }
    else
    {
        C<T> prefix{(T) 0, (T) 0}, acc{(T) 0, (T) 0};
        for (int q = q0; q < q1; ++q)
        {
            const T* jq = jones + W * ((size_t) q * num_sources + i);
            const C<T> j{jq[0], jq[1]};
            const C<T> t = cmulc_(prefix, j);
            acc.re += t.re;
            acc.im += t.im;
            prefix.re += j.re;
            prefix.im += j.im;
        }
        const C<T> terms[3] = {acc, prefix, prefix};
#pragma unroll
        for (int t = 0; t < 3; ++t)
        {
            o[(size_t) t * W * num_sources + W * (size_t) i] = terms[t].re;
            o[(size_t) t * W * num_sources + W * (size_t) i + 1] =
                    terms[t].im;
        }
    }
}

// Combines the segments in order: total = sum_g [pair_g + P_g S_g^H] with
// P_g the sum of J_p B over the segments before g and S_g segment g's sum
// of J_q.
template <typename T, bool MATRIX>
__global__ void __launch_bounds__(kThreads) cross_power_combine_kernel(
        int num_sources, int num_segments, const T* __restrict__ ws, T norm,
        int offset_out, T* __restrict__ out)
{
    constexpr int W = MATRIX ? 8 : 2;
    constexpr int NC = W / 2;
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < num_sources;
            i += gridDim.x * kThreads)
    {
        C<T> total[NC] = {}, before[NC] = {};
        for (int g = 0; g < num_segments; ++g)
        {
            const T* o = ws + (size_t) g * 3 * W * num_sources +
                    W * (size_t) i;
            C<T> pair[NC], pb[NC], sj[NC];
#pragma unroll
            for (int k = 0; k < NC; ++k)
            {
                pair[k] = C<T>{o[2 * k], o[2 * k + 1]};
                pb[k] = C<T>{o[(size_t) W * num_sources + 2 * k],
                        o[(size_t) W * num_sources + 2 * k + 1]};
                sj[k] = C<T>{o[(size_t) 2 * W * num_sources + 2 * k],
                        o[(size_t) 2 * W * num_sources + 2 * k + 1]};
            }
            if constexpr (MATRIX)
                add_mul_herm(total, before, sj);
            else
            {
                const C<T> t = cmulc_(before[0], sj[0]);
                total[0].re += t.re;
                total[0].im += t.im;
            }
#pragma unroll
            for (int k = 0; k < NC; ++k)
            {
                total[k].re += pair[k].re;
                total[k].im += pair[k].im;
                before[k].re += pb[k].re;
                before[k].im += pb[k].im;
            }
        }
        T* dst = out + W * ((size_t) i + offset_out);
#pragma unroll
        for (int k = 0; k < NC; ++k)
        {
            dst[2 * k] = total[k].re * norm;
            dst[2 * k + 1] = total[k].im * norm;
        }
    }
}

int num_sms() { return device_sm_count(); }

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
    // Few directions: split the stations into segments so that about
    // eight CTAs per SM run, each segment at least 32 stations long.
    const int blocks = (num_sources + kThreads - 1) / kThreads;
    int segments = 1;
    while (segments < 64 && (long long) blocks * segments < 8LL * num_sms()
            && num_stations / (2 * segments) >= 32)
        segments *= 2;
    cudaStream_t st = as_stream(stream);
    T* ws = nullptr;
    if (segments > 1)
    {
        const size_t bytes = (size_t) segments * 3 * (matrix ? 8 : 2) *
                num_sources * sizeof(T);
        if (scratch_alloc((void**) &ws, bytes, st) != cudaSuccess)
        {
            cudaGetLastError();  // no room: one pass per direction
            ws = nullptr;
            segments = 1;
        }
    }
    if (segments == 1)
    {
        if (matrix)
            cross_power_kernel<T, true><<<grid_for(num_sources), kThreads, 0,
                    st>>>(num_sources, num_stations, jones, I, Q, U, V, norm,
                    offset_out, out);
        else
            cross_power_kernel<T, false><<<grid_for(num_sources), kThreads,
                    0, st>>>(num_sources, num_stations, jones, I, Q, U, V,
                    norm, offset_out, out);
        return check_launch("evaluate_cross_power");
    }
    const int seg_len = (num_stations + segments - 1) / segments;
    const dim3 grid(blocks, segments);
    if (matrix)
    {
        cross_power_segments_kernel<T, true><<<grid, kThreads, 0, st>>>(
                num_sources, num_stations, seg_len, jones, I, Q, U, V, ws);
        cross_power_combine_kernel<T, true><<<grid_for(num_sources),
                kThreads, 0, st>>>(num_sources, segments, ws, norm,
                offset_out, out);
    }
    else
    {
        cross_power_segments_kernel<T, false><<<grid, kThreads, 0, st>>>(
                num_sources, num_stations, seg_len, jones, I, Q, U, V, ws);
        cross_power_combine_kernel<T, false><<<grid_for(num_sources),
                kThreads, 0, st>>>(num_sources, segments, ws, norm,
                offset_out, out);
    }
    const int err = check_launch("evaluate_cross_power");
    scratch_free(ws, st);
    return err;
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

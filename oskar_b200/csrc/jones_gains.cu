// Per-station terms applied to a Jones array in place: cable-length phase
// errors and complex station gains.
//
// Jones arrays are [station][source] (interferometer/private_jones.h:34-41).
// A CTA works on one station row at a time (blockIdx.y strides over
// stations), so each thread forms the station's gain once per row and then
// streams several sources of that row: the kernels are HBM-bound (FP64
// matrix Jones: 64 B read + 64 B written per station-source).
//
// References: interferometer/define_jones_apply_cable_length_errors.h:3-74
// (gain diag(e^{i k dx}, e^{i k dy}), k = 2 pi f / c; scalar Jones take the
// x term only and are left alone without x errors) and
// interferometer/define_jones_apply_station_gains.h:3-45 (J <- G J).
#include "common.cuh"

namespace oskb {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ void m_sincos(float x, float* s, float* c)
{
    sincosf(x, s, c);
}
__device__ __forceinline__ void m_sincos(double x, double* s, double* c)
{
    sincos(x, s, c);
}

// Grid: x covers a station row's sources (capped so each thread streams
// several), y strides over stations.
dim3 row_grid(int num_sources, int num_stations)
{
    const int num_sms = device_sm_count();
    int gx = (num_sources + kThreads - 1) / kThreads;
    int gy = num_stations < 65535 ? num_stations : 65535;
    const long long cap = (long long) num_sms * 8;
    while ((long long) gx * gy > cap && gx > 1) gx = (gx + 1) / 2;
    return dim3(gx < 1 ? 1 : gx, gy < 1 ? 1 : gy);
}

template <typename T>
struct C2
{
    T re, im;
};

template <typename T>
__device__ __forceinline__ C2<T> cx_mul(C2<T> x, C2<T> y)
{
    return C2<T>{x.re * y.re - x.im * y.im, x.re * y.im + x.im * y.re};
}

template <typename T, bool MATRIX>
__global__ void __launch_bounds__(kThreads) cable_kernel(int num_sources,
        int num_stations, T wavenumber, const T* __restrict__ ex,
        const T* __restrict__ ey, T* jones)
{
    for (int p = blockIdx.y; p < num_stations; p += gridDim.y)
    {
        C2<T> gx{1, 0}, gy{1, 0};
        if (ex) m_sincos(wavenumber * ex[p], &gx.im, &gx.re);
        if (ey) m_sincos(wavenumber * ey[p], &gy.im, &gy.re);
        T* row = jones + (size_t) (MATRIX ? 8 : 2) * num_sources * p;
        for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < num_sources;
                s += gridDim.x * blockDim.x)
        {
            T* e = row + (size_t) (MATRIX ? 8 : 2) * s;
            if constexpr (!MATRIX)
            {
                const C2<T> r = cx_mul(gx, C2<T>{e[0], e[1]});
                e[0] = r.re;
                e[1] = r.im;
            }
            else
            {
                T v[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) v[k] = e[k];
#pragma unroll
                for (int k = 0; k < 4; ++k)
                {
                    // rows a, b take the x gain; rows c, d the y gain
                    const C2<T> r = cx_mul(k < 2 ? gx : gy,
                            C2<T>{v[2 * k], v[2 * k + 1]});
                    v[2 * k] = r.re;
                    v[2 * k + 1] = r.im;
                }
#pragma unroll
                for (int k = 0; k < 8; ++k) e[k] = v[k];
            }
        }
    }
}

template <typename T, bool MATRIX>
__global__ void __launch_bounds__(kThreads) gains_kernel(int num_sources,
        int num_stations, const T* __restrict__ gains, T* jones)
{
    constexpr int W = MATRIX ? 8 : 2;
    for (int p = blockIdx.y; p < num_stations; p += gridDim.y)
    {
        T g[W];
#pragma unroll
        for (int k = 0; k < W; ++k) g[k] = gains[(size_t) W * p + k];
        T* row = jones + (size_t) W * num_sources * p;
        for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < num_sources;
                s += gridDim.x * blockDim.x)
        {
            T* e = row + (size_t) W * s;
            if constexpr (!MATRIX)
            {
                const C2<T> r = cx_mul(C2<T>{g[0], g[1]}, C2<T>{e[0], e[1]});
                e[0] = r.re;
                e[1] = r.im;
            }
            else
            {
                T v[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) v[k] = e[k];
                const C2<T> ga{g[0], g[1]}, gb{g[2], g[3]}, gc{g[4], g[5]},
                        gd{g[6], g[7]}, ja{v[0], v[1]}, jb{v[2], v[3]},
                        jc{v[4], v[5]}, jd{v[6], v[7]};
                C2<T> o[4];
                C2<T> t0 = cx_mul(ga, ja), t1 = cx_mul(gb, jc);
                o[0] = C2<T>{t0.re + t1.re, t0.im + t1.im};
                t0 = cx_mul(ga, jb); t1 = cx_mul(gb, jd);
                o[1] = C2<T>{t0.re + t1.re, t0.im + t1.im};
                t0 = cx_mul(gc, ja); t1 = cx_mul(gd, jc);
                o[2] = C2<T>{t0.re + t1.re, t0.im + t1.im};
                t0 = cx_mul(gc, jb); t1 = cx_mul(gd, jd);
                o[3] = C2<T>{t0.re + t1.re, t0.im + t1.im};
#pragma unroll
                for (int k = 0; k < 4; ++k)
                {
                    e[2 * k] = o[k].re;
                    e[2 * k + 1] = o[k].im;
                }
            }
        }
    }
}

template <typename T>
int apply_cable(int matrix, int num_sources, int num_stations, T wavenumber,
        const T* ex, const T* ey, T* jones, void* stream)
{
    if (num_sources < 0 || num_stations < 0) return OSKB_ERR_INVALID_ARGUMENT;
    if (!ex && !ey) return 0;
    if (!matrix && !ex) return 0;
    if (num_sources == 0 || num_stations == 0) return 0;
    if (!jones) return OSKB_ERR_INVALID_ARGUMENT;
    const dim3 grid = row_grid(num_sources, num_stations);
    if (matrix)
        cable_kernel<T, true><<<grid, kThreads, 0, as_stream(stream)>>>(
                num_sources, num_stations, wavenumber, ex, ey, jones);
    else
        cable_kernel<T, false><<<grid, kThreads, 0, as_stream(stream)>>>(
                num_sources, num_stations, wavenumber, ex, nullptr, jones);
    return check_launch("jones_apply_cable_length_errors");
}

template <typename T>
int apply_gains(int matrix, int num_sources, int num_stations,
        const T* gains, T* jones, void* stream)
{
    if (num_sources < 0 || num_stations < 0) return OSKB_ERR_INVALID_ARGUMENT;
    if (num_sources == 0 || num_stations == 0) return 0;
    if (!gains || !jones) return OSKB_ERR_INVALID_ARGUMENT;
    const dim3 grid = row_grid(num_sources, num_stations);
    if (matrix)
        gains_kernel<T, true><<<grid, kThreads, 0, as_stream(stream)>>>(
                num_sources, num_stations, gains, jones);
    else
        gains_kernel<T, false><<<grid, kThreads, 0, as_stream(stream)>>>(
                num_sources, num_stations, gains, jones);
    return check_launch("jones_apply_station_gains");
}

}  // namespace
}  // namespace oskb

extern "C" {

int oskb_jones_apply_cable_length_errors_d(int matrix, int num_sources,
        int num_stations, double wavenumber, const double* errors_x,
        const double* errors_y, double* jones, void* stream)
{
    return oskb::apply_cable<double>(matrix, num_sources, num_stations,
            wavenumber, errors_x, errors_y, jones, stream);
}

int oskb_jones_apply_cable_length_errors_f(int matrix, int num_sources,
        int num_stations, float wavenumber, const float* errors_x,
        const float* errors_y, float* jones, void* stream)
{
    return oskb::apply_cable<float>(matrix, num_sources, num_stations,
            wavenumber, errors_x, errors_y, jones, stream);
}

int oskb_jones_apply_station_gains_d(int matrix, int num_sources,
        int num_stations, const double* gains, double* jones, void* stream)
{
    return oskb::apply_gains<double>(matrix, num_sources, num_stations,
            gains, jones, stream);
}

int oskb_jones_apply_station_gains_f(int matrix, int num_sources,
        int num_stations, const float* gains, float* jones, void* stream)
{
    return oskb::apply_gains<float>(matrix, num_sources, num_stations,
            gains, jones, stream);
}

}  // extern "C"

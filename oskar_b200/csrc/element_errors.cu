// Element weight factors of aperture-array stations: time-variable element
// gain and phase errors, and apodisation.
//
// Replaces oskar_evaluate_element_weights_errors
// (oskar/telescope/station/src/oskar_evaluate_element_weights_errors.c:
// 19-110 with define_evaluate_element_weights_errors.h:3-16) and the
// random fill it calls (oskar/mem/src/oskar_mem_random_gaussian.c:14-191,
// GPU form in oskar_mem_random_gaussian_cuda.cu): per element a Gaussian
// pair (g, h) from Philox4x32-10 with key {seed, 0xCAFEF00D} and counter
// {element / 2, time index, station id, 0x12345678}, then the factor
// (gain + gain_error g) e^{i (phase + phase_error h)}. The station-beam
// kernel takes the product of these factors and the apodisation weights
// (oskar_station_evaluate_element_weights.c:33-64 multiplies the DFT
// weights by each in turn) as one complex factor per element.
//
// Philox4x32-10 is restated from its paper (J. K. Salmon, M. A. Moraes,
// R. O. Dror, D. E. Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC11, 2011). One thread draws the four values of one counter, i.e. the
// pairs of two elements; the whole [station][element] array is one launch.
#include <algorithm>

#include "common.cuh"

namespace oskb {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0)
{
    uint32_t k1 = 0xCAFEF00Du;
#pragma unroll
    for (int r = 0; r < 10; ++r)
    {
        if (r > 0)
        {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const uint32_t lo0 = 0xD2511F53u * c.x;
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
    }
    return c;
}

// Box-Muller pair as the reference's GPU path forms it
// (math/private_random_helpers.h:42-107): angle pi x with
// x = u0 2^-31 + 2^-32 through sincospi, radius sqrt(-2 log y) with
// y = u1 2^-32 + 2^-33.
__device__ __forceinline__ void box_muller(uint32_t u0, uint32_t u1,
        double* f0, double* f1)
{
    const double x = (double) u0 * 0x1p-31 + 0x1p-32;
    const double y = (double) u1 * 0x1p-32 + 0x1p-33;
    sincospi(x, f0, f1);
    const double r = sqrt(-2.0 * log(y));
    *f0 *= r;
    *f1 *= r;
}
__device__ __forceinline__ void box_muller(uint32_t u0, uint32_t u1,
        float* f0, float* f1)
{
    const float x = (float) u0 * 0x1p-31f + 0x1p-32f;
    const float y = (float) u1 * 0x1p-32f + 0x1p-33f;
    sincospif(x, f0, f1);
    const float r = sqrtf(-2.0f * logf(y));
    *f0 *= r;
    *f1 *= r;
}

__device__ __forceinline__ void m_sincos(float x, float* s, float* c)
{
    sincosf(x, s, c);
}
__device__ __forceinline__ void m_sincos(double x, double* s, double* c)
{
    sincos(x, s, c);
}

// factors[s][e] = errors (if gain != NULL) x apodisation[s][e] (if given);
// station s has id first_station_id + s. Error arrays are [station][element]
// when per_station, else one [element] array shared by all stations.
template <typename T>
__global__ void __launch_bounds__(kThreads) factors_kernel(int num_elements,
        int num_stations, int first_station_id, unsigned int seed,
        int time_index, const T* __restrict__ gain,
        const T* __restrict__ gain_error, const T* __restrict__ phase,
        const T* __restrict__ phase_error, int per_station,
        const T* __restrict__ apodisation, T* __restrict__ factors)
{
    typedef typename vec2<T>::type T2;
    const int num_pairs = (num_elements + 1) / 2;
    const long long total = (long long) num_pairs * num_stations;
    for (long long it = blockIdx.x * (long long) kThreads + threadIdx.x;
            it < total; it += (long long) gridDim.x * kThreads)
    {
        const int st = (int) (it / num_pairs);
        const int q = (int) (it - (long long) st * num_pairs);
        T g[4] = {(T) 0, (T) 0, (T) 0, (T) 0};
        if (gain)
        {
            const uint4 u = philox4x32_10(make_uint4((uint32_t) q,
                    (uint32_t) time_index,
                    (uint32_t) (first_station_id + st), 0x12345678u), seed);
            box_muller(u.x, u.y, &g[0], &g[1]);
            box_muller(u.z, u.w, &g[2], &g[3]);
        }
#pragma unroll
        for (int h = 0; h < 2; ++h)
        {
            const int e = 2 * q + h;
            if (e >= num_elements) break;
            const size_t i = (size_t) st * num_elements + e;
            const size_t ie = per_station ? i : (size_t) e;
            T2 f{(T) 1, (T) 0};
            if (gain)
            {
                const T amp = g[2 * h] * gain_error[ie] + gain[ie];
                const T ph = g[2 * h + 1] * phase_error[ie] + phase[ie];
                T sn, cs;
                m_sincos(ph, &sn, &cs);
                f = T2{cs * amp, sn * amp};
            }
            if (apodisation)
            {
                const T2 a = reinterpret_cast<const T2*>(apodisation)[i];
                f = T2{f.x * a.x - f.y * a.y, f.x * a.y + f.y * a.x};
            }
            reinterpret_cast<T2*>(factors)[i] = f;
        }
    }
}

template <typename T>
int weight_factors(int num_stations, int num_elements, int first_station_id,
        unsigned int seed, int time_index, const T* gain,
        const T* gain_error, const T* phase, const T* phase_error,
        int per_station, const T* apodisation, T* factors, void* stream)
{
    if (num_stations < 0 || num_elements < 0) return OSKB_ERR_INVALID_ARGUMENT;
    if (num_stations == 0 || num_elements == 0) return 0;
    if (!factors) return OSKB_ERR_INVALID_ARGUMENT;
    if (gain && (!gain_error || !phase || !phase_error))
        return OSKB_ERR_INVALID_ARGUMENT;
    const long long total = (long long) ((num_elements + 1) / 2) *
            num_stations;
    const int grid = (int) std::min<long long>((total + kThreads - 1) /
            kThreads, 1 << 20);
    factors_kernel<T><<<grid, kThreads, 0, as_stream(stream)>>>(
            num_elements, num_stations, first_station_id, seed, time_index,
            gain, gain_error, phase, phase_error, per_station, apodisation,
            factors);
    return check_launch("element_weight_factors");
}

}  // namespace
}  // namespace oskb

extern "C" {

int oskb_evaluate_element_weights_errors_d(int num_elements,
        const double* gain, const double* gain_error, const double* phase,
        const double* phase_error, unsigned int random_seed, int time_index,
        int station_id, double* errors, void* stream)
{
    if (!gain) return OSKB_ERR_INVALID_ARGUMENT;
    return oskb::weight_factors<double>(1, num_elements, station_id,
            random_seed, time_index, gain, gain_error, phase, phase_error, 1,
            nullptr, errors, stream);
}

int oskb_evaluate_element_weights_errors_f(int num_elements,
        const float* gain, const float* gain_error, const float* phase,
        const float* phase_error, unsigned int random_seed, int time_index,
        int station_id, float* errors, void* stream)
{
    if (!gain) return OSKB_ERR_INVALID_ARGUMENT;
    return oskb::weight_factors<float>(1, num_elements, station_id,
            random_seed, time_index, gain, gain_error, phase, phase_error, 1,
            nullptr, errors, stream);
}

int oskb_station_element_weight_factors_d(int num_stations,
        int num_elements, int first_station_id, unsigned int random_seed,
        int time_index, const double* gain, const double* gain_error,
        const double* phase, const double* phase_error, int per_station,
        const double* apodisation, double* factors, void* stream)
{
    return oskb::weight_factors<double>(num_stations, num_elements,
            first_station_id, random_seed, time_index, gain, gain_error,
            phase, phase_error, per_station, apodisation, factors, stream);
}

int oskb_station_element_weight_factors_f(int num_stations,
        int num_elements, int first_station_id, unsigned int random_seed,
        int time_index, const float* gain, const float* gain_error,
        const float* phase, const float* phase_error, int per_station,
        const float* apodisation, float* factors, void* stream)
{
    return oskb::weight_factors<float>(num_stations, num_elements,
            first_station_id, random_seed, time_index, gain, gain_error,
            phase, phase_error, per_station, apodisation, factors, stream);
}

}  // extern "C"

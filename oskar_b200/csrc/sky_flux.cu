// Sky flux scaling with frequency on the device.
//
// The sky table is column-major: column k of source s at
// table[capacity * k + s], the columns of one type adjacent and in index
// order, and num_valid_columns[s * 20 + type] counts the columns of each
// type that hold data for source s (reference layout:
// oskar/sky/private_sky.h, oskar/sky/src/oskar_sky_sort_columns.c; column
// types oskar/sky/oskar_sky_enum.h:14-35). One thread scales one
// (channel, source) pair; consecutive threads take consecutive sources, so
// every column read and every output write is coalesced. The multi-channel
// entry scales the whole band in one launch: the reference rescales the sky
// once per (dump, channel) inside its block loop
// (oskar_interferometer_run_block.c:183-190), though the result depends on
// the channel only.
//
// Reference kernel: oskar/sky/define_sky_scale_flux_with_frequency.h:3-253.
// A column index outside [0, num_columns) reads as 0, where the reference
// would read outside its table.
#include "common.cuh"

namespace oskb {
namespace {

// Column types (oskar/sky/oskar_sky_enum.h:14-35).
enum
{
    kTyI = 3, kTyQ = 4, kTyU = 5, kTyV = 6, kTyRefHz = 7, kTySpx = 8,
    kTyRm = 9, kTyLinSi = 13, kTyPolA = 14, kTyPolF = 15, kTyRefWave = 16,
    kTyCurv = 17, kTyLineWidth = 18, kTyIncHz = 19, kNumTypes = 20
};

// First-column slots, in the reference kernel's argument order.
enum
{
    kCI = 0, kCQ, kCU, kCV, kCRef, kCLin, kCSpx, kCRm, kCPolF, kCPolA,
    kCRefWave, kCCurv, kCLineWidth, kCInc, kNumSlots
};

struct FluxCols
{
    int c[kNumSlots];
};

__device__ __forceinline__ float m_exp(float x) { return expf(x); }
__device__ __forceinline__ double m_exp(double x) { return exp(x); }
__device__ __forceinline__ float m_log(float x) { return logf(x); }
__device__ __forceinline__ double m_log(double x) { return log(x); }
__device__ __forceinline__ float m_log10(float x) { return log10f(x); }
__device__ __forceinline__ double m_log10(double x) { return log10(x); }
__device__ __forceinline__ float m_pow(float x, float y) { return powf(x, y); }
__device__ __forceinline__ double m_pow(double x, double y)
{
    return pow(x, y);
}
__device__ __forceinline__ float m_atan2(float y, float x)
{
    return atan2f(y, x);
}
__device__ __forceinline__ double m_atan2(double y, double x)
{
    return atan2(y, x);
}
__device__ __forceinline__ float m_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double m_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ void m_sincos(float x, float* s, float* c)
{
    sincosf(x, s, c);
}
__device__ __forceinline__ void m_sincos(double x, double* s, double* c)
{
    sincos(x, s, c);
}

template <typename T>
struct SkyTable
{
    const T* __restrict__ data;
    int capacity, num_columns;
    __device__ __forceinline__ T at(int column, int s) const
    {
        return (column >= 0 && column < num_columns) ?
                data[(size_t) capacity * column + s] : (T) 0;
    }
};

template <typename T>
__device__ __forceinline__ T nan_to_zero(T x) { return x != x ? (T) 0 : x; }

// Per-source column counts this scaling reads.
struct Counts
{
    int i, q, u, v, ref, spx, rm, lin, pola, polf, refw, curv, lw, inc;
};

__device__ __forceinline__ Counts load_counts(const int* __restrict__ nv)
{
    Counts n;
    n.i = __ldg(nv + kTyI); n.q = __ldg(nv + kTyQ); n.u = __ldg(nv + kTyU);
    n.v = __ldg(nv + kTyV); n.ref = __ldg(nv + kTyRefHz);
    n.spx = __ldg(nv + kTySpx); n.rm = __ldg(nv + kTyRm);
    n.lin = __ldg(nv + kTyLinSi); n.pola = __ldg(nv + kTyPolA);
    n.polf = __ldg(nv + kTyPolF); n.refw = __ldg(nv + kTyRefWave);
    n.curv = __ldg(nv + kTyCurv); n.lw = __ldg(nv + kTyLineWidth);
    n.inc = __ldg(nv + kTyIncHz);
    return n;
}

// Stokes I of source s at freq, from its value i_in at freq0
// (define_sky_scale_flux_with_frequency.h:5-86).
template <typename T>
__device__ T stokes_i_at(const SkyTable<T>& tab, const FluxCols& col,
        const Counts& n, int s, T i_in, T freq, T freq0)
{
    if (n.lw > 0)
    {
        // Sum of Gaussian line profiles, one per I column.
        const T inc = n.inc > 0 ? tab.at(col.c[kCInc], s) : (T) 0;
        T sum = 0;
        for (int c = 0; c < n.i; ++c)
        {
            const T amp = tab.at(col.c[kCI] + c, s);
            const T ref = c < n.ref ? tab.at(col.c[kCRef] + c, s) :
                    tab.at(col.c[kCRef], s) + c * inc;
            const T sigma = tab.at(col.c[kCLineWidth] + (c < n.lw ? c : 0),
                    s);
            const T x = freq - ref;
            sum += amp * m_exp(-(x * x) / (2 * sigma * sigma));
        }
        return sum;
    }
    if (n.i > 1) return i_in;  // tabulated flux: no spectral model
    if (n.curv > 0)
    {
        // Curved power law (Callingham et al. 2017, eq. 2).
        const T spx = n.spx > 0 ? nan_to_zero(tab.at(col.c[kCSpx], s)) :
                (T) 0;
        const T q = nan_to_zero(tab.at(col.c[kCCurv], s));
        const T ratio = freq / freq0;
        const T lr = m_log(ratio);
        return i_in * m_exp(q * (lr * lr)) * m_pow(ratio, spx);
    }
    const T lin = n.lin > 0 ? tab.at(col.c[kCLin], s) : (T) 0;
    T acc = 0;
    if (lin == (T) 0)
    {
        // Logarithmic spectral-index polynomial, Horner's rule.
        const T base = m_log10(freq / freq0);
        for (int c = n.spx - 1; c >= 0; --c)
            acc = base * acc + nan_to_zero(tab.at(col.c[kCSpx] + c, s));
        return i_in * m_pow((T) 10, base * acc);
    }
    // Linear spectral-index polynomial.
    const T base = freq / freq0 - (T) 1;
    for (int c = n.spx - 1; c >= 0; --c)
        acc = base * acc + nan_to_zero(tab.at(col.c[kCSpx] + c, s));
    return i_in + base * acc;
}

template <typename T>
__global__ void __launch_bounds__(256) scale_flux_kernel(int num_sources,
        int num_channels, T freq_single, const double* __restrict__ freqs,
        const SkyTable<T> tab, const int* __restrict__ num_valid,
        const FluxCols col, long long out_stride, T* __restrict__ out_i,
        T* __restrict__ out_q, T* __restrict__ out_u, T* __restrict__ out_v)
{
    const T kC0 = (T) 299792458;
    const long long total = (long long) num_sources * num_channels;
    for (long long idx = (long long) blockIdx.x * blockDim.x + threadIdx.x;
            idx < total; idx += (long long) gridDim.x * blockDim.x)
    {
        const int s = (int) (idx % num_sources);
        const int ch = (int) (idx / num_sources);
        const T freq = freqs ? (T) freqs[ch] : freq_single;
        const Counts n = load_counts(num_valid + (size_t) s * kNumTypes);

        // Reference channel nearest freq.
        T diff = (T) 1e38, f0 = 0;
        int chan = 0;
        const bool regular = n.inc == 1 && n.ref == 1;
        const T start = tab.at(col.c[kCRef], s);
        const T step = regular ? tab.at(col.c[kCInc], s) : (T) 0;
        for (int j = 0; j < n.i; ++j)
        {
            const T tf = regular ? start + j * step :
                    tab.at(col.c[kCRef] + j, s);
            const T d = fabs(tf - freq);
            if (d < diff)
            {
                diff = d;
                chan = j;
                f0 = tf;
            }
        }
        // Stokes values of that channel (NaN -> 0).
        T iquv[4];
        const int nq[4] = {n.i, n.q, n.u, n.v};
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            T x = 0;
            if (nq[j] > 0)
                x = tab.at(col.c[kCI + j] + (chan < nq[j] ? chan : 0), s);
            iquv[j] = nan_to_zero(x);
        }
        // Q, U from polarisation angle and fraction where not given.
        if (n.pola > 0 && n.polf > 0 && (n.q <= 0 || n.u <= 0))
        {
            const T ang = tab.at(col.c[kCPolA] + (chan < n.pola ? chan : 0),
                    s);
            const T frac = tab.at(col.c[kCPolF] + (chan < n.polf ? chan : 0),
                    s);
            T sn, cs;
            m_sincos(2 * ang, &sn, &cs);
            iquv[1] = frac * iquv[0] * cs;
            iquv[2] = frac * iquv[0] * sn;
        }
        T oi = iquv[0], oq = iquv[1], ou = iquv[2], ov = iquv[3];
        if (f0 != (T) 0)
        {
            oi = stokes_i_at(tab, col, n, s, iquv[0], freq, f0);
            const T scale = iquv[0] != (T) 0 ? oi / iquv[0] : (T) 0;
            if (n.rm > 0)
            {
                // Faraday rotation of the polarisation angle.
                const T rm = nan_to_zero(tab.at(col.c[kCRm], s));
                const T lambda = kC0 / freq;
                T chi0, frac;
                if (n.pola <= 0 || n.polf <= 0)
                {
                    const T lambda0 = n.refw > 0 ?
                            tab.at(col.c[kCRefWave], s) : kC0 / f0;
                    const T i_ref = stokes_i_at(tab, col, n, s, iquv[0],
                            freq, kC0 / lambda0);
                    chi0 = (T) 0.5 * m_atan2(iquv[2], iquv[1]) -
                            lambda0 * lambda0 * rm;
                    frac = m_sqrt(iquv[1] * iquv[1] + iquv[2] * iquv[2]) /
                            i_ref;
                }
                else
                {
                    chi0 = tab.at(col.c[kCPolA] +
                            (chan < n.pola ? chan : 0), s);
                    frac = tab.at(col.c[kCPolF] +
                            (chan < n.polf ? chan : 0), s);
                }
                const T chi = chi0 + rm * (lambda * lambda);
                T sn, cs;
                m_sincos(2 * chi, &sn, &cs);
                oq = frac * oi * cs;
                ou = frac * oi * sn;
            }
            else
            {
                oq = scale * iquv[1];
                ou = scale * iquv[2];
            }
            ov = scale * iquv[3];
        }
        const size_t o = (size_t) ch * out_stride + s;
        out_i[o] = oi;
        out_q[o] = oq;
        out_u[o] = ou;
        out_v[o] = ov;
    }
}

int flux_grid(long long n)
{
    const int num_sms = device_sm_count();
    long long blocks = (n + 255) / 256;
    const long long cap = (long long) num_sms * 8;
    if (blocks > cap) blocks = cap;
    return (int) (blocks < 1 ? 1 : blocks);
}

template <typename T>
int scale_flux(int num_sources, int capacity, int num_columns,
        int num_channels, T freq_single, const double* freqs, const T* table,
        const int* num_valid, const int* cols, long long out_stride,
        T* out_i, T* out_q, T* out_u, T* out_v, void* stream)
{
    if (num_sources < 0 || num_channels < 0 || capacity < num_sources ||
            num_columns < 0)
        return OSKB_ERR_INVALID_ARGUMENT;
    if (cols[kCI] < 0) return OSKB_ERR_INVALID_ARGUMENT;  // no Stokes I
    if (num_sources == 0 || num_channels == 0) return 0;
    if (!table || !num_valid || !out_i || !out_q || !out_u || !out_v ||
            (num_channels > 1 && out_stride < num_sources))
        return OSKB_ERR_INVALID_ARGUMENT;
    SkyTable<T> tab;
    tab.data = table;
    tab.capacity = capacity;
    tab.num_columns = num_columns;
    FluxCols col;
    for (int k = 0; k < kNumSlots; ++k) col.c[k] = cols[k];
    const long long total = (long long) num_sources * num_channels;
    scale_flux_kernel<T><<<flux_grid(total), 256, 0, as_stream(stream)>>>(
            num_sources, num_channels, freq_single, freqs, tab, num_valid,
            col, out_stride, out_i, out_q, out_u, out_v);
    return check_launch("sky_scale_flux_with_frequency");
}

}  // namespace
}  // namespace oskb

extern "C" {

#define OSKB_FLUX_ENTRIES(T, S)                                              \
int oskb_sky_scale_flux_with_frequency_##S(int num_sources, int capacity,    \
        int num_columns, T freq_hz, const T* table,                          \
        const int* num_valid_columns, int col_i, int col_q, int col_u,       \
        int col_v, int col_ref_freq, int col_lin_sp_index, int col_sp_index, \
        int col_rot_meas, int col_pol_frac, int col_pol_ang,                 \
        int col_ref_wavelength, int col_sp_curvature, int col_line_width,    \
        int col_freq_inc, T* out_i, T* out_q, T* out_u, T* out_v,            \
        void* stream)                                                        \
{                                                                            \
    const int cols[14] = {col_i, col_q, col_u, col_v, col_ref_freq,          \
            col_lin_sp_index, col_sp_index, col_rot_meas, col_pol_frac,      \
            col_pol_ang, col_ref_wavelength, col_sp_curvature,               \
            col_line_width, col_freq_inc};                                   \
    return oskb::scale_flux<T>(num_sources, capacity, num_columns, 1,        \
            freq_hz, nullptr, table, num_valid_columns, cols, num_sources,   \
            out_i, out_q, out_u, out_v, stream);                             \
}                                                                            \
int oskb_sky_scale_flux_channels_##S(int num_sources, int capacity,          \
        int num_columns, int num_channels, const double* frequency_hz,       \
        const T* table, const int* num_valid_columns, const int* columns,    \
        long long out_channel_stride, T* out_i, T* out_q, T* out_u,          \
        T* out_v, void* stream)                                              \
{                                                                            \
    if (!frequency_hz || !columns) return OSKB_ERR_INVALID_ARGUMENT;         \
    return oskb::scale_flux<T>(num_sources, capacity, num_columns,           \
            num_channels, (T) 0, frequency_hz, table, num_valid_columns,     \
            columns, out_channel_stride, out_i, out_q, out_u, out_v,         \
            stream);                                                         \
}

OSKB_FLUX_ENTRIES(double, d)
OSKB_FLUX_ENTRIES(float, f)
#undef OSKB_FLUX_ENTRIES

}  // extern "C"

// Device-side sky and baseline preparation around the hot path:
//  - (lon, lat) -> direction cosines relative to a phase centre
//    (convert/define_convert_lon_lat_to_relative_directions.h:3-19);
//  - apparent (RA, Dec) -> ENU direction cosines for every station at once
//    (convert/define_convert_apparent_ra_dec_to_enu_directions.h:3-30; the
//    reference converts per station model in a host loop);
//  - horizon mask over all stations and order-preserving compaction of the
//    sky columns (sky/src/oskar_sky_horizon_clip.c:18-96 with
//    sky/define_update_horizon_mask.h:3-12);
//  - station (u, v, w) -> baseline (uu, vv, ww)
//    (convert/src/oskar_convert_station_uvw_to_baseline_uvw.c:13-29).
// All elementwise: HBM-bound (a few bytes per source or baseline).
#include <math.h>
#include <stdlib.h>

#include <vector>

#include "common.cuh"

namespace oskb {
namespace {

template <typename T>
__global__ void lonlat_kernel(int num, const T* __restrict__ lon,
        const T* __restrict__ lat, T lon0, T cos_lat0, T sin_lat0,
        T* __restrict__ l, T* __restrict__ m, T* __restrict__ n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= num) return;
    T sl, cl, sb, cb;
    sincos(lon[i] - lon0, &sl, &cl);
    sincos(lat[i], &sb, &cb);
    l[i] = cb * sl;
    m[i] = cos_lat0 * sb - sin_lat0 * cb * cl;
    if (n) n[i] = sin_lat0 * sb + cos_lat0 * cb * cl;
}

// One launch for every station: (x, y, z)[station][source].
template <typename T>
__global__ void radec_enu_kernel(int num, const T* __restrict__ ra,
        const T* __restrict__ dec, const double* __restrict__ lst_rad,
        const double* __restrict__ lat_rad, T* __restrict__ x,
        T* __restrict__ y, T* __restrict__ z)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int st = blockIdx.y;
    if (i >= num) return;
    // the reference's driver forms sin/cos of the latitude in double
    const T sin_lat = (T) sin(lat_rad[st]), cos_lat = (T) cos(lat_rad[st]);
    const T lst = (T) lst_rad[st];
    T sh, ch, sd, cd;
    sincos(lst - ra[i], &sh, &ch);
    sincos(dec[i], &sd, &cd);
    const size_t o = (size_t) st * num + i;
    x[o] = -cd * sh;
    y[o] = cos_lat * sd - sin_lat * cd * ch;
    z[o] = sin_lat * sd + cos_lat * cd * ch;
}

// mask[i] |= source i above the horizon of any station (multipliers
// [station][3] formed in double on the host, rounded to T).
template <typename T>
__global__ void horizon_kernel(int num, const T* __restrict__ l,
        const T* __restrict__ m, const T* __restrict__ n, int num_st,
        const T* __restrict__ mul, int* __restrict__ mask)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= num) return;
    const T li = l[i], mi = m[i], ni = n[i];
    int v = mask[i];
    for (int s = 0; s < num_st && !v; ++s)
        v |= (li * mul[3 * s] + mi * mul[3 * s + 1] + ni * mul[3 * s + 2]) >
                (T) 0;
    mask[i] = v;
}

constexpr int kScanBlock = 1024;

__global__ void count_kernel(int num, const int* __restrict__ mask,
        int* __restrict__ block_count)
{
    const int i = blockIdx.x * kScanBlock + threadIdx.x;
    const int v = i < num && mask[i] != 0;
    const int c = __syncthreads_count(v);
    if (threadIdx.x == 0) block_count[blockIdx.x] = c;
}

// Exclusive scan of the block counts (one CTA, sequential over chunks of
// kScanBlock); block_count[num_blocks] receives the total.
__global__ void scan_kernel(int num_blocks, int* __restrict__ block_count)
{
    __shared__ int warp_sums[kScanBlock / 32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < num_blocks; base += kScanBlock)
    {
        const int i = base + threadIdx.x;
        const int v = i < num_blocks ? block_count[i] : 0;
        int x = v;
        for (int d = 1; d < 32; d <<= 1)
        {
            const int y = __shfl_up_sync(0xffffffffu, x, d);
            if ((threadIdx.x & 31) >= d) x += y;
        }
        if ((threadIdx.x & 31) == 31) warp_sums[threadIdx.x >> 5] = x;
        __syncthreads();
        if (threadIdx.x < 32)
        {
            int w = warp_sums[threadIdx.x];
            for (int d = 1; d < 32; d <<= 1)
            {
                const int y = __shfl_up_sync(0xffffffffu, w, d);
                if (threadIdx.x >= d) w += y;
            }
            warp_sums[threadIdx.x] = w;
        }
        __syncthreads();
        const int incl = x + ((threadIdx.x >> 5) ? warp_sums[(threadIdx.x >> 5)
                - 1] : 0);
        if (i < num_blocks) block_count[i] = carry + incl - v;
        __syncthreads();
        if (threadIdx.x == kScanBlock - 1) carry += incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) block_count[num_blocks] = carry;
}

template <typename T>
__global__ void scatter_kernel(int num, const int* __restrict__ mask,
        const int* __restrict__ block_offset, int num_cols,
        const T* const* __restrict__ in, T* const* __restrict__ out)
{
    __shared__ int warp_base[kScanBlock / 32];
    const int i = blockIdx.x * kScanBlock + threadIdx.x;
    const int v = i < num && mask[i] != 0;
    const unsigned bal = __ballot_sync(0xffffffffu, v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) warp_base[w] = __popc(bal);
    __syncthreads();
    if (threadIdx.x == 0)
    {
        int s = 0;
        for (int k = 0; k < kScanBlock / 32; ++k)
        {
            const int c = warp_base[k];
            warp_base[k] = s;
            s += c;
        }
    }
    __syncthreads();
    if (!v) return;
    const int o = block_offset[blockIdx.x] + warp_base[w] +
            __popc(bal & ((1u << lane) - 1u));
    for (int c = 0; c < num_cols; ++c) out[c][o] = in[c][i];
}

template <typename T>
__global__ void baseline_uvw_kernel(int casa, int num, int offset_in,
        const T* __restrict__ u, const T* __restrict__ v,
        const T* __restrict__ w, int offset_out, T* __restrict__ uu,
        T* __restrict__ vv, T* __restrict__ ww)
{
    const int s2 = blockIdx.x * blockDim.x + threadIdx.x;
    const int s1 = blockIdx.y;
    if (s2 <= s1 || s2 >= num) return;
    const T f = casa ? (T) -1 : (T) 1;
    const long long b = (long long) s1 * (num - 1) -
            (long long) (s1 - 1) * s1 / 2 + s2 - s1 - 1 + offset_out;
    uu[b] = f * (u[s2 + offset_in] - u[s1 + offset_in]);
    vv[b] = f * (v[s2 + offset_in] - v[s1 + offset_in]);
    ww[b] = f * (w[s2 + offset_in] - w[s1 + offset_in]);
}

}  // namespace
}  // namespace oskb

extern "C" {

#define OSKB_PREP_ENTRIES(T, S)                                              \
int oskb_convert_lon_lat_to_relative_directions_##S(int num, const T* lon,   \
        const T* lat, double lon0_rad, double lat0_rad, T* l, T* m, T* n,    \
        void* stream)                                                        \
{                                                                            \
    if (num < 0) return OSKB_ERR_INVALID_ARGUMENT;                           \
    if (num == 0) return 0;                                                  \
    if (!lon || !lat || !l || !m) return OSKB_ERR_INVALID_ARGUMENT;          \
    oskb::lonlat_kernel<T><<<(num + 255) / 256, 256, 0,                      \
            oskb::as_stream(stream)>>>(num, lon, lat, (T) lon0_rad,          \
            (T) cos(lat0_rad), (T) sin(lat0_rad), l, m, n);                  \
    return oskb::check_launch("lon_lat_to_relative_directions");            \
}                                                                            \
int oskb_convert_ra_dec_to_enu_directions_##S(int num_sources, const T* ra, \
        const T* dec, int num_stations, const double* lst_rad,               \
        const double* lat_rad, T* x, T* y, T* z, void* stream)               \
{                                                                            \
    if (num_sources < 0 || num_stations < 0 || num_stations > 65535)         \
        return OSKB_ERR_INVALID_ARGUMENT;                                    \
    if (!num_sources || !num_stations) return 0;                             \
    if (!ra || !dec || !lst_rad || !lat_rad || !x || !y || !z)               \
        return OSKB_ERR_INVALID_ARGUMENT;                                    \
    oskb::radec_enu_kernel<T><<<dim3((num_sources + 255) / 256,              \
            num_stations), 256, 0, oskb::as_stream(stream)>>>(num_sources,   \
            ra, dec, lst_rad, lat_rad, x, y, z);                             \
    return oskb::check_launch("ra_dec_to_enu_directions");                  \
}                                                                            \
int oskb_sky_horizon_mask_##S(int num_sources, const T* l, const T* m,       \
        const T* n, int num_stations, const double* ha0_rad_host,            \
        const double* lat_rad_host, double dec0_rad, int* mask,              \
        void* stream)                                                        \
{                                                                            \
    if (num_sources < 0 || num_stations < 0) return OSKB_ERR_INVALID_ARGUMENT;\
    if (!num_sources || !num_stations) return 0;                             \
    if (!l || !m || !n || !ha0_rad_host || !lat_rad_host || !mask)           \
        return OSKB_ERR_INVALID_ARGUMENT;                                    \
    std::vector<T> h(3 * (size_t) num_stations);                             \
    for (int s = 0; s < num_stations; ++s)                                   \
    {                                                                        \
        /* oskar_update_horizon_mask.c:36-43, per station */                 \
        const double ch = cos(ha0_rad_host[s]), sd = sin(dec0_rad);          \
        const double cd = cos(dec0_rad), sl = sin(lat_rad_host[s]);          \
        const double cl = cos(lat_rad_host[s]);                              \
        h[3 * s] = (T) (cl * sin(ha0_rad_host[s]));                          \
        h[3 * s + 1] = (T) (sl * cd - cl * ch * sd);                         \
        h[3 * s + 2] = (T) (sl * sd + cl * ch * cd);                         \
    }                                                                        \
    cudaStream_t st = oskb::as_stream(stream);                               \
    T* d = nullptr;                                                          \
    if (cudaMalloc(&d, sizeof(T) * h.size()) != cudaSuccess ||               \
            cudaMemcpy(d, h.data(), sizeof(T) * h.size(),                    \
            cudaMemcpyHostToDevice) != cudaSuccess)                          \
    {                                                                        \
        oskb::set_last_error("sky_horizon_mask", cudaGetLastError());        \
        cudaFree(d);                                                         \
        return OSKB_ERR_MEMORY_ALLOC_FAILURE;                                \
    }                                                                        \
    oskb::horizon_kernel<T><<<(num_sources + 255) / 256, 256, 0, st>>>(      \
            num_sources, l, m, n, num_stations, d, mask);                    \
    const int err = oskb::check_launch("sky_horizon_mask");                  \
    cudaStreamSynchronize(st);                                               \
    cudaFree(d);                                                             \
    return err;                                                              \
}                                                                            \
int oskb_sky_compact_##S(int num, const int* mask, int num_columns,          \
        const T* const* columns_in, T* const* columns_out, int* num_out,     \
        void* stream)                                                        \
{                                                                            \
    if (num < 0 || num_columns < 0 || !num_out)                              \
        return OSKB_ERR_INVALID_ARGUMENT;                                    \
    *num_out = 0;                                                            \
    if (!num) return 0;                                                      \
    if (!mask || (num_columns && (!columns_in || !columns_out)))             \
        return OSKB_ERR_INVALID_ARGUMENT;                                    \
    cudaStream_t st = oskb::as_stream(stream);                               \
    const int nb = (num + oskb::kScanBlock - 1) / oskb::kScanBlock;          \
    int* offs = nullptr;                                                     \
    const T** cols = nullptr;                                                \
    if (cudaMalloc(&offs, sizeof(int) * (nb + 1)) != cudaSuccess ||          \
            cudaMalloc(&cols, sizeof(T*) * 2 * (num_columns + 1)) !=         \
            cudaSuccess)                                                     \
    {                                                                        \
        oskb::set_last_error("sky_compact", cudaGetLastError());             \
        cudaFree(offs);                                                      \
        return OSKB_ERR_MEMORY_ALLOC_FAILURE;                                \
    }                                                                        \
    std::vector<const T*> hc(2 * (size_t) num_columns + 2);                  \
    for (int c = 0; c < num_columns; ++c)                                    \
    {                                                                        \
        hc[c] = columns_in[c];                                               \
        hc[num_columns + c] = columns_out[c];                                \
    }                                                                        \
    cudaMemcpy(cols, hc.data(), sizeof(T*) * 2 * num_columns,                \
            cudaMemcpyHostToDevice);                                         \
    oskb::count_kernel<<<nb, oskb::kScanBlock, 0, st>>>(num, mask, offs);    \
    oskb::scan_kernel<<<1, oskb::kScanBlock, 0, st>>>(nb, offs);             \
    oskb::scatter_kernel<T><<<nb, oskb::kScanBlock, 0, st>>>(num, mask,      \
            offs, num_columns, cols, (T* const*) (cols + num_columns));      \
    int err = oskb::check_launch("sky_compact");                             \
    if (!err && cudaMemcpyAsync(num_out, offs + nb, sizeof(int),             \
            cudaMemcpyDeviceToHost, st) != cudaSuccess)                      \
        err = OSKB_ERR_MEMORY_COPY_FAILURE;                                  \
    cudaStreamSynchronize(st);                                               \
    cudaFree(offs);                                                          \
    cudaFree(cols);                                                          \
    return err;                                                              \
}                                                                            \
int oskb_convert_station_uvw_to_baseline_uvw_##S(int use_casa, int num,      \
        int offset_in, const T* u, const T* v, const T* w, int offset_out,   \
        T* uu, T* vv, T* ww, void* stream)                                   \
{                                                                            \
    if (num < 0 || num > 65535) return OSKB_ERR_INVALID_ARGUMENT;            \
    if (num < 2) return 0;                                                   \
    if (!u || !v || !w || !uu || !vv || !ww) return OSKB_ERR_INVALID_ARGUMENT;\
    oskb::baseline_uvw_kernel<T><<<dim3((num + 127) / 128, num), 128, 0,     \
            oskb::as_stream(stream)>>>(use_casa, num, offset_in, u, v, w,    \
            offset_out, uu, vv, ww);                                         \
    return oskb::check_launch("station_uvw_to_baseline_uvw");               \
}

OSKB_PREP_ENTRIES(double, d)
OSKB_PREP_ENTRIES(float, f)
#undef OSKB_PREP_ENTRIES

}  // extern "C"

// Weighted DFT of element signals (station beam array pattern).
//
// Replaces the kernels behind oskar_dftw (oskar/math/define_dftw_c2c.h:24-77,
// oskar/math/define_dftw_m2m.h:24-107). One thread per output direction;
// element coordinates, weights and data indices are staged in shared memory
// in chunks of kChunk elements. Each element-direction costs one phase
// (2-3 FMA), one sincos, one complex weight multiply and 1 (c2c) or 4 (m2m)
// complex multiply-adds; the direction's data rows are read through L1 since
// all threads of a warp read consecutive directions.
#include "common.cuh"

namespace oskb {
namespace {

constexpr int kChunk = 512;
constexpr int kThreads = 128;

template <typename T, bool MATRIX, bool IS3D>
__global__ void __launch_bounds__(kThreads)
dftw_kernel(int num_in, T wavenumber, const T* __restrict__ weights_in,
        const T* __restrict__ x_in, const T* __restrict__ y_in,
        const T* __restrict__ z_in, int offset_coord_out, int num_out,
        const T* __restrict__ x_out, const T* __restrict__ y_out,
        const T* __restrict__ z_out, const int* __restrict__ data_idx,
        const T* __restrict__ data, int eval_x, int eval_y, int offset_out,
        T* __restrict__ output, T norm_factor)
{
    typedef typename vec2<T>::type T2;
    __shared__ T2 s_w[kChunk];
    __shared__ T s_x[kChunk], s_y[kChunk], s_z[IS3D ? kChunk : 1];
    __shared__ int s_idx[kChunk];
    const int d = blockIdx.x * kThreads + threadIdx.x;
    const bool active = d < num_out;
    T xo = 0, yo = 0, zo = 0;
    if (active)
    {
        xo = wavenumber * x_out[d + offset_coord_out];
        yo = wavenumber * y_out[d + offset_coord_out];
        if (IS3D) zo = wavenumber * z_out[d + offset_coord_out];
    }
    constexpr int NC = MATRIX ? 4 : 1;
    T2 acc[NC];
#pragma unroll
    for (int k = 0; k < NC; ++k) acc[k].x = acc[k].y = (T) 0;
    const int k0 = (MATRIX && !eval_x) ? 2 : 0;
    const int k1 = MATRIX ? (eval_y ? 4 : 2) : 1;
    const T2* data2 = reinterpret_cast<const T2*>(data);

    for (int e0 = 0; e0 < num_in; e0 += kChunk)
    {
        const int ne = min(kChunk, num_in - e0);
        for (int t = threadIdx.x; t < ne; t += kThreads)
        {
            const int g = e0 + t;
            s_w[t] = reinterpret_cast<const T2*>(weights_in)[g];
            s_x[t] = x_in[g];
            s_y[t] = y_in[g];
            if (IS3D) s_z[t] = z_in[g];
            s_idx[t] = data_idx ? data_idx[g] : g;
        }
        __syncthreads();
        if (active)
        {
            for (int i = 0; i < ne; ++i)
            {
                T ph = xo * s_x[i] + yo * s_y[i];
                if (IS3D) ph += zo * s_z[i];
                T sn, cs;
                sincos(ph, &sn, &cs);
                const T2 w = s_w[i];
                const T re = cs * w.x - w.y * sn;
                const T im = sn * w.x + w.y * cs;
                const size_t base = (size_t) s_idx[i] * num_out + d;
                if (MATRIX)
                {
                    for (int k = k0; k < k1; ++k)
                    {
                        const T2 v = __ldg(&data2[4 * base + k]);
                        acc[k].x += v.x * re - v.y * im;
                        acc[k].y += v.y * re + v.x * im;
                    }
                }
                else
                {
                    const T2 v = __ldg(&data2[base]);
                    acc[0].x += v.x * re - v.y * im;
                    acc[0].y += v.y * re + v.x * im;
                }
            }
        }
        __syncthreads();
    }
    if (!active) return;
    T2* out2 = reinterpret_cast<T2*>(output);
    if (MATRIX)
    {
        for (int k = k0; k < k1; ++k)
            out2[4 * ((size_t) d + offset_out) + k] =
                    T2{acc[k].x * norm_factor, acc[k].y * norm_factor};
    }
    else
    {
        out2[(size_t) d + offset_out] =
                T2{acc[0].x * norm_factor, acc[0].y * norm_factor};
    }
}

template <typename T>
int dftw(int matrix, int num_in, T wavenumber, const T* weights_in,
        const T* x_in, const T* y_in, const T* z_in, int offset_coord_out,
        int num_out, const T* x_out, const T* y_out, const T* z_out,
        const int* data_idx, const T* data, int eval_x, int eval_y,
        int offset_out, T* output, T norm_factor, void* stream)
{
    if (num_in < 0 || num_out < 0) return OSKB_ERR_INVALID_ARGUMENT;
    if (num_out == 0) return 0;
    if (!weights_in || !x_in || !y_in || !x_out || !y_out || !data ||
            !output)
        return OSKB_ERR_INVALID_ARGUMENT;
    const bool is3d = (z_in != nullptr && z_out != nullptr);
    const int grid = (num_out + kThreads - 1) / kThreads;
    cudaStream_t s = as_stream(stream);
#define OSKB_DFTW(M, D) dftw_kernel<T, M, D><<<grid, kThreads, 0, s>>>(       \
        num_in, wavenumber, weights_in, x_in, y_in, z_in, offset_coord_out,  \
        num_out, x_out, y_out, z_out, data_idx, data, eval_x, eval_y,        \
        offset_out, output, norm_factor)
    if (matrix) { if (is3d) OSKB_DFTW(true, true); else OSKB_DFTW(true, false); }
    else { if (is3d) OSKB_DFTW(false, true); else OSKB_DFTW(false, false); }
#undef OSKB_DFTW
    return check_launch("dftw");
}

}  // namespace
}  // namespace oskb

extern "C" {

int oskb_dftw_d(int matrix, int num_in, double wavenumber,
        const double* weights_in, const double* x_in, const double* y_in,
        const double* z_in, int offset_coord_out, int num_out,
        const double* x_out, const double* y_out, const double* z_out,
        const int* data_idx, const double* data, int eval_x, int eval_y,
        int offset_out, double* output, double norm_factor, void* stream)
{
    return oskb::dftw<double>(matrix, num_in, wavenumber, weights_in, x_in,
            y_in, z_in, offset_coord_out, num_out, x_out, y_out, z_out,
            data_idx, data, eval_x, eval_y, offset_out, output, norm_factor,
            stream);
}

int oskb_dftw_f(int matrix, int num_in, float wavenumber,
        const float* weights_in, const float* x_in, const float* y_in,
        const float* z_in, int offset_coord_out, int num_out,
        const float* x_out, const float* y_out, const float* z_out,
        const int* data_idx, const float* data, int eval_x, int eval_y,
        int offset_out, float* output, float norm_factor, void* stream)
{
    return oskb::dftw<float>(matrix, num_in, wavenumber, weights_in, x_in,
            y_in, z_in, offset_coord_out, num_out, x_out, y_out, z_out,
            data_idx, data, eval_x, eval_y, offset_out, output, norm_factor,
            stream);
}

}  // extern "C"

// Weighted DFT of element signals (station beam array pattern).
//
// Replaces the kernels behind oskar_dftw (oskar/math/define_dftw_c2c.h:24-77,
// oskar/math/define_dftw_m2m.h:24-107). One thread per output direction;
// element coordinates, weights and data indices are staged in shared memory
// in chunks of kChunk elements. Each element-direction costs one phase
// (2-3 FMA), one sincos, one complex weight multiply and 1 (c2c) or 4 (m2m)
// complex multiply-adds; the direction's data rows are read through L1 since
// all threads of a warp read consecutive directions.
//
// A station beam has a few thousand to a few tens of thousands of
// directions, which at one thread per direction leaves most of the 148 SMs
// idle. When the direction grid is small the elements are split into
// `slices` contiguous ranges, one per CTA of a thread-block cluster
// (gridDim.y == cluster height); each CTA sums its range and CTA 0 of the
// cluster adds the partial sums from the others' shared memory in rank
// order, so the result does not depend on scheduling. The accumulators are
// fully unrolled with the eval_x/eval_y selection as a predicate so they
// stay in registers. In FP64 the phase factors come from a shared-memory
// table (trig_table.cuh) instead of a library sincos per element-direction.
#include "trig_table.cuh"

#include <algorithm>
#include <cooperative_groups.h>

namespace oskb {
namespace {

namespace cg = cooperative_groups;

constexpr int kChunk = 256;
constexpr int kThreads = 128;
constexpr int kMaxSlices = 8;      // portable cluster size
constexpr int kMinSliceElements = 16;
constexpr int kTableMinElements = 64;

// acc[k] += w e^{i ph} data[idx][d][k] for the evaluated k.
template <typename T, int NC>
__device__ __forceinline__ void accumulate(typename vec2<T>::type* acc,
        const typename vec2<T>::type* __restrict__ data2,
        typename vec2<T>::type w, int idx, int num_out, int d, int k0,
        int k1, T sn, T cs)
{
    const T re = cs * w.x - w.y * sn;
    const T im = sn * w.x + w.y * cs;
    const size_t base = (size_t) idx * num_out + d;
#pragma unroll
    for (int k = 0; k < NC; ++k)
    {
        if (k < k0 || k >= k1) continue;
        const typename vec2<T>::type v = __ldg(&data2[(size_t) NC * base + k]);
        acc[k].x += v.x * re - v.y * im;
        acc[k].y += v.y * re + v.x * im;
    }
}

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
    constexpr int NC = MATRIX ? 4 : 1;
    __shared__ T2 s_w[kChunk];
    __shared__ T s_x[kChunk], s_y[kChunk], s_z[IS3D ? kChunk : 1];
    __shared__ int s_idx[kChunk];
    __shared__ double2 s_trig[sizeof(T) == 8 ? kTrigTableSize : 1];
    const int d = blockIdx.x * kThreads + threadIdx.x;
    const bool active = d < num_out;
    T xo = 0, yo = 0, zo = 0;
    if (active)
    {
        // radians in FP32, table steps (radians x 64 / pi) in FP64
        const T k = sizeof(T) == 8 ? (T) (wavenumber * kTrigStepsPerRadian)
                                   : wavenumber;
        xo = k * x_out[d + offset_coord_out];
        yo = k * y_out[d + offset_coord_out];
        if (IS3D) zo = k * z_out[d + offset_coord_out];
    }
    T2 acc[NC];
#pragma unroll
    for (int k = 0; k < NC; ++k) acc[k].x = acc[k].y = (T) 0;
    const int k0 = (MATRIX && !eval_x) ? 2 : 0;
    const int k1 = MATRIX ? (eval_y ? 4 : 2) : 1;
    const T2* data2 = reinterpret_cast<const T2*>(data);

    // this CTA's element range
    const int slices = gridDim.y;
    const int per = (num_in + slices - 1) / slices;
    const int lo = min(num_in, (int) blockIdx.y * per);
    const int hi = min(num_in, lo + per);
    // The table costs 128 sincospi per CTA: worth it from about 64 elements.
    const bool use_table = sizeof(T) == 8 && hi - lo >= kTableMinElements;
    if (use_table) trig_table_fill(s_trig);  // synced in the chunk loop
    for (int e0 = lo; e0 < hi; e0 += kChunk)
    {
        const int ne = min(kChunk, hi - e0);
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
            if constexpr (sizeof(T) == 8)
            {
                bool exact = !use_table;
                if (use_table)
                {
                    // Branch-free table loop; a thread that met a phase
                    // the table does not cover redoes the chunk exactly.
                    T2 acc0[NC];
#pragma unroll
                    for (int k = 0; k < NC; ++k) acc0[k] = acc[k];
                    bool covered = true;
#pragma unroll 2
                    for (int i = 0; i < ne; ++i)
                    {
                        T ph = xo * s_x[i] + yo * s_y[i];
                        if (IS3D) ph += zo * s_z[i];
                        T sn, cs;
                        trig_steps_sincos(s_trig, ph, &sn, &cs, covered);
                        accumulate<T, NC>(acc, data2, s_w[i], s_idx[i],
                                num_out, d, k0, k1, sn, cs);
                    }
                    if (!covered)
                    {
#pragma unroll
                        for (int k = 0; k < NC; ++k) acc[k] = acc0[k];
                        exact = true;
                    }
                }
                if (exact)
                {
                    for (int i = 0; i < ne; ++i)
                    {
                        T ph = xo * s_x[i] + yo * s_y[i];
                        if (IS3D) ph += zo * s_z[i];
                        T sn, cs;
                        trig_steps_exact(ph, &sn, &cs);
                        accumulate<T, NC>(acc, data2, s_w[i], s_idx[i],
                                num_out, d, k0, k1, sn, cs);
                    }
                }
            }
            else
            {
                for (int i = 0; i < ne; ++i)
                {
                    T ph = xo * s_x[i] + yo * s_y[i];
                    if (IS3D) ph += zo * s_z[i];
                    T sn, cs;
                    sincosf(ph, &sn, &cs);
                    accumulate<T, NC>(acc, data2, s_w[i], s_idx[i], num_out,
                            d, k0, k1, sn, cs);
                }
            }
        }
        __syncthreads();
    }
    if (slices > 1)
    {
        // partial sums of the cluster's CTAs, added in rank order by rank 0
        __shared__ T2 s_part[NC][kThreads];
#pragma unroll
        for (int k = 0; k < NC; ++k) s_part[k][threadIdx.x] = acc[k];
        cg::cluster_group cluster = cg::this_cluster();
        cluster.sync();
        if (blockIdx.y == 0)
        {
            for (int r = 1; r < slices; ++r)
            {
                const T2* p = cluster.map_shared_rank(&s_part[0][0], r);
#pragma unroll
                for (int k = 0; k < NC; ++k)
                {
                    const T2 v = p[k * kThreads + threadIdx.x];
                    acc[k].x += v.x;
                    acc[k].y += v.y;
                }
            }
        }
        // keep every CTA's shared memory alive until rank 0 has read it
        cluster.sync();
        if (blockIdx.y != 0) return;
    }
    if (!active) return;
    T2* out2 = reinterpret_cast<T2*>(output);
#pragma unroll
    for (int k = 0; k < NC; ++k)
    {
        if (k < k0 || k >= k1) continue;
        out2[(size_t) NC * ((size_t) d + offset_out) + k] =
                T2{acc[k].x * norm_factor, acc[k].y * norm_factor};
    }
}

int num_sms() { return device_sm_count(); }

// Number of element slices: grow the cluster while the direction grid is
// below about 8 CTAs (32 warps) per SM and each slice keeps at least
// kMinSliceElements elements.
int choose_slices(int num_in, int blocks_x)
{
    const long long target = 8LL * num_sms();
    int s = 1;
    while (s < kMaxSlices && (long long) blocks_x * s < target &&
            num_in / (2 * s) >= kMinSliceElements)
        s *= 2;
    return s;
}

template <typename T, bool MATRIX, bool IS3D>
int launch_dftw(int slices, int blocks_x, cudaStream_t s, int num_in,
        T wavenumber, const T* weights_in, const T* x_in, const T* y_in,
        const T* z_in, int offset_coord_out, int num_out, const T* x_out,
        const T* y_out, const T* z_out, const int* data_idx, const T* data,
        int eval_x, int eval_y, int offset_out, T* output, T norm_factor)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks_x, slices, 1);
    cfg.blockDim = dim3(kThreads, 1, 1);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 1;
    attr[0].val.clusterDim.y = slices;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = slices > 1 ? 1 : 0;
    cudaError_t e = cudaLaunchKernelEx(&cfg, dftw_kernel<T, MATRIX, IS3D>,
            num_in, wavenumber, weights_in, x_in, y_in, z_in,
            offset_coord_out, num_out, x_out, y_out, z_out, data_idx, data,
            eval_x, eval_y, offset_out, output, norm_factor);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        set_last_error("dftw", e);
        return OSKB_ERR_KERNEL_LAUNCH_FAILURE;
    }
    return check_launch("dftw");
}

__global__ void __launch_bounds__(kThreads) phase_factors_kernel(int n,
        const double* __restrict__ steps, double2* __restrict__ out)
{
    __shared__ double2 s_trig[kTrigTableSize];
    trig_table_fill(s_trig);
    __syncthreads();
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n;
            i += gridDim.x * kThreads)
    {
        double s, c;
        trig_steps_checked(s_trig, steps[i], &s, &c);
        out[i] = make_double2(c, s);
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
    const int blocks_x = (num_out + kThreads - 1) / kThreads;
    const int slices = choose_slices(num_in, blocks_x);
    cudaStream_t s = as_stream(stream);
#define OSKB_DFTW(M, D) return launch_dftw<T, M, D>(slices, blocks_x, s,      \
        num_in, wavenumber, weights_in, x_in, y_in, z_in, offset_coord_out,  \
        num_out, x_out, y_out, z_out, data_idx, data, eval_x, eval_y,        \
        offset_out, output, norm_factor)
    if (matrix) { if (is3d) OSKB_DFTW(true, true); else OSKB_DFTW(true, false); }
    else { if (is3d) OSKB_DFTW(false, true); else OSKB_DFTW(false, false); }
#undef OSKB_DFTW
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

int oskb_phase_factors_d(int n, const double* steps, double* out,
        void* stream)
{
    if (n < 0) return OSKB_ERR_INVALID_ARGUMENT;
    if (n == 0) return 0;
    if (!steps || !out) return OSKB_ERR_INVALID_ARGUMENT;
    const int grid = (int) std::min<long long>(
            (n + oskb::kThreads - 1) / oskb::kThreads,
            8LL * oskb::num_sms());
    oskb::phase_factors_kernel<<<grid, oskb::kThreads, 0,
            oskb::as_stream(stream)>>>(n, steps,
            reinterpret_cast<double2*>(out));
    return oskb::check_launch("phase_factors");
}

}  // extern "C"

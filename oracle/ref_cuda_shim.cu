// The reference's own GPU weighted-DFT kernels (math/define_dftw_m2m.h,
// math/define_dftw_c2c.h, instantiated here under exported names) with a
// launcher that sizes the launch as the reference's oskar_dftw does
// (math/src/oskar_dftw.c:34-40, 303-371: blocks of up to 256 threads, one
// output per thread, 256-element input chunks staged in dynamic shared
// memory). TEST INFRASTRUCTURE ONLY: the GPU baseline and a GPU parity pin
// for the station-beam DFT; nothing in the product links it. Built by
// `make -C oracle ref_cuda` together with the reference's CUDA
// cross-correlation sources.
#include <cuda_runtime.h>

#include "utility/oskar_kernel_macros.h"
#include "utility/oskar_vector_types.h"
// the reference registers its kernels with a run-time table; not needed here
#define OSKAR_CUDA_KERNEL(NAME)
#include "math/define_dftw_c2c.h"
#include "math/define_dftw_m2m.h"

OSKAR_DFTW_M2M_GPU(ref_k_dftw_m2m_2d_double, 0, double, double2)
OSKAR_DFTW_M2M_GPU(ref_k_dftw_m2m_3d_double, 1, double, double2)
OSKAR_DFTW_M2M_GPU(ref_k_dftw_m2m_2d_float, 0, float, float2)
OSKAR_DFTW_M2M_GPU(ref_k_dftw_m2m_3d_float, 1, float, float2)
OSKAR_DFTW_C2C_GPU(ref_k_dftw_c2c_2d_double, 0, double, double2)
OSKAR_DFTW_C2C_GPU(ref_k_dftw_c2c_3d_double, 1, double, double2)
OSKAR_DFTW_C2C_GPU(ref_k_dftw_c2c_2d_float, 0, float, float2)
OSKAR_DFTW_C2C_GPU(ref_k_dftw_c2c_3d_float, 1, float, float2)

namespace {

const int kMaxInChunk = 256;

int block_size(int num_out)
{
    const int b = (num_out + 31) / 32 * 32;
    return b > 256 ? 256 : (b < 32 ? 32 : b);
}

// Dynamic shared memory in the order the kernel carves it: weights (FP2),
// coordinates (FP2), indices (int), z (FP, 3-D only).
size_t smem_bytes(size_t fp, int is_3d)
{
    return kMaxInChunk * (4 * fp + sizeof(int) + (is_3d ? fp : 0));
}

}  // namespace

#define REF_DFTW_LAUNCHER(S, FP, FP2)                                        \
extern "C" int ref_cuda_dftw_##S(int matrix, int is_3d, int num_in,          \
        FP wavenumber, const FP* weights_in, const FP* x_in,                 \
        const FP* y_in, const FP* z_in, int offset_coord_out, int num_out,   \
        const FP* x_out, const FP* y_out, const FP* z_out,                   \
        const int* data_idx, const FP* data, int eval_x, int eval_y,         \
        int offset_out, FP* output, FP norm_factor, void* stream)            \
{                                                                            \
    if (num_out <= 0) return 0;                                              \
    const int block = block_size(num_out);                                   \
    const int grid = (num_out + block - 1) / block;                          \
    const size_t smem = smem_bytes(sizeof(FP), is_3d);                       \
    cudaStream_t s = (cudaStream_t) stream;                                  \
    const FP2* w = (const FP2*) weights_in;                                  \
    const FP2* d = (const FP2*) data;                                        \
    FP2* o = (FP2*) output;                                                  \
    if (matrix && is_3d)                                                     \
        ref_k_dftw_m2m_3d_##S<<<grid, block, smem, s>>>(num_in, wavenumber,  \
                w, x_in, y_in, z_in, offset_coord_out, num_out, x_out,       \
                y_out, z_out, data_idx, d, eval_x, eval_y, offset_out, o,    \
                norm_factor, kMaxInChunk);                                   \
    else if (matrix)                                                         \
        ref_k_dftw_m2m_2d_##S<<<grid, block, smem, s>>>(num_in, wavenumber,  \
                w, x_in, y_in, 0, offset_coord_out, num_out, x_out, y_out,   \
                0, data_idx, d, eval_x, eval_y, offset_out, o, norm_factor,  \
                kMaxInChunk);                                                \
    else if (is_3d)                                                          \
        ref_k_dftw_c2c_3d_##S<<<grid, block, smem, s>>>(num_in, wavenumber,  \
                w, x_in, y_in, z_in, offset_coord_out, num_out, x_out,       \
                y_out, z_out, data_idx, d, eval_x, eval_y, offset_out, o,    \
                norm_factor, kMaxInChunk);                                   \
    else                                                                     \
        ref_k_dftw_c2c_2d_##S<<<grid, block, smem, s>>>(num_in, wavenumber,  \
                w, x_in, y_in, 0, offset_coord_out, num_out, x_out, y_out,   \
                0, data_idx, d, eval_x, eval_y, offset_out, o, norm_factor,  \
                kMaxInChunk);                                                \
    return (int) cudaGetLastError();                                         \
}

REF_DFTW_LAUNCHER(double, double, double2)
REF_DFTW_LAUNCHER(float, float, float2)

// The reference's GPU beam-pattern cross-power kernel
// (correlate/define_evaluate_cross_power.h, instantiated for CUDA by
// correlate/src/oskar_evaluate_cross_power.c:41-42) with the reference's
// launch: one thread per source, blocks of 64 (FP64) or 128 (FP32)
// threads (oskar_evaluate_cross_power.c:109-131).
#include "math/define_multiply.h"
#include "correlate/define_correlate_utils.h"
#include "correlate/define_evaluate_cross_power.h"

OSKAR_CROSS_POWER_MATRIX(ref_k_cross_power_double, double, double2, double4c)
OSKAR_CROSS_POWER_MATRIX(ref_k_cross_power_float, float, float2, float4c)

#define REF_CROSS_POWER_LAUNCHER(S, FP, FP4c, BLOCK)                          \
extern "C" int ref_cuda_cross_power_##S(int num_sources, int num_stations,  \
        const void* jones, FP src_I, FP src_Q, FP src_U, FP src_V, FP norm,  \
        int offset_out, void* out, void* stream)                             \
{                                                                            \
    if (num_sources <= 0) return 0;                                          \
    const int grid = (num_sources + BLOCK - 1) / BLOCK;                      \
    ref_k_cross_power_##S<<<grid, BLOCK, 0, (cudaStream_t) stream>>>(        \
            num_sources, num_stations, (const FP4c*) jones, src_I, src_Q,    \
            src_U, src_V, norm, offset_out, (FP4c*) out);                    \
    return (int) cudaGetLastError();                                         \
}
REF_CROSS_POWER_LAUNCHER(double, double, double4c, 64)
REF_CROSS_POWER_LAUNCHER(float, float, float4c, 128)

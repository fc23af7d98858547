// Internal interface of the tensor-core block correlation, shared by the
// device-buffer entry point (xcorr_tc.cu) and the host-buffer driver
// (block_host.cu).
#pragma once

namespace oskb {
namespace tc {

// Contraction forms; kFormDefault follows the environment (OSKB_TC_ARITH,
// OSKB_TC_TILE), the others fix the form (2 is not a form).
enum Form
{
    kFormDefault = 0,
    kFormI8 = 1,        // integer, 128 x 128 tiles
    kFormF16 = 3,       // FP16 hi/lo, 128 x 128 tiles
    kFormF16Wide = 4,   // FP16 hi/lo, 128 x 256 tiles
    kFormF16Pair = 5    // FP16 hi/lo, 256 x 256 tiles on CTA pairs
};

// oskb_correlate_block_tc with a hook: after_group (if set) is called on the
// host once the contraction of problems [p0, p0 + np) has been enqueued on
// the stream, so the caller can enqueue work that depends on those
// visibilities (for example their download) while later groups compute;
// autos (if set) receives the auto-correlations from the same contraction
// ([time][channel][station][2x2], added). E is FP32 or FP64 (float or
// double instantiations); form fixes the contraction form.
template <typename TE>
int correlate_block(int casa, int num_sources, int num_stations,
        int num_times, int num_channels, const TE* E, const double* l,
        const double* m, const double* n, const double* I, const double* Q,
        const double* U, const double* V, const double* station_uvw,
        const double* inv_wavelength, double uv_min_lambda,
        double uv_max_lambda, double* vis, void* workspace,
        size_t workspace_bytes, void* stream,
        void (*after_group)(void* ctx, int p0, int np), void* ctx,
        double* autos = nullptr, int form = kFormDefault);

// The per-device launch set-up of the contraction kernels (shared-memory
// opt-ins), done before a stream capture so that none happens inside it.
int setup_device();

}  // namespace tc
}  // namespace oskb

// Learned station-beam surrogate: array-factor training samples, and the
// station beam with the array factor taken from a per-station-type network
// outside a main-lobe radius, audited against the exact sum.
//
// For a planar station whose elements share one pattern and whose weights
// phase it to the pointing b (oskar_station_evaluate_element_weights.c:
// 25-31 without cable errors), the array factor in direction d is
//     AF(d) = (1/N) sum_e exp(i k r_e . (d - b)) = A(kappa),
//     kappa = k (d - b) projected on the station plane,
// a function of two variables per station layout. Stations of one type are
// the same layout rotated by an angle; in the station frame they share A.
// So one network per type learns A(kappa) (two inputs, complex output); the
// element pattern stays analytic. The beam is
//     E(d) = s_final * s_elem * P(d) * A(kappa(d)),
// with P the dipole pattern, s_elem the element normalisation at the pole,
// and s_final = 1 / |E(b)| (the normalisation direction is the pointing,
// where A = 1 exactly), blanked below the horizon - the composition of
// oskar_station_beam / oskar_evaluate_station_beam_aperture_array for such
// stations (see beam.cu).
//
// Evaluation of one block (oskb_station_beam_surrogate_f):
//  1. classify: each (station, direction) inside |kappa| < kappa_main (the
//     main lobe) or below the horizon gets the exact A; every other one is
//     queued for its type's network with features kappa / kappa_scale;
//  2. the networks run over their queues (oskb_mlp_infer);
//  3. audit: every audit_stride-th queued entry is recomputed exactly; the
//     largest |A_net - A_exact| (A is 1 at the pointing) is the block's
//     audit error. Above the bound, every queued entry is recomputed exactly
//     (the fallback), so the block is exact;
//  4. assemble the beam.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "beam_common.cuh"

struct oskb_Mlp;
extern "C" int oskb_mlp_infer(oskb_Mlp* n, long long count, const float* x,
        float* y, int chunk, void* stream);

namespace oskb {
namespace {

constexpr int kThreads = 256;

// Exact normalised array factor for station-frame kappa (rad/m), FP64
// phases, from the layout (ex, ey) of num_el elements.
__device__ __forceinline__ float2 array_factor(int num_el,
        const float* __restrict__ ex, const float* __restrict__ ey,
        double kx, double ky)
{
    double re = 0, im = 0;
    for (int e = 0; e < num_el; ++e)
    {
        double s, c;
        sincos(kx * (double) ex[e] + ky * (double) ey[e], &s, &c);
        re += c;
        im += s;
    }
    return make_float2((float) (re / num_el), (float) (im / num_el));
}

__global__ void af_samples_kernel(int num_el, const float* __restrict__ ex,
        const float* __restrict__ ey, long long count,
        const float* __restrict__ kx, const float* __restrict__ ky,
        float* __restrict__ af)
{
    const long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float2 a = array_factor(num_el, ex, ey, kx[i], ky[i]);
    af[2 * i] = a.x;
    af[2 * i + 1] = a.y;
}

struct SurrogateArgs
{
    int num_st, num_dir, num_types, num_el;
    const int* station_type;       // [station]
    const double* rotation;        // [station] rad
    const float* layout_x;         // [type][element] station frame
    const float* layout_y;
    const double* beam_enu;        // [station][3]
    const float *dx, *dy, *dz;     // [station][direction]
    double wavenumber, kappa_main, kappa_scale;
    float2* af;                    // [station][direction]
    int* queue_count;              // [type]
    int* queue_index;              // [type][capacity] -> st * num_dir + d
    float* queue_x;                // [type][capacity][2]
    long long capacity;
};

__device__ __forceinline__ void station_kappa(const SurrogateArgs& a, int st,
        float X, float Y, double& kx, double& ky)
{
    const double ex = a.wavenumber * ((double) X - a.beam_enu[3 * st]);
    const double ey = a.wavenumber * ((double) Y - a.beam_enu[3 * st + 1]);
    double s, c;
    sincos(a.rotation[st], &s, &c);
    // rotate by -rotation into the station (layout) frame
    kx = c * ex + s * ey;
    ky = -s * ex + c * ey;
}

__global__ void classify_kernel(SurrogateArgs a)
{
    const long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if (i >= (long long) a.num_st * a.num_dir) return;
    const int st = (int) (i / a.num_dir);
    const int type = a.station_type[st];
    const float X = a.dx[i], Y = a.dy[i], Z = a.dz[i];
    double kx, ky;
    station_kappa(a, st, X, Y, kx, ky);
    const bool main_lobe = kx * kx + ky * ky < a.kappa_main * a.kappa_main;
    if (Z < 0.f)
    {
        a.af[i] = make_float2(0.f, 0.f);  // blanked anyway
        return;
    }
    if (main_lobe)
    {
        a.af[i] = array_factor(a.num_el, a.layout_x + (size_t) type *
                a.num_el, a.layout_y + (size_t) type * a.num_el, kx, ky);
        return;
    }
    const int slot = atomicAdd(&a.queue_count[type], 1);
    if (slot >= a.capacity) return;  // cannot happen: capacity = all entries
    const size_t q = (size_t) type * a.capacity + slot;
    a.queue_index[q] = (int) i;
    a.queue_x[2 * q] = (float) (kx / a.kappa_scale);
    a.queue_x[2 * q + 1] = (float) (ky / a.kappa_scale);
}

// Scatters network outputs; for every stride-th entry (or every entry when
// exact_all) computes the exact A and, for audited entries, the error.
__global__ void scatter_audit_kernel(SurrogateArgs a, int type, int count,
        const float* __restrict__ y, int stride, int exact_all,
        unsigned int* __restrict__ max_err_bits, double* __restrict__ sum_sq,
        int* __restrict__ num_audited)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) return;
    const size_t q = (size_t) type * a.capacity + j;
    const long long i = a.queue_index[q];
    float2 v = make_float2(y[2 * j], y[2 * j + 1]);
    const bool audit = stride > 0 && j % stride == 0;
    if (audit || exact_all)
    {
        const int st = (int) (i / a.num_dir);
        double kx, ky;
        station_kappa(a, st, a.dx[i], a.dy[i], kx, ky);
        const float2 e = array_factor(a.num_el, a.layout_x + (size_t) type *
                a.num_el, a.layout_y + (size_t) type * a.num_el, kx, ky);
        if (audit)
        {
            const float err = hypotf(v.x - e.x, v.y - e.y);
            atomicMax(max_err_bits, __float_as_uint(err));
            atomicAdd(sum_sq, (double) err * err);
            atomicAdd(num_audited, 1);
        }
        if (exact_all) v = e;
    }
    a.af[i] = v;
}

// E = s_final s_elem P(d) A, blanked below the horizon.
template <bool NORM_ELEMENT>
__global__ void assemble_kernel(SurrogateArgs a, float kL, float cos_kL,
        float* __restrict__ beam)
{
    const long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if (i >= (long long) a.num_st * a.num_dir) return;
    const int st = (int) (i / a.num_dir);
    // The station's dipoles turn with it: both element Euler angles equal
    // the station rotation, so (as in beam.cu) dphi1 = -rot and
    // dphi2 = pi/2 - rot.
    const double rot = a.rotation[st];
    const float dphi1 = (float) (kPi / 2 - (rot + kPi / 2));
    const float dphi2 = (float) (kPi / 2 - rot);
    float p[4], pb[4], pp[4];
    element_pattern<float>(a.dx[i], a.dy[i], a.dz[i], false, dphi1, dphi2,
            kL, cos_kL, 0, p);
    element_pattern<float>((float) a.beam_enu[3 * st],
            (float) a.beam_enu[3 * st + 1], (float) a.beam_enu[3 * st + 2],
            false, dphi1, dphi2, kL, cos_kL, 0, pb);
    float s_elem = 1.f;
    if (NORM_ELEMENT)
    {
        element_pattern<float>(0.f, 0.f, 1.f, true, dphi1, dphi2, kL, cos_kL,
                0, pp);
        s_elem = 1.f / sqrtf((pp[0] * pp[0] + pp[1] * pp[1] + pp[2] * pp[2] +
                pp[3] * pp[3]) / 2.f);
    }
    // final normalisation: |E(b)| with A(b) = 1
    const float nb = sqrtf((pb[0] * pb[0] + pb[1] * pb[1] + pb[2] * pb[2] +
            pb[3] * pb[3]) * s_elem * s_elem / 2.f);
    const float s = s_elem / nb;
    const float2 A = a.af[i];
    float* o = beam + 8 * i;
    const bool blank = a.dz[i] < 0.f;
    for (int k = 0; k < 4; ++k)
    {
        o[2 * k] = blank ? 0.f : p[k] * s * A.x;
        o[2 * k + 1] = blank ? 0.f : p[k] * s * A.y;
    }
}

}  // namespace
}  // namespace oskb

extern "C" {

int oskb_array_factor_samples_f(int num_elements, const float* layout_x,
        const float* layout_y, long long count, const float* kappa_x,
        const float* kappa_y, float* af, void* stream)
{
    if (num_elements < 1 || count < 0) return OSKB_ERR_INVALID_ARGUMENT;
    if (count == 0) return 0;
    if (!layout_x || !layout_y || !kappa_x || !kappa_y || !af)
        return OSKB_ERR_INVALID_ARGUMENT;
    oskb::af_samples_kernel<<<(unsigned) ((count + 255) / 256), 256, 0,
            oskb::as_stream(stream)>>>(num_elements, layout_x, layout_y,
            count, kappa_x, kappa_y, af);
    return oskb::check_launch("oskb_array_factor_samples_f");
}

int oskb_station_beam_surrogate_f(int num_stations, int num_types,
        int num_elements, const int* station_type_host,
        const double* rotation_rad, const float* layout_x,
        const float* layout_y, oskb_Mlp* const* networks,
        double dipole_length_m, int normalise_element, double frequency_hz,
        const double* beam_enu, int num_directions, const float* x,
        const float* y, const float* z, double kappa_main,
        double kappa_scale, int audit_stride, double audit_bound,
        float* beam, double* audit, void* stream)
{
    using namespace oskb;
    if (num_stations < 0 || num_directions < 0 || num_types < 1 ||
            num_elements < 1)
        return OSKB_ERR_INVALID_ARGUMENT;
    if (num_stations == 0 || num_directions == 0) return 0;
    if (!station_type_host || !rotation_rad || !layout_x || !layout_y ||
            !networks || !beam_enu || !x || !y || !z || !beam ||
            kappa_scale <= 0)
        return OSKB_ERR_INVALID_ARGUMENT;
    cudaStream_t s = as_stream(stream);
    const long long total = (long long) num_stations * num_directions;
    // Per-type queue capacity: stations of that type x directions.
    std::vector<long long> per_type(num_types, 0);
    for (int st = 0; st < num_stations; ++st)
    {
        const int t = station_type_host[st];
        if (t < 0 || t >= num_types || !networks[t])
            return OSKB_ERR_INVALID_ARGUMENT;
        per_type[t] += num_directions;
    }
    long long cap = 0;
    for (long long c : per_type) cap = c > cap ? c : cap;
    // Workspace (stream-ordered): A per entry, queues, counters, audit.
    SurrogateArgs a;
    a.num_st = num_stations; a.num_dir = num_directions;
    a.num_types = num_types; a.num_el = num_elements;
    a.rotation = rotation_rad; a.layout_x = layout_x; a.layout_y = layout_y;
    a.beam_enu = beam_enu; a.dx = x; a.dy = y; a.dz = z;
    a.wavenumber = 2.0 * kPi * frequency_hz / 299792458.0;
    a.kappa_main = kappa_main; a.kappa_scale = kappa_scale;
    a.capacity = cap;
    int* d_type = nullptr;
    float* queue_y = nullptr;
    unsigned char* stats = nullptr;  // max bits, count, sum_sq
    const size_t qn = (size_t) num_types * cap;
    bool ok = scratch_alloc((void**) &d_type, sizeof(int) * num_stations,
            s) == cudaSuccess &&
            scratch_alloc((void**) &a.af, sizeof(float2) * total, s) ==
            cudaSuccess &&
            scratch_alloc((void**) &a.queue_count, sizeof(int) * num_types,
            s) == cudaSuccess &&
            scratch_alloc((void**) &a.queue_index, sizeof(int) * qn, s) ==
            cudaSuccess &&
            scratch_alloc((void**) &a.queue_x, sizeof(float) * 2 * qn, s) ==
            cudaSuccess &&
            scratch_alloc((void**) &queue_y, sizeof(float) * 2 * qn, s) ==
            cudaSuccess &&
            scratch_alloc((void**) &stats, 16, s) == cudaSuccess;
    int err = 0;
    if (!ok)
    {
        set_last_error("oskb_station_beam_surrogate_f", cudaGetLastError());
        err = OSKB_ERR_MEMORY_ALLOC_FAILURE;
    }
    a.station_type = d_type;
    unsigned int* max_bits = (unsigned int*) stats;
    int* n_aud = (int*) (stats + 4);
    double* sum_sq = (double*) (stats + 8);
    std::vector<int> counts(num_types, 0);
    if (!err)
    {
        cudaMemcpyAsync(d_type, station_type_host, sizeof(int) * num_stations,
                cudaMemcpyHostToDevice, s);
        cudaMemsetAsync(a.queue_count, 0, sizeof(int) * num_types, s);
        cudaMemsetAsync(stats, 0, 16, s);
        classify_kernel<<<(unsigned) ((total + kThreads - 1) / kThreads),
                kThreads, 0, s>>>(a);
        err = check_launch("surrogate classify");
        if (!err)
        {
            cudaMemcpyAsync(counts.data(), a.queue_count,
                    sizeof(int) * num_types, cudaMemcpyDeviceToHost, s);
            if (cudaStreamSynchronize(s) != cudaSuccess)
            {
                set_last_error("surrogate", cudaGetLastError());
                err = OSKB_ERR_KERNEL_LAUNCH_FAILURE;
            }
        }
    }
    // Networks over their queues, then scatter with the audit.
    for (int t = 0; t < num_types && !err; ++t)
    {
        if (!counts[t]) continue;
        const size_t q0 = (size_t) t * cap;
        err = oskb_mlp_infer(networks[t], counts[t], a.queue_x + 2 * q0,
                queue_y + 2 * q0, 1 << 18, stream);
        if (!err)
        {
            scatter_audit_kernel<<<(counts[t] + kThreads - 1) / kThreads,
                    kThreads, 0, s>>>(a, t, counts[t], queue_y + 2 * q0,
                    audit_stride, 0, max_bits, sum_sq, n_aud);
            err = check_launch("surrogate scatter");
        }
    }
    double max_err = 0, rms = 0;
    int n_audited = 0, fallback = 0;
    if (!err)
    {
        unsigned char h[16];
        cudaMemcpyAsync(h, stats, 16, cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess)
        {
            set_last_error("surrogate", cudaGetLastError());
            err = OSKB_ERR_KERNEL_LAUNCH_FAILURE;
        }
        unsigned int mb;
        double ss;
        memcpy(&mb, h, 4);
        memcpy(&n_audited, h + 4, 4);
        memcpy(&ss, h + 8, 8);
        float mf;
        memcpy(&mf, &mb, 4);
        max_err = mf;
        rms = n_audited ? sqrt(ss / n_audited) : 0;
        // Fallback: the exact sum for every queued entry.
        fallback = !(max_err <= audit_bound);
        for (int t = 0; t < num_types && !err && fallback; ++t)
        {
            if (!counts[t]) continue;
            const size_t q0 = (size_t) t * cap;
            scatter_audit_kernel<<<(counts[t] + kThreads - 1) / kThreads,
                    kThreads, 0, s>>>(a, t, counts[t], queue_y + 2 * q0, 0,
                    1, max_bits, sum_sq, n_aud);
            err = check_launch("surrogate fallback");
        }
    }
    if (!err)
    {
        const double kL = dipole_length_m * (kPi * frequency_hz /
                299792458.0);
        const unsigned grid = (unsigned) ((total + kThreads - 1) / kThreads);
        if (normalise_element)
            assemble_kernel<true><<<grid, kThreads, 0, s>>>(a, (float) kL,
                    (float) cos(kL), beam);
        else
            assemble_kernel<false><<<grid, kThreads, 0, s>>>(a, (float) kL,
                    (float) cos(kL), beam);
        err = check_launch("surrogate assemble");
    }
    scratch_free(d_type, s); scratch_free(a.af, s);
    scratch_free(a.queue_count, s); scratch_free(a.queue_index, s);
    scratch_free(a.queue_x, s); scratch_free(queue_y, s);
    scratch_free(stats, s);
    if (audit)
    {
        long long surrogate = 0;
        for (int c : counts) surrogate += c;
        audit[0] = max_err;
        audit[1] = rms;
        audit[2] = n_audited;
        audit[3] = fallback;
        audit[4] = (double) surrogate;
    }
    return err;
}

}  // extern "C"

// Drop-in oskar_interferometer_run_block: the reference's per-block driver
// (oskar/interferometer/src/oskar_interferometer_run_block.c:28-153, with
// sim_baselines at :156-336) re-implemented on the B200 kernels of this
// library. It is built into liboskar_b200_dropin.so, which a process loads
// ahead of an unmodified reference liboskar (LD_PRELOAD, or linked first):
// the reference's own oskar_interferometer_run, its Python wrapper and any
// user code then reach this function through the PLT, with the reference's
// settings, sky, telescope and output code around it.
//
// What it does per call, in the reference's order:
//  - checks that the simulator was initialised (h->header set);
//  - picks the GPU: h->gpu_ids[device_id] when the reference was given GPUs,
//    otherwise device_id modulo the visible GPUs (a CPU-only reference
//    configuration still correlates on the GPU); one CUDA stream per
//    (simulator, device_id), so the reference's device threads run
//    concurrently;
//  - claims (time, sky chunk) work units from the shared counter under
//    h->mutex (:88-103) until none are left;
//  - per unit: uploads the chunk's sky table when the chunk changes (the
//    reference's d->previous_chunk_index cache), horizon-clips it on the
//    device, then for each channel of the block: flux scaling with
//    frequency, station (u, v, w), station beams E, parallactic R and
//    E R, Jones K, K (E R), cable-length errors, auto- and
//    cross-correlation, all on the device;
//  - writes the block (resized, start indices set) into
//    h->d[device_id].vis_block_cpu[block_index % 2] (:146-151), which the
//    reference's oskar_interferometer_finalise_block combines over devices.
//
// Station beams: isotropic stations (identity E, or zero while the station
// beam direction is below the horizon, oskar_station_beam.c:84-93, 141-144)
// and aperture-array stations without child stations whose elements share
// one orientation and one set of data for both feeds (dipole or isotropic
// elements, up to four element types, cosine or Gaussian tapers, measured
// positions and cable-length errors in the weights, array, element and
// final normalisation), through the fused station-beam kernels. Other
// station types and features (child stations, element errors, apodisation,
// numerical element patterns, HARP data, ionospheric screens, gain models)
// return OSKAR_ERR_FUNCTION_NOT_AVAILABLE with a log message: there is no
// CPU fallback.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "oskar_b200.h"
#include "ref_abi.h"

#define DROPIN_EXPORT extern "C" __attribute__((visibility("default")))

namespace {

constexpr double kC0 = 299792458.0;

// FP64 point-source correlation without smearing on the FP64-class
// integer tensor-core form (oskb_cross_correlate_tc64_d) unless the
// environment variable OSKB_DROPIN_TC64 is 0 (then the FP64 direct
// kernels, as for every other case).
bool use_tc64()
{
    static const bool on = [] {
        const char* e = getenv("OSKB_DROPIN_TC64");
        return !(e && e[0] == '0');
    }();
    return on;
}

// FP32 point-source correlation without smearing on the integer
// tensor-core form (oskb_cross_correlate_tc_f: error ~4e-7, inside FP32's
// own) unless OSKB_DROPIN_TC32 is 0.
bool use_tc32()
{
    static const bool on = [] {
        const char* e = getenv("OSKB_DROPIN_TC32");
        return !(e && e[0] == '0');
    }();
    return on;
}

// ---------------------------------------------------------------- buffers
struct DevBuf
{
    void* p = nullptr;
    size_t bytes = 0;

    int ensure(size_t need)
    {
        if (need <= bytes) return 0;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        if (need == 0) return 0;
        if (cudaMalloc(&p, need) != cudaSuccess)
        {
            cudaGetLastError();
            return REF_ERR_MEMORY_ALLOC_FAILURE;
        }
        bytes = need;
        return 0;
    }
    template <typename T> T* as() const { return (T*) p; }
};

// Device state of one (simulator, device_id) pair.
struct State
{
    int cuda_dev = -1;
    cudaStream_t stream = nullptr;
    // sky chunk, as uploaded ([num_columns][capacity] table, [capacity][20]
    // valid-column counts) and after the horizon clip
    int num_in = 0, capacity = 0, num_columns = 0;
    DevBuf table, valid, clip_table, clip_valid, mask, index;
    // telescope
    DevBuf st_xyz, cable[2], lat, station_off;
    // per channel
    DevBuf uvw, uvw64, flux, E, R, K, J;
    // the block's visibilities
    DevBuf vis, autos;
    // workspace of the tensor-core correlation (FP64-class or FP32 form)
    DevBuf tc64ws;
    int* host_count = nullptr;   // page-locked: sources kept by the clip
};

std::mutex g_states_mutex;
std::map<std::pair<const void*, int>, State*> g_states;

State* state_for(const void* h, int device_id)
{
    std::lock_guard<std::mutex> lock(g_states_mutex);
    State*& s = g_states[std::make_pair(h, device_id)];
    if (!s) s = new State();
    return s;
}

// ---------------------------------------------------------------- kernels
// Isotropic station beams: identity (matrix) or 1 (scalar) per
// station-source where station_off[p] == 0, zero where it is 1 (the beam
// direction is below the horizon); rows with 2 are left as they are.
template <typename T>
__global__ void isotropic_beam_kernel(int num_src, int num_st, int matrix,
        const int* __restrict__ station_off, T* __restrict__ E)
{
    const size_t n = (size_t) num_src * num_st;
    const int w = matrix ? 8 : 2;
    for (size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
            i += (size_t) gridDim.x * blockDim.x)
    {
        const int p = (int) (i / num_src);
        if (station_off[p] == 2) continue;   // computed by the AA kernel
        const T one = station_off[p] ? (T) 0 : (T) 1;
        T* e = E + w * i;
        e[0] = one;
        e[1] = 0;
        if (matrix)
        {
            e[2] = 0; e[3] = 0; e[4] = 0; e[5] = 0;
            e[6] = one; e[7] = 0;
        }
    }
}

// Exclusive prefix sum of the horizon mask in one block (index[s] = number
// of kept sources before s; index[num] = total), then the order-preserving
// copy of every table column and valid-count row of the kept sources: the
// copy step of oskar_sky_horizon_clip (sky/src/oskar_sky_horizon_clip.c:
// 80-95, via oskar_sky_copy_source_data).
__global__ void __launch_bounds__(1024) scan_mask_kernel(int num,
        const int* __restrict__ mask, int* __restrict__ index, int* total)
{
    __shared__ int warp_sums[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < num; base += 1024)
    {
        const int s = base + (int) threadIdx.x;
        const int v = (s < num && mask[s]) ? 1 : 0;
        int x = v;
        for (int o = 1; o < 32; o <<= 1)
        {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sums[warp] = x;
        __syncthreads();
        if (warp == 0)
        {
            int t = warp_sums[lane];
            for (int o = 1; o < 32; o <<= 1)
            {
                const int y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            warp_sums[lane] = t;
        }
        __syncthreads();
        const int before = carry + (warp ? warp_sums[warp - 1] : 0) + x - v;
        if (s < num) index[s] = before;
        __syncthreads();
        if (threadIdx.x == 1023) carry = before + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

template <typename T>
__global__ void compact_rows_kernel(int num, int capacity, int num_columns,
        const int* __restrict__ mask, const int* __restrict__ index,
        const T* __restrict__ table, const int* __restrict__ valid,
        T* __restrict__ table_out, int* __restrict__ valid_out)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= num || !mask[s]) return;
    const int d = index[s];
    for (int k = 0; k < num_columns; ++k)
        table_out[(size_t) k * capacity + d] =
                table[(size_t) k * capacity + s];
    for (int j = 0; j < REF_SKY_NUM_FIXED_COLUMN_TYPES; ++j)
        valid_out[(size_t) d * REF_SKY_NUM_FIXED_COLUMN_TYPES + j] =
                valid[(size_t) s * REF_SKY_NUM_FIXED_COLUMN_TYPES + j];
}

// FP32 station (u, v, w) with the reference's single-precision arithmetic
// (convert/define_convert_ecef_to_station_uvw.h:3-28: products and sums
// rounded one at a time, trigonometric factors rounded from FP64).
__global__ void station_uvw_f_kernel(int num, const float* __restrict__ x,
        const float* __restrict__ y, const float* __restrict__ z,
        float sin_ha0, float cos_ha0, float sin_dec0, float cos_dec0,
        int ignore_w, float* __restrict__ u, float* __restrict__ v,
        float* __restrict__ w)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= num) return;
    const float x_ = x[i], y_ = y[i], z_ = z[i];
    const float t = __fsub_rn(__fmul_rn(x_, cos_ha0), __fmul_rn(y_, sin_ha0));
    u[i] = __fadd_rn(__fmul_rn(x_, sin_ha0), __fmul_rn(y_, cos_ha0));
    v[i] = __fsub_rn(__fmul_rn(z_, cos_dec0), __fmul_rn(t, sin_dec0));
    w[i] = ignore_w ? 0.0f :
            __fadd_rn(__fmul_rn(z_, sin_dec0), __fmul_rn(t, cos_dec0));
}

int launch_ok(const char* what, oskar_Log* log)
{
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return 0;
    oskar_log_error(log, "B200 drop-in: %s: %s", what, cudaGetErrorString(e));
    return REF_ERR_KERNEL_LAUNCH_FAILURE;
}

// ---------------------------------------------------------------- helpers
// Direction cosines (east, north, up) of a station's beam direction given
// in RA/Dec at local sidereal time lst and latitude lat: only its elevation
// is used (a beam below the horizon zeroes the station's beam,
// oskar_station_beam.c:84-93).
double beam_elevation(const oskar_Station* st, double gast)
{
    const double lat = oskar_station_lat_rad(st);
    const double lon = oskar_station_lon_rad(st);
    const double b_lon = oskar_station_beam_lon_rad(st);
    const double b_lat = oskar_station_beam_lat_rad(st);
    if (oskar_station_beam_coord_type(st) == REF_COORDS_AZEL) return b_lat;
    const double ha = gast + lon - b_lon;
    const double sin_el = sin(lat) * sin(b_lat) +
            cos(lat) * cos(b_lat) * cos(ha);
    return asin(fmax(-1.0, fmin(1.0, sin_el)));
}

struct Block
{
    int chan_start, num_chans, time_start, num_times;
};

// Copies a reference oskar_Mem's data to the device buffer (any location).
int upload(DevBuf& dst, const oskar_Mem* m, size_t elem, cudaStream_t s)
{
    const size_t n = oskar_mem_length(m) * elem;
    int err = dst.ensure(n);
    if (err || n == 0) return err;
    if (cudaMemcpyAsync(dst.p, oskar_mem_void_const(m), n, cudaMemcpyDefault,
            s) != cudaSuccess)
    {
        cudaGetLastError();
        return REF_ERR_MEMORY_COPY_FAILURE;
    }
    return 0;
}

size_t elem_bytes(int type)
{
    size_t b = (type & 0x0F) == REF_DOUBLE ? 8 : 4;
    if (type & REF_COMPLEX) b *= 2;
    if (type & REF_MATRIX) b *= 4;
    return b;
}

// ------------------------------------------------------------- the driver
template <typename T>
class Runner
{
public:
    Runner(RefInterferometer* h, State* st, int device_id, int* status)
        : h_(h), st_(st), dev_id_(device_id), status_(status),
          log_(h->log), tel_(h->tel), s_(st->stream) {}

    void run_block(int block_index);

private:
    void fail(int code, const char* msg)
    {
        if (!*status_) *status_ = code;
        oskar_log_error(log_, "B200 drop-in: %s", msg);
    }
    bool ok() const { return *status_ == 0; }
    long long num_baselines() const
    {
        return (long long) num_st_ * (num_st_ - 1) / 2;
    }
    void check(int err, const char* what)
    {
        if (err && !*status_)
        {
            *status_ = err;
            oskar_log_error(log_, "B200 drop-in: %s failed (status %d): %s",
                    what, err, oskb_last_error());
        }
    }

    void upload_chunk(const RefSky* sky);
    int horizon_clip(const RefSky* sky, double gast);
    void sim_baselines(const RefSky* sky, int num_src, const T* table,
            const int* valid, int chan_block, int time_block, int chan_sim,
            int time_sim);
    void station_beams(int num_src, double gast, const T* ra, const T* dec,
            double freq);

    RefInterferometer* h_;
    State* st_;
    int dev_id_;
    int* status_;
    oskar_Log* log_;
    oskar_Telescope* tel_;
    cudaStream_t s_;
    Block blk_{};
    int num_st_ = 0, matrix_ = 1, vis_type_ = 0;
    bool has_cross_ = false, has_auto_ = false;
};

template <typename T>
void Runner<T>::upload_chunk(const RefSky* sky)
{
    if (!ok()) return;
    // The mirrored private layout must agree with the reference's own
    // accessors before anything is read through it.
    const oskar_Sky* osky = reinterpret_cast<const oskar_Sky*>(sky);
    if (sky->attr_int[REF_SKY_NUM_SOURCES] !=
            oskar_sky_int(osky, REF_SKY_NUM_SOURCES) ||
            sky->attr_int[REF_SKY_CAPACITY] !=
            oskar_sky_int(osky, REF_SKY_CAPACITY))
    {
        fail(REF_ERR_FUNCTION_NOT_AVAILABLE, "sky model layout differs "
                "from the one this library was built for");
        return;
    }
    st_->num_in = sky->attr_int[REF_SKY_NUM_SOURCES];
    st_->capacity = sky->attr_int[REF_SKY_CAPACITY];
    st_->num_columns = sky->attr_int[REF_SKY_NUM_COLUMNS];
    if ((oskar_mem_type(sky->table) & 0x0F) != (sizeof(T) == 8 ?
            REF_DOUBLE : REF_SINGLE))
    {
        fail(REF_ERR_TYPE_MISMATCH, "sky precision differs from the "
                "simulator's");
        return;
    }
    check(upload(st_->table, sky->table, sizeof(T), s_), "sky table upload");
    check(upload(st_->valid, sky->num_valid_columns, sizeof(int), s_),
            "sky column counts upload");
}

// Horizon clip of the uploaded chunk for one dump (sky/src/
// oskar_sky_horizon_clip.c:18-96): the mask over all station models, then
// the order-preserving copy. Returns the number of sources kept.
template <typename T>
int Runner<T>::horizon_clip(const RefSky* sky, double gast)
{
    const oskar_Sky* osky = reinterpret_cast<const oskar_Sky*>(sky);
    const int n = st_->num_in, cap = st_->capacity;
    const size_t tbytes = (size_t) st_->num_columns * cap * sizeof(T);
    check(st_->clip_table.ensure(tbytes), "clip buffers");
    check(st_->clip_valid.ensure((size_t) cap * REF_SKY_NUM_FIXED_COLUMN_TYPES
            * sizeof(int)), "clip buffers");
    check(st_->mask.ensure(((size_t) n + 1) * sizeof(int)), "clip buffers");
    check(st_->index.ensure(((size_t) n + 1) * sizeof(int)), "clip buffers");
    if (!ok() || n == 0) return 0;
    const double ra0 = oskar_sky_double(osky, REF_SKY_REF_RA_RAD);
    const double dec0 = oskar_sky_double(osky, REF_SKY_REF_DEC_RAD);
    const int nmod = oskar_telescope_num_station_models(tel_);
    std::vector<double> ha0(nmod), lat(nmod);
    for (int i = 0; i < nmod; ++i)
    {
        const oskar_Station* s = oskar_telescope_station_const(tel_, i);
        ha0[i] = (gast + oskar_station_lon_rad(s)) - ra0;
        lat[i] = oskar_station_lat_rad(s);
    }
    const T* tab = st_->table.as<T>();
    const int cl = oskar_sky_first_column(osky, REF_SKY_SCRATCH_L);
    const int cm = oskar_sky_first_column(osky, REF_SKY_SCRATCH_M);
    const int cn = oskar_sky_first_column(osky, REF_SKY_SCRATCH_N);
    if (cl < 0 || cm < 0 || cn < 0)
    {
        fail(REF_ERR_INVALID_ARGUMENT, "sky chunk has no direction cosines");
        return 0;
    }
    cudaMemsetAsync(st_->mask.p, 0, (size_t) n * sizeof(int), s_);
    int err;
    if (sizeof(T) == 8)
        err = oskb_sky_horizon_mask_d(n, (const double*) tab + (size_t) cl *
                cap, (const double*) tab + (size_t) cm * cap,
                (const double*) tab + (size_t) cn * cap, nmod, ha0.data(),
                lat.data(), dec0, st_->mask.as<int>(), s_);
    else
        err = oskb_sky_horizon_mask_f(n, (const float*) tab + (size_t) cl *
                cap, (const float*) tab + (size_t) cm * cap,
                (const float*) tab + (size_t) cn * cap, nmod, ha0.data(),
                lat.data(), dec0, st_->mask.as<int>(), s_);
    check(err, "horizon mask");
    if (!ok()) return 0;
    int* total = st_->index.as<int>() + n;
    scan_mask_kernel<<<1, 1024, 0, s_>>>(n, st_->mask.as<int>(),
            st_->index.as<int>(), total);
    compact_rows_kernel<T><<<(n + 255) / 256, 256, 0, s_>>>(n, cap,
            st_->num_columns, st_->mask.as<int>(), st_->index.as<int>(), tab,
            st_->valid.as<int>(), st_->clip_table.as<T>(),
            st_->clip_valid.as<int>());
    check(launch_ok("horizon clip", log_), "horizon clip");
    cudaMemcpyAsync(st_->host_count, total, sizeof(int),
            cudaMemcpyDeviceToHost, s_);
    if (cudaStreamSynchronize(s_) != cudaSuccess)
        check(launch_ok("horizon clip", log_), "horizon clip");
    return ok() ? *st_->host_count : 0;
}

// Station beams E [station][source] for this dump and channel.
// One aperture-array station model, as the fused station-beam kernel takes
// it (oskar_evaluate_station_beam_aperture_array.c:153-240 for a station
// without child stations, elements of common orientation and one set of
// element data for both feeds).
struct AaModel
{
    int model;                    // index of the station model
    int num_elements, num_types;
    int norm_element, norm_array, norm_final, swap_xy, is_3d;
    std::vector<double> length, taper_param;   // per element type
    std::vector<int> length_units, kind, taper;
    double euler_x, euler_y;
    double lat, lst;
    double beam_enu[3], norm_enu[3];

    bool same_launch(const AaModel& o) const
    {
        return num_elements == o.num_elements && num_types == o.num_types &&
                norm_element == o.norm_element &&
                norm_array == o.norm_array && norm_final == o.norm_final &&
                swap_xy == o.swap_xy && is_3d == o.is_3d &&
                length == o.length && length_units == o.length_units &&
                kind == o.kind && taper == o.taper &&
                taper_param == o.taper_param;
    }
};

// Copies a station model's beams into the rows of the stations that use
// it: E[p] = E_model[slot[p]] (rows of num_src values of w reals).
template <typename T>
__global__ void gather_beams_kernel(int num_src, int num_st, int w,
        const int* __restrict__ slot, const T* __restrict__ Em,
        T* __restrict__ E)
{
    const size_t row = (size_t) num_src * w;
    const size_t n = row * num_st;
    for (size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
            i += (size_t) gridDim.x * blockDim.x)
    {
        const size_t p = i / row, k = i - p * row;
        E[i] = Em[(size_t) slot[p] * row + k];
    }
}

// Station beams E [station][source] for this dump and channel: each station
// model that the stations use is evaluated once (the reference's
// oskar_evaluate_jones_E with station-beam duplication, :140-188, or every
// station without it), then copied to its stations.
template <typename T>
void Runner<T>::station_beams(int num_src, double gast, const T* ra,
        const T* dec, double freq)
{
    if (!ok()) return;
    const int dup = oskar_telescope_allow_station_beam_duplication(tel_);
    const int* type_map = nullptr;
    if (dup)
    {
        const oskar_Mem* m = oskar_telescope_station_type_map_const(tel_);
        if (m && oskar_mem_location(m) == REF_CPU &&
                (int) oskar_mem_length(m) >= num_st_)
            type_map = (const int*) oskar_mem_void_const(m);
    }
    // models to evaluate, in order of first use, and each station's slot
    std::vector<int> models, slot(num_st_);
    std::map<int, int> slot_of_model;
    for (int p = 0; p < num_st_; ++p)
    {
        const int model = type_map ? type_map[p] : p;
        auto it = slot_of_model.find(model);
        if (it == slot_of_model.end())
        {
            slot_of_model[model] = (int) models.size();
            slot[p] = (int) models.size();
            models.push_back(model);
        }
        else
            slot[p] = it->second;
    }
    const int nm = (int) models.size();
    // per model: 0 = identity (isotropic), 1 = zero (beam direction below
    // the horizon, oskar_station_beam.c:84-93), 2 = aperture array
    std::vector<int> mode(nm, 0);
    std::vector<AaModel> aa;
    const double c0 = 299792458.0;
    const int pc_type = oskar_telescope_phase_centre_coord_type(tel_);
    const double pc_lon = oskar_telescope_phase_centre_longitude_rad(tel_);
    const double pc_lat = oskar_telescope_phase_centre_latitude_rad(tel_);
    for (int k = 0; k < nm; ++k)
    {
        const oskar_Station* st = oskar_telescope_station_const(tel_,
                models[k]);
        if (!st)
        {
            fail(REF_ERR_SETTINGS_TELESCOPE, "missing station model");
            return;
        }
        const int type = oskar_station_type(st);
        if (beam_elevation(st, gast) < 0.0)
        {
            mode[k] = 1;
            continue;
        }
        if (type == REF_STATION_TYPE_ISOTROPIC) continue;
        if (type != REF_STATION_TYPE_AA)
        {
            fail(REF_ERR_FUNCTION_NOT_AVAILABLE, "Gaussian and VLA station "
                    "beams are not built in this drop-in");
            return;
        }
        if (oskar_station_has_child(st) ||
                !oskar_station_common_element_orientation(st) ||
                !oskar_station_enable_array_pattern(st) ||
                (matrix_ && !oskar_station_common_pol_beams(st)) ||
                oskar_station_apply_element_errors(st) ||
                oskar_station_apply_element_weight(st) ||
                oskar_gains_defined(oskar_station_gains_const(st)) ||
                oskar_station_harp_data_const(st, freq) ||
                oskar_station_num_element_types(st) > 4)
        {
            fail(REF_ERR_FUNCTION_NOT_AVAILABLE, "this aperture-array station "
                    "(child stations, per-element orientations, separate "
                    "feed data, element errors, apodisation, gain models, "
                    "HARP data or more than four element types) is not "
                    "built in this drop-in");
            return;
        }
        AaModel a;
        a.model = models[k];
        a.num_elements = oskar_station_num_elements(st);
        a.num_types = oskar_station_num_element_types(st);
        a.norm_element = oskar_station_normalise_element_pattern(st);
        a.norm_array = oskar_station_normalise_array_pattern(st);
        a.norm_final = oskar_station_normalise_final_beam(st);
        a.swap_xy = oskar_station_swap_xy(st);
        a.is_3d = oskar_station_array_is_3d(st);
        for (int t = 0; t < a.num_types; ++t)
        {
            const oskar_Element* e = oskar_station_element_const(st, t);
            if (!e || oskar_element_num_freq(e) > 0)
            {
                fail(REF_ERR_FUNCTION_NOT_AVAILABLE, "numerical element "
                        "patterns are not built in this drop-in");
                return;
            }
            a.kind.push_back(oskar_element_is_isotropic(e) ?
                    OSKB_ELEMENT_ISOTROPIC : OSKB_ELEMENT_DIPOLE);
            a.taper.push_back(oskar_element_taper_type(e));
            a.taper_param.push_back(a.taper.back() == OSKB_TAPER_COSINE ?
                    oskar_element_cosine_power(e) :
                    a.taper.back() == OSKB_TAPER_GAUSSIAN ?
                    oskar_element_gaussian_fwhm_rad(e) : 0.0);
            a.length.push_back(oskar_element_dipole_length(e));
            a.length_units.push_back(oskar_element_dipole_length_units(e));
        }
        a.euler_x = oskar_station_element_euler_index_rad(st, 0, 0, 0);
        a.euler_y = oskar_station_element_euler_index_rad(st, 1, 0, 0);
        a.lat = oskar_station_lat_rad(st);
        a.lst = gast + oskar_station_lon_rad(st);
        int stt = 0;
        oskar_station_beam_horizon_direction(st, gast, &a.beam_enu[0],
                &a.beam_enu[1], &a.beam_enu[2], &stt);
        if (stt) check(stt, "station beam direction");
        // normalisation direction: the phase centre
        // (oskar_station_beam.c:108-126)
        if (pc_type == REF_COORDS_RADEC)
        {
            const double ha = a.lst - pc_lon;
            const double sh = sin(ha), ch = cos(ha);
            const double sd = sin(pc_lat), cd = cos(pc_lat);
            const double sl = sin(a.lat), cl = cos(a.lat);
            a.norm_enu[0] = -cd * sh;
            a.norm_enu[1] = cl * sd - sl * cd * ch;
            a.norm_enu[2] = sl * sd + cl * cd * ch;
        }
        else
        {
            fail(REF_ERR_FUNCTION_NOT_AVAILABLE, "beam normalisation needs "
                    "an RA/Dec phase centre in this drop-in");
            return;
        }
        mode[k] = 2;
        aa.push_back(a);
    }
    if (!ok()) return;
    const int w = matrix_ ? 8 : 2;
    const size_t row = (size_t) num_src * w;
    DevBuf& em = st_->J;   // model beams (J is free until K is joined)
    check(em.ensure((size_t) nm * row * sizeof(T)), "beam buffers");
    check(st_->E.ensure((size_t) num_st_ * row * sizeof(T)), "beam buffers");
    if (!ok()) return;

    // ---- aperture-array models, one launch per group of alike models
    std::vector<int> aa_slot;
    for (int k = 0; k < nm; ++k)
        if (mode[k] == 2) aa_slot.push_back(k);
    std::vector<char> done(aa.size(), 0);
    for (size_t g0 = 0; g0 < aa.size() && ok(); ++g0)
    {
        if (done[g0]) continue;
        std::vector<size_t> grp;
        for (size_t j = g0; j < aa.size(); ++j)
            if (!done[j] && aa[j].same_launch(aa[g0]))
            {
                grp.push_back(j);
                done[j] = 1;
            }
        const AaModel& r = aa[g0];
        const int ng = (int) grp.size(), ne = r.num_elements;
        std::vector<T> el((size_t) 7 * ng * ne);
        std::vector<int> etype((size_t) ng * ne);
        std::vector<double> geo((size_t) 10 * ng);   // lat, lst, beam, norm
        bool have_cable = false;
        for (int gi = 0; gi < ng && ok(); ++gi)
        {
            const AaModel& a = aa[grp[gi]];
            const oskar_Station* st = oskar_telescope_station_const(tel_,
                    a.model);
            for (int d = 0; d < 3; ++d)
            {
                const oskar_Mem* tm =
                        oskar_station_element_true_enu_metres_const(st, 0, d);
                const oskar_Mem* mm =
                        oskar_station_element_measured_enu_metres_const(st, 0,
                        d);
                if (!tm || !mm || (int) oskar_mem_length(tm) < ne ||
                        (int) oskar_mem_length(mm) < ne)
                {
                    fail(REF_ERR_SETTINGS_TELESCOPE, "element coordinates");
                    return;
                }
                memcpy(&el[((size_t) d * ng + gi) * ne],
                        oskar_mem_void_const(tm), ne * sizeof(T));
                memcpy(&el[((size_t) (3 + d) * ng + gi) * ne],
                        oskar_mem_void_const(mm), ne * sizeof(T));
            }
            const oskar_Mem* cm =
                    oskar_station_element_cable_length_error_metres_const(st,
                    0);
            if (cm && (int) oskar_mem_length(cm) >= ne)
            {
                memcpy(&el[((size_t) 6 * ng + gi) * ne],
                        oskar_mem_void_const(cm), ne * sizeof(T));
                have_cable = true;
            }
            const int* types = oskar_station_element_types_cpu_const(st);
            for (int e = 0; e < ne; ++e)
                etype[(size_t) gi * ne + e] = types ? types[e] : 0;
            geo[gi] = a.lat;
            geo[ng + gi] = a.lst;
            for (int d = 0; d < 3; ++d)
            {
                geo[2 * ng + 3 * gi + d] = a.beam_enu[d];
                geo[5 * ng + 3 * gi + d] = a.norm_enu[d];
            }
            geo[8 * ng + gi] = a.euler_x;
            geo[9 * ng + gi] = a.euler_y;
        }
        // per-type host parameters at this frequency
        std::vector<double> len(r.num_types), orient((size_t) 2 * ng *
                r.num_types);
        for (int t = 0; t < r.num_types; ++t)
            len[t] = r.length_units[t] == REF_WAVELENGTHS ?
                    r.length[t] * (c0 / freq) : r.length[t];
        for (int gi = 0; gi < ng; ++gi)
            for (int t = 0; t < r.num_types; ++t)
            {
                orient[(size_t) gi * r.num_types + t] = geo[8 * ng + gi];
                orient[(size_t) (ng + gi) * r.num_types + t] =
                        geo[9 * ng + gi];
            }
        const size_t ebytes = el.size() * sizeof(T);
        const size_t tbytes = etype.size() * sizeof(int);
        const size_t gbytes = (size_t) 8 * ng * sizeof(double);
        const size_t obytes = orient.size() * sizeof(double);
        const size_t dirs = (size_t) 3 * ng * num_src * sizeof(T);
        DevBuf& buf = st_->uvw64;
        check(buf.ensure(ebytes + tbytes + gbytes + obytes + dirs + 1024),
                "beam buffers");
        if (!ok()) return;
        uint8_t* b = buf.as<uint8_t>();
        T* d_el = (T*) b;
        int* d_type = (int*) (b + ebytes);
        double* d_geo = (double*) (b + ebytes + tbytes);
        double* d_orient = (double*) (b + ebytes + tbytes + gbytes);
        T* d_dirs = (T*) (b + ((ebytes + tbytes + gbytes + obytes + 255) &
                ~(size_t) 255));
        cudaMemcpyAsync(d_el, el.data(), ebytes, cudaMemcpyHostToDevice, s_);
        cudaMemcpyAsync(d_type, etype.data(), tbytes, cudaMemcpyHostToDevice,
                s_);
        cudaMemcpyAsync(d_geo, geo.data(), gbytes, cudaMemcpyHostToDevice,
                s_);
        cudaMemcpyAsync(d_orient, orient.data(), obytes,
                cudaMemcpyHostToDevice, s_);
        T* dx = d_dirs;
        T* dy = dx + (size_t) ng * num_src;
        T* dz = dy + (size_t) ng * num_src;
        // source directions (east, north, up) at each model's station
        int err = sizeof(T) == 8 ?
                oskb_convert_ra_dec_to_enu_directions_d(num_src,
                (const double*) ra, (const double*) dec, ng, d_geo + ng,
                d_geo, (double*) dx, (double*) dy, (double*) dz, s_) :
                oskb_convert_ra_dec_to_enu_directions_f(num_src,
                (const float*) ra, (const float*) dec, ng, d_geo + ng, d_geo,
                (float*) dx, (float*) dy, (float*) dz, s_);
        check(err, "source directions");
        // the group's models take consecutive slots of a staging area after
        // the nm model rows: evaluated there, then copied to their slots
        std::vector<int> kinds(r.kind), tapers(r.taper);
        std::vector<double> tparam(r.taper_param);
        const size_t ge = (size_t) ng * ne;
        check(st_->R.ensure((size_t) ng * row * sizeof(T)), "beam buffers");
        if (!ok()) return;
        T* out = st_->R.as<T>();
        const T* cab = have_cable ? d_el + 6 * ge : nullptr;
        const int nf = r.norm_final;
        if (sizeof(T) == 8 && matrix_)
            err = oskb_station_beam_aa_types_d(ng, ne, (const double*) d_el,
                    (const double*) d_el + ge, (const double*) d_el + 2 * ge,
                    (const double*) d_el + 3 * ge,
                    (const double*) d_el + 4 * ge,
                    (const double*) d_el + 5 * ge, (const double*) cab,
                    nullptr, r.num_types, d_type, len.data(), kinds.data(),
                    tapers.data(), tparam.data(), d_orient,
                    d_orient + (size_t) ng * r.num_types, r.norm_element,
                    r.norm_array, nf, r.swap_xy, r.is_3d, freq, d_geo + 2 * ng,
                    d_geo + 5 * ng, num_src, (const double*) dx,
                    (const double*) dy, (const double*) dz, 1, (double*) out,
                    s_);
        else if (sizeof(T) == 8)
            err = oskb_station_beam_aa_scalar_d(ng, ne, (const double*) d_el,
                    (const double*) d_el + ge, (const double*) d_el + 2 * ge,
                    (const double*) d_el + 3 * ge,
                    (const double*) d_el + 4 * ge,
                    (const double*) d_el + 5 * ge, (const double*) cab,
                    nullptr, r.num_types, d_type, len.data(), kinds.data(),
                    tapers.data(), tparam.data(), d_orient,
                    d_orient + (size_t) ng * r.num_types, r.norm_element,
                    r.norm_array, nf, r.swap_xy, r.is_3d, freq, d_geo + 2 * ng,
                    d_geo + 5 * ng, num_src, (const double*) dx,
                    (const double*) dy, (const double*) dz, 1, (double*) out,
                    s_);
        else if (matrix_)
            err = oskb_station_beam_aa_types_f(ng, ne, (const float*) d_el,
                    (const float*) d_el + ge, (const float*) d_el + 2 * ge,
                    (const float*) d_el + 3 * ge, (const float*) d_el + 4 * ge,
                    (const float*) d_el + 5 * ge, (const float*) cab, nullptr,
                    r.num_types, d_type, len.data(), kinds.data(),
                    tapers.data(), tparam.data(), d_orient,
                    d_orient + (size_t) ng * r.num_types, r.norm_element,
                    r.norm_array, nf, r.swap_xy, r.is_3d, freq, d_geo + 2 * ng,
                    d_geo + 5 * ng, num_src, (const float*) dx,
                    (const float*) dy, (const float*) dz, 1, (float*) out, s_);
        else
            err = oskb_station_beam_aa_scalar_f(ng, ne, (const float*) d_el,
                    (const float*) d_el + ge, (const float*) d_el + 2 * ge,
                    (const float*) d_el + 3 * ge, (const float*) d_el + 4 * ge,
                    (const float*) d_el + 5 * ge, (const float*) cab, nullptr,
                    r.num_types, d_type, len.data(), kinds.data(),
                    tapers.data(), tparam.data(), d_orient,
                    d_orient + (size_t) ng * r.num_types, r.norm_element,
                    r.norm_array, nf, r.swap_xy, r.is_3d, freq, d_geo + 2 * ng,
                    d_geo + 5 * ng, num_src, (const float*) dx,
                    (const float*) dy, (const float*) dz, 1, (float*) out, s_);
        check(err, "aperture-array station beams");
        for (int gi = 0; gi < ng && ok(); ++gi)
            cudaMemcpyAsync(em.as<T>() + (size_t) aa_slot[grp[gi]] * row,
                    out + (size_t) gi * row, row * sizeof(T),
                    cudaMemcpyDeviceToDevice, s_);
        // host vectors must outlive their copies
        cudaStreamSynchronize(s_);
    }
    if (!ok()) return;

    // ---- isotropic and below-horizon models, then the copy to stations
    DevBuf& flags = st_->station_off;
    check(flags.ensure((size_t) (nm + num_st_) * sizeof(int)),
            "beam buffers");
    if (!ok()) return;
    std::vector<int> host(nm + num_st_);
    for (int k = 0; k < nm; ++k) host[k] = mode[k];
    for (int p = 0; p < num_st_; ++p) host[nm + p] = slot[p];
    cudaMemcpyAsync(flags.p, host.data(), host.size() * sizeof(int),
            cudaMemcpyHostToDevice, s_);
    const size_t n = (size_t) nm * num_src;
    int grid = (int) std::min<size_t>((n + 255) / 256, 148 * 16);
    isotropic_beam_kernel<T><<<grid, 256, 0, s_>>>(num_src, nm, matrix_,
            flags.as<int>(), em.as<T>());
    const size_t ns = (size_t) num_st_ * row;
    grid = (int) std::min<size_t>((ns + 255) / 256, 148 * 16);
    gather_beams_kernel<T><<<grid, 256, 0, s_>>>(num_src, num_st_, w,
            flags.as<int>() + nm, em.as<T>(), st_->E.as<T>());
    check(launch_ok("station beams", log_), "station beams");
    cudaStreamSynchronize(s_);
}

template <typename T>
void Runner<T>::sim_baselines(const RefSky* sky, int num_src, const T* tab,
        const int* valid, int chan_block, int time_block, int chan_sim,
        int time_sim)
{
    const oskar_Sky* osky = reinterpret_cast<const oskar_Sky*>(sky);
    if (!ok() || num_src == 0 || time_block >= blk_.num_times ||
            chan_block >= blk_.num_chans)
        return;
    const int cap = st_->capacity;
    const bool dbl = sizeof(T) == 8;
    const double dt_days = h_->time_inc_sec / 86400.0;
    const double t_start = h_->time_start_mjd_utc;
    const double t_dump = t_start + dt_days * (time_sim + 0.5);
    const double gast = oskar_convert_mjd_to_gast_fast(t_dump);
    const double freq = h_->freq_start_hz + chan_sim * h_->freq_inc_hz;
    auto col = [&](int type) -> const T* {
        const int k = oskar_sky_first_column(osky, type);
        return k < 0 ? nullptr : tab + (size_t) k * cap;
    };
    auto colidx = [&](int type) {
        return oskar_sky_first_column(osky, type);
    };

    // ---- flux scaled to this channel (run_block.c:183-190)
    check(st_->flux.ensure((size_t) 4 * cap * sizeof(T)), "flux buffers");
    if (!ok()) return;
    T* fI = st_->flux.as<T>();
    T *fQ = fI + cap, *fU = fI + 2 * (size_t) cap, *fV = fI + 3 * (size_t) cap;
    int err;
    if (dbl)
        err = oskb_sky_scale_flux_with_frequency_d(num_src, cap,
                st_->num_columns, freq, (const double*) tab, valid,
                colidx(REF_SKY_I_JY), colidx(REF_SKY_Q_JY),
                colidx(REF_SKY_U_JY), colidx(REF_SKY_V_JY),
                colidx(REF_SKY_REF_HZ), colidx(REF_SKY_LIN_SI),
                colidx(REF_SKY_SPEC_IDX), colidx(REF_SKY_RM_RAD),
                colidx(REF_SKY_POLF), colidx(REF_SKY_POLA_RAD),
                colidx(REF_SKY_REF_WAVE_M), colidx(REF_SKY_SPEC_CURV),
                colidx(REF_SKY_LINE_WIDTH_HZ), colidx(REF_SKY_INC_HZ),
                (double*) fI, (double*) fQ, (double*) fU, (double*) fV, s_);
    else
        err = oskb_sky_scale_flux_with_frequency_f(num_src, cap,
                st_->num_columns, (float) freq, (const float*) tab, valid,
                colidx(REF_SKY_I_JY), colidx(REF_SKY_Q_JY),
                colidx(REF_SKY_U_JY), colidx(REF_SKY_V_JY),
                colidx(REF_SKY_REF_HZ), colidx(REF_SKY_LIN_SI),
                colidx(REF_SKY_SPEC_IDX), colidx(REF_SKY_RM_RAD),
                colidx(REF_SKY_POLF), colidx(REF_SKY_POLA_RAD),
                colidx(REF_SKY_REF_WAVE_M), colidx(REF_SKY_SPEC_CURV),
                colidx(REF_SKY_LINE_WIDTH_HZ), colidx(REF_SKY_INC_HZ),
                (float*) fI, (float*) fQ, (float*) fU, (float*) fV, s_);
    check(err, "flux scaling");

    // ---- station (u, v, w) of this dump, true coordinates
    // (oskar_telescope_uvw.c:15-102 with one time sample)
    const int azel = oskar_telescope_phase_centre_coord_type(tel_) ==
            REF_COORDS_AZEL;
    const double lon0 = oskar_telescope_phase_centre_longitude_rad(tel_);
    const double lat0 = oskar_telescope_phase_centre_latitude_rad(tel_);
    check(st_->uvw.ensure((size_t) 3 * num_st_ * sizeof(T)), "uvw buffers");
    if (!ok()) return;
    T* u = st_->uvw.as<T>();
    T *v = u + num_st_, *w = u + 2 * num_st_;
    const T* sx = st_->st_xyz.as<T>();
    const T *sy = sx + num_st_, *sz = sx + 2 * num_st_;
    if (azel)
    {
        // drift scans take their (u, v, w) from the ENU coordinates and
        // their directions from apparent RA/Dec per dump (run_block.c:
        // 211-227): not built here
        fail(REF_ERR_FUNCTION_NOT_AVAILABLE, "drift-scan (AZEL) phase "
                "centres are not built in this drop-in");
        return;
    }
    if (dbl)
    {
        check(oskb_convert_ecef_to_station_uvw_d(num_st_, (const double*) sx,
                (const double*) sy, (const double*) sz, lon0, lat0, gast, 0,
                0, (double*) u, (double*) v, (double*) w, s_),
                "station uvw");
    }
    else
    {
        const double ha0 = gast - lon0;
        station_uvw_f_kernel<<<(num_st_ + 127) / 128, 128, 0, s_>>>(num_st_,
                (const float*) sx, (const float*) sy, (const float*) sz,
                (float) sin(ha0), (float) cos(ha0), (float) sin(lat0),
                (float) cos(lat0), 0, (float*) u, (float*) v, (float*) w);
        check(launch_ok("station uvw", log_), "station uvw");
    }

    // ---- source direction cosines
    const T *l = col(REF_SKY_SCRATCH_L), *m = col(REF_SKY_SCRATCH_M),
            *n = col(REF_SKY_SCRATCH_N);
    if (!l || !m || !n)
    {
        fail(REF_ERR_INVALID_ARGUMENT, "sky chunk has no direction cosines");
        return;
    }

    // ---- Jones E, R and E R
    station_beams(num_src, gast, col(REF_SKY_RA_RAD), col(REF_SKY_DEC_RAD),
            freq);
    if (!ok()) return;
    const size_t njones = (size_t) num_st_ * num_src;
    const size_t mat = njones * 8 * sizeof(T), cpx = njones * 2 * sizeof(T);
    check(st_->K.ensure(cpx), "Jones buffers");
    check(st_->J.ensure(mat), "Jones buffers");
    check(st_->R.ensure(mat), "Jones buffers");
    if (!ok()) return;
    const bool have_R = h_->d[dev_id_].R != nullptr;
    T* EJ = st_->E.as<T>();    // becomes the joined Jones
    if (have_R)
    {
        // R per station (its latitude and local sidereal time), or station
        // 0's for all when station beams are shared
        // (oskar_evaluate_jones_R.c:37-70, 129-140)
        const int dup = oskar_telescope_allow_station_beam_duplication(tel_);
        std::vector<double> lat(num_st_), lst(num_st_);
        for (int p = 0; p < num_st_; ++p)
        {
            const oskar_Station* s = oskar_telescope_station_const(tel_,
                    dup ? 0 : p);
            lat[p] = oskar_station_lat_rad(s);
            lst[p] = gast + oskar_station_lon_rad(s);
        }
        check(st_->lat.ensure(2 * num_st_ * sizeof(double)), "R buffers");
        if (!ok()) return;
        double* dlat = st_->lat.as<double>();
        cudaMemcpyAsync(dlat, lat.data(), num_st_ * sizeof(double),
                cudaMemcpyHostToDevice, s_);
        cudaMemcpyAsync(dlat + num_st_, lst.data(), num_st_ * sizeof(double),
                cudaMemcpyHostToDevice, s_);
        const T* ra = col(REF_SKY_RA_RAD);
        const T* dec = col(REF_SKY_DEC_RAD);
        if (dbl)
            err = oskb_evaluate_jones_R_d(num_src, (const double*) ra,
                    (const double*) dec, num_st_, dlat, dlat + num_st_,
                    st_->R.as<double>(), s_);
        else
            err = oskb_evaluate_jones_R_f(num_src, (const float*) ra,
                    (const float*) dec, num_st_, dlat, dlat + num_st_,
                    st_->R.as<float>(), s_);
        check(err, "Jones R");
        // R <- E R (oskar_jones_join(d->R, d->E, d->R), run_block.c:259-274)
        if (dbl)
            err = oskb_mem_multiply_d(OSKB_MUL_MM_M, 0, 0, 0, njones,
                    (const double*) EJ, st_->R.as<double>(),
                    st_->J.as<double>(), s_);
        else
            err = oskb_mem_multiply_f(OSKB_MUL_MM_M, 0, 0, 0, njones,
                    (const float*) EJ, st_->R.as<float>(),
                    st_->J.as<float>(), s_);
        check(err, "join E R");
        cudaStreamSynchronize(s_);   // lat/lst host vectors
    }

    // ---- Jones K (run_block.c:277-281)
    const double wavenumber = 2.0 * M_PI * freq / kC0;
    if (dbl)
        err = oskb_evaluate_jones_K_d(num_src, (const double*) l,
                (const double*) m, (const double*) n, num_st_,
                (const double*) u, (const double*) v, (const double*) w,
                wavenumber, (const double*) fI, h_->source_min_jy,
                h_->source_max_jy, h_->ignore_w_components,
                st_->K.as<double>(), s_);
    else
        err = oskb_evaluate_jones_K_f(num_src, (const float*) l,
                (const float*) m, (const float*) n, num_st_,
                (const float*) u, (const float*) v, (const float*) w,
                (float) wavenumber, (const float*) fI,
                (float) h_->source_min_jy, (float) h_->source_max_jy,
                h_->ignore_w_components, st_->K.as<float>(), s_);
    check(err, "Jones K");

    // ---- J = K (E R) or K E (run_block.c:284-286), into the E buffer
    const T* second = have_R ? st_->J.as<T>() : st_->E.as<T>();
    T* joined = have_R ? st_->E.as<T>() : st_->J.as<T>();
    const int kind = matrix_ ? OSKB_MUL_CM_M : OSKB_MUL_CC_C;
    if (dbl)
        err = oskb_mem_multiply_d(kind, 0, 0, 0, njones,
                st_->K.as<double>(), (const double*) second,
                (double*) joined, s_);
    else
        err = oskb_mem_multiply_f(kind, 0, 0, 0, njones, st_->K.as<float>(),
                (const float*) second, (float*) joined, s_);
    check(err, "join K");
    EJ = joined;

    // ---- gains (run_block.c:288-295): HDF5 gain tables are not built
    if (oskar_gains_defined(oskar_telescope_gains(tel_)))
    {
        fail(REF_ERR_FUNCTION_NOT_AVAILABLE, "station gain models are not "
                "built in this drop-in");
        return;
    }

    // ---- cable-length errors (run_block.c:297-304)
    const T* cx = st_->cable[0].p ? st_->cable[0].as<T>() : nullptr;
    const T* cy = st_->cable[1].p ? st_->cable[1].as<T>() : nullptr;
    if (cx || cy)
    {
        if (dbl)
            err = oskb_jones_apply_cable_length_errors_d(matrix_, num_src,
                    num_st_, wavenumber, (const double*) cx,
                    (const double*) cy, (double*) EJ, s_);
        else
            err = oskb_jones_apply_cable_length_errors_f(matrix_, num_src,
                    num_st_, (float) wavenumber, (const float*) cx,
                    (const float*) cy, (float*) EJ, s_);
        check(err, "cable-length errors");
    }

    // ---- correlation (run_block.c:306-334)
    const int offset = blk_.num_chans * time_block + chan_block;
    if (has_auto_)
    {
        if (dbl)
            err = oskb_auto_correlate_d(matrix_, num_src, num_st_,
                    num_st_ * offset, (const double*) EJ, (const double*) fI,
                    (const double*) fQ, (const double*) fU,
                    (const double*) fV, st_->autos.as<double>(), s_);
        else
            err = oskb_auto_correlate_f(matrix_, num_src, num_st_,
                    num_st_ * offset, (const float*) EJ, (const float*) fI,
                    (const float*) fQ, (const float*) fU, (const float*) fV,
                    st_->autos.as<float>(), s_);
        check(err, "auto-correlation");
    }
    if (has_cross_)
    {
        // the dispatcher's parameters (correlate/src/oskar_cross_correlate.c:
        // 40-71)
        const int gaussian = oskar_sky_int(osky, REF_SKY_USE_EXTENDED) == 1;
        const double inv_wl = fabs(freq) / kC0;
        const double frac_bw = oskar_telescope_channel_bandwidth_hz(tel_) /
                fabs(freq);
        double time_avg = 0.0, gha0 = 0.0, dec0 = 0.0;
        if (!azel)
        {
            time_avg = oskar_telescope_time_average_sec(tel_);
            gha0 = gast - lon0;
            dec0 = lat0;
        }
        double uv_min = oskar_telescope_uv_filter_min(tel_);
        double uv_max = oskar_telescope_uv_filter_max(tel_);
        if (oskar_telescope_uv_filter_units(tel_) == REF_METRES)
        {
            uv_min *= inv_wl;
            uv_max *= inv_wl;
        }
        if (uv_max < 0.0 || uv_max > 3.402823466e38) uv_max = 3.402823466e38;
        const T *ea = gaussian ? col(REF_SKY_SCRATCH_EXT_A) : nullptr,
                *eb = gaussian ? col(REF_SKY_SCRATCH_EXT_B) : nullptr,
                *ec = gaussian ? col(REF_SKY_SCRATCH_EXT_C) : nullptr;
        const size_t out = (size_t) num_baselines() * offset;
        // Point sources without smearing: the FP64-class tensor-core form
        // in FP64 (the dispatcher's branch oskar_cross_correlate.c:
        // 434-455), the integer form in FP32 (:413-433), unless a
        // brightness matrix of the chunk is not positive semi-definite,
        // which they report having added nothing; then, and for every
        // other case, the direct kernels
        bool done = false;
        if (matrix_ && !gaussian && frac_bw == 0.0 && time_avg == 0.0 &&
                (dbl ? use_tc64() : use_tc32()))
        {
            check(st_->tc64ws.ensure(dbl ?
                    oskb_cross_correlate_tc64_workspace_bytes(num_src,
                            num_st_) :
                    oskb_cross_correlate_tc_f_workspace_bytes(num_src,
                            num_st_)), "tensor-core correlation workspace");
            if (!ok()) return;
            if (dbl)
                err = oskb_cross_correlate_tc64_d(h_->casa_phase_convention,
                        num_src, num_st_, (int) out, (const double*) EJ,
                        (const double*) fI, (const double*) fQ,
                        (const double*) fU, (const double*) fV,
                        (const double*) u, (const double*) v, uv_min, uv_max,
                        inv_wl, st_->vis.as<double>(), st_->tc64ws.p,
                        st_->tc64ws.bytes, s_);
            else
                err = oskb_cross_correlate_tc_f(h_->casa_phase_convention,
                        num_src, num_st_, (int) out, (const float*) EJ,
                        (const float*) fI, (const float*) fQ,
                        (const float*) fU, (const float*) fV,
                        (const float*) u, (const float*) v, (float) uv_min,
                        (float) uv_max, (float) inv_wl,
                        st_->vis.as<float>(), st_->tc64ws.p,
                        st_->tc64ws.bytes, s_);
            check(err, "cross-correlation (tensor cores)");
            if (!ok()) return;
            int flags = 0, wait_error = 0;
            check(cudaStreamSynchronize(s_) == cudaSuccess ?
                    oskb_tc_status(st_->tc64ws.p, &flags, &wait_error) :
                    REF_ERR_KERNEL_LAUNCH_FAILURE,
                    "tensor-core correlation status");
            if (!ok()) return;
            if (wait_error)
            {
                fail(REF_ERR_KERNEL_LAUNCH_FAILURE, "tensor-core correlation: "
                        "a bounded device-side wait expired");
                return;
            }
            done = !(flags & 1);
        }
        if (done)
            err = 0;
        else if (dbl && matrix_)
            err = oskb_cross_correlate_d(h_->casa_phase_convention, gaussian,
                    num_src, num_st_, (int) out, (const double*) EJ,
                    (const double*) fI, (const double*) fQ,
                    (const double*) fU, (const double*) fV,
                    (const double*) l, (const double*) m, (const double*) n,
                    (const double*) ea, (const double*) eb,
                    (const double*) ec, (const double*) u, (const double*) v,
                    (const double*) w, (const double*) sx,
                    (const double*) sy, uv_min, uv_max, inv_wl, frac_bw,
                    time_avg, gha0, dec0, st_->vis.as<double>(), s_);
        else if (matrix_)
            err = oskb_cross_correlate_f(h_->casa_phase_convention, gaussian,
                    num_src, num_st_, (int) out, (const float*) EJ,
                    (const float*) fI, (const float*) fQ, (const float*) fU,
                    (const float*) fV, (const float*) l, (const float*) m,
                    (const float*) n, (const float*) ea, (const float*) eb,
                    (const float*) ec, (const float*) u, (const float*) v,
                    (const float*) w, (const float*) sx, (const float*) sy,
                    (float) uv_min, (float) uv_max, (float) inv_wl,
                    (float) frac_bw, (float) time_avg, (float) gha0,
                    (float) dec0, st_->vis.as<float>(), s_);
        else if (dbl)
            err = oskb_cross_correlate_scalar_d(h_->casa_phase_convention,
                    gaussian, num_src, num_st_, (int) out,
                    (const double*) EJ, (const double*) fI,
                    (const double*) l, (const double*) m, (const double*) n,
                    (const double*) ea, (const double*) eb,
                    (const double*) ec, (const double*) u, (const double*) v,
                    (const double*) w, (const double*) sx,
                    (const double*) sy, uv_min, uv_max, inv_wl, frac_bw,
                    time_avg, gha0, dec0, st_->vis.as<double>(), s_);
        else
            err = oskb_cross_correlate_scalar_f(h_->casa_phase_convention,
                    gaussian, num_src, num_st_, (int) out, (const float*) EJ,
                    (const float*) fI, (const float*) l, (const float*) m,
                    (const float*) n, (const float*) ea, (const float*) eb,
                    (const float*) ec, (const float*) u, (const float*) v,
                    (const float*) w, (const float*) sx, (const float*) sy,
                    (float) uv_min, (float) uv_max, (float) inv_wl,
                    (float) frac_bw, (float) time_avg, (float) gha0,
                    (float) dec0, st_->vis.as<float>(), s_);
        check(err, "cross-correlation");
    }
}

template <typename T>
void Runner<T>::run_block(int block_index)
{
    RefDeviceData* d = &h_->d[dev_id_];
    const int total_chunks = h_->num_sky_chunks;
    const int total_chans = h_->num_channels;
    const int total_times = h_->num_time_steps;
    // block extent (run_block.c:55-84)
    const int nbc = (total_chans + h_->max_channels_per_block - 1) /
            h_->max_channels_per_block;
    const int ibc = block_index % nbc, ibt = block_index / nbc;
    blk_.chan_start = ibc * h_->max_channels_per_block;
    int chan_end = blk_.chan_start + h_->max_channels_per_block - 1;
    blk_.time_start = ibt * h_->max_times_per_block;
    int time_end = blk_.time_start + h_->max_times_per_block - 1;
    if (time_end >= total_times) time_end = total_times - 1;
    if (chan_end >= total_chans) chan_end = total_chans - 1;
    blk_.num_times = 1 + time_end - blk_.time_start;
    blk_.num_chans = 1 + chan_end - blk_.chan_start;

    oskar_VisBlock* vb = d->vis_block_cpu[block_index % 2];
    num_st_ = oskar_vis_block_num_stations(vb);
    oskar_vis_block_resize(vb, blk_.num_times, blk_.num_chans, num_st_,
            status_);
    oskar_vis_block_set_start_time_index(vb, blk_.time_start);
    oskar_vis_block_set_start_channel_index(vb, blk_.chan_start);
    if (!ok()) return;
    has_cross_ = oskar_vis_block_has_cross_correlations(vb) != 0;
    has_auto_ = oskar_vis_block_has_auto_correlations(vb) != 0;
    oskar_Mem* xc = oskar_vis_block_cross_correlations(vb);
    oskar_Mem* ac = oskar_vis_block_auto_correlations(vb);
    vis_type_ = oskar_mem_type(xc);
    matrix_ = (vis_type_ & REF_MATRIX) != 0;
    if (num_st_ != oskar_telescope_num_stations(tel_))
    {
        fail(REF_ERR_SETTINGS_TELESCOPE, "station count differs between "
                "the telescope and the visibility block");
        return;
    }
    const size_t xbytes = oskar_mem_length(xc) * elem_bytes(vis_type_);
    const size_t abytes = oskar_mem_length(ac) * elem_bytes(
            oskar_mem_type(ac));
    check(st_->vis.ensure(xbytes), "visibility buffers");
    check(st_->autos.ensure(abytes), "visibility buffers");
    if (!ok()) return;
    if (xbytes) cudaMemsetAsync(st_->vis.p, 0, xbytes, s_);
    if (abytes) cudaMemsetAsync(st_->autos.p, 0, abytes, s_);

    // telescope arrays: true station coordinates (ECEF offsets, or ENU for
    // a drift scan) and cable-length errors, in the simulator's precision
    const int azel = oskar_telescope_phase_centre_coord_type(tel_) ==
            REF_COORDS_AZEL;
    check(st_->st_xyz.ensure((size_t) 3 * num_st_ * sizeof(T)),
            "telescope buffers");
    for (int i = 0; i < 3 && ok(); ++i)
    {
        const oskar_Mem* c = azel ?
                oskar_telescope_station_true_enu_metres_const(tel_, i) :
                oskar_telescope_station_true_offset_ecef_metres_const(tel_,
                i);
        if (!c || (int) oskar_mem_length(c) < num_st_ ||
                (oskar_mem_type(c) & 0x0F) != (sizeof(T) == 8 ? REF_DOUBLE :
                REF_SINGLE))
        {
            fail(REF_ERR_TYPE_MISMATCH, "station coordinates");
            return;
        }
        cudaMemcpyAsync(st_->st_xyz.as<T>() + (size_t) i * num_st_,
                oskar_mem_void_const(c), num_st_ * sizeof(T),
                cudaMemcpyDefault, s_);
    }
    for (int f = 0; f < 2 && ok(); ++f)
    {
        const oskar_Mem* c = oskar_telescope_station_cable_length_error_const(
                tel_, f);
        if (c && (int) oskar_mem_length(c) >= num_st_)
        {
            if ((oskar_mem_type(c) & 0x0F) != (sizeof(T) == 8 ? REF_DOUBLE :
                    REF_SINGLE))
            {
                fail(REF_ERR_TYPE_MISMATCH, "cable-length errors");
                return;
            }
            check(upload(st_->cable[f], c, sizeof(T), s_), "cable errors");
        }
        else if (st_->cable[f].p)
        {
            cudaFree(st_->cable[f].p);
            st_->cable[f] = DevBuf();
        }
    }
    if (oskar_telescope_ionosphere_screen_type(tel_) != 'N' &&
            oskar_telescope_ionosphere_screen_type(tel_) != 0)
    {
        fail(REF_ERR_FUNCTION_NOT_AVAILABLE, "ionospheric screens are not "
                "built in this drop-in");
        return;
    }

    // work units (time, chunk), claimed under the simulator's mutex
    // (run_block.c:88-145)
    while (!h_->coords_only && ok())
    {
        oskar_mutex_lock(h_->mutex);
        const int unit = (h_->work_unit_index)++;
        oskar_mutex_unlock(h_->mutex);
        if (unit >= blk_.num_times * total_chunks || !ok()) break;
        const int i_chunk = unit / blk_.num_times;
        const int i_time = unit - i_chunk * blk_.num_times;
        const int sim_time = blk_.time_start + i_time;
        const RefSky* sky =
                reinterpret_cast<const RefSky*>(h_->sky_chunks[i_chunk]);
        if (i_chunk != d->previous_chunk_index) upload_chunk(sky);
        d->previous_chunk_index = i_chunk;
        if (!ok()) break;
        if (oskar_telescope_harp_data(tel_, h_->freq_start_hz))
        {
            fail(REF_ERR_FUNCTION_NOT_AVAILABLE, "HARP element data are not "
                    "built in this drop-in");
            break;
        }
        int num_src = st_->num_in;
        const T* tab = st_->table.as<T>();
        const int* valid = st_->valid.as<int>();
        if (h_->apply_horizon_clip)
        {
            const double mjd = h_->time_start_mjd_utc +
                    h_->time_inc_sec / 86400.0 * (sim_time + 0.5);
            num_src = horizon_clip(sky, oskar_convert_mjd_to_gast_fast(mjd));
            tab = st_->clip_table.as<T>();
            valid = st_->clip_valid.as<int>();
        }
        for (int c = 0; c < blk_.num_chans && ok(); ++c)
            sim_baselines(sky, num_src, tab, valid, c, i_time,
                    blk_.chan_start + c, sim_time);
    }

    // the block into the host visibility buffer the reference finalises
    if (ok())
    {
        if (xbytes)
            cudaMemcpyAsync(oskar_mem_void(xc), st_->vis.p, xbytes,
                    cudaMemcpyDefault, s_);
        if (abytes)
            cudaMemcpyAsync(oskar_mem_void(ac), st_->autos.p, abytes,
                    cudaMemcpyDefault, s_);
    }
    if (cudaStreamSynchronize(s_) != cudaSuccess)
        check(launch_ok("block", log_), "block");
}

}  // namespace

// oskar/interferometer/oskar_interferometer.h:80-81
DROPIN_EXPORT void oskar_interferometer_run_block(oskar_Interferometer* hh,
        int block_index, int device_id, int* status)
{
    if (!status || *status) return;
    RefInterferometer* h = reinterpret_cast<RefInterferometer*>(hh);
    if (!h)
    {
        *status = REF_ERR_INVALID_ARGUMENT;
        return;
    }
    // The simulator's private layout is mirrored: check it against the
    // reference's accessors before using it.
    if (h->num_devices != oskar_interferometer_num_devices(hh) ||
            h->num_gpus != oskar_interferometer_num_gpus(hh) ||
            h->coords_only != oskar_interferometer_coords_only(hh) ||
            h->casa_phase_convention !=
            oskar_interferometer_casa_phase_convention(hh) ||
            h->log != oskar_interferometer_log(hh))
    {
        *status = REF_ERR_FUNCTION_NOT_AVAILABLE;
        oskar_log_error(oskar_interferometer_log(hh), "B200 drop-in: the "
                "simulator's layout differs from the one this library was "
                "built for");
        return;
    }
    if (!h->header)
    {
        *status = REF_ERR_MEMORY_NOT_ALLOCATED;
        oskar_log_error(h->log, "Simulator not initalised. "
                "Call oskar_interferometer_check_init() first.");
        return;
    }
    if (device_id < 0 || device_id >= h->num_devices)
    {
        *status = REF_ERR_INVALID_ARGUMENT;
        return;
    }
    int ngpu = 0;
    if (cudaGetDeviceCount(&ngpu) != cudaSuccess || ngpu < 1)
    {
        cudaGetLastError();
        *status = REF_ERR_CUDA_NOT_AVAILABLE;
        oskar_log_error(h->log, "B200 drop-in: no CUDA device");
        return;
    }
    State* st = state_for(h, device_id);
    const int dev = (device_id < h->num_gpus && h->gpu_ids) ?
            h->gpu_ids[device_id] : device_id % ngpu;
    if (cudaSetDevice(dev) != cudaSuccess)
    {
        cudaGetLastError();
        *status = REF_ERR_CUDA_NOT_AVAILABLE;
        return;
    }
    if (st->cuda_dev != dev)
    {
        if (cudaStreamCreateWithFlags(&st->stream, cudaStreamNonBlocking) !=
                cudaSuccess ||
                cudaHostAlloc((void**) &st->host_count, sizeof(int),
                cudaHostAllocDefault) != cudaSuccess)
        {
            cudaGetLastError();
            *status = REF_ERR_CUDA_NOT_AVAILABLE;
            return;
        }
        st->cuda_dev = dev;
    }
    if (h->prec == REF_DOUBLE)
        Runner<double>(h, st, device_id, status).run_block(block_index);
    else if (h->prec == REF_SINGLE)
        Runner<float>(h, st, device_id, status).run_block(block_index);
    else
        *status = REF_ERR_BAD_DATA_TYPE;
}

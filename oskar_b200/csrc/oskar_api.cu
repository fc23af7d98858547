// OSKAR-named host API for the hot path (include/oskar_b200_api.h): minimal
// containers and the reference's entry points with their argument checks,
// dispatching to the oskb_* CUDA kernels. Host code only; there is no CPU
// compute path (CPU-located data returns OSKAR_ERR_BAD_LOCATION).
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "common.cuh"
#include "oskar_b200_api.h"

struct oskar_Mem
{
    int type;
    int location;
    size_t num_elements;
    void* data;
};

struct oskar_Jones
{
    oskar_Mem* data;
    int num_stations, num_sources;
};

struct oskar_Telescope
{
    int precision, location, num_stations;
    oskar_Mem* true_offset_ecef[3];
    double channel_bandwidth_hz, time_average_sec;
    int coord_type;
    double lon_rad, lat_rad;
    double uv_min, uv_max;
    int uv_units;
};

namespace {

constexpr double kC0 = 299792458.0;

bool valid_type(int type)
{
    const int base = type & 0x0F;
    if (base != OSKAR_CHAR && base != OSKAR_INT && base != OSKAR_SINGLE &&
            base != OSKAR_DOUBLE)
        return false;
    if ((type & (OSKAR_COMPLEX | OSKAR_MATRIX)) &&
            base != OSKAR_SINGLE && base != OSKAR_DOUBLE)
        return false;
    if ((type & OSKAR_MATRIX) && !(type & OSKAR_COMPLEX)) return false;
    return (type & ~(0x0F | OSKAR_COMPLEX | OSKAR_MATRIX)) == 0;
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------- oskar_Mem
size_t oskar_mem_element_size(int type)
{
    size_t s = 0;
    switch (type & 0x0F)
    {
    case OSKAR_CHAR: s = 1; break;
    case OSKAR_INT: s = sizeof(int); break;
    case OSKAR_SINGLE: s = sizeof(float); break;
    case OSKAR_DOUBLE: s = sizeof(double); break;
    default: return 0;
    }
    if (type & OSKAR_COMPLEX) s *= 2;
    if (type & OSKAR_MATRIX) s *= 4;
    return s;
}

oskar_Mem* oskar_mem_create(int type, int location, size_t num_elements,
        int* status)
{
    if (*status) return nullptr;
    if (!valid_type(type))
    {
        *status = OSKAR_ERR_BAD_DATA_TYPE;
        return nullptr;
    }
    if (location != OSKAR_CPU && location != OSKAR_GPU)
    {
        *status = OSKAR_ERR_BAD_LOCATION;
        return nullptr;
    }
    oskar_Mem* m = (oskar_Mem*) calloc(1, sizeof(oskar_Mem));
    if (!m)
    {
        *status = OSKAR_ERR_MEMORY_ALLOC_FAILURE;
        return nullptr;
    }
    m->type = type;
    m->location = location;
    m->num_elements = num_elements;
    const size_t bytes = num_elements * oskar_mem_element_size(type);
    if (bytes)
    {
        if (location == OSKAR_CPU)
            m->data = calloc(1, bytes);
        else if (cudaMalloc(&m->data, bytes) == cudaSuccess)
            cudaMemset(m->data, 0, bytes);
        else
            m->data = nullptr;
        if (!m->data)
        {
            if (location == OSKAR_GPU)
                oskb::set_last_error("oskar_mem_create", cudaGetLastError());
            free(m);
            *status = OSKAR_ERR_MEMORY_ALLOC_FAILURE;
            return nullptr;
        }
    }
    return m;
}

void oskar_mem_free(oskar_Mem* mem, int* status)
{
    (void) status;  // frees even after an error, as the reference does
    if (!mem) return;
    if (mem->data)
    {
        if (mem->location == OSKAR_CPU) free(mem->data);
        else cudaFree(mem->data);
    }
    free(mem);
}

int oskar_mem_type(const oskar_Mem* mem) { return mem->type; }
int oskar_mem_precision(const oskar_Mem* mem) { return mem->type & 0x0F; }
int oskar_mem_location(const oskar_Mem* mem) { return mem->location; }
size_t oskar_mem_length(const oskar_Mem* mem) { return mem->num_elements; }
int oskar_mem_is_complex(const oskar_Mem* mem)
{
    return (mem->type & OSKAR_COMPLEX) ? 1 : 0;
}
int oskar_mem_is_matrix(const oskar_Mem* mem)
{
    return (mem->type & OSKAR_MATRIX) ? 1 : 0;
}
int oskar_mem_is_double(const oskar_Mem* mem)
{
    return (mem->type & 0x0F) == OSKAR_DOUBLE;
}
void* oskar_mem_void(oskar_Mem* mem) { return mem->data; }
const void* oskar_mem_void_const(const oskar_Mem* mem) { return mem->data; }

void oskar_mem_copy_contents(oskar_Mem* dst, const oskar_Mem* src,
        size_t offset_dst, size_t offset_src, size_t num_elements,
        int* status)
{
    if (*status || num_elements == 0) return;
    if (src->type != dst->type)
    {
        *status = OSKAR_ERR_TYPE_MISMATCH;
        return;
    }
    if (offset_src + num_elements > src->num_elements ||
            offset_dst + num_elements > dst->num_elements)
    {
        *status = OSKAR_ERR_OUT_OF_RANGE;
        return;
    }
    const size_t es = oskar_mem_element_size(src->type);
    if (src->location == OSKAR_CPU && dst->location == OSKAR_CPU)
    {
        memmove((char*) dst->data + offset_dst * es,
                (const char*) src->data + offset_src * es, num_elements * es);
        return;
    }
    const cudaMemcpyKind kind[2][2] = {
        {cudaMemcpyHostToHost, cudaMemcpyHostToDevice},
        {cudaMemcpyDeviceToHost, cudaMemcpyDeviceToDevice}};
    if (cudaMemcpy((char*) dst->data + offset_dst * es,
            (const char*) src->data + offset_src * es, num_elements * es,
            kind[src->location][dst->location]) != cudaSuccess)
    {
        oskb::set_last_error("oskar_mem_copy_contents", cudaGetLastError());
        *status = OSKAR_ERR_MEMORY_COPY_FAILURE;
    }
}

void oskar_mem_clear_contents(oskar_Mem* mem, int* status)
{
    if (*status || !mem->data) return;
    const size_t bytes = mem->num_elements *
            oskar_mem_element_size(mem->type);
    if (mem->location == OSKAR_CPU) memset(mem->data, 0, bytes);
    else if (cudaMemset(mem->data, 0, bytes) != cudaSuccess)
        *status = OSKAR_ERR_MEMORY_COPY_FAILURE;
}

// -------------------------------------------------------------- oskar_Jones
oskar_Jones* oskar_jones_create(int type, int location, int num_stations,
        int num_sources, int* status)
{
    if (*status) return nullptr;
    if (!(type & OSKAR_COMPLEX))
    {
        *status = OSKAR_ERR_BAD_DATA_TYPE;
        return nullptr;
    }
    if (num_stations < 0 || num_sources < 0)
    {
        *status = OSKAR_ERR_INVALID_ARGUMENT;
        return nullptr;
    }
    oskar_Jones* j = (oskar_Jones*) calloc(1, sizeof(oskar_Jones));
    j->num_stations = num_stations;
    j->num_sources = num_sources;
    j->data = oskar_mem_create(type, location,
            (size_t) num_stations * num_sources, status);
    if (*status)
    {
        free(j);
        return nullptr;
    }
    return j;
}

void oskar_jones_free(oskar_Jones* jones, int* status)
{
    if (!jones) return;
    oskar_mem_free(jones->data, status);
    free(jones);
}

oskar_Mem* oskar_jones_mem(oskar_Jones* j) { return j->data; }
const oskar_Mem* oskar_jones_mem_const(const oskar_Jones* j) { return j->data; }
int oskar_jones_num_stations(const oskar_Jones* j) { return j->num_stations; }
int oskar_jones_num_sources(const oskar_Jones* j) { return j->num_sources; }
int oskar_jones_type(const oskar_Jones* j) { return j->data->type; }
int oskar_jones_mem_location(const oskar_Jones* j)
{
    return j->data->location;
}

// ---------------------------------------------------------- oskar_Telescope
oskar_Telescope* oskar_telescope_create(int type, int location,
        int num_stations, int* status)
{
    if (*status) return nullptr;
    if (type != OSKAR_SINGLE && type != OSKAR_DOUBLE)
    {
        *status = OSKAR_ERR_BAD_DATA_TYPE;
        return nullptr;
    }
    oskar_Telescope* t = (oskar_Telescope*) calloc(1, sizeof(oskar_Telescope));
    t->precision = type;
    t->location = location;
    t->num_stations = num_stations;
    for (int i = 0; i < 3; ++i)
        t->true_offset_ecef[i] = oskar_mem_create(type, location,
                num_stations, status);
    t->coord_type = OSKAR_COORDS_RADEC;
    t->uv_max = -1.0;  // no upper limit, as the reference's default
    t->uv_units = OSKAR_WAVELENGTHS;
    if (*status)
    {
        int s = 0;
        oskar_telescope_free(t, &s);
        return nullptr;
    }
    return t;
}

void oskar_telescope_free(oskar_Telescope* t, int* status)
{
    if (!t) return;
    for (int i = 0; i < 3; ++i) oskar_mem_free(t->true_offset_ecef[i], status);
    free(t);
}

int oskar_telescope_num_stations(const oskar_Telescope* t)
{
    return t->num_stations;
}
int oskar_telescope_mem_location(const oskar_Telescope* t)
{
    return t->location;
}
oskar_Mem* oskar_telescope_station_true_offset_ecef_metres(
        oskar_Telescope* t, int dim)
{
    return (dim >= 0 && dim < 3) ? t->true_offset_ecef[dim] : nullptr;
}
void oskar_telescope_set_channel_bandwidth(oskar_Telescope* t, double bw)
{
    t->channel_bandwidth_hz = bw;
}
void oskar_telescope_set_time_average(oskar_Telescope* t, double s)
{
    t->time_average_sec = s;
}
void oskar_telescope_set_phase_centre(oskar_Telescope* t, int coord_type,
        double lon, double lat)
{
    t->coord_type = coord_type;
    t->lon_rad = lon;
    t->lat_rad = lat;
}
void oskar_telescope_set_uv_filter(oskar_Telescope* t, double mn, double mx,
        int units)
{
    t->uv_min = mn;
    t->uv_max = mx;
    t->uv_units = units;
}

}  // extern "C"

namespace {

// OSKAR_CORRELATE: "TC" the tensor-core compensated form (1e-6), "TC64"
// the FP64-class tensor-core form (FP64 accuracy); 0 otherwise.
int tc_mode()
{
    const char* e = getenv("OSKAR_CORRELATE");
    if (!e) return 0;
    if (strcmp(e, "TC") == 0 || strcmp(e, "tc") == 0) return 1;
    if (strcmp(e, "TC64") == 0 || strcmp(e, "tc64") == 0) return 2;
    return 0;
}

const float* F(const oskar_Mem* m)
{
    return m ? static_cast<const float*>(m->data) : nullptr;
}
const double* D(const oskar_Mem* m)
{
    return m ? static_cast<const double*>(m->data) : nullptr;
}

// Grows a device array to at least n elements, keeping its contents
// (the role of oskar_mem_ensure, oskar/mem/src/oskar_mem_ensure.c).
void mem_ensure(oskar_Mem* m, size_t n, int* status)
{
    if (*status || m->num_elements >= n) return;
    int s = 0;
    oskar_Mem* t = oskar_mem_create(m->type, m->location, n, &s);
    if (s) { *status = s; return; }
    oskar_mem_copy_contents(t, m, 0, 0, m->num_elements, &s);
    if (s) { *status = s; oskar_mem_free(t, &s); return; }
    if (m->location == OSKAR_CPU) free(m->data); else cudaFree(m->data);
    m->data = t->data;
    m->num_elements = n;
    free(t);
}

}  // namespace

extern "C" {

// oskar/correlate/src/oskar_cross_correlate.c:20-743 (argument handling and
// checks in the same order; GPU dispatch to the oskb kernels).
void oskar_cross_correlate(int casa, int source_type, int num_sources,
        const oskar_Jones* jones, const oskar_Mem* const src_flux[4],
        const oskar_Mem* const src_dir[3], const oskar_Mem* const src_ext[3],
        const oskar_Telescope* tel, const oskar_Mem* const station_uvw[3],
        double gast, double frequency_hz, int offset_out, oskar_Mem* vis,
        int* status)
{
    double time_avg = 0.0, gha0 = 0.0, dec0 = 0.0;
    if (*status) return;
    const int num_stations = tel->num_stations;
    const int use_extended = (source_type == 1);
    frequency_hz = fabs(frequency_hz);
    const double inv_wavelength = frequency_hz / kC0;
    const double frac_bandwidth = tel->channel_bandwidth_hz / frequency_hz;
    if (tel->coord_type != OSKAR_COORDS_AZEL)
    {
        time_avg = tel->time_average_sec;
        gha0 = gast - tel->lon_rad;
        dec0 = tel->lat_rad;
    }
    double uv_min = tel->uv_min, uv_max = tel->uv_max;
    if (tel->uv_units == OSKAR_METRES)
    {
        uv_min *= inv_wavelength;
        uv_max *= inv_wavelength;
    }
    if (uv_max < 0.0 || uv_max > FLT_MAX) uv_max = FLT_MAX;
    const int location = jones->data->location;
    if (tel->location != location || vis->location != location ||
            station_uvw[0]->location != location ||
            station_uvw[1]->location != location ||
            station_uvw[2]->location != location)
    {
        *status = OSKAR_ERR_LOCATION_MISMATCH;
        return;
    }
    const int jones_type = jones->data->type;
    const int base_type = jones_type & 0x0F;
    if ((vis->type & 0x0F) != base_type ||
            station_uvw[0]->type != base_type ||
            station_uvw[1]->type != base_type ||
            station_uvw[2]->type != base_type || vis->type != jones_type)
    {
        *status = OSKAR_ERR_TYPE_MISMATCH;
        return;
    }
    if (jones->num_sources < num_sources ||
            (int) station_uvw[0]->num_elements != num_stations ||
            (int) station_uvw[1]->num_elements != num_stations ||
            (int) station_uvw[2]->num_elements != num_stations)
    {
        *status = OSKAR_ERR_DIMENSION_MISMATCH;
        return;
    }
    if (location != OSKAR_GPU)
    {
        *status = OSKAR_ERR_BAD_LOCATION;
        return;
    }
    const oskar_Mem* x = tel->true_offset_ecef[0];
    const oskar_Mem* y = tel->true_offset_ecef[1];
    const oskar_Mem *a = use_extended ? src_ext[0] : nullptr,
            *b = use_extended ? src_ext[1] : nullptr,
            *c = use_extended ? src_ext[2] : nullptr;
    switch (vis->type)
    {
    case OSKAR_SINGLE_COMPLEX_MATRIX:
    {
        // OSKAR_CORRELATE=TC: point sources without smearing on the integer
        // tensor-core form (FP32 in and out); nothing is added if a
        // brightness matrix is not positive semi-definite (status flags
        // bit 0), then the direct kernel
        bool done = false;
        if (tc_mode() == 1 && !use_extended && frac_bandwidth == 0.0 &&
                time_avg == 0.0)
        {
            *status = oskb_cross_correlate_tc_f(casa, num_sources,
                    num_stations, offset_out, F(jones->data), F(src_flux[0]),
                    F(src_flux[1]), F(src_flux[2]), F(src_flux[3]),
                    F(station_uvw[0]), F(station_uvw[1]), (float) uv_min,
                    (float) uv_max, (float) inv_wavelength,
                    (float*) vis->data, nullptr, 0, 0);
            int flags = 0, wait_error = 0;
            if (!*status)
                *status = cudaStreamSynchronize(0) == cudaSuccess ?
                        oskb_tc_status(nullptr, &flags, &wait_error) :
                        OSKB_ERR_KERNEL_LAUNCH_FAILURE;
            if (!*status && wait_error)
                *status = OSKB_ERR_KERNEL_LAUNCH_FAILURE;
            done = *status != 0 || !(flags & 1);
        }
        if (!done)
        *status = oskb_cross_correlate_f(casa, use_extended, num_sources,
                num_stations, offset_out, F(jones->data), F(src_flux[0]),
                F(src_flux[1]), F(src_flux[2]), F(src_flux[3]), F(src_dir[0]),
                F(src_dir[1]), F(src_dir[2]), F(a), F(b), F(c),
                F(station_uvw[0]), F(station_uvw[1]), F(station_uvw[2]), F(x),
                F(y), (float) uv_min, (float) uv_max, (float) inv_wavelength,
                (float) frac_bandwidth, (float) time_avg, (float) gha0,
                (float) dec0, (float*) vis->data, 0);
        break;
    }
    case OSKAR_DOUBLE_COMPLEX_MATRIX:
    {
        const int mode = tc_mode();
        const bool point = !use_extended && frac_bandwidth == 0.0 &&
                time_avg == 0.0;
        bool done = false;
        if (mode == 1 && point)
        {
            *status = oskb_cross_correlate_tc_d(casa, num_sources,
                    num_stations, offset_out, D(jones->data), D(src_flux[0]),
                    D(src_flux[1]), D(src_flux[2]), D(src_flux[3]),
                    D(station_uvw[0]), D(station_uvw[1]), uv_min, uv_max,
                    inv_wavelength, (double*) vis->data, nullptr, 0, 0);
            done = true;
        }
        else if (mode == 2 && point)
        {
            // nothing is added if a brightness matrix is not positive
            // semi-definite (status flags bit 0): then the direct kernel
            *status = oskb_cross_correlate_tc64_d(casa, num_sources,
                    num_stations, offset_out, D(jones->data), D(src_flux[0]),
                    D(src_flux[1]), D(src_flux[2]), D(src_flux[3]),
                    D(station_uvw[0]), D(station_uvw[1]), uv_min, uv_max,
                    inv_wavelength, (double*) vis->data, nullptr, 0, 0);
            int flags = 0, wait_error = 0;
            if (!*status)
                *status = cudaStreamSynchronize(0) == cudaSuccess ?
                        oskb_tc_status(nullptr, &flags, &wait_error) :
                        OSKB_ERR_KERNEL_LAUNCH_FAILURE;
            if (!*status && wait_error)
                *status = OSKB_ERR_KERNEL_LAUNCH_FAILURE;
            done = *status != 0 || !(flags & 1);
        }
        if (!done)
            *status = oskb_cross_correlate_d(casa, use_extended, num_sources,
                    num_stations, offset_out, D(jones->data), D(src_flux[0]),
                    D(src_flux[1]), D(src_flux[2]), D(src_flux[3]),
                    D(src_dir[0]), D(src_dir[1]), D(src_dir[2]), D(a), D(b),
                    D(c), D(station_uvw[0]), D(station_uvw[1]),
                    D(station_uvw[2]), D(x), D(y), uv_min, uv_max,
                    inv_wavelength, frac_bandwidth, time_avg, gha0, dec0,
                    (double*) vis->data, 0);
        break;
    }
    case OSKAR_SINGLE_COMPLEX:
        *status = oskb_cross_correlate_scalar_f(casa, use_extended,
                num_sources, num_stations, offset_out, F(jones->data),
                F(src_flux[0]), F(src_dir[0]), F(src_dir[1]), F(src_dir[2]),
                F(a), F(b), F(c), F(station_uvw[0]), F(station_uvw[1]),
                F(station_uvw[2]), F(x), F(y), (float) uv_min, (float) uv_max,
                (float) inv_wavelength, (float) frac_bandwidth,
                (float) time_avg, (float) gha0, (float) dec0,
                (float*) vis->data, 0);
        break;
    case OSKAR_DOUBLE_COMPLEX:
        *status = oskb_cross_correlate_scalar_d(casa, use_extended,
                num_sources, num_stations, offset_out, D(jones->data),
                D(src_flux[0]), D(src_dir[0]), D(src_dir[1]), D(src_dir[2]),
                D(a), D(b), D(c), D(station_uvw[0]), D(station_uvw[1]),
                D(station_uvw[2]), D(x), D(y), uv_min, uv_max,
                inv_wavelength, frac_bandwidth, time_avg, gha0, dec0,
                (double*) vis->data, 0);
        break;
    default:
        *status = OSKAR_ERR_BAD_DATA_TYPE;
    }
}

// oskar/correlate/src/oskar_auto_correlate.c:22-80
void oskar_auto_correlate(int num_sources, const oskar_Jones* jones,
        const oskar_Mem* const src_flux[4], int offset_out, oskar_Mem* vis,
        int* status)
{
    if (*status) return;
    const oskar_Mem* J = jones->data;
    if (vis->location != J->location)
    {
        *status = OSKAR_ERR_LOCATION_MISMATCH;
        return;
    }
    if (J->type != vis->type)
    {
        *status = OSKAR_ERR_TYPE_MISMATCH;
        return;
    }
    if (jones->num_sources < num_sources)
    {
        *status = OSKAR_ERR_DIMENSION_MISMATCH;
        return;
    }
    if (J->location != OSKAR_GPU)
    {
        *status = OSKAR_ERR_BAD_LOCATION;
        return;
    }
    const int ns = jones->num_stations;
    switch (vis->type)
    {
    case OSKAR_SINGLE_COMPLEX_MATRIX:
    case OSKAR_SINGLE_COMPLEX:
        *status = oskb_auto_correlate_f(oskar_mem_is_matrix(vis),
                num_sources, ns, offset_out, F(J), F(src_flux[0]),
                F(src_flux[1]), F(src_flux[2]), F(src_flux[3]),
                (float*) vis->data, 0);
        break;
    case OSKAR_DOUBLE_COMPLEX_MATRIX:
    case OSKAR_DOUBLE_COMPLEX:
        *status = oskb_auto_correlate_d(oskar_mem_is_matrix(vis),
                num_sources, ns, offset_out, D(J), D(src_flux[0]),
                D(src_flux[1]), D(src_flux[2]), D(src_flux[3]),
                (double*) vis->data, 0);
        break;
    default:
        *status = OSKAR_ERR_BAD_DATA_TYPE;
    }
}

// oskar/mem/src/oskar_mem_multiply.c:36-314 (inputs on another location are
// copied to the output's location first, as the reference does).
void oskar_mem_multiply(oskar_Mem* out, const oskar_Mem* in1,
        const oskar_Mem* in2, size_t offset_out, size_t offset_in1,
        size_t offset_in2, size_t num_elements, int* status)
{
    if (num_elements == 0 || *status) return;
    const int location = out->location;
    oskar_Mem *t1 = nullptr, *t2 = nullptr;
    const oskar_Mem *a = in1, *b = in2;
    if (in1->location != location)
    {
        t1 = oskar_mem_create(in1->type, location, in1->num_elements, status);
        oskar_mem_copy_contents(t1, in1, 0, 0, in1->num_elements, status);
        a = t1;
    }
    if (in2->location != location)
    {
        t2 = oskar_mem_create(in2->type, location, in2->num_elements, status);
        oskar_mem_copy_contents(t2, in2, 0, 0, in2->num_elements, status);
        b = t2;
    }
    int kind = -1;
    const int prec = out->type & 0x0F;
    if (!*status)
    {
        if ((a->type & 0x0F) != prec || (b->type & 0x0F) != prec)
            *status = OSKAR_ERR_TYPE_MISMATCH;
        else if (out->type == a->type && out->type == b->type)
            kind = (out->type & OSKAR_MATRIX) ? OSKB_MUL_MM_M :
                   (out->type & OSKAR_COMPLEX) ? OSKB_MUL_CC_C : OSKB_MUL_RR_R;
        else if (out->type & OSKAR_MATRIX)
        {
            const bool ac = (a->type & OSKAR_COMPLEX) &&
                    !(a->type & OSKAR_MATRIX);
            const bool bc = (b->type & OSKAR_COMPLEX) &&
                    !(b->type & OSKAR_MATRIX);
            if (ac && bc) kind = OSKB_MUL_CC_M;
            else if (ac && b->type == out->type) kind = OSKB_MUL_CM_M;
            else if (a->type == out->type && bc) kind = OSKB_MUL_MC_M;
            else *status = OSKAR_ERR_TYPE_MISMATCH;
        }
        else
            *status = OSKAR_ERR_TYPE_MISMATCH;
    }
    if (!*status && location != OSKAR_GPU) *status = OSKAR_ERR_BAD_LOCATION;
    if (!*status)
    {
        if (prec == OSKAR_DOUBLE)
            *status = oskb_mem_multiply_d(kind, offset_in1, offset_in2,
                    offset_out, num_elements, D(a), D(b),
                    (double*) out->data, 0);
        else if (prec == OSKAR_SINGLE)
            *status = oskb_mem_multiply_f(kind, offset_in1, offset_in2,
                    offset_out, num_elements, F(a), F(b),
                    (float*) out->data, 0);
        else
            *status = OSKAR_ERR_BAD_DATA_TYPE;
    }
    int s = 0;
    oskar_mem_free(t1, &s);
    oskar_mem_free(t2, &s);
}

// oskar/interferometer/src/oskar_jones_join.c:13-41
void oskar_jones_join(oskar_Jones* j3, oskar_Jones* j1, const oskar_Jones* j2,
        int* status)
{
    if (*status) return;
    if (!j3) j3 = j1;
    if (j1->num_sources != j2->num_sources ||
            j1->num_sources != j3->num_sources ||
            j1->num_stations != j2->num_stations ||
            j1->num_stations != j3->num_stations)
    {
        *status = OSKAR_ERR_DIMENSION_MISMATCH;
        return;
    }
    const size_t n = (size_t) j1->num_sources * j1->num_stations;
    oskar_mem_multiply(j3->data, j1->data, j2->data, 0, 0, 0, n, status);
}

// oskar/interferometer/src/oskar_jones_apply_cable_length_errors.c:23-141.
// Error arrays must have the Jones array's precision and location (the
// reference launches without checking them).
void oskar_jones_apply_cable_length_errors(oskar_Jones* jones,
        double frequency_hz, const oskar_Mem* errors_x,
        const oskar_Mem* errors_y, int* status)
{
    if (*status) return;
    if (!errors_x && !errors_y) return;
    const oskar_Mem* J = jones->data;
    const int precision = J->type & 0x0F;
    const int num_stations = jones->num_stations;
    if ((errors_x && (int) errors_x->num_elements < num_stations) ||
            (errors_y && (int) errors_y->num_elements < num_stations))
    {
        *status = OSKAR_ERR_DIMENSION_MISMATCH;
        return;
    }
    const oskar_Mem* e[2] = {errors_x, errors_y};
    for (const oskar_Mem* m : e)
    {
        if (!m) continue;
        if (m->location != J->location)
        {
            *status = OSKAR_ERR_LOCATION_MISMATCH;
            return;
        }
        if (m->type != precision)
        {
            *status = OSKAR_ERR_TYPE_MISMATCH;
            return;
        }
    }
    if (J->location != OSKAR_GPU)
    {
        *status = OSKAR_ERR_BAD_LOCATION;
        return;
    }
    const int matrix = (J->type & OSKAR_MATRIX) != 0;
    if (!(J->type & OSKAR_COMPLEX))
    {
        *status = OSKAR_ERR_BAD_DATA_TYPE;
        return;
    }
    const double k = 2.0 * M_PI * frequency_hz / kC0;
    if (precision == OSKAR_DOUBLE)
        *status = oskb_jones_apply_cable_length_errors_d(matrix,
                jones->num_sources, num_stations, k,
                errors_x ? (const double*) errors_x->data : nullptr,
                errors_y ? (const double*) errors_y->data : nullptr,
                (double*) J->data, 0);
    else
        *status = oskb_jones_apply_cable_length_errors_f(matrix,
                jones->num_sources, num_stations, (float) k,
                errors_x ? (const float*) errors_x->data : nullptr,
                errors_y ? (const float*) errors_y->data : nullptr,
                (float*) J->data, 0);
}

// oskar/interferometer/src/oskar_jones_apply_station_gains.c:23-121.
// The gains must have the Jones array's type and location (the reference
// launches by the gains' type alone).
void oskar_jones_apply_station_gains(oskar_Jones* jones, oskar_Mem* gains,
        int* status)
{
    if (*status) return;
    const oskar_Mem* J = jones->data;
    if ((int) gains->num_elements < jones->num_stations)
    {
        *status = OSKAR_ERR_DIMENSION_MISMATCH;
        return;
    }
    if (gains->location != J->location)
    {
        *status = OSKAR_ERR_LOCATION_MISMATCH;
        return;
    }
    if (gains->type != J->type)
    {
        *status = OSKAR_ERR_TYPE_MISMATCH;
        return;
    }
    if (J->location != OSKAR_GPU)
    {
        *status = OSKAR_ERR_BAD_LOCATION;
        return;
    }
    if (!(J->type & OSKAR_COMPLEX))
    {
        *status = OSKAR_ERR_BAD_DATA_TYPE;
        return;
    }
    const int matrix = (J->type & OSKAR_MATRIX) != 0;
    if ((J->type & 0x0F) == OSKAR_DOUBLE)
        *status = oskb_jones_apply_station_gains_d(matrix, jones->num_sources,
                jones->num_stations, (const double*) gains->data,
                (double*) J->data, 0);
    else
        *status = oskb_jones_apply_station_gains_f(matrix, jones->num_sources,
                jones->num_stations, (const float*) gains->data,
                (float*) J->data, 0);
}

// oskar/telescope/station/src/oskar_evaluate_element_weights_errors.c:
// 19-110: the same location, type and length checks, then the random
// errors on the device.
void oskar_evaluate_element_weights_errors(int num_elements,
        const oskar_Mem* gain, const oskar_Mem* gain_error,
        const oskar_Mem* phase, const oskar_Mem* phase_error,
        unsigned int random_seed, int time_index, int station_id,
        oskar_Mem* errors, int* status)
{
    if (*status) return;
    const int location = errors->location;
    const int precision = errors->type & 0x0F;
    if (gain->location != location || gain_error->location != location ||
            phase->location != location || phase_error->location != location)
    {
        *status = OSKAR_ERR_LOCATION_MISMATCH;
        return;
    }
    if (gain->type != precision || phase->type != precision ||
            gain_error->type != precision || phase_error->type != precision)
    {
        *status = OSKAR_ERR_TYPE_MISMATCH;
        return;
    }
    if ((int) errors->num_elements < num_elements ||
            (int) gain->num_elements < num_elements ||
            (int) gain_error->num_elements < num_elements ||
            (int) phase->num_elements < num_elements ||
            (int) phase_error->num_elements < num_elements)
    {
        *status = OSKAR_ERR_DIMENSION_MISMATCH;
        return;
    }
    if (location != OSKAR_GPU)
    {
        *status = OSKAR_ERR_BAD_LOCATION;
        return;
    }
    if (errors->type == OSKAR_DOUBLE_COMPLEX)
        *status = oskb_evaluate_element_weights_errors_d(num_elements,
                D(gain), D(gain_error), D(phase), D(phase_error),
                random_seed, time_index, station_id, (double*) errors->data,
                0);
    else if (errors->type == OSKAR_SINGLE_COMPLEX)
        *status = oskb_evaluate_element_weights_errors_f(num_elements,
                (const float*) gain->data, (const float*) gain_error->data,
                (const float*) phase->data, (const float*) phase_error->data,
                random_seed, time_index, station_id, (float*) errors->data,
                0);
    else
        *status = OSKAR_ERR_BAD_DATA_TYPE;
}

// oskar/interferometer/src/oskar_evaluate_jones_K.c:19-157
void oskar_evaluate_jones_K(oskar_Jones* K, int num_sources,
        const oskar_Mem* l, const oskar_Mem* m, const oskar_Mem* n,
        const oskar_Mem* u, const oskar_Mem* v, const oskar_Mem* w,
        double frequency_hz, const oskar_Mem* source_filter,
        double source_filter_min, double source_filter_max,
        int ignore_w_components, int* status)
{
    if (*status) return;
    const int type = K->data->type;
    const int precision = type & 0x0F;
    const int location = K->data->location;
    const int num_stations = K->num_stations;
    const double wavenumber = 2.0 * M_PI * frequency_hz / kC0;
    if (l->location != location || m->location != location ||
            n->location != location || source_filter->location != location ||
            u->location != location || v->location != location ||
            w->location != location)
    {
        *status = OSKAR_ERR_LOCATION_MISMATCH;
        return;
    }
    if (precision != l->type || precision != m->type ||
            precision != n->type || precision != u->type ||
            precision != v->type || precision != w->type ||
            precision != source_filter->type)
    {
        *status = OSKAR_ERR_TYPE_MISMATCH;
        return;
    }
    if (location != OSKAR_GPU)
    {
        *status = OSKAR_ERR_BAD_LOCATION;
        return;
    }
    if (type == OSKAR_SINGLE_COMPLEX)
        *status = oskb_evaluate_jones_K_f(num_sources, F(l), F(m), F(n),
                num_stations, F(u), F(v), F(w), (float) wavenumber,
                F(source_filter), (float) source_filter_min,
                (float) source_filter_max, ignore_w_components,
                (float*) K->data->data, 0);
    else if (type == OSKAR_DOUBLE_COMPLEX)
        *status = oskb_evaluate_jones_K_d(num_sources, D(l), D(m), D(n),
                num_stations, D(u), D(v), D(w), wavenumber,
                D(source_filter), source_filter_min, source_filter_max,
                ignore_w_components, (double*) K->data->data, 0);
    else
        *status = OSKAR_ERR_BAD_DATA_TYPE;
}

// oskar/math/src/oskar_dftw.c:42-374
void oskar_dftw(int normalise, int num_in, double wavenumber,
        const oskar_Mem* weights_in, const oskar_Mem* x_in,
        const oskar_Mem* y_in, const oskar_Mem* z_in, int offset_coord_out,
        int num_out, const oskar_Mem* x_out, const oskar_Mem* y_out,
        const oskar_Mem* z_out, const oskar_Mem* data_idx,
        const oskar_Mem* data, int eval_x, int eval_y, int offset_out,
        oskar_Mem* output, int* status)
{
    if (*status) return;
    const int location = output->location;
    const int type = output->type & 0x0F;
    const int is_3d = (z_in != nullptr && z_out != nullptr);
    const int is_matrix = oskar_mem_is_matrix(output);
    const double norm_factor = normalise ? 1.0 / num_in : 1.0;
    if (!oskar_mem_is_complex(output) || !oskar_mem_is_complex(weights_in) ||
            oskar_mem_is_matrix(weights_in))
    {
        *status = OSKAR_ERR_BAD_DATA_TYPE;
        return;
    }
    if (data->location != location || weights_in->location != location ||
            x_in->location != location || y_in->location != location ||
            x_out->location != location || y_out->location != location)
    {
        *status = OSKAR_ERR_LOCATION_MISMATCH;
        return;
    }
    if ((weights_in->type & 0x0F) != type || x_in->type != type ||
            y_in->type != type || x_out->type != type ||
            y_out->type != type)
    {
        *status = OSKAR_ERR_TYPE_MISMATCH;
        return;
    }
    if (!oskar_mem_is_complex(data) || data->type != output->type)
    {
        *status = OSKAR_ERR_TYPE_MISMATCH;
        return;
    }
    if (is_3d)
    {
        if (z_in->location != location || z_out->location != location)
        {
            *status = OSKAR_ERR_LOCATION_MISMATCH;
            return;
        }
        if (z_in->type != type || z_out->type != type)
        {
            *status = OSKAR_ERR_TYPE_MISMATCH;
            return;
        }
    }
    if (location != OSKAR_GPU)
    {
        *status = OSKAR_ERR_BAD_LOCATION;
        return;
    }
    mem_ensure(output, (size_t) offset_out + num_out, status);
    if (*status) return;
    const int* idx = data_idx ? (const int*) data_idx->data : nullptr;
    if (type == OSKAR_DOUBLE)
        *status = oskb_dftw_d(is_matrix, num_in, wavenumber, D(weights_in),
                D(x_in), D(y_in), is_3d ? D(z_in) : nullptr,
                offset_coord_out, num_out, D(x_out), D(y_out),
                is_3d ? D(z_out) : nullptr, idx, D(data), eval_x, eval_y,
                offset_out, (double*) output->data, norm_factor, 0);
    else if (type == OSKAR_SINGLE)
        *status = oskb_dftw_f(is_matrix, num_in, (float) wavenumber,
                F(weights_in), F(x_in), F(y_in), is_3d ? F(z_in) : nullptr,
                offset_coord_out, num_out, F(x_out), F(y_out),
                is_3d ? F(z_out) : nullptr, idx, F(data), eval_x, eval_y,
                offset_out, (float*) output->data, (float) norm_factor, 0);
    else
        *status = OSKAR_ERR_BAD_DATA_TYPE;
}

// oskar/convert/src/oskar_convert_ecef_to_station_uvw.c (FP64 on the GPU)
void oskar_convert_ecef_to_station_uvw(int num_stations, const oskar_Mem* x,
        const oskar_Mem* y, const oskar_Mem* z, double ra0_rad,
        double dec0_rad, double gast, int ignore_w_components,
        int offset_out, oskar_Mem* u, oskar_Mem* v, oskar_Mem* w, int* status)
{
    if (*status) return;
    const int type = x->type, location = x->location;
    if (y->location != location || z->location != location ||
            u->location != location || v->location != location ||
            w->location != location)
    {
        *status = OSKAR_ERR_LOCATION_MISMATCH;
        return;
    }
    if (y->type != type || z->type != type || u->type != type ||
            v->type != type || w->type != type)
    {
        *status = OSKAR_ERR_TYPE_MISMATCH;
        return;
    }
    if (location != OSKAR_GPU)
    {
        *status = OSKAR_ERR_BAD_LOCATION;
        return;
    }
    if (type != OSKAR_DOUBLE)
    {
        *status = OSKAR_ERR_BAD_DATA_TYPE;
        return;
    }
    mem_ensure(u, (size_t) offset_out + num_stations, status);
    mem_ensure(v, (size_t) offset_out + num_stations, status);
    mem_ensure(w, (size_t) offset_out + num_stations, status);
    if (*status) return;
    *status = oskb_convert_ecef_to_station_uvw_d(num_stations, D(x), D(y),
            D(z), ra0_rad, dec0_rad, gast, ignore_w_components, offset_out,
            (double*) u->data, (double*) v->data, (double*) w->data, 0);
}

}  // extern "C"

namespace {

// Common checks of the conversion wrappers: same location and precision
// for every array, GPU only, FP32 or FP64.
int check_arrays(const oskar_Mem* const* a, int n, int* type)
{
    const oskar_Mem* first = nullptr;
    for (int i = 0; i < n; ++i)
    {
        if (!a[i]) continue;
        if (!first) { first = a[i]; continue; }
        if (a[i]->location != first->location)
            return OSKAR_ERR_LOCATION_MISMATCH;
        if (a[i]->type != first->type) return OSKAR_ERR_TYPE_MISMATCH;
    }
    if (!first) return OSKAR_ERR_INVALID_ARGUMENT;
    if (first->location != OSKAR_GPU) return OSKAR_ERR_BAD_LOCATION;
    if (first->type != OSKAR_DOUBLE && first->type != OSKAR_SINGLE)
        return OSKAR_ERR_BAD_DATA_TYPE;
    *type = first->type;
    return 0;
}

}  // namespace

extern "C" {

// oskar/convert/src/oskar_convert_station_uvw_to_baseline_uvw.c:34-100
void oskar_convert_station_uvw_to_baseline_uvw(int use_casa_phase_convention,
        int num_stations, int offset_in, const oskar_Mem* u,
        const oskar_Mem* v, const oskar_Mem* w, int offset_out,
        oskar_Mem* uu, oskar_Mem* vv, oskar_Mem* ww, int* status)
{
    if (*status) return;
    const oskar_Mem* all[6] = {u, v, w, uu, vv, ww};
    int type = 0;
    for (int i = 0; i < 6; ++i)
        if (!all[i]) { *status = OSKAR_ERR_INVALID_ARGUMENT; return; }
    if ((*status = check_arrays(all, 6, &type))) return;
    const size_t nbl = (size_t) num_stations * (num_stations - 1) / 2;
    mem_ensure(uu, offset_out + nbl, status);
    mem_ensure(vv, offset_out + nbl, status);
    mem_ensure(ww, offset_out + nbl, status);
    if (*status) return;
    if (type == OSKAR_DOUBLE)
        *status = oskb_convert_station_uvw_to_baseline_uvw_d(
                use_casa_phase_convention, num_stations, offset_in, D(u),
                D(v), D(w), offset_out, (double*) uu->data,
                (double*) vv->data, (double*) ww->data, 0);
    else
        *status = oskb_convert_station_uvw_to_baseline_uvw_f(
                use_casa_phase_convention, num_stations, offset_in, F(u),
                F(v), F(w), offset_out, (float*) uu->data,
                (float*) vv->data, (float*) ww->data, 0);
}

// oskar/convert/oskar_convert_lon_lat_to_relative_directions.h:154-157
// (n may be NULL: the 2-D form)
void oskar_convert_lon_lat_to_relative_directions(int num_points,
        const oskar_Mem* lon_rad, const oskar_Mem* lat_rad, double lon0_rad,
        double lat0_rad, oskar_Mem* l, oskar_Mem* m, oskar_Mem* n,
        int* status)
{
    if (*status) return;
    if (!lon_rad || !lat_rad || !l || !m)
    {
        *status = OSKAR_ERR_INVALID_ARGUMENT;
        return;
    }
    const oskar_Mem* all[5] = {lon_rad, lat_rad, l, m, n};
    int type = 0;
    if ((*status = check_arrays(all, 5, &type))) return;
    mem_ensure(l, num_points, status);
    mem_ensure(m, num_points, status);
    if (n) mem_ensure(n, num_points, status);
    if (*status) return;
    if (type == OSKAR_DOUBLE)
        *status = oskb_convert_lon_lat_to_relative_directions_d(num_points,
                D(lon_rad), D(lat_rad), lon0_rad, lat0_rad,
                (double*) l->data, (double*) m->data,
                n ? (double*) n->data : nullptr, 0);
    else
        *status = oskb_convert_lon_lat_to_relative_directions_f(num_points,
                F(lon_rad), F(lat_rad), lon0_rad, lat0_rad,
                (float*) l->data, (float*) m->data,
                n ? (float*) n->data : nullptr, 0);
}

// oskar/convert/oskar_convert_apparent_ra_dec_to_enu_directions.h:41-45
void oskar_convert_apparent_ra_dec_to_enu_directions(int num_points,
        const oskar_Mem* ra_rad, const oskar_Mem* dec_rad, double lst_rad,
        double latitude_rad, int offset_out, oskar_Mem* x, oskar_Mem* y,
        oskar_Mem* z, int* status)
{
    if (*status) return;
    if (!ra_rad || !dec_rad || !x || !y || !z)
    {
        *status = OSKAR_ERR_INVALID_ARGUMENT;
        return;
    }
    const oskar_Mem* all[5] = {ra_rad, dec_rad, x, y, z};
    int type = 0;
    if ((*status = check_arrays(all, 5, &type))) return;
    mem_ensure(x, (size_t) offset_out + num_points, status);
    mem_ensure(y, (size_t) offset_out + num_points, status);
    mem_ensure(z, (size_t) offset_out + num_points, status);
    if (*status || num_points == 0) return;
    // one station: its LST and latitude as one-element device arrays
    double h[2] = {lst_rad, latitude_rad};
    double* d = nullptr;
    if (cudaMalloc(&d, sizeof(h)) != cudaSuccess ||
            cudaMemcpy(d, h, sizeof(h), cudaMemcpyHostToDevice) !=
            cudaSuccess)
    {
        oskb::set_last_error("oskar_convert_apparent_ra_dec_to_enu_"
                "directions", cudaGetLastError());
        cudaFree(d);
        *status = OSKAR_ERR_MEMORY_ALLOC_FAILURE;
        return;
    }
    if (type == OSKAR_DOUBLE)
        *status = oskb_convert_ra_dec_to_enu_directions_d(num_points,
                D(ra_rad), D(dec_rad), 1, d, d + 1,
                (double*) x->data + offset_out,
                (double*) y->data + offset_out,
                (double*) z->data + offset_out, 0);
    else
        *status = oskb_convert_ra_dec_to_enu_directions_f(num_points,
                F(ra_rad), F(dec_rad), 1, d, d + 1,
                (float*) x->data + offset_out, (float*) y->data + offset_out,
                (float*) z->data + offset_out, 0);
    cudaStreamSynchronize(0);
    cudaFree(d);
}

}  // extern "C"

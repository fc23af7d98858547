/*
 * OSKAR-named host API for the visibility hot path, implemented by
 * liboskar_b200.so on top of the oskb_* kernels (include/oskar_b200.h).
 *
 * The functions below keep the names, argument meaning, status-code
 * behaviour and data layouts of the reference's functions for this path, so
 * code written against the reference (for these calls) runs unchanged:
 *  - status: every function returns immediately if *status != 0 on entry
 *    and reports errors with the reference's codes (oskar/oskar_global.h);
 *  - type codes are the reference's (oskar/binary/oskar_binary_data_types.h:
 *    OSKAR_SINGLE 0x04, OSKAR_DOUBLE 0x08, OSKAR_COMPLEX 0x20,
 *    OSKAR_MATRIX 0x40) and locations OSKAR_CPU 0 / OSKAR_GPU 1
 *    (oskar/mem/oskar_mem.h:38-41).
 * The containers (oskar_Mem, oskar_Jones, oskar_Telescope) are this
 * library's own minimal implementations of the reference's opaque types,
 * with the accessors this path uses. Compute functions run on OSKAR_GPU
 * data only: there is no CPU implementation here, and CPU-located inputs
 * return OSKAR_ERR_BAD_LOCATION (the reference's CPU path stays the
 * reference's).
 */
#ifndef OSKAR_B200_API_H_
#define OSKAR_B200_API_H_

#include <stddef.h>

#include "oskar_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

enum oskb_oskar_type_codes
{
    OSKAR_CHAR = 0x01, OSKAR_INT = 0x02, OSKAR_SINGLE = 0x04,
    OSKAR_DOUBLE = 0x08, OSKAR_COMPLEX = 0x20, OSKAR_MATRIX = 0x40,
    OSKAR_SINGLE_COMPLEX = 0x24, OSKAR_DOUBLE_COMPLEX = 0x28,
    OSKAR_SINGLE_COMPLEX_MATRIX = 0x64, OSKAR_DOUBLE_COMPLEX_MATRIX = 0x68
};
enum oskb_oskar_locations { OSKAR_CPU = 0, OSKAR_GPU = 1 };
enum oskb_oskar_units { OSKAR_METRES = 0, OSKAR_WAVELENGTHS = 1 };
/* oskar/oskar_global.h:89-97 */
enum oskb_oskar_coords
{
    OSKAR_COORDS_REL_DIR = 0, OSKAR_COORDS_ENU_DIR = 1, OSKAR_COORDS_RADEC = 2,
    OSKAR_COORDS_HADEC = 3, OSKAR_COORDS_AZEL = 4, OSKAR_COORDS_GALACTIC = 5
};
enum oskb_oskar_errors
{
    OSKAR_ERR_INVALID_ARGUMENT = -3, OSKAR_ERR_FUNCTION_NOT_AVAILABLE = -4,
    OSKAR_ERR_OUT_OF_RANGE = -5, OSKAR_ERR_MEMORY_ALLOC_FAILURE = -6,
    OSKAR_ERR_MEMORY_COPY_FAILURE = -7, OSKAR_ERR_TYPE_MISMATCH = -9,
    OSKAR_ERR_LOCATION_MISMATCH = -10, OSKAR_ERR_DIMENSION_MISMATCH = -11,
    OSKAR_ERR_BAD_DATA_TYPE = -13, OSKAR_ERR_BAD_LOCATION = -14,
    OSKAR_ERR_KERNEL_LAUNCH_FAILURE = -18
};

typedef struct oskar_Mem oskar_Mem;
typedef struct oskar_Jones oskar_Jones;
typedef struct oskar_Telescope oskar_Telescope;

/* ---- oskar_Mem (oskar/mem/oskar_mem.h) ---- */
OSKB_API oskar_Mem* oskar_mem_create(int type, int location,
        size_t num_elements, int* status);
OSKB_API void oskar_mem_free(oskar_Mem* mem, int* status);
OSKB_API int oskar_mem_type(const oskar_Mem* mem);
OSKB_API int oskar_mem_precision(const oskar_Mem* mem);
OSKB_API int oskar_mem_location(const oskar_Mem* mem);
OSKB_API size_t oskar_mem_length(const oskar_Mem* mem);
OSKB_API int oskar_mem_is_complex(const oskar_Mem* mem);
OSKB_API int oskar_mem_is_matrix(const oskar_Mem* mem);
OSKB_API int oskar_mem_is_double(const oskar_Mem* mem);
OSKB_API size_t oskar_mem_element_size(int type);
OSKB_API void* oskar_mem_void(oskar_Mem* mem);
OSKB_API const void* oskar_mem_void_const(const oskar_Mem* mem);
OSKB_API void oskar_mem_copy_contents(oskar_Mem* dst, const oskar_Mem* src,
        size_t offset_dst, size_t offset_src, size_t num_elements,
        int* status);
OSKB_API void oskar_mem_clear_contents(oskar_Mem* mem, int* status);

/* ---- oskar_Jones (oskar/interferometer/oskar_jones.h) ---- */
OSKB_API oskar_Jones* oskar_jones_create(int type, int location,
        int num_stations, int num_sources, int* status);
OSKB_API void oskar_jones_free(oskar_Jones* jones, int* status);
OSKB_API oskar_Mem* oskar_jones_mem(oskar_Jones* jones);
OSKB_API const oskar_Mem* oskar_jones_mem_const(const oskar_Jones* jones);
OSKB_API int oskar_jones_num_stations(const oskar_Jones* jones);
OSKB_API int oskar_jones_num_sources(const oskar_Jones* jones);
OSKB_API int oskar_jones_type(const oskar_Jones* jones);
OSKB_API int oskar_jones_mem_location(const oskar_Jones* jones);

/* ---- oskar_Telescope: the fields the correlator reads
 * (oskar/telescope/oskar_telescope_accessors.h) ---- */
OSKB_API oskar_Telescope* oskar_telescope_create(int type, int location,
        int num_stations, int* status);
OSKB_API void oskar_telescope_free(oskar_Telescope* tel, int* status);
OSKB_API int oskar_telescope_num_stations(const oskar_Telescope* tel);
OSKB_API int oskar_telescope_mem_location(const oskar_Telescope* tel);
OSKB_API oskar_Mem* oskar_telescope_station_true_offset_ecef_metres(
        oskar_Telescope* tel, int dim);
OSKB_API void oskar_telescope_set_channel_bandwidth(oskar_Telescope* tel,
        double bandwidth_hz);
OSKB_API void oskar_telescope_set_time_average(oskar_Telescope* tel,
        double time_average_sec);
OSKB_API void oskar_telescope_set_phase_centre(oskar_Telescope* tel,
        int coord_type, double longitude_rad, double latitude_rad);
OSKB_API void oskar_telescope_set_uv_filter(oskar_Telescope* tel,
        double uv_filter_min, double uv_filter_max, int units);

/* ---- hot-path functions ---- */
/* oskar/correlate/oskar_cross_correlate.h:49-63. Point sources without
 * smearing use the tensor-core kernel when the environment variable
 * OSKAR_CORRELATE is "TC" (relative error <= 1e-6 instead of FP64's
 * 1e-12; positive semi-definite brightness required); every other case, and
 * the default, uses the direct kernel. */
OSKB_API void oskar_cross_correlate(int use_casa_phase_convention,
        int source_type, int num_sources, const oskar_Jones* jones,
        const oskar_Mem* const src_flux[4], const oskar_Mem* const src_dir[3],
        const oskar_Mem* const src_ext[3], const oskar_Telescope* tel,
        const oskar_Mem* const station_uvw[3], double gast,
        double frequency_hz, int offset_out, oskar_Mem* vis, int* status);
/* oskar/correlate/oskar_auto_correlate.h:37 */
OSKB_API void oskar_auto_correlate(int num_sources, const oskar_Jones* jones,
        const oskar_Mem* const src_flux[4], int offset_out, oskar_Mem* vis,
        int* status);
/* oskar/interferometer/oskar_jones_join.h:69 */
OSKB_API void oskar_jones_join(oskar_Jones* j3, oskar_Jones* j1,
        const oskar_Jones* j2, int* status);
/* oskar/interferometer/oskar_jones_apply_cable_length_errors.h:37-43.
 * The error arrays must match the Jones array's precision and location. */
OSKB_API void oskar_jones_apply_cable_length_errors(oskar_Jones* jones,
        double frequency_hz, const oskar_Mem* errors_x,
        const oskar_Mem* errors_y, int* status);
/* oskar/interferometer/oskar_jones_apply_station_gains.h:32-36. The gains
 * must match the Jones array's type and location. */
OSKB_API void oskar_jones_apply_station_gains(oskar_Jones* jones,
        oskar_Mem* gains, int* status);
/* oskar/telescope/station/oskar_evaluate_element_weights_errors.h:62-66.
 * The gain and phase arrays must have the precision and location of the
 * complex errors array. */
OSKB_API void oskar_evaluate_element_weights_errors(int num_elements,
        const oskar_Mem* gain, const oskar_Mem* gain_error,
        const oskar_Mem* phase, const oskar_Mem* phase_error,
        unsigned int random_seed, int time_index, int station_id,
        oskar_Mem* errors, int* status);
/* oskar/mem/oskar_mem_multiply.h:63 */
OSKB_API void oskar_mem_multiply(oskar_Mem* out, const oskar_Mem* in1,
        const oskar_Mem* in2, size_t offset_out, size_t offset_in1,
        size_t offset_in2, size_t num_elements, int* status);
/* oskar/interferometer/oskar_evaluate_jones_K.h:49 */
OSKB_API void oskar_evaluate_jones_K(oskar_Jones* K, int num_sources,
        const oskar_Mem* l, const oskar_Mem* m, const oskar_Mem* n,
        const oskar_Mem* u, const oskar_Mem* v, const oskar_Mem* w,
        double frequency_hz, const oskar_Mem* source_filter,
        double source_filter_min, double source_filter_max,
        int ignore_w_components, int* status);
/* oskar/math/oskar_dftw.h:92-111 */
OSKB_API void oskar_dftw(int normalise, int num_in, double wavenumber,
        const oskar_Mem* weights_in, const oskar_Mem* x_in,
        const oskar_Mem* y_in, const oskar_Mem* z_in, int offset_coord_out,
        int num_out, const oskar_Mem* x_out, const oskar_Mem* y_out,
        const oskar_Mem* z_out, const oskar_Mem* data_idx,
        const oskar_Mem* data, int eval_x, int eval_y, int offset_out,
        oskar_Mem* output, int* status);
/* oskar/convert/oskar_convert_ecef_to_station_uvw.h:67 */
OSKB_API void oskar_convert_ecef_to_station_uvw(int num_stations,
        const oskar_Mem* x, const oskar_Mem* y, const oskar_Mem* z,
        double ra0_rad, double dec0_rad, double gast,
        int ignore_w_components, int offset_out, oskar_Mem* u, oskar_Mem* v,
        oskar_Mem* w, int* status);

/* oskar/convert/oskar_convert_station_uvw_to_baseline_uvw.h:39-49 */
OSKB_API void oskar_convert_station_uvw_to_baseline_uvw(
        int use_casa_phase_convention, int num_stations, int offset_in,
        const oskar_Mem* u, const oskar_Mem* v, const oskar_Mem* w,
        int offset_out, oskar_Mem* uu, oskar_Mem* vv, oskar_Mem* ww,
        int* status);
/* oskar/convert/oskar_convert_lon_lat_to_relative_directions.h:154-157 */
OSKB_API void oskar_convert_lon_lat_to_relative_directions(int num_points,
        const oskar_Mem* lon_rad, const oskar_Mem* lat_rad, double lon0_rad,
        double lat0_rad, oskar_Mem* l, oskar_Mem* m, oskar_Mem* n,
        int* status);
/* oskar/convert/oskar_convert_apparent_ra_dec_to_enu_directions.h:41-45 */
OSKB_API void oskar_convert_apparent_ra_dec_to_enu_directions(int num_points,
        const oskar_Mem* ra_rad, const oskar_Mem* dec_rad, double lst_rad,
        double latitude_rad, int offset_out, oskar_Mem* x, oskar_Mem* y,
        oskar_Mem* z, int* status);

#ifdef __cplusplus
}
#endif

#endif /* OSKAR_B200_API_H_ */

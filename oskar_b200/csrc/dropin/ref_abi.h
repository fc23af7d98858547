// The part of the reference library's interface that the drop-in
// oskar_interferometer_run_block reads: enumerator values, prototypes of
// exported accessor functions (resolved at run time from the liboskar the
// drop-in is loaded next to), and the two private structures that have no
// accessors for what run_block needs (the simulator object with its
// per-device data, and the sky model's data table).
//
// Everything here restates the reference's own declarations, because the
// drop-in must bind to them exactly: values, names, argument lists and field
// order are the reference's; the file and line each one follows is given.
#pragma once

#include <stddef.h>

extern "C" {

// ---- opaque reference types -------------------------------------------
typedef struct oskar_Mem oskar_Mem;
typedef struct oskar_Sky oskar_Sky;
typedef struct oskar_Telescope oskar_Telescope;
typedef struct oskar_Station oskar_Station;
typedef struct oskar_VisBlock oskar_VisBlock;
typedef struct oskar_Mutex oskar_Mutex;
typedef struct oskar_Log oskar_Log;
typedef struct oskar_Gains oskar_Gains;
typedef struct oskar_Harp oskar_Harp;
typedef struct oskar_Interferometer oskar_Interferometer;

// ---- enumerators -------------------------------------------------------
// oskar/oskar_global.h:23-55 (status codes used here)
enum {
    REF_ERR_INVALID_ARGUMENT = -3,
    REF_ERR_FUNCTION_NOT_AVAILABLE = -4,
    REF_ERR_MEMORY_ALLOC_FAILURE = -6,
    REF_ERR_MEMORY_COPY_FAILURE = -7,
    REF_ERR_MEMORY_NOT_ALLOCATED = -8,
    REF_ERR_TYPE_MISMATCH = -9,
    REF_ERR_BAD_DATA_TYPE = -13,
    REF_ERR_BAD_LOCATION = -14,
    REF_ERR_CUDA_NOT_AVAILABLE = -16,
    REF_ERR_KERNEL_LAUNCH_FAILURE = -18,
    REF_ERR_SETTINGS_TELESCOPE = -23
};
// oskar/oskar_global.h:79-83
enum { REF_METRES = 0, REF_WAVELENGTHS = 1 };
// oskar/oskar_global.h:88-96
enum { REF_COORDS_RADEC = 2, REF_COORDS_AZEL = 4 };
// oskar/mem/oskar_mem.h:36-42 and the type flags of oskar/oskar_global.h
enum { REF_CPU = 0, REF_GPU = 1 };
enum {
    REF_SINGLE = 0x04, REF_DOUBLE = 0x08, REF_COMPLEX = 0x20,
    REF_MATRIX = 0x40
};
// oskar/telescope/station/oskar_station.h:25-31
enum {
    REF_STATION_TYPE_AA = 0, REF_STATION_TYPE_ISOTROPIC = 1,
    REF_STATION_TYPE_GAUSSIAN_BEAM = 2, REF_STATION_TYPE_VLA_PBCOR = 3
};
// oskar/sky/oskar_sky_enum.h:9-50 (column types used here)
enum {
    REF_SKY_RA_RAD = 1, REF_SKY_DEC_RAD = 2, REF_SKY_I_JY = 3,
    REF_SKY_Q_JY = 4, REF_SKY_U_JY = 5, REF_SKY_V_JY = 6,
    REF_SKY_REF_HZ = 7, REF_SKY_SPEC_IDX = 8, REF_SKY_RM_RAD = 9,
    REF_SKY_LIN_SI = 13, REF_SKY_POLA_RAD = 14, REF_SKY_POLF = 15,
    REF_SKY_REF_WAVE_M = 16, REF_SKY_SPEC_CURV = 17,
    REF_SKY_LINE_WIDTH_HZ = 18, REF_SKY_INC_HZ = 19,
    REF_SKY_NUM_FIXED_COLUMN_TYPES = 20,
    REF_SKY_SCRATCH_EXT_A = 0x100, REF_SKY_SCRATCH_EXT_B = 0x101,
    REF_SKY_SCRATCH_EXT_C = 0x102, REF_SKY_SCRATCH_L = 0x103,
    REF_SKY_SCRATCH_M = 0x104, REF_SKY_SCRATCH_N = 0x105
};
// oskar/sky/oskar_sky_enum.h:55-73
enum {
    REF_SKY_PRECISION = 0, REF_SKY_MEM_LOCATION = 1, REF_SKY_CAPACITY = 2,
    REF_SKY_NUM_SOURCES = 3, REF_SKY_NUM_COLUMNS = 4,
    REF_SKY_USE_EXTENDED = 5, REF_SKY_NUM_ATTRIBUTES_INT = 6
};
enum {
    REF_SKY_REF_RA_RAD = 0, REF_SKY_REF_DEC_RAD = 1,
    REF_SKY_NUM_ATTRIBUTES_DOUBLE = 2
};
// oskar/telescope/oskar_telescope.h:25-29
enum { REF_POL_MODE_FULL = 0, REF_POL_MODE_SCALAR = 1 };

// ---- private structures ------------------------------------------------
// oskar/interferometer/private_interferometer.h:22-46 (struct DeviceData)
struct RefDeviceData
{
    oskar_VisBlock* vis_block_cpu[2];
    int previous_chunk_index;
    oskar_VisBlock* vis_block;
    oskar_Mem *lmn[3], *uvw[3];
    oskar_Sky* chunk;
    oskar_Sky* chunk_clip;
    oskar_Telescope* tel;
    void *J, *R, *E, *K;                 // oskar_Jones*
    oskar_Mem* gains;
    void* station_work;                  // oskar_StationWork*
    void *tmr_compute, *tmr_copy, *tmr_clip, *tmr_correlate, *tmr_join,
            *tmr_E, *tmr_K;               // oskar_Timer*
};

// oskar/interferometer/private_interferometer.h:50-86
// (struct oskar_Interferometer)
struct RefInterferometer
{
    int prec, num_devices, num_gpus_avail, dev_loc, num_gpus, *gpu_ids;
    int num_channels, num_time_steps;
    int max_sources_per_chunk, max_times_per_block, max_channels_per_block;
    int apply_horizon_clip, force_polarised_ms, zero_failed_gaussians;
    int coords_only, ignore_w_components;
    int casa_phase_convention;
    double freq_start_hz, freq_inc_hz, time_start_mjd_utc, time_inc_sec;
    double source_min_jy, source_max_jy;
    double ms_dish_diameter;
    char correlation_type, *vis_name, *ms_name, *settings_path;
    int init_sky, work_unit_index;
    oskar_Mutex* mutex;
    void* barrier;                       // oskar_Barrier*
    oskar_Log* log;
    int num_sources_total, num_sky_chunks;
    oskar_Sky** sky_chunks;
    oskar_Telescope* tel;
    void* header;                        // oskar_VisHeader*
    void* ms;                            // oskar_MeasurementSet*
    void* vis;                           // oskar_Binary*
    oskar_Mem* temp;
    void *tmr_sim, *tmr_write;           // oskar_Timer*
    RefDeviceData* d;
};

// oskar/sky/private_sky.h:18-33 (struct oskar_Sky)
struct RefSky
{
    double attr_double[REF_SKY_NUM_ATTRIBUTES_DOUBLE];
    int attr_int[REF_SKY_NUM_ATTRIBUTES_INT];
    oskar_Mem* table;                    // [num_columns][capacity]
    oskar_Mem* num_valid_columns;        // [capacity][20] int
    oskar_Mem** columns;
    int* column_type;
    int* column_attr;
};

// ---- exported functions --------------------------------------------------
// oskar/utility/oskar_thread.h
void oskar_mutex_lock(oskar_Mutex* mutex);
void oskar_mutex_unlock(oskar_Mutex* mutex);
// oskar/log/oskar_log.h
void oskar_log_error(oskar_Log* log, const char* format, ...);
// oskar/mem/oskar_mem_accessors.h
void* oskar_mem_void(oskar_Mem* mem);
const void* oskar_mem_void_const(const oskar_Mem* mem);
int oskar_mem_type(const oskar_Mem* mem);
int oskar_mem_location(const oskar_Mem* mem);
size_t oskar_mem_length(const oskar_Mem* mem);
// oskar/convert/oskar_convert_mjd_to_gast_fast.h
double oskar_convert_mjd_to_gast_fast(double mjd);
// oskar/interferometer/oskar_interferometer_accessors.h
int oskar_interferometer_num_devices(const oskar_Interferometer* h);
int oskar_interferometer_num_gpus(const oskar_Interferometer* h);
int oskar_interferometer_coords_only(const oskar_Interferometer* h);
int oskar_interferometer_casa_phase_convention(
        const oskar_Interferometer* h);
oskar_Log* oskar_interferometer_log(oskar_Interferometer* h);
// oskar/vis/oskar_vis_block_accessors.h, oskar_vis_block_resize.h
oskar_Mem* oskar_vis_block_cross_correlations(oskar_VisBlock* vis);
oskar_Mem* oskar_vis_block_auto_correlations(oskar_VisBlock* vis);
int oskar_vis_block_has_cross_correlations(const oskar_VisBlock* vis);
int oskar_vis_block_has_auto_correlations(const oskar_VisBlock* vis);
int oskar_vis_block_num_stations(const oskar_VisBlock* vis);
void oskar_vis_block_resize(oskar_VisBlock* vis, int num_times,
        int num_channels, int num_stations, int* status);
void oskar_vis_block_set_start_time_index(oskar_VisBlock* vis,
        int global_index);
void oskar_vis_block_set_start_channel_index(oskar_VisBlock* vis,
        int global_index);
// oskar/sky/oskar_sky_accessors.h
int oskar_sky_int(const oskar_Sky* sky, int attribute);
double oskar_sky_double(const oskar_Sky* sky, int attribute);
int oskar_sky_first_column(const oskar_Sky* sky, int column_type);
// oskar/telescope/oskar_telescope_accessors.h
int oskar_telescope_num_stations(const oskar_Telescope* model);
int oskar_telescope_num_station_models(const oskar_Telescope* model);
int oskar_telescope_pol_mode(const oskar_Telescope* model);
int oskar_telescope_phase_centre_coord_type(const oskar_Telescope* model);
double oskar_telescope_phase_centre_longitude_rad(
        const oskar_Telescope* model);
double oskar_telescope_phase_centre_latitude_rad(
        const oskar_Telescope* model);
double oskar_telescope_lon_rad(const oskar_Telescope* model);
double oskar_telescope_lat_rad(const oskar_Telescope* model);
double oskar_telescope_channel_bandwidth_hz(const oskar_Telescope* model);
double oskar_telescope_time_average_sec(const oskar_Telescope* model);
double oskar_telescope_uv_filter_min(const oskar_Telescope* model);
double oskar_telescope_uv_filter_max(const oskar_Telescope* model);
int oskar_telescope_uv_filter_units(const oskar_Telescope* model);
int oskar_telescope_allow_station_beam_duplication(
        const oskar_Telescope* model);
char oskar_telescope_ionosphere_screen_type(const oskar_Telescope* model);
const oskar_Mem* oskar_telescope_station_type_map_const(
        const oskar_Telescope* model);
const oskar_Mem* oskar_telescope_station_true_offset_ecef_metres_const(
        const oskar_Telescope* model, int dim);
const oskar_Mem* oskar_telescope_station_true_enu_metres_const(
        const oskar_Telescope* model, int dim);
const oskar_Mem* oskar_telescope_station_cable_length_error_const(
        const oskar_Telescope* model, int feed);
const oskar_Station* oskar_telescope_station_const(
        const oskar_Telescope* model, int i);
oskar_Gains* oskar_telescope_gains(oskar_Telescope* model);
oskar_Harp* oskar_telescope_harp_data(oskar_Telescope* model,
        double freq_hz);
// oskar/gains/oskar_gains.h
int oskar_gains_defined(const oskar_Gains* h);
typedef struct oskar_Element oskar_Element;
// oskar/telescope/station/oskar_station_accessors.h
int oskar_station_num_elements(const oskar_Station* model);
int oskar_station_num_element_types(const oskar_Station* model);
int oskar_station_normalise_array_pattern(const oskar_Station* model);
int oskar_station_normalise_element_pattern(const oskar_Station* model);
int oskar_station_enable_array_pattern(const oskar_Station* model);
int oskar_station_common_element_orientation(const oskar_Station* model);
int oskar_station_common_pol_beams(const oskar_Station* model);
int oskar_station_apply_element_errors(const oskar_Station* model);
int oskar_station_apply_element_weight(const oskar_Station* model);
int oskar_station_swap_xy(const oskar_Station* model);
int oskar_station_array_is_3d(const oskar_Station* model);
int oskar_station_has_child(const oskar_Station* model);
double oskar_station_element_euler_index_rad(const oskar_Station* model,
        int feed, int dim, int index);
const oskar_Mem* oskar_station_element_true_enu_metres_const(
        const oskar_Station* model, int feed, int dim);
const oskar_Mem* oskar_station_element_measured_enu_metres_const(
        const oskar_Station* model, int feed, int dim);
const oskar_Mem* oskar_station_element_cable_length_error_metres_const(
        const oskar_Station* model, int feed);
const int* oskar_station_element_types_cpu_const(const oskar_Station* model);
const oskar_Element* oskar_station_element_const(const oskar_Station* model,
        int element_type_index);
const oskar_Gains* oskar_station_gains_const(const oskar_Station* model);
const oskar_Harp* oskar_station_harp_data_const(const oskar_Station* model,
        double freq_hz);
void oskar_station_beam_horizon_direction(const oskar_Station* station,
        const double gast_rad, double* x, double* y, double* z, int* status);
// oskar/telescope/station/element/oskar_element_accessors.h
int oskar_element_num_freq(const oskar_Element* data);
int oskar_element_is_isotropic(const oskar_Element* data);
int oskar_element_taper_type(const oskar_Element* data);
double oskar_element_cosine_power(const oskar_Element* data);
double oskar_element_gaussian_fwhm_rad(const oskar_Element* data);
double oskar_element_dipole_length(const oskar_Element* data);
int oskar_element_dipole_length_units(const oskar_Element* data);
// oskar/telescope/station/oskar_station_accessors.h
int oskar_station_type(const oskar_Station* model);
int oskar_station_normalise_final_beam(const oskar_Station* model);
double oskar_station_lon_rad(const oskar_Station* model);
double oskar_station_lat_rad(const oskar_Station* model);
double oskar_station_beam_lon_rad(const oskar_Station* model);
double oskar_station_beam_lat_rad(const oskar_Station* model);
int oskar_station_beam_coord_type(const oskar_Station* model);

}  // extern "C"

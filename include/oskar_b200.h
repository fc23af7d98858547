/*
 * oskar_b200 -- B200 (sm_100a) kernels for OSKAR's interferometer visibility
 * hot path: station-beam DFT, Jones K and join, cross-/auto-correlation.
 *
 * This is the C ABI of liboskar_b200.so. Every entry point takes plain
 * pointers, sizes and a CUDA stream (passed as void*, 0 = legacy default
 * stream). Unless stated otherwise all array pointers are DEVICE pointers.
 *
 * Conventions (the same as the reference's kernel launchers):
 *  - a complex value is two reals {re, im}; a 2x2 complex matrix is eight
 *    reals {a, b, c, d} = {xx, xy, yx, yy}
 *    (oskar/utility/oskar_vector_types.h:85-98);
 *  - Jones arrays are [station][source], source fastest
 *    (oskar/interferometer/private_jones.h:34-41);
 *  - visibility index of the baseline between stations q < p is
 *    q*(N-1) - (q-1)*q/2 + p - q - 1, plus offset_out
 *    (oskar/correlate/define_correlate_utils.h:42);
 *  - correlation outputs are ACCUMULATED (+=) into vis, as in the reference;
 *  - every function returns 0 on success or a negative OSKAR error code
 *    (oskar/oskar_global.h:20-55); nothing is launched after an error.
 *
 * Each function names the reference interface it replaces.
 */
#ifndef OSKAR_B200_H_
#define OSKAR_B200_H_

#include <stddef.h>

#if defined(__GNUC__)
#define OSKB_API __attribute__((visibility("default")))
#else
#define OSKB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes shared with the reference (oskar/oskar_global.h:20-55). */
#define OSKB_ERR_INVALID_ARGUMENT      (-3)
#define OSKB_ERR_OUT_OF_RANGE          (-5)
#define OSKB_ERR_MEMORY_ALLOC_FAILURE  (-6)
#define OSKB_ERR_MEMORY_COPY_FAILURE   (-7)
#define OSKB_ERR_TYPE_MISMATCH         (-9)
#define OSKB_ERR_LOCATION_MISMATCH     (-10)
#define OSKB_ERR_DIMENSION_MISMATCH    (-11)
#define OSKB_ERR_BAD_DATA_TYPE         (-13)
#define OSKB_ERR_CUDA_NOT_AVAILABLE    (-16)
#define OSKB_ERR_KERNEL_LAUNCH_FAILURE (-18)

/* Library version string and the CUDA error text of the last failure. */
OSKB_API const char* oskb_version(void);
OSKB_API const char* oskb_last_error(void);

/* Per-call temporaries (partial sums of source slices and the like) come
 * from a library-owned stream-ordered pool that keeps up to 4 GiB cached
 * across host synchronisations; this returns the cached blocks to the
 * driver. No OSKAR counterpart. */
OSKB_API int oskb_scratch_release(void);

/* ------------------------------------------------------------------------
 * Cross-correlation, direct kernel (all source types and smearing modes).
 * ------------------------------------------------------------------------
 * V[bl] += sum_s smear(s, bl) * J_p(s) B(s) J_q(s)^H, with the brightness
 * matrix B built from Stokes I, Q, U, V. Bandwidth smearing is on when
 * frac_bandwidth != 0, time-average smearing when time_int_sec != 0.
 * gaussian != 0 selects Gaussian sources (a, b, c used); else a, b, c may be
 * NULL.
 * Replaces oskar_cross_correlate_{point,gaussian}_cuda_{f,d}
 * (oskar/correlate/oskar_cross_correlate_cuda.h:60-71, 113-124, 172-184,
 * 232-244). The FP64 form matches the reference CPU FP64 path to 1e-12
 * relative; the FP32 form accumulates per source chunk with compensated
 * cross-chunk sums. */
OSKB_API int oskb_cross_correlate_d(int use_casa_phase_convention, int gaussian,
        int num_sources, int num_stations, int offset_out,
        const double* jones, const double* I, const double* Q,
        const double* U, const double* V, const double* l, const double* m,
        const double* n, const double* a, const double* b, const double* c,
        const double* station_u, const double* station_v,
        const double* station_w, const double* station_x,
        const double* station_y, double uv_min_lambda, double uv_max_lambda,
        double inv_wavelength, double frac_bandwidth, double time_int_sec,
        double gha0_rad, double dec0_rad, double* vis, void* stream);
OSKB_API int oskb_cross_correlate_f(int use_casa_phase_convention, int gaussian,
        int num_sources, int num_stations, int offset_out,
        const float* jones, const float* I, const float* Q,
        const float* U, const float* V, const float* l, const float* m,
        const float* n, const float* a, const float* b, const float* c,
        const float* station_u, const float* station_v,
        const float* station_w, const float* station_x,
        const float* station_y, float uv_min_lambda, float uv_max_lambda,
        float inv_wavelength, float frac_bandwidth, float time_int_sec,
        float gha0_rad, float dec0_rad, float* vis, void* stream);

/* Scalar (Stokes-I only) polarisation mode: V += sum smear * I J_p conj(J_q).
 * jones is complex [station][source]. Replaces
 * oskar_cross_correlate_scalar_{point,gaussian}_cuda_{f,d}
 * (oskar/correlate/oskar_cross_correlate_scalar_cuda.h:56, 103, 156, 211). */
OSKB_API int oskb_cross_correlate_scalar_d(int use_casa_phase_convention,
        int gaussian, int num_sources, int num_stations, int offset_out,
        const double* jones, const double* I, const double* l,
        const double* m, const double* n, const double* a, const double* b,
        const double* c, const double* station_u, const double* station_v,
        const double* station_w, const double* station_x,
        const double* station_y, double uv_min_lambda, double uv_max_lambda,
        double inv_wavelength, double frac_bandwidth, double time_int_sec,
        double gha0_rad, double dec0_rad, double* vis, void* stream);
OSKB_API int oskb_cross_correlate_scalar_f(int use_casa_phase_convention,
        int gaussian, int num_sources, int num_stations, int offset_out,
        const float* jones, const float* I, const float* l,
        const float* m, const float* n, const float* a, const float* b,
        const float* c, const float* station_u, const float* station_v,
        const float* station_w, const float* station_x,
        const float* station_y, float uv_min_lambda, float uv_max_lambda,
        float inv_wavelength, float frac_bandwidth, float time_int_sec,
        float gha0_rad, float dec0_rad, float* vis, void* stream);

/* Auto-correlation: vis[s + offset_out] += sum_src J B J^H (matrix) or
 * sum |J|^2 I (scalar, real part only). Replaces the kernels behind
 * oskar_auto_correlate (oskar/correlate/oskar_auto_correlate.h:37;
 * oskar/correlate/define_auto_correlate.h:8-82). */
OSKB_API int oskb_auto_correlate_d(int matrix, int num_sources, int num_stations,
        int offset_out, const double* jones, const double* I,
        const double* Q, const double* U, const double* V, double* vis,
        void* stream);
OSKB_API int oskb_auto_correlate_f(int matrix, int num_sources, int num_stations,
        int offset_out, const float* jones, const float* I,
        const float* Q, const float* U, const float* V, float* vis,
        void* stream);

/* ------------------------------------------------------------------------
 * Jones K and join.
 * ------------------------------------------------------------------------
 * K[station][source] = exp(i wavenumber (u l + v m + w (n - 1))), zero for
 * sources whose filter value lies outside (filter_min, filter_max].
 * Replaces the kernels behind oskar_evaluate_jones_K
 * (oskar/interferometer/oskar_evaluate_jones_K.h:49;
 *  oskar/interferometer/define_evaluate_jones_K.h:22-70). */
OSKB_API int oskb_evaluate_jones_K_d(int num_sources, const double* l,
        const double* m, const double* n, int num_stations, const double* u,
        const double* v, const double* w, double wavenumber,
        const double* source_filter, double filter_min, double filter_max,
        int ignore_w_components, double* jones, void* stream);
OSKB_API int oskb_evaluate_jones_K_f(int num_sources, const float* l,
        const float* m, const float* n, int num_stations, const float* u,
        const float* v, const float* w, float wavenumber,
        const float* source_filter, float filter_min, float filter_max,
        int ignore_w_components, float* jones, void* stream);

/* Element-wise products c[i+off_c] = a[i+off_a] * b[i+off_b] behind
 * oskar_jones_join / oskar_mem_multiply
 * (oskar/interferometer/oskar_jones_join.h:69; oskar/mem/oskar_mem_multiply.h:63;
 *  kernels oskar/mem/define_mem_multiply.h:3-89). kind selects the operand
 * shapes: OSKB_MUL_RR_R (real*real), OSKB_MUL_CC_C (complex*complex),
 * OSKB_MUL_CC_M (complex*complex -> diagonal matrix), OSKB_MUL_CM_M
 * (complex*matrix), OSKB_MUL_MC_M (matrix*complex), OSKB_MUL_MM_M
 * (matrix*matrix). c may alias a or b exactly. */
#define OSKB_MUL_RR_R 0
#define OSKB_MUL_CC_C 1
#define OSKB_MUL_CC_M 2
#define OSKB_MUL_CM_M 3
#define OSKB_MUL_MC_M 4
#define OSKB_MUL_MM_M 5
OSKB_API int oskb_mem_multiply_d(int kind, size_t off_a, size_t off_b, size_t off_c,
        size_t n, const double* a, const double* b, double* c, void* stream);
OSKB_API int oskb_mem_multiply_f(int kind, size_t off_a, size_t off_b, size_t off_c,
        size_t n, const float* a, const float* b, float* c, void* stream);

/* ------------------------------------------------------------------------
 * Station beam: weighted DFT and beamforming weights.
 * ------------------------------------------------------------------------
 * output[d + offset_out] = norm_factor * sum_e w_e
 *     * exp(i wavenumber (x_e X_d + y_e Y_d [+ z_e Z_d])) * data[idx_e][d]
 * with (X, Y, Z) = (x_out, y_out, z_out)[d + offset_coord_out]; 3-D when
 * both z_in and z_out are non-NULL; idx_e = data_idx[e] or e if data_idx is
 * NULL. matrix = 0: data complex [n_idx][num_out], output complex;
 * matrix = 1: data [n_idx][num_out][2x2], output 2x2, the xx/xy pair written
 * if eval_x and the yx/yy pair if eval_y.
 * Replaces the kernels behind oskar_dftw (oskar/math/oskar_dftw.h:92-111;
 * oskar/math/define_dftw_c2c.h:24-77, define_dftw_m2m.h:24-107). */
OSKB_API int oskb_dftw_d(int matrix, int num_in, double wavenumber,
        const double* weights_in, const double* x_in, const double* y_in,
        const double* z_in, int offset_coord_out, int num_out,
        const double* x_out, const double* y_out, const double* z_out,
        const int* data_idx, const double* data, int eval_x, int eval_y,
        int offset_out, double* output, double norm_factor, void* stream);
OSKB_API int oskb_dftw_f(int matrix, int num_in, float wavenumber,
        const float* weights_in, const float* x_in, const float* y_in,
        const float* z_in, int offset_coord_out, int num_out,
        const float* x_out, const float* y_out, const float* z_out,
        const int* data_idx, const float* data, int eval_x, int eval_y,
        int offset_out, float* output, float norm_factor, void* stream);

/* out[2 i], out[2 i + 1] = cos, sin of (pi / 64) steps[i]: a phase given
 * in steps of 2 pi / 128, by the table-driven method the FP64 element loops
 * of the weighted DFT and the station beam use (128-entry table, Taylor
 * series of the remainder; sincospi(steps / 64) where the table does not
 * reach, beyond |steps| = 2^32). Device arrays. No OSKAR counterpart:
 * exposed so the method can be checked against exact values. */
OSKB_API int oskb_phase_factors_d(int n, const double* steps, double* out,
        void* stream);

/* Beamforming weights w_e = exp(-i wavenumber (x x1 + y y1 + z z1 + cable_e)),
 * z and cable_length_error may be NULL (zero).
 * Replaces the kernel behind oskar_evaluate_element_weights_dft
 * (oskar/telescope/station/oskar_evaluate_element_weights_dft.h:66;
 *  define_evaluate_element_weights_dft.h:3-16). */
OSKB_API int oskb_evaluate_element_weights_dft_d(int num_elements, const double* x,
        const double* y, const double* z, const double* cable_length_error,
        double wavenumber, double x1, double y1, double z1, double* weights,
        void* stream);
OSKB_API int oskb_evaluate_element_weights_dft_f(int num_elements, const float* x,
        const float* y, const float* z, const float* cable_length_error,
        float wavenumber, float x1, float y1, float z1, float* weights,
        void* stream);

/* Station ECEF offsets to (u, v, w) metres at hour angle ha0 = gast - ra0.
 * Replaces the kernel behind oskar_convert_ecef_to_station_uvw
 * (oskar/convert/oskar_convert_ecef_to_station_uvw.h:67;
 *  define_convert_ecef_to_station_uvw.h:3-29). */
OSKB_API int oskb_convert_ecef_to_station_uvw_d(int num_stations, const double* x,
        const double* y, const double* z, double ra0_rad, double dec0_rad,
        double gast, int ignore_w_components, int offset_out, double* u,
        double* v, double* w, void* stream);

/* Aperture-array station beam (Jones E) of num_stations stations in one
 * launch: dipole element pattern (optionally normalised at the pole), array
 * factor with weights from the measured element positions (true positions
 * where meas_* is NULL) and cable-length errors (NULL: none), optional 1/N
 * array normalisation, horizon blanking, and optional division by the beam
 * amplitude in the normalisation direction. Replaces the chain of
 * oskar_station_beam (oskar/telescope/station/src/oskar_station_beam.c:
 * 84-182) and oskar_evaluate_station_beam_aperture_array
 * (oskar_evaluate_station_beam_aperture_array.c:150-240) for stations with
 * one dipole element type, common orientation, no child stations.
 *   el_*, meas_*, cable_length_error: [station][element] metres (ENU);
 *   orientation_{x,y}_rad: [station] element Euler angles (the reference's
 *     oskar_station_element_euler_index_rad(s, 0|1, 0, 0));
 *   beam_enu, norm_enu: [station][3] ENU direction cosines (double);
 *   x, y, z: ENU direction cosines, [station][num_directions] when
 *     directions_per_station, else [num_directions] shared;
 *   beam: [station][num_directions] complex 2x2 (the Jones E layout).
 * All pointers are device memory. */
OSKB_API int oskb_station_beam_aa_d(int num_stations, int num_elements,
        const double* el_x, const double* el_y, const double* el_z,
        const double* meas_x, const double* meas_y, const double* meas_z,
        const double* cable_length_error, const double* orientation_x_rad,
        const double* orientation_y_rad, double dipole_length_m,
        int normalise_element, int normalise_array, int normalise_final,
        int swap_xy, int is_3d, double frequency_hz, const double* beam_enu,
        const double* norm_enu, int num_directions, const double* x,
        const double* y, const double* z, int directions_per_station,
        double* beam, void* stream);
OSKB_API int oskb_station_beam_aa_f(int num_stations, int num_elements,
        const float* el_x, const float* el_y, const float* el_z,
        const float* meas_x, const float* meas_y, const float* meas_z,
        const float* cable_length_error, const double* orientation_x_rad,
        const double* orientation_y_rad, double dipole_length_m,
        int normalise_element, int normalise_array, int normalise_final,
        int swap_xy, int is_3d, double frequency_hz, const double* beam_enu,
        const double* norm_enu, int num_directions, const float* x,
        const float* y, const float* z, int directions_per_station,
        float* beam, void* stream);

/* oskb_station_beam_aa with one complex factor per element multiplying the
 * element's DFT weight: element_weight_factors [station][element] complex
 * (NULL: none), e.g. the product of time-variable element errors and
 * apodisation from oskb_station_element_weight_factors, as
 * oskar_station_evaluate_element_weights
 * (oskar/telescope/station/src/oskar_station_evaluate_element_weights.c:
 * 33-64) applies them to the weights; the normalisation direction uses the
 * same weights. */
OSKB_API int oskb_station_beam_aa_weighted_d(int num_stations,
        int num_elements, const double* el_x, const double* el_y,
        const double* el_z, const double* meas_x, const double* meas_y,
        const double* meas_z, const double* cable_length_error,
        const double* element_weight_factors,
        const double* orientation_x_rad, const double* orientation_y_rad,
        double dipole_length_m, int normalise_element, int normalise_array,
        int normalise_final, int swap_xy, int is_3d, double frequency_hz,
        const double* beam_enu, const double* norm_enu, int num_directions,
        const double* x, const double* y, const double* z,
        int directions_per_station, double* beam, void* stream);
OSKB_API int oskb_station_beam_aa_weighted_f(int num_stations,
        int num_elements, const float* el_x, const float* el_y,
        const float* el_z, const float* meas_x, const float* meas_y,
        const float* meas_z, const float* cable_length_error,
        const float* element_weight_factors,
        const double* orientation_x_rad, const double* orientation_y_rad,
        double dipole_length_m, int normalise_element, int normalise_array,
        int normalise_final, int swap_xy, int is_3d, double frequency_hz,
        const double* beam_enu, const double* norm_enu, int num_directions,
        const float* x, const float* y, const float* z,
        int directions_per_station, float* beam, void* stream);

#define OSKB_ELEMENT_DIPOLE    0
#define OSKB_ELEMENT_ISOTROPIC 1
#define OSKB_TAPER_NONE        0
#define OSKB_TAPER_COSINE      1
#define OSKB_TAPER_GAUSSIAN    2

/* oskb_station_beam_aa_weighted for stations with up to 4 element types
 * (oskar_evaluate_station_beam_aperture_array.c:158-202 and its oskar_dftw
 * with data index = element type): element e has type
 * element_type[station][e] (device; NULL: all type 0); type t is a dipole
 * of length dipole_length_m[t] (host array of num_element_types) with
 * Euler angles orientation_{x,y}_rad[station][t] (device) and its own pole
 * normalisation; beam = sum over types of the type's pattern times the
 * array factor of its elements. Host arrays per type (each may be NULL):
 * element_kind OSKB_ELEMENT_DIPOLE or OSKB_ELEMENT_ISOTROPIC (the identity
 * pattern); taper_kind OSKB_TAPER_NONE, OSKB_TAPER_COSINE (cos(theta) to the
 * power taper_param) or OSKB_TAPER_GAUSSIAN (FWHM taper_param radians in
 * theta), applied after the pole normalisation (oskar_element_evaluate.c:
 * 82-87, 159-174). A station whose elements differ in
 * orientation (the reference's per-element branch, :180-202) maps onto
 * this when its distinct (element model, orientation) pairs number at most
 * four: one type per pair. An element whose type is outside
 * [0, num_element_types) adds nothing (the reference stops with
 * OSKAR_ERR_OUT_OF_RANGE). num_element_types > 4: OSKB_ERR_OUT_OF_RANGE. */
OSKB_API int oskb_station_beam_aa_types_d(int num_stations, int num_elements,
        const double* el_x, const double* el_y, const double* el_z,
        const double* meas_x, const double* meas_y, const double* meas_z,
        const double* cable_length_error,
        const double* element_weight_factors, int num_element_types,
        const int* element_type, const double* dipole_length_m,
        const int* element_kind, const int* taper_kind,
        const double* taper_param,
        const double* orientation_x_rad, const double* orientation_y_rad,
        int normalise_element, int normalise_array, int normalise_final,
        int swap_xy, int is_3d, double frequency_hz, const double* beam_enu,
        const double* norm_enu, int num_directions, const double* x,
        const double* y, const double* z, int directions_per_station,
        double* beam, void* stream);
OSKB_API int oskb_station_beam_aa_types_f(int num_stations, int num_elements,
        const float* el_x, const float* el_y, const float* el_z,
        const float* meas_x, const float* meas_y, const float* meas_z,
        const float* cable_length_error,
        const float* element_weight_factors, int num_element_types,
        const int* element_type, const double* dipole_length_m,
        const int* element_kind, const int* taper_kind,
        const double* taper_param,
        const double* orientation_x_rad, const double* orientation_y_rad,
        int normalise_element, int normalise_array, int normalise_final,
        int swap_xy, int is_3d, double frequency_hz, const double* beam_enu,
        const double* norm_enu, int num_directions, const float* x,
        const float* y, const float* z, int directions_per_station,
        float* beam, void* stream);

/* oskb_station_beam_aa_types in the scalar (Stokes-I) polarisation mode:
 * each type's pattern is its amplitude sqrt((a^2 + b^2 + c^2 + d^2) / 2)
 * (the reference's scalar dipole response,
 * oskar/telescope/station/element/define_evaluate_dipole_pattern.h:51-75;
 * 1 for isotropic elements), the beam is complex [station][direction] and
 * the final normalisation divides by its magnitude in the normalisation
 * direction (oskar/mem/define_mem_normalise.h:13-29). */
OSKB_API int oskb_station_beam_aa_scalar_d(int num_stations, int num_elements,
        const double* el_x, const double* el_y, const double* el_z,
        const double* meas_x, const double* meas_y, const double* meas_z,
        const double* cable_length_error,
        const double* element_weight_factors, int num_element_types,
        const int* element_type, const double* dipole_length_m,
        const int* element_kind, const int* taper_kind,
        const double* taper_param,
        const double* orientation_x_rad, const double* orientation_y_rad,
        int normalise_element, int normalise_array, int normalise_final,
        int swap_xy, int is_3d, double frequency_hz, const double* beam_enu,
        const double* norm_enu, int num_directions, const double* x,
        const double* y, const double* z, int directions_per_station,
        double* beam, void* stream);
OSKB_API int oskb_station_beam_aa_scalar_f(int num_stations, int num_elements,
        const float* el_x, const float* el_y, const float* el_z,
        const float* meas_x, const float* meas_y, const float* meas_z,
        const float* cable_length_error,
        const float* element_weight_factors, int num_element_types,
        const int* element_type, const double* dipole_length_m,
        const int* element_kind, const int* taper_kind,
        const double* taper_param,
        const double* orientation_x_rad, const double* orientation_y_rad,
        int normalise_element, int normalise_array, int normalise_final,
        int swap_xy, int is_3d, double frequency_hz, const double* beam_enu,
        const double* norm_enu, int num_directions, const float* x,
        const float* y, const float* z, int directions_per_station,
        float* beam, void* stream);

/* oskb_station_beam_aa_types for stations whose two feeds have element
 * data of their own (the reference's num_feeds = 2 when a station is not
 * common_pol_beams: per-feed positions, cable errors, gains, errors or
 * apodisation; oskar_evaluate_station_beam_aperture_array.c:208-223).
 * el_*, meas_*, cable_length_error: [feed][station][element];
 * element_weight_factors: [feed][station][element] complex (NULL: none);
 * the x feed's array factor forms the (xx, xy) row, the y feed's the
 * (yx, yy) row; the final normalisation uses both. num_feeds = 1 is
 * oskb_station_beam_aa_types. */
OSKB_API int oskb_station_beam_aa_feeds_d(int num_feeds, int num_stations,
        int num_elements, const double* el_x, const double* el_y,
        const double* el_z, const double* meas_x, const double* meas_y,
        const double* meas_z, const double* cable_length_error,
        const double* element_weight_factors, int num_element_types,
        const int* element_type, const double* dipole_length_m,
        const int* element_kind, const int* taper_kind,
        const double* taper_param,
        const double* orientation_x_rad, const double* orientation_y_rad,
        int normalise_element, int normalise_array, int normalise_final,
        int swap_xy, int is_3d, double frequency_hz, const double* beam_enu,
        const double* norm_enu, int num_directions, const double* x,
        const double* y, const double* z, int directions_per_station,
        double* beam, void* stream);
OSKB_API int oskb_station_beam_aa_feeds_f(int num_feeds, int num_stations,
        int num_elements, const float* el_x, const float* el_y,
        const float* el_z, const float* meas_x, const float* meas_y,
        const float* meas_z, const float* cable_length_error,
        const float* element_weight_factors, int num_element_types,
        const int* element_type, const double* dipole_length_m,
        const int* element_kind, const int* taper_kind,
        const double* taper_param,
        const double* orientation_x_rad, const double* orientation_y_rad,
        int normalise_element, int normalise_array, int normalise_final,
        int swap_xy, int is_3d, double frequency_hz, const double* beam_enu,
        const double* norm_enu, int num_directions, const float* x,
        const float* y, const float* z, int directions_per_station,
        float* beam, void* stream);

/* Beam-pattern power terms for one source of brightness (I, Q, U, V):
 * auto power out[i + offset_out] = J B J^H of jones[i + offset_in] (|J|^2
 * for scalar Jones), and cross power out[s + offset_out] =
 * 2 / (N (N - 1)) sum_{p<q} (J_p B) J_q^H over the N stations of
 * jones[station][source] (scalar: J_p conj(J_q)); matrix selects 2x2 Jones.
 * The cross power takes one pass over the stations with running prefix
 * sums, O(N) per source where the reference loops over pairs. Replace the
 * kernels behind oskar_evaluate_auto_power and oskar_evaluate_cross_power
 * (oskar/correlate/oskar_evaluate_{auto,cross}_power.h;
 * define_evaluate_auto_power.h:3-40, define_evaluate_cross_power.h:3-72). */
OSKB_API int oskb_evaluate_auto_power_d(int matrix, int n, int offset_in,
        const double* jones, double src_I, double src_Q, double src_U,
        double src_V, int offset_out, double* out, void* stream);
OSKB_API int oskb_evaluate_auto_power_f(int matrix, int n, int offset_in,
        const float* jones, float src_I, float src_Q, float src_U,
        float src_V, int offset_out, float* out, void* stream);
OSKB_API int oskb_evaluate_cross_power_d(int matrix, int num_sources,
        int num_stations, const double* jones, double src_I, double src_Q,
        double src_U, double src_V, int offset_out, double* out,
        void* stream);
OSKB_API int oskb_evaluate_cross_power_f(int matrix, int num_sources,
        int num_stations, const float* jones, float src_I, float src_Q,
        float src_U, float src_V, int offset_out, float* out, void* stream);

/* Time-variable element gain and phase errors of one station:
 * errors[e] = (gain[e] + gain_error[e] g) exp(i (phase[e] + phase_error[e] h))
 * with (g, h) a standard Gaussian pair per element drawn from Philox4x32-10
 * (key {random_seed, 0xCAFEF00D}, counter {e / 2, time_index, station_id,
 * 0x12345678}) and the Box-Muller transform, as the reference draws them.
 * errors: complex [element]. Replaces oskar_evaluate_element_weights_errors
 * (oskar/telescope/station/oskar_evaluate_element_weights_errors.h;
 * src/oskar_evaluate_element_weights_errors.c:19-110) with the random fill
 * of oskar_mem_random_gaussian (oskar/mem/src/oskar_mem_random_gaussian.c). */
OSKB_API int oskb_evaluate_element_weights_errors_d(int num_elements,
        const double* gain, const double* gain_error, const double* phase,
        const double* phase_error, unsigned int random_seed, int time_index,
        int station_id, double* errors, void* stream);
OSKB_API int oskb_evaluate_element_weights_errors_f(int num_elements,
        const float* gain, const float* gain_error, const float* phase,
        const float* phase_error, unsigned int random_seed, int time_index,
        int station_id, float* errors, void* stream);

/* Element weight factors of num_stations stations in one launch:
 * factors[s][e] = errors (as oskb_evaluate_element_weights_errors, station
 * id first_station_id + s; skipped when gain is NULL) times
 * apodisation[s][e] (complex; skipped when NULL); 1 when both are skipped.
 * gain, gain_error, phase, phase_error: [station][element] when
 * per_station, else [element] shared by every station. No single OSKAR
 * counterpart: the per-station steps of
 * oskar_station_evaluate_element_weights.c:33-64 for all stations. */
OSKB_API int oskb_station_element_weight_factors_d(int num_stations,
        int num_elements, int first_station_id, unsigned int random_seed,
        int time_index, const double* gain, const double* gain_error,
        const double* phase, const double* phase_error, int per_station,
        const double* apodisation, double* factors, void* stream);
OSKB_API int oskb_station_element_weight_factors_f(int num_stations,
        int num_elements, int first_station_id, unsigned int random_seed,
        int time_index, const float* gain, const float* gain_error,
        const float* phase, const float* phase_error, int per_station,
        const float* apodisation, float* factors, void* stream);

/* Two-level (hierarchical) aperture-array station: a station of num_tiles
 * tiles at ENU positions tile_x/y/z [tile] (true positions, metres), tile t
 * a dipole array of layout tile_type[t] (NULL: every tile of layout 0, the
 * reference's identical children); layout i has num_elements dipoles at
 * el_x/y/z [i][element] and orientations orientation_x/y_rad [i]. Beam
 * [direction][2x2] = (1/num_tiles if normalise_station_array) x
 * sum_t w_t exp(i k r_t . d) x tilebeam[type(t)][d], with parent weights
 * w_t = exp(-i k r_t . b) for the pointing b = (beam_x, beam_y, beam_z)
 * (host, ENU), and each tile beam the fused single-level beam
 * (oskb_station_beam_aa: dipole pattern, tile array factor pointed at b,
 * normalise_element / normalise_tile_array, blanked below the horizon).
 * The two-level case of the reference's recursion
 * (oskar_evaluate_station_beam_aperture_array.c:242-287, child beams as the
 * parent's weighted-DFT data, oskar_dftw with element weights from
 * oskar_station_evaluate_element_weights.c:15-66); the normalisation to
 * the beam direction (oskar_station_beam.c:108-135) is the caller's, as in
 * the reference. workspace: device, at least
 * oskb_station_beam_two_level_workspace_bytes(sizeof(T), num_tile_types,
 * num_tiles, num_directions) bytes. Directions x, y, z: device [direction],
 * ENU direction cosines. */
OSKB_API size_t oskb_station_beam_two_level_workspace_bytes(
        int precision_bytes, int num_tile_types, int num_tiles,
        int num_directions);
OSKB_API int oskb_station_beam_two_level_d(int num_tile_types,
        int num_elements, const double* el_x, const double* el_y,
        const double* el_z, const double* orientation_x_rad,
        const double* orientation_y_rad, double dipole_length_m,
        int normalise_element, int normalise_tile_array, int num_tiles,
        const double* tile_x, const double* tile_y, const double* tile_z,
        const int* tile_type, int normalise_station_array, int swap_xy,
        int is_3d, double frequency_hz, double beam_x, double beam_y,
        double beam_z, int num_directions, const double* x, const double* y,
        const double* z, void* workspace, size_t workspace_bytes,
        double* beam, void* stream);
OSKB_API int oskb_station_beam_two_level_f(int num_tile_types,
        int num_elements, const float* el_x, const float* el_y,
        const float* el_z, const double* orientation_x_rad,
        const double* orientation_y_rad, double dipole_length_m,
        int normalise_element, int normalise_tile_array, int num_tiles,
        const float* tile_x, const float* tile_y, const float* tile_z,
        const int* tile_type, int normalise_station_array, int swap_xy,
        int is_3d, double frequency_hz, double beam_x, double beam_y,
        double beam_z, int num_directions, const float* x, const float* y,
        const float* z, void* workspace, size_t workspace_bytes,
        float* beam, void* stream);

/* Relative direction cosines (l, m, n) about a sky position (ra0, dec0) to
 * ENU direction cosines (x, y, z) of a station at latitude lat, for hour
 * angle ha0 = lst - ra0 (radians). All arrays device [num]. Replaces the
 * kernel behind oskar_convert_relative_directions_to_enu_directions
 * (oskar/convert/define_convert_relative_directions_to_enu_directions.h;
 * src/oskar_convert_relative_directions_to_enu_directions.c:18-60), the
 * conversion the beam-pattern application applies to its pixel grid. */
OSKB_API int oskb_convert_relative_directions_to_enu_directions_d(int num,
        const double* l, const double* m, const double* n, double ha0_rad,
        double dec0_rad, double lat_rad, double* x, double* y, double* z,
        void* stream);
OSKB_API int oskb_convert_relative_directions_to_enu_directions_f(int num,
        const float* l, const float* m, const float* n, double ha0_rad,
        double dec0_rad, double lat_rad, float* x, float* y, float* z,
        void* stream);

/* Beam-image pixel grid: direction cosines (l, m, n) of num_l x num_m
 * pixels (m slowest, l fastest, l decreasing with the pixel index as FITS
 * images run) over a field of fov_lon x fov_lat radians; centred (the
 * beam-pattern application's grid): the axes run evenly between +-sin(fov
 * / 2); otherwise pixel centres step by the cell size asin(2 sin(fov / 2) /
 * num) from the centre pixel num / 2. Pixels beyond the sphere are NaN.
 * Host arrays [num_l * num_m]. Restates oskar_evaluate_image_lmn_grid_d
 * (oskar/math/src/oskar_evaluate_image_lmn_grid.c:149-227). */
OSKB_API int oskb_evaluate_image_lmn_grid(int num_l, int num_m,
        double fov_lon_rad, double fov_lat_rad, int centred, double* l,
        double* m, double* n);

/* Hierarchical aperture-array station of any depth (num_levels 2..16).
 * Level 0 holds num_types[0] leaf layouts (dipole arrays: num_elements
 * dipoles each at el_x/y/z [type][element], orientations orientation_x/y_rad
 * [type], one dipole length); each level l = 1..num_levels-1 holds
 * num_types[l] node types, each an array of children of level l - 1; the top
 * level holds one node type, the station (num_types[num_levels-1] == 1).
 * Node types are numbered level by level from level 1 upward (node n); node
 * n has the children child_start[n] .. child_start[n+1]-1 (host, CSR,
 * child_start[0] == 0, at least one child each) at ENU positions
 * child_x/y/z [child] (device, true positions in metres, relative to the
 * node's own centre) with child_type [child] (device, the index of the
 * child's node type in the level below, which must be less than that
 * level's num_types; NULL: every child is type 0, the reference's identical
 * children). normalise_array [level] (host): divide that level's array sum
 * by its number of children (level 0: the leaf array, by num_elements).
 * beam_enu [level][3] (host): the ENU pointing of that level's weights, the
 * reference's oskar_station_beam_horizon_direction of a station at that
 * depth. Beam [direction][2x2] of the station: at every level above 0,
 * sum_c w_c exp(i k r_c . d) x beam(type(c))[d] with w_c = exp(-i k r_c . b)
 * (oskar_dftw with the weights of oskar_station_evaluate_element_weights.c:
 * 15-66); level 0 is the fused single-level beam (oskb_station_beam_aa:
 * dipole pattern, leaf array factor, normalise_element, blanked below the
 * horizon). Replaces the recursion of
 * oskar_evaluate_station_beam_aperture_array.c:242-287 (each distinct node
 * type is evaluated once; identical or repeated children are indexed, not
 * copied); the normalisation to the beam direction
 * (oskar_station_beam.c:108-135) is the caller's, as in the reference.
 * workspace: device, at least oskb_station_beam_hierarchical_workspace_bytes
 * bytes (0 there: the description is invalid). Directions x, y, z: device
 * [direction], ENU direction cosines. oskb_station_beam_two_level_{d,f} is
 * the case num_levels = 2. */
OSKB_API size_t oskb_station_beam_hierarchical_workspace_bytes(
        int precision_bytes, int num_levels, const int* num_types,
        const int* child_start, int num_directions);
OSKB_API int oskb_station_beam_hierarchical_d(int num_levels,
        const int* num_types, int num_elements, const double* el_x,
        const double* el_y, const double* el_z,
        const double* orientation_x_rad, const double* orientation_y_rad,
        double dipole_length_m, int normalise_element,
        const int* normalise_array, const int* child_start,
        const double* child_x, const double* child_y, const double* child_z,
        const int* child_type, int swap_xy, int is_3d, double frequency_hz,
        const double* beam_enu, int num_directions, const double* x,
        const double* y, const double* z, void* workspace,
        size_t workspace_bytes, double* beam, void* stream);
OSKB_API int oskb_station_beam_hierarchical_f(int num_levels,
        const int* num_types, int num_elements, const float* el_x,
        const float* el_y, const float* el_z,
        const double* orientation_x_rad, const double* orientation_y_rad,
        double dipole_length_m, int normalise_element,
        const int* normalise_array, const int* child_start,
        const float* child_x, const float* child_y, const float* child_z,
        const int* child_type, int swap_xy, int is_3d, double frequency_hz,
        const double* beam_enu, int num_directions, const float* x,
        const float* y, const float* z, void* workspace,
        size_t workspace_bytes, float* beam, void* stream);

/* ------------------------------------------------------------------------
 * Sky and baseline preparation on the device.
 * ------------------------------------------------------------------------
 * (lon, lat) -> direction cosines (l, m[, n]) about (lon0, lat0); n may be
 * NULL. Replaces the kernel behind oskar_convert_lon_lat_to_relative_
 * directions (convert/define_convert_lon_lat_to_relative_directions.h). */
OSKB_API int oskb_convert_lon_lat_to_relative_directions_d(int num,
        const double* lon, const double* lat, double lon0_rad,
        double lat0_rad, double* l, double* m, double* n, void* stream);
OSKB_API int oskb_convert_lon_lat_to_relative_directions_f(int num,
        const float* lon, const float* lat, double lon0_rad,
        double lat0_rad, float* l, float* m, float* n, void* stream);
/* Apparent (RA, Dec) -> ENU direction cosines [station][source] for every
 * station in one launch (station st at local sidereal time lst_rad[st] and
 * latitude lat_rad[st], device double arrays). Replaces the per-station
 * kernel of oskar_convert_apparent_ra_dec_to_enu_directions
 * (convert/define_convert_apparent_ra_dec_to_enu_directions.h). */
OSKB_API int oskb_convert_ra_dec_to_enu_directions_d(int num_sources,
        const double* ra, const double* dec, int num_stations,
        const double* lst_rad, const double* lat_rad, double* x, double* y,
        double* z, void* stream);
OSKB_API int oskb_convert_ra_dec_to_enu_directions_f(int num_sources,
        const float* ra, const float* dec, int num_stations,
        const double* lst_rad, const double* lat_rad, float* x, float* y,
        float* z, void* stream);
/* mask[s] |= source s (direction cosines l, m, n about the phase centre) is
 * above the horizon of any of the stations (hour angle of the phase centre
 * ha0_rad_host[st], latitude lat_rad_host[st]: host arrays). The mask step
 * of oskar_sky_horizon_clip (sky/src/oskar_sky_horizon_clip.c:63-79,
 * sky/define_update_horizon_mask.h). */
OSKB_API int oskb_sky_horizon_mask_d(int num_sources, const double* l,
        const double* m, const double* n, int num_stations,
        const double* ha0_rad_host, const double* lat_rad_host,
        double dec0_rad, int* mask, void* stream);
OSKB_API int oskb_sky_horizon_mask_f(int num_sources, const float* l,
        const float* m, const float* n, int num_stations,
        const double* ha0_rad_host, const double* lat_rad_host,
        double dec0_rad, int* mask, void* stream);
/* Order-preserving compaction of num_columns sky columns by mask (the copy
 * step of oskar_sky_horizon_clip, sky/src/oskar_sky_horizon_clip.c:80-95):
 * columns_in / columns_out are host arrays of device pointers; *num_out
 * (host) receives the number kept. Synchronises the stream. */
OSKB_API int oskb_sky_compact_d(int num, const int* mask, int num_columns,
        const double* const* columns_in, double* const* columns_out,
        int* num_out, void* stream);
OSKB_API int oskb_sky_compact_f(int num, const int* mask, int num_columns,
        const float* const* columns_in, float* const* columns_out,
        int* num_out, void* stream);
/* Station (u, v, w) -> baseline (uu, vv, ww) = station q - station p for
 * p < q in the reference's baseline order, negated in the CASA convention
 * (convert/src/oskar_convert_station_uvw_to_baseline_uvw.c:13-29). */
OSKB_API int oskb_convert_station_uvw_to_baseline_uvw_d(int use_casa,
        int num_stations, int offset_in, const double* u, const double* v,
        const double* w, int offset_out, double* uu, double* vv, double* ww,
        void* stream);
OSKB_API int oskb_convert_station_uvw_to_baseline_uvw_f(int use_casa,
        int num_stations, int offset_in, const float* u, const float* v,
        const float* w, int offset_out, float* uu, float* vv, float* ww,
        void* stream);

/* Scaled Stokes I, Q, U, V of every source at freq_hz from the spectral
 * columns of a sky table: the reference channel nearest freq_hz, Q and U
 * from polarisation angle and fraction where only those are given, then
 * Gaussian line profiles, a curved power law, or a logarithmic or linear
 * spectral-index polynomial for I (Q, U, V follow I's ratio), or Faraday
 * rotation with a rotation measure. NaN coefficients count as 0; a source
 * whose nearest reference frequency is 0 keeps its values.
 * The arguments are those of the reference's kernel
 * (sky/src/oskar_sky_scale_flux_with_frequency.c:127-152, body
 * sky/define_sky_scale_flux_with_frequency.h:89-253), plus num_columns:
 * the table holds num_columns columns of capacity values (column k of
 * source s at table[capacity * k + s]); num_valid_columns is
 * [source][20] counts per column type (sky/oskar_sky_enum.h:14-35); a
 * col_ argument is the first column of its type, -1 if absent; a column
 * index outside [0, num_columns) reads as 0. col_i < 0 is
 * OSKB_ERR_INVALID_ARGUMENT (the reference's "no Stokes I column",
 * oskar_sky_scale_flux_with_frequency.c:57-62). All arrays on the device. */
OSKB_API int oskb_sky_scale_flux_with_frequency_d(int num_sources,
        int capacity, int num_columns, double freq_hz, const double* table,
        const int* num_valid_columns, int col_i, int col_q, int col_u,
        int col_v, int col_ref_freq, int col_lin_sp_index, int col_sp_index,
        int col_rot_meas, int col_pol_frac, int col_pol_ang,
        int col_ref_wavelength, int col_sp_curvature, int col_line_width,
        int col_freq_inc, double* out_i, double* out_q, double* out_u,
        double* out_v, void* stream);
OSKB_API int oskb_sky_scale_flux_with_frequency_f(int num_sources,
        int capacity, int num_columns, float freq_hz, const float* table,
        const int* num_valid_columns, int col_i, int col_q, int col_u,
        int col_v, int col_ref_freq, int col_lin_sp_index, int col_sp_index,
        int col_rot_meas, int col_pol_frac, int col_pol_ang,
        int col_ref_wavelength, int col_sp_curvature, int col_line_width,
        int col_freq_inc, float* out_i, float* out_q, float* out_u,
        float* out_v, void* stream);
/* The same for every channel of a band in one launch: frequency_hz is a
 * device array [num_channels]; columns is a host array of the 14 first
 * columns in the order of the col_ arguments above; outputs are
 * [channel][source], channel c at c * out_channel_stride
 * (>= num_sources when num_channels > 1). The FP32 variant rounds each
 * frequency to float, as the reference's FP32 kernel receives it. */
OSKB_API int oskb_sky_scale_flux_channels_d(int num_sources, int capacity,
        int num_columns, int num_channels, const double* frequency_hz,
        const double* table, const int* num_valid_columns,
        const int* columns, long long out_channel_stride, double* out_i,
        double* out_q, double* out_u, double* out_v, void* stream);
OSKB_API int oskb_sky_scale_flux_channels_f(int num_sources, int capacity,
        int num_columns, int num_channels, const double* frequency_hz,
        const float* table, const int* num_valid_columns,
        const int* columns, long long out_channel_stride, float* out_i,
        float* out_q, float* out_u, float* out_v, void* stream);

/* Cable-length phase errors applied in place to Jones [station][source]:
 * J <- diag(e^{i k dx_p}, e^{i k dy_p}) J for matrix Jones (matrix != 0;
 * an absent array keeps gain 1), J <- e^{i k dx_p} J for scalar Jones
 * (nothing without errors_x); wavenumber k = 2 pi f / c
 * (interferometer/define_jones_apply_cable_length_errors.h:3-74, called
 * from interferometer/src/oskar_jones_apply_cable_length_errors.c:23-141).
 * errors_x, errors_y: [station] metres, device, either may be NULL. */
OSKB_API int oskb_jones_apply_cable_length_errors_d(int matrix,
        int num_sources, int num_stations, double wavenumber,
        const double* errors_x, const double* errors_y, double* jones,
        void* stream);
OSKB_API int oskb_jones_apply_cable_length_errors_f(int matrix,
        int num_sources, int num_stations, float wavenumber,
        const float* errors_x, const float* errors_y, float* jones,
        void* stream);
/* Station gains applied in place: J[p][s] <- G_p J[p][s], G_p a 2x2
 * complex matrix (matrix != 0) or a complex scalar
 * (interferometer/define_jones_apply_station_gains.h:3-45, called from
 * interferometer/src/oskar_jones_apply_station_gains.c:23-121). gains:
 * [station], device. */
OSKB_API int oskb_jones_apply_station_gains_d(int matrix, int num_sources,
        int num_stations, const double* gains, double* jones, void* stream);
OSKB_API int oskb_jones_apply_station_gains_f(int matrix, int num_sources,
        int num_stations, const float* gains, float* jones, void* stream);

/* ------------------------------------------------------------------------
 * Learned station-beam surrogate.
 * ------------------------------------------------------------------------
 * A multilayer perceptron with sine activations (dims[0] -> ... ->
 * dims[num_layers]; sin(omega0 z) after every layer but the last), trained
 * and evaluated by this library's own FP32 kernels. Parameters are one
 * device array: per layer W [out][in] then b [out].
 *   oskb_mlp_forward keeps the activations of the batch for
 *   oskb_mlp_backward, which overwrites the gradients (same layout as the
 *   parameters) with d loss / d parameter for the output gradient dy;
 *   oskb_mlp_mse: loss += mean (y - t)^2, dy = 2 (y - t) / count (dy may
 *   alias y; loss may be NULL);
 *   oskb_mlp_train: steps of Adam (beta 0.9, 0.999) on random minibatches
 *   of the (x, target) samples with a cosine-decayed learning rate; the
 *   loss of every report_every-th step (and of the last) goes to
 *   loss_history (host, (steps - 1) / report_every + 2 entries);
 *   oskb_mlp_infer: outputs for count inputs, in chunks.
 * x, y, target, dy: device, row-major [sample][feature]. */
typedef struct oskb_Mlp oskb_Mlp;
OSKB_API oskb_Mlp* oskb_mlp_create(int num_layers, const int* dims,
        float omega0, unsigned long long seed, int* status);
OSKB_API void oskb_mlp_free(oskb_Mlp* net);
OSKB_API int oskb_mlp_num_params(const oskb_Mlp* net);
OSKB_API float* oskb_mlp_params(oskb_Mlp* net);
OSKB_API float* oskb_mlp_grads(oskb_Mlp* net);
/* which: 0 parameters, 1 gradients; host arrays of oskb_mlp_num_params. */
OSKB_API int oskb_mlp_copy_to_host(const oskb_Mlp* net, int which,
        float* host);
OSKB_API int oskb_mlp_set_params(oskb_Mlp* net, const float* host);
OSKB_API int oskb_mlp_forward(oskb_Mlp* net, int batch, const float* x,
        float* y, void* stream);
OSKB_API int oskb_mlp_backward(oskb_Mlp* net, int batch, const float* dy,
        void* stream);
OSKB_API int oskb_mlp_mse(long long count, const float* y,
        const float* target, float* dy, float* loss, void* stream);
OSKB_API int oskb_mlp_adam_step(oskb_Mlp* net, float lr, float beta1,
        float beta2, float eps, void* stream);
OSKB_API int oskb_mlp_train(oskb_Mlp* net, int num_samples, const float* x,
        const float* target, int batch, int steps, float lr_max,
        unsigned long long seed, int report_every, float* loss_history,
        void* stream);
OSKB_API int oskb_mlp_infer(oskb_Mlp* net, long long count, const float* x,
        float* y, int chunk, void* stream);

/* Exact normalised array factor A(kappa) = (1/N) sum_e exp(i (x_e kx +
 * y_e ky)) of a planar layout, for training samples (FP64 phases, FP32
 * output [count][2]). kappa in rad/m, layout in metres; device arrays. */
OSKB_API int oskb_array_factor_samples_f(int num_elements,
        const float* layout_x, const float* layout_y, long long count,
        const float* kappa_x, const float* kappa_y, float* af, void* stream);

/* Station beam (Jones E, FP32) of stations built from num_types planar
 * dipole layouts, station st being layout station_type_host[st] rotated by
 * rotation_rad[st] (elements and dipole orientation: Euler angles x = y =
 * rotation), phased to beam_enu[st] and normalised there (array and final
 * normalisation on, element normalisation optional) - the beam that
 * oskb_station_beam_aa_f gives for those stations. The array factor comes
 * from networks[type] (trained on A(kappa) with inputs kappa / kappa_scale)
 * wherever |kappa| >= kappa_main and from the exact sum inside the main
 * lobe. Every audit_stride-th network value is checked against the exact
 * sum; if the largest difference exceeds audit_bound (A is 1 at the
 * pointing), every network value is replaced by the exact sum. audit (host,
 * 5 values): largest audited |A_net - A|, rms audited error, number
 * audited, 1 if the fallback ran, number of network evaluations.
 * station_type_host and networks are host arrays; the rest device. */
OSKB_API int oskb_station_beam_surrogate_f(int num_stations, int num_types,
        int num_elements, const int* station_type_host,
        const double* rotation_rad, const float* layout_x,
        const float* layout_y, oskb_Mlp* const* networks,
        double dipole_length_m, int normalise_element, double frequency_hz,
        const double* beam_enu, int num_directions, const float* x,
        const float* y, const float* z, double kappa_main,
        double kappa_scale, int audit_stride, double audit_bound,
        float* beam, double* audit, void* stream);

/* Parallactic-angle rotation R [station][source] (real 2x2 rotation) for
 * stations at latitude lat_rad[station] and local sidereal time
 * lst_rad[station] = gast + longitude. Replaces the kernel behind
 * oskar_evaluate_jones_R (oskar/interferometer/src/oskar_evaluate_jones_R.c:
 * 21-147; define_evaluate_jones_R.h:3-29). Device pointers. */
OSKB_API int oskb_evaluate_jones_R_d(int num_sources, const double* ra_rad,
        const double* dec_rad, int num_stations, const double* lat_rad,
        const double* lst_rad, double* jones, void* stream);
OSKB_API int oskb_evaluate_jones_R_f(int num_sources, const float* ra_rad,
        const float* dec_rad, int num_stations, const double* lat_rad,
        const double* lst_rad, float* jones, void* stream);

/* ------------------------------------------------------------------------
 * Tensor-core compensated cross-correlation (point sources, no smearing).
 * ------------------------------------------------------------------------
 * Same result as oskb_cross_correlate_d with gaussian = 0,
 * frac_bandwidth = 0 and time_int_sec = 0, computed as a Hermitian rank-k
 * update on the sm_100a tensor cores (tcgen05; by default the integer form:
 * 24-bit fixed-point entries in three signed 8-bit limbs, the sources in
 * amplitude buckets with a scale each, exact S32 accumulation; else the
 * FP16 hi/lo form: three products, FP32 accumulation drained to FP64; see
 * oskb_tc_arithmetic); relative visibility error against FP64 below 1e-6
 * (L2 and max). Every brightness matrix must be positive
 * semi-definite (I >= sqrt(Q^2 + U^2 + V^2)); oskb_tc_status() reports a
 * violation. It is the fast branch of oskar_cross_correlate
 * (oskar/correlate/oskar_cross_correlate.h:49) for source_type 0 without
 * smearing; station_u/v are only used by the uv filter.
 * workspace: device scratch of at least
 * oskb_cross_correlate_tc_workspace_bytes() bytes, or NULL to let the library
 * keep one per device (allocated on first use, grown on demand). */
OSKB_API size_t oskb_cross_correlate_tc_workspace_bytes(int num_sources,
        int num_stations);
OSKB_API int oskb_cross_correlate_tc_d(int use_casa_phase_convention,
        int num_sources, int num_stations, int offset_out,
        const double* jones, const double* I, const double* Q,
        const double* U, const double* V, const double* station_u,
        const double* station_v, double uv_min_lambda, double uv_max_lambda,
        double inv_wavelength, double* vis, void* workspace,
        size_t workspace_bytes, void* stream);

/* FP32 form of oskb_cross_correlate_tc_d: J, fluxes, station u, v and vis
 * in FP32 (as oskb_cross_correlate_f takes them), the sums formed by the
 * integer tensor-core form (FP64 sums of exact integer products, error
 * ~4e-7 against FP64, inside FP32's own 1e-5) and added into vis once per
 * call. Replaces oskar_cross_correlate's FP32 point-source branch without
 * smearing (oskar/correlate/src/oskar_cross_correlate.c:413-433, the CUDA
 * call of the single-precision matrix case) where every brightness matrix
 * is positive semi-definite: otherwise nothing is added and
 * oskb_tc_status(workspace) reports flags bit 0 (then use
 * oskb_cross_correlate_f). jones must be 16-byte aligned. workspace: at
 * least oskb_cross_correlate_tc_f_workspace_bytes() bytes, or NULL. */
OSKB_API size_t oskb_cross_correlate_tc_f_workspace_bytes(int num_sources,
        int num_stations);
OSKB_API int oskb_cross_correlate_tc_f(int use_casa_phase_convention,
        int num_sources, int num_stations, int offset_out, const float* jones,
        const float* I, const float* Q, const float* U, const float* V,
        const float* station_u, const float* station_v, float uv_min_lambda,
        float uv_max_lambda, float inv_wavelength, float* vis,
        void* workspace, size_t workspace_bytes, void* stream);

/* FP64-class tensor-core cross-correlation (no counterpart in the
 * reference; replaces oskar_cross_correlate's FP64 point-source branch
 * without smearing, oskar/correlate/src/oskar_cross_correlate.c:434-455,
 * where every brightness matrix is positive semi-definite). Same arguments
 * and result as oskb_cross_correlate_tc_d, computed on the 8-bit integer
 * tensor cores to FP64-class accuracy: each entry of J C (FP64, C the
 * Cholesky factor of the brightness) as a 48-bit fixed-point integer in six
 * signed 8-bit limbs, the sources ordered into amplitude buckets with a
 * scale each, the limb products of weight >= 2^-40 (21 per K step) summed
 * exactly in 32-bit integer accumulators and combined in FP64; relative
 * visibility error against the FP64 direct kernel ~1e-14 (tested <= 1e-12,
 * L2 and max). If a brightness matrix is not positive semi-definite,
 * nothing is added to vis and oskb_tc_status(workspace) reports flags bit
 * 0: correlate that call with oskb_cross_correlate_d instead.
 * workspace: device scratch of at least
 * oskb_cross_correlate_tc64_workspace_bytes() bytes (56 B per
 * station-source, rounded up to blocks of 32 x 32, plus about 8 B per
 * source), or NULL to let the library keep one per device and stream. */
OSKB_API size_t oskb_cross_correlate_tc64_workspace_bytes(int num_sources,
        int num_stations);
OSKB_API int oskb_cross_correlate_tc64_d(int use_casa_phase_convention,
        int num_sources, int num_stations, int offset_out,
        const double* jones, const double* I, const double* Q,
        const double* U, const double* V, const double* station_u,
        const double* station_v, double uv_min_lambda, double uv_max_lambda,
        double inv_wavelength, double* vis, void* workspace,
        size_t workspace_bytes, void* stream);

/* FP64-class fused block (no counterpart in the reference; replaces the
 * per-channel Jones K -> join -> FP64 correlate sequence of sim_baselines,
 * oskar/interferometer/src/oskar_interferometer_run_block.c:277-334, for
 * point sources without smearing whose brightness matrices are positive
 * semi-definite): the same block as oskb_correlate_block_tc_d (E FP64
 * [station][source][2x2] shared by the block, station_uvw
 * [time][3][station] metres, inv_wavelength[channel], vis
 * [time][channel][baseline][2x2] FP64, added), at FP64-class accuracy:
 * K E C formed in FP64 (phase reduced mod 1, sincospi) as 48-bit fixed
 * point in six 8-bit limbs per amplitude bucket, contracted on the integer
 * tensor cores as oskb_cross_correlate_tc64_d. If a brightness matrix is
 * not positive semi-definite, nothing is added and oskb_tc_status reports
 * flags bit 0 (then use oskb_correlate_block_direct_d). Problems are
 * processed in groups that fit the workspace (NULL: library-kept). */
OSKB_API size_t oskb_correlate_block_tc64_workspace_bytes(int num_sources,
        int num_stations, int num_problems);
OSKB_API int oskb_correlate_block_tc64_d(int use_casa_phase_convention,
        int num_sources, int num_stations, int num_times, int num_channels,
        const double* E, const double* l, const double* m, const double* n,
        const double* I, const double* Q, const double* U, const double* V,
        const double* station_uvw, const double* inv_wavelength,
        double uv_min_lambda, double uv_max_lambda, double* vis,
        void* workspace, size_t workspace_bytes, void* stream);

/* The same, with the auto-correlations of every station from the same
 * contraction (the diagonal station pairs of the diagonal tiles, V_pp =
 * J_p B J_p^H) added into autos [num_times][num_channels][num_stations]
 * [2x2] FP64, as oskb_correlate_block_tc_auto does for the 1e-6 form
 * (the reference's oskar_auto_correlate per (dump, channel),
 * oskar/correlate/define_auto_correlate.h:8-82). */
OSKB_API int oskb_correlate_block_tc64_auto_d(int use_casa_phase_convention,
        int num_sources, int num_stations, int num_times, int num_channels,
        const double* E, const double* l, const double* m, const double* n,
        const double* I, const double* Q, const double* U, const double* V,
        const double* station_uvw, const double* inv_wavelength,
        double uv_min_lambda, double uv_max_lambda, double* vis,
        double* autos, void* workspace, size_t workspace_bytes,
        void* stream);

/* Direct (FP64 or FP32) block correlator with smearing: for every (dump t,
 * channel c) of a block, in ONE persistent launch,
 *   vis[t][c][pq] += sum_s smear_pq(s) (J_p B J_q^H)(s),  J = K(t, c) E,
 * with K exactly as oskar_evaluate_jones_K forms it (phase
 * 2 pi / lambda_c (u l + v m + w (n - 1)) in the working precision; K = 0
 * where I is outside (source_filter_min, source_filter_max]), and smear_pq
 * the Gaussian, bandwidth and time-average factors of the reference's
 * correlator (oskar/correlate/define_cross_correlate.h:16-111). Replaces
 * the per-(dump, chunk, channel) sequence Jones K -> join -> correlate of
 * sim_baselines (oskar/interferometer/src/oskar_interferometer_run_block.c:
 * 156-336); K and J are formed in shared memory, never stored.
 *   E: [station][source] 2x2 (or [dump][station][source] if E_per_dump);
 *      NULL for identity (J = K);
 *   a, b, c: Gaussian shape per source, or all NULL for point sources.
 *      Sources of the reference's point-source chunks carry a = b = c = 0
 *      (exp(-0) = 1 exactly), so one call covers chunks of both kinds;
 *   station_uvw: [dump][3][station] metres; station_x/y: ECEF offsets
 *      (time smearing only); inv_wavelength: [channel] = f_c / c0;
 *      gha0_rad: [dump] Greenwich hour angle of the phase centre (time
 *      smearing only);
 *   uv_filter_units: 0 metres (scaled per channel), 1 wavelengths;
 *   vis: [dump][channel][baseline][2x2], accumulated.
 * All arrays are device memory; inv_wavelength and gha0_rad are double in
 * both precisions. The launch schedule (grid, item order) is chosen per
 * block shape by timing candidates on a sample of the block the first time
 * that shape is seen (OSKB_AUTOTUNE=0: fixed default; OSKB_BLOCK_SCHEDULE=
 * "ctas_per_sm,tile_major": forced). Results do not depend on it. */
OSKB_API int oskb_correlate_block_direct_d(int casa, int num_sources,
        int num_stations, int num_times, int num_channels, const double* E,
        int E_per_dump, const double* I, const double* Q, const double* U,
        const double* V, const double* l, const double* m, const double* n,
        const double* a, const double* b, const double* c,
        const double* station_uvw, const double* station_x,
        const double* station_y, const double* inv_wavelength,
        double channel_bandwidth_hz, double time_average_sec,
        const double* gha0_rad, double dec0_rad, double uv_min,
        double uv_max, int uv_filter_units, double source_filter_min,
        double source_filter_max, double* vis, void* stream);
OSKB_API int oskb_correlate_block_direct_f(int casa, int num_sources,
        int num_stations, int num_times, int num_channels, const float* E,
        int E_per_dump, const float* I, const float* Q, const float* U,
        const float* V, const float* l, const float* m, const float* n,
        const float* a, const float* b, const float* c,
        const float* station_uvw, const float* station_x,
        const float* station_y, const double* inv_wavelength,
        double channel_bandwidth_hz, double time_average_sec,
        const double* gha0_rad, double dec0_rad, double uv_min,
        double uv_max, int uv_filter_units, double source_filter_min,
        double source_filter_max, float* vis, void* stream);
/* As oskb_correlate_block_direct, with the brightness of every channel:
 * I, Q, U, V hold [channel][source] values, channel c at
 * c * flux_channel_stride (>= num_sources; 0 = one set for every channel),
 * e.g. from oskb_sky_scale_flux_channels. The source filter applies to
 * each channel's own I, as the reference filters on the flux scaled to the
 * channel frequency (oskar_interferometer_run_block.c:183-190, 277-281). */
OSKB_API int oskb_correlate_block_direct_spectral_d(int casa,
        int num_sources, int num_stations, int num_times, int num_channels,
        const double* E, int E_per_dump, const double* I, const double* Q,
        const double* U, const double* V, long long flux_channel_stride,
        const double* l, const double* m, const double* n, const double* a,
        const double* b, const double* c, const double* station_uvw,
        const double* station_x, const double* station_y,
        const double* inv_wavelength, double channel_bandwidth_hz,
        double time_average_sec, const double* gha0_rad, double dec0_rad,
        double uv_min, double uv_max, int uv_filter_units,
        double source_filter_min, double source_filter_max, double* vis,
        void* stream);
OSKB_API int oskb_correlate_block_direct_spectral_f(int casa,
        int num_sources, int num_stations, int num_times, int num_channels,
        const float* E, int E_per_dump, const float* I, const float* Q,
        const float* U, const float* V, long long flux_channel_stride,
        const float* l, const float* m, const float* n, const float* a,
        const float* b, const float* c, const float* station_uvw,
        const float* station_x, const float* station_y,
        const double* inv_wavelength, double channel_bandwidth_hz,
        double time_average_sec, const double* gha0_rad, double dec0_rad,
        double uv_min, double uv_max, int uv_filter_units,
        double source_filter_min, double source_filter_max, float* vis,
        void* stream);
/* Text report of the schedules the block autotuner has chosen (one line
 * per block shape, with the sample time of every candidate). Returns the
 * number of characters written. */
OSKB_API int oskb_block_tune_report(char* buf, int len);

/* Block plan: the host driver of oskb_correlate_block_direct for one block
 * shape. It keeps the sky, station offsets and beam on the device, and
 * page-locked host buffers for the per-block inputs (station uvw
 * [dump][3][station] and Greenwich hour angle [dump] of the phase centre)
 * and the output (visibilities [dump][channel][baseline][2x2]). Execute
 * runs: upload uvw and hour angles, clear, correlate, download, on the
 * plan's own stream; the first execute runs eagerly and captures the
 * sequence as a CUDA graph, later executes replay the graph. Arrays passed
 * to the setters are host arrays of the plan's precision (precision_bytes
 * 8: double, 4: float); frequency_hz is a host array [num_channels]. The
 * other arguments mean what they mean for oskb_correlate_block_direct. */
typedef struct oskb_BlockPlan oskb_BlockPlan;
OSKB_API oskb_BlockPlan* oskb_block_plan_create(int precision_bytes,
        int casa, int num_stations, int num_sources, int num_times,
        int num_channels, int gaussian, int with_beam, int beam_per_dump,
        const double* frequency_hz, double channel_bandwidth_hz,
        double time_average_sec, double dec0_rad, double uv_min,
        double uv_max, int uv_filter_units, double source_filter_min,
        double source_filter_max, int* status);
OSKB_API int oskb_block_plan_set_sky(oskb_BlockPlan* plan, const void* I,
        const void* Q, const void* U, const void* V, const void* l,
        const void* m, const void* n, const void* a, const void* b,
        const void* c);
/* Spectral sky: the plan scales the brightness of every source to every
 * channel once, on the device (oskb_sky_scale_flux_channels), and each
 * block correlates with those per-channel values; the reference rescales
 * per dump and channel inside its block loop
 * (oskar_interferometer_run_block.c:183-190). table: host [num_columns]
 * [capacity] sky table of the plan's precision; num_valid_columns: host
 * [num_sources][20]; columns: host, the 14 first-column indices in the
 * order of oskb_sky_scale_flux_with_frequency's col_ arguments. Once it is
 * set, oskb_block_plan_set_sky may pass NULL for I, Q, U and V. */
OSKB_API int oskb_block_plan_set_spectral_sky(oskb_BlockPlan* plan,
        int capacity, int num_columns, const void* table,
        const int* num_valid_columns, const int* columns);
OSKB_API int oskb_block_plan_set_stations(oskb_BlockPlan* plan,
        const void* ecef_x, const void* ecef_y);
OSKB_API int oskb_block_plan_set_beam(oskb_BlockPlan* plan, const void* E);
OSKB_API void* oskb_block_plan_host_uvw(oskb_BlockPlan* plan);
OSKB_API double* oskb_block_plan_host_gha0(oskb_BlockPlan* plan);
OSKB_API const void* oskb_block_plan_host_vis(oskb_BlockPlan* plan);
OSKB_API int oskb_block_plan_execute(oskb_BlockPlan* plan);
OSKB_API int oskb_block_plan_synchronize(oskb_BlockPlan* plan);
/* Graph replays so far, or -1 while the plan runs without a graph. */
OSKB_API int oskb_block_plan_graph_launches(const oskb_BlockPlan* plan);
OSKB_API void oskb_block_plan_free(oskb_BlockPlan* plan);

/* Pipelined tensor-core blocks: a plan with two slots of device buffers.
 * oskb_tc_plan_enqueue returns at once; it uploads the block's E
 * ([station][source][2x2] FP32) and station uvw ([time][3][station]) from
 * host memory on a copy-in stream, correlates the block (as
 * oskb_correlate_block_tc, the visibility block cleared first) on a compute
 * stream once the upload and the slot's previous download are done, and
 * downloads the visibilities ([time][channel][baseline][2x2] FP64) group by
 * group on a copy-out stream. So block b + 1's upload overlaps block b's
 * correlation. Host buffers must stay valid until oskb_tc_plan_wait (they
 * should be page-locked for the copies to overlap); the sky (l, m, n and
 * Stokes, host arrays) is uploaded once by oskb_tc_plan_set_sky.
 * The plan owns its contraction workspace (up to 16 problems' operand
 * images, at most half the device memory free at creation). The first
 * enqueue picks the contraction form by timing the integer form, FP16
 * square tiles and FP16 wide tiles on its own block (it waits for them;
 * environment OSKB_TC_PLAN_FORM = 1, 3, 4 or 5 fixes a form instead, 0 the
 * library default; OSKB_TC_PLAN_TUNE=0 skips the timing); each slot's
 * compute work is then captured into a CUDA graph at its first block and
 * replayed for the later ones (OSKB_TC_PLAN_GRAPH=0: launched eagerly). The
 * downloads stay outside the graph. No reference counterpart (the
 * reference's block loop is oskar_interferometer_run_block.c:28-153). */
typedef struct oskb_TcPlan oskb_TcPlan;
OSKB_API oskb_TcPlan* oskb_tc_plan_create(int casa, int num_sources,
        int num_stations, int num_times, int num_channels,
        const double* freqs_hz, double uv_min_lambda, double uv_max_lambda,
        int* status);
OSKB_API int oskb_tc_plan_set_sky(oskb_TcPlan* plan, const double* l,
        const double* m, const double* n, const double* I, const double* Q,
        const double* U, const double* V);
OSKB_API int oskb_tc_plan_enqueue(oskb_TcPlan* plan, const float* E_host,
        const double* station_uvw_host, double* vis_host);
OSKB_API int oskb_tc_plan_wait(oskb_TcPlan* plan);
OSKB_API void oskb_tc_plan_free(oskb_TcPlan* plan);
/* The plan's contraction form: 0 library default, 1 integer (square
 * tiles), 3 FP16 square, 4 FP16 wide, 5 FP16 pairs (2 is not a form). */
OSKB_API int oskb_tc_plan_form(const oskb_TcPlan* plan);
/* Graph replays so far (0 while the plan runs eagerly). */
OSKB_API int oskb_tc_plan_graph_launches(const oskb_TcPlan* plan);
/* The tuning times (ms) of forms 1, 3 and 4 on the first block, -1 where
 * not timed. ms: host [3]. */
OSKB_API int oskb_tc_plan_tuning_ms(const oskb_TcPlan* plan, double* ms);

/* Fused block: for every (time t, channel c) of a block,
 *   vis[t][c] += sum_s (K_p E_p C)(s) (K_q E_q C)(s)^H
 * with K_p(s) = exp(2 pi i (u_p l + v_p m + w_p (n - 1)) / lambda_c) formed
 * in FP64 (mod-1 reduced) from station_uvw[t][3][num_stations] (metres) and
 * inv_wavelength[c]; E is FP32 [station][source][2x2], shared by the whole
 * block. vis is [num_times][num_channels][num_baselines][2x2] FP64 in the
 * reference's baseline order. This replaces the per-channel sequence
 * Jones K -> join -> correlate of sim_baselines
 * (oskar/interferometer/src/oskar_interferometer_run_block.c:277-334) for
 * point sources without smearing. The (t, c) problems are processed in
 * groups that fit the workspace (NULL: a library-kept workspace sized for
 * the whole block; query oskb_correlate_block_tc_workspace_bytes with
 * num_problems = num_times * num_channels). */
OSKB_API size_t oskb_correlate_block_tc_workspace_bytes(int num_sources,
        int num_stations, int num_problems);
OSKB_API int oskb_correlate_block_tc(int use_casa_phase_convention,
        int num_sources, int num_stations, int num_times, int num_channels,
        const float* E, const double* l, const double* m, const double* n,
        const double* I, const double* Q, const double* U, const double* V,
        const double* station_uvw, const double* inv_wavelength,
        double uv_min_lambda, double uv_max_lambda, double* vis,
        void* workspace, size_t workspace_bytes, void* stream);
/* The same with E in FP64 [station][source][2x2] (an FP64 caller's Jones E
 * or R E as it comes, e.g. oskar_Jones of type OSKAR_DOUBLE_COMPLEX_MATRIX):
 * each entry is rounded to FP32 once on load before the FP16 hi/lo split,
 * and that rounding (2^-24 relative) is part of the stated 1e-6 error
 * against the FP64 chain. */
OSKB_API int oskb_correlate_block_tc_d(int use_casa_phase_convention,
        int num_sources, int num_stations, int num_times, int num_channels,
        const double* E, const double* l, const double* m, const double* n,
        const double* I, const double* Q, const double* U, const double* V,
        const double* station_uvw, const double* inv_wavelength,
        double uv_min_lambda, double uv_max_lambda, double* vis,
        void* workspace, size_t workspace_bytes, void* stream);
/* The same, with the auto-correlations of every station from the same
 * contraction: the diagonal station pairs of the diagonal tiles are
 * V_pp = J_p B J_p^H, added into autos [num_times][num_channels]
 * [num_stations][2x2] FP64 (the reference's oskar_auto_correlate per
 * (dump, channel), oskar/correlate/define_auto_correlate.h:8-82, fused into
 * the correlation at no extra tensor work). */
OSKB_API int oskb_correlate_block_tc_auto(int use_casa_phase_convention,
        int num_sources, int num_stations, int num_times, int num_channels,
        const float* E, const double* l, const double* m, const double* n,
        const double* I, const double* Q, const double* U, const double* V,
        const double* station_uvw, const double* inv_wavelength,
        double uv_min_lambda, double uv_max_lambda, double* vis,
        double* autos, void* workspace, size_t workspace_bytes,
        void* stream);

/* Host-buffer block driver: the same computation as
 * oskb_correlate_block_tc with every array in HOST memory (page-locked for
 * full-speed copies): the inputs are copied to library-kept device buffers,
 * the visibility block is cleared, correlated and copied back into vis
 * ([num_times][num_channels][num_baselines][2x2] FP64, overwritten). The
 * call returns when vis holds the result. freqs_hz has num_channels
 * entries. The role of oskar_interferometer_run_block
 * (oskar/interferometer/oskar_interferometer.h:80) for a block of point
 * sources without smearing. */
OSKB_API int oskb_run_block_tc_host(int use_casa_phase_convention,
        int num_sources, int num_stations, int num_times, int num_channels,
        const float* E, const double* l, const double* m, const double* n,
        const double* I, const double* Q, const double* U, const double* V,
        const double* station_uvw, const double* freqs_hz,
        double uv_min_lambda, double uv_max_lambda, double* vis,
        void* stream);

/* Timing of the tensor-core contraction kernel: while enabled, CUDA events
 * are recorded around every launch of it; oskb_tc_timing_read() waits for
 * them and returns the summed milliseconds and the launch count since the
 * last read (or enable). No effect on results. */
OSKB_API int oskb_tc_timing(int enable);
OSKB_API int oskb_tc_timing_read(double* total_ms, int* launches);

/* Allocation-free form of oskb_cross_correlate_tc_d (no counterpart in the
 * reference). For callers that cannot allocate device memory while they
 * correlate: a process holding a fixed device-memory budget reserved at
 * start-up (for example a real-time pipeline stage sharing the GPU), or a
 * latency-critical loop that cannot afford the device-wide synchronisation
 * that cudaMalloc may cause. It computes the same visibilities but takes its
 * scratch from a 64 MiB array that the library declares in device memory
 * (held by every GPU that loads the library until the process exits), and
 * calls no cudaMalloc, cudaFree or allocating library routine.
 *  - Limit: 32 bytes per station-source after rounding up to blocks of 32
 *    stations x 32 sources, plus 256 bytes (e.g. 512 stations x 4,064
 *    sources; 4,096 sources do not fit): the FP16 form's operand image,
 *    so the limit holds whichever contraction form runs (the default
 *    integer form's image is 24 bytes per station-source, with up to 15
 *    more blocks of sources of bucket padding, and its source-order tables
 *    about 8 bytes per source: smaller for all but a few sources, and the
 *    check takes the larger of the two). Larger calls return
 *    OSKB_ERR_OUT_OF_RANGE (-5) with the sizes in oskb_last_error(); split
 *    the sources into chunks, since vis is accumulated.
 *  - The first call on a device takes the array's device address
 *    (cudaGetSymbolAddress, with that device current); make that first call
 *    before any stream capture.
 *  - Every call shares the one array: calls whose work overlaps on the GPU
 *    (different streams without ordering between them, or several host
 *    threads) race and corrupt each other's results. Order them, for example
 *    on one stream.
 *  - oskb_tc_status() does not read this array: oskb_tc_noalloc_status()
 *    does (below). */
OSKB_API int oskb_cross_correlate_tc_noalloc_d(int use_casa_phase_convention,
        int num_sources, int num_stations, int offset_out,
        const double* jones, const double* I, const double* Q,
        const double* U, const double* V, const double* station_u,
        const double* station_v, double uv_min_lambda, double uv_max_lambda,
        double inv_wavelength, double* vis, void* stream);

/* Status words of the last oskb_cross_correlate_tc_noalloc_d call on the
 * current device (no counterpart in the reference), read from the header of
 * the library's static scratch array without allocating: flags bit 0 = a
 * brightness matrix was not positive semi-definite; wait_error != 0 = a
 * bounded device-side wait expired, so that call's visibilities are
 * incomplete. Synchronises with the device. */
OSKB_API int oskb_tc_noalloc_status(int* flags, int* wait_error);

/* Status words of the last tensor-core call that used this workspace (NULL:
 * the library-kept workspace used last on the current device, each host
 * stream having its own; synchronises with the device): flags bit 0 = a
 * brightness matrix was not positive semi-definite; wait_error != 0 = a
 * bounded device-side wait expired (the call's result is invalid). */
OSKB_API int oskb_tc_status(const void* workspace, int* flags,
        int* wait_error);
/* Tile shape of the last tensor-core contraction launched, 0 before the
 * first. FP16 form: 128 (128 x 128 tiles of G per CTA), 256 (128 x 256 per
 * CTA) or 512 (256 x 256 per pair of CTAs, cta_group::2); the environment
 * variable OSKB_TC_TILE (128, 256 or 512) selects the FP16 form with that
 * tile (with OSKB_TC_ARITH=fp16 and no tile set: wide tiles when a launch
 * has at least two per SM, else square). Integer form: 128 (128 x 128 per
 * CTA). */
OSKB_API int oskb_tc_tile_columns(void);
/* Arithmetic of the last tensor-core contraction launched, 0 before the
 * first: 8 for the default integer form (the sources ordered into
 * amplitude buckets, factor 2 apart, each with its own scale; each scaled
 * entry a 24-bit fixed-point integer held as three signed 8-bit limbs; six
 * 8-bit tcgen05 MMAs per K step into exact S32 accumulators, square tiles),
 * 16 for the FP16 hi/lo form (three FP16 MMAs per K step into FP32
 * accumulators drained to FP64), which OSKB_TC_ARITH=fp16, or any
 * OSKB_TC_TILE setting, selects. */
OSKB_API int oskb_tc_arithmetic(void);

/* ------------------------------------------------------------------------
 * Visibility files (.vis, OSKAR binary format version 2): block
 * finalisation / output, replacing oskar_vis_header_write
 * (oskar/vis/src/oskar_vis_header_write.c:20-253) and
 * oskar_vis_block_write (oskar/vis/src/oskar_vis_block_write.c:16-70).
 * ------------------------------------------------------------------------
 * HOST pointers throughout. oskb_vis_file_create opens the file, writes the
 * file header and the visibility header: amp_type is the OSKAR type code
 * of the visibilities (complex, or complex matrix for 4 polarisations;
 * single 0x04 or double 0x08 | complex 0x20 | matrix 0x40),
 * coord_precision 0x04 or 0x08 the type of station_x/y/z (offset ECEF,
 * [station]), element_x/y/z (ENU, [station][element], num_elements
 * [station] or NULL) and of the per-block station (u, v, w);
 * element_feed_angles: double [feed X, Y][angle a, b, c][all elements] or
 * NULL; station_diameter_m [station] or NULL (0); station_names
 * [station] or NULL (""); telescope_path, settings (file contents) may be
 * NULL. date_time, version, cwd, username: the metadata strings, NULL for
 * the current time, this library's version, the working directory and
 * $USERNAME / $USER. max_times_per_block / max_channels_per_block <= 0
 * mean all. On error returns NULL with *status set.
 * oskb_vis_file_write_block writes one block: dimensions, then the
 * auto-correlations [time][channel][station] (if the file has them), the
 * cross-correlations [time][channel][baseline] and, when all three are
 * given, station u, v, w [time][station] metres. */
typedef struct oskb_VisFile oskb_VisFile;
OSKB_API oskb_VisFile* oskb_vis_file_create(const char* filename,
        int amp_type, int coord_precision, int max_times_per_block,
        int num_times_total, int max_channels_per_block,
        int num_channels_total, int num_stations, int write_autocorr,
        int write_crosscorr, int casa_phase_convention, double freq_start_hz,
        double freq_inc_hz, double channel_bandwidth_hz,
        double time_start_mjd_utc, double time_inc_sec,
        double time_average_sec, int phase_centre_coord_type,
        double phase_centre_lon_deg, double phase_centre_lat_deg,
        double telescope_lon_deg, double telescope_lat_deg,
        double telescope_alt_m, const void* station_x, const void* station_y,
        const void* station_z, const double* station_diameter_m,
        const char* const* station_names, const int* num_elements,
        const void* element_x, const void* element_y, const void* element_z,
        const double* element_feed_angles, const char* telescope_path,
        const char* settings, const char* date_time, const char* version,
        const char* cwd, const char* username, int* status);
OSKB_API int oskb_vis_file_write_block(oskb_VisFile* file, int block_index,
        int start_time_index, int start_channel_index, int num_times,
        int num_channels, const void* cross_correlations,
        const void* auto_correlations, const void* station_u,
        const void* station_v, const void* station_w);
OSKB_API int oskb_vis_file_close(oskb_VisFile* file);

#ifdef __cplusplus
}
#endif

#endif /* OSKAR_B200_H_ */

/*
 * CPU oracle for the visibility hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is a plain-C restatement of the
 * reference's CPU kernels for the station-beam DFT, the Jones K / join steps
 * and the cross-correlation. It is the checker for the CUDA library, never a
 * product code path: only tests/, __graft_entry__.smoke() and the CPU-baseline
 * leg of bench.py may load it.
 *
 * Parity is pinned: tests/test_oracle_pin.py compares every function here
 * against the reference's own CPU kernels compiled from their sources
 * (oracle/Makefile target "ref", output in oracle/_ref/), and
 * tests/test_golden.py checks it against fixtures generated from those
 * kernels (tests/golden/make_golden.py).
 *
 * Array layouts follow the reference:
 *   - a complex 2x2 matrix is 8 reals {a.re, a.im, b.re, b.im, c.re, c.im,
 *     d.re, d.im} (utility/oskar_vector_types.h:85-98);
 *   - Jones arrays are [station][source] (interferometer/private_jones.h:34-41);
 *   - the baseline index of stations (q < p) is
 *     q*(N-1) - (q-1)*q/2 + p - q - 1 (correlate/define_correlate_utils.h:42).
 */
#ifndef OSKAR_ORACLE_H_
#define OSKAR_ORACLE_H_

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_DECLARE(REAL, S) \
void orc_xcorr_matrix_##S(int casa, int gaussian, int num_src, int num_st, \
        int offset_out, const REAL* jones, const REAL* I, const REAL* Q, \
        const REAL* U, const REAL* V, const REAL* l, const REAL* m, \
        const REAL* n, const REAL* a, const REAL* b, const REAL* c, \
        const REAL* st_u, const REAL* st_v, const REAL* st_w, \
        const REAL* st_x, const REAL* st_y, REAL uv_min_lambda, \
        REAL uv_max_lambda, REAL inv_wavelength, REAL frac_bandwidth, \
        REAL time_int_sec, REAL gha0_rad, REAL dec0_rad, REAL* vis); \
void orc_xcorr_scalar_##S(int casa, int gaussian, int num_src, int num_st, \
        int offset_out, const REAL* jones, const REAL* I, const REAL* Q, \
        const REAL* U, const REAL* V, const REAL* l, const REAL* m, \
        const REAL* n, const REAL* a, const REAL* b, const REAL* c, \
        const REAL* st_u, const REAL* st_v, const REAL* st_w, \
        const REAL* st_x, const REAL* st_y, REAL uv_min_lambda, \
        REAL uv_max_lambda, REAL inv_wavelength, REAL frac_bandwidth, \
        REAL time_int_sec, REAL gha0_rad, REAL dec0_rad, REAL* vis); \
void orc_acorr_matrix_##S(int num_src, int num_st, int offset_out, \
        const REAL* jones, const REAL* I, const REAL* Q, const REAL* U, \
        const REAL* V, REAL* vis); \
void orc_acorr_scalar_##S(int num_src, int num_st, int offset_out, \
        const REAL* jones, const REAL* I, REAL* vis); \
void orc_jones_k_##S(int num_src, const REAL* l, const REAL* m, \
        const REAL* n, int num_st, const REAL* u, const REAL* v, \
        const REAL* w, REAL wavenumber, const REAL* filter, \
        REAL filter_min, REAL filter_max, int ignore_w, REAL* jones); \
void orc_mem_mul_cc_c_##S(int n, const REAL* a, const REAL* b, REAL* c); \
void orc_mem_mul_cc_m_##S(int n, const REAL* a, const REAL* b, REAL* c); \
void orc_mem_mul_cm_m_##S(int n, const REAL* a, const REAL* b, REAL* c); \
void orc_mem_mul_mc_m_##S(int n, const REAL* a, const REAL* b, REAL* c); \
void orc_mem_mul_mm_m_##S(int n, const REAL* a, const REAL* b, REAL* c); \
void orc_dftw_##S(int matrix, int is_3d, int num_in, REAL wavenumber, \
        const REAL* weights_in, const REAL* x_in, const REAL* y_in, \
        const REAL* z_in, int offset_coord_out, int num_out, \
        const REAL* x_out, const REAL* y_out, const REAL* z_out, \
        const int* data_idx, const REAL* data, int eval_x, int eval_y, \
        int offset_out, REAL* output, REAL norm_factor); \
void orc_element_weights_dft_##S(int n, const REAL* x, const REAL* y, \
        const REAL* z, const REAL* cable_length_error, REAL wavenumber, \
        REAL x1, REAL y1, REAL z1, REAL* weights); \
void orc_ecef_to_station_uvw_##S(int n, const REAL* x, const REAL* y, \
        const REAL* z, REAL sin_ha0, REAL cos_ha0, REAL sin_dec0, \
        REAL cos_dec0, int ignore_w, int offset_out, REAL* u, REAL* v, \
        REAL* w); \
void orc_enu_to_theta_phi_##S(int off_in, int num, const REAL* x, \
        const REAL* y, const REAL* z, int extra_point_at_pole, REAL dphi1, \
        REAL dphi2, REAL* theta, REAL* phi1, REAL* phi2); \
void orc_dipole_pattern_##S(int n, const REAL* theta, const REAL* phi_x, \
        const REAL* phi_y, REAL kL, REAL cos_kL, int swap_xy, \
        int offset_out, REAL* pattern); \
void orc_mem_normalise_matrix_##S(int offset, int n, REAL* a, int idx); \
void orc_blank_below_horizon_##S(int off_mask, int n, const REAL* mask, \
        int off_out, REAL* jones); \
void orc_jones_r_##S(int num_sources, const REAL* ra, const REAL* dec, \
        REAL cos_lat, REAL sin_lat, REAL lst_rad, int offset_out, \
        REAL* jones); \
void orc_station_beam_aa_types_##S(int num_el, int num_feeds, \
        const REAL* x, \
        const REAL* y, const REAL* z, const REAL* x_meas, \
        const REAL* y_meas, const REAL* z_meas, const REAL* cable, \
        const REAL* weight_factors, int num_types, const int* element_type, \
        const double* dipole_length_per_type, const int* kind_per_type, \
        const int* taper_per_type, const double* taper_param_per_type, \
        const double* orientation_x_per_type, \
        const double* orientation_y_per_type, int norm_element, \
        int norm_array, int norm_final, int swap_xy, int scalar, int is_3d, \
        double frequency_hz, double bx, double by, double bz, double nx, \
        double ny, double nz, int num_dir, const REAL* dx, const REAL* dy, \
        const REAL* dz, REAL* beam); \
void orc_station_beam_aa_weighted_##S(int num_el, const REAL* x, \
        const REAL* y, const REAL* z, const REAL* x_meas, \
        const REAL* y_meas, const REAL* z_meas, const REAL* cable, \
        const REAL* weight_factors, double orientation_x_rad, \
        double orientation_y_rad, double dipole_length_m, int norm_element, \
        int norm_array, int norm_final, int swap_xy, int is_3d, \
        double frequency_hz, double bx, double by, double bz, double nx, \
        double ny, double nz, int num_dir, const REAL* dx, const REAL* dy, \
        const REAL* dz, REAL* beam); \
void orc_station_beam_aa_##S(int num_el, const REAL* x, const REAL* y, \
        const REAL* z, const REAL* x_meas, const REAL* y_meas, \
        const REAL* z_meas, const REAL* cable, double orientation_x_rad, \
        double orientation_y_rad, double dipole_length_m, int norm_element, \
        int norm_array, int norm_final, int swap_xy, int is_3d, \
        double frequency_hz, double bx, double by, double bz, double nx, \
        double ny, double nz, int num_dir, const REAL* dx, const REAL* dy, \
        const REAL* dz, REAL* beam); \
void orc_sky_scale_flux_##S(int num_sources, int capacity, \
        int num_columns, REAL freq_hz, const REAL* table, \
        const int* num_valid, int col_i, int col_q, int col_u, int col_v, \
        int col_ref_freq, int col_lin_sp_index, int col_sp_index, \
        int col_rot_meas, int col_pol_frac, int col_pol_ang, \
        int col_ref_wavelength, int col_sp_curvature, int col_line_width, \
        int col_freq_inc, REAL* out_i, REAL* out_q, REAL* out_u, \
        REAL* out_v); \
void orc_cable_length_errors_##S(int matrix, int num_sources, \
        int num_stations, REAL wavenumber, const REAL* errors_x, \
        const REAL* errors_y, REAL* jones); \
void orc_station_gains_##S(int matrix, int num_sources, int num_stations, \
        const REAL* gains, REAL* jones); \
void orc_auto_power_##S(int matrix, int n, int offset_in, \
        const REAL* jones, REAL I, REAL Q, REAL U, REAL V, int offset_out, \
        REAL* out); \
void orc_cross_power_##S(int matrix, int num_sources, int num_stations, \
        const REAL* jones, REAL I, REAL Q, REAL U, REAL V, REAL norm, \
        int offset_out, REAL* out); \
void orc_random_gaussian_##S(unsigned int n, REAL* data, unsigned int seed, \
        unsigned int c1, unsigned int c2, unsigned int c3, REAL std); \
void orc_element_weights_errors_##S(int n, const REAL* gain, \
        const REAL* gain_error, const REAL* phase, const REAL* phase_error, \
        unsigned int seed, int time_index, int station_id, REAL* errors);

ORC_DECLARE(double, d)
ORC_DECLARE(float, f)

#undef ORC_DECLARE

#ifdef __cplusplus
}
#endif

#endif

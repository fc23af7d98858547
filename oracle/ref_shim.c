/*
 * Instantiates the reference's own CPU kernels (their macro bodies, included
 * from the reference source tree) under exported names, so that tests can
 * run them next to the oracle. Built by `make -C oracle ref` into
 * oracle/_ref/liboskar_ref.so; nothing in the product links it.
 * The cross-correlation CPU kernels come from the reference's
 * correlate/src/oskar_cross_correlate{,_scalar}_omp.cpp, compiled as they are.
 */
#include <stddef.h>
#include "oskar_global.h"
#include "utility/oskar_kernel_macros.h"
#include "utility/oskar_vector_types.h"
#include "math/define_multiply.h"
#include "correlate/define_correlate_utils.h"
#include "correlate/define_auto_correlate.h"
#include "interferometer/define_evaluate_jones_K.h"
#include "mem/define_mem_multiply.h"
#include "math/define_dftw_c2c.h"
#include "math/define_dftw_m2m.h"
#include "telescope/station/define_evaluate_element_weights_dft.h"
#include "convert/define_convert_ecef_to_station_uvw.h"
#include "convert/define_convert_enu_directions_to_theta_phi.h"
#include "telescope/station/element/define_evaluate_dipole_pattern.h"
#include "telescope/station/define_blank_below_horizon.h"
#include "mem/define_mem_normalise.h"
#include "interferometer/define_evaluate_jones_R.h"
#include "convert/define_convert_lon_lat_to_relative_directions.h"
#include "convert/define_convert_apparent_ra_dec_to_enu_directions.h"
#include "sky/define_update_horizon_mask.h"
#include "correlate/define_evaluate_auto_power.h"
#include "correlate/define_evaluate_cross_power.h"

#define INST(REAL, S, REAL2, REAL4c) \
OSKAR_ACORR_CPU(k_acorr_##S, REAL, REAL2, REAL4c) \
OSKAR_ACORR_SCALAR_CPU(k_acorr_scalar_##S, REAL, REAL2) \
OSKAR_JONES_K_CPU(k_jones_k_##S, REAL, REAL2) \
OSKAR_MEM_MUL_CC_C(k_mul_cc_c_##S, REAL2) \
OSKAR_MEM_MUL_CC_M(k_mul_cc_m_##S, REAL, REAL2, REAL4c) \
OSKAR_MEM_MUL_CM_M(k_mul_cm_m_##S, REAL2, REAL4c) \
OSKAR_MEM_MUL_MC_M(k_mul_mc_m_##S, REAL2, REAL4c) \
OSKAR_MEM_MUL_MM_M(k_mul_mm_m_##S, REAL2, REAL4c) \
OSKAR_DFTW_C2C_CPU(k_dftw_c2c_2d_##S, 0, REAL, REAL2) \
OSKAR_DFTW_C2C_CPU(k_dftw_c2c_3d_##S, 1, REAL, REAL2) \
OSKAR_DFTW_M2M_CPU(k_dftw_m2m_2d_##S, 0, REAL, REAL2) \
OSKAR_DFTW_M2M_CPU(k_dftw_m2m_3d_##S, 1, REAL, REAL2) \
OSKAR_ELEMENT_WEIGHTS_DFT(k_weights_##S, REAL, REAL2) \
OSKAR_CONVERT_ECEF_TO_STATION_UVW(k_uvw_##S, REAL) \
void ref_acorr_matrix_##S(int ns, int nst, int off, const REAL4c* j, \
        const REAL* sI, const REAL* sQ, const REAL* sU, const REAL* sV, \
        REAL4c* vis) \
{ k_acorr_##S(ns, nst, off, sI, sQ, sU, sV, j, vis); } \
void ref_acorr_scalar_##S(int ns, int nst, int off, const REAL2* j, \
        const REAL* sI, REAL2* vis) \
{ k_acorr_scalar_##S(ns, nst, off, sI, sI, sI, sI, j, vis); } \
void ref_jones_k_##S(int ns, const REAL* l, const REAL* m, const REAL* n, \
        int nst, const REAL* u, const REAL* v, const REAL* w, REAL k, \
        const REAL* f, REAL fmin, REAL fmax, int ignore_w, REAL2* out) \
{ k_jones_k_##S(ns, l, m, n, nst, u, v, w, k, f, fmin, fmax, ignore_w, out); } \
void ref_mem_mul_cc_c_##S(int n, const REAL2* a, const REAL2* b, REAL2* c) \
{ k_mul_cc_c_##S(0, 0, 0, (unsigned) n, a, b, c); } \
void ref_mem_mul_cc_m_##S(int n, const REAL2* a, const REAL2* b, REAL4c* c) \
{ k_mul_cc_m_##S(0, 0, 0, (unsigned) n, a, b, c); } \
void ref_mem_mul_cm_m_##S(int n, const REAL2* a, const REAL4c* b, REAL4c* c) \
{ k_mul_cm_m_##S(0, 0, 0, (unsigned) n, a, b, c); } \
void ref_mem_mul_mc_m_##S(int n, const REAL4c* a, const REAL2* b, REAL4c* c) \
{ k_mul_mc_m_##S(0, 0, 0, (unsigned) n, a, b, c); } \
void ref_mem_mul_mm_m_##S(int n, const REAL4c* a, const REAL4c* b, REAL4c* c) \
{ k_mul_mm_m_##S(0, 0, 0, (unsigned) n, a, b, c); } \
void ref_dftw_##S(int matrix, int is_3d, int num_in, REAL k, \
        const REAL2* w, const REAL* xi, const REAL* yi, const REAL* zi, \
        int off_coord, int num_out, const REAL* xo, const REAL* yo, \
        const REAL* zo, const int* idx, const REAL2* data, int ex, int ey, \
        int off_out, REAL2* out, REAL norm) \
{ \
    if (!matrix && !is_3d) k_dftw_c2c_2d_##S(num_in, k, w, xi, yi, zi, \
            off_coord, num_out, xo, yo, zo, idx, data, ex, ey, off_out, out, \
            norm, 0); \
    else if (!matrix) k_dftw_c2c_3d_##S(num_in, k, w, xi, yi, zi, \
            off_coord, num_out, xo, yo, zo, idx, data, ex, ey, off_out, out, \
            norm, 0); \
    else if (!is_3d) k_dftw_m2m_2d_##S(num_in, k, w, xi, yi, zi, \
            off_coord, num_out, xo, yo, zo, idx, data, ex, ey, off_out, out, \
            norm, 0); \
    else k_dftw_m2m_3d_##S(num_in, k, w, xi, yi, zi, \
            off_coord, num_out, xo, yo, zo, idx, data, ex, ey, off_out, out, \
            norm, 0); \
} \
void ref_element_weights_dft_##S(int n, const REAL* x, const REAL* y, \
        const REAL* z, const REAL* cable, REAL k, REAL x1, REAL y1, REAL z1, \
        REAL2* w) \
{ k_weights_##S(n, x, y, z, cable, k, x1, y1, z1, w); } \
void ref_ecef_to_station_uvw_##S(int n, const REAL* x, const REAL* y, \
        const REAL* z, REAL sh, REAL ch, REAL sd, REAL cd, int ignore_w, \
        int off, REAL* u, REAL* v, REAL* w) \
{ k_uvw_##S(n, x, y, z, sh, ch, sd, cd, ignore_w, off, u, v, w); }

INST(double, d, double2, double4c)
INST(float, f, float2, float4c)

/* Station-beam pieces: element coordinates, dipole pattern, normalisation,
 * horizon blanking and the parallactic-angle rotation R. */
#define INST_BEAM(REAL, S, REAL2, REAL4c) \
OSKAR_CONVERT_ENU_DIR_TO_THETA_PHI(k_theta_phi_##S, REAL) \
OSKAR_EVALUATE_DIPOLE_PATTERN(k_dipole_##S, REAL, REAL2, REAL4c) \
OSKAR_BLANK_BELOW_HORIZON_MATRIX(k_blank_##S, REAL, REAL4c) \
OSKAR_MEM_NORMALISE_MATRIX_CPU(k_normalise_##S, REAL, REAL4c) \
OSKAR_JONES_R(k_jones_r_##S, REAL, REAL4c) \
void ref_enu_to_theta_phi_##S(int off_in, int num, const REAL* x, \
        const REAL* y, const REAL* z, int extra_point_at_pole, REAL dphi1, \
        REAL dphi2, REAL* theta, REAL* phi1, REAL* phi2) \
{ k_theta_phi_##S(off_in, num, x, y, z, extra_point_at_pole, dphi1, dphi2, \
        theta, phi1, phi2); } \
void ref_dipole_pattern_##S(int n, const REAL* theta, const REAL* phi_x, \
        const REAL* phi_y, REAL kL, REAL cos_kL, int swap_xy, \
        int offset_out, REAL4c* pattern) \
{ k_dipole_##S(n, theta, phi_x, phi_y, kL, cos_kL, swap_xy, offset_out, \
        pattern); } \
void ref_blank_below_horizon_##S(int off_mask, int n, const REAL* mask, \
        int off_out, REAL4c* jones) \
{ k_blank_##S(off_mask, n, mask, off_out, jones); } \
void ref_mem_normalise_matrix_##S(int offset, int n, REAL4c* a, int idx) \
{ k_normalise_##S((unsigned) offset, (unsigned) n, a, (unsigned) idx); } \
void ref_jones_r_##S(int num_sources, const REAL* ra, const REAL* dec, \
        REAL cos_lat, REAL sin_lat, REAL lst_rad, int offset_out, \
        REAL4c* jones) \
{ k_jones_r_##S(num_sources, ra, dec, cos_lat, sin_lat, lst_rad, \
        offset_out, jones); }

INST_BEAM(double, d, double2, double4c)
INST_BEAM(float, f, float2, float4c)

/* Direction conversions and the horizon mask. */
#define INST_DIR(REAL, S) \
OSKAR_CONVERT_LON_LAT_TO_REL_DIR(k_lonlat_3d_##S, 1, REAL) \
OSKAR_CONVERT_LON_LAT_TO_REL_DIR(k_lonlat_2d_##S, 0, REAL) \
OSKAR_CONVERT_RA_DEC_TO_ENU_DIR(k_radec_enu_##S, REAL) \
OSKAR_UPDATE_HORIZON_MASK(k_horizon_##S, REAL) \
void ref_lon_lat_to_relative_directions_##S(int num, const REAL* lon, \
        const REAL* lat, REAL lon0, REAL cos_lat0, REAL sin_lat0, REAL* l, \
        REAL* m, REAL* n) \
{ \
    if (n) k_lonlat_3d_##S(num, lon, lat, lon0, cos_lat0, sin_lat0, l, m, \
            n); \
    else k_lonlat_2d_##S(num, lon, lat, lon0, cos_lat0, sin_lat0, l, m, n); \
} \
void ref_ra_dec_to_enu_directions_##S(int num, const REAL* ra, \
        const REAL* dec, REAL lst, REAL sin_lat, REAL cos_lat, \
        int offset_out, REAL* x, REAL* y, REAL* z) \
{ k_radec_enu_##S(num, ra, dec, lst, sin_lat, cos_lat, offset_out, x, y, \
        z); } \
void ref_update_horizon_mask_##S(int num, const REAL* l, const REAL* m, \
        const REAL* n, REAL l_mul, REAL m_mul, REAL n_mul, int* mask) \
{ k_horizon_##S(num, l, m, n, l_mul, m_mul, n_mul, mask); }

INST_DIR(double, d)
INST_DIR(float, f)

/* Sky flux scaling with frequency; station cable-length phases and station
 * gains applied to Jones arrays. The flux kernel's calc_stokes_i_flux_<FP>
 * helpers must carry these exact names (the kernel body refers to them).
 * The ref_ wrapper takes the oracle's extra num_columns argument and
 * ignores it. */
#include "sky/oskar_sky_enum.h"
#include "sky/define_sky_scale_flux_with_frequency.h"
#include "interferometer/define_jones_apply_cable_length_errors.h"
#include "interferometer/define_jones_apply_station_gains.h"

OSKAR_SKY_CALC_STOKES_I_FLUX(calc_stokes_i_flux_float, float)
OSKAR_SKY_CALC_STOKES_I_FLUX(calc_stokes_i_flux_double, double)

#define INST_SKY(REAL, S, REAL2, REAL4c) \
OSKAR_SKY_SCALE_FLUX_WITH_FREQUENCY(k_scale_flux_##S, REAL) \
OSKAR_JONES_APPLY_CABLE_LENGTH_ERRORS_M(k_cable_m_##S, REAL, REAL4c) \
OSKAR_JONES_APPLY_CABLE_LENGTH_ERRORS_C(k_cable_c_##S, REAL, REAL2) \
OSKAR_JONES_APPLY_STATION_GAINS_M(k_gains_m_##S, REAL4c) \
OSKAR_JONES_APPLY_STATION_GAINS_C(k_gains_c_##S, REAL2) \
void ref_sky_scale_flux_##S(int num_sources, int capacity, int num_columns, \
        REAL freq_hz, const REAL* table, const int* num_valid, int col_i, \
        int col_q, int col_u, int col_v, int col_ref_freq, \
        int col_lin_sp_index, int col_sp_index, int col_rot_meas, \
        int col_pol_frac, int col_pol_ang, int col_ref_wavelength, \
        int col_sp_curvature, int col_line_width, int col_freq_inc, \
        REAL* out_i, REAL* out_q, REAL* out_u, REAL* out_v) \
{ \
    (void) num_columns; \
    k_scale_flux_##S(num_sources, capacity, freq_hz, table, num_valid, \
            col_i, col_q, col_u, col_v, col_ref_freq, col_lin_sp_index, \
            col_sp_index, col_rot_meas, col_pol_frac, col_pol_ang, \
            col_ref_wavelength, col_sp_curvature, col_line_width, \
            col_freq_inc, out_i, out_q, out_u, out_v); \
} \
void ref_cable_length_errors_##S(int matrix, int num_sources, \
        int num_stations, REAL wavenumber, const REAL* errors_x, \
        const REAL* errors_y, void* jones) \
{ \
    if (matrix) k_cable_m_##S(num_sources, num_stations, wavenumber, \
            errors_x != 0, errors_y != 0, errors_x, errors_y, \
            (REAL4c*) jones); \
    else k_cable_c_##S(num_sources, num_stations, wavenumber, \
            errors_x != 0, errors_y != 0, errors_x, errors_y, \
            (REAL2*) jones); \
} \
void ref_station_gains_##S(int matrix, int num_sources, int num_stations, \
        const void* gains, void* jones) \
{ \
    if (matrix) k_gains_m_##S(num_sources, num_stations, \
            (const REAL4c*) gains, (REAL4c*) jones); \
    else k_gains_c_##S(num_sources, num_stations, (const REAL2*) gains, \
            (REAL2*) jones); \
}

INST_SKY(double, d, double2, double4c)
INST_SKY(float, f, float2, float4c)

/* Beam-pattern auto and cross power (correlate/define_evaluate_auto_power.h,
 * define_evaluate_cross_power.h), CPU forms. */
#define INST_POWER(REAL, S, REAL2, REAL4c) \
OSKAR_AUTO_POWER_MATRIX(k_auto_power_m_##S, REAL, REAL2, REAL4c) \
OSKAR_AUTO_POWER_SCALAR(k_auto_power_s_##S, REAL, REAL2) \
OSKAR_CROSS_POWER_MATRIX(k_cross_power_m_##S, REAL, REAL2, REAL4c) \
OSKAR_CROSS_POWER_SCALAR(k_cross_power_s_##S, REAL, REAL2) \
void ref_auto_power_##S(int matrix, int n, int offset_in, const void* jones, \
        REAL sI, REAL sQ, REAL sU, REAL sV, int offset_out, void* out) \
{ \
    if (matrix) k_auto_power_m_##S(n, offset_in, (const REAL4c*) jones, \
            sI, sQ, sU, sV, offset_out, (REAL4c*) out); \
    else k_auto_power_s_##S(n, offset_in, (const REAL2*) jones, sI, sQ, sU, sV, \
            offset_out, (REAL2*) out); \
} \
void ref_cross_power_##S(int matrix, int ns, int nst, const void* jones, \
        REAL sI, REAL sQ, REAL sU, REAL sV, REAL norm, int offset_out, \
        void* out) \
{ \
    if (matrix) k_cross_power_m_##S(ns, nst, (const REAL4c*) jones, sI, sQ, \
            sU, sV, norm, offset_out, (REAL4c*) out); \
    else k_cross_power_s_##S(ns, nst, (const REAL2*) jones, sI, sQ, sU, \
            sV, norm, offset_out, (REAL2*) out); \
}
INST_POWER(double, d, double2, double4c)
INST_POWER(float, f, float2, float4c)

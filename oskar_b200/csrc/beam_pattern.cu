// Pieces of the beam-pattern application (oskar/beam_pattern/) that run
// under its station beams: the beam-image pixel grid and the rotation of
// relative direction cosines about a sky position into a station's ENU
// frame at an hour angle. The driver that loops over times, channels and
// pixel chunks, forms station beams, auto and cross power and writes images
// is oskar_b200/beam_pattern.py; the station beams and power terms are the
// library's fused kernels (beam.cu, beam_power.cu).
#include <math.h>

#include "common.cuh"

namespace oskb {
namespace {

// (l, m, n) about (ra0, dec0) -> ENU direction cosines at hour angle
// ha0 = lst - ra0 and latitude lat; the rotation of
// oskar/convert/define_convert_relative_directions_to_enu_directions.h
// (the same products in the same order).
template <typename T>
__global__ void rel_to_enu_kernel(int num, const T* __restrict__ l,
        const T* __restrict__ m, const T* __restrict__ n, T sin_ha0,
        T cos_ha0, T sin_dec0, T cos_dec0, T sin_lat, T cos_lat,
        T* __restrict__ x, T* __restrict__ y, T* __restrict__ z)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < num;
            i += gridDim.x * blockDim.x)
    {
        const T l_ = l[i], m_ = m[i], n_ = n[i];
        x[i] = l_ * cos_ha0 + m_ * sin_ha0 * sin_dec0 -
                n_ * sin_ha0 * cos_dec0;
        T t = sin_lat * cos_ha0;
        y[i] = -l_ * sin_lat * sin_ha0 +
                m_ * (cos_lat * cos_dec0 + t * sin_dec0) +
                n_ * (cos_lat * sin_dec0 - t * cos_dec0);
        t = cos_lat * cos_ha0;
        z[i] = l_ * cos_lat * sin_ha0 +
                m_ * (sin_lat * cos_dec0 - t * sin_dec0) +
                n_ * (sin_lat * sin_dec0 + t * cos_dec0);
    }
}

template <typename T>
int rel_to_enu(int num, const T* l, const T* m, const T* n, double ha0,
        double dec0, double lat, T* x, T* y, T* z, void* stream)
{
    if (num < 0) return OSKB_ERR_INVALID_ARGUMENT;
    if (num == 0) return 0;
    if (!l || !m || !n || !x || !y || !z) return OSKB_ERR_INVALID_ARGUMENT;
    // the reference forms the sines and cosines in FP64 and rounds them to
    // the working precision
    const int grid = (num + 255) / 256 < 65535 ? (num + 255) / 256 : 65535;
    rel_to_enu_kernel<T><<<grid, 256, 0, as_stream(stream)>>>(num, l, m, n,
            (T) sin(ha0), (T) cos(ha0), (T) sin(dec0), (T) cos(dec0),
            (T) sin(lat), (T) cos(lat), x, y, z);
    return check_launch("convert_relative_directions_to_enu_directions");
}

// Evenly spaced values from a to b inclusive (the reference's
// oskar_linspace_d, oskar/math/src/oskar_linspace.c:12-26: a + i (b - a) /
// (n - 1), the midpoint alone for n = 1).
void linspace(double* v, double a, double b, int n)
{
    if (n <= 0) return;
    if (n == 1)
    {
        v[0] = (a + b) / 2;
        return;
    }
    const double inc = (b - a) / (n - 1);
    for (int i = 0; i < n; ++i) v[i] = a + i * inc;
}

}  // namespace
}  // namespace oskb

extern "C" {

int oskb_convert_relative_directions_to_enu_directions_d(int num,
        const double* l, const double* m, const double* n, double ha0_rad,
        double dec0_rad, double lat_rad, double* x, double* y, double* z,
        void* stream)
{
    return oskb::rel_to_enu<double>(num, l, m, n, ha0_rad, dec0_rad, lat_rad,
            x, y, z, stream);
}

int oskb_convert_relative_directions_to_enu_directions_f(int num,
        const float* l, const float* m, const float* n, double ha0_rad,
        double dec0_rad, double lat_rad, float* x, float* y, float* z,
        void* stream)
{
    return oskb::rel_to_enu<float>(num, l, m, n, ha0_rad, dec0_rad, lat_rad,
            x, y, z, stream);
}

int oskb_evaluate_image_lmn_grid(int num_l, int num_m, double fov_lon_rad,
        double fov_lat_rad, int centred, double* l, double* m, double* n)
{
    if (num_l < 1 || num_m < 1 || !l || !m || !n)
        return OSKB_ERR_INVALID_ARGUMENT;
    const double nan = NAN;
    if (centred)
    {
        // FITS convention: l increases to the left
        const double l_max = -sin(0.5 * fov_lon_rad);
        const double m_max = sin(0.5 * fov_lat_rad);
        double* lv = new double[num_l];
        double* mv = new double[num_m];
        oskb::linspace(lv, -l_max, l_max, num_l);
        oskb::linspace(mv, -m_max, m_max, num_m);
        for (int j = 0, p = 0; j < num_m; ++j)
            for (int i = 0; i < num_l; ++i, ++p)
            {
                const double r = sqrt(lv[i] * lv[i] + mv[j] * mv[j]);
                if (r > 1.0)
                {
                    l[p] = m[p] = n[p] = nan;
                }
                else
                {
                    l[p] = lv[i];
                    m[p] = mv[j];
                    n[p] = sqrt(1.0 - l[p] * l[p] - m[p] * m[p]);
                }
            }
        delete[] lv;
        delete[] mv;
    }
    else
    {
        // cell size from the field of view: asin(2 sin(fov / 2) / n)
        const double dl = sin(asin(2.0 * sin(0.5 * fov_lon_rad) / num_l));
        const double dm = sin(asin(2.0 * sin(0.5 * fov_lat_rad) / num_m));
        for (int j = 0, p = 0; j < num_m; ++j)
        {
            const double mm = (-(num_m / 2) + j) * dm;
            for (int i = 0; i < num_l; ++i, ++p)
            {
                const double ll = ((num_l / 2) - i) * dl;
                const double r = sqrt(ll * ll + mm * mm);
                if (r > 1.0)
                {
                    l[p] = m[p] = n[p] = nan;
                }
                else
                {
                    l[p] = ll;
                    m[p] = mm;
                    n[p] = sqrt(1.0 - ll * ll - mm * mm);
                }
            }
        }
    }
    return 0;
}

}  // extern "C"

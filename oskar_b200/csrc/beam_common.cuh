// Element-pattern device functions shared by the exact station beam
// (beam.cu) and the learned-surrogate beam (surrogate.cu).
#pragma once

#include "common.cuh"

namespace oskb {

// Dipole far field along phi for a direction with (sin, cos) theta
// (oskar/telescope/station/element/define_evaluate_dipole_pattern.h:3-15).
template <typename T>
__device__ __forceinline__ void dipole(T kL, T cos_kL, T sin_th, T cos_th,
        T phi, T& e_theta, T& e_phi)
{
    T sp, cp;
    sincos(phi, &sp, &cp);
    const T denom = (T) 1 + cp * cp * (cos_th * cos_th - (T) 1);
    if (denom == (T) 0)
    {
        e_theta = e_phi = (T) 0;
        return;
    }
    const T t = (cos(kL * cp * sin_th) - cos_kL) / denom;
    e_theta = -cp * cos_th * t;
    e_phi = sp * t;
}

// Real element-pattern matrix {a, b, c, d} for one direction
// (define_convert_enu_directions_to_theta_phi.h:3-31 then
// define_evaluate_dipole_pattern.h:17-48). pole: the extra point at theta = 0
// whose phi values are the unwrapped offsets.
template <typename T>
__device__ __forceinline__ void element_pattern(T X, T Y, T Z, bool pole,
        T dphi1, T dphi2, T kL, T cos_kL, int swap_xy, T p[4])
{
    T theta, phi1, phi2;
    if (pole)
    {
        theta = (T) 0;
        phi1 = dphi1;
        phi2 = dphi2;
    }
    else
    {
        const T twopi = (T) 2 * (T) kPi;
        const T p0 = atan2(Y, X);
        phi1 = fmod(p0 + dphi1, twopi);
        phi2 = fmod(p0 + dphi2, twopi);
        if (phi1 < (T) 0) phi1 += twopi;
        if (phi2 < (T) 0) phi2 += twopi;
        theta = atan2(sqrt(X * X + Y * Y), Z);
    }
    T st, ct, xt, xp, yt, yp;
    sincos(theta, &st, &ct);
    dipole(kL, cos_kL, st, ct, phi1, xt, xp);
    dipole(kL, cos_kL, st, ct, phi2, yt, yp);
    p[0] = swap_xy ? yt : xt;
    p[1] = swap_xy ? yp : xp;
    p[2] = swap_xy ? xt : yt;
    p[3] = swap_xy ? xp : yp;
}

}  // namespace oskb

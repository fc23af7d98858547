// Aperture-array station beam (Jones E) for many stations in one launch, and
// the parallactic-angle rotation (Jones R).
//
// Replaces the chain the reference runs per station and per feed
// (oskar/telescope/station/src/oskar_station_beam.c:84-182 and
// oskar_evaluate_station_beam_aperture_array.c:150-240): element pattern
// (dipole, oskar_element_evaluate.c:76-157), element weights
// (define_evaluate_element_weights_dft.h:3-16), weighted DFT
// (define_dftw_m2m.h:24-107), horizon blanking
// (define_blank_below_horizon.h:15-29) and final normalisation
// (define_mem_normalise.h:31-51). The reference runs these as six kernels
// with five round trips through a per-station signal buffer; here one thread
// owns one (station, direction) and the pieces stay in registers.
//
// With a single element type the weighted DFT of the element signals is
// pattern(dir) x AF(dir), AF = sum_e w_e exp(i k r_e . dir): the pattern is
// evaluated once per direction and the element loop carries only the array
// factor (one sincos and one complex multiply-add per element-direction).
// Element weights and positions are staged in shared memory in chunks.
// The normalisation direction's beam (one per station) is recomputed by each
// CTA cooperatively before the main loop, so there is no second launch.
// In FP64 the element loops take their phase factors from a shared-memory
// table (trig_table.cuh) instead of a library sincos per element-direction.
#include <climits>

#include "beam_common.cuh"
#include "trig_table.cuh"

namespace oskb {
namespace {

constexpr int kThreads = 128;
constexpr int kChunk = 512;

struct BeamFlags
{
    int normalise_element, normalise_array, normalise_final, swap_xy;
    int scalar;  // complex beam of the pattern amplitude (Stokes-I mode)
};

// e^{i ph} for the normalisation direction: ph in table steps through
// the shared table in FP64, in radians through sincosf in FP32.
__device__ __forceinline__ void phase_factor(const double2* table, double ph,
        double* s, double* c)
{
    trig_steps_checked(table, ph, s, c);
}
__device__ __forceinline__ void phase_factor(const double2*, float ph,
        float* s, float* c)
{
    sincosf(ph, s, c);
}

template <typename T>
__device__ __forceinline__ T half_frobenius(const T p[4], T ar, T ai)
{
    // |p * af|_F^2 / 2 with p real and af complex.
    const T a2 = ar * ar + ai * ai;
    return (p[0] * p[0] + p[1] * p[1] + p[2] * p[2] + p[3] * p[3]) * a2 /
            (T) 2;
}

// Up to kMaxTypes element types per station (a dipole length each).
constexpr int kMaxTypes = 4;

template <typename T>
struct TypeParams
{
    T kL[kMaxTypes];      // dipole length x pi f / c
    T cos_kL[kMaxTypes];
    int kind[kMaxTypes];  // 0 dipole, 1 isotropic
    int taper[kMaxTypes]; // 0 none, 1 cos(theta)^p, 2 Gaussian in theta
    T taper_param[kMaxTypes];  // p, or 4 ln 2 / FWHM^2
};

// Real pattern {a, b, c, d} of element type t in direction (X, Y, Z): the
// dipole's, or the identity for an isotropic element
// (oskar_element_evaluate.c:82-87).
template <typename T>
__device__ __forceinline__ void type_pattern(const TypeParams<T>& tp, int t,
        T X, T Y, T Z, bool pole, T dphi1, T dphi2, int swap_xy, T p[4])
{
    if (tp.kind[t] == 1)
    {
        p[0] = p[3] = (T) 1;
        p[1] = p[2] = (T) 0;
        return;
    }
    element_pattern<T>(X, Y, Z, pole, dphi1, dphi2, tp.kL[t], tp.cos_kL[t],
            swap_xy, p);
}

// Element taper of type t at polar angle theta = atan2(|(X, Y)|, Z),
// applied after the pole normalisation (oskar_element_evaluate.c:159-174;
// define_apply_element_taper_{cosine,gaussian}.h).
template <typename T>
__device__ __forceinline__ T type_taper(const TypeParams<T>& tp, int t, T X,
        T Y, T Z)
{
    if (tp.taper[t] == 0) return (T) 1;
    const T theta = atan2(sqrt(X * X + Y * Y), Z);
    if (tp.taper[t] == 1) return pow(cos(theta), tp.taper_param[t]);
    return exp(-(theta * theta) * tp.taper_param[t]);
}

// (ar, ai)[t] += w e^{i ph} for the element's type t only: register selects
// over a compile-time number of types, so the accumulators stay in
// registers. One type: the plain complex multiply-add.
template <typename T, int NT>
__device__ __forceinline__ void add_term(T* ar, T* ai,
        typename vec2<T>::type w, int type, T sn, T cs)
{
    if constexpr (NT == 1)
    {
        ar[0] += cs * w.x - w.y * sn;
        ai[0] += sn * w.x + w.y * cs;
    }
    else
    {
#pragma unroll
        for (int t = 0; t < NT; ++t)
        {
            const T wx = type == t ? w.x : (T) 0;
            const T wy = type == t ? w.y : (T) 0;
            ar[t] += cs * wx - wy * sn;
            ai[t] += sn * wx + wy * cs;
        }
    }
}

template <typename T, bool IS3D, int NT>
__global__ void __launch_bounds__(kThreads)
station_beam_kernel(int num_elements, const T* __restrict__ el_x,
        const T* __restrict__ el_y, const T* __restrict__ el_z,
        const T* __restrict__ meas_x, const T* __restrict__ meas_y,
        const T* __restrict__ meas_z, const T* __restrict__ cable,
        const T* __restrict__ weight_factors,
        const int* __restrict__ element_type,
        const double* __restrict__ orientation_x,
        const double* __restrict__ orientation_y, TypeParams<T> tp,
        BeamFlags flags, T wavenumber, const double* __restrict__ beam_enu,
        const double* __restrict__ norm_enu, int num_dir,
        const T* __restrict__ dir_x, const T* __restrict__ dir_y,
        const T* __restrict__ dir_z, int directions_per_station, int rows,
        T* __restrict__ norm_af, T* __restrict__ beam)
{
    // rows: 0 all four; 1 the x feed's (xx, xy); 2 the y feed's (yx, yy).
    // With one feed per launch the final normalisation needs both feeds'
    // array factors at the normalisation direction: the launch writes its
    // own to norm_af[station][type] (complex) and leaves the scaling to
    // feeds_finalise_kernel.
    typedef typename vec2<T>::type T2;
    __shared__ T2 s_w[kChunk];
    __shared__ T s_x[kChunk], s_y[kChunk], s_z[IS3D ? kChunk : 1];
    __shared__ int s_type[NT > 1 ? kChunk : 1];
    __shared__ T s_red[2][NT][kThreads / 32];
    // FP64: phase factors of the element loops from the shared table
    __shared__ double2 s_trig[sizeof(T) == 8 ? kTrigTableSize : 1];
    const int st = blockIdx.y;
    const int d = blockIdx.x * kThreads + threadIdx.x;
    const bool active = d < num_dir;
    const size_t el0 = (size_t) st * num_elements;
    const size_t dir0 = directions_per_station ? (size_t) st * num_dir : 0;
    const int per_dir = flags.scalar ? 1 : 4;
    T2* out = reinterpret_cast<T2*>(beam) +
            per_dir * ((size_t) st * num_dir + d);

    const T bx = (T) beam_enu[3 * st], by = (T) beam_enu[3 * st + 1],
            bz = (T) beam_enu[3 * st + 2];
    if (beam_enu[3 * st + 2] < 0.0)  // pointing below the horizon
    {
        if (active)
            for (int k = 0; k < per_dir; ++k) out[k] = T2{(T) 0, (T) 0};
        return;
    }
    if constexpr (sizeof(T) == 8)
    {
        trig_table_fill(s_trig);
        __syncthreads();
    }
    // element orientations per (station, type)
    T dphi1[NT], dphi2[NT];
#pragma unroll
    for (int t = 0; t < NT; ++t)
    {
        dphi1[t] = (T) (kPi / 2 - (orientation_x[st * NT + t] + kPi / 2));
        dphi2[t] = (T) (kPi / 2 - orientation_y[st * NT + t]);
    }

    T X = 0, Y = 0, Z = 0;
    if (active)
    {
        X = dir_x[dir0 + d];
        Y = dir_y[dir0 + d];
        Z = dir_z[dir0 + d];
    }
    T nX = 0, nY = 0, nZ = 1;
    if (flags.normalise_final)
    {
        nX = (T) norm_enu[3 * st];
        nY = (T) norm_enu[3 * st + 1];
        nZ = (T) norm_enu[3 * st + 2];
    }
    // Phase factors per element coordinate: radians in FP32, table steps
    // (radians x 64 / pi) in FP64.
    const T to_steps = sizeof(T) == 8 ? (T) kTrigStepsPerRadian : (T) 1;
    const T kX = wavenumber * X * to_steps, kY = wavenumber * Y * to_steps,
            kZ = wavenumber * Z * to_steps;
    const T knX = wavenumber * nX * to_steps, knY = wavenumber * nY * to_steps,
            knZ = wavenumber * nZ * to_steps;

    // array factors per element type: this thread's direction (ar, ai) and
    // the normalisation direction (nr, ni)
    T ar[NT], ai[NT], nr[NT], ni[NT];
#pragma unroll
    for (int t = 0; t < NT; ++t) ar[t] = ai[t] = nr[t] = ni[t] = (T) 0;
    for (int e0 = 0; e0 < num_elements; e0 += kChunk)
    {
        const int ne = min(kChunk, num_elements - e0);
        for (int t = threadIdx.x; t < ne; t += kThreads)
        {
            const size_t g = el0 + e0 + t;
            const T mx = meas_x ? meas_x[g] : el_x[g];
            const T my = meas_y ? meas_y[g] : el_y[g];
            const T mz = meas_z ? meas_z[g] : (el_z ? el_z[g] : (T) 0);
            const T p = wavenumber * (mx * bx + my * by + mz * bz +
                    (cable ? cable[g] : (T) 0));
            T sn, cs;
            sincos(-p, &sn, &cs);
            if (weight_factors)
            {
                // element errors x apodisation, applied to the DFT weight
                const T2 f = reinterpret_cast<const T2*>(weight_factors)[g];
                const T re = cs * f.x - sn * f.y;
                sn = cs * f.y + sn * f.x;
                cs = re;
            }
            s_w[t] = T2{cs, sn};
            int type = 0;
            if constexpr (NT > 1)
            {
                type = element_type ? element_type[g] : 0;
                s_type[t] = type;
            }
            s_x[t] = el_x[g];
            s_y[t] = el_y[g];
            if (IS3D) s_z[t] = el_z[g];
            // The normalisation direction: elements split across threads.
            if (flags.normalise_final)
            {
                T ph = knX * s_x[t] + knY * s_y[t];
                if (IS3D) ph += knZ * s_z[t];
                T s2, c2;
                phase_factor(s_trig, ph, &s2, &c2);
                add_term<T, NT>(nr, ni, T2{cs, sn}, type, s2, c2);
            }
        }
        __syncthreads();
        if (active)
        {
            if constexpr (sizeof(T) == 8)
            {
                // Branch-free table loop; a thread that met a phase the
                // table does not cover redoes the chunk with sincos.
                T ar0[NT], ai0[NT];
#pragma unroll
                for (int t = 0; t < NT; ++t)
                {
                    ar0[t] = ar[t];
                    ai0[t] = ai[t];
                }
                bool covered = true;
#pragma unroll 4
                for (int i = 0; i < ne; ++i)
                {
                    T ph = kX * s_x[i] + kY * s_y[i];
                    if (IS3D) ph += kZ * s_z[i];
                    T sn, cs;
                    trig_steps_sincos(s_trig, ph, &sn, &cs, covered);
                    add_term<T, NT>(ar, ai, s_w[i], NT > 1 ? s_type[i] : 0,
                            sn, cs);
                }
                if (!covered)
                {
#pragma unroll
                    for (int t = 0; t < NT; ++t)
                    {
                        ar[t] = ar0[t];
                        ai[t] = ai0[t];
                    }
                    for (int i = 0; i < ne; ++i)
                    {
                        T ph = kX * s_x[i] + kY * s_y[i];
                        if (IS3D) ph += kZ * s_z[i];
                        T sn, cs;
                        trig_steps_exact(ph, &sn, &cs);
                        add_term<T, NT>(ar, ai, s_w[i],
                                NT > 1 ? s_type[i] : 0, sn, cs);
                    }
                }
            }
            else
            {
#pragma unroll 4
                for (int i = 0; i < ne; ++i)
                {
                    T ph = kX * s_x[i] + kY * s_y[i];
                    if (IS3D) ph += kZ * s_z[i];
                    T sn, cs;
                    sincosf(ph, &sn, &cs);
                    add_term<T, NT>(ar, ai, s_w[i], NT > 1 ? s_type[i] : 0,
                            sn, cs);
                }
            }
        }
        __syncthreads();
    }

    // Element normalisation: 1 / |pattern at the pole|, per type.
    T pole_scale[NT];
#pragma unroll
    for (int t = 0; t < NT; ++t)
    {
        pole_scale[t] = (T) 1;
        if (flags.normalise_element)
        {
            T pp[4];
            type_pattern<T>(tp, t, 0, 0, 1, true, dphi1[t], dphi2[t],
                    flags.swap_xy, pp);
            pole_scale[t] = (T) 1 / sqrt(half_frobenius<T>(pp, 1, 0));
        }
    }
    const T array_scale = flags.normalise_array ?
            (T) (1.0 / num_elements) : (T) 1;

    // Final normalisation: amplitude of the beam in the normalisation
    // direction (block reduction of its array factors first).
    T final_scale = (T) 1;
    if (flags.normalise_final)
    {
#pragma unroll
        for (int t = 0; t < NT; ++t)
        {
            for (int o = 16; o > 0; o >>= 1)
            {
                nr[t] += __shfl_xor_sync(0xffffffffu, nr[t], o);
                ni[t] += __shfl_xor_sync(0xffffffffu, ni[t], o);
            }
            if ((threadIdx.x & 31) == 0)
            {
                s_red[0][t][threadIdx.x >> 5] = nr[t];
                s_red[1][t][threadIdx.x >> 5] = ni[t];
            }
        }
        __syncthreads();
#pragma unroll
        for (int t = 0; t < NT; ++t)
        {
            nr[t] = ni[t] = 0;
            for (int w = 0; w < kThreads / 32; ++w)
            {
                nr[t] += s_red[0][t][w];
                ni[t] += s_red[1][t][w];
            }
            // A normalisation direction below the horizon is blanked, as in
            // the reference, which then divides by zero.
            if (nZ < (T) 0) nr[t] = ni[t] = (T) 0;
        }
        if (rows != 0)
        {
            if (blockIdx.x == 0 && threadIdx.x == 0)
            {
#pragma unroll
                for (int t = 0; t < NT; ++t)
                {
                    norm_af[2 * ((size_t) st * NT + t)] = nr[t];
                    norm_af[2 * ((size_t) st * NT + t) + 1] = ni[t];
                }
            }
        }
        else if (flags.scalar)
        {
            // |sum_t amplitude_t AF_t| (define_mem_normalise.h:13-29)
            T vr = 0, vi = 0;
#pragma unroll
            for (int t = 0; t < NT; ++t)
            {
                T pn[4];
                type_pattern<T>(tp, t, nX, nY, nZ, false, dphi1[t],
                        dphi2[t], flags.swap_xy, pn);
                const T a = sqrt(half_frobenius<T>(pn, 1, 0)) *
                        type_taper<T>(tp, t, nX, nY, nZ) * pole_scale[t] *
                        array_scale;
                vr += a * nr[t];
                vi += a * ni[t];
            }
            final_scale = (T) 1 / sqrt(vr * vr + vi * vi);
        }
        else if constexpr (NT == 1)
        {
            T pn[4];
            type_pattern<T>(tp, 0, nX, nY, nZ, false, dphi1[0], dphi2[0],
                    flags.swap_xy, pn);
            const T taper = type_taper<T>(tp, 0, nX, nY, nZ);
            for (int k = 0; k < 4; ++k)
                pn[k] *= pole_scale[0] * taper * array_scale;
            final_scale = (T) 1 / sqrt(half_frobenius<T>(pn, nr[0], ni[0]));
        }
        else
        {
            // |sum_t pattern_t AF_t|_F^2 / 2 over the four polarisations
            T pn[NT][4];
#pragma unroll
            for (int t = 0; t < NT; ++t)
            {
                type_pattern<T>(tp, t, nX, nY, nZ, false, dphi1[t],
                        dphi2[t], flags.swap_xy, pn[t]);
                const T taper = type_taper<T>(tp, t, nX, nY, nZ);
                for (int k = 0; k < 4; ++k) pn[t][k] *= taper;
            }
            T amp = 0;
            for (int k = 0; k < 4; ++k)
            {
                T vr = 0, vi = 0;
#pragma unroll
                for (int t = 0; t < NT; ++t)
                {
                    const T pk = pn[t][k] * pole_scale[t] * array_scale;
                    vr += pk * nr[t];
                    vi += pk * ni[t];
                }
                amp += vr * vr + vi * vi;
            }
            final_scale = (T) 1 / sqrt(amp / (T) 2);
        }
    }
    if (!active) return;

    const bool blank = Z < (T) 0;
    if (flags.scalar)
    {
        // pattern amplitude sqrt(sum p_k^2 / 2)
        // (define_evaluate_dipole_pattern.h:51-75) times the array factor
        T2 v{(T) 0, (T) 0};
#pragma unroll
        for (int t = 0; t < NT; ++t)
        {
            T pt[4];
            type_pattern<T>(tp, t, X, Y, Z, false, dphi1[t], dphi2[t],
                    flags.swap_xy, pt);
            const T a = sqrt(half_frobenius<T>(pt, 1, 0)) *
                    type_taper<T>(tp, t, X, Y, Z) * pole_scale[t];
            v.x += a * ar[t] * array_scale;
            v.y += a * ai[t] * array_scale;
        }
        if (blank) v = T2{(T) 0, (T) 0};
        out[0] = T2{v.x * final_scale, v.y * final_scale};
        return;
    }
    T p[NT][4];
#pragma unroll
    for (int t = 0; t < NT; ++t)
    {
        type_pattern<T>(tp, t, X, Y, Z, false, dphi1[t], dphi2[t],
                flags.swap_xy, p[t]);
        const T taper = type_taper<T>(tp, t, X, Y, Z);
        for (int k = 0; k < 4; ++k) p[t][k] *= taper;
    }
    for (int k = 0; k < 4; ++k)
    {
        // The reference's order: pattern (normalised), times the weighted
        // element sum, times the DFT norm, then the final scale.
        T2 v{(T) 0, (T) 0};
#pragma unroll
        for (int t = 0; t < NT; ++t)
        {
            const T pk = p[t][k] * pole_scale[t];
            v.x += pk * ar[t] * array_scale;
            v.y += pk * ai[t] * array_scale;
        }
        if (blank) v = T2{(T) 0, (T) 0};
        v.x *= final_scale;
        v.y *= final_scale;
        if (rows == 0 || (rows == 1) == (k < 2)) out[k] = v;
    }
}

// Final normalisation of a station beam evaluated one feed per launch:
// the beam in the normalisation direction takes its (xx, xy) row from the
// x feed's array factors and its (yx, yy) row from the y feed's
// (norm_af[feed][station][type], complex); every direction of the station
// is divided by that matrix's amplitude (define_mem_normalise.h:31-51).
template <typename T, int NT>
__global__ void __launch_bounds__(256)
feeds_finalise_kernel(int num_stations, int num_elements,
        const double* __restrict__ orientation_x,
        const double* __restrict__ orientation_y, TypeParams<T> tp,
        BeamFlags flags, const double* __restrict__ beam_enu,
        const double* __restrict__ norm_enu, int num_dir,
        const T* __restrict__ norm_af, T* __restrict__ beam)
{
    const int st = blockIdx.y;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    // a pointing below the horizon left a zero beam and no array factors
    if (d >= num_dir || beam_enu[3 * st + 2] < 0.0) return;
    const T nX = (T) norm_enu[3 * st], nY = (T) norm_enu[3 * st + 1],
            nZ = (T) norm_enu[3 * st + 2];
    const T array_scale = flags.normalise_array ?
            (T) (1.0 / num_elements) : (T) 1;
    T amp = 0;
    T pn[NT][4], pole[NT];
#pragma unroll
    for (int t = 0; t < NT; ++t)
    {
        const T dphi1 = (T) (kPi / 2 - (orientation_x[st * NT + t] + kPi / 2));
        const T dphi2 = (T) (kPi / 2 - orientation_y[st * NT + t]);
        pole[t] = (T) 1;
        if (flags.normalise_element)
        {
            T pp[4];
            type_pattern<T>(tp, t, 0, 0, 1, true, dphi1, dphi2,
                    flags.swap_xy, pp);
            pole[t] = (T) 1 / sqrt(half_frobenius<T>(pp, 1, 0));
        }
        type_pattern<T>(tp, t, nX, nY, nZ, false, dphi1, dphi2,
                flags.swap_xy, pn[t]);
        const T taper = type_taper<T>(tp, t, nX, nY, nZ);
        for (int k = 0; k < 4; ++k) pn[t][k] *= taper;
    }
    for (int k = 0; k < 4; ++k)
    {
        const T* af = norm_af + 2 * (size_t) NT *
                ((size_t) (k < 2 ? 0 : 1) * num_stations + st);
        T vr = 0, vi = 0;
#pragma unroll
        for (int t = 0; t < NT; ++t)
        {
            const T pk = pn[t][k] * pole[t] * array_scale;
            vr += pk * af[2 * t];
            vi += pk * af[2 * t + 1];
        }
        amp += vr * vr + vi * vi;
    }
    const T scale = (T) 1 / sqrt(amp / (T) 2);
    T* b = beam + 8 * ((size_t) st * num_dir + d);
#pragma unroll
    for (int i = 0; i < 8; ++i) b[i] *= scale;
}

template <typename T>
__global__ void __launch_bounds__(256)
jones_r_kernel(int num_sources, const T* __restrict__ ra,
        const T* __restrict__ dec, const double* __restrict__ lat_rad,
        const double* __restrict__ lst_rad, T* __restrict__ jones)
{
    typedef typename vec2<T>::type T2;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int st = blockIdx.y;
    if (s >= num_sources) return;
    // (define_evaluate_jones_R.h:3-29; per-station latitude and LST as the
    // driver oskar_evaluate_jones_R.c:42-49 derives them in double.)
    const T cos_lat = (T) cos(lat_rad[st]), sin_lat = (T) sin(lat_rad[st]);
    const T lst = (T) lst_rad[st];
    T sh, ch, sd, cd, sq, cq;
    sincos(lst - ra[s], &sh, &ch);
    sincos(dec[s], &sd, &cd);
    const T q = atan2(cos_lat * sh, sin_lat * cd - cos_lat * sd * ch);
    sincos(q, &sq, &cq);
    T2* o = reinterpret_cast<T2*>(jones) + 4 * ((size_t) st * num_sources + s);
    o[0] = T2{cq, (T) 0};
    o[1] = T2{-sq, (T) 0};
    o[2] = T2{sq, (T) 0};
    o[3] = T2{cq, (T) 0};
}

}  // namespace
}  // namespace oskb

namespace oskb {
namespace {

// Per-type parameters from host arrays (NULL kinds: dipoles; NULL tapers:
// none). Returns an OSKAR status.
template <typename T>
int make_type_params(int num_types, const double* dipole_length_m,
        const int* element_kind, const int* taper_kind,
        const double* taper_param, double frequency_hz, TypeParams<T>* tp)
{
    if (num_types < 1 || !dipole_length_m) return OSKB_ERR_INVALID_ARGUMENT;
    if (num_types > kMaxTypes) return OSKB_ERR_OUT_OF_RANGE;
    const double c0 = 299792458.0;
    for (int t = 0; t < kMaxTypes; ++t)
    {
        const bool on = t < num_types;
        const double kL = on ?
                dipole_length_m[t] * (kPi * frequency_hz / c0) : 0.0;
        tp->kL[t] = (T) kL;
        tp->cos_kL[t] = (T) cos(kL);
        tp->kind[t] = on && element_kind ? element_kind[t] : 0;
        tp->taper[t] = on && taper_kind ? taper_kind[t] : 0;
        if (tp->kind[t] < 0 || tp->kind[t] > 1 || tp->taper[t] < 0 ||
                tp->taper[t] > 2 || (tp->taper[t] && !taper_param))
            return OSKB_ERR_INVALID_ARGUMENT;
        double q = 0.0;
        if (tp->taper[t] == 1) q = taper_param[t];
        if (tp->taper[t] == 2)
        {
            const double fwhm = taper_param[t];
            if (!(fwhm > 0.0)) return OSKB_ERR_INVALID_ARGUMENT;
            q = 4.0 * log(2.0) / (fwhm * fwhm);
        }
        tp->taper_param[t] = (T) q;
    }
    return 0;
}

template <typename T>
int station_beam_aa(int num_stations, int num_elements, const T* el_x,
        const T* el_y, const T* el_z, const T* meas_x, const T* meas_y,
        const T* meas_z, const T* cable, const T* weight_factors,
        int num_element_types, const int* element_type,
        const double* orientation_x,
        const double* orientation_y, const double* dipole_length_m,
        const int* element_kind, const int* taper_kind,
        const double* taper_param,
        int normalise_element, int normalise_array, int normalise_final,
        int swap_xy, int is_3d, double frequency_hz, const double* beam_enu,
        const double* norm_enu, int num_directions, const T* x, const T* y,
        const T* z, int directions_per_station, T* beam, void* stream,
        int rows = 0, T* norm_af = nullptr, int scalar = 0)
{
    if (num_stations < 0 || num_elements < 0 || num_directions < 0)
        return OSKB_ERR_INVALID_ARGUMENT;
    if (num_stations == 0 || num_directions == 0) return 0;
    if (num_elements == 0 || !el_x || !el_y || (is_3d && !el_z) ||
            !orientation_x || !orientation_y || !beam_enu ||
            (normalise_final && !norm_enu) || !x || !y || !z || !beam)
        return OSKB_ERR_INVALID_ARGUMENT;
    if (num_stations > 65535) return OSKB_ERR_INVALID_ARGUMENT;
    TypeParams<T> tp;
    if (int err = make_type_params<T>(num_element_types, dipole_length_m,
            element_kind, taper_kind, taper_param, frequency_hz, &tp))
        return err;
    const double c0 = 299792458.0;
    const T wavenumber = (T) (2.0 * kPi * frequency_hz / c0);
    BeamFlags flags{normalise_element, normalise_array, normalise_final,
            swap_xy, scalar};
    dim3 grid((num_directions + kThreads - 1) / kThreads, num_stations);
    cudaStream_t s = as_stream(stream);
#define OSKB_BEAM(D, NT) station_beam_kernel<T, D, NT><<<grid, kThreads, 0,    \
        s>>>(num_elements, el_x, el_y, el_z, meas_x, meas_y, meas_z, cable,  \
        weight_factors, element_type, orientation_x, orientation_y, tp,      \
        flags, wavenumber, beam_enu, norm_enu, num_directions, x, y, z,      \
        directions_per_station, rows, norm_af, beam)
#define OSKB_BEAM_NT(D)                                                      \
    switch (num_element_types)                                               \
    {                                                                        \
    case 1: OSKB_BEAM(D, 1); break;                                          \
    case 2: OSKB_BEAM(D, 2); break;                                          \
    case 3: OSKB_BEAM(D, 3); break;                                          \
    default: OSKB_BEAM(D, 4); break;                                         \
    }
    if (is_3d) { OSKB_BEAM_NT(true) } else { OSKB_BEAM_NT(false) }
#undef OSKB_BEAM_NT
#undef OSKB_BEAM
    return check_launch("station_beam_aa");
}

// Stations whose two feeds have their own element data (the reference's
// num_feeds = 2 when a station is not common_pol_beams,
// oskar_evaluate_station_beam_aperture_array.c:208-223): element arrays
// are [feed][station][element]; one launch per feed writes that feed's
// rows, then the final normalisation combines both feeds.
template <typename T>
int station_beam_aa_feeds(int num_feeds, int num_stations, int num_elements,
        const T* el_x, const T* el_y, const T* el_z, const T* meas_x,
        const T* meas_y, const T* meas_z, const T* cable,
        const T* weight_factors, int num_element_types,
        const int* element_type, const double* orientation_x,
        const double* orientation_y, const double* dipole_length_m,
        const int* element_kind, const int* taper_kind,
        const double* taper_param,
        int normalise_element, int normalise_array, int normalise_final,
        int swap_xy, int is_3d, double frequency_hz, const double* beam_enu,
        const double* norm_enu, int num_directions, const T* x, const T* y,
        const T* z, int directions_per_station, T* beam, void* stream)
{
    if (num_feeds == 1)
        return station_beam_aa<T>(num_stations, num_elements, el_x, el_y,
                el_z, meas_x, meas_y, meas_z, cable, weight_factors,
                num_element_types, element_type, orientation_x,
                orientation_y, dipole_length_m, element_kind, taper_kind,
                taper_param, normalise_element,
                normalise_array, normalise_final, swap_xy, is_3d,
                frequency_hz, beam_enu, norm_enu, num_directions, x, y, z,
                directions_per_station, beam, stream);
    if (num_feeds != 2) return OSKB_ERR_INVALID_ARGUMENT;
    if (num_stations <= 0 || num_directions <= 0)
        return num_stations < 0 || num_directions < 0 ?
                OSKB_ERR_INVALID_ARGUMENT : 0;
    TypeParams<T> tp;
    if (int err = make_type_params<T>(num_element_types, dipole_length_m,
            element_kind, taper_kind, taper_param, frequency_hz, &tp))
        return err;
    cudaStream_t s = as_stream(stream);
    T* norm_af = nullptr;
    const size_t af_count = (size_t) 2 * num_stations * num_element_types * 2;
    if (normalise_final)
    {
        if (scratch_alloc((void**) &norm_af, af_count * sizeof(T), s) !=
                cudaSuccess)
        {
            cudaGetLastError();
            return OSKB_ERR_MEMORY_ALLOC_FAILURE;
        }
    }
    const size_t n = (size_t) num_stations * num_elements;
    int err = 0;
    for (int f = 0; f < 2 && !err; ++f)
    {
        const size_t o = f * n;
        err = station_beam_aa<T>(num_stations, num_elements, el_x + o,
                el_y + o, el_z ? el_z + o : nullptr,
                meas_x ? meas_x + o : nullptr, meas_y ? meas_y + o : nullptr,
                meas_z ? meas_z + o : nullptr, cable ? cable + o : nullptr,
                weight_factors ? weight_factors + 2 * o : nullptr,
                num_element_types, element_type, orientation_x,
                orientation_y, dipole_length_m, element_kind, taper_kind,
                taper_param, normalise_element,
                normalise_array, normalise_final, swap_xy, is_3d,
                frequency_hz, beam_enu, norm_enu, num_directions, x, y, z,
                directions_per_station, beam, stream, 1 + f,
                norm_af ? norm_af + f * (af_count / 2) : nullptr);
    }
    if (!err && normalise_final)
    {
        BeamFlags flags{normalise_element, normalise_array, normalise_final,
                swap_xy, 0};
        dim3 grid((num_directions + 255) / 256, num_stations);
#define OSKB_FIN(NT) feeds_finalise_kernel<T, NT><<<grid, 256, 0, s>>>(       \
        num_stations, num_elements, orientation_x, orientation_y, tp, flags, \
        beam_enu, norm_enu, num_directions, norm_af, beam)
        switch (num_element_types)
        {
        case 1: OSKB_FIN(1); break;
        case 2: OSKB_FIN(2); break;
        case 3: OSKB_FIN(3); break;
        default: OSKB_FIN(4); break;
        }
#undef OSKB_FIN
        err = check_launch("station_beam_feeds_finalise");
    }
    if (norm_af) scratch_free(norm_af, s);
    return err;
}

template <typename T>
int jones_r(int num_sources, const T* ra, const T* dec, int num_stations,
        const double* lat_rad, const double* lst_rad, T* jones, void* stream)
{
    if (num_sources < 0 || num_stations < 0 || num_stations > 65535)
        return OSKB_ERR_INVALID_ARGUMENT;
    if (num_sources == 0 || num_stations == 0) return 0;
    if (!ra || !dec || !lat_rad || !lst_rad || !jones)
        return OSKB_ERR_INVALID_ARGUMENT;
    dim3 grid((num_sources + 255) / 256, num_stations);
    jones_r_kernel<T><<<grid, 256, 0, as_stream(stream)>>>(num_sources, ra,
            dec, lat_rad, lst_rad, jones);
    return check_launch("evaluate_jones_R");
}

}  // namespace
}  // namespace oskb

extern "C" {

#define OSKB_BEAM_ENTRY(T, S)                                                \
int oskb_station_beam_aa_##S(int num_stations, int num_elements,             \
        const T* el_x, const T* el_y, const T* el_z, const T* meas_x,        \
        const T* meas_y, const T* meas_z, const T* cable_length_error,       \
        const double* orientation_x_rad, const double* orientation_y_rad,    \
        double dipole_length_m, int normalise_element, int normalise_array,  \
        int normalise_final, int swap_xy, int is_3d, double frequency_hz,    \
        const double* beam_enu, const double* norm_enu, int num_directions,  \
        const T* x, const T* y, const T* z, int directions_per_station,      \
        T* beam, void* stream)                                               \
{                                                                            \
    return oskb::station_beam_aa<T>(num_stations, num_elements, el_x, el_y,  \
            el_z, meas_x, meas_y, meas_z, cable_length_error, nullptr, 1,    \
            nullptr, orientation_x_rad, orientation_y_rad, &dipole_length_m, \
            nullptr, nullptr, nullptr,                                       \
            normalise_element, normalise_array, normalise_final, swap_xy,    \
            is_3d, frequency_hz, beam_enu, norm_enu, num_directions, x, y,   \
            z, directions_per_station, beam, stream);                        \
}                                                                            \
int oskb_station_beam_aa_weighted_##S(int num_stations, int num_elements,    \
        const T* el_x, const T* el_y, const T* el_z, const T* meas_x,        \
        const T* meas_y, const T* meas_z, const T* cable_length_error,       \
        const T* element_weight_factors,                                     \
        const double* orientation_x_rad, const double* orientation_y_rad,    \
        double dipole_length_m, int normalise_element, int normalise_array,  \
        int normalise_final, int swap_xy, int is_3d, double frequency_hz,    \
        const double* beam_enu, const double* norm_enu, int num_directions,  \
        const T* x, const T* y, const T* z, int directions_per_station,      \
        T* beam, void* stream)                                               \
{                                                                            \
    return oskb::station_beam_aa<T>(num_stations, num_elements, el_x, el_y,  \
            el_z, meas_x, meas_y, meas_z, cable_length_error,                \
            element_weight_factors, 1, nullptr, orientation_x_rad,           \
            orientation_y_rad, &dipole_length_m, nullptr, nullptr, nullptr,  \
            normalise_element,                                               \
            normalise_array, normalise_final, swap_xy, is_3d, frequency_hz,  \
            beam_enu, norm_enu, num_directions, x, y, z,                     \
            directions_per_station, beam, stream);                           \
}                                                                            \
int oskb_station_beam_aa_types_##S(int num_stations, int num_elements,       \
        const T* el_x, const T* el_y, const T* el_z, const T* meas_x,        \
        const T* meas_y, const T* meas_z, const T* cable_length_error,       \
        const T* element_weight_factors, int num_element_types,              \
        const int* element_type, const double* dipole_length_m,              \
        const int* element_kind, const int* taper_kind,                      \
        const double* taper_param,                                           \
        const double* orientation_x_rad, const double* orientation_y_rad,    \
        int normalise_element, int normalise_array, int normalise_final,     \
        int swap_xy, int is_3d, double frequency_hz,                         \
        const double* beam_enu, const double* norm_enu, int num_directions,  \
        const T* x, const T* y, const T* z, int directions_per_station,      \
        T* beam, void* stream)                                               \
{                                                                            \
    return oskb::station_beam_aa<T>(num_stations, num_elements, el_x, el_y,  \
            el_z, meas_x, meas_y, meas_z, cable_length_error,                \
            element_weight_factors, num_element_types, element_type,         \
            orientation_x_rad, orientation_y_rad, dipole_length_m,           \
            element_kind, taper_kind, taper_param,                           \
            normalise_element, normalise_array, normalise_final, swap_xy,    \
            is_3d, frequency_hz, beam_enu, norm_enu, num_directions, x, y,   \
            z, directions_per_station, beam, stream);                        \
}                                                                            \
int oskb_station_beam_aa_scalar_##S(int num_stations, int num_elements,      \
        const T* el_x, const T* el_y, const T* el_z, const T* meas_x,        \
        const T* meas_y, const T* meas_z, const T* cable_length_error,       \
        const T* element_weight_factors, int num_element_types,              \
        const int* element_type, const double* dipole_length_m,              \
        const int* element_kind, const int* taper_kind,                      \
        const double* taper_param,                                           \
        const double* orientation_x_rad, const double* orientation_y_rad,    \
        int normalise_element, int normalise_array, int normalise_final,     \
        int swap_xy, int is_3d, double frequency_hz,                         \
        const double* beam_enu, const double* norm_enu, int num_directions,  \
        const T* x, const T* y, const T* z, int directions_per_station,      \
        T* beam, void* stream)                                               \
{                                                                            \
    return oskb::station_beam_aa<T>(num_stations, num_elements, el_x, el_y,  \
            el_z, meas_x, meas_y, meas_z, cable_length_error,                \
            element_weight_factors, num_element_types, element_type,         \
            orientation_x_rad, orientation_y_rad, dipole_length_m,           \
            element_kind, taper_kind, taper_param,                           \
            normalise_element, normalise_array, normalise_final, swap_xy,    \
            is_3d, frequency_hz, beam_enu, norm_enu, num_directions, x, y,   \
            z, directions_per_station, beam, stream, 0, nullptr, 1);         \
}                                                                            \
int oskb_station_beam_aa_feeds_##S(int num_feeds, int num_stations,        \
        int num_elements, const T* el_x, const T* el_y, const T* el_z,       \
        const T* meas_x, const T* meas_y, const T* meas_z,                   \
        const T* cable_length_error, const T* element_weight_factors,        \
        int num_element_types, const int* element_type,                     \
        const double* dipole_length_m, const int* element_kind,              \
        const int* taper_kind, const double* taper_param,                    \
        const double* orientation_x_rad,                                     \
        const double* orientation_y_rad, int normalise_element,              \
        int normalise_array, int normalise_final, int swap_xy, int is_3d,    \
        double frequency_hz, const double* beam_enu, const double* norm_enu, \
        int num_directions, const T* x, const T* y, const T* z,              \
        int directions_per_station, T* beam, void* stream)                   \
{                                                                            \
    return oskb::station_beam_aa_feeds<T>(num_feeds, num_stations,           \
            num_elements, el_x, el_y, el_z, meas_x, meas_y, meas_z,          \
            cable_length_error, element_weight_factors, num_element_types,   \
            element_type, orientation_x_rad, orientation_y_rad,              \
            dipole_length_m, element_kind, taper_kind, taper_param,          \
            normalise_element, normalise_array,                              \
            normalise_final, swap_xy, is_3d, frequency_hz, beam_enu,         \
            norm_enu, num_directions, x, y, z, directions_per_station, beam, \
            stream);                                                         \
}                                                                            \
int oskb_evaluate_jones_R_##S(int num_sources, const T* ra_rad,              \
        const T* dec_rad, int num_stations, const double* lat_rad,           \
        const double* lst_rad, T* jones, void* stream)                       \
{                                                                            \
    return oskb::jones_r<T>(num_sources, ra_rad, dec_rad, num_stations,      \
            lat_rad, lst_rad, jones, stream);                                \
}

OSKB_BEAM_ENTRY(double, d)
OSKB_BEAM_ENTRY(float, f)
#undef OSKB_BEAM_ENTRY

}  // extern "C"

// ---------------------------------------------------------------------------
// Hierarchical aperture-array stations of any depth: level 0 holds the leaf
// layouts (dipole arrays), each node type of level l > 0 is an array of
// children of level l - 1, and the top level is the station itself. The
// reference recurses (oskar_evaluate_station_beam_aperture_array.c:242-287):
// it evaluates every child station's beam, copying the first child's beam to
// all children when they are identical, then forms the parent's weighted DFT
// over its children with the child beams as the data. Here the recursion runs
// bottom-up over node TYPES instead of over the tree: one fused station-beam
// launch evaluates every leaf layout once, however many tiles share it, and
// each node type of each higher level is one launch of DFT weights and one
// weighted DFT whose data index is the child's type, so identical children
// (and any repeated sub-tree) cost no copies and no re-evaluation. Levels
// alternate between two beam buffers of the workspace; the top level writes
// the caller's beam.
// ---------------------------------------------------------------------------
namespace oskb {
namespace {

__global__ void hierarchy_setup_kernel(int num_types, double bx, double by,
        double bz, double* pointing, int num_zero, int* zero_idx)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x;
            i < num_types || i < num_zero; i += gridDim.x * blockDim.x)
    {
        if (i < num_types)
        {
            pointing[3 * i] = bx;
            pointing[3 * i + 1] = by;
            pointing[3 * i + 2] = bz;
        }
        if (zero_idx && i < num_zero) zero_idx[i] = 0;
    }
}

size_t align256(size_t b) { return (b + 255) & ~(size_t) 255; }

constexpr int kMaxLevels = 16;

// Checks the tree description; on success gives the most node types of the
// even and of the odd levels below the top (the two beam buffers) and the
// most children of any node (weights and the zero data index).
int hierarchy_shape(int num_levels, const int* num_types,
        const int* child_start, int& max_types_even, int& max_types_odd,
        int& max_children)
{
    if (num_levels < 2 || num_levels > kMaxLevels || !num_types ||
            !child_start)
        return OSKB_ERR_INVALID_ARGUMENT;
    for (int l = 0; l < num_levels; ++l)
        if (num_types[l] < 1 || num_types[l] > 65535)
            return OSKB_ERR_INVALID_ARGUMENT;
    if (num_types[num_levels - 1] != 1) return OSKB_ERR_INVALID_ARGUMENT;
    max_types_even = max_types_odd = max_children = 0;
    for (int l = 0; l < num_levels - 1; ++l)
    {
        int& m = (l % 2) ? max_types_odd : max_types_even;
        if (num_types[l] > m) m = num_types[l];
    }
    if (child_start[0] != 0) return OSKB_ERR_INVALID_ARGUMENT;
    int nodes = 0;
    for (int l = 1; l < num_levels; ++l) nodes += num_types[l];
    for (int n = 0; n < nodes; ++n)
    {
        const long long c = (long long) child_start[n + 1] - child_start[n];
        if (c < 1 || c > INT_MAX / 2) return OSKB_ERR_INVALID_ARGUMENT;
        if (c > max_children) max_children = (int) c;
    }
    return 0;
}

size_t hierarchy_workspace(size_t elem, int num_directions,
        int max_types_even, int max_types_odd, int max_children,
        int num_leaf_types)
{
    return align256(elem * 8 * (size_t) max_types_even * num_directions) +
            align256(elem * 8 * (size_t) max_types_odd * num_directions) +
            align256(elem * 2 * (size_t) max_children) +
            align256(sizeof(double) * 3 * (size_t) num_leaf_types) +
            align256(sizeof(int) * (size_t) max_children);
}

template <typename T>
int station_beam_hierarchical(int num_levels, const int* num_types,
        int num_elements, const T* el_x, const T* el_y, const T* el_z,
        const double* orientation_x, const double* orientation_y,
        double dipole_length_m, int normalise_element,
        const int* normalise_array, const int* child_start,
        const T* child_x, const T* child_y, const T* child_z,
        const int* child_type, int swap_xy, int is_3d, double frequency_hz,
        const double* beam_enu, int num_directions, const T* x, const T* y,
        const T* z, void* workspace, size_t workspace_bytes, T* beam,
        void* stream)
{
    int max_even = 0, max_odd = 0, max_children = 0;
    if (int err = hierarchy_shape(num_levels, num_types, child_start,
            max_even, max_odd, max_children))
        return err;
    if (num_directions < 0 || !normalise_array || !beam_enu)
        return OSKB_ERR_INVALID_ARGUMENT;
    if (num_directions == 0) return 0;
    if (!child_x || !child_y || (is_3d && !child_z) || !workspace || !beam)
        return OSKB_ERR_INVALID_ARGUMENT;
    if (workspace_bytes < hierarchy_workspace(sizeof(T), num_directions,
            max_even, max_odd, max_children, num_types[0]))
        return OSKB_ERR_MEMORY_ALLOC_FAILURE;
    uint8_t* w = static_cast<uint8_t*>(workspace);
    T* level_beams[2];
    level_beams[0] = reinterpret_cast<T*>(w);
    w += align256(sizeof(T) * 8 * (size_t) max_even * num_directions);
    level_beams[1] = reinterpret_cast<T*>(w);
    w += align256(sizeof(T) * 8 * (size_t) max_odd * num_directions);
    T* weights = reinterpret_cast<T*>(w);
    w += align256(sizeof(T) * 2 * (size_t) max_children);
    double* pointing = reinterpret_cast<double*>(w);
    w += align256(sizeof(double) * 3 * (size_t) num_types[0]);
    int* zero_idx = child_type ? nullptr : reinterpret_cast<int*>(w);
    cudaStream_t s = as_stream(stream);
    const int n = num_types[0] > max_children ? num_types[0] : max_children;
    hierarchy_setup_kernel<<<(n + 255) / 256, 256, 0, s>>>(num_types[0],
            beam_enu[0], beam_enu[1], beam_enu[2], pointing, max_children,
            zero_idx);
    if (int err = check_launch("station_beam_hierarchical")) return err;
    // leaf beams [type][direction]: element pattern x leaf array factor,
    // blanked below the horizon, no final normalisation
    if (int err = station_beam_aa<T>(num_types[0], num_elements, el_x, el_y,
            el_z, nullptr, nullptr, nullptr, nullptr, nullptr, 1, nullptr,
            orientation_x, orientation_y, &dipole_length_m, nullptr, nullptr,
            nullptr, normalise_element, normalise_array[0], 0, swap_xy,
            is_3d, frequency_hz, pointing, nullptr, num_directions, x, y, z,
            0, level_beams[0], stream))
        return err;
    const double k = 2.0 * kPi * frequency_hz / 299792458.0;
    const T* zo = is_3d ? z : nullptr;
    const size_t beam_stride = (size_t) 8 * num_directions;
    int node = 0;
    for (int l = 1; l < num_levels; ++l)
    {
        const T* data = level_beams[(l - 1) % 2];
        const double* b = beam_enu + 3 * l;
        for (int j = 0; j < num_types[l]; ++j, ++node)
        {
            const int c0 = child_start[node];
            const int nc = child_start[node + 1] - c0;
            const T* cz = is_3d ? child_z + c0 : nullptr;
            const int* idx = child_type ? child_type + c0 : zero_idx;
            T* out = (l == num_levels - 1) ? beam :
                    level_beams[l % 2] + beam_stride * j;
            const T norm = normalise_array[l] ? (T) (1.0 / nc) : (T) 1;
            if constexpr (sizeof(T) == 8)
            {
                if (int err = oskb_evaluate_element_weights_dft_d(nc,
                        child_x + c0, child_y + c0, cz, nullptr, k, b[0],
                        b[1], is_3d ? b[2] : 0.0, weights, stream))
                    return err;
                if (int err = oskb_dftw_d(1, nc, k, weights, child_x + c0,
                        child_y + c0, cz, 0, num_directions, x, y, zo, idx,
                        data, 1, 1, 0, out, norm, stream))
                    return err;
            }
            else
            {
                if (int err = oskb_evaluate_element_weights_dft_f(nc,
                        child_x + c0, child_y + c0, cz, nullptr, (float) k,
                        (float) b[0], (float) b[1],
                        (float) (is_3d ? b[2] : 0.0), weights, stream))
                    return err;
                if (int err = oskb_dftw_f(1, nc, (float) k, weights,
                        child_x + c0, child_y + c0, cz, 0, num_directions, x,
                        y, zo, idx, data, 1, 1, 0, out, norm, stream))
                    return err;
            }
        }
    }
    return 0;
}

}  // namespace
}  // namespace oskb

extern "C" {

size_t oskb_station_beam_hierarchical_workspace_bytes(int precision_bytes,
        int num_levels, const int* num_types, const int* child_start,
        int num_directions)
{
    int max_even = 0, max_odd = 0, max_children = 0;
    if ((precision_bytes != 4 && precision_bytes != 8) ||
            num_directions < 0 || oskb::hierarchy_shape(num_levels,
                num_types, child_start, max_even, max_odd, max_children))
        return 0;
    return oskb::hierarchy_workspace((size_t) precision_bytes,
            num_directions, max_even, max_odd, max_children, num_types[0]);
}

size_t oskb_station_beam_two_level_workspace_bytes(int precision_bytes,
        int num_tile_types, int num_tiles, int num_directions)
{
    if (num_tiles < 1)
        return num_tile_types >= 1 && num_tiles == 0 &&
                num_directions >= 0 ? 256 : 0;
    const int types[2] = {num_tile_types, 1};
    const int start[2] = {0, num_tiles};
    return oskb_station_beam_hierarchical_workspace_bytes(precision_bytes,
            2, types, start, num_directions);
}

#define OSKB_HIERARCHICAL_ENTRY(T, S)                                        \
int oskb_station_beam_hierarchical_##S(int num_levels,                       \
        const int* num_types, int num_elements, const T* el_x,               \
        const T* el_y, const T* el_z, const double* orientation_x_rad,       \
        const double* orientation_y_rad, double dipole_length_m,             \
        int normalise_element, const int* normalise_array,                   \
        const int* child_start, const T* child_x, const T* child_y,          \
        const T* child_z, const int* child_type, int swap_xy, int is_3d,     \
        double frequency_hz, const double* beam_enu, int num_directions,     \
        const T* x, const T* y, const T* z, void* workspace,                 \
        size_t workspace_bytes, T* beam, void* stream)                       \
{                                                                            \
    return oskb::station_beam_hierarchical<T>(num_levels, num_types,         \
            num_elements, el_x, el_y, el_z, orientation_x_rad,               \
            orientation_y_rad, dipole_length_m, normalise_element,           \
            normalise_array, child_start, child_x, child_y, child_z,         \
            child_type, swap_xy, is_3d, frequency_hz, beam_enu,              \
            num_directions, x, y, z, workspace, workspace_bytes, beam,       \
            stream);                                                         \
}

OSKB_HIERARCHICAL_ENTRY(double, d)
OSKB_HIERARCHICAL_ENTRY(float, f)
#undef OSKB_HIERARCHICAL_ENTRY

// The two-level station is the hierarchy {tile layouts, station}.
#define OSKB_TWO_LEVEL_ENTRY(T, S)                                           \
int oskb_station_beam_two_level_##S(int num_tile_types, int num_elements,    \
        const T* el_x, const T* el_y, const T* el_z,                         \
        const double* orientation_x_rad, const double* orientation_y_rad,    \
        double dipole_length_m, int normalise_element,                       \
        int normalise_tile_array, int num_tiles, const T* tile_x,            \
        const T* tile_y, const T* tile_z, const int* tile_type,              \
        int normalise_station_array, int swap_xy, int is_3d,                 \
        double frequency_hz, double beam_x, double beam_y, double beam_z,    \
        int num_directions, const T* x, const T* y, const T* z,              \
        void* workspace, size_t workspace_bytes, T* beam, void* stream)      \
{                                                                            \
    if (num_tile_types < 1 || num_tiles < 0 || num_directions < 0)           \
        return OSKB_ERR_INVALID_ARGUMENT;                                    \
    if (num_tiles == 0 || num_directions == 0) return 0;                     \
    const int types[2] = {num_tile_types, 1};                                \
    const int start[2] = {0, num_tiles};                                     \
    const int norm[2] = {normalise_tile_array, normalise_station_array};     \
    const double b[6] = {beam_x, beam_y, beam_z, beam_x, beam_y, beam_z};    \
    return oskb::station_beam_hierarchical<T>(2, types, num_elements, el_x,  \
            el_y, el_z, orientation_x_rad, orientation_y_rad,                \
            dipole_length_m, normalise_element, norm, start, tile_x, tile_y, \
            tile_z, tile_type, swap_xy, is_3d, frequency_hz, b,              \
            num_directions, x, y, z, workspace, workspace_bytes, beam,       \
            stream);                                                         \
}

OSKB_TWO_LEVEL_ENTRY(double, d)
OSKB_TWO_LEVEL_ENTRY(float, f)
#undef OSKB_TWO_LEVEL_ENTRY

}  // extern "C"

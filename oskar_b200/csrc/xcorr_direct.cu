// Direct cross-correlation kernel (all source types and smearing modes).
//
// Replaces the reference's warp-per-baseline kernel
// (oskar/correlate/src/oskar_cross_correlate_cuda.cu:45-224) with a
// register-tiled form: one CTA owns a 32 x 32 block of stations (rows p,
// columns q, lower triangle p > q as in the reference), each thread a 2 x 2
// group of baselines. Sources are staged through shared memory in chunks:
// the "left" factor J B (or I J in scalar mode) and the "right" factor J are
// computed once per station-source for the whole CTA, so the per
// source-baseline work is the 8 complex MACs of (J_p B) J_q^H. Smearing
// arguments are per-station source phases (phi_p - phi_q), which turns the
// reference's three multiply-adds per source-baseline into one subtraction.
// FP64 mode accumulates in FP64; FP32 mode sums each chunk in FP32 and the
// chunk sums in FP64.
#include "common.cuh"

namespace oskb {
namespace {

constexpr int kTile = 32;      // stations per block edge
constexpr int kChunk = 16;     // sources per shared-memory chunk
constexpr int kThreads = 256;  // 16 x 16 threads, 2 x 2 baselines each

template <typename T>
struct XcorrParams
{
    int num_src, num_st, offset_out;
    const T* jones;
    const T *I, *Q, *U, *V, *l, *m, *n, *a, *b, *c;
    const T *st_u, *st_v, *st_w, *st_x, *st_y;
    double uv_min, uv_max, inv_wavelength;
    double bw_scale;  // pi * frac_bandwidth * inv_wavelength
    double ts_scale;  // pi * inv_wavelength * omega_earth * time_int_sec
    double s_ha, c_ha, s_dec, c_dec;
    T* vis;
};

template <typename T, bool MATRIX>
struct Smem
{
    typedef typename vec2<T>::type T2;
    static constexpr int NCOMP = MATRIX ? 4 : 1;
    // [comp][chunk][tile] complex, for the row (p) and column (q) blocks
    T2 row[NCOMP][kChunk][kTile];
    T2 col[NCOMP][kChunk][kTile];
    T ph_row[kChunk][kTile], ph_col[kChunk][kTile];  // bandwidth phases
    T ps_row[kChunk][kTile], ps_col[kChunk][kTile];  // time-smearing phases
    T ga[kChunk], gb[kChunk], gc[kChunk];
};

template <typename T>
__device__ __forceinline__ T sinc(T x)
{
    return x == (T) 0 ? (T) 1 : sin(x) / x;
}

// Maps a linear block index to (bp, bq) with bp >= bq.
__device__ __forceinline__ void tri_block(int k, int& bp, int& bq)
{
    int p = (int) ((sqrt(8.0 * k + 1.0) - 1.0) * 0.5);
    while ((p + 1) * (p + 2) / 2 <= k) ++p;
    while (p * (p + 1) / 2 > k) --p;
    bp = p;
    bq = k - p * (p + 1) / 2;
}

template <typename T, bool MATRIX, bool GAUSS, bool BW, bool TS, bool CASA>
__global__ void __launch_bounds__(kThreads, 1)
xcorr_direct_kernel(const XcorrParams<T> prm)
{
    typedef typename vec2<T>::type T2;
    typedef Smem<T, MATRIX> S;
    constexpr int NC = S::NCOMP;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    S& sm = *reinterpret_cast<S*>(smem_raw);

    int bp, bq;
    tri_block(blockIdx.x, bp, bq);
    const int p0 = bp * kTile, q0 = bq * kTile;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int N = prm.num_st;

    // Per-thread baseline terms.
    bool valid[2][2];
    T uu2[2][2], vv2[2][2], uuvv[2][2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
        {
            // Baseline terms as the reference forms them
            // (oskar/correlate/define_correlate_utils.h:5-13).
            const int p = p0 + ty + 16 * i, q = q0 + tx + 16 * j;
            bool ok = (p < N) && (q < p);
            T uu = 0, vv = 0;
            if (ok)
            {
                uu = (prm.st_u[p] - prm.st_u[q]) * (T) prm.inv_wavelength;
                vv = (prm.st_v[p] - prm.st_v[q]) * (T) prm.inv_wavelength;
                const T len = sqrt(uu * uu + vv * vv);
                ok = !(len < (T) prm.uv_min || len > (T) prm.uv_max);
            }
            valid[i][j] = ok;
            uu2[i][j] = uu * uu;
            vv2[i][j] = vv * vv;
            uuvv[i][j] = 2 * uu * vv;
        }

    // Accumulators: FP64 always; FP32 mode adds per-chunk FP32 partials.
    double acc[2][2][2 * NC];
    T part[2][2][2 * NC];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int k = 0; k < 2 * NC; ++k)
            {
                acc[i][j][k] = 0;
                part[i][j][k] = 0;
            }

    for (int s0 = 0; s0 < prm.num_src; s0 += kChunk)
    {
        const int ns = min(kChunk, prm.num_src - s0);
        // ---- stage the chunk: 2 blocks x kTile stations x kChunk sources
        for (int it = tid; it < 2 * kTile * kChunk; it += kThreads)
        {
            const int blk = it / (kTile * kChunk);
            const int rem = it - blk * (kTile * kChunk);
            const int sl = rem % kChunk, stl = rem / kChunk;
            const int st = (blk ? q0 : p0) + stl, s = s0 + sl;
            const bool in = (st < N) && (sl < ns);
            // Left factor (J B, or I J) lives in the row block unless CASA.
            const bool left = (blk == 0) != CASA;
            T2 (*dst)[kChunk][kTile] = blk ? sm.col : sm.row;
            if (MATRIX)
            {
                Mat2<T> J;
                if (in)
                    J = load_mat(prm.jones + 8 * ((size_t) st * prm.num_src + s));
                else
                    J.a = J.b = J.c = J.d = T2{0, 0};
                if (left && in)
                {
                    const T I = prm.I[s], Q = prm.Q[s];
                    const T2 buv = T2{prm.U[s], prm.V[s]};
                    const T2 buvc = T2{prm.U[s], -prm.V[s]};
                    const T xx = I + Q, yy = I - Q;
                    Mat2<T> M;
                    const T2 t0 = cmul<T>(J.b, buvc), t1 = cmul<T>(J.d, buvc);
                    const T2 t2 = cmul<T>(J.a, buv), t3 = cmul<T>(J.c, buv);
                    M.a = T2{J.a.x * xx + t0.x, J.a.y * xx + t0.y};
                    M.c = T2{J.c.x * xx + t1.x, J.c.y * xx + t1.y};
                    M.b = T2{J.b.x * yy + t2.x, J.b.y * yy + t2.y};
                    M.d = T2{J.d.x * yy + t3.x, J.d.y * yy + t3.y};
                    J = M;
                }
                dst[0][sl][stl] = J.a;
                dst[1][sl][stl] = J.b;
                dst[2][sl][stl] = J.c;
                dst[3][sl][stl] = J.d;
            }
            else
            {
                T2 J = T2{0, 0};
                if (in)
                    J = reinterpret_cast<const T2*>(prm.jones)[
                            (size_t) st * prm.num_src + s];
                if (left && in)
                {
                    const T I = prm.I[s];
                    J.x *= I; J.y *= I;
                }
                dst[0][sl][stl] = J;
            }
            if (BW || TS)
            {
                T ph = 0, ps = 0;
                if (in)
                {
                    const double l = prm.l[s], m = prm.m[s];
                    const double n1 = (double) prm.n[s] - 1.0;
                    if (BW)
                        ph = (T) (((double) prm.st_u[st] * l +
                                (double) prm.st_v[st] * m +
                                (double) prm.st_w[st] * n1) * prm.bw_scale);
                    if (TS)
                    {
                        const double x = prm.st_x[st], y = prm.st_y[st];
                        ps = (T) (((x * prm.c_ha - y * prm.s_ha) * l +
                                (x * prm.s_ha + y * prm.c_ha) *
                                (prm.s_dec * m - prm.c_dec * n1)) *
                                prm.ts_scale);
                    }
                }
                if (blk) { sm.ph_col[sl][stl] = ph; sm.ps_col[sl][stl] = ps; }
                else { sm.ph_row[sl][stl] = ph; sm.ps_row[sl][stl] = ps; }
            }
        }
        if (GAUSS && tid < kChunk)
        {
            const bool in = tid < ns;
            sm.ga[tid] = in ? prm.a[s0 + tid] : (T) 0;
            sm.gb[tid] = in ? prm.b[s0 + tid] : (T) 0;
            sm.gc[tid] = in ? prm.c[s0 + tid] : (T) 0;
        }
        __syncthreads();

        // ---- accumulate
        for (int sl = 0; sl < ns; ++sl)
        {
            T2 R[2][NC], C[2][NC];
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int k = 0; k < NC; ++k)
                {
                    R[i][k] = sm.row[k][sl][ty + 16 * i];
                    C[i][k] = sm.col[k][sl][tx + 16 * i];
                }
            T smear[2][2];
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j)
                {
                    T f = (T) 1;
                    if (GAUSS)
                        f = exp(-(sm.ga[sl] * uu2[i][j] + sm.gb[sl] * uuvv[i][j]
                                + sm.gc[sl] * vv2[i][j]));
                    if (BW)
                        f *= sinc<T>(sm.ph_row[sl][ty + 16 * i] -
                                sm.ph_col[sl][tx + 16 * j]);
                    if (TS)
                        f *= sinc<T>(sm.ps_row[sl][ty + 16 * i] -
                                sm.ps_col[sl][tx + 16 * j]);
                    smear[i][j] = f;
                }
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j)
                {
                    // L * conj-transpose(Rt): L = left factor, Rt = right.
                    const T2* L = CASA ? C[j] : R[i];
                    const T2* Rt = CASA ? R[i] : C[j];
                    T t[2 * NC];
                    if constexpr (MATRIX)
                    {
                        // a = La Ra* + Lb Rb*, b = La Rc* + Lb Rd*,
                        // c = Lc Ra* + Ld Rb*, d = Lc Rc* + Ld Rd*
#define OSKB_CMAC2(OUT, X0, Y0, X1, Y1) \
                        OUT[0] = X0.x * Y0.x + X0.y * Y0.y + X1.x * Y1.x + X1.y * Y1.y; \
                        OUT[1] = X0.y * Y0.x - X0.x * Y0.y + X1.y * Y1.x - X1.x * Y1.y;
                        OSKB_CMAC2((t + 0), L[0], Rt[0], L[1], Rt[1])
                        OSKB_CMAC2((t + 2), L[0], Rt[2], L[1], Rt[3])
                        OSKB_CMAC2((t + 4), L[2], Rt[0], L[3], Rt[1])
                        OSKB_CMAC2((t + 6), L[2], Rt[2], L[3], Rt[3])
#undef OSKB_CMAC2
                    }
                    else
                    {
                        t[0] = L[0].x * Rt[0].x + L[0].y * Rt[0].y;
                        t[1] = L[0].y * Rt[0].x - L[0].x * Rt[0].y;
                    }
                    if (GAUSS || BW || TS)
                    {
#pragma unroll
                        for (int k = 0; k < 2 * NC; ++k)
                            part[i][j][k] += t[k] * smear[i][j];
                    }
                    else
                    {
#pragma unroll
                        for (int k = 0; k < 2 * NC; ++k)
                            part[i][j][k] += t[k];
                    }
                }
        }
        if (sizeof(T) == 4)
        {
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j)
#pragma unroll
                    for (int k = 0; k < 2 * NC; ++k)
                    {
                        acc[i][j][k] += (double) part[i][j][k];
                        part[i][j][k] = 0;
                    }
        }
        __syncthreads();
    }

    // ---- write out: each baseline is owned by exactly one thread
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
        {
            if (!valid[i][j]) continue;
            const int p = p0 + ty + 16 * i, q = q0 + tx + 16 * j;
            T* out = prm.vis + (size_t) (2 * NC) *
                    (size_t) (baseline_index(N, p, q) + prm.offset_out);
#pragma unroll
            for (int k = 0; k < 2 * NC; ++k)
            {
                const double v = (sizeof(T) == 4) ? acc[i][j][k]
                                                  : (double) part[i][j][k];
                out[k] = (T) ((double) out[k] + v);
            }
        }
}

template <typename T, bool MATRIX, bool GAUSS, bool BW, bool TS>
void launch_casa(bool casa, const XcorrParams<T>& p, int grid,
        cudaStream_t stream)
{
    const size_t smem = sizeof(Smem<T, MATRIX>);
    if (casa)
    {
        auto k = xcorr_direct_kernel<T, MATRIX, GAUSS, BW, TS, true>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                (int) smem);
        k<<<grid, kThreads, smem, stream>>>(p);
    }
    else
    {
        auto k = xcorr_direct_kernel<T, MATRIX, GAUSS, BW, TS, false>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                (int) smem);
        k<<<grid, kThreads, smem, stream>>>(p);
    }
}

template <typename T, bool MATRIX>
int xcorr_dispatch(bool casa, bool gauss, const XcorrParams<T>& p,
        bool bw, bool ts, cudaStream_t stream)
{
    if (p.num_st < 2 || p.num_src <= 0) return 0;
    const int nb = (p.num_st + kTile - 1) / kTile;
    const int grid = nb * (nb + 1) / 2;
#define OSKB_SEL(G, B, S) launch_casa<T, MATRIX, G, B, S>(casa, p, grid, stream)
    if (gauss)
    {
        if (!bw && !ts) OSKB_SEL(true, false, false);
        else if (bw && !ts) OSKB_SEL(true, true, false);
        else if (!bw && ts) OSKB_SEL(true, false, true);
        else OSKB_SEL(true, true, true);
    }
    else
    {
        if (!bw && !ts) OSKB_SEL(false, false, false);
        else if (bw && !ts) OSKB_SEL(false, true, false);
        else if (!bw && ts) OSKB_SEL(false, false, true);
        else OSKB_SEL(false, true, true);
    }
#undef OSKB_SEL
    return check_launch("xcorr_direct");
}

template <typename T>
XcorrParams<T> make_params(int num_sources, int num_stations, int offset_out,
        const T* jones, const T* I, const T* Q, const T* U, const T* V,
        const T* l, const T* m, const T* n, const T* a, const T* b,
        const T* c, const T* su, const T* sv, const T* sw, const T* sx,
        const T* sy, T uv_min, T uv_max, T inv_wavelength, T frac_bandwidth,
        T time_int_sec, T gha0, T dec0, T* vis)
{
    XcorrParams<T> p;
    p.num_src = num_sources; p.num_st = num_stations; p.offset_out = offset_out;
    p.jones = jones; p.I = I; p.Q = Q; p.U = U; p.V = V;
    p.l = l; p.m = m; p.n = n; p.a = a; p.b = b; p.c = c;
    p.st_u = su; p.st_v = sv; p.st_w = sw; p.st_x = sx; p.st_y = sy;
    p.uv_min = uv_min; p.uv_max = uv_max; p.inv_wavelength = inv_wavelength;
    p.bw_scale = kPi * (double) frac_bandwidth * (double) inv_wavelength;
    p.ts_scale = kPi * (double) inv_wavelength * kOmegaEarth *
            (double) time_int_sec;
    p.s_ha = sin((double) gha0); p.c_ha = cos((double) gha0);
    p.s_dec = sin((double) dec0); p.c_dec = cos((double) dec0);
    p.vis = vis;
    return p;
}

template <typename T>
int check_args(int gaussian, int num_sources, int num_stations,
        const T* jones, const T* I, const T* a, const T* b, const T* c,
        const T* vis, bool ts, const T* sx, const T* sy)
{
    if (num_sources < 0 || num_stations < 0) return OSKB_ERR_INVALID_ARGUMENT;
    if (num_sources == 0 || num_stations < 2) return 0;
    if (!jones || !I || !vis) return OSKB_ERR_INVALID_ARGUMENT;
    if (gaussian && (!a || !b || !c)) return OSKB_ERR_INVALID_ARGUMENT;
    if (ts && (!sx || !sy)) return OSKB_ERR_INVALID_ARGUMENT;
    return 0;
}

}  // namespace
}  // namespace oskb

using namespace oskb;

#define OSKB_XCORR_ENTRY(NAME, T, MATRIX)                                      \
int NAME(int casa, int gaussian, int num_sources, int num_stations,           \
        int offset_out, const T* jones, const T* I, const T* Q, const T* U,   \
        const T* V, const T* l, const T* m, const T* n, const T* a,           \
        const T* b, const T* c, const T* su, const T* sv, const T* sw,       \
        const T* sx, const T* sy, T uv_min, T uv_max, T inv_wavelength,       \
        T frac_bandwidth, T time_int_sec, T gha0, T dec0, T* vis,             \
        void* stream)                                                          \
{                                                                              \
    const bool bw = frac_bandwidth != (T) 0, ts = time_int_sec != (T) 0;      \
    int err = check_args<T>(gaussian, num_sources, num_stations, jones, I,    \
            a, b, c, vis, ts, sx, sy);                                         \
    if (err || num_sources == 0 || num_stations < 2) return err;              \
    if (MATRIX && (!Q || !U || !V)) return OSKB_ERR_INVALID_ARGUMENT;         \
    if ((bw || ts) && (!l || !m || !n)) return OSKB_ERR_INVALID_ARGUMENT;     \
    XcorrParams<T> p = make_params<T>(num_sources, num_stations, offset_out,  \
            jones, I, Q, U, V, l, m, n, a, b, c, su, sv, sw, sx, sy, uv_min,  \
            uv_max, inv_wavelength, frac_bandwidth, time_int_sec, gha0, dec0, \
            vis);                                                              \
    return xcorr_dispatch<T, MATRIX>(casa != 0, gaussian != 0, p, bw, ts,     \
            as_stream(stream));                                                \
}

extern "C" {

OSKB_XCORR_ENTRY(oskb_cross_correlate_d, double, true)
OSKB_XCORR_ENTRY(oskb_cross_correlate_f, float, true)

int oskb_cross_correlate_scalar_d(int casa, int gaussian, int num_sources,
        int num_stations, int offset_out, const double* jones,
        const double* I, const double* l, const double* m, const double* n,
        const double* a, const double* b, const double* c, const double* su,
        const double* sv, const double* sw, const double* sx,
        const double* sy, double uv_min, double uv_max, double inv_wavelength,
        double frac_bandwidth, double time_int_sec, double gha0, double dec0,
        double* vis, void* stream);
int oskb_cross_correlate_scalar_f(int casa, int gaussian, int num_sources,
        int num_stations, int offset_out, const float* jones, const float* I,
        const float* l, const float* m, const float* n, const float* a,
        const float* b, const float* c, const float* su, const float* sv,
        const float* sw, const float* sx, const float* sy, float uv_min,
        float uv_max, float inv_wavelength, float frac_bandwidth,
        float time_int_sec, float gha0, float dec0, float* vis, void* stream);
}

namespace {
OSKB_XCORR_ENTRY(scalar_impl_d, double, false)
OSKB_XCORR_ENTRY(scalar_impl_f, float, false)
}

extern "C" int oskb_cross_correlate_scalar_d(int casa, int gaussian,
        int num_sources, int num_stations, int offset_out,
        const double* jones, const double* I, const double* l,
        const double* m, const double* n, const double* a, const double* b,
        const double* c, const double* su, const double* sv, const double* sw,
        const double* sx, const double* sy, double uv_min, double uv_max,
        double inv_wavelength, double frac_bandwidth, double time_int_sec,
        double gha0, double dec0, double* vis, void* stream)
{
    return scalar_impl_d(casa, gaussian, num_sources, num_stations,
            offset_out, jones, I, nullptr, nullptr, nullptr, l, m, n, a, b, c,
            su, sv, sw, sx, sy, uv_min, uv_max, inv_wavelength,
            frac_bandwidth, time_int_sec, gha0, dec0, vis, stream);
}

extern "C" int oskb_cross_correlate_scalar_f(int casa, int gaussian,
        int num_sources, int num_stations, int offset_out, const float* jones,
        const float* I, const float* l, const float* m, const float* n,
        const float* a, const float* b, const float* c, const float* su,
        const float* sv, const float* sw, const float* sx, const float* sy,
        float uv_min, float uv_max, float inv_wavelength,
        float frac_bandwidth, float time_int_sec, float gha0, float dec0,
        float* vis, void* stream)
{
    return scalar_impl_f(casa, gaussian, num_sources, num_stations,
            offset_out, jones, I, nullptr, nullptr, nullptr, l, m, n, a, b, c,
            su, sv, sw, sx, sy, uv_min, uv_max, inv_wavelength,
            frac_bandwidth, time_int_sec, gha0, dec0, vis, stream);
}

// Element-wise and per-station kernels on the hot path: Jones K, the Jones
// join products, auto-correlation, beamforming weights, station (u, v, w).
// All are HBM-bound; they use one thread per output element with vectorised
// 16-byte loads and grid-stride loops sized to a multiple of the SM count.
#include <string.h>

#include "common.cuh"

namespace oskb {

static thread_local char g_last_error[256] = "";

void set_last_error(const char* where, cudaError_t err)
{
    snprintf(g_last_error, sizeof(g_last_error), "%s: %s", where,
            cudaGetErrorString(err));
}

void set_last_error_msg(const char* msg)
{
    snprintf(g_last_error, sizeof(g_last_error), "%s", msg);
}

namespace {

int grid_for(size_t n, int threads)
{
    const int num_sms = device_sm_count();
    size_t blocks = (n + threads - 1) / threads;
    const size_t cap = (size_t) num_sms * 16;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    return (int) blocks;
}

// ---- Jones K (interferometer/define_evaluate_jones_K.h:56-70 order of
// operations: phase = u l + v m [+ w (n - 1)], then * wavenumber).
template <typename T>
__global__ void jones_k_kernel(int num_src, const T* __restrict__ l,
        const T* __restrict__ m, const T* __restrict__ n, int num_st,
        const T* __restrict__ u, const T* __restrict__ v,
        const T* __restrict__ w, T wavenumber, const T* __restrict__ filter,
        T fmin, T fmax, int ignore_w, typename vec2<T>::type* jones)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int a = blockIdx.y;
    if (s >= num_src) return;
    typename vec2<T>::type out;
    out.x = out.y = (T) 0;
    const T f = filter[s];
    if (f > fmin && f <= fmax)
    {
        T ph = u[a] * l[s] + v[a] * m[s];
        if (!ignore_w) ph += w[a] * (n[s] - (T) 1);
        ph *= wavenumber;
        T sn, cs;
        sincos(ph, &sn, &cs);
        out.x = cs; out.y = sn;
    }
    jones[(size_t) s + (size_t) num_src * a] = out;
}

// ---- element-wise products (mem/define_mem_multiply.h:3-89)
template <typename T>
struct Cx { T re, im; };

template <typename T>
__device__ __forceinline__ Cx<T> cm(Cx<T> x, Cx<T> y)
{
    return Cx<T>{x.re * y.re - x.im * y.im, x.re * y.im + x.im * y.re};
}

template <typename T, int KIND>
__global__ void mem_mul_kernel(size_t off_a, size_t off_b, size_t off_c,
        size_t n, const T* a, const T* b, T* c)
{
    const size_t stride = (size_t) gridDim.x * blockDim.x;
    for (size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
            i += stride)
    {
        if (KIND == OSKB_MUL_RR_R)
        {
            c[i + off_c] = a[i + off_a] * b[i + off_b];
        }
        else if (KIND == OSKB_MUL_CC_C || KIND == OSKB_MUL_CC_M)
        {
            const Cx<T> x{a[2 * (i + off_a)], a[2 * (i + off_a) + 1]};
            const Cx<T> y{b[2 * (i + off_b)], b[2 * (i + off_b) + 1]};
            const Cx<T> r = cm(x, y);
            if (KIND == OSKB_MUL_CC_C)
            {
                c[2 * (i + off_c)] = r.re; c[2 * (i + off_c) + 1] = r.im;
            }
            else
            {
                T* o = c + 8 * (i + off_c);
                o[0] = r.re; o[1] = r.im; o[2] = 0; o[3] = 0;
                o[4] = 0; o[5] = 0; o[6] = r.re; o[7] = r.im;
            }
        }
        else if (KIND == OSKB_MUL_CM_M || KIND == OSKB_MUL_MC_M)
        {
            const T* sp = (KIND == OSKB_MUL_CM_M) ? a + 2 * (i + off_a)
                                                  : b + 2 * (i + off_b);
            const T* mp = (KIND == OSKB_MUL_CM_M) ? b + 8 * (i + off_b)
                                                  : a + 8 * (i + off_a);
            const Cx<T> s{sp[0], sp[1]};
            T mv[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) mv[k] = mp[k];
            T* o = c + 8 * (i + off_c);
#pragma unroll
            for (int k = 0; k < 4; ++k)
            {
                const Cx<T> r = cm(Cx<T>{mv[2 * k], mv[2 * k + 1]}, s);
                o[2 * k] = r.re; o[2 * k + 1] = r.im;
            }
        }
        else  // OSKB_MUL_MM_M
        {
            T x[8], y[8];
#pragma unroll
            for (int k = 0; k < 8; ++k)
            {
                x[k] = a[8 * (i + off_a) + k];
                y[k] = b[8 * (i + off_b) + k];
            }
            const Cx<T> xa{x[0], x[1]}, xb{x[2], x[3]}, xc{x[4], x[5]},
                    xd{x[6], x[7]}, ya{y[0], y[1]}, yb{y[2], y[3]},
                    yc{y[4], y[5]}, yd{y[6], y[7]};
            Cx<T> r[4];
            Cx<T> t0 = cm(xa, ya), t1 = cm(xb, yc);
            r[0] = Cx<T>{t0.re + t1.re, t0.im + t1.im};
            t0 = cm(xa, yb); t1 = cm(xb, yd);
            r[1] = Cx<T>{t0.re + t1.re, t0.im + t1.im};
            t0 = cm(xc, ya); t1 = cm(xd, yc);
            r[2] = Cx<T>{t0.re + t1.re, t0.im + t1.im};
            t0 = cm(xc, yb); t1 = cm(xd, yd);
            r[3] = Cx<T>{t0.re + t1.re, t0.im + t1.im};
            T* o = c + 8 * (i + off_c);
#pragma unroll
            for (int k = 0; k < 4; ++k)
            {
                o[2 * k] = r[k].re; o[2 * k + 1] = r[k].im;
            }
        }
    }
}

// ---- auto-correlation (correlate/define_auto_correlate.h:8-101): one CTA
// per station, sources strided over threads, warp-shuffle then smem reduce.
template <typename T, bool MATRIX>
__global__ void acorr_kernel(int num_src, int num_st, int offset_out,
        const T* __restrict__ jones, const T* __restrict__ I,
        const T* __restrict__ Q, const T* __restrict__ U,
        const T* __restrict__ V, T* vis)
{
    constexpr int NC = MATRIX ? 8 : 1;
    __shared__ double red[32][NC];
    const int st = blockIdx.x;
    double sum[NC];
#pragma unroll
    for (int k = 0; k < NC; ++k) sum[k] = 0;
    for (int s = threadIdx.x; s < num_src; s += blockDim.x)
    {
        if (MATRIX)
        {
            const T* jp = jones + 8 * ((size_t) st * num_src + s);
            const Cx<T> a{jp[0], jp[1]}, b{jp[2], jp[3]}, c{jp[4], jp[5]},
                    d{jp[6], jp[7]};
            const T i_ = I[s], q_ = Q[s];
            const Cx<T> uv{U[s], V[s]}, uvc{U[s], -V[s]};
            // M = J B
            Cx<T> t0 = cm(b, uvc), t1 = cm(d, uvc), t2 = cm(a, uv),
                    t3 = cm(c, uv);
            const Cx<T> ma{a.re * (i_ + q_) + t0.re, a.im * (i_ + q_) + t0.im};
            const Cx<T> mc{c.re * (i_ + q_) + t1.re, c.im * (i_ + q_) + t1.im};
            const Cx<T> mb{b.re * (i_ - q_) + t2.re, b.im * (i_ - q_) + t2.im};
            const Cx<T> md{d.re * (i_ - q_) + t3.re, d.im * (i_ - q_) + t3.im};
            // M J^H
            const Cx<T> X[4] = {ma, mb, mc, md}, Y[4] = {a, b, c, d};
            const int li[4] = {0, 0, 2, 2}, ri[4] = {0, 2, 0, 2};
#pragma unroll
            for (int k = 0; k < 4; ++k)
            {
                const Cx<T> x0 = X[li[k]], x1 = X[li[k] + 1];
                const Cx<T> y0 = Y[ri[k]], y1 = Y[ri[k] + 1];
                sum[2 * k] += x0.re * y0.re + x0.im * y0.im +
                        x1.re * y1.re + x1.im * y1.im;
                sum[2 * k + 1] += x0.im * y0.re - x0.re * y0.im +
                        x1.im * y1.re - x1.re * y1.im;
            }
        }
        else
        {
            const T* jp = jones + 2 * ((size_t) st * num_src + s);
            sum[0] += (jp[0] * jp[0] + jp[1] * jp[1]) * I[s];
        }
    }
#pragma unroll
    for (int k = 0; k < NC; ++k)
        for (int o = 16; o > 0; o >>= 1)
            sum[k] += __shfl_xor_sync(0xffffffffu, sum[k], o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
        for (int k = 0; k < NC; ++k) red[warp][k] = sum[k];
    __syncthreads();
    if (threadIdx.x == 0)
    {
        const int nw = blockDim.x >> 5;
        for (int w = 1; w < nw; ++w)
            for (int k = 0; k < NC; ++k) sum[k] += red[w][k];
        if (MATRIX)
        {
            sum[1] = sum[7] = 0;
            T* o = vis + 8 * (size_t) (st + offset_out);
            for (int k = 0; k < 8; ++k) o[k] = (T) ((double) o[k] + sum[k]);
        }
        else
        {
            T* o = vis + 2 * (size_t) (st + offset_out);
            o[0] = (T) ((double) o[0] + sum[0]);
        }
    }
}

// ---- beamforming weights (define_evaluate_element_weights_dft.h:3-16)
template <typename T>
__global__ void weights_kernel(int n, const T* x, const T* y, const T* z,
        const T* cable, T k, T x1, T y1, T z1, T* w)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // z or cable NULL: zero (a 2-D layout; no cable errors)
    const T p = k * (x[i] * x1 + y[i] * y1 + (z ? z[i] * z1 : (T) 0) +
            (cable ? cable[i] : (T) 0));
    T sn, cs;
    sincos(-p, &sn, &cs);
    w[2 * i] = cs;
    w[2 * i + 1] = sn;
}

// ---- station (u, v, w) (define_convert_ecef_to_station_uvw.h:3-29)
__global__ void uvw_kernel(int n, const double* x, const double* y,
        const double* z, double sh, double ch, double sd, double cd,
        int ignore_w, int off, double* u, double* v, double* w)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double xx = x[i], yy = y[i], zz = z[i];
    const double t = xx * ch - yy * sh;
    u[i + off] = xx * sh + yy * ch;
    v[i + off] = zz * cd - t * sd;
    w[i + off] = ignore_w ? 0.0 : zz * sd + t * cd;
}

template <typename T>
int jones_k(int num_src, const T* l, const T* m, const T* n, int num_st,
        const T* u, const T* v, const T* w, T k, const T* f, T fmin, T fmax,
        int ignore_w, T* jones, void* stream)
{
    if (num_src < 0 || num_st < 0) return OSKB_ERR_INVALID_ARGUMENT;
    if (num_src == 0 || num_st == 0) return 0;
    if (!l || !m || !n || !u || !v || !w || !f || !jones)
        return OSKB_ERR_INVALID_ARGUMENT;
    if (num_st > 65535) return OSKB_ERR_OUT_OF_RANGE;
    dim3 grid((num_src + 255) / 256, num_st);
    jones_k_kernel<T><<<grid, 256, 0, as_stream(stream)>>>(num_src, l, m, n,
            num_st, u, v, w, k, f, fmin, fmax, ignore_w,
            reinterpret_cast<typename vec2<T>::type*>(jones));
    return check_launch("evaluate_jones_K");
}

template <typename T>
int mem_mul(int kind, size_t off_a, size_t off_b, size_t off_c, size_t n,
        const T* a, const T* b, T* c, void* stream)
{
    if (n == 0) return 0;
    if (!a || !b || !c) return OSKB_ERR_INVALID_ARGUMENT;
    const int threads = 256, grid = grid_for(n, threads);
    cudaStream_t s = as_stream(stream);
    switch (kind)
    {
    case OSKB_MUL_RR_R:
        mem_mul_kernel<T, OSKB_MUL_RR_R><<<grid, threads, 0, s>>>(off_a,
                off_b, off_c, n, a, b, c); break;
    case OSKB_MUL_CC_C:
        mem_mul_kernel<T, OSKB_MUL_CC_C><<<grid, threads, 0, s>>>(off_a,
                off_b, off_c, n, a, b, c); break;
    case OSKB_MUL_CC_M:
        mem_mul_kernel<T, OSKB_MUL_CC_M><<<grid, threads, 0, s>>>(off_a,
                off_b, off_c, n, a, b, c); break;
    case OSKB_MUL_CM_M:
        mem_mul_kernel<T, OSKB_MUL_CM_M><<<grid, threads, 0, s>>>(off_a,
                off_b, off_c, n, a, b, c); break;
    case OSKB_MUL_MC_M:
        mem_mul_kernel<T, OSKB_MUL_MC_M><<<grid, threads, 0, s>>>(off_a,
                off_b, off_c, n, a, b, c); break;
    case OSKB_MUL_MM_M:
        mem_mul_kernel<T, OSKB_MUL_MM_M><<<grid, threads, 0, s>>>(off_a,
                off_b, off_c, n, a, b, c); break;
    default:
        return OSKB_ERR_BAD_DATA_TYPE;
    }
    return check_launch("mem_multiply");
}

template <typename T>
int acorr(int matrix, int num_src, int num_st, int off, const T* jones,
        const T* I, const T* Q, const T* U, const T* V, T* vis, void* stream)
{
    if (num_src < 0 || num_st < 0) return OSKB_ERR_INVALID_ARGUMENT;
    if (num_src == 0 || num_st == 0) return 0;
    if (!jones || !I || !vis || (matrix && (!Q || !U || !V)))
        return OSKB_ERR_INVALID_ARGUMENT;
    if (matrix)
        acorr_kernel<T, true><<<num_st, 256, 0, as_stream(stream)>>>(num_src,
                num_st, off, jones, I, Q, U, V, vis);
    else
        acorr_kernel<T, false><<<num_st, 256, 0, as_stream(stream)>>>(num_src,
                num_st, off, jones, I, Q, U, V, vis);
    return check_launch("auto_correlate");
}

template <typename T>
int weights(int n, const T* x, const T* y, const T* z, const T* cable, T k,
        T x1, T y1, T z1, T* w, void* stream)
{
    if (n < 0) return OSKB_ERR_INVALID_ARGUMENT;
    if (n == 0) return 0;
    if (!x || !y || !w) return OSKB_ERR_INVALID_ARGUMENT;
    weights_kernel<T><<<(n + 255) / 256, 256, 0, as_stream(stream)>>>(n, x,
            y, z, cable, k, x1, y1, z1, w);
    return check_launch("element_weights_dft");
}

}  // namespace
}  // namespace oskb

using namespace oskb;

extern "C" {

const char* oskb_version(void) { return "oskar_b200 0.1.0 (sm_100a)"; }
const char* oskb_last_error(void) { return oskb::g_last_error; }

int oskb_evaluate_jones_K_d(int num_sources, const double* l, const double* m,
        const double* n, int num_stations, const double* u, const double* v,
        const double* w, double wavenumber, const double* filter,
        double fmin, double fmax, int ignore_w, double* jones, void* stream)
{
    return jones_k<double>(num_sources, l, m, n, num_stations, u, v, w,
            wavenumber, filter, fmin, fmax, ignore_w, jones, stream);
}

int oskb_evaluate_jones_K_f(int num_sources, const float* l, const float* m,
        const float* n, int num_stations, const float* u, const float* v,
        const float* w, float wavenumber, const float* filter, float fmin,
        float fmax, int ignore_w, float* jones, void* stream)
{
    return jones_k<float>(num_sources, l, m, n, num_stations, u, v, w,
            wavenumber, filter, fmin, fmax, ignore_w, jones, stream);
}

int oskb_mem_multiply_d(int kind, size_t off_a, size_t off_b, size_t off_c,
        size_t n, const double* a, const double* b, double* c, void* stream)
{
    return mem_mul<double>(kind, off_a, off_b, off_c, n, a, b, c, stream);
}

int oskb_mem_multiply_f(int kind, size_t off_a, size_t off_b, size_t off_c,
        size_t n, const float* a, const float* b, float* c, void* stream)
{
    return mem_mul<float>(kind, off_a, off_b, off_c, n, a, b, c, stream);
}

int oskb_auto_correlate_d(int matrix, int num_sources, int num_stations,
        int offset_out, const double* jones, const double* I,
        const double* Q, const double* U, const double* V, double* vis,
        void* stream)
{
    return acorr<double>(matrix, num_sources, num_stations, offset_out,
            jones, I, Q, U, V, vis, stream);
}

int oskb_auto_correlate_f(int matrix, int num_sources, int num_stations,
        int offset_out, const float* jones, const float* I, const float* Q,
        const float* U, const float* V, float* vis, void* stream)
{
    return acorr<float>(matrix, num_sources, num_stations, offset_out,
            jones, I, Q, U, V, vis, stream);
}

int oskb_evaluate_element_weights_dft_d(int n, const double* x,
        const double* y, const double* z, const double* cable, double k,
        double x1, double y1, double z1, double* w, void* stream)
{
    return weights<double>(n, x, y, z, cable, k, x1, y1, z1, w, stream);
}

int oskb_evaluate_element_weights_dft_f(int n, const float* x,
        const float* y, const float* z, const float* cable, float k,
        float x1, float y1, float z1, float* w, void* stream)
{
    return weights<float>(n, x, y, z, cable, k, x1, y1, z1, w, stream);
}

int oskb_convert_ecef_to_station_uvw_d(int num_stations, const double* x,
        const double* y, const double* z, double ra0_rad, double dec0_rad,
        double gast, int ignore_w, int offset_out, double* u, double* v,
        double* w, void* stream)
{
    if (num_stations < 0) return OSKB_ERR_INVALID_ARGUMENT;
    if (num_stations == 0) return 0;
    if (!x || !y || !z || !u || !v || !w) return OSKB_ERR_INVALID_ARGUMENT;
    const double ha0 = gast - ra0_rad;
    uvw_kernel<<<(num_stations + 127) / 128, 128, 0, as_stream(stream)>>>(
            num_stations, x, y, z, sin(ha0), cos(ha0), sin(dec0_rad),
            cos(dec0_rad), ignore_w, offset_out, u, v, w);
    return check_launch("ecef_to_station_uvw");
}

}  // extern "C"

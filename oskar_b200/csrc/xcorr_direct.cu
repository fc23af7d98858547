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
#include <stdlib.h>
#include <string.h>

#include "common.cuh"

namespace oskb {
namespace {

constexpr int kTile = 32;      // stations per block edge
constexpr int kChunk = 8;      // sources per shared-memory chunk
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
    // Source slices: CTA (tile, y) sums sources [y * slice_len,
    // (y + 1) * slice_len). With more than one slice, each CTA writes its
    // sums to partial[y][baseline][comp] and reduce_partials adds them to
    // vis in slice order (deterministic); with one slice it adds to vis.
    int slice_len;
    double* partial;
};

template <typename T, bool MATRIX>
struct Staging
{
    // Bytes of one Jones element and the cp.async copy size used for it.
    static constexpr int ELEM = (int) sizeof(T) * (MATRIX ? 8 : 2);
    static constexpr int COPY = ELEM >= 16 ? 16 : ELEM;
    static constexpr int PIECES = ELEM / COPY;
};

// Per-source arrays staged with each chunk.
enum SrcArr { kI = 0, kQ, kU, kV, kL, kM, kN, kGa, kGb, kGc, kNumSrcArr };

template <typename T, bool MATRIX>
struct Smem
{
    typedef typename vec2<T>::type T2;
    typedef Staging<T, MATRIX> G;
    static constexpr int NCOMP = MATRIX ? 4 : 1;
    // Raw Jones of the next chunk, landed by cp.async:
    // [block][piece][source][station] x COPY bytes, so that a warp's
    // transform reads consecutive stations (conflict-free).
    __align__(16) unsigned char raw[2][G::PIECES][kChunk][kTile][G::COPY];
    T raw_src[kNumSrcArr][kChunk];
    // Factors of the current chunk: [comp][source][station] complex for the
    // row (p) and column (q) blocks.
    T2 row[NCOMP][kChunk][kTile];
    T2 col[NCOMP][kChunk][kTile];
    T ph_row[kChunk][kTile], ph_col[kChunk][kTile];  // bandwidth phases
    T ps_row[kChunk][kTile], ps_col[kChunk][kTile];  // time-smearing phases
    T ga[kChunk], gb[kChunk], gc[kChunk];
    // Per-station phase terms, loaded once per CTA: u, v, w (bandwidth)
    // and the rotated x, y pair (time smearing).
    double st_terms[2][kTile][5];
};

__device__ __forceinline__ void cp_async(void* smem, const void* gmem,
        bool in_range, int bytes)
{
    const unsigned s = (unsigned) __cvta_generic_to_shared(smem);
    const int src = in_range ? bytes : 0;  // 0: zero-fill, nothing read
    if (bytes == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n"
                :: "r"(s), "l"(gmem), "r"(src) : "memory");
    else if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n"
                :: "r"(s), "l"(gmem), "r"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n"
                :: "r"(s), "l"(gmem), "r"(src) : "memory");
}

__device__ __forceinline__ void cp_async_commit()
{
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

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

// Issues the cp.async copies of one chunk (sources [s0, min(s0 + kChunk,
// src_end))) of both station blocks and of the per-source arrays; entries
// outside the stations or sources are zero-filled without a global read.
template <typename T, bool MATRIX, bool GAUSS, bool LMN>
__device__ __forceinline__ void issue_chunk(Smem<T, MATRIX>& sm,
        const XcorrParams<T>& prm, int p0, int q0, int s0, int src_end)
{
    typedef Staging<T, MATRIX> G;
    const int tid = threadIdx.x, N = prm.num_st;
    const unsigned char* jb = reinterpret_cast<const unsigned char*>(prm.jones);
    // Thread mapping: 8 stations x PIECES x 4 station groups x sources x
    // blocks, so a warp reads whole elements of 8 stations and writes 8
    // consecutive station slots per piece.
    constexpr int total = 2 * G::PIECES * kChunk * kTile;
    for (int it = tid; it < total; it += kThreads)
    {
        const int a = it & 7;
        const int pc = (it >> 3) % G::PIECES;
        const int rest = (it >> 3) / G::PIECES;
        const int stl = a + 8 * (rest & 3);
        const int rest2 = rest >> 2;
        const int sl = rest2 % kChunk, blk = rest2 / kChunk;
        const int st = (blk ? q0 : p0) + stl, s = s0 + sl;
        const bool in = st < N && s < src_end;
        const unsigned char* src = in ? jb + ((size_t) st * prm.num_src + s) *
                G::ELEM + pc * G::COPY : jb;
        cp_async(sm.raw[blk][pc][sl][stl], src, in, G::COPY);
    }
    // Per-source arrays: only those this variant reads.
    const T* arrs[kNumSrcArr] = {prm.I, prm.Q, prm.U, prm.V, prm.l, prm.m,
            prm.n, prm.a, prm.b, prm.c};
    for (int it = tid; it < kNumSrcArr * kChunk; it += kThreads)
    {
        const int k = it / kChunk, sl = it % kChunk;
        const bool want = (k == kI) || (MATRIX && k <= kV) ||
                (LMN && k >= kL && k <= kN) || (GAUSS && k >= kGa);
        if (!want) continue;
        const int s = s0 + sl;
        const bool in = s < src_end;
        cp_async(&sm.raw_src[k][sl], in ? arrs[k] + s : arrs[kI], in,
                (int) sizeof(T));
    }
    cp_async_commit();
}

template <typename T, bool MATRIX, bool GAUSS, bool BW, bool TS, bool CASA>
__global__ void __launch_bounds__(kThreads,
        (sizeof(T) == 8 && !(MATRIX && (GAUSS || BW || TS))) ? 2 : 1)
xcorr_direct_kernel(const XcorrParams<T> prm)
{
    typedef typename vec2<T>::type T2;
    typedef Smem<T, MATRIX> S;
    typedef Staging<T, MATRIX> G;
    constexpr int NC = S::NCOMP;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    S& sm = *reinterpret_cast<S*>(smem_raw);

    int bp, bq;
    tri_block(blockIdx.x, bp, bq);
    const int p0 = bp * kTile, q0 = bq * kTile;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int N = prm.num_st;
    const int src_begin = blockIdx.y * prm.slice_len;
    const int src_end = min(prm.num_src, src_begin + prm.slice_len);

    // First chunk in flight while the per-baseline terms are set up.
    if (src_begin < src_end)
        issue_chunk<T, MATRIX, GAUSS, BW || TS>(sm, prm, p0, q0, src_begin,
                src_end);

    if (BW || TS)
    {
        for (int it = tid; it < 2 * kTile; it += kThreads)
        {
            const int blk = it / kTile, stl = it % kTile;
            const int st = (blk ? q0 : p0) + stl;
            double* t = sm.st_terms[blk][stl];
            t[0] = t[1] = t[2] = t[3] = t[4] = 0;
            if (st < N)
            {
                t[0] = prm.st_u[st]; t[1] = prm.st_v[st]; t[2] = prm.st_w[st];
                if (TS)
                {
                    const double x = prm.st_x[st], y = prm.st_y[st];
                    t[3] = x * prm.c_ha - y * prm.s_ha;
                    t[4] = x * prm.s_ha + y * prm.c_ha;
                }
            }
        }
    }

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

    for (int s0 = src_begin; s0 < src_end; s0 += kChunk)
    {
        const int ns = min(kChunk, src_end - s0);
        cp_async_wait_all();
        __syncthreads();  // chunk landed; previous chunk's factors consumed

        // ---- transform the raw chunk into the factors (shared to shared)
        for (int it = tid; it < 2 * kTile * kChunk; it += kThreads)
        {
            const int blk = it / (kTile * kChunk);
            const int rem = it - blk * (kTile * kChunk);
            const int stl = rem % kTile, sl = rem / kTile;
            T v[2 * NC];
#pragma unroll
            for (int pc = 0; pc < G::PIECES; ++pc)
            {
                constexpr int PER = G::COPY / (int) sizeof(T);
                if constexpr (G::COPY == 16)
                {
                    const uint4 u = *reinterpret_cast<const uint4*>(
                            sm.raw[blk][pc][sl][stl]);
                    memcpy(&v[pc * PER], &u, 16);
                }
                else
                {
                    const uint2 u = *reinterpret_cast<const uint2*>(
                            sm.raw[blk][pc][sl][stl]);
                    memcpy(&v[pc * PER], &u, 8);
                }
            }
            // Left factor (J B, or I J) lives in the row block unless CASA.
            const bool left = (blk == 0) != CASA;
            T2 (*dst)[kChunk][kTile] = blk ? sm.col : sm.row;
            if (MATRIX)
            {
                Mat2<T> J;
                J.a = T2{v[0], v[1]}; J.b = T2{v[2], v[3]};
                J.c = T2{v[4], v[5]}; J.d = T2{v[6], v[7]};
                if (left)
                {
                    const T I = sm.raw_src[kI][sl], Q = sm.raw_src[kQ][sl];
                    const T2 buv = T2{sm.raw_src[kU][sl], sm.raw_src[kV][sl]};
                    const T2 buvc = T2{buv.x, -buv.y};
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
                T2 J = T2{v[0], v[1]};
                if (left)
                {
                    const T I = sm.raw_src[kI][sl];
                    J.x *= I; J.y *= I;
                }
                dst[0][sl][stl] = J;
            }
            if (BW || TS)
            {
                // Per-station source phases (phi_p - phi_q is the
                // reference's baseline argument), in FP64.
                const double* t = sm.st_terms[blk][stl];
                const double l = sm.raw_src[kL][sl], m = sm.raw_src[kM][sl];
                const double n1 = (double) sm.raw_src[kN][sl] - 1.0;
                T ph = 0, ps = 0;
                if (BW)
                    ph = (T) ((t[0] * l + t[1] * m + t[2] * n1) *
                            prm.bw_scale);
                if (TS)
                    ps = (T) ((t[3] * l + t[4] * (prm.s_dec * m -
                            prm.c_dec * n1)) * prm.ts_scale);
                if (blk) { sm.ph_col[sl][stl] = ph; sm.ps_col[sl][stl] = ps; }
                else { sm.ph_row[sl][stl] = ph; sm.ps_row[sl][stl] = ps; }
            }
        }
        if (GAUSS && tid < kChunk)
        {
            sm.ga[tid] = sm.raw_src[kGa][tid];
            sm.gb[tid] = sm.raw_src[kGb][tid];
            sm.gc[tid] = sm.raw_src[kGc][tid];
        }
        __syncthreads();  // factors ready; the raw buffer is free

        // ---- next chunk's copies overlap this chunk's arithmetic
        if (s0 + kChunk < src_end)
            issue_chunk<T, MATRIX, GAUSS, BW || TS>(sm, prm, p0, q0,
                    s0 + kChunk, src_end);

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
            if constexpr (!(GAUSS || BW || TS))
            {
                // No smearing: 32 FMAs per source-baseline (matrix), i.e.
                // exactly the 64 algorithmic flops, accumulated straight
                // into the sums. Term-major order: each pass adds one term
                // to all 32 sums of the thread, so consecutive FMAs never
                // depend on each other.
#pragma unroll
                for (int u = 0; u < (MATRIX ? 2 : 1); ++u)
#pragma unroll
                    for (int i = 0; i < 2; ++i)
#pragma unroll
                        for (int j = 0; j < 2; ++j)
                        {
                            const T2* L = CASA ? C[j] : R[i];
                            const T2* Rt = CASA ? R[i] : C[j];
                            T* o = part[i][j];
#pragma unroll
                            for (int e = 0; e < NC; ++e)
                            {
                                // element e = (r, c) of the 2x2 output:
                                // sum_u L[2r + u] conj(Rt[2c + u])
                                const T2 x = L[MATRIX ? 2 * (e >> 1) + u : 0];
                                const T2 y = Rt[MATRIX ? 2 * (e & 1) + u : 0];
                                o[2 * e] = fma(x.x, y.x, o[2 * e]);
                                o[2 * e + 1] = fma(x.y, y.x, o[2 * e + 1]);
                            }
#pragma unroll
                            for (int e = 0; e < NC; ++e)
                            {
                                const T2 x = L[MATRIX ? 2 * (e >> 1) + u : 0];
                                const T2 y = Rt[MATRIX ? 2 * (e & 1) + u : 0];
                                o[2 * e] = fma(x.y, y.y, o[2 * e]);
                                o[2 * e + 1] = fma(-x.x, y.y, o[2 * e + 1]);
                            }
                        }
            }
            else
            {
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j)
                {
                    // L * conj-transpose(Rt): L = left factor, Rt = right.
                    const T2* L = CASA ? C[j] : R[i];
                    const T2* Rt = CASA ? R[i] : C[j];
                    T* o = part[i][j];
                    {
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
#pragma unroll
                        for (int k = 0; k < 2 * NC; ++k)
                            o[k] = fma(t[k], smear[i][j], o[k]);
                    }
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
    }

    // ---- write out: each baseline is owned by exactly one thread
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
        {
            const int p = p0 + ty + 16 * i, q = q0 + tx + 16 * j;
            if (p >= N || q >= p) continue;
            const long long bl = baseline_index(N, p, q);
            if (prm.partial)
            {
                // Every baseline of the slice is written (zero where the uv
                // filter drops it), so the reduction reads no stale data.
                const long long nbl = (long long) N * (N - 1) / 2;
                double* out = prm.partial + (size_t) (2 * NC) *
                        (size_t) (blockIdx.y * nbl + bl);
#pragma unroll
                for (int k = 0; k < 2 * NC; ++k)
                    out[k] = !valid[i][j] ? 0.0 : (sizeof(T) == 4) ?
                            acc[i][j][k] : (double) part[i][j][k];
                continue;
            }
            if (!valid[i][j]) continue;
            T* out = prm.vis + (size_t) (2 * NC) *
                    (size_t) (bl + prm.offset_out);
#pragma unroll
            for (int k = 0; k < 2 * NC; ++k)
            {
                const double v = (sizeof(T) == 4) ? acc[i][j][k]
                                                  : (double) part[i][j][k];
                out[k] = (T) ((double) out[k] + v);
            }
        }
}

// Adds the slices' partial sums to the visibilities, in slice order.
template <typename T>
__global__ void __launch_bounds__(256)
reduce_partials_kernel(const double* __restrict__ partial, int num_slices,
        long long n, long long offset, T* __restrict__ vis)
{
    const long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if (i >= n) return;
    double sum = 0;
    for (int y = 0; y < num_slices; ++y) sum += partial[(size_t) y * n + i];
    T* out = vis + offset + i;
    *out = (T) ((double) *out + sum);
}

int num_sms()
{
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev)
            != cudaSuccess || n <= 0)
        return 148;
    return n;
}

template <typename T, bool MATRIX, bool GAUSS, bool BW, bool TS>
void launch_casa(bool casa, const XcorrParams<T>& p, dim3 grid,
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
int xcorr_dispatch(bool casa, bool gauss, XcorrParams<T> p,
        bool bw, bool ts, cudaStream_t stream)
{
    if (p.num_st < 2 || p.num_src <= 0) return 0;
    // The staging copies whole Jones elements in COPY-byte pieces, so the
    // Jones array must be aligned to COPY bytes (any cudaMalloc'd array,
    // or an offset into one by whole elements, is).
    if ((uintptr_t) p.jones % Staging<T, MATRIX>::COPY != 0)
        return OSKB_ERR_INVALID_ARGUMENT;
    const int nb = (p.num_st + kTile - 1) / kTile;
    const int tiles = nb * (nb + 1) / 2;
    // Split the sources into slices so that about four waves of two CTAs
    // per SM are in flight, each slice at least 64 sources long.
    const int max_slices = (p.num_src + 8 * kChunk - 1) / (8 * kChunk);
    int slices = (8 * num_sms() + tiles - 1) / tiles;
    slices = max(1, min(slices, max_slices));
    if (const char* e = getenv("OSKB_XCORR_SLICES")) slices = max(1, atoi(e));
    int slice_len = (p.num_src + slices - 1) / slices;
    slice_len = (slice_len + kChunk - 1) / kChunk * kChunk;
    slices = (p.num_src + slice_len - 1) / slice_len;
    constexpr int ncomp2 = MATRIX ? 8 : 2;
    const long long nbl = (long long) p.num_st * (p.num_st - 1) / 2;
    p.slice_len = slice_len;
    p.partial = nullptr;
    if (slices > 1)
    {
        const size_t bytes = (size_t) slices * nbl * ncomp2 * sizeof(double);
        if (cudaMallocAsync((void**) &p.partial, bytes, stream) !=
                cudaSuccess)
        {
            cudaGetLastError();  // no room for partials: one slice
            p.partial = nullptr;
            slices = 1;
            p.slice_len = p.num_src;
        }
    }
    const dim3 grid(tiles, slices);
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
    int err = check_launch("xcorr_direct");
    if (p.partial)
    {
        const long long n = nbl * ncomp2;
        if (!err)
        {
            reduce_partials_kernel<T><<<(unsigned) ((n + 255) / 256), 256, 0,
                    stream>>>(p.partial, slices, n,
                    (long long) p.offset_out * ncomp2, p.vis);
            err = check_launch("xcorr_direct reduce");
        }
        cudaFreeAsync(p.partial, stream);
    }
    return err;
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

// Direct cross-correlation kernel (all source types and smearing modes), and
// its batched form over whole (dump x channel) blocks.
//
// Replaces the reference's warp-per-baseline kernel
// (oskar/correlate/src/oskar_cross_correlate_cuda.cu:45-224) with a
// register-tiled form: one CTA owns a 32 x 32 block of stations (rows p,
// columns q, lower triangle p > q as in the reference), each thread a 2 x 2
// group of baselines. Sources are staged through shared memory in chunks of
// 8: cp.async lands the next chunk's raw Jones while the current chunk is
// correlated, then a shared-to-shared transform forms the "left" factor J B
// (or I J in scalar mode) and the "right" factor J once per station-source
// for the whole CTA, so the per source-baseline work is the 8 complex MACs
// of (J_p B) J_q^H. Smearing arguments are per-station source phases
// (phi_p - phi_q), which turns the reference's three multiply-adds per
// source-baseline into one subtraction. FP64 mode accumulates in FP64; FP32
// mode sums each chunk in FP32 and the chunk sums in FP64.
//
// Work items. A launch covers items (dump t, channel c, station tile, source
// slice); each CTA loops over items. The single-call entry points are one
// dump and one channel with the sources split into slices (partial sums
// reduced in slice order); the block entry point (oskb_correlate_block_direct)
// covers every (t, c) of a block in one persistent launch with one slice per
// item, and forms J = K(t, c) E in the staging transform, so neither K nor J
// is ever written to memory (the reference's sim_baselines,
// oskar/interferometer/src/oskar_interferometer_run_block.c:156-336, runs
// K, join and correlate as separate launches per (t, chunk, c)).
#include <stdlib.h>
#include <string.h>

#include <mutex>

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
    int src_stride;  // sources per station row of jones (= num_src)
    const T* jones;  // J [station][source], or E when K is fused
    const T *I, *Q, *U, *V, *l, *m, *n, *a, *b, *c;
    // Station (u, v, w) metres of dump t at st_u + t * uvw_time_stride
    // (v and w follow at +num_st and +2 num_st in block mode).
    const T *st_u, *st_v, *st_w, *st_x, *st_y;
    long long uvw_time_stride;
    double uv_min, uv_max;  // wavelengths (single call) or metres (block)
    int uv_filter_in_metres;
    double inv_wavelength;            // single call
    const double* inv_wavelength_c;   // block: [channel]
    double bw_scale;  // pi * frac_bandwidth * inv_wavelength (= pi bw / c0)
    double ts_base;   // pi * omega_earth * time_int_sec (x inv_wavelength)
    double gha0;                      // single call
    const double* gha0_t;             // block: [dump]
    double s_dec, c_dec;
    T* vis;
    // Items: num_times x num_channels x tiles x slices, in that nesting
    // (slices fastest). Source slice y covers [y * slice_len,
    // (y + 1) * slice_len). With more than one slice (single call only),
    // each CTA writes its sums to partial[y][baseline][comp] and
    // reduce_partials adds them to vis in slice order (deterministic).
    int num_times, num_channels, tiles, slices, slice_len;
    int tile_major;  // item order: tile outermost instead of innermost
    double* partial;
    // Fused Jones K (block mode): J = K E, K = exp(i 2 pi / lambda (u l +
    // v m + w (n - 1))), zero where I is outside (filter_min, filter_max].
    long long e_time_stride;  // E of dump t at jones + t * e_time_stride
    double filter_min, filter_max;
    // Brightness per channel (block mode): I, Q, U, V of channel c at
    // + c * flux_channel_stride (0: the same for every channel).
    long long flux_channel_stride;
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
    // Per-station smearing phases phi and their sin, cos:
    // [block][phi, sin, cos][source][station], bandwidth (ph) and time (ps).
    T ph[2][3][kChunk][kTile];
    T ps[2][3][kChunk][kTile];
    T ga[kChunk], gb[kChunk], gc[kChunk];
    // Per-station terms, loaded once per item: u, v, w (bandwidth phase and
    // fused K) and the rotated x, y pair (time smearing).
    T st_uvw[2][kTile][3];
    double st_xy[2][kTile][2];
};

// Per-item constants.
struct ItemCtx
{
    int t, c, p0, q0, src_begin, src_end;
    double inv_wavelength, ts_scale, s_ha, c_ha;
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

// Waits until at most N of this thread's cp.async groups are pending.
template <int N>
__device__ __forceinline__ void cp_async_wait_group()
{
    asm volatile("cp.async.wait_group %0;\n" :: "n"(N) : "memory");
}

// sinc(phi_p - phi_q) = sin(phi_p - phi_q) / (phi_p - phi_q), the
// reference's smearing factor (define_cross_correlate.h:16-32), from the
// per-station sin and cos: sin(a - b) = sin a cos b - cos a sin b. Where the
// difference d is small the identity loses relative accuracy (its absolute
// error is a few ulp of 1), so below |d| = tau the Taylor series of sinc is
// summed instead, 1 - d^2/6 + d^4/120 - d^6/5040 + d^8/362880, whose
// truncation error d^10/39916800 is below 1e-20 (FP64, tau = 0.05) and
// 3e-11 (FP32, tau = 0.5); above tau the identity's relative error is below
// ~1e-14 (FP64) and ~1e-6 (FP32).
template <typename T>
__device__ __forceinline__ T sinc_series(T d)
{
    const T d2 = d * d;
    return (T) 1 + d2 * ((T) (-1.0 / 6) + d2 * ((T) (1.0 / 120) +
            d2 * ((T) (-1.0 / 5040) + d2 * (T) (1.0 / 362880))));
}

// 1 / d for |d| >= 0.05 (FP64): the hardware's reciprocal approximation
// refined by two steps of Newton's method for 1 / d, y' = y + y (1 - d y),
// each of which squares the relative error (from ~2^-23 to below 2^-52,
// then rounding). A short dependent chain instead of the IEEE division's;
// the quotient is within an ulp or two of the correctly rounded one.
__device__ __forceinline__ double recip_newton(double d)
{
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(d));
    double e = fma(-d, y, 1.0);
    y = fma(y, e, y);
    e = fma(-d, y, 1.0);
    return fma(y, e, y);
}

template <typename T>
__device__ __forceinline__ T sinc_diff(T pa, T sa, T ca, T pb, T sb, T cb)
{
    const T d = pa - pb;
    const T tau = sizeof(T) == 8 ? (T) 0.05 : (T) 0.5;
    if constexpr (sizeof(T) == 8)
    {
        // both forms, then a select: no divergence between the lanes of a
        // warp whose baselines fall on either side of tau
        const bool small = fabs(d) < tau;
        const T by_identity = (sa * cb - ca * sb) *
                recip_newton(small ? (T) 1 : d);
        const T by_series = sinc_series(d);
        return small ? by_series : by_identity;
    }
    else
    {
        if (fabs(d) < tau) return sinc_series(d);
        return (sa * cb - ca * sb) / d;
    }
}

// The same factor as a numerator and a denominator (sin d, d), or
// (series, 1) below tau, so that the bandwidth and time factors of one
// source-baseline share a single division: used in FP32, where it is
// faster (in FP64 the two divisions measured faster than the shared one).
template <typename T>
__device__ __forceinline__ void sinc_parts(T pa, T sa, T ca, T pb, T sb,
        T cb, T& num, T& den)
{
    const T d = pa - pb;
    const T tau = sizeof(T) == 8 ? (T) 0.05 : (T) 0.5;
    // both forms, then a select (no divergence within a warp)
    const bool small = fabs(d) < tau;
    const T by_series = sinc_series(d);
    num = small ? by_series : sa * cb - ca * sb;
    den = small ? (T) 1 : d;
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
// jsrc: the Jones (or, fused, E) array of this item; NULL for identity E.
template <typename T, bool MATRIX, bool GAUSS, bool LMN>
__device__ __forceinline__ void issue_chunk(Smem<T, MATRIX>& sm,
        const XcorrParams<T>& prm, const T* jsrc, const ItemCtx& it_ctx,
        int s0)
{
    typedef Staging<T, MATRIX> G;
    const int tid = threadIdx.x, N = prm.num_st;
    const int src_end = it_ctx.src_end;
    if (jsrc)
    {
        const unsigned char* jb = reinterpret_cast<const unsigned char*>(jsrc);
        // Thread mapping: 8 stations x PIECES x 4 station groups x sources
        // x blocks, so a warp reads whole elements of 8 stations and writes
        // 8 consecutive station slots per piece.
        constexpr int total = 2 * G::PIECES * kChunk * kTile;
        for (int it = tid; it < total; it += kThreads)
        {
            const int a = it & 7;
            const int pc = (it >> 3) % G::PIECES;
            const int rest = (it >> 3) / G::PIECES;
            const int stl = a + 8 * (rest & 3);
            const int rest2 = rest >> 2;
            const int sl = rest2 % kChunk, blk = rest2 / kChunk;
            const int st = (blk ? it_ctx.q0 : it_ctx.p0) + stl, s = s0 + sl;
            const bool in = st < N && s < src_end;
            const unsigned char* src = in ? jb + ((size_t) st *
                    prm.src_stride + s) * G::ELEM + pc * G::COPY : jb;
            cp_async(sm.raw[blk][pc][sl][stl], src, in, G::COPY);
        }
    }
    // Per-source arrays: only those this variant reads. (A select chain,
    // not an array of pointers, which would live in local memory.)
    for (int it = tid; it < kNumSrcArr * kChunk; it += kThreads)
    {
        const int k = it / kChunk, sl = it % kChunk;
        const bool want = (k == kI) || (MATRIX && k <= kV) ||
                (LMN && k >= kL && k <= kN) || (GAUSS && k >= kGa);
        if (!want) continue;
        const T* arr = k == kI ? prm.I : k == kQ ? prm.Q : k == kU ? prm.U :
                k == kV ? prm.V : k == kL ? prm.l : k == kM ? prm.m :
                k == kN ? prm.n : k == kGa ? prm.a : k == kGb ? prm.b :
                prm.c;
        const int s = s0 + sl;
        const bool in = s < src_end;
        const long long off = k <= kV ? it_ctx.c * prm.flux_channel_stride :
                0;
        cp_async(&sm.raw_src[k][sl], in ? arr + off + s : prm.I, in,
                (int) sizeof(T));
    }
    cp_async_commit();
}

template <typename T, bool MATRIX, bool GAUSS, bool BW, bool TS, bool CASA,
        bool FUSED>
__global__ void __launch_bounds__(kThreads,
        (sizeof(T) == 8 && !FUSED && (MATRIX ? !(GAUSS || BW || TS) : !GAUSS))
        ? 2 : 1)
xcorr_direct_kernel(const XcorrParams<T> prm)
{
    typedef typename vec2<T>::type T2;
    typedef Smem<T, MATRIX> S;
    typedef Staging<T, MATRIX> G;
    constexpr int NC = S::NCOMP;
    constexpr bool LMN = BW || TS || FUSED;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    S& sm = *reinterpret_cast<S*>(smem_raw);
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int N = prm.num_st;
    const long long nbl = (long long) N * (N - 1) / 2;
    const int num_items = prm.num_times * prm.num_channels * prm.tiles *
            prm.slices;

    for (int item = blockIdx.x; item < num_items; item += gridDim.x)
    {
    // ---- item: (dump, channel, station tile, source slice)
    ItemCtx ctx;
    int r = item;
    const int slice = r % prm.slices; r /= prm.slices;
    int tile;
    if (prm.tile_major)
    {
        // Consecutive items share a station tile (its E rows stay in L2).
        const int tc = r % (prm.num_times * prm.num_channels);
        tile = r / (prm.num_times * prm.num_channels);
        ctx.c = tc % prm.num_channels;
        ctx.t = tc / prm.num_channels;
    }
    else
    {
        tile = r % prm.tiles;
        r /= prm.tiles;
        ctx.c = r % prm.num_channels;
        ctx.t = r / prm.num_channels;
    }
    {
        int bp, bq;
        tri_block(tile, bp, bq);
        ctx.p0 = bp * kTile;
        ctx.q0 = bq * kTile;
    }
    ctx.src_begin = slice * prm.slice_len;
    ctx.src_end = min(prm.num_src, ctx.src_begin + prm.slice_len);
    ctx.inv_wavelength = prm.inv_wavelength_c ?
            prm.inv_wavelength_c[ctx.c] : prm.inv_wavelength;
    ctx.ts_scale = prm.ts_base * ctx.inv_wavelength;
    ctx.s_ha = ctx.c_ha = 0;
    if (TS) sincos(prm.gha0_t ? prm.gha0_t[ctx.t] : prm.gha0, &ctx.s_ha,
            &ctx.c_ha);
    const T* su = prm.st_u + ctx.t * prm.uvw_time_stride;
    const T* sv = prm.st_v + ctx.t * prm.uvw_time_stride;
    const T* sw = prm.st_w + ctx.t * prm.uvw_time_stride;
    const T* jsrc = !FUSED ? prm.jones : (prm.jones ?
            prm.jones + ctx.t * prm.e_time_stride : nullptr);
    const T wavenumber = (T) (2.0 * kPi * ctx.inv_wavelength);
    const double uv_scale = prm.uv_filter_in_metres ? ctx.inv_wavelength :
            1.0;
    const T uv_lo = (T) (prm.uv_min * uv_scale);
    const T uv_hi = (T) (prm.uv_max * uv_scale);

    __syncthreads();  // the previous item is done with shared memory
    // First chunk in flight while the per-station and baseline terms are
    // set up.
    if (ctx.src_begin < ctx.src_end)
        issue_chunk<T, MATRIX, GAUSS, LMN>(sm, prm, jsrc, ctx,
                ctx.src_begin);

    if (LMN)
    {
        for (int it = tid; it < 2 * kTile; it += kThreads)
        {
            const int blk = it / kTile, stl = it % kTile;
            const int st = (blk ? ctx.q0 : ctx.p0) + stl;
            T* u = sm.st_uvw[blk][stl];
            double* xy = sm.st_xy[blk][stl];
            u[0] = u[1] = u[2] = 0;
            xy[0] = xy[1] = 0;
            if (st < N)
            {
                u[0] = su[st]; u[1] = sv[st]; u[2] = sw[st];
                if (TS)
                {
                    const double x = prm.st_x[st], y = prm.st_y[st];
                    xy[0] = x * ctx.c_ha - y * ctx.s_ha;
                    xy[1] = x * ctx.s_ha + y * ctx.c_ha;
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
            const int p = ctx.p0 + ty + 16 * i, q = ctx.q0 + tx + 16 * j;
            bool ok = (p < N) && (q < p);
            T uu = 0, vv = 0;
            if (ok)
            {
                uu = (su[p] - su[q]) * (T) ctx.inv_wavelength;
                vv = (sv[p] - sv[q]) * (T) ctx.inv_wavelength;
                const T len = sqrt(uu * uu + vv * vv);
                ok = !(len < uv_lo || len > uv_hi);
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

    for (int s0 = ctx.src_begin; s0 < ctx.src_end; s0 += kChunk)
    {
        const int ns = min(kChunk, ctx.src_end - s0);
        cp_async_wait_all();
        __syncthreads();  // chunk landed; previous chunk's factors consumed

        // ---- transform the raw chunk into the factors (shared to shared)
        for (int it = tid; it < 2 * kTile * kChunk; it += kThreads)
        {
            const int blk = it / (kTile * kChunk);
            const int rem = it - blk * (kTile * kChunk);
            const int stl = rem % kTile, sl = rem / kTile;
            T v[2 * NC];
            if (jsrc)
            {
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
            }
            else
            {
                // Identity E (fused mode without a station beam).
#pragma unroll
                for (int k = 0; k < 2 * NC; ++k) v[k] = (T) 0;
                v[0] = (T) 1;
                if (MATRIX) v[6] = (T) 1;
            }
            if (FUSED)
            {
                // J = K E with the reference's K
                // (oskar/interferometer/define_evaluate_jones_K.h:53-70).
                const T* u = sm.st_uvw[blk][stl];
                const T l = sm.raw_src[kL][sl], m = sm.raw_src[kM][sl];
                const T n1 = sm.raw_src[kN][sl] - (T) 1;
                const T flux = sm.raw_src[kI][sl];
                const T phase = (u[0] * l + u[1] * m + u[2] * n1) * wavenumber;
                T ks, kc;
                sincos(phase, &ks, &kc);
                if (!(sl < ns && flux > (T) prm.filter_min &&
                        flux <= (T) prm.filter_max))
                    ks = kc = (T) 0;
#pragma unroll
                for (int k = 0; k < NC; ++k)
                {
                    const T re = v[2 * k], im = v[2 * k + 1];
                    v[2 * k] = kc * re - ks * im;
                    v[2 * k + 1] = kc * im + ks * re;
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
                const T* u = sm.st_uvw[blk][stl];
                const double* xy = sm.st_xy[blk][stl];
                const double l = sm.raw_src[kL][sl], m = sm.raw_src[kM][sl];
                const double n1 = (double) sm.raw_src[kN][sl] - 1.0;
                T ph = 0, ps = 0;
                if (BW)
                    ph = (T) (((double) u[0] * l + (double) u[1] * m +
                            (double) u[2] * n1) * prm.bw_scale);
                if (TS)
                    ps = (T) ((xy[0] * l + xy[1] * (prm.s_dec * m -
                            prm.c_dec * n1)) * ctx.ts_scale);
                if (BW)
                {
                    T sn, cs;
                    sincos(ph, &sn, &cs);
                    sm.ph[blk][0][sl][stl] = ph;
                    sm.ph[blk][1][sl][stl] = sn;
                    sm.ph[blk][2][sl][stl] = cs;
                }
                if (TS)
                {
                    T sn, cs;
                    sincos(ps, &sn, &cs);
                    sm.ps[blk][0][sl][stl] = ps;
                    sm.ps[blk][1][sl][stl] = sn;
                    sm.ps[blk][2][sl][stl] = cs;
                }
            }
        }
        int g = 0;
        if (GAUSS && tid < kChunk)
        {
            sm.ga[tid] = sm.raw_src[kGa][tid];
            sm.gb[tid] = sm.raw_src[kGb][tid];
            sm.gc[tid] = sm.raw_src[kGc][tid];
            g = sm.ga[tid] != (T) 0 || sm.gb[tid] != (T) 0 ||
                    sm.gc[tid] != (T) 0;
        }
        // Factors ready; the raw buffer is free. A chunk of point sources
        // (a = b = c = 0, exp(-0) = 1 exactly) skips the Gaussian factor.
        const bool gauss_chunk = GAUSS && __syncthreads_or(g);
        if (!GAUSS) __syncthreads();

        // ---- next chunk's copies overlap this chunk's arithmetic
        if (s0 + kChunk < ctx.src_end)
            issue_chunk<T, MATRIX, GAUSS, LMN>(sm, prm, jsrc, ctx,
                    s0 + kChunk);
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
                    if (GAUSS && gauss_chunk)
                        f = exp(-(sm.ga[sl] * uu2[i][j] + sm.gb[sl] * uuvv[i][j]
                                + sm.gc[sl] * vv2[i][j]));
                    const int pr = ty + 16 * i, qc = tx + 16 * j;
                    if constexpr (sizeof(T) == 8)
                    {
                        if (BW)
                            f *= sinc_diff<T>(sm.ph[0][0][sl][pr],
                                    sm.ph[0][1][sl][pr], sm.ph[0][2][sl][pr],
                                    sm.ph[1][0][sl][qc], sm.ph[1][1][sl][qc],
                                    sm.ph[1][2][sl][qc]);
                        if (TS)
                            f *= sinc_diff<T>(sm.ps[0][0][sl][pr],
                                    sm.ps[0][1][sl][pr], sm.ps[0][2][sl][pr],
                                    sm.ps[1][0][sl][qc], sm.ps[1][1][sl][qc],
                                    sm.ps[1][2][sl][qc]);
                    }
                    else if (BW || TS)
                    {
                        T num = (T) 1, den = (T) 1;
                        if (BW)
                            sinc_parts<T>(sm.ph[0][0][sl][pr],
                                    sm.ph[0][1][sl][pr], sm.ph[0][2][sl][pr],
                                    sm.ph[1][0][sl][qc], sm.ph[1][1][sl][qc],
                                    sm.ph[1][2][sl][qc], num, den);
                        if (TS)
                        {
                            T n2, d2;
                            sinc_parts<T>(sm.ps[0][0][sl][pr],
                                    sm.ps[0][1][sl][pr], sm.ps[0][2][sl][pr],
                                    sm.ps[1][0][sl][qc], sm.ps[1][1][sl][qc],
                                    sm.ps[1][2][sl][qc], n2, d2);
                            num *= n2;
                            den *= d2;
                        }
                        // |den| >= 0.25 here (each factor's d is 1 or
                        // at least tau = 0.5), well inside the range where
                        // the fast division is accurate to 2 ulp
                        f *= __fdividef(num, den);
                    }
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
            const int p = ctx.p0 + ty + 16 * i, q = ctx.q0 + tx + 16 * j;
            if (p >= N || q >= p) continue;
            const long long bl = baseline_index(N, p, q);
            if (prm.partial)
            {
                // Every baseline of the slice is written (zero where the uv
                // filter drops it), so the reduction reads no stale data.
                double* out = prm.partial + (size_t) (2 * NC) * (size_t) (
                        ((long long) slice * prm.num_times * prm.num_channels
                        + (long long) ctx.t * prm.num_channels + ctx.c) *
                        nbl + bl);
#pragma unroll
                for (int k = 0; k < 2 * NC; ++k)
                    out[k] = !valid[i][j] ? 0.0 : (sizeof(T) == 4) ?
                            acc[i][j][k] : (double) part[i][j][k];
                continue;
            }
            if (!valid[i][j]) continue;
            // Block layout [dump][channel][baseline] (the reference's
            // oskar_VisBlock order, private_vis_block.h:33-57).
            T* out = prm.vis + (size_t) (2 * NC) * (size_t) (((long long)
                    ctx.t * prm.num_channels + ctx.c) * nbl + bl +
                    prm.offset_out);
#pragma unroll
            for (int k = 0; k < 2 * NC; ++k)
            {
                const double v = (sizeof(T) == 4) ? acc[i][j][k]
                                                  : (double) part[i][j][k];
                out[k] = (T) ((double) out[k] + v);
            }
        }
    }  // items
}

// ---------------------------------------------------------------------------
// FP64 tensor-core form: staging, transform and kernel.
// ---------------------------------------------------------------------------
// Fragment-ordered operands of one chunk: per block (rows, columns),
// kChunk / 2 k4 steps x 16 tiles of 8 rows x kFragTile doubles.
constexpr int kFragTile = 33;
constexpr int kFragK4 = (4 * kTile / 8) * kFragTile;
constexpr int kFragBlock = (kChunk / 2) * kFragK4;

// Shared memory of the FP64 tensor-core kernel: the raw Jones of two
// chunks and the fragment-ordered operands of two chunks, so that one
// chunk's products run while the next chunk is transformed (one barrier per
// chunk).
struct DmmaSmem
{
    // [buffer][block][piece][source][station] x 16 bytes
    __align__(16) unsigned char raw[2][2][4][kChunk][kTile][16];
    double src[2][kChunk][4];        // [buffer][source][I, Q, U, V]
    double frag[2][2 * kFragBlock];  // [buffer][rows block, columns block]
};

__device__ __forceinline__ void dmma_m8n8k4(double& d0, double& d1,
        double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 "
                 "{%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1) : "d"(a), "d"(b));
}

// Warp w stages and transforms source sl = w of every chunk, both blocks
// (64 elements): its copies land 8 stations x 4 pieces per instruction
// (whole 64-byte elements of 8 stations, coalesced; 4 x 128 contiguous
// bytes in shared memory), and its own cp.async wait plus __syncwarp make
// them visible to its lanes, so no block barrier is needed before the
// transform. Lanes 0-3 stage the source's I, Q, U, V.
__device__ __forceinline__ void dmma_issue(DmmaSmem& sm, int buf,
        const XcorrParams<double>& prm, const ItemCtx& ctx, int s0)
{
    const int lane = threadIdx.x & 31, sl = threadIdx.x >> 5;
    const unsigned char* jb = reinterpret_cast<const unsigned char*>(
            prm.jones);
    const int s = s0 + sl;
    const bool src_in = s < ctx.src_end;
    const int a = lane & 7, pc = lane >> 3;
#pragma unroll
    for (int i = 0; i < 8; ++i)
    {
        const int blk = i >> 2, stl = 8 * (i & 3) + a;
        const int st = (blk ? ctx.q0 : ctx.p0) + stl;
        const bool in = st < prm.num_st && src_in;
        const unsigned char* src = in ? jb + ((size_t) st * prm.src_stride +
                s) * 64 + 16 * pc : jb;
        cp_async(sm.raw[buf][blk][pc][sl][stl], src, in, 16);
    }
    if (lane < 4)
    {
        const double* arr = lane == 0 ? prm.I : lane == 1 ? prm.Q :
                lane == 2 ? prm.U : prm.V;
        cp_async(&sm.src[buf][sl][lane], src_in ? arr + s : prm.I, src_in,
                8);
    }
    cp_async_commit();
}

// Left factor J B (rows unless CASA) and right factor J of lane stl's two
// elements of the warp's source, written in fragment order: W entry (row
// r, k) of a block at frag[k / 4][r / 8][4 (r % 8) + k % 4] (tiles of 8 rows
// padded to kFragTile doubles against bank conflicts), so the mma.sync
// operand of lane (g, t) = (r % 8, k % 4) is one 8-byte load per lane (row
// r = 4 stl + 2 i + c, k = 2 sl + kk).
template <bool CASA>
__device__ __forceinline__ void dmma_transform(DmmaSmem& sm, int buf,
        int fbuf)
{
    typedef double2 T2;
    const int stl = threadIdx.x & 31, sl = threadIdx.x >> 5;
    __syncwarp();  // the warp's own copies, landed, visible to all lanes
#pragma unroll
    for (int blk = 0; blk < 2; ++blk)
    {
        Mat2<double> J;
        J.a = *reinterpret_cast<const T2*>(sm.raw[buf][blk][0][sl][stl]);
        J.b = *reinterpret_cast<const T2*>(sm.raw[buf][blk][1][sl][stl]);
        J.c = *reinterpret_cast<const T2*>(sm.raw[buf][blk][2][sl][stl]);
        J.d = *reinterpret_cast<const T2*>(sm.raw[buf][blk][3][sl][stl]);
        if ((blk == 0) != CASA)
        {
            const double I = sm.src[buf][sl][0], Q = sm.src[buf][sl][1];
            const T2 buv = T2{sm.src[buf][sl][2], sm.src[buf][sl][3]};
            const T2 buvc = T2{buv.x, -buv.y};
            const double xx = I + Q, yy = I - Q;
            Mat2<double> M;
            const T2 t0 = cmul<double>(J.b, buvc), t1 = cmul<double>(J.d, buvc);
            const T2 t2 = cmul<double>(J.a, buv), t3 = cmul<double>(J.c, buv);
            M.a = T2{J.a.x * xx + t0.x, J.a.y * xx + t0.y};
            M.c = T2{J.c.x * xx + t1.x, J.c.y * xx + t1.y};
            M.b = T2{J.b.x * yy + t2.x, J.b.y * yy + t2.y};
            M.d = T2{J.d.x * yy + t3.x, J.d.y * yy + t3.y};
            J = M;
        }
        double* frag = sm.frag[fbuf] + (blk ? kFragBlock : 0);
#define OSKB_FRAG(I, KK, C, VAL)                                             \
        frag[((2 * sl + KK) >> 2) * kFragK4 +                                \
                ((4 * stl + 2 * I + C) >> 3) * kFragTile +                   \
                4 * ((4 * stl + 2 * I + C) & 7) + ((2 * sl + KK) & 3)] = VAL;
        OSKB_FRAG(0, 0, 0, J.a.x) OSKB_FRAG(0, 0, 1, J.a.y)
        OSKB_FRAG(0, 1, 0, J.b.x) OSKB_FRAG(0, 1, 1, J.b.y)
        OSKB_FRAG(1, 0, 0, J.c.x) OSKB_FRAG(1, 0, 1, J.c.y)
        OSKB_FRAG(1, 1, 0, J.d.x) OSKB_FRAG(1, 1, 1, J.d.y)
#undef OSKB_FRAG
    }
}

// FP64 tensor-core form for point sources without smearing (matrix, FP64):
// the product of each 32 x 32 station tile on the FP64 tensor pipe with
// mma.sync m8n8k4 f64. Real embedding: with M = left factor (station p,
// rows) and R = right factor (station q, columns), entries
// W[(s, i, c)][(src, k)] = Re (c = 0) or Im (c = 1) of the 2x2 entry (i, k),
// and
//     G = W_M W_R^T,  Re V_ij = G[(p,i,0)][(q,j,0)] + G[(p,i,1)][(q,j,1)],
//                     Im V_ij = G[(p,i,1)][(q,j,0)] - G[(p,i,0)][(q,j,1)].
// The 128 x 128 G tile is split over 8 warps as 4 (rows) x 2 (columns) warp
// tiles of 32 x 64 = 4 x 8 m8n8 accumulators; a k4 step is two sources.
// Accumulation is FP64 throughout (no brightness factorisation, so any B).
// Pipeline per chunk c: copies of chunk c + 2 in flight, products of chunk
// c on the tensor pipe, transform of chunk c + 1 on the FP64 pipe, one
// barrier.
template <bool CASA>
__global__ void __launch_bounds__(kThreads, 1)
xcorr_dmma_kernel(const XcorrParams<double> prm)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    DmmaSmem& sm = *reinterpret_cast<DmmaSmem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 3, wn = warp >> 2;   // warp tile: rows, columns
    const int g = lane >> 2, t = lane & 3;     // mma fragment coordinates
    const int N = prm.num_st;
    const long long nbl = (long long) N * (N - 1) / 2;
    const int num_items = prm.tiles * prm.slices;

    for (int item = blockIdx.x; item < num_items; item += gridDim.x)
    {
    ItemCtx ctx;
    const int slice = item % prm.slices;
    const int tile = item / prm.slices;
    ctx.t = ctx.c = 0;
    {
        int bp, bq;
        tri_block(tile, bp, bq);
        ctx.p0 = bp * kTile;
        ctx.q0 = bq * kTile;
    }
    ctx.src_begin = slice * prm.slice_len;
    ctx.src_end = min(prm.num_src, ctx.src_begin + prm.slice_len);
    const int nchunks = ctx.src_end > ctx.src_begin ?
            (ctx.src_end - ctx.src_begin + kChunk - 1) / kChunk : 0;

    double acc[4][8][2];
#pragma unroll
    for (int ms = 0; ms < 4; ++ms)
#pragma unroll
        for (int ns = 0; ns < 8; ++ns) acc[ms][ns][0] = acc[ms][ns][1] = 0.0;

    __syncthreads();  // the previous item is done with shared memory
    if (nchunks > 0)
    {
        dmma_issue(sm, 0, prm, ctx, ctx.src_begin);
        if (nchunks > 1)
        {
            dmma_issue(sm, 1, prm, ctx, ctx.src_begin + kChunk);
            cp_async_wait_group<1>();
        }
        else
        {
            cp_async_wait_group<0>();
        }
        dmma_transform<CASA>(sm, 0, 0);
        __syncthreads();
    }
    for (int c = 0; c < nchunks; ++c)
    {
        const int s0 = ctx.src_begin + c * kChunk;
        // copies of chunk c + 2 into the raw buffer chunk c used (this
        // warp transformed its own elements of it already)
        if (c + 2 < nchunks)
            dmma_issue(sm, c & 1, prm, ctx, s0 + 2 * kChunk);
        // ---- products of chunk c: 4 k4 steps of 2 sources
        const double* fbase = sm.frag[c & 1];
#pragma unroll
        for (int k4 = 0; k4 < kChunk / 2; ++k4)
        {
            const double* fa = fbase + k4 * kFragK4;
            const double* fb = fa + kFragBlock;
            double a[4], b[8];
#pragma unroll
            for (int ms = 0; ms < 4; ++ms)
                a[ms] = fa[(4 * wm + ms) * kFragTile + lane];
#pragma unroll
            for (int ns = 0; ns < 8; ++ns)
                b[ns] = fb[(8 * wn + ns) * kFragTile + lane];
#pragma unroll
            for (int ms = 0; ms < 4; ++ms)
#pragma unroll
                for (int ns = 0; ns < 8; ++ns)
                    dmma_m8n8k4(acc[ms][ns][0], acc[ms][ns][1], a[ms],
                            b[ns]);
        }
        // ---- transform of chunk c + 1 while the products run
        if (c + 1 < nchunks)
        {
            if (c + 2 < nchunks) cp_async_wait_group<1>();
            else cp_async_wait_group<0>();
            dmma_transform<CASA>(sm, (c + 1) & 1, (c + 1) & 1);
        }
        __syncthreads();
    }

    // ---- visibilities: thread pairs (rows c = 0, 1: lanes l, l ^ 4) form
    // Re (c = 0) and Im (c = 1) of V_ij for their (p, q, i, j)
    const double kw = prm.inv_wavelength;
    const double* su = prm.st_u;
    const double* sv = prm.st_v;
    const double uv_lo = prm.uv_min, uv_hi = prm.uv_max;
#pragma unroll
    for (int ms = 0; ms < 4; ++ms)
#pragma unroll
        for (int ns = 0; ns < 8; ++ns)
        {
            const double d0 = acc[ms][ns][0], d1 = acc[ms][ns][1];
            const double other = __shfl_xor_sync(0xffffffffu, d1, 4);
            const int r = 32 * wm + 8 * ms + g;
            const int c = r & 1, i = (r >> 1) & 1;
            const int p = ctx.p0 + (r >> 2);
            const int n0 = 64 * wn + 8 * ns + 2 * t;
            const int j = (n0 >> 1) & 1;
            const int q = ctx.q0 + (n0 >> 2);
            if (p >= N || q >= p) continue;
            const double val = c ? d0 - other : d0 + other;
            // V'_ji = conj(V_ij) in the CASA convention
            const int e = CASA ? 2 * j + i : 2 * i + j;
            const double out_val = (CASA && c) ? -val : val;
            const double uu = (su[p] - su[q]) * kw;
            const double vv = (sv[p] - sv[q]) * kw;
            const double len = sqrt(uu * uu + vv * vv);
            const bool ok = !(len < uv_lo || len > uv_hi);
            const long long bl = baseline_index(N, p, q);
            if (prm.partial)
            {
                prm.partial[(size_t) 8 * (slice * nbl + bl) + 2 * e + c] =
                        ok ? out_val : 0.0;
                continue;
            }
            if (!ok) continue;
            double* o = prm.vis + (size_t) 8 * (bl + prm.offset_out) +
                    2 * e + c;
            *o += out_val;
        }
    }  // items
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

int num_sms() { return device_sm_count(); }

template <typename T, bool MATRIX, bool GAUSS, bool BW, bool TS, bool CASA,
        bool FUSED>
void launch_one(const XcorrParams<T>& p, int grid, cudaStream_t stream)
{
    const size_t smem = sizeof(Smem<T, MATRIX>);
    auto k = xcorr_direct_kernel<T, MATRIX, GAUSS, BW, TS, CASA, FUSED>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
            (int) smem);
    k<<<grid, kThreads, smem, stream>>>(p);
}

// Selects the kernel variant. FUSED (K formed in the staging) exists for
// the matrix form only.
template <typename T, bool MATRIX, bool FUSED>
void launch_variant(bool casa, bool gauss, bool bw, bool ts,
        const XcorrParams<T>& p, int grid, cudaStream_t s)
{
#define OSKB_L(G, B, S)                                                      \
    (casa ? launch_one<T, MATRIX, G, B, S, true, FUSED>(p, grid, s)          \
          : launch_one<T, MATRIX, G, B, S, false, FUSED>(p, grid, s))
    if (gauss)
    {
        if (!bw && !ts) OSKB_L(true, false, false);
        else if (bw && !ts) OSKB_L(true, true, false);
        else if (!bw && ts) OSKB_L(true, false, true);
        else OSKB_L(true, true, true);
    }
    else
    {
        if (!bw && !ts) OSKB_L(false, false, false);
        else if (bw && !ts) OSKB_L(false, true, false);
        else if (!bw && ts) OSKB_L(false, false, true);
        else OSKB_L(false, true, true);
    }
#undef OSKB_L
}

// FP64 matrix point sources without smearing run on the FP64 tensor pipe
// (xcorr_dmma_kernel) by default: with the transform of the next chunk
// overlapping the current chunk's products it measured 8 % faster than the
// SIMT kernel (256 against 236 G source-baselines/s at 512 stations x 8,000
// sources on one B200). OSKB_XCORR_DMMA=0 selects the SIMT kernel.
template <typename T, bool MATRIX>
bool use_dmma(bool gauss, bool bw, bool ts)
{
    if (sizeof(T) != 8 || !MATRIX || gauss || bw || ts) return false;
    const char* e = getenv("OSKB_XCORR_DMMA");
    return !(e && e[0] == '0');
}

template <typename T>
void launch_dmma(bool casa, const XcorrParams<T>& p, int grid,
        cudaStream_t stream)
{
    if constexpr (sizeof(T) == 8)
    {
        const size_t smem = sizeof(DmmaSmem);
        if (casa)
        {
            auto k = xcorr_dmma_kernel<true>;
            cudaFuncSetAttribute(k,
                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
            k<<<grid, kThreads, smem, stream>>>(p);
        }
        else
        {
            auto k = xcorr_dmma_kernel<false>;
            cudaFuncSetAttribute(k,
                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
            k<<<grid, kThreads, smem, stream>>>(p);
        }
    }
}

int tiles_for(int num_st)
{
    const int nb = (num_st + kTile - 1) / kTile;
    return nb * (nb + 1) / 2;
}

// One call: one dump, one channel, sources split into slices.
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
    const int tiles = tiles_for(p.num_st);
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
    p.num_times = p.num_channels = 1;
    p.tiles = tiles;
    p.slices = slices;
    p.slice_len = slice_len;
    p.tile_major = 0;
    p.partial = nullptr;
    if (slices > 1)
    {
        const size_t bytes = (size_t) slices * nbl * ncomp2 * sizeof(double);
        if (scratch_alloc((void**) &p.partial, bytes, stream) !=
                cudaSuccess)
        {
            cudaGetLastError();  // no room for partials: one slice
            p.partial = nullptr;
            p.slices = slices = 1;
            p.slice_len = p.num_src;
        }
    }
    if (use_dmma<T, MATRIX>(gauss, bw, ts))
        launch_dmma(casa, p, tiles * slices, stream);
    else
        launch_variant<T, MATRIX, false>(casa, gauss, bw, ts, p,
                tiles * slices, stream);
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
        scratch_free(p.partial, stream);
    }
    return err;
}

// ---------------------------------------------------------------- blocks
// Schedule of one block launch: grid size (CTAs; 0 = one per item) and
// item order. Picked per block shape by timing the candidates on a sample
// of the block (the first dump, the first 4,096 sources) into scratch
// visibilities; cached for the process. Every schedule sums each
// (dump, channel, baseline) over the sources in the same order, so the
// choice changes speed only, never a bit of the result.
struct BlockSchedule
{
    int ctas_per_sm;  // grid = ctas_per_sm x SMs; 0: one CTA per item
    int tile_major;
};

constexpr int kNumCandidates = 8;
const BlockSchedule kCandidates[kNumCandidates] = {
    {2, 0}, {2, 1}, {4, 0}, {4, 1}, {8, 0}, {8, 1}, {0, 0}, {0, 1}};

struct TuneEntry
{
    long long key[10];
    BlockSchedule sched;
    float ms[kNumCandidates];
};

TuneEntry g_tune[64];
int g_num_tune = 0;
std::mutex g_tune_mutex;

int grid_for(const BlockSchedule& s, int items)
{
    if (s.ctas_per_sm <= 0) return items;
    return max(1, min(items, s.ctas_per_sm * num_sms()));
}

template <typename T>
BlockSchedule block_schedule(bool casa, bool gauss, bool bw, bool ts,
        const XcorrParams<T>& p, cudaStream_t stream)
{
    const BlockSchedule dflt = {2, 1};
    if (const char* e = getenv("OSKB_BLOCK_SCHEDULE"))
    {
        BlockSchedule s = dflt;
        if (sscanf(e, "%d,%d", &s.ctas_per_sm, &s.tile_major) == 2) return s;
    }
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    int dev = 0;
    cudaGetDevice(&dev);
    (void) dev;
    const long long key[10] = {(long long) sizeof(T), casa, gauss, bw, ts,
            p.num_st, p.num_src, p.num_times, p.num_channels,
            p.jones != nullptr};
    for (int i = 0; i < g_num_tune; ++i)
        if (!memcmp(g_tune[i].key, key, sizeof(key))) return g_tune[i].sched;
    const char* at = getenv("OSKB_AUTOTUNE");
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(stream, &cap);
    if ((at && at[0] == '0') || cap != cudaStreamCaptureStatusNone ||
            g_num_tune >= 64)
        return dflt;

    // Sample: the first dump, all channels, up to 4,096 sources.
    XcorrParams<T> q = p;
    q.num_times = 1;
    q.num_src = min(p.num_src, 4096);
    q.slice_len = q.num_src;
    const long long nbl = (long long) p.num_st * (p.num_st - 1) / 2;
    const size_t vis_bytes = (size_t) q.num_channels * nbl * 8 * sizeof(T);
    TuneEntry ent;
    memcpy(ent.key, key, sizeof(key));
    ent.sched = dflt;
    if (scratch_alloc((void**) &q.vis, vis_bytes, stream) != cudaSuccess)
    {
        cudaGetLastError();
        return dflt;
    }
    cudaMemsetAsync(q.vis, 0, vis_bytes, stream);
    q.offset_out = 0;
    const int items = q.num_times * q.num_channels * q.tiles;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 3e38f;
    for (int i = 0; i < kNumCandidates; ++i)
    {
        q.tile_major = kCandidates[i].tile_major;
        const int grid = grid_for(kCandidates[i], items);
        launch_variant<T, true, true>(casa, gauss, bw, ts, q, grid, stream);
        cudaEventRecord(e0, stream);
        launch_variant<T, true, true>(casa, gauss, bw, ts, q, grid, stream);
        cudaEventRecord(e1, stream);
        float ms = 3e38f;
        if (cudaEventSynchronize(e1) == cudaSuccess)
            cudaEventElapsedTime(&ms, e0, e1);
        ent.ms[i] = ms;
        if (ms < best)
        {
            best = ms;
            ent.sched = kCandidates[i];
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    scratch_free(q.vis, stream);
    cudaGetLastError();
    g_tune[g_num_tune++] = ent;
    return ent.sched;
}

// A whole block: every (dump, channel) in one persistent launch, K fused.
template <typename T>
int block_dispatch(bool casa, bool gauss, bool bw, bool ts, XcorrParams<T> p,
        cudaStream_t stream)
{
    if (p.num_st < 2 || p.num_src <= 0 || p.num_times <= 0 ||
            p.num_channels <= 0)
        return 0;
    if (p.jones && (uintptr_t) p.jones % Staging<T, true>::COPY != 0)
        return OSKB_ERR_INVALID_ARGUMENT;
    p.tiles = tiles_for(p.num_st);
    p.slices = 1;
    p.slice_len = p.num_src;
    p.partial = nullptr;
    const long long tc_items = (long long) p.num_times * p.num_channels *
            p.tiles;
    if (tc_items > 0x7fffffffLL) return OSKB_ERR_INVALID_ARGUMENT;
    const BlockSchedule s = block_schedule<T>(casa, gauss, bw, ts, p, stream);
    p.tile_major = s.tile_major;
    // Too few (dump, channel, tile) items to fill the GPU: split the
    // sources too (at least 64 per slice), the slices' sums reduced into
    // vis in slice order afterwards.
    const long long want = 4LL * num_sms();
    if (tc_items < want)
    {
        const int max_slices = (p.num_src + 8 * kChunk - 1) / (8 * kChunk);
        int slices = (int) min((long long) max_slices,
                (want + tc_items - 1) / tc_items);
        if (slices > 1)
        {
            int len = (p.num_src + slices - 1) / slices;
            len = (len + kChunk - 1) / kChunk * kChunk;
            slices = (p.num_src + len - 1) / len;
            const size_t bytes = (size_t) slices * tc_items / p.tiles *
                    ((size_t) p.num_st * (p.num_st - 1) / 2) * 8 *
                    sizeof(double);
            if (slices > 1 && scratch_alloc((void**) &p.partial, bytes,
                    stream) == cudaSuccess)
            {
                p.slices = slices;
                p.slice_len = len;
            }
            else
            {
                cudaGetLastError();
                p.partial = nullptr;
            }
        }
    }
    const long long items = tc_items * p.slices;
    launch_variant<T, true, true>(casa, gauss, bw, ts, p,
            grid_for(s, (int) items), stream);
    int err = check_launch("correlate_block_direct");
    if (p.partial)
    {
        const long long n = (long long) p.num_times * p.num_channels *
                ((long long) p.num_st * (p.num_st - 1) / 2) * 8;
        if (!err)
        {
            reduce_partials_kernel<T><<<(unsigned) ((n + 255) / 256), 256, 0,
                    stream>>>(p.partial, p.slices, n, 0, p.vis);
            err = check_launch("correlate_block_direct reduce");
        }
        scratch_free(p.partial, stream);
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
    memset(&p, 0, sizeof(p));
    p.num_src = num_sources; p.num_st = num_stations; p.offset_out = offset_out;
    p.src_stride = num_sources;
    p.jones = jones; p.I = I; p.Q = Q; p.U = U; p.V = V;
    p.l = l; p.m = m; p.n = n; p.a = a; p.b = b; p.c = c;
    p.st_u = su; p.st_v = sv; p.st_w = sw; p.st_x = sx; p.st_y = sy;
    p.uv_min = uv_min; p.uv_max = uv_max; p.inv_wavelength = inv_wavelength;
    p.bw_scale = kPi * (double) frac_bandwidth * (double) inv_wavelength;
    p.ts_base = kPi * kOmegaEarth * (double) time_int_sec;
    p.gha0 = gha0;
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

namespace oskb {
namespace {

template <typename T>
int correlate_block_direct(int casa, int num_sources, int num_stations,
        int num_times, int num_channels, const T* E, int E_per_dump,
        const T* I, const T* Q, const T* U, const T* V, const T* l,
        const T* m, const T* n, const T* a, const T* b, const T* c,
        const T* station_uvw, const T* station_x, const T* station_y,
        const double* inv_wavelength, double channel_bandwidth_hz,
        double time_average_sec, const double* gha0_rad, double dec0_rad,
        double uv_min, double uv_max, int uv_filter_units,
        double source_filter_min, double source_filter_max, T* vis,
        void* stream, long long flux_channel_stride)
{
    if (num_sources < 0 || num_stations < 0 || num_times < 0 ||
            num_channels < 0)
        return OSKB_ERR_INVALID_ARGUMENT;
    if (flux_channel_stride != 0 && flux_channel_stride < num_sources)
        return OSKB_ERR_INVALID_ARGUMENT;
    if (num_sources == 0 || num_stations < 2 || num_times == 0 ||
            num_channels == 0)
        return 0;
    const bool bw = channel_bandwidth_hz != 0.0;
    const bool ts = time_average_sec != 0.0;
    const bool gauss = a && b && c;
    if (!I || !Q || !U || !V || !l || !m || !n || !station_uvw ||
            !inv_wavelength || !vis || (ts && (!station_x || !station_y ||
            !gha0_rad)))
        return OSKB_ERR_INVALID_ARGUMENT;
    XcorrParams<T> p;
    memset(&p, 0, sizeof(p));
    p.num_src = num_sources;
    p.src_stride = num_sources;
    p.num_st = num_stations;
    p.jones = E;
    p.e_time_stride = E_per_dump ? 8LL * num_stations * num_sources : 0;
    p.I = I; p.Q = Q; p.U = U; p.V = V; p.l = l; p.m = m; p.n = n;
    p.a = a; p.b = b; p.c = c;
    p.st_u = station_uvw;
    p.st_v = station_uvw + num_stations;
    p.st_w = station_uvw + 2 * (size_t) num_stations;
    p.uvw_time_stride = 3LL * num_stations;
    p.st_x = station_x; p.st_y = station_y;
    p.uv_min = uv_min; p.uv_max = uv_max;
    p.uv_filter_in_metres = uv_filter_units == 0;
    p.inv_wavelength_c = inv_wavelength;
    p.bw_scale = kPi * channel_bandwidth_hz / 299792458.0;
    p.ts_base = kPi * kOmegaEarth * time_average_sec;
    p.gha0_t = gha0_rad;
    p.s_dec = sin(dec0_rad); p.c_dec = cos(dec0_rad);
    p.vis = vis;
    p.num_times = num_times;
    p.num_channels = num_channels;
    p.filter_min = source_filter_min;
    p.filter_max = source_filter_max;
    p.flux_channel_stride = flux_channel_stride;
    return block_dispatch<T>(casa != 0, gauss, bw, ts, p, as_stream(stream));
}

}  // namespace
}  // namespace oskb

extern "C" {

#define OSKB_BLOCK_ENTRY(T, S)                                               \
int oskb_correlate_block_direct_##S(int casa, int num_sources,               \
        int num_stations, int num_times, int num_channels, const T* E,       \
        int E_per_dump, const T* I, const T* Q, const T* U, const T* V,      \
        const T* l, const T* m, const T* n, const T* a, const T* b,          \
        const T* c, const T* station_uvw, const T* station_x,                \
        const T* station_y, const double* inv_wavelength,                    \
        double channel_bandwidth_hz, double time_average_sec,                \
        const double* gha0_rad, double dec0_rad, double uv_min,              \
        double uv_max, int uv_filter_units, double source_filter_min,        \
        double source_filter_max, T* vis, void* stream)                      \
{                                                                            \
    return oskb::correlate_block_direct<T>(casa, num_sources, num_stations,  \
            num_times, num_channels, E, E_per_dump, I, Q, U, V, l, m, n, a,  \
            b, c, station_uvw, station_x, station_y, inv_wavelength,         \
            channel_bandwidth_hz, time_average_sec, gha0_rad, dec0_rad,      \
            uv_min, uv_max, uv_filter_units, source_filter_min,              \
            source_filter_max, vis, stream, 0);                              \
}                                                                            \
int oskb_correlate_block_direct_spectral_##S(int casa, int num_sources,      \
        int num_stations, int num_times, int num_channels, const T* E,       \
        int E_per_dump, const T* I, const T* Q, const T* U, const T* V,      \
        long long flux_channel_stride, const T* l, const T* m, const T* n,   \
        const T* a, const T* b, const T* c, const T* station_uvw,            \
        const T* station_x, const T* station_y,                              \
        const double* inv_wavelength, double channel_bandwidth_hz,           \
        double time_average_sec, const double* gha0_rad, double dec0_rad,    \
        double uv_min, double uv_max, int uv_filter_units,                   \
        double source_filter_min, double source_filter_max, T* vis,          \
        void* stream)                                                        \
{                                                                            \
    return oskb::correlate_block_direct<T>(casa, num_sources, num_stations,  \
            num_times, num_channels, E, E_per_dump, I, Q, U, V, l, m, n, a,  \
            b, c, station_uvw, station_x, station_y, inv_wavelength,         \
            channel_bandwidth_hz, time_average_sec, gha0_rad, dec0_rad,      \
            uv_min, uv_max, uv_filter_units, source_filter_min,              \
            source_filter_max, vis, stream, flux_channel_stride);            \
}

OSKB_BLOCK_ENTRY(double, d)
OSKB_BLOCK_ENTRY(float, f)
#undef OSKB_BLOCK_ENTRY

int oskb_block_tune_report(char* buf, int len)
{
    std::lock_guard<std::mutex> lock(oskb::g_tune_mutex);
    int used = 0;
    if (len > 0) buf[0] = 0;
    for (int i = 0; i < oskb::g_num_tune && used < len; ++i)
    {
        const oskb::TuneEntry& e = oskb::g_tune[i];
        used += snprintf(buf + used, len - used,
                "fp%lld casa=%lld gauss=%lld bw=%lld ts=%lld stations=%lld "
                "sources=%lld dumps=%lld channels=%lld beam=%lld -> "
                "ctas_per_sm=%d tile_major=%d; sample ms:",
                8 * e.key[0], e.key[1], e.key[2], e.key[3], e.key[4],
                e.key[5], e.key[6], e.key[7], e.key[8], e.key[9],
                e.sched.ctas_per_sm, e.sched.tile_major);
        for (int k = 0; k < oskb::kNumCandidates && used < len; ++k)
            used += snprintf(buf + used, len - used, " %.3f", e.ms[k]);
        if (used < len) used += snprintf(buf + used, len - used, "\n");
    }
    return used < len ? used : len;
}

}  // extern "C"

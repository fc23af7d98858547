// Tensor-core (tcgen05) compensated cross-correlation of point sources
// without smearing.
//
// Algebra. With the brightness factored as B(s) = C(s) C(s)^H (C the lower
// Cholesky factor of [[I+Q, U+iV], [U-iV, I-Q]]), A_p(s) = J_p(s) C(s) and
//     V_pq = sum_s A_p(s) A_q(s)^H,
// i.e. V = X X^H, a Hermitian rank-k update over sources. Interleaving the
// real and imaginary parts as rows, W[(p, i, c)][(s, kk)] = part c of
// A_p(s)[i][kk], turns it into the real symmetric product G = W W^T:
//     Re V_pq[i][j] = G[(p,i,0),(q,j,0)] + G[(p,i,1),(q,j,1)]
//     Im V_pq[i][j] = G[(p,i,1),(q,j,0)] - G[(p,i,0),(q,j,1)]
// and only the upper block triangle of G is computed.
//
// Precision. W is scaled by a power of two S (largest |entry| -> 2^14) and
// split into two FP16 pieces, W = hi + lo (22 significant bits); G is formed
// from the three products hi hi^T + hi lo^T + lo hi^T on the tensor cores
// (FP16 x FP16 products are exact in FP32), accumulated in FP32 in TMEM for
// a bounded number of k-blocks and then added into FP64 registers (the
// cross-tile sum is FP64). The hi hi^T products go to their own TMEM
// accumulator: the tensor core rounds its FP32 accumulator once per MMA,
// and keeping the 2^-11-smaller correction products out of it leaves only
// four full-size accumulate steps per k-block. The interferometer phase is formed in FP64 and
// reduced mod 1 cycle before an FP32 sincospi.
//
// Layout of the operand image (per problem): tiles of 128 rows (32 stations)
// x 64 columns (32 sources) of FP16, each 16 KB, stored exactly as the MMA
// reads them from shared memory (K-major, 128-byte swizzle), hi tile then lo
// tile, ordered [row block][k block][hi, lo]. A pipeline stage is therefore
// one 32 KB bulk copy per operand.
#include <cuda.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <utility>
#include <vector>

#include "common.cuh"
#include "tc_ptx.cuh"
#include "xcorr_tc.cuh"

namespace oskb {
namespace tc {

constexpr int kStPerBlock = 32;              // stations per 128-row block
constexpr int kSrcPerBlock = 32;             // sources per 64-column block
constexpr int kTileBytes = 128 * 128;        // 128 rows x 128 bytes
constexpr int kPairBytes = 2 * kTileBytes;   // hi + lo
constexpr int kKSteps = 4;                   // K = 16 MMA steps per k block
constexpr float kScaleTarget = 16384.0f;     // largest scaled |entry|

__host__ __device__ inline size_t image_bytes(int num_st, int num_src)
{
    const size_t nrb = (num_st + kStPerBlock - 1) / kStPerBlock;
    const size_t nkb = (num_src + kSrcPerBlock - 1) / kSrcPerBlock;
    return nrb * nkb * kPairBytes;
}

// Power-of-two scale that maps the largest |entry| to at most 2^14.
__device__ __forceinline__ float scale_from_bits(unsigned int bits)
{
    const float m = __uint_as_float(bits);
    if (!(m > 0.0f) || !isfinite(m)) return 1.0f;
    const float e = floorf(log2f(kScaleTarget / m));
    return exp2f(fminf(fmaxf(e, -100.0f), 100.0f));
}

// Integer operand image (the default contraction): every entry x is the
// fixed-point integer a = round(x q), |a| <= 127 * 2^16 (plus rounding),
// held as three signed 8-bit limbs a = a0 2^16 + a1 2^8 + a2 with a1, a2
// in [-128, 127] (balanced digits, so that the left-out product a2 b2 has
// no bias). They are the bytes of t = a + 0x8080 with the two low bytes'
// top bits flipped: t = a0 2^16 + (a1 + 128) 2^8 + (a2 + 128), and
// a0 = t >> 16 stays in [-127, 127]. Per 32-station x 32-source block:
// three limb tiles of 128 rows x 64 bytes (one byte per K column), stored
// with the 64-byte swizzle.
constexpr int kI8Tile = 128 * 64;
constexpr int kI8Block = 3 * kI8Tile;
constexpr float kI8Target = 8323072.0f;      // 127 * 2^16

// Sources of the integer image are ordered by amplitude bucket: bucket b
// holds the sources whose largest |entry| over the stations is in
// (m 2^-(b+1), m 2^-b] (m the largest of all; the last bucket also takes
// everything fainter), each bucket padded to whole 32-source blocks and
// scaled by its own q_b = q 2^b, so a source's entries use the limbs' full
// range whatever its flux. The k blocks of one problem's image are the
// padded, ordered sources (i8_kb_cap bounds their number).
constexpr int kI8Buckets = 16;
constexpr int kI8DrainKb = 512;

// Each non-empty bucket pads to whole blocks, so the k blocks are at most
// sum_b ceil(n_b / 32) <= (num_src + 31 B) / 32 for B non-empty buckets,
// B <= min(kI8Buckets, num_src).
__host__ __device__ inline int i8_kb_cap(int num_src)
{
    const int nb = num_src < kI8Buckets ? num_src : kI8Buckets;
    return (int) (((long long) num_src + (long long) (kSrcPerBlock - 1) * nb)
            / kSrcPerBlock);
}

__host__ __device__ inline size_t image_bytes_i8(int num_st, int num_src)
{
    const size_t nrb = (num_st + kStPerBlock - 1) / kStPerBlock;
    return nrb * (size_t) i8_kb_cap(num_src) * kI8Block;
}

// The contraction's chunks (accumulator drain intervals): one or more per
// bucket, at most drain_kb k blocks each (kI8DrainKb for the three-limb
// image).
__host__ __device__ inline int i8_max_chunks(int num_src, int drain_kb)
{
    return (i8_kb_cap(num_src) + drain_kb - 1) / drain_kb + kI8Buckets;
}

// Source order and scales of one call (device, in the workspace before the
// image): counts[0] = k blocks used, counts[1] = chunks; chunk c covers k
// blocks [chunk_kb[c], chunk_kb[c + 1]) of bucket chunk_bucket[c]; kb_bucket
// is the bucket of each k block; perm maps each padded source position to
// its source (-1: padding); amp_bits holds each source's largest |entry|.
struct I8Order
{
    int* counts;
    int* chunk_kb;
    int* chunk_bucket;
    int* kb_bucket;
    int* perm;
    unsigned int* amp_bits;
};

__host__ __device__ inline size_t align256_t(size_t b)
{
    return (b + 255) & ~(size_t) 255;
}

// Bytes of the tables for num_src sources and chunks of at most drain_kb
// k blocks; with base set, also their addresses.
__host__ __device__ inline size_t i8_order_bytes(int num_src, int drain_kb,
        uint8_t* base, I8Order* o)
{
    const size_t cap = (size_t) i8_kb_cap(num_src);
    const size_t mc = (size_t) i8_max_chunks(num_src, drain_kb);
    size_t off = 0;
    const size_t sizes[6] = {align256_t(2 * sizeof(int)),
            align256_t((mc + 1) * sizeof(int)), align256_t(mc * sizeof(int)),
            align256_t(cap * sizeof(int)),
            align256_t(cap * kSrcPerBlock * sizeof(int)),
            align256_t((size_t) num_src * sizeof(unsigned int))};
    if (base && o)
    {
        o->counts = reinterpret_cast<int*>(base + off); off += sizes[0];
        o->chunk_kb = reinterpret_cast<int*>(base + off); off += sizes[1];
        o->chunk_bucket = reinterpret_cast<int*>(base + off); off += sizes[2];
        o->kb_bucket = reinterpret_cast<int*>(base + off); off += sizes[3];
        o->perm = reinterpret_cast<int*>(base + off); off += sizes[4];
        o->amp_bits = reinterpret_cast<unsigned int*>(base + off);
        off += sizes[5];
        return off;
    }
    for (size_t k = 0; k < 6; ++k) off += sizes[k];
    return off;
}

// Fixed-point scale q (not a power of two) for the largest |entry| m.
__device__ __forceinline__ float i8_scale_from_bits(unsigned int bits)
{
    const float m = __uint_as_float(bits);
    if (!(m > 0.0f) || !isfinite(m)) return 1.0f;
    return kI8Target / m;
}

// Bucket of a source whose largest |entry| is a, for the largest of all m
// (both as float bits): floor(log2(m / a)) in [0, kI8Buckets - 1] (so
// a <= m 2^-b). For normal floats it is the exponent difference, less one
// where a's significand exceeds m's (exact); zero sources go to the last
// bucket.
__device__ __forceinline__ int i8_bucket(unsigned int a_bits,
        unsigned int m_bits)
{
    const float a = __uint_as_float(a_bits), m = __uint_as_float(m_bits);
    if (!(a > 0.0f) || !(m > 0.0f) || !isfinite(m))
        return a > 0.0f ? 0 : kI8Buckets - 1;
    const int ea = (int) (a_bits >> 23), em = (int) (m_bits >> 23);
    int b;
    if (ea > 0 && em > 0)
        b = em - ea - ((m_bits & 0x7fffffu) < (a_bits & 0x7fffffu) ? 1 : 0);
    else
        b = (int) floor(log2((double) m / (double) a));
    return b < 0 ? 0 : (b >= kI8Buckets ? kI8Buckets - 1 : b);
}

// Byte offset of K column c (0..63) of row r in a limb tile.
__device__ __forceinline__ uint32_t swz64_offset(int r, int c)
{
    return (uint32_t) (r * 64 + ((((c >> 4) ^ (r >> 1)) & 3) << 4) +
                       (c & 15));
}

// Writes one station-source's 2x2 A (already scaled by q) as 4 rows of the
// three limb tiles of its block.
__device__ __forceinline__ void store_entry_i8(uint8_t* block, int pl,
        int sl, const float A[2][2][2])
{
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int c = 0; c < 2; ++c)
        {
            const int r = 4 * pl + 2 * i + c;
            const int t0 = __float2int_rn(A[i][0][c]) + 0x8080;
            const int t1 = __float2int_rn(A[i][1][c]) + 0x8080;
            const uint32_t off = swz64_offset(r, 2 * sl);
            // limb k of both K columns: byte 2 - k of each t, the low limbs
            // with their top bit flipped
#pragma unroll
            for (int limb = 0; limb < 3; ++limb)
                *reinterpret_cast<uint16_t*>(block + limb * kI8Tile + off) =
                        (uint16_t) (__byte_perm(t0, t1,
                                (2 - limb) | ((6 - limb) << 4)) ^
                                (limb ? 0x8080u : 0u));
        }
}

// Byte offset of the 4-byte word holding columns (2*sl, 2*sl+1) of tile row
// r, with the 128-byte swizzle applied (16-byte chunk index XOR row % 8).
__device__ __forceinline__ uint32_t swz_offset(int r, int sl)
{
    return (uint32_t) (r * 128 + ((((sl >> 2) ^ (r & 7)) & 7) << 4) +
                       (sl & 3) * 4);
}

// Lower Cholesky factor C of B = [[I+Q, U+iV], [U-iV, I-Q]]:
// C = [[c11, 0], [c21, c22]], c11 and c22 real. Returns false when B is not
// positive semi-definite (beyond rounding); C is then the factor of the
// nearest PSD matrix with that diagonal clipped at zero.
template <typename T>
__device__ __forceinline__ bool brightness_factor(double I, double Q,
        double U, double V, T& c11, T& c21r, T& c21i, T& c22)
{
    const double xx = I + Q, yy = I - Q;
    const double tol = 1e-12 * (fabs(I) + fabs(Q) + fabs(U) + fabs(V));
    bool ok = true;
    if (xx > tol)
    {
        const double a = sqrt(xx);
        const double br = U / a, bi = -V / a;
        const double d = yy - (br * br + bi * bi);
        if (d < -tol) ok = false;
        c11 = (T) a; c21r = (T) br; c21i = (T) bi;
        c22 = (T) sqrt(fmax(d, 0.0));
    }
    else
    {
        if (xx < -tol || fabs(U) > tol || fabs(V) > tol) ok = false;
        c11 = 0; c21r = 0; c21i = 0;
        c22 = (T) sqrt(fmax(yy, 0.0));
    }
    return ok;
}

// A = J C for a 2x2 complex J (row-major {a, b, c, d}) and lower-triangular
// C; out[i][kk][part].
__device__ __forceinline__ void apply_factor(const float* J, float c11,
        float c21r, float c21i, float c22, float out[2][2][2])
{
#pragma unroll
    for (int i = 0; i < 2; ++i)
    {
        const float j0r = J[4 * i + 0], j0i = J[4 * i + 1];
        const float j1r = J[4 * i + 2], j1i = J[4 * i + 3];
        out[i][0][0] = j0r * c11 + (j1r * c21r - j1i * c21i);
        out[i][0][1] = j0i * c11 + (j1r * c21i + j1i * c21r);
        out[i][1][0] = j1r * c22;
        out[i][1][1] = j1i * c22;
    }
}

template <typename TJ>
__device__ __forceinline__ void load_jones(const TJ* p, float* J)
{
#pragma unroll
    for (int k = 0; k < 8; ++k) J[k] = (float) p[k];
}

template <>
__device__ __forceinline__ void load_jones<float>(const float* p, float* J)
{
    const float4 a = __ldg(reinterpret_cast<const float4*>(p));
    const float4 b = __ldg(reinterpret_cast<const float4*>(p) + 1);
    J[0] = a.x; J[1] = a.y; J[2] = a.z; J[3] = a.w;
    J[4] = b.x; J[5] = b.y; J[6] = b.z; J[7] = b.w;
}

template <>
__device__ __forceinline__ void load_jones<double>(const double* p, float* J)
{
    const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
    for (int k = 0; k < 4; ++k)
    {
        const double2 v = __ldg(q + k);
        J[2 * k] = (float) v.x; J[2 * k + 1] = (float) v.y;
    }
}

// Writes one station-source's 2x2 A (already scaled) as 4 tile rows of the
// hi and lo tiles.
__device__ __forceinline__ void store_entry(uint8_t* tile_hi, int pl, int sl,
        const float A[2][2][2])
{
    uint8_t* tile_lo = tile_hi + kTileBytes;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int c = 0; c < 2; ++c)
        {
            const int r = 4 * pl + 2 * i + c;
            const float x0 = A[i][0][c], x1 = A[i][1][c];
            const __half h0 = __float2half_rn(x0), h1 = __float2half_rn(x1);
            const __half l0 = __float2half_rn(x0 - __half2float(h0));
            const __half l1 = __float2half_rn(x1 - __half2float(h1));
            const uint32_t off = swz_offset(r, sl);
            *reinterpret_cast<__half2*>(tile_hi + off) = __halves2half2(h0, h1);
            *reinterpret_cast<__half2*>(tile_lo + off) = __halves2half2(l0, l1);
        }
}

// ---------------------------------------------------------------------------
// Largest |component| of J C over all station-sources (-> the scale S).
// ---------------------------------------------------------------------------
// The bound uses the complex modulus of each entry, so it also holds after
// the unit-modulus phase K is applied.
template <typename TJ, typename TF>
__global__ void __launch_bounds__(256) maxabs_kernel(const TJ* __restrict__ jones,
        int num_src, int num_st, const TF* __restrict__ I,
        const TF* __restrict__ Q, const TF* __restrict__ U,
        const TF* __restrict__ V, unsigned int* maxabs_bits, int* flags)
{
    float mx = 0.0f;
    bool psd = true;
    const size_t total = (size_t) num_st * num_src;
    for (size_t idx = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
            idx < total; idx += (size_t) gridDim.x * blockDim.x)
    {
        const int s = (int) (idx % num_src);
        float c11, c21r, c21i, c22, J[8], A[2][2][2];
        psd &= brightness_factor(I[s], Q[s], U[s], V[s], c11, c21r, c21i,
                c22);
        load_jones<TJ>(jones + 8 * idx, J);
        apply_factor(J, c11, c21r, c21i, c22, A);
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int kk = 0; kk < 2; ++kk)
                mx = fmaxf(mx, hypotf(A[i][kk][0], A[i][kk][1]));
    }
    for (int o = 16; o > 0; o >>= 1)
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(maxabs_bits, __float_as_uint(mx));
    if (!psd) atomicOr(flags, 1);
}

// ---------------------------------------------------------------------------
// Largest |entry| of J C per source over the stations (amp_bits, cleared
// before) and of all (maxabs_bits), for the integer image's buckets and
// scales. One thread per source and station range (blockIdx.y of
// gridDim.y), the stations in a loop (coalesced over sources); positive
// floats order as their bit patterns, so the maxima are integer atomics.
// ---------------------------------------------------------------------------
template <typename TJ, typename TF>
__global__ void __launch_bounds__(256) maxabs_src_kernel(
        const TJ* __restrict__ jones, int num_src, int num_st,
        const TF* __restrict__ I, const TF* __restrict__ Q,
        const TF* __restrict__ U, const TF* __restrict__ V,
        unsigned int* __restrict__ amp_bits, unsigned int* maxabs_bits,
        int* flags)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int per = (num_st + gridDim.y - 1) / gridDim.y;
    const int pa = blockIdx.y * per, pb = min(num_st, pa + per);
    float mx = 0.0f;
    bool psd = true;
    if (s < num_src && pa < pb)
    {
        float c11, c21r, c21i, c22, J[8], A[2][2][2];
        psd = brightness_factor(I[s], Q[s], U[s], V[s], c11, c21r, c21i,
                c22);
        for (int p = pa; p < pb; ++p)
        {
            load_jones<TJ>(jones + 8 * ((size_t) p * num_src + s), J);
            apply_factor(J, c11, c21r, c21i, c22, A);
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int kk = 0; kk < 2; ++kk)
                    mx = fmaxf(mx, hypotf(A[i][kk][0], A[i][kk][1]));
        }
        atomicMax(amp_bits + s, __float_as_uint(mx));
    }
    for (int o = 16; o > 0; o >>= 1)
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(maxabs_bits, __float_as_uint(mx));
    if (!psd) atomicOr(flags, 1);
}

// ---------------------------------------------------------------------------
// The integer image's source order (one CTA of kOrderThreads = 32 warps):
// sources are taken kOrderThreads at a time in source order (coalesced).
// Pass 1 counts the sources per bucket (the lanes of a warp that share a
// bucket found with __match_any_sync, one shared-memory add per group);
// then the bucket starts (each bucket padded to whole 32-source blocks),
// the chunk table and the bucket of every k block. Pass 2 places every
// source at its bucket's start plus the number of sources before it in the
// same bucket (earlier rounds' running count, earlier warps of this round,
// earlier lanes of its warp), so each bucket keeps the sources in their
// original order (deterministic); then the padding.
// ---------------------------------------------------------------------------
constexpr int kOrderThreads = 1024;

__global__ void __launch_bounds__(kOrderThreads) i8_order_kernel(
        int num_src, int drain_kb,
        const unsigned int* __restrict__ maxabs_bits, I8Order o)
{
    constexpr int kWarps = kOrderThreads / 32;
    __shared__ int total[kI8Buckets], start[kI8Buckets + 1];
    __shared__ int running[kI8Buckets];
    __shared__ int wcnt[kWarps][kI8Buckets];
    __shared__ int woff[kWarps][kI8Buckets];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const unsigned int m_bits = *maxabs_bits;
    const unsigned int lt = (1u << lane) - 1u;
    if (t < kI8Buckets)
    {
        total[t] = 0;
        running[t] = 0;
    }
    __syncthreads();
    // ---- pass 1: bucket sizes
    for (int s0 = 0; s0 < num_src; s0 += kOrderThreads)
    {
        const int s = s0 + t;
        const int b = s < num_src ? i8_bucket(o.amp_bits[s], m_bits) : -1;
        const unsigned int same = __match_any_sync(0xffffffffu, b);
        if (b >= 0 && (same & lt) == 0)
            atomicAdd(&total[b], __popc(same));
    }
    __syncthreads();
    if (t == 0)
    {
        start[0] = 0;
        for (int b = 0; b < kI8Buckets; ++b)
            start[b + 1] = start[b] + (total[b] + kSrcPerBlock - 1) /
                    kSrcPerBlock * kSrcPerBlock;
        const int nkb = start[kI8Buckets] / kSrcPerBlock;
        int nchunk = 0;
        for (int b = 0; b < kI8Buckets; ++b)
            for (int k = start[b] / kSrcPerBlock;
                    k < start[b + 1] / kSrcPerBlock; k += drain_kb)
            {
                o.chunk_kb[nchunk] = k;
                o.chunk_bucket[nchunk] = b;
                ++nchunk;
            }
        o.chunk_kb[nchunk] = nkb;
        o.counts[0] = nkb;
        o.counts[1] = nchunk;
    }
    __syncthreads();
    // ---- pass 2: positions, round by round in source order
    for (int s0 = 0; s0 < num_src; s0 += kOrderThreads)
    {
        if (lane < kI8Buckets) wcnt[warp][lane] = 0;
        __syncthreads();
        const int s = s0 + t;
        const int b = s < num_src ? i8_bucket(o.amp_bits[s], m_bits) : -1;
        const unsigned int same = __match_any_sync(0xffffffffu, b);
        if (b >= 0 && (same & lt) == 0) wcnt[warp][b] = __popc(same);
        __syncthreads();
        // warp k < kI8Buckets: exclusive scan of bucket k over the warps
        if (warp < kI8Buckets)
        {
            const int v = wcnt[lane][warp];
            int incl = v;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1)
            {
                const int u = __shfl_up_sync(0xffffffffu, incl, d);
                if (lane >= d) incl += u;
            }
            const int base = running[warp];
            woff[lane][warp] = base + incl - v;
            __syncwarp();
            if (lane == 31) running[warp] = base + incl;
        }
        __syncthreads();
        if (b >= 0)
            o.perm[start[b] + woff[warp][b] + __popc(same & lt)] = s;
    }
    // ---- padding and the bucket of every k block
    const int npos = start[kI8Buckets];
    for (int i = t; i < npos; i += kOrderThreads)
    {
        int b = 0;
        while (i >= start[b + 1]) ++b;
        if (i >= start[b] + total[b]) o.perm[i] = -1;
        if (i % kSrcPerBlock == 0) o.kb_bucket[i / kSrcPerBlock] = b;
    }
}

// ---------------------------------------------------------------------------
// Operand image from joined Jones J (the oskar_cross_correlate input).
// grid (k blocks, row blocks, problems); 8 warps, warp = 4 stations,
// lane = source.
// ---------------------------------------------------------------------------
template <typename TJ>
__global__ void __launch_bounds__(256) prep_jones_kernel(
        const TJ* __restrict__ jones, int num_src, int num_st,
        const TJ* __restrict__ I, const TJ* __restrict__ Q,
        const TJ* __restrict__ U, const TJ* __restrict__ V,
        const unsigned int* __restrict__ maxabs_bits, uint8_t* W)
{
    const int kb = blockIdx.x, rb = blockIdx.y, nkb = gridDim.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int s = kb * kSrcPerBlock + lane;
    const bool src_ok = s < num_src;
    float c11 = 0, c21r = 0, c21i = 0, c22 = 0;
    if (src_ok) brightness_factor(I[s], Q[s], U[s], V[s], c11, c21r, c21i, c22);
    const float S = scale_from_bits(*maxabs_bits);
    uint8_t* tile = W + (size_t) (rb * nkb + kb) * kPairBytes;
    for (int pl = warp; pl < kStPerBlock; pl += 8)
    {
        const int p = rb * kStPerBlock + pl;
        float A[2][2][2] = {{{0, 0}, {0, 0}}, {{0, 0}, {0, 0}}};
        if (src_ok && p < num_st)
        {
            float J[8];
            load_jones<TJ>(jones + 8 * ((size_t) p * num_src + s), J);
            apply_factor(J, c11, c21r, c21i, c22, A);
#pragma unroll
            for (int k = 0; k < 8; ++k) (&A[0][0][0])[k] *= S;
        }
        store_entry(tile, pl, lane, A);
    }
}

// Integer image from joined Jones J: the sources in bucket order (o.perm),
// each k block scaled by its bucket's q 2^b. grid (kb cap, row blocks);
// blocks past the used k blocks return.
template <typename TJ>
__global__ void __launch_bounds__(256) prep_jones_i8_kernel(
        const TJ* __restrict__ jones, int num_src, int num_st,
        const TJ* __restrict__ I, const TJ* __restrict__ Q,
        const TJ* __restrict__ U, const TJ* __restrict__ V,
        const unsigned int* __restrict__ maxabs_bits, const I8Order o,
        uint8_t* W)
{
    const int kb = blockIdx.x, rb = blockIdx.y, nkb_cap = gridDim.x;
    if (kb >= o.counts[0]) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int s = o.perm[kb * kSrcPerBlock + lane];
    const bool src_ok = s >= 0;
    float c11 = 0, c21r = 0, c21i = 0, c22 = 0;
    if (src_ok) brightness_factor(I[s], Q[s], U[s], V[s], c11, c21r, c21i, c22);
    const float q = scalbnf(i8_scale_from_bits(*maxabs_bits),
            o.kb_bucket[kb]);
    uint8_t* tile = W + (size_t) (rb * nkb_cap + kb) * kI8Block;
    for (int pl = warp; pl < kStPerBlock; pl += 8)
    {
        const int p = rb * kStPerBlock + pl;
        float A[2][2][2] = {{{0, 0}, {0, 0}}, {{0, 0}, {0, 0}}};
        if (src_ok && p < num_st)
        {
            float J[8];
            load_jones<TJ>(jones + 8 * ((size_t) p * num_src + s), J);
            apply_factor(J, c11, c21r, c21i, c22, A);
#pragma unroll
            for (int k = 0; k < 8; ++k) (&A[0][0][0])[k] *= q;
        }
        store_entry_i8(tile, pl, lane, A);
    }
}

// ---------------------------------------------------------------------------
// Fused operand image: A = K (E C) with the interferometer phase
//   K_p(s) = exp(2 pi i x),  x = (u_p l + v_p m + w_p (n - 1)) / lambda,
// x formed in FP64 and reduced to [-1/2, 1/2] before an FP32 sincospi.
// E is FP32 or FP64 [station][source][2x2] (rounded to FP32 on load, then
// split into the 22-bit FP16 hi/lo pair), shared by every problem. Problems are
// (time, channel) pairs, prob = t * nch + c: station (u, v, w) of time t at
// uvw[t][3][num_st], 1/lambda of channel c. One launch writes the images of
// problems [p0, p0 + np) (image prob - p0 at W + (prob - p0) * image_stride),
// reading E and forming E C once per station-source for all of them.
// grid (k blocks, row blocks); 8 warps, warp = 4 stations, lane = source.
// ---------------------------------------------------------------------------
template <typename TE>
__global__ void __launch_bounds__(256) prep_fused_kernel(
        const TE* __restrict__ E, int num_src, int num_st,
        const double* __restrict__ l, const double* __restrict__ m,
        const double* __restrict__ n, const double* __restrict__ I,
        const double* __restrict__ Q, const double* __restrict__ U,
        const double* __restrict__ V, const double* __restrict__ uvw,
        const double* __restrict__ inv_wavelength, int nch, int p0, int np,
        const unsigned int* __restrict__ maxabs_bits, uint8_t* W,
        size_t image_stride)
{
    const int kb = blockIdx.x, rb = blockIdx.y;
    const int nkb = gridDim.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int s = kb * kSrcPerBlock + lane;
    const bool src_ok = s < num_src;
    float c11 = 0, c21r = 0, c21i = 0, c22 = 0;
    double sl = 0, sm = 0, sn1 = 0;
    if (src_ok)
    {
        brightness_factor(I[s], Q[s], U[s], V[s], c11, c21r, c21i, c22);
        sl = l[s]; sm = m[s]; sn1 = n[s] - 1.0;
    }
    const float S = scale_from_bits(*maxabs_bits);
    uint8_t* tile0 = W + (size_t) (rb * nkb + kb) * kPairBytes;
    for (int pl = warp; pl < kStPerBlock; pl += 8)
    {
        const int p = rb * kStPerBlock + pl;
        const bool ok = src_ok && p < num_st;
        float A0[2][2][2] = {{{0, 0}, {0, 0}}, {{0, 0}, {0, 0}}};
        if (ok)
        {
            float J[8];
            load_jones<TE>(E + 8 * ((size_t) p * num_src + s), J);
            apply_factor(J, c11, c21r, c21i, c22, A0);
#pragma unroll
            for (int k = 0; k < 8; ++k) (&A0[0][0][0])[k] *= S;
        }
        for (int j = 0; j < np; ++j)
        {
            const int prob = p0 + j, t = prob / nch, c = prob - t * nch;
            float A[2][2][2] = {{{0, 0}, {0, 0}}, {{0, 0}, {0, 0}}};
            if (ok)
            {
                const double* pu = uvw + (size_t) t * 3 * num_st;
                const double x = (pu[p] * sl + pu[num_st + p] * sm +
                                  pu[2 * num_st + p] * sn1) *
                                 inv_wavelength[c];
                const float f = (float) (x - rint(x));
                float sn, cs;
                sincospif(2.0f * f, &sn, &cs);
#pragma unroll
                for (int i = 0; i < 2; ++i)
#pragma unroll
                    for (int kk = 0; kk < 2; ++kk)
                    {
                        const float re = A0[i][kk][0], im = A0[i][kk][1];
                        A[i][kk][0] = re * cs - im * sn;
                        A[i][kk][1] = re * sn + im * cs;
                    }
            }
            store_entry(tile0 + (size_t) j * image_stride, pl, lane, A);
        }
    }
}

// ---------------------------------------------------------------------------
// Integer form of prep_fused_kernel: the same A = K (E C) per station-source
// and problem, written as the three limb tiles of the block. Each block of
// one problem (24 KB, contiguous in the image) is assembled in shared memory
// and leaves with one bulk copy, double-buffered so that the copy of one
// problem's block overlaps forming the next. A thread keeps E C of its four
// stations (8 values each) in registers across the problems.
// grid (k blocks, row blocks); 8 warps, warp = 4 stations, lane = source.
// ---------------------------------------------------------------------------
template <typename TE>
__global__ void __launch_bounds__(256, 4) prep_fused_i8_kernel(
        const TE* __restrict__ E, int num_src, int num_st,
        const double* __restrict__ l, const double* __restrict__ m,
        const double* __restrict__ n, const double* __restrict__ I,
        const double* __restrict__ Q, const double* __restrict__ U,
        const double* __restrict__ V, const double* __restrict__ uvw,
        const double* __restrict__ inv_wavelength, int nch, int p0, int np,
        const unsigned int* __restrict__ maxabs_bits, const I8Order o,
        uint8_t* W, size_t image_stride)
{
    // two blocks: the 48 KB of static shared memory a kernel may declare
    __shared__ __align__(128) uint8_t buf[2 * kI8Block];
    const int kb = blockIdx.x, rb = blockIdx.y;
    const int nkb = gridDim.x;
    if (kb >= o.counts[0]) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int s = o.perm[kb * kSrcPerBlock + lane];
    const bool src_ok = s >= 0;
    float c11 = 0, c21r = 0, c21i = 0, c22 = 0;
    double sl = 0, sm = 0, sn1 = 0;
    if (src_ok)
    {
        brightness_factor(I[s], Q[s], U[s], V[s], c11, c21r, c21i, c22);
        sl = l[s]; sm = m[s]; sn1 = n[s] - 1.0;
    }
    const float q = scalbnf(i8_scale_from_bits(*maxabs_bits),
            o.kb_bucket[kb]);
    float A0[4][2][2][2];
#pragma unroll
    for (int k = 0; k < 4; ++k)
    {
        const int p = rb * kStPerBlock + warp + 8 * k;
        float* a = &A0[k][0][0][0];
#pragma unroll
        for (int e = 0; e < 8; ++e) a[e] = 0.0f;
        if (src_ok && p < num_st)
        {
            float J[8];
            load_jones<TE>(E + 8 * ((size_t) p * num_src + s), J);
            apply_factor(J, c11, c21r, c21i, c22, A0[k]);
#pragma unroll
            for (int e = 0; e < 8; ++e) a[e] *= q;
        }
    }
    uint8_t* dst0 = W + (size_t) (rb * nkb + kb) * kI8Block;
    // u l + v m + w (n - 1) of the thread's four stations at dump t_cur
    // (the channels of one dump share it)
    double base[4] = {0.0, 0.0, 0.0, 0.0};
    int t_cur = -1;
    for (int j = 0; j < np; ++j)
    {
        uint8_t* b = buf + (size_t) (j & 1) * kI8Block;
        if (j >= 2)
        {
            // the copy that read this buffer (problem j - 2) is done
            if (threadIdx.x == 0) ptx::bulk_wait_read<1>();
            __syncthreads();
        }
        const int prob = p0 + j, t = prob / nch, c = prob - t * nch;
        if (t != t_cur)
        {
            t_cur = t;
            const double* pu = uvw + (size_t) t * 3 * num_st;
#pragma unroll
            for (int k = 0; k < 4; ++k)
            {
                const int p = rb * kStPerBlock + warp + 8 * k;
                base[k] = (src_ok && p < num_st) ? pu[p] * sl +
                        pu[num_st + p] * sm + pu[2 * num_st + p] * sn1 : 0.0;
            }
        }
        const double kw = inv_wavelength[c];
#pragma unroll
        for (int k = 0; k < 4; ++k)
        {
            const int pl = warp + 8 * k;
            const int p = rb * kStPerBlock + pl;
            float A[2][2][2] = {{{0, 0}, {0, 0}}, {{0, 0}, {0, 0}}};
            if (src_ok && p < num_st)
            {
                const double x = base[k] * kw;
                const float f = (float) (x - rint(x));
                float sn, cs;
                sincospif(2.0f * f, &sn, &cs);
#pragma unroll
                for (int i = 0; i < 2; ++i)
#pragma unroll
                    for (int kk = 0; kk < 2; ++kk)
                    {
                        const float re = A0[k][i][kk][0];
                        const float im = A0[k][i][kk][1];
                        A[i][kk][0] = re * cs - im * sn;
                        A[i][kk][1] = re * sn + im * cs;
                    }
            }
            store_entry_i8(b, pl, lane, A);
        }
        ptx::fence_proxy_async_smem();
        __syncthreads();
        if (threadIdx.x == 0)
        {
            ptx::bulk_s2g(dst0 + (size_t) j * image_stride, b, kI8Block);
            ptx::bulk_commit();
        }
    }
    if (threadIdx.x == 0) ptx::bulk_wait<0>();
}

}  // namespace tc
}  // namespace oskb

// ===========================================================================
// G = W W^T on the tensor cores, upper block triangle, fused visibility
// epilogue. Persistent CTAs (one per SM) walk the task list
//     task = problem * ntile + tile,  tile -> (rb <= cb)
// Warp roles (320 threads):
//   warp 0 (one lane): bulk copies of the A (row block rb) and B (row block
//     cb) hi/lo tile pairs into a kStages-deep shared-memory ring;
//   warp 1 (one lane): issues the tcgen05 MMAs (3 products per 16-wide k
//     step) into one of two TMEM buffers, each a pair of 128-column FP32
//     accumulators (hi hi^T, and hi lo^T + lo hi^T);
//   warps 2-9: drain the accumulator every drain_kb k-blocks into FP64
//     registers (one TMEM lane = one row of G, 64 columns per warp), then
//     form the four polarisations and add them into vis.
// ===========================================================================
namespace oskb {
namespace tc {

constexpr int kStages = 3;
constexpr int kStageBytes = 2 * kPairBytes;   // A pair + B pair
constexpr int kGemmThreads = 320;
constexpr int kAccCols = 128;                 // one FP32 accumulator
constexpr int kBufCols = 2 * kAccCols;        // main + correction
constexpr uint32_t kTmemCols = 2 * kBufCols;  // double-buffered: all 512

struct GemmParams
{
    const uint8_t* W;
    size_t image_stride;        // bytes per problem
    int nrb, nkb, num_problems, num_st;
    int drain_kb;
    const unsigned int* maxabs_bits;
    int maxabs_stride;          // 0: one scale for all problems
    // Problem j of this launch is global problem g = prob0 + j of a
    // (time, channel) block, g = t * nch + c.
    int prob0, nch;
    double* vis;                // vis of global problem g at
    size_t vis_stride;          //   vis + 8 * (g * vis_stride + offset_out)
    int offset_out;
    const double* st_u;         // station u, v (metres) of time t at
    const double* st_v;         //   st_u + t * uv_stride, st_v + ...
    size_t uv_stride;
    const double* inv_wavelength;  // [nch], or NULL: use kw_scalar
    double kw_scalar;
    double uv_min, uv_max;
    int casa;
    int i8;                     // operand image is the three-limb integer one
    // integer image only: k blocks used (i8_counts[0]), chunks
    // (i8_counts[1]) and the chunk table (I8Order); nkb is then the image's
    // k-block capacity (its row-block stride)
    const int* i8_counts;
    const int* i8_chunk_kb;
    const int* i8_chunk_bucket;
    int form;                   // Form (kFormDefault: the environment's)
    // six-limb form only: when set and bit 0 of *skip_flags is set (a
    // brightness matrix was not positive semi-definite), the contraction
    // adds nothing
    const int* skip_flags = nullptr;
    int* err;
    // Auto-correlations (optional): the diagonal station pairs of the
    // diagonal tiles, V_pp = J_p B J_p^H, added into
    // autos[(g * num_st + p) * 8 + 2 x 2] for global problem g; NULL: none.
    double* autos;
};

struct GemmCtl
{
    uint64_t full[kStages], empty[kStages], tfull[2], tempty[2], done;
    uint32_t tmem_base;
    int abort;
};

constexpr size_t gemm_smem_bytes()
{
    return 1024 + (size_t) kStages * kStageBytes + sizeof(GemmCtl);
}

__device__ __forceinline__ void tile_of(int t, int& rb, int& cb)
{
    int c = (int) ((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
    while ((c + 1) * (c + 2) / 2 <= t) ++c;
    while (c * (c + 1) / 2 > t) --c;
    cb = c;
    rb = t - c * (c + 1) / 2;
}

// Visibilities of one task from the FP64 sums of the thread's NQ column
// stations: row `row` of row block rb against column stations q_first ..
// q_first + NQ - 1 of column block cb; scaled by inv_s2.
template <int NQ>
__device__ __forceinline__ void task_store(const GemmParams& prm,
        const double (&accR)[NQ], const double (&accI)[NQ], double inv_s2,
        int row, int q_first, int prob, int rb, int cb)
{
    const int c = row & 1;
    const int g = prm.prob0 + prob, t = g / prm.nch;
    const int chan = g - t * prm.nch;
    const int i = (row >> 1) & 1;
    const int p = rb * kStPerBlock + (row >> 2);
    const int N = prm.num_st;
    const double* su = prm.st_u + prm.uv_stride * t;
    const double* sv = prm.st_v + prm.uv_stride * t;
    const double kw = prm.inv_wavelength ? prm.inv_wavelength[chan]
                                          : prm.kw_scalar;
    double* vbase = prm.vis + 8 * ((size_t) g * prm.vis_stride +
            (size_t) prm.offset_out);
    if (prm.autos && rb == cb && p < N)
    {
        // column station q = p of this thread's NQ: V_pp[i][c]
        const int ql = p - cb * kStPerBlock - q_first;
#pragma unroll
        for (int k = 0; k < NQ; ++k)
            if (k == ql)
            {
                double* o = prm.autos + 8 * ((size_t) g * N + p) +
                        2 * (2 * i + c);
                o[0] += accR[k] * inv_s2;
                o[1] += accI[k] * inv_s2;
            }
    }
#pragma unroll
    for (int ql = 0; ql < NQ; ++ql)
    {
        const int q = cb * kStPerBlock + q_first + ql;
        if (p < q && q < N)
        {
            const double uu = (su[p] - su[q]) * kw;
            const double vv = (sv[p] - sv[q]) * kw;
            const double len = sqrt(uu * uu + vv * vv);
            if (!(len < prm.uv_min || len > prm.uv_max))
            {
                const double re = accR[ql] * inv_s2;
                const double im = accI[ql] * inv_s2;
                // this thread holds V_pq[i][j] with j = c; the
                // reference stores J_q B J_p^H (p < q) unless CASA
                const int ro = prm.casa ? i : c;
                const int co = prm.casa ? c : i;
                double* o = vbase + 8 * (size_t) baseline_index(N, q, p)
                        + 2 * (2 * ro + co);
                o[0] += re;
                o[1] += prm.casa ? im : -im;
            }
        }
    }
}

// task_store for a square (128 x 128) task: the thread's 16 column
// stations of column half h.
__device__ __forceinline__ void square_task_store(const GemmParams& prm,
        const double (&accR)[16], const double (&accI)[16], double inv_s2,
        int row, int h, int prob, int rb, int cb)
{
    task_store<16>(prm, accR, accI, inv_s2, row, 16 * h, prob, rb, cb);
}

__global__ void __launch_bounds__(kGemmThreads, 1)
gemm_kernel(const GemmParams prm)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(
            (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t) 1023);
    GemmCtl* ctl = reinterpret_cast<GemmCtl*>(smem + kStages * kStageBytes);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    volatile int* abort = &ctl->abort;

    if (threadIdx.x == 0)
    {
        for (int s = 0; s < kStages; ++s)
        {
            ptx::mbar_init(&ctl->full[s], 1);
            ptx::mbar_init(&ctl->empty[s], 1);
        }
        for (int b = 0; b < 2; ++b)
        {
            ptx::mbar_init(&ctl->tfull[b], 1);
            ptx::mbar_init(&ctl->tempty[b], 8);
        }
        ptx::mbar_init(&ctl->done, 1);
        ctl->abort = 0;
        ptx::fence_mbar_init();
    }
    if (warp == 1) ptx::tmem_alloc(&ctl->tmem_base, kTmemCols);
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    const uint32_t tmem = ctl->tmem_base;

    const int ntile = prm.nrb * (prm.nrb + 1) / 2;
    const int ntasks = ntile * prm.num_problems;
    const int nchunk = (prm.nkb + prm.drain_kb - 1) / prm.drain_kb;

    if (warp == 0)
    {
        if (lane == 0)
        {
            // ---------------- producer
            int stage = 0;
            uint32_t phase = 0;
            uint32_t issued = 0, issued_par = 0;  // bit s: stage s
            for (int task = blockIdx.x; task < ntasks && !*abort;
                    task += gridDim.x)
            {
                const int prob = task / ntile;
                int rb, cb;
                tile_of(task - prob * ntile, rb, cb);
                const bool diag = rb == cb;
                const uint8_t* img = prm.W + (size_t) prob * prm.image_stride;
                for (int kb = 0; kb < prm.nkb; ++kb)
                {
                    if (!ptx::mbar_wait(&ctl->empty[stage], phase ^ 1,
                            prm.err, 11, abort))
                        break;
                    uint8_t* dst = smem + (size_t) stage * kStageBytes;
                    ptx::mbar_arrive_expect_tx(&ctl->full[stage],
                            diag ? kPairBytes : 2 * kPairBytes);
                    ptx::bulk_g2s(dst, img + ((size_t) rb * prm.nkb + kb) *
                            kPairBytes, kPairBytes, &ctl->full[stage]);
                    if (!diag)
                        ptx::bulk_g2s(dst + kPairBytes, img +
                                ((size_t) cb * prm.nkb + kb) * kPairBytes,
                                kPairBytes, &ctl->full[stage]);
                    issued |= 1u << stage;
                    issued_par = (issued_par & ~(1u << stage)) |
                            (phase << stage);
                    if (++stage == kStages) { stage = 0; phase ^= 1; }
                }
            }
            // Copies still in flight must land before the CTA can exit.
            for (int s = 0; s < kStages; ++s)
                if ((issued >> s) & 1)
                    ptx::mbar_wait(&ctl->full[s], (issued_par >> s) & 1,
                            prm.err, 12, abort);
        }
        __syncwarp();
    }
    else if (warp == 1)
    {
        if (lane == 0)
        {
            // ---------------- MMA issuer
            // hi hi^T and hi lo^T in one N = 256 MMA: the B hi and lo tiles
            // are consecutive in shared memory, so they form one 256-row
            // operand whose result columns land in the main (0-127) and
            // correction (128-255) accumulators of the buffer.
            const uint32_t idesc2 = ptx::idesc_f16_f32(128, 2 * kAccCols);
            const uint32_t idesc = ptx::idesc_f16_f32(128, kAccCols);
            int stage = 0;
            uint32_t phase = 0, tpar = 0;  // tpar bit b: use parity of buf b
            int buf = 0;
            bool ok = true;
            for (int task = blockIdx.x; task < ntasks && ok;
                    task += gridDim.x)
            {
                const int prob = task / ntile;
                int rb, cb;
                tile_of(task - prob * ntile, rb, cb);
                const bool diag = rb == cb;
                for (int ch = 0; ch < nchunk && ok; ++ch)
                {
                    if (!ptx::mbar_wait(&ctl->tempty[buf],
                            ((tpar >> buf) & 1) ^ 1, prm.err, 13, abort))
                    {
                        ok = false;
                        break;
                    }
                    ptx::tc_fence_after();
                    const uint32_t d = tmem + (uint32_t) (buf * kBufCols);
                    const uint32_t dc = d + kAccCols;
                    const int kb0 = ch * prm.drain_kb;
                    const int kb1 = min(prm.nkb, kb0 + prm.drain_kb);
                    for (int kb = kb0; kb < kb1; ++kb)
                    {
                        if (!ptx::mbar_wait(&ctl->full[stage], phase, prm.err,
                                14, abort))
                        {
                            ok = false;
                            break;
                        }
                        ptx::tc_fence_after();
                        const uint32_t a = ptx::smem_u32(smem +
                                (size_t) stage * kStageBytes);
                        const uint32_t b = diag ? a : a + kPairBytes;
#pragma unroll
                        for (int k = 0; k < kKSteps; ++k)
                        {
                            const uint64_t ah = ptx::sdesc_sw128(a + 32 * k);
                            const uint64_t al = ptx::sdesc_sw128(
                                    a + kTileBytes + 32 * k);
                            const uint64_t bh = ptx::sdesc_sw128(b + 32 * k);
                            const uint32_t acc =
                                    (kb > kb0 || k > 0) ? 1u : 0u;
                            ptx::mma_f16(d, ah, bh, idesc2, acc);
                            ptx::mma_f16(dc, al, bh, idesc, 1u);
                        }
                        ptx::mma_commit(&ctl->empty[stage]);
                        if (++stage == kStages) { stage = 0; phase ^= 1; }
                    }
                    if (!ok) break;
                    ptx::mma_commit(&ctl->tfull[buf]);
                    tpar ^= 1u << buf;
                    buf ^= 1;
                }
            }
            // All issued MMAs must finish before TMEM is released.
            ptx::mma_commit(&ctl->done);
            ptx::mbar_wait(&ctl->done, 0, prm.err, 15, abort);
        }
        __syncwarp();
    }
    else
    {
        // ---------------- epilogue: 8 warps
        const int q4 = warp & 3;          // TMEM lane quadrant of this warp
        const int h = (warp - 2) >> 2;    // column half
        const int row = 32 * q4 + lane;   // row of the G tile
        const uint32_t taddr = tmem + ((uint32_t) (32 * q4) << 16) +
                (uint32_t) (64 * h);
        int buf = 0;
        uint32_t tpar = 0;
        bool ok = true;
        for (int task = blockIdx.x; task < ntasks && ok; task += gridDim.x)
        {
            const int prob = task / ntile;
            int rb, cb;
            tile_of(task - prob * ntile, rb, cb);
            // FP64 sums of Re V (accR) and Im V (accI) of the 16 baselines
            // (station columns) this thread owns: thread (row c) keeps the
            // polarisation j = c of its row's pair.
            const int c = row & 1;
            double accR[16], accI[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) accR[j] = accI[j] = 0.0;
            for (int ch = 0; ch < nchunk; ++ch)
            {
                if (!ptx::mbar_wait(&ctl->tfull[buf], (tpar >> buf) & 1,
                        prm.err, 16, abort))
                {
                    ok = false;
                    break;
                }
                ptx::tc_fence_after();
                const uint32_t ta = taddr + (uint32_t) (buf * kBufCols);
#pragma unroll
                for (int j0 = 0; j0 < 64; j0 += 16)
                {
                    uint32_t vm[16], vc[16];
                    ptx::tmem_ld16(ta + j0, vm);
                    ptx::tmem_ld16(ta + kAccCols + j0, vc);
                    ptx::tmem_ld_wait();
                    float v[16];
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                        v[j] = __uint_as_float(vm[j]) + __uint_as_float(vc[j]);
                    // Re V = G00 + G11, Im V = G10 - G01 (rows c = 0, 1 of
                    // the pair are lanes l, l ^ 1; columns 2j + c' of the
                    // group of four): combined in FP32 before the FP64
                    // accumulation, which halves the FP32 -> FP64
                    // conversions of the drain.
#pragma unroll
                    for (int qq = 0; qq < 4; ++qq)
                    {
                        const int jb = 4 * qq;
                        const float s0 = c ? v[jb + 0] : v[jb + 2];
                        const float s1 = c ? v[jb + 1] : v[jb + 3];
                        const float r0 = __shfl_xor_sync(0xffffffffu, s0, 1);
                        const float r1 = __shfl_xor_sync(0xffffffffu, s1, 1);
                        const float g00 = c ? r0 : v[jb + 0];
                        const float g01 = c ? r1 : v[jb + 1];
                        const float g10 = c ? v[jb + 2] : r0;
                        const float g11 = c ? v[jb + 3] : r1;
                        accR[j0 / 4 + qq] += (double) (g00 + g11);
                        accI[j0 / 4 + qq] += (double) (g10 - g01);
                    }
                }
                ptx::tc_fence_before();
                __syncwarp();
                if (lane == 0) ptx::mbar_arrive(&ctl->tempty[buf]);
                tpar ^= 1u << buf;
                buf ^= 1;
            }
            if (!ok) break;
            // ---- visibilities of this tile
            const int g = prm.prob0 + prob;
            const float S = scale_from_bits(
                    prm.maxabs_bits[prm.maxabs_stride * g]);
            const double inv_s2 = 1.0 / ((double) S * (double) S);
            square_task_store(prm, accR, accI, inv_s2, row, h, prob, rb, cb);
        }
    }

    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    if (warp == 1) ptx::tmem_dealloc(tmem, kTmemCols);
}

// ===========================================================================
// Wide tiles: 128 rows x 256 columns of G per task (row block rb, column
// blocks 2 cp and 2 cp + 1), so every A tile pair loaded feeds twice the
// products of the 128 x 128 kernel: 96 KB of operands per k block for six
// 128x128x64 products, where the square tiles load 64 KB for three. The
// contraction is bound by how fast operands reach shared memory, so fewer
// bytes per product is the lever.
// TMEM holds a 256-column main accumulator (hi hi^T) and a 256-column
// correction accumulator (hi lo^T + lo hi^T), both single-buffered. The
// main accumulator is drained every drain_kb k blocks; while it drains, the
// MMA issuer already issues the next k block's correction products, and
// only then waits for the main accumulator. The correction accumulator
// (2^-11 of the main one) is drained every kCorrPeriods main drains and at
// the end of each task.
// Warp roles: warpgroup 0 = producer (warp 0), MMA issuer (warp 1) and two
// other warps, all releasing registers down to kWLowRegs; warpgroups 1 and
// 2 = eight epilogue warps of 128 columns each, raised to kWHighRegs so that
// the 64 FP64 sums per thread and two 32-column TMEM loads stay in
// registers. Budget: 128 x kWLowRegs + 256 x kWHighRegs must not exceed the
// 384 x (registers per thread at launch) the block starts with; the host
// checks the compiled count before the first launch.
// ===========================================================================
constexpr int kWThreads = 384;
constexpr int kWEpiWarps = 8;
constexpr int kWEpiCols = 128;                // columns per epilogue thread
constexpr int kWLowRegs = 72;
constexpr int kWHighRegs = 216;
constexpr int kWStages = 2;
constexpr int kWStageBytes = 3 * kPairBytes;  // A pair + B hi x2 + B lo x2
constexpr int kWCols = 256;                   // one accumulator
constexpr uint32_t kWTmemCols = 512;          // main + correction
constexpr int kCorrPeriods = 8;

struct WideCtl
{
    uint64_t full[kWStages], empty[kWStages], mfull, mempty, cfull, cempty,
            done;
    uint32_t tmem_base;
    int abort;
};

constexpr size_t gemm_wide_smem_bytes()
{
    return 1024 + (size_t) kWStages * kWStageBytes + sizeof(WideCtl);
}

// Wide task t of one problem -> (rb, cp): column pair cp holds the tasks
// [cp (cp + 1), cp (cp + 1) + 2 cp + 2), rb = t - cp (cp + 1) (the last pair
// of an odd number of row blocks holds 2 cp + 1 of them).
__device__ __forceinline__ void wide_tile_of(int t, int& rb, int& cp)
{
    int c = (int) ((sqrt(4.0 * t + 1.0) - 1.0) * 0.5);
    while ((c + 1) * (c + 2) <= t) ++c;
    while (c * (c + 1) > t) --c;
    cp = c;
    rb = t - c * (c + 1);
}

__host__ __device__ inline int wide_tiles(int nrb)
{
    int n = 0;
    for (int cp = 0; 2 * cp < nrb; ++cp)
        n += (2 * cp + 2 < nrb) ? 2 * cp + 2 : nrb;
    return n;
}

__device__ __forceinline__ bool corr_drain_at(int ch, int nchunk)
{
    return (ch % kCorrPeriods) == kCorrPeriods - 1 || ch == nchunk - 1;
}

// ---------------------------------------------------------------------------
// Epilogue of one wide or pair task, run by each of the eight epilogue
// warps. The thread's TMEM lane is row `row` of the task's 128-row block;
// its 128 columns (taddr) are 32 stations x (polarisation j, part c') of G.
// Every drain loads them (32 columns per TMEM load; 16 main and 16
// correction columns when the correction accumulator is due), folds each
// group of four into the real and imaginary parts of this thread's
// visibility (Re V = G00 + G11, Im V = G10 - G01 across the row pair, lanes
// l and l ^ 1) in FP32 and adds those into FP64 sums: the cross-tile sum is
// FP64. At the end of the task the sums are scaled and added into vis (and
// autos). Returns false if a bounded wait expired.
// ---------------------------------------------------------------------------
template <class Arrive>
__device__ __forceinline__ bool wide_task_epilogue(const GemmParams& prm,
        uint64_t* mfull, uint64_t* cfull, uint32_t& mpar, uint32_t& cpar,
        volatile int* abort, uint32_t taddr, int row, int lane, int prob,
        int rb, int q0, int nchunk, Arrive arrive)
{
    const int c = row & 1;
    double accR[32], accI[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) accR[j] = accI[j] = 0.0;
    for (int ch = 0; ch < nchunk; ++ch)
    {
        const bool with_corr = corr_drain_at(ch, nchunk);
        if (!ptx::mbar_wait(mfull, mpar, prm.err, 27, abort) ||
                (with_corr && !ptx::mbar_wait(cfull, cpar, prm.err, 28,
                abort)))
            return false;
        ptx::tc_fence_after();
#define OSKB_WIDE_FOLD(V, J0, NQ)                                              \
        _Pragma("unroll")                                                      \
        for (int qq = 0; qq < (NQ); ++qq)                                      \
        {                                                                      \
            const int jb = 4 * qq;                                             \
            const float s0 = c ? V[jb + 0] : V[jb + 2];                        \
            const float s1 = c ? V[jb + 1] : V[jb + 3];                        \
            const float r0 = __shfl_xor_sync(0xffffffffu, s0, 1);              \
            const float r1 = __shfl_xor_sync(0xffffffffu, s1, 1);              \
            const float g00 = c ? r0 : V[jb + 0];                              \
            const float g01 = c ? r1 : V[jb + 1];                              \
            const float g10 = c ? V[jb + 2] : r0;                              \
            const float g11 = c ? V[jb + 3] : r1;                              \
            accR[(J0) / 4 + qq] += (double) (g00 + g11);                       \
            accI[(J0) / 4 + qq] += (double) (g10 - g01);                       \
        }
        if (!with_corr)
        {
#pragma unroll
            for (int j0 = 0; j0 < 128; j0 += 32)
            {
                uint32_t va[32];
                ptx::tmem_ld32(taddr + j0, va);
                ptx::tmem_ld_wait();
                float v[32];
#pragma unroll
                for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(va[j]);
                OSKB_WIDE_FOLD(v, j0, 8)
            }
        }
        else
        {
#pragma unroll
            for (int j0 = 0; j0 < 128; j0 += 16)
            {
                uint32_t va[16], vb[16];
                ptx::tmem_ld16(taddr + j0, va);
                ptx::tmem_ld16(taddr + kWCols + j0, vb);
                ptx::tmem_ld_wait();
                float v[16];
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    v[j] = __uint_as_float(va[j]) + __uint_as_float(vb[j]);
                OSKB_WIDE_FOLD(v, j0, 4)
            }
        }
#undef OSKB_WIDE_FOLD
        ptx::tc_fence_before();
        __syncwarp();
        if (lane == 0) arrive(with_corr);
        mpar ^= 1;
        if (with_corr) cpar ^= 1;
    }
    // ---- visibilities of this thread's row of the tile
    const int g = prm.prob0 + prob, t = g / prm.nch;
    const int chan = g - t * prm.nch;
    const float S = scale_from_bits(prm.maxabs_bits[prm.maxabs_stride * g]);
    const double inv_s2 = 1.0 / ((double) S * (double) S);
    const int i = (row >> 1) & 1;
    const int p = rb * kStPerBlock + (row >> 2);
    const int N = prm.num_st;
    const double* su = prm.st_u + prm.uv_stride * t;
    const double* sv = prm.st_v + prm.uv_stride * t;
    const double kw = prm.inv_wavelength ? prm.inv_wavelength[chan]
                                          : prm.kw_scalar;
    double* vbase = prm.vis + 8 * ((size_t) g * prm.vis_stride +
            (size_t) prm.offset_out);
    if (prm.autos && p < N)
    {
        // the column station q = p, where this thread's 32 hold it
        const int ql = p - q0;
#pragma unroll
        for (int k = 0; k < 32; ++k)
            if (k == ql)
            {
                double* o = prm.autos + 8 * ((size_t) g * N + p) +
                        2 * (2 * i + c);
                o[0] += accR[k] * inv_s2;
                o[1] += accI[k] * inv_s2;
            }
    }
#pragma unroll
    for (int ql = 0; ql < 32; ++ql)
    {
        const int q = q0 + ql;
        if (p < q && q < N)
        {
            const double uu = (su[p] - su[q]) * kw;
            const double vv = (sv[p] - sv[q]) * kw;
            const double len = sqrt(uu * uu + vv * vv);
            if (!(len < prm.uv_min || len > prm.uv_max))
            {
                const double re = accR[ql] * inv_s2;
                const double im = accI[ql] * inv_s2;
                // this thread holds V_pq[i][j] with j = c; the reference
                // stores J_q B J_p^H (p < q) unless CASA
                const int ro = prm.casa ? i : c;
                const int co = prm.casa ? c : i;
                double* o = vbase + 8 * (size_t) baseline_index(N, q, p) +
                        2 * (2 * ro + co);
                o[0] += re;
                o[1] += prm.casa ? im : -im;
            }
        }
    }
    return true;
}

__global__ void __launch_bounds__(kWThreads, 1)
gemm_wide_kernel(const GemmParams prm)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(
            (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t) 1023);
    WideCtl* ctl = reinterpret_cast<WideCtl*>(smem + kWStages * kWStageBytes);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    volatile int* abort = &ctl->abort;

    if (threadIdx.x == 0)
    {
        for (int s = 0; s < kWStages; ++s)
        {
            ptx::mbar_init(&ctl->full[s], 1);
            ptx::mbar_init(&ctl->empty[s], 1);
        }
        ptx::mbar_init(&ctl->mfull, 1);
        ptx::mbar_init(&ctl->mempty, kWEpiWarps);
        ptx::mbar_init(&ctl->cfull, 1);
        ptx::mbar_init(&ctl->cempty, kWEpiWarps);
        ptx::mbar_init(&ctl->done, 1);
        ctl->abort = 0;
        ptx::fence_mbar_init();
    }
    if (warp == 1) ptx::tmem_alloc(&ctl->tmem_base, kWTmemCols);
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    const uint32_t tmem = ctl->tmem_base;

    const int ntile = wide_tiles(prm.nrb);
    const int ntasks = ntile * prm.num_problems;
    const int nchunk = (prm.nkb + prm.drain_kb - 1) / prm.drain_kb;

    if (warp < 4)
    {
    ptx::regs_release<kWLowRegs>();
    if (warp == 0)
    {
        if (lane == 0)
        {
            // ---------------- producer: A pair, then the hi tiles of both
            // column blocks (one 256-row operand), then their lo tiles
            int stage = 0;
            uint32_t phase = 0;
            uint32_t issued = 0, issued_par = 0;  // bit s: stage s
            for (int task = blockIdx.x; task < ntasks && !*abort;
                    task += gridDim.x)
            {
                const int prob = task / ntile;
                int rb, cp;
                wide_tile_of(task - prob * ntile, rb, cp);
                const int cb0 = 2 * cp;
                // an odd last column block: its partner repeats it (the
                // columns are discarded by the q < N test)
                const int cb1 = cb0 + 1 < prm.nrb ? cb0 + 1 : cb0;
                const uint8_t* img = prm.W + (size_t) prob * prm.image_stride;
                for (int kb = 0; kb < prm.nkb; ++kb)
                {
                    if (!ptx::mbar_wait(&ctl->empty[stage], phase ^ 1,
                            prm.err, 21, abort))
                        break;
                    uint8_t* dst = smem + (size_t) stage * kWStageBytes;
                    const uint8_t* a = img + ((size_t) rb * prm.nkb + kb) *
                            kPairBytes;
                    const uint8_t* b0 = img + ((size_t) cb0 * prm.nkb + kb) *
                            kPairBytes;
                    const uint8_t* b1 = img + ((size_t) cb1 * prm.nkb + kb) *
                            kPairBytes;
                    ptx::mbar_arrive_expect_tx(&ctl->full[stage],
                            kWStageBytes);
                    ptx::bulk_g2s(dst, a, kPairBytes, &ctl->full[stage]);
                    ptx::bulk_g2s(dst + kPairBytes, b0, kTileBytes,
                            &ctl->full[stage]);
                    ptx::bulk_g2s(dst + kPairBytes + kTileBytes, b1,
                            kTileBytes, &ctl->full[stage]);
                    ptx::bulk_g2s(dst + 2 * kPairBytes, b0 + kTileBytes,
                            kTileBytes, &ctl->full[stage]);
                    ptx::bulk_g2s(dst + 2 * kPairBytes + kTileBytes,
                            b1 + kTileBytes, kTileBytes, &ctl->full[stage]);
                    issued |= 1u << stage;
                    issued_par = (issued_par & ~(1u << stage)) |
                            (phase << stage);
                    if (++stage == kWStages) { stage = 0; phase ^= 1; }
                }
            }
            for (int s = 0; s < kWStages; ++s)
                if ((issued >> s) & 1)
                    ptx::mbar_wait(&ctl->full[s], (issued_par >> s) & 1,
                            prm.err, 22, abort);
        }
        __syncwarp();
    }
    else if (warp == 1)
    {
        if (lane == 0)
        {
            // ---------------- MMA issuer
            const uint32_t idesc = ptx::idesc_f16_f32(128, kWCols);
            const uint32_t dm = tmem, dcr = tmem + kWCols;
            int stage = 0;
            uint32_t phase = 0, mpar = 0, cpar = 0;
            bool ok = true;
            for (int task = blockIdx.x; task < ntasks && ok;
                    task += gridDim.x)
            {
                for (int ch = 0; ch < nchunk && ok; ++ch)
                {
                    const bool fresh = (ch % kCorrPeriods) == 0;
                    if (fresh)
                    {
                        if (!ptx::mbar_wait(&ctl->cempty, cpar ^ 1, prm.err,
                                23, abort))
                        {
                            ok = false;
                            break;
                        }
                        ptx::tc_fence_after();
                    }
                    const int kb0 = ch * prm.drain_kb;
                    const int kb1 = min(prm.nkb, kb0 + prm.drain_kb);
                    for (int kb = kb0; kb < kb1; ++kb)
                    {
                        if (!ptx::mbar_wait(&ctl->full[stage], phase, prm.err,
                                24, abort))
                        {
                            ok = false;
                            break;
                        }
                        ptx::tc_fence_after();
                        const uint32_t a = ptx::smem_u32(smem +
                                (size_t) stage * kWStageBytes);
                        const uint32_t al = a + kTileBytes;
                        const uint32_t bh = a + kPairBytes;
                        const uint32_t bl = a + 2 * kPairBytes;
                        // correction products first: they do not need the
                        // main accumulator, which may still be draining
#pragma unroll
                        for (int k = 0; k < kKSteps; ++k)
                        {
                            const uint32_t first =
                                    (fresh && kb == kb0 && k == 0) ? 0u : 1u;
                            ptx::mma_f16(dcr, ptx::sdesc_sw128(a + 32 * k),
                                    ptx::sdesc_sw128(bl + 32 * k), idesc,
                                    first);
                            ptx::mma_f16(dcr, ptx::sdesc_sw128(al + 32 * k),
                                    ptx::sdesc_sw128(bh + 32 * k), idesc, 1u);
                        }
                        if (kb == kb0)
                        {
                            if (!ptx::mbar_wait(&ctl->mempty, mpar ^ 1,
                                    prm.err, 25, abort))
                            {
                                ok = false;
                                break;
                            }
                            ptx::tc_fence_after();
                        }
#pragma unroll
                        for (int k = 0; k < kKSteps; ++k)
                            ptx::mma_f16(dm, ptx::sdesc_sw128(a + 32 * k),
                                    ptx::sdesc_sw128(bh + 32 * k), idesc,
                                    (kb > kb0 || k > 0) ? 1u : 0u);
                        ptx::mma_commit(&ctl->empty[stage]);
                        if (++stage == kWStages) { stage = 0; phase ^= 1; }
                    }
                    if (!ok) break;
                    ptx::mma_commit(&ctl->mfull);
                    mpar ^= 1;
                    if (corr_drain_at(ch, nchunk))
                    {
                        ptx::mma_commit(&ctl->cfull);
                        cpar ^= 1;
                    }
                }
            }
            ptx::mma_commit(&ctl->done);
            ptx::mbar_wait(&ctl->done, 0, prm.err, 26, abort);
        }
        __syncwarp();
    }
    }  // warpgroup 0
    else
    {
        // ---------------- epilogue warps (4 and up), kWEpiCols columns each
        ptx::regs_request<kWHighRegs>();
        const int q4 = warp & 3;          // TMEM lane quadrant of this warp
        const int h = (warp - 4) >> 2;    // column slice
        const int row = 32 * q4 + lane;   // row of the G tile
        const uint32_t taddr = tmem + ((uint32_t) (32 * q4) << 16) +
                (uint32_t) (kWEpiCols * h);
        uint32_t mpar = 0, cpar = 0;
        auto arrive = [&](bool with_corr) {
            ptx::mbar_arrive(&ctl->mempty);
            if (with_corr) ptx::mbar_arrive(&ctl->cempty);
        };
        for (int task = blockIdx.x; task < ntasks; task += gridDim.x)
        {
            const int prob = task / ntile;
            int rb, cp;
            wide_tile_of(task - prob * ntile, rb, cp);
            if (!wide_task_epilogue(prm, &ctl->mfull, &ctl->cfull, mpar,
                    cpar, abort, taddr, row, lane, prob, rb,
                    2 * cp * kStPerBlock + (kWEpiCols / 4) * h, nchunk,
                    arrive))
                break;
        }
    }

    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    if (warp == 1) ptx::tmem_dealloc(tmem, kWTmemCols);
}

// ===========================================================================
// Pair tiles: two CTAs of a cluster (cta_group::2) compute one 256 x 256
// tile of G: row blocks 2i and 2i + 1 (one per CTA) against column blocks
// 2j and 2j + 1 (i <= j). Each CTA brings only its own row block (A) and
// its own column block (half of B) into shared memory, 64 KB per k block,
// and the even CTA issues M = 256, N = 256 MMAs that read A and B from both
// CTAs' shared memory; each CTA's TMEM receives its 128 rows. Against the
// wide tiles (96 KB per CTA per k block for the same products per CTA) this
// moves a third fewer operand bytes per product from L2, and three 64 KB
// stages fit where two 96 KB stages did.
// Synchronisation between the two CTAs:
//  - each CTA's producer fills its own half of a stage with tensor-map
//    copies (cta_group::2 form, no multicast) whose completion is counted
//    on the even CTA's full barrier, which the even CTA's producer arms with
//    both halves' bytes; so the MMA issuer's one wait covers both halves;
//  - the MMA issuer's commits arrive on the empty, mfull and cfull barriers
//    at the same offset in both CTAs (multicast commit);
//  - the epilogue warps of both CTAs arrive on the even CTA's mempty and
//    cempty barriers (16 arrivals each) before the accumulators are reused.
// Everything else (drain interval, correction period, register split,
// epilogue) is that of the wide kernel.
// ===========================================================================
constexpr int kPStages = 3;
constexpr int kPStageBytes = 2 * kPairBytes;  // A pair + B pair (own half)

struct PairCtl
{
    uint64_t full[kPStages], empty[kPStages], mfull, mempty, cfull, cempty,
            done;
    uint32_t tmem_base;
    int abort;
};

constexpr size_t gemm_pair_smem_bytes()
{
    return 1024 + (size_t) kPStages * kPStageBytes + sizeof(PairCtl);
}

__host__ __device__ inline int pair_tiles(int nrb)
{
    const int np = (nrb + 1) / 2;
    return np * (np + 1) / 2;
}

// The operand image as a 2-D tensor for the copies: rows of 128 bytes (16
// 8-byte elements), row r at byte 128 r of the workspace's image area; a
// box is 256 rows, one hi + lo tile pair.
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kWThreads, 1)
gemm_pair_kernel(const GemmParams prm, const __grid_constant__ CUtensorMap tmap)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(
            (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t) 1023);
    PairCtl* ctl = reinterpret_cast<PairCtl*>(smem + kPStages * kPStageBytes);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = ptx::cluster_ctarank();
    volatile int* abort = &ctl->abort;

    if (threadIdx.x == 0)
    {
        for (int s = 0; s < kPStages; ++s)
        {
            ptx::mbar_init(&ctl->full[s], 1);
            ptx::mbar_init(&ctl->empty[s], 1);
        }
        ptx::mbar_init(&ctl->mfull, 1);
        ptx::mbar_init(&ctl->mempty, 2 * kWEpiWarps);
        ptx::mbar_init(&ctl->cfull, 1);
        ptx::mbar_init(&ctl->cempty, 2 * kWEpiWarps);
        ptx::mbar_init(&ctl->done, 1);
        ctl->abort = 0;
        ptx::fence_mbar_init();
    }
    if (warp == 1) ptx::tmem_alloc_pair(&ctl->tmem_base, kWTmemCols);
    ptx::tc_fence_before();
    // both CTAs' barriers initialised and TMEM allocated before any
    // cross-CTA arrive or MMA
    ptx::cluster_sync();
    ptx::tc_fence_after();
    const uint32_t tmem = ctl->tmem_base;

    const int np = (prm.nrb + 1) / 2;
    const int ntile = pair_tiles(prm.nrb);
    const int npairs = gridDim.x >> 1;
    const int pair = blockIdx.x >> 1;
    const int ntasks = ntile * prm.num_problems;
    const int nchunk = (prm.nkb + prm.drain_kb - 1) / prm.drain_kb;
    (void) np;

    if (warp < 4)
    {
    ptx::regs_release<kWLowRegs>();
    if (warp == 0)
    {
        if (lane == 0)
        {
            // ---------------- producer: this CTA's row block (A pair) and
            // column block (B pair) of every k block, counted on the even
            // CTA's full barrier
            const uint32_t full0 = ptx::mapa_shared(
                    ptx::smem_u32(&ctl->full[0]), 0);
            int stage = 0;
            uint32_t phase = 0;
            uint32_t issued = 0, issued_par = 0;
            for (int task = pair; task < ntasks && !*abort; task += npairs)
            {
                const int prob = task / ntile;
                int ti, tj;
                tile_of(task - prob * ntile, ti, tj);
                // a missing odd block (odd number of row blocks) repeats the
                // even one; its rows and columns are discarded (p, q >= N)
                int rb = 2 * ti + (int) rank, cb = 2 * tj + (int) rank;
                if (rb >= prm.nrb) rb = prm.nrb - 1;
                if (cb >= prm.nrb) cb = prm.nrb - 1;
                const long long row0 = (long long) prob * (long long)
                        (prm.image_stride / 128);
                for (int kb = 0; kb < prm.nkb; ++kb)
                {
                    if (!ptx::mbar_wait(&ctl->empty[stage], phase ^ 1,
                            prm.err, 31, abort))
                        break;
                    uint8_t* dst = smem + (size_t) stage * kPStageBytes;
                    if (rank == 0)
                        ptx::mbar_arrive_expect_tx(&ctl->full[stage],
                                2 * kPStageBytes);
                    const uint32_t bar = full0 +
                            (uint32_t) (stage * sizeof(uint64_t));
                    ptx::tma_load_2d_pair(dst, &tmap, 0, (int) (row0 +
                            ((long long) rb * prm.nkb + kb) * 256), bar);
                    ptx::tma_load_2d_pair(dst + kPairBytes, &tmap, 0,
                            (int) (row0 + ((long long) cb * prm.nkb + kb) *
                            256), bar);
                    issued |= 1u << stage;
                    issued_par = (issued_par & ~(1u << stage)) |
                            (phase << stage);
                    if (++stage == kPStages) { stage = 0; phase ^= 1; }
                }
            }
            // the even CTA's full barrier counts both CTAs' copies: its
            // producer waits for every stage's last phase before the CTAs
            // can leave
            if (rank == 0)
                for (int s = 0; s < kPStages; ++s)
                    if ((issued >> s) & 1)
                        ptx::mbar_wait(&ctl->full[s], (issued_par >> s) & 1,
                                prm.err, 32, abort);
        }
        __syncwarp();
    }
    else if (warp == 1)
    {
        if (lane == 0 && rank == 0)
        {
            // ---------------- MMA issuer (even CTA only)
            const uint32_t idesc = ptx::idesc_f16_f32(256, kWCols);
            const uint32_t dm = tmem, dcr = tmem + kWCols;
            int stage = 0;
            uint32_t phase = 0, mpar = 0, cpar = 0;
            bool ok = true;
            for (int task = pair; task < ntasks && ok; task += npairs)
            {
                for (int ch = 0; ch < nchunk && ok; ++ch)
                {
                    const bool fresh = (ch % kCorrPeriods) == 0;
                    if (fresh)
                    {
                        if (!ptx::mbar_wait_cluster(&ctl->cempty, cpar ^ 1,
                                prm.err, 33, abort))
                        {
                            ok = false;
                            break;
                        }
                        ptx::tc_fence_after();
                    }
                    const int kb0 = ch * prm.drain_kb;
                    const int kb1 = min(prm.nkb, kb0 + prm.drain_kb);
                    for (int kb = kb0; kb < kb1; ++kb)
                    {
                        if (!ptx::mbar_wait_cluster(&ctl->full[stage], phase,
                                prm.err, 34, abort))
                        {
                            ok = false;
                            break;
                        }
                        ptx::tc_fence_after();
                        const uint32_t a = ptx::smem_u32(smem +
                                (size_t) stage * kPStageBytes);
                        const uint32_t al = a + kTileBytes;
                        const uint32_t bh = a + kPairBytes;
                        const uint32_t bl = bh + kTileBytes;
                        // correction products first (hi lo^T + lo hi^T)
#pragma unroll
                        for (int k = 0; k < kKSteps; ++k)
                        {
                            const uint32_t first =
                                    (fresh && kb == kb0 && k == 0) ? 0u : 1u;
                            ptx::mma_f16_pair(dcr,
                                    ptx::sdesc_sw128(a + 32 * k),
                                    ptx::sdesc_sw128(bl + 32 * k), idesc,
                                    first);
                            ptx::mma_f16_pair(dcr,
                                    ptx::sdesc_sw128(al + 32 * k),
                                    ptx::sdesc_sw128(bh + 32 * k), idesc, 1u);
                        }
                        if (kb == kb0)
                        {
                            if (!ptx::mbar_wait_cluster(&ctl->mempty,
                                    mpar ^ 1, prm.err, 36, abort))
                            {
                                ok = false;
                                break;
                            }
                            ptx::tc_fence_after();
                        }
#pragma unroll
                        for (int k = 0; k < kKSteps; ++k)
                            ptx::mma_f16_pair(dm,
                                    ptx::sdesc_sw128(a + 32 * k),
                                    ptx::sdesc_sw128(bh + 32 * k), idesc,
                                    (kb > kb0 || k > 0) ? 1u : 0u);
                        ptx::mma_commit_pair(&ctl->empty[stage]);
                        if (++stage == kPStages) { stage = 0; phase ^= 1; }
                    }
                    if (!ok) break;
                    ptx::mma_commit_pair(&ctl->mfull);
                    mpar ^= 1;
                    if (corr_drain_at(ch, nchunk))
                    {
                        ptx::mma_commit_pair(&ctl->cfull);
                        cpar ^= 1;
                    }
                }
            }
            // every tcgen05 instruction of this kernel is cta_group::2
            ptx::mma_commit_pair(&ctl->done);
            ptx::mbar_wait(&ctl->done, 0, prm.err, 37, abort);
        }
        __syncwarp();
    }
    }  // warpgroup 0
    else
    {
        // ---------------- epilogue warps (4 and up), kWEpiCols columns each
        ptx::regs_request<kWHighRegs>();
        const int q4 = warp & 3;
        const int h = (warp - 4) >> 2;
        const int row = 32 * q4 + lane;
        const uint32_t taddr = tmem + ((uint32_t) (32 * q4) << 16) +
                (uint32_t) (kWEpiCols * h);
        const uint32_t mempty0 = ptx::mapa_shared(
                ptx::smem_u32(&ctl->mempty), 0);
        const uint32_t cempty0 = ptx::mapa_shared(
                ptx::smem_u32(&ctl->cempty), 0);
        uint32_t mpar = 0, cpar = 0;
        auto arrive = [&](bool with_corr) {
            ptx::mbar_arrive_cluster(mempty0);
            if (with_corr) ptx::mbar_arrive_cluster(cempty0);
        };
        for (int task = pair; task < ntasks; task += npairs)
        {
            const int prob = task / ntile;
            int ti, tj;
            tile_of(task - prob * ntile, ti, tj);
            // columns 0-127 of the accumulator are column block 2 tj,
            // 128-255 column block 2 tj + 1
            if (!wide_task_epilogue(prm, &ctl->mfull, &ctl->cfull, mpar,
                    cpar, abort, taddr, row, lane, prob,
                    2 * ti + (int) rank,
                    2 * tj * kStPerBlock + (kWEpiCols / 4) * h, nchunk,
                    arrive))
                break;
        }
    }

    ptx::tc_fence_before();
    // no CTA leaves (or frees TMEM) while its peer may still arrive on its
    // barriers or its MMAs read the other's shared memory
    ptx::cluster_sync();
    ptx::tc_fence_after();
    if (warp == 1) ptx::tmem_dealloc_pair(tmem, kWTmemCols);
}

// ===========================================================================
// Integer contraction (the default): G = W W^T from the three-limb 8-bit
// image on the tcgen05 integer path (signed 8-bit MMAs). With
// a = a0 2^16 + a1 2^8 + a2 and b likewise,
//     a b / 2^16 = a0 b0 2^16 + (a0 b1 + a1 b0) 2^8 + (a0 b2 + a1 b1 + a2 b0)
//                  + (a1 b2 + a2 b1) 2^-8 + a2 b2 2^-16,
// the last two classes left out: six 8-bit MMAs per 32-wide K step feed
// three S32 TMEM accumulators (D0 .. D2, 128 columns each) of 128 x 128
// tiles. The limbs are balanced digits (each in [-128, 127]), so the left-out
// terms have mean zero and add at most 2^-23 of the largest product at
// their k block's scale (|a1 b2 + a2 b1| 2^-8 <= 2^7 against 2^30). The
// image orders the sources by amplitude bucket, each bucket with its own
// scale q 2^b, so that bound follows every source's own size instead of
// the brightest source's (without the buckets, a sky of many faint sources
// would lose ~1e-6 of the visibilities' L2 norm to the uniform low digits
// of its faint entries).
// The integer sums are exact: no rounding happens in the tensor core, so
// the accumulators only need draining before they could overflow (at most
// kI8DrainKb k blocks per chunk: one k block adds at most 3 x 64 x 2^14 <
// 2^21.6 to |D2|, so 512 blocks stay below 2^31), at the end of each bucket
// (a chunk never spans two scales) and of a task, where
// (D0 2^16 + D1 2^8 + D2) 2^-2b is formed in FP64 and folded into the
// visibility sums.
// Warp roles (320 threads): warp 0 producer (one bulk copy per operand per
// k block into a kI8Stages-deep ring of 48 KB stages), warp 1 MMA issuer,
// warps 2-9 epilogue (64 columns each, as the square FP16 kernel).
// ===========================================================================
constexpr int kI8Stages = 4;
constexpr int kI8StageBytes = 2 * kI8Block;   // A block + B block
constexpr uint32_t kI8TmemCols = 512;         // D0, D1, D2 (+ 128 unused)

struct I8Ctl
{
    uint64_t full[kI8Stages], empty[kI8Stages], dfull, dempty, done;
    uint32_t tmem_base;
    int abort;
};

constexpr size_t gemm_i8_smem_bytes()
{
    return 1024 + (size_t) kI8Stages * kI8StageBytes + sizeof(I8Ctl);
}

// One drain of the three integer accumulators over this thread's 64
// columns (taddr): (D0 2^16 + D1 2^8 + D2) scale per column (exact before
// the scale, |.| < 2^48), folded into the Re V and Im V sums of its 16
// column stations.
__device__ __forceinline__ void i8_drain64(uint32_t taddr, int c,
        double scale, double (&accR)[16], double (&accI)[16])
{
#pragma unroll
    for (int j0 = 0; j0 < 64; j0 += 16)
    {
        uint32_t v0[16], v1[16], v2[16];
        ptx::tmem_ld16(taddr + j0, v0);
        ptx::tmem_ld16(taddr + 128 + j0, v1);
        ptx::tmem_ld16(taddr + 256 + j0, v2);
        ptx::tmem_ld_wait();
        double v[16];
#pragma unroll
        for (int j = 0; j < 16; ++j)
            v[j] = ((double) (int) v0[j] * 65536.0 +
                    (double) (int) v1[j] * 256.0 +
                    (double) (int) v2[j]) * scale;
        // Re V = G00 + G11, Im V = G10 - G01 across the row pair
        // (lanes l, l ^ 1), as the FP16 kernels fold
#pragma unroll
        for (int qq = 0; qq < 4; ++qq)
        {
            const int jb = 4 * qq;
            const double s0 = c ? v[jb + 0] : v[jb + 2];
            const double s1 = c ? v[jb + 1] : v[jb + 3];
            const double r0 = __shfl_xor_sync(0xffffffffu, s0, 1);
            const double r1 = __shfl_xor_sync(0xffffffffu, s1, 1);
            const double g00 = c ? r0 : v[jb + 0];
            const double g01 = c ? r1 : v[jb + 1];
            const double g10 = c ? v[jb + 2] : r0;
            const double g11 = c ? v[jb + 3] : r1;
            accR[j0 / 4 + qq] += g00 + g11;
            accI[j0 / 4 + qq] += g10 - g01;
        }
    }
}

__global__ void __launch_bounds__(kGemmThreads, 1)
gemm_i8_kernel(const GemmParams prm)
{
    // a brightness matrix that is not positive semi-definite: nothing is
    // added when the caller asked so (the FP32 entry point)
    if (prm.skip_flags && (*prm.skip_flags & 1)) return;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(
            (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t) 1023);
    I8Ctl* ctl = reinterpret_cast<I8Ctl*>(smem + kI8Stages * kI8StageBytes);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    volatile int* abort = &ctl->abort;

    if (threadIdx.x == 0)
    {
        for (int s = 0; s < kI8Stages; ++s)
        {
            ptx::mbar_init(&ctl->full[s], 1);
            ptx::mbar_init(&ctl->empty[s], 1);
        }
        ptx::mbar_init(&ctl->dfull, 1);
        ptx::mbar_init(&ctl->dempty, 8);
        ptx::mbar_init(&ctl->done, 1);
        ctl->abort = 0;
        ptx::fence_mbar_init();
    }
    if (warp == 1) ptx::tmem_alloc(&ctl->tmem_base, kI8TmemCols);
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    const uint32_t tmem = ctl->tmem_base;

    const int ntile = prm.nrb * (prm.nrb + 1) / 2;
    const int ntasks = ntile * prm.num_problems;
    const int nkb_used = prm.i8_counts[0];
    const int nchunk = prm.i8_counts[1];

    if (warp == 0)
    {
        if (lane == 0)
        {
            // ---------------- producer: A block, then B block (not on
            // diagonal tiles, whose B is A); the image's row blocks are
            // prm.nkb (its capacity) apart, nkb_used of them filled
            int stage = 0;
            uint32_t phase = 0;
            uint32_t issued = 0, issued_par = 0;  // bit s: stage s
            for (int task = blockIdx.x; task < ntasks && !*abort;
                    task += gridDim.x)
            {
                const int prob = task / ntile;
                int rb, cb;
                tile_of(task - prob * ntile, rb, cb);
                const bool diag = rb == cb;
                const uint8_t* img = prm.W + (size_t) prob * prm.image_stride;
                for (int kb = 0; kb < nkb_used; ++kb)
                {
                    if (!ptx::mbar_wait(&ctl->empty[stage], phase ^ 1,
                            prm.err, 31, abort))
                        break;
                    uint8_t* dst = smem + (size_t) stage * kI8StageBytes;
                    ptx::mbar_arrive_expect_tx(&ctl->full[stage],
                            diag ? kI8Block : 2 * kI8Block);
                    ptx::bulk_g2s(dst, img + ((size_t) rb * prm.nkb + kb) *
                            kI8Block, kI8Block, &ctl->full[stage]);
                    if (!diag)
                        ptx::bulk_g2s(dst + kI8Block, img +
                                ((size_t) cb * prm.nkb + kb) * kI8Block,
                                kI8Block, &ctl->full[stage]);
                    issued |= 1u << stage;
                    issued_par = (issued_par & ~(1u << stage)) |
                            (phase << stage);
                    if (++stage == kI8Stages) { stage = 0; phase ^= 1; }
                }
            }
            for (int s = 0; s < kI8Stages; ++s)
                if ((issued >> s) & 1)
                    ptx::mbar_wait(&ctl->full[s], (issued_par >> s) & 1,
                            prm.err, 32, abort);
        }
        __syncwarp();
    }
    else if (warp == 1)
    {
        if (lane == 0)
        {
            // ---------------- MMA issuer
            const uint32_t idesc = ptx::idesc_i8_s32(128, 128, true, true);
            const uint32_t d0 = tmem, d1 = tmem + 128, d2 = tmem + 256;
            int stage = 0;
            uint32_t phase = 0, dpar = 0;
            bool ok = true;
            for (int task = blockIdx.x; task < ntasks && ok;
                    task += gridDim.x)
            {
                const int prob = task / ntile;
                int rb, cb;
                tile_of(task - prob * ntile, rb, cb);
                const bool diag = rb == cb;
                for (int ch = 0; ch < nchunk && ok; ++ch)
                {
                    // the epilogue has read the accumulators' last sums
                    if (!ptx::mbar_wait(&ctl->dempty, dpar ^ 1, prm.err, 33,
                            abort))
                    {
                        ok = false;
                        break;
                    }
                    ptx::tc_fence_after();
                    const int kb0 = prm.i8_chunk_kb[ch];
                    const int kb1 = prm.i8_chunk_kb[ch + 1];
                    for (int kb = kb0; kb < kb1; ++kb)
                    {
                        if (!ptx::mbar_wait(&ctl->full[stage], phase, prm.err,
                                34, abort))
                        {
                            ok = false;
                            break;
                        }
                        ptx::tc_fence_after();
                        const uint32_t a = ptx::smem_u32(smem +
                                (size_t) stage * kI8StageBytes);
                        const uint32_t b = diag ? a : a + kI8Block;
#pragma unroll
                        for (int k = 0; k < 2; ++k)
                        {
                            const uint64_t a0 = ptx::sdesc_sw64(a + 32 * k);
                            const uint64_t a1 = ptx::sdesc_sw64(
                                    a + kI8Tile + 32 * k);
                            const uint64_t a2 = ptx::sdesc_sw64(
                                    a + 2 * kI8Tile + 32 * k);
                            const uint64_t b0 = ptx::sdesc_sw64(b + 32 * k);
                            const uint64_t b1 = ptx::sdesc_sw64(
                                    b + kI8Tile + 32 * k);
                            const uint64_t b2 = ptx::sdesc_sw64(
                                    b + 2 * kI8Tile + 32 * k);
                            const uint32_t acc =
                                    (kb > kb0 || k > 0) ? 1u : 0u;
                            // grouped by A limb, A kept in the collector
                            // buffer across its group; the first MMA into
                            // each accumulator (program order) resets it
                            ptx::mma_i8_col<0>(d0, a0, b0, idesc, acc);
                            ptx::mma_i8_col<1>(d1, a0, b1, idesc, acc);
                            ptx::mma_i8_col<2>(d2, a0, b2, idesc, acc);
                            ptx::mma_i8_col<0>(d1, a1, b0, idesc, 1u);
                            ptx::mma_i8_col<2>(d2, a1, b1, idesc, 1u);
                            ptx::mma_i8(d2, a2, b0, idesc, 1u);
                        }
                        ptx::mma_commit(&ctl->empty[stage]);
                        if (++stage == kI8Stages) { stage = 0; phase ^= 1; }
                    }
                    if (!ok) break;
                    ptx::mma_commit(&ctl->dfull);
                    dpar ^= 1;
                }
            }
            // All issued MMAs must finish before TMEM is released.
            ptx::mma_commit(&ctl->done);
            ptx::mbar_wait(&ctl->done, 0, prm.err, 35, abort);
        }
        __syncwarp();
    }
    else
    {
        // ---------------- epilogue: 8 warps, 64 columns each
        const int q4 = warp & 3;          // TMEM lane quadrant of this warp
        const int h = (warp - 2) >> 2;    // column half
        const int row = 32 * q4 + lane;   // row of the G tile
        const int c = row & 1;
        const uint32_t taddr = tmem + ((uint32_t) (32 * q4) << 16) +
                (uint32_t) (64 * h);
        uint32_t dpar = 0;
        bool ok = true;
        for (int task = blockIdx.x; task < ntasks && ok; task += gridDim.x)
        {
            const int prob = task / ntile;
            int rb, cb;
            tile_of(task - prob * ntile, rb, cb);
            // sums of Re V and Im V, in units of 2^16 / q^2, of the
            // thread's 16 column stations
            double accR[16], accI[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) accR[j] = accI[j] = 0.0;
            for (int ch = 0; ch < nchunk; ++ch)
            {
                if (!ptx::mbar_wait(&ctl->dfull, dpar, prm.err, 36, abort))
                {
                    ok = false;
                    break;
                }
                ptx::tc_fence_after();
                // the chunk's bucket b: its entries carry q 2^b each
                i8_drain64(taddr, c, ldexp(1.0, -2 * prm.i8_chunk_bucket[ch]),
                        accR, accI);
                ptx::tc_fence_before();
                __syncwarp();
                if (lane == 0) ptx::mbar_arrive(&ctl->dempty);
                dpar ^= 1;
            }
            if (!ok) break;
            const int g = prm.prob0 + prob;
            const double q = (double) i8_scale_from_bits(
                    prm.maxabs_bits[prm.maxabs_stride * g]);
            square_task_store(prm, accR, accI, 65536.0 / (q * q), row, h,
                    prob, rb, cb);
        }
    }

    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    if (warp == 1) ptx::tmem_dealloc(tmem, kI8TmemCols);
}

// ===========================================================================
// FP64-class integer contraction (oskb_cross_correlate_tc64_d): the entries
// of A = J C (FP64) as 48-bit fixed point, a = round(x q 2^b) with
// q = 127 2^40 / max|A| and b the source's amplitude bucket, held as six
// balanced 8-bit limbs a = sum_k a_k 2^(8 (5 - k)) (a_0 signed, a_1 .. a_5
// in [-128, 127]). With b likewise,
//     a b / 2^40 = sum_{i + j = c} a_i b_j 2^(8 (5 - c)),  c = 0 .. 10,
// of which the classes c <= 5 (21 products) are kept: the rest add at most
// ~2^-41 of the largest product at the block's scale. Tiles are 128 rows
// x 64 columns (half of a column block) so that the six S32 accumulators
// D0 .. D5 fit TMEM (64 columns each); 21 MMAs (M = 128, N = 64, K = 32)
// per K step, A held in the collector buffer across its limb's products.
// The accumulators are drained every kL6DrainKb k blocks (a k block adds at
// most 6 x 64 x 2^14 < 2^22.6 to |D5|), at each bucket's end and at the
// task's end: sum_c D_c 2^(8 (5 - c)) in FP64 (Horner), times 2^-2b.
// Warp roles as gemm_i8_kernel; the epilogue warps take 32 columns each.
// ===========================================================================
constexpr int kL6Limbs = 6;
constexpr int kL6Block = kL6Limbs * kI8Tile;        // 48 KB per k block
constexpr int kL6HalfB = kL6Limbs * (kI8Tile / 2);  // 24 KB: 64 rows each
constexpr int kL6StageBytes = kL6Block + kL6HalfB;  // 72 KB
constexpr int kL6Stages = 3;
constexpr int kL6DrainKb = 256;
constexpr uint32_t kL6TmemCols = 512;               // D0 .. D5, 64 each
constexpr double kL6Target = 127.0 * 1099511627776.0;   // 127 x 2^40

__host__ __device__ inline size_t image_bytes_l6(int num_st, int num_src)
{
    const size_t nrb = (num_st + kStPerBlock - 1) / kStPerBlock;
    return nrb * (size_t) i8_kb_cap(num_src) * kL6Block;
}

__device__ __forceinline__ double l6_scale_from_bits(unsigned int bits)
{
    const float m = __uint_as_float(bits);
    if (!(m > 0.0f) || !isfinite(m)) return 1.0;
    return kL6Target / (double) m;
}

// A = J C in FP64 (J row-major {a, b, c, d} complex, C lower triangular).
__device__ __forceinline__ void apply_factor_d(const double* J, double c11,
        double c21r, double c21i, double c22, double out[2][2][2])
{
#pragma unroll
    for (int i = 0; i < 2; ++i)
    {
        const double j0r = J[4 * i + 0], j0i = J[4 * i + 1];
        const double j1r = J[4 * i + 2], j1i = J[4 * i + 3];
        out[i][0][0] = j0r * c11 + (j1r * c21r - j1i * c21i);
        out[i][0][1] = j0i * c11 + (j1r * c21i + j1i * c21r);
        out[i][1][0] = j1r * c22;
        out[i][1][1] = j1i * c22;
    }
}

// Writes one station-source's scaled 2x2 A as 4 rows of the six limb tiles
// of its block: t = a + 0x8080808080, limb k = byte 5 - k of t (the low
// limbs with their top bit flipped: balanced digits).
__device__ __forceinline__ void store_entry_l6(uint8_t* block, int pl,
        int sl, const double A[2][2][2])
{
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int c = 0; c < 2; ++c)
        {
            const int r = 4 * pl + 2 * i + c;
            const long long t0 = __double2ll_rn(A[i][0][c]) +
                    0x8080808080LL;
            const long long t1 = __double2ll_rn(A[i][1][c]) +
                    0x8080808080LL;
            const uint32_t lo0 = (uint32_t) t0, hi0 = (uint32_t) (t0 >> 32);
            const uint32_t lo1 = (uint32_t) t1, hi1 = (uint32_t) (t1 >> 32);
            const uint32_t off = swz64_offset(r, 2 * sl);
#pragma unroll
            for (int limb = 0; limb < kL6Limbs; ++limb)
            {
                const int byte = 5 - limb;
                const uint32_t v = byte >= 4 ?
                        __byte_perm(hi0, hi1, (byte - 4) | ((byte) << 4)) :
                        __byte_perm(lo0, lo1, byte | ((byte + 4) << 4));
                *reinterpret_cast<uint16_t*>(block + limb * kI8Tile + off) =
                        (uint16_t) (v ^ (limb ? 0x8080u : 0u));
            }
        }
}

// Six-limb image from joined Jones J (FP64): the sources in bucket order
// (o.perm), each k block scaled by q 2^b of its bucket. grid (k-block
// capacity, row blocks); blocks past the used k blocks return.
__global__ void __launch_bounds__(256) prep_jones_l6_kernel(
        const double* __restrict__ jones, int num_src, int num_st,
        const double* __restrict__ I, const double* __restrict__ Q,
        const double* __restrict__ U, const double* __restrict__ V,
        const unsigned int* __restrict__ maxabs_bits, const I8Order o,
        uint8_t* W)
{
    const int kb = blockIdx.x, rb = blockIdx.y, nkb_cap = gridDim.x;
    if (kb >= o.counts[0]) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int s = o.perm[kb * kSrcPerBlock + lane];
    const bool src_ok = s >= 0;
    double c11 = 0, c21r = 0, c21i = 0, c22 = 0;
    if (src_ok) brightness_factor(I[s], Q[s], U[s], V[s], c11, c21r, c21i, c22);
    const double q = ldexp(l6_scale_from_bits(*maxabs_bits), o.kb_bucket[kb]);
    uint8_t* blk = W + (size_t) (rb * nkb_cap + kb) * kL6Block;
    for (int pl = warp; pl < kStPerBlock; pl += 8)
    {
        const int p = rb * kStPerBlock + pl;
        double A[2][2][2] = {{{0, 0}, {0, 0}}, {{0, 0}, {0, 0}}};
        if (src_ok && p < num_st)
        {
            const double2* jp = reinterpret_cast<const double2*>(
                    jones + 8 * ((size_t) p * num_src + s));
            double J[8];
#pragma unroll
            for (int k = 0; k < 4; ++k)
            {
                const double2 v = __ldg(jp + k);
                J[2 * k] = v.x;
                J[2 * k + 1] = v.y;
            }
            apply_factor_d(J, c11, c21r, c21i, c22, A);
#pragma unroll
            for (int k = 0; k < 8; ++k) (&A[0][0][0])[k] *= q;
        }
        store_entry_l6(blk, pl, lane, A);
    }
}

// Six-limb image of a block of problems (t, c) from E (FP32 or FP64
// [station][source][2x2], shared by the block) with the interferometer
// phase in FP64: entry = K_p(s) (E_p C)(s) scaled by q 2^b of the source's
// bucket, K_p(s) = exp(2 pi i (u_p l + v_p m + w_p (n - 1)) / lambda_c),
// the argument reduced mod 1 in FP64 and its sine and cosine by sincospi
// (FP64). grid (k-block capacity, row blocks); a thread takes one source
// and stations warp + 8 k, and for each station every problem of the
// group [p0, p0 + np) (problem j's image at W + j image_stride).
template <typename TE>
__global__ void __launch_bounds__(256) prep_fused_l6_kernel(
        const TE* __restrict__ E, int num_src, int num_st,
        const double* __restrict__ l, const double* __restrict__ m,
        const double* __restrict__ n, const double* __restrict__ I,
        const double* __restrict__ Q, const double* __restrict__ U,
        const double* __restrict__ V, const double* __restrict__ uvw,
        const double* __restrict__ inv_wavelength, int nch, int p0, int np,
        const unsigned int* __restrict__ maxabs_bits, const I8Order o,
        uint8_t* W, size_t image_stride)
{
    const int kb = blockIdx.x, rb = blockIdx.y, nkb_cap = gridDim.x;
    if (kb >= o.counts[0]) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int s = o.perm[kb * kSrcPerBlock + lane];
    const bool src_ok = s >= 0;
    double c11 = 0, c21r = 0, c21i = 0, c22 = 0;
    double sl = 0, sm = 0, sn1 = 0;
    if (src_ok)
    {
        brightness_factor(I[s], Q[s], U[s], V[s], c11, c21r, c21i, c22);
        sl = l[s]; sm = m[s]; sn1 = n[s] - 1.0;
    }
    const double q = ldexp(l6_scale_from_bits(*maxabs_bits), o.kb_bucket[kb]);
    uint8_t* blk0 = W + (size_t) (rb * nkb_cap + kb) * kL6Block;
    for (int pl = warp; pl < kStPerBlock; pl += 8)
    {
        const int p = rb * kStPerBlock + pl;
        const bool ok = src_ok && p < num_st;
        double A0[2][2][2] = {{{0, 0}, {0, 0}}, {{0, 0}, {0, 0}}};
        if (ok)
        {
            double J[8];
            const TE* e = E + 8 * ((size_t) p * num_src + s);
#pragma unroll
            for (int k = 0; k < 8; ++k) J[k] = (double) e[k];
            apply_factor_d(J, c11, c21r, c21i, c22, A0);
#pragma unroll
            for (int k = 0; k < 8; ++k) (&A0[0][0][0])[k] *= q;
        }
        double base = 0.0;
        int t_cur = -1;
        for (int j = 0; j < np; ++j)
        {
            const int prob = p0 + j, t = prob / nch, c = prob - t * nch;
            double A[2][2][2] = {{{0, 0}, {0, 0}}, {{0, 0}, {0, 0}}};
            if (ok)
            {
                if (t != t_cur)
                {
                    t_cur = t;
                    const double* pu = uvw + (size_t) t * 3 * num_st;
                    base = pu[p] * sl + pu[num_st + p] * sm +
                            pu[2 * num_st + p] * sn1;
                }
                const double x = base * inv_wavelength[c];
                double sn, cs;
                sincospi(2.0 * (x - rint(x)), &sn, &cs);
#pragma unroll
                for (int i = 0; i < 2; ++i)
#pragma unroll
                    for (int kk = 0; kk < 2; ++kk)
                    {
                        const double re = A0[i][kk][0], im = A0[i][kk][1];
                        A[i][kk][0] = re * cs - im * sn;
                        A[i][kk][1] = re * sn + im * cs;
                    }
            }
            store_entry_l6(blk0 + (size_t) j * image_stride, pl, lane, A);
        }
    }
}

struct L6Ctl
{
    uint64_t full[kL6Stages], empty[kL6Stages], dfull, dempty, done;
    uint32_t tmem_base;
    int abort;
};

constexpr size_t gemm_l6_smem_bytes()
{
    return 1024 + (size_t) kL6Stages * kL6StageBytes + sizeof(L6Ctl);
}

// One drain of the six accumulators over this thread's 32 columns (taddr,
// 64 columns per accumulator): sum_c D_c 2^(8 (5 - c)) scale per column,
// folded into the Re V and Im V sums of its 8 column stations.
__device__ __forceinline__ void l6_drain32(uint32_t taddr, int c,
        double scale, double (&accR)[8], double (&accI)[8])
{
#pragma unroll
    for (int j0 = 0; j0 < 32; j0 += 16)
    {
        double v[16];
        {
            uint32_t u0[16], u1[16], u2[16];
            ptx::tmem_ld16(taddr + j0, u0);
            ptx::tmem_ld16(taddr + 64 + j0, u1);
            ptx::tmem_ld16(taddr + 128 + j0, u2);
            ptx::tmem_ld_wait();
#pragma unroll
            for (int j = 0; j < 16; ++j)
                v[j] = ((double) (int) u0[j] * 256.0 + (double) (int) u1[j])
                        * 256.0 + (double) (int) u2[j];
        }
        {
            uint32_t u3[16], u4[16], u5[16];
            ptx::tmem_ld16(taddr + 192 + j0, u3);
            ptx::tmem_ld16(taddr + 256 + j0, u4);
            ptx::tmem_ld16(taddr + 320 + j0, u5);
            ptx::tmem_ld_wait();
#pragma unroll
            for (int j = 0; j < 16; ++j)
                v[j] = (((v[j] * 256.0 + (double) (int) u3[j]) * 256.0 +
                        (double) (int) u4[j]) * 256.0 +
                        (double) (int) u5[j]) * scale;
        }
        // Re V = G00 + G11, Im V = G10 - G01 across the row pair
        // (lanes l, l ^ 1), as i8_drain64
#pragma unroll
        for (int qq = 0; qq < 4; ++qq)
        {
            const int jb = 4 * qq;
            const double s0 = c ? v[jb + 0] : v[jb + 2];
            const double s1 = c ? v[jb + 1] : v[jb + 3];
            const double r0 = __shfl_xor_sync(0xffffffffu, s0, 1);
            const double r1 = __shfl_xor_sync(0xffffffffu, s1, 1);
            const double g00 = c ? r0 : v[jb + 0];
            const double g01 = c ? r1 : v[jb + 1];
            const double g10 = c ? v[jb + 2] : r0;
            const double g11 = c ? v[jb + 3] : r1;
            accR[j0 / 4 + qq] += g00 + g11;
            accI[j0 / 4 + qq] += g10 - g01;
        }
    }
}

// Tasks: (problem, square tile (rb <= cb), column half); 2 per tile.
__global__ void __launch_bounds__(kGemmThreads, 1)
gemm_l6_kernel(const GemmParams prm)
{
    // a brightness matrix that is not positive semi-definite: nothing is
    // added (the caller correlates those sources another way)
    if (prm.skip_flags && (*prm.skip_flags & 1)) return;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(
            (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t) 1023);
    L6Ctl* ctl = reinterpret_cast<L6Ctl*>(smem + kL6Stages * kL6StageBytes);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    volatile int* abort = &ctl->abort;

    if (threadIdx.x == 0)
    {
        for (int s = 0; s < kL6Stages; ++s)
        {
            ptx::mbar_init(&ctl->full[s], 1);
            ptx::mbar_init(&ctl->empty[s], 1);
        }
        ptx::mbar_init(&ctl->dfull, 1);
        ptx::mbar_init(&ctl->dempty, 8);
        ptx::mbar_init(&ctl->done, 1);
        ctl->abort = 0;
        ptx::fence_mbar_init();
    }
    if (warp == 1) ptx::tmem_alloc(&ctl->tmem_base, kL6TmemCols);
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    const uint32_t tmem = ctl->tmem_base;

    const int ntile = prm.nrb * (prm.nrb + 1);     // two halves per tile
    const int ntasks = ntile * prm.num_problems;
    const int nkb_used = prm.i8_counts[0];
    const int nchunk = prm.i8_counts[1];

    if (warp == 0)
    {
        if (lane == 0)
        {
            // ---------------- producer: the row block's six limb tiles
            // (one copy), then rows 64 h .. 64 h + 63 of the column
            // block's (six copies; none on diagonal tiles, whose B rows
            // are in A)
            int stage = 0;
            uint32_t phase = 0;
            uint32_t issued = 0, issued_par = 0;  // bit s: stage s
            for (int task = blockIdx.x; task < ntasks && !*abort;
                    task += gridDim.x)
            {
                const int prob = task / ntile;
                const int tt = task - prob * ntile;
                const int half = tt & 1;
                int rb, cb;
                tile_of(tt >> 1, rb, cb);
                const bool diag = rb == cb;
                const uint8_t* img = prm.W + (size_t) prob * prm.image_stride;
                for (int kb = 0; kb < nkb_used; ++kb)
                {
                    if (!ptx::mbar_wait(&ctl->empty[stage], phase ^ 1,
                            prm.err, 51, abort))
                        break;
                    uint8_t* dst = smem + (size_t) stage * kL6StageBytes;
                    ptx::mbar_arrive_expect_tx(&ctl->full[stage],
                            diag ? kL6Block : kL6StageBytes);
                    ptx::bulk_g2s(dst, img + ((size_t) rb * prm.nkb + kb) *
                            kL6Block, kL6Block, &ctl->full[stage]);
                    if (!diag)
                    {
                        const uint8_t* srcb = img + ((size_t) cb * prm.nkb +
                                kb) * kL6Block + half * (kI8Tile / 2);
#pragma unroll
                        for (int l = 0; l < kL6Limbs; ++l)
                            ptx::bulk_g2s(dst + kL6Block + l * (kI8Tile / 2),
                                    srcb + l * kI8Tile, kI8Tile / 2,
                                    &ctl->full[stage]);
                    }
                    issued |= 1u << stage;
                    issued_par = (issued_par & ~(1u << stage)) |
                            (phase << stage);
                    if (++stage == kL6Stages) { stage = 0; phase ^= 1; }
                }
            }
            for (int s = 0; s < kL6Stages; ++s)
                if ((issued >> s) & 1)
                    ptx::mbar_wait(&ctl->full[s], (issued_par >> s) & 1,
                            prm.err, 52, abort);
        }
        __syncwarp();
    }
    else if (warp == 1)
    {
        if (lane == 0)
        {
            // ---------------- MMA issuer
            const uint32_t idesc = ptx::idesc_i8_s32(128, 64, true, true);
            uint32_t d[kL6Limbs];
#pragma unroll
            for (int c = 0; c < kL6Limbs; ++c) d[c] = tmem + 64 * c;
            int stage = 0;
            uint32_t phase = 0, dpar = 0;
            bool ok = true;
            for (int task = blockIdx.x; task < ntasks && ok;
                    task += gridDim.x)
            {
                const int prob = task / ntile;
                const int tt = task - prob * ntile;
                const int half = tt & 1;
                int rb, cb;
                tile_of(tt >> 1, rb, cb);
                const bool diag = rb == cb;
                for (int ch = 0; ch < nchunk && ok; ++ch)
                {
                    // the epilogue has read the accumulators' last sums
                    if (!ptx::mbar_wait(&ctl->dempty, dpar ^ 1, prm.err, 53,
                            abort))
                    {
                        ok = false;
                        break;
                    }
                    ptx::tc_fence_after();
                    const int kb0 = prm.i8_chunk_kb[ch];
                    const int kb1 = prm.i8_chunk_kb[ch + 1];
                    for (int kb = kb0; kb < kb1; ++kb)
                    {
                        if (!ptx::mbar_wait(&ctl->full[stage], phase, prm.err,
                                54, abort))
                        {
                            ok = false;
                            break;
                        }
                        ptx::tc_fence_after();
                        const uint32_t a = ptx::smem_u32(smem +
                                (size_t) stage * kL6StageBytes);
                        // B limb l: rows 64 half .. of A's limb tile l on a
                        // diagonal tile, else the staged half
                        const uint32_t b = diag ? a + half * (kI8Tile / 2)
                                                : a + kL6Block;
                        const uint32_t bstep = diag ? kI8Tile : kI8Tile / 2;
#pragma unroll
                        for (int k = 0; k < 2; ++k)
                        {
                            uint64_t ad[kL6Limbs], bd[kL6Limbs];
#pragma unroll
                            for (int l = 0; l < kL6Limbs; ++l)
                            {
                                ad[l] = ptx::sdesc_sw64(a + l * kI8Tile +
                                        32 * k);
                                bd[l] = ptx::sdesc_sw64(b + l * bstep +
                                        32 * k);
                            }
                            const uint32_t acc =
                                    (kb > kb0 || k > 0) ? 1u : 0u;
                            // grouped by A limb i (collector buffer), the
                            // products a_i b_j into D_(i+j), i + j <= 5;
                            // the i = 0 group writes every accumulator
                            // first (program order), so it resets them
                            ptx::mma_i8_col<0>(d[0], ad[0], bd[0], idesc, acc);
                            ptx::mma_i8_col<1>(d[1], ad[0], bd[1], idesc, acc);
                            ptx::mma_i8_col<1>(d[2], ad[0], bd[2], idesc, acc);
                            ptx::mma_i8_col<1>(d[3], ad[0], bd[3], idesc, acc);
                            ptx::mma_i8_col<1>(d[4], ad[0], bd[4], idesc, acc);
                            ptx::mma_i8_col<2>(d[5], ad[0], bd[5], idesc, acc);
                            ptx::mma_i8_col<0>(d[1], ad[1], bd[0], idesc, 1u);
                            ptx::mma_i8_col<1>(d[2], ad[1], bd[1], idesc, 1u);
                            ptx::mma_i8_col<1>(d[3], ad[1], bd[2], idesc, 1u);
                            ptx::mma_i8_col<1>(d[4], ad[1], bd[3], idesc, 1u);
                            ptx::mma_i8_col<2>(d[5], ad[1], bd[4], idesc, 1u);
                            ptx::mma_i8_col<0>(d[2], ad[2], bd[0], idesc, 1u);
                            ptx::mma_i8_col<1>(d[3], ad[2], bd[1], idesc, 1u);
                            ptx::mma_i8_col<1>(d[4], ad[2], bd[2], idesc, 1u);
                            ptx::mma_i8_col<2>(d[5], ad[2], bd[3], idesc, 1u);
                            ptx::mma_i8_col<0>(d[3], ad[3], bd[0], idesc, 1u);
                            ptx::mma_i8_col<1>(d[4], ad[3], bd[1], idesc, 1u);
                            ptx::mma_i8_col<2>(d[5], ad[3], bd[2], idesc, 1u);
                            ptx::mma_i8_col<0>(d[4], ad[4], bd[0], idesc, 1u);
                            ptx::mma_i8_col<2>(d[5], ad[4], bd[1], idesc, 1u);
                            ptx::mma_i8(d[5], ad[5], bd[0], idesc, 1u);
                        }
                        ptx::mma_commit(&ctl->empty[stage]);
                        if (++stage == kL6Stages) { stage = 0; phase ^= 1; }
                    }
                    if (!ok) break;
                    ptx::mma_commit(&ctl->dfull);
                    dpar ^= 1;
                }
            }
            // All issued MMAs must finish before TMEM is released.
            ptx::mma_commit(&ctl->done);
            ptx::mbar_wait(&ctl->done, 0, prm.err, 55, abort);
        }
        __syncwarp();
    }
    else
    {
        // ---------------- epilogue: 8 warps, 32 columns each
        const int q4 = warp & 3;          // TMEM lane quadrant of this warp
        const int h = (warp - 2) >> 2;    // 32-column half of the 64
        const int row = 32 * q4 + lane;   // row of the G tile
        const int c = row & 1;
        const uint32_t taddr = tmem + ((uint32_t) (32 * q4) << 16) +
                (uint32_t) (32 * h);
        uint32_t dpar = 0;
        bool ok = true;
        for (int task = blockIdx.x; task < ntasks && ok; task += gridDim.x)
        {
            const int prob = task / ntile;
            const int tt = task - prob * ntile;
            const int half = tt & 1;
            int rb, cb;
            tile_of(tt >> 1, rb, cb);
            double accR[8], accI[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) accR[j] = accI[j] = 0.0;
            for (int ch = 0; ch < nchunk; ++ch)
            {
                if (!ptx::mbar_wait(&ctl->dfull, dpar, prm.err, 56, abort))
                {
                    ok = false;
                    break;
                }
                ptx::tc_fence_after();
                // the chunk's bucket b: its entries carry q 2^b each
                l6_drain32(taddr, c, ldexp(1.0, -2 * prm.i8_chunk_bucket[ch]),
                        accR, accI);
                ptx::tc_fence_before();
                __syncwarp();
                if (lane == 0) ptx::mbar_arrive(&ctl->dempty);
                dpar ^= 1;
            }
            if (!ok) break;
            const int g = prm.prob0 + prob;
            const double q = l6_scale_from_bits(
                    prm.maxabs_bits[prm.maxabs_stride * g]);
            task_store<8>(prm, accR, accI, 1099511627776.0 / (q * q), row,
                    16 * half + 8 * h, prob, rb, cb);
        }
    }

    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    if (warp == 1) ptx::tmem_dealloc(tmem, kL6TmemCols);
}

// FP32 entry point helpers: station u, v widened to FP64; the FP64 sums
// added into the FP32 visibilities (8 reals per baseline).
__global__ void __launch_bounds__(256) widen_uv_kernel(int n,
        const float* __restrict__ u, const float* __restrict__ v,
        double* __restrict__ du, double* __restrict__ dv)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
    {
        du[i] = (double) u[i];
        dv[i] = (double) v[i];
    }
}

__global__ void __launch_bounds__(256) add_vis_f_kernel(size_t n,
        const double* __restrict__ sums, float* __restrict__ vis)
{
    for (size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
            i += (size_t) gridDim.x * blockDim.x)
        vis[i] = (float) ((double) vis[i] + sums[i]);
}

}  // namespace tc
}  // namespace oskb

// ===========================================================================
// Host side
// ===========================================================================
namespace oskb {
namespace tc {
namespace {

constexpr size_t kHeaderBytes = 256;  // maxabs bits, flags, error word

struct Header
{
    unsigned int maxabs_bits;
    int flags;   // bit 0: a brightness matrix was not positive semi-definite
    int err;     // non-zero: a bounded wait expired (code of the wait)
};

int num_sms() { return device_sm_count(); }

int drain_kblocks()
{
    static int d = 0;
    if (!d)
    {
        // every 2 k blocks (8 main-product MMA steps) by default. The FP32
        // accumulator's error grows with the interval (at 512 stations x
        // 100,000 sources, against the FP64 kernel: L2 / max relative
        // 2.55e-7 / 3.36e-7 at 2, 3.46e-7 / 5.07e-7 at 3, 4.56e-7 / 7.02e-7
        // at 4) while the drain's cost falls (46.1, 43.0, 40.9 ms per
        // launch); at 3 a 31-station x 100-source case already reached
        // 1.007e-6 max relative, past the 1e-6 bound, so 2 stays
        const char* e = getenv("OSKB_TC_DRAIN_KB");
        d = e ? atoi(e) : 2;
        if (d < 1) d = 1;
    }
    return d;
}

// Problems per group when the library keeps the workspace (each problem's
// operand image is 32 bytes per station-source).
int max_group()
{
    static int g = 0;
    if (!g)
    {
        const char* e = getenv("OSKB_TC_MAX_GROUP");
        g = e ? atoi(e) : 16;
        if (g < 1) g = 1;
    }
    return g;
}

// Library-kept workspaces, one per (device, stream), grown on demand. A
// workspace is only ever used by work on its own stream, so growing it
// (which first waits for that stream) cannot pull memory from under work
// queued on another stream or by another host thread.
struct CachedWorkspace
{
    int dev;
    cudaStream_t stream;
    void* ptr;
    size_t bytes;
};
std::mutex g_ws_mutex;
std::vector<CachedWorkspace> g_ws;
void* g_ws_last[64] = {};   // last library-kept workspace used per device

int get_workspace(void*& ws, size_t& ws_bytes, size_t need,
        cudaStream_t stream)
{
    if (ws)
        return ws_bytes >= need ? 0 : OSKB_ERR_MEMORY_ALLOC_FAILURE;
    const int dev = current_device();
    if (dev < 0 || dev >= 64) return OSKB_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(g_ws_mutex);
    CachedWorkspace* c = nullptr;
    for (auto& w : g_ws)
        if (w.dev == dev && w.stream == stream) c = &w;
    if (!c)
    {
        g_ws.push_back(CachedWorkspace{dev, stream, nullptr, 0});
        c = &g_ws.back();
    }
    if (c->bytes < need)
    {
        if (c->ptr)
        {
            cudaStreamSynchronize(stream);
            cudaFree(c->ptr);
        }
        c->ptr = nullptr;
        c->bytes = 0;
        if (cudaMalloc(&c->ptr, need) != cudaSuccess)
        {
            c->ptr = nullptr;
            set_last_error("tc workspace", cudaGetLastError());
            return OSKB_ERR_MEMORY_ALLOC_FAILURE;
        }
        c->bytes = need;
    }
    ws = c->ptr;
    ws_bytes = c->bytes;
    g_ws_last[dev] = c->ptr;
    return 0;
}

// Optional CUDA-event timing of every GEMM launch (for roofline reports),
// guarded by a lock so that launches from several host threads are all
// recorded.
std::mutex g_timing_mutex;
bool g_timing = false;
std::vector<std::pair<cudaEvent_t, cudaEvent_t>> g_ev;
size_t g_ev_used = 0;

// Tile shape of the contraction: OSKB_TC_TILE=128 (square 128 x 128
// tiles), 256 (wide 128 x 256 tiles) or 512 (256 x 256 pair tiles on two
// CTAs); unset: wide tiles when a launch has at least two per SM, else
// square tiles (with fewer tasks, the smaller tiles keep more SMs busy).
int tile_setting()
{
    const char* e = getenv("OSKB_TC_TILE");
    const int t = e ? atoi(e) : 0;
    return (t == 128 || t == 256 || t == 512) ? t : 0;
}

std::atomic<int> g_last_tile{0};
std::atomic<int> g_last_arith{0};

// Arithmetic of the contraction: the three-limb 8-bit integer form unless
// OSKB_TC_ARITH=fp16 or an FP16 tile shape is fixed by OSKB_TC_TILE.
bool arith_i8()
{
    const char* e = getenv("OSKB_TC_ARITH");
    if (e && strcmp(e, "fp16") == 0) return false;
    return tile_setting() == 0;
}

size_t image_bytes_for(bool i8, int num_st, int num_src)
{
    return i8 ? image_bytes_i8(num_st, num_src)
              : image_bytes(num_st, num_src);
}

// Per-device launch set-up: the dynamic shared-memory opt-in of both
// contraction kernels (a per-device attribute) and whether the wide
// kernel's register split fits the registers its blocks are launched with
// (kWLowRegs / kWHighRegs against the compiled count; otherwise the
// epilogue's request would never be granted).
struct DeviceSetup
{
    bool done;
    bool wide_fits;
    bool pair_fits;
};
std::mutex g_setup_mutex;
DeviceSetup g_setup[64] = {};

int device_setup(bool& wide_fits, bool& pair_fits)
{
    const int dev = current_device();
    if (dev < 0 || dev >= 64) return OSKB_ERR_CUDA_NOT_AVAILABLE;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    DeviceSetup& d = g_setup[dev];
    if (!d.done)
    {
        if (cudaFuncSetAttribute(gemm_kernel,
                cudaFuncAttributeMaxDynamicSharedMemorySize,
                (int) gemm_smem_bytes()) != cudaSuccess ||
                cudaFuncSetAttribute(gemm_wide_kernel,
                cudaFuncAttributeMaxDynamicSharedMemorySize,
                (int) gemm_wide_smem_bytes()) != cudaSuccess ||
                cudaFuncSetAttribute(gemm_pair_kernel,
                cudaFuncAttributeMaxDynamicSharedMemorySize,
                (int) gemm_pair_smem_bytes()) != cudaSuccess ||
                cudaFuncSetAttribute(gemm_i8_kernel,
                cudaFuncAttributeMaxDynamicSharedMemorySize,
                (int) gemm_i8_smem_bytes()) != cudaSuccess ||
                cudaFuncSetAttribute(gemm_l6_kernel,
                cudaFuncAttributeMaxDynamicSharedMemorySize,
                (int) gemm_l6_smem_bytes()) != cudaSuccess)
        {
            set_last_error("tc gemm attributes", cudaGetLastError());
            return OSKB_ERR_KERNEL_LAUNCH_FAILURE;
        }
        cudaFuncAttributes fa;
        d.wide_fits = cudaFuncGetAttributes(&fa, gemm_wide_kernel) ==
                cudaSuccess && (long long) fa.numRegs * kWThreads >=
                128LL * kWLowRegs + (kWThreads - 128LL) * kWHighRegs;
        if (!d.wide_fits)
            set_last_error_msg("tc: wide contraction tiles disabled "
                    "(register budget)");
        d.pair_fits = cudaFuncGetAttributes(&fa, gemm_pair_kernel) ==
                cudaSuccess && (long long) fa.numRegs * kWThreads >=
                128LL * kWLowRegs + (kWThreads - 128LL) * kWHighRegs;
        if (!d.pair_fits)
            set_last_error_msg("tc: pair contraction tiles disabled "
                    "(register budget)");
        d.done = true;
    }
    wide_fits = d.wide_fits;
    pair_fits = d.pair_fits;
    return 0;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point, so that
// the library links only the CUDA runtime and still loads on a host without
// a driver (the host-only entry points stay callable there).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType,
        cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*,
        const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
        CUtensorMapSwizzle, CUtensorMapL2promotion,
        CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled_fn()
{
    static std::atomic<EncodeTiledFn> fn{nullptr};
    EncodeTiledFn f = fn.load();
    if (f) return f;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p,
            cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
        return nullptr;
    f = reinterpret_cast<EncodeTiledFn>(p);
    fn.store(f);
    return f;
}

// Records the start event of a timed contraction launch (when timing is
// on) and returns the event to record after it, else nullptr.
cudaEvent_t timing_start(cudaStream_t stream)
{
    std::lock_guard<std::mutex> lock(g_timing_mutex);
    if (!g_timing) return nullptr;
    // a launch being captured into a graph is not timed (its replays would
    // all record into the one pair of events)
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(stream, &cs) == cudaSuccess &&
            cs != cudaStreamCaptureStatusNone)
        return nullptr;
    if (g_ev_used == g_ev.size())
    {
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        g_ev.emplace_back(e0, e1);
    }
    cudaEventRecord(g_ev[g_ev_used].first, stream);
    return g_ev[g_ev_used++].second;
}

int launch_gemm(GemmParams& gp, cudaStream_t stream)
{
    bool wide_fits = false, pair_fits = false;
    const int serr = device_setup(wide_fits, pair_fits);
    if (serr) return serr;
    const long long square = (long long) gp.nrb * (gp.nrb + 1) / 2 *
            gp.num_problems;
    if (gp.i8)
    {
        // square tiles (the integer image's only shape)
        g_last_arith.store(8);
        const int grid = (int) (square < num_sms() ? square : num_sms());
        g_last_tile.store(128);
        cudaEvent_t ev_stop = timing_start(stream);
        gemm_i8_kernel<<<grid, kGemmThreads, gemm_i8_smem_bytes(), stream>>>(
                gp);
        if (ev_stop) cudaEventRecord(ev_stop, stream);
        return check_launch("tc gemm (integer)");
    }
    const long long wide_n = (long long) wide_tiles(gp.nrb) *
            gp.num_problems;
    const long long pair_n = (long long) pair_tiles(gp.nrb) *
            gp.num_problems;
    const int setting = gp.form == kFormF16 ? 128 :
            gp.form == kFormF16Wide ? 256 : gp.form == kFormF16Pair ? 512 :
            tile_setting();
    const int pairs = num_sms() / 2;
    // pair tiles only on request: on one B200 at 512 stations x 100,000
    // sources x 16 channels they measured 52.6 ms per launch against 46.1 ms
    // for the wide tiles (drain every 2 blocks), 44.8 against 43.0 (every 3)
    const bool pair = pair_fits && setting == 512;
    const bool wide = !pair && wide_fits && (setting == 256 ||
            (setting == 0 && wide_n >= 2LL * num_sms()));
    const long long ntasks = pair ? pair_n : wide ? wide_n : square;
    int grid = (int) (ntasks < num_sms() ? ntasks : num_sms());
    if (pair)
        grid = 2 * (int) (pair_n < pairs ? pair_n : pairs);
    g_last_tile.store(pair ? 512 : wide ? 256 : 128);
    g_last_arith.store(16);
    gp.drain_kb = drain_kblocks();
    cudaEvent_t ev_stop = timing_start(stream);
    CUtensorMap tmap;
    if (pair)
    {
        // the operand image area as rows of 128 bytes (see gemm_pair_kernel)
        const size_t bytes = gp.image_stride ?
                gp.image_stride * (size_t) gp.num_problems :
                (size_t) gp.nrb * gp.nkb * kPairBytes;
        const cuuint64_t gdim[2] = {16, bytes / 128};
        const cuuint64_t gstride[1] = {128};
        const cuuint32_t box[2] = {16, 256};
        const cuuint32_t estride[2] = {1, 1};
        EncodeTiledFn encode = encode_tiled_fn();
        if (!encode || bytes / 128 >= (1ull << 31) ||
                encode(&tmap, CU_TENSOR_MAP_DATA_TYPE_UINT64,
                2, (void*) gp.W, gdim, gstride, box, estride,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        {
            set_last_error_msg("tc: operand tensor map");
            return OSKB_ERR_KERNEL_LAUNCH_FAILURE;
        }
    }
    if (pair)
        gemm_pair_kernel<<<grid, kWThreads, gemm_pair_smem_bytes(),
                stream>>>(gp, tmap);
    else if (wide)
        gemm_wide_kernel<<<grid, kWThreads, gemm_wide_smem_bytes(),
                stream>>>(gp);
    else
        gemm_kernel<<<grid, kGemmThreads, gemm_smem_bytes(), stream>>>(gp);
    if (ev_stop) cudaEventRecord(ev_stop, stream);
    return check_launch("tc gemm");
}

// Workspace layout: the Header, then (integer form) the source-order tables
// (I8Order), then the operand images.
size_t tables_bytes_for(bool i8, int num_src)
{
    return i8 ? i8_order_bytes(num_src, kI8DrainKb, nullptr, nullptr) : 0;
}

// Workspace bytes of np problems' images that suit either form.
size_t workspace_bytes_any(int num_st, int num_src, int np)
{
    const size_t f16 = (size_t) np * image_bytes(num_st, num_src);
    const size_t i8 = tables_bytes_for(true, num_src) +
            (size_t) np * image_bytes_i8(num_st, num_src);
    return kHeaderBytes + (f16 > i8 ? f16 : i8);
}

// The integer image's scale, buckets and source order for a J (or E) block
// of num_st x num_src ([station][source][2x2], shared by all problems):
// per-source and overall largest |entry| of J C, then the order tables.
template <typename TJ, typename TF = double>
int i8_order(const TJ* jones, int num_src, int num_st, const TF* I,
        const TF* Q, const TF* U, const TF* V, Header* hdr,
        const I8Order& o, cudaStream_t s, int drain_kb = kI8DrainKb)
{
    if (cudaMemsetAsync(o.amp_bits, 0, sizeof(unsigned int) * num_src, s) !=
            cudaSuccess)
    {
        set_last_error("tc source order clear", cudaGetLastError());
        return OSKB_ERR_KERNEL_LAUNCH_FAILURE;
    }
    const int gx = (num_src + 255) / 256;
    int gy = (4 * num_sms() + gx - 1) / gx;
    if (gy > num_st) gy = num_st;
    if (gy < 1) gy = 1;
    maxabs_src_kernel<TJ, TF><<<dim3(gx, gy), 256, 0, s>>>(jones,
            num_src, num_st, I, Q, U, V, o.amp_bits, &hdr->maxabs_bits,
            &hdr->flags);
    int err = check_launch("tc source amplitudes");
    if (err) return err;
    i8_order_kernel<<<1, kOrderThreads, 0, s>>>(num_src, drain_kb,
            &hdr->maxabs_bits, o);
    return check_launch("tc source order");
}

// One J block (oskb_cross_correlate_tc_d and the allocation-free entry
// point): scale, operand image and contraction, in the workspace at ws
// (the Header first; workspace_bytes_any(num_stations, num_sources, 1)
// bytes).
int jones_block(int casa, int num_sources, int num_stations, int offset_out,
        const double* jones, const double* I, const double* Q,
        const double* U, const double* V, const double* station_u,
        const double* station_v, double uv_min_lambda, double uv_max_lambda,
        double inv_wavelength, double* vis, uint8_t* ws, cudaStream_t s)
{
    Header* hdr = reinterpret_cast<Header*>(ws);
    // the status words start at zero; the image is rewritten
    if (cudaMemsetAsync(hdr, 0, sizeof(Header), s) != cudaSuccess)
    {
        set_last_error("tc header clear", cudaGetLastError());
        return OSKB_ERR_KERNEL_LAUNCH_FAILURE;
    }
    const int nrb = (num_stations + kStPerBlock - 1) / kStPerBlock;
    const int nkb = (num_sources + kSrcPerBlock - 1) / kSrcPerBlock;
    const bool i8 = arith_i8();
    GemmParams gp;
    gp.i8 = i8;
    gp.form = kFormDefault;
    gp.i8_counts = gp.i8_chunk_kb = gp.i8_chunk_bucket = nullptr;
    int err = 0;
    if (i8)
    {
        I8Order o;
        uint8_t* W = ws + kHeaderBytes + i8_order_bytes(num_sources,
                kI8DrainKb, ws + kHeaderBytes, &o);
        if ((err = i8_order<double>(jones, num_sources, num_stations, I, Q,
                U, V, hdr, o, s)))
            return err;
        const int cap = i8_kb_cap(num_sources);
        prep_jones_i8_kernel<double><<<dim3(cap, nrb), 256, 0, s>>>(jones,
                num_sources, num_stations, I, Q, U, V, &hdr->maxabs_bits, o,
                W);
        gp.W = W;
        gp.nkb = cap;
        gp.i8_counts = o.counts;
        gp.i8_chunk_kb = o.chunk_kb;
        gp.i8_chunk_bucket = o.chunk_bucket;
    }
    else
    {
        maxabs_kernel<double, double><<<num_sms() * 8, 256, 0, s>>>(jones,
                num_sources, num_stations, I, Q, U, V, &hdr->maxabs_bits,
                &hdr->flags);
        if ((err = check_launch("tc maxabs"))) return err;
        uint8_t* W = ws + kHeaderBytes;
        prep_jones_kernel<double><<<dim3(nkb, nrb), 256, 0, s>>>(jones,
                num_sources, num_stations, I, Q, U, V, &hdr->maxabs_bits, W);
        gp.W = W;
        gp.nkb = nkb;
    }
    if ((err = check_launch("tc prep"))) return err;
    gp.image_stride = 0; gp.nrb = nrb;
    gp.num_problems = 1; gp.num_st = num_stations;
    gp.maxabs_bits = &hdr->maxabs_bits; gp.maxabs_stride = 0;
    gp.prob0 = 0; gp.nch = 1;
    gp.vis = vis; gp.vis_stride = 0; gp.offset_out = offset_out;
    gp.st_u = station_u; gp.st_v = station_v; gp.uv_stride = 0;
    gp.inv_wavelength = nullptr; gp.kw_scalar = inv_wavelength;
    gp.uv_min = uv_min_lambda; gp.uv_max = uv_max_lambda;
    gp.casa = casa; gp.err = &hdr->err; gp.autos = nullptr;
    return launch_gemm(gp, s);
}

// Workspace of the FP64-class form: Header, source-order tables (chunks of
// kL6DrainKb k blocks), six-limb image.
size_t l6_workspace_bytes(int num_st, int num_src)
{
    return kHeaderBytes + i8_order_bytes(num_src, kL6DrainKb, nullptr,
            nullptr) + image_bytes_l6(num_st, num_src);
}

// One J block through the FP64-class form in the workspace at ws.
int l6_block(int casa, int num_sources, int num_stations, int offset_out,
        const double* jones, const double* I, const double* Q,
        const double* U, const double* V, const double* station_u,
        const double* station_v, double uv_min_lambda, double uv_max_lambda,
        double inv_wavelength, double* vis, uint8_t* ws, cudaStream_t s)
{
    bool wide_fits = false, pair_fits = false;
    int err = device_setup(wide_fits, pair_fits);
    if (err) return err;
    Header* hdr = reinterpret_cast<Header*>(ws);
    if (cudaMemsetAsync(hdr, 0, sizeof(Header), s) != cudaSuccess)
    {
        set_last_error("tc64 header clear", cudaGetLastError());
        return OSKB_ERR_KERNEL_LAUNCH_FAILURE;
    }
    const int nrb = (num_stations + kStPerBlock - 1) / kStPerBlock;
    I8Order o;
    uint8_t* W = ws + kHeaderBytes + i8_order_bytes(num_sources, kL6DrainKb,
            ws + kHeaderBytes, &o);
    if ((err = i8_order<double>(jones, num_sources, num_stations, I, Q, U,
            V, hdr, o, s, kL6DrainKb)))
        return err;
    const int cap = i8_kb_cap(num_sources);
    prep_jones_l6_kernel<<<dim3(cap, nrb), 256, 0, s>>>(jones, num_sources,
            num_stations, I, Q, U, V, &hdr->maxabs_bits, o, W);
    if ((err = check_launch("tc64 prep"))) return err;
    GemmParams gp;
    gp.i8 = 1;
    gp.form = kFormDefault;
    gp.i8_counts = o.counts;
    gp.i8_chunk_kb = o.chunk_kb;
    gp.i8_chunk_bucket = o.chunk_bucket;
    gp.skip_flags = &hdr->flags;
    gp.W = W; gp.image_stride = 0; gp.nrb = nrb; gp.nkb = cap;
    gp.num_problems = 1; gp.num_st = num_stations;
    gp.maxabs_bits = &hdr->maxabs_bits; gp.maxabs_stride = 0;
    gp.prob0 = 0; gp.nch = 1;
    gp.vis = vis; gp.vis_stride = 0; gp.offset_out = offset_out;
    gp.st_u = station_u; gp.st_v = station_v; gp.uv_stride = 0;
    gp.inv_wavelength = nullptr; gp.kw_scalar = inv_wavelength;
    gp.uv_min = uv_min_lambda; gp.uv_max = uv_max_lambda;
    gp.casa = casa; gp.err = &hdr->err; gp.autos = nullptr;
    const long long ntasks = (long long) nrb * (nrb + 1);
    const int grid = (int) (ntasks < num_sms() ? ntasks : num_sms());
    cudaEvent_t ev_stop = timing_start(s);
    gemm_l6_kernel<<<grid, kGemmThreads, gemm_l6_smem_bytes(), s>>>(gp);
    if (ev_stop) cudaEventRecord(ev_stop, s);
    return check_launch("tc64 gemm");
}

// Workspace of the FP32 entry point: Header, order tables, the integer
// image, FP64 sums of the visibilities, FP64 station u and v.
size_t tcf_workspace_bytes(int num_st, int num_src)
{
    const size_t nbl = (size_t) num_st * (num_st - 1) / 2;
    return kHeaderBytes + i8_order_bytes(num_src, kI8DrainKb, nullptr,
            nullptr) + image_bytes_i8(num_st, num_src) +
            align256_t(nbl * 8 * sizeof(double)) +
            2 * align256_t((size_t) num_st * sizeof(double));
}

// One FP32 J block through the integer form.
int tcf_block(int casa, int num_sources, int num_stations, int offset_out,
        const float* jones, const float* I, const float* Q, const float* U,
        const float* V, const float* station_u, const float* station_v,
        double uv_min_lambda, double uv_max_lambda, double inv_wavelength,
        float* vis, uint8_t* ws, cudaStream_t s)
{
    bool wide_fits = false, pair_fits = false;
    int err = device_setup(wide_fits, pair_fits);
    if (err) return err;
    Header* hdr = reinterpret_cast<Header*>(ws);
    const size_t nbl = (size_t) num_stations * (num_stations - 1) / 2;
    I8Order o;
    uint8_t* W = ws + kHeaderBytes + i8_order_bytes(num_sources, kI8DrainKb,
            ws + kHeaderBytes, &o);
    double* sums = reinterpret_cast<double*>(W +
            image_bytes_i8(num_stations, num_sources));
    double* du = reinterpret_cast<double*>(reinterpret_cast<uint8_t*>(sums)
            + align256_t(nbl * 8 * sizeof(double)));
    double* dv = reinterpret_cast<double*>(reinterpret_cast<uint8_t*>(du) +
            align256_t((size_t) num_stations * sizeof(double)));
    if (cudaMemsetAsync(hdr, 0, sizeof(Header), s) != cudaSuccess ||
            cudaMemsetAsync(sums, 0, nbl * 8 * sizeof(double), s) !=
            cudaSuccess)
    {
        set_last_error("tc (FP32) clear", cudaGetLastError());
        return OSKB_ERR_KERNEL_LAUNCH_FAILURE;
    }
    widen_uv_kernel<<<(num_stations + 255) / 256, 256, 0, s>>>(num_stations,
            station_u, station_v, du, dv);
    if ((err = check_launch("tc (FP32) uv"))) return err;
    if ((err = i8_order<float, float>(jones, num_sources, num_stations, I, Q,
            U, V, hdr, o, s)))
        return err;
    const int nrb = (num_stations + kStPerBlock - 1) / kStPerBlock;
    const int cap = i8_kb_cap(num_sources);
    prep_jones_i8_kernel<float><<<dim3(cap, nrb), 256, 0, s>>>(jones,
            num_sources, num_stations, I, Q, U, V, &hdr->maxabs_bits, o, W);
    if ((err = check_launch("tc (FP32) prep"))) return err;
    GemmParams gp;
    gp.i8 = 1;
    gp.form = kFormI8;
    gp.i8_counts = o.counts;
    gp.i8_chunk_kb = o.chunk_kb;
    gp.i8_chunk_bucket = o.chunk_bucket;
    gp.skip_flags = &hdr->flags;
    gp.W = W; gp.image_stride = 0; gp.nrb = nrb; gp.nkb = cap;
    gp.num_problems = 1; gp.num_st = num_stations;
    gp.maxabs_bits = &hdr->maxabs_bits; gp.maxabs_stride = 0;
    gp.prob0 = 0; gp.nch = 1;
    gp.vis = sums; gp.vis_stride = 0; gp.offset_out = 0;
    gp.st_u = du; gp.st_v = dv; gp.uv_stride = 0;
    gp.inv_wavelength = nullptr; gp.kw_scalar = inv_wavelength;
    gp.uv_min = uv_min_lambda; gp.uv_max = uv_max_lambda;
    gp.casa = casa; gp.err = &hdr->err; gp.autos = nullptr;
    if ((err = launch_gemm(gp, s))) return err;
    const size_t n = nbl * 8;
    const int grid = (int) std::min<size_t>((n + 255) / 256,
            (size_t) num_sms() * 8);
    add_vis_f_kernel<<<grid, 256, 0, s>>>(n, sums,
            vis + 8 * (size_t) offset_out);
    return check_launch("tc (FP32) add");
}

// The FP64-class block (oskb_correlate_block_tc64_d): as correlate_block
// with the six-limb image. Workspace: Header, tables, group x image.
int correlate_block_l6(int casa, int num_sources, int num_stations,
        int num_times, int num_channels, const double* E, const double* l,
        const double* m, const double* n, const double* I, const double* Q,
        const double* U, const double* V, const double* station_uvw,
        const double* inv_wavelength, double uv_min_lambda,
        double uv_max_lambda, double* vis, double* autos, void* workspace,
        size_t workspace_bytes, cudaStream_t s)
{
    const int num_problems = num_times * num_channels;
    const size_t img = image_bytes_l6(num_stations, num_sources);
    const size_t tb = i8_order_bytes(num_sources, kL6DrainKb, nullptr,
            nullptr);
    int group = num_problems;
    if (workspace)
    {
        if (workspace_bytes < kHeaderBytes + tb + img)
            return OSKB_ERR_MEMORY_ALLOC_FAILURE;
        const size_t fit = (workspace_bytes - kHeaderBytes - tb) / img;
        if ((size_t) group > fit) group = (int) fit;
    }
    else
    {
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        size_t fit = free_b / 2 / img;
        if (fit < 1) fit = 1;
        if ((size_t) group > fit) group = (int) fit;
        if (group > max_group()) group = max_group();
    }
    int err = get_workspace(workspace, workspace_bytes,
            kHeaderBytes + tb + (size_t) group * img, s);
    if (err) return err;
    bool wide_fits = false, pair_fits = false;
    if ((err = device_setup(wide_fits, pair_fits))) return err;
    uint8_t* ws = reinterpret_cast<uint8_t*>(workspace);
    Header* hdr = reinterpret_cast<Header*>(ws);
    uint8_t* W = ws + kHeaderBytes + tb;
    if (cudaMemsetAsync(hdr, 0, sizeof(Header), s) != cudaSuccess)
    {
        set_last_error("tc64 header clear", cudaGetLastError());
        return OSKB_ERR_KERNEL_LAUNCH_FAILURE;
    }
    I8Order o;
    i8_order_bytes(num_sources, kL6DrainKb, ws + kHeaderBytes, &o);
    // |K| = 1: one scale and source order from E C for the whole block
    if ((err = i8_order<double>(E, num_sources, num_stations, I, Q, U, V,
            hdr, o, s, kL6DrainKb)))
        return err;
    const int nrb = (num_stations + kStPerBlock - 1) / kStPerBlock;
    const int cap = i8_kb_cap(num_sources);
    const size_t nbl = (size_t) num_stations * (num_stations - 1) / 2;
    for (int p0 = 0; p0 < num_problems; p0 += group)
    {
        const int np = min(group, num_problems - p0);
        prep_fused_l6_kernel<double><<<dim3(cap, nrb), 256, 0, s>>>(E,
                num_sources, num_stations, l, m, n, I, Q, U, V, station_uvw,
                inv_wavelength, num_channels, p0, np, &hdr->maxabs_bits, o, W,
                img);
        if ((err = check_launch("tc64 prep fused"))) return err;
        GemmParams gp;
        gp.i8 = 1;
        gp.form = kFormDefault;
        gp.i8_counts = o.counts;
        gp.i8_chunk_kb = o.chunk_kb;
        gp.i8_chunk_bucket = o.chunk_bucket;
        gp.skip_flags = &hdr->flags;
        gp.W = W; gp.image_stride = img; gp.nrb = nrb; gp.nkb = cap;
        gp.num_problems = np; gp.num_st = num_stations;
        gp.maxabs_bits = &hdr->maxabs_bits; gp.maxabs_stride = 0;
        gp.prob0 = p0; gp.nch = num_channels;
        gp.vis = vis; gp.vis_stride = nbl; gp.offset_out = 0;
        gp.st_u = station_uvw; gp.st_v = station_uvw + num_stations;
        gp.uv_stride = 3 * (size_t) num_stations;
        gp.inv_wavelength = inv_wavelength; gp.kw_scalar = 0.0;
        gp.uv_min = uv_min_lambda; gp.uv_max = uv_max_lambda;
        gp.casa = casa; gp.err = &hdr->err; gp.autos = autos;
        const long long ntasks = (long long) nrb * (nrb + 1) * np;
        const int grid = (int) (ntasks < num_sms() ? ntasks : num_sms());
        cudaEvent_t ev_stop = timing_start(s);
        gemm_l6_kernel<<<grid, kGemmThreads, gemm_l6_smem_bytes(), s>>>(gp);
        if (ev_stop) cudaEventRecord(ev_stop, s);
        if ((err = check_launch("tc64 gemm"))) return err;
    }
    return 0;
}

}  // namespace
}  // namespace tc
}  // namespace oskb

using namespace oskb;
using namespace oskb::tc;

extern "C" {

size_t oskb_cross_correlate_tc_workspace_bytes(int num_sources,
        int num_stations)
{
    if (num_sources <= 0 || num_stations <= 0) return kHeaderBytes;
    return workspace_bytes_any(num_stations, num_sources, 1);
}

int oskb_cross_correlate_tc_d(int casa, int num_sources, int num_stations,
        int offset_out, const double* jones, const double* I,
        const double* Q, const double* U, const double* V,
        const double* station_u, const double* station_v,
        double uv_min_lambda, double uv_max_lambda, double inv_wavelength,
        double* vis, void* workspace, size_t workspace_bytes, void* stream)
{
    if (num_sources < 0 || num_stations < 0) return OSKB_ERR_INVALID_ARGUMENT;
    if (num_sources == 0 || num_stations < 2) return 0;
    if (!jones || !I || !Q || !U || !V || !station_u || !station_v || !vis)
        return OSKB_ERR_INVALID_ARGUMENT;
    const size_t need = oskb_cross_correlate_tc_workspace_bytes(num_sources,
            num_stations);
    cudaStream_t s = as_stream(stream);
    int err = get_workspace(workspace, workspace_bytes, need, s);
    if (err) return err;
    return jones_block(casa, num_sources, num_stations, offset_out, jones, I,
            Q, U, V, station_u, station_v, uv_min_lambda, uv_max_lambda,
            inv_wavelength, vis, reinterpret_cast<uint8_t*>(workspace), s);
}

size_t oskb_cross_correlate_tc_f_workspace_bytes(int num_sources,
        int num_stations)
{
    if (num_sources <= 0 || num_stations <= 0) return kHeaderBytes;
    return tcf_workspace_bytes(num_stations, num_sources);
}

int oskb_cross_correlate_tc_f(int casa, int num_sources, int num_stations,
        int offset_out, const float* jones, const float* I, const float* Q,
        const float* U, const float* V, const float* station_u,
        const float* station_v, float uv_min_lambda, float uv_max_lambda,
        float inv_wavelength, float* vis, void* workspace,
        size_t workspace_bytes, void* stream)
{
    if (num_sources < 0 || num_stations < 0) return OSKB_ERR_INVALID_ARGUMENT;
    if (num_sources == 0 || num_stations < 2) return 0;
    if (!jones || !I || !Q || !U || !V || !station_u || !station_v || !vis)
        return OSKB_ERR_INVALID_ARGUMENT;
    // 16 B per element of J: whole elements
    if ((uintptr_t) jones % 16 != 0) return OSKB_ERR_INVALID_ARGUMENT;
    const size_t need = oskb_cross_correlate_tc_f_workspace_bytes(
            num_sources, num_stations);
    cudaStream_t s = as_stream(stream);
    int err = get_workspace(workspace, workspace_bytes, need, s);
    if (err) return err;
    return tcf_block(casa, num_sources, num_stations, offset_out, jones, I, Q,
            U, V, station_u, station_v, uv_min_lambda, uv_max_lambda,
            inv_wavelength, vis, reinterpret_cast<uint8_t*>(workspace), s);
}

size_t oskb_cross_correlate_tc64_workspace_bytes(int num_sources,
        int num_stations)
{
    if (num_sources <= 0 || num_stations <= 0) return kHeaderBytes;
    return l6_workspace_bytes(num_stations, num_sources);
}

int oskb_cross_correlate_tc64_d(int casa, int num_sources, int num_stations,
        int offset_out, const double* jones, const double* I,
        const double* Q, const double* U, const double* V,
        const double* station_u, const double* station_v,
        double uv_min_lambda, double uv_max_lambda, double inv_wavelength,
        double* vis, void* workspace, size_t workspace_bytes, void* stream)
{
    if (num_sources < 0 || num_stations < 0) return OSKB_ERR_INVALID_ARGUMENT;
    if (num_sources == 0 || num_stations < 2) return 0;
    if (!jones || !I || !Q || !U || !V || !station_u || !station_v || !vis)
        return OSKB_ERR_INVALID_ARGUMENT;
    const size_t need = oskb_cross_correlate_tc64_workspace_bytes(
            num_sources, num_stations);
    cudaStream_t s = as_stream(stream);
    int err = get_workspace(workspace, workspace_bytes, need, s);
    if (err) return err;
    return l6_block(casa, num_sources, num_stations, offset_out, jones, I, Q,
            U, V, station_u, station_v, uv_min_lambda, uv_max_lambda,
            inv_wavelength, vis, reinterpret_cast<uint8_t*>(workspace), s);
}

size_t oskb_correlate_block_tc64_workspace_bytes(int num_sources,
        int num_stations, int num_problems)
{
    if (num_sources <= 0 || num_stations <= 0 || num_problems <= 0)
        return kHeaderBytes;
    return kHeaderBytes + i8_order_bytes(num_sources, kL6DrainKb, nullptr,
            nullptr) + (size_t) num_problems *
            image_bytes_l6(num_stations, num_sources);
}

int oskb_correlate_block_tc64_d(int casa, int num_sources, int num_stations,
        int num_times, int num_channels, const double* E, const double* l,
        const double* m, const double* n, const double* I, const double* Q,
        const double* U, const double* V, const double* station_uvw,
        const double* inv_wavelength, double uv_min_lambda,
        double uv_max_lambda, double* vis, void* workspace,
        size_t workspace_bytes, void* stream)
{
    if (num_sources < 0 || num_stations < 0 || num_times < 0 ||
            num_channels < 0)
        return OSKB_ERR_INVALID_ARGUMENT;
    if (num_sources == 0 || num_stations < 2 ||
            num_times * num_channels == 0)
        return 0;
    if (!E || !l || !m || !n || !I || !Q || !U || !V || !station_uvw ||
            !inv_wavelength || !vis)
        return OSKB_ERR_INVALID_ARGUMENT;
    return correlate_block_l6(casa, num_sources, num_stations, num_times,
            num_channels, E, l, m, n, I, Q, U, V, station_uvw,
            inv_wavelength, uv_min_lambda, uv_max_lambda, vis, nullptr,
            workspace, workspace_bytes, as_stream(stream));
}

int oskb_correlate_block_tc64_auto_d(int casa, int num_sources,
        int num_stations, int num_times, int num_channels, const double* E,
        const double* l, const double* m, const double* n, const double* I,
        const double* Q, const double* U, const double* V,
        const double* station_uvw, const double* inv_wavelength,
        double uv_min_lambda, double uv_max_lambda, double* vis,
        double* autos, void* workspace, size_t workspace_bytes, void* stream)
{
    if (num_sources < 0 || num_stations < 0 || num_times < 0 ||
            num_channels < 0)
        return OSKB_ERR_INVALID_ARGUMENT;
    if (num_sources == 0 || num_stations < 2 ||
            num_times * num_channels == 0)
        return 0;
    if (!E || !l || !m || !n || !I || !Q || !U || !V || !station_uvw ||
            !inv_wavelength || !vis || !autos)
        return OSKB_ERR_INVALID_ARGUMENT;
    return correlate_block_l6(casa, num_sources, num_stations, num_times,
            num_channels, E, l, m, n, I, Q, U, V, station_uvw,
            inv_wavelength, uv_min_lambda, uv_max_lambda, vis, autos,
            workspace, workspace_bytes, as_stream(stream));
}

size_t oskb_correlate_block_tc_workspace_bytes(int num_sources,
        int num_stations, int num_problems)
{
    if (num_sources <= 0 || num_stations <= 0 || num_problems <= 0)
        return kHeaderBytes;
    return workspace_bytes_any(num_stations, num_sources, num_problems);
}

int oskb_correlate_block_tc(int casa, int num_sources, int num_stations,
        int num_times, int num_channels, const float* E, const double* l,
        const double* m, const double* n, const double* I, const double* Q,
        const double* U, const double* V, const double* station_uvw,
        const double* inv_wavelength, double uv_min_lambda,
        double uv_max_lambda, double* vis, void* workspace,
        size_t workspace_bytes, void* stream)
{
    return oskb::tc::correlate_block<float>(casa, num_sources, num_stations,
            num_times, num_channels, E, l, m, n, I, Q, U, V, station_uvw,
            inv_wavelength, uv_min_lambda, uv_max_lambda, vis, workspace,
            workspace_bytes, stream, nullptr, nullptr, nullptr);
}

int oskb_correlate_block_tc_auto(int casa, int num_sources,
        int num_stations, int num_times, int num_channels, const float* E,
        const double* l, const double* m, const double* n, const double* I,
        const double* Q, const double* U, const double* V,
        const double* station_uvw, const double* inv_wavelength,
        double uv_min_lambda, double uv_max_lambda, double* vis,
        double* autos, void* workspace, size_t workspace_bytes, void* stream)
{
    return oskb::tc::correlate_block<float>(casa, num_sources, num_stations,
            num_times, num_channels, E, l, m, n, I, Q, U, V, station_uvw,
            inv_wavelength, uv_min_lambda, uv_max_lambda, vis, workspace,
            workspace_bytes, stream, nullptr, nullptr, autos);
}

int oskb_correlate_block_tc_d(int casa, int num_sources, int num_stations,
        int num_times, int num_channels, const double* E, const double* l,
        const double* m, const double* n, const double* I, const double* Q,
        const double* U, const double* V, const double* station_uvw,
        const double* inv_wavelength, double uv_min_lambda,
        double uv_max_lambda, double* vis, void* workspace,
        size_t workspace_bytes, void* stream)
{
    return oskb::tc::correlate_block<double>(casa, num_sources, num_stations,
            num_times, num_channels, E, l, m, n, I, Q, U, V, station_uvw,
            inv_wavelength, uv_min_lambda, uv_max_lambda, vis, workspace,
            workspace_bytes, stream, nullptr, nullptr, nullptr);
}

}  // extern "C"

namespace oskb {
namespace tc {

template <typename TE>
int correlate_block(int casa, int num_sources, int num_stations,
        int num_times, int num_channels, const TE* E, const double* l,
        const double* m, const double* n, const double* I, const double* Q,
        const double* U, const double* V, const double* station_uvw,
        const double* inv_wavelength, double uv_min_lambda,
        double uv_max_lambda, double* vis, void* workspace,
        size_t workspace_bytes, void* stream,
        void (*after_group)(void* ctx, int p0, int np), void* ctx,
        double* autos, int form)
{
    if (num_sources < 0 || num_stations < 0 || num_times < 0 ||
            num_channels < 0)
        return OSKB_ERR_INVALID_ARGUMENT;
    const int num_problems = num_times * num_channels;
    if (num_sources == 0 || num_stations < 2 || num_problems == 0) return 0;
    if (!E || !l || !m || !n || !I || !Q || !U || !V || !station_uvw ||
            !inv_wavelength || !vis)
        return OSKB_ERR_INVALID_ARGUMENT;
    // Problems (t, c) are processed in groups that fit the workspace.
    const bool i8 = form ? form == kFormI8 : arith_i8();
    const size_t img = image_bytes_for(i8, num_stations, num_sources);
    const size_t tb = tables_bytes_for(i8, num_sources);
    int group = num_problems;
    if (workspace)
    {
        if (workspace_bytes < kHeaderBytes + tb + img)
            return OSKB_ERR_MEMORY_ALLOC_FAILURE;
        const size_t fit = (workspace_bytes - kHeaderBytes - tb) / img;
        if ((size_t) group > fit) group = (int) fit;
    }
    else
    {
        // Library-kept workspace: at most max_group() images, and no more
        // than half of the device memory that is free now.
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        size_t fit = free_b / 2 / img;
        if (fit < 1) fit = 1;
        if ((size_t) group > fit) group = (int) fit;
        if (group > max_group()) group = max_group();
    }
    cudaStream_t s = as_stream(stream);
    int err = get_workspace(workspace, workspace_bytes,
            kHeaderBytes + tb + (size_t) group * img, s);
    if (err) return err;
    uint8_t* ws = reinterpret_cast<uint8_t*>(workspace);
    Header* hdr = reinterpret_cast<Header*>(ws);
    uint8_t* W = ws + kHeaderBytes + tb;
    if (cudaMemsetAsync(hdr, 0, sizeof(Header), s) != cudaSuccess)
    {
        set_last_error("tc header clear", cudaGetLastError());
        return OSKB_ERR_KERNEL_LAUNCH_FAILURE;
    }
    // |K| = 1: one scale (and, for the integer image, one source order)
    // from E C serves every problem of the block.
    I8Order o = {};
    if (i8)
    {
        i8_order_bytes(num_sources, kI8DrainKb, ws + kHeaderBytes, &o);
        if ((err = i8_order<TE>(E, num_sources, num_stations, I, Q, U, V,
                hdr, o, s)))
            return err;
    }
    else
    {
        maxabs_kernel<TE, double><<<num_sms() * 8, 256, 0, s>>>(E,
                num_sources, num_stations, I, Q, U, V, &hdr->maxabs_bits,
                &hdr->flags);
        if ((err = check_launch("tc maxabs"))) return err;
    }
    const int nrb = (num_stations + kStPerBlock - 1) / kStPerBlock;
    const int nkb = (num_sources + kSrcPerBlock - 1) / kSrcPerBlock;
    const int cap = i8_kb_cap(num_sources);
    const size_t nbl = (size_t) num_stations * (num_stations - 1) / 2;
    for (int p0 = 0; p0 < num_problems; p0 += group)
    {
        const int np = min(group, num_problems - p0);
        if (i8)
            prep_fused_i8_kernel<TE><<<dim3(cap, nrb), 256, 0, s>>>(E,
                    num_sources, num_stations,
                    l, m, n, I, Q, U, V, station_uvw, inv_wavelength,
                    num_channels, p0, np, &hdr->maxabs_bits, o, W, img);
        else
            prep_fused_kernel<TE><<<dim3(nkb, nrb), 256, 0, s>>>(E,
                    num_sources, num_stations, l, m, n, I, Q, U, V,
                    station_uvw, inv_wavelength, num_channels, p0, np,
                    &hdr->maxabs_bits, W, img);
        if ((err = check_launch("tc prep fused"))) return err;
        GemmParams gp;
        gp.i8 = i8;
        gp.i8_counts = o.counts;
        gp.i8_chunk_kb = o.chunk_kb;
        gp.i8_chunk_bucket = o.chunk_bucket;
        gp.form = form;
        gp.W = W; gp.image_stride = img; gp.nrb = nrb;
        gp.nkb = i8 ? cap : nkb;
        gp.num_problems = np; gp.num_st = num_stations;
        gp.maxabs_bits = &hdr->maxabs_bits; gp.maxabs_stride = 0;
        gp.prob0 = p0; gp.nch = num_channels;
        gp.vis = vis; gp.vis_stride = nbl; gp.offset_out = 0;
        gp.st_u = station_uvw; gp.st_v = station_uvw + num_stations;
        gp.uv_stride = 3 * (size_t) num_stations;
        gp.inv_wavelength = inv_wavelength; gp.kw_scalar = 0.0;
        gp.uv_min = uv_min_lambda; gp.uv_max = uv_max_lambda;
        gp.casa = casa; gp.err = &hdr->err; gp.autos = autos;
        if ((err = launch_gemm(gp, s))) return err;
        if (after_group) after_group(ctx, p0, np);
    }
    return 0;
}

template int correlate_block<float>(int, int, int, int, int, const float*,
        const double*, const double*, const double*, const double*,
        const double*, const double*, const double*, const double*,
        const double*, double, double, double*, void*, size_t, void*,
        void (*)(void*, int, int), void*, double*, int);
template int correlate_block<double>(int, int, int, int, int, const double*,
        const double*, const double*, const double*, const double*,
        const double*, const double*, const double*, const double*,
        const double*, double, double, double*, void*, size_t, void*,
        void (*)(void*, int, int), void*, double*, int);

int setup_device()
{
    bool wide_fits = false, pair_fits = false;
    return device_setup(wide_fits, pair_fits);
}

}  // namespace tc
}  // namespace oskb

extern "C" {

int oskb_tc_timing(int enable)
{
    std::lock_guard<std::mutex> lock(g_timing_mutex);
    g_timing = enable != 0;
    g_ev_used = 0;
    return 0;
}

int oskb_tc_timing_read(double* total_ms, int* launches)
{
    std::lock_guard<std::mutex> lock(g_timing_mutex);
    double sum = 0.0;
    for (size_t i = 0; i < g_ev_used; ++i)
    {
        float ms = 0.0f;
        if (cudaEventSynchronize(g_ev[i].second) != cudaSuccess ||
                cudaEventElapsedTime(&ms, g_ev[i].first, g_ev[i].second)
                != cudaSuccess)
            return OSKB_ERR_KERNEL_LAUNCH_FAILURE;
        sum += ms;
    }
    if (total_ms) *total_ms = sum;
    if (launches) *launches = (int) g_ev_used;
    g_ev_used = 0;
    return 0;
}

int oskb_tc_tile_columns(void)
{
    return g_last_tile.load();
}

int oskb_tc_arithmetic(void)
{
    return g_last_arith.load();
}

int oskb_tc_status(const void* workspace, int* flags, int* wait_error)
{
    const void* ws = workspace;
    if (!ws)
    {
        const int dev = current_device();
        std::lock_guard<std::mutex> lock(g_ws_mutex);
        ws = (dev >= 0 && dev < 64) ? g_ws_last[dev] : nullptr;
    }
    if (!ws) return OSKB_ERR_INVALID_ARGUMENT;
    Header h;
    if (cudaMemcpy(&h, ws, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess)
        return OSKB_ERR_MEMORY_COPY_FAILURE;
    if (flags) *flags = h.flags;
    if (wait_error) *wait_error = h.err;
    return 0;
}

}  // extern "C"

// ===========================================================================
// Allocation-free form of the tensor-core correlation.
//
// Some callers cannot allocate device memory at the time they correlate: a
// process that reserves a fixed device-memory budget at start-up (a real-time
// correlator or pipeline stage sharing the GPU with other software) must not
// grow past it, and cudaMalloc may synchronise the whole device, which a
// latency-critical caller cannot afford in its processing loop. For them this
// entry point takes its scratch (status words and the FP16 operand image)
// from a file-scope device array of fixed size instead of a workspace.
// ===========================================================================
#include <mutex>

namespace oskb {
namespace tc {
namespace {

// Maximum scratch of the allocation-free entry point: 64 MiB, held by every
// GPU that loads the library until the process exits. Beside a 256-byte
// status header, the operand image needs 32 bytes per station-source in the
// FP16 form (an FP16 hi and lo word for each of the 8 real parts of J C),
// 24 in the integer form (three limbs each) plus its source-order tables
// (about 8 bytes per source), rounded up to blocks of 32 stations x 32
// sources (the integer form's buckets pad up to 15 more source blocks); the
// size check takes the larger of the two whichever form runs: e.g. up to
// 512 stations x 4,064 sources per call (4,096 sources no longer fit).
constexpr size_t kStaticScratchBytes = (size_t) 64 << 20;

static __device__ __align__(256) uint8_t g_static_scratch[kStaticScratchBytes];

// Device address of g_static_scratch for each device, taken once per device
// with that device current (the host-side symbol is not a device address).
std::mutex g_static_mutex;
void* g_static_ptr[64] = {};

int static_scratch(void** ptr)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
        return OSKB_ERR_CUDA_NOT_AVAILABLE;
    std::lock_guard<std::mutex> lock(g_static_mutex);
    if (!g_static_ptr[dev])
    {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p)
        {
            set_last_error("static scratch address", e);
            return OSKB_ERR_CUDA_NOT_AVAILABLE;
        }
        g_static_ptr[dev] = p;
    }
    *ptr = g_static_ptr[dev];
    return 0;
}

}  // namespace
}  // namespace tc
}  // namespace oskb

extern "C" int oskb_cross_correlate_tc_noalloc_d(int casa, int num_sources,
        int num_stations, int offset_out, const double* jones,
        const double* I, const double* Q, const double* U, const double* V,
        const double* station_u, const double* station_v,
        double uv_min_lambda, double uv_max_lambda, double inv_wavelength,
        double* vis, void* stream)
{
    if (num_sources < 0 || num_stations < 0) return OSKB_ERR_INVALID_ARGUMENT;
    if (num_sources == 0 || num_stations < 2) return 0;
    if (!jones || !I || !Q || !U || !V || !station_u || !station_v || !vis)
        return OSKB_ERR_INVALID_ARGUMENT;
    const size_t need = workspace_bytes_any(num_stations, num_sources, 1);
    if (need > kStaticScratchBytes)
    {
        char msg[200];
        snprintf(msg, sizeof(msg), "oskb_cross_correlate_tc_noalloc_d: %d "
                "stations x %d sources need %zu bytes of scratch; the static "
                "scratch holds %zu (split the sources into chunks)",
                num_stations, num_sources, need, kStaticScratchBytes);
        set_last_error_msg(msg);
        return OSKB_ERR_OUT_OF_RANGE;
    }
    void* scratch = nullptr;
    int err = static_scratch(&scratch);
    if (err) return err;
    // The array keeps the previous call's contents: the status words are
    // cleared and the tables and operand image rewritten by the call.
    return jones_block(casa, num_sources, num_stations, offset_out, jones, I,
            Q, U, V, station_u, station_v, uv_min_lambda, uv_max_lambda,
            inv_wavelength, vis, reinterpret_cast<uint8_t*>(scratch),
            as_stream(stream));
}

// Status words of the last allocation-free call on the current device: the
// header of the static array, read with a plain device-to-host copy (no
// allocation). Synchronises with the device.
extern "C" int oskb_tc_noalloc_status(int* flags, int* wait_error)
{
    void* scratch = nullptr;
    const int err = static_scratch(&scratch);
    if (err) return err;
    Header h;
    const cudaError_t e = cudaMemcpy(&h, scratch, sizeof(h),
            cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
    {
        set_last_error("static scratch status", e);
        return OSKB_ERR_MEMORY_COPY_FAILURE;
    }
    if (flags) *flags = h.flags;
    if (wait_error) *wait_error = h.err;
    return 0;
}

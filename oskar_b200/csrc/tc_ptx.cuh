// Thin inline-PTX wrappers for sm_100a: mbarriers, bulk (TMA) copies and the
// tcgen05 tensor-core instructions (TMEM allocation, MMA, commit, loads).
// Every wait is bounded in wall-clock time: on expiry it records an error
// code in a global flag and returns false, so no kernel can spin forever.
#pragma once

#include <stdint.h>

namespace oskb {
namespace ptx {

// Wait limit for any single barrier wait (nanoseconds of %globaltimer).
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t) __cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---- mbarrier
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;"
                 :: "r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];"
                 :: "r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar,
        uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, "
                 "[%0], %1;" :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}

// Waits for the phase with the given parity to complete. Returns false (and
// sets *err = code unless already set) if it has not completed within
// kWaitLimitNs, or if *abort became non-zero meanwhile.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
        int* err, int code, volatile int* abort)
{
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t it = 1;; ++it)
    {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 255u) == 0)
        {
            if (*abort) return false;
            if (global_ns() - t0 > kWaitLimitNs)
            {
                if (err) atomicCAS(err, 0, code);
                *abort = 1;
                return false;
            }
        }
    }
}

// ---- bulk copy global -> shared (TMA engine, non-tensor form). Both
// addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst_smem, const void* src,
        uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx"
                 "::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_u32(dst_smem)), "l"(src), "r"(bytes),
                    "r"(smem_u32(bar)) : "memory");
}

// ---- bulk copy shared -> global (TMA engine, non-tensor form), bulk-group
// completion. Both addresses 16-byte aligned, bytes a multiple of 16.
// Shared-memory writes by threads must be made visible to the copy first
// (fence_proxy_async_smem by the writing threads, then a block barrier).
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void bulk_s2g(void* dst, const void* src_smem,
        uint32_t bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;"
                 :: "l"(dst), "r"(smem_u32(src_smem)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_commit()
{
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// Waits until at most N committed bulk groups still read shared memory.
template <int N>
__device__ __forceinline__ void bulk_wait_read()
{
    asm volatile("cp.async.bulk.wait_group.read %0;" :: "n"(N) : "memory");
}

// Waits until at most N committed bulk groups are incomplete.
template <int N>
__device__ __forceinline__ void bulk_wait()
{
    asm volatile("cp.async.bulk.wait_group %0;" :: "n"(N) : "memory");
}

// ---- tcgen05: TMEM allocation (whole warp), MMA, commit, loads, fences
__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 "
                 "[%0], %1;" :: "r"(smem_u32(dst_smem)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;"
                 ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :: "r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_fence_before()
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_after()
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, kind::f16 (FP16 inputs, FP32 accumulate)
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a_desc,
        uint64_t b_desc, uint32_t idesc, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                 :: "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc),
                    "r"(accumulate) : "memory");
}

// D (S32, TMEM) (+)= A B^T for 8-bit A and B (signedness in the instruction
// descriptor; K = 32 per instruction, both K-major in shared memory), no
// output lanes disabled.
__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t a_desc,
        uint64_t b_desc, uint32_t idesc, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, "
                 "{%5, %6, %7, %8}, p;\n\t}"
                 :: "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc),
                    "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                 : "memory");
}

// mma_i8 with the A operand kept in the tensor core's collector buffer for
// the next MMAs of the same A: Use = 0 reads A and fills the buffer, 1 reuses
// it, 2 reuses it for the last time.
template <int Use>
__device__ __forceinline__ void mma_i8_col(uint32_t d_tmem, uint64_t a_desc,
        uint64_t b_desc, uint32_t idesc, uint32_t accumulate)
{
    if constexpr (Use == 0)
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "setp.ne.b32 p, %4, 0;\n\t"
                     "tcgen05.mma.cta_group::1.kind::i8.collector::a::fill "
                     "[%0], %1, %2, %3, p;\n\t}"
                     :: "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc),
                        "r"(accumulate) : "memory");
    else if constexpr (Use == 1)
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "setp.ne.b32 p, %4, 0;\n\t"
                     "tcgen05.mma.cta_group::1.kind::i8.collector::a::use "
                     "[%0], %1, %2, %3, p;\n\t}"
                     :: "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc),
                        "r"(accumulate) : "memory");
    else
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "setp.ne.b32 p, %4, 0;\n\t"
                     "tcgen05.mma.cta_group::1.kind::i8.collector::a::lastuse "
                     "[%0], %1, %2, %3, p;\n\t}"
                     :: "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc),
                        "r"(accumulate) : "memory");
}

// Arrives on an mbarrier once all previously issued MMAs have completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one"
                 ".shared::cluster.b64 [%0];" :: "r"(smem_u32(bar))
                 : "memory");
}

// 32 consecutive 32-bit TMEM columns of this thread's lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t* v)
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                 "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, "
                 "%24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]),
                   "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                   "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                   "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
                   "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]),
                   "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
                   "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
                   "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                 : "r"(taddr) : "memory");
}

// 16 consecutive 32-bit TMEM columns of this thread's lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* v)
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                 "%13, %14, %15}, [%16];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]),
                   "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                   "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                   "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                 : "r"(taddr) : "memory");
}

// Per-thread register budget of the executing warp (whole warpgroup, all
// lanes converged): release down to N, or request up to N (waits until
// the block's released registers cover it).
template <int N>
__device__ __forceinline__ void regs_release()
{
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" :: "n"(N) : "memory");
}

template <int N>
__device__ __forceinline__ void regs_request()
{
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" :: "n"(N) : "memory");
}

__device__ __forceinline__ void tmem_ld_wait()
{
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Shared-memory matrix descriptor for a K-major operand tile stored with the
// 128-byte swizzle: rows of 128 bytes, 8-row groups 1024 bytes apart, tile
// base 1024-byte aligned (sm_100 descriptor format, version 1).
__device__ __forceinline__ uint64_t sdesc_sw128(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t) ((saddr & 0x3FFFFu) >> 4);  // start address
    d |= (uint64_t) 1 << 16;                     // leading byte offset (unused)
    d |= (uint64_t) (1024u >> 4) << 32;          // stride byte offset
    d |= (uint64_t) 1 << 46;                     // descriptor version
    d |= (uint64_t) 2 << 61;                     // 128-byte swizzle
    return d;
}

// The same for a tile stored with the 64-byte swizzle: rows of 64 bytes,
// 8-row groups 512 bytes apart, tile base 512-byte aligned; byte c of row r
// sits at r * 64 + ((c / 16) ^ ((r / 2) % 4)) * 16 + c % 16.
__device__ __forceinline__ uint64_t sdesc_sw64(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t) ((saddr & 0x3FFFFu) >> 4);  // start address
    d |= (uint64_t) 1 << 16;                     // leading byte offset (unused)
    d |= (uint64_t) (512u >> 4) << 32;           // stride byte offset
    d |= (uint64_t) 1 << 46;                     // descriptor version
    d |= (uint64_t) 4 << 61;                     // 64-byte swizzle
    return d;
}

// ---- thread-block pairs (cluster of two CTAs, cta_group::2)
__device__ __forceinline__ uint32_t cluster_ctarank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// All threads of both CTAs of the cluster.
__device__ __forceinline__ void cluster_sync()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\t"
                 "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Shared::cluster address of the variable at local shared address saddr in
// the CTA of the given rank.
__device__ __forceinline__ uint32_t mapa_shared(uint32_t saddr, uint32_t rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;"
                 : "=r"(r) : "r"(saddr), "r"(rank));
    return r;
}

// Arrive (release at cluster scope) on an mbarrier given by its
// shared::cluster address, possibly in the peer CTA.
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t cluster_addr)
{
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, "
                 "[%0];" :: "r"(cluster_addr) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait_cluster(uint64_t* bar,
        uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 "
                 "p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}

// mbar_wait for barriers that threads of the peer CTA arrive on: the
// acquire is at cluster scope, the limit and abort as in mbar_wait.
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t* bar,
        uint32_t parity, int* err, int code, volatile int* abort)
{
    if (mbar_try_wait_cluster(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t it = 1;; ++it)
    {
        if (mbar_try_wait_cluster(bar, parity)) return true;
        if ((it & 255u) == 0)
        {
            if (*abort) return false;
            if (global_ns() - t0 > kWaitLimitNs)
            {
                if (err) atomicCAS(err, 0, code);
                *abort = 1;
                return false;
            }
        }
    }
}

// Tensor-map (TMA) load of a 2-D box into this CTA's shared memory whose
// completion is reported to an mbarrier of either CTA of the pair (its
// shared::cluster address): the copy form of cta_group::2. No multicast.
// The box's innermost coordinate x must be a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_2d_pair(void* dst_smem,
        const void* tmap, int x, int y, uint32_t mbar_cluster)
{
    asm volatile("cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global"
                 ".mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                 :: "r"(smem_u32(dst_smem)), "l"(tmap), "r"(x), "r"(y),
                    "r"(mbar_cluster) : "memory");
}

// TMEM of both CTAs of a pair: one warp of each CTA (the same warp index),
// the same shared-memory destination offset in both.
__device__ __forceinline__ void tmem_alloc_pair(uint32_t* dst_smem,
        uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 "
                 "[%0], %1;" :: "r"(smem_u32(dst_smem)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;"
                 ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc_pair(uint32_t taddr,
        uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;"
                 :: "r"(taddr), "r"(ncols) : "memory");
}

// Pair MMA, issued by one thread of the even CTA: D (M = 256: rows 0-127 in
// the even CTA's TMEM, 128-255 in the odd CTA's) (+)= A B^T, A's rows
// 0-127 and 128-255 read from the two CTAs' shared memory at the same
// offset, B's N rows split the same way (first N/2 from the even CTA).
__device__ __forceinline__ void mma_f16_pair(uint32_t d_tmem, uint64_t a_desc,
        uint64_t b_desc, uint32_t idesc, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                 :: "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc),
                    "r"(accumulate) : "memory");
}

// Arrives on the mbarrier at the same shared offset in both CTAs of the
// pair once all previously issued pair MMAs have completed.
__device__ __forceinline__ void mma_commit_pair(uint64_t* bar)
{
    const uint16_t mask = 0x3;
    asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one"
                 ".shared::cluster.multicast::cluster.b64 [%0], %1;"
                 :: "r"(smem_u32(bar)), "h"(mask) : "memory");
}

// Instruction descriptor: FP16 A and B (K-major), FP32 accumulator, M x N.
__host__ __device__ constexpr uint32_t idesc_f16_f32(int m, int n)
{
    return (1u << 4) | ((uint32_t) (n >> 3) << 17) |
           ((uint32_t) (m >> 4) << 24);
}

// Instruction descriptor of kind::i8: S32 accumulator (bits 4-5 = 2), A and
// B 8-bit, signed (1) or unsigned (0) at bits 7-9 and 10-12, both K-major,
// N / 8 at bit 17, M / 16 at bit 24.
__host__ __device__ constexpr uint32_t idesc_i8_s32(int m, int n,
        bool a_signed, bool b_signed)
{
    return (2u << 4) | ((a_signed ? 1u : 0u) << 7) |
           ((b_signed ? 1u : 0u) << 10) |
           ((uint32_t) (n >> 3) << 17) | ((uint32_t) (m >> 4) << 24);
}

}  // namespace ptx
}  // namespace oskb

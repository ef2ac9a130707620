// sm_100a building blocks for the tensor-core convolution kernels: mbarriers
// with bounded waits, TMA tensor-map tile loads (this GPU's own memory, no
// multicast), and the tcgen05 tensor-core / tensor-memory instructions.
//
// Shared-memory matrix descriptors follow the PTX ISA "tcgen05 shared memory
// descriptor" layout: start address >> 4 in bits 0-13, leading byte offset
// >> 4 in bits 16-29, stride byte offset >> 4 in bits 32-45, the fixed value
// 0b001 in bits 46-48, base offset 0 in bits 49-51, swizzle mode in bits
// 61-63 (2 = 128-byte swizzle). Instruction descriptors for kind::f16: D format in bits 4-5
// (1 = f32), A/B formats in bits 7-9 / 10-12 (1 = bf16), A/B major in bits
// 15 / 16 (0 = K-major, 1 = MN-major), N >> 3 in bits 17-22, M >> 4 in bits
// 24-28.
#pragma once

#include <cstdint>
#include <cuda.h>

namespace mlb {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---- mbarriers --------------------------------------------------------------

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_barrier_init()
{
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async()
{
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
               :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
  uint32_t ok;
  asm volatile(
    "{\n\t.reg .pred p;\n\t"
    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
    "selp.u32 %0, 1, 0, p;\n\t}"
    : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
  return ok != 0;
}
// Wait for the phase of parity `parity` to complete; gives up after about
// 2^31 clock cycles (about a second) and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
  if(mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while(!mbar_try_wait(bar, parity))
    if(clock64() - t0 > (1ll << 31)) return false;
  return true;
}

// ---- TMA tile loads (tensor maps over this GPU's global memory) ----------------

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1,
                                            int c2, uint64_t* bar)
{
  asm volatile(
    "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
    " [%0], [%1, {%2, %3, %4}], [%5];"
    :: "r"(smem_u32(dst)), "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
    : "memory");
}
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1,
                                            int c2, int c3, uint64_t* bar)
{
  asm volatile(
    "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
    " [%0], [%1, {%2, %3, %4, %5}], [%6];"
    :: "r"(smem_u32(dst)), "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
    : "memory");
}
// shared memory -> global tile store (this GPU's memory); completes through
// the bulk async-group of the issuing thread
__device__ __forceinline__ void tma_store_4d(const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                             const void* src)
{
  asm volatile(
    "cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4}], [%5];"
    :: "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(src)) : "memory");
}
__device__ __forceinline__ void bulk_commit()
{
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// the issuing thread's committed stores have finished reading shared memory
__device__ __forceinline__ void bulk_wait_read_all()
{
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
// ... and have completed their global writes
__device__ __forceinline__ void bulk_wait_all()
{
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// named barrier `id` over `n` threads (a multiple of 32)
__device__ __forceinline__ void named_sync(int id, int n)
{
  asm volatile("bar.sync %0, %1;" :: "r"(id), "r"(n) : "memory");
}
// named barrier that also returns the AND of `v` over its `n` threads, so
// every participant takes the same branch afterwards
__device__ __forceinline__ bool named_and(int id, int n, bool v)
{
  uint32_t r;
  asm volatile(
    "{\n\t.reg .pred pi, po;\n\t"
    "setp.ne.u32 pi, %1, 0;\n\t"
    "bar.red.and.pred po, %2, %3, pi;\n\t"
    "selp.u32 %0, 1, 0, po;\n\t}"
    : "=r"(r) : "r"(static_cast<uint32_t>(v)), "r"(id), "r"(n) : "memory");
  return r != 0;
}

__device__ __forceinline__ void prefetch_map(const CUtensorMap* map)
{
  asm volatile("prefetch.tensormap [%0];" :: "l"(map) : "memory");
}

// ---- tcgen05 ------------------------------------------------------------------

// whole warp; writes the TMEM base address to *dst (shared memory)
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols)
{
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
               :: "r"(smem_u32(dst)), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tmem_relinquish()
{
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
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

// D[tmem] (+)= A[smem] * B[smem]^T, one thread issues. No memory clobber:
// the operands are ordered by the mbarrier waits before and the commits
// after (both volatile with clobbers), and a memory clobber here costs
// issue slots on every MMA.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc,
                                         uint32_t idesc, uint32_t accumulate)
{
  asm volatile(
    "{\n\t.reg .pred p;\n\t"
    "setp.ne.b32 p, %4, 0;\n\t"
    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
    :: "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate));
}
// The same MMA with the A-operand collector buffer: COLL 1 fills it from
// shared memory (A read as usual, then kept), 2 reads A from it, 3 reads A
// from it for the last time. A run fill, use..., lastuse lets consecutive
// MMAs that share A (same descriptor) but take different B read A from
// shared memory once.
template<int COLL>
__device__ __forceinline__ void mma_bf16_coll(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc,
                                              uint32_t idesc, uint32_t accumulate)
{
  static_assert(COLL >= 0 && COLL <= 3, "collector usage");
  if constexpr(COLL == 0)
    mma_bf16(d_tmem, a_desc, b_desc, idesc, accumulate);
  else if constexpr(COLL == 1)
    asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16.collector::a::fill [%0], %1, %2, %3, p;\n\t}"
      :: "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate));
  else if constexpr(COLL == 2)
    asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16.collector::a::use [%0], %1, %2, %3, p;\n\t}"
      :: "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate));
  else
    asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16.collector::a::lastuse [%0], %1, %2, %3, p;\n\t}"
      :: "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate));
}
// arrive on `bar` once every tcgen05.mma issued so far by this thread is done
__device__ __forceinline__ void mma_commit(uint64_t* bar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :: "r"(smem_u32(bar)) : "memory");
}

// 32 lanes x 32 consecutive 32-bit columns: thread t gets lane (base lane + t)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v)
{
  uint32_t r[32];
  asm volatile(
    "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
    "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
    "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
      "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
      "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
      "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
      "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
    : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for(int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v)
{
  uint32_t r[16];
  asm volatile(
    "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
    "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
      "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
      "=r"(r[14]), "=r"(r[15])
    : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for(int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// ---- descriptors ----------------------------------------------------------------

// 128-byte-swizzled operand tile in shared memory. K-major: rows of 128 bytes
// (64 bf16 along K), 8-row groups `sbo` bytes apart (lbo unused). MN-major:
// rows are K indices holding 64 bf16 along M/N, 8-row K groups `sbo` apart,
// 64-element M/N groups `lbo` apart. The 128-byte swizzle is a function of
// the absolute shared-memory address (16-byte chunk bits 4-6 XOR row bits
// 7-9), the same one TMA applies when it writes a tile to a 1024-aligned
// address, so a matrix may start at any 128-byte row inside such a tile
// with the base-offset field left 0 (the convolution kernels rely on this;
// their GPU tests check it against the CPU oracle).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
  uint64_t d = 0;
  d |= static_cast<uint64_t>((saddr & 0x3FFFFu) >> 4);
  d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
  d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
  d |= 1ull << 46;
  d |= 2ull << 61;
  return d;
}

__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N, int a_mn_major, int b_mn_major)
{
  return (1u << 4) | (1u << 7) | (1u << 10) |
         (static_cast<uint32_t>(a_mn_major) << 15) | (static_cast<uint32_t>(b_mn_major) << 16) |
         (static_cast<uint32_t>(N >> 3) << 17) | (static_cast<uint32_t>(M >> 4) << 24);
}

} // namespace tc
} // namespace mlb

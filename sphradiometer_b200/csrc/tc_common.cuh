// tc_common.cuh -- PTX wrappers for sm_100a shared by the tcgen05 kernels:
// mbarriers with bounded waits, TMA / bulk copies, UMMA descriptors,
// tcgen05.mma (kind::f16, bf16 operands, FP32 accumulation in TMEM),
// commits and TMEM loads.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace sphrad {

constexpr unsigned long long kWaitCycles = 4000000000ull;  // ~2 s bound on every wait

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t) __cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
	asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_arrive_tx(uint32_t bar, uint32_t bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity)
{
	uint32_t ok;
	asm volatile(
		"{\n\t.reg .pred P;\n\t"
		"mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
		"selp.u32 %0, 1, 0, P;\n\t}"
		: "=r"(ok)
		: "r"(bar), "r"(parity)
		: "memory");
	return ok != 0;
}

// bounded wait: false on timeout after limit clock cycles (sets the abort
// flag and the error word) or when another role has aborted
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int *abort_flag, unsigned *err, unsigned code,
					  unsigned long long limit = kWaitCycles)
{
	const unsigned long long t0 = clock64();
	while(true) {
		if(mbar_try(bar, parity))
			return true;
		if(*abort_flag)
			return false;
		if(clock64() - t0 > limit) {
			*abort_flag = 1;
			atomicExch(err, code);
			return false;
		}
	}
}

// bounded wait that ignores the abort flag (draining copies in flight)
__device__ __forceinline__ void mbar_drain(uint32_t bar, uint32_t parity, unsigned long long limit = kWaitCycles)
{
	const unsigned long long t0 = clock64();
	while(!mbar_try(bar, parity) && clock64() - t0 < limit) {
	}
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, uint32_t bar, int x, int y, int z)
{
	asm volatile(
		"cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(dst),
		"l"((uint64_t) map), "r"(bar), "r"(x), "r"(y), "r"(z)
		: "memory");
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, uint32_t bar, int x, int y)
{
	asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(dst), "l"((uint64_t) map),
		     "r"(bar), "r"(x), "r"(y)
		     : "memory");
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
		     : "memory");
}

// 16-byte asynchronous copy global -> shared by this thread, L1 bypassed;
// src_bytes < 16 fills the rest with zeros (0: all zeros, src unread but a
// valid address).  Completion is per thread: commit groups, then wait.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, uint32_t src_bytes)
{
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// arrive on an mbarrier once every cp.async this thread has issued so far
// has landed (the barrier's expected count includes this arrival)
__device__ __forceinline__ void cp_async_arrive_noinc(uint32_t bar) { asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(bar) : "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// wait until at most N of this thread's committed groups are in flight
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// UMMA shared-memory descriptor, K-major, no swizzle: core matrices of
// 8 rows x 16 bytes; LBO = byte step between core matrices along K, SBO =
// byte step between 8-row groups; version field 1 (sm100).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
	uint64_t d = 0;
	d |= (uint64_t) ((saddr >> 4) & 0x3FFF);
	d |= (uint64_t) ((lbo >> 4) & 0x3FFF) << 16;
	d |= (uint64_t) ((sbo >> 4) & 0x3FFF) << 32;
	d |= (uint64_t) 1 << 46;
	return d;
}

// the same for a K-major operand in the 128-byte swizzled layout a TMA
// copy with CU_TENSOR_MAP_SWIZZLE_128B writes (rows of 64 bf16 = 128 B, 8-row
// groups 1024 B apart, the tile 1024-byte aligned): SBO 1024, LBO unused,
// swizzle mode 2; the K steps of 16 elements inside the 128-byte row advance
// the start address by 32 B
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr)
{
	uint64_t d = 0;
	d |= (uint64_t) ((saddr >> 4) & 0x3FFF);
	d |= (uint64_t) 1 << 16;
	d |= (uint64_t) (1024 >> 4) << 32;
	d |= (uint64_t) 1 << 46;
	d |= (uint64_t) 2 << 61;
	return d;
}

__device__ __forceinline__ void umma_bf16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate)
{
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"setp.ne.b32 p, %4, 0;\n\t"
		"tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
		"l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// the same MMA with the A operand in tensor memory (K-major: row m in lane
// m, bf16 elements k = 2c, 2c + 1 packed in column c, even k in the low half)
__device__ __forceinline__ void umma_bf16_tmem_a(uint32_t dtmem, uint32_t atmem, uint64_t bdesc, uint32_t idesc, uint32_t accumulate)
{
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"setp.ne.b32 p, %4, 0;\n\t"
		"tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(dtmem),
		"r"(atmem), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// two consecutive 32-bit columns of this thread's lane (warp w may store to
// lanes 32 (w % 4) .. 32 (w % 4) + 31 only)
__device__ __forceinline__ void tmem_st2(uint32_t taddr, uint32_t v0, uint32_t v1)
{
	asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(taddr), "r"(v0), "r"(v1) : "memory");
}

__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void umma_commit(uint32_t bar)
{
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t *v)
{
	asm volatile(
		"tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
		: "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]),
		  "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
		: "r"(taddr));
	asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ uint32_t pack_bf16(float lo_elem, float hi_elem)
{
	const __nv_bfloat16 a = __float2bfloat16_rn(lo_elem);
	const __nv_bfloat16 b = __float2bfloat16_rn(hi_elem);
	return (uint32_t) __bfloat16_as_ushort(a) | ((uint32_t) __bfloat16_as_ushort(b) << 16);
}


// TMEM allocation of ncols columns (a power of two >= 32) by one whole
// warp; the address lands in *slot (shared memory)
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols)
{
	asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols));
	asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}

__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols)
{
	asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

// instruction descriptor of tcgen05.mma kind::f16: FP32 accumulator, bf16
// A and B, both K-major, N x M tile
__host__ __device__ __forceinline__ uint32_t idesc_bf16(int M, int N)
{
	return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t) (N >> 3) << 17) | ((uint32_t) (M >> 4) << 24);
}

}  // namespace sphrad

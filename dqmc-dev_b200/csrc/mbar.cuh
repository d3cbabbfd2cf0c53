// mbarrier, TMA and timer helpers shared by the kernels that wait on
// asynchronous copies (the TMA-fed GEMM, the clustered update).  Every wait
// is bounded: after 1 s it sets an error bit and returns instead of spinning
// on, so that no kernel can hang the device on a copy that never lands.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace dq {

__device__ inline uint32_t smem_u32(const void *p)
{
	return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ inline void mbar_init(uint32_t a, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}

__device__ inline void mbar_arrive(uint32_t a)
{
	asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}"
	             ::"r"(a) : "memory");
}

__device__ inline void mbar_arrive_tx(uint32_t a, uint32_t tx)
{
	asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}"
	             ::"r"(a), "r"(tx) : "memory");
}

__device__ inline bool mbar_try_wait(uint32_t a, uint32_t parity)
{
	uint32_t ok;
	asm volatile("{\n\t.reg .pred p;\n\t"
	             "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
	             "selp.u32 %0, 1, 0, p;\n\t}"
	             : "=r"(ok) : "r"(a), "r"(parity) : "memory");
	return ok != 0;
}

__device__ inline uint64_t global_ns()
{
	uint64_t t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

// wait for phase `parity` of the mbarrier at `a` for at most 1 s; on
// timeout (or once another thread of the CTA has timed out) flag the error
// and return, so that no thread can wait forever
__device__ inline void mbar_wait_bounded(uint32_t a, uint32_t parity, volatile int *abort,
		unsigned *err)
{
	if (*abort) return;
	if (mbar_try_wait(a, parity)) return;
	const uint64_t t0 = global_ns();
	while (!mbar_try_wait(a, parity)) {
		if (*abort) return;
		if (global_ns() - t0 > 1000000000ull) {
			*abort = 1;
			if (err) atomicOr(err, DQ_ERR_TIMEOUT);
			return;
		}
	}
}

// tiled TMA loads of one box into this CTA's shared memory (no multicast),
// completing the box's bytes on the mbarrier at `mbar`; `tmap` is the
// address of a CUtensorMap in kernel-parameter or global memory
__device__ inline void tma_load_3d(uint32_t dst, const void *tmap, int x, int y, int z, uint32_t mbar)
{
	asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
	             " [%0], [%1, {%2, %3, %4}], [%5];"
	             ::"r"(dst), "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(mbar) : "memory");
}

__device__ inline void tma_load_4d(uint32_t dst, const void *tmap, int x, int y, int z, int w,
		uint32_t mbar)
{
	asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
	             " [%0], [%1, {%2, %3, %4, %5}], [%6];"
	             ::"r"(dst), "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(w), "r"(mbar) : "memory");
}

}  // namespace dq

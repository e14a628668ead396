// Bulk prefetch into L2 for the per-element table readers.
#pragma once

#include <cstdint>

namespace tfiga {

// Prefetches [p, p + bytes) into L2 with cp.async.bulk.prefetch (no shared memory, nothing to wait
// for); p 16-byte aligned, bytes a multiple of 16.  Issued in 16 KiB pieces by the calling thread.
__device__ __forceinline__ void PrefetchL2(const void* p, uint32_t bytes)
{
	const char* c = static_cast<const char*>(p);
	for (uint32_t off = 0; off < bytes; off += 16384u) {
		const uint32_t n = bytes-off < 16384u ? bytes-off : 16384u;
		asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" :: "l"(c+off), "r"(n) : "memory");
	}
}

} // namespace tfiga

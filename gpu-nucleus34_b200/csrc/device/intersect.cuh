// Warp-cooperative 3-way intersection of a triangle's three incidence lists.
//
// Reference: for_each_clique_of (nucleus/cuNucleus34_ondemand.cu:136-170) walks
// the three lists with one thread in a 3-way zipper, O(|L(a)|+|L(b)|+|L(c)|)
// dependent steps per triangle. Here the shortest list drives: each lane takes
// one entry x of it and binary-searches x in the other two lists; a ballot
// over the 32 lanes yields the common thirds of 32 driver entries per step.
// After each step the search windows of the other lists start at the position
// lane 31 reached (the driver is sorted, so later x are larger).
#pragma once

#include "common.cuh"

namespace n34 {

// f(found, x, pd, p1, p2) is called by ALL lanes once per 32-entry step (so it
// may use warp collectives); pd/p1/p2 are positions in third[]/tri[] of x in
// the driver list and the two other lists (valid only when found).
template <class F>
__device__ __forceinline__ void warp_intersect3(const uint32_t *__restrict__ third, uint64_t b0, uint64_t e0,
												uint64_t b1, uint64_t e1, uint64_t b2, uint64_t e2, F &&f)
{
	// pick the shortest list as the driver
	uint64_t bd = b0, ed = e0, lo1 = b1, hi1 = e1, lo2 = b2, hi2 = e2;
	if (e1 - b1 < ed - bd)
	{
		bd = b1;
		ed = e1;
		lo1 = b0;
		hi1 = e0;
	}
	if (e2 - b2 < ed - bd)
	{
		// driver becomes list 2; the previous driver moves into slot 2
		lo2 = bd;
		hi2 = ed;
		bd = b2;
		ed = e2;
	}
	const uint32_t lane = lane_id();
	for (uint64_t base = bd; base < ed; base += 32)
	{
		if (lo1 >= hi1 || lo2 >= hi2)
			break; // warp-uniform
		const uint64_t i = base + lane;
		const bool valid = i < ed;
		const uint32_t x = valid ? __ldg(third + i) : 0xffffffffu;
		uint64_t p1 = hi1, p2 = hi2;
		bool found = false;
		if (valid)
		{
			p1 = lower_bound_u32(third, lo1, hi1, x);
			p2 = lower_bound_u32(third, lo2, hi2, x);
			found = p1 < hi1 && __ldg(third + p1) == x && p2 < hi2 && __ldg(third + p2) == x;
		}
		f(found, x, i, p1, p2);
		lo1 = __shfl_sync(FULL, p1, 31);
		lo2 = __shfl_sync(FULL, p2, 31);
	}
}

} // namespace n34

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
// the driver list and the two other lists (valid only when found). Positions
// are 32-bit: the incidence holds 3T < 2^32 entries (checked by the driver).
template <class F>
__device__ __forceinline__ void warp_intersect3(const uint32_t *__restrict__ third, uint32_t b0, uint32_t e0,
												uint32_t b1, uint32_t e1, uint32_t b2, uint32_t e2, F &&f)
{
	// pick the shortest list as the driver
	uint32_t bd = b0, ed = e0, lo1 = b1, hi1 = e1, lo2 = b2, hi2 = e2;
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
	for (uint32_t base = bd; base < ed; base += 32)
	{
		if (lo1 >= hi1 || lo2 >= hi2)
			break; // warp-uniform
		const uint32_t i = base + lane;
		const bool valid = i < ed;
		const uint32_t x = valid ? __ldg(third + i) : 0xffffffffu;
		uint32_t p1 = hi1, p2 = hi2;
		bool found = false;
		if (valid)
		{
			p1 = lower_bound32(third, lo1, hi1, x);
			if (p1 < hi1 && __ldg(third + p1) == x)
			{
				p2 = lower_bound32(third, lo2, hi2, x);
				found = p2 < hi2 && __ldg(third + p2) == x;
			}
		}
		f(found, x, i, p1, p2);
		// later chunks hold larger x: the highest lane that searched a list
		// leaves a lower bound that stays valid for that list
		const uint32_t m1 = __ballot_sync(FULL, valid);
		const uint32_t m2 = __ballot_sync(FULL, valid && p1 < hi1 && __ldg(third + p1) == x);
		if (m1)
			lo1 = __shfl_sync(FULL, p1, 31 - __clz(m1));
		if (m2)
			lo2 = __shfl_sync(FULL, p2, 31 - __clz(m2));
	}
}

// The shortest of the three lists drives; the other two are searched.
struct Driver
{
	uint32_t bd, ed, lo1, hi1, lo2, hi2;
};

__device__ __forceinline__ Driver pick_driver(uint32_t b0, uint32_t e0, uint32_t b1, uint32_t e1, uint32_t b2,
											  uint32_t e2)
{
	Driver d{b0, e0, b1, e1, b2, e2};
	if (e1 - b1 < d.ed - d.bd)
	{
		d.bd = b1;
		d.ed = e1;
		d.lo1 = b0;
		d.hi1 = e0;
	}
	if (e2 - b2 < d.ed - d.bd)
	{
		d.lo2 = d.bd;
		d.hi2 = d.ed;
		d.bd = b2;
		d.ed = e2;
	}
	return d;
}

// Driver length up to which one lane handles a triangle on its own (the
// lanes of a warp then work on 32 different triangles at once).
constexpr uint32_t THREAD_MODE_MAX = 16;

// Thread-local 3-way intersection for a short driver list: f(x, pd, p1, p2)
// per common third. Windows only move forward because the driver is sorted.
template <class F>
__device__ __forceinline__ void thread_intersect3(const uint32_t *__restrict__ third, Driver d, F &&f)
{
	for (uint32_t i = d.bd; i < d.ed && d.lo1 < d.hi1 && d.lo2 < d.hi2; ++i)
	{
		const uint32_t x = __ldg(third + i);
		d.lo1 = lower_bound32(third, d.lo1, d.hi1, x);
		if (d.lo1 >= d.hi1)
			break;
		if (__ldg(third + d.lo1) != x)
			continue;
		d.lo2 = lower_bound32(third, d.lo2, d.hi2, x);
		if (d.lo2 >= d.hi2)
			break;
		if (__ldg(third + d.lo2) != x)
			continue;
		f(x, i, d.lo1, d.lo2);
	}
}

} // namespace n34

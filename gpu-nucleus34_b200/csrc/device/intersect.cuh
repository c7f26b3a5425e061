// Intersection of a triangle's incidence lists.
//
// Reference: for_each_clique_of (nucleus/cuNucleus34_ondemand.cu:136-170) walks
// the three lists of triangle t=(u,v,w) in one thread with a 3-way zipper,
// O(|L(a)|+|L(b)|+|L(c)|) dependent steps.
//
// Two facts shape the device version:
//  1. Any two of the three lists suffice to find the cliques: x in L(u,w) and
//     in L(u,v) is adjacent to u, v and w, so {u,v,w,x} is a four-clique and x
//     is in L(v,w) as well. The common thirds of the two SHORTEST lists are
//     exactly t's cliques; the longest list is only searched, for a found x,
//     when the partner triangle on that edge is needed.
//  2. On skewed graphs the two shortest lists are usually of similar length,
//     so a merge beats per-entry binary searches. One warp merges 32 + 32
//     entries per step with coalesced loads: each lane locates its A entry in
//     the B tile held in registers by a 5-step shuffle search, and the tile
//     whose last entry is smaller is consumed. When B is far longer than A,
//     the lanes binary-search B instead; short A lists are handled by a single
//     lane (see THREAD_MODE_MAX).
#pragma once

#include "common.cuh"

namespace n34 {

// A triangle's three lists as [begin, end) positions in third[] / tri[],
// ordered by length: A shortest, B middle, C longest. Positions are 32-bit:
// the incidence holds 3T < 2^32 entries (checked before it is built).
struct Lists
{
	uint32_t a0, a1, b0, b1, c0, c1;
};

__device__ __forceinline__ Lists order_lists(uint32_t x0, uint32_t x1, uint32_t y0, uint32_t y1, uint32_t z0,
											 uint32_t z1)
{
	// sort three (begin, end) pairs by length
	uint32_t p0 = x0, p1 = x1, q0 = y0, q1 = y1, r0 = z0, r1 = z1, t;
	if (q1 - q0 < p1 - p0)
	{
		t = p0; p0 = q0; q0 = t;
		t = p1; p1 = q1; q1 = t;
	}
	if (r1 - r0 < q1 - q0)
	{
		t = q0; q0 = r0; r0 = t;
		t = q1; q1 = r1; r1 = t;
	}
	if (q1 - q0 < p1 - p0)
	{
		t = p0; p0 = q0; q0 = t;
		t = p1; p1 = q1; q1 = t;
	}
	return Lists{p0, p1, q0, q1, r0, r1};
}

// Shortest-list length up to which one lane handles a triangle on its own
// (the default; the on-demand variant's scheduling settings instantiate the
// support count and the peel debit with 8, 16 or 32).
constexpr uint32_t THREAD_MODE_MAX = 16;
// B longer than this multiple of A: binary-search B instead of merging.
constexpr uint32_t MERGE_RATIO = 24;
// Search ranges at least this long start with a warp-wide sample of 32
// evenly spaced entries (one round trip instead of five halvings).
#ifndef N34_SAMPLE_MIN
#define N34_SAMPLE_MIN 256u
#endif

// Loads of the incidence's triangle words (which carry the death flags).
// Kernels that only read them during their run use the read-only path; a
// kernel that also writes flags in an earlier phase of the same launch (the
// cooperative small-round peel) must read them through L2.
template <bool COHERENT>
__device__ __forceinline__ uint32_t ld_tri(const uint32_t *p)
{
	if (COHERENT)
		return __ldcg(p);
	return __ldg(p);
}

__device__ __forceinline__ bool use_merge(const Lists &L)
{
	return (L.b1 - L.b0) <= MERGE_RATIO * (L.a1 - L.a0);
}

// L2 prefetch of a list range by the bulk-copy engine (one instruction per
// 64 KB, issued by one lane): later tile loads of a long list then hit L2
// instead of DRAM. The range is widened to 16-byte boundaries, which stay
// inside the array because allocations are 256-byte aligned and padded.
#ifndef N34_L2_PREFETCH_MIN
#define N34_L2_PREFETCH_MIN 64u
#endif
__device__ __forceinline__ void prefetch_range_l2(const uint32_t *base, uint32_t lo, uint32_t hi)
{
	if (hi - lo < N34_L2_PREFETCH_MIN)
		return;
	uintptr_t a = reinterpret_cast<uintptr_t>(base + lo) & ~uintptr_t(15);
	const uintptr_t e = (reinterpret_cast<uintptr_t>(base + hi) + 15) & ~uintptr_t(15);
	while (a < e)
	{
		const uint32_t n = uint32_t((e - a) > 65536 ? 65536 : (e - a));
		asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"(n) : "memory");
		a += n;
	}
}

// Warp lower bounds: every lane with want gets the first position in [lo, hi)
// whose entry is >= its x (hi if none). Long ranges are first narrowed to
// 1/32 by a sample of 32 evenly spaced entries loaded at once, so the
// per-lane binary searches start five levels down. A sample of a list can be
// taken once and reused while the searched range only moves forward.
struct WarpSample
{
	uint32_t sp; // sample position of this lane (end of slice lane)
	uint32_t sv; // entry there
	bool on;     // range long enough to be sampled (warp-uniform)
};

__device__ __forceinline__ WarpSample warp_sample(const uint32_t *__restrict__ a, uint32_t lo, uint32_t hi)
{
	WarpSample s{0u, 0u, (hi - lo) >= N34_SAMPLE_MIN};
	if (s.on)
	{
		const uint32_t n = hi - lo;
		// sample i sits at the end of slice i: lo + ceil(n * (i+1) / 32) - 1
		s.sp = lo + uint32_t((uint64_t(n) * (lane_id() + 1) + 31) >> 5) - 1;
		s.sv = __ldg(a + s.sp);
	}
	return s;
}

// Lower bounds in [lo, hi) using a sample taken over [lo0, hi) with lo0 <= lo
// (every entry before lo is below every x searched now). Called by all lanes.
__device__ __forceinline__ uint32_t sampled_lower_bound(const uint32_t *__restrict__ a, const WarpSample &s,
														uint32_t lo, uint32_t hi, bool want, uint32_t x)
{
	uint32_t l = lo, h = hi;
	if (s.on) // warp-uniform
	{
		// first sample >= x (31 if none)
		uint32_t j = 0;
#pragma unroll
		for (uint32_t step = 16; step > 0; step >>= 1)
		{
			const uint32_t probe = __shfl_sync(FULL, s.sv, (j + step - 1) & 31);
			if (probe < x)
				j += step;
		}
		const uint32_t last = __shfl_sync(FULL, s.sv, 31);
		const uint32_t sj = __shfl_sync(FULL, s.sp, j & 31);
		const uint32_t sprev = __shfl_sync(FULL, s.sp, (j + 31) & 31);
		if (last < x)
		{
			l = hi;
			h = hi;
		}
		else
		{
			const uint32_t from = j ? sprev + 1 : lo;
			l = from > lo ? from : lo;
			h = sj; // a[sj] >= x: the bound is at most sj (and at least lo)
		}
	}
	uint32_t r = hi;
	if (want)
		r = lower_bound32(a, l, h, x);
	return r;
}

__device__ __forceinline__ uint32_t warp_lower_bound(const uint32_t *__restrict__ a, uint32_t lo, uint32_t hi,
													 bool want, uint32_t x)
{
	return sampled_lower_bound(a, warp_sample(a, lo, hi), lo, hi, want, x);
}

// Warp tile merge of A and B. f(found, x, pa, pb, qa, qb) is called by all
// lanes once per step; found lanes hold x = third[pa] = third[pb], and with
// WITH_TRI also qa = itri[pa], qb = itri[pb] (the partner tiles are loaded
// together with the third tiles, saving a dependent round trip). Each common
// x is seen exactly once, in ascending order across steps.
template <bool WITH_TRI, class F, bool COH = false>
__device__ __forceinline__ void warp_merge2(const uint32_t *__restrict__ third, const uint32_t *__restrict__ itri,
											uint32_t a0, uint32_t a1, uint32_t b0, uint32_t b1, F &&f)
{
	const uint32_t lane = lane_id();
	while (a0 < a1 && b0 < b1) // warp-uniform
	{
		const uint32_t ai = a0 + lane, bi = b0 + lane;
		const bool av_ok = ai < a1, bv_ok = bi < b1;
		const uint32_t av = av_ok ? __ldg(third + ai) : 0xffffffffu;
		const uint32_t bv = bv_ok ? __ldg(third + bi) : 0xffffffffu;
		uint32_t at = 0, bt = 0;
		if (WITH_TRI)
		{
			at = av_ok ? ld_tri<COH>(itri + ai) : 0u;
			bt = bv_ok ? ld_tri<COH>(itri + bi) : 0u;
		}
		const uint32_t amax = __shfl_sync(FULL, av, 31), bmax = __shfl_sync(FULL, bv, 31);
		const uint32_t m = amax < bmax ? amax : bmax;
		// first lane j of the B tile with bv_j >= av (31 if none: then no match)
		uint32_t pos = 0;
#pragma unroll
		for (uint32_t step = 16; step > 0; step >>= 1)
		{
			const uint32_t probe = __shfl_sync(FULL, bv, (pos + step - 1) & 31);
			if (probe < av)
				pos += step;
		}
		const uint32_t hitv = __shfl_sync(FULL, bv, pos & 31);
		const uint32_t qb = WITH_TRI ? __shfl_sync(FULL, bt, pos & 31) : 0u;
		const bool found = av_ok && av <= m && hitv == av && b0 + pos < b1;
		f(found, av, ai, b0 + pos, at, qb);
		// everything <= m is consumed; at least one tile is used up entirely
		a0 += __popc(__ballot_sync(FULL, av_ok && av <= m));
		b0 += __popc(__ballot_sync(FULL, bv_ok && bv <= m));
	}
}

// Warp binary search of A's entries in B (B much longer than A).
template <bool WITH_TRI, class F, bool COH = false>
__device__ __forceinline__ void warp_search2(const uint32_t *__restrict__ third, const uint32_t *__restrict__ itri,
											 uint32_t a0, uint32_t a1, uint32_t b0, uint32_t b1, F &&f)
{
	const uint32_t lane = lane_id();
	for (uint32_t base = a0; base < a1; base += 32)
	{
		if (b0 >= b1)
			break; // warp-uniform
		const uint32_t ai = base + lane;
		const bool ok = ai < a1;
		const uint32_t x = ok ? __ldg(third + ai) : 0xffffffffu;
		const uint32_t at = (WITH_TRI && ok) ? ld_tri<COH>(itri + ai) : 0u;
		const uint32_t p = warp_lower_bound(third, b0, b1, ok, x);
		const bool found = ok && p < b1 && __ldg(third + p) == x;
		const uint32_t bt = (WITH_TRI && found) ? ld_tri<COH>(itri + p) : 0u;
		f(found, x, ai, p, at, bt);
		// later steps hold larger x: the highest searching lane's bound stays valid
		const uint32_t msk = __ballot_sync(FULL, ok);
		b0 = __shfl_sync(FULL, p, 31 - __clz(msk));
	}
}

// Warp dispatch between merge and search for the two shortest lists.
template <bool WITH_TRI = false, bool COH = false, class F>
__device__ __forceinline__ void warp_intersect2(const uint32_t *__restrict__ third, const uint32_t *__restrict__ itri,
												const Lists &L, F &&f)
{
	if (use_merge(L))
		warp_merge2<WITH_TRI, F &, COH>(third, itri, L.a0, L.a1, L.b0, L.b1, f);
	else
		warp_search2<WITH_TRI, F &, COH>(third, itri, L.a0, L.a1, L.b0, L.b1, f);
}

// One lane on its own: each entry of A binary-searched in B (the window only
// moves forward). f(x, pa, pb) per common x, ascending.
template <class F>
__device__ __forceinline__ void lane_intersect2(const uint32_t *__restrict__ third, const Lists &L, F &&f)
{
	uint32_t lo = L.b0;
	for (uint32_t i = L.a0; i < L.a1 && lo < L.b1; ++i)
	{
		const uint32_t x = __ldg(third + i);
		lo = lower_bound32(third, lo, L.b1, x);
		if (lo < L.b1 && __ldg(third + lo) == x)
			f(x, i, lo);
	}
}

} // namespace n34

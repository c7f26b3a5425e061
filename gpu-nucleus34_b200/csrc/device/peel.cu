// Device-resident, level-synchronous bucketed peel of triangle support.
//
// Reference: the direct program launches peel_fourcliques over ALL triangles
// once per level with a host round trip each (nucleus/cuNucleus34.cu:107-141,
// 675-714; claim flags per clique), the on-demand program runs
// min_alive_support / mark_dying / debit_partners with three device->host
// copies and two syncs per round (cuNucleus34_ondemand.cu:203-305, 599-682);
// the CPU form is bucket_ex::peeling_par (nucleus/bucket_ex.hpp:274-360).
// All produce the unique (3,4)-nucleus number of each triangle.
//
// Here a round is a fixed sequence of kernels that read their work sizes from
// a device control block, so the host only launches batches of rounds and
// reads one flag per batch:
//   scan_min / gather  (only when the frontier is empty): next level = min
//                      alive support; frontier = alive triangles at it.
//   mark               K[t] = level, R[t] = round for the frontier.
//   debit              each dying triangle enumerates its cliques (on-demand:
//                      3-way intersection of its incidence lists; direct: its
//                      clique ids); the clique belongs to its first member to
//                      die, ties to the lowest id (the death-stamp rule of
//                      debit_partners, cuNucleus34_ondemand.cu:237-276); the
//                      owner debits every alive partner with atomicSub. A
//                      partner whose support falls from level+1 to level is
//                      appended to the next frontier (exactly once).
//   advance            swap frontiers, advance the round.
// The result is independent of thread timing: ownership depends only on the
// stamps, and crossing detection catches every triangle that reaches the level.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "intersect.cuh"
#include "pipeline.cuh"

namespace n34 {

namespace {

constexpr uint32_t INF = 0xffffffffu;
constexpr int PEEL_THREADS = 256;
// The device loop stops a peel that has run this long (device time) and the
// call returns NUCLEUS34_E_TIMEOUT: a bound on a loop that would otherwise
// only end by the round bound. R-MAT scale 20 peels in about 2 s.
constexpr unsigned long long PEEL_TIME_LIMIT_NS = 600ull * 1000000000ull;

struct CtlX
{
	PeelCtl c;
	uint32_t scan;        // 1 while the next frontier must come from a scan
	uint32_t next_found;  // k_scan_min's snapshot: k_gather_next found a frontier
	uint32_t compact_now; // set by k_compact_gate for the replay's compaction
	uint32_t compact_div; // compaction gate divisor (0: never compact)
	unsigned long long sort_min; // frontiers at least this large are put in id order
	unsigned long long peeled_at_compact;
	unsigned long long live_at_compact;
	uint32_t compactions;
	unsigned long long t0_ns; // %globaltimer at the peel's start (device-loop time bound)
	uint32_t timed_out;       // the device loop stopped at its round or time bound
	uint32_t small_rounds;    // rounds run inside k_small_rounds
	uint32_t loop_passes;     // passes of the device loop's body
	// profiling counters of k_debit_flags_warp (filled only when stats is set)
	uint32_t stats;
	unsigned long long st_tri, st_merge_entries, st_steps, st_lookups, st_resolves, st_staged, st_found;
	uint32_t cursor; // next unclaimed frontier position / bitmap word (warp debit with a cursor)
};

// A frontier is a list F[0, nF) (default) or, in the memory-lean peel, a
// bitmap of T bits (one u32 word per 32 triangles; no list at all). Two of
// each alternate between the current and the next round.
struct Frontier
{
	uint32_t *F0, *F1; // lists (null in bitmap mode)
	uint32_t *B0, *B1; // bitmaps (null in list mode)
	uint64_t W;        // bitmap words
	__device__ __forceinline__ bool bits() const { return B0 != nullptr; }
	__device__ __forceinline__ uint32_t *cur_list(uint32_t cur) const { return cur ? F1 : F0; }
	__device__ __forceinline__ uint32_t *next_list(uint32_t cur) const { return cur ? F0 : F1; }
	__device__ __forceinline__ uint32_t *cur_bits(uint32_t cur) const { return cur ? B1 : B0; }
	__device__ __forceinline__ uint32_t *next_bits(uint32_t cur) const { return cur ? B0 : B1; }
};

// f(t) for every triangle of the current frontier, grid-stride over threads;
// in bitmap mode one thread takes one word, and with clear it zeroes the
// word afterwards (the last kernel of a round frees the bitmap for reuse).
template <class Fn>
__device__ __forceinline__ void frontier_each_thread(const Frontier fr, uint32_t cur, uint32_t nF, bool clear,
													 Fn &&f)
{
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	const uint64_t tid = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
	if (fr.bits())
	{
		uint32_t *B = fr.cur_bits(cur);
		for (uint64_t w = tid; w < fr.W; w += stride)
		{
			uint32_t word = B[w];
			if (!word)
				continue;
			if (clear)
				B[w] = 0;
			while (word)
			{
				const uint32_t b = __ffs(word) - 1;
				word &= word - 1;
				f(uint32_t(w * 32 + b));
			}
		}
	}
	else
	{
		const uint32_t *F = fr.cur_list(cur);
		for (uint64_t i = tid; i < nF; i += stride)
			f(F[i]);
	}
}

// K null: k is kept in S (a dead triangle holds -1 - k there), as in the
// memory-lean peel; otherwise every k starts at -1 (not peeled).
__global__ void k_peel_init(int32_t *__restrict__ K, uint64_t T, CtlX *ctl, uint32_t compact_div,
							unsigned long long sort_min)
{
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	if (K)
		for (uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < T; t += stride)
			K[t] = -1;
	if (blockIdx.x == 0 && threadIdx.x == 0)
	{
		PeelCtl z{};
		z.minS = INF;
		z.level = 0xffffffffu; // "-1": the first level change tries level 0
		ctl->c = z;
		ctl->scan = 1;
		ctl->next_found = 0;
		ctl->compact_now = 0;
		ctl->compact_div = compact_div;
		ctl->sort_min = sort_min;
		ctl->cursor = 0;
		ctl->peeled_at_compact = 0;
		ctl->live_at_compact = T;
		unsigned long long now;
		asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
		ctl->t0_ns = now;
		ctl->timed_out = 0;
		ctl->small_rounds = 0;
		ctl->loop_passes = 0;
		ctl->compactions = 0;
		ctl->st_tri = ctl->st_merge_entries = ctl->st_steps = ctl->st_lookups = 0;
		ctl->st_resolves = ctl->st_staged = ctl->st_found = 0;
	}
}

// Level change (frontier empty): every alive triangle has S > level, and dead
// ones hold S = INT_MAX. First try the next level directly (the usual case);
// only if nothing sits at level+1 compute the minimum and gather at it.
// Dead triangles hold S = -1 - k < 0; live supports are never negative.
__device__ __forceinline__ void gather_take(const Frontier fr, CtlX *ctl, bool take, uint64_t t, uint64_t T)
{
	const uint32_t slot = warp_append(take, &ctl->c.nF);
	if (take)
	{
		if (fr.bits())
			atomicOr(fr.cur_bits(ctl->c.cur) + (t >> 5), 1u << (t & 31));
		else if (slot < T)
			fr.cur_list(ctl->c.cur)[slot] = uint32_t(t);
		else
			atomicOr(&ctl->c.error, 1u);
	}
}

// Level-change scans. With vec (the default) each thread reads eight
// consecutive supports per step as two aligned 16-byte loads, so that a warp
// keeps 1 KB in flight instead of 128 bytes, and a warp appends its step's
// takes with one atomic on the frontier counter (a warp scan of the lanes'
// counts) instead of one ballot and atomic per 32 supports. Without vec:
// one support per thread per step (kept for comparison,
// NUCLEUS34_OPT_SCALAR_SCANS).
constexpr uint32_t SCAN_VEC = 8;

// v[j] = S[t0 + j] for t0 + j < T, else -1 (never taken); t0 is a multiple of
// 8 and S is 256-byte aligned, so the vector loads are aligned.
__device__ __forceinline__ void load_supports8(const int32_t *__restrict__ S, uint64_t T, uint64_t t0, int32_t v[8])
{
	if (t0 + SCAN_VEC <= T)
	{
		const int4 a = __ldg(reinterpret_cast<const int4 *>(S + t0));
		const int4 b = __ldg(reinterpret_cast<const int4 *>(S + t0 + 4));
		v[0] = a.x;
		v[1] = a.y;
		v[2] = a.z;
		v[3] = a.w;
		v[4] = b.x;
		v[5] = b.y;
		v[6] = b.z;
		v[7] = b.w;
	}
	else
	{
#pragma unroll
		for (uint32_t j = 0; j < SCAN_VEC; ++j)
			v[j] = t0 + j < T ? S[t0 + j] : -1;
	}
}

// Appends every t whose support is in [0, hi] (all threads of the grid call).
__device__ __forceinline__ void gather_range8(const Frontier fr, CtlX *ctl, const int32_t *__restrict__ S,
											  uint64_t T, uint32_t hi)
{
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x * SCAN_VEC;
	const uint32_t lane = lane_id();
	for (uint64_t b0 = uint64_t(blockIdx.x) * blockDim.x * SCAN_VEC; b0 < T; b0 += stride)
	{
		const uint64_t t0 = b0 + uint64_t(threadIdx.x) * SCAN_VEC;
		int32_t v[SCAN_VEC];
		load_supports8(S, T, t0, v);
		uint32_t mask = 0;
#pragma unroll
		for (uint32_t j = 0; j < SCAN_VEC; ++j)
			if (v[j] >= 0 && uint32_t(v[j]) <= hi)
				mask |= 1u << j;
		const uint32_t cnt = __popc(mask);
		uint32_t x = cnt; // inclusive warp scan of the counts
#pragma unroll
		for (uint32_t o = 1; o < 32; o <<= 1)
		{
			const uint32_t y = __shfl_up_sync(FULL, x, o);
			if (lane >= o)
				x += y;
		}
		const uint32_t total = __shfl_sync(FULL, x, 31);
		if (total == 0)
			continue; // warp-uniform: b0 is the same for the whole block
		uint32_t base = 0;
		if (lane == 31)
			base = atomicAdd(&ctl->c.nF, total);
		base = __shfl_sync(FULL, base, 31);
		uint32_t pos = base + x - cnt;
		while (mask)
		{
			const uint32_t j = __ffs(mask) - 1;
			mask &= mask - 1;
			const uint64_t t = t0 + j;
			if (fr.bits())
				atomicOr(fr.cur_bits(ctl->c.cur) + (t >> 5), 1u << (t & 31));
			else if (pos < T)
				fr.cur_list(ctl->c.cur)[pos] = uint32_t(t);
			else
				atomicOr(&ctl->c.error, 1u);
			++pos;
		}
	}
}

__global__ void __launch_bounds__(PEEL_THREADS) k_gather_next(CtlX *ctl, const int32_t *__restrict__ S, uint64_t T,
															  Frontier fr, bool vec)
{
	if (ctl->c.done || !ctl->scan)
		return;
	const int32_t want = int32_t(ctl->c.level) + 1;
	if (vec)
	{
		gather_range8(fr, ctl, S, T, uint32_t(want));
		return;
	}
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t t0 = uint64_t(blockIdx.x) * blockDim.x; t0 < T; t0 += stride)
	{
		const uint64_t t = t0 + threadIdx.x;
		bool take = false;
		if (t < T)
		{
			const int32_t s = S[t];
			take = s >= 0 && s <= want;
		}
		gather_take(fr, ctl, take, t, T);
	}
}

__global__ void __launch_bounds__(PEEL_THREADS) k_scan_min(CtlX *ctl, const int32_t *__restrict__ S, uint64_t T,
														   bool vec)
{
	if (ctl->c.done || !ctl->scan)
		return;
	// nF is final here (k_gather_next has finished); k_gather, which appends
	// to nF itself, decides from this snapshot instead of reading nF
	const uint32_t nf = ctl->c.nF;
	if (blockIdx.x == 0 && threadIdx.x == 0)
		ctl->next_found = nf != 0;
	if (nf)
		return;
	uint32_t mn = INF;
	if (vec)
	{
		const uint64_t vstride = uint64_t(gridDim.x) * blockDim.x * SCAN_VEC;
		for (uint64_t t0 = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) * SCAN_VEC; t0 < T; t0 += vstride)
		{
			int32_t v[SCAN_VEC];
			load_supports8(S, T, t0, v);
#pragma unroll
			for (uint32_t j = 0; j < SCAN_VEC; ++j)
				if (v[j] >= 0)
					mn = min(mn, uint32_t(v[j]));
		}
	}
	else
	{
		const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
		for (uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < T; t += stride)
		{
			const int32_t s = S[t];
			if (s >= 0)
				mn = min(mn, uint32_t(s));
		}
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		mn = min(mn, __shfl_xor_sync(FULL, mn, o));
	if (lane_id() == 0 && mn != INF)
		atomicMin(&ctl->c.minS, mn);
}

// Second chance of the level change: gather at the minimum (or finish).
__global__ void __launch_bounds__(PEEL_THREADS) k_gather(CtlX *ctl, const int32_t *__restrict__ S, uint64_t T,
														 Frontier fr, bool vec)
{
	if (ctl->c.done || !ctl->scan)
		return;
	if (ctl->next_found)
	{ // k_gather_next found the frontier at level+1
		if (blockIdx.x == 0 && threadIdx.x == 0)
			ctl->c.level = ctl->c.level + 1;
		return;
	}
	const uint32_t mn = ctl->c.minS;
	if (mn == INF)
	{
		if (blockIdx.x == 0 && threadIdx.x == 0)
			ctl->c.done = 1;
		return;
	}
	// every alive triangle sits above the old level, so the minimum is the new one
	if (blockIdx.x == 0 && threadIdx.x == 0)
		ctl->c.level = mn;
	if (vec)
	{
		gather_range8(fr, ctl, S, T, mn);
		return;
	}
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t t0 = uint64_t(blockIdx.x) * blockDim.x; t0 < T; t0 += stride)
	{
		const uint64_t t = t0 + threadIdx.x;
		bool take = false;
		if (t < T)
		{
			const int32_t s = S[t];
			take = s >= 0 && uint32_t(s) <= mn;
		}
		gather_take(fr, ctl, take, t, T);
	}
}

__global__ void k_mark(CtlX *ctl, const uint32_t *__restrict__ F0, const uint32_t *__restrict__ F1,
					   int32_t *__restrict__ K, uint32_t *__restrict__ R, int32_t *__restrict__ S)
{
	if (ctl->c.done)
		return;
	const uint32_t nF = ctl->c.nF;
	const uint32_t *F = ctl->c.cur ? F1 : F0;
	const int32_t level = int32_t(ctl->c.level);
	const uint32_t round = ctl->c.round;
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nF; i += stride)
	{
		const uint32_t t = F[i];
		K[t] = level;
		R[t] = round;
		S[t] = -1 - level; // dead: out of every later scan (dead triangles are never debited)
	}
}

// Ownership + debit of one clique seen by dying triangle t (all lanes call).
__device__ __forceinline__ void settle_clique(bool found, uint32_t t, uint32_t p0, uint32_t p1, uint32_t p2,
											  const int32_t *__restrict__ K, const uint32_t *__restrict__ R,
											  int32_t *__restrict__ S, uint32_t round, int32_t level,
											  uint32_t *__restrict__ Fn, uint32_t *nNext, uint64_t cap,
											  uint32_t *err)
{
	bool owner = found;
	bool alive0 = false, alive1 = false, alive2 = false;
	if (found)
	{
		const uint32_t p[3] = {p0, p1, p2};
		bool al[3];
#pragma unroll
		for (int s = 0; s < 3; ++s)
		{
			const int32_t k = K[p[s]];
			al[s] = k == -1;
			if (!al[s])
			{
				const uint32_t r = R[p[s]];
				if (r < round || p[s] < t)
					owner = false;
			}
		}
		alive0 = owner && al[0];
		alive1 = owner && al[1];
		alive2 = owner && al[2];
	}
	bool hit0 = false, hit1 = false, hit2 = false;
	if (alive0)
		hit0 = atomicSub(S + p0, 1) == level + 1;
	if (alive1)
		hit1 = atomicSub(S + p1, 1) == level + 1;
	if (alive2)
		hit2 = atomicSub(S + p2, 1) == level + 1;
	// capacity guard: a triangle reaches the frontier at most once, so T slots suffice
	uint32_t slot = warp_append(hit0, nNext);
	if (hit0)
	{
		if (slot < cap)
			Fn[slot] = p0;
		else
			atomicOr(err, 1u);
	}
	slot = warp_append(hit1, nNext);
	if (hit1)
	{
		if (slot < cap)
			Fn[slot] = p1;
		else
			atomicOr(err, 1u);
	}
	slot = warp_append(hit2, nNext);
	if (hit2)
	{
		if (slot < cap)
			Fn[slot] = p2;
		else
			atomicOr(err, 1u);
	}
}

__device__ __forceinline__ Lists frontier_lists(uint32_t t, const uint32_t *__restrict__ tris,
											   const uint2 *__restrict__ span)
{
	const uint32_t ea = __ldg(tris + 3 * uint64_t(t)), eb = __ldg(tris + 3 * uint64_t(t) + 1),
				   ec = __ldg(tris + 3 * uint64_t(t) + 2);
	const uint2 sa = __ldg(span + ea), sb = __ldg(span + eb), sc = __ldg(span + ec);
	return order_lists(sa.x, sa.y, sb.x, sb.y, sc.x, sc.y);
}

// On-demand debit with the round-stamp owner test (used when triangle ids do
// not leave room for flag bits): one warp per dying triangle; the partner on
// the longest list is found by a forward-moving binary search.
__global__ void __launch_bounds__(PEEL_THREADS) k_debit_ondemand(
	CtlX *ctl, uint32_t *__restrict__ F0, uint32_t *__restrict__ F1, const uint32_t *__restrict__ tris,
	const uint2 *__restrict__ span, const uint32_t *__restrict__ third, const uint32_t *__restrict__ itri,
	const int32_t *__restrict__ K, const uint32_t *__restrict__ R, int32_t *__restrict__ S, uint64_t T)
{
	if (ctl->c.done)
		return;
	const uint32_t nF = ctl->c.nF;
	const uint32_t *F = ctl->c.cur ? F1 : F0;
	uint32_t *Fn = ctl->c.cur ? F0 : F1;
	const int32_t level = int32_t(ctl->c.level);
	const uint32_t round = ctl->c.round;
	const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
	for (uint64_t i = warp; i < nF; i += nwarps)
	{
		const uint32_t t = F[i];
		const Lists L = frontier_lists(t, tris, span);
		uint32_t lo_c = L.c0;
		warp_intersect2<true>(third, itri, L, [&](bool found, uint32_t x, uint32_t, uint32_t, uint32_t qa,
												  uint32_t qb) {
			const uint32_t fm = __ballot_sync(FULL, found);
			if (!fm)
				return;
			const uint32_t pc = warp_lower_bound(third, lo_c, L.c1, found, x);
			lo_c = __shfl_sync(FULL, pc, 31 - __clz(fm));
			found = found && pc < L.c1; // always true without compaction
			uint32_t q0 = 0, q1 = 0, q2 = 0;
			if (found)
			{
				q0 = qa;
				q1 = qb;
				q2 = __ldg(itri + pc);
			}
			settle_clique(found, t, q0, q1, q2, K, R, S, round, level, Fn, &ctl->c.nNext, T, &ctl->c.error);
		});
	}
}

// Direct variant: a dying triangle walks its clique ids. A clique destroyed in
// an earlier round carries a set byte in `destroyed` (written by its owner), so
// later members skip it with one byte load; otherwise the members are read and
// the round-stamp owner rule decides.
__global__ void __launch_bounds__(PEEL_THREADS) k_debit_direct(
	CtlX *ctl, uint32_t *__restrict__ F0, uint32_t *__restrict__ F1, const uint64_t *__restrict__ coff,
	const uint32_t *__restrict__ cids, const uint4 *__restrict__ quds, const int32_t *__restrict__ K,
	const uint32_t *__restrict__ R, int32_t *__restrict__ S, uint8_t *__restrict__ destroyed, uint64_t T)
{
	if (ctl->c.done)
		return;
	const uint32_t nF = ctl->c.nF;
	const uint32_t *F = ctl->c.cur ? F1 : F0;
	uint32_t *Fn = ctl->c.cur ? F0 : F1;
	const int32_t level = int32_t(ctl->c.level);
	const uint32_t round = ctl->c.round;
	const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
	for (uint64_t i = warp; i < nF; i += nwarps)
	{
		const uint32_t t = F[i];
		const uint64_t b = coff[t], e = coff[t + 1];
		for (uint64_t base = b; base < e; base += 32)
		{
			const uint64_t j = base + lane_id();
			bool live = false;
			uint32_t q = 0, q0 = 0, q1 = 0, q2 = 0;
			if (j < e)
			{
				q = cids[j];
				live = !destroyed[q];
			}
			if (live)
			{
				const uint4 x = quds[q];
				// the three members other than t
				const uint32_t m[4] = {x.x, x.y, x.z, x.w};
				uint32_t o[3] = {0, 0, 0};
				int k = 0;
#pragma unroll
				for (int s = 0; s < 4; ++s)
					if (m[s] != t && k < 3)
						o[k++] = m[s];
				q0 = o[0];
				q1 = o[1];
				q2 = o[2];
			}
			bool owner = live;
			bool al[3] = {false, false, false};
			if (live)
			{
				const uint32_t p[3] = {q0, q1, q2};
#pragma unroll
				for (int s = 0; s < 3; ++s)
				{
					al[s] = K[p[s]] == -1;
					if (!al[s] && (R[p[s]] < round || p[s] < t))
						owner = false;
				}
			}
			bool hit[3] = {false, false, false};
			if (owner)
			{
				destroyed[q] = 1;
				if (al[0])
					hit[0] = atomicSub(S + q0, 1) == level + 1;
				if (al[1])
					hit[1] = atomicSub(S + q1, 1) == level + 1;
				if (al[2])
					hit[2] = atomicSub(S + q2, 1) == level + 1;
			}
			const uint32_t qs[3] = {q0, q1, q2};
#pragma unroll
			for (int r = 0; r < 3; ++r)
			{
				const uint32_t slot = warp_append(hit[r], &ctl->c.nNext);
				if (hit[r])
				{
					if (slot < T)
						Fn[slot] = qs[r];
					else
						atomicOr(&ctl->c.error, 1u);
				}
			}
		}
	}
}

// ---- on-demand peel with death flags kept in the incidence entries ----------
//
// Each triangle owns one entry in each of its three edges' lists; bit 31 of the
// entry's triangle id means "died in an earlier round", bit 30 "dies in this
// round". The owner rule then reads nothing but the three entries the 3-way
// intersection already located, and a dead driver entry skips its searches.
constexpr uint32_t DEAD = INC_DEAD;
constexpr uint32_t DYING = 0x40000000u;
constexpr uint32_t ID_MASK = 0x3fffffffu;
static_assert(ID_MASK == FLAG_PEEL_MAX_TRIANGLES, "death-flag id range");

// positions of triangle t's three entries: under b (third w), a (third v), c (third u);
// read from tpos when the incidence keeps them, else searched
__device__ __forceinline__ void entry_positions(uint32_t t, const uint32_t *__restrict__ tris,
												const uint32_t *__restrict__ src, const uint32_t *__restrict__ E,
												const uint2 *__restrict__ span, const uint32_t *__restrict__ third,
												const uint32_t *__restrict__ tpos, uint64_t pos[3])
{
	if (tpos)
	{
		pos[0] = tpos[3 * uint64_t(t)];
		pos[1] = tpos[3 * uint64_t(t) + 1];
		pos[2] = tpos[3 * uint64_t(t) + 2];
		return;
	}
	const uint32_t a = __ldg(tris + 3 * uint64_t(t)), b = __ldg(tris + 3 * uint64_t(t) + 1),
				   c = __ldg(tris + 3 * uint64_t(t) + 2);
	const uint32_t u = __ldg(src + b), v = __ldg(E + b), w = __ldg(E + c);
	const uint2 sa = __ldg(span + a), sb = __ldg(span + b), sc = __ldg(span + c);
	pos[0] = lower_bound32(third, sb.x, sb.y, w);
	pos[1] = lower_bound32(third, sa.x, sa.y, v);
	pos[2] = lower_bound32(third, sc.x, sc.y, u);
}

__global__ void k_mark_flags(CtlX *ctl, Frontier fr, int32_t *__restrict__ K, int32_t *__restrict__ S,
							 const uint32_t *__restrict__ tris, const uint32_t *__restrict__ src,
							 const uint32_t *__restrict__ E, const uint2 *__restrict__ span,
							 const uint32_t *__restrict__ third, const uint32_t *__restrict__ tpos,
							 uint32_t *__restrict__ itri, uint64_t n3, uint32_t *__restrict__ R)
{
	if (ctl->c.done)
		return;
	const int32_t level = int32_t(ctl->c.level);
	const uint32_t round = ctl->c.round;
	frontier_each_thread(fr, ctl->c.cur, ctl->c.nF, false, [&](uint32_t t) {
		if (K)
			K[t] = level;
		S[t] = -1 - level; // dead from now on: out of every later scan
		if (R)
			R[t] = round;
		uint64_t pos[3];
		entry_positions(t, tris, src, E, span, third, tpos, pos);
#pragma unroll
		for (int r = 0; r < 3; ++r)
			if (pos[r] < n3)
				itri[pos[r]] = t | DYING;
	});
}

__global__ void k_finalize_flags(CtlX *ctl, Frontier fr, const uint32_t *__restrict__ tris,
								 const uint32_t *__restrict__ src, const uint32_t *__restrict__ E,
								 const uint2 *__restrict__ span, const uint32_t *__restrict__ third,
								 const uint32_t *__restrict__ tpos, uint32_t *__restrict__ itri, uint64_t n3)
{
	if (ctl->c.done)
		return;
	// the round's last frontier kernel: a bitmap frontier is cleared here
	frontier_each_thread(fr, ctl->c.cur, ctl->c.nF, true, [&](uint32_t t) {
		uint64_t pos[3];
		entry_positions(t, tris, src, E, span, third, tpos, pos);
#pragma unroll
		for (int r = 0; r < 3; ++r)
			if (pos[r] < n3)
				itri[pos[r]] = t | DEAD;
	});
}

// Owner rule on flagged entries: q0..q2 are the three partners' entries (no
// DEAD bit); t owns the clique unless a partner dying this round has a
// smaller id. Returns which partners crossed level+1 -> level.
__device__ __forceinline__ void settle_flags(uint32_t t, uint32_t q0, uint32_t q1, uint32_t q2,
											 int32_t *__restrict__ S, int32_t level, bool hit[3])
{
	hit[0] = hit[1] = hit[2] = false;
	if (((q0 & DYING) && (q0 & ID_MASK) < t) || ((q1 & DYING) && (q1 & ID_MASK) < t) ||
		((q2 & DYING) && (q2 & ID_MASK) < t))
		return;
	if (!(q0 & DYING))
		hit[0] = atomicSub(S + q0, 1) == level + 1;
	if (!(q1 & DYING))
		hit[1] = atomicSub(S + q1, 1) == level + 1;
	if (!(q2 & DYING))
		hit[2] = atomicSub(S + q2, 1) == level + 1;
}

// Debit of dying triangles whose shortest list is short: one thread each, so a
// small frontier still spreads over the whole GPU. Dead entries of the
// shortest list are skipped before any search. After a compaction the entry
// of a partner that died earlier is gone; a third that is not found on an edge
// therefore means the clique was destroyed before.
// Debit of dying triangles with long lists: one warp each, tile merge (or
// binary search) of the two shortest lists. A common third whose two
// partners on A and B are alive is queued in shared memory; the queue is
// resolved 32 entries at a time (each lane one lookup on the longest list),
// so the dependent search chain is paid once per 32 live cliques instead of
// once per merge step that has any.
#ifndef N34_L2_PREFETCH
#define N34_L2_PREFETCH 1
#endif
#ifndef N34_C_STAGE
#define N34_C_STAGE 768
#endif
// Work counters of the warp debit in profiling runs (a diagnostic build
// option: the counters cost registers in the hot loop).
#ifndef N34_PEEL_STATS
#define N34_PEEL_STATS 0
#endif
#ifndef N34_DEBIT_MINB
#define N34_DEBIT_MINB 6
#endif
// Claims the next `claim` positions below cap from *cursor into [cpos, cend);
// false when none are left. Called by all lanes with warp-uniform values.
// Positions are 32-bit: the death-flag peel has T <= 2^30, and the cursor
// passes cap by at most one claim per warp.
__device__ __forceinline__ bool claim_range(uint32_t *cursor, uint32_t claim, uint32_t cap, uint32_t &cpos,
											uint32_t &cend)
{
	uint32_t b = 0;
	if (lane_id() == 0)
		b = atomicAdd(cursor, claim);
	b = __shfl_sync(FULL, b, 0);
	if (b >= cap)
		return false;
	cpos = b;
	cend = cap - b > claim ? b + claim : cap;
	return true;
}

// Shared memory of one warp of the warp debit: the queue of lookups on the
// longest list, and a copy of that list's thirds when it is short.
struct DebitSmem
{
	uint32_t *bx, *b0, *b1; // 64 entries each
	uint32_t *cstage;       // N34_C_STAGE entries (unused when 0)
};

// Debit of one dying triangle t by one warp (all lanes call): tile merge (or
// binary search) of the two shortest lists; a common third whose partners on
// A and B are alive, and not owned by a dying partner of smaller id, is queued
// in shared memory; the queue is resolved 32 entries at a time (each lane one
// lookup on the longest list), so the dependent search chain is paid once per
// 32 live cliques instead of once per merge step that has any. Next-frontier
// appends go to the list Fn (or bitmap Bn with BITS). COH: the flags are read
// through L2 (a kernel that wrote them earlier in the same launch).
template <bool BITS, bool COH>
__device__ __forceinline__ void debit_warp_tri(uint32_t t, const Lists &L, const DebitSmem &sm, CtlX *ctl,
											   uint32_t *__restrict__ Fn, uint32_t *__restrict__ Bn,
											   const uint32_t *__restrict__ third, const uint32_t *itri,
											   int32_t *__restrict__ S, int32_t level, uint64_t T)
{
	const uint32_t lane = lane_id();
	uint32_t *nNext = &ctl->c.nNext;
	uint32_t *err = &ctl->c.error;
	uint32_t *bx = sm.bx, *b0 = sm.b0, *b1 = sm.b1;
#if N34_L2_PREFETCH
	if (lane == 0 && use_merge(L))
	{
		prefetch_range_l2(third, L.a0, L.a1);
		prefetch_range_l2(third, L.b0, L.b1);
		prefetch_range_l2(itri, L.a0, L.a1);
		prefetch_range_l2(itri, L.b0, L.b1);
	}
#endif
#if N34_PEEL_STATS
	const bool st = ctl->stats != 0;
#else
	constexpr bool st = false;
#endif
	unsigned long long n_steps = 0, n_lookups = 0, n_resolves = 0, n_staged = 0, n_found = 0;
	uint32_t lo_c = L.c0;
	uint32_t queued = 0; // warp-uniform
	// How the lookups on C are served, decided at the first resolve
	// (warp-uniform): 0 undecided, 1 from a copy of C's thirds staged in
	// shared memory (C short against the lookups: one coalesced read of
	// C instead of a search path per lookup), 2 by sampled binary
	// searches in global memory (one sample of C per triangle).
	uint32_t mode = 0, stage_base = 0, stage_len = 0;
	WarpSample cs{0u, 0u, false};
#if N34_C_STAGE > 0
	uint32_t *cstage = sm.cstage;
#endif
	// resolves the first n (<= 32) queued entries; called by all lanes
	auto resolve = [&](uint32_t n) {
		__syncwarp();
		if (mode == 0)
		{
			const uint32_t len = L.c1 - lo_c;
#if N34_C_STAGE > 0
			if (len <= N34_C_STAGE && len <= 32u * n)
			{
				for (uint32_t i = lane; i < len; i += 32)
					cstage[i] = __ldg(third + lo_c + i);
				__syncwarp();
				stage_base = lo_c;
				stage_len = len;
				mode = 1;
			}
			else
#endif
			{
				cs = warp_sample(third, lo_c, L.c1);
				mode = 2;
			}
		}
		const bool v = lane < n;
		const uint32_t x = v ? bx[lane] : 0xffffffffu;
		const uint32_t q0 = v ? b0[lane] : DEAD, q1 = v ? b1[lane] : DEAD;
		uint32_t pc = L.c1, xc = 0xffffffffu, q2 = DEAD;
#if N34_C_STAGE > 0
		if (mode == 1)
		{
			if (v)
			{
				// lower bound of x in the staged thirds from lo_c on
				uint32_t lo = lo_c - stage_base, cnt = stage_len - lo;
				while (cnt > 0)
				{
					const uint32_t half = cnt >> 1;
					const bool less = cstage[lo + half] < x;
					lo = less ? lo + half + 1 : lo;
					cnt = less ? cnt - half - 1 : half;
				}
				pc = stage_base + lo;
				if (lo < stage_len)
					xc = cstage[lo];
				if (xc == x)
					q2 = ld_tri<COH>(itri + pc);
			}
		}
		else
#endif
		{
			pc = sampled_lower_bound(third, cs, lo_c, L.c1, v, x);
			if (v && pc < L.c1)
			{
				xc = __ldg(third + pc);
				q2 = ld_tri<COH>(itri + pc);
			}
		}
		lo_c = __shfl_sync(FULL, pc, n - 1); // thirds ascend through the queue
		if (st)
		{
			n_lookups += n;
			n_resolves += 1;
			n_staged += mode == 1;
			n_found += __popc(__ballot_sync(FULL, v && xc == x));
		}
		bool hit[3] = {false, false, false};
		// absent from C: that partner died and was compacted away (clique destroyed)
		if (v && xc == x && !(q2 & DEAD))
			settle_flags(t, q0, q1, q2, S, level, hit);
		const uint32_t qs[3] = {q0, q1, q2};
#pragma unroll
		for (int r = 0; r < 3; ++r)
		{
			const uint32_t slot = warp_append(hit[r], nNext);
			if (hit[r])
			{
				if (BITS)
					atomicOr(Bn + (qs[r] >> 5), 1u << (qs[r] & 31));
				else if (slot < T)
					Fn[slot] = qs[r];
				else
					atomicOr(err, 1u);
			}
		}
		__syncwarp();
	};
	warp_intersect2<true, COH>(third, itri, L, [&](bool found, uint32_t x, uint32_t, uint32_t, uint32_t qa,
												   uint32_t qb) {
		n_steps += st;
		// a clique is looked up on C only if its partners on A and B are
		// alive and neither is a dying triangle of smaller id (its owner)
		const bool live = found && !(qa & DEAD) && !(qb & DEAD) && !((qa & DYING) && (qa & ID_MASK) < t) &&
						  !((qb & DYING) && (qb & ID_MASK) < t);
		const uint32_t fm = __ballot_sync(FULL, live);
		if (!fm)
			return;
		const uint32_t o = queued + __popc(fm & lanemask_lt());
		if (live)
		{
			bx[o] = x;
			b0[o] = qa;
			b1[o] = qb;
		}
		queued += __popc(fm);
		if (queued >= 32)
		{
			resolve(32);
			// move the overflow [32, queued) to the front (ranges do not overlap)
			const uint32_t rest = queued - 32;
			uint32_t mx = 0, m0 = 0, m1 = 0;
			if (lane < rest)
			{
				mx = bx[32 + lane];
				m0 = b0[32 + lane];
				m1 = b1[32 + lane];
			}
			__syncwarp();
			if (lane < rest)
			{
				bx[lane] = mx;
				b0[lane] = m0;
				b1[lane] = m1;
			}
			queued = rest;
		}
	});
	if (queued)
		resolve(queued);
	__syncwarp();
	if (st && lane == 0)
	{
		atomicAdd(&ctl->st_tri, 1ull);
		atomicAdd(&ctl->st_merge_entries, (unsigned long long)(L.a1 - L.a0 + L.b1 - L.b0));
		atomicAdd(&ctl->st_steps, n_steps);
		atomicAdd(&ctl->st_lookups, n_lookups);
		atomicAdd(&ctl->st_resolves, n_resolves);
		atomicAdd(&ctl->st_staged, n_staged);
		atomicAdd(&ctl->st_found, n_found);
	}
}

// Debit of one dying triangle whose shortest list is short, by one thread
// (see k_debit_flags_thread). Returns without work when the list is longer.
template <uint32_t LANE_MAX, bool BITS, bool COH>
__device__ __forceinline__ void debit_thread_tri(uint32_t t, const Lists &L, CtlX *ctl, uint32_t *__restrict__ Fn,
												 uint32_t *__restrict__ Bn, const uint32_t *__restrict__ third,
												 const uint32_t *itri, int32_t *__restrict__ S, int32_t level,
												 uint64_t T)
{
	uint32_t lo_b = L.b0, lo_c = L.c0;
	for (uint32_t i = L.a0; i < L.a1 && lo_b < L.b1; ++i)
	{
		const uint32_t q0 = ld_tri<COH>(itri + i);
		if (q0 & DEAD)
			continue;
		const uint32_t x = __ldg(third + i);
		lo_b = lower_bound32(third, lo_b, L.b1, x);
		if (lo_b >= L.b1)
			break;
		if (__ldg(third + lo_b) != x)
			continue;
		const uint32_t q1 = ld_tri<COH>(itri + lo_b);
		if (q1 & DEAD)
			continue;
		lo_c = lower_bound32(third, lo_c, L.c1, x);
		if (lo_c >= L.c1 || __ldg(third + lo_c) != x)
			continue; // the partner on the longest list was compacted away
		const uint32_t q2 = ld_tri<COH>(itri + lo_c);
		if (q2 & DEAD)
			continue;
		bool hit[3];
		settle_flags(t, q0, q1, q2, S, level, hit);
		const uint32_t qs[3] = {q0, q1, q2};
#pragma unroll
		for (int r = 0; r < 3; ++r)
			if (hit[r])
			{
				const uint32_t slot = atomicAdd(&ctl->c.nNext, 1u);
				if (BITS)
					atomicOr(Bn + (qs[r] >> 5), 1u << (qs[r] & 31));
				else if (slot < T)
					Fn[slot] = qs[r];
				else
					atomicOr(&ctl->c.error, 1u);
			}
	}
}

template <uint32_t LANE_MAX>
__global__ void __launch_bounds__(PEEL_THREADS) k_debit_flags_thread(
	CtlX *ctl, Frontier fr, const uint32_t *__restrict__ tris, const uint2 *__restrict__ span,
	const uint32_t *__restrict__ third, const uint32_t *__restrict__ itri, int32_t *__restrict__ S, uint64_t T,
	bool chunked)
{
	if (ctl->c.done || (chunked && !fr.bits()))
		return; // chunked: the warp kernel's lanes take the short lists too
	const uint32_t cur = ctl->c.cur;
	const int32_t level = int32_t(ctl->c.level);
	uint32_t *Fn = fr.bits() ? nullptr : fr.next_list(cur);
	uint32_t *Bn = fr.bits() ? fr.next_bits(cur) : nullptr;
	const bool bits = fr.bits();
	frontier_each_thread(fr, cur, ctl->c.nF, false, [&](uint32_t t) {
		const Lists L = frontier_lists(t, tris, span);
		if (L.a1 - L.a0 > LANE_MAX)
			return; // the warp kernel takes it
		if (bits)
			debit_thread_tri<LANE_MAX, true, false>(t, L, ctl, Fn, Bn, third, itri, S, level, T);
		else
			debit_thread_tri<LANE_MAX, false, false>(t, L, ctl, Fn, Bn, third, itri, S, level, T);
	});
}

// Debit of the round's dying triangles whose shortest list is longer than
// LANE_MAX, one warp per triangle (shorter ones: k_debit_flags_thread).
// BITS: bitmap frontiers (memory-lean layout) instead of lists. The other
// parameters choose how warps walk a list frontier; all give the same k:
// CHUNKED, a warp loads up to 32 triangles' records at once and its lanes
// also debit the short lists; PIPE, the next triangles' ids and records are
// loaded ahead of the current debit; CURSOR, one wave of blocks claims
// positions from an atomic cursor. Default: a fixed warp stride.
// The pipelined instantiation returns before the generic walk below.
#pragma nv_diag_suppress 128
template <bool BITS, uint32_t LANE_MAX, bool CHUNKED = false, bool PIPE = false, bool CURSOR = false>
__global__ void __launch_bounds__(PEEL_THREADS, PIPE ? 5 : N34_DEBIT_MINB) k_debit_flags_warp(
	CtlX *ctl, uint32_t *__restrict__ F0, uint32_t *__restrict__ F1, uint32_t *__restrict__ B0,
	uint32_t *__restrict__ B1, uint64_t W, const uint32_t *__restrict__ tris, const uint2 *__restrict__ span,
	const uint32_t *__restrict__ third, const uint32_t *__restrict__ itri, int32_t *__restrict__ S, uint64_t T)
{
	constexpr int WARPS = PEEL_THREADS / 32;
	__shared__ uint32_t qx[WARPS][64], qp0[WARPS][64], qp1[WARPS][64];
#if N34_C_STAGE > 0
	__shared__ uint32_t cstage_all[WARPS][N34_C_STAGE];
#endif
	if (ctl->c.done)
		return;
	uint32_t *Fn = ctl->c.cur ? F0 : F1;
	uint32_t *Bn = ctl->c.cur ? B0 : B1;
	const int32_t level = int32_t(ctl->c.level);
	const uint32_t wib = threadIdx.x >> 5;
#if N34_C_STAGE > 0
	const DebitSmem sm{qx[wib], qp0[wib], qp1[wib], cstage_all[wib]};
#else
	const DebitSmem sm{qx[wib], qp0[wib], qp1[wib], nullptr};
#endif
	const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
	const uint32_t nF = ctl->c.nF;
	const uint32_t *F = ctl->c.cur ? F1 : F0;
	const uint32_t *Bc = ctl->c.cur ? B1 : B0;
	uint32_t word = 0; // bits of word fi not yet taken (bitmap mode)
	if (!BITS && CHUNKED)
	{
		// Chunked schedule (list frontiers): a warp takes ch consecutive
		// frontier triangles, its lanes load their records and spans at once
		// (one dependent chain per chunk instead of one per triangle), lanes
		// debit the short lists themselves, then the warp debits the long
		// ones. ch doubles while every warp still gets two chunks, so small
		// frontiers keep one triangle per warp.
		const uint32_t lane = lane_id();
		uint32_t ch = 1;
		while (ch < 32 && uint64_t(ch) * 2 * nwarps <= nF)
			ch <<= 1;
		for (uint64_t base = warp * ch; base < nF; base += nwarps * ch)
		{
			const uint64_t i = base + lane;
			const bool have = lane < ch && i < nF;
			uint32_t t = 0;
			Lists L{0, 0, 0, 0, 0, 0};
			if (have)
			{
				t = F[i];
				L = frontier_lists(t, tris, span);
			}
			const bool is_long = have && (L.a1 - L.a0 > LANE_MAX);
			if (have && !is_long)
				debit_thread_tri<LANE_MAX, false, false>(t, L, ctl, Fn, nullptr, third, itri, S, level, T);
			uint32_t longs = __ballot_sync(FULL, is_long);
			while (longs)
			{
				const uint32_t sl = __ffs(longs) - 1;
				longs &= longs - 1;
				const uint32_t tt = __shfl_sync(FULL, t, sl);
				// its lists again (record and spans were just loaded: cache hits)
				// rather than six more registers held across the long debits
				const Lists LL = frontier_lists(tt, tris, span);
				debit_warp_tri<false, false>(tt, LL, sm, ctl, Fn, nullptr, third, itri, S, level, T);
			}
		}
		return;
	}
	if (!BITS && PIPE)
	{
		// Software-pipelined walk of this warp's frontier positions: the id of
		// the triangle two ahead and the record (three edge ids) of the one
		// after the current are loaded before the current triangle's debit and
		// used after it, so only the spans' load waits at the top of each step.
		uint64_t fi = warp;
		uint32_t tc = fi < nF ? F[fi] : 0;
		uint32_t tn = fi + nwarps < nF ? F[fi + nwarps] : 0;
		uint32_t ea = 0, eb = 0, ec = 0;
		if (fi < nF)
		{
			ea = __ldg(tris + 3 * uint64_t(tc));
			eb = __ldg(tris + 3 * uint64_t(tc) + 1);
			ec = __ldg(tris + 3 * uint64_t(tc) + 2);
		}
		for (; fi < nF; fi += nwarps)
		{
			const uint64_t f2 = fi + 2 * nwarps;
			const uint32_t t2 = f2 < nF ? F[f2] : 0;
			uint32_t na = 0, nb = 0, nc = 0;
			if (fi + nwarps < nF)
			{
				na = __ldg(tris + 3 * uint64_t(tn));
				nb = __ldg(tris + 3 * uint64_t(tn) + 1);
				nc = __ldg(tris + 3 * uint64_t(tn) + 2);
			}
			const uint2 sa = __ldg(span + ea), sb = __ldg(span + eb), sc = __ldg(span + ec);
			const Lists L = order_lists(sa.x, sa.y, sb.x, sb.y, sc.x, sc.y);
			if (L.a1 - L.a0 > LANE_MAX) // warp-uniform; short lists: the thread kernel
				debit_warp_tri<false, false>(tc, L, sm, ctl, Fn, nullptr, third, itri, S, level, T);
			tc = tn;
			tn = t2;
			ea = na;
			eb = nb;
			ec = nc;
		}
		return;
	}
	// The warp's next triangle comes either from the positions (list) or
	// bitmap words it claims, CLAIM at a time, from the round's cursor (CURSOR:
	// one wave of blocks, balanced at run time), or from a fixed warp stride
	// over the frontier. [cpos, cend): the current claim; fi: the stride's
	// position (list) or bitmap word, advanced by each branch itself.
	constexpr uint32_t CLAIM = BITS ? 4 : 16;
	const uint32_t cap = BITS ? uint32_t(W) : nF;
	uint32_t cpos = 0, cend = 0;
	uint64_t fi = warp;
	for (;;)
	{
		uint32_t t;
		if (CURSOR && BITS)
		{
			// next nonzero word of the claim, claiming again when it is used up
			while (!word)
			{
				if (cpos >= cend && !claim_range(&ctl->cursor, CLAIM, cap, cpos, cend))
					break;
				word = Bc[cpos];
				if (!word)
					++cpos;
			}
			if (!word)
				break;
			t = uint32_t(cpos * 32 + (__ffs(word) - 1));
			word &= word - 1;
			if (!word)
				++cpos;
		}
		else if (CURSOR)
		{
			if (cpos >= cend && !claim_range(&ctl->cursor, CLAIM, cap, cpos, cend))
				break;
			t = F[cpos++];
		}
		else if (BITS)
		{
			while (!word && fi < W)
			{
				word = Bc[fi];
				if (!word)
					fi += nwarps;
			}
			if (!word)
				break;
			t = uint32_t(fi * 32 + (__ffs(word) - 1));
			word &= word - 1;
			if (!word)
				fi += nwarps;
		}
		else
		{
			if (fi >= nF)
				break;
			t = F[fi];
			fi += nwarps;
		}
		const Lists L = frontier_lists(t, tris, span);
		if (L.a1 - L.a0 <= LANE_MAX)
			continue; // the thread kernel took it (warp-uniform)
		debit_warp_tri<BITS, false>(t, L, sm, ctl, Fn, Bn, third, itri, S, level, T);
	}
}
#pragma nv_diag_default 128

// Ordering of large frontiers. Appends leave the next frontier in random
// order; the debit of a random order reads every dying triangle's lists from
// DRAM, while in id order (edge-major, as the triangles are numbered)
// neighbouring warps share lists in L2. A frontier of at least
// max(T >> sort_shift, SORT_MIN) triangles (ctl->sort_min) is therefore
// rewritten in id order through a bitmap: set bits, count per chunk, scan the
// counts, write the ids back (clearing the bits).
#ifndef N34_SORT_MIN
#define N34_SORT_MIN 4096ull
#endif
constexpr uint32_t SORT_CHUNK_WORDS = 1024; // bitmap words per chunk (4 per thread)
constexpr int SORT_THREADS = 256;

__device__ __forceinline__ bool sort_wanted(const CtlX *ctl, uint64_t T)
{
	return !ctl->c.done && ctl->c.nNext >= ctl->sort_min && ctl->c.nNext <= T;
}

// Sort key of a frontier triangle: its id, or, with cpos (the entry
// positions of the triangles' c edges, 3t + 2 of tpos), the position of its
// entry under c. Entry positions are edge-major, so the second order groups
// the triangles that share their c edge (v -> w, between the two vertices of
// higher degree: usually their longest list, the one every lookup searches).
__global__ void k_fsort_set(const CtlX *ctl, const uint32_t *__restrict__ F0, const uint32_t *__restrict__ F1,
							uint32_t *__restrict__ bits, uint64_t T, const uint32_t *__restrict__ tpos,
							uint64_t keys)
{
	if (!sort_wanted(ctl, T))
		return;
	const uint32_t *Fn = ctl->c.cur ? F0 : F1;
	const uint32_t n = ctl->c.nNext;
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
	{
		const uint32_t t = Fn[i];
		if (t >= T)
			continue;
		const uint32_t k = tpos ? tpos[3 * uint64_t(t) + 2] : t;
		if (k < keys)
			atomicOr(bits + (k >> 5), 1u << (k & 31));
	}
}

__global__ void __launch_bounds__(SORT_THREADS) k_fsort_count(const CtlX *ctl, const uint32_t *__restrict__ bits,
															   uint64_t W, uint32_t *__restrict__ chunk, uint64_t T)
{
	if (!sort_wanted(ctl, T))
		return;
	const uint64_t nchunks = (W + SORT_CHUNK_WORDS - 1) / SORT_CHUNK_WORDS;
	__shared__ uint32_t wsum[SORT_THREADS / 32];
	for (uint64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x)
	{
		uint32_t cnt = 0;
#pragma unroll
		for (int k = 0; k < 4; ++k)
		{
			const uint64_t w = ch * SORT_CHUNK_WORDS + uint64_t(k) * SORT_THREADS + threadIdx.x;
			if (w < W)
				cnt += __popc(bits[w]);
		}
#pragma unroll
		for (int o = 16; o > 0; o >>= 1)
			cnt += __shfl_xor_sync(FULL, cnt, o);
		if (lane_id() == 0)
			wsum[threadIdx.x >> 5] = cnt;
		__syncthreads();
		if (threadIdx.x == 0)
		{
			uint32_t tot = 0;
			for (int i = 0; i < SORT_THREADS / 32; ++i)
				tot += wsum[i];
			chunk[ch] = tot;
		}
		__syncthreads();
	}
}

// exclusive scan of the chunk counts, one block
__global__ void __launch_bounds__(1024) k_fsort_scan(const CtlX *ctl, uint32_t *__restrict__ chunk, uint64_t nchunks,
													  uint64_t T)
{
	if (!sort_wanted(ctl, T))
		return;
	__shared__ uint32_t part[32];
	__shared__ uint32_t carry;
	if (threadIdx.x == 0)
		carry = 0;
	__syncthreads();
	for (uint64_t base = 0; base < nchunks; base += 1024)
	{
		const uint64_t i = base + threadIdx.x;
		const uint32_t v = i < nchunks ? chunk[i] : 0u;
		uint32_t x = v; // inclusive warp scan
#pragma unroll
		for (int o = 1; o < 32; o <<= 1)
		{
			const uint32_t y = __shfl_up_sync(FULL, x, o);
			if (lane_id() >= uint32_t(o))
				x += y;
		}
		if (lane_id() == 31)
			part[threadIdx.x >> 5] = x;
		__syncthreads();
		if (threadIdx.x < 32)
		{
			uint32_t p = part[threadIdx.x];
#pragma unroll
			for (int o = 1; o < 32; o <<= 1)
			{
				const uint32_t y = __shfl_up_sync(FULL, p, o);
				if (lane_id() >= uint32_t(o))
					p += y;
			}
			part[threadIdx.x] = p; // inclusive over warps
		}
		__syncthreads();
		const uint32_t wbase = (threadIdx.x >> 5) ? part[(threadIdx.x >> 5) - 1] : 0u;
		if (i < nchunks)
			chunk[i] = carry + wbase + x - v;
		__syncthreads();
		if (threadIdx.x == 0)
			carry += part[31];
		__syncthreads();
	}
}

__global__ void __launch_bounds__(SORT_THREADS) k_fsort_write(const CtlX *ctl, uint32_t *__restrict__ bits,
															   uint64_t W, const uint32_t *__restrict__ chunk,
															   uint32_t *__restrict__ F0, uint32_t *__restrict__ F1,
															   uint64_t T, const uint32_t *__restrict__ itri)
{
	if (!sort_wanted(ctl, T))
		return;
	uint32_t *Fn = ctl->c.cur ? F0 : F1;
	const uint32_t n = ctl->c.nNext;
	const uint64_t nchunks = (W + SORT_CHUNK_WORDS - 1) / SORT_CHUNK_WORDS;
	__shared__ uint32_t wsum[SORT_THREADS / 32];
	for (uint64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x)
	{
		// each thread owns 4 consecutive words so that its ids come out in order
		const uint64_t w0 = ch * SORT_CHUNK_WORDS + 4 * uint64_t(threadIdx.x);
		uint32_t wv[4];
		uint32_t cnt = 0;
#pragma unroll
		for (int k = 0; k < 4; ++k)
		{
			wv[k] = (w0 + k < W) ? bits[w0 + k] : 0u;
			cnt += __popc(wv[k]);
		}
		uint32_t x = cnt; // inclusive block scan of the thread counts
#pragma unroll
		for (int o = 1; o < 32; o <<= 1)
		{
			const uint32_t y = __shfl_up_sync(FULL, x, o);
			if (lane_id() >= uint32_t(o))
				x += y;
		}
		if (lane_id() == 31)
			wsum[threadIdx.x >> 5] = x;
		__syncthreads();
		uint32_t wb = 0;
		for (uint32_t i = 0; i < (threadIdx.x >> 5); ++i)
			wb += wsum[i];
		uint32_t pos = chunk[ch] + wb + x - cnt;
#pragma unroll
		for (int k = 0; k < 4; ++k)
		{
			uint32_t m = wv[k];
			while (m)
			{
				const uint32_t b = __ffs(m) - 1;
				m &= m - 1;
				if (pos < n)
				{
					const uint32_t key = uint32_t((w0 + k) * 32 + b);
					// an entry position names its triangle (flags masked)
					Fn[pos] = itri ? (itri[key] & ID_MASK) : key;
				}
				++pos;
			}
			if (wv[k])
				bits[w0 + k] = 0u;
		}
		__syncthreads();
	}
}

// Compaction gate, run after each replay: once the triangles peeled since
// the last compaction reach 1/compact_div of the live ones then, the next
// k_compact_spans drops the dead entries. A compaction reads every remaining
// entry once, so the passes form a geometric series (at most compact_div
// passes over the full incidence in total).
__global__ void k_compact_gate(CtlX *ctl, uint64_t T)
{
	const unsigned long long peeled = ctl->c.peeled;
	ctl->compact_now = 0;
	if (ctl->c.done || peeled >= T)
		return;
	if (ctl->compact_div &&
		(unsigned long long)ctl->compact_div * (peeled - ctl->peeled_at_compact) >= ctl->live_at_compact)
	{
		ctl->compact_now = 1;
		ctl->peeled_at_compact = peeled;
		ctl->live_at_compact = T - peeled;
		ctl->compactions++;
	}
}

// In-place compaction of every edge list (one warp per edge): live entries
// move to the front of the list, keeping their order, and the span's end is
// lowered. A tile is fully read (warp ballot) before any lane writes, and the
// write cursor never passes the tile's start, so unread entries stay intact.
__global__ void __launch_bounds__(PEEL_THREADS) k_compact_spans(const CtlX *ctl, uint2 *__restrict__ span,
																  uint64_t m, uint32_t *__restrict__ third,
																  uint32_t *__restrict__ itri, uint32_t *__restrict__ tpos)
{
	if (!ctl->compact_now)
		return;
	const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
	const uint32_t lane = lane_id();
	for (uint64_t e = warp; e < m; e += nwarps)
	{
		const uint2 sp = span[e];
		uint32_t out = sp.x;
		for (uint32_t base = sp.x; base < sp.y; base += 32)
		{
			const uint32_t i = base + lane;
			uint32_t t = DEAD, x = 0;
			if (i < sp.y)
			{
				t = itri[i];
				x = third[i];
			}
			const bool keep = !(t & DEAD);
			const uint32_t bal = __ballot_sync(FULL, keep);
			const uint32_t o = out + __popc(bal & lanemask_lt());
			if (keep && o != i)
			{
				third[o] = x;
				itri[o] = t;
				if (tpos)
				{
					// the moved entry is the one of t's three recorded at i
					uint32_t *tp = tpos + 3 * uint64_t(t);
					const uint32_t r = tp[0] == i ? 0u : (tp[1] == i ? 1u : 2u);
					tp[r] = o;
				}
			}
			out += __popc(bal);
		}
		if (lane == 0 && out != sp.y)
			span[e].y = out;
	}
}

__global__ void k_advance(CtlX *ctl)
{
	PeelCtl &c = ctl->c;
	if (c.done)
		return;
	if (c.nF)
	{
		c.peeled += c.nF;
		c.rounds++;
	}
	c.round++;
	c.cur ^= 1u;
	c.nF = c.nNext;
	c.nNext = 0;
	c.minS = INF;
	ctl->scan = c.nF == 0;
	ctl->cursor = 0;
}

// ---- small rounds in one cooperative launch ----------------------------------
//
// Most rounds of a peel are small cascades (R-MAT scale 20: about 4300 of 5500
// rounds have fewer than 2^16 dying triangles), and as separate launches each
// pays a dozen kernels' fixed cost. k_small_rounds runs such rounds back to
// back in one cooperative launch: mark, debit, finalize and advance of a round
// are phases separated by grid barriers. It returns as soon as the frontier
// is empty (a level change: the regular kernels scan), larger than
// small_max, or the peel is done; the regular round that follows takes over.
// The rules are those of the regular kernels (same device functions); flags
// written in one phase are read in the next through L2 (__ldcg), never
// through the read-only path.

struct GridBar
{
	unsigned int count; // blocks arrived at the current barrier
	unsigned int gen;   // barriers completed
	unsigned int abort; // a wait ran past its time bound
	unsigned int pad;
};

__device__ __forceinline__ unsigned long long global_ns()
{
	unsigned long long t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

// Barrier of all blocks of a cooperative launch (all resident at once by
// construction). Waits are bounded: past the deadline a block sets abort and
// leaves; every block then sees abort (here or at its next barrier) and
// returns false, so the kernel ends in any case.
__device__ __forceinline__ bool grid_barrier(GridBar *bar, uint32_t &gen, unsigned long long deadline)
{
	__shared__ uint32_t ok_s;
	__syncthreads();
	if (threadIdx.x == 0)
	{
		__threadfence();
		const uint32_t g = gen;
		if (atomicAdd(&bar->count, 1u) == gridDim.x - 1)
		{
			atomicExch(&bar->count, 0u);
			__threadfence();
			atomicExch(&bar->gen, g + 1);
		}
		else
		{
			uint32_t spins = 0;
			while (__ldcg(&bar->gen) == g)
			{
				if (__ldcg(&bar->abort))
					break;
				if ((++spins & 255u) == 0 && global_ns() > deadline)
				{
					atomicExch(&bar->abort, 1u);
					break;
				}
				__nanosleep(64);
			}
		}
		gen = g + 1;
		__threadfence();
		ok_s = __ldcg(&bar->abort) == 0;
	}
	__syncthreads();
	return ok_s != 0;
}

#ifndef N34_SMALL_MAX
#define N34_SMALL_MAX 8192u
#endif
// Time bound of one k_small_rounds launch (its rounds take microseconds each).
constexpr unsigned long long SMALL_ROUNDS_LIMIT_NS = 10ull * 1000000000ull;
// Rounds of one k_small_rounds launch at most (each peels at least one triangle).
constexpr uint32_t SMALL_ROUNDS_MAX_ITER = 1u << 16;

template <uint32_t LANE_MAX>
__global__ void __launch_bounds__(PEEL_THREADS, 4) k_small_rounds(
	CtlX *ctl, GridBar *bar, uint32_t *F0, uint32_t *F1, const uint32_t *__restrict__ tris,
	const uint32_t *__restrict__ src, const uint32_t *__restrict__ E, const uint2 *__restrict__ span,
	const uint32_t *__restrict__ third, const uint32_t *__restrict__ tpos, uint32_t *itri, uint64_t n3,
	int32_t *K, int32_t *S, uint32_t *R, uint64_t T, uint32_t small_max)
{
	constexpr int WARPS = PEEL_THREADS / 32;
	__shared__ uint32_t qx[WARPS][64], qp0[WARPS][64], qp1[WARPS][64];
#if N34_C_STAGE > 0
	__shared__ uint32_t cstage_all[WARPS][N34_C_STAGE];
#endif
	__shared__ uint32_t s_go, s_nF, s_cur, s_level, s_round;
	const uint32_t lane = lane_id(), wib = threadIdx.x >> 5;
#if N34_C_STAGE > 0
	const DebitSmem sm{qx[wib], qp0[wib], qp1[wib], cstage_all[wib]};
#else
	const DebitSmem sm{qx[wib], qp0[wib], qp1[wib], nullptr};
#endif
	const uint64_t tid = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
	const uint64_t nthreads = uint64_t(gridDim.x) * blockDim.x;
	const uint64_t warp = tid >> 5, nwarps = nthreads >> 5;
	uint32_t gen = 0;
	if (threadIdx.x == 0)
		gen = __ldcg(&bar->gen);
	const unsigned long long deadline = global_ns() + SMALL_ROUNDS_LIMIT_NS;
	bool aborted = false;
	for (uint32_t it = 0; it < SMALL_ROUNDS_MAX_ITER; ++it)
	{
		if (threadIdx.x == 0)
		{
			const uint32_t nF = __ldcg(&ctl->c.nF);
			s_go = !__ldcg(&ctl->c.done) && !__ldcg(&ctl->c.error) && !__ldcg(&ctl->scan) && nF > 0 &&
				   nF <= small_max;
			s_nF = nF;
			s_cur = __ldcg(&ctl->c.cur);
			s_level = __ldcg(&ctl->c.level);
			s_round = __ldcg(&ctl->c.round);
		}
		__syncthreads();
		if (!s_go) // the same for every block: ctl was last written before a barrier
			break;
		const uint32_t nF = s_nF, cur = s_cur, round = s_round;
		const int32_t level = int32_t(s_level);
		const uint32_t *F = cur ? F1 : F0;
		uint32_t *Fn = cur ? F0 : F1;
		// mark: k and the dying flag of every frontier triangle
		for (uint64_t i = tid; i < nF; i += nthreads)
		{
			const uint32_t t = __ldcg(F + i);
			if (K)
				K[t] = level;
			S[t] = -1 - level;
			if (R)
				R[t] = round;
			uint64_t pos[3];
			entry_positions(t, tris, src, E, span, third, tpos, pos);
#pragma unroll
			for (int r = 0; r < 3; ++r)
				if (pos[r] < n3)
					itri[pos[r]] = t | DYING;
		}
		if (!grid_barrier(bar, gen, deadline))
		{
			aborted = true;
			break;
		}
		// debit: triangles whose shortest list is short one thread each, then
		// the others one warp each (the split of the regular kernels; both
		// passes only append to the next frontier, so no barrier between)
		for (uint64_t i = tid; i < nF; i += nthreads)
		{
			const uint32_t t = __ldcg(F + i);
			const Lists L = frontier_lists(t, tris, span);
			if (L.a1 - L.a0 <= LANE_MAX)
				debit_thread_tri<LANE_MAX, false, true>(t, L, ctl, Fn, nullptr, third, itri, S, level, T);
		}
		for (uint64_t i = warp; i < nF; i += nwarps)
		{
			const uint32_t t = __ldcg(F + i);
			const Lists L = frontier_lists(t, tris, span);
			if (L.a1 - L.a0 > LANE_MAX) // warp-uniform
				debit_warp_tri<false, true>(t, L, sm, ctl, Fn, nullptr, third, itri, S, level, T);
		}
		if (!grid_barrier(bar, gen, deadline))
		{
			aborted = true;
			break;
		}
		// finalize: dying -> dead
		for (uint64_t i = tid; i < nF; i += nthreads)
		{
			const uint32_t t = __ldcg(F + i);
			uint64_t pos[3];
			entry_positions(t, tris, src, E, span, third, tpos, pos);
#pragma unroll
			for (int r = 0; r < 3; ++r)
				if (pos[r] < n3)
					itri[pos[r]] = t | DEAD;
		}
		if (!grid_barrier(bar, gen, deadline))
		{
			aborted = true;
			break;
		}
		// advance (as k_advance)
		if (blockIdx.x == 0 && threadIdx.x == 0)
		{
			PeelCtl &c = ctl->c;
			const uint32_t nNext = __ldcg(&c.nNext);
			c.peeled += nF;
			c.rounds++;
			c.round = round + 1;
			c.cur = cur ^ 1u;
			c.nF = nNext;
			c.nNext = 0;
			c.minS = INF;
			ctl->scan = nNext == 0;
			ctl->small_rounds++;
			ctl->cursor = 0;
		}
		if (!grid_barrier(bar, gen, deadline))
		{
			aborted = true;
			break;
		}
	}
	if (aborted && threadIdx.x == 0)
	{
		atomicOr(&ctl->c.error, 4u);
		atomicExch(&ctl->timed_out, 1u);
	}
}

// End of one pass of the device loop's body: go on while the peel is neither
// done nor failed, within its round bound and its time bound.
__global__ void k_loop_cond(CtlX *ctl, cudaGraphConditionalHandle h, uint32_t max_rounds,
							unsigned long long limit_ns)
{
	unsigned long long now;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
	ctl->loop_passes++;
	bool more = !ctl->c.done && !ctl->c.error;
	if (more && (ctl->c.round > max_rounds || now - ctl->t0_ns > limit_ns))
	{
		ctl->timed_out = 1;
		more = false;
	}
	cudaGraphSetConditional(h, more ? 1u : 0u);
}

__global__ void k_s_to_k(int32_t *__restrict__ S, uint64_t T)
{
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < T; t += stride)
		S[t] = -1 - S[t];
}

__global__ void k_stats(CtlX *ctl, const int32_t *__restrict__ K, uint64_t T)
{
	unsigned long long sum = 0;
	uint32_t mx = 0, unp = 0;
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < T; t += stride)
	{
		const int32_t k = K[t];
		if (k < 0)
			unp++;
		else
		{
			sum += uint64_t(k);
			mx = max(mx, uint32_t(k));
		}
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
	{
		sum += __shfl_xor_sync(FULL, sum, o);
		mx = max(mx, __shfl_xor_sync(FULL, mx, o));
		unp += __shfl_xor_sync(FULL, unp, o);
	}
	if (lane_id() == 0)
	{
		if (sum)
			atomicAdd(&ctl->c.ksum, sum);
		if (mx)
			atomicMax(&ctl->c.kmax, mx);
		if (unp)
			atomicAdd(&ctl->c.unpeeled, unp);
	}
}

// The two debit kernels of the death-flag peel with one lane/warp split
// (LM); ev5 (profiling only) is recorded between them.
template <uint32_t LM>
void launch_debit_flags(cudaStream_t st, uint32_t gscan, uint32_t gwarp, bool lean, CtlX *ctl, const Frontier &fr,
						const uint32_t *tris, const Incidence &inc, int32_t *S, uint64_t T, cudaEvent_t ev5,
						bool chunked, bool pipelined, bool cursor)
{
	k_debit_flags_thread<LM><<<gscan, PEEL_THREADS, 0, st>>>(ctl, fr, tris, inc.span, inc.third, inc.tri, S, T,
															 chunked);
	if (ev5)
		cudaEventRecord(ev5, st);
	if (cursor)
	{
		// one wave: as many blocks as can be resident at once on every SM
		int dev = 0, sms = 1, per_sm = 1;
		if (cudaGetDevice(&dev) != cudaSuccess ||
			cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
			cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm,
														  lean ? k_debit_flags_warp<true, LM, false, false, true>
															   : k_debit_flags_warp<false, LM, false, false, true>,
														  PEEL_THREADS, 0) != cudaSuccess ||
			per_sm < 1)
		{
			cudaGetLastError();
			per_sm = 1;
		}
		gwarp = uint32_t(per_sm) * uint32_t(sms > 0 ? sms : 1);
	}
	if (lean && cursor)
		k_debit_flags_warp<true, LM, false, false, true><<<gwarp, PEEL_THREADS, 0, st>>>(
			ctl, fr.F0, fr.F1, fr.B0, fr.B1, fr.W, tris, inc.span, inc.third, inc.tri, S, T);
	else if (lean)
		k_debit_flags_warp<true, LM><<<gwarp, PEEL_THREADS, 0, st>>>(ctl, fr.F0, fr.F1, fr.B0, fr.B1, fr.W, tris,
																	 inc.span, inc.third, inc.tri, S, T);
	else if (chunked)
		k_debit_flags_warp<false, LM, true><<<gwarp, PEEL_THREADS, 0, st>>>(ctl, fr.F0, fr.F1, fr.B0, fr.B1, fr.W,
																			tris, inc.span, inc.third, inc.tri, S, T);
	else if (pipelined)
		k_debit_flags_warp<false, LM, false, true><<<gwarp, PEEL_THREADS, 0, st>>>(
			ctl, fr.F0, fr.F1, fr.B0, fr.B1, fr.W, tris, inc.span, inc.third, inc.tri, S, T);
	else if (cursor)
		k_debit_flags_warp<false, LM, false, false, true><<<gwarp, PEEL_THREADS, 0, st>>>(
			ctl, fr.F0, fr.F1, fr.B0, fr.B1, fr.W, tris, inc.span, inc.third, inc.tri, S, T);
	else
		k_debit_flags_warp<false, LM><<<gwarp, PEEL_THREADS, 0, st>>>(ctl, fr.F0, fr.F1, fr.B0, fr.B1, fr.W, tris,
																	  inc.span, inc.third, inc.tri, S, T);
}

// Cooperative launch of k_small_rounds (capturable into a CUDA graph).
template <uint32_t LM>
cudaError_t launch_small_rounds(cudaStream_t st, uint32_t grid, CtlX *ctl, GridBar *bar, const Frontier &fr,
								const uint32_t *tris, const uint32_t *src, const uint32_t *E, const Incidence &inc,
								int32_t *K, int32_t *S, uint32_t *R, uint64_t T, uint32_t small_max)
{
	cudaLaunchConfig_t cfg{};
	cfg.gridDim = dim3(grid);
	cfg.blockDim = dim3(PEEL_THREADS);
	cfg.dynamicSmemBytes = 0;
	cfg.stream = st;
	cudaLaunchAttribute at[1];
	at[0].id = cudaLaunchAttributeCooperative;
	at[0].val.cooperative = 1;
	cfg.attrs = at;
	cfg.numAttrs = 1;
	return cudaLaunchKernelEx(&cfg, k_small_rounds<LM>, ctl, bar, fr.F0, fr.F1, tris, src, E,
							  static_cast<const uint2 *>(inc.span), static_cast<const uint32_t *>(inc.third),
							  static_cast<const uint32_t *>(inc.tpos), inc.tri, uint64_t(3 * T), K, S, R, T, small_max);
}

template <uint32_t LM>
uint32_t small_rounds_grid(int sm_count)
{
	int per_sm = 0;
	if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_small_rounds<LM>, PEEL_THREADS, 0) != cudaSuccess ||
		per_sm < 1)
	{
		cudaGetLastError();
		return 0;
	}
	return uint32_t(per_sm) * uint32_t(sm_count);
}

} // namespace

int peel(Ctx &c, int variant, const Incidence &inc, const CliqueCsr &csr, int32_t *S, int32_t *K, PeelCtl *hctl)
{
	const uint64_t T = c.T;
	uint32_t *R = nullptr, *F0 = nullptr, *F1 = nullptr, *B0 = nullptr, *B1 = nullptr, *fbits = nullptr,
			 *fchunk = nullptr;
	uint8_t *destroyed = nullptr;
	CtlX *ctl = nullptr;
	GridBar *bar = nullptr;
	int rc = NUCLEUS34_OK;
	auto cleanup = [&] {
		c.release(R);
		c.release(F0);
		c.release(F1);
		c.release(B0);
		c.release(B1);
		c.release(fbits);
		c.release(fchunk);
		c.release(ctl);
		c.release(bar);
		c.release(destroyed);
	};
	// death flags live in the incidence entries when triangle ids leave the
	// top two bits free (the incidence is discarded after the peel)
	const bool flags = variant == NUCLEUS34_ONDEMAND && T <= ID_MASK && !(c.opt_flags & NUCLEUS34_OPT_STAMP_PEEL);
	// death rounds: the round-stamp owner test needs them; the death-flag
	// path records them only to keep them for nucleus34_ctx_verify
	const bool keep_rounds = (c.opt_flags & NUCLEUS34_OPT_VERIFIABLE) != 0;
	// Memory-lean peel (death-flag path only): frontiers as two bitmaps of T
	// bits instead of two lists of T ids, and, when the caller passes K == S,
	// k kept in S (a dead triangle holds -1 - k) and converted at the end.
	const bool lean = flags && c.lean_run;
	// level-change scans with vector loads unless the scalar ones are asked for
	const bool vec_scans = !(c.opt_flags & NUCLEUS34_OPT_SCALAR_SCANS);
	// chunked debit schedule (list frontiers) when asked for; the split one
	// (a thread per short-list triangle, a warp per long one) by default
	const bool chunked = !lean && (c.opt_flags & NUCLEUS34_OPT_CHUNKED_DEBIT);
	// software-pipelined warp debit (list frontiers) when asked for
	const bool pipelined = !lean && !chunked && (c.opt_flags & NUCLEUS34_OPT_PIPELINED_DEBIT);
	// warp debit on one wave that claims frontier positions from a cursor
	const bool cursor = !chunked && !pipelined && (c.opt_flags & NUCLEUS34_OPT_DEBIT_CURSOR);
	const bool k_in_s = (K == S);
	int32_t *Kw = k_in_s ? nullptr : K;
	const uint64_t fwords = (T + 31) / 32;
	// scheduling settings of this run (identical results for any of them)
	const nucleus34_tune tn = tune_filled(c.tune);
	const bool sort_on = tn.sort_shift != NUCLEUS34_TUNE_NEVER;
	const unsigned long long sort_min =
		sort_on ? std::max<unsigned long long>(T >> tn.sort_shift, N34_SORT_MIN) : ~0ull;
	const uint32_t compact_div = tn.compact_div == NUCLEUS34_TUNE_NEVER ? 0u : tn.compact_div;
	const uint32_t rpr = tn.rounds_per_replay;
	do
	{
		if (k_in_s && !lean)
		{
			rc = fail(NUCLEUS34_E_INVALID, "internal: k kept in S outside the lean peel");
			break;
		}
		if ((!flags || keep_rounds) && (rc = dalloc(c, &R, T, "peel round stamps")))
			break;
		if (lean)
		{
			if ((rc = dalloc(c, &B0, fwords, "frontier bitmap 0")) || (rc = dalloc(c, &B1, fwords, "frontier bitmap 1")))
				break;
			if (cudaMemsetAsync(B0, 0, fwords * 4, c.stream) != cudaSuccess ||
				cudaMemsetAsync(B1, 0, fwords * 4, c.stream) != cudaSuccess)
			{
				rc = fail(NUCLEUS34_E_CUDA, "memset");
				break;
			}
		}
		else
		{
			if ((rc = dalloc(c, &F0, T, "frontier 0")))
				break;
			if ((rc = dalloc(c, &F1, T, "frontier 1")))
				break;
		}
		const Frontier fr{F0, F1, B0, B1, fwords};
		if ((rc = dalloc(c, &ctl, 1, "peel control")))
			break;
		// Small cascade rounds in one cooperative launch (death-flag peel with
		// list frontiers; not in profiling mode, whose per-step events need the
		// separate kernels).
		const bool profile_mode = (c.opt_flags & NUCLEUS34_OPT_PROFILE_PEEL) != 0;
		uint32_t gsmall = 0;
		if (flags && !lean && !profile_mode && !(c.opt_flags & NUCLEUS34_OPT_NO_SMALL_ROUNDS))
		{
			int coop = 0;
			if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c.device) != cudaSuccess)
				coop = 0;
			cudaGetLastError();
			if (coop)
				gsmall = tn.lane_max == 8	 ? small_rounds_grid<8>(c.sm_count)
						 : tn.lane_max == 32 ? small_rounds_grid<32>(c.sm_count)
											 : small_rounds_grid<THREAD_MODE_MAX>(c.sm_count);
		}
		if (gsmall)
		{
			if ((rc = dalloc(c, &bar, 1, "peel grid barrier")))
				break;
			if (cudaMemsetAsync(bar, 0, sizeof(GridBar), c.stream) != cudaSuccess)
			{
				rc = fail(NUCLEUS34_E_CUDA, "memset");
				break;
			}
		}
		const uint32_t small_max =
			uint32_t(std::min<unsigned long long>(N34_SMALL_MAX, sort_min > 0 ? sort_min - 1 : 0));
		// frontier ordering bitmap (optional: skipped without room for it;
		// a bitmap frontier is in id order already)
		// keyed by the c-edge entry position (3T keys) when asked and the entry
		// positions exist (death-flag peel), else by triangle id (T keys)
		const bool order_by_c = flags && inc.tpos && (c.opt_flags & NUCLEUS34_OPT_FRONTIER_BY_C);
		const uint64_t fkeys = order_by_c ? 3 * T : T;
		const uint64_t skeys_words = (fkeys + 31) / 32;
		const uint64_t fchunks = (skeys_words + SORT_CHUNK_WORDS - 1) / SORT_CHUNK_WORDS;
		if (!sort_on || lean || (c.opt_flags & NUCLEUS34_OPT_LEAN_MEMORY) ||
			dalloc(c, &fbits, skeys_words, "frontier order bitmap") ||
			dalloc(c, &fchunk, fchunks, "frontier order chunks"))
		{
			c.release(fbits);
			c.release(fchunk);
			fbits = nullptr;
			fchunk = nullptr;
			clear_error();
		}
		else if (cudaMemsetAsync(fbits, 0, skeys_words * 4, c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "memset");
			break;
		}
		const uint32_t gsort = uint32_t(std::min<uint64_t>(fchunks, uint64_t(c.sm_count) * 8));
		if (variant == NUCLEUS34_DIRECT)
		{
			if ((rc = dalloc(c, &destroyed, c.Q ? c.Q : 1, "clique destroyed flags")))
				break;
			if (cudaMemsetAsync(destroyed, 0, c.Q ? c.Q : 1, c.stream) != cudaSuccess)
			{
				rc = fail(NUCLEUS34_E_CUDA, "memset");
				break;
			}
		}
		const uint32_t gscan = grid_for(c, T, PEEL_THREADS, 8);
		const uint32_t gwarp = grid_for(c, T, PEEL_THREADS / 32, 16);
		k_peel_init<<<gscan, PEEL_THREADS, 0, c.stream>>>(Kw, T, ctl, compact_div, sort_min);
		c.launches++;
		{
			const uint32_t on = (c.opt_flags & NUCLEUS34_OPT_PROFILE_PEEL) ? 1u : 0u;
			if (cudaMemcpyAsync(&ctl->stats, &on, 4, cudaMemcpyHostToDevice, c.stream) != cudaSuccess)
			{
				rc = fail(NUCLEUS34_E_CUDA, "peel control");
				break;
			}
		}
		// Profiling (NUCLEUS34_OPT_PROFILE_PEEL): rounds run as plain launches
		// with an event after every step; per-step totals go to stderr.
		const bool profile = (c.opt_flags & NUCLEUS34_OPT_PROFILE_PEEL) != 0;
		constexpr int PROF_STEPS = 8;
		static const char *const prof_names[PROF_STEPS] = {"gather_next", "scan_min", "gather",	   "mark",
														   "debit_thread", "debit_warp", "finalize", "order+advance"};
		// One round = a fixed kernel sequence that reads its sizes from ctl.
		auto launch_round = [&](cudaEvent_t *ev, uint32_t *trace) {
			auto tick = [&](int j) {
				if (ev)
					cudaEventRecord(ev[j], c.stream);
			};
			if (gsmall)
			{
				const uint32_t lm = tn.lane_max;
				if (lm == 8)
					launch_small_rounds<8>(c.stream, gsmall, ctl, bar, fr, c.dtris, c.dsrc, c.dE, inc, Kw, S, R, T,
										   small_max);
				else if (lm == 32)
					launch_small_rounds<32>(c.stream, gsmall, ctl, bar, fr, c.dtris, c.dsrc, c.dE, inc, Kw, S, R, T,
											small_max);
				else
					launch_small_rounds<THREAD_MODE_MAX>(c.stream, gsmall, ctl, bar, fr, c.dtris, c.dsrc, c.dE, inc,
														 Kw, S, R, T, small_max);
			}
			tick(0);
			k_gather_next<<<gscan, PEEL_THREADS, 0, c.stream>>>(ctl, S, T, fr, vec_scans);
			tick(1);
			k_scan_min<<<gscan, PEEL_THREADS, 0, c.stream>>>(ctl, S, T, vec_scans);
			tick(2);
			k_gather<<<gscan, PEEL_THREADS, 0, c.stream>>>(ctl, S, T, fr, vec_scans);
			tick(3);
			if (trace)
				cudaMemcpyAsync(trace, &ctl->c, 3 * sizeof(uint32_t), cudaMemcpyDeviceToHost, c.stream);
			if (flags)
			{
				k_mark_flags<<<gscan, PEEL_THREADS, 0, c.stream>>>(ctl, fr, Kw, S, c.dtris, c.dsrc, c.dE, inc.span,
																   inc.third, inc.tpos, inc.tri, 3 * T, R);
				tick(4);
				cudaEvent_t ev5 = ev ? ev[5] : nullptr;
				static_assert(THREAD_MODE_MAX == TUNE_LANE_MAX, "default lane/warp split");
				if (tn.lane_max == 8)
					launch_debit_flags<8>(c.stream, gscan, gwarp, lean, ctl, fr, c.dtris, inc, S, T, ev5, chunked,
											pipelined, cursor);
				else if (tn.lane_max == 32)
					launch_debit_flags<32>(c.stream, gscan, gwarp, lean, ctl, fr, c.dtris, inc, S, T, ev5, chunked,
											pipelined, cursor);
				else
					launch_debit_flags<THREAD_MODE_MAX>(c.stream, gscan, gwarp, lean, ctl, fr, c.dtris, inc, S, T,
														ev5, chunked, pipelined, cursor);
				tick(6);
				k_finalize_flags<<<gscan, PEEL_THREADS, 0, c.stream>>>(ctl, fr, c.dtris, c.dsrc, c.dE, inc.span,
																	   inc.third, inc.tpos, inc.tri, 3 * T);
				tick(7);
			}
			else
			{
				k_mark<<<gscan, PEEL_THREADS, 0, c.stream>>>(ctl, F0, F1, K, R, S);
				tick(4);
				if (variant == NUCLEUS34_ONDEMAND)
					k_debit_ondemand<<<gwarp, PEEL_THREADS, 0, c.stream>>>(ctl, F0, F1, c.dtris, inc.span, inc.third,
																		   inc.tri, K, R, S, T);
				else
					k_debit_direct<<<gwarp, PEEL_THREADS, 0, c.stream>>>(
						ctl, F0, F1, csr.off, csr.ids, reinterpret_cast<const uint4 *>(c.dquds), K, R, S, destroyed,
						T);
				tick(5);
				tick(6);
				tick(7);
			}
			if (fbits)
			{
				k_fsort_set<<<gscan, PEEL_THREADS, 0, c.stream>>>(ctl, F0, F1, fbits, T,
																  order_by_c ? inc.tpos : nullptr, fkeys);
				k_fsort_count<<<gsort, SORT_THREADS, 0, c.stream>>>(ctl, fbits, skeys_words, fchunk, T);
				k_fsort_scan<<<1, 1024, 0, c.stream>>>(ctl, fchunk, fchunks, T);
				k_fsort_write<<<gsort, SORT_THREADS, 0, c.stream>>>(ctl, fbits, skeys_words, fchunk, F0, F1, T,
																	order_by_c ? inc.tri : nullptr);
			}
			k_advance<<<1, 1, 0, c.stream>>>(ctl);
			if (ev)
				cudaEventRecord(ev[PROF_STEPS], c.stream);
		};
		const uint32_t per_round = (flags ? 8u : 6u) + (fbits ? 4u : 0u) + (gsmall ? 1u : 0u);
		const uint32_t gcompact = grid_for(c, c.m, PEEL_THREADS / 32, 16);
		// after every rpr rounds: the gated in-place compaction
		const bool compaction = flags && compact_div != 0;
		auto launch_compaction = [&]() {
			if (!compaction)
				return;
			k_compact_gate<<<1, 1, 0, c.stream>>>(ctl, T);
			k_compact_spans<<<gcompact, PEEL_THREADS, 0, c.stream>>>(ctl, inc.span, c.m, inc.third, inc.tri,
																	  inc.tpos);
		};
		const uint32_t per_replay = compaction ? 2u : 0u;
		// Bounds of the peel: every round that is not a no-op peels at least
		// one triangle, so T + 1 rounds suffice; the bound leaves a wide margin.
		const uint64_t max_rounds = 2 * T + 4096;
		const uint32_t max_rounds32 = uint32_t(std::min<uint64_t>(max_rounds, 0xfffffff0ull));
		const unsigned long long limit_ns = (c.opt_flags & NUCLEUS34_OPT_PROFILE_PEEL) ? ~0ull : PEEL_TIME_LIMIT_NS;
		uint64_t rounds = 0;
		// Device loop: one CUDA graph whose while node repeats a body of rpr
		// rounds, the compaction and k_loop_cond, which ends the loop when the
		// peel is done, a device check failed, or a bound was reached. The host
		// launches it once and waits once: no host round trip between rounds.
		cudaGraph_t loop_graph = nullptr;
		cudaGraphExec_t loop_exec = nullptr;
		bool device_loop = false;
		if (!profile && !(c.opt_flags & NUCLEUS34_OPT_HOST_LOOP))
		{
			cudaGraphConditionalHandle cond{};
			cudaGraphNodeParams cp{};
			cudaGraphNode_t cnode = nullptr;
			if (cudaGraphCreate(&loop_graph, 0) == cudaSuccess &&
				cudaGraphConditionalHandleCreate(&cond, loop_graph, 1, cudaGraphCondAssignDefault) == cudaSuccess)
			{
				cp.type = cudaGraphNodeTypeConditional;
				cp.conditional.handle = cond;
				cp.conditional.type = cudaGraphCondTypeWhile;
				cp.conditional.size = 1;
				if (cudaGraphAddNode(&cnode, loop_graph, nullptr, 0, &cp) == cudaSuccess &&
					cudaStreamBeginCaptureToGraph(c.stream, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
												  cudaStreamCaptureModeThreadLocal) == cudaSuccess)
				{
					for (uint32_t r = 0; r < rpr; ++r)
						launch_round(nullptr, nullptr);
					launch_compaction();
					k_loop_cond<<<1, 1, 0, c.stream>>>(ctl, cond, max_rounds32, limit_ns);
					cudaGraph_t body = nullptr;
					device_loop = cudaStreamEndCapture(c.stream, &body) == cudaSuccess &&
								  cudaGraphInstantiate(&loop_exec, loop_graph, 0) == cudaSuccess;
				}
			}
			cudaGetLastError();
			if (!device_loop)
			{
				if (loop_exec)
					cudaGraphExecDestroy(loop_exec);
				loop_exec = nullptr;
			}
		}
		if (device_loop)
		{
			if (cudaGraphLaunch(loop_exec, c.stream) != cudaSuccess ||
				cudaStreamSynchronize(c.stream) != cudaSuccess)
				rc = fail(NUCLEUS34_E_CUDA, std::string("peel device loop: ") + cudaGetErrorString(cudaGetLastError()));
			CtlX hx{};
			if (!rc && cudaMemcpy(&hx, ctl, sizeof(CtlX), cudaMemcpyDeviceToHost) != cudaSuccess)
				rc = fail(NUCLEUS34_E_CUDA, "peel control");
			if (!rc && std::getenv("NUCLEUS34_PEEL_VERBOSE"))
				std::fprintf(stderr, "[peel] rounds=%u peeling_rounds=%u small_rounds=%u loop_passes=%u compactions=%u\n",
							 hx.c.round, hx.c.rounds, hx.small_rounds, hx.loop_passes, hx.compactions);
			if (!rc)
			{
				rounds = hx.c.round;
				c.launches += (uint64_t(rounds + rpr - 1) / rpr) * (uint64_t(rpr) * per_round + per_replay + 1);
				if (hx.timed_out || (!hx.c.done && !hx.c.error))
					rc = fail(NUCLEUS34_E_TIMEOUT, "peel did not converge within its round and time bounds");
			}
			cudaGraphExecDestroy(loop_exec);
			cudaGraphDestroy(loop_graph);
			loop_graph = nullptr;
			if (rc)
				break;
		}
		if (loop_graph)
			cudaGraphDestroy(loop_graph);
		// Host loop (profiling, or where the device loop could not be built):
		// rounds are replayed from a CUDA graph of rpr rounds; the host reads
		// the control block once per replay. Rounds after the last one are
		// no-ops.
		cudaGraph_t graph = nullptr;
		cudaGraphExec_t exec = nullptr;
		bool use_graph = !device_loop && !profile &&
						 cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
		if (use_graph)
		{
			for (uint32_t r = 0; r < rpr; ++r)
				launch_round(nullptr, nullptr);
			launch_compaction();
			use_graph = cudaStreamEndCapture(c.stream, &graph) == cudaSuccess && graph &&
						cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
		}
		cudaGetLastError();
		std::vector<cudaEvent_t> events;
		double prof_ms[PROF_STEPS] = {};
		uint32_t *trace_buf = nullptr; // (level, round, frontier size) per round
		if (profile)
		{
			if (cudaMallocHost(&trace_buf, 3 * sizeof(uint32_t) * rpr) != cudaSuccess)
			{
				trace_buf = nullptr; // profile without the per-round lines
				cudaGetLastError();
			}
			events.resize(size_t(rpr) * (PROF_STEPS + 1));
			for (auto &e : events)
				cudaEventCreate(&e);
		}
		// The next replay is queued before the host reads the control block of
		// the previous one (pinned ring of two), so the GPU never waits on the
		// host; after the last round the queued replay is all no-ops.
		PeelCtl *ring = nullptr;
		cudaEvent_t ring_ev[2] = {nullptr, nullptr};
		if (!device_loop &&
			(cudaMallocHost(&ring, 2 * sizeof(PeelCtl)) != cudaSuccess ||
			 cudaEventCreateWithFlags(&ring_ev[0], cudaEventDisableTiming) != cudaSuccess ||
			 cudaEventCreateWithFlags(&ring_ev[1], cudaEventDisableTiming) != cudaSuccess))
			rc = fail(NUCLEUS34_E_CUDA, "peel control ring");
		auto enqueue = [&](int slot) -> bool {
			if (use_graph)
			{
				if (cudaGraphLaunch(exec, c.stream) != cudaSuccess)
					return false;
			}
			else
			{
				for (uint32_t r = 0; r < rpr; ++r)
					launch_round(profile ? &events[size_t(r) * (PROF_STEPS + 1)] : nullptr,
								 trace_buf ? trace_buf + 3 * r : nullptr);
				launch_compaction();
			}
			rounds += rpr;
			c.launches += uint64_t(rpr) * per_round + per_replay;
			return cudaMemcpyAsync(&ring[slot], &ctl->c, sizeof(PeelCtl), cudaMemcpyDeviceToHost, c.stream) ==
					   cudaSuccess &&
				   cudaEventRecord(ring_ev[slot], c.stream) == cudaSuccess;
		};
		// profiling reads per-round events, so it runs one replay at a time
		const int depth = profile ? 1 : 2;
		uint64_t issued = 0, consumed = 0;
		while (!rc && !device_loop && issued < uint64_t(depth))
		{
			if (!enqueue(int(issued & 1)))
				rc = fail(NUCLEUS34_E_CUDA, "peel replay launch");
			++issued;
		}
		while (!rc && !device_loop)
		{
			const int slot = int(consumed & 1);
			if (cudaEventSynchronize(ring_ev[slot]) != cudaSuccess || cudaGetLastError() != cudaSuccess)
			{
				rc = fail(NUCLEUS34_E_CUDA, std::string("peel rounds: ") + cudaGetErrorString(cudaGetLastError()));
				break;
			}
			const PeelCtl hc = ring[slot];
			++consumed;
			if (profile)
			{
				for (uint32_t r = 0; r < rpr; ++r)
				{
					const uint32_t *tr = trace_buf ? trace_buf + 3 * r : nullptr;
					if (tr && !tr[2])
						continue; // no-op round
					if (tr)
						std::fprintf(stderr, "[peel-round] level=%u round=%u frontier=%u", tr[0], tr[1], tr[2]);
					for (int j = 0; j < PROF_STEPS; ++j)
					{
						float ms = 0;
						const size_t b = size_t(r) * (PROF_STEPS + 1);
						if (cudaEventElapsedTime(&ms, events[b + j], events[b + j + 1]) == cudaSuccess)
							prof_ms[j] += ms;
						if (tr)
							std::fprintf(stderr, " %.3f", ms);
					}
					if (tr)
						std::fprintf(stderr, "\n");
				}
				cudaGetLastError();
			}
			if (hc.done)
				break;
			if (rounds > max_rounds)
			{
				rc = fail(NUCLEUS34_E_TIMEOUT, "peel did not converge within its round bound");
				break;
			}
			if (!enqueue(int(issued & 1)))
			{
				rc = fail(NUCLEUS34_E_CUDA, "peel replay launch");
				break;
			}
			++issued;
		}
		// the replay still queued (no-op rounds) completes before the stats
		if (cudaStreamSynchronize(c.stream) != cudaSuccess && !rc)
			rc = fail(NUCLEUS34_E_CUDA, "peel drain");
		for (auto &e : ring_ev)
			if (e)
				cudaEventDestroy(e);
		if (ring)
			cudaFreeHost(ring);
		for (auto &e : events)
			cudaEventDestroy(e);
		if (trace_buf)
			cudaFreeHost(trace_buf);
		if (profile)
		{
			CtlX hx{};
			cudaMemcpy(&hx, ctl, sizeof(CtlX), cudaMemcpyDeviceToHost);
			if (N34_PEEL_STATS)
				std::fprintf(stderr,
						 "[peel-counters] warp-debit triangles=%llu merged_entries=%llu merge_steps=%llu lookups=%llu "
						 "resolves=%llu staged_resolves=%llu found_on_c=%llu\n",
						 hx.st_tri, hx.st_merge_entries, hx.st_steps, hx.st_lookups, hx.st_resolves, hx.st_staged,
						 hx.st_found);
			std::fprintf(stderr, "[peel-profile] rounds=%llu compactions=%u", (unsigned long long)rounds,
						 hx.compactions);
			for (int j = 0; j < PROF_STEPS; ++j)
				std::fprintf(stderr, " %s=%.1fms", prof_names[j], prof_ms[j]);
			std::fprintf(stderr, "\n");
			// steps 4 and 5: the debit kernels (thread + warp, or the single
			// stamp/direct debit in slot 4)
			c.peel_debit_sec = (prof_ms[4] + prof_ms[5]) * 1e-3;
		}
		if (exec)
			cudaGraphExecDestroy(exec);
		if (graph)
			cudaGraphDestroy(graph);
		if (rc)
			break;
		if (k_in_s)
		{
			// -1 - k of every peeled triangle back to k (unpeeled ones stay negative)
			k_s_to_k<<<gscan, PEEL_THREADS, 0, c.stream>>>(S, T);
			c.launches++;
		}
		k_stats<<<gscan, PEEL_THREADS, 0, c.stream>>>(ctl, K, T);
		c.launches++;
		if (cudaMemcpyAsync(hctl, &ctl->c, sizeof(PeelCtl), cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaStreamSynchronize(c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "peel stats");
			break;
		}
		if (hctl->error & 4u)
		{
			rc = fail(NUCLEUS34_E_TIMEOUT, "peel: a grid barrier of the small-round kernel ran past its time bound");
			break;
		}
		if (hctl->error)
		{
			rc = fail(NUCLEUS34_E_CUDA, "internal: peel check failed (" +
									   std::string(hctl->error & 2u ? "compaction bound" : "frontier overflow") + ")");
			break;
		}
		if (keep_rounds)
		{
			c.dR = R; // kept for nucleus34_ctx_verify
			R = nullptr;
		}
	} while (false);
	cleanup();
	return rc;
}

} // namespace n34

// Four-clique support per triangle, and the direct variant's clique list and
// triangle -> clique CSR.
//
// Reference: count_support (nucleus/cuNucleus34_ondemand.cu:176-194) counts
// cliques per triangle through the 3-way zipper; the direct program lists the
// cliques over the triangle graph (cu_cliques_quds, nucleus/utils.cuh:550-619)
// in atomic order and builds the triangle -> clique incidence by
// sort_by_key + lower_bound (cuNucleus34.cu:627-669).
//
// Here: the two shortest incidence lists of each triangle are intersected
// (intersect.cuh) by one lane (short lists) or one warp (tile merge).
// Every clique is listed once, by its lowest triangle id, in ascending order of
// its fourth vertex: a count pass, a scan and a write pass give a
// deterministic clique order with no sort. The triangle -> clique CSR uses the
// supports as counts (support[t] = cliques on t), a scan, and an atomic
// scatter of clique ids (the order inside a triangle's list does not affect
// the peel result).
#include "intersect.cuh"
#include "pipeline.cuh"

namespace n34 {

namespace {

constexpr int SUP_THREADS = 256;

struct TriEdges
{
	uint32_t b0, e0, b1, e1, b2, e2;
};

__device__ __forceinline__ TriEdges tri_lists(const uint32_t *__restrict__ tris, const uint2 *__restrict__ span,
											  uint64_t t)
{
	const uint32_t a = __ldg(tris + 3 * t + 0), b = __ldg(tris + 3 * t + 1), c = __ldg(tris + 3 * t + 2);
	const uint2 sa = __ldg(span + a), sb = __ldg(span + b), sc = __ldg(span + c);
	return TriEdges{sa.x, sa.y, sb.x, sb.y, sc.x, sc.y};
}

__device__ __forceinline__ Lists tri_order(const uint32_t *__restrict__ tris, const uint2 *__restrict__ span,
										   uint64_t t)
{
	const TriEdges E = tri_lists(tris, span, t);
	return order_lists(E.b0, E.e0, E.b1, E.e1, E.b2, E.e2);
}

// Support count. Each warp takes 32 consecutive triangles, one per lane: a
// lane whose shortest list is short intersects its two shortest lists alone;
// the warp then intersects the remaining triangles one at a time (tile merge,
// or binary search when the lists are very unequal). With WITH_OWN it also
// counts the cliques whose lowest triangle id is t (the direct variant's
// clique-list sizes); that needs the partner on the longest list too, found
// by a forward-moving binary search. LANE_MAX is the shortest-list length up
// to which a lane works alone (any value gives the same counts).
template <uint32_t LANE_MAX, bool WITH_OWN>
__global__ void __launch_bounds__(SUP_THREADS, 4) k_support(const uint32_t *__restrict__ tris, uint64_t T,
															const uint2 *__restrict__ span,
															const uint32_t *__restrict__ third,
															const uint32_t *__restrict__ itri,
															int32_t *__restrict__ support, uint32_t *__restrict__ own,
															unsigned long long *__restrict__ total)
{
	const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
	const uint32_t lane = lane_id();
	unsigned long long acc = 0;
	for (uint64_t base = warp * 32; base < T; base += nwarps * 32)
	{
		const uint64_t t = base + lane;
		const bool valid = t < T;
		Lists L{};
		if (valid)
			L = tri_order(tris, span, t);
		const bool small = valid && L.a1 - L.a0 <= LANE_MAX;
		if (small)
		{
			uint32_t cnt = 0, mine = 0, lo_c = L.c0;
			lane_intersect2(third, L, [&](uint32_t x, uint32_t pa, uint32_t pb) {
				++cnt;
				if (WITH_OWN)
				{
					lo_c = lower_bound32(third, lo_c, L.c1, x);
					mine += uint32_t(t) < __ldg(itri + pa) && uint32_t(t) < __ldg(itri + pb) &&
							uint32_t(t) < __ldg(itri + lo_c);
				}
			});
			support[t] = int32_t(cnt);
			if (WITH_OWN)
				own[t] = mine;
			acc += cnt;
		}
		uint32_t large = __ballot_sync(FULL, valid && !small);
		while (large)
		{
			const int j = __ffs(large) - 1;
			large &= large - 1;
			const uint32_t tj = uint32_t(base) + uint32_t(j);
			const Lists Lj{__shfl_sync(FULL, L.a0, j), __shfl_sync(FULL, L.a1, j), __shfl_sync(FULL, L.b0, j),
						   __shfl_sync(FULL, L.b1, j), __shfl_sync(FULL, L.c0, j), __shfl_sync(FULL, L.c1, j)};
			uint32_t cnt = 0, mine = 0, lo_c = Lj.c0;
			warp_intersect2<WITH_OWN>(third, itri, Lj, [&](bool found, uint32_t x, uint32_t, uint32_t, uint32_t qa,
														   uint32_t qb) {
				const uint32_t fm = __ballot_sync(FULL, found);
				cnt += __popc(fm);
				if (WITH_OWN && fm)
				{
					// the longest list is searched only where t is below the other two
					const bool cand = found && tj < qa && tj < qb;
					const uint32_t pc = warp_lower_bound(third, lo_c, Lj.c1, cand, x);
					const bool m = cand && pc < Lj.c1 && tj < __ldg(itri + pc);
					mine += __popc(__ballot_sync(FULL, m));
					const uint32_t cm = __ballot_sync(FULL, cand);
					if (cm)
						lo_c = __shfl_sync(FULL, pc, 31 - __clz(cm));
				}
			});
			if (lane == uint32_t(j))
			{
				support[tj] = int32_t(cnt);
				if (WITH_OWN)
					own[tj] = mine;
				acc += cnt;
			}
		}
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		acc += __shfl_xor_sync(FULL, acc, o);
	if (lane == 0 && acc)
		atomicAdd(total, acc);
}

__device__ __forceinline__ void sort3(uint32_t &a, uint32_t &b, uint32_t &c)
{
	uint32_t t;
	if (a > b)
	{
		t = a;
		a = b;
		b = t;
	}
	if (b > c)
	{
		t = b;
		b = c;
		c = t;
	}
	if (a > b)
	{
		t = a;
		a = b;
		b = t;
	}
}

// Writes each triangle's owned cliques (lowest member t) at qoff[t], in
// ascending fourth-vertex order; same hybrid thread/warp split as k_support.
__global__ void __launch_bounds__(SUP_THREADS, 4) k_clique_write(const uint32_t *__restrict__ tris, uint64_t T,
																 const uint2 *__restrict__ span,
																 const uint32_t *__restrict__ third,
																 const uint32_t *__restrict__ itri,
																 const uint64_t *__restrict__ qoff,
																 uint4 *__restrict__ quds)
{
	const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
	const uint32_t lane = lane_id();
	for (uint64_t base = warp * 32; base < T; base += nwarps * 32)
	{
		const uint64_t t = base + lane;
		bool work = false;
		Lists L{};
		uint64_t out = 0, out_end = 0;
		if (t < T)
		{
			out = qoff[t];
			out_end = qoff[t + 1];
			work = out < out_end;
			if (work)
				L = tri_order(tris, span, t);
		}
		const bool small = work && L.a1 - L.a0 <= THREAD_MODE_MAX;
		if (small)
		{
			uint32_t lo_c = L.c0;
			lane_intersect2(third, L, [&](uint32_t x, uint32_t pa, uint32_t pb) {
				lo_c = lower_bound32(third, lo_c, L.c1, x);
				uint32_t q0 = __ldg(itri + pa), q1 = __ldg(itri + pb), q2 = __ldg(itri + lo_c);
				if (uint32_t(t) < q0 && uint32_t(t) < q1 && uint32_t(t) < q2 && out < out_end)
				{
					sort3(q0, q1, q2);
					quds[out++] = make_uint4(uint32_t(t), q0, q1, q2);
				}
			});
		}
		uint32_t large = __ballot_sync(FULL, work && !small);
		while (large)
		{
			const int j = __ffs(large) - 1;
			large &= large - 1;
			const uint32_t tj = uint32_t(base) + uint32_t(j);
			uint64_t o = __shfl_sync(FULL, out, j);
			const uint64_t oe = __shfl_sync(FULL, out_end, j);
			const Lists Lj{__shfl_sync(FULL, L.a0, j), __shfl_sync(FULL, L.a1, j), __shfl_sync(FULL, L.b0, j),
						   __shfl_sync(FULL, L.b1, j), __shfl_sync(FULL, L.c0, j), __shfl_sync(FULL, L.c1, j)};
			uint32_t lo_c = Lj.c0;
			warp_intersect2<true>(third, itri, Lj, [&](bool found, uint32_t x, uint32_t, uint32_t, uint32_t qa,
													   uint32_t qb) {
				// the longest list is searched only where t is below the other two
				const bool cand = found && tj < qa && tj < qb;
				const uint32_t cm = __ballot_sync(FULL, cand);
				if (!cm)
					return;
				const uint32_t pc = warp_lower_bound(third, lo_c, Lj.c1, cand, x);
				lo_c = __shfl_sync(FULL, pc, 31 - __clz(cm));
				uint32_t q0 = qa, q1 = qb, q2 = 0;
				bool mine = false;
				if (cand && pc < Lj.c1)
				{
					q2 = __ldg(itri + pc);
					mine = tj < q2;
				}
				const uint32_t word = __ballot_sync(FULL, mine);
				const uint64_t at = o + __popc(word & lanemask_lt());
				if (mine && at < oe) // capacity guard (the count pass sized it)
				{
					sort3(q0, q1, q2);
					quds[at] = make_uint4(tj, q0, q1, q2);
				}
				o += __popc(word);
			});
		}
	}
}

__global__ void k_clique_fill(const uint4 *__restrict__ quds, uint64_t Q, const uint64_t *__restrict__ coff,
							  uint32_t *__restrict__ cursor, uint32_t *__restrict__ ids, uint32_t *__restrict__ err)
{
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t q = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < Q; q += stride)
	{
		const uint4 x = quds[q];
		const uint32_t m4[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
		for (int r = 0; r < 4; ++r)
		{
			const uint64_t at = coff[m4[r]] + atomicAdd(cursor + m4[r], 1u);
			// capacity guard: counts are the supports, which list every clique of t once
			if (at < coff[m4[r] + 1])
				ids[at] = uint32_t(q);
			else
				atomicOr(err, 1u);
		}
	}
}

} // namespace

int count_support(Ctx &c, const Incidence &inc, int32_t *support, uint64_t *total, uint32_t *own)
{
	unsigned long long *dtot = nullptr;
	N34_TRY(dalloc(c, &dtot, 1, "support total"));
	int rc = NUCLEUS34_OK;
	do
	{
		if (cudaMemsetAsync(dtot, 0, 8, c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "memset");
			break;
		}
		const uint32_t grid = grid_for(c, (c.T + 31) / 32, SUP_THREADS / 32, 32);
		static_assert(THREAD_MODE_MAX == TUNE_LANE_MAX, "default lane/warp split");
		if (own) // the direct variant: default split
			k_support<THREAD_MODE_MAX, true><<<grid, SUP_THREADS, 0, c.stream>>>(
				c.dtris, c.T, inc.span, inc.third, inc.tri, support, own, dtot);
		else if (c.tune.lane_max == 8)
			k_support<8, false><<<grid, SUP_THREADS, 0, c.stream>>>(c.dtris, c.T, inc.span, inc.third, inc.tri,
																	support, nullptr, dtot);
		else if (c.tune.lane_max == 32)
			k_support<32, false><<<grid, SUP_THREADS, 0, c.stream>>>(c.dtris, c.T, inc.span, inc.third, inc.tri,
																	 support, nullptr, dtot);
		else
			k_support<THREAD_MODE_MAX, false><<<grid, SUP_THREADS, 0, c.stream>>>(
				c.dtris, c.T, inc.span, inc.third, inc.tri, support, nullptr, dtot);
		c.launches++;
		unsigned long long h = 0;
		if (cudaGetLastError() != cudaSuccess ||
			cudaMemcpyAsync(&h, dtot, 8, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaStreamSynchronize(c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "support count");
			break;
		}
		*total = h;
	} while (false);
	c.release(dtot);
	return rc;
}

int list_cliques(Ctx &c, const Incidence &inc, const int32_t *support, const uint32_t *own, CliqueCsr &csr)
{
	const uint64_t T = c.T;
	uint32_t *cursor = nullptr, *errf = nullptr;
	uint64_t *qoff = nullptr;
	int rc = NUCLEUS34_OK;
	auto cleanup = [&] {
		c.release(cursor);
		c.release(qoff);
		c.release(errf);
	};
	do
	{
		if ((rc = dalloc(c, &qoff, T + 1, "clique offsets")))
			break;
		const uint32_t grid = grid_for(c, (T + 31) / 32, SUP_THREADS / 32, 32);
		if ((rc = scan_u32(c, own, qoff, T)))
			break;
		uint64_t Q = 0;
		if (cudaMemcpyAsync(&Q, qoff + T, 8, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaStreamSynchronize(c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "clique count");
			break;
		}
		if (Q > 0xffffffffull)
		{
			rc = fail(NUCLEUS34_E_RANGE32, "four-clique count " + std::to_string(Q) +
											   " exceeds the 32-bit clique id range of the direct variant; "
											   "use the on-demand variant");
			break;
		}
		c.Q = Q;
		if (Q == 0)
			break;
		if ((rc = dalloc(c, &c.dquds, 4 * Q, "four-cliques")))
			break;
		k_clique_write<<<grid, SUP_THREADS, 0, c.stream>>>(c.dtris, T, inc.span, inc.third, inc.tri, qoff,
														   reinterpret_cast<uint4 *>(c.dquds));
		c.launches++;
		c.release(qoff);
		qoff = nullptr;
		// triangle -> clique CSR: counts are the supports
		if ((rc = dalloc(c, &csr.off, T + 1, "clique csr offsets")))
			break;
		static_assert(sizeof(int32_t) == sizeof(uint32_t), "support layout");
		if ((rc = scan_u32(c, reinterpret_cast<const uint32_t *>(support), csr.off, T)))
			break;
		if ((rc = dalloc(c, &csr.ids, 4 * Q, "clique csr ids")))
			break;
		if ((rc = dalloc(c, &cursor, T, "clique csr cursor")))
			break;
		if ((rc = dalloc(c, &errf, 1, "clique check")))
			break;
		if (cudaMemsetAsync(cursor, 0, T * 4, c.stream) != cudaSuccess ||
			cudaMemsetAsync(errf, 0, 4, c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "memset");
			break;
		}
		k_clique_fill<<<grid_for(c, Q, 256), 256, 0, c.stream>>>(reinterpret_cast<const uint4 *>(c.dquds), Q,
																  csr.off, cursor, csr.ids, errf);
		c.launches++;
		uint32_t herr = 0;
		if (cudaGetLastError() != cudaSuccess ||
			cudaMemcpyAsync(&herr, errf, 4, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaStreamSynchronize(c.stream) != cudaSuccess)
			rc = fail(NUCLEUS34_E_CUDA, "clique kernels");
		else if (herr)
			rc = fail(NUCLEUS34_E_CUDA, "internal: clique incidence overflow");
	} while (false);
	cleanup();
	return rc;
}

void free_clique_csr(Ctx &c, CliqueCsr &csr)
{
	c.release(csr.off);
	c.release(csr.ids);
	csr = CliqueCsr{};
}

} // namespace n34

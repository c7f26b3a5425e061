// Certificate check of a finished peel (nucleus34_ctx_verify).
//
// With k(t) the reported number and r(t) the round in which t died:
//   (A) t lies in at least k(t) four-cliques whose other three triangles all
//       have k >= k(t): the triangles with k >= L then form a subgraph in
//       which each has >= L cliques, so every k is at most the true number;
//   (B) t lies in at most k(t) cliques whose other three triangles died in
//       r(t) or later (its support when its round began);
//   (C) all triangles of one round share one level, and the level never
//       decreases from round to round.
// (B) and (C) make every k at least the true number: in the true k*(t)-
// nucleus containing t, the first triangle to die had all of the nucleus
// alive, hence support >= k*(t) <= its level <= k(t). So the three together
// hold exactly when k equals the (3,4)-nucleus numbers. The check costs one
// enumeration of all cliques (the support count's pass) plus random reads of
// the partners' k and r.
#include "intersect.cuh"
#include "pipeline.cuh"

#include <vector>

namespace n34 {

namespace {

constexpr int VER_THREADS = 256;

__global__ void k_max_round(const uint32_t *__restrict__ R, uint64_t T, uint32_t *__restrict__ mx)
{
	uint32_t m = 0;
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < T; t += stride)
		m = max(m, R[t]);
#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		m = max(m, __shfl_xor_sync(FULL, m, o));
	if (lane_id() == 0)
		atomicMax(mx, m);
}

__global__ void k_round_levels(const int32_t *__restrict__ K, const uint32_t *__restrict__ R, uint64_t T,
							   uint32_t nrounds, int32_t *__restrict__ lvmin, int32_t *__restrict__ lvmax,
							   unsigned long long *__restrict__ bad)
{
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < T; t += stride)
	{
		const int32_t k = K[t];
		const uint32_t r = R[t];
		if (k < 0 || r >= nrounds)
			atomicAdd(bad, 1ull);
		else
		{
			atomicMin(lvmin + r, k);
			atomicMax(lvmax + r, k);
		}
	}
}

__global__ void __launch_bounds__(VER_THREADS) k_verify(const uint32_t *__restrict__ tris, uint64_t T,
														 const uint2 *__restrict__ span,
														 const uint32_t *__restrict__ third,
														 const uint32_t *__restrict__ itri,
														 const int32_t *__restrict__ K, const uint32_t *__restrict__ R,
														 unsigned long long *__restrict__ bad)
{
	const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
	for (uint64_t t = warp; t < T; t += nwarps)
	{
		const uint32_t a = __ldg(tris + 3 * t), b = __ldg(tris + 3 * t + 1), c = __ldg(tris + 3 * t + 2);
		const uint2 sa = __ldg(span + a), sb = __ldg(span + b), sc = __ldg(span + c);
		const Lists L = order_lists(sa.x, sa.y, sb.x, sb.y, sc.x, sc.y);
		const int32_t kt = K[t];
		const uint32_t rt = R[t];
		uint32_t cnt_a = 0, cnt_b = 0, lo_c = L.c0;
		const WarpSample cs = warp_sample(third, L.c0, L.c1);
		warp_intersect2<true>(third, itri, L, [&](bool found, uint32_t x, uint32_t, uint32_t, uint32_t qa,
												  uint32_t qb) {
			const uint32_t fm = __ballot_sync(FULL, found);
			if (!fm)
				return;
			const uint32_t pc = sampled_lower_bound(third, cs, lo_c, L.c1, found, x);
			lo_c = __shfl_sync(FULL, pc, 31 - __clz(fm));
			bool ok_a = false, ok_b = false;
			if (found && pc < L.c1)
			{
				const uint32_t qc = __ldg(itri + pc);
				const int32_t km = min(min(K[qa], K[qb]), K[qc]);
				ok_a = km >= kt;
				ok_b = R[qa] >= rt && R[qb] >= rt && R[qc] >= rt;
			}
			cnt_a += __popc(__ballot_sync(FULL, ok_a));
			cnt_b += __popc(__ballot_sync(FULL, ok_b));
		});
		if (lane_id() == 0 && (kt < 0 || int64_t(cnt_a) < int64_t(kt) || int64_t(cnt_b) > int64_t(kt)))
			atomicAdd(bad, 1ull);
	}
}

} // namespace

int verify(Ctx &c, uint64_t *violations, uint64_t *checked)
{
	if (!c.have_result)
		return fail(NUCLEUS34_E_STATE, "no result");
	if (c.T && !c.dR && c.Q + c.res.four_clique_count)
		return fail(NUCLEUS34_E_STATE, "death rounds were not kept: run with NUCLEUS34_OPT_VERIFIABLE");
	N34_CUDA(cudaSetDevice(c.device));
	*violations = 0;
	*checked = c.T;
	if (!c.T)
		return NUCLEUS34_OK;
	if (!c.dR)
	{
		// no cliques: every k must be 0
		std::vector<int32_t> k(c.T);
		N34_CUDA(cudaMemcpyAsync(k.data(), c.dK, c.T * 4, cudaMemcpyDeviceToHost, c.stream));
		N34_CUDA(cudaStreamSynchronize(c.stream));
		for (auto v : k)
			*violations += v != 0;
		return NUCLEUS34_OK;
	}
	uint32_t *mx = nullptr;
	int32_t *lv = nullptr;
	unsigned long long *bad = nullptr;
	Incidence inc;
	int rc = NUCLEUS34_OK;
	do
	{
		if ((rc = dalloc(c, &mx, 1, "verify round max")) || (rc = dalloc(c, &bad, 1, "verify counter")))
			break;
		if (cudaMemsetAsync(mx, 0, 4, c.stream) != cudaSuccess || cudaMemsetAsync(bad, 0, 8, c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "memset");
			break;
		}
		k_max_round<<<grid_for(c, c.T, 256), 256, 0, c.stream>>>(c.dR, c.T, mx);
		uint32_t hmx = 0;
		if (cudaMemcpyAsync(&hmx, mx, 4, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaStreamSynchronize(c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "verify rounds");
			break;
		}
		const uint32_t nrounds = hmx + 1;
		if ((rc = dalloc(c, &lv, 2 * uint64_t(nrounds), "verify round levels")))
			break;
		std::vector<int32_t> init(2 * size_t(nrounds));
		for (uint32_t r = 0; r < nrounds; ++r)
		{
			init[r] = INT32_MAX;
			init[nrounds + r] = -1;
		}
		if (cudaMemcpyAsync(lv, init.data(), init.size() * 4, cudaMemcpyHostToDevice, c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "verify init");
			break;
		}
		k_round_levels<<<grid_for(c, c.T, 256), 256, 0, c.stream>>>(c.dK, c.dR, c.T, nrounds, lv, lv + nrounds, bad);
		if ((rc = build_incidence(c, inc, false)))
			break;
		k_verify<<<grid_for(c, c.T, VER_THREADS / 32, 16), VER_THREADS, 0, c.stream>>>(
			c.dtris, c.T, inc.span, inc.third, inc.tri, c.dK, c.dR, bad);
		unsigned long long hbad = 0;
		if (cudaMemcpyAsync(init.data(), lv, init.size() * 4, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaMemcpyAsync(&hbad, bad, 8, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaStreamSynchronize(c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "verify kernels");
			break;
		}
		// (C): one level per round, non-decreasing
		int32_t prev = -1;
		for (uint32_t r = 0; r < nrounds; ++r)
		{
			const int32_t lo = init[r], hi = init[nrounds + r];
			if (hi < 0)
				continue; // nobody died in this round
			if (lo != hi || lo < prev)
				++hbad;
			prev = hi;
		}
		*violations = hbad;
	} while (false);
	free_incidence(c, inc);
	c.release(mx);
	c.release(lv);
	c.release(bad);
	return rc;
}

} // namespace n34

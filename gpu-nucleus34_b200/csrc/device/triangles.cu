// Triangle listing in canonical (a,b) order, written directly (no sort).
//
// Reference: cu_cliques_tris + intersect_lists (nucleus/utils.cuh:259-343) list
// triangles per vertex by a zipper against materialised length-2 paths
// (cu_multi_arrange, utils.cuh:515-548), append them in atomic order and sort
// them afterwards by tri_t::operator< (utils.cuh:98-101, 1901;
// cuNucleus34_ondemand.cu:499).
//
// Here: for a vertex u with out-list N+(u) of length d, the triangles with
// source u are exactly the pairs (ia, ib) of positions in N+(u) such that
// w = N+(u)[ia] is an out-neighbour of v = N+(u)[ib]; the triangle is
// (a = O[u]+ia, b = O[u]+ib, c = position of w in N+(v)). Enumerating pairs in
// row-major (ia, ib) order IS the canonical (a, b) order, because a and b are
// both out-edges of u and canonical order is u-major. One warp owns a vertex;
// 32 consecutive pairs form one ballot word. Pass 1 stores the ballot words
// (scratch bitmap) and counts; a scan gives each vertex its output offset;
// pass 2 walks the set bits and binary-searches c. When the bitmap would not
// fit the budget, pass 2 recomputes the membership tests instead.
#include "pipeline.cuh"

namespace n34 {

namespace {

constexpr int TRI_THREADS = 256;
constexpr int TRI_WARPS = TRI_THREADS / 32;

__global__ void __launch_bounds__(256) k_build_src(const uint32_t *__restrict__ O, uint64_t n,
												   uint32_t *__restrict__ src)
{
	const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
	for (uint64_t u = warp; u < n; u += nwarps)
	{
		const uint32_t b = O[u], e = O[u + 1];
		for (uint32_t j = b + lane_id(); j < e; j += 32)
			src[j] = uint32_t(u);
	}
}

// words[u] = ceil(d*d / 32)
__global__ void k_pair_words(const uint32_t *__restrict__ O, uint64_t n, uint64_t *__restrict__ words)
{
	const uint64_t u = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
	if (u < n)
	{
		const uint64_t d = O[u + 1] - O[u];
		words[u] = (d * d + 31) / 32;
	}
}

// Membership test of pair p of vertex u: is N+(u)[p / d] in N+(N+(u)[p % d])?
// Returns the position of w in E (c) or UINT32_MAX.
__device__ __forceinline__ void pair_split(uint64_t p, uint32_t d, uint32_t &ia, uint32_t &ib)
{
	if (p <= 0xffffffffull)
	{
		ia = uint32_t(p) / d;
		ib = uint32_t(p) - ia * d;
	}
	else
	{
		ia = uint32_t(p / d);
		ib = uint32_t(p - uint64_t(ia) * d);
	}
}

__device__ __forceinline__ uint32_t pair_test(const uint32_t *__restrict__ O, const uint32_t *__restrict__ E,
											  uint32_t ob, uint32_t d, uint64_t p)
{
	uint32_t ia, ib;
	pair_split(p, d, ia, ib);
	if (ia == ib)
		return UINT32_MAX;
	const uint32_t w = __ldg(E + ob + ia);
	const uint32_t v = __ldg(E + ob + ib);
	const uint32_t vb = __ldg(O + v), ve = __ldg(O + v + 1);
	const uint64_t pos = lower_bound_u32(E, vb, ve, w);
	return (pos < ve && __ldg(E + pos) == w) ? uint32_t(pos) : UINT32_MAX;
}

// Pass 1: per-vertex triangle counts (+ ballot words when bits != nullptr).
__global__ void __launch_bounds__(TRI_THREADS) k_tri_count(const uint32_t *__restrict__ O,
														   const uint32_t *__restrict__ E, uint64_t n,
														   const uint64_t *__restrict__ woff,
														   uint32_t *__restrict__ bits,
														   uint32_t *__restrict__ cnt)
{
	const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
	for (uint64_t u = warp; u < n; u += nwarps)
	{
		const uint32_t ob = O[u], d = O[u + 1] - ob;
		const uint64_t pairs = uint64_t(d) * d;
		uint32_t total = 0;
		uint64_t w = 0;
		for (uint64_t base = 0; base < pairs; base += 32, ++w)
		{
			const uint64_t p = base + lane_id();
			const bool hit = p < pairs && pair_test(O, E, ob, d, p) != UINT32_MAX;
			const uint32_t word = __ballot_sync(FULL, hit);
			if (bits && lane_id() == 0)
				bits[woff[u] + w] = word;
			total += __popc(word);
		}
		if (lane_id() == 0)
			cnt[u] = total;
	}
}

// Pass 2: emit (a,b,c) at toff[u] in row-major pair order = canonical order.
__global__ void __launch_bounds__(TRI_THREADS) k_tri_write(const uint32_t *__restrict__ O,
														   const uint32_t *__restrict__ E, uint64_t n,
														   const uint64_t *__restrict__ woff,
														   const uint32_t *__restrict__ bits,
														   const uint64_t *__restrict__ toff,
														   uint32_t *__restrict__ tris)
{
	const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
	for (uint64_t u = warp; u < n; u += nwarps)
	{
		const uint64_t out0 = toff[u], outN = toff[u + 1];
		if (out0 == outN)
			continue;
		const uint32_t ob = O[u], d = O[u + 1] - ob;
		const uint64_t pairs = uint64_t(d) * d;
		uint64_t out = out0;
		uint64_t w = 0;
		for (uint64_t base = 0; base < pairs && out < outN; base += 32, ++w)
		{
			const uint64_t p = base + lane_id();
			uint32_t word;
			uint32_t c = UINT32_MAX;
			if (bits)
			{
				word = bits[woff[u] + w]; // same value in every lane
				if ((word >> lane_id()) & 1u)
					c = pair_test(O, E, ob, d, p);
			}
			else
			{
				if (p < pairs)
					c = pair_test(O, E, ob, d, p);
				word = __ballot_sync(FULL, c != UINT32_MAX);
			}
			if ((word >> lane_id()) & 1u)
			{
				const uint64_t at = out + __popc(word & lanemask_lt());
				uint32_t ia, ib;
				pair_split(p, d, ia, ib);
				tris[3 * at + 0] = ob + ia;
				tris[3 * at + 1] = ob + ib;
				tris[3 * at + 2] = c;
			}
			out += __popc(word);
		}
	}
}

} // namespace

int build_src(Ctx &c)
{
	if (c.m == 0)
		return NUCLEUS34_OK;
	N34_LAUNCH(c, k_build_src, grid_for(c, c.n, TRI_WARPS), TRI_THREADS, 0, c.dO, c.n, c.dsrc);
	return NUCLEUS34_OK;
}

// Launch helpers for callers that manage their own memory (no context):
// pass 1 (counts only, no bitmap) and pass 2 (recomputing the membership tests).
cudaError_t launch_tri_count(const uint32_t *O, const uint32_t *E, uint64_t n, uint32_t *cnt, int sm_count,
							 cudaStream_t s)
{
	uint64_t g = (n + TRI_WARPS - 1) / TRI_WARPS;
	g = g > uint64_t(sm_count) * 32 ? uint64_t(sm_count) * 32 : (g ? g : 1);
	k_tri_count<<<uint32_t(g), TRI_THREADS, 0, s>>>(O, E, n, nullptr, nullptr, cnt);
	return cudaGetLastError();
}

cudaError_t launch_tri_write(const uint32_t *O, const uint32_t *E, uint64_t n, const uint64_t *toff,
							 uint32_t *tris, int sm_count, cudaStream_t s)
{
	uint64_t g = (n + TRI_WARPS - 1) / TRI_WARPS;
	g = g > uint64_t(sm_count) * 32 ? uint64_t(sm_count) * 32 : (g ? g : 1);
	k_tri_write<<<uint32_t(g), TRI_THREADS, 0, s>>>(O, E, n, nullptr, nullptr, toff, tris);
	return cudaGetLastError();
}

// Lists the triangles of the resident graph into c.dtris (3*T u32) and sets c.T.
int list_triangles(Ctx &c)
{
	c.T = 0;
	if (c.m == 0)
		return NUCLEUS34_OK;
	const uint64_t n = c.n;
	uint64_t *words = nullptr, *woff = nullptr, *toff = nullptr;
	uint32_t *cnt = nullptr, *bits = nullptr;
	int rc = NUCLEUS34_OK;
	auto cleanup = [&] {
		c.release(words);
		c.release(woff);
		c.release(toff);
		c.release(cnt);
		c.release(bits);
	};
	do
	{
		if ((rc = dalloc(c, &words, n, "pair words")))
			break;
		if ((rc = dalloc(c, &woff, n + 1, "pair word offsets")))
			break;
		k_pair_words<<<uint32_t((n + 255) / 256), 256, 0, c.stream>>>(c.dO, n, words);
		c.launches++;
		if ((rc = scan_u64(c, words, woff, n)))
			break;
		uint64_t nwords = 0;
		if (cudaMemcpyAsync(&nwords, woff + n, 8, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaStreamSynchronize(c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "pair word count");
			break;
		}
		c.release(words);
		words = nullptr;
		// The bitmap is a cache: skip it if it would take more than a quarter
		// of what the budget has left.
		const uint64_t room = c.budget > c.in_use ? c.budget - c.in_use : 0;
		if (nwords * 4 <= room / 4)
		{
			if (dalloc(c, &bits, nwords ? nwords : 1, "pair bitmap"))
			{
				bits = nullptr;
				fail(0, "");
			}
		}
		if ((rc = dalloc(c, &cnt, n, "triangle counts")))
			break;
		if ((rc = dalloc(c, &toff, n + 1, "triangle offsets")))
			break;
		const uint32_t grid = grid_for(c, n, TRI_WARPS, 32);
		k_tri_count<<<grid, TRI_THREADS, 0, c.stream>>>(c.dO, c.dE, n, woff, bits, cnt);
		c.launches++;
		if ((rc = scan_u32(c, cnt, toff, n)))
			break;
		uint64_t T = 0;
		if (cudaMemcpyAsync(&T, toff + n, 8, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaStreamSynchronize(c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "triangle count");
			break;
		}
		if (T > 0xffffffffull)
		{
			rc = fail(NUCLEUS34_E_RANGE32, "triangle count " + std::to_string(T) + " exceeds 32-bit triangle ids");
			break;
		}
		c.T = T;
		if (T == 0)
			break;
		if ((rc = dalloc(c, &c.dtris, 3 * T, "triangles")))
			break;
		k_tri_write<<<grid, TRI_THREADS, 0, c.stream>>>(c.dO, c.dE, n, woff, bits, toff, c.dtris);
		c.launches++;
		if (cudaGetLastError() != cudaSuccess)
			rc = fail(NUCLEUS34_E_CUDA, "triangle kernels");
	} while (false);
	cleanup();
	return rc;
}

} // namespace n34

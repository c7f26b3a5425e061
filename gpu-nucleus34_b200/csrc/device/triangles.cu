// Triangle listing in canonical (a,b) order, written directly (no sort).
//
// Reference: cu_cliques_tris + intersect_lists (nucleus/utils.cuh:259-343) list
// triangles per vertex by a zipper against materialised length-2 paths
// (cu_multi_arrange, utils.cuh:515-548), append them in atomic order and sort
// them afterwards by tri_t::operator< (utils.cuh:98-101, 1901;
// cuNucleus34_ondemand.cu:499).
//
// Here a triangle {u, v, w} with u -> v, u -> w, v -> w in the orientation is
// (a = edge u->w, b = edge u->v, c = edge v->w), and canonical order is (a, b):
// u-major, then w's position ia in N+(u), then v's position ib. For a source
// u with out-degree d, the triangles form a d x d bit matrix M[ia][ib].
//   1. columns  one warp per oriented edge b = (u, v) merges N+(u) with N+(v)
//               in 32-entry tiles (coalesced loads, a 5-step shuffle search of
//               each A entry in the B tile); tile k of N+(u) gives word k of
//               column ib: M[32k .. 32k+31][ib].
//   2. rows     one warp per source transposes 32 x 32 blocks of those column
//               words with 32 ballots into row words M[ia][32q .. 32q+31], and
//               stores beside each row word the number of set bits before it
//               in the row; the row totals are the triangles per edge a.
//   3. offsets  scan of the per-edge-a counts: where each a's triangles start.
//   4. write    the merges of step 1 run again; a common w at A position ia
//               and B position pb is triangle (O[u]+ia, b, O[v]+pb), and its
//               canonical position is offset(a) + the row prefix + the set
//               bits of its row word below ib. No search is needed for c.
// Steps 1-2 hold 3 words of bits per (column, row tile) of each source; when
// those do not fit the budget the sources are taken in chunks, counting all
// of them first and repeating steps 1-2 before each chunk's writes.
//
// The pair-test kernels below (every (ia, ib) tested by a binary search of w
// in N+(v)) serve callers that manage their own memory and cannot give the
// listing scratch for bits (nucleus34_list_triangles_noalloc).
#include "pipeline.cuh"

#include <algorithm>
#include <cstdlib>
#include <vector>

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

// ---- merge-based listing ---------------------------------------------------

// words[u] = d * ceil(d / 32): one word per (column, row tile) of u's matrix
__global__ void k_list_words(const uint32_t *__restrict__ O, uint64_t n, uint64_t *__restrict__ words)
{
	const uint64_t u = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
	if (u < n)
	{
		const uint64_t d = O[u + 1] - O[u];
		words[u] = d * ((d + 31) / 32);
	}
}

// Warp tile merge of A = N+(u) (d entries) and B = N+(v) (dv entries), both
// ascending. For every 32-entry tile k of A, in order, f(k, found, pb) is
// called by all lanes: found = A[32k + lane] occurs in B, at B position pb.
// With all_tiles false the walk stops once B is used up (later tiles can have
// no match); with it set the remaining tiles are reported empty.
template <class F>
__device__ __forceinline__ void out_list_merge(const uint32_t *__restrict__ A, uint32_t d,
											   const uint32_t *__restrict__ B, uint32_t dv, bool all_tiles, F &&f)
{
	const uint32_t lane = lane_id();
	uint32_t bp = 0;                 // B entries before bp are below every A entry still to come
	uint32_t tile_at = 0xffffffffu;  // start of the B tile held in bt
	uint32_t bt = 0xffffffffu;
	const uint32_t tiles = (d + 31) >> 5;
	for (uint32_t k = 0; k < tiles; ++k)
	{
		if (bp >= dv)
		{
			if (!all_tiles)
				return;
			f(k, false, 0u);
			continue;
		}
		const uint32_t ai = (k << 5) + lane;
		const uint32_t av = ai < d ? __ldg(A + ai) : 0xffffffffu;
		const uint32_t alast = d - (k << 5) > 32 ? 31u : d - (k << 5) - 1;
		const uint32_t amax = __shfl_sync(FULL, av, alast);
		bool found = false;
		uint32_t pb = 0;
		uint32_t nb = 0;
		while (bp < dv) // warp-uniform
		{
			if (tile_at != bp)
			{
				bt = bp + lane < dv ? __ldg(B + bp + lane) : 0xffffffffu;
				tile_at = bp;
			}
			nb = dv - bp > 32 ? 32u : dv - bp;
			// first lane j of the B tile with bt_j >= av
			uint32_t pos = 0;
#pragma unroll
			for (uint32_t step = 16; step > 0; step >>= 1)
			{
				const uint32_t probe = __shfl_sync(FULL, bt, (pos + step - 1) & 31);
				if (probe < av)
					pos += step;
			}
			const uint32_t hv = __shfl_sync(FULL, bt, pos & 31);
			if (ai < d && pos < nb && hv == av)
			{
				found = true;
				pb = bp + pos;
			}
			const uint32_t blast = __shfl_sync(FULL, bt, nb - 1);
			if (blast > amax)
				break; // the tile reaches past this A tile: keep it
			bp += nb;  // the whole tile is <= amax: used up
		}
		f(k, found, pb);
		// entries of the held tile that are <= amax cannot match a later A entry
		if (bp < dv && tile_at == bp)
			bp += __popc(__ballot_sync(FULL, lane < nb && bt <= amax));
	}
}

// Step 1: column words. One warp per oriented edge b = (u, v) in [j0, j1);
// word k of column ib = j - O[u] sits at cols[woff[u] - wbase + ib * W + k].
__global__ void __launch_bounds__(TRI_THREADS) k_list_cols(const uint32_t *__restrict__ O,
														   const uint32_t *__restrict__ E,
														   const uint32_t *__restrict__ src, uint64_t j0,
														   uint64_t j1, const uint64_t *__restrict__ woff,
														   uint64_t wbase, uint32_t *__restrict__ cols)
{
	const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
	for (uint64_t j = j0 + warp; j < j1; j += nwarps)
	{
		const uint32_t u = __ldg(src + j), ob = __ldg(O + u), d = __ldg(O + u + 1) - ob;
		const uint32_t v = __ldg(E + j), vb = __ldg(O + v), dv = __ldg(O + v + 1) - vb;
		const uint32_t W = (d + 31) >> 5, ib = uint32_t(j - ob);
		uint32_t *col = cols + (woff[u] - wbase) + uint64_t(ib) * W;
		uint32_t held = 0; // word k is kept by lane k % 32 and stored 32 at a time
		out_list_merge(E + ob, d, E + vb, dv, true, [&](uint32_t k, bool found, uint32_t) {
			const uint32_t word = __ballot_sync(FULL, found);
			if (lane_id() == (k & 31))
				held = word;
			if ((k & 31) == 31 || k + 1 == W)
			{
				const uint32_t k0 = k & ~31u;
				if (lane_id() <= (k & 31))
					col[k0 + lane_id()] = held;
			}
		});
	}
}

// Step 2: row words, row prefixes and per-edge-a counts. One warp per source
// u in [u0, u1); 32 x 32 blocks of column words are transposed by ballots.
__global__ void __launch_bounds__(TRI_THREADS) k_list_rows(const uint32_t *__restrict__ O, uint64_t u0, uint64_t u1,
														   const uint64_t *__restrict__ woff, uint64_t wbase,
														   const uint32_t *__restrict__ cols,
														   uint32_t *__restrict__ rows, uint32_t *__restrict__ pre,
														   uint32_t *__restrict__ rowcnt)
{
	const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
	const uint32_t lane = lane_id();
	for (uint64_t u = u0 + warp; u < u1; u += nwarps)
	{
		const uint32_t ob = O[u], d = O[u + 1] - ob;
		if (d == 0)
			continue;
		const uint32_t W = (d + 31) >> 5;
		const uint64_t base = woff[u] - wbase;
		for (uint32_t r = 0; r < W; ++r)
		{
			const uint32_t row = (r << 5) + lane;
			uint32_t tot = 0;
			for (uint32_t q = 0; q < W; ++q)
			{
				const uint32_t col = (q << 5) + lane;
				const uint32_t w = col < d ? cols[base + uint64_t(col) * W + r] : 0u;
				uint32_t rw = 0;
#pragma unroll
				for (uint32_t i = 0; i < 32; ++i)
				{
					const uint32_t b = __ballot_sync(FULL, (w >> i) & 1u);
					if (lane == i)
						rw = b;
				}
				if (row < d)
				{
					rows[base + uint64_t(row) * W + q] = rw;
					pre[base + uint64_t(row) * W + q] = tot;
				}
				tot += __popc(rw);
			}
			if (row < d)
				rowcnt[ob + row] = tot;
		}
	}
}

// Step 4: the triangles at their canonical positions. One warp per oriented
// edge b in [j0, j1), the merge of step 1 again.
__global__ void __launch_bounds__(TRI_THREADS) k_list_write(const uint32_t *__restrict__ O,
															const uint32_t *__restrict__ E,
															const uint32_t *__restrict__ src, uint64_t j0,
															uint64_t j1, const uint64_t *__restrict__ woff,
															uint64_t wbase, const uint32_t *__restrict__ rows,
															const uint32_t *__restrict__ pre,
															const uint64_t *__restrict__ aoff, uint64_t T,
															uint32_t *__restrict__ tris, uint32_t *__restrict__ err)
{
	const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
	for (uint64_t j = j0 + warp; j < j1; j += nwarps)
	{
		const uint32_t u = __ldg(src + j), ob = __ldg(O + u), d = __ldg(O + u + 1) - ob;
		const uint32_t v = __ldg(E + j), vb = __ldg(O + v), dv = __ldg(O + v + 1) - vb;
		const uint32_t W = (d + 31) >> 5, ib = uint32_t(j - ob);
		const uint64_t base = woff[u] - wbase;
		const uint32_t q = ib >> 5, below = (1u << (ib & 31)) - 1u;
		out_list_merge(E + ob, d, E + vb, dv, false, [&](uint32_t k, bool found, uint32_t pb) {
			if (!found)
				return;
			const uint32_t ia = (k << 5) + lane_id();
			const uint64_t at = base + uint64_t(ia) * W + q;
			const uint64_t pos = aoff[ob + ia] + pre[at] + __popc(rows[at] & below);
			if (pos < T)
			{
				tris[3 * pos + 0] = ob + ia;
				tris[3 * pos + 1] = uint32_t(j);
				tris[3 * pos + 2] = vb + pb;
			}
			else
				atomicOr(err, 1u);
		});
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
	const uint64_t n = c.n, m = c.m;
	uint64_t *words = nullptr, *woff = nullptr, *aoff = nullptr;
	uint32_t *rowcnt = nullptr, *cols = nullptr, *rows = nullptr, *pre = nullptr, *err = nullptr;
	int rc = NUCLEUS34_OK;
	auto cleanup = [&] {
		c.release(words);
		c.release(woff);
		c.release(aoff);
		c.release(rowcnt);
		c.release(cols);
		c.release(rows);
		c.release(pre);
		c.release(err);
	};
	do
	{
		if ((rc = dalloc(c, &words, n, "listing words")) || (rc = dalloc(c, &woff, n + 1, "listing word offsets")) ||
			(rc = dalloc(c, &err, 1, "listing check")))
			break;
		if (cudaMemsetAsync(err, 0, 4, c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "memset");
			break;
		}
		k_list_words<<<uint32_t((n + 255) / 256), 256, 0, c.stream>>>(c.dO, n, words);
		c.launches++;
		if ((rc = scan_u64(c, words, woff, n)))
			break;
		uint64_t nwords = 0;
		if (cudaMemcpyAsync(&nwords, woff + n, 8, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaStreamSynchronize(c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "listing word count");
			break;
		}
		c.release(words);
		words = nullptr;
		if ((rc = dalloc(c, &rowcnt, m, "triangles per edge")) || (rc = dalloc(c, &aoff, m + 1, "triangle offsets")))
			break;
		// Chunks of sources whose bit words (3 arrays) fit a quarter of the
		// room left; one chunk when all of them do.
		const uint64_t room = c.budget > c.in_use ? c.budget - c.in_use : 0;
		uint64_t cap_words = std::max<uint64_t>(room / 4 / 12, uint64_t(1) << 20);
		// NUCLEUS34_LIST_CHUNK_WORDS=N caps the chunk at N words (a test hook
		// for the chunked path, which budgets alone reach only on large graphs)
		if (const char *e = std::getenv("NUCLEUS34_LIST_CHUNK_WORDS"))
			if (const uint64_t forced = std::strtoull(e, nullptr, 10))
				cap_words = forced;
		std::vector<uint64_t> cuts; // source boundaries: chunk i is [cuts[i], cuts[i+1])
		if (nwords <= cap_words)
			cuts = {0, n};
		else
		{
			std::vector<uint64_t> hw(n + 1);
			if (cudaMemcpyAsync(hw.data(), woff, (n + 1) * 8, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
				cudaStreamSynchronize(c.stream) != cudaSuccess)
			{
				rc = fail(NUCLEUS34_E_CUDA, "listing word offsets");
				break;
			}
			cuts.push_back(0);
			while (cuts.back() < n)
			{
				const uint64_t u0 = cuts.back();
				// last u1 > u0 with hw[u1] - hw[u0] <= cap_words (at least one source)
				uint64_t u1 = uint64_t(std::upper_bound(hw.begin() + u0 + 1, hw.end(), hw[u0] + cap_words) -
									   hw.begin()) - 1;
				if (u1 <= u0)
					u1 = u0 + 1;
				cuts.push_back(u1);
			}
		}
		std::vector<uint32_t> hO(cuts.size());
		for (size_t i = 0; i < cuts.size(); ++i)
		{
			if (cudaMemcpyAsync(&hO[i], c.dO + cuts[i], 4, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess)
			{
				rc = fail(NUCLEUS34_E_CUDA, "listing chunk edges");
				break;
			}
		}
		if (rc)
			break;
		std::vector<uint64_t> hwc(cuts.size());
		for (size_t i = 0; i < cuts.size(); ++i)
			if (cudaMemcpyAsync(&hwc[i], woff + cuts[i], 8, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess)
			{
				rc = fail(NUCLEUS34_E_CUDA, "listing chunk words");
				break;
			}
		if (rc || cudaStreamSynchronize(c.stream) != cudaSuccess)
		{
			rc = rc ? rc : fail(NUCLEUS34_E_CUDA, "listing chunks");
			break;
		}
		uint64_t maxw = 0;
		for (size_t i = 0; i + 1 < cuts.size(); ++i)
			maxw = std::max(maxw, hwc[i + 1] - hwc[i]);
		const uint64_t alloc_w = maxw ? maxw : 1;
		if ((rc = dalloc(c, &cols, alloc_w, "listing column words")) ||
			(rc = dalloc(c, &rows, alloc_w, "listing row words")) ||
			(rc = dalloc(c, &pre, alloc_w, "listing row prefixes")))
			break;
		const size_t nchunks = cuts.size() - 1;
		auto bits_of_chunk = [&](size_t i) -> int {
			const uint64_t u0 = cuts[i], u1 = cuts[i + 1], j0 = hO[i], j1 = hO[i + 1];
			if (j1 > j0)
				N34_LAUNCH(c, k_list_cols, grid_for(c, j1 - j0, TRI_WARPS, 32), TRI_THREADS, 0, c.dO, c.dE, c.dsrc,
						   j0, j1, woff, hwc[i], cols);
			N34_LAUNCH(c, k_list_rows, grid_for(c, u1 - u0, TRI_WARPS, 32), TRI_THREADS, 0, c.dO, u0, u1, woff,
					   hwc[i], cols, rows, pre, rowcnt);
			return NUCLEUS34_OK;
		};
		// counts of every chunk, then the offsets
		for (size_t i = 0; i < nchunks && !rc; ++i)
			rc = bits_of_chunk(i);
		if (rc || (rc = scan_u32(c, rowcnt, aoff, m)))
			break;
		uint64_t T = 0;
		if (cudaMemcpyAsync(&T, aoff + m, 8, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
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
		for (size_t i = 0; i < nchunks && !rc; ++i)
		{
			// a single chunk still holds its bits from the count
			if (nchunks > 1 && (rc = bits_of_chunk(i)))
				break;
			const uint64_t j0 = hO[i], j1 = hO[i + 1];
			if (j1 > j0)
			{
				k_list_write<<<grid_for(c, j1 - j0, TRI_WARPS, 32), TRI_THREADS, 0, c.stream>>>(
					c.dO, c.dE, c.dsrc, j0, j1, woff, hwc[i], rows, pre, aoff, T, c.dtris, err);
				c.launches++;
			}
		}
		if (rc)
			break;
		uint32_t herr = 0;
		if (cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaStreamSynchronize(c.stream) != cudaSuccess || cudaGetLastError() != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "triangle kernels");
			break;
		}
		if (herr)
			rc = fail(NUCLEUS34_E_CUDA, "internal: triangle listing check failed");
	} while (false);
	cleanup();
	return rc;
}

} // namespace n34

// Oriented CSR of an edge list built on the device (nucleus34_ctx_upload_edges).
//
// Reference: graph_t::from_edges (nucleus/graph/graph.hpp:356-411:
// symmetrise, drop self-loops, parallel sort + unique of the pairs, n = max
// id + 1 over the non-loop pairs) followed by make_oriented (graph.hpp:176-218:
// keep (u,v) iff (deg u, u) < (deg v, v) on the undirected degree), both on
// the host. The library's host build (csrc/host/graph_io.cpp) has the same
// semantics; this is its device form, for inputs whose pairs are already in
// host memory:
//   largest id       one pass over the pairs (non-loop pairs only)
//   raw counts       both directions of every non-loop pair (duplicates kept)
//   scatter          into per-vertex segments (scan of the counts)
//   sort             each segment ascending (the incidence's segmented sort)
//   unique degree    distinct neighbours per vertex (one warp per vertex)
//   orientation      out-degree under the (degree, id) order, scan, then the
//                    kept neighbours written in ascending order
// The result is left resident in the context exactly as nucleus34_ctx_upload
// leaves a host CSR: dO (n+1), dE (m), dsrc (m).
#include "pipeline.cuh"

namespace n34 {

namespace {

constexpr int CB_THREADS = 256;
constexpr int CB_WARPS = CB_THREADS / 32;

__global__ void k_edges_max(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst, uint64_t P,
							unsigned int *__restrict__ mx, unsigned long long *__restrict__ nonloop)
{
	uint32_t m = 0;
	unsigned long long k = 0;
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < P; i += stride)
	{
		const uint32_t s = src[i], d = dst[i];
		if (s != d)
		{
			m = max(m, max(s, d));
			++k;
		}
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
	{
		m = max(m, __shfl_xor_sync(FULL, m, o));
		k += __shfl_xor_sync(FULL, k, o);
	}
	if (lane_id() == 0)
	{
		atomicMax(mx, m);
		if (k)
			atomicAdd(nonloop, k);
	}
}

// Raw count of vertex u: both directions of every non-loop pair.
__global__ void k_edges_count(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst, uint64_t P,
							  uint64_t n, unsigned long long *__restrict__ cnt, uint32_t *__restrict__ err)
{
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < P; i += stride)
	{
		const uint32_t s = src[i], d = dst[i];
		if (s == d)
			continue;
		if (s >= n || d >= n)
		{
			atomicOr(err, 1u);
			continue;
		}
		atomicAdd(cnt + s, 1ull);
		atomicAdd(cnt + d, 1ull);
	}
}

// Scatter into the segments: keys[off[u] + slot] = v (as a 64-bit sort key).
__global__ void k_edges_scatter(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst, uint64_t P,
								uint64_t n, const uint64_t *__restrict__ off, unsigned long long *__restrict__ cur,
								unsigned long long *__restrict__ keys, uint32_t *__restrict__ err)
{
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < P; i += stride)
	{
		const uint32_t s = src[i], d = dst[i];
		if (s == d || s >= n || d >= n)
			continue;
		const uint64_t ps = off[s] + atomicAdd(cur + s, 1ull);
		const uint64_t pd = off[d] + atomicAdd(cur + d, 1ull);
		if (ps >= off[s + 1] || pd >= off[d + 1])
		{
			atomicOr(err, 2u);
			continue;
		}
		keys[ps] = d;
		keys[pd] = s;
	}
}

// Distinct neighbours of each vertex in its sorted segment (warp per vertex).
__global__ void __launch_bounds__(CB_THREADS) k_adj_unique(const uint64_t *__restrict__ off, uint64_t n,
															const unsigned long long *__restrict__ keys,
															uint32_t *__restrict__ udeg)
{
	const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
	const uint32_t lane = lane_id();
	for (uint64_t u = warp; u < n; u += nwarps)
	{
		const uint64_t b = off[u], e = off[u + 1];
		uint32_t k = 0;
		for (uint64_t j0 = b; j0 < e; j0 += 32)
		{
			const uint64_t j = j0 + lane;
			bool first = false;
			if (j < e)
				first = j == b || keys[j] != keys[j - 1];
			k += __popc(__ballot_sync(FULL, first));
		}
		if (lane == 0)
			udeg[u] = k;
	}
}

// u keeps v iff (deg u, u) < (deg v, v) on the undirected degree.
__device__ __forceinline__ bool keeps(uint32_t du, uint64_t u, uint32_t dv, uint32_t v)
{
	return du < dv || (du == dv && u < v);
}

// Out-degree of each vertex under the orientation (warp per vertex).
__global__ void __launch_bounds__(CB_THREADS) k_adj_outdeg(const uint64_t *__restrict__ off, uint64_t n,
															const unsigned long long *__restrict__ keys,
															const uint32_t *__restrict__ udeg,
															uint32_t *__restrict__ D)
{
	const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
	const uint32_t lane = lane_id();
	for (uint64_t u = warp; u < n; u += nwarps)
	{
		const uint64_t b = off[u], e = off[u + 1];
		const uint32_t du = udeg[u];
		uint32_t k = 0;
		for (uint64_t j0 = b; j0 < e; j0 += 32)
		{
			const uint64_t j = j0 + lane;
			bool take = false;
			if (j < e && (j == b || keys[j] != keys[j - 1]))
			{
				const uint32_t v = uint32_t(keys[j]);
				take = keeps(du, u, udeg[v], v);
			}
			k += __popc(__ballot_sync(FULL, take));
		}
		if (lane == 0)
			D[u] = k;
	}
}

// 64-bit offsets to the 32-bit O of the CSR (the total is checked on the host).
__global__ void k_offsets_u32(const uint64_t *__restrict__ o64, uint64_t n1, uint32_t *__restrict__ O)
{
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n1; i += stride)
		O[i] = uint32_t(o64[i]);
}

// The kept neighbours of each vertex, ascending, at O[u] (warp per vertex).
__global__ void __launch_bounds__(CB_THREADS) k_adj_write(const uint64_t *__restrict__ off, uint64_t n,
														   const unsigned long long *__restrict__ keys,
														   const uint32_t *__restrict__ udeg,
														   const uint32_t *__restrict__ O, uint64_t m,
														   uint32_t *__restrict__ E, uint32_t *__restrict__ err)
{
	const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
	const uint32_t lane = lane_id();
	for (uint64_t u = warp; u < n; u += nwarps)
	{
		const uint64_t b = off[u], e = off[u + 1];
		const uint32_t du = udeg[u];
		uint64_t w = O[u];
		const uint64_t wend = O[u + 1];
		for (uint64_t j0 = b; j0 < e; j0 += 32)
		{
			const uint64_t j = j0 + lane;
			bool take = false;
			uint32_t v = 0;
			if (j < e && (j == b || keys[j] != keys[j - 1]))
			{
				v = uint32_t(keys[j]);
				take = keeps(du, u, udeg[v], v);
			}
			const uint32_t bal = __ballot_sync(FULL, take);
			const uint64_t p = w + __popc(bal & lanemask_lt());
			if (take)
			{
				if (p < wend && p < m)
					E[p] = v;
				else
					atomicOr(err, 4u);
			}
			w += __popc(bal);
		}
	}
}

__global__ void k_max_u32(const uint32_t *__restrict__ a, uint64_t n, unsigned int *__restrict__ mx)
{
	uint32_t m = 0;
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
		m = max(m, a[i]);
#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		m = max(m, __shfl_xor_sync(FULL, m, o));
	if (lane_id() == 0 && m)
		atomicMax(mx, m);
}

} // namespace

int upload_edges(Ctx &c, const uint32_t *src, const uint32_t *dst, uint64_t P)
{
	if (P && (!src || !dst))
		return fail(NUCLEUS34_E_INVALID, "null edge arrays");
	N34_CUDA(cudaSetDevice(c.device));
	c.release_results();
	c.release_graph();
	c.seg_eoff.clear();
	uint32_t *dsrc_in = nullptr, *ddst_in = nullptr, *udeg = nullptr, *D = nullptr, *O = nullptr, *E = nullptr,
			 *err = nullptr;
	unsigned int *mx = nullptr;
	unsigned long long *cnt = nullptr, *keys = nullptr, *nonloop = nullptr;
	uint64_t *off = nullptr, *o64 = nullptr;
	int rc = NUCLEUS34_OK;
	auto cleanup = [&] {
		c.release(dsrc_in);
		c.release(ddst_in);
		c.release(udeg);
		c.release(D);
		c.release(err);
		c.release(mx);
		c.release(cnt);
		c.release(keys);
		c.release(nonloop);
		c.release(off);
		c.release(o64);
		c.release(O);
		c.release(E);
	};
	do
	{
		// pairs to the device; largest id and non-loop pair count
		if ((rc = dalloc(c, &dsrc_in, P ? P : 1, "edge sources")) ||
			(rc = dalloc(c, &ddst_in, P ? P : 1, "edge destinations")) ||
			(rc = dalloc(c, &mx, 1, "largest vertex id")) || (rc = dalloc(c, &nonloop, 1, "non-loop pairs")) ||
			(rc = dalloc(c, &err, 1, "build check")))
			break;
		if ((P && (cudaMemcpyAsync(dsrc_in, src, P * 4, cudaMemcpyHostToDevice, c.stream) != cudaSuccess ||
				   cudaMemcpyAsync(ddst_in, dst, P * 4, cudaMemcpyHostToDevice, c.stream) != cudaSuccess)) ||
			cudaMemsetAsync(mx, 0, 4, c.stream) != cudaSuccess ||
			cudaMemsetAsync(nonloop, 0, 8, c.stream) != cudaSuccess ||
			cudaMemsetAsync(err, 0, 4, c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "edge upload");
			break;
		}
		if (P)
		{
			k_edges_max<<<grid_for(c, P, CB_THREADS), CB_THREADS, 0, c.stream>>>(dsrc_in, ddst_in, P, mx, nonloop);
			c.launches++;
		}
		unsigned int hmax = 0;
		unsigned long long hnl = 0;
		if (cudaMemcpyAsync(&hmax, mx, 4, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaMemcpyAsync(&hnl, nonloop, 8, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaStreamSynchronize(c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "edge scan");
			break;
		}
		// n = max id + 1 over the non-loop pairs (1 when there are none)
		const uint64_t n = uint64_t(hmax) + 1;
		if (n >= 0xffffffffull)
		{
			rc = fail(NUCLEUS34_E_RANGE32, "graph exceeds 32-bit vertex ids");
			break;
		}
		const uint64_t total = 2 * hnl;
		if ((rc = dalloc(c, &cnt, n, "raw degrees")) || (rc = dalloc(c, &off, n + 1, "raw offsets")) ||
			(rc = dalloc(c, &keys, total ? total : 1, "adjacency keys")))
			break;
		if (cudaMemsetAsync(cnt, 0, n * 8, c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "memset");
			break;
		}
		if (P)
		{
			k_edges_count<<<grid_for(c, P, CB_THREADS), CB_THREADS, 0, c.stream>>>(dsrc_in, ddst_in, P, n, cnt,
																				   err);
			c.launches++;
		}
		if ((rc = scan_u64(c, reinterpret_cast<const uint64_t *>(cnt), off, n)))
			break;
		if (cudaMemsetAsync(cnt, 0, n * 8, c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "memset");
			break;
		}
		if (P)
		{
			k_edges_scatter<<<grid_for(c, P, CB_THREADS), CB_THREADS, 0, c.stream>>>(dsrc_in, ddst_in, P, n, off,
																					 cnt, keys, err);
			c.launches++;
		}
		c.release(dsrc_in);
		c.release(ddst_in);
		c.release(cnt);
		dsrc_in = ddst_in = nullptr;
		cnt = nullptr;
		if ((rc = sort_segments_u64(c, keys, off, n)))
			break;
		// undirected degree, orientation, offsets
		if ((rc = dalloc(c, &udeg, n, "undirected degrees")) || (rc = dalloc(c, &D, n, "out-degrees")) ||
			(rc = dalloc(c, &o64, n + 1, "oriented offsets")))
			break;
		const uint32_t gv = grid_for(c, n, CB_WARPS);
		k_adj_unique<<<gv, CB_THREADS, 0, c.stream>>>(off, n, keys, udeg);
		k_adj_outdeg<<<gv, CB_THREADS, 0, c.stream>>>(off, n, keys, udeg, D);
		c.launches += 2;
		if ((rc = scan_u32(c, D, o64, n)))
			break;
		uint64_t m = 0;
		uint32_t herr = 0;
		if (cudaMemcpyAsync(&m, o64 + n, 8, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaStreamSynchronize(c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "orientation");
			break;
		}
		if (herr)
		{
			rc = fail(NUCLEUS34_E_CUDA, "internal: edge build check failed (" + std::to_string(herr) + ")");
			break;
		}
		if (m > 0xffffffffull)
		{
			rc = fail(NUCLEUS34_E_RANGE32, "oriented edge count exceeds 32-bit edge ids");
			break;
		}
		if ((rc = dalloc(c, &O, n + 1, "CSR offsets")) || (rc = dalloc(c, &E, m ? m : 1, "CSR destinations")))
			break;
		k_offsets_u32<<<grid_for(c, n + 1, CB_THREADS), CB_THREADS, 0, c.stream>>>(o64, n + 1, O);
		k_adj_write<<<gv, CB_THREADS, 0, c.stream>>>(off, n, keys, udeg, O, m, E, err);
		c.launches += 2;
		// largest out-degree (the tune table's skew class)
		if (cudaMemsetAsync(mx, 0, 4, c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "memset");
			break;
		}
		k_max_u32<<<grid_for(c, n, CB_THREADS), CB_THREADS, 0, c.stream>>>(D, n, mx);
		c.launches++;
		if (cudaMemcpyAsync(&hmax, mx, 4, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaStreamSynchronize(c.stream) != cudaSuccess || cudaGetLastError() != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "edge build kernels");
			break;
		}
		if (herr)
		{
			rc = fail(NUCLEUS34_E_CUDA, "internal: edge build check failed (" + std::to_string(herr) + ")");
			break;
		}
		// resident like an uploaded CSR
		c.dO = O;
		c.dE = E;
		O = E = nullptr;
		c.n = n;
		c.m = m;
		c.max_out = hmax;
		if ((rc = dalloc(c, &c.dsrc, m ? m : 1, "CSR sources")))
		{
			c.release_graph();
			break;
		}
		if ((rc = build_src(c)))
		{
			c.release_graph();
			break;
		}
		if (cudaStreamSynchronize(c.stream) != cudaSuccess)
		{
			c.release_graph();
			rc = fail(NUCLEUS34_E_CUDA, "CSR sources");
		}
	} while (false);
	cleanup();
	return rc;
}

} // namespace n34

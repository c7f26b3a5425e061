// Edge -> triangle incidence: for every oriented edge e, the triangles that
// contain e, each as (third vertex x, triangle id), sorted by x.
//
// Reference: build_incidence_entries + thrust::sort_by_key on the 64-bit key
// (edge<<32 | third) + split_keys + lower_bound (nucleus/cuNucleus34_ondemand.cu:
// 92-128, 513-549): one global radix sort of 3T 64-bit keys.
//
// Here: per-edge counts (atomics) -> exclusive scan -> scatter of 64-bit
// (x<<32 | t) entries into their edge's segment -> a segmented sort of each
// segment by x (segments are short: a warp bitonic network on registers for
// <= 256 entries, a shared-memory block bitonic sort up to SEG_SMEM, a
// global-memory bitonic sort on a padded copy beyond that) -> split into the third[] and tri[]
// arrays the 3-way intersection reads. Triangle t = (a,b,c) with u = src[b],
// v = E[b], w = E[c] is listed under b with x = w, under a with x = v and under
// c with x = u, exactly the reference's three entries.
#include "pipeline.cuh"

#include <algorithm>

namespace n34 {

namespace {

constexpr int SEG_WARP_MAX = 256;     // keys per warp sort (8 registers per lane)
constexpr int SEG_SMEM = 8192;        // keys per block sort (64 KB smem)
constexpr int SEG_BLOCK = 512;

// Entry storage of the sorts: the 64-bit (x<<32 | t) keys, or, in the
// memory-lean build, the third[] and tri[] arrays themselves (sorted as pairs
// in place, so that no key array coexists with them).
struct EntryStore
{
	unsigned long long *keys; // null: use third / tri
	uint32_t *third, *tri;
	__device__ __forceinline__ unsigned long long ld(uint64_t i) const
	{
		return keys ? keys[i] : ((unsigned long long)third[i] << 32) | tri[i];
	}
	__device__ __forceinline__ void st(uint64_t i, unsigned long long v) const
	{
		if (keys)
			keys[i] = v;
		else
		{
			third[i] = uint32_t(v >> 32);
			tri[i] = uint32_t(v);
		}
	}
};

__global__ void k_inc_count(const uint32_t *__restrict__ tris, uint64_t T, uint32_t *__restrict__ cnt)
{
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < T; t += stride)
	{
		atomicAdd(cnt + tris[3 * t + 0], 1u);
		atomicAdd(cnt + tris[3 * t + 1], 1u);
		atomicAdd(cnt + tris[3 * t + 2], 1u);
	}
}

__global__ void k_inc_scatter(const uint32_t *__restrict__ tris, uint64_t T, const uint32_t *__restrict__ src,
							  const uint32_t *__restrict__ E, const uint64_t *__restrict__ incO,
							  uint32_t *__restrict__ cursor, EntryStore keys, uint32_t *__restrict__ err,
							  bool slot_bits)
{
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < T; t += stride)
	{
		const uint32_t a = tris[3 * t + 0], b = tris[3 * t + 1], c = tris[3 * t + 2];
		const uint32_t u = src[b], v = E[b], w = E[c];
		const uint32_t e3[3] = {b, a, c};
		const uint32_t x3[3] = {w, v, u};
#pragma unroll
		for (int r = 0; r < 3; ++r)
		{
			const uint32_t e = e3[r];
			const uint32_t s = atomicAdd(cursor + e, 1u);
			// capacity guard: the counts pass sized every segment exactly
			if (incO[e] + s < incO[e + 1])
				keys.st(incO[e] + s, (uint64_t(x3[r]) << 32) | (slot_bits ? (t | (uint64_t(r) << 30)) : t));
			else
				atomicOr(err, 1u);
		}
	}
}

// Classifies edges by segment length into three work lists.
__global__ void k_seg_classify(const uint64_t *__restrict__ incO, uint64_t m, uint32_t *__restrict__ lists,
							   uint32_t *__restrict__ counts, uint64_t list_cap, unsigned long long *max_len)
{
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t e0 = uint64_t(blockIdx.x) * blockDim.x; e0 < m; e0 += stride)
	{
		const uint64_t e = e0 + threadIdx.x;
		uint64_t len = 0;
		if (e < m)
			len = incO[e + 1] - incO[e];
		const int cls = len < 2 ? -1 : (len <= SEG_WARP_MAX ? 0 : (len <= SEG_SMEM ? 1 : 2));
#pragma unroll
		for (int k = 0; k < 3; ++k)
		{
			const uint32_t slot = warp_append(cls == k, counts + k);
			if (cls == k)
				lists[uint64_t(k) * list_cap + slot] = uint32_t(e);
		}
		if (cls == 2)
			atomicMax(max_len, (unsigned long long)len);
	}
}

// Bitonic network over 32*K keys held K per lane (element k*32 + lane in
// v[k]): strides below 32 pair lanes (shuffles), larger ones pair registers
// of the same lane.
template <int K>
__device__ __forceinline__ void warp_bitonic(unsigned long long (&v)[K])
{
	const uint32_t lane = lane_id();
#pragma unroll
	for (uint32_t size = 2; size <= 32u * K; size <<= 1)
	{
#pragma unroll
		for (uint32_t stride = size >> 1; stride > 0; stride >>= 1)
		{
			if (stride >= 32)
			{
				const uint32_t ks = stride >> 5;
#pragma unroll
				for (int k = 0; k < K; ++k)
				{
					if ((uint32_t(k) & ks) == 0)
					{
						const int k2 = int(uint32_t(k) | ks);
						const bool up = ((uint32_t(k) * 32 + lane) & size) == 0;
						const unsigned long long a = v[k], b = v[k2];
						if ((a > b) == up)
						{
							v[k] = b;
							v[k2] = a;
						}
					}
				}
			}
			else
			{
#pragma unroll
				for (int k = 0; k < K; ++k)
				{
					const unsigned long long o = __shfl_xor_sync(FULL, v[k], stride);
					const bool up = ((uint32_t(k) * 32 + lane) & size) == 0;
					const bool lower = (lane & stride) == 0;
					const unsigned long long mn = v[k] < o ? v[k] : o, mx = v[k] < o ? o : v[k];
					v[k] = (lower == up) ? mn : mx;
				}
			}
		}
	}
}

template <int K>
__device__ __forceinline__ void warp_sort_segment(const EntryStore &keys, uint64_t b, uint32_t len)
{
	const uint32_t lane = lane_id();
	unsigned long long v[K];
#pragma unroll
	for (int k = 0; k < K; ++k)
	{
		const uint32_t i = uint32_t(k) * 32 + lane;
		v[k] = i < len ? keys.ld(b + i) : ~0ull;
	}
	warp_bitonic<K>(v);
#pragma unroll
	for (int k = 0; k < K; ++k)
	{
		const uint32_t i = uint32_t(k) * 32 + lane;
		if (i < len)
			keys.st(b + i, v[k]);
	}
}

// Warp per segment (<= SEG_WARP_MAX entries): register bitonic network of
// the smallest power of two that holds it.
__global__ void k_seg_sort_warp(const uint32_t *__restrict__ list, const uint32_t *__restrict__ count,
								const uint64_t *__restrict__ incO, EntryStore keys)
{
	const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
	const uint32_t n = *count;
	for (uint64_t i = warp; i < n; i += nwarps)
	{
		const uint32_t e = list[i];
		const uint64_t b = incO[e];
		const uint32_t len = uint32_t(incO[e + 1] - b);
		if (len <= 32)
			warp_sort_segment<1>(keys, b, len);
		else if (len <= 64)
			warp_sort_segment<2>(keys, b, len);
		else if (len <= 128)
			warp_sort_segment<4>(keys, b, len);
		else
			warp_sort_segment<8>(keys, b, len);
	}
}

// Block bitonic sort of n (padded to pow2 P) keys in `s` (shared or global).
__device__ __forceinline__ void block_bitonic(unsigned long long *s, uint32_t P)
{
	for (uint32_t size = 2; size <= P; size <<= 1)
		for (uint32_t stride = size >> 1; stride > 0; stride >>= 1)
		{
			for (uint32_t i = threadIdx.x; i < P / 2; i += blockDim.x)
			{
				const uint32_t lo = 2 * i - (i & (stride - 1));
				const uint32_t hi = lo + stride;
				const bool up = (lo & size) == 0;
				unsigned long long x = s[lo], y = s[hi];
				if ((x > y) == up)
				{
					s[lo] = y;
					s[hi] = x;
				}
			}
			__syncthreads();
		}
}

__global__ void __launch_bounds__(SEG_BLOCK) k_seg_sort_block(const uint32_t *__restrict__ list,
															  const uint32_t *__restrict__ count,
															  const uint64_t *__restrict__ incO,
															  EntryStore keys)
{
	extern __shared__ unsigned long long sm[];
	const uint32_t n = *count;
	for (uint32_t i = blockIdx.x; i < n; i += gridDim.x)
	{
		const uint32_t e = list[i];
		const uint64_t b = incO[e];
		const uint32_t len = uint32_t(incO[e + 1] - b);
		uint32_t P = 64;
		while (P < len)
			P <<= 1;
		for (uint32_t j = threadIdx.x; j < P; j += blockDim.x)
			sm[j] = j < len ? keys.ld(b + j) : ~0ull;
		__syncthreads();
		block_bitonic(sm, P);
		for (uint32_t j = threadIdx.x; j < len; j += blockDim.x)
			keys.st(b + j, sm[j]);
		__syncthreads();
	}
}

// Long segments: padded copy in global scratch (one region per block).
__global__ void __launch_bounds__(SEG_BLOCK) k_seg_sort_global(const uint32_t *__restrict__ list,
															   const uint32_t *__restrict__ count,
															   const uint64_t *__restrict__ incO,
															   EntryStore keys,
															   unsigned long long *__restrict__ scratch,
															   uint64_t region)
{
	const uint32_t n = *count;
	unsigned long long *s = scratch + uint64_t(blockIdx.x) * region;
	for (uint32_t i = blockIdx.x; i < n; i += gridDim.x)
	{
		const uint32_t e = list[i];
		const uint64_t b = incO[e];
		const uint64_t len = incO[e + 1] - b;
		uint64_t P = 64;
		while (P < len)
			P <<= 1;
		if (P > region)
			continue; // cannot happen: region is sized from the longest segment
		for (uint64_t j = threadIdx.x; j < P; j += blockDim.x)
			s[j] = j < len ? keys.ld(b + j) : ~0ull;
		__syncthreads();
		block_bitonic(s, uint32_t(P));
		for (uint64_t j = threadIdx.x; j < len; j += blockDim.x)
			keys.st(b + j, s[j]);
		__syncthreads();
	}
}

__global__ void k_sum_sq(const uint64_t *__restrict__ off, uint64_t m, unsigned long long *__restrict__ out)
{
	unsigned long long acc = 0;
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t e = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < m; e += stride)
	{
		const unsigned long long d = off[e + 1] - off[e];
		acc += d * d;
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		acc += __shfl_xor_sync(FULL, acc, o);
	if (lane_id() == 0 && acc)
		atomicAdd(out, acc);
}

// Splits the sorted keys into third[] and tri[]; with tpos, the key's slot
// bits (30-31: which of the triangle's three entries) give tpos[3t + slot].
__global__ void k_inc_split(const unsigned long long *__restrict__ keys, uint64_t n, uint32_t *__restrict__ third,
							uint32_t *__restrict__ tri, uint32_t *__restrict__ tpos)
{
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
	{
		const unsigned long long k = keys[i];
		third[i] = uint32_t(k >> 32);
		const uint32_t lo = uint32_t(k);
		if (tpos)
		{
			const uint32_t t = lo & 0x3fffffffu;
			tri[i] = t;
			tpos[3 * uint64_t(t) + (lo >> 30)] = uint32_t(i);
		}
		else
			tri[i] = lo;
	}
}

// Per-edge list bounds as 32-bit (begin, end) pairs (3T < 2^32 entries).
__global__ void k_make_spans(const uint64_t *__restrict__ off, uint64_t m, uint2 *__restrict__ span)
{
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t e = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < m; e += stride)
		span[e] = make_uint2(uint32_t(off[e]), uint32_t(off[e + 1]));
}

} // namespace

int build_incidence(Ctx &c, Incidence &inc, bool want_tpos, bool lean)
{
	const uint64_t T = c.T, m = c.m, n3 = 3 * T;
	uint32_t *cnt = nullptr, *lists = nullptr, *counts = nullptr, *errf = nullptr;
	unsigned long long *keys = nullptr, *scratch = nullptr, *maxlen = nullptr, *sumsq = nullptr;
	uint64_t *off = nullptr;
	int rc = NUCLEUS34_OK;
	auto cleanup = [&] {
		c.release(off);
		c.release(cnt);
		c.release(lists);
		c.release(counts);
		c.release(keys);
		c.release(scratch);
		c.release(maxlen);
		c.release(errf);
		c.release(sumsq);
	};
	do
	{
		if ((rc = dalloc(c, &off, m + 1, "incidence offsets")))
			break;
		if ((rc = dalloc(c, &cnt, m, "incidence counts")))
			break;
		if (cudaMemsetAsync(cnt, 0, m * 4, c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "memset");
			break;
		}
		k_inc_count<<<grid_for(c, T, 256), 256, 0, c.stream>>>(c.dtris, T, cnt);
		c.launches++;
		if ((rc = scan_u32(c, cnt, off, m)))
			break;
		// lean: the entries are scattered straight into third[] / tri[] and
		// sorted there as pairs (no 8-byte key per entry beside them)
		if (lean)
		{
			if ((rc = dalloc(c, &inc.third, n3, "incidence third")))
				break;
			if ((rc = dalloc(c, &inc.tri, n3, "incidence tri")))
				break;
		}
		else if ((rc = dalloc(c, &keys, n3, "incidence keys")))
			break;
		const EntryStore store{keys, inc.third, inc.tri};
		if (cudaMemsetAsync(cnt, 0, m * 4, c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "memset");
			break;
		}
		if ((rc = dalloc(c, &errf, 1, "incidence check")))
			break;
		if (cudaMemsetAsync(errf, 0, 4, c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "memset");
			break;
		}
		// entry positions per triangle (the on-demand peel's death flags);
		// optional: without room for them the peel searches instead
		if (want_tpos && !lean && T <= 0x3fffffffull)
		{
			if (dalloc(c, &inc.tpos, 3 * T, "triangle entry positions"))
			{
				inc.tpos = nullptr;
				clear_error();
			}
		}
		k_inc_scatter<<<grid_for(c, T, 256), 256, 0, c.stream>>>(c.dtris, T, c.dsrc, c.dE, off, cnt, store, errf,
																 inc.tpos != nullptr);
		c.launches++;
		c.release(cnt);
		cnt = nullptr;
		// segmented sort
		if ((rc = dalloc(c, &lists, 3 * m, "segment lists")))
			break;
		if ((rc = dalloc(c, &counts, 4, "segment counts")))
			break;
		if ((rc = dalloc(c, &maxlen, 1, "segment max")))
			break;
		if ((rc = dalloc(c, &sumsq, 1, "segment square sum")))
			break;
		if (cudaMemsetAsync(counts, 0, 16, c.stream) != cudaSuccess ||
			cudaMemsetAsync(maxlen, 0, 8, c.stream) != cudaSuccess ||
			cudaMemsetAsync(sumsq, 0, 8, c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "memset");
			break;
		}
		k_seg_classify<<<grid_for(c, m, 256), 256, 0, c.stream>>>(off, m, lists, counts, m, maxlen);
		c.launches++;
		k_sum_sq<<<grid_for(c, m, 256), 256, 0, c.stream>>>(off, m, sumsq);
		c.launches++;
		uint32_t hcounts[4] = {0, 0, 0, 0};
		unsigned long long hmax = 0;
		uint32_t herr = 0;
		if (cudaMemcpyAsync(&inc.sum_te_sq, sumsq, 8, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaMemcpyAsync(&herr, errf, 4, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaMemcpyAsync(hcounts, counts, 16, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaMemcpyAsync(&hmax, maxlen, 8, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaStreamSynchronize(c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "segment classify");
			break;
		}
		if (herr)
		{
			rc = fail(NUCLEUS34_E_CUDA, "internal: incidence segment overflow");
			break;
		}
		if (hcounts[0])
		{
			k_seg_sort_warp<<<grid_for(c, hcounts[0], 8, 32), 256, 0, c.stream>>>(lists, counts + 0, off, store);
			c.launches++;
		}
		if (hcounts[1])
		{
			const size_t smem = SEG_SMEM * sizeof(unsigned long long);
			cudaFuncSetAttribute(k_seg_sort_block, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
			k_seg_sort_block<<<grid_for(c, hcounts[1], 1, 2), SEG_BLOCK, smem, c.stream>>>(lists + m, counts + 1,
																							off, store);
			c.launches++;
		}
		if (hcounts[2])
		{
			uint64_t P = 64;
			while (P < hmax)
				P <<= 1;
			const uint32_t blocks = std::min<uint32_t>(hcounts[2], uint32_t(c.sm_count));
			if ((rc = dalloc(c, &scratch, P * blocks, "segment sort scratch")))
				break;
			k_seg_sort_global<<<blocks, SEG_BLOCK, 0, c.stream>>>(lists + 2 * m, counts + 2, off, store,
																  scratch, P);
			c.launches++;
		}
		if (!lean)
		{
			if ((rc = dalloc(c, &inc.third, n3, "incidence third")))
				break;
			if ((rc = dalloc(c, &inc.tri, n3, "incidence tri")))
				break;
			k_inc_split<<<grid_for(c, n3, 256), 256, 0, c.stream>>>(keys, n3, inc.third, inc.tri, inc.tpos);
			c.launches++;
		}
		if ((rc = dalloc(c, &inc.span, m ? m : 1, "incidence spans")))
			break;
		k_make_spans<<<grid_for(c, m, 256), 256, 0, c.stream>>>(off, m, inc.span);
		c.launches++;
		if (cudaGetLastError() != cudaSuccess)
			rc = fail(NUCLEUS34_E_CUDA, "incidence kernels");
	} while (false);
	cleanup();
	return rc;
}

// The segmented sort above for other builders: every segment
// [off[s], off[s+1]) of keys (nseg < 2^32 segments) ascending, with the same
// three size classes and kernels as the incidence build.
int sort_segments_u64(Ctx &c, unsigned long long *keys, const uint64_t *off, uint64_t nseg)
{
	if (nseg == 0)
		return NUCLEUS34_OK;
	if (nseg > 0xffffffffull)
		return fail(NUCLEUS34_E_RANGE32, "segment count exceeds 32-bit segment ids");
	uint32_t *lists = nullptr, *counts = nullptr;
	unsigned long long *scratch = nullptr, *maxlen = nullptr;
	int rc = NUCLEUS34_OK;
	const EntryStore store{keys, nullptr, nullptr};
	do
	{
		if ((rc = dalloc(c, &lists, 3 * nseg, "segment lists")) || (rc = dalloc(c, &counts, 4, "segment counts")) ||
			(rc = dalloc(c, &maxlen, 1, "segment max")))
			break;
		if (cudaMemsetAsync(counts, 0, 16, c.stream) != cudaSuccess ||
			cudaMemsetAsync(maxlen, 0, 8, c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "memset");
			break;
		}
		k_seg_classify<<<grid_for(c, nseg, 256), 256, 0, c.stream>>>(off, nseg, lists, counts, nseg, maxlen);
		c.launches++;
		uint32_t hcounts[4] = {0, 0, 0, 0};
		unsigned long long hmax = 0;
		if (cudaMemcpyAsync(hcounts, counts, 16, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaMemcpyAsync(&hmax, maxlen, 8, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaStreamSynchronize(c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "segment classify");
			break;
		}
		if (hcounts[0])
		{
			k_seg_sort_warp<<<grid_for(c, hcounts[0], 8, 32), 256, 0, c.stream>>>(lists, counts + 0, off, store);
			c.launches++;
		}
		if (hcounts[1])
		{
			const size_t smem = SEG_SMEM * sizeof(unsigned long long);
			cudaFuncSetAttribute(k_seg_sort_block, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
			k_seg_sort_block<<<grid_for(c, hcounts[1], 1, 2), SEG_BLOCK, smem, c.stream>>>(lists + nseg,
																							counts + 1, off, store);
			c.launches++;
		}
		if (hcounts[2])
		{
			uint64_t P = 64;
			while (P < hmax)
				P <<= 1;
			if (P > 0xffffffffull)
			{
				rc = fail(NUCLEUS34_E_RANGE32, "segment longer than the sort's 32-bit index range");
				break;
			}
			const uint32_t blocks = std::min<uint32_t>(hcounts[2], uint32_t(c.sm_count));
			if ((rc = dalloc(c, &scratch, P * blocks, "segment sort scratch")))
				break;
			k_seg_sort_global<<<blocks, SEG_BLOCK, 0, c.stream>>>(lists + 2 * nseg, counts + 2, off, store, scratch,
																  P);
			c.launches++;
		}
		if (cudaGetLastError() != cudaSuccess)
			rc = fail(NUCLEUS34_E_CUDA, "segment sort kernels");
	} while (false);
	c.release(lists);
	c.release(counts);
	c.release(maxlen);
	c.release(scratch);
	return rc;
}

void free_incidence(Ctx &c, Incidence &inc)
{
	c.release(inc.span);
	c.release(inc.tpos);
	c.release(inc.third);
	c.release(inc.tri);
	inc = Incidence{};
}

} // namespace n34

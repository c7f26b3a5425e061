// Device exclusive scan (u32 or u64 in -> u64 out, out[n] = total), used for
// every CSR offset array of the pipeline (replaces thrust::inclusive_scan /
// exclusive_scan / lower_bound offset builds, nucleus/utils.cuh:410,1906;
// cuNucleus34.cu:650-653; cuNucleus34_ondemand.cu:546-549).
// Three phases: tile sums, scan of the tile sums (recursive), tile scan + base.
#include "common.cuh"

namespace n34 {

namespace {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ uint64_t block_exclusive_scan(uint64_t v, uint64_t *warp_sums, uint64_t &block_total)
{
	const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
	uint64_t x = v;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1)
	{
		uint64_t y = __shfl_up_sync(FULL, x, o);
		if (lane >= o)
			x += y;
	}
	if (lane == 31)
		warp_sums[wid] = x;
	__syncthreads();
	if (wid == 0)
	{
		uint64_t s = lane < (SCAN_THREADS / 32) ? warp_sums[lane] : 0;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1)
		{
			uint64_t y = __shfl_up_sync(FULL, s, o);
			if (lane >= o)
				s += y;
		}
		if (lane < (SCAN_THREADS / 32))
			warp_sums[lane] = s; // inclusive over warps
	}
	__syncthreads();
	const uint64_t warp_base = wid ? warp_sums[wid - 1] : 0;
	block_total = warp_sums[SCAN_THREADS / 32 - 1];
	return warp_base + x - v;
}

template <typename Tin>
__global__ void __launch_bounds__(SCAN_THREADS) k_tile_sums(const Tin *__restrict__ in, uint64_t n,
															uint64_t *__restrict__ sums)
{
	__shared__ uint64_t red[SCAN_THREADS / 32];
	const uint64_t base = uint64_t(blockIdx.x) * SCAN_TILE;
	uint64_t s = 0;
#pragma unroll
	for (int k = 0; k < SCAN_ITEMS; ++k)
	{
		const uint64_t i = base + uint64_t(k) * SCAN_THREADS + threadIdx.x;
		if (i < n)
			s += uint64_t(in[i]);
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		s += __shfl_down_sync(FULL, s, o);
	if ((threadIdx.x & 31) == 0)
		red[threadIdx.x >> 5] = s;
	__syncthreads();
	if (threadIdx.x == 0)
	{
		uint64_t t = 0;
		for (int w = 0; w < SCAN_THREADS / 32; ++w)
			t += red[w];
		sums[blockIdx.x] = t;
	}
}

template <typename Tin>
__global__ void __launch_bounds__(SCAN_THREADS) k_tile_scan(const Tin *__restrict__ in, uint64_t n,
															const uint64_t *__restrict__ tile_base,
															uint64_t *__restrict__ out)
{
	__shared__ uint64_t tile[SCAN_TILE];
	__shared__ uint64_t warp_sums[SCAN_THREADS / 32];
	const uint64_t base = uint64_t(blockIdx.x) * SCAN_TILE;
#pragma unroll
	for (int k = 0; k < SCAN_ITEMS; ++k)
	{
		const uint32_t j = uint32_t(k) * SCAN_THREADS + threadIdx.x;
		const uint64_t i = base + j;
		tile[j] = i < n ? uint64_t(in[i]) : 0;
	}
	__syncthreads();
	uint64_t local[SCAN_ITEMS];
	uint64_t run = 0;
#pragma unroll
	for (int k = 0; k < SCAN_ITEMS; ++k)
	{
		local[k] = run;
		run += tile[threadIdx.x * SCAN_ITEMS + k];
	}
	uint64_t total;
	const uint64_t tb = (tile_base ? tile_base[blockIdx.x] : 0);
	const uint64_t excl = block_exclusive_scan(run, warp_sums, total) + tb;
	__syncthreads();
#pragma unroll
	for (int k = 0; k < SCAN_ITEMS; ++k)
		tile[threadIdx.x * SCAN_ITEMS + k] = excl + local[k];
	__syncthreads();
#pragma unroll
	for (int k = 0; k < SCAN_ITEMS; ++k)
	{
		const uint32_t j = uint32_t(k) * SCAN_THREADS + threadIdx.x;
		const uint64_t i = base + j;
		if (i < n)
			out[i] = tile[j];
	}
	if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0)
		out[n] = tb + total;
}

template <typename Tin>
int scan_impl(Ctx &c, const Tin *in, uint64_t *out, uint64_t n)
{
	if (n == 0)
	{
		N34_CUDA(cudaMemsetAsync(out, 0, sizeof(uint64_t), c.stream));
		return NUCLEUS34_OK;
	}
	const uint64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
	if (tiles > 0x7fffffffull)
		return fail(NUCLEUS34_E_RANGE32, "scan too large");
	if (tiles == 1)
	{
		N34_LAUNCH(c, k_tile_scan<Tin>, 1, SCAN_THREADS, 0, in, n, nullptr, out);
		return NUCLEUS34_OK;
	}
	uint64_t *sums = nullptr, *bases = nullptr;
	N34_TRY(dalloc(c, &sums, tiles, "scan sums"));
	int rc = dalloc(c, &bases, tiles + 1, "scan bases");
	if (rc)
	{
		c.release(sums);
		return rc;
	}
	{
		k_tile_sums<Tin><<<uint32_t(tiles), SCAN_THREADS, 0, c.stream>>>(in, n, sums);
		c.launches++;
		rc = cudaGetLastError() == cudaSuccess ? 0 : fail(NUCLEUS34_E_CUDA, "scan launch");
		if (!rc)
			rc = scan_impl<uint64_t>(c, sums, bases, tiles);
		if (!rc)
		{
			k_tile_scan<Tin><<<uint32_t(tiles), SCAN_THREADS, 0, c.stream>>>(in, n, bases, out);
			c.launches++;
			rc = cudaGetLastError() == cudaSuccess ? 0 : fail(NUCLEUS34_E_CUDA, "scan launch");
		}
	}
	c.release(sums);
	c.release(bases);
	return rc;
}

} // namespace

int scan_u32(Ctx &c, const uint32_t *in, uint64_t *out, uint64_t n) { return scan_impl<uint32_t>(c, in, out, n); }
int scan_u64(Ctx &c, const uint64_t *in, uint64_t *out, uint64_t n) { return scan_impl<uint64_t>(c, in, out, n); }

} // namespace n34

// Triangle listing that allocates nothing.
//
// Some callers cannot allocate device memory while they run:
// - services that reserve all of HBM up front and hand slices of it out
//   themselves;
// - host processes whose framework allocator owns the device and would be
//   bypassed or starved by a cudaMalloc;
// - real-time loops where an allocation's latency or failure is not acceptable.
//
// nucleus34_list_triangles_noalloc serves them. The caller passes its own
// device buffers for the oriented CSR and the output triangle list, and every
// temporary of the two listing passes lives in the file-scope array below:
// per-vertex counts, output offsets, scan partials and a check flag. Its size
// is fixed, so the entry point accepts graphs of at most
// NOALLOC_MAX_VERTICES vertices.
//
// The array exists once per GPU that loads the library and stays allocated
// until the process exits. Every call on a device shares it and finds the
// previous call's contents there. Calls that overlap on the same GPU
// (different streams or host threads) race on it and must be serialised by
// the caller.
#include "pipeline.cuh"

#include <string>

namespace n34 {

namespace {

// 2^20 vertices: 4 MiB of counts + 8 MiB of offsets + scan partials.
constexpr uint64_t NOALLOC_MAX_VERTICES = uint64_t(1) << 20;
constexpr uint32_t NA_TILE = 2048; // scan tile (256 threads x 8)
constexpr uint64_t NA_MAX_TILES = (NOALLOC_MAX_VERTICES + NA_TILE - 1) / NA_TILE;
// layout, in 64-bit words
constexpr uint64_t NA_COUNTS = 0;                                   // u32[MAX]
constexpr uint64_t NA_OFFSETS = NA_COUNTS + NOALLOC_MAX_VERTICES / 2; // u64[MAX + 1]
constexpr uint64_t NA_TILE_SUMS = NA_OFFSETS + NOALLOC_MAX_VERTICES + 1;
constexpr uint64_t NA_TILE_BASES = NA_TILE_SUMS + NA_MAX_TILES;
constexpr uint64_t NA_FLAG = NA_TILE_BASES + NA_MAX_TILES + 1;
constexpr uint64_t NA_WORDS = NA_FLAG + 1;

static __device__ __align__(256) unsigned long long g_noalloc_scratch[NA_WORDS];

// Set-up, run at the start of every call with the call's device current: the
// address of the array as that device's current context sees it. Host code
// must not use the symbol's name as a pointer (it names a host-side stand-in).
// The address is not cached: a device reset reloads the module, and the array
// may then sit elsewhere; the lookup costs far less than the call's own
// synchronisation.
int scratch_for_current_device(unsigned long long **out)
{
	void *p = nullptr;
	const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
	if (e != cudaSuccess || !p)
	{
		cudaGetLastError();
		return fail(NUCLEUS34_E_CUDA, std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e));
	}
	*out = static_cast<unsigned long long *>(p);
	return NUCLEUS34_OK;
}

// Makes `device` current for the call and gives the caller's current device
// back on every return path.
struct DeviceGuard
{
	int saved = -1;
	cudaError_t enter(int device)
	{
		cudaError_t e = cudaGetDevice(&saved);
		if (e != cudaSuccess)
		{
			saved = -1;
			return e;
		}
		return saved == device ? cudaSuccess : cudaSetDevice(device);
	}
	~DeviceGuard()
	{
		int now = -1;
		if (saved >= 0 && cudaGetDevice(&now) == cudaSuccess && now != saved)
			cudaSetDevice(saved);
	}
};

// Same checks as the context upload: ids < n, no self-loops, ascending lists,
// O monotone with O[n] == m; and each undirected edge stored once: for an
// edge u->v, u must not be in N+(v) (a symmetric CSR would list every
// triangle more than once). Sets flag on any violation (the flag is cleared
// by the host before this kernel).
__global__ void k_na_validate(const uint32_t *__restrict__ O, const uint32_t *__restrict__ E, uint64_t n,
							  uint64_t m, unsigned long long *__restrict__ flag)
{
	const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
	if (blockIdx.x == 0 && threadIdx.x == 0 && uint64_t(O[n]) != m)
		atomicOr(flag, 1ull);
	for (uint64_t u = warp; u < n; u += nwarps)
	{
		const uint32_t b = O[u], e = O[u + 1];
		bool ok = b <= e && e <= m;
		for (uint32_t j = b + lane_id(); ok && j < e; j += 32)
		{
			const uint32_t v = E[j];
			if (v >= n || v == u || (j > b && E[j - 1] >= v))
				ok = false;
			else
			{
				// reverse edge v->u present? (N+(v) is searched only within [O[v], O[v+1]) <= m)
				const uint32_t vb = O[v], ve = O[v + 1];
				if (vb <= ve && ve <= m)
				{
					const uint64_t pos = lower_bound_u32(E, vb, ve, uint32_t(u));
					if (pos < ve && E[pos] == uint32_t(u))
						ok = false;
				}
			}
		}
		if (!__all_sync(FULL, ok) && lane_id() == 0)
			atomicOr(flag, 1ull);
	}
}

// Exclusive scan of u32 counts into u64 offsets (offsets[n] = total), tile
// sums -> one-block scan of the sums -> tile scans, all in the scratch.
__global__ void __launch_bounds__(256) k_na_tile_sums(const uint32_t *__restrict__ cnt, uint64_t n,
													  unsigned long long *__restrict__ sums)
{
	__shared__ unsigned long long red[8];
	const uint64_t base = uint64_t(blockIdx.x) * NA_TILE;
	unsigned long long s = 0;
	for (uint32_t k = 0; k < 8; ++k)
	{
		const uint64_t i = base + uint64_t(k) * 256 + threadIdx.x;
		if (i < n)
			s += cnt[i];
	}
	for (int o = 16; o > 0; o >>= 1)
		s += __shfl_down_sync(FULL, s, o);
	if ((threadIdx.x & 31) == 0)
		red[threadIdx.x >> 5] = s;
	__syncthreads();
	if (threadIdx.x == 0)
	{
		unsigned long long t = 0;
		for (int w = 0; w < 8; ++w)
			t += red[w];
		sums[blockIdx.x] = t;
	}
}

__global__ void __launch_bounds__(1024) k_na_scan_sums(const unsigned long long *__restrict__ sums, uint32_t tiles,
													   unsigned long long *__restrict__ bases)
{
	__shared__ unsigned long long sh[1024];
	// tiles <= NA_MAX_TILES = 512 <= blockDim
	const uint32_t i = threadIdx.x;
	sh[i] = i < tiles ? sums[i] : 0;
	__syncthreads();
	for (uint32_t o = 1; o < 1024; o <<= 1)
	{
		const unsigned long long v = i >= o ? sh[i - o] : 0;
		__syncthreads();
		sh[i] += v;
		__syncthreads();
	}
	if (i < tiles)
		bases[i] = i ? sh[i - 1] : 0; // exclusive
	if (i == 0)
		bases[tiles] = sh[tiles - 1];
}

__global__ void __launch_bounds__(256) k_na_tile_scan(const uint32_t *__restrict__ cnt, uint64_t n,
													  const unsigned long long *__restrict__ bases,
													  unsigned long long *__restrict__ off, uint32_t tiles)
{
	__shared__ unsigned long long tile[NA_TILE];
	__shared__ unsigned long long warp_sums[8];
	const uint64_t base = uint64_t(blockIdx.x) * NA_TILE;
	for (uint32_t k = 0; k < 8; ++k)
	{
		const uint32_t j = k * 256 + threadIdx.x;
		tile[j] = base + j < n ? cnt[base + j] : 0;
	}
	__syncthreads();
	unsigned long long local[8], run = 0;
	for (int k = 0; k < 8; ++k)
	{
		local[k] = run;
		run += tile[threadIdx.x * 8 + k];
	}
	// block exclusive scan of the per-thread runs
	const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
	unsigned long long x = run;
	for (int o = 1; o < 32; o <<= 1)
	{
		const unsigned long long y = __shfl_up_sync(FULL, x, o);
		if (lane >= uint32_t(o))
			x += y;
	}
	if (lane == 31)
		warp_sums[wid] = x;
	__syncthreads();
	unsigned long long wbase = 0;
	for (uint32_t w = 0; w < wid; ++w)
		wbase += warp_sums[w];
	const unsigned long long excl = bases[blockIdx.x] + wbase + x - run;
	__syncthreads();
	for (int k = 0; k < 8; ++k)
		tile[threadIdx.x * 8 + k] = excl + local[k];
	__syncthreads();
	for (uint32_t k = 0; k < 8; ++k)
	{
		const uint32_t j = k * 256 + threadIdx.x;
		if (base + j < n)
			off[base + j] = tile[j];
	}
	if (blockIdx.x == 0 && threadIdx.x == 0)
		off[n] = bases[tiles];
}

int list_noalloc(const uint32_t *d_O, const uint32_t *d_E, uint64_t n, uint64_t m, uint32_t *d_tris,
				 uint64_t capacity, uint64_t *count, int device, void *stream)
{
	if (!count)
		return fail(NUCLEUS34_E_INVALID, "null count output");
	*count = 0;
	if (n > NOALLOC_MAX_VERTICES)
		return fail(NUCLEUS34_E_INVALID, "graph has " + std::to_string(n) +
											 " vertices; the no-allocation listing handles at most " +
											 std::to_string(NOALLOC_MAX_VERTICES) +
											 " (its scratch is a fixed static array)");
	if (m > 0xffffffffull)
		return fail(NUCLEUS34_E_RANGE32, "edge count exceeds 32-bit edge ids");
	if (n == 0)
		return NUCLEUS34_OK;
	if (!d_O || (m && !d_E) || (capacity && !d_tris))
		return fail(NUCLEUS34_E_INVALID, "null device pointer");
	DeviceGuard guard;
	N34_CUDA(guard.enter(device));
	unsigned long long *scr = nullptr;
	N34_TRY(scratch_for_current_device(&scr));
	int sms = 0;
	N34_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
	if (sms < 1)
		sms = 1;
	cudaStream_t s = static_cast<cudaStream_t>(stream);
	uint32_t *cnt = reinterpret_cast<uint32_t *>(scr + NA_COUNTS);
	unsigned long long *off = scr + NA_OFFSETS;
	unsigned long long *sums = scr + NA_TILE_SUMS;
	unsigned long long *bases = scr + NA_TILE_BASES;
	unsigned long long *flag = scr + NA_FLAG;
	const uint32_t tiles = uint32_t((n + NA_TILE - 1) / NA_TILE);

	// the flag keeps the last call's value: clear it
	N34_CUDA(cudaMemsetAsync(flag, 0, sizeof(unsigned long long), s));
	{
		uint64_t g = (n + 7) / 8;
		g = g > uint64_t(sms) * 8 ? uint64_t(sms) * 8 : g;
		k_na_validate<<<uint32_t(g), 256, 0, s>>>(d_O, d_E, n, m, flag);
		N34_CUDA(cudaGetLastError());
	}
	unsigned long long hflag = 0;
	N34_CUDA(cudaMemcpyAsync(&hflag, flag, sizeof(hflag), cudaMemcpyDeviceToHost, s));
	N34_CUDA(cudaStreamSynchronize(s));
	if (hflag)
		return fail(NUCLEUS34_E_INVALID,
					"CSR must hold O[n] == m, ids < n, no self-loops, strictly ascending adjacency and each "
					"undirected edge once (no u->v beside v->u)");
	// pass 1 counts (every entry of cnt[0..n) is written), scan, pass 2 writes
	N34_CUDA(launch_tri_count(d_O, d_E, n, cnt, sms, s));
	k_na_tile_sums<<<tiles, 256, 0, s>>>(cnt, n, sums);
	N34_CUDA(cudaGetLastError());
	k_na_scan_sums<<<1, 1024, 0, s>>>(sums, tiles, bases);
	N34_CUDA(cudaGetLastError());
	k_na_tile_scan<<<tiles, 256, 0, s>>>(cnt, n, bases, off, tiles);
	N34_CUDA(cudaGetLastError());
	unsigned long long T = 0;
	N34_CUDA(cudaMemcpyAsync(&T, off + n, sizeof(T), cudaMemcpyDeviceToHost, s));
	N34_CUDA(cudaStreamSynchronize(s));
	*count = T;
	if (T == 0 || (!d_tris && capacity == 0)) // nothing to write, or a count-only query
		return NUCLEUS34_OK;
	if (T > capacity)
		return fail(NUCLEUS34_E_INVALID, "output holds " + std::to_string(capacity) + " triangles, the graph has " +
											 std::to_string(T) + " (the count is returned; call again with room)");
	N34_CUDA(launch_tri_write(d_O, d_E, n, reinterpret_cast<const uint64_t *>(off), d_tris, sms,
							  s));
	N34_CUDA(cudaStreamSynchronize(s));
	return NUCLEUS34_OK;
}

} // namespace

} // namespace n34

extern "C" int nucleus34_list_triangles_noalloc(const uint32_t *d_O, const uint32_t *d_E, uint64_t n, uint64_t m,
												uint32_t *d_tris, uint64_t tris_capacity,
												uint64_t *triangle_count, int device, void *stream)
{
	try
	{
		n34::clear_error();
		return n34::list_noalloc(d_O, d_E, n, m, d_tris, tris_capacity, triangle_count, device, stream);
	}
	catch (...)
	{
		return n34::fail(NUCLEUS34_E_INVALID, "unexpected host error");
	}
}

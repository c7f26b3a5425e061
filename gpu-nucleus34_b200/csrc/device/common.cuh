// Device-side building blocks shared by the sm_100a kernels of libnucleus34:
// warp helpers, bounded searches and the context that owns streams, budgeted
// allocations and launch accounting.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "nucleus34.h"
#include "tune.h"

namespace n34 {

int fail(int code, const std::string &msg);
void clear_error();

constexpr int WARP = 32;
constexpr uint32_t FULL = 0xffffffffu;

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint32_t lanemask_lt() { return (1u << lane_id()) - 1u; }

// First position in a[lo,hi) with a[pos] >= x.
__device__ __forceinline__ uint64_t lower_bound_u32(const uint32_t *__restrict__ a, uint64_t lo, uint64_t hi,
													uint32_t x)
{
	while (lo < hi)
	{
		const uint64_t mid = (lo + hi) >> 1;
		if (__ldg(a + mid) < x)
			lo = mid + 1;
		else
			hi = mid;
	}
	return lo;
}

// Same on 32-bit positions, branch-free: the trip count depends only on the
// window length, so lanes searching the same window stay converged.
__device__ __forceinline__ uint32_t lower_bound32(const uint32_t *__restrict__ a, uint32_t lo, uint32_t hi, uint32_t x)
{
	uint32_t n = hi - lo;
	while (n > 0)
	{
		const uint32_t half = n >> 1;
		const uint32_t mid = lo + half;
		const bool less = __ldg(a + mid) < x;
		lo = less ? mid + 1 : lo;
		n = less ? n - half - 1 : half;
	}
	return lo;
}

// Warp-aggregated append: every lane with pred set gets a distinct slot.
__device__ __forceinline__ uint32_t warp_append(bool pred, uint32_t *counter)
{
	const uint32_t mask = __ballot_sync(FULL, pred);
	uint32_t base = 0;
	const uint32_t leader = mask ? (__ffs(mask) - 1) : 0;
	if (mask && lane_id() == leader)
		base = atomicAdd(counter, __popc(mask));
	base = __shfl_sync(FULL, base, leader);
	return base + __popc(mask & lanemask_lt());
}

// Peel control block (device resident; one per run).
struct PeelCtl
{
	uint32_t level;      // current peel level
	uint32_t round;      // current round (death stamp)
	uint32_t nF;         // frontier size of this round
	uint32_t nNext;      // appended to the next frontier
	uint32_t cur;        // which frontier buffer is current (0/1)
	uint32_t minS;       // scan result: min alive support (0xffffffff = none)
	uint32_t done;       // 1 when every triangle is peeled
	uint32_t pad0;
	unsigned long long peeled;
	unsigned long long ksum;
	uint32_t kmax;
	uint32_t unpeeled;
	uint32_t rounds;
	uint32_t error;      // nonzero: a device-side check failed (code)
};

// Library context: one device, one stream, budgeted allocations.
struct Ctx
{
	int device = 0;
	int sm_count = 148;
	cudaStream_t stream = nullptr;
	uint64_t budget = 0;
	uint64_t in_use = 0;
	uint64_t peak = 0;
	uint64_t launches = 0;
	std::vector<TuneRule> tune_rules; // the context's tune table (empty: defaults)
	bool tune_pinned = false;         // settings pinned by nucleus34_ctx_set_tune
	nucleus34_tune tune_pin{};
	nucleus34_tune tune = tune_filled(nucleus34_tune{}); // settings of the current / last run
	uint32_t opt_flags = 0;
	double peel_debit_sec = 0; // profiling only: debit kernels' device time
	bool lean_run = false;     // this run uses the memory-lean layout
	std::mutex mu;

	// resident graph
	uint64_t n = 0, m = 0;
	uint32_t max_out = 0;   // maximum out-degree (the tune table's skew class)
	uint32_t *dO = nullptr; // n+1
	uint32_t *dE = nullptr; // m
	uint32_t *dsrc = nullptr; // m

	// results of the last run
	bool have_result = false;
	int variant = 0;
	uint64_t T = 0, Q = 0;
	uint32_t *dtris = nullptr; // 3T
	int32_t *dK = nullptr;     // T
	uint32_t *dquds = nullptr; // 4Q (direct)
	uint32_t *dR = nullptr;    // T death rounds (kept with NUCLEUS34_OPT_VERIFIABLE)
	nucleus34_result res{};

	// Segments (batched graphs decomposed as one disjoint union): seg_eoff
	// holds count+1 edge offsets of the member graphs; empty for a single
	// graph. After a run the per-segment triangle offsets, clique counts and
	// k statistics are in the host vectors.
	std::vector<uint64_t> seg_eoff;
	std::vector<uint64_t> seg_toff, seg_q, seg_ksum;
	std::vector<uint32_t> seg_kmax;
	uint64_t *dseg = nullptr; // device: eoff (count+1), toff (count+1), q, ksum (count), kmax (count, u32 words)

	std::unordered_map<void *, uint64_t> sizes; // live allocations
	// Released blocks kept for reuse by a later allocation of the same size
	// on this context's stream (contexts that run the same graph again: every
	// run then finds its blocks, and the device pool never has to grow in
	// the middle of a phase). Off unless keep_blocks; trimmed when the budget
	// or the device needs the memory, and when the context is destroyed.
	bool keep_blocks = false;
	std::unordered_multimap<uint64_t, void *> kept;
	uint64_t kept_bytes = 0;

	int alloc(void **p, uint64_t bytes, const char *what);
	void release(void *p);
	void trim_kept();
	void release_results();
	void release_graph();
};

// Host vectors whose resize leaves new elements uninitialised, for large
// buffers that are written in full right after (batch unions and slices).
template <class T>
struct NoInitAlloc : std::allocator<T>
{
	template <class U>
	struct rebind
	{
		using other = NoInitAlloc<U>;
	};
	NoInitAlloc() = default;
	template <class U>
	NoInitAlloc(const NoInitAlloc<U> &) noexcept
	{
	}
	template <class U>
	void construct(U *p) noexcept
	{
		::new (static_cast<void *>(p)) U;
	}
	template <class U, class... A>
	void construct(U *p, A &&...a)
	{
		::new (static_cast<void *>(p)) U(std::forward<A>(a)...);
	}
};
using HostU32 = std::vector<uint32_t, NoInitAlloc<uint32_t>>;

template <class T>
inline int dalloc(Ctx &c, T **p, uint64_t count, const char *what)
{
	return c.alloc(reinterpret_cast<void **>(p), count * sizeof(T), what);
}

#define N34_CUDA(expr)                                                                          \
	do                                                                                          \
	{                                                                                           \
		cudaError_t e__ = (expr);                                                               \
		if (e__ != cudaSuccess)                                                                 \
			return ::n34::fail(NUCLEUS34_E_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e__)); \
	} while (0)

#define N34_TRY(expr)        \
	do                       \
	{                        \
		int r__ = (expr);    \
		if (r__ != 0)        \
			return r__;      \
	} while (0)

// Launch with accounting; checks the launch itself.
#define N34_LAUNCH(ctx, kernel, grid, block, smem, ...)                                     \
	do                                                                                      \
	{                                                                                       \
		kernel<<<(grid), (block), (smem), (ctx).stream>>>(__VA_ARGS__);                     \
		(ctx).launches++;                                                                   \
		cudaError_t e__ = cudaGetLastError();                                               \
		if (e__ != cudaSuccess)                                                             \
			return ::n34::fail(NUCLEUS34_E_CUDA, std::string("launch " #kernel ": ") + cudaGetErrorString(e__)); \
	} while (0)

inline uint32_t grid_for(const Ctx &c, uint64_t items, uint32_t per_block, uint32_t max_per_sm = 16)
{
	uint64_t g = (items + per_block - 1) / per_block;
	const uint64_t cap = uint64_t(c.sm_count) * max_per_sm;
	if (g > cap)
		g = cap;
	if (g == 0)
		g = 1;
	return uint32_t(g);
}

// exclusive scan: out[0..n] with out[n] = total; in may be u32 or u64
int scan_u32(Ctx &c, const uint32_t *in, uint64_t *out, uint64_t n);
int scan_u64(Ctx &c, const uint64_t *in, uint64_t *out, uint64_t n);

} // namespace n34

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
#include "intersect.cuh"
#include "pipeline.cuh"

namespace n34 {

namespace {

constexpr uint32_t INF = 0xffffffffu;
constexpr int PEEL_THREADS = 256;

struct CtlX
{
	PeelCtl c;
	uint32_t scan; // 1 while the next frontier must come from a scan
};

__global__ void k_peel_init(int32_t *__restrict__ K, uint64_t T, CtlX *ctl)
{
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < T; t += stride)
		K[t] = -1;
	if (blockIdx.x == 0 && threadIdx.x == 0)
	{
		PeelCtl z{};
		z.minS = INF;
		ctl->c = z;
		ctl->scan = 1;
	}
}

__global__ void __launch_bounds__(PEEL_THREADS) k_scan_min(CtlX *ctl, const int32_t *__restrict__ S,
														   const int32_t *__restrict__ K, uint64_t T)
{
	if (ctl->c.done || !ctl->scan)
		return;
	uint32_t mn = INF;
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < T; t += stride)
		if (K[t] == -1)
		{
			const int32_t s = S[t];
			mn = min(mn, uint32_t(s < 0 ? 0 : s));
		}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		mn = min(mn, __shfl_xor_sync(FULL, mn, o));
	if (lane_id() == 0 && mn != INF)
		atomicMin(&ctl->c.minS, mn);
}

__global__ void __launch_bounds__(PEEL_THREADS) k_gather(CtlX *ctl, const int32_t *__restrict__ S,
														 const int32_t *__restrict__ K, uint64_t T,
														 uint32_t *__restrict__ F0, uint32_t *__restrict__ F1)
{
	if (ctl->c.done || !ctl->scan)
		return;
	const uint32_t mn = ctl->c.minS;
	if (mn == INF)
	{
		if (blockIdx.x == 0 && threadIdx.x == 0)
			ctl->c.done = 1;
		return;
	}
	if (blockIdx.x == 0 && threadIdx.x == 0)
		ctl->c.level = max(ctl->c.level, mn);
	uint32_t *F = ctl->c.cur ? F1 : F0;
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t t0 = uint64_t(blockIdx.x) * blockDim.x; t0 < T; t0 += stride)
	{
		const uint64_t t = t0 + threadIdx.x;
		bool take = false;
		if (t < T && K[t] == -1)
		{
			const int32_t s = S[t];
			take = uint32_t(s < 0 ? 0 : s) <= mn;
		}
		const uint32_t slot = warp_append(take, &ctl->c.nF);
		if (take)
		{
			if (slot < T)
				F[slot] = uint32_t(t);
			else
				atomicOr(&ctl->c.error, 1u);
		}
	}
}

__global__ void k_mark(CtlX *ctl, const uint32_t *__restrict__ F0, const uint32_t *__restrict__ F1,
					   int32_t *__restrict__ K, uint32_t *__restrict__ R)
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

__global__ void __launch_bounds__(PEEL_THREADS) k_debit_ondemand(
	CtlX *ctl, uint32_t *__restrict__ F0, uint32_t *__restrict__ F1, const uint32_t *__restrict__ tris,
	const uint64_t *__restrict__ incO, const uint32_t *__restrict__ third, const uint32_t *__restrict__ itri,
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
		const uint32_t a = __ldg(tris + 3 * uint64_t(t)), b = __ldg(tris + 3 * uint64_t(t) + 1),
					   c = __ldg(tris + 3 * uint64_t(t) + 2);
		warp_intersect3(third, incO[a], incO[a + 1], incO[b], incO[b + 1], incO[c], incO[c + 1],
						[&](bool found, uint32_t, uint64_t pd, uint64_t p1, uint64_t p2) {
							uint32_t q0 = 0, q1 = 0, q2 = 0;
							if (found)
							{
								q0 = __ldg(itri + pd);
								q1 = __ldg(itri + p1);
								q2 = __ldg(itri + p2);
							}
							settle_clique(found, t, q0, q1, q2, K, R, S, round, level, Fn, &ctl->c.nNext, T, &ctl->c.error);
						});
	}
}

__global__ void __launch_bounds__(PEEL_THREADS) k_debit_direct(
	CtlX *ctl, uint32_t *__restrict__ F0, uint32_t *__restrict__ F1, const uint64_t *__restrict__ coff,
	const uint32_t *__restrict__ cids, const uint4 *__restrict__ quds, const int32_t *__restrict__ K,
	const uint32_t *__restrict__ R, int32_t *__restrict__ S, uint64_t T)
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
			const bool found = j < e;
			uint32_t q0 = 0, q1 = 0, q2 = 0;
			if (found)
			{
				const uint4 q = quds[cids[j]];
				// the three members other than t
				const uint32_t m[4] = {q.x, q.y, q.z, q.w};
				uint32_t o[3];
				int k = 0;
#pragma unroll
				for (int s = 0; s < 4; ++s)
					if (m[s] != t && k < 3)
						o[k++] = m[s];
				q0 = o[0];
				q1 = o[1];
				q2 = o[2];
			}
			settle_clique(found, t, q0, q1, q2, K, R, S, round, level, Fn, &ctl->c.nNext, T, &ctl->c.error);
		}
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

} // namespace

int peel(Ctx &c, int variant, const Incidence &inc, const CliqueCsr &csr, int32_t *S, int32_t *K, PeelCtl *hctl)
{
	const uint64_t T = c.T;
	uint32_t *R = nullptr, *F0 = nullptr, *F1 = nullptr;
	CtlX *ctl = nullptr;
	int rc = NUCLEUS34_OK;
	auto cleanup = [&] {
		c.release(R);
		c.release(F0);
		c.release(F1);
		c.release(ctl);
	};
	do
	{
		if ((rc = dalloc(c, &R, T, "peel round stamps")))
			break;
		if ((rc = dalloc(c, &F0, T, "frontier 0")))
			break;
		if ((rc = dalloc(c, &F1, T, "frontier 1")))
			break;
		if ((rc = dalloc(c, &ctl, 1, "peel control")))
			break;
		const uint32_t gscan = grid_for(c, T, PEEL_THREADS, 8);
		const uint32_t gwarp = grid_for(c, T, PEEL_THREADS / 32, 16);
		k_peel_init<<<gscan, PEEL_THREADS, 0, c.stream>>>(K, T, ctl);
		c.launches++;
		// Bounded host loop: at most one peel per triangle per round and each
		// level costs at least one round, so T + levels + a margin bounds it.
		const uint64_t max_rounds = 2 * T + 4096;
		uint64_t rounds = 0;
		uint32_t batch = 4;
		bool done = false;
		while (!done)
		{
			for (uint32_t r = 0; r < batch; ++r)
			{
				k_scan_min<<<gscan, PEEL_THREADS, 0, c.stream>>>(ctl, S, K, T);
				k_gather<<<gscan, PEEL_THREADS, 0, c.stream>>>(ctl, S, K, T, F0, F1);
				k_mark<<<gscan, PEEL_THREADS, 0, c.stream>>>(ctl, F0, F1, K, R);
				if (variant == NUCLEUS34_ONDEMAND)
					k_debit_ondemand<<<gwarp, PEEL_THREADS, 0, c.stream>>>(ctl, F0, F1, c.dtris, inc.off, inc.third,
																		   inc.tri, K, R, S, T);
				else
					k_debit_direct<<<gwarp, PEEL_THREADS, 0, c.stream>>>(
						ctl, F0, F1, csr.off, csr.ids, reinterpret_cast<const uint4 *>(c.dquds), K, R, S, T);
				k_advance<<<1, 1, 0, c.stream>>>(ctl);
				c.launches += 5;
			}
			rounds += batch;
			uint32_t hdone = 0;
			if (cudaGetLastError() != cudaSuccess ||
				cudaMemcpyAsync(&hdone, &ctl->c.done, 4, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
				cudaStreamSynchronize(c.stream) != cudaSuccess)
			{
				rc = fail(NUCLEUS34_E_CUDA, std::string("peel rounds: ") + cudaGetErrorString(cudaGetLastError()));
				break;
			}
			done = hdone != 0;
			if (!done && rounds > max_rounds)
			{
				rc = fail(NUCLEUS34_E_TIMEOUT, "peel did not converge within its round bound");
				break;
			}
			if (batch < 64)
				batch *= 2;
		}
		if (rc)
			break;
		k_stats<<<gscan, PEEL_THREADS, 0, c.stream>>>(ctl, K, T);
		c.launches++;
		if (cudaMemcpyAsync(hctl, &ctl->c, sizeof(PeelCtl), cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaStreamSynchronize(c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "peel stats");
			break;
		}
		if (hctl->error)
		{
			rc = fail(NUCLEUS34_E_CUDA, "internal: peel frontier overflow");
			break;
		}
	} while (false);
	cleanup();
	return rc;
}

} // namespace n34

// Batched decomposition: many independent graphs in one device pass.
//
// The graphs are decomposed as their disjoint union. Vertex ids of graph g
// are shifted by the vertices before it and its oriented edges follow the
// edges before it, so:
//   - orientation ((deg, id) order between the two ends of an edge) and the
//     ascending adjacency of every vertex are those of the graph alone;
//   - triangles and four-cliques never span two graphs, and the canonical
//     (a,b) order of the union lists graph 0's triangles first, each graph's
//     in its own canonical order (edge ids shifted by the graph's offset);
//   - the (3,4)-nucleus number of a triangle depends only on the cliques of
//     its own graph, so every k equals the one of the graph decomposed alone.
// One pipeline (listing, incidence, support, peel) then serves the whole
// batch: one set of launches and one peel whose rounds advance all graphs at
// once, instead of a launch sequence per graph. Per-graph counts and k
// statistics come from segment reductions over the shared arrays.
//
// The reference has no batched form (one graph per process); every graph's
// results keep the reference's per-graph semantics.
#include "pipeline.cuh"

#include <algorithm>
#include <chrono>
#include <string>
#include <vector>

// A batch is split into chunks whose unions stay within the 32-bit entry
// positions of the incidence (3T < 2^32); each chunk is one device pass in
// its own context, and its results stay resident until nucleus34_batch_free,
// unless they were moved to host memory (hk, htris) to make room for a later
// pass; the context then keeps only the per-graph statistics.
struct BatchChunk
{
	nucleus34_ctx ctx = nullptr;
	uint64_t first = 0, count = 0; // member graphs [first, first + count)
	bool on_host = false;
	std::vector<int32_t> hk;      // T (on_host)
	std::vector<uint32_t> htris;  // 3T (on_host)
};

struct nucleus34_batch_s
{
	std::vector<BatchChunk> chunks;
	std::vector<uint32_t> chunk_of; // graph -> chunk
	uint64_t count = 0;
};

namespace n34 {

namespace {

// first triangle whose edge a is >= the segment's first edge
__global__ void k_seg_tri_offsets(const uint32_t *__restrict__ tris, uint64_t T, const uint64_t *__restrict__ eoff,
								  uint64_t count, uint64_t *__restrict__ toff)
{
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; g <= count; g += stride)
	{
		const uint64_t e = eoff[g];
		uint64_t lo = 0, n = T;
		while (n > 0)
		{
			const uint64_t half = n >> 1;
			const bool less = uint64_t(tris[3 * (lo + half)]) < e;
			lo = less ? lo + half + 1 : lo;
			n = less ? n - half - 1 : half;
		}
		toff[g] = lo;
	}
}

// warp per segment: sum of the support (each clique counted by its 4 triangles)
__global__ void k_seg_support(const int32_t *__restrict__ S, const uint64_t *__restrict__ toff, uint64_t count,
							  unsigned long long *__restrict__ q)
{
	const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
	for (uint64_t g = warp; g < count; g += nwarps)
	{
		unsigned long long acc = 0;
		for (uint64_t t = toff[g] + lane_id(); t < toff[g + 1]; t += 32)
			acc += uint64_t(uint32_t(S[t]));
#pragma unroll
		for (int o = 16; o > 0; o >>= 1)
			acc += __shfl_xor_sync(FULL, acc, o);
		if (lane_id() == 0)
			q[g] = acc;
	}
}

__global__ void k_seg_kstats(const int32_t *__restrict__ K, const uint64_t *__restrict__ toff, uint64_t count,
							 unsigned long long *__restrict__ ksum, uint32_t *__restrict__ kmax)
{
	const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
	for (uint64_t g = warp; g < count; g += nwarps)
	{
		unsigned long long acc = 0;
		uint32_t mx = 0;
		for (uint64_t t = toff[g] + lane_id(); t < toff[g + 1]; t += 32)
		{
			const int32_t k = K[t];
			const uint32_t kk = k < 0 ? 0u : uint32_t(k);
			acc += kk;
			mx = kk > mx ? kk : mx;
		}
#pragma unroll
		for (int o = 16; o > 0; o >>= 1)
		{
			acc += __shfl_xor_sync(FULL, acc, o);
			mx = max(mx, __shfl_xor_sync(FULL, mx, o));
		}
		if (lane_id() == 0)
		{
			ksum[g] = acc;
			kmax[g] = mx;
		}
	}
}

// triangles per member graph from per-vertex counts (warp per graph)
__global__ void k_seg_vertex_sums(const uint32_t *__restrict__ cnt, const uint64_t *__restrict__ voff, uint64_t count,
								  unsigned long long *__restrict__ out)
{
	const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
	for (uint64_t g = warp; g < count; g += nwarps)
	{
		unsigned long long acc = 0;
		for (uint64_t u = voff[g] + lane_id(); u < voff[g + 1]; u += 32)
			acc += cnt[u];
#pragma unroll
		for (int o = 16; o > 0; o >>= 1)
			acc += __shfl_xor_sync(FULL, acc, o);
		if (lane_id() == 0)
			out[g] = acc;
	}
}

// device layout of c.dseg
struct SegView
{
	uint64_t *eoff, *toff;
	unsigned long long *q, *ksum;
	uint32_t *kmax;
};

SegView seg_view(Ctx &c)
{
	const uint64_t n = c.seg_eoff.size() - 1;
	SegView v;
	v.eoff = c.dseg;
	v.toff = v.eoff + (n + 1);
	v.q = reinterpret_cast<unsigned long long *>(v.toff + (n + 1));
	v.ksum = v.q + n;
	v.kmax = reinterpret_cast<uint32_t *>(v.ksum + n);
	return v;
}

uint64_t seg_words(uint64_t n) { return 2 * (n + 1) + 2 * n + (n + 1) / 2 + 1; }

} // namespace

int segments_after_listing(Ctx &c)
{
	if (c.seg_eoff.empty())
		return NUCLEUS34_OK;
	const uint64_t n = c.seg_eoff.size() - 1;
	if (!c.dseg)
	{
		N34_TRY(dalloc(c, &c.dseg, seg_words(n), "batch segments"));
		N34_CUDA(cudaMemsetAsync(c.dseg, 0, seg_words(n) * 8, c.stream));
		N34_CUDA(cudaMemcpyAsync(c.dseg, c.seg_eoff.data(), (n + 1) * 8, cudaMemcpyHostToDevice, c.stream));
	}
	const SegView v = seg_view(c);
	N34_LAUNCH(c, k_seg_tri_offsets, grid_for(c, n + 1, 256), 256, 0, c.dtris, c.T, v.eoff, n, v.toff);
	return NUCLEUS34_OK;
}

int segments_after_support(Ctx &c, const int32_t *support)
{
	if (c.seg_eoff.empty())
		return NUCLEUS34_OK;
	const uint64_t n = c.seg_eoff.size() - 1;
	const SegView v = seg_view(c);
	if (c.T)
		N34_LAUNCH(c, k_seg_support, grid_for(c, n, 8), 256, 0, support, v.toff, n, v.q);
	else
		N34_CUDA(cudaMemsetAsync(v.q, 0, n * 8, c.stream));
	return NUCLEUS34_OK;
}

int segments_after_peel(Ctx &c)
{
	if (c.seg_eoff.empty())
		return NUCLEUS34_OK;
	const uint64_t n = c.seg_eoff.size() - 1;
	const SegView v = seg_view(c);
	if (c.T)
		N34_LAUNCH(c, k_seg_kstats, grid_for(c, n, 8), 256, 0, c.dK, v.toff, n, v.ksum, v.kmax);
	else
	{
		N34_CUDA(cudaMemsetAsync(v.ksum, 0, n * 8, c.stream));
		N34_CUDA(cudaMemsetAsync(v.kmax, 0, n * 4, c.stream));
	}
	c.seg_toff.assign(n + 1, 0);
	c.seg_q.assign(n, 0);
	c.seg_ksum.assign(n, 0);
	c.seg_kmax.assign(n, 0);
	N34_CUDA(cudaMemcpyAsync(c.seg_toff.data(), v.toff, (n + 1) * 8, cudaMemcpyDeviceToHost, c.stream));
	N34_CUDA(cudaMemcpyAsync(c.seg_q.data(), v.q, n * 8, cudaMemcpyDeviceToHost, c.stream));
	N34_CUDA(cudaMemcpyAsync(c.seg_ksum.data(), v.ksum, n * 8, cudaMemcpyDeviceToHost, c.stream));
	N34_CUDA(cudaMemcpyAsync(c.seg_kmax.data(), v.kmax, n * 4, cudaMemcpyDeviceToHost, c.stream));
	N34_CUDA(cudaStreamSynchronize(c.stream));
	for (auto &q : c.seg_q)
		q /= 4;
	return NUCLEUS34_OK;
}

// Builds the union CSR of the member graphs on the host.
int build_union(const nucleus34_csr *graphs, uint64_t count, HostU32 &O, HostU32 &D, HostU32 &E,
				std::vector<uint64_t> &voff, std::vector<uint64_t> &eoff)
{
	voff.assign(count + 1, 0);
	eoff.assign(count + 1, 0);
	for (uint64_t g = 0; g < count; ++g)
	{
		const nucleus34_csr &x = graphs[g];
		if ((x.n && !x.D) || (x.m && !x.E))
			return fail(NUCLEUS34_E_INVALID, "batch graph " + std::to_string(g) + ": null CSR array");
		voff[g + 1] = voff[g] + x.n;
		eoff[g + 1] = eoff[g] + x.m;
	}
	if (voff[count] >= 0xffffffffull || eoff[count] > 0xffffffffull)
		return fail(NUCLEUS34_E_RANGE32, "batch union exceeds 32-bit vertex/edge ids");
	O.resize(voff[count] + 1);
	D.resize(voff[count]);
	E.resize(eoff[count]);
	// member graphs in parallel (disjoint ranges); a graph that fails its
	// checks records why, and the first such graph is reported
	std::vector<uint8_t> why(count, 0);
#pragma omp parallel for schedule(dynamic, 8)
	for (int64_t gi = 0; gi < int64_t(count); ++gi)
	{
		const uint64_t g = uint64_t(gi);
		const nucleus34_csr &x = graphs[g];
		uint64_t s = eoff[g];
		for (uint64_t u = 0; u < x.n; ++u)
		{
			O[voff[g] + u] = uint32_t(s);
			D[voff[g] + u] = x.D[u];
			s += x.D[u];
		}
		if (s != eoff[g + 1])
		{
			why[g] = 1;
			continue;
		}
		const uint32_t vo = uint32_t(voff[g]);
		for (uint64_t j = 0; j < x.m; ++j)
		{
			if (x.E[j] >= x.n)
			{
				why[g] = 2;
				break;
			}
			E[eoff[g] + j] = x.E[j] + vo;
		}
	}
	for (uint64_t g = 0; g < count; ++g)
		if (why[g])
			return fail(NUCLEUS34_E_INVALID, "batch graph " + std::to_string(g) +
												 (why[g] == 1 ? ": sum of D does not equal m" : ": edge id out of range"));
	O[voff[count]] = uint32_t(eoff[count]);
	return NUCLEUS34_OK;
}

// Triangles of every member graph: the listing's count pass over the union
// already uploaded to c, summed per graph.
int triangles_per_graph(Ctx &c, const std::vector<uint64_t> &voff, std::vector<uint64_t> &tcount)
{
	const uint64_t count = voff.size() - 1;
	tcount.assign(count, 0);
	if (!c.m)
		return NUCLEUS34_OK;
	uint32_t *cnt = nullptr;
	uint64_t *dv = nullptr;
	unsigned long long *dout = nullptr;
	int rc = NUCLEUS34_OK;
	do
	{
		if ((rc = dalloc(c, &cnt, c.n, "batch triangle counts")) || (rc = dalloc(c, &dv, count + 1, "batch offsets")) ||
			(rc = dalloc(c, &dout, count, "batch sums")))
			break;
		if (launch_tri_count(c.dO, c.dE, c.n, cnt, c.sm_count, c.stream) != cudaSuccess ||
			cudaMemcpyAsync(dv, voff.data(), (count + 1) * 8, cudaMemcpyHostToDevice, c.stream) != cudaSuccess)
		{
			rc = fail(NUCLEUS34_E_CUDA, "batch triangle count");
			break;
		}
		k_seg_vertex_sums<<<grid_for(c, count, 8), 256, 0, c.stream>>>(cnt, dv, count, dout);
		c.launches += 2;
		if (cudaMemcpyAsync(tcount.data(), dout, count * 8, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
			cudaStreamSynchronize(c.stream) != cudaSuccess)
			rc = fail(NUCLEUS34_E_CUDA, "batch triangle count");
	} while (false);
	c.release(cnt);
	c.release(dv);
	c.release(dout);
	return rc;
}

// Union of the member graphs [first, last) of the full union (O, D, E),
// re-based to start at vertex 0 and edge 0.
void slice_union(const HostU32 &O, const HostU32 &D, const HostU32 &E, const std::vector<uint64_t> &voff,
				 const std::vector<uint64_t> &eoff, uint64_t first, uint64_t last, HostU32 &So, HostU32 &Sd,
				 HostU32 &Se)
{
	const uint64_t v0 = voff[first], v1 = voff[last], e0 = eoff[first], e1 = eoff[last];
	So.resize(v1 - v0 + 1);
	Sd.resize(v1 - v0);
	Se.resize(e1 - e0);
#pragma omp parallel for schedule(static)
	for (int64_t u = int64_t(v0); u <= int64_t(v1); ++u)
	{
		So[uint64_t(u) - v0] = uint32_t(O[uint64_t(u)] - e0);
		if (uint64_t(u) < v1)
			Sd[uint64_t(u) - v0] = D[uint64_t(u)];
	}
#pragma omp parallel for schedule(static)
	for (int64_t j = int64_t(e0); j < int64_t(e1); ++j)
		Se[uint64_t(j) - e0] = uint32_t(E[uint64_t(j)] - v0);
}

} // namespace n34

using namespace n34;

// Moves a finished pass's k and triangle list to host memory and frees its
// device memory (results and graph); the per-graph statistics stay.
static int move_results_to_host(BatchChunk &ch)
{
	Ctx &c = ch.ctx->c;
	std::lock_guard<std::mutex> lk(c.mu);
	if (ch.on_host)
		return NUCLEUS34_OK;
	N34_CUDA(cudaSetDevice(c.device));
	const uint64_t T = c.T;
	ch.hk.resize(T);
	ch.htris.resize(3 * T);
	if (T)
	{
		N34_CUDA(cudaMemcpyAsync(ch.hk.data(), c.dK, T * 4, cudaMemcpyDeviceToHost, c.stream));
		N34_CUDA(cudaMemcpyAsync(ch.htris.data(), c.dtris, T * 12, cudaMemcpyDeviceToHost, c.stream));
	}
	N34_CUDA(cudaStreamSynchronize(c.stream));
	std::vector<uint64_t> toff = std::move(c.seg_toff), q = std::move(c.seg_q), ks = std::move(c.seg_ksum);
	std::vector<uint32_t> km = std::move(c.seg_kmax);
	c.release_results();
	c.release_graph();
	c.seg_toff = std::move(toff);
	c.seg_q = std::move(q);
	c.seg_ksum = std::move(ks);
	c.seg_kmax = std::move(km);
	N34_CUDA(cudaStreamSynchronize(c.stream));
	ch.on_host = true;
	return NUCLEUS34_OK;
}

// Device memory a new context could use now: free memory plus what the
// stream-ordered pool holds unused, at the 90% a default budget takes.
static uint64_t device_room(int dev)
{
	size_t fb = 0, tb = 0;
	if (cudaSetDevice(dev) != cudaSuccess || cudaMemGetInfo(&fb, &tb) != cudaSuccess)
	{
		cudaGetLastError();
		return 0;
	}
	uint64_t cached = 0;
	cudaMemPool_t pool;
	uint64_t reserved = 0, used = 0;
	if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess &&
		cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
		cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess && reserved > used)
		cached = reserved - used;
	cudaGetLastError();
	return uint64_t(double(fb + cached) * 0.9);
}

template <class F>
static int batch_guarded(F &&f)
{
	clear_error();
	try
	{
		return f();
	}
	catch (const std::bad_alloc &)
	{
		return fail(NUCLEUS34_E_OOM_BUDGET, "host allocation failed");
	}
	catch (const std::exception &e)
	{
		return fail(NUCLEUS34_E_INVALID, e.what());
	}
}

extern "C" {

int nucleus34_batch_decompose(const nucleus34_csr *graphs, uint64_t count, const nucleus34_opts *opts,
							  nucleus34_batch_result *res, nucleus34_batch *out)
{
	if (!graphs || !count || !out)
		return fail(NUCLEUS34_E_INVALID, "null argument or empty batch");
	*out = nullptr;
	return batch_guarded([&]() -> int {
		const auto h0 = std::chrono::steady_clock::now();
		HostU32 O, D, E;
		std::vector<uint64_t> voff, eoff;
		N34_TRY(build_union(graphs, count, O, D, E, voff, eoff));
		auto *b = new (std::nothrow) nucleus34_batch_s();
		if (!b)
			return fail(NUCLEUS34_E_OOM_BUDGET, "host allocation failed");
		b->count = count;
		b->chunk_of.assign(count, 0);
		nucleus34_batch_result br{};
		br.graphs = count;
		double t_upload = 0;
		auto finish = [&](int rc) {
			if (rc)
				nucleus34_batch_free(b);
			return rc;
		};
		// pass 0: the whole union, counted per graph
		nucleus34_ctx ctx0 = nullptr;
		int rc = create_ctx(opts, &ctx0);
		if (rc)
			return finish(rc);
		{
			const nucleus34_csr u{voff[count], eoff[count], O.data(), D.data(), E.empty() ? nullptr : E.data()};
			rc = upload(ctx0->c, &u);
		}
		std::vector<uint64_t> tcount;
		if (!rc)
			rc = triangles_per_graph(ctx0->c, voff, tcount);
		if (rc)
		{
			destroy_ctx(ctx0);
			return finish(rc);
		}
		// chunks: greedy in graph order, 3T < 2^32 entry positions each, at
		// most FLAG_PEEL_MAX_TRIANGLES (so that every pass of several graphs
		// peels with death flags), and about PASS_BYTES_PER_TRIANGLE bytes of a
		// pass's peak per triangle within the memory budget (a single graph
		// over that still runs alone)
		constexpr uint64_t PASS_BYTES_PER_TRIANGLE = 80;
		const uint64_t range_limit = 0xffffffffull / 3;
		const uint64_t csr_bytes = 4 * (voff[count] + 1) + 8 * eoff[count];
		const uint64_t budget = ctx0->c.budget;
		const uint64_t mem_limit = budget > csr_bytes ? (budget - csr_bytes) / PASS_BYTES_PER_TRIANGLE : 0;
		const uint64_t limit =
			std::max<uint64_t>(1, std::min(std::min(range_limit, FLAG_PEEL_MAX_TRIANGLES), mem_limit));
		std::vector<uint64_t> cut{0};
		uint64_t acc = 0;
		for (uint64_t g = 0; g < count; ++g)
		{
			if (tcount[g] > range_limit)
			{
				destroy_ctx(ctx0);
				return finish(fail(NUCLEUS34_E_RANGE32, "batch graph " + std::to_string(g) + " alone has " +
															 std::to_string(tcount[g]) + " triangles (incidence "
															 "exceeds the 32-bit position range)"));
			}
			if (acc && acc + tcount[g] > limit)
			{
				cut.push_back(g);
				acc = 0;
			}
			acc += tcount[g];
		}
		cut.push_back(count);
		const uint64_t nchunks = cut.size() - 1;
		t_upload += std::chrono::duration<double>(std::chrono::steady_clock::now() - h0).count();
		const bool to_host = opts && (opts->flags & NUCLEUS34_OPT_HOST_RESULTS);
		const int dev = opts ? opts->device : 0;
		for (uint64_t ci = 0; ci < nchunks; ++ci)
		{
			const uint64_t f = cut[ci], l = cut[ci + 1];
			const auto c0 = std::chrono::steady_clock::now();
			if (ci > 0 && !b->chunks.back().on_host)
			{
				// the results kept on the device must leave room for this pass
				uint64_t tri = 0;
				for (uint64_t g = f; g < l; ++g)
					tri += tcount[g];
				const uint64_t need = PASS_BYTES_PER_TRIANGLE * tri + 4 * (voff[l] - voff[f] + 1) +
									  8 * (eoff[l] - eoff[f]);
				if (to_host || need > device_room(dev))
					for (auto &ch : b->chunks)
						if ((rc = move_results_to_host(ch)))
							return finish(rc);
			}
			nucleus34_ctx ctx = nullptr;
			if (nchunks == 1)
			{
				ctx = ctx0; // the union is already resident
				ctx0 = nullptr;
			}
			else
			{
				if (ctx0)
				{
					destroy_ctx(ctx0);
					ctx0 = nullptr;
				}
				if ((rc = create_ctx(opts, &ctx)))
					return finish(rc);
				HostU32 So, Sd, Se;
				slice_union(O, D, E, voff, eoff, f, l, So, Sd, Se);
				const nucleus34_csr u{voff[l] - voff[f], eoff[l] - eoff[f], So.data(), Sd.data(),
									  Se.empty() ? nullptr : Se.data()};
				if ((rc = upload(ctx->c, &u)))
				{
					destroy_ctx(ctx);
					return finish(rc);
				}
			}
			b->chunks.push_back(BatchChunk{ctx, f, l - f});
			for (uint64_t g = f; g < l; ++g)
				b->chunk_of[g] = uint32_t(ci);
			Ctx &c = ctx->c;
			c.seg_eoff.resize(l - f + 1);
			for (uint64_t g = f; g <= l; ++g)
				c.seg_eoff[g - f] = eoff[g] - eoff[f];
			t_upload += std::chrono::duration<double>(std::chrono::steady_clock::now() - c0).count();
			nucleus34_result r{};
			if ((rc = run(c, NUCLEUS34_ONDEMAND, &r)))
				return finish(rc);
			br.triangle_count += r.triangle_count;
			br.four_clique_count += r.four_clique_count;
			br.peeling_iterations += r.peeling_iterations;
			br.t_triangles += r.t_triangles;
			br.t_incidence += r.t_incidence;
			br.t_support += r.t_support;
			br.t_peel += r.t_peel;
			br.t_total += r.t_total;
			br.gpu_launches += r.gpu_launches;
			br.peak_device_bytes = std::max<uint64_t>(br.peak_device_bytes, r.peak_device_bytes);
		}
		if (to_host)
			for (auto &ch : b->chunks)
				if ((rc = move_results_to_host(ch)))
					return finish(rc);
		br.t_upload = t_upload;
		br.chunks = nchunks;
		if (res)
			*res = br;
		*out = b;
		return int(NUCLEUS34_OK);
	});
}

static const BatchChunk *chunk_for(nucleus34_batch b, uint64_t index, uint64_t *local)
{
	if (!b || index >= b->count)
		return nullptr;
	const BatchChunk &ch = b->chunks[b->chunk_of[index]];
	*local = index - ch.first;
	return &ch;
}

int nucleus34_batch_summary(nucleus34_batch b, uint64_t index, nucleus34_graph_summary *out)
{
	uint64_t i = 0;
	const BatchChunk *ch = chunk_for(b, index, &i);
	if (!ch || !out)
		return fail(NUCLEUS34_E_INVALID, "null argument or graph index out of range");
	const Ctx &c = ch->ctx->c;
	if (c.seg_toff.size() != ch->count + 1)
		return fail(NUCLEUS34_E_STATE, "batch has no result");
	nucleus34_graph_summary s{};
	s.triangle_count = c.seg_toff[i + 1] - c.seg_toff[i];
	s.four_clique_count = c.seg_q[i];
	s.k_max = c.seg_kmax[i];
	// same arithmetic as a single decomposition: 64-bit integer sum / T
	s.k_avg = s.triangle_count ? double(c.seg_ksum[i]) / double(s.triangle_count) : 0.0;
	*out = s;
	return NUCLEUS34_OK;
}

int nucleus34_batch_copy_k(nucleus34_batch b, uint64_t index, int32_t *k_out, uint32_t *tris_out)
{
	uint64_t i = 0;
	const BatchChunk *ch = chunk_for(b, index, &i);
	if (!ch)
		return fail(NUCLEUS34_E_INVALID, "null argument or graph index out of range");
	return batch_guarded([&]() -> int {
		Ctx &c = ch->ctx->c;
		std::lock_guard<std::mutex> lk(c.mu);
		if (c.seg_toff.size() != ch->count + 1)
			return fail(NUCLEUS34_E_STATE, "batch has no result");
		const uint64_t t0 = c.seg_toff[i], T = c.seg_toff[i + 1] - t0;
		if (!T)
			return int(NUCLEUS34_OK);
		if (ch->on_host)
		{
			if (k_out)
				std::copy(ch->hk.begin() + t0, ch->hk.begin() + t0 + T, k_out);
			if (tris_out)
			{
				const uint32_t eo = uint32_t(c.seg_eoff[i]);
				for (uint64_t j = 0; j < 3 * T; ++j)
					tris_out[j] = ch->htris[3 * t0 + j] - eo;
			}
			return int(NUCLEUS34_OK);
		}
		N34_CUDA(cudaSetDevice(c.device));
		if (k_out)
			N34_CUDA(cudaMemcpyAsync(k_out, c.dK + t0, T * 4, cudaMemcpyDeviceToHost, c.stream));
		if (tris_out)
			N34_CUDA(cudaMemcpyAsync(tris_out, c.dtris + 3 * t0, T * 12, cudaMemcpyDeviceToHost, c.stream));
		N34_CUDA(cudaStreamSynchronize(c.stream));
		if (tris_out)
		{
			// edge ids of the graph alone
			const uint32_t eo = uint32_t(c.seg_eoff[i]);
			for (uint64_t j = 0; j < 3 * T; ++j)
				tris_out[j] -= eo;
		}
		return int(NUCLEUS34_OK);
	});
}

void nucleus34_batch_free(nucleus34_batch b)
{
	if (!b)
		return;
	for (auto &ch : b->chunks)
		destroy_ctx(ch.ctx);
	delete b;
}

} // extern "C"

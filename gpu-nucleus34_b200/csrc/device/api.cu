// C-ABI of the decomposition: contexts (device, stream, budgeted memory,
// resident graph), the pipeline driver and the result accessors.
//
// Reference counterparts: the two programs' device pipelines
// (nucleus/cuNucleus34.cu:283-721, nucleus/cuNucleus34_ondemand.cu:407-690);
// their CSR upload (cuNucleus34.cu:290-293) is nucleus34_ctx_upload, their
// phase timers (hrc::now() around synchronised phases) become CUDA events on
// the library stream.
#include "pipeline.cuh"

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <new>
#include <string>
#include <unordered_map>
#include <vector>

#include <omp.h>

struct nucleus34_state
{
	nucleus34_ctx ctx = nullptr;
};

namespace n34 {

void clear_error();

namespace {

__global__ void k_validate(const uint32_t *__restrict__ O, const uint32_t *__restrict__ E, uint64_t n,
						   uint32_t *__restrict__ bad)
{
	const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
	for (uint64_t u = warp; u < n; u += nwarps)
	{
		const uint32_t b = O[u], e = O[u + 1];
		bool ok = b <= e;
		for (uint32_t j = b + lane_id(); ok && j < e; j += 32)
		{
			const uint32_t v = E[j];
			if (v >= n || v == u || (j > b && E[j - 1] >= v))
				ok = false;
		}
		if (!ok)
			atomicOr(bad, 1u);
	}
}

__global__ void k_zero_k(int32_t *K, uint64_t T)
{
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < T; t += stride)
		K[t] = 0;
}

struct Events
{
	cudaEvent_t e[6] = {};
	bool ok = true;
	explicit Events()
	{
		for (auto &x : e)
			ok = ok && cudaEventCreate(&x) == cudaSuccess;
	}
	~Events()
	{
		for (auto &x : e)
			if (x)
				cudaEventDestroy(x);
	}
	double sec(int a, int b)
	{
		float ms = 0.f;
		if (cudaEventElapsedTime(&ms, e[a], e[b]) != cudaSuccess)
			return 0.0;
		return double(ms) * 1e-3;
	}
};

int set_device(Ctx &c)
{
	N34_CUDA(cudaSetDevice(c.device));
	return NUCLEUS34_OK;
}

} // namespace

// Failure injection for tests of the error paths: with
// NUCLEUS34_FAIL_ALLOC_AT=N in the environment, the process's Nth device
// allocation fails once with E_OOM_BUDGET (a host-side fake of an
// out-of-memory; no device fault). Read once; unset means never.
static bool injected_alloc_failure()
{
	static std::atomic<long long> countdown{[] {
		const char *v = std::getenv("NUCLEUS34_FAIL_ALLOC_AT");
		const long long n = v ? std::atoll(v) : 0;
		return n > 0 ? n : 0LL;
	}()};
	if (countdown.load(std::memory_order_relaxed) <= 0)
		return false;
	return countdown.fetch_sub(1) == 1;
}

int Ctx::alloc(void **p, uint64_t bytes, const char *what)
{
	*p = nullptr;
	if (injected_alloc_failure())
		return fail(NUCLEUS34_E_OOM_BUDGET, std::string("injected allocation failure (NUCLEUS34_FAIL_ALLOC_AT) at ") +
												what);
	if (bytes == 0)
		bytes = 16;
	bytes = (bytes + 255) & ~uint64_t(255);
	auto hit = kept.find(bytes);
	if (hit != kept.end())
	{
		*p = hit->second;
		kept.erase(hit);
		kept_bytes -= bytes;
		in_use += bytes;
		peak = std::max(peak, in_use);
		sizes[*p] = bytes;
		return NUCLEUS34_OK;
	}
	if (in_use + kept_bytes + bytes > budget)
		trim_kept();
	if (in_use + bytes > budget)
		return fail(NUCLEUS34_E_OOM_BUDGET, std::string("device memory budget exceeded allocating ") + what + " (" +
												std::to_string(bytes >> 20) + " MiB; in use " +
												std::to_string(in_use >> 20) + " of " + std::to_string(budget >> 20) +
												" MiB)");
	cudaError_t e = cudaMallocAsync(p, bytes, stream);
	if (e == cudaErrorMemoryAllocation && kept_bytes)
	{
		cudaGetLastError();
		trim_kept();
		e = cudaMallocAsync(p, bytes, stream);
	}
	if (e != cudaSuccess)
	{
		cudaGetLastError();
		*p = nullptr;
		return fail(e == cudaErrorMemoryAllocation ? NUCLEUS34_E_OOM_BUDGET : NUCLEUS34_E_CUDA,
					std::string("cudaMallocAsync ") + what + ": " + cudaGetErrorString(e));
	}
	in_use += bytes;
	peak = std::max(peak, in_use);
	sizes[*p] = bytes;
	return NUCLEUS34_OK;
}

void Ctx::release(void *p)
{
	if (!p)
		return;
	auto it = sizes.find(p);
	if (it != sizes.end())
	{
		in_use -= it->second;
		if (keep_blocks)
		{
			kept.emplace(it->second, p);
			kept_bytes += it->second;
			sizes.erase(it);
			return;
		}
		sizes.erase(it);
	}
	cudaFreeAsync(p, stream);
}

void Ctx::trim_kept()
{
	for (auto &kv : kept)
		cudaFreeAsync(kv.second, stream);
	kept.clear();
	kept_bytes = 0;
}

void Ctx::release_results()
{
	release(dseg);
	dseg = nullptr;
	seg_toff.clear();
	seg_q.clear();
	seg_ksum.clear();
	seg_kmax.clear();
	release(dR);
	dR = nullptr;
	release(dtris);
	release(dK);
	release(dquds);
	dtris = nullptr;
	dK = nullptr;
	dquds = nullptr;
	T = Q = 0;
	have_result = false;
}

void Ctx::release_graph()
{
	release(dO);
	release(dE);
	release(dsrc);
	dO = dE = dsrc = nullptr;
	n = m = 0;
	max_out = 0;
}

// The upload proper; upload() below releases the validation flag and, on any
// failure, the partly uploaded graph, so that a failed upload leaves no graph
// that a later run could take for a valid one.
static int upload_graph(Ctx &c, const nucleus34_csr *csr, uint32_t *&bad)
{
	const uint64_t n = csr->n, m = csr->m;
	std::vector<uint32_t> O(n + 1);
	uint64_t s = 0;
	uint32_t max_out = 0;
	for (uint64_t u = 0; u < n; ++u)
	{
		if (csr->O && csr->O[u] != s)
			return fail(NUCLEUS34_E_INVALID, "O is not the exclusive scan of D");
		O[u] = uint32_t(s);
		s += csr->D[u];
		max_out = csr->D[u] > max_out ? csr->D[u] : max_out;
	}
	if (s != m)
		return fail(NUCLEUS34_E_INVALID, "sum of D does not equal m");
	O[n] = uint32_t(m);
	N34_TRY(dalloc(c, &c.dO, n + 1, "CSR offsets"));
	N34_TRY(dalloc(c, &c.dE, m ? m : 1, "CSR destinations"));
	N34_TRY(dalloc(c, &c.dsrc, m ? m : 1, "CSR sources"));
	N34_CUDA(cudaMemcpyAsync(c.dO, O.data(), (n + 1) * 4, cudaMemcpyHostToDevice, c.stream));
	if (m)
		N34_CUDA(cudaMemcpyAsync(c.dE, csr->E, m * 4, cudaMemcpyHostToDevice, c.stream));
	c.n = n;
	c.m = m;
	c.max_out = max_out;
	N34_TRY(dalloc(c, &bad, 1, "validation flag"));
	N34_CUDA(cudaMemsetAsync(bad, 0, 4, c.stream));
	if (n)
		N34_LAUNCH(c, k_validate, grid_for(c, n, 8), 256, 0, c.dO, c.dE, n, bad);
	uint32_t hbad = 0;
	N34_CUDA(cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, c.stream));
	N34_CUDA(cudaStreamSynchronize(c.stream));
	if (hbad)
		return fail(NUCLEUS34_E_INVALID, "CSR adjacency must hold ids < n, no self-loops, strictly ascending per vertex");
	N34_TRY(build_src(c));
	N34_CUDA(cudaStreamSynchronize(c.stream));
	return NUCLEUS34_OK;
}

int upload(Ctx &c, const nucleus34_csr *csr)
{
	if (!csr || (csr->n && !csr->D) || (csr->m && !csr->E))
		return fail(NUCLEUS34_E_INVALID, "null CSR array");
	if (csr->m > 0xffffffffull || csr->n >= 0xffffffffull)
		return fail(NUCLEUS34_E_RANGE32, "graph exceeds 32-bit vertex/edge ids");
	N34_TRY(set_device(c));
	c.release_results();
	c.release_graph();
	c.seg_eoff.clear();
	uint32_t *bad = nullptr;
	const int rc = upload_graph(c, csr, bad);
	c.release(bad);
	if (rc)
	{
		cudaStreamSynchronize(c.stream);
		c.release_graph();
	}
	return rc;
}

// Settings of this run: the direct variant keeps the defaults (its clique
// order must not depend on them); the on-demand one takes the pinned
// settings, else the tune table's line for the graph's class, else the
// defaults. Called once T is known.
void select_tune(Ctx &c, int variant)
{
	c.tune = tune_filled(nucleus34_tune{});
	if (variant != NUCLEUS34_ONDEMAND)
		return;
	if (c.tune_pinned)
	{
		c.tune = tune_filled(c.tune_pin);
		return;
	}
	if (c.tune_rules.empty())
		return;
	int32_t size = 0, skew = 0;
	tune_class(c.T, c.n, c.m, c.max_out, size, skew);
	if (const TuneRule *r = tune_match(c.tune_rules, size, skew))
		c.tune = tune_filled(r->tune);
}

int run(Ctx &c, int variant, nucleus34_result *out)
{
	if (variant != NUCLEUS34_DIRECT && variant != NUCLEUS34_ONDEMAND)
		return fail(NUCLEUS34_E_INVALID, "unknown variant");
	if (!c.dO)
		return fail(NUCLEUS34_E_STATE, "no graph uploaded");
	N34_TRY(set_device(c));
	c.release_results();
	const uint64_t launches0 = c.launches;
	c.peak = c.in_use;
	Events ev;
	if (!ev.ok)
		return fail(NUCLEUS34_E_CUDA, "event creation");
	nucleus34_result r{};
	r.variant = variant;
	Incidence inc;
	CliqueCsr csr;
	int32_t *S = nullptr;
	uint32_t *own = nullptr;
	int rc = NUCLEUS34_OK;
	PeelCtl pc{};
	bool peeled = false;
	do
	{
		c.peel_debit_sec = 0;
		N34_CUDA(cudaEventRecord(ev.e[0], c.stream));
		if ((rc = list_triangles(c)))
			break;
		if ((rc = segments_after_listing(c)))
			break;
		N34_CUDA(cudaEventRecord(ev.e[1], c.stream));
		r.triangle_count = c.T;
		r.incidence_entries = 3 * c.T;
		select_tune(c, variant);
		// The incidence is addressed with 32-bit positions, the limit the
		// reference also enforces (cuNucleus34_ondemand.cu:505-511).
		if (3 * c.T > 0xffffffffull)
		{
			rc = fail(NUCLEUS34_E_RANGE32, "incidence size " + std::to_string(3 * c.T) +
											   " exceeds the 32-bit position range");
			break;
		}
		c.lean_run = false;
		if (c.T)
		{
			// The on-demand peel with death flags (T < 2^30) uses either the
			// regular layout (64-bit sort keys beside the entries, each
			// triangle's entry positions, two frontier lists, k apart from the
			// support: about 60 bytes per triangle at the incidence build) or,
			// by request or when that does not fit in the memory left, the
			// memory-lean one (entries sorted in place, no entry positions,
			// bitmap frontiers, k kept in the support array: about 28 bytes
			// per triangle beside the triangle list).
			const bool flags_path = variant == NUCLEUS34_ONDEMAND && c.T <= 0x3fffffffull &&
									!(c.opt_flags & NUCLEUS34_OPT_STAMP_PEEL);
			const uint64_t room = c.budget > c.in_use ? c.budget - c.in_use : 0;
			const uint64_t regular = 60 * c.T + 40 * c.m;
			c.lean_run = flags_path && ((c.opt_flags & NUCLEUS34_OPT_LEAN_MEMORY) || regular > room);
			const bool want_tpos = flags_path && !c.lean_run;
			if ((rc = build_incidence(c, inc, want_tpos, c.lean_run)))
				break;
			r.sum_te_sq = inc.sum_te_sq;
		}
		N34_CUDA(cudaEventRecord(ev.e[2], c.stream));
		uint64_t total = 0;
		if (c.T)
		{
			if ((rc = dalloc(c, &S, c.T, "support")))
				break;
			if (variant == NUCLEUS34_DIRECT && (rc = dalloc(c, &own, c.T, "clique owner counts")))
				break;
			if ((rc = count_support(c, inc, S, &total, own)))
				break;
			if (total % 4)
			{
				rc = fail(NUCLEUS34_E_CUDA, "internal: clique incidences not a multiple of 4");
				break;
			}
		}
		if ((rc = segments_after_support(c, S)))
			break;
		r.four_clique_count = total / 4;
		N34_CUDA(cudaEventRecord(ev.e[3], c.stream));
		if (variant == NUCLEUS34_DIRECT && total)
		{
			if ((rc = list_cliques(c, inc, S, own, csr)))
				break;
			if (c.Q != total / 4)
			{
				rc = fail(NUCLEUS34_E_CUDA, "internal: clique list size differs from support total");
				break;
			}
		}
		c.release(own);
		own = nullptr;
		if (variant == NUCLEUS34_DIRECT)
			free_incidence(c, inc);
		N34_CUDA(cudaEventRecord(ev.e[4], c.stream));
		if (c.T && c.lean_run)
		{
			// k is kept in the support array and becomes the result
			if (total)
			{
				if ((rc = peel(c, variant, inc, csr, S, S, &pc)))
					break;
				peeled = true;
			}
			else
			{
				N34_LAUNCH(c, k_zero_k, grid_for(c, c.T, 256), 256, 0, S, c.T);
			}
			c.dK = S;
			S = nullptr;
		}
		else if (c.T)
		{
			if ((rc = dalloc(c, &c.dK, c.T, "k values")))
				break;
			if (total)
			{
				if ((rc = peel(c, variant, inc, csr, S, c.dK, &pc)))
					break;
				peeled = true;
			}
			else
			{
				N34_LAUNCH(c, k_zero_k, grid_for(c, c.T, 256), 256, 0, c.dK, c.T);
			}
		}
		N34_CUDA(cudaEventRecord(ev.e[5], c.stream));
		if ((rc = segments_after_peel(c)))
			break;
		N34_CUDA(cudaStreamSynchronize(c.stream));
	} while (false);
	free_incidence(c, inc);
	free_clique_csr(c, csr);
	c.release(S);
	c.release(own);
	if (rc)
	{
		c.release_results();
		cudaStreamSynchronize(c.stream);
		return rc;
	}
	r.t_triangles = ev.sec(0, 1);
	r.t_incidence = ev.sec(1, 2);
	r.t_support = ev.sec(2, 3);
	r.t_cliques = ev.sec(3, 4);
	r.t_peel = ev.sec(4, 5);
	r.t_peel_debit = c.peel_debit_sec;
	r.t_total = r.t_triangles + r.t_incidence + r.t_support + r.t_cliques + r.t_peel;
	if (peeled)
	{
		r.peeling_iterations = pc.rounds;
		r.unpeeled_count = pc.unpeeled;
		r.k_max = pc.kmax;
		r.k_avg = c.T ? double(pc.ksum) / double(c.T) : 0.0;
	}
	r.gpu_launches = c.launches - launches0;
	r.peak_device_bytes = c.peak;
	c.variant = variant;
	c.have_result = true;
	c.res = r;
	if (out)
		*out = r;
	return NUCLEUS34_OK;
}

int copy_k(Ctx &c, int32_t *k_out, uint32_t *tris_out)
{
	if (!c.have_result)
		return fail(NUCLEUS34_E_STATE, "no result");
	N34_TRY(set_device(c));
	if (k_out && c.T)
		N34_CUDA(cudaMemcpyAsync(k_out, c.dK, c.T * 4, cudaMemcpyDeviceToHost, c.stream));
	if (tris_out && c.T)
		N34_CUDA(cudaMemcpyAsync(tris_out, c.dtris, c.T * 12, cudaMemcpyDeviceToHost, c.stream));
	N34_CUDA(cudaStreamSynchronize(c.stream));
	return NUCLEUS34_OK;
}

// Autotuner: coordinate descent over the settings of the on-demand variant.
// Every trial is a full run whose k is compared with the default run's.
int autotune(Ctx &c, const char *path, nucleus34_tune *best_out, double *best_sec, double *default_sec)
{
	if (!c.dO)
		return fail(NUCLEUS34_E_STATE, "no graph uploaded");
	const bool pinned0 = c.tune_pinned;
	const nucleus34_tune pin0 = c.tune_pin;
	std::vector<int32_t> ref, got;
	nucleus34_result r0{};
	bool have_ref = false;
	// one run under t, timed on the device (t_total); the first one sets the
	// reference result
	auto trial = [&](const nucleus34_tune &t, double &sec) -> int {
		c.tune_pinned = true;
		c.tune_pin = t;
		nucleus34_result r{};
		N34_TRY(run(c, NUCLEUS34_ONDEMAND, &r));
		sec = r.t_total;
		std::vector<int32_t> &dst = have_ref ? got : ref;
		dst.resize(c.T);
		N34_TRY(copy_k(c, dst.data(), nullptr));
		if (!have_ref)
		{
			r0 = r;
			have_ref = true;
		}
		else if (r.triangle_count != r0.triangle_count || r.four_clique_count != r0.four_clique_count ||
				 got != ref)
			return fail(NUCLEUS34_E_CUDA, "autotune: the settings " + tune_line(TuneRule{0, 0, t, 0, 0, 0}) +
											  " changed the result");
		return NUCLEUS34_OK;
	};
	auto body = [&]() -> int {
		const nucleus34_tune def = tune_filled(nucleus34_tune{});
		double s0 = 0, s1 = 0, s2 = 0;
		N34_TRY(trial(def, s0)); // warm-up and reference
		N34_TRY(trial(def, s1));
		N34_TRY(trial(def, s2));
		const double t_def = std::min(s1, s2);
		nucleus34_tune best = def;
		double t_best = t_def;
		const uint32_t NEVER = NUCLEUS34_TUNE_NEVER;
		// candidates around each default; replay length and compaction
		// frequency move the peel the most, so they get the finest steps
		const std::vector<uint32_t> lanes = {8, 16, 32}, divs = {4, 6, 8, 12, 16, NEVER},
									shifts = {10, 11, 12, 13, 14, NEVER}, rounds = {8, 12, 16, 24, 32};
		using Member = uint32_t nucleus34_tune::*;
		struct Field
		{
			Member f;
			const std::vector<uint32_t> *values;
		};
		const Field fields[] = {{&nucleus34_tune::lane_max, &lanes},
								{&nucleus34_tune::compact_div, &divs},
								{&nucleus34_tune::sort_shift, &shifts},
								{&nucleus34_tune::rounds_per_replay, &rounds}};
		for (const Field &fd : fields)
			for (uint32_t v : *fd.values)
			{
				if (best.*fd.f == v)
					continue;
				nucleus34_tune cand = best;
				cand.*fd.f = v;
				double a = 0, b = 0;
				N34_TRY(trial(cand, a));
				if (a >= 0.99 * t_best)
					continue;
				N34_TRY(trial(cand, b)); // confirm: both runs 1% faster
				if (b >= 0.99 * t_best)
					continue;
				best = cand;
				t_best = 0.5 * (a + b);
			}
		if (best_out)
			*best_out = best;
		if (best_sec)
			*best_sec = t_best;
		if (default_sec)
			*default_sec = t_def;
		if (path)
		{
			TuneRule rule;
			tune_class(c.T, c.n, c.m, c.max_out, rule.size, rule.skew);
			rule.tune = best;
			rule.sec = t_best;
			rule.default_sec = t_def;
			N34_TRY(tune_store(path, rule));
			// later unpinned runs of this context use the new line too
			bool replaced = false;
			for (auto &x : c.tune_rules)
				if (x.size == rule.size && x.skew == rule.skew)
				{
					x = rule;
					replaced = true;
				}
			if (!replaced)
				c.tune_rules.push_back(rule);
		}
		return NUCLEUS34_OK;
	};
	const int rc = body();
	c.tune_pinned = pinned0;
	c.tune_pin = pin0;
	return rc;
}

// One k-file row "(a,b,c)\t<k>\n" (the reference's format,
// cuNucleus34_ondemand.cu:724-733) at p, returning its length: the same bytes
// as printf's "%u" and "%d", without the format parsing (at most 47 bytes).
static inline char *put_u32(char *p, uint32_t v)
{
	char tmp[10];
	int n = 0;
	do
	{
		tmp[n++] = char('0' + v % 10);
		v /= 10;
	} while (v);
	while (n)
		*p++ = tmp[--n];
	return p;
}

static inline size_t kfile_row(char *line, uint32_t a, uint32_t b, uint32_t c, int32_t k)
{
	char *p = line;
	*p++ = '(';
	p = put_u32(p, a);
	*p++ = ',';
	p = put_u32(p, b);
	*p++ = ',';
	p = put_u32(p, c);
	*p++ = ')';
	*p++ = '\t';
	if (k < 0)
	{
		*p++ = '-';
		p = put_u32(p, uint32_t(0) - uint32_t(k));
	}
	else
		p = put_u32(p, uint32_t(k));
	*p++ = '\n';
	return size_t(p - line);
}

int write_kfile(Ctx &c, const char *path)
{
	std::vector<int32_t> k(c.T);
	std::vector<uint32_t> t(3 * c.T);
	N34_TRY(copy_k(c, k.data(), t.data()));
	FILE *f = std::fopen(path, "wb");
	if (!f)
		return fail(NUCLEUS34_E_IO, std::string("Failed to open output file: ") + path);
	const uint64_t T = c.T, chunk = 1u << 18;
	const uint64_t nchunks = (T + chunk - 1) / chunk;
	bool ok = true;
	// format chunks in parallel, write them in order
	for (uint64_t c0 = 0; c0 < nchunks && ok; c0 += 64)
	{
		const uint64_t c1 = std::min(nchunks, c0 + 64);
		std::vector<std::string> bufs(c1 - c0);
#pragma omp parallel for schedule(dynamic, 1)
		for (int64_t ci = int64_t(c0); ci < int64_t(c1); ++ci)
		{
			std::string &b = bufs[size_t(ci - int64_t(c0))];
			const uint64_t s = uint64_t(ci) * chunk, e = std::min(T, s + chunk);
			b.resize((e - s) * 48); // the longest row is 47 bytes
			size_t len = 0;
			for (uint64_t i = s; i < e; ++i)
				len += kfile_row(&b[len], t[3 * i], t[3 * i + 1], t[3 * i + 2], k[i]);
			b.resize(len);
		}
		for (auto &b : bufs)
			ok = ok && std::fwrite(b.data(), 1, b.size(), f) == b.size();
	}
	ok = (std::fclose(f) == 0) && ok;
	return ok ? NUCLEUS34_OK : fail(NUCLEUS34_E_IO, "short write");
}

int create_ctx(const nucleus34_opts *opts, nucleus34_ctx *out)
{
	*out = nullptr;
	int dev = opts ? opts->device : 0;
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
	{
		cudaGetLastError();
		return fail(NUCLEUS34_E_NODEVICE, "no CUDA device visible");
	}
	if (dev < 0 || dev >= ndev)
		return fail(NUCLEUS34_E_INVALID, "device ordinal out of range");
	// a tune table is read and checked up front: a bad one fails the call
	std::vector<TuneRule> rules;
	if (opts && opts->tune_table)
		N34_TRY(tune_read(opts->tune_table, rules));
	cudaDeviceProp prop{};
	N34_CUDA(cudaGetDeviceProperties(&prop, dev));
	if (prop.major < 10)
		return fail(NUCLEUS34_E_NODEVICE, std::string("this build targets sm_100a; device is ") + prop.name);
	N34_CUDA(cudaSetDevice(dev));
	auto *x = new (std::nothrow) nucleus34_ctx_s();
	if (!x)
		return fail(NUCLEUS34_E_INVALID, "host allocation failed");
	Ctx &c = x->c;
	c.device = dev;
	c.tune_rules = std::move(rules);
	c.sm_count = prop.multiProcessorCount;
	if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess)
	{
		delete x;
		return fail(NUCLEUS34_E_CUDA, "stream creation");
	}
	// Keep freed blocks mapped in the stream-ordered pool between phases and
	// runs: re-mapping tens of GB costs far more than the kernels themselves.
	{
		cudaMemPool_t pool;
		if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess)
		{
			uint64_t thr = UINT64_MAX;
			cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
		}
		cudaGetLastError();
	}
	size_t fb = 0, tb = 0;
	cudaMemGetInfo(&fb, &tb);
	// memory cached in the pool by earlier calls is available to this one too
	uint64_t cached = 0;
	{
		cudaMemPool_t pool;
		uint64_t reserved = 0, used = 0;
		if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess &&
			cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
			cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess && reserved > used)
			cached = reserved - used;
		cudaGetLastError();
	}
	c.budget = (opts && opts->mem_budget_bytes) ? opts->mem_budget_bytes : uint64_t(double(fb + cached) * 0.9);
	if (opts)
		c.opt_flags = opts->flags;
	*out = x;
	return NUCLEUS34_OK;
}

void destroy_ctx(nucleus34_ctx x)
{
	if (!x)
		return;
	Ctx &c = x->c;
	cudaSetDevice(c.device);
	c.release_results();
	c.release_graph();
	c.trim_kept();
	c.keep_blocks = false;
	for (auto &kv : c.sizes)
		cudaFreeAsync(kv.first, c.stream);
	c.sizes.clear();
	if (c.stream)
	{
		cudaStreamSynchronize(c.stream);
		cudaStreamDestroy(c.stream);
	}
	// the freed blocks stay cached in the device's pool for the next call;
	// nucleus34_release_cached_memory returns them to the driver
	delete x;
}

template <class F>
int guarded(F &&f)
{
	clear_error();
	try
	{
		return f();
	}
	catch (const std::bad_alloc &)
	{
		return fail(NUCLEUS34_E_INVALID, "host allocation failed");
	}
	catch (const std::exception &e)
	{
		return fail(NUCLEUS34_E_INVALID, e.what());
	}
	catch (...)
	{
		return fail(NUCLEUS34_E_INVALID, "unknown error");
	}
}

int decompose_impl(const nucleus34_csr *csr, const nucleus34_opts *opts, nucleus34_result *res,
				   nucleus34_handle *out, int variant)
{
	if (!out)
		return fail(NUCLEUS34_E_INVALID, "null handle output");
	*out = nullptr;
	nucleus34_ctx ctx = nullptr;
	N34_TRY(create_ctx(opts, &ctx));
	int rc;
	{
		std::lock_guard<std::mutex> lk(ctx->c.mu);
		rc = upload(ctx->c, csr);
		if (!rc)
			rc = run(ctx->c, variant, res);
	}
	if (rc)
	{
		destroy_ctx(ctx);
		return rc;
	}
	auto *h = new (std::nothrow) nucleus34_state();
	if (!h)
	{
		destroy_ctx(ctx);
		return fail(NUCLEUS34_E_INVALID, "host allocation failed");
	}
	h->ctx = ctx;
	*out = h;
	return NUCLEUS34_OK;
}

} // namespace n34

using namespace n34;

extern "C" {

int nucleus34_ctx_create(const nucleus34_opts *opts, nucleus34_ctx *out)
{
	if (!out)
		return fail(NUCLEUS34_E_INVALID, "null output");
	return guarded([&] {
		const int rc = create_ctx(opts, out);
		// a resident context usually runs again: it keeps its blocks
		if (!rc)
			(*out)->c.keep_blocks = true;
		return rc;
	});
}

int nucleus34_ctx_upload(nucleus34_ctx ctx, const nucleus34_csr *csr)
{
	if (!ctx)
		return fail(NUCLEUS34_E_INVALID, "null context");
	return guarded([&] {
		std::lock_guard<std::mutex> lk(ctx->c.mu);
		return upload(ctx->c, csr);
	});
}

int nucleus34_ctx_run(nucleus34_ctx ctx, int variant, nucleus34_result *res)
{
	if (!ctx)
		return fail(NUCLEUS34_E_INVALID, "null context");
	return guarded([&] {
		std::lock_guard<std::mutex> lk(ctx->c.mu);
		return run(ctx->c, variant, res);
	});
}

int nucleus34_ctx_copy_k(nucleus34_ctx ctx, int32_t *k_out, uint32_t *tris_out)
{
	if (!ctx)
		return fail(NUCLEUS34_E_INVALID, "null context");
	return guarded([&] {
		std::lock_guard<std::mutex> lk(ctx->c.mu);
		return copy_k(ctx->c, k_out, tris_out);
	});
}

void nucleus34_ctx_destroy(nucleus34_ctx ctx) { destroy_ctx(ctx); }

int nucleus34_ctx_upload_edges(nucleus34_ctx ctx, const uint32_t *src, const uint32_t *dst, uint64_t count,
							   uint64_t *n_out, uint64_t *m_out)
{
	if (!ctx)
		return fail(NUCLEUS34_E_INVALID, "null context");
	return guarded([&]() -> int {
		std::lock_guard<std::mutex> lk(ctx->c.mu);
		N34_TRY(upload_edges(ctx->c, src, dst, count));
		if (n_out)
			*n_out = ctx->c.n;
		if (m_out)
			*m_out = ctx->c.m;
		return NUCLEUS34_OK;
	});
}

int nucleus34_ctx_copy_csr(nucleus34_ctx ctx, uint32_t *O, uint32_t *D, uint32_t *E)
{
	if (!ctx)
		return fail(NUCLEUS34_E_INVALID, "null context");
	return guarded([&]() -> int {
		std::lock_guard<std::mutex> lk(ctx->c.mu);
		Ctx &c = ctx->c;
		if (!c.dO)
			return fail(NUCLEUS34_E_STATE, "no graph uploaded");
		N34_TRY(set_device(c));
		std::vector<uint32_t> h(c.n + 1);
		N34_CUDA(cudaMemcpyAsync(h.data(), c.dO, (c.n + 1) * 4, cudaMemcpyDeviceToHost, c.stream));
		if (E && c.m)
			N34_CUDA(cudaMemcpyAsync(E, c.dE, c.m * 4, cudaMemcpyDeviceToHost, c.stream));
		N34_CUDA(cudaStreamSynchronize(c.stream));
		if (O)
			std::copy(h.begin(), h.end(), O);
		if (D)
			for (uint64_t u = 0; u < c.n; ++u)
				D[u] = h[u + 1] - h[u];
		return NUCLEUS34_OK;
	});
}

int nucleus34_ctx_set_tune(nucleus34_ctx ctx, const nucleus34_tune *tune)
{
	if (!ctx)
		return fail(NUCLEUS34_E_INVALID, "null context");
	return guarded([&]() -> int {
		if (tune)
			N34_TRY(tune_check(*tune));
		std::lock_guard<std::mutex> lk(ctx->c.mu);
		ctx->c.tune_pinned = tune != nullptr;
		ctx->c.tune_pin = tune ? *tune : nucleus34_tune{};
		return NUCLEUS34_OK;
	});
}

int nucleus34_ctx_last_tune(nucleus34_ctx ctx, nucleus34_tune *out)
{
	if (!ctx || !out)
		return fail(NUCLEUS34_E_INVALID, "null argument");
	return guarded([&]() -> int {
		std::lock_guard<std::mutex> lk(ctx->c.mu);
		*out = tune_filled(ctx->c.tune);
		return NUCLEUS34_OK;
	});
}

int nucleus34_ctx_autotune(nucleus34_ctx ctx, const char *path, nucleus34_tune *best, double *best_sec,
						   double *default_sec)
{
	if (!ctx)
		return fail(NUCLEUS34_E_INVALID, "null context");
	return guarded([&] {
		std::lock_guard<std::mutex> lk(ctx->c.mu);
		return autotune(ctx->c, path, best, best_sec, default_sec);
	});
}

int nucleus34_ctx_verify(nucleus34_ctx ctx, uint64_t *violations, uint64_t *checked)
{
	if (!ctx || !violations || !checked)
		return fail(NUCLEUS34_E_INVALID, "null argument");
	return guarded([&] {
		std::lock_guard<std::mutex> lk(ctx->c.mu);
		return verify(ctx->c, violations, checked);
	});
}

int nucleus34_decompose(const nucleus34_csr *csr, const nucleus34_opts *opts, nucleus34_result *res,
						nucleus34_handle *out)
{
	return guarded([&] { return decompose_impl(csr, opts, res, out, NUCLEUS34_DIRECT); });
}

int nucleus34_decompose_ondemand(const nucleus34_csr *csr, const nucleus34_opts *opts, nucleus34_result *res,
								 nucleus34_handle *out)
{
	return guarded([&] { return decompose_impl(csr, opts, res, out, NUCLEUS34_ONDEMAND); });
}

int nucleus34_copy_k(nucleus34_handle h, int32_t *k_out, uint32_t *tris_out)
{
	if (!h || !h->ctx)
		return fail(NUCLEUS34_E_INVALID, "null handle");
	return nucleus34_ctx_copy_k(h->ctx, k_out, tris_out);
}

int nucleus34_copy_quds(nucleus34_handle h, uint64_t first, uint64_t count, uint32_t *quds_out)
{
	if (!h || !h->ctx || (count && !quds_out))
		return fail(NUCLEUS34_E_INVALID, "null argument");
	return guarded([&] {
		Ctx &c = h->ctx->c;
		std::lock_guard<std::mutex> lk(c.mu);
		if (!c.have_result || c.variant != NUCLEUS34_DIRECT)
			return fail(NUCLEUS34_E_STATE, "four-clique list exists only after a direct decomposition");
		if (first > c.Q || count > c.Q - first)
			return fail(NUCLEUS34_E_INVALID, "clique range out of bounds");
		if (!count)
			return int(NUCLEUS34_OK);
		N34_TRY(set_device(c));
		N34_CUDA(cudaMemcpyAsync(quds_out, c.dquds + 4 * first, count * 16, cudaMemcpyDeviceToHost, c.stream));
		N34_CUDA(cudaStreamSynchronize(c.stream));
		return int(NUCLEUS34_OK);
	});
}

int nucleus34_write_kfile(nucleus34_handle h, const char *path)
{
	if (!h || !h->ctx || !path)
		return fail(NUCLEUS34_E_INVALID, "null argument");
	return guarded([&] {
		std::lock_guard<std::mutex> lk(h->ctx->c.mu);
		return write_kfile(h->ctx->c, path);
	});
}

int nucleus34_release_cached_memory(int device)
{
	return guarded([&]() -> int {
		int ndev = 0;
		if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
		{
			cudaGetLastError();
			return fail(NUCLEUS34_E_NODEVICE, "no CUDA device");
		}
		if (device < 0 || device >= ndev)
			return fail(NUCLEUS34_E_INVALID, "device ordinal out of range");
		cudaMemPool_t pool;
		N34_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
		N34_CUDA(cudaMemPoolTrimTo(pool, 0));
		return NUCLEUS34_OK;
	});
}

void nucleus34_free(nucleus34_handle h)
{
	if (!h)
		return;
	destroy_ctx(h->ctx);
	delete h;
}

} // extern "C"

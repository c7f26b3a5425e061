// Serving: a request loop that keeps graph state on the device and batches
// requests continuously (nucleus34_server_*).
//
// Each worker owns a context (device, stream, pooled memory) on one device
// slot; a slot is a device with its own memory budget, and several slots may
// name one GPU. A worker takes the pending requests in arrival order that fit
// the memory still free in its slot (estimated per request from its CSR) and
// within the 32-bit ranges, on-demand unions also within the 2^30 triangles
// of the death-flag peel (same-variant requests further back in the queue
// join too, past requests of the other variant), decomposes them in one pass
// as a disjoint union
// (the batched form), copies every request's results to the host and signals
// it. Requests that arrive while passes run are admitted by the next free
// worker, so with two or more workers their passes overlap on the device.
//
// Routing. Each request's variant is fixed at submission by its memory
// estimate: the direct variant (four-clique list kept and peeled by clique
// ids) when its estimate is at most 1/direct_div of a slot's budget, the
// on-demand variant (cliques re-enumerated) otherwise; a request for its
// clique list is always direct. The direct estimate counts out-triples
// sum_u C(d+(u), 3), which bound the four-cliques (every four-clique has one
// lowest vertex in the orientation with the other three among its
// out-neighbours); a direct union is cut so that this bound stays below
// 2^32, the direct variant's clique-id range. This generalises the
// reference's projection of the direct peel's memory (cuNucleus34.cu:563-585),
// which reports whether that peel will fit but does not choose.
//
// Results do not depend on the mix: a graph's triangles, cliques and k in a
// union equal those of the graph alone (the batched form's argument).
#include "admission.h"
#include "pipeline.cuh"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace n34 {
int build_union(const nucleus34_csr *graphs, uint64_t count, HostU32 &O, HostU32 &D, HostU32 &E,
				std::vector<uint64_t> &voff, std::vector<uint64_t> &eoff);
}

using namespace n34;

namespace {

using clk = std::chrono::steady_clock;

struct Request
{
	uint64_t id = 0;
	uint32_t flags = 0;
	// owned copy of the CSR
	uint64_t n = 0, m = 0;
	std::vector<uint32_t> O, D, E;
	uint64_t est_bytes = 0;     // admission estimate of the pass memory it needs (its variant)
	uint64_t est_triangles = 0; // upper bound (out-wedges)
	uint64_t est_cliques = 0;   // upper bound (out-triples)
	bool direct = false;        // variant chosen at submission
	// result
	bool done = false;
	int status = NUCLEUS34_OK;
	std::string error;
	nucleus34_graph_summary summary{};
	std::vector<int32_t, NoInitAlloc<int32_t>> k;
	HostU32 tris;
	HostU32 quds;
	clk::time_point t_submit, t_start, t_done;
	uint64_t pass = 0; // pass that served it
};

// The admission constants (bytes per triangle, edge and clique bound) and
// the default direct share live with the estimates in admission.h.

struct Slot
{
	int device = 0;
	uint64_t budget = 0;
	uint64_t in_flight = 0;
	uint32_t running = 0; // passes inside their decomposition
};

} // namespace

struct nucleus34_server_s
{
	nucleus34_opts opts{};
	std::vector<Slot> slots;      // device slots, each with its own budget
	uint64_t max_batch = 256;     // graphs per pass
	uint32_t route = NUCLEUS34_ROUTE_MEMORY;
	uint32_t direct_div = DEFAULT_DIRECT_DIV;
	uint32_t max_running = 0;     // decompositions at once per slot, 0 = no limit
	std::mutex mu;
	std::condition_variable cv_work, cv_done, cv_run;
	std::deque<std::shared_ptr<Request>> pending;
	std::map<uint64_t, std::shared_ptr<Request>> all;
	uint64_t next_id = 1, passes = 0, served = 0, direct_served = 0, busy_workers = 0;
	bool stop = false;
	std::vector<std::thread> workers;
	std::vector<nucleus34_ctx> ctxs;   // one per worker
	std::vector<size_t> worker_slot;   // slot of each worker
};

namespace {

// Entry to and exit from a slot's decompositions (at most max_running at
// once when set). The union build, upload and result copies stay outside, so
// one worker prepares or drains a pass while another computes.
void run_enter(nucleus34_server_s *s, Slot &slot)
{
	std::unique_lock<std::mutex> lk(s->mu);
	s->cv_run.wait(lk, [&] { return s->max_running == 0 || slot.running < s->max_running; });
	slot.running++;
}

void run_exit(nucleus34_server_s *s, Slot &slot)
{
	{
		std::lock_guard<std::mutex> lk(s->mu);
		slot.running--;
	}
	s->cv_run.notify_all();
}

// one pass over a set of requests of one variant (their union) on context c
void serve_union(nucleus34_server_s *s, Slot &slot, Ctx &c, std::vector<std::shared_ptr<Request>> &batch,
				 bool direct)
{
	std::vector<nucleus34_csr> csrs(batch.size());
	for (size_t i = 0; i < batch.size(); ++i)
		csrs[i] = nucleus34_csr{batch[i]->n, batch[i]->m, batch[i]->O.data(), batch[i]->D.data(),
								batch[i]->E.empty() ? nullptr : batch[i]->E.data()};
	HostU32 O, D, E;
	std::vector<uint64_t> voff, eoff;
	clear_error();
	int rc = build_union(csrs.data(), csrs.size(), O, D, E, voff, eoff);
	if (!rc)
	{
		const nucleus34_csr u{voff.back(), eoff.back(), O.data(), D.data(), E.empty() ? nullptr : E.data()};
		rc = upload(c, &u);
	}
	nucleus34_result r{};
	if (!rc)
	{
		c.seg_eoff = eoff;
		run_enter(s, slot);
		rc = run(c, direct ? NUCLEUS34_DIRECT : NUCLEUS34_ONDEMAND, &r);
		run_exit(s, slot);
	}
	// results to the host, each request's slices copied straight into its own
	// buffers (left uninitialised until the copy): k of every request, the
	// triangle and clique lists of those that ask
	if (!rc)
	{
		uint64_t q0 = 0; // first clique of request i in the union's list (cliques are listed by lowest triangle)
		for (size_t i = 0; i < batch.size() && !rc; ++i)
		{
			Request &q = *batch[i];
			const uint64_t t0 = c.seg_toff[i], T = c.seg_toff[i + 1] - t0;
			const uint64_t Qi = c.seg_q[i];
			q.summary.triangle_count = T;
			q.summary.four_clique_count = Qi;
			q.summary.k_max = c.seg_kmax[i];
			q.summary.k_avg = T ? double(c.seg_ksum[i]) / double(T) : 0.0;
			q.k.resize(T);
			if (q.flags & NUCLEUS34_REQ_TRIANGLES)
				q.tris.resize(3 * T);
			if (direct && (q.flags & NUCLEUS34_REQ_CLIQUES))
				q.quds.resize(4 * Qi);
			if ((T && cudaMemcpyAsync(q.k.data(), c.dK + t0, T * 4, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess) ||
				(T && !q.tris.empty() &&
				 cudaMemcpyAsync(q.tris.data(), c.dtris + 3 * t0, T * 12, cudaMemcpyDeviceToHost, c.stream) !=
					 cudaSuccess) ||
				(Qi && !q.quds.empty() &&
				 cudaMemcpyAsync(q.quds.data(), c.dquds + 4 * q0, Qi * 16, cudaMemcpyDeviceToHost, c.stream) !=
					 cudaSuccess))
				rc = fail(NUCLEUS34_E_CUDA, "serving: result copy");
			q0 += Qi;
		}
		if (!rc && cudaStreamSynchronize(c.stream) != cudaSuccess)
			rc = fail(NUCLEUS34_E_CUDA, "serving: result copy");
	}
	// a finished pass holds nothing on the device (admission counts on it)
	const std::vector<uint64_t> toff = std::move(c.seg_toff);
	c.release_results();
	c.release_graph();
	// ids of the union back to each request's own (edge ids, triangle ids)
	const std::string err = rc ? std::string(nucleus34_last_error()) : std::string();
	for (size_t i = 0; i < batch.size(); ++i)
	{
		Request &q = *batch[i];
		q.status = rc;
		q.error = err;
		if (rc)
		{
			decltype(q.k)().swap(q.k);
			decltype(q.tris)().swap(q.tris);
			decltype(q.quds)().swap(q.quds);
			continue;
		}
		const uint32_t eo = uint32_t(eoff[i]);
		if (eo)
			for (auto &x : q.tris)
				x -= eo;
		const uint32_t to = uint32_t(toff[i]);
		if (to)
			for (auto &x : q.quds)
				x -= to;
	}
}

void worker_loop(nucleus34_server_s *s, size_t wi)
{
	Ctx &c = s->ctxs[wi]->c;
	Slot &slot = s->slots[s->worker_slot[wi]];
	cudaSetDevice(c.device);
	const uint64_t range_limit = 0xffffffffull / 3; // 3T incidence entries in 32-bit positions
	// on-demand unions stay within the death-flag peel's triangle range
	const uint64_t ondemand_limit = std::min(range_limit, FLAG_PEEL_MAX_TRIANGLES);
	const uint64_t clique_limit = 0xffffffffull;     // direct: clique ids in 32 bits
	for (;;)
	{
		std::vector<std::shared_ptr<Request>> batch;
		bool direct = false;
		uint64_t take_bytes = 0;
		{
			std::unique_lock<std::mutex> lk(s->mu);
			s->cv_work.wait(lk, [&] {
				if (s->pending.empty())
					return s->stop;
				// the head fits the memory left in this slot, or nothing else
				// runs there; while stopping too, so that the queued requests
				// are finished under the same budget (a running pass always
				// ends and wakes the waiting workers)
				const uint64_t free_b = slot.budget > slot.in_flight ? slot.budget - slot.in_flight : 0;
				return s->pending.front()->est_bytes <= free_b || slot.in_flight == 0;
			});
			if (s->pending.empty())
				return; // stopping, nothing queued
			const uint64_t free_b = slot.budget > slot.in_flight ? slot.budget - slot.in_flight : 0;
			// admission in arrival order: the head always (it fits, or runs
			// alone on an idle slot), then, in order, the pending requests of
			// the same variant that fit, looking past requests of the other
			// variant (they stay queued for the next pass) within a bounded
			// window, so that interleaved variants still fill their passes
			auto head = s->pending.front();
			direct = head->direct;
			batch.push_back(head);
			s->pending.pop_front();
			take_bytes = head->est_bytes;
			uint64_t tri_bound = head->est_triangles, clique_bound = head->est_cliques;
			const size_t window = 4 * s->max_batch;
			for (size_t i = 0; i < s->pending.size() && i < window && batch.size() < s->max_batch;)
			{
				auto &q = s->pending[i];
				if (q->direct != direct || take_bytes + q->est_bytes > free_b ||
					tri_bound + q->est_triangles > (direct ? range_limit : ondemand_limit) ||
					(direct && clique_bound + q->est_cliques > clique_limit))
				{
					++i;
					continue;
				}
				take_bytes += q->est_bytes;
				tri_bound += q->est_triangles;
				clique_bound += q->est_cliques;
				batch.push_back(q);
				s->pending.erase(s->pending.begin() + std::ptrdiff_t(i));
			}
			slot.in_flight += take_bytes;
			s->busy_workers++;
			const auto now = clk::now();
			for (auto &q : batch)
				q->t_start = now;
		}
		serve_union(s, slot, c, batch, direct);
		{
			std::lock_guard<std::mutex> lk(s->mu);
			slot.in_flight -= take_bytes;
			s->busy_workers--;
			s->passes++;
			if (direct)
				s->direct_served += batch.size();
			const auto now = clk::now();
			for (auto &q : batch)
			{
				q->done = true;
				q->t_done = now;
				q->pass = s->passes;
				// the CSR copy is no longer needed
				std::vector<uint32_t>().swap(q->O);
				std::vector<uint32_t>().swap(q->D);
				std::vector<uint32_t>().swap(q->E);
			}
			s->served += batch.size();
		}
		s->cv_done.notify_all();
		s->cv_work.notify_all();
	}
}

std::shared_ptr<Request> find(nucleus34_server s, uint64_t id)
{
	auto it = s->all.find(id);
	return it == s->all.end() ? nullptr : it->second;
}

} // namespace

extern "C" {

int nucleus34_server_create(const nucleus34_opts *opts, const nucleus34_server_opts *sopts, nucleus34_server *out)
{
	if (!out)
		return fail(NUCLEUS34_E_INVALID, "null argument");
	*out = nullptr;
	clear_error();
	if (sopts && sopts->device_count && !sopts->devices)
		return fail(NUCLEUS34_E_INVALID, "device_count without devices");
	if (sopts && sopts->route > NUCLEUS34_ROUTE_ONDEMAND)
		return fail(NUCLEUS34_E_INVALID, "unknown route");
	auto *s = new (std::nothrow) nucleus34_server_s();
	if (!s)
		return fail(NUCLEUS34_E_OOM_BUDGET, "host allocation failed");
	if (opts)
		s->opts = *opts;
	s->opts.tune_table = nullptr; // read by each worker context as it is created; not kept
	const uint32_t per_dev = (sopts && sopts->workers) ? sopts->workers : 3u;
	s->max_batch = (sopts && sopts->max_batch_graphs) ? sopts->max_batch_graphs : 256;
	s->route = sopts ? sopts->route : NUCLEUS34_ROUTE_MEMORY;
	s->direct_div = (sopts && sopts->direct_div) ? sopts->direct_div : DEFAULT_DIRECT_DIV;
	s->max_running = sopts ? sopts->concurrent_runs : 0;
	std::vector<int> devs;
	if (sopts && sopts->device_count)
		devs.assign(sopts->devices, sopts->devices + sopts->device_count);
	else
		devs.push_back(opts ? opts->device : 0);
	for (size_t d = 0; d < devs.size(); ++d)
	{
		Slot sl;
		sl.device = devs[d];
		s->slots.push_back(sl);
	}
	// workers: per_dev on every slot, interleaved (worker w on slot w % slots)
	const size_t nw = size_t(per_dev) * devs.size();
	for (size_t w = 0; w < nw; ++w)
	{
		nucleus34_opts o = opts ? *opts : nucleus34_opts{};
		const size_t si = w % devs.size();
		o.device = devs[si];
		nucleus34_ctx ctx = nullptr;
		int rc = create_ctx(&o, &ctx);
		if (rc)
		{
			for (auto x : s->ctxs)
				destroy_ctx(x);
			delete s;
			return rc;
		}
		s->ctxs.push_back(ctx);
		s->worker_slot.push_back(si);
		// one budget per slot, shared by the passes in flight there
		if (w < devs.size())
			s->slots[si].budget = ctx->c.budget;
	}
	for (size_t w = 0; w < nw; ++w)
		s->ctxs[w]->c.budget = s->slots[s->worker_slot[w]].budget;
	for (size_t w = 0; w < nw; ++w)
		s->workers.emplace_back(worker_loop, s, w);
	*out = s;
	return NUCLEUS34_OK;
}

int nucleus34_server_submit(nucleus34_server s, const nucleus34_csr *csr, uint32_t flags, uint64_t *id)
{
	if (!s || !csr || !id || (csr->n && !csr->D) || (csr->m && !csr->E))
		return fail(NUCLEUS34_E_INVALID, "null argument");
	clear_error();
	if (csr->m > 0xffffffffull || csr->n >= 0xffffffffull)
		return fail(NUCLEUS34_E_RANGE32, "graph exceeds 32-bit vertex/edge ids");
	auto q = std::make_shared<Request>();
	q->flags = flags;
	q->n = csr->n;
	q->m = csr->m;
	q->O.resize(csr->n + 1);
	q->D.assign(csr->D, csr->D + csr->n);
	q->E.assign(csr->E, csr->E + csr->m);
	uint64_t acc = 0;
	for (uint64_t u = 0; u < csr->n; ++u)
	{
		q->O[u] = uint32_t(acc);
		acc += csr->D[u];
	}
	if (acc != csr->m)
		return fail(NUCLEUS34_E_INVALID, "sum of D does not equal m");
	q->O[csr->n] = uint32_t(acc);
	// routing by the memory estimate (the smallest slot budget is the limit)
	uint64_t min_budget = ~uint64_t(0);
	for (auto &sl : s->slots)
		min_budget = std::min(min_budget, sl.budget);
	nucleus34_request_estimate est{};
	request_estimate(csr->D, csr->n, csr->m, min_budget, s->route, s->direct_div, flags, est);
	q->est_triangles = est.triangle_bound;
	q->est_cliques = est.clique_bound;
	q->direct = est.direct != 0;
	q->est_bytes = q->direct ? est.direct_bytes : est.ondemand_bytes;
	q->t_submit = clk::now();
	{
		std::lock_guard<std::mutex> lk(s->mu);
		q->id = s->next_id++;
		s->all[q->id] = q;
		s->pending.push_back(q);
	}
	*id = q->id;
	s->cv_work.notify_one();
	return NUCLEUS34_OK;
}

int nucleus34_server_wait(nucleus34_server s, uint64_t id, int64_t timeout_ms, nucleus34_request_info *info)
{
	if (!s)
		return fail(NUCLEUS34_E_INVALID, "null server");
	clear_error();
	std::unique_lock<std::mutex> lk(s->mu);
	auto q = find(s, id);
	if (!q)
		return fail(NUCLEUS34_E_INVALID, "unknown request id");
	auto ready = [&] { return q->done; };
	if (timeout_ms < 0)
		s->cv_done.wait(lk, ready);
	else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
		return fail(NUCLEUS34_E_TIMEOUT, "request not finished within the timeout");
	if (info)
	{
		nucleus34_request_info x{};
		x.status = q->status;
		x.summary = q->summary;
		x.queue_seconds = std::chrono::duration<double>(q->t_start - q->t_submit).count();
		x.latency_seconds = std::chrono::duration<double>(q->t_done - q->t_submit).count();
		x.pass = q->pass;
		x.direct = q->direct ? 1 : 0;
		*info = x;
	}
	if (q->status)
		return fail(q->status, q->error);
	return NUCLEUS34_OK;
}

int nucleus34_server_copy_k(nucleus34_server s, uint64_t id, int32_t *k_out, uint32_t *tris_out)
{
	if (!s)
		return fail(NUCLEUS34_E_INVALID, "null server");
	std::lock_guard<std::mutex> lk(s->mu);
	auto q = find(s, id);
	if (!q || !q->done)
		return fail(NUCLEUS34_E_STATE, "request unknown or not finished");
	if (q->status)
		return fail(q->status, q->error);
	if (k_out && !q->k.empty())
		std::copy(q->k.begin(), q->k.end(), k_out);
	if (tris_out)
	{
		if (q->tris.size() != 3 * q->summary.triangle_count)
			return fail(NUCLEUS34_E_STATE, "the request did not ask for its triangle list");
		std::copy(q->tris.begin(), q->tris.end(), tris_out);
	}
	return NUCLEUS34_OK;
}

int nucleus34_server_copy_quds(nucleus34_server s, uint64_t id, uint64_t first, uint64_t count, uint32_t *quds_out)
{
	if (!s || (count && !quds_out))
		return fail(NUCLEUS34_E_INVALID, "null argument");
	std::lock_guard<std::mutex> lk(s->mu);
	auto q = find(s, id);
	if (!q || !q->done)
		return fail(NUCLEUS34_E_STATE, "request unknown or not finished");
	if (!(q->flags & NUCLEUS34_REQ_CLIQUES))
		return fail(NUCLEUS34_E_STATE, "the request did not ask for its four-clique list");
	const uint64_t Q = q->quds.size() / 4;
	if (first > Q || count > Q - first)
		return fail(NUCLEUS34_E_INVALID, "clique range out of bounds");
	std::copy(q->quds.begin() + 4 * first, q->quds.begin() + 4 * (first + count), quds_out);
	return NUCLEUS34_OK;
}

int nucleus34_server_release(nucleus34_server s, uint64_t id)
{
	if (!s)
		return fail(NUCLEUS34_E_INVALID, "null server");
	std::lock_guard<std::mutex> lk(s->mu);
	auto it = s->all.find(id);
	if (it == s->all.end() || !it->second->done)
		return fail(NUCLEUS34_E_STATE, "request unknown or not finished");
	s->all.erase(it);
	return NUCLEUS34_OK;
}

int nucleus34_server_stats(nucleus34_server s, nucleus34_server_counters *out)
{
	if (!s || !out)
		return fail(NUCLEUS34_E_INVALID, "null argument");
	std::lock_guard<std::mutex> lk(s->mu);
	nucleus34_server_counters x{};
	x.passes = s->passes;
	x.served = s->served;
	x.pending = s->pending.size();
	x.busy_workers = s->busy_workers;
	x.workers = s->workers.size();
	for (auto &sl : s->slots)
	{
		x.in_flight_bytes += sl.in_flight;
		x.budget_bytes += sl.budget;
	}
	x.direct_served = s->direct_served;
	x.devices = s->slots.size();
	*out = x;
	return NUCLEUS34_OK;
}

void nucleus34_server_destroy(nucleus34_server s)
{
	if (!s)
		return;
	{
		std::lock_guard<std::mutex> lk(s->mu);
		s->stop = true;
	}
	s->cv_work.notify_all();
	for (auto &t : s->workers)
		t.join();
	for (auto x : s->ctxs)
		destroy_ctx(x);
	delete s;
}

} // extern "C"

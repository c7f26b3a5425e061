// Splitting independent graphs over several GPUs (replicas, no collective):
// the host-side router of the batched form and of multi-device serving.
//
// Every graph is decomposed on one device only, so a split is a partition of
// the graphs into `parts` shares of similar estimated cost. The plan is the
// greedy longest-processing-time rule: graphs in decreasing cost (ties by
// index) each go to the currently least-loaded share (ties by share number).
// It is deterministic, so every rank of a multi-process run derives the same
// plan from the same inputs without exchanging it. Its makespan is within
// 4/3 of the optimum.
//
// Cost of a graph: its oriented edges plus its out-wedges sum_u C(d+(u), 2),
// the bound on its triangles that the admission estimates also use; both the
// listing and the peel grow with them.
//
// No reference counterpart: the reference runs one graph per process.
#include "host_internal.h"

#include <algorithm>
#include <functional>
#include <numeric>
#include <queue>
#include <utility>
#include <vector>

namespace n34 {

uint64_t graph_cost(const nucleus34_csr &g)
{
	uint64_t w = 0;
	for (uint64_t u = 0; u < g.n; ++u)
	{
		const uint64_t d = g.D[u];
		w += d * (d ? d - 1 : 0) / 2;
	}
	return g.m + w;
}

int split_plan(const uint64_t *cost, uint64_t count, uint32_t parts, uint32_t *part_of, uint64_t *load)
{
	if (parts == 0)
		return fail(NUCLEUS34_E_INVALID, "split into zero parts");
	if (count && (!cost || !part_of))
		return fail(NUCLEUS34_E_INVALID, "null argument");
	std::vector<uint64_t> order(count);
	std::iota(order.begin(), order.end(), uint64_t(0));
	std::stable_sort(order.begin(), order.end(), [&](uint64_t a, uint64_t b) { return cost[a] > cost[b]; });
	// min-heap of (load, share)
	using Share = std::pair<uint64_t, uint32_t>;
	std::priority_queue<Share, std::vector<Share>, std::greater<Share>> heap;
	for (uint32_t p = 0; p < parts; ++p)
		heap.push({0, p});
	std::vector<uint64_t> loads(parts, 0);
	for (uint64_t i : order)
	{
		Share s = heap.top();
		heap.pop();
		part_of[i] = s.second;
		s.first += cost[i];
		loads[s.second] = s.first;
		heap.push(s);
	}
	if (load)
		std::copy(loads.begin(), loads.end(), load);
	return NUCLEUS34_OK;
}

} // namespace n34

extern "C" {

int nucleus34_graph_cost(const nucleus34_csr *g, uint64_t *cost)
{
	if (!g || !cost || (g->n && !g->D))
		return n34::fail(NUCLEUS34_E_INVALID, "null argument");
	n34::clear_error();
	*cost = n34::graph_cost(*g);
	return NUCLEUS34_OK;
}

int nucleus34_split_plan(const uint64_t *cost, uint64_t count, uint32_t parts, uint32_t *part_of, uint64_t *load)
{
	n34::clear_error();
	try
	{
		return n34::split_plan(cost, count, parts, part_of, load);
	}
	catch (...)
	{
		return n34::fail(NUCLEUS34_E_INVALID, "host allocation failed");
	}
}

} // extern "C"

// Admission estimates and variant routing of the serving loop: host-only
// arithmetic on a request's out-degrees, shared by nucleus34_server_submit
// and nucleus34_server_estimate (so that it runs, and is tested, without a
// GPU).
#pragma once

#include "nucleus34.h"

#include <cstdint>

namespace n34 {

// Bytes of one pass per triangle (peak: listing, incidence build, support,
// peel arrays) and per oriented edge (CSR, sources, spans, counts); the
// direct variant adds its clique list and triangle->clique incidence (16 +
// 16 bytes per clique) and one destroyed flag per clique. Applied to the
// out-wedge and out-triple bounds, not to the true counts, so they
// overestimate; the GPU tests check them against measured peaks.
constexpr uint64_t PASS_BYTES_PER_TRIANGLE = 80;
constexpr uint64_t PASS_BYTES_PER_EDGE = 40;
constexpr uint64_t DIRECT_BYTES_PER_CLIQUE = 33;

// Direct share of a slot's budget (1/64). Alone, a graph is decomposed
// faster by the direct variant up to about 1e8 four-cliques, but a direct
// union of many such graphs streams its clique list from DRAM where the
// graph alone kept it in L2: on the full serving mix (edges up to 1e7) a
// share of 1/8 served 13.3-13.7 graphs/s, 1/64 14.2 and on-demand only 14.3.
constexpr uint32_t DEFAULT_DIRECT_DIV = 64;

// Out-wedges sum_u C(d, 2) (bound on the triangles) and out-triples
// sum_u C(d, 3) (bound on the four-cliques); the triples saturate at 2^63.
void out_bounds(const uint32_t *D, uint64_t n, uint64_t &wedges, uint64_t &triples);

// A request's estimates and variant: direct if it asks for its clique list
// (NUCLEUS34_REQ_CLIQUES), or, with NUCLEUS34_ROUTE_MEMORY, if its direct
// estimate is at most budget / direct_div (0: DEFAULT_DIRECT_DIV) and its
// clique bound fits the direct variant's 32-bit clique ids.
void request_estimate(const uint32_t *D, uint64_t n, uint64_t m, uint64_t budget, uint32_t route,
					  uint32_t direct_div, uint32_t flags, nucleus34_request_estimate &out);

} // namespace n34

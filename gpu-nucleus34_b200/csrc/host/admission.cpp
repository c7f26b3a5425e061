// Admission estimates and variant routing of the serving loop (host only).
//
// No reference counterpart: the reference projects the direct peel's memory
// (cuNucleus34.cu:563-585) only to report whether it will fit; the serving
// loop uses the same kind of projection to choose the variant per request.
#include "admission.h"
#include "host_internal.h"

namespace n34 {

void out_bounds(const uint32_t *D, uint64_t n, uint64_t &wedges, uint64_t &triples)
{
	wedges = 0;
	triples = 0;
	for (uint64_t u = 0; u < n; ++u)
	{
		const uint64_t d = D[u];
		wedges += d * (d ? d - 1 : 0) / 2;
		const unsigned __int128 t3 = d >= 3 ? (unsigned __int128)d * (d - 1) * (d - 2) / 6 : 0;
		const unsigned __int128 sum = (unsigned __int128)triples + t3;
		triples = sum > ((unsigned __int128)1 << 63) ? (uint64_t(1) << 63) : uint64_t(sum);
	}
}

void request_estimate(const uint32_t *D, uint64_t n, uint64_t m, uint64_t budget, uint32_t route,
					  uint32_t direct_div, uint32_t flags, nucleus34_request_estimate &out)
{
	uint64_t w = 0, t3 = 0;
	out_bounds(D, n, w, t3);
	const uint64_t est_on = PASS_BYTES_PER_EDGE * m + PASS_BYTES_PER_TRIANGLE * w;
	const unsigned __int128 est_dir128 = (unsigned __int128)est_on + (unsigned __int128)DIRECT_BYTES_PER_CLIQUE * t3;
	const uint64_t est_dir = est_dir128 > ~uint64_t(0) ? ~uint64_t(0) : uint64_t(est_dir128);
	const uint32_t div = direct_div ? direct_div : DEFAULT_DIRECT_DIV;
	bool direct = false;
	if (flags & NUCLEUS34_REQ_CLIQUES)
		direct = true;
	else if (route == NUCLEUS34_ROUTE_MEMORY)
		direct = est_dir <= budget / div && t3 < 0xffffffffull;
	out.ondemand_bytes = est_on;
	out.direct_bytes = est_dir;
	out.triangle_bound = w;
	out.clique_bound = t3;
	out.direct = direct ? 1 : 0;
}

} // namespace n34

extern "C" {

int nucleus34_server_estimate(const nucleus34_csr *csr, uint64_t budget, uint32_t route, uint32_t direct_div,
							  uint32_t flags, nucleus34_request_estimate *out)
{
	if (!csr || !out || (csr->n && !csr->D))
		return n34::fail(NUCLEUS34_E_INVALID, "null argument");
	if (route > NUCLEUS34_ROUTE_ONDEMAND)
		return n34::fail(NUCLEUS34_E_INVALID, "unknown route");
	n34::clear_error();
	uint64_t sum = 0;
	for (uint64_t u = 0; u < csr->n; ++u)
		sum += csr->D[u];
	if (sum != csr->m)
		return n34::fail(NUCLEUS34_E_INVALID, "sum of D does not equal m");
	n34::request_estimate(csr->D, csr->n, csr->m, budget, route, direct_div, flags, *out);
	return NUCLEUS34_OK;
}

} // extern "C"

// Stages of the device pipeline and the data they hand to each other.
#pragma once

#include "common.cuh"

namespace n34 {

// Edge -> triangle incidence, per edge sorted by third vertex. Edge e's list
// is [span[e].x, span[e].y) in third[] / tri[] (32-bit positions: the
// incidence holds 3T < 2^32 entries). The peel may shorten a list in place
// (dead entries dropped, span[e].y lowered); begins never move.
struct Incidence
{
	uint2 *span = nullptr;     // m
	uint32_t *third = nullptr; // 3T
	uint32_t *tri = nullptr;   // 3T
	// optional (on-demand peel with death flags): tpos[3t + r] = position of
	// triangle t's entry under its edge b (r=0), a (r=1), c (r=2)
	uint32_t *tpos = nullptr;
	unsigned long long sum_te_sq = 0; // sum over edges of (list length)^2
};

// Bit of an incidence entry's tri word that marks a peeled triangle (on-demand
// peel with death flags; the incidence is discarded after the peel).
constexpr uint32_t INC_DEAD = 0x80000000u;
// Most triangles the on-demand peel keeps its death flags in the incidence
// for (ids leave the top two bits of a tri word free); above it the slower
// round-stamp peel runs. Union passes (batched form, serving) are cut below it.
constexpr uint64_t FLAG_PEEL_MAX_TRIANGLES = 0x3fffffffull;

// Triangle -> four-clique incidence of the direct variant.
struct CliqueCsr
{
	uint64_t *off = nullptr; // T+1
	uint32_t *ids = nullptr; // 4Q clique ids
};

int build_src(Ctx &c);
// Triangle-listing passes on caller-owned memory (no bitmap cache).
cudaError_t launch_tri_count(const uint32_t *O, const uint32_t *E, uint64_t n, uint32_t *cnt, int sm_count,
							 cudaStream_t s);
cudaError_t launch_tri_write(const uint32_t *O, const uint32_t *E, uint64_t n, const uint64_t *toff,
							 uint32_t *tris, int sm_count, cudaStream_t s);
int list_triangles(Ctx &c);
// lean: no 64-bit key array (entries sorted in place as pairs) and no tpos.
int build_incidence(Ctx &c, Incidence &inc, bool want_tpos, bool lean = false);
void free_incidence(Ctx &c, Incidence &inc);
// Sorts every segment [off[s], off[s+1]) of keys ascending (incidence.cu's
// segmented sort; nseg < 2^32).
int sort_segments_u64(Ctx &c, unsigned long long *keys, const uint64_t *off, uint64_t nseg);
// Oriented CSR of an edge list built on the device and made resident in c
// (csr_build.cu), with the host build's semantics.
int upload_edges(Ctx &c, const uint32_t *src, const uint32_t *dst, uint64_t count);
// support[t] = number of four-cliques on t; returns sum(support) in *total.
// own (optional): cliques whose lowest triangle is t (direct variant sizes).
int count_support(Ctx &c, const Incidence &inc, int32_t *support, uint64_t *total, uint32_t *own);
// Direct variant: canonical clique list (c.dquds, c.Q) and triangle->clique CSR.
int list_cliques(Ctx &c, const Incidence &inc, const int32_t *support, const uint32_t *own, CliqueCsr &csr);
void free_clique_csr(Ctx &c, CliqueCsr &csr);
// Per-segment statistics of a batched (disjoint union) run; no-ops when the
// context holds a single graph. After listing: triangle offsets per member
// graph; after the support count: clique counts; after the peel: k max/sum.
int segments_after_listing(Ctx &c);
int segments_after_support(Ctx &c, const int32_t *support);
int segments_after_peel(Ctx &c);
// Device-resident peel; K receives the final k of every triangle.
int peel(Ctx &c, int variant, const Incidence &inc, const CliqueCsr &csr, int32_t *support, int32_t *K,
		 PeelCtl *hctl);

// Certificate check of the last run (verify.cu); needs the kept death rounds.
int verify(Ctx &c, uint64_t *violations, uint64_t *checked);
// Context entry points shared by the C-ABI front ends (api.cu, batch.cu).
int upload(Ctx &c, const nucleus34_csr *csr);
int run(Ctx &c, int variant, nucleus34_result *out);
int create_ctx(const nucleus34_opts *opts, nucleus34_ctx *out);
void destroy_ctx(nucleus34_ctx x);

} // namespace n34

struct nucleus34_ctx_s
{
	n34::Ctx c;
};

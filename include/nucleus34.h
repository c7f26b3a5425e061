/*
 * nucleus34.h -- C-ABI of the B200-native (3,4)-nucleus decomposition.
 *
 * Plain pointers and sizes only; no exception crosses this boundary and every
 * entry point returns a status code (0 = success, negative = NUCLEUS34_E_*).
 *
 * Vertex and edge ids are uint32, exactly as the reference's CSR holds them
 * (graph_t<EDGE_T=unsigned, VERTEX_T=unsigned>, nucleus/graph/graph_api.hpp:17-52):
 * an oriented edge id is its position in the degree-oriented CSR whose
 * adjacency lists are in ascending vertex-id order. A triangle is the triple
 * (a,b,c) of oriented-edge ids (u,w),(u,v),(v,w) (tri_t, nucleus/utils.cuh:93-102);
 * triangle ids are positions in the canonical (a,b) order.
 *
 * Threading: each call is synchronous on a library-owned stream of
 * opts->device. Calls on distinct handles/contexts may run concurrently from
 * different host threads.
 */
#ifndef NUCLEUS34_H_
#define NUCLEUS34_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NUCLEUS34_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------ */
enum
{
	NUCLEUS34_OK = 0,
	NUCLEUS34_E_INVALID = -1,     /* bad argument or malformed CSR */
	NUCLEUS34_E_OOM_BUDGET = -2,  /* device memory budget exceeded (reference: bad_alloc /
	                                 segment retry exhausted, nucleus/utils.cuh:1580-1581) */
	NUCLEUS34_E_RANGE32 = -3,     /* a 32-bit id range would overflow (reference guards:
	                                 nucleus/cuNucleus34.cu:617-624, cuNucleus34_ondemand.cu:505-511) */
	NUCLEUS34_E_CUDA = -4,        /* CUDA runtime error */
	NUCLEUS34_E_TIMEOUT = -5,     /* a bounded device wait ran out */
	NUCLEUS34_E_IO = -6,          /* file could not be opened/read/written */
	NUCLEUS34_E_FORMAT = -7,      /* unknown extension or malformed file
	                                 (reference: "Unknown dataset format", cuNucleus34.cu:253-256) */
	NUCLEUS34_E_NODEVICE = -8,    /* no CUDA device / wrong architecture */
	NUCLEUS34_E_STATE = -9        /* call out of order (e.g. run before upload) */
};

enum
{
	NUCLEUS34_DIRECT = 0,    /* materialise four-cliques + triangle->clique CSR (cuNucleus34) */
	NUCLEUS34_ONDEMAND = 1   /* edge->triangle incidence, re-enumerate at death (cuNucleus34_ondemand) */
};

/* ---- inputs and results ------------------------------------------------ */

/* Oriented CSR on the HOST. O may be NULL (then built from D); when given it
 * holds n entries, O[u] = first out-edge of u, like graph_t::O
 * (nucleus/graph/graph.hpp:523-536). D[u] = out-degree, E = destinations. */
typedef struct
{
	uint64_t n;
	uint64_t m;
	const uint32_t *O;
	const uint32_t *D;
	const uint32_t *E;
} nucleus34_csr;

typedef struct
{
	uint64_t mem_budget_bytes; /* 0 = 90% of the device's free memory */
	int device;                /* CUDA ordinal */
	uint32_t parts;            /* accepted for CLI parity (cuNucleus34.cu:161-169); one GPU */
	const char *tune_table;    /* tune table path (see nucleus34_tune below), read and checked when
	                              the context is created; NULL = built-in defaults */
	uint32_t flags;            /* NUCLEUS34_OPT_* bits, 0 = defaults */
} nucleus34_opts;

/* opts.flags: force the round-stamp ownership test in the on-demand peel
 * (the default keeps death flags inside the incidence entries when T < 2^30). */
#define NUCLEUS34_OPT_STAMP_PEEL 0x1u
/* opts.flags: run the peel rounds as plain launches with CUDA events around
 * every step and print per-step device times to stderr (diagnostics only;
 * slower than the default graph replay). */
#define NUCLEUS34_OPT_PROFILE_PEEL 0x2u
/* opts.flags: the memory-lean layout of the on-demand variant (T < 2^30):
 * incidence entries sorted in place (no 64-bit sort keys beside them), no
 * per-triangle entry positions (the peel searches for a triangle's entries),
 * frontiers as two bitmaps instead of two lists, and k kept in the support
 * array; about 28 bytes per triangle beside the triangle list instead of
 * about 60. Chosen automatically when the regular layout does not fit in
 * the memory budget left after the triangle listing. Results are identical. */
#define NUCLEUS34_OPT_LEAN_MEMORY 0x4u
/* opts.flags: keep each triangle's death round after the peel, so that
 * nucleus34_ctx_verify can certify the result (costs 4 bytes per triangle). */
#define NUCLEUS34_OPT_VERIFIABLE 0x8u
/* opts.flags (batched form): each finished pass's k and triangle lists move
 * to host memory and its device memory is freed before the next pass. Also
 * chosen automatically when the next pass would not fit beside the results
 * kept on the device. Results and accessors are unchanged. */
#define NUCLEUS34_OPT_HOST_RESULTS 0x10u
/* opts.flags: drive the peel rounds from the host (a CUDA graph of a fixed
 * number of rounds replayed, the host reading the control block after each
 * replay) instead of the default device loop (one CUDA graph whose while
 * node repeats the rounds until the peel is done, launched once). Results
 * are identical; kept for comparison and for drivers without conditional
 * graph nodes. */
#define NUCLEUS34_OPT_HOST_LOOP 0x20u
/* opts.flags: run every peel round as separate kernel launches, instead of
 * running consecutive small cascade rounds (at most 8192 dying triangles, no
 * level change) inside one cooperative launch with grid barriers between the
 * steps of a round (the default for the on-demand peel with death flags).
 * Results are identical; kept for comparison. */
#define NUCLEUS34_OPT_NO_SMALL_ROUNDS 0x40u
/* opts.flags: put large peel frontiers in the order of their triangles'
 * entries under their c edges (edge-major: triangles that share their c edge,
 * usually their longest list, become neighbours) instead of triangle-id
 * order. Results are identical. */
#define NUCLEUS34_OPT_FRONTIER_BY_C 0x80u
/* opts.flags: the chunked debit schedule of the death-flag peel: warps take
 * chunks of up to 32 frontier triangles, load their lists in parallel and
 * debit the short and the long ones, instead of one thread per dying
 * triangle with a short list and one warp per triangle with a long one (two
 * kernels). Results are identical; measured on one B200 it is 3% faster on
 * RGG 4M and 4.5% slower on R-MAT scale 20, so it is not the default. */
#define NUCLEUS34_OPT_CHUNKED_DEBIT 0x100u
/* opts.flags: the peel's level-change scans with one 4-byte load per thread
 * per step and a ballot and atomic per 32 supports, instead of two 16-byte
 * loads per thread per step and one atomic per warp step. Results are
 * identical; kept for comparison. */
#define NUCLEUS34_OPT_SCALAR_SCANS 0x200u
/* opts.flags: the warp debit of the death-flag peel loads the next dying
 * triangles' ids and records before the current one's debit (a software
 * pipeline; 5 instead of 6 blocks per SM). Results are identical. */
#define NUCLEUS34_OPT_PIPELINED_DEBIT 0x400u
/* opts.flags: the warp debit of the death-flag peel runs as one wave of
 * blocks whose warps claim frontier positions from an atomic cursor (work
 * balanced at run time) instead of a fixed warp stride. Results are
 * identical. */
#define NUCLEUS34_OPT_DEBIT_CURSOR 0x800u

typedef struct
{
	uint64_t triangle_count;
	uint64_t four_clique_count;
	uint64_t peeling_iterations;  /* peel rounds executed */
	uint64_t unpeeled_count;      /* triangles left at -1 (0 on success) */
	uint32_t k_max;
	double k_avg;                 /* sum(k) / T, accumulated in 64-bit integers */
	/* device-side phase times, seconds, CUDA events on the library stream */
	double t_triangles;           /* triangle listing */
	double t_incidence;           /* edge -> triangle incidence */
	double t_support;             /* four-clique support count */
	double t_cliques;             /* direct only: clique list + triangle->clique CSR */
	double t_peel;                /* device-resident bucketed peel */
	double t_total;               /* sum of the above (reference total_time_sec accounting) */
	uint64_t incidence_entries;   /* 3 * triangle_count */
	uint64_t gpu_launches;        /* kernels this run launched */
	uint64_t peak_device_bytes;   /* high-water mark of the library's device allocations */
	int variant;                  /* NUCLEUS34_DIRECT or NUCLEUS34_ONDEMAND */
	uint64_t sum_te_sq;           /* sum over edges of T(e)^2, T(e) = triangles on edge e
	                                 (work measure of the 3-way intersections) */
	/* with NUCLEUS34_OPT_PROFILE_PEEL only (0 otherwise): device time of the
	 * peel's re-enumeration kernels summed over all rounds, seconds */
	double t_peel_debit;
} nucleus34_result;

typedef struct nucleus34_state *nucleus34_handle;

/* ---- one-shot decomposition (drop-in for the two programs' device pipelines) */

/* Replaces the device pipeline of the direct program, nucleus/cuNucleus34.cu:283-721
 * (triangle listing, triangle graph, four-clique list, triangle->clique incidence,
 * claim peel). Uploads the host CSR, runs on the device, keeps k (and the
 * triangle and clique lists) behind *out until nucleus34_free. */
int nucleus34_decompose(const nucleus34_csr *csr, const nucleus34_opts *opts,
						nucleus34_result *res, nucleus34_handle *out);

/* Replaces the device pipeline of nucleus/cuNucleus34_ondemand.cu:407-690
 * (triangles, sorted incidence, support count, re-enumerating round peel). */
int nucleus34_decompose_ondemand(const nucleus34_csr *csr, const nucleus34_opts *opts,
								 nucleus34_result *res, nucleus34_handle *out);

/* k_out: int32[triangle_count] in canonical order (may be NULL);
 * tris_out: uint32[3*triangle_count] as (a,b,c) (may be NULL). */
int nucleus34_copy_k(nucleus34_handle h, int32_t *k_out, uint32_t *tris_out);

/* Direct variant only: count cliques starting at index first, each as four
 * ascending triangle ids, in the library's canonical clique order (grouped by
 * lowest member, then by the fourth vertex's id). */
int nucleus34_copy_quds(nucleus34_handle h, uint64_t first, uint64_t count, uint32_t *quds_out);

/* Writes the per-triangle file, one row "(a,b,c)\t<k>" per triangle in
 * canonical order (layout of cuNucleus34_ondemand.cu:724-733). */
int nucleus34_write_kfile(nucleus34_handle h, const char *path);

/* Releases the handle's device memory into the device's stream-ordered pool,
 * where it stays cached for later calls (re-mapping tens of GB would cost more
 * than the decomposition); nucleus34_release_cached_memory hands it back. */
void nucleus34_free(nucleus34_handle h);

/* Returns the device memory cached by earlier calls (the default memory pool
 * of `device`, trimmed to zero) to the driver. */
int nucleus34_release_cached_memory(int device);

const char *nucleus34_strerror(int code);
/* Detail of the calling thread's last failure ("" if none). */
const char *nucleus34_last_error(void);

/* ---- device-resident context (inputs stay in HBM across runs) ------------ */

typedef struct nucleus34_ctx_s *nucleus34_ctx;

/* A context keeps the device blocks its runs release and reuses them for
 * allocations of the same size, so a graph run again allocates nothing new;
 * the kept blocks count toward opts.mem_budget_bytes, are given back when an
 * allocation needs the room, and are freed by nucleus34_ctx_destroy. */
int nucleus34_ctx_create(const nucleus34_opts *opts, nucleus34_ctx *out);
/* H2D copy of the CSR into context-owned device memory (replaces the
 * thrust::device_vector uploads, cuNucleus34.cu:290-293). */
int nucleus34_ctx_upload(nucleus34_ctx ctx, const nucleus34_csr *csr);
/* The oriented CSR of an edge list, built on the device and made resident:
 * the same graph as nucleus34_graph_from_edges followed by
 * nucleus34_ctx_upload (symmetrise, drop self-loops, sort + unique,
 * n = max id + 1 over the non-loop pairs, degree orientation; graph.hpp:
 * 356-411, 176-218), with only the pairs crossing to the device. src and dst
 * are host arrays of count pairs; *n_out and *m_out (optional) receive the
 * vertex and oriented edge counts. */
int nucleus34_ctx_upload_edges(nucleus34_ctx ctx, const uint32_t *src, const uint32_t *dst, uint64_t count,
							   uint64_t *n_out, uint64_t *m_out);
/* Copies the resident oriented CSR to the host: O (n+1 entries), D (n), E (m);
 * each may be NULL. */
int nucleus34_ctx_copy_csr(nucleus34_ctx ctx, uint32_t *O, uint32_t *D, uint32_t *E);
/* Runs one decomposition of the resident graph; results stay on the device. */
int nucleus34_ctx_run(nucleus34_ctx ctx, int variant, nucleus34_result *res);
int nucleus34_ctx_copy_k(nucleus34_ctx ctx, int32_t *k_out, uint32_t *tris_out);
void nucleus34_ctx_destroy(nucleus34_ctx ctx);
/* Certifies the last run's k (needs NUCLEUS34_OPT_VERIFIABLE): every
 * triangle t must lie in at least k(t) cliques whose triangles all have
 * k >= k(t), must have had at most k(t) cliques with all partners alive when
 * its round began, and the level must never decrease from round to round.
 * Together these hold exactly for the (3,4)-nucleus numbers. *violations
 * receives the number of triangles (and rounds) that fail; *checked the
 * number of triangles examined. Rebuilds the edge->triangle incidence. */
int nucleus34_ctx_verify(nucleus34_ctx ctx, uint64_t *violations, uint64_t *checked);

/* ---- tuning (scheduling settings of the on-demand variant) -------------- */

/* Every setting gives bit-identical results: a setting only moves a
 * triangle between the lane and warp kernels, or changes when the incidence
 * is compacted, when a frontier is put in id order and how many peel rounds
 * one CUDA graph replay holds. A zero field means the built-in default. The
 * direct variant always runs with the defaults. No reference counterpart:
 * the reference's kernels run with fixed launch shapes and one peel round per
 * host iteration (cuNucleus34_ondemand.cu:599-682). */
#define NUCLEUS34_TUNE_NEVER 0xffffffffu
typedef struct
{
	uint32_t lane_max;          /* shortest-list length up to which one lane rather than a warp
	                               takes a triangle (support count and peel): 8, 16 (default), 32 */
	uint32_t compact_div;       /* compact the incidence once the triangles peeled since the last
	                               compaction reach 1/compact_div of the live ones: 1..64
	                               (default 8), or NUCLEUS34_TUNE_NEVER */
	uint32_t sort_shift;        /* put a frontier of at least max(T >> sort_shift, 4096) triangles
	                               in id order: 1..31 (default 12), or NUCLEUS34_TUNE_NEVER */
	uint32_t rounds_per_replay; /* peel rounds per CUDA graph replay: 1..64 (default 16) */
} nucleus34_tune;

/* A tune table is a text file of lines
 *     size=<s> skew=<w> [lane_max=..] [compact_div=..|never] [sort_shift=..|never]
 *     [rounds_per_replay=..] [sec=..] [default_sec=..]
 * ('#' starts a comment). A graph's class is size = floor(log2 T) and
 * skew = floor(log2(max out-degree * n / m)) of its degree-oriented CSR
 * (0 when m = 0). A run takes the line of its skew class whose size is
 * nearest, if within 2 (ties to the earlier line); otherwise the defaults.
 * sec and default_sec record the autotuner's timings and are not used. */

/* The settings that the table at path gives a graph of `triangles`
 * triangles whose oriented CSR has n vertices, m edges and maximum
 * out-degree max_out; defaults filled in. *matched (if non-NULL) = 1 when a
 * line applied. E_IO: unreadable; E_INVALID: a malformed line (the detail
 * names it). */
int nucleus34_tune_lookup(const char *path, uint64_t triangles, uint64_t n, uint64_t m, uint32_t max_out,
						  nucleus34_tune *out, int *matched);
/* Writes `tune` (defaults filled in) as the line of that graph's class into
 * the table at path, replacing a line of the same class or appending one
 * (the file is created when missing and rewritten through a temporary and a
 * rename; a table that does not parse is left alone: E_INVALID). sec and
 * default_sec are recorded as given. */
int nucleus34_tune_store(const char *path, uint64_t triangles, uint64_t n, uint64_t m, uint32_t max_out,
						 const nucleus34_tune *tune, double sec, double default_sec);
/* Pins the settings of the context's later on-demand runs (NULL: back to
 * its tune table, or the defaults). E_INVALID for a value out of range. */
int nucleus34_ctx_set_tune(nucleus34_ctx ctx, const nucleus34_tune *tune);
/* The settings the last run used, defaults filled in. */
int nucleus34_ctx_last_tune(nucleus34_ctx ctx, nucleus34_tune *out);
/* Autotuner for the uploaded graph: times its on-demand decomposition under
 * the defaults, then under candidate settings, one field at a time (each
 * field keeps the best value found before the next is tried; a candidate
 * must beat the best so far by 1% twice). Every run's k must equal the
 * default run's bit for bit (E_CUDA otherwise). The best settings go to
 * *best, their time and the default time (s, device-timed t_total) to
 * *best_sec and *default_sec, and, when path is non-NULL, into the table
 * at path as the line of this graph's class (a line of the same class is
 * replaced; the file is rewritten through a temporary and a rename).
 * Needs host memory for two copies of k (8 bytes per triangle). The
 * context's pinned settings are restored afterwards. */
int nucleus34_ctx_autotune(nucleus34_ctx ctx, const char *path, nucleus34_tune *best, double *best_sec,
						   double *default_sec);

/* ---- batched decomposition ------------------------------------------------ */

/* Many independent graphs decomposed in one device pass (their disjoint
 * union: one listing, incidence, support count and peel for the whole
 * batch; a batch beyond 2^32/3 triangles is cut into several such passes,
 * after one counting pass over the whole union). Every graph's triangle list, counts and k equal those of
 * nucleus34_decompose_ondemand on that graph alone. No reference
 * counterpart: the reference decomposes one graph per process. */
typedef struct nucleus34_batch_s *nucleus34_batch;

typedef struct
{
	uint64_t graphs;
	uint64_t triangle_count;      /* over all graphs */
	uint64_t four_clique_count;   /* over all graphs */
	uint64_t peeling_iterations;  /* rounds of the shared peel */
	double t_upload;              /* host union build + upload, seconds (wall) */
	double t_triangles, t_incidence, t_support, t_peel;
	double t_total;               /* device time of the shared pass */
	uint64_t gpu_launches;
	uint64_t peak_device_bytes;   /* largest pass */
	uint64_t chunks;              /* device passes: unions are cut so that 3T < 2^32 each */
} nucleus34_batch_result;

typedef struct
{
	uint64_t triangle_count;
	uint64_t four_clique_count;
	uint32_t k_max;
	double k_avg;                 /* sum(k) / T in 64-bit integers, as for one graph */
} nucleus34_graph_summary;

int nucleus34_batch_decompose(const nucleus34_csr *graphs, uint64_t count, const nucleus34_opts *opts,
							  nucleus34_batch_result *res, nucleus34_batch *out);
int nucleus34_batch_summary(nucleus34_batch b, uint64_t index, nucleus34_graph_summary *out);
/* Graph `index`'s k in its canonical order and, if tris_out is not NULL, its
 * triangles as (a,b,c) edge ids of that graph alone. */
int nucleus34_batch_copy_k(nucleus34_batch b, uint64_t index, int32_t *k_out, uint32_t *tris_out);
void nucleus34_batch_free(nucleus34_batch b);

/* ---- replicas over several GPUs: the split of independent graphs ---------- */

/* No reference counterpart (the reference runs one graph per process). A
 * graph's estimated cost: its oriented edges plus its out-wedges
 * sum_u d+(u)(d+(u)-1)/2 (the admission estimates' bound on its triangles). */
int nucleus34_graph_cost(const nucleus34_csr *g, uint64_t *cost);
/* Partitions `count` graphs of the given costs into `parts` shares
 * (part_of[i] in [0, parts)) by the greedy longest-processing-time rule:
 * decreasing cost, ties by index, each to the least-loaded share (ties by
 * share number). Deterministic, so every rank derives the same plan. load
 * (optional, parts entries) receives each share's total cost. */
int nucleus34_split_plan(const uint64_t *cost, uint64_t count, uint32_t parts, uint32_t *part_of, uint64_t *load);

/* ---- serving: continuous batching of decomposition requests -------------- */

/* A request loop with device-resident state. Workers (one context and stream
 * each, spread over one or more devices) admit pending requests in arrival
 * order while their estimated memory fits what their device's budget
 * (opts.mem_budget_bytes per device) has left, decompose them in one union
 * pass, and copy each request's results to the host. Requests that arrive
 * while passes run join the next pass; passes of different workers overlap
 * on the device. Each request's variant is chosen at submission by its
 * memory estimate (bytes per oriented edge and per out-wedge, plus, for the
 * direct variant, per out-triple sum_u C(d+(u), 3), the bound on its
 * four-cliques that the clique list grows with): with NUCLEUS34_ROUTE_MEMORY
 * it is the direct variant when that estimate is at most 1/direct_div of a
 * device's budget, else on-demand; requests flagged NUCLEUS34_REQ_CLIQUES are
 * always direct. A pass holds requests of one variant; direct unions stay
 * below 2^32 four-cliques by the same bound. A request's results equal those
 * of the graph decomposed alone. No reference counterpart: the reference's
 * projection of the direct peel's memory (cuNucleus34.cu:563-585) only
 * reports whether that peel will fit. */
typedef struct nucleus34_server_s *nucleus34_server;

#define NUCLEUS34_REQ_CLIQUES 0x1u   /* direct variant: keep the four-clique list */
#define NUCLEUS34_REQ_TRIANGLES 0x2u /* keep the triangle list (k alone otherwise) */

#define NUCLEUS34_ROUTE_MEMORY 0u    /* direct when its estimate fits 1/direct_div of a device's budget */
#define NUCLEUS34_ROUTE_ONDEMAND 1u  /* on-demand unless the request asks for its clique list */

typedef struct
{
	uint32_t workers;             /* concurrent passes per device, 0 = 3 */
	uint64_t max_batch_graphs;    /* requests per pass, 0 = 256 */
	uint32_t route;               /* NUCLEUS34_ROUTE_* */
	uint32_t direct_div;          /* ROUTE_MEMORY: direct estimate <= budget / direct_div; 0 = 64 */
	uint32_t device_count;        /* 0: opts.device alone; else devices[0..device_count) */
	const int *devices;           /* ordinals (one may repeat: several budgets on one GPU) */
	uint32_t concurrent_runs;     /* decompositions running at once per slot (the other workers
	                               * build unions and copy results meanwhile); 0 = no limit */
} nucleus34_server_opts;

typedef struct
{
	int status;                   /* the request's own result code */
	nucleus34_graph_summary summary;
	double queue_seconds;         /* submit -> admitted to a pass */
	double latency_seconds;       /* submit -> results on the host */
	uint64_t pass;                /* sequence number of the pass that served it */
	int direct;                   /* 1 if routed to the direct variant */
} nucleus34_request_info;

typedef struct
{
	uint64_t passes, served, pending, busy_workers, workers, in_flight_bytes, budget_bytes;
	uint64_t direct_served;       /* requests served by the direct variant */
	uint64_t devices;             /* device slots */
} nucleus34_server_counters;

/* A request's admission estimates and variant, as nucleus34_server_submit
 * computes them (host only; needs no device). */
typedef struct
{
	uint64_t ondemand_bytes;      /* pass memory estimate of the on-demand variant */
	uint64_t direct_bytes;        /* the same with the direct variant's clique list (saturates) */
	uint64_t triangle_bound;      /* out-wedges sum_u C(d+(u), 2) >= triangles */
	uint64_t clique_bound;        /* out-triples sum_u C(d+(u), 3) >= four-cliques (saturates at 2^63) */
	int direct;                   /* 1 if the request would be routed to the direct variant */
} nucleus34_request_estimate;

/* Estimates and routes a request without submitting it: budget is the
 * smallest slot budget the server would see, route and direct_div as in
 * nucleus34_server_opts (direct_div 0 = 64), flags as in submit. Reads only
 * csr->D (sum must equal m). No reference counterpart. */
int nucleus34_server_estimate(const nucleus34_csr *csr, uint64_t budget, uint32_t route, uint32_t direct_div,
                              uint32_t flags, nucleus34_request_estimate *out);

int nucleus34_server_create(const nucleus34_opts *opts, const nucleus34_server_opts *sopts, nucleus34_server *out);
/* Copies the CSR and queues it; returns at once with the request id. */
int nucleus34_server_submit(nucleus34_server s, const nucleus34_csr *csr, uint32_t flags, uint64_t *id);
/* Waits for request id (timeout_ms < 0: without limit; NUCLEUS34_E_TIMEOUT when
 * it runs out); returns the request's own status and fills info. */
int nucleus34_server_wait(nucleus34_server s, uint64_t id, int64_t timeout_ms, nucleus34_request_info *info);
int nucleus34_server_copy_k(nucleus34_server s, uint64_t id, int32_t *k_out, uint32_t *tris_out);
int nucleus34_server_copy_quds(nucleus34_server s, uint64_t id, uint64_t first, uint64_t count, uint32_t *quds_out);
/* Forgets a finished request and its host results. */
int nucleus34_server_release(nucleus34_server s, uint64_t id);
int nucleus34_server_stats(nucleus34_server s, nucleus34_server_counters *out);
/* Finishes the queued requests, then stops the workers. */
void nucleus34_server_destroy(nucleus34_server s);

/* ---- triangle listing without allocation --------------------------------- */

/* No counterpart in the reference. For callers that cannot allocate device
 * memory while they run (all of HBM reserved up front by their own pool, a
 * framework allocator that must not be bypassed, latency-critical loops):
 * lists the triangles of an oriented CSR already in device memory, in
 * canonical (a,b) order, into a caller-owned device buffer, and allocates
 * nothing. d_O holds n+1 offsets (O[n] = m), d_E the m destinations; d_tris
 * receives 3 u32 per triangle. The CSR must be acyclically oriented with each
 * undirected edge stored once and ascending adjacency lists, as
 * nucleus34_graph_from_edges and nucleus34_graph_load produce; a CSR that
 * breaks O[n] == m, holds an id >= n, a self-loop, an unsorted list or an
 * edge stored in both directions is rejected with NUCLEUS34_E_INVALID and
 * nothing is written (a longer cycle in the orientation is not detected: its
 * triangles would be missed). The count is always returned in
 * *triangle_count; if it exceeds tris_capacity nothing is written and the
 * call returns NUCLEUS34_E_INVALID (call again with room; capacity 0 and a
 * NULL d_tris is a count-only query). At most 2^20 vertices: larger graphs
 * are rejected with NUCLEUS34_E_INVALID. The temporaries live in a fixed
 * static device array (about 12.6 MB, held by every GPU that loads the
 * library until exit) shared by all calls: calls that overlap on one GPU race
 * and must be serialised by the caller. Every call looks up that array's
 * address on `device` and restores the caller's current device before it
 * returns. stream is a cudaStream_t (NULL = default stream); the call
 * synchronises it before returning. */
int nucleus34_list_triangles_noalloc(const uint32_t *d_O, const uint32_t *d_E, uint64_t n, uint64_t m,
									 uint32_t *d_tris, uint64_t tris_capacity, uint64_t *triangle_count,
									 int device, void *stream);

/* ---- host graph layer (reference reader/orientation semantics) ----------- */

/* Library-owned oriented CSR; O has n+1 entries here. */
typedef struct
{
	uint64_t n;
	uint64_t m;
	uint32_t *O;
	uint32_t *D;
	uint32_t *E;
} nucleus34_graph;

/* Dispatch by extension like the mains (cuNucleus34.cu:235-256):
 * .mtx -> from_edges(mtx header) + make_oriented; .edges/.txt -> from_edges
 * (first non-comment line consumed as a header, graph.hpp:307-318) +
 * make_oriented; .grh -> deserialize + build_offset (already oriented). */
int nucleus34_graph_load(const char *path, nucleus34_graph *g);
/* Same semantics from an in-memory list (no header line): symmetrise, drop
 * self-loops, sort + unique, n = max id + 1, orient (graph.hpp:356-411,176-218). */
int nucleus34_graph_from_edges(const uint32_t *src, const uint32_t *dst, uint64_t count,
							   nucleus34_graph *g);
/* .grh writer (graph_t::serialize layout, graph.hpp:465-488). */
int nucleus34_graph_save_grh(const nucleus34_graph *g, const char *path);
void nucleus34_graph_release(nucleus34_graph *g);
/* View of a loaded graph as the decomposition input. */
nucleus34_csr nucleus34_graph_csr(const nucleus34_graph *g);

/* ---- seeded synthetic inputs (no datasets on this system) ---------------- */

typedef struct
{
	uint64_t count;
	uint32_t *src;
	uint32_t *dst;
} nucleus34_edges;

/* Each generator returns the cleaned undirected list: u < v, unique, no loops,
 * sorted. Counter-based streams (splitmix64 of seed and index) make the output
 * independent of the thread count. */
int nucleus34_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c,
					   uint64_t seed, nucleus34_edges *out);
int nucleus34_gen_rgg(uint64_t n, double expected_degree, uint64_t seed, nucleus34_edges *out);
int nucleus34_gen_ws(uint64_t n, uint32_t k, double beta, uint64_t seed, nucleus34_edges *out);
/* Bare .edges file with a sacrificial first line (a repeat of the first edge),
 * so the reference reader's first-line drop loses nothing. */
int nucleus34_edges_write(const nucleus34_edges *e, const char *path);
void nucleus34_edges_release(nucleus34_edges *e);
uint64_t nucleus34_splitmix64(uint64_t x);

#ifdef __cplusplus
}
#endif
#endif /* NUCLEUS34_H_ */

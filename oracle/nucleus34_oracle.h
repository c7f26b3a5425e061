/*
 * CPU oracle for the (3,4)-nucleus decomposition -- TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C restatement of the reference's algorithm, used by the
 * tests, by the smoke check and by the bench's CPU-baseline leg to check the
 * CUDA path. It is never linked into, loaded by or called from the product
 * library. Each function cites the reference file:line it follows.
 *
 * Parity pinning: the restatement is checked against the outputs of the
 * reference's own host code (oracle/_ref/cpu_ref, compiled from the reference
 * sources by oracle/Makefile) on the committed fixtures in tests/golden/.
 */
#ifndef NUCLEUS34_ORACLE_H_
#define NUCLEUS34_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Oriented CSR exactly as graph_t<EDGE_T,VERTEX_T> holds it after
 * make_oriented (nucleus/graph/graph.hpp:176-218): O has n+1 entries here
 * (the reference keeps n and uses m for the last end). */
typedef struct
{
	uint64_t n;     /* vertices (max id + 1) */
	uint64_t m;     /* oriented edges */
	uint32_t *O;    /* n+1 */
	uint32_t *D;    /* n, out-degree */
	uint32_t *E;    /* m, ascending vertex id within each list */
} oracle_graph;

typedef struct
{
	uint64_t T;          /* triangles */
	uint64_t Q;          /* four-cliques */
	int32_t k_max;
	double k_avg;
	uint32_t *tris;      /* 3T: (a,b,c) oriented-edge ids, canonical (a,b) order */
	int32_t *support;    /* T: initial four-clique support */
	int32_t *k;          /* T: final k per triangle */
	uint32_t *quds;      /* 4 * min(Q, quds_cap): first cliques, canonical order */
	uint64_t quds_len;
} oracle_result;

/* Error codes: 0 ok, -1 I/O, -2 format, -3 out of memory, -4 range. */
int oracle_read_graph(const char *path, oracle_graph *g);
/* Same semantics as reading a bare edge list whose first line was already
 * consumed: symmetrise, drop self-loops, sort + unique, n = max id + 1, then
 * orient by (undirected degree, id). */
int oracle_graph_from_pairs(const uint32_t *src, const uint32_t *dst, uint64_t count,
							oracle_graph *g);
int oracle_graph_from_oriented(uint64_t n, uint64_t m, const uint32_t *D, const uint32_t *E,
							   oracle_graph *g);
void oracle_graph_free(oracle_graph *g);

/* Full decomposition. quds_cap = how many canonical four-cliques to keep. */
int oracle_decompose(const oracle_graph *g, uint64_t quds_cap, oracle_result *r);
void oracle_result_free(oracle_result *r);

/* Triangle count only (listing without storage). */
uint64_t oracle_count_triangles(const oracle_graph *g);
/* four-cliques counted by oriented neighbourhoods (independent of the incidence) */
uint64_t oracle_count_k4(const oracle_graph *g);
/* Level-synchronous peel (the device peel's rules) on the canonical triangle
 * list tris (3T): k and each triangle's death round. */
int oracle_peel_rounds(const oracle_graph *g, const uint32_t *tris, uint64_t T, int32_t *k, uint32_t *rounds);
/* Certificate check of (k, rounds): number of failing triangles and rounds
 * (0: k are exactly the (3,4)-nucleus numbers), or a negative error code. */
int64_t oracle_certify(const oracle_graph *g, const uint32_t *tris, uint64_t T, const int32_t *k,
					   const uint32_t *rounds);

#ifdef __cplusplus
}
#endif
#endif

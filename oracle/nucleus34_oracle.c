/*
 * CPU oracle for the (3,4)-nucleus decomposition -- TEST INFRASTRUCTURE ONLY.
 * Not product code: only tests/, the smoke check and the bench's CPU-baseline
 * leg load it, and only as the checker. The product library never links it.
 *
 * Plain-C restatement of the reference algorithm. Every step cites the
 * reference source it restates (paths relative to the reference project).
 */
#define _GNU_SOURCE
#include "nucleus34_oracle.h"

#include <errno.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_OK 0
#define OR_EIO (-1)
#define OR_EFORMAT (-2)
#define OR_ENOMEM (-3)
#define OR_ERANGE (-4)

/* ------------------------------------------------------------------------- */
/* small helpers                                                             */
/* ------------------------------------------------------------------------- */

static int cmp_u64(const void *x, const void *y)
{
	uint64_t a = *(const uint64_t *)x, b = *(const uint64_t *)y;
	return (a > b) - (a < b);
}

/* LSD radix sort of u64 keys (8 passes of 8 bits); used for the pair sort of
 * from_edges (graph.hpp:384, std::sort of (s,d) pairs) and the incidence sort
 * (cuNucleus34_ondemand.cu:535, sort_by_key on (edge<<32|third)). */
static int radix_sort_u64(uint64_t *a, uint64_t n, uint64_t *payload_opt)
{
	if (n < 2)
		return OR_OK;
	if (n < 4096 && !payload_opt)
	{
		qsort(a, n, sizeof(uint64_t), cmp_u64);
		return OR_OK;
	}
	uint64_t *tmp = malloc(n * sizeof(uint64_t));
	uint64_t *ptmp = payload_opt ? malloc(n * sizeof(uint64_t)) : NULL;
	if (!tmp || (payload_opt && !ptmp))
	{
		free(tmp);
		free(ptmp);
		return OR_ENOMEM;
	}
	uint64_t *src = a, *dst = tmp, *psrc = payload_opt, *pdst = ptmp;
	for (int pass = 0; pass < 8; ++pass)
	{
		const int sh = pass * 8;
		uint64_t cnt[257] = {0};
		for (uint64_t i = 0; i < n; ++i)
			cnt[((src[i] >> sh) & 0xff) + 1]++;
		{ /* every key shares this digit: the pass is the identity */
			int skip = 0;
			for (int d = 1; d <= 256; ++d)
				if (cnt[d] == n)
					skip = 1;
			if (skip)
				continue;
		}
		for (int d = 0; d < 256; ++d)
			cnt[d + 1] += cnt[d];
		for (uint64_t i = 0; i < n; ++i)
		{
			uint64_t pos = cnt[(src[i] >> sh) & 0xff]++;
			dst[pos] = src[i];
			if (psrc)
				pdst[pos] = psrc[i];
		}
		uint64_t *t = src;
		src = dst;
		dst = t;
		if (psrc)
		{
			t = psrc;
			psrc = pdst;
			pdst = t;
		}
	}
	if (src != a)
	{
		memcpy(a, src, n * sizeof(uint64_t));
		if (payload_opt)
			memcpy(payload_opt, psrc, n * sizeof(uint64_t));
	}
	free(tmp);
	free(ptmp);
	return OR_OK;
}

void oracle_graph_free(oracle_graph *g)
{
	if (!g)
		return;
	free(g->O);
	free(g->D);
	free(g->E);
	memset(g, 0, sizeof(*g));
}

/* ------------------------------------------------------------------------- */
/* graph construction                                                        */
/* ------------------------------------------------------------------------- */

/* Undirected CSR from symmetrised, sorted, unique pairs (key = s<<32|d), then
 * orientation. Restates graph_t::from_edges' tail (graph.hpp:383-410: sort,
 * unique, resize(max_node+1), D[s]++, build_offset) and make_oriented
 * (graph.hpp:176-218) with vertex_less (graph_api.hpp:124-127): keep (u,v) iff
 * (deg u, u) < (deg v, v) on the UNDIRECTED degree, adjacency order kept. */
static int orient_from_sorted_pairs(const uint64_t *pairs, uint64_t np, uint64_t n, oracle_graph *g)
{
	memset(g, 0, sizeof(*g));
	uint32_t *Du = calloc(n ? n : 1, sizeof(uint32_t));
	if (!Du)
		return OR_ENOMEM;
	for (uint64_t i = 0; i < np; ++i)
		Du[pairs[i] >> 32]++;
	g->n = n;
	g->O = calloc(n + 1, sizeof(uint32_t));
	g->D = calloc(n ? n : 1, sizeof(uint32_t));
	uint64_t m = 0;
	for (uint64_t i = 0; i < np; ++i)
	{
		uint32_t u = (uint32_t)(pairs[i] >> 32), v = (uint32_t)pairs[i];
		if (Du[u] < Du[v] || (Du[u] == Du[v] && u < v))
			m++;
	}
	g->m = m;
	g->E = malloc((m ? m : 1) * sizeof(uint32_t));
	if (!g->O || !g->D || !g->E)
	{
		free(Du);
		oracle_graph_free(g);
		return OR_ENOMEM;
	}
	uint64_t k = 0;
	for (uint64_t i = 0; i < np; ++i)
	{
		uint32_t u = (uint32_t)(pairs[i] >> 32), v = (uint32_t)pairs[i];
		if (Du[u] < Du[v] || (Du[u] == Du[v] && u < v))
		{
			g->E[k++] = v;
			g->D[u]++;
		}
	}
	for (uint64_t u = 0; u < n; ++u)
		g->O[u + 1] = g->O[u] + g->D[u];
	free(Du);
	return OR_OK;
}

/* pairs: symmetrise + self-loop drop (graph.hpp:359-376), sort + unique
 * (graph.hpp:383-388). max_node tracks only non-self-loop endpoints. */
static int finish_pairs(uint64_t *pairs, uint64_t np, uint32_t max_node, int any, oracle_graph *g)
{
	int rc = radix_sort_u64(pairs, np, NULL);
	if (rc)
		return rc;
	uint64_t w = 0;
	for (uint64_t i = 0; i < np; ++i)
		if (w == 0 || pairs[i] != pairs[w - 1])
			pairs[w++] = pairs[i];
	(void)any;
	return orient_from_sorted_pairs(pairs, w, (uint64_t)max_node + 1, g);
}

int oracle_graph_from_pairs(const uint32_t *src, const uint32_t *dst, uint64_t count, oracle_graph *g)
{
	uint64_t *pairs = malloc((2 * count + 1) * sizeof(uint64_t));
	if (!pairs)
		return OR_ENOMEM;
	uint64_t np = 0;
	uint32_t max_node = 0;
	for (uint64_t i = 0; i < count; ++i)
	{
		uint32_t s = src[i], d = dst[i];
		if (s == d)
			continue;
		if (s > max_node)
			max_node = s;
		if (d > max_node)
			max_node = d;
		pairs[np++] = ((uint64_t)s << 32) | d;
		pairs[np++] = ((uint64_t)d << 32) | s;
	}
	int rc = finish_pairs(pairs, np, max_node, 1, g);
	free(pairs);
	return rc;
}

int oracle_graph_from_oriented(uint64_t n, uint64_t m, const uint32_t *D, const uint32_t *E, oracle_graph *g)
{
	memset(g, 0, sizeof(*g));
	g->n = n;
	g->m = m;
	g->O = calloc(n + 1, sizeof(uint32_t));
	g->D = malloc((n ? n : 1) * sizeof(uint32_t));
	g->E = malloc((m ? m : 1) * sizeof(uint32_t));
	if (!g->O || !g->D || !g->E)
	{
		oracle_graph_free(g);
		return OR_ENOMEM;
	}
	memcpy(g->D, D, n * sizeof(uint32_t));
	memcpy(g->E, E, m * sizeof(uint32_t));
	uint64_t s = 0;
	for (uint64_t u = 0; u < n; ++u)
	{
		g->O[u] = (uint32_t)s;
		s += D[u];
	}
	g->O[n] = (uint32_t)s;
	if (s != m)
	{
		oracle_graph_free(g);
		return OR_EFORMAT;
	}
	return OR_OK;
}

/* Parses "<uint> <uint>" at the start of a line, as `ss >> s >> d` does for
 * well-formed input (graph.hpp:361-363); returns 0 if two numbers are not
 * present (the reference reads uninitialised values there; this oracle
 * skips the line). */
static int parse_two(const char *p, uint32_t *s, uint32_t *d)
{
	char *end;
	while (*p == ' ' || *p == '\t')
		p++;
	if (*p < '0' || *p > '9')
		return 0;
	errno = 0;
	unsigned long long a = strtoull(p, &end, 10);
	if (end == p || errno)
		return 0;
	p = end;
	while (*p == ' ' || *p == '\t')
		p++;
	if (*p < '0' || *p > '9')
		return 0;
	unsigned long long b = strtoull(p, &end, 10);
	if (end == p || errno || a > 0xffffffffULL || b > 0xffffffffULL)
		return 0;
	*s = (uint32_t)a;
	*d = (uint32_t)b;
	return 1;
}

static const char *file_ext(const char *path)
{
	const char *dot = strrchr(path, '.');
	return dot ? dot : "";
}

/* Reads .mtx/.edges/.txt like graph_t::from_edges (graph.hpp:285-411) followed
 * by make_oriented, and .grh like deserialize + build_offset
 * (graph.hpp:491-536), dispatched by extension as the mains do
 * (cuNucleus34.cu:238-256). Quirk kept: the first non-comment line of a bare
 * edge list is consumed as a "header" and discarded (graph.hpp:307-318). */
int oracle_read_graph(const char *path, oracle_graph *g)
{
	const char *ext = file_ext(path);
	memset(g, 0, sizeof(*g));
	if (!strcmp(ext, ".grh"))
	{
		FILE *f = fopen(path, "rb");
		if (!f)
			return OR_EIO;
		uint64_t sv = 0, nV = 0, nE = 0;
		if (fread(&sv, 8, 1, f) != 1 || fread(&nV, 8, 1, f) != 1 || fread(&nE, 8, 1, f) != 1 || sv != 4)
		{
			fclose(f);
			return OR_EFORMAT;
		}
		uint32_t *D = malloc((nV ? nV : 1) * 4), *E = malloc((nE ? nE : 1) * 4);
		if (!D || !E)
		{
			free(D);
			free(E);
			fclose(f);
			return OR_ENOMEM;
		}
		int ok = fread(D, 4, nV, f) == nV && fread(E, 4, nE, f) == nE;
		fclose(f);
		int rc = ok ? oracle_graph_from_oriented(nV, nE, D, E, g) : OR_EFORMAT;
		free(D);
		free(E);
		return rc;
	}
	int mtx = !strcmp(ext, ".mtx");
	if (!mtx && strcmp(ext, ".edges") && strcmp(ext, ".txt"))
		return OR_EFORMAT;

	FILE *f = fopen(path, "r");
	if (!f)
		return OR_EIO;
	char *line = NULL;
	size_t cap = 0;
	ssize_t len;
	int have_line = 0;
	/* skip leading comment lines: line[0] in "#%" (graph.hpp:307-314) */
	while ((len = getline(&line, &cap, f)) >= 0)
	{
		if (line[0] != '#' && line[0] != '%')
		{
			have_line = 1;
			break;
		}
	}
	if (mtx)
	{
		/* header: 2 or 3 tokens (graph.hpp:318-354) */
		if (!have_line)
		{
			free(line);
			fclose(f);
			return OR_EFORMAT;
		}
		int ntok = 0;
		unsigned long long tok[4] = {0};
		char *save = NULL;
		for (char *t = strtok_r(line, " \t\r\n", &save); t; t = strtok_r(NULL, " \t\r\n", &save))
		{
			if (ntok < 4)
			{
				char *end;
				tok[ntok] = strtoull(t, &end, 0);
				if (end == t)
				{
					free(line);
					fclose(f);
					return OR_EFORMAT;
				}
			}
			ntok++;
		}
		if (ntok != 2 && ntok != 3)
		{
			free(line);
			fclose(f);
			return OR_EFORMAT;
		}
		unsigned long long nvtx = ntok == 2 ? tok[0] : (tok[0] > tok[1] ? tok[0] : tok[1]);
		unsigned long long nedge = ntok == 2 ? tok[1] : tok[2];
		if (nedge > 0xffffffffULL || nvtx > 0xffffffffULL)
		{
			free(line);
			fclose(f);
			return OR_ERANGE;
		}
	}
	uint64_t cap_pairs = 1 << 16, np = 0;
	uint64_t *pairs = malloc(cap_pairs * sizeof(uint64_t));
	uint32_t max_node = 0;
	if (!pairs)
	{
		free(line);
		fclose(f);
		return OR_ENOMEM;
	}
	while ((len = getline(&line, &cap, f)) >= 0)
	{
		uint32_t s, d;
		if (!parse_two(line, &s, &d))
			continue;
		if (s == d)
			continue;
		if (np + 2 > cap_pairs)
		{
			cap_pairs *= 2;
			uint64_t *p2 = realloc(pairs, cap_pairs * sizeof(uint64_t));
			if (!p2)
			{
				free(pairs);
				free(line);
				fclose(f);
				return OR_ENOMEM;
			}
			pairs = p2;
		}
		if (s > max_node)
			max_node = s;
		if (d > max_node)
			max_node = d;
		pairs[np++] = ((uint64_t)s << 32) | d;
		pairs[np++] = ((uint64_t)d << 32) | s;
	}
	free(line);
	fclose(f);
	int rc = finish_pairs(pairs, np, max_node, 1, g);
	free(pairs);
	return rc;
}

/* ------------------------------------------------------------------------- */
/* triangles                                                                 */
/* ------------------------------------------------------------------------- */

/* Zipper listing of cliques_tri_seq (cliques.hpp:42-92; device twin
 * utils.cuh:259-343): for u, for each out-edge j=(u,v), intersect E[O[u]..)
 * with E over v's out-edges; a match at i1 (in u's list) and o (in v's list)
 * is the triangle {a=i1, b=j, c=o}. emit==NULL counts only. */
static uint64_t list_triangles_of(const oracle_graph *g, uint64_t u, uint32_t *emit)
{
	uint64_t cnt = 0;
	const uint32_t d1 = g->O[u], d2 = g->O[u + 1];
	for (uint32_t j = d1; j < d2; ++j)
	{
		const uint32_t v = g->E[j];
		uint32_t i1 = d1, o = g->O[v];
		const uint32_t oe = g->O[v + 1];
		while (i1 < d2 && o < oe)
		{
			const uint32_t p = g->E[i1], q = g->E[o];
			if (p < q)
				i1++;
			else
			{
				if (p == q)
				{
					if (emit)
					{
						emit[3 * cnt + 0] = i1;
						emit[3 * cnt + 1] = j;
						emit[3 * cnt + 2] = o;
					}
					cnt++;
					i1++;
				}
				o++;
			}
		}
	}
	return cnt;
}

uint64_t oracle_count_triangles(const oracle_graph *g)
{
	uint64_t T = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : T)
	for (uint64_t u = 0; u < g->n; ++u)
		T += list_triangles_of(g, u, NULL);
	return T;
}

/* Four-clique count by oriented neighbourhoods, independent of the
 * edge->triangle incidence and of any peel: with the degree orientation every
 * four-clique has exactly one vertex u that points to the other three, and
 * among those one v that points to the other two, and so on; so it is counted
 * once as u -> v -> w (a triangle of u's out-lists) plus an x in
 * N+(u) & N+(v) & N+(w). Used as an independent check of the clique totals on
 * graphs too large for the full oracle (no counterpart in the reference). */
static uint64_t count3(const uint32_t *a, uint32_t na, const uint32_t *b, uint32_t nb, const uint32_t *c,
					   uint32_t nc)
{
	uint64_t cnt = 0;
	uint32_t i = 0, j = 0, k = 0;
	while (i < na && j < nb && k < nc)
	{
		const uint32_t x = a[i], y = b[j], z = c[k];
		if (x == y && y == z)
		{
			++cnt;
			++i, ++j, ++k;
			continue;
		}
		const uint32_t mx = x > y ? (x > z ? x : z) : (y > z ? y : z);
		if (x < mx)
			++i;
		if (y < mx)
			++j;
		if (z < mx)
			++k;
	}
	return cnt;
}

uint64_t oracle_count_k4(const oracle_graph *g)
{
	uint64_t Q = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : Q)
	for (uint64_t u = 0; u < g->n; ++u)
	{
		const uint32_t *nu = g->E + g->O[u];
		const uint32_t du = g->O[u + 1] - g->O[u];
		for (uint32_t i = 0; i < du; ++i)
		{
			const uint32_t v = nu[i];
			const uint32_t *nv = g->E + g->O[v];
			const uint32_t dv = g->O[v + 1] - g->O[v];
			/* w in N+(u) & N+(v) */
			uint32_t p = 0, q = 0;
			while (p < du && q < dv)
			{
				if (nu[p] < nv[q])
					++p;
				else if (nu[p] > nv[q])
					++q;
				else
				{
					const uint32_t w = nu[p];
					Q += count3(nu, du, nv, dv, g->E + g->O[w], g->O[w + 1] - g->O[w]);
					++p, ++q;
				}
			}
		}
	}
	return Q;
}

/* canonical order: tuple sort on (a,b) (graph.hpp:108, helpers.hpp:305-317;
 * tri_t::operator< utils.cuh:98-101). Since a and b are both out-edges of the
 * same vertex u, the order is u-major; sort within each vertex's block. */
static int cmp_ab(const void *x, const void *y)
{
	const uint32_t *a = x, *b = y;
	if (a[0] != b[0])
		return a[0] < b[0] ? -1 : 1;
	if (a[1] != b[1])
		return a[1] < b[1] ? -1 : 1;
	return 0;
}

/* ------------------------------------------------------------------------- */
/* edge -> triangle incidence and the 3-way zipper                           */
/* ------------------------------------------------------------------------- */

typedef struct
{
	uint64_t *off;      /* m+1 */
	uint32_t *third;    /* 3T, per edge ascending */
	uint32_t *tri;      /* 3T */
} incidence;

/* build_incidence_entries + sort_by_key + split + lower_bound
 * (cuNucleus34_ondemand.cu:92-128, 513-549): triangle i=(a,b,c) with
 * u=src[b], v=E[b], w=E[c] is listed under b with third w, under a with third
 * v and under c with third u. */
static int build_incidence(const oracle_graph *g, const uint32_t *tris, uint64_t T, incidence *inc)
{
	memset(inc, 0, sizeof(*inc));
	const uint64_t n3 = 3 * T;
	uint32_t *src = malloc((g->m ? g->m : 1) * sizeof(uint32_t));
	uint64_t *keys = malloc((n3 ? n3 : 1) * sizeof(uint64_t));
	uint64_t *vals = malloc((n3 ? n3 : 1) * sizeof(uint64_t));
	inc->off = calloc(g->m + 1, sizeof(uint64_t));
	inc->third = malloc((n3 ? n3 : 1) * sizeof(uint32_t));
	inc->tri = malloc((n3 ? n3 : 1) * sizeof(uint32_t));
	if (!src || !keys || !vals || !inc->off || !inc->third || !inc->tri)
	{
		free(src);
		free(keys);
		free(vals);
		free(inc->off);
		free(inc->third);
		free(inc->tri);
		return OR_ENOMEM;
	}
	for (uint64_t u = 0; u < g->n; ++u)
		for (uint32_t e = g->O[u]; e < g->O[u + 1]; ++e)
			src[e] = (uint32_t)u;
	for (uint64_t i = 0; i < T; ++i)
	{
		const uint32_t a = tris[3 * i], b = tris[3 * i + 1], c = tris[3 * i + 2];
		const uint32_t u = src[b], v = g->E[b], w = g->E[c];
		keys[3 * i + 0] = ((uint64_t)b << 32) | w;
		keys[3 * i + 1] = ((uint64_t)a << 32) | v;
		keys[3 * i + 2] = ((uint64_t)c << 32) | u;
		vals[3 * i + 0] = vals[3 * i + 1] = vals[3 * i + 2] = i;
	}
	int rc = radix_sort_u64(keys, n3, vals);
	if (rc == OR_OK)
	{
		for (uint64_t i = 0; i < n3; ++i)
		{
			inc->off[(keys[i] >> 32) + 1]++;
			inc->third[i] = (uint32_t)keys[i];
			inc->tri[i] = (uint32_t)vals[i];
		}
		for (uint64_t e = 0; e < g->m; ++e)
			inc->off[e + 1] += inc->off[e];
	}
	free(src);
	free(keys);
	free(vals);
	return rc;
}

static void free_incidence(incidence *inc)
{
	free(inc->off);
	free(inc->third);
	free(inc->tri);
}

/* 3-way zipper of for_each_clique_of (cuNucleus34_ondemand.cu:136-170): every
 * common third vertex x of the lists of the triangle's three edges is one
 * four-clique; the partners are the (b,x), (a,x), (c,x) triangles. */
typedef void (*clique_fn)(void *ctx, uint32_t x, uint32_t p1, uint32_t p2, uint32_t p3);

static uint32_t for_each_clique(const incidence *inc, const uint32_t *t3, clique_fn fn, void *ctx)
{
	uint64_t i = inc->off[t3[1]], iE = inc->off[t3[1] + 1];
	uint64_t j = inc->off[t3[0]], jE = inc->off[t3[0] + 1];
	uint64_t k = inc->off[t3[2]], kE = inc->off[t3[2] + 1];
	uint32_t cnt = 0;
	while (i < iE && j < jE && k < kE)
	{
		const uint32_t x1 = inc->third[i], x2 = inc->third[j], x3 = inc->third[k];
		if (x1 == x2 && x2 == x3)
		{
			if (fn)
				fn(ctx, x1, inc->tri[i], inc->tri[j], inc->tri[k]);
			cnt++;
			i++;
			j++;
			k++;
		}
		else
		{
			uint32_t mx = x1 > x2 ? x1 : x2;
			mx = mx > x3 ? mx : x3;
			if (x1 < mx)
				i++;
			if (x2 < mx)
				j++;
			if (x3 < mx)
				k++;
		}
	}
	return cnt;
}

/* ------------------------------------------------------------------------- */
/* bucket peel                                                               */
/* ------------------------------------------------------------------------- */

/* Restates bucket_ex (bucket_ex.hpp:31-64 construction, 132-146 decrease,
 * 148-163 peel, 210-220 pop_min, 246-264 peeling_seq, 92-99 support): a
 * bin-sorted permutation with per-value bin starts; pop the minimum, and for
 * each clique of the popped triangle that no earlier-popped member destroyed,
 * decrease every member whose value is above the current level (clamped at
 * the level). Zero-support triangles are never popped and report k = 0. */
typedef struct
{
	int64_t *val;      /* current value; popped: level-1 */
	uint32_t *perm;    /* bin-sorted keys */
	uint64_t *pos;     /* perm^-1 */
	uint64_t *bin;     /* bin[v] = first position of value v (v >= 1) */
	int64_t last;      /* last popped value */
} bucket;

static void bucket_decrease(bucket *B, uint32_t key)
{
	int64_t v = B->val[key];
	uint64_t p = B->pos[key];
	uint64_t s = B->bin[v]; /* start of bin v */
	uint32_t other = B->perm[s];
	B->perm[s] = key;
	B->perm[p] = other;
	B->pos[key] = s;
	B->pos[other] = p;
	B->bin[v]++;
	B->val[key] = v - 1;
}

typedef struct
{
	bucket *B;
} peel_ctx;

static void peel_clique(void *vctx, uint32_t x, uint32_t p1, uint32_t p2, uint32_t p3)
{
	(void)x;
	bucket *B = ((peel_ctx *)vctx)->B;
	const uint32_t m[3] = {p1, p2, p3};
	for (int s = 0; s < 3; ++s)
		if (B->val[m[s]] < B->last)
			return; /* destroyed by an earlier pop */
	for (int s = 0; s < 3; ++s)
		if (B->val[m[s]] != B->last)
			bucket_decrease(B, m[s]);
}

/* canonical four-clique listing for the direct variant's record: each clique
 * is listed once, under its lowest triangle id, in ascending x. */
typedef struct
{
	uint32_t owner;
	uint32_t *out;
	uint64_t cap, len;
} qud_ctx;

static int cmp_u32(const void *x, const void *y)
{
	uint32_t a = *(const uint32_t *)x, b = *(const uint32_t *)y;
	return (a > b) - (a < b);
}

static void collect_qud(void *vctx, uint32_t x, uint32_t p1, uint32_t p2, uint32_t p3)
{
	(void)x;
	qud_ctx *c = vctx;
	if (c->len >= c->cap)
		return;
	if (p1 < c->owner || p2 < c->owner || p3 < c->owner)
		return;
	uint32_t *q = c->out + 4 * c->len;
	q[0] = c->owner;
	q[1] = p1;
	q[2] = p2;
	q[3] = p3;
	qsort(q, 4, sizeof(uint32_t), cmp_u32);
	c->len++;
}

void oracle_result_free(oracle_result *r)
{
	if (!r)
		return;
	free(r->tris);
	free(r->support);
	free(r->k);
	free(r->quds);
	memset(r, 0, sizeof(*r));
}

int oracle_decompose(const oracle_graph *g, uint64_t quds_cap, oracle_result *r)
{
	memset(r, 0, sizeof(*r));
	/* triangle listing (cliques.hpp:98-226), per-vertex counts then writes */
	uint64_t *toff = calloc(g->n + 1, sizeof(uint64_t));
	if (!toff)
		return OR_ENOMEM;
#pragma omp parallel for schedule(dynamic, 64)
	for (uint64_t u = 0; u < g->n; ++u)
		toff[u + 1] = list_triangles_of(g, u, NULL);
	for (uint64_t u = 0; u < g->n; ++u)
		toff[u + 1] += toff[u];
	const uint64_t T = toff[g->n];
	r->T = T;
	if (T > 0xffffffffULL)
	{
		free(toff);
		return OR_ERANGE;
	}
	r->tris = malloc((T ? 3 * T : 1) * sizeof(uint32_t));
	if (!r->tris)
	{
		free(toff);
		return OR_ENOMEM;
	}
#pragma omp parallel for schedule(dynamic, 64)
	for (uint64_t u = 0; u < g->n; ++u)
	{
		uint32_t *blk = r->tris + 3 * toff[u];
		uint64_t c = list_triangles_of(g, u, blk);
		qsort(blk, c, 3 * sizeof(uint32_t), cmp_ab);
	}
	free(toff);
	if (T == 0)
		return OR_OK;

	incidence inc;
	int rc = build_incidence(g, r->tris, T, &inc);
	if (rc)
		return rc;

	/* support (count_support, cuNucleus34_ondemand.cu:176-194) */
	r->support = malloc(T * sizeof(int32_t));
	r->k = malloc(T * sizeof(int32_t));
	if (!r->support || !r->k)
	{
		free_incidence(&inc);
		return OR_ENOMEM;
	}
	uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : total)
	for (uint64_t t = 0; t < T; ++t)
	{
		uint32_t c = for_each_clique(&inc, r->tris + 3 * t, NULL, NULL);
		r->support[t] = (int32_t)c;
		total += c;
	}
	r->Q = total / 4;

	if (quds_cap)
	{
		uint64_t cap = quds_cap < r->Q ? quds_cap : r->Q;
		r->quds = malloc((cap ? cap : 1) * 4 * sizeof(uint32_t));
		qud_ctx qc = {0, r->quds, cap, 0};
		for (uint64_t t = 0; t < T && qc.len < cap; ++t)
		{
			qc.owner = (uint32_t)t;
			for_each_clique(&inc, r->tris + 3 * t, collect_qud, &qc);
		}
		r->quds_len = qc.len;
	}

	/* bucket construction (bucket_ex.hpp:31-64) */
	int64_t maxv = 0;
	for (uint64_t t = 0; t < T; ++t)
		if (r->support[t] > maxv)
			maxv = r->support[t];
	bucket B;
	B.val = malloc(T * sizeof(int64_t));
	B.perm = malloc(T * sizeof(uint32_t));
	B.pos = malloc(T * sizeof(uint64_t));
	B.bin = calloc((size_t)maxv + 2, sizeof(uint64_t));
	if (!B.val || !B.perm || !B.pos || !B.bin)
	{
		free(B.val);
		free(B.perm);
		free(B.pos);
		free(B.bin);
		free_incidence(&inc);
		return OR_ENOMEM;
	}
	for (uint64_t t = 0; t < T; ++t)
		B.bin[r->support[t] + 1]++;
	for (int64_t v = 0; v <= maxv; ++v)
		B.bin[v + 1] += B.bin[v];
	/* B.bin[v] is now the start of bin v; place keys (counting sort) */
	{
		uint64_t *cur = malloc(((size_t)maxv + 1) * sizeof(uint64_t));
		if (!cur)
		{
			free(B.val);
			free(B.perm);
			free(B.pos);
			free(B.bin);
			free_incidence(&inc);
			return OR_ENOMEM;
		}
		memcpy(cur, B.bin, ((size_t)maxv + 1) * sizeof(uint64_t));
		for (uint64_t t = 0; t < T; ++t)
		{
			uint64_t p = cur[r->support[t]]++;
			B.perm[p] = (uint32_t)t;
			B.pos[t] = p;
		}
		free(cur);
	}
	for (uint64_t t = 0; t < T; ++t)
		B.val[t] = r->support[t] ? r->support[t] : -1; /* replace_copy 0 -> -1 */
	uint64_t min_id = B.bin[1 <= maxv ? 1 : maxv + 1];
	if (maxv == 0)
		min_id = T;
	B.last = 0;
	peel_ctx pc = {&B};
	while (min_id < T)
	{
		/* pop_min (bucket_ex.hpp:210-220) */
		const uint32_t key = B.perm[min_id++];
		B.last = B.val[key];
		for_each_clique(&inc, r->tris + 3 * (uint64_t)key, peel_clique, &pc);
		B.val[key]--; /* mark popped (bucket_ex.hpp:261) */
	}
	int64_t kmax = 0;
	long long ksum = 0;
	for (uint64_t t = 0; t < T; ++t)
	{
		const int32_t kv = (int32_t)(B.val[t] + 1); /* support(): value + 1 */
		r->k[t] = kv;
		ksum += kv;
		if (kv > kmax)
			kmax = kv;
	}
	r->k_max = (int32_t)kmax;
	r->k_avg = (double)ksum / (double)T;
	free(B.val);
	free(B.perm);
	free(B.pos);
	free(B.bin);
	free_incidence(&inc);
	return OR_OK;
}

/* ------------------------------------------------------------------------- */
/* level-synchronous peel with death rounds, and the result certificate      */
/* (checker side; no counterpart in the reference)                           */
/* ------------------------------------------------------------------------- */

/* The device peel's rules, restated on one thread: rounds at a level; a
 * round's frontier dies together; a clique belongs to its first member to
 * die, ties to the lowest id, and its owner debits the members still alive;
 * a triangle whose support reaches the level joins the next round; an empty
 * frontier moves the level to level+1 if some support is there, else to the
 * minimum support. Gives the same k as the bucket peel (the numbers are
 * unique) plus each triangle's death round. */
typedef struct
{
	const uint8_t *state; /* 0 alive, 1 dying this round, 2 dead */
	int32_t *S;
	int64_t level;
	uint32_t t;
	uint32_t *next;
	uint64_t nnext;
} round_ctx;

static void round_clique(void *vctx, uint32_t x, uint32_t p1, uint32_t p2, uint32_t p3)
{
	(void)x;
	round_ctx *c = vctx;
	const uint32_t m[3] = {p1, p2, p3};
	for (int s = 0; s < 3; ++s)
	{
		if (c->state[m[s]] == 2)
			return; /* destroyed in an earlier round */
		if (c->state[m[s]] == 1 && m[s] < c->t)
			return; /* owned by a lower dying member */
	}
	for (int s = 0; s < 3; ++s)
		if (c->state[m[s]] == 0 && --c->S[m[s]] == c->level)
			c->next[c->nnext++] = m[s];
}

int oracle_peel_rounds(const oracle_graph *g, const uint32_t *tris, uint64_t T, int32_t *k, uint32_t *rounds)
{
	if (T == 0)
		return OR_OK;
	incidence inc;
	int rc = build_incidence(g, tris, T, &inc);
	if (rc)
		return rc;
	int32_t *S = malloc(T * sizeof(int32_t));
	uint8_t *state = calloc(T, 1);
	uint32_t *front = malloc(T * sizeof(uint32_t)), *next = malloc(T * sizeof(uint32_t));
	if (!S || !state || !front || !next)
	{
		free(S), free(state), free(front), free(next);
		free_incidence(&inc);
		return OR_ENOMEM;
	}
	for (uint64_t t = 0; t < T; ++t)
		S[t] = (int32_t)for_each_clique(&inc, tris + 3 * t, NULL, NULL);
	int64_t level = -1;
	uint32_t round = 0;
	uint64_t nf = 0, peeled = 0;
	while (peeled < T)
	{
		if (nf == 0)
		{
			/* level change */
			int64_t mn = INT64_MAX;
			for (uint64_t t = 0; t < T; ++t)
				if (state[t] == 0 && S[t] < mn)
					mn = S[t];
			level = mn <= level + 1 ? level + 1 : mn;
			for (uint64_t t = 0; t < T; ++t)
				if (state[t] == 0 && S[t] <= level)
					front[nf++] = (uint32_t)t;
		}
		for (uint64_t i = 0; i < nf; ++i)
		{
			k[front[i]] = (int32_t)level;
			rounds[front[i]] = round;
			state[front[i]] = 1;
		}
		round_ctx rc2 = {state, S, level, 0, next, 0};
		for (uint64_t i = 0; i < nf; ++i)
		{
			rc2.t = front[i];
			for_each_clique(&inc, tris + 3 * (uint64_t)front[i], round_clique, &rc2);
		}
		for (uint64_t i = 0; i < nf; ++i)
			state[front[i]] = 2;
		peeled += nf;
		memcpy(front, next, rc2.nnext * sizeof(uint32_t));
		nf = rc2.nnext;
		++round;
	}
	free(S), free(state), free(front), free(next);
	free_incidence(&inc);
	return OR_OK;
}

/* Certificate of a peel result, the conditions the device check applies:
 * (A) t has at least k(t) cliques whose other triangles all have k >= k(t);
 * (B) t has at most k(t) cliques whose other triangles died in round r(t) or
 *     later (its support when its round began);
 * (C) the triangles of a round share one level, non-decreasing over rounds.
 * Returns the number of failing triangles plus failing rounds, or a negative
 * error code. */
typedef struct
{
	const int32_t *k;
	const uint32_t *r;
	int32_t kt;
	uint32_t rt;
	uint32_t a, b;
} cert_ctx;

static void cert_clique(void *vctx, uint32_t x, uint32_t p1, uint32_t p2, uint32_t p3)
{
	(void)x;
	cert_ctx *c = vctx;
	if (c->k[p1] >= c->kt && c->k[p2] >= c->kt && c->k[p3] >= c->kt)
		c->a++;
	if (c->r[p1] >= c->rt && c->r[p2] >= c->rt && c->r[p3] >= c->rt)
		c->b++;
}

int64_t oracle_certify(const oracle_graph *g, const uint32_t *tris, uint64_t T, const int32_t *k,
					   const uint32_t *rounds)
{
	if (T == 0)
		return 0;
	incidence inc;
	int rc = build_incidence(g, tris, T, &inc);
	if (rc)
		return rc;
	int64_t bad = 0;
	uint32_t rmax = 0;
	for (uint64_t t = 0; t < T; ++t)
	{
		cert_ctx c = {k, rounds, k[t], rounds[t], 0, 0};
		for_each_clique(&inc, tris + 3 * t, cert_clique, &c);
		if (k[t] < 0 || (int64_t)c.a < k[t] || (int64_t)c.b > k[t])
			++bad;
		if (rounds[t] > rmax)
			rmax = rounds[t];
	}
	free_incidence(&inc);
	int32_t *lo = malloc(((uint64_t)rmax + 1) * sizeof(int32_t)), *hi = malloc(((uint64_t)rmax + 1) * sizeof(int32_t));
	if (!lo || !hi)
	{
		free(lo), free(hi);
		return OR_ENOMEM;
	}
	for (uint64_t r = 0; r <= rmax; ++r)
		lo[r] = INT32_MAX, hi[r] = -1;
	for (uint64_t t = 0; t < T; ++t)
	{
		if (k[t] < lo[rounds[t]])
			lo[rounds[t]] = k[t];
		if (k[t] > hi[rounds[t]])
			hi[rounds[t]] = k[t];
	}
	int32_t prev = -1;
	for (uint64_t r = 0; r <= rmax; ++r)
	{
		if (hi[r] < 0)
			continue;
		if (lo[r] != hi[r] || lo[r] < prev)
			++bad;
		prev = hi[r];
	}
	free(lo), free(hi);
	return bad;
}

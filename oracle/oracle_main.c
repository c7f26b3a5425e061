/*
 * Command-line front end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.
 * Prints one JSON object with the counts, K_max, K_avg and the decomposition
 * time; with a second argument writes "(a,b,c)\t<k>" per triangle in
 * canonical order (the on-demand program's k-file layout,
 * cuNucleus34_ondemand.cu:724-733).
 */
#include <stdio.h>
#include <stdlib.h>
#include <time.h>

#include "nucleus34_oracle.h"

#ifdef _OPENMP
#include <omp.h>
#endif

static double now_s(void)
{
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

int main(int argc, char **argv)
{
	if (argc < 2)
	{
		fprintf(stderr, "usage: %s <graph> [kfile]\n", argv[0]);
		return 2;
	}
	oracle_graph g;
	double t0 = now_s();
	int rc = oracle_read_graph(argv[1], &g);
	if (rc)
	{
		fprintf(stderr, "read failed: %d\n", rc);
		return 1;
	}
	double t_load = now_s() - t0;
	oracle_result r;
	t0 = now_s();
	rc = oracle_decompose(&g, 5, &r);
	double t_dec = now_s() - t0;
	if (rc)
	{
		fprintf(stderr, "decompose failed: %d\n", rc);
		return 1;
	}
	int threads = 1;
#ifdef _OPENMP
	threads = omp_get_max_threads();
#endif
	printf("{\"vertex_count\": %llu, \"edge_count\": %llu, \"triangle_count\": %llu, "
		   "\"four_clique_count\": %llu, \"K_max\": %d, \"K_avg\": %.17g, \"threads\": %d, "
		   "\"t_load\": %.6f, \"t_decomp\": %.6f}\n",
		   (unsigned long long)g.n, (unsigned long long)(2 * g.m), (unsigned long long)r.T,
		   (unsigned long long)r.Q, r.k_max, r.k_avg, threads, t_load, t_dec);
	if (argc > 2)
	{
		FILE *f = fopen(argv[2], "w");
		if (!f)
			return 1;
		for (unsigned long long i = 0; i < r.T; ++i)
			fprintf(f, "(%u,%u,%u)\t%d\n", r.tris[3 * i], r.tris[3 * i + 1], r.tris[3 * i + 2], r.k[i]);
		fclose(f);
	}
	oracle_result_free(&r);
	oracle_graph_free(&g);
	return 0;
}

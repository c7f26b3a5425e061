// Test infrastructure (oracle side), not product code.
//
// A small driver, written for this project, that runs the reference's OWN
// host-side (3,4)-nucleus path by including its headers where they lie (the
// build recipe in oracle/Makefile points -I at the reference tree; nothing of
// the reference is copied here). The call sequence is the one the reference's
// CPU code composes:
//
//   graph_t<EDGE_T,VERTEX_T>::from_edges / deserialize   nucleus/graph/graph.hpp:285-411, 491-520
//   make_oriented                                        nucleus/graph/graph.hpp:176-218
//   make_split_parts(nprocs)                             nucleus/graph/graph.hpp:581-605
//   cliques_tri_par                                      nucleus/cliques.hpp:98-226
//   graph_t<U,V,2>(tris, m, true)   (sorts by (a,b))     nucleus/graph/graph.hpp:100-131
//   cliques_qud_par                                      nucleus/cliques.hpp:570-711
//   graph_t<U,V,3>(quds, T, false)                       nucleus/graph/graph.hpp:132-173
//   bucket_ex<V,long>(qg.D).peeling_par(qg).support()    nucleus/bucket_ex.hpp:31-99, 274-360
//
// Output (stdout): one JSON object with vertex_count, edge_count, triangle_count,
// four_clique_count, K_max, K_avg and phase times. With a second argument, the
// per-triangle file "(a,b,c)\t<k>" in canonical (a,b) order is written there.
#include <chrono>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "bucket_ex.hpp"
#include "cliques.hpp"
#include "graph/graph.hpp"
#include "utility/def_system.hpp"

using clk = std::chrono::steady_clock;

static double since(clk::time_point t0)
{
	return std::chrono::duration<double>(clk::now() - t0).count();
}

int main(int argc, char **argv)
{
	if (argc < 2)
	{
		std::cerr << "usage: " << argv[0] << " <graph .edges|.txt|.mtx|.grh> [kfile]\n";
		return 2;
	}
	const std::string path(argv[1]);
	const std::string kfile = argc > 2 ? argv[2] : "";
	const int nprocs = omp_get_num_procs();

	auto t0 = clk::now();
	graph_t<EDGE_T, VERTEX_T> g;
	const auto ext = get_ext(path);
	if (ext == ".mtx")
	{
		g.from_edges(path, true);
		g.make_oriented();
	}
	else if (ext == ".edges" || ext == ".txt")
	{
		g.from_edges(path, false);
		g.make_oriented();
	}
	else if (ext == ".grh")
	{
		g.deserialize(path);
		g.build_offset();
	}
	else
	{
		std::cerr << "unknown extension " << ext << "\n";
		return 2;
	}
	g.make_split_parts(nprocs);
	const double t_load = since(t0);

	const size_t nV = g.size_vertices(), nE = g.size_edges();

	t0 = clk::now();
	auto tris = cliques_tri_par(g);
	const double t_tri = since(t0);
	const size_t T = tris.size();

	double t_qud = 0, t_peel = 0;
	size_t Q = 0;
	long kmax = 0;
	double kavg = 0;
	std::vector<long> k;

	t0 = clk::now();
	graph_t<EDGE_T, VERTEX_T, 2> tg(tris, nE, true); // sorts tris by (a,b) in place
	tg.make_split_parts(nprocs);
	auto quds = cliques_qud_par(tg);
	t_qud = since(t0);
	Q = quds.size();

	if (T)
	{
		t0 = clk::now();
		graph_t<EDGE_T, VERTEX_T, 3> qg(quds, T, false);
		bucket_ex<VERTEX_T, long> bkt(qg.D);
		bkt.peeling_par(qg);
		k = bkt.support();
		t_peel = since(t0);
		long long s = 0;
		for (auto v : k)
		{
			s += v;
			kmax = std::max(kmax, v);
		}
		kavg = k.empty() ? 0.0 : static_cast<double>(s) / static_cast<double>(k.size());
	}

	std::cout << "{\"vertex_count\": " << nV << ", \"edge_count\": " << 2 * nE
			  << ", \"triangle_count\": " << T << ", \"four_clique_count\": " << Q
			  << ", \"K_max\": " << kmax << ", \"K_avg\": " << kavg
			  << ", \"threads\": " << nprocs
			  << ", \"t_load\": " << t_load << ", \"t_triangles\": " << t_tri
			  << ", \"t_four_cliques\": " << t_qud << ", \"t_peel\": " << t_peel
			  << ", \"t_decomp\": " << (t_tri + t_qud + t_peel) << "}" << std::endl;

	if (!kfile.empty())
	{
		std::ofstream out(kfile);
		for (size_t i = 0; i < T; ++i)
			out << '(' << tris[i][0] << ',' << tris[i][1] << ',' << tris[i][2] << ")\t" << k[i] << '\n';
	}
	return 0;
}

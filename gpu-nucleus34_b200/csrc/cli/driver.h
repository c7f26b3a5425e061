// The drop-in program flow shared by cuNucleus34 and cuNucleus34_ondemand:
// argv -> load (by extension) -> C-ABI decomposition -> JSON record on stdout,
// "[phase]" lines on stderr, optional per-triangle k file. Mirrors the
// reference mains (nucleus/cuNucleus34.cu:144-839,
// nucleus/cuNucleus34_ondemand.cu:308-784) field by field; the differences are
// listed where they occur.
#pragma once

#include "record.h"

namespace rec {

struct ProgramSpec
{
	bool direct;
	const char *app;
	const char *version;
};

inline int run_program(const ProgramSpec &spec, int argc, char **argv)
{
	const char *prog = argv[0];
	if (argc < 2)
	{
		std::cerr << "Usage: " << strip_path(prog) << " <dataset file (.mtx or .grh)>"
				  << (spec.direct ? " [parts (default 1; >1 enables the parted multi-GPU pipeline)]" : "")
				  << " [results output file (optional)]" << std::endl;
		return EXIT_FAILURE;
	}
	const std::string dataset(argv[1]);
	size_t parts = 1;
	std::string output;
	if (spec.direct)
	{
		if (argc > 2)
		{
			try
			{
				parts = size_t(std::stoul(argv[2]));
			}
			catch (...)
			{
				parts = 1;
			}
			if (parts < 1)
				parts = 1;
		}
		if (argc > 3)
			output = argv[3];
	}
	else if (argc > 2)
		output = argv[2];

	std::string step;
	phase(step, "0.1 Environment info collection");
	Json j;
	environment(j, spec.app, spec.version, spec.direct, parts);
	j.begin(false, "dataset");
	j.field(true, "file", strip_path(dataset));

	nucleus34_handle h = nullptr;
	try
	{
		phase(step, "0.2 Data loading and graph construction");
		nucleus34_graph g{};
		auto t0 = std::chrono::steady_clock::now();
		check(nucleus34_graph_load(dataset.c_str(), &g), "load");
		const double t_data = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
		j.field(false, "vertex_count", size_t(g.n));
		j.field(false, "edge_count", size_t(g.m) * 2);
		j.raw(false, "data_loading_time_sec", fixed2(t_data));
		if (spec.direct)
			j.field(false, "data_memory_bytes", size_t(4 * (g.n + 1) + 4 * g.n + 4 * g.m));
		mem_note("graph", "vertices=" + std::to_string(g.n) + " oriented_edges=" + std::to_string(g.m) +
							  " host_graph=" + std::to_string((4 * (2 * g.n + 1) + 4 * g.m) >> 20) + " MiB load=" +
							  secs1(t_data));

		phase(step, spec.direct ? "1.1 Triangle counting, four-cliques and peeling (device)"
								: "1.1 Triangle counting, incidence, support and peeling (device)");
		nucleus34_opts opts{};
		opts.device = 0;
		opts.parts = uint32_t(parts);
		// scheduling table of the on-demand variant (argv stays the reference's)
		const char *tune = std::getenv("NUCLEUS34_TUNE_TABLE");
		if (tune && *tune)
			opts.tune_table = tune;
		nucleus34_result r{};
		const nucleus34_csr csr = nucleus34_graph_csr(&g);
		int rc = spec.direct ? nucleus34_decompose(&csr, &opts, &r, &h) : nucleus34_decompose_ondemand(&csr, &opts, &r, &h);
		nucleus34_graph_release(&g);
		check(rc, "decompose");
		{
			const uint64_t T = r.triangle_count, Q = r.four_clique_count;
			if (spec.direct)
			{
				mem_note("tri-done", "triangles=" + std::to_string(T) + " device_tris=" +
										 std::to_string((12 * T) >> 20) + " MiB time=" + secs1(r.t_triangles));
				mem_note("fc-done", "four_cliques=" + std::to_string(Q) + " peak_device=" +
										std::to_string(r.peak_device_bytes >> 20) + " MiB time=" + secs1(r.t_support));
				if (Q)
					mem_note("inc-done", "triangle->four-clique CSR built");
			}
			else
			{
				mem_note("incidence", "entries=" + std::to_string(r.incidence_entries) + " bytes=" +
										  std::to_string((r.incidence_entries * 8) >> 20) + " MiB");
				std::cerr << "[mem] support four_cliques=" << Q << " incidences=" << 4 * Q
						  << " time=" << secs1(r.t_support) << std::endl;
			}
		}

		const uint64_t T = r.triangle_count;
		std::vector<int32_t> k(T);
		std::vector<uint32_t> tris(3 * T);
		check(nucleus34_copy_k(h, k.data(), tris.data()), "copy_k");

		j.field(false, "triangle_time_sec", r.t_triangles);
		j.field(false, "triangle_count", size_t(T));
		if (spec.direct)
		{
			// canonical (sorted) order; the reference prints its unsorted,
			// atomically ordered list here (cuNucleus34.cu:430-436)
			std::vector<const uint32_t *> first;
			for (uint64_t i = 0; i < std::min<uint64_t>(PRINT_CAP, T); ++i)
				first.push_back(&tris[3 * i]);
			j.array(false, "triangles", first.begin(), first.end(),
					[](std::ostream &os, const uint32_t *t) { print_tri(os, t); });
		}
		if (!T)
		{ // early finish without triangles (cuNucleus34.cu:439-446)
			j.end();
			j.last();
			j.print();
			nucleus34_free(h);
			return EXIT_SUCCESS;
		}
		if (spec.direct)
			j.field(false, "triangle_graph_time_sec", r.t_incidence);
		else
		{
			j.field(false, "incidence_time_sec", r.t_incidence);
			j.field(false, "incidence_entries", size_t(r.incidence_entries));
		}
		j.field(false, "four_clique_time_sec", r.t_support);
		j.field(false, "four_clique_count", size_t(r.four_clique_count));
		if (spec.direct)
		{
			const uint64_t nq = std::min<uint64_t>(PRINT_CAP, r.four_clique_count);
			std::vector<uint32_t> q(4 * nq);
			if (nq)
				check(nucleus34_copy_quds(h, 0, nq, q.data()), "copy_quds");
			std::vector<const uint32_t *> first;
			for (uint64_t i = 0; i < nq; ++i)
				first.push_back(&q[4 * i]);
			j.array(false, "four-cliques", first.begin(), first.end(),
					[](std::ostream &os, const uint32_t *x) { print_qud(os, x); });
		}
		if (!r.four_clique_count)
		{ // early finish without four-cliques (cuNucleus34.cu:598-605)
			j.end();
			j.last();
			j.print();
			nucleus34_free(h);
			return EXIT_SUCCESS;
		}
		if (spec.direct)
		{
			j.field(false, "four_clique_graph_time_sec", r.t_cliques);
			j.field(false, "peeling_mode", std::string("resident-direct"));
			j.field(false, "peeling_preprocess_time_sec", 0.0);
		}
		else
		{
			j.field(false, "unpeeled_count", size_t(r.unpeeled_count));
			if (r.unpeeled_count)
				std::cerr << "[warn] " << r.unpeeled_count << " triangles left unpeeled" << std::endl;
			j.field(false, "peeling_mode", std::string("ondemand-reenumerate"));
		}
		j.field(false, "peeling_time_sec", r.t_peel);
		j.field(false, "peeling_iterations", size_t(r.peeling_iterations));
		j.field(false, "K_max", r.k_max);
		j.field(false, "total_time_sec", r.t_total);
		phase(step, "4.3 Finalizing results on host");
		j.field(false, "K_count", k.size());
		j.array(false, "K", k.begin(), k.begin() + std::min<size_t>(PRINT_CAP, k.size()),
				[](std::ostream &os, int32_t v) { os << v; });
		if (!output.empty())
			check(nucleus34_write_kfile(h, output.c_str()), "write k file");
		j.field(false, "K_avg", r.k_avg);
		j.end();
		j.last();
		j.print();
	}
	catch (const Error &e)
	{
		std::cerr << "Dataset: " << dataset << std::endl
				  << "Step: " << step << std::endl
				  << "Error: " << e.msg << std::endl;
		j.field(false, "errorstep", step);
		j.field(false, "error", e.msg);
		j.end();
		j.last();
		j.print();
	}
	catch (const std::exception &e)
	{
		std::cerr << "Dataset: " << dataset << std::endl << "Step: " << step << std::endl << "Error: " << e.what() << std::endl;
		j.field(false, "errorstep", step);
		j.field(false, "error", std::string(e.what()));
		j.end();
		j.last();
		j.print();
	}
	nucleus34_free(h);
	// handled errors still exit 0, as the reference does (cuNucleus34.cu:838)
	return EXIT_SUCCESS;
}

} // namespace rec

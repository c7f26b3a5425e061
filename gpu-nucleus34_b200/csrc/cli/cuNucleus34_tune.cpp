// cuNucleus34_tune <dataset> <tune table>: autotunes the on-demand variant for
// the dataset's graph class (nucleus34_ctx_autotune) and writes the fastest
// settings into the table, which cuNucleus34_ondemand then reads from
// NUCLEUS34_TUNE_TABLE. Prints one JSON line: the class, the settings and the
// device times of the default and the tuned decomposition, and of a last
// unpinned run that takes its settings from the table. Exit code 1 on any
// error (the JSON then holds "error").
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>

#include "nucleus34.h"

namespace {

int finish_error(const char *what, int rc)
{
	std::printf("{\"error\": \"%s: %s (%s)\"}\n", what, nucleus34_strerror(rc), nucleus34_last_error());
	return EXIT_FAILURE;
}

std::string setting(uint32_t v) { return v == NUCLEUS34_TUNE_NEVER ? "\"never\"" : std::to_string(v); }

} // namespace

int main(int argc, char **argv)
{
	if (argc < 3)
	{
		std::fprintf(stderr, "Usage: %s <dataset file (.mtx, .edges, .txt or .grh)> <tune table>\n", argv[0]);
		return EXIT_FAILURE;
	}
	nucleus34_graph g{};
	int rc = nucleus34_graph_load(argv[1], &g);
	if (rc)
		return finish_error("load", rc);
	nucleus34_opts opts{};
	nucleus34_ctx ctx = nullptr;
	rc = nucleus34_ctx_create(&opts, &ctx);
	if (rc)
	{
		nucleus34_graph_release(&g);
		return finish_error("context", rc);
	}
	const nucleus34_csr csr = nucleus34_graph_csr(&g);
	rc = nucleus34_ctx_upload(ctx, &csr);
	nucleus34_graph_release(&g);
	nucleus34_tune applied{};
	double best_sec = 0, default_sec = 0;
	if (!rc)
		rc = nucleus34_ctx_autotune(ctx, argv[2], nullptr, &best_sec, &default_sec);
	// a final unpinned run takes its settings from the table just written
	nucleus34_result r{};
	if (!rc)
		rc = nucleus34_ctx_run(ctx, NUCLEUS34_ONDEMAND, &r);
	if (!rc)
		rc = nucleus34_ctx_last_tune(ctx, &applied);
	nucleus34_ctx_destroy(ctx);
	if (rc)
		return finish_error("autotune", rc);
	std::printf("{\"table\": \"%s\", \"triangle_count\": %llu, \"four_clique_count\": %llu, "
				"\"lane_max\": %s, \"compact_div\": %s, \"sort_shift\": %s, \"rounds_per_replay\": %s, "
				"\"default_sec\": %.4f, \"tuned_sec\": %.4f, \"check_sec\": %.4f}\n",
				argv[2], (unsigned long long)r.triangle_count, (unsigned long long)r.four_clique_count,
				setting(applied.lane_max).c_str(), setting(applied.compact_div).c_str(),
				setting(applied.sort_shift).c_str(), setting(applied.rounds_per_replay).c_str(), default_sec, best_sec,
				r.t_total);
	return EXIT_SUCCESS;
}

// C-ABI entry points of the host graph layer and generators, plus the shared
// error reporting. No exception leaves this file.
#include "host_internal.h"

#include <cstdlib>
#include <cstring>
#include <exception>
#include <new>

namespace n34 {

namespace {
thread_local std::string g_last_error;
}

int fail(int code, const std::string &msg)
{
	g_last_error = msg;
	return code;
}

void clear_error() { g_last_error.clear(); }

int export_graph(HostGraph &&hg, nucleus34_graph *g)
{
	g->n = hg.n;
	g->m = hg.m;
	g->O = static_cast<uint32_t *>(std::malloc((hg.n + 1) * sizeof(uint32_t)));
	g->D = static_cast<uint32_t *>(std::malloc((hg.n ? hg.n : 1) * sizeof(uint32_t)));
	g->E = static_cast<uint32_t *>(std::malloc((hg.m ? hg.m : 1) * sizeof(uint32_t)));
	if (!g->O || !g->D || !g->E)
	{
		nucleus34_graph_release(g);
		return fail(NUCLEUS34_E_INVALID, "host allocation failed");
	}
	std::memcpy(g->O, hg.O.data(), (hg.n + 1) * sizeof(uint32_t));
	if (hg.n)
		std::memcpy(g->D, hg.D.data(), hg.n * sizeof(uint32_t));
	if (hg.m)
		std::memcpy(g->E, hg.E.data(), hg.m * sizeof(uint32_t));
	return NUCLEUS34_OK;
}

int gen_rmat(uint32_t, uint32_t, double, double, double, uint64_t, nucleus34_edges *);
int gen_rgg(uint64_t, double, uint64_t, nucleus34_edges *);
int gen_ws(uint64_t, uint32_t, double, uint64_t, nucleus34_edges *);
int write_edges(const nucleus34_edges *, const char *);
uint64_t splitmix64(uint64_t);

template <class F>
int guarded(F &&f)
{
	clear_error();
	try
	{
		return f();
	}
	catch (const std::bad_alloc &)
	{
		return fail(NUCLEUS34_E_INVALID, "host allocation failed");
	}
	catch (const std::exception &e)
	{
		return fail(NUCLEUS34_E_INVALID, e.what());
	}
	catch (...)
	{
		return fail(NUCLEUS34_E_INVALID, "unknown host error");
	}
}

} // namespace n34

using namespace n34;

extern "C" {

const char *nucleus34_strerror(int code)
{
	switch (code)
	{
	case NUCLEUS34_OK:
		return "success";
	case NUCLEUS34_E_INVALID:
		return "invalid argument";
	case NUCLEUS34_E_OOM_BUDGET:
		return "device memory budget exceeded";
	case NUCLEUS34_E_RANGE32:
		return "32-bit id range exceeded";
	case NUCLEUS34_E_CUDA:
		return "CUDA error";
	case NUCLEUS34_E_TIMEOUT:
		return "bounded device wait timed out";
	case NUCLEUS34_E_IO:
		return "I/O error";
	case NUCLEUS34_E_FORMAT:
		return "unknown or malformed dataset format";
	case NUCLEUS34_E_NODEVICE:
		return "no usable CUDA device";
	case NUCLEUS34_E_STATE:
		return "call out of order";
	default:
		return "unknown error";
	}
}

const char *nucleus34_last_error(void) { return g_last_error.c_str(); }

int nucleus34_graph_load(const char *path, nucleus34_graph *g)
{
	if (!g)
		return fail(NUCLEUS34_E_INVALID, "null graph");
	std::memset(g, 0, sizeof(*g));
	return guarded([&] {
		HostGraph hg;
		int rc = load_graph(path, hg);
		return rc ? rc : export_graph(std::move(hg), g);
	});
}

int nucleus34_graph_from_edges(const uint32_t *src, const uint32_t *dst, uint64_t count, nucleus34_graph *g)
{
	if (!g || (count && (!src || !dst)))
		return fail(NUCLEUS34_E_INVALID, "null argument");
	std::memset(g, 0, sizeof(*g));
	return guarded([&] {
		HostGraph hg;
		int rc = build_oriented(src, dst, count, hg);
		return rc ? rc : export_graph(std::move(hg), g);
	});
}

int nucleus34_graph_save_grh(const nucleus34_graph *g, const char *path)
{
	if (!g || !path)
		return fail(NUCLEUS34_E_INVALID, "null argument");
	return guarded([&] { return save_grh(g, path); });
}

void nucleus34_graph_release(nucleus34_graph *g)
{
	if (!g)
		return;
	std::free(g->O);
	std::free(g->D);
	std::free(g->E);
	std::memset(g, 0, sizeof(*g));
}

nucleus34_csr nucleus34_graph_csr(const nucleus34_graph *g)
{
	nucleus34_csr c{};
	if (g)
	{
		c.n = g->n;
		c.m = g->m;
		c.O = g->O;
		c.D = g->D;
		c.E = g->E;
	}
	return c;
}

int nucleus34_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
					   nucleus34_edges *out)
{
	if (!out)
		return fail(NUCLEUS34_E_INVALID, "null output");
	std::memset(out, 0, sizeof(*out));
	return guarded([&] { return gen_rmat(scale, edge_factor, a, b, c, seed, out); });
}

int nucleus34_gen_rgg(uint64_t n, double expected_degree, uint64_t seed, nucleus34_edges *out)
{
	if (!out)
		return fail(NUCLEUS34_E_INVALID, "null output");
	std::memset(out, 0, sizeof(*out));
	return guarded([&] { return gen_rgg(n, expected_degree, seed, out); });
}

int nucleus34_gen_ws(uint64_t n, uint32_t k, double beta, uint64_t seed, nucleus34_edges *out)
{
	if (!out)
		return fail(NUCLEUS34_E_INVALID, "null output");
	std::memset(out, 0, sizeof(*out));
	return guarded([&] { return gen_ws(n, k, beta, seed, out); });
}

int nucleus34_edges_write(const nucleus34_edges *e, const char *path)
{
	if (!e || !path)
		return fail(NUCLEUS34_E_INVALID, "null argument");
	return guarded([&] { return write_edges(e, path); });
}

void nucleus34_edges_release(nucleus34_edges *e)
{
	if (!e)
		return;
	std::free(e->src);
	std::free(e->dst);
	std::memset(e, 0, sizeof(*e));
}

uint64_t nucleus34_splitmix64(uint64_t x) { return splitmix64(x); }

} // extern "C"

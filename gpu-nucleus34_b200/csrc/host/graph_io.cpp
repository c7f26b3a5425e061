// Host graph layer: readers (.mtx/.edges/.txt/.grh), undirected CSR build,
// degree orientation and the .grh writer, with the reference's semantics:
//   from_edges      nucleus/graph/graph.hpp:285-411
//   make_oriented   nucleus/graph/graph.hpp:176-218 (vertex_less, graph_api.hpp:124-127)
//   deserialize     nucleus/graph/graph.hpp:491-520, build_offset :523-536
//   serialize       nucleus/graph/graph.hpp:465-488
// The parse is parallel (OpenMP over line-aligned chunks) and the pair
// sort + unique of from_edges is done as a counting sort by source followed by
// a per-list sort + unique, which yields the same sorted unique adjacency.
#include "host_internal.h"

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <fcntl.h>
#include <memory>
#include <omp.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

namespace n34 {

namespace {

bool is_digit(char c) { return c >= '0' && c <= '9'; }

// "<uint> <uint>" at the start of a line, as `ss >> s >> d` reads well-formed
// input (graph.hpp:361-363). Lines without two numbers are skipped (the
// reference reads uninitialised values for them). Reads from p up to end and
// reports where it stopped; the caller skips the rest of the line from there.
// A line's numbers cannot run past its newline: '\n' is neither a digit, a
// space nor a tab.
inline bool parse_two_at(const char *p, const char *end, uint32_t &s, uint32_t &d, const char *&stop)
{
	stop = p;
	while (p < end && (*p == ' ' || *p == '\t'))
		++p;
	if (p >= end || !is_digit(*p))
	{
		stop = p;
		return false;
	}
	uint64_t a = 0;
	while (p < end && is_digit(*p))
	{
		a = a * 10 + uint64_t(*p - '0');
		if (a > 0xffffffffull)
		{
			stop = p;
			return false;
		}
		++p;
	}
	while (p < end && (*p == ' ' || *p == '\t'))
		++p;
	if (p >= end || !is_digit(*p))
	{
		stop = p;
		return false;
	}
	uint64_t b = 0;
	while (p < end && is_digit(*p))
	{
		b = b * 10 + uint64_t(*p - '0');
		if (b > 0xffffffffull)
		{
			stop = p;
			return false;
		}
		++p;
	}
	stop = p;
	s = uint32_t(a);
	d = uint32_t(b);
	return true;
}

std::string file_ext(const std::string &path)
{
	auto dot = path.find_last_of('.');
	auto slash = path.find_last_of('/');
	if (dot == std::string::npos || (slash != std::string::npos && dot < slash))
		return "";
	return path.substr(dot);
}

int read_file(const char *path, std::vector<char> &buf)
{
	FILE *f = std::fopen(path, "rb");
	if (!f)
		return fail(NUCLEUS34_E_IO, std::string("Dataset ") + path + " is not accessible!");
	std::fseek(f, 0, SEEK_END);
	long sz = std::ftell(f);
	std::fseek(f, 0, SEEK_SET);
	if (sz < 0)
	{
		std::fclose(f);
		return fail(NUCLEUS34_E_IO, "cannot size file");
	}
	buf.resize(size_t(sz) + 1);
	size_t got = sz ? std::fread(buf.data(), 1, size_t(sz), f) : 0;
	std::fclose(f);
	if (got != size_t(sz))
		return fail(NUCLEUS34_E_IO, "short read");
	buf[size_t(sz)] = '\n';
	buf.resize(size_t(sz));
	return NUCLEUS34_OK;
}

} // namespace

namespace {

// A text file mapped read-only (or, where mapping fails, read into memory).
struct MappedText
{
	const char *data = nullptr;
	size_t size = 0;
	void *map = nullptr;
	std::vector<char> copy;
	int open(const char *path)
	{
		const int fd = ::open(path, O_RDONLY);
		if (fd < 0)
			return fail(NUCLEUS34_E_IO, std::string("Dataset ") + path + " is not accessible!");
		struct stat st;
		if (fstat(fd, &st) == 0 && st.st_size > 0)
		{
			void *m = mmap(nullptr, size_t(st.st_size), PROT_READ, MAP_PRIVATE, fd, 0);
			if (m != MAP_FAILED)
			{
				madvise(m, size_t(st.st_size), MADV_SEQUENTIAL);
				map = m;
				data = static_cast<const char *>(m);
				size = size_t(st.st_size);
				::close(fd);
				return NUCLEUS34_OK;
			}
		}
		::close(fd);
		const int rc = read_file(path, copy);
		data = copy.data();
		size = copy.size();
		return rc;
	}
	~MappedText()
	{
		if (map)
			munmap(map, size);
	}
};

// A slice of the input pairs; the parser hands over its per-thread slices
// as they are, without concatenating them.
struct PairSlice
{
	const uint32_t *src, *dst;
	uint64_t count;
};

int build_oriented_slices(const std::vector<PairSlice> &parts, HostGraph &out)
{
	const int nth = std::max(1, omp_get_max_threads());
	const int64_t np = int64_t(parts.size());
	// max_node over non-self-loop pairs only (graph.hpp:365-369)
	uint32_t max_node = 0;
#pragma omp parallel for reduction(max : max_node) schedule(dynamic, 1) num_threads(nth)
	for (int64_t pi = 0; pi < np; ++pi)
	{
		const PairSlice &ps = parts[size_t(pi)];
		for (uint64_t i = 0; i < ps.count; ++i)
			if (ps.src[i] != ps.dst[i])
				max_node = std::max(max_node, std::max(ps.src[i], ps.dst[i]));
	}
	const uint64_t n = uint64_t(max_node) + 1;

	// Undirected CSR, both directions, built in buckets of 2^SH vertices so
	// that every write stays in cache: each thread counts and then scatters
	// its slices of the pairs into the buckets' regions (the entry carries its
	// source's low SH bits), and each bucket is then counting-sorted by source
	// in place, where its lists are sorted and deduplicated. Thread t takes
	// slices t, t + nth, ... in both passes.
	constexpr uint32_t SH = 12;
	const uint64_t nb = (n >> SH) + 1;
	std::vector<uint64_t> cursor(uint64_t(nth) * nb, 0);
#pragma omp parallel num_threads(nth)
	{
		const int t = omp_get_thread_num();
		uint64_t *h = cursor.data() + uint64_t(t) * nb;
		for (int64_t pi = t; pi < np; pi += nth)
		{
			const PairSlice &ps = parts[size_t(pi)];
			for (uint64_t i = 0; i < ps.count; ++i)
				if (ps.src[i] != ps.dst[i])
				{
					h[ps.src[i] >> SH]++;
					h[ps.dst[i] >> SH]++;
				}
		}
	}
	std::vector<uint64_t> bstart(nb + 1, 0);
	uint64_t run = 0;
	for (uint64_t b = 0; b < nb; ++b)
	{
		bstart[b] = run;
		for (int t = 0; t < nth; ++t)
		{
			const uint64_t c = cursor[uint64_t(t) * nb + b];
			cursor[uint64_t(t) * nb + b] = run;
			run += c;
		}
	}
	bstart[nb] = run;
	const uint64_t total = run;
	std::vector<uint32_t> adj(total ? total : 1);
	std::vector<uint16_t> low(total ? total : 1);
#pragma omp parallel num_threads(nth)
	{
		const int t = omp_get_thread_num();
		uint64_t *h = cursor.data() + uint64_t(t) * nb;
		constexpr uint32_t MASK = (1u << SH) - 1;
		for (int64_t pi = t; pi < np; pi += nth)
		{
			const PairSlice &ps = parts[size_t(pi)];
			for (uint64_t i = 0; i < ps.count; ++i)
			{
				const uint32_t u = ps.src[i], v = ps.dst[i];
				if (u == v)
					continue;
				uint64_t p = h[u >> SH]++;
				adj[p] = v;
				low[p] = uint16_t(u & MASK);
				p = h[v >> SH]++;
				adj[p] = u;
				low[p] = uint16_t(v & MASK);
			}
		}
	}
	std::vector<uint64_t> off(n + 1, 0);
	off[n] = total;
	// per-list sort + unique == global pair sort + unique (graph.hpp:383-388)
	std::vector<uint32_t> udeg(n, 0);
#pragma omp parallel num_threads(nth)
	{
		std::vector<uint64_t> cnt((1u << SH) + 1);
		std::vector<uint32_t> tmp;
#pragma omp for schedule(dynamic, 4)
		for (int64_t b = 0; b < int64_t(nb); ++b)
		{
			const uint64_t s0 = bstart[b], e0 = bstart[b + 1];
			const uint64_t v0 = uint64_t(b) << SH;
			const uint64_t nv = std::min<uint64_t>(uint64_t(1) << SH, n - std::min(n, v0));
			std::fill(cnt.begin(), cnt.end(), 0);
			for (uint64_t p = s0; p < e0; ++p)
				cnt[low[p] + 1]++;
			for (uint64_t j = 0; j < nv; ++j)
			{
				cnt[j + 1] += cnt[j];
				off[v0 + j] = s0 + cnt[j];
			}
			tmp.resize(e0 - s0);
			for (uint64_t p = s0; p < e0; ++p)
				tmp[cnt[low[p]]++] = adj[p];
			std::copy(tmp.begin(), tmp.end(), adj.begin() + s0);
			for (uint64_t j = 0; j < nv; ++j)
			{
				uint32_t *lb = adj.data() + off[v0 + j];
				uint32_t *le = adj.data() + (j + 1 < nv ? off[v0 + j + 1] : e0);
				std::sort(lb, le);
				udeg[v0 + j] = uint32_t(std::unique(lb, le) - lb);
			}
		}
	}
	// orientation on the undirected degree (graph.hpp:196-213)
	out.n = n;
	out.O.assign(n + 1, 0);
	out.D.assign(n, 0);
#pragma omp parallel for schedule(dynamic, 256)
	for (int64_t u = 0; u < int64_t(n); ++u)
	{
		uint32_t k = 0;
		const uint32_t du = udeg[u];
		for (uint64_t j = off[u]; j < off[u] + udeg[u]; ++j)
		{
			const uint32_t v = adj[j];
			if (du < udeg[v] || (du == udeg[v] && uint32_t(u) < v))
				++k;
		}
		out.D[u] = k;
	}
	for (uint64_t u = 0; u < n; ++u)
	{
		if (uint64_t(out.O[u]) + out.D[u] > 0xffffffffull)
			return fail(NUCLEUS34_E_RANGE32, "oriented edge count exceeds 32-bit edge ids");
		out.O[u + 1] = out.O[u] + out.D[u];
	}
	out.m = out.O[n];
	out.E.assign(out.m ? out.m : 1, 0);
	out.E.resize(out.m);
#pragma omp parallel for schedule(dynamic, 256)
	for (int64_t u = 0; u < int64_t(n); ++u)
	{
		uint32_t w = out.O[u];
		const uint32_t du = udeg[u];
		for (uint64_t j = off[u]; j < off[u] + udeg[u]; ++j)
		{
			const uint32_t v = adj[j];
			if (du < udeg[v] || (du == udeg[v] && uint32_t(u) < v))
				out.E[w++] = v;
		}
	}
	return NUCLEUS34_OK;
}

} // namespace

int build_oriented(const uint32_t *src, const uint32_t *dst, uint64_t count, HostGraph &out)
{
	const uint64_t nth = uint64_t(std::max(1, omp_get_max_threads()));
	std::vector<PairSlice> parts;
	for (uint64_t t = 0; t < nth; ++t)
	{
		const uint64_t lo = count * t / nth, hi = count * (t + 1) / nth;
		parts.push_back(PairSlice{src + lo, dst + lo, hi - lo});
	}
	return build_oriented_slices(parts, out);
}

int load_graph(const char *path, HostGraph &g)
{
	if (!path)
		return fail(NUCLEUS34_E_INVALID, "null path");
	const std::string ext = file_ext(path);
	if (ext == ".grh")
	{
		FILE *f = std::fopen(path, "rb");
		if (!f)
			return fail(NUCLEUS34_E_IO, "Can't open file for reading.");
		uint64_t sv = 0, nV = 0, nE = 0;
		bool ok = std::fread(&sv, 8, 1, f) == 1 && std::fread(&nV, 8, 1, f) == 1 &&
				  std::fread(&nE, 8, 1, f) == 1;
		if (!ok || sv != sizeof(uint32_t))
		{
			std::fclose(f);
			return fail(NUCLEUS34_E_FORMAT, "Incompatible types in dataset.");
		}
		if (nE > 0xffffffffull)
		{
			std::fclose(f);
			return fail(NUCLEUS34_E_RANGE32, "edge count exceeds 32-bit edge ids");
		}
		g.n = nV;
		g.D.resize(nV);
		g.E.resize(nE);
		ok = (nV == 0 || std::fread(g.D.data(), 4, nV, f) == nV) &&
			 (nE == 0 || std::fread(g.E.data(), 4, nE, f) == nE);
		std::fclose(f);
		if (!ok)
			return fail(NUCLEUS34_E_FORMAT, "truncated .grh file");
		g.O.assign(nV + 1, 0);
		for (uint64_t u = 0; u < nV; ++u)
			g.O[u + 1] = g.O[u] + g.D[u];
		if (g.O[nV] != nE)
			return fail(NUCLEUS34_E_FORMAT, ".grh degree sum does not match its edge count");
		g.m = nE;
		return NUCLEUS34_OK;
	}
	const bool mtx = ext == ".mtx";
	if (!mtx && ext != ".edges" && ext != ".txt")
		return fail(NUCLEUS34_E_FORMAT, "Unknown dataset format: " + ext);

	// the text is mapped, not copied (a read into memory is the fallback)
	MappedText text;
	int rc = text.open(path);
	if (rc)
		return rc;
	const char *p = text.data, *end = text.data + text.size;

	// Skip leading comment lines: a line whose first character is '#' or '%'
	// (graph.hpp:307-314). The first other line is the header: parsed for
	// .mtx, consumed and discarded for bare edge lists (graph.hpp:318-359).
	const char *line = p;
	const char *header = nullptr, *header_end = nullptr;
	while (line < end)
	{
		const char *nl = static_cast<const char *>(std::memchr(line, '\n', size_t(end - line)));
		const char *le = nl ? nl : end;
		const char *next = nl ? nl + 1 : end;
		if (le == line || (*line != '#' && *line != '%'))
		{
			header = line;
			header_end = le;
			line = next;
			break;
		}
		line = next;
	}
	if (mtx)
	{
		if (!header)
			return fail(NUCLEUS34_E_FORMAT, "Wrong header for mtx format!");
		std::vector<unsigned long long> tok;
		std::string h(header, header_end);
		char *save = nullptr;
		for (char *t = strtok_r(h.data(), " \t\r", &save); t; t = strtok_r(nullptr, " \t\r", &save))
		{
			char *e2 = nullptr;
			errno = 0;
			unsigned long long v = std::strtoull(t, &e2, 0);
			if (e2 == t || errno)
				return fail(NUCLEUS34_E_FORMAT, "Wrong header for mtx format!");
			tok.push_back(v);
		}
		if (tok.size() != 2 && tok.size() != 3)
			return fail(NUCLEUS34_E_FORMAT, "Wrong header for mtx format!");
		unsigned long long nv = tok.size() == 2 ? tok[0] : std::max(tok[0], tok[1]);
		unsigned long long ne = tok.size() == 2 ? tok[1] : tok[2];
		if (ne > 0xffffffffull)
			return fail(NUCLEUS34_E_RANGE32, "Edges size are larger than defined type.");
		if (nv > 0xffffffffull)
			return fail(NUCLEUS34_E_RANGE32, "Vertices id are larger than defined type.");
	}
	if (!header)
		line = end; // nothing but comments

	// parallel parse of the remaining lines
	const size_t body = size_t(end - line);
	const int nth = std::max(1, omp_get_max_threads());
	const int nchunks = body < (1u << 20) ? 1 : nth * 4;
	std::vector<const char *> cb(nchunks + 1);
	cb[0] = line;
	cb[nchunks] = end;
	for (int c = 1; c < nchunks; ++c)
	{
		const char *q = line + body * size_t(c) / size_t(nchunks);
		if (q < cb[c - 1])
			q = cb[c - 1];
		const char *nl = static_cast<const char *>(std::memchr(q, '\n', size_t(end - q)));
		cb[c] = nl ? nl + 1 : end;
	}
	// Each chunk parses into its own uninitialised buffers, sized for the
	// most pair lines it can hold (a pair line has at least 4 characters,
	// "1 2\n"). The two numbers are read in one pass from the line start
	// (parse_two_at stops at the first character that is neither a digit, a
	// space nor a tab, so the bound is the chunk end), then the rest of the
	// line is skipped.
	std::vector<std::unique_ptr<uint32_t[]>> ps(nchunks), pd(nchunks);
	std::vector<uint64_t> pn(nchunks, 0);
#pragma omp parallel for schedule(dynamic, 1)
	for (int c = 0; c < nchunks; ++c)
	{
		const char *q = cb[c], *qe = cb[c + 1];
		const size_t cap = size_t(qe - q) / 4 + 1;
		ps[c].reset(new uint32_t[cap]);
		pd[c].reset(new uint32_t[cap]);
		uint32_t *S = ps[c].get(), *Dd = pd[c].get();
		uint64_t k = 0;
		while (q < qe)
		{
			const char *stop = q;
			uint32_t s, d;
			if (parse_two_at(q, qe, s, d, stop))
			{
				S[k] = s;
				Dd[k] = d;
				++k;
			}
			const char *nl = static_cast<const char *>(std::memchr(stop, '\n', size_t(qe - stop)));
			q = nl ? nl + 1 : qe;
		}
		pn[c] = k;
	}
	// the parsed chunks go to the CSR build in file order, as they are
	std::vector<PairSlice> parts(static_cast<size_t>(nchunks));
	for (int c = 0; c < nchunks; ++c)
		parts[size_t(c)] = PairSlice{ps[c].get(), pd[c].get(), pn[c]};
	return build_oriented_slices(parts, g);
}

int save_grh(const nucleus34_graph *g, const char *path)
{
	FILE *f = std::fopen(path, "wb");
	if (!f)
		return fail(NUCLEUS34_E_IO, "Can't open file for serializing.");
	uint64_t hdr[3] = {sizeof(uint32_t), g->n, g->m};
	bool ok = std::fwrite(hdr, 8, 3, f) == 3 &&
			  (g->n == 0 || std::fwrite(g->D, 4, g->n, f) == g->n) &&
			  (g->m == 0 || std::fwrite(g->E, 4, g->m, f) == g->m);
	ok = (std::fclose(f) == 0) && ok;
	return ok ? NUCLEUS34_OK : fail(NUCLEUS34_E_IO, "short write");
}

} // namespace n34

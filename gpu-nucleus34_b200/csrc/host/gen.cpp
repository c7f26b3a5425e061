// Seeded synthetic graph generators (there are no datasets on this system):
// R-MAT, 2D random geometric graphs and Watts-Strogatz rings. Every random
// draw comes from a counter-based stream (splitmix64 keyed by the seed and an
// index), so the output does not depend on the number of host threads.
// Each generator returns the cleaned undirected list (u < v, unique, sorted).
#include "host_internal.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <omp.h>

namespace n34 {

namespace {

inline uint64_t mix64(uint64_t z)
{
	z += 0x9E3779B97F4A7C15ull;
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
	return z ^ (z >> 31);
}

struct Stream
{
	uint64_t s;
	Stream(uint64_t seed, uint64_t index) : s(mix64(seed ^ mix64(index ^ 0xD1B54A32D192ED03ull))) {}
	uint64_t next()
	{
		s += 0x9E3779B97F4A7C15ull;
		uint64_t z = s;
		z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
		z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
		return z ^ (z >> 31);
	}
	double uniform() { return double(next() >> 11) * 0x1.0p-53; }
	uint64_t below(uint64_t n) { return n ? next() % n : 0; }
};

// Parallel LSD radix sort of u64 keys, 8-bit digits, passes whose digit is
// constant over all keys are skipped.
void radix_sort(std::vector<uint64_t> &a)
{
	const size_t n = a.size();
	if (n < (1u << 16))
	{
		std::sort(a.begin(), a.end());
		return;
	}
	std::vector<uint64_t> tmp(n);
	uint64_t *src = a.data(), *dst = tmp.data();
	const int T = std::max(1, omp_get_max_threads());
	std::vector<size_t> hist(size_t(T) * 256);
	for (int pass = 0; pass < 8; ++pass)
	{
		const int sh = 8 * pass;
		std::fill(hist.begin(), hist.end(), 0);
#pragma omp parallel num_threads(T)
		{
			const int t = omp_get_thread_num();
			const size_t b = n * size_t(t) / size_t(T), e = n * size_t(t + 1) / size_t(T);
			size_t *h = hist.data() + size_t(t) * 256;
			for (size_t i = b; i < e; ++i)
				h[(src[i] >> sh) & 0xff]++;
		}
		bool trivial = false;
		for (int d = 0; d < 256 && !trivial; ++d)
		{
			size_t c = 0;
			for (int t = 0; t < T; ++t)
				c += hist[size_t(t) * 256 + d];
			trivial = c == n;
		}
		if (trivial)
			continue;
		size_t run = 0;
		for (int d = 0; d < 256; ++d)
			for (int t = 0; t < T; ++t)
			{
				size_t c = hist[size_t(t) * 256 + d];
				hist[size_t(t) * 256 + d] = run;
				run += c;
			}
#pragma omp parallel num_threads(T)
		{
			const int t = omp_get_thread_num();
			const size_t b = n * size_t(t) / size_t(T), e = n * size_t(t + 1) / size_t(T);
			size_t *h = hist.data() + size_t(t) * 256;
			for (size_t i = b; i < e; ++i)
				dst[h[(src[i] >> sh) & 0xff]++] = src[i];
		}
		std::swap(src, dst);
	}
	if (src != a.data())
		std::memcpy(a.data(), src, n * sizeof(uint64_t));
}

// keys (u<<32|v) with u != v -> canonical (min,max), sorted unique, exported.
int finish(std::vector<uint64_t> &keys, nucleus34_edges *out)
{
	size_t w = 0;
	for (size_t i = 0; i < keys.size(); ++i)
	{
		uint32_t u = uint32_t(keys[i] >> 32), v = uint32_t(keys[i]);
		if (u == v)
			continue;
		if (u > v)
			std::swap(u, v);
		keys[w++] = (uint64_t(u) << 32) | v;
	}
	keys.resize(w);
	radix_sort(keys);
	keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
	const uint64_t c = keys.size();
	out->count = c;
	out->src = static_cast<uint32_t *>(std::malloc((c ? c : 1) * sizeof(uint32_t)));
	out->dst = static_cast<uint32_t *>(std::malloc((c ? c : 1) * sizeof(uint32_t)));
	if (!out->src || !out->dst)
	{
		std::free(out->src);
		std::free(out->dst);
		out->src = out->dst = nullptr;
		out->count = 0;
		return fail(NUCLEUS34_E_INVALID, "host allocation failed");
	}
#pragma omp parallel for schedule(static)
	for (int64_t i = 0; i < int64_t(c); ++i)
	{
		out->src[i] = uint32_t(keys[i] >> 32);
		out->dst[i] = uint32_t(keys[i]);
	}
	return NUCLEUS34_OK;
}

} // namespace

uint64_t splitmix64(uint64_t x) { return mix64(x); }

int gen_rmat(uint32_t scale, uint32_t ef, double a, double b, double c, uint64_t seed, nucleus34_edges *out)
{
	if (!out || scale == 0 || scale > 31 || ef == 0 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0)
		return fail(NUCLEUS34_E_INVALID, "bad R-MAT parameters");
	const uint64_t m = uint64_t(ef) << scale;
	std::vector<uint64_t> keys(m);
	const double ab = a + b, abc = a + b + c;
#pragma omp parallel for schedule(static)
	for (int64_t i = 0; i < int64_t(m); ++i)
	{
		Stream st(seed, uint64_t(i));
		uint32_t u = 0, v = 0;
		for (uint32_t l = 0; l < scale; ++l)
		{
			const double r = st.uniform();
			uint32_t bu = 0, bv = 0;
			if (r < a)
			{
			}
			else if (r < ab)
				bv = 1;
			else if (r < abc)
				bu = 1;
			else
				bu = bv = 1;
			u = (u << 1) | bu;
			v = (v << 1) | bv;
		}
		keys[i] = (uint64_t(u) << 32) | v;
	}
	return finish(keys, out);
}

int gen_rgg(uint64_t n, double deg, uint64_t seed, nucleus34_edges *out)
{
	if (!out || n < 2 || n > 0xffffffffull || !(deg > 0))
		return fail(NUCLEUS34_E_INVALID, "bad RGG parameters");
	const double r = std::sqrt(deg / (M_PI * double(n)));
	const double r2 = r * r;
	std::vector<double> x(n), y(n);
#pragma omp parallel for schedule(static)
	for (int64_t i = 0; i < int64_t(n); ++i)
	{
		Stream st(seed, uint64_t(i));
		x[i] = st.uniform();
		y[i] = st.uniform();
	}
	const uint64_t G = std::max<uint64_t>(1, uint64_t(std::floor(1.0 / r)));
	auto cell_of = [&](uint64_t i) {
		uint64_t cx = std::min<uint64_t>(G - 1, uint64_t(x[i] * double(G)));
		uint64_t cy = std::min<uint64_t>(G - 1, uint64_t(y[i] * double(G)));
		return cy * G + cx;
	};
	std::vector<uint64_t> coff(G * G + 1, 0);
	std::vector<uint32_t> cid(n);
	for (uint64_t i = 0; i < n; ++i)
		coff[cell_of(i) + 1]++;
	for (uint64_t c = 0; c < G * G; ++c)
		coff[c + 1] += coff[c];
	{
		std::vector<uint64_t> cur(coff.begin(), coff.end() - 1);
		for (uint64_t i = 0; i < n; ++i)
			cid[cur[cell_of(i)]++] = uint32_t(i);
	}
	const int T = std::max(1, omp_get_max_threads());
	std::vector<std::vector<uint64_t>> local(T);
#pragma omp parallel num_threads(T)
	{
		auto &L = local[omp_get_thread_num()];
#pragma omp for schedule(dynamic, 64)
		for (int64_t c = 0; c < int64_t(G * G); ++c)
		{
			const int64_t cy = c / int64_t(G), cx = c % int64_t(G);
			for (uint64_t pi = coff[c]; pi < coff[c + 1]; ++pi)
			{
				const uint32_t i = cid[pi];
				for (int64_t dy = -1; dy <= 1; ++dy)
					for (int64_t dx = -1; dx <= 1; ++dx)
					{
						const int64_t ny = cy + dy, nx = cx + dx;
						if (ny < 0 || nx < 0 || ny >= int64_t(G) || nx >= int64_t(G))
							continue;
						const uint64_t nc = uint64_t(ny) * G + uint64_t(nx);
						for (uint64_t pj = coff[nc]; pj < coff[nc + 1]; ++pj)
						{
							const uint32_t j = cid[pj];
							if (j <= i)
								continue;
							const double ddx = x[i] - x[j], ddy = y[i] - y[j];
							if (ddx * ddx + ddy * ddy < r2)
								L.push_back((uint64_t(i) << 32) | j);
						}
					}
			}
		}
	}
	size_t total = 0;
	for (auto &L : local)
		total += L.size();
	std::vector<uint64_t> keys;
	keys.reserve(total);
	for (auto &L : local)
	{
		keys.insert(keys.end(), L.begin(), L.end());
		std::vector<uint64_t>().swap(L);
	}
	return finish(keys, out);
}

// Watts-Strogatz ring with rewiring, in the order of the standard algorithm:
// ring lattice with k/2 neighbours per side, then for each distance j and
// each node u in order, with probability beta replace (u, u+j) by (u, w) for a
// uniform w that is neither u nor already adjacent (skipped if u is full).
int gen_ws(uint64_t n, uint32_t k, double beta, uint64_t seed, nucleus34_edges *out)
{
	if (!out || n < 3 || n > 0xffffffffull || k < 2 || k >= n || beta < 0 || beta > 1)
		return fail(NUCLEUS34_E_INVALID, "bad Watts-Strogatz parameters");
	std::vector<std::vector<uint32_t>> adj(n);
	auto has = [&](uint32_t u, uint32_t v) {
		const auto &A = adj[u];
		return std::find(A.begin(), A.end(), v) != A.end();
	};
	auto add = [&](uint32_t u, uint32_t v) {
		adj[u].push_back(v);
		adj[v].push_back(u);
	};
	auto del = [&](uint32_t u, uint32_t v) {
		auto &A = adj[u];
		A.erase(std::find(A.begin(), A.end(), v));
		auto &B = adj[v];
		B.erase(std::find(B.begin(), B.end(), u));
	};
	const uint32_t half = k / 2;
	for (uint32_t j = 1; j <= half; ++j)
		for (uint64_t u = 0; u < n; ++u)
		{
			const uint32_t v = uint32_t((u + j) % n);
			if (!has(uint32_t(u), v))
				add(uint32_t(u), v);
		}
	Stream st(seed, 0);
	for (uint32_t j = 1; j <= half; ++j)
		for (uint64_t u = 0; u < n; ++u)
		{
			const uint32_t v = uint32_t((u + j) % n);
			if (st.uniform() >= beta)
				continue;
			uint32_t w = uint32_t(st.below(n));
			bool skip = false;
			while (w == u || has(uint32_t(u), w))
			{
				if (adj[u].size() >= n - 1)
				{
					skip = true;
					break;
				}
				w = uint32_t(st.below(n));
			}
			if (!skip && has(uint32_t(u), v))
			{
				del(uint32_t(u), v);
				add(uint32_t(u), w);
			}
		}
	std::vector<uint64_t> keys;
	for (uint64_t u = 0; u < n; ++u)
		for (uint32_t v : adj[u])
			if (u < v)
				keys.push_back((u << 32) | v);
	return finish(keys, out);
}

int write_edges(const nucleus34_edges *e, const char *path)
{
	FILE *f = std::fopen(path, "wb");
	if (!f)
		return fail(NUCLEUS34_E_IO, std::string("cannot write ") + path);
	const uint64_t c = e->count;
	bool ok = true;
	if (c)
		ok = std::fprintf(f, "%u %u\n", e->src[0], e->dst[0]) > 0;
	const uint64_t chunk = 1u << 20;
	std::vector<char> buf;
	for (uint64_t b = 0; b < c && ok; b += chunk)
	{
		const uint64_t end = std::min(c, b + chunk);
		buf.resize((end - b) * 23);
		size_t w = 0;
		for (uint64_t i = b; i < end; ++i)
			w += size_t(std::snprintf(buf.data() + w, 23, "%u %u\n", e->src[i], e->dst[i]));
		ok = std::fwrite(buf.data(), 1, w, f) == w;
	}
	ok = (std::fclose(f) == 0) && ok;
	return ok ? NUCLEUS34_OK : fail(NUCLEUS34_E_IO, "short write");
}

} // namespace n34

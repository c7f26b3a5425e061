// Tune tables: parsing, graph classes, the selection rule, the writer and the
// C-ABI lookup. Host only; no exception leaves the C-ABI function.
#include "tune.h"

#include "host_internal.h"

#include <unistd.h>

#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

namespace n34 {

nucleus34_tune tune_filled(const nucleus34_tune &t)
{
	nucleus34_tune r = t;
	if (!r.lane_max)
		r.lane_max = TUNE_LANE_MAX;
	if (!r.compact_div)
		r.compact_div = TUNE_COMPACT_DIV;
	if (!r.sort_shift)
		r.sort_shift = TUNE_SORT_SHIFT;
	if (!r.rounds_per_replay)
		r.rounds_per_replay = TUNE_ROUNDS;
	return r;
}

int tune_check(const nucleus34_tune &t)
{
	if (t.lane_max && t.lane_max != 8 && t.lane_max != 16 && t.lane_max != 32)
		return fail(NUCLEUS34_E_INVALID, "tune: lane_max must be 8, 16 or 32");
	if (t.compact_div != NUCLEUS34_TUNE_NEVER && t.compact_div > 64)
		return fail(NUCLEUS34_E_INVALID, "tune: compact_div must be 1..64 or never");
	if (t.sort_shift != NUCLEUS34_TUNE_NEVER && t.sort_shift > 31)
		return fail(NUCLEUS34_E_INVALID, "tune: sort_shift must be 1..31 or never");
	if (t.rounds_per_replay > 64)
		return fail(NUCLEUS34_E_INVALID, "tune: rounds_per_replay must be 1..64");
	return NUCLEUS34_OK;
}

void tune_class(uint64_t T, uint64_t n, uint64_t m, uint32_t max_out, int32_t &size, int32_t &skew)
{
	size = T > 1 ? 63 - __builtin_clzll(T) : 0;
	skew = 0;
	if (!m)
		return;
	const unsigned __int128 top = (unsigned __int128)max_out * n;
	while (skew < 64 && ((unsigned __int128)m << (skew + 1)) <= top)
		++skew;
}

namespace {

bool parse_u32(const std::string &v, uint32_t lo, uint32_t hi, bool never_ok, uint32_t &out)
{
	if (never_ok && v == "never")
	{
		out = NUCLEUS34_TUNE_NEVER;
		return true;
	}
	if (v.empty() || v.size() > 10 || v.find_first_not_of("0123456789") != std::string::npos)
		return false;
	const unsigned long long x = std::strtoull(v.c_str(), nullptr, 10);
	if (x < lo || x > hi)
		return false;
	out = uint32_t(x);
	return true;
}

bool parse_sec(const std::string &v, double &out)
{
	if (v.empty())
		return false;
	char *end = nullptr;
	errno = 0;
	const double x = std::strtod(v.c_str(), &end);
	if (errno || !end || *end || !(x >= 0) || x > 1e9)
		return false;
	out = x;
	return true;
}

// 0: nothing on the line; 1: a rule; an error code with the detail set.
int parse_line(const std::string &raw, const char *path, int lineno, TuneRule &r)
{
	std::string text = raw.substr(0, raw.find('#'));
	std::istringstream in(text);
	std::string tok;
	r = TuneRule{};
	r.line = lineno;
	bool any = false, have_size = false, have_skew = false;
	std::vector<std::string> seen;
	auto bad = [&](const std::string &why) {
		return fail(NUCLEUS34_E_INVALID,
					std::string("tune table ") + path + ":" + std::to_string(lineno) + ": " + why);
	};
	while (in >> tok)
	{
		any = true;
		const size_t eq = tok.find('=');
		if (eq == std::string::npos || eq == 0)
			return bad("expected key=value, got '" + tok + "'");
		const std::string k = tok.substr(0, eq), v = tok.substr(eq + 1);
		for (const auto &s : seen)
			if (s == k)
				return bad("'" + k + "' given twice");
		seen.push_back(k);
		uint32_t u = 0;
		bool ok;
		if (k == "size")
		{
			ok = have_size = parse_u32(v, 0, 64, false, u);
			r.size = int32_t(u);
		}
		else if (k == "skew")
		{
			ok = have_skew = parse_u32(v, 0, 64, false, u);
			r.skew = int32_t(u);
		}
		else if (k == "lane_max")
			ok = parse_u32(v, 8, 32, false, r.tune.lane_max) && (r.tune.lane_max & (r.tune.lane_max - 1)) == 0;
		else if (k == "compact_div")
			ok = parse_u32(v, 1, 64, true, r.tune.compact_div);
		else if (k == "sort_shift")
			ok = parse_u32(v, 1, 31, true, r.tune.sort_shift);
		else if (k == "rounds_per_replay")
			ok = parse_u32(v, 1, 64, false, r.tune.rounds_per_replay);
		else if (k == "sec")
			ok = parse_sec(v, r.sec);
		else if (k == "default_sec")
			ok = parse_sec(v, r.default_sec);
		else
			return bad("unknown key '" + k + "'");
		if (!ok)
			return bad("bad value for '" + k + "': '" + v + "'");
	}
	if (!any)
		return 0;
	if (!have_size || !have_skew)
		return bad("size= and skew= are required");
	return 1;
}

} // namespace

int tune_read(const char *path, std::vector<TuneRule> &rules)
{
	rules.clear();
	if (!path || !*path)
		return fail(NUCLEUS34_E_INVALID, "null tune table path");
	std::ifstream f(path);
	if (!f)
		return fail(NUCLEUS34_E_IO, std::string("cannot open tune table ") + path);
	std::string line;
	int lineno = 0;
	while (std::getline(f, line))
	{
		++lineno;
		TuneRule r;
		const int rc = parse_line(line, path, lineno, r);
		if (rc < 0)
			return rc;
		if (rc == 1)
			rules.push_back(r);
	}
	if (f.bad())
		return fail(NUCLEUS34_E_IO, std::string("error reading tune table ") + path);
	return NUCLEUS34_OK;
}

const TuneRule *tune_match(const std::vector<TuneRule> &rules, int32_t size, int32_t skew)
{
	const TuneRule *best = nullptr;
	int32_t best_d = 3;
	for (const auto &r : rules)
	{
		if (r.skew != skew)
			continue;
		const int32_t d = r.size > size ? r.size - size : size - r.size;
		if (d < best_d)
		{
			best = &r;
			best_d = d;
		}
	}
	return best;
}

std::string tune_line(const TuneRule &r)
{
	const nucleus34_tune t = tune_filled(r.tune);
	auto never_or = [](uint32_t v) { return v == NUCLEUS34_TUNE_NEVER ? std::string("never") : std::to_string(v); };
	char sec[64];
	std::snprintf(sec, sizeof sec, " sec=%.4f default_sec=%.4f", r.sec, r.default_sec);
	return "size=" + std::to_string(r.size) + " skew=" + std::to_string(r.skew) +
		   " lane_max=" + std::to_string(t.lane_max) + " compact_div=" + never_or(t.compact_div) +
		   " sort_shift=" + never_or(t.sort_shift) + " rounds_per_replay=" + std::to_string(t.rounds_per_replay) +
		   sec;
}

int tune_store(const char *path, const TuneRule &r)
{
	if (!path || !*path)
		return fail(NUCLEUS34_E_INVALID, "null tune table path");
	std::vector<std::string> keep;
	{
		std::ifstream f(path);
		if (f)
		{
			std::string line;
			int lineno = 0;
			while (std::getline(f, line))
			{
				++lineno;
				TuneRule old;
				const int rc = parse_line(line, path, lineno, old);
				if (rc < 0)
					return rc; // never overwrite a table that does not parse
				if (rc == 1 && old.size == r.size && old.skew == r.skew)
					continue;
				keep.push_back(line);
			}
		}
		else
			keep.push_back("# nucleus34 tune table: size = floor(log2 T), skew = floor(log2(max out-degree * n / m))");
	}
	keep.push_back(tune_line(r));
	const std::string tmp = std::string(path) + ".tmp." + std::to_string(long(::getpid()));
	{
		std::ofstream o(tmp, std::ios::trunc);
		if (!o)
			return fail(NUCLEUS34_E_IO, "cannot write " + tmp);
		for (const auto &l : keep)
			o << l << '\n';
		o.flush();
		if (!o)
		{
			std::remove(tmp.c_str());
			return fail(NUCLEUS34_E_IO, "short write to " + tmp);
		}
	}
	if (std::rename(tmp.c_str(), path) != 0)
	{
		std::remove(tmp.c_str());
		return fail(NUCLEUS34_E_IO, std::string("cannot replace ") + path);
	}
	return NUCLEUS34_OK;
}

} // namespace n34

using namespace n34;

extern "C" int nucleus34_tune_lookup(const char *path, uint64_t triangles, uint64_t n, uint64_t m, uint32_t max_out,
									 nucleus34_tune *out, int *matched)
{
	clear_error();
	if (!out)
		return fail(NUCLEUS34_E_INVALID, "null output");
	try
	{
		std::vector<TuneRule> rules;
		const int rc = tune_read(path, rules);
		if (rc)
			return rc;
		int32_t size = 0, skew = 0;
		tune_class(triangles, n, m, max_out, size, skew);
		const TuneRule *r = tune_match(rules, size, skew);
		*out = tune_filled(r ? r->tune : nucleus34_tune{});
		if (matched)
			*matched = r ? 1 : 0;
		return NUCLEUS34_OK;
	}
	catch (const std::exception &e)
	{
		return fail(NUCLEUS34_E_INVALID, e.what());
	}
}

extern "C" int nucleus34_tune_store(const char *path, uint64_t triangles, uint64_t n, uint64_t m, uint32_t max_out,
									const nucleus34_tune *tune, double sec, double default_sec)
{
	clear_error();
	if (!tune)
		return fail(NUCLEUS34_E_INVALID, "null settings");
	if (!(sec >= 0) || !(default_sec >= 0) || sec > 1e9 || default_sec > 1e9)
		return fail(NUCLEUS34_E_INVALID, "times must be in [0, 1e9] s");
	try
	{
		const int rc = tune_check(*tune);
		if (rc)
			return rc;
		TuneRule r;
		tune_class(triangles, n, m, max_out, r.size, r.skew);
		r.tune = tune_filled(*tune);
		r.sec = sec;
		r.default_sec = default_sec;
		return tune_store(path, r);
	}
	catch (const std::exception &e)
	{
		return fail(NUCLEUS34_E_INVALID, e.what());
	}
}

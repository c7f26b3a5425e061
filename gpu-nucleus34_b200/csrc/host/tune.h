// Tune tables of the on-demand variant: graph classes, line parsing, the
// selection rule and the table writer (host code, shared by the device-side
// context). Every setting gives identical results; the table only picks the
// fastest schedule per graph class.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "nucleus34.h"

namespace n34 {

// Built-in defaults (the values the kernels were tuned with on R-MAT scale 20).
constexpr uint32_t TUNE_LANE_MAX = 16;
constexpr uint32_t TUNE_COMPACT_DIV = 8;
constexpr uint32_t TUNE_SORT_SHIFT = 12;
constexpr uint32_t TUNE_ROUNDS = 16;

struct TuneRule
{
	int32_t size = 0; // floor(log2 T)
	int32_t skew = 0; // floor(log2(max out-degree * n / m))
	nucleus34_tune tune{};
	double sec = 0, default_sec = 0; // autotuner timings (informative)
	int line = 0;                     // line number in its file
};

// Zero fields replaced by the defaults.
nucleus34_tune tune_filled(const nucleus34_tune &t);
// NUCLEUS34_OK, or E_INVALID (with a detail) for a value out of range.
int tune_check(const nucleus34_tune &t);
// Class of a graph: size = floor(log2 T) (0 for T <= 1), skew = the largest
// w with m * 2^w <= max_out * n (0 when m = 0), both exact in integers.
void tune_class(uint64_t T, uint64_t n, uint64_t m, uint32_t max_out, int32_t &size, int32_t &skew);
// Reads and checks a whole table. E_IO: unreadable; E_INVALID: malformed.
int tune_read(const char *path, std::vector<TuneRule> &rules);
// The rule of the same skew class with the nearest size (at most 2 away;
// ties to the earlier line), or null.
const TuneRule *tune_match(const std::vector<TuneRule> &rules, int32_t size, int32_t skew);
// One table line for r (no newline).
std::string tune_line(const TuneRule &r);
// Replaces the line of r's class in the table at path (or appends it; the
// file is created when missing), through a temporary file and a rename.
int tune_store(const char *path, const TuneRule &r);

} // namespace n34

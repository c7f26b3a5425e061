// Internal declarations shared by the host-side sources of libnucleus34.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "nucleus34.h"

namespace n34 {

struct HostGraph
{
	uint64_t n = 0;
	uint64_t m = 0;
	std::vector<uint32_t> O; // n+1
	std::vector<uint32_t> D; // n
	std::vector<uint32_t> E; // m
};

// Records a thread-local detail message and returns code.
int fail(int code, const std::string &msg);
void clear_error();

int build_oriented(const uint32_t *src, const uint32_t *dst, uint64_t count, HostGraph &out);
int load_graph(const char *path, HostGraph &g);
int save_grh(const nucleus34_graph *g, const char *path);

// Moves a HostGraph into a malloc-owned C struct.
int export_graph(HostGraph &&hg, nucleus34_graph *g);

} // namespace n34

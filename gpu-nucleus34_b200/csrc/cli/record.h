// Shared front-end pieces of the two drop-in programs: the JSON result record
// in the reference's exact layout (nucleus/utility/json.h:9-92), the
// environment object (cuNucleus34.cu:197-226, utility/cpuinfo.hpp:43-160), the
// "[phase]" progress lines (utility/defs.hpp:71) and helpers.
#pragma once

#include <cuda_runtime_api.h>

#include <sched.h>
#include <unistd.h>

#include <algorithm>
#include <cctype>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include <omp.h>

#include "nucleus34.h"

namespace rec {

constexpr size_t PRINT_CAP = 5; // utility/defs.hpp:25

inline std::string escape(const std::string &s)
{
	std::string out;
	out += '"';
	for (unsigned char c : s)
	{
		switch (c)
		{
		case '"':
			out += "\\\"";
			break;
		case '\\':
			out += "\\\\";
			break;
		case '\b':
			out += "\\b";
			break;
		case '\f':
			out += "\\f";
			break;
		case '\n':
			out += "\\n";
			break;
		case '\r':
			out += "\\r";
			break;
		case '\t':
			out += "\\t";
			break;
		default:
			if (c < 0x20)
			{
				char buf[7];
				std::snprintf(buf, sizeof(buf), "\\u%04x", c);
				out += buf;
			}
			else
				out += char(c);
		}
	}
	out += '"';
	return out;
}

// The record is built in a string stream exactly like g_jsonSS and printed once.
struct Json
{
	std::ostringstream ss;
	void field(bool first, const std::string &k, const std::string &v)
	{
		ss << (first ? "{" : ",") << "\n\t\t\"" << k << "\": " << escape(v);
	}
	void field(bool first, const std::string &k, const char *v) { field(first, k, std::string(v ? v : "")); }
	template <class T>
	void field(bool first, const std::string &k, const T &v)
	{
		ss << (first ? "{" : ",") << "\n\t\t\"" << k << "\": " << v;
	}
	void raw(bool first, const std::string &k, const std::string &v)
	{
		ss << (first ? "{" : ",") << "\n\t\t\"" << k << "\": " << v;
	}
	template <class It, class Fmt>
	void array(bool first, const std::string &k, It b, It e, Fmt fmt)
	{
		ss << (first ? "{" : ",") << "\n\t\t\"" << k << "\": [";
		bool fe = true;
		for (auto it = b; it != e; ++it)
		{
			if (!fe)
				ss << ", ";
			fmt(ss, *it);
			fe = false;
		}
		ss << "]";
	}
	void begin(bool first, const std::string &k) { ss << (first ? "{" : ",") << "\n\t\"" << k << "\":"; }
	void end() { ss << "\n\t}"; }
	void last() { ss << "\n}"; }
	void print() { std::cout << ss.str() << std::endl; }
};

inline void phase(std::string &step, const char *s)
{
	step = s;
	std::cerr << "[phase] " << step << std::endl;
}

inline std::string strip_path(const std::string &f) { return f.substr(f.find_last_of("/\\") + 1); }

inline std::string env(const char *e)
{
	const char *v = std::getenv(e);
	return v ? std::string(v) : std::string();
}

inline std::string hostname()
{
	char h[256] = {0};
	if (gethostname(h, sizeof(h) - 1))
		return "";
	return h;
}

inline std::vector<std::map<std::string, std::string>> cpuinfo()
{
	auto trim = [](std::string s) {
		s.erase(s.begin(), std::find_if(s.begin(), s.end(), [](int ch) { return !std::isspace(ch); }));
		s.erase(std::find_if(s.rbegin(), s.rend(), [](int ch) { return !std::isspace(ch); }).base(), s.end());
		return s;
	};
	std::vector<std::map<std::string, std::string>> cpus;
	std::map<std::string, std::string> inf;
	std::ifstream f("/proc/cpuinfo");
	std::string line;
	while (std::getline(f, line))
	{
		auto pos = line.find(':');
		if (pos == std::string::npos)
		{
			if (!inf.empty())
			{
				cpus.push_back(inf);
				inf.clear();
			}
			continue;
		}
		inf[trim(line.substr(0, pos))] = trim(line.substr(pos + 1));
	}
	if (!inf.empty())
		cpus.push_back(inf);
	return cpus;
}

inline std::string cpu_affinity()
{
	cpu_set_t set;
	if (sched_getaffinity(0, sizeof(set), &set))
		return "";
	std::string a;
	int first = -1, last = -1;
	auto flush = [&] {
		if (first > -1)
		{
			a += (a.empty() ? "" : "-") + std::to_string(first);
			if (last > -1)
				a += ":" + std::to_string(last);
		}
		first = last = -1;
	};
	for (int c = 0; c < CPU_SETSIZE; ++c)
	{
		if (CPU_ISSET(c, &set))
		{
			if (first < 0)
				first = c;
			else
				last = c;
		}
		else
			flush();
	}
	flush();
	return a;
}

// GPU properties under the same keys as gpuinfo() (cpuinfo.hpp:43-86), in
// std::map (sorted) order, one block per visible device.
inline std::vector<std::map<std::string, std::string>> gpuinfo()
{
	std::vector<std::map<std::string, std::string>> out;
	int count = 0;
	if (cudaGetDeviceCount(&count) != cudaSuccess)
	{
		cudaGetLastError();
		return out;
	}
	for (int i = 0; i < count; ++i)
	{
		cudaDeviceProp p{};
		if (cudaGetDeviceProperties(&p, i) != cudaSuccess)
			continue;
		std::map<std::string, std::string> inf;
		int clk = 0;
		cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, i);
		inf["Name"] = p.name;
		inf["Compute capability"] = std::to_string(p.major) + "." + std::to_string(p.minor);
		inf["Clock rate"] = std::to_string(clk);
		inf["Device copy overlap"] = p.asyncEngineCount > 0 ? "Enabled" : "Disabled";
		inf["Kernel execution timeout"] = "N/A";
		inf["Total global mem"] = std::to_string(p.totalGlobalMem);
		inf["Total constant Mem"] = std::to_string(p.totalConstMem);
		inf["Max mem pitch"] = std::to_string(p.memPitch);
		inf["Texture Alignment"] = std::to_string(p.textureAlignment);
		inf["Multiprocessor count"] = std::to_string(p.multiProcessorCount);
		inf["Shared mem per mp"] = std::to_string(p.sharedMemPerBlock);
		inf["Registers per mp"] = std::to_string(p.regsPerBlock);
		inf["Threads in warp"] = std::to_string(p.warpSize);
		inf["Max threads per block"] = std::to_string(p.maxThreadsPerBlock);
		inf["Max thread dimensions"] = std::to_string(p.maxThreadsDim[0]) + "x" + std::to_string(p.maxThreadsDim[1]) +
									   "x" + std::to_string(p.maxThreadsDim[2]);
		inf["Max grid dimensions"] = std::to_string(p.maxGridSize[0]) + "x" + std::to_string(p.maxGridSize[1]) + "x" +
									 std::to_string(p.maxGridSize[2]);
		out.push_back(inf);
	}
	return out;
}

inline std::string gxx_version()
{
	return std::to_string(__GNUC__) + "." + std::to_string(__GNUC_MINOR__) + "-" + std::to_string(__GNUC_PATCHLEVEL__);
}

// common environment object; `direct` adds the direct program's extra keys
inline void environment(Json &j, const char *app, const char *ver, bool direct, size_t parts)
{
	auto cpus = cpuinfo();
	auto gpus = gpuinfo();
	j.begin(true, "environment");
	j.field(true, "app", app);
	j.field(false, "version", ver);
	j.field(false, "g++", gxx_version());
	j.field(false, "cuda", CUDART_VERSION); // compile-time toolkit version, as the reference reports it
	if (direct)
	{
		j.field(false, "parts", parts);
		j.field(false, "slurm_requested_gpus", env("SLURM_GPUS"));
		j.field(false, "slurm_available_gpus", env("SLURM_VISIBLE_DEVICES"));
		j.field(false, "slurm_job_gpus", env("SLURM_JOB_GPUS"));
		j.field(false, "peer_gpu_count", size_t(0));
	}
	j.field(false, "thrust", "unused");
	j.field(false, "policy", "omp");
	j.field(false, "procs", omp_get_num_procs());
	j.field(false, "cpu_core_count", cpus.size());
	if (direct)
		j.field(false, "cpu_affinity", cpu_affinity());
	j.field(false, "cpu_model", cpus.size() ? cpus[0]["model name"] : std::string("Unknown"));
	if (direct)
		j.field(false, "cpu_physical_cores", cpus.size() ? cpus[0]["cpu cores"] : std::string("Unknown"));
	for (const auto &g : gpus)
		for (const auto &kv : g)
		{
			std::string key = "gpu_" + kv.first;
			std::replace(key.begin(), key.end(), ' ', '_');
			j.field(false, key, kv.second);
		}
	j.field(false, "host", hostname());
	j.end();
}

// "[mem] <tag> <detail> | gpu_free=<free>/<total> MiB" on stderr: the
// reference's memory milestone line (cuNucleus34.cu:72-79,
// cuNucleus34_ondemand.cu:556-562, 585-588).
inline void mem_note(const char *tag, const std::string &detail)
{
	size_t fb = 0, tb = 0;
	if (cudaMemGetInfo(&fb, &tb) != cudaSuccess)
	{
		cudaGetLastError();
		fb = tb = 0;
	}
	std::cerr << "[mem] " << tag << ' ' << detail << " | gpu_free=" << (fb >> 20) << "/" << (tb >> 20) << " MiB"
			  << std::endl;
}

inline std::string secs1(double v)
{
	std::ostringstream os;
	os << std::fixed << std::setprecision(1) << v << "s";
	return os.str();
}

inline std::string fixed2(double v)
{
	std::ostringstream os;
	os << std::fixed << std::setprecision(2) << v;
	return os.str();
}

inline void print_tri(std::ostream &os, const uint32_t *t)
{
	os << "\"(" << t[0] << "," << t[1] << "," << t[2] << ")\"";
}

inline void print_qud(std::ostream &os, const uint32_t *q)
{
	os << "\"(" << q[0] << "," << q[1] << "," << q[2] << "," << q[3] << ")\"";
}

struct Error
{
	int code;
	std::string msg;
};

// The record's "error" is the exception text the reference would print
// (e.what(), cuNucleus34_ondemand.cu:762-778): the library's detail message,
// which repeats the reference's texts for reader errors ("Dataset <f> is not
// accessible!", "Unknown dataset format: <ext>", ...); the call and status
// name only when there is no detail.
inline void check(int rc, const char *what)
{
	if (rc == NUCLEUS34_OK)
		return;
	const std::string detail = nucleus34_last_error();
	throw Error{rc, detail.empty() ? std::string(what) + ": " + nucleus34_strerror(rc) : detail};
}

} // namespace rec

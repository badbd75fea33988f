// Library-wide C-ABI helpers: per-thread last-error text and the version string.
#include <cstdio>
#include <cstring>

#include "awcm_b200.h"
#include "awcm_common.cuh"

namespace awcm {

static thread_local char g_last_error[512] = "";

void set_last_error(const char* msg, const char* file, int line)
{
    const char* base = std::strrchr(file, '/');
    std::snprintf(g_last_error, sizeof(g_last_error), "%s (%s:%d)", msg, base ? base + 1 : file, line);
}

}  // namespace awcm

extern "C" {

const char* awcm_last_error(void) { return awcm::g_last_error; }

const char* awcm_version(void) { return "awcm-b200 0.1 (sm_100a, fp64)"; }

}  // extern "C"

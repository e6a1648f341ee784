// Internal declarations shared by the host-side sources (no CUDA).
#pragma once

#include <string>

#include "rrg.h"

namespace rrg {

// Records the calling thread's last error message (read by rrg_last_error(NULL)).
void set_thread_error(const std::string& msg);
const char* io_error();

// Fills a grid description from params.json values the way io_json.cpp:28-40 does.
void grid_from_values(int nx, double dx, double bc_frac, rrg_grid_info* g);

}  // namespace rrg

// gfb_internal.h -- helpers shared between the translation units of libgfb.
#pragma once

#include <vector>

#include "../../include/gfb.h"

namespace gfb {

// Record `msg` as this thread's gfb_last_error() and return `st`.
gfb_status set_error(gfb_status st, const char* msg);

// GLL weights and derivative matrix for ngll points per axis.
bool gll_tables_for(int ngll, std::vector<double>& w, std::vector<double>& D);

}  // namespace gfb

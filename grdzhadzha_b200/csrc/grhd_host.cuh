// grhd_host.cuh -- host helpers of the C ABI shared between its files.
#pragma once

#include "grhd_b200.h"
#include "grhd_kernels.cuh"

namespace grhd {
namespace host {
Options options_of(const grhd_params &p);
Background background_of(const grhd_params &p, double t);
BoxDev box_of(const grhd_box *b, int64_t state_cs);
bool box_valid(const grhd_box *b);
bool box_whole_domain(const grhd_box *b);
} // namespace host
} // namespace grhd

// gs_host.h — host helpers shared by the C ABI implementation.
#pragma once
#include <string>

#include "gs_internal.h"

namespace gs {
// Validate and copy a caller descriptor; empty string on success, else the reason.
std::string CopyGrid(const gs_grid_desc* d, HostGrid& g);
void FillInfo(const HostGrid& g, const Symbolic& s, gs_grid_info* info);
}  // namespace gs

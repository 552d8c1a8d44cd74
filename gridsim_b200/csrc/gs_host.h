// gs_host.h — host helpers shared by the C ABI implementation.
#pragma once
#include <string>

#include "gs_internal.h"

namespace gs {
// Validate and copy a caller descriptor; empty string on success, else the reason.
std::string CopyGrid(const gs_grid_desc* d, HostGrid& g);
void FillInfo(const HostGrid& g, const Symbolic& s, gs_grid_info* info);
// Topology verdicts of single-branch outages (-1 = the intact grid): splits[k] when removing idx[k] leaves more
// connected parts, unsolvable[k] when the grid without it has a part no Newton solve can converge (gs_topology.cpp).
// Either output may be null; empty string on success.
std::string OutageTopology(const HostGrid& h, double tol, int nOut, const int* idx, uint8_t* splits,
                           uint8_t* unsolvable);
// The same verdicts for one multi-branch outage (every branch in `removed` out at once).
std::string OutageSetTopology(const HostGrid& h, double tol, const std::vector<int>& removed, bool& splits,
                              bool& unsolvable);
}  // namespace gs

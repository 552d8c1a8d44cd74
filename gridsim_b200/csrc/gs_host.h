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
// An element outage for the topology verdicts: branches out, a unit out (-1 none), a bus out (-1 none; its branches
// listed too), and the reference moved from one bus to another (-1 none) when the outage took its last unit.
struct ElementCut {
    std::vector<int> branches;
    int gen = -1, bus = -1, slackFrom = -1, slackTo = -1;
};
// The same verdicts for one element outage (several branches, a unit, a bus).
std::string ElementTopology(const HostGrid& h, double tol, const ElementCut& e, bool& splits, bool& unsolvable);
}  // namespace gs

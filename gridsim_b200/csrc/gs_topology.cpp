// gs_topology.cpp — the host topology pass of the contingency screen.
//
// For every single-branch outage of a screen it answers two questions without solving anything:
//   * does the outage split the network into more connected parts than the grid has
//     (ContingencyAnalysis.Splits / ConnectedParts, Analysis/ContingencyAnalysis.cs:1665-1687)?
//   * does the grid without the branch hold a connected part that ProvablyUnsolvablePart (:1750-1830) proves no
//     Newton solve can bring to convergence (no reference bus, and a real-power balance no state can meet)?
// The screen reports the second kind at once (ScreenStateCore :1118-1127) and sends only the rest to the device.
//
// The reference rebuilds the reduced model and runs a union-find over it per outage. Here one iterative depth-first
// pass over the in-service branches gives every bridge (a branch whose removal splits its part, found by low-link
// values over branch ids, so parallel branches are never bridges) and, in preorder, prefix sums of the per-part
// facts the proof reads (reference buses, lossy and negative-loss elements). A bridge's child subtree is one side of
// the split and its preorder range, so each outage costs O(1) for those facts. The net injection of a side with no
// reference bus is summed over its buses in model order, as the reference sums it, so the verdict rounds the same
// way.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <unordered_set>
#include <vector>

#include "gs_host.h"

namespace gs {

namespace {

// Margin of the proof (ContingencyAnalysis.UnsolvableMarginPu, :1700-1705).
constexpr double kUnsolvableMarginPu = 1e-6;

struct Dfs {
    std::vector<int> pre, size, low, parentEdge, comp, ord;
};

// Iterative depth-first search over the in-service branches, roots in bus order.
Dfs Search(const HostGrid& h, const std::vector<int>& adjPtr, const std::vector<int>& adj) {
    const int n = h.n;
    Dfs d;
    d.pre.assign(n, -1);
    d.size.assign(n, 1);
    d.low.assign(n, 0);
    d.parentEdge.assign(n, -1);
    d.comp.assign(n, -1);
    d.ord.reserve(n);
    std::vector<int> stack, cursor(n, 0);
    for (int r = 0; r < n; r++) {
        if (d.pre[r] >= 0) continue;
        d.pre[r] = d.low[r] = (int)d.ord.size();
        d.ord.push_back(r);
        d.comp[r] = r;
        stack.push_back(r);
        cursor[r] = adjPtr[r];
        while (!stack.empty()) {
            const int v = stack.back();
            if (cursor[v] < adjPtr[v + 1]) {
                const int e = adj[cursor[v]++];
                if (e == d.parentEdge[v]) continue;
                const int w = h.brF[e] == v ? h.brT[e] : h.brF[e];
                if (d.pre[w] < 0) {
                    d.pre[w] = d.low[w] = (int)d.ord.size();
                    d.ord.push_back(w);
                    d.parentEdge[w] = e;
                    d.comp[w] = r;
                    cursor[w] = adjPtr[w];
                    stack.push_back(w);
                } else {
                    d.low[v] = std::min(d.low[v], d.pre[w]);
                }
            } else {
                stack.pop_back();
                if (d.parentEdge[v] >= 0) {
                    const int e = d.parentEdge[v];
                    const int u = h.brF[e] == v ? h.brT[e] : h.brF[e];
                    d.low[u] = std::min(d.low[u], d.low[v]);
                    d.size[u] += d.size[v];
                }
            }
        }
    }
    return d;
}

}  // namespace

std::string OutageTopology(const HostGrid& h, double tol, int nOut, const int* idx, uint8_t* splits,
                           uint8_t* unsolvable) {
    const int n = h.n, nb = h.nbr;
    for (int k = 0; k < nOut; k++)
        if (idx[k] < -1 || idx[k] >= nb) return "outage index out of range";
    std::vector<int> adjPtr(n + 1, 0), adj;
    for (int e = 0; e < nb; e++)
        if (h.brOn[e]) { adjPtr[h.brF[e] + 1]++; adjPtr[h.brT[e] + 1]++; }
    for (int i = 0; i < n; i++) adjPtr[i + 1] += adjPtr[i];
    adj.resize(adjPtr[n]);
    {
        std::vector<int> fill(adjPtr.begin(), adjPtr.end() - 1);
        for (int e = 0; e < nb; e++)
            if (h.brOn[e]) { adj[fill[h.brF[e]]++] = e; adj[fill[h.brT[e]]++] = e; }
    }
    const Dfs d = Search(h, adjPtr, adj);
    // the child end of each bridge (-1: not a bridge or not in service)
    std::vector<int> bridgeChild(nb, -1);
    for (int v = 0; v < n; v++) {
        const int e = d.parentEdge[v];
        if (e < 0) continue;
        const int u = h.brF[e] == v ? h.brT[e] : h.brF[e];
        if (d.low[v] > d.pre[u]) bridgeChild[e] = v;
    }
    if (splits)
        for (int k = 0; k < nOut; k++) splits[k] = idx[k] >= 0 && bridgeChild[idx[k]] >= 0;
    if (!unsolvable) return "";
    std::fill(unsolvable, unsolvable + nOut, 0);

    // The cases in which the reference gives no proof for any outage (:1752-1790).
    if (!(tol > 0.0) || !std::isfinite(tol)) return "";
    {
        std::unordered_set<int> ids;
        for (int i = 0; i < n; i++)
            if (!ids.insert(h.busId[i]).second) return "";  // a duplicate bus id is the engine's to refuse
    }
    std::vector<double> pgBus(n, 0.0);
    for (int g = 0; g < h.ngen; g++)
        if (h.genOn[g]) pgBus[h.genBus[g]] += h.pg[g];  // in generator order, as the reference sums
    for (int i = 0; i < n; i++)
        if (!std::isfinite(h.gsh[i]) || !std::isfinite(h.pd[i]) || !std::isfinite(pgBus[i])) return "";
    int badR = 0;
    for (int e = 0; e < nb; e++)
        if (h.brOn[e] && !std::isfinite(h.r[e])) badR++;

    // Per-vertex facts in preorder; a branch counts at its end discovered later (inside every subtree that holds
    // both ends).
    std::vector<int> slackAt(n, 0), lossyAt(n, 0), negAt(n, 0);
    for (int i = 0; i < n; i++) {
        slackAt[d.pre[i]] += h.busType[i] == 3;
        lossyAt[d.pre[i]] += h.gsh[i] != 0.0;
        negAt[d.pre[i]] += h.gsh[i] < 0.0;
    }
    for (int e = 0; e < nb; e++) {
        if (!h.brOn[e]) continue;
        const int p = std::max(d.pre[h.brF[e]], d.pre[h.brT[e]]);
        lossyAt[p] += h.r[e] != 0.0;
        negAt[p] += h.r[e] < 0.0;
    }
    std::vector<int> slackSum(n + 1, 0), lossySum(n + 1, 0), negSum(n + 1, 0);
    for (int p = 0; p < n; p++) {
        slackSum[p + 1] = slackSum[p] + slackAt[p];
        lossySum[p + 1] = lossySum[p] + lossyAt[p];
        negSum[p + 1] = negSum[p] + negAt[p];
    }
    auto range = [](const std::vector<int>& s, int a, int len) { return s[a + len] - s[a]; };
    auto netOf = [&](std::vector<int>& buses) {  // (sum Pg - Pd) / base over the buses, in model order
        std::sort(buses.begin(), buses.end());
        double net = 0.0;
        for (int i : buses) net += (pgBus[i] - h.pd[i]) / h.base;
        return net;
    };
    auto verdict = [&](int count, int slack, int lossy, int neg, double net) {
        if (slack > 0 || neg > 0) return false;
        const double margin = count * tol + kUnsolvableMarginPu;
        if (net <= -margin) return true;                          // a load part: its losses cannot be negative
        return lossy == 0 && std::fabs(net) >= margin;            // a lossless part that cannot balance
    };
    // the intact grid's parts, their facts and nets (summed in bus order per part)
    std::vector<double> compNet(n, 0.0);
    for (int i = 0; i < n; i++) compNet[d.comp[i]] += (pgBus[i] - h.pd[i]) / h.base;
    std::vector<uint8_t> compBad(n, 0);
    int nBad = 0;
    for (int r = 0; r < n; r++) {
        if (d.comp[r] != r) continue;
        const int a = d.pre[r], len = d.size[r];
        compBad[r] = verdict(len, range(slackSum, a, len), range(lossySum, a, len), range(negSum, a, len), compNet[r]);
        nBad += compBad[r];
    }
    for (int k = 0; k < nOut; k++) {
        const int e = idx[k];
        if (badR - (e >= 0 && h.brOn[e] && !std::isfinite(h.r[e])) > 0) continue;  // no proof (:1806)
        if (e < 0 || !h.brOn[e]) { unsolvable[k] = nBad > 0; continue; }
        const int c = d.comp[h.brF[e]];
        const int a = d.pre[c], len = d.size[c];
        const int lossyE = h.r[e] != 0.0, negE = h.r[e] < 0.0;
        int bad = nBad - compBad[c];
        const int v = bridgeChild[e];
        if (v < 0) {  // the part stays whole, less one branch
            bad += verdict(len, range(slackSum, a, len), range(lossySum, a, len) - lossyE, range(negSum, a, len) - negE,
                           compNet[c]);
        } else {      // the part splits into the subtree of v and the rest
            const int sa = d.pre[v], sl = d.size[v];
            const int subSlack = range(slackSum, sa, sl);
            const int subLossy = range(lossySum, sa, sl) - lossyE, subNeg = range(negSum, sa, sl) - negE;
            const int restSlack = range(slackSum, a, len) - subSlack;
            const int restLossy = range(lossySum, a, len) - range(lossySum, sa, sl);
            const int restNeg = range(negSum, a, len) - range(negSum, sa, sl);
            if (subSlack == 0 && subNeg == 0) {
                std::vector<int> buses(d.ord.begin() + sa, d.ord.begin() + sa + sl);
                bad += verdict(sl, 0, subLossy, 0, netOf(buses));
            }
            if (restSlack == 0 && restNeg == 0) {
                std::vector<int> buses;
                buses.reserve(len - sl);
                for (int p = a; p < a + len; p++)
                    if (p < sa || p >= sa + sl) buses.push_back(d.ord[p]);
                bad += verdict(len - sl, 0, restLossy, 0, netOf(buses));
            }
        }
        unsolvable[k] = bad > 0;
    }
    return "";
}

// The same two verdicts for an element outage (ScreenElementOutage, :1355-1437): the grid without the branches
// e.branches, without unit e.gen (its output lost), without bus e.bus (its branches are among e.branches), and with
// the reference moved from e.slackFrom to e.slackTo where the outage took the reference's last unit (ReelectReference
// :1440-1488). One union-find over the remaining in-service branches: O(buses + branches) per outage.
std::string ElementTopology(const HostGrid& h, double tol, const ElementCut& e, bool& splits, bool& unsolvable) {
    const int n = h.n, nb = h.nbr;
    splits = unsolvable = false;
    std::vector<uint8_t> gone(nb, 0);
    for (int k : e.branches) {
        if (k < 0 || k >= nb) return "outage index out of range";
        gone[k] = 1;
    }
    if (e.bus >= n || e.gen >= h.ngen) return "outage index out of range";
    std::vector<int> parent(n), partsAt(2, n);
    auto find = [&](int x) { while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; } return x; };
    partsAt[1] = n - (e.bus >= 0 ? 1 : 0);  // a removed bus is not a part of the reduced model
    for (int pass = 0; pass < 2; pass++) {  // 0: the intact grid, 1: the reduced one
        for (int i = 0; i < n; i++) parent[i] = i;
        for (int k = 0; k < nb; k++) {
            if (!h.brOn[k] || (pass == 1 && gone[k])) continue;
            const int a = find(h.brF[k]), c = find(h.brT[k]);
            if (a != c) { parent[a] = c; partsAt[pass]--; }
        }
    }
    splits = partsAt[1] > partsAt[0];
    // ProvablyUnsolvablePart of the reduced grid (parent holds its parts)
    if (!(tol > 0.0) || !std::isfinite(tol)) return "";
    {
        std::unordered_set<int> ids;
        for (int i = 0; i < n; i++)
            if (i != e.bus && !ids.insert(h.busId[i]).second) return "";
    }
    std::vector<double> pgBus(n, 0.0);
    for (int g = 0; g < h.ngen; g++)
        if (h.genOn[g] && g != e.gen && h.genBus[g] != e.bus) pgBus[h.genBus[g]] += h.pg[g];
    std::vector<int> count(n, 0), slack(n, 0), lossy(n, 0), neg(n, 0);
    std::vector<double> net(n, 0.0);
    for (int i = 0; i < n; i++) {
        if (i == e.bus) continue;
        if (!std::isfinite(h.gsh[i]) || !std::isfinite(h.pd[i]) || !std::isfinite(pgBus[i])) return "";
        const int r = find(i);
        const bool isSlack = (h.busType[i] == 3 && i != e.slackFrom) || i == e.slackTo;
        count[r]++;
        slack[r] += isSlack;
        lossy[r] += h.gsh[i] != 0.0;
        neg[r] += h.gsh[i] < 0.0;
        net[r] += (pgBus[i] - h.pd[i]) / h.base;  // bus order within each part
    }
    for (int k = 0; k < nb; k++) {
        if (!h.brOn[k] || gone[k]) continue;
        if (!std::isfinite(h.r[k])) return "";
        const int r = find(h.brF[k]);
        lossy[r] += h.r[k] != 0.0;
        neg[r] += h.r[k] < 0.0;
    }
    for (int r = 0; r < n && !unsolvable; r++) {
        if (count[r] == 0 || slack[r] > 0 || neg[r] > 0) continue;
        const double margin = count[r] * tol + kUnsolvableMarginPu;
        unsolvable = net[r] <= -margin || (lossy[r] == 0 && std::fabs(net[r]) >= margin);
    }
    return "";
}

}  // namespace gs

extern "C" int gs_outage_topology(const gs_grid_desc* desc, double tolerance, int32_t nOut, const int32_t* idx,
                                  uint8_t* splits, uint8_t* unsolvable) {
    if (!desc || nOut < 0 || (nOut > 0 && !idx)) return GS_ERR_INVALID_ARG;
    gs::HostGrid g;
    if (!gs::CopyGrid(desc, g).empty()) return GS_ERR_INVALID_ARG;
    return gs::OutageTopology(g, tolerance, nOut, idx, splits, unsolvable).empty() ? GS_OK : GS_ERR_INVALID_ARG;
}

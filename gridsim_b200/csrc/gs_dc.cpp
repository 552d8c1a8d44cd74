// gs_dc.cpp — DC power-flow start angles for the DC-angle retry (host side).
//
// NewtonShell.TrySeedDcAngles (src/GridSim.Core/PowerFlow/NewtonShell.cs:282-299) starts a stalled case again from
// the angles of the DC power flow (Analysis/DcPowerFlow.cs on DcDemand.LegacyView, DcDemand.cs:36-50: every tap 1,
// no phase shift, no Gs): B' from b = 1/x of the in-service branches with non-zero reactance, injections sum(Pg) - Pd,
// one island referenced at the slack. The retried Newton solves run on the device; these angles are their start
// point, computed once per stalled case (a few per screen), by a sparse elimination in minimum-degree order of the
// reduced B' (symmetric positive definite on a single island, so no pivoting is needed).
#include <algorithm>
#include <cmath>
#include <map>
#include <numeric>
#include <vector>

#include "gs_internal.h"

namespace gs {

bool DcAngles(const HostGrid& h, const Symbolic& s, const std::vector<int>& skip, int slack, const double* loadScale,
              std::vector<double>& thetaDeg, int deadBus, int specBus, double specDpPu) {
    const int n = h.n;
    std::vector<int> parent(n);
    std::iota(parent.begin(), parent.end(), 0);
    auto find = [&](int a) {
        while (parent[a] != a) a = parent[a] = parent[parent[a]];
        return a;
    };
    std::vector<int> red(n, -1);
    int nr = 0;
    for (int i = 0; i < n; i++) if (i != slack && i != deadBus) red[i] = nr++;
    std::vector<std::map<int, double>> rows(nr);
    for (int k = 0; k < h.nbr; k++) {
        if (!h.brOn[k] || h.x[k] == 0.0 || std::find(skip.begin(), skip.end(), k) != skip.end()) continue;
        parent[find(h.brF[k])] = find(h.brT[k]);
        const double b = 1.0 / h.x[k];
        const int f = red[h.brF[k]], t = red[h.brT[k]];
        if (f >= 0) rows[f][f] += b;
        if (t >= 0) rows[t][t] += b;
        if (f >= 0 && t >= 0) { rows[f][t] -= b; rows[t][f] -= b; }
    }
    int islands = 0;
    for (int i = 0; i < n; i++) if (i != deadBus && find(i) == i) islands++;  // a removed bus is not in the model
    if (islands != 1 || nr == 0) return false;
    // minimum-degree order of the pattern
    std::vector<int> rowPtr(nr + 1, 0), col;
    for (int r = 0; r < nr; r++) {
        for (auto& kv : rows[r]) col.push_back(kv.first);
        rowPtr[r + 1] = (int)col.size();
    }
    const std::vector<int> perm = MinimumDegreeOrder(nr, rowPtr, col);
    std::vector<int> pinv(nr);
    for (int k = 0; k < nr; k++) pinv[perm[k]] = k;
    std::vector<std::map<int, double>> a(nr);
    for (int r = 0; r < nr; r++)
        for (auto& kv : rows[r]) a[pinv[r]][pinv[kv.first]] = kv.second;
    std::vector<double> rhs(nr, 0.0);
    for (int i = 0; i < n; i++)
        if (red[i] >= 0)  // injections sum(Pg) - Pd (pu), the load scaled as the case's
            rhs[pinv[red[i]]] = (loadScale ? s.pspec[i] - (loadScale[i] - 1.0) * h.pd[i] / h.base : s.pspec[i]) -
                                (i == specBus ? specDpPu : 0.0);
    // elimination (rows keep their upper parts; the pattern is symmetric, so row k's upper columns are the rows
    // that hold column k)
    for (int k = 0; k < nr; k++) {
        const double piv = a[k][k];
        if (!(std::fabs(piv) > 0.0) || !std::isfinite(piv)) return false;
        for (auto it = a[k].upper_bound(k); it != a[k].end(); ++it) {
            const int j = it->first;
            auto jk = a[j].find(k);
            if (jk == a[j].end()) continue;
            const double l = jk->second / piv;
            a[j].erase(jk);
            for (auto c = a[k].upper_bound(k); c != a[k].end(); ++c) a[j][c->first] -= l * c->second;
            rhs[j] -= l * rhs[k];
        }
    }
    std::vector<double> x(nr, 0.0);
    for (int k = nr - 1; k >= 0; k--) {
        double v = rhs[k];
        for (auto c = a[k].upper_bound(k); c != a[k].end(); ++c) v -= c->second * x[c->first];
        x[k] = v / a[k][k];
        if (!std::isfinite(x[k])) return false;
    }
    thetaDeg.assign(n, 0.0);
    for (int i = 0; i < n; i++)
        if (red[i] >= 0) thetaDeg[i] = x[pinv[red[i]]] * 180.0 / 3.14159265358979323846;
    return true;
}

}  // namespace gs

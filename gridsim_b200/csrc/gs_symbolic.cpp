// gs_symbolic.cpp — host symbolic analysis of the gridsim_b200 engine.
//
// One analysis per grid, shared by every system of every batch (contingencies of that grid, load
// scalings, serving requests). It covers:
//   * the Y-bus of the intact grid, stamped as SparseNewtonRaphsonPowerFlow.BuildY does
//     (src/GridSim.Core/PowerFlow/SparseNewtonRaphsonPowerFlow.cs:382-402, AdmittanceStamp.cs:35-76,
//     cell order and summation order of ComplexCsr.Builder, Numerics/Sparse.cs:134-224), and for every
//     branch the values its four cells take when that branch is out (a single-branch outage is a
//     rank-2 change of Y; the replacement values are summed in the order a rebuilt Y would sum them);
//   * the bus specification and equation numbering (NewtonShell.BuildBusSpec :433-486,
//     EquationPositions :327-336) and the Jacobian superset pattern (BuildJacobianStructure :296-332);
//   * a minimum-degree order of that pattern (the same exact-degree method as
//     Numerics/MinimumDegreeOrdering.cs:23-121) and the static-pivot LU pattern it implies: pivots on
//     the permuted diagonal, so L and U^T share the pattern of the symmetric symbolic factor;
//   * the elimination-tree levels and, per level, the warp tasks of the fused "Crout" factorisation
//     with forward substitution: every L/U entry is its own sparse dot product over the row subtree of
//     its node, with the index pairs precomputed here.
#include <algorithm>
#include <functional>
#include <limits>
#include <cmath>
#include <complex>
#include <cstring>
#include <numeric>

#include "gs_internal.h"

namespace gs {

// Shared memory a one-system walk may hold the top of the elimination tree in.
constexpr size_t kTopBudgetBytes = 200 * 1024;
namespace {

using cplx = std::complex<double>;
constexpr double kPi = 3.14159265358979323846;

struct Stamp { cplx yff, ytt, yft, ytf; };

Stamp BranchStamp(double r, double x, double b, double tapRatio, double shiftDeg) {
    cplx ys = cplx(1.0, 0.0) / cplx(r, x);
    cplx bc(0.0, b / 2.0);
    double a = tapRatio == 0 ? 1.0 : tapRatio;
    double sh = shiftDeg * kPi / 180.0;
    cplx t(a * std::cos(sh), a * std::sin(sh));
    return {(ys + bc) / (a * a), ys + bc, -ys / std::conj(t), -ys / t};
}

}  // namespace

std::vector<int> MinimumDegreeOrder(int n, const std::vector<int>& rowPtr, const std::vector<int>& col) {
    // Explicit elimination graph with exact degrees; bucket lists by degree, most recent insertion first;
    // initial insertion in descending index so that the lowest index wins the first ties.
    std::vector<int> order(n);
    std::vector<std::vector<int>> adj(n);
    for (int i = 0; i < n; i++)
        for (int p = rowPtr[i]; p < rowPtr[i + 1]; p++) {
            int j = col[p];
            if (j != i) { adj[i].push_back(j); adj[j].push_back(i); }
        }
    for (auto& a : adj) { std::sort(a.begin(), a.end()); a.erase(std::unique(a.begin(), a.end()), a.end()); }
    std::vector<int> head(n + 1, -1), nxt(n, -1), prv(n, -1), deg(n, 0);
    auto push = [&](int v, int d) {
        deg[v] = d; prv[v] = -1; nxt[v] = head[d];
        if (head[d] >= 0) prv[head[d]] = v;
        head[d] = v;
    };
    auto pop = [&](int v) {
        if (prv[v] >= 0) nxt[prv[v]] = nxt[v]; else head[deg[v]] = nxt[v];
        if (nxt[v] >= 0) prv[nxt[v]] = prv[v];
    };
    for (int i = n - 1; i >= 0; i--) push(i, (int)adj[i].size());
    std::vector<char> gone(n, 0);
    std::vector<int> mark(n, -1), nbr;
    int dmin = 0;
    for (int s = 0; s < n; s++) {
        while (head[dmin] < 0) dmin++;
        int v = head[dmin];
        pop(v);
        gone[v] = 1;
        order[s] = v;
        nbr.clear();
        for (int u : adj[v]) if (!gone[u]) nbr.push_back(u);
        for (int u : nbr) mark[u] = s;
        for (int u : nbr) {
            pop(u);
            std::vector<int>& au = adj[u];
            size_t w = 0;
            for (size_t p = 0; p < au.size(); p++) {
                int x = au[p];
                if (x != v && !gone[x] && mark[x] != s) au[w++] = x;
            }
            au.resize(w);
            for (int y : nbr) if (y != u) au.push_back(y);
            push(u, (int)au.size());
        }
        std::vector<int>().swap(adj[v]);
        if (dmin > 0) dmin--;
    }
    return order;
}

std::string Analyze(const HostGrid& g, Symbolic& s, bool qlim) {
    const int n = g.n;
    s = Symbolic();
    s.n = n;
    s.nbr = g.nbr;
    s.qlim = qlim;

    // ---------------- Y-bus (stamping order: in-service branches in order, then bus shunts) ----------------
    struct Contribution { int row, col, owner; double gv, bv; };  // owner: branch index or -1 (shunt)
    std::vector<Contribution> contrib;
    contrib.reserve(4 * g.nbr + n);
    s.brStamp.assign(8 * (size_t)g.nbr, 0.0);
    for (int k = 0; k < g.nbr; k++) {
        Stamp st = BranchStamp(g.r[k], g.x[k], g.b[k], g.tap[k], g.shift[k]);
        double* o = &s.brStamp[8 * (size_t)k];
        o[0] = st.yff.real(); o[1] = st.yff.imag(); o[2] = st.ytt.real(); o[3] = st.ytt.imag();
        o[4] = st.yft.real(); o[5] = st.yft.imag(); o[6] = st.ytf.real(); o[7] = st.ytf.imag();
        if (!g.brOn[k]) continue;
        int f = g.brF[k], t = g.brT[k];
        const cplx v[4] = {st.yff, st.ytt, st.yft, st.ytf};
        const int rr[4] = {f, t, f, t}, cc[4] = {f, t, t, f};
        for (int q = 0; q < 4; q++)
            if (!(v[q].real() == 0.0 && v[q].imag() == 0.0)) contrib.push_back({rr[q], cc[q], k, v[q].real(), v[q].imag()});
    }
    for (int i = 0; i < n; i++)
        if (!(g.gsh[i] == 0 && g.bsh[i] == 0)) contrib.push_back({i, i, -1, g.gsh[i] / g.base, g.bsh[i] / g.base});
    // cells: per row, columns ascending with the diagonal always present; contributions kept in order
    std::vector<std::vector<int>> rowCols(n);
    for (auto& c : contrib) rowCols[c.row].push_back(c.col);
    s.yRowPtr.assign(n + 1, 0);
    for (int i = 0; i < n; i++) {
        auto& rc = rowCols[i];
        rc.push_back(i);
        std::sort(rc.begin(), rc.end());
        rc.erase(std::unique(rc.begin(), rc.end()), rc.end());
        s.yRowPtr[i + 1] = s.yRowPtr[i] + (int)rc.size();
    }
    s.nnzY = s.yRowPtr[n];
    s.yCol.resize(s.nnzY);
    for (int i = 0; i < n; i++) std::copy(rowCols[i].begin(), rowCols[i].end(), s.yCol.begin() + s.yRowPtr[i]);
    auto cellOf = [&](int i, int j) {
        auto b = s.yCol.begin() + s.yRowPtr[i], e = s.yCol.begin() + s.yRowPtr[i + 1];
        return (int)(std::lower_bound(b, e, j) - s.yCol.begin());
    };
    std::vector<std::vector<int>> cellContrib(s.nnzY);
    for (int c = 0; c < (int)contrib.size(); c++) cellContrib[cellOf(contrib[c].row, contrib[c].col)].push_back(c);
    s.yG.assign(s.nnzY, 0.0);
    s.yB.assign(s.nnzY, 0.0);
    for (int p = 0; p < s.nnzY; p++) {
        double gv = 0.0, bv = 0.0;
        for (int c : cellContrib[p]) { gv += contrib[c].gv; bv += contrib[c].bv; }
        s.yG[p] = gv;
        s.yB[p] = bv;
    }
    s.ccPtr.assign(s.nnzY + 1, 0);
    for (int p = 0; p < s.nnzY; p++) s.ccPtr[p + 1] = s.ccPtr[p] + (int)cellContrib[p].size();
    s.ccOwner.resize(s.ccPtr[s.nnzY]);
    s.ccG.resize(s.ccPtr[s.nnzY]);
    s.ccB.resize(s.ccPtr[s.nnzY]);
    for (int p = 0; p < s.nnzY; p++)
        for (size_t q = 0; q < cellContrib[p].size(); q++) {
            const Contribution& c = contrib[cellContrib[p][q]];
            s.ccOwner[s.ccPtr[p] + q] = c.owner;
            s.ccG[s.ccPtr[p] + q] = c.gv;
            s.ccB[s.ccPtr[p] + q] = c.bv;
        }
    s.brCell.assign(4 * (size_t)g.nbr, -1);
    s.brRed.assign(8 * (size_t)g.nbr, 0.0);
    for (int k = 0; k < g.nbr; k++) {
        if (!g.brOn[k]) continue;
        int f = g.brF[k], t = g.brT[k];
        const int rr[4] = {f, t, f, t}, cc[4] = {f, t, t, f};
        for (int q = 0; q < 4; q++) {
            int p = cellOf(rr[q], cc[q]);
            s.brCell[4 * (size_t)k + q] = p;
            double gv = 0.0, bv = 0.0;
            for (int c : cellContrib[p]) if (contrib[c].owner != k) { gv += contrib[c].gv; bv += contrib[c].bv; }
            s.brRed[8 * (size_t)k + 2 * q] = gv;
            s.brRed[8 * (size_t)k + 2 * q + 1] = bv;
        }
    }

    // ---------------- bus specification and equation numbering ----------------
    std::vector<double> pgB(n, 0), qgB(n, 0), vgB(n, 0);
    std::vector<char> hasGen(n, 0);
    s.qminMvar.assign(n, 0.0);
    s.qmaxMvar.assign(n, 0.0);
    for (int k = 0; k < g.ngen; k++) {
        if (!g.genOn[k]) continue;
        int i = g.genBus[k];
        pgB[i] += g.pg[k];
        qgB[i] += g.qg[k];
        s.qminMvar[i] += g.qmin[k];  // the bus's aggregate reactive limits (NewtonShell.BuildBusSpec)
        s.qmaxMvar[i] += g.qmax[k];
        vgB[i] = g.vg[k];  // the last unit at the bus sets the voltage
        hasGen[i] = 1;
    }
    s.type0.resize(n); s.vm0.resize(n); s.va0.resize(n); s.pspec.resize(n); s.qspec.resize(n);
    for (int i = 0; i < n; i++) {
        int t = g.busType[i];
        s.type0[i] = (t == 2 && !hasGen[i]) ? 1 : t;  // a PV bus with no unit is solved as PQ
        bool vc = s.type0[i] == 3 || s.type0[i] == 2;
        s.vm0[i] = (vc && hasGen[i]) ? vgB[i] : g.vm[i];
        s.va0[i] = g.vaDeg[i] * kPi / 180.0;
        s.pspec[i] = (pgB[i] - g.pd[i]) / g.base;
        s.qspec[i] = (qgB[i] - g.qd[i]) / g.base;
    }
    s.pPos.assign(n, -1);
    s.qPos.assign(n, -1);
    int m = 0;
    // with qlim every bus has both rows: a PV bus may become PQ (Q limits, a generator outage), a reference bus may
    // lose its units and the reference move, a bus may be removed; a row that is not an equation in a system is an
    // identity row there
    for (int i = 0; i < n; i++) if (qlim || s.type0[i] != 3) s.pPos[i] = m++;
    for (int i = 0; i < n; i++) {
        if (s.type0[i] == 1) s.npq++;
        if (qlim || s.type0[i] == 1) s.qPos[i] = m++;
    }
    for (int i = 0; i < n; i++) if (s.type0[i] == 2) s.npv++;
    s.m = m;
    if (m == 0) return "the grid has no unknowns";

    // ---------------- Jacobian superset pattern ----------------
    std::vector<std::vector<int>> jr(m);
    for (int i = 0; i < n; i++) {
        int pi = s.pPos[i], qi = s.qPos[i];
        if (pi < 0 && qi < 0) continue;
        for (int p = s.yRowPtr[i]; p < s.yRowPtr[i + 1]; p++) {
            int j = s.yCol[p], pj = s.pPos[j], qj = s.qPos[j];
            if (pi >= 0 && pj >= 0) jr[pi].push_back(pj);
            if (pi >= 0 && qj >= 0) jr[pi].push_back(qj);
            if (qi >= 0 && pj >= 0) jr[qi].push_back(pj);
            if (qi >= 0 && qj >= 0) jr[qi].push_back(qj);
        }
    }
    s.jRowPtr.assign(m + 1, 0);
    for (int a = 0; a < m; a++) {
        jr[a].push_back(a);
        std::sort(jr[a].begin(), jr[a].end());
        jr[a].erase(std::unique(jr[a].begin(), jr[a].end()), jr[a].end());
        s.jRowPtr[a + 1] = s.jRowPtr[a] + (int)jr[a].size();
    }
    s.nnzJ = s.jRowPtr[m];
    s.jCol.resize(s.nnzJ);
    for (int a = 0; a < m; a++) std::copy(jr[a].begin(), jr[a].end(), s.jCol.begin() + s.jRowPtr[a]);

    return FactorSymbolic(s, [&](const std::function<int64_t(int, int)>& slotOf, std::vector<char>& hasA) {
        // Y cell -> the four Jacobian blocks' LU slots
        s.ySlot.assign(4 * (size_t)s.nnzY, -1);
        for (int i = 0; i < n; i++) {
            int pi = s.pPos[i], qi = s.qPos[i];
            for (int p = s.yRowPtr[i]; p < s.yRowPtr[i + 1]; p++) {
                int j = s.yCol[p], pj = s.pPos[j], qj = s.qPos[j];
                int* o = &s.ySlot[4 * (size_t)p];
                if (pi >= 0 && pj >= 0) o[0] = (int)slotOf(s.pinv[pi], s.pinv[pj]);
                if (pi >= 0 && qj >= 0) o[1] = (int)slotOf(s.pinv[pi], s.pinv[qj]);
                if (qi >= 0 && pj >= 0) o[2] = (int)slotOf(s.pinv[qi], s.pinv[pj]);
                if (qi >= 0 && qj >= 0) o[3] = (int)slotOf(s.pinv[qi], s.pinv[qj]);
            }
        }
        s.busP.assign(n, -1);
        s.busQ.assign(n, -1);
        for (int i = 0; i < n; i++) {
            if (s.pPos[i] >= 0) s.busP[i] = s.pinv[s.pPos[i]];
            if (s.qPos[i] >= 0) s.busQ[i] = s.pinv[s.qPos[i]];
        }
        // which LU slots hold a Jacobian value (the rest are fill, which start from zero)
        for (int v : s.ySlot) if (v >= 0) hasA[v] = 1;
        // the Jacobian's cells in equation order: LU slot, and the Y cell between their buses
        std::vector<int> eqBus(m, -1);
        for (int i = 0; i < n; i++) {
            if (s.pPos[i] >= 0) eqBus[s.pPos[i]] = i;
            if (s.qPos[i] >= 0) eqBus[s.qPos[i]] = i;
        }
        s.jSlot.assign(s.nnzJ, -1);
        s.jYcell.assign(s.nnzJ, -1);
        for (int r = 0; r < m; r++)
            for (int q = s.jRowPtr[r]; q < s.jRowPtr[r + 1]; q++) {
                const int c = s.jCol[q];
                s.jSlot[q] = (int32_t)slotOf(s.pinv[r], s.pinv[c]);
                const int bi = eqBus[r], bj = eqBus[c];
                if (bi == bj) continue;
                for (int p = s.yRowPtr[bi]; p < s.yRowPtr[bi + 1]; p++)
                    if (s.yCol[p] == bj) { s.jYcell[q] = p; break; }
            }
    });
}

std::string FactorSymbolic(Symbolic& s, const std::function<void(const std::function<int64_t(int, int)>&,
                                                                 std::vector<char>&)>& mapA) {
    const int m = s.m;
    // ---------------- ordering and static-pivot LU pattern ----------------
    s.perm = MinimumDegreeOrder(m, s.jRowPtr, s.jCol);
    s.pinv.assign(m, -1);
    for (int k = 0; k < m; k++) s.pinv[s.perm[k]] = k;
    s.parent.assign(m, -1);
    std::vector<std::vector<int>> children(m);
    std::vector<std::vector<int>> P(m);
    std::vector<int> mark(m, -1);
    for (int k = 0; k < m; k++) {
        std::vector<int>& pk = P[k];
        mark[k] = k;
        int a = s.perm[k];
        for (int p = s.jRowPtr[a]; p < s.jRowPtr[a + 1]; p++) {
            int l = s.pinv[s.jCol[p]];
            if (l > k && mark[l] != k) { mark[l] = k; pk.push_back(l); }
        }
        for (int c : children[k])
            for (int l : P[c])
                if (l > k && mark[l] != k) { mark[l] = k; pk.push_back(l); }
        std::sort(pk.begin(), pk.end());
        if (!pk.empty()) { s.parent[k] = pk[0]; children[pk[0]].push_back(k); }
    }
    s.luBase.resize(m + 1);
    s.luCnt.resize(m);
    s.pRowPtr.assign(m + 1, 0);
    int64_t off = 0;
    for (int k = 0; k < m; k++) {
        s.luBase[k] = off;
        s.luCnt[k] = (int)P[k].size();
        off += 1 + 2 * (int64_t)P[k].size();
        s.pRowPtr[k + 1] = s.pRowPtr[k] + (int)P[k].size();
    }
    s.luBase[m] = off;
    s.nnzLU = off;
    if (off >= (int64_t)INT32_MAX) return "the LU factor is too large for 32-bit slot indices";
    s.pRows.resize(s.pRowPtr[m]);
    for (int k = 0; k < m; k++) std::copy(P[k].begin(), P[k].end(), s.pRows.begin() + s.pRowPtr[k]);
    auto posIn = [&](int k, int l) {  // index of l in P_k (l > k)
        const int* b = &s.pRows[s.pRowPtr[k]];
        const int* e = b + s.luCnt[k];
        const int* it = std::lower_bound(b, e, l);
        return (it != e && *it == l) ? (int)(it - b) : -1;
    };
    auto slotOf = [&](int k, int l) -> int64_t {  // LU slot of permuted cell (k, l)
        if (k == l) return s.luBase[k];
        if (k < l) { int t = posIn(k, l); return t < 0 ? -1 : s.luBase[k] + 1 + t; }
        int t = posIn(l, k);
        return t < 0 ? -1 : s.luBase[l] + 1 + s.luCnt[l] + t;
    };
    std::vector<char> hasA(s.nnzLU, 0);
    mapA(slotOf, hasA);
    {
        // the cells that receive a value of A, by column: node k holds (k, k), U(k, l) and L(l, k) for l in P_k
        std::vector<std::vector<std::pair<int, int32_t>>> cols(m);
        for (int k = 0; k < m; k++) {
            const int64_t b0 = s.luBase[k];
            const int c = s.luCnt[k];
            if (hasA[b0]) cols[k].push_back({k, (int32_t)b0});
            for (int t = 0; t < c; t++) {
                const int l = s.pRows[s.pRowPtr[k] + t];
                if (hasA[b0 + 1 + t]) cols[l].push_back({k, (int32_t)(b0 + 1 + t)});
                if (hasA[b0 + 1 + c + t]) cols[k].push_back({l, (int32_t)(b0 + 1 + c + t)});
            }
        }
        s.aColPtr.assign(m + 1, 0);
        s.aRow.clear();
        s.aSlot.clear();
        for (int l = 0; l < m; l++) {
            std::sort(cols[l].begin(), cols[l].end());
            for (const auto& e : cols[l]) { s.aRow.push_back(e.first); s.aSlot.push_back(e.second); }
            s.aColPtr[l + 1] = (int32_t)s.aRow.size();
        }
    }

    // ---------------- levels ----------------
    s.level.assign(m, 0);
    for (int k = 0; k < m; k++)
        if (s.parent[k] >= 0) s.level[s.parent[k]] = std::max(s.level[s.parent[k]], s.level[k] + 1);
    s.nLevels = 0;
    for (int k = 0; k < m; k++) s.nLevels = std::max(s.nLevels, s.level[k] + 1);
    s.levelNodePtr.assign(s.nLevels + 1, 0);
    for (int k = 0; k < m; k++) s.levelNodePtr[s.level[k] + 1]++;
    for (int l = 0; l < s.nLevels; l++) s.levelNodePtr[l + 1] += s.levelNodePtr[l];
    s.levelNodes.resize(m);
    {
        std::vector<int> fill(s.levelNodePtr.begin(), s.levelNodePtr.end() - 1);
        for (int k = 0; k < m; k++) s.levelNodes[fill[s.level[k]]++] = k;
    }

    // ---------------- Crout entries and their index pairs ----------------
    // Row subtree J_k = { j < k : k in P_j }, ascending.
    std::vector<std::vector<int>> rowSub(m);
    for (int j = 0; j < m; j++)
        for (int t = s.pRowPtr[j]; t < s.pRowPtr[j + 1]; t++) rowSub[s.pRows[t]].push_back(j);
    // Per node k the entries are: diag, U(k, P_k[t]) for each t, forward y(k), L(P_k[t], k) for each t.
    s.entPairPtr.assign(1, 0);
    s.diagPairNode.assign(m, -1);
    std::vector<int> posK(m, -1);
    std::vector<int64_t> cnt;
    std::vector<std::vector<int32_t>> lists;
    s.flops = 0;
    for (int k = 0; k < m; k++) {
        const int c = s.luCnt[k];
        const int nE = 2 * c + 2;
        for (int t = 0; t < c; t++) posK[s.pRows[s.pRowPtr[k] + t]] = t;
        lists.assign(nE, {});
        // entry indices: 0 diag, 1..c upper, c+1 fwd, c+2..2c+1 lower
        for (int j : rowSub[k]) {
            int tk = posIn(j, k);
            int cj = s.luCnt[j];
            int64_t Lkj = s.luBase[j] + 1 + cj + tk, Ujk = s.luBase[j] + 1 + tk;
            lists[0].push_back((int32_t)Lkj); lists[0].push_back((int32_t)Ujk);
            lists[c + 1].push_back((int32_t)Lkj); lists[c + 1].push_back(j);
            for (int t = tk + 1; t < cj; t++) {
                int r = s.pRows[s.pRowPtr[j] + t];
                int tr = posK[r];  // r in P_k by the fill property
                int64_t Ujr = s.luBase[j] + 1 + t, Lrj = s.luBase[j] + 1 + cj + t;
                lists[1 + tr].push_back((int32_t)Lkj); lists[1 + tr].push_back((int32_t)Ujr);
                lists[c + 2 + tr].push_back((int32_t)Lrj); lists[c + 2 + tr].push_back((int32_t)Ujk);
            }
        }
        int e0 = (int)s.entSlot.size();
        s.diagPairNode[k] = e0;
        for (int e = 0; e < nE; e++) {
            int32_t slot, kind;
            if (e == 0) { slot = (int32_t)s.luBase[k]; kind = kDiag; }
            else if (e <= c) { slot = (int32_t)(s.luBase[k] + e); kind = kUpper; }
            else if (e == c + 1) { slot = k; kind = kFwd; }
            else { slot = (int32_t)(s.luBase[k] + 1 + c + (e - c - 2)); kind = kLower; }
            s.entSlot.push_back(slot);
            s.entKind.push_back(kind);
            s.entHasA.push_back(kind == kFwd ? 1 : (int32_t)hasA[slot]);
            s.pairs.insert(s.pairs.end(), lists[e].begin(), lists[e].end());
            s.entPairPtr.push_back((int64_t)s.pairs.size() / 2);
            s.flops += (int64_t)lists[e].size() / 2;
        }
        for (int t = 0; t < c; t++) posK[s.pRows[s.pRowPtr[k] + t]] = -1;
    }

    // ---------------- work schedules per level ----------------
    s.entNode.assign(s.entSlot.size(), 0);
    for (int k = 0; k < m; k++)
        for (int e = s.diagPairNode[k]; e < s.diagPairNode[k] + 2 * s.luCnt[k] + 2; e++) s.entNode[e] = k;
    // Short pieces (at most kShort pairs) are packed kPack to an item (the most lane groups a warp has:
    // 4 for FP32, 8 for FP64 -- the kernels take the first `count`); longer ones get a warp each.
    const int kShort = 32, kPack = 8;
    // The short pieces of a level are ordered longest first; the one-system walks give those with more than kMid
    // pairs a group of lanes each (levelMid counts them).
    const int kMid = 8;
    auto pack = [&](Symbolic::Schedule& sc, const std::vector<int32_t>& list, const std::vector<int64_t>& len,
                    int64_t midAbove) {
        std::vector<std::pair<int64_t, int32_t>> shortLen;
        int wide = 0;
        for (size_t q = 0; q < list.size(); q++) {
            if (len[q] > kShort) {
                sc.work.push_back(list[q]);
                sc.items.push_back((int32_t)sc.work.size() - 1);
                sc.items.push_back(-1);
                wide++;
            } else {
                shortLen.push_back({len[q], list[q]});
            }
        }
        std::stable_sort(shortLen.begin(), shortLen.end(),
                         [](const std::pair<int64_t, int32_t>& a, const std::pair<int64_t, int32_t>& b) { return a.first > b.first; });
        std::vector<int32_t> shortOnes;
        int mid = 0;
        for (auto& pr : shortLen) {
            shortOnes.push_back(pr.second);
            if (pr.first > midAbove) mid++;
        }
        sc.levelMid.push_back(mid);
        for (size_t q = 0; q < shortOnes.size(); q += kPack) {
            int cnt = (int)std::min<size_t>(kPack, shortOnes.size() - q);
            sc.items.push_back((int32_t)sc.work.size());
            sc.items.push_back(cnt);
            for (int t = 0; t < cnt; t++) sc.work.push_back(shortOnes[q + t]);
        }
        sc.levelItemPtr.push_back((int32_t)sc.items.size() / 2);
        sc.levelWorkPtr.push_back((int32_t)sc.work.size());
        sc.levelWide.push_back(wide);
    };
    for (Symbolic::Schedule* sc : {&s.factor, &s.backward, &s.forward}) {
        sc->levelItemPtr.assign(1, 0);
        sc->levelWorkPtr.assign(1, 0);
    }
    for (int l = 0; l < s.nLevels; l++) {
        std::vector<int32_t> phaseA, phaseB, bwd, fwd;
        std::vector<int64_t> lenA, lenB, lenBwd, lenFwd;
        for (int q = s.levelNodePtr[l]; q < s.levelNodePtr[l + 1]; q++) {
            const int k = s.levelNodes[q];
            const int e0 = s.diagPairNode[k], c = s.luCnt[k];
            for (int e = e0; e < e0 + 2 * c + 2; e++) {
                const int64_t np = s.entPairPtr[e + 1] - s.entPairPtr[e];
                const int kind = s.entKind[e];
                // an upper or forward entry with no pairs keeps its value where it already is
                if ((kind == kUpper || kind == kFwd) && np == 0 && s.entHasA[e]) continue;
                if (kind == kLower) { phaseB.push_back(e); lenB.push_back(np); }
                else { phaseA.push_back(e); lenA.push_back(np); }
                if (kind == kFwd) { fwd.push_back(e); lenFwd.push_back(np); }
            }
            bwd.push_back(q);
            lenBwd.push_back(c);
        }
        pack(s.factor, phaseA, lenA, kMid);
        pack(s.factor, phaseB, lenB, kMid);
        pack(s.backward, bwd, lenBwd, kMid);
        pack(s.forward, fwd, lenFwd, kMid);
    }

    // ---------------- the paired schedule (Symbolic::PairSchedule) ----------------
    {
        Symbolic::PairSchedule& P = s.ps;
        P = Symbolic::PairSchedule();
        // units: k, k + 1 paired when parent(k) = k + 1, |P_k| = |P_{k+1}| + 1 (so P_k = {k + 1} + P_{k+1} by the
        // fill property) and the row subtree of k + 1 is that of k plus k; every other node alone
        std::vector<int> unitOf(m, -1), unitFirst;
        std::vector<char> unitPair;
        for (int k = 0; k < m;) {
            bool pair = false;
            if (k + 1 < m && s.parent[k] == k + 1 && s.luCnt[k] == s.luCnt[k + 1] + 1) {
                const std::vector<int>& a = rowSub[k];
                const std::vector<int>& b2 = rowSub[k + 1];
                pair = b2.size() == a.size() + 1 && b2.back() == k && std::equal(a.begin(), a.end(), b2.begin());
            }
            unitOf[k] = (int)unitFirst.size();
            if (pair) unitOf[k + 1] = (int)unitFirst.size();
            unitFirst.push_back(k);
            unitPair.push_back(pair ? 1 : 0);
            k += pair ? 2 : 1;
        }
        const int nU = (int)unitFirst.size();
        std::vector<int> uLevel(nU, 0);
        for (int u = 0; u < nU; u++) {  // a unit's parent unit holds the parent of its last node (a later unit)
            const int par = s.parent[unitFirst[u] + unitPair[u]];
            if (par >= 0) uLevel[unitOf[par]] = std::max(uLevel[unitOf[par]], uLevel[u] + 1);
        }
        int nL = 0;
        for (int u = 0; u < nU; u++) nL = std::max(nL, uLevel[u] + 1);
        std::vector<std::vector<int>> byLevel(nL);
        for (int u = 0; u < nU; u++) byLevel[uLevel[u]].push_back(u);
        auto npairs = [&]() { return (int64_t)P.pairs.size() / 2; };
        auto addTask = [&](int64_t q0, int kindFlags, int k, int64_t s0, int64_t s1, int64_t aux) {
            P.taskA.insert(P.taskA.end(), {(int32_t)q0, (int32_t)npairs(), kindFlags, k});
            P.taskB.insert(P.taskB.end(), {(int32_t)s0, (int32_t)s1, (int32_t)aux, 0});
            return (int32_t)(P.taskA.size() / 4 - 1);
        };
        auto addBack = [&](int r0, int r1, int kind, int k, int64_t s0, int64_t s1, int64_t aux) {
            P.bTaskA.insert(P.bTaskA.end(), {r0, r1, kind, k});
            P.bTaskB.insert(P.bTaskB.end(), {(int32_t)s0, (int32_t)s1, (int32_t)aux, 0});
            return (int32_t)(P.bTaskA.size() / 4 - 1);
        };
        auto hb = [&](int64_t slot) { return (int)hasA[slot]; };
        for (Symbolic::Schedule* sc : {&P.factor, &P.backward, &P.forward}) {
            sc->levelItemPtr.assign(1, 0);
            sc->levelWorkPtr.assign(1, 0);
        }
        std::vector<int> posK1(m, -1);
        std::vector<std::vector<int32_t>> up, lo;
        std::vector<int32_t> dg, fw;
        for (int l = 0; l < nL; l++) {
            std::vector<int32_t> phA, phB, bwd, fwd;
            std::vector<int64_t> lenA, lenB, lenBwd, lenFwd;
            for (int u : byLevel[l]) {
                const int k = unitFirst[u];
                if (!unitPair[u]) {  // a single node: its entries as in the scalar schedule
                    const int e0 = s.diagPairNode[k], c = s.luCnt[k];
                    for (int e = e0; e < e0 + 2 * c + 2; e++) {
                        const int64_t p0 = s.entPairPtr[e], p1 = s.entPairPtr[e + 1];
                        const int kind = s.entKind[e];
                        if ((kind == kUpper || kind == kFwd) && p1 == p0 && s.entHasA[e]) continue;
                        const int64_t q0 = npairs();
                        P.pairs.insert(P.pairs.end(), s.pairs.begin() + 2 * p0, s.pairs.begin() + 2 * p1);
                        const int32_t t = addTask(q0, kind | (s.entHasA[e] << 3), k, s.entSlot[e], 0, 0);
                        if (kind == kLower) { phB.push_back(t); lenB.push_back(p1 - p0); }
                        else { phA.push_back(t); lenA.push_back(p1 - p0); }
                        if (kind == kFwd) { fwd.push_back(t); lenFwd.push_back(p1 - p0); }
                    }
                    bwd.push_back(addBack(s.pRowPtr[k], s.pRowPtr[k + 1], kBNode, k, s.luBase[k], 0, 0));
                    lenBwd.push_back(c);
                    continue;
                }
                // a pair k, k + 1: c = |P_{k+1}|, |P_k| = c + 1. Slots: U(k, k + 1) = bk + 1, L(k + 1, k) = bk + 2 + c,
                // U(k, P_{k+1}[t]) = bk + 2 + t, L(P_{k+1}[t], k) = bk + 3 + c + t, U(k + 1, P_{k+1}[t]) = bk1 + 1 + t,
                // L(P_{k+1}[t], k + 1) = bk1 + 1 + c + t
                const int c = s.luCnt[k + 1];
                const int64_t bk = s.luBase[k], bk1 = s.luBase[k + 1];
                const int64_t sUkk1 = bk + 1, sLk1k = bk + 2 + c;
                for (int t = 0; t < c; t++) posK1[s.pRows[s.pRowPtr[k + 1] + t]] = t;
                up.assign(c, {});
                lo.assign(c, {});
                dg.clear();
                fw.clear();
                for (int j : rowSub[k]) {
                    const int cj = s.luCnt[j];
                    const int tk = posIn(j, k);  // k + 1 follows at tk + 1 (the pairing rule)
                    if (tk < 0 || tk + 1 >= cj || s.pRows[s.pRowPtr[j] + tk + 1] != k + 1)
                        return "paired schedule: node " + std::to_string(j) + " breaks the pair " + std::to_string(k);
                    const int64_t Lkj = s.luBase[j] + 1 + cj + tk, Ujk = s.luBase[j] + 1 + tk;
                    dg.push_back((int32_t)Lkj); dg.push_back((int32_t)Ujk);
                    fw.push_back((int32_t)Lkj); fw.push_back(j);
                    for (int t2 = tk + 2; t2 < cj; t2++) {  // r of P_j beyond k + 1 lies in P_{k+1}
                        const int tr = posK1[s.pRows[s.pRowPtr[j] + t2]];
                        if (tr < 0) return "paired schedule: fill outside P_{k+1} at node " + std::to_string(k);
                        up[tr].push_back((int32_t)Lkj); up[tr].push_back((int32_t)(s.luBase[j] + 1 + t2));
                        lo[tr].push_back((int32_t)(s.luBase[j] + 1 + cj + t2)); lo[tr].push_back((int32_t)Ujk);
                    }
                }
                int64_t q0 = npairs();
                P.pairs.insert(P.pairs.end(), dg.begin(), dg.end());
                int32_t t = addTask(q0, kPDiag | (hb(bk) | hb(sUkk1) << 1 | hb(sLk1k) << 2 | hb(bk1) << 3) << 3, k, bk, bk1, c);
                phA.push_back(t);
                lenA.push_back((int64_t)dg.size());  // four products a pair
                q0 = npairs();
                P.pairs.insert(P.pairs.end(), fw.begin(), fw.end());
                t = addTask(q0, kPFwd, k, k, 0, sLk1k);
                phB.push_back(t);
                lenB.push_back((int64_t)fw.size() / 2);
                fwd.push_back(t);
                lenFwd.push_back((int64_t)fw.size() / 2);
                for (int tt = 0; tt < c; tt++) {
                    const int64_t sU0 = bk + 2 + tt, sU1 = bk1 + 1 + tt, sL0 = bk + 3 + c + tt, sL1 = bk1 + 1 + c + tt;
                    q0 = npairs();
                    P.pairs.insert(P.pairs.end(), up[tt].begin(), up[tt].end());
                    t = addTask(q0, kPUpper | (hb(sU0) | hb(sU1) << 1) << 3, k, sU0, sU1, sLk1k);
                    phB.push_back(t);
                    lenB.push_back((int64_t)up[tt].size() / 2);
                    q0 = npairs();
                    P.pairs.insert(P.pairs.end(), lo[tt].begin(), lo[tt].end());
                    t = addTask(q0, kPLower | (hb(sL0) | hb(sL1) << 1) << 3, k, sL0, sL1, sUkk1);
                    phB.push_back(t);
                    lenB.push_back((int64_t)lo[tt].size() / 2);
                }
                for (int tt = 0; tt < c; tt++) posK1[s.pRows[s.pRowPtr[k + 1] + tt]] = -1;
                bwd.push_back(addBack(s.pRowPtr[k + 1], s.pRowPtr[k + 1] + c, kBPair, k, bk + 2, bk1 + 1, sUkk1));
                lenBwd.push_back(c);
                P.nPaired++;
            }
            // the cluster walk keeps four pairs in flight a lane on this schedule: pieces above four pairs go to
            // 8-lane groups
            pack(P.factor, phA, lenA, 4);
            pack(P.factor, phB, lenB, 4);
            pack(P.backward, bwd, lenBwd, 4);
            pack(P.forward, fwd, lenFwd, 4);
        }
        if (npairs() >= (int64_t)INT32_MAX) return "the paired schedule is too large for 32-bit pair indices";
        P.nUnits = nU;
        P.nLevels = nL;
        P.unitOf = unitOf;
        P.unitLevel = uLevel;
        P.unitParent.assign(nU, -1);
        for (int u = 0; u < nU; u++) {
            const int par = s.parent[unitFirst[u] + unitPair[u]];
            if (par >= 0) P.unitParent[u] = unitOf[par];
        }
        P.on = true;
    }
    BuildTopPart(s, 0, sizeof(double), kTopBudgetBytes);
    BuildTopPart(s, 1, sizeof(float), kTopBudgetBytes);
    return "";
}

std::string AnalyzeMatrix(int n, const int* rowPtr, const int* colIdx, Symbolic& s, std::vector<int>& aSlot) {
    s = Symbolic();
    if (n <= 0) return "the matrix has no rows";
    if (rowPtr[0] != 0) return "row_ptr[0] must be 0";
    for (int i = 0; i < n; i++)
        if (rowPtr[i + 1] < rowPtr[i]) return "row_ptr must not decrease";
    const int nnz = rowPtr[n];
    std::vector<std::vector<int>> jr(n);
    for (int i = 0; i < n; i++) {
        for (int p = rowPtr[i]; p < rowPtr[i + 1]; p++) {
            const int j = colIdx[p];
            if (j < 0 || j >= n) return "a column index is out of range";
            jr[i].push_back(j);
            jr[j].push_back(i);
        }
        jr[i].push_back(i);
    }
    for (int i = 0; i < n; i++) {  // a column twice in one row is malformed (CsrMatrix holds each cell once)
        std::vector<int> row(colIdx + rowPtr[i], colIdx + rowPtr[i + 1]);
        std::sort(row.begin(), row.end());
        if (std::adjacent_find(row.begin(), row.end()) != row.end()) return "a row names a column twice";
    }
    s.n = n;
    s.m = n;
    s.jRowPtr.assign(n + 1, 0);
    for (int a = 0; a < n; a++) {
        std::sort(jr[a].begin(), jr[a].end());
        jr[a].erase(std::unique(jr[a].begin(), jr[a].end()), jr[a].end());
        s.jRowPtr[a + 1] = s.jRowPtr[a] + (int)jr[a].size();
    }
    s.nnzJ = s.jRowPtr[n];
    s.jCol.resize(s.nnzJ);
    for (int a = 0; a < n; a++) std::copy(jr[a].begin(), jr[a].end(), s.jCol.begin() + s.jRowPtr[a]);
    s.yRowPtr.assign(n + 1, 0);  // no Y: the value kernels of the load flow are not used on a bare matrix
    s.busP.assign(n, -1);
    s.busQ.assign(n, -1);
    return FactorSymbolic(s, [&](const std::function<int64_t(int, int)>& slotOf, std::vector<char>& hasA) {
        aSlot.assign(nnz, -1);
        for (int i = 0; i < n; i++)
            for (int p = rowPtr[i]; p < rowPtr[i + 1]; p++) {
                aSlot[p] = (int)slotOf(s.pinv[i], s.pinv[colIdx[p]]);
                hasA[aSlot[p]] = 1;
            }
    });
}

SubtreeSchedule BuildSubtrees(const Symbolic& s, int cut) {
    SubtreeSchedule out;
    const Symbolic::PairSchedule& P = s.ps;
    if (!P.on || cut < 0) return out;
    cut = std::min(cut, P.nLevels - 1);
    const int nU = P.nUnits;
    // the subtree root of every unit at or below the cut
    std::vector<int> root(nU, -1);
    for (int u = 0; u < nU; u++) {
        if (P.unitLevel[u] > cut) continue;
        int r = u;
        while (P.unitParent[r] >= 0 && P.unitLevel[P.unitParent[r]] <= cut) r = P.unitParent[r];
        root[u] = r;
    }
    std::vector<int> subOf(nU, -1), rootsOrder;
    for (int u = 0; u < nU; u++)
        if (root[u] == u) { subOf[u] = (int)rootsOrder.size(); rootsOrder.push_back(u); }
    const int nSub = (int)rootsOrder.size();
    // per subtree and stage (level, phase): its work positions
    std::vector<std::vector<std::vector<int32_t>>> lists(nSub, std::vector<std::vector<int32_t>>(2 * (cut + 1)));
    std::vector<int64_t> pairs(nSub, 0), entries(nSub, 0);
    int64_t allPairs = 0, below = 0;
    for (int l = 0; l < P.nLevels; l++)
        for (int ph = 0; ph < 2; ph++)
            for (int w = P.factor.levelWorkPtr[2 * l + ph]; w < P.factor.levelWorkPtr[2 * l + ph + 1]; w++) {
                const int t = P.factor.work[w];
                const int64_t np = (int64_t)P.taskA[4 * t + 1] - P.taskA[4 * t];
                allPairs += np;
                if (l > cut) continue;
                const int u = P.unitOf[P.taskA[4 * t + 3]];
                const int sub = subOf[root[u]];
                lists[sub][2 * l + ph].push_back(w);
                pairs[sub] += np;
                below += np;
            }
    // the LU entries of each subtree: its nodes' diagonal, U row and L column
    for (int k = 0; k < s.m; k++) {
        const int u = P.unitOf[k];
        if (root[u] >= 0) entries[subOf[root[u]]] += 1 + 2 * (int64_t)s.luCnt[k];
    }
    std::vector<int> order(nSub);
    for (int q = 0; q < nSub; q++) order[q] = q;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return pairs[a] > pairs[b]; });
    out.cut = cut;
    out.nSub = nSub;
    out.subStage.push_back(0);
    out.stagePtr.push_back(0);
    for (int q : order) {
        for (const auto& st : lists[q]) {
            if (st.empty()) continue;
            out.work.insert(out.work.end(), st.begin(), st.end());
            out.stagePtr.push_back((int32_t)out.work.size());
        }
        out.subStage.push_back((int32_t)out.stagePtr.size() - 1);
        out.maxEntries = std::max(out.maxEntries, entries[q]);
    }
    out.pairShare = allPairs > 0 ? (double)below / (double)allPairs : 0.0;
    return out;
}

void BuildTopPart(Symbolic& s, int which, size_t elem, size_t budget) {
    Symbolic::TopPart& t = s.top[which];
    t = Symbolic::TopPart();
    const int m = s.m, L = s.nLevels;
    // values (LU + right-hand side) of the top from each level up
    std::vector<int64_t> vals(L + 1, 0);
    for (int l = L - 1; l >= 0; l--) {
        int64_t v = 0;
        for (int q = s.levelNodePtr[l]; q < s.levelNodePtr[l + 1]; q++) v += 2 * (int64_t)s.luCnt[s.levelNodes[q]] + 2;
        vals[l] = vals[l + 1] + v;
    }
    int L0 = L;
    while (L0 > 0 && (size_t)vals[L0 - 1] * elem <= budget) L0--;
    t.L0 = L0;
    if (L0 >= L) return;
    const int nTop = L - L0;
    t.smemBase.assign(m, -1);
    t.yIdx.assign(m, -1);
    for (int l = L0; l < L; l++)
        for (int q = s.levelNodePtr[l]; q < s.levelNodePtr[l + 1]; q++) {
            const int k = s.levelNodes[q];
            t.smemBase[k] = t.nSlots;
            for (int x = 0; x < 2 * s.luCnt[k] + 1; x++) {
                t.slotGlobal.push_back((int32_t)(s.luBase[k] + x));
                t.slotDiagNode.push_back(x == 0 ? k : -1);
            }
            t.nSlots += 2 * s.luCnt[k] + 1;
            t.nodes.push_back(k);
        }
    t.nNodes = (int)t.nodes.size();
    for (int i = 0; i < t.nNodes; i++) t.yIdx[t.nodes[i]] = t.nSlots + i;
    std::vector<int> slotNode(s.nnzLU);
    for (int k = 0; k < m; k++)
        for (int64_t x = s.luBase[k]; x < s.luBase[k] + 2 * s.luCnt[k] + 1; x++) slotNode[x] = k;
    // entries of the top nodes and their pairs split into internal (smem) and external (global) ones
    constexpr int kWideTop = 32, kWideExt = 16;
    std::vector<int32_t> nInt, nExt, kindOf;
    t.intPtr.assign(1, 0);
    t.extPtr.assign(1, 0);
    std::vector<int32_t> firstEnt(m, -1);
    for (int k : t.nodes) {
        firstEnt[k] = (int32_t)t.ent.size();
        const int e0 = s.diagPairNode[k];
        for (int e = e0; e < e0 + 2 * s.luCnt[k] + 2; e++) {
            const int kind = s.entKind[e];
            t.ent.push_back(e);
            t.entSm.push_back(kind == kFwd ? t.yIdx[k] : t.smemBase[k] + (int32_t)(s.entSlot[e] - s.luBase[k]));
            int ni = 0, nx = 0;
            for (int64_t q = s.entPairPtr[e]; q < s.entPairPtr[e + 1]; q++) {
                const int left = s.pairs[2 * q], right = s.pairs[2 * q + 1];
                const int j = slotNode[left];
                if (s.level[j] >= L0) {
                    t.intPairs.push_back(t.smemBase[j] + (int32_t)(left - s.luBase[j]));
                    t.intPairs.push_back(kind == kFwd ? t.yIdx[right] : t.smemBase[j] + (int32_t)(right - s.luBase[j]));
                    ni++;
                } else {
                    t.extPairs.push_back(left);
                    t.extPairs.push_back(right);
                    nx++;
                }
            }
            t.intPtr.push_back((int32_t)(t.intPairs.size() / 2));
            t.extPtr.push_back((int32_t)(t.extPairs.size() / 2));
            nInt.push_back(ni);
            nExt.push_back(nx);
            kindOf.push_back(kind);
        }
    }
    const int nEnt = (int)t.ent.size();
    for (int ti = 0; ti < nEnt; ti++) if (nExt[ti] > kWideExt) t.loadList.push_back(ti);
    t.loadWide = (int)t.loadList.size();
    for (int ti = 0; ti < nEnt; ti++) if (nExt[ti] <= kWideExt) t.loadList.push_back(ti);
    for (int ti = 0; ti < nEnt; ti++) if (kindOf[ti] == kFwd && nExt[ti] > kWideExt) t.fwdLoadList.push_back(ti);
    t.fwdLoadWide = (int)t.fwdLoadList.size();
    for (int ti = 0; ti < nEnt; ti++) if (kindOf[ti] == kFwd && nExt[ti] <= kWideExt) t.fwdLoadList.push_back(ti);
    // walks per top level
    auto addWide = [&](std::vector<int32_t>& walk, std::vector<int32_t>& wideCnt, std::vector<int32_t>& ptr,
                       const std::vector<int32_t>& list, const std::vector<int32_t>& len, int wideAt) {
        int w = 0;
        for (size_t q = 0; q < list.size(); q++) if (len[q] > wideAt) { walk.push_back(list[q]); w++; }
        for (size_t q = 0; q < list.size(); q++) if (len[q] <= wideAt) walk.push_back(list[q]);
        wideCnt.push_back(w);
        ptr.push_back((int32_t)walk.size());
    };
    t.fWalkPtr.assign(1, 0);
    t.vWalkPtr.assign(1, 0);
    t.bWalkPtr.assign(1, 0);
    std::vector<int32_t> nodeIndex(m, -1);
    for (int i = 0; i < t.nNodes; i++) nodeIndex[t.nodes[i]] = i;
    for (int lt = 0; lt < nTop; lt++) {
        const int l = L0 + lt;
        std::vector<int32_t> pa, pb, pf, la, lb, lf, bn, lbn;
        for (int q = s.levelNodePtr[l]; q < s.levelNodePtr[l + 1]; q++) {
            const int k = s.levelNodes[q];
            const int c = s.luCnt[k];
            for (int ti = firstEnt[k]; ti < firstEnt[k] + 2 * c + 2; ti++) {
                const int kind = kindOf[ti];
                // after the load an upper or forward entry without internal pairs holds its final value
                if (kind == kLower) { pb.push_back(ti); lb.push_back(nInt[ti]); }
                else if (kind == kDiag || nInt[ti] > 0) { pa.push_back(ti); la.push_back(nInt[ti]); }
                if (kind == kFwd && nInt[ti] > 0) { pf.push_back(ti); lf.push_back(nInt[ti]); }
            }
            bn.push_back(nodeIndex[k]);
            lbn.push_back(c);
        }
        addWide(t.fWalk, t.fWalkWide, t.fWalkPtr, pa, la, kWideTop);
        addWide(t.fWalk, t.fWalkWide, t.fWalkPtr, pb, lb, kWideTop);
        addWide(t.vWalk, t.vWalkWide, t.vWalkPtr, pf, lf, kWideTop);
        addWide(t.bWalk, t.bWalkWide, t.bWalkPtr, bn, lbn, kWideTop);
    }
    t.bRowPtr.assign(1, 0);
    for (int i = 0; i < t.nNodes; i++) {
        const int k = t.nodes[i];
        for (int q = s.pRowPtr[k]; q < s.pRowPtr[k + 1]; q++) t.bRowSm.push_back(t.yIdx[s.pRows[q]]);
        t.bRowPtr.push_back((int32_t)t.bRowSm.size());
    }
}

int AddOutageSet(const Symbolic& s, const std::vector<int>& b, OutageSetTable& t) {
    std::vector<int> cells;
    for (int k : b)
        for (int q = 0; q < 4; q++) cells.push_back(s.brCell[4 * (size_t)k + q]);
    std::sort(cells.begin(), cells.end());
    cells.erase(std::unique(cells.begin(), cells.end()), cells.end());
    const int q = t.n++;
    t.br.resize((size_t)t.n * kSetBranches, -1);
    t.cell.resize((size_t)t.n * kSetStride, std::numeric_limits<int>::max());
    t.red.resize((size_t)t.n * 2 * kSetStride, 0.0);
    for (size_t j = 0; j < b.size(); j++) t.br[(size_t)q * kSetBranches + j] = b[j];
    for (size_t c = 0; c < cells.size(); c++) {
        const int p = cells[c];
        double gv = 0.0, bv = 0.0;  // the cell's stamps in stamping order, the set's own left out
        for (int e = s.ccPtr[p]; e < s.ccPtr[p + 1]; e++)
            if (std::find(b.begin(), b.end(), s.ccOwner[e]) == b.end()) { gv += s.ccG[e]; bv += s.ccB[e]; }
        t.cell[(size_t)q * kSetStride + c] = p;
        t.red[(size_t)q * 2 * kSetStride + 2 * c] = gv;
        t.red[(size_t)q * 2 * kSetStride + 2 * c + 1] = bv;
    }
    return q;
}

}  // namespace gs

// gs_oracle.cpp — CPU ORACLE for the gridsim_b200 load-flow path. TEST INFRASTRUCTURE ONLY.
//
// A plain C++17 restatement of GridSim.Core's FP64 sparse polar Newton-Raphson load flow and its N-1
// branch-outage screen, operation for operation where cheap. It exists to check the CUDA engine (tests,
// the smoke check and the CPU-baseline leg of the benchmark); the product never links or calls it.
// Every function cites the reference file:line it follows (paths relative to the GridSim source tree).
//
// Deliberate deviations (documented in the design notes):
//   * sin/cos come from libm, not the reference's fdlibm port (Numerics/DetMath.cs:66-71); the parity
//     target (1e-8) does not need cross-OS bit identity.
//   * the DC power flow of the DC-angle retry assumes the reference bus of a single-island DC model is the
//     case's slack (DistributionFactors picks it as the AC island pre-pass does); other cases get no retry.
#include "../include/gridsim_b200.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <map>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

namespace {

using cplx = std::complex<double>;
constexpr double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------------------------------------
// Model: the GridModel fields the load flow reads (Model/Model.cs:20-35, 91-114, 253-275).
struct Gen {
    int bus;
    double pg, qg, vg, qmin, qmax;
    // machine data, read only by the outage dispatch by governor droop or inertia (ShareLostPower)
    double pmin = 0.0, pmax = std::numeric_limits<double>::infinity(), mbase = 100.0, h = 0.0;
    bool sync = true;  // a synchronous machine with a governor: not power-flow-only, not converter plant
};
struct Br {
    int f, t;
    double r, x, b, tap, shift, rateA;
    bool inService;
    double rateB, rateC;
};
// Boundary (Model/Model.cs:516-560) with its branch names resolved to positions.
struct Bnd {
    double limitMw;
    std::vector<std::pair<int, int>> members;  // (branch position, direction)
};
struct Model {
    int n = 0;
    double base = 100.0;
    std::vector<int> id, type;  // 1 PQ, 2 PV, 3 slack
    std::vector<double> pd, qd, gs, bs, vm, vaDeg, vmin, vmax;
    std::vector<Gen> gens;      // in-service units only (GridModel.Generators)
    std::vector<int> genOfDesc; // descriptor unit -> position in gens (-1: out of service)
    std::vector<Br> br;         // GridModel.Branches order
    std::vector<Bnd> bnd;
    std::vector<double> zip;    // [6 n] Ap Bp Cp Aq Bq Cq per bus (Bus.Zip, Model/Model.cs:33,45-90); empty: none
};

Model FromDesc(const gs_grid_desc* d) {
    Model m;
    m.n = d->n_bus;
    m.base = d->base_mva;
    m.id.assign(d->bus_id, d->bus_id + m.n);
    m.type.assign(d->bus_type, d->bus_type + m.n);
    m.pd.assign(d->pd, d->pd + m.n);
    m.qd.assign(d->qd, d->qd + m.n);
    m.gs.assign(d->gs, d->gs + m.n);
    m.bs.assign(d->bs, d->bs + m.n);
    m.vm.assign(d->vm, d->vm + m.n);
    m.vaDeg.assign(d->va_deg, d->va_deg + m.n);
    const double nan = std::numeric_limits<double>::quiet_NaN();
    m.vmin.assign(m.n, nan);
    m.vmax.assign(m.n, nan);
    if (d->vmin_pu) m.vmin.assign(d->vmin_pu, d->vmin_pu + m.n);
    if (d->vmax_pu) m.vmax.assign(d->vmax_pu, d->vmax_pu + m.n);
    m.genOfDesc.assign(d->n_gen, -1);
    for (int g = 0; g < d->n_gen; g++) {
        if (d->gen_in_service && !d->gen_in_service[g]) continue;
        m.genOfDesc[g] = (int)m.gens.size();
        m.gens.push_back({d->gen_bus[g], d->pg[g], d->qg[g], d->vg[g], d->qmin[g], d->qmax[g]});
    }
    for (int k = 0; k < d->n_branch; k++) {
        m.br.push_back({d->br_from[k], d->br_to[k], d->r[k], d->x[k], d->b[k], d->tap[k], d->shift_deg[k],
                        d->rate_a[k], d->br_in_service ? d->br_in_service[k] != 0 : true,
                        d->rate_b ? d->rate_b[k] : 0.0, d->rate_c ? d->rate_c[k] : 0.0});
    }
    if (d->zip) m.zip.assign(d->zip, d->zip + 6 * (size_t)m.n);
    for (int q = 0; q < d->n_boundary; q++) {
        Bnd b{d->bnd_limit_mw[q], {}};
        for (int e = d->bnd_ptr[q]; e < d->bnd_ptr[q + 1]; e++) b.members.push_back({d->bnd_branch[e], d->bnd_dir[e]});
        m.bnd.push_back(b);
    }
    return m;
}

// Machine data per descriptor unit for the shared outage dispatch (0 reference bus, 1 governor droop, 2 inertia).
struct GsoMachines {
    int32_t dispatch;
    const double *pmin, *pmax, *mbase, *h;
    const uint8_t* sync;
};

void AttachMachines(Model& m, const GsoMachines* mc) {
    for (size_t g = 0; g < m.genOfDesc.size(); g++) {
        const int p = m.genOfDesc[g];
        if (p < 0) continue;
        Gen& u = m.gens[p];
        u.pmin = mc->pmin[g];
        u.pmax = mc->pmax[g];
        u.mbase = mc->mbase[g];
        u.h = mc->h[g];
        u.sync = mc->sync[g] != 0;
    }
}

// ---------------------------------------------------------------------------------------------
// AdmittanceStamp.Branch / FromAdmittance (PowerFlow/AdmittanceStamp.cs:35-76), h = 1.
struct Stamp { cplx yff, ytt, yft, ytf; };
Stamp BranchStamp(double r, double x, double b, double tapRatio, double shiftDeg) {
    cplx ys = cplx(1.0, 0.0) / cplx(r, x);
    cplx bc(0.0, b / 2.0);
    double a = tapRatio == 0 ? 1.0 : tapRatio;
    double shift = shiftDeg * kPi / 180.0;
    cplx tap(a * std::cos(shift), a * std::sin(shift));
    Stamp s;
    s.yff = (ys + bc) / (a * a);
    s.ytt = ys + bc;
    s.yft = -ys / std::conj(tap);
    s.ytf = -ys / tap;
    return s;
}

// ---------------------------------------------------------------------------------------------
// ComplexCsr and its builder (Numerics/Sparse.cs:134-224): insertion order kept per cell (stable by
// column), duplicates summed in that order from +0.0, a zero diagonal injected where none is stamped.
struct ComplexCsr {
    int n = 0;
    std::vector<int> rowPtr, colIdx, diag;
    std::vector<double> G, B;
};
struct ComplexBuilder {
    int n;
    std::vector<int> r, c;
    std::vector<double> g, b;
    explicit ComplexBuilder(int n_) : n(n_) {}
    void Add(int row, int col, double gv, double bv) {
        if (gv == 0.0 && bv == 0.0) return;  // Sparse.cs:151
        r.push_back(row); c.push_back(col); g.push_back(gv); b.push_back(bv);
    }
    ComplexCsr Build() const {
        int nnz = (int)g.size();
        std::vector<int> rowStart(n + 1, 0);
        for (int t = 0; t < nnz; t++) rowStart[r[t] + 1]++;
        for (int i = 0; i < n; i++) rowStart[i + 1] += rowStart[i];
        std::vector<int> col(nnz), fill(rowStart);
        std::vector<double> gv(nnz), bv(nnz);
        for (int t = 0; t < nnz; t++) { int p = fill[r[t]]++; col[p] = c[t]; gv[p] = g[t]; bv[p] = b[t]; }
        ComplexCsr y;
        y.n = n;
        y.rowPtr.assign(n + 1, 0);
        y.diag.assign(n, -1);
        std::vector<int> order;
        for (int i = 0; i < n; i++) {
            int s = rowStart[i], e = rowStart[i + 1];
            order.resize(e - s);
            for (int k = 0; k < e - s; k++) order[k] = s + k;
            std::stable_sort(order.begin(), order.end(), [&](int a, int bb) { return col[a] < col[bb]; });
            y.rowPtr[i] = (int)y.colIdx.size();
            int prev = std::numeric_limits<int>::min();
            bool diagWritten = false;
            for (int o : order) {
                int cc = col[o];
                if (cc == prev) { y.G.back() += gv[o]; y.B.back() += bv[o]; continue; }
                if (!diagWritten && prev < i && cc > i) {
                    y.diag[i] = (int)y.colIdx.size();
                    y.colIdx.push_back(i); y.G.push_back(0); y.B.push_back(0);
                    diagWritten = true;
                }
                y.colIdx.push_back(cc); y.G.push_back(0.0 + gv[o]); y.B.push_back(0.0 + bv[o]);
                prev = cc;
                if (cc == i) { y.diag[i] = (int)y.colIdx.size() - 1; diagWritten = true; }
            }
            if (!diagWritten) {
                y.diag[i] = (int)y.colIdx.size();
                y.colIdx.push_back(i); y.G.push_back(0); y.B.push_back(0);
            }
        }
        y.rowPtr[n] = (int)y.colIdx.size();
        return y;
    }
};

// SparseNewtonRaphsonPowerFlow.BuildY (:382-402). `skip` removes one branch (ScreenOutageCore's
// WithoutMany, ContingencyAnalysis.cs:1839-1845, keeps the remaining branches in model order).
ComplexCsr BuildY(const Model& m, int skip) {
    ComplexBuilder b(m.n);
    for (int k = 0; k < (int)m.br.size(); k++) {
        const Br& br = m.br[k];
        if (k == skip || !br.inService) continue;
        Stamp s = BranchStamp(br.r, br.x, br.b, br.tap, br.shift);
        b.Add(br.f, br.f, s.yff.real(), s.yff.imag());
        b.Add(br.t, br.t, s.ytt.real(), s.ytt.imag());
        b.Add(br.f, br.t, s.yft.real(), s.yft.imag());
        b.Add(br.t, br.f, s.ytf.real(), s.ytf.imag());
    }
    for (int i = 0; i < m.n; i++) {
        if (m.gs[i] == 0 && m.bs[i] == 0) continue;
        b.Add(i, i, m.gs[i] / m.base, m.bs[i] / m.base);
    }
    return b.Build();
}

// ---------------------------------------------------------------------------------------------
// Real CSR with the CsrMatrix.Builder semantics (Numerics/Sparse.cs:33-127).
struct Csr {
    int n = 0;
    std::vector<int> rowPtr, colIdx;
    std::vector<double> val;
};
Csr BuildCsrPattern(int n, const std::vector<std::pair<int, int>>& cells) {
    // Every cell carries the placeholder 1.0, so duplicates only merge; the diagonal is injected where
    // absent (ensureDiagonal, the Build() default).
    std::vector<std::vector<int>> rows(n);
    for (auto& rc : cells) rows[rc.first].push_back(rc.second);
    Csr a;
    a.n = n;
    a.rowPtr.assign(n + 1, 0);
    for (int i = 0; i < n; i++) {
        auto& r = rows[i];
        r.push_back(i);
        std::sort(r.begin(), r.end());
        r.erase(std::unique(r.begin(), r.end()), r.end());
        a.rowPtr[i] = (int)a.colIdx.size();
        for (int c : r) a.colIdx.push_back(c);
    }
    a.rowPtr[n] = (int)a.colIdx.size();
    a.val.assign(a.colIdx.size(), 1.0);
    return a;
}
int Locate(const Csr& a, int row, int col) {  // SparseNewtonRaphsonPowerFlow.Locate (:335-336)
    auto b = a.colIdx.begin() + a.rowPtr[row], e = a.colIdx.begin() + a.rowPtr[row + 1];
    auto it = std::lower_bound(b, e, col);
    return (it != e && *it == col) ? (int)(it - a.colIdx.begin()) : -1;
}

// ---------------------------------------------------------------------------------------------
// MinimumDegreeOrdering.Order (Numerics/MinimumDegreeOrdering.cs:23-121): exact minimum degree on the
// pattern of A + A^T, explicit elimination graph, LIFO bucket queue, initial insertion in descending index.
std::vector<int> MinimumDegree(int n, const std::vector<int>& rowPtr, const std::vector<int>& colIdx) {
    std::vector<int> order(n);
    if (n == 0) return order;
    std::vector<int> cnt(n, 0);
    for (int i = 0; i < n; i++)
        for (int k = rowPtr[i]; k < rowPtr[i + 1]; k++) {
            int j = colIdx[k];
            if (j != i) { cnt[i]++; cnt[j]++; }
        }
    std::vector<std::vector<int>> adj(n);
    for (int i = 0; i < n; i++) adj[i].resize(cnt[i]);
    std::vector<int> len(n, 0);
    for (int i = 0; i < n; i++)
        for (int k = rowPtr[i]; k < rowPtr[i + 1]; k++) {
            int j = colIdx[k];
            if (j == i) continue;
            adj[i][len[i]++] = j;
            adj[j][len[j]++] = i;
        }
    std::vector<int> stamp(n, 0);
    int st = 0;
    for (int i = 0; i < n; i++) {
        st++;
        int w = 0;
        for (int p = 0; p < len[i]; p++) {
            int j = adj[i][p];
            if (stamp[j] != st) { stamp[j] = st; adj[i][w++] = j; }
        }
        len[i] = w;
    }
    std::vector<int> head(n + 1, -1), next(n), prev(n), deg(n);
    auto insert = [&](int v, int d) {
        deg[v] = d; prev[v] = -1; next[v] = head[d];
        if (head[d] >= 0) prev[head[d]] = v;
        head[d] = v;
    };
    auto remove = [&](int v) {
        int d = deg[v];
        if (prev[v] >= 0) next[prev[v]] = next[v]; else head[d] = next[v];
        if (next[v] >= 0) prev[next[v]] = prev[v];
    };
    for (int i = n - 1; i >= 0; i--) insert(i, len[i]);
    std::vector<char> dead(n, 0);
    std::vector<int> nb(n);
    int minDeg = 0;
    for (int s = 0; s < n; s++) {
        while (head[minDeg] < 0) minDeg++;
        int v = head[minDeg];
        remove(v);
        dead[v] = 1;
        order[s] = v;
        int nbCount = 0;
        for (int p = 0; p < len[v]; p++) {
            int u = adj[v][p];
            if (!dead[u]) nb[nbCount++] = u;
        }
        st++;
        for (int t = 0; t < nbCount; t++) stamp[nb[t]] = st;
        int nbStamp = st;
        for (int t = 0; t < nbCount; t++) {
            int u = nb[t];
            remove(u);
            auto& au = adj[u];
            int w = 0;
            for (int p = 0; p < len[u]; p++) {
                int x = au[p];
                if (x != v && !dead[x] && stamp[x] != nbStamp) au[w++] = x;
            }
            int need = w + nbCount - 1;
            if ((int)au.size() < need) au.resize(std::max(need, (int)au.size() * 2));
            for (int q = 0; q < nbCount; q++)
                if (nb[q] != u) au[w++] = nb[q];
            len[u] = w;
            insert(u, w);
        }
        adj[v].clear();
        len[v] = 0;
        if (minDeg > 0) minDeg--;
    }
    return order;
}

// ---------------------------------------------------------------------------------------------
// SparseLuFactorization.Factor (Numerics/SparseLuFactorization.cs:69-195) with SpSolve / Reach / Dfs
// (:753-821): left-looking Gilbert-Peierls LU = P A Q, partial pivoting with the per-row floor
// 1e-12 * max|A(row,:)| (NumericTolerances.cs:36, RowPivotFloorsCsc :99-116). Solve (:338-371).
struct SparseLu {
    int n = 0;
    std::vector<int> lp, li, up, ui, pinv, q;
    std::vector<double> lx, ux;
    std::vector<double> Solve(const std::vector<double>& b) const {
        std::vector<double> x(n), out(n);
        for (int k = 0; k < n; k++) x[pinv[k]] = b[k];
        for (int j = 0; j < n; j++) {
            double xj = x[j];
            for (int p = lp[j] + 1; p < lp[j + 1]; p++) x[li[p]] -= lx[p] * xj;
        }
        for (int j = n - 1; j >= 0; j--) {
            double xj = x[j] / ux[up[j + 1] - 1];
            x[j] = xj;
            for (int p = up[j]; p < up[j + 1] - 1; p++) x[ui[p]] -= ux[p] * xj;
        }
        for (int k = 0; k < n; k++) out[q[k]] = x[k];
        return out;
    }
};

// Returns false when singular (the reference returns null).
bool GpFactor(int n, const std::vector<int>& ap, const std::vector<int>& ai, const std::vector<double>& ax,
              const std::vector<int>& q, SparseLu& F) {
    int nnzA = ap[n];
    double aNorm = 0.0;
    for (int p = 0; p < nnzA; p++) {
        if (std::isnan(ax[p])) return false;  // the reference throws; SolveStep refused non-finite J already
        aNorm = std::max(aNorm, std::fabs(ax[p]));
    }
    if (std::isinf(aNorm)) return false;
    std::vector<double> rowFloor(n, 0.0);
    for (int p = 0; p < nnzA; p++) rowFloor[ai[p]] = std::max(rowFloor[ai[p]], std::fabs(ax[p]));
    for (int r = 0; r < n; r++) rowFloor[r] *= 1e-12;

    F.n = n;
    F.q = q;
    F.lp.assign(n + 1, 0);
    F.up.assign(n + 1, 0);
    F.li.clear(); F.lx.clear(); F.ui.clear(); F.ux.clear();
    F.pinv.assign(n, -1);
    std::vector<double> x(n, 0.0);
    std::vector<int> xi(n), pstack(n);
    std::vector<char> marked(n, 0);

    auto dfs = [&](int j, int top) {
        int head = 0;
        xi[0] = j;
        while (head >= 0) {
            j = xi[head];
            int jcol = F.pinv[j];
            if (!marked[j]) {
                marked[j] = 1;
                pstack[head] = jcol < 0 ? 0 : F.lp[jcol] + 1;
            }
            bool done = true;
            int pend = jcol < 0 ? 0 : F.lp[jcol + 1];
            for (int p = pstack[head]; p < pend; p++) {
                int i = F.li[p];
                if (marked[i]) continue;
                pstack[head] = p + 1;
                xi[++head] = i;
                done = false;
                break;
            }
            if (done) { head--; xi[--top] = j; }
        }
        return top;
    };

    for (int k = 0; k < n; k++) {
        F.lp[k] = (int)F.li.size();
        F.up[k] = (int)F.ui.size();
        int col = q[k];
        // Reach (:783-792)
        int top = n;
        for (int p = ap[col]; p < ap[col + 1]; p++) {
            int j = ai[p];
            if (!marked[j]) top = dfs(j, top);
        }
        for (int p = top; p < n; p++) marked[xi[p]] = 0;
        // SpSolve (:753-780)
        for (int p = top; p < n; p++) x[xi[p]] = 0.0;
        for (int p = ap[col]; p < ap[col + 1]; p++) x[ai[p]] = ax[p];
        for (int px = top; px < n; px++) {
            int j = xi[px];
            int jcol = F.pinv[j];
            if (jcol < 0) continue;
            double xj = x[j];
            for (int p = F.lp[jcol] + 1; p < F.lp[jcol + 1]; p++) x[F.li[p]] -= F.lx[p] * xj;
        }
        // partial pivot (:129-162)
        int ipiv = -1;
        double best = -1.0;
        for (int px = top; px < n; px++) {
            int i = xi[px];
            if (F.pinv[i] < 0) {
                double t = std::fabs(x[i]);
                if (t > best) { best = t; ipiv = i; }
            } else {
                F.ui.push_back(F.pinv[i]);
                F.ux.push_back(x[i]);
            }
        }
        if (ipiv < 0 || best <= rowFloor[ipiv]) return false;
        double pivot = x[ipiv];
        F.ui.push_back(k); F.ux.push_back(pivot);
        F.pinv[ipiv] = k;
        F.li.push_back(ipiv); F.lx.push_back(1.0);
        for (int px = top; px < n; px++) {
            int i = xi[px];
            if (F.pinv[i] < 0) { F.li.push_back(i); F.lx.push_back(x[i] / pivot); }
            x[i] = 0.0;
        }
    }
    F.lp[n] = (int)F.li.size();
    F.up[n] = (int)F.ui.size();
    for (auto& r : F.li) r = F.pinv[r];
    return true;
}

// CpuSparseLuSolver (PowerFlow/CpuSparseLuSolver.cs:30-48): MD ordering cached by CSR pattern, then
// SparseLu.ToCsc that DROPS exact zeros (Numerics/SparseLu.cs:63-91), then the factorisation.
struct CpuSparseLuSolver {
    std::vector<int> q, rowPtr, colIdx;
    bool Solve(const Csr& a, const std::vector<double>& b, std::vector<double>& x) {
        int n = a.n;
        if (q.empty() || rowPtr != a.rowPtr || colIdx != a.colIdx) {
            q = MinimumDegree(n, a.rowPtr, a.colIdx);
            rowPtr = a.rowPtr;
            colIdx = a.colIdx;
        }
        std::vector<int> ap(n + 1, 0);
        for (size_t k = 0; k < a.colIdx.size(); k++)
            if (a.val[k] != 0.0) ap[a.colIdx[k] + 1]++;
        for (int c = 0; c < n; c++) ap[c + 1] += ap[c];
        std::vector<int> ai(ap[n]), fill(ap.begin(), ap.end() - 1);
        std::vector<double> ax(ap[n]);
        for (int i = 0; i < n; i++)
            for (int k = a.rowPtr[i]; k < a.rowPtr[i + 1]; k++) {
                double v = a.val[k];
                if (v == 0.0) continue;
                int dst = fill[a.colIdx[k]]++;
                ai[dst] = i;
                ax[dst] = v;
            }
        SparseLu F;
        if (!GpFactor(n, ap, ai, ax, q, F)) return false;
        for (double v : b)
            if (!std::isfinite(v)) return false;
        x = F.Solve(b);
        return true;
    }
};

// ---------------------------------------------------------------------------------------------
// The SolveStep fallback when the sparse LU reports singular (NewtonShell.cs:100-105): ILU(0) with the
// row-relative pivot guard (Numerics/Sparse.cs:232-300, NumericTolerances.Ilu0PivotGuard :226-234) and
// ILU-preconditioned BiCGSTAB with the true-residual acceptance (Sparse.cs:305-405), tolerance
// min(1e-10, tol*1e-3) and cap 4m + 200 (NumericTolerances.cs:256-260).
void CsrMultiply(const Csr& a, const std::vector<double>& x, std::vector<double>& y) {
    for (int i = 0; i < a.n; i++) {
        double s = 0;
        for (int k = a.rowPtr[i]; k < a.rowPtr[i + 1]; k++) s += a.val[k] * x[a.colIdx[k]];
        y[i] = s;
    }
}
struct Ilu0 {
    const Csr* a = nullptr;
    std::vector<double> lu;
    std::vector<int> diag;
    void Factor(const Csr& A) {
        a = &A;
        int n = A.n;
        diag.assign(n, -1);
        for (int i = 0; i < n; i++)
            for (int k = A.rowPtr[i]; k < A.rowPtr[i + 1]; k++)
                if (A.colIdx[k] == i) diag[i] = k;
        lu = A.val;
        std::vector<int> iw(n, -1);
        for (int i = 0; i < n; i++) {
            for (int k = A.rowPtr[i]; k < A.rowPtr[i + 1]; k++) iw[A.colIdx[k]] = k;
            for (int k = A.rowPtr[i]; k < diag[i]; k++) {
                int j = A.colIdx[k];
                double piv = lu[diag[j]];
                double lij = (piv != 0.0) ? lu[k] / piv : 0.0;
                lu[k] = lij;
                if (lij == 0.0) continue;
                for (int kk = diag[j] + 1; kk < A.rowPtr[j + 1]; kk++) {
                    int pos = iw[A.colIdx[kk]];
                    if (pos != -1) lu[pos] -= lij * lu[kk];
                }
            }
            double rowScale = 0.0;
            for (int k = A.rowPtr[i]; k < A.rowPtr[i + 1]; k++) rowScale = std::max(rowScale, std::fabs(A.val[k]));
            double guard = 1e-12 * (rowScale > 0.0 ? rowScale : 1.0);
            double d = lu[diag[i]];
            if (std::fabs(d) < guard) lu[diag[i]] = d < 0 ? -guard : guard;
            for (int k = A.rowPtr[i]; k < A.rowPtr[i + 1]; k++) iw[A.colIdx[k]] = -1;
        }
    }
    void Apply(const std::vector<double>& r, std::vector<double>& z) const {
        int n = a->n;
        for (int i = 0; i < n; i++) {
            double s = r[i];
            for (int k = a->rowPtr[i]; k < diag[i]; k++) s -= lu[k] * z[a->colIdx[k]];
            z[i] = s;
        }
        for (int i = n - 1; i >= 0; i--) {
            double s = z[i];
            for (int k = diag[i] + 1; k < a->rowPtr[i + 1]; k++) s -= lu[k] * z[a->colIdx[k]];
            z[i] = s / lu[diag[i]];
        }
    }
};
double Dot(const std::vector<double>& a, const std::vector<double>& b) {
    double s = 0;
    for (size_t i = 0; i < a.size(); i++) s += a[i] * b[i];
    return s;
}
bool BiCgStab(const Csr& a, const std::vector<double>& b, std::vector<double>& x, const Ilu0& pc, double tol,
              int maxIter) {
    int n = a.n;
    x.assign(n, 0.0);
    std::vector<double> r = b, rhat = b, p(n, 0), v(n, 0), s(n), t(n), ph(n), sh(n);
    double bnorm = std::sqrt(Dot(b, b));
    if (bnorm == 0) {
        for (double bi : b) if (bi != 0.0) return false;
        return true;
    }
    auto trueResidual = [&]() {
        CsrMultiply(a, x, t);
        double sum = 0;
        for (int i = 0; i < n; i++) { double d = b[i] - t[i]; sum += d * d; }
        return std::sqrt(sum) / bnorm < tol;
    };
    double rho = 1, alpha = 1, omega = 1;
    const double underflowGuard = 1e-300;
    for (int it = 0; it < maxIter; it++) {
        double rhoNew = Dot(rhat, r);
        if (std::fabs(rhoNew) < underflowGuard || std::isnan(rhoNew)) return false;
        double beta = (rhoNew / rho) * (alpha / omega);
        for (int i = 0; i < n; i++) p[i] = r[i] + beta * (p[i] - omega * v[i]);
        pc.Apply(p, ph);
        CsrMultiply(a, ph, v);
        double rhatV = Dot(rhat, v);
        if (rhatV == 0.0 || std::isnan(rhatV)) return false;
        alpha = rhoNew / rhatV;
        for (int i = 0; i < n; i++) s[i] = r[i] - alpha * v[i];
        if (std::sqrt(Dot(s, s)) / bnorm < tol) {
            for (int i = 0; i < n; i++) x[i] += alpha * ph[i];
            return trueResidual();
        }
        pc.Apply(s, sh);
        CsrMultiply(a, sh, t);
        double tt = Dot(t, t);
        omega = tt > 0 ? Dot(t, s) / tt : 0.0;
        for (int i = 0; i < n; i++) { x[i] += alpha * ph[i] + omega * sh[i]; r[i] = s[i] - omega * t[i]; }
        rho = rhoNew;
        if (std::sqrt(Dot(r, r)) / bnorm < tol) return trueResidual();
        if (omega == 0) return false;
    }
    return false;
}

// ---------------------------------------------------------------------------------------------
// NewtonShell.BuildBusSpec (PowerFlow/NewtonShell.cs:433-486).
struct BusSpec {
    std::vector<int> type0;  // 1 PQ, 2 PV, 3 slack
    std::vector<double> vm, va, pspec, qspec, qd, qmin, qmax, vg;
    // voltage-dependent loads (BuildBusSpec :482): per bus its ZIP coefficients when they vary with voltage
    // (ZipLoad.VariesWithVoltage), and the nominal load Pd, Qd (MW, MVAr) they scale
    std::vector<char> hasZip;
    std::vector<double> zip, pd;
    bool anyZip = false;
};

// ZipLoad.PMultiplier / QMultiplier / DPMultiplier / DQMultiplier (Model/Model.cs:51-63)
inline double ZipMult(const double* c, double v) { return c[0] * v * v + c[1] * v + c[2]; }
inline double ZipDMult(const double* c, double v) { return 2 * c[0] * v + c[1]; }
BusSpec BuildBusSpec(const Model& m, bool flatStart) {
    int n = m.n;
    BusSpec s;
    std::vector<double> pg(n, 0), qg(n, 0), vg(n, 0);
    std::vector<char> hasGen(n, 0);
    s.qmin.assign(n, 0); s.qmax.assign(n, 0);
    for (const Gen& g : m.gens) {
        pg[g.bus] += g.pg;
        qg[g.bus] += g.qg;
        s.qmin[g.bus] += g.qmin;
        s.qmax[g.bus] += g.qmax;
        vg[g.bus] = g.vg;  // the last generator at the bus wins (:448)
        hasGen[g.bus] = 1;
    }
    s.type0.resize(n); s.vm.resize(n); s.va.resize(n); s.pspec.resize(n); s.qspec.resize(n);
    s.qd = m.qd;
    s.pd = m.pd;
    s.vg = vg;
    s.hasZip.assign(n, 0);
    s.zip.assign(6 * (size_t)n, 0.0);
    if (!m.zip.empty())
        for (int i = 0; i < n; i++) {
            const double* c = &m.zip[6 * (size_t)i];
            if (c[0] != 0 || c[1] != 0 || c[3] != 0 || c[4] != 0) {  // VariesWithVoltage
                s.hasZip[i] = 1;
                s.anyZip = true;
                std::copy(c, c + 6, s.zip.begin() + 6 * (size_t)i);
            }
        }
    for (int i = 0; i < n; i++) {
        s.type0[i] = (m.type[i] == 2 && !hasGen[i]) ? 1 : m.type[i];
        bool vc = s.type0[i] == 3 || s.type0[i] == 2;
        s.vm[i] = (vc && hasGen[i]) ? vg[i] : (s.type0[i] == 3 ? m.vm[i] : (flatStart ? 1.0 : m.vm[i]));
        s.va[i] = m.type[i] == 3 ? m.vaDeg[i] * kPi / 180.0 : (flatStart ? 0.0 : m.vaDeg[i] * kPi / 180.0);
        s.pspec[i] = (pg[i] - m.pd[i]) / m.base;
        s.qspec[i] = (qg[i] - m.qd[i]) / m.base;
    }
    return s;
}

// NewtonShell.EquationPositions (:327-336).
int EquationPositions(const std::vector<int>& type, std::vector<int>& pPos, std::vector<int>& qPos) {
    int n = (int)type.size();
    pPos.assign(n, -1);
    qPos.assign(n, -1);
    int m = 0;
    for (int i = 0; i < n; i++) if (type[i] != 3) pPos[i] = m++;
    for (int i = 0; i < n; i++) if (type[i] == 1) qPos[i] = m++;
    return m;
}

// SparseNewtonRaphsonPowerFlow.ComputeInjections (:269-289).
void ComputeInjections(const ComplexCsr& y, const std::vector<double>& Vm, const std::vector<double>& Va,
                       std::vector<double>& P, std::vector<double>& Q) {
    for (int i = 0; i < y.n; i++) {
        double pi = 0, qi = 0, vai = Va[i];
        for (int k = y.rowPtr[i]; k < y.rowPtr[i + 1]; k++) {
            int j = y.colIdx[k];
            double th = vai - Va[j];
            double sn = std::sin(th), cs = std::cos(th);
            double vmj = Vm[j];
            pi += vmj * (y.G[k] * cs + y.B[k] * sn);
            qi += vmj * (y.G[k] * sn - y.B[k] * cs);
        }
        P[i] = Vm[i] * pi;
        Q[i] = Vm[i] * qi;
    }
}

// BuildJacobianStructure (:296-332).
Csr BuildJacobianStructure(const ComplexCsr& y, const std::vector<int>& pPos, const std::vector<int>& qPos, int m,
                           std::vector<int>& slots) {
    std::vector<std::pair<int, int>> cells;
    for (int i = 0; i < y.n; i++) {
        int pi = pPos[i], qi = qPos[i];
        if (pi < 0 && qi < 0) continue;
        for (int k = y.rowPtr[i]; k < y.rowPtr[i + 1]; k++) {
            int j = y.colIdx[k], pj = pPos[j], qj = qPos[j];
            if (pi >= 0 && pj >= 0) cells.push_back({pi, pj});
            if (pi >= 0 && qj >= 0) cells.push_back({pi, qj});
            if (qi >= 0 && pj >= 0) cells.push_back({qi, pj});
            if (qi >= 0 && qj >= 0) cells.push_back({qi, qj});
        }
    }
    Csr jac = BuildCsrPattern(m, cells);
    slots.assign(4 * y.rowPtr[y.n], -1);
    for (int i = 0; i < y.n; i++) {
        int pi = pPos[i], qi = qPos[i];
        for (int k = y.rowPtr[i]; k < y.rowPtr[i + 1]; k++) {
            int j = y.colIdx[k], pj = pPos[j], qj = qPos[j];
            slots[4 * k + 0] = (pi >= 0 && pj >= 0) ? Locate(jac, pi, pj) : -1;
            slots[4 * k + 1] = (pi >= 0 && qj >= 0) ? Locate(jac, pi, qj) : -1;
            slots[4 * k + 2] = (qi >= 0 && pj >= 0) ? Locate(jac, qi, pj) : -1;
            slots[4 * k + 3] = (qi >= 0 && qj >= 0) ? Locate(jac, qi, qj) : -1;
        }
    }
    return jac;
}

// RefillJacobian (:342-380).
void RefillJacobian(Csr& jac, const std::vector<int>& slots, const ComplexCsr& y, const std::vector<double>& Vm,
                    const std::vector<double>& Va, const std::vector<double>& P, const std::vector<double>& Q) {
    std::fill(jac.val.begin(), jac.val.end(), 0.0);
    for (int i = 0; i < y.n; i++) {
        for (int k = y.rowPtr[i]; k < y.rowPtr[i + 1]; k++) {
            int j = y.colIdx[k];
            double Gij = y.G[k], Bij = y.B[k];
            double H, N, M, L;
            if (i == j) {
                H = -Q[i] - Bij * Vm[i] * Vm[i];
                N = P[i] / Vm[i] + Gij * Vm[i];
                M = P[i] - Gij * Vm[i] * Vm[i];
                L = Q[i] / Vm[i] - Bij * Vm[i];
            } else {
                double th = Va[i] - Va[j];
                double sn = std::sin(th), cs = std::cos(th);
                H = Vm[i] * Vm[j] * (Gij * sn - Bij * cs);
                N = Vm[i] * (Gij * cs + Bij * sn);
                M = -Vm[i] * Vm[j] * (Gij * cs + Bij * sn);
                L = Vm[i] * (Gij * sn - Bij * cs);
            }
            int s;
            if ((s = slots[4 * k + 0]) >= 0) jac.val[s] = H;
            if ((s = slots[4 * k + 1]) >= 0) jac.val[s] = N;
            if ((s = slots[4 * k + 2]) >= 0) jac.val[s] = M;
            if ((s = slots[4 * k + 3]) >= 0) jac.val[s] = L;
        }
    }
}

constexpr double kMaxUndampedStep = 0.4;  // NewtonShell.cs:38
constexpr double kVmFloorPu = 0.01;       // NewtonShell.cs:48
constexpr double kQLimitTolMva = 1e-3;    // NewtonShell.cs:26
constexpr double kRevertVoltTolPu = 1e-4; // NewtonShell.cs:31

// How a Newton run ended (NewtonShell.NewtonRunEnd, NewtonShell.cs:170-174): its start mismatch, the mismatch it
// took its last step from, its steps and whether the iteration cap stopped it.
struct RunEnd {
    bool converged = false, diverged = false, capReached = false;
    int iters = 0;
    double maxMis = INFINITY, startMis = NAN, beforeLast = NAN;
};

// RunNewton (:168-265) with NewtonShell.SolveStep (:74-120) and ApplyStep (:128-136).
// ZIP loads (zs non-null with anyZip): the deviation of each load from its nominal value at the present voltage comes off
// the mismatch (:223-231, NewtonShell.ZipDeviationPu :396-402), its derivative onto the N and L diagonals of buses
// with a voltage column (:241-248, NewtonShell.ZipJacobianDiagPu :407-413).
RunEnd RunNewton(CpuSparseLuSolver& solver, const ComplexCsr& y, const std::vector<int>& type, std::vector<double>& Vm,
                 std::vector<double>& Va, const std::vector<double>& Pspec, const std::vector<double>& Qspec,
                 std::vector<double>& P, std::vector<double>& Q, const gs_pf_opts& opt, const BusSpec* zs = nullptr,
                 double base = 100.0) {
    const bool zip = zs && zs->anyZip;
    int n = y.n;
    std::vector<int> pPos, qPos;
    int m = EquationPositions(type, pPos, qPos);
    std::vector<double> f(m), dx(m);
    std::vector<int> slots;
    Csr jac = BuildJacobianStructure(y, pPos, qPos, m, slots);
    RunEnd r;
    double startMis = NAN;
    int iter = 0;
    for (;; iter++) {
        ComputeInjections(y, Vm, Va, P, Q);
        for (int i = 0; i < n; i++) {
            if (pPos[i] >= 0) f[pPos[i]] = Pspec[i] - P[i];
            if (qPos[i] >= 0) f[qPos[i]] = Qspec[i] - Q[i];
        }
        if (zip)
            for (int i = 0; i < n; i++) {
                if (!zs->hasZip[i]) continue;
                const double* c = &zs->zip[6 * (size_t)i];
                if (pPos[i] >= 0) f[pPos[i]] -= zs->pd[i] * (ZipMult(c, Vm[i]) - 1.0) / base;
                if (qPos[i] >= 0) f[qPos[i]] -= zs->qd[i] * (ZipMult(c + 3, Vm[i]) - 1.0) / base;
            }
        double maxMis = 0;
        for (int k = 0; k < m; k++) maxMis = std::max(maxMis, std::fabs(f[k]));
        // Math.Max propagates NaN; std::max does not: restate the .NET rule explicitly.
        for (int k = 0; k < m; k++) if (std::isnan(f[k])) maxMis = NAN;
        r.maxMis = maxMis;
        if (iter == 0) startMis = maxMis;
        if (maxMis < opt.tolerance) { r.converged = true; break; }
        // NewtonShell.DivergedBeyondLimit (:177-178): Math.Max propagates a NaN, which then compares false.
        double lim = std::isnan(startMis) ? NAN : std::max(opt.diverge_limit_pu, startMis);
        if (maxMis > lim) { r.diverged = true; break; }
        if (iter >= opt.max_iterations) break;
        RefillJacobian(jac, slots, y, Vm, Va, P, Q);
        if (zip)
            for (int i = 0; i < n; i++) {
                if (qPos[i] < 0 || !zs->hasZip[i]) continue;
                const double* c = &zs->zip[6 * (size_t)i];
                if (pPos[i] >= 0) jac.val[Locate(jac, pPos[i], qPos[i])] += zs->pd[i] * ZipDMult(c, Vm[i]) / base;
                jac.val[Locate(jac, qPos[i], qPos[i])] += zs->qd[i] * ZipDMult(c + 3, Vm[i]) / base;
            }
        bool ok = true;
        for (double v : jac.val) if (!std::isfinite(v)) { ok = false; break; }
        if (ok) for (double v : f) if (!std::isfinite(v)) { ok = false; break; }
        std::vector<double> sol;
        if (!ok) break;
        if (!solver.Solve(jac, f, sol)) {
            Ilu0 pc;
            pc.Factor(jac);
            if (!BiCgStab(jac, f, sol, pc, std::min(1e-10, opt.tolerance * 1e-3), 4 * m + 200)) break;
        }
        double maxAbs = 0;
        for (int k = 0; k < m; k++) {
            if (!std::isfinite(sol[k])) { ok = false; break; }
            maxAbs = std::max(maxAbs, std::fabs(sol[k]));
        }
        if (!ok) break;
        r.beforeLast = maxMis;  // the retry's stall test only (SparseNewtonRaphsonPowerFlow.cs:259)
        dx = sol;
        double damp = maxAbs > kMaxUndampedStep ? kMaxUndampedStep / maxAbs : 1.0;
        for (int i = 0; i < n; i++) {
            if (pPos[i] >= 0) Va[i] += damp * dx[pPos[i]];
            if (qPos[i] >= 0) { Vm[i] += damp * dx[qPos[i]]; if (Vm[i] < kVmFloorPu) Vm[i] = kVmFloorPu; }
        }
    }
    r.iters = iter;
    r.startMis = startMis;
    r.capReached = !r.converged && !r.diverged && iter >= opt.max_iterations;
    return r;
}

enum QPin { kPinNone = 0, kPinMax = 1, kPinMin = -1, kPinFixed = 2 };

// NewtonShell.TryRevertPin (:563-576).
bool TryRevertPin(int i, std::vector<int>& eff, std::vector<double>& vm, const std::vector<double>& vg,
                  std::vector<int>& pinned, std::vector<int>& revertCount) {
    if (pinned[i] == kPinNone || pinned[i] == kPinFixed || revertCount[i] >= 1) return false;
    bool rMax = pinned[i] == kPinMax && vm[i] > vg[i] + kRevertVoltTolPu;
    bool rMin = pinned[i] == kPinMin && vm[i] < vg[i] - kRevertVoltTolPu;
    if (!(rMax || rMin)) return false;
    eff[i] = 2;
    vm[i] = vg[i];
    pinned[i] = kPinNone;
    revertCount[i]++;
    return true;
}

// NewtonShell.ApplyQLimits (:519-558), revert off by default; the generators' output is the net injection plus the
// load drawn at the solved voltage (LoadAtVoltage.QMvar, :533-537 and PowerFlow/LoadAtVoltage.cs:29-30).
bool ApplyQLimits(const BusSpec& s, std::vector<int>& eff, const std::vector<double>& Q, std::vector<double>& qspec,
                  double base, std::vector<double>& vm, std::vector<int>& pinned, std::vector<int>& revertCount,
                  bool revert) {
    bool changed = false;
    for (size_t i = 0; i < eff.size(); i++) {
        if (s.type0[i] != 2) continue;
        if (eff[i] == 2) {
            double qGen = Q[i] * base + (s.hasZip[i] ? s.qd[i] * ZipMult(&s.zip[6 * i + 3], vm[i]) : s.qd[i]);
            if (qGen > s.qmax[i] + kQLimitTolMva) {
                eff[i] = 1;
                qspec[i] = (s.qmax[i] - s.qd[i]) / base;
                pinned[i] = s.qmin[i] == s.qmax[i] ? kPinFixed : kPinMax;
                changed = true;
            } else if (qGen < s.qmin[i] - kQLimitTolMva) {
                eff[i] = 1;
                qspec[i] = (s.qmin[i] - s.qd[i]) / base;
                pinned[i] = s.qmin[i] == s.qmax[i] ? kPinFixed : kPinMin;
                changed = true;
            }
        } else if (revert) {
            if (TryRevertPin((int)i, eff, vm, s.vg, pinned, revertCount)) changed = true;
        }
    }
    return changed;
}

// RevertBrokenPins (:593-603).
bool RevertBrokenPins(const BusSpec& s, std::vector<int>& eff, std::vector<double>& vm, std::vector<int>& pinned,
                      std::vector<int>& revertCount) {
    bool changed = false;
    for (size_t i = 0; i < eff.size(); i++) {
        if (s.type0[i] != 2 || eff[i] != 1) continue;
        if (TryRevertPin((int)i, eff, vm, s.vg, pinned, revertCount)) changed = true;
    }
    return changed;
}

struct SolveOut {
    int status = GS_PF_NOT_RUN;
    int iterations = 0;
    double maxMis = NAN;
    std::vector<double> vm, va, p, q;  // va in radians; p, q in pu
    bool available = true;    // false: the DC-angle start could not be formed (nothing was solved)
    bool newtonFailed = false;  // the last Newton run did not converge (the retry's trigger)
    RunEnd runEnd;            // how that run ended
};

// DcPowerFlow.Solve on DcDemand.LegacyView (Analysis/DcPowerFlow.cs:40-51, DcDemand.cs:36-50): every tap 1, no
// phase shift, no Gs; B' from b = 1/x of the in-service branches with non-zero reactance (the outaged one removed);
// injections sum(Pg) - Pd; the slack is the single island's reference. Returns false (no angles) unless the DC
// model is one island, or when B' is singular.
bool DcAngles(const Model& m, int skip, int slack, std::vector<double>& thetaDeg) {
    const int n = m.n;
    std::vector<int> parent(n);
    std::iota(parent.begin(), parent.end(), 0);
    std::function<int(int)> find = [&](int a) { return parent[a] == a ? a : parent[a] = find(parent[a]); };
    std::vector<std::pair<int, int>> cells;
    std::vector<double> vals;
    std::vector<int> red(n, -1);
    int nr = 0;
    for (int i = 0; i < n; i++) if (i != slack) red[i] = nr++;
    std::map<std::pair<int, int>, double> acc;
    for (int k = 0; k < (int)m.br.size(); k++) {
        const Br& br = m.br[k];
        if (!br.inService || k == skip || br.x == 0.0) continue;
        parent[find(br.f)] = find(br.t);
        const double b = 1.0 / br.x;
        const int f = red[br.f], t = red[br.t];
        if (f >= 0) acc[{f, f}] += b;
        if (t >= 0) acc[{t, t}] += b;
        if (f >= 0 && t >= 0) { acc[{f, t}] -= b; acc[{t, f}] -= b; }
    }
    int islands = 0;
    for (int i = 0; i < n; i++) if (find(i) == i) islands++;
    if (islands != 1 || nr == 0) return false;
    Csr a;
    a.n = nr;
    a.rowPtr.assign(nr + 1, 0);
    for (auto& kv : acc) a.rowPtr[kv.first.first + 1]++;
    for (int r = 0; r < nr; r++) a.rowPtr[r + 1] += a.rowPtr[r];
    for (auto& kv : acc) { a.colIdx.push_back(kv.first.second); a.val.push_back(kv.second); }  // map order: row-major
    std::vector<double> pinj(n, 0.0), rhs(nr), th;
    for (const Gen& g : m.gens) pinj[g.bus] += g.pg;
    for (int i = 0; i < n; i++) if (red[i] >= 0) rhs[red[i]] = (pinj[i] - m.pd[i]) / m.base;
    CpuSparseLuSolver solver;
    if (!solver.Solve(a, rhs, th)) return false;
    thetaDeg.assign(n, 0.0);
    for (int i = 0; i < n; i++) if (red[i] >= 0) thetaDeg[i] = th[red[i]] * 180.0 / kPi;
    return true;
}

// NewtonShell.TrySeedDcAngles (:282-299): every non-slack start angle from the DC power flow, reduced to
// [-180, 180] degrees, offset by the slack's own start angle; magnitudes unchanged. False: no single slack, or no
// single-island DC model.
bool TrySeedDcAngles(const Model& m, int skip, BusSpec& s) {
    int slack = -1, slacks = 0;
    for (int i = 0; i < m.n; i++) if (s.type0[i] == 3) { slack = i; slacks++; }
    if (slacks != 1) return false;
    std::vector<double> th;
    if (!DcAngles(m, skip, slack, th)) return false;
    const double va0 = s.va[slack];
    for (int i = 0; i < m.n; i++)
        if (i != slack) s.va[i] = va0 + std::remainder(th[i], 360.0) * kPi / 180.0;
    return true;
}

constexpr double kRetryStallFactor = 1e-3;        // NewtonShell.cs:146
constexpr double kRetryLastStepFactor = 0.5;      // NewtonShell.cs:167
constexpr double kMaxRetryBranchAngleDeg = 90.0;  // NewtonShell.cs:142

// NewtonShell.Stalled (:162, :200-206): a run that did not converge stalled (or diverged) rather than being cut off
// by the iteration cap while still converging.
bool Stalled(const RunEnd& r, double finalMis) {
    if (r.capReached && r.iters == 0) return false;
    if (finalMis <= kRetryStallFactor * r.startMis) return false;  // a NaN on either side counts as stalled
    if (r.capReached && r.iters >= 2 && finalMis <= kRetryLastStepFactor * r.beforeLast) return false;
    return true;
}

// NewtonShell.MaxBranchAngleDeg: the largest angle across an in-service branch, net of its phase shift, wrapped
// to [-180, 180] degrees.
double MaxBranchAngleDeg(const Model& m, int skip, const std::vector<double>& vaRad) {
    double mx = 0.0;
    for (int k = 0; k < (int)m.br.size(); k++) {
        const Br& br = m.br[k];
        if (!br.inService || k == skip) continue;
        const double a = std::fabs(std::remainder((vaRad[br.f] - vaRad[br.t]) * 180.0 / kPi - br.shift, 360.0));
        mx = std::max(mx, a);
    }
    return mx;
}

// SparseNewtonRaphsonPowerFlow.SolveAcAttempt (:69-166) + NewtonShell.AssembleResult status (:649-693).
// `vmStart/vaStart` (radians) replace the model's stored start when given (warm start, GridScenario.cs:35-52).
SolveOut SolveModel(const Model& m, int skip, const gs_pf_opts& opt, const double* vmStart, const double* vaStartRad,
                    bool dcStart = false) {
    int n = m.n;
    ComplexCsr y = BuildY(m, skip);
    Model mm;  // only the start values can differ
    const Model* src = &m;
    if (vmStart) {
        mm = m;
        for (int i = 0; i < n; i++) { mm.vm[i] = vmStart[i]; mm.vaDeg[i] = vaStartRad[i] * 180.0 / kPi; }
        src = &mm;
    }
    BusSpec s = BuildBusSpec(*src, opt.flat_start != 0);
    if (vmStart) {  // keep the radian start exactly (the degree round trip is not needed)
        for (int i = 0; i < n; i++)
            if (src->type[i] != 3 && !opt.flat_start) s.va[i] = vaStartRad[i];
    }
    if (dcStart && !TrySeedDcAngles(m, skip, s)) {
        SolveOut none;
        none.available = false;
        return none;
    }
    std::vector<int> eff = s.type0, pinned(n, kPinNone), revertCount(n, 0);
    std::vector<double> Vm = s.vm, Va = s.va, P(n), Q(n), qspec = s.qspec;
    CpuSparseLuSolver solver;
    bool converged = false;
    int total = 0;
    RunEnd re;
    // PowerFlowOptions.MaxQLimitPasses (:101, default 100) and RevertQLimits (:110, default off)
    int qPasses = opt.enforce_q_limits ? (opt.max_q_limit_passes > 0 ? opt.max_q_limit_passes : 100) : 1;
    bool switchPending = false;
    for (int qp = 0; qp < qPasses; qp++) {
        switchPending = false;
        re = RunNewton(solver, y, eff, Vm, Va, s.pspec, qspec, P, Q, opt, &s, m.base);
        converged = re.converged;
        total += re.iters;
        if (!opt.enforce_q_limits) break;
        if (!converged) break;
        bool changed = ApplyQLimits(s, eff, Q, qspec, m.base, Vm, pinned, revertCount, opt.revert_q_limits != 0);
        if (!changed) changed = RevertBrokenPins(s, eff, Vm, pinned, revertCount);
        switchPending = changed;
        if (!changed) break;
    }
    if (switchPending) {
        re = RunNewton(solver, y, eff, Vm, Va, s.pspec, qspec, P, Q, opt, &s, m.base);
        total += re.iters;
        converged = false;
    }
    const bool newtonFailed = !re.converged;
    ComputeInjections(y, Vm, Va, P, Q);
    SolveOut o;
    bool finite = std::isfinite(re.maxMis);
    for (int i = 0; i < n; i++)
        finite = finite && std::isfinite(Vm[i]) && std::isfinite(Va[i]) && std::isfinite(P[i] * m.base) &&
                 std::isfinite(Q[i] * m.base);
    o.status = !finite ? GS_PF_NON_FINITE
             : converged ? GS_PF_CONVERGED
             : (!converged && re.diverged) ? GS_PF_DIVERGED
             : GS_PF_MAX_ITERATIONS;
    o.iterations = total;
    o.maxMis = re.maxMis;
    o.newtonFailed = newtonFailed;
    o.runEnd = re;
    o.vm = Vm; o.va = Va; o.p = P; o.q = Q;
    return o;
}

// NewtonShell.SolveWithRetry (:227-268): the ordinary solve; when its last Newton run failed to converge and stalled
// (and the option is on, with a cap above 1), the solve again from DC power-flow angles, kept only if it converges
// with every branch angle within 90 degrees.
SolveOut SolveWithRetry(const Model& m, int skip, const gs_pf_opts& opt, const double* vmStart, const double* vaStartRad) {
    SolveOut first = SolveModel(m, skip, opt, vmStart, vaStartRad, false);
    if (first.status == GS_PF_CONVERGED || !first.newtonFailed || !opt.retry_from_dc_start || opt.max_iterations <= 1 ||
        !Stalled(first.runEnd, first.maxMis))
        return first;
    SolveOut retry = SolveModel(m, skip, opt, vmStart, vaStartRad, true);
    if (!retry.available) return first;
    if (retry.status == GS_PF_CONVERGED && MaxBranchAngleDeg(m, skip, retry.va) <= kMaxRetryBranchAngleDeg) return retry;
    return first;
}

// NewtonShell.ComputeLineFlows (:699-734): per-branch complex flows (MVA) and loading %.
void LineFlows(const Model& m, int skip, const std::vector<double>& vm, const std::vector<double>& va,
               double* loading, double* sf, double* st) {
    for (int k = 0; k < (int)m.br.size(); k++) {
        const Br& br = m.br[k];
        if (k == skip || !br.inService) {
            if (loading) loading[k] = 0;
            if (sf) { sf[2 * k] = 0; sf[2 * k + 1] = 0; }
            if (st) { st[2 * k] = 0; st[2 * k + 1] = 0; }
            continue;
        }
        cplx vf = std::polar(vm[br.f], va[br.f]);
        cplx vt = std::polar(vm[br.t], va[br.t]);
        Stamp s = BranchStamp(br.r, br.x, br.b, br.tap, br.shift);
        cplx iF = s.yff * vf + s.yft * vt;
        cplx iT = s.ytf * vf + s.ytt * vt;
        cplx sF = vf * std::conj(iF) * m.base;
        cplx sT = vt * std::conj(iT) * m.base;
        double mva = std::max(std::abs(sF), std::abs(sT));
        if (loading) loading[k] = br.rateA > 0 ? mva / br.rateA * 100.0 : 0.0;
        if (sf) { sf[2 * k] = sF.real(); sf[2 * k + 1] = sF.imag(); }
        if (st) { st[2 * k] = sT.real(); st[2 * k + 1] = sT.imag(); }
    }
}

struct Violation { int kind, element; double value; };

// ContingencyAnalysis.ScreenStateCore (:1105-1238), converged branch: thermal (:1150-1180, keyed by the
// ORIGINAL branch index, threshold 100 %; an outage state judged against RateB / RateC when asked, falling back to
// the RateA loading where that rating is 0, PostFaultLoadingPercent :1273-1284), boundaries
// (BoundaryAnalysis.EvaluateAfterOutage, Analysis/BoundaryAnalysis.cs:43-68: the signed sum of the members' from-end
// MW, a limit of 0 = none), then voltage per-bus (:1196-1223) or the 0.94/1.06 band (:1226-1235,
// VoltageLimits.cs:28-31).
void Classify(const Model& m, int skip, bool postFault, const std::vector<double>& vm, const std::vector<double>& va,
              bool perBus, int postRating, double& maxLoad, double& worstBnd, double& minVm, double& maxVm,
              std::vector<Violation>& out, const std::vector<int>* original = nullptr) {
    const int nb = (int)m.br.size();
    std::vector<double> loading(nb), sf(2 * (size_t)nb), st(2 * (size_t)nb);
    LineFlows(m, skip, vm, va, loading.data(), sf.data(), st.data());
    maxLoad = 0;
    for (int k = 0; k < nb; k++) {
        if (k == skip) continue;  // the reduced model has no such branch
        double l = loading[k];
        if (postFault && postRating != GS_RATE_A) {
            const double rating = postRating == GS_RATE_B ? m.br[k].rateB : m.br[k].rateC;
            if (rating > 0) {
                const double mva = std::max(std::abs(cplx(sf[2 * k], sf[2 * k + 1])), std::abs(cplx(st[2 * k], st[2 * k + 1])));
                l = mva / rating * 100.0;
            }
        }
        if (l > maxLoad) maxLoad = l;
        if (l > 100.0) out.push_back({GS_VIOL_BRANCH_OVERLOAD, original ? (*original)[k] : k, l});  // keyed by the
                                                                                                  // original index
    }
    worstBnd = 0;
    for (int q = 0; q < (int)m.bnd.size(); q++) {
        const Bnd& b = m.bnd[q];
        double flow = 0;
        for (const auto& mem : b.members)
            if (mem.first != skip) flow += mem.second * sf[2 * mem.first];  // an out-of-service branch carries 0
        const bool limited = b.limitMw > 0;
        const double l = limited ? std::fabs(flow) / b.limitMw * 100.0 : 0.0;
        if (l > worstBnd) worstBnd = l;
        if (limited && std::fabs(flow) > b.limitMw) out.push_back({GS_VIOL_BOUNDARY_OVERLOAD, q, l});
    }
    minVm = INFINITY; maxVm = -INFINITY;
    for (int i = 0; i < m.n; i++) { minVm = std::min(minVm, vm[i]); maxVm = std::max(maxVm, vm[i]); }
    bool hasPerBus = false;
    for (int i = 0; i < m.n; i++) if (!std::isnan(m.vmin[i]) || !std::isnan(m.vmax[i])) hasPerBus = true;
    for (int i = 0; i < m.n; i++) {
        double lo = 0.94, hi = 1.06;
        if (perBus && hasPerBus) {
            if (!std::isnan(m.vmin[i])) lo = m.vmin[i];
            if (!std::isnan(m.vmax[i])) hi = m.vmax[i];
        }
        if (vm[i] < lo) out.push_back({GS_VIOL_UNDERVOLTAGE, m.id[i], vm[i]});
        else if (vm[i] > hi) out.push_back({GS_VIOL_OVERVOLTAGE, m.id[i], vm[i]});
    }
}

// ContingencyAnalysis.ConnectedParts (:1671-1687) of the model without branch `skip`: buses joined by in-service
// branches (union-find).
int ConnectedParts(const Model& m, int skip) {
    std::vector<int> parent(m.n);
    std::iota(parent.begin(), parent.end(), 0);
    auto find = [&](int x) { while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; } return x; };
    int parts = m.n;
    for (int k = 0; k < (int)m.br.size(); k++) {
        if (k == skip || !m.br[k].inService) continue;
        int a = find(m.br[k].f), c = find(m.br[k].t);
        if (a != c) { parent[a] = c; parts--; }
    }
    return parts;
}

// ContingencyAnalysis.ProvablyUnsolvablePart (:1750-1830) of the model without branch `skip`: true when a connected
// part has no reference bus, no negative R or Gs, and either its demand exceeds its generation by more than
// count * tol + 1e-6 pu, or it is lossless (every R and Gs zero) and unbalanced by at least that much.
bool ProvablyUnsolvablePart(const Model& m, int skip, double tol) {
    if (!(tol > 0.0) || !std::isfinite(tol)) return false;
    if (!(m.base > 0.0) || !std::isfinite(m.base)) return false;
    {
        std::vector<int> ids(m.id);
        std::sort(ids.begin(), ids.end());
        if (std::adjacent_find(ids.begin(), ids.end()) != ids.end()) return false;
    }
    const int n = m.n;
    std::vector<int> parent(n);
    std::iota(parent.begin(), parent.end(), 0);
    auto find = [&](int x) { while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; } return x; };
    for (int k = 0; k < (int)m.br.size(); k++) {
        if (k == skip || !m.br[k].inService) continue;
        int a = find(m.br[k].f), c = find(m.br[k].t);
        if (a != c) parent[a] = c;
    }
    std::vector<double> pgByBus(n, 0.0);
    for (const Gen& g : m.gens) pgByBus[g.bus] += g.pg;
    std::vector<int> order, count(n, 0);
    std::vector<char> hasSlack(n, 0), anyNeg(n, 0), anyLoss(n, 0);
    std::vector<double> net(n, 0.0);
    for (int i = 0; i < n; i++) {
        int r = find(i);
        if (count[r] == 0) order.push_back(r);
        count[r]++;
        if (m.type[i] == 3) hasSlack[r] = 1;
        if (!std::isfinite(m.gs[i]) || !std::isfinite(m.pd[i]) || !std::isfinite(pgByBus[i])) return false;
        if (m.gs[i] < 0.0) anyNeg[r] = 1;
        if (m.gs[i] != 0.0) anyLoss[r] = 1;
        net[r] += (pgByBus[i] - m.pd[i]) / m.base;
    }
    for (int k = 0; k < (int)m.br.size(); k++) {
        if (k == skip || !m.br[k].inService) continue;
        int r = find(m.br[k].f);
        if (!std::isfinite(m.br[k].r)) return false;
        if (m.br[k].r < 0.0) anyNeg[r] = 1;
        if (m.br[k].r != 0.0) anyLoss[r] = 1;
    }
    for (int r : order) {
        if (hasSlack[r] || anyNeg[r]) continue;
        double slack = count[r] * tol + 1e-6;  // UnsolvableMarginPu (:1700-1705)
        if (net[r] <= -slack) return true;
        if (!anyLoss[r] && std::fabs(net[r]) >= slack) return true;
    }
    return false;
}

// ScreenElementOutage (ContingencyAnalysis.cs:1355-1437): the reduced model of one element outage, built as the
// reference builds it. kind 1: the in-service unit `index` (a descriptor position) goes; kind 2: bus `index` goes with
// every branch touching it, its units and its load (the buses after it move up one position). When the outage takes
// a reference bus or its last unit, ReelectReference (:1440-1488) moves the reference to the bus of the largest
// remaining unit by |Pg| (first in model order) in the part the reference served; `noReference` when none is left.
// original[k] = the full model's index of the reduced model's branch k; busOf[i] = the reduced position of bus i
// (-1: removed).
struct Reduced {
    Model m;
    std::vector<int> original, busOf;
    bool noReference = false;
};

Reduced ReduceForElement(const Model& m, int kind, int index) {
    Reduced r;
    r.m = m;
    const int n = m.n;
    r.busOf.resize(n);
    std::iota(r.busOf.begin(), r.busOf.end(), 0);
    r.original.resize(m.br.size());
    std::iota(r.original.begin(), r.original.end(), 0);
    int affected = -1, removedBus = -1;
    if (kind == 1) {
        const int gi = m.genOfDesc[index];
        affected = m.gens[gi].bus;
        r.m.gens.erase(r.m.gens.begin() + gi);
    } else {
        removedBus = affected = index;
    }
    // ReelectReference on the full model's buses (positions), before any renumbering
    if (m.type[affected] == 3) {
        bool left = false;
        for (const Gen& g : r.m.gens) if (g.bus == affected && removedBus < 0) left = true;
        if (!left) {
            std::vector<std::vector<int>> adj(n);
            for (size_t k = 0; k < m.br.size(); k++)
                if (m.br[k].inService && m.br[k].f != removedBus && m.br[k].t != removedBus) {
                    adj[m.br[k].f].push_back(m.br[k].t);
                    adj[m.br[k].t].push_back(m.br[k].f);
                }
            std::vector<int> seeds;
            if (removedBus < 0) seeds.push_back(affected);
            else
                for (const Br& b : m.br)
                    if (b.inService && (b.f == removedBus || b.t == removedBus)) seeds.push_back(b.f == removedBus ? b.t : b.f);
            std::vector<char> reach(n, 0);
            std::vector<int> queue;
            for (int x : seeds) if (!reach[x]) { reach[x] = 1; queue.push_back(x); }
            for (size_t q = 0; q < queue.size(); q++)
                for (int v : adj[queue[q]]) if (v != removedBus && !reach[v]) { reach[v] = 1; queue.push_back(v); }
            const Gen* best = nullptr;
            for (const Gen& g : r.m.gens)
                if (g.bus != removedBus && reach[g.bus] && (!best || std::fabs(g.pg) > std::fabs(best->pg))) best = &g;
            if (!best) { r.noReference = true; return r; }
            if (removedBus < 0) r.m.type[affected] = 1;
            if (r.m.type[best->bus] != 3) r.m.type[best->bus] = 3;
        }
    }
    if (removedBus >= 0) {  // the bus, its branches and its units leave the model
        Model red;
        red.n = n - 1;
        red.base = m.base;
        for (int i = 0, j = 0; i < n; i++) {
            if (i == removedBus) { r.busOf[i] = -1; continue; }
            r.busOf[i] = j++;
            red.id.push_back(r.m.id[i]); red.type.push_back(r.m.type[i]);
            red.pd.push_back(m.pd[i]); red.qd.push_back(m.qd[i]); red.gs.push_back(m.gs[i]); red.bs.push_back(m.bs[i]);
            if (!m.zip.empty()) red.zip.insert(red.zip.end(), m.zip.begin() + 6 * i, m.zip.begin() + 6 * i + 6);
            red.vm.push_back(m.vm[i]); red.vaDeg.push_back(m.vaDeg[i]);
            red.vmin.push_back(m.vmin[i]); red.vmax.push_back(m.vmax[i]);
        }
        for (const Gen& g : r.m.gens)
            if (g.bus != removedBus) { Gen h = g; h.bus = r.busOf[g.bus]; red.gens.push_back(h); }
        r.original.clear();
        std::vector<int> newIndex(m.br.size(), -1);
        for (size_t k = 0; k < m.br.size(); k++) {
            const Br& b = m.br[k];
            if (b.f == removedBus || b.t == removedBus) continue;
            Br c = b;
            c.f = r.busOf[b.f];
            c.t = r.busOf[b.t];
            newIndex[k] = (int)red.br.size();
            red.br.push_back(c);
            r.original.push_back((int)k);
        }
        for (const Bnd& b : m.bnd) {  // a boundary member that went with the bus contributes nothing
            Bnd c{b.limitMw, {}};
            for (const auto& mem : b.members)
                if (newIndex[mem.first] >= 0) c.members.push_back({newIndex[mem.first], mem.second});
            red.bnd.push_back(c);
        }
        r.m = std::move(red);
    }
    return r;
}

// ParticipationWeights (ContingencyAnalysis.cs:1588-1645): a unit takes part when it is a synchronous machine on a bus
// that in-service branches connect to a reference bus (within the part `island` names, when given); its weight is
// its effective machine base (MachineBase.EffectiveMva: MBase, or the system base when MBase is 0 or less) for
// governor droop, H times that for inertia; a weight that is not a positive finite number takes no part. A
// participant with Pmin above Pmax has no range to share within: false (the reference refuses it).
bool ParticipationWeights(const Model& m, int dispatch, const std::vector<int>* island, std::vector<double>& w) {
    std::vector<std::vector<int>> adj(m.n);
    for (const Br& b : m.br)
        if (b.inService) { adj[b.f].push_back(b.t); adj[b.t].push_back(b.f); }
    auto flood = [&](std::vector<int> queue) {
        std::vector<char> seen(m.n, 0);
        for (int x : queue) seen[x] = 1;
        for (size_t q = 0; q < queue.size(); q++)
            for (int v : adj[queue[q]]) if (!seen[v]) { seen[v] = 1; queue.push_back(v); }
        return seen;
    };
    std::vector<int> refs;
    for (int i = 0; i < m.n; i++) if (m.type[i] == 3) refs.push_back(i);
    std::vector<char> reach = flood(refs);
    if (island) {
        std::vector<char> part = flood(*island);
        for (int i = 0; i < m.n; i++) reach[i] = reach[i] && part[i];
    }
    w.assign(m.gens.size(), 0.0);
    for (size_t i = 0; i < m.gens.size(); i++) {
        const Gen& g = m.gens[i];
        if (!g.sync || !reach[g.bus]) continue;
        const double mva = g.mbase > 0.0 ? g.mbase : m.base;
        const double x = dispatch == 1 ? mva : g.h * mva;
        if (!(x > 0.0) || !std::isfinite(x)) continue;
        if (g.pmin > g.pmax) return false;
        w[i] = x;
    }
    return true;
}

// ShareLostPower (ContingencyAnalysis.cs:1509-1579): the net lost MW (positive: generation lost) shared among the
// participants in proportion to their weights, each within [Pmin, Pmax] from its scheduled Pg; a unit whose share
// exceeds its headroom is fixed at its limit and the rest shared again (units visited in model order). `stats`:
// lost MW, participants, units fixed at a limit, MW left to the reference. False for a lost MW that is not finite
// or a participant with crossed limits.
bool ShareLostPower(Model& m, double lostMw, int dispatch, const std::vector<int>* island, double stats[4]) {
    if (!std::isfinite(lostMw)) return false;
    stats[0] = lostMw; stats[1] = 0; stats[2] = 0; stats[3] = 0;
    if (lostMw == 0.0) return true;
    std::vector<double> weights;
    if (!ParticipationWeights(m, dispatch, island, weights)) return false;
    const size_t n = m.gens.size();
    std::vector<double> weight(n, 0.0), room(n, 0.0), delta(n, 0.0);
    std::vector<int> active;
    const bool raise = lostMw > 0.0;
    for (size_t i = 0; i < n; i++) {
        const Gen& g = m.gens[i];
        const double w = weights[i];
        if (!(w > 0.0)) continue;
        const double r = raise ? g.pmax - g.pg : g.pg - g.pmin;
        if (!(r > 0.0)) continue;
        weight[i] = w;
        room[i] = r;
        active.push_back((int)i);
    }
    double remaining = std::fabs(lostMw);
    int fixedAtLimit = 0;
    const int participants = (int)active.size();
    while (!active.empty() && remaining > 0.0) {
        double wsum = 0.0;
        for (int i : active) wsum += weight[i];
        std::vector<int> capped;
        for (int i : active) if (remaining * weight[i] / wsum > room[i]) capped.push_back(i);
        if (capped.empty()) {
            for (int i : active) delta[i] += remaining * weight[i] / wsum;
            remaining = 0.0;
            break;
        }
        for (int i : capped) {
            delta[i] += room[i];
            remaining -= room[i];
            active.erase(std::find(active.begin(), active.end(), i));
            fixedAtLimit++;
        }
        if (remaining < 0.0) remaining = 0.0;
    }
    const double sign = raise ? 1.0 : -1.0;
    for (size_t i = 0; i < n; i++)
        if (delta[i] != 0.0) m.gens[i].pg = m.gens[i].pg + sign * delta[i];
    stats[1] = participants;
    stats[2] = fixedAtLimit;
    stats[3] = remaining;
    return true;
}

bool OptionsSupported(const gs_pf_opts* o) { return o != nullptr; }

}  // namespace

// =============================================================================================
// C API of the oracle (test infrastructure). All outputs are caller-owned.
extern "C" {

int gso_pf_solve(const gs_grid_desc* d, const gs_pf_opts* opt, gs_pf_result* res) {
    if (!d || !res || !OptionsSupported(opt)) return GS_ERR_INVALID_ARG;
    Model m = FromDesc(d);
    SolveOut o = SolveWithRetry(m, -1, *opt, nullptr, nullptr);
    res->status = o.status;
    res->iterations = o.iterations;
    res->max_mismatch = o.maxMis;
    for (int i = 0; i < m.n; i++) {
        if (res->vm) res->vm[i] = o.vm[i];
        if (res->va_deg) res->va_deg[i] = o.va[i] * 180.0 / kPi;
        if (res->p_inj_mw) res->p_inj_mw[i] = o.p[i] * m.base;
        if (res->q_inj_mvar) res->q_inj_mvar[i] = o.q[i] * m.base;
    }
    LineFlows(m, -1, o.vm, o.va, res->loading_pct, res->sf_mva, res->st_mva);
    return GS_OK;
}

// Jacobian of the intact grid at its start point, in the reference's own CSR (for kernel checks).
// Returns m; fills rowPtr [m+1], colIdx/val [nnz] when the capacities allow (nnz returned in *nnz).
int gso_jacobian(const gs_grid_desc* d, int32_t* m_out, int32_t* nnz_out, int32_t* rowPtr, int32_t* colIdx,
                 double* val, int32_t cap, double* mismatch, int32_t mis_cap) {
    if (!d) return GS_ERR_INVALID_ARG;
    Model mdl = FromDesc(d);
    ComplexCsr y = BuildY(mdl, -1);
    BusSpec s = BuildBusSpec(mdl, false);
    std::vector<int> pPos, qPos, slots;
    int m = EquationPositions(s.type0, pPos, qPos);
    Csr jac = BuildJacobianStructure(y, pPos, qPos, m, slots);
    std::vector<double> P(mdl.n), Q(mdl.n);
    ComputeInjections(y, s.vm, s.va, P, Q);
    RefillJacobian(jac, slots, y, s.vm, s.va, P, Q);
    *m_out = m;
    *nnz_out = (int32_t)jac.colIdx.size();
    if (mismatch && mis_cap >= m) {
        for (int i = 0; i < mdl.n; i++) {
            if (pPos[i] >= 0) mismatch[pPos[i]] = s.pspec[i] - P[i];
            if (qPos[i] >= 0) mismatch[qPos[i]] = s.qspec[i] - Q[i];
        }
    }
    if (cap < (int)jac.colIdx.size()) return GS_ERR_CAPACITY;
    for (int i = 0; i <= m; i++) rowPtr[i] = jac.rowPtr[i];
    for (size_t k = 0; k < jac.colIdx.size(); k++) { colIdx[k] = jac.colIdx[k]; val[k] = jac.val[k]; }
    return GS_OK;
}

// The max |mismatch| of `count` given states (system-major [count][n], Va in radians), each on the grid with branch
// outage[s] removed (-1 or a null `outage`: the intact grid): Y rebuilt as BuildY does (:382-402), the bus
// specification of BuildBusSpec (NewtonShell.cs:433-486), the injections of ComputeInjections (:269-289) and the
// infinity norm of RunNewton's mismatch vector (:216-235). NaN when a mismatch is not finite.
int gso_max_mismatch(const gs_grid_desc* d, int32_t count, const int32_t* outage, const double* vm, const double* va,
                     double* out) {
    if (!d || count < 0 || (count > 0 && (!vm || !va || !out))) return GS_ERR_INVALID_ARG;
    Model mdl = FromDesc(d);
    const int n = mdl.n;
    BusSpec s = BuildBusSpec(mdl, false);
    std::vector<int> pPos, qPos;
    EquationPositions(s.type0, pPos, qPos);
    std::vector<double> V(n), A(n), P(n), Q(n);
    for (int c = 0; c < count; c++) {
        const int o = outage ? outage[c] : -1;
        if (o >= (int)mdl.br.size()) return GS_ERR_INVALID_ARG;
        ComplexCsr y = BuildY(mdl, o);
        for (int i = 0; i < n; i++) { V[i] = vm[(size_t)c * n + i]; A[i] = va[(size_t)c * n + i]; }
        ComputeInjections(y, V, A, P, Q);
        double mx = 0.0;
        bool finite = true;
        for (int i = 0; i < n; i++) {
            const double* z = &s.zip[6 * (size_t)i];
            const double dP = s.hasZip[i] ? s.pd[i] * (ZipMult(z, V[i]) - 1.0) / mdl.base : 0.0;
            const double dQ = s.hasZip[i] ? s.qd[i] * (ZipMult(z + 3, V[i]) - 1.0) / mdl.base : 0.0;
            if (pPos[i] >= 0) { double f = s.pspec[i] - P[i] - dP; finite = finite && std::isfinite(f); mx = std::max(mx, std::fabs(f)); }
            if (qPos[i] >= 0) { double f = s.qspec[i] - Q[i] - dQ; finite = finite && std::isfinite(f); mx = std::max(mx, std::fabs(f)); }
        }
        out[c] = finite ? mx : NAN;
    }
    return GS_OK;
}

// Minimum-degree order of a CSR pattern (for ordering tests).
int gso_md_order(int32_t n, const int32_t* rowPtr, const int32_t* colIdx, int32_t* order) {
    std::vector<int> rp(rowPtr, rowPtr + n + 1), ci(colIdx, colIdx + rowPtr[n]);
    std::vector<int> q = MinimumDegree(n, rp, ci);
    for (int i = 0; i < n; i++) order[i] = q[i];
    return GS_OK;
}

// Sparse direct solve A x = b (ISparseLinearSolver via CpuSparseLuSolver). Returns 1 when singular, 2 when the
// matrix factorises but b has a non-finite entry (the ArgumentException CpuSparseLuSolver.cs:41-47 throws after the
// factorisation, so a singular matrix stays 1 whatever b holds).
int gso_sparse_solve(int32_t n, const int32_t* rowPtr, const int32_t* colIdx, const double* val, const double* b,
                     double* x) {
    Csr a;
    a.n = n;
    a.rowPtr.assign(rowPtr, rowPtr + n + 1);
    a.colIdx.assign(colIdx, colIdx + rowPtr[n]);
    a.val.assign(val, val + rowPtr[n]);
    CpuSparseLuSolver s;
    std::vector<double> bv(b, b + n), xv;
    bool bFinite = true;
    for (double v : bv) bFinite = bFinite && std::isfinite(v);
    if (!bFinite) return s.Solve(a, std::vector<double>(n, 0.0), xv) ? 2 : 1;
    if (!s.Solve(a, bv, xv)) return 1;
    for (int i = 0; i < n; i++) x[i] = xv[i];
    return GS_OK;
}

// The singular-step fallback's two pieces on their own, for pinning them on the reference's known answers:
// Ilu0.Factor then Apply (Numerics/Sparse.cs:240-300), and BiCgStab.Solve with that preconditioner
// (Sparse.cs:319-405; maxIter 0 = the shared cap 4n + 200, NumericTolerances.cs:256-260). BiCGSTAB returns 1 when
// it is not accepted.
int gso_ilu0_apply(int32_t n, const int32_t* rowPtr, const int32_t* colIdx, const double* val, const double* r,
                   double* z) {
    Csr a;
    a.n = n;
    a.rowPtr.assign(rowPtr, rowPtr + n + 1);
    a.colIdx.assign(colIdx, colIdx + rowPtr[n]);
    a.val.assign(val, val + rowPtr[n]);
    Ilu0 pc;
    pc.Factor(a);
    std::vector<double> rv(r, r + n), zv(n, 0.0);
    pc.Apply(rv, zv);
    for (int i = 0; i < n; i++) z[i] = zv[i];
    return GS_OK;
}
int gso_bicgstab(int32_t n, const int32_t* rowPtr, const int32_t* colIdx, const double* val, const double* b,
                 double tol, int32_t maxIter, double* x) {
    Csr a;
    a.n = n;
    a.rowPtr.assign(rowPtr, rowPtr + n + 1);
    a.colIdx.assign(colIdx, colIdx + rowPtr[n]);
    a.val.assign(val, val + rowPtr[n]);
    Ilu0 pc;
    pc.Factor(a);
    std::vector<double> bv(b, b + n), xv;
    const bool ok = BiCgStab(a, bv, xv, pc, tol, maxIter > 0 ? maxIter : 4 * n + 200);
    for (int i = 0; i < n; i++) x[i] = xv[i];
    return ok ? GS_OK : 1;
}

}  // extern "C"

namespace {

// The screen of outages given as lists of branches taken out together (ScreenOutageCore, :1087-1097): one branch is
// the N-1 path (the branch skipped in the Y build), several are taken out of a copy of the model.
int ScreenLists(const Model& m, const std::vector<std::vector<int>>& lists, const gs_pf_opts* opt, int threads,
                gs_n1_result* res) {
    const int nOut = (int)lists.size();
    for (const auto& l : lists)
        for (int k : l)
            if (k < 0 || k >= (int)m.br.size() || !m.br[k].inService) return GS_ERR_INVALID_ARG;
    std::vector<double> vm0, va0;
    res->base_status = GS_PF_NOT_RUN;
    res->base_iterations = 0;
    if (opt->warm_start_from_base) {
        SolveOut b = SolveWithRetry(m, -1, *opt, nullptr, nullptr);
        res->base_status = b.status;
        res->base_iterations = b.iterations;
        vm0 = b.vm;
        va0 = b.va;
    }
    std::vector<SolveOut> outs(nOut);
    std::vector<std::vector<Violation>> viol(nOut);
    std::vector<double> maxLoad(nOut, 0), worstBnd(nOut, 0), minVm(nOut, 0), maxVm(nOut, 0);
    std::vector<uint8_t> islanded(nOut, 0);
    const int partsBefore = ConnectedParts(m, -1);
    std::atomic<int> cursor{0};
    auto work = [&]() {
        for (;;) {
            int k = cursor.fetch_add(1);
            if (k >= nOut) return;
            const std::vector<int>& l = lists[k];
            Model reduced;
            const Model* mk = &m;
            int skip = l.size() == 1 ? l[0] : -1;
            if (l.size() > 1) {
                reduced = m;
                for (int b : l) reduced.br[b].inService = false;
                mk = &reduced;
            }
            // ScreenStateCore (:1118-1127): a provably unsolvable state is reported without a solve
            if (ProvablyUnsolvablePart(*mk, skip, opt->tolerance)) {
                outs[k].status = GS_PF_UNSOLVABLE_PART;
                outs[k].iterations = 0;
                outs[k].maxMis = 0;
                outs[k].vm.assign(m.n, 0.0);
                outs[k].va.assign(m.n, 0.0);
            } else {
                outs[k] = SolveWithRetry(*mk, skip, *opt, vm0.empty() ? nullptr : vm0.data(),
                                         va0.empty() ? nullptr : va0.data());
            }
            if (outs[k].status == GS_PF_CONVERGED)
                Classify(*mk, skip, !l.empty(), outs[k].vm, outs[k].va, opt->per_bus_voltage_limits != 0,
                         opt->post_fault_rating, maxLoad[k], worstBnd[k], minVm[k], maxVm[k], viol[k]);
            else  // NonConverged(label, Splits(before, reduced)) (:1661-1665)
                islanded[k] = ConnectedParts(*mk, skip) > partsBefore;
        }
    };
    int nt = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
    nt = std::max(1, std::min(nt, std::max(1, nOut)));
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; t++) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();

    int total = 0;
    for (int k = 0; k < nOut; k++) total += (int)viol[k].size();
    res->viol_count = total;
    bool fits = total <= res->viol_capacity;
    int w = 0;
    for (int k = 0; k < nOut; k++) {
        if (res->status) res->status[k] = outs[k].status;
        if (res->iterations) res->iterations[k] = outs[k].iterations;
        if (res->max_mismatch) res->max_mismatch[k] = outs[k].maxMis;
        if (res->min_vm) res->min_vm[k] = minVm[k];
        if (res->max_vm) res->max_vm[k] = maxVm[k];
        if (res->max_loading_pct) res->max_loading_pct[k] = maxLoad[k];
        if (res->worst_boundary_pct) res->worst_boundary_pct[k] = worstBnd[k];
        if (res->islanded) res->islanded[k] = islanded[k];
        if (res->viol_ptr) res->viol_ptr[k] = w;
        for (const Violation& v : viol[k]) {
            if (fits && res->viol_kind) {
                res->viol_kind[w] = v.kind;
                res->viol_element[w] = v.element;
                res->viol_value[w] = v.value;
            }
            w++;
        }
        if (res->vm)
            for (int i = 0; i < m.n; i++) res->vm[(size_t)k * m.n + i] = outs[k].vm[i];
        if (res->va_deg)
            for (int i = 0; i < m.n; i++) res->va_deg[(size_t)k * m.n + i] = outs[k].va[i] * 180.0 / kPi;
    }
    if (res->viol_ptr) res->viol_ptr[nOut] = w;
    return fits ? GS_OK : GS_ERR_CAPACITY;
}

}  // namespace

extern "C" {

// ScreenBranchesParallel (ContingencyAnalysis.cs:323-344): one outage per task on `threads` host threads
// (0 = all). Output layout is gs_n1_result's; -1 is the intact grid (ScreenBaseCase). With warm_start_from_base the
// intact grid is solved first and its state starts every outage (GridScenario.WithSolvedVoltages).
int gso_n1_screen(const gs_grid_desc* d, int32_t nOut, const int32_t* idx, const gs_pf_opts* opt, int32_t threads,
                  gs_n1_result* res) {
    if (!d || !res || !OptionsSupported(opt) || nOut < 0) return GS_ERR_INVALID_ARG;
    Model m = FromDesc(d);
    std::vector<std::vector<int>> lists(nOut);
    for (int k = 0; k < nOut; k++) {
        if (idx[k] < -1) return GS_ERR_INVALID_ARG;
        if (idx[k] >= 0) lists[k].push_back(idx[k]);
    }
    return ScreenLists(m, lists, opt, threads, res);
}

// ScreenOutageCore over several indices per outage (the N-k screens' unit of work): outage j takes out every branch
// sets[j*k .. j*k+k-1] that is not -1.
int gso_nk_screen(const gs_grid_desc* d, int32_t nOut, int32_t k, const int32_t* sets, const gs_pf_opts* opt,
                  int32_t threads, gs_n1_result* res) {
    if (!d || !res || !OptionsSupported(opt) || nOut < 0 || k < 1) return GS_ERR_INVALID_ARG;
    Model m = FromDesc(d);
    std::vector<std::vector<int>> lists(nOut);
    for (int j = 0; j < nOut; j++)
        for (int q = 0; q < k; q++) {
            const int b = sets[(size_t)j * k + q];
            if (b < -1) return GS_ERR_INVALID_ARG;
            if (b >= 0) lists[j].push_back(b);
        }
    return ScreenLists(m, lists, opt, threads, res);
}

// ScreenElementOutages (ContingencyAnalysis.cs:1309-1437) with the reference-bus dispatch: outage j is the branch,
// unit or bus index[j] of kind[j] (0, 1, 2). Results in gs_n1_result's layout over the full model's buses; a removed
// bus's state entries are 0 and it is in neither Vmin / Vmax nor the voltage violations.
int gso_element_screen(const gs_grid_desc* d, int32_t nOut, const int32_t* kind, const int32_t* index,
                       const gs_pf_opts* opt, int32_t threads, const GsoMachines* mach, double* share, gs_n1_result* res) {
    if (!d || !res || !OptionsSupported(opt) || nOut < 0) return GS_ERR_INVALID_ARG;
    Model m = FromDesc(d);
    const int dispatch = mach ? mach->dispatch : 0;
    if (mach) AttachMachines(m, mach);
    for (int j = 0; j < nOut; j++) {
        if (kind[j] == 0 && (index[j] < 0 || index[j] >= (int)m.br.size() || !m.br[index[j]].inService)) return GS_ERR_INVALID_ARG;
        if (kind[j] == 1 && (index[j] < 0 || index[j] >= (int)m.genOfDesc.size() || m.genOfDesc[index[j]] < 0)) return GS_ERR_INVALID_ARG;
        if (kind[j] == 2 && (index[j] < 0 || index[j] >= m.n)) return GS_ERR_INVALID_ARG;
        if (kind[j] < 0 || kind[j] > 2) return GS_ERR_INVALID_ARG;
    }
    std::vector<double> vm0, va0;
    res->base_status = GS_PF_NOT_RUN;
    res->base_iterations = 0;
    if (opt->warm_start_from_base) {
        SolveOut b = SolveWithRetry(m, -1, *opt, nullptr, nullptr);
        res->base_status = b.status;
        res->base_iterations = b.iterations;
        vm0 = b.vm;
        va0 = b.va;
    }
    const int n = m.n;
    std::vector<SolveOut> outs(nOut);
    std::vector<std::vector<Violation>> viol(nOut);
    std::vector<double> maxLoad(nOut, 0), worstBnd(nOut, 0), minVm(nOut, 0), maxVm(nOut, 0);
    std::vector<uint8_t> islanded(nOut, 0);
    std::vector<std::vector<int>> busOf(nOut);
    const int partsBefore = ConnectedParts(m, -1);
    if (share)
        for (int j = 0; j < nOut; j++)
            for (int q = 0; q < 4; q++) share[4 * j + q] = q == 0 ? std::numeric_limits<double>::quiet_NaN() : 0.0;
    std::atomic<int> cursor{0};
    std::atomic<int> refused{0};
    auto work = [&]() {
        for (;;) {
            const int j = cursor.fetch_add(1);
            if (j >= nOut) return;
            Reduced r;
            int skip = -1;
            if (kind[j] == 0) {
                r.m = m;
                r.busOf.resize(n);
                std::iota(r.busOf.begin(), r.busOf.end(), 0);
                skip = index[j];
            } else {
                r = ReduceForElement(m, kind[j], index[j]);
                // ScreenElementOutage (:1370-1374, :1410-1421): a shared dispatch moves the remaining units before
                // the re-solve; the part that lost the power is the unit's bus, or the removed bus's neighbours
                if (dispatch != 0 && !r.noReference) {
                    double lost;
                    std::vector<int> island;
                    if (kind[j] == 1) {
                        const Gen& g = m.gens[m.genOfDesc[index[j]]];
                        lost = g.pg;
                        island.push_back(g.bus);
                    } else {
                        double lostGen = 0.0;
                        for (const Gen& g : m.gens) if (g.bus == index[j]) lostGen += g.pg;
                        lost = lostGen - m.pd[index[j]];
                        for (const Br& b : m.br)
                            if (b.inService && (b.f == index[j] || b.t == index[j])) {
                                const int nb = r.busOf[b.f == index[j] ? b.t : b.f];
                                if (nb >= 0) island.push_back(nb);
                            }
                    }
                    double st[4];
                    if (!ShareLostPower(r.m, lost, dispatch, &island, st)) { refused = 1; busOf[j] = r.busOf; continue; }
                    if (share) for (int q = 0; q < 4; q++) share[4 * j + q] = st[q];
                }
            }
            busOf[j] = r.busOf;
            const Model& red = r.m;
            const bool splits = ConnectedParts(red, skip) > partsBefore;
            if (r.noReference || ProvablyUnsolvablePart(red, skip, opt->tolerance)) {
                outs[j].status = GS_PF_UNSOLVABLE_PART;
                outs[j].iterations = 0;
                outs[j].maxMis = 0;
                outs[j].vm.assign(red.n, 0.0);
                outs[j].va.assign(red.n, 0.0);
                islanded[j] = splits;
                continue;
            }
            std::vector<double> v0, a0;
            if (!vm0.empty())
                for (int i = 0; i < n; i++)
                    if (r.busOf[i] >= 0) { v0.push_back(vm0[i]); a0.push_back(va0[i]); }
            outs[j] = SolveWithRetry(red, skip, *opt, v0.empty() ? nullptr : v0.data(), a0.empty() ? nullptr : a0.data());
            if (outs[j].status == GS_PF_CONVERGED)
                Classify(red, skip, true, outs[j].vm, outs[j].va, opt->per_bus_voltage_limits != 0, opt->post_fault_rating,
                         maxLoad[j], worstBnd[j], minVm[j], maxVm[j], viol[j], kind[j] == 2 ? &r.original : nullptr);
            else
                islanded[j] = splits;
        }
    };
    int nt = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
    nt = std::max(1, std::min(nt, std::max(1, nOut)));
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; t++) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
    if (refused) return GS_ERR_INVALID_ARG;
    int total = 0;
    for (int j = 0; j < nOut; j++) total += (int)viol[j].size();
    res->viol_count = total;
    const bool fits = total <= res->viol_capacity;
    int w = 0;
    for (int j = 0; j < nOut; j++) {
        if (res->status) res->status[j] = outs[j].status;
        if (res->iterations) res->iterations[j] = outs[j].iterations;
        if (res->max_mismatch) res->max_mismatch[j] = outs[j].maxMis;
        if (res->min_vm) res->min_vm[j] = minVm[j];
        if (res->max_vm) res->max_vm[j] = maxVm[j];
        if (res->max_loading_pct) res->max_loading_pct[j] = maxLoad[j];
        if (res->worst_boundary_pct) res->worst_boundary_pct[j] = worstBnd[j];
        if (res->islanded) res->islanded[j] = islanded[j];
        if (res->viol_ptr) res->viol_ptr[j] = w;
        for (const Violation& v : viol[j]) {
            if (fits && res->viol_kind) {
                res->viol_kind[w] = v.kind;
                res->viol_element[w] = v.element;
                res->viol_value[w] = v.value;
            }
            w++;
        }
        for (int i = 0; i < n; i++) {
            const int p = busOf[j][i];
            if (res->vm) res->vm[(size_t)j * n + i] = p >= 0 ? outs[j].vm[p] : 0.0;
            if (res->va_deg) res->va_deg[(size_t)j * n + i] = p >= 0 ? outs[j].va[p] * 180.0 / kPi : 0.0;
        }
    }
    if (res->viol_ptr) res->viol_ptr[nOut] = w;
    return fits ? GS_OK : GS_ERR_CAPACITY;
}

// The topology verdicts of single-branch outages (the product's gs_outage_topology), the reference's way: per outage,
// ConnectedParts of the reduced model against the intact one and ProvablyUnsolvablePart of the reduced model.
// ShareLostPower on the model of `d` (no outage taken): `lostMw` shared by mach->dispatch among its units, within the
// part the island bus positions name (n_island < 0: the whole network). pg_out [n_gen] receives every descriptor
// unit's scheduled output after the sharing; stats [4]: lost MW, participants, units fixed at a limit, MW left to
// the reference. GS_ERR_INVALID_ARG for the reference-bus dispatch, a lost MW that is not finite, or a participant
// with Pmin above Pmax (the reference refuses each).
int gso_share_lost_power(const gs_grid_desc* d, double lostMw, const GsoMachines* mach, int32_t nIsland,
                         const int32_t* island, double* pgOut, double* stats) {
    if (!d || !mach || !pgOut || !stats || mach->dispatch < 1 || mach->dispatch > 2) return GS_ERR_INVALID_ARG;
    Model m = FromDesc(d);
    AttachMachines(m, mach);
    std::vector<int> isl;
    if (nIsland >= 0) isl.assign(island, island + nIsland);
    if (!ShareLostPower(m, lostMw, mach->dispatch, nIsland >= 0 ? &isl : nullptr, stats)) return GS_ERR_INVALID_ARG;
    for (int g = 0; g < d->n_gen; g++) pgOut[g] = m.genOfDesc[g] >= 0 ? m.gens[m.genOfDesc[g]].pg : d->pg[g];
    return GS_OK;
}

int gso_outage_topology(const gs_grid_desc* d, double tol, int32_t nOut, const int32_t* idx, uint8_t* splits,
                        uint8_t* unsolvable) {
    if (!d || nOut < 0) return GS_ERR_INVALID_ARG;
    Model m = FromDesc(d);
    const int before = ConnectedParts(m, -1);
    for (int k = 0; k < nOut; k++) {
        if (idx[k] < -1 || idx[k] >= (int)m.br.size()) return GS_ERR_INVALID_ARG;
        if (splits) splits[k] = ConnectedParts(m, idx[k]) > before;
        if (unsolvable) unsolvable[k] = ProvablyUnsolvablePart(m, idx[k], tol);
    }
    return GS_OK;
}

}  // extern "C"

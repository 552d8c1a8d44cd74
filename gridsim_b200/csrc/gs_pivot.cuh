// gs_pivot.cuh — per-system sparse LU with row partial pivoting, for the systems whose static diagonal pivot
// collapsed (included by gs_engine.cu).
//
// The batched kernels pivot statically on the diagonal of a minimum-degree order. A system whose pivot falls below
// its floor is solved again here the way the reference factors every system: the left-looking Gilbert-Peierls LU
// with row partial pivoting (SparseLuFactorization.Factor, Numerics/SparseLuFactorization.cs:69-195: the reach of
// each column by depth-first search through the columns of L computed so far (Reach / Dfs :783-821), a sparse
// triangular solve over the reach in topological order (SpSolve :753-780), the largest remaining magnitude as the
// pivot, refused at or below the row's floor 1e-12 x max |A(row, :)| (:129-162, NumericTolerances.cs:36,
// RowPivotFloorsCsc :99-116)), then the forward and backward solve (:314-371). Cells whose value is exactly zero
// are left out, as SparseLu.ToCsc does (Numerics/SparseLu.cs:63-91). The column order is the static order itself:
// the matrix is held in pivot order, which is the minimum-degree order of its pattern. On a symmetric pattern (every
// Jacobian) that is the order the reference's CpuSparseLuSolver takes (PowerFlow/CpuSparseLuSolver.cs:30-48); on a
// nonsymmetric bare matrix the reference breaks minimum-degree ties by its scan order of A and may order it
// differently.
//
// One warp per system. The reach is a sequential depth-first search (lane 0); the column updates, the pivot search
// and the writes of L and U are spread over the lanes. The factors live in global scratch of a fixed capacity per
// system; a system that needs more reports GP_CAPACITY.
#pragma once

namespace gs {

enum : int32_t { GP_OK = 0, GP_SINGULAR = 1, GP_CAPACITY = 2, GP_NON_FINITE = 3 };

// The matrix's own cells by column in pivot order (row = pivot-order row, slot = its LU slot in the batch layout) and
// the per-system scratch of the factorisation; q-th listed system at offset q * (m or m + 1 or cap).
struct GpView {
    int m;
    int64_t cap;  // L and U entries each, per system
    const int* colPtr;
    const int* row;
    const int* slot;
    double* x;       // [m] dense work column, all zero between columns
    unsigned long long* rowMax;  // [m] max |A(row, :)| as the bits of a non-negative double
    int* xi;         // [m] depth-first stack and reach (topological order from `top` on)
    int* pstack;     // [m]
    int* mark;       // [m] column stamp of the last visit
    int* pinv;       // [m] row -> its pivot column, -1 while not pivoted
    int* lp;         // [m + 1]
    int* up;         // [m + 1]
    int* li;         // [cap] rows (pivot positions after the factorisation)
    int* ui;         // [cap]
    double* lx;      // [cap]
    double* ux;      // [cap]
    int* result;     // [listed systems] GP_*
};

__device__ __forceinline__ void gpAtomicMax(unsigned long long* a, double v) {
    atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

// Reach of column entry j (Dfs, SparseLuFactorization.cs:795-821): the rows j reaches through the columns of L
// found so far, pushed on xi below `top` in reverse finishing order. Lane 0 only.
__device__ int gpDfs(int j, int top, int stamp, int* xi, int* pstack, int* mark, const int* pinv, const int* lp,
                     const int* li) {
    int head = 0;
    xi[0] = j;
    while (head >= 0) {
        j = xi[head];
        const int jcol = pinv[j];
        if (mark[j] != stamp) {
            mark[j] = stamp;
            pstack[head] = jcol < 0 ? 0 : lp[jcol] + 1;
        }
        bool done = true;
        const int pend = jcol < 0 ? 0 : lp[jcol + 1];
        for (int p = pstack[head]; p < pend; p++) {
            const int i = li[p];
            if (mark[i] == stamp) continue;
            pstack[head] = p + 1;
            xi[++head] = i;
            done = false;
            break;
        }
        if (done) {
            head--;
            xi[--top] = j;
        }
    }
    return top;
}

// Factor and solve the listed systems of a batch: A(row, col) = lu[slot * B + s] (the Jacobian or the loaded matrix,
// before any static factorisation), right-hand side y[row * B + s] in pivot order, overwritten with the solution
// (pivot order). v.result[q] reports each listed system; y is left as it was unless the result is GP_OK.
__global__ void __launch_bounds__(32) k_gp_solve(GpView v, const double* __restrict__ lu, double* y, int B,
                                                 const int* list, int nList) {
    const int q = blockIdx.x;
    if (q >= nList) return;
    const int s = list ? list[q] : q;
    const int lane = threadIdx.x;
    const unsigned full = 0xffffffffu;
    const int m = v.m;
    const int64_t cap = v.cap;
    double* x = v.x + (size_t)q * m;
    unsigned long long* rowMax = v.rowMax + (size_t)q * m;
    int* xi = v.xi + (size_t)q * m;
    int* pstack = v.pstack + (size_t)q * m;
    int* mark = v.mark + (size_t)q * m;
    int* pinv = v.pinv + (size_t)q * m;
    int* lp = v.lp + (size_t)q * (m + 1);
    int* up = v.up + (size_t)q * (m + 1);
    int* li = v.li + (size_t)q * cap;
    int* ui = v.ui + (size_t)q * cap;
    double* lx = v.lx + (size_t)q * cap;
    double* ux = v.ux + (size_t)q * cap;
    const size_t Bz = (size_t)B;

    for (int r = lane; r < m; r += 32) {
        x[r] = 0.0;
        rowMax[r] = 0ull;
        mark[r] = -1;
        pinv[r] = -1;
    }
    __syncwarp();
    // row floors (RowPivotFloorsCsc): the largest magnitude of each row; a NaN or Inf anywhere ends the solve
    int bad = 0;
    for (int c = 0; c < m; c++)
        for (int p = v.colPtr[c] + lane; p < v.colPtr[c + 1]; p += 32) {
            const double a = lu[(size_t)v.slot[p] * Bz + s];
            if (!isfinite(a)) bad = 1;
            else if (a != 0.0) gpAtomicMax(&rowMax[v.row[p]], fabs(a));
        }
    if (__any_sync(full, bad)) {
        if (lane == 0) v.result[q] = GP_NON_FINITE;
        return;
    }
    __syncwarp();
    int64_t nl = 0, nu = 0;  // entries of L and U so far (uniform across the warp)
    for (int k = 0; k < m; k++) {
        if (lane == 0) { lp[k] = (int)nl; up[k] = (int)nu; }
        const int c0 = v.colPtr[k], c1 = v.colPtr[k + 1];
        // reach of the column's nonzero rows (lane 0), in topological order xi[top .. m)
        int top = m;
        if (lane == 0) {
            for (int p = c0; p < c1; p++) {
                const int j = v.row[p];
                if (lu[(size_t)v.slot[p] * Bz + s] == 0.0) continue;
                if (mark[j] != k) top = gpDfs(j, top, k, xi, pstack, mark, pinv, lp, li);
            }
        }
        top = __shfl_sync(full, top, 0);
        __syncwarp();
        // scatter A(:, k); the sparse triangular solve over the reach in topological order
        for (int p = c0 + lane; p < c1; p += 32) {
            const double a = lu[(size_t)v.slot[p] * Bz + s];
            if (a != 0.0) x[v.row[p]] = a;
        }
        __syncwarp();
        for (int px = top; px < m; px++) {
            const int j = xi[px];
            const int jc = pinv[j];
            if (jc < 0) continue;
            const double xj = x[j];
            const int e1 = lp[jc + 1];
            for (int p = lp[jc] + 1 + lane; p < e1; p += 32) x[li[p]] -= lx[p] * xj;
            __syncwarp();
        }
        // partial pivot: the first largest magnitude among the rows not yet pivoted, in reach order
        double best = -1.0;
        int bestPx = m;
        for (int px = top + lane; px < m; px += 32) {
            const int i = xi[px];
            if (pinv[i] < 0) {
                const double t = fabs(x[i]);
                if (t > best) { best = t; bestPx = px; }
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_xor_sync(full, best, o);
            const int op = __shfl_xor_sync(full, bestPx, o);
            if (ob > best || (ob == best && op < bestPx)) { best = ob; bestPx = op; }
        }
        const int reach = m - top;
        if (bestPx >= m || !(best > __longlong_as_double((long long)rowMax[xi[bestPx]]) * 1e-12)) {
            if (lane == 0) v.result[q] = GP_SINGULAR;
            return;
        }
        if (nl + reach > cap || nu + reach > cap) {
            if (lane == 0) v.result[q] = GP_CAPACITY;
            return;
        }
        const int ipiv = xi[bestPx];
        const double pivot = x[ipiv];
        // U: the pivoted rows of the reach (their pivot columns), then the diagonal; L: the pivot row (unit), then
        // the rows not pivoted, divided by the pivot; both in reach order
        int64_t uo = nu, lo = nl + 1;
        for (int base = top; base < m; base += 32) {
            const int px = base + lane;
            const bool in = px < m;
            const int i = in ? xi[px] : 0;
            const int pc = in ? pinv[i] : -1;
            const bool isU = in && pc >= 0;
            const bool isL = in && pc < 0 && px != bestPx;
            const unsigned mu = __ballot_sync(full, isU), ml = __ballot_sync(full, isL);
            const unsigned below = (1u << lane) - 1u;
            if (isU) { const int64_t d = uo + __popc(mu & below); ui[d] = pc; ux[d] = x[i]; }
            if (isL) { const int64_t d = lo + __popc(ml & below); li[d] = i; lx[d] = x[i] / pivot; }
            uo += __popc(mu);
            lo += __popc(ml);
        }
        __syncwarp();
        if (lane == 0) {
            ui[uo] = k;
            ux[uo] = pivot;
            li[nl] = ipiv;
            lx[nl] = 1.0;
            pinv[ipiv] = k;
        }
        nu = uo + 1;
        nl = lo;
        __syncwarp();
        for (int px = top + lane; px < m; px += 32) x[xi[px]] = 0.0;
        __syncwarp();
    }
    if (lane == 0) { lp[m] = (int)nl; up[m] = (int)nu; }
    __syncwarp();
    for (int64_t p = lane; p < nl; p += 32) li[p] = pinv[li[p]];
    // solve: x(pinv(r)) = b(r); L (unit lower, by columns); U (by columns, the diagonal last in each)
    for (int r = lane; r < m; r += 32) x[pinv[r]] = y[(size_t)r * Bz + s];
    __syncwarp();
    for (int j = 0; j < m; j++) {
        const double xj = x[j];
        const int e1 = lp[j + 1];
        for (int p = lp[j] + 1 + lane; p < e1; p += 32) x[li[p]] -= lx[p] * xj;
        __syncwarp();
    }
    for (int j = m - 1; j >= 0; j--) {
        const int u1 = up[j + 1] - 1;
        const double xj = x[j] / ux[u1];
        __syncwarp();
        if (lane == 0) x[j] = xj;
        for (int p = up[j] + lane; p < u1; p += 32) x[ui[p]] -= ux[p] * xj;
        __syncwarp();
    }
    int fin = 1;
    for (int k = lane; k < m; k += 32) fin &= isfinite(x[k]) ? 1 : 0;
    if (!__all_sync(full, fin)) {
        if (lane == 0) v.result[q] = GP_NON_FINITE;
        return;
    }
    // the column order is the identity: the unknowns come out in pivot order
    for (int k = lane; k < m; k += 32) {
        y[(size_t)k * Bz + s] = x[k];
        x[k] = 0.0;
    }
    if (lane == 0) v.result[q] = GP_OK;
}

// ---------------------------------------------------------------------------------------------
// The step of a system whose matrix the factorisation found singular: ILU(0) with the row-relative pivot guard
// (Numerics/Sparse.cs:232-300, NumericTolerances.Ilu0PivotGuard :226-234) and ILU-preconditioned BiCGSTAB with the
// true-residual acceptance (Sparse.cs:305-405), tolerance min(1e-10, tol x 1e-3), at most 4 m + 200 iterations
// (NumericTolerances.cs:256-260), as NewtonShell.SolveStep falls back to (NewtonShell.cs:96-105). It runs on the
// Jacobian in equation order, on the cells of the system's own grid: a cell between two buses exists only while
// one of the branches stamped into it is in service in the system (the reference rebuilds Y without the outage's
// branches). Identity rows (a PV bus's Q row, a reference or removed bus) stay identities through ILU(0) and keep
// their components at zero through BiCGSTAB, so the iteration is that of the reference's reduced system.
// One warp per system, for the listed systems whose result is GP_SINGULAR: GP_ITERATIVE when BiCGSTAB is accepted,
// else GP_SINGULAR stays; a run longer than `budgetNs` gives up as GP_TIMEOUT.
enum : int32_t { GP_ITERATIVE = 4, GP_TIMEOUT = 5 };

struct IterView {
    int m, nnz, nbr;
    const int* rowPtr;   // Jacobian, equation order
    const int* col;
    const int* slot;     // LU slot of each cell
    const int* ycell;    // Y cell between the cell's buses, -1 within one bus
    const int* pinv;     // equation -> pivot position (where y holds its right-hand side and solution)
    const int* ccPtr;    // per Y cell its stamps' owners (branch, or -1 for a shunt)
    const int* ccOwner;
    const int* setBr;    // outage sets: kSetBranches branches each (-1 after the last), ids nbr ...
    const int* outage;   // per system of the batch: branch, set id, or -1
    double tol;
    int maxIter;
    long long budgetNs;
    double* val;         // [nnz] per listed system: ILU(0) values
    double* a;           // [nnz] the matrix's values
    int* present;        // [nnz]
    int* diag;           // [m]
    int* iw;             // [m]
    double* vec;         // [10 m]: x r rhat p v s t ph sh b
    int* result;
};

__device__ __forceinline__ long long gpNowNs() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return (long long)t;
}

// Sums in the reference's order (index order, one accumulator): the null-space component of a singular system's
// BiCGSTAB solution follows its rounding, so the reductions keep the reference's sequence. Lane 0 sums; all get it.
// Products and sums rounded one by one (no fused multiply-add), as the reference's C# evaluates them
__device__ __forceinline__ double fmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double fadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double fsub(double a, double b) { return __dsub_rn(a, b); }

__device__ double gpDot(const double* a, const double* b, int m, int lane) {
    double t = 0.0;
    if (lane == 0)
        for (int i = 0; i < m; i++) t = fadd(t, fmul(a[i], b[i]));
    return __shfl_sync(0xffffffffu, t, 0);
}

__device__ void gpSpMV(const IterView& v, const double* A, const int* pres, const double* x, double* y, int lane) {
    for (int i = lane; i < v.m; i += 32) {
        double t = 0.0;
        for (int q = v.rowPtr[i]; q < v.rowPtr[i + 1]; q++)
            if (pres[q]) t = fadd(t, fmul(A[q], x[v.col[q]]));
        y[i] = t;
    }
    __syncwarp();
}

// z = (LU)^-1 r with the ILU(0) factors (Ilu0.Apply): rows in order, then in reverse, each row's terms subtracted
// one by one in the reference's order (lane 0)
__device__ void gpIluApply(const IterView& v, const double* lu, const int* pres, const int* diag, const double* r,
                           double* z, int lane) {
    if (lane == 0) {
        for (int i = 0; i < v.m; i++) {
            double t = r[i];
            for (int q = v.rowPtr[i]; q < diag[i]; q++)
                if (pres[q]) t = fsub(t, fmul(lu[q], z[v.col[q]]));
            z[i] = t;
        }
        for (int i = v.m - 1; i >= 0; i--) {
            double t = z[i];
            for (int q = diag[i] + 1; q < v.rowPtr[i + 1]; q++)
                if (pres[q]) t = fsub(t, fmul(lu[q], z[v.col[q]]));
            z[i] = t / lu[diag[i]];
        }
    }
    __syncwarp();
}

__global__ void __launch_bounds__(32) k_gp_iterative(IterView v, const double* __restrict__ lu, double* y, int B,
                                                     const int* list, int nList, int nbrSet) {
    const int q = blockIdx.x;
    if (q >= nList || v.result[q] != GP_SINGULAR) return;
    const long long t0 = gpNowNs();
    const int s = list ? list[q] : q;
    const int lane = threadIdx.x;
    const int m = v.m, nnz = v.nnz;
    const size_t Bz = (size_t)B;
    double* val = v.val + (size_t)q * nnz;
    double* A = v.a + (size_t)q * nnz;
    int* pres = v.present + (size_t)q * nnz;
    int* diag = v.diag + (size_t)q * m;
    int* iw = v.iw + (size_t)q * m;
    double* x = v.vec + (size_t)q * 10 * m;
    double *r = x + m, *rhat = r + m, *p = rhat + m, *vv = p + m, *sv = vv + m, *t = sv + m, *ph = t + m, *sh = ph + m,
           *b = sh + m;
    // the outage's branches
    const int o = v.outage[s];
    int outBr[kSetBranches];
    int nOut = 0;
    if (o >= 0 && o < nbrSet) outBr[nOut++] = o;
    else if (o >= nbrSet)
        for (int j = 0; j < kSetBranches; j++) {
            const int br = v.setBr[(size_t)kSetBranches * (o - nbrSet) + j];
            if (br < 0) break;
            outBr[nOut++] = br;
        }
    // the cells of the system's own grid, their values
    for (int c = lane; c < nnz; c += 32) {
        int here = 1;
        const int yc = v.ycell[c];
        if (yc >= 0 && nOut > 0) {
            here = 0;
            for (int e = v.ccPtr[yc]; e < v.ccPtr[yc + 1] && !here; e++) {
                const int ow = v.ccOwner[e];
                bool gone = false;
                for (int j = 0; j < nOut; j++) gone |= ow == outBr[j];
                if (!gone) here = 1;
            }
        }
        pres[c] = here;
        A[c] = lu[(size_t)v.slot[c] * Bz + s];
        val[c] = A[c];
    }
    int noDiag = 0;
    for (int i = lane; i < m; i += 32) {
        iw[i] = -1;
        b[i] = y[(size_t)v.pinv[i] * Bz + s];
        int d = -1;
        for (int c = v.rowPtr[i]; c < v.rowPtr[i + 1]; c++)
            if (v.col[c] == i) d = c;
        diag[i] = d;
        noDiag |= d < 0;
    }
    if (__any_sync(0xffffffffu, noDiag)) return;  // every Jacobian row holds its diagonal cell; stays GP_SINGULAR
    __syncwarp();
    // ILU(0) (Ilu0.Factor)
    for (int i = 0; i < m; i++) {
        const int r0 = v.rowPtr[i], r1 = v.rowPtr[i + 1];
        for (int c = r0 + lane; c < r1; c += 32)
            if (pres[c]) iw[v.col[c]] = c;
        __syncwarp();
        for (int k = r0; k < diag[i]; k++) {
            if (!pres[k]) continue;
            const int j = v.col[k];
            const double piv = val[diag[j]];
            const double lij = piv != 0.0 ? val[k] / piv : 0.0;
            __syncwarp();
            if (lane == 0) val[k] = lij;
            __syncwarp();
            if (lij == 0.0) continue;
            for (int kk = diag[j] + 1 + lane; kk < v.rowPtr[j + 1]; kk += 32) {
                if (!pres[kk]) continue;
                const int pos = iw[v.col[kk]];
                if (pos != -1) val[pos] = fsub(val[pos], fmul(lij, val[kk]));
            }
            __syncwarp();
        }
        double rs = 0.0;
        for (int c = r0 + lane; c < r1; c += 32)
            if (pres[c]) rs = fmax(rs, fabs(A[c]));
        for (int o2 = 16; o2 > 0; o2 >>= 1) rs = fmax(rs, __shfl_xor_sync(0xffffffffu, rs, o2));
        const double guard = 1e-12 * (rs > 0.0 ? rs : 1.0);
        const double d = val[diag[i]];
        __syncwarp();
        if (lane == 0 && fabs(d) < guard) val[diag[i]] = d < 0 ? -guard : guard;
        for (int c = r0 + lane; c < r1; c += 32)
            if (pres[c]) iw[v.col[c]] = -1;
        __syncwarp();
    }
    // BiCGSTAB (BiCgStab)
    for (int i = lane; i < m; i += 32) {
        x[i] = 0.0; r[i] = b[i]; rhat[i] = b[i]; p[i] = 0.0; vv[i] = 0.0;
    }
    __syncwarp();
    const double bnorm = sqrt(gpDot(b, b, m, lane));
    int ok = 0;
    if (bnorm == 0.0) {
        ok = 1;  // b is zero (a NaN makes bnorm NaN, which fails below)
    } else {
        auto trueResidual = [&]() {
            gpSpMV(v, A, pres, x, t, lane);
            double sum = 0.0;
            if (lane == 0)
                for (int i = 0; i < m; i++) { const double d = b[i] - t[i]; sum = fadd(sum, fmul(d, d)); }
            sum = __shfl_sync(0xffffffffu, sum, 0);
            return sqrt(sum) / bnorm < v.tol ? 1 : 0;
        };
        double rho = 1.0, alpha = 1.0, omega = 1.0;
        for (int it = 0; it < v.maxIter; it++) {
            if (gpNowNs() - t0 > v.budgetNs) { ok = -1; break; }
            const double rhoNew = gpDot(rhat, r, m, lane);
            if (fabs(rhoNew) < 1e-300 || isnan(rhoNew)) break;
            const double beta = (rhoNew / rho) * (alpha / omega);
            for (int i = lane; i < m; i += 32) p[i] = fadd(r[i], fmul(beta, fsub(p[i], fmul(omega, vv[i]))));
            __syncwarp();
            gpIluApply(v, val, pres, diag, p, ph, lane);
            gpSpMV(v, A, pres, ph, vv, lane);
            const double rhatV = gpDot(rhat, vv, m, lane);
            if (rhatV == 0.0 || isnan(rhatV)) break;
            alpha = rhoNew / rhatV;
            for (int i = lane; i < m; i += 32) sv[i] = fsub(r[i], fmul(alpha, vv[i]));
            __syncwarp();
            if (sqrt(gpDot(sv, sv, m, lane)) / bnorm < v.tol) {
                for (int i = lane; i < m; i += 32) x[i] = fadd(x[i], fmul(alpha, ph[i]));
                __syncwarp();
                ok = trueResidual();
                break;
            }
            gpIluApply(v, val, pres, diag, sv, sh, lane);
            gpSpMV(v, A, pres, sh, t, lane);
            const double tt = gpDot(t, t, m, lane);
            omega = tt > 0 ? gpDot(t, sv, m, lane) / tt : 0.0;
            for (int i = lane; i < m; i += 32) {
                x[i] = fadd(x[i], fadd(fmul(alpha, ph[i]), fmul(omega, sh[i])));
                r[i] = fsub(sv[i], fmul(omega, t[i]));
            }
            __syncwarp();
            rho = rhoNew;
            if (sqrt(gpDot(r, r, m, lane)) / bnorm < v.tol) { ok = trueResidual(); break; }
            if (omega == 0.0) break;
        }
    }
    if (ok == 1) {
        for (int i = lane; i < m; i += 32) y[(size_t)v.pinv[i] * Bz + s] = x[i];
        if (lane == 0) v.result[q] = GP_ITERATIVE;
    } else if (ok < 0 && lane == 0) {
        v.result[q] = GP_TIMEOUT;
    }
}

}  // namespace gs

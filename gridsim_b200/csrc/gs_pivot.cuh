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
// the matrix is held in pivot order, which is the minimum-degree order of its pattern, the order the reference's
// CpuSparseLuSolver takes (PowerFlow/CpuSparseLuSolver.cs:30-48).
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

}  // namespace gs

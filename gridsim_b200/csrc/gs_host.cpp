// gs_host.cpp — host-only parts of the C ABI: descriptor validation and copy, the symbolic analysis
// without a device, status strings, option defaults.
#include <cmath>
#include <cstring>

#include "gs_host.h"

namespace gs {

std::string CopyGrid(const gs_grid_desc* d, HostGrid& g) {
    if (!d) return "null grid descriptor";
    if (d->n_bus <= 0 || d->n_gen < 0 || d->n_branch < 0) return "bus/generator/branch counts must be positive";
    if (!(d->base_mva > 0) || !std::isfinite(d->base_mva)) return "base_mva must be a finite number above 0";
    const void* need[] = {d->bus_id, d->bus_type, d->pd, d->qd, d->gs, d->bs, d->vm, d->va_deg};
    for (const void* p : need) if (!p) return "a required bus array is null";
    if (d->n_gen > 0 && (!d->gen_bus || !d->pg || !d->qg || !d->vg || !d->qmin || !d->qmax))
        return "a required generator array is null";
    if (d->n_branch > 0 && (!d->br_from || !d->br_to || !d->r || !d->x || !d->b || !d->tap || !d->shift_deg || !d->rate_a))
        return "a required branch array is null";
    int n = d->n_bus;
    g = HostGrid();
    g.n = n; g.ngen = d->n_gen; g.nbr = d->n_branch; g.base = d->base_mva;
    g.busId.assign(d->bus_id, d->bus_id + n);
    g.busType.assign(d->bus_type, d->bus_type + n);
    g.pd.assign(d->pd, d->pd + n); g.qd.assign(d->qd, d->qd + n);
    g.gsh.assign(d->gs, d->gs + n); g.bsh.assign(d->bs, d->bs + n);
    g.vm.assign(d->vm, d->vm + n); g.vaDeg.assign(d->va_deg, d->va_deg + n);
    g.vmin.assign(n, NAN); g.vmax.assign(n, NAN);
    if (d->vmin_pu) g.vmin.assign(d->vmin_pu, d->vmin_pu + n);
    if (d->vmax_pu) g.vmax.assign(d->vmax_pu, d->vmax_pu + n);
    int slack = 0;
    for (int i = 0; i < n; i++) {
        if (g.busType[i] < 1 || g.busType[i] > 3) return "bus_type must be 1 (PQ), 2 (PV) or 3 (slack)";
        if (g.busType[i] == 3) slack++;
        if (!std::isfinite(g.vm[i]) || !std::isfinite(g.vaDeg[i])) return "bus start voltages must be finite";
    }
    if (slack == 0) return "the grid has no slack bus";
    int ng = d->n_gen;
    if (ng > 0) {
        g.genBus.assign(d->gen_bus, d->gen_bus + ng);
        g.pg.assign(d->pg, d->pg + ng); g.qg.assign(d->qg, d->qg + ng); g.vg.assign(d->vg, d->vg + ng);
        g.qmin.assign(d->qmin, d->qmin + ng); g.qmax.assign(d->qmax, d->qmax + ng);
    }
    g.genOn.assign(ng, 1);
    if (d->gen_in_service && ng > 0) g.genOn.assign(d->gen_in_service, d->gen_in_service + ng);
    for (int k = 0; k < ng; k++) if (g.genBus[k] < 0 || g.genBus[k] >= n) return "gen_bus out of range";
    int nb = d->n_branch;
    if (nb > 0) {
        g.brF.assign(d->br_from, d->br_from + nb); g.brT.assign(d->br_to, d->br_to + nb);
        g.r.assign(d->r, d->r + nb); g.x.assign(d->x, d->x + nb); g.b.assign(d->b, d->b + nb);
        g.tap.assign(d->tap, d->tap + nb); g.shift.assign(d->shift_deg, d->shift_deg + nb);
        g.rateA.assign(d->rate_a, d->rate_a + nb);
    }
    g.rateB.assign(nb, 0.0);
    g.rateC.assign(nb, 0.0);
    if (d->rate_b && nb > 0) g.rateB.assign(d->rate_b, d->rate_b + nb);
    if (d->rate_c && nb > 0) g.rateC.assign(d->rate_c, d->rate_c + nb);
    if (d->zip) {  // kept only when some load varies with voltage (ZipLoad.VariesWithVoltage, Model/Model.cs:49)
        bool varies = false;
        for (int i = 0; i < n; i++) {
            const double* c = d->zip + 6 * (size_t)i;
            for (int q = 0; q < 6; q++)
                if (!std::isfinite(c[q])) return "zip coefficients must be finite numbers";
            varies = varies || c[0] != 0 || c[1] != 0 || c[3] != 0 || c[4] != 0;
        }
        if (varies) g.zip.assign(d->zip, d->zip + 6 * (size_t)n);
    }
    g.brOn.assign(nb, 1);
    if (d->br_in_service && nb > 0) g.brOn.assign(d->br_in_service, d->br_in_service + nb);
    for (int k = 0; k < nb; k++) {
        if (g.brF[k] < 0 || g.brF[k] >= n || g.brT[k] < 0 || g.brT[k] >= n) return "branch end out of range";
        if (g.brF[k] == g.brT[k]) return "a branch joins a bus to itself";
        if (g.tap[k] < 0 || std::isnan(g.tap[k])) return "a tap ratio must be 0 (a line) or above";  // AdmittanceStamp.cs:63-66
        // ScreenStateCore refuses a NaN rating A/B/C by name (ContingencyAnalysis.cs:1160-1168)
        if (std::isnan(g.rateA[k]) || std::isnan(g.rateB[k]) || std::isnan(g.rateC[k]))
            return "a rating must be 0 (unrated) or a number above 0";
        if (g.r[k] == 0 && g.x[k] == 0) return "a branch has zero impedance";
    }
    // boundaries (Model/Model.cs:516-560; the limit rule of BoundaryAnalysis.EvaluateAfterOutage :60-62, the
    // direction rule of JsonGridLoader.cs:219-223)
    if (d->n_boundary < 0) return "n_boundary must be 0 or more";
    g.nBnd = d->n_boundary;
    g.bndPtr.assign(1, 0);
    if (g.nBnd > 0) {
        if (!d->bnd_ptr || !d->bnd_limit_mw) return "a required boundary array is null";
        if (d->bnd_ptr[0] != 0) return "bnd_ptr[0] must be 0";
        for (int q = 0; q < g.nBnd; q++)
            if (d->bnd_ptr[q + 1] < d->bnd_ptr[q]) return "bnd_ptr must not decrease";
        const int nm = d->bnd_ptr[g.nBnd];
        if (nm > 0 && (!d->bnd_branch || !d->bnd_dir)) return "a required boundary array is null";
        g.bndPtr.assign(d->bnd_ptr, d->bnd_ptr + g.nBnd + 1);
        g.bndBranch.assign(d->bnd_branch, d->bnd_branch + nm);
        g.bndDir.assign(d->bnd_dir, d->bnd_dir + nm);
        g.bndLimit.assign(d->bnd_limit_mw, d->bnd_limit_mw + g.nBnd);
        for (int e = 0; e < nm; e++) {
            if (g.bndBranch[e] < 0 || g.bndBranch[e] >= nb) return "a boundary names a branch out of range";
            if (g.bndDir[e] != 1 && g.bndDir[e] != -1) return "a boundary branch direction must be 1 or -1";
        }
        for (int q = 0; q < g.nBnd; q++)
            if (!std::isfinite(g.bndLimit[q]) || g.bndLimit[q] < 0)
                return "a boundary transfer limit must be a finite non-negative MW value (0 = no limit set)";
    }
    return "";
}

void FillInfo(const HostGrid& g, const Symbolic& s, gs_grid_info* info) {
    std::memset(info, 0, sizeof(*info));
    info->n_bus = g.n;
    info->n_branch = g.nbr;
    info->n_pv = s.npv;
    info->n_pq = s.npq;
    info->m = s.m;
    info->nnz_y = s.nnzY;
    info->nnz_j = s.nnzJ;
    info->nnz_lu = s.nnzLU;
    info->lu_flops = s.flops;
    info->n_levels = s.nLevels;
}

}  // namespace gs

extern "C" {

int gs_abi_version(void) { return GS_ABI_VERSION; }

const char* gs_status_str(int st) {
    switch (st) {
        case GS_OK: return "ok";
        case GS_ERR_INVALID_ARG: return "invalid argument";
        case GS_ERR_CUDA: return "CUDA error";
        case GS_ERR_OOM: return "out of device memory";
        case GS_ERR_NO_DEVICE: return "no usable CUDA device";
        case GS_ERR_TIMEOUT: return "timed out";
        case GS_ERR_STATE: return "wrong call order";
        case GS_ERR_UNSUPPORTED: return "unsupported option";
        case GS_ERR_INTERNAL: return "internal error";
        case GS_ERR_CAPACITY: return "output capacity too small";
        default: return "unknown status";
    }
}

void gs_pf_opts_default(gs_pf_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->tolerance = 1e-8;        // PowerFlowOptions.cs:20-32
    o->diverge_limit_pu = 10.0; // :92
    o->max_iterations = 30;     // :53-65
    o->precision = GS_PREC_FP64;
}

int gs_analyze_host(const gs_grid_desc* desc, gs_grid_info* info) {
    if (!info) return GS_ERR_INVALID_ARG;
    gs::HostGrid g;
    if (!gs::CopyGrid(desc, g).empty()) return GS_ERR_INVALID_ARG;
    gs::Symbolic s;
    if (!gs::Analyze(g, s).empty()) return GS_ERR_INVALID_ARG;
    gs::FillInfo(g, s, info);
    return GS_OK;
}

}  // extern "C"

// Batched 2D2V steps: many independent runs of uneven sizes advanced in
// lockstep, one launch per substep for all runs.
//
// vp_batch2d_plan resolves everything a step needs into one flat table of
// plain argument blocks (the same blocks the single-run kernels take) plus
// per-sweep item offsets; the caller copies the table to the device once.
// vp_batch2d_step then only launches kernels whose arguments point into the
// device copy (the fused runs' tensor maps are copied from the host table
// into the plane kernels' parameters), so a sequence of steps is capturable
// in a CUDA graph. The runs whose layout the fused drift pairs take (FP32,
// 32 <= ny <= 64 a multiple of 8, nvy a multiple of 16; several column
// groups of a run per CTA) make three passes over f: x then y with the rho partials
// (f -> s2), the fused kick (s2 -> s1), y then x (s1 -> f); the others one
// sweep per axis: x (f -> s1), y + rho partials (s1 -> s2), kick (s2 -> s1),
// y (s1 -> s2), x (s2 -> f). Each kind of pass is one launch for all runs
// that take it, plus the rho finalize, 3 Poisson kernels and the
// diagnostics: at most 14 launches per step for up to 64 runs (the fused
// passes launch once per box class and per 64 runs: their tensor maps are
// launch parameters; the launches of a pass chain as programmatic dependents).
// Every run's arithmetic is that of vp_step2d (same item bodies, same
// weights, same reduction order for the default tile shapes).
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "launch.h"

namespace vp {

namespace {

constexpr char kMagic[8] = {'V', 'P', 'B', 'A', 'T', 'C', 'H', '1'};

struct BatchHeader {
    char magic[8];
    int32_t n_runs, dtype, phys, diag;
    int32_t vec_x, nt_x, wrap_x;  // x drifts
    int32_t vec_y, nt_y, wrap_y;  // y drifts
    int32_t vec_k;                // fused kick
    int32_t block[VP_BATCH_KINDS];
    int32_t grid[VP_BATCH_KINDS];  // persistent CTAs of each sweep kind
    int32_t max_nx, max_ny;
    int64_t max_points;  // max nx*ny
    int64_t kick_smem;
    // byte offsets of the arrays inside the table
    int64_t off_x1, off_y1, off_y2, off_x2;  // StridedArgs[n]
    int64_t off_start_x, off_start_y1, off_start_y2, off_start_k;  // int64[n+1]
    int64_t off_kick;  // Kick2dArgs[n]
    int64_t off_pois;  // Pois2dRun[n]
    int64_t off_rfin;  // RhoFinRun[n]
    int64_t off_diag;  // DiagArgs[n]
    int64_t off_p1, off_p2;    // plane-pass records (x then y, y then x), 64-byte aligned
    int32_t n_plane, n_plane_full;  // fused runs: records 0 .. n_plane - 1, whole-box ones first,
                                    // longest lines first in each class
    int64_t off_sp1, off_sp2;  // int64[n+1]: prefix sums of the two passes' plane items over the records
    int64_t plane_items1, plane_items2;  // all runs' plane items (0: no fused runs)
    int32_t p1_slab_rows, p2_slab_rows;  // the largest ring slab of the fused runs
    int64_t sweep_items;     // all runs' x-drift items (0: every run fused)
    int64_t total_bytes;
};

size_t al16(size_t b) { return (b + 15) & ~size_t(15); }
size_t al64(size_t b) { return (b + 63) & ~size_t(63); }

struct Layout {
    int64_t off_x1, off_y1, off_y2, off_x2, off_sx, off_sy1, off_sy2, off_sk, off_kick, off_pois, off_rfin, off_diag,
        off_p1, off_p2, off_sp1, off_sp2, total;
};

Layout layout_for(int n) {
    Layout L;
    size_t off = al16(sizeof(BatchHeader));
    auto take = [&](size_t b) {
        const size_t o = off;
        off += al16(b);
        return (int64_t)o;
    };
    L.off_x1 = take(sizeof(StridedArgs) * n);
    L.off_y1 = take(sizeof(StridedArgs) * n);
    L.off_y2 = take(sizeof(StridedArgs) * n);
    L.off_x2 = take(sizeof(StridedArgs) * n);
    L.off_sx = take(sizeof(int64_t) * (n + 1));
    L.off_sy1 = take(sizeof(int64_t) * (n + 1));
    L.off_sy2 = take(sizeof(int64_t) * (n + 1));
    L.off_sk = take(sizeof(int64_t) * (n + 1));
    L.off_kick = take(sizeof(Kick2dArgs) * n);
    L.off_pois = take(sizeof(Pois2dRun) * n);
    L.off_rfin = take(sizeof(RhoFinRun) * n);
    L.off_diag = take(sizeof(DiagArgs) * n);
    L.off_sp1 = take(sizeof(int64_t) * (n + 1));
    L.off_sp2 = take(sizeof(int64_t) * (n + 1));
    off = al64(off);  // tensor maps inside the plane records need 64-byte alignment
    L.off_p1 = (int64_t)off;
    off += al64(plane_run_bytes() * n);
    L.off_p2 = (int64_t)off;
    off += al64(plane_run_bytes() * n);
    L.total = (int64_t)off;
    return L;
}

template <typename T>
T* at(void* base, int64_t off) {
    return reinterpret_cast<T*>(static_cast<char*>(base) + off);
}
template <typename T>
const T* at(const void* base, int64_t off) {
    return reinterpret_cast<const T*>(static_cast<const char*>(base) + off);
}

int grid_for(int ctas_per_sm, int64_t items) {
    const int per_sm = ctas_per_sm > 0 ? ctas_per_sm : 2;  // the sweeps' occupancy limit
    return (int)std::max<int64_t>(1, std::min<int64_t>(items, (int64_t)sm_count() * per_sm));
}

}  // namespace
}  // namespace vp

using namespace vp;

extern "C" {

size_t vp_batch2d_table_bytes(int32_t n_runs) {
    if (n_runs <= 0) return 0;
    return (size_t)layout_for(n_runs).total;
}

int vp_batch2d_plan(int32_t dtype, int32_t physics_mode, int32_t diagnostics, const vp_batch2d_run* runs,
                    int32_t n_runs, const vp_batch_tiles* tiles, void* table, size_t table_bytes) {
    if (dtype != VP_F32 && dtype != VP_F64 && dtype != VP_BF16)
        return set_error(VP_ERR_DTYPE, "vp_batch2d_plan: unknown dtype");
    if (!runs || !table || n_runs <= 0) return set_error(VP_ERR_ARG, "vp_batch2d_plan: null pointer or no runs");
    if (table_bytes < vp_batch2d_table_bytes(n_runs))
        return set_error(VP_ERR_WORKSPACE, "vp_batch2d_plan: table too small");
    if (diagnostics != 0 && diagnostics != 1)
        return set_error(VP_ERR_ARG, "vp_batch2d_plan: diagnostics must be 0 or 1");
    if (diagnostics && !physics_mode)
        return set_error(VP_ERR_UNSUPPORTED, "vp_batch2d_plan: diagnostics need physics_mode");
    int32_t block[VP_BATCH_KINDS], per_sm[VP_BATCH_KINDS], segs[VP_BATCH_KINDS];
    for (int k = 0; k < VP_BATCH_KINDS; ++k) {
        block[k] = tiles && tiles->block[k] ? tiles->block[k] : 256;
        per_sm[k] = tiles ? tiles->ctas_per_sm[k] : 0;
        segs[k] = tiles && tiles->segments[k] ? tiles->segments[k] : 1;
        if (block[k] != 128 && block[k] != 256)
            return set_error(VP_ERR_ARG, "vp_batch2d_plan: tile block must be 128 or 256");
        if (per_sm[k] < 0 || per_sm[k] > 2)
            return set_error(VP_ERR_ARG, "vp_batch2d_plan: ctas_per_sm must be 0, 1 or 2");
        if (segs[k] != 1 && segs[k] != 2 && segs[k] != 4)
            return set_error(VP_ERR_ARG, "vp_batch2d_plan: segments must be 1, 2 or 4");
    }
    const Layout L = layout_for(n_runs);
    std::memset(table, 0, (size_t)L.total);
    BatchHeader h{};
    std::memcpy(h.magic, kMagic, 8);
    h.n_runs = n_runs;
    h.dtype = dtype;
    h.phys = physics_mode ? 1 : 0;
    h.diag = diagnostics;
    const bool phys = h.phys != 0;
    StridedArgs* x1 = at<StridedArgs>(table, L.off_x1);
    StridedArgs* y1 = at<StridedArgs>(table, L.off_y1);
    StridedArgs* y2 = at<StridedArgs>(table, L.off_y2);
    StridedArgs* x2 = at<StridedArgs>(table, L.off_x2);
    Kick2dArgs* kk = at<Kick2dArgs>(table, L.off_kick);
    Pois2dRun* pr = at<Pois2dRun>(table, L.off_pois);
    RhoFinRun* rf = at<RhoFinRun>(table, L.off_rfin);
    DiagArgs* dg = at<DiagArgs>(table, L.off_diag);
    int vx_min = 4, ntx_min = 7, vy_min = 4, nty_min = 7, vk_min = 4;
    bool wrap_x = false, wrap_y = false;  // some run sweeps whole lines of a multiple of 8 rows
    const bool sweeps_only = tiles && tiles->sweeps_only;
    int64_t* sp1 = at<int64_t>(table, L.off_sp1);
    int64_t* sp2 = at<int64_t>(table, L.off_sp2);
    std::vector<char> fused(n_runs, 0);
    sp1[0] = sp2[0] = 0;
    int slab1 = 0, slab2 = 0;
    for (int r = 0; r < n_runs; ++r) {
        const vp_batch2d_run& d = runs[r];
        if (d.nx <= 0 || d.ny <= 0 || d.nvx <= 1 || d.nvy <= 1)
            return set_error(VP_ERR_ARG, "vp_batch2d_plan: bad run size");
        if (!d.f || !d.s1 || !d.s2 || d.f == d.s1 || d.f == d.s2 || d.s1 == d.s2)
            return set_error(VP_ERR_ARG, "vp_batch2d_plan: f, s1, s2 must be distinct non-null buffers");
        if (!d.shift_x || !d.W_x || !d.shift_y || !d.W_y)
            return set_error(VP_ERR_ARG, "vp_batch2d_plan: null drift table");
        if (phys && (!d.kx || !d.ky || !d.inv_ksq))
            return set_error(VP_ERR_ARG, "vp_batch2d_plan: null spectral arrays");
        if (d.dvx == 0.0 || d.dvy == 0.0) return set_error(VP_ERR_ARG, "vp_batch2d_plan: zero velocity spacing");
        if (d.test_stall != 0 && d.test_stall != 1) return set_error(VP_ERR_ARG, "vp_batch2d_plan: test_stall must be 0 or 1");
        for (int sg : {d.segments_x, d.segments_y})
            if (sg != 0 && sg != 1 && sg != 2 && sg != 4)
                return set_error(VP_ERR_ARG, "vp_batch2d_plan: run segments must be 0, 1, 2 or 4");
        if (d.nx > 4096 || d.ny > 1024)
            return set_error(VP_ERR_ARG, "vp_batch2d_plan: nx must be <= 4096 and ny <= 1024");
        if (phys && !poisson2d_fits(d.nx, d.ny))
            return set_error(VP_ERR_UNSUPPORTED, "vp_batch2d_plan: a run's field solve needs nx below about 1800 "
                                                 "and ny below about 3600 (shared memory)");
        const size_t need = step2d_layout(d.nx, d.ny, d.nvx, d.nvy, nullptr, nullptr);
        if (!d.workspace || d.workspace_bytes < need)
            return set_error(VP_ERR_WORKSPACE, "vp_batch2d_plan: run workspace too small");
        if (phys && !kick2d_fits(dtype, d.nvy, d.f, d.s1, d.s2))
            return set_error(VP_ERR_UNSUPPORTED, "vp_batch2d_plan: a plane row must fit one warp (nvy <= 128)");
        Step2dWs w;
        step2d_layout(d.nx, d.ny, d.nvx, d.nvy, static_cast<char*>(d.workspace), &w);
        const int64_t nx = d.nx, ny = d.ny, nvx = d.nvx, nvy = d.nvy;
        const bool want_rho = phys || diagnostics;
        // the fused drift pairs: f -> s2 (x then y, the rho partials), then
        // s1 -> f (after the kick) or s2 -> f (without it)
        fused[r] = !sweeps_only && plane_batch_fits(dtype, nx, ny, nvx, nvy, d.f, d.s1, d.s2);
        int v, nt;
        // x drifts: f -> s1 and s2 -> f (with the kicks) or s1 -> f (without)
        strided_batch_args(dtype, d.f, d.s1, 1, nx, ny * nvx * nvy, nvy, nvx, d.shift_spread_x, d.shift_x, d.W_x,
                           nullptr, block[0], &x1[r], &v, &nt);
        if (!fused[r]) {
            vx_min = std::min(vx_min, v);
            ntx_min = std::min(ntx_min, nt);
        }
        void* last_src = phys ? d.s2 : d.s1;
        strided_batch_args(dtype, last_src, d.f, 1, nx, ny * nvx * nvy, nvy, nvx, d.shift_spread_x, d.shift_x,
                           d.W_x, nullptr, block[0], &x2[r], &v, &nt);
        if (!fused[r]) {
            vx_min = std::min(vx_min, v);
            ntx_min = std::min(ntx_min, nt);
        }
        // y drifts: s1 -> s2 (+rho), then s1 -> s2 (kicks) or s2 -> s1 (no kicks)
        strided_batch_args(dtype, d.s1, d.s2, nx, ny, nvx * nvy, 1, nvy, d.shift_spread_y, d.shift_y, d.W_y,
                           want_rho ? w.part : nullptr, block[1], &y1[r], &v, &nt);
        if (!fused[r]) {
            vy_min = std::min(vy_min, v);
            nty_min = std::min(nty_min, nt);
        }
        strided_batch_args(dtype, phys ? d.s1 : d.s2, phys ? d.s2 : d.s1, nx, ny, nvx * nvy, 1, nvy,
                           d.shift_spread_y, d.shift_y, d.W_y, nullptr, block[1], &y2[r], &v, &nt);
        if (!fused[r]) {
            vy_min = std::min(vy_min, v);
            nty_min = std::min(nty_min, nt);
        }
        if (phys) {
            kick2d_batch_args(dtype, d.s2, d.s1, nx * ny, nvx, nvy, w.ex, w.ey, d.dt, d.dvx, d.dvy, d.window, &kk[r],
                              &v);
            vk_min = std::min(vk_min, v);
            pois2d_run_args(w.rho, nx, ny, d.kx, d.ky, d.inv_ksq, w.ex, w.ey, d.drho, d.phi, w.pois, &pr[r],
                            nullptr);
        }
        rf[r].part = w.part;
        rf[r].n_outer = nx;
        rf[r].n_line = (int)ny;
        rf[r].scale = d.dvx * d.dvy;
        rf[r].offset = 0.0;
        rf[r].rho = w.rho;
        if (diagnostics) {
            DiagArgs& a = dg[r];
            a.mass_part = pr[r].mass_part;
            a.n_mass = (int)nx;
            a.we_part = pr[r].we_part;
            a.n_we = (int)nx;
            a.emax_part = pr[r].emax_part;
            a.n_emax = (int)nx;
            a.mass_scale = d.dx * d.dy;
            a.we_scale = 0.5 * d.dx * d.dy;
            a.dv_scale = d.dx * d.dy * d.dvx * d.dvy;
            a.shift_x = d.dt / d.dvx;
            a.shift_y = d.dt / d.dvy;
            a.diag = d.diag;
            a.slot_stride = d.diag_slot_stride;
            a.status = d.status;
        }
        h.max_nx = std::max<int32_t>(h.max_nx, d.nx);
        h.max_ny = std::max<int32_t>(h.max_ny, d.ny);
        h.max_points = std::max<int64_t>(h.max_points, nx * ny);
        const int sgx = d.segments_x ? d.segments_x : segs[0];
        const int sgy = d.segments_y ? d.segments_y : segs[1];
        wrap_x = wrap_x || (sgx == 1 && nx % 8 == 0);
        wrap_y = wrap_y || (sgy == 1 && ny % 8 == 0);
    }
    // one kernel variant per sweep kind: the widest form every run supports
    const int pref = strided_batch_pref_vec(dtype);
    h.vec_x = vx_min >= pref ? pref : 1;
    h.nt_x = 6;  // the x shift follows vx, shared by the VEC columns of a thread
    (void)ntx_min;
    h.vec_y = vy_min >= pref ? pref : 1;
    h.nt_y = (h.vec_y == pref && nty_min == 7) ? 7 : 6;
    if (h.vec_y == pref && nty_min != 7) h.vec_y = 1;  // per-element weights need the 7-row form
    h.vec_k = vk_min;
    h.wrap_x = wrap_x;
    h.wrap_y = wrap_y;
    int64_t* sx = at<int64_t>(table, L.off_sx);
    int64_t* sy1 = at<int64_t>(table, L.off_sy1);
    int64_t* sy2 = at<int64_t>(table, L.off_sy2);
    int64_t* sk = at<int64_t>(table, L.off_sk);
    sx[0] = sy1[0] = sy2[0] = sk[0] = 0;
    int64_t kick_smem = 0;
    for (int r = 0; r < n_runs; ++r) {
        const int sgx = runs[r].segments_x ? runs[r].segments_x : segs[0];
        const int sgy = runs[r].segments_y ? runs[r].segments_y : segs[1];
        for (StridedArgs* a : {&x1[r], &x2[r]}) {
            strided_batch_finish(a, h.vec_x, block[0]);
            a->seg = (a->n_line + sgx - 1) / sgx;
            a->nseg = (a->n_line + a->seg - 1) / a->seg;
            a->items *= a->nseg;
        }
        for (StridedArgs* a : {&y1[r], &y2[r]}) {
            strided_batch_finish(a, h.vec_y, block[1]);
            a->seg = (a->n_line + sgy - 1) / sgy;
            a->nseg = (a->n_line + a->seg - 1) / a->seg;
            a->items *= a->nseg;
        }
        rf[r].tiles = y1[r].tiles;
        if (fused[r]) {
            // no sweeps for this run; its density partials are per group
            for (StridedArgs* a : {&x1[r], &x2[r], &y1[r], &y2[r]}) a->items = 0;
            rf[r].tiles = (int)plane_part_tiles(runs[r].nvx, runs[r].nvy);
        }
        sx[r + 1] = sx[r] + x1[r].items;
        sy1[r + 1] = sy1[r] + y1[r].items;
        sy2[r + 1] = sy2[r] + y2[r].items;
        if (phys) {
            int64_t items = 0;
            if (kk[r].nvy / h.vec_k > 32)
                return set_error(VP_ERR_UNSUPPORTED, "vp_batch2d_plan: runs need different kick vector widths");
            kick_smem = std::max<int64_t>(kick_smem, kick2d_batch_finish(&kk[r], dtype, h.vec_k, block[2], &items));
            sk[r + 1] = sk[r] + items;
        } else {
            sk[r + 1] = sk[r];
        }
    }
    // the fused runs' plane records, longest lines first: a CTA takes the
    // packs b, b + G, ... of the launch in record order, so that each round
    // deals packs of about one length (C4: the longest CTA share 387 row
    // steps against 435 in run order, 346 the even share)
    std::vector<int> order;
    for (int r = 0; r < n_runs; ++r)
        if (fused[r]) order.push_back(r);
    // runs with nvy % 32 == 0 first (whole-box launch), then the others (half boxes)
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        const bool ha = runs[a].nvy % 32 != 0, hb = runs[b].nvy % 32 != 0;
        return ha != hb ? !ha : runs[a].nx > runs[b].nx;
    });
    int n_full = 0;
    for (int r : order) n_full += runs[r].nvy % 32 == 0 ? 1 : 0;
    for (size_t i = 0; i < order.size(); ++i) {
        const int r = order[i];
        const vp_batch2d_run& d = runs[r];
        Step2dWs w;
        step2d_layout(d.nx, d.ny, d.nvx, d.nvy, static_cast<char*>(d.workspace), &w);
        int64_t items1 = 0, items2 = 0;
        int rows1 = 0, rows2 = 0;
        int rc = plane_batch_run(static_cast<char*>(table) + L.off_p1 + i * plane_run_bytes(), true, d.f, d.s2, d.nx,
                                 d.ny, d.nvx, d.nvy, d.shift_x, d.W_x, d.shift_y, d.W_y,
                                 (phys || diagnostics) ? w.part : nullptr, d.status, d.test_stall, &items1, &rows1);
        if (!rc)
            rc = plane_batch_run(static_cast<char*>(table) + L.off_p2 + i * plane_run_bytes(), false,
                                 phys ? d.s1 : d.s2, d.f, d.nx, d.ny, d.nvx, d.nvy, d.shift_x, d.W_x, d.shift_y,
                                 d.W_y, nullptr, d.status, d.test_stall, &items2, &rows2);
        if (rc) return rc;
        slab1 = std::max(slab1, rows1);
        slab2 = std::max(slab2, rows2);
        sp1[i + 1] = sp1[i] + items1;
        sp2[i + 1] = sp2[i] + items2;
    }
    h.n_plane = (int32_t)order.size();
    h.n_plane_full = n_full;
    for (int k = 0; k < VP_BATCH_KINDS; ++k) h.block[k] = block[k];
    h.grid[0] = grid_for(per_sm[0], sx[n_runs]);
    h.grid[1] = grid_for(per_sm[1], std::max(sy1[n_runs], sy2[n_runs]));
    h.grid[2] = grid_for(per_sm[2], std::max<int64_t>(sk[n_runs], 1));
    h.kick_smem = kick_smem;
    h.plane_items1 = sp1[h.n_plane];
    h.plane_items2 = sp2[h.n_plane];
    h.p1_slab_rows = slab1;
    h.p2_slab_rows = slab2;
    h.sweep_items = sx[n_runs];
    h.off_p1 = L.off_p1;
    h.off_p2 = L.off_p2;
    h.off_sp1 = L.off_sp1;
    h.off_sp2 = L.off_sp2;
    h.off_x1 = L.off_x1;
    h.off_y1 = L.off_y1;
    h.off_y2 = L.off_y2;
    h.off_x2 = L.off_x2;
    h.off_start_x = L.off_sx;
    h.off_start_y1 = L.off_sy1;
    h.off_start_y2 = L.off_sy2;
    h.off_start_k = L.off_sk;
    h.off_kick = L.off_kick;
    h.off_pois = L.off_pois;
    h.off_rfin = L.off_rfin;
    h.off_diag = L.off_diag;
    h.total_bytes = L.total;
    std::memcpy(table, &h, sizeof(h));
    return VP_OK;
}

int vp_batch2d_step(const void* table, const void* table_dev, int32_t slot, void* const* events, void* stream) {
    if (!table || !table_dev) return set_error(VP_ERR_ARG, "vp_batch2d_step: null table");
    BatchHeader h;
    std::memcpy(&h, table, sizeof(h));
    if (std::memcmp(h.magic, kMagic, 8) != 0) return set_error(VP_ERR_ARG, "vp_batch2d_step: not a batch table");
    if (slot < 0) return set_error(VP_ERR_ARG, "vp_batch2d_step: negative slot");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int n = h.n_runs;
    const int64_t* sx = at<int64_t>(table_dev, h.off_start_x);
    const int64_t* sy1 = at<int64_t>(table_dev, h.off_start_y1);
    const int64_t* sy2 = at<int64_t>(table_dev, h.off_start_y2);
    const int64_t* sk = at<int64_t>(table_dev, h.off_start_k);
    int rc;
    auto mark = [&](int i) -> int {
        if (!events || !events[i]) return VP_OK;
        if (cudaEventRecord(static_cast<cudaEvent_t>(events[i]), st) != cudaSuccess)
            return set_cuda_error("cudaEventRecord(timing event)");
        return VP_OK;
    };
    const bool want_rho = h.phys || h.diag;
    const bool sweeps = h.sweep_items > 0;
    const int64_t* sp1 = at<int64_t>(table_dev, h.off_sp1);
    const int64_t* sp2 = at<int64_t>(table_dev, h.off_sp2);
    // the fused runs: x then y (dt/2 each) with the rho partials, f -> s2;
    // the others: x drift (dt/2), f -> s1
    if ((rc = mark(2 * VP_PHASE_DRIFT_X1))) return rc;
    rc = launch_plane_batch(true, want_rho, at<char>(table_dev, h.off_p1), at<char>(table, h.off_p1), sp1,
                            at<int64_t>(table, h.off_sp1), h.n_plane_full, h.n_plane, h.plane_items1, h.p1_slab_rows,
                            st);
    if (rc) return rc;
    // the other runs' x sweep starts its CTAs as the plane pass's leave
    const bool after_planes = h.n_plane > 0;
    if (sweeps) {
        rc = launch_strided_batch(h.dtype, h.vec_x, h.nt_x, false, h.wrap_x, at<StridedArgs>(table_dev, h.off_x1), sx,
                                  n, h.block[0], h.grid[0], 0, after_planes, st);
        if (rc) return rc;
    }
    if ((rc = mark(2 * VP_PHASE_DRIFT_X1 + 1)) || (rc = mark(2 * VP_PHASE_DRIFT_Y1))) return rc;
    // y drift (dt/2) fused with the rho partials: s1 -> s2
    if (sweeps) {
        rc = launch_strided_batch(h.dtype, h.vec_y, h.nt_y, want_rho, h.wrap_y && !want_rho,
                                  at<StridedArgs>(table_dev, h.off_y1), sy1, n, h.block[1], h.grid[1], h.max_ny, false,
                                  st);
        if (rc) return rc;
    }
    if (h.phys) {
        if ((rc = launch_rho_finalize_batch(at<RhoFinRun>(table_dev, h.off_rfin), n, h.max_nx, h.max_ny, st))) return rc;
    }
    if ((rc = mark(2 * VP_PHASE_DRIFT_Y1 + 1)) || (rc = mark(2 * VP_PHASE_FIELD))) return rc;
    if (h.phys) {
        if ((rc = launch_poisson2d_batch(at<Pois2dRun>(table_dev, h.off_pois), n, h.max_nx, h.max_ny, st)))
            return rc;
    }
    if ((rc = mark(2 * VP_PHASE_FIELD + 1)) || (rc = mark(2 * VP_PHASE_KICK))) return rc;
    if (h.phys) {
        // vx(dt) + vy(dt): s2 -> s1
        rc = launch_kick2d_batch(h.dtype, h.vec_k, at<Kick2dArgs>(table_dev, h.off_kick), sk, n, h.block[2],
                                 h.grid[2], (size_t)h.kick_smem, st);
        if (rc) return rc;
    }
    if ((rc = mark(2 * VP_PHASE_KICK + 1)) || (rc = mark(2 * VP_PHASE_DRIFT_Y2))) return rc;
    // y drift (dt/2)
    if (sweeps) {
        rc = launch_strided_batch(h.dtype, h.vec_y, h.nt_y, false, h.wrap_y, at<StridedArgs>(table_dev, h.off_y2), sy2,
                                  n, h.block[1], h.grid[1], 0, false, st);
        if (rc) return rc;
    }
    if ((rc = mark(2 * VP_PHASE_DRIFT_Y2 + 1)) || (rc = mark(2 * VP_PHASE_DRIFT_X2))) return rc;
    // the fused runs: y then x back into f; the others: x drift back into f
    rc = launch_plane_batch(false, false, at<char>(table_dev, h.off_p2), at<char>(table, h.off_p2), sp2,
                            at<int64_t>(table, h.off_sp2), h.n_plane_full, h.n_plane, h.plane_items2, h.p2_slab_rows,
                            st);
    if (rc) return rc;
    if (sweeps) {
        rc = launch_strided_batch(h.dtype, h.vec_x, h.nt_x, false, h.wrap_x, at<StridedArgs>(table_dev, h.off_x2), sx,
                                  n, h.block[0], h.grid[0], 0, after_planes, st);
        if (rc) return rc;
    }
    if ((rc = mark(2 * VP_PHASE_DRIFT_X2 + 1)) || (rc = mark(2 * VP_PHASE_DIAG))) return rc;
    if (h.diag && (rc = launch_diag_finalize_batch(at<DiagArgs>(table_dev, h.off_diag), n, slot, st))) return rc;
    return mark(2 * VP_PHASE_DIAG + 1);
}

}  // extern "C"

// Batches of independent problems (no reference counterpart: the reference builds one
// Elliptic::Problem per design and load case, src/elliptic/Problem.hpp:80-140).
//
// A batch is created from P problem descriptions and stored as ONE handle over the disjoint
// union of their meshes: member s's nodes, cells, essential-BC dofs and traction faces are
// offset by the sizes of members 0..s-1.  Every element kernel, the block pattern, the
// assembly, the Dirichlet elimination and the SELL conversions run unchanged over the union
// (its block pattern is the members' patterns on the diagonal), so one launch per stage
// serves all members.  Only the Krylov solver and the criterion value need member-wise
// reductions (fcg_batch in mixed.cu, launch_energy_segments in element_kernels.cu).
#include <algorithm>
#include <cmath>
#include <vector>

#include "plato_internal.cuh"

namespace plato {

int solve_state(plato_problem* h, const double* z, const double* u0, double* u, plato_solve_stats* st);

void batch_release(plato_problem* h) {
    BatchState& b = h->batch;
    for (int32_t** p : {&b.cta_seg, &b.cta_row0, &b.cta_row1, &b.seg_cta0, &b.cell_off_d, &b.ndone})
        if (*p) { cudaFree(*p); *p = nullptr; }
    for (double** p : {&b.partials, &b.values})
        if (*p) { cudaFree(*p); *p = nullptr; }
    if (b.S) { cudaFree(b.S); b.S = nullptr; }
    if (b.S_host) { cudaFreeHost(b.S_host); b.S_host = nullptr; }
    b.nseg = 0;
}

namespace {

// Tiles of at most b.tile_rows rows that never straddle two members; inside a member the
// tiles after the first start on multiples of tile_rows (aligned with the SELL slices).
// Rebuilt when the autotuner changes the tile size.
void free_tiles(BatchState& b) {
    for (int32_t** p : {&b.cta_seg, &b.cta_row0, &b.cta_row1, &b.seg_cta0})
        if (*p) { cudaFree(*p); *p = nullptr; }
    if (b.partials) { cudaFree(b.partials); b.partials = nullptr; }
}

int setup_tiles(plato_problem* h) {
    BatchState& b = h->batch;
    const int64_t T = b.tile_rows;
    free_tiles(b);
    std::vector<int32_t> seg, r0, r1, first(b.nseg + 1, 0);
    for (int s = 0; s < b.nseg; ++s) {
        first[s] = int32_t(seg.size());
        int64_t a = b.node_off[s];
        const int64_t e = b.node_off[s + 1];
        while (a < e) {
            const int64_t next = std::min<int64_t>(e, (a / T + 1) * T);
            seg.push_back(s);
            r0.push_back(int32_t(a));
            r1.push_back(int32_t(next));
            a = next;
        }
    }
    first[b.nseg] = int32_t(seg.size());
    b.ncta = int32_t(seg.size());
    PLATO_CUDA(h, cudaMalloc(&b.cta_seg, sizeof(int32_t) * b.ncta));
    PLATO_CUDA(h, cudaMalloc(&b.cta_row0, sizeof(int32_t) * b.ncta));
    PLATO_CUDA(h, cudaMalloc(&b.cta_row1, sizeof(int32_t) * b.ncta));
    PLATO_CUDA(h, cudaMalloc(&b.seg_cta0, sizeof(int32_t) * (b.nseg + 1)));
    PLATO_CUDA(h, cudaMalloc(&b.partials, sizeof(double) * 2 * b.ncta));
    if (!b.cell_off_d) PLATO_CUDA(h, cudaMalloc(&b.cell_off_d, sizeof(int32_t) * (b.nseg + 1)));
    if (!b.ndone) PLATO_CUDA(h, cudaMalloc(&b.ndone, sizeof(int32_t)));
    if (!b.values) PLATO_CUDA(h, cudaMalloc(&b.values, sizeof(double) * size_t(b.nseg) * kEnergySplit));
    if (!b.S) {
        PLATO_CUDA(h, cudaMalloc(&b.S, sizeof(SegScalars) * b.nseg));
        PLATO_CUDA(h, cudaMemset(b.S, 0, sizeof(SegScalars) * b.nseg));
    }
    if (!b.S_host) PLATO_CUDA(h, cudaMallocHost(reinterpret_cast<void**>(&b.S_host), sizeof(SegScalars) * b.nseg));
    PLATO_CUDA(h, cudaMemcpy(b.cta_seg, seg.data(), sizeof(int32_t) * b.ncta, cudaMemcpyHostToDevice));
    PLATO_CUDA(h, cudaMemcpy(b.cta_row0, r0.data(), sizeof(int32_t) * b.ncta, cudaMemcpyHostToDevice));
    PLATO_CUDA(h, cudaMemcpy(b.cta_row1, r1.data(), sizeof(int32_t) * b.ncta, cudaMemcpyHostToDevice));
    PLATO_CUDA(h, cudaMemcpy(b.seg_cta0, first.data(), sizeof(int32_t) * (b.nseg + 1), cudaMemcpyHostToDevice));
    PLATO_CUDA(h, cudaMemcpy(b.cell_off_d, b.cell_off.data(), sizeof(int32_t) * (b.nseg + 1), cudaMemcpyHostToDevice));
    return PLATO_OK;
}

bool same_physics(const plato_problem_desc& a, const plato_problem_desc& b) {
    return a.material.youngs_modulus == b.material.youngs_modulus &&
           a.material.poissons_ratio == b.material.poissons_ratio && a.penalty.exponent == b.penalty.exponent &&
           a.penalty.minimum_value == b.penalty.minimum_value;
}

}  // namespace
}  // namespace plato

using namespace plato;

extern "C" {

int plato_create_batch(int32_t count, const plato_problem_desc* descs, plato_problem** out) {
    if (!out) return plato_fail(nullptr, PLATO_BAD_INPUT, "null output handle pointer");
    *out = nullptr;
    if (count < 1 || !descs) return plato_fail(nullptr, PLATO_BAD_INPUT, "a batch needs count >= 1 descriptions");
    int64_t nodes = 0, cells = 0;
    for (int32_t s = 0; s < count; ++s) {
        const plato_problem_desc& d = descs[s];
        if (d.mesh.num_nodes < 1 || d.mesh.num_cells < 1 || !d.mesh.coords || !d.mesh.connectivity)
            return plato_fail(nullptr, PLATO_BAD_INPUT, "every batch member needs a non-empty mesh");
        if (!same_physics(d, descs[0]))
            return plato_fail(nullptr, PLATO_BAD_INPUT, "batch members must share material and penalty");
        if (d.essential_bcs.num_dofs < 0 || d.num_natural_bcs < 0 || (d.num_natural_bcs > 0 && !d.natural_bcs) ||
            (d.essential_bcs.num_dofs > 0 && (!d.essential_bcs.dofs || !d.essential_bcs.values)))
            return plato_fail(nullptr, PLATO_BAD_INPUT, "malformed boundary conditions in a batch member");
        nodes += d.mesh.num_nodes;
        cells += d.mesh.num_cells;
    }
    if (nodes * 3 > INT32_MAX || cells * 4 > INT32_MAX || count > 65535)
        return plato_fail(nullptr, PLATO_BAD_INPUT, "batch too large for int32 ordinals");
    const plato_solver_opts& o = descs[0].solver;
    if (o.operator_kind != PLATO_OPERATOR_ASSEMBLED || o.coarse_cells[0] > 0)
        return plato_fail(nullptr, PLATO_NOT_SUPPORTED,
                          "batched solves use the assembled operator without a coarse space");

    // union arrays
    std::vector<double> coords;
    std::vector<int32_t> conn, bc_dofs, node_off(count + 1, 0), cell_off(count + 1, 0);
    std::vector<double> bc_vals;
    coords.reserve(size_t(3 * nodes));
    conn.reserve(size_t(4 * cells));
    std::vector<std::vector<int32_t>> face_cells;  // per natural BC, offset cell ids
    std::vector<plato_natural_bc> nbcs;
    for (int32_t s = 0; s < count; ++s) {
        const plato_problem_desc& d = descs[s];
        const int32_t no = node_off[s], co = cell_off[s];
        coords.insert(coords.end(), d.mesh.coords, d.mesh.coords + 3 * int64_t(d.mesh.num_nodes));
        for (int64_t k = 0; k < 4 * int64_t(d.mesh.num_cells); ++k) {
            const int32_t v = d.mesh.connectivity[k];
            if (v < 0 || v >= d.mesh.num_nodes)
                return plato_fail(nullptr, PLATO_BAD_INPUT, "connectivity entry out of range in a batch member");
            conn.push_back(v + no);
        }
        for (int32_t i = 0; i < d.essential_bcs.num_dofs; ++i) {
            const int32_t dof = d.essential_bcs.dofs[i];
            if (dof < 0 || dof >= 3 * d.mesh.num_nodes)
                return plato_fail(nullptr, PLATO_BAD_INPUT, "essential BC dof out of range in a batch member");
            bc_dofs.push_back(dof + 3 * no);
            bc_vals.push_back(d.essential_bcs.values[i]);
        }
        for (int32_t k = 0; k < d.num_natural_bcs; ++k) {
            const plato_natural_bc& nb = d.natural_bcs[k];
            if (nb.num_faces < 0 || (nb.num_faces > 0 && (!nb.face_cells || !nb.face_local_nodes)))
                return plato_fail(nullptr, PLATO_BAD_INPUT, "natural BC needs face cells and local nodes");
            std::vector<int32_t> fc(nb.face_cells, nb.face_cells + nb.num_faces);
            for (int32_t& c : fc) {
                if (c < 0 || c >= d.mesh.num_cells)
                    return plato_fail(nullptr, PLATO_BAD_INPUT, "natural BC face cell out of range in a batch member");
                c += co;
            }
            face_cells.push_back(std::move(fc));
            nbcs.push_back(nb);
        }
        node_off[s + 1] = no + d.mesh.num_nodes;
        cell_off[s + 1] = co + d.mesh.num_cells;
    }
    for (size_t k = 0; k < nbcs.size(); ++k) nbcs[k].face_cells = face_cells[k].data();

    plato_problem_desc u = descs[0];
    u.mesh.num_nodes = int32_t(nodes);
    u.mesh.num_cells = int32_t(cells);
    u.mesh.coords = coords.data();
    u.mesh.connectivity = conn.data();
    u.num_natural_bcs = int32_t(nbcs.size());
    u.natural_bcs = nbcs.empty() ? nullptr : nbcs.data();
    u.essential_bcs.num_dofs = int32_t(bc_dofs.size());
    u.essential_bcs.dofs = bc_dofs.empty() ? nullptr : bc_dofs.data();
    u.essential_bcs.values = bc_vals.empty() ? nullptr : bc_vals.data();

    plato_problem* h = nullptr;
    if (int rc = plato_create(&u, &h)) return rc;
    h->batch.nseg = count;
    h->batch.node_off = node_off;
    h->batch.cell_off = cell_off;
    if (int rc = setup_tiles(h)) {
        const std::string msg = h->last_error;
        plato_destroy(h);
        return plato_fail(nullptr, rc, msg);
    }
    *out = h;
    return PLATO_OK;
}

int plato_batch_info(const plato_problem* h, int32_t* count, int32_t* node_offsets, int32_t* cell_offsets) {
    if (!h) return PLATO_BAD_INPUT;
    const BatchState& b = h->batch;
    const int32_t n = b.nseg > 0 ? b.nseg : 1;
    if (count) *count = n;
    for (int32_t s = 0; s <= n; ++s) {
        if (node_offsets) node_offsets[s] = b.nseg > 0 ? b.node_off[s] : (s ? h->N : 0);
        if (cell_offsets) cell_offsets[s] = b.nseg > 0 ? b.cell_off[s] : (s ? h->C : 0);
    }
    return PLATO_OK;
}

int plato_batch_last_stats(const plato_problem* h, plato_solve_stats* stats) {
    if (!h || !stats) return PLATO_BAD_INPUT;
    const BatchState& b = h->batch;
    if (b.nseg == 0 || int32_t(b.last.size()) != b.nseg)
        return plato_fail(const_cast<plato_problem*>(h), PLATO_BAD_INPUT, "no batched solve has run on this handle");
    std::copy(b.last.begin(), b.last.end(), stats);
    return PLATO_OK;
}

// The project's autotuner of the batched solve: every (tile rows, CTAs per SM) candidate runs
// kAutotuneIterations flexible-CG iterations of this batch (assembly and preconditioner set-up
// included, the same for every candidate) on a scratch state; the fastest pair is kept.
int plato_batch_autotune(plato_problem* h, const double* z, plato_batch_tuning* out) {
    if (!h) return PLATO_BAD_INPUT;
    if (!z || !out) return plato_fail(h, PLATO_BAD_INPUT, "null pointer");
    BatchState& b = h->batch;
    if (b.nseg == 0) return plato_fail(h, PLATO_BAD_INPUT, "not a batch handle");
    static const int32_t kRows[] = {128, 256, 512};
    static const int32_t kCtas[] = {2, 4, 8, 16};
    constexpr int32_t kAutotuneIterations = 8;
    double* x = nullptr;
    PLATO_CUDA(h, cudaMalloc(&x, sizeof(double) * 3 * size_t(h->N)));
    const plato_solver_opts saved = h->opts;
    h->opts.max_iterations = kAutotuneIterations;
    h->opts.fallback_max_iterations = -1;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int best = -1, k = 0, rc = PLATO_OK;
    double best_ms = 0.0;
    *out = plato_batch_tuning{};
    for (int32_t rows : kRows)
        for (int32_t ctas : kCtas) {
            b.tile_rows = rows;
            b.ctas_per_sm = ctas;
            rc = setup_tiles(h);
            if (rc) break;
            plato_solve_stats st{};
            float ms = 0.f;
            // the first run of a candidate warms it up; the second is timed
            for (int rep = 0; rep < 2 && rc == PLATO_OK; ++rep) {
                cudaEventRecord(e0, h->stream);
                const int r = solve_state(h, z, nullptr, x, &st);
                cudaEventRecord(e1, h->stream);
                if (r != PLATO_OK && r != PLATO_NOT_CONVERGED) rc = r;
            }
            if (rc) break;
            cudaEventSynchronize(e1);
            cudaEventElapsedTime(&ms, e0, e1);
            out->tile_rows_tried[k] = rows;
            out->ctas_per_sm_tried[k] = ctas;
            out->ms_tried[k] = ms;
            if (best < 0 || ms < best_ms) { best = k; best_ms = ms; }
            ++k;
        }
    h->opts = saved;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(x);
    h->last_error.clear();
    if (rc) return rc;
    out->candidates = k;
    out->tile_rows = out->tile_rows_tried[best];
    out->ctas_per_sm = out->ctas_per_sm_tried[best];
    out->iterations = kAutotuneIterations;
    b.tile_rows = out->tile_rows;
    b.ctas_per_sm = out->ctas_per_sm;
    b.tuned = 1;
    return setup_tiles(h);
}

int plato_batch_criterion_values(plato_problem* h, const double* z, const double* u, double* values) {
    if (!h) return PLATO_BAD_INPUT;
    if (!z || !u || !values) return plato_fail(h, PLATO_BAD_INPUT, "null device pointer");
    if (h->batch.nseg == 0) return plato_fail(h, PLATO_BAD_INPUT, "not a batch handle");
    int rc = launch_energy_segments(h, u, z, values);
    if (rc) return rc;
    PLATO_CUDA(h, cudaStreamSynchronize(h->stream));
    return PLATO_OK;
}

}  // extern "C"

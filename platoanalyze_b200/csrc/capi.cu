// C ABI entry points (declared in include/plato_b200.h).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include <map>
#include <mutex>
#include <utility>

#include "plato_internal.cuh"

namespace plato {
int build_graph(plato_problem* h);
int launch_internal_force(plato_problem* h, const double* u, const double* z, double* R, double scale_F);
int launch_traction(plato_problem* h, int32_t nfaces, const int32_t* fcell, const int32_t* floc, const double t[3]);
int launch_nodal_control_derivative(plato_problem* h, int mode, const double* u, const double* z,
                                    const double* lam, double* cellbuf, double* out, int accumulate);
int launch_energy(plato_problem* h, const double* u, const double* z, double* result);
int launch_energy_and_gradient(plato_problem* h, const double* u, const double* z, double* result, double* dfdz);
int launch_assemble_jacobian(plato_problem* h, const double* z, double* entries);
int launch_assemble_gradient_z(plato_problem* h, const double* u, const double* z, double* entries);
int launch_dirichlet(plato_problem* h, double* A, double* rhs, double scale);
int launch_matvec_plus(plato_problem* h, int rb, int cb, const double* A, const double* x, double* y);
int launch_axpby(plato_problem* h, int64_t n, double a, const double* x, double b, double* y);
int build_sell_pattern(plato_problem* h);
int prepare_operator(plato_problem* h, const double* crs, const double* z = nullptr);
int assembly_direct_sell_ok(plato_problem* h, int* ok);
int pcg_fp64(plato_problem* h, const double* b, double* x, plato_solve_stats* stats);
int solve_state(plato_problem* h, const double* z, const double* u0, double* u, plato_solve_stats* stats);
int solve_adjoint(plato_problem* h, const double* z, const double* rhs, double* lam, plato_solve_stats* stats);
int prepare_mixed(plato_problem* h, const double* crs, const double* z);
int prepare_coarse(plato_problem* h, const double* z);
int prepare_coarse_start(plato_problem* h);
int fcg_poly(plato_problem* h, const double* b, double* x, plato_solve_stats* stats);
int matfree_rhs(plato_problem* h, double* b, double scale);
int launch_dirichlet_rhs(plato_problem* h, double* rhs, double scale);
int launch_ebe_apply64_unmasked(plato_problem* h, const double* x, double* y);
int launch_masked_axpy(plato_problem* h, double a, const double* x, double* y);
int matfree_setup(plato_problem* h, const double* z);
int launch_ebe_apply64(plato_problem* h, const double* x, double* y, const PcgScalars* S);
int launch_mask_copy(plato_problem* h, const double* x, double* y);
int launch_sell_spmv(plato_problem* h, const double* vals, const double* x, double* y);
int launch_volume(plato_problem* h, const Material& pen, const double* z, double* result);
int launch_volume_gradient(plato_problem* h, const Material& pen, const double* z, double* dvdz);
}  // namespace plato

using namespace plato;

static thread_local std::string g_create_error;

int plato_fail(plato_problem* h, int status, const std::string& msg) {
    if (h) h->last_error = msg; else g_create_error = msg;
    return status;
}

int plato_cuda_fail(plato_problem* h, cudaError_t e, const char* what, const char* file, int line) {
    char buf[512];
    std::snprintf(buf, sizeof buf, "CUDA error %s (%s) in %s at %s:%d", cudaGetErrorName(e),
                  cudaGetErrorString(e), what, file, line);
    // clear the runtime's last-error slot so a later launch check does not report this
    // (non-sticky) error again; sticky errors persist in the context regardless
    (void)cudaGetLastError();
    const int status = (e == cudaErrorMemoryAllocation) ? PLATO_OUT_OF_MEMORY : PLATO_CUDA_ERROR;
    return plato_fail(h, status, buf);
}

namespace plato {
int ensure_smem_attribute(plato_problem* h, const void* kernel, int bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, int> granted;
    int dev = 0;
    PLATO_CUDA(h, cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    int& have = granted[{dev, kernel}];
    if (bytes <= have) return PLATO_OK;
    PLATO_CUDA(h, cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    have = bytes;
    return PLATO_OK;
}
}  // namespace plato

namespace {

template <typename T>
int dmalloc(plato_problem* h, T** p, int64_t count) {
    if (*p) return PLATO_OK;
    const size_t bytes = size_t(count > 0 ? count : 1) * sizeof(T);
    PLATO_CUDA(h, cudaMalloc(reinterpret_cast<void**>(p), bytes));
    return PLATO_OK;
}

template <typename T>
void dfree(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

bool finite_array(const double* a, int64_t n) {
    for (int64_t i = 0; i < n; ++i)
        if (!std::isfinite(a[i])) return false;
    return true;
}

int check_opts(plato_problem* h, const plato_solver_opts& o) {
    if (!(o.tolerance > 0.0) || !std::isfinite(o.tolerance))
        return plato_fail(h, PLATO_BAD_INPUT, "solver tolerance must be a positive finite number");
    if (o.max_iterations < 1) return plato_fail(h, PLATO_BAD_INPUT, "solver max_iterations must be >= 1");
    if (o.operator_kind != PLATO_OPERATOR_ASSEMBLED && o.operator_kind != PLATO_OPERATOR_MATRIX_FREE)
        return plato_fail(h, PLATO_BAD_INPUT, "unknown operator_kind");
    if (o.precision < PLATO_PRECISION_FP64 || o.precision > PLATO_PRECISION_MIXED_FP32_ASSEMBLED)
        return plato_fail(h, PLATO_BAD_INPUT, "unknown precision");
    if (o.precision == PLATO_PRECISION_MIXED_FP32_ASSEMBLED && o.operator_kind != PLATO_OPERATOR_MATRIX_FREE)
        return plato_fail(h, PLATO_BAD_INPUT, "FP32 element assembly pairs with the matrix-free FP64 operator");
    if (o.chebyshev_kind != 0 && o.chebyshev_kind != 1 && o.chebyshev_kind != 4)
        return plato_fail(h, PLATO_BAD_INPUT, "chebyshev_kind must be 0 or 1 (first kind) or 4 (fourth kind)");
    if (o.sweep_steps < 0 || o.sweep_steps > 16) return plato_fail(h, PLATO_BAD_INPUT, "sweep_steps must be in 0..16");
    if (o.sweep_lag < 0) return plato_fail(h, PLATO_BAD_INPUT, "sweep_lag must be >= 0");
    return PLATO_OK;
}

#define RC(expr)                   \
    do {                           \
        int _rc = (expr);          \
        if (_rc) return _rc;       \
    } while (0)

#define NEED(h, cond, msg)                                             \
    do {                                                               \
        if (!(h)) return PLATO_BAD_INPUT;                              \
        if (!(cond)) return plato_fail((h), PLATO_BAD_INPUT, (msg));   \
    } while (0)

}  // namespace

extern "C" {

const char* plato_last_error(const plato_problem* h) {
    return h ? h->last_error.c_str() : g_create_error.c_str();
}

int plato_destroy(plato_problem* h) {
    if (!h) return PLATO_OK;
    cudaStreamSynchronize(h->stream);
    dfree(h->conn); dfree(h->coords); dfree(h->row_map); dfree(h->cols); dfree(h->diag);
    dfree(h->n2c_ptr); dfree(h->n2c); dfree(h->F); dfree(h->bc_dofs); dfree(h->bc_values);
    dfree(h->asm_plan); dfree(h->asm_wide); dfree(h->asm_mirror); dfree(h->asm_wideflag); dfree(h->ritz_small);
    dfree(h->bc_mask); dfree(h->K); dfree(h->KT); dfree(h->v_r); dfree(h->v_z); dfree(h->v_p);
    dfree(h->v_Ap); dfree(h->v_dinv); dfree(h->v_b); dfree(h->v_x); dfree(h->v_tmp);
    dfree(h->partials); dfree(h->cellbuf); dfree(h->scal); dfree(h->red_out); dfree(h->red_ticket);
    dfree(h->f_r); dfree(h->f_z); dfree(h->f_p); dfree(h->f_Ap); dfree(h->f_x); dfree(h->f_dinv);
    dfree(h->f_K); dfree(h->h_K); dfree(h->f_coords); dfree(h->f_z_ctrl); dfree(h->d_z_ctrl);
    dfree(h->d_z_in); dfree(h->d_u_out); dfree(h->d_g_out);
    dfree(h->sell.width); dfree(h->sell.ptr); dfree(h->sell.cols); dfree(h->sell.dcols);
    dfree(h->sell64); dfree(h->sell32);
    if (h->sell16) cudaFree(h->sell16);
    if (h->sell16s) cudaFree(h->sell16s);
    dfree(h->f_sq); dfree(h->f_isq);
    dfree(h->mf_w64); dfree(h->mf_w32); dfree(h->v_q);
    dfree(h->f_res); dfree(h->f_d0); dfree(h->f_d1); dfree(h->f_y); dfree(h->f_w);
    dfree(h->wave_flags); dfree(h->wave_ctl); dfree(h->lanczos);
    for (int32_t*& o : h->wave_order) dfree(o);
    if (h->scal_host) cudaFreeHost(h->scal_host);
    for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
    for (cudaEvent_t e : h->poll_ev)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : h->asm_ev)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : h->coarse_ev)
        if (e) cudaEventDestroy(e);
    coarse_release(h);
    batch_release(h);
    if (h->ritz_scratch) cudaFree(h->ritz_scratch);
    dfree(h->helm_K); dfree(h->helm_sell); dfree(h->helm_D); dfree(h->helm_Dsell); dfree(h->helm_dinv); dfree(h->helm_fcell); dfree(h->helm_floc);
    delete h;
    return PLATO_OK;
}

int plato_create(const plato_problem_desc* d, plato_problem** out) {
    if (!out) return plato_fail(nullptr, PLATO_BAD_INPUT, "null output handle pointer");
    *out = nullptr;
    if (!d) return plato_fail(nullptr, PLATO_BAD_INPUT, "null problem description");
    const plato_mesh_desc& m = d->mesh;
    if (m.num_nodes < 1 || m.num_cells < 1 || !m.coords || !m.connectivity)
        return plato_fail(nullptr, PLATO_BAD_INPUT, "mesh needs num_nodes >= 1, num_cells >= 1, coords and connectivity");
    if (int64_t(m.num_nodes) * 3 > INT32_MAX || int64_t(m.num_cells) * 4 > INT32_MAX)
        return plato_fail(nullptr, PLATO_BAD_INPUT, "mesh too large for int32 dof / connectivity ordinals");
    if (!finite_array(m.coords, 3 * int64_t(m.num_nodes)))
        return plato_fail(nullptr, PLATO_BAD_INPUT, "non-finite nodal coordinate");
    const double E = d->material.youngs_modulus, nu = d->material.poissons_ratio;
    if (!std::isfinite(E) || !std::isfinite(nu) || nu <= -1.0 || nu >= 0.5)
        return plato_fail(nullptr, PLATO_BAD_INPUT, "material needs finite E and -1 < nu < 0.5");
    if (!std::isfinite(d->penalty.exponent) || !std::isfinite(d->penalty.minimum_value))
        return plato_fail(nullptr, PLATO_BAD_INPUT, "non-finite penalty parameter");

    plato_problem* h = new plato_problem();
    h->N = m.num_nodes;
    h->C = m.num_cells;
    h->opts = d->solver;
    for (int dd = 0; dd < 3; ++dd) {
        h->bbox_min[dd] = m.coords[dd];
        h->bbox_max[dd] = m.coords[dd];
    }
    for (int64_t p = 1; p < m.num_nodes; ++p)
        for (int dd = 0; dd < 3; ++dd) {
            const double v = m.coords[3 * p + dd];
            if (v < h->bbox_min[dd]) h->bbox_min[dd] = v;
            if (v > h->bbox_max[dd]) h->bbox_max[dd] = v;
        }
    if (int rc = check_opts(h, h->opts)) { g_create_error = h->last_error; delete h; return rc; }
    cudaGetDevice(&h->device);

    // IsotropicLinearElasticMaterial<3> constants, src/IsotropicLinearElasticMaterial.cpp:86-110
    const double coef = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
    h->material.c00 = coef * (1.0 - nu);
    h->material.c01 = coef * nu;
    h->material.c33 = 1.0 / 2.0 * coef * (1.0 - 2.0 * nu);
    h->material.p = d->penalty.exponent;
    h->material.rho_min = d->penalty.minimum_value;
    h->material.p_int = (d->penalty.exponent >= 0.0 && d->penalty.exponent <= 16.0 &&
                         std::floor(d->penalty.exponent) == d->penalty.exponent)
                            ? int(d->penalty.exponent) : -1;

    auto fail_create = [&](int rc) {
        g_create_error = h->last_error;
        plato_destroy(h);
        return rc;
    };
#define CRC(expr)                          \
    do {                                   \
        int _rc = (expr);                  \
        if (_rc) return fail_create(_rc);  \
    } while (0)
#define CCUDA(expr)                                                                 \
    do {                                                                            \
        cudaError_t _e = (expr);                                                    \
        if (_e != cudaSuccess) return fail_create(plato_cuda_fail(h, _e, #expr, __FILE__, __LINE__)); \
    } while (0)

    const int64_t n = 3 * int64_t(h->N);
    CRC(dmalloc(h, &h->conn, h->C));
    CRC(dmalloc(h, &h->coords, n));
    CCUDA(cudaMemcpy(h->conn, m.connectivity, sizeof(int4) * size_t(h->C), cudaMemcpyHostToDevice));
    CCUDA(cudaMemcpy(h->coords, m.coords, sizeof(double) * size_t(n), cudaMemcpyHostToDevice));
    CRC(build_graph(h));
    CRC(build_sell_pattern(h));

    // essential BCs
    const plato_essential_bcs& bc = d->essential_bcs;
    if (bc.num_dofs < 0 || (bc.num_dofs > 0 && (!bc.dofs || !bc.values)))
        return fail_create(plato_fail(h, PLATO_BAD_INPUT, "essential BCs need dofs and values"));
    std::vector<uint8_t> mask(n, 0);
    for (int32_t i = 0; i < bc.num_dofs; ++i) {
        if (bc.dofs[i] < 0 || bc.dofs[i] >= n)
            return fail_create(plato_fail(h, PLATO_BAD_INPUT, "essential BC dof out of range"));
        if (!std::isfinite(bc.values[i]))
            return fail_create(plato_fail(h, PLATO_BAD_INPUT, "non-finite essential BC value"));
        mask[bc.dofs[i]] = 1;
        if (bc.values[i] != 0.0) h->bc_nonzero = 1;
    }
    h->nbc = bc.num_dofs;
    CRC(dmalloc(h, &h->bc_dofs, h->nbc));
    CRC(dmalloc(h, &h->bc_values, h->nbc));
    CRC(dmalloc(h, &h->bc_mask, n));
    if (h->nbc) {
        CCUDA(cudaMemcpy(h->bc_dofs, bc.dofs, sizeof(int32_t) * h->nbc, cudaMemcpyHostToDevice));
        CCUDA(cudaMemcpy(h->bc_values, bc.values, sizeof(double) * h->nbc, cudaMemcpyHostToDevice));
    }
    CCUDA(cudaMemcpy(h->bc_mask, mask.data(), size_t(n), cudaMemcpyHostToDevice));

    // work vectors and reduction scratch
    for (double** v : {&h->F, &h->v_r, &h->v_z, &h->v_p, &h->v_Ap, &h->v_dinv, &h->v_b, &h->v_x, &h->v_tmp})
        CRC(dmalloc(h, v, n));
    h->partials_len = 148 * 64;
    CRC(dmalloc(h, &h->partials, 4 * int64_t(h->partials_len)));
    CRC(dmalloc(h, &h->cellbuf, h->C));
    CRC(dmalloc(h, &h->scal, 1));
    CRC(dmalloc(h, &h->red_out, 4));  // up to 4 reduction results
    CRC(dmalloc(h, &h->red_ticket, 1));
    CCUDA(cudaMemset(h->red_ticket, 0, sizeof(uint32_t)));
    CCUDA(cudaMemset(h->scal, 0, sizeof(PcgScalars)));
    CCUDA(cudaMallocHost(reinterpret_cast<void**>(&h->scal_host), 2 * sizeof(PcgScalars)));

    // external load F from the natural BCs (constant in u and z)
    CCUDA(cudaMemset(h->F, 0, sizeof(double) * size_t(n)));
    for (int32_t k = 0; k < d->num_natural_bcs; ++k) {
        const plato_natural_bc& nb = d->natural_bcs[k];
        if (nb.num_faces < 0 || (nb.num_faces > 0 && (!nb.face_cells || !nb.face_local_nodes)))
            return fail_create(plato_fail(h, PLATO_BAD_INPUT, "natural BC needs face cells and local nodes"));
        for (int32_t f = 0; f < nb.num_faces; ++f) {
            if (nb.face_cells[f] < 0 || nb.face_cells[f] >= h->C)
                return fail_create(plato_fail(h, PLATO_BAD_INPUT, "natural BC face cell out of range"));
            for (int a = 0; a < 3; ++a)
                if (nb.face_local_nodes[3 * int64_t(f) + a] < 0 || nb.face_local_nodes[3 * int64_t(f) + a] > 3)
                    return fail_create(plato_fail(h, PLATO_BAD_INPUT, "natural BC local node ordinal out of range"));
        }
        if (nb.num_faces == 0) continue;
        int32_t *fc = nullptr, *fl = nullptr;
        CCUDA(cudaMalloc(&fc, sizeof(int32_t) * nb.num_faces));
        CCUDA(cudaMalloc(&fl, sizeof(int32_t) * 3 * size_t(nb.num_faces)));
        CCUDA(cudaMemcpy(fc, nb.face_cells, sizeof(int32_t) * nb.num_faces, cudaMemcpyHostToDevice));
        CCUDA(cudaMemcpy(fl, nb.face_local_nodes, sizeof(int32_t) * 3 * size_t(nb.num_faces), cudaMemcpyHostToDevice));
        const int rc = launch_traction(h, nb.num_faces, fc, fl, nb.vector);
        cudaStreamSynchronize(h->stream);
        cudaFree(fc);
        cudaFree(fl);
        CRC(rc);
    }
    CCUDA(cudaStreamSynchronize(h->stream));
#undef CRC
#undef CCUDA
    *out = h;
    return PLATO_OK;
}

int plato_set_stream(plato_problem* h, void* stream) {
    if (!h) return PLATO_BAD_INPUT;
    h->stream = static_cast<cudaStream_t>(stream);
    return PLATO_OK;
}

int plato_set_control_layout(plato_problem* h, int32_t layout) {
    if (!h) return plato_fail(nullptr, PLATO_BAD_INPUT, "null handle");
    if (layout != PLATO_CONTROL_NODAL && layout != PLATO_CONTROL_ELEMENT)
        return plato_fail(h, PLATO_BAD_INPUT, "unknown control layout");
    if (layout == PLATO_CONTROL_ELEMENT && (h->batch.nseg > 0 || h->physics != 0))
        return plato_fail(h, PLATO_NOT_SUPPORTED, "element control is for single elastostatic problems");
    h->material.cell_control = layout == PLATO_CONTROL_ELEMENT ? 1 : 0;
    return PLATO_OK;
}

int plato_set_solver_opts(plato_problem* h, const plato_solver_opts* o) {
    NEED(h, o != nullptr, "null solver options");
    RC(check_opts(h, *o));
    if (h->batch.nseg > 0 && (o->operator_kind != PLATO_OPERATOR_ASSEMBLED || o->coarse_cells[0] > 0))
        return plato_fail(h, PLATO_NOT_SUPPORTED, "batched solves use the assembled operator without a coarse space");
    h->opts = *o;
    return PLATO_OK;
}

int plato_set_timing(plato_problem* h, int32_t enable) {
    if (!h) return PLATO_BAD_INPUT;
    h->timing = enable ? 1 : 0;
    return PLATO_OK;
}

int plato_get_instrumentation(const plato_problem* h, int64_t* launches, double* op_ms_total,
                              int64_t* op_timed) {
    if (!h) return PLATO_BAD_INPUT;
    if (launches) *launches = h->launches;
    if (op_ms_total) *op_ms_total = h->op_ms_total;
    if (op_timed) *op_timed = h->op_timed;
    return PLATO_OK;
}

// Element-kernel timing: begin/end bracket one launch group of kind k (0 residual, 1 energy,
// 2 control derivative) on the handle's stream; a previous pair of the same kind is read
// first (it has completed by then or is waited for).
static int elem_time_flush(plato_problem* h, int k) {
    auto& t = h->elem_timing[k];
    if (!t.pending) return PLATO_OK;
    PLATO_CUDA(h, cudaEventSynchronize(t.e1));
    float ms = 0.f;
    PLATO_CUDA(h, cudaEventElapsedTime(&ms, t.e0, t.e1));
    t.ms += ms;
    t.count += 1;
    t.pending = 0;
    return PLATO_OK;
}

static int elem_time_begin(plato_problem* h, int k) {
    if (!h->timing) return PLATO_OK;
    auto& t = h->elem_timing[k];
    RC(elem_time_flush(h, k));
    if (!t.e0) PLATO_CUDA(h, cudaEventCreate(&t.e0));
    if (!t.e1) PLATO_CUDA(h, cudaEventCreate(&t.e1));
    PLATO_CUDA(h, cudaEventRecord(t.e0, h->stream));
    return PLATO_OK;
}

static int elem_time_end(plato_problem* h, int k) {
    if (!h->timing) return PLATO_OK;
    auto& t = h->elem_timing[k];
    PLATO_CUDA(h, cudaEventRecord(t.e1, h->stream));
    t.pending = 1;
    return PLATO_OK;
}

int plato_get_kernel_timing(const plato_problem* hc, int32_t kind, double* ms_total, int64_t* count) {
    if (!hc || !ms_total || !count) return PLATO_BAD_INPUT;
    plato_problem* h = const_cast<plato_problem*>(hc);  // reading the totals completes pending pairs
    if (kind >= 5 && kind <= 8) {
        RC(elem_time_flush(h, kind - 5));
        *ms_total = h->elem_timing[kind - 5].ms;
        *count = h->elem_timing[kind - 5].count;
        return PLATO_OK;
    }
    if (kind == 0) { *ms_total = h->op_ms_total; *count = h->op_timed; }
    else if (kind == 1) { *ms_total = h->inner_ms_total; *count = h->inner_timed; }
    else if (kind == 2) { *ms_total = h->asm_ms_total; *count = h->asm_timed; }
    else if (kind == 3) { *ms_total = h->coarse_gal_ms; *count = h->coarse_timed; }
    else if (kind == 4) { *ms_total = h->coarse_inv_ms; *count = h->coarse_timed; }
    else return PLATO_BAD_INPUT;
    return PLATO_OK;
}

int plato_test_stall_next_sweep(plato_problem* h) {
    if (!h) return PLATO_BAD_INPUT;
    h->wave_stall = 1;
    return PLATO_OK;
}

int plato_get_sweep_info(const plato_problem* h, int32_t* steps_per_launch, int32_t* halo_tiles) {
    if (!h || !steps_per_launch || !halo_tiles) return PLATO_BAD_INPUT;
    *steps_per_launch = h->sweep_steps_used > 0 ? h->sweep_steps_used : 1;
    *halo_tiles = h->wave_halo >= 0 ? h->wave_halo : -1;
    return PLATO_OK;
}

int plato_get_sell_info(const plato_problem* h, int64_t* total_slots, int32_t* column_bytes) {
    if (!h || !total_slots || !column_bytes) return PLATO_BAD_INPUT;
    *total_slots = h->sell.total_slots;
    *column_bytes = h->sell.dcols ? 2 : 4;
    return PLATO_OK;
}

int plato_reset_instrumentation(plato_problem* h) {
    if (!h) return PLATO_BAD_INPUT;
    h->launches = 0;
    h->op_ms_total = 0.0;
    h->op_timed = 0;
    h->inner_ms_total = 0.0;
    h->inner_timed = 0;
    h->asm_ms_total = 0.0;
    h->asm_timed = 0;
    for (auto& t : h->elem_timing) {
        if (t.pending && t.e1) cudaEventSynchronize(t.e1);
        t.pending = 0;
        t.ms = 0.0;
        t.count = 0;
    }
    h->coarse_gal_ms = 0.0;
    h->coarse_inv_ms = 0.0;
    h->coarse_timed = 0;
    return PLATO_OK;
}

int plato_get_sizes(const plato_problem* h, int32_t* nn, int32_t* nc, int64_t* nb) {
    if (!h) return PLATO_BAD_INPUT;
    if (nn) *nn = h->N;
    if (nc) *nc = h->C;
    if (nb) *nb = h->nblocks;
    return PLATO_OK;
}

int plato_jacobian_pattern(plato_problem* h, int32_t* row_map, int32_t* cols) {
    NEED(h, row_map && cols, "null pattern output");
    PLATO_CUDA(h, cudaMemcpyAsync(row_map, h->row_map, sizeof(int32_t) * (h->N + 1), cudaMemcpyDeviceToDevice, h->stream));
    PLATO_CUDA(h, cudaMemcpyAsync(cols, h->cols, sizeof(int32_t) * size_t(h->nblocks), cudaMemcpyDeviceToDevice, h->stream));
    return PLATO_OK;
}

int plato_vf_value(plato_problem* h, const double* u, const double* z, double* R) {
    NEED(h, u && z && R, "null device pointer");
    RC(elem_time_begin(h, 0));
    RC(launch_internal_force(h, u, z, R, -1.0));
    return elem_time_end(h, 0);
}

int plato_vf_gradient_u(plato_problem* h, const double* u, const double* z, double* entries) {
    NEED(h, z && entries, "null device pointer");
    (void)u;  // linear elasticity: K does not depend on u
    return launch_assemble_jacobian(h, z, entries);
}

int plato_vf_gradient_u_T(plato_problem* h, const double* u, const double* z, double* entries) {
    // The closed-form isotropic element blocks satisfy K_ab = K_ba^T term by term, so the
    // transpose assembly produces the same entries as gradient_u.
    return plato_vf_gradient_u(h, u, z, entries);
}

int plato_vf_gradient_z(plato_problem* h, const double* u, const double* z, double* entries) {
    if (h && h->material.cell_control)
        return plato_fail(h, PLATO_NOT_SUPPORTED, "the (dR/dz)^T block matrix needs nodal control");
    NEED(h, u && z && entries, "null device pointer");
    return launch_assemble_gradient_z(h, u, z, entries);
}

int plato_vf_gradient_z_apply(plato_problem* h, const double* u, const double* z, const double* lam, double* out) {
    NEED(h, u && z && lam && out, "null device pointer");
    return launch_nodal_control_derivative(h, 3, u, z, lam, h->cellbuf, out, 1);
}

int plato_sf_value(plato_problem* h, const double* u, const double* z, double* value) {
    NEED(h, u && z && value, "null pointer");
    RC(elem_time_begin(h, 1));
    RC(launch_energy(h, u, z, h->red_out));
    RC(elem_time_end(h, 1));
    PLATO_CUDA(h, cudaMemcpyAsync(value, h->red_out, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    PLATO_CUDA(h, cudaStreamSynchronize(h->stream));
    return PLATO_OK;
}

int plato_sf_gradient_u(plato_problem* h, const double* u, const double* z, double* dfdu) {
    NEED(h, u && z && dfdu, "null device pointer");
    return launch_internal_force(h, u, z, dfdu, 0.0);
}

int plato_sf_gradient_z(plato_problem* h, const double* u, const double* z, double* dfdz) {
    NEED(h, u && z && dfdz, "null device pointer");
    return launch_nodal_control_derivative(h, 1, u, z, nullptr, h->cellbuf, dfdz, 0);
}

static Material volume_penalty(const plato_penalty* p, const plato_problem* h) {
    Material m{};
    m.cell_control = h->material.cell_control;
    m.p = p->exponent;
    m.rho_min = p->minimum_value;
    m.p_int = (p->exponent >= 0.0 && p->exponent <= 16.0 && std::floor(p->exponent) == p->exponent)
                  ? int(p->exponent) : -1;
    return m;
}

int plato_volume_value(plato_problem* h, const double* z, const plato_penalty* penalty, double* value) {
    NEED(h, z && penalty && value, "null pointer");
    NEED(h, std::isfinite(penalty->exponent) && std::isfinite(penalty->minimum_value), "non-finite penalty");
    RC(launch_volume(h, volume_penalty(penalty, h), z, h->red_out));
    PLATO_CUDA(h, cudaMemcpyAsync(value, h->red_out, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    PLATO_CUDA(h, cudaStreamSynchronize(h->stream));
    return PLATO_OK;
}

int plato_volume_gradient_z(plato_problem* h, const double* z, const plato_penalty* penalty, double* dvdz) {
    NEED(h, z && penalty && dvdz, "null pointer");
    NEED(h, std::isfinite(penalty->exponent) && std::isfinite(penalty->minimum_value), "non-finite penalty");
    return launch_volume_gradient(h, volume_penalty(penalty, h), z, dvdz);
}

int plato_apply_constraints(plato_problem* h, double* entries, double* rhs, double scale) {
    NEED(h, entries != nullptr, "null matrix entries");
    return launch_dirichlet(h, entries, rhs, scale);
}

int plato_matvec_plus(plato_problem* h, int32_t rb, int32_t cb, const double* entries, const double* x, double* y) {
    NEED(h, entries && x && y, "null device pointer");
    return launch_matvec_plus(h, rb, cb, entries, x, y);
}

int plato_apply_operator(plato_problem* h, const double* z, int32_t operator_kind, const double* x, double* y) {
    NEED(h, z && x && y, "null device pointer");
    if (operator_kind == PLATO_OPERATOR_MATRIX_FREE) {
        RC(matfree_setup(h, z));
        RC(launch_ebe_apply64(h, x, y, nullptr));
        return launch_mask_copy(h, x, y);
    }
    if (operator_kind != PLATO_OPERATOR_ASSEMBLED) return plato_fail(h, PLATO_BAD_INPUT, "unknown operator_kind");
    RC(dmalloc(h, &h->K, 9 * h->nblocks));
    RC(launch_assemble_jacobian(h, z, h->K));
    RC(launch_dirichlet(h, h->K, nullptr, 0.0));
    RC(prepare_operator(h, h->K, z));
    return launch_sell_spmv(h, h->sell64, x, y);
}

int plato_solver_solve(plato_problem* h, const double* entries, double* x, const double* b,
                       plato_solve_stats* stats) {
    NEED(h, entries && x && b, "null device pointer");
    plato_solve_stats local{};
    plato_solve_stats* st = stats ? stats : &local;
    // the matrix is given: the assembled operator is used whatever operator_kind says
    if (h->batch.nseg > 0) {
        RC(prepare_mixed(h, entries, nullptr));
        return fcg_batch(h, b, x, st);
    }
    if (h->opts.precision == PLATO_PRECISION_FP64 && h->opts.chebyshev_degree <= 0) {
        RC(prepare_operator(h, entries));
        return pcg_fp64(h, b, x, st);
    }
    const int32_t kind = h->opts.operator_kind;
    h->opts.operator_kind = PLATO_OPERATOR_ASSEMBLED;
    h->coarse.active = 0;  // the coarse operator needs the control, which this entry point lacks
    int rc = prepare_mixed(h, entries, nullptr);
    if (!rc) rc = fcg_poly(h, b, x, st);
    h->opts.operator_kind = kind;
    return rc;
}

int plato_problem_solution(plato_problem* h, const double* z, const double* u0, double* u,
                           plato_solve_stats* stats) {
    NEED(h, z && u, "null device pointer");
    plato_solve_stats local{};
    return solve_state(h, z, u0, u, stats ? stats : &local);
}

int plato_problem_solution_subspace(plato_problem* h, const double* z, const double* u0, const double* W, int32_t k,
                                    double* u, plato_solve_stats* stats, double* residual_ratio) {
    NEED(h, z && u, "null device pointer");
    NEED(h, k >= 0 && k <= 8 && (k == 0 || W), "subspace needs 0 <= k <= 8 columns");
    if (k > 0 && (h->batch.nseg > 0 || h->opts.operator_kind != PLATO_OPERATOR_ASSEMBLED))
        return plato_fail(h, PLATO_NOT_SUPPORTED, "subspace initial guesses need a single problem on the assembled operator");
    plato_solve_stats local{};
    h->ritz_W = W;
    h->ritz_k = k;
    h->ritz_rel_gain = 1.0;
    const int rc = solve_state(h, z, u0, u, stats ? stats : &local);
    h->ritz_W = nullptr;
    h->ritz_k = 0;
    if (residual_ratio) *residual_ratio = h->ritz_rel_gain;
    return rc;
}

int plato_problem_solution_deflated(plato_problem* h, const double* z, const double* u0, const double* W, int32_t k,
                                    double* u, plato_solve_stats* stats, double* residual_ratio) {
    NEED(h, z && u, "null device pointer");
    NEED(h, k >= 1 && k <= 8 && W, "deflation needs 1 <= k <= 8 columns");
    if (h->batch.nseg > 0 || h->opts.operator_kind != PLATO_OPERATOR_ASSEMBLED)
        return plato_fail(h, PLATO_NOT_SUPPORTED, "deflation needs a single problem on the assembled operator");
    plato_solve_stats local{};
    h->ritz_W = W;
    h->ritz_k = k;
    h->ritz_rel_gain = 1.0;
    h->ritz_deflate = 1;
    h->ritz_deflating = 0;
    const int rc = solve_state(h, z, u0, u, stats ? stats : &local);
    h->ritz_W = nullptr;
    h->ritz_k = 0;
    h->ritz_deflate = 0;
    h->ritz_deflating = 0;
    if (residual_ratio) *residual_ratio = h->ritz_rel_gain;
    return rc;
}

int plato_problem_criterion_value(plato_problem* h, const double* z, const double* u, double* value) {
    return plato_sf_value(h, u, z, value);
}

int plato_problem_criterion_value_and_gradient(plato_problem* h, const double* z, const double* u, double* value,
                                               double* dfdz, plato_solve_stats* stats) {
    NEED(h, z && u && value && dfdz, "null pointer");
    if (!h->opts.self_adjoint || h->batch.nseg > 0) {  // the adjoint solve, or per-member values: two calls
        RC(plato_problem_criterion_value(h, z, u, value));
        return plato_problem_criterion_gradient(h, z, u, dfdz, stats);
    }
    if (stats) { stats->iterations = 0; stats->refinements = 0; stats->relative_residual = 0.0;
                 stats->converged = 1; stats->status = 0; stats->fallback = 0; }
    RC(elem_time_begin(h, 3));
    RC(launch_energy_and_gradient(h, u, z, h->red_out, dfdz));
    RC(elem_time_end(h, 3));
    PLATO_CUDA(h, cudaMemcpyAsync(value, h->red_out, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    PLATO_CUDA(h, cudaStreamSynchronize(h->stream));
    return PLATO_OK;
}

int plato_problem_criterion_gradient(plato_problem* h, const double* z, const double* u, double* dfdz,
                                     plato_solve_stats* stats) {
    NEED(h, z && u && dfdz, "null device pointer");
    plato_solve_stats local{};
    plato_solve_stats* st = stats ? stats : &local;
    if (h->opts.self_adjoint) {
        // lambda = -u (src/elliptic/Problem.hpp:423-427): dfdz + (dR/dz)^T lambda fused per cell
        st->iterations = 0; st->refinements = 0; st->relative_residual = 0.0; st->converged = 1; st->status = 0;
        RC(elem_time_begin(h, 2));
        RC(launch_nodal_control_derivative(h, 2, u, z, nullptr, h->cellbuf, dfdz, 0));
        return elem_time_end(h, 2);
    }
    // adjoint: K^T lambda = -df/du with zero-valued constraints (Problem.hpp:429-441, 701-713)
    const int64_t n = 3 * int64_t(h->N);
    RC(launch_internal_force(h, u, z, h->v_tmp, 0.0));
    RC(launch_axpby(h, n, -1.0, h->v_tmp, 0.0, h->v_tmp));
    RC(solve_adjoint(h, z, h->v_tmp, h->v_x, st));
    return launch_nodal_control_derivative(h, 4, u, z, h->v_x, h->cellbuf, dfdz, 0);
}

int plato_problem_solve_and_gradient_host(plato_problem* h, const double* z_host, const double* u0_host,
                                          double* u_host, double* value_host, double* dfdz_host,
                                          plato_solve_stats* stats) {
    NEED(h, z_host != nullptr, "null control");
    const int64_t n = 3 * int64_t(h->N);
    // control entries: one per node, or one per cell with element control (buffers sized for both)
    const int64_t nz = h->material.cell_control ? h->C : h->N;
    const int64_t zcap = h->C > h->N ? h->C : h->N;
    RC(dmalloc(h, &h->d_z_in, zcap));
    RC(dmalloc(h, &h->d_u_out, n));
    RC(dmalloc(h, &h->d_g_out, zcap));
    cudaStream_t s = h->stream;
    PLATO_CUDA(h, cudaMemcpyAsync(h->d_z_in, z_host, sizeof(double) * nz, cudaMemcpyHostToDevice, s));
    const double* u0 = nullptr;
    if (u0_host) {
        PLATO_CUDA(h, cudaMemcpyAsync(h->d_u_out, u0_host, sizeof(double) * n, cudaMemcpyHostToDevice, s));
        u0 = h->d_u_out;
    }
    plato_solve_stats local{};
    plato_solve_stats* st = stats ? stats : &local;
    int rc = solve_state(h, h->d_z_in, u0, h->d_u_out, st);
    if (rc && rc != PLATO_NOT_CONVERGED) return rc;
    const int solve_rc = rc;
    if (value_host && dfdz_host) {  // ComputeCriterion: value and gradient together
        plato_solve_stats adj{};
        RC(plato_problem_criterion_value_and_gradient(h, h->d_z_in, h->d_u_out, value_host, h->d_g_out, &adj));
        PLATO_CUDA(h, cudaMemcpyAsync(dfdz_host, h->d_g_out, sizeof(double) * nz, cudaMemcpyDeviceToHost, s));
    } else if (value_host) {
        RC(plato_sf_value(h, h->d_u_out, h->d_z_in, value_host));
    } else if (dfdz_host) {
        plato_solve_stats adj{};
        RC(plato_problem_criterion_gradient(h, h->d_z_in, h->d_u_out, h->d_g_out, &adj));
        PLATO_CUDA(h, cudaMemcpyAsync(dfdz_host, h->d_g_out, sizeof(double) * nz, cudaMemcpyDeviceToHost, s));
    }
    if (u_host) PLATO_CUDA(h, cudaMemcpyAsync(u_host, h->d_u_out, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    PLATO_CUDA(h, cudaStreamSynchronize(s));
    return solve_rc;
}

}  // extern "C"

namespace plato {

static bool plain_method(const plato_solver_opts& o) {
    return o.operator_kind == PLATO_OPERATOR_ASSEMBLED && o.precision == PLATO_PRECISION_FP64 &&
           o.chebyshev_degree <= 0 && o.coarse_cells[0] <= 0;
}

// The plain method is the fallback of the others.  When a flexible-CG solve (status
// `failed`) did not meet the tolerance or broke down: if a subspace guess seeded it, the same
// method is retried from a zero guess; if that fails too, or there was no such guess, the
// plain FP64 Jacobi-PCG solves from a zero guess with fallback_max_iterations (0: the
// max_iterations cap).  h->v_b holds the constrained right-hand side.  For the matrix-free
// operator (z given) the constrained block matrix is assembled first.
static int fallback_solve(plato_problem* h, double* x, plato_solve_stats* st, int failed,
                          const double* z = nullptr) {
    const int32_t cap = h->opts.fallback_max_iterations;
    const size_t bytes = sizeof(double) * 3 * size_t(h->N);
    h->ritz_deflating = 0;  // deflation needs the Galerkin guess, which the retries drop
    if (h->ritz_W && h->ritz_k > 0) {
        PLATO_CUDA(h, cudaMemsetAsync(x, 0, bytes, h->stream));
        const int rc = fcg_poly(h, h->v_b, x, st);
        if (rc != PLATO_NOT_CONVERGED && rc != PLATO_NONFINITE) {
            st->fallback = 1;
            return rc;
        }
        failed = rc;
    }
    if (cap < 0) return failed;
    if (z) {  // matrix-free: the assembled constrained operator (right-hand side already built)
        RC(dmalloc(h, &h->K, 9 * h->nblocks));
        RC(launch_assemble_jacobian(h, z, h->K));
        RC(launch_dirichlet(h, h->K, nullptr, 0.0));
        RC(prepare_operator(h, h->K, z));
    }
    // the SELL FP64 copy and its Jacobi diagonal were made for the flexible CG's operator
    const int32_t saved = h->opts.max_iterations;
    if (cap > 0) h->opts.max_iterations = cap;
    PLATO_CUDA(h, cudaMemsetAsync(x, 0, bytes, h->stream));
    const int rc = pcg_fp64(h, h->v_b, x, st);
    h->opts.max_iterations = saved;
    st->fallback = 2;
    return rc;
}

// Builds the constrained operator of control z and the right-hand side (rhs with the
// Dirichlet rows/columns eliminated, values scaled by bc_scale), then solves into x (which
// holds the initial guess).  Plain method: assembled block matrix + Jacobi-PCG.  Otherwise:
// flexible CG with the Chebyshev preconditioner on the assembled or matrix-free operator.
static int solve_constrained(plato_problem* h, const double* z, const double* rhs, double bc_scale, double* x,
                             plato_solve_stats* st) {
    const int64_t n = 3 * int64_t(h->N);
    if (rhs != h->v_b)
        PLATO_CUDA(h, cudaMemcpyAsync(h->v_b, rhs, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->stream));
    h->coarse.active = 0;
    if (h->opts.operator_kind == PLATO_OPERATOR_MATRIX_FREE) {
        RC(prepare_coarse_start(h));
        RC(prepare_coarse(h, z));  // starts on its own stream, overlapping what follows
        RC(prepare_mixed(h, nullptr, z));
        RC(matfree_rhs(h, h->v_b, bc_scale));
        int rc = fcg_poly(h, h->v_b, x, st);
        const int crc = coarse_finish(h);
        if (crc && rc == PLATO_OK) rc = crc;
        if (rc != PLATO_NOT_CONVERGED && rc != PLATO_NONFINITE) return rc;
        return fallback_solve(h, x, st, rc, z);
    }
    // Homogeneous essential BCs and no high-valence rows: the solver's SELL copies are assembled
    // straight from z with the constraints applied (no CRS copy); otherwise K is assembled into
    // the block CRS, constrained there (lifting inhomogeneous values) and converted.
    int direct = 0;
    RC(assembly_direct_sell_ok(h, &direct));
    if (h->timing)
        for (cudaEvent_t& e : h->asm_ev)
            if (!e) PLATO_CUDA(h, cudaEventCreate(&e));
    const double* crs = nullptr;
    if (direct) {
        RC(launch_dirichlet_rhs(h, h->v_b, bc_scale));
    } else {
        RC(dmalloc(h, &h->K, 9 * h->nblocks));
        if (h->timing) PLATO_CUDA(h, cudaEventRecord(h->asm_ev[0], h->stream));
        RC(launch_assemble_jacobian(h, z, h->K));
        if (h->timing) PLATO_CUDA(h, cudaEventRecord(h->asm_ev[1], h->stream));
        RC(launch_dirichlet(h, h->K, h->v_b, bc_scale));
        crs = h->K;
    }
    int rc;
    if (h->batch.nseg > 0) {  // member-wise flexible CG over the union (Jacobi when no degree is set)
        RC(prepare_mixed(h, crs, z));
        rc = fcg_batch(h, h->v_b, x, st);
    } else if (plain_method(h->opts)) {
        RC(prepare_operator(h, crs, z));
        RC(ritz_guess(h, h->v_b, x));
        rc = pcg_fp64(h, h->v_b, x, st);
    } else {
        // the fine-level set-up is queued first (a few launches), then the coarse set-up on its
        // own stream, overlapping it from the point where z is final
        RC(prepare_coarse_start(h));
        RC(prepare_mixed(h, crs, z));
        RC(prepare_coarse(h, z));
        RC(ritz_guess(h, h->v_b, x));
        rc = fcg_poly(h, h->v_b, x, st);
        const int crc = coarse_finish(h);  // the overlapped coarse set-up: timing and its check
        if (crc && rc == PLATO_OK) rc = crc;
        if (rc == PLATO_NOT_CONVERGED || rc == PLATO_NONFINITE) rc = fallback_solve(h, x, st, rc);
    }
    if (h->timing) {  // the solver has synchronised the stream
        float ms = 0.f;
        PLATO_CUDA(h, cudaEventElapsedTime(&ms, h->asm_ev[0], h->asm_ev[1]));
        h->asm_ms_total += ms;
        h->asm_timed += 1;
    }
    return rc;
}

// Problem::solution (src/elliptic/Problem.hpp:237-292), one Newton step from u = 0:
// R = -value(0, z) = F, J = gradient_u, applyStateConstraints(J, R, 1), solve J d = R.
// (value(0, z) = 0 - F exactly, so F is used directly.)  u0, when given, seeds the solve.
int solve_state(plato_problem* h, const double* z, const double* u0, double* u, plato_solve_stats* st) {
    const int64_t n = 3 * int64_t(h->N);
    if (u0) {
        if (u0 != u) PLATO_CUDA(h, cudaMemcpyAsync(u, u0, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->stream));
    } else {
        PLATO_CUDA(h, cudaMemsetAsync(u, 0, sizeof(double) * n, h->stream));
    }
    return solve_constrained(h, z, h->F, 1.0, u, st);
}

// Adjoint solve K^T lambda = rhs with zero-valued constraints (K is symmetric).
int solve_adjoint(plato_problem* h, const double* z, const double* rhs, double* lam, plato_solve_stats* st) {
    PLATO_CUDA(h, cudaMemsetAsync(lam, 0, sizeof(double) * 3 * size_t(h->N), h->stream));
    return solve_constrained(h, z, rhs, 0.0, lam, st);
}

// Matrix-free right-hand side: b_free -= (K g)_free for inhomogeneous values g, b_d = scale g_d.
int matfree_rhs(plato_problem* h, double* b, double scale) {
    if (scale != 0.0 && h->bc_nonzero) {
        const int64_t n = 3 * int64_t(h->N);
        PLATO_CUDA(h, cudaMemsetAsync(h->v_tmp, 0, sizeof(double) * n, h->stream));
        RC(launch_dirichlet_rhs(h, h->v_tmp, scale));
        RC(launch_ebe_apply64_unmasked(h, h->v_tmp, h->v_q));
        RC(launch_masked_axpy(h, -1.0, h->v_q, b));
    }
    return launch_dirichlet_rhs(h, b, scale);
}

}  // namespace plato

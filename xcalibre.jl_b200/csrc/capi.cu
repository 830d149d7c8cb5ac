// capi.cu -- extern "C" entry points of libxcal_b200.so (include/xcal_b200.h).
// Every call catches library errors and turns them into a status code plus a
// message retrievable with xcal_last_error; nothing aborts the process.
#include <cstddef>
#include <exception>
#include <vector>
#include <new>

#include "case.hpp"
#include "dev_common.cuh"
#include "kernels.hpp"

namespace xcal {
DevMesh* upload_mesh(const xcal_mesh_desc* d, cudaStream_t s);
std::atomic<long long> g_launch_count{0};
thread_local long long t_launch_count = 0;
thread_local size_t* t_alloc_acc = nullptr;
}
using namespace xcal;

static int set_error(xcal_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->set_error(msg);
    return code;
}

#define XCAL_GUARD(ctx, ...)                                                  \
    try {                                                                     \
        __VA_ARGS__;                                                          \
        return XCAL_OK;                                                       \
    } catch (const ::xcal::Error& e) {                                        \
        return set_error(ctx, e.code, e.msg);                                 \
    } catch (const std::bad_alloc&) {                                         \
        return set_error(ctx, XCAL_ERR_OOM, "host allocation failed");        \
    } catch (const std::exception& e) {                                       \
        return set_error(ctx, XCAL_ERR_INVALID, e.what());                    \
    }

static int select_device(xcal_ctx* ctx) {
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return set_error(ctx, XCAL_ERR_CUDA, cudaGetErrorString(e));
    return XCAL_OK;
}

extern "C" {

const char* xcal_version(void) { return "xcal_b200 0.1 (sm_100a, FP64 hot path)"; }

int32_t xcal_det_math(int32_t which, const double* in, double* out, int64_t n) {
    if (!in || !out || n < 0 || which < 0 || which > 3) return XCAL_ERR_INVALID;
    for (int64_t i = 0; i < n; ++i)
        out[i] = which == 0   ? det_exp_neg(in[i])
                 : which == 1 ? det_log(in[i])
                 : which == 2 ? det_tanh_pos(in[i])
                              : det_pow(in[i], -1.30);
    return XCAL_OK;
}

#define XCAL_OFF(T, f) (int64_t) offsetof(T, f)
int32_t xcal_abi_layout(int32_t which, int64_t* out, int32_t cap) {
    std::vector<int64_t> v;
    switch (which) {
        case XCAL_LAYOUT_MESH_DESC: {
            using T = xcal_mesh_desc;
            v = {sizeof(T), XCAL_OFF(T, n_cells), XCAL_OFF(T, n_faces), XCAL_OFF(T, n_bfaces),
                 XCAL_OFF(T, face_owner), XCAL_OFF(T, face_neigh), XCAL_OFF(T, face_centre),
                 XCAL_OFF(T, face_normal), XCAL_OFF(T, face_e), XCAL_OFF(T, face_area), XCAL_OFF(T, face_delta),
                 XCAL_OFF(T, face_weight), XCAL_OFF(T, cell_centre), XCAL_OFF(T, cell_volume),
                 XCAL_OFF(T, cell_faces_offset), XCAL_OFF(T, cell_faces), XCAL_OFF(T, cell_nsign),
                 XCAL_OFF(T, cell_neighbours), XCAL_OFF(T, boundary_cellsID), XCAL_OFF(T, n_patches),
                 XCAL_OFF(T, patch_start), XCAL_OFF(T, patch_count), XCAL_OFF(T, dim)};
            break;
        }
        case XCAL_LAYOUT_BC: {
            using T = xcal_bc;
            v = {sizeof(T), XCAL_OFF(T, type), XCAL_OFF(T, patch), XCAL_OFF(T, value), XCAL_OFF(T, face_values),
                 XCAL_OFF(T, face_map), XCAL_OFF(T, distance), XCAL_OFF(T, partner_patch), XCAL_OFF(T, wall)};
            break;
        }
        case XCAL_LAYOUT_SOLVER_SETUP: {
            using T = xcal_solver_setup;
            v = {sizeof(T), XCAL_OFF(T, solver), XCAL_OFF(T, precond), XCAL_OFF(T, convergence), XCAL_OFF(T, relax),
                 XCAL_OFF(T, atol), XCAL_OFF(T, rtol), XCAL_OFF(T, itmax), XCAL_OFF(T, smoother_loops),
                 XCAL_OFF(T, smoother_omega)};
            break;
        }
        case XCAL_LAYOUT_SCHEMES: {
            using T = xcal_schemes;
            v = {sizeof(T), XCAL_OFF(T, time), XCAL_OFF(T, divergence), XCAL_OFF(T, gradient), XCAL_OFF(T, limiter),
                 XCAL_OFF(T, limiter_level)};
            break;
        }
        case XCAL_LAYOUT_CONFIG: {
            using T = xcal_config;
            v = {sizeof(T),
                 XCAL_OFF(T, algorithm), XCAL_OFF(T, turbulence), XCAL_OFF(T, nu), XCAL_OFF(T, smagorinsky_C),
                 XCAL_OFF(T, les_delta_distance), XCAL_OFF(T, les_delta_power), XCAL_OFF(T, U_schemes),
                 XCAL_OFF(T, p_schemes), XCAL_OFF(T, U_solver), XCAL_OFF(T, p_solver), XCAL_OFF(T, iterations),
                 XCAL_OFF(T, dt), XCAL_OFF(T, has_pref), XCAL_OFF(T, pref), XCAL_OFF(T, inner_loops),
                 XCAL_OFF(T, ncorrectors), XCAL_OFF(T, precision), XCAL_OFF(T, inner_rtol), XCAL_OFF(T, n_bc_U),
                 XCAL_OFF(T, n_bc_p), XCAL_OFF(T, n_bc_nut), XCAL_OFF(T, bc_U), XCAL_OFF(T, bc_p),
                 XCAL_OFF(T, bc_nut), XCAL_OFF(T, kw_beta_star), XCAL_OFF(T, kw_alpha1), XCAL_OFF(T, kw_beta1),
                 XCAL_OFF(T, kw_sigma_k), XCAL_OFF(T, kw_sigma_omega), XCAL_OFF(T, k_schemes),
                 XCAL_OFF(T, omega_schemes), XCAL_OFF(T, k_solver), XCAL_OFF(T, omega_solver), XCAL_OFF(T, n_bc_k),
                 XCAL_OFF(T, n_bc_omega), XCAL_OFF(T, bc_k), XCAL_OFF(T, bc_omega), XCAL_OFF(T, sst_beta2),
                 XCAL_OFF(T, sst_sigma_k2), XCAL_OFF(T, sst_sigma_omega2), XCAL_OFF(T, y_schemes),
                 XCAL_OFF(T, y_solver), XCAL_OFF(T, n_bc_y), XCAL_OFF(T, bc_y),
                 XCAL_OFF(T, keq_ck), XCAL_OFF(T, keq_ce), XCAL_OFF(T, lke_Tu), XCAL_OFF(T, kl_schemes),
                 XCAL_OFF(T, kl_solver), XCAL_OFF(T, n_bc_kl), XCAL_OFF(T, bc_kl)};
            break;
        }
        case XCAL_LAYOUT_POLYMESH_DESC: {
            using T = xcal_polymesh_desc;
            v = {sizeof(T), XCAL_OFF(T, n_points), XCAL_OFF(T, points), XCAL_OFF(T, n_faces),
                 XCAL_OFF(T, face_offsets), XCAL_OFF(T, face_nodes), XCAL_OFF(T, owner),
                 XCAL_OFF(T, n_internal_faces), XCAL_OFF(T, neighbour), XCAL_OFF(T, n_patches),
                 XCAL_OFF(T, patch_sizes)};
            break;
        }
        case XCAL_LAYOUT_MESH_BUFFERS: {
            using T = xcal_mesh_buffers;
            v = {sizeof(T), XCAL_OFF(T, face_owner), XCAL_OFF(T, face_neigh), XCAL_OFF(T, face_centre),
                 XCAL_OFF(T, face_normal), XCAL_OFF(T, face_e), XCAL_OFF(T, face_area), XCAL_OFF(T, face_delta),
                 XCAL_OFF(T, face_weight), XCAL_OFF(T, cell_centre), XCAL_OFF(T, cell_volume),
                 XCAL_OFF(T, cell_faces_offset), XCAL_OFF(T, cell_faces), XCAL_OFF(T, cell_nsign),
                 XCAL_OFF(T, cell_neighbours), XCAL_OFF(T, boundary_cellsID), XCAL_OFF(T, patch_start),
                 XCAL_OFF(T, patch_count)};
            break;
        }
        case XCAL_LAYOUT_TERM: {
            using T = xcal_term;
            v = {sizeof(T), XCAL_OFF(T, op), XCAL_OFF(T, scheme), XCAL_OFF(T, sign), XCAL_OFF(T, flux),
                 XCAL_OFF(T, value)};
            break;
        }
        case XCAL_LAYOUT_SOURCE: {
            using T = xcal_source;
            v = {sizeof(T), XCAL_OFF(T, sign), XCAL_OFF(T, field), XCAL_OFF(T, value)};
            break;
        }
        default:
            return XCAL_ERR_INVALID;
    }
    if (!out || cap < (int32_t)v.size()) return XCAL_ERR_INVALID;
    for (size_t k = 0; k < v.size(); ++k) out[k] = v[k];
    return (int32_t)v.size();
}
#undef XCAL_OFF

int32_t xcal_ctx_create(int32_t device, xcal_ctx** out) {
    if (!out) return XCAL_ERR_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) return XCAL_ERR_CUDA;
    if (cudaSetDevice(device) != cudaSuccess) return XCAL_ERR_CUDA;
    cudaFree(nullptr);  // create the context now
    xcal_ctx* c = new (std::nothrow) xcal_ctx();
    if (!c) return XCAL_ERR_OOM;
    c->device = device;
    *out = c;
    return XCAL_OK;
}

int32_t xcal_ctx_destroy(xcal_ctx* ctx) {
    delete ctx;
    return XCAL_OK;
}

const char* xcal_last_error(const xcal_ctx* ctx) {
    return ctx ? const_cast<xcal_ctx*>(ctx)->last_error() : "no context";
}

int32_t xcal_mesh_upload(xcal_ctx* ctx, const xcal_mesh_desc* desc, xcal_mesh** out) {
    if (!ctx || !out) return XCAL_ERR_INVALID;
    *out = nullptr;
    if (int e = select_device(ctx)) return e;
    XCAL_GUARD(ctx, {
        std::unique_ptr<DevMesh> m(upload_mesh(desc, 0));
        xcal_mesh* h = new xcal_mesh();
        h->ctx = ctx;
        h->m = std::move(m);
        *out = h;
    })
}

int32_t xcal_mesh_destroy(xcal_mesh* mesh) {
    delete mesh;
    return XCAL_OK;
}

int32_t xcal_case_create(xcal_ctx* ctx, const xcal_mesh* mesh, const xcal_config* cfg, xcal_case** out) {
    if (!ctx || !mesh || !cfg || !out) return XCAL_ERR_INVALID;
    *out = nullptr;
    if (int e = select_device(ctx)) return e;
    XCAL_GUARD(ctx, {
        std::unique_ptr<Case> c(new Case(ctx, mesh->m.get(), cfg));
        xcal_case* h = new xcal_case();
        h->c = std::move(c);
        *out = h;
    })
}

int32_t xcal_case_destroy(xcal_case* cs) {
    delete cs;
    return XCAL_OK;
}

int32_t xcal_case_nnz(const xcal_case* cs, int32_t eqn, int64_t* nnz) {
    if (!cs || !nnz || (eqn != XCAL_EQN_U && eqn != XCAL_EQN_P)) return XCAL_ERR_INVALID;
    *nnz = eqn == XCAL_EQN_U ? cs->c->U.nnz_csr : cs->c->P.nnz_csr;
    return XCAL_OK;
}

int32_t xcal_case_csr_pattern(const xcal_case* cs, int32_t eqn, int32_t* rowptr, int32_t* colval) {
    if (!cs || !rowptr || !colval || (eqn != XCAL_EQN_U && eqn != XCAL_EQN_P)) return XCAL_ERR_INVALID;
    const Equation& E = eqn == XCAL_EQN_U ? cs->c->U : cs->c->P;
    const DevMesh& m = *cs->c->mesh;
    // export in the original numbering (rows are stored in storage order)
    rowptr[0] = 0;
    long k = 0;
    for (int i = 0; i < E.n; ++i) {
        int st = m.inv[i];
        for (int q = 0; q < E.len[st]; ++q) colval[k++] = m.perm[E.colval[E.base(st) + SELL_C * q]];
        rowptr[i + 1] = (int32_t)k;
    }
    return XCAL_OK;
}

int32_t xcal_case_get_system(const xcal_case* cs, int32_t eqn, int32_t component, double* nzval, double* b) {
    if (!cs || (eqn != XCAL_EQN_U && eqn != XCAL_EQN_P)) return XCAL_ERR_INVALID;
    Case* c = cs->c.get();
    XCAL_GUARD(c->ctx, {
        const Equation& E = eqn == XCAL_EQN_U ? c->U : c->P;
        if (eqn == XCAL_EQN_U && (component < -1 || component > 2)) fail(XCAL_ERR_INVALID, "component");
        c->sync();
        const DevMesh& m = *c->mesh;
        if (nzval) {
            std::vector<double> nz(E.nnz);
            XCAL_CUDA(cudaMemcpy(nz.data(), E.nz.p, E.nnz * sizeof(double), cudaMemcpyDeviceToHost));
            if (eqn == XCAL_EQN_U && component < 0) {
                std::vector<double> d0(E.n);
                XCAL_CUDA(cudaMemcpy(d0.data(), E.diag0.p, E.n * sizeof(double), cudaMemcpyDeviceToHost));
                for (int st = 0; st < E.n; ++st) nz[E.diag[st]] = d0[st];
                // periodic pair slots are 0 in A0 (only the BCs write them)
                for (const std::vector<int>* v : {&c->bcU.h_pNP, &c->bcU.h_pPN})
                    for (int s : *v)
                        if (s >= 0) nz[s] = 0.0;
            }
            long k = 0;
            for (int i = 0; i < E.n; ++i) {
                int st = m.inv[i];
                for (int q = 0; q < E.len[st]; ++q) nzval[k++] = nz[E.base(st) + SELL_C * q];
            }
        }
        if (b) {
            int bc = eqn == XCAL_EQN_U ? (component < 0 ? 0 : component) : 0;
            std::vector<double> tmp(E.n);
            XCAL_CUDA(cudaMemcpy(tmp.data(), E.b[bc].p, E.n * sizeof(double), cudaMemcpyDeviceToHost));
            for (int i = 0; i < E.n; ++i) b[i] = tmp[m.inv[i]];
        }
    })
}

static int field_io(xcal_case* cs, int32_t field, double* host, int64_t count, bool set) {
    if (!cs || !host || field < 0 || field >= XCAL_FIELD_COUNT) return XCAL_ERR_INVALID;
    Case* c = cs->c.get();
    XCAL_GUARD(c->ctx, {
        int ncomp = field == XCAL_FIELD_U || field == XCAL_FIELD_GRADP || field == XCAL_FIELD_HV ||
                            field == XCAL_FIELD_UF
                        ? 3
                        : (field == XCAL_FIELD_GRADU ? 9 : 1);
        long per = 0;
        c->field_comp(field, 0, per);
        if (count != (int64_t)ncomp * per) fail(XCAL_ERR_INVALID, "field size mismatch");
        // device arrays are in storage order, the ABI uses the original order:
        // each component is staged in original order and permuted on the
        // device (set: field[st] = io[perm[st]]; get: io[i] = field[inv[i]])
        bool face = field == XCAL_FIELD_MDOTF || field == XCAL_FIELD_NUEFF || field == XCAL_FIELD_NUTF ||
                    field == XCAL_FIELD_UF || field == XCAL_FIELD_PF || field == XCAL_FIELD_RDF;
        const DevMesh& m = *c->mesh;
        const int* to_storage = face ? m.d_fperm.p : m.d_perm.p;
        const int* to_original = face ? m.d_finv.p : m.d_inv.p;
        for (int d = 0; d < ncomp; ++d) {
            long n = 0;
            double* p = c->field_comp(field, d, n);
            double* h = host + (size_t)d * per;
            if (set) {
                XCAL_CUDA(cudaMemcpyAsync(c->io.p, h, per * sizeof(double), cudaMemcpyHostToDevice, c->stream));
                launch_gather(c->stream, per, c->io.p, to_storage, p);
            } else {
                launch_gather(c->stream, per, p, to_original, c->io.p);
                XCAL_CUDA(cudaMemcpyAsync(h, c->io.p, per * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
            }
        }
        c->sync();
    })
}

int32_t xcal_case_set_field(xcal_case* cs, int32_t field, const double* host, int64_t count) {
    return field_io(cs, field, const_cast<double*>(host), count, true);
}

int32_t xcal_case_get_field(const xcal_case* cs, int32_t field, double* host, int64_t count) {
    return field_io(const_cast<xcal_case*>(cs), field, host, count, false);
}

int32_t xcal_case_set_bc_values(xcal_case* cs, int32_t eqn, int32_t bc_index, const double* values, int64_t count) {
    if (!cs || !values || (eqn != XCAL_EQN_U && eqn != XCAL_EQN_P)) return XCAL_ERR_INVALID;
    Case* c = cs->c.get();
    XCAL_GUARD(c->ctx, {
        BCTable& T = eqn == XCAL_EQN_U ? c->bcU : c->bcP;
        int ncomp = eqn == XCAL_EQN_U ? 3 : 1;
        if (bc_index < 0 || bc_index >= (int)T.src.size()) fail(XCAL_ERR_INVALID, "bc_index");
        const xcal_bc& bc = T.src[bc_index];
        if (bc.type != XCAL_BC_DIRICHLET_FUNCTION) fail(XCAL_ERR_INVALID, "BC is not a DirichletFunction");
        int start = c->mesh->patch_start[bc.patch], n = c->mesh->patch_count[bc.patch];
        if (count != (int64_t)ncomp * n) fail(XCAL_ERR_INVALID, "value count mismatch");
        for (int i = 0; i < n; ++i)
            for (int d = 0; d < ncomp; ++d) T.val[3 * (size_t)(start + i) + d] = values[(size_t)ncomp * i + d];
        c->sync();
        XCAL_CUDA(cudaMemcpy(T.d_val.p, T.val.data(), T.val.size() * sizeof(double), cudaMemcpyHostToDevice));
    })
}

int32_t xcal_simple_iterate(xcal_case* cs, int32_t n_iter, double* res_hist, int32_t* n_done, int32_t* converged) {
    if (!cs || n_iter < 0) return XCAL_ERR_INVALID;
    Case* c = cs->c.get();
    if (n_done) *n_done = 0;
    if (converged) *converged = 0;
    XCAL_GUARD(c->ctx, {
        for (int k = 0; k < n_iter; ++k) {
            double r[4];
            bool conv = c->simple_iteration(r);
            if (res_hist)
                for (int q = 0; q < 4; ++q) res_hist[4 * k + q] = r[q];
            if (n_done) *n_done = k + 1;
            if (conv) {
                if (converged) *converged = 1;
                break;
            }
        }
    })
}

int32_t xcal_piso_step(xcal_case* cs, int32_t n_steps, double* res_hist, double* courant, int32_t* n_done) {
    if (!cs || n_steps < 0) return XCAL_ERR_INVALID;
    Case* c = cs->c.get();
    if (n_done) *n_done = 0;
    XCAL_GUARD(c->ctx, {
        for (int k = 0; k < n_steps; ++k) {
            double r[4];
            double co = c->piso_step(r);
            if (res_hist)
                for (int q = 0; q < 4; ++q) res_hist[4 * k + q] = r[q];
            if (courant) courant[k] = co;
            if (n_done) *n_done = k + 1;
        }
    })
}

#define XCAL_STEP(name, ...)                            \
    int32_t name {                                      \
        if (!cs) return XCAL_ERR_INVALID;               \
        Case* c = cs->c.get();                          \
        XCAL_GUARD(c->ctx, { __VA_ARGS__; c->sync(); }) \
    }

XCAL_STEP(xcal_initial_calculations(xcal_case* cs), c->initial_calculations())
XCAL_STEP(xcal_discretise(xcal_case* cs, int32_t eqn), c->discretise(eqn))
XCAL_STEP(xcal_apply_boundary_conditions(xcal_case* cs, int32_t eqn, int32_t component),
          c->apply_bcs(eqn, component))
XCAL_STEP(xcal_implicit_relaxation_diagdom(xcal_case* cs, int32_t component), c->relax_U(component))
XCAL_STEP(xcal_set_reference(xcal_case* cs), c->set_reference())
XCAL_STEP(xcal_update_preconditioner(xcal_case* cs, int32_t eqn), c->update_precond(eqn))
XCAL_STEP(xcal_pressure_predictor(xcal_case* cs), c->pressure_predictor(true))
XCAL_STEP(xcal_flux_divergence(xcal_case* cs), {
    c->flux_divergence();
    XCAL_CUDA(cudaMemcpyAsync(c->prev.p, c->p.p, c->mesh->nC * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
})
XCAL_STEP(xcal_explicit_relaxation_p(xcal_case* cs, double alpha), c->explicit_relaxation_p(alpha))
XCAL_STEP(xcal_grad_p(xcal_case* cs), c->grad_p())
XCAL_STEP(xcal_correct(xcal_case* cs), c->correct())
XCAL_STEP(xcal_turbulence(xcal_case* cs), c->turbulence())

int32_t xcal_solve_system(xcal_case* cs, int32_t eqn, int32_t component, double* residual, int32_t* iterations) {
    if (!cs) return XCAL_ERR_INVALID;
    Case* c = cs->c.get();
    XCAL_GUARD(c->ctx, {
        int it = 0;
        double r = c->solve_system(eqn, eqn == XCAL_EQN_U ? component : 0, &it);
        if (residual) *residual = r;
        if (iterations) *iterations = it;
    })
}

int32_t xcal_solve_equation(xcal_case* cs, int32_t eqn, double* res) {
    if (!cs || !res) return XCAL_ERR_INVALID;
    Case* c = cs->c.get();
    XCAL_GUARD(c->ctx, {
        if (eqn == XCAL_EQN_U)
            c->solve_equation_U(res);
        else
            res[0] = c->solve_equation_p();
    })
}

int32_t xcal_max_courant(xcal_case* cs, double* courant) {
    if (!cs || !courant) return XCAL_ERR_INVALID;
    Case* c = cs->c.get();
    XCAL_GUARD(c->ctx, { *courant = c->max_courant(); })
}

int32_t xcal_get_timings(const xcal_case* cs, double* ms, int32_t n) {
    if (!cs || !ms) return XCAL_ERR_INVALID;
    int k = n < 6 ? n : 6;
    for (int i = 0; i < k; ++i) ms[i] = cs->c->ms[i];
    return k;
}

int32_t xcal_get_launch_count(const xcal_case* cs, int64_t* count) {
    (void)cs;  // the count is library-wide; cs may be NULL
    if (!count) return XCAL_ERR_INVALID;
    *count = g_launch_count.load();
    return XCAL_OK;
}

int32_t xcal_case_stream(const xcal_case* cs, void** stream) {
    if (!cs || !stream) return XCAL_ERR_INVALID;
    *stream = (void*)cs->c->stream;
    return XCAL_OK;
}

int32_t xcal_case_set_profiling(xcal_case* cs, int32_t enable) {
    if (!cs) return XCAL_ERR_INVALID;
    cs->c->profiling = enable != 0;
    return XCAL_OK;
}

int32_t xcal_case_mark_initialised(xcal_case* cs) {
    if (!cs) return XCAL_ERR_INVALID;
    cs->c->initialised = true;
    return XCAL_OK;
}

int32_t xcal_case_set_persistent(xcal_case* cs, int32_t mode) {
    if (!cs) return XCAL_ERR_INVALID;
    if (mode != 0 && mode != 1 && mode != 2 && mode != PERSIST_MT1024 && mode != PERSIST_MT512 && mode != 256 &&
        mode != 512 && mode != 1024)
        return XCAL_ERR_INVALID;
    cs->c->persistent_cg = mode;
    return XCAL_OK;
}

int32_t xcal_case_solve_report(const xcal_case* cs, int32_t* iters7, int32_t* status7, int64_t* itmax_hits) {
    if (!cs) return XCAL_ERR_INVALID;
    const Case* c = cs->c.get();
    for (int k = 0; k < 7; ++k) {
        if (iters7) iters7[k] = c->last_iters[k];
        if (status7) status7[k] = c->last_status[k];
    }
    if (itmax_hits) *itmax_hits = c->itmax_hits;
    return XCAL_OK;
}

int32_t xcal_case_set_inner_cg(xcal_case* cs, int32_t mode) {
    if (!cs || mode < 0 || mode >= 2 + 16) return XCAL_ERR_INVALID;
    XCAL_GUARD(cs->c->ctx, cs->c->set_inner_cg(mode));
}

int32_t xcal_case_set_dilu_mode(xcal_case* cs, int32_t mode) {
    if (!cs || mode < 0 || mode > 3) return XCAL_ERR_INVALID;
    Case* c = cs->c.get();
    c->dilu_mode = mode;
    if (mode != 0) {
        c->U.use_block = c->P.use_block = mode == 1;
        c->U.use_grid = c->P.use_grid = mode == 3;
    }
    if (c->step_graph) {  // a captured step holds the previous form
        c->sync();
        cudaGraphExecDestroy(c->step_graph);
        c->step_graph = nullptr;
    }
    return XCAL_OK;
}

int32_t xcal_case_tuning(xcal_case* cs, int32_t* out6) {
    if (!cs || !out6) return XCAL_ERR_INVALID;
    Case* c = cs->c.get();
    XCAL_GUARD(c->ctx, {
        c->autotune();
        const Equation* E[2] = {&c->U, &c->P};
        for (int e = 0; e < 2; ++e) {
            out6[3 * e] = E[e]->spmv_shape.rows_per_thread;
            out6[3 * e + 1] = E[e]->spmv_shape.block;
            out6[3 * e + 2] = E[e]->use_block ? 1 : (E[e]->use_grid ? 2 : 0);
        }
    })
}

int32_t xcal_case_set_graph_mode(xcal_case* cs, int32_t enable) {
    if (!cs) return XCAL_ERR_INVALID;
    Case* c = cs->c.get();
    XCAL_GUARD(c->ctx, { c->set_graph_mode(enable != 0); })
}

int32_t xcal_case_get_profile(const xcal_case* cs, int32_t which, double* ms, int64_t* launches) {
    if (!cs || which < 0 || which > 5) return XCAL_ERR_INVALID;
    if (ms) *ms = cs->c->prof_ms[which];
    if (launches) *launches = cs->c->prof_n[which];
    return XCAL_OK;
}

}  // extern "C"

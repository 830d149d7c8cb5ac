// terms.cu -- scalar equations built from XCALibre's operator DSL.
//
// The reference writes an equation as a list of operators with signs
// (ModelFramework_1_operations.jl:3-63: `-` sets sign = -1 on the operator
// that follows it) equal to a list of sources, e.g.
//     (Time{Euler}(T) + Divergence{Upwind}(mdotf, T)
//        - Laplacian{Linear}(kappa, T) + Si(d, T) == Source(s)) -> ScalarEquation
// and assembles it term by term (Discretise_2_generated_distretisation.jl:
// 90-168) and boundary condition by boundary condition
// (Discretise_5_apply_bcs.jl, boundary_conditions/*.jl).  The SIMPLE/PISO
// drivers use fixed term lists (kernels_fv.cu); an xcal_equation takes any
// list of Time / Divergence / Laplacian / Si terms and sources across the
// C boundary, with the same per-term arithmetic in the reference's order:
//   per cell, per internal face (cell_faces order): AC = sum_t ac_t, AN =
//   sum_t an_t (t in term order, from 0); a_ij = AN, ac_sum += AC;
//   per cell: a_ii = ac_sum + sum_t ac_t(source part), b_i = sum_s
//   (sign_s field_s) V + sum_t b_t;
//   per boundary face (ascending face id per cell): a_ii += sum_t ap_t,
//   b_i += sum_t bp_t.
#include <cmath>
#include <functional>
#include <memory>

#include "case.hpp"
#include "dev_common.cuh"
#include "kernels.hpp"

namespace xcal {

constexpr int TERMS_MAX = 8;
constexpr int SOURCES_MAX = 8;

// a term / source list as kernels read it: flux arrays in storage order
// (face arrays for Divergence / Laplacian, cell arrays for Time / Si), or
// null for a constant
struct TermList {
    int nt, ns;
    int op[TERMS_MAX], scheme[TERMS_MAX];
    double sign[TERMS_MAX], value[TERMS_MAX];
    const double* flux[TERMS_MAX];
    double ssign[SOURCES_MAX], svalue[SOURCES_MAX];
    const double* sfield[SOURCES_MAX];
};

__device__ __forceinline__ double term_flux(const TermList& T, int t, int idx) {
    return T.flux[t] ? T.flux[t][idx] : T.value[t];
}

// scheme! of one term on internal face f seen from the cell with normal
// sign ns (Discretise_1_schemes.jl:12-218)
__device__ __forceinline__ void term_face(const MeshView& m, const TermList& T, int t, int f, int ns, double& ac,
                                          double& an) {
    const double dns = (double)ns;
    switch (T.op[t]) {
        case XCAL_OP_LAPLACIAN: {  // :68-110 (|E_f| does not depend on ns)
            const double ap = (T.sign[t] * (term_flux(T, t, f) * m.Efmag[f])) / m.delta[f];
            ac = -ap;
            an = ap;
            return;
        }
        case XCAL_OP_DIVERGENCE: {  // :114-180
            const double ap = T.sign[t] * (term_flux(T, t, f) * dns);
            if (T.scheme[t] == XCAL_DIV_LINEAR) {
                double w = m.weight[f];
                w = 0.5 + dns * (w - 0.5);
                ac = ap * w;
                an = ap * (1.0 - w);
            } else if (T.scheme[t] == XCAL_DIV_UPWIND) {
                ac = jl_max(ap, 0.0);
                an = -jl_max(-ap, 0.0);
            } else {  // LUST: 0.75 Linear + 0.25 Upwind
                double w = m.weight[f];
                if (ns < 0) w = 1.0 - w;
                const double acL = ap * w, anL = ap * (1.0 - w);
                const double acU = jl_max(ap, 0.0), anU = -jl_max(-ap, 0.0);
                ac = 0.75 * acL + 0.25 * acU;
                an = 0.75 * anL + 0.25 * anU;
            }
            return;
        }
        default:  // Time, Si: nothing on faces
            ac = 0.0;
            an = 0.0;
    }
}

// scheme_source! of one term in cell i (Discretise_1_schemes.jl:26-45, 211-218)
__device__ __forceinline__ void term_cell(const TermList& T, int t, int i, double V, const double* prev, double dt,
                                          double& ac, double& b) {
    ac = 0.0;
    b = 0.0;
    if (T.op[t] == XCAL_OP_TIME && T.scheme[t] == XCAL_TIME_EULER) {
        const double vol_rdt = (term_flux(T, t, i) * V) / dt;
        ac = vol_rdt;
        b = prev[i] * vol_rdt;
    } else if (T.op[t] == XCAL_OP_SI) {
        ac = (T.sign[t] * term_flux(T, t, i)) * V;
    }
}

// _discretise_scalar_model! (Discretise_2_generated_distretisation.jl:125-167)
__global__ void k_assemble_terms(MeshView m, CSRView A, TermList T, const double* __restrict__ prev, double dt,
                                 double* nz, double* b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nC) return;
    double ac_sum = 0.0;
    for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
        const int f = m.cf_face[k];
        const int ns = m.cf_sign[k];
        double AC = 0.0, AN = 0.0;
        for (int t = 0; t < T.nt; ++t) {
            double ac, an;
            term_face(m, T, t, f, ns, ac, an);
            AC = AC + ac;
            AN = AN + an;
        }
        ac_sum = ac_sum + AC;
        nz[A.cf_slot[k]] = AN;
    }
    const double V = m.vol[i];
    double acs = 0.0, bs = 0.0;
    for (int t = 0; t < T.nt; ++t) {
        double ac, bt;
        term_cell(T, t, i, V, prev, dt, ac, bt);
        acs = acs + ac;
        bs = bs + bt;
    }
    nz[A.diag[i]] = ac_sum + acs;
    double b2 = 0.0;
    for (int s = 0; s < T.ns; ++s) b2 = b2 + (T.ssign[s] * (T.sfield[s] ? T.sfield[s][i] : T.svalue[s])) * V;
    b[i] = b2 + bs;
}

// the boundary functors of one term on boundary face f of `cell` for a
// scalar field (boundary_conditions/*.jl: Time and Si contribute nothing)
__device__ __forceinline__ void term_bc(const MeshView& m, const BCView& bc, const TermList& T, int t, int f, int cell,
                                        const double* phi, double& ap, double& bp) {
    ap = 0.0;
    bp = 0.0;
    const int type = bc.type[f];
    if (T.op[t] == XCAL_OP_LAPLACIAN) {
        const double J = term_flux(T, t, f);
        switch (type) {
            case XCAL_BC_DIRICHLET:
            case XCAL_BC_DIRICHLET_FUNCTION: {  // dirichlet.jl:19-25
                const double fl = (J * m.area[f]) / m.delta[f];
                ap = T.sign[t] * (-fl);
                bp = ap * bc.val[3 * f];
                break;
            }
            case XCAL_BC_EXTRAPOLATED:  // extrapolated.jl:21-30
            case XCAL_BC_OMEGA_WALL: {
                const double fl = ((-J) * m.area[f]) / m.delta[f];
                ap = T.sign[t] * fl;
                bp = ap * phi[cell];
                break;
            }
            case XCAL_BC_NEUMANN:  // neumann.jl:23-31
                bp = (J * m.area[f]) * bc.val[3 * f];
                break;
            default:  // Wall, Zerogradient, Symmetry, Empty, wall functions: (0, 0)
                break;
        }
    } else if (T.op[t] == XCAL_OP_DIVERGENCE) {
        const double J = term_flux(T, t, f);
        switch (type) {
            case XCAL_BC_DIRICHLET:
            case XCAL_BC_DIRICHLET_FUNCTION:  // dirichlet.jl:27-31
                bp = (T.sign[t] * (-J)) * bc.val[3 * f];
                break;
            case XCAL_BC_NEUMANN: {  // neumann.jl:33-59
                const double a = T.sign[t] * J;
                ap = a;
                bp = ((-bc.val[3 * f]) * a) * m.delta[f];
                break;
            }
            case XCAL_BC_EMPTY:  // empty.jl:60-102
                break;
            default:  // Wall, Zerogradient, Symmetry, Extrapolated, wall functions
                ap = T.sign[t] * J;
                break;
        }
    }
}

// apply_boundary_conditions! (Discretise_5_apply_bcs.jl) for a term list:
// each cell's boundary faces in ascending face id
__global__ void k_bc_terms(MeshView m, CSRView A, BCView bc, TermList T, const double* __restrict__ phi, double* nz,
                           double* b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nC) return;
    const int ds = A.diag[i];
    double d = nz[ds], bi = b[i];
    for (int k = m.bf_off[i]; k < m.bf_off[i + 1]; ++k) {
        const int f = m.bf_face[k];
        double ap = 0.0, bp = 0.0;
        for (int t = 0; t < T.nt; ++t) {
            double a, q;
            term_bc(m, bc, T, t, f, i, phi, a, q);
            ap = ap + a;
            bp = bp + q;
        }
        d = d + ap;
        bi = bi + bp;
    }
    nz[ds] = d;
    b[i] = bi;
}

}  // namespace xcal

using namespace xcal;

struct xcal_equation {
    Case* c = nullptr;  // not owned; the equation lives on its case's mesh and stream
    Equation E;
    BCTable bc;
    TermList T{};
    std::vector<std::unique_ptr<DBuf<double>>> arrays;  // term fluxes and source fields, storage order
    DBuf<double> prev, phi, stage;
    bool euler = false, extrapolated = false;
};

namespace {

// host values in original order -> device storage order (face or cell arrays)
const double* upload_permuted(xcal_equation* q, const double* host, bool face) {
    const DevMesh& m = *q->c->mesh;
    const long n = face ? m.nF : m.nC;
    q->arrays.emplace_back(new DBuf<double>());
    DBuf<double>& d = *q->arrays.back();
    d.alloc(n);
    q->stage.alloc(n);
    XCAL_CUDA(cudaMemcpyAsync(q->stage.p, host, n * sizeof(double), cudaMemcpyHostToDevice, q->c->stream));
    launch_gather(q->c->stream, n, q->stage.p, face ? m.d_fperm.p : m.d_perm.p, d.p);
    q->c->sync();
    return d.p;
}

void load_cells(xcal_equation* q, const double* host, DBuf<double>& dst) {
    const DevMesh& m = *q->c->mesh;
    if (dst.n != (size_t)m.nC) dst.alloc(m.nC);
    q->stage.alloc(m.nC);
    XCAL_CUDA(cudaMemcpyAsync(q->stage.p, host, m.nC * sizeof(double), cudaMemcpyHostToDevice, q->c->stream));
    launch_gather(q->c->stream, m.nC, q->stage.p, m.d_perm.p, dst.p);
}

int guard(xcal_ctx* ctx, const std::function<void()>& f) {
    try {
        f();
        return XCAL_OK;
    } catch (const Error& e) {
        if (ctx) ctx->set_error(e.msg);
        return e.code;
    } catch (const std::bad_alloc&) {
        if (ctx) ctx->set_error("host allocation failed");
        return XCAL_ERR_OOM;
    } catch (const std::exception& e) {
        if (ctx) ctx->set_error(e.what());
        return XCAL_ERR_INVALID;
    }
}

int nblocks(int n) { return (n + 255) / 256; }

}  // namespace

extern "C" {

int32_t xcal_equation_create(xcal_case* cs, int32_t n_terms, const xcal_term* terms, int32_t n_sources,
                             const xcal_source* sources, int32_t n_bcs, const xcal_bc* bcs, xcal_equation** out) {
    if (!cs || !out || !terms || n_terms < 1 || n_terms > TERMS_MAX || n_sources < 0 || n_sources > SOURCES_MAX ||
        (n_sources > 0 && !sources) || n_bcs < 0 || (n_bcs > 0 && !bcs))
        return XCAL_ERR_INVALID;
    *out = nullptr;
    Case* c = cs->c.get();
    auto q = std::make_unique<xcal_equation>();
    q->c = c;
    const int code = guard(c->ctx, [&] {
        const DevMesh& m = *c->mesh;
        for (int b = 0; b < n_bcs; ++b)
            if (bcs[b].type == XCAL_BC_PERIODIC || bcs[b].type == XCAL_BC_PERIODIC_PARENT)
                fail(XCAL_ERR_UNSUPPORTED, "equation: periodic boundaries are not supported for term lists");
        std::vector<xcal_bc> bv(bcs, bcs + n_bcs);
        build_equation(q->E, m, bv, 1, true, c->stream);
        build_bc_table(q->bc, m, bcs, n_bcs, 1, &q->E, c->stream);
        q->E.b[0].alloc(m.nC);
        q->E.b[0].zero(c->stream);
        TermList& T = q->T;
        T.nt = n_terms;
        T.ns = n_sources;
        for (int t = 0; t < n_terms; ++t) {
            const xcal_term& tm = terms[t];
            if (tm.op < XCAL_OP_TIME || tm.op > XCAL_OP_SI) fail(XCAL_ERR_INVALID, "equation: unknown operator");
            if (tm.op == XCAL_OP_TIME && tm.scheme != XCAL_TIME_STEADY && tm.scheme != XCAL_TIME_EULER)
                fail(XCAL_ERR_UNSUPPORTED, "equation: Time schemes are SteadyState and Euler");
            if (tm.op == XCAL_OP_DIVERGENCE && (tm.scheme < XCAL_DIV_LINEAR || tm.scheme > XCAL_DIV_LUST))
                fail(XCAL_ERR_UNSUPPORTED, "equation: Divergence schemes are Linear, Upwind and LUST");
            if (!(tm.sign == 1.0 || tm.sign == -1.0)) fail(XCAL_ERR_INVALID, "equation: a term's sign is +1 or -1");
            T.op[t] = tm.op;
            T.scheme[t] = tm.scheme;
            T.sign[t] = tm.sign;
            T.value[t] = tm.value;
            const bool face = tm.op == XCAL_OP_DIVERGENCE || tm.op == XCAL_OP_LAPLACIAN;
            T.flux[t] = tm.flux ? upload_permuted(q.get(), tm.flux, face) : nullptr;
            q->euler |= tm.op == XCAL_OP_TIME && tm.scheme == XCAL_TIME_EULER;
        }
        for (int s = 0; s < n_sources; ++s) {
            if (!(sources[s].sign == 1.0 || sources[s].sign == -1.0))
                fail(XCAL_ERR_INVALID, "equation: a source's sign is +1 or -1");
            T.ssign[s] = sources[s].sign;
            T.svalue[s] = sources[s].value;
            T.sfield[s] = sources[s].field ? upload_permuted(q.get(), sources[s].field, false) : nullptr;
        }
        for (int b = 0; b < n_bcs; ++b)
            q->extrapolated |= bcs[b].type == XCAL_BC_EXTRAPOLATED || bcs[b].type == XCAL_BC_OMEGA_WALL;
        q->phi.alloc(m.nC);
        q->phi.zero(c->stream);
        c->sync();
    });
    if (code != XCAL_OK) return code;
    *out = q.release();
    return XCAL_OK;
}

// frees the equation's device memory (cudaFree waits for work using it);
// touches nothing of its case, which may already be gone
int32_t xcal_equation_destroy(xcal_equation* q) {
    delete q;
    return XCAL_OK;
}

int32_t xcal_equation_discretise(xcal_equation* q, const double* prev, double dt) {
    if (!q) return XCAL_ERR_INVALID;
    Case* c = q->c;
    return guard(c->ctx, [&] {
        if (q->euler) {
            if (!prev) fail(XCAL_ERR_INVALID, "equation: Time{Euler} needs the previous values");
            if (!(dt > 0.0)) fail(XCAL_ERR_INVALID, "equation: Time{Euler} needs dt > 0");
            load_cells(q, prev, q->prev);
        }
        k_assemble_terms<<<nblocks(c->mesh->nC), 256, 0, c->stream>>>(c->mv(), q->E.view(), q->T,
                                                                       q->euler ? q->prev.p : nullptr, dt,
                                                                       q->E.nz.p, q->E.b[0].p);
        XCAL_CHECK_LAUNCH();
        c->sync();
    });
}

int32_t xcal_equation_apply_bcs(xcal_equation* q, const double* phi) {
    if (!q) return XCAL_ERR_INVALID;
    Case* c = q->c;
    return guard(c->ctx, [&] {
        if (q->extrapolated && !phi) fail(XCAL_ERR_INVALID, "equation: Extrapolated boundaries need the field");
        if (phi) load_cells(q, phi, q->phi);
        k_bc_terms<<<nblocks(c->mesh->nC), 256, 0, c->stream>>>(c->mv(), q->E.view(), q->bc.view(), q->T, q->phi.p,
                                                                 q->E.nz.p, q->E.b[0].p);
        XCAL_CHECK_LAUNCH();
        c->sync();
    });
}

int32_t xcal_equation_nnz(const xcal_equation* q, int64_t* nnz) {
    if (!q || !nnz) return XCAL_ERR_INVALID;
    *nnz = q->E.nnz_csr;
    return XCAL_OK;
}

int32_t xcal_equation_get_system(const xcal_equation* q, int32_t* rowptr, int32_t* colval, double* nzval,
                                 double* b) {
    if (!q) return XCAL_ERR_INVALID;
    Case* c = q->c;
    return guard(c->ctx, [&] {
        c->sync();
        const Equation& E = q->E;
        const DevMesh& m = *c->mesh;
        std::vector<double> nz(E.nnz), bs(E.n);
        XCAL_CUDA(cudaMemcpy(nz.data(), E.nz.p, E.nnz * sizeof(double), cudaMemcpyDeviceToHost));
        XCAL_CUDA(cudaMemcpy(bs.data(), E.b[0].p, E.n * sizeof(double), cudaMemcpyDeviceToHost));
        // rows in the original numbering, entries in the reference's CSR order
        long k = 0;
        if (rowptr) rowptr[0] = 0;
        for (int i = 0; i < E.n; ++i) {
            const int st = m.inv[i];
            for (int e = 0; e < E.len[st]; ++e, ++k) {
                const int slot = E.base(st) + SELL_C * e;
                if (colval) colval[k] = m.perm[E.colval[slot]];
                if (nzval) nzval[k] = nz[slot];
            }
            if (rowptr) rowptr[i + 1] = (int32_t)k;
            if (b) b[i] = bs[st];
        }
    });
}

int32_t xcal_equation_solve(xcal_equation* q, const xcal_solver_setup* setup, double* phi, double* residual,
                            int32_t* iterations) {
    if (!q || !setup || !phi) return XCAL_ERR_INVALID;
    Case* c = q->c;
    return guard(c->ctx, [&] {
        if (setup->solver != XCAL_SOLVER_CG && setup->solver != XCAL_SOLVER_BICGSTAB)
            fail(XCAL_ERR_INVALID, "equation: solver");
        if (setup->precond < XCAL_PRECOND_NONE || setup->precond > XCAL_PRECOND_DILU)
            fail(XCAL_ERR_INVALID, "equation: preconditioner");
        const DevMesh& m = *c->mesh;
        load_cells(q, phi, q->phi);
        c->update_precond_E(q->E, setup->precond);
        if (setup->smoother_loops > 0)
            kr_jacobi_smooth(c->stream, q->E.view(), q->E.nz.p, q->E.b[0].p, q->phi.p, c->ws.t.p,
                             setup->smoother_loops, setup->smoother_omega);
        // the p system's Krylov workspace and scalars (report slot 6); FP64
        // whatever the case's precision
        Case::SolveRef R{&q->E, *setup, q->phi.p, q->E.b[0].p, 0, 1, 6};
        int its = 0;
        const double r = c->solve_system_ref(R, &its, true);
        launch_gather(c->stream, m.nC, q->phi.p, m.d_inv.p, c->io.p);
        XCAL_CUDA(cudaMemcpyAsync(phi, c->io.p, m.nC * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        c->sync();
        if (residual) *residual = r;
        if (iterations) *iterations = its;
    });
}

}  // extern "C"

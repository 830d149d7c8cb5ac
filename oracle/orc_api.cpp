// orc_api.cpp -- C entry points of the CPU oracle (loaded by the tests with
// ctypes).  TEST INFRASTRUCTURE ONLY (see orc_common.hpp).
#include "orc_internal.hpp"

#include <cstring>
#include <exception>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {
void initial_calculations(Case& C);
void solve_equation_U(Case& C, double res[3], int iters[3]);
double solve_equation_p(Case& C, int* iters);
void pressure_predictor(Case& C, bool with_H);
void H(Case& C);
void flux_divergence(Case& C);
void explicit_relaxation_p(Case& C, double alpha);
void correct(Case& C);
void turbulence(Case& C);
double max_courant(Case& C);
bool simple_iteration(Case& C, double* res4);
double piso_step(Case& C, double* res4);
void o_discretise(Case& C, int eqn);
void o_apply_bcs(Case& C, int eqn, int comp);
void o_relax(Case& C, int comp);
void o_set_reference(Case& C);
void o_update_precond(Case& C, int eqn);
double o_solve_system(Case& C, int eqn, int comp, int* iters);
void o_grad_p(Case& C);
void o_dilu(const CSR& A, std::vector<double>& D);
void o_dilu_ldiv(const CSR& A, const std::vector<double>& D, std::vector<double>& x, const std::vector<double>& b);
void jacobi_smooth(const CSR& A, const double* b, double* x, int loops, double omega);

Mesh* mesh_from_desc(const xcal_mesh_desc* d) {
    Mesh* m = new Mesh();
    m->n_cells = d->n_cells;
    m->n_faces = d->n_faces;
    m->n_bfaces = d->n_bfaces;
    m->n_ifaces = d->n_faces - d->n_bfaces;
    int nF = d->n_faces, nC = d->n_cells;
    m->owner.assign(d->face_owner, d->face_owner + nF);
    m->neigh.assign(d->face_neigh, d->face_neigh + nF);
    auto v3 = [](const double* p, int n, std::vector<V3>& out) {
        out.resize(n);
        for (int i = 0; i < n; ++i) out[i] = {p[3 * i], p[3 * i + 1], p[3 * i + 2]};
    };
    v3(d->face_centre, nF, m->fcentre);
    v3(d->face_normal, nF, m->fnormal);
    v3(d->face_e, nF, m->fe);
    m->farea.assign(d->face_area, d->face_area + nF);
    m->fdelta.assign(d->face_delta, d->face_delta + nF);
    m->fweight.assign(d->face_weight, d->face_weight + nF);
    v3(d->cell_centre, nC, m->ccentre);
    m->cvol.assign(d->cell_volume, d->cell_volume + nC);
    m->cf_off.assign(d->cell_faces_offset, d->cell_faces_offset + nC + 1);
    int nk = m->cf_off[nC];
    m->cell_faces.assign(d->cell_faces, d->cell_faces + nk);
    m->cell_nsign.assign(d->cell_nsign, d->cell_nsign + nk);
    m->cell_neigh.assign(d->cell_neighbours, d->cell_neighbours + nk);
    m->bcell.assign(d->boundary_cellsID, d->boundary_cellsID + d->n_bfaces);
    m->patch_start.assign(d->patch_start, d->patch_start + d->n_patches);
    m->patch_count.assign(d->patch_count, d->patch_count + d->n_patches);
    m->dim = d->dim == 2 ? 2 : 3;
    return m;
}
}  // namespace orc

using namespace orc;

static void set_err(char* err, int len, const char* msg) {
    if (err && len > 0) {
        std::strncpy(err, msg, len - 1);
        err[len - 1] = 0;
    }
}

static std::vector<double>* field_ptr(Case* C, int field, int& ncomp, int& per) {
    ncomp = 1;
    per = C->nC;
    switch (field) {
        case XCAL_FIELD_U: ncomp = 3; return C->U;
        case XCAL_FIELD_P: return &C->p;
        case XCAL_FIELD_MDOTF: per = C->nF; return &C->mdotf;
        case XCAL_FIELD_NUEFF: per = C->nF; return &C->nueff;
        case XCAL_FIELD_GRADP: ncomp = 3; return C->gradp;
        case XCAL_FIELD_GRADU: ncomp = 9; return C->gradU;
        case XCAL_FIELD_RD: return &C->rD;
        case XCAL_FIELD_HV: ncomp = 3; return C->Hv;
        case XCAL_FIELD_DIVHV: return &C->divHv;
        case XCAL_FIELD_NUT: return &C->nut;
        case XCAL_FIELD_NUTF: per = C->nF; return &C->nutf;
        case XCAL_FIELD_UF: ncomp = 3; per = C->nF; return C->Uf;
        case XCAL_FIELD_PF: per = C->nF; return &C->pf;
        case XCAL_FIELD_RDF: per = C->nF; return &C->rDf;
        case XCAL_FIELD_DELTA: return &C->Delta;
        case XCAL_FIELD_K: return &C->k;
        case XCAL_FIELD_OMEGA: return &C->omega;
        case XCAL_FIELD_WALLDIST: return &C->yw;
        case XCAL_FIELD_PK: return &C->Pk;
        case XCAL_FIELD_DK: return &C->Dk;
        case XCAL_FIELD_DW: return &C->Dw;
        case XCAL_FIELD_KL: return C->kl.empty() ? nullptr : &C->kl;
        case XCAL_FIELD_GAMMA: return C->gam.empty() ? nullptr : &C->gam;
        default: return nullptr;
    }
}

extern "C" {

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int orc_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void* orc_mesh_build(int np, const double* pts, int nf, const int* face_off, const int* face_nodes,
                     const int* owner, int nif, const int* neigh, int npatch, const int* patch_nfaces,
                     char* err, int errlen) {
    try {
        return build_foam_mesh(np, pts, nf, face_off, face_nodes, owner, nif, neigh, npatch, patch_nfaces);
    } catch (std::exception& e) {
        set_err(err, errlen, e.what());
        return nullptr;
    }
}

void* orc_mesh_from_desc(const xcal_mesh_desc* d) { return mesh_from_desc(d); }

void orc_mesh_free(void* m) { delete (Mesh*)m; }

void orc_mesh_sizes(void* mp, int* out) {
    Mesh* m = (Mesh*)mp;
    out[0] = m->n_cells;
    out[1] = m->n_faces;
    out[2] = m->n_bfaces;
    out[3] = m->n_ifaces;
    out[4] = (int)m->patch_start.size();
    out[5] = (int)m->cell_nodes.size();
    out[6] = (int)m->points.size();
}

void orc_mesh_export(void* mp, int* owner, int* neigh, double* fcentre, double* fnormal, double* fe,
                     double* farea, double* fdelta, double* fweight, double* ccentre, double* cvol, int* cf_off,
                     int* cell_faces, int* cell_nsign, int* cell_neigh, int* bcell, int* patch_start,
                     int* patch_count) {
    Mesh* m = (Mesh*)mp;
    for (int f = 0; f < m->n_faces; ++f) {
        owner[f] = m->owner[f];
        neigh[f] = m->neigh[f];
        fcentre[3 * f] = m->fcentre[f].x;
        fcentre[3 * f + 1] = m->fcentre[f].y;
        fcentre[3 * f + 2] = m->fcentre[f].z;
        fnormal[3 * f] = m->fnormal[f].x;
        fnormal[3 * f + 1] = m->fnormal[f].y;
        fnormal[3 * f + 2] = m->fnormal[f].z;
        fe[3 * f] = m->fe[f].x;
        fe[3 * f + 1] = m->fe[f].y;
        fe[3 * f + 2] = m->fe[f].z;
        farea[f] = m->farea[f];
        fdelta[f] = m->fdelta[f];
        fweight[f] = m->fweight[f];
    }
    for (int c = 0; c < m->n_cells; ++c) {
        ccentre[3 * c] = m->ccentre[c].x;
        ccentre[3 * c + 1] = m->ccentre[c].y;
        ccentre[3 * c + 2] = m->ccentre[c].z;
        cvol[c] = m->cvol[c];
    }
    for (int c = 0; c <= m->n_cells; ++c) cf_off[c] = m->cf_off[c];
    for (size_t k = 0; k < m->cell_faces.size(); ++k) {
        cell_faces[k] = m->cell_faces[k];
        cell_nsign[k] = m->cell_nsign[k];
        cell_neigh[k] = m->cell_neigh[k];
    }
    for (int f = 0; f < m->n_bfaces; ++f) bcell[f] = m->bcell[f];
    for (size_t p = 0; p < m->patch_start.size(); ++p) {
        patch_start[p] = m->patch_start[p];
        patch_count[p] = m->patch_count[p];
    }
}

int orc_construct_periodic(void* mp, int p1, int p2, double tol, int* map1, int* map2, double* dist) {
    return construct_periodic((Mesh*)mp, p1, p2, tol, map1, map2, dist);
}

void* orc_case_create(void* mp, const xcal_config* cfg, char* err, int errlen) {
    try {
        return case_create((Mesh*)mp, cfg);
    } catch (std::exception& e) {
        set_err(err, errlen, e.what());
        return nullptr;
    }
}

void orc_case_free(void* c) { delete (Case*)c; }

long orc_case_nnz(void* cp, int eqn) {
    Case* C = (Case*)cp;
    return (long)(eqn == XCAL_EQN_U ? C->AU.colval.size() : C->Ap.colval.size());
}

void orc_case_pattern(void* cp, int eqn, int* rowptr, int* colval) {
    Case* C = (Case*)cp;
    const CSR& A = eqn == XCAL_EQN_U ? C->AU : C->Ap;
    for (int i = 0; i <= A.n; ++i) rowptr[i] = A.rowptr[i];
    for (size_t k = 0; k < A.colval.size(); ++k) colval[k] = A.colval[k];
}

void orc_case_get_system(void* cp, int eqn, int comp, double* nzval, double* b) {
    Case* C = (Case*)cp;
    if (eqn == XCAL_EQN_U) {
        const CSR& A = comp < 0 ? C->AU0 : C->AU;
        if (nzval) std::memcpy(nzval, A.nzval.data(), A.nzval.size() * sizeof(double));
        if (b) std::memcpy(b, C->bU[comp < 0 ? 0 : comp].data(), C->nC * sizeof(double));
    } else {
        if (nzval) std::memcpy(nzval, C->Ap.nzval.data(), C->Ap.nzval.size() * sizeof(double));
        if (b) std::memcpy(b, C->bp.data(), C->nC * sizeof(double));
    }
}

int orc_case_set_field(void* cp, int field, const double* host, long count) {
    Case* C = (Case*)cp;
    int ncomp, per;
    std::vector<double>* f = field_ptr(C, field, ncomp, per);
    if (!f || count != (long)ncomp * per) return XCAL_ERR_INVALID;
    for (int d = 0; d < ncomp; ++d) std::memcpy(f[d].data(), host + (size_t)d * per, per * sizeof(double));
    return 0;
}

// the state set by orc_case_set_field is complete: the next iteration does
// not redo the run's initial calculations (checkpoint restore)
int orc_case_mark_initialised(void* cp) {
    ((Case*)cp)->initialised = true;
    return 0;
}

int orc_case_get_field(void* cp, int field, double* host, long count) {
    Case* C = (Case*)cp;
    int ncomp, per;
    std::vector<double>* f = field_ptr(C, field, ncomp, per);
    if (!f || count != (long)ncomp * per) return XCAL_ERR_INVALID;
    for (int d = 0; d < ncomp; ++d) std::memcpy(host + (size_t)d * per, f[d].data(), per * sizeof(double));
    return 0;
}

int orc_simple_iterate(void* cp, int n, double* res, int* n_done, int* converged) {
    Case* C = (Case*)cp;
    *converged = 0;
    int k = 0;
    for (; k < n; ++k) {
        bool conv = simple_iteration(*C, res + 4 * k);
        if (conv) {
            *converged = 1;
            ++k;
            break;
        }
    }
    *n_done = k;
    return 0;
}

int orc_piso_step(void* cp, int n, double* res, double* courant) {
    Case* C = (Case*)cp;
    for (int k = 0; k < n; ++k) {
        double co = piso_step(*C, res + 4 * k);
        if (courant) courant[k] = co;
    }
    return 0;
}

void orc_initial_calculations(void* cp) { initial_calculations(*(Case*)cp); }
void orc_discretise(void* cp, int eqn) { o_discretise(*(Case*)cp, eqn); }
void orc_apply_bcs(void* cp, int eqn, int comp) { o_apply_bcs(*(Case*)cp, eqn, comp); }
void orc_relax(void* cp, int comp) { o_relax(*(Case*)cp, comp); }
void orc_set_reference(void* cp) { o_set_reference(*(Case*)cp); }
void orc_update_precond(void* cp, int eqn) { o_update_precond(*(Case*)cp, eqn); }
double orc_solve_system(void* cp, int eqn, int comp, int* iters) {
    return o_solve_system(*(Case*)cp, eqn, comp, iters);
}
void orc_solve_equation(void* cp, int eqn, double* res) {
    Case* C = (Case*)cp;
    if (eqn == XCAL_EQN_U)
        solve_equation_U(*C, res, nullptr);
    else
        res[0] = solve_equation_p(*C, nullptr);
}
void orc_pressure_predictor(void* cp) { pressure_predictor(*(Case*)cp, true); }
void orc_flux_divergence(void* cp) { flux_divergence(*(Case*)cp); }
void orc_prev_from_p(void* cp) {
    Case* C = (Case*)cp;
    C->prev = C->p;
}
void orc_explicit_relaxation_p(void* cp, double a) { explicit_relaxation_p(*(Case*)cp, a); }
void orc_grad_p(void* cp) { o_grad_p(*(Case*)cp); }
void orc_correct(void* cp) { correct(*(Case*)cp); }
void orc_turbulence(void* cp) { turbulence(*(Case*)cp); }
double orc_max_courant(void* cp) { return max_courant(*(Case*)cp); }

double orc_canonical_sum(const double* v, long n) {
    return creduce(n, [&](int64_t i) { return v[i]; });
}

// DILU on an arbitrary CSR (sorted columns, diagonal present)
void orc_dilu(int n, const int* rowptr, const int* colval, const double* nzval, double* D) {
    CSR A;
    A.n = n;
    A.rowptr.assign(rowptr, rowptr + n + 1);
    A.colval.assign(colval, colval + rowptr[n]);
    A.nzval.assign(nzval, nzval + rowptr[n]);
    A.diag.resize(n);
    for (int i = 0; i < n; ++i) A.diag[i] = A.find(i, i);
    std::vector<double> d(n);
    o_dilu(A, d);
    std::memcpy(D, d.data(), n * sizeof(double));
}

void orc_dilu_ldiv(int n, const int* rowptr, const int* colval, const double* nzval, const double* D, double* x,
                   const double* b) {
    CSR A;
    A.n = n;
    A.rowptr.assign(rowptr, rowptr + n + 1);
    A.colval.assign(colval, colval + rowptr[n]);
    A.nzval.assign(nzval, nzval + rowptr[n]);
    A.diag.resize(n);
    for (int i = 0; i < n; ++i) A.diag[i] = A.find(i, i);
    std::vector<double> dv(D, D + n), xv(n), bv(b, b + n);
    o_dilu_ldiv(A, dv, xv, bv);
    std::memcpy(x, xv.data(), n * sizeof(double));
}

// the Jacobi smoother on an arbitrary CSR (sorted columns, diagonal present)
void orc_jacobi_smooth(int n, const int* rowptr, const int* colval, const double* nzval, const double* b, double* x,
                       int loops, double omega) {
    CSR A;
    A.n = n;
    A.rowptr.assign(rowptr, rowptr + n + 1);
    A.colval.assign(colval, colval + rowptr[n]);
    A.nzval.assign(nzval, nzval + rowptr[n]);
    A.diag.resize(n);
    for (int i = 0; i < n; ++i) A.diag[i] = A.find(i, i);
    jacobi_smooth(A, b, x, loops, omega);
}

}  // extern "C"

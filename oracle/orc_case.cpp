// orc_case.cpp -- oracle restatement of the SIMPLE/PISO hot path.
//
// TEST INFRASTRUCTURE ONLY (see orc_common.hpp).  Every function cites the
// XCALibre.jl source it restates (paths relative to the project root).
#include "orc_internal.hpp"

#include <cstring>
#include <stdexcept>

namespace orc {

// ---------------------------------------------------------------------------
// CSR helpers
// ---------------------------------------------------------------------------
// spindex (src/ModelFramework/ModelFramework_0_types.jl:246-258), 0-based
int CSR::find(int i, int j) const {
    for (int k = rowptr[i]; k < rowptr[i + 1]; ++k)
        if (colval[k] == j) return k;
    return -1;
}

// sparse_matrix_connectivity (ModelFramework_0_types.jl:223-243) + periodic
// extend_matrix (periodic.jl:219-254) + sparsecsr (sorted rows, merged
// duplicates, explicit zeros kept).
static void build_pattern(const Mesh& m, const std::vector<BC>& bcs, CSR& A) {
    int n = m.n_cells;
    std::vector<std::vector<int>> rows(n);
    for (int c = 0; c < n; ++c) {
        rows[c].push_back(c);
        for (int k = m.cf_off[c]; k < m.cf_off[c + 1]; ++k) rows[c].push_back(m.cell_neigh[k]);
    }
    for (const BC& bc : bcs) {
        if (bc.type != XCAL_BC_PERIODIC_PARENT) continue;
        for (int i = 0; i < bc.count; ++i) {
            int f1 = bc.start + i, f2 = bc.face_map[i];
            int c1 = m.owner[f1], c2 = m.owner[f2];
            rows[c1].push_back(c2);
            rows[c2].push_back(c1);
        }
    }
    A.n = n;
    A.rowptr.assign(n + 1, 0);
    A.colval.clear();
    for (int c = 0; c < n; ++c) {
        std::sort(rows[c].begin(), rows[c].end());
        rows[c].erase(std::unique(rows[c].begin(), rows[c].end()), rows[c].end());
        for (int j : rows[c]) A.colval.push_back(j);
        A.rowptr[c + 1] = (int)A.colval.size();
    }
    A.nzval.assign(A.colval.size(), 0.0);
    A.diag.resize(n);
    for (int c = 0; c < n; ++c) A.diag[c] = A.find(c, c);
}

static void spmv(const CSR& A, const std::vector<double>& x, std::vector<double>& y) {
    // xmul! (src/Multithread/spmvm.jl:35-59): sequential per row from 0
#pragma omp parallel for schedule(static)
    for (int i = 0; i < A.n; ++i) {
        double acc = 0.0;
        for (int k = A.rowptr[i]; k < A.rowptr[i + 1]; ++k) acc = acc + A.nzval[k] * x[A.colval[k]];
        y[i] = acc;
    }
}

// dot product summed in the canonical tree over the rows in order `ord`
static double cdot(const int* ord, const std::vector<double>& a, const std::vector<double>& b) {
    const double* pa = a.data();
    const double* pb = b.data();
    return creduce((int64_t)a.size(), [&](int64_t s) {
        int64_t i = ord ? ord[s] : s;
        return pa[i] * pb[i];
    });
}

// ---------------------------------------------------------------------------
// case construction
// ---------------------------------------------------------------------------
static void copy_bcs(const Mesh& m, const xcal_bc* src, int n, std::vector<BC>& dst, int ncomp) {
    dst.clear();
    for (int b = 0; b < n; ++b) {
        BC bc;
        bc.type = src[b].type;
        bc.patch = src[b].patch;
        if (bc.patch < 0 || bc.patch >= (int)m.patch_start.size()) throw std::runtime_error("bad patch");
        for (int c = 0; c < 3; ++c) bc.value[c] = src[b].value[c];
        bc.start = m.patch_start[bc.patch];
        bc.count = m.patch_count[bc.patch];
        for (int c = 0; c < 5; ++c) bc.wall[c] = src[b].wall[c];
        if (bc.type == XCAL_BC_DIRICHLET_FUNCTION) {
            if (!src[b].face_values) throw std::runtime_error("DirichletFunction without values");
            bc.face_values.assign(src[b].face_values, src[b].face_values + (size_t)ncomp * bc.count);
        }
        if (bc.type == XCAL_BC_PERIODIC || bc.type == XCAL_BC_PERIODIC_PARENT) {
            if (!src[b].face_map) throw std::runtime_error("periodic without face_map");
            bc.face_map.assign(src[b].face_map, src[b].face_map + bc.count);
            bc.distance = {src[b].distance[0], src[b].distance[1], src[b].distance[2]};
            bc.partner_patch = src[b].partner_patch;
        }
        dst.push_back(bc);
    }
}

static void wall_distance(Case& C);

Case* case_create(const Mesh* m, const xcal_config* cfg) {
    Case* C = new Case();
    C->m = m;
    C->cfg = *cfg;
    C->nC = m->n_cells;
    C->nF = m->n_faces;
    C->nB = m->n_bfaces;
    copy_bcs(*m, cfg->bc_U, cfg->n_bc_U, C->bcU, 3);
    copy_bcs(*m, cfg->bc_p, cfg->n_bc_p, C->bcP, 1);
    copy_bcs(*m, cfg->bc_nut, cfg->n_bc_nut, C->bcNut, 1);
    C->cfg.bc_U = C->cfg.bc_p = C->cfg.bc_nut = nullptr;
    const bool lke = cfg->turbulence == XCAL_TURB_KOMEGA_LKE;
    const bool has_y = cfg->turbulence == XCAL_TURB_KOMEGA_SST || lke;
    if (cfg->turbulence == XCAL_TURB_KOMEGA || cfg->turbulence == XCAL_TURB_KOMEGA_SST || lke) {
        copy_bcs(*m, cfg->bc_k, cfg->n_bc_k, C->bcK, 1);
        copy_bcs(*m, cfg->bc_omega, cfg->n_bc_omega, C->bcOmega, 1);
    }
    if (cfg->turbulence == XCAL_TURB_KEQUATION) copy_bcs(*m, cfg->bc_k, cfg->n_bc_k, C->bcK, 1);
    if (has_y) copy_bcs(*m, cfg->bc_y, cfg->n_bc_y, C->bcY, 1);
    if (lke) copy_bcs(*m, cfg->bc_kl, cfg->n_bc_kl, C->bcKl, 1);
    C->cfg.bc_k = C->cfg.bc_omega = C->cfg.bc_y = C->cfg.bc_kl = nullptr;
    int nC = C->nC, nF = C->nF;
    for (int d = 0; d < 3; ++d) {
        C->U[d].assign(nC, 0.0);
        C->gradp[d].assign(nC, 0.0);
        C->Hv[d].assign(nC, 0.0);
        C->Uf[d].assign(nF, 0.0);
        C->bU[d].assign(nC, 0.0);
    }
    for (int d = 0; d < 9; ++d) C->gradU[d].assign(nC, 0.0);
    C->p.assign(nC, 0.0);
    C->mdotf.assign(nF, 0.0);
    C->nueff.assign(nF, 0.0);
    C->rD.assign(nC, 0.0);
    C->divHv.assign(nC, 0.0);
    C->nut.assign(nC, 0.0);
    C->nutf.assign(nF, 0.0);
    C->pf.assign(nF, 0.0);
    C->rDf.assign(nF, 1.0);  // initialise!(rDf, 1.0) (Solvers_1_SIMPLE.jl:61)
    C->Delta.assign(nC, 0.0);
    for (std::vector<double>* v : {&C->k, &C->omega, &C->Pk, &C->Pw, &C->Dk, &C->Dw, &C->Pkw}) v->assign(nC, 0.0);
    C->mueffk.assign(nF, 0.0);
    C->mueffw.assign(nF, 0.0);
    if (lke) {
        for (std::vector<double>* v : {&C->kl, &C->PkL, &C->DkL, &C->S2, &C->normU, &C->divU, &C->ReL, &C->gam,
                                       &C->nueffS, &C->Pkl})
            v->assign(nC, 0.0);
        C->mueffl.assign(nF, 0.0);
        // eta = 0.02974 tanh(59.79 Tu^1.191 + 1.65e-13) (RANS_kOmegaLKE.jl:97)
        C->lke_eta = 0.02974 * det_tanh_pos(59.79 * det_pow(cfg->lke_Tu, 1.191) + 1.65e-13);
    }
    if (has_y) {
        for (std::vector<double>* v : {&C->yw, &C->F1, &C->F2, &C->Om, &C->D2, &C->Pww}) v->assign(nC, 0.0);
        for (int d = 0; d < 3; ++d) {
            C->gk[d].assign(nC, 0.0);
            C->gw[d].assign(nC, 0.0);
        }
        C->kfs.assign(nF, 0.0);
        C->wfs.assign(nF, 0.0);
    }
    C->prev.assign(nC, 0.0);
    C->cellsCourant.assign(nC, 0.0);
    C->bp.assign(nC, 0.0);
    build_pattern(*m, C->bcU, C->AU);
    build_pattern(*m, C->bcP, C->Ap);
    C->rorder = morton_order(m->ccentre);
    C->AU.ord = C->rorder.data();
    C->Ap.ord = C->rorder.data();
    C->AU0 = C->AU;
    C->PU.assign(nC, 0.0);
    C->Pp.assign(nC, 0.0);
    // LES{Smagorinsky} initialise (LES_Smagorinsky.jl:84-101, LES_functions.jl:1-55);
    // LES{KEquation} initialise (LES_KEquation.jl:85-94): delta! alone
    const bool keq = cfg->turbulence == XCAL_TURB_KEQUATION;
    if (cfg->turbulence == XCAL_TURB_SMAGORINSKY || keq) {
        double distance = 1.0, power = 1.0 / 3.0;
        if (cfg->les_delta_power > 0.0) {  // delta_scaling evaluated by the caller
            distance = cfg->les_delta_distance;
            power = cfg->les_delta_power;
        } else
        for (const BC& bc : C->bcU)
            if (bc.type == XCAL_BC_EMPTY) {
                // 2D slab: distance between the Empty patches (delta_scaling,
                // Mesh3): the box of the boundary faces' nodes when the mesh
                // has them, else of the boundary-face centres
                V3 pmin{0, 0, 0}, pmax{0, 0, 0};
                const bool nodes = !m->fn_off.empty();
                for (int f = 0; f < C->nB; ++f) {
                    const int k0 = nodes ? m->fn_off[f] : 0, k1 = nodes ? m->fn_off[f + 1] : 1;
                    for (int k = k0; k < k1; ++k) {
                        V3 c = nodes ? m->points[m->face_nodes[k]] : m->fcentre[f];
                        pmin = {std::min(pmin.x, c.x), std::min(pmin.y, c.y), std::min(pmin.z, c.z)};
                        pmax = {std::max(pmax.x, c.x), std::max(pmax.y, c.y), std::max(pmax.z, c.z)};
                    }
                }
                V3 n = m->fnormal[bc.start];
                distance = std::fabs(dot(pmin, n)) + std::fabs(dot(pmax, n));
                power = 0.5;
                break;
            }
        for (int i = 0; i < nC; ++i) {
            double d = std::pow(m->cvol[i] / distance, power);
            double dc = d * cfg->smagorinsky_C;
            C->Delta[i] = keq ? d : dc * dc;
        }
    }
    if (has_y) wall_distance(*C);  // initialise (RANS_kOmegaSST.jl:167, RANS_kOmegaLKE.jl:236)
    return C;
}

// ---------------------------------------------------------------------------
// discretisation
// ---------------------------------------------------------------------------
enum TermKind { T_TIME, T_DIV, T_LAP, T_SI };
struct Term {
    TermKind kind;
    double sign;
    const std::vector<double>* flux;  // face flux (Div: mdotf, Lap: nueff/rDf); Si: cell coefficient
    int scheme;                       // time or divergence scheme
};

// terms of U_eqn: Time(U) + Divergence(mdotf,U) - Laplacian(nueff,U) == -Source(grad p)
// (Solvers_1_SIMPLE.jl:68-74)
static std::vector<Term> u_terms(Case& C) {
    return {{T_TIME, 1.0, nullptr, C.cfg.U_schemes.time},
            {T_DIV, 1.0, &C.mdotf, C.cfg.U_schemes.divergence},
            {T_LAP, -1.0, &C.nueff, 0}};
}
// p_eqn: -Laplacian(rDf, p) == -Source(divHv) (Solvers_1_SIMPLE.jl:76-78)
static std::vector<Term> p_terms(Case& C) { return {{T_LAP, -1.0, &C.rDf, 0}}; }

// scheme! (src/Discretise/Discretise_1_schemes.jl)
static void scheme(const Mesh& m, const Term& t, int fID, int ns, double& ac, double& an) {
    if (t.kind == T_TIME || t.kind == T_SI) {  // :12-23, :26-34, Si :204-210
        ac = 0.0;
        an = 0.0;
        return;
    }
    double dns = (double)ns;
    double flux = (*t.flux)[fID];
    if (t.kind == T_LAP) {  // Laplacian{Linear} :68-110
        V3 Sf = (dns * m.farea[fID]) * m.fnormal[fID];
        V3 e = dns * m.fe[fID];
        V3 Ef = (dot(Sf, Sf) / dot(Sf, e)) * e;
        double Ef_mag = norm(Ef);
        double ap = (t.sign * (flux * Ef_mag)) / m.fdelta[fID];
        ac = -ap;
        an = ap;
        return;
    }
    double ap = t.sign * (flux * dns);
    if (t.scheme == XCAL_DIV_LINEAR) {  // :114-134
        double w = m.fweight[fID];
        w = 0.5 + dns * (w - 0.5);
        ac = ap * w;
        an = ap * (1.0 - w);
    } else if (t.scheme == XCAL_DIV_UPWIND) {  // :137-152
        ac = jl_max(ap, 0.0);
        an = -jl_max(-ap, 0.0);
    } else {  // LUST :155-180
        double w = m.fweight[fID];
        if (ns < 0) w = 1.0 - w;
        double acL = ap * w, anL = ap * (1.0 - w);
        double acU = jl_max(ap, 0.0), anU = -jl_max(-ap, 0.0);
        ac = 0.75 * acL + 0.25 * acU;
        an = 0.75 * anL + 0.25 * anU;
    }
}

// scheme_source! for Time{Euler} (:36-45); zero for every other term
static void scheme_source(const Case& C, const Term& t, int c, double prev, double& ac, double& b) {
    if (t.kind == T_TIME && t.scheme == XCAL_TIME_EULER) {
        double vol_rdt = (1.0 * C.m->cvol[c]) / C.cfg.dt;
        ac = vol_rdt;
        b = prev * vol_rdt;
    } else if (t.kind == T_SI) {  // Si (:211-218): sign * flux[c] * volume
        ac = (t.sign * (*t.flux)[c]) * C.m->cvol[c];
        b = 0.0;
    } else {
        ac = 0.0;
        b = 0.0;
    }
}

// _discretise_vector_model! (Discretise_2_generated_distretisation.jl:39-87)
static void discretise_U(Case& C) {
    const Mesh& m = *C.m;
    std::vector<Term> terms = u_terms(C);
    CSR& A0 = C.AU0;
    std::fill(A0.nzval.begin(), A0.nzval.end(), 0.0);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < C.nC; ++i) {
        double ac_sum = 0.0;
        for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
            int fID = m.cell_faces[k], ns = m.cell_nsign[k], nID = m.cell_neigh[k];
            int nIndex = A0.find(i, nID);
            double AC = 0.0, AN = 0.0;
            for (const Term& t : terms) {
                double ac, an;
                scheme(m, t, fID, ns, ac, an);
                AC = AC + ac;
                AN = AN + an;
            }
            ac_sum = ac_sum + AC;
            A0.nzval[nIndex] = AN;
        }
        double AC = 0.0, BX = 0.0, BY = 0.0, BZ = 0.0;
        for (const Term& t : terms) {
            double ac, bx, by, bz;
            scheme_source(C, t, i, C.U[0][i], ac, bx);
            scheme_source(C, t, i, C.U[1][i], ac, by);
            scheme_source(C, t, i, C.U[2][i], ac, bz);
            AC = AC + ac;
            BX = BX + bx;
            BY = BY + by;
            BZ = BZ + bz;
        }
        A0.nzval[A0.diag[i]] = ac_sum + AC;
        // _sources!: -Source(grad p): Bx += sign*field.x*volume
        double V = m.cvol[i];
        double Bx = 0.0 + (-1.0 * C.gradp[0][i]) * V;
        double By = 0.0 + (-1.0 * C.gradp[1][i]) * V;
        double Bz = 0.0 + (-1.0 * C.gradp[2][i]) * V;
        C.bU[0][i] = BX + Bx;
        C.bU[1][i] = BY + By;
        C.bU[2][i] = BZ + Bz;
    }
}

// _discretise_scalar_model! (:125-167)
static void discretise_p(Case& C) {
    const Mesh& m = *C.m;
    std::vector<Term> terms = p_terms(C);
    CSR& A = C.Ap;
    std::fill(A.nzval.begin(), A.nzval.end(), 0.0);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < C.nC; ++i) {
        double ac_sum = 0.0;
        for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
            int fID = m.cell_faces[k], ns = m.cell_nsign[k], nID = m.cell_neigh[k];
            int nIndex = A.find(i, nID);
            double AC = 0.0, AN = 0.0;
            for (const Term& t : terms) {
                double ac, an;
                scheme(m, t, fID, ns, ac, an);
                AC = AC + ac;
                AN = AN + an;
            }
            ac_sum = ac_sum + AC;
            A.nzval[nIndex] = AN;
        }
        double AC = 0.0, B = 0.0;
        for (const Term& t : terms) {
            double ac, b;
            scheme_source(C, t, i, 0.0, ac, b);
            AC = AC + ac;
            B = B + b;
        }
        A.nzval[A.diag[i]] = ac_sum + AC;
        double b2 = 0.0 + (-1.0 * C.divHv[i]) * m.cvol[i];
        C.bp[i] = b2 + B;
    }
}

// ---------------------------------------------------------------------------
// boundary conditions (Discretise_5_apply_bcs.jl + boundary_conditions/*.jl)
// ---------------------------------------------------------------------------
static const BC* find_bc(const std::vector<BC>& bcs, int f) {
    for (const BC& bc : bcs)
        if (f >= bc.start && f < bc.start + bc.count) return &bc;
    return nullptr;
}

struct BCCtx {
    Case* C;
    CSR* A;
    bool vector;
    int comp;                     // component (vector fields)
    const std::vector<double>* phi;  // component values / scalar values
};

static double bc_value(const BC& bc, bool vector, int comp, int i) {
    if (bc.type == XCAL_BC_DIRICHLET_FUNCTION) return vector ? bc.face_values[3 * i + comp] : bc.face_values[i];
    return vector ? bc.value[comp] : bc.value[0];
}

// one BC functor call: returns (ap, bp); periodic parents also update A
static void bc_functor(BCCtx& X, const BC& bc, const Term& t, int f, double& ap, double& bp) {
    Case& C = *X.C;
    const Mesh& m = *C.m;
    int i = f - bc.start;
    int cell = m.bcell[f];
    ap = 0.0;
    bp = 0.0;
    if (t.kind == T_TIME || t.kind == T_SI) return;  // Discretise_3_boundary_conditions.jl:2-9; Si: (0, 0)
    double flux = (*t.flux)[f];
    switch (bc.type) {
        case XCAL_BC_DIRICHLET:
        case XCAL_BC_DIRICHLET_FUNCTION: {  // dirichlet.jl, dirichletFunction.jl
            double val = bc_value(bc, X.vector, X.comp, i);
            if (t.kind == T_LAP) {
                double fl = (flux * m.farea[f]) / m.fdelta[f];
                double a = t.sign * (-fl);
                ap = a;
                bp = a * val;
            } else {
                double fl = -flux;
                double a = t.sign * fl;
                ap = 0.0;
                bp = a * val;
            }
            return;
        }
        case XCAL_BC_WALL: {  // wall.jl
            if (t.kind == T_LAP) {
                if (!X.vector) return;
                double fl = (flux * m.farea[f]) / m.fdelta[f];
                double a = t.sign * (-fl);
                V3 n = m.fnormal[f];
                V3 vb{bc.value[0], bc.value[1], bc.value[2]};
                V3 vc{C.U[0][cell], C.U[1][cell], C.U[2][cell]};
                V3 vc_n = dot(vc, n) * n;
                V3 vb_n = dot(vb, n) * n;
                V3 vb_p = vb - vb_n;
                ap = a;
                bp = a * (comp(vb_p, X.comp) + comp(vc_n, X.comp));
            } else {
                if (X.vector) return;
                ap = t.sign * flux;
            }
            return;
        }
        case XCAL_BC_ZEROGRADIENT:  // zerogradient.jl
        case XCAL_BC_K_WALL:        // Discretise_3_boundary_conditions.jl:12-51 (Laplacian (0, 0))
        case XCAL_BC_NUT_WALL:
            if (t.kind == T_DIV) ap = t.sign * flux;
            return;
        case XCAL_BC_OMEGA_WALL:    // Discretise_3_boundary_conditions.jl:28-61 (as Extrapolated)
        case XCAL_BC_EXTRAPOLATED:  // extrapolated.jl
            if (t.kind == T_LAP) {
                double fl = ((-flux) * m.farea[f]) / m.fdelta[f];
                double a = t.sign * fl;
                ap = a;
                bp = a * (*X.phi)[cell];
            } else {
                ap = t.sign * flux;
            }
            return;
        case XCAL_BC_EMPTY:
        case XCAL_BC_PERIODIC:
            return;
        case XCAL_BC_SYMMETRY: {  // symmetry.jl
            if (t.kind == T_LAP) {
                if (!X.vector) return;
                double fl = (flux * m.farea[f]) / m.fdelta[f];
                double a = t.sign * (-fl);
                V3 n = m.fnormal[f];
                V3 vc{C.U[0][cell], C.U[1][cell], C.U[2][cell]};
                V3 vn = dot(vc, n) * n;
                V3 vp = vc - vn;
                ap = a;
                bp = a * comp(vp, X.comp);
            } else {
                double a = t.sign * flux;
                if (!X.vector) {
                    ap = a;
                    return;
                }
                V3 n = m.fnormal[f];
                V3 vc{C.U[0][cell], C.U[1][cell], C.U[2][cell]};
                V3 vn = dot(vc, n) * n;
                ap = a;
                bp = a * comp(vn, X.comp);
            }
            return;
        }
        case XCAL_BC_NEUMANN: {  // neumann.jl (scalar)
            if (t.kind == T_LAP) {
                double fl = flux * m.farea[f];
                ap = 0.0;
                bp = fl * bc.value[0];
            } else {
                double a = t.sign * flux;
                ap = a;
                bp = ((-bc.value[0]) * a) * m.fdelta[f];
            }
            return;
        }
        case XCAL_BC_PERIODIC_PARENT: {  // periodic.jl:261-443
            CSR& A = *X.A;
            int pfID = bc.face_map[i];
            int pcell = m.owner[pfID];
            int NN = A.find(pcell, pcell), NP = A.find(pcell, cell), PN = A.find(cell, pcell);
            if (t.kind == T_LAP) {
                V3 C1 = m.ccentre[cell];
                V3 C2 = m.ccentre[pcell] - bc.distance;
                V3 d = C2 - C1;
                double Delta = norm(d);
                V3 Sf = m.farea[f] * m.fnormal[f];
                V3 e = m.fe[f];
                V3 Ef = (dot(Sf, Sf) / dot(Sf, e)) * e;
                double Ef_mag = norm(Ef);
                double gamma = ((-t.sign) * (flux * Ef_mag)) / Delta;
                A.nzval[NN] = A.nzval[NN] + gamma;
                A.nzval[NP] = A.nzval[NP] + (-gamma);
                A.nzval[PN] = A.nzval[PN] + (-gamma);
                ap = gamma;
                return;
            }
            if (t.scheme == XCAL_DIV_UPWIND) {
                double mdot = t.sign * flux;
                double a = jl_max(mdot, 0.0), an = -jl_max(-mdot, 0.0);
                A.nzval[NN] = A.nzval[NN] + (-an);
                A.nzval[NP] = A.nzval[NP] + (-a);
                A.nzval[PN] = A.nzval[PN] + an;
                ap = a;
                return;
            }
            V3 C1 = m.ccentre[cell];
            V3 C2 = m.ccentre[pcell] - bc.distance;
            V3 Cf = m.fcentre[f], n = m.fnormal[f];
            V3 Pf = Cf - C1, PNv = C2 - C1;
            double wn = dot(Pf, n) / dot(PNv, n);
            double w = 1.0 - wn;
            double ac, an;
            if (t.scheme == XCAL_DIV_LINEAR) {
                double a = t.sign * flux;
                ac = a * w;
                an = a * wn;
            } else {  // LUST
                double mdot = t.sign * flux;
                double acL = mdot * w, anL = mdot * wn;
                double acU = jl_max(mdot, 0.0), anU = -jl_max(-mdot, 0.0);
                ac = 0.75 * acL + 0.25 * acU;
                an = 0.75 * anL + 0.25 * anU;
            }
            A.nzval[NN] = A.nzval[NN] + (-an);
            A.nzval[NP] = A.nzval[NP] + (-ac);
            A.nzval[PN] = A.nzval[PN] + an;
            ap = ac;
            return;
        }
        default:
            return;
    }
}

// apply_boundary_conditions! in boundary-face order (the reference's atomics
// are applied here in ascending face id order)
static void apply_bcs(Case& C, bool vector, int comp) {
    const Mesh& m = *C.m;
    std::vector<Term> terms = vector ? u_terms(C) : p_terms(C);
    CSR& A = vector ? C.AU : C.Ap;
    std::vector<double>& b = vector ? C.bU[comp] : C.bp;
    const std::vector<BC>& bcs = vector ? C.bcU : C.bcP;
    BCCtx X{&C, &A, vector, comp, vector ? &C.U[comp] : &C.p};
    for (int f = 0; f < C.nB; ++f) {
        const BC* bc = find_bc(bcs, f);
        if (!bc) continue;
        int cell = m.bcell[f];
        double AP = 0.0, BP = 0.0;
        for (const Term& t : terms) {
            double ap, bp;
            bc_functor(X, *bc, t, f, ap, bp);
            AP = AP + ap;
            BP = BP + bp;
        }
        A.nzval[A.diag[cell]] = A.nzval[A.diag[cell]] + AP;
        b[cell] = b[cell] + BP;
    }
}

// update_equation! (:305-330) A <- A0
static void update_equation(Case& C) { C.AU.nzval = C.AU0.nzval; }

// implicit_relaxation_diagdom! (src/Solve/Solve_1_api.jl:388-411)
static void relax_diagdom(Case& C, int comp) {
    CSR& A = C.AU;
    std::vector<double>& b = C.bU[comp];
    const std::vector<double>& field = C.U[comp];
    double alpha = C.cfg.U_solver.relax;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < A.n; ++i) {
        int c = A.diag[i];
        double sumv = 0.0;
        for (int k = A.rowptr[i]; k < A.rowptr[i + 1]; ++k) sumv = sumv + std::fabs(A.nzval[k]);
        sumv = sumv - std::fabs(A.nzval[c]);
        double D0 = A.nzval[c];
        double D_max = jl_max(std::fabs(D0), sumv) / alpha;
        A.nzval[c] = D_max;
        b[i] = b[i] + (D_max - D0) * field[i];
    }
}

// setReference! (Solve_1_api.jl:414-439), cellID = 1
static void set_reference(Case& C) {
    if (!C.cfg.has_pref) return;
    CSR& A = C.Ap;
    int c = A.diag[0];
    C.bp[0] = A.nzval[c] * C.cfg.pref;
    A.nzval[c] = A.nzval[c] + A.nzval[c];
}

// update_preconditioner! (preconditioners_2_functions.jl:65-108; DILU
// preconditioners_1_DILU.jl:43-82)
static void update_precond(const CSR& A, int type, std::vector<double>& P) {
    if (type == XCAL_PRECOND_JACOBI) {
        for (int i = 0; i < A.n; ++i) {
            double d = std::fabs(A.nzval[A.diag[i]]);
            P[i] = 1.0 / d;
        }
    } else if (type == XCAL_PRECOND_DILU) {
        for (int i = 0; i < A.n; ++i) P[i] = A.nzval[A.diag[i]];
        for (int i = 0; i < A.n; ++i) {
            for (int k = A.rowptr[i]; k < A.rowptr[i + 1]; ++k) {
                int j = A.colval[k];
                if (j > i) {
                    int k2 = A.find(j, i);
                    if (k2 >= 0) P[j] = P[j] - (A.nzval[k] * A.nzval[k2]) / P[i];
                }
            }
        }
    }
}

// forward/backward_substitution! (preconditioners_1_DILU.jl:84-120)
static void dilu_ldiv(const CSR& A, const std::vector<double>& D, std::vector<double>& x,
                      const std::vector<double>& b) {
    int n = A.n;
    for (int i = 0; i < n; ++i) {
        double sum = 0.0;
        for (int k = A.rowptr[i]; k < A.diag[i]; ++k) {
            int j = A.colval[k];
            sum = sum + (A.nzval[k] * x[j]) * (1.0 / D[j]);
        }
        x[i] = b[i] - sum;
    }
    for (int i = n - 1; i >= 0; --i) {
        double sum = 0.0;
        for (int k = A.diag[i] + 1; k < A.rowptr[i + 1]; ++k) sum = sum + A.nzval[k] * x[A.colval[k]];
        x[i] = (x[i] - sum) / D[i];
    }
}

static void apply_M(const CSR& A, int type, const std::vector<double>& P, std::vector<double>& out,
                    const std::vector<double>& in) {
    if (type == XCAL_PRECOND_JACOBI) {
        for (int i = 0; i < A.n; ++i) out[i] = P[i] * in[i];
    } else if (type == XCAL_PRECOND_DILU) {
        dilu_ldiv(A, P, out, in);
    } else {
        out = in;
    }
}

// ---------------------------------------------------------------------------
// Krylov.jl 0.10 restatements (warm start x0 = field values)
// ---------------------------------------------------------------------------
// CG (Hestenes-Stiefel) as in Krylov.jl cg!: x0 = 0 plus warm-start shift
static int krylov_cg(const CSR& A, const std::vector<double>& b, std::vector<double>& field, int ptype,
                     const std::vector<double>& P, const xcal_solver_setup& S, Krylov& K) {
    int n = A.n;
    K.dx = field;
    K.x.assign(n, 0.0);
    K.r.assign(n, 0.0);
    K.p.assign(n, 0.0);
    K.q.assign(n, 0.0);
    K.z.assign(n, 0.0);
    spmv(A, K.dx, K.r);
    for (int i = 0; i < n; ++i) K.r[i] = b[i] - K.r[i];
    bool MisI = ptype == XCAL_PRECOND_NONE;
    std::vector<double>& z = MisI ? K.r : K.z;
    if (!MisI) apply_M(A, ptype, P, z, K.r);
    K.p = z;
    double gamma = cdot(A.ord, K.r, z);
    double rNorm = std::sqrt(gamma);
    int iter = 0;
    if (gamma == 0.0) {
        for (int i = 0; i < n; ++i) K.x[i] = K.x[i] + K.dx[i];
        field = K.x;
        K.niter = 0;
        return 0;
    }
    int itmax = S.itmax == 0 ? 2 * n : S.itmax;
    double pNorm2 = gamma;
    double eps_ = S.atol + S.rtol * rNorm;
    const double epsT = std::numeric_limits<double>::epsilon();
    bool solved = rNorm <= eps_, tired = iter >= itmax, zero_curv = false;
    while (!(solved || tired || zero_curv)) {
        spmv(A, K.p, K.q);
        double pAp = cdot(A.ord, K.p, K.q);
        if (pAp <= epsT * pNorm2) {
            if (std::fabs(pAp) <= epsT * pNorm2) zero_curv = true;
        }
        if (zero_curv) continue;
        double alpha = gamma / pAp;
        for (int i = 0; i < n; ++i) K.x[i] = K.x[i] + alpha * K.p[i];
        for (int i = 0; i < n; ++i) K.r[i] = K.r[i] + (-alpha) * K.q[i];
        if (!MisI) apply_M(A, ptype, P, z, K.r);
        double gamma_next = cdot(A.ord, K.r, z);
        rNorm = std::sqrt(gamma_next);
        bool mach = (rNorm + 1.0 <= 1.0);
        solved = (rNorm <= eps_) || mach;
        if (!solved) {
            double beta = gamma_next / gamma;
            pNorm2 = gamma_next + (beta * beta) * pNorm2;
            gamma = gamma_next;
            for (int i = 0; i < n; ++i) K.p[i] = z[i] + beta * K.p[i];
        }
        iter = iter + 1;
        tired = iter >= itmax;
    }
    for (int i = 0; i < n; ++i) K.x[i] = K.x[i] + K.dx[i];
    field = K.x;
    K.niter = iter;
    return iter;
}

// BiCGSTAB (van der Vorst) as in Krylov.jl bicgstab! with left preconditioner
// M, c = b (shadow residual), warm start.
static int krylov_bicgstab(const CSR& A, const std::vector<double>& b, std::vector<double>& field, int ptype,
                           const std::vector<double>& P, const xcal_solver_setup& S, Krylov& K) {
    int n = A.n;
    bool MisI = ptype == XCAL_PRECOND_NONE;
    K.dx = field;
    K.x.assign(n, 0.0);
    K.s.assign(n, 0.0);
    K.v.assign(n, 0.0);
    K.r.assign(n, 0.0);
    K.q.assign(n, 0.0);
    K.t.assign(n, 0.0);
    std::vector<double> r0(n);
    spmv(A, K.dx, r0);
    for (int i = 0; i < n; ++i) r0[i] = b[i] - r0[i];
    if (!MisI)
        apply_M(A, ptype, P, K.r, r0);
    else
        K.r = r0;
    K.p = K.r;
    const std::vector<double>& c = b;
    double rNorm = std::sqrt(cdot(A.ord, K.r, K.r));
    int iter = 0;
    if (rNorm == 0.0) {
        for (int i = 0; i < n; ++i) K.x[i] = K.x[i] + K.dx[i];
        field = K.x;
        K.niter = 0;
        return 0;
    }
    int itmax = S.itmax == 0 ? 2 * n : S.itmax;
    double eps_ = S.atol + S.rtol * rNorm;
    double next_rho = cdot(A.ord, c,K.r);
    if (next_rho == 0.0) {
        for (int i = 0; i < n; ++i) K.x[i] = K.x[i] + K.dx[i];
        field = K.x;
        K.niter = 0;
        return 0;
    }
    bool solved = rNorm <= eps_, tired = iter >= itmax, breakdown = false;
    std::vector<double> d(n);
    while (!(solved || tired || breakdown)) {
        iter = iter + 1;
        double rho = next_rho;
        spmv(A, K.p, K.q);  // q = A y, y = p
        if (!MisI)
            apply_M(A, ptype, P, K.v, K.q);
        else
            K.v = K.q;
        double alpha = rho / cdot(A.ord, c,K.v);
        for (int i = 0; i < n; ++i) K.s[i] = K.r[i] + (-alpha) * K.v[i];
        for (int i = 0; i < n; ++i) K.x[i] = K.x[i] + alpha * K.p[i];
        spmv(A, K.s, d);  // d = A z, z = s
        if (!MisI)
            apply_M(A, ptype, P, K.t, d);
        else
            K.t = d;
        std::vector<double>& tt = K.t;
        double omega = cdot(A.ord, tt,K.s) / cdot(A.ord, tt,tt);
        for (int i = 0; i < n; ++i) K.x[i] = K.x[i] + omega * K.s[i];
        for (int i = 0; i < n; ++i) K.r[i] = K.s[i] + (-omega) * tt[i];
        next_rho = cdot(A.ord, c,K.r);
        double beta = (next_rho / rho) * (alpha / omega);
        for (int i = 0; i < n; ++i) K.p[i] = K.r[i] + beta * (K.p[i] + (-omega) * K.v[i]);
        rNorm = std::sqrt(cdot(A.ord, K.r, K.r));
        bool mach = (rNorm + 1.0 <= 1.0);
        solved = (rNorm <= eps_) || mach;
        tired = iter >= itmax;
        breakdown = (alpha == 0.0) || std::isnan(alpha);
    }
    for (int i = 0; i < n; ++i) K.x[i] = K.x[i] + K.dx[i];
    field = K.x;
    K.niter = iter;
    return iter;
}

// residual (Solve_1_api.jl:441-464)
static double residual(const CSR& A, const std::vector<double>& b, const std::vector<double>& x) {
    std::vector<double> Fx(A.n);
    spmv(A, x, Fx);
    const double* pb = b.data();
    const double* pf = Fx.data();
    const int* ord = A.ord;
    double sR = creduce(A.n, [&](int64_t s) {
        int64_t i = ord ? ord[s] : s;
        double d = pb[i] - pf[i];
        return d * d;
    });
    double normb = std::sqrt(creduce(A.n, [&](int64_t s) {
        int64_t i = ord ? ord[s] : s;
        return pb[i] * pb[i];
    }));
    double denom = normb > jl_eps(normb) ? normb : 1.0;
    return std::sqrt(sR) / denom;
}

// apply_smoother!(JacobiSmoother) (Smoothers_jacobi.jl:73-86, multiply_row
// :112-131): `loops` sweeps; per row the sum over the row from 0, less
// a_ii x_i, then omega (1/a_ii) (b_i - sum) + (1 - omega) x_i into a scratch
// vector, copied back after each sweep
void jacobi_smooth(const CSR& A, const double* b, double* x, int loops, double omega) {
    std::vector<double> xt(A.n);
    for (int l = 0; l < loops; ++l) {
#pragma omp parallel for schedule(static)
        for (int i = 0; i < A.n; ++i) {
            double sum = 0.0;
            for (int k = A.rowptr[i]; k < A.rowptr[i + 1]; ++k) sum = sum + A.nzval[k] * x[A.colval[k]];
            const double a_ii = A.nzval[A.diag[i]];
            const double xi = x[i];
            sum = sum - a_ii * xi;
            const double rD = 1.0 / a_ii;
            xt[i] = omega * rD * (b[i] - sum) + (1.0 - omega) * xi;
        }
        std::copy(xt.begin(), xt.end(), x);
    }
}

// solve_system! (Solve_1_api.jl:268-307)
static double solve_system(Case& C, bool vector, int comp, int* iters) {
    const xcal_solver_setup& S = vector ? C.cfg.U_solver : C.cfg.p_solver;
    CSR& A = vector ? C.AU : C.Ap;
    std::vector<double>& b = vector ? C.bU[comp] : C.bp;
    std::vector<double>& field = vector ? C.U[comp] : C.p;
    if (S.smoother_loops > 0) jacobi_smooth(A, b.data(), field.data(), S.smoother_loops, S.smoother_omega);
    std::vector<double>& P = vector ? C.PU : C.Pp;
    Krylov& K = vector ? C.kU : C.kp;
    int it = S.solver == XCAL_SOLVER_CG ? krylov_cg(A, b, field, S.precond, P, S, K)
                                        : krylov_bicgstab(A, b, field, S.precond, P, S, K);
    if (iters) *iters = it;
    return residual(A, b, field);
}

// ---------------------------------------------------------------------------
// calculus: interpolation, boundaries, gradients, divergence, flux
// ---------------------------------------------------------------------------
// interpolate_Scalar! (Calculate_2_interpolation.jl:58-76)
static void interpolate(const Mesh& m, const std::vector<double>& phi, std::vector<double>& phif) {
#pragma omp parallel for schedule(static)
    for (int f = 0; f < m.n_faces; ++f) {
        double w = m.fweight[f];
        double omw = 1.0 - w;
        phif[f] = w * phi[m.owner[f]] + omw * phi[m.neigh[f]];
    }
}

// boundary_interpolation! for every BC (1_boundary_interpolation.jl and the
// *_interpolation.jl files); vector fields pass all three components
static void correct_boundaries(Case& C, const std::vector<BC>& bcs, std::vector<double>* phif,
                               const std::vector<double>* phi, bool vector) {
    const Mesh& m = *C.m;
    int ncomp = vector ? 3 : 1;
    for (int f = 0; f < C.nB; ++f) {
        const BC* bc = find_bc(bcs, f);
        if (!bc) continue;
        int i = f - bc->start;
        int c = m.bcell[f];
        switch (bc->type) {
            case XCAL_BC_DIRICHLET:
            case XCAL_BC_DIRICHLET_FUNCTION:
                for (int d = 0; d < ncomp; ++d) phif[d][f] = bc_value(*bc, vector, d, i);
                break;
            case XCAL_BC_WALL:
                if (vector)
                    for (int d = 0; d < 3; ++d) phif[d][f] = bc->value[d];
                else
                    phif[0][f] = phi[0][c];
                break;
            case XCAL_BC_ZEROGRADIENT:
            case XCAL_BC_OMEGA_WALL:
            case XCAL_BC_K_WALL:
            case XCAL_BC_NUT_WALL:
            case XCAL_BC_EXTRAPOLATED:
                for (int d = 0; d < ncomp; ++d) phif[d][f] = phi[d][c];
                break;
            case XCAL_BC_EMPTY:
                for (int d = 0; d < ncomp; ++d) phif[d][f] = 0.0;
                break;
            case XCAL_BC_SYMMETRY:
                if (!vector) {
                    phif[0][f] = phi[0][c];
                } else {
                    V3 n = m.fnormal[f];
                    V3 pc{phi[0][c], phi[1][c], phi[2][c]};
                    V3 pn = dot(pc, n) * n;
                    V3 r = pc - pn;
                    phif[0][f] = r.x;
                    phif[1][f] = r.y;
                    phif[2][f] = r.z;
                }
                break;
            case XCAL_BC_NEUMANN:
                phif[0][f] = phi[0][c] + m.fdelta[f] * bc->value[0];
                break;
            case XCAL_BC_PERIODIC:
                break;
            case XCAL_BC_PERIODIC_PARENT: {
                int pfID = bc->face_map[i];
                int pc = m.owner[pfID];
                int cID = m.owner[f];
                V3 Pf = m.fcentre[f] - m.ccentre[cID];
                V3 PN = (m.ccentre[pc] - bc->distance) - m.ccentre[cID];
                V3 n = m.fnormal[f];
                double wn = dot(Pf, n) / dot(PN, n);
                double w = 1.0 - wn;
                for (int d = 0; d < ncomp; ++d) {
                    double v = w * phi[d][cID] + wn * phi[d][pc];
                    phif[d][f] = v;
                    phif[d][pfID] = v;
                }
                break;
            }
            default:
                break;
        }
    }
}

// green_gauss! scalar -> vector (Calculate_1_green_gauss.jl:5-78)
static void green_gauss(const Mesh& m, const std::vector<double>& phif, std::vector<double>* g) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < m.n_cells; ++i) {
        V3 res{0, 0, 0};
        for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
            int f = m.cell_faces[k];
            V3 Sf = (m.farea[f] * m.fnormal[f]) * (double)m.cell_nsign[k];
            res = res + phif[f] * Sf;
        }
        res = res / m.cvol[i];
        g[0][i] = res.x;
        g[1][i] = res.y;
        g[2][i] = res.z;
    }
    for (int f = 0; f < m.n_bfaces; ++f) {
        int c = m.owner[f];
        V3 res = phif[f] * (m.farea[f] * m.fnormal[f]);
        res = res / m.cvol[c];
        g[0][c] = g[0][c] + res.x;
        g[1][c] = g[1][c] + res.y;
        g[2][c] = g[2][c] + res.z;
    }
}

// green_gauss! vector -> tensor (Calculate_1_green_gauss.jl:82-173)
static void green_gauss_tensor(const Mesh& m, const std::vector<double>* psif, std::vector<double>* g) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < m.n_cells; ++i) {
        double res[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
            int f = m.cell_faces[k];
            V3 Sf = (m.farea[f] * m.fnormal[f]) * (double)m.cell_nsign[k];
            double u[3] = {psif[0][f], psif[1][f], psif[2][f]};
            double s[3] = {Sf.x, Sf.y, Sf.z};
            for (int a = 0; a < 3; ++a)
                for (int bb = 0; bb < 3; ++bb) res[3 * a + bb] = res[3 * a + bb] + u[a] * s[bb];
        }
        for (int q = 0; q < 9; ++q) g[q][i] = res[q] / m.cvol[i];
    }
    for (int f = 0; f < m.n_bfaces; ++f) {
        int c = m.owner[f];
        V3 Sf = m.farea[f] * m.fnormal[f];
        double u[3] = {psif[0][f], psif[1][f], psif[2][f]};
        double s[3] = {Sf.x, Sf.y, Sf.z};
        for (int a = 0; a < 3; ++a)
            for (int bb = 0; bb < 3; ++bb) {
                double r = (u[a] * s[bb]) / m.cvol[c];
                g[3 * a + bb][c] = g[3 * a + bb][c] + r;
            }
    }
}

// div! of a face scalar (Calculate_0_divergence.jl:99-170)
static void divergence(const Mesh& m, const std::vector<double>& psif, std::vector<double>& out) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < m.n_cells; ++i) {
        double red = 0.0;
        for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k)
            red = red + psif[m.cell_faces[k]] * (double)m.cell_nsign[k];
        out[i] = red / m.cvol[i];
    }
    for (int f = 0; f < m.n_bfaces; ++f) {
        int c = m.owner[f];
        out[c] = out[c] + psif[f] / m.cvol[c];
    }
}

// flux! (Solvers_0_functions.jl:41-62)
static void flux(const Mesh& m, const std::vector<double>* Uf, std::vector<double>& mdot) {
#pragma omp parallel for schedule(static)
    for (int f = 0; f < m.n_faces; ++f) {
        V3 Sf = m.farea[f] * m.fnormal[f];
        V3 u{Uf[0][f], Uf[1][f], Uf[2][f]};
        mdot[f] = dot(u, Sf);
    }
}

// correct_interpolation_periodic (Solvers_1_SIMPLE.jl:427-470)
static void correct_interp_periodic(Case& C, std::vector<double>& phif, const std::vector<double>& phi) {
    const Mesh& m = *C.m;
    for (const BC& bc : C.bcU) {
        if (bc.type != XCAL_BC_PERIODIC_PARENT) continue;
        for (int i = 0; i < bc.count; ++i) {
            int f = bc.start + i, pf = bc.face_map[i];
            int c = m.owner[f], pc = m.owner[pf];
            double w = m.fdelta[pf] / (m.fdelta[f] + m.fdelta[pf]);
            double omw = 1.0 - w;
            double v = w * phi[c] + omw * phi[pc];
            phif[f] = v;
            phif[pf] = v;
        }
    }
}

// grad!(grad p) (Calculate_0_gradient.jl:105-111)
// Midpoint gradient (Calculate_0_gradient.jl:170-262): internal faces get
// 0.5 (phi1 + phi2) (interpolate_midpoint!, boundary faces as for Gauss),
// Green-Gauss, then twice: phif = 0.5 (phi1 + phi2) + (0.5 (grad1 + grad2)).Ri
// with Ri = rf - 0.5 (rP + rN) (correct_interpolation!) and Green-Gauss.
static V3 mid_R(const Mesh& m, int f) {
    return m.fcentre[f] - 0.5 * (m.ccentre[m.owner[f]] + m.ccentre[m.neigh[f]]);
}

// limit_gradient!(CellBased(level), grad F, F)
// (Calculate_0_gradient_cell_limiter.jl:68-108), F scalar (grad F = g[0..2])
// or one component of U with its row of grad U (:47-63): per cell the
// neighbours' max/min of F, then the smallest ratio over its internal faces
// of the allowed change to the gradient-extrapolated change (fc - cc).grad,
// |change| > 10 eps(F_P); grad *= 1 - level (1 - limiter)
static void limit_cell(Case& C, const std::vector<double>& F, std::vector<double>* g, double level) {
    const Mesh& m = *C.m;
    for (int i = 0; i < C.nC; ++i) {
        const double phiP = F[i];
        double phiMax = phiP, phiMin = phiP;
        for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
            const double phiN = F[m.cell_neigh[k]];
            phiMax = jl_max(phiN, phiMax);
            phiMin = jl_min(phiN, phiMin);
        }
        const V3 g0 = {g[0][i], g[1][i], g[2][i]};
        double lim = 1.0;
        const double e = 10.0 * jl_eps(phiP);
        for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
            const int f = m.cell_faces[k];
            const double d = dot(m.fcentre[f] - m.ccentre[i], g0);
            if (d > e)
                lim = jl_min(lim, (phiMax - phiP) / d);
            else if (d < -e)
                lim = jl_min(lim, (phiMin - phiP) / d);
        }
        lim = 1.0 - level * (1.0 - lim);
        g[0][i] = g0.x * lim;
        g[1][i] = g0.y * lim;
        g[2][i] = g0.z * lim;
    }
}

// limit_gradient!(FaceBased) (Calculate_0_gradient_face_limiter.jl:31-92,
// 152-170): each internal face lowers both cells' limiters (an atomic
// minimum in the reference, so a cell's limiter is the smallest candidate
// of its faces and 1 in any order; here each cell's faces in turn).  Per
// face the bounds min/max(F_owner, F_neighbour) widened by their difference,
// the cell's extrapolated change dF = grad . (fc - cc) and the candidate
// (Fmax - F)/dF (dF > Fmax - F) or (Fmin - F)/dF (dF < Fmin - F); then
// grad *= limiter.
static void lower_limiter(double& lim, double Fmax, double Fmin, double dF, double F) {
    const double dmax = Fmax - F, dmin = Fmin - F;
    if (dF > dmax) {
        const double v = dmax / dF;
        if (v < lim) lim = v;
    } else if (dF < dmin) {
        const double v = dmin / dF;
        if (v < lim) lim = v;
    }
}
static void limit_face_scalar(Case& C, const std::vector<double>& F, std::vector<double>* g) {
    const Mesh& m = *C.m;
    for (int i = 0; i < C.nC; ++i) {
        const V3 g0 = {g[0][i], g[1][i], g[2][i]};
        double lim = 1.0;
        for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
            const int f = m.cell_faces[k];
            const double F1 = F[m.owner[f]], F2 = F[m.neigh[f]];
            double mn = jl_min(F1, F2), mx = jl_max(F1, F2);
            const double dl = mx - mn;
            mn = mn - dl;
            mx = mx + dl;
            lower_limiter(lim, mx, mn, dot(g0, m.fcentre[f] - m.ccentre[i]), F[i]);
        }
        g[0][i] = g0.x * lim;
        g[1][i] = g0.y * lim;
        g[2][i] = g0.z * lim;
    }
}
// the vector form (:94-151): gradf = grad U (fc - cc) (row a . d), both
// cells' U projected on it, measure gradf . gradf; one limiter per cell
// scales all nine components
static void limit_face_vector(Case& C, std::vector<double>* g) {
    const Mesh& m = *C.m;
    for (int i = 0; i < C.nC; ++i) {
        double lim = 1.0;
        for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
            const int f = m.cell_faces[k];
            const V3 d = m.fcentre[f] - m.ccentre[i];
            double gf[3];
            for (int a = 0; a < 3; ++a)
                gf[a] = (g[3 * a][i] * d.x + g[3 * a + 1][i] * d.y) + g[3 * a + 2][i] * d.z;
            const int o = m.owner[f], n = m.neigh[f];
            const double vOwn = (gf[0] * C.U[0][o] + gf[1] * C.U[1][o]) + gf[2] * C.U[2][o];
            const double vNei = (gf[0] * C.U[0][n] + gf[1] * C.U[1][n]) + gf[2] * C.U[2][n];
            double mx = jl_max(vOwn, vNei), mn = jl_min(vOwn, vNei);
            const double dl = mx - mn;
            mx = mx + dl;
            mn = mn - dl;
            lower_limiter(lim, mx, mn, (gf[0] * gf[0] + gf[1] * gf[1]) + gf[2] * gf[2], i == o ? vOwn : vNei);
        }
        for (int q = 0; q < 9; ++q) g[q][i] = g[q][i] * lim;
    }
}

// limit_gradient!(::MFaceBased) (Calculate_0_gradient_mface_limiter.jl):
// the face kernel run on one thread, face by face in ascending id; a face's
// two updates touch different cells, so each cell takes its own internal
// faces' corrections in ascending face order (set_limiter, :62-74):
// grad += d (bound - grad . d) / (d . d) where grad . d leaves
// [min, max](F_own, F_nei) - F_cell, d = fc - cc
static std::vector<int> sorted_internal_faces(const Mesh& m, int i) {
    std::vector<int> fs(m.cell_faces.begin() + m.cf_off[i], m.cell_faces.begin() + m.cf_off[i + 1]);
    std::sort(fs.begin(), fs.end());
    return fs;
}
static void limit_mface_scalar(Case& C, const std::vector<double>& F, std::vector<double>* g) {
    const Mesh& m = *C.m;
    for (int i = 0; i < C.nC; ++i) {
        V3 gr = {g[0][i], g[1][i], g[2][i]};
        for (int f : sorted_internal_faces(m, i)) {
            const double F1 = F[m.owner[f]], F2 = F[m.neigh[f]];
            const double dmax = jl_max(F1, F2) - F[i], dmin = jl_min(F1, F2) - F[i];
            const V3 d = m.fcentre[f] - m.ccentre[i];
            const double fval = dot(gr, d), d2 = dot(d, d);
            if (fval > dmax)
                gr = {gr.x + (d.x * (dmax - fval)) / d2, gr.y + (d.y * (dmax - fval)) / d2,
                      gr.z + (d.z * (dmax - fval)) / d2};
            else if (fval < dmin)
                gr = {gr.x + (d.x * (dmin - fval)) / d2, gr.y + (d.y * (dmin - fval)) / d2,
                      gr.z + (d.z * (dmin - fval)) / d2};
        }
        g[0][i] = gr.x;
        g[1][i] = gr.y;
        g[2][i] = gr.z;
    }
}
// Julia's isless on Float64 and Base's lexicographic isless of vectors
// (cmp: the first entry not isequal decides); min / max(x, y) of two
// vectors are whole vectors: isless(y, x) ? y : x and isless(y, x) ? x : y
static bool jl_isless_d(double a, double b) {
    if (std::isnan(a)) return false;
    if (std::isnan(b)) return true;
    return a < b || (a == b && std::signbit(a) && !std::signbit(b));
}
static bool lex_isless(const double* a, const double* b) {
    for (int j = 0; j < 3; ++j) {
        const bool eq = (std::isnan(a[j]) && std::isnan(b[j])) ||
                        (a[j] == b[j] && std::signbit(a[j]) == std::signbit(b[j]));
        if (!eq) return jl_isless_d(a[j], b[j]);
    }
    return false;
}
// the tensor form (:76-113): row a of grad U against component a
static void limit_mface_vector(Case& C, std::vector<double>* g) {
    const Mesh& m = *C.m;
    for (int i = 0; i < C.nC; ++i) {
        double G[9];
        for (int q = 0; q < 9; ++q) G[q] = g[q][i];
        const double ui[3] = {C.U[0][i], C.U[1][i], C.U[2][i]};
        for (int f : sorted_internal_faces(m, i)) {
            const int o = m.owner[f], n = m.neigh[f];
            const double F1[3] = {C.U[0][o], C.U[1][o], C.U[2][o]};
            const double F2[3] = {C.U[0][n], C.U[1][n], C.U[2][n]};
            const bool lt = lex_isless(F2, F1);
            const double* mx = lt ? F1 : F2;
            const double* mn = lt ? F2 : F1;
            const V3 d = m.fcentre[f] - m.ccentre[i];
            const double dv[3] = {d.x, d.y, d.z};
            const double d2 = dot(d, d);
            for (int a = 0; a < 3; ++a) {
                const double dmax = mx[a] - ui[a], dmin = mn[a] - ui[a];
                const double fval = (G[3 * a] * d.x + G[3 * a + 1] * d.y) + G[3 * a + 2] * d.z;
                if (fval > dmax)
                    for (int b = 0; b < 3; ++b) G[3 * a + b] = G[3 * a + b] + (dv[b] * (dmax - fval)) / d2;
                else if (fval < dmin)
                    for (int b = 0; b < 3; ++b) G[3 * a + b] = G[3 * a + b] + (dv[b] * (dmin - fval)) / d2;
            }
        }
        for (int q = 0; q < 9; ++q) g[q][i] = G[q];
    }
}

static void grad_p_only(Case& C);

static void grad_p(Case& C) {
    grad_p_only(C);
    if (C.cfg.p_schemes.limiter == XCAL_LIMITER_CELL) limit_cell(C, C.p, C.gradp, C.cfg.p_schemes.limiter_level);
    if (C.cfg.p_schemes.limiter == XCAL_LIMITER_FACE) limit_face_scalar(C, C.p, C.gradp);
    if (C.cfg.p_schemes.limiter == XCAL_LIMITER_MFACE) limit_mface_scalar(C, C.p, C.gradp);
}

static void grad_p_only(Case& C) {
    const Mesh& m = *C.m;
    interpolate(m, C.p, C.pf);
    correct_boundaries(C, C.bcP, &C.pf, &C.p, false);
    if (C.cfg.p_schemes.gradient != XCAL_GRAD_MIDPOINT) {
        green_gauss(m, C.pf, C.gradp);
        return;
    }
    for (int f = C.nB; f < C.nF; ++f) C.pf[f] = 0.5 * (C.p[m.owner[f]] + C.p[m.neigh[f]]);
    green_gauss(m, C.pf, C.gradp);
    for (int it = 0; it < 2; ++it) {
        for (int f = C.nB; f < C.nF; ++f) {
            const int c1 = m.owner[f], c2 = m.neigh[f];
            const V3 g1 = {C.gradp[0][c1], C.gradp[1][c1], C.gradp[2][c1]};
            const V3 g2 = {C.gradp[0][c2], C.gradp[1][c2], C.gradp[2][c2]};
            C.pf[f] = 0.5 * (C.p[c1] + C.p[c2]) + dot(0.5 * (g1 + g2), mid_R(m, f));
        }
        green_gauss(m, C.pf, C.gradp);
    }
}

// grad!(grad U) (Calculate_0_gradient.jl:113-119)
static void grad_U_only(Case& C);

static void grad_U(Case& C) {  // grad! + limit_gradient!(schemes.U.limiter) (RANS_laminar.jl:76-77)
    grad_U_only(C);
    if (C.cfg.U_schemes.limiter == XCAL_LIMITER_CELL)
        for (int a = 0; a < 3; ++a) limit_cell(C, C.U[a], C.gradU + 3 * a, C.cfg.U_schemes.limiter_level);
    if (C.cfg.U_schemes.limiter == XCAL_LIMITER_FACE) limit_face_vector(C, C.gradU);
    if (C.cfg.U_schemes.limiter == XCAL_LIMITER_MFACE) limit_mface_vector(C, C.gradU);
}

static void grad_U_only(Case& C) {
    const Mesh& m = *C.m;
    for (int d = 0; d < 3; ++d) interpolate(m, C.U[d], C.Uf[d]);
    correct_boundaries(C, C.bcU, C.Uf, C.U, true);
    if (C.cfg.U_schemes.gradient != XCAL_GRAD_MIDPOINT) {
        green_gauss_tensor(m, C.Uf, C.gradU);
        return;
    }
    for (int f = C.nB; f < C.nF; ++f)
        for (int d = 0; d < 3; ++d) C.Uf[d][f] = 0.5 * (C.U[d][m.owner[f]] + C.U[d][m.neigh[f]]);
    green_gauss_tensor(m, C.Uf, C.gradU);
    for (int it = 0; it < 2; ++it) {
        for (int f = C.nB; f < C.nF; ++f) {
            const int c1 = m.owner[f], c2 = m.neigh[f];
            const V3 R = mid_R(m, f);
            for (int a = 0; a < 3; ++a) {
                const double M0 = 0.5 * (C.gradU[3 * a][c1] + C.gradU[3 * a][c2]);
                const double M1 = 0.5 * (C.gradU[3 * a + 1][c1] + C.gradU[3 * a + 1][c2]);
                const double M2 = 0.5 * (C.gradU[3 * a + 2][c1] + C.gradU[3 * a + 2][c2]);
                // (grad*Ri)_a = (M[a,1] R1 + M[a,2] R2) + M[a,3] R3
                C.Uf[a][f] = 0.5 * (C.U[a][c1] + C.U[a][c2]) + (M0 * R.x + M1 * R.y + M2 * R.z);
            }
        }
        green_gauss_tensor(m, C.Uf, C.gradU);
    }
}

// update_nueff! (Solvers_0_functions.jl:5-35)
static void update_nueff(Case& C) {
    for (int f = 0; f < C.nF; ++f)
        C.nueff[f] = C.cfg.turbulence == XCAL_TURB_LAMINAR ? C.cfg.nu : C.cfg.nu + C.nutf[f];
}

// ---------------------------------------------------------------------------
// SIMPLE / PISO building blocks
// ---------------------------------------------------------------------------
void initial_calculations(Case& C) {  // Solvers_1_SIMPLE.jl:150-156
    for (int d = 0; d < 3; ++d) interpolate(*C.m, C.U[d], C.Uf[d]);
    correct_boundaries(C, C.bcU, C.Uf, C.U, true);
    flux(*C.m, C.Uf, C.mdotf);
    grad_p(C);
    update_nueff(C);
    C.initialised = true;
}

void solve_equation_U(Case& C, double res[3], int iters[3]) {  // Solve_1_api.jl:233-266
    discretise_U(C);
    for (int d = 0; d < 3; ++d) {
        update_equation(C);
        apply_bcs(C, true, d);
        relax_diagdom(C, d);
        if (d == 0) update_precond(C.AU, C.cfg.U_solver.precond, C.PU);
        res[d] = solve_system(C, true, d, iters ? &iters[d] : nullptr);
    }
}

double solve_equation_p(Case& C, int* iters) {  // Solve_1_api.jl:214-231
    discretise_p(C);
    apply_bcs(C, false, 0);
    set_reference(C);
    update_precond(C.Ap, C.cfg.p_solver.precond, C.Pp);
    return solve_system(C, false, 0, iters);
}

void pressure_predictor(Case& C, bool with_H) {  // Solvers_1_SIMPLE.jl:170-174
    const Mesh& m = *C.m;
    CSR& A = C.AU;
    for (int i = 0; i < C.nC; ++i) C.rD[i] = m.cvol[i] / A.nzval[A.diag[i]];
    interpolate(m, C.rD, C.rDf);
    correct_interp_periodic(C, C.rDf, C.rD);
    // remove_pressure_source! (Solvers_0_functions.jl:156-181), source sign -1
    for (int i = 0; i < C.nC; ++i) {
        double V = m.cvol[i];
        for (int d = 0; d < 3; ++d) {
            double calc = (-1.0 * C.gradp[d][i]) * V;
            C.bU[d][i] = C.bU[d][i] - calc;
        }
    }
    if (with_H) {
        extern void H(Case & C);
        H(C);
    }
}

// H! (Solvers_0_functions.jl:184-249)
void H(Case& C) {
    CSR& A = C.AU;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < C.nC; ++i) {
        double sx = 0.0, sy = 0.0, sz = 0.0;
        for (int k = A.rowptr[i]; k < A.rowptr[i + 1]; ++k) {
            int j = A.colval[k];
            double val = A.nzval[k];
            sx = sx + val * C.U[0][j];
            sy = sy + val * C.U[1][j];
            sz = sz + val * C.U[2][j];
        }
        double D = A.nzval[A.diag[i]];
        sx = sx - D * C.U[0][i];
        sy = sy - D * C.U[1][i];
        sz = sz - D * C.U[2][i];
        double rD = 1.0 / D;
        C.Hv[0][i] = (C.bU[0][i] - sx) * rD;
        C.Hv[1][i] = (C.bU[1][i] - sy) * rD;
        C.Hv[2][i] = (C.bU[2][i] - sz) * rD;
    }
}

void flux_divergence(Case& C) {  // Solvers_1_SIMPLE.jl:177-185
    for (int d = 0; d < 3; ++d) interpolate(*C.m, C.Hv[d], C.Uf[d]);
    correct_boundaries(C, C.bcU, C.Uf, C.Hv, true);
    flux(*C.m, C.Uf, C.mdotf);
    divergence(*C.m, C.mdotf, C.divHv);
}

void explicit_relaxation_p(Case& C, double alpha) {  // Solve_1_api.jl:317-335
    for (int i = 0; i < C.nC; ++i) C.p[i] = C.prev[i] + alpha * (C.p[i] - C.prev[i]);
}

// correct_mass_flux! (Solvers_1_SIMPLE.jl:340-557) + correct_velocity!
void correct(Case& C) {
    const Mesh& m = *C.m;
    CSR& A = C.Ap;
    for (int f = C.nB; f < C.nF; ++f) {
        int c1 = m.owner[f], c2 = m.neigh[f];
        double aN = A.nzval[A.find(c1, c2)];
        C.mdotf[f] = C.mdotf[f] + aN * (C.p[c2] - C.p[c1]);
    }
    for (const BC& bc : C.bcP) {
        if (bc.type != XCAL_BC_PERIODIC_PARENT) continue;
        for (int i = 0; i < bc.count; ++i) {
            int f = bc.start + i, pf = bc.face_map[i];
            int c1 = m.owner[f], c2 = m.owner[pf];
            double aN = A.nzval[A.find(c1, c2)];
            double corr = aN * (C.p[c2] - C.p[c1]);
            C.mdotf[f] = C.mdotf[f] + corr;
            C.mdotf[pf] = -C.mdotf[f];
        }
    }
    for (int f = 0; f < C.nB; ++f) {
        const BC* bc = find_bc(C.bcP, f);
        if (!bc) continue;
        int c = m.bcell[f];
        if (bc->type == XCAL_BC_DIRICHLET || bc->type == XCAL_BC_DIRICHLET_FUNCTION) {
            double fl = (C.rDf[f] * m.farea[f]) / m.fdelta[f];
            double ap = -1.0 * (-fl);
            double val = bc_value(*bc, false, 0, f - bc->start);
            C.mdotf[f] = C.mdotf[f] + ap * (C.p[c] - val);
        } else if (bc->type == XCAL_BC_NEUMANN) {
            C.mdotf[f] = C.mdotf[f] - (C.rDf[f] * m.farea[f]) * bc->value[0];
        }
    }
    // correct_velocity! (Solvers_0_functions.jl:126-151)
    for (int i = 0; i < C.nC; ++i) {
        double r = C.rD[i];
        for (int d = 0; d < 3; ++d) C.U[d][i] = C.Hv[d][i] - C.gradp[d][i] * r;
    }
}

// ---------------------------------------------------------------------------
// RANS{KOmega} (src/ModelPhysics/Turbulence/RANS_kOmega.jl)
// ---------------------------------------------------------------------------
// _discretise_scalar_model! (Discretise_2_generated_distretisation.jl:125-167)
// with a field `phi` (Time terms) and +Source(src)
static void discretise_scalar(Case& C, const std::vector<Term>& terms, CSR& A, std::vector<double>& b,
                              const std::vector<double>& phi, const std::vector<double>& src) {
    const Mesh& m = *C.m;
    std::fill(A.nzval.begin(), A.nzval.end(), 0.0);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < C.nC; ++i) {
        double ac_sum = 0.0;
        for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
            int fID = m.cell_faces[k], ns = m.cell_nsign[k], nID = m.cell_neigh[k];
            double AC = 0.0, AN = 0.0;
            for (const Term& t : terms) {
                double ac, an;
                scheme(m, t, fID, ns, ac, an);
                AC = AC + ac;
                AN = AN + an;
            }
            ac_sum = ac_sum + AC;
            A.nzval[A.find(i, nID)] = AN;
        }
        double AC = 0.0, B = 0.0;
        for (const Term& t : terms) {
            double ac, bb;
            scheme_source(C, t, i, phi[i], ac, bb);
            AC = AC + ac;
            B = B + bb;
        }
        A.nzval[A.diag[i]] = ac_sum + AC;
        double b2 = 0.0 + (1.0 * src[i]) * m.cvol[i];  // _sources!: +Source(src)
        b[i] = b2 + B;
    }
}

// apply_boundary_conditions! of a scalar equation, ascending boundary face id
static void apply_bcs_scalar(Case& C, const std::vector<Term>& terms, CSR& A, std::vector<double>& b,
                             const std::vector<BC>& bcs, const std::vector<double>& phi) {
    const Mesh& m = *C.m;
    BCCtx X{&C, &A, false, 0, &phi};
    for (int f = 0; f < C.nB; ++f) {
        const BC* bc = find_bc(bcs, f);
        if (!bc) continue;
        int cell = m.bcell[f];
        double AP = 0.0, BP = 0.0;
        for (const Term& t : terms) {
            double ap, bp;
            bc_functor(X, *bc, t, f, ap, bp);
            AP = AP + ap;
            BP = BP + bp;
        }
        A.nzval[A.diag[cell]] = A.nzval[A.diag[cell]] + AP;
        b[cell] = b[cell] + BP;
    }
}

// implicit_relaxation_diagdom! (Solve_1_api.jl:388-411) of a scalar equation
static void relax_scalar(CSR& A, std::vector<double>& b, const std::vector<double>& field, double alpha) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < A.n; ++i) {
        int c = A.diag[i];
        double sumv = 0.0;
        for (int k = A.rowptr[i]; k < A.rowptr[i + 1]; ++k) sumv = sumv + std::fabs(A.nzval[k]);
        sumv = sumv - std::fabs(A.nzval[c]);
        double D0 = A.nzval[c];
        double D_max = jl_max(std::fabs(D0), sumv) / alpha;
        A.nzval[c] = D_max;
        b[i] = b[i] + (D_max - D0) * field[i];
    }
}

// constrain_equation!(omega_eqn, OmegaWallFunction) (RANS_functions.jl:376-429):
// per wall face, in BC order then face order, the wall cell's row becomes
// omega = omega_log (y+ > yPlusLam) or omega_vis, from the current k
static void constrain_omega(Case& C, CSR& A, std::vector<double>& b) {
    const Mesh& m = *C.m;
    const double nu = C.cfg.nu;
    for (const BC& bc : C.bcOmega) {
        if (bc.type != XCAL_BC_OMEGA_WALL) continue;
        const double kappa = bc.wall[0], beta1 = bc.wall[1], c25 = bc.wall[2], yPlusLam = bc.wall[3];
        for (int f = bc.start; f < bc.start + bc.count; ++f) {
            const int c = m.bcell[f];
            const double y = m.fdelta[f];
            const double w_vis = (6.0 * nu) / (beta1 * (y * y));          // omega_vis (:50)
            const double w_log = std::sqrt(C.k[c]) / ((c25 * kappa) * y);  // omega_log (:51)
            const double yplus = ((c25 * y) * std::sqrt(C.k[c])) / nu;    // y_plus (:52)
            const double wc = yplus > yPlusLam ? w_log : w_vis;
            for (int e = A.rowptr[c]; e < A.rowptr[c + 1]; ++e) A.nzval[e] = 0.0;
            A.nzval[A.diag[c]] = 1.0;
            b[c] = wc;
        }
    }
}

// bound! (RANS_functions.jl:2-41): each cell from the values before the
// call (the reference updates in place while neighbours read, so its result
// can depend on thread order where adjacent cells are both clipped)
static void bound_field(const Mesh& m, std::vector<double>& v) {
    const double mzero = jl_eps(1.0);
    const std::vector<double> old(v);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < (int)v.size(); ++i) {
        double sum_flux = 0.0;
        int sum_area = 0;
        for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
            sum_flux = sum_flux + jl_max(old[m.cell_neigh[k]], mzero);
            sum_area += 1;
        }
        const double average = sum_flux / (double)sum_area;
        // average * signbit(v): average, or a zero with average's sign
        const double s = std::signbit(old[i]) ? average : std::copysign(0.0, average);
        v[i] = jl_max(jl_max(old[i], s), mzero);
    }
}

// nut_wall (RANS_functions.jl:61-63)
static double nut_wall(double nu, double yplus, double kappa, double E) {
    return jl_max(nu * (((yplus * kappa) / det_log(jl_max(E * yplus, 1.0 + 1e-4))) - 1.0), 0.0);
}

// correct_production!(Pk, KWallFunction) (RANS_functions.jl:66-117): per
// wall face (BC order, face order), the cell's production from the log law
static void kwall_production(Case& C) {
    const Mesh& m = *C.m;
    const double nu = C.cfg.nu;
    for (const BC& bc : C.bcK) {
        if (bc.type != XCAL_BC_K_WALL) continue;
        const double kappa = bc.wall[0], c25 = bc.wall[2], yPlusLam = bc.wall[3], E = bc.wall[4];
        for (int f = bc.start; f < bc.start + bc.count; ++f) {
            const int c = m.bcell[f];
            const double delta = m.fdelta[f];
            const V3 n = m.fnormal[f];
            const double sk = std::sqrt(C.k[c]);
            const double uStar = c25 * sk;
            const double dUdy = uStar / (kappa * delta);
            const double yplus = ((c25 * delta) * sk) / nu;
            const double nutw = nut_wall(nu, yplus, kappa, E);
            const V3 Ud = {C.U[0][c] - 0.0, C.U[1][c] - 0.0, C.U[2][c] - 0.0};  // Ui - Uw, Uw = 0
            const V3 Up = Ud - dot(Ud, n) * n;
            const V3 g = Up / delta;
            const double mag = std::sqrt(g.x * g.x + g.y * g.y + g.z * g.z);
            C.Pk[c] = yplus > yPlusLam ? ((nu + nutw) * mag) * dUdy : 0.0;
        }
    }
}

// correct_eddy_viscosity!(nutf, NutWallFunction) (RANS_functions.jl:119-172)
static void nutwall_correct(Case& C) {
    const Mesh& m = *C.m;
    const double nu = C.cfg.nu;
    for (const BC& bc : C.bcNut) {
        if (bc.type != XCAL_BC_NUT_WALL) continue;
        const double kappa = bc.wall[0], c25 = bc.wall[2], yPlusLam = bc.wall[3], E = bc.wall[4];
        for (int f = bc.start; f < bc.start + bc.count; ++f) {
            const int c = m.bcell[f];
            const double yplus = ((c25 * m.fdelta[f]) * std::sqrt(C.k[c])) / nu;
            C.nutf[f] = yplus > yPlusLam ? nut_wall(nu, yplus, kappa, E) : 0.0;
        }
    }
}

// solve_system! of k or omega on the shared scalar system
static double solve_scalar(Case& C, const xcal_solver_setup& SS0, int ptype, std::vector<double>& field,
                           std::vector<double>& P) {
    xcal_solver_setup SS = SS0;
    SS.precond = ptype;
    CSR& A = C.Ap;
    if (SS.smoother_loops > 0) jacobi_smooth(A, C.bp.data(), field.data(), SS.smoother_loops, SS.smoother_omega);
    if (SS.solver == XCAL_SOLVER_CG)
        krylov_cg(A, C.bp, field, SS.precond, P, SS, C.kp);
    else
        krylov_bicgstab(A, C.bp, field, SS.precond, P, SS, C.kp);
    return residual(A, C.bp, field);
}

// turbulence!(::KOmegaModel) after grad!(gradU) (RANS_kOmega.jl:146-210)
static void komega(Case& C) {
    const Mesh& m = *C.m;
    const xcal_config& cf = C.cfg;
    for (int i = 0; i < C.nC; ++i) {
        // magnitude2!(Pk, S, scale_factor = 2) (RANS_tensor_algebra.jl:81-99), S = 0.5 (G + G')
        double sum = 0.0;
        for (int j = 0; j < 3; ++j)
            for (int q = 0; q < 3; ++q) {
                const double s = 0.5 * (C.gradU[3 * j + q][i] + C.gradU[3 * q + j][i]);
                sum = sum + s * s;
            }
        const double mag = sum * 2.0;
        C.Pw[i] = cf.kw_alpha1 * mag;           // rho alpha1 Pk (rho = 1)
        C.Pk[i] = C.nut[i] * mag;               // rho nut Pk
        C.Dw[i] = cf.kw_beta1 * C.omega[i];     // rho beta1 omega
        C.Dk[i] = cf.kw_beta_star * C.omega[i];  // rho beta+ omega
    }
    kwall_production(C);
    for (int f = 0; f < C.nF; ++f) {  // rhof (nuf + sigma nutf), rhof = 1
        C.mueffw[f] = cf.nu + cf.kw_sigma_omega * C.nutf[f];
        C.mueffk[f] = cf.nu + cf.kw_sigma_k * C.nutf[f];
    }
    const int ptype = cf.k_solver.precond;
    // omega: Time + Div(mdotf) - Lap(mueffw) + Si(Dw) == Source(Pw)
    std::vector<Term> tw = {{T_TIME, 1.0, nullptr, cf.omega_schemes.time},
                            {T_DIV, 1.0, &C.mdotf, cf.omega_schemes.divergence},
                            {T_LAP, -1.0, &C.mueffw, 0},
                            {T_SI, 1.0, &C.Dw, 0}};
    discretise_scalar(C, tw, C.Ap, C.bp, C.omega, C.Pw);
    apply_bcs_scalar(C, tw, C.Ap, C.bp, C.bcOmega, C.omega);
    relax_scalar(C.Ap, C.bp, C.omega, cf.omega_solver.relax);
    constrain_omega(C, C.Ap, C.bp);
    update_precond(C.Ap, ptype, C.Pkw);
    C.res_omega = solve_scalar(C, cf.omega_solver, ptype, C.omega, C.Pkw);
    bound_field(m, C.omega);
    // k: Time + Div(mdotf) - Lap(mueffk) + Si(Dk) == Source(Pk)
    std::vector<Term> tk = {{T_TIME, 1.0, nullptr, cf.k_schemes.time},
                            {T_DIV, 1.0, &C.mdotf, cf.k_schemes.divergence},
                            {T_LAP, -1.0, &C.mueffk, 0},
                            {T_SI, 1.0, &C.Dk, 0}};
    discretise_scalar(C, tk, C.Ap, C.bp, C.k, C.Pk);
    apply_bcs_scalar(C, tk, C.Ap, C.bp, C.bcK, C.k);
    relax_scalar(C.Ap, C.bp, C.k, cf.k_solver.relax);
    update_precond(C.Ap, ptype, C.Pkw);
    C.res_k = solve_scalar(C, cf.k_solver, ptype, C.k, C.Pkw);
    bound_field(m, C.k);
    for (int i = 0; i < C.nC; ++i) C.nut[i] = C.k[i] / C.omega[i];
    interpolate(m, C.nut, C.nutf);
    correct_boundaries(C, C.bcNut, &C.nutf, &C.nut, false);
    nutwall_correct(C);
}

// turbulence!(::KEquationModel) after grad!(gradU) and its limiter
// (LES_KEquation.jl:134-186), rho = 1: mueffk = nu + nut_f; per cell
// Pk = 2 nut (grad U . dev(S)) (the Frobenius product over the column-major
// entries, S = (G + G')/2, dev(S) = S - tr(S)/3 I), Dkf = ce sqrt(k) / Delta,
// divU = 2/3 tr(grad U); the k equation Time + Div(mdotf) - Lap(mueffk) +
// Si(Dkf) + Si(divU) == Source(Pk), its BCs, implicit relaxation, solve,
// bound!; nut = ck Delta sqrt(k), interpolated with its BCs and the wall
// functions (correct_eddy_viscosity!)
static void kequation(Case& C) {
    const Mesh& m = *C.m;
    const xcal_config& cf = C.cfg;
    for (int i = 0; i < C.nC; ++i) {
        double G[3][3], S[3][3];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) G[a][b] = C.gradU[3 * a + b][i];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) S[a][b] = 0.5 * (G[a][b] + G[b][a]);
        const double third = (1.0 / 3.0) * ((S[0][0] + S[1][1]) + S[2][2]);
        double dot = 0.0;
        bool first = true;
        for (int b = 0; b < 3; ++b)
            for (int a = 0; a < 3; ++a) {
                const double pr = G[a][b] * (a == b ? S[a][b] - third : S[a][b]);
                dot = first ? pr : dot + pr;
                first = false;
            }
        C.Pk[i] = (2.0 * C.nut[i]) * dot;
        C.Dk[i] = (cf.keq_ce * std::sqrt(C.k[i])) / C.Delta[i];
        C.Dw[i] = (2.0 / 3.0) * ((G[0][0] + G[1][1]) + G[2][2]);
    }
    for (int f = 0; f < C.nF; ++f) C.mueffk[f] = cf.nu + C.nutf[f];
    const int ptype = cf.k_solver.precond;
    std::vector<Term> tk = {{T_TIME, 1.0, nullptr, cf.k_schemes.time},
                            {T_DIV, 1.0, &C.mdotf, cf.k_schemes.divergence},
                            {T_LAP, -1.0, &C.mueffk, 0},
                            {T_SI, 1.0, &C.Dk, 0},
                            {T_SI, 1.0, &C.Dw, 0}};
    discretise_scalar(C, tk, C.Ap, C.bp, C.k, C.Pk);
    apply_bcs_scalar(C, tk, C.Ap, C.bp, C.bcK, C.k);
    relax_scalar(C.Ap, C.bp, C.k, cf.k_solver.relax);
    update_precond(C.Ap, ptype, C.Pkw);
    C.res_k = solve_scalar(C, cf.k_solver, ptype, C.k, C.Pkw);
    bound_field(m, C.k);
    for (int i = 0; i < C.nC; ++i) C.nut[i] = (cf.keq_ck * C.Delta[i]) * std::sqrt(C.k[i]);
    interpolate(m, C.nut, C.nutf);
    correct_boundaries(C, C.bcNut, &C.nutf, &C.nut, false);
    nutwall_correct(C);
}

// grad! of a scalar with its BCs, Gauss or Midpoint (Calculate_0_gradient.jl)
static void scalar_grad(Case& C, const std::vector<double>& phi, std::vector<double>& phif, const std::vector<BC>& bcs,
                        int scheme, std::vector<double>* g) {
    const Mesh& m = *C.m;
    interpolate(m, phi, phif);
    correct_boundaries(C, bcs, &phif, &phi, false);
    green_gauss(m, phif, g);
    if (scheme != XCAL_GRAD_MIDPOINT) return;
    for (int f = C.nB; f < C.nF; ++f) phif[f] = 0.5 * (phi[m.owner[f]] + phi[m.neigh[f]]);
    green_gauss(m, phif, g);
    for (int it = 0; it < 2; ++it) {
        for (int f = C.nB; f < C.nF; ++f) {
            const int c1 = m.owner[f], c2 = m.neigh[f];
            const V3 g1 = {g[0][c1], g[1][c1], g[2][c1]};
            const V3 g2 = {g[0][c2], g[1][c2], g[2][c2]};
            phif[f] = 0.5 * (phi[c1] + phi[c2]) + dot(0.5 * (g1 + g2), mid_R(m, f));
        }
        green_gauss(m, phif, g);
    }
}

// wall_distance! (Calculate_4_wall_distance.jl:4-78): -Laplacian(1, phi) ==
// Source(1) with the wall BCs, solved (y_solver) and explicitly relaxed up to
// 1000 times until its residual is below the convergence, then
// y = -|grad phi| + sqrt(|grad phi|^2 + 2 phi) (:80-92)
static void wall_distance(Case& C) {
    const xcal_solver_setup& SS = C.cfg.y_solver;
    std::vector<double> phi(C.nC, 0.0), prev(C.nC), ones_f(C.nF, 1.0), ones_c(C.nC, 1.0), phif(C.nF), g[3];
    for (int d = 0; d < 3; ++d) g[d].assign(C.nC, 0.0);
    std::vector<Term> terms = {{T_LAP, -1.0, &ones_f, 0}};
    scalar_grad(C, phi, phif, C.bcY, C.cfg.y_schemes.gradient, g);
    for (int it = 0; it < 1000; ++it) {
        prev = phi;
        discretise_scalar(C, terms, C.Ap, C.bp, phi, ones_c);
        apply_bcs_scalar(C, terms, C.Ap, C.bp, C.bcY, phi);
        update_precond(C.Ap, SS.precond, C.Pkw);
        const double res = solve_scalar(C, SS, SS.precond, phi, C.Pkw);
        for (int i = 0; i < C.nC; ++i) phi[i] = prev[i] + SS.relax * (phi[i] - prev[i]);
        if (res < SS.convergence) break;
    }
    scalar_grad(C, phi, phif, C.bcY, C.cfg.y_schemes.gradient, g);
    for (int i = 0; i < C.nC; ++i) {
        const double gm = std::sqrt(g[0][i] * g[0][i] + g[1][i] * g[1][i] + g[2][i] * g[2][i]);
        C.yw[i] = (-gm) + std::sqrt(gm * gm + 2.0 * phi[i]);
    }
}

// turbulence!(::KOmegaSSTModel) after grad!(gradU) (RANS_kOmegaSST.jl:190-315)
static void komega_sst(Case& C) {
    const Mesh& m = *C.m;
    const xcal_config& cf = C.cfg;
    const double bs = cf.kw_beta_star, al1 = cf.kw_alpha1, b1 = cf.kw_beta1, b2 = cf.sst_beta2;
    const double sk1 = cf.kw_sigma_k, sk2 = cf.sst_sigma_k2, sw1 = cf.kw_sigma_omega, sw2 = cf.sst_sigma_omega2;
    const double nu = cf.nu, eps = jl_eps(1.0);
    scalar_grad(C, C.omega, C.wfs, C.bcOmega, cf.p_schemes.gradient, C.gw);  // Grad{schemes.p.gradient}(omega)
    scalar_grad(C, C.k, C.kfs, C.bcK, cf.k_schemes.gradient, C.gk);
    for (int i = 0; i < C.nC; ++i) {
        double sum = 0.0;  // magnitude2!(Pk, S, 2)
        for (int j = 0; j < 3; ++j)
            for (int q = 0; q < 3; ++q) {
                const double s = 0.5 * (C.gradU[3 * j + q][i] + C.gradU[3 * q + j][i]);
                sum = sum + s * s;
            }
        const double mag = sum * 2.0;
        C.Om[i] = std::sqrt(mag);  // Omega = sqrt(Pk)
        const double w = C.omega[i], kk = C.k[i], y = C.yw[i];
        const double dkdw = (C.gk[0][i] * C.gw[0][i] + C.gk[1][i] * C.gw[1][i]) + C.gk[2][i] * C.gw[2][i];
        const double CD = jl_max(((2.0 * sw2) * dkdw) / w, 1e-10);
        const double sq = std::sqrt(jl_max(kk, eps));
        const double a1 = jl_min(jl_min(jl_max(sq / ((bs * w) * y), (500.0 * nu) / (w * (y * y))),
                                        ((4.0 * sw2) * kk) / (CD * (y * y))),
                                 10.0);
        const double a2 = jl_min(jl_max((2.0 * sq) / ((bs * w) * y), (500.0 * nu) / ((y * y) * w)), 100.0);
        const double f2 = det_tanh_pos(a2 * a2);
        const double f1 = det_tanh_pos((a1 * a1) * (a1 * a1));
        C.F1[i] = f1;
        C.F2[i] = f2;
        const double beta = b1 * f1 + (1.0 - f1) * b2;
        const double gamma = (5.0 / 9.0) * f1 + (1.0 - f1) * 0.44;
        C.Dw[i] = beta * w;
        C.Dk[i] = bs * w;
        C.Pw[i] = gamma * jl_min(mag, (((10.0 / al1) * bs) * w) * jl_max(al1 * w, f2 * C.Om[i]));
        C.Pk[i] = jl_min(mag * C.nut[i], ((10.0 * bs) * kk) * w);
        C.D2[i] = ((((2.0 * (f1 - 1.0)) * sw2) * dkdw) / w) / w;
    }
    kwall_production(C);
    for (int f = 0; f < C.nF; ++f) {  // interpolate!(F1f, F1); sigma blending; mueff
        const double wt = m.fweight[f];
        const double F1f = wt * C.F1[m.owner[f]] + (1.0 - wt) * C.F1[m.neigh[f]];
        const double sk = sk1 * F1f + (1.0 - F1f) * sk2;
        const double sw = sw1 * F1f + (1.0 - F1f) * sw2;
        C.mueffw[f] = nu + sw * C.nutf[f];
        C.mueffk[f] = nu + sk * C.nutf[f];
    }
    // omega: Time + Div - Lap(mueffw) + Si(Dw) + Si(D2) == Source(Pw), its own preconditioner
    std::vector<Term> tw = {{T_TIME, 1.0, nullptr, cf.omega_schemes.time},
                            {T_DIV, 1.0, &C.mdotf, cf.omega_schemes.divergence},
                            {T_LAP, -1.0, &C.mueffw, 0},
                            {T_SI, 1.0, &C.Dw, 0},
                            {T_SI, 1.0, &C.D2, 0}};
    discretise_scalar(C, tw, C.Ap, C.bp, C.omega, C.Pw);
    apply_bcs_scalar(C, tw, C.Ap, C.bp, C.bcOmega, C.omega);
    relax_scalar(C.Ap, C.bp, C.omega, cf.omega_solver.relax);
    constrain_omega(C, C.Ap, C.bp);
    update_precond(C.Ap, cf.omega_solver.precond, C.Pww);
    C.res_omega = solve_scalar(C, cf.omega_solver, cf.omega_solver.precond, C.omega, C.Pww);
    bound_field(m, C.omega);
    std::vector<Term> tk = {{T_TIME, 1.0, nullptr, cf.k_schemes.time},
                            {T_DIV, 1.0, &C.mdotf, cf.k_schemes.divergence},
                            {T_LAP, -1.0, &C.mueffk, 0},
                            {T_SI, 1.0, &C.Dk, 0}};
    discretise_scalar(C, tk, C.Ap, C.bp, C.k, C.Pk);
    apply_bcs_scalar(C, tk, C.Ap, C.bp, C.bcK, C.k);
    relax_scalar(C.Ap, C.bp, C.k, cf.k_solver.relax);
    update_precond(C.Ap, cf.k_solver.precond, C.Pkw);
    C.res_k = solve_scalar(C, cf.k_solver, cf.k_solver.precond, C.k, C.Pkw);
    bound_field(m, C.k);
    for (int i = 0; i < C.nC; ++i) C.nut[i] = (al1 * C.k[i]) / jl_max(al1 * C.omega[i], C.F2[i] * C.Om[i]);
    interpolate(m, C.nut, C.nutf);
    correct_boundaries(C, C.bcNut, &C.nutf, &C.nut, false);
    nutwall_correct(C);
}

// solve one transport equation of k-omega LKE on the shared scalar system
// (RANS_kOmegaLKE.jl:339-345, :393-399, :427-433): discretise!,
// apply_boundary_conditions!, implicit_relaxation!, (omega: constrain),
// update_preconditioner!, solve_system!, bound!
static double lke_solve(Case& C, const std::vector<Term>& t, std::vector<double>& phi, const std::vector<double>& src,
                        const std::vector<BC>& bcs, const xcal_solver_setup& SS, std::vector<double>& Pre,
                        bool constrain) {
    discretise_scalar(C, t, C.Ap, C.bp, phi, src);
    apply_bcs_scalar(C, t, C.Ap, C.bp, bcs, phi);
    relax_scalar(C.Ap, C.bp, phi, SS.relax);
    if (constrain) constrain_omega(C, C.Ap, C.bp);
    update_precond(C.Ap, SS.precond, Pre);
    const double r = solve_scalar(C, SS, SS.precond, phi, Pre);
    bound_field(*C.m, phi);
    return r;
}

// the diffusivity of a k-omega LKE equation: the cell field interpolated,
// boundary faces from nut's BCs (interpolate! + correct_boundaries!)
static void lke_face(Case& C, const std::vector<double>& cell, std::vector<double>& face) {
    interpolate(*C.m, cell, face);
    correct_boundaries(C, C.bcNut, &face, &cell, false);
}

// Re_upsilon^-1.30, Re_upsilon = sqrt(sqrt(2 nu^2 kl / y^2)) y / nu
static double lke_reu_pow(double nu, double kl, double y) {
    const double ru = (std::sqrt(std::sqrt(((2.0 * (nu * nu)) * kl) / (y * y))) * y) / nu;
    return det_pow(ru, -1.30);
}

// turbulence!(::KOmegaLKEModel) after grad!(gradU) and its limiter
// (RANS_kOmegaLKE.jl:262-474), rho = 1, the model's constants (:83-98)
static void komega_lke(Case& C) {
    const xcal_config& cf = C.cfg;
    const double nu = cf.nu, eta = C.lke_eta;
    const double Cmu = 0.09, Cw1 = 0.52, Cw2 = 0.0708, Ccrit = 76500.0, CSS = 1.45, Cv = 0.43, sk = 0.5,
                 sd = 0.125, skl = 0.0125, sw = 0.5;
    for (int i = 0; i < C.nC; ++i) {
        // :284-306.  S_dev = (g + g')/2 - tr(g)/3 I; S2 = 2 sum(S_dev.^2);
        // Omega = sqrt(2 sum(((g - g')/2).^2)); Pk = sum(g .* 2*S_dev), which
        // Julia reads as the matrix product (g .* 2) * S_dev (.* and * share
        // a precedence level, left to right).  Sums run over the column-major
        // entries from the first; a product entry is ((a1 b1 + a2 b2) + a3 b3)
        double G[3][3], Sd[3][3];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) G[a][b] = C.gradU[3 * a + b][i];
        const double divU = (G[0][0] + G[1][1]) + G[2][2];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
                Sd[a][b] = 0.5 * (G[a][b] + G[b][a]);
                if (a == b) Sd[a][b] = Sd[a][b] - divU / 3.0;
            }
        double s2 = 0.0, om = 0.0, pk = 0.0;
        for (int b = 0; b < 3; ++b)
            for (int a = 0; a < 3; ++a) {
                const double sq = Sd[a][b] * Sd[a][b];
                const double w = 0.5 * (G[a][b] - G[b][a]);
                double mab = (G[a][0] * 2.0) * Sd[0][b];
                mab = mab + (G[a][1] * 2.0) * Sd[1][b];
                mab = mab + (G[a][2] * 2.0) * Sd[2][b];
                if (a == 0 && b == 0) {
                    s2 = sq;
                    om = w * w;
                    pk = mab;
                } else {
                    s2 = s2 + sq;
                    om = om + w * w;
                    pk = pk + mab;
                }
            }
        C.divU[i] = divU;
        C.S2[i] = 2.0 * s2;
        C.Om[i] = std::sqrt(2.0 * om);
        C.Pk[i] = pk;
        const double u0 = C.U[0][i], u1 = C.U[1][i], u2 = C.U[2][i];
        C.normU[i] = std::sqrt((u0 * u0 + u1 * u1) + u2 * u2);
        C.ReL[i] = (jl_max(C.normU[i], std::sqrt(jl_eps(1.0))) * C.yw[i]) / nu;  // kMin = eps()
    }
    for (int i = 0; i < C.nC; ++i) {
        // :309-335 (Re_lambda^0.5 as sqrt)
        const double y = C.yw[i], kl = C.kl[i], S2 = C.S2[i];
        const double pru = lke_reu_pow(nu, kl, y), prl = std::sqrt(C.ReL[i]);
        const double uy = C.normU[i] / y;
        const double nutL1 = ((((eta * kl) * std::sqrt(S2)) * pru) * prl) / jl_max(S2, uy * uy);
        const double ReLt = jl_min((kl / jl_max(jl_min(nu, nutL1), 1e-15)) / jl_max(C.Om[i], 1e-15), 5000.0);
        C.gam[i] = jl_min(ReLt * ReLt, Ccrit) / Ccrit;
        C.PkL[i] = (((std::sqrt(S2) * eta) * kl) * pru) * prl;
        C.DkL[i] = (2.0 * nu) / (y * y);
        C.nueffS[i] = nu + (skl * std::sqrt(kl)) * y;
    }
    // kl: Time + Div(mdotf) - Lap(nueffkL) + Si(DkLf) == Source(PkL) (:165-173, :337-345)
    lke_face(C, C.nueffS, C.mueffl);
    const std::vector<Term> tl = {{T_TIME, 1.0, nullptr, cf.kl_schemes.time},
                                  {T_DIV, 1.0, &C.mdotf, cf.kl_schemes.divergence},
                                  {T_LAP, -1.0, &C.mueffl, 0},
                                  {T_SI, 1.0, &C.DkL, 0}};
    C.res_kl = lke_solve(C, tl, C.kl, C.PkL, C.bcKl, cf.kl_solver, C.Pkl, false);
    // cross diffusion (:371-374): grad omega with p's gradient scheme, grad k
    scalar_grad(C, C.omega, C.wfs, C.bcOmega, cf.p_schemes.gradient, C.gw);
    scalar_grad(C, C.k, C.kfs, C.bcK, cf.k_schemes.gradient, C.gk);
    for (int i = 0; i < C.nC; ++i) {  // :377-387
        const double w = C.omega[i], sw_ = jl_max(w, 1e-15);
        C.Pw[i] = Cw1 * C.Pk[i];
        C.Pw[i] = C.Pw[i] - (((2.0 / 3.0) * Cw1) * C.divU[i]) * w;
        C.Dw[i] = Cw2 * w;
        C.nueffS[i] = nu + sw * (C.k[i] / sw_);
        const double dkdw = (C.gk[0][i] * C.gw[0][i] + C.gk[1][i] * C.gw[1][i]) + C.gk[2][i] * C.gw[2][i];
        C.D2[i] = jl_max((sd / (sw_ * sw_)) * dkdw, 0.0);
    }
    // omega: Time + Div - Lap(nueffw) + Si(Dwf) - Si(dkdomegadx) == Source(Pw) (:185-195)
    lke_face(C, C.nueffS, C.mueffw);
    const std::vector<Term> tw = {{T_TIME, 1.0, nullptr, cf.omega_schemes.time},
                                  {T_DIV, 1.0, &C.mdotf, cf.omega_schemes.divergence},
                                  {T_LAP, -1.0, &C.mueffw, 0},
                                  {T_SI, 1.0, &C.Dw, 0},
                                  {T_SI, -1.0, &C.D2, 0}};
    C.res_omega = lke_solve(C, tw, C.omega, C.Pw, C.bcOmega, cf.omega_solver, C.Pww, true);
    for (int i = 0; i < C.nC; ++i) {  // :401-420
        const double w = C.omega[i], g = C.gam[i];
        const double sw_ = jl_max(w, 1e-15), sk_ = jl_max(C.k[i], 1e-15), snu = jl_max(nu, 1e-15);
        const double fv = 1.0 - det_exp_neg((-std::sqrt(sk_ / (snu * sw_))) / Cv);
        const double pku = ((fv * (sk_ / sw_)) * C.Pk[i]) * g;
        const double pkl = jl_min(pku, ((20.0 * Cmu) * sk_) * w);
        C.Pk[i] = pkl - ((2.0 / 3.0) * C.divU[i]) * C.k[i];
        C.Dk[i] = (Cmu * g) * w;
        C.nueffS[i] = nu + sk * (sk_ / sw_);
    }
    lke_face(C, C.nueffS, C.mueffk);
    kwall_production(C);  // correct_production! (:424)
    const std::vector<Term> tk = {{T_TIME, 1.0, nullptr, cf.k_schemes.time},
                                  {T_DIV, 1.0, &C.mdotf, cf.k_schemes.divergence},
                                  {T_LAP, -1.0, &C.mueffk, 0},
                                  {T_SI, 1.0, &C.Dk, 0}};
    C.res_k = lke_solve(C, tk, C.k, C.Pk, C.bcK, cf.k_solver, C.Pkw, false);
    for (int i = 0; i < C.nC; ++i) {  // :436-460
        const double kl = C.kl[i], y = C.yw[i], S2 = C.S2[i];
        const double sw_ = jl_max(C.omega[i], 1e-15), sk_ = jl_max(C.k[i], 1e-15);
        const double PkLv = (((std::sqrt(S2) * eta) * kl) * lke_reu_pow(nu, kl, y)) * std::sqrt(C.ReL[i]);
        const double uy = C.normU[i] / y;
        const double nuL = PkLv / jl_max(S2, uy * uy);
        const double x = ((CSS * nu) * C.Om[i]) / sk_;
        const double fSS = det_exp_neg(-(x * x));
        const double nuts = fSS * (sk_ / sw_);
        C.nut[i] = nuts + nuL;
    }
    interpolate(*C.m, C.nut, C.nutf);
    correct_boundaries(C, C.bcNut, &C.nutf, &C.nut, false);
    nutwall_correct(C);
}

void turbulence(Case& C) {
    grad_U(C);  // RANS_laminar.jl:73-79, LES_Smagorinsky.jl:117, RANS_kOmega.jl:167-168
    if (C.cfg.turbulence == XCAL_TURB_KOMEGA_LKE) komega_lke(C);
    if (C.cfg.turbulence == XCAL_TURB_KOMEGA_SST) komega_sst(C);
    if (C.cfg.turbulence == XCAL_TURB_KOMEGA) komega(C);
    if (C.cfg.turbulence == XCAL_TURB_KEQUATION) kequation(C);
    if (C.cfg.turbulence == XCAL_TURB_SMAGORINSKY) {
        // LES_Smagorinsky.jl:122-131
        for (int i = 0; i < C.nC; ++i) {
            double G[3][3];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) G[a][b] = C.gradU[3 * a + b][i];
            double S[3][3];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) S[a][b] = 0.5 * (G[a][b] + G[b][a]);
            // (2.0*S) . S over column-major linear index
            double acc = 0.0;
            bool first = true;
            for (int b = 0; b < 3; ++b)
                for (int a = 0; a < 3; ++a) {
                    double pr = (2.0 * S[a][b]) * S[a][b];
                    acc = first ? pr : acc + pr;
                    first = false;
                }
            double magS = std::sqrt(acc);
            C.nut[i] = C.Delta[i] * magS;
        }
        interpolate(*C.m, C.nut, C.nutf);
        correct_boundaries(C, C.bcNut, &C.nutf, &C.nut, false);
    }
    update_nueff(C);
}

double max_courant(Case& C) {  // Solvers_0_functions.jl:253-285 (Mesh3 / Mesh2 kernels)
    double mx = -std::numeric_limits<double>::infinity();
    for (int i = 0; i < C.nC; ++i) {
        V3 u{C.U[0][i], C.U[1][i], C.U[2][i]};
        double umag = norm(u);
        double V = C.m->cvol[i];
        double dx = C.m->dim == 2 ? std::sqrt(V) : std::pow(V, 1.0 / 3.0);
        double co = (umag * C.cfg.dt) / dx;
        C.cellsCourant[i] = co;
        mx = (i == 0) ? co : jl_max(mx, co);
    }
    return mx;
}

// one SIMPLE iteration (Solvers_1_SIMPLE.jl:164-240); returns converged
// nonorthogonal_face_correction (Solvers_1_SIMPLE.jl:267-318) with
// correction_weight (:320-333): over every internal face
//   w      = |c2 - f'| / |c2 - c1|, f' = c1 - q (c1 - c2),
//            q = ((xf - c1).(c2 - c1)) / ((c2 - c1).(c2 - c1))
//   gradi  = w grad[c1] + (1 - w) grad[c2]
//   gradf  = gradi + ((p2 - p1)/delta - gradi.e) e
//   T      = Sf - Ef, Sf = area n, Ef = dPN (|n|^2 / (dPN.n)) area
//   corr   = (rDf_f gradf) . T;  b[c1] += corr, b[c2] -= corr
// The reference adds with atomics (any order); here each cell adds its
// faces' corrections in its cell_faces order, which the product follows.
static double nonorth_face(const Case& C, int f) {
    const Mesh& m = *C.m;
    const int c1 = m.owner[f], c2 = m.neigh[f];
    const V3 xC = m.ccentre[c1], xN = m.ccentre[c2], xf = m.fcentre[f], n = m.fnormal[f], e = m.fe[f];
    const V3 c1f = xf - xC, c1c2 = xN - xC;
    const double q = dot(c1f, c1c2) / dot(c1c2, c1c2);
    const V3 fp = xC - q * (xC - xN);
    const double w = norm(xN - fp) / norm(xN - xC);
    const V3 dPN = xN - xC;
    const V3 g1 = {C.gradp[0][c1], C.gradp[1][c1], C.gradp[2][c1]};
    const V3 g2 = {C.gradp[0][c2], C.gradp[1][c2], C.gradp[2][c2]};
    const V3 gi = w * g1 + (1.0 - w) * g2;
    const double s = (C.p[c2] - C.p[c1]) / m.fdelta[f] - dot(gi, e);
    const V3 gf = gi + s * e;
    const double a = m.farea[f];
    const V3 Sf = a * n;
    const double nn = norm(n) * norm(n);
    const V3 Ef = (dPN * (nn / dot(dPN, n))) * a;
    const V3 T = Sf - Ef;
    return dot(C.rDf[f] * gf, T);
}

static void nonorthogonal_correction(Case& C) {
    const Mesh& m = *C.m;
    for (int i = 0; i < C.nC; ++i) {
        double bi = C.bp[i];
        for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
            const int f = m.cell_faces[k];
            const double corr = nonorth_face(C, f);
            bi = m.owner[f] == i ? bi + corr : bi - corr;
        }
        C.bp[i] = bi;
    }
}

bool simple_iteration(Case& C, double* res4) {
    if (!C.initialised) initial_calculations(C);
    C.iteration += 1;
    double r3[3];
    solve_equation_U(C, r3, nullptr);
    pressure_predictor(C, true);
    flux_divergence(C);
    C.prev = C.p;
    double rp = solve_equation_p(C, nullptr);
    explicit_relaxation_p(C, C.cfg.p_solver.relax);
    grad_p(C);
    // non-orthogonal correctors (Solvers_1_SIMPLE.jl:196-206): re-assemble
    // p with its BCs (no reference pressure), add the face corrections,
    // solve with the preconditioner of the first solve, relax against the
    // p of before the first solve, new gradient
    for (int k = 0; k < C.cfg.ncorrectors; ++k) {
        discretise_p(C);
        apply_bcs(C, false, 0);
        nonorthogonal_correction(C);
        rp = solve_system(C, false, 0, nullptr);
        explicit_relaxation_p(C, C.cfg.p_solver.relax);
        grad_p(C);
    }
    correct(C);
    turbulence(C);
    res4[0] = r3[0];
    res4[1] = r3[1];
    res4[2] = r3[2];
    res4[3] = rp;
    bool turb_conv = C.cfg.turbulence == XCAL_TURB_LAMINAR;
    // Uz enters the test on 3D meshes only (Solvers_1_SIMPLE.jl:220-223)
    const bool uz_conv = C.m->dim == 2 || r3[2] <= C.cfg.U_solver.convergence;
    return r3[0] <= C.cfg.U_solver.convergence && r3[1] <= C.cfg.U_solver.convergence && uz_conv &&
           rp <= C.cfg.p_solver.convergence && turb_conv;
}

// one PISO time step (Solvers_2_PISO.jl:108-187); returns the Courant number
double piso_step(Case& C, double* res4) {
    if (!C.initialised) initial_calculations(C);
    C.iteration += 1;
    C.time = C.time + C.cfg.dt;
    double r3[3];
    solve_equation_U(C, r3, nullptr);
    pressure_predictor(C, false);
    double rp = 0.0;
    int inner = C.cfg.inner_loops;
    for (int it = 1; it <= inner; ++it) {
        H(C);
        flux_divergence(C);
        C.prev = C.p;
        rp = solve_equation_p(C, nullptr);
        explicit_relaxation_p(C, it == inner ? 1.0 : C.cfg.p_solver.relax);
        grad_p(C);
        correct(C);
    }
    turbulence(C);
    double co = max_courant(C);
    res4[0] = r3[0];
    res4[1] = r3[1];
    res4[2] = r3[2];
    res4[3] = rp;
    return co;
}

// expose the internal steps to the C API
void o_discretise(Case& C, int eqn) {
    if (eqn == XCAL_EQN_U)
        discretise_U(C);
    else
        discretise_p(C);
}
void o_apply_bcs(Case& C, int eqn, int comp) {
    if (eqn == XCAL_EQN_U) {
        update_equation(C);
        apply_bcs(C, true, comp);
    } else {
        apply_bcs(C, false, 0);
    }
}
void o_relax(Case& C, int comp) { relax_diagdom(C, comp); }
void o_set_reference(Case& C) { set_reference(C); }
void o_update_precond(Case& C, int eqn) {
    if (eqn == XCAL_EQN_U)
        update_precond(C.AU, C.cfg.U_solver.precond, C.PU);
    else
        update_precond(C.Ap, C.cfg.p_solver.precond, C.Pp);
}
double o_solve_system(Case& C, int eqn, int comp, int* iters) {
    return solve_system(C, eqn == XCAL_EQN_U, comp, iters);
}
void o_grad_p(Case& C) { grad_p(C); }
void o_dilu(const CSR& A, std::vector<double>& D) { update_precond(A, XCAL_PRECOND_DILU, D); }
void o_dilu_ldiv(const CSR& A, const std::vector<double>& D, std::vector<double>& x, const std::vector<double>& b) {
    dilu_ldiv(A, D, x, b);
}

}  // namespace orc

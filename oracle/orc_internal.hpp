// orc_internal.hpp -- data structures of the CPU oracle (test infrastructure).
#pragma once
#include "orc_common.hpp"
#include "../include/xcal_b200.h"

#include <string>
#include <vector>

namespace orc {

// Mesh3 contract (src/Mesh/Mesh_0_types.jl), SoA, 0-based.
struct Mesh {
    int n_cells = 0, n_faces = 0, n_bfaces = 0, n_ifaces = 0;
    int dim = 3;  // 2 for a Mesh2
    std::vector<V3> points;
    std::vector<int> owner, neigh;  // ownerCells[1], ownerCells[2]
    std::vector<V3> fcentre, fnormal, fe;
    std::vector<double> farea, fdelta, fweight;
    std::vector<int> fn_off, face_nodes;
    std::vector<V3> ccentre;
    std::vector<double> cvol;
    std::vector<int> cf_off, cell_faces, cell_nsign, cell_neigh;
    std::vector<int> cn_off, cell_nodes;
    std::vector<int> bcell;  // boundary_cellsID
    std::vector<int> patch_start, patch_count;
};

Mesh* build_foam_mesh(int n_points, const double* points, int n_faces, const int* face_off,
                      const int* face_nodes, const int* owner, int n_ifaces, const int* neighbour,
                      int n_patches, const int* patch_nfaces);
Mesh* mesh_from_desc(const xcal_mesh_desc* d);
int construct_periodic(const Mesh* m, int patch1, int patch2, double tol, int* map1, int* map2,
                       double* distance);

// compressed sparse row matrix (SparseMatricesCSR semantics: sorted columns,
// duplicates merged)
struct CSR {
    int n = 0;
    std::vector<int> rowptr, colval;
    std::vector<double> nzval;
    std::vector<int> diag;  // diagonal_indices!
    const int* ord = nullptr;  // row order of the canonical reductions (null: 0..n-1)
    int find(int i, int j) const;  // spindex (0-based, -1 when absent)
};

struct BC {
    int type = 0;
    int patch = 0;
    double value[3] = {0, 0, 0};
    std::vector<double> face_values;  // DirichletFunction
    std::vector<int> face_map;        // periodic
    V3 distance{0, 0, 0};
    int partner_patch = -1;
    int start = 0, count = 0;  // IDs_range
    double wall[5] = {0, 0, 0, 0, 0};  // wall functions: kappa, beta1, cmu^0.25, yPlusLam, E
};

struct Krylov {
    // workspace vectors
    std::vector<double> x, r, p, q, z, v, s, t, dx, c;
    int niter = 0;
};

struct Case {
    const Mesh* m = nullptr;
    xcal_config cfg{};
    std::vector<BC> bcU, bcP, bcNut, bcK, bcOmega, bcY, bcKl;
    int nC = 0, nF = 0, nB = 0;

    // fields
    std::vector<double> U[3], p, mdotf, nueff, gradp[3], gradU[9], rD, Hv[3], divHv, nut, nutf, Uf[3], pf,
        rDf, Delta, prev, cellsCourant;
    // equations
    CSR AU, AU0, Ap;
    std::vector<double> bU[3], bp;
    // preconditioners
    std::vector<double> PU, Pp;  // Jacobi storage (1/|A_ii|) or DILU D
    Krylov kU, kp;
    // RANS{KOmega}: fields, production / dissipation, face diffusivities,
    // the k/omega preconditioner (shared, RANS_kOmega.jl:84-85), residuals
    std::vector<double> k, omega, Pk, Pw, Dk, Dw, mueffk, mueffw, Pkw;
    double res_k = 0.0, res_omega = 0.0;
    // RANS{KOmegaSST}: wall distance, blending, |S|, the second omega Si
    // coefficient, grad k / grad omega, their face values, omega's own
    // preconditioner
    std::vector<double> yw, F1, F2, Om, D2, gk[3], gw[3], kfs, wfs, Pww;
    // RANS{KOmegaLKE}: kl, its source and Si coefficient, the flow quantities
    // of one turbulence! call (Omega in Om, the cross diffusion in D2), the
    // intermittency gamma, a cell diffusivity and kl's face diffusivity and
    // preconditioner; eta from Tu
    std::vector<double> kl, PkL, DkL, S2, normU, divU, ReL, gam, nueffS, mueffl, Pkl;
    double res_kl = 0.0, lke_eta = 0.0;
    std::vector<int> rorder;  // morton_order of the cell centres
    double time = 0.0;
    bool initialised = false;
    int iteration = 0;
    std::string err;
};

Case* case_create(const Mesh* m, const xcal_config* cfg);

}  // namespace orc

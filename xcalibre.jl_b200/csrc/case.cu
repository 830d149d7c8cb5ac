// case.cu -- host orchestration of the hot path (mesh upload, equation
// patterns, BC tables, SIMPLE/PISO steps).  Host floating-point code is
// compiled without contraction so precomputed geometry matches the reference
// formulas bit for bit.
#include <algorithm>
#include <cmath>
#include <numeric>

#include "case.hpp"
#include "kernels.hpp"
#include "dev_common.cuh"

namespace xcal {

// ---------------------------------------------------------------------------
// views
// ---------------------------------------------------------------------------
MeshView DevMesh::view() const {
    MeshView v;
    v.nC = nC;
    v.nF = nF;
    v.nB = nB;
    v.owner = d_owner.p;
    v.neigh = d_neigh.p;
    v.area = d_area.p;
    v.delta = d_delta.p;
    v.weight = d_weight.p;
    v.Sx = d_Sx.p;
    v.Sy = d_Sy.p;
    v.Sz = d_Sz.p;
    v.nx = d_nx.p;
    v.ny = d_ny.p;
    v.nz = d_nz.p;
    v.Efmag = d_Ef.p;
    v.vol = d_vol.p;
    v.cf_off = d_cf_off.p;
    v.cf_face = d_cf_face.p;
    v.cf_nb = d_cf_nb.p;
    v.cf_sign = d_cf_sign.p;
    v.bf_off = d_bf_off.p;
    v.bf_face = d_bf_face.p;
    v.bcell = d_bcell.p;
    v.bcells = d_bcells.p;
    v.n_bcells = (int)bcells.size();
    return v;
}

CSRView Equation::view() const {
    CSRView v;
    v.n = n;
    v.slice = d_slice.p;
    v.len = d_len.p;
    v.colval = d_colval.p;
    v.diag = d_diag.p;
    v.trans = d_trans.p;
    v.cf_slot = d_cf_slot.p;
    v.fslot = d_fslot.p;
    return v;
}

int Equation::find(int i, int j) const {
    // rows are ordered by original column, not by storage column: linear scan
    int b = base(i);
    for (int k = 0; k < len[i]; ++k)
        if (colval[b + SELL_C * k] == j) return b + SELL_C * k;
    return -1;
}

BCView BCTable::view() const {
    BCView v;
    v.type = d_type.p;
    v.val = d_val.p;
    v.peer_face = d_peer_face.p;
    v.peer_cell = d_peer_cell.p;
    v.pw = d_pw.p;
    v.pwn = d_pwn.p;
    v.pEf = d_pEf.p;
    v.pDelta = d_pDelta.p;
    v.pwdelta = d_pwdelta.p;
    v.pNN = d_pNN.p;
    v.pNP = d_pNP.p;
    v.pPN = d_pPN.p;
    v.pe_off = d_pe_off.p;
    v.pe_face = d_pe_face.p;
    return v;
}

// ---------------------------------------------------------------------------
// mesh upload
// ---------------------------------------------------------------------------
// Storage (locality) order of cells: ascending 63-bit Morton key of the cell
// centre quantised to 21 bits per axis over the centres' bounding box, ties by
// index.  perm[s] = original cell stored at position s.  The canonical
// reduction tree runs over this order (the oracle uses the same definition).
void locality_order(int n, const double* c, std::vector<int>& perm) {
    double lo[3] = {c[0], c[1], c[2]}, hi[3] = {c[0], c[1], c[2]};
    for (int i = 1; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
            lo[d] = std::min(lo[d], c[3 * i + d]);
            hi[d] = std::max(hi[d], c[3 * i + d]);
        }
    auto spread = [](uint64_t v) {  // 21 bits -> every third bit
        v &= 0x1fffffULL;
        v = (v | (v << 32)) & 0x1f00000000ffffULL;
        v = (v | (v << 16)) & 0x1f0000ff0000ffULL;
        v = (v | (v << 8)) & 0x100f00f00f00f00fULL;
        v = (v | (v << 4)) & 0x10c30c30c30c30c3ULL;
        v = (v | (v << 2)) & 0x1249249249249249ULL;
        return v;
    };
    std::vector<uint64_t> key(n);
    for (int i = 0; i < n; ++i) {
        uint64_t q[3];
        for (int d = 0; d < 3; ++d) {
            double span = hi[d] - lo[d];
            double u = span > 0.0 ? (c[3 * i + d] - lo[d]) / span : 0.0;
            double t = u * 2097151.0;
            uint64_t qq = t > 0.0 ? (uint64_t)t : 0;
            q[d] = qq > 2097151ULL ? 2097151ULL : qq;
        }
        key[i] = spread(q[0]) | (spread(q[1]) << 1) | (spread(q[2]) << 2);
    }
    // (key, index) pairs sorted in place: the order of (key, then index),
    // without an indirect key lookup per comparison
    std::vector<std::pair<uint64_t, int>> kv(n);
    for (int i = 0; i < n; ++i) kv[i] = {key[i], i};
    std::sort(kv.begin(), kv.end());
    perm.resize(n);
    for (int i = 0; i < n; ++i) perm[i] = kv[i].second;
}

static DevMesh* upload_mesh_ordered(const xcal_mesh_desc* d, cudaStream_t s, std::unique_ptr<DevMesh> m);

DevMesh* upload_mesh(const xcal_mesh_desc* d0, cudaStream_t s) {
    if (!d0 || d0->n_cells <= 0 || d0->n_faces <= 0 || d0->n_bfaces < 0 || d0->n_bfaces > d0->n_faces)
        fail(XCAL_ERR_INVALID, "mesh: invalid sizes");
    if (!d0->face_owner || !d0->face_neigh || !d0->face_normal || !d0->face_area || !d0->face_delta ||
        !d0->face_weight || !d0->face_e || !d0->cell_volume || !d0->cell_faces_offset || !d0->cell_faces ||
        !d0->cell_nsign || !d0->cell_neighbours || !d0->boundary_cellsID || !d0->cell_centre || !d0->face_centre)
        fail(XCAL_ERR_INVALID, "mesh: missing array");
    const int nC = d0->n_cells, nF = d0->n_faces, nB = d0->n_bfaces;
    for (int f = 0; f < nF; ++f)
        if (d0->face_owner[f] < 0 || d0->face_owner[f] >= nC || d0->face_neigh[f] < 0 || d0->face_neigh[f] >= nC)
            fail(XCAL_ERR_INVALID, "mesh: face cell index out of range");
    for (int f = 0; f < nB; ++f)
        if (d0->boundary_cellsID[f] < 0 || d0->boundary_cellsID[f] >= nC)
            fail(XCAL_ERR_INVALID, "mesh: boundary_cellsID out of range");
    if (d0->cell_faces_offset[0] != 0 || d0->cell_faces_offset[nC] != 2 * (nF - nB))
        fail(XCAL_ERR_INVALID, "mesh: cell_faces_offset mismatch");
    for (int c = 0; c < nC; ++c)
        if (d0->cell_faces_offset[c + 1] < d0->cell_faces_offset[c])
            fail(XCAL_ERR_INVALID, "mesh: decreasing cell_faces_offset");
    for (int k = 0; k < 2 * (nF - nB); ++k)
        if (d0->cell_faces[k] < nB || d0->cell_faces[k] >= nF || d0->cell_neighbours[k] < 0 ||
            d0->cell_neighbours[k] >= nC)
            fail(XCAL_ERR_INVALID, "mesh: invalid cell_faces entry");
    auto m = std::make_unique<DevMesh>();
    AllocScope acc(&m->bytes);
    // cell order and face order (boundary faces keep their ids; internal faces
    // follow their storage owner/neighbour)
    locality_order(nC, d0->cell_centre, m->perm);
    m->inv.resize(nC);
    for (int st = 0; st < nC; ++st) m->inv[m->perm[st]] = st;
    // internal faces by (storage owner, storage neighbour, id): a counting
    // sort on the storage owner (ids ascending within each owner), then each
    // owner's few faces by (storage neighbour, id)
    m->fperm.resize(nF);
    std::iota(m->fperm.begin(), m->fperm.begin() + nB, 0);
    {
        std::vector<int> start(nC + 1, 0);
        for (int f = nB; f < nF; ++f) ++start[m->inv[d0->face_owner[f]] + 1];
        for (int c = 0; c < nC; ++c) start[c + 1] += start[c];
        std::vector<int> next(start.begin(), start.end() - 1);
        for (int f = nB; f < nF; ++f) m->fperm[nB + next[m->inv[d0->face_owner[f]]]++] = f;
        for (int c = 0; c < nC; ++c) {
            int* b = m->fperm.data() + nB + start[c];
            const int len = start[c + 1] - start[c];
            for (int a = 1; a < len; ++a) {  // insertion sort by (neighbour, id)
                const int f = b[a], nf = m->inv[d0->face_neigh[f]];
                int j = a - 1;
                while (j >= 0) {
                    const int g = b[j], ng = m->inv[d0->face_neigh[g]];
                    if (ng < nf || (ng == nf && g < f)) break;
                    b[j + 1] = g;
                    --j;
                }
                b[j + 1] = f;
            }
        }
    }
    m->finv.resize(nF);
    for (int fs = 0; fs < nF; ++fs) m->finv[m->fperm[fs]] = fs;
    // permuted copies of the Mesh3 arrays
    std::vector<int> owner(nF), neigh(nF), cf_off(nC + 1, 0), cf(2 * (nF - nB)), nsign(2 * (nF - nB)),
        nbr(2 * (nF - nB)), bcell(nB);
    std::vector<double> fc(3 * (size_t)nF), fnrm(3 * (size_t)nF), fe(3 * (size_t)nF), area(nF), delta(nF), weight(nF),
        cc(3 * (size_t)nC), vol(nC);
    for (int fs = 0; fs < nF; ++fs) {
        int f = m->fperm[fs];
        owner[fs] = m->inv[d0->face_owner[f]];
        neigh[fs] = m->inv[d0->face_neigh[f]];
        for (int k = 0; k < 3; ++k) {
            fc[3 * fs + k] = d0->face_centre[3 * f + k];
            fnrm[3 * fs + k] = d0->face_normal[3 * f + k];
            fe[3 * fs + k] = d0->face_e[3 * f + k];
        }
        area[fs] = d0->face_area[f];
        delta[fs] = d0->face_delta[f];
        weight[fs] = d0->face_weight[f];
    }
    for (int st = 0; st < nC; ++st) {
        int c = m->perm[st];
        for (int k = 0; k < 3; ++k) cc[3 * st + k] = d0->cell_centre[3 * c + k];
        vol[st] = d0->cell_volume[c];
        cf_off[st + 1] = cf_off[st] + (d0->cell_faces_offset[c + 1] - d0->cell_faces_offset[c]);
        int k2 = cf_off[st];
        for (int k = d0->cell_faces_offset[c]; k < d0->cell_faces_offset[c + 1]; ++k, ++k2) {
            cf[k2] = m->finv[d0->cell_faces[k]];
            nsign[k2] = d0->cell_nsign[k];
            nbr[k2] = m->inv[d0->cell_neighbours[k]];
        }
    }
    for (int f = 0; f < nB; ++f) bcell[f] = m->inv[d0->boundary_cellsID[f]];
    xcal_mesh_desc d = *d0;
    d.face_owner = owner.data();
    d.face_neigh = neigh.data();
    d.face_centre = fc.data();
    d.face_normal = fnrm.data();
    d.face_e = fe.data();
    d.face_area = area.data();
    d.face_delta = delta.data();
    d.face_weight = weight.data();
    d.cell_centre = cc.data();
    d.cell_volume = vol.data();
    d.cell_faces_offset = cf_off.data();
    d.cell_faces = cf.data();
    d.cell_nsign = nsign.data();
    d.cell_neighbours = nbr.data();
    d.boundary_cellsID = bcell.data();
    return upload_mesh_ordered(&d, s, std::move(m));
}

// the Mesh3 arrays already in storage order
static DevMesh* upload_mesh_ordered(const xcal_mesh_desc* d, cudaStream_t s, std::unique_ptr<DevMesh> m) {
    int nC = m->nC = d->n_cells, nF = m->nF = d->n_faces, nB = m->nB = d->n_bfaces;
    int nI = m->nI = nF - nB;
    m->owner.assign(d->face_owner, d->face_owner + nF);
    m->neigh.assign(d->face_neigh, d->face_neigh + nF);
    m->cf_off.assign(d->cell_faces_offset, d->cell_faces_offset + nC + 1);
    if (m->cf_off[0] != 0 || m->cf_off[nC] != 2 * nI) fail(XCAL_ERR_INVALID, "mesh: cell_faces_offset mismatch");
    for (int c = 0; c < nC; ++c)
        if (m->cf_off[c + 1] < m->cf_off[c]) fail(XCAL_ERR_INVALID, "mesh: decreasing cell_faces_offset");
    int nk = 2 * nI;
    m->cf_face.assign(d->cell_faces, d->cell_faces + nk);
    m->cf_nb.assign(d->cell_neighbours, d->cell_neighbours + nk);
    m->cf_sign.resize(nk);
    for (int k = 0; k < nk; ++k) {
        int sgn = d->cell_nsign[k];
        if ((sgn != 1 && sgn != -1) || m->cf_face[k] < nB || m->cf_face[k] >= nF || m->cf_nb[k] < 0 ||
            m->cf_nb[k] >= nC)
            fail(XCAL_ERR_INVALID, "mesh: invalid cell_faces entry");
        m->cf_sign[k] = (signed char)sgn;
    }
    for (int f = 0; f < nF; ++f)
        if (m->owner[f] < 0 || m->owner[f] >= nC || m->neigh[f] < 0 || m->neigh[f] >= nC)
            fail(XCAL_ERR_INVALID, "mesh: face cell index out of range");
    m->bcell.assign(d->boundary_cellsID, d->boundary_cellsID + nB);
    m->patch_start.assign(d->patch_start, d->patch_start + d->n_patches);
    m->patch_count.assign(d->patch_count, d->patch_count + d->n_patches);
    if (d->dim != 0 && d->dim != 2 && d->dim != 3) fail(XCAL_ERR_INVALID, "mesh: dim must be 0, 2 or 3");
    m->dim = d->dim == 2 ? 2 : 3;
    // cell -> boundary faces (ascending face id)
    std::vector<int> cnt(nC, 0);
    for (int f = 0; f < nB; ++f) {
        if (m->bcell[f] < 0 || m->bcell[f] >= nC) fail(XCAL_ERR_INVALID, "mesh: boundary_cellsID out of range");
        cnt[m->bcell[f]]++;
    }
    m->bf_off.assign(nC + 1, 0);
    for (int c = 0; c < nC; ++c) m->bf_off[c + 1] = m->bf_off[c] + cnt[c];
    m->bf_face.resize(nB);
    {
        std::vector<int> cur(m->bf_off.begin(), m->bf_off.end() - 1);
        for (int f = 0; f < nB; ++f) m->bf_face[cur[m->bcell[f]]++] = f;
    }
    for (int c = 0; c < nC; ++c)
        if (cnt[c]) m->bcells.push_back(c);
    // geometry
    m->vol.assign(d->cell_volume, d->cell_volume + nC);
    m->area.assign(d->face_area, d->face_area + nF);
    m->delta.assign(d->face_delta, d->face_delta + nF);
    std::vector<double> Sx(nF), Sy(nF), Sz(nF), Ef(nF);
    m->nxh.resize(nF);
    m->nyh.resize(nF);
    m->nzh.resize(nF);
    m->ex.resize(nF);
    m->ey.resize(nF);
    m->ez.resize(nF);
    m->fcx.resize(nF);
    m->fcy.resize(nF);
    m->fcz.resize(nF);
    for (int f = 0; f < nF; ++f) {
        double a = d->face_area[f];
        double nx = d->face_normal[3 * f], ny = d->face_normal[3 * f + 1], nz = d->face_normal[3 * f + 2];
        double ex = d->face_e[3 * f], ey = d->face_e[3 * f + 1], ez = d->face_e[3 * f + 2];
        m->nxh[f] = nx;
        m->nyh[f] = ny;
        m->nzh[f] = nz;
        m->ex[f] = ex;
        m->ey[f] = ey;
        m->ez[f] = ez;
        m->fcx[f] = d->face_centre[3 * f];
        m->fcy[f] = d->face_centre[3 * f + 1];
        m->fcz[f] = d->face_centre[3 * f + 2];
        // Sf = area*normal (flux!, green_gauss!)
        double sx = a * nx, sy = a * ny, sz = a * nz;
        Sx[f] = sx;
        Sy[f] = sy;
        Sz[f] = sz;
        // |E_f| with Sf = (ns*area)*normal and e' = ns*e; independent of the
        // sign ns (Discretise_1_schemes.jl:77-93)
        double ss = sx * sx + sy * sy + sz * sz;
        double se = sx * ex + sy * ey + sz * ez;
        double r = ss / se;
        double efx = r * ex, efy = r * ey, efz = r * ez;
        Ef[f] = std::sqrt(efx * efx + efy * efy + efz * efz);
    }
    m->ccx.resize(nC);
    m->ccy.resize(nC);
    m->ccz.resize(nC);
    for (int c = 0; c < nC; ++c) {
        m->ccx[c] = d->cell_centre[3 * c];
        m->ccy[c] = d->cell_centre[3 * c + 1];
        m->ccz[c] = d->cell_centre[3 * c + 2];
    }
    // device copies
    m->d_owner.upload(m->owner, s);
    m->d_neigh.upload(m->neigh, s);
    m->d_cf_off.upload(m->cf_off, s);
    m->d_cf_face.upload(m->cf_face, s);
    m->d_cf_nb.upload(m->cf_nb, s);
    m->d_cf_sign.upload(m->cf_sign, s);
    m->d_bf_off.upload(m->bf_off, s);
    m->d_bf_face.upload(m->bf_face, s);
    m->d_bcell.upload(m->bcell, s);
    m->d_bcells.upload(m->bcells, s);
    m->d_area.upload(m->area, s);
    m->d_delta.upload(m->delta, s);
    m->d_weight.upload(d->face_weight, nF, s);
    m->d_Sx.upload(Sx, s);
    m->d_Sy.upload(Sy, s);
    m->d_Sz.upload(Sz, s);
    m->d_nx.upload(m->nxh, s);
    m->d_ny.upload(m->nyh, s);
    m->d_nz.upload(m->nzh, s);
    m->d_Ef.upload(Ef, s);
    m->d_vol.upload(m->vol, s);
    m->d_perm.upload(m->perm, s);
    m->d_inv.upload(m->inv, s);
    m->d_fperm.upload(m->fperm, s);
    m->d_finv.upload(m->finv, s);
    XCAL_CUDA(cudaStreamSynchronize(s));
    return m.release();
}

// Off-diagonal SELL-32 storage of an equation for the folded FP32 CG
// (cg_folded.cu): per 32-row slice, width = the longest row's off-diagonal
// count; each row keeps its entries' order with the diagonal left out; map =
// the entry's slot in E's own storage.  When padding every slice to the
// longest row of all costs at most a quarter more slots (hexahedral meshes:
// 6 per row), every slice takes that width and padding slots hold the row's
// own column (value 0), so the kernel reads a fixed number of slots per row
// at computed addresses.  Built once, on first use.
static void build_fold(Equation& E, cudaStream_t s, bool uniform_ok) {
    if (E.fold_built && E.fold_uniform_ok == uniform_ok) return;
    E.fold_uniform_ok = uniform_ok;
    const int n = E.n, nsl = (n + SELL_C - 1) / SELL_C;
    std::vector<int> fsl(nsl + 1, 0);
    std::vector<unsigned char> flen((size_t)nsl * SELL_C, 0);  // whole slices
    for (int r = 0; r < n; ++r) {
        if (E.diag[r] < 0) fail(XCAL_ERR_INVALID, "folded CG: a row has no diagonal entry");
        if (E.len[r] - 1 > 127) fail(XCAL_ERR_UNSUPPORTED, "folded CG: a row has more than 127 off-diagonals");
        flen[r] = (unsigned char)(E.len[r] - 1);
    }
    long narrow = 0;
    int W = 0;
    for (int sl = 0; sl < nsl; ++sl) {
        int w = 0;
        for (int r = sl * SELL_C; r < std::min(n, (sl + 1) * SELL_C); ++r) w = std::max(w, (int)flen[r]);
        fsl[sl + 1] = fsl[sl] + SELL_C * w;
        narrow += (long)SELL_C * w;
        W = std::max(W, w);
    }
    const bool uniform = uniform_ok && W > 0 && (long)nsl * SELL_C * W <= narrow + narrow / 4 &&
                         (long)nsl * SELL_C * W <= 2147483647L;
    if (uniform)
        for (int sl = 0; sl <= nsl; ++sl) fsl[sl] = SELL_C * W * sl;
    const long nslots = fsl[nsl];
    std::vector<int> fcol(nslots, 0), fmap(nslots, 0);
    for (int r = 0; r < n; ++r) {
        const int b = E.base(r), fb = fsl[r / SELL_C] + r % SELL_C;
        if (uniform)
            for (int m = flen[r]; m < W; ++m) fcol[fb + SELL_C * m] = r;  // padding: own column, value 0
        int m = 0;
        for (int k = 0; k < E.len[r]; ++k) {
            const int slot = b + SELL_C * k;
            if (slot == E.diag[r]) continue;
            fcol[fb + SELL_C * m] = E.colval[slot];
            fmap[fb + SELL_C * m] = slot;
            ++m;
        }
    }
    E.f_slice.upload(fsl, s);
    E.f_len.upload(flen, s);
    E.f_col.upload(fcol, s);
    E.f_map.upload(fmap, s);
    E.f_val.alloc(nslots);
    E.f_val.zero(s);
    XCAL_CUDA(cudaStreamSynchronize(s));  // the host vectors go out of scope
    E.f_W = uniform ? W : 0;
    E.fold_built = true;
}

// ---------------------------------------------------------------------------
// equation pattern (sparse_matrix_connectivity + extend_matrix + sparsecsr)
// ---------------------------------------------------------------------------
void build_equation(Equation& E, const DevMesh& m, const std::vector<xcal_bc>& bcs, int nvec,
                           bool need_dilu, cudaStream_t s) {
    int n = E.n = m.nC;
    E.use_block = n <= DILU_BLOCK_MAX_ROWS;
    std::vector<std::vector<int>> extra(n);
    for (const xcal_bc& bc : bcs) {
        if (bc.type != XCAL_BC_PERIODIC_PARENT) continue;
        E.has_periodic = true;
        int start = m.patch_start[bc.patch], count = m.patch_count[bc.patch];
        for (int i = 0; i < count; ++i) {
            int f1 = start + i, f2 = bc.face_map[i];
            int c1 = m.owner[f1], c2 = m.owner[f2];
            extra[c1].push_back(c2);
            extra[c2].push_back(c1);
        }
    }
    // rows are stored in storage order; the entries of a row keep the
    // reference's order (ascending ORIGINAL column), so row sums are unchanged
    std::vector<std::vector<int>> rows_s(n);
    std::vector<int> row;
    E.nnz_csr = 0;
    for (int c = 0; c < n; ++c) {
        row.clear();
        row.push_back(m.perm[c]);
        for (int k = m.cf_off[c]; k < m.cf_off[c + 1]; ++k) row.push_back(m.perm[m.cf_nb[k]]);
        for (int j : extra[c]) row.push_back(m.perm[j]);
        std::sort(row.begin(), row.end());
        row.erase(std::unique(row.begin(), row.end()), row.end());
        if (row.size() > 255) fail(XCAL_ERR_UNSUPPORTED, "a matrix row has more than 255 entries");
        for (int j : row) rows_s[c].push_back(m.inv[j]);
        E.nnz_csr += (long)row.size();
    }
    // SELL-32 layout: slice width = longest row of the slice
    int nsl = (n + SELL_C - 1) / SELL_C;
    E.slice.assign(nsl + 1, 0);
    E.len.resize(n);
    for (int sl = 0; sl < nsl; ++sl) {
        size_t w = 0;
        for (int r = sl * SELL_C; r < std::min(n, (sl + 1) * SELL_C); ++r) w = std::max(w, rows_s[r].size());
        if ((long)E.slice[sl] + (long)SELL_C * (long)w > 2147483647L) fail(XCAL_ERR_UNSUPPORTED, "matrix too large");
        E.slice[sl + 1] = E.slice[sl] + SELL_C * (int)w;
    }
    E.nnz = E.slice[nsl];
    E.colval.assign(E.nnz, 0);
    for (int r = 0; r < n; ++r) {
        E.len[r] = (unsigned char)rows_s[r].size();
        int b = E.base(r);
        for (int k = 0; k < E.len[r]; ++k) E.colval[b + SELL_C * k] = rows_s[r][k];
        for (int k = E.len[r]; b + SELL_C * k < E.slice[r / SELL_C + 1]; ++k) E.colval[b + SELL_C * k] = r;
    }
    rows_s.clear();
    rows_s.shrink_to_fit();
    E.diag.resize(n);
    for (int c = 0; c < n; ++c) E.diag[c] = E.find(c, c);
    std::vector<int> trans(E.nnz, 0), cf_slot(m.cf_face.size()), fslot(m.nI);
    for (int c = 0; c < n; ++c)
        for (int k = m.cf_off[c]; k < m.cf_off[c + 1]; ++k) cf_slot[k] = E.find(c, m.cf_nb[k]);
    for (int f = m.nB; f < m.nF; ++f) fslot[f - m.nB] = E.find(m.owner[f], m.neigh[f]);
    // trans: the slot of (col, row) per entry.  The diagonal is its own; an
    // internal face pairs (owner, neigh) with (neigh, owner); the periodic
    // couplings (no face) are looked up row by row
    {
        std::vector<char> set(E.nnz, 0);
        for (int c = 0; c < n; ++c) {
            trans[E.diag[c]] = E.diag[c];
            set[E.diag[c]] = 1;
        }
        for (int f = m.nB; f < m.nF; ++f) {
            const int a = fslot[f - m.nB], b = E.find(m.neigh[f], m.owner[f]);
            trans[a] = b;
            trans[b] = a;
            set[a] = set[b] = 1;
        }
        for (int i = 0; i < n; ++i)
            for (int k = 0, b = E.base(i); k < E.len[i]; ++k) {
                const int e = b + SELL_C * k;
                if (!set[e]) trans[e] = E.find(E.colval[e], i);
            }
    }
    E.d_slice.upload(E.slice, s);
    E.d_len.upload(E.len, s);
    E.d_colval.upload(E.colval, s);
    E.d_diag.upload(E.diag, s);
    E.d_trans.upload(trans, s);
    E.d_cf_slot.upload(cf_slot, s);
    E.d_fslot.upload(fslot, s);
    E.nz.alloc(E.nnz);
    E.nz.zero(s);
    if (E.has_periodic) {
        E.nz0.alloc(E.nnz);
        E.nz0.zero(s);
    }
    E.diag0.alloc(n);
    E.diag0.zero(s);
    E.P.alloc(n);
    E.P.zero(s);
    for (int d = 0; d < nvec; ++d) {
        E.b[d].alloc(n);
        E.b[d].zero(s);
    }
    if (need_dilu) {
        // dependency levels of the lower (ascending) and upper (descending)
        // triangular sweeps in the ORIGINAL numbering
        // (rows visited in ascending original index; lvl indexed by storage row)
        std::vector<int> lvl(n, 0);
        int maxl = 0;
        for (int io = 0; io < n; ++io) {
            int i = m.inv[io];
            int l = 0;
            for (int e = E.base(i); e < E.diag[i]; e += SELL_C) l = std::max(l, lvl[E.colval[e]] + 1);
            lvl[i] = l;
            maxl = std::max(maxl, l);
        }
        std::vector<int> rows(n);
        E.lower_off.assign(maxl + 2, 0);
        for (int i = 0; i < n; ++i) E.lower_off[lvl[i] + 1]++;
        for (int l = 0; l <= maxl; ++l) E.lower_off[l + 1] += E.lower_off[l];
        {
            std::vector<int> cur(E.lower_off.begin(), E.lower_off.end() - 1);
            for (int i = 0; i < n; ++i) rows[cur[lvl[i]]++] = i;
        }
        E.d_lower_rows.upload(rows, s);
        E.h_lower_rows = rows;
        E.d_lower_off.upload(E.lower_off, s);
        std::fill(lvl.begin(), lvl.end(), 0);
        maxl = 0;
        for (int io = n - 1; io >= 0; --io) {
            int i = m.inv[io];
            int l = 0;
            for (int e = E.diag[i] + SELL_C; e < E.base(i) + SELL_C * E.len[i]; e += SELL_C)
                l = std::max(l, lvl[E.colval[e]] + 1);
            lvl[i] = l;
            maxl = std::max(maxl, l);
        }
        E.upper_off.assign(maxl + 2, 0);
        for (int i = 0; i < n; ++i) E.upper_off[lvl[i] + 1]++;
        for (int l = 0; l <= maxl; ++l) E.upper_off[l + 1] += E.upper_off[l];
        {
            std::vector<int> cur(E.upper_off.begin(), E.upper_off.end() - 1);
            for (int i = 0; i < n; ++i) rows[cur[lvl[i]]++] = i;
        }
        E.d_upper_rows.upload(rows, s);
        E.h_upper_rows = rows;
        E.d_upper_off.upload(E.upper_off, s);
        // level-ordered copies of the strictly lower / upper entries
        for (int tri = 0; tri < 2; ++tri) {
            const std::vector<int>& order = tri == 0 ? E.h_lower_rows : E.h_upper_rows;
            LevelSell& L = tri == 0 ? E.lsell : E.usell;
            const int nsl2 = (n + SELL_C - 1) / SELL_C;
            std::vector<int> sl(nsl2 + 1, 0);
            std::vector<unsigned char> cnt(n);
            for (int k = 0; k < n; ++k) {
                int i = order[k];
                int c = tri == 0 ? (E.diag[i] - E.base(i)) / SELL_C : (int)E.len[i] - 1 - (E.diag[i] - E.base(i)) / SELL_C;
                cnt[k] = (unsigned char)c;
            }
            for (int sidx = 0; sidx < nsl2; ++sidx) {
                int w = 0;
                for (int k = sidx * SELL_C; k < std::min(n, sidx * SELL_C + SELL_C); ++k) w = std::max(w, (int)cnt[k]);
                sl[sidx + 1] = sl[sidx] + SELL_C * w;
            }
            L.nslots = sl[nsl2];
            std::vector<int> col(std::max(L.nslots, 1L)), src(std::max(L.nslots, 1L));
            for (int k = 0; k < n; ++k) {
                int i = order[k];
                int b0 = sl[k / SELL_C] + k % SELL_C;
                int first = tri == 0 ? E.base(i) : E.diag[i] + SELL_C;
                int w = (sl[k / SELL_C + 1] - sl[k / SELL_C]) / SELL_C;
                for (int j = 0; j < w; ++j) {
                    int e = b0 + SELL_C * j;
                    if (j < cnt[k]) {
                        src[e] = first + SELL_C * j;
                        col[e] = E.colval[src[e]];
                    } else {  // padding: never read
                        src[e] = E.diag[i];
                        col[e] = i;
                    }
                }
            }
            L.slice.upload(sl, s);
            L.cnt.upload(cnt, s);
            L.col.upload(col, s);
            L.src.upload(src, s);
            if (tri == 0) {  // what the DILU factor reads besides: a_ji's slot, each row's diagonal slot
                std::vector<int> tsrc(src.size()), dslot(n);
                for (size_t e = 0; e < src.size(); ++e) tsrc[e] = trans[src[e]];
                for (int k = 0; k < n; ++k) dslot[k] = E.diag[order[k]];
                L.tsrc.upload(tsrc, s);
                L.dslot.upload(dslot, s);
            }
            L.val.alloc(std::max(L.nslots, 1L));
            L.val.zero(s);
            if (tri == 0) {
                L.dinv.alloc(std::max(L.nslots, 1L));
                L.dinv.zero(s);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// BC tables
// ---------------------------------------------------------------------------
void build_bc_table(BCTable& T, const DevMesh& m, const xcal_bc* bcs, int nbc, int ncomp, const Equation* E,
                           cudaStream_t s) {
    int nB = m.nB;
    T.src.assign(bcs, bcs + nbc);
    T.type.assign(nB, 0);
    T.val.assign(3 * (size_t)nB, 0.0);
    std::vector<int> peer_face(nB, -1), peer_cell(nB, -1), pNN(nB, -1), pNP(nB, -1), pPN(nB, -1);
    std::vector<double> pw(nB, 0.0), pwn(nB, 0.0), pEf(nB, 0.0), pDelta(nB, 0.0), pwdelta(nB, 0.0);
    int np = (int)m.patch_start.size();
    for (int b = 0; b < nbc; ++b) {
        const xcal_bc& bc = bcs[b];
        if (bc.patch < 0 || bc.patch >= np) fail(XCAL_ERR_INVALID, "bc: patch index out of range");
        if (bc.type < XCAL_BC_DIRICHLET || bc.type > XCAL_BC_NUT_WALL)
            fail(XCAL_ERR_INVALID, "bc: unknown type");
        if (ncomp == 3 && bc.type == XCAL_BC_NEUMANN)
            fail(XCAL_ERR_UNSUPPORTED, "Neumann boundary condition for vector fields is not implemented");
        int start = m.patch_start[bc.patch], count = m.patch_count[bc.patch];
        for (int i = 0; i < count; ++i) {
            int f = start + i;
            if (T.type[f] != 0) continue;  // first BC listed for a face wins
            T.type[f] = (signed char)bc.type;
            for (int c = 0; c < 3; ++c) {
                double v = bc.value[c];
                if (bc.type == XCAL_BC_DIRICHLET_FUNCTION) {
                    if (!bc.face_values) fail(XCAL_ERR_INVALID, "DirichletFunction without face values");
                    v = c < ncomp ? bc.face_values[(size_t)ncomp * i + c] : 0.0;
                }
                T.val[3 * (size_t)f + c] = v;
            }
            if (bc.type == XCAL_BC_PERIODIC || bc.type == XCAL_BC_PERIODIC_PARENT) {
                if (!bc.face_map) fail(XCAL_ERR_INVALID, "periodic BC without face_map");
                int pf = bc.face_map[i];
                if (pf < 0 || pf >= nB) fail(XCAL_ERR_INVALID, "periodic face_map out of range");
                T.has_periodic = true;
                peer_face[f] = pf;
                int c1 = m.owner[f], c2 = m.owner[pf];
                peer_cell[f] = c2;
                if (bc.type == XCAL_BC_PERIODIC_PARENT) {
                    double dx = bc.distance[0], dy = bc.distance[1], dz = bc.distance[2];
                    // periodic.jl:282-296, 336-346; periodic_interpolation.jl:58-66
                    double C1x = m.ccx[c1], C1y = m.ccy[c1], C1z = m.ccz[c1];
                    double C2x = m.ccx[c2] - dx, C2y = m.ccy[c2] - dy, C2z = m.ccz[c2] - dz;
                    double Pfx = m.fcx[f] - C1x, Pfy = m.fcy[f] - C1y, Pfz = m.fcz[f] - C1z;
                    double PNx = C2x - C1x, PNy = C2y - C1y, PNz = C2z - C1z;
                    double nx = m.nxh[f], ny = m.nyh[f], nz = m.nzh[f];
                    double wn = (Pfx * nx + Pfy * ny + Pfz * nz) / (PNx * nx + PNy * ny + PNz * nz);
                    pwn[f] = wn;
                    pw[f] = 1.0 - wn;
                    pDelta[f] = std::sqrt(PNx * PNx + PNy * PNy + PNz * PNz);
                    double a = m.area[f];
                    double sx = a * nx, sy = a * ny, sz = a * nz;
                    double ss = sx * sx + sy * sy + sz * sz;
                    double se = sx * m.ex[f] + sy * m.ey[f] + sz * m.ez[f];
                    double r = ss / se;
                    double efx = r * m.ex[f], efy = r * m.ey[f], efz = r * m.ez[f];
                    pEf[f] = std::sqrt(efx * efx + efy * efy + efz * efz);
                    pwdelta[f] = m.delta[pf] / (m.delta[f] + m.delta[pf]);  // Solvers_1_SIMPLE.jl:463
                    if (E) {
                        // the periodic slots start from 0 at every assembly:
                        // a pair that is also an internal neighbour (or the
                        // cell itself) would share a slot with the face loop
                        if (c1 == c2) fail(XCAL_ERR_UNSUPPORTED, "periodic pair maps a cell onto itself");
                        for (int k = m.cf_off[c1]; k < m.cf_off[c1 + 1]; ++k)
                            if (m.cf_nb[k] == c2)
                                fail(XCAL_ERR_UNSUPPORTED, "periodic partners are also internal neighbours");
                        pNN[f] = E->find(c2, c2);
                        pNP[f] = E->find(c2, c1);
                        pPN[f] = E->find(c1, c2);
                        if (pNN[f] < 0 || pNP[f] < 0 || pPN[f] < 0)
                            fail(XCAL_ERR_INVALID, "periodic pair missing from the matrix pattern");
                    }
                }
            }
        }
    }
    T.d_type.upload(T.type, s);
    T.d_val.upload(T.val, s);
    T.d_peer_face.upload(peer_face, s);
    T.d_peer_cell.upload(peer_cell, s);
    T.d_pw.upload(pw, s);
    T.d_pwn.upload(pwn, s);
    T.d_pEf.upload(pEf, s);
    T.d_pDelta.upload(pDelta, s);
    T.d_pwdelta.upload(pwdelta, s);
    T.d_pNN.upload(pNN, s);
    T.d_pNP.upload(pNP, s);
    T.d_pPN.upload(pPN, s);
    T.h_pNP = pNP;
    T.h_pPN = pPN;
    // partner events: cell owner[face_map[f]] of every parent face f
    if (T.has_periodic) {
        const int nC = m.nC;
        std::vector<int> off(nC + 1, 0), face;
        for (int f = 0; f < nB; ++f)
            if (T.type[f] == XCAL_BC_PERIODIC_PARENT) ++off[peer_cell[f] + 1];
        for (int c = 0; c < nC; ++c) off[c + 1] += off[c];
        face.assign(off[nC], 0);
        std::vector<int> pos(off.begin(), off.end() - 1);
        for (int f = 0; f < nB; ++f)  // ascending f: each cell's list is ascending
            if (T.type[f] == XCAL_BC_PERIODIC_PARENT) face[pos[peer_cell[f]]++] = f;
        T.d_pe_off.upload(off, s);
        T.d_pe_face.upload(face, s);
    }
}

// ---------------------------------------------------------------------------
// case
// ---------------------------------------------------------------------------
Case::Case(xcal_ctx* c, const DevMesh* m, const xcal_config* cf) : ctx(c), mesh(m), cfg(*cf) {
    AllocScope acc(&bytes);
    if (cfg.U_solver.relax <= 0.0 || cfg.p_solver.relax <= 0.0) fail(XCAL_ERR_INVALID, "relax must be > 0");
    if (cfg.algorithm == XCAL_ALGO_PISO && cfg.dt <= 0.0) fail(XCAL_ERR_INVALID, "PISO needs dt > 0");
    if (cfg.ncorrectors < 0) fail(XCAL_ERR_INVALID, "ncorrectors must be >= 0");
    if (cfg.ncorrectors > 0 && cfg.algorithm != XCAL_ALGO_SIMPLE)
        fail(XCAL_ERR_UNSUPPORTED, "non-orthogonal correctors are implemented for SIMPLE");
    if (cfg.precision != XCAL_PREC_FP64 && cfg.precision != XCAL_PREC_MIXED)
        fail(XCAL_ERR_INVALID, "unknown precision mode");
    for (auto* ss : {&cfg.U_solver, &cfg.p_solver}) {
        if (ss->solver != XCAL_SOLVER_CG && ss->solver != XCAL_SOLVER_BICGSTAB)
            fail(XCAL_ERR_UNSUPPORTED, "solver must be Cg or Bicgstab");
        if (ss->precond < XCAL_PRECOND_NONE || ss->precond > XCAL_PRECOND_DILU)
            fail(XCAL_ERR_UNSUPPORTED, "unknown preconditioner");
    }
    XCAL_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    for (auto& e : ev) XCAL_CUDA(cudaEventCreate(&e));
    XCAL_CUDA(cudaMallocHost(&h_S, 2 * sizeof(KScalars)));
    XCAL_CUDA(cudaMallocHost(&h_res, 16 * sizeof(double)));
    int nC = m->nC, nF = m->nF;
    std::vector<xcal_bc> bU(cfg.bc_U, cfg.bc_U + cfg.n_bc_U), bP(cfg.bc_p, cfg.bc_p + cfg.n_bc_p);
    build_equation(U, *m, bU, 3, cfg.U_solver.precond == XCAL_PRECOND_DILU, stream);
    // the p system's storage also carries k, omega, kl and the wall distance:
    // its DILU levels are needed when any solve on it is DILU-preconditioned
    auto dilu = [](const xcal_solver_setup& ss) { return ss.precond == XCAL_PRECOND_DILU; };
    const bool p_dilu = dilu(cfg.p_solver) || (has_k() && dilu(cfg.k_solver)) ||
                        (rans_kw() && dilu(cfg.omega_solver)) || (lke() && dilu(cfg.kl_solver)) ||
                        (has_y() && dilu(cfg.y_solver));
    build_equation(P, *m, bP, 1, p_dilu, stream);
    build_bc_table(bcU, *m, cfg.bc_U, cfg.n_bc_U, 3, &U, stream);
    build_bc_table(bcP, *m, cfg.bc_p, cfg.n_bc_p, 1, &P, stream);
    build_bc_table(bcNut, *m, cfg.bc_nut, cfg.n_bc_nut, 1, nullptr, stream);
    for (const BCTable* T : {&bcU, &bcP})
        for (const xcal_bc& bc : T->src)
            if (bc.type == XCAL_BC_OMEGA_WALL || bc.type == XCAL_BC_K_WALL || bc.type == XCAL_BC_NUT_WALL)
                fail(XCAL_ERR_INVALID, "wall functions apply to k, omega and nut only");
    for (const xcal_bc& bc : bcNut.src)
        if (bc.type == XCAL_BC_OMEGA_WALL || bc.type == XCAL_BC_K_WALL)
            fail(XCAL_ERR_INVALID, "OmegaWallFunction / KWallFunction do not apply to nut");
    if (keq()) {
        // LES{KEquation}: the subgrid k equation shares the p system (its
        // periodic pairs resolve to the p system's partner slots)
        build_bc_table(bcK, *m, cfg.bc_k, cfg.n_bc_k, 1, &P, stream);
        for (DBuf<double>* b : {&kfld, &Pk, &Dk, &Dw, &kwtmp}) {
            b->alloc(m->nC);
            b->zero(stream);
        }
        build_wall_table(*m);
    } else if (rans_kw()) {
        // RANS{KOmega} / RANS{KOmegaSST}: k / omega share the p system (their
        // periodic pairs resolve to the p system's partner slots)
        build_bc_table(bcK, *m, cfg.bc_k, cfg.n_bc_k, 1, &P, stream);
        build_bc_table(bcOmega, *m, cfg.bc_omega, cfg.n_bc_omega, 1, &P, stream);
        if (has_y()) build_bc_table(bcY, *m, cfg.bc_y, cfg.n_bc_y, 1, &P, stream);
        for (DBuf<double>* b : {&kfld, &omega, &Pk, &Pw, &Dk, &Dw, &kwtmp}) {
            b->alloc(m->nC);
            b->zero(stream);
        }
        if (lke()) {
            // RANS{KOmegaLKE}: kl on the p system too; eta from Tu (RANS_kOmegaLKE.jl:97)
            if (!(cfg.lke_Tu >= 0.0)) fail(XCAL_ERR_INVALID, "RANS{KOmegaLKE} needs Tu >= 0");
            build_bc_table(bcKl, *m, cfg.bc_kl, cfg.n_bc_kl, 1, &P, stream);
            for (DBuf<double>* b : {&kl, &PkL, &DkL, &S2b, &normUb, &divUb, &ReLb, &gam, &nueffS}) {
                b->alloc(m->nC);
                b->zero(stream);
            }
            fmu.alloc(m->nF);
            fmu.zero(stream);
            lke_eta = 0.02974 * det_tanh_pos(59.79 * det_pow(cfg.lke_Tu, 1.191) + 1.65e-13);
        }
        if (has_y()) {
            for (DBuf<double>* b : {&yw, &yphi, &F1b, &F2b, &Omb, &D2b, &gkv[0], &gkv[1], &gkv[2], &gwv[0], &gwv[1],
                                    &gwv[2]}) {
                b->alloc(m->nC);
                b->zero(stream);
            }
            fscr.alloc(m->nF);
        }
        build_wall_table(*m);
    } else if (cfg.turbulence != XCAL_TURB_LAMINAR && cfg.turbulence != XCAL_TURB_SMAGORINSKY) {
        fail(XCAL_ERR_INVALID, "unknown turbulence model");
    }
    cfg.bc_U = cfg.bc_p = cfg.bc_nut = nullptr;  // not retained
    cfg.bc_kl = nullptr;
    for (int d = 0; d < 3; ++d) {
        Uc[d].alloc(nC);
        gradp[d].alloc(nC);
        Hv[d].alloc(nC);
        Uf[d].alloc(nF);
    }
    for (int d = 0; d < 9; ++d) gradU[d].alloc(nC);
    for (DBuf<double>* b : {&p, &rD, &divHv, &nut, &Delta, &prev, &courant, &dx13}) b->alloc(nC);
    for (DBuf<double>* b : {&mdot, &nueff, &nutf, &pf, &rDf}) b->alloc(nF);
    if (cfg.ncorrectors > 0) build_nonorth(*m, stream);
    for (int g : {cfg.U_schemes.gradient, cfg.p_schemes.gradient})
        if (g != XCAL_GRAD_GAUSS && g != XCAL_GRAD_MIDPOINT) fail(XCAL_ERR_INVALID, "unknown gradient scheme");
    if (has_y())
        for (int g : {cfg.k_schemes.gradient, cfg.y_schemes.gradient})
            if (g != XCAL_GRAD_GAUSS && g != XCAL_GRAD_MIDPOINT) fail(XCAL_ERR_INVALID, "unknown gradient scheme");
    if (cfg.U_schemes.gradient == XCAL_GRAD_MIDPOINT || cfg.p_schemes.gradient == XCAL_GRAD_MIDPOINT ||
        (has_y() && (cfg.k_schemes.gradient == XCAL_GRAD_MIDPOINT || cfg.y_schemes.gradient == XCAL_GRAD_MIDPOINT)))
        build_midpoint(*m, stream);
    for (const xcal_schemes* sc : {&cfg.U_schemes, &cfg.p_schemes}) {
        if (sc->limiter != XCAL_LIMITER_NONE && sc->limiter != XCAL_LIMITER_CELL && sc->limiter != XCAL_LIMITER_FACE &&
            sc->limiter != XCAL_LIMITER_MFACE)
            fail(XCAL_ERR_UNSUPPORTED, "gradient limiter: CellBased, FaceBased or MFaceBased");
        if (sc->limiter == XCAL_LIMITER_CELL && !(sc->limiter_level >= 0.0 && sc->limiter_level <= 1.0))
            fail(XCAL_ERR_INVALID, "CellBased limiter level must be in [0, 1]");
    }
    if (cfg.U_schemes.limiter != XCAL_LIMITER_NONE || cfg.p_schemes.limiter != XCAL_LIMITER_NONE)
        build_limiter(*m, stream);
    for (int d = 0; d < 3; ++d) {
        Uc[d].zero(stream);
        gradp[d].zero(stream);
        Hv[d].zero(stream);
        Uf[d].zero(stream);
    }
    for (int d = 0; d < 9; ++d) gradU[d].zero(stream);
    for (DBuf<double>* b : {&p, &rD, &divHv, &nut, &Delta, &prev, &courant, &mdot, &nueff, &nutf, &pf})
        b->zero(stream);
    launch_fill(stream, rDf.p, 1.0, nF);  // initialise!(rDf, 1.0) (Solvers_1_SIMPLE.jl:61)
    // Krylov workspace
    int T = (nC + 2047) / 2048;
    for (DBuf<double>* b : {&ws.x, &ws.dx, &ws.r, &ws.z, &ws.p, &ws.q, &ws.v, &ws.s, &ws.t}) {
        b->alloc(nC);
        b->zero(stream);
    }
    if (cfg.precision == XCAL_PREC_MIXED) {
        for (DBuf<float>* b : {&ws.fx, &ws.fr, &ws.fz, &ws.fp, &ws.fq, &ws.fv, &ws.fs, &ws.ft, &ws.fd}) {
            b->alloc(nC);
            b->zero(stream);
        }
        ws.fpart.alloc(2 * FOLD_MAX_BLOCKS);
        ws.fpart.zero(stream);
        ws.frp.alloc(2L * nC);
        ws.frp.zero(stream);
        for (Equation* E : {&U, &P}) {
            E->nz32.alloc(E->nnz);
            E->nz32.zero(stream);
            E->P32.alloc(E->n);
            E->P32.zero(stream);
            for (LevelSell* L : {&E->lsell, &E->usell})
                if (L->nslots > 0) {
                    L->val32.alloc(L->nslots);
                    L->val32.zero(stream);
                    if (L == &E->lsell) {
                        L->dinv32.alloc(L->nslots);
                        L->dinv32.zero(stream);
                    }
                }
        }
    }
    ws.part0.alloc(T);
    ws.part1.alloc(T);
    ws.bar.alloc(2);
    ws.bar.zero(stream);
    ws.err.alloc(1);
    ws.err.zero(stream);
    ws.S.alloc(2);
    ws.S.zero(stream);
    resbuf.alloc(8);
    resbuf.zero(stream);
    io.alloc(std::max(nC, nF));
    cmax.alloc(T);
    cmax_ctr.alloc(1);
    cmax_ctr.zero(stream);
    gres.alloc(GRES_N);
    gres.zero(stream);
    giters.alloc(2 * GRES_N);
    giters.zero(stream);
    dlaunch.alloc(1);
    dlaunch.zero(stream);
    XCAL_CUDA(cudaMallocHost(&h_iters, 2 * GRES_N * sizeof(int)));
    XCAL_CUDA(cudaMallocHost(&h_launch, sizeof(unsigned long long)));
    XCAL_CUDA(cudaMallocHost(&h_perr, sizeof(int)));
    // host-side per-cell constants: V^(1/3) (Courant) and the LES filter
    std::vector<double> h(nC);
    // Courant cell size: V^(1/3) (Mesh3), sqrt(V) (Mesh2, Solvers_0_functions.jl:277-285)
    for (int i = 0; i < nC; ++i) h[i] = m->dim == 2 ? std::sqrt(m->vol[i]) : std::pow(m->vol[i], 1.0 / 3.0);
    XCAL_CUDA(cudaMemcpyAsync(dx13.p, h.data(), nC * sizeof(double), cudaMemcpyHostToDevice, stream));
    if (cfg.turbulence == XCAL_TURB_SMAGORINSKY || keq()) {
        // LES_Smagorinsky.jl:84-101 + LES_functions.jl:1-55 (delta! with
        // delta_scaling); Smagorinsky keeps (C Delta)^2, KEquation Delta
        double distance = 1.0, power = 1.0 / 3.0;
        if (cfg.les_delta_power > 0.0) {
            distance = cfg.les_delta_distance;
            power = cfg.les_delta_power;
        } else
        for (const xcal_bc& bc : bcU.src)
            if (bc.type == XCAL_BC_EMPTY) {
                double pmin[3] = {0, 0, 0}, pmax[3] = {0, 0, 0};
                for (int f = 0; f < m->nB; ++f) {
                    double c3[3] = {m->fcx[f], m->fcy[f], m->fcz[f]};
                    for (int k = 0; k < 3; ++k) {
                        pmin[k] = std::min(pmin[k], c3[k]);
                        pmax[k] = std::max(pmax[k], c3[k]);
                    }
                }
                int f0 = m->patch_start[bc.patch];
                double n3[3] = {m->nxh[f0], m->nyh[f0], m->nzh[f0]};
                double d1 = std::fabs(pmin[0] * n3[0] + pmin[1] * n3[1] + pmin[2] * n3[2]);
                double d2 = std::fabs(pmax[0] * n3[0] + pmax[1] * n3[1] + pmax[2] * n3[2]);
                distance = d1 + d2;
                power = 0.5;
                break;
            }
        for (int i = 0; i < nC; ++i) {
            double dd = std::pow(m->vol[i] / distance, power);
            double dc = dd * cfg.smagorinsky_C;
            h[i] = keq() ? dd : dc * dc;
        }
        XCAL_CUDA(cudaMemcpyAsync(Delta.p, h.data(), nC * sizeof(double), cudaMemcpyHostToDevice, stream));
    }
    XCAL_CUDA(cudaStreamSynchronize(stream));
    // initialise(::KOmegaSST) (RANS_kOmegaSST.jl:167), initialise(::KOmegaLKE) (RANS_kOmegaLKE.jl:236)
    if (has_y()) wall_distance();
}

Case::~Case() {
    if (stream) cudaStreamSynchronize(stream);
    for (auto& row : chunk_graph)
        for (auto& g : row)
            if (g.exec) cudaGraphExecDestroy(g.exec);
    for (auto& row : gev)
        for (auto& e : row)
            if (e) cudaEventDestroy(e);
    for (auto& e : ev) cudaEventDestroy(e);
    for (auto& e : pev) cudaEventDestroy(e);
    if (h_S) cudaFreeHost(h_S);
    if (h_res) cudaFreeHost(h_res);
    if (h_iters) cudaFreeHost(h_iters);
    if (h_perr) cudaFreeHost(h_perr);
    if (h_launch) cudaFreeHost(h_launch);
    if (step_graph) cudaGraphExecDestroy(step_graph);
    for (cudaStream_t& sd : side)
        if (sd) cudaStreamDestroy(sd);
    if (stream && own_stream) cudaStreamDestroy(stream);
}

void Case::sync() { XCAL_CUDA(cudaStreamSynchronize(stream)); }

// Capture `body` (a fixed sequence of launches on the case stream) once,
// then replay it.  Launch counts follow the replays, not the capture.
template <class F>
void Case::replay_chunk(ChunkGraph& g, F&& body) {
    if (!g.exec) {
        const long long t0 = t_launch_count;
        cudaGraph_t graph = nullptr;
        XCAL_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        try {
            body();
        } catch (...) {
            cudaStreamEndCapture(stream, &graph);
            if (graph) cudaGraphDestroy(graph);
            throw;
        }
        XCAL_CUDA(cudaStreamEndCapture(stream, &graph));
        const long long captured = t_launch_count - t0;
        g_launch_count.fetch_sub(captured, std::memory_order_relaxed);
        t_launch_count = t0;
        cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
        cudaGraphDestroy(graph);
        XCAL_CUDA(e);
        g.launches = captured;
    }
    XCAL_CUDA(cudaGraphLaunch(g.exec, stream));
    g_launch_count.fetch_add(g.launches, std::memory_order_relaxed);
    t_launch_count += g.launches;
}

void Case::prof_reserve(int pairs) {
    while ((int)pev.size() < 2 * pairs) {
        cudaEvent_t e;
        XCAL_CUDA(cudaEventCreate(&e));
        pev.push_back(e);
    }
}

double* Case::field_comp(int field, int comp, long& count) {
    count = mesh->nC;
    switch (field) {
        case XCAL_FIELD_U: return Uc[comp].p;
        case XCAL_FIELD_P: return p.p;
        case XCAL_FIELD_MDOTF: count = mesh->nF; return mdot.p;
        case XCAL_FIELD_NUEFF: count = mesh->nF; return nueff.p;
        case XCAL_FIELD_GRADP: return gradp[comp].p;
        case XCAL_FIELD_GRADU: return gradU[comp].p;
        case XCAL_FIELD_RD: return rD.p;
        case XCAL_FIELD_HV: return Hv[comp].p;
        case XCAL_FIELD_DIVHV: return divHv.p;
        case XCAL_FIELD_NUT: return nut.p;
        case XCAL_FIELD_NUTF: count = mesh->nF; return nutf.p;
        case XCAL_FIELD_UF: count = mesh->nF; return Uf[comp].p;
        case XCAL_FIELD_PF: count = mesh->nF; return pf.p;
        case XCAL_FIELD_RDF: count = mesh->nF; return rDf.p;
        case XCAL_FIELD_DELTA: return Delta.p;
        case XCAL_FIELD_K:
        case XCAL_FIELD_OMEGA:
            if (field == XCAL_FIELD_K && keq()) return kfld.p;
            if (!rans_kw())
                fail(XCAL_ERR_INVALID, "k / omega fields need RANS{KOmega}, RANS{KOmegaSST} or (k) LES{KEquation}");
            return field == XCAL_FIELD_K ? kfld.p : omega.p;
        case XCAL_FIELD_WALLDIST:
            if (!has_y()) fail(XCAL_ERR_INVALID, "the wall distance needs RANS{KOmegaSST} or RANS{KOmegaLKE}");
            return yw.p;
        case XCAL_FIELD_KL:
        case XCAL_FIELD_GAMMA:
            if (!lke()) fail(XCAL_ERR_INVALID, "kl / gamma need RANS{KOmegaLKE}");
            return field == XCAL_FIELD_KL ? kl.p : gam.p;
        case XCAL_FIELD_PK:
        case XCAL_FIELD_DK:
        case XCAL_FIELD_DW:
            if (!has_k()) fail(XCAL_ERR_INVALID, "k-equation sources need RANS{KOmega} or LES{KEquation}");
            return field == XCAL_FIELD_PK ? Pk.p : field == XCAL_FIELD_DK ? Dk.p : Dw.p;
        default: return nullptr;
    }
}

// ---------------------------------------------------------------------------
// steps
// ---------------------------------------------------------------------------
void Case::initial_calculations() {  // Solvers_1_SIMPLE.jl:150-156
    const double* Ucp[3] = {Uc[0].p, Uc[1].p, Uc[2].p};
    double* Ufp[3] = {Uf[0].p, Uf[1].p, Uf[2].p};
    launch_interp_U(stream, mv(), bcU.view(), Ucp, Ufp, mdot.p);
    grad_p();
    // update_nueff! (Solvers_0_functions.jl:5-35) from the nutf as it stands
    if (cfg.turbulence == XCAL_TURB_LAMINAR)
        launch_fill(stream, nueff.p, cfg.nu, mesh->nF);
    else
        launch_nueff(stream, mesh->nF, nutf.p, nueff.p, cfg.nu);
    initialised = true;
}

// The omega wall constraint's rows (constrain_equation!, RANS_functions.jl:
// 376-429): BCs in order, each BC's faces in order, so a cell's row ends as
// its last such face sets it; per wall cell that face's y = delta and the
// BC's constants
void Case::build_wall_table(const DevMesh& m) {
    std::vector<int> win(m.nC, -1), wf, wb;
    for (int b = 0; b < (int)bcOmega.src.size(); ++b) {
        const xcal_bc& bc = bcOmega.src[b];
        if (bc.type != XCAL_BC_OMEGA_WALL) continue;
        const int start = m.patch_start[bc.patch], count = m.patch_count[bc.patch];
        for (int f = start; f < start + count; ++f) {
            win[m.bcell[f]] = (int)wf.size();
            wf.push_back(f);
            wb.push_back(b);
        }
    }
    std::vector<int> cells;
    std::vector<double> par;
    for (int c = 0; c < m.nC; ++c) {
        if (win[c] < 0) continue;
        const int f = wf[win[c]];
        const xcal_bc& bc = bcOmega.src[wb[win[c]]];
        cells.push_back(c);
        for (double v : {m.delta[f], bc.wall[0], bc.wall[1], bc.wall[2], bc.wall[3]}) par.push_back(v);
    }
    nwall = (int)cells.size();
    if (nwall) {
        wcell.upload(cells, stream);
        wpar.upload(par, stream);
    }
    // KWallFunction (set_production!, RANS_functions.jl:66-117): the last
    // face per cell in BC then face order; NutWallFunction faces
    std::vector<int> kwin(m.nC, -1), kf, kc, nf;
    std::vector<double> kp, np_;
    for (const xcal_bc& bc : bcK.src) {
        if (bc.type != XCAL_BC_K_WALL) continue;
        const int start = m.patch_start[bc.patch], count = m.patch_count[bc.patch];
        for (int f = start; f < start + count; ++f) {
            const int c = m.bcell[f];
            if (kwin[c] < 0) {
                kwin[c] = (int)kc.size();
                kc.push_back(c);
                kf.push_back(f);
                kp.insert(kp.end(), {0, 0, 0, 0});
            }
            const int t = kwin[c];
            kf[t] = f;
            for (int q = 0; q < 4; ++q) kp[4 * t + q] = q == 0 ? bc.wall[0] : bc.wall[q + 1];
        }
    }
    for (const xcal_bc& bc : bcNut.src) {
        if (bc.type != XCAL_BC_NUT_WALL) continue;
        const int start = m.patch_start[bc.patch], count = m.patch_count[bc.patch];
        for (int f = start; f < start + count; ++f) {
            nf.push_back(f);
            for (double v : {bc.wall[0], bc.wall[2], bc.wall[3], bc.wall[4]}) np_.push_back(v);
        }
    }
    nkwall = (int)kc.size();
    nnutwall = (int)nf.size();
    if (nkwall) {
        kwcell.upload(kc, stream);
        kwface.upload(kf, stream);
        kwpar.upload(kp, stream);
    }
    if (nnutwall) {
        nwface.upload(nf, stream);
        nwpar.upload(np_, stream);
    }
}

// turbulence!(::KOmegaModel) after grad!(gradU) (RANS_kOmega.jl:146-210):
// production and dissipation coefficients, then the omega and k equations
// (Time + Div - Lap(nu + sigma nutf) + Si == Source) on the p system, each
// relaxed, solved and bounded (omega's wall rows constrained first), then
// nut = k / omega, nutf with its BCs and nueff
void Case::komega() {
    const double* g[9];
    for (int q = 0; q < 9; ++q) g[q] = gradU[q].p;
    const bool S = sst();
    if (S) {
        // RANS_kOmegaSST.jl:214-266: grad omega (p's gradient scheme), grad k, then the cell fields
        double* gw[3] = {gwv[0].p, gwv[1].p, gwv[2].p};
        double* gk[3] = {gkv[0].p, gkv[1].p, gkv[2].p};
        scalar_grad(omega.p, bcOmega, cfg.p_schemes.gradient, gw);
        scalar_grad(kfld.p, bcK, cfg.k_schemes.gradient, gk);
        const double* gwc[3] = {gw[0], gw[1], gw[2]};
        const double* gkc[3] = {gk[0], gk[1], gk[2]};
        launch_sst_fields(stream, mesh->nC, g, gkc, gwc, kfld.p, omega.p, nut.p, yw.p, F1b.p, F2b.p, Omb.p, Pk.p, Pw.p,
                          Dk.p, Dw.p, D2b.p, cfg.kw_beta_star, cfg.kw_alpha1, cfg.kw_beta1, cfg.sst_beta2,
                          cfg.sst_sigma_omega2, cfg.nu);
    } else {
        launch_kw_sources(stream, mesh->nC, g, nut.p, omega.p, Pk.p, Pw.p, Dk.p, Dw.p, cfg.kw_alpha1, cfg.kw_beta1,
                          cfg.kw_beta_star);
    }
    const double* Ucp[3] = {Uc[0].p, Uc[1].p, Uc[2].p};
    launch_kwall_production(stream, nkwall, mv(), kwcell.p, kwface.p, kwpar.p, kfld.p, Ucp, cfg.nu, Pk.p);
    for (int e : {(int)XCAL_EQN_OMEGA, (int)XCAL_EQN_K}) {
        const bool w = e == XCAL_EQN_OMEGA;
        double* phi = w ? omega.p : kfld.p;
        const xcal_schemes& sc = w ? cfg.omega_schemes : cfg.k_schemes;
        const double sigma = w ? cfg.kw_sigma_omega : cfg.kw_sigma_k;
        const double sigma2 = w ? cfg.sst_sigma_omega2 : cfg.sst_sigma_k2;
        const double* F1 = S ? F1b.p : nullptr;
        const double* D2 = (S && w) ? D2b.p : nullptr;
        launch_assemble_scalar(stream, mv(), P.view(), mdot.p, nutf.p, cfg.nu, sigma, F1, sigma2, phi,
                               w ? Dw.p : Dk.p, D2, w ? Pw.p : Pk.p, P.nz.p, P.b[0].p, sc.time, sc.divergence, cfg.dt);
        launch_bc_relax_scalar(stream, mv(), P.view(), (w ? bcOmega : bcK).view(), P.nz.p, P.b[0].p, mdot.p, nutf.p,
                               cfg.nu, sigma, F1, sigma2, D2 ? 1 : 0, phi, (w ? cfg.omega_solver : cfg.k_solver).relax,
                               sc.divergence);
        if (w && nwall) launch_omega_constrain(stream, nwall, P.view(), wcell.p, wpar.p, kfld.p, cfg.nu, P.nz.p, P.b[0].p);
        update_precond(e);
        const double r = solve_system(e, 0, &last_iters[w ? 5 : 4]);
        (w ? res_omega : res_k) = r;
        XCAL_CUDA(cudaMemcpyAsync(kwtmp.p, phi, (size_t)mesh->nC * sizeof(double), cudaMemcpyDeviceToDevice, stream));
        launch_bound(stream, mv(), kwtmp.p, phi);
    }
    if (S)
        launch_sst_nut(stream, mesh->nC, kfld.p, omega.p, F2b.p, Omb.p, cfg.kw_alpha1, nut.p);
    else
        launch_kw_nut(stream, mesh->nC, kfld.p, omega.p, nut.p);
    launch_interp_scalar(stream, mv(), bcNut.view(), nut.p, nutf.p, nueff.p, cfg.nu);
    launch_nutwall(stream, nnutwall, mv(), nwface.p, nwpar.p, kfld.p, cfg.nu, nutf.p, nueff.p);
}

// turbulence!(::KEquationModel) (LES_KEquation.jl:134-186), grad U already
// formed (and limited): the cell sources from the previous nut and k, the k
// equation Time + Div(mdotf) - Lap(nu + nut_f) + Si(Dk) + Si(Dw) ==
// Source(Pk) assembled on the p system with k's BCs and implicit
// relaxation, solved, bounded; then nut = ck Delta sqrt(k), its faces with
// their BCs and the wall functions' nut (correct_eddy_viscosity!)
void Case::kequation() {
    const double* g[9];
    for (int q = 0; q < 9; ++q) g[q] = gradU[q].p;
    launch_keq_sources(stream, mesh->nC, g, nut.p, kfld.p, Delta.p, cfg.keq_ce, Pk.p, Dk.p, Dw.p);
    const xcal_schemes& sc = cfg.k_schemes;
    launch_assemble_scalar(stream, mv(), P.view(), mdot.p, nutf.p, cfg.nu, 1.0, nullptr, 0.0, kfld.p, Dk.p, Dw.p,
                           Pk.p, P.nz.p, P.b[0].p, sc.time, sc.divergence, cfg.dt);
    launch_bc_relax_scalar(stream, mv(), P.view(), bcK.view(), P.nz.p, P.b[0].p, mdot.p, nutf.p, cfg.nu, 1.0, nullptr,
                           0.0, 1, kfld.p, cfg.k_solver.relax, sc.divergence);
    update_precond(XCAL_EQN_K);
    res_k = solve_system(XCAL_EQN_K, 0, &last_iters[4]);
    XCAL_CUDA(cudaMemcpyAsync(kwtmp.p, kfld.p, (size_t)mesh->nC * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    launch_bound(stream, mv(), kwtmp.p, kfld.p);
    launch_keq_nut(stream, mesh->nC, kfld.p, Delta.p, cfg.keq_ck, nut.p);
    launch_interp_scalar(stream, mv(), bcNut.view(), nut.p, nutf.p, nueff.p, cfg.nu);
    launch_nutwall(stream, nnutwall, mv(), nwface.p, nwpar.p, kfld.p, cfg.nu, nutf.p, nueff.p);
}

// turbulence!(::KOmegaLKEModel) after grad!(gradU) and its limiter
// (RANS_kOmegaLKE.jl:262-474), rho = 1.  Each equation Time + Div(mdotf) -
// Lap(nueff_f) + Si(D) [- Si(D2)] == Source(P) goes on the p system with
// its own BCs, implicit relaxation and preconditioner and is bounded after
// its solve; nueff_f is the equation's cell diffusivity interpolated with
// nut's BCs (interpolate! + correct_boundaries!).  Order: the cell fields
// and gamma, kl; grad omega, grad k and the omega equation (its wall rows
// constrained from the current k); the k equation (KWallFunction production
// after its cell loop); nut = fSS k / omega + nuL, nutf with nut's BCs and
// the wall functions
void Case::komega_lke() {
    LkeView V{};
    for (int q = 0; q < 9; ++q) V.g[q] = gradU[q].p;
    for (int d = 0; d < 3; ++d) {
        V.U[d] = Uc[d].p;
        V.gk[d] = gkv[d].p;
        V.gw[d] = gwv[d].p;
    }
    V.y = yw.p;
    V.kl = kl.p;
    V.k = kfld.p;
    V.omega = omega.p;
    V.divU = divUb.p;
    V.S2 = S2b.p;
    V.Om = Omb.p;
    V.normU = normUb.p;
    V.ReL = ReLb.p;
    V.gam = gam.p;
    V.Pk = Pk.p;
    V.Pw = Pw.p;
    V.PkL = PkL.p;
    V.Dk = Dk.p;
    V.Dw = Dw.p;
    V.DkL = DkL.p;
    V.D2 = D2b.p;
    V.nueffS = nueffS.p;
    V.nut = nut.p;
    V.nC = mesh->nC;
    V.nu = cfg.nu;
    V.eta = lke_eta;
    // D2 (omega's cross diffusion) enters with sign -1: - Si(dkdomegadx, omega)
    auto transport = [&](int e, double* phi, const BCTable& T, const xcal_schemes& sc, const xcal_solver_setup& SS,
                         const double* D, const double* D2, const double* src, bool constrain, int slot) {
        launch_interp_scalar(stream, mv(), bcNut.view(), nueffS.p, fmu.p, nullptr, 0.0);
        launch_assemble_scalar(stream, mv(), P.view(), mdot.p, fmu.p, 0.0, 1.0, nullptr, 0.0, phi, D, D2, src, P.nz.p,
                               P.b[0].p, sc.time, sc.divergence, cfg.dt, /*d2_sign=*/-1.0);
        launch_bc_relax_scalar(stream, mv(), P.view(), T.view(), P.nz.p, P.b[0].p, mdot.p, fmu.p, 0.0, 1.0, nullptr,
                               0.0, D2 ? 1 : 0, phi, SS.relax, sc.divergence);
        if (constrain && nwall)
            launch_omega_constrain(stream, nwall, P.view(), wcell.p, wpar.p, kfld.p, cfg.nu, P.nz.p, P.b[0].p);
        update_precond(e);
        const double r = solve_system(e, 0, &last_iters[slot]);
        XCAL_CUDA(cudaMemcpyAsync(kwtmp.p, phi, (size_t)mesh->nC * sizeof(double), cudaMemcpyDeviceToDevice, stream));
        launch_bound(stream, mv(), kwtmp.p, phi);
        return r;
    };
    launch_lke_fields(stream, V);
    res_kl = transport(XCAL_EQN_KL, kl.p, bcKl, cfg.kl_schemes, cfg.kl_solver, DkL.p, nullptr, PkL.p, false, 7);
    double* gw[3] = {gwv[0].p, gwv[1].p, gwv[2].p};
    double* gk[3] = {gkv[0].p, gkv[1].p, gkv[2].p};
    scalar_grad(omega.p, bcOmega, cfg.p_schemes.gradient, gw);  // Grad{schemes.p.gradient}(omega) (:177)
    scalar_grad(kfld.p, bcK, cfg.k_schemes.gradient, gk);
    launch_lke_omega(stream, V);
    // omega: ... + Si(Dw) - Si(cross diffusion) == Source(Pw)
    res_omega = transport(XCAL_EQN_OMEGA, omega.p, bcOmega, cfg.omega_schemes, cfg.omega_solver, Dw.p, D2b.p, Pw.p,
                          true, 5);
    launch_lke_k(stream, V);
    const double* Ucp[3] = {Uc[0].p, Uc[1].p, Uc[2].p};
    launch_kwall_production(stream, nkwall, mv(), kwcell.p, kwface.p, kwpar.p, kfld.p, Ucp, cfg.nu, Pk.p);
    res_k = transport(XCAL_EQN_K, kfld.p, bcK, cfg.k_schemes, cfg.k_solver, Dk.p, nullptr, Pk.p, false, 4);
    launch_lke_nut(stream, V);
    launch_interp_scalar(stream, mv(), bcNut.view(), nut.p, nutf.p, nueff.p, cfg.nu);
    launch_nutwall(stream, nnutwall, mv(), nwface.p, nwpar.p, kfld.p, cfg.nu, nutf.p, nueff.p);
}

// grad! of a scalar with its BCs (Calculate_0_gradient.jl): Gauss, or the
// Midpoint passes (as grad p)
void Case::scalar_grad(const double* phi, const BCTable& T, int scheme, double* const g[3]) {
    launch_interp_scalar(stream, mv(), T.view(), phi, fscr.p, nullptr, 0.0);
    launch_green_gauss(stream, mv(), fscr.p, g);
    if (scheme != XCAL_GRAD_MIDPOINT) return;
    const double* gc[3] = {g[0], g[1], g[2]};
    launch_mid_scalar(stream, mv(), phi, fscr.p);
    launch_green_gauss(stream, mv(), fscr.p, g);
    for (int it = 0; it < 2; ++it) {
        launch_mid_correct_scalar(stream, mv(), midR.p, phi, gc, fscr.p);
        launch_green_gauss(stream, mv(), fscr.p, g);
    }
}

// wall_distance! (Calculate_4_wall_distance.jl:4-92), once at case creation:
// -Laplacian(1, phi) == Source(1) with the wall BCs on the p system (the p
// assembly with rDf = 1 and divHv = -1 gives the same coefficients), solved
// and explicitly relaxed until the residual is below y_solver.convergence
// (1000 at most); y = -|grad phi| + sqrt(|grad phi|^2 + 2 phi)
void Case::wall_distance() {
    const int nC = mesh->nC, nF = mesh->nF;
    DBuf<double> ones_f, mone_c;
    ones_f.alloc(nF);
    mone_c.alloc(nC);
    launch_fill(stream, ones_f.p, 1.0, nF);
    launch_fill(stream, mone_c.p, -1.0, nC);
    const xcal_solver_setup& SS = cfg.y_solver;
    for (int it = 0; it < 1000; ++it) {
        XCAL_CUDA(cudaMemcpyAsync(kwtmp.p, yphi.p, (size_t)nC * sizeof(double), cudaMemcpyDeviceToDevice, stream));
        launch_assemble_p(stream, mv(), P.view(), ones_f.p, mone_c.p, P.nz.p, P.b[0].p);
        launch_bc_p(stream, mv(), P.view(), bcY.view(), P.nz.p, P.b[0].p, ones_f.p, yphi.p);
        update_precond(XCAL_EQN_WALLDIST);
        const double res = solve_system(XCAL_EQN_WALLDIST, 0, &last_iters[6]);
        launch_relax_explicit(stream, nC, yphi.p, kwtmp.p, SS.relax);
        if (res < SS.convergence) break;
    }
    double* g[3] = {gkv[0].p, gkv[1].p, gkv[2].p};
    scalar_grad(yphi.p, bcY, cfg.y_schemes.gradient, g);
    const double* gc[3] = {g[0], g[1], g[2]};
    launch_walldist(stream, nC, yphi.p, gc, yw.p);
    sync();
}

void Case::discretise(int eqn) {
    if (eqn != XCAL_EQN_U && eqn != XCAL_EQN_P) fail(XCAL_ERR_INVALID, "discretise: equation must be U or p");
    if (eqn == XCAL_EQN_U) {
        const double* Ucp[3] = {Uc[0].p, Uc[1].p, Uc[2].p};
        const double* gp[3] = {gradp[0].p, gradp[1].p, gradp[2].p};
        double* bp[3] = {U.b[0].p, U.b[1].p, U.b[2].p};
        launch_assemble_U(stream, mv(), U.view(), mdot.p, nueff.p, Ucp, gp, U.nz.p, U.diag0.p, bp,
                          cfg.U_schemes.time, cfg.U_schemes.divergence, cfg.dt);
    } else {
        launch_assemble_p(stream, mv(), P.view(), rDf.p, divHv.p, P.nz.p, P.b[0].p);
    }
}

// update_equation! + apply_boundary_conditions! (+ relaxation for U, fused)
void Case::apply_bcs(int eqn, int comp) {
    if (eqn != XCAL_EQN_U && eqn != XCAL_EQN_P) fail(XCAL_ERR_INVALID, "apply_bcs: equation must be U or p");
    if (eqn == XCAL_EQN_U) {
        const double* Ucp[3] = {Uc[0].p, Uc[1].p, Uc[2].p};
        launch_bc_relax_U(stream, mv(), U.view(), bcU.view(), comp, cfg.U_schemes.divergence, U.nz.p, U.diag0.p,
                          U.b[comp].p, mdot.p, nueff.p, Ucp, cfg.U_solver.relax, BCR_DIAG0 | BCR_BC);
    } else {
        launch_bc_p(stream, mv(), P.view(), bcP.view(), P.nz.p, P.b[0].p, rDf.p, p.p);
    }
}

void Case::relax_U(int comp) {
    const double* Ucp[3] = {Uc[0].p, Uc[1].p, Uc[2].p};
    launch_bc_relax_U(stream, mv(), U.view(), bcU.view(), comp, cfg.U_schemes.divergence, U.nz.p, U.diag0.p,
                      U.b[comp].p, mdot.p, nueff.p, Ucp, cfg.U_solver.relax, BCR_RELAX);
}

void Case::bc_relax_U(int comp) {
    const double* Ucp[3] = {Uc[0].p, Uc[1].p, Uc[2].p};
    launch_bc_relax_U(stream, mv(), U.view(), bcU.view(), comp, cfg.U_schemes.divergence, U.nz.p, U.diag0.p,
                      U.b[comp].p, mdot.p, nueff.p, Ucp, cfg.U_solver.relax, BCR_DIAG0 | BCR_BC | BCR_RELAX);
}

void Case::set_reference() {
    if (cfg.has_pref) launch_set_reference(stream, P.view(), P.nz.p, P.b[0].p, cfg.pref, mesh->inv[0]);
}

bool Case::coop_ok_here() {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(stream, &st) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return st == cudaStreamCaptureStatusNone || kr_coop_capture_ok(side_depth > 0);
}

void Case::update_precond(int eqn) {
    const SolveRef R = solve_ref(eqn, 0);
    update_precond_E(*R.E, R.SS.precond);
}

void Case::update_precond_E(Equation& E, int pt) {
    if (pt == XCAL_PRECOND_JACOBI) {
        kr_jacobi_update(stream, E.view(), E.nz.p, E.P.p);
    } else if (pt == XCAL_PRECOND_DILU) {
        if (E.dilu_block()) {
            kr_dilu_D_lv_block(stream, E.n, level_d_view(E), E.nz.p, E.P.p);
            return;
        }
        if (E.use_grid && coop_ok_here() && kr_dilu_D_lv_grid(stream, level_d_view(E), E.nz.p, E.P.p, ws.bar.p, ws.err.p))
            return;
        for (size_t l = 0; l + 1 < E.lower_off.size(); ++l)
            kr_dilu_D(stream, E.d_lower_rows.p + E.lower_off[l], E.lower_off[l + 1] - E.lower_off[l], E.view(),
                      E.nz.p, E.P.p);
    }
}

template <class T>
void Case::dilu_ldiv(Equation& E, const T* nz, const T* D, const T* b, T* out, const KScalars* S) {
    // both paths read the level-ordered triangles (values and 1/D refreshed
    // by dilu_refresh before the solve); nz is the matrix those mirror
    (void)nz;
    if (E.dilu_block()) {
        kr_dilu_block(stream, E.n, level_view<T>(E, 0), level_view<T>(E, 1), D, b, out, S);
        return;
    }
    if (E.use_grid && coop_ok_here() &&
        kr_dilu_grid(stream, level_view<T>(E, 0), level_view<T>(E, 1), D, b, out, ws.bar.p, ws.err.p, S))
        return;
    const LevelView<T> lo = level_view<T>(E, 0);
    const T* uv = sizeof(T) == 8 ? (const T*)E.usell.val.p : (const T*)E.usell.val32.p;
    for (size_t l = 0; l + 1 < E.lower_off.size(); ++l)
        kr_dilu_fwd_lv(stream, E.lower_off[l], E.lower_off[l + 1], E.d_lower_rows.p, E.lsell.slice.p, E.lsell.cnt.p,
                       E.lsell.col.p, lo.val, lo.dinv, b, out, S);
    for (size_t l = 0; l + 1 < E.upper_off.size(); ++l)
        kr_dilu_bwd_lv(stream, E.upper_off[l], E.upper_off[l + 1], E.d_upper_rows.p, E.usell.slice.p, E.usell.cnt.p,
                       E.usell.col.p, uv, D, out, S);
}

// copy the current off-diagonal values into the level-ordered triangles and
// form the lower triangle's 1/D per slot (FP64 values and D, or the FP32
// copies nz32 / P32 for the mixed inner solves); D must be current
void Case::dilu_refresh(Equation& E, bool fp32) {
    if (E.lower_off.empty()) return;
    for (LevelSell* L : {&E.lsell, &E.usell}) {
        if (fp32) {
            kr_gather_vals(stream, L->nslots, L->src.p, E.nz32.p, L->val32.p);
        } else {
            kr_gather_vals(stream, L->nslots, L->src.p, E.nz.p, L->val.p);
        }
    }
    if (fp32)
        kr_level_dinv(stream, E.lsell.nslots, E.lsell.col.p, E.P32.p, E.lsell.dinv32.p);
    else
        kr_level_dinv(stream, E.lsell.nslots, E.lsell.col.p, E.P.p, E.lsell.dinv.p);
}

LevelDView level_d_view(const Equation& E) {
    const LevelSell& L = E.lsell;
    return LevelDView{E.d_lower_rows.p, E.d_lower_off.p, (int)E.lower_off.size() - 1, L.slice.p, L.cnt.p,
                      L.col.p, L.src.p, L.tsrc.p, L.dslot.p};
}

template <class T>
LevelView<T> level_view(const Equation& E, int tri) {
    const LevelSell& L = tri == 0 ? E.lsell : E.usell;
    LevelView<T> v;
    v.rows = tri == 0 ? E.d_lower_rows.p : E.d_upper_rows.p;
    v.off = tri == 0 ? E.d_lower_off.p : E.d_upper_off.p;
    const std::vector<int>& off = tri == 0 ? E.lower_off : E.upper_off;
    v.nlev = off.empty() ? 0 : (int)off.size() - 1;
    v.slice = L.slice.p;
    v.cnt = L.cnt.p;
    v.col = L.col.p;
    v.val = sizeof(T) == 8 ? (const T*)L.val.p : (const T*)L.val32.p;
    v.dinv = sizeof(T) == 8 ? (const T*)L.dinv.p : (const T*)L.dinv32.p;
    return v;
}
template LevelView<double> level_view<double>(const Equation&, int);
template LevelView<float> level_view<float>(const Equation&, int);

template <class T>
void Case::apply_M(Equation& E, int ptype, const T* nz, const T* P, const T* in, T* out, const KScalars* S) {
    if (ptype == XCAL_PRECOND_JACOBI)
        kr_jacobi_apply(stream, E.n, P, in, out, S);
    else if (ptype == XCAL_PRECOND_DILU)
        dilu_ldiv(E, nz, P, in, out, S);
    else
        kr_copy(stream, E.n, in, out, S);
}

// Start of a Krylov solve from its initial residual.  CG: V.r holds r0.
// BiCGSTAB: r0 holds the unpreconditioned r0 and c is Krylov.jl's shadow
// vector (the right-hand side).
template <class T>
void Case::krylov_start(Equation& E, const xcal_solver_setup& SS, const T* nz, const T* P, const T* c, const T* r0,
                        const KrylovVecs<T>& V, KScalars* S) {
    const int n = E.n;
    const int pt = SS.precond;
    if (SS.solver == XCAL_SOLVER_CG) {
        T* zz = pt == XCAL_PRECOND_NONE ? V.r : V.z;
        if (pt != XCAL_PRECOND_NONE) apply_M(E, pt, nz, P, (const T*)V.r, zz, (const KScalars*)nullptr);
        kr_cg_start(stream, n, (const T*)V.r, (const T*)zz, V.p, S, ws.part0.p);
    } else {
        apply_M(E, pt, nz, P, r0, V.r, (const KScalars*)nullptr);
        kr_bicg_start(stream, n, c, (const T*)V.r, V.p, S, ws.part0.p, ws.part1.p);
    }
}

// One Krylov iteration (every kernel returns at once when the solve is done).
// ev (optional): CG -- events before the SpMV, between SpMV and update, after
// the update; BiCGSTAB -- around both SpMVs and both preconditioner
// applications.  in_capture: record the events as graph event nodes.
template <class T>
void Case::krylov_step(Equation& E, const xcal_solver_setup& SS, const T* nz, const T* P, const T* c,
                       const KrylovVecs<T>& V, KScalars* S, cudaEvent_t* ev, bool in_capture) {
    const int n = E.n;
    const int pt = SS.precond;
    CSRView A = E.view();
    auto rec = [&](cudaEvent_t e) {
        if (in_capture)
            XCAL_CUDA(cudaEventRecordWithFlags(e, stream, cudaEventRecordExternal));
        else
            XCAL_CUDA(cudaEventRecord(e, stream));
    };
    T *x = V.x, *r = V.r, *pp = V.p, *q = V.q, *v = V.v, *s = V.s, *t = V.t;
    if (SS.solver == XCAL_SOLVER_CG) {
        T* zz = pt == XCAL_PRECOND_NONE ? r : V.z;
        if (ev) rec(ev[0]);
        // p_k alternates between pp (even k) and v (odd k)
        kr_cg_spmv(stream, A, nz, (const T*)zz, pp, v, q, S, ws.part0.p);
        if (ev) rec(ev[1]);
        if (pt == XCAL_PRECOND_JACOBI) {
            kr_cg_update(stream, n, x, (const T*)pp, (const T*)v, r, (const T*)q, zz, P, 1, S, ws.part0.p);
        } else {
            kr_cg_update(stream, n, x, (const T*)pp, (const T*)v, r, (const T*)q, zz, P, 0, S, ws.part0.p);
            if (pt == XCAL_PRECOND_DILU) dilu_ldiv(E, nz, P, (const T*)r, zz, (const KScalars*)S);
            kr_cg_rz(stream, n, (const T*)r, (const T*)zz, S, ws.part0.p);
        }
        if (ev) rec(ev[2]);
    } else {
        if (ev) rec(ev[0]);
        kr_spmv_shaped(stream, E.spmv_shape, A, nz, (const T*)pp, q, (const KScalars*)S);
        if (ev) rec(ev[1]);
        apply_M(E, pt, nz, P, (const T*)q, v, (const KScalars*)S);
        if (ev) rec(ev[2]);
        kr_bicg_alpha(stream, n, c, (const T*)v, S, ws.part0.p);
        kr_bicg_s(stream, n, (const T*)r, (const T*)v, (const T*)pp, s, x, (const KScalars*)S);
        if (ev) rec(ev[3]);
        kr_spmv_shaped(stream, E.spmv_shape, A, nz, (const T*)s, q, (const KScalars*)S);
        if (ev) rec(ev[4]);
        apply_M(E, pt, nz, P, (const T*)q, t, (const KScalars*)S);
        if (ev) rec(ev[5]);
        kr_bicg_omega(stream, n, (const T*)t, (const T*)s, S, ws.part0.p, ws.part1.p);
        kr_bicg_xr(stream, n, x, (const T*)s, (const T*)t, r, c, S, ws.part0.p, ws.part1.p);
        kr_bicg_p(stream, n, (const T*)r, (const T*)v, pp, (const KScalars*)S);
    }
}

// Host-polled Krylov loop: chunks of iterations (4 -> 32 CG, 1 -> 8
// BiCGSTAB), the steady-state chunk replayed as a cached CUDA graph, the
// host reading the device's `done` flag after each chunk.  gk selects the
// cached chunk graphs.
template <class T>
void Case::krylov_iterate(Equation& E, const xcal_solver_setup& SS, const T* nz, const T* P, const T* c,
                          const T* r0, const KrylovVecs<T>& V, KScalars* S, KScalars* hS, int gk) {
    const bool cg = SS.solver == XCAL_SOLVER_CG;
    const int pt = SS.precond;
    if (profiling)
        for (auto& e : gev[gk])
            if (!e) XCAL_CUDA(cudaEventCreate(&e));
    krylov_start(E, SS, nz, P, c, r0, V, S);
    // the whole loop in one cooperative launch (falls through when the
    // system's tiles cannot all be co-resident).  Measured on B200 against
    // the two-kernel loop: faster at every size tried (1.2k-2.1M cells), in
    // FP64 and FP32 (2.1M cells, FP32: 51.7 vs 59 us per iteration).
    if (cg && persistent_cg && (pt == XCAL_PRECOND_JACOBI || pt == XCAL_PRECOND_NONE)) {
        const int it0 = 0;
        if (profiling) XCAL_CUDA(cudaEventRecord(ev[5], stream));
        T* zz = pt == XCAL_PRECOND_NONE ? V.r : V.z;
        if (kr_cg_persist(stream, E.view(), nz, P, pt == XCAL_PRECOND_JACOBI ? 1 : 0, V.x, V.r, zz, V.p, V.v, S,
                          ws.part0.p, ws.part1.p, ws.bar.p, ws.err.p, hS->itmax + 1,
                          persistent_cg > 1 ? persistent_cg : 0,
                          E.nnz * (long)(sizeof(T) + 4) <= PERSIST_PF_MAX_BYTES ? 256 : 0)) {
            if (profiling) XCAL_CUDA(cudaEventRecord(ev[6], stream));
            int errflag = 0;
            XCAL_CUDA(cudaMemcpyAsync(hS, S, sizeof(KScalars), cudaMemcpyDeviceToHost, stream));
            XCAL_CUDA(cudaMemcpyAsync(&errflag, ws.err.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
            sync();
            if (errflag) fail(XCAL_ERR_TIMEOUT, "persistent CG: a grid barrier wait gave up");
            if (!hS->done) fail(XCAL_ERR_TIMEOUT, "persistent CG did not report completion");
            if (profiling) {
                float t = 0;
                XCAL_CUDA(cudaEventElapsedTime(&t, ev[5], ev[6]));
                const int real = hS->iter - it0 + (hS->status == KS_ZERO_CURV ? 1 : 0);
                prof_ms[5] += t;
                prof_n[5] += hS->iter - it0;
                prof_n[4] += real;
            }
            return;
        }
    }
    const int CHUNK = cg ? 32 : 8;
    const int nev = cg ? 3 : 6;  // events per timed iteration
    int chunk = cg ? 4 : 1;
    long launched = 0;
    for (;;) {
        if ((launched += chunk) > (long)hS->itmax + 2 * CHUNK + 32)
            fail(XCAL_ERR_TIMEOUT, cg ? "CG did not report completion within itmax iterations"
                                      : "BiCGSTAB did not report completion within itmax iterations");
        int it0 = hS->iter;
        const bool graphed = chunk == CHUNK;
        // (iteration index within the chunk, its events); graphed chunks time
        // the iterations with c % 8 == 4
        std::vector<std::pair<int, cudaEvent_t*>> samples;
        if (graphed) {
            if (profiling)
                for (int c8 = 4; c8 < CHUNK; c8 += 8) samples.push_back({c8, &gev[gk][nev * (c8 / 8)]});
            replay_chunk(chunk_graph[gk][profiling ? 1 : 0], [&] {
                for (int ci = 0; ci < CHUNK; ++ci)
                    krylov_step(E, SS, nz, P, c, V, S, profiling && ci % 8 == 4 ? &gev[gk][nev * (ci / 8)] : nullptr,
                                true);
            });
        } else {
            if (profiling) prof_reserve((nev * chunk + 1) / 2 + 1);
            for (int ci = 0; ci < chunk; ++ci) {
                krylov_step(E, SS, nz, P, c, V, S, profiling ? &pev[nev * ci] : nullptr, false);
                if (profiling) samples.push_back({ci, &pev[nev * ci]});
            }
        }
        XCAL_CUDA(cudaMemcpyAsync(hS, S, sizeof(KScalars), cudaMemcpyDeviceToHost, stream));
        sync();
        const int done_it = hS->iter - it0;
        if (cg) {
            // launches that did work: one per completed iteration, plus a
            // final SpMV that detected zero curvature
            const int real = done_it + (hS->status == KS_ZERO_CURV ? 1 : 0);
            if (profiling) prof_n[4] += real;
            for (auto& sm : samples) {
                if (sm.first >= real) continue;
                float tm = 0, tu = 0;
                XCAL_CUDA(cudaEventElapsedTime(&tm, sm.second[0], sm.second[1]));
                prof_ms[0] += tm;
                prof_n[0] += 1;
                if (sm.first < done_it) {
                    XCAL_CUDA(cudaEventElapsedTime(&tu, sm.second[1], sm.second[2]));
                    prof_ms[3] += tu;
                    prof_n[3] += 1;
                }
            }
        } else {
            for (auto& sm : samples) {
                if (sm.first >= done_it) continue;
                cudaEvent_t* e = sm.second;
                float t0 = 0, t1 = 0, t2 = 0, t3 = 0;
                XCAL_CUDA(cudaEventElapsedTime(&t0, e[0], e[1]));
                XCAL_CUDA(cudaEventElapsedTime(&t1, e[3], e[4]));
                XCAL_CUDA(cudaEventElapsedTime(&t2, e[1], e[2]));
                XCAL_CUDA(cudaEventElapsedTime(&t3, e[4], e[5]));
                prof_ms[1] += t0 + t1;
                prof_n[1] += 2;
                if (pt == XCAL_PRECOND_DILU) {
                    prof_ms[2] += t2 + t3;
                    prof_n[2] += 2;
                }
            }
        }
        if (hS->done) break;
        if (chunk < CHUNK) chunk *= 2;
    }
}

// ---------------------------------------------------------------------------
// graph mode
// ---------------------------------------------------------------------------
// Add a conditional WHILE node at the current point of the capture running on
// `stream`; body(h) launches the loop body (captured into the node's body
// graph on a side stream) and must end with a kernel that sets h.
template <class F>
void Case::capture_while(F&& body) {
    if (side_depth >= 2) fail(XCAL_ERR_INVALID, "graph mode: WHILE loops nest at most two deep");
    cudaStreamCaptureStatus st;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    XCAL_CUDA(cudaStreamGetCaptureInfo(stream, &st, nullptr, &g, &deps, &nd));
    if (st != cudaStreamCaptureStatusActive) fail(XCAL_ERR_CUDA, "graph mode: no active capture");
    cudaGraphConditionalHandle h;
    XCAL_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
    // enter the loop with the condition set explicitly (also when the
    // enclosing body runs again)
    kr_set_cond(stream, h, 1u);
    XCAL_CUDA(cudaStreamGetCaptureInfo(stream, &st, nullptr, &g, &deps, &nd));
    cudaGraphNodeParams prm = {};
    prm.type = cudaGraphNodeTypeConditional;
    prm.conditional.handle = h;
    prm.conditional.type = cudaGraphCondTypeWhile;
    prm.conditional.size = 1;
    cudaGraphNode_t node;
    XCAL_CUDA(cudaGraphAddNode(&node, g, deps, nd, &prm));
    cudaGraph_t bodyg = prm.conditional.phGraph_out[0];
    if (!side[side_depth]) XCAL_CUDA(cudaStreamCreateWithFlags(&side[side_depth], cudaStreamNonBlocking));
    cudaStream_t outer = stream;
    stream = side[side_depth++];
    const long long kb = t_launch_count;
    XCAL_CUDA(cudaStreamBeginCaptureToGraph(stream, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    try {
        body(h);
    } catch (...) {
        cudaGraph_t tmp;
        cudaStreamEndCapture(stream, &tmp);
        stream = outer;
        --side_depth;
        throw;
    }
    cudaGraph_t tmp;
    XCAL_CUDA(cudaStreamEndCapture(stream, &tmp));
    stream = outer;
    --side_depth;
    last_body_kernels = t_launch_count - kb;
    if (side_depth == 0) body_kernels_captured += last_body_kernels;
    XCAL_CUDA(cudaStreamUpdateCaptureDependencies(stream, &node, 1, cudaStreamSetCaptureDependencies));
}

// solve_system! captured: per-solve setup, the Krylov loop as a WHILE node
// (bodies of 4 CG / 1 BiCGSTAB iterations, at most itmax/BODY + 2 bodies), the FP64 residual
// into gres and (iterations, status) into giters.  Mixed precision nests the
// inner loop in a WHILE node over defect-correction steps.
void Case::solve_captured(int eqn, int comp) {
    const SolveRef R = solve_ref(eqn, comp);
    Equation& E = *R.E;
    const xcal_solver_setup& SS = R.SS;
    double* field = R.field;
    const double* b = R.b;
    KScalars* S = ws.S.p + R.kslot;
    const int n = E.n;
    const int slot = R.slot;
    CSRView A = E.view();
    const int itmax = SS.itmax == 0 ? 2 * n : SS.itmax;
    // iterations per loop body: a finished solve wastes at most BODY-1
    // early-exit iterations; a BiCGSTAB iteration is already tens of
    // launches (two SpMVs, two preconditioner sweeps), a CG iteration two
    const int BODY = SS.solver == XCAL_SOLVER_CG ? 4 : 1;
    const int cap = itmax / BODY + 2;
    const bool mixed = cfg.precision == XCAL_PREC_MIXED;
    const double inner_rtol = cfg.inner_rtol > 0 ? cfg.inner_rtol : 1e-3;
    kr_ks_init(stream, S, SS.atol, SS.rtol, itmax, mixed ? 1 : 0, inner_rtol);
    // the CG loop as one cooperative kernel node where the driver runs those
    // in graphs (top level; inside the mixed outer WHILE body), its barrier
    // error flag cleared once per step and read after each replay
    // (only the launch forms the driver runs inside graphs; -1: none)
    int pwidth = persistent_cg > 1 ? persistent_cg : 0;
    if (!kr_cluster_capture_ok(mixed)) {
        if (pwidth == PERSIST_CLUSTER_ONLY) pwidth = -1;
        if (pwidth == 0) pwidth = PERSIST_COOP_ONLY;
    }
    if (!kr_coop_capture_ok(mixed) && pwidth != PERSIST_CLUSTER_ONLY && pwidth != -1)
        pwidth = pwidth == 0 ? PERSIST_CLUSTER_ONLY : -1;
    const bool persist = SS.solver == XCAL_SOLVER_CG && persistent_cg && pwidth != -1 &&
                         (SS.precond == XCAL_PRECOND_JACOBI || SS.precond == XCAL_PRECOND_NONE);
    const int jac = SS.precond == XCAL_PRECOND_JACOBI ? 1 : 0;
    if (!mixed) {
        if (SS.precond == XCAL_PRECOND_DILU) dilu_refresh(E, false);
        KrylovVecs<double> V{ws.x.p, ws.r.p, ws.z.p, ws.p.p, ws.q.p, ws.v.p, ws.s.p, ws.t.p};
        const double* r0 = SS.solver == XCAL_SOLVER_CG ? V.r : V.q;
        kr_init_resid(stream, A, E.nz.p, b, field, ws.dx.p, V.x, SS.solver == XCAL_SOLVER_CG ? V.r : V.q);
        krylov_start<double>(E, SS, E.nz.p, E.P.p, b, r0, V, S);
        const bool ran = persist && kr_cg_persist(stream, A, E.nz.p, E.P.p, jac, V.x, V.r, jac ? V.z : V.r, V.p, V.v,
                                                  S, ws.part0.p, ws.part1.p, ws.bar.p, ws.err.p, itmax + 1, pwidth,
                                                  E.nnz * 12L <= PERSIST_PF_MAX_BYTES ? 256 : 0, false);
        if (!ran)
            capture_while([&](cudaGraphConditionalHandle h) {
                const long long k0 = t_launch_count;
                for (int i = 0; i < BODY; ++i) krylov_step<double>(E, SS, E.nz.p, E.P.p, b, V, S, nullptr, true);
                kr_loop_cond(stream, h, S, cap, (int)(t_launch_count - k0) + 1, dlaunch.p);
            });
        kr_finish(stream, n, V.x, ws.dx.p, field);
    } else if (use_fold(E, SS, true) && E.fold_built && E.fold_uniform_ok == fold_uniform_ok()) {
        // folded FP32 CG (cg_folded.cu): each defect step is the scaled
        // defect, the start, and one cooperative node that also applies the
        // correction
        kr_fold_scale(stream, E.fold_mut(), E.nz.p, E.d_diag.p, E.P.p);
        KrylovVecs<float> V{ws.fx.p, ws.fr.p, ws.fz.p, ws.fp.p, ws.fq.p, ws.fv.p, ws.fs.p, ws.ft.p};
        capture_while([&](cudaGraphConditionalHandle ho) {
            const long long k0 = t_launch_count;
            kr_outer_prep(stream, S);
            kr_fold_defect(stream, A, E.nz.p, b, field, E.P.p, ws.frp.p);
            kr_fold_start(stream, n, ws.frp.p, S, ws.part0.p);
            if (!kr_cgf_persist(stream, E.fold_view(), ws.frp.p, ws.frp.p + n, V.x, field, E.P.p, S, ws.fpart.p,
                                ws.fpart.p + FOLD_MAX_BLOCKS, ws.bar.p, ws.err.p, itmax + 1, false, fold_form(),
                                fold_smem()))
                fail(XCAL_ERR_UNSUPPORTED, "folded CG: the system does not fit one block per SM");
            kr_outer_cond(stream, ho, S, 64, (int)(t_launch_count - k0) + 1, dlaunch.p);
        });
    } else {
        kr_to_float(stream, E.nnz, E.nz.p, E.nz32.p);
        if (SS.precond != XCAL_PRECOND_NONE) kr_to_float(stream, n, E.P.p, E.P32.p);
        if (SS.precond == XCAL_PRECOND_DILU) dilu_refresh(E, true);
        KrylovVecs<float> V{ws.fx.p, ws.fr.p, ws.fz.p, ws.fp.p, ws.fq.p, ws.fv.p, ws.fs.p, ws.ft.p};
        const bool cg = SS.solver == XCAL_SOLVER_CG;
        float* rhs = cg ? V.r : ws.fd.p;
        capture_while([&](cudaGraphConditionalHandle ho) {
            const long long k0 = t_launch_count;
            kr_outer_prep(stream, S);
            kr_defect(stream, A, E.nz.p, b, field, rhs, V.x);
            krylov_start<float>(E, SS, E.nz32.p, E.P32.p, (const float*)rhs, (const float*)rhs, V, S);
            const bool ran =
                persist && kr_cg_persist(stream, A, E.nz32.p, E.P32.p, jac, V.x, V.r, jac ? V.z : V.r, V.p, V.v, S,
                                         ws.part0.p, ws.part1.p, ws.bar.p, ws.err.p, itmax + 1, pwidth,
                                         E.nnz * 8L <= PERSIST_PF_MAX_BYTES ? 256 : 0, false);
            if (!ran)
                capture_while([&](cudaGraphConditionalHandle hi) {
                    const long long k1 = t_launch_count;
                    for (int i = 0; i < BODY; ++i)
                        krylov_step<float>(E, SS, E.nz32.p, E.P32.p, (const float*)rhs, V, S, nullptr, true);
                    kr_loop_cond(stream, hi, S, cap, (int)(t_launch_count - k1) + 1, dlaunch.p);
                });
            const long long inner_body = ran ? 0 : last_body_kernels;
            kr_correct_masked(stream, n, field, V.x, S);
            // this body's own kernels (the inner loop's bodies count themselves)
            const long long outer_kernels = t_launch_count - k0 - inner_body + 1;
            kr_outer_cond(stream, ho, S, 64, (int)outer_kernels, dlaunch.p);
        });
    }
    kr_residual(stream, A, E.nz.p, field, b, S, ws.part0.p, ws.part1.p, gres.p + slot);
    kr_record(stream, S, giters.p + 2 * slot);
}

// apply_smoother!(setup.smoother, values, A, b) (Solve_1_api.jl:284): the
// Jacobi smoother on the field, before the Krylov solve of (eqn, comp)
void Case::smooth(int eqn, int comp) {
    const SolveRef R = solve_ref(eqn, comp);
    if (R.SS.smoother_loops <= 0) return;
    kr_jacobi_smooth(stream, R.E->view(), R.E->nz.p, R.b, R.field, ws.t.p, R.SS.smoother_loops, R.SS.smoother_omega);
}

Case::SolveRef Case::solve_ref(int eqn, int comp) {
    switch (eqn) {
        case XCAL_EQN_U:
            return {&U, cfg.U_solver, Uc[comp].p, U.b[comp].p, GRES_U + comp, 0, comp};
        case XCAL_EQN_P:
            return {&P, cfg.p_solver, p.p, P.b[0].p, GRES_P, 1, 3};
        case XCAL_EQN_K:
        case XCAL_EQN_OMEGA: {
            if (eqn == XCAL_EQN_K && keq()) return {&P, cfg.k_solver, kfld.p, P.b[0].p, (int)GRES_K, 1, 4};
            if (!rans_kw()) fail(XCAL_ERR_INVALID, "k / omega equations need RANS{KOmega} or RANS{KOmegaSST}");
            const bool w = eqn == XCAL_EQN_OMEGA;
            SolveRef r{&P, w ? cfg.omega_solver : cfg.k_solver, w ? omega.p : kfld.p, P.b[0].p,
                       w ? (int)GRES_OMEGA : (int)GRES_K, 1, w ? 5 : 4};
            // k-omega: omega with k's preconditioner; SST and LKE: each its own
            // (RANS_kOmegaSST.jl:163-164, RANS_kOmegaLKE.jl:210-212)
            r.SS.precond = (w && (sst() || lke())) ? cfg.omega_solver.precond : cfg.k_solver.precond;
            return r;
        }
        case XCAL_EQN_KL:
            if (!lke()) fail(XCAL_ERR_INVALID, "the kl equation needs RANS{KOmegaLKE}");
            return {&P, cfg.kl_solver, kl.p, P.b[0].p, GRES_KL, 1, 7};
        case XCAL_EQN_WALLDIST:
            if (!has_y()) fail(XCAL_ERR_INVALID, "the wall distance needs RANS{KOmegaSST} or RANS{KOmegaLKE}");
            return {&P, cfg.y_solver, yphi.p, P.b[0].p, GRES_K, 1, 6};
        default:
            fail(XCAL_ERR_INVALID, "unknown equation");
    }
    return {};
}

// solve_system! (Solve_1_api.jl:268-307)
double Case::solve_system(int eqn, int comp, int* iters) {
    smooth(eqn, comp);
    if (capturing) {  // graph mode: residual goes to gres
        solve_captured(eqn, comp);
        return 0.0;
    }
    return solve_system_ref(solve_ref(eqn, comp), iters, false);
}

// the host-polled solve of one system R (fp64: the plain FP64 path whatever
// the case's precision)
double Case::solve_system_ref(const SolveRef& R, int* iters, bool fp64) {
    static const char* const names[7] = {"solve Ux", "solve Uy", "solve Uz", "solve p", "solve k", "solve omega",
                                         "solve wall distance"};
    NvtxRange range(names[R.gk >= 0 && R.gk < 7 ? R.gk : 3]);
    Equation& E = *R.E;
    const xcal_solver_setup& SS = R.SS;
    double* field = R.field;
    const double* b = R.b;
    KScalars* S = ws.S.p + R.kslot;
    KScalars* hS = h_S + R.kslot;
    int n = E.n;
    CSRView A = E.view();
    const double* nz = E.nz.p;
    std::memset(hS, 0, sizeof(KScalars));
    hS->atol = SS.atol;
    hS->rtol = SS.rtol;
    hS->itmax = SS.itmax == 0 ? 2 * n : SS.itmax;
    const int gk = R.gk;
    // the DILU factor and applications as cooperative launches report a
    // barrier wait that gave up through ws.err, read back with the residual
    // below (it stays 0 otherwise)
    const bool grid_dilu = SS.precond == XCAL_PRECOND_DILU && E.use_grid && !E.dilu_block();
    if (cfg.precision == XCAL_PREC_MIXED && !fp64) {
        solve_mixed(E, SS, field, b, S, hS, gk, iters);
    } else {
        XCAL_CUDA(cudaMemcpyAsync(S, hS, sizeof(KScalars), cudaMemcpyHostToDevice, stream));
        if (SS.precond == XCAL_PRECOND_DILU) dilu_refresh(E, false);
        KrylovVecs<double> V{ws.x.p, ws.r.p, ws.z.p, ws.p.p, ws.q.p, ws.v.p, ws.s.p, ws.t.p};
        if (SS.solver == XCAL_SOLVER_CG) {
            kr_init_resid(stream, A, nz, b, field, ws.dx.p, V.x, V.r);
            krylov_iterate<double>(E, SS, nz, E.P.p, b, V.r, V, S, hS, gk);
        } else {
            kr_init_resid(stream, A, nz, b, field, ws.dx.p, V.x, V.q);  // r0 in q
            krylov_iterate<double>(E, SS, nz, E.P.p, b, V.q, V, S, hS, gk);
        }
        kr_finish(stream, n, V.x, ws.dx.p, field);
        if (iters) *iters = hS->iter;
    }
    note_status(gk, hS->status);
    // residual (Solve_1_api.jl:441-464), FP64 in both modes
    kr_residual(stream, A, nz, field, b, S, ws.part0.p, ws.part1.p, resbuf.p);
    XCAL_CUDA(cudaMemcpyAsync(h_res, resbuf.p, sizeof(double), cudaMemcpyDeviceToHost, stream));
    if (grid_dilu) XCAL_CUDA(cudaMemcpyAsync(h_perr, ws.err.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
    sync();
    if (grid_dilu && *h_perr) fail(XCAL_ERR_TIMEOUT, "DILU sweep: a grid barrier wait gave up");
    return h_res[0];
}

bool Case::use_fold(const Equation& E, const xcal_solver_setup& SS, bool captured) const {
    if (cfg.precision != XCAL_PREC_MIXED || inner_cg == 1 || !persistent_cg) return false;
    if (SS.solver != XCAL_SOLVER_CG || SS.precond != XCAL_PRECOND_JACOBI) return false;
    if (captured && !kr_coop_capture_ok(true)) return false;
    return fold_shape(E.n, fold_form(), fold_smem()).blocks > 0;
}

void Case::fold_iterate(Equation& E, double* field, const KrylovVecs<float>& V, KScalars* S, KScalars* hS, int gk) {
    (void)gk;
    kr_fold_start(stream, E.n, ws.frp.p, S, ws.part0.p);
    if (profiling) XCAL_CUDA(cudaEventRecord(ev[5], stream));
    if (!kr_cgf_persist(stream, E.fold_view(), ws.frp.p, ws.frp.p + E.n, V.x, field, E.P.p, S, ws.fpart.p,
                        ws.fpart.p + FOLD_MAX_BLOCKS, ws.bar.p, ws.err.p, hS->itmax + 1, true, fold_form(),
                        fold_smem()))
        fail(XCAL_ERR_UNSUPPORTED, "folded CG: the system does not fit one block per SM");
    if (profiling) XCAL_CUDA(cudaEventRecord(ev[6], stream));
    int errflag = 0;
    XCAL_CUDA(cudaMemcpyAsync(hS, S, sizeof(KScalars), cudaMemcpyDeviceToHost, stream));
    XCAL_CUDA(cudaMemcpyAsync(&errflag, ws.err.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
    sync();
    if (errflag) fail(XCAL_ERR_TIMEOUT, "folded CG: a grid barrier wait gave up");
    if (!hS->done) fail(XCAL_ERR_TIMEOUT, "folded CG did not report completion");
    if (profiling) {
        float t = 0;
        XCAL_CUDA(cudaEventElapsedTime(&t, ev[5], ev[6]));
        prof_ms[5] += t;
        prof_n[5] += hS->iter;
        prof_n[4] += hS->iter + (hS->status == KS_ZERO_CURV ? 1 : 0);
    }
}

// Mixed precision: FP64 defect correction around FP32 Krylov solves.  Each
// step forms d = b - A x in FP64 (A, b, x all FP64), solves A32 e = d32 in
// FP32 from e = 0 with the FP32 copy of the preconditioner, and adds e to x
// in FP64.  The loop ends when the inner solver's initial monitored norm of a
// fresh defect is below the FP64 path's own target atol + rtol*||r0|| (r0 =
// the first defect), so both modes stop on the same criterion; each inner
// solve stops at max(target, inner_rtol * its initial norm).
void Case::solve_mixed(Equation& E, const xcal_solver_setup& SS, double* field, const double* b, KScalars* S,
                       KScalars* hS, int gk, int* iters) {
    const int n = E.n;
    CSRView A = E.view();
    const bool fold = use_fold(E, SS, false);
    if (fold) {
        build_fold(E, stream, fold_uniform_ok());
        kr_fold_scale(stream, E.fold_mut(), E.nz.p, E.d_diag.p, E.P.p);
    } else {
        kr_to_float(stream, E.nnz, E.nz.p, E.nz32.p);
        if (SS.precond != XCAL_PRECOND_NONE) kr_to_float(stream, n, E.P.p, E.P32.p);
        if (SS.precond == XCAL_PRECOND_DILU) dilu_refresh(E, true);
    }
    KrylovVecs<float> V{ws.fx.p, ws.fr.p, ws.fz.p, ws.fp.p, ws.fq.p, ws.fv.p, ws.fs.p, ws.ft.p};
    hS->mixed = 1;
    hS->inner_rtol = cfg.inner_rtol > 0 ? cfg.inner_rtol : 1e-3;
    int total = 0;
    const int max_outer = 64;
    for (int outer = 0; outer < max_outer; ++outer) {
        hS->outer = outer;
        hS->iter = 0;
        hS->done = 0;
        hS->status = KS_RUNNING;
        XCAL_CUDA(cudaMemcpyAsync(S, hS, sizeof(KScalars), cudaMemcpyHostToDevice, stream));
        if (fold) {
            // scaled defect, inner solve, and the correction applied by the
            // solve's own kernel (unless this defect met the target)
            kr_fold_defect(stream, A, E.nz.p, b, field, E.P.p, ws.frp.p);
            fold_iterate(E, field, V, S, hS, gk);
            if (hS->outer_conv) break;
            total += hS->iter;
            if (hS->status == KS_ZERO_CURV || hS->status == KS_BREAKDOWN || hS->status == KS_TIRED) break;
            if (hS->status == KS_SOLVED && hS->eps <= hS->eps_outer) break;
            continue;
        }
        if (SS.solver == XCAL_SOLVER_CG) {
            kr_defect(stream, A, E.nz.p, b, field, V.r, V.x);
            krylov_iterate<float>(E, SS, E.nz32.p, E.P32.p, (const float*)V.r, V.r, V, S, hS, gk);
        } else {
            kr_defect(stream, A, E.nz.p, b, field, ws.fd.p, V.x);
            krylov_iterate<float>(E, SS, E.nz32.p, E.P32.p, (const float*)ws.fd.p, ws.fd.p, V, S, hS, gk);
        }
        if (hS->outer_conv) break;  // this defect already met the target
        total += hS->iter;
        kr_correct(stream, n, field, V.x);
        if (hS->status == KS_ZERO_CURV || hS->status == KS_BREAKDOWN || hS->status == KS_TIRED) break;
        // An inner solve whose own target was the outer target and that met
        // it leaves a defect at that target up to FP32 rounding of d (about
        // 1e-7 relative): no further FP64 check is needed.
        if (hS->status == KS_SOLVED && hS->eps <= hS->eps_outer) break;
    }
    last_outer[gk] = hS->outer + 1;
    if (iters) *iters = total;
}

void Case::solve_equation_U(double res[3]) {  // Solve_1_api.jl:233-266
    discretise(XCAL_EQN_U);
    for (int d = 0; d < 3; ++d) {
        bc_relax_U(d);
        if (d == 0) update_precond(XCAL_EQN_U);
        res[d] = solve_system(XCAL_EQN_U, d, &last_iters[d]);
    }
}

double Case::solve_equation_p() {  // Solve_1_api.jl:214-231
    discretise(XCAL_EQN_P);
    apply_bcs(XCAL_EQN_P, 0);
    set_reference();
    update_precond(XCAL_EQN_P);
    return solve_system(XCAL_EQN_P, 0, &last_iters[3]);
}

void Case::pressure_predictor(bool with_H) {  // Solvers_1_SIMPLE.jl:170-174
    const double* Ucp[3] = {Uc[0].p, Uc[1].p, Uc[2].p};
    const double* gp[3] = {gradp[0].p, gradp[1].p, gradp[2].p};
    double* bp[3] = {U.b[0].p, U.b[1].p, U.b[2].p};
    double* Hp[3] = {Hv[0].p, Hv[1].p, Hv[2].p};
    launch_rD_remove_H(stream, mv(), U.view(), U.nz.p, Ucp, gp, bp, rD.p, Hp, with_H ? 1 : 0);
    launch_interp_rD(stream, mv(), bcU.view(), rD.p, rDf.p);
}

void Case::H() {
    const double* Ucp[3] = {Uc[0].p, Uc[1].p, Uc[2].p};
    const double* bp[3] = {U.b[0].p, U.b[1].p, U.b[2].p};
    double* Hp[3] = {Hv[0].p, Hv[1].p, Hv[2].p};
    launch_H(stream, mv(), U.view(), U.nz.p, Ucp, bp, Hp);
}

void Case::flux_divergence() {  // Solvers_1_SIMPLE.jl:177-185
    const double* Hp[3] = {Hv[0].p, Hv[1].p, Hv[2].p};
    double* Ufp[3] = {Uf[0].p, Uf[1].p, Uf[2].p};
    launch_interp_U(stream, mv(), bcU.view(), Hp, Ufp, mdot.p);
    launch_div(stream, mv(), mdot.p, divHv.p);
}

void Case::explicit_relaxation_p(double a) { launch_relax_explicit(stream, mesh->nC, p.p, prev.p, a); }

// The face constants of nonorthogonal_face_correction (Solvers_1_SIMPLE.jl:
// 267-333), per internal face in storage order, on the host once: the
// interpolation weight w of correction_weight, e, and T = Sf - Ef with
// Ef = dPN (|n|^2 / (dPN.n)) area.  Layout: 7 arrays of nI (w, ex, ey, ez,
// Tx, Ty, Tz).
void Case::build_nonorth(const DevMesh& m, cudaStream_t s) {
    const int nB = m.nB, nI = m.nI;
    std::vector<double> t(7 * (size_t)nI);
    for (int j = 0; j < nI; ++j) {
        const int f = nB + j, c1 = m.owner[f], c2 = m.neigh[f];
        const double xCx = m.ccx[c1], xCy = m.ccy[c1], xCz = m.ccz[c1];
        const double xNx = m.ccx[c2], xNy = m.ccy[c2], xNz = m.ccz[c2];
        // correction_weight
        const double afx = m.fcx[f] - xCx, afy = m.fcy[f] - xCy, afz = m.fcz[f] - xCz;
        const double acx = xNx - xCx, acy = xNy - xCy, acz = xNz - xCz;
        const double q = (afx * acx + afy * acy + afz * acz) / (acx * acx + acy * acy + acz * acz);
        const double fpx = xCx - q * (xCx - xNx), fpy = xCy - q * (xCy - xNy), fpz = xCz - q * (xCz - xNz);
        const double d1x = xNx - fpx, d1y = xNy - fpy, d1z = xNz - fpz;
        const double d2x = xNx - xCx, d2y = xNy - xCy, d2z = xNz - xCz;
        const double w = std::sqrt(d1x * d1x + d1y * d1y + d1z * d1z) / std::sqrt(d2x * d2x + d2y * d2y + d2z * d2z);
        // T = Sf - Ef
        const double nx = m.nxh[f], ny = m.nyh[f], nz = m.nzh[f], a = m.area[f];
        const double nr = std::sqrt(nx * nx + ny * ny + nz * nz);
        const double nn = nr * nr;
        const double dn = acx * nx + acy * ny + acz * nz;
        const double r = nn / dn;
        t[j] = w;
        t[nI + (size_t)j] = m.ex[f];
        t[2 * (size_t)nI + j] = m.ey[f];
        t[3 * (size_t)nI + j] = m.ez[f];
        t[4 * (size_t)nI + j] = a * nx - (acx * r) * a;
        t[5 * (size_t)nI + j] = a * ny - (acy * r) * a;
        t[6 * (size_t)nI + j] = a * nz - (acz * r) * a;
    }
    nonorth.upload(t, s);
}

void Case::nonorth_correct() {
    const double* gp[3] = {gradp[0].p, gradp[1].p, gradp[2].p};
    launch_nonorth_correct(stream, mv(), nonorth.p, p.p, gp, rDf.p, P.b[0].p);
}

// the non-orthogonal correctors of a SIMPLE iteration (Solvers_1_SIMPLE.jl:
// 196-206); rp becomes the last corrector solve's residual
void Case::nonorth_correctors(double& rp) {
    for (int k = 0; k < cfg.ncorrectors; ++k) {
        discretise(XCAL_EQN_P);
        apply_bcs(XCAL_EQN_P, 0);
        nonorth_correct();
        rp = solve_system(XCAL_EQN_P, 0, &last_iters[3]);
        explicit_relaxation_p(cfg.p_solver.relax);
        grad_p();
    }
}

// grad! + limit_gradient!(schemes.p.limiter) (Solvers_1_SIMPLE.jl:153-154,
// 192-193, 205-206): Gauss (Calculate_0_gradient.jl:105-111) or Midpoint
// (:249-258), then the CellBased limiter when configured
void Case::grad_p() {
    launch_interp_scalar(stream, mv(), bcP.view(), p.p, pf.p, nullptr, 0.0);
    double* gp[3] = {gradp[0].p, gradp[1].p, gradp[2].p};
    if (cfg.p_schemes.gradient == XCAL_GRAD_MIDPOINT) {
        const double* gc[3] = {gradp[0].p, gradp[1].p, gradp[2].p};
        launch_mid_scalar(stream, mv(), p.p, pf.p);
        launch_green_gauss(stream, mv(), pf.p, gp);
        for (int it = 0; it < 2; ++it) {
            launch_mid_correct_scalar(stream, mv(), midR.p, p.p, gc, pf.p);
            launch_green_gauss(stream, mv(), pf.p, gp);
        }
    } else {
        launch_green_gauss(stream, mv(), pf.p, gp);
    }
    if (cfg.p_schemes.limiter == XCAL_LIMITER_CELL)
        launch_limit_cell(stream, mv(), limD.p, p.p, gp, cfg.p_schemes.limiter_level);
    else if (cfg.p_schemes.limiter == XCAL_LIMITER_FACE)
        launch_limit_face_scalar(stream, mv(), limD.p, p.p, gp);
    else if (cfg.p_schemes.limiter == XCAL_LIMITER_MFACE)
        launch_limit_mface_scalar(stream, mv(), limOrd.p, limD.p, p.p, gp);
}

// fc - cc per cell_faces entry (storage order), 3 arrays of 2 nI
void Case::build_limiter(const DevMesh& m, cudaStream_t s) {
    const size_t nk = m.cf_face.size();
    std::vector<double> t(3 * nk);
    for (int i = 0; i < m.nC; ++i)
        for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
            const int f = m.cf_face[k];
            t[k] = m.fcx[f] - m.ccx[i];
            t[nk + k] = m.fcy[f] - m.ccy[i];
            t[2 * nk + k] = m.fcz[f] - m.ccz[i];
        }
    limD.upload(t, s);
    // MFaceBased: per cell its entries by the reference's face id (fperm
    // maps storage faces back to it)
    std::vector<int> ord(nk);
    for (int i = 0; i < m.nC; ++i) {
        std::iota(ord.begin() + m.cf_off[i], ord.begin() + m.cf_off[i + 1], m.cf_off[i]);
        std::sort(ord.begin() + m.cf_off[i], ord.begin() + m.cf_off[i + 1],
                  [&](int a, int b) { return m.fperm[m.cf_face[a]] < m.fperm[m.cf_face[b]]; });
    }
    limOrd.upload(ord, s);
}

// Ri = rf - 0.5 (rP + rN) per internal face (correct_interpolation!,
// Calculate_0_gradient.jl:214-246), storage order; 3 arrays of nI
void Case::build_midpoint(const DevMesh& m, cudaStream_t s) {
    const int nB = m.nB, nI = m.nI;
    std::vector<double> t(3 * (size_t)nI);
    for (int j = 0; j < nI; ++j) {
        const int f = nB + j, c1 = m.owner[f], c2 = m.neigh[f];
        t[j] = m.fcx[f] - 0.5 * (m.ccx[c1] + m.ccx[c2]);
        t[nI + (size_t)j] = m.fcy[f] - 0.5 * (m.ccy[c1] + m.ccy[c2]);
        t[2 * (size_t)nI + j] = m.fcz[f] - 0.5 * (m.ccz[c1] + m.ccz[c2]);
    }
    midR.upload(t, s);
}

void Case::correct() {  // Solvers_1_SIMPLE.jl:210-211
    launch_correct_mdot(stream, mv(), P.view(), bcP.view(), P.nz.p, p.p, rDf.p, mdot.p);
    double* Hp[3] = {Hv[0].p, Hv[1].p, Hv[2].p};
    const double* gp[3] = {gradp[0].p, gradp[1].p, gradp[2].p};
    double* Ucp[3] = {Uc[0].p, Uc[1].p, Uc[2].p};
    launch_correct_U(stream, mesh->nC, Hp, gp, rD.p, Ucp);
}

void Case::turbulence() {
    const double* Ucp[3] = {Uc[0].p, Uc[1].p, Uc[2].p};
    double* Ufp[3] = {Uf[0].p, Uf[1].p, Uf[2].p};
    launch_interp_U(stream, mv(), bcU.view(), Ucp, Ufp, nullptr);
    double* g[9];
    for (int q = 0; q < 9; ++q) g[q] = gradU[q].p;
    const bool les = cfg.turbulence == XCAL_TURB_SMAGORINSKY;  // nut from grad U alone
    const bool limit = cfg.U_schemes.limiter != XCAL_LIMITER_NONE;
    // nut fused into the last Green-Gauss pass unless the limiter comes between
    double* nut_gg = les && !limit ? nut.p : nullptr;
    if (cfg.U_schemes.gradient == XCAL_GRAD_MIDPOINT) {
        // Midpoint (Calculate_0_gradient.jl:249-258); nut from the last pass
        const double* gc[9];
        for (int q = 0; q < 9; ++q) gc[q] = gradU[q].p;
        launch_mid_vector(stream, mv(), Ucp, Ufp);
        launch_green_gauss_tensor(stream, mv(), Ufp, g, Delta.p, nullptr);
        for (int it = 0; it < 2; ++it) {
            launch_mid_correct_vector(stream, mv(), midR.p, Ucp, gc, Ufp);
            launch_green_gauss_tensor(stream, mv(), Ufp, g, Delta.p, it == 1 ? nut_gg : nullptr);
        }
    } else {
        launch_green_gauss_tensor(stream, mv(), Ufp, g, Delta.p, nut_gg);
    }
    if (limit) {
        // limit_gradient!(schemes.U.limiter, gradU, U) (RANS_laminar.jl:77,
        // LES_Smagorinsky.jl:120): CellBased once per component row,
        // FaceBased and MFaceBased once for the tensor
        if (cfg.U_schemes.limiter == XCAL_LIMITER_FACE)
            launch_limit_face_vector(stream, mv(), limD.p, Ucp, g);
        else if (cfg.U_schemes.limiter == XCAL_LIMITER_MFACE)
            launch_limit_mface_vector(stream, mv(), limOrd.p, limD.p, Ucp, g);
        else
            for (int a = 0; a < 3; ++a)
                launch_limit_cell(stream, mv(), limD.p, Uc[a].p, g + 3 * a, cfg.U_schemes.limiter_level);
        if (les) launch_smag_nut(stream, mesh->nC, g, Delta.p, nut.p);
    }
    if (lke())
        komega_lke();
    else if (rans_kw())
        komega();
    else if (keq())
        kequation();
    else if (les)
        launch_interp_scalar(stream, mv(), bcNut.view(), nut.p, nutf.p, nueff.p, cfg.nu);
    else
        launch_fill(stream, nueff.p, cfg.nu, mesh->nF);
}

// max Courant number into gres[GRES_CO] (device); the stream-mode caller reads it
void Case::courant_to_slot() {
    const double* Ucp[3] = {Uc[0].p, Uc[1].p, Uc[2].p};
    launch_courant_max(stream, mesh->nC, Ucp, dx13.p, cfg.dt, cmax.p, cmax_ctr.p, gres.p + GRES_CO);
}

double Case::max_courant() {
    courant_to_slot();
    XCAL_CUDA(cudaMemcpyAsync(h_res, gres.p + GRES_CO, sizeof(double), cudaMemcpyDeviceToHost, stream));
    sync();
    return h_res[0];
}

// One SIMPLE iteration's launches (Solvers_1_SIMPLE.jl:164-240).  Eager:
// residuals returned, phases timed with events.  Under capture: residuals
// land in gres, no events.
void Case::simple_body(double r3[3], double& rp, bool timed) {
    NvtxRange range("SIMPLE iteration");
    if (timed) XCAL_CUDA(cudaEventRecord(ev[0], stream));
    {
        NvtxRange r("momentum predictor");
        solve_equation_U(r3);
    }
    if (timed) XCAL_CUDA(cudaEventRecord(ev[1], stream));
    {
        NvtxRange r("pressure predictor + flux divergence");
        pressure_predictor(true);
        flux_divergence();
    }
    XCAL_CUDA(cudaMemcpyAsync(prev.p, p.p, mesh->nC * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    if (timed) XCAL_CUDA(cudaEventRecord(ev[2], stream));
    {
        NvtxRange r("pressure equation");
        rp = solve_equation_p();
        explicit_relaxation_p(cfg.p_solver.relax);
        grad_p();
        nonorth_correctors(rp);
    }
    if (timed) XCAL_CUDA(cudaEventRecord(ev[3], stream));
    {
        NvtxRange r("correction + turbulence");
        correct();
        turbulence();
    }
    if (timed) XCAL_CUDA(cudaEventRecord(ev[4], stream));
}

// One PISO time step's launches (Solvers_2_PISO.jl:108-187); the Courant
// number is left in gres[GRES_CO].
void Case::piso_body(double r3[3], double& rp) {
    NvtxRange range("PISO step");
    {
        NvtxRange r("momentum predictor");
        solve_equation_U(r3);
    }
    pressure_predictor(false);
    rp = 0.0;
    for (int it = 1; it <= cfg.inner_loops; ++it) {
        NvtxRange r("pressure corrector");
        H();
        flux_divergence();
        XCAL_CUDA(cudaMemcpyAsync(prev.p, p.p, mesh->nC * sizeof(double), cudaMemcpyDeviceToDevice, stream));
        rp = solve_equation_p();
        explicit_relaxation_p(it == cfg.inner_loops ? 1.0 : cfg.p_solver.relax);
        grad_p();
        correct();
    }
    {
        NvtxRange r("turbulence");
        turbulence();
    }
    courant_to_slot();
}

// Capture one step (SIMPLE iteration or PISO step, by the configured
// algorithm) into step_graph.  Everything a step reads is either device state
// or fixed for the case (coefficients, relaxation, dt), so the graph is
// captured once and replayed for every later step.
void Case::capture_step() {
    if (step_graph) return;
    autotune();
    sync();
    const long long t0 = t_launch_count;
    body_kernels_captured = 0;
    capturing = true;
    cudaGraph_t g = nullptr;
    // decided before the capture (the check runs graphs of its own)
    kr_coop_capture_ok(false);
    kr_cluster_capture_ok(false);
    if (cfg.precision == XCAL_PREC_MIXED) {
        kr_coop_capture_ok(true);
        kr_cluster_capture_ok(true);
        // the folded inner CG's storage (uploads) cannot be made under capture
        if (use_fold(P, cfg.p_solver, true)) build_fold(P, stream, fold_uniform_ok());
    }
    XCAL_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    try {
        XCAL_CUDA(cudaMemsetAsync(ws.err.p, 0, sizeof(int), stream));
        double r3[3], rp;
        if (cfg.algorithm == XCAL_ALGO_PISO)
            piso_body(r3, rp);
        else
            simple_body(r3, rp, false);
    } catch (...) {
        capturing = false;
        cudaStreamEndCapture(stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    capturing = false;
    XCAL_CUDA(cudaStreamEndCapture(stream, &g));
    const long long captured = t_launch_count - t0;
    g_launch_count.fetch_sub(captured, std::memory_order_relaxed);
    t_launch_count = t0;
    step_top_kernels = captured - body_kernels_captured;
    cudaError_t e = cudaGraphInstantiate(&step_graph, g, 0);
    cudaGraphDestroy(g);
    XCAL_CUDA(e);
}

// Replay the step graph; one host synchronisation reads the residuals, the
// Courant number, the solves' iteration counts and the body-kernel count.
void Case::run_step_graph(double res[4], double* courant) {
    capture_step();
    XCAL_CUDA(cudaEventRecord(ev[0], stream));
    XCAL_CUDA(cudaGraphLaunch(step_graph, stream));
    XCAL_CUDA(cudaEventRecord(ev[1], stream));
    XCAL_CUDA(cudaMemcpyAsync(h_res, gres.p, GRES_N * sizeof(double), cudaMemcpyDeviceToHost, stream));
    XCAL_CUDA(cudaMemcpyAsync(h_iters, giters.p, 2 * GRES_N * sizeof(int), cudaMemcpyDeviceToHost, stream));
    XCAL_CUDA(cudaMemcpyAsync(h_launch, dlaunch.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream));
    XCAL_CUDA(cudaMemsetAsync(dlaunch.p, 0, sizeof(unsigned long long), stream));
    XCAL_CUDA(cudaMemcpyAsync(h_perr, ws.err.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
    sync();
    if (*h_perr) fail(XCAL_ERR_TIMEOUT, "persistent CG: a grid barrier wait gave up (graph mode)");
    long long nk = step_top_kernels + (long long)h_launch[0];
    g_launch_count.fetch_add(nk, std::memory_order_relaxed);
    t_launch_count += nk;
    float t = 0;
    cudaEventElapsedTime(&t, ev[0], ev[1]);
    ms[5] += t;
    for (int k = 0; k < 4; ++k) {
        res[k] = h_res[k];
        last_iters[k] = h_iters[2 * k];
        if (h_iters[2 * k + 1] == KS_LOOP_CAP)
            fail(XCAL_ERR_TIMEOUT, "a Krylov solve did not finish within its loop-body cap");
        note_status(k, h_iters[2 * k + 1]);
    }
    if (courant) *courant = h_res[GRES_CO];
}

bool Case::simple_iteration(double res[4]) {  // Solvers_1_SIMPLE.jl:164-240
    if (!initialised) initial_calculations();
    autotune();
    iteration += 1;
    double r3[3], rp;
    if (graph_mode) {
        double r[4];
        run_step_graph(r, nullptr);
        r3[0] = r[0];
        r3[1] = r[1];
        r3[2] = r[2];
        rp = r[3];
    } else {
        simple_body(r3, rp, true);
        sync();
        float a = 0, b = 0, c = 0, d = 0;
        cudaEventElapsedTime(&a, ev[0], ev[1]);
        cudaEventElapsedTime(&b, ev[1], ev[2]);
        cudaEventElapsedTime(&c, ev[2], ev[3]);
        cudaEventElapsedTime(&d, ev[3], ev[4]);
        ms[1] += a;
        ms[3] += b + d;
        ms[2] += c;
        ms[5] += a + b + c + d;
    }
    res[0] = r3[0];
    res[1] = r3[1];
    res[2] = r3[2];
    res[3] = rp;
    for (int k = 0; k < 4; ++k)
        if (std::isnan(res[k]) || std::isinf(res[k])) fail(XCAL_ERR_DIVERGED, "residual is NaN/Inf");
    bool turb_conv = cfg.turbulence == XCAL_TURB_LAMINAR;
    // Uz enters the test on 3D meshes only (Solvers_1_SIMPLE.jl:220-223)
    const bool uz_conv = mesh->dim == 2 || r3[2] <= cfg.U_solver.convergence;
    return r3[0] <= cfg.U_solver.convergence && r3[1] <= cfg.U_solver.convergence && uz_conv &&
           rp <= cfg.p_solver.convergence && turb_conv;
}

double Case::piso_step(double res[4]) {  // Solvers_2_PISO.jl:108-187
    if (!initialised) initial_calculations();
    autotune();
    iteration += 1;
    time = time + cfg.dt;
    double r3[3], rp, co;
    if (graph_mode) {
        double r[4];
        run_step_graph(r, &co);
        r3[0] = r[0];
        r3[1] = r[1];
        r3[2] = r[2];
        rp = r[3];
    } else {
        XCAL_CUDA(cudaEventRecord(ev[0], stream));
        piso_body(r3, rp);
        XCAL_CUDA(cudaEventRecord(ev[1], stream));
        XCAL_CUDA(cudaMemcpyAsync(h_res + GRES_CO, gres.p + GRES_CO, sizeof(double), cudaMemcpyDeviceToHost, stream));
        sync();
        co = h_res[GRES_CO];
        float t = 0;
        cudaEventElapsedTime(&t, ev[0], ev[1]);
        ms[5] += t;
    }
    res[0] = r3[0];
    res[1] = r3[1];
    res[2] = r3[2];
    res[3] = rp;
    return co;
}

void Case::set_inner_cg(int mode) {
    if (mode == inner_cg) return;
    sync();
    inner_cg = mode;
    if (step_graph) {
        cudaGraphExecDestroy(step_graph);
        step_graph = nullptr;
    }
}

void Case::set_graph_mode(bool on) {
    if (on == graph_mode) return;
    sync();
    if (step_graph) {
        cudaGraphExecDestroy(step_graph);
        step_graph = nullptr;
    }
    graph_mode = on;
}

template void Case::dilu_ldiv<double>(Equation&, const double*, const double*, const double*, double*,
                                      const KScalars*);
template void Case::dilu_ldiv<float>(Equation&, const float*, const float*, const float*, float*, const KScalars*);

}  // namespace xcal

// foam_import.cu -- host-side polyMesh -> Mesh3 import (no GPU needed).
//
// Builds the Mesh3 contract exactly as XCALibre's FOAM3D_mesh does, with every
// floating-point operation in the Julia source's order (host code is compiled
// with -ffp-contract=off):
//   src/FoamMesh/FoamMesh_1_read.jl:25-43      boundary neighbour = owner
//   src/FoamMesh/FoamMesh_2_connect.jl:24-69   cell -> internal faces (owner first, ascending)
//   src/FoamMesh/FoamMesh_2_connect.jl:71-146  cell nodes, first-seen order
//   src/FoamMesh/FoamMesh_2_connect.jl:148-195 boundary faces first
//   src/FoamMesh/FoamMesh_4_geometry.jl:2-158  centres, fan geometry, orientation, volumes
//   src/Mesh/Mesh_1_functions.jl:20-51         weight / delta / e
#include <algorithm>
#include <cmath>
#include <limits>
#include <vector>

#include "../../include/xcal_b200.h"

namespace {

struct P3 {
    double x, y, z;
};
inline P3 add(P3 a, P3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline P3 sub(P3 a, P3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline P3 scl(double s, P3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline P3 dvd(P3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline double dotp(P3 a, P3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double nrm(P3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
inline P3 crs(P3 a, P3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double eps_of(double v) {
    v = std::fabs(v);
    return std::nextafter(v, std::numeric_limits<double>::infinity()) - v;
}
inline double jmax(double x, double y) {  // Julia max for floats
    bool ty = (y > x) || (std::signbit(y) < std::signbit(x));
    return ty ? (std::isnan(x) ? x : y) : (std::isnan(y) ? y : x);
}

int check_pm(const xcal_polymesh_desc* pm) {
    if (!pm || pm->n_points <= 0 || pm->n_faces <= 0 || pm->n_internal_faces < 0 ||
        pm->n_internal_faces > pm->n_faces || !pm->points || !pm->face_offsets || !pm->face_nodes || !pm->owner ||
        (pm->n_internal_faces && !pm->neighbour) || pm->n_patches < 0 || (pm->n_patches && !pm->patch_sizes))
        return XCAL_ERR_INVALID;
    return XCAL_OK;
}

int n_cells_of(const xcal_polymesh_desc* pm) {
    int mx = -1;
    for (int f = 0; f < pm->n_faces; ++f) mx = std::max(mx, pm->owner[f]);
    for (int f = 0; f < pm->n_internal_faces; ++f) mx = std::max(mx, pm->neighbour[f]);
    return mx + 1;
}

}  // namespace

extern "C" int32_t xcal_foam_mesh_sizes(const xcal_polymesh_desc* pm, int32_t* sizes) {
    if (check_pm(pm) || !sizes) return XCAL_ERR_INVALID;
    sizes[0] = n_cells_of(pm);
    sizes[1] = pm->n_faces;
    sizes[2] = pm->n_faces - pm->n_internal_faces;
    return XCAL_OK;
}

extern "C" int32_t xcal_foam_mesh_build(const xcal_polymesh_desc* pm, const xcal_mesh_buffers* o) {
    if (check_pm(pm) || !o) return XCAL_ERR_INVALID;
    const int nF = pm->n_faces, nI = pm->n_internal_faces, nB = nF - nI, nP = pm->n_points;
    const int nC = n_cells_of(pm);
    if (nC <= 0) return XCAL_ERR_INVALID;
    long total_bf = 0;
    for (int p = 0; p < pm->n_patches; ++p) total_bf += pm->patch_sizes[p];
    if (total_bf != nB) return XCAL_ERR_INVALID;
    for (int f = 0; f < nF; ++f)
        if (pm->owner[f] < 0 || pm->face_offsets[f + 1] < pm->face_offsets[f]) return XCAL_ERR_INVALID;
    const int* fo = pm->face_offsets;
    const int* fn = pm->face_nodes;
    for (int k = 0; k < fo[nF]; ++k)
        if (fn[k] < 0 || fn[k] >= nP) return XCAL_ERR_INVALID;
    auto pt = [&](int i) { return P3{pm->points[3 * i], pm->points[3 * i + 1], pm->points[3 * i + 2]}; };
    auto fneigh = [&](int fi) { return fi < nI ? pm->neighbour[fi] : pm->owner[fi]; };

    // cell -> internal faces: counts, offsets, fill in increasing fi, owner then neighbour
    std::vector<int> off(nC + 1, 0);
    for (int fi = 0; fi < nI; ++fi) {
        off[pm->owner[fi] + 1]++;
        off[pm->neighbour[fi] + 1]++;
    }
    for (int c = 0; c < nC; ++c) off[c + 1] += off[c];
    {
        std::vector<int> cur(off.begin(), off.end() - 1);
        for (int fi = 0; fi < nI; ++fi) {
            int a = pm->owner[fi], b = pm->neighbour[fi], fid = fi + nB;
            int k = cur[a]++;
            o->cell_faces[k] = fid;
            o->cell_nsign[k] = 1;
            o->cell_neighbours[k] = b;
            k = cur[b]++;
            o->cell_faces[k] = fid;
            o->cell_nsign[k] = -1;
            o->cell_neighbours[k] = a;
        }
        for (int c = 0; c <= nC; ++c) o->cell_faces_offset[c] = off[c];
    }

    // mesh face order: boundary faces (foam nI..nF-1) then internal (0..nI-1)
    auto src_of = [&](int fid) { return fid < nB ? nI + fid : fid - nB; };
    for (int fid = 0; fid < nF; ++fid) {
        int s = src_of(fid);
        o->face_owner[fid] = pm->owner[s];
        o->face_neigh[fid] = fneigh(s);
    }
    {
        int start = 0;
        for (int p = 0; p < pm->n_patches; ++p) {
            o->patch_start[p] = start;
            o->patch_count[p] = pm->patch_sizes[p];
            start += pm->patch_sizes[p];
        }
    }
    for (int f = 0; f < nB; ++f) o->boundary_cellsID[f] = o->face_owner[f];

    // cell nodes in first-seen order of the raw per-cell list (faces in foam
    // order; owner role then neighbour role) -> cell centres
    {
        std::vector<int> cnt(nC, 0);
        for (int fi = 0; fi < nF; ++fi) {
            int nn = fo[fi + 1] - fo[fi];
            cnt[pm->owner[fi]] += nn;
            cnt[fneigh(fi)] += nn;
        }
        std::vector<long> roff(nC + 1, 0);
        for (int c = 0; c < nC; ++c) roff[c + 1] = roff[c] + cnt[c];
        std::vector<int> raw(roff[nC]);
        std::vector<long> cur(roff.begin(), roff.end() - 1);
        for (int fi = 0; fi < nF; ++fi) {
            int a = pm->owner[fi], b = fneigh(fi);
            for (int k = fo[fi]; k < fo[fi + 1]; ++k) raw[cur[a]++] = fn[k];
            for (int k = fo[fi]; k < fo[fi + 1]; ++k) raw[cur[b]++] = fn[k];
        }
        std::vector<int> seen(nP, -1);
        for (int c = 0; c < nC; ++c) {
            P3 s{0, 0, 0};
            int m = 0;
            for (long k = roff[c]; k < roff[c + 1]; ++k) {
                int nid = raw[k];
                if (seen[nid] != c) {
                    seen[nid] = c;
                    s = add(s, pt(nid));
                    ++m;
                }
            }
            P3 cc = dvd(s, (double)m);
            o->cell_centre[3 * c] = cc.x;
            o->cell_centre[3 * c + 1] = cc.y;
            o->cell_centre[3 * c + 2] = cc.z;
        }
    }
    auto cc = [&](int c) { return P3{o->cell_centre[3 * c], o->cell_centre[3 * c + 1], o->cell_centre[3 * c + 2]}; };

    // faces: node-average apex, fan triangles, orientation, weight/delta/e
    for (int fid = 0; fid < nF; ++fid) {
        int s = src_of(fid);
        int b = fo[s], n = fo[s + 1] - b;
        P3 sum{0, 0, 0};
        for (int k = 0; k < n; ++k) sum = add(sum, pt(fn[b + k]));
        P3 apex = dvd(sum, (double)n);
        P3 area_vec{0, 0, 0}, centre_sum{0, 0, 0};
        double sum_area = 0.0;
        for (int i = 0; i < n; ++i) {
            int j = (i == n - 1) ? 0 : i + 1;
            P3 p1 = pt(fn[b + i]), p2 = pt(fn[b + j]);
            P3 tri = dvd(crs(sub(p1, apex), sub(p2, apex)), 2.0);
            double ta = nrm(tri);
            if (!(ta > 0.0)) continue;
            area_vec = add(area_vec, tri);
            centre_sum = add(centre_sum, dvd(scl(ta, add(add(apex, p1), p2)), 3.0));
            sum_area = sum_area + ta;
        }
        double mag = nrm(area_vec);
        P3 normal = mag > 0.0 ? dvd(area_vec, mag) : P3{0, 0, 0};
        P3 centre = sum_area > 0.0 ? dvd(centre_sum, sum_area) : apex;
        double weight, delta;
        P3 e;
        if (fid < nB) {
            P3 C1F1 = sub(centre, cc(o->face_owner[fid]));
            if (dotp(C1F1, normal) < 0.0) normal = scl(-1.0, normal);
            weight = 1.0;
            delta = nrm(C1F1);
            e = delta > 0.0 ? dvd(C1F1, delta) : normal;
            delta = jmax(delta, eps_of(1.0));
        } else {
            P3 C1 = cc(o->face_owner[fid]), C2 = cc(o->face_neigh[fid]);
            P3 C1F1 = sub(centre, C1), C2F1 = sub(centre, C2), C1C2 = sub(C2, C1);
            if (dotp(C1C2, normal) < 0.0) normal = scl(-1.0, normal);
            double proj = dotp(C1C2, normal);
            if (std::isfinite(proj) && std::fabs(proj) > eps_of(proj)) {
                double wi = dotp(C1F1, normal) / proj;
                weight = 1.0 - wi;
            } else {
                double d1 = nrm(C1F1), d2 = nrm(C2F1), ds = d1 + d2;
                weight = ds > 0.0 ? d2 / ds : 0.5;
            }
            delta = nrm(C1C2);
            if (delta > 0.0) {
                e = dvd(C1C2, delta);
            } else {
                delta = nrm(C1F1) + nrm(C2F1);
                e = normal;
            }
            delta = jmax(delta, eps_of(1.0));
            weight = weight > 1.0 ? 1.0 : (weight < 0.0 ? 0.0 : weight);
        }
        // (the negation -normal of the reference flips each sign exactly like -1.0*normal)
        o->face_centre[3 * fid] = centre.x;
        o->face_centre[3 * fid + 1] = centre.y;
        o->face_centre[3 * fid + 2] = centre.z;
        o->face_normal[3 * fid] = normal.x;
        o->face_normal[3 * fid + 1] = normal.y;
        o->face_normal[3 * fid + 2] = normal.z;
        o->face_e[3 * fid] = e.x;
        o->face_e[3 * fid + 1] = e.y;
        o->face_e[3 * fid + 2] = e.z;
        o->face_area[fid] = mag;
        o->face_delta[fid] = delta;
        o->face_weight[fid] = weight;
    }

    // volumes: internal faces in cell_faces order, then boundary faces ascending
    {
        const double oneThird = 1.0 / 3.0;
        std::vector<double> vol(nC, 0.0), maxa(nC, 0.0);
        auto fc = [&](int f) { return P3{o->face_centre[3 * f], o->face_centre[3 * f + 1], o->face_centre[3 * f + 2]}; };
        auto fnm = [&](int f) { return P3{o->face_normal[3 * f], o->face_normal[3 * f + 1], o->face_normal[3 * f + 2]}; };
        for (int c = 0; c < nC; ++c)
            for (int k = off[c]; k < off[c + 1]; ++k) {
                int f = o->cell_faces[k];
                P3 xf = sub(fc(f), cc(c));
                vol[c] = vol[c] + ((oneThird * dotp(xf, fnm(f))) * (double)o->cell_nsign[k]) * o->face_area[f];
                maxa[c] = jmax(maxa[c], o->face_area[f]);
            }
        for (int f = 0; f < nB; ++f) {
            int c = o->boundary_cellsID[f];
            P3 xf = sub(fc(f), cc(c));
            vol[c] = vol[c] + (oneThird * dotp(xf, fnm(f))) * o->face_area[f];
            maxa[c] = jmax(maxa[c], o->face_area[f]);
        }
        for (int c = 0; c < nC; ++c) {
            double V = vol[c];
            if (!(std::isfinite(V) && V > 0.0)) {
                double est = std::pow(maxa[c], 1.5) * 1e-3;
                V = jmax(std::isfinite(V) ? std::fabs(V) : 0.0, est);
            }
            o->cell_volume[c] = V;
        }
    }
    return XCAL_OK;
}

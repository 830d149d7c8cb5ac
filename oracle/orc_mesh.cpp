// orc_mesh.cpp -- oracle restatement of FOAM3D_mesh and construct_periodic.
//
// TEST INFRASTRUCTURE ONLY (see orc_common.hpp).
//
// Follows, step by step:
//   src/FoamMesh/FoamMesh_1_read.jl:25-43      assign_faces! (boundary neighbour = owner)
//   src/FoamMesh/FoamMesh_2_connect.jl:24-69   connect_cell_faces
//   src/FoamMesh/FoamMesh_2_connect.jl:71-146  connect_cell_nodes (dedup in first-seen order)
//   src/FoamMesh/FoamMesh_2_connect.jl:148-195 connect_face_nodes (boundary faces first)
//   src/FoamMesh/FoamMesh_3_generate.jl:2-82   generate_mesh / faces / boundaries
//   src/FoamMesh/FoamMesh_4_geometry.jl:2-158  compute_geometry!
//   src/Mesh/Mesh_1_functions.jl:20-51         weight_delta_e
//   src/Discretise/boundary_conditions/periodic.jl:95-217 construct_periodic
// Indices are 0-based here (the Julia code is 1-based).
#include "orc_internal.hpp"

#include <numeric>
#include <stdexcept>

namespace orc {

Mesh* build_foam_mesh(int n_points, const double* points, int n_faces, const int* face_off,
                      const int* face_nodes_in, const int* owner_in, int n_ifaces,
                      const int* neighbour_in, int n_patches, const int* patch_nfaces) {
    Mesh* m = new Mesh();
    m->n_faces = n_faces;
    m->n_ifaces = n_ifaces;
    m->n_bfaces = n_faces - n_ifaces;
    int max_cell = -1;
    for (int f = 0; f < n_faces; ++f) max_cell = std::max(max_cell, owner_in[f]);
    for (int f = 0; f < n_ifaces; ++f) max_cell = std::max(max_cell, neighbour_in[f]);
    m->n_cells = max_cell + 1;
    const int nC = m->n_cells, nB = m->n_bfaces;

    m->points.resize(n_points);
    for (int i = 0; i < n_points; ++i)
        m->points[i] = {points[3 * i], points[3 * i + 1], points[3 * i + 2]};

    // assign_faces!: foam-order owner/neighbour, boundary neighbour = owner
    std::vector<int> f_owner(owner_in, owner_in + n_faces), f_neigh(n_faces);
    for (int fi = 0; fi < n_ifaces; ++fi) f_neigh[fi] = neighbour_in[fi];
    for (int fi = n_ifaces; fi < n_faces; ++fi) f_neigh[fi] = f_owner[fi];

    // connect_cell_faces
    std::vector<int> count(nC, 0);
    for (int fi = 0; fi < n_ifaces; ++fi) {
        count[f_owner[fi]]++;
        count[f_neigh[fi]]++;
    }
    m->cf_off.assign(nC + 1, 0);
    for (int c = 0; c < nC; ++c) m->cf_off[c + 1] = m->cf_off[c] + count[c];
    m->cell_faces.resize(2 * (size_t)n_ifaces);
    m->cell_nsign.resize(2 * (size_t)n_ifaces);
    m->cell_neigh.resize(2 * (size_t)n_ifaces);
    {
        std::vector<int> cursor(m->cf_off.begin(), m->cf_off.end() - 1);
        for (int fi = 0; fi < n_ifaces; ++fi) {
            int o = f_owner[fi], nb = f_neigh[fi], fID = fi + nB;
            int k = cursor[o]++;
            m->cell_faces[k] = fID;
            m->cell_nsign[k] = 1;
            m->cell_neigh[k] = nb;
            k = cursor[nb]++;
            m->cell_faces[k] = fID;
            m->cell_nsign[k] = -1;
            m->cell_neigh[k] = o;
        }
    }

    // connect_cell_nodes: raw lists (owner role then neighbour role per face,
    // global foam face order), then first-seen dedup per cell
    {
        std::vector<int> rcount(nC, 0);
        for (int fi = 0; fi < n_faces; ++fi) {
            int nn = face_off[fi + 1] - face_off[fi];
            rcount[f_owner[fi]] += nn;
            rcount[f_neigh[fi]] += nn;
        }
        std::vector<int64_t> roff(nC + 1, 0);
        for (int c = 0; c < nC; ++c) roff[c + 1] = roff[c] + rcount[c];
        std::vector<int> raw(roff[nC]);
        std::vector<int64_t> rcur(roff.begin(), roff.end() - 1);
        for (int fi = 0; fi < n_faces; ++fi) {
            int o = f_owner[fi];
            for (int k = face_off[fi]; k < face_off[fi + 1]; ++k) raw[rcur[o]++] = face_nodes_in[k];
            int nb = f_neigh[fi];
            for (int k = face_off[fi]; k < face_off[fi + 1]; ++k) raw[rcur[nb]++] = face_nodes_in[k];
        }
        std::vector<int> seen(n_points, -1);
        m->cn_off.assign(nC + 1, 0);
        m->cell_nodes.clear();
        for (int c = 0; c < nC; ++c) {
            for (int64_t k = roff[c]; k < roff[c + 1]; ++k) {
                int nid = raw[k];
                if (seen[nid] != c) {
                    m->cell_nodes.push_back(nid);
                    seen[nid] = c;
                }
            }
            m->cn_off[c + 1] = (int)m->cell_nodes.size();
        }
    }

    // connect_face_nodes: boundary faces first, then internal faces
    m->fn_off.assign(n_faces + 1, 0);
    m->face_nodes.clear();
    {
        int fID = 0;
        auto push = [&](int src) {
            for (int k = face_off[src]; k < face_off[src + 1]; ++k) m->face_nodes.push_back(face_nodes_in[k]);
            m->fn_off[fID + 1] = (int)m->face_nodes.size();
            ++fID;
        };
        for (int src = n_ifaces; src < n_faces; ++src) push(src);
        for (int src = 0; src < n_ifaces; ++src) push(src);
    }

    // generate_faces: mesh fID -> foam source index
    m->owner.resize(n_faces);
    m->neigh.resize(n_faces);
    for (int fID = 0; fID < n_faces; ++fID) {
        int src = fID < nB ? (n_ifaces + fID) : (fID - nB);
        m->owner[fID] = f_owner[src];
        m->neigh[fID] = f_neigh[src];
    }
    // generate_boundaries: consecutive ranges from face 0
    {
        int start = 0;
        for (int p = 0; p < n_patches; ++p) {
            m->patch_start.push_back(start);
            m->patch_count.push_back(patch_nfaces[p]);
            start += patch_nfaces[p];
        }
        if (start != nB) {
            delete m;
            throw std::runtime_error("patch face counts do not cover the boundary faces");
        }
    }
    // generate_boundary_cells
    m->bcell.resize(nB);
    for (int p = 0; p < n_patches; ++p)
        for (int f = m->patch_start[p]; f < m->patch_start[p] + m->patch_count[p]; ++f) m->bcell[f] = m->owner[f];

    // ---- compute_geometry! ----
    m->ccentre.resize(nC);
    m->cvol.resize(nC);
    for (int c = 0; c < nC; ++c) {  // calculate_cell_centres!
        V3 s{0, 0, 0};
        int cnt = m->cn_off[c + 1] - m->cn_off[c];
        for (int k = m->cn_off[c]; k < m->cn_off[c + 1]; ++k) s = s + m->points[m->cell_nodes[k]];
        m->ccentre[c] = s / (double)cnt;
    }
    m->fcentre.resize(n_faces);
    for (int f = 0; f < n_faces; ++f) {  // calculate_face_centres!
        V3 s{0, 0, 0};
        int cnt = m->fn_off[f + 1] - m->fn_off[f];
        for (int k = m->fn_off[f]; k < m->fn_off[f + 1]; ++k) s = s + m->points[m->face_nodes[k]];
        m->fcentre[f] = s / (double)cnt;
    }
    m->fnormal.resize(n_faces);
    m->fe.resize(n_faces);
    m->farea.resize(n_faces);
    m->fdelta.resize(n_faces);
    m->fweight.resize(n_faces);
    // _face_geometry (FoamMesh_4_geometry.jl:48-70)
    auto face_geometry = [&](int f, V3 apex, V3& normal, double& mag, V3& centre) {
        V3 area_vec{0, 0, 0}, centre_sum{0, 0, 0};
        double sum_area = 0.0;
        int b = m->fn_off[f], n = m->fn_off[f + 1] - b;
        for (int i = 0; i < n; ++i) {
            int j = (i == n - 1) ? 0 : i + 1;
            V3 p1 = m->points[m->face_nodes[b + i]];
            V3 p2 = m->points[m->face_nodes[b + j]];
            V3 tri_vec = cross(p1 - apex, p2 - apex) / 2.0;
            double tri_area = norm(tri_vec);
            if (!(tri_area > 0.0)) continue;
            area_vec = area_vec + tri_vec;
            centre_sum = centre_sum + (tri_area * ((apex + p1) + p2)) / 3.0;
            sum_area = sum_area + tri_area;
        }
        mag = norm(area_vec);
        normal = mag > 0.0 ? area_vec / mag : V3{0, 0, 0};
        centre = sum_area > 0.0 ? centre_sum / sum_area : apex;
    };
    for (int f = 0; f < nB; ++f) {  // boundary faces
        V3 normal, centre;
        double area;
        face_geometry(f, m->fcentre[f], normal, area, centre);
        V3 C1 = m->ccentre[m->owner[f]];
        V3 C1F1 = centre - C1;
        if (dot(C1F1, normal) < 0.0) normal = -normal;
        // weight_delta_e(C1F1, normal) (Mesh_1_functions.jl:45-51)
        double weight = 1.0;
        double delta = norm(C1F1);
        V3 e = delta > 0.0 ? C1F1 / delta : normal;
        delta = jl_max(delta, jl_eps(1.0));
        m->fcentre[f] = centre;
        m->fnormal[f] = normal;
        m->farea[f] = area;
        m->fdelta[f] = delta;
        m->fe[f] = e;
        m->fweight[f] = weight;
    }
    for (int f = nB; f < n_faces; ++f) {  // internal faces
        V3 normal, centre;
        double area;
        face_geometry(f, m->fcentre[f], normal, area, centre);
        V3 C1 = m->ccentre[m->owner[f]], C2 = m->ccentre[m->neigh[f]];
        V3 C1F1 = centre - C1, C2F1 = centre - C2, C1C2 = C2 - C1;
        if (dot(C1C2, normal) < 0.0) normal = -normal;
        // weight_delta_e(C1F1, C2F1, C1C2, normal) (Mesh_1_functions.jl:20-42)
        double weight;
        double projection = dot(C1C2, normal);
        if (std::isfinite(projection) && std::fabs(projection) > jl_eps(projection)) {
            double wi = dot(C1F1, normal) / projection;
            weight = 1.0 - wi;
        } else {
            double d1 = norm(C1F1), d2 = norm(C2F1), dsum = d1 + d2;
            weight = dsum > 0.0 ? d2 / dsum : 0.5;
        }
        double delta = norm(C1C2);
        V3 e;
        if (delta > 0.0) {
            e = C1C2 / delta;
        } else {
            delta = norm(C1F1) + norm(C2F1);
            e = normal;
        }
        delta = jl_max(delta, jl_eps(1.0));
        weight = jl_clamp(weight, 0.0, 1.0);
        m->fcentre[f] = centre;
        m->fnormal[f] = normal;
        m->farea[f] = area;
        m->fdelta[f] = delta;
        m->fe[f] = e;
        m->fweight[f] = weight;
    }
    // calculate_cell_volumes!: internal faces per cell, then boundary faces
    {
        const double oneThird = 1.0 / 3.0;
        std::vector<double> vol(nC, 0.0), max_area(nC, 0.0);
        for (int c = 0; c < nC; ++c) {
            for (int k = m->cf_off[c]; k < m->cf_off[c + 1]; ++k) {
                int f = m->cell_faces[k];
                V3 xf = m->fcentre[f] - m->ccentre[c];
                vol[c] = vol[c] + ((oneThird * dot(xf, m->fnormal[f])) * (double)m->cell_nsign[k]) * m->farea[f];
                max_area[c] = jl_max(max_area[c], m->farea[f]);
            }
        }
        for (int p = 0; p < n_patches; ++p) {
            for (int f = m->patch_start[p]; f < m->patch_start[p] + m->patch_count[p]; ++f) {
                int c = m->bcell[f];
                V3 xf = m->fcentre[f] - m->ccentre[c];
                vol[c] = vol[c] + (oneThird * dot(xf, m->fnormal[f])) * m->farea[f];
                max_area[c] = jl_max(max_area[c], m->farea[f]);
            }
        }
        for (int c = 0; c < nC; ++c) {
            double V = vol[c];
            if (!(std::isfinite(V) && V > 0.0)) {
                double estimate = std::pow(max_area[c], 1.5) * 1e-3;
                V = jl_max(std::isfinite(V) ? std::fabs(V) : 0.0, estimate);
            }
            m->cvol[c] = V;
        }
    }
    return m;
}

// Julia's pairwise `sum` over a vector (mapreduce_impl, blocksize 1024) with
// sequential leaves; used by `mean` in construct_periodic.
static V3 pairwise_sum(const std::vector<V3>& a, int64_t lo, int64_t hi) {  // [lo, hi]
    if (lo == hi) return a[lo];
    if (hi - lo < 1024) {
        V3 v = a[lo] + a[lo + 1];
        for (int64_t i = lo + 2; i <= hi; ++i) v = v + a[i];
        return v;
    }
    int64_t mid = lo + ((hi - lo) >> 1);
    V3 v1 = pairwise_sum(a, lo, mid);
    V3 v2 = pairwise_sum(a, mid + 1, hi);
    return v1 + v2;
}

int construct_periodic(const Mesh* m, int patch1, int patch2, double tol, int* map1, int* map2,
                       double* distance) {
    int s1 = m->patch_start[patch1], n1 = m->patch_count[patch1];
    int s2 = m->patch_start[patch2], n2 = m->patch_count[patch2];
    if (n1 != n2) return -1;
    int nf = n1;
    std::vector<V3> c1(nf), c2(nf);
    for (int i = 0; i < nf; ++i) {
        c1[i] = m->fcentre[s1 + i];
        c2[i] = m->fcentre[s2 + i];
    }
    V3 mean1 = pairwise_sum(c1, 0, nf - 1) / (double)nf;
    V3 mean2 = pairwise_sum(c2, 0, nf - 1) / (double)nf;
    V3 tr = mean2 - mean1;
    std::vector<V3> targets(nf);
    for (int i = 0; i < nf; ++i) targets[i] = c1[i] + tr;
    // extent of the targets (minimum/maximum over SVectors is lexicographic
    // in Julia: min_bound/max_bound are the lexicographic extremes)
    V3 mn = targets[0], mx = targets[0];
    auto lexless = [](V3 a, V3 b) {
        if (a.x != b.x) return a.x < b.x;
        if (a.y != b.y) return a.y < b.y;
        return a.z < b.z;
    };
    for (int i = 1; i < nf; ++i) {
        if (lexless(targets[i], mn)) mn = targets[i];
        if (lexless(mx, targets[i])) mx = targets[i];
    }
    V3 ext = mx - mn;
    int axis = 0;
    double best = ext.x;
    if (ext.y > best) { axis = 1; best = ext.y; }
    if (ext.z > best) { axis = 2; best = ext.z; }
    std::vector<int> p1(nf), p2(nf);
    std::iota(p1.begin(), p1.end(), 0);
    std::iota(p2.begin(), p2.end(), 0);
    std::stable_sort(p1.begin(), p1.end(), [&](int a, int b) { return comp(targets[a], axis) < comp(targets[b], axis); });
    std::stable_sort(p2.begin(), p2.end(), [&](int a, int b) { return comp(c2[a], axis) < comp(c2[b], axis); });
    int search_start = 0;
    for (int i = 0; i < nf; ++i) {
        V3 t = targets[p1[i]];
        double tv = comp(t, axis);
        while (search_start < nf && comp(c2[p2[search_start]], axis) < tv - tol) ++search_start;
        double best_dist = std::numeric_limits<double>::infinity();
        int best_j = -1;
        for (int j = search_start; j < nf; ++j) {
            V3 s = c2[p2[j]];
            double axis_dist = comp(s, axis) - tv;
            if (axis_dist > tol) break;
            double d = norm(t - s);
            if (d < best_dist) {
                best_dist = d;
                best_j = j;
            }
        }
        if (best_j < 0 || !(best_dist < tol)) return -2;
        int l1 = p1[i], l2 = p2[best_j];
        map1[l1] = s2 + l2;
        map2[l2] = s1 + l1;
    }
    distance[0] = tr.x;
    distance[1] = tr.y;
    distance[2] = tr.z;
    return 0;
}

}  // namespace orc

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

#include <math_constants.h>

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

namespace {
int device_geometry(const xcal_polymesh_desc* pm, const xcal_mesh_buffers* o, int nC, int nB,
                    const std::vector<long>& roff, const std::vector<int>& raw, const std::vector<int>& off);
}  // namespace

// the Mesh3 of a polyMesh: topology on the host, then the geometry on the
// host or (device) on the current GPU with the same arithmetic
static int32_t foam_build(const xcal_polymesh_desc* pm, const xcal_mesh_buffers* o, bool device) {
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
        if (device) return device_geometry(pm, o, nC, nB, roff, raw, off);
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

extern "C" int32_t xcal_foam_mesh_build(const xcal_polymesh_desc* pm, const xcal_mesh_buffers* o) {
    return foam_build(pm, o, false);
}

// ---------------------------------------------------------------------------
// device geometry: the host loops above as kernels (one thread per cell or
// face, the same operations in the same order; device code is compiled
// without contraction)
// ---------------------------------------------------------------------------
namespace {

struct D3 {
    double x, y, z;
};
__device__ __forceinline__ D3 dadd(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 dsub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 dscl(double s, D3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ D3 ddvd(D3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ double ddot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double dnrm(D3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ D3 dcrs(D3 a, D3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double deps(double v) {
    v = fabs(v);
    return nextafter(v, CUDART_INF) - v;
}
__device__ __forceinline__ double djmax(double x, double y) {
    bool ty = (y > x) || (signbit(y) < signbit(x));
    return ty ? (isnan(x) ? x : y) : (isnan(y) ? y : x);
}
__device__ __forceinline__ D3 dpt(const double* p, int i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }

// cell centres: the mean of the cell's nodes in first-seen order of its raw
// node list (faces in foam order, owner role then neighbour role)
__global__ void k_geo_centres(int nC, const long* __restrict__ roff, const int* __restrict__ raw,
                              const double* __restrict__ pts, double* cc) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    D3 s{0, 0, 0};
    int m = 0;
    for (long k = roff[c]; k < roff[c + 1]; ++k) {
        const int nid = raw[k];
        bool seen = false;
        for (long q = roff[c]; q < k; ++q)
            if (raw[q] == nid) {
                seen = true;
                break;
            }
        if (seen) continue;
        s = dadd(s, dpt(pts, nid));
        ++m;
    }
    const D3 r = ddvd(s, (double)m);
    cc[3 * c] = r.x;
    cc[3 * c + 1] = r.y;
    cc[3 * c + 2] = r.z;
}

// per face: node-average apex, fan triangles, orientation, weight/delta/e
__global__ void k_geo_faces(int nF, int nB, int nI, const int* __restrict__ fo, const int* __restrict__ fn,
                            const double* __restrict__ pts, const int* __restrict__ owner,
                            const int* __restrict__ neigh, const double* __restrict__ cc, double* fcen, double* fnor,
                            double* fe, double* farea, double* fdelta, double* fweight) {
    int fid = blockIdx.x * blockDim.x + threadIdx.x;
    if (fid >= nF) return;
    const int s = fid < nB ? nI + fid : fid - nB;
    const int b = fo[s], n = fo[s + 1] - b;
    D3 sum{0, 0, 0};
    for (int k = 0; k < n; ++k) sum = dadd(sum, dpt(pts, fn[b + k]));
    const D3 apex = ddvd(sum, (double)n);
    D3 area_vec{0, 0, 0}, centre_sum{0, 0, 0};
    double sum_area = 0.0;
    for (int i = 0; i < n; ++i) {
        const int j = (i == n - 1) ? 0 : i + 1;
        const D3 p1 = dpt(pts, fn[b + i]), p2 = dpt(pts, fn[b + j]);
        const D3 tri = ddvd(dcrs(dsub(p1, apex), dsub(p2, apex)), 2.0);
        const double ta = dnrm(tri);
        if (!(ta > 0.0)) continue;
        area_vec = dadd(area_vec, tri);
        centre_sum = dadd(centre_sum, ddvd(dscl(ta, dadd(dadd(apex, p1), p2)), 3.0));
        sum_area = sum_area + ta;
    }
    const double mag = dnrm(area_vec);
    D3 normal = mag > 0.0 ? ddvd(area_vec, mag) : D3{0, 0, 0};
    const D3 centre = sum_area > 0.0 ? ddvd(centre_sum, sum_area) : apex;
    const D3 C1 = dpt(cc, owner[fid]);
    double weight, delta;
    D3 e;
    if (fid < nB) {
        const D3 C1F1 = dsub(centre, C1);
        if (ddot(C1F1, normal) < 0.0) normal = dscl(-1.0, normal);
        weight = 1.0;
        delta = dnrm(C1F1);
        e = delta > 0.0 ? ddvd(C1F1, delta) : normal;
        delta = djmax(delta, deps(1.0));
    } else {
        const D3 C2 = dpt(cc, neigh[fid]);
        const D3 C1F1 = dsub(centre, C1), C2F1 = dsub(centre, C2), C1C2 = dsub(C2, C1);
        if (ddot(C1C2, normal) < 0.0) normal = dscl(-1.0, normal);
        const double proj = ddot(C1C2, normal);
        if (isfinite(proj) && fabs(proj) > deps(proj)) {
            const double wi = ddot(C1F1, normal) / proj;
            weight = 1.0 - wi;
        } else {
            const double d1 = dnrm(C1F1), d2 = dnrm(C2F1), ds = d1 + d2;
            weight = ds > 0.0 ? d2 / ds : 0.5;
        }
        delta = dnrm(C1C2);
        if (delta > 0.0) {
            e = ddvd(C1C2, delta);
        } else {
            delta = dnrm(C1F1) + dnrm(C2F1);
            e = normal;
        }
        delta = djmax(delta, deps(1.0));
        weight = weight > 1.0 ? 1.0 : (weight < 0.0 ? 0.0 : weight);
    }
    fcen[3 * fid] = centre.x;
    fcen[3 * fid + 1] = centre.y;
    fcen[3 * fid + 2] = centre.z;
    fnor[3 * fid] = normal.x;
    fnor[3 * fid + 1] = normal.y;
    fnor[3 * fid + 2] = normal.z;
    fe[3 * fid] = e.x;
    fe[3 * fid + 1] = e.y;
    fe[3 * fid + 2] = e.z;
    farea[fid] = mag;
    fdelta[fid] = delta;
    fweight[fid] = weight;
}

// volumes: internal faces in cell_faces order, then boundary faces ascending
__global__ void k_geo_volumes(int nC, const int* __restrict__ off, const int* __restrict__ cf,
                              const int* __restrict__ nsign, const int* __restrict__ bf_off,
                              const int* __restrict__ bf_face, const double* __restrict__ fcen,
                              const double* __restrict__ fnor, const double* __restrict__ farea,
                              const double* __restrict__ cc, double* vol_out) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    const double oneThird = 1.0 / 3.0;
    const D3 C = dpt(cc, c);
    double vol = 0.0, maxa = 0.0;
    for (int k = off[c]; k < off[c + 1]; ++k) {
        const int f = cf[k];
        const D3 xf = dsub(dpt(fcen, f), C);
        vol = vol + ((oneThird * ddot(xf, dpt(fnor, f))) * (double)nsign[k]) * farea[f];
        maxa = djmax(maxa, farea[f]);
    }
    for (int k = bf_off[c]; k < bf_off[c + 1]; ++k) {
        const int f = bf_face[k];
        const D3 xf = dsub(dpt(fcen, f), C);
        vol = vol + (oneThird * ddot(xf, dpt(fnor, f))) * farea[f];
        maxa = djmax(maxa, farea[f]);
    }
    double V = vol;
    if (!(isfinite(V) && V > 0.0)) {  // degenerate cell (pow's last bit may differ from the host's)
        const double est = pow(maxa, 1.5) * 1e-3;
        V = djmax(isfinite(V) ? fabs(V) : 0.0, est);
    }
    vol_out[c] = V;
}

template <class T>
struct DArr {
    T* p = nullptr;
    ~DArr() {
        if (p) cudaFree(p);
    }
    cudaError_t put(const T* h, size_t n) {
        cudaError_t e = cudaMalloc(&p, (n ? n : 1) * sizeof(T));
        if (e != cudaSuccess || !n) return e;
        return cudaMemcpy(p, h, n * sizeof(T), cudaMemcpyHostToDevice);
    }
    cudaError_t get(T* h, size_t n) const { return n ? cudaMemcpy(h, p, n * sizeof(T), cudaMemcpyDeviceToHost) : cudaSuccess; }
};

int device_geometry(const xcal_polymesh_desc* pm, const xcal_mesh_buffers* o, int nC, int nB,
                    const std::vector<long>& roff, const std::vector<int>& raw, const std::vector<int>& off) {
    const int nF = pm->n_faces, nI = pm->n_internal_faces, nP = pm->n_points;
    const int* fo = pm->face_offsets;
    // cell -> boundary faces, ascending
    std::vector<int> bf_off(nC + 1, 0), bf_face(nB);
    for (int f = 0; f < nB; ++f) bf_off[o->boundary_cellsID[f] + 1]++;
    for (int c = 0; c < nC; ++c) bf_off[c + 1] += bf_off[c];
    {
        std::vector<int> cur(bf_off.begin(), bf_off.end() - 1);
        for (int f = 0; f < nB; ++f) bf_face[cur[o->boundary_cellsID[f]]++] = f;
    }
    const long nk = off[nC];
    DArr<double> d_pts, d_cc, d_fc, d_fn, d_fe, d_fa, d_fd, d_fw, d_vol;
    DArr<long> d_roff;
    DArr<int> d_raw, d_fo, d_fnodes, d_own, d_nei, d_off, d_cf, d_ns, d_bfo, d_bff;
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
        return e == cudaSuccess;
    };
    ok(d_pts.put(pm->points, 3 * (size_t)nP));
    ok(d_roff.put(roff.data(), roff.size()));
    ok(d_raw.put(raw.data(), raw.size()));
    ok(d_fo.put(fo, nF + 1));
    ok(d_fnodes.put(pm->face_nodes, fo[nF]));
    ok(d_own.put(o->face_owner, nF));
    ok(d_nei.put(o->face_neigh, nF));
    ok(d_off.put(off.data(), off.size()));
    ok(d_cf.put(o->cell_faces, nk));
    ok(d_ns.put(o->cell_nsign, nk));
    ok(d_bfo.put(bf_off.data(), bf_off.size()));
    ok(d_bff.put(bf_face.data(), bf_face.size()));
    for (DArr<double>* a : {&d_cc, &d_vol}) ok(cudaMalloc(&a->p, (size_t)nC * 3 * sizeof(double)));
    for (DArr<double>* a : {&d_fc, &d_fn, &d_fe}) ok(cudaMalloc(&a->p, (size_t)nF * 3 * sizeof(double)));
    for (DArr<double>* a : {&d_fa, &d_fd, &d_fw}) ok(cudaMalloc(&a->p, (size_t)nF * sizeof(double)));
    if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? XCAL_ERR_OOM : XCAL_ERR_CUDA;
    const int T = 256;
    k_geo_centres<<<(nC + T - 1) / T, T>>>(nC, d_roff.p, d_raw.p, d_pts.p, d_cc.p);
    k_geo_faces<<<(nF + T - 1) / T, T>>>(nF, nB, nI, d_fo.p, d_fnodes.p, d_pts.p, d_own.p, d_nei.p, d_cc.p, d_fc.p,
                                         d_fn.p, d_fe.p, d_fa.p, d_fd.p, d_fw.p);
    k_geo_volumes<<<(nC + T - 1) / T, T>>>(nC, d_off.p, d_cf.p, d_ns.p, d_bfo.p, d_bff.p, d_fc.p, d_fn.p, d_fa.p,
                                           d_cc.p, d_vol.p);
    ok(cudaGetLastError());
    ok(cudaDeviceSynchronize());
    ok(d_cc.get(o->cell_centre, 3 * (size_t)nC));
    ok(d_fc.get(o->face_centre, 3 * (size_t)nF));
    ok(d_fn.get(o->face_normal, 3 * (size_t)nF));
    ok(d_fe.get(o->face_e, 3 * (size_t)nF));
    ok(d_fa.get(o->face_area, nF));
    ok(d_fd.get(o->face_delta, nF));
    ok(d_fw.get(o->face_weight, nF));
    ok(d_vol.get(o->cell_volume, nC));
    return e == cudaSuccess ? XCAL_OK : XCAL_ERR_CUDA;
}

}  // namespace

extern "C" int32_t xcal_foam_mesh_build_device(int32_t device, const xcal_polymesh_desc* pm,
                                               const xcal_mesh_buffers* o) {
    if (cudaSetDevice(device) != cudaSuccess) return XCAL_ERR_CUDA;
    return foam_build(pm, o, true);
}

// kernels_fv.cu -- finite-volume kernels of the SIMPLE/PISO path (FP64).
//
// Each kernel restates one reference kernel; the operation order inside every
// expression is the Julia source's (cited per kernel).  Gathers replace the
// reference's Atomix scatters: boundary contributions to a cell are applied by
// the thread owning the cell, in ascending boundary-face order.
#include "dev_common.cuh"
#include <algorithm>

#include "kernels.hpp"

namespace xcal {

constexpr int TPB = 256;
static inline int nblk(long n) { return (int)((n + TPB - 1) / TPB); }

// ---------------------------------------------------------------------------
// boundary-condition functors (src/Discretise/boundary_conditions/*.jl)
// ---------------------------------------------------------------------------
// value of a Dirichlet-like BC at boundary face f, component c
__device__ __forceinline__ double bc_val(const BCView& bc, int f, int c) { return bc.val[3 * f + c]; }

// Periodic parent face f (periodic.jl:261-443), one term at a time: the term
// adds ac to the own diagonal and an to the (own, partner) slot, and -an to
// the partner diagonal and -ac to the (partner, own) slot.
// Divergence (sign +1, flux mdot_f):
__device__ __forceinline__ void periodic_div(const BCView& bc, int f, double mdotf, int div_scheme, double& ac,
                                             double& an) {
    if (div_scheme == XCAL_DIV_UPWIND) {
        double md = 1.0 * mdotf;
        ac = jl_max(md, 0.0);
        an = -jl_max(-md, 0.0);
        return;
    }
    double w = bc.pw[f], wn = bc.pwn[f];
    if (div_scheme == XCAL_DIV_LINEAR) {
        double a = 1.0 * mdotf;
        ac = a * w;
        an = a * wn;
    } else {  // LUST
        double md = 1.0 * mdotf;
        double acL = md * w, anL = md * wn;
        double acU = jl_max(md, 0.0), anU = -jl_max(-md, 0.0);
        ac = 0.75 * acL + 0.25 * acU;
        an = 0.75 * anL + 0.25 * anU;
    }
}
// Laplacian (sign -1, flux Gamma_f): gamma = (1 * (Gamma |E_f|)) / Delta;
// ac = gamma, an = -gamma
__device__ __forceinline__ void periodic_lap(const BCView& bc, int f, double flux, double& ac, double& an) {
    double gamma = (1.0 * (flux * bc.pEf[f])) / bc.pDelta[f];
    ac = gamma;
    an = -gamma;
}

// U equation: terms Time + Divergence(mdotf,U) - Laplacian(nueff,U); returns
// (AP, BP) summed over the terms in order (apply!, Discretise_5_apply_bcs.jl:158-183)
__device__ void bc_U(const MeshView& m, const BCView& bc, int f, int cell, int comp, int div_scheme,
                     const double* mdot, const double* nueff, const double* Ux, const double* Uy,
                     const double* Uz, double& AP, double& BP) {
    int type = bc.type[f];
    double ap_d = 0.0, bp_d = 0.0, ap_l = 0.0, bp_l = 0.0;
    switch (type) {
        case XCAL_BC_DIRICHLET:
        case XCAL_BC_DIRICHLET_FUNCTION: {  // dirichlet.jl:46-75
            double val = bc_val(bc, f, comp);
            double fl = -mdot[f];
            double a = 1.0 * fl;
            ap_d = 0.0;
            bp_d = a * val;
            double fll = (nueff[f] * m.area[f]) / m.delta[f];
            double al = -1.0 * (-fll);
            ap_l = al;
            bp_l = al * val;
            break;
        }
        case XCAL_BC_WALL: {  // wall.jl:26-42
            double fll = (nueff[f] * m.area[f]) / m.delta[f];
            double al = -1.0 * (-fll);
            double nx = m.nx[f], ny = m.ny[f], nz = m.nz[f];
            double vbx = bc_val(bc, f, 0), vby = bc_val(bc, f, 1), vbz = bc_val(bc, f, 2);
            double vcx = Ux[cell], vcy = Uy[cell], vcz = Uz[cell];
            double dc = vcx * nx + vcy * ny + vcz * nz;
            double db = vbx * nx + vby * ny + vbz * nz;
            double vcn = comp == 0 ? dc * nx : (comp == 1 ? dc * ny : dc * nz);
            double vbn = comp == 0 ? db * nx : (comp == 1 ? db * ny : db * nz);
            double vb = comp == 0 ? vbx : (comp == 1 ? vby : vbz);
            double vbp = vb - vbn;
            ap_l = al;
            bp_l = al * (vbp + vcn);
            break;
        }
        case XCAL_BC_ZEROGRADIENT:  // zerogradient.jl:40-46
            ap_d = 1.0 * mdot[f];
            break;
        case XCAL_BC_EXTRAPOLATED: {  // extrapolated.jl:21-41
            ap_d = 1.0 * mdot[f];
            double fll = ((-nueff[f]) * m.area[f]) / m.delta[f];
            double al = -1.0 * fll;
            const double* U = comp == 0 ? Ux : (comp == 1 ? Uy : Uz);
            ap_l = al;
            bp_l = al * U[cell];
            break;
        }
        case XCAL_BC_SYMMETRY: {  // symmetry.jl:23-41, 103-117
            double nx = m.nx[f], ny = m.ny[f], nz = m.nz[f];
            double vcx = Ux[cell], vcy = Uy[cell], vcz = Uz[cell];
            double dc = vcx * nx + vcy * ny + vcz * nz;
            double vn = comp == 0 ? dc * nx : (comp == 1 ? dc * ny : dc * nz);
            double vc = comp == 0 ? vcx : (comp == 1 ? vcy : vcz);
            double a = 1.0 * mdot[f];
            ap_d = a;
            bp_d = a * vn;
            double fll = (nueff[f] * m.area[f]) / m.delta[f];
            double al = -1.0 * (-fll);
            ap_l = al;
            bp_l = al * (vc - vn);
            break;
        }
        case XCAL_BC_PERIODIC_PARENT: {  // own-row share; slots in k_bc_relax_U
            double an;
            periodic_div(bc, f, mdot[f], div_scheme, ap_d, an);
            periodic_lap(bc, f, nueff[f], ap_l, an);
            break;
        }
        default:  // Empty, Periodic (shadow), none
            break;
    }
    double ap = 0.0, bp = 0.0;
    ap = ap + 0.0;  // Time term (Discretise_3_boundary_conditions.jl:2-9)
    bp = bp + 0.0;
    ap = ap + ap_d;
    bp = bp + bp_d;
    ap = ap + ap_l;
    bp = bp + bp_l;
    AP = ap;
    BP = bp;
}

// p equation: single term -Laplacian(rDf, p)
__device__ void bc_p(const MeshView& m, const BCView& bc, int f, int cell, const double* rDf, const double* p,
                     double& AP, double& BP) {
    int type = bc.type[f];
    double a = 0.0, b = 0.0;
    switch (type) {
        case XCAL_BC_DIRICHLET:
        case XCAL_BC_DIRICHLET_FUNCTION: {  // dirichlet.jl:19-25
            double fl = (rDf[f] * m.area[f]) / m.delta[f];
            a = -1.0 * (-fl);
            b = a * bc_val(bc, f, 0);
            break;
        }
        case XCAL_BC_EXTRAPOLATED: {  // extrapolated.jl:21-33
            double fl = ((-rDf[f]) * m.area[f]) / m.delta[f];
            a = -1.0 * fl;
            b = a * p[cell];
            break;
        }
        case XCAL_BC_NEUMANN: {  // neumann.jl:23-30
            double fl = rDf[f] * m.area[f];
            a = 0.0;
            b = fl * bc_val(bc, f, 0);
            break;
        }
        case XCAL_BC_PERIODIC_PARENT: {  // own-row share; slots in k_bc_p
            double an;
            periodic_lap(bc, f, rDf[f], a, an);
            break;
        }
        default:  // Wall, Zerogradient, Empty, Symmetry, Periodic shadow: (0, 0)
            break;
    }
    AP = 0.0 + a;
    BP = 0.0 + b;
}

// ---------------------------------------------------------------------------
// assembly: _discretise_vector_model! / _discretise_scalar_model!
// (Discretise_2_generated_distretisation.jl:39-87, 125-167)
// ---------------------------------------------------------------------------
__global__ void k_assemble_U(MeshView m, CSRView A, const double* __restrict__ mdot,
                             const double* __restrict__ nueff, const double* __restrict__ Ux,
                             const double* __restrict__ Uy, const double* __restrict__ Uz,
                             const double* __restrict__ gx, const double* __restrict__ gy,
                             const double* __restrict__ gz, double* nz, double* diag0, double* bx, double* by,
                             double* bz, int time_scheme, int div_scheme, double dt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nC) return;
    double ac_sum = 0.0;
    for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
        int f = m.cf_face[k];
        int ns = m.cf_sign[k];
        double dns = (double)ns;
        double AC = 0.0, AN = 0.0;
        AC = AC + 0.0;  // Time{...} scheme! (Discretise_1_schemes.jl:12-34)
        AN = AN + 0.0;
        // Divergence (Discretise_1_schemes.jl:114-180)
        double ap = 1.0 * (mdot[f] * dns);
        double ac, an;
        if (div_scheme == XCAL_DIV_LINEAR) {
            double w = m.weight[f];
            w = 0.5 + dns * (w - 0.5);
            ac = ap * w;
            an = ap * (1.0 - w);
        } else if (div_scheme == XCAL_DIV_UPWIND) {
            ac = jl_max(ap, 0.0);
            an = -jl_max(-ap, 0.0);
        } else {
            double w = m.weight[f];
            if (ns < 0) w = 1.0 - w;
            double acL = ap * w, anL = ap * (1.0 - w);
            double acU = jl_max(ap, 0.0), anU = -jl_max(-ap, 0.0);
            ac = 0.75 * acL + 0.25 * acU;
            an = 0.75 * anL + 0.25 * anU;
        }
        AC = AC + ac;
        AN = AN + an;
        // Laplacian{Linear}, sign -1 (Discretise_1_schemes.jl:68-110)
        double apl = (-1.0 * (nueff[f] * m.Efmag[f])) / m.delta[f];
        AC = AC + (-apl);
        AN = AN + apl;
        ac_sum = ac_sum + AC;
        nz[A.cf_slot[k]] = AN;
    }
    double V = m.vol[i];
    double acs = 0.0, bxs = 0.0, bys = 0.0, bzs = 0.0;  // _scheme_source!
    if (time_scheme == XCAL_TIME_EULER) {
        double vol_rdt = (1.0 * V) / dt;  // Discretise_1_schemes.jl:36-45
        acs = acs + vol_rdt;
        bxs = bxs + Ux[i] * vol_rdt;
        bys = bys + Uy[i] * vol_rdt;
        bzs = bzs + Uz[i] * vol_rdt;
    } else {
        acs = acs + 0.0;
        bxs = bxs + 0.0;
        bys = bys + 0.0;
        bzs = bzs + 0.0;
    }
    acs = acs + 0.0;  // Divergence, Laplacian scheme_source!
    bxs = bxs + 0.0;
    bys = bys + 0.0;
    bzs = bzs + 0.0;
    acs = acs + 0.0;
    bxs = bxs + 0.0;
    bys = bys + 0.0;
    bzs = bzs + 0.0;
    double d = ac_sum + acs;
    nz[A.diag[i]] = d;
    diag0[i] = d;
    // _sources!: -Source(grad p)
    double Bx = 0.0 + (-1.0 * gx[i]) * V;
    double By = 0.0 + (-1.0 * gy[i]) * V;
    double Bz = 0.0 + (-1.0 * gz[i]) * V;
    bx[i] = bxs + Bx;
    by[i] = bys + By;
    bz[i] = bzs + Bz;
}

__global__ void k_assemble_p(MeshView m, CSRView A, const double* __restrict__ rDf,
                             const double* __restrict__ divHv, double* nz, double* b) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nC) return;
    double ac_sum = 0.0;
    for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
        int f = m.cf_face[k];
        double ap = (-1.0 * (rDf[f] * m.Efmag[f])) / m.delta[f];
        double AC = 0.0 + (-ap);
        double AN = 0.0 + ap;
        ac_sum = ac_sum + AC;
        nz[A.cf_slot[k]] = AN;
    }
    double acs = 0.0 + 0.0, bs = 0.0 + 0.0;
    nz[A.diag[i]] = ac_sum + acs;
    double b2 = 0.0 + (-1.0 * divHv[i]) * m.vol[i];
    b[i] = b2 + bs;
}

// ---------------------------------------------------------------------------
// boundary conditions + implicit relaxation (U), per row
// apply_boundary_conditions! (Discretise_5_apply_bcs.jl:84-123) then
// implicit_relaxation_diagdom! (Solve_1_api.jl:388-411)
// ---------------------------------------------------------------------------
__global__ void k_bc_relax_U(MeshView m, CSRView A, BCView bc, int comp, int div_scheme, double* nz,
                             const double* __restrict__ diag0, double* b, const double* __restrict__ mdot,
                             const double* __restrict__ nueff, const double* __restrict__ Ux,
                             const double* __restrict__ Uy, const double* __restrict__ Uz, double alpha,
                             int flags) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nC) return;
    int ds = A.diag[i];
    double d = (flags & BCR_DIAG0) ? diag0[i] : nz[ds];
    double bi = b[i];
    if (flags & BCR_BC) {
        // own boundary faces and the periodic parent faces this cell partners,
        // merged in ascending face order (the reference's face loop order)
        int k = m.bf_off[i], ke = m.bf_off[i + 1];
        int q = bc.pe_off ? bc.pe_off[i] : 0, qe = bc.pe_off ? bc.pe_off[i + 1] : 0;
        while (k < ke || q < qe) {
            int fo = k < ke ? m.bf_face[k] : 0x7fffffff;
            int fp = q < qe ? bc.pe_face[q] : 0x7fffffff;
            if (fo < fp) {
                double AP, BP;
                bc_U(m, bc, fo, i, comp, div_scheme, mdot, nueff, Ux, Uy, Uz, AP, BP);
                d = d + AP;
                bi = bi + BP;
                if (bc.type[fo] == XCAL_BC_PERIODIC_PARENT) {  // (own, partner) slot from A0 = 0
                    double acd, and_, acl, anl;
                    periodic_div(bc, fo, mdot[fo], div_scheme, acd, and_);
                    periodic_lap(bc, fo, nueff[fo], acl, anl);
                    double v = 0.0;
                    v = v + and_;
                    v = v + anl;
                    nz[bc.pPN[fo]] = v;
                }
                ++k;
            } else {  // this cell is the partner of parent face fp
                double acd, and_, acl, anl;
                periodic_div(bc, fp, mdot[fp], div_scheme, acd, and_);
                periodic_lap(bc, fp, nueff[fp], acl, anl);
                d = d + (-and_);
                d = d + (-anl);
                double v = 0.0;
                v = v + (-acd);
                v = v + (-acl);
                nz[bc.pNP[fp]] = v;
                ++q;
            }
        }
    }
    if (!(flags & BCR_RELAX)) {
        nz[ds] = d;
        b[i] = bi;
        return;
    }
    double sumv = 0.0;
    const int rb = row_base(A, i), rl = A.len[i];
    for (int k = 0; k < rl; ++k) {
        int e = rb + SELL_C * k;
        sumv = sumv + fabs(e == ds ? d : nz[e]);
    }
    sumv = sumv - fabs(d);
    double D0 = d;
    double Dmax = jl_max(fabs(D0), sumv) / alpha;
    nz[ds] = Dmax;
    const double* U = comp == 0 ? Ux : (comp == 1 ? Uy : Uz);
    b[i] = bi + (Dmax - D0) * U[i];
}

// ---------------------------------------------------------------------------
// RANS{KOmega} (RANS_kOmega.jl): the k and omega equations
//   Time + Divergence(mdot, phi) - Laplacian(mueff, phi) + Si(D, phi) == Source(P)
// with mueff = nu + sigma nutf (rho = 1), on the p system's storage
// ---------------------------------------------------------------------------
// production / dissipation (RANS_kOmega.jl:170-178): magnitude2!(S, 2)
// (RANS_tensor_algebra.jl:81-99, S = 0.5 (G + G'), rows outer) into
// Pw = alpha1 |S|^2, Pk = nut |S|^2; Dw = beta1 omega, Dk = beta+ omega
__global__ void k_kw_sources(int nC, const double* __restrict__ g0, const double* __restrict__ g1,
                             const double* __restrict__ g2, const double* __restrict__ g3,
                             const double* __restrict__ g4, const double* __restrict__ g5,
                             const double* __restrict__ g6, const double* __restrict__ g7,
                             const double* __restrict__ g8, const double* __restrict__ nut,
                             const double* __restrict__ omega, double* Pk, double* Pw, double* Dk, double* Dw,
                             double alpha1, double beta1, double beta_star) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nC) return;
    const double G[9] = {g0[i], g1[i], g2[i], g3[i], g4[i], g5[i], g6[i], g7[i], g8[i]};
    double sum = 0.0;
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const double s = 0.5 * (G[3 * j + q] + G[3 * q + j]);
            sum = sum + s * s;
        }
    const double mag = sum * 2.0;
    Pw[i] = alpha1 * mag;
    Pk[i] = nut[i] * mag;
    const double w = omega[i];
    Dw[i] = beta1 * w;
    Dk[i] = beta_star * w;
}

// _discretise_scalar_model! (Discretise_2_generated_distretisation.jl:125-167)
// of the k / omega equation: terms Time, Divergence, Laplacian, Si in order
// face diffusivity nu + sigma nutf; with F1 (k-omega SST) sigma blends as
// s1 F1f + (1 - F1f) s2, F1f the plain interpolation of F1.  k-omega LKE
// passes its interpolated face diffusivity as nutf with nu = 0, sigma = 1
// (0 + 1 x = x)
__device__ __forceinline__ double kw_mueff(const MeshView& m, int f, const double* nutf, double nu, double s1,
                                           const double* F1, double s2) {
    if (!F1) return nu + s1 * nutf[f];
    const double w = m.weight[f];
    const double F1f = w * F1[m.owner[f]] + (1.0 - w) * F1[m.neigh[f]];
    const double sg = s1 * F1f + (1.0 - F1f) * s2;
    return nu + sg * nutf[f];
}

__global__ void k_assemble_scalar(MeshView m, CSRView A, const double* __restrict__ mdot,
                                  const double* __restrict__ nutf, double nu, double sigma,
                                  const double* __restrict__ F1, double sigma2, const double* __restrict__ phi,
                                  const double* __restrict__ D, const double* __restrict__ D2,
                                  const double* __restrict__ P, double* nz, double* b, int time_scheme,
                                  int div_scheme, double dt, double d2_sign) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nC) return;
    double ac_sum = 0.0;
    for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
        int f = m.cf_face[k];
        int ns = m.cf_sign[k];
        double dns = (double)ns;
        double AC = 0.0, AN = 0.0;
        AC = AC + 0.0;  // Time
        AN = AN + 0.0;
        double ap = 1.0 * (mdot[f] * dns);  // Divergence (Discretise_1_schemes.jl:114-180)
        double ac, an;
        if (div_scheme == XCAL_DIV_LINEAR) {
            double w = m.weight[f];
            w = 0.5 + dns * (w - 0.5);
            ac = ap * w;
            an = ap * (1.0 - w);
        } else if (div_scheme == XCAL_DIV_UPWIND) {
            ac = jl_max(ap, 0.0);
            an = -jl_max(-ap, 0.0);
        } else {
            double w = m.weight[f];
            if (ns < 0) w = 1.0 - w;
            double acL = ap * w, anL = ap * (1.0 - w);
            double acU = jl_max(ap, 0.0), anU = -jl_max(-ap, 0.0);
            ac = 0.75 * acL + 0.25 * acU;
            an = 0.75 * anL + 0.25 * anU;
        }
        AC = AC + ac;
        AN = AN + an;
        const double muf = kw_mueff(m, f, nutf, nu, sigma, F1, sigma2);
        double apl = (-1.0 * (muf * m.Efmag[f])) / m.delta[f];  // Laplacian, sign -1
        AC = AC + (-apl);
        AN = AN + apl;
        AC = AC + 0.0;  // Si (:204-210)
        AN = AN + 0.0;
        if (D2) {  // a second Si (omega of k-omega SST)
            AC = AC + 0.0;
            AN = AN + 0.0;
        }
        ac_sum = ac_sum + AC;
        nz[A.cf_slot[k]] = AN;
    }
    const double V = m.vol[i];
    double acs = 0.0, bs = 0.0;
    if (time_scheme == XCAL_TIME_EULER) {
        double vol_rdt = (1.0 * V) / dt;  // Discretise_1_schemes.jl:36-45
        acs = acs + vol_rdt;
        bs = bs + phi[i] * vol_rdt;
    } else {
        acs = acs + 0.0;
        bs = bs + 0.0;
    }
    acs = acs + 0.0;  // Divergence, Laplacian
    bs = bs + 0.0;
    acs = acs + 0.0;
    bs = bs + 0.0;
    acs = acs + (1.0 * D[i]) * V;  // Si (:211-218)
    bs = bs + 0.0;
    if (D2) {
        acs = acs + (d2_sign * D2[i]) * V;
        bs = bs + 0.0;
    }
    nz[A.diag[i]] = ac_sum + acs;
    const double b2 = 0.0 + (1.0 * P[i]) * V;  // +Source(P)
    b[i] = b2 + bs;
}

// one boundary face of the k / omega equation (Time, Divergence, Laplacian,
// Si; Discretise_3_boundary_conditions.jl, boundary_conditions/*.jl):
// OmegaWallFunction contributes as Extrapolated (its wall rows are then
// constrained)
__device__ void bc_scalar_transport(const MeshView& m, const BCView& bc, int f, int cell, const double* mdot,
                                    double muf, const double* phi, bool si2, int div_scheme, double& AP,
                                    double& BP) {
    double ap_d = 0.0, bp_d = 0.0, ap_l = 0.0, bp_l = 0.0;
    switch (bc.type[f]) {
        case XCAL_BC_DIRICHLET:
        case XCAL_BC_DIRICHLET_FUNCTION: {  // dirichlet.jl:19-31
            const double val = bc_val(bc, f, 0);
            bp_d = (1.0 * (-mdot[f])) * val;
            double fl = (muf * m.area[f]) / m.delta[f];
            double al = -1.0 * (-fl);
            ap_l = al;
            bp_l = al * val;
            break;
        }
        case XCAL_BC_WALL:  // wall.jl:43-102 (scalar)
        case XCAL_BC_ZEROGRADIENT:
        case XCAL_BC_SYMMETRY:
        case XCAL_BC_K_WALL:  // Discretise_3_boundary_conditions.jl:12-51 (Laplacian (0, 0))
        case XCAL_BC_NUT_WALL:
            ap_d = 1.0 * mdot[f];
            break;
        case XCAL_BC_EXTRAPOLATED:  // extrapolated.jl:21-45
        case XCAL_BC_OMEGA_WALL: {
            ap_d = 1.0 * mdot[f];
            double fl = ((-muf) * m.area[f]) / m.delta[f];
            double al = -1.0 * fl;
            ap_l = al;
            bp_l = al * phi[cell];
            break;
        }
        case XCAL_BC_NEUMANN: {  // neumann.jl (scalar)
            const double val = bc_val(bc, f, 0);
            double a = 1.0 * mdot[f];
            ap_d = a;
            bp_d = ((-val) * a) * m.delta[f];
            bp_l = (muf * m.area[f]) * val;
            break;
        }
        case XCAL_BC_PERIODIC_PARENT: {  // own-row share; slots in k_bc_relax_scalar
            double an;
            periodic_div(bc, f, mdot[f], div_scheme, ap_d, an);
            periodic_lap(bc, f, muf, ap_l, an);
            break;
        }
        default:  // Empty, the periodic partner faces
            break;
    }
    double ap = 0.0, bp = 0.0;
    ap = ap + 0.0;  // Time
    bp = bp + 0.0;
    ap = ap + ap_d;
    bp = bp + bp_d;
    ap = ap + ap_l;
    bp = bp + bp_l;
    ap = ap + 0.0;  // Si
    bp = bp + 0.0;
    if (si2) {
        ap = ap + 0.0;
        bp = bp + 0.0;
    }
    AP = ap;
    BP = bp;
}

// apply_boundary_conditions! (ascending face id per cell) then
// implicit_relaxation_diagdom! (Solve_1_api.jl:388-411) of the k / omega
// equation, one thread per row.  Periodic pairs (periodic.jl:261-443): a
// parent face adds its own-row share through the functor and writes the
// (own, partner) slot; the partner cell adds its diagonal share and writes
// the (partner, own) slot -- its own boundary faces and the parent faces it
// partners merged in ascending face order, the reference's face loop order.
__global__ void k_bc_relax_scalar(MeshView m, CSRView A, BCView bc, double* nz, double* b,
                                  const double* __restrict__ mdot, const double* __restrict__ nutf, double nu,
                                  double sigma, const double* __restrict__ F1, double sigma2, int si2,
                                  const double* __restrict__ phi, double alpha, int div_scheme) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nC) return;
    const int ds = A.diag[i];
    double d = nz[ds];
    double bi = b[i];
    int k = m.bf_off[i];
    const int ke = m.bf_off[i + 1];
    int q = bc.pe_off ? bc.pe_off[i] : 0;
    const int qe = bc.pe_off ? bc.pe_off[i + 1] : 0;
    while (k < ke || q < qe) {
        const int fo = k < ke ? m.bf_face[k] : 0x7fffffff;
        const int fp = q < qe ? bc.pe_face[q] : 0x7fffffff;
        if (fo < fp) {
            const double muf = kw_mueff(m, fo, nutf, nu, sigma, F1, sigma2);
            double AP, BP;
            bc_scalar_transport(m, bc, fo, i, mdot, muf, phi, si2 != 0, div_scheme, AP, BP);
            d = d + AP;
            bi = bi + BP;
            if (bc.type[fo] == XCAL_BC_PERIODIC_PARENT) {  // (own, partner) slot from A0 = 0
                double acd, and_, acl, anl;
                periodic_div(bc, fo, mdot[fo], div_scheme, acd, and_);
                periodic_lap(bc, fo, muf, acl, anl);
                double v = 0.0;
                v = v + and_;
                v = v + anl;
                nz[bc.pPN[fo]] = v;
            }
            ++k;
        } else {  // this cell is the partner of parent face fp
            const double muf = kw_mueff(m, fp, nutf, nu, sigma, F1, sigma2);
            double acd, and_, acl, anl;
            periodic_div(bc, fp, mdot[fp], div_scheme, acd, and_);
            periodic_lap(bc, fp, muf, acl, anl);
            d = d + (-and_);
            d = d + (-anl);
            double v = 0.0;
            v = v + (-acd);
            v = v + (-acl);
            nz[bc.pNP[fp]] = v;
            ++q;
        }
    }
    double sumv = 0.0;
    const int rb = row_base(A, i), rl = A.len[i];
    for (int k = 0; k < rl; ++k) {
        int e = rb + SELL_C * k;
        sumv = sumv + fabs(e == ds ? d : nz[e]);
    }
    sumv = sumv - fabs(d);
    const double D0 = d;
    const double Dmax = jl_max(fabs(D0), sumv) / alpha;
    nz[ds] = Dmax;
    b[i] = bi + (Dmax - D0) * phi[i];
}

// constrain!(omega_eqn, OmegaWallFunction) (RANS_functions.jl:380-429) per
// wall cell: the row becomes omega = omega_log (y+ > yPlusLam) or omega_vis
// (:46-52) from the current k; par: y, kappa, beta1, cmu^0.25, yPlusLam
__global__ void k_omega_constrain(int nw, CSRView A, const int* __restrict__ wcell, const double* __restrict__ par,
                                  const double* __restrict__ k, double nu, double* nz, double* b) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nw) return;
    const int c = wcell[t];
    const double y = par[5 * t], kappa = par[5 * t + 1], beta1 = par[5 * t + 2], c25 = par[5 * t + 3],
                 yPlusLam = par[5 * t + 4];
    const double sk = sqrt(k[c]);
    const double w_vis = (6.0 * nu) / (beta1 * (y * y));
    const double w_log = sk / ((c25 * kappa) * y);
    const double yplus = ((c25 * y) * sk) / nu;
    const double wc = yplus > yPlusLam ? w_log : w_vis;
    const int rb = row_base(A, c), rl = A.len[c];
    for (int q = 0; q < rl; ++q) nz[rb + SELL_C * q] = 0.0;
    nz[A.diag[c]] = 1.0;
    b[c] = wc;
}

// bound! (RANS_functions.jl:2-41) from a copy of the values before the call
__global__ void k_bound(MeshView m, const double* __restrict__ old, double* v) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nC) return;
    const double mzero = jl_eps(1.0);
    double sum_flux = 0.0;
    int sum_area = 0;
    for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
        sum_flux = sum_flux + jl_max(old[m.cf_nb[k]], mzero);
        sum_area += 1;
    }
    const double average = sum_flux / (double)sum_area;
    const double vi = old[i];
    const double s = signbit(vi) ? average : copysign(0.0, average);
    v[i] = jl_max(jl_max(vi, s), mzero);
}

// k-omega SST cell fields (RANS_kOmegaSST.jl:214-266): |S|^2 (as k-omega),
// Omega = sqrt(2|S|^2), CDkw, arg1/arg2, F1 = tanh(arg1^4), F2 = tanh(arg2^2),
// beta and gamma blends, Dw = beta w, Dk = beta+ w, the limited productions
// and the cross-diffusion Si coefficient D2; g: grad U, gk / gw: grad k /
// grad omega
__global__ void k_sst_fields(int nC, const double* __restrict__ g0, const double* __restrict__ g1,
                             const double* __restrict__ g2, const double* __restrict__ g3,
                             const double* __restrict__ g4, const double* __restrict__ g5,
                             const double* __restrict__ g6, const double* __restrict__ g7,
                             const double* __restrict__ g8, const double* __restrict__ gkx,
                             const double* __restrict__ gky, const double* __restrict__ gkz,
                             const double* __restrict__ gwx, const double* __restrict__ gwy,
                             const double* __restrict__ gwz, const double* __restrict__ kf,
                             const double* __restrict__ omega, const double* __restrict__ nut,
                             const double* __restrict__ yw, double* F1o, double* F2o, double* Omo, double* Pk,
                             double* Pw, double* Dk, double* Dw, double* D2, double bs, double al1, double b1,
                             double b2, double sw2, double nu) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nC) return;
    const double G[9] = {g0[i], g1[i], g2[i], g3[i], g4[i], g5[i], g6[i], g7[i], g8[i]};
    double sum = 0.0;
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const double s = 0.5 * (G[3 * j + q] + G[3 * q + j]);
            sum = sum + s * s;
        }
    const double mag = sum * 2.0;
    const double Om = sqrt(mag);
    const double w = omega[i], kk = kf[i], y = yw[i];
    const double dkdw = (gkx[i] * gwx[i] + gky[i] * gwy[i]) + gkz[i] * gwz[i];
    const double CD = jl_max(((2.0 * sw2) * dkdw) / w, 1e-10);
    const double sq = sqrt(jl_max(kk, jl_eps(1.0)));
    const double a1 = jl_min(jl_min(jl_max(sq / ((bs * w) * y), (500.0 * nu) / (w * (y * y))),
                                    ((4.0 * sw2) * kk) / (CD * (y * y))),
                             10.0);
    const double a2 = jl_min(jl_max((2.0 * sq) / ((bs * w) * y), (500.0 * nu) / ((y * y) * w)), 100.0);
    const double f2 = det_tanh_pos(a2 * a2);
    const double f1 = det_tanh_pos((a1 * a1) * (a1 * a1));
    const double beta = b1 * f1 + (1.0 - f1) * b2;
    const double gamma = (5.0 / 9.0) * f1 + (1.0 - f1) * 0.44;
    F1o[i] = f1;
    F2o[i] = f2;
    Omo[i] = Om;
    Dw[i] = beta * w;
    Dk[i] = bs * w;
    Pw[i] = gamma * jl_min(mag, (((10.0 / al1) * bs) * w) * jl_max(al1 * w, f2 * Om));
    Pk[i] = jl_min(mag * nut[i], ((10.0 * bs) * kk) * w);
    D2[i] = ((((2.0 * (f1 - 1.0)) * sw2) * dkdw) / w) / w;
}

// nut = alpha1 k / max(alpha1 omega, F2 Omega) (RANS_kOmegaSST.jl:303-306)
__global__ void k_sst_nut(int nC, const double* __restrict__ k, const double* __restrict__ omega,
                          const double* __restrict__ F2, const double* __restrict__ Om, double al1, double* nut) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nC) nut[i] = (al1 * k[i]) / jl_max(al1 * omega[i], F2[i] * Om[i]);
}

// normal_distance! (Calculate_4_wall_distance.jl:80-92)
__global__ void k_walldist(int nC, const double* __restrict__ phi, const double* __restrict__ gx,
                           const double* __restrict__ gy, const double* __restrict__ gz, double* y) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nC) return;
    const double gm = sqrt(gx[i] * gx[i] + gy[i] * gy[i] + gz[i] * gz[i]);
    y[i] = (-gm) + sqrt(gm * gm + 2.0 * phi[i]);
}

// nut_wall (RANS_functions.jl:61-63)
__device__ __forceinline__ double nut_wall(double nu, double yplus, double kappa, double E) {
    return jl_max(nu * (((yplus * kappa) / det_log(jl_max(E * yplus, 1.0 + 1e-4))) - 1.0), 0.0);
}

// set_production!(Pk, KWallFunction) (RANS_functions.jl:84-117) per wall
// cell (its constraining face f): log-law production or 0 below yPlusLam;
// par per entry: kappa, cmu^0.25, yPlusLam, E
__global__ void k_kwall_production(int nw, MeshView m, const int* __restrict__ cell, const int* __restrict__ face,
                                   const double* __restrict__ par, const double* __restrict__ k,
                                   const double* __restrict__ Ux, const double* __restrict__ Uy,
                                   const double* __restrict__ Uz, double nu, double* Pk) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nw) return;
    const int c = cell[t], f = face[t];
    const double kappa = par[4 * t], c25 = par[4 * t + 1], yPlusLam = par[4 * t + 2], E = par[4 * t + 3];
    const double delta = m.delta[f];
    const double nx = m.nx[f], ny = m.ny[f], nz = m.nz[f];
    const double sk = sqrt(k[c]);
    const double uStar = c25 * sk;
    const double dUdy = uStar / (kappa * delta);
    const double yplus = ((c25 * delta) * sk) / nu;
    const double nutw = nut_wall(nu, yplus, kappa, E);
    const double ux = Ux[c] - 0.0, uy = Uy[c] - 0.0, uz = Uz[c] - 0.0;
    const double dn = ux * nx + uy * ny + uz * nz;
    const double gx = (ux - dn * nx) / delta, gy = (uy - dn * ny) / delta, gz = (uz - dn * nz) / delta;
    const double mag = sqrt(gx * gx + gy * gy + gz * gz);
    Pk[c] = yplus > yPlusLam ? ((nu + nutw) * mag) * dUdy : 0.0;
}

// correct_nut_wall!(nutf, NutWallFunction) (RANS_functions.jl:135-172) per
// wall face, then nueff = nu + nutf there
__global__ void k_nutwall(int nw, MeshView m, const int* __restrict__ face, const double* __restrict__ par,
                          const double* __restrict__ k, double nu, double* nutf, double* nueff) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nw) return;
    const int f = face[t], c = m.owner[f];
    const double kappa = par[4 * t], c25 = par[4 * t + 1], yPlusLam = par[4 * t + 2], E = par[4 * t + 3];
    const double yplus = ((c25 * m.delta[f]) * sqrt(k[c])) / nu;
    const double v = yplus > yPlusLam ? nut_wall(nu, yplus, kappa, E) : 0.0;
    nutf[f] = v;
    nueff[f] = nu + v;
}

// nut = k / omega (RANS_kOmega.jl:201)
__global__ void k_kw_nut(int nC, const double* __restrict__ k, const double* __restrict__ omega, double* nut) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nC) nut[i] = k[i] / omega[i];
}

// update_nueff_turbulent! (Solvers_0_functions.jl:30-35)
__global__ void k_nueff(int nF, const double* __restrict__ nutf, double* nueff, double nu) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f < nF) nueff[f] = nu + nutf[f];
}

// boundary conditions of the p equation (cells owning boundary faces)
__global__ void k_bc_p(MeshView m, CSRView A, BCView bc, double* nz, double* b, const double* __restrict__ rDf,
                       const double* __restrict__ p) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m.n_bcells) return;
    int i = m.bcells[t];
    int ds = A.diag[i];
    double d = nz[ds];
    double bi = b[i];
    // own boundary faces merged with the periodic parent faces this cell
    // partners, in ascending face order (see k_bc_relax_U)
    int k = m.bf_off[i], ke = m.bf_off[i + 1];
    int q = bc.pe_off ? bc.pe_off[i] : 0, qe = bc.pe_off ? bc.pe_off[i + 1] : 0;
    while (k < ke || q < qe) {
        int fo = k < ke ? m.bf_face[k] : 0x7fffffff;
        int fp = q < qe ? bc.pe_face[q] : 0x7fffffff;
        if (fo < fp) {
            double AP, BP;
            bc_p(m, bc, fo, i, rDf, p, AP, BP);
            d = d + AP;
            bi = bi + BP;
            if (bc.type[fo] == XCAL_BC_PERIODIC_PARENT) {
                double ac, an;
                periodic_lap(bc, fo, rDf[fo], ac, an);
                nz[bc.pPN[fo]] = 0.0 + an;
            }
            ++k;
        } else {
            double ac, an;
            periodic_lap(bc, fp, rDf[fp], ac, an);
            d = d + (-an);
            nz[bc.pNP[fp]] = 0.0 + (-ac);
            ++q;
        }
    }
    nz[ds] = d;
    b[i] = bi;
}

// setReference! (Solve_1_api.jl:431-439) on the row of the mesh's first cell
__global__ void k_set_reference(CSRView A, double* nz, double* b, double pref, int row) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        int c = A.diag[row];
        b[row] = nz[c] * pref;
        nz[c] = nz[c] + nz[c];
    }
}

// ---------------------------------------------------------------------------
// face interpolation + boundary values (+ flux)
// interpolate_Vector! (Calculate_2_interpolation.jl:374-397), correct_boundaries!
// (1_boundary_interpolation.jl), flux! (Solvers_0_functions.jl:51-62)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void periodic_interp3(const MeshView& m, const BCView& bc, int pf, const double* ux,
                                                 const double* uy, const double* uz, double& fx, double& fy,
                                                 double& fz) {
    // value written by the parent face pf (periodic_interpolation.jl:45-73)
    int c = m.owner[pf], pc = bc.peer_cell[pf];
    double w = bc.pw[pf], wn = bc.pwn[pf];
    fx = w * ux[c] + wn * ux[pc];
    fy = w * uy[c] + wn * uy[pc];
    fz = w * uz[c] + wn * uz[pc];
}

__global__ void k_interp_U(MeshView m, BCView bc, const double* __restrict__ ux, const double* __restrict__ uy,
                           const double* __restrict__ uz, double* fx, double* fy, double* fz, double* mdot) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nF) return;
    int o = m.owner[f], n = m.neigh[f];
    double w = m.weight[f];
    double omw = 1.0 - w;
    double vx = w * ux[o] + omw * ux[n];
    double vy = w * uy[o] + omw * uy[n];
    double vz = w * uz[o] + omw * uz[n];
    if (f < m.nB) {
        switch (bc.type[f]) {
            case XCAL_BC_DIRICHLET:
            case XCAL_BC_DIRICHLET_FUNCTION:
            case XCAL_BC_WALL:
                vx = bc_val(bc, f, 0);
                vy = bc_val(bc, f, 1);
                vz = bc_val(bc, f, 2);
                break;
            case XCAL_BC_ZEROGRADIENT:
            case XCAL_BC_EXTRAPOLATED:
                vx = ux[o];
                vy = uy[o];
                vz = uz[o];
                break;
            case XCAL_BC_EMPTY:
                vx = 0.0;
                vy = 0.0;
                vz = 0.0;
                break;
            case XCAL_BC_SYMMETRY: {
                double nx = m.nx[f], ny = m.ny[f], nz = m.nz[f];
                double px = ux[o], py = uy[o], pz = uz[o];
                double dd = px * nx + py * ny + pz * nz;
                vx = px - dd * nx;
                vy = py - dd * ny;
                vz = pz - dd * nz;
                break;
            }
            case XCAL_BC_PERIODIC_PARENT:
                periodic_interp3(m, bc, f, ux, uy, uz, vx, vy, vz);
                break;
            case XCAL_BC_PERIODIC:
                periodic_interp3(m, bc, bc.peer_face[f], ux, uy, uz, vx, vy, vz);
                break;
            default:
                break;
        }
    }
    if (fx) {
        fx[f] = vx;
        fy[f] = vy;
        fz[f] = vz;
    }
    if (mdot) mdot[f] = vx * m.Sx[f] + vy * m.Sy[f] + vz * m.Sz[f];
}

// scalar interpolation with the boundary values of a scalar field
// (p: Calculate_0_gradient.jl:105-111; nut: LES_Smagorinsky.jl:129-130)
__global__ void k_interp_scalar(MeshView m, BCView bc, const double* __restrict__ phi, double* phif,
                                double* nueff_out, double nu) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nF) return;
    int o = m.owner[f], n = m.neigh[f];
    double w = m.weight[f];
    double omw = 1.0 - w;
    double v = w * phi[o] + omw * phi[n];
    if (f < m.nB) {
        switch (bc.type[f]) {
            case XCAL_BC_DIRICHLET:
            case XCAL_BC_DIRICHLET_FUNCTION:
                v = bc_val(bc, f, 0);
                break;
            case XCAL_BC_WALL:
            case XCAL_BC_ZEROGRADIENT:
            case XCAL_BC_EXTRAPOLATED:
            case XCAL_BC_OMEGA_WALL:
            case XCAL_BC_K_WALL:
            case XCAL_BC_NUT_WALL:
            case XCAL_BC_SYMMETRY:
                v = phi[o];
                break;
            case XCAL_BC_EMPTY:
                v = 0.0;
                break;
            case XCAL_BC_NEUMANN:
                v = phi[o] + m.delta[f] * bc_val(bc, f, 0);
                break;
            case XCAL_BC_PERIODIC_PARENT: {
                int c = m.owner[f], pc = bc.peer_cell[f];
                v = bc.pw[f] * phi[c] + bc.pwn[f] * phi[pc];
                break;
            }
            case XCAL_BC_PERIODIC: {
                int pf = bc.peer_face[f];
                int c = m.owner[pf], pc = bc.peer_cell[pf];
                v = bc.pw[pf] * phi[c] + bc.pwn[pf] * phi[pc];
                break;
            }
            default:
                break;
        }
    }
    phif[f] = v;
    if (nueff_out) nueff_out[f] = nu + v;  // update_nueff_turbulent! (Solvers_0_functions.jl:30-35)
}

// interpolate!(rDf, rD) + correct_interpolation_periodic (Solvers_1_SIMPLE.jl:427-470)
__global__ void k_interp_rD(MeshView m, BCView bcU, const double* __restrict__ rD, double* rDf) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nF) return;
    int o = m.owner[f], n = m.neigh[f];
    double w = m.weight[f];
    double omw = 1.0 - w;
    double v = w * rD[o] + omw * rD[n];
    if (f < m.nB) {
        int pf = -1;
        if (bcU.type[f] == XCAL_BC_PERIODIC_PARENT) pf = f;
        if (bcU.type[f] == XCAL_BC_PERIODIC) pf = bcU.peer_face[f];
        if (pf >= 0) {
            double wp = bcU.pwdelta[pf];
            double omwp = 1.0 - wp;
            v = wp * rD[m.owner[pf]] + omwp * rD[bcU.peer_cell[pf]];
        }
    }
    rDf[f] = v;
}

__global__ void k_fill(double* a, double v, long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = v;
}

// ---------------------------------------------------------------------------
// Green-Gauss gradients (Calculate_1_green_gauss.jl:27-78, 106-173)
// ---------------------------------------------------------------------------
__global__ void k_green_gauss(MeshView m, const double* __restrict__ phif, double* gx, double* gy, double* gz) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nC) return;
    double rx = 0.0, ry = 0.0, rz = 0.0;
    for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
        int f = m.cf_face[k];
        double s = (double)m.cf_sign[k];
        double v = phif[f];
        rx = rx + v * (m.Sx[f] * s);
        ry = ry + v * (m.Sy[f] * s);
        rz = rz + v * (m.Sz[f] * s);
    }
    double V = m.vol[i];
    rx = rx / V;
    ry = ry / V;
    rz = rz / V;
    for (int k = m.bf_off[i]; k < m.bf_off[i + 1]; ++k) {
        int f = m.bf_face[k];
        double v = phif[f];
        rx = rx + (v * m.Sx[f]) / V;
        ry = ry + (v * m.Sy[f]) / V;
        rz = rz + (v * m.Sz[f]) / V;
    }
    gx[i] = rx;
    gy[i] = ry;
    gz[i] = rz;
}

// vector -> tensor; with Smagorinsky also nut = (C Delta)^2 sqrt(2 S:S)
// (LES_Smagorinsky.jl:122-127)
// |S| = sqrt((2S).S), S = 0.5 (G + G') over the column-major linear index
// (LES_Smagorinsky.jl:124-125); G row-major, G[3a+b] = dU_a/dx_b
__device__ __forceinline__ double smag_magS(const double r[9]) {
    double acc = 0.0;
    bool first = true;
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            double s = 0.5 * (r[3 * a + b] + r[3 * b + a]);
            double pr = (2.0 * s) * s;
            acc = first ? pr : acc + pr;
            first = false;
        }
    return sqrt(acc);
}

__global__ void k_green_gauss_tensor(MeshView m, const double* __restrict__ fx, const double* __restrict__ fy,
                                     const double* __restrict__ fz, double* g0, double* g1, double* g2, double* g3,
                                     double* g4, double* g5, double* g6, double* g7, double* g8,
                                     const double* __restrict__ Delta, double* nut) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nC) return;
    double r[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) r[q] = 0.0;
    for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
        int f = m.cf_face[k];
        double s = (double)m.cf_sign[k];
        double S[3] = {m.Sx[f] * s, m.Sy[f] * s, m.Sz[f] * s};
        double u[3] = {fx[f], fy[f], fz[f]};
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) r[3 * a + b] = r[3 * a + b] + u[a] * S[b];
    }
    double V = m.vol[i];
#pragma unroll
    for (int q = 0; q < 9; ++q) r[q] = r[q] / V;
    for (int k = m.bf_off[i]; k < m.bf_off[i + 1]; ++k) {
        int f = m.bf_face[k];
        double S[3] = {m.Sx[f], m.Sy[f], m.Sz[f]};
        double u[3] = {fx[f], fy[f], fz[f]};
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) r[3 * a + b] = r[3 * a + b] + (u[a] * S[b]) / V;
    }
    g0[i] = r[0];
    g1[i] = r[1];
    g2[i] = r[2];
    g3[i] = r[3];
    g4[i] = r[4];
    g5[i] = r[5];
    g6[i] = r[6];
    g7[i] = r[7];
    g8[i] = r[8];
    if (nut) nut[i] = Delta[i] * smag_magS(r);
}

// nut = Delta |S| from a stored grad U (LES_Smagorinsky.jl:122-127), for
// when grad U is limited between the gradient and nut
__global__ void k_smag_nut(int nC, const double* __restrict__ g0, const double* __restrict__ g1,
                           const double* __restrict__ g2, const double* __restrict__ g3, const double* __restrict__ g4,
                           const double* __restrict__ g5, const double* __restrict__ g6, const double* __restrict__ g7,
                           const double* __restrict__ g8, const double* __restrict__ Delta, double* nut) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nC) return;
    const double r[9] = {g0[i], g1[i], g2[i], g3[i], g4[i], g5[i], g6[i], g7[i], g8[i]};
    nut[i] = Delta[i] * smag_magS(r);
}

// div! of a face scalar (Calculate_0_divergence.jl:129-170)
__global__ void k_div(MeshView m, const double* __restrict__ psif, double* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nC) return;
    double red = 0.0;
    for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) red = red + psif[m.cf_face[k]] * (double)m.cf_sign[k];
    double V = m.vol[i];
    double r = red / V;
    for (int k = m.bf_off[i]; k < m.bf_off[i + 1]; ++k) r = r + psif[m.bf_face[k]] / V;
    out[i] = r;
}

// ---- Midpoint gradient (Calculate_0_gradient.jl:170-262) ----
// interpolate_midpoint! on internal faces (boundary faces keep the values the
// boundary interpolation gave them): phif = 0.5 (phi1 + phi2)
__global__ void k_mid_scalar(MeshView m, const double* __restrict__ phi, double* phif) {
    int f = m.nB + blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nF) return;
    phif[f] = 0.5 * (phi[m.owner[f]] + phi[m.neigh[f]]);
}
__global__ void k_mid_vector(MeshView m, const double* __restrict__ ux, const double* __restrict__ uy,
                             const double* __restrict__ uz, double* fx, double* fy, double* fz) {
    int f = m.nB + blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nF) return;
    const int o = m.owner[f], n = m.neigh[f];
    fx[f] = 0.5 * (ux[o] + ux[n]);
    fy[f] = 0.5 * (uy[o] + uy[n]);
    fz[f] = 0.5 * (uz[o] + uz[n]);
}
// correct_interpolation!: phif = 0.5 (phi1 + phi2) + (0.5 (grad1 + grad2)).Ri
__global__ void k_mid_correct_scalar(MeshView m, const double* __restrict__ R, const double* __restrict__ phi,
                                     const double* __restrict__ gx, const double* __restrict__ gy,
                                     const double* __restrict__ gz, double* phif) {
    int f = m.nB + blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nF) return;
    const int nI = m.nF - m.nB, j = f - m.nB, o = m.owner[f], n = m.neigh[f];
    const double ax = 0.5 * (gx[o] + gx[n]), ay = 0.5 * (gy[o] + gy[n]), az = 0.5 * (gz[o] + gz[n]);
    phif[f] = 0.5 * (phi[o] + phi[n]) + (ax * R[j] + ay * R[nI + j] + az * R[2 * nI + j]);
}
// vector field, tensor gradient g[3a+b] = d u_a / d x_b:
// phif_a = 0.5 (u_a1 + u_a2) + ((M[a,1] R1 + M[a,2] R2) + M[a,3] R3), M = 0.5 (grad1 + grad2)
struct Grad9 {
    const double* g[9];
};
__global__ void k_mid_correct_vector(MeshView m, const double* __restrict__ R, const double* __restrict__ ux,
                                     const double* __restrict__ uy, const double* __restrict__ uz, Grad9 G,
                                     double* fx, double* fy, double* fz) {
    int f = m.nB + blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nF) return;
    const int nI = m.nF - m.nB, j = f - m.nB, o = m.owner[f], n = m.neigh[f];
    const double Rx = R[j], Ry = R[nI + j], Rz = R[2 * nI + j];
    const double* u[3] = {ux, uy, uz};
    double* out[3] = {fx, fy, fz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double M0 = 0.5 * (G.g[3 * a][o] + G.g[3 * a][n]);
        const double M1 = 0.5 * (G.g[3 * a + 1][o] + G.g[3 * a + 1][n]);
        const double M2 = 0.5 * (G.g[3 * a + 2][o] + G.g[3 * a + 2][n]);
        out[a][f] = 0.5 * (u[a][o] + u[a][n]) + (M0 * Rx + M1 * Ry + M2 * Rz);
    }
}

// limit_gradient!(CellBased(level)) (Calculate_0_gradient_cell_limiter.jl:
// 68-108), one thread per cell, for a scalar field F and its gradient (one
// row of grad U for a vector field): F's max/min over the cell's neighbours,
// the smallest ratio over its internal faces of the allowed change to the
// extrapolated change d.grad (d = fc - cc, D: 3 arrays over the cell_faces
// entries), |d.grad| > 10 eps(F_P); grad *= 1 - level (1 - limiter)
__global__ void k_limit_cell(MeshView m, const double* __restrict__ D, const double* __restrict__ F, double* gx,
                             double* gy, double* gz, double level) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nC) return;
    const int nk = 2 * (m.nF - m.nB);
    const double phiP = F[i];
    double phiMax = phiP, phiMin = phiP;
    for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
        const double phiN = F[m.cf_nb[k]];
        phiMax = jl_max(phiN, phiMax);
        phiMin = jl_min(phiN, phiMin);
    }
    const double x = gx[i], y = gy[i], z = gz[i];
    double lim = 1.0;
    const double e = 10.0 * jl_eps(phiP);
    for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
        const double d = D[k] * x + D[nk + k] * y + D[2 * nk + k] * z;
        if (d > e)
            lim = jl_min(lim, (phiMax - phiP) / d);
        else if (d < -e)
            lim = jl_min(lim, (phiMin - phiP) / d);
    }
    lim = 1.0 - level * (1.0 - lim);
    gx[i] = x * lim;
    gy[i] = y * lim;
    gz[i] = z * lim;
}

// limit_gradient!(FaceBased) (Calculate_0_gradient_face_limiter.jl:31-113,
// 152-170) as a gather, one thread per cell.  The reference runs one thread
// per internal face, each lowering both of its cells' limiters with an
// atomic minimum (compare-and-swap while the value is smaller); a cell's
// limiter is thus the smallest of its faces' candidate ratios and 1, the
// same in any order -- here its faces in cell_faces order.  Per face: the
// bounds min/max(F_own, F_nei) widened by their difference, this cell's
// extrapolated change dF = grad . (fc - cc) (D), and the candidate
// (Fmax - F)/dF when dF > Fmax - F, (Fmin - F)/dF when dF < Fmin - F; then
// grad *= limiter.
__global__ void k_limit_face_scalar(MeshView m, const double* __restrict__ D, const double* __restrict__ F,
                                    double* gx, double* gy, double* gz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nC) return;
    const int nk = 2 * (m.nF - m.nB);
    const double x = gx[i], y = gy[i], z = gz[i];
    const double Fi = F[i];
    double lim = 1.0;
    for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
        const double Fo = F[m.cf_nb[k]];
        const bool own = m.cf_sign[k] > 0;
        double mn = own ? jl_min(Fi, Fo) : jl_min(Fo, Fi);
        double mx = own ? jl_max(Fi, Fo) : jl_max(Fo, Fi);
        const double dl = mx - mn;
        mn = mn - dl;
        mx = mx + dl;
        const double dF = (x * D[k] + y * D[nk + k]) + z * D[2 * nk + k];
        const double dmax = mx - Fi, dmin = mn - Fi;
        if (dF > dmax) {
            const double v = dmax / dF;
            if (v < lim) lim = v;
        } else if (dF < dmin) {
            const double v = dmin / dF;
            if (v < lim) lim = v;
        }
    }
    gx[i] = x * lim;
    gy[i] = y * lim;
    gz[i] = z * lim;
}

// the vector form (:94-151, OpenFOAM's faceLimitedGrad<vector>): per face
// side the gradient tensor times (fc - cc) gives gradf; both cells' values
// projected on it bound this cell's projected value, the extrapolation
// measure is gradf . gradf; one limiter scales all nine components.
// G[a][b] = g[3 a + b] is entry (a, b) of the tensor.
struct GradW9 {
    double* g[9];
};
__global__ void k_limit_face_vector(MeshView m, const double* __restrict__ D, const double* __restrict__ U0,
                                    const double* __restrict__ U1, const double* __restrict__ U2, GradW9 Gd) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nC) return;
    const int nk = 2 * (m.nF - m.nB);
    double G[9];
    for (int q = 0; q < 9; ++q) G[q] = Gd.g[q][i];
    const double ui[3] = {U0[i], U1[i], U2[i]};
    double lim = 1.0;
    for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
        const int o = m.cf_nb[k];
        const double uo[3] = {U0[o], U1[o], U2[o]};
        const double d[3] = {D[k], D[nk + k], D[2 * nk + k]};
        double gf[3];
        for (int a = 0; a < 3; ++a) gf[a] = (G[3 * a] * d[0] + G[3 * a + 1] * d[1]) + G[3 * a + 2] * d[2];
        const double vi = (gf[0] * ui[0] + gf[1] * ui[1]) + gf[2] * ui[2];
        const double vo = (gf[0] * uo[0] + gf[1] * uo[1]) + gf[2] * uo[2];
        const bool own = m.cf_sign[k] > 0;
        const double vOwn = own ? vi : vo, vNei = own ? vo : vi;
        double mx = jl_max(vOwn, vNei), mn = jl_min(vOwn, vNei);
        const double dl = mx - mn;
        mx = mx + dl;
        mn = mn - dl;
        const double dF = (gf[0] * gf[0] + gf[1] * gf[1]) + gf[2] * gf[2];
        const double dmax = mx - vi, dmin = mn - vi;
        if (dF > dmax) {
            const double v = dmax / dF;
            if (v < lim) lim = v;
        } else if (dF < dmin) {
            const double v = dmin / dF;
            if (v < lim) lim = v;
        }
    }
    for (int q = 0; q < 9; ++q) Gd.g[q][i] = G[q] * lim;
}

// nonorthogonal_face_correction (Solvers_1_SIMPLE.jl:267-318), one thread
// per cell: b_i gets each of its internal faces' correction, in its
// cell_faces order (+ as owner, - as neighbour; the reference adds with
// atomics in no fixed order).  t: per internal face w, ex, ey, ez, Tx, Ty,
// Tz (Case::build_nonorth).
__global__ void k_nonorth_correct(MeshView m, const double* __restrict__ t, const double* __restrict__ p,
                                  const double* __restrict__ gx, const double* __restrict__ gy,
                                  const double* __restrict__ gz, const double* __restrict__ rDf, double* b) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nC) return;
    const int nI = m.nF - m.nB;
    double bi = b[i];
    for (int k = m.cf_off[i]; k < m.cf_off[i + 1]; ++k) {
        const int f = m.cf_face[k], j = f - m.nB, c1 = m.owner[f], c2 = m.neigh[f];
        const double w = t[j], ex = t[nI + j], ey = t[2 * nI + j], ez = t[3 * nI + j];
        const double Tx = t[4 * nI + j], Ty = t[5 * nI + j], Tz = t[6 * nI + j];
        const double w1 = 1.0 - w;
        // gradi = w grad[c1] + (1 - w) grad[c2]
        const double gix = w * gx[c1] + w1 * gx[c2], giy = w * gy[c1] + w1 * gy[c2], giz = w * gz[c1] + w1 * gz[c2];
        // gradf = gradi + ((p2 - p1)/delta - gradi.e) e
        const double s = (p[c2] - p[c1]) / m.delta[f] - (gix * ex + giy * ey + giz * ez);
        const double gfx = gix + s * ex, gfy = giy + s * ey, gfz = giz + s * ez;
        // (rDf gradf) . T
        const double r = rDf[f];
        const double corr = (r * gfx) * Tx + (r * gfy) * Ty + (r * gfz) * Tz;
        bi = c1 == i ? bi + corr : bi - corr;
    }
    b[i] = bi;
}

// ---------------------------------------------------------------------------
// pressure-velocity coupling (Solvers_0_functions.jl, Solvers_1_SIMPLE.jl)
// ---------------------------------------------------------------------------
// inverse_diagonal! (:108-120) + remove_pressure_source! (:170-181) + H! (:201-249)
__global__ void k_rD_remove_H(MeshView m, CSRView A, const double* __restrict__ nz, const double* __restrict__ Ux,
                              const double* __restrict__ Uy, const double* __restrict__ Uz,
                              const double* __restrict__ gx, const double* __restrict__ gy,
                              const double* __restrict__ gz, double* bx, double* by, double* bz, double* rD,
                              double* Hx, double* Hy, double* Hz, int do_H) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nC) return;
    double V = m.vol[i];
    double D = nz[A.diag[i]];
    rD[i] = V / D;
    double cx = (-1.0 * gx[i]) * V, cy = (-1.0 * gy[i]) * V, cz = (-1.0 * gz[i]) * V;
    double bxi = bx[i] - cx, byi = by[i] - cy, bzi = bz[i] - cz;
    bx[i] = bxi;
    by[i] = byi;
    bz[i] = bzi;
    if (!do_H) return;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    const int rb = row_base(A, i), rl = A.len[i];
    for (int k = 0; k < rl; ++k) {
        int e = rb + SELL_C * k;
        int j = A.colval[e];
        double val = nz[e];
        sx = sx + val * Ux[j];
        sy = sy + val * Uy[j];
        sz = sz + val * Uz[j];
    }
    sx = sx - D * Ux[i];
    sy = sy - D * Uy[i];
    sz = sz - D * Uz[i];
    double r = 1.0 / D;
    Hx[i] = (bxi - sx) * r;
    Hy[i] = (byi - sy) * r;
    Hz[i] = (bzi - sz) * r;
}

// H! alone (PISO correctors, Solvers_2_PISO.jl:122)
__global__ void k_H(MeshView m, CSRView A, const double* __restrict__ nz, const double* __restrict__ Ux,
                    const double* __restrict__ Uy, const double* __restrict__ Uz, const double* __restrict__ bx,
                    const double* __restrict__ by, const double* __restrict__ bz, double* Hx, double* Hy,
                    double* Hz) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nC) return;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    const int rb = row_base(A, i), rl = A.len[i];
    for (int k = 0; k < rl; ++k) {
        int e = rb + SELL_C * k;
        int j = A.colval[e];
        double val = nz[e];
        sx = sx + val * Ux[j];
        sy = sy + val * Uy[j];
        sz = sz + val * Uz[j];
    }
    double D = nz[A.diag[i]];
    sx = sx - D * Ux[i];
    sy = sy - D * Uy[i];
    sz = sz - D * Uz[i];
    double r = 1.0 / D;
    Hx[i] = (bx[i] - sx) * r;
    Hy[i] = (by[i] - sy) * r;
    Hz[i] = (bz[i] - sz) * r;
}

// correct_mass_flux! (Solvers_1_SIMPLE.jl:371-388), periodic (:403-425),
// boundary (:474-557)
__global__ void k_correct_mdot(MeshView m, CSRView A, BCView bcp, const double* __restrict__ nz,
                               const double* __restrict__ p, const double* __restrict__ rDf, double* mdot) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nF) return;
    if (f >= m.nB) {
        int o = m.owner[f], n = m.neigh[f];
        double aN = nz[A.fslot[f - m.nB]];
        mdot[f] = mdot[f] + aN * (p[n] - p[o]);
        return;
    }
    int c = m.bcell[f];
    switch (bcp.type[f]) {
        case XCAL_BC_DIRICHLET:
        case XCAL_BC_DIRICHLET_FUNCTION: {
            double fl = (rDf[f] * m.area[f]) / m.delta[f];
            double ap = -1.0 * (-fl);
            mdot[f] = mdot[f] + ap * (p[c] - bc_val(bcp, f, 0));
            break;
        }
        case XCAL_BC_NEUMANN:
            mdot[f] = mdot[f] - (rDf[f] * m.area[f]) * bc_val(bcp, f, 0);
            break;
        case XCAL_BC_PERIODIC_PARENT: {
            int pf = bcp.peer_face[f];
            int c2 = bcp.peer_cell[f];
            double aN = nz[bcp.pPN[f]];
            double corr = aN * (p[c2] - p[c]);
            double v = mdot[f] + corr;
            mdot[f] = v;
            mdot[pf] = -v;
            break;
        }
        default:
            break;
    }
}

// correct_velocity! (Solvers_0_functions.jl:136-151)
__global__ void k_correct_U(int n, const double* __restrict__ Hx, const double* __restrict__ Hy,
                            const double* __restrict__ Hz, const double* __restrict__ gx,
                            const double* __restrict__ gy, const double* __restrict__ gz,
                            const double* __restrict__ rD, double* Ux, double* Uy, double* Uz) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double r = rD[i];
    Ux[i] = Hx[i] - gx[i] * r;
    Uy[i] = Hy[i] - gy[i] * r;
    Uz[i] = Hz[i] - gz[i] * r;
}

// explicit_relaxation! (Solve_1_api.jl:327-335)
__global__ void k_relax_explicit(int n, double* phi, const double* __restrict__ phi0, double alpha) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    phi[i] = phi0[i] + alpha * (phi[i] - phi0[i]);
}

// _max_courant_number! (Solvers_0_functions.jl:267-276): per-cell Courant
// number and its maximum (Julia max; exact, so the tree order is free), the
// last block writing the result
__global__ void k_courant_max(int n, const double* __restrict__ Ux, const double* __restrict__ Uy,
                              const double* __restrict__ Uz, const double* __restrict__ dx, double dt, double* part,
                              unsigned int* counter, double* out) {
    __shared__ double sm[8];
    double mx = -INFINITY;
    for (int k = 0; k < RED_ITEMS; ++k) {
        int i = tile_row(k);
        if (i < n) {
            double umag = sqrt(Ux[i] * Ux[i] + Uy[i] * Uy[i] + Uz[i] * Uz[i]);
            mx = jl_max(mx, (umag * dt) / dx[i]);
        }
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) mx = jl_max(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sm[warp] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = sm[0];
        for (int w = 1; w < RED_THREADS / 32; ++w) b = jl_max(b, sm[w]);
        part[blockIdx.x] = b;
    }
    if (!last_block(counter)) return;
    if (threadIdx.x == 0) {
        int T = gridDim.x;
        double r = __ldcg(part);
        for (int t = 1; t < T; ++t) r = jl_max(r, __ldcg(part + t));
        *out = r;
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
void launch_assemble_U(cudaStream_t s, const MeshView& m, const CSRView& A, const double* mdot, const double* nueff,
                       const double* const U[3], const double* const g[3], double* nz, double* diag0,
                       double* const b[3], int time_scheme, int div_scheme, double dt) {
    k_assemble_U<<<nblk(m.nC), TPB, 0, s>>>(m, A, mdot, nueff, U[0], U[1], U[2], g[0], g[1], g[2], nz, diag0, b[0],
                                            b[1], b[2], time_scheme, div_scheme, dt);
    XCAL_CHECK_LAUNCH();
}
void launch_assemble_p(cudaStream_t s, const MeshView& m, const CSRView& A, const double* rDf, const double* divHv,
                       double* nz, double* b) {
    k_assemble_p<<<nblk(m.nC), TPB, 0, s>>>(m, A, rDf, divHv, nz, b);
    XCAL_CHECK_LAUNCH();
}
void launch_bc_relax_U(cudaStream_t s, const MeshView& m, const CSRView& A, const BCView& bc, int comp,
                       int div_scheme, double* nz, const double* diag0, double* b, const double* mdot,
                       const double* nueff, const double* const U[3], double alpha, int flags) {
    k_bc_relax_U<<<nblk(m.nC), TPB, 0, s>>>(m, A, bc, comp, div_scheme, nz, diag0, b, mdot, nueff, U[0], U[1], U[2],
                                            alpha, flags);
    XCAL_CHECK_LAUNCH();
}
void launch_bc_p(cudaStream_t s, const MeshView& m, const CSRView& A, const BCView& bc, double* nz, double* b,
                 const double* rDf, const double* p) {
    if (m.n_bcells == 0) return;
    k_bc_p<<<nblk(m.n_bcells), TPB, 0, s>>>(m, A, bc, nz, b, rDf, p);
    XCAL_CHECK_LAUNCH();
}
void launch_set_reference(cudaStream_t s, const CSRView& A, double* nz, double* b, double pref, int row) {
    k_set_reference<<<1, 32, 0, s>>>(A, nz, b, pref, row);
    XCAL_CHECK_LAUNCH();
}
void launch_interp_U(cudaStream_t s, const MeshView& m, const BCView& bc, const double* const U[3], double* const Uf[3],
                     double* mdot) {
    k_interp_U<<<nblk(m.nF), TPB, 0, s>>>(m, bc, U[0], U[1], U[2], Uf ? Uf[0] : nullptr, Uf ? Uf[1] : nullptr,
                                          Uf ? Uf[2] : nullptr, mdot);
    XCAL_CHECK_LAUNCH();
}
void launch_interp_scalar(cudaStream_t s, const MeshView& m, const BCView& bc, const double* phi, double* phif,
                          double* nueff, double nu) {
    k_interp_scalar<<<nblk(m.nF), TPB, 0, s>>>(m, bc, phi, phif, nueff, nu);
    XCAL_CHECK_LAUNCH();
}
void launch_interp_rD(cudaStream_t s, const MeshView& m, const BCView& bcU, const double* rD, double* rDf) {
    k_interp_rD<<<nblk(m.nF), TPB, 0, s>>>(m, bcU, rD, rDf);
    XCAL_CHECK_LAUNCH();
}
void launch_fill(cudaStream_t s, double* a, double v, long n) {
    if (n <= 0) return;
    k_fill<<<(int)((n + TPB - 1) / TPB), TPB, 0, s>>>(a, v, n);
    XCAL_CHECK_LAUNCH();
}
void launch_green_gauss(cudaStream_t s, const MeshView& m, const double* phif, double* const g[3]) {
    k_green_gauss<<<nblk(m.nC), TPB, 0, s>>>(m, phif, g[0], g[1], g[2]);
    XCAL_CHECK_LAUNCH();
}
void launch_green_gauss_tensor(cudaStream_t s, const MeshView& m, double* const Uf[3], double* const g[9],
                               const double* Delta, double* nut) {
    k_green_gauss_tensor<<<nblk(m.nC), TPB, 0, s>>>(m, Uf[0], Uf[1], Uf[2], g[0], g[1], g[2], g[3], g[4], g[5], g[6],
                                                    g[7], g[8], Delta, nut);
    XCAL_CHECK_LAUNCH();
}
static inline int nblk_i(const MeshView& m) { return std::max(1, (m.nF - m.nB + TPB - 1) / TPB); }
void launch_mid_scalar(cudaStream_t s, const MeshView& m, const double* phi, double* phif) {
    if (m.nF == m.nB) return;
    k_mid_scalar<<<nblk_i(m), TPB, 0, s>>>(m, phi, phif);
    XCAL_CHECK_LAUNCH();
}
void launch_mid_vector(cudaStream_t s, const MeshView& m, const double* const U[3], double* const Uf[3]) {
    if (m.nF == m.nB) return;
    k_mid_vector<<<nblk_i(m), TPB, 0, s>>>(m, U[0], U[1], U[2], Uf[0], Uf[1], Uf[2]);
    XCAL_CHECK_LAUNCH();
}
void launch_mid_correct_scalar(cudaStream_t s, const MeshView& m, const double* R, const double* phi,
                               const double* const g[3], double* phif) {
    if (m.nF == m.nB) return;
    k_mid_correct_scalar<<<nblk_i(m), TPB, 0, s>>>(m, R, phi, g[0], g[1], g[2], phif);
    XCAL_CHECK_LAUNCH();
}
void launch_mid_correct_vector(cudaStream_t s, const MeshView& m, const double* R, const double* const U[3],
                               const double* const g[9], double* const Uf[3]) {
    if (m.nF == m.nB) return;
    Grad9 G;
    for (int q = 0; q < 9; ++q) G.g[q] = g[q];
    k_mid_correct_vector<<<nblk_i(m), TPB, 0, s>>>(m, R, U[0], U[1], U[2], G, Uf[0], Uf[1], Uf[2]);
    XCAL_CHECK_LAUNCH();
}
void launch_limit_cell(cudaStream_t s, const MeshView& m, const double* D, const double* F, double* const g[3],
                       double level) {
    k_limit_cell<<<nblk(m.nC), TPB, 0, s>>>(m, D, F, g[0], g[1], g[2], level);
    XCAL_CHECK_LAUNCH();
}
// limit_gradient!(::MFaceBased) (Calculate_0_gradient_mface_limiter.jl):
// each internal face moves both cells' gradients so that the extrapolation
// grad . d (d = fc - cc) stays within [min, max](F_own, F_nei) - F_cell,
// grad += d (bound - grad . d) / (d . d).  A face's two updates read and
// write different cells, so a cell's result is its own faces' updates
// applied in turn; here in ascending face order (ord: the cell's cell_faces
// entries sorted by the reference's face id), the reference's kernel run on
// one thread.  (Its parallel runs race on cells that share faces.)
__global__ void k_limit_mface_scalar(MeshView m, const int* __restrict__ ord, const double* __restrict__ D,
                                     const double* __restrict__ F, double* gx, double* gy, double* gz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nC) return;
    const int nk = 2 * (m.nF - m.nB);
    double x = gx[i], y = gy[i], z = gz[i];
    const double Fi = F[i];
    for (int e = m.cf_off[i]; e < m.cf_off[i + 1]; ++e) {
        const int k = ord[e];
        const double Fo = F[m.cf_nb[k]];
        const bool own = m.cf_sign[k] > 0;
        const double F1 = own ? Fi : Fo, F2 = own ? Fo : Fi;
        const double dmax = jl_max(F1, F2) - Fi, dmin = jl_min(F1, F2) - Fi;
        const double d0 = D[k], d1 = D[nk + k], d2 = D[2 * nk + k];
        const double fval = (x * d0 + y * d1) + z * d2;
        const double dd = (d0 * d0 + d1 * d1) + d2 * d2;
        if (fval > dmax || fval < dmin) {
            const double t = (fval > dmax ? dmax : dmin) - fval;
            x = x + (d0 * t) / dd;
            y = y + (d1 * t) / dd;
            z = z + (d2 * t) / dd;
        }
    }
    gx[i] = x;
    gy[i] = y;
    gz[i] = z;
}

// Julia's isless / isequal on Float64 (NaN above everything, -0.0 < 0.0)
__device__ __forceinline__ bool jl_isless(double a, double b) {
    if (isnan(a)) return false;
    if (isnan(b)) return true;
    return a < b || (a == b && signbit(a) && !signbit(b));
}
__device__ __forceinline__ bool jl_isequal(double a, double b) {
    if (isnan(a) || isnan(b)) return isnan(a) && isnan(b);
    return a == b && signbit(a) == signbit(b);
}
// isless of two 3-vectors: Base's lexicographic cmp (the first entry that
// differs by isequal decides by isless)
__device__ __forceinline__ bool lex_isless(const double* a, const double* b) {
    for (int j = 0; j < 3; ++j)
        if (!jl_isequal(a[j], b[j])) return jl_isless(a[j], b[j]);
    return false;
}

// the tensor form: min / max(U_own, U_nei) are Base's generic min / max of
// two vectors, whole vectors chosen by the lexicographic isless; each row a
// of grad U (d u_a / d x_b) is corrected against component a of the bounds
__global__ void k_limit_mface_vector(MeshView m, const int* __restrict__ ord, const double* __restrict__ D,
                                     const double* __restrict__ U0, const double* __restrict__ U1,
                                     const double* __restrict__ U2, GradW9 Gd) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nC) return;
    const int nk = 2 * (m.nF - m.nB);
    double G[9];
    for (int q = 0; q < 9; ++q) G[q] = Gd.g[q][i];
    const double ui[3] = {U0[i], U1[i], U2[i]};
    for (int e = m.cf_off[i]; e < m.cf_off[i + 1]; ++e) {
        const int k = ord[e];
        const int o = m.cf_nb[k];
        const double uo[3] = {U0[o], U1[o], U2[o]};
        const bool own = m.cf_sign[k] > 0;
        const double* F1 = own ? ui : uo;
        const double* F2 = own ? uo : ui;
        const bool lt = lex_isless(F2, F1);  // max = F1 if F2 < F1, min = F2 then
        const double* mx = lt ? F1 : F2;
        const double* mn = lt ? F2 : F1;
        const double d[3] = {D[k], D[nk + k], D[2 * nk + k]};
        const double dd = (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2];
        for (int a = 0; a < 3; ++a) {
            const double dmax = mx[a] - ui[a], dmin = mn[a] - ui[a];
            const double fval = (G[3 * a] * d[0] + G[3 * a + 1] * d[1]) + G[3 * a + 2] * d[2];
            if (fval > dmax || fval < dmin) {
                const double t = (fval > dmax ? dmax : dmin) - fval;
                for (int b = 0; b < 3; ++b) G[3 * a + b] = G[3 * a + b] + (d[b] * t) / dd;
            }
        }
    }
    for (int q = 0; q < 9; ++q) Gd.g[q][i] = G[q];
}

void launch_limit_mface_scalar(cudaStream_t s, const MeshView& m, const int* ord, const double* D, const double* F,
                               double* const g[3]) {
    k_limit_mface_scalar<<<nblk(m.nC), TPB, 0, s>>>(m, ord, D, F, g[0], g[1], g[2]);
    XCAL_CHECK_LAUNCH();
}
void launch_limit_mface_vector(cudaStream_t s, const MeshView& m, const int* ord, const double* D,
                               const double* const U[3], double* const g[9]) {
    GradW9 G;
    for (int q = 0; q < 9; ++q) G.g[q] = g[q];
    k_limit_mface_vector<<<nblk(m.nC), TPB, 0, s>>>(m, ord, D, U[0], U[1], U[2], G);
    XCAL_CHECK_LAUNCH();
}
void launch_limit_face_scalar(cudaStream_t s, const MeshView& m, const double* D, const double* F,
                              double* const g[3]) {
    k_limit_face_scalar<<<nblk(m.nC), TPB, 0, s>>>(m, D, F, g[0], g[1], g[2]);
    XCAL_CHECK_LAUNCH();
}
void launch_limit_face_vector(cudaStream_t s, const MeshView& m, const double* D, const double* const U[3],
                              double* const g[9]) {
    GradW9 G;
    for (int q = 0; q < 9; ++q) G.g[q] = g[q];
    k_limit_face_vector<<<nblk(m.nC), TPB, 0, s>>>(m, D, U[0], U[1], U[2], G);
    XCAL_CHECK_LAUNCH();
}
void launch_kw_sources(cudaStream_t s, int nC, const double* const g[9], const double* nut, const double* omega,
                       double* Pk, double* Pw, double* Dk, double* Dw, double alpha1, double beta1, double beta_star) {
    k_kw_sources<<<nblk(nC), TPB, 0, s>>>(nC, g[0], g[1], g[2], g[3], g[4], g[5], g[6], g[7], g[8], nut, omega, Pk, Pw,
                                          Dk, Dw, alpha1, beta1, beta_star);
    XCAL_CHECK_LAUNCH();
}
void launch_assemble_scalar(cudaStream_t s, const MeshView& m, const CSRView& A, const double* mdot,
                            const double* nutf, double nu, double sigma, const double* F1, double sigma2,
                            const double* phi, const double* D, const double* D2, const double* P, double* nz,
                            double* b, int time_scheme, int div_scheme, double dt, double d2_sign) {
    k_assemble_scalar<<<nblk(m.nC), TPB, 0, s>>>(m, A, mdot, nutf, nu, sigma, F1, sigma2, phi, D, D2, P, nz, b,
                                                 time_scheme, div_scheme, dt, d2_sign);
    XCAL_CHECK_LAUNCH();
}
void launch_bc_relax_scalar(cudaStream_t s, const MeshView& m, const CSRView& A, const BCView& bc, double* nz,
                            double* b, const double* mdot, const double* nutf, double nu, double sigma,
                            const double* F1, double sigma2, int si2, const double* phi, double alpha,
                            int div_scheme) {
    k_bc_relax_scalar<<<nblk(m.nC), TPB, 0, s>>>(m, A, bc, nz, b, mdot, nutf, nu, sigma, F1, sigma2, si2, phi, alpha,
                                                 div_scheme);
    XCAL_CHECK_LAUNCH();
}
void launch_sst_fields(cudaStream_t s, int nC, const double* const g[9], const double* const gk[3],
                       const double* const gw[3], const double* k, const double* omega, const double* nut,
                       const double* yw, double* F1, double* F2, double* Om, double* Pk, double* Pw, double* Dk,
                       double* Dw, double* D2, double bs, double al1, double b1, double b2, double sw2, double nu) {
    k_sst_fields<<<nblk(nC), TPB, 0, s>>>(nC, g[0], g[1], g[2], g[3], g[4], g[5], g[6], g[7], g[8], gk[0], gk[1],
                                          gk[2], gw[0], gw[1], gw[2], k, omega, nut, yw, F1, F2, Om, Pk, Pw, Dk, Dw,
                                          D2, bs, al1, b1, b2, sw2, nu);
    XCAL_CHECK_LAUNCH();
}
void launch_sst_nut(cudaStream_t s, int nC, const double* k, const double* omega, const double* F2, const double* Om,
                    double al1, double* nut) {
    k_sst_nut<<<nblk(nC), TPB, 0, s>>>(nC, k, omega, F2, Om, al1, nut);
    XCAL_CHECK_LAUNCH();
}
void launch_kwall_production(cudaStream_t s, int nw, const MeshView& m, const int* cell, const int* face,
                             const double* par, const double* k, const double* const U[3], double nu, double* Pk) {
    if (nw <= 0) return;
    k_kwall_production<<<nblk(nw), TPB, 0, s>>>(nw, m, cell, face, par, k, U[0], U[1], U[2], nu, Pk);
    XCAL_CHECK_LAUNCH();
}
void launch_nutwall(cudaStream_t s, int nw, const MeshView& m, const int* face, const double* par, const double* k,
                    double nu, double* nutf, double* nueff) {
    if (nw <= 0) return;
    k_nutwall<<<nblk(nw), TPB, 0, s>>>(nw, m, face, par, k, nu, nutf, nueff);
    XCAL_CHECK_LAUNCH();
}
void launch_walldist(cudaStream_t s, int nC, const double* phi, const double* const g[3], double* y) {
    k_walldist<<<nblk(nC), TPB, 0, s>>>(nC, phi, g[0], g[1], g[2], y);
    XCAL_CHECK_LAUNCH();
}
void launch_omega_constrain(cudaStream_t s, int nw, const CSRView& A, const int* wcell, const double* par,
                            const double* k, double nu, double* nz, double* b) {
    if (nw <= 0) return;
    k_omega_constrain<<<nblk(nw), TPB, 0, s>>>(nw, A, wcell, par, k, nu, nz, b);
    XCAL_CHECK_LAUNCH();
}
void launch_bound(cudaStream_t s, const MeshView& m, const double* old, double* v) {
    k_bound<<<nblk(m.nC), TPB, 0, s>>>(m, old, v);
    XCAL_CHECK_LAUNCH();
}
// LES{KEquation} cell sources (LES_KEquation.jl:164-168), rho = 1:
//   Pk = 2 nut (grad U . dev(S)), the Frobenius product over the tensor's
//        column-major entries in order, S = (G + G')/2, dev(S) = S - tr(S)/3 I
//   Dk = ce sqrt(k) / Delta      (Si on k)
//   Dw = 2/3 tr(grad U)          (a second Si on k)
// G[a][b] = g[3 a + b] is entry (a, b) of the tensor the reference builds.
__global__ void k_keq_sources(int nC, const double* __restrict__ g0, const double* __restrict__ g1,
                              const double* __restrict__ g2, const double* __restrict__ g3,
                              const double* __restrict__ g4, const double* __restrict__ g5,
                              const double* __restrict__ g6, const double* __restrict__ g7,
                              const double* __restrict__ g8, const double* __restrict__ nut,
                              const double* __restrict__ k, const double* __restrict__ Delta, double ce, double* Pk,
                              double* Dk, double* Dw) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nC) return;
    const double G[3][3] = {{g0[i], g1[i], g2[i]}, {g3[i], g4[i], g5[i]}, {g6[i], g7[i], g8[i]}};
    double S[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) S[a][b] = 0.5 * (G[a][b] + G[b][a]);
    const double trS = (S[0][0] + S[1][1]) + S[2][2];
    const double third = (1.0 / 3.0) * trS;
    double dot = 0.0;
    bool first = true;
    for (int b = 0; b < 3; ++b)
        for (int a = 0; a < 3; ++a) {
            const double dev = a == b ? S[a][b] - third : S[a][b];
            const double pr = G[a][b] * dev;
            dot = first ? pr : dot + pr;
            first = false;
        }
    Pk[i] = (2.0 * nut[i]) * dot;
    Dk[i] = (ce * sqrt(k[i])) / Delta[i];
    Dw[i] = (2.0 / 3.0) * ((G[0][0] + G[1][1]) + G[2][2]);
}

// nut = ck Delta sqrt(k) (LES_KEquation.jl:180-183)
__global__ void k_keq_nut(int nC, const double* __restrict__ k, const double* __restrict__ Delta, double ck,
                          double* nut) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nC) nut[i] = (ck * Delta[i]) * sqrt(k[i]);
}

// ---- RANS{KOmegaLKE} (RANS_kOmegaLKE.jl) ---------------------------------
// the model's constants (:83-98)
constexpr double LKE_CMU = 0.09, LKE_CW1 = 0.52, LKE_CW2 = 0.0708, LKE_CCRIT = 76500.0, LKE_CSS = 1.45,
                 LKE_CV = 0.43, LKE_SK = 0.5, LKE_SD = 0.125, LKE_SKL = 0.0125, LKE_SW = 0.5;

// Re_upsilon = sqrt(sqrt(2 nu^2 kl / y^2)) y / nu and its power -1.30 (:321, :447)
__device__ __forceinline__ double lke_reu_pow(double nu, double kl, double y) {
    const double ru = (sqrt(sqrt(((2.0 * (nu * nu)) * kl) / (y * y))) * y) / nu;
    return det_pow(ru, -1.30);
}

// the first two cell loops of turbulence! (:284-335), after grad U: div U,
// S2 = 2 |dev(S)|^2, Omega = sqrt(2) |skew(grad U)|, Pk = sum((2 grad U)
// dev(S)) (the code's `g .* 2*S_dev` is a matrix product: .* and * share a
// precedence level and associate left), |U|, Re_lambda; then gamma, the kl
// equation's source and Si coefficient and its cell diffusivity.  Sums over
// the 3x3 entries run in column-major order from the first entry; the
// product's entries are ((a1 b1 + a2 b2) + a3 b3)
__global__ void k_lke_fields(LkeView V) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V.nC) return;
    double G[3][3];
    for (int q = 0; q < 9; ++q) G[q / 3][q % 3] = V.g[q][i];
    const double divU = (G[0][0] + G[1][1]) + G[2][2];
    const double d3 = divU / 3.0;
    double Sd[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            const double sy = 0.5 * (G[a][b] + G[b][a]);
            Sd[a][b] = a == b ? sy - d3 : sy;
        }
    double s2 = 0.0, om = 0.0, pk = 0.0;
    for (int b = 0; b < 3; ++b)
        for (int a = 0; a < 3; ++a) {
            const double sq = Sd[a][b] * Sd[a][b];
            const double w = 0.5 * (G[a][b] - G[b][a]);
            const double m = (((G[a][0] * 2.0) * Sd[0][b]) + ((G[a][1] * 2.0) * Sd[1][b])) + ((G[a][2] * 2.0) * Sd[2][b]);
            const bool first = a == 0 && b == 0;
            s2 = first ? sq : s2 + sq;
            om = first ? w * w : om + w * w;
            pk = first ? m : pk + m;
        }
    const double S2 = 2.0 * s2, Om = sqrt(2.0 * om);
    const double u0 = V.U[0][i], u1 = V.U[1][i], u2 = V.U[2][i];
    const double normU = sqrt((u0 * u0 + u1 * u1) + u2 * u2);
    const double nu = V.nu, y = V.y[i], kl = V.kl[i];
    const double ReL = (jl_max(normU, 1.4901161193847656e-08) * y) / nu;  // sqrt(eps())
    V.divU[i] = divU;
    V.S2[i] = S2;
    V.Om[i] = Om;
    V.Pk[i] = pk;
    V.normU[i] = normU;
    V.ReL[i] = ReL;
    // :312-335
    const double pru = lke_reu_pow(nu, kl, y), prl = sqrt(ReL), sS2 = sqrt(S2);
    const double uy = normU / y;
    const double nutL1 = ((((V.eta * kl) * sS2) * pru) * prl) / jl_max(S2, uy * uy);
    const double ReLt = jl_min((kl / jl_max(jl_min(nu, nutL1), 1e-15)) / jl_max(Om, 1e-15), 5000.0);
    V.gam[i] = jl_min(ReLt * ReLt, LKE_CCRIT) / LKE_CCRIT;
    V.PkL[i] = (((sS2 * V.eta) * kl) * pru) * prl;
    V.DkL[i] = (2.0 * nu) / (y * y);
    V.nueffS[i] = nu + ((LKE_SKL * sqrt(kl)) * y);
}

// the omega equation's cell loop (:377-387): production from the loop's Pk,
// Cw2 omega, the diffusivity nu + sigma_w k / omega, the cross diffusion
// max(sigma_d / omega^2 grad k . grad omega, 0)
__global__ void k_lke_omega(LkeView V) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V.nC) return;
    const double w = V.omega[i], sw = jl_max(w, 1e-15);
    double pw = LKE_CW1 * V.Pk[i];
    pw = pw - ((((2.0 / 3.0) * LKE_CW1) * V.divU[i]) * w);
    V.Pw[i] = pw;
    V.Dw[i] = LKE_CW2 * w;
    V.nueffS[i] = V.nu + LKE_SW * (V.k[i] / sw);
    const double dkdw = (V.gk[0][i] * V.gw[0][i] + V.gk[1][i] * V.gw[1][i]) + V.gk[2][i] * V.gw[2][i];
    V.D2[i] = jl_max((LKE_SD / (sw * sw)) * dkdw, 0.0);
}

// the k equation's cell loop (:401-420), after the omega solve: fv, the
// limited production Pk, Cmu gamma omega, the diffusivity nu + sigma_k k / omega
__global__ void k_lke_k(LkeView V) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V.nC) return;
    const double w = V.omega[i], gam = V.gam[i], kk = V.k[i];
    const double sw = jl_max(w, 1e-15), sk = jl_max(kk, 1e-15), snu = jl_max(V.nu, 1e-15);
    const double fv = 1.0 - det_exp_neg((-sqrt(sk / (snu * sw))) / LKE_CV);
    const double pku = ((fv * (sk / sw)) * V.Pk[i]) * gam;
    const double pkl = jl_min(pku, ((20.0 * LKE_CMU) * sk) * w);
    V.Pk[i] = pkl - (((2.0 / 3.0) * V.divU[i]) * kk);
    V.Dk[i] = (LKE_CMU * gam) * w;
    V.nueffS[i] = V.nu + LKE_SK * (sk / sw);
}

// nut = fSS k / omega + nuL from the solved kl, k, omega (:435-460)
__global__ void k_lke_nut(LkeView V) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V.nC) return;
    const double kl = V.kl[i], nu = V.nu, y = V.y[i], S2 = V.S2[i], normU = V.normU[i];
    const double sw = jl_max(V.omega[i], 1e-15), sk = jl_max(V.k[i], 1e-15);
    const double PkL = (((sqrt(S2) * V.eta) * kl) * lke_reu_pow(nu, kl, y)) * sqrt(V.ReL[i]);
    const double uy = normU / y;
    const double nuL = PkL / jl_max(S2, uy * uy);
    const double x = ((LKE_CSS * nu) * V.Om[i]) / sk;
    const double fSS = det_exp_neg(-(x * x));
    V.nut[i] = fSS * (sk / sw) + nuL;
}

void launch_lke_fields(cudaStream_t s, const LkeView& V) {
    k_lke_fields<<<nblk(V.nC), TPB, 0, s>>>(V);
    XCAL_CHECK_LAUNCH();
}
void launch_lke_omega(cudaStream_t s, const LkeView& V) {
    k_lke_omega<<<nblk(V.nC), TPB, 0, s>>>(V);
    XCAL_CHECK_LAUNCH();
}
void launch_lke_k(cudaStream_t s, const LkeView& V) {
    k_lke_k<<<nblk(V.nC), TPB, 0, s>>>(V);
    XCAL_CHECK_LAUNCH();
}
void launch_lke_nut(cudaStream_t s, const LkeView& V) {
    k_lke_nut<<<nblk(V.nC), TPB, 0, s>>>(V);
    XCAL_CHECK_LAUNCH();
}

void launch_keq_sources(cudaStream_t s, int nC, const double* const g[9], const double* nut, const double* k,
                        const double* Delta, double ce, double* Pk, double* Dk, double* Dw) {
    k_keq_sources<<<nblk(nC), TPB, 0, s>>>(nC, g[0], g[1], g[2], g[3], g[4], g[5], g[6], g[7], g[8], nut, k, Delta, ce,
                                           Pk, Dk, Dw);
    XCAL_CHECK_LAUNCH();
}
void launch_keq_nut(cudaStream_t s, int nC, const double* k, const double* Delta, double ck, double* nut) {
    k_keq_nut<<<nblk(nC), TPB, 0, s>>>(nC, k, Delta, ck, nut);
    XCAL_CHECK_LAUNCH();
}
void launch_kw_nut(cudaStream_t s, int nC, const double* k, const double* omega, double* nut) {
    k_kw_nut<<<nblk(nC), TPB, 0, s>>>(nC, k, omega, nut);
    XCAL_CHECK_LAUNCH();
}
void launch_nueff(cudaStream_t s, int nF, const double* nutf, double* nueff, double nu) {
    k_nueff<<<nblk(nF), TPB, 0, s>>>(nF, nutf, nueff, nu);
    XCAL_CHECK_LAUNCH();
}
void launch_smag_nut(cudaStream_t s, int nC, const double* const g[9], const double* Delta, double* nut) {
    k_smag_nut<<<nblk(nC), TPB, 0, s>>>(nC, g[0], g[1], g[2], g[3], g[4], g[5], g[6], g[7], g[8], Delta, nut);
    XCAL_CHECK_LAUNCH();
}
void launch_nonorth_correct(cudaStream_t s, const MeshView& m, const double* t, const double* p,
                            const double* const g[3], const double* rDf, double* b) {
    k_nonorth_correct<<<nblk(m.nC), TPB, 0, s>>>(m, t, p, g[0], g[1], g[2], rDf, b);
    XCAL_CHECK_LAUNCH();
}
void launch_div(cudaStream_t s, const MeshView& m, const double* psif, double* out) {
    k_div<<<nblk(m.nC), TPB, 0, s>>>(m, psif, out);
    XCAL_CHECK_LAUNCH();
}
void launch_rD_remove_H(cudaStream_t s, const MeshView& m, const CSRView& A, const double* nz,
                        const double* const U[3], const double* const g[3], double* const b[3], double* rD,
                        double* const H[3], int do_H) {
    k_rD_remove_H<<<nblk(m.nC), TPB, 0, s>>>(m, A, nz, U[0], U[1], U[2], g[0], g[1], g[2], b[0], b[1], b[2], rD,
                                             H[0], H[1], H[2], do_H);
    XCAL_CHECK_LAUNCH();
}
void launch_H(cudaStream_t s, const MeshView& m, const CSRView& A, const double* nz, const double* const U[3],
              const double* const b[3], double* const H[3]) {
    k_H<<<nblk(m.nC), TPB, 0, s>>>(m, A, nz, U[0], U[1], U[2], b[0], b[1], b[2], H[0], H[1], H[2]);
    XCAL_CHECK_LAUNCH();
}
void launch_correct_mdot(cudaStream_t s, const MeshView& m, const CSRView& A, const BCView& bcp, const double* nz,
                         const double* p, const double* rDf, double* mdot) {
    k_correct_mdot<<<nblk(m.nF), TPB, 0, s>>>(m, A, bcp, nz, p, rDf, mdot);
    XCAL_CHECK_LAUNCH();
}
void launch_correct_U(cudaStream_t s, int n, double* const H[3], const double* const g[3], const double* rD,
                      double* const U[3]) {
    k_correct_U<<<nblk(n), TPB, 0, s>>>(n, H[0], H[1], H[2], g[0], g[1], g[2], rD, U[0], U[1], U[2]);
    XCAL_CHECK_LAUNCH();
}
void launch_relax_explicit(cudaStream_t s, int n, double* phi, const double* phi0, double alpha) {
    k_relax_explicit<<<nblk(n), TPB, 0, s>>>(n, phi, phi0, alpha);
    XCAL_CHECK_LAUNCH();
}
// dst[i] = src[idx[i]]: the storage <-> original permutation of a field
__global__ void k_gather(long n, const double* __restrict__ src, const int* __restrict__ idx, double* dst) {
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[idx[i]];
}
void launch_gather(cudaStream_t s, long n, const double* src, const int* idx, double* dst) {
    if (n <= 0) return;
    k_gather<<<nblk(n), TPB, 0, s>>>(n, src, idx, dst);
    XCAL_CHECK_LAUNCH();
}

void launch_courant_max(cudaStream_t s, int n, const double* const U[3], const double* dx, double dt, double* part,
                        unsigned int* counter, double* out) {
    k_courant_max<<<(n + RED_TILE - 1) / RED_TILE, RED_THREADS, 0, s>>>(n, U[0], U[1], U[2], dx, dt, part, counter,
                                                                        out);
    XCAL_CHECK_LAUNCH();
}

}  // namespace xcal

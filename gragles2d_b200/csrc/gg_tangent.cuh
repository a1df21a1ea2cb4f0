// Tangent-linear (forward-mode) derivative of the plain FP64 step with
// respect to the four calibration parameters
//   p0 = theta_ref (Read-Shockley cut-off angle, radians),
//   p1 = gamma_HAGB (high-angle boundary energy),
//   p2 = m_HAGB (high-angle boundary mobility),
//   p3 = Lambda (triple-junction drag, TriplePointDrag).
// Four tangent fields d phi / d p_k ride along the distance field through
// every stage with the step's discrete decisions held fixed: the comparison's
// winners, the contour's edges, the redistancing sweeps' accepted candidates,
// the corrector's sectors and pixel projections.  With four parameters and
// scalar losses this carries the same information as a reverse adjoint of
// the same linearised stages, without a tape.
//
// Stage by stage (reference routines in brackets):
//  - convolution (src/box.cpp:622-695): linear, d psi = K d phi (k_conv_dft, tk >= 0);
//  - corrector (src/box.cpp:428-510): psi' = phi + (psi - phi) w(p), so
//    d psi' = (1 - w) d phi + w d psi + (psi - phi) dw/dp, with dw/dp from the
//    Read-Shockley / mobility-model / junction-drag formulas in dual numbers;
//  - comparison (src/box.cpp:838-1025): the winner's d psi' routed through
//    the maximum, then the set-comparison blend;
//  - contour area (src/grainBoundary.cpp:201-213): each contour point moves
//    with the zero crossing of its grid edge;
//  - redistancing (src/box.cpp:1259-1399): every output carries the
//    derivative of the zero-crossing value it was propagated from.
#pragma once

#include "gg_corrector.cuh"
#include "gg_kernels.cuh"

namespace gg {
namespace {

constexpr int kNP = 4;  // tangent parameters

struct D4 {
    double v;
    double d[kNP];
};

__device__ __forceinline__ D4 dconst(double v) {
    D4 r;
    r.v = v;
    for (int k = 0; k < kNP; ++k) r.d[k] = 0.0;
    return r;
}
__device__ __forceinline__ D4 dadd(const D4& a, const D4& b) {
    D4 r;
    r.v = a.v + b.v;
    for (int k = 0; k < kNP; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
__device__ __forceinline__ D4 dsub(const D4& a, const D4& b) {
    D4 r;
    r.v = a.v - b.v;
    for (int k = 0; k < kNP; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
__device__ __forceinline__ D4 dmul(const D4& a, const D4& b) {
    D4 r;
    r.v = a.v * b.v;
    for (int k = 0; k < kNP; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
__device__ __forceinline__ D4 dscale(const D4& a, double s) {
    D4 r;
    r.v = a.v * s;
    for (int k = 0; k < kNP; ++k) r.d[k] = a.d[k] * s;
    return r;
}
__device__ __forceinline__ D4 drecip(const D4& a) {
    D4 r;
    r.v = 1 / a.v;
    const double q = -1 / (a.v * a.v);
    for (int k = 0; k < kNP; ++k) r.d[k] = a.d[k] * q;
    return r;
}

// read_shockley (LSbox::GBEnergyReadShockley, src/box.cpp:1785-1823) with its
// derivatives in theta_ref (p0) and gamma_HAGB (p1); same value arithmetic.
__device__ D4 read_shockley_d(double theta, const NetConst& C) {
    if (C.isotropic) return dconst(1.0);
    const double gamma_hagb = C.gamma_hagb, theta_ref = C.theta_ref;
    D4 r = dconst(0.0);
    if (theta > theta_ref) {
        r.v = gamma_hagb;
        r.d[1] = 1.0;
        return r;
    }
    if (theta < 1.0 * kPi / 180.0) theta = 1.0 * kPi / 180.0;
    const double x = theta / theta_ref, lx = log(theta / theta_ref);
    r.v = gamma_hagb * (theta / theta_ref) * (1.0 - log(theta / theta_ref));
    if (r.v != r.v) return dconst(0.01);
    r.d[0] = gamma_hagb * x * lx / theta_ref;  // d/dtheta_ref of gamma x (1 - ln x), x = theta / theta_ref
    r.d[1] = x * (1.0 - lx);
    return r;
}

// mobility_model (LSbox::GBmobilityModel, src/box.cpp:1825-1865, model 1)
// with its derivatives in theta_ref (p0) and m_HAGB (p2).
__device__ D4 mobility_model_d(double theta, const NetConst& C) {
    if (C.use_mobility_model == 0 || C.isotropic) return dconst(1.0);
    const double u = pow(theta / C.theta_ref, 9.0), e = exp(-5.0 * u);
    const double m = 1 - (0.99 * exp(-5.0 * (pow(theta / C.theta_ref, 9.0))));
    D4 r = dconst(C.m_hagb * m);
    r.d[0] = -44.55 * C.m_hagb * u * e / C.theta_ref;  // d/dtheta_ref: 0.99 * 5 * 9 = 44.55
    r.d[2] = m;
    return r;
}

// getGBEnergyTimesGBMobility floor (src/box.cpp:554-561)
__device__ __forceinline__ D4 gb_floor_d(const D4& e, const D4& m) {
    const D4 w = dmul(e, m);
    return w.v > 0.01 ? w : dconst(0.01);
}

// Characteristic of id in owner's direct-neighbour list as (energy, mobility)
// duals from its stored misorientation; absent or removed: (1, 1) constant.
__device__ bool characteristic_d(const NetConst& C, int owner, int id, D4* e, D4* m) {
    const Neighbour* c = find_characteristic(C, owner, id);
    if (!c) {
        *e = dconst(1.0);
        *m = dconst(1.0);
        return false;
    }
    *e = read_shockley_d(c->misori, C);
    *m = mobility_model_d(c->misori, C);
    return true;
}

// GrainJunction::getWeight (src/junction.cpp:23-192) in dual numbers, one thread.
__device__ D4 junction_weight_d(const NetConst& C, const Junction& J, int me) {
    uint32_t nbr[4] = {0xFFFFFFu, 0xFFFFFFu, 0xFFFFFFu, 0xFFFFFFu};
    for (int i = 0, j = 0; i < J.type && i < 4; i++)
        if ((uint32_t)me != J.grains[i]) nbr[j++] = J.grains[i];
    if (nbr[0] == 0xFFFFFFu || nbr[1] == 0xFFFFFFu) return dconst(1.0);
    const int n0 = (int)nbr[0], n1 = (int)nbr[1];
    if (n0 > C.N || n1 > C.N) return dconst(1.0);
    const double* qm = C.quat + 4 * (int64_t)me;
    const double* q0 = C.quat + 4 * (int64_t)n0;
    const double* q1 = C.quat + 4 * (int64_t)n1;
    const double t0 = grain_misorientation(qm, q0), t1 = grain_misorientation(q0, q1),
                 t2 = grain_misorientation(qm, q1);
    D4 e01, m01;
    characteristic_d(C, n0, n1, &e01, &m01);
    D4 avg = dconst(0.0);
    avg = dadd(avg, mobility_model_d(t0, C));
    avg = dadd(avg, m01);
    avg = dadd(avg, mobility_model_d(t2, C));
    D4 sigma = dadd(dsub(read_shockley_d(t0, C), read_shockley_d(t1, C)), read_shockley_d(t2, C));
    if (!C.isotropic && C.use_mobility_model > 0 && C.tpd > 0) {
        avg = dscale(avg, 1.0 / 3);
        D4 lam = dconst(C.tpd);
        lam.d[3] = 1.0;
        const D4 a = drecip(dscale(lam, C.ds));  // 1 / (ds Lambda)
        const D4 drag = drecip(dadd(a, drecip(avg)));
        sigma = dmul(sigma, drag);
    }
    if (sigma.v < 0.01) return dconst(0.01);
    return sigma;
}

// Dual weights of a grain's sectors and neighbour table.
struct SectorDuals {
    D4 cs[kMaxConstSectors];
    D4 lw[kMaxInterpSectors], rw[kMaxInterpSectors], bw[kMaxInterpSectors];
    D4 nb[48];
    int nb_id[48];
    int nb_n;
};

__device__ __forceinline__ D4 table_weight_d(const SectorDuals& T, const uint32_t* idl, const Box& ib, int row,
                                             int col) {
    uint32_t k;
    if (!buf_index(ib, row, col, &k)) return dconst(1.0);
    const int id = (int)idl[k];
    for (int e = 0; e < T.nb_n; ++e)
        if (T.nb_id[e] == id) return T.nb[e];
    return dconst(1.0);
}

// Tangent of the anisotropic corrector, run before the value corrector (it
// reads the unmodified convolution): per pixel of IDLocal box x current box
// with phi > -delta, d psi' = (1 - w) d phi + w d psi + (psi - phi) dw;
// below, psi' = -delta is constant.  The sectors are rebuilt exactly as the
// value corrector builds them.
__global__ void __launch_bounds__(128) k_corrector_t(NetConst C, NetState* S) {
    const int g = blockIdx.x + 1;
    if (g > C.N || C.state[g] != G_EXISTS || C.regular[g] == 0 || S->loop == 0 || halted(S)) return;
    __shared__ SectorSet sec;
    __shared__ double jw[64];
    __shared__ uint32_t s_st;
    __shared__ double s_per;
    __shared__ NbTable nbt;
    __shared__ double s_seg[kSegShared];
    __shared__ int jl[64], jr[64];
    __shared__ SectorDuals sd;
    __shared__ D4 jwd[64];
    __shared__ double s_dlen[kMaxInterpSectors][kNP];
    const CPoint* P = S->contPrev + S->coff_prev[g];
    const int size = S->cn_prev[g];
    if (size < 2) return;
    double* seg = size - 1 <= kSegShared ? s_seg : S->segPrev + S->coff_prev[g];
    const Box ib = S->box_prev[g];
    const uint32_t* idl = S->idPrev + S->off_prev[g];
    prepare_sectors(C, S, g, P, size, seg, sec, jw, &s_st, &s_per, nbt, jl, jr);
    // dual weights: junctions, neighbour table, constant and interpolating sectors
    const Junction* J = S->jPrev + (int64_t)g * C.jmax;
    const int nj = min(S->jn_prev[g], 64);
    for (int q = threadIdx.x; q < nj; q += blockDim.x) jwd[q] = junction_weight_d(C, J[q], g);
    {
        const Neighbour* nb = C.nb + (int64_t)g * C.nbmax;
        const int n = min(C.nb_n[g], 48);
        if (threadIdx.x == 0) sd.nb_n = n;
        for (int e = threadIdx.x; e < n; e += blockDim.x) {
            const int id = nb[e].id;
            const bool gone = id < 0 || id > C.N || (id != 0 && C.state[id] == G_GONE);
            sd.nb_id[e] = gone ? -2 : id;
            sd.nb[e] = gb_floor_d(read_shockley_d(nb[e].misori, C), mobility_model_d(nb[e].misori, C));
        }
    }
    __syncthreads();
    for (int s = threadIdx.x; s < sec.nconst; s += blockDim.x) {
        D4 w = dconst(0.0);
        for (int q = 0; q < sec.cs[s].nj; ++q) w = dadd(w, jwd[sec.cs[s].js[q] < 64 ? sec.cs[s].js[q] : 63]);
        sd.cs[s] = dscale(w, 1.0 / (double)sec.cs[s].nj);
    }
    __syncthreads();
    const int real = size - 1;
    for (int s = threadIdx.x; s < sec.ninterp; s += blockDim.x) {
        const InterpSector& q = sec.is[s];
        sd.lw[s] = q.lb >= 0 ? sd.cs[q.lb] : table_weight_d(sd, idl, ib, (int)P[q.left].y, (int)P[q.left].x);
        sd.rw[s] = q.rb >= 0 ? sd.cs[q.rb] : table_weight_d(sd, idl, ib, (int)P[q.right].y, (int)P[q.right].x);
        sd.bw[s] = dconst(0.0);
        if (q.lb >= 0 && q.rb >= 0) {
            const CPoint& smp = P[(q.right + 1) % real];
            sd.bw[s] = table_weight_d(sd, idl, ib, (int)smp.y, (int)smp.x);
        }
    }
    // the previous contour moves with the parameters too: segment-length
    // tangents, then each interpolating sector's length tangent over the
    // segments its length summed
    const double* dP = S->dcontPrev + 8 * S->coff_prev[g];
    double* dsg = C.dseg + 4 * S->coff_prev[g];
    for (int k = threadIdx.x; k < real; k += blockDim.x) {
        const double ex = P[k + 1].x - P[k].x, ey = P[k + 1].y - P[k].y;
        const double len = sqrt(ex * ex + ey * ey);
        for (int t = 0; t < kNP; ++t) {
            const double ddx = dP[8 * (k + 1) + t] - dP[8 * k + t];
            const double ddy = dP[8 * (k + 1) + 4 + t] - dP[8 * k + 4 + t];
            dsg[4 * k + t] = len > 0 ? C.h * (ex * ddx + ey * ddy) / len : 0.0;
        }
    }
    __syncthreads();
    for (int q = threadIdx.x; q < sec.ninterp; q += blockDim.x) {
        double dl[kNP] = {0, 0, 0, 0};
        const InterpSector& is = sec.is[q];
        if (is.len0 >= 0) {
            int it = 0;
            for (int k = is.len0;; k = wrap_next(k, real)) {
                for (int t = 0; t < kNP; ++t) dl[t] += dsg[4 * k + t];
                if (k == is.len1 || ++it > size) break;
            }
        }
        for (int t = 0; t < kNP; ++t) s_dlen[q][t] = dl[t];
    }
    __syncthreads();
    const Box bo = S->box_cur[g];
    const int x0 = ib.x0 < bo.x0 ? bo.x0 : ib.x0;
    const int y0 = ib.y0 < bo.y0 ? bo.y0 : ib.y0;
    const int x1 = ib.x1 > bo.x1 ? bo.x1 : ib.x1;
    const int y1 = ib.y1 > bo.y1 ? bo.y1 : ib.y1;
    if (x1 <= x0 || y1 <= y0) return;
    const int w = x1 - x0;
    const int64_t cnt = (int64_t)w * (y1 - y0);
    const double* phi = phiA_of<double>(S) + S->off_cur[g];
    const double* psi = phiB_of<double>(S) + S->off_cur[g];
    const double* dphi = reinterpret_cast<const double*>(S->dphiA) + S->off_cur[g];
    double* dpsi = reinterpret_cast<double*>(S->dphiB) + S->off_cur[g];
    const int64_t cap = S->phi_cap;
    const int wo = box_w(bo);
    const double delta = C.delta;
    for (int64_t p = threadIdx.x; p < cnt; p += blockDim.x) {
        const int i = y0 + (int)(p / w), j = x0 + (int)(p % w);
        const int64_t k = (int64_t)(i - bo.y0) * wo + (j - bo.x0);
        const double val = phi[k];
        if (!(val > -delta)) {
            for (int t = 0; t < kNP; ++t) dpsi[t * cap + k] = 0.0;
            continue;
        }
        // the value corrector's pixel weight, as a dual
        double lambda = 0.0;
        const int segment = project_to_boundary(P, size, (double)j, (double)i, &lambda);
        int sid = -1;
        double interpolator = 0;
        for (int q = 0; q < sec.nconst && sid == -1; q++)
            if (within(sec.cs[q].left, sec.cs[q].right, real, segment)) sid = q;
        for (int q = 0; q < sec.ninterp && sid == -1; q++)
            if (within(sec.is[q].left, sec.is[q].right, real, segment)) sid = -2 - q;
        D4 wd;
        if (sid >= 0) {
            wd = sd.cs[sid];
        } else if (sid == -1) {
            wd = table_weight_d(sd, idl, ib, i, j);
        } else {
            const InterpSector& s = sec.is[-2 - sid];
            double dacc[kNP] = {0, 0, 0, 0};
            int it = 0;
            for (int kk = s.right; kk != segment; kk = wrap_next(kk, real)) {
                interpolator += seg[kk];
                for (int t = 0; t < kNP; ++t) dacc[t] += dsg[4 * kk + t];
                if (++it > size) break;
            }
            const int kn = wrap_next(segment, real);
            const double ux = P[kn].x - P[segment].x, uy = P[kn].y - P[segment].y;
            const double ax = ux * lambda, ay = uy * lambda;
            const double partial = sqrt(ax * ax + ay * ay);
            interpolator += partial;
            const double iraw = interpolator / s.length;
            interpolator /= s.length;
            if (interpolator < 0) interpolator = 0;
            if (interpolator > 1) interpolator = 1;
            // tangent of the interpolator through the moving contour: the
            // partial segment |u| lambda (lambda the pixel's projection onto
            // segment (a, a + u)), the summed segments and the sector length
            double dI[kNP] = {0, 0, 0, 0};
            const double uu = ux * ux + uy * uy, ul = sqrt(uu);
            if (iraw > 0 && iraw < 1 && uu > 0) {
                const double px = (double)j - P[segment].x, py = (double)i - P[segment].y;
                const double lraw = (px * ux + py * uy) / uu;
                for (int t = 0; t < kNP; ++t) {
                    const double dax = dP[8 * segment + t], day = dP[8 * segment + 4 + t];
                    const double dux = dP[8 * kn + t] - dax, duy = dP[8 * kn + 4 + t] - day;
                    const double udu = ux * dux + uy * duy;
                    double dl = 0;
                    if (lraw > 0 && lraw < 1) dl = (-(dax * ux + day * uy) + (px * dux + py * duy)) / uu - lraw * 2 * udu / uu;
                    const double dpart = lambda * udu / ul + ul * dl;
                    dI[t] = (dacc[t] + dpart) / s.length - iraw * s_dlen[-2 - sid][t] / s.length;
                }
            }
            const D4 lw = sd.lw[-2 - sid], rw = sd.rw[-2 - sid];
            const double I = interpolator;
            if (s.lb >= 0 && s.rb >= 0) {
                const double isr = C.isr;
                const double quot = (s.length > 2 * isr ? 2 * isr : s.length);
                const D4 mid = dscale(dadd(lw, rw), 0.5);
                const D4 amplitude = dadd(dscale(dsub(sd.bw[-2 - sid], mid), quot / (2 * isr)), mid);
                const D4 a0 = dscale(rw, 2), a1 = dscale(amplitude, -4), a2 = dscale(lw, 2);
                const D4 A = dadd(dadd(a0, a1), a2);
                const D4 B = dscale(dadd(dadd(dscale(a0, 1.5), a1), dscale(a2, 0.5)), -1);
                const D4 Cc = dscale(a0, 0.5);
                wd = dadd(dadd(dscale(A, I * I), dscale(B, I)), Cc);
                const double dw_dI = 2 * A.v * I + B.v;
                const double dw_dquot = (-4 * I * I + 4 * I) * (sd.bw[-2 - sid].v - mid.v) / (2 * isr);
                for (int t = 0; t < kNP; ++t)
                    wd.d[t] += dw_dI * dI[t] + (s.length > 2 * isr ? 0.0 : dw_dquot * s_dlen[-2 - sid][t]);
            } else {
                wd = dadd(dscale(lw, I), dscale(rw, 1 - I));
                for (int t = 0; t < kNP; ++t) wd.d[t] += (lw.v - rw.v) * dI[t];
            }
        }
        const double diff = psi[k] - val;
        for (int t = 0; t < kNP; ++t)
            dpsi[t * cap + k] = (1 - wd.v) * dphi[t * cap + k] + wd.v * dpsi[t * cap + k] + diff * wd.d[t];
    }
}

// Tangent of the comparison and set comparison: the winner of each pixel's
// maximum (list members in order, strict '>', then the wall) is found again
// on the corrected fields and its tangent routed through; inside the 0.7
// delta tube d chi = (d psi'_own - d out) / 2, elsewhere d psi'_own.  Reads
// arena B (psi', d psi'), writes d chi into tangent arena A.
__global__ void __launch_bounds__(256) k_compare_t(NetConst C, NetState* S) {
    const int g = blockIdx.x + 1;
    if (g > C.N || C.state[g] != G_EXISTS || halted(S)) return;
    const int K = C.kmax;
    const int nl = C.cmp_n[g] < kListMaxSmem ? C.cmp_n[g] : kListMaxSmem;
    const int* ids = C.cmp_ids + (int64_t)g * K;
    const Box bc = S->box_cur[g];
    const int w = box_w(bc);
    const int64_t area = box_area(bc);
    const int b = C.b, m = C.m;
    const int lo = b + b, hi = m - b - b;
    const bool bnd = !(bc.x0 > lo && bc.x1 < hi && bc.y0 > lo && bc.y1 < hi);
    const double* conv = phiB_of<double>(S);
    const double* dconv = reinterpret_cast<const double*>(S->dphiB);
    double* dchi = reinterpret_cast<double*>(S->dphiA) + S->off_cur[g];
    const int64_t cap = S->phi_cap;
    const int64_t self = S->off_cur[g];
    const double tube = 0.7 * C.delta;
    for (int64_t p = threadIdx.x; p < area; p += blockDim.x) {
        const int i = bc.y0 + (int)(p / w);
        const int j = bc.x0 + (int)(p - (int64_t)(i - bc.y0) * w);
        double out = -1.0;
        int64_t win = -1;  // arena index of the winning neighbour's pixel
        for (int q = 0; q < nl; ++q) {
            const int id = ids[q];
            const Box bk = S->box_cur[id];
            if (i >= bk.y0 && i < bk.y1 && j >= bk.x0 && j < bk.x1) {
                const int64_t idx = S->off_cur[id] + (int64_t)(i - bk.y0) * (bk.x1 - bk.x0) + (j - bk.x0);
                const double d = conv[idx];
                if (d > out) {
                    out = d;
                    win = idx;
                }
            }
        }
        if (bnd) {
            const int dxmin = -(j - b), dymin = -(i - b);
            const int dxmax = (j - (m - b)), dymax = (i - (m - b));
            const int dx = (abs(dxmin) < abs(dxmax)) ? dxmin : dxmax;
            const int dy = (abs(dymin) < abs(dymax)) ? dymin : dymax;
            double dist = 0;
            if (dx > 0 && dy > 0)
                dist = sqrt((double)dx * dx + dy * dy);
            else if (dx < 0 && dy > 0)
                dist = dy;
            else if (dx > 0 && dy < 0)
                dist = dx;
            else if (dx < 0 && dy < 0)
                dist = dx > dy ? dx : dy;
            else if (dx == 0)
                dist = dy > 0 ? dy : 0;
            else
                dist = dx > 0 ? dx : 0;
            if (dist * C.h > out) win = -1;  // the wall is constant
        }
        const double in = conv[self + p];
        const bool blend = fabs(in) < tube;
        for (int t = 0; t < kNP; ++t) {
            const double dout = win >= 0 ? dconv[t * cap + win] : 0.0;
            const double din = dconv[t * cap + self + p];
            dchi[t * cap + p] = blend ? 0.5 * (din - dout) : din;
        }
    }
}

// d area / d p_k of the contour just extracted (LSbox::computeVolume,
// src/grainBoundary.cpp:201-213): a point on a vertical grid edge (integer x)
// moves in y with the zero crossing between rows floor(y) and floor(y) + 1,
// a point on a horizontal edge in x; points on a grid node (both integer, as
// the box-border cases of generatePoint) are fixed.  The point tangents are
// kept for the next step's corrector.  One thread per grain.
__global__ void k_area_t(NetConst C, NetState* S) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (g > C.N) return;
    double* out = C.dvol + kNP * (int64_t)g;
    for (int t = 0; t < kNP; ++t) out[t] = 0.0;
    if (C.state[g] != G_EXISTS || halted(S)) return;
    const int n = S->cn_cur[g];
    if (n < 2) return;
    const CPoint* P = S->contCur + S->coff_cur[g];
    const Box bc = S->box_cur[g];
    const int w = box_w(bc);
    const double* chi = phiA_of<double>(S) + S->off_cur[g];
    const double* dchi = reinterpret_cast<const double*>(S->dphiA) + S->off_cur[g];
    const int64_t cap = S->phi_cap;
    auto inside = [&](int r, int c) { return r >= bc.y0 && r < bc.y1 && c >= bc.x0 && c < bc.x1; };
    auto at = [&](int r, int c) { return (int64_t)(r - bc.y0) * w + (c - bc.x0); };
    // d(x_i), d(y_i) of point i for parameter t
    auto dpoint = [&](int i, int t, double* dx, double* dy) {
        *dx = 0.0;
        *dy = 0.0;
        const double x = P[i].x, y = P[i].y;
        const double fx = floor(x), fy = floor(y);
        int r0, c0, r1, c1;
        bool vertical;
        if (x == fx && y != fy) {
            vertical = true;
            c0 = c1 = (int)fx;
            r0 = (int)fy;
            r1 = r0 + 1;
        } else if (y == fy && x != fx) {
            vertical = false;
            r0 = r1 = (int)fy;
            c0 = (int)fx;
            c1 = c0 + 1;
        } else {
            return;
        }
        if (!inside(r0, c0) || !inside(r1, c1)) return;
        const double a = chi[at(r0, c0)], b = chi[at(r1, c1)];
        const double da = dchi[t * cap + at(r0, c0)], db = dchi[t * cap + at(r1, c1)];
        const double den = (a - b) * (a - b);
        if (!(den > 0)) return;
        const double d = (a * db - b * da) / den;  // position = first + a / (a - b)
        if (vertical)
            *dy = d;
        else
            *dx = d;
    };
    double* dP = S->dcontCur + 8 * S->coff_cur[g];  // kept for the next step's corrector
    for (int i = 0; i < n; ++i)
        for (int t = 0; t < kNP; ++t) dpoint(i, t, &dP[8 * i + t], &dP[8 * i + 4 + t]);
    double s = 0;
    for (int i = 0; i < n - 1; i++) s += (P[i].y + P[i + 1].y) * (P[i].x - P[i + 1].x);
    const double sg = s > 0 ? 1.0 : (s < 0 ? -1.0 : 0.0);
    for (int t = 0; t < kNP; ++t) {
        double ds = 0;
        double dx0 = dP[t], dy0 = dP[4 + t], dx1, dy1;
        for (int i = 0; i < n - 1; i++) {
            dx1 = dP[8 * (i + 1) + t];
            dy1 = dP[8 * (i + 1) + 4 + t];
            ds += (dy0 + dy1) * (P[i].x - P[i + 1].x) + (P[i].y + P[i + 1].y) * (dx0 - dx1);
            dx0 = dx1;
            dy0 = dy1;
        }
        out[t] = sg * ds * C.h * C.h * 0.5;
    }
}

// Redistancing with tangents (replaces k_redistance_s in tangent mode; the
// value arithmetic is the same, in global memory).  Every output value is a
// zero-crossing value -dz sgn(slope) = a h s / (c - a) plus steps of +-h, so
// it carries that crossing's tangent h s (c da - a dc) / (c - a)^2; the -1
// start values and clamped outputs carry none.
__global__ void __launch_bounds__(64) k_redistance_t(NetConst C, NetState* S) {
    const int g = blockIdx.x + 1;
    if (g > C.N || C.state[g] != G_EXISTS || halted(S)) return;
    const Box bi = S->box_cur[g], bo = S->box_new[g];
    const double h = C.h, delta = C.delta;
    const double* in = phiA_of<double>(S) + S->off_cur[g];
    const double* din = reinterpret_cast<const double*>(S->dphiA) + S->off_cur[g];
    double* out = phiB_of<double>(S) + S->off_new[g];
    double* dout = reinterpret_cast<double*>(S->dphiB) + S->off_new[g];
    const int64_t cap = S->phi_cap;
    const int wi = box_w(bi), wo = box_w(bo);
    const int64_t ao = box_area(bo);
    for (int64_t p = threadIdx.x; p < ao; p += blockDim.x) {
        out[p] = -1.0;
        for (int t = 0; t < kNP; ++t) dout[t * cap + p] = 0.0;
    }
    __syncthreads();
    const int ixmin = (bi.x0 < bo.x0) ? bo.x0 : bi.x0;
    const int iymin = (bi.y0 < bo.y0) ? bo.y0 : bi.y0;
    const int ixmax = (bi.x1 < bo.x1) ? bi.x1 : bo.x1;
    const int iymax = (bi.y1 < bo.y1) ? bi.y1 : bo.y1;
    auto II = [&](int i, int j) { return (int64_t)(i - bi.y0) * wi + (j - bi.x0); };
    auto OI = [&](int i, int j) { return (int64_t)(i - bo.y0) * wo + (j - bo.x0); };
    // tangent of the crossing value between input pixels ia (value a) and ic (value c)
    auto cross_d = [&](int64_t ia, int64_t ic, double a, double c, double s, double* d) {
        const double den = (c - a) * (c - a);
        for (int t = 0; t < kNP; ++t)
            d[t] = den > 0 ? h * s * (c * din[t * cap + ia] - a * din[t * cap + ic]) / den : 0.0;
    };
    double dcur[kNP], dcand[kNP];
    // y forward / backward per column
    for (int j = ixmin + (int)threadIdx.x; j < bo.x1; j += blockDim.x) {
        if (iymin < bo.y1 - 1) {
            double cur = out[OI(iymin, j)];
            for (int t = 0; t < kNP; ++t) dcur[t] = dout[t * cap + OI(iymin, j)];
            for (int i = iymin; i < bo.y1 - 1; i++) {
                double nxt = out[OI(i + 1, j)];
                double cand;
                if (j < ixmax && i < iymax - 1) {
                    const double a = in[II(i, j)], c = in[II(i + 1, j)];
                    if (a * c <= 0.0) {
                        const double slope = (c - a) / h;
                        const double dz = -a / slope;
                        if (fabs(cur) > fabs(dz)) {
                            cur = -dz * sgn(slope);
                            out[OI(i, j)] = cur;
                            cross_d(II(i, j), II(i + 1, j), a, c, (double)sgn(slope), dcur);
                            for (int t = 0; t < kNP; ++t) dout[t * cap + OI(i, j)] = dcur[t];
                        }
                    }
                    cand = cur + (sgn(c) * h);
                } else {
                    cand = cur + (sgn(nxt) * h);
                }
                if (fabs(cand) < fabs(nxt)) {
                    nxt = cand;
                    out[OI(i + 1, j)] = nxt;
                    for (int t = 0; t < kNP; ++t) dout[t * cap + OI(i + 1, j)] = dcur[t];
                } else {
                    for (int t = 0; t < kNP; ++t) dcur[t] = dout[t * cap + OI(i + 1, j)];
                }
                cur = nxt;
            }
        }
        if (iymax - 1 > bo.y0) {
            double cur = out[OI(iymax - 1, j)];
            for (int t = 0; t < kNP; ++t) dcur[t] = dout[t * cap + OI(iymax - 1, j)];
            for (int i = iymax - 1; i > bo.y0; i--) {
                double prv = out[OI(i - 1, j)];
                double cand;
                if (j < ixmax && i > iymin)
                    cand = cur + (sgn(in[II(i - 1, j)]) * h);
                else
                    cand = cur + (sgn(prv) * h);
                if (fabs(cand) < fabs(prv)) {
                    prv = cand;
                    out[OI(i - 1, j)] = prv;
                    for (int t = 0; t < kNP; ++t) dout[t * cap + OI(i - 1, j)] = dcur[t];
                } else {
                    for (int t = 0; t < kNP; ++t) dcur[t] = dout[t * cap + OI(i - 1, j)];
                }
                cur = prv;
            }
        }
    }
    __syncthreads();
    // x forward / backward per row
    for (int i = iymin + (int)threadIdx.x; i < bo.y1; i += blockDim.x) {
        if (ixmin < bo.x1 - 1) {
            double cur = out[OI(i, ixmin)];
            for (int t = 0; t < kNP; ++t) dcur[t] = dout[t * cap + OI(i, ixmin)];
            for (int j = ixmin; j < bo.x1 - 1; j++) {
                double nxt = out[OI(i, j + 1)];
                double cand;
                if (j < ixmax - 1 && i < iymax) {
                    const double a = in[II(i, j)], c = in[II(i, j + 1)];
                    if (a * c <= 0.0) {
                        const double slope = (c - a) / h;
                        const double dz = -a / slope;
                        if (fabs(cur) > fabs(dz)) {
                            cur = -dz * sgn(slope);
                            out[OI(i, j)] = cur;
                            cross_d(II(i, j), II(i, j + 1), a, c, (double)sgn(slope), dcur);
                            for (int t = 0; t < kNP; ++t) dout[t * cap + OI(i, j)] = dcur[t];
                        }
                    }
                    cand = cur + (sgn(c) * h);
                } else {
                    cand = cur + (sgn(nxt) * h);
                }
                if (fabs(cand) < fabs(nxt)) {
                    nxt = cand;
                    out[OI(i, j + 1)] = nxt;
                    for (int t = 0; t < kNP; ++t) dout[t * cap + OI(i, j + 1)] = dcur[t];
                } else {
                    for (int t = 0; t < kNP; ++t) dcur[t] = dout[t * cap + OI(i, j + 1)];
                }
                cur = nxt;
            }
        }
        if (ixmax - 1 > bo.x0) {
            double cur = out[OI(i, ixmax - 1)];
            for (int t = 0; t < kNP; ++t) dcur[t] = dout[t * cap + OI(i, ixmax - 1)];
            for (int j = ixmax - 1; j > bo.x0; j--) {
                double prv = out[OI(i, j - 1)];
                double cand;
                if (j > ixmin && i < iymax)
                    cand = cur + (sgn(in[II(i, j - 1)]) * h);
                else
                    cand = cur + sgn(prv) * h;
                if (fabs(cand) < fabs(prv)) {
                    prv = cand;
                    out[OI(i, j - 1)] = prv;
                    for (int t = 0; t < kNP; ++t) dout[t * cap + OI(i, j - 1)] = dcur[t];
                } else {
                    for (int t = 0; t < kNP; ++t) dcur[t] = dout[t * cap + OI(i, j - 1)];
                }
                cur = prv;
            }
        }
    }
    __syncthreads();
    for (int64_t p = threadIdx.x; p < ao; p += blockDim.x) {  // clampValues(-delta, delta)
        double v = out[p];
        if (v < -delta || v > delta) {
            v = v < -delta ? -delta : delta;
            for (int t = 0; t < kNP; ++t) dout[t * cap + p] = 0.0;
        }
        out[p] = v;
    }
    (void)dcand;
}

}  // namespace
}  // namespace gg

// Warp-per-grain versions of the per-grain sequential stages (level set,
// volume/energy/neighbours, second-order lists).  The parts of each
// reference routine that are independent per pixel, per contour point or per
// list entry run across the 32 lanes; every order-dependent part (the
// marching-squares walk, list construction, sums) runs on lane 0 in the
// reference's order, so the FP64 form stays bit-identical.
#pragma once

#include "gg_grain.cuh"
#include "gg_kernels.cuh"

namespace gg {
namespace {  // internal linkage: each form's translation unit has its own copy

constexpr int kGrainsPerBlock = 4;  // warps (grains) per CTA of the warp kernels

__device__ __forceinline__ int warp_min_i(int v) {
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// First pixel of the box (row-major) with phi >= 0, as the scan of
// generateContour (src/marchingSquares.cpp:32-42); -1 if none.
template <typename R>
__device__ int first_inside_warp(const Field<R>& f, int lane) {
    const int w = box_w(f.b), h = box_h(f.b);
    for (int r = 0; r < h; ++r) {
        int best = 0x7fffffff;
        for (int c = lane; c < w; c += 32)
            if ((double)f.v[r * w + c] >= 0) {
                best = c;
                break;
            }
        best = warp_min_i(best);
        if (best != 0x7fffffff) return r * w + best;
    }
    return -1;
}

// Marching-squares walk from a known start pixel (src/marchingSquares.cpp:44-187).
// The four corner values of the current square are kept in registers and
// only the two corners a move uncovers are loaded; the last emitted point
// is kept in registers for insertPoint's duplicate test; junction corners
// are only read where a junction is possible (at most two inside corners).
template <typename R>
__device__ void ms_walk(const Field<R>& f, const uint32_t* idl, uint32_t own, int startX, int startY,
                        ContourOut& o) {
    o.n = 0;
    o.jn = 0;
    const Box b = f.b;
    const int w = b.x1 - b.x0;
    auto val = [&](int row, int col, double* v) -> bool {  // value and isInside
        if (row < b.y0 || row >= b.y1 || col < b.x0 || col >= b.x1) {
            *v = -1.0;
            return false;
        }
        *v = (double)f.v[(row - b.y0) * w + (col - b.x0)];
        return *v >= 0;
    };
    int left = startX - 1, right = startX, top = startY - 1, bottom = startY;
    double vTL, vTR, vBL, vBR;
    bool iTL = val(top, left, &vTL), iTR = val(top, right, &vTR);
    bool iBL = val(bottom, left, &vBL), iBR = val(bottom, right, &vBR);
    int next = MS_NONE, prev = MS_NONE;
    double lastx = 0, lasty = 0, firstx = 0, firsty = 0;
    const long limit = 4L * (w + 2) * (box_h(b) + 2) + 16;
    long it = 0;
    do {
        int mask = 0;
        if (iTL) mask |= C_TL;
        if (iTR) mask |= C_TR;
        if (iBL) mask |= C_BL;
        if (iBR) mask |= C_BR;
        bool emit = true;
        switch (mask) {
            case C_TL: next = MS_UP; break;
            case C_TR: next = MS_RIGHT; break;
            case C_TL | C_TR: next = MS_RIGHT; break;
            case C_BL: next = MS_LEFT; break;
            case C_BL | C_TL: next = MS_UP; break;
            case C_BL | C_TR:
                next = (prev == MS_UP) ? MS_RIGHT : MS_LEFT;
                emit = false;
                break;
            case C_BL | C_TR | C_TL: next = MS_RIGHT; break;
            case C_BR: next = MS_DOWN; break;
            case C_BR | C_TL:
                next = (prev == MS_RIGHT) ? MS_DOWN : MS_UP;
                emit = false;
                break;
            case C_BR | C_TR: next = MS_DOWN; break;
            case C_BR | C_TR | C_TL: next = MS_DOWN; break;
            case C_BR | C_BL: next = MS_LEFT; break;
            case C_BR | C_BL | C_TL: next = MS_UP; break;
            case C_BR | C_BL | C_TR: next = MS_LEFT; break;
            default: emit = false; break;
        }
        if (emit) {  // generatePoint (src/marchingSquares.cpp:204-265) on the cached corners
            double px, py, delta, position;
            switch (next) {
                case MS_LEFT:
                    px = left;
                    if (top < b.y0) {
                        py = bottom;
                    } else {
                        delta = vBL - vTL;
                        position = bottom - vBL / delta;
                        py = position;
                    }
                    break;
                case MS_RIGHT:
                    px = right;
                    if (bottom >= b.y1) {
                        py = top;
                    } else {
                        delta = vTR - vBR;
                        position = top + vTR / delta;
                        py = position;
                    }
                    break;
                case MS_UP:
                    py = top;
                    if (right >= b.x1) {
                        px = left;
                    } else {
                        delta = vTL - vTR;
                        position = left + vTL / delta;
                        px = position;
                    }
                    break;
                default:
                    py = bottom;
                    if (left < b.x0) {
                        px = right;
                    } else {
                        delta = vBR - vBL;
                        position = right - vBR / delta;
                        px = position;
                    }
                    break;
            }
            if (o.n == 0 || px != lastx || py != lasty) {  // insertPoint
                if (o.n >= o.cap) {
                    o.status |= S_CONTOUR_OVERFLOW;
                } else {
                    CPoint& q = o.pts[o.n];
                    q.x = px;
                    q.y = py;
                    q.energy = -1.0;
                    q.mob = -1.0;
                    if (o.n == 0) {
                        firstx = px;
                        firsty = py;
                    }
                    o.n++;
                    lastx = px;
                    lasty = py;
                }
            }
        }
        if (__popc(mask) < 3) ms_junction(f, idl, own, mask, top, bottom, left, right, o);
        switch (next) {
            case MS_UP:
                top--;
                bottom--;
                vBL = vTL;
                vBR = vTR;
                iBL = iTL;
                iBR = iTR;
                iTL = val(top, left, &vTL);
                iTR = val(top, right, &vTR);
                break;
            case MS_DOWN:
                top++;
                bottom++;
                vTL = vBL;
                vTR = vBR;
                iTL = iBL;
                iTR = iBR;
                iBL = val(bottom, left, &vBL);
                iBR = val(bottom, right, &vBR);
                break;
            case MS_LEFT:
                left--;
                right--;
                vTR = vTL;
                vBR = vBL;
                iTR = iTL;
                iBR = iBL;
                iTL = val(top, left, &vTL);
                iBL = val(bottom, left, &vBL);
                break;
            case MS_RIGHT:
                left++;
                right++;
                vTL = vTR;
                vBL = vBR;
                iTL = iTR;
                iBL = iBR;
                iTR = val(top, right, &vTR);
                iBR = val(bottom, right, &vBR);
                break;
            default: break;
        }
        prev = next;
        if (++it > limit) {
            o.status |= S_WALK_LIMIT;
            break;
        }
    } while (left != startX - 1 || bottom != startY);
    if (o.n > 0 && (firstx != lastx || firsty != lasty)) {
        if (o.n >= o.cap) {
            o.status |= S_CONTOUR_OVERFLOW;
        } else {
            o.pts[o.n] = o.pts[0];
            o.n++;
        }
    }
}

// Contour + junctions of one grain by one warp; returns false if no pixel
// has phi >= 0.  Junctions are projected one lane per junction.
template <typename R>
__device__ bool extract_warp(const Field<R>& f, const uint32_t* idl, uint32_t own, ContourOut& o, int lane) {
    const int start = first_inside_warp(f, lane);
    if (start < 0) {
        o.n = 0;
        o.jn = 0;
        return false;
    }
    const int w = box_w(f.b);
    if (lane == 0) ms_walk(f, idl, own, f.b.x0 + start % w, f.b.y0 + start / w, o);
    o.n = __shfl_sync(0xffffffffu, o.n, 0);
    o.jn = __shfl_sync(0xffffffffu, o.jn, 0);
    o.status = __shfl_sync(0xffffffffu, o.status, 0);
    __syncwarp();
    if (o.n >= 2) {
        for (int j = lane; j < o.jn; j += 32) {
            double lambda = 0.0;
            const int seg = project_to_boundary(o.pts, o.n, o.js[j].x, o.js[j].y, &lambda);
            const int nx = periodic(seg + 1, o.n);
            o.js[j].x = o.pts[seg].x + (o.pts[nx].x - o.pts[seg].x) * lambda;
            o.js[j].y = o.pts[seg].y + (o.pts[nx].y - o.pts[seg].y) * lambda;
            o.js[j].segment = seg;
            o.js[j].lambda = lambda;
        }
    }
    __syncwarp();
    return true;
}

// grainhdl::level_set -> LSbox::extractContour (src/grainhdl.cpp:830-848,
// src/box.cpp:1089-1153), one warp per grain.
template <typename R>
__global__ void __launch_bounds__(32 * kGrainsPerBlock) k_levelset_w(NetConst C, NetState* S) {
    const int lane = threadIdx.x & 31;
    const int g = blockIdx.x * kGrainsPerBlock + (threadIdx.x >> 5) + 1;
    if (g > C.N || halted(S)) return;
    const int st = C.state[g];
    const Box bc = S->box_cur[g];
    if (st != G_EXISTS) {
        if (lane == 0) {
            if (st == G_VANISHED) C.state[g] = G_GONE;
            S->box_new[g] = bc;
            S->cn_cur[g] = 0;
            S->jn_cur[g] = 0;
        }
        return;
    }
    const int old_len = S->cn_prev[g];
    R* phi = phiA_of<R>(S) + S->off_cur[g];
    Field<R> f{phi, bc};
    const uint32_t* idl = S->idCur + S->off_cur[g];
    ContourOut o{S->contCur + S->coff_cur[g], S->ccap_cur[g], 0, S->jCur + (int64_t)g * C.jmax, C.jmax, 0, 0};
    bool ok = extract_warp(f, idl, (uint32_t)g, o, lane);
    int irregular = 0;
    if (ok) {
        double newVolume = 0;
        bool regular_motion = true;
        if (lane == 0) {
            newVolume = contour_volume(o.pts, o.n, C.h);
            regular_motion = motion_regular(old_len, o.n, C.volume[g], newVolume, C.dt, &irregular);
        }
        regular_motion = __shfl_sync(0xffffffffu, regular_motion, 0);
        int tries = 0;
        while (!regular_motion) {  // clear the grain area and extract again (src/box.cpp:1099-1114)
            if (lane == 0 && !clear_contour_area(phi, bc, o.pts, o.n, C.h)) o.status |= S_INDEX;
            __syncwarp();
            ok = extract_warp(f, idl, (uint32_t)g, o, lane);
            if (!ok) break;
            if (lane == 0) {
                newVolume = contour_volume(o.pts, o.n, C.h);
                regular_motion = motion_regular(old_len, o.n, C.volume[g], newVolume, C.dt, &irregular);
                if (++tries > 64) {
                    o.status |= S_RETRY_LIMIT;
                    regular_motion = true;
                }
            }
            regular_motion = __shfl_sync(0xffffffffu, regular_motion, 0);
        }
    }
    if (lane != 0) return;
    if (o.status) set_status(S, o.status);
    C.regular[g] = 1;
    if (!ok) {
        C.state[g] = G_VANISHED;
        S->box_new[g] = bc;
        S->cn_cur[g] = 0;
        S->jn_cur[g] = 0;
        return;
    }
    if (irregular) C.regular[g] = 0;
    int* nb = C.newbb + 4 * (int64_t)g;
    Box nbx = bc;
    if (!C.decouple) {
        if (nb[0] < 0) nb[0] = 0;
        if (nb[2] < 0) nb[2] = 0;
        if (nb[1] > C.m) nb[1] = C.m;
        if (nb[3] > C.m) nb[3] = C.m;
        nbx = resize_to_square(Box{nb[0], nb[1], nb[2], nb[3]}, C.m);
    }
    S->box_new[g] = nbx;
    C.perimeter[g] = contour_perimeter(o.pts, o.n, C.h);
    S->cn_cur[g] = o.n;
    S->jn_cur[g] = o.jn;
}

// Per contour point result of the neighbour probe of buildDirectNeighbours.
struct PointInfo {
    int32_t cid;
    int32_t pad;
    double theta;
    double len;
};

// LSbox::computeVolumeAndEnergy + ExplicitGrainBoundary::buildDirectNeighbours
// (src/box.cpp:1201-1228, src/grainBoundary.cpp:85-199), one warp per grain:
// lanes probe contour points and evaluate the per-pair physics, lane 0 builds
// the neighbour list and the sums in contour order.
template <typename R>
__global__ void __launch_bounds__(32 * kGrainsPerBlock) k_neighbours_w(NetConst C, NetState* S, PointInfo* scratch) {
    const int lane = threadIdx.x & 31;
    const int g = blockIdx.x * kGrainsPerBlock + (threadIdx.x >> 5) + 1;
    if (g > C.N || C.state[g] != G_EXISTS || C.regular[g] == 0 || halted(S)) return;
    const int loop = S->loop;
    CPoint* P = S->contCur + S->coff_cur[g];
    PointInfo* info = scratch + S->coff_cur[g];
    const int n = S->cn_cur[g];
    const double h = C.h;
    const Box bc = S->box_cur[g];
    const R* phi = phiA_of<R>(S) + S->off_cur[g];
    const uint32_t* idl = S->idCur + S->off_cur[g];
    const double* qg = C.quat + 4 * (int64_t)g;
    // probes, in parallel; the first failing point ends the reference's loop
    int first_bad = 0x7fffffff;
    for (int i = lane; i < n - 1; i += 32) {
        const double px = P[i].x, py = P[i].y;
        int pxGrid = (int)px, pyGrid = (int)py;
        uint32_t k;
        bool bad = false;
        if (!buf_index(bc, pyGrid, pxGrid, &k)) bad = true;
        if (!bad && (double)phi[k] > 0) {
            pxGrid = (int)(px + 1);
            if (!buf_index(bc, pyGrid, pxGrid, &k)) bad = true;
            if (!bad && (double)phi[k] > 0) {
                pyGrid = (int)(py + 1);
                if (!buf_index(bc, pyGrid, pxGrid, &k)) bad = true;
                if (!bad && (double)phi[k] > 0) pxGrid = (int)px;
            }
        }
        if (!bad && (pyGrid < 0 || pyGrid >= bc.y1 || pxGrid < 0 || pxGrid >= bc.x1)) bad = true;
        if (!bad && !buf_index(bc, pyGrid, pxGrid, &k)) bad = true;
        uint32_t cid = 0;
        if (!bad) {
            cid = idl[k];
            if (cid != 0 && (cid > (uint32_t)C.N || C.state[cid] == G_GONE)) bad = true;
        }
        if (bad) {
            first_bad = min(first_bad, i);
            info[i].cid = -1;
            continue;
        }
        info[i].cid = (int)cid;
        const double theta = grain_misorientation(qg, C.quat + 4 * (int64_t)cid);
        info[i].theta = theta;
        const double dx = P[i].x - P[i + 1].x, dy = P[i].y - P[i + 1].y;
        info[i].len = sqrt(dx * dx + dy * dy) * h;
    }
    first_bad = warp_min_i(first_bad);
    const int upto = first_bad < n - 1 ? first_bad : n - 1;
    __syncwarp();
    for (int i = lane; i < upto; i += 32) {  // points before the first failure get their physics
        const double theta = info[i].theta;
        P[i].mob = mobility_model(theta, C);
        P[i].energy = read_shockley(theta, C);
    }
    __syncwarp();
    if (lane != 0) return;
    const double newVolume = fabs(contour_volume(P, n, h));
    Neighbour* nb = C.nb + (int64_t)g * C.nbmax;
    int nn = 0;
    bool overflow = false;
    for (int i = 0; i < upto; i++) {
        const int cid = info[i].cid;
        int e = 0;
        for (; e < nn; ++e)
            if (nb[e].id == cid) break;
        if (e == nn) {
            if (nn >= C.nbmax) {
                overflow = true;
                continue;
            }
            nb[nn].id = cid;
            nb[nn].length = 0;
            nb[nn].energy = P[i].energy;
            nb[nn].misori = info[i].theta;
            nb[nn].mobility = P[i].mob;
            nn++;
        }
        nb[e].length += info[i].len;
    }
    C.nb_n[g] = nn;
    if (overflow) set_status(S, S_NEIGHBOUR_OVERFLOW);
    if (first_bad < n - 1) {
        C.regular[g] = 0;  // markAsInvalidMotion (src/box.cpp:1939-1945)
    } else if (n > 0) {
        P[n - 1].energy = P[0].energy;
        P[n - 1].mob = P[0].mob;
    }
    C.energy[g] = contour_energy(P, n, h);
    double dA = newVolume - C.volume[g];
    dA = dA / C.dt;
    dA = dA * (3 / kPi);
    const unsigned int lp = (unsigned int)loop;
    if ((unsigned long)(lp - 1u) % (unsigned long)C.analysis_timestep == 0 || lp == 0) C.meanda[g] = 0;
    C.meanda[g] += dA;
    C.volume[g] = newVolume;
}

// LSbox::computeSecondOrderNeighbours (src/box.cpp:1027-1068), one warp per
// grain: candidates of each member's list are tested across lanes and the
// accepted ones appended in list order.
__global__ void __launch_bounds__(32 * kGrainsPerBlock) k_second_order_w(NetConst C, NetState* S) {
    const int lane = threadIdx.x & 31;
    const int g = blockIdx.x * kGrainsPerBlock + (threadIdx.x >> 5) + 1;
    if (g > C.N || C.state[g] != G_EXISTS) return;
    const int K = C.kmax;
    const int* sec = C.sec_ids + (int64_t)g * K;
    const int ns = C.sec_n[g];
    int* cmp = C.cmp_ids + (int64_t)g * K;
    const unsigned lt = (1u << lane) - 1u;
    int nc = 0;
    bool overflow = false;
    for (int a0 = 0; a0 < ns; a0 += 32) {  // existing members, in order
        const int a = a0 + lane;
        const bool take = a < ns && C.state[sec[a]] == G_EXISTS;
        const unsigned bal = __ballot_sync(0xffffffffu, take);
        if (take) {
            const int pos = nc + __popc(bal & lt);
            if (pos < K) cmp[pos] = sec[a]; else overflow = true;
        }
        nc += __popc(bal);
    }
    if (nc > K) nc = K;
    __syncwarp();
    const Box mine = S->box_cur[g];
    for (int a = 0; a < ns; ++a) {
        const int id = sec[a];
        const int* s2 = C.sec_ids + (int64_t)id * K;
        const int n2 = C.sec_n[id];
        for (int q0 = 0; q0 < n2; q0 += 32) {
            const int q = q0 + lane;
            bool take = false;
            int c = 0;
            if (q < n2) {
                c = s2[q];
                take = C.state[c] == G_EXISTS && boxes_intersect(mine, S->box_cur[c]) && c != g && c != 0;
                if (take)
                    for (int e = 0; e < nc; ++e)
                        if (cmp[e] == c) {
                            take = false;
                            break;
                        }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, take);
            if (take) {
                const int pos = nc + __popc(bal & lt);
                if (pos < K) cmp[pos] = c; else overflow = true;
            }
            nc += __popc(bal);
            if (nc > K) nc = K;
            __syncwarp();
        }
    }
    if (lane == 0) {
        C.cmp_n[g] = nc;
        if (overflow) set_status(S, S_LIST_OVERFLOW);
    }
}

// LSbox::executeRedistancing (src/box.cpp:1259-1399), one warp per grain:
// lanes take columns for the two y sweeps, then rows for the two x sweeps
// (each column / row is a sequential recurrence, as in the reference).
template <typename R>
__global__ void __launch_bounds__(32 * kGrainsPerBlock) k_redistance_w(NetConst C, NetState* S) {
    const int lane = threadIdx.x & 31;
    const int g = blockIdx.x * kGrainsPerBlock + (threadIdx.x >> 5) + 1;
    if (g > C.N || C.state[g] != G_EXISTS || halted(S)) return;
    const R* __restrict__ in = phiA_of<R>(S) + S->off_cur[g];
    R* __restrict__ out = phiB_of<R>(S) + S->off_new[g];
    const Box bi = S->box_cur[g], bo = S->box_new[g];
    const R h = (R)C.h, delta = (R)C.delta;
    const int wi = box_w(bi), wo = box_w(bo);
    const int64_t ao = box_area(bo);
    for (int64_t p = lane; p < ao; p += 32) out[p] = (R)-1.0;
    __syncwarp();
    const int ixmin = (bi.x0 < bo.x0) ? bo.x0 : bi.x0;
    const int iymin = (bi.y0 < bo.y0) ? bo.y0 : bi.y0;
    const int ixmax = (bi.x1 < bo.x1) ? bi.x1 : bo.x1;
    const int iymax = (bi.y1 < bo.y1) ? bi.y1 : bo.y1;
#define GG_IN(i, j) in[(int64_t)((i) - bi.y0) * wi + ((j) - bi.x0)]
#define GG_OUT(i, j) out[(int64_t)((i) - bo.y0) * wo + ((j) - bo.x0)]
    for (int j = ixmin + lane; j < bo.x1; j += 32) {
        for (int i = iymin; i < bo.y1 - 1; i++) {  // y forward
            R cand;
            if (j < ixmax && i < iymax - 1) {
                const R a = GG_IN(i, j), c = GG_IN(i + 1, j);
                if (a * c <= (R)0.0) {
                    const R slope = (c - a) / h;
                    const R dz = -a / slope;
                    if (fabs(GG_OUT(i, j)) > fabs(dz)) GG_OUT(i, j) = -dz * (R)sgn(slope);
                }
                cand = GG_OUT(i, j) + ((R)sgn(c) * h);
            } else {
                cand = GG_OUT(i, j) + ((R)sgn(GG_OUT(i + 1, j)) * h);
            }
            if (fabs(cand) < fabs(GG_OUT(i + 1, j))) GG_OUT(i + 1, j) = cand;
        }
        for (int i = iymax - 1; i > bo.y0; i--) {  // y backward
            R cand;
            if (j < ixmax && i > iymin)
                cand = GG_OUT(i, j) + ((R)sgn(GG_IN(i - 1, j)) * h);
            else
                cand = GG_OUT(i, j) + ((R)sgn(GG_OUT(i - 1, j)) * h);
            if (fabs(cand) < fabs(GG_OUT(i - 1, j))) GG_OUT(i - 1, j) = cand;
        }
    }
    __syncwarp();
    for (int i = iymin + lane; i < bo.y1; i += 32) {
        for (int j = ixmin; j < bo.x1 - 1; j++) {  // x forward
            R cand;
            if (j < ixmax - 1 && i < iymax) {
                const R a = GG_IN(i, j), c = GG_IN(i, j + 1);
                if (a * c <= (R)0.0) {
                    const R slope = (c - a) / h;
                    const R dz = -a / slope;
                    if (fabs(GG_OUT(i, j)) > fabs(dz)) GG_OUT(i, j) = -dz * (R)sgn(slope);
                }
                cand = GG_OUT(i, j) + ((R)sgn(c) * h);
            } else {
                cand = GG_OUT(i, j) + ((R)sgn(GG_OUT(i, j + 1)) * h);
            }
            if (fabs(cand) < fabs(GG_OUT(i, j + 1))) GG_OUT(i, j + 1) = cand;
        }
        for (int j = ixmax - 1; j > bo.x0; j--) {  // x backward
            R cand;
            if (j > ixmin && i < iymax)
                cand = GG_OUT(i, j) + ((R)sgn(GG_IN(i, j - 1)) * h);
            else
                cand = GG_OUT(i, j) + (R)sgn(GG_OUT(i, j - 1)) * h;
            if (fabs(cand) < fabs(GG_OUT(i, j - 1))) GG_OUT(i, j - 1) = cand;
        }
    }
#undef GG_IN
#undef GG_OUT
    __syncwarp();
    for (int64_t p = lane; p < ao; p += 32) {  // clampValues(-delta, delta)
        const R v = out[p];
        if (v < -delta)
            out[p] = -delta;
        else if (v > delta)
            out[p] = delta;
    }
}

}  // namespace
}  // namespace gg

/*
 * CPU restatement of GraGLeS2D's per-grain level-set routines.
 *
 * Test infrastructure: only tests/, __graft_entry__.smoke() and bench.py's
 * CPU arm use it, as the checker; the product never links it.  Each function
 * follows the reference routine cited at its head; FP64 throughout, compiled
 * with -ffp-contract=off so every operation rounds as in the reference.
 * Parity pinned against the reference's own dumps: tests/test_oracle_port.py.
 */
#include "gg_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OR_PI 3.14159265358979323846 /* src/ggLS.h:26 */

static int bw(const int* b) { return b[1] - b[0]; }
static int bh(const int* b) { return b[3] - b[2]; }

/* ---- convolution ---------------------------------------------------------- */

static void twiddle(int n, int k, double* re, double* im) {
    double ang = (2.0 * OR_PI * (double)k) / (double)n;
    *re = cos(ang);
    *im = -sin(ang);
}

/* src/box.cpp:622-695: r2c, G(i2, j2) multiply, c2r (FFTW semantics as in
 * oracle/shim/fft_shim.c). */
void gg_or_convolve(int n, const double* in, double* out, double dt, int real_domain_size) {
    const int half = n / 2 + 1;
    double* w = (double*)malloc(sizeof(double) * 2 * (size_t)n);
    double* t = (double*)malloc(sizeof(double) * 2 * (size_t)n * half);
    double* y = (double*)malloc(sizeof(double) * 2 * (size_t)n * half);
    for (int k = 0; k < n; ++k) twiddle(n, k, &w[2 * k], &w[2 * k + 1]);
    /* rows: real -> half spectrum */
    for (int r = 0; r < n; ++r)
        for (int f = 0; f < half; ++f) {
            double re = 0.0, im = 0.0;
            for (int c = 0; c < n; ++c) {
                int k = (int)(((long)f * c) % n);
                re = re + in[(size_t)r * n + c] * w[2 * k];
                im = im + in[(size_t)r * n + c] * w[2 * k + 1];
            }
            t[2 * ((size_t)r * half + f)] = re;
            t[2 * ((size_t)r * half + f) + 1] = im;
        }
    /* columns */
    for (int f = 0; f < half; ++f)
        for (int q = 0; q < n; ++q) {
            double re = 0.0, im = 0.0;
            for (int r = 0; r < n; ++r) {
                int k = (int)(((long)q * r) % n);
                double a = t[2 * ((size_t)r * half + f)], b = t[2 * ((size_t)r * half + f) + 1];
                re = re + (a * w[2 * k] - b * w[2 * k + 1]);
                im = im + (a * w[2 * k + 1] + b * w[2 * k]);
            }
            y[2 * ((size_t)q * half + f)] = re;
            y[2 * ((size_t)q * half + f) + 1] = im;
        }
    /* Gaussian multiplier, src/box.cpp:674-687 */
    {
        double nsq = real_domain_size * real_domain_size;
        double n_nsq = n * n;
        for (int i = 0; i < half; i++) {
            int i2 = i > n - i ? n - i : i;
            for (int j = 0; j < n; j++) {
                int j2 = j > n - j ? n - j : j;
                double G = exp(-sqrt(2 / OR_PI) * (i2 * i2 + j2 * j2) * 4.0 * dt * nsq / n_nsq * OR_PI * OR_PI) / n_nsq;
                y[2 * ((size_t)j * half + i)] = y[2 * ((size_t)j * half + i)] * G;
                y[2 * ((size_t)j * half + i) + 1] = y[2 * ((size_t)j * half + i) + 1] * G;
            }
        }
    }
    /* inverse columns */
    for (int f = 0; f < half; ++f)
        for (int r = 0; r < n; ++r) {
            double re = 0.0, im = 0.0;
            for (int q = 0; q < n; ++q) {
                int k = (int)(((long)q * r) % n);
                double a = y[2 * ((size_t)q * half + f)], b = y[2 * ((size_t)q * half + f) + 1];
                double wc = w[2 * k], ws = -w[2 * k + 1];
                re = re + (a * wc - b * ws);
                im = im + (a * ws + b * wc);
            }
            t[2 * ((size_t)r * half + f)] = re;
            t[2 * ((size_t)r * half + f) + 1] = im;
        }
    /* rows: half spectrum -> real */
    const int hmax = (n - 1) / 2;
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) {
            double acc = t[2 * ((size_t)r * half)];
            for (int f = 1; f <= hmax; ++f) {
                int k = (int)(((long)f * c) % n);
                acc = acc + 2.0 * (t[2 * ((size_t)r * half + f)] * w[2 * k] + t[2 * ((size_t)r * half + f) + 1] * w[2 * k + 1]);
            }
            if ((n & 1) == 0) {
                double nyq = t[2 * ((size_t)r * half + n / 2)];
                acc = acc + ((c & 1) ? -nyq : nyq);
            }
            out[(size_t)r * n + c] = acc;
        }
    free(w);
    free(t);
    free(y);
}

/* ---- comparison ------------------------------------------------------------ */

/* boundaryCondition's wall distance (src/box.cpp:968-1025) */
static double wall_distance(int i, int j, int b, int m) {
    int dxmin = -(j - b), dymin = -(i - b), dxmax = j - (m - b), dymax = i - (m - b);
    int dx = abs(dxmin) < abs(dxmax) ? dxmin : dxmax;
    int dy = abs(dymin) < abs(dymax) ? dymin : dymax;
    if (dx > 0 && dy > 0) return sqrt((double)dx * dx + dy * dy);
    if (dx < 0 && dy > 0) return dy;
    if (dx > 0 && dy < 0) return dx;
    if (dx < 0 && dy < 0) return dx > dy ? dx : dy;
    if (dx == 0) return dy > 0 ? dy : 0;
    return dx > 0 ? dx : 0;
}

void gg_or_compare(const int* box, const double* own_conv, int nlist, const int* nbr_box,
                   const double* const* nbr_conv, const unsigned* nbr_id, const int* prev_box,
                   const unsigned* idprev, int m, int b, double h, double delta, double* cmp_out,
                   unsigned* id_out, int* newbb) {
    const int w = bw(box), hh = bh(box);
    const long area = (long)w * hh, parea = (long)bw(prev_box) * bh(prev_box);
    /* IDLocal resized from the previous box: the linear prefix survives */
    for (long p = 0; p < area; ++p) id_out[p] = p < parea ? idprev[p] : 0u;
    double* out = cmp_out;
    for (long p = 0; p < area; ++p) out[p] = -1.0;
    /* executeComparison: members in list order, strict '>' */
    for (int k = 0; k < nlist; ++k) {
        const int* nb = nbr_box + 4 * k;
        int x0 = box[0] < nb[0] ? nb[0] : box[0], x1 = box[1] > nb[1] ? nb[1] : box[1];
        int y0 = box[2] < nb[2] ? nb[2] : box[2], y1 = box[3] > nb[3] ? nb[3] : box[3];
        for (int i = y0; i < y1; i++)
            for (int j = x0; j < x1; j++) {
                double d = nbr_conv[k][(long)(i - nb[2]) * bw(nb) + (j - nb[0])];
                long p = (long)(i - box[2]) * w + (j - box[0]);
                if (d > out[p]) {
                    out[p] = d;
                    id_out[p] = nbr_id[k];
                }
            }
    }
    /* BoundaryIntersection (src/box.cpp:945-962) and boundaryCondition */
    const int lo = b + b, hi = m - b - b;
    if (!(box[0] > lo && box[1] < hi && box[2] > lo && box[3] < hi)) {
        for (int i = box[2]; i < box[3]; i++)
            for (int j = box[0]; j < box[1]; j++) {
                double d = wall_distance(i, j, b, m);
                long p = (long)(i - box[2]) * w + (j - box[0]);
                if (d * h > out[p]) {
                    out[p] = d * h;
                    id_out[p] = 0u;
                }
            }
    }
    /* executeSetComparison */
    int nx0 = box[1], nx1 = box[0], ny0 = box[3], ny1 = box[2];
    for (int i = box[2]; i < box[3]; i++)
        for (int j = box[0]; j < box[1]; j++) {
            long p = (long)(i - box[2]) * w + (j - box[0]);
            double in = own_conv[p];
            out[p] = fabs(in) < 0.7 * delta ? 0.5 * (in - out[p]) : in;
            if (out[p] >= 0) {
                if (i < ny0) ny0 = i;
                if (i > ny1) ny1 = i;
                if (j < nx0) nx0 = j;
                if (j > nx1) nx1 = j;
            }
        }
    nx0 -= b;
    nx1 += b;
    ny0 -= b;
    ny1 += b;
    if (nx0 >= nx1 || ny0 >= ny1) {
        nx0 = box[0];
        nx1 = box[1];
        ny0 = box[2];
        ny1 = box[3];
    }
    newbb[0] = nx0;
    newbb[1] = nx1;
    newbb[2] = ny0;
    newbb[3] = ny1;
}

/* ---- marching squares --------------------------------------------------------- */

enum { UP, DOWN, LEFT, RIGHT, NONE };
enum { TL = 1, TR = 2, BL = 4, BR = 8 };

typedef struct {
    const double* v;
    const int* box;
} field;

static int inside(const field* f, int row, int col) {
    const int* b = f->box;
    if (row < b[2] || row >= b[3] || col < b[0] || col >= b[1]) return 0;
    return f->v[(long)(row - b[2]) * bw(b) + (col - b[0])] >= 0;
}

static double at(const field* f, int row, int col) {
    return f->v[(long)(row - f->box[2]) * bw(f->box) + (col - f->box[0])];
}

/* projectToGrainBondary (src/grainBoundary.cpp:365-447) on (x, y) pairs */
static int project(const double* P, int asize, double px, double py, double* out_lambda) {
    double minDist = 1000000.0, dist = 0, lam = *out_lambda;
    int seg = 0, nearest = -1;
    for (int k = 0; k < asize - 1; k++) {
        double dx = px - P[2 * k], dy = py - P[2 * k + 1];
        dist = dx * dx + dy * dy;
        if (dist < minDist) {
            nearest = k;
            minDist = dist;
            seg = k;
        }
    }
    if (nearest < 0) return 0;
    minDist = 1000000.0;
    for (int side = 0; side < 2; ++side) {
        int a, c;
        if (side == 0) {
            a = nearest;
            c = nearest + 1;
        } else {
            if (nearest == 0) nearest = asize - 1;
            a = nearest - 1;
            c = nearest;
        }
        double ux = P[2 * c] - P[2 * a], uy = P[2 * c + 1] - P[2 * a + 1];
        double lambda = (px - P[2 * a]) * ux + (py - P[2 * a + 1]) * uy;
        lambda /= (ux * ux + uy * uy);
        double dx, dy;
        if (lambda < 0) {
            dx = px - P[2 * a];
            dy = py - P[2 * a + 1];
        } else if (lambda > 1) {
            dx = P[2 * c] - px;
            dy = P[2 * c + 1] - py;
        } else {
            dx = px - (P[2 * a] + ux * lambda);
            dy = py - (P[2 * a + 1] + uy * lambda);
        }
        dist = dx * dx + dy * dy;
        if (dist < minDist) {
            seg = a;
            minDist = dist;
            lam = lambda;
        }
    }
    if (lam > 1) lam = 1;
    if (lam < 0) lam = 0;
    *out_lambda = lam;
    return seg;
}

int gg_or_contour(const double* phi, const int* box, const unsigned* idl, unsigned own, double* pts, int cap,
                  int* jtype, unsigned* jgrains, int* jseg, double* jlam, double* jxy, int jcap, int* njunc) {
    field f = {phi, box};
    const int w = bw(box);
    int n = 0, nj = 0;
    int startX = -1, startY = -1;
    for (int i = box[2]; i < box[3] && startX < 0; i++)
        for (int j = box[0]; j < box[1]; j++)
            if (inside(&f, i, j)) {
                startX = j;
                startY = i;
                break;
            }
    *njunc = 0;
    if (startX == -1) return 0;
    int left = startX - 1, right = startX, top = startY - 1, bottom = startY;
    int next = NONE, prev = NONE;
    long guard = 4L * (w + 2) * (bh(box) + 2) + 16;
    do {
        int mask = (inside(&f, top, left) ? TL : 0) | (inside(&f, top, right) ? TR : 0) |
                   (inside(&f, bottom, left) ? BL : 0) | (inside(&f, bottom, right) ? BR : 0);
        int emit = 1;
        switch (mask) {
            case TL: next = UP; break;
            case TR: next = RIGHT; break;
            case TL | TR: next = RIGHT; break;
            case BL: next = LEFT; break;
            case BL | TL: next = UP; break;
            case BL | TR: next = prev == UP ? RIGHT : LEFT; emit = 0; break;
            case BL | TR | TL: next = RIGHT; break;
            case BR: next = DOWN; break;
            case BR | TL: next = prev == RIGHT ? DOWN : UP; emit = 0; break;
            case BR | TR: next = DOWN; break;
            case BR | TR | TL: next = DOWN; break;
            case BR | BL: next = LEFT; break;
            case BR | BL | TL: next = UP; break;
            case BR | BL | TR: next = LEFT; break;
            default: emit = 0; break;
        }
        if (emit) { /* generatePoint (src/marchingSquares.cpp:204-265) */
            double x, y, delta;
            if (next == LEFT) {
                x = left;
                if (top < box[2]) {
                    y = bottom;
                } else {
                    delta = at(&f, bottom, left) - at(&f, top, left);
                    y = bottom - at(&f, bottom, left) / delta;
                }
            } else if (next == RIGHT) {
                x = right;
                if (bottom >= box[3]) {
                    y = top;
                } else {
                    delta = at(&f, top, right) - at(&f, bottom, right);
                    y = top + at(&f, top, right) / delta;
                }
            } else if (next == UP) {
                y = top;
                if (right >= box[1]) {
                    x = left;
                } else {
                    delta = at(&f, top, left) - at(&f, top, right);
                    x = left + at(&f, top, left) / delta;
                }
            } else {
                y = bottom;
                if (left < box[0]) {
                    x = right;
                } else {
                    delta = at(&f, bottom, right) - at(&f, bottom, left);
                    x = right - at(&f, bottom, right) / delta;
                }
            }
            if ((n == 0 || x != pts[2 * (n - 1)] || y != pts[2 * (n - 1) + 1]) && n < cap) { /* insertPoint */
                pts[2 * n] = x;
                pts[2 * n + 1] = y;
                n++;
            }
        }
        /* generateJunction (src/marchingSquares.cpp:266-301) */
        if (bottom >= box[2] && bottom < box[3] && top >= box[2] && top < box[3] && left >= box[0] &&
            left < box[1] && right >= box[0] && right < box[1]) {
            unsigned ids[4] = {0xFFFFFFu, 0xFFFFFFu, 0xFFFFFFu, 0xFFFFFFu}, v[4];
            int order = 0;
            v[0] = (mask & BL) ? own : idl[(long)(bottom - box[2]) * w + (left - box[0])];
            v[1] = (mask & TL) ? own : idl[(long)(top - box[2]) * w + (left - box[0])];
            v[2] = (mask & BR) ? own : idl[(long)(bottom - box[2]) * w + (right - box[0])];
            v[3] = (mask & TR) ? own : idl[(long)(top - box[2]) * w + (right - box[0])];
            for (int q = 0; q < 4; ++q) {
                int found = 0;
                for (int e = 0; e < order; ++e)
                    if (ids[e] == v[q]) found = 1;
                if (!found) ids[order++] = v[q];
            }
            if (order > 2 && nj < jcap) {
                jtype[nj] = order;
                for (int q = 0; q < 4; ++q) jgrains[4 * nj + q] = q < order ? ids[q] : 0xFFFFFFFFu;
                jxy[2 * nj] = left + 0.5;
                jxy[2 * nj + 1] = top + 0.5;
                nj++;
            }
        }
        if (next == UP) {
            top--;
            bottom--;
        } else if (next == DOWN) {
            top++;
            bottom++;
        } else if (next == LEFT) {
            left--;
            right--;
        } else if (next == RIGHT) {
            left++;
            right++;
        }
        prev = next;
    } while ((left != startX - 1 || bottom != startY) && --guard > 0);
    if (n > 0 && (pts[0] != pts[2 * (n - 1)] || pts[1] != pts[2 * (n - 1) + 1]) && n < cap) {
        pts[2 * n] = pts[0];
        pts[2 * n + 1] = pts[1];
        n++;
    }
    /* junctions projected onto the contour (src/grainBoundary.cpp:51-61) */
    double lambda = 0;
    for (int q = 0; q < nj && n >= 2; ++q) {
        int s = project(pts, n, jxy[2 * q], jxy[2 * q + 1], &lambda);
        int nx = (s + 1) % (n - 1);
        jxy[2 * q] = pts[2 * s] + (pts[2 * nx] - pts[2 * s]) * lambda;
        jxy[2 * q + 1] = pts[2 * s + 1] + (pts[2 * nx + 1] - pts[2 * s + 1]) * lambda;
        jseg[q] = s;
        jlam[q] = lambda;
    }
    *njunc = nj;
    return n;
}

double gg_or_area(const double* P, int n, double h) {
    double v = 0;
    for (int i = 0; i < n - 1; i++) v += (P[2 * i + 1] + P[2 * i + 3]) * (P[2 * i] - P[2 * i + 2]);
    return fabs(v) * h * h * 0.5;
}

double gg_or_perimeter(const double* P, int n, double h) {
    double p = 0;
    for (int i = 0; i < n - 1; i++) {
        double dx = P[2 * i] - P[2 * i + 2], dy = P[2 * i + 1] - P[2 * i + 3];
        p += sqrt(dx * dx + dy * dy) * h;
    }
    return p;
}

void gg_or_new_box(const int* nb, int m, int* out) {
    int x0 = nb[0] < 0 ? 0 : nb[0], x1 = nb[1] > m ? m : nb[1];
    int y0 = nb[2] < 0 ? 0 : nb[2], y1 = nb[3] > m ? m : nb[3];
    int gs = m - 1;
    unsigned height = y1 - y0, width = x1 - x0;
    if (width > height) {
        int d = width - height;
        y0 -= d / 2;
        y1 += d / 2 + d % 2;
    } else if (height > width) {
        int d = height - width;
        x0 -= d / 2;
        x1 += d / 2 + d % 2;
    }
    if (width != height) {
        if (x0 < 0) {
            x1 -= x0;
            x0 = 0;
        } else if (x1 > gs) {
            x0 += gs - x1;
            x1 = gs;
        }
        if (y0 < 0) {
            y1 -= y0;
            y0 = 0;
        } else if (y1 > gs) {
            y0 += gs - y1;
            y1 = gs;
        }
    }
    out[0] = x0;
    out[1] = x1;
    out[2] = y0;
    out[3] = y1;
}

/* ---- redistancing ------------------------------------------------------------ */

static int sgn(double v) { return (0.0 < v) - (v < 0.0); }

void gg_or_redistance(const double* in, const int* bi, double* out, const int* bo, double h, double delta) {
    const int wi = bw(bi), wo = bw(bo);
#define IN(i, j) in[(long)((i) - bi[2]) * wi + ((j) - bi[0])]
#define OUT(i, j) out[(long)((i) - bo[2]) * wo + ((j) - bo[0])]
    for (long p = 0; p < (long)wo * bh(bo); ++p) out[p] = -1.0;
    int ixmin = bi[0] < bo[0] ? bo[0] : bi[0], iymin = bi[2] < bo[2] ? bo[2] : bi[2];
    int ixmax = bi[1] < bo[1] ? bi[1] : bo[1], iymax = bi[3] < bo[3] ? bi[3] : bo[3];
    double cand, slope, dz;
    for (int j = ixmin; j < bo[1]; j++)
        for (int i = iymin; i < bo[3] - 1; i++) {
            if (j < ixmax && i < iymax - 1) {
                if (IN(i, j) * IN(i + 1, j) <= 0.0) {
                    slope = (IN(i + 1, j) - IN(i, j)) / h;
                    dz = -IN(i, j) / slope;
                    if (fabs(OUT(i, j)) > fabs(dz)) OUT(i, j) = -dz * sgn(slope);
                }
                cand = OUT(i, j) + (sgn(IN(i + 1, j)) * h);
            } else {
                cand = OUT(i, j) + (sgn(OUT(i + 1, j)) * h);
            }
            if (fabs(cand) < fabs(OUT(i + 1, j))) OUT(i + 1, j) = cand;
        }
    for (int j = ixmin; j < bo[1]; j++)
        for (int i = iymax - 1; i > bo[2]; i--) {
            if (j < ixmax && i > iymin)
                cand = OUT(i, j) + (sgn(IN(i - 1, j)) * h);
            else
                cand = OUT(i, j) + (sgn(OUT(i - 1, j)) * h);
            if (fabs(cand) < fabs(OUT(i - 1, j))) OUT(i - 1, j) = cand;
        }
    for (int i = iymin; i < bo[3]; i++)
        for (int j = ixmin; j < bo[1] - 1; j++) {
            if (j < ixmax - 1 && i < iymax) {
                if (IN(i, j) * IN(i, j + 1) <= 0.0) {
                    slope = (IN(i, j + 1) - IN(i, j)) / h;
                    dz = -IN(i, j) / slope;
                    if (fabs(OUT(i, j)) > fabs(dz)) OUT(i, j) = -dz * sgn(slope);
                }
                cand = OUT(i, j) + (sgn(IN(i, j + 1)) * h);
            } else {
                cand = OUT(i, j) + (sgn(OUT(i, j + 1)) * h);
            }
            if (fabs(cand) < fabs(OUT(i, j + 1))) OUT(i, j + 1) = cand;
        }
    for (int i = iymin; i < bo[3]; i++)
        for (int j = ixmax - 1; j > bo[0]; j--) {
            if (j > ixmin && i < iymax)
                cand = OUT(i, j) + (sgn(IN(i, j - 1)) * h);
            else
                cand = OUT(i, j) + sgn(OUT(i, j - 1)) * h;
            if (fabs(cand) < fabs(OUT(i, j - 1))) OUT(i, j - 1) = cand;
        }
    for (long p = 0; p < (long)wo * bh(bo); ++p) {
        if (out[p] < -delta)
            out[p] = -delta;
        else if (out[p] > delta)
            out[p] = delta;
    }
#undef IN
#undef OUT
}

/* LSbox::isMotionRegular (src/box.cpp:1156-1190): 1 regular, 0 irregular;
 * *flagged set when the grey zone lets the grain pass flagged. */
int gg_or_motion_regular(int old_contour, int new_contour, double old_volume, double new_volume, double dt,
                         int* flagged) {
    double mullins = (new_volume - old_volume) / dt * (3 / OR_PI);
    double contour_ratio = ((double)new_contour) / old_contour;
    double volume_ratio = new_volume / old_volume;
    *flagged = 0;
    if (mullins > -6.0) return 1;
    if (volume_ratio < 0.10) return 0;
    if (contour_ratio < 0.35) return 0;
    if (contour_ratio > 0.7) return 1;
    *flagged = 1;
    return 1;
}

/* ---- contour input ------------------------------------------------------------ */

void gg_or_polygon_phi(const double* pts, int n, const int* bo, int blowup, double h, double delta, double* out) {
    const int w = bo[1] - bo[0];
    for (int i = bo[2]; i < bo[3]; ++i)
        for (int j = bo[0]; j < bo[1]; ++j) {
            const double tx = (j - blowup) * h, ty = (i - blowup) * h;
            int inside = 0;
            for (int k = 1, l = 0; k < n; l = k++) {
                const double lx = pts[2 * l], ly = pts[2 * l + 1], kx = pts[2 * k], ky = pts[2 * k + 1];
                if (((ly > ty) != (ky > ty)) && (tx < (kx - lx) * (ty - ly) / (ky - ly) + lx)) inside = !inside;
            }
            double best = 1000000.0;
            for (int k = 1, l = 0; k < n; l = k++) {
                const double lx = pts[2 * l], ly = pts[2 * l + 1], kx = pts[2 * k], ky = pts[2 * k + 1];
                const double ux = kx - lx, uy = ky - ly;
                double lambda = (tx - lx) * ux + (ty - ly) * uy;
                lambda /= ux * ux + uy * uy;
                double d;
                if (lambda <= 0)
                    d = sqrt((tx - lx) * (tx - lx) + (ty - ly) * (ty - ly));
                else if (lambda >= 1)
                    d = sqrt((kx - tx) * (kx - tx) + (ky - ty) * (ky - ty));
                else {
                    const double fx = lx + ux * lambda, fy = ly + uy * lambda;
                    d = sqrt((tx - fx) * (tx - fx) + (ty - fy) * (ty - fy));
                }
                if (d < best) best = d; /* std::min(best, d): NaN leaves best */
            }
            if (best > delta) best = delta;
            out[(i - bo[2]) * w + (j - bo[0])] = inside ? best : -best;
        }
}

void gg_or_polygon_box(const double* pts, int n, int m, int blowup, double h, int* out) {
    int xmax = 0, xmin = m, ymax = 0, ymin = m;
    for (int k = 0; k < n; ++k) {
        const double x = pts[2 * k], y = pts[2 * k + 1];
        if (y / h < ymin) ymin = (int)(y / h);
        if (y / h > ymax) ymax = (int)(y / h);
        if (x / h < xmin) xmin = (int)(x / h);
        if (x / h > xmax) xmax = (int)(x / h);
    }
    xmax += 2 * blowup;
    ymax += 2 * blowup;
    if (ymax > m) ymax = m;
    if (xmax > m) xmax = m;
    out[0] = xmin;
    out[1] = xmax;
    out[2] = ymin;
    out[3] = ymax;
}

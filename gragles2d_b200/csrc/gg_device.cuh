// Device data model of the level-set network and the per-grain sequential
// routines shared by the plain (FP64) and batched (FP32) kernels.
//
// Data layout in HBM
//  - Each grain g (1..N; slot 0 is the domain-boundary grain) owns a square
//    box [x0,x1) x [y0,y1) in global grid coordinates (the reference's
//    DimensionalBuffer, src/dimensionalBuffer.h:34-211).  Its distance field
//    is stored row-major inside a flat arena at offset off[g]; offsets are a
//    device-side prefix sum over box areas, recomputed every step because
//    boxes move and change size every step (src/box.cpp:1146-1147).
//  - Two distance arenas ping-pong per step: A holds phi_t, then the
//    comparison result; B holds the convolution, then phi_{t+1}.
//  - IDLocal (nearest competing grain per pixel) lives in two u32 arenas with
//    the reference's resize-without-remap semantics (the linear buffer keeps
//    its prefix, src/dimensionalBuffer.h:108-115).
//  - Contours (x, y, energy, mobility per point, first point repeated at the
//    end) and junctions live in per-grain slots of two ping-pong arenas.
//  - Comparison / second-order / direct-neighbour lists are fixed-capacity
//    per-grain rows, in the reference's order.
#pragma once

#include <cstdint>

#ifndef GG_HD
#define GG_HD __host__ __device__ __forceinline__
#endif

namespace gg {

enum : int32_t { G_GONE = 0, G_EXISTS = 1, G_VANISHED = 2 };

enum : uint32_t {
    S_ARENA_FULL = 1u << 0,
    S_LIST_OVERFLOW = 1u << 1,
    S_CONTOUR_OVERFLOW = 1u << 2,
    S_JUNCTION_OVERFLOW = 1u << 3,
    S_WALK_LIMIT = 1u << 4,
    S_TABLE_RANGE = 1u << 5,
    S_NEIGHBOUR_OVERFLOW = 1u << 6,
    S_NAN = 1u << 7,
    S_INDEX = 1u << 8,
    S_SECTOR_GUARD = 1u << 9,   // a sector walk met a zero-length contour
    S_RETRY_LIMIT = 1u << 10    // more than 64 contour re-extractions
};

struct Box {
    int32_t x0, x1, y0, y1;  // [x0,x1) x [y0,y1): getMinX/getMaxX/getMinY/getMaxY
};

GG_HD int box_w(const Box& b) { return b.x1 - b.x0; }
GG_HD int box_h(const Box& b) { return b.y1 - b.y0; }
GG_HD int64_t box_area(const Box& b) { return (int64_t)(b.x1 - b.x0) * (int64_t)(b.y1 - b.y0); }

// DimensionalBuffer::getValueAt addressing (src/dimensionalBuffer.h:68-73):
// unsigned 32-bit arithmetic on (row - yMin) * width + (col - xMin), then a
// bounds check against the buffer length (std::vector::at).  An index left of
// the box therefore lands in the previous row, exactly as in the reference.
GG_HD bool buf_index(const Box& b, int row, int col, uint32_t* idx) {
    const uint32_t w = (uint32_t)(b.x1 - b.x0);
    const uint32_t k = ((uint32_t)row - (uint32_t)b.y0) * w + ((uint32_t)col - (uint32_t)b.x0);
    *idx = k;
    const int64_t size = box_area(b);
    return (int64_t)k < size;
}

GG_HD bool box_contains(const Box& b, int row, int col) {
    return row >= b.y0 && row < b.y1 && col >= b.x0 && col < b.x1;
}

template <typename T>
GG_HD int sgn(T v) {  // src/utilities.h:27-30
    return (T(0) < v) - (v < T(0));
}

struct CPoint {  // SPoint (src/spoint.h:29-87)
    double x, y, energy, mob;
};

struct Junction {  // GrainJunction (src/junction.h:45-67)
    int32_t type;  // 3 triple, 4 quadruple
    uint32_t grains[4];
    int32_t segment;
    double lambda;
    double x, y;
};

struct Neighbour {  // characteristics (src/charasteristic.h:29-62)
    int32_t id;
    int32_t pad;
    double length, energy, misori, mobility;
};

// Constant description of the network (passed by value to every kernel).
struct NetConst {
    int32_t N;       // grain slots: IDs 1..N (arrays sized N+1)
    int32_t m;       // ngridpoints = realDomainSize + 2 b
    int32_t b;       // grid_blowup (DomainBorderSize)
    int32_t nn;      // realDomainSize
    int32_t kmax;    // comparison / second-order list capacity
    int32_t nbmax;   // direct-neighbour list capacity
    int32_t jmax;    // junction slots per grain
    int32_t tmax;    // largest box edge with tables
    int32_t isotropic;
    int32_t use_mobility_model;
    int32_t analysis_timestep;
    int32_t decouple;
    // batched form's launch bins (autotuned, gg_autotune): boxes with an
    // edge above big_edge are redistanced by the large-box kernel; the
    // convolution keeps its row-pass intermediate in shared memory up to
    // conv_smem_edge
    int32_t big_edge;
    int32_t conv_smem_edge;
    double h, delta, dt;
    double csr, isr;  // sector radii (already scaled by h)
    double ds;        // (2 CSR + 2 ISR) / realDomainSize in grid points, src/grainhdl.cpp:81-82
    double tpd;       // TriplePointDrag
    double theta_ref, gamma_hagb, m_hagb;

    // per grain (fixed roles)
    int32_t* state;
    int32_t* regular;
    int32_t* inter_bnd;
    int32_t* newbb;  // 4 per grain: m_newXMin, m_newXMax, m_newYMin, m_newYMax
    double* volume;
    double* energy;
    double* perimeter;
    double* meanda;
    double* quat;    // 4 per grain (q0..q3); slot 0 = boundary (identity)
    int32_t* cmp_n;
    int32_t* cmp_ids;  // kmax per grain
    int32_t* sec_n;
    int32_t* sec_ids;
    int32_t* nb_n;
    Neighbour* nb;     // nbmax per grain
    int32_t* gone_loop;  // loop of the step whose level set deleted the grain, else -1
    double* stored;      // UseStoredElasticEnergy: scaled stored energy per grain, slot 0 = boundary (else null)
    double* magnetic;    // UseMagneticField: magnetic energy per grain, slot 0 = boundary (else null)
    double time_slope;   // GaussianKernelUserDefTimeSlope

    // tables (host-computed, libm on the host)
    const double* tw;        // twiddles exp(-2 pi i k / n), interleaved, at tw_off[n]
    const int64_t* tw_off;   // [tmax+1]
    const double* gk;        // Gaussian multipliers G(i2, j2) at gk_off[n], (n/2+1)^2 each
    const int64_t* gk_off;   // [tmax+1]
    const float* ck;         // separable real-space kernel per n at ck_off[n] (batched form)
    const int64_t* ck_off;
    void* ptinfo;            // per-contour-point probe scratch (contCur offsets), 32 bytes each
    double* dvol;            // tangent mode: d area / d p_k of the last level set, 4 per grain (else null)
    double* dseg;            // tangent mode: d segment length / d p_k, 4 per previous-contour point (scratch)
    // batched form: sectors built one step ahead for the corrector (k_sectors):
    // one SectorPack per grain, and per contour point (at the contour's
    // offsets) the sector of the segment starting there and, for an
    // interpolating sector, the arc length from the sector's right end
    void* secpack;
    int16_t* segsec;
    float* segacc;
};

// Per-step rotating state, resident in device memory (kernels read it
// through a pointer; a one-thread kernel rotates the roles at the end of a
// step, so a captured graph of one step can be replayed step after step).
struct NetState {
    Box* box_prev;  // IDLocal box before the convolution-stage resize
    Box* box_cur;   // box of phi_t / convolution / comparison
    Box* box_new;   // box of phi_{t+1}
    int64_t* off_prev;
    int64_t* off_cur;
    int64_t* off_new;
    int64_t* soff_cur;  // spectral scratch offsets (plain convolution)
    int64_t* soff_new;
    void* phiA;
    void* phiB;
    uint32_t* idPrev;
    uint32_t* idCur;
    CPoint* contPrev;
    CPoint* contCur;
    int64_t* coff_prev;
    int64_t* coff_cur;
    int64_t* coff_new;
    int32_t* ccap_prev;
    int32_t* ccap_cur;
    int32_t* ccap_new;
    int32_t* cn_prev;
    int32_t* cn_cur;
    double* segPrev;     // per-contour-point segment lengths (corrector scratch, contPrev offsets)
    Junction* jPrev;
    Junction* jCur;
    int32_t* jn_prev;
    int32_t* jn_cur;
    void* spec;          // spectral scratch arena (plain convolution)
    int64_t phi_cap;     // elements per distance arena
    int64_t spec_cap;    // elements of spec
    int64_t cont_cap;    // points per contour arena
    int64_t phi_used;
    int64_t spec_used;
    int64_t cont_used;
    int32_t loop;
    uint32_t status;
    int32_t live;        // grains not removed (grainhdl::currentNrGrains)
    int32_t n_big;       // entries of big_list
    double max_volume;
    unsigned long long updates;   // sum over steps of grains alive at step start
    unsigned long long t_area;    // traffic model scratch (k_traffic)
    unsigned long long t_overlap;
    unsigned long long t_exists;
    // tangent fields d phi / d p_k of the four calibration parameters (plain
    // form only; null unless enabled): 4 x phi_cap doubles each, parameter k
    // at offset k * phi_cap, same per-grain offsets as phiA / phiB
    void* dphiA;
    void* dphiB;
    // tangents of the contour points (8 doubles per point: dx / dp_k, then
    // dy / dp_k), same offsets and rotation as contPrev / contCur
    double* dcontPrev;
    double* dcontCur;
    // batched form: the per-grain launches' work queue, grain IDs by
    // descending box edge (rebuilt after every change of the boxes); null in
    // the plain form, whose launches take grains in ID order
    int32_t* order;
    // batched form: grains whose previous contour is longer than the main
    // corrector stages (kCorrStagedPts), flagged per grain and listed
    // (n_big entries) for the large-contour corrector; rebuilt with the work
    // queue, so each grain has exactly one corrector launch
    int32_t* big_flag;
    int32_t* big_list;
};

// The initial neighbour search's grid of grain bins (kNeighbourBin cells a
// side, nc x nc of them): counts, starts (nc * nc + 1) and the binned grain
// IDs, with the total written back for the host to size `items`.
constexpr int kNeighbourBin = 64;
struct NeighbourBins {
    int nc;
    int* count;
    int* start;
    int* items;
    int* total;
};

// Contour points the main batched corrector stages in shared memory; longer
// contours go to the large-contour corrector.
constexpr int kCorrStagedPts = 512;

// The grain that work slot `slot` (0-based, < N) of a per-grain launch
// processes: largest boxes first when the queue exists, else ID order.  Every
// per-grain kernel writes only its own grain's outputs, so the order changes
// when a grain runs, never what it computes.
GG_HD int grain_at(const NetState* S, int slot) { return S->order ? S->order[slot] : slot + 1; }

GG_HD void set_status(NetState* S, uint32_t bits) {
#ifdef __CUDA_ARCH__
    atomicOr(&S->status, bits);
#else
    S->status |= bits;
#endif
}

GG_HD int contour_capacity(int n) { return 8 * n + 64; }

// Arena offsets are only valid while no allocation overflowed; every kernel
// that addresses an arena returns early once this bit is set.
GG_HD bool halted(const NetState* S) { return (S->status & S_ARENA_FULL) != 0; }

}  // namespace gg

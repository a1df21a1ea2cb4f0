/*
 * Oracle harness around GraGLeS2D's own C++ (test infrastructure only; it
 * is never linked into the product and only tests, smoke() and bench.py's
 * reference/CPU arms run it).
 *
 * It links the reference sources where they lie (compiled by
 * oracle/Makefile with the FFTW / libnuma / voro++ shims in oracle/shim)
 * and replaces the reference's main (src/ggLS.cpp:24-61) with a driver
 * that
 *   - reads parameters.xml through Settings::initializeParameters
 *     (src/Settings.cpp:84-289);
 *   - builds grainhdl in zeroed storage, so the member the reference never
 *     initialises without a magnetic field (m_Energy_deltaMAX,
 *     src/grainhdl.h:53, used by src/grainhdl.cpp:250-274) reads 0 and dt
 *     keeps its documented value;
 *   - runs run_sim's prologue and loop body (src/grainhdl.cpp:1035-1142)
 *     stage by stage, skipping the analysis file writers (save_Texture /
 *     save_NetworkPlot / save_NrGrainsStats / restart files), which change
 *     no grain state, unless an analysis directory is given: then
 *     save_Texture, save_NrGrainsStats and save_Full_Microstructure_for_Restart
 *     run on the reference's schedule (src/grainhdl.cpp:1098-1112) with that
 *     directory as the working directory;
 *   - writes a binary dump of every LSbox after initialisation and after
 *     chosen steps (format below), and the loop's wall time.
 *
 * Usage: gg_ref <parameters.xml> <dump.bin|-> [dump_every] [quiet] [analysis_dir]
 *   dump_every = k > 0 dumps after every k-th step (and after init);
 *   0 dumps only the initial and final states.
 *
 * Dump format (little endian):
 *   "GGD1", i32 version=1, i32 N, i32 ngridpoints, i32 realDomainSize,
 *   f64 h, f64 delta, f64 dt, then records.  Each record: i32 tag=0x52454344,
 *   i32 loop (steps completed), i32 n_grains_alive, then for id = 1..N:
 *     i32 id, i32 state (0 gone, 1 exists, 2 marked not existing),
 *     i32 motion_regular, i32 intersects_boundary,
 *     f64 volume, energy, perimeter, meanDa,
 *     box phi  (i32 xmin,xmax,ymin,ymax) + f64 values (current phi = out),
 *     box IDLocal (4 x i32) + u32 values,
 *     i32 nCmp + i32 ids, i32 nSec + i32 ids,
 *     i32 nContour + 4 f64 each (x, y, energy, mob),
 *     i32 nJunction + (i32 type, 4 x u32 grains, i32 segment, f64 lambda,
 *                      f64 x, f64 y) each,
 *     i32 nNeighbour + (i32 id, f64 length, f64 energy, f64 misori,
 *                       f64 mobility) each,
 *     i32 newXMin, newXMax, newYMin, newYMax.
 */
#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <iterator>
#include <limits>
#include <list>
#include <map>
#include <memory>
#include <new>
#include <numeric>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>
#include <omp.h>
#include <sched.h>
#include <sys/time.h>
#include <unistd.h>

// Test-only access to the reference's private/protected state for dumping.
// Every standard header is included above, so only the reference's own
// declarations are affected; object layout is unchanged.
#define private public
#define protected public
#include "ggLS.h"
#include "Settings.h"
#include "box.h"
#include "grainhdl.h"
#undef private
#undef protected

namespace {

double now_s() {
    timeval t;
    gettimeofday(&t, nullptr);
    return t.tv_sec + t.tv_usec * 1e-6;
}

struct Writer {
    FILE* f = nullptr;
    void i32(int32_t v) { fwrite(&v, 4, 1, f); }
    void u32(uint32_t v) { fwrite(&v, 4, 1, f); }
    void f64(double v) { fwrite(&v, 8, 1, f); }
};

void dump_state(Writer& w, grainhdl* sim, int steps_done) {
    w.i32(0x52454344);
    w.i32(steps_done);
    w.i32((int32_t)sim->currentNrGrains);
    const int N = (int)Settings::NumberOfParticles;
    for (int id = 1; id <= N; ++id) {
        LSbox* g = (id < (int)sim->grains.size()) ? sim->grains[id] : nullptr;
        w.i32(id);
        if (!g) {
            w.i32(0);
            continue;
        }
        w.i32(g->m_exists ? 1 : 2);
        w.i32(g->m_isMotionRegular ? 1 : 0);
        w.i32(g->m_intersectsBoundaryGrain ? 1 : 0);
        w.f64(g->m_volume);
        w.f64(g->m_energy);
        w.f64(g->m_perimeter);
        w.f64(g->m_meanDa);
        DimensionalBufferReal* phi = g->m_outputDistance;
        w.i32(phi->getMinX());
        w.i32(phi->getMaxX());
        w.i32(phi->getMinY());
        w.i32(phi->getMaxY());
        const size_t nphi = (size_t)(phi->getMaxX() - phi->getMinX()) * (phi->getMaxY() - phi->getMinY());
        for (size_t k = 0; k < nphi; ++k) w.f64(phi->m_values[k]);
        DimensionalBufferIDLocal& idl = g->m_IDLocal;
        w.i32(idl.getMinX());
        w.i32(idl.getMaxX());
        w.i32(idl.getMinY());
        w.i32(idl.getMaxY());
        const size_t nid = (size_t)(idl.getMaxX() - idl.getMinX()) * (idl.getMaxY() - idl.getMinY());
        for (size_t k = 0; k < nid; ++k) w.u32(k < idl.m_values.size() ? idl.m_values[k].grainID : 0xFFFFFFFFu);
        w.i32((int32_t)g->m_comparisonList.size());
        for (LSbox* b : g->m_comparisonList) w.i32((int32_t)b->getID());
        w.i32((int32_t)g->m_secondOrderNeighbours.size());
        for (LSbox* b : g->m_secondOrderNeighbours) w.i32((int32_t)b->getID());
        std::vector<SPoint>& contour = g->m_grainBoundary.m_grainBoundary;
        w.i32((int32_t)contour.size());
        for (const SPoint& p : contour) {
            w.f64(p.x);
            w.f64(p.y);
            w.f64(p.energy);
            w.f64(p.mob);
        }
        std::vector<GrainJunction>& js = g->m_grainBoundary.m_grainJunctions;
        w.i32((int32_t)js.size());
        for (const GrainJunction& j : js) {
            w.i32((int32_t)j.junction_type);
            for (int q = 0; q < 4; ++q) w.u32(q < (int)j.junction_type ? j.grains[q] : 0xFFFFFFFFu);
            w.i32(j.contourSegment);
            w.f64(j.lambda);
            w.f64(j.coordinates.x);
            w.f64(j.coordinates.y);
        }
        std::vector<characteristics>& nb = g->m_grainBoundary.m_directNeighbourhood;
        w.i32((int32_t)nb.size());
        for (const characteristics& c : nb) {
            w.i32(c.directNeighbour ? (int32_t)c.directNeighbour->getID() : -1);
            w.f64(c.length);
            w.f64(c.energyDensity);
            w.f64(c.mis_ori);
            w.f64(c.mobility);
        }
        w.i32(g->m_newXMin);
        w.i32(g->m_newXMax);
        w.i32(g->m_newYMin);
        w.i32(g->m_newYMax);
    }
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s parameters.xml dump.bin|- [dump_every] [quiet]\n", argv[0]);
        return 2;
    }
    const std::string dump_path = argv[2];
    const int dump_every = argc > 3 ? std::atoi(argv[3]) : 0;
    const bool quiet = argc > 4 && std::atoi(argv[4]) != 0;
    const char* analysis_dir = argc > 5 ? argv[5] : nullptr;

    std::streambuf* saved = nullptr;
    std::ofstream devnull;
    if (quiet) {
        devnull.open("/dev/null");
        saved = std::cout.rdbuf(devnull.rdbuf());
    }

    Settings::initializeParameters(argv[1]);
    void* storage = std::calloc(1, sizeof(grainhdl));
    grainhdl* sim = new (storage) grainhdl();
    sim->setResearchAdjustments(Settings::ResearchProject);
    sim->setSimulationParameter();

    Writer w;
    if (dump_path != "-") {
        w.f = std::fopen(dump_path.c_str(), "wb");
        if (!w.f) {
            std::fprintf(stderr, "cannot open %s\n", dump_path.c_str());
            return 2;
        }
        std::fwrite("GGD1", 1, 4, w.f);
        w.i32(1);
        w.i32((int32_t)Settings::NumberOfParticles);
        w.i32(sim->get_ngridpoints());
        w.i32(sim->get_realDomainSize());
        w.f64(sim->get_h());
        w.f64(sim->delta);
        w.f64(sim->get_dt());
    }

    if (analysis_dir && chdir(analysis_dir) != 0) {
        std::fprintf(stderr, "cannot enter %s\n", analysis_dir);
        return 2;
    }

    // run_sim prologue (src/grainhdl.cpp:1041-1048)
    const double t_init0 = now_s();
    sim->distanceInitialisation();
    sim->get_biggestGrainVol();
    sim->Realtime = 0.0;
    sim->find_neighbors();
    const double t_init = now_s() - t_init0;
    if (w.f) dump_state(w, sim, 0);

    // run_sim loop body (src/grainhdl.cpp:1049-1142)
    double t_loop = 0.0;
    unsigned long grain_updates = 0;
    int steps = 0;
    std::vector<double> step_s;
    std::vector<unsigned> step_grains;
    for (sim->loop = Settings::StartTime; sim->loop <= Settings::StartTime + Settings::NumberOfTimesteps;
         sim->loop++) {
        const double t0 = now_s();
        grain_updates += sim->currentNrGrains;
        step_grains.push_back(sim->currentNrGrains);
        double overhead = 0;
        sim->gridCoarsement();
        sim->convolution(overhead);
        sim->switchDistancebuffer();
        sim->updateSecondOrderNeighbors();
        if (Settings::DecoupleGrains != 1) {
            sim->comparison_box();
            sim->switchDistancebuffer();
        } else {
            sim->tweakIDLocal();
        }
        sim->level_set();
        sim->redistancing();
        if (analysis_dir && (((sim->loop - Settings::StartTime) % int(Settings::AnalysisTimestep)) == 0 ||
                             sim->loop == Settings::NumberOfTimesteps)) {
            sim->save_Texture();
            sim->save_NrGrainsStats();
            if ((Settings::MicrostructureGenMode == E_READ_VOXELIZED_MICROSTRUCTURE && sim->loop == 0) ||
                sim->loop == Settings::NumberOfTimesteps)
                sim->save_Full_Microstructure_for_Restart();
        }
        sim->Realtime += (sim->get_dt() * (Settings::Physical_Domain_Size * Settings::Physical_Domain_Size) /
                          (sim->TimeSlope * Settings::HAGB_Energy * Settings::HAGB_Mobility));
        sim->get_biggestGrainVol();
        step_s.push_back(now_s() - t0);
        t_loop += step_s.back();
        ++steps;
        const bool last = sim->loop == Settings::StartTime + Settings::NumberOfTimesteps;
        const bool brk = sim->currentNrGrains < Settings::BreakupNumber;
        if (w.f && ((dump_every > 0 && steps % dump_every == 0) || last || brk)) dump_state(w, sim, steps);
        if (brk) break;
    }
    if (w.f) std::fclose(w.f);
    if (quiet) std::cout.rdbuf(saved);
    std::printf("{\"steps\": %d, \"grain_updates\": %lu, \"loop_s\": %.6f, \"init_s\": %.6f, \"threads\": %d, "
                "\"grains_left\": %u, \"step_s\": [",
                steps, grain_updates, t_loop, t_init, omp_get_max_threads(), sim->currentNrGrains);
    for (size_t k = 0; k < step_s.size(); ++k) std::printf("%s%.6f", k ? ", " : "", step_s[k]);
    std::printf("], \"step_grains\": [");
    for (size_t k = 0; k < step_grains.size(); ++k) std::printf("%s%u", k ? ", " : "", step_grains[k]);
    std::printf("]}\n");
    return 0;
}

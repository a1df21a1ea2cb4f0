/*
 * Test-infrastructure shim (oracle only).  GraGLeS2D's Voronoi generator
 * (src/grainhdl.cpp:513-603, microstructure mode 1) links a prebuilt voro++
 * archive that is not built from source here.  The oracle always reads
 * mode-4 voxel input (src/grainhdl.cpp:336-511), so the voro++ symbols are
 * bound (linker --defsym, see oracle/Makefile) to this function, which
 * aborts if the Voronoi path is ever reached.
 */
#include <stdio.h>
#include <stdlib.h>

void gg_voro_unavailable(void) {
    fprintf(stderr, "oracle: voro++ is not available; use MicrostructureGenMode 4\n");
    abort();
}

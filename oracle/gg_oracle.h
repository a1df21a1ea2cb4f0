/*
 * CPU restatement of GraGLeS2D's per-grain level-set routines (test
 * infrastructure only: tests and bench.py's CPU arm may call it; the product
 * never links it).  Plain C, FP64, no FMA contraction, each function
 * following the reference routine cited beside it operation for operation.
 *
 * Boxes are int[4] = {xmin, xmax, ymin, ymax} in global grid coordinates,
 * fields row-major over the box.  Parity of this restatement is pinned
 * against dumps of the reference's own run (tests/test_oracle_port.py).
 */
#ifndef GG_ORACLE_H
#define GG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* LSbox::convolutionGeneratorFFTW, Gaussian mode (src/box.cpp:622-695), with
 * the FFTW transforms as the separable direct DFTs of oracle/shim/fft_shim.c. */
void gg_or_convolve(int n, const double* in, double* out, double dt, int real_domain_size);

/* LSbox::executeComparison + boundaryCondition + executeSetComparison
 * (src/box.cpp:890-1025, 838-879) for one grain.  nbr_conv[k] is the
 * convolved field of list member k over nbr_box[4k..4k+3]; idprev is the
 * IDLocal buffer of the previous box (keep-prefix resize,
 * src/dimensionalBuffer.h:108-115).  Outputs the compared field, IDLocal and
 * the unclipped new bounding box. */
void gg_or_compare(const int* box, const double* own_conv, int nlist, const int* nbr_box,
                   const double* const* nbr_conv, const unsigned* nbr_id, const int* prev_box,
                   const unsigned* idprev, int m, int b, double h, double delta, double* cmp_out,
                   unsigned* id_out, int* newbb);

/* MarchingSquaresAlgorithm::generateContour (src/marchingSquares.cpp:28-301)
 * with the junction projection of extractBoundaryAndJunctions
 * (src/grainBoundary.cpp:51-61).  Returns the number of contour points
 * written to pts (x, y pairs; 0 if no pixel has phi >= 0); junctions go to
 * jtype, jgrains (4 each), jseg, jlam, jxy (x, y). */
int gg_or_contour(const double* phi, const int* box, const unsigned* idl, unsigned own, double* pts, int cap,
                  int* jtype, unsigned* jgrains, int* jseg, double* jlam, double* jxy, int jcap, int* njunc);

/* ExplicitGrainBoundary::computeVolume / computePerimeter
 * (src/grainBoundary.cpp:201-213, 224-231). */
double gg_or_area(const double* pts, int n, double h);
double gg_or_perimeter(const double* pts, int n, double h);

/* LSbox::isMotionRegular (src/box.cpp:1156-1190): returns 1 when the motion
 * is regular (or passes flagged: *flagged = 1), 0 when the contour must be
 * re-extracted. */
int gg_or_motion_regular(int old_contour, int new_contour, double old_volume, double new_volume, double dt,
                         int* flagged);

/* The new box of LSbox::extractContour (src/box.cpp:1118-1148): clip the
 * set-comparison bounding box to the grid and make it square
 * (DimensionalBuffer::resizeToSquare, src/dimensionalBuffer.h:123-160). */
void gg_or_new_box(const int* newbb, int m, int* out);

/* LSbox::executeRedistancing (src/box.cpp:1259-1399). */
void gg_or_redistance(const double* in, const int* bi, double* out, const int* bo, double h, double delta);

/* LSbox::calculateDistanceFunction for contour input (src/box.cpp:342-400):
 * the signed distance of every pixel of box `bo` (xmin, xmax, ymin, ymax) to
 * the polygon pts[2k], pts[2k+1] (k < n, domain coordinates), clamped to
 * delta, positive inside by the crossing-number test. */
void gg_or_polygon_phi(const double* pts, int n, const int* bo, int blowup, double h, double delta, double* out);

/* The box of the contour constructor (src/box.cpp:108-159) before it is made
 * square: out = xmin, xmax, ymin, ymax. */
void gg_or_polygon_box(const double* pts, int n, int m, int blowup, double h, int* out);

#ifdef __cplusplus
}
#endif

#endif

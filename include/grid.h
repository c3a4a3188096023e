/* grid.h — square velocity grids (real/complex, N x N and padded 2N x 2N).
 *
 * Same types and entry points as the upstream include/grid.h:34-104 so that
 * callers compiled against the upstream headers link against libqbgpu.
 * Differences, all source compatible:
 *   - N_GRID may be set by the build (-DN_GRID=...); the default is the
 *     upstream value 32 (include/grid.h:34).  The library is built once per
 *     N_GRID because every grid type below has a compile-time size.
 *   - restrict_ falls back to __restrict__ when the includer does not define
 *     it (upstream callers pass -Drestrict_=__restrict__, bin/makefile:12).
 *
 * Index convention (upstream src/quadrature.c:186-187): element (l, k) of an
 * N x N grid is data[k + N*l]; l is the slow (v_x / first Fourier) index.
 */
#ifndef GRID_H
#define GRID_H

#include <fftw3.h>

#ifndef restrict_
#define restrict_ __restrict__
#endif

#ifndef N_GRID
#define N_GRID 32                   /* grid points per direction */
#endif
#define N_MASK (N_GRID - 1)          /* modulo-N mask; N must be a power of 2 */

#ifdef __cplusplus
extern "C" {
#endif

/* real N x N grid (upstream grid.h:42-47) */
typedef struct { double data[N_GRID*N_GRID]; } grid_t;

/* real 2N x 2N grid (upstream grid.h:53-58) */
typedef struct { double data[4*N_GRID*N_GRID]; } grid2_t;

/* complex N x N grid (upstream grid.h:64-69) */
typedef struct { fftw_complex data[N_GRID*N_GRID]; } cgrid_t;

/* complex 2N x 2N grid (upstream grid.h:75-80) */
typedef struct { fftw_complex data[4*N_GRID*N_GRID]; } cgrid2_t;

/* Pointwise products (upstream src/grid.c:33-164). */
void MultiplyPointwiseRR (const   grid_t *restrict_ f, const   grid_t *restrict_ g,   grid_t *restrict_ ret);
void MultiplyPointwiseRC (const   grid_t *restrict_ f, const  cgrid_t *restrict_ g,  cgrid_t *restrict_ ret);
void MultiplyPointwiseCC (const  cgrid_t *restrict_ f, const  cgrid_t *restrict_ g,  cgrid_t *restrict_ ret);
void MultiplyPointwiseRR2(const  grid2_t *restrict_ f, const  grid2_t *restrict_ g,  grid2_t *restrict_ ret);
void MultiplyPointwiseCC2(const cgrid2_t *restrict_ f, const cgrid2_t *restrict_ g, cgrid2_t *restrict_ ret);

void MultiplyPointwiseAssignRR (const   grid_t *restrict_ f,   grid_t *restrict_ ret);
void MultiplyPointwiseAssignRC (const   grid_t *restrict_ f,  cgrid_t *restrict_ ret);
void MultiplyPointwiseAssignRC2(const  grid2_t *restrict_ f, cgrid2_t *restrict_ ret);
void MultiplyPointwiseAssignCC2(const cgrid2_t *restrict_ f, cgrid2_t *restrict_ ret);

/* Embed an FFT-ordered N x N grid in the corner quadrants of a zeroed 2N x 2N
 * grid, and the inverse (upstream src/grid.c:171-210). */
void GridZeroPad(const cgrid_t *restrict_ f, cgrid2_t *restrict_ ret);
void GridExtract(const cgrid2_t *restrict_ f, cgrid_t *restrict_ ret);

#ifdef __cplusplus
}
#endif

#endif /* GRID_H */

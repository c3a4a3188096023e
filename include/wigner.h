/* wigner.h — Wigner state of a spin-1/2 particle in the Pauli basis.
 *
 * Same layout as upstream include/wigner.h:35-50: four components
 * (trace, sigma_x, sigma_y, sigma_z), each an N x N grid.  In velocity space
 * the components are real and the velocities along each axis are
 * [0:N/2-1, -N/2:-1] * (2L)/N; in Fourier space they are complex.
 */
#ifndef WIGNER_H
#define WIGNER_H

#include "grid.h"

/* velocity-space state (upstream wigner.h:35-39) */
typedef struct { grid_t comp[4]; } wignerV_t;

/* Fourier-space state (upstream wigner.h:46-50) */
typedef struct { cgrid_t comp[4]; } wignerF_t;

#endif /* WIGNER_H */

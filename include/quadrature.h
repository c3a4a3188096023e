/* quadrature.h — quadrature tables for the I1..I4 collision integrals.
 *
 * Same structs and entry points as upstream include/quadrature.h:35-97.
 * The tables live in caller-visible host memory exactly as upstream
 * (psiR1/psiR2 arrays of num grids).  libqbgpu builds them on the GPU,
 * copies them into these host arrays, and keeps a compact device copy keyed
 * by the psiR1 pointer until QuadI*_Delete (tables built by Fourier*() are
 * treated as read-only by the caller, as they are upstream).
 */
#ifndef QUADRATURE_H
#define QUADRATURE_H

#include "grid.h"

#ifdef __cplusplus
extern "C" {
#endif

/* I1 / I4 quadrature (upstream quadrature.h:35-43) */
typedef struct
{
	unsigned int num;   /* number of terms */
	grid2_t *psiR1;     /* num real 2N x 2N grids */
	grid_t  *psiR2;     /* num real  N x  N grids */
}
quadI1_t;

void QuadI1_Allocate(const unsigned int num, quadI1_t *quad);
void QuadI1_Delete(quadI1_t *quad);

/* I2 quadrature (upstream quadrature.h:52-60) */
typedef struct
{
	unsigned int num;
	grid_t *psiR1;      /* num real N x N grids */
	grid_t *psiR2;      /* num real N x N grids */
}
quadI2_t;

void QuadI2_Allocate(const unsigned int J, quadI2_t *quad);
void QuadI2_Delete(quadI2_t *quad);

/* I3 quadrature (upstream quadrature.h:69-77) */
typedef struct
{
	unsigned int num;   /* J*M terms */
	cgrid_t *psiR1;     /* num complex N x N grids (plane waves) */
	grid2_t *psiR2;     /* num real 2N x 2N grids */
}
quadI3_t;

void QuadI3_Allocate(const unsigned int num, quadI3_t *quad);
void QuadI3_Delete(quadI3_t *quad);

/* Table builders (upstream src/quadrature.c:150,245,395,473). */
void FourierI1(const unsigned int J, const double L, const double R, quadI1_t *quad);
void FourierI2(const unsigned int J, const double L, const double R, quadI2_t *quad);
void FourierI3(const unsigned int J, const double L, const double R, const unsigned int M, quadI3_t *quad);
void FourierI4(const unsigned int J, const double L, const double R, quadI1_t *quad);

/* Legendre-Gauss nodes and weights on [a,b] (upstream src/quadrature.c:293);
 * not in the upstream header, but declared by test/lgwt_test.c:37. */
void LegendreGaussQuad(const unsigned int M, const double a, const double b, double *x, double *w);

#ifdef __cplusplus
}
#endif

#endif /* QUADRATURE_H */

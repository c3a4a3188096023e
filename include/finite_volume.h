/* finite_volume.h — minmod slope-limiter transport steps in one dimension.
 *
 * Entry points as upstream include/finite_volume.h:29-41 (src/finite_volume.c:52-323):
 * one step of u_t + A u_x = 0 with the slope-limiter scheme of LeVeque (1992),
 * Eq. (16.57), for periodic, Dirichlet and Maxwell-reflection boundaries.
 * Every step is evaluated on the GPU; for a single line the call uploads the
 * line, runs the stencil kernel and downloads the result.  The floating-point
 * operation order matches upstream without fused multiply-adds, so results
 * are bit-identical to upstream's IEEE double arithmetic.
 */
#ifndef FINITE_VOLUME_H
#define FINITE_VOLUME_H

#ifndef restrict_
#define restrict_ __restrict__
#endif

#ifdef __cplusplus
extern "C" {
#endif

void SlopeLimiterStepPeriodic(const double h, const double dt, const double A, const unsigned int N, const double *restrict_ Un, double *restrict_ Un1);

void SlopeLimiterStepDirichlet(const double h, const double dt, const double A, const unsigned int N, const double *restrict_ Un, double *restrict_ Un1);

double CalculateRightwardFlux(const unsigned int m, const double *restrict_ A, const double *restrict_ U);

double CalculateLeftwardFlux(const unsigned int m, const double *restrict_ A, const double *restrict_ U);

void SlopeLimiterStepMaxwell(const double h, const double dt, const unsigned int m, const double *restrict_ A, const unsigned int N,
	const double lambda, const double fluxL, const double fluxR, const double *restrict_ UmaxwL, const double *restrict_ UmaxwR, const double *restrict_ Un, double *restrict_ Un1);

#ifdef __cplusplus
}
#endif

#endif /* FINITE_VOLUME_H */

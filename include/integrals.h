/* integrals.h — the I1 (and I4), I2 and I3 collision integrals.
 *
 * Entry points and argument meaning as upstream include/integrals.h:56-138:
 *   I1 = (1/(4N^2))^2 sum_j Extract(IFFT(h^ . FFT(psiR1_j . IFFT(f^ . FFT(Pad(psiR2_j . g))))))
 *   I2 = (1/(4N^2))   sum_j Extract(IFFT(FFT(Pad(psiR1_j f)) . FFT(Pad(psiR2_j g)) . h^))
 *   I3 = (1/(4N^2))^2 sum_j Extract(IFFT(FFT(Pad(psiR1_j f)) . FFT(psiR2_j . IFFT(g^ . FFT(Pad(psiR1_j h))))))
 * with x^ = FFT(Pad(x)) on the 2N x 2N grid (upstream src/integrals.c:90-379).
 *
 * The intermediate structs keep their upstream names and remain complete
 * types, but their contents differ: upstream holds FFTW plans and host
 * scratch grids (integrals.h:36-51,88-112); here each holds a handle to a
 * GPU workspace (device scratch, stream) created by *_Create and released by
 * *_Delete.  Callers only ever pass their address, so this is source
 * compatible.  Each call copies its inputs to the GPU, evaluates there and
 * copies the result back; the call returns after the result is on the host.
 */
#ifndef INTEGRALS_H
#define INTEGRALS_H

#include "grid.h"
#include "quadrature.h"

#ifdef __cplusplus
extern "C" {
#endif

struct qb_workspace;

typedef struct { struct qb_workspace *ws; } I1interm_t;
typedef struct { struct qb_workspace *ws; } I2interm_t;
typedef struct { struct qb_workspace *ws; } I3interm_t;

void I1interm_Create(I1interm_t *interm);
void I1interm_Delete(I1interm_t *interm);
void I1integral(const cgrid_t *restrict_ f, const cgrid_t *restrict_ g, const cgrid_t *restrict_ h, const quadI1_t *restrict_ quad, I1interm_t *restrict_ interm, cgrid_t *restrict_ I1);

void I2interm_Create(I2interm_t *interm);
void I2interm_Delete(I2interm_t *interm);
void I2integral(const cgrid_t *restrict_ f, const cgrid_t *restrict_ g, const cgrid_t *restrict_ h, const quadI2_t *restrict_ quad, I2interm_t *restrict_ interm, cgrid_t *restrict_ I2);

void I3interm_Create(I3interm_t *interm);
void I3interm_Delete(I3interm_t *interm);
void I3integral(const cgrid_t *restrict_ f, const cgrid_t *restrict_ g, const cgrid_t *restrict_ h, const quadI3_t *restrict_ quad, I3interm_t *restrict_ interm, cgrid_t *restrict_ I3);

#ifdef __cplusplus
}
#endif

#endif /* INTEGRALS_H */

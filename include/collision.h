/* collision.h — conservative (Cc) and dissipative (Cd) collision operators.
 *
 * Entry points as upstream include/collision.h:46-73 (src/collision.c:74,209):
 *   Cc[W]: cross-product terms built from 6 I1 integrals; Cc_0 = 0.
 *   Cd[W]: 16 I2, 16 I3 and 12 I4 integrals combined with eta = diag(1,-1,-1,-1).
 * W and the results are Fourier-space Wigner states (wignerF_t).
 *
 * CdInterm_t / CcInterm_t hold a GPU workspace handle instead of the upstream
 * nested FFTW scratch (collision.h:36-42,56-62); callers only pass their
 * address.  On the GPU the integrals are evaluated in factored form (sums
 * over quadrature terms moved inside the outer FFTs, shared transforms
 * computed once); results agree with the upstream loop order to rounding.
 */
#ifndef COLLISION_H
#define COLLISION_H

#include "integrals.h"
#include "wigner.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { struct qb_workspace *ws; } CdInterm_t;

void CdInterm_Create(CdInterm_t *interm);
void CdInterm_Delete(CdInterm_t *interm);
void CdInt(const wignerF_t *restrict_ W, const quadI2_t *restrict_ quadI2, const quadI3_t *restrict_ quadI3, const quadI1_t *restrict_ quadI4, CdInterm_t *restrict_ interm, wignerF_t *restrict_ Cd);

typedef struct { struct qb_workspace *ws; } CcInterm_t;

void CcInterm_Create(CcInterm_t *interm);
void CcInterm_Delete(CcInterm_t *interm);
void CcInt(const wignerF_t *restrict_ W, const quadI1_t *restrict_ quadI1, CcInterm_t *restrict_ interm, wignerF_t *restrict_ Cc);

#ifdef __cplusplus
}
#endif

#endif /* COLLISION_H */

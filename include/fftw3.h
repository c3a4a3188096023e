/* fftw3.h — the subset of the FFTW 3 C API that the collision/transport
 * library, its callers and its test drivers use.
 *
 * The upstream solver includes <fftw3.h> from include/grid.h:28 and calls
 * FFTW directly from its drivers (test/Cc_test.c:104-106, test/Cd_test.c:105-107,
 * test/coll_step_test.c:110-112, src/main_hom.c:61,105).  FFTW itself is not
 * part of this project: this header only declares the entry points with
 * FFTW's published signatures and constants so that those drivers compile
 * unchanged.  Two implementations exist:
 *   - libqbgpu (the product) runs every planned transform on the GPU with the
 *     project's own FFT kernels;
 *   - the oracle (oracle/fftw_cpu.c) is a CPU restatement of the DFT used only
 *     by tests to build the upstream sources as a checker.
 *
 * Conventions (FFTW's): FORWARD uses exp(-2 pi i jk/n), BACKWARD exp(+2 pi i jk/n),
 * no normalisation; 2-D arrays are row-major with the last index fastest.
 */
#ifndef QB_FFTW3_H
#define QB_FFTW3_H

#include <stddef.h>
#include <stdio.h>   /* the upstream drivers rely on <fftw3.h> pulling in stdio */

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct fftw_plan_s *fftw_plan;

#define FFTW_FORWARD  (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE  (0U)
#define FFTW_ESTIMATE (1U << 6)

void *fftw_malloc(size_t n);
void fftw_free(void *p);

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out, unsigned flags);

void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void fftw_cleanup(void);

#ifdef __cplusplus
}
#endif

#endif /* QB_FFTW3_H */

/* ref_harness.c — ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * Compiled together with the unmodified upstream sources
 * (src/{collision,finite_volume,grid,integrals,quadrature,simulation,util}.c,
 * upstream headers, N_GRID = 32) and oracle/fftw_cpu.c into
 * oracle/_ref/libqbref_n32.so.  It exposes flat entry points (plain double
 * arrays) around the upstream API so that Python tests can run the real
 * upstream code as a second checker beside the restatement in qb_oracle.c.
 * This file is project code; it only calls the upstream functions.
 */
#include "simulation.h"
#include "finite_volume.h"
#include "util.h"
#include <stdlib.h>
#include <string.h>

void LegendreGaussQuad(const unsigned int M, const double a, const double b, double *x, double *w);

int ref_n_grid(void) { return N_GRID; }

typedef struct {
	quadI1_t q1; quadI2_t q2; quadI3_t q3; quadI1_t q4;
} ref_ctx;

void *ref_ctx_create(unsigned J, unsigned M, double L, double R)
{
	ref_ctx *c = calloc(1, sizeof(*c));
	FourierI1(J, L, R, &c->q1);
	FourierI2(J, L, R, &c->q2);
	FourierI3(J, L, R, M, &c->q3);
	FourierI4(J, L, R, &c->q4);
	return c;
}

void ref_ctx_free(void *p)
{
	ref_ctx *c = p;
	QuadI1_Delete(&c->q4); QuadI3_Delete(&c->q3); QuadI2_Delete(&c->q2); QuadI1_Delete(&c->q1);
	free(c);
}

/* table copies: which = 1..4, part = 1 (psiR1) or 2 (psiR2) */
unsigned ref_table_num(void *p, int which)
{
	ref_ctx *c = p;
	return which == 1 ? c->q1.num : which == 2 ? c->q2.num : which == 3 ? c->q3.num : c->q4.num;
}

void ref_table_copy(void *p, int which, int part, double *out)
{
	ref_ctx *c = p;
	size_t n;
	const void *src;
	switch (which) {
	case 1: n = c->q1.num * (part == 1 ? sizeof(grid2_t) : sizeof(grid_t)); src = part == 1 ? (void *)c->q1.psiR1 : (void *)c->q1.psiR2; break;
	case 2: n = c->q2.num * sizeof(grid_t); src = part == 1 ? (void *)c->q2.psiR1 : (void *)c->q2.psiR2; break;
	case 3: n = c->q3.num * (part == 1 ? sizeof(cgrid_t) : sizeof(grid2_t)); src = part == 1 ? (void *)c->q3.psiR1 : (void *)c->q3.psiR2; break;
	default: n = c->q4.num * (part == 1 ? sizeof(grid2_t) : sizeof(grid_t)); src = part == 1 ? (void *)c->q4.psiR1 : (void *)c->q4.psiR2; break;
	}
	memcpy(out, src, n);
}

/* I-integrals with the context's tables (which = 1: I1, 4: I4 via I1integral) */
void ref_i1(void *p, int which, const double *f, const double *g, const double *h, double *out)
{
	ref_ctx *c = p;
	I1interm_t it; I1interm_Create(&it);
	I1integral((const cgrid_t *)f, (const cgrid_t *)g, (const cgrid_t *)h, which == 4 ? &c->q4 : &c->q1, &it, (cgrid_t *)out);
	I1interm_Delete(&it);
}

void ref_i2(void *p, const double *f, const double *g, const double *h, double *out)
{
	ref_ctx *c = p;
	I2interm_t it; I2interm_Create(&it);
	I2integral((const cgrid_t *)f, (const cgrid_t *)g, (const cgrid_t *)h, &c->q2, &it, (cgrid_t *)out);
	I2interm_Delete(&it);
}

void ref_i3(void *p, const double *f, const double *g, const double *h, double *out)
{
	ref_ctx *c = p;
	I3interm_t it; I3interm_Create(&it);
	I3integral((const cgrid_t *)f, (const cgrid_t *)g, (const cgrid_t *)h, &c->q3, &it, (cgrid_t *)out);
	I3interm_Delete(&it);
}

void ref_cc(void *p, const double *W, double *out)
{
	ref_ctx *c = p;
	CcInterm_t it; CcInterm_Create(&it);
	CcInt((const wignerF_t *)W, &c->q1, &it, (wignerF_t *)out);
	CcInterm_Delete(&it);
}

void ref_cd(void *p, const double *W, double *out)
{
	ref_ctx *c = p;
	CdInterm_t it; CdInterm_Create(&it);
	CdInt((const wignerF_t *)W, &c->q2, &c->q3, &c->q4, &it, (wignerF_t *)out);
	CdInterm_Delete(&it);
}

void ref_collision_step(void *p, const double *W, double dt, const double *B, double *out)
{
	ref_ctx *c = p;
	collisionInterm_t it; CollisionInterm_Create(&it);
	CollisionStep((const wignerF_t *)W, &c->q1, &c->q2, &c->q3, &c->q4, dt, B, &it, (wignerF_t *)out);
	CollisionInterm_Delete(&it);
}

/* bc: 0 periodic, 1 Dirichlet */
void ref_inhom_step(void *p, int bc, unsigned numVol, double L, const double *W, double h, double dt, const double *Bext, double *out)
{
	ref_ctx *c = p;
	inhomStepInterm_t it; InhomStepInterm_Create(numVol, L, &it);
	if (bc == 0) InhomStepPeriodic((const wignerV_t *)W, &c->q1, &c->q2, &c->q3, &c->q4, h, dt, Bext, &it, (wignerV_t *)out);
	else         InhomStepDirichlet((const wignerV_t *)W, &c->q1, &c->q2, &c->q3, &c->q4, h, dt, Bext, &it, (wignerV_t *)out);
	InhomStepInterm_Delete(&it);
}

void ref_inhom_step_maxwell(void *p, unsigned numVol, double L, const double *W, double h, double dt, double lambda,
                            const double *WL, const double *WR, const double *Bext, double *out)
{
	ref_ctx *c = p;
	inhomStepInterm_t it; InhomStepInterm_Create(numVol, L, &it);
	InhomStepMaxwell((const wignerV_t *)W, &c->q1, &c->q2, &c->q3, &c->q4, h, dt, lambda,
	                 (const wignerV_t *)WL, (const wignerV_t *)WR, Bext, &it, (wignerV_t *)out);
	InhomStepInterm_Delete(&it);
}

void ref_sim_hom(void *p, const double *W0, double dt, unsigned numsteps, const double *B, double *out)
{
	ref_ctx *c = p;
	simulationHomInterm_t it; SimulationHomInterm_Create(&it);
	SimulationHomogeneous((const wignerV_t *)W0, &c->q1, &c->q2, &c->q3, &c->q4, dt, numsteps, B, &it, (wignerV_t *)out);
	SimulationHomInterm_Delete(&it);
}

/* InternalFourierCollisionStep's transform to Fourier space, as the upstream
 * test drivers do it (test/Cc_test.c:99-136): r2c, 1/N^2, Hermitian fill */
void ref_to_fourier(const double *Wv, double *Wf)
{
	const int N = N_GRID;
	cgrid_t *WFh = fftw_malloc(sizeof(cgrid_t));
	double *in = fftw_malloc(sizeof(grid_t));
	for (int i = 0; i < 4; i++) {
		memcpy(in, Wv + i * N * N, sizeof(grid_t));
		fftw_plan plan = fftw_plan_dft_r2c_2d(N, N, in, WFh->data, FFTW_ESTIMATE);
		fftw_execute(plan);
		fftw_destroy_plan(plan);
		const double scale = 1.0 / (N * N);
		double *o = Wf + 2 * i * N * N;
		for (int l = 0; l < N; l++) {
			const int lc = (N - l) & N_MASK;
			for (int k = 0; k <= N / 2; k++) {
				o[2 * (N * l + k)]     = WFh->data[(N / 2 + 1) * l + k][0] * scale;
				o[2 * (N * l + k) + 1] = WFh->data[(N / 2 + 1) * l + k][1] * scale;
			}
			for (int k = N / 2 + 1; k < N; k++) {
				const int kc = N - k;
				o[2 * (N * l + k)]     =  WFh->data[(N / 2 + 1) * lc + kc][0] * scale;
				o[2 * (N * l + k) + 1] = -WFh->data[(N / 2 + 1) * lc + kc][1] * scale;
			}
		}
	}
	fftw_free(in);
	fftw_free(WFh);
}

/* SimulationInhomogeneousPeriodic (src/simulation.c:1288-1301): numsteps
 * frames of numVol cells, frame 0 = W0, written to Wevolv */
void ref_sim_inhom_periodic(void *p, unsigned numVol, double L, const double *W0, double h, double dt,
                            unsigned numsteps, const double *Bext, double *Wevolv)
{
	ref_ctx *c = p;
	inhomStepInterm_t it; InhomStepInterm_Create(numVol, L, &it);
	SimulationInhomogeneousPeriodic((const wignerV_t *)W0, &c->q1, &c->q2, &c->q3, &c->q4, h, dt, numsteps, Bext, &it,
	                                (wignerV_t *)Wevolv);
	InhomStepInterm_Delete(&it);
}

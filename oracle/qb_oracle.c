/* qb_oracle.c — ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the upstream solver's time step with the grid size
 * N as a run-time parameter.  It follows the upstream loop structure term by
 * term (no factoring), so it is slow by design: it is the checker that the
 * GPU path is compared against, and is only called from tests/, the smoke
 * check and bench.py's CPU-baseline leg.  Independent integrals of one
 * operator evaluation run in parallel (pthreads, ORC_THREADS, default all
 * cores); every sum is accumulated in the upstream order.
 *
 * Array conventions: a complex N x N grid is 2*N*N doubles (re, im
 * interleaved), element (l, k) at index k + N*l; P = 2N is the padded size;
 * a Wigner state is 4 consecutive grids (trace, x, y, z); a cell array is
 * cell-major (numVol consecutive Wigner states).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#include <assert.h>
#include <pthread.h>
#include <unistd.h>
#include "qb_oracle.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

void orc_fft2d(double *a, int n0, int n1, int sign);   /* fftw_cpu.c */

static inline double sq(double x) { return x * x; }

/* ---- a minimal parallel-for over independent tasks (pthreads) ------------ */
typedef struct { void (*fn)(int, void *); void *ctx; int n; int next; pthread_mutex_t lock; } par_job;

static void *par_worker(void *arg)
{
	par_job *jb = arg;
	for (;;) {
		pthread_mutex_lock(&jb->lock);
		const int t = jb->next++;
		pthread_mutex_unlock(&jb->lock);
		if (t >= jb->n) return NULL;
		jb->fn(t, jb->ctx);
	}
}

static int par_threads(void)
{
	const char *e = getenv("ORC_THREADS");
	long n = e ? atol(e) : sysconf(_SC_NPROCESSORS_ONLN);
	return n < 1 ? 1 : (n > 64 ? 64 : (int)n);
}

static __thread int par_inside;   /* nested par_for calls run serially */

static void *par_worker_outer(void *arg)
{
	par_inside = 1;
	return par_worker(arg);
}

/* runs fn(0..n-1, ctx) on up to ORC_THREADS threads (default: all cores) */
static void par_for(int n, void (*fn)(int, void *), void *ctx)
{
	int nt = par_inside ? 1 : par_threads();
	if (nt > n) nt = n;
	par_job jb = { fn, ctx, n, 0, PTHREAD_MUTEX_INITIALIZER };
	if (nt <= 1) { for (int t = 0; t < n; t++) fn(t, ctx); return; }
	pthread_t th[64];
	for (int i = 0; i < nt; i++) pthread_create(&th[i], NULL, par_worker_outer, &jb);
	for (int i = 0; i < nt; i++) pthread_join(th[i], NULL);
}
static inline int kgrid(int N, int k)  { return k < N / 2 ? k : k - N; }       /* quadrature.c:163-166 */
static inline int kgrid2(int N, int k) { return k < N ? k : k - 2 * N; }       /* quadrature.c:167-170 */

/* ---- grid helpers (upstream src/grid.c) ---------------------------------- */

/* GridZeroPad, grid.c:171-188: corner quadrants of the 2N x 2N grid */
void orc_zero_pad(int N, const double *f, double *ret)
{
	const int P = 2 * N;
	memset(ret, 0, sizeof(double) * 2 * P * P);
	for (int l = 0; l < N; l++) {
		const int lp = (l < N / 2) ? l : (N + l);          /* row in the padded grid */
		for (int k = 0; k < N; k++) {
			const int kp = (k < N / 2) ? k : (N + k);
			ret[2 * (kp + P * lp)]     = f[2 * (k + N * l)];
			ret[2 * (kp + P * lp) + 1] = f[2 * (k + N * l) + 1];
		}
	}
}

/* GridExtract, grid.c:195-210 */
void orc_extract(int N, const double *f, double *ret)
{
	const int P = 2 * N;
	for (int l = 0; l < N; l++) {
		const int lp = (l < N / 2) ? l : (N + l);
		for (int k = 0; k < N; k++) {
			const int kp = (k < N / 2) ? k : (N + k);
			ret[2 * (k + N * l)]     = f[2 * (kp + P * lp)];
			ret[2 * (k + N * l) + 1] = f[2 * (kp + P * lp) + 1];
		}
	}
}

/* ret = f .* ret, complex (MultiplyPointwiseAssignCC2, grid.c:152-164) */
static void mul_assign_cc(long n, const double *f, double *ret)
{
	for (long i = 0; i < n; i++) {
		const double re = ret[2 * i], im = ret[2 * i + 1];
		ret[2 * i]     = f[2 * i] * re - f[2 * i + 1] * im;
		ret[2 * i + 1] = f[2 * i] * im + f[2 * i + 1] * re;
	}
}

/* ret = f .* g, complex (MultiplyPointwiseCC / CC2, grid.c:61-73,107-119) */
static void mul_cc(long n, const double *f, const double *g, double *ret)
{
	for (long i = 0; i < n; i++) {
		ret[2 * i]     = f[2 * i] * g[2 * i] - f[2 * i + 1] * g[2 * i + 1];
		ret[2 * i + 1] = f[2 * i] * g[2 * i + 1] + f[2 * i + 1] * g[2 * i];
	}
}

/* ret = f .* g, real x complex (MultiplyPointwiseRC, grid.c:47-55) */
static void mul_rc(long n, const double *f, const double *g, double *ret)
{
	for (long i = 0; i < n; i++) { ret[2 * i] = f[i] * g[2 * i]; ret[2 * i + 1] = f[i] * g[2 * i + 1]; }
}

/* ret *= f, real x complex (MultiplyPointwiseAssignRC2, grid.c:137-145) */
static void mul_assign_rc(long n, const double *f, double *ret)
{
	for (long i = 0; i < n; i++) { ret[2 * i] *= f[i]; ret[2 * i + 1] *= f[i]; }
}

/* ---- quadrature tables (upstream src/quadrature.c) ----------------------- */

static double orc_sin_sinc(double x) { return fabs(x) < 1e-8 ? x : sq(sin(x)) / x; }   /* :116-126 */
static double orc_sinc(double x)     { return fabs(x) < 1e-8 ? 1 : sin(x) / x; }       /* :132-142 */

/* FourierI1, quadrature.c:150-238: J*J terms; psiR1[i+J*j] = psi1_i (2N grid),
 * psiR2[i+J*j] = weight_ij * psi2_j (N grid) */
void orc_fourier_i1(int N, int J, double L, double R, double *psiR1, double *psiR2)
{
	const int P = 2 * N;
	const double dth = M_PI / J;
	const double s = R * M_PI / (2 * L);
	for (int i = 0; i < J; i++) {
		const double th1 = i * dth, c = cos(th1), sn = sin(th1);
		double *g = psiR1 + (long)i * P * P;
		for (int l = 0; l < P; l++)
			for (int k = 0; k < P; k++)
				g[k + P * l] = R * orc_sin_sinc(s * (kgrid2(N, l) * c + kgrid2(N, k) * sn));
		for (int j = 1; j < J; j++) memcpy(psiR1 + (long)(i + J * j) * P * P, g, sizeof(double) * P * P);
	}
	for (int j = 0; j < J; j++) {
		const double th2 = j * dth + 0.5 * dth, c = cos(th2), sn = sin(th2);
		double *g = psiR2 + (long)(J * j) * N * N;
		for (int l = 0; l < N; l++)
			for (int k = 0; k < N; k++)
				g[k + N * l] = R * orc_sin_sinc(s * (kgrid(N, l) * c + kgrid(N, k) * sn));
		for (int i = 1; i < J; i++) memcpy(psiR2 + (long)(i + J * j) * N * N, g, sizeof(double) * N * N);
	}
	for (int j = 0; j < J; j++)
		for (int i = 0; i < J; i++) {
			const double th1 = i * dth, th2 = j * dth + 0.5 * dth;
			const double weight = -sq(2 * M_PI / J) / cos(th1 - th2);
			double *g = psiR2 + (long)(i + J * j) * N * N;
			for (int q = 0; q < N * N; q++) g[q] *= weight;
		}
}

/* FourierI2, quadrature.c:245-286 */
void orc_fourier_i2(int N, int J, double L, double R, double *psiR1, double *psiR2)
{
	const double f1 = 2 * R, f2 = 2 * R * M_PI / J, s = R * M_PI / L;
	for (int j = 0; j < J; j++) {
		const double th = j * M_PI / J, c = cos(th), sn = sin(th);
		for (int l = 0; l < N; l++)
			for (int k = 0; k < N; k++) {
				psiR1[(long)j * N * N + k + N * l] = f1 * orc_sinc(s * ( kgrid(N, l) * c + kgrid(N, k) * sn));
				psiR2[(long)j * N * N + k + N * l] = f2 * orc_sinc(s * (-kgrid(N, l) * sn + kgrid(N, k) * c));
			}
	}
}

/* LegendreGaussQuad, quadrature.c:293-388 (Newton iteration on P_M) */
void orc_lgwt(int M, double a, double b, double *x, double *w)
{
	const double invN = 1.0 / (M - 1);
	double *y = malloc(sizeof(double) * M), *y0 = malloc(sizeof(double) * M);
	double *Lv = calloc((size_t)M * (M + 1), sizeof(double)), *Lp = calloc(M, sizeof(double));
	for (int i = 0; i < M; i++) {
		const double xu = -1.0 + 2 * i * invN;
		y[i] = cos((2 * i + 1) * M_PI / (2 * M)) + 0.27 / M * sin(M_PI * xu * (M - 1) / (M + 1));
		y0[i] = 2;
	}
	double diff = 0;
	for (int i = 0; i < M; i++) diff = fmax(diff, fabs(y[i] - y0[i]));
	int iter = 0;
	while (diff > DBL_EPSILON && iter++ < 1000) {
		for (int i = 0; i < M; i++) { Lv[i] = 1; Lv[i + M] = y[i]; }
		for (int k = 1; k < M; k++)
			for (int i = 0; i < M; i++)
				Lv[i + (k + 1) * M] = ((2 * k + 1) * y[i] * Lv[i + k * M] - k * Lv[i + (k - 1) * M]) / (k + 1);
		for (int i = 0; i < M; i++)
			Lp[i] = (M + 1) * (Lv[i + (M - 1) * M] - y[i] * Lv[i + M * M]) / (1 - sq(y[i]));
		memcpy(y0, y, sizeof(double) * M);
		diff = 0;
		for (int i = 0; i < M; i++) {
			const double t = Lv[i + M * M] / Lp[i];
			y[i] -= t;
			diff = fmax(diff, fabs(t));
		}
	}
	for (int i = 0; i < M; i++) {
		x[i] = (a * (1 - y[i]) + b * (1 + y[i])) / 2;
		w[i] = (b - a) / ((1 - sq(y[i])) * sq(Lp[i])) * sq((double)(M + 1) / M);
	}
	free(Lv); free(Lp); free(y0); free(y);
}

/* FourierI3, quadrature.c:395-466: J*M terms, index m + j*M */
void orc_fourier_i3(int N, int J, double L, double R, int M, double *psiR1, double *psiR2)
{
	const int P = 2 * N;
	double *rho = malloc(sizeof(double) * M), *w = malloc(sizeof(double) * M);
	orc_lgwt(M, -R, R, rho, w);
	const double s2 = M_PI * R / L;
	for (int j = 0; j < J; j++) {
		const double th = j * M_PI / J, c = cos(th), sn = sin(th);
		for (int m = 0; m < M; m++) {
			double *g1 = psiR1 + (long)(m + j * M) * 2 * N * N;
			double *g2 = psiR2 + (long)(m + j * M) * P * P;
			const double s1 = rho[m] * M_PI / L;
			const double f2 = 2 * R * w[m] * M_PI / J;
			for (int l = 0; l < N; l++)
				for (int k = 0; k < N; k++) {
					const double t = s1 * (kgrid(N, l) * c + kgrid(N, k) * sn);
					g1[2 * (k + N * l)] = cos(t);
					g1[2 * (k + N * l) + 1] = sin(t);
				}
			for (int l = 0; l < P; l++)
				for (int k = 0; k < P; k++)
					g2[k + P * l] = f2 * orc_sinc(s2 * (-kgrid2(N, l) * sn + kgrid2(N, k) * c));
		}
	}
	free(w); free(rho);
}

/* FourierI4, quadrature.c:473-527 */
void orc_fourier_i4(int N, int J, double L, double R, double *psiR1, double *psiR2)
{
	const int P = 2 * N;
	const double f1 = 2 * R, f2 = 2 * R * M_PI / J, s = M_PI * R / L;
	for (int j = 0; j < J; j++) {
		const double th = j * M_PI / J, c = cos(th), sn = sin(th);
		for (int l = 0; l < P; l++)
			for (int k = 0; k < P; k++)
				psiR1[(long)j * P * P + k + P * l] = f1 * orc_sinc(s * (kgrid2(N, l) * c + kgrid2(N, k) * sn));
		for (int l = 0; l < N; l++)
			for (int k = 0; k < N; k++)
				psiR2[(long)j * N * N + k + N * l] = f2 * orc_sinc(s * (-kgrid(N, l) * sn + kgrid(N, k) * c));
	}
}

/* ---- integrals (upstream src/integrals.c) -------------------------------- */

/* I1integral, integrals.c:90-133 (also I4) */
void orc_i1(int N, const double *f, const double *g, const double *h,
            int num, const double *psiR1, const double *psiR2, double *I1)
{
	const int P = 2 * N;
	const long nn = (long)N * N, pp = (long)P * P;
	const double scale = sq(1.0 / (4.0 * N * N));
	double *f2F = malloc(sizeof(double) * 2 * pp), *h2F = malloc(sizeof(double) * 2 * pp);
	double *tmp = malloc(sizeof(double) * 2 * nn), *t2 = malloc(sizeof(double) * 2 * pp);
	orc_zero_pad(N, f, f2F); orc_fft2d(f2F, P, P, -1);
	orc_zero_pad(N, h, h2F); orc_fft2d(h2F, P, P, -1);
	memset(I1, 0, sizeof(double) * 2 * nn);
	for (int j = 0; j < num; j++) {
		mul_rc(nn, psiR2 + (long)j * nn, g, tmp);
		orc_zero_pad(N, tmp, t2);
		orc_fft2d(t2, P, P, -1);
		mul_assign_cc(pp, f2F, t2);
		orc_fft2d(t2, P, P, +1);
		mul_assign_rc(pp, psiR1 + (long)j * pp, t2);
		orc_fft2d(t2, P, P, -1);
		mul_assign_cc(pp, h2F, t2);
		orc_fft2d(t2, P, P, +1);
		orc_extract(N, t2, tmp);
		for (long i = 0; i < 2 * nn; i++) I1[i] += scale * tmp[i];
	}
	free(t2); free(tmp); free(h2F); free(f2F);
}

/* I2integral, integrals.c:211-251 */
void orc_i2(int N, const double *f, const double *g, const double *h,
            int num, const double *psiR1, const double *psiR2, double *I2)
{
	const int P = 2 * N;
	const long nn = (long)N * N, pp = (long)P * P;
	const double scale = 1.0 / (4.0 * N * N);
	double *h2F = malloc(sizeof(double) * 2 * pp), *fp = malloc(sizeof(double) * 2 * nn), *gp = malloc(sizeof(double) * 2 * nn);
	double *fP = malloc(sizeof(double) * 2 * pp), *gP = malloc(sizeof(double) * 2 * pp), *t2 = malloc(sizeof(double) * 2 * pp);
	double *tmp = malloc(sizeof(double) * 2 * nn);
	orc_zero_pad(N, h, h2F); orc_fft2d(h2F, P, P, -1);
	memset(I2, 0, sizeof(double) * 2 * nn);
	for (int j = 0; j < num; j++) {
		mul_rc(nn, psiR1 + (long)j * nn, f, fp);
		mul_rc(nn, psiR2 + (long)j * nn, g, gp);
		orc_zero_pad(N, fp, fP); orc_zero_pad(N, gp, gP);
		orc_fft2d(fP, P, P, -1); orc_fft2d(gP, P, P, -1);
		mul_cc(pp, fP, gP, t2);
		mul_assign_cc(pp, h2F, t2);
		orc_fft2d(t2, P, P, +1);
		orc_extract(N, t2, tmp);
		for (long i = 0; i < 2 * nn; i++) I2[i] += scale * tmp[i];
	}
	free(tmp); free(t2); free(gP); free(fP); free(gp); free(fp); free(h2F);
}

/* I3integral, integrals.c:332-379 */
void orc_i3(int N, const double *f, const double *g, const double *h,
            int num, const double *psiR1, const double *psiR2, double *I3)
{
	const int P = 2 * N;
	const long nn = (long)N * N, pp = (long)P * P;
	const double scale = sq(1.0 / (4.0 * N * N));
	double *g2F = malloc(sizeof(double) * 2 * pp), *fp = malloc(sizeof(double) * 2 * nn), *hp = malloc(sizeof(double) * 2 * nn);
	double *fP = malloc(sizeof(double) * 2 * pp), *hP = malloc(sizeof(double) * 2 * pp), *t2 = malloc(sizeof(double) * 2 * pp);
	double *tmp = malloc(sizeof(double) * 2 * nn);
	orc_zero_pad(N, g, g2F); orc_fft2d(g2F, P, P, -1);
	memset(I3, 0, sizeof(double) * 2 * nn);
	for (int j = 0; j < num; j++) {
		mul_cc(nn, psiR1 + (long)j * 2 * nn, f, fp);
		mul_cc(nn, psiR1 + (long)j * 2 * nn, h, hp);
		orc_zero_pad(N, fp, fP); orc_zero_pad(N, hp, hP);
		orc_fft2d(fP, P, P, -1); orc_fft2d(hP, P, P, -1);
		mul_cc(pp, g2F, hP, t2);
		orc_fft2d(t2, P, P, +1);
		mul_assign_rc(pp, psiR2 + (long)j * pp, t2);
		orc_fft2d(t2, P, P, -1);
		mul_assign_cc(pp, fP, t2);
		orc_fft2d(t2, P, P, +1);
		orc_extract(N, t2, tmp);
		for (long i = 0; i < 2 * nn; i++) I3[i] += scale * tmp[i];
	}
	free(tmp); free(t2); free(hP); free(fP); free(hp); free(fp); free(g2F);
}

/* ---- quadrature bundle --------------------------------------------------- */

orc_quad *orc_quad_create(int N, int J, int M, double L, double R)
{
	const long P = 2 * N;
	orc_quad *q = calloc(1, sizeof(*q));
	q->N = N; q->J = J; q->M = M; q->L = L; q->R = R;
	q->n1 = J * J; q->n2 = J; q->n3 = J * M; q->n4 = J;
	q->i1r1 = malloc(sizeof(double) * q->n1 * P * P); q->i1r2 = malloc(sizeof(double) * q->n1 * N * N);
	q->i2r1 = malloc(sizeof(double) * q->n2 * N * N); q->i2r2 = malloc(sizeof(double) * q->n2 * N * N);
	q->i3r1 = malloc(sizeof(double) * q->n3 * 2 * N * N); q->i3r2 = malloc(sizeof(double) * q->n3 * P * P);
	q->i4r1 = malloc(sizeof(double) * q->n4 * P * P); q->i4r2 = malloc(sizeof(double) * q->n4 * N * N);
	orc_fourier_i1(N, J, L, R, q->i1r1, q->i1r2);
	orc_fourier_i2(N, J, L, R, q->i2r1, q->i2r2);
	orc_fourier_i3(N, J, L, R, M, q->i3r1, q->i3r2);
	orc_fourier_i4(N, J, L, R, q->i4r1, q->i4r2);
	return q;
}

void orc_quad_free(orc_quad *q)
{
	if (!q) return;
	free(q->i1r1); free(q->i1r2); free(q->i2r1); free(q->i2r2);
	free(q->i3r1); free(q->i3r2); free(q->i4r1); free(q->i4r2);
	free(q);
}

/* ---- collision operators (upstream src/collision.c) ---------------------- */

typedef struct { const orc_quad *q; const double *W, *Wtr2m1; double *res; const int *gi, *hi; } cc_task;

static void cc_run(int t, void *p)
{
	cc_task *c = p;
	const long g = 2L * c->q->N * c->q->N;
	orc_i1(c->q->N, c->Wtr2m1, c->W + c->gi[t] * g, c->W + c->hi[t] * g, c->q->n1, c->q->i1r1, c->q->i1r2, c->res + t * g);
}

/* CcInt, collision.c:209-254: six I1 integrals (independent; run in parallel,
 * combined in upstream order). */
void orc_cc(const orc_quad *q, const double *W, double *Cc)
{
	const int N = q->N;
	const long nn = (long)N * N;
	double *Wtr2m1 = malloc(sizeof(double) * 2 * nn);
	for (long k = 0; k < 2 * nn; k++) Wtr2m1[k] = -4 * W[k];
	Wtr2m1[0] += 2;
	/* (output comp, g, h) pairs: Cc_1 = I1(.,W2,W3) - I1(.,W3,W2) etc. */
	static const int gi[6] = { 2, 3, 3, 1, 1, 2 };
	static const int hi[6] = { 3, 2, 1, 3, 2, 1 };
	double *res = malloc(sizeof(double) * 6 * 2 * nn);
	cc_task ct = { q, W, Wtr2m1, res, gi, hi };
	par_for(6, cc_run, &ct);
	memset(Cc, 0, sizeof(double) * 4 * 2 * nn);
	for (int b = 0; b < 3; b++) {
		double *o = Cc + (b + 1) * 2 * nn;
		memcpy(o, res + (2 * b) * 2 * nn, sizeof(double) * 2 * nn);
		for (long k = 0; k < 2 * nn; k++) o[k] -= res[(2 * b + 1) * 2 * nn + k];
	}
	free(res); free(Wtr2m1);
}

typedef struct { const orc_quad *q; const double *W, *Wt, *Wt0; double *r2, *r3, *r4; } cd_task;

static void cd_run(int t, void *p)
{
	cd_task *c = p;
	const orc_quad *q = c->q;
	const int N = q->N;
	const long g = 2L * N * N;
	const double *W = c->W;
	if (t < 16) {            /* I3 first: the expensive ones */
		const int j = t / 4, i = t % 4;
		orc_i3(N, W + i * g, W + i * g, W + j * g, q->n3, q->i3r1, q->i3r2, c->r3 + t * g);
	} else if (t < 32) {
		const int u = t - 16, j = u / 4, i = u % 4;
		orc_i2(N, W + i * g, W + i * g, c->Wt + j * g, q->n2, q->i2r1, q->i2r2, c->r2 + u * g);
	} else {
		const int u = t - 32, grp = u / 4, j = u % 4;
		const double *gg = (grp == 1) ? W : W + j * g;
		const double *hh = (grp == 0) ? W : W + j * g;
		orc_i1(N, c->Wt0, gg, hh, q->n4, q->i4r1, q->i4r2, c->r4 + u * g);
	}
}

/* CdInt, collision.c:74-168: 16 I2 + 16 I3 + 12 I4 integrals (computed in
 * parallel, accumulated in upstream order). */
void orc_cd(const orc_quad *q, const double *W, double *Cd)
{
	const int N = q->N;
	const long nn = (long)N * N, g = 2 * nn;
	static const double eta[4] = { 1, -1, -1, -1 };
	static const double eta2[4] = { 2, -2, -2, -2 };
	double *Wt = malloc(sizeof(double) * 4 * g);
	for (long k = 0; k < 4 * g; k++) Wt[k] = -W[k];
	Wt[0] += 1;
	double *Wt0 = malloc(sizeof(double) * g);    /* 2 W_0 - 1 */
	for (long k = 0; k < g; k++) Wt0[k] = 2 * W[k];
	Wt0[0] -= 1;
	double *r2 = malloc(sizeof(double) * 16 * g), *r3 = malloc(sizeof(double) * 16 * g), *r4 = malloc(sizeof(double) * 12 * g);
	cd_task ct = { q, W, Wt, Wt0, r2, r3, r4 };
	par_for(44, cd_run, &ct);
	memset(Cd, 0, sizeof(double) * 4 * g);
	for (int j = 0; j < 4; j++)
		for (int i = 0; i < 4; i++)
			for (long k = 0; k < g; k++) Cd[j * g + k] += eta2[i] * r2[(j * 4 + i) * g + k];
	for (int j = 0; j < 4; j++)
		for (int i = 0; i < 4; i++)
			for (long k = 0; k < g; k++) Cd[j * g + k] -= eta[i] * eta2[j] * r3[(j * 4 + i) * g + k];
	for (int j = 0; j < 4; j++)
		for (long k = 0; k < g; k++) Cd[j * g + k] += eta2[j] * r4[j * g + k];
	for (int j = 0; j < 4; j++)
		for (long k = 0; k < g; k++) Cd[j * g + k] += 2 * r4[(4 + j) * g + k];
	for (int j = 0; j < 4; j++)
		for (long k = 0; k < g; k++) Cd[k] -= 2 * r4[(8 + j) * g + k];
	free(r4); free(r3); free(r2); free(Wt0); free(Wt);
}

/* MagneticRotation, simulation.c:75-98 */
void orc_magnetic_rotation(int N, const double *W, const double B[3], double *CB)
{
	const long g = 2L * N * N;
	memset(CB, 0, sizeof(double) * g);
	for (long k = 0; k < g; k++) {
		CB[1 * g + k] = 2 * (B[1] * W[3 * g + k] - B[2] * W[2 * g + k]);
		CB[2 * g + k] = 2 * (B[2] * W[1 * g + k] - B[0] * W[3 * g + k]);
		CB[3 * g + k] = 2 * (B[0] * W[2 * g + k] - B[1] * W[1 * g + k]);
	}
}

/* right-hand side Cc + Cd + CB, each accumulated as upstream does in the update */
static void rhs_parts(const orc_quad *q, const double *W, const double B[3], double *Cc, double *Cd, double *CB)
{
	orc_cc(q, W, Cc);
	orc_cd(q, W, Cd);
	orc_magnetic_rotation(q->N, W, B, CB);
}

/* CollisionStep, simulation.c:105-136 (midpoint rule) */
void orc_collision_step(const orc_quad *q, const double *W, double dt, const double B[3], double *Wnext)
{
	const long n = 4L * 2 * q->N * q->N;
	double *Cc = malloc(sizeof(double) * n), *Cd = malloc(sizeof(double) * n), *CB = malloc(sizeof(double) * n);
	double *Wmid = malloc(sizeof(double) * n);
	rhs_parts(q, W, B, Cc, Cd, CB);
	const double dth = 0.5 * dt;
	for (long k = 0; k < n; k++) Wmid[k] = W[k] + dth * (Cc[k] + Cd[k] + CB[k]);
	rhs_parts(q, Wmid, B, Cc, Cd, CB);
	for (long k = 0; k < n; k++) Wnext[k] = W[k] + dt * (Cc[k] + Cd[k] + CB[k]);
	free(Wmid); free(CB); free(Cd); free(Cc);
}

/* Classical RK4 on the same right-hand side (extension used by the
 * homogeneous RK4 workloads; upstream only has the midpoint rule). */
void orc_collision_step_rk4(const orc_quad *q, const double *W, double dt, const double B[3], double *Wnext)
{
	const long n = 4L * 2 * q->N * q->N;
	double *Cc = malloc(sizeof(double) * n), *Cd = malloc(sizeof(double) * n), *CB = malloc(sizeof(double) * n);
	double *k1 = malloc(sizeof(double) * n), *k2 = malloc(sizeof(double) * n), *k3 = malloc(sizeof(double) * n), *k4 = malloc(sizeof(double) * n);
	double *Ws = malloc(sizeof(double) * n);
	rhs_parts(q, W, B, Cc, Cd, CB);
	for (long k = 0; k < n; k++) { k1[k] = Cc[k] + Cd[k] + CB[k]; Ws[k] = W[k] + 0.5 * dt * k1[k]; }
	rhs_parts(q, Ws, B, Cc, Cd, CB);
	for (long k = 0; k < n; k++) { k2[k] = Cc[k] + Cd[k] + CB[k]; Ws[k] = W[k] + 0.5 * dt * k2[k]; }
	rhs_parts(q, Ws, B, Cc, Cd, CB);
	for (long k = 0; k < n; k++) { k3[k] = Cc[k] + Cd[k] + CB[k]; Ws[k] = W[k] + dt * k3[k]; }
	rhs_parts(q, Ws, B, Cc, Cd, CB);
	for (long k = 0; k < n; k++) { k4[k] = Cc[k] + Cd[k] + CB[k]; Wnext[k] = W[k] + dt / 6.0 * (k1[k] + 2 * k2[k] + 2 * k3[k] + k4[k]); }
	free(Ws); free(k4); free(k3); free(k2); free(k1); free(CB); free(Cd); free(Cc);
}

/* ---- Fourier representation (upstream simulation.c:224-283) -------------- */

/* one real component -> Fourier grid: FFT / N^2, Hermitian completion (:224-261) */
static void to_fourier_comp(int N, const double *Wv, double *Wf)
{
	const long nn = (long)N * N;
	double *a = malloc(sizeof(double) * 2 * nn);
	for (long i = 0; i < nn; i++) { a[2 * i] = Wv[i]; a[2 * i + 1] = 0; }
	orc_fft2d(a, N, N, -1);
	const double scale = 1.0 / (N * N);
	for (int l = 0; l < N; l++) {
		const int lc = (N - l) % N;
		for (int k = 0; k <= N / 2; k++) {
			Wf[2 * (N * l + k)]     = a[2 * (N * l + k)] * scale;
			Wf[2 * (N * l + k) + 1] = a[2 * (N * l + k) + 1] * scale;
		}
		for (int k = N / 2 + 1; k < N; k++) {
			const int kc = N - k;
			Wf[2 * (N * l + k)]     =  a[2 * (N * lc + kc)] * scale;
			Wf[2 * (N * l + k) + 1] = -a[2 * (N * lc + kc) + 1] * scale;
		}
	}
	free(a);
}

void orc_to_fourier(int N, int ncells, const double *Wv, double *Wf)
{
	const long nn = (long)N * N;
	for (long c = 0; c < 4L * ncells; c++) to_fourier_comp(N, Wv + c * nn, Wf + c * 2 * nn);
}

/* backward c2c N x N, real part (:270-283) */
void orc_from_fourier(int N, int ncells, const double *Wf, double *Wv)
{
	const long nn = (long)N * N;
	double *a = malloc(sizeof(double) * 2 * nn);
	for (long c = 0; c < 4L * ncells; c++) {
		memcpy(a, Wf + c * 2 * nn, sizeof(double) * 2 * nn);
		orc_fft2d(a, N, N, +1);
		for (long i = 0; i < nn; i++) Wv[c * nn + i] = a[2 * i];
	}
	free(a);
}

/* ---- finite volumes (upstream src/finite_volume.c) ----------------------- */

static inline double minmod(double a, double b)   /* :35-38 */
{
	return 0.5 * (copysign(1, a) + copysign(1, b)) * fmin(fabs(a), fabs(b));
}

/* SlopeLimiterStepPeriodic, finite_volume.c:52-104 */
void orc_slope_periodic(double h, double dt, double A, int N, const double *Un, double *Un1)
{
	const double Aabs = fabs(A), nu = dt * A / h;
	const double S = 0.5 * A * (copysign(1, nu) - nu), Sabs = 0.5 * Aabs * (copysign(1, nu) - nu);
	double *al = malloc(sizeof(double) * N), *hb = malloc(sizeof(double) * N);
	for (int j = 0; j < N - 1; j++) al[j] = Un[j + 1] - Un[j];
	al[N - 1] = Un[0] - Un[N - 1];
	for (int j = 1; j < N; j++) hb[j] = minmod(al[j], al[j - 1]);
	hb[0] = minmod(al[0], al[N - 1]);
	const double scale = dt / (2 * h);
	for (int j = 0; j < N; j++) {
		const int jp = (j + 1) % N, jm = (j + N - 1) % N;
		Un1[j] = Un[j] + scale * (
			- A * (Un[jp] - Un[jm]) + Aabs * (Un[jp] - 2 * Un[j] + Un[jm])
			- S * (hb[jp] - hb[jm]) + Sabs * (hb[jp] - 2 * hb[j] + hb[jm]));
	}
	free(hb); free(al);
}

/* SlopeLimiterStepDirichlet, finite_volume.c:118-179 */
void orc_slope_dirichlet(double h, double dt, double A, int N, const double *Un, double *Un1)
{
	const double Aabs = fabs(A), nu = dt * A / h;
	const double S = 0.5 * A * (copysign(1, nu) - nu), Sabs = 0.5 * Aabs * (copysign(1, nu) - nu);
	double *al = malloc(sizeof(double) * N), *hb = malloc(sizeof(double) * N);
	for (int j = 0; j < N - 1; j++) al[j] = Un[j + 1] - Un[j];
	al[N - 1] = 0;
	for (int j = 1; j < N - 1; j++) hb[j] = minmod(al[j], al[j - 1]);
	hb[0] = 0; hb[N - 1] = 0;
	const double scale = dt / (2 * h);
	for (int j = 1; j < N - 1; j++)
		Un1[j] = Un[j] + scale * (
			- A * (Un[j + 1] - Un[j - 1]) + Aabs * (Un[j + 1] - 2 * Un[j] + Un[j - 1])
			- S * (hb[j + 1] - hb[j - 1]) + Sabs * (hb[j + 1] - 2 * hb[j] + hb[j - 1]));
	if (A >= 0) {
		Un1[0] = Un[0];
		Un1[N - 1] = Un[N - 1] + 2 * scale * (- A * (Un[N - 1] - Un[N - 2]) - S * (hb[N - 1] - hb[N - 2]));
	} else {
		Un1[0] = Un[0] + 2 * scale * (- A * (Un[1] - Un[0]) - S * (hb[1] - hb[0]));
		Un1[N - 1] = Un[N - 1];
	}
	free(hb); free(al);
}

/* CalculateRightwardFlux / CalculateLeftwardFlux, finite_volume.c:186-216 */
double orc_flux_right(int m, const double *A, const double *U)
{
	double flux = 0;
	for (int i = 0; i < m / 2; i++) flux += A[i] * U[i];
	return flux;
}

double orc_flux_left(int m, const double *A, const double *U)
{
	double flux = 0;
	for (int i = m / 2; i < m; i++) flux += fabs(A[i]) * U[i];
	return flux;
}

/* SlopeLimiterStepMaxwell, finite_volume.c:241-323; Un is m x N (index i + m*j) */
void orc_slope_maxwell(double h, double dt, int m, const double *A, int N, double lambda, double fluxL, double fluxR,
                       const double *UmaxwL, const double *UmaxwR, const double *Un, double *Un1)
{
	double *Um1 = malloc(sizeof(double) * m), *UN1 = malloc(sizeof(double) * m);
	for (int i = 0; i < m / 2; i++) {
		UN1[i] = Un[i + m * (N - 1)];
		Um1[i] = (1 - lambda) * Un[m - 1 - i] + lambda * fluxL * UmaxwL[i];
	}
	for (int i = m / 2; i < m; i++) {
		Um1[i] = Un[i];
		UN1[i] = (1 - lambda) * Un[m - 1 - i + m * (N - 1)] + lambda * fluxR * UmaxwR[i];
	}
	double *Vb = malloc(sizeof(double) * (N + 4)), *ab = malloc(sizeof(double) * (N + 3)), *hbb = malloc(sizeof(double) * (N + 2));
	double *V = Vb + 2, *al = ab + 2, *hb = hbb + 1;
	for (int i = 0; i < m; i++) {
		const double Aabs = fabs(A[i]), nu = dt * A[i] / h;
		const double S = 0.5 * A[i] * (copysign(1, nu) - nu), Sabs = 0.5 * Aabs * (copysign(1, nu) - nu);
		V[-2] = Um1[i]; V[-1] = Um1[i];
		for (int j = 0; j < N; j++) V[j] = Un[i + m * j];
		V[N] = UN1[i]; V[N + 1] = UN1[i];
		for (int j = -2; j <= N; j++) al[j] = V[j + 1] - V[j];
		for (int j = -1; j <= N; j++) hb[j] = minmod(al[j], al[j - 1]);
		const double scale = dt / (2 * h);
		for (int j = 0; j < N; j++)
			Un1[i + m * j] = V[j] + scale * (
				- A[i] * (V[j + 1] - V[j - 1]) + Aabs * (V[j + 1] - 2 * V[j] + V[j - 1])
				- S * (hb[j + 1] - hb[j - 1]) + Sabs * (hb[j + 1] - 2 * hb[j] + hb[j - 1]));
	}
	free(hbb); free(ab); free(Vb); free(UN1); free(Um1);
}

/* ---- inhomogeneous steps (upstream simulation.c, non-MPI paths) ---------- */

static void vgrid_of(int N, double L, double *vgrid)     /* simulation.c:151-154 */
{
	const double scale = 2 * L / N;
	for (int k = 0; k < N; k++) vgrid[k] = k < N / 2 ? scale * k : scale * (k - N);
}

/* half-step transport of every x-line (simulation.c:426-448); bc 0 periodic, 1 Dirichlet */
static void transport_lines(int N, int numVol, double L, double h, double dt, int bc, const double *W, double *Wout)
{
	const long nn = (long)N * N, cs = 4 * nn;   /* cell stride */
	double *vg = malloc(sizeof(double) * N);
	vgrid_of(N, L, vg);
	double *x = malloc(sizeof(double) * numVol), *x1 = malloc(sizeof(double) * numVol);
	for (long line = 0; line < cs; line++) {
		const int l = (int)((line % nn) / N);
		for (int i = 0; i < numVol; i++) x[i] = W[i * cs + line];
		if (bc == 0) orc_slope_periodic(h, 0.5 * dt, vg[l], numVol, x, x1);
		else         orc_slope_dirichlet(h, 0.5 * dt, vg[l], numVol, x, x1);
		for (int i = 0; i < numVol; i++) Wout[i * cs + line] = x1[i];
	}
	free(x1); free(x);
	free(vg);
}

/* InternalFourierCollisionStep, simulation.c:214-284 (cells i0..i1-1, in place) */
typedef struct { const orc_quad *q; int i0; double dt; const double *Bext; double *Wv; } fc_task;

static void fc_run(int t, void *p)
{
	fc_task *c = p;
	const int N = c->q->N, i = c->i0 + t;
	const long nn = (long)N * N;
	double *Wf = malloc(sizeof(double) * 8 * nn), *Wf2 = malloc(sizeof(double) * 8 * nn);
	orc_to_fourier(N, 1, c->Wv + i * 4 * nn, Wf);
	orc_collision_step(c->q, Wf, c->dt, c->Bext + 3 * i, Wf2);
	orc_from_fourier(N, 1, Wf2, c->Wv + i * 4 * nn);
	free(Wf2); free(Wf);
}

/* cells are independent: with several cells they run in parallel (each
 * cell's integrals then run serially inside its thread) */
static void fourier_collision_cells(const orc_quad *q, int i0, int i1, double dt, const double *Bext, double *Wv)
{
	fc_task ct = { q, i0, dt, Bext, Wv };
	if (i1 - i0 >= 4) par_for(i1 - i0, fc_run, &ct);
	else for (int t = 0; t < i1 - i0; t++) fc_run(t, &ct);
}

/* InhomStepPeriodic (:307-555) and InhomStepDirichlet (:562-830), non-MPI */
void orc_inhom_step(const orc_quad *q, int bc, int numVol, const double *W, double h, double dt, const double *Bext, double *Wnext)
{
	const int N = q->N;
	const long cs = 4L * N * N;
	double *Wtmp = malloc(sizeof(double) * cs * numVol);
	transport_lines(N, numVol, q->L, h, dt, bc, W, Wtmp);
	if (bc == 0) fourier_collision_cells(q, 0, numVol, dt, Bext, Wtmp);
	else         fourier_collision_cells(q, 1, numVol - 1, dt, Bext, Wtmp);
	transport_lines(N, numVol, q->L, h, dt, bc, Wtmp, Wnext);
	free(Wtmp);
}

/* Maxwell velocity remapping (simulation.c:837-872) */
static void to_maxwell(int N, const double *comp, double *maxw)
{
	const long nn = (long)N * N;
	memcpy(maxw, comp + N, sizeof(double) * nn / 2);
	memcpy(maxw + nn / 2, comp + nn / 2, sizeof(double) * nn / 2);
}

static void from_maxwell(int N, const double *maxw, const double *v0, double *comp)
{
	const long nn = (long)N * N;
	memcpy(comp, v0, sizeof(double) * N);
	memcpy(comp + N, maxw, sizeof(double) * (nn / 2 - N));
	memcpy(comp + nn / 2, maxw + nn / 2, sizeof(double) * nn / 2);
}

static void maxwell_transport(int N, int numVol, double h, double dt, double lambda, const double *vx,
                              double fluxL, double fluxR, const double *WLeff, const double *WReff,
                              const double *Win, double *Wout)
{
	const long nn = (long)N * N, cs = 4 * nn;
	double *x = malloc(sizeof(double) * nn * numVol), *x1 = malloc(sizeof(double) * nn * numVol);
	for (int j = 0; j < 4; j++) {
		for (int i = 0; i < numVol; i++) to_maxwell(N, Win + i * cs + j * nn, x + i * nn);
		orc_slope_maxwell(h, 0.5 * dt, (int)nn, vx, numVol, lambda, fluxL, fluxR, WLeff + j * nn, WReff + j * nn, x, x1);
		for (int i = 0; i < numVol; i++) from_maxwell(N, x1 + i * nn, Win + i * cs + j * nn, Wout + i * cs + j * nn);
	}
	free(x1); free(x);
}

/* InhomStepMaxwell, simulation.c:879-1165 (non-MPI path) */
void orc_inhom_step_maxwell(const orc_quad *q, int numVol, const double *W, double h, double dt, double lambda,
                            const double *WMaxwL, const double *WMaxwR, const double *Bext, double *Wnext)
{
	const int N = q->N;
	const long nn = (long)N * N, cs = 4 * nn;
	const double scale = 2 * q->L / N;
	double *vx = malloc(sizeof(double) * nn);
	for (int l = 0; l < N; l++)
		for (int k = 0; k < N; k++) vx[k + N * l] = l < N / 2 ? scale * (l + 1) : scale * (l - N);
	double *WLeff = malloc(sizeof(double) * cs), *WReff = malloc(sizeof(double) * cs);
	for (int j = 0; j < 4; j++) { to_maxwell(N, WMaxwL + j * nn, WLeff + j * nn); to_maxwell(N, WMaxwR + j * nn, WReff + j * nn); }
	const double normL = 1.0 / orc_flux_right((int)nn, vx, WLeff);
	const double normR = 1.0 / orc_flux_left((int)nn, vx, WReff);
	for (long k = 0; k < cs; k++) { WLeff[k] *= normL; WReff[k] *= normR; }
	double *tr = malloc(sizeof(double) * nn);
	to_maxwell(N, W, tr);
	double fluxL = orc_flux_left((int)nn, vx, tr);
	to_maxwell(N, W + (numVol - 1) * cs, tr);
	double fluxR = orc_flux_right((int)nn, vx, tr);
	double *Wtmp = malloc(sizeof(double) * cs * numVol);
	maxwell_transport(N, numVol, h, dt, lambda, vx, fluxL, fluxR, WLeff, WReff, W, Wtmp);
	fourier_collision_cells(q, 0, numVol, dt, Bext, Wtmp);
	to_maxwell(N, Wtmp, tr);
	fluxL = orc_flux_left((int)nn, vx, tr);
	to_maxwell(N, Wtmp + (numVol - 1) * cs, tr);
	fluxR = orc_flux_right((int)nn, vx, tr);
	maxwell_transport(N, numVol, h, dt, lambda, vx, fluxL, fluxR, WLeff, WReff, Wtmp, Wnext);
	free(Wtmp); free(tr); free(WReff); free(WLeff); free(vx);
}

/* SimulationHomogeneous, simulation.c:1219-1281: Wevolv[0] = W0, then steps */
void orc_simulation_homogeneous(const orc_quad *q, const double *W0, double dt, int numsteps, const double B[3], double *Wevolv)
{
	const int N = q->N;
	const long cs = 4L * N * N;
	memcpy(Wevolv, W0, sizeof(double) * cs);
	for (int it = 1; it < numsteps; it++) {
		memcpy(Wevolv + it * cs, Wevolv + (it - 1) * cs, sizeof(double) * cs);
		fourier_collision_cells(q, 0, 1, dt, B, Wevolv + it * cs);
	}
}

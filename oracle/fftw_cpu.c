/* fftw_cpu.c — ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * A CPU implementation of the FFTW-API subset declared in include/fftw3.h,
 * written from the DFT definition (mixed-radix Cooley-Tukey, radix 2 and 3,
 * direct DFT for other prime factors).  It exists so that
 *   - the upstream C sources (which call FFTW, e.g. src/integrals.c:48-51,97)
 *     can be compiled unchanged into oracle/_ref as a checker, and
 *   - the C restatement in oracle/qb_oracle.c has a transform to call.
 * Nothing in the product library links or calls this file.
 *
 * Conventions follow FFTW: FORWARD = exp(-2 pi i jk/n), BACKWARD = exp(+...),
 * unnormalised, row-major 2-D arrays with the last index fastest.  An r2c
 * plan writes the n0 x (n1/2+1) half spectrum.
 */
#include <fftw3.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

typedef struct { double re, im; } cplx;

/* ---- twiddle cache: w[k] = exp(-2 pi i k / n), k < n --------------------- */
#define TW_MAX 64
static struct { int n; cplx *w; } tw_cache[TW_MAX];
static pthread_mutex_t tw_lock = PTHREAD_MUTEX_INITIALIZER;

static const cplx *twiddles(int n)
{
	/* lock-free hit path: a slot's table is published before its size */
	for (int i = 0; i < TW_MAX; i++) {
		int ni = __atomic_load_n(&tw_cache[i].n, __ATOMIC_ACQUIRE);
		if (ni == n) return tw_cache[i].w;
		if (ni == 0) break;
	}
	pthread_mutex_lock(&tw_lock);
	for (int i = 0; i < TW_MAX; i++) {
		if (tw_cache[i].n == n) { const cplx *w = tw_cache[i].w; pthread_mutex_unlock(&tw_lock); return w; }
	}
	cplx *w = malloc((size_t)n * sizeof(cplx));
	for (int k = 0; k < n; k++) {
		double a = -2.0 * M_PI * (double)k / (double)n;
		w[k].re = cos(a);
		w[k].im = sin(a);
	}
	/* exact values at quarter points */
	if (n % 4 == 0) {
		w[0].re = 1; w[0].im = 0;
		w[n/4].re = 0; w[n/4].im = -1;
		w[n/2].re = -1; w[n/2].im = 0;
		w[3*n/4].re = 0; w[3*n/4].im = 1;
	}
	int slot = -1;
	for (int i = 0; i < TW_MAX; i++) if (tw_cache[i].n == 0) { slot = i; break; }
	if (slot < 0) { pthread_mutex_unlock(&tw_lock); abort(); }   /* more distinct sizes than any caller uses */
	tw_cache[slot].w = w;
	__atomic_store_n(&tw_cache[slot].n, n, __ATOMIC_RELEASE);
	pthread_mutex_unlock(&tw_lock);
	return w;
}

/* twiddle exp(sign * 2 pi i e / n) from the forward table; every caller
 * passes 0 <= e < n (exponents are reduced by construction) */
static inline cplx tw_get(const cplx *w, int n, long e, int sign)
{
	(void)n;
	cplx t = w[e];
	if (sign > 0) t.im = -t.im;
	return t;
}

static inline cplx cmul(cplx a, cplx b) { cplx r = { a.re*b.re - a.im*b.im, a.re*b.im + a.im*b.re }; return r; }

/* Recursive mixed-radix DFT of length n with input stride `is`,
 * out[k] = sum_j in[j*is] exp(sign 2 pi i jk/n); `w` is the table for the
 * top-level length `ntop` (n divides ntop), scratch has room for n values. */
static void dft_rec(const cplx *in, long is, cplx *out, int n, int sign, const cplx *w, int ntop, cplx *scratch)
{
	if (n == 1) { out[0] = in[0]; return; }
	int p;
	if (n % 4 == 0) p = 4;
	else if (n % 2 == 0) p = 2;
	else if (n % 3 == 0) p = 3;
	else { p = 0; for (int d = 5; d * d <= n; d += 2) if (n % d == 0) { p = d; break; } if (!p || p > 64) p = n; }

	const int m = n / p;
	const int step = ntop / n;   /* w_n^e = w_ntop^(e*step) */
	if (p == n) {
		/* direct DFT of prime length */
		for (int k = 0; k < n; k++) {
			cplx s = { 0, 0 };
			for (int j = 0; j < n; j++) {
				cplx t = tw_get(w, ntop, (long)j * k % n * step, sign);
				cplx x = in[j * is];
				s.re += x.re*t.re - x.im*t.im;
				s.im += x.re*t.im + x.im*t.re;
			}
			out[k] = s;
		}
		return;
	}
	/* decimation in time: sub-transforms of the p residue classes */
	for (int r = 0; r < p; r++)
		dft_rec(in + r * is, is * p, scratch + r * m, m, sign, w, ntop, out);
	/* combine: out[k + m*q] = sum_r w_n^{r(k+m q)} sub_r[k] */
	for (int k = 0; k < m; k++) {
		cplx v[16];
		cplx vs[64];
		cplx *vv = (p <= 16) ? v : vs;
		for (int r = 0; r < p; r++) vv[r] = cmul(scratch[r * m + k], tw_get(w, ntop, (long)r * k * step, sign));
		if (p == 2) {
			out[k].re = vv[0].re + vv[1].re; out[k].im = vv[0].im + vv[1].im;
			out[k + m].re = vv[0].re - vv[1].re; out[k + m].im = vv[0].im - vv[1].im;
		} else if (p == 4) {
			cplx a = { vv[0].re + vv[2].re, vv[0].im + vv[2].im };
			cplx b = { vv[0].re - vv[2].re, vv[0].im - vv[2].im };
			cplx c = { vv[1].re + vv[3].re, vv[1].im + vv[3].im };
			cplx d = { vv[1].re - vv[3].re, vv[1].im - vv[3].im };
			/* multiply d by sign*i */
			cplx di = (sign < 0) ? (cplx){ d.im, -d.re } : (cplx){ -d.im, d.re };
			out[k].re = a.re + c.re;           out[k].im = a.im + c.im;
			out[k + m].re = b.re + di.re;      out[k + m].im = b.im + di.im;
			out[k + 2*m].re = a.re - c.re;     out[k + 2*m].im = a.im - c.im;
			out[k + 3*m].re = b.re - di.re;    out[k + 3*m].im = b.im - di.im;
		} else {
			for (int q = 0; q < p; q++) {
				cplx s = { 0, 0 };
				for (int r = 0; r < p; r++) {
					cplx t = tw_get(w, ntop, (long)r * q % p * (ntop / p), sign);
					s.re += vv[r].re*t.re - vv[r].im*t.im;
					s.im += vv[r].re*t.im + vv[r].im*t.re;
				}
				out[k + m * q] = s;
			}
		}
	}
}

/* 1-D transform of n values at stride `stride` (in place, via a buffer) */
static void fft1d_strided(cplx *data, long stride, int n, int sign, cplx *buf)
{
	const cplx *w = twiddles(n);
	cplx *in = buf, *out = buf + n, *scr = buf + 2 * n;
	for (int j = 0; j < n; j++) in[j] = data[j * stride];
	dft_rec(in, 1, out, n, sign, w, n, scr);
	for (int j = 0; j < n; j++) data[j * stride] = out[j];
}

/* 2-D complex transform in place: rows (length n1) then columns (length n0) */
static void fft2d_inplace(cplx *a, int n0, int n1, int sign)
{
	int nmax = n0 > n1 ? n0 : n1;
	cplx *buf = malloc((size_t)4 * nmax * sizeof(cplx));
	for (int r = 0; r < n0; r++) fft1d_strided(a + (long)r * n1, 1, n1, sign, buf);
	for (int c = 0; c < n1; c++) fft1d_strided(a + c, n1, n0, sign, buf);
	free(buf);
}

/* ---- FFTW API ------------------------------------------------------------ */

struct fftw_plan_s {
	int r2c;
	int n0, n1, sign;
	void *in;
	fftw_complex *out;
};

void *fftw_malloc(size_t n)
{
	void *p = NULL;
	if (posix_memalign(&p, 64, n ? n : 1) != 0) return NULL;
	return p;
}

void fftw_free(void *p) { free(p); }

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned flags)
{
	(void)flags;
	fftw_plan p = calloc(1, sizeof(*p));
	p->r2c = 0; p->n0 = n0; p->n1 = n1; p->sign = sign; p->in = in; p->out = out;
	return p;
}

fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out, unsigned flags)
{
	(void)flags;
	fftw_plan p = calloc(1, sizeof(*p));
	p->r2c = 1; p->n0 = n0; p->n1 = n1; p->sign = FFTW_FORWARD; p->in = in; p->out = out;
	return p;
}

void fftw_execute(const fftw_plan p)
{
	const long n = (long)p->n0 * p->n1;
	cplx *a = malloc((size_t)n * sizeof(cplx));
	if (p->r2c) {
		const double *x = (const double *)p->in;
		for (long i = 0; i < n; i++) { a[i].re = x[i]; a[i].im = 0; }
	} else {
		memcpy(a, p->in, (size_t)n * sizeof(cplx));
	}
	fft2d_inplace(a, p->n0, p->n1, p->sign);
	if (p->r2c) {
		const int nh = p->n1 / 2 + 1;
		for (int r = 0; r < p->n0; r++)
			for (int c = 0; c < nh; c++) {
				p->out[(long)r * nh + c][0] = a[(long)r * p->n1 + c].re;
				p->out[(long)r * nh + c][1] = a[(long)r * p->n1 + c].im;
			}
	} else {
		memcpy(p->out, a, (size_t)n * sizeof(cplx));
	}
	free(a);
}

void fftw_destroy_plan(fftw_plan p) { free(p); }

void fftw_cleanup(void) {}

/* Direct entry for the oracle restatement: 2-D complex transform in place. */
void orc_fft2d(double *a, int n0, int n1, int sign)
{
	fft2d_inplace((cplx *)a, n0, n1, sign);
}

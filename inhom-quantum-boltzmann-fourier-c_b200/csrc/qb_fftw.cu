// qb_fftw.cu — the FFTW-API subset of include/fftw3.h, executed on the GPU.
//
// The upstream drivers plan and execute FFTW transforms themselves (for
// example test/Cc_test.c:104-106 transforms W to Fourier space with an r2c
// plan).  libqbgpu provides those symbols so the drivers link unchanged; a
// planned transform runs on the GPU through the project's FFT kernels (square
// 8..64 grids).  Other shapes are rejected loudly: there is no host FFT here.
#include "qb_engine.h"

extern "C" {
#include <fftw3.h>
}

#include <cstdlib>
#include <cstring>

struct fftw_plan_s {
	int r2c, n0, n1, sign;
	void *in;
	fftw_complex *out;
};

namespace {
struct Ctx {
	int device = -1;
	cudaStream_t s = nullptr;
	qb::DevBuf buf;
	~Ctx() { if (s) cudaStreamDestroy(s); }
};
Ctx &ctx() {
	thread_local Ctx c;
	int d = 0;
	QB_CUDA(cudaGetDevice(&d));
	if (c.s == nullptr || c.device != d) {
		if (c.s) cudaStreamDestroy(c.s);
		c.buf.release();
		QB_CUDA(cudaStreamCreateWithFlags(&c.s, cudaStreamNonBlocking));
		c.device = d;
	}
	return c;
}

fftw_plan make_plan(int r2c, int n0, int n1, int sign, void *in, fftw_complex *out) {
	if (!qb::fft2_generic_supported(n0, n1))
		QB_FAIL("fftw_plan: only square 8x8 .. 64x64 transforms are provided (requested " + std::to_string(n0) + "x" + std::to_string(n1) + ")");
	if (sign != FFTW_FORWARD && sign != FFTW_BACKWARD) QB_FAIL("fftw_plan: sign must be FFTW_FORWARD or FFTW_BACKWARD");
	fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
	p->r2c = r2c; p->n0 = n0; p->n1 = n1; p->sign = sign; p->in = in; p->out = out;
	return p;
}
}  // namespace

extern "C" {

void *fftw_malloc(size_t n) {
	void *p = nullptr;
	if (posix_memalign(&p, 64, n ? n : 1) != 0) return nullptr;
	return p;
}

void fftw_free(void *p) { free(p); }

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned flags) {
	(void)flags;
	return make_plan(0, n0, n1, sign, in, out);
}

fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out, unsigned flags) {
	(void)flags;
	return make_plan(1, n0, n1, FFTW_FORWARD, in, out);
}

void fftw_execute(const fftw_plan p) {
	if (p == nullptr) QB_FAIL("fftw_execute: null plan");
	Ctx &c = ctx();
	const size_t n = (size_t)p->n0 * p->n1;
	const size_t ib = p->r2c ? n * sizeof(double) : n * sizeof(fftw_complex);
	const size_t ob = p->r2c ? (size_t)p->n0 * (p->n1 / 2 + 1) * sizeof(fftw_complex) : n * sizeof(fftw_complex);
	c.buf.ensure(ib + ob + 16);
	char *d = c.buf.as<char>();
	double2 *dout = (double2 *)(d + ((ib + 15) & ~(size_t)15));
	QB_CUDA(cudaMemcpyAsync(d, p->in, ib, cudaMemcpyHostToDevice, c.s));
	qb::fft2_generic(p->n0, p->sign, p->r2c != 0, d, dout, c.s);
	QB_CUDA(cudaMemcpyAsync(p->out, dout, ob, cudaMemcpyDeviceToHost, c.s));
	QB_CUDA(cudaStreamSynchronize(c.s));
}

void fftw_destroy_plan(fftw_plan p) { free(p); }

void fftw_cleanup(void) {}

}  // extern "C"

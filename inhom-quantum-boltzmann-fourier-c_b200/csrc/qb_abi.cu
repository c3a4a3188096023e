// qb_abi.cu — the upstream C API (include/*.h, compile-time N_GRID) on the GPU engine.
//
// Every entry point keeps the upstream signature and argument meaning.  Host
// inputs are copied to the device, the engine evaluates on the GPU, results
// are copied back, and the call returns once they are on the host.  There is
// no CPU fallback: a CUDA failure is reported (qb_last_error) and, unless
// QB_ABORT_ON_ERROR=0, aborts the process.
#include "qb_engine.h"

extern "C" {
#include "simulation.h"
#include "finite_volume.h"
#include "util.h"
}

#include <cstdlib>
#include <cstring>
#include <unordered_map>
#include <vector>

namespace {

constexpr int NG = N_GRID;
constexpr long NN = (long)NG * NG;
constexpr long PP = 4 * NN;

// ---- quadrature registry ----------------------------------------------------
// Tables built by FourierI1..I4 keep a compact device copy keyed by the host
// psiR1 pointer (upstream stores J*J duplicated grids for I1; the device copy
// stores J folded terms).  Tables filled by the caller (test/I2_test.c builds
// quadI2_t by hand) are uploaded as generic term lists on every call.
enum Kind { K_I1 = 1, K_I2, K_I3, K_I4 };
struct Entry {
	Kind kind;
	int device;
	unsigned num;
	qb::DevI1 i1;
	qb::DevI2 i2;
	qb::DevI3 i3;
};
std::mutex g_reg_mu;
std::unordered_map<const void *, std::unique_ptr<Entry>> g_reg;

int cur_device() { int d = 0; QB_CUDA(cudaGetDevice(&d)); return d; }

Entry *lookup(const void *key, Kind kind, unsigned num) {
	std::lock_guard<std::mutex> lk(g_reg_mu);
	auto it = g_reg.find(key);
	if (it == g_reg.end()) return nullptr;
	Entry *e = it->second.get();
	if (e->kind != kind || e->num != num || e->device != cur_device()) return nullptr;
	return e;
}

void reg_put(const void *key, std::unique_ptr<Entry> e) {
	std::lock_guard<std::mutex> lk(g_reg_mu);
	g_reg[key] = std::move(e);
}

void reg_drop(const void *key) {
	std::lock_guard<std::mutex> lk(g_reg_mu);
	g_reg.erase(key);
}

// per-thread helper workspace for entry points without an interm struct
qb_workspace &thread_ws() {
	thread_local std::unique_ptr<qb_workspace> ws;
	if (!ws || ws->device != cur_device()) ws = std::make_unique<qb_workspace>(NG);
	return *ws;
}

qb_workspace *need(qb_workspace *ws, const char *fn) {
	if (ws == nullptr) QB_FAIL(std::string(fn) + ": intermediate struct was not created (call the matching *_Create first)");
	return ws;
}

void h2d(void *dst, const void *src, size_t bytes, cudaStream_t s) { QB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s)); }
void d2h(void *dst, const void *src, size_t bytes, cudaStream_t s) { QB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s)); }
void sync(cudaStream_t s) { QB_CUDA(cudaStreamSynchronize(s)); }

// device table views for a quad struct (registered or uploaded into `tmp`)
const qb::DevI1 *dev_quad1(const quadI1_t *q, Kind kind, qb::DevI1 &tmp, cudaStream_t s) {
	if (Entry *e = lookup(q->psiR1, kind, q->num)) return &e->i1;
	if (Entry *e = lookup(q->psiR1, kind == K_I1 ? K_I4 : K_I1, q->num)) return &e->i1;
	qb::upload_i1(NG, (int)q->num, (const double *)q->psiR1, (const double *)q->psiR2, tmp, s);
	return &tmp;
}
const qb::DevI2 *dev_quad2(const quadI2_t *q, qb::DevI2 &tmp, cudaStream_t s) {
	if (Entry *e = lookup(q->psiR1, K_I2, q->num)) return &e->i2;
	qb::upload_i2(NG, (int)q->num, (const double *)q->psiR1, (const double *)q->psiR2, tmp, s);
	return &tmp;
}
const qb::DevI3 *dev_quad3(const quadI3_t *q, qb::DevI3 &tmp, cudaStream_t s) {
	if (Entry *e = lookup(q->psiR1, K_I3, q->num)) return &e->i3;
	qb::upload_i3(NG, (int)q->num, (const double *)q->psiR1, (const double *)q->psiR2, tmp, s);
	return &tmp;
}

struct Quads {
	qb::DevI1 t1, t4; qb::DevI2 t2; qb::DevI3 t3;
	qb::QuadSet set;
	Quads(const quadI1_t *q1, const quadI2_t *q2, const quadI3_t *q3, const quadI1_t *q4, cudaStream_t s) {
		if (q1) set.i1 = dev_quad1(q1, K_I1, t1, s);
		if (q2) set.i2 = dev_quad2(q2, t2, s);
		if (q3) set.i3 = dev_quad3(q3, t3, s);
		if (q4) set.i4 = dev_quad1(q4, K_I4, t4, s);
	}
};

void alloc_ws(qb_workspace **slot) { *slot = new qb_workspace(NG); }
void free_ws(qb_workspace **slot) { delete *slot; *slot = nullptr; }

}  // namespace

// ---- grid.h (upstream src/grid.c) --------------------------------------------
// Pointwise products and pad/extract run as GPU kernels on copies of the
// caller's grids, with explicitly rounded products (no FMA contraction) so the
// results equal upstream's double arithmetic.
namespace {
__global__ void k_pointwise(long n, int mode, const double *__restrict__ f, const double *__restrict__ g, double *__restrict__ r) {
	const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	switch (mode) {
	case 0: r[i] = __dmul_rn(f[i], g[i]); break;                                                        // RR
	case 1: r[2 * i] = __dmul_rn(f[i], g[2 * i]); r[2 * i + 1] = __dmul_rn(f[i], g[2 * i + 1]); break;     // RC
	case 2: {                                                                                           // CC
		const double a = f[2 * i], b = f[2 * i + 1], c = g[2 * i], d = g[2 * i + 1];
		r[2 * i] = __dsub_rn(__dmul_rn(a, c), __dmul_rn(b, d)); r[2 * i + 1] = __dadd_rn(__dmul_rn(a, d), __dmul_rn(b, c)); break;
	}
	case 3: r[i] = __dmul_rn(r[i], f[i]); break;                                                        // assign RR
	case 4: r[2 * i] = __dmul_rn(r[2 * i], f[i]); r[2 * i + 1] = __dmul_rn(r[2 * i + 1], f[i]); break;      // assign RC
	case 5: {                                                                                           // assign CC
		const double re = r[2 * i], im = r[2 * i + 1], a = f[2 * i], b = f[2 * i + 1];
		r[2 * i] = __dsub_rn(__dmul_rn(a, re), __dmul_rn(b, im)); r[2 * i + 1] = __dadd_rn(__dmul_rn(a, im), __dmul_rn(b, re)); break;
	}
	}
}
// GridZeroPad (dir 0) / GridExtract (dir 1)
__global__ void k_padx(int N, int dir, const double2 *__restrict__ in, double2 *__restrict__ out) {
	const int P = 2 * N;
	const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
	if (dir == 0) {
		if (i >= (long)P * P) return;
		const int lp = (int)(i / P), kp = (int)(i % P);
		const int l = lp < N / 2 ? lp : (lp >= 3 * N / 2 ? lp - N : -1);
		const int k = kp < N / 2 ? kp : (kp >= 3 * N / 2 ? kp - N : -1);
		out[i] = (l >= 0 && k >= 0) ? in[k + N * l] : make_double2(0.0, 0.0);
	} else {
		if (i >= (long)N * N) return;
		const int l = (int)(i / N), k = (int)(i % N);
		const int lp = l < N / 2 ? l : l + N, kp = k < N / 2 ? k : k + N;
		out[i] = in[kp + P * lp];
	}
}

// r (n values; complex when `rc`) = op(f, g, r)
void pointwise(int mode, long n, const void *f, size_t fb, const void *g, size_t gb, void *r, size_t rb, bool r_in) {
	qb_workspace &ws = thread_ws();
	cudaStream_t s = ws.stream;
	ws.io_in.ensure(fb + gb + rb);
	char *d = ws.io_in.as<char>();
	h2d(d, f, fb, s);
	if (g) h2d(d + fb, g, gb, s);
	if (r_in) h2d(d + fb + gb, r, rb, s);
	k_pointwise<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, mode, (const double *)d, (const double *)(d + fb), (double *)(d + fb + gb));
	QB_CUDA(cudaGetLastError());
	d2h(r, d + fb + gb, rb, s);
	sync(s);
}

void padx(int dir, const void *in, void *out) {
	qb_workspace &ws = thread_ws();
	cudaStream_t s = ws.stream;
	const size_t ib = sizeof(double2) * (dir == 0 ? NN : PP), ob = sizeof(double2) * (dir == 0 ? PP : NN);
	ws.io_in.ensure(ib + ob);
	char *d = ws.io_in.as<char>();
	h2d(d, in, ib, s);
	const long n = dir == 0 ? PP : NN;
	k_padx<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(NG, dir, (const double2 *)d, (double2 *)(d + ib));
	QB_CUDA(cudaGetLastError());
	d2h(out, d + ib, ob, s);
	sync(s);
}
}  // namespace

extern "C" {

void MultiplyPointwiseRR(const grid_t *restrict_ f, const grid_t *restrict_ g, grid_t *restrict_ ret) {
	pointwise(0, NN, f, sizeof(grid_t), g, sizeof(grid_t), ret, sizeof(grid_t), false);
}
void MultiplyPointwiseRC(const grid_t *restrict_ f, const cgrid_t *restrict_ g, cgrid_t *restrict_ ret) {
	pointwise(1, NN, f, sizeof(grid_t), g, sizeof(cgrid_t), ret, sizeof(cgrid_t), false);
}
void MultiplyPointwiseCC(const cgrid_t *restrict_ f, const cgrid_t *restrict_ g, cgrid_t *restrict_ ret) {
	pointwise(2, NN, f, sizeof(cgrid_t), g, sizeof(cgrid_t), ret, sizeof(cgrid_t), false);
}
void MultiplyPointwiseRR2(const grid2_t *restrict_ f, const grid2_t *restrict_ g, grid2_t *restrict_ ret) {
	pointwise(0, PP, f, sizeof(grid2_t), g, sizeof(grid2_t), ret, sizeof(grid2_t), false);
}
void MultiplyPointwiseCC2(const cgrid2_t *restrict_ f, const cgrid2_t *restrict_ g, cgrid2_t *restrict_ ret) {
	pointwise(2, PP, f, sizeof(cgrid2_t), g, sizeof(cgrid2_t), ret, sizeof(cgrid2_t), false);
}
void MultiplyPointwiseAssignRR(const grid_t *restrict_ f, grid_t *restrict_ ret) {
	pointwise(3, NN, f, sizeof(grid_t), nullptr, 0, ret, sizeof(grid_t), true);
}
void MultiplyPointwiseAssignRC(const grid_t *restrict_ f, cgrid_t *restrict_ ret) {
	pointwise(4, NN, f, sizeof(grid_t), nullptr, 0, ret, sizeof(cgrid_t), true);
}
void MultiplyPointwiseAssignRC2(const grid2_t *restrict_ f, cgrid2_t *restrict_ ret) {
	pointwise(4, PP, f, sizeof(grid2_t), nullptr, 0, ret, sizeof(cgrid2_t), true);
}
void MultiplyPointwiseAssignCC2(const cgrid2_t *restrict_ f, cgrid2_t *restrict_ ret) {
	pointwise(5, PP, f, sizeof(cgrid2_t), nullptr, 0, ret, sizeof(cgrid2_t), true);
}
void GridZeroPad(const cgrid_t *restrict_ f, cgrid2_t *restrict_ ret) { padx(0, f, ret); }
void GridExtract(const cgrid2_t *restrict_ f, cgrid_t *restrict_ ret) { padx(1, f, ret); }

// ---- quadrature.h (upstream src/quadrature.c) -----------------------------------
void QuadI1_Allocate(const unsigned int num, quadI1_t *quad) {
	quad->num = num;
	quad->psiR1 = (grid2_t *)fftw_malloc(num * sizeof(grid2_t));
	quad->psiR2 = (grid_t *)fftw_malloc(num * sizeof(grid_t));
}
void QuadI1_Delete(quadI1_t *quad) {
	reg_drop(quad->psiR1);
	fftw_free(quad->psiR2);
	fftw_free(quad->psiR1);
	quad->num = 0;
}
void QuadI2_Allocate(const unsigned int num, quadI2_t *quad) {
	quad->num = num;
	quad->psiR1 = (grid_t *)fftw_malloc(num * sizeof(grid_t));
	quad->psiR2 = (grid_t *)fftw_malloc(num * sizeof(grid_t));
}
void QuadI2_Delete(quadI2_t *quad) {
	reg_drop(quad->psiR1);
	fftw_free(quad->psiR2);
	fftw_free(quad->psiR1);
	quad->num = 0;
}
void QuadI3_Allocate(const unsigned int num, quadI3_t *quad) {
	quad->num = num;
	quad->psiR1 = (cgrid_t *)fftw_malloc(num * sizeof(cgrid_t));
	quad->psiR2 = (grid2_t *)fftw_malloc(num * sizeof(grid2_t));
}
void QuadI3_Delete(quadI3_t *quad) {
	reg_drop(quad->psiR1);
	fftw_free(quad->psiR2);
	fftw_free(quad->psiR1);
	quad->num = 0;
}

void FourierI1(const unsigned int J, const double L, const double R, quadI1_t *quad) {
	QuadI1_Allocate(J * J, quad);
	auto e = std::make_unique<Entry>();
	e->kind = K_I1; e->device = cur_device(); e->num = J * J;
	qb::build_i1(NG, (int)J, L, R, e->i1, (double *)quad->psiR1, (double *)quad->psiR2, thread_ws().stream);
	reg_put(quad->psiR1, std::move(e));
}
void FourierI2(const unsigned int J, const double L, const double R, quadI2_t *quad) {
	QuadI2_Allocate(J, quad);
	auto e = std::make_unique<Entry>();
	e->kind = K_I2; e->device = cur_device(); e->num = J;
	qb::build_i2(NG, (int)J, L, R, e->i2, (double *)quad->psiR1, (double *)quad->psiR2, thread_ws().stream);
	reg_put(quad->psiR1, std::move(e));
}
void FourierI3(const unsigned int J, const double L, const double R, const unsigned int M, quadI3_t *quad) {
	QuadI3_Allocate(J * M, quad);
	auto e = std::make_unique<Entry>();
	e->kind = K_I3; e->device = cur_device(); e->num = J * M;
	qb::build_i3(NG, (int)J, L, R, (int)M, e->i3, (double *)quad->psiR1, (double *)quad->psiR2, thread_ws().stream);
	reg_put(quad->psiR1, std::move(e));
}
void FourierI4(const unsigned int J, const double L, const double R, quadI1_t *quad) {
	QuadI1_Allocate(J, quad);
	auto e = std::make_unique<Entry>();
	e->kind = K_I4; e->device = cur_device(); e->num = J;
	qb::build_i4(NG, (int)J, L, R, e->i1, (double *)quad->psiR1, (double *)quad->psiR2, thread_ws().stream);
	reg_put(quad->psiR1, std::move(e));
}
void LegendreGaussQuad(const unsigned int M, const double a, const double b, double *x, double *w) {
	qb::lgwt_device((int)M, a, b, x, w, thread_ws().stream);
}

// ---- integrals.h (upstream src/integrals.c) ------------------------------------
void I1interm_Create(I1interm_t *interm) { alloc_ws(&interm->ws); }
void I1interm_Delete(I1interm_t *interm) { free_ws(&interm->ws); }
void I2interm_Create(I2interm_t *interm) { alloc_ws(&interm->ws); }
void I2interm_Delete(I2interm_t *interm) { free_ws(&interm->ws); }
void I3interm_Create(I3interm_t *interm) { alloc_ws(&interm->ws); }
void I3interm_Delete(I3interm_t *interm) { free_ws(&interm->ws); }

#define QB_INTEGRAL_BODY(UPLOAD_QUAD, CALL)                                                         \
	qb_workspace &ws = *need(interm->ws, __func__);                                                  \
	cudaStream_t s = ws.stream;                                                                      \
	ws.io_in.ensure(sizeof(cgrid_t) * 4);                                                            \
	double2 *d = ws.io_in.as<double2>();                                                             \
	h2d(d, f, sizeof(cgrid_t), s); h2d(d + NN, g, sizeof(cgrid_t), s); h2d(d + 2 * NN, h, sizeof(cgrid_t), s); \
	UPLOAD_QUAD;                                                                                     \
	CALL;                                                                                            \
	d2h(out, d + 3 * NN, sizeof(cgrid_t), s);                                                        \
	sync(s);

void I1integral(const cgrid_t *restrict_ f, const cgrid_t *restrict_ g, const cgrid_t *restrict_ h, const quadI1_t *restrict_ quad, I1interm_t *restrict_ interm, cgrid_t *restrict_ I1) {
	cgrid_t *out = I1;
	qb::DevI1 tmp;
	QB_INTEGRAL_BODY(const qb::DevI1 *t = dev_quad1(quad, K_I1, tmp, s),
	                 qb::integral_i1(ws, *t, d, d + NN, d + 2 * NN, d + 3 * NN, s))
}
void I2integral(const cgrid_t *restrict_ f, const cgrid_t *restrict_ g, const cgrid_t *restrict_ h, const quadI2_t *restrict_ quad, I2interm_t *restrict_ interm, cgrid_t *restrict_ I2) {
	cgrid_t *out = I2;
	qb::DevI2 tmp;
	QB_INTEGRAL_BODY(const qb::DevI2 *t = dev_quad2(quad, tmp, s),
	                 qb::integral_i2(ws, *t, d, d + NN, d + 2 * NN, d + 3 * NN, s))
}
void I3integral(const cgrid_t *restrict_ f, const cgrid_t *restrict_ g, const cgrid_t *restrict_ h, const quadI3_t *restrict_ quad, I3interm_t *restrict_ interm, cgrid_t *restrict_ I3) {
	cgrid_t *out = I3;
	qb::DevI3 tmp;
	QB_INTEGRAL_BODY(const qb::DevI3 *t = dev_quad3(quad, tmp, s),
	                 qb::integral_i3(ws, *t, d, d + NN, d + 2 * NN, d + 3 * NN, s))
}

// ---- collision.h (upstream src/collision.c) --------------------------------------
void CdInterm_Create(CdInterm_t *interm) { alloc_ws(&interm->ws); }
void CdInterm_Delete(CdInterm_t *interm) { free_ws(&interm->ws); }
void CcInterm_Create(CcInterm_t *interm) { alloc_ws(&interm->ws); }
void CcInterm_Delete(CcInterm_t *interm) { free_ws(&interm->ws); }

static void operators_call(qb_workspace &ws, const wignerF_t *W, const Quads &q, int parts, wignerF_t *out) {
	cudaStream_t s = ws.stream;
	ws.io_in.ensure(sizeof(wignerF_t) * 2);
	double2 *d = ws.io_in.as<double2>();
	h2d(d, W, sizeof(wignerF_t), s);
	qb::collision_operators(ws, q.set, 1, d, parts, parts == qb::RHS_CC ? d + 4 * NN : nullptr,
	                        parts == qb::RHS_CD ? d + 4 * NN : nullptr, s);
	d2h(out, d + 4 * NN, sizeof(wignerF_t), s);
	sync(s);
}

void CdInt(const wignerF_t *restrict_ W, const quadI2_t *restrict_ quadI2, const quadI3_t *restrict_ quadI3, const quadI1_t *restrict_ quadI4, CdInterm_t *restrict_ interm, wignerF_t *restrict_ Cd) {
	qb_workspace &ws = *need(interm->ws, __func__);
	Quads q(nullptr, quadI2, quadI3, quadI4, ws.stream);
	operators_call(ws, W, q, qb::RHS_CD, Cd);
}

void CcInt(const wignerF_t *restrict_ W, const quadI1_t *restrict_ quadI1, CcInterm_t *restrict_ interm, wignerF_t *restrict_ Cc) {
	qb_workspace &ws = *need(interm->ws, __func__);
	Quads q(quadI1, nullptr, nullptr, nullptr, ws.stream);
	operators_call(ws, W, q, qb::RHS_CC, Cc);
}

// ---- simulation.h (upstream src/simulation.c) -------------------------------------
void CollisionInterm_Create(collisionInterm_t *interm) { alloc_ws(&interm->ws); }
void CollisionInterm_Delete(collisionInterm_t *interm) { free_ws(&interm->ws); }

void CollisionStep(const wignerF_t *restrict_ W, const quadI1_t *restrict_ quadI1, const quadI2_t *restrict_ quadI2, const quadI3_t *restrict_ quadI3, const quadI1_t *restrict_ quadI4,
                   const double dt, const double Bext[3], collisionInterm_t *restrict_ interm, wignerF_t *restrict_ Wnext) {
	qb_workspace &ws = *need(interm->ws, __func__);
	cudaStream_t s = ws.stream;
	Quads q(quadI1, quadI2, quadI3, quadI4, s);
	ws.io_in.ensure(sizeof(wignerF_t) * 2 + 64);
	double2 *d = ws.io_in.as<double2>();
	double *B = (double *)(d + 8 * NN);
	h2d(d, W, sizeof(wignerF_t), s);
	h2d(B, Bext, 3 * sizeof(double), s);
	qb::collision_step(ws, q.set, 1, d, B, dt, d + 4 * NN, s);
	d2h(Wnext, d + 4 * NN, sizeof(wignerF_t), s);
	sync(s);
}

void InhomStepInterm_Create(const unsigned int numVol, const double L, inhomStepInterm_t *interm) {
	interm->numVol = numVol;
	const double scale = (2 * L) / N_GRID;
	for (int k = 0; k < N_GRID; k++) interm->vgrid[k] = k < N_GRID / 2 ? scale * k : scale * (k - N_GRID);   // simulation.c:151-154
	for (int l = 0; l < N_GRID; l++)                                                                          // simulation.c:156-162
		for (int k = 0; k < N_GRID; k++)
			interm->vxgridMaxw.data[k + N_GRID * l] = l < N_GRID / 2 ? scale * (l + 1) : scale * (l - N_GRID);
	alloc_ws(&interm->ws);
	// device velocity tables: the transport velocity of every point of a cell
	// ([4][N*N], v_x = vgrid of the slow index) followed by the Maxwell grid
	std::vector<double> A(5 * NN);
	for (long j = 0; j < 4 * NN; j++) A[j] = interm->vgrid[(j % NN) / NG];
	memcpy(A.data() + 4 * NN, interm->vxgridMaxw.data, sizeof(double) * NN);
	interm->ws->vgrid.ensure(sizeof(double) * 5 * NN);
	h2d(interm->ws->vgrid.p, A.data(), sizeof(double) * 5 * NN, interm->ws->stream);
	sync(interm->ws->stream);
}

void InhomStepInterm_Delete(inhomStepInterm_t *interm) { free_ws(&interm->ws); }

static void inhom_call(const wignerV_t *W, const Quads &q, double h, double dt, const double *Bext, inhomStepInterm_t *interm, wignerV_t *Wnext, int bc) {
	qb_workspace &ws = *need(interm->ws, "InhomStep");
	cudaStream_t s = ws.stream;
	const unsigned n = interm->numVol;
	ws.io_in.ensure(sizeof(wignerV_t) * n);
	ws.io_out.ensure(sizeof(wignerV_t) * n);
	ws.bext.ensure(sizeof(double) * 3 * n);
	h2d(ws.io_in.p, W, sizeof(wignerV_t) * n, s);
	h2d(ws.bext.p, Bext, sizeof(double) * 3 * n, s);
	qb::inhom_step(ws, q.set, (int)n, ws.io_in.as<double>(), ws.io_out.as<double>(), ws.vgrid.as<double>(), h, dt, ws.bext.as<double>(), bc, s);
	d2h(Wnext, ws.io_out.p, sizeof(wignerV_t) * n, s);
	sync(s);
}

void InhomStepPeriodic(const wignerV_t *restrict_ W, const quadI1_t *restrict_ quadI1, const quadI2_t *restrict_ quadI2, const quadI3_t *restrict_ quadI3, const quadI1_t *restrict_ quadI4,
                       const double h, const double dt, const double *restrict_ Bext, inhomStepInterm_t *restrict_ interm, wignerV_t *restrict_ Wnext) {
	Quads q(quadI1, quadI2, quadI3, quadI4, need(interm->ws, __func__)->stream);
	inhom_call(W, q, h, dt, Bext, interm, Wnext, 0);
}

void InhomStepDirichlet(const wignerV_t *restrict_ W, const quadI1_t *restrict_ quadI1, const quadI2_t *restrict_ quadI2, const quadI3_t *restrict_ quadI3, const quadI1_t *restrict_ quadI4,
                        const double h, const double dt, const double *restrict_ Bext, inhomStepInterm_t *restrict_ interm, wignerV_t *restrict_ Wnext) {
	Quads q(quadI1, quadI2, quadI3, quadI4, need(interm->ws, __func__)->stream);
	inhom_call(W, q, h, dt, Bext, interm, Wnext, 1);
}

static void maxwell_call(const wignerV_t *W, const Quads &q, double h, double dt, double lambda, const wignerV_t *WL, const wignerV_t *WR,
                         const double *Bext, inhomStepInterm_t *interm, wignerV_t *Wnext, unsigned numsteps, wignerV_t *Wevolv) {
	qb_workspace &ws = *need(interm->ws, "InhomStepMaxwell");
	cudaStream_t s = ws.stream;
	const unsigned n = interm->numVol;
	ws.io_in.ensure(sizeof(wignerV_t) * n);
	ws.io_out.ensure(sizeof(wignerV_t) * n);
	ws.bext.ensure(sizeof(double) * 3 * n + 2 * sizeof(wignerV_t));
	double *B = ws.bext.as<double>(), *wl = B + 3 * n, *wr = wl + 4 * NN;
	double *a = ws.io_in.as<double>(), *b = ws.io_out.as<double>();
	h2d(a, W, sizeof(wignerV_t) * n, s);
	h2d(B, Bext, sizeof(double) * 3 * n, s);
	h2d(wl, WL, sizeof(wignerV_t), s);
	h2d(wr, WR, sizeof(wignerV_t), s);
	const double *vx = ws.vgrid.as<double>() + 4 * NN;
	if (Wevolv == nullptr) {
		qb::inhom_step_maxwell(ws, q.set, (int)n, a, b, vx, h, dt, lambda, wl, wr, B, s);
		d2h(Wnext, b, sizeof(wignerV_t) * n, s);
	} else {
		for (unsigned it = 1; it < numsteps; it++) {
			qb::inhom_step_maxwell(ws, q.set, (int)n, a, b, vx, h, dt, lambda, wl, wr, B, s);
			d2h(&Wevolv[(size_t)it * n], b, sizeof(wignerV_t) * n, s);
			std::swap(a, b);
		}
	}
	sync(s);
}

void InhomStepMaxwell(const wignerV_t *restrict_ W, const quadI1_t *restrict_ quadI1, const quadI2_t *restrict_ quadI2, const quadI3_t *restrict_ quadI3, const quadI1_t *restrict_ quadI4,
                      const double h, const double dt, const double lambda, const wignerV_t *restrict_ WMaxwL, const wignerV_t *restrict_ WMaxwR, const double *restrict_ Bext, inhomStepInterm_t *restrict_ interm, wignerV_t *restrict_ Wnext) {
	Quads q(quadI1, quadI2, quadI3, quadI4, need(interm->ws, __func__)->stream);
	maxwell_call(W, q, h, dt, lambda, WMaxwL, WMaxwR, Bext, interm, Wnext, 0, nullptr);
}

void SimulationHomInterm_Create(simulationHomInterm_t *interm) { alloc_ws(&interm->ws); }
void SimulationHomInterm_Delete(simulationHomInterm_t *interm) { free_ws(&interm->ws); }

void SimulationHomogeneous(const wignerV_t *restrict_ W0, const quadI1_t *restrict_ quadI1, const quadI2_t *restrict_ quadI2, const quadI3_t *restrict_ quadI3, const quadI1_t *restrict_ quadI4,
                           const double dt, const unsigned int numsteps, const double Bext[3], simulationHomInterm_t *restrict_ interm, wignerV_t *restrict_ Wevolv) {
	qb_workspace &ws = *need(interm->ws, __func__);
	cudaStream_t s = ws.stream;
	Quads q(quadI1, quadI2, quadI3, quadI4, s);
	if (numsteps == 0) return;
	memcpy(Wevolv, W0, sizeof(wignerV_t));
	ws.va.ensure(sizeof(wignerV_t));
	ws.fa.ensure(sizeof(wignerF_t) * 2);
	ws.bext.ensure(sizeof(double) * 3);
	double *V = ws.va.as<double>();
	double2 *F = ws.fa.as<double2>();
	h2d(V, W0, sizeof(wignerV_t), s);
	h2d(ws.bext.p, Bext, 3 * sizeof(double), s);
	for (unsigned it = 1; it < numsteps; it++) {
		qb::to_fourier(NG, 4, V, F, s);
		qb::collision_step(ws, q.set, 1, F, ws.bext.as<double>(), dt, F + 4 * NN, s);
		qb::from_fourier(NG, 4, F + 4 * NN, V, s);
		d2h(&Wevolv[it], V, sizeof(wignerV_t), s);
	}
	sync(s);
}

static void sim_inhom(const wignerV_t *W0, const Quads &q, double h, double dt, unsigned numsteps, const double *Bext, inhomStepInterm_t *interm, wignerV_t *Wevolv, int bc) {
	qb_workspace &ws = *need(interm->ws, "SimulationInhomogeneous");
	cudaStream_t s = ws.stream;
	const unsigned n = interm->numVol;
	if (numsteps == 0) return;
	memcpy(Wevolv, W0, sizeof(wignerV_t) * n);
	ws.io_in.ensure(sizeof(wignerV_t) * n);
	ws.io_out.ensure(sizeof(wignerV_t) * n);
	ws.bext.ensure(sizeof(double) * 3 * n);
	double *a = ws.io_in.as<double>(), *b = ws.io_out.as<double>();
	h2d(a, W0, sizeof(wignerV_t) * n, s);
	h2d(ws.bext.p, Bext, sizeof(double) * 3 * n, s);
	for (unsigned it = 1; it < numsteps; it++) {
		qb::inhom_step(ws, q.set, (int)n, a, b, ws.vgrid.as<double>(), h, dt, ws.bext.as<double>(), bc, s);
		d2h(&Wevolv[(size_t)it * n], b, sizeof(wignerV_t) * n, s);
		std::swap(a, b);
	}
	sync(s);
}

void SimulationInhomogeneousPeriodic(const wignerV_t *restrict_ W0, const quadI1_t *restrict_ quadI1, const quadI2_t *restrict_ quadI2, const quadI3_t *restrict_ quadI3, const quadI1_t *restrict_ quadI4,
                                     const double h, const double dt, const unsigned int numsteps, const double *restrict_ Bext, inhomStepInterm_t *restrict_ interm, wignerV_t *restrict_ Wevolv) {
	Quads q(quadI1, quadI2, quadI3, quadI4, need(interm->ws, __func__)->stream);
	sim_inhom(W0, q, h, dt, numsteps, Bext, interm, Wevolv, 0);
}

void SimulationInhomogeneousDirichlet(const wignerV_t *restrict_ W0, const quadI1_t *restrict_ quadI1, const quadI2_t *restrict_ quadI2, const quadI3_t *restrict_ quadI3, const quadI1_t *restrict_ quadI4,
                                      const double h, const double dt, const unsigned int numsteps, const double *restrict_ Bext, inhomStepInterm_t *restrict_ interm, wignerV_t *restrict_ Wevolv) {
	Quads q(quadI1, quadI2, quadI3, quadI4, need(interm->ws, __func__)->stream);
	sim_inhom(W0, q, h, dt, numsteps, Bext, interm, Wevolv, 1);
}

void SimulationInhomogeneousMaxwell(const wignerV_t *restrict_ W0, const quadI1_t *restrict_ quadI1, const quadI2_t *restrict_ quadI2, const quadI3_t *restrict_ quadI3, const quadI1_t *restrict_ quadI4,
                                    const double h, const double dt, const double lambda, const wignerV_t *restrict_ WMaxwL, const wignerV_t *restrict_ WMaxwR, const unsigned int numsteps, const double *restrict_ Bext, inhomStepInterm_t *restrict_ interm, wignerV_t *restrict_ Wevolv) {
	Quads q(quadI1, quadI2, quadI3, quadI4, need(interm->ws, __func__)->stream);
	if (numsteps == 0) return;
	memcpy(Wevolv, W0, sizeof(wignerV_t) * interm->numVol);
	maxwell_call(W0, q, h, dt, lambda, WMaxwL, WMaxwR, Bext, interm, nullptr, numsteps, Wevolv);
}

// ---- finite_volume.h (upstream src/finite_volume.c) ----------------------------------
// Single lines run through the same stencil kernels as the batched transport.
static void slope_line(const double h, const double dt, const double A, const unsigned N, const double *Un, double *Un1, int bc) {
	if (N == 0) return;
	qb_workspace &ws = thread_ws();
	cudaStream_t s = ws.stream;
	ws.io_in.ensure(sizeof(double) * (2 * (size_t)N + 1));
	double *d = ws.io_in.as<double>();
	h2d(d, Un, sizeof(double) * N, s);
	h2d(d + 2 * N, &A, sizeof(double), s);
	qb::transport(1, (int)N, d, d + N, d + 2 * N, h, dt, bc, s);
	d2h(Un1, d + N, sizeof(double) * N, s);
	sync(s);
}

void SlopeLimiterStepPeriodic(const double h, const double dt, const double A, const unsigned int N, const double *restrict_ Un, double *restrict_ Un1) {
	slope_line(h, dt, A, N, Un, Un1, 0);
}
void SlopeLimiterStepDirichlet(const double h, const double dt, const double A, const unsigned int N, const double *restrict_ Un, double *restrict_ Un1) {
	slope_line(h, dt, A, N, Un, Un1, 1);
}

static void flux_call(const unsigned m, const double *A, const double *U, double out[2]) {
	qb_workspace &ws = thread_ws();
	cudaStream_t s = ws.stream;
	ws.io_in.ensure(sizeof(double) * (2 * (size_t)m + 2));
	double *d = ws.io_in.as<double>();
	h2d(d, A, sizeof(double) * m, s);
	h2d(d + m, U, sizeof(double) * m, s);
	qb::flux_pair((int)m, d, d + m, d + 2 * m, s);
	d2h(out, d + 2 * m, 2 * sizeof(double), s);
	sync(s);
}
double CalculateRightwardFlux(const unsigned int m, const double *restrict_ A, const double *restrict_ U) {
	double f[2];
	flux_call(m, A, U, f);
	return f[0];
}
double CalculateLeftwardFlux(const unsigned int m, const double *restrict_ A, const double *restrict_ U) {
	double f[2];
	flux_call(m, A, U, f);
	return f[1];
}

void SlopeLimiterStepMaxwell(const double h, const double dt, const unsigned int m, const double *restrict_ A, const unsigned int N,
                             const double lambda, const double fluxL, const double fluxR, const double *restrict_ UmaxwL, const double *restrict_ UmaxwR, const double *restrict_ Un, double *restrict_ Un1) {
	if (N == 0 || m == 0) return;
	qb_workspace &ws = thread_ws();
	cudaStream_t s = ws.stream;
	const size_t mn = (size_t)m * N;
	ws.io_in.ensure(sizeof(double) * (2 * mn + 3 * (size_t)m + 2));
	double *in = ws.io_in.as<double>(), *out = in + mn, *a = out + mn, *ul = a + m, *ur = ul + m, *fl = ur + m;
	const double flux[2] = { fluxL, fluxR };
	h2d(in, Un, sizeof(double) * mn, s);
	h2d(a, A, sizeof(double) * m, s);
	h2d(ul, UmaxwL, sizeof(double) * m, s);
	h2d(ur, UmaxwR, sizeof(double) * m, s);
	h2d(fl, flux, sizeof(flux), s);
	qb::transport_maxwell_lines((int)m, (int)N, in, out, a, h, dt, lambda, fl, ul, ur, s);
	d2h(Un1, out, sizeof(double) * mn, s);
	sync(s);
}

// ---- util.h (upstream src/util.c): raw binary I/O ---------------------------------------
int ReadData(const char *filename, void *data, const size_t size, const size_t n) {
	FILE *fd = fopen(filename, "rb");
	if (fd == NULL) { fprintf(stderr, "ReadData: cannot open '%s' for reading\n", filename); return -1; }
	fseek(fd, 0, SEEK_END);
	const long filesize = ftell(fd);
	rewind(fd);
	if ((size_t)filesize != n * size) {
		fprintf(stderr, "ReadData: '%s' holds %ld bytes, the caller expects %zu\n", filename, filesize, n * size);
		fclose(fd);
		return -2;
	}
	if (fread(data, size, n, fd) != n) { fprintf(stderr, "ReadData: short read from '%s'\n", filename); fclose(fd); return -3; }
	fclose(fd);
	return 0;
}

int WriteData(const char *filename, const void *data, const size_t size, const size_t n, const bool append) {
	FILE *fd = fopen(filename, append ? "ab" : "wb");
	if (fd == NULL) { fprintf(stderr, "WriteData: cannot open '%s' for writing\n", filename); return -1; }
	if (fwrite(data, size, n, fd) != n) { fprintf(stderr, "WriteData: short write to '%s'\n", filename); fclose(fd); return -3; }
	fclose(fd);
	return 0;
}

}  // extern "C"

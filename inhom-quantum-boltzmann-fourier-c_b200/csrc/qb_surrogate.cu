// qb_surrogate.cu — Strang step whose collision half takes the learned
// operator C~[W] (qb_fno) where it is accurate enough, with the exact
// collision operator as judge and per-cell fallback.
//
// The step is the one of qb_inhom_step (upstream SimulationInhomogeneous,
// src/simulation.c:294-330 with InternalFourierCollisionStep,
// src/simulation.c:214-284): half a transport step, the collision step, half
// a transport step.  For a surrogate cell the collision step is the midpoint
// rule of upstream CollisionStep (src/simulation.c:105-136) with C~ in place
// of Cc + Cd:
//     Wm = W + dt/2 (C~[W] + CB[W]),   W' = W + dt (C~[Wm] + CB[Wm])
// evaluated in velocity space (CB, the magnetic precession -i[B, W], is
// pointwise and linear, so it reads the same there).  Before use, C~ is
// projected so that the trace component conserves mass, momentum and energy:
// c0 -= |w0| (l0 + l1 i + l2 j + l3 (i^2 + j^2)) with the l solving the 4 x 4
// normal equations, (i, j) the velocity in units of the grid spacing (the
// same span as the physical velocities).  Every `check_every`-th step runs
// both the network's step and the exact one on every cell, keeps the exact one, and
// marks the cells whose collision increment from the network differs from the
// exact increment by more than `tol` (relative L1); marked cells take the
// exact step until the next check.  Judging the step rather than C itself
// costs no evaluation of the exact operator beyond the exact step.  The exact
// operator is reached only through the library's public entry point
// qb_fourier_collision, so the judge is the same code the parity tests pin.
#include "qb_engine.h"

extern "C" {
#include "qbgpu.h"
}

#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

namespace {

constexpr int kThreads = 256;

// block-wide sum of `nv` doubles per thread, fixed order; result in red[0..nv)
template <int NV>
__device__ void block_sums(double (&v)[NV], double *red) {
	__shared__ double sh[NV][kThreads / 32];
	const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
	for (int k = 0; k < NV; k++) {
		double x = v[k];
		for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
		if (lane == 0) sh[k][wid] = x;
	}
	__syncthreads();
	if (threadIdx.x < NV) {
		double x = 0;
		for (int w = 0; w < kThreads / 32; w++) x += sh[threadIdx.x][w];
		red[threadIdx.x] = x;
	}
	__syncthreads();
}

// velocity of grid index k in units of the grid spacing: the velocity grid
// is in FFT order, 0, 1, ..., N/2 - 1, -N/2, ..., -1 (upstream
// src/simulation.c:150-154)
__device__ __forceinline__ double vidx(int N, int k) { return k < N / 2 ? (double)k : (double)(k - N); }

// conservation projection of the trace component of C (one CTA per cell)
__global__ void __launch_bounds__(kThreads) k_project(int N, double *__restrict__ C, const double *__restrict__ V) {
	__shared__ double red[14];
	__shared__ double lam[4];
	const int NN = N * N;
	double *c0 = C + (long)blockIdx.x * 4 * NN;
	const double *w0 = V + (long)blockIdx.x * 4 * NN;
	double acc[14];
	for (int k = 0; k < 14; k++) acc[k] = 0;
	for (int p = threadIdx.x; p < NN; p += kThreads) {
		const double i = vidx(N, p / N), j = vidx(N, p % N);
		const double phi[4] = { 1.0, i, j, i * i + j * j };
		const double a = fabs(w0[p]), c = c0[p];
		int t = 0;
		for (int r = 0; r < 4; r++)
			for (int q = r; q < 4; q++) acc[t++] += a * phi[r] * phi[q];
		for (int r = 0; r < 4; r++) acc[10 + r] += c * phi[r];
	}
	block_sums<14>(acc, red);
	if (threadIdx.x == 0) {
		// G lam = rhs, G symmetric from the 10 sums; Gaussian elimination with partial pivoting
		double G[4][5];
		int t = 0;
		for (int r = 0; r < 4; r++)
			for (int q = r; q < 4; q++) { G[r][q] = red[t]; G[q][r] = red[t]; t++; }
		for (int r = 0; r < 4; r++) G[r][4] = red[10 + r];
		bool ok = true;
		for (int col = 0; col < 4; col++) {
			int piv = col;
			for (int r = col + 1; r < 4; r++) if (fabs(G[r][col]) > fabs(G[piv][col])) piv = r;
			if (!(fabs(G[piv][col]) > 1e-300)) { ok = false; break; }
			if (piv != col) for (int q = 0; q < 5; q++) { const double x = G[col][q]; G[col][q] = G[piv][q]; G[piv][q] = x; }
			for (int r = col + 1; r < 4; r++) {
				const double f = G[r][col] / G[col][col];
				for (int q = col; q < 5; q++) G[r][q] -= f * G[col][q];
			}
		}
		for (int r = 3; r >= 0; r--) {
			double x = ok ? G[r][4] : 0.0;
			if (ok) {
				for (int q = r + 1; q < 4; q++) x -= G[r][q] * lam[q];
				x /= G[r][r];
			}
			lam[r] = x;
		}
	}
	__syncthreads();
	for (int p = threadIdx.x; p < NN; p += kThreads) {
		const double i = vidx(N, p / N), j = vidx(N, p % N);
		c0[p] -= fabs(w0[p]) * (lam[0] + lam[1] * i + lam[2] * j + lam[3] * (i * i + j * j));
	}
}

// out = V + a (C + CB[U]) over ncells velocity-space cells; B: 3 per cell or null
__global__ void k_stage(int NN, int ncells, const double *__restrict__ V, const double *__restrict__ U, const double *__restrict__ C,
                        const double *__restrict__ B, double a, double *__restrict__ out) {
	const long n = (long)ncells * NN;
	for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
		const long cell = t / NN, p = t % NN;
		const long base = cell * 4 * NN + p;
		double cb[4] = { 0, 0, 0, 0 };
		if (B != nullptr) {
			const double *b = B + cell * 3;
			const double u1 = U[base + NN], u2 = U[base + 2 * NN], u3 = U[base + 3 * NN];
			cb[1] = 2 * (b[1] * u3 - b[2] * u2);
			cb[2] = 2 * (b[2] * u1 - b[0] * u3);
			cb[3] = 2 * (b[0] * u2 - b[1] * u1);
		}
		for (int c = 0; c < 4; c++) out[base + c * NN] = V[base + c * NN] + a * (C[base + c * NN] + cb[c]);
	}
}

// out[cell] = sum |A - B| / sum |B - V| over the cell's `per` values: the
// relative L1 difference of two steps A, B from the same state V, measured on
// the increment B - V
__global__ void __launch_bounds__(kThreads) k_step_residual(long per, const double *__restrict__ A, const double *__restrict__ B,
                                                            const double *__restrict__ V, double *__restrict__ out) {
	__shared__ double red[2];
	const double *a = A + blockIdx.x * per, *b = B + blockIdx.x * per, *v = V + blockIdx.x * per;
	double acc[2] = { 0, 0 };
	for (long p = threadIdx.x; p < per; p += kThreads) {
		acc[0] += fabs(a[p] - b[p]);
		acc[1] += fabs(b[p] - v[p]);
	}
	block_sums<2>(acc, red);
	if (threadIdx.x == 0) out[blockIdx.x] = red[1] > 0 ? red[0] / red[1] : (red[0] > 0 ? INFINITY : 0.0);
}

// dst[k] = src[idx[k]] (to_gathered) or dst[idx[k]] = src[k], cells of `per` doubles
__global__ void k_move_cells(long per, int count, const int *__restrict__ idx, const double *__restrict__ src, double *__restrict__ dst, int to_gathered) {
	const long n = per * count;
	for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
		const long k = t / per, p = t % per;
		if (to_gathered) dst[t] = src[(long)idx[k] * per + p];
		else dst[(long)idx[k] * per + p] = src[t];
	}
}

unsigned grid_for(long n) { return (unsigned)std::max<long>(1, std::min<long>((n + 255) / 256, 148L * 16)); }

template <class... P, class... A>
void launch(const char *name, void (*k)(P...), unsigned grid, unsigned block, cudaStream_t s, A... args) {
	qb::ProfScope ps(name, s);
	k<<<grid, block, 0, s>>>(args...);
	QB_CUDA(cudaGetLastError());
}

void api(int rc, const char *what) {
	if (rc != 0) QB_FAIL(std::string("surrogate step: ") + what + " failed: " + qb_last_error());
}

}  // namespace

struct qb_surrogate {
	qb_fno *net = nullptr;
	double tol = 0;
	unsigned check_every = 1;
	unsigned long step = 0;
	long n_sur = 0, n_ex = 0;
	double last_res = 0;
	std::vector<unsigned char> exact;            // per cell: take the exact step until the next check
	std::vector<int> idx;
	std::vector<double> resid_h;
	qb::DevBuf vt, vm, vc, c1, vs, resid, gath, bg, didx;
};

extern "C" {

qb_surrogate *qb_surrogate_create(qb_fno *net, double tol, unsigned check_every) {
	try {
		if (net == nullptr) QB_FAIL("qb_surrogate_create: null network");
		if (!(tol >= 0)) QB_FAIL("qb_surrogate_create: tol must be >= 0");
		if (check_every == 0) QB_FAIL("qb_surrogate_create: check_every must be positive");
		auto s = std::make_unique<qb_surrogate>();
		s->net = net;
		s->tol = tol;
		s->check_every = check_every;
		return s.release();
	} catch (const std::exception &) {
		return nullptr;
	}
}

void qb_surrogate_free(qb_surrogate *s) { delete s; }

int qb_surrogate_stats(const qb_surrogate *s, long *surrogate_cells, long *exact_cells, double *last_max_residual) {
	if (s == nullptr) {
		try { QB_FAIL("qb_surrogate_stats: null handle"); } catch (const std::exception &) {}
		return -1;
	}
	if (surrogate_cells) *surrogate_cells = s->n_sur;
	if (exact_cells) *exact_cells = s->n_ex;
	if (last_max_residual) *last_max_residual = s->last_res;
	return 0;
}

int qb_surrogate_inhom_step(qb_surrogate *sg, qb_workspace *ws, const qb_quad *q, int ncells, const double *W, double *Wnext,
                            double h, double dt, const double *Bext, void *stream) {
	try {
		if (sg == nullptr || ws == nullptr || q == nullptr) QB_FAIL("qb_surrogate_inhom_step: null handle");
		if (W == nullptr || Wnext == nullptr) QB_FAIL("qb_surrogate_inhom_step: null state");
		if (qb_fno_grid_size(sg->net) != ws->N) QB_FAIL("qb_surrogate_inhom_step: the network and the workspace are for different grid sizes");
		const int N = ws->N;
		if (q->q->N != N) QB_FAIL("qb_surrogate_inhom_step: workspace and quadrature tables are for different grid sizes");
		if (N > 64 || ncells <= 0) QB_FAIL("qb_surrogate_inhom_step: bad grid size or cell count");
		if (W == Wnext) QB_FAIL("qb_surrogate_inhom_step: Wnext must not alias W");
		const double L = q->q->L;
		const int NN = N * N;
		const long cs = 4L * NN;
		cudaStream_t s = (cudaStream_t)stream;
		sg->vt.ensure(sizeof(double) * cs * ncells);
		sg->vc.ensure(sizeof(double) * cs * ncells);
		sg->c1.ensure(sizeof(double) * cs * ncells);
		double *Vt = sg->vt.as<double>(), *Vc = sg->vc.as<double>(), *C1 = sg->c1.as<double>();

		api(qb_transport(N, L, ncells, W, Vt, h, 0.5 * dt, 0, s), "transport");
		const bool check = (sg->step % sg->check_every == 0) || sg->exact.size() != (size_t)ncells;
		// the network's midpoint step of every cell from Vt into out
		auto network_step = [&](double *out) {
			sg->vm.ensure(sizeof(double) * cs * ncells);
			double *Vm = sg->vm.as<double>();
			const long nv = (long)ncells * NN;
			api(qb_fno_forward(sg->net, ncells, Vt, C1, s), "network");
			launch("surrogate_project", k_project, ncells, kThreads, s, N, C1, (const double *)Vt);
			launch("surrogate_stage", k_stage, grid_for(nv), 256, s, NN, ncells, (const double *)Vt, (const double *)Vt, (const double *)C1, Bext, 0.5 * dt, Vm);
			api(qb_fno_forward(sg->net, ncells, Vm, C1, s), "network");
			launch("surrogate_project", k_project, ncells, kThreads, s, N, C1, (const double *)Vm);
			launch("surrogate_stage", k_stage, grid_for(nv), 256, s, NN, ncells, (const double *)Vt, (const double *)Vm, (const double *)C1, Bext, dt, out);
		};
		if (check) {
			// both steps on every cell; the exact one is kept, the network's is
			// judged by the relative L1 difference of its collision increment
			sg->vs.ensure(sizeof(double) * cs * ncells);
			sg->resid.ensure(sizeof(double) * ncells);
			network_step(sg->vs.as<double>());
			QB_CUDA(cudaMemcpyAsync(Vc, Vt, sizeof(double) * cs * ncells, cudaMemcpyDeviceToDevice, s));
			api(qb_fourier_collision(ws, q, ncells, Vc, Bext, dt, s), "exact collision");
			launch("surrogate_residual", k_step_residual, ncells, kThreads, s, cs, (const double *)sg->vs.as<double>(), (const double *)Vc,
			       (const double *)Vt, sg->resid.as<double>());
			sg->resid_h.resize(ncells);
			QB_CUDA(cudaMemcpyAsync(sg->resid_h.data(), sg->resid.p, sizeof(double) * ncells, cudaMemcpyDeviceToHost, s));
			QB_CUDA(cudaStreamSynchronize(s));
			sg->exact.assign(ncells, 0);
			double mx = 0;
			for (int c = 0; c < ncells; c++) {
				const double r = sg->resid_h[c];
				mx = std::max(mx, std::isnan(r) ? INFINITY : r);
				sg->exact[c] = !(r <= sg->tol);
			}
			sg->last_res = mx;
			sg->n_ex += ncells;
		} else {
			network_step(Vc);
			sg->idx.clear();
			for (int c = 0; c < ncells; c++) if (sg->exact[c]) sg->idx.push_back(c);
			const int nf = (int)sg->idx.size();
			if (nf > 0) {
				sg->gath.ensure(sizeof(double) * cs * nf);
				sg->didx.ensure(sizeof(int) * nf);
				QB_CUDA(cudaMemcpyAsync(sg->didx.p, sg->idx.data(), sizeof(int) * nf, cudaMemcpyHostToDevice, s));
				launch("surrogate_gather", k_move_cells, grid_for(cs * nf), 256, s, cs, nf, (const int *)sg->didx.as<int>(), (const double *)Vt,
				       sg->gath.as<double>(), 1);
				const double *Bg = nullptr;
				if (Bext != nullptr) {
					sg->bg.ensure(sizeof(double) * 3 * nf);
					launch("surrogate_gather", k_move_cells, grid_for(3L * nf), 256, s, 3L, nf, (const int *)sg->didx.as<int>(), Bext, sg->bg.as<double>(), 1);
					Bg = sg->bg.as<double>();
				}
				api(qb_fourier_collision(ws, q, nf, sg->gath.as<double>(), Bg, dt, s), "exact collision");
				launch("surrogate_scatter", k_move_cells, grid_for(cs * nf), 256, s, cs, nf, (const int *)sg->didx.as<int>(),
				       (const double *)sg->gath.as<double>(), Vc, 0);
				// the index list is read by the copy above until the copy has
				// been staged (pageable memory), which the call itself waits for
			}
			sg->n_sur += ncells - nf;
			sg->n_ex += nf;
		}
		api(qb_transport(N, L, ncells, Vc, Wnext, h, 0.5 * dt, 0, s), "transport");
		sg->step++;
		return 0;
	} catch (const std::exception &) {
		return -1;
	}
}

}  // extern "C"

// qb_tables.cu — quadrature tables of the collision integrals, built on the GPU.
//
// Each table follows the formula of the upstream builder cited beside it
// (src/quadrature.c); the upstream host layout is produced for the caller's
// quad structs, and compact device forms are kept for the kernels:
//   I1: psi1_i (J distinct 2N grids), psi2_j (J distinct N grids) and the
//       J x J principal-value weights w_ij fold into Phi_j = sum_i w_ij psi1_i,
//       so the J*J-term upstream sum becomes J terms (phi = Phi_j, psi2 = psi2_j).
//   I3: psi2_{j,m} = c_m * S_j with S_j a sinc table per angle (stored
//       transposed for the column pass) and c_m = 2 R w_m pi / J.
#include "qb_engine.h"
#include <cmath>
#include <vector>

namespace qb {

namespace {

__device__ __forceinline__ int kg(int N, int k) { return k < N / 2 ? k : k - N; }       // quadrature.c:163-166
__device__ __forceinline__ int kg2(int N, int k) { return k < N ? k : k - 2 * N; }      // quadrature.c:167-170
__device__ __forceinline__ double d_sin_sinc(double x) {                                // quadrature.c:116-126
	if (fabs(x) < 1e-8) return x;
	const double s = sin(x);
	return (s * s) / x;
}
__device__ __forceinline__ double d_sinc(double x) { return fabs(x) < 1e-8 ? 1.0 : sin(x) / x; }   // :132-142

// I1 (FourierI1, quadrature.c:150-238)
__global__ void k_i1_psi1(int N, int J, double L, double R, double *out) {   // [J][P*P]
	const int P = 2 * N, i = blockIdx.y;
	const double th = i * (M_PI / J), c = cos(th), sn = sin(th), s = R * M_PI / (2 * L);
	for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < P * P; q += gridDim.x * blockDim.x) {
		const int l = q / P, k = q % P;
		out[(long)i * P * P + q] = R * d_sin_sinc(s * (kg2(N, l) * c + kg2(N, k) * sn));
	}
}
__global__ void k_i1_psi2(int N, int J, double L, double R, double *out) {   // [J][N*N], theta2 grid
	const int j = blockIdx.y;
	const double dth = M_PI / J, th = j * dth + 0.5 * dth, c = cos(th), sn = sin(th), s = R * M_PI / (2 * L);
	for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < N * N; q += gridDim.x * blockDim.x) {
		const int l = q / N, k = q % N;
		out[(long)j * N * N + q] = R * d_sin_sinc(s * (kg(N, l) * c + kg(N, k) * sn));
	}
}
__device__ __forceinline__ double i1_weight(int J, int i, int j) {
	const double dth = M_PI / J, th1 = i * dth, th2 = j * dth + 0.5 * dth, a = 2 * M_PI / J;
	return -(a * a) / cos(th1 - th2);
}
__global__ void k_i1_phi(int N, int J, const double *psi1, double *phi) {   // Phi_j = sum_i w_ij psi1_i
	const int P = 2 * N, j = blockIdx.y;
	for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < P * P; q += gridDim.x * blockDim.x) {
		double s = 0;
		for (int i = 0; i < J; i++) s += i1_weight(J, i, j) * psi1[(long)i * P * P + q];
		phi[(long)j * P * P + q] = s;
	}
}
// upstream layout: psiR1[i+J*j] = psi1_i, psiR2[i+J*j] = psi2_j * w_ij
__global__ void k_i1_full(int N, int J, const double *psi1, const double *psi2, double *r1, double *r2) {
	const int P = 2 * N, t = blockIdx.y, i = t % J, j = t / J;
	const double w = i1_weight(J, i, j);
	for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < P * P; q += gridDim.x * blockDim.x) {
		r1[(long)t * P * P + q] = psi1[(long)i * P * P + q];
		if (q < N * N) r2[(long)t * N * N + q] = psi2[(long)j * N * N + q] * w;
	}
}

// I2 (FourierI2, quadrature.c:245-286)
__global__ void k_i2(int N, int J, double L, double R, double *r1, double *r2) {
	const int j = blockIdx.y;
	const double th = j * (M_PI / J), c = cos(th), sn = sin(th);
	const double f1 = 2 * R, f2 = 2 * R * M_PI / J, s = R * M_PI / L;
	for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < N * N; q += gridDim.x * blockDim.x) {
		const int l = q / N, k = q % N;
		r1[(long)j * N * N + q] = f1 * d_sinc(s * (kg(N, l) * c + kg(N, k) * sn));
		r2[(long)j * N * N + q] = f2 * d_sinc(s * (-kg(N, l) * sn + kg(N, k) * c));
	}
}

// Legendre-Gauss nodes/weights (LegendreGaussQuad, quadrature.c:293-388): one
// thread runs the upstream Newton iteration (bounded); scratch holds M*(M+1)+4M doubles
__global__ void k_lgwt(int M, double a, double b, double *x, double *w, double *scr) {
	if (threadIdx.x != 0 || blockIdx.x != 0) return;
	double *Lv = scr, *Lp = scr + (long)M * (M + 1), *y = Lp + M, *y0 = y + M;
	const double invN = 1.0 / (M - 1);
	for (int i = 0; i < M; i++) {
		const double xu = -1.0 + 2 * i * invN;
		y[i] = cos((2 * i + 1) * M_PI / (2 * M)) + 0.27 / M * sin(M_PI * xu * (M - 1) / (M + 1));
		y0[i] = 2;
		Lp[i] = 0;
	}
	double diff = 0;
	for (int i = 0; i < M; i++) diff = fmax(diff, fabs(y[i] - y0[i]));
	for (int it = 0; diff > 2.220446049250313e-16 && it < 1000; it++) {
		for (int i = 0; i < M; i++) { Lv[i] = 1; Lv[i + M] = y[i]; }
		for (int k = 1; k < M; k++)
			for (int i = 0; i < M; i++)
				Lv[i + (k + 1) * M] = ((2 * k + 1) * y[i] * Lv[i + k * M] - k * Lv[i + (k - 1) * M]) / (k + 1);
		for (int i = 0; i < M; i++) Lp[i] = (M + 1) * (Lv[i + (M - 1) * M] - y[i] * Lv[i + M * M]) / (1 - y[i] * y[i]);
		diff = 0;
		for (int i = 0; i < M; i++) {
			const double t = Lv[i + M * M] / Lp[i];
			y0[i] = y[i];
			y[i] -= t;
			diff = fmax(diff, fabs(t));
		}
	}
	for (int i = 0; i < M; i++) {
		x[i] = (a * (1 - y[i]) + b * (1 + y[i])) / 2;
		const double r = (double)(M + 1) / M;
		w[i] = (b - a) / ((1 - y[i] * y[i]) * (Lp[i] * Lp[i])) * (r * r);
	}
}

// I3 (FourierI3, quadrature.c:395-466): term t = m + j*M
__global__ void k_i3_psi1(int N, int J, int M, double L, const double *rho, double2 *psi1) {
	const int t = blockIdx.y, j = t / M, m = t % M;
	const double th = j * (M_PI / J), c = cos(th), sn = sin(th), s1 = rho[m] * M_PI / L;
	for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < N * N; q += gridDim.x * blockDim.x) {
		const int l = q / N, k = q % N;
		double sv, cv;
		sincos(s1 * (kg(N, l) * c + kg(N, k) * sn), &sv, &cv);
		psi1[(long)t * N * N + q] = make_double2(cv, sv);
	}
}
// S_j stored transposed: ST[j][k][l] = sinc(s2*(-kgrid2[l] sin + kgrid2[k] cos))
__global__ void k_i3_sinc(int N, int J, double L, double R, double *ST) {
	const int P = 2 * N, j = blockIdx.y;
	const double th = j * (M_PI / J), c = cos(th), sn = sin(th), s2 = M_PI * R / L;
	for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < P * P; q += gridDim.x * blockDim.x) {
		const int k = q / P, l = q % P;
		ST[(long)j * P * P + q] = d_sinc(s2 * (-kg2(N, l) * sn + kg2(N, k) * c));
	}
}
__global__ void k_i3_terms(int J, int M, double R, const double *wq, int *idx, double *scale) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= J * M) return;
	const int m = t % M;
	idx[t] = t / M;
	scale[t] = 2 * R * wq[m] * M_PI / J;
}
// upstream layout psiR2[t][l][k] = scale[t] * S_j[l][k]
__global__ void k_i3_full(int N, int nterms, const double *ST, const int *idx, const double *scale, double *r2) {
	const int P = 2 * N, t = blockIdx.y;
	for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < P * P; q += gridDim.x * blockDim.x) {
		const int l = q / P, k = q % P;
		r2[(long)t * P * P + q] = scale[t] * ST[(long)idx[t] * P * P + k * P + l];
	}
}
__global__ void k_transpose(int P, int ntab, const double *in, double *out) {   // out[t][k][l] = in[t][l][k]
	const int t = blockIdx.y;
	for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < P * P; q += gridDim.x * blockDim.x) {
		const int k = q / P, l = q % P;
		out[(long)t * P * P + q] = in[(long)t * P * P + l * P + k];
	}
}
__global__ void k_iota_ones(int n, int *idx, double *scale) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t < n) { idx[t] = t; scale[t] = 1.0; }
}

// I4 (FourierI4, quadrature.c:473-527)
__global__ void k_i4(int N, int J, double L, double R, double *r1, double *r2) {
	const int P = 2 * N, j = blockIdx.y;
	const double th = j * (M_PI / J), c = cos(th), sn = sin(th);
	const double f1 = 2 * R, f2 = 2 * R * M_PI / J, s = M_PI * R / L;
	for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < P * P; q += gridDim.x * blockDim.x) {
		const int l = q / P, k = q % P;
		r1[(long)j * P * P + q] = f1 * d_sinc(s * (kg2(N, l) * c + kg2(N, k) * sn));
		if (q < N * N) {
			const int l2 = q / N, k2 = q % N;
			r2[(long)j * N * N + q] = f2 * d_sinc(s * (-kg(N, l2) * sn + kg(N, k2) * c));
		}
	}
}

dim3 tab_grid(long per, int ny) { return dim3((unsigned)((per + 255) / 256 < 64 ? (per + 255) / 256 : 64), (unsigned)ny); }

void d2h(double *host, const void *dev, size_t bytes, cudaStream_t s) {
	if (host == nullptr) return;
	QB_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, s));
}

}  // namespace

void build_i1(int N, int J, double L, double R, DevI1 &dev, double *host_psiR1, double *host_psiR2, cudaStream_t s) {
	if (J < 1) QB_FAIL("FourierI1: J must be positive");
	const long P = 2 * N;
	DevBuf psi1;
	psi1.ensure(sizeof(double) * J * P * P);
	dev.N = N; dev.nterms = J;
	dev.psi2.ensure(sizeof(double) * J * N * N);
	dev.phi.ensure(sizeof(double) * J * P * P);
	k_i1_psi1<<<tab_grid(P * P, J), 256, 0, s>>>(N, J, L, R, psi1.as<double>());
	k_i1_psi2<<<tab_grid(N * N, J), 256, 0, s>>>(N, J, L, R, dev.psi2.as<double>());
	k_i1_phi<<<tab_grid(P * P, J), 256, 0, s>>>(N, J, psi1.as<double>(), dev.phi.as<double>());
	QB_CUDA(cudaGetLastError());
	if (host_psiR1 || host_psiR2) {
		DevBuf r1, r2;
		r1.ensure(sizeof(double) * (long)J * J * P * P);
		r2.ensure(sizeof(double) * (long)J * J * N * N);
		k_i1_full<<<tab_grid(P * P, J * J), 256, 0, s>>>(N, J, psi1.as<double>(), dev.psi2.as<double>(), r1.as<double>(), r2.as<double>());
		QB_CUDA(cudaGetLastError());
		d2h(host_psiR1, r1.p, r1.bytes, s);
		d2h(host_psiR2, r2.p, r2.bytes, s);
		QB_CUDA(cudaStreamSynchronize(s));
	}
	QB_CUDA(cudaStreamSynchronize(s));
}

void build_i2(int N, int J, double L, double R, DevI2 &dev, double *host_psiR1, double *host_psiR2, cudaStream_t s) {
	if (J < 1) QB_FAIL("FourierI2: J must be positive");
	dev.N = N; dev.nterms = J;
	dev.psi1.ensure(sizeof(double) * J * N * N);
	dev.psi2.ensure(sizeof(double) * J * N * N);
	k_i2<<<tab_grid((long)N * N, J), 256, 0, s>>>(N, J, L, R, dev.psi1.as<double>(), dev.psi2.as<double>());
	QB_CUDA(cudaGetLastError());
	d2h(host_psiR1, dev.psi1.p, dev.psi1.bytes, s);
	d2h(host_psiR2, dev.psi2.p, dev.psi2.bytes, s);
	QB_CUDA(cudaStreamSynchronize(s));
}

void lgwt_device(int M, double a, double b, double *x_host, double *w_host, cudaStream_t s) {
	if (M < 2) QB_FAIL("LegendreGaussQuad: M must be at least 2");
	DevBuf xw, scr;
	xw.ensure(sizeof(double) * 2 * M);
	scr.ensure(sizeof(double) * ((long)M * (M + 1) + 4 * M));
	k_lgwt<<<1, 32, 0, s>>>(M, a, b, xw.as<double>(), xw.as<double>() + M, scr.as<double>());
	QB_CUDA(cudaGetLastError());
	QB_CUDA(cudaMemcpyAsync(x_host, xw.as<double>(), sizeof(double) * M, cudaMemcpyDeviceToHost, s));
	QB_CUDA(cudaMemcpyAsync(w_host, xw.as<double>() + M, sizeof(double) * M, cudaMemcpyDeviceToHost, s));
	QB_CUDA(cudaStreamSynchronize(s));
}

void build_i3(int N, int J, double L, double R, int M, DevI3 &dev, double *host_psiR1, double *host_psiR2, cudaStream_t s) {
	if (J < 1 || M < 2) QB_FAIL("FourierI3: J must be positive and M at least 2");
	const long P = 2 * N;
	const int nt = J * M;
	DevBuf xw, scr;
	xw.ensure(sizeof(double) * 2 * M);
	scr.ensure(sizeof(double) * ((long)M * (M + 1) + 4 * M));
	k_lgwt<<<1, 32, 0, s>>>(M, -R, R, xw.as<double>(), xw.as<double>() + M, scr.as<double>());
	dev.N = N; dev.nterms = nt;
	dev.psi1.ensure(sizeof(double2) * nt * N * N);
	dev.psi2T.ensure(sizeof(double) * J * P * P);
	dev.idx.ensure(sizeof(int) * nt);
	dev.scale.ensure(sizeof(double) * nt);
	k_i3_psi1<<<tab_grid((long)N * N, nt), 256, 0, s>>>(N, J, M, L, xw.as<double>(), dev.psi1.as<double2>());
	k_i3_sinc<<<tab_grid(P * P, J), 256, 0, s>>>(N, J, L, R, dev.psi2T.as<double>());
	k_i3_terms<<<(nt + 255) / 256, 256, 0, s>>>(J, M, R, xw.as<double>() + M, dev.idx.as<int>(), dev.scale.as<double>());
	QB_CUDA(cudaGetLastError());
	d2h(host_psiR1, dev.psi1.p, dev.psi1.bytes, s);
	if (host_psiR2) {
		DevBuf r2;
		r2.ensure(sizeof(double) * nt * P * P);
		k_i3_full<<<tab_grid(P * P, nt), 256, 0, s>>>(N, nt, dev.psi2T.as<double>(), dev.idx.as<int>(), dev.scale.as<double>(), r2.as<double>());
		QB_CUDA(cudaGetLastError());
		d2h(host_psiR2, r2.p, r2.bytes, s);
		QB_CUDA(cudaStreamSynchronize(s));
	}
	QB_CUDA(cudaStreamSynchronize(s));
}

void build_i4(int N, int J, double L, double R, DevI1 &dev, double *host_psiR1, double *host_psiR2, cudaStream_t s) {
	if (J < 1) QB_FAIL("FourierI4: J must be positive");
	const long P = 2 * N;
	dev.N = N; dev.nterms = J;
	dev.phi.ensure(sizeof(double) * J * P * P);
	dev.psi2.ensure(sizeof(double) * J * N * N);
	k_i4<<<tab_grid(P * P, J), 256, 0, s>>>(N, J, L, R, dev.phi.as<double>(), dev.psi2.as<double>());
	QB_CUDA(cudaGetLastError());
	d2h(host_psiR1, dev.phi.p, dev.phi.bytes, s);
	d2h(host_psiR2, dev.psi2.p, dev.psi2.bytes, s);
	QB_CUDA(cudaStreamSynchronize(s));
}

void upload_i1(int N, int num, const double *psiR1, const double *psiR2, DevI1 &dev, cudaStream_t s) {
	const long P = 2 * N;
	dev.N = N; dev.nterms = num;
	dev.phi.ensure(sizeof(double) * num * P * P);
	dev.psi2.ensure(sizeof(double) * num * N * N);
	QB_CUDA(cudaMemcpyAsync(dev.phi.p, psiR1, sizeof(double) * num * P * P, cudaMemcpyHostToDevice, s));
	QB_CUDA(cudaMemcpyAsync(dev.psi2.p, psiR2, sizeof(double) * num * N * N, cudaMemcpyHostToDevice, s));
}

void upload_i2(int N, int num, const double *psiR1, const double *psiR2, DevI2 &dev, cudaStream_t s) {
	dev.N = N; dev.nterms = num;
	dev.psi1.ensure(sizeof(double) * num * N * N);
	dev.psi2.ensure(sizeof(double) * num * N * N);
	QB_CUDA(cudaMemcpyAsync(dev.psi1.p, psiR1, sizeof(double) * num * N * N, cudaMemcpyHostToDevice, s));
	QB_CUDA(cudaMemcpyAsync(dev.psi2.p, psiR2, sizeof(double) * num * N * N, cudaMemcpyHostToDevice, s));
}

void upload_i3(int N, int num, const double *psiR1, const double *psiR2, DevI3 &dev, cudaStream_t s) {
	const long P = 2 * N;
	dev.N = N; dev.nterms = num;
	dev.psi1.ensure(sizeof(double2) * num * N * N);
	dev.psi2T.ensure(sizeof(double) * num * P * P);
	dev.idx.ensure(sizeof(int) * num);
	dev.scale.ensure(sizeof(double) * num);
	DevBuf raw;
	raw.ensure(sizeof(double) * num * P * P);
	QB_CUDA(cudaMemcpyAsync(dev.psi1.p, psiR1, sizeof(double2) * num * N * N, cudaMemcpyHostToDevice, s));
	QB_CUDA(cudaMemcpyAsync(raw.p, psiR2, sizeof(double) * num * P * P, cudaMemcpyHostToDevice, s));
	k_transpose<<<tab_grid(P * P, num), 256, 0, s>>>((int)P, num, raw.as<double>(), dev.psi2T.as<double>());
	k_iota_ones<<<(num + 255) / 256, 256, 0, s>>>(num, dev.idx.as<int>(), dev.scale.as<double>());
	QB_CUDA(cudaGetLastError());
	QB_CUDA(cudaStreamSynchronize(s));
}

std::unique_ptr<Quad> make_quad(int N, int J, int M, double L, double R, cudaStream_t s) {
	if (!supported_n(N)) QB_FAIL("grid size N=" + std::to_string(N) + " has no compiled kernels");
	auto q = std::make_unique<Quad>();
	q->N = N; q->J = J; q->M = M; q->L = L; q->R = R;
	build_i1(N, J, L, R, q->i1, nullptr, nullptr, s);
	build_i2(N, J, L, R, q->i2, nullptr, nullptr, s);
	build_i3(N, J, L, R, M, q->i3, nullptr, nullptr, s);
	build_i4(N, J, L, R, q->i4, nullptr, nullptr, s);
	return q;
}

}  // namespace qb

// qb_batch.cu — spatially homogeneous collision steps for a batch of
// independent instances of different grid sizes (the time loop of upstream
// SimulationHomogeneous, src/simulation.c:1219-1281, run on many instances
// at once).
//
// Instances of equal grid size are gathered into one contiguous batch and
// advanced together: one batched launch sequence per grid size and step, so
// a batch of thousands of small instances costs a few launches per size
// instead of a few per instance.  The quadrature tables and workspaces are
// built once per (grid size, J, M, L, R) and kept for later calls.
#include "qb_engine.h"

extern "C" {
#include "qbgpu.h"
}

#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

namespace {

// dst[i * per + k] = src[i][k]
__global__ void k_gather(const double2 *const *__restrict__ src, long per, int count, double2 *__restrict__ dst) {
	const long n = per * count;
	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
		dst[i] = src[i / per][i % per];
}
// dst[i][k] = src[i * per + k]
__global__ void k_scatter(const double2 *__restrict__ src, long per, int count, double2 *const *__restrict__ dst) {
	const long n = per * count;
	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
		dst[i / per][i % per] = src[i];
}

using QuadKey = std::tuple<int, int, int, int, double, double>;   // device, N, J, M, L, R
std::mutex g_mu;
std::map<QuadKey, std::unique_ptr<qb::Quad>> g_quads;
std::map<std::tuple<int, int, int>, std::unique_ptr<qb::Workspace>> g_ws;   // (device, N, precision)

struct Group {
	qb::DevBuf ptrs, state_a, state_b, bfield;
};
std::map<std::pair<int, int>, std::unique_ptr<Group>> g_groups;      // (device, N)

}  // namespace

extern "C" int qb_homogeneous_batch_ex(int ninst, const int *n, void *const *W, const double *B, double dt, unsigned steps, int rk4,
                                       int precision, int J, int M, double L, double R, void *stream) {
	try {
		if (precision != 64 && precision != 32) QB_FAIL("qb_homogeneous_batch_ex: precision must be 64 or 32");
		if (ninst <= 0 || steps == 0) return 0;
		if (n == nullptr || W == nullptr) QB_FAIL("qb_homogeneous_batch: null size or state array");
		std::lock_guard<std::mutex> lk(g_mu);
		int dev = 0;
		QB_CUDA(cudaGetDevice(&dev));
		cudaStream_t s = (cudaStream_t)stream;
		std::map<int, std::vector<int>> by_n;
		for (int i = 0; i < ninst; i++) {
			if (!qb::supported_n(n[i])) QB_FAIL("qb_homogeneous_batch: grid size N=" + std::to_string(n[i]) + " of instance " + std::to_string(i) + " has no compiled kernels");
			if (W[i] == nullptr) QB_FAIL("qb_homogeneous_batch: null state of instance " + std::to_string(i));
			by_n[n[i]].push_back(i);
		}
		for (auto &kv : by_n) {
			const int N = kv.first;
			const std::vector<int> &idx = kv.second;
			const int g = (int)idx.size();
			const long per = 4L * N * N;
			auto &quad = g_quads[QuadKey(dev, N, J, M, L, R)];
			if (!quad) quad = qb::make_quad(N, J, M, L, R, s);
			auto &ws = g_ws[std::make_tuple(dev, N, precision)];
			if (!ws) {
				ws = std::make_unique<qb::Workspace>(N);
				ws->prec = precision;
			}
			auto &grp = g_groups[{ dev, N }];
			if (!grp) grp = std::make_unique<Group>();
			std::vector<const double2 *> src(g);
			std::vector<double> bh(3L * g, 0.0);
			for (int k = 0; k < g; k++) {
				src[k] = (const double2 *)W[idx[k]];
				if (B) for (int c = 0; c < 3; c++) bh[3L * k + c] = B[3L * idx[k] + c];
			}
			grp->ptrs.ensure(sizeof(double2 *) * g);
			grp->state_a.ensure(sizeof(double2) * per * g);
			grp->state_b.ensure(sizeof(double2) * per * g);
			grp->bfield.ensure(sizeof(double) * 3 * g);
			// pageable sources: the copies have been staged when the calls return
			QB_CUDA(cudaMemcpyAsync(grp->ptrs.p, src.data(), sizeof(double2 *) * g, cudaMemcpyHostToDevice, s));
			QB_CUDA(cudaMemcpyAsync(grp->bfield.p, bh.data(), sizeof(double) * 3 * g, cudaMemcpyHostToDevice, s));
			const unsigned nb = (unsigned)std::min<long>((per * g + 255) / 256, 148L * 16);
			k_gather<<<nb, 256, 0, s>>>(grp->ptrs.as<const double2 *const>(), per, g, grp->state_a.as<double2>());
			QB_CUDA(cudaGetLastError());
			double2 *cur = grp->state_a.as<double2>(), *nxt = grp->state_b.as<double2>();
			for (unsigned st = 0; st < steps; st++) {
				if (rk4) qb::collision_step_rk4(*ws, quad->set(), g, cur, grp->bfield.as<double>(), dt, nxt, s);
				else qb::collision_step(*ws, quad->set(), g, cur, grp->bfield.as<double>(), dt, nxt, s);
				std::swap(cur, nxt);
			}
			k_scatter<<<nb, 256, 0, s>>>(cur, per, g, grp->ptrs.as<double2 *const>());
			QB_CUDA(cudaGetLastError());
			// the host vectors above are read by the asynchronous copies only
			// until they return (pageable memory is staged); the device
			// buffers of this group are reused by the next call on `s`
		}
		return 0;
	} catch (const std::exception &) {
		return -1;
	}
}

extern "C" int qb_homogeneous_batch(int ninst, const int *n, void *const *W, const double *B, double dt, unsigned steps, int rk4,
                                    int J, int M, double L, double R, void *stream) {
	return qb_homogeneous_batch_ex(ninst, n, W, B, dt, steps, rk4, 64, J, M, L, R, stream);
}

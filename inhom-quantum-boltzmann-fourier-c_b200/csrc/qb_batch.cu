// qb_batch.cu — spatially homogeneous collision steps for a batch of
// independent instances of different grid sizes (the time loop of upstream
// SimulationHomogeneous, src/simulation.c:1219-1281, run on many instances
// at once).
//
// Instances of equal grid size are gathered into one contiguous group and
// advanced together: one batched launch sequence per group and step, so a
// batch of thousands of small instances costs a few launches per size
// instead of a few per instance.  On top of that:
//   - every group runs on its own stream, forked from and joined to the
//     caller's stream with events, so the groups of different sizes overlap
//     on the GPU;
//   - the first call for a (device, size, instance count, precision, method,
//     tables) tunes the group's schedule by timing candidate settings on the
//     device -- multipliers of the heuristic chunk counts of the quadrature
//     sums, and where they exist the alternative I3 schedules (the term ranges
//     or the (cell, chunk) grid of the FP64 sums at N = 32; the FFT kernels or
//     the tensor-core DFT-GEMMs of the FP32 form at N = 16), or for the sizes
//     of the any-N engine its radix schedules, tile heights and wave budgets
//     -- and keeps the fastest;
//   - the steps of all groups are captured once into a CUDA graph of two
//     steps (state a -> b -> a), which is then relaunched.
// The quadrature tables, workspaces, group buffers, schedules and the graph
// are kept for later calls.
#include "qb_engine.h"

extern "C" {
#include "qbgpu.h"
}

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
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
	cudaStream_t stream = nullptr;
	cudaEvent_t done = nullptr;
	~Group() {
		if (done) cudaEventDestroy(done);
		if (stream) cudaStreamDestroy(stream);
	}
};
std::map<std::tuple<int, int, int>, std::unique_ptr<Group>> g_groups;      // (device, N, precision)

// a group's schedule: the workspace knobs (qb::Workspace) and its measured step time
struct Sched {
	float s12 = 1.0f, s3 = 1.0f;
	int ranges = -1, variant = 0;
	int plan = 0, lines = 0;          // any-N engine: radix-plan variant, lines per tile (0: default)
	int fused = -1;                   // any-N engine: whole-grid I3 chains (1), three passes (0), default (-1)
	float wave_mb = 0.0f;             // any-N engine: wave budget (0: default)
	double ms = 0.0;
};
// (device, N, precision, instances, rk4, J, M, L, R)
using SchedKey = std::tuple<int, int, int, int, int, int, int, double, double>;
std::map<SchedKey, Sched> g_sched;

struct BatchGraph {
	std::vector<double> key;
	cudaGraphExec_t exec = nullptr;
	unsigned long long generation = 0;   // buffer_generation() at capture
};
std::map<int, BatchGraph> g_graph;                 // per device: the graph of the last batch layout
// per device: the fork event of the groups' streams, and the stream the graph
// is captured and launched on (the caller's stream may be the legacy default
// stream, which cannot be captured) with the events that order it after and
// before the caller's stream
struct DevSync {
	cudaEvent_t fork = nullptr, in = nullptr, out = nullptr;
	cudaStream_t cap = nullptr;
};
std::map<int, DevSync> g_sync;

bool env_on(const char *name) {
	const char *e = getenv(name);
	return e == nullptr || strcmp(e, "0") != 0;
}

void apply(qb::Workspace &ws, const Sched &sc) {
	ws.chunk_scale12 = sc.s12;
	ws.chunk_scale3 = sc.s3;
	ws.i3_ranges = sc.ranges;
	ws.i3_variant = sc.variant;
	ws.anyn_plan = sc.plan;
	ws.anyn_lines = sc.lines;
	ws.anyn_wave_mb = sc.wave_mb;
	ws.anyn_fused = sc.fused;
}

void step_one(qb::Workspace &ws, const qb::Quad &q, int g, const double2 *in, const double *B, double dt, double2 *out, int rk4,
              cudaStream_t s) {
	if (rk4) qb::collision_step_rk4(ws, q.set(), g, in, B, dt, out, s);
	else qb::collision_step(ws, q.set(), g, in, B, dt, out, s);
}

// time the candidate schedules of one group on its stream: one warm-up step
// with the default schedule, then one timed step per candidate (input a,
// output b: the state is not advanced); the fastest is applied and returned.
// A group whose default step takes longer than kTuneLimitMs already fills
// the GPU with work units: it keeps the default without trying the others.
constexpr double kTuneLimitMs = 500.0;
Sched autotune(qb::Workspace &ws, const qb::Quad &q, int N, int prec, int g, const double2 *a, double2 *b, const double *B,
               double dt, int rk4, cudaStream_t s) {
	std::vector<Sched> cand(1);
	if (qb::anyn_route(N)) {
		// the any-N engine: radix schedules (fewest stages, radix 8 first, radix 3
		// first, radix 4 only), tile heights (lines per tile), wave budgets, and the
		// three-pass I3 chains against the whole-grid ones (both forced; the
		// default picks by precision)
		// (the engine's defaults: tiles of about 4096 elements in FP32, 2048 in
		// FP64; a 64 MB wave budget)
		const int P = 2 * N, dl = std::max(1, (prec == 32 ? 4096 : 2048) / P);
		for (int v : { 1, 2, 3 }) { Sched c; c.plan = v; cand.push_back(c); }
		for (int nl : { dl / 2, 2 * dl }) if (nl >= 1 && nl <= P) { Sched c; c.lines = nl; cand.push_back(c); }
		for (float mb : { 24.0f, 128.0f }) { Sched c; c.wave_mb = mb; cand.push_back(c); }
		for (int f : { 0, 1 }) { Sched c; c.fused = f; cand.push_back(c); }
	} else {
		cand.resize(5);
		cand[1].s12 = 0.5f;
		cand[2].s12 = 2.0f;
		cand[3].s3 = 0.5f;
		cand[4].s3 = 2.0f;
		if (N == 32 && prec == 64) { Sched c; c.ranges = 0; cand.push_back(c); }
		if (N == 16 && prec == 32) { Sched c; c.variant = 1; cand.push_back(c); }
	}
	cudaEvent_t e0, e1;
	QB_CUDA(cudaEventCreate(&e0));
	QB_CUDA(cudaEventCreate(&e1));
	apply(ws, cand[0]);
	step_one(ws, q, g, a, B, dt, b, rk4, s);
	Sched best;
	best.ms = 1e300;
	for (Sched &c : cand) {
		apply(ws, c);
		if (&c != &cand[0]) step_one(ws, q, g, a, B, dt, b, rk4, s);     // sizes the buffers of this schedule
		QB_CUDA(cudaEventRecord(e0, s));
		step_one(ws, q, g, a, B, dt, b, rk4, s);
		QB_CUDA(cudaEventRecord(e1, s));
		QB_CUDA(cudaEventSynchronize(e1));
		float ms = 0.0f;
		QB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
		c.ms = ms;
		if (c.ms < best.ms) best = c;
		if (&c == &cand[0] && c.ms > kTuneLimitMs) break;
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	apply(ws, best);
	return best;
}

struct Live {             // one group of this call
	int N, g;
	long per;
	qb::Workspace *ws;
	qb::Quad *quad;
	Group *grp;
	double2 *cur, *nxt;
};

// one step of every group, each on its own stream between a fork and a join on s
void step_all(std::vector<Live> &lv, double dt, int rk4, cudaEvent_t fork, cudaStream_t s) {
	QB_CUDA(cudaEventRecord(fork, s));
	for (Live &l : lv) {
		QB_CUDA(cudaStreamWaitEvent(l.grp->stream, fork, 0));
		step_one(*l.ws, *l.quad, l.g, l.cur, l.grp->bfield.as<double>(), dt, l.nxt, rk4, l.grp->stream);
		QB_CUDA(cudaEventRecord(l.grp->done, l.grp->stream));
		std::swap(l.cur, l.nxt);
	}
	for (Live &l : lv) QB_CUDA(cudaStreamWaitEvent(s, l.grp->done, 0));
}

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
		const bool tune = env_on("QB_BATCH_TUNE");
		std::vector<Live> lv;
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
			auto &grp = g_groups[std::make_tuple(dev, N, precision)];
			if (!grp) {
				grp = std::make_unique<Group>();
				QB_CUDA(cudaStreamCreateWithFlags(&grp->stream, cudaStreamNonBlocking));
				QB_CUDA(cudaEventCreateWithFlags(&grp->done, cudaEventDisableTiming));
			}
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
			const SchedKey sk(dev, N, precision, g, rk4 ? 1 : 0, J, M, L, R);
			auto it = g_sched.find(sk);
			if (it != g_sched.end()) {
				apply(*ws, it->second);
			} else if (tune) {
				g_sched[sk] = autotune(*ws, *quad, N, precision, g, grp->state_a.as<double2>(), grp->state_b.as<double2>(),
				                       grp->bfield.as<double>(), dt, rk4, s);
			} else {
				apply(*ws, Sched{});
			}
			lv.push_back(Live{ N, g, per, ws.get(), quad.get(), grp.get(), grp->state_a.as<double2>(), grp->state_b.as<double2>() });
		}
		DevSync &ds = g_sync[dev];
		if (ds.fork == nullptr) {
			QB_CUDA(cudaEventCreateWithFlags(&ds.fork, cudaEventDisableTiming));
			QB_CUDA(cudaEventCreateWithFlags(&ds.in, cudaEventDisableTiming));
			QB_CUDA(cudaEventCreateWithFlags(&ds.out, cudaEventDisableTiming));
			QB_CUDA(cudaStreamCreateWithFlags(&ds.cap, cudaStreamNonBlocking));
		}
		unsigned done = 0;
		if (steps >= 2 && env_on("QB_CUDA_GRAPHS")) {
			// the layout and parameters the graph is captured for
			std::vector<double> key = { dt, (double)rk4, (double)precision, (double)J, (double)M, L, R };
			for (const Live &l : lv) {
				key.push_back((double)l.N);
				key.push_back((double)l.g);
				key.push_back((double)(uintptr_t)l.cur);
				key.push_back((double)(uintptr_t)l.nxt);
				key.push_back((double)(uintptr_t)l.grp->bfield.p);
			}
			BatchGraph &bg = g_graph[dev];
			if (bg.key != key || bg.generation != qb::buffer_generation()) {
				if (bg.exec) { cudaGraphExecDestroy(bg.exec); bg.exec = nullptr; }
				bg.key = key;
			}
			// two steps run directly until none of them reallocated a buffer (the
			// first steps of a layout size the buffers of its schedules); then two
			// steps are captured (a -> b -> a) on the capture stream and relaunched
			while (done + 2 <= steps && bg.exec == nullptr) {
				const unsigned long long gen0 = qb::buffer_generation();
				step_all(lv, dt, rk4, ds.fork, s);
				step_all(lv, dt, rk4, ds.fork, s);
				done += 2;
				if (qb::buffer_generation() == gen0) {
					cudaGraph_t gr = nullptr;
					QB_CUDA(cudaStreamBeginCapture(ds.cap, cudaStreamCaptureModeThreadLocal));
					step_all(lv, dt, rk4, ds.fork, ds.cap);
					step_all(lv, dt, rk4, ds.fork, ds.cap);
					QB_CUDA(cudaStreamEndCapture(ds.cap, &gr));
					QB_CUDA(cudaGraphInstantiate(&bg.exec, gr, 0));
					cudaGraphDestroy(gr);
					bg.generation = qb::buffer_generation();
				}
			}
			if (bg.exec != nullptr && done + 2 <= steps) {
				QB_CUDA(cudaEventRecord(ds.in, s));
				QB_CUDA(cudaStreamWaitEvent(ds.cap, ds.in, 0));
				while (done + 2 <= steps) {
					QB_CUDA(cudaGraphLaunch(bg.exec, ds.cap));
					done += 2;
				}
				QB_CUDA(cudaEventRecord(ds.out, ds.cap));
				QB_CUDA(cudaStreamWaitEvent(s, ds.out, 0));
			}
		}
		while (done < steps) {
			step_all(lv, dt, rk4, ds.fork, s);
			done++;
		}
		for (const Live &l : lv) {
			const unsigned nb = (unsigned)std::min<long>((l.per * l.g + 255) / 256, 148L * 16);
			k_scatter<<<nb, 256, 0, s>>>(l.cur, l.per, l.g, l.grp->ptrs.as<double2 *const>());
			QB_CUDA(cudaGetLastError());
		}
		// the host vectors above are read by the asynchronous copies only until
		// they return (pageable memory is staged); the device buffers of the
		// groups are reused by the next call on `s`
		return 0;
	} catch (const std::exception &) {
		return -1;
	}
}

extern "C" int qb_homogeneous_batch(int ninst, const int *n, void *const *W, const double *B, double dt, unsigned steps, int rk4,
                                    int J, int M, double L, double R, void *stream) {
	return qb_homogeneous_batch_ex(ninst, n, W, B, dt, steps, rk4, 64, J, M, L, R, stream);
}

extern "C" int qb_batch_schedules(char *buf, int len) {
	std::lock_guard<std::mutex> lk(g_mu);
	std::string out = "[";
	for (const auto &kv : g_sched) {
		const SchedKey &k = kv.first;
		const Sched &c = kv.second;
		char line[448];
		snprintf(line, sizeof(line),
		         "%s{\"device\": %d, \"N\": %d, \"precision\": %d, \"instances\": %d, \"rk4\": %d, \"J\": %d, \"M\": %d, "
		         "\"chunk_scale_i1_i2_i4\": %g, \"chunk_scale_i3\": %g, \"i3_ranges\": %d, \"i3_variant\": %d, "
		         "\"anyn_plan\": %d, \"anyn_lines\": %d, \"anyn_wave_mb\": %g, \"anyn_fused\": %d, \"step_ms\": %.4f}",
		         out.size() > 1 ? ", " : "", std::get<0>(k), std::get<1>(k), std::get<2>(k), std::get<3>(k), std::get<4>(k),
		         std::get<5>(k), std::get<6>(k), c.s12, c.s3, c.ranges, c.variant, c.plan, c.lines, c.wave_mb, c.fused, c.ms);
		out += line;
	}
	out += "]";
	if (buf != nullptr && len > 0) {
		strncpy(buf, out.c_str(), (size_t)len - 1);
		buf[len - 1] = 0;
	}
	return (int)out.size();
}

// qb_engine.h — internal C++ interface of the GPU engine (run-time grid size N).
//
// The C-ABI layers (qb_abi.cu: the upstream API at compile-time N_GRID;
// qb_ext.cu: the batched device-pointer API) are thin clients of this.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

namespace qb {

// ---- errors ---------------------------------------------------------------
// Every failed CUDA call or invalid argument records a message retrievable
// through qb_last_error(); unless QB_ABORT_ON_ERROR=0 the process then aborts,
// because the upstream entry points return void and callers could otherwise
// continue with garbage.
void fail(const char *file, int line, const std::string &msg);
#define QB_FAIL(msg) ::qb::fail(__FILE__, __LINE__, (msg))
#define QB_CUDA(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) ::qb::fail(__FILE__, __LINE__, std::string(#call) + ": " + cudaGetErrorString(e_)); } while (0)
bool supported_n(int N);      // grid sizes with kernels: the fixed sizes 8, 16, 32, 64 and the any-N engine's

// ---- device buffers ---------------------------------------------------------
// Process-wide count of device-buffer reallocations and releases: a captured
// CUDA graph holds raw buffer addresses, so it is replayed only while this
// count is unchanged since its capture.
unsigned long long buffer_generation();
struct DevBuf {
	void *p = nullptr;
	size_t bytes = 0;
	int device = -1;
	DevBuf() = default;
	DevBuf(const DevBuf &) = delete;
	DevBuf &operator=(const DevBuf &) = delete;
	DevBuf(DevBuf &&o) noexcept : p(o.p), bytes(o.bytes), device(o.device) { o.p = nullptr; o.bytes = 0; }
	DevBuf &operator=(DevBuf &&o) noexcept {
		if (this != &o) { release(); p = o.p; bytes = o.bytes; device = o.device; o.p = nullptr; o.bytes = 0; }
		return *this;
	}
	void ensure(size_t n);        // grow (contents discarded)
	void release();
	~DevBuf() { release(); }
	template <class T> T *as() const { return static_cast<T *>(p); }
};

// ---- quadrature tables on the device -----------------------------------------
// I1-type (I1 and I4):  S = sum_t phi_t . IFFT2(F . FFT2(Pad(psi2_t . g)))
// Each table set also holds FP32 roundings of its tables (the *f buffers),
// made on first use by the FP32 precision form.
struct DevI1 { int N = 0, nterms = 0; DevBuf psi2, phi; mutable DevBuf psi2f, phif; };
// I2-type: Q = sum_t FFT2(Pad(psi1_t f)) . FFT2(Pad(psi2_t g))
struct DevI2 { int N = 0, nterms = 0; DevBuf psi1, psi2; mutable DevBuf psi1f, psi2f; };
// I3-type: psi1_t complex N x N; psi2_t = scale[t] * table[idx[t]] (tables stored transposed)
struct DevI3 { int N = 0, nterms = 0; DevBuf psi1, psi2T, idx, scale; mutable DevBuf psi1f, psi2Tf; };

struct QuadSet { const DevI1 *i1 = nullptr; const DevI2 *i2 = nullptr; const DevI3 *i3 = nullptr; const DevI1 *i4 = nullptr; };

// Builders (all on the GPU).  `host_*` receive the upstream-layout tables
// when non-null (FourierI* fill the caller's quad structs with them).
void build_i1(int N, int J, double L, double R, DevI1 &dev, double *host_psiR1, double *host_psiR2, cudaStream_t s);
void build_i2(int N, int J, double L, double R, DevI2 &dev, double *host_psiR1, double *host_psiR2, cudaStream_t s);
void build_i3(int N, int J, double L, double R, int M, DevI3 &dev, double *host_psiR1, double *host_psiR2, cudaStream_t s);
void build_i4(int N, int J, double L, double R, DevI1 &dev, double *host_psiR1, double *host_psiR2, cudaStream_t s);
void lgwt_device(int M, double a, double b, double *x_host, double *w_host, cudaStream_t s);
// upload caller-built tables (upstream layouts) as generic term lists
void upload_i1(int N, int num, const double *psiR1, const double *psiR2, DevI1 &dev, cudaStream_t s);
void upload_i2(int N, int num, const double *psiR1, const double *psiR2, DevI2 &dev, cudaStream_t s);
void upload_i3(int N, int num, const double *psiR1, const double *psiR2, DevI3 &dev, cudaStream_t s);

// A complete (N, J, M, L, R) table set
struct Quad {
	int N, J, M; double L, R;
	DevI1 i1, i4; DevI2 i2; DevI3 i3;
	QuadSet set() const { QuadSet q; q.i1 = &i1; q.i2 = &i2; q.i3 = &i3; q.i4 = &i4; return q; }
};
std::unique_ptr<Quad> make_quad(int N, int J, int M, double L, double R, cudaStream_t s);

// ---- workspace: scratch for one evaluation stream ------------------------------
struct Workspace {
	int N = 0, device = -1;
	int prec = 64;                           // working precision of the collision operator: 64 (FP64) or 32 (FP32 form)
	int conserve = 0;                        // restore the collision invariants after each velocity-space collision step
	cudaStream_t stream = nullptr;           // own stream (upstream API calls)
	DevBuf What, i1cc, i1i4, i2p, i3p, fs, fs4, wmid;      // collision scratch
	DevBuf fa, fb, va, vb;                   // state scratch (Fourier / velocity)
	DevBuf io_in, io_out, bext, vgrid;       // staging for host-pointer calls
	DevBuf aux, aux2;
	DevBuf inv;                              // per-cell collision invariants (conservation on)
	DevBuf scr128a, scr128b;                 // N = 64: per-cluster spectra of the I3 terms, first I2 spectra
	DevBuf i3kind;                           // FP32 I3 sums: per-cell form (0 real, 1 complex)
	DevBuf i3stats;                          // FP32 I3 sums: cells evaluated by the real form, by either form (2 x u64)
	DevBuf kerr;                             // device error word of kernels with bounded waits (nonzero: a wait ran out)
	DevBuf wave1, wave2;                     // any-N engine: per-wave scratch of the quadrature sums, assembly scratch
	// any-N engine knobs (0: default): radix-plan variant, lines per tile, wave budget in MB
	int anyn_plan = 0, anyn_lines = 0;
	int anyn_fused = -1;                     // any-N engine: whole-grid I3 chains (1), three passes (0), the engine's default (-1)
	float anyn_wave_mb = 0.0f;
	DevBuf anyn_tw;                          // any-N engine: roots of unity of the padded grid (double2, then float2)
	int i3_variant = 0;                      // I3 sums: 0 the FFT kernels, 1 DFT-GEMMs on the tensor cores (FP32 form, N = 16)
	// schedule knobs (set by the batch autotuner): multipliers of the heuristic
	// chunk counts of the I1/I2/I4 sums and of the I3 sums, and the FP64 I3
	// schedule at N = 32 (-1: the default, 0: (cell, chunk) grid, 1: term ranges)
	float chunk_scale12 = 1.0f, chunk_scale3 = 1.0f;
	int i3_ranges = -1;
	double tables_L = -1.0;                  // box half-width the velocity tables in `vgrid` were built for
	// replay of repeated Strang steps (batched API): the launch sequence of a
	// (pointers, parameters) key is captured on its second call and relaunched
	// afterwards; a few keys are kept, so that ping-pong buffers replay too
	struct GraphEntry {
		std::vector<double> key;
		cudaGraphExec_t exec = nullptr;
		unsigned long long generation = 0;   // buffer_generation() when the key was sized / captured
		unsigned long long last_use = 0;
		long kernels = 0;                    // kernel nodes of the captured sequence
	};
	static constexpr int kGraphSlots = 4;
	std::vector<GraphEntry> graphs;
	unsigned long long graph_clock = 0;
	long graph_replays = 0;                  // launches served by an instantiated graph
	cudaEvent_t ev_in = nullptr, ev_out = nullptr;
	// the sharded step (qb_sharded_step): a second workspace for the edge cells,
	// which collide on the caller's stream while the interior collides on `stream`
	std::unique_ptr<Workspace> edge;
	cudaEvent_t ev_t = nullptr, ev_i = nullptr;
	explicit Workspace(int N);
	~Workspace();
};

// a kernel that allocates tensor memory, for the co-residency check
struct TmemKernel { const void *fn; size_t dyn_smem; int threads; int cols; const char *name; };
std::vector<TmemKernel> dftmma_tmem_kernels();
std::vector<TmemKernel> fno_tmem_kernels();
// before the first launch of a tensor-memory kernel on a device: no set of
// tensor-memory kernels that can share an SM asks for more than 512 columns
void ensure_tmem_coresidency();

// chunking of the quadrature-term sums over CTAs (picked per launch shape)
struct Chunks {
	int i1 = 1, i2 = 1, i3 = 1;
	int i3_slots = 0;                        // > 0: the I3 sums run as that many contiguous (cell, term) ranges instead of chunks
};
Chunks pick_chunks(int N, int ncells, const QuadSet &q, int prec);

// ---- operators (device pointers, stream-ordered) ------------------------------
enum RhsParts { RHS_CC = 1, RHS_CD = 2, RHS_ALL = 3 };

// Cc and/or Cd of ncells Fourier states W ([cell][4][N*N] complex):
// out_cc / out_cd may be null when not requested.
void collision_operators(Workspace &ws, const QuadSet &q, int ncells, const double2 *W, int parts,
                         double2 *out_cc, double2 *out_cd, cudaStream_t s);
// out = base + dtc * (Cc + Cd + CB)(wcur)
void collision_update(Workspace &ws, const QuadSet &q, int ncells, const double2 *base, const double2 *wcur,
                      const double *B, double dtc, double2 *out, cudaStream_t s);
// midpoint collision step (upstream CollisionStep), Wnext may not alias W
void collision_step(Workspace &ws, const QuadSet &q, int ncells, const double2 *W, const double *B, double dt,
                    double2 *Wnext, cudaStream_t s);
// classical RK4 on the same right-hand side (extension; upstream has midpoint only)
void collision_step_rk4(Workspace &ws, const QuadSet &q, int ncells, const double2 *W, const double *B, double dt,
                        double2 *Wnext, cudaStream_t s);

// generic single-triple integrals (upstream I1integral / I2integral / I3integral)
void integral_i1(Workspace &ws, const DevI1 &t, const double2 *f, const double2 *g, const double2 *h, double2 *out, cudaStream_t s);
void integral_i2(Workspace &ws, const DevI2 &t, const double2 *f, const double2 *g, const double2 *h, double2 *out, cudaStream_t s);
void integral_i3(Workspace &ws, const DevI3 &t, const double2 *f, const double2 *g, const double2 *h, double2 *out, cudaStream_t s);

// the any-N engine (qb_anyn.cu): grid sizes N with 2N = 2^a 3^b up to 128
// that have no fixed-size kernels (N = 24, 48, 96, 128, ...); QB_ANYN=1
// routes the fixed sizes through it too (a cross-check of the two engines)
bool anyn_supported(int N);
bool anyn_route(int N);
void anyn_operators(Workspace &ws, const QuadSet &q, int ncells, const double2 *W, int parts, double2 *out_cc, double2 *out_cd, cudaStream_t s);
void anyn_update(Workspace &ws, const QuadSet &q, int ncells, const double2 *base, const double2 *wcur, const double *B, double dtc,
                 double2 *out, cudaStream_t s);
// the twiddle table ws.anyn_tw (made at construction, outside any graph capture)
void anyn_build_twiddles(Workspace &ws);
void anyn_to_fourier(int N, int ngrids, const double *Wv, double2 *Wf, cudaStream_t s);
void anyn_from_fourier(int N, int ngrids, const double2 *Wf, double *Wv, cudaStream_t s);
// The FP32 I3 sums take the real form for the cells whose Nyquist content and
// anti-Hermitian part are at most 1e-6 of the state (QB_I3_KERNEL=complex or
// pair: never).  i3_form_kinds writes the per-cell form (0 real, 1 complex) of
// W [ncells][4][N*N] into ws.i3kind, counts the cells in ws.i3stats and
// returns the device array.
bool real_form_enabled();
int *i3_form_kinds(Workspace &ws, int ncells, const double2 *W, cudaStream_t s);
// FP32 roundings of a table set (made once, on the caller's stream, which is then synchronised)
void prepare_f32_tables(const QuadSet &q, cudaStream_t s);

void to_fourier(int N, int ngrids, const double *Wv, double2 *Wf, cudaStream_t s);
void from_fourier(int N, int ngrids, const double2 *Wf, double *Wv, cudaStream_t s);
// One limiter step for ncells cells of npts points ([cell][npts] layout) with
// per-point velocity A (device array of npts); dt is the step handed to the
// limiter (the Strang half step in a simulation); bc 0 periodic, 1 Dirichlet.
void transport(int npts, int ncells, const double *in, double *out, const double *A_dev, double h, double dt, int bc, cudaStream_t s);
// Maxwell-boundary limiter step on caller data (SlopeLimiterStepMaxwell):
// m points per cell, flux_dev = {fluxL, fluxR}, UL/UR m values each
void transport_maxwell_lines(int m, int ncells, const double *in, double *out, const double *A_dev, double h, double dt,
                             double lambda, const double *flux_dev, const double *UL, const double *UR, cudaStream_t s);
// sequential upstream-order flux sums: out_dev[0] rightward, out_dev[1] leftward
void flux_pair(int m, const double *A_dev, const double *U_dev, double *out_dev, cudaStream_t s);

// collision part of a Strang step on ncells velocity-space cells, in place:
// to Fourier space, CollisionStep, back (upstream InternalFourierCollisionStep);
// with ws.conserve set it also restores the trace component's mass, momentum
// and energy
void fourier_collision(Workspace &ws, const QuadSet &q, int ncells, double *V, const double *B, double dt, cudaStream_t s);
// one Strang step over ncells cells (V space): 1/2 transport, collision, 1/2 transport.
// A_dev: per-point velocities of a cell ([4][N*N], v_x of the slow index).
// bc 0 periodic (all cells collide), 1 Dirichlet (first and last cell skip the collision)
void inhom_step(Workspace &ws, const QuadSet &q, int ncells, const double *W, double *Wnext, const double *A_dev,
                double h, double dt, const double *Bext, int bc, cudaStream_t s);
// Maxwell boundaries: vx_dev = N*N Maxwell-grid x velocities, WL/WR one
// velocity-space state each (device)
void inhom_step_maxwell(Workspace &ws, const QuadSet &q, int ncells, const double *W, double *Wnext, const double *vx_dev,
                        double h, double dt, double lambda, const double *WL, const double *WR, const double *Bext, cudaStream_t s);

// generic 2-D FFT of one L x L grid (FFTW-API plans): r2c writes L x (L/2+1)
bool fft2_generic_supported(int n0, int n1);
void fft2_generic(int L, int dir, bool r2c, const void *in_dev, double2 *out_dev, cudaStream_t s);

std::string last_error();

// ---- launch accounting -------------------------------------------------------
// Every kernel launch of the engine goes through prof_launch(): it counts
// launches and, while profiling is enabled, brackets the launch with CUDA
// events on its stream so per-kernel device time can be read back.
void prof_enable(bool on);
bool prof_enabled();
void prof_reset();
// kernels launched so far, the nodes of replayed CUDA graphs included
long launch_count();
void add_launches(long n);
// total device milliseconds and launches recorded for kernels whose name starts with `prefix`
void prof_read(const char *prefix, double *ms, long *launches);
struct ProfScope {
	const char *name; cudaStream_t s; cudaEvent_t e0 = nullptr, e1 = nullptr;
	ProfScope(const char *n, cudaStream_t st);
	~ProfScope();
};

}  // namespace qb

// opaque handle types of the C headers
struct qb_workspace : public qb::Workspace {
	using qb::Workspace::Workspace;
};
struct qb_quad {
	std::unique_ptr<qb::Quad> q;
};

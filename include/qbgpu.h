/* qbgpu.h — batched, device-resident extension API of libqbgpu.
 *
 * The upstream API (collision.h, integrals.h, simulation.h, ...) works on one
 * host state per call with a compile-time N_GRID.  These entry points take
 * the grid size at run time, operate on many cells per call, and take DEVICE
 * pointers plus a CUDA stream (cudaStream_t; NULL = the legacy default stream),
 * so a caller
 * that keeps the state resident in HBM pays no host transfers per step.
 * Layouts are the upstream ones laid end to end: a velocity-space cell is
 * wignerV_t (4 real N x N grids), a Fourier-space cell is wignerF_t (4 complex
 * N x N grids, interleaved re/im), cells are consecutive.
 *
 * Every function returns 0 on success.  On failure it records a message for
 * qb_last_error() and, unless the environment sets QB_ABORT_ON_ERROR=0,
 * aborts the process; with QB_ABORT_ON_ERROR=0 it returns -1.
 * None of these has an upstream counterpart; each names the upstream function
 * whose arithmetic it batches.
 */
#ifndef QBGPU_H
#define QBGPU_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct qb_quad qb_quad;              /* device quadrature tables for (N, J, M, L, R) */
typedef struct qb_workspace qb_workspace;    /* device scratch + stream for one grid size */

const char *qb_last_error(void);
int qb_n_grid(void);                          /* N_GRID this library's upstream API was built for */
int qb_supported_n(int N);                    /* 1 if kernels for grid size N are compiled */

/* FourierI1..I4 (upstream src/quadrature.c:150-527) built on the GPU */
qb_quad *qb_quad_create(int N, int J, int M, double L, double R);
void qb_quad_free(qb_quad *q);

qb_workspace *qb_workspace_create(int N);
void qb_workspace_free(qb_workspace *ws);

/* working precision of the collision operator evaluated through `ws`:
 * 64 (default) is the plain FP64 path of the upstream code; 32 is the FP32
 * precision form, which has no upstream counterpart: the Wigner state, the
 * Pauli-blocking assembly, the magnetic term and the time update stay FP64,
 * while the spectra, the quadrature tables (rounded once per table set) and
 * every FFT of the factored integrals run in FP32.  Transport is unaffected.
 * The first FP32 evaluation with a table set rounds its tables and
 * synchronises the stream, so it must not be inside a stream capture. */
int qb_workspace_set_precision(qb_workspace *ws, int bits);
int qb_workspace_precision(const qb_workspace *ws);

/* I3 sums of the collision operator (no upstream counterpart): variant 0
 * (default) runs the hand-written FFT kernels; variant 1 runs every 1-D pass
 * of the I3 chains as a GEMM against the DFT matrix on the tensor cores
 * (tcgen05.mma, TF32 operands split hi + lo, FP32 accumulation).  Variant 1
 * applies to the FP32 form at N = 16; other sizes and FP64 ignore it. */
int qb_workspace_set_i3_variant(qb_workspace *ws, int variant);

/* Synchronises the workspace's device and returns (then clears) its device
 * error word: 0 when no kernel with a bounded wait (the tensor-core I3
 * variant) gave up on a wait since the last call, 1 if one did (its outputs
 * are NaN), -1 on a host error. */
int qb_workspace_device_errors(qb_workspace *ws);

/* on != 0: the velocity-space steps through `ws` (qb_inhom_step,
 * qb_inhom_step_maxwell, qb_fourier_collision, qb_simulate_record) restore,
 * after each collision, the mass, momentum and energy of the trace component
 * w0 -- the invariants of the continuous collision operator, which the
 * discrete one keeps only to its quadrature accuracy -- by the least change
 * w0 += |w0| (l0 + l1 v_x + l2 v_y + l3 |v|^2) that puts them back.  No
 * upstream counterpart; off by default (the upstream step). */
int qb_workspace_set_conservation(qb_workspace *ws, int on);

/* The FP32 form (every N): the I3 sums of a cell whose Fourier state has a
 * Nyquist content (sum of |W| on row and column N/2 over sum of |W|, the 4
 * components) and an anti-Hermitian part of at most 1e-6 of the state run in
 * real arithmetic, two quadrature chains
 * per complex transform (exact when that content is zero); the other cells
 * take the complex kernel.  Reports the cells evaluated so far through `ws`
 * by the real form and by either form (synchronises the device); reset != 0
 * zeroes both counts. */
int qb_workspace_i3_forms(qb_workspace *ws, long long *real_cells, long long *all_cells, int reset);

/* Cc and/or Cd (CcInt / CdInt, upstream src/collision.c:74-254) of ncells
 * Fourier states; parts: 1 = Cc, 2 = Cd, 3 = both; cc / cd may be NULL. */
int qb_collision_operators(qb_workspace *ws, const qb_quad *q, int ncells, const void *W, int parts,
                           void *cc, void *cd, void *stream);

/* CollisionStep (midpoint, upstream src/simulation.c:105-136) of ncells
 * Fourier states, B = 3 doubles per cell (NULL: no field); rk4 != 0 uses
 * classical RK4 on the same right-hand side instead.  Wnext must not alias W. */
int qb_collision_step(qb_workspace *ws, const qb_quad *q, int ncells, const void *W, const double *B,
                      double dt, void *Wnext, int rk4, void *stream);

/* Spatially homogeneous collision steps for a batch of ninst independent
 * instances of possibly different grid sizes (the time loop of
 * SimulationHomogeneous, upstream src/simulation.c:1219-1281, over many
 * instances): instance i has grid size n[i] (8, 16, 32 or 64) and its Fourier
 * state at the device pointer W[i] (4 complex n[i] x n[i] grids, updated in
 * place); B (host, may be NULL = 0) holds 3 doubles per instance.  Every
 * instance advances `steps` collision steps of size dt: midpoint
 * (CollisionStep), or classical RK4 with rk4 != 0.  Instances of equal size
 * are gathered and advanced together, one batched launch sequence per size
 * and step; the quadrature (J, M, L, R) is common and its tables are built
 * once per size and kept.  Calls are serialised on the host; their GPU work
 * shares internal buffers, so calls on different streams must not overlap. */
int qb_homogeneous_batch(int ninst, const int *n, void *const *W, const double *B, double dt, unsigned steps, int rk4,
                         int J, int M, double L, double R, void *stream);
/* the same in a chosen working precision: 64 (the call above) or 32 (the
 * FP32 form of qb_workspace_set_precision: FP32 spectra, tables and FFTs, FP64
 * state and update).  The first FP32 call with a table set synchronises. */
int qb_homogeneous_batch_ex(int ninst, const int *n, void *const *W, const double *B, double dt, unsigned steps, int rk4,
                            int precision, int J, int M, double L, double R, void *stream);

/* The schedules the batch calls above have tuned so far (no upstream
 * counterpart), as a JSON array: per (device, N, precision, instance count,
 * method, J, M) the chosen multipliers of the heuristic chunk counts, the I3
 * schedule and variant, and the measured step time.  Writes at most len - 1
 * characters and a terminating zero; returns the full length.  The first batch
 * call for such a key times the candidates on the device (synchronising);
 * QB_BATCH_TUNE=0 keeps the defaults.  All groups of a call advance
 * concurrently on their own streams.  Within a call, once two direct steps
 * have reallocated no buffer, two steps at a time replay a CUDA graph of all
 * groups (QB_CUDA_GRAPHS=0: direct launches only). */
int qb_batch_schedules(char *buf, int len);

/* one Strang step of InhomStepPeriodic (bc = 0) / InhomStepDirichlet (bc = 1)
 * (upstream src/simulation.c:307-830) over ncells velocity-space cells with
 * box half-width L; Bext = 3 doubles per cell (NULL: no field).  Wnext must
 * not alias W.
 * The workspace keeps the CUDA graphs of its last 4 distinct argument sets:
 * a call whose arguments match one of them (e.g. steps that alternate two
 * state buffers) relaunches the graph captured on that set's second call.
 * QB_CUDA_GRAPHS=0, or kernel profiling being on, launches kernel by kernel. */
int qb_inhom_step(qb_workspace *ws, const qb_quad *q, int ncells, const double *W, double *Wnext,
                  double h, double dt, const double *Bext, int bc, void *stream);

/* InhomStepMaxwell (upstream src/simulation.c:879-1165); WL / WR one
 * velocity-space state each. */
int qb_inhom_step_maxwell(qb_workspace *ws, const qb_quad *q, int ncells, const double *W, double *Wnext,
                          double h, double dt, double lambda, const double *WL, const double *WR,
                          const double *Bext, void *stream);

/* One Strang step of this rank's block of a sharded periodic domain, for
 * hosts that distribute the x-cells themselves (MPI ranks, or NCCL from C);
 * it replaces upstream's MPI path of InhomStepPeriodic (src/simulation.c:
 * 316-418).  ext_a and ext_b are device buffers of ncells + 4 velocity-space
 * cells each, the haloed line [2 | local | 2]: the rank's cells start in
 * ext_a[2 .. ncells + 1], and there the step leaves them.  exchange(ext,
 * ncells, stream, user) must fill the halo cells 0, 1 and ncells + 2,
 * ncells + 3 of `ext` with the last two cells of the left neighbour and the
 * first two of the right neighbour on the periodic ring (ext's cells 2 ..
 * ncells + 1 are this rank's), ordered on `stream` (e.g. ncclSend/ncclRecv
 * there) or complete on return; it returns 0 on success.  It is called twice
 * per step: before the first half step of transport, and after the collision
 * of the two edge cells on each side, while the interior cells collide on
 * the workspace's own stream (ncells >= 6; fewer cells collide all first).
 * Bext: 3 doubles per local cell, or NULL. */
typedef int (*qb_halo_exchange_fn)(double *ext, int ncells, void *stream, void *user);
int qb_sharded_step(qb_workspace *ws, const qb_quad *q, int ncells, double *ext_a, double *ext_b, double h, double dt,
                    const double *Bext, qb_halo_exchange_fn exchange, void *user, void *stream);

/* velocity space <-> Fourier space for ngrids N x N components
 * (upstream src/simulation.c:224-283) */
int qb_to_fourier(int N, int ngrids, const double *Wv, void *Wf, void *stream);
int qb_from_fourier(int N, int ngrids, const void *Wf, double *Wv, void *stream);

/* single I1 / I2 / I3 / I4 integral (which = 1..4) of Fourier grids f, g, h
 * with the quad's tables (upstream src/integrals.c:90-382) */
int qb_integral(qb_workspace *ws, const qb_quad *q, int which, const void *f, const void *g, const void *h,
                void *out, void *stream);

/* one half-step of transport (SlopeLimiterStepPeriodic / Dirichlet over every
 * x-line, upstream src/simulation.c:426-448) for ncells velocity-space cells
 * of grid size N in a box of half-width L: out = limiter(in) with step dt. */
int qb_transport(int N, double L, int ncells, const double *in, double *out, double h, double dt, int bc, void *stream);

/* the collision part of a Strang step on ncells velocity-space cells, in
 * place: to Fourier space, CollisionStep, back (InternalFourierCollisionStep,
 * upstream src/simulation.c:214-284) */
int qb_fourier_collision(qb_workspace *ws, const qb_quad *q, int ncells, double *W, const double *Bext, double dt, void *stream);

/* Strang steps of ncells cells (bc 0 periodic, 1 Dirichlet) from the HOST
 * initial state W0, state resident on the device; frame 0 (= W0) and every
 * record_every-th state are appended to `path` in the upstream trajectory
 * format (raw wignerV_t frames, as SimulationInhomogeneous* + WriteData
 * produce, upstream src/simulation.c:1288-1341, src/util.c:70-91), each frame
 * written while the GPU computes the following steps.  With record_every = 1
 * the file equals upstream's Wevolv file.  numsteps counts frames including
 * the initial one, as upstream.  The final state goes to final_out (host) if
 * non-null; path may be NULL (no recording).  Returns the number of frames
 * written, or -1. */
long qb_simulate_record(qb_workspace *ws, const qb_quad *q, int ncells, const double *W0, double h, double dt, unsigned numsteps,
                        const double *Bext, int bc, unsigned record_every, const char *path, double *final_out);

/* per-cell diagnostics of velocity-space states W (device): out (device) gets
 * 10 doubles per cell: w_tr, w_x, w_y, w_z (integrals, dv^2 included), mean
 * velocity u_x, u_y, energy per particle, smallest and largest eigenvalue of
 * W(v) over the grid, and the Fermi-Dirac entropy (upstream
 * visualization/wignerMoments.m:15-37, visualization/entropy.m). */
int qb_diagnostics(int N, double L, int ncells, const double *W, double *out, void *stream);

/* Fermi-Dirac equilibrium with the conserved moments (spin density matrix,
 * mean velocity, energy) of each of ncells velocity-space states W (device),
 * written to WFD (device, same layout) (upstream visualization/asymptoticFD.m,
 * calculateFDparams.m, createFD.m; the moments as qb_diagnostics).  The
 * inverse temperature and the two chemical potentials solve the 3 moment
 * equations by Newton's method on the host from the upstream starting points
 * (1, 1, 1), then (1, 1, 0.5).  params (host, may be NULL) gets 9 doubles per
 * cell: beta, mu_1, mu_2 (smaller / larger density eigenvalue), u_x, u_y,
 * the unit spin direction n_x, n_y, n_z of the larger eigenvalue, and the
 * residual norm of the moment equations.  Synchronises `stream`; N <= 64. */
int qb_fermi_dirac_equilibrium(int N, double L, int ncells, const double *W, double *WFD, double *params, void *stream);

/* per cell 2 doubles into out (device): the quantum relative entropy of W(v)
 * to WFD(v) (eigenvalues clamped to [eps, 1 - eps]) summed over the points
 * with WFD_0(v) > 1e-6, times dv^2, and the distance sum_j ||W_j - WFD_j||_1 dv^2
 * in the matrix 1-norm (largest sum over v_y at fixed v_x) (upstream
 * visualization/relentropy.m, visualization/visualizeHomBoltzmann.m:116-148).
 * N <= 64. */
int qb_relative_entropy(int N, double L, int ncells, const double *W, const double *WFD, double *out, void *stream);

/* launch accounting: every engine kernel launch is counted; while profiling
 * is on, launches are bracketed by CUDA events on their stream.
 * qb_profile_read sums device milliseconds and launches of kernels whose
 * name starts with `prefix` ("i3_cluster", "i1_terms", "i2_terms",
 * "pad_fft", "fft_full", "assemble", "to_fourier", "from_fourier",
 * "transport"; "" = all). */
int qb_profile_enable(int on);
int qb_profile_reset(void);
int qb_profile_read(const char *prefix, double *ms, long *launches);
/* Tensor-core self-check (no upstream counterpart): D (128 x 64) = A (128 x 64)
 * x B (64 x 64) through tcgen05.mma kind::tf32 in one CTA, with both
 * operands in the K-major shared-memory layout that the DFT-as-GEMM kernels
 * use; Bt is B transposed (row n = column n of B).  Operands are rounded to
 * TF32 (nearest); device pointers, row-major FP32. */
int qb_umma_selftest(const float *A, const float *Bt, float *D, void *stream);

/* kernels launched so far by this library, the kernel nodes of replayed CUDA
 * graphs included */
long qb_launch_count(void);
/* Strang steps of qb_inhom_step served by relaunching a captured CUDA graph */
long qb_workspace_graph_replays(const qb_workspace *ws);

/* The I3 integral of qb_integral(q, 3, ...) for callers that cannot allocate
 * device memory (a stream being captured into a CUDA graph, a host
 * application that owns all device memory, a latency-critical loop).  It has
 * no counterpart in the upstream code.  All scratch comes from one static
 * device array of 4 MiB compiled into the library; every GPU that loads the
 * library holds it until exit, and the call itself allocates nothing.  The
 * first call on a device looks up the array's address (cudaGetSymbolAddress)
 * and must come before any stream capture on that device.  Calls share the
 * array: calls that can overlap on the GPU race, so serialise them.  Grid
 * sizes up to N = 32 fit; larger ones are rejected with an error. f, g, h,
 * out: device N x N complex grids. */
int qb_integral_i3_noalloc(const qb_quad *q, const void *f, const void *g, const void *h, void *out, void *stream);

/* measured FP64 FMA throughput of the current device in TFLOP/s (a dependent-
 * free DFMA loop on every SM, ~tens of ms) -- the denominator of the FP64
 * roofline of the collision kernels. */
double qb_fp64_peak_tflops(void);

/* ---- learned surrogate of the collision operator (no upstream counterpart) --
 * A Fourier neural operator maps one velocity-space cell W (4 real N x N
 * grids, FP64) to an approximation of C[W] = Cc + Cd (velocity space, FP64).
 * Its input features are the 4 Pauli components and their 10 pairwise
 * products w_i w_j (i <= j, order (0,0), (0,1), ..., (3,3)), each times a
 * fixed input scale; a lift to `width` channels, `layers` spectral layers
 * (truncated DFT to `modes` x (2 modes - 1) frequencies, complex mode mixing,
 * inverse DFT, plus a pointwise map; GELU between layers) and a projection to
 * 4 channels follow, whose outputs are multiplied by the per-component output
 * scales.  Arithmetic is FP32; the forward pass, the backward pass and Adam
 * are the library's own kernels, and every reduction is in a fixed order, so
 * gradients and trained weights are deterministic.  All state pointers are
 * device pointers. */
typedef struct qb_fno qb_fno;
/* N even, 4..64; 1 <= width <= 64; 2 modes - 1 <= N; 1 <= layers <= 16.
 * Weights are drawn from a seeded normal distribution.  NULL on error. */
qb_fno *qb_fno_create(int N, int width, int modes, int layers, unsigned long long seed);
void qb_fno_free(qb_fno *net);
long qb_fno_num_params(const qb_fno *net);
int qb_fno_grid_size(const qb_fno *net);                         /* N, or -1 for NULL */
/* all weights as one FP32 array of qb_fno_num_params() values (host memory):
 * A[width][14], a[width], per layer Rr[width][width][K], Ri[..], W[width][width],
 * b[width], then Q[4][width], q[4]; K = (2 modes - 1) modes, frequency
 * k = (kx + modes - 1) modes + ky */
int qb_fno_get_params(const qb_fno *net, float *host);
int qb_fno_set_params(qb_fno *net, const float *host);
int qb_fno_set_scale(qb_fno *net, const double *scale);          /* 4 output scales (> 0) */
int qb_fno_set_input_scale(qb_fno *net, const double *scale);    /* 14 input scales (> 0) */
/* Extension, no counterpart in the reference: on != 0 runs the pointwise
 * channel maps (the lift, each layer's W, the projection, and their
 * transposes in the backward pass) and the truncated DFTs and their inverses
 * on the tensor cores with BF16 operands and FP32 accumulation (tcgen05.mma,
 * accumulator in tensor memory); the mode mixing and the weight gradients
 * stay FP32.  Off by default. */
int qb_fno_set_tensor_cores(qb_fno *net, int on);
/* nonzero when a tensor-core MMA of the network did not complete within its
 * poll limit (its outputs are then undefined); 0 otherwise */
int qb_fno_device_errors(const qb_fno *net);
/* C[b] ~ C[W[b]] for `batch` cells */
int qb_fno_forward(qb_fno *net, int batch, const double *W, double *C, void *stream);
/* loss = mean over all outputs of (y - target / scale)^2 (y: the unscaled
 * network output) and its gradient with respect to every weight (copied to
 * grad_host when non-NULL, same layout as qb_fno_get_params); synchronises */
int qb_fno_gradients(qb_fno *net, int batch, const double *W, const double *target, float *grad_host, double *loss, void *stream);
/* one Adam step (beta 0.9 / 0.999, eps 1e-8, bias-corrected) on that loss;
 * the loss is read back, so the call synchronises */
int qb_fno_train_step(qb_fno *net, int batch, const double *W, const double *target, float lr, double *loss, void *stream);

/* Strang step (the step of qb_inhom_step, periodic boundaries) whose
 * collision half uses the network with the exact operator as judge:
 *  - every `check_every`-th step (the first included) runs both collision
 *    steps on every cell, keeps the exact one, and marks for the following
 *    steps each cell whose collision increment from the network differs from
 *    the exact increment by more than `tol` (relative L1);
 *  - the other steps take the network's C (a midpoint step with the magnetic
 *    term and a network evaluation at the midpoint) for unmarked cells and
 *    the exact collision for marked ones.
 * The network's C is projected before use onto mass, momentum and energy
 * conservation of the trace component w0 (the least change |w0| (l0 + l1 v_x +
 * l2 v_y + l3 |v|^2), the same moments the exact operator conserves), so the
 * surrogate steps keep them to round-off.  tol = 0 gives the exact step.
 * The surrogate holds `net`, which must outlive it. */
typedef struct qb_surrogate qb_surrogate;
qb_surrogate *qb_surrogate_create(qb_fno *net, double tol, unsigned check_every);
void qb_surrogate_free(qb_surrogate *s);
int qb_surrogate_inhom_step(qb_surrogate *s, qb_workspace *ws, const qb_quad *q, int ncells, const double *W, double *Wnext,
                            double h, double dt, const double *Bext, void *stream);
/* cell-steps taken by the network and by the exact operator so far, and the
 * largest residual (relative increment difference) of the last check step */
int qb_surrogate_stats(const qb_surrogate *s, long *surrogate_cells, long *exact_cells, double *last_max_residual);

#ifdef __cplusplus
}
#endif

#endif /* QBGPU_H */

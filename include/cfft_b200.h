/*
 * libcfft_b200 — C ABI of the B200 (sm_100a) symmetry-reduced crystallographic FFT
 * (KRFFT) and SCFT pseudo-spectral diffusion step.
 *
 * The entry points replace the plan/execute surface of CrystallographicFFT.jl for
 * the hot path; each declaration names the reference function it stands in for
 * (file:line within the reference project).  A Julia caller binds them with
 * `ccall`.
 *
 * Conventions
 *  - Grids are column-major, x fastest (Julia Array layout == C [z][y][x]).
 *  - Real fields are float (precision 4) or double (precision 8); spectra are
 *    interleaved complex of the same precision, in spectral-ASU order (sorted
 *    lexicographically by (h1, h2, h3), as calc_spectral_asu returns them).
 *  - A batch of B fields is B contiguous fields (f0: B * M1*M2*M3 reals,
 *    spectra: B * n_spec complex).
 *  - Operations: R is row-major int32[9] (x'_i = sum_j R[3i+j] x_j + t_i), t is
 *    int32[3] in grid units; a 2-D problem passes dim = 2 and 4-entry R / 2-entry t
 *    packed into the 3-D slots with R33 = 1, t3 = 0 (N3 = 1).
 *  - Execute calls take device pointers owned by the caller and a cudaStream_t
 *    passed as void*; they are stream-ordered and never alias outputs.
 *  - Plans are not thread-safe (as in the reference); use one plan per stream.
 *  - Every call returns a cfft_status; cfft_last_error() gives a message.
 */
#ifndef CFFT_B200_H
#define CFFT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum cfft_status {
  CFFT_OK = 0,
  CFFT_ERR_INVALID = 1,          /* bad argument / size mismatch */
  CFFT_ERR_CUDA = 2,             /* CUDA runtime error (message in cfft_last_error) */
  CFFT_ERR_NOT_COMMENSURATE = 3, /* translation not commensurate with the grid */
  CFFT_ERR_UNSUPPORTED = 4,      /* size / group outside what the library handles */
  CFFT_ERR_TIMEOUT = 5,          /* a bounded device wait gave up */
  CFFT_ERR_ALLOC = 6,            /* device or host allocation failed */
  CFFT_ERR_NOT_REACHABLE = 7     /* a subgrid parity class has no operation */
} cfft_status;

typedef enum cfft_path {
  CFFT_PATH_AUTO = 0,     /* centred fold when applicable, else M2 (plan_krfft_centered) */
  CFFT_PATH_M2 = 1,       /* plain stride-L path: plan_krfft + plan_m2_backward */
  CFFT_PATH_CENTERED = 2, /* same as AUTO: plan_krfft_centered falls back to M2 itself */
  CFFT_PATH_M2Q = 3,      /* plan_m2_q (src/q_fused_krfft.jl:83): plain stride-L FFT; the SCFT
                             step applies the Q-matrix first row (d-tap gather) to the subgrid
                             spectrum instead of going through the spectral ASU */
  CFFT_PATH_M7 = 4,       /* plan_m7_scft (src/q_fused_krfft.jl:822): centring fold + channel FFTs
                             + Q-multiply + unfold; centred lattices only, like the reference */
  CFFT_PATH_FULLGRID = 5  /* full-grid plan, L = 1: the forward is the centring prefold of the whole
                             grid u into parity channels of (N/2)^3 + channel FFTs + merge onto the
                             spectral ASU (CenteringPreFoldPlan, _merge_channels!,
                             src/centering_prefold.jl:27-257); the backward returns the whole grid
                             with the symmetry fill (src/recursive_blocks_backward.jl:531-545).
                             Fields are N1 x N2 x N3 (M = N in cfft_info). */
} cfft_path;

typedef enum cfft_centering {
  CFFT_CENT_P = 0, CFFT_CENT_C = 1, CFFT_CENT_A = 2, CFFT_CENT_I = 3, CFFT_CENT_F = 4
} cfft_centering;

typedef struct cfft_desc {
  int dim;               /* 2 or 3 */
  int N[3];              /* full grid (N[2] ignored for dim = 2) */
  int n_ops;
  const int32_t* R;      /* n_ops * 9 */
  const int32_t* t;      /* n_ops * 3, shifted operations (find_optimal_shift) */
  double lattice[9];     /* lattice vectors in columns, column-major */
  double ds;             /* Δs of K(h) = exp(-Δs |2π A^-T h|^2) */
  int precision;         /* 4 (float) or 8 (double) */
  int max_batch;         /* largest batch any call will pass */
  int path;              /* cfft_path */
} cfft_desc;

typedef struct cfft_plan_s* cfft_plan;

typedef struct cfft_info {
  int N[3], L[3], M[3], H[3];
  int n_spec;            /* spectral-ASU size */
  int n_ops;             /* shifted operations held by the plan */
  int n_rep;             /* prod(L): representative operations (fiber length d) */
  int centering;         /* cfft_centering */
  int centered;          /* 1 if the centring fold is used */
  int n_channels;        /* alive parity channels (1 on the M2 path) */
  int n_orbits;          /* backward orbit representatives */
  int n_rem_ops;         /* even-translation operations used for orbit expansion */
  int precision;
  int max_batch;
  int P;                 /* lcm(N): phase denominator */
  int64_t workspace_bytes;
  int exec_path;         /* bit 0: compile-time sized kernels; bit 1: packed quad backward gather;
                            bit 2: fused 8-CTA cluster kernels; bit 3 / bit 4: persistent bulk-copy
                            (TMA) forward / backward plane kernels; bit 5: backward gather in
                            groups of 16 (FP32) / 8 (FP64) fields; bit 6: separable Q-multiply
                            (Pmmm-like M2Q plans) (0 for host-only plans) */
  int chunk;             /* fields per workspace chunk */
  int lanes;             /* concurrent chunk lanes */
} cfft_info;

/* ---------------- plan-time functions (host only, no GPU needed) ---------------- */

/* ---------------- legacy block path (plan_cfft, mul! / ldiv!) ----------------
 * plan_cfft (src/cfft_plan.jl:15-41) packs the real-space ASU (cfft_calc_asu + the
 * host-side pack_asu) into rectangular blocks and plans one FFT per block shape;
 * mul! / ldiv! (src/execution.jl:16-60, src/cfft_plan.jl:43-66) transform every block.
 * A block plan holds n_blocks block shapes dims[3 b + {0, 1, 2}] (unused dimensions 1);
 * `in` / `out` are device arrays of the blocks' complex data concatenated in plan order,
 * each block column-major.  Forward is unnormalised, backward divides by the block size,
 * as FFTW's plan * x and plan \ x.  `in` and `out` must not overlap. */
typedef struct cfft_block_plan_s* cfft_block_plan;
cfft_status cfft_block_plan_create(int n_blocks, const int32_t* dims, int precision, cfft_block_plan* plan);
cfft_status cfft_block_plan_destroy(cfft_block_plan plan);
cfft_status cfft_block_forward(cfft_block_plan plan, const void* in, void* out, void* stream);
cfft_status cfft_block_backward(cfft_block_plan plan, const void* in, void* out, void* stream);

/* build_recursive_tree + collect_leaves (src/fractal_krfft.jl:300-636): the recursive
 * parity tree that the fractal plans (plan_fractal_krfft, src/fractal_krfft.jl:678-723;
 * plan_fractal_krfft_v2/v3) are built on, from the operations (R row-major n_ops x 9,
 * t n_ops x 3, grid units).  leaves receives n_leaves x 10 int32 (grid size[3],
 * stride[3], offset[3] in the full grid, depth below the root) in collect_leaves
 * order, *n_inner the number of inner nodes; call with leaves = NULL to query
 * *n_leaves.  flags = 0 follows the
 * current source; bit 0 takes child translations from the half-grid-shifted
 * operations and bit 1 skips the centring split (the construction of the reference
 * version that wrote its tree survey, test/debug_tree_output.log). */
cfft_status cfft_fractal_tree(int dim, const int* N, int n_ops, const int32_t* R, const int32_t* t, int flags, int cap,
                              int* n_leaves, int* n_inner, int32_t* leaves);

/* calc_asu(N, ops) (src/asu.jl:216-324): real-space asymmetric unit by recursive parity
 * splitting of the grid under shifted operations.  n_points points sorted by grid index,
 * each with idx[3] (0-based grid coordinates), depth[3] (even splits per dimension) and
 * mult (orbit size within its leaf).  Call with idx = depth = mult = NULL to query
 * n_points. */
cfft_status cfft_calc_asu(int dim, const int* N, int n_ops, const int32_t* R, const int32_t* t, int cap,
                          int* n_points, int32_t* idx, int32_t* depth, int32_t* mult);

/* _build_q_matrices! (src/q_fused_krfft.jl:182-413) tables of an M2Q / M7 plan (also
 * host plans): Q first row Q[(b * Mvol + q) * 2 + {re, im}] and gather[b * Mvol + q]
 * (0-based column-major subgrid index of R_b^T q mod M), b < n_rep, q < M1 M2 M3.
 * Either pointer may be NULL.  CFFT_UNSUPPORTED for plans of the other paths. */
cfft_status cfft_plan_q_tables(cfft_plan plan, double* Q, int32_t* gather);

/* get_ops(sg, dim, N) (src/symmetry_ops.jl:51-53): operations of space group `sg`
 * (plane group for dim = 2) in ITA order, converted to grid units like convert_op
 * (src/symmetry_ops.jl:38-46).  Call with R = t = NULL to query *n_ops. */
cfft_status cfft_get_ops(int sg, int dim, const int* N, int cap, int* n_ops, int32_t* R, int32_t* t);

/* Space-group numbers the built-in table holds for `dim` (query with out = NULL). */
int cfft_list_groups(int dim, int* out, int cap);

/* find_optimal_shift(ops, N) (src/asu.jl:281-347): writes the fractional shift
 * (dim doubles) and the shifted translations (n_ops * 3). */
cfft_status cfft_find_optimal_shift(int dim, const int* N, int n_ops, const int32_t* R, const int32_t* t,
                                    double* shift, int32_t* t_shifted);

/* _count_special_positions_fast (src/asu.jl:372-438). */
int cfft_count_special_positions(int dim, const int* N, int n_ops, const int32_t* R, const int32_t* t);

/* auto_L(ops_shifted) (src/krfft.jl:225-279): writes L[3]. */
cfft_status cfft_auto_L(int dim, int n_ops, const int32_t* R, const int32_t* t, int* L);

/* detect_centering_type(ops, N) (src/symmetry_ops.jl:133-179): returns cfft_centering. */
int cfft_detect_centering(int dim, const int* N, int n_ops, const int32_t* R, const int32_t* t);

/* calc_spectral_asu(ops, dim, N) (src/spectral_indexing.jl:22-176): representatives
 * (n_spec * 3, 0-based) and multiplicities.  Query with idx = mult = NULL. */
cfft_status cfft_spectral_asu(int dim, const int* N, int n_ops, const int32_t* R, const int32_t* t, int cap,
                              int* n_spec, int32_t* idx, int32_t* mult);

/* ---------------- plans ---------------- */

/* plan_krfft_centered(spec, ops) / plan_krfft(spec, ops) + plan_m2_backward /
 * plan_centered_ikrfft / plan_centered_scft / plan_m2_scft
 * (src/centering_fold.jl:328,630,868; src/krfft.jl:301,1101; src/q_fused_krfft.jl:948):
 * one plan holds the forward, backward and diffusion-step state for a batch. */
cfft_status cfft_plan_create(const cfft_desc* desc, cfft_plan* plan);
/* Execution choices of one plan (no reference counterpart: the autotuner's knobs).
 * Zero / -1 fields keep the default (the environment switch of the same name, then the
 * built-in default measured best on Im-3m 128^3). */
typedef struct cfft_tuning {
  int64_t chunk_bytes;   /* channel workspace per chunk (CFFT_CHUNK_BYTES; 64 MiB) */
  int lanes;             /* concurrent chunk lanes 1..4 (CFFT_LANES; 2 for batches >= 8) */
  int zr_slots;          /* workspace slots per CTA of the fused z FFT + gather, 2 or 4 (CFFT_ZR_SLOTS; 4) */
  int wide;              /* backward gather in 128-byte field groups: 0, 1 (CFFT_WIDE; 1) */
  int tma;               /* bulk-copy plane kernels: 0, 1 forward, 2 backward, 3 both (CFFT_TMA; 0) */
  int cluster;           /* fused cluster kernels: 0, 8 or 16 CTAs (CFFT_CLUSTER; 0) */
} cfft_tuning;
/* cfft_plan_create with explicit execution choices (tuning may be NULL). */
cfft_status cfft_plan_create_tuned(const cfft_desc* desc, const cfft_tuning* tuning, cfft_plan* plan);
/* Same plan-time tables without any device state (no GPU needed); execute calls on
 * such a plan return CFFT_ERR_INVALID.  For table inspection and host tooling. */
cfft_status cfft_plan_create_host(const cfft_desc* desc, cfft_plan* plan);
cfft_status cfft_plan_destroy(cfft_plan plan);
cfft_status cfft_plan_info(cfft_plan plan, cfft_info* info);

/* Host copies of the plan's integer tables for bit-exact checks:
 * spectral ASU (n_spec*3 idx, n_spec mult), representative ops (n_rep*9, n_rep*3). */
cfft_status cfft_plan_spectral_asu(cfft_plan plan, int32_t* idx, int32_t* mult);
cfft_status cfft_plan_rep_ops(cfft_plan plan, int32_t* R, int32_t* t);
/* Backward orbit tables: orbit_rep (n_orbits), inv_spec and inv_phase (n_orbits * n_rep). */
cfft_status cfft_plan_backward_tables(cfft_plan plan, int32_t* orbit_rep, int32_t* inv_spec, int32_t* inv_phase);
/* K_spec (n_spec doubles) as plan_centered_scft computes it. */
cfft_status cfft_plan_kernel(cfft_plan plan, double* K);

/* update_kernel! / update_m2_kernel! (src/centering_fold.jl:939-953,
 * src/q_fused_krfft.jl:1036-1052): recompute K for a new Δs (lattice may be NULL
 * to keep the plan's). */
cfft_status cfft_update_kernel(cfft_plan plan, double ds, const double* lattice);

/* ---------------- execution (device pointers, stream-ordered) ---------------- */

/* fft_reconstruct_centered! / fft_reconstruct! (src/centering_fold.jl:421-431,
 * src/krfft.jl:554-562): f0 (B x M-grid real) -> F (B x n_spec complex). */
cfft_status cfft_forward(cfft_plan plan, const void* f0, void* F, int batch, void* stream);

/* ifft_unrecon_centered! / execute_m2_backward! (src/centering_fold.jl:745-775,
 * src/krfft.jl:1269-1277): F -> f0 (real part). */
cfft_status cfft_backward(cfft_plan plan, const void* F, void* f0, int batch, void* stream);

/* Batched forms over an array of plans (no reference counterpart: a caller of the
 * reference runs its plans one call each): plan i runs cfft_forward (cfft_backward) on
 * batch[i] fields from f0[i] into F[i] (F[i] into f0[i]), the plans in array order on
 * the one stream.  Each call is the single-plan call; the first failing plan stops the
 * loop, and its status is returned with "plan i: " before its message. */
cfft_status cfft_forward_plans(int n_plans, const cfft_plan* plans, const void* const* f0, void* const* F,
                               const int* batch, void* stream);
cfft_status cfft_backward_plans(int n_plans, const cfft_plan* plans, const void* const* F, void* const* f0,
                                const int* batch, void* stream);

/* execute_centered_scft! / execute_m2_scft! (src/centering_fold.jl:908-931,
 * src/q_fused_krfft.jl:989-1026): f0 <- IKRFFT(K . KRFFT(f0)), in place. */
cfft_status cfft_scft_step(cfft_plan plan, void* f0, int batch, void* stream);

/* step_diffusion! (src/diffusion_solver.jl:254-282) applied n_steps times:
 * q <- e^{-w dt/2} D(e^{-w dt/2} q), D = the plan's diffusion operator.  w has the
 * layout of q (B x M-grid). */
cfft_status cfft_step_diffusion(cfft_plan plan, void* q, const void* w, double dt, int n_steps, int batch,
                                void* stream);

/* fullgrid_to_subgrid! / subgrid_to_fullgrid! (src/q_fused_krfft.jl:681-719):
 * u (B x N-grid real) <-> f0 (B x M-grid real). */
cfft_status cfft_fullgrid_to_subgrid(cfft_plan plan, const void* u, void* f0, int batch, void* stream);
cfft_status cfft_subgrid_to_fullgrid(cfft_plan plan, const void* f0, void* u, int batch, void* stream);

/* Subgrid spectrum G0 = FFT_M(f0) of each field, [batch][M3][M2][M1] complex: the
 * F000 array returned by execute_staged! / execute_staged_full! (src/staged_krfft.jl:
 * 562-567,883-889) and the Y buffer of execute_m2_q! (src/q_fused_krfft.jl:553-576); on
 * the centred path the assembled G0 of fft_channels! + assemble_G0! (src/centering_fold.jl:
 * 264-296).  Compile-time sized channel grids only (CFFT_UNSUPPORTED otherwise). */
cfft_status cfft_subgrid_spectrum(cfft_plan plan, const void* f0, void* G0, int batch, void* stream);

/* Allocation-free forward.  No counterpart in the reference: it exists for callers
 * that cannot allocate device memory themselves or through this library -- for
 * example a process whose device memory is owned entirely by another allocator, or
 * code that must not enter the driver's allocator while it runs.  It computes what
 * cfft_forward computes, but its workspace, geometry and twiddle tables live in one
 * static device array of 32 MiB compiled into the library (every GPU that loads the
 * library holds it until the process exits), so a plan from cfft_plan_create_host is
 * enough; f0 and F are the caller's device buffers.  Any batch size is processed in
 * chunks that fit the array; a problem whose single field needs more scratch than
 * 32 MiB is rejected with CFFT_ERR_UNSUPPORTED.  The first call on each device (and
 * the first after the device's primary context was reset) looks up the array's
 * device address and sets kernel attributes, so make that first call before any
 * stream capture.  Geometry and tables reach the array as kernel parameters, with no
 * host staging buffer.  It never calls cudaMalloc or cudaFree.  All calls share
 * the one array: calls that overlap on the GPU (other streams, other host threads)
 * race and must be serialised by the caller. */
cfft_status cfft_forward_noalloc(cfft_plan plan, const void* f0, void* F, int batch, void* stream);

/* Host-buffer forms of the three execute calls (the reference's execute_*! take
 * host arrays): copy in, run, copy out on the plan's own stream, then synchronise. */
cfft_status cfft_forward_host(cfft_plan plan, const void* f0_host, void* F_host, int batch);
cfft_status cfft_backward_host(cfft_plan plan, const void* F_host, void* f0_host, int batch);
cfft_status cfft_scft_step_host(cfft_plan plan, void* f0_host, int batch);

/* Status of the plan's bounded device waits.  No reference counterpart: the
 * persistent bulk-copy kernels bound every wait on a copy (CFFT_WAIT_TIMEOUT_NS,
 * default one second); a wait that runs out records CFFT_ERR_TIMEOUT here, and every
 * later execute call on the plan returns CFFT_ERR_TIMEOUT until it is cleared.  Call
 * after synchronising the stream; clear != 0 resets the status. */
cfft_status cfft_plan_device_status(cfft_plan plan, int clear);
/* Self-test of that mechanism: launches one kernel on `stream` whose bounded wait
 * waits for bytes that never arrive, so after timeout_ns it records CFFT_ERR_TIMEOUT
 * in the plan's status and returns (the GPU context stays usable). */
cfft_status cfft_wait_selftest(cfft_plan plan, unsigned long long timeout_ns, void* stream);

/* ---------------- SCFT driver (AB diblock melt) ----------------
 * No reference counterpart: the reference stops at the contour step these entries run
 * on (step_diffusion!, src/diffusion_solver.jl:254-282; execute_m2_scft!,
 * src/q_fused_krfft.jl:989-1026).  The self-consistent field iteration of an
 * incompressible AB diblock melt (Gaussian chain, lengths in the plan's lattice units,
 * contour s in [0, 1], ds = 1/Ns; the plan's ds must equal 1/Ns and its max_batch be
 * at least 2): propagators q, q_dagger (one two-field batch of the plan's contour
 * step), Q = <q(r, 1)>, densities by Simpson's rule, residuals
 * d_A = chiN (phi_B - 1/2) + (w_B - w_A)/2, d_B = chiN (phi_A - 1/2) + (w_A - w_B)/2,
 * err = sqrt(sum d^2 / sum w^2), F = -ln Q + <(w_B - w_A)^2 / (4 chiN) - (w_A + w_B) / 2> + chiN / 4
 * (the field-theoretic Hamiltonian: equal to -ln Q + <chiN phi_A phi_B - w_A phi_A - w_B phi_B>
 * at the saddle point and stationary there, so its error is second order in the residual),
 * simple mixing for the first min_simple iterations and above anderson_start, Anderson
 * mixing after.  Q, F, the residual
 * norms, the Anderson Gram matrix and its least-squares solve are FP64 on the device.
 * Fields are [w_A | w_B] on the plan's M-grid (2 x M1 M2 M3 reals of the plan's
 * precision, device memory). */
typedef struct cfft_scft_params {
  double f;              /* A-block fraction, 0 < f < 1 */
  double chiN;           /* chi N */
  int Ns;                /* contour steps */
  int history;           /* Anderson history depth, 0..32 */
  double tol;            /* stop when err < tol */
  int max_iter;
  double lam_simple;     /* simple-mixing step (err > anderson_start) */
  double lam_anderson;   /* Anderson mixing step */
  double anderson_start; /* residual below which Anderson mixing runs */
  int min_simple;        /* simple-mixing iterations before Anderson mixing may start: from a
                            near-uniform start the ordered structure must first grow out of the
                            unstable modes, or Anderson mixing converges to the disordered state */
} cfft_scft_params;
typedef struct cfft_scft_state {
  double Q, F, err;
  int iterations;
  int converged;
} cfft_scft_state;
typedef struct cfft_scft_s* cfft_scft;
cfft_status cfft_scft_create(cfft_plan plan, const cfft_scft_params* params, cfft_scft* scft);
cfft_status cfft_scft_destroy(cfft_scft scft);
/* One evaluation of fields w: Q, F, err into *state; densities [phi_A | phi_B] into phi
 * and residuals [d_A | d_B] into d when not NULL.  Synchronises the stream. */
cfft_status cfft_scft_evaluate(cfft_scft scft, const void* w, void* phi, void* d, cfft_scft_state* state,
                               void* stream);
/* Iterate from w (in/out) until err < tol or max_iter; *state holds the last
 * evaluation.  One stream synchronisation per iteration (the convergence test). */
cfft_status cfft_scft_solve(cfft_scft scft, void* w, cfft_scft_state* state, void* stream);
/* Densities [phi_A | phi_B] of the last evaluation (device copy on `stream`). */
cfft_status cfft_scft_densities(cfft_scft scft, void* phi, void* stream);

/* ---------------- learned warm start (spectral neural operator) ----------------
 * No reference counterpart: a network that predicts SCFT fields [w_A | w_B] of an AB
 * diblock melt from (chiN, f) and the space group (one-hot slot 0 Im-3m, 1 Ia-3d,
 * 2 Pm-3m), trained on converged fields of the SCFT driver above, used as its starting
 * point.  Lift of 21 input channels (chiN, f, the group one-hot and the symmetrised
 * plane waves of 8 reflections) to 32 channels, 4 Fourier layers (a 1 x 1 channel map
 * plus a spectral convolution with one real 32 x 32 matrix per mode class, 12 retained
 * modes per axis, gelu), a 32 -> 64 -> 2 projection.  The spectral convolution runs on
 * the plan's own KRFFT (the 32 channels of every sample as one batch); the channel maps
 * run on the tensor cores with BF16 weights and FP32 accumulation.  Fields live on the
 * plan's M-grid: FP32 plans of a cubic group on a cubic grid with M1 M2 M3 a multiple of
 * 128, max_batch >= 32 * max_samples, max_samples <= 32.  A model's weights are shared
 * by all its bound contexts (one per plan), so one model trains on several groups and
 * grids; parameters are cfft_sno_param_count() floats in the library's fixed order. */
typedef struct cfft_sno_config {
  double lr, beta1, beta2, eps, weight_decay; /* Adam (decoupled weight decay) */
} cfft_sno_config;
typedef struct cfft_sno_s* cfft_sno;
typedef struct cfft_sno_ctx_s* cfft_sno_ctx;
int64_t cfft_sno_param_count(void);
/* A model with seeded initial weights (cfg may be NULL for the defaults 1e-3, 0.9,
 * 0.999, 1e-8, 0). */
cfft_status cfft_sno_create(const cfft_sno_config* cfg, cfft_sno* model);
cfft_status cfft_sno_destroy(cfft_sno model);
cfft_status cfft_sno_set_params(cfft_sno model, const float* host);
cfft_status cfft_sno_get_params(cfft_sno model, float* host);
/* Gradients of the last cfft_sno_train call (host copy, parameter order). */
cfft_status cfft_sno_get_grads(cfft_sno model, float* host);
/* Data-parallel training over several GPUs (one process per GPU): each rank calls
 * cfft_sno_train with step = 0 on its own samples, copies the gradients into a device
 * buffer of cfft_sno_param_count() floats with cfft_sno_grads_device, averages that
 * buffer over the ranks (an NCCL all-reduce), and then applies one Adam step from it
 * with cfft_sno_apply_grads (grads = NULL uses the model's own gradient buffer).
 * cfft_sno_train with step != 0 equals cfft_sno_train with step = 0 followed by
 * cfft_sno_apply_grads(model, NULL, lr).  cfft_sno_apply_grads synchronises the stream. */
cfft_status cfft_sno_grads_device(cfft_sno model, void* dst, void* stream);
cfft_status cfft_sno_apply_grads(cfft_sno model, const void* grads, double lr, void* stream);
/* Binds the model to a plan: shift is the fractional origin shift of the plan's
 * operations (find_optimal_shift), so the input features are the same functions of
 * position on every grid. */
cfft_status cfft_sno_bind(cfft_sno model, cfft_plan plan, int group_slot, const double* shift, int max_samples,
                          cfft_sno_ctx* ctx);
cfft_status cfft_sno_unbind(cfft_sno_ctx ctx);
/* params = n_samples pairs (chiN, f) on the host; w_out = n_samples x [w_A | w_B]
 * (n_samples x 2 x M-grid floats, device).  Synchronises the stream. */
cfft_status cfft_sno_predict(cfft_sno_ctx ctx, const double* params, int n_samples, void* w_out, void* stream);
/* Loss (mean square of (w - w_target) / chiN over samples, both fields and grid
 * points) and gradients for targets w_target (device, the layout of w_out); step != 0
 * then applies one Adam step with learning rate lr.  Synchronises the stream. */
cfft_status cfft_sno_train(cfft_sno_ctx ctx, const double* params, int n_samples, const void* w_target, double lr,
                           int step, double* loss, void* stream);

/* ---------------- diagnostics ---------------- */
/* Forward then backward of one batch with a CUDA event between every launch;
 * stage_ms receives up to 8 per-stage device times (plane/fold+xy FFT, z FFT,
 * reconstruct, inverse reconstruct, inverse z FFT, inverse xy FFT + unfold) and
 * *n_stages their number.  Synchronises the stream.  No reference counterpart:
 * it backs the per-kernel timing of the benchmark. */
cfft_status cfft_profile_roundtrip(cfft_plan plan, const void* f0, void* F, void* f0_out, int batch, void* stream,
                                   float* stage_ms, int* n_stages);
const char* cfft_status_string(cfft_status s);
const char* cfft_last_error(void);
int cfft_version(void);
/* Number of kernel launches this library issued on this thread since the last reset. */
int64_t cfft_launch_count(int reset);

#ifdef __cplusplus
}
#endif

#endif /* CFFT_B200_H */

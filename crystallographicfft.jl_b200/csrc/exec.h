// Device-side plan object and execution entry points of libcfft_b200.
#pragma once

#include <string>

#include "cfft_internal.h"

namespace cfft {

// Per-plan execution choices (cfft_plan_create_tuned); unset fields (0 / -1) fall back
// to the process defaults (environment switches, then built-in defaults).
struct Tuning {
  int64_t chunk_bytes = 0;  // channel workspace per chunk
  int lanes = 0;            // concurrent chunk lanes
  int zr_slots = 0;         // slots per CTA of the fused z FFT + gather (2 or 4)
  int wide = -1;            // backward gather in 128-byte field groups
  int tma = -1;             // bulk-copy plane kernels: bit 0 forward, bit 1 backward
  int cluster = -1;         // fused cluster kernels: 0, 8 or 16 CTAs
};

struct Plan {
  PlanTables T;
  Tuning tune;
  int precision = 4;   // 4 = float, 8 = double
  int max_batch = 1;
  double lattice[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  double ds = 0.0;
  int n_mask_words = 1;
  std::vector<int32_t> fill_map;  // N-grid -> M-grid linear index (built on first use)
  // device buffers (owned)
  void* d_geom = nullptr;       // DevGeom
  void* d_tables = nullptr;     // twiddles / phases (complex T)
  void* d_spec_h = nullptr;     // packed h per spectral point
  void* d_K = nullptr;          // K per spectral point (T)
  void* d_orbit_rep = nullptr;
  void* d_inv_spec = nullptr;
  void* d_inv_phase = nullptr;
  void* d_img_mask = nullptr;   // distinct-image masks per orbit representative
  void* d_fill_map = nullptr;
  void* d_work_T = nullptr;     // B x n_ch x H-grid complex
  void* d_work_F = nullptr;     // B x n_spec complex
  void* d_work_E = nullptr;     // B x M-grid real (interaction factors)
  void* d_stage_in = nullptr;   // host-API staging
  void* d_stage_out = nullptr;
  void* d_expand = nullptr;     // fast path: per channel position (orbit index, phase numerator)
  void* d_g0r = nullptr;        // fast path: G0 at orbit representatives (per lane)
  void* d_ft = nullptr;         // packed backward path: spectra regrouped in quads of fields (per lane)
  void* d_inv_pk = nullptr;     // fast path: packed alias table for the shared-memory gather
  void* d_zr_units = nullptr;   // fused z FFT + gather: uint4 per unit (c | ya | yb, first point, count)
  void* d_zr_pts = nullptr;     // fused z FFT + gather: spectral indices grouped by unit
  void* own_stream = nullptr;
  static constexpr int kMaxLanes = 4;
  void* lane_stream[kMaxLanes] = {};  // concurrent chunk lanes (fork/join on the caller's stream)
  void* ev_fork = nullptr;
  void* ev_join[kMaxLanes] = {};
  // host-buffer entry points: pieces of the batch flow H2D (h2d_stream) -> compute
  // (own_stream) -> D2H (d2h_stream), so the copies of neighbouring pieces overlap.
  static constexpr int kHostPieces = 8;
  void* h2d_stream = nullptr;
  void* d2h_stream = nullptr;
  void* ev_in[kHostPieces] = {};
  void* ev_done[kHostPieces] = {};
  size_t w_lane_bytes = 0, g0r_lane_bytes = 0, ft_lane_bytes = 0;
  size_t workspace_bytes = 0;
  // launch geometry
  int threads_xy = 0, threads_z = 0;
  int fast_h = 0;               // cubic channel edge of the compile-time sized kernels (0 = generic)
  int chunk = 1;                // fields per workspace chunk
  int lanes = 1;                // concurrent chunk lanes
  int cent_type = 0;            // plane-kernel centring (0 plain, 1 I, 2 F, 3 C, 4 A)
  bool rep_perm = false;        // representative ops are signed permutations
  bool rep_diag8 = false;       // representative ops are the 8 diagonal sign matrices
  bool reps_quad = false;       // packed alias rows; fields gathered and expanded in quads
  bool reps_wide = false;       // the same in groups of 128 / sizeof(complex) fields (one line per point)
  bool zrecon = false;          // forward z FFT fused with the diagonal-sign gather (stage 6)
  int zr_units = 0;             // units of the fused kernel (channel + mirrored row pair)
  bool cluster = false;         // fused cluster kernels: fold+xyz FFT and expand+xyz IFFT+unfold
  // Q-matrix diffusion step (M2Q: plain path, M7: centred path): host tables and their
  // channel-point ordered device copies, plus a second channel workspace per lane.
  // Contour-loop graphs of cfft_step_diffusion: the n_steps forward + K + backward
  // steps on a fixed field buffer, captured once and replayed (a cudaGraphExec_t each).
  struct StepGraph {
    void* q;
    int batch, n_steps;
    void* exec;
    int64_t kernels;   // kernel launches one replay stands for
    uint64_t last_use;
  };
  std::vector<StepGraph> step_graphs;
  uint64_t graph_clock = 0;
  int qmode = 0;                // 0 none, 3 M2Q, 4 M7 (the cfft_path value)
  std::vector<double> q_host;   // d x Mvol complex (re, im)
  std::vector<int32_t> q_gather;  // d x Mvol
  void* d_qt = nullptr;         // d x n_ch x H^3 complex coefficients
  void* d_gt = nullptr;         // d x n_ch x H^3 int32 workspace index (-1: extinct class)
  void* d_work_Q = nullptr;     // lanes x channel workspace (Q-multiply output)
  bool qsep = false;            // separable Q-multiply (Pmmm-like M2Q plans, CFFT_QSEP=0 turns it off)
  void* d_qsep = nullptr;       // its 1-D twiddles (3 x H) and kernel factors (3 x 2H), complex
  int cluster_ctas = 8;         // CTAs per cluster
  // Status word of the bounded device waits (mapped pinned host memory, so the host
  // reads it without a synchronisation): 0, or CFFT_ERR_TIMEOUT once a wait ran out.
  int* h_status = nullptr;
  int* d_status = nullptr;
  unsigned long long timeout_ns = 1000000000ull;  // limit of one device wait (CFFT_WAIT_TIMEOUT_NS)
  size_t smem_xy = 0, smem_z = 0;
};

Status plan_device_init(Plan* p, std::string* err);
void plan_device_free(Plan* p);
Status plan_upload_kernel(Plan* p, std::string* err);

Status exec_forward(Plan* p, const void* f0, void* F, int B, void* stream, std::string* err);
Status exec_backward(Plan* p, const void* F, void* f0, int B, void* stream, std::string* err);
Status exec_scft_step(Plan* p, void* f0, int B, void* stream, std::string* err);
Status exec_step_diffusion(Plan* p, void* q, const void* w, double dt, int n_steps, int B, void* stream,
                           std::string* err);
Status exec_full_to_sub(Plan* p, const void* u, void* f0, int B, void* stream, std::string* err);
Status exec_sub_to_full(Plan* p, const void* f0, void* u, int B, void* stream, std::string* err);
// Legacy block plan (plan_cfft): per-block DFTs of the packed real-space ASU.
constexpr int kBlockLineElems = 1024;  // elements of the lines one CTA of the block transform stages
constexpr int kBlockMaxLen = 4096;     // longest block edge
constexpr int kBlockSmemMax = (2 * kBlockMaxLen + kBlockMaxLen) * 16;
struct BlockPlan {
  int n_blocks = 0;
  long long total = 0;  // elements over all blocks
  int precision = 8;
  void* d_dims = nullptr;
  void* d_off = nullptr;
  void* d_work = nullptr;
  void* d_items = nullptr;  // per axis: int4 (block, first line, lines, 0) work items
  int item_off[3] = {0, 0, 0}, n_items[3] = {0, 0, 0}, max_len[3] = {0, 0, 0};
};
Status block_plan_create(int n_blocks, const int32_t* dims, int precision, BlockPlan** out, std::string* err);
void block_plan_destroy(BlockPlan* bp);
Status block_execute(BlockPlan* bp, const void* in, void* out, bool inverse, void* stream, std::string* err);
Status exec_subgrid_spectrum(Plan* p, const void* f0, void* G0, int B, void* stream, std::string* err);
Status exec_host(Plan* p, int which, const void* in, void* out, int B, std::string* err);
Status exec_profile_roundtrip(Plan* p, const void* f0, void* F, void* f0_out, int B, void* stream, float* ms,
                              int* n, std::string* err);

Status exec_forward_noalloc(const Plan* p, const void* f0, void* F, int B, void* stream, std::string* err);
// Status of the plan's bounded device waits (after the caller synchronised): kOk or
// kTimeout; `clear` resets it.
Status plan_device_status(Plan* p, bool clear, std::string* err);
// Bounded-wait self-test on the plan's status word (see k_wait_selftest).
Status plan_wait_selftest(Plan* p, unsigned long long timeout_ns, void* stream, std::string* err);

int64_t launch_count(bool reset);
// Adds n to the launch counter (kernels launched outside exec.cu).
void add_launches(int64_t n);

// One contour step of a batch with per-field interaction factors E (B x M-grid):
// out = E . IKRFFT(K . KRFFT(E . in)), in and out distinct buffers of B fields.
Status exec_contour_step(Plan* p, const void* in, void* out, const void* E, int B, void* stream, std::string* err);

}  // namespace cfft

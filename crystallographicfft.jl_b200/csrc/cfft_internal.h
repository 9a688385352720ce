// Internal declarations shared by the host plan layer (C++) and the device
// execution layer (CUDA) of libcfft_b200.
#pragma once

#include <array>
#include <complex>
#include <cstdint>
#include <string>
#include <vector>

namespace cfft {

enum class Status : int {
  kOk = 0,
  kInvalid = 1,
  kCuda = 2,
  kNotCommensurate = 3,
  kUnsupported = 4,
  kTimeout = 5,
  kAlloc = 6,
  kNotReachable = 7,
};

// Seitz operation in grid units: x' = R x + t (mod N).  Always stored 3-D; a 2-D
// problem is embedded with N3 = 1, R33 = 1 and t3 = 0.
struct SymOp {
  int R[3][3];
  int t[3];
};

enum Centering : int { kCentP = 0, kCentC = 1, kCentA = 2, kCentI = 3, kCentF = 4 };

struct SpecPoint {
  int h[3];  // 0-based frequency indices in [0, N)
  int mult;  // orbit size under the dual point group
};

// ---- space-group table (spacegroups.cpp) ----
bool has_group(int sg, int dim);
int list_groups(int dim, int* out, int cap);
Status get_ops(int sg, int dim, const int* N, std::vector<SymOp>* out, std::string* err);

// ---- plan-time geometry (planner.cpp) ----
long floor_mod(long a, long n);
bool check_shift_invariance(const std::vector<SymOp>& ops, const double* shift, const int* N, int dim,
                            std::vector<std::array<int, 3>>* deltas);
int count_special_positions_fast(const int* N, int dim, const std::vector<SymOp>& ops);
void find_optimal_shift(const std::vector<SymOp>& ops, const int* N, int dim, double* shift_out,
                        std::vector<SymOp>* shifted);
std::vector<SymOp> dual_ops(const std::vector<SymOp>& ops);
std::vector<SpecPoint> calc_spectral_asu(const std::vector<SymOp>& ops, const int* N, int dim);
std::array<int, 3> auto_L(const std::vector<SymOp>& ops, int dim);
Status select_rep_ops(const std::vector<SymOp>& ops, const std::array<int, 3>& L, const int* N,
                      std::vector<SymOp>* rep, std::string* err);
Centering detect_centering_type(const std::vector<SymOp>& ops, const int* N, int dim);
int alive_offsets(Centering c, std::array<int, 3>* offsets);  // returns n_channels (0 for P)
void get_k_vector(const SpecPoint& p, const int* N, int* k);

// Backward-transform lookup: every full-grid frequency h that is equivalent to a
// spectral-ASU point s under the group (or its Hermitian image) maps to
// (s, phase numerator j, conj): F(h) = e^{2 pi i j / P} * F(s) (or conj(F(s))),
// P = lcm(N).  Mirrors _build_spectral_reverse_lookup (src/krfft.jl:1183-1255).
struct ReverseEntry {
  int32_t spec;  // 1-based; 0 = frequency outside every ASU orbit (extinct)
  int32_t phase;  // numerator over P
  bool conj;
};

struct PlanTables {
  int dim = 3;
  int N[3] = {1, 1, 1};
  int L[3] = {1, 1, 1};
  int M[3] = {1, 1, 1};
  int P = 1;  // lcm(N1,N2,N3): phase denominator for recon weights
  int d = 1;  // prod(L)
  Centering centering = kCentP;
  bool centered = false;  // true: centering fold path (n_ch channels of H)
  int n_ch = 1;
  int H[3] = {1, 1, 1};  // channel grid (= M on the plain path)
  std::array<int, 3> offsets[8];
  int chan_of_parity[8];  // parity class (p0 + 2 p1 + 4 p2) -> channel or -1
  std::vector<SymOp> ops;      // shifted operations (all)
  std::vector<SymOp> rep_ops;  // one per parity class, canonical order
  std::vector<SpecPoint> spec;
  // Backward: orbit representatives of the channel grid under the even-translation
  // subgroup; per representative d entries (spec index signed for conjugation,
  // phase numerator over P) with the 1/d weight applied in the kernel.
  std::vector<SymOp> rem_ops;        // (R, s = t/2) acting on the M-grid
  std::vector<int32_t> orbit_rep;    // linear M-grid index of each representative
  std::vector<int32_t> inv_spec;     // n_orbits * d
  std::vector<int32_t> inv_phase;    // n_orbits * d
  std::vector<double> K;             // diffusion kernel per spectral point
};

Status build_tables(const std::vector<SymOp>& shifted_ops, const int* N, int dim, bool want_centered,
                    PlanTables* T, std::string* err, bool full_grid = false);
void compute_kernel(const PlanTables& T, const double* lattice, double ds, std::vector<double>* K);
struct AsuPoint {
  int idx[3];    // grid coordinates (0-based)
  int depth[3];  // even-split count per dimension
  int mult;      // orbit size at the leaf
};
std::vector<AsuPoint> calc_asu(const std::vector<SymOp>& ops, const int* N, int dim);
Status build_q_tables(const PlanTables& T, const double* lattice, double ds, std::vector<double>* Q,
                      std::vector<int32_t>* gather, std::string* err);

}  // namespace cfft

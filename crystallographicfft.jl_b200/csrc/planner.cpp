// Host plan layer: magic shift, spectral ASU, stride-L selection, representative
// operations, centering detection, backward orbit tables and the diffusion kernel.
// Each routine follows the reference algorithm cited beside it so that every
// integer table (spectral-ASU points, multiplicities, L, M, fold offsets) is
// identical to the reference's.
#include <algorithm>
#include <array>
#include <atomic>
#include <climits>
#include <cmath>
#include <complex>
#include <numeric>
#include <set>
#include <thread>
#include <unordered_map>

#include "cfft_internal.h"
#include "fractal_tree.h"

namespace cfft {

long floor_mod(long a, long n) {
  long r = a % n;
  return r < 0 ? r + n : r;
}

static bool is_identity_R(const SymOp& op) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      if (op.R[i][j] != (i == j ? 1 : 0)) return false;
  return true;
}

// check_shift_invariance (src/symmetry_ops.jl:81-94): delta = (R s - s) .* N must be integral.
bool check_shift_invariance(const std::vector<SymOp>& ops, const double* shift, const int* N, int dim,
                            std::vector<std::array<int, 3>>* deltas) {
  deltas->assign(ops.size(), {0, 0, 0});
  for (size_t k = 0; k < ops.size(); ++k) {
    for (int i = 0; i < dim; ++i) {
      double rs = 0.0;
      for (int j = 0; j < dim; ++j) rs += ops[k].R[i][j] * shift[j];
      const double df = (rs - shift[i]) * N[i];
      const double di = std::nearbyint(df);
      if (std::fabs(df - di) > 1e-5) return false;
      (*deltas)[k][i] = static_cast<int>(di);
    }
  }
  return true;
}

// True when the affine operations x -> R x + t (mod n, first dim axes) contain the
// identity and are closed under composition.  The orbit of x is then exactly
// {R x + t}, and one pass of the operations over x replaces the closure walk that
// applies every operation to every orbit member.  Matrices are compared entry by
// entry and translations mod n, so a list that is closed only as maps on the grid
// counts as open and keeps the walk (same result, more work).
static bool affine_ops_form_group(const std::vector<SymOp>& ops, const int* n, int dim) {
  auto same = [&](const int (&R)[3][3], const long* t, const SymOp& o) {
    for (int i = 0; i < dim; ++i) {
      if (floor_mod(t[i] - o.t[i], n[i]) != 0) return false;
      for (int j = 0; j < dim; ++j)
        if (R[i][j] != o.R[i][j]) return false;
    }
    return true;
  };
  int I[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  const long zero[3] = {0, 0, 0};
  bool has_id = false;
  for (const auto& o : ops) has_id = has_id || same(I, zero, o);
  if (!has_id) return false;
  for (const auto& a : ops)
    for (const auto& b : ops) {
      int R[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      long t[3] = {0, 0, 0};
      for (int i = 0; i < dim; ++i) {
        t[i] = a.t[i];
        for (int k = 0; k < dim; ++k) t[i] += static_cast<long>(a.R[i][k]) * b.t[k];
        for (int j = 0; j < dim; ++j)
          for (int k = 0; k < dim; ++k) R[i][j] += a.R[i][k] * b.R[k][j];
      }
      bool found = false;
      for (const auto& c : ops)
        if (same(R, t, c)) { found = true; break; }
      if (!found) return false;
    }
  return true;
}

// _count_special_positions_fast (src/asu.jl:372-438): number of orbits shorter than |ops|.
int count_special_positions_fast(const int* N, int dim, const std::vector<SymOp>& ops) {
  const int n1 = N[0], n2 = dim > 1 ? N[1] : 1, n3 = dim > 2 ? N[2] : 1;
  const long total = static_cast<long>(n1) * n2 * n3;
  std::vector<char> visited(total, 0);
  std::vector<long> orbit;
  int sp = 0;
  const int n[3] = {n1, n2, n3};
  const bool closed = affine_ops_form_group(ops, n, dim);
  for (long lin = 0; lin < total; ++lin) {
    if (visited[lin]) continue;
    orbit.clear();
    orbit.push_back(lin);
    visited[lin] = 1;
    if (closed) {  // the orbit is {g x}: one pass of the operations
      long rem = lin;
      int x[3];
      x[0] = rem % n1; rem /= n1; x[1] = rem % n2; x[2] = rem / n2;
      long size = 1;
      for (const auto& op : ops) {
        long li = 0, stride = 1;
        for (int d = 0; d < 3; ++d) {
          long s = (d < dim) ? op.t[d] : 0;
          for (int j = 0; j < 3; ++j) s += op.R[d][j] * x[j];
          li += floor_mod(s, n[d]) * stride;
          stride *= n[d];
        }
        if (!visited[li]) { visited[li] = 1; ++size; }
      }
      if (size < static_cast<long>(ops.size())) ++sp;
      continue;
    }
    for (size_t w = 0; w < orbit.size(); ++w) {
      long rem = orbit[w];
      int x[3];
      x[0] = rem % n1; rem /= n1; x[1] = rem % n2; x[2] = rem / n2;
      for (const auto& op : ops) {
        long li = 0, stride = 1;
        for (int d = 0; d < 3; ++d) {
          long s = (d < dim) ? op.t[d] : 0;
          for (int j = 0; j < 3; ++j) s += op.R[d][j] * x[j];
          li += floor_mod(s, n[d]) * stride;
          stride *= n[d];
        }
        if (!visited[li]) { visited[li] = 1; orbit.push_back(li); }
      }
    }
    if (static_cast<long>(orbit.size()) < static_cast<long>(ops.size())) ++sp;
  }
  return sp;
}

static int odd_dims_product(const std::vector<SymOp>& ops, int dim) {
  int p = 1;
  for (int d = 0; d < dim; ++d) {
    bool any = false;
    for (const auto& op : ops)
      if (floor_mod(op.t[d], 2) == 1) { any = true; break; }
    p *= any ? 2 : 1;
  }
  return p;
}

// find_optimal_shift (src/asu.jl:281-347).
void find_optimal_shift(const std::vector<SymOp>& ops, const int* N, int dim, double* shift_out,
                        std::vector<SymOp>* shifted) {
  int Np[3] = {1, 1, 1};
  for (int d = 0; d < dim; ++d) Np[d] = 12;
  // _rescale_ops (src/asu.jl:355-363): t_new = t * 12 ÷ N (truncating division)
  std::vector<SymOp> proxy = ops;
  for (auto& op : proxy)
    for (int d = 0; d < dim; ++d) op.t[d] = static_cast<int>((static_cast<long>(op.t[d]) * Np[d]) / N[d]);
  const double fracs[4] = {0.0, 0.5, 1.0 / 3.0, 0.25};
  double best_frac = 0.0;
  int min_sp = INT32_MAX;
  std::vector<std::array<int, 3>> deltas;
  for (double frac : fracs) {
    double s[3] = {0, 0, 0};
    for (int d = 0; d < dim; ++d) s[d] = frac / Np[d];
    if (!check_shift_invariance(proxy, s, Np, dim, &deltas)) continue;
    std::vector<SymOp> cur = proxy;
    for (size_t k = 0; k < cur.size(); ++k)
      for (int d = 0; d < dim; ++d) cur[k].t[d] += deltas[k][d];
    const int sp = count_special_positions_fast(Np, dim, cur);
    if (sp < min_sp) { min_sp = sp; best_frac = frac; }
    if (min_sp == 0) break;
  }
  double shift[3] = {0, 0, 0};
  for (int d = 0; d < dim; ++d) shift[d] = best_frac / N[d];
  std::vector<SymOp> best = ops;
  if (check_shift_invariance(ops, shift, N, dim, &deltas)) {
    for (size_t k = 0; k < best.size(); ++k)
      for (int d = 0; d < dim; ++d) best[k].t[d] += deltas[k][d];
  } else {
    for (int d = 0; d < dim; ++d) shift[d] = 0.0;
  }
  // Half-grid shift when it raises the number of dimensions with odd translations.
  double half[3] = {0, 0, 0};
  for (int d = 0; d < dim; ++d) half[d] = 0.5 / N[d];
  if (check_shift_invariance(ops, half, N, dim, &deltas)) {
    std::vector<SymOp> oh = ops;
    for (size_t k = 0; k < oh.size(); ++k)
      for (int d = 0; d < dim; ++d) oh[k].t[d] += deltas[k][d];
    if (odd_dims_product(oh, dim) > odd_dims_product(best, dim)) {
      for (int d = 0; d < dim; ++d) shift[d] = half[d];
      best = oh;
    }
  }
  for (int d = 0; d < 3; ++d) shift_out[d] = d < dim ? shift[d] : 0.0;
  *shifted = best;
}

// Integer inverse of a unimodular 3x3 matrix.
static void int_inverse(const int R[3][3], int out[3][3]) {
  const long det = static_cast<long>(R[0][0]) * (R[1][1] * R[2][2] - R[1][2] * R[2][1]) -
                   static_cast<long>(R[0][1]) * (R[1][0] * R[2][2] - R[1][2] * R[2][0]) +
                   static_cast<long>(R[0][2]) * (R[1][0] * R[2][1] - R[1][1] * R[2][0]);
  int adj[3][3];
  adj[0][0] = R[1][1] * R[2][2] - R[1][2] * R[2][1];
  adj[0][1] = R[0][2] * R[2][1] - R[0][1] * R[2][2];
  adj[0][2] = R[0][1] * R[1][2] - R[0][2] * R[1][1];
  adj[1][0] = R[1][2] * R[2][0] - R[1][0] * R[2][2];
  adj[1][1] = R[0][0] * R[2][2] - R[0][2] * R[2][0];
  adj[1][2] = R[0][2] * R[1][0] - R[0][0] * R[1][2];
  adj[2][0] = R[1][0] * R[2][1] - R[1][1] * R[2][0];
  adj[2][1] = R[0][1] * R[2][0] - R[0][0] * R[2][1];
  adj[2][2] = R[0][0] * R[1][1] - R[0][1] * R[1][0];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) out[i][j] = static_cast<int>(adj[i][j] / det);
}

// dual_ops (src/symmetry_ops.jl:103-112): R* = (R^-1)^T, t = 0.
std::vector<SymOp> dual_ops(const std::vector<SymOp>& ops) {
  std::vector<SymOp> out(ops.size());
  for (size_t k = 0; k < ops.size(); ++k) {
    int inv[3][3];
    int_inverse(ops[k].R, inv);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) out[k].R[i][j] = inv[j][i];
    out[k].t[0] = out[k].t[1] = out[k].t[2] = 0;
  }
  return out;
}

// The distinct rotation parts of a list of operations (centring copies share one R).
static std::vector<SymOp> distinct_rotations(const std::vector<SymOp>& ops) {
  std::vector<SymOp> out;
  for (const auto& op : ops) {
    bool dup = false;
    for (const auto& o : out) {
      bool same = true;
      for (int i = 0; i < 3 && same; ++i)
        for (int j = 0; j < 3 && same; ++j) same = o.R[i][j] == op.R[i][j];
      if (same) { dup = true; break; }
    }
    if (!dup) out.push_back(op);
  }
  return out;
}

// True when the rotations contain the identity and are closed under multiplication
// (a point group).  Then the orbit of k is exactly {R k}, with no closure walk.
static bool rotations_form_group(const std::vector<SymOp>& rots) {
  bool has_id = false;
  for (const auto& r : rots) has_id = has_id || is_identity_R(r);
  if (!has_id) return false;
  for (const auto& a : rots)
    for (const auto& b : rots) {
      int p[3][3];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          p[i][j] = 0;
          for (int k = 0; k < 3; ++k) p[i][j] += a.R[i][k] * b.R[k][j];
        }
      bool found = false;
      for (const auto& c : rots) {
        bool same = true;
        for (int i = 0; i < 3 && same; ++i)
          for (int j = 0; j < 3 && same; ++j) same = c.R[i][j] == p[i][j];
        if (same) { found = true; break; }
      }
      if (!found) return false;
    }
  return true;
}

// Stabiliser-phase extinction filter of calc_spectral_asu (src/spectral_indexing.jl:143-171):
// a representative kr is kept when |sum over g with R_g kr = kr (mod N) of
// exp(-2 pi i kr.t_g / N)| > 1e-5.
static bool spectral_alive(const std::vector<SymOp>& ops, const std::vector<SymOp>& rec, const int* kr, const int* n,
                           int dim) {
  double sr = 0.0, si = 0.0;
  for (size_t g = 0; g < rec.size(); ++g) {
    bool stab = true;
    for (int d = 0; d < 3 && stab; ++d) {
      long s = 0;
      for (int j = 0; j < 3; ++j) s += rec[g].R[d][j] * kr[j];
      if ((s - kr[d]) % n[d] != 0) stab = false;
    }
    if (!stab) continue;
    double phase = 0.0;
    for (int d = 0; d < dim; ++d) phase += static_cast<double>(kr[d]) * ops[g].t[d] / n[d];
    sr += std::cos(2.0 * M_PI * phase);
    si -= std::sin(2.0 * M_PI * phase);
  }
  return std::hypot(sr, si) > 1e-5;
}

// Representatives of a closed point group without a visited array: k (column-major
// index lin) is the smallest member of its orbit {R k} exactly when no rotation maps it
// to a smaller index, which most points fail after one or two rotations.  The test is
// arithmetic only, so it runs on host threads over ranges of lin; the orbit size (the
// number of distinct images) and the extinction filter are evaluated at representatives.
static std::vector<SpecPoint> spectral_asu_closed(const std::vector<SymOp>& ops, const std::vector<SymOp>& rec,
                                                  const std::vector<SymOp>& rots, const int* n, int dim) {
  const long total = static_cast<long>(n[0]) * n[1] * n[2];
  std::vector<std::array<int, 9>> R;
  for (const auto& r : rots) {
    if (is_identity_R(r)) continue;
    std::array<int, 9> a{};
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) a[3 * i + j] = r.R[i][j];
    R.push_back(a);
  }
  // Rotation entries of crystallographic groups are small, so an image coordinate lies
  // within a few multiples of N of [0, N) and is wrapped by adding or subtracting N.
  int amax = 0;
  for (const auto& a : R)
    for (int v : a) amax = std::max(amax, std::abs(v));
  const bool small = amax <= 2;
  auto image = [&](const std::array<int, 9>& a, const int* k) {
    long li = 0, stride = 1;
    for (int d = 0; d < 3; ++d) {
      long s = static_cast<long>(a[3 * d]) * k[0] + static_cast<long>(a[3 * d + 1]) * k[1] +
               static_cast<long>(a[3 * d + 2]) * k[2];
      if (small) {
        while (s < 0) s += n[d];
        while (s >= n[d]) s -= n[d];
      } else {
        s = floor_mod(s, n[d]);
      }
      li += s * stride;
      stride *= n[d];
    }
    return li;
  };
  const long nthreads = std::max(1L, std::min<long>(std::min(16u, std::max(1u, std::thread::hardware_concurrency())),
                                                    total / 65536));
  std::vector<std::vector<SpecPoint>> part(nthreads);
  auto work = [&](long t) {
    const long l0 = total * t / nthreads, l1 = total * (t + 1) / nthreads;
    std::vector<long> imgs;
    // Move-to-front: the rotation that rejected the previous point is tried first, since
    // neighbouring points are usually rejected by the same one.
    std::vector<int> order(R.size());
    std::iota(order.begin(), order.end(), 0);
    for (long lin = l0; lin < l1; ++lin) {
      const int k[3] = {static_cast<int>(lin % n[0]), static_cast<int>((lin / n[0]) % n[1]),
                        static_cast<int>(lin / (static_cast<long>(n[0]) * n[1]))};
      bool rep = true;
      for (size_t i = 0; i < order.size(); ++i)
        if (image(R[order[i]], k) < lin) {
          rep = false;
          if (i) std::swap(order[0], order[i]);
          break;
        }
      if (!rep) continue;
      imgs.assign(1, lin);
      for (const auto& a : R) imgs.push_back(image(a, k));
      std::sort(imgs.begin(), imgs.end());
      const int mult = static_cast<int>(std::unique(imgs.begin(), imgs.end()) - imgs.begin());
      if (!spectral_alive(ops, rec, k, n, dim)) continue;
      SpecPoint p;
      p.h[0] = k[0]; p.h[1] = k[1]; p.h[2] = k[2];
      p.mult = mult;
      part[t].push_back(p);
    }
  };
  std::vector<std::thread> pool;
  for (long t = 1; t < nthreads; ++t) pool.emplace_back(work, t);
  work(0);
  for (auto& th : pool) th.join();
  std::vector<SpecPoint> pts;
  for (auto& v : part) pts.insert(pts.end(), v.begin(), v.end());
  return pts;
}

// calc_spectral_asu (src/spectral_indexing.jl:22-176): orbit representatives of the
// dual point group (smallest column-major index), with the stabiliser-phase
// extinction filter, sorted lexicographically by (h1, h2, h3).
//
// The reference grows each orbit by a closure walk that applies every operation to
// every member, O(N^3 |G|).  When the distinct dual rotations form a group (always,
// for a space group's operations) the representatives are found directly
// (spectral_asu_closed); the result is identical.  Operation lists that are not closed
// keep the closure walk.  The last result is kept per host thread, so the query and the
// fill call of the C ABI and the plan build on the same operations compute it once.
std::vector<SpecPoint> calc_spectral_asu(const std::vector<SymOp>& ops, const int* N, int dim) {
  const int n[3] = {N[0], dim > 1 ? N[1] : 1, dim > 2 ? N[2] : 1};
  thread_local std::vector<long> cache_key;
  thread_local std::vector<SpecPoint> cache_pts;
  std::vector<long> key{dim, n[0], n[1], n[2]};
  for (const auto& op : ops) {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) key.push_back(op.R[i][j]);
    for (int i = 0; i < 3; ++i) key.push_back(op.t[i]);
  }
  if (key == cache_key) return cache_pts;
  const long total = static_cast<long>(n[0]) * n[1] * n[2];
  const std::vector<SymOp> rec = dual_ops(ops);
  const std::vector<SymOp> rots = distinct_rotations(rec);
  std::vector<SpecPoint> pts;
  if (rotations_form_group(rots)) {
    pts = spectral_asu_closed(ops, rec, rots, n, dim);
  } else {
    std::vector<char> visited(total, 0);
    std::vector<long> work;
    for (long lin = 0; lin < total; ++lin) {
      if (visited[lin]) continue;
      visited[lin] = 1;
      int orbit = 1;
      long min_lin = lin;
      work.clear();
      work.push_back(lin);
      for (size_t w = 0; w < work.size(); ++w) {
        long r2 = work[w];
        int kk[3];
        kk[0] = r2 % n[0]; r2 /= n[0]; kk[1] = r2 % n[1]; kk[2] = r2 / n[1];
        for (const auto& op : rec) {
          long li = 0, stride = 1;
          for (int d = 0; d < 3; ++d) {
            long s = 0;
            for (int j = 0; j < 3; ++j) s += op.R[d][j] * kk[j];
            li += floor_mod(s, n[d]) * stride;
            stride *= n[d];
          }
          if (!visited[li]) {
            visited[li] = 1;
            ++orbit;
            work.push_back(li);
            if (li < min_lin) min_lin = li;
          }
        }
      }
      int kr[3];
      long rem = min_lin;
      kr[0] = rem % n[0]; rem /= n[0]; kr[1] = rem % n[1]; kr[2] = rem / n[1];
      if (!spectral_alive(ops, rec, kr, n, dim)) continue;
      SpecPoint p;
      p.h[0] = kr[0]; p.h[1] = kr[1]; p.h[2] = kr[2];
      p.mult = orbit;
      pts.push_back(p);
    }
  }
  std::sort(pts.begin(), pts.end(), [](const SpecPoint& a, const SpecPoint& b) {
    if (a.h[0] != b.h[0]) return a.h[0] < b.h[0];
    if (a.h[1] != b.h[1]) return a.h[1] < b.h[1];
    return a.h[2] < b.h[2];
  });
  cache_key.swap(key);
  cache_pts = pts;
  return pts;
}

// get_k_vector (src/spectral_indexing.jl:195-238): wrap to (-N/2, N/2].
void get_k_vector(const SpecPoint& p, const int* N, int* k) {
  for (int d = 0; d < 3; ++d) {
    const int n = N[d], v = p.h[d];
    k[d] = (v >= n - n / 2) ? v - n : v;
  }
}

// auto_L (src/krfft.jl:225-279).
std::array<int, 3> auto_L(const std::vector<SymOp>& ops, int dim) {
  std::array<int, 3> Lmax = {1, 1, 1};
  for (const auto& op : ops)
    for (int d = 0; d < dim; ++d)
      if (floor_mod(op.t[d], 2) == 1) Lmax[d] = 2;
  const int nsub = Lmax[0] * Lmax[1] * Lmax[2];
  if (nsub <= 1) return Lmax;
  auto reach_count = [&](const std::array<int, 3>& L) {
    std::set<std::array<int, 3>> reach;
    for (const auto& op : ops)
      reach.insert({static_cast<int>(floor_mod(op.t[0], L[0])), static_cast<int>(floor_mod(op.t[1], L[1])),
                    static_cast<int>(floor_mod(op.t[2], L[2]))});
    return static_cast<int>(reach.size());
  };
  if (reach_count(Lmax) == nsub) return Lmax;
  std::array<int, 3> best = {1, 1, 1};
  for (int mask = 1; mask < (1 << dim); ++mask) {
    std::array<int, 3> Lt = {1, 1, 1};
    for (int d = 0; d < dim; ++d)
      if (((mask >> d) & 1) && Lmax[d] == 2) Lt[d] = 2;
    const int ns = Lt[0] * Lt[1] * Lt[2];
    if (reach_count(Lt) == ns && ns > best[0] * best[1] * best[2]) best = Lt;
  }
  return best;
}

// _select_rep_ops (src/krfft.jl:958-987): one operation per parity class x0 = t mod L,
// preferring diagonal R with t in {0, N-1}; classes enumerated with x0[0] fastest.
Status select_rep_ops(const std::vector<SymOp>& ops, const std::array<int, 3>& L, const int* N,
                      std::vector<SymOp>* rep, std::string* err) {
  const int d = L[0] * L[1] * L[2];
  std::vector<int> best(d, -1), quality(d, -1);
  for (size_t k = 0; k < ops.size(); ++k) {
    const auto& op = ops[k];
    const int x0 = static_cast<int>(floor_mod(op.t[0], L[0]) + L[0] * (floor_mod(op.t[1], L[1]) + L[1] * floor_mod(op.t[2], L[2])));
    bool diag = true;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        if (i != j && op.R[i][j] != 0) diag = false;
    bool simple = true;
    for (int dd = 0; dd < 3; ++dd) {
      const long tm = floor_mod(op.t[dd], N[dd]);
      if (!(tm == 0 || tm == N[dd] - 1)) simple = false;
    }
    const int q = diag ? (simple ? 2 : 1) : 0;
    if (best[x0] < 0 || q > quality[x0]) { best[x0] = static_cast<int>(k); quality[x0] = q; }
  }
  rep->clear();
  for (int c = 0; c < d; ++c) {
    if (best[c] < 0) { *err = "subgrid parity class not reachable; auto_L should have prevented this"; return Status::kNotReachable; }
    rep->push_back(ops[best[c]]);
  }
  return Status::kOk;
}

// detect_centering_type (src/symmetry_ops.jl:133-179).
Centering detect_centering_type(const std::vector<SymOp>& ops, const int* N, int dim) {
  bool any = false, xyz = false, x0yz = false, xx0z = false, xy0 = false;
  for (const auto& op : ops) {
    if (!is_identity_R(op)) continue;
    bool zero = true;
    for (int d = 0; d < dim; ++d)
      if (op.t[d] != 0) zero = false;
    if (zero) continue;
    bool half[3] = {false, false, false};
    for (int d = 0; d < dim; ++d) half[d] = std::fabs(std::fabs(static_cast<double>(op.t[d])) / N[d] - 0.5) < 0.01;
    any = true;
    if (dim < 3) continue;
    if (half[0] && half[1] && half[2]) xyz = true;
    if (!half[0] && half[1] && half[2]) x0yz = true;
    if (half[0] && !half[1] && half[2]) xx0z = true;
    if (half[0] && half[1] && !half[2]) xy0 = true;
  }
  if (!any || dim < 3) return kCentP;
  if (static_cast<int>(x0yz) + static_cast<int>(xx0z) + static_cast<int>(xy0) >= 2) return kCentF;
  if (xyz) return kCentI;
  if (xy0) return kCentC;
  if (x0yz) return kCentA;
  if (xx0z) return kCentA;  // B centring is classified as A, as in the reference
  return kCentP;
}

// _alive_offsets (src/centering_fold.jl:111-127).
int alive_offsets(Centering c, std::array<int, 3>* o) {
  switch (c) {
    case kCentI: o[0] = {0, 0, 0}; o[1] = {1, 1, 0}; o[2] = {1, 0, 1}; o[3] = {0, 1, 1}; return 4;
    case kCentF: o[0] = {0, 0, 0}; o[1] = {1, 1, 1}; return 2;
    case kCentC: o[0] = {0, 0, 0}; o[1] = {1, 1, 0}; o[2] = {0, 0, 1}; o[3] = {1, 1, 1}; return 4;
    case kCentA: o[0] = {0, 0, 0}; o[1] = {0, 1, 1}; o[2] = {1, 0, 0}; o[3] = {1, 1, 1}; return 4;
    default: return 0;
  }
}

static long lcm_l(long a, long b) { return a / std::gcd(a, b) * b; }

Status build_tables(const std::vector<SymOp>& shifted_ops, const int* N_in, int dim, bool want_centered,
                    PlanTables* T, std::string* err, bool full_grid) {
  if (shifted_ops.empty()) { *err = "empty operation list"; return Status::kInvalid; }
  T->dim = dim;
  for (int d = 0; d < 3; ++d) T->N[d] = d < dim ? N_in[d] : 1;
  const int* N = T->N;
  for (int d = 0; d < 3; ++d)
    if (N[d] < 1 || N[d] > 1024) { *err = "grid edge must be in [1, 1024]"; return Status::kInvalid; }
  T->ops = shifted_ops;
  for (auto& op : T->ops)
    for (int d = dim; d < 3; ++d) {
      op.t[d] = 0;
      for (int j = 0; j < 3; ++j) op.R[d][j] = op.R[j][d] = (d == j);
    }
  // Full-grid plans (the centring prefold, src/centering_prefold.jl) keep L = 1: the
  // "subgrid" is the whole grid and the identity is the only representative.
  const std::array<int, 3> L = full_grid ? std::array<int, 3>{1, 1, 1} : auto_L(T->ops, dim);
  for (int d = 0; d < 3; ++d) {
    T->L[d] = L[d];
    if (N[d] % L[d] != 0) { *err = "Grid size N not divisible by auto L"; return Status::kNotCommensurate; }
    T->M[d] = N[d] / L[d];
  }
  T->d = L[0] * L[1] * L[2];
  long P = 1;
  for (int d = 0; d < 3; ++d) P = lcm_l(P, N[d]);
  if (P > (1 << 20)) { *err = "lcm of grid edges too large"; return Status::kUnsupported; }
  T->P = static_cast<int>(P);
  Status st = select_rep_ops(T->ops, L, N, &T->rep_ops, err);
  if (st != Status::kOk) return st;
  if (!is_identity_R(T->rep_ops[0]) || T->rep_ops[0].t[0] || T->rep_ops[0].t[1] || T->rep_ops[0].t[2]) {
    *err = "the identity operation must represent parity class 0";
    return Status::kInvalid;
  }
  T->spec = calc_spectral_asu(T->ops, N, dim);
  T->centering = detect_centering_type(T->ops, N, dim);
  // plan_krfft_centered falls back to the plain path for P, L != 2, or odd M
  // (src/centering_fold.jl:339-352).
  // Full-grid plans fold the whole grid into the parity channels of (N/2)^3, which is
  // exact for any field; the centring only decides which channels exist.
  T->centered = want_centered && T->centering != kCentP && dim == 3 &&
                (full_grid || (L[0] == 2 && L[1] == 2 && L[2] == 2)) &&
                T->M[0] % 2 == 0 && T->M[1] % 2 == 0 && T->M[2] % 2 == 0;
  for (int p = 0; p < 8; ++p) T->chan_of_parity[p] = -1;
  if (T->centered) {
    T->n_ch = alive_offsets(T->centering, T->offsets);
    for (int d = 0; d < 3; ++d) T->H[d] = T->M[d] / 2;
    for (int c = 0; c < T->n_ch; ++c)
      T->chan_of_parity[T->offsets[c][0] + 2 * T->offsets[c][1] + 4 * T->offsets[c][2]] = c;
  } else {
    T->n_ch = 1;
    for (int d = 0; d < 3; ++d) T->H[d] = T->M[d];
    T->offsets[0] = {0, 0, 0};
  }

  // ---- reverse lookup (src/krfft.jl:1183-1255) ----
  // For a full-grid frequency key, the entry of _build_spectral_reverse_lookup: the
  // spectral point s whose orbit holds the key (direct) or its negative (conjugate),
  // with the symmetry phase, the first writer winning in the reference's order (for
  // each s: itself, then per operation j its image R_j^T h_s and the negative, then -h_s).
  const long n1 = N[0], n2 = N[1], n3 = N[2];
  const long total = n1 * n2 * n3;
  auto lin = [&](long a, long b, long c) { return a + n1 * (b + n2 * c); };
  auto phase_num = [&](const int* h, const int* t) {
    long j = 0;
    for (int d = 0; d < 3; ++d) j += static_cast<long>(h[d]) * t[d] * (P / N[d]);
    return static_cast<int32_t>(floor_mod(j, P));
  };
  const int nspec = static_cast<int>(T->spec.size());
  const std::vector<SymOp> rev_rots = distinct_rotations(dual_ops(T->ops));
  const bool rev_closed = rotations_form_group(rev_rots);
  // Non-closed operation lists: the reference's dense table over the full grid.
  std::vector<int32_t> rs, rp;
  std::vector<char> rc;
  if (!rev_closed) {
    rs.assign(total, 0);
    rp.assign(total, 0);
    rc.assign(total, 0);
    for (int s = 0; s < nspec; ++s) {
      const int* h = T->spec[s].h;
      long key = lin(h[0], h[1], h[2]);
      if (!rs[key]) { rs[key] = s + 1; rp[key] = 0; rc[key] = 0; }
      for (const auto& op : T->ops) {
        long hr[3];
        for (int d = 0; d < 3; ++d) {
          long v = 0;
          for (int d2 = 0; d2 < 3; ++d2) v += static_cast<long>(op.R[d2][d]) * h[d2];
          hr[d] = floor_mod(v, N[d]);
        }
        const int32_t ph = phase_num(h, op.t);
        key = lin(hr[0], hr[1], hr[2]);
        if (!rs[key]) { rs[key] = s + 1; rp[key] = ph; rc[key] = 0; }
        key = lin(floor_mod(-hr[0], n1), floor_mod(-hr[1], n2), floor_mod(-hr[2], n3));
        if (!rs[key]) { rs[key] = s + 1; rp[key] = static_cast<int32_t>(floor_mod(-static_cast<long>(ph), P)); rc[key] = 1; }
      }
      key = lin(floor_mod(-h[0], n1), floor_mod(-h[1], n2), floor_mod(-h[2], n3));
      if (!rs[key]) { rs[key] = s + 1; rp[key] = 0; rc[key] = 1; }
    }
  }
  // Closed groups: each queried key is answered directly.  The spectral points are the
  // smallest members of their orbits, so the candidates are s_d = the point at the
  // orbit minimum of k (a direct entry) and s_c = that of -k (a conjugate entry); the
  // smaller s wins, and within one s the first operation in list order.
  std::unordered_map<long, int> spec_at;
  if (rev_closed) {
    spec_at.reserve(2 * static_cast<size_t>(nspec) + 1);
    for (int s = 0; s < nspec; ++s) spec_at[lin(T->spec[s].h[0], T->spec[s].h[1], T->spec[s].h[2])] = s;
  }
  auto orbit_min = [&](const long* k) {
    long best = LONG_MAX;
    for (const auto& r : rev_rots) {
      long v[3];
      for (int d = 0; d < 3; ++d) {
        long x = 0;
        for (int j = 0; j < 3; ++j) x += static_cast<long>(r.R[d][j]) * k[j];
        v[d] = floor_mod(x, N[d]);
      }
      best = std::min(best, lin(v[0], v[1], v[2]));
    }
    return best;
  };
  // (signed spectral index + 1 as in the dense table: 0 = absent, < 0 conjugate; phase)
  auto lookup = [&](const long* k, int32_t* sgn, int32_t* ph) {
    if (!rev_closed) {
      const long key = lin(k[0], k[1], k[2]);
      *sgn = rs[key] ? (rc[key] ? -rs[key] : rs[key]) : 0;
      *ph = rs[key] ? rp[key] : 0;
      return;
    }
    const long nk[3] = {floor_mod(-k[0], n1), floor_mod(-k[1], n2), floor_mod(-k[2], n3)};
    auto find = [&](long key) {
      auto it = spec_at.find(key);
      return it == spec_at.end() ? -1 : it->second;
    };
    const int sd = find(orbit_min(k)), sc = find(orbit_min(nk));
    if (sd < 0 && sc < 0) { *sgn = 0; *ph = 0; return; }
    const long big = 4L * static_cast<long>(T->ops.size()) + 8;
    // order of the first direct write of k by sd, and of the first conjugate write by sc
    auto first_write = [&](int s, bool conj, int32_t* phase) -> long {
      const int* h = T->spec[s].h;
      if (!conj && h[0] == k[0] && h[1] == k[1] && h[2] == k[2]) { *phase = 0; return -1; }
      for (size_t j = 0; j < T->ops.size(); ++j) {
        const auto& op = T->ops[j];
        long hr[3];
        for (int d = 0; d < 3; ++d) {
          long v = 0;
          for (int d2 = 0; d2 < 3; ++d2) v += static_cast<long>(op.R[d2][d]) * h[d2];
          hr[d] = floor_mod(conj ? -v : v, N[d]);
        }
        if (hr[0] == k[0] && hr[1] == k[1] && hr[2] == k[2]) {
          const int32_t p0 = phase_num(h, op.t);
          *phase = conj ? static_cast<int32_t>(floor_mod(-static_cast<long>(p0), P)) : p0;
          return 2 * static_cast<long>(j) + (conj ? 1 : 0);
        }
      }
      if (conj && floor_mod(-h[0], n1) == k[0] && floor_mod(-h[1], n2) == k[1] && floor_mod(-h[2], n3) == k[2]) {
        *phase = 0;
        return 2 * static_cast<long>(T->ops.size());
      }
      *phase = 0;
      return big;  // not written by s (does not happen for a closed group)
    };
    int32_t pd = 0, pc = 0;
    const long od = sd >= 0 ? first_write(sd, false, &pd) : big;
    const long oc = sc >= 0 ? first_write(sc, true, &pc) : big;
    const bool take_d = sd >= 0 && od < big && (sc < 0 || oc >= big || sd < sc || (sd == sc && od < oc));
    if (take_d) { *sgn = sd + 1; *ph = pd; return; }
    if (sc >= 0 && oc < big) { *sgn = -(sc + 1); *ph = pc; return; }
    *sgn = 0;
    *ph = 0;
  };

  // ---- orbit structure on the M-grid under the even-translation subgroup ----
  // (src/centering_fold.jl:643-687, generalised to any L by s = t / L)
  T->rem_ops.clear();
  for (const auto& op : T->ops) {
    bool ok = true;
    for (int d = 0; d < 3 && ok; ++d)
      if (floor_mod(op.t[d], L[d]) != 0) ok = false;
    SymOp r{};
    for (int i = 0; i < 3 && ok; ++i)
      for (int j = 0; j < 3 && ok; ++j) {
        const long v = static_cast<long>(op.R[i][j]) * L[j];
        if (v % L[i] != 0) ok = false;
        r.R[i][j] = static_cast<int>(v / L[i]);
      }
    if (!ok) continue;
    for (int d = 0; d < 3; ++d) r.t[d] = static_cast<int>(floor_mod(op.t[d] / L[d], T->M[d]));
    T->rem_ops.push_back(r);
  }
  const int* M = T->M;
  const long mtot = static_cast<long>(M[0]) * M[1] * M[2];
  std::vector<char> seen(mtot, 0);
  T->orbit_rep.clear();
  T->inv_spec.clear();
  T->inv_phase.clear();
  const int d = T->d;
  for (long m = 0; m < mtot; ++m) {
    if (seen[m]) continue;
    int q[3];
    long r = m;
    q[0] = r % M[0]; r /= M[0]; q[1] = r % M[1]; q[2] = r / M[1];
    const int par = (q[0] & 1) + 2 * (q[1] & 1) + 4 * (q[2] & 1);
    const bool alive = !T->centered || T->chan_of_parity[par] >= 0;
    for (const auto& op : T->rem_ops) {
      long li = 0, stride = 1;
      for (int dd = 0; dd < 3; ++dd) {
        long v = 0;
        for (int d2 = 0; d2 < 3; ++d2) v += static_cast<long>(op.R[d2][dd]) * q[d2];
        li += floor_mod(v, M[dd]) * stride;
        stride *= M[dd];
      }
      seen[li] = 1;
    }
    seen[m] = 1;
    if (!alive) continue;
    T->orbit_rep.push_back(static_cast<int32_t>(m));
  }
  // d aliases h_a = q + M .* alpha_a per representative, alpha with the first axis
  // fastest; the lookups are independent and run on host threads.
  const long n_orb_all = static_cast<long>(T->orbit_rep.size());
  T->inv_spec.assign(static_cast<size_t>(n_orb_all) * d, 0);
  T->inv_phase.assign(static_cast<size_t>(n_orb_all) * d, 0);
  auto fill = [&](long o0, long o1) {
    for (long o = o0; o < o1; ++o) {
      long rr = T->orbit_rep[o];
      long q[3];
      q[0] = rr % M[0]; rr /= M[0]; q[1] = rr % M[1]; q[2] = rr / M[1];
      for (int a = 0; a < d; ++a) {
        int alpha[3];
        int rem = a;
        for (int dd = 0; dd < 3; ++dd) { alpha[dd] = rem % L[dd]; rem /= L[dd]; }
        long hk[3];
        for (int dd = 0; dd < 3; ++dd) hk[dd] = floor_mod(q[dd] + static_cast<long>(M[dd]) * alpha[dd], N[dd]);
        lookup(hk, &T->inv_spec[o * d + a], &T->inv_phase[o * d + a]);
      }
    }
  };
  const long nth = rev_closed ? std::max(1L, std::min<long>(std::min(16u, std::max(1u, std::thread::hardware_concurrency())),
                                                            n_orb_all / 2048))
                              : 1;
  {
    std::vector<std::thread> pool;
    for (long t = 1; t < nth; ++t) pool.emplace_back(fill, n_orb_all * t / nth, n_orb_all * (t + 1) / nth);
    fill(0, n_orb_all / nth);
    for (auto& th : pool) th.join();
  }
  // Order the representatives by the spectral index of their first alias so that
  // neighbouring device threads gather neighbouring spectrum entries.
  const size_t n_orb = T->orbit_rep.size();
  std::vector<size_t> perm(n_orb);
  std::iota(perm.begin(), perm.end(), 0);
  std::stable_sort(perm.begin(), perm.end(), [&](size_t a, size_t b) {
    return std::abs(T->inv_spec[a * d]) < std::abs(T->inv_spec[b * d]);
  });
  std::vector<int32_t> rep2(n_orb), spec2(n_orb * d), phase2(n_orb * d);
  for (size_t k = 0; k < n_orb; ++k) {
    rep2[k] = T->orbit_rep[perm[k]];
    for (int a = 0; a < d; ++a) {
      spec2[k * d + a] = T->inv_spec[perm[k] * d + a];
      phase2[k * d + a] = T->inv_phase[perm[k] * d + a];
    }
  }
  T->orbit_rep.swap(rep2);
  T->inv_spec.swap(spec2);
  T->inv_phase.swap(phase2);
  return Status::kOk;
}

// K(h) = exp(-ds |2 pi A^-T h_c|^2), h_c = h >= N÷2 ? h - N : h
// (src/centering_fold.jl:881-891, src/q_fused_krfft.jl:967-974).
void compute_kernel(const PlanTables& T, const double* lattice, double ds, std::vector<double>* K) {
  // lattice is column-major 3x3 (lattice vectors in columns), as a Julia Matrix.
  double A[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) A[i][j] = lattice[i + 3 * j];
  if (T.dim == 2) {
    for (int i = 0; i < 3; ++i) { A[i][2] = (i == 2); A[2][i] = (i == 2); }
  }
  const double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                     A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                     A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
  double inv[3][3];
  inv[0][0] = (A[1][1] * A[2][2] - A[1][2] * A[2][1]) / det;
  inv[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) / det;
  inv[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) / det;
  inv[1][0] = (A[1][2] * A[2][0] - A[1][0] * A[2][2]) / det;
  inv[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) / det;
  inv[1][2] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) / det;
  inv[2][0] = (A[1][0] * A[2][1] - A[1][1] * A[2][0]) / det;
  inv[2][1] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) / det;
  inv[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) / det;
  K->resize(T.spec.size());
  for (size_t s = 0; s < T.spec.size(); ++s) {
    double hc[3];
    for (int d = 0; d < 3; ++d) {
      const int v = T.spec[s].h[d];
      hc[d] = (v >= T.N[d] / 2) ? v - T.N[d] : v;
      if (d >= T.dim) hc[d] = 0.0;
    }
    double k2 = 0.0;
    for (int i = 0; i < 3; ++i) {
      // recip_B = 2 pi inv(A)^T  =>  k_i = 2 pi sum_j inv[j][i] h_j
      double k = 0.0;
      for (int j = 0; j < 3; ++j) k += inv[j][i] * hc[j];
      k *= 2.0 * M_PI;
      k2 += k * k;
    }
    (*K)[s] = std::exp(-k2 * ds);
  }
}

// Q-matrix tables of the M2+Q / M7 diffusion step (plan_m2_q, _build_q_matrices!,
// src/q_fused_krfft.jl:83-169,182-413).  For each subgrid point q (column-major) and
// parity class a, h_a = q + M.alpha_a (classes in Iterators.product order, first axis
// fastest), B[a][b] = e^{-2 pi i h_a.t_b / N} over the representative operations b and
// K_a = exp(-ds |2 pi A^-T h_a,c|^2).  Q(q) = B^-1 diag(K) B; only its first row is
// used: Q[b] = sum_a y_a K_a B[a][b] with B^T y = e_0.  gather[b][q] = lin(R_b^T q mod M).
// Q is returned interleaved (re, im) as Q[(b * Mvol + q) * 2 + {0, 1}].
Status build_q_tables(const PlanTables& T, const double* lattice, double ds, std::vector<double>* Q,
                      std::vector<int32_t>* gather, std::string* err) {
  using cd = std::complex<double>;
  const int d = static_cast<int>(T.rep_ops.size());
  const long Mvol = static_cast<long>(T.M[0]) * T.M[1] * T.M[2];
  if (d < 1 || d > 8) { *err = "Q tables need 1..8 representative operations"; return Status::kInvalid; }
  double A[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) A[i][j] = lattice[i + 3 * j];
  if (T.dim == 2)
    for (int i = 0; i < 3; ++i) { A[i][2] = (i == 2); A[2][i] = (i == 2); }
  const double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                     A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                     A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
  if (det == 0.0) { *err = "singular lattice"; return Status::kInvalid; }
  double inv[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      const int i1 = (j + 1) % 3, i2 = (j + 2) % 3, j1 = (i + 1) % 3, j2 = (i + 2) % 3;
      inv[i][j] = (A[i1][j1] * A[i2][j2] - A[i1][j2] * A[i2][j1]) / det;  // adjugate / det
    }
  // parity classes alpha_a, first axis fastest
  std::vector<std::array<int, 3>> alpha(d);
  for (int a = 0; a < d; ++a) {
    int r = a;
    for (int k = 0; k < 3; ++k) { alpha[a][k] = r % T.L[k]; r /= T.L[k]; }
  }
  if (T.L[0] * T.L[1] * T.L[2] != d) { *err = "parity classes do not match the representatives"; return Status::kInvalid; }
  Q->assign(static_cast<size_t>(d) * Mvol * 2, 0.0);
  gather->assign(static_cast<size_t>(d) * Mvol, 0);
  // Fibers are independent: contiguous ranges of q go to host threads, each fiber's
  // entries are computed exactly as in a serial pass.
  std::atomic<bool> singular{false};
  auto fibers = [&](long q0, long q1) {
  for (long q = q0; q < q1 && !singular.load(std::memory_order_relaxed); ++q) {
    const long qv[3] = {q % T.M[0], (q / T.M[0]) % T.M[1], q / (static_cast<long>(T.M[0]) * T.M[1])};
    cd Bm[8][8];
    double Kv[8];
    for (int a = 0; a < d; ++a) {
      long h[3];
      double hc[3];
      for (int k = 0; k < 3; ++k) {
        h[k] = qv[k] + static_cast<long>(T.M[k]) * alpha[a][k];
        hc[k] = (h[k] >= T.N[k] / 2) ? static_cast<double>(h[k] - T.N[k]) : static_cast<double>(h[k]);
        if (k >= T.dim) hc[k] = 0.0;
      }
      double k2 = 0.0;
      for (int i = 0; i < 3; ++i) {
        double kk = 0.0;
        for (int j = 0; j < 3; ++j) kk += inv[j][i] * hc[j];
        kk *= 2.0 * M_PI;
        k2 += kk * kk;
      }
      Kv[a] = std::exp(-k2 * ds);
      for (int b = 0; b < d; ++b) {
        double ph = 0.0;
        for (int k = 0; k < T.dim; ++k) ph += static_cast<double>(h[k]) * T.rep_ops[b].t[k] / T.N[k];
        Bm[a][b] = std::polar(1.0, -2.0 * M_PI * ph);
      }
    }
    // Solve B^T y = e_0 by Gaussian elimination with partial pivoting.
    cd Mx[8][9];
    for (int i = 0; i < d; ++i) {
      for (int j = 0; j < d; ++j) Mx[i][j] = Bm[j][i];
      Mx[i][d] = (i == 0) ? cd(1.0, 0.0) : cd(0.0, 0.0);
    }
    for (int c = 0; c < d; ++c) {
      int piv = c;
      for (int i = c + 1; i < d; ++i)
        if (std::abs(Mx[i][c]) > std::abs(Mx[piv][c])) piv = i;
      if (std::abs(Mx[piv][c]) < 1e-12) { singular = true; return; }
      if (piv != c)
        for (int j = 0; j <= d; ++j) std::swap(Mx[c][j], Mx[piv][j]);
      for (int i = c + 1; i < d; ++i) {
        const cd f = Mx[i][c] / Mx[c][c];
        for (int j = c; j <= d; ++j) Mx[i][j] -= f * Mx[c][j];
      }
    }
    cd y[8];
    for (int i = d - 1; i >= 0; --i) {
      cd acc = Mx[i][d];
      for (int j = i + 1; j < d; ++j) acc -= Mx[i][j] * y[j];
      y[i] = acc / Mx[i][i];
    }
    for (int b = 0; b < d; ++b) {
      cd acc(0.0, 0.0);
      for (int a = 0; a < d; ++a) acc += y[a] * Kv[a] * Bm[a][b];
      (*Q)[(static_cast<size_t>(b) * Mvol + q) * 2] = acc.real();
      (*Q)[(static_cast<size_t>(b) * Mvol + q) * 2 + 1] = acc.imag();
      long g = 0, stride = 1;
      for (int k = 0; k < 3; ++k) {
        long v = 0;
        for (int j = 0; j < 3; ++j) v += static_cast<long>(T.rep_ops[b].R[j][k]) * qv[j];  // (R^T q)_k
        g += floor_mod(v, T.M[k]) * stride;
        stride *= T.M[k];
      }
      (*gather)[static_cast<size_t>(b) * Mvol + q] = static_cast<int32_t>(g);
    }
  }
  };
  const long nthreads = std::max(1L, std::min<long>(std::min(16u, std::max(1u, std::thread::hardware_concurrency())),
                                                    Mvol / 4096));
  std::vector<std::thread> pool;
  const long per = (Mvol + nthreads - 1) / nthreads;
  for (long k = 1; k < nthreads; ++k) pool.emplace_back(fibers, std::min(Mvol, k * per), std::min(Mvol, (k + 1) * per));
  fibers(0, std::min(Mvol, per));
  for (auto& th : pool) th.join();
  if (singular) { *err = "singular alias matrix B"; return Status::kInvalid; }
  return Status::kOk;
}

// Real-space asymmetric unit by recursive parity splitting (calc_asu(N, ops),
// src/asu.jl:216-324).  A state is a sub-problem on curr_N points with operations
// acting on it, mapped to the full grid by x = scale .* p + offset.  Each active
// dimension whose parity every operation preserves splits into its even and odd
// halves (S = 2); the operations of a half are R' = S^-1 R S, t' = S^-1 (R p + t - p)
// and the half is dropped when they are not integral.  Odd halves and dimensions that
// cannot split become general-position leaves; a leaf lists one point per orbit of
// its operations (the lexicographically smallest member) with the orbit size.  The
// result is sorted by grid index.
std::vector<AsuPoint> calc_asu(const std::vector<SymOp>& ops_in, const int* N_in, int dim) {
  struct State {
    int n[3], scale[3], offset[3], depth[3];
    bool gp[3];
    std::vector<SymOp> ops;
  };
  std::vector<AsuPoint> out;
  std::vector<State> stack;
  State s0{};
  for (int d = 0; d < 3; ++d) {
    s0.n[d] = d < dim ? N_in[d] : 1;
    s0.scale[d] = 1;
    s0.offset[d] = 0;
    s0.depth[d] = 0;
    s0.gp[d] = d >= dim;  // unused dimensions never split
  }
  s0.ops = ops_in;
  stack.push_back(std::move(s0));
  auto apply = [&](const SymOp& op, const int* x, const int* n, int* y) {
    for (int i = 0; i < dim; ++i) {
      long v = op.t[i];
      for (int j = 0; j < dim; ++j) v += static_cast<long>(op.R[i][j]) * x[j];
      y[i] = static_cast<int>(floor_mod(v, n[i]));
    }
  };
  while (!stack.empty()) {
    State st = std::move(stack.back());
    stack.pop_back();
    bool empty = false, all_gp = true, all_small = true;
    for (int d = 0; d < dim; ++d) {
      if (st.n[d] == 0) empty = true;
      if (!st.gp[d]) all_gp = false;
      if (st.n[d] > 1) all_small = false;
    }
    if (empty) continue;
    if (all_gp || all_small) {
      const long total = static_cast<long>(st.n[0]) * st.n[1] * st.n[2];
      std::vector<char> seen(total, 0);
      std::vector<long> orbit;
      const bool closed = affine_ops_form_group(st.ops, st.n, dim);
      for (long lin = 0; lin < total; ++lin) {
        if (seen[lin]) continue;
        orbit.assign(1, lin);
        seen[lin] = 1;
        if (closed) {  // the orbit is {g x}: one pass of the operations
          const int x[3] = {static_cast<int>(lin % st.n[0]), static_cast<int>((lin / st.n[0]) % st.n[1]),
                            static_cast<int>(lin / (static_cast<long>(st.n[0]) * st.n[1]))};
          for (const auto& op : st.ops) {
            int y[3] = {0, 0, 0};
            apply(op, x, st.n, y);
            const long li = y[0] + static_cast<long>(st.n[0]) * (y[1] + static_cast<long>(st.n[1]) * y[2]);
            if (!seen[li]) { seen[li] = 1; orbit.push_back(li); }
          }
        }
        for (size_t w = closed ? orbit.size() : 0; w < orbit.size(); ++w) {
          long r = orbit[w];
          int x[3] = {static_cast<int>(r % st.n[0]), static_cast<int>((r / st.n[0]) % st.n[1]),
                      static_cast<int>(r / (static_cast<long>(st.n[0]) * st.n[1]))};
          for (const auto& op : st.ops) {
            int y[3] = {0, 0, 0};
            apply(op, x, st.n, y);
            const long li = y[0] + static_cast<long>(st.n[0]) * (y[1] + static_cast<long>(st.n[1]) * y[2]);
            if (!seen[li]) { seen[li] = 1; orbit.push_back(li); }
          }
        }
        // lexicographically smallest member (first coordinate most significant)
        std::array<int, 3> best{INT32_MAX, INT32_MAX, INT32_MAX};
        for (long r : orbit) {
          std::array<int, 3> x{static_cast<int>(r % st.n[0]), static_cast<int>((r / st.n[0]) % st.n[1]),
                               static_cast<int>(r / (static_cast<long>(st.n[0]) * st.n[1]))};
          if (x < best) best = x;
        }
        AsuPoint pt{};
        for (int d = 0; d < 3; ++d) {
          pt.idx[d] = st.scale[d] * best[d] + st.offset[d];
          pt.depth[d] = st.depth[d];
        }
        pt.mult = static_cast<int>(orbit.size());
        out.push_back(pt);
      }
      continue;
    }
    bool egp[3] = {st.gp[0], st.gp[1], st.gp[2]};
    for (int d = 0; d < dim; ++d) {
      if (st.gp[d]) continue;
      int pe[3] = {0, 0, 0}, po[3] = {0, 0, 0}, y[3];
      po[d] = 1;
      for (const auto& op : st.ops) {
        apply(op, pe, st.n, y);
        if (y[d] % 2 != 0) { egp[d] = true; break; }
        apply(op, po, st.n, y);
        if (y[d] % 2 != 1) { egp[d] = true; break; }
      }
    }
    int hi[3];
    for (int d = 0; d < 3; ++d) hi[d] = (egp[d] || st.n[d] <= 1) ? 0 : 1;
    for (int p2 = 0; p2 <= hi[2]; ++p2)
      for (int p1 = 0; p1 <= hi[1]; ++p1)
        for (int p0 = 0; p0 <= hi[0]; ++p0) {
          const int par[3] = {p0, p1, p2};
          int S[3];
          for (int d = 0; d < 3; ++d) S[d] = egp[d] ? 1 : 2;
          State nx{};
          bool valid = true;
          for (const auto& op : st.ops) {
            SymOp q{};
            for (int i = 0; i < 3 && valid; ++i) {
              long t = op.t[i] - par[i];
              for (int j = 0; j < 3; ++j) {
                t += static_cast<long>(op.R[i][j]) * par[j];
                const long rv = static_cast<long>(op.R[i][j]) * S[j];
                if (rv % S[i] != 0) valid = false;
                q.R[i][j] = static_cast<int>(rv / S[i]);
              }
              if (t % S[i] != 0) valid = false;
              q.t[i] = static_cast<int>(t / S[i]);
            }
            if (!valid) break;
            nx.ops.push_back(q);
          }
          if (!valid) continue;
          for (int d = 0; d < 3; ++d) {
            nx.n[d] = egp[d] ? st.n[d] : st.n[d] / 2;
            nx.gp[d] = egp[d] || par[d] == 1;
            nx.depth[d] = egp[d] ? st.depth[d] : st.depth[d] + (par[d] == 0 ? 1 : 0);
            nx.scale[d] = st.scale[d] * S[d];
            nx.offset[d] = st.scale[d] * par[d] + st.offset[d];
          }
          stack.push_back(std::move(nx));
        }
  }
  std::sort(out.begin(), out.end(), [](const AsuPoint& a, const AsuPoint& b) {
    return std::lexicographical_compare(a.idx, a.idx + 3, b.idx, b.idx + 3);
  });
  return out;
}

// ---------------------------------------------------------------------------------
// Recursive parity tree of the fractal KRFFT plans (build_recursive_tree and
// collect_leaves, src/fractal_krfft.jl:133-636).  A node splits the dimensions whose
// parity every diagonal operation preserves into even and odd sectors; sectors related
// by an operation of the half-grid-shifted group (t' = t + (I - R)/2 mod N, rounded
// half to even as the reference rounds it) share one representative child, which keeps
// the operations that map its sector to itself, rewritten in its own coordinates:
// R' = S^-1 R S, t' = S^-1 (R p + t - p).  A node whose operations are all pure
// translations splits into its alive (non-extinct) sectors, each a leaf.
namespace {

struct TreeOp {
  int R[3][3];
  long t[3];
};
struct TreeNode {
  int n[3], scale[3], offset[3], depth = 0;
  std::vector<TreeOp> ops;
  std::vector<int> children;
  bool leaf = false;
};

long round_half_even_twice(long x2) {  // round(x2 / 2), ties to even
  const long q = (x2 >= 0) ? x2 / 2 : -((-x2 + 1) / 2);  // floor(x2 / 2)
  if (x2 - 2 * q == 0) return q;
  return (q % 2 == 0) ? q : q + 1;
}

bool tree_identity(const int (&R)[3][3], int D) {
  for (int i = 0; i < D; ++i)
    for (int j = 0; j < D; ++j)
      if (R[i][j] != (i == j ? 1 : 0)) return false;
  return true;
}

}  // namespace

void fractal_tree(const std::vector<SymOp>& ops_in, const int* N, int D, int flags, std::vector<TreeLeaf>* leaves,
                  int* n_inner) {
  const bool child_shifted_t = flags & 1, centering_split = !(flags & 2);
  std::vector<TreeNode> nodes(1);
  for (int d = 0; d < 3; ++d) {
    nodes[0].n[d] = d < D ? N[d] : 1;
    nodes[0].scale[d] = 1;
    nodes[0].offset[d] = 0;
  }
  for (const auto& op : ops_in) {
    TreeOp o{};
    for (int i = 0; i < 3; ++i) {
      o.t[i] = i < D ? op.t[i] : 0;
      for (int j = 0; j < 3; ++j) o.R[i][j] = (i < D && j < D) ? op.R[i][j] : (i == j);
    }
    nodes[0].ops.push_back(o);
  }
  std::vector<int> stack{0};
  while (!stack.empty()) {
    const int id = stack.back();
    stack.pop_back();
    int cN[3];
    for (int d = 0; d < 3; ++d) cN[d] = nodes[id].n[d];
    bool zero = false;
    for (int d = 0; d < D; ++d) zero = zero || cN[d] == 0;
    if (zero) { nodes[id].leaf = true; continue; }
    const std::vector<TreeOp> ops = nodes[id].ops;  // copy: nodes may grow below
    bool nontrivial = false;
    for (const auto& o : ops) nontrivial = nontrivial || !tree_identity(o.R, D);
    if (!nontrivial) {
      // centring translations only (_setup_centering_split!, src/fractal_krfft.jl:535-604)
      std::vector<std::array<long, 3>> cent;
      for (const auto& o : ops) {
        std::array<long, 3> tm{0, 0, 0};
        bool any = false;
        for (int d = 0; d < D; ++d) { tm[d] = floor_mod(o.t[d], cN[d]); any = any || tm[d] != 0; }
        if (any) cent.push_back(tm);
      }
      bool big = true;
      for (int d = 0; d < D; ++d) big = big && cN[d] >= 2;
      if (!(centering_split && !cent.empty() && big)) { nodes[id].leaf = true; continue; }
      std::vector<int> split;
      for (int d = 0; d < D; ++d)
        if (cN[d] >= 2 && cN[d] % 2 == 0) split.push_back(d);
      std::set<std::array<long, 3>> group{{0, 0, 0}};
      std::vector<std::array<long, 3>> queue{{0, 0, 0}};
      for (const auto& t : cent)
        if (group.insert(t).second) queue.push_back(t);
      while (!queue.empty()) {
        const auto g = queue.back();
        queue.pop_back();
        for (const auto& t : cent) {
          std::array<long, 3> h{0, 0, 0};
          for (int d = 0; d < D; ++d) h[d] = floor_mod(g[d] + t[d], cN[d]);
          if (group.insert(h).second) queue.push_back(h);
        }
      }
      const int nsec = 1 << split.size();
      for (int bits = 0; bits < nsec; ++bits) {
        int p[3] = {0, 0, 0};
        for (size_t k = 0; k < split.size(); ++k) p[split[k]] = (bits >> k) & 1;
        double re = 0.0, im = 0.0;
        for (const auto& tau : group) {
          double ph = 0.0;
          for (int d = 0; d < D; ++d) ph += static_cast<double>(p[d]) * tau[d] / cN[d];
          re += std::cos(2.0 * M_PI * ph);
          im -= std::sin(2.0 * M_PI * ph);
        }
        if (std::hypot(re, im) < 0.5) continue;  // extinct sector
        TreeNode c;
        for (int d = 0; d < 3; ++d) {
          const bool sp = std::find(split.begin(), split.end(), d) != split.end();
          c.n[d] = sp ? cN[d] / 2 : cN[d];
          c.scale[d] = nodes[id].scale[d] * (sp ? 2 : 1);
          c.offset[d] = nodes[id].scale[d] * p[d] + nodes[id].offset[d];
        }
        c.leaf = true;
        c.depth = nodes[id].depth + 1;
        nodes.push_back(c);
        nodes[id].children.push_back(static_cast<int>(nodes.size()) - 1);
      }
      continue;
    }
    // splittable dimensions (find_split_dims, src/fractal_krfft.jl:159-186)
    std::vector<int> split;
    for (int d = 0; d < D; ++d) {
      if (cN[d] % 2 != 0 || cN[d] <= 1) continue;
      bool ok = true;
      for (const auto& o : ops) {
        bool diag = true;
        for (int i = 0; i < D && diag; ++i)
          for (int j = 0; j < D && diag; ++j)
            if (i != j && o.R[i][j] != 0) diag = false;
        if (!diag) continue;
        if (floor_mod(o.t[d], 2) != 0 || floor_mod(o.R[d][d] + o.t[d], 2) != 1) { ok = false; break; }
      }
      if (ok) split.push_back(d);
    }
    bool all_small = true;
    for (int d = 0; d < D; ++d) all_small = all_small && cN[d] <= 1;
    if (split.empty() || all_small) { nodes[id].leaf = true; continue; }
    const int nsec = 1 << split.size();
    std::vector<std::array<int, 3>> par(nsec);
    for (int bits = 0; bits < nsec; ++bits) {
      par[bits] = {0, 0, 0};
      for (size_t k = 0; k < split.size(); ++k) par[bits][split[k]] = (bits >> k) & 1;
    }
    auto in_split = [&](int d) { return std::find(split.begin(), split.end(), d) != split.end(); };
    // half-grid-shifted translations (shift_ops_half_grid, src/fractal_krfft.jl:262-283)
    std::vector<std::array<long, 3>> tsh(ops.size());
    for (size_t k = 0; k < ops.size(); ++k)
      for (int d = 0; d < 3; ++d) {
        if (d >= D) { tsh[k][d] = 0; continue; }
        long x2 = 2 * ops[k].t[d];
        for (int j = 0; j < D; ++j) x2 += (d == j ? 1 : 0) - ops[k].R[d][j];
        tsh[k][d] = round_half_even_twice(floor_mod(x2, 2L * cN[d]));
      }
    auto image = [&](size_t k, const std::array<int, 3>& p, int* img) {
      for (int d = 0; d < D; ++d) {
        long s = tsh[k][d];
        for (int j = 0; j < D; ++j) s += static_cast<long>(ops[k].R[d][j]) * p[j];
        img[d] = static_cast<int>(floor_mod(s, 2));
      }
    };
    // sector orbits (find_sector_orbits, src/fractal_krfft.jl:203-250)
    auto sector_of = [&](const int* img) {
      int bits = 0;
      for (size_t k = 0; k < split.size(); ++k) bits |= img[split[k]] << k;
      return bits;
    };
    std::vector<int> orbit_rep(nsec);
    std::vector<char> visited(nsec, 0);
    for (int i = 0; i < nsec; ++i) orbit_rep[i] = i;
    for (int i = 0; i < nsec; ++i) {
      if (visited[i]) continue;
      visited[i] = 1;
      for (size_t k = 0; k < ops.size(); ++k) {
        int img[3] = {0, 0, 0};
        image(k, par[i], img);
        const int j = sector_of(img);  // non-split dimensions are ignored
        if (!visited[j]) { visited[j] = 1; orbit_rep[j] = i; }
      }
    }
    std::vector<int> reps(orbit_rep.begin(), orbit_rep.end());
    std::sort(reps.begin(), reps.end());
    reps.erase(std::unique(reps.begin(), reps.end()), reps.end());
    int S[3];
    for (int d = 0; d < 3; ++d) S[d] = in_split(d) ? 2 : 1;
    for (int ri : reps) {
      const auto& p = par[ri];
      TreeNode c;
      for (int d = 0; d < 3; ++d) {
        c.n[d] = in_split(d) ? cN[d] / 2 : cN[d];
        c.scale[d] = nodes[id].scale[d] * S[d];
        c.offset[d] = nodes[id].scale[d] * p[d] + nodes[id].offset[d];
      }
      for (size_t k = 0; k < ops.size(); ++k) {
        int img[3] = {0, 0, 0};
        image(k, p, img);
        bool self = true;
        for (int d : split) self = self && img[d] == p[d];
        if (!self) continue;
        TreeOp o{};
        bool valid = true;
        for (int i = 0; i < 3 && valid; ++i) {
          for (int j = 0; j < 3; ++j) {
            const long rv = static_cast<long>(ops[k].R[i][j]) * S[j];
            if (rv % S[i] != 0) { valid = false; break; }
            o.R[i][j] = static_cast<int>(rv / S[i]);
          }
          if (!valid || i >= D) { o.t[i] = 0; continue; }
          long tv = (child_shifted_t ? tsh[k][i] : ops[k].t[i]) - p[i];
          for (int j = 0; j < D; ++j) tv += static_cast<long>(ops[k].R[i][j]) * p[j];
          if (tv % S[i] != 0) { valid = false; break; }
          o.t[i] = tv / S[i];
        }
        if (!valid) continue;
        bool dup = false;  // _deduplicate_ops: exact (R, t)
        for (const auto& e : c.ops) {
          bool same = true;
          for (int i = 0; i < 3 && same; ++i) {
            same = e.t[i] == o.t[i];
            for (int j = 0; j < 3 && same; ++j) same = e.R[i][j] == o.R[i][j];
          }
          if (same) { dup = true; break; }
        }
        if (!dup) c.ops.push_back(o);
      }
      c.depth = nodes[id].depth + 1;
      nodes.push_back(std::move(c));
      const int cid = static_cast<int>(nodes.size()) - 1;
      nodes[id].children.push_back(cid);
      stack.push_back(cid);
    }
  }
  // collect_leaves: depth first, children in order
  leaves->clear();
  *n_inner = 0;
  std::vector<int> order{0};
  while (!order.empty()) {
    const int id = order.back();
    order.pop_back();
    const TreeNode& nd = nodes[id];
    if (nd.leaf) {
      TreeLeaf l{};
      for (int d = 0; d < 3; ++d) { l.n[d] = nd.n[d]; l.scale[d] = nd.scale[d]; l.offset[d] = nd.offset[d]; }
      l.depth = nd.depth;
      leaves->push_back(l);
      continue;
    }
    ++*n_inner;
    for (auto it = nd.children.rbegin(); it != nd.children.rend(); ++it) order.push_back(*it);
  }
}

}  // namespace cfft

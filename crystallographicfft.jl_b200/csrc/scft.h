// SCFT driver (AB diblock melt) on a KRFFT plan: see scft.cu.
#pragma once

#include <string>

#include "exec.h"

namespace cfft {

constexpr int kScftMaxHistory = 32;

struct ScftParams {
  double f = 0.4;             // A-block fraction
  double chiN = 20.0;         // Flory-Huggins parameter times N
  int Ns = 100;               // contour steps (the plan's ds must be 1 / Ns)
  int history = 20;           // Anderson history depth
  double tol = 1e-6;          // stop when the relative residual is below tol
  int max_iter = 1000;
  double lam_simple = 0.1;    // simple-mixing step while err > anderson_start
  double lam_anderson = 1.0;  // Anderson mixing step
  double anderson_start = 0.2;
  int min_simple = 0;         // simple-mixing iterations before Anderson mixing may start
};

struct ScftState {
  double Q = 0, F = 0, err = 0;
  int iterations = 0;
  int converged = 0;
};

struct Scft;
Status scft_create(Plan* p, const ScftParams& prm, Scft** out, std::string* err);
void scft_destroy(Scft* s);
// Propagators, densities, residual, Q and F of the fields w = [w_A | w_B] (2 x M-grid);
// phi (2 x M-grid) and d (2 x M-grid) may be null.  Synchronises the stream.
Status scft_evaluate(Scft* s, const void* w, void* phi, void* d, ScftState* out, void* stream, std::string* err);
// Iterates from w (in/out) until err < tol or max_iter iterations; one stream
// synchronisation per iteration (the convergence test).
Status scft_solve(Scft* s, void* w, ScftState* out, void* stream, std::string* err);
// Densities of the last evaluation (2 x M-grid, device).
Status scft_densities(const Scft* s, void* phi, void* stream, std::string* err);

}  // namespace cfft

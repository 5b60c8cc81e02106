// Device-resident restarted GMRES (left preconditioned), restating
// jax.scipy.sparse.linalg.gmres as called at steppers.py:466 / :476.
#pragma once

#include "sisl_core.cuh"

namespace sisl {

constexpr int GM_MAXR = 128;     // largest supported restart (Krylov) dimension
constexpr int GM_MAXBLOCKS = 1184;  // 8 * 148 SMs: reduction partials per kernel

// Scalars and small dense matrices of one solve, all float64, in workspace.
struct GState {
  double h[GM_MAXR + 2];            // projections of the new vector (scaled)
  double s[GM_MAXR + 2];            // inverse norms of the stored basis vectors
  double H[GM_MAXR][GM_MAXR + 1];   // Hessenberg rows (batched) or rotated R rows (incremental)
  double givens[GM_MAXR][2];
  double beta[GM_MAXR + 1];
  double coef[GM_MAXR + 2];         // coefficients of the pending multi-axpy
  double hn0;                       // ||M A v_j|| before orthogonalisation
  double bnorm, mbnorm, rnorm, atol, ptol, tol, atol_in, eps;
  double err;                       // incremental residual estimate
  int active;                       // 1 while the current cycle continues
  int kdone;                        // Arnoldi steps taken in the current cycle
  int restart;
  int method;                       // 0 batched, 1 incremental
  int breakdown;
  unsigned int counter;             // last-block-done ticket
  int cycles, steps;                // restart cycles and Arnoldi steps taken (graph mode)
};

// Per-solve statistics written on the device in graph mode; the same layout
// as SislSolveInfo.
struct GDevInfo {
  int32_t cycles, arnoldi_steps, converged, pad;
  double residual_norm, atol, b_norm;
};

// Host-visible summary copied back once per restart cycle.
struct GHostView {
  double rnorm, atol, bnorm;
  int kdone;
  int pad;
};

}  // namespace sisl

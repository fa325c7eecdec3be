// Device-resident data layout of a registration batch.
//
// A context holds P independent pairs (source landmarks + target varifold).  All
// pairs share the dimension D, the deformation kernel family and the varifold
// kernel types (template parameters of the kernels) and the number of time
// points; sizes, widths and weights are per pair.
//
// Point-indexed arrays concatenate the pairs' points, each pair padded to a
// multiple of kTile with zero-weight points (alpha = 0, area = 0), so the all-pairs
// loops need no bounds checks: a padded j contributes exactly zero.
//
// FP64 optimisation vectors (alpha, gradient, L-BFGS history) concatenate the
// pairs' unpadded variables in the reference's C++ layout: coordinate fastest,
// then node, then time step (Cpp/src/objgrd.cpp:47-50).
#pragma once

#include <cstdint>

namespace lddmm {

constexpr int kMaxMem = 32;  // largest L-BFGS memory (optdata.memNum) supported

struct PairDesc {
  int N, Npad;        // landmarks; padded count (multiple of kTile)
  int Ed, Edpad;      // deformed elements (segments / triangles)
  int Et, Etpad;      // target elements
  int pt_off;         // first point in point arrays
  int el_off;         // first deformed element in element arrays
  int tg_off;         // first target element in target arrays
  int itile_off;      // first 64-row i-tile of this pair (per-step sweep partials)
  int grp_off;        // first 8-row group of this pair (persistent sweep partials)
  int etile_off;      // first element tile of this pair (varifold partials)
  int adj_off;        // first entry of this pair's vertex CSR pointer array
  int chunk_off, nchunk;  // vector-pass chunks of this pair
  long long var_off;  // first FP64 variable
  long long var_num;  // D * N * T
  float kscale;       // coordinate scale of the deformation kernel (ex2 argument)
  float cscale;       // centre scale of the varifold centre kernel
  double dt;          // time step
  double dis_wgt;     // varifold weight
  double pd_fac;      // dq factor: pdot = pd_fac * sum(lr * W * dq_scaled)
  double dc_fac;      // varifold dc factor (without the 2 a_i): -2 / (sigma_W^2 * cscale)
  double tt;          // target self-term, FP64, computed once
};

// L-BFGS + line-search state of one pair (FP64 scalars), after Cpp/src/LBFGS.cpp
// and Cpp/src/lineSearch.cpp.
enum Phase : int {
  kPhaseInit = 0,    // initial point pending evaluation
  kPhaseLS = 1,      // a line-search trial point pending evaluation
  kPhaseDone = 2,    // converged or iteration budget exhausted
  kPhaseFailed = 3,  // line search failed (status 1/2/3) or non-finite values
};

enum Action : int { kActNone = 0, kActAcceptInit = 1, kActAccept = 2 };

struct PairState {
  double f;        // objective at the current point
  double f_try;    // objective at the trial point
  double glen;     // |g| at the current point
  double f_prev;   // objective before the last accepted step
  double t, relL, relR;  // line search: relative step and bracket
  double slp, dlen;      // g.d and |d| of the current direction
  double H0;             // initial inverse Hessian scale s.y / y.y
  double stp;            // last accepted step length (t * |d|)
  int bisMax, epdMax, bisCnt, epdCnt, objCnt;
  int newIdx, hisNum, itr;
  int phase, status, action, need_dir;
  int evals, iters;
  int active;            // evaluate this pair in the next objective sweep
  int pad_;
};

struct OptParams {
  int itr_max;
  int mem_num;
  double tol;
  double wolfe1, wolfe2;
  double rel_obj_tol;    // stop when |f_prev - f| <= rel_obj_tol * |f_prev| (0: off)
  int rec_cap;           // per-pair iteration records kept (0: none)
};

}  // namespace lddmm

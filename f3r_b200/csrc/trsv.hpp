// trsv.hpp -- Jacobi-iteration triangular solves on SELL-32 (trsv.cu).
//
// The reference's alternatives to an exact triangular solve
// (umineko-sparse/trsv/jacobi.hpp:290-505 and trsv/baj.hpp:95-190): instead
// of a sequential sweep, a few fully parallel sweeps of
//   Jacobi  y0 = om D^-1 in;   y <- om D^-1 (in - N y) + (1 - om) y
//   BAJ     y  = D^-1 in;      y <- D^-1 (in - N y), in place
// with N the strictly triangular part.  Each sweep is one SpMV over N, which
// on the GPU is the TMA-fed SELL kernel with a Jacobi epilogue; the BAJ sweep
// updates the vector in place (a row may read values another warp already
// replaced in this sweep, as in the reference), so its intermediate results
// depend on scheduling and only its fixed point is deterministic.
#pragma once

#include <vector>

#include "objects.cuh"

namespace f3r {

enum TrsvForm : int { FORM_LOWER = 0, FORM_LOWER_D = 1, FORM_D_UPPER = 2 };
enum TrsvKind : int { TRSV_JACOBI = 0, TRSV_BAJ = 1 };

struct JacobiTrsv {
  DeviceSell off;             // N in the vector order, fp16 values, original column order per row
  __half *dinv = nullptr;     // fp16(1 / d_ii) by vector position; nullptr for FORM_LOWER
  __half *tmp = nullptr;      // second buffer of the synchronous sweeps
  int32_t n = 0, form = FORM_LOWER, kind = TRSV_JACOBI, iters = 0;
  double omega = 1.0;
  bool reverse = false;       // BAJ: visit slices from the bottom (D_UPPER)

  // M: the triangular factor in its stored form (CSR, original numbering);
  // perm (nullable): vector position -> original row
  Status build(Context &c, const HostCSR &M, int form_, int kind_, int32_t iters_, double omega_,
               const std::vector<int32_t> *perm);
  // out = the approximate M^-1 in (fp16 device vectors, in distinct from out);
  // ome (nullable, device): the result is multiplied by *ome, rounded again
  Status apply(Context &c, const __half *in, __half *out, const __half *ome);
  void release();
};

// Raises the shared-memory limit of the sweep kernel (before graph capture).
Status jacobi_trsv_prepare(Context &c);

}  // namespace f3r

struct f3r_trsv {
  f3r_context *ctx = nullptr;
  f3r::JacobiTrsv t;
};

// Brick-tiled multigrid / CG kernels (pr_mg.cu).
#pragma once

#include <cmath>

#include "pr_ops.cuh"

namespace pr {

// Galerkin operator of one multigrid level: interior constants and the 8 x 27 table of
// low-face coefficients (mask bit a set = node index 0 on axis a), FP64 on the host.
struct LevelCoef {
  uint32_t depth = 0;
  double shift = 0.0;
  double c0 = 0, ce = 0, cc = 0, cf = 0;
  double table[8][27];
  bool has_faces = false;
};

// Level l of a hierarchy whose finest depth is D; shift_l is added to the diagonal.
LevelCoef level_coef(uint32_t D, uint32_t l, double shift_l);

// Every launch below takes `clouds`: packed vectors of that many independent systems of the same
// level (cloud k's slice of a level-l vector at k 8^l, of the per-block partials at k mg_blocks),
// one launch for all of them.

// One smoothing sweep over all blocks of the level, out of place.  mode 0: xo = sweep(xi);
// 1: xo = sweep(0) (xi unused); 2: xo = sweep(xi + P ec).  part (nullable): per-block f.xo
// (mg_blocks entries).
template <typename T>
void mg_smooth(cudaStream_t s, const LevelCoef& L, const T* table, const T* xi, T* xo, const T* f, const T* ec,
               int mode, bool forward, double* part, uint32_t clouds = 1);
// CG update x += alpha d, r -= alpha q (in place) fused with the first pre-smoothing sweep from
// zero of the finest level (depth >= 4): xo = sweep(0) on the new r; part = per-block r.r
template <typename T>
struct CgFuse {
  T* x = nullptr;
  const T* d = nullptr;
  const T* q = nullptr;
  T* r = nullptr;
  T alpha = 0;
  const double* alpha_dev = nullptr;  // packed launches: per-cloud alpha in place of `alpha`
};
template <typename T>
void mg_cg_update_presmooth(cudaStream_t s, const LevelCoef& L, const T* table, const CgFuse<T>& cg, T* xo,
                            double* part, uint32_t clouds = 1);
// fc = P^T (f - A_l e); face: scratch of mg_face_entries(depth) values per cloud (levels >= 4)
template <typename T>
void mg_resid_restrict(cudaStream_t s, const LevelCoef& L, const T* table, const T* e, const T* f, T* fc, T* face,
                       uint32_t clouds = 1);
size_t mg_face_entries(uint32_t depth);
// finest level only.  xpby: dn = z + beta d, q = A dn; else q = A d.  Stencil part only;
// per-block (dn or d).q into part.  beta_dev (packed, nullable): per-cloud beta.
template <typename T>
void mg_spmv(cudaStream_t s, const LevelCoef& L, const T* table, const T* z, const T* d, T* dn, double beta,
             bool xpby, T* q, double* part, uint32_t clouds = 1, const double* beta_dev = nullptr);
uint32_t mg_blocks(uint32_t depth);
// finest level (depth >= 4), FP64: xn = x + scale * e (e: correction, float or double),
// r = b - K xn (stencil part; the screening is applied separately).  x, xn: distinct buffers.
// scale_dev (packed, nullable): per-cloud scale.
template <typename E>
void mg_resid_update(cudaStream_t s, const LevelCoef& L, const double* x, const E* e, double scale, double* xn,
                     const double* b, double* r, uint32_t clouds = 1, const double* scale_dev = nullptr);
// out = sum(part[0:np]) + scale2 * sum(part2[0:np2]), fixed order; per cloud (cloud k's partials
// at k np and k np2, its sum at out[k])
void sum_parts(cudaStream_t s, const double* part, int np, double scale2, const double* part2, int np2, double* out,
               uint32_t clouds = 1);

// The z-segment choices of the 16^3 block kernels made so far in this process (one line per
// kernel family, level and launch size, with the timings).
std::string autotune_log();

// Time `reps` launches of one kernel (ids: 0 spmv, 1 spmv+xpby, 2 smooth from zero,
// 3 smooth, 4 smooth+prolongation+dot, 5 residual+restriction, 6 per-node stencil) at
// depth D on context-owned buffers; returns ms per launch and the algorithmic bytes.
double kernel_bench(pr_context* c, int kid, uint32_t D, int precision, int reps, double* bytes);

}  // namespace pr

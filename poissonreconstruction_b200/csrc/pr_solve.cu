// Solve stage: the crate's fine system A x = b (src/fem_tree.rs:180-299) solved to a
// relative FP64 residual ||b - A x|| / ||b||.
//
// The crate runs a two-level cascade of sequential Gauss-Seidel and plain CG
// (src/fem_tree.rs:458-487, src/solvers.rs:20-69,164-175) and stops it far from
// convergence.  Its fine system is SPD, so its solution is unique: here it is reached with
// CG preconditioned by a geometric multigrid V-cycle, in two precisions:
//   * FP64: preconditioned CG in FP64 throughout;
//   * mixed: preconditioned CG in FP32 (operator, vectors and V-cycle in FP32) inside an
//     FP64 iterative-refinement loop: r = b - A x is formed in FP64, scaled to unit norm,
//     solved approximately in FP32, and the correction is added to the FP64 x.
// The V-cycle works on the constant-coefficient stencil A' = K + wg I of every depth
// (rediscretised: the Galerkin coarse stiffness of nested trilinear spaces), relaxed with
// multicolour block Gauss-Seidel (forward before, backward after the coarse correction, so
// the preconditioner is symmetric), coarsest level 4^3 solved with a dense inverse.  The
// per-point screening terms are in A but not in A' (they are below 1e-5 of the stiffness
// diagonal at depth >= 8 and only slow convergence, never prevent it).
#include <cmath>
#include <cstdio>
#include <vector>

#include "pr_ops.cuh"

namespace pr {

namespace {

constexpr uint32_t kCoarseDepth = 2;

// Dense inverse of the constant stencil at depth Dc (Morton order), FP64 Cholesky.
std::vector<double> dense_inverse(uint32_t Dc, const Coef<double>& c) {
  const int res = 1 << Dc;
  const int n = res * res * res;
  std::vector<double> A((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) {
    uint32_t ix, iy, iz;
    unmorton3((uint32_t)i, ix, iy, iz);
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          int jx = (int)ix + dx, jy = (int)iy + dy, jz = (int)iz + dz;
          if (jx < 0 || jx >= res || jy < 0 || jy >= res || jz < 0 || jz >= res) continue;
          int nz = (dx != 0) + (dy != 0) + (dz != 0);
          double v = nz == 0 ? c.c0 : (nz == 2 ? c.ce : (nz == 3 ? c.cc : 0.0));
          A[(size_t)i * n + morton3(jx, jy, jz)] = v;
        }
  }
  // Cholesky A = L L^T (lower, in place)
  for (int j = 0; j < n; ++j) {
    double d = A[(size_t)j * n + j];
    for (int k = 0; k < j; ++k) d -= A[(size_t)j * n + k] * A[(size_t)j * n + k];
    if (!(d > 0.0)) throw Error(PR_ERR_INTERNAL, "coarse operator is not positive definite");
    d = std::sqrt(d);
    A[(size_t)j * n + j] = d;
    for (int i = j + 1; i < n; ++i) {
      double s = A[(size_t)i * n + j];
      for (int k = 0; k < j; ++k) s -= A[(size_t)i * n + k] * A[(size_t)j * n + k];
      A[(size_t)i * n + j] = s / d;
    }
  }
  // inverse column by column: solve L L^T x = e_c
  std::vector<double> inv((size_t)n * n), y(n);
  for (int col = 0; col < n; ++col) {
    for (int i = 0; i < n; ++i) {
      double s = (i == col) ? 1.0 : 0.0;
      for (int k = 0; k < i; ++k) s -= A[(size_t)i * n + k] * y[k];
      y[i] = s / A[(size_t)i * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {
      double s = y[i];
      for (int k = i + 1; k < n; ++k) s -= A[(size_t)k * n + i] * inv[(size_t)k * n + col];
      inv[(size_t)i * n + col] = s / A[(size_t)i * n + i];
    }
  }
  return inv;
}

// Multigrid V-cycle preconditioner on A' (constant stencil per depth)
template <typename T>
struct Multigrid {
  pr_context* c = nullptr;
  uint32_t D = 0, Dc = 0;
  int sweeps = 1;
  std::vector<Coef<T>> coef;
  std::vector<T*> f, e, r;
  T* inv = nullptr;
  uint32_t nc = 0;

  void init(pr_context* ctx, uint32_t depth, double wg, int nsweeps) {
    c = ctx;
    D = depth;
    Dc = std::min<uint32_t>(D, kCoarseDepth);
    sweeps = std::max(1, nsweeps);
    coef.assign(D + 1, Coef<T>{});
    f.assign(D + 1, nullptr);
    e.assign(D + 1, nullptr);
    r.assign(D + 1, nullptr);
    for (uint32_t l = Dc; l <= D; ++l) {
      double shift = wg * std::pow(8.0, (double)(D - l));
      coef[l] = cast_coef<T>(stencil_coef(l, shift));
      uint64_t nl = 1ull << (3 * l);
      std::string sfx = std::string("_") + tname<T>() + "_" + std::to_string(l);
      if (l < D) {
        f[l] = c->buf<T>("mg_f" + sfx, nl);
        e[l] = c->buf<T>("mg_e" + sfx, nl);
      }
      if (l > Dc) r[l] = c->buf<T>("mg_r" + sfx, nl);
    }
    nc = 1u << (3 * Dc);
    std::vector<double> invd = dense_inverse(Dc, stencil_coef(Dc, wg * std::pow(8.0, (double)(D - Dc))));
    std::vector<T> invt(invd.begin(), invd.end());
    inv = c->buf<T>(std::string("mg_inv_") + tname<T>(), invt.size());
    PR_CUDA(cudaMemcpyAsync(inv, invt.data(), invt.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream));
    c->sync();  // invt is a host temporary
  }

  void vcycle(uint32_t l, const T* fl, T* el) {
    cudaStream_t s = c->stream;
    if (l == Dc) {
      dense_solve<T>(s, nc, inv, fl, el);
      return;
    }
    const uint64_t nl = 1ull << (3 * l);
    PR_CUDA(cudaMemsetAsync(el, 0, nl * sizeof(T), s));
    for (int k = 0; k < sweeps; ++k) gs_sweep<T>(s, l, el, fl, coef[l], true);
    stencil_apply<T>(s, l, el, fl, r[l], coef[l], 1);
    restrict_to_coarse<T>(s, l, r[l], f[l - 1]);
    vcycle(l - 1, f[l - 1], e[l - 1]);
    prolong_add<T>(s, l, e[l - 1], el);
    for (int k = 0; k < sweeps; ++k) gs_sweep<T>(s, l, el, fl, coef[l], false);
  }
  void apply(const T* rhs, T* z) { vcycle(D, rhs, z); }
};

struct PcgResult {
  int iters = 0;
  double rr = 0.0;
  bool broke = false;
};

// Preconditioned CG from x = 0 on A x = b, until ||r|| <= tol_abs or maxit iterations.
template <typename T>
PcgResult pcg(pr_context* c, const FineOp<T>& A, Multigrid<T>& M, const T* b, T* x, double tol_abs, int maxit) {
  const uint64_t n = c->n;
  cudaStream_t s = c->stream;
  std::string t = tname<T>();
  T* r = c->buf<T>("cg_r_" + t, n);
  T* z = c->buf<T>("cg_z_" + t, n);
  T* d = c->buf<T>("cg_d_" + t, n);
  T* q = c->buf<T>("cg_q_" + t, n);
  PcgResult res;
  PR_CUDA(cudaMemsetAsync(x, 0, n * sizeof(T), s));
  PR_CUDA(cudaMemcpyAsync(r, b, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
  double rr = dot<T>(c, r, r, n);
  res.rr = rr;
  if (!(std::sqrt(rr) > tol_abs) || maxit <= 0) return res;
  M.apply(r, z);
  PR_CUDA(cudaMemcpyAsync(d, z, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
  double rz = dot<T>(c, r, z, n);
  for (int it = 0; it < maxit; ++it) {
    A.apply(s, d, q);
    double dq = dot<T>(c, d, q, n);
    if (!(dq > 0.0) || !std::isfinite(dq) || !(rz > 0.0)) {
      res.broke = true;
      break;
    }
    double alpha = rz / dq;
    rr = cg_update<T>(c, n, alpha, d, q, x, r);
    res.iters = it + 1;
    res.rr = rr;
    if (!std::isfinite(rr)) {
      res.broke = true;
      break;
    }
    if (std::sqrt(rr) <= tol_abs) break;
    M.apply(r, z);
    double rz_new = dot<T>(c, r, z, n);
    double beta = rz_new / rz;
    rz = rz_new;
    xpby<T>(s, n, z, beta, d);
  }
  return res;
}

// Algorithmic HBM bytes of one PCG iteration / V-cycle (element size es), used for the
// solve GB/s figure: SpMV reads x writes y; CG update reads x,d,r,q writes x,r; xpby reads
// z,d writes d; two dot products read 2 vectors each; the V-cycle per level l: 2 GS sweeps
// (read x,f write x), residual (read e,f write r), restriction (read r, write 1/8),
// prolongation (read 1/8 + e, write e).
double iter_bytes(uint64_t n, double es, uint64_t pin, double pes) {
  double spmv = 2.0 * n * es + pin * (8.0 * pes + 8.0 * 4.0) * 2.0;
  double upd = 6.0 * n * es, xp = 3.0 * n * es, dots = 4.0 * n * es;
  return spmv + upd + xp + dots;
}
double vcycle_bytes(uint32_t D, double es, int sweeps) {
  double b = 0.0;
  for (uint32_t l = 3; l <= D; ++l) {
    double nl = (double)(1ull << (3 * l));
    b += nl * es * (2.0 * sweeps * 3.0 + 3.0 + 1.125 + 2.125);
  }
  return b;
}

}  // namespace

void stage_solve(pr_context* c, const pr_params& p, pr_stats& st) {
  const uint64_t n = c->n;
  cudaStream_t s = c->stream;
  const double h = 1.0 / (double)(1u << c->D);
  const double wg = c->pw > 0.0 ? (c->pw * (h * h * h) / 1.5) * 0.005 : 0.0;
  const double* b = c->get<double>("b64");
  double* x = c->buf<double>("x64", n);
  double* r = c->buf<double>("r64", n);
  const double target = p.target_rel_residual > 0.0 ? p.target_rel_residual : 1e-6;
  const int max_iters = p.max_iters > 0 ? (int)p.max_iters : 200;
  const int sweeps = p.smooth_sweeps > 0 ? (int)p.smooth_sweeps : 1;

  st.pcg_iterations = 0;
  st.refinement_steps = 0;
  st.solve_bytes = 0.0;
  PR_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), s));
  double bn = std::sqrt(dot<double>(c, b, b, n));
  if (bn == 0.0) {
    st.rel_residual = 0.0;
    st.converged = 1;
    c->have_coeffs = true;
    return;
  }
  FineOp<double> A64 = make_fine_op<double>(c, wg);
  PR_CUDA(cudaMemcpyAsync(r, b, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  double rn = bn;
  int used = 0;
  const bool mixed = p.precision != PR_PRECISION_FP64;
  const double es = mixed ? 4.0 : 8.0;
  const double per_iter = iter_bytes(n, es, c->P_in, es) + vcycle_bytes(c->D, es, sweeps);

  if (mixed) {
    FineOp<float> A32 = make_fine_op<float>(c, wg);
    Multigrid<float> M32;
    M32.init(c, c->D, wg, sweeps);
    float* r32 = c->buf<float>("r32", n);
    float* e32 = c->buf<float>("e32", n);
    const double inner = p.inner_rel_tol > 0.0 ? p.inner_rel_tol : 1e-4;
    while (rn > target * bn && used < max_iters) {
      scale_convert<double, float>(s, n, 1.0 / rn, r, r32);
      double tol = std::max(inner, 0.5 * target * bn / rn);
      PcgResult pr_ = pcg<float>(c, A32, M32, r32, e32, tol, max_iters - used);
      used += pr_.iters;
      axpy<float, double>(s, n, rn, e32, x);
      A64.residual(s, x, b, r);
      double rn_new = std::sqrt(dot<double>(c, r, r, n));
      st.refinement_steps++;
      st.solve_bytes += pr_.iters * per_iter + 2.0 * n * 4.0 + 2.0 * n * 8.0 /*convert, axpy*/ +
                        (3.0 * n * 8.0 + c->P_in * 2.0 * (8.0 * 8.0 + 32.0)) /*FP64 residual*/ + 2.0 * n * 8.0;
      if (pr_.iters == 0 || !(rn_new < rn)) {  // no progress: stop
        rn = rn_new;
        break;
      }
      rn = rn_new;
    }
  } else {
    Multigrid<double> M64;
    M64.init(c, c->D, wg, sweeps);
    double* e64 = c->buf<double>("e64", n);
    while (rn > target * bn && used < max_iters) {
      double tol = 0.5 * target * bn;  // absolute, on the current residual system
      PcgResult pr_ = pcg<double>(c, A64, M64, r, e64, tol, max_iters - used);
      used += pr_.iters;
      axpy<double, double>(s, n, 1.0, e64, x);
      A64.residual(s, x, b, r);
      double rn_new = std::sqrt(dot<double>(c, r, r, n));
      st.refinement_steps++;
      st.solve_bytes += pr_.iters * per_iter + 3.0 * n * 8.0 + (3.0 * n * 8.0 + c->P_in * 2.0 * (8.0 * 8.0 + 32.0)) +
                        2.0 * n * 8.0;
      if (pr_.iters == 0 || !(rn_new < rn)) {
        rn = rn_new;
        break;
      }
      rn = rn_new;
    }
  }
  st.pcg_iterations = (uint32_t)used;
  st.rel_residual = rn / bn;
  st.converged = st.rel_residual <= target ? 1 : 0;
  c->have_coeffs = true;
}

// ------------------------------------------------------------------ operator access for tests
void apply_operator64(pr_context* c, const double* d_x, double* d_y) {
  const double h = 1.0 / (double)(1u << c->D);
  const double wg = c->pw > 0.0 ? (c->pw * (h * h * h) / 1.5) * 0.005 : 0.0;
  make_fine_op<double>(c, wg).apply(c->stream, d_x, d_y);
}
void apply_operator32(pr_context* c, const float* d_x, float* d_y) {
  const double h = 1.0 / (double)(1u << c->D);
  const double wg = c->pw > 0.0 ? (c->pw * (h * h * h) / 1.5) * 0.005 : 0.0;
  make_fine_op<float>(c, wg).apply(c->stream, d_x, d_y);
}

}  // namespace pr

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
// The V-cycle works on A' = K + wg I and its exact Galerkin coarse operators (P^T A' P for
// the linear B-spline prolongation P), relaxed with multicolour Gauss-Seidel inside
// 8^3 / 16^3 blocks (forward before, backward after the coarse correction, so the
// preconditioner is symmetric); the coarsest level, 4^3, is solved with a dense inverse.
// The per-point screening terms are in A but not in A' (below 1e-5 of the stiffness
// diagonal at depth >= 8; they only slow convergence, never prevent it).
#include <cmath>
#include <cstdio>
#include <vector>

#include "pr_mg.cuh"

namespace pr {

namespace {

constexpr uint32_t kCoarseDepth = 2;

// Dense inverse of a level's Galerkin operator (depth Dc <= 2, Morton order), FP64 Cholesky.
std::vector<double> dense_inverse(const LevelCoef& L) {
  const uint32_t Dc = L.depth;
  const int res = 1 << Dc;
  const int n = res * res * res;
  std::vector<double> A((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) {
    uint32_t ix, iy, iz;
    unmorton3((uint32_t)i, ix, iy, iz);
    int mask = L.has_faces ? ((ix == 0) | ((iy == 0) << 1) | ((iz == 0) << 2)) : 0;
    for (int o = 0; o < 27; ++o) {
      int dx = o % 3 - 1, dy = (o / 3) % 3 - 1, dz = o / 9 - 1;
      int jx = (int)ix + dx, jy = (int)iy + dy, jz = (int)iz + dz;
      if (jx < 0 || jx >= res || jy < 0 || jy >= res || jz < 0 || jz >= res) continue;
      A[(size_t)i * n + morton3(jx, jy, jz)] = L.table[mask][o];
    }
  }
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

// Multigrid V-cycle preconditioner on A' = K + wg I with Galerkin coarse levels.
// Level l holds f_l (right-hand side), a_l (after pre-smoothing) and e_l (result);
// sweeps beyond the first ping-pong through t_l.
template <typename T>
struct Multigrid {
  pr_context* c = nullptr;
  uint32_t D = 0, Dc = 0;
  int sweeps = 1;
  std::vector<LevelCoef> L;
  std::vector<T*> f, a, e, t, face;
  T* tables = nullptr;  // [D+1][8*27]
  T* inv = nullptr;
  uint32_t nc = 0;

  void init(pr_context* ctx, uint32_t depth, double wg, int nsweeps) {
    c = ctx;
    D = depth;
    Dc = std::min<uint32_t>(D, kCoarseDepth);
    sweeps = std::max(1, nsweeps);
    L.assign(D + 1, LevelCoef());
    f.assign(D + 1, nullptr);
    a.assign(D + 1, nullptr);
    e.assign(D + 1, nullptr);
    t.assign(D + 1, nullptr);
    face.assign(D + 1, nullptr);
    std::vector<T> tab((size_t)(D + 1) * 216, (T)0);
    for (uint32_t l = Dc; l <= D; ++l) {
      L[l] = level_coef(D, l, wg * std::pow(8.0, (double)(D - l)));
      for (int m = 0; m < 8; ++m)
        for (int o = 0; o < 27; ++o) tab[(size_t)l * 216 + 27 * m + o] = (T)L[l].table[m][o];
      const uint64_t nl = 1ull << (3 * l);
      const std::string sfx = std::string("_") + tname<T>() + "_" + std::to_string(l);
      if (l < D) {
        f[l] = c->buf<T>("mg_f" + sfx, nl);
        e[l] = c->buf<T>("mg_e" + sfx, nl);
      }
      if (l > Dc) {
        a[l] = c->buf<T>("mg_a" + sfx, nl);
        if (mg_face_entries(l)) face[l] = c->buf<T>("mg_face" + sfx, mg_face_entries(l));
        if (sweeps > 1) t[l] = c->buf<T>("mg_t" + sfx, nl);
      }
    }
    tables = c->buf<T>(std::string("mg_tab_") + tname<T>(), tab.size());
    nc = 1u << (3 * Dc);
    std::vector<double> invd = dense_inverse(L[Dc]);
    std::vector<T> invt(invd.begin(), invd.end());
    inv = c->buf<T>(std::string("mg_inv_") + tname<T>(), invt.size());
    PR_CUDA(cudaMemcpyAsync(tables, tab.data(), tab.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream));
    PR_CUDA(cudaMemcpyAsync(inv, invt.data(), invt.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream));
    c->sync();  // host temporaries
  }
  const T* table(uint32_t l) const { return tables + (size_t)l * 216; }

  // el = V(fl); at the finest level `part` (nullable) receives per-block fl.el partials.
  // presmoothed: the first pre-smoothing sweep of this level is already in a_l.
  void vcycle(uint32_t l, const T* fl, T* el, double* part, bool presmoothed = false) {
    cudaStream_t s = c->stream;
    if (l == Dc) {
      dense_solve<T>(s, nc, inv, fl, el);
      return;
    }
    // pre-smoothing (forward) from zero; result in a_l
    T* cur = a[l];
    if (!presmoothed) mg_smooth<T>(s, L[l], table(l), nullptr, cur, fl, nullptr, 1, true, nullptr);
    for (int k = 1; k < sweeps; ++k) {
      T* nxt = (cur == a[l]) ? t[l] : a[l];
      mg_smooth<T>(s, L[l], table(l), cur, nxt, fl, nullptr, 0, true, nullptr);
      cur = nxt;
    }
    mg_resid_restrict<T>(s, L[l], table(l), cur, fl, f[l - 1], face[l]);
    vcycle(l - 1, f[l - 1], e[l - 1], nullptr);
    // post-smoothing (backward): first sweep on cur + P e_{l-1}; the last sweep writes el
    for (int k = 0; k < sweeps; ++k) {
      const bool last = (k == sweeps - 1);
      T* nxt = last ? el : ((cur == a[l]) ? t[l] : a[l]);
      mg_smooth<T>(s, L[l], table(l), cur, nxt, fl, e[l - 1], k == 0 ? 2 : 0, false, last ? part : nullptr);
      cur = nxt;
    }
  }
  // The CG update can be fused with the first pre-smoothing sweep of the finest level.
  bool fuses_cg_update() const { return D >= 4 && D > Dc; }
  // x += alpha d, r -= alpha q, first pre-smoothing sweep of r into a_D; returns r.r
  double cg_update_presmooth(double alpha, const T* d, const T* q, T* x, T* r) {
    double* part = c->buf<double>("mg_part", mg_blocks(D));
    double* out = c->buf<double>("mg_out", 1);
    CgFuse<T> cg;
    cg.x = x;
    cg.d = d;
    cg.q = q;
    cg.r = r;
    cg.alpha = (T)alpha;
    mg_cg_update_presmooth<T>(c->stream, L[D], table(D), cg, a[D], part);
    sum_parts(c->stream, part, (int)mg_blocks(D), 0.0, part, 0, out);
    PR_CUDA(cudaMemcpyAsync(c->h_scalars, out, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    c->sync();
    return c->h_scalars[0];
  }
  // z = M r; returns r.z.  presmoothed: a_D already holds the first sweep on r.
  double apply(const T* r, T* z, bool presmoothed = false) {
    const uint64_t n = 1ull << (3 * D);
    if (D == Dc) {
      dense_solve<T>(c->stream, nc, inv, r, z);
      return dot<T>(c, r, z, n);
    }
    double* part = c->buf<double>("mg_part", mg_blocks(D));
    double* out = c->buf<double>("mg_out", 1);
    vcycle(D, r, z, part, presmoothed);
    sum_parts(c->stream, part, (int)mg_blocks(D), 0.0, part, 0, out);
    PR_CUDA(cudaMemcpyAsync(c->h_scalars, out, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    c->sync();
    return c->h_scalars[0];
  }
};

// Fine operator for CG: tiled stencil SpMV (optionally fused with dn = z + beta d) plus
// the per-point screening terms; returns dn.A dn from the fused partial sums.
template <typename T>
struct CgOperator {
  pr_context* c = nullptr;
  LevelCoef Lf;
  T* table = nullptr;
  Screen<T> scr;
  uint32_t D = 0;
  void init(pr_context* ctx, double wg) {
    c = ctx;
    D = c->D;
    Lf = level_coef(D, D, wg);
    std::vector<T> tab(216);
    for (int m = 0; m < 8; ++m)
      for (int o = 0; o < 27; ++o) tab[27 * m + o] = (T)Lf.table[m][o];
    table = c->buf<T>(std::string("cg_tab_") + tname<T>(), 216);
    PR_CUDA(cudaMemcpyAsync(table, tab.data(), 216 * sizeof(T), cudaMemcpyHostToDevice, c->stream));
    c->sync();
    scr = make_fine_op<T>(c, wg).scr;
  }
  // xpby: dn = z + beta d, q = A dn; else q = A d (dn unused).  Returns (dn or d).q
  double apply_dot(const T* z, const T* d, T* dn, double beta, bool xpby, T* q) {
    cudaStream_t s = c->stream;
    const uint64_t n = c->n;
    const T* dd = xpby ? dn : d;
    if (D < 3) {  // grids below one 8^3 block: per-node kernels
      if (xpby) {
        PR_CUDA(cudaMemcpyAsync(dn, d, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
        pr::xpby<T>(s, n, z, beta, dn);
      }
      stencil_apply<T>(s, D, dd, nullptr, q, cast_coef<T>(stencil_coef(D, Lf.shift)), 0);
      screen_apply<T>(s, scr, dd, q, +1);
      return dot<T>(c, dd, q, n);
    }
    double* part = c->buf<double>("cg_part", mg_blocks(D));
    double* part2 = c->buf<double>("cg_part2", kDotBlocks);
    double* out = c->buf<double>("cg_out", 1);
    mg_spmv<T>(s, Lf, table, z, d, dn, beta, xpby, q, part);
    int np2 = 0;
    if (scr.active()) {
      screen_project_sq<T>(s, scr, dd, part2, kDotBlocks);
      screen_gather<T>(s, scr, q, +1);
      np2 = kDotBlocks;
    }
    sum_parts(s, part, (int)mg_blocks(D), (double)scr.wh3, part2, np2, out);
    PR_CUDA(cudaMemcpyAsync(c->h_scalars, out, sizeof(double), cudaMemcpyDeviceToHost, s));
    c->sync();
    return c->h_scalars[0];
  }
};

struct PcgResult {
  int iters = 0;
  double rr = 0.0;
  bool broke = false;
};

// Preconditioned CG from x = 0 on A x = b, until ||r|| <= tol_abs or maxit iterations; rr0 = b . b
// when the caller knows it (else negative). The search direction ping-pongs between two buffers
// (the SpMV reads d with halos).
template <typename T>
PcgResult pcg(pr_context* c, CgOperator<T>& A, Multigrid<T>& M, const T* b, T* x, double tol_abs, int maxit,
              double rr0 = -1.0) {
  const uint64_t n = c->n;
  cudaStream_t s = c->stream;
  const std::string tn = tname<T>();
  T* r = c->buf<T>("cg_r_" + tn, n);
  T* z = c->buf<T>("cg_z_" + tn, n);
  T* dA = c->buf<T>("cg_d_" + tn, n);
  T* dB = c->buf<T>("cg_d2_" + tn, n);
  T* q = c->buf<T>("cg_q_" + tn, n);
  PcgResult res;
  PR_CUDA(cudaMemsetAsync(x, 0, n * sizeof(T), s));
  PR_CUDA(cudaMemcpyAsync(r, b, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
  double rr = rr0 >= 0.0 ? rr0 : dot<T>(c, r, r, n);
  res.rr = rr;
  if (!(std::sqrt(rr) > tol_abs) || maxit <= 0) return res;
  double rz = M.apply(r, z);
  double beta = 0.0;
  T* d = nullptr;  // current search direction
  for (int it = 0; it < maxit; ++it) {
    double dq;
    if (it == 0) {
      dq = A.apply_dot(z, z, nullptr, 0.0, false, q);  // d = z
      d = z;
    } else {
      T* dn = (d == dA) ? dB : dA;
      dq = A.apply_dot(z, d, dn, beta, true, q);
      d = dn;
    }
    if (!(dq > 0.0) || !std::isfinite(dq) || !(rz > 0.0)) {
      res.broke = true;
      break;
    }
    const double alpha = rz / dq;
    const bool fused = M.fuses_cg_update();
    rr = fused ? M.cg_update_presmooth(alpha, d, q, x, r) : cg_update<T>(c, n, alpha, d, q, x, r);
    res.iters = it + 1;
    res.rr = rr;
    if (!std::isfinite(rr)) {
      res.broke = true;
      break;
    }
    if (std::sqrt(rr) <= tol_abs) break;
    if (d == z) {  // the first direction aliases z: keep it before z is overwritten
      PR_CUDA(cudaMemcpyAsync(dA, z, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
      d = dA;
    }
    const double rz_new = M.apply(r, z, fused);
    beta = rz_new / rz;
    rz = rz_new;
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
  double* xA = c->buf<double>("x64", c->n);
  solve_system(c, p, st, c->get<double>("b64"), xA);
  c->have_coeffs = true;
}

// A x = b on the current system (the fine operator of the last setup), x = 0 initially.
void solve_system(pr_context* c, const pr_params& p, pr_stats& st, const double* b, double* xA) {
  const uint64_t n = c->n;
  const uint32_t D = c->D;
  cudaStream_t s = c->stream;
  const double h = 1.0 / (double)(1u << D);
  const double wg = c->pw > 0.0 ? (c->pw * (h * h * h) / 1.5) * 0.005 : 0.0;
  double* xB = c->buf<double>("x64b", n);
  double* r = c->buf<double>("r64", n);
  const double target = p.target_rel_residual > 0.0 ? p.target_rel_residual : 1e-6;
  const int max_iters = p.max_iters > 0 ? (int)p.max_iters : 200;
  const int sweeps = p.smooth_sweeps > 0 ? (int)p.smooth_sweeps : 1;
  const bool mixed = p.precision != PR_PRECISION_FP64;

  st.pcg_iterations = 0;
  st.refinement_steps = 0;
  st.solve_bytes = 0.0;
  PR_CUDA(cudaMemsetAsync(xA, 0, n * sizeof(double), s));
  // mixed: the FP32 system is the current FP64 residual rounded (unscaled: residuals stay far
  // above the bottom of the FP32 range), its norm computed in the same pass
  float* r32 = mixed ? c->buf<float>("r32", n) : nullptr;
  const double bn = mixed ? convert_norm(c, b, r32, n) : std::sqrt(dot<double>(c, b, b, n));
  if (bn == 0.0) {
    st.rel_residual = 0.0;
    st.converged = 1;
    return;
  }
  FineOp<double> A64 = make_fine_op<double>(c, wg);
  const LevelCoef L64 = level_coef(D, D, wg);
  const bool fused = D >= 4;  // tiled residual-update kernel
  const double es = mixed ? 4.0 : 8.0;
  const double per_iter = iter_bytes(n, es, c->P_in, es) + vcycle_bytes(D, es, sweeps);
  const double resid_bytes = 36.0 * n + c->P_in * 2.0 * (8.0 * 8.0 + 32.0) + 8.0 * n;  // update+residual, norm

  // x <- x + scale * e and r = b - A x (FP64); with_norm: returns ||r|| (else 0).  x ping-pongs
  // between xA and xB.
  double* x = xA;
  auto update_residual = [&](const void* e, bool e_is_float, double scale, bool with_norm = true) -> double {
    if (fused) {
      double* xn = (x == xA) ? xB : xA;
      if (e_is_float) mg_resid_update<float>(s, L64, x, (const float*)e, scale, xn, b, r);
      else mg_resid_update<double>(s, L64, x, (const double*)e, scale, xn, b, r);
      x = xn;
      if (A64.scr.active()) {
        screen_project<double>(s, A64.scr, x);
        screen_gather<double>(s, A64.scr, r, -1);
      }
    } else {
      if (e_is_float) axpy<float, double>(s, n, scale, (const float*)e, x);
      else axpy<double, double>(s, n, scale, (const double*)e, x);
      A64.residual(s, x, b, r);
    }
    return with_norm ? std::sqrt(dot<double>(c, r, r, n)) : 0.0;
  };

  double rn = bn;
  const double* rsrc = b;  // current residual (b while x = 0)
  int used = 0;
  if (mixed) {
    CgOperator<float> A32;
    A32.init(c, wg);
    Multigrid<float> M32;
    M32.init(c, D, wg, sweeps);
    float* e32 = c->buf<float>("e32", n);
    const double inner = p.inner_rel_tol > 0.0 ? p.inner_rel_tol : 1e-4;
    while (rn > target * bn && used < max_iters) {
      const double tol = std::max(inner, 0.5 * target * bn / rn);
      // r32 . r32 differs from rn^2 only by the FP32 rounding of r32: good enough for the entry test
      const PcgResult pr_ = pcg<float>(c, A32, M32, r32, e32, tol * rn, max_iters - used, rn * rn);
      used += pr_.iters;
      update_residual(e32, true, 1.0, false);
      const double rn_new = convert_norm(c, r, r32, n);
      rsrc = r;
      st.refinement_steps++;
      st.solve_bytes += pr_.iters * per_iter + 12.0 * n + resid_bytes;
      if (pr_.iters == 0 || !(rn_new < rn)) {  // no progress: stop
        rn = rn_new;
        break;
      }
      rn = rn_new;
    }
  } else {
    Multigrid<double> M64;
    M64.init(c, D, wg, sweeps);
    CgOperator<double> A64cg;
    A64cg.init(c, wg);
    double* e64 = c->buf<double>("e64", n);
    while (rn > target * bn && used < max_iters) {
      const double tol = 0.5 * target * bn;  // absolute, on the current residual system
      const PcgResult pr_ = pcg<double>(c, A64cg, M64, rsrc, e64, tol, max_iters - used, rn * rn);
      used += pr_.iters;
      const double rn_new = update_residual(e64, false, 1.0);
      rsrc = r;
      st.refinement_steps++;
      st.solve_bytes += pr_.iters * per_iter + 8.0 * n + resid_bytes;
      if (pr_.iters == 0 || !(rn_new < rn)) {
        rn = rn_new;
        break;
      }
      rn = rn_new;
    }
  }
  if (x != xA) PR_CUDA(cudaMemcpyAsync(xA, x, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  st.pcg_iterations = (uint32_t)used;
  st.rel_residual = rn / bn;
  st.converged = st.rel_residual <= target ? 1 : 0;
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

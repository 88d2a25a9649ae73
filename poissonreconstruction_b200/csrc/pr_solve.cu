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
#include <cstdlib>
#include <string>
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

// ------------------------------------------------------------------ packed systems
// `clouds` degree-1 systems of one depth D and one screening weight, solved together: every
// vector holds the clouds' slices back to back (cloud k at k 8^D) and every step is one launch for
// all of them (blockIdx.y = cloud).  A single reconstruction is a pack of one.  Per-cloud scalars
// (CG's alpha and beta, the refinement scale, the dot products) pass through pinned host slots;
// packed launches read alpha, beta and the scale from their device copies, a pack of one takes them
// as kernel arguments.
struct Pack {
  pr_context* c = nullptr;  // stream and buffers of the solve
  uint32_t D = 0, clouds = 1;
  uint64_t n = 0;           // nodes per cloud
  double wg = 0.0;          // diagonal shift of the multigrid operator
  ScreenPack scr;           // screening of every cloud (inactive without points or weight)
  FineOp<double> op64;      // a pack of one below depth 4: the per-node operator
  FineOp<float> op32;
  std::vector<uint64_t> P_in;
  double* h = nullptr;      // pinned, kSlots x clouds
  double* d = nullptr;      // device, kSlots x clouds
  enum { kOut, kAlpha, kBeta, kScale, kSlots };
  uint64_t N() const { return n * clouds; }
  double* hs(int k) const { return h + (size_t)k * clouds; }
  double* ds(int k) const { return d + (size_t)k * clouds; }
  // the device results in slot kOut after the stream's work so far
  std::vector<double> fetch() {
    PR_CUDA(cudaMemcpyAsync(hs(kOut), ds(kOut), clouds * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    c->sync();
    return std::vector<double>(hs(kOut), hs(kOut) + clouds);
  }
  // per-cloud values for a packed launch (device slot k), or null for a pack of one.  The host slot
  // is rewritten only after a later fetch, so the copy has run by then.
  const double* upload(int k, const std::vector<double>& v) {
    if (clouds == 1) return nullptr;
    std::copy(v.begin(), v.end(), hs(k));
    PR_CUDA(cudaMemcpyAsync(ds(k), hs(k), clouds * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    return ds(k);
  }
  void init_slots() {
    h = c->pinned_scalars((size_t)kSlots * clouds);
    d = c->buf<double>("pk_scal", (size_t)kSlots * clouds);
  }
};

bool any(const std::vector<char>& v) {
  for (char x : v)
    if (x) return true;
  return false;
}

// Multigrid V-cycle preconditioner on A' = K + wg I with Galerkin coarse levels.
// Level l holds f_l (right-hand side), a_l (after pre-smoothing) and e_l (result);
// sweeps beyond the first ping-pong through t_l.
template <typename T>
struct Multigrid {
  Pack* pk = nullptr;
  pr_context* c = nullptr;
  uint32_t D = 0, Dc = 0, clouds = 1;
  int sweeps = 1;
  std::vector<LevelCoef> L;
  std::vector<T*> f, a, e, t, face;
  T* tables = nullptr;  // [D+1][8*27]
  T* inv = nullptr;
  uint32_t nc = 0;

  void init(Pack& p, int nsweeps) {
    pk = &p;
    c = p.c;
    D = p.D;
    clouds = p.clouds;
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
      L[l] = level_coef(D, l, p.wg * std::pow(8.0, (double)(D - l)));
      for (int m = 0; m < 8; ++m)
        for (int o = 0; o < 27; ++o) tab[(size_t)l * 216 + 27 * m + o] = (T)L[l].table[m][o];
      const uint64_t nl = (1ull << (3 * l)) * clouds;
      const std::string sfx = std::string("_") + tname<T>() + "_" + std::to_string(l);
      if (l < D) {
        f[l] = c->buf<T>("mg_f" + sfx, nl);
        e[l] = c->buf<T>("mg_e" + sfx, nl);
      }
      if (l > Dc) {
        a[l] = c->buf<T>("mg_a" + sfx, nl);
        if (mg_face_entries(l)) face[l] = c->buf<T>("mg_face" + sfx, mg_face_entries(l) * clouds);
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
      dense_solve<T>(s, nc, inv, fl, el, clouds);
      return;
    }
    // pre-smoothing (forward) from zero; result in a_l
    T* cur = a[l];
    if (!presmoothed) mg_smooth<T>(s, L[l], table(l), nullptr, cur, fl, nullptr, 1, true, nullptr, clouds);
    for (int k = 1; k < sweeps; ++k) {
      T* nxt = (cur == a[l]) ? t[l] : a[l];
      mg_smooth<T>(s, L[l], table(l), cur, nxt, fl, nullptr, 0, true, nullptr, clouds);
      cur = nxt;
    }
    mg_resid_restrict<T>(s, L[l], table(l), cur, fl, f[l - 1], face[l], clouds);
    vcycle(l - 1, f[l - 1], e[l - 1], nullptr);
    // post-smoothing (backward): first sweep on cur + P e_{l-1}; the last sweep writes el
    for (int k = 0; k < sweeps; ++k) {
      const bool last = (k == sweeps - 1);
      T* nxt = last ? el : ((cur == a[l]) ? t[l] : a[l]);
      mg_smooth<T>(s, L[l], table(l), cur, nxt, fl, e[l - 1], k == 0 ? 2 : 0, false, last ? part : nullptr, clouds);
      cur = nxt;
    }
  }
  // The CG update can be fused with the first pre-smoothing sweep of the finest level.
  bool fuses_cg_update() const { return D >= 4 && D > Dc; }
  // x += alpha d, r -= alpha q, first pre-smoothing sweep of r into a_D; returns r.r per cloud.
  // A cloud with alpha 0 keeps x and r.
  std::vector<double> cg_update_presmooth(const std::vector<double>& alpha, const T* d, const T* q, T* x, T* r) {
    double* part = c->buf<double>("mg_part", (size_t)mg_blocks(D) * clouds);
    CgFuse<T> cg;
    cg.x = x;
    cg.d = d;
    cg.q = q;
    cg.r = r;
    cg.alpha = (T)alpha[0];
    cg.alpha_dev = pk->upload(Pack::kAlpha, alpha);
    mg_cg_update_presmooth<T>(c->stream, L[D], table(D), cg, a[D], part, clouds);
    sum_parts(c->stream, part, (int)mg_blocks(D), 0.0, part, 0, pk->ds(Pack::kOut), clouds);
    return pk->fetch();
  }
  // z = M r; returns r.z per cloud.  presmoothed: a_D already holds the first sweep on r.
  // After the first V-cycle of a solve (which runs plainly: the kernels' z segments are tuned on
  // first use) the V-cycle is replayed from a CUDA graph kept by the context.
  std::vector<double> apply(const T* r, T* z, bool presmoothed = false) {
    const uint64_t n = 1ull << (3 * D);
    if (D == Dc) {
      dense_solve<T>(c->stream, nc, inv, r, z, clouds);
      double* part = c->buf<double>("pk_dot_part", (size_t)kDotBlocks * clouds);
      dots_pk<T>(c->stream, r, z, n, clouds, part, pk->ds(Pack::kOut));
      return pk->fetch();
    }
    double* part = c->buf<double>("mg_part", (size_t)mg_blocks(D) * clouds);
    auto body = [&] {
      vcycle(D, r, z, part, presmoothed);
      sum_parts(c->stream, part, (int)mg_blocks(D), 0.0, part, 0, pk->ds(Pack::kOut), clouds);
    };
    const char* gr = std::getenv("PR_GRAPHS");
    if (applies++ == 0 || (gr && std::atoi(gr) == 0)) body();
    else c->run_graph(graph_key(r, z, part, presmoothed), body);
    return pk->fetch();
  }
  int applies = 0;
  // everything a captured V-cycle depends on: sizes, the shift (kernel arguments), every buffer
  std::string graph_key(const T* r, const T* z, const double* part, bool presmoothed) const {
    char b[96];
    std::snprintf(b, sizeof(b), "vcycle/%s/%u/%u/%d/%d/%a", tname<T>(), D, clouds, sweeps, presmoothed ? 1 : 0, pk->wg);
    std::string k = b;
    auto add = [&](const void* p) {
      std::snprintf(b, sizeof(b), "/%p", p);
      k += b;
    };
    add(r);
    add(z);
    add(part);
    add(pk->ds(Pack::kOut));
    add(tables);
    add(inv);
    for (uint32_t l = Dc; l <= D; ++l) {
      add(f[l]);
      add(e[l]);
      add(a[l]);
      add(t[l]);
      add(face[l]);
    }
    for (const char* v : {"PR_ZT", "PR_AUTOTUNE", "PR_ZT_SPMV16", "PR_ZT_RESID16", "PR_ZT_SMOOTH16"}) {
      const char* x = std::getenv(v);
      k += "/";
      k += x ? x : "-";
    }
    return k;
  }
};

// Fine operator for CG: tiled stencil SpMV (optionally fused with dn = z + beta d) plus
// the per-point screening terms; returns dn.A dn per cloud from the fused partial sums.
template <typename T>
struct CgOperator {
  Pack* pk = nullptr;
  pr_context* c = nullptr;
  LevelCoef Lf;
  T* table = nullptr;
  uint32_t D = 0, clouds = 1;
  void init(Pack& p) {
    pk = &p;
    c = p.c;
    D = p.D;
    clouds = p.clouds;
    Lf = level_coef(D, D, p.wg);
    std::vector<T> tab(216);
    for (int m = 0; m < 8; ++m)
      for (int o = 0; o < 27; ++o) tab[27 * m + o] = (T)Lf.table[m][o];
    table = c->buf<T>(std::string("cg_tab_") + tname<T>(), 216);
    PR_CUDA(cudaMemcpyAsync(table, tab.data(), 216 * sizeof(T), cudaMemcpyHostToDevice, c->stream));
    c->sync();
  }
  const FineOp<T>& small_op() const;
  // xpby: dn = z + beta d, q = A dn; else q = A d (dn unused).  Returns (dn or d).q per cloud
  std::vector<double> apply_dot(const T* z, const T* d, T* dn, const std::vector<double>& beta, bool xpby, T* q) {
    cudaStream_t s = c->stream;
    const uint64_t n = pk->n;
    const T* dd = xpby ? dn : d;
    if (D < 3) {  // grids below one 8^3 block (a pack of one): per-node kernels
      if (xpby) {
        PR_CUDA(cudaMemcpyAsync(dn, d, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
        pr::xpby<T>(s, n, z, beta[0], dn);
      }
      stencil_apply<T>(s, D, dd, nullptr, q, cast_coef<T>(stencil_coef(D, Lf.shift)), 0);
      screen_apply<T>(s, small_op().scr, dd, q, +1);
      return std::vector<double>(1, dot<T>(c, dd, q, n));
    }
    double* part = c->buf<double>("cg_part", (size_t)mg_blocks(D) * clouds);
    double* part2 = c->buf<double>("cg_part2", (size_t)kDotBlocks * clouds);
    mg_spmv<T>(s, Lf, table, z, d, dn, beta[0], xpby, q, part, clouds, xpby ? pk->upload(Pack::kBeta, beta) : nullptr);
    int np2 = 0;
    if (pk->scr.active()) {
      screen_project_pk<T>(s, pk->scr, dd, n, part2, kDotBlocks);
      screen_gather_pk<T>(s, pk->scr, q, n, +1);
      np2 = kDotBlocks;
    }
    sum_parts(s, part, (int)mg_blocks(D), (double)(T)pk->scr.wh3, part2, np2, pk->ds(Pack::kOut), clouds);
    return pk->fetch();
  }
};
template <>
const FineOp<float>& CgOperator<float>::small_op() const { return pk->op32; }
template <>
const FineOp<double>& CgOperator<double>::small_op() const { return pk->op64; }

struct PcgResult {
  std::vector<int> iters;
  std::vector<double> rr;
  std::vector<char> broke;
};

// Preconditioned CG from x = 0 on A x = b for every cloud with want[k], until ||r_k|| <= tol_abs[k]
// or maxit[k] iterations; rr0[k] = b_k . b_k.  The clouds run in lockstep: one that has stopped
// gets alpha 0 (its x and r stay) and its other results are ignored.  The search direction
// ping-pongs between two buffers (the SpMV reads d with halos).
template <typename T>
PcgResult pcg(Pack& pk, CgOperator<T>& A, Multigrid<T>& M, const T* b, T* x, const std::vector<double>& tol_abs,
              const std::vector<int>& maxit, const std::vector<double>& rr0, const std::vector<char>& want) {
  pr_context* c = pk.c;
  const uint32_t K = pk.clouds;
  const uint64_t N = pk.N();
  cudaStream_t s = c->stream;
  const std::string tn = tname<T>();
  T* r = c->buf<T>("cg_r_" + tn, N);
  T* z = c->buf<T>("cg_z_" + tn, N);
  T* dA = c->buf<T>("cg_d_" + tn, N);
  T* dB = c->buf<T>("cg_d2_" + tn, N);
  T* q = c->buf<T>("cg_q_" + tn, N);
  PcgResult res;
  res.iters.assign(K, 0);
  res.rr = rr0;
  res.broke.assign(K, 0);
  PR_CUDA(cudaMemsetAsync(x, 0, N * sizeof(T), s));
  PR_CUDA(cudaMemcpyAsync(r, b, N * sizeof(T), cudaMemcpyDeviceToDevice, s));
  std::vector<char> act(K, 0);
  for (uint32_t k = 0; k < K; ++k) act[k] = want[k] && std::sqrt(rr0[k]) > tol_abs[k] && maxit[k] > 0;
  if (!any(act)) return res;
  std::vector<double> rz = M.apply(r, z), beta(K, 0.0), alpha(K, 0.0);
  T* d = nullptr;  // current search direction
  for (int it = 0;; ++it) {
    std::vector<double> dq;
    if (it == 0) {
      dq = A.apply_dot(z, z, nullptr, beta, false, q);  // d = z
      d = z;
    } else {
      T* dn = (d == dA) ? dB : dA;
      dq = A.apply_dot(z, d, dn, beta, true, q);
      d = dn;
    }
    for (uint32_t k = 0; k < K; ++k) {
      alpha[k] = 0.0;
      if (!act[k]) continue;
      if (!(dq[k] > 0.0) || !std::isfinite(dq[k]) || !(rz[k] > 0.0)) {
        res.broke[k] = 1;
        act[k] = 0;
        continue;
      }
      alpha[k] = rz[k] / dq[k];
    }
    if (!any(act)) break;
    const bool fused = M.fuses_cg_update();
    const std::vector<double> rr =
        fused ? M.cg_update_presmooth(alpha, d, q, x, r)
              : std::vector<double>(1, cg_update<T>(c, pk.n, alpha[0], d, q, x, r));  // a pack of one
    for (uint32_t k = 0; k < K; ++k) {
      if (!act[k]) continue;
      res.iters[k] = it + 1;
      res.rr[k] = rr[k];
      if (!std::isfinite(rr[k])) {
        res.broke[k] = 1;
        act[k] = 0;
      } else if (std::sqrt(rr[k]) <= tol_abs[k] || it + 1 >= maxit[k]) {
        act[k] = 0;
      }
    }
    if (!any(act)) break;
    if (d == z) {  // the first direction aliases z: keep it before z is overwritten
      PR_CUDA(cudaMemcpyAsync(dA, z, N * sizeof(T), cudaMemcpyDeviceToDevice, s));
      d = dA;
    }
    const std::vector<double> rz_new = M.apply(r, z, fused);
    for (uint32_t k = 0; k < K; ++k) {
      beta[k] = 0.0;
      if (!act[k]) continue;
      beta[k] = rz_new[k] / rz[k];
      rz[k] = rz_new[k];
    }
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

// A_k x_k = b_k for every cloud of the pack (b, x: packed FP64 vectors, x = 0 initially), to the
// relative FP64 residual target; st[k] gets the cloud's solve figures.
void solve_pack(Pack& pk, const pr_params& p, const double* b, double* xA, std::vector<pr_stats>& st) {
  pr_context* c = pk.c;
  const uint32_t K = pk.clouds, D = pk.D;
  const uint64_t n = pk.n, N = pk.N();
  cudaStream_t s = c->stream;
  double* xB = c->buf<double>("x64b", N);
  double* r = c->buf<double>("r64", N);
  const double target = p.target_rel_residual > 0.0 ? p.target_rel_residual : 1e-6;
  const int max_iters = p.max_iters > 0 ? (int)p.max_iters : 200;
  const int sweeps = p.smooth_sweeps > 0 ? (int)p.smooth_sweeps : 1;
  const bool mixed = p.precision != PR_PRECISION_FP64;
  double* part = c->buf<double>("pk_dot_part", (size_t)kDotBlocks * K);

  for (uint32_t k = 0; k < K; ++k) {
    st[k].pcg_iterations = 0;
    st[k].refinement_steps = 0;
    st[k].solve_bytes = 0.0;
  }
  PR_CUDA(cudaMemsetAsync(xA, 0, N * sizeof(double), s));
  // mixed: the FP32 system is the current FP64 residual rounded (unscaled: residuals stay far
  // above the bottom of the FP32 range), its norm computed in the same pass
  float* r32 = mixed ? c->buf<float>("r32", N) : nullptr;
  auto norms_of = [&](const double* v, float* v32) {  // per-cloud ||v|| (and v32 = (float) v)
    if (v32) convert_sq_pk(s, v, v32, n, K, part, pk.ds(Pack::kOut));
    else dots_pk<double>(s, v, v, n, K, part, pk.ds(Pack::kOut));
    std::vector<double> out = pk.fetch();
    for (double& x : out) x = std::sqrt(x);
    return out;
  };
  const std::vector<double> bn = norms_of(b, r32);
  std::vector<char> done(K, 0);
  std::vector<double> rn = bn;
  std::vector<int> used(K, 0);
  for (uint32_t k = 0; k < K; ++k)
    if (bn[k] == 0.0) done[k] = 1;
  const LevelCoef L64 = level_coef(D, D, pk.wg);
  const bool fused = D >= 4;  // tiled residual-update kernel
  const double es = mixed ? 4.0 : 8.0;

  // x <- x + scale_k e and r = b - A x (FP64) per cloud; scale 0 keeps a cloud's x.  x ping-pongs
  // between xA and xB.
  double* x = xA;
  auto update_residual = [&](const void* e, bool e_is_float, const std::vector<double>& scale) {
    if (fused) {
      double* xn = (x == xA) ? xB : xA;
      const double* sd = pk.upload(Pack::kScale, scale);
      if (e_is_float) mg_resid_update<float>(s, L64, x, (const float*)e, scale[0], xn, b, r, K, sd);
      else mg_resid_update<double>(s, L64, x, (const double*)e, scale[0], xn, b, r, K, sd);
      x = xn;
      if (pk.scr.active()) {
        screen_project_pk<double>(s, pk.scr, x, n);
        screen_gather_pk<double>(s, pk.scr, r, n, -1);
      }
    } else {  // a pack of one below depth 4
      if (e_is_float) axpy<float, double>(s, n, scale[0], (const float*)e, x);
      else axpy<double, double>(s, n, scale[0], (const double*)e, x);
      pk.op64.residual(s, x, b, r);
    }
  };

  const double* rsrc = b;  // current residual (b while x = 0)
  auto round = [&](auto tag) {
    using T = decltype(tag);
    CgOperator<T> A;
    A.init(pk);
    Multigrid<T> M;
    M.init(pk, sweeps);
    T* e = c->buf<T>(std::string("e") + (sizeof(T) == 4 ? "32" : "64"), N);
    const double inner = p.inner_rel_tol > 0.0 ? p.inner_rel_tol : 1e-4;
    const double per_iter = 0.0;
    (void)per_iter;
    for (;;) {
      std::vector<char> want(K, 0);
      std::vector<double> tol(K, 0.0), rr0(K, 0.0), scale(K, 0.0);
      std::vector<int> maxit(K, 0);
      for (uint32_t k = 0; k < K; ++k) {
        want[k] = !done[k] && rn[k] > target * bn[k] && used[k] < max_iters;
        if (!want[k]) continue;
        // mixed: an inner tolerance relative to the current residual; FP64: absolute, on the
        // current residual system
        tol[k] = mixed ? std::max(inner, 0.5 * target * bn[k] / rn[k]) * rn[k] : 0.5 * target * bn[k];
        rr0[k] = rn[k] * rn[k];
        maxit[k] = max_iters - used[k];
        scale[k] = 1.0;
      }
      if (!any(want)) break;
      // r32 . r32 differs from rn^2 only by the FP32 rounding of r32: good enough for the entry test
      const T* rhs = mixed ? (const T*)(const void*)r32 : (const T*)(const void*)rsrc;
      const PcgResult pr_ = pcg<T>(pk, A, M, rhs, e, tol, maxit, rr0, want);
      update_residual(e, mixed, scale);
      const std::vector<double> rn_new = norms_of(r, r32);
      rsrc = r;
      for (uint32_t k = 0; k < K; ++k) {
        if (!want[k]) continue;
        used[k] += pr_.iters[k];
        st[k].refinement_steps++;
        const double pib = iter_bytes(n, es, pk.P_in[k], es) + vcycle_bytes(D, es, sweeps);
        const double resid_bytes = 36.0 * n + pk.P_in[k] * 2.0 * (8.0 * 8.0 + 32.0) + 8.0 * n;
        st[k].solve_bytes += pr_.iters[k] * pib + (mixed ? 12.0 : 8.0) * n + resid_bytes;
        if (pr_.iters[k] == 0 || !(rn_new[k] < rn[k])) done[k] = 1;  // no progress: stop
        rn[k] = rn_new[k];
      }
    }
  };
  if (mixed) round(float());
  else round(double());
  if (x != xA) PR_CUDA(cudaMemcpyAsync(xA, x, N * sizeof(double), cudaMemcpyDeviceToDevice, s));
  for (uint32_t k = 0; k < K; ++k) {
    st[k].pcg_iterations = (uint32_t)used[k];
    st[k].rel_residual = bn[k] == 0.0 ? 0.0 : rn[k] / bn[k];
    st[k].converged = st[k].rel_residual <= target ? 1 : 0;
  }
}

double diag_shift(uint32_t D, double pw) {
  const double h = 1.0 / (double)(1u << D);
  return pw > 0.0 ? (pw * (h * h * h) / 1.5) * 0.005 : 0.0;
}

// The screening payload of cloud k of a pack (its context's setup buffers), with projection
// scratch at proj32 / proj64.
ScreenDesc screen_desc(pr_context* cl, float* proj32, double* proj64) {
  ScreenDesc d;
  if (!(cl->pw > 0.0 && cl->S > 0)) return d;
  d.key = cl->get<uint32_t>("scr_kin");
  d.phi32 = cl->get<float>("phi32");
  d.phi64 = cl->get<double>("phi64");
  d.snode = cl->get<uint32_t>("scr_runkey");
  d.soff = cl->get<uint32_t>("scr_runoff");
  d.sval = cl->get<uint32_t>("scr_val");
  d.proj32 = proj32;
  d.proj64 = proj64;
  d.P = cl->P;
  d.S = cl->S;
  return d;
}

// The pack of the clouds' systems on the stream and buffers of sc (sc may be clouds[0]).
void make_pack(Pack& pk, pr_context* sc, const std::vector<pr_context*>& cl) {
  pk.c = sc;
  pk.clouds = (uint32_t)cl.size();
  pk.D = cl[0]->D;
  pk.n = cl[0]->n;
  const double pw = cl[0]->pw;
  pk.wg = diag_shift(pk.D, pw);
  pk.init_slots();
  uint64_t sumP = 0;
  for (pr_context* x : cl) {
    PR_REQUIRE(x->D == pk.D && x->pw == pw && x->degree == 1, PR_ERR_INTERNAL,
               "a packed solve needs degree-1 systems of one depth and screening weight");
    pk.P_in.push_back(x->P_in);
    sumP += x->P;
  }
  std::vector<ScreenDesc> desc;
  float* p32 = sc->buf<float>("pk_proj32", std::max<uint64_t>(sumP, 1));
  double* p64 = sc->buf<double>("pk_proj64", std::max<uint64_t>(sumP, 1));
  uint64_t off = 0;
  for (pr_context* x : cl) {
    desc.push_back(screen_desc(x, p32 + off, p64 + off));
    off += x->P;
    pk.scr.maxP = std::max<uint64_t>(pk.scr.maxP, desc.back().P);
    pk.scr.maxS = std::max<uint64_t>(pk.scr.maxS, desc.back().S);
  }
  ScreenDesc* dd = sc->buf<ScreenDesc>("pk_screen", desc.size());
  PR_CUDA(cudaMemcpyAsync(dd, desc.data(), desc.size() * sizeof(ScreenDesc), cudaMemcpyHostToDevice, sc->stream));
  sc->sync();  // host descriptors
  pk.scr.desc = dd;
  pk.scr.clouds = pk.clouds;
  pk.scr.sentinel = 1u << (3 * pk.D);
  const double h = 1.0 / (double)(1u << pk.D);
  pk.scr.wh3 = pw * (h * h * h) / 1.5;
  if (pk.clouds == 1 && pk.D < 4) {
    pk.op64 = make_fine_op<double>(cl[0], pk.wg);
    pk.op32 = make_fine_op<float>(cl[0], pk.wg);
  }
}

}  // namespace

void stage_solve(pr_context* c, const pr_params& p, pr_stats& st) {
  double* xA = c->buf<double>("x64", c->n);
  solve_system(c, p, st, c->get<double>("b64"), xA);
  c->have_coeffs = true;
}

// A x = b on the current system (the fine operator of the last setup), x = 0 initially.
void solve_system(pr_context* c, const pr_params& p, pr_stats& st, const double* b, double* xA) {
  Pack pk;
  make_pack(pk, c, std::vector<pr_context*>(1, c));
  std::vector<pr_stats> sts(1, st);
  solve_pack(pk, p, b, xA, sts);
  st = sts[0];
}

void solve_packed(pr_context* sc, const std::vector<pr_context*>& cl, const pr_params& p, std::vector<pr_stats>& st) {
  PR_REQUIRE(!cl.empty() && st.size() == cl.size(), PR_ERR_INTERNAL, "solve_packed: one stats entry per cloud");
  PR_REQUIRE(cl[0]->D >= 5, PR_ERR_INTERNAL, "solve_packed: depth >= 5");
  Pack pk;
  make_pack(pk, sc, cl);
  const uint64_t n = pk.n, N = pk.N();
  double* b = sc->buf<double>("pk_b64", N);
  double* x = sc->buf<double>("pk_x64", N);
  for (size_t k = 0; k < cl.size(); ++k)
    PR_CUDA(cudaMemcpyAsync(b + k * n, cl[k]->get<double>("b64"), n * sizeof(double), cudaMemcpyDeviceToDevice,
                            sc->stream));
  solve_pack(pk, p, b, x, st);
  for (size_t k = 0; k < cl.size(); ++k) {
    double* xk = cl[k]->buf<double>("x64", n);
    PR_CUDA(cudaMemcpyAsync(xk, x + k * n, n * sizeof(double), cudaMemcpyDeviceToDevice, sc->stream));
    cl[k]->have_coeffs = true;
  }
  sc->sync();
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

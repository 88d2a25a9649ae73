// Reference-schedule solve: the crate's cascade (FEMTree::solve_cascadic,
// src/fem_tree.rs:458-487) on the GPU, step for step, with one change: Gauss-Seidel sweeps
// relax the 8 parity colours of the grid in turn (each colour in parallel) instead of one
// node at a time in Morton order (src/solvers.rs:164-175).  A partially converged solve
// depends on the relaxation order, so this mode tracks but does not reproduce the crate's
// coefficients; its CG (src/solvers.rs:20-69) is replicated exactly.
//
//   coarse depth D-2 (0 if D <= 2): stiffness at the coarse h, diagonal += wh3'*1.005 with
//   pw' = pw * 4^(D-d), RHS = sum of (v.x + v.y + v.z) over the fine nodes of each coarse
//   cell + wh3'*0.5  (build_system_at_depth, src/fem_tree.rs:346-404)
//   GS(20) + CG(cg_iters) on it; one-level prolongation stencil applied across the gap
//   (prolongate, src/fem_tree.rs:310-343); GS(20) + CG(cg_iters/4) on the fine system.
#include <cmath>

#include "pr_ops.cuh"

namespace pr {

namespace {

constexpr int kThreads = 256;

inline unsigned grid_for(uint64_t n, int threads = kThreads, uint64_t cap = 1u << 22) {
  uint64_t g = (n + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (unsigned)g;
}

// Coarse RHS (src/fem_tree.rs:386-402): fine nodes of a coarse cell are one contiguous
// Morton range, visited in the crate's order (ascending fine FEM index).
__global__ void k_coarse_rhs(const uint32_t* __restrict__ tnode, uint64_t T, const double* __restrict__ v,
                             uint32_t Dc, uint32_t gap, double add, double* __restrict__ brhs) {
  const uint64_t nc = 1ull << (3 * Dc);
  for (uint64_t cc = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; cc < nc; cc += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t lo = cc << (3 * gap), hi = (cc + 1) << (3 * gap);
    // lower_bound(lo) in the sorted touched-node list
    uint64_t a = 0, b = T;
    while (a < b) {
      uint64_t m = (a + b) >> 1;
      if ((uint64_t)tnode[m] < lo) a = m + 1;
      else b = m;
    }
    double acc = 0.0;
    for (uint64_t t = a; t < T && (uint64_t)tnode[t] < hi; ++t)
      acc = xadd(acc, xadd(xadd(v[t], v[T + t]), v[2 * T + t]));
    if (add > 0.0) acc = xadd(acc, add);
    brhs[cc] = acc;
  }
}

// prolongate (src/fem_tree.rs:310-343): fine f receives coarse c with f = 2c + d - 1,
// d in {0,1,2}, weight bw[dx]*bw[dy]*bw[dz], coarse nodes in lexicographic (z,y,x) order.
__global__ void k_prolong_reference(const double* __restrict__ coarse, uint32_t Dc, uint32_t Df,
                                    double* __restrict__ fine) {
  const int cres = 1 << Dc;
  const uint64_t nf = 1ull << (3 * Df);
  const double bw[3] = {0.5, 1.0, 0.5};
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nf; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t f[3];
    unmorton3((uint32_t)i, f[0], f[1], f[2]);
    int cand[3][2], dd[3][2], nc[3];
    for (int a = 0; a < 3; ++a) {
      nc[a] = 0;
      int fa = (int)f[a];
      // ascending coarse coordinate: c = (f-1)/2 (d = 2) before c = (f+1)/2 (d = 0)
      for (int d = 2; d >= 0; --d) {
        int t = fa + 1 - d;
        if (t < 0 || (t & 1)) continue;
        int c = t >> 1;
        if (c >= cres) continue;
        cand[a][nc[a]] = c;
        dd[a][nc[a]] = d;
        ++nc[a];
      }
    }
    double acc = 0.0;
    for (int z = 0; z < nc[2]; ++z)
      for (int y = 0; y < nc[1]; ++y)
        for (int x = 0; x < nc[0]; ++x) {
          double vv = coarse[morton3(cand[0][x], cand[1][y], cand[2][z])];
          if (vv == 0.0) continue;
          double w = xmul(xmul(bw[dd[0][x]], bw[dd[1][y]]), bw[dd[2][z]]);
          acc = xadd(acc, xmul(vv, w));
        }
    fine[i] = acc;
  }
}

__global__ void k_fill_map(const uint32_t* __restrict__ snode, uint64_t S, uint32_t* __restrict__ smap) {
  for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < S; u += (uint64_t)gridDim.x * blockDim.x)
    smap[snode[u]] = (uint32_t)u;
}

// One parity colour of a Gauss-Seidel sweep on K + wg I (+ screening if smap != NULL):
// x_i = (b_i - sum_{j != i} A_ij x_j) / A_ii.  proj holds phi(p).x for the current x;
// same-colour nodes never share a point, so proj stays valid during the colour.
__global__ void k_gs_colour(uint32_t D, int colour, double* __restrict__ x, const double* __restrict__ b, double c0,
                            double ce, double cc, const uint32_t* __restrict__ smap, const uint32_t* __restrict__ soff,
                            const uint32_t* __restrict__ sval, const double* __restrict__ phi,
                            const double* __restrict__ proj, double wh3) {
  const int res = 1 << D;
  const uint64_t n = 1ull << (3 * D);
  const uint64_t cnt = (n + 7 - colour) / 8;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < cnt; t += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t i = (uint32_t)((t << 3) | (uint64_t)colour);
    uint32_t ix, iy, iz;
    unmorton3(i, ix, iy, iz);
    double se = 0.0, sc = 0.0;
    for (int dz = -1; dz <= 1; ++dz) {
      int jz = (int)iz + dz;
      if (jz < 0 || jz >= res) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        int jy = (int)iy + dy;
        if (jy < 0 || jy >= res) continue;
        for (int dx = -1; dx <= 1; ++dx) {
          int jx = (int)ix + dx;
          if (jx < 0 || jx >= res) continue;
          int nz = (dx != 0) + (dy != 0) + (dz != 0);
          if (nz < 2) continue;
          double v = x[morton3(jx, jy, jz)];
          if (nz == 2) se += v;
          else sc += v;
        }
      }
    }
    double diag = c0, off = ce * se + cc * sc;
    if (smap) {
      uint32_t u = smap[i];
      if (u != 0xffffffffu) {
        double xi = x[i], sd = 0.0, so = 0.0;
        for (uint32_t e = soff[u]; e < soff[u + 1]; ++e) {
          uint32_t pk = sval[e];
          double ph = phi[pk];
          sd += ph * ph;
          so += ph * (proj[pk >> 3] - ph * xi);
        }
        diag += wh3 * sd;
        off += wh3 * so;
      }
    }
    x[i] = (b[i] - off) / diag;
  }
}

// src/solvers.rs:20-69 with the GPU operator; delta (host, may be NULL) receives ||r||^2 before
// the first iteration and after each one
uint64_t solve_cg_reference(pr_context* c, const FineOp<double>& A, const double* b, double* x, uint64_t n,
                            uint64_t max_iters, double accuracy, double* delta = nullptr) {
  cudaStream_t s = c->stream;
  double* r = c->buf<double>("rcg_r", n);
  double* d = c->buf<double>("rcg_d", n);
  double* q = c->buf<double>("rcg_q", n);
  A.residual(s, x, b, r);
  PR_CUDA(cudaMemcpyAsync(d, r, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  double delta_new = dot<double>(c, r, r, n);
  const double delta_0 = delta_new;
  if (delta) delta[0] = delta_new;
  if (delta_new == 0.0) return 0;
  for (uint64_t iter = 0; iter < max_iters; ++iter) {
    A.apply(s, d, q);
    double dq = dot<double>(c, d, q, n);
    if (dq == 0.0) return iter + 1;
    double alpha = delta_new / dq;
    double delta_old = delta_new;
    if ((iter + 1) % 10 == 0) {
      axpy<double, double>(s, n, alpha, d, x);
      A.residual(s, x, b, r);
      delta_new = dot<double>(c, r, r, n);
    } else {
      delta_new = cg_update<double>(c, n, alpha, d, q, x, r);
    }
    if (delta) delta[iter + 1] = delta_new;
    if (delta_new <= delta_0 * accuracy * accuracy) return iter + 1;
    double beta = delta_new / delta_old;
    if (std::isnan(beta) || std::isinf(beta)) break;
    xpby<double>(s, n, r, beta, d);
  }
  return max_iters;
}

void gs_sweeps(pr_context* c, uint32_t D, double* x, const double* b, const Coef<double>& k, const Screen<double>* scr,
               const uint32_t* smap, int sweeps) {
  const uint64_t n = 1ull << (3 * D);
  for (int sw = 0; sw < sweeps; ++sw)
    for (int col = 0; col < 8; ++col) {
      uint64_t cnt = (n + 7 - col) / 8;
      if (cnt == 0) continue;
      const double* proj = nullptr;
      if (scr && scr->active()) {
        screen_project<double>(c->stream, *scr, x);
        proj = scr->proj;
      }
      k_gs_colour<<<grid_for(cnt), kThreads, 0, c->stream>>>(
          D, col, x, b, k.c0, k.ce, k.cc, proj ? smap : nullptr, proj ? scr->soff : nullptr,
          proj ? scr->sval : nullptr, proj ? scr->phi : nullptr, proj, proj ? (double)scr->wh3 : 0.0);
      PR_CHECK_LAUNCH();
    }
}

}  // namespace

void stage_solve_reference(pr_context* c, const pr_params& p, pr_stats& st) {
  const uint32_t D = c->D;
  const uint64_t n = c->n;
  const double pw = c->pw;
  const int gs = 20;
  cudaStream_t s = c->stream;
  const double h = 1.0 / (double)(1u << D);
  const double wg = pw > 0.0 ? (pw * (h * h * h) / 1.5) * 0.005 : 0.0;
  FineOp<double> A = make_fine_op<double>(c, wg);
  const double* b = c->get<double>("b64");
  double* x = c->buf<double>("x64", n);
  const uint32_t Dc = D > 2 ? D - 2 : 0;
  const uint64_t ncoarse = 1ull << (3 * Dc);

  // --- coarse system (build_system_at_depth)
  const double hc = 1.0 / (double)(1u << Dc);
  const double eff_pw = pw * (double)(1ull << (2 * (D - Dc)));
  const double wh3c = eff_pw > 0.0 ? eff_pw * (hc * hc * hc) / 1.5 : 0.0;
  FineOp<double> Ac;
  Ac.D = Dc;
  Ac.coef = stencil_coef(Dc, eff_pw > 0.0 ? wh3c * 1.005 : 0.0);
  double* brhs = c->buf<double>("ref_brhs", ncoarse);
  c->have_ref_coarse = true;
  c->ref_coarse_D = Dc;
  double* csol = c->buf<double>("ref_csol", ncoarse);
  k_coarse_rhs<<<grid_for(ncoarse), kThreads, 0, s>>>(c->get<uint32_t>("splat_runkey"), c->T, c->get<double>("nfield"),
                                                     Dc, D - Dc, eff_pw > 0.0 ? wh3c * 0.5 : 0.0, brhs);
  PR_CHECK_LAUNCH();
  PR_CUDA(cudaMemsetAsync(csol, 0, ncoarse * sizeof(double), s));
  gs_sweeps(c, Dc, csol, brhs, Ac.coef, nullptr, nullptr, gs);
  uint64_t itc = solve_cg_reference(c, Ac, brhs, csol, ncoarse, p.cg_iters, p.cg_accuracy);

  // --- prolongation + fine relaxation
  k_prolong_reference<<<grid_for(n), kThreads, 0, s>>>(csol, Dc, D, x);
  PR_CHECK_LAUNCH();
  uint32_t* smap = nullptr;
  if (A.scr.active()) {
    smap = c->buf<uint32_t>("ref_smap", n);
    PR_CUDA(cudaMemsetAsync(smap, 0xff, n * sizeof(uint32_t), s));
    k_fill_map<<<grid_for(A.scr.S), kThreads, 0, s>>>(A.scr.snode, A.scr.S, smap);
    PR_CHECK_LAUNCH();
  }
  Coef<double> kf = stencil_coef(D, wg);
  gs_sweeps(c, D, x, b, kf, &A.scr, smap, gs);
  uint64_t itf = solve_cg_reference(c, A, b, x, n, p.cg_iters / 4, p.cg_accuracy);

  double* r = c->buf<double>("r64", n);
  A.residual(s, x, b, r);
  double bn = dot<double>(c, b, b, n), rn = dot<double>(c, r, r, n);
  st.rel_residual = bn > 0.0 ? std::sqrt(rn / bn) : 0.0;
  st.pcg_iterations = (uint32_t)(itc + itf);
  st.refinement_steps = 0;
  st.converged = 0;
  c->have_coeffs = true;
  if (smap) c->release("ref_smap");
}

uint64_t cg_reference_fine(pr_context* c, double* d_x, uint64_t max_iters, double accuracy, double* delta) {
  const uint32_t D = c->D;
  const double h = 1.0 / (double)(1u << D);
  const double wg = c->pw > 0.0 ? (c->pw * (h * h * h) / 1.5) * 0.005 : 0.0;
  FineOp<double> A = make_fine_op<double>(c, wg);
  const uint64_t it = solve_cg_reference(c, A, c->get<double>("b64"), d_x, c->n, max_iters, accuracy, delta);
  c->release("rcg_r");
  c->release("rcg_d");
  c->release("rcg_q");
  return it;
}

}  // namespace pr

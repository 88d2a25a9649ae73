// Adjoint of the reconstruction: gradients of a loss on the implicit function at query
// points w.r.t. the input points' positions and normals.  No counterpart in the reference
// crate; it differentiates the crate's forward path:
//   splat      nf_j = -(sum_i phi_j(u_i) nu_i) / w_j,  w_j = sum_i phi_j(u_i)
//              (floor cells, src/fem_tree.rs:130-178)
//   RHS        b = G nf + (wh3/2) sum_i psi(u_i)   (divergence stencil :251-274, screening
//              RHS on trunc cells :276-297)
//   operator   A = K + wg I + wh3 sum_i psi(u_i) psi(u_i)^T   (:180-249)
//   solve      A x = b;  chi(q) = evaluate(x, q)   (:490-513)
// With g = dL/dchi at the queries, lambda = A^{-1} E^T g (A symmetric), and
//   dL/dnu_i = -sum_j (phi_j(u_i)/w_j) mu_j,                         mu = G^T lambda
//   dL/du_i  = -sum_j (grad phi_j(u_i)/w_j) mu_j.(nu_i + nf_j)
//              + (wh3/2) grad Lambda(u_i) - wh3 (grad Lambda X + Lambda grad X)(u_i)
// where Lambda(u) = sum psi_l(u) lambda_l and X(u) = sum psi_l(u) x_l.  Model space: u = s p +
// c with the unit-cube transform held fixed; nu = v/|v| with v = s n.
//
// Every sum has a fixed order (sort-based scatter for E^T g, per-point gathers with the
// corner loop for the rest), so the result is deterministic.  adjoint_backward2 is the same for
// the quadratic node functions of pr_params.degree = 2.
#include <cstring>

#include "pr_internal.cuh"

namespace pr {

namespace {

constexpr int kThreads = 256;
constexpr uint32_t kEmpty = 0xffffffffu;

inline unsigned grid_for(uint64_t n, uint64_t cap = 1u << 20) {
  uint64_t g = (n + kThreads - 1) / kThreads;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (unsigned)g;
}

struct Affine {
  double m[16];  // column-major m[col*4+row]
};

// Mat4::transform_point (src/geometry.rs:256-262), the operation order of the forward transform
__global__ void k_query_unit(const double* __restrict__ q3, uint64_t K, Affine M, double* __restrict__ qu) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < K; i += (uint64_t)gridDim.x * blockDim.x) {
    const double* p = q3 + 3 * i;
#pragma unroll
    for (int r = 0; r < 3; ++r)
      qu[3 * i + r] =
          xadd(xadd(xadd(xmul(M.m[r], p[0]), xmul(M.m[4 + r], p[1])), xmul(M.m[8 + r], p[2])), M.m[12 + r]);
  }
}

// g = upstream gradient, or 2 chi / K for the mean-square loss
__global__ void k_upstream(const double* __restrict__ chi, const double* __restrict__ dl, uint64_t K,
                           double* __restrict__ g) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < K; i += (uint64_t)gridDim.x * blockDim.x)
    g[i] = dl ? dl[i] : 2.0 * chi[i] / (double)K;
}

__device__ __forceinline__ double bspline1(double t) {
  if (t < 0.0 || t > 2.0) return 0.0;
  if (t <= 1.0) return t;
  return xsub(2.0, t);
}

// evaluate()'s basis on one axis (src/fem_tree.rs:490-513, :640-649): nodes o[2], weights b[2]
__device__ __forceinline__ void eval_axis(double u, double h, int64_t res, uint32_t* o, double* b) {
  const double s = xdiv(u, h);
  const int64_t f = sat_i64(floor(s));
  int64_t lo = f - 1, hi = f;
  lo = lo < 0 ? 0 : (lo > res - 1 ? res - 1 : lo);
  hi = hi < 0 ? 0 : (hi > res - 1 ? res - 1 : hi);
  o[0] = (uint32_t)lo;
  o[1] = (uint32_t)hi;
  b[0] = bspline1(xsub(s, (double)o[0]));
  b[1] = bspline1(xsub(s, (double)o[1]));
}

// (node, 8k + term) pairs of E^T: term e = a | b<<1 | c<<2 over evaluate()'s 2x2x2 loop;
// terms that evaluate() skips (a zero weight) get the sentinel key 2^(3D).
__global__ void k_eval_pairs(const double* __restrict__ qu, uint64_t K, uint32_t D, uint32_t* __restrict__ keys,
                             uint32_t* __restrict__ vals) {
  const int64_t res = 1ll << D;
  const double h = 1.0 / (double)res;
  const uint32_t sentinel = 1u << (3 * D);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < K; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t o[3][2];
    double b[3][2];
#pragma unroll
    for (int a = 0; a < 3; ++a) eval_axis(qu[3 * i + a], h, res, o[a], b[a]);
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int a = e & 1, bb = (e >> 1) & 1, cc = e >> 2;
      const bool ok = b[0][a] != 0.0 && b[1][bb] != 0.0 && b[2][cc] != 0.0;
      keys[8 * i + e] = ok ? morton3(o[0][a], o[1][bb], o[2][cc]) : sentinel;
      vals[8 * i + e] = (uint32_t)(8 * i + e);
    }
  }
}

// rhs[node] = sum over the node's (query, term) pairs in query order of g_k * basis weight
__global__ void k_eval_scatter(const uint32_t* __restrict__ run_key, const uint32_t* __restrict__ run_off,
                               uint64_t R, const uint32_t* __restrict__ sval, const double* __restrict__ qu,
                               const double* __restrict__ g, uint32_t D, double* __restrict__ rhs) {
  const int64_t res = 1ll << D;
  const double h = 1.0 / (double)res;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < R; t += (uint64_t)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (uint32_t e = run_off[t]; e < run_off[t + 1]; ++e) {
      const uint32_t pk = sval[e];
      const uint32_t k = pk >> 3, term = pk & 7u;
      uint32_t o[2];
      double bx[2], by[2], bz[2];
      eval_axis(qu[3 * k], h, res, o, bx);
      eval_axis(qu[3 * k + 1], h, res, o, by);
      eval_axis(qu[3 * k + 2], h, res, o, bz);
      acc = xadd(acc, xmul(xmul(xmul(g[k], bx[term & 1u]), by[(term >> 1) & 1u]), bz[term >> 2]));
    }
    rhs[run_key[t]] = acc;
  }
}

__device__ __forceinline__ double mass1(int d) { return d == 0 ? 2.0 / 3.0 : 1.0 / 6.0; }
__device__ __forceinline__ double dmass1(int d) { return d == 0 ? 0.0 : (d == 1 ? -0.5 : 0.5); }

// mu_t = (G^T lambda) at splat node t: row i = j - d of the divergence stencil sees node j at
// offset d with weights h^2 dm(dx) m(dy) m(dz) (x component) and permutations.
__global__ void k_mu(const uint32_t* __restrict__ run_key, uint64_t T, const double* __restrict__ lam, uint32_t D,
                     double* __restrict__ mu) {
  const int res = 1 << D;
  const double h = 1.0 / (double)res;
  const double h2 = h * h;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < T; t += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t jx, jy, jz;
    unmorton3(run_key[t], jx, jy, jz);
    double m0 = 0.0, m1 = 0.0, m2 = 0.0;
    for (int dx = -1; dx <= 1; ++dx) {
      const int ix = (int)jx - dx;
      if (ix < 0 || ix >= res) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        const int iy = (int)jy - dy;
        if (iy < 0 || iy >= res) continue;
        for (int dz = -1; dz <= 1; ++dz) {
          const int iz = (int)jz - dz;
          if (iz < 0 || iz >= res) continue;
          const double l = lam[morton3(ix, iy, iz)] * h2;
          m0 += l * dmass1(dx) * mass1(dy) * mass1(dz);
          m1 += l * mass1(dx) * dmass1(dy) * mass1(dz);
          m2 += l * mass1(dx) * mass1(dy) * dmass1(dz);
        }
      }
    }
    mu[t] = m0;
    mu[T + t] = m1;
    mu[2 * T + t] = m2;
  }
}

// Trilinear corner basis: value and gradient (unit-cube coordinates) of corner d of the cell
// with in-cell coordinates t.
__device__ __forceinline__ void corner_basis(const double* t, int dx, int dy, int dz, double inv_h, double& phi,
                                             double* gp) {
  const double bx = dx ? t[0] : 1.0 - t[0], by = dy ? t[1] : 1.0 - t[1], bz = dz ? t[2] : 1.0 - t[2];
  const double gx = dx ? inv_h : -inv_h, gy = dy ? inv_h : -inv_h, gz = dz ? inv_h : -inv_h;
  phi = bx * by * bz;
  gp[0] = gx * by * bz;
  gp[1] = bx * gy * bz;
  gp[2] = bx * by * gz;
}

struct PointGradArgs {
  const double* upos;  // 3 x P (SoA)
  const double* unrm;
  const double* ulen;
  uint64_t P;
  uint32_t D;
  const uint32_t* map;  // node -> splat slot
  const double* nfield;  // 4 x T: nf x y z, w
  const double* mu;      // 3 x T
  uint64_t T;
  const double* lam;  // n
  const double* x;    // n
  double wh3;         // 0 without screening
  double s;           // model -> unit scale
  double* dpos;       // P x 3
  double* dnrm;       // P x 3
};

__global__ void k_point_grad(PointGradArgs a) {
  const uint32_t res = 1u << a.D;
  const double h = 1.0 / (double)res;
  const double inv_h = (double)res;
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < a.P; p += (uint64_t)gridDim.x * blockDim.x) {
    const double u[3] = {a.upos[p], a.upos[a.P + p], a.upos[2 * a.P + p]};
    const double nu[3] = {a.unrm[p], a.unrm[a.P + p], a.unrm[2 * a.P + p]};
    double gu[3] = {0.0, 0.0, 0.0}, gn[3] = {0.0, 0.0, 0.0};
    {  // splat, floor cells
      int64_t c[3];
      double t[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double sk = xdiv(u[k], h);
        c[k] = sat_i64(floor(sk));
        t[k] = xsub(sk, (double)c[k]);
      }
      for (int kk = 0; kk < 8; ++kk) {
        const int dx = kk & 1, dy = (kk >> 1) & 1, dz = kk >> 2;
        const uint64_t ox = (uint64_t)c[0] + dx, oy = (uint64_t)c[1] + dy, oz = (uint64_t)c[2] + dz;
        if (ox >= res || oy >= res || oz >= res) continue;
        const uint32_t slot = a.map[morton3((uint32_t)ox, (uint32_t)oy, (uint32_t)oz)];
        if (slot == kEmpty) continue;
        const double w = a.nfield[3 * a.T + slot];
        if (!(w > 0.0)) continue;
        double phi, gp[3];
        corner_basis(t, dx, dy, dz, inv_h, phi, gp);
        const double m[3] = {a.mu[slot], a.mu[a.T + slot], a.mu[2 * a.T + slot]};
        const double nf[3] = {a.nfield[slot], a.nfield[a.T + slot], a.nfield[2 * a.T + slot]};
        const double sdot = m[0] * (nu[0] + nf[0]) + m[1] * (nu[1] + nf[1]) + m[2] * (nu[2] + nf[2]);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          gn[k] -= phi / w * m[k];
          gu[k] -= gp[k] / w * sdot;
        }
      }
    }
    if (a.wh3 > 0.0) {  // screening RHS and matrix, trunc cells
      int64_t c[3];
      double t[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double sk = xdiv(u[k], h);
        c[k] = sat_i64(sk);
        t[k] = xsub(sk, (double)c[k]);
      }
      double Lv = 0.0, Xv = 0.0, gL[3] = {0.0, 0.0, 0.0}, gX[3] = {0.0, 0.0, 0.0};
      for (int kk = 0; kk < 8; ++kk) {
        const int dx = kk & 1, dy = (kk >> 1) & 1, dz = kk >> 2;
        const uint32_t ox = (uint32_t)((uint64_t)c[0] + dx), oy = (uint32_t)((uint64_t)c[1] + dy),
                       oz = (uint32_t)((uint64_t)c[2] + dz);
        if (ox >= res || oy >= res || oz >= res) continue;
        const uint32_t j = morton3(ox, oy, oz);
        double phi, gp[3];
        corner_basis(t, dx, dy, dz, inv_h, phi, gp);
        const double lj = a.lam[j], xj = a.x[j];
        Lv += phi * lj;
        Xv += phi * xj;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          gL[k] += gp[k] * lj;
          gX[k] += gp[k] * xj;
        }
      }
#pragma unroll
      for (int k = 0; k < 3; ++k) gu[k] += a.wh3 * 0.5 * gL[k] - a.wh3 * (gL[k] * Xv + Lv * gX[k]);
    }
    const double len = a.ulen[p];
    const double ng = nu[0] * gn[0] + nu[1] * gn[1] + nu[2] * gn[2];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      a.dpos[3 * p + k] = a.s * gu[k];
      a.dnrm[3 * p + k] = len > 0.0 ? a.s / len * (gn[k] - nu[k] * ng) : 0.0;
    }
  }
}

// ------------------------------------------------------------------ degree 2
// The same adjoint for quadratic B-spline node functions (pr_params.degree = 2): the forward is
// the degree-2 system (27 nodes per point for the splat and the screening, floor cells, the
// divergence stencil h^2 (G M M) per component), its vectors in natural order.  With the 1-D
// integrals m, g at offsets -2..2:
//   mu_j^a = h^2 sum_d lambda_{j-d} W_a(d),  W_x(d) = g(dx) m(dy) m(dz) (permuted for y, z),
// and the per-point formulas above with the degree-2 basis and its gradient.

// degree-2 basis of one axis: nodes c-1, c, c+1 with values b and derivatives db (d/du)
__device__ __forceinline__ void axis2_grad(double u, double h, int64_t& c, double* b, double* db) {
  const double s = xdiv(u, h);
  c = sat_i64(floor(s));
  const double t = xsub(s, (double)c);
  const double omt = xsub(1.0, t);
  b[0] = xmul(xmul(0.5, omt), omt);
  b[1] = xmul(0.5, xadd(xadd(xmul(xmul(-2.0, t), t), xmul(2.0, t)), 1.0));
  b[2] = xmul(xmul(0.5, t), t);
  const double ih = 1.0 / h;
  db[0] = -omt * ih;
  db[1] = (1.0 - 2.0 * t) * ih;
  db[2] = t * ih;
}

// (node, 27 k + term) pairs of E^T for the degree-2 evaluation: natural node index, sentinel
// 2^(3D) outside the grid
__global__ void k_eval_pairs2(const double* __restrict__ qu, uint64_t K, uint32_t D, uint32_t* __restrict__ keys,
                              uint32_t* __restrict__ vals) {
  const int64_t res = 1ll << D;
  const double h = 1.0 / (double)res;
  const uint32_t sentinel = 1u << (3 * D);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < 27 * K; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = i / 27;
    const int e = (int)(i - 27 * k), dx = e % 3, dy = (e / 3) % 3, dz = e / 9;
    int64_t c[3];
    double b[3], db[3];
    axis2_grad(qu[3 * k], h, c[0], b, db);
    axis2_grad(qu[3 * k + 1], h, c[1], b, db);
    axis2_grad(qu[3 * k + 2], h, c[2], b, db);
    const int64_t x = c[0] + dx - 1, y = c[1] + dy - 1, z = c[2] + dz - 1;
    const bool ok = x >= 0 && y >= 0 && z >= 0 && x < res && y < res && z < res;
    keys[i] = ok ? (uint32_t)(x + res * (y + res * z)) : sentinel;
    vals[i] = (uint32_t)i;
  }
}

// rhs[node] = sum over the node's (query, term) pairs in query order of g_k * basis value
__global__ void k_eval_scatter2(const uint32_t* __restrict__ run_key, const uint32_t* __restrict__ run_off,
                                uint64_t R, const uint32_t* __restrict__ sval, const double* __restrict__ qu,
                                const double* __restrict__ g, uint32_t D, double* __restrict__ rhs) {
  const double h = 1.0 / (double)(1u << D);
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < R; t += (uint64_t)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (uint32_t e = run_off[t]; e < run_off[t + 1]; ++e) {
      const uint32_t pk = sval[e];
      const uint32_t k = pk / 27, term = pk % 27;
      int64_t c;
      double bx[3], by[3], bz[3], db[3];
      axis2_grad(qu[3 * k], h, c, bx, db);
      axis2_grad(qu[3 * k + 1], h, c, by, db);
      axis2_grad(qu[3 * k + 2], h, c, bz, db);
      acc = xadd(acc, xmul(g[k], xmul(xmul(bx[term % 3], by[(term / 3) % 3]), bz[term / 9])));
    }
    rhs[run_key[t]] = acc;
  }
}

struct Deg2K {
  double m[5], g[5];
};
// mu at the touched nodes (natural run keys), 3 x T
__global__ void k_mu2(const uint32_t* __restrict__ run_key, uint64_t T, const double* __restrict__ lam, uint32_t D,
                      Deg2K k, double* __restrict__ mu) {
  const int res = 1 << D;
  const double h = 1.0 / (double)res;
  const double h2 = h * h;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < T; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t j = run_key[t];
    const int jx = (int)(j & (res - 1)), jy = (int)((j >> D) & (res - 1)), jz = (int)(j >> (2 * D));
    double m0 = 0.0, m1 = 0.0, m2 = 0.0;
    for (int dz = -2; dz <= 2; ++dz) {
      const int iz = jz - dz;
      if (iz < 0 || iz >= res) continue;
      for (int dy = -2; dy <= 2; ++dy) {
        const int iy = jy - dy;
        if (iy < 0 || iy >= res) continue;
        for (int dx = -2; dx <= 2; ++dx) {
          const int ix = jx - dx;
          if (ix < 0 || ix >= res) continue;
          const double l = lam[(uint64_t)ix + (uint64_t)res * (iy + (uint64_t)res * iz)] * h2;
          m0 += l * k.g[dx + 2] * k.m[dy + 2] * k.m[dz + 2];
          m1 += l * k.m[dx + 2] * k.g[dy + 2] * k.m[dz + 2];
          m2 += l * k.m[dx + 2] * k.m[dy + 2] * k.g[dz + 2];
        }
      }
    }
    mu[t] = m0;
    mu[T + t] = m1;
    mu[2 * T + t] = m2;
  }
}

// per run: w = sum phi (point order, the splat's own sum) and runidx[pair] = run
__global__ void k_run_weights2(const uint32_t* __restrict__ run_off, uint64_t T, const uint32_t* __restrict__ sval,
                               const double* __restrict__ phi, double* __restrict__ w, uint32_t* __restrict__ runidx) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < T; t += (uint64_t)gridDim.x * blockDim.x) {
    double sw = 0.0;
    for (uint32_t e = run_off[t]; e < run_off[t + 1]; ++e) {
      sw = xadd(sw, phi[sval[e]]);
      runidx[sval[e]] = (uint32_t)t;
    }
    w[t] = sw;
  }
}

__global__ void k_point_grad2(PointGrad2In a) {
  const double h = 1.0 / (double)(1u << a.D);
  const uint32_t sentinel = a.sentinel;
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < a.P; p += (uint64_t)gridDim.x * blockDim.x) {
    const double nu[3] = {a.unrm[p], a.unrm[a.P + p], a.unrm[2 * a.P + p]};
    int64_t c[3];
    double b[3][3], db[3][3];
    for (int k = 0; k < 3; ++k) axis2_grad(a.upos[(uint64_t)k * a.P + p], h, c[k], b[k], db[k]);
    double gu[3] = {0.0, 0.0, 0.0}, gn[3] = {0.0, 0.0, 0.0};
    double Lv = 0.0, Xv = 0.0, gL[3] = {0.0, 0.0, 0.0}, gX[3] = {0.0, 0.0, 0.0};
    for (int e = 0; e < 27; ++e) {
      const uint32_t node = a.key[27 * p + e];
      if (node == sentinel) continue;
      const int ix = e % 3, iy = (e / 3) % 3, iz = e / 9;
      const double phi = b[0][ix] * b[1][iy] * b[2][iz];
      const double gp[3] = {db[0][ix] * b[1][iy] * b[2][iz], b[0][ix] * db[1][iy] * b[2][iz],
                            b[0][ix] * b[1][iy] * db[2][iz]};
      const uint32_t t = a.runidx[27 * p + e];
      const double wt = a.w[t];
      if (wt > 0.0) {  // splat
        const double m[3] = {a.mu[t], a.mu[a.T + t], a.mu[2 * a.T + t]};
        const double nf[3] = {a.nfc[a.nfc_aos ? 3 * t : t], a.nfc[a.nfc_aos ? 3 * t + 1 : a.T + t],
                              a.nfc[a.nfc_aos ? 3 * t + 2 : 2 * a.T + t]};
        const double sdot = m[0] * (nu[0] + nf[0]) + m[1] * (nu[1] + nf[1]) + m[2] * (nu[2] + nf[2]);
        for (int k = 0; k < 3; ++k) {
          gn[k] -= phi / wt * m[k];
          gu[k] -= gp[k] / wt * sdot;
        }
      }
      if (a.wh3 > 0.0) {
        const double lj = a.lam[node], xj = a.x[node];
        Lv += phi * lj;
        Xv += phi * xj;
        for (int k = 0; k < 3; ++k) {
          gL[k] += gp[k] * lj;
          gX[k] += gp[k] * xj;
        }
      }
    }
    if (a.wh3 > 0.0)
      for (int k = 0; k < 3; ++k) gu[k] += a.wh3 * 0.5 * gL[k] - a.wh3 * (gL[k] * Xv + Lv * gX[k]);
    const double len = a.ulen[p];
    const double ng = nu[0] * gn[0] + nu[1] * gn[1] + nu[2] * gn[2];
    for (int k = 0; k < 3; ++k) {
      const double dp = a.s * gu[k], dn = len > 0.0 ? a.s / len * (gn[k] - nu[k] * ng) : 0.0;
      a.dpos[3 * p + k] = a.accumulate ? a.dpos[3 * p + k] + dp : dp;
      a.dnrm[3 * p + k] = a.accumulate ? a.dnrm[3 * p + k] + dn : dn;
    }
  }
}

}  // namespace

void point_grad2(pr_context* c, const PointGrad2In& a) {
  if (a.P == 0) return;
  k_point_grad2<<<grid_for(a.P), kThreads, 0, c->stream>>>(a);
  PR_CHECK_LAUNCH();
}
void run_weights2(pr_context* c, const uint32_t* run_off, uint64_t T, const uint32_t* sval, const double* phi, double* w,
                  uint32_t* runidx) {
  if (T == 0) return;
  k_run_weights2<<<grid_for(T), kThreads, 0, c->stream>>>(run_off, T, sval, phi, w, runidx);
  PR_CHECK_LAUNCH();
}
void mu2_dense(pr_context* c, const uint32_t* run_key, uint64_t T, const double* lam, uint32_t D, double* mu) {
  if (T == 0) return;
  Deg2K k;
  double s5[5];
  deg2_constants(k.m, s5, k.g);
  k_mu2<<<grid_for(T), kThreads, 0, c->stream>>>(run_key, T, lam, D, k, mu);
  PR_CHECK_LAUNCH();
}

void adjoint_backward2(pr_context* c, const double* d_q3, uint64_t K, const double* d_dl, double* d_chi,
                       double* d_dpos, double* d_dnrm, pr_adjoint_stats& st) {
  const uint32_t D = c->D;
  const uint64_t n = c->n, P = c->P, T = c->T;
  cudaStream_t s = c->stream;
  Affine M;
  for (int k = 0; k < 16; ++k) M.m[k] = c->M[k];
  double* qu = c->buf<double>("adj_qu", 3 * K);
  k_query_unit<<<grid_for(K), kThreads, 0, s>>>(d_q3, K, M, qu);
  PR_CHECK_LAUNCH();
  // the forward solution, kept apart from the solver's buffers the adjoint solve reuses
  double* x = c->buf<double>("adj2_x", n);
  PR_CUDA(cudaMemcpyAsync(x, c->d2_xnat, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  c->d2_xnat = x;
  evaluate_points(c, D, x, qu, 3, K, d_chi, 3);
  double* g = c->buf<double>("adj_g", K);
  k_upstream<<<grid_for(K), kThreads, 0, s>>>(d_chi, d_dl, K, g);
  PR_CHECK_LAUNCH();
  st.loss = d_dl ? dot64(c, d_dl, d_chi, K) : dot64(c, d_chi, d_chi, K) / (double)K;

  uint32_t* kin = c->buf<uint32_t>("adj_kin", 27 * K);
  uint32_t* vin = c->buf<uint32_t>("adj_vin", 27 * K);
  k_eval_pairs2<<<grid_for(27 * K), kThreads, 0, s>>>(qu, K, D, kin, vin);
  PR_CHECK_LAUNCH();
  const uint64_t R = sort_and_segment(c, "adjq", kin, vin, 27 * K, D);
  double* rhs = c->buf<double>("adj_rhs", n);
  PR_CUDA(cudaMemsetAsync(rhs, 0, n * sizeof(double), s));
  if (R > 0) {
    k_eval_scatter2<<<grid_for(R), kThreads, 0, s>>>(c->get<uint32_t>("adjq_runkey"), c->get<uint32_t>("adjq_runoff"),
                                                      R, c->get<uint32_t>("adjq_val"), qu, g, D, rhs);
    PR_CHECK_LAUNCH();
  }
  c->release("adj_kin");
  c->release("adj_vin");

  pr_stats sst;
  std::memset(&sst, 0, sizeof(sst));
  c->sync();
  const double t0 = now_seconds();
  solve_deg2(c, c->params, sst, rhs);
  c->sync();
  st.time_solve = now_seconds() - t0;
  st.rel_residual = sst.rel_residual;
  st.pcg_iterations = sst.pcg_iterations;
  st.refinement_steps = sst.refinement_steps;
  st.converged = sst.converged;
  double* lam = c->buf<double>("adj_lambda", n);
  PR_CUDA(cudaMemcpyAsync(lam, c->d2_xnat, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  c->d2_xnat = x;  // the context keeps the forward solution
  c->x64_ready = false;

  double* mu = c->buf<double>("adj_mu", 3 * std::max<uint64_t>(T, 1));
  double* w = c->buf<double>("adj_w", std::max<uint64_t>(T, 1));
  uint32_t* runidx = c->buf<uint32_t>("adj_runidx", 27 * P);
  if (T > 0) {
    Deg2K k;
    double s5[5];
    deg2_constants(k.m, s5, k.g);
    k_mu2<<<grid_for(T), kThreads, 0, s>>>(c->get<uint32_t>("d2s_runkey"), T, lam, D, k, mu);
    PR_CHECK_LAUNCH();
    k_run_weights2<<<grid_for(T), kThreads, 0, s>>>(c->get<uint32_t>("d2s_runoff"), T, c->get<uint32_t>("d2s_val"),
                                                      c->get<double>("d2_phi64"), w, runidx);
    PR_CHECK_LAUNCH();
  }
  const double h = 1.0 / (double)(1u << D);
  PointGrad2In a;
  a.sentinel = 1u << (3 * D);
  a.accumulate = 0;
  a.upos = c->get<double>("upos");
  a.unrm = c->get<double>("unrm");
  a.ulen = c->get<double>("ulen");
  a.P = P;
  a.D = D;
  a.key = c->get<uint32_t>("d2_kin");
  a.runidx = runidx;
  a.nfc = c->get<double>("d2_nfc");
  a.w = w;
  a.mu = mu;
  a.T = T;
  a.lam = lam;
  a.x = x;
  a.wh3 = c->pw > 0.0 ? c->pw * (h * h * h) / 1.5 : 0.0;
  a.s = c->M[0];
  a.dpos = d_dpos;
  a.dnrm = d_dnrm;
  point_grad2(c, a);
  c->release("adj_runidx");
}

// d_q3: K model-space queries (device); d_dl: K upstream gradients or nullptr (mean chi^2);
// outputs on the device: d_chi (K), d_dpos and d_dnrm (P x 3).
void adjoint_backward(pr_context* c, const double* d_q3, uint64_t K, const double* d_dl, double* d_chi,
                      double* d_dpos, double* d_dnrm, pr_adjoint_stats& st) {
  const uint32_t D = c->D;
  const uint64_t n = c->n, P = c->P, T = c->T;
  cudaStream_t s = c->stream;
  Affine M;
  for (int k = 0; k < 16; ++k) M.m[k] = c->M[k];
  double* qu = c->buf<double>("adj_qu", 3 * K);
  k_query_unit<<<grid_for(K), kThreads, 0, s>>>(d_q3, K, M, qu);
  PR_CHECK_LAUNCH();
  const double* x = coeffs_morton(c);
  evaluate_points(c, D, x, qu, 3, K, d_chi);
  double* g = c->buf<double>("adj_g", K);
  k_upstream<<<grid_for(K), kThreads, 0, s>>>(d_chi, d_dl, K, g);
  PR_CHECK_LAUNCH();
  st.loss = d_dl ? dot64(c, d_dl, d_chi, K) : dot64(c, d_chi, d_chi, K) / (double)K;

  // E^T g by a stable sort of (node, query-term) pairs
  uint32_t* kin = c->buf<uint32_t>("adj_kin", 8 * K);
  uint32_t* vin = c->buf<uint32_t>("adj_vin", 8 * K);
  k_eval_pairs<<<grid_for(K), kThreads, 0, s>>>(qu, K, D, kin, vin);
  PR_CHECK_LAUNCH();
  const uint64_t R = sort_and_segment(c, "adjq", kin, vin, 8 * K, D);
  double* rhs = c->buf<double>("adj_rhs", n);
  PR_CUDA(cudaMemsetAsync(rhs, 0, n * sizeof(double), s));
  if (R > 0) {
    k_eval_scatter<<<grid_for(R), kThreads, 0, s>>>(c->get<uint32_t>("adjq_runkey"), c->get<uint32_t>("adjq_runoff"),
                                                     R, c->get<uint32_t>("adjq_val"), qu, g, D, rhs);
    PR_CHECK_LAUNCH();
  }

  // adjoint solve with the forward's solver settings
  double* lam = c->buf<double>("adj_lambda", n);
  pr_stats sst;
  std::memset(&sst, 0, sizeof(sst));
  c->sync();
  const double t0 = now_seconds();
  solve_system(c, c->params, sst, rhs, lam);
  c->sync();
  st.time_solve = now_seconds() - t0;
  st.rel_residual = sst.rel_residual;
  st.pcg_iterations = sst.pcg_iterations;
  st.refinement_steps = sst.refinement_steps;
  st.converged = sst.converged;

  double* mu = c->buf<double>("adj_mu", 3 * std::max<uint64_t>(T, 1));
  if (T > 0) {
    k_mu<<<grid_for(T), kThreads, 0, s>>>(c->get<uint32_t>("splat_runkey"), T, lam, D, mu);
    PR_CHECK_LAUNCH();
  }
  const double h = 1.0 / (double)(1u << D);
  PointGradArgs a;
  a.upos = c->get<double>("upos");
  a.unrm = c->get<double>("unrm");
  a.ulen = c->get<double>("ulen");
  a.P = P;
  a.D = D;
  a.map = c->get<uint32_t>("map");
  a.nfield = c->get<double>("nfield");
  a.mu = mu;
  a.T = T;
  a.lam = lam;
  a.x = x;
  a.wh3 = c->pw > 0.0 ? c->pw * (h * h * h) / 1.5 : 0.0;
  a.s = c->M[0];
  a.dpos = d_dpos;
  a.dnrm = d_dnrm;
  k_point_grad<<<grid_for(P), kThreads, 0, s>>>(a);
  PR_CHECK_LAUNCH();
}

}  // namespace pr

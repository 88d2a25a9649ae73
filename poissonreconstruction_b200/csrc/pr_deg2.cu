// Degree-2 (quadratic B-spline) reconstruction: an extension.  The crate's degree-2 code
// (src/bspline.rs:74-123, 322-417) is not on its reconstruction path; this builds the degree-2
// system on the crate's degree-1 conventions:
//   node functions phi_i(x) = N2(x/h - i + 1), i in [0, res) per axis (cell-centred quadratic
//   B-splines, N2 the canonical quadratic B-spline of src/bspline.rs:334-345);
//   A = h (S (x) M (x) M + M (x) S (x) M + M (x) M (x) S) + wg I + wh3 sum_p phi(p) phi(p)^T, with
//   m, s the 1-D integrals of N2 N2 and N2' N2' at offsets -2..2 on every row and neighbours
//   outside the grid omitted (as the crate's degree-1 stiffness, src/fem_tree.rs:180-249);
//   b = h^2 sum_a (G (x) M (x) M)_a nf_a + (wh3 / 2) sum_p phi(p), G the 1-D integrals of N2' N2,
//   nf the normalised, negated splat of the normals with the same 27 functions per point;
//   wh3 = pw h^3 / 1.5, wg = wh3 / 200 (src/fem_tree.rs:195-200, 276-280).
//
// Layout: grid vectors in natural order (x fastest, index x + res (y + res z)).  Every operator
// is a sum of tensor products of banded 1-D matrices.  One kernel (k_op2) applies a level's
// operator in a single pass over HBM: a CTA owns 32 x 8 columns and streams up to 64 z planes;
// per plane it stages the 36 x 12 haloed input in shared memory, filters along x (M and S),
// then along y (three products) into registers, and keeps a five-plane register window for
// the z filter.  The epilogue forms A x, f - A x or a Chebyshev smoothing step.
//
// Solver: conjugate gradients preconditioned by a multigrid V-cycle on K + wg I.  Coarse
// levels are Galerkin products of the 1-D matrices (P^T X P, P the B2 subdivision
// [1/4 3/4 3/4 1/4] per axis, fine functions outside the grid omitted) with the shift wg;
// smoothing is Chebyshev of degree 3 on the Jacobi-scaled operator over [2.1 / 15, 2.1]; the
// 4^3 level is solved with a dense inverse.  FP32 inner solves with FP64 residual refinement,
// or FP64 throughout.  The solved coefficients are permuted to the Morton order of the
// degree-1 path for evaluation and marching cubes.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "pr_internal.cuh"
#include "pr_ops.cuh"

namespace pr {

namespace {

constexpr int kThreads = 256;
constexpr int TX = 32, TY = 8;           // output columns of a CTA
constexpr int SW = TX + 4, SH = TY + 4;  // staged input plane (halo 2)
constexpr int kZChunk = 64;              // output planes per CTA
constexpr int kChebSteps = 3;            // Chebyshev degree of one smoothing
constexpr double kLamMax = 2.1;          // bound of the spectrum of D^-1 (K + wg I) on every level
constexpr double kLamRatio = 15.0;       // smoothed interval [kLamMax / kLamRatio, kLamMax]

inline unsigned grid_for(uint64_t n, uint64_t cap = 1u << 22) {
  uint64_t g = (n + kThreads - 1) / kThreads;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (unsigned)g;
}

// ------------------------------------------------------------------ 1-D integrals (host)
double h_n2(double x) {
  if (x <= 0.0 || x >= 3.0) return 0.0;
  if (x <= 1.0) return 0.5 * x * x;
  if (x <= 2.0) return 0.5 * (-2.0 * x * x + 6.0 * x - 3.0);
  const double t = 3.0 - x;
  return 0.5 * t * t;
}
double h_dn2(double x) {
  if (x <= 0.0 || x >= 3.0) return 0.0;
  if (x <= 1.0) return x;
  if (x <= 2.0) return 3.0 - 2.0 * x;
  return x - 3.0;
}
// m, s, g at offsets -2..2 (index d + 2): integrals over R of N2(t) N2(t-d), N2'(t) N2'(t-d) and
// N2'(t) N2(t-d), by 3-point Gauss-Legendre per unit cell (exact for these polynomial pieces)
struct Consts {
  double m[5], s[5], g[5];
  Consts() {
    const double gx[3] = {-std::sqrt(0.6), 0.0, std::sqrt(0.6)}, gw[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
    for (int d = -2; d <= 2; ++d) {
      double am = 0, as = 0, ag = 0;
      for (int c = -1; c < 5; ++c)
        for (int q = 0; q < 3; ++q) {
          const double t = c + 0.5 + 0.5 * gx[q], w = 0.5 * gw[q];
          am += w * h_n2(t) * h_n2(t - d);
          as += w * h_dn2(t) * h_dn2(t - d);
          ag += w * h_dn2(t) * h_n2(t - d);
        }
      m[d + 2] = am;
      s[d + 2] = as;
      g[d + 2] = ag;
    }
  }
};
const Consts& consts() {
  static const Consts k;
  return k;
}

// banded 1-D matrix: row i, entry (i, i + d) for d in -2..2 at [5 i + d + 2]; 0 outside the grid
typedef std::vector<double> Band;
Band toeplitz(int res, const double* c5) {
  Band b(5 * (size_t)res, 0.0);
  for (int i = 0; i < res; ++i)
    for (int d = -2; d <= 2; ++d)
      if (i + d >= 0 && i + d < res) b[5 * i + d + 2] = c5[d + 2];
  return b;
}
// P^T X P for the subdivision P: fine 2c + k <- coarse c with weights 1/4, 3/4, 3/4, 1/4 (k = -1..2)
double sub_weight(int f, int c) {
  const int k = f - 2 * c;
  return k == -1 || k == 2 ? 0.25 : (k == 0 || k == 1 ? 0.75 : 0.0);
}
Band galerkin(const Band& X, int resf) {
  const int resc = resf / 2;
  Band out(5 * (size_t)resc, 0.0);
  for (int c = 0; c < resc; ++c)
    for (int dc = -2; dc <= 2; ++dc) {
      const int c2 = c + dc;
      if (c2 < 0 || c2 >= resc) continue;
      double v = 0.0;
      for (int f = 2 * c - 1; f <= 2 * c + 2; ++f) {
        if (f < 0 || f >= resf) continue;
        for (int d = -2; d <= 2; ++d) {
          const int f2 = f + d;
          if (f2 < 0 || f2 >= resf) continue;
          v += sub_weight(f, c) * X[5 * f + d + 2] * sub_weight(f2, c2);
        }
      }
      out[5 * c + dc + 2] = v;
    }
  return out;
}

// ------------------------------------------------------------------ the level operator
template <typename T>
struct LevelView {
  const T* tM;  // 5 res: banded 1-D mass matrix of the level
  const T* tS;  // 5 res: banded 1-D stiffness matrix
  int L;        // log2 res
  T H, wg;      // A = H (S M M + M S M + M M S) + wg I
};

enum { kOpApply = 0, kOpResid = 1, kOpCheb = 2 };

// One pass of the level operator over a CTA's 32 x 8 columns and up to kZChunk planes.
//   kOpApply: out = A x
//   kOpResid: out = f - A x
//   kOpCheb:  out = x + ca (x - xp) + cb D^-1 (f - A x)   (xp null: previous iterate 0); out may
//             alias xp (each element is read before it is written by the same thread), never x.
template <typename T, int MODE>
__global__ void __launch_bounds__(kThreads) k_op2(const T* __restrict__ x, const T* __restrict__ f, const T* xp,
                                                  T* out, LevelView<T> lv, T ca, T cb) {
  __shared__ T s_in[SH][SW];
  __shared__ T s_um[SH][TX];
  __shared__ T s_us[SH][TX];
  const int res = 1 << lv.L;
  const int64_t plane = (int64_t)res * res;
  const int t = threadIdx.x, tx = t & 31, ty = t >> 5;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  const int z0 = blockIdx.z * kZChunk, z1 = min(z0 + kZChunk, res);
  const int gx = x0 + tx, gy = y0 + ty;
  const bool own = gx < res && gy < res;
  T cmx[5], csx[5], cmy[5], csy[5];
#pragma unroll
  for (int d = 0; d < 5; ++d) {
    cmx[d] = gx < res ? lv.tM[5 * gx + d] : T(0);
    csx[d] = gx < res ? lv.tS[5 * gx + d] : T(0);
    cmy[d] = gy < res ? lv.tM[5 * gy + d] : T(0);
    csy[d] = gy < res ? lv.tS[5 * gy + d] : T(0);
  }
  // the (at most two) staged elements of this thread
  const int e0 = t, e1 = t + kThreads;
  const bool has1 = e1 < SH * SW;
  const int r0 = e0 / SW, c0 = e0 % SW, r1 = has1 ? e1 / SW : 0, c1 = has1 ? e1 % SW : 0;
  const int X0 = x0 - 2 + c0, Y0 = y0 - 2 + r0, X1 = x0 - 2 + c1, Y1 = y0 - 2 + r1;
  const bool ok0 = X0 >= 0 && X0 < res && Y0 >= 0 && Y0 < res;
  const bool ok1 = has1 && X1 >= 0 && X1 < res && Y1 >= 0 && Y1 < res;
  const int64_t o0 = ok0 ? (int64_t)X0 + (int64_t)res * Y0 : 0, o1 = ok1 ? (int64_t)X1 + (int64_t)res * Y1 : 0;
  T p0, p1;
  {
    const int z = z0 - 2;
    const bool zin = z >= 0 && z < res;
    p0 = (ok0 && zin) ? x[o0 + z * plane] : T(0);
    p1 = (ok1 && zin) ? x[o1 + z * plane] : T(0);
  }
  T wa[5], wb[5], wc[3];  // windows: M-filtered (S M + M S) terms, S-filtered M M terms, centre x
#pragma unroll
  for (int k = 0; k < 5; ++k) wa[k] = wb[k] = T(0);
  wc[0] = wc[1] = wc[2] = T(0);
  for (int zin = z0 - 2; zin <= z1 + 1; ++zin) {
    s_in[r0][c0] = p0;
    if (has1) s_in[r1][c1] = p1;
    __syncthreads();
    {
      const int z = zin + 1;
      const bool zin_ok = z >= 0 && z < res && z <= z1 + 1;
      p0 = (ok0 && zin_ok) ? x[o0 + z * plane] : T(0);
      p1 = (ok1 && zin_ok) ? x[o1 + z * plane] : T(0);
    }
    // x filter: rows ty and ty + 8 of the 12 staged rows
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int r = ty + 8 * k;
      if (r < SH) {
        T um = 0, us = 0;
#pragma unroll
        for (int d = 0; d < 5; ++d) {
          const T v = s_in[r][tx + d];
          um += cmx[d] * v;
          us += csx[d] * v;
        }
        s_um[r][tx] = um;
        s_us[r][tx] = us;
      }
    }
    const T xc = s_in[ty + 2][tx + 2];
    __syncthreads();
    // y filter into registers
    T vmm = 0, vsm = 0, vms = 0;
#pragma unroll
    for (int d = 0; d < 5; ++d) {
      const T a = s_um[ty + d][tx], b = s_us[ty + d][tx];
      vmm += cmy[d] * a;
      vsm += cmy[d] * b;
      vms += csy[d] * a;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      wa[k] = wa[k + 1];
      wb[k] = wb[k + 1];
    }
    wa[4] = vsm + vms;
    wb[4] = vmm;
    wc[0] = wc[1];
    wc[1] = wc[2];
    wc[2] = xc;
    const int zo = zin - 2;
    if (own && zo >= z0 && zo < z1) {
      T cmz[5], csz[5];
#pragma unroll
      for (int d = 0; d < 5; ++d) {
        cmz[d] = lv.tM[5 * zo + d];
        csz[d] = lv.tS[5 * zo + d];
      }
      T acc = 0;
#pragma unroll
      for (int d = 0; d < 5; ++d) acc += cmz[d] * wa[d] + csz[d] * wb[d];
      const T xo = wc[0];
      const T ax = lv.H * acc + lv.wg * xo;
      const int64_t i = (int64_t)gx + (int64_t)res * gy + plane * zo;
      if (MODE == kOpApply) {
        out[i] = ax;
      } else if (MODE == kOpResid) {
        out[i] = f[i] - ax;
      } else {
        const T r = f[i] - ax;
        const T dg = lv.H * (csx[2] * cmy[2] * cmz[2] + cmx[2] * csy[2] * cmz[2] + cmx[2] * cmy[2] * csz[2]) + lv.wg;
        const T prev = xp ? xp[i] : T(0);
        out[i] = xo + ca * (xo - prev) + cb * r / dg;
      }
    }
  }
}

// first Chebyshev step from x = 0: out = cb D^-1 f
template <typename T>
__global__ void k_cheb_first2(const T* __restrict__ f, T* __restrict__ out, LevelView<T> lv, T cb) {
  const int L = lv.L;
  const uint64_t n = 1ull << (3 * L), m = (1ull << L) - 1;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i & m), y = (int)((i >> L) & m), z = (int)(i >> (2 * L));
    const T mx = lv.tM[5 * x + 2], my = lv.tM[5 * y + 2], mz = lv.tM[5 * z + 2];
    const T sx = lv.tS[5 * x + 2], sy = lv.tS[5 * y + 2], sz = lv.tS[5 * z + 2];
    const T dg = lv.H * (sx * my * mz + mx * sy * mz + mx * my * sz) + lv.wg;
    out[i] = cb * f[i] / dg;
  }
}

// fc = P^T rf (fine level Lf -> coarse Lf - 1): coarse c <- fine 2c + k, k = -1..2 per axis
template <typename T>
__global__ void k_restrict2(const T* __restrict__ rf, int Lf, T* __restrict__ fc) {
  const int Lc = Lf - 1, rf_res = 1 << Lf;
  const uint64_t nc = 1ull << (3 * Lc), m = (1ull << Lc) - 1;
  const int64_t pf = (int64_t)rf_res * rf_res;
  const T w[4] = {T(0.25), T(0.75), T(0.75), T(0.25)};
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nc; i += (uint64_t)gridDim.x * blockDim.x) {
    const int cx = (int)(i & m), cy = (int)((i >> Lc) & m), cz = (int)(i >> (2 * Lc));
    T acc = 0;
#pragma unroll
    for (int kz = 0; kz < 4; ++kz) {
      const int fz = 2 * cz - 1 + kz;
      if (fz < 0 || fz >= rf_res) continue;
      T az = 0;
#pragma unroll
      for (int ky = 0; ky < 4; ++ky) {
        const int fy = 2 * cy - 1 + ky;
        if (fy < 0 || fy >= rf_res) continue;
        const T* row = rf + fz * pf + (int64_t)fy * rf_res;
        T ay = 0;
#pragma unroll
        for (int kx = 0; kx < 4; ++kx) {
          const int fx = 2 * cx - 1 + kx;
          if (fx >= 0 && fx < rf_res) ay += w[kx] * row[fx];
        }
        az += w[ky] * ay;
      }
      acc += w[kz] * az;
    }
    fc[i] = acc;
  }
}

// out = xf + P ec (coarse Lf - 1 -> fine Lf); fine f <- coarse f/2 (3/4) and f/2 - 1 (1/4) for f
// even, (f-1)/2 (3/4) and (f+1)/2 (1/4) for f odd
template <typename T>
__global__ void k_prolong2(const T* __restrict__ xf, const T* __restrict__ ec, int Lf, T* __restrict__ out) {
  const int Lc = Lf - 1, rc = 1 << Lc;
  const uint64_t n = 1ull << (3 * Lf), m = (1ull << Lf) - 1;
  const int64_t pc = (int64_t)rc * rc;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const int f[3] = {(int)(i & m), (int)((i >> Lf) & m), (int)(i >> (2 * Lf))};
    int c[3][2];
    T w[3][2];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      c[a][0] = f[a] >> 1;
      w[a][0] = T(0.75);
      c[a][1] = (f[a] & 1) ? (f[a] >> 1) + 1 : (f[a] >> 1) - 1;
      w[a][1] = (c[a][1] >= 0 && c[a][1] < rc) ? T(0.25) : T(0);
      if (w[a][1] == T(0)) c[a][1] = c[a][0];
    }
    T acc = 0;
#pragma unroll
    for (int kz = 0; kz < 2; ++kz)
#pragma unroll
      for (int ky = 0; ky < 2; ++ky) {
        const T* row = ec + c[2][kz] * pc + (int64_t)c[1][ky] * rc;
        acc += w[2][kz] * w[1][ky] * (w[0][0] * row[c[0][0]] + w[0][1] * row[c[0][1]]);
      }
    out[i] = xf[i] + acc;
  }
}

// ------------------------------------------------------------------ setup kernels
// degree-2 basis of one axis at unit coordinate u: nodes c-1, c, c+1 (the oracle's expressions)
__device__ __forceinline__ void axis2(double u, double h, int64_t& c, double* b) {
  const double s = xdiv(u, h);
  c = sat_i64(floor(s));
  const double t = xsub(s, (double)c);
  const double omt = xsub(1.0, t);
  b[0] = xmul(xmul(0.5, omt), omt);
  b[1] = xmul(0.5, xadd(xadd(xmul(xmul(-2.0, t), t), xmul(2.0, t)), 1.0));
  b[2] = xmul(xmul(0.5, t), t);
}

// (node, 27 p + k) pairs with the natural node index (sentinel 2^(3D) outside the grid), k =
// 9 (dz + 1) + 3 (dy + 1) + (dx + 1); basis values (FP64, FP32); count of points with a node
__global__ void k_pair_keys2(const double* __restrict__ upos, uint64_t P, uint32_t D, uint32_t* __restrict__ keys,
                             uint32_t* __restrict__ vals, double* __restrict__ phi64, float* __restrict__ phi32,
                             unsigned long long* __restrict__ nin) {
  const int64_t res = 1ll << D;
  const double h = 1.0 / (double)res;
  const uint32_t sentinel = 1u << (3 * D);
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < P; p += (uint64_t)gridDim.x * blockDim.x) {
    int64_t c[3];
    double b[3][3];
    axis2(upos[p], h, c[0], b[0]);
    axis2(upos[P + p], h, c[1], b[1]);
    axis2(upos[2 * P + p], h, c[2], b[2]);
    bool any = false;
    for (int k = 0; k < 27; ++k) {
      const int dx = k % 3, dy = (k / 3) % 3, dz = k / 9;
      const int64_t x = c[0] + dx - 1, y = c[1] + dy - 1, z = c[2] + dz - 1;
      const bool ok = x >= 0 && y >= 0 && z >= 0 && x < res && y < res && z < res;
      any |= ok;
      keys[27 * p + k] = ok ? (uint32_t)(x + res * (y + res * z)) : sentinel;
      vals[27 * p + k] = (uint32_t)(27 * p + k);
      const double phi = ok ? xmul(xmul(b[0][dx], b[1][dy]), b[2][dz]) : 0.0;
      phi64[27 * p + k] = phi;
      phi32[27 * p + k] = (float)phi;
    }
    if (any) atomicAdd(nin, 1ull);
  }
}

// splat per touched node, points in input order: nf = -(sum phi n) / (sum phi), w = sum phi
__global__ void k_splat2(const uint32_t* __restrict__ run_key, const uint32_t* __restrict__ run_off, uint64_t T,
                         const uint32_t* __restrict__ sval, const double* __restrict__ phi,
                         const double* __restrict__ unrm, uint64_t P, uint64_t n, double* __restrict__ nf,
                         double* __restrict__ w) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < T; t += (uint64_t)gridDim.x * blockDim.x) {
    double fx = 0.0, fy = 0.0, fz = 0.0, sw = 0.0;
    for (uint32_t e = run_off[t]; e < run_off[t + 1]; ++e) {
      const uint32_t pk = sval[e];
      const uint32_t p = pk / 27;
      const double wgt = phi[pk];
      fx = xadd(fx, xmul(unrm[p], wgt));
      fy = xadd(fy, xmul(unrm[P + p], wgt));
      fz = xadd(fz, xmul(unrm[2 * P + p], wgt));
      sw = xadd(sw, wgt);
    }
    if (sw > 0.0) {
      fx = xdiv(-fx, sw);
      fy = xdiv(-fy, sw);
      fz = xdiv(-fz, sw);
    }
    const uint32_t node = run_key[t];
    nf[node] = fx;
    nf[n + node] = fy;
    nf[2 * n + node] = fz;
    w[node] = sw;
  }
}

// b = h^2 sum_a (G_a M M) nf_a on the finest level, streamed like k_op2 (three inputs)
struct RhsCoef {
  double g[5], m[5], h2;
};
__global__ void __launch_bounds__(kThreads) k_rhs2(const double* __restrict__ nf, int L, RhsCoef k,
                                                   double* __restrict__ b) {
  __shared__ double s_in[3][SH][SW];
  __shared__ double s_u[3][SH][TX];
  const int res = 1 << L;
  const int64_t plane = (int64_t)res * res, n = plane * res;
  const int t = threadIdx.x, tx = t & 31, ty = t >> 5;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  const int z0 = blockIdx.z * kZChunk, z1 = min(z0 + kZChunk, res);
  const int gx = x0 + tx, gy = y0 + ty;
  const bool own = gx < res && gy < res;
  const int e0 = t, e1 = t + kThreads;
  const bool has1 = e1 < SH * SW;
  const int r0 = e0 / SW, c0 = e0 % SW, r1 = has1 ? e1 / SW : 0, c1 = has1 ? e1 % SW : 0;
  const int X0 = x0 - 2 + c0, Y0 = y0 - 2 + r0, X1 = x0 - 2 + c1, Y1 = y0 - 2 + r1;
  const bool ok0 = X0 >= 0 && X0 < res && Y0 >= 0 && Y0 < res;
  const bool ok1 = has1 && X1 >= 0 && X1 < res && Y1 >= 0 && Y1 < res;
  const int64_t o0 = ok0 ? (int64_t)X0 + (int64_t)res * Y0 : 0, o1 = ok1 ? (int64_t)X1 + (int64_t)res * Y1 : 0;
  double wa[5], wb[5];
#pragma unroll
  for (int q = 0; q < 5; ++q) wa[q] = wb[q] = 0.0;
  for (int zin = z0 - 2; zin <= z1 + 1; ++zin) {
    const bool zok = zin >= 0 && zin < res;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      s_in[a][r0][c0] = (ok0 && zok) ? nf[a * n + o0 + zin * plane] : 0.0;
      if (has1) s_in[a][r1][c1] = (ok1 && zok) ? nf[a * n + o1 + zin * plane] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int r = ty + 8 * q;
      if (r < SH) {
        double u0 = 0.0, u1 = 0.0, u2 = 0.0;
#pragma unroll
        for (int d = 0; d < 5; ++d) {
          u0 += k.g[d] * s_in[0][r][tx + d];
          u1 += k.m[d] * s_in[1][r][tx + d];
          u2 += k.m[d] * s_in[2][r][tx + d];
        }
        s_u[0][r][tx] = u0;
        s_u[1][r][tx] = u1;
        s_u[2][r][tx] = u2;
      }
    }
    __syncthreads();
    double v0 = 0.0, v1 = 0.0, v2 = 0.0;
#pragma unroll
    for (int d = 0; d < 5; ++d) {
      v0 += k.m[d] * s_u[0][ty + d][tx];
      v1 += k.g[d] * s_u[1][ty + d][tx];
      v2 += k.m[d] * s_u[2][ty + d][tx];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      wa[q] = wa[q + 1];
      wb[q] = wb[q + 1];
    }
    wa[4] = v0 + v1;
    wb[4] = v2;
    const int zo = zin - 2;
    if (own && zo >= z0 && zo < z1) {
      double acc = 0.0;
#pragma unroll
      for (int d = 0; d < 5; ++d) acc += k.m[d] * wa[d] + k.g[d] * wb[d];
      b[(int64_t)gx + (int64_t)res * gy + plane * zo] = k.h2 * acc;
    }
  }
}

// screening right-hand side: b[node] += (wh3 / 2) sum of phi over the node's pairs
__global__ void k_screen_rhs2(const uint32_t* __restrict__ snode, const uint32_t* __restrict__ soff, uint64_t S,
                              const uint32_t* __restrict__ sval, const double* __restrict__ phi, double wt,
                              double* __restrict__ b) {
  for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < S; u += (uint64_t)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (uint32_t e = soff[u]; e < soff[u + 1]; ++e) acc += phi[sval[e]];
    b[snode[u]] += wt * acc;
  }
}

// screening operator wh3 Phi (Phi^T x): per point projection, then a per node gather
template <typename T>
__global__ void k_screen_proj2(const uint32_t* __restrict__ key, const T* __restrict__ phi, uint64_t P,
                               uint32_t sentinel, const T* __restrict__ x, T* __restrict__ proj) {
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < P; p += (uint64_t)gridDim.x * blockDim.x) {
    T s = 0;
    for (int k = 0; k < 27; ++k) {
      const uint32_t kk = key[27 * p + k];
      if (kk != sentinel) s += phi[27 * p + k] * x[kk];
    }
    proj[p] = s;
  }
}
template <typename T>
__global__ void k_screen_gather2(const uint32_t* __restrict__ snode, const uint32_t* __restrict__ soff, uint64_t S,
                                 const uint32_t* __restrict__ sval, const T* __restrict__ phi,
                                 const T* __restrict__ proj, T wh3s, T* __restrict__ y) {
  for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < S; u += (uint64_t)gridDim.x * blockDim.x) {
    T acc = 0;
    for (uint32_t e = soff[u]; e < soff[u + 1]; ++e) {
      const uint32_t pk = sval[e];
      acc += phi[pk] * proj[pk / 27];
    }
    y[snode[u]] += wh3s * acc;
  }
}

// natural <-> Morton
template <typename T>
__global__ void k_nat_to_morton(const T* __restrict__ in, uint32_t D, T* __restrict__ out) {
  const uint64_t n = 1ull << (3 * D), m = (1ull << D) - 1;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[morton3((uint32_t)(i & m), (uint32_t)((i >> D) & m), (uint32_t)(i >> (2 * D)))] = in[i];
}
template <typename T>
__global__ void k_morton_to_nat(const T* __restrict__ in, uint32_t D, T* __restrict__ out) {
  const uint64_t n = 1ull << (3 * D), m = (1ull << D) - 1;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = in[morton3((uint32_t)(i & m), (uint32_t)((i >> D) & m), (uint32_t)(i >> (2 * D)))];
}
// AoS (n x 3, Morton) from three natural-order components
__global__ void k_nat3_to_morton_aos(const double* __restrict__ nf, uint32_t D, double* __restrict__ out) {
  const uint64_t n = 1ull << (3 * D), m = (1ull << D) - 1;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t j = morton3((uint32_t)(i & m), (uint32_t)((i >> D) & m), (uint32_t)(i >> (2 * D)));
    out[3 * j] = nf[i];
    out[3 * j + 1] = nf[n + i];
    out[3 * j + 2] = nf[2 * n + i];
  }
}

// ------------------------------------------------------------------ host: the system
template <typename T>
struct Level2 {
  int L = 0;
  uint64_t n = 0;
  T* tM = nullptr;
  T* tS = nullptr;
  double H = 0, wg = 0;
  T* f = nullptr;  // right-hand side (coarse levels)
  T* x = nullptr;  // iterate (coarse levels)
  T* y = nullptr;  // scratch
  LevelView<T> view() const { return LevelView<T>{tM, tS, L, (T)H, (T)wg}; }
};

template <typename T>
struct Screen2 {
  const uint32_t* key = nullptr;   // 27 P node keys (natural index or sentinel)
  const T* phi = nullptr;          // 27 P basis values
  const uint32_t* snode = nullptr; // S screened nodes
  const uint32_t* soff = nullptr;  // S + 1
  const uint32_t* sval = nullptr;  // node-sorted pairs 27 p + k
  uint64_t P = 0, S = 0, pairs = 0;
  uint32_t sentinel = 0;
  double wh3 = 0;
  T* proj = nullptr;
};

template <typename T>
const char* tn2() {
  return sizeof(T) == 4 ? "f32" : "f64";
}

template <typename T>
struct System2 {
  pr_context* c = nullptr;
  uint32_t D = 0;
  std::vector<Level2<T>> lv;  // lv[0] finest
  T* inv = nullptr;           // dense inverse of the coarsest level
  int nc = 0;
  Screen2<T> scr;
  double bytes = 0.0;         // algorithmic HBM bytes of the launched kernels

  // levels D (finest) down to the dense 4^3 level; `multigrid` false: the finest level only
  void init(pr_context* ctx, uint32_t depth, double pw, bool multigrid) {
    c = ctx;
    D = depth;
    const double h = 1.0 / (double)(1u << D);
    const double wh3 = pw > 0.0 ? pw * h * h * h / 1.5 : 0.0;
    const double wg = wh3 * 0.005;
    const std::string tn = tn2<T>();
    Band M = toeplitz(1 << D, consts().m), S = toeplitz(1 << D, consts().s);
    const int lmin = multigrid ? std::min<int>((int)D, 2) : (int)D;
    lv.clear();
    for (int l = (int)D; l >= lmin; --l) {
      Level2<T> q;
      q.L = l;
      q.n = 1ull << (3 * l);
      q.H = h;
      q.wg = wg;
      const std::string sfx = std::string("_") + tn + "_" + std::to_string(l);
      auto upload = [&](const Band& b, const std::string& nm) {
        std::vector<T> tb(b.begin(), b.end());
        T* p = c->buf<T>("d2_" + nm + sfx, tb.size());
        PR_CUDA(cudaMemcpyAsync(p, tb.data(), tb.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream));
        c->sync();
        return p;
      };
      q.tM = upload(M, "tM");
      q.tS = upload(S, "tS");
      if (multigrid) {
        q.y = c->buf<T>("d2_y" + sfx, q.n);
        if (l != (int)D) {
          q.f = c->buf<T>("d2_f" + sfx, q.n);
          q.x = c->buf<T>("d2_x" + sfx, q.n);
        }
      }
      lv.push_back(q);
      if (l == lmin) {
        if (multigrid) build_dense(M, S, 1 << l, wg, h);
        break;
      }
      M = galerkin(M, 1 << l);
      S = galerkin(S, 1 << l);
    }
  }

  // dense inverse of the coarsest operator (Cholesky on the host, FP64)
  void build_dense(const Band& M, const Band& S, int r, double wg, double H) {
    nc = r * r * r;
    std::vector<double> A((size_t)nc * nc, 0.0);
    auto at = [&](const Band& b, int i, int j) { return (j - i >= -2 && j - i <= 2) ? b[5 * i + (j - i) + 2] : 0.0; };
    for (int i = 0; i < nc; ++i)
      for (int j = 0; j < nc; ++j) {
        const int ix = i % r, iy = (i / r) % r, iz = i / (r * r), jx = j % r, jy = (j / r) % r, jz = j / (r * r);
        double v = H * (at(S, ix, jx) * at(M, iy, jy) * at(M, iz, jz) + at(M, ix, jx) * at(S, iy, jy) * at(M, iz, jz) +
                        at(M, ix, jx) * at(M, iy, jy) * at(S, iz, jz));
        if (i == j) v += wg;
        A[(size_t)i * nc + j] = v;
      }
    std::vector<double> Lc((size_t)nc * nc, 0.0);
    for (int i = 0; i < nc; ++i)
      for (int j = 0; j <= i; ++j) {
        double s = A[(size_t)i * nc + j];
        for (int k = 0; k < j; ++k) s -= Lc[(size_t)i * nc + k] * Lc[(size_t)j * nc + k];
        if (i == j) {
          PR_REQUIRE(s > 0.0, PR_ERR_INTERNAL, "degree-2 coarsest operator is not positive definite");
          Lc[(size_t)i * nc + i] = std::sqrt(s);
        } else {
          Lc[(size_t)i * nc + j] = s / Lc[(size_t)j * nc + j];
        }
      }
    std::vector<T> invt((size_t)nc * nc);
    std::vector<double> y(nc), col(nc);
    for (int cc = 0; cc < nc; ++cc) {
      for (int i = 0; i < nc; ++i) {
        double s = (i == cc) ? 1.0 : 0.0;
        for (int k = 0; k < i; ++k) s -= Lc[(size_t)i * nc + k] * y[k];
        y[i] = s / Lc[(size_t)i * nc + i];
      }
      for (int i = nc - 1; i >= 0; --i) {
        double s = y[i];
        for (int k = i + 1; k < nc; ++k) s -= Lc[(size_t)k * nc + i] * col[k];
        col[i] = s / Lc[(size_t)i * nc + i];
      }
      for (int i = 0; i < nc; ++i) invt[(size_t)i * nc + cc] = (T)col[i];
    }
    inv = c->buf<T>(std::string("d2_inv_") + tn2<T>(), invt.size());
    PR_CUDA(cudaMemcpyAsync(inv, invt.data(), invt.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream));
    c->sync();
  }

  void set_screen(const T* phi) {
    if (!(c->pw > 0.0) || c->S == 0) return;
    const double h = 1.0 / (double)(1u << D);
    scr.key = c->get<uint32_t>("d2_kin");
    scr.phi = phi;
    scr.snode = c->get<uint32_t>("d2s_runkey");
    scr.soff = c->get<uint32_t>("d2s_runoff");
    scr.sval = c->get<uint32_t>("d2s_val");
    scr.P = c->P;
    scr.S = c->S;
    scr.pairs = c->S_pairs;
    scr.sentinel = 1u << (3 * D);
    scr.wh3 = c->pw * h * h * h / 1.5;
    scr.proj = c->buf<T>(std::string("d2_proj_") + tn2<T>(), c->P);
  }

  // y += sign wh3 Phi Phi^T x
  void screen(const T* x, T* y, int sign) {
    if (scr.S == 0) return;
    cudaStream_t s = c->stream;
    k_screen_proj2<T><<<grid_for(scr.P, 1u << 20), kThreads, 0, s>>>(scr.key, scr.phi, scr.P, scr.sentinel, x,
                                                                      scr.proj);
    PR_CHECK_LAUNCH();
    k_screen_gather2<T><<<grid_for(scr.S, 1u << 20), kThreads, 0, s>>>(scr.snode, scr.soff, scr.S, scr.sval, scr.phi,
                                                                        scr.proj, (T)(sign * scr.wh3), y);
    PR_CHECK_LAUNCH();
    bytes += (double)scr.P * 27 * (4 + 2 * sizeof(T)) + (double)scr.P * sizeof(T) +
             (double)scr.pairs * (4 + 2 * sizeof(T)) + (double)scr.S * (8 + 2 * sizeof(T));
  }

  void op(int li, int mode, const T* x, const T* f, const T* xp, T* out, double a = 0.0, double b = 0.0) {
    const Level2<T>& q = lv[li];
    const int res = 1 << q.L;
    dim3 grid((res + TX - 1) / TX, (res + TY - 1) / TY, (res + kZChunk - 1) / kZChunk);
    cudaStream_t s = c->stream;
    const LevelView<T> v = q.view();
    if (mode == kOpApply) k_op2<T, kOpApply><<<grid, kThreads, 0, s>>>(x, f, xp, out, v, (T)a, (T)b);
    else if (mode == kOpResid) k_op2<T, kOpResid><<<grid, kThreads, 0, s>>>(x, f, xp, out, v, (T)a, (T)b);
    else k_op2<T, kOpCheb><<<grid, kThreads, 0, s>>>(x, f, xp, out, v, (T)a, (T)b);
    PR_CHECK_LAUNCH();
    bytes += (double)q.n * sizeof(T) * (2 + (mode != kOpApply ? 1 : 0) + (xp ? 1 : 0));
  }

  // Chebyshev smoothing on level li.  From zero (pre-smoothing): x1 in x, x2 in y, x3 in x.
  // From y0 held in y (post-smoothing): y1 in x, y2 in y, y3 in x.
  void chebyshev(int li, const T* f, T* x, T* y, bool from_zero) {
    const Level2<T>& q = lv[li];
    const double hi = kLamMax, lo = kLamMax / kLamRatio;
    const double th = 0.5 * (hi + lo), de = 0.5 * (hi - lo), sig = th / de;
    double rho = 1.0 / sig;
    if (from_zero) {
      k_cheb_first2<T><<<grid_for(q.n), kThreads, 0, c->stream>>>(f, x, q.view(), (T)(1.0 / th));
      PR_CHECK_LAUNCH();
      bytes += 2.0 * q.n * sizeof(T);
    } else {
      op(li, kOpCheb, y, f, nullptr, x, 0.0, 1.0 / th);
    }
    T* cur = x;
    T* prev = from_zero ? nullptr : y;
    for (int k = 1; k < kChebSteps; ++k) {
      const double rn = 1.0 / (2.0 * sig - rho);
      T* dst = (cur == x) ? y : x;
      op(li, kOpCheb, cur, f, prev, dst, rn * rho, 2.0 * rn / de);
      prev = cur;
      cur = dst;
      rho = rn;
    }
    PR_REQUIRE(cur == x, PR_ERR_INTERNAL, "Chebyshev smoothing must end in its output buffer");
  }

  // X = V(f) on level li (f read only)
  void vcycle(int li, const T* f, T* X) {
    cudaStream_t s = c->stream;
    if (li == (int)lv.size() - 1) {
      dense_solve<T>(s, (uint32_t)nc, inv, f, X);
      bytes += 2.0 * nc * sizeof(T);
      return;
    }
    Level2<T>& q = lv[li];
    Level2<T>& qc = lv[li + 1];
    chebyshev(li, f, X, q.y, true);
    op(li, kOpResid, X, f, nullptr, q.y);
    k_restrict2<T><<<grid_for(qc.n), kThreads, 0, s>>>(q.y, q.L, qc.f);
    PR_CHECK_LAUNCH();
    bytes += (double)(q.n + qc.n) * sizeof(T);
    vcycle(li + 1, qc.f, qc.x);
    k_prolong2<T><<<grid_for(q.n), kThreads, 0, s>>>(X, qc.x, q.L, q.y);
    PR_CHECK_LAUNCH();
    bytes += (double)(2 * q.n + qc.n) * sizeof(T);
    chebyshev(li, f, X, q.y, false);
  }
};

// preconditioned CG on the finest level from x = 0 to ||r|| <= tol_abs; r holds b on entry and
// is overwritten with the recursively updated residual
template <typename T>
int pcg2(pr_context* c, System2<T>& sys, T* r, T* x, double tol_abs, int maxit) {
  const uint64_t n = sys.lv[0].n;
  cudaStream_t s = c->stream;
  const std::string tn = tn2<T>();
  T* z = c->buf<T>("d2cg_z_" + tn, n);
  T* d = c->buf<T>("d2cg_d_" + tn, n);
  T* q = c->buf<T>("d2cg_q_" + tn, n);
  PR_CUDA(cudaMemsetAsync(x, 0, n * sizeof(T), s));
  double rr = dot<T>(c, r, r, n);
  sys.bytes += 2.0 * n * sizeof(T);
  if (!(std::sqrt(rr) > tol_abs)) return 0;
  sys.vcycle(0, r, z);
  double rz = dot<T>(c, r, z, n);
  PR_CUDA(cudaMemcpyAsync(d, z, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
  sys.bytes += 4.0 * n * sizeof(T);
  int it = 0;
  while (it < maxit) {
    sys.op(0, kOpApply, d, nullptr, nullptr, q);
    sys.screen(d, q, +1);
    const double dq = dot<T>(c, d, q, n);
    if (!(dq > 0.0) || !(rz > 0.0)) break;
    const double alpha = rz / dq;
    rr = cg_update<T>(c, n, alpha, d, q, x, r);
    sys.bytes += 8.0 * n * sizeof(T);
    ++it;
    if (!std::isfinite(rr) || std::sqrt(rr) <= tol_abs) break;
    sys.vcycle(0, r, z);
    const double rz_new = dot<T>(c, r, z, n);
    const double beta = rz_new / rz;
    rz = rz_new;
    xpby<T>(s, n, z, beta, d);
    sys.bytes += 5.0 * n * sizeof(T);
  }
  return it;
}

}  // namespace

// ------------------------------------------------------------------ stages
// Splat, right-hand side and screening payload of the degree-2 system (natural order).
void stage_setup_deg2(pr_context* c, uint32_t D, double pw) {
  const uint64_t P = c->P;
  const uint64_t n = 1ull << (3 * D);
  const uint64_t m = 27 * P;
  PR_REQUIRE(m < (1ull << 31), PR_ERR_INVALID_ARGUMENT, "degree 2 takes at most 79,536,431 points per call");
  c->D = D;
  c->n = n;
  c->pw = pw;
  cudaStream_t s = c->stream;
  const double* upos = c->get<double>("upos");
  const double* unrm = c->get<double>("unrm");
  uint32_t* kin = c->buf<uint32_t>("d2_kin", m);
  uint32_t* vin = c->buf<uint32_t>("d2_vin", m);
  double* phi64 = c->buf<double>("d2_phi64", m);
  float* phi32 = c->buf<float>("d2_phi32", m);
  unsigned long long* nin = c->buf<unsigned long long>("d2_nin", 1);
  PR_CUDA(cudaMemsetAsync(nin, 0, sizeof(unsigned long long), s));
  k_pair_keys2<<<grid_for(P, 1u << 20), kThreads, 0, s>>>(upos, P, D, kin, vin, phi64, phi32, nin);
  PR_CHECK_LAUNCH();
  const uint64_t T = sort_and_segment(c, "d2s", kin, vin, m, D);
  unsigned long long h_nin = 0;
  PR_CUDA(cudaMemcpyAsync(&h_nin, nin, sizeof(h_nin), cudaMemcpyDeviceToHost, s));
  uint32_t h_pairs = 0;
  if (T > 0)
    PR_CUDA(cudaMemcpyAsync(&h_pairs, c->get<uint32_t>("d2s_runoff") + T, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  c->sync();
  c->T = T;
  c->P_in = h_nin;
  double* nf = c->buf<double>("d2_nf", 3 * n);
  double* w = c->buf<double>("d2_w", n);
  PR_CUDA(cudaMemsetAsync(nf, 0, 3 * n * sizeof(double), s));
  PR_CUDA(cudaMemsetAsync(w, 0, n * sizeof(double), s));
  if (T > 0) {
    k_splat2<<<grid_for(T, 1u << 20), kThreads, 0, s>>>(c->get<uint32_t>("d2s_runkey"), c->get<uint32_t>("d2s_runoff"),
                                                        T, c->get<uint32_t>("d2s_val"), phi64, unrm, P, n, nf, w);
    PR_CHECK_LAUNCH();
  }
  const double h = 1.0 / (double)(1u << D);
  RhsCoef k;
  for (int d = 0; d < 5; ++d) {
    k.g[d] = consts().g[d];
    k.m[d] = consts().m[d];
  }
  k.h2 = h * h;
  double* b = c->buf<double>("d2_b", n);
  const int res = 1 << D;
  dim3 grid((res + TX - 1) / TX, (res + TY - 1) / TY, (res + kZChunk - 1) / kZChunk);
  k_rhs2<<<grid, kThreads, 0, s>>>(nf, (int)D, k, b);
  PR_CHECK_LAUNCH();
  c->S = 0;
  c->S_pairs = 0;
  if (pw > 0.0 && T > 0) {
    // screening payload: the node-sorted (node, 27 p + k) pairs of the splat
    c->S = T;
    c->S_pairs = h_pairs;
    const double wh3 = pw * h * h * h / 1.5;
    k_screen_rhs2<<<grid_for(T, 1u << 20), kThreads, 0, s>>>(c->get<uint32_t>("d2s_runkey"),
                                                             c->get<uint32_t>("d2s_runoff"), T,
                                                             c->get<uint32_t>("d2s_val"), phi64, 0.5 * wh3, b);
    PR_CHECK_LAUNCH();
  }
  c->have_state = true;
}

// Solve of the degree-2 system; fills "d2_x" (natural order) and "x64" (Morton order).
void stage_solve_deg2(pr_context* c, const pr_params& p, pr_stats& st) {
  const uint32_t D = c->D;
  const uint64_t n = c->n;
  cudaStream_t s = c->stream;
  const double* b = c->get<double>("d2_b");
  double* x = c->buf<double>("d2_x", n);
  double* r = c->buf<double>("d2_r", n);
  PR_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), s));
  const double target = p.target_rel_residual > 0.0 ? p.target_rel_residual : 1e-6;
  const int max_iters = p.max_iters > 0 ? (int)p.max_iters : 200;
  const bool mixed = p.precision != PR_PRECISION_FP64;
  st.pcg_iterations = 0;
  st.refinement_steps = 0;
  const double bn = std::sqrt(dot<double>(c, b, b, n));
  double bytes = 2.0 * n * 8;
  System2<double> sys64;
  sys64.init(c, D, c->pw, !mixed);
  sys64.set_screen(c->get<double>("d2_phi64"));
  double rn = bn;
  int used = 0;
  if (bn > 0.0) {
    if (mixed) {
      System2<float> sys32;
      sys32.init(c, D, c->pw, true);
      sys32.set_screen(c->get<float>("d2_phi32"));
      float* r32 = c->buf<float>("d2_r32", n);
      float* e32 = c->buf<float>("d2_e32", n);
      const double inner = p.inner_rel_tol > 0.0 ? p.inner_rel_tol : 1e-4;
      rn = convert_norm(c, b, r32, n);
      bytes += 12.0 * n;
      while (rn > target * bn && used < max_iters) {
        const double tol = std::max(inner, 0.5 * target * bn / rn);
        const int it = pcg2<float>(c, sys32, r32, e32, tol * rn, max_iters - used);
        used += it;
        axpy<float, double>(s, n, 1.0, e32, x);
        sys64.op(0, kOpResid, x, b, nullptr, r);  // r = b - A x
        sys64.screen(x, r, -1);
        const double rn_new = convert_norm(c, r, r32, n);
        bytes += 20.0 * n + 12.0 * n;
        st.refinement_steps++;
        const bool stalled = it == 0 || !(rn_new < rn);
        rn = rn_new;
        if (stalled) break;
      }
      bytes += sys32.bytes;
    } else {
      double* e64 = c->buf<double>("d2_e64", n);
      PR_CUDA(cudaMemcpyAsync(r, b, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
      bytes += 16.0 * n;
      while (rn > target * bn && used < max_iters) {
        const int it = pcg2<double>(c, sys64, r, e64, 0.5 * target * bn, max_iters - used);
        used += it;
        axpy<double, double>(s, n, 1.0, e64, x);
        sys64.op(0, kOpResid, x, b, nullptr, r);
        sys64.screen(x, r, -1);
        const double rn_new = std::sqrt(dot<double>(c, r, r, n));
        bytes += 24.0 * n + 16.0 * n;
        st.refinement_steps++;
        const bool stalled = it == 0 || !(rn_new < rn);
        rn = rn_new;
        if (stalled) break;
      }
    }
  }
  bytes += sys64.bytes;
  st.pcg_iterations = (uint32_t)used;
  st.rel_residual = bn > 0.0 ? rn / bn : 0.0;
  st.converged = st.rel_residual <= target ? 1 : 0;
  st.solve_bytes = bytes;
  double* xm = c->buf<double>("x64", n);
  k_nat_to_morton<double><<<grid_for(n), kThreads, 0, s>>>(x, D, xm);
  PR_CHECK_LAUNCH();
  c->have_coeffs = true;
}

// accessors in Morton order (the order of the degree-1 vectors and of the oracle)
void deg2_rhs_morton(pr_context* c, double* d_out) {
  k_nat_to_morton<double><<<grid_for(c->n), kThreads, 0, c->stream>>>(c->get<double>("d2_b"), c->D, d_out);
  PR_CHECK_LAUNCH();
}
void deg2_normal_field_morton(pr_context* c, double* d_nf3, double* d_w) {
  k_nat3_to_morton_aos<<<grid_for(c->n), kThreads, 0, c->stream>>>(c->get<double>("d2_nf"), c->D, d_nf3);
  PR_CHECK_LAUNCH();
  k_nat_to_morton<double><<<grid_for(c->n), kThreads, 0, c->stream>>>(c->get<double>("d2_w"), c->D, d_w);
  PR_CHECK_LAUNCH();
}
// y = A x with the screening, x and y in Morton order (device)
template <typename T>
void deg2_apply_morton(pr_context* c, const T* d_x, T* d_y) {
  const uint64_t n = c->n;
  const std::string tn = tn2<T>();
  T* xn = c->buf<T>("d2_acc_xn_" + tn, n);
  T* yn = c->buf<T>("d2_acc_yn_" + tn, n);
  k_morton_to_nat<T><<<grid_for(n), kThreads, 0, c->stream>>>(d_x, c->D, xn);
  PR_CHECK_LAUNCH();
  System2<T> sys;
  sys.init(c, c->D, c->pw, false);
  sys.set_screen(sizeof(T) == 8 ? (const T*)c->get<double>("d2_phi64") : (const T*)c->get<float>("d2_phi32"));
  sys.op(0, kOpApply, xn, nullptr, nullptr, yn);
  sys.screen(xn, yn, +1);
  k_nat_to_morton<T><<<grid_for(n), kThreads, 0, c->stream>>>(yn, c->D, d_y);
  PR_CHECK_LAUNCH();
}
template void deg2_apply_morton<double>(pr_context*, const double*, double*);
template void deg2_apply_morton<float>(pr_context*, const float*, float*);

}  // namespace pr

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
// is a sum of tensor products of banded 1-D matrices, applied in a single pass over HBM that
// streams z planes through a CTA and keeps the z filter in registers; the epilogue forms A x,
// f - A x, a Chebyshev step or a fused CG / refinement update.  Levels with res >= 64 stage their
// planes with TMA: k_op3r on the finest level (x filter from the stage, y and z in registers),
// k_op3 on the Galerkin coarse levels (interior and face tiles); smaller levels use k_op2
// (32 x 8 columns, plain loads into shared memory).  The grid transfers and the right-hand side
// stream the same way (k_restrict3, k_prolong3).  The right-hand side is built per 8^3 brick from
// the normal field of the touched nodes only (k_rhs2_bricks).
//
// Solver: conjugate gradients preconditioned by a multigrid V-cycle on K + wg I.  Coarse
// levels are Galerkin products of the 1-D matrices (P^T X P, P the B2 subdivision
// [1/4 3/4 3/4 1/4] per axis, fine functions outside the grid omitted) with the shift wg;
// smoothing is Chebyshev of degree 3 on the Jacobi-scaled operator over [2.1 / 15, 2.1]; the
// 4^3 level is solved with a dense inverse.  FP32 inner solves with FP64 residual refinement,
// or FP64 throughout.  The solved coefficients are permuted to the Morton order of the
// degree-1 path for evaluation and marching cubes.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <cuda.h>

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
constexpr int kZChunk = 64;              // output planes per CTA (k_op2)
constexpr int kZChunk3 = 76;             // output planes per CTA (k_op3): 80 staged planes = 16 x 5
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

// ------------------------------------------------------------------ the TMA-fed operator
// For levels with res >= 64 (k_op2 serves the smaller ones).  A CTA owns 64 x 8 columns, each
// thread an x-adjacent pair of them, and streams up to 64 z planes.  One elected thread keeps five
// planes in flight: per plane a tiled TMA load of the haloed input (box BW x 12 x 1 from a 16-byte
// aligned x; the tensor map's zero fill supplies the halo outside the grid) and, for the epilogue,
// the f / xp planes of the output two planes behind (box 64 x 8 x 1), completing on the stage's
// mbarrier.  The five stages are also the five-plane z window, so the plane loop is unrolled by
// five and every window index is static.
//
// Interior CTAs (all outputs at least `edge` rows from the x and y faces, where the level's 1-D
// matrices equal their interior row) take the coefficients from the kernel parameters; the CTAs
// along the x and y faces run the EDGE instantiation with per-thread rows.  Planes within `edge`
// of the z faces read their z row from the tables in both.
//
// Waits are bounded: a wait that runs out sets *err, the CTA stops after the next barrier and
// thread 0 waits (bounded again) for the loads it still has in flight.
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// false once 2^22 polls have failed (each poll may itself suspend the thread for a while)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (uint32_t k = 0; k < (1u << 22); ++k)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

template <typename T>
struct Geo3 {
  static constexpr int NS = 5;                          // stages = z window
  static constexpr int TXP = 64;                        // output columns in x (32 pairs)
  static constexpr int BW = sizeof(T) == 4 ? 72 : 68;   // staged width from a 16-byte aligned start
  static constexpr int XOFF = sizeof(T) == 4 ? 2 : 0;   // stage column of global x0 - 2
  static constexpr uint32_t XBYTES = BW * SH * sizeof(T);
  static constexpr uint32_t OBYTES = TXP * TY * sizeof(T);
  static constexpr size_t OFF_X = 0;
  static constexpr size_t OFF_F = OFF_X + (size_t)NS * XBYTES;
  static constexpr size_t OFF_P = OFF_F + (size_t)NS * OBYTES;
  static constexpr size_t OFF_UM = OFF_P + (size_t)NS * OBYTES;
  static constexpr size_t OFF_US = OFF_UM + 2 * (size_t)SH * TXP * sizeof(T);
  static constexpr size_t OFF_K = OFF_US + 2 * (size_t)SH * TXP * sizeof(T);  // EDGE, kOpChebF: D^-1 scale
  static constexpr size_t OFF_DX = OFF_K + (size_t)SH * BW * sizeof(T);      // EDGE: diagonal entries
  static constexpr size_t OFF_BAR = OFF_DX + (size_t)(BW + SH) * 2 * sizeof(T);
  static constexpr size_t BYTES = OFF_BAR + NS * 8 + 16;
};

template <typename T>
struct Vec2;
template <>
struct Vec2<float> {
  typedef float2 type;
};
template <>
struct Vec2<double> {
  typedef double2 type;
};

// kOpChebF:  out = (1 + ca) x1 + cb D^-1 (f - A x1), x1 = c0 D^-1 f (the first step from zero,
//            then the second); the staged input is f.
// kOpChebPF: out = x + ca (x - xp) + cb D^-1 (f - A x) with xp = c0 D^-1 f (the third step after
//            kOpChebF: its previous iterate is recomputed from f).
// kOpApplyD: the preconditioned CG direction update fused into the operator pass (second staged
//            plane z): d = z + s1 dold (staged: dold, z), out = A d, out2 = d, xacc += s2 dold,
//            dot d . out
// kOpRefine: the FP64 refinement step on a level without boundary rows (k_op3r only): staged x
//            (skipped when xzero), the FP32 correction e and b; xn = x + e (written to out2),
//            out = b - A xn, r32 = (float) out, dot out . out
enum { kOpChebF = 3, kOpChebPF = 4, kOpApplyD = 5, kOpRefine = 6 };

template <typename T>
struct Op3Args {
  LevelView<T> lv;
  T im[5], is[5];  // interior rows of the 1-D matrices
  T invd;          // 1 / interior diagonal
  int edge;        // rows [edge, res - edge) equal the interior row
  T ca, cb, c0;
  int use_p;       // kOpCheb: xp given
  int nbx, nby;    // tiles per axis (x: 64 columns, y: 8 rows)
  int all;         // EDGE: the grid enumerates every tile, not only the face tiles
  int ox, oy;      // interior: tile of block (i, j) is (i + ox, j + oy)
  int oz;          // interior: z run of block k is k + oz
  int* err;
  double* dot;     // optional per-CTA partials: kOpApply x . out, kOpCheb f . out, kOpApplyD d . out
  int dot_base;    // index of this launch's first partial
  T s1, s2;        // kOpApplyD: beta, alpha of the previous step
  T* out2;         // kOpApplyD: d
  T* xacc;         // kOpApplyD: the CG iterate
  int xmode;       // kOpApplyD: 0 leave xacc alone, 1 xacc = s2 dold (not read), 2 xacc += s2 dold
  float* r32;      // kOpRefine: the residual rounded to FP32
  int xzero;       // kOpRefine: x = 0 (not staged)
};

// the (x, y) tile of an EDGE CTA: the first and the last tile row, then the first and the last
// tile of every row in between
__device__ __forceinline__ void edge_tile(int j, int nbx, int nby, int all, int& bx, int& by) {
  if (all || nbx <= 2 || nby <= 2) {
    bx = j % nbx;
    by = j / nbx;
  } else if (j < 2 * nbx) {
    bx = j % nbx;
    by = j < nbx ? 0 : nby - 1;
  } else {
    const int k = j - 2 * nbx;
    bx = (k & 1) ? nbx - 1 : 0;
    by = 1 + (k >> 1);
  }
}

// 5-tap filters of the face tiles (general rows).
template <typename T>
__device__ __forceinline__ T filt(const T* v, const T* c) {
  return c[0] * v[0] + c[1] * v[1] + c[2] * v[2] + c[3] * v[3] + c[4] * v[4];
}

// Pair arithmetic for the two x-adjacent outputs of a thread: FP32 pairs use the packed two-wide
// instructions (one instruction for both lanes), FP64 pairs two scalar operations.
__device__ __forceinline__ float2 p_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 p_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 p_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ double2 p_add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 p_mul(double2 a, double2 b) { return make_double2(a.x * b.x, a.y * b.y); }
__device__ __forceinline__ double2 p_fma(double2 a, double2 b, double2 c) {
  return make_double2(__fma_rn(a.x, b.x, c.x), __fma_rn(a.y, b.y, c.y));
}
template <typename V2, typename T>
__device__ __forceinline__ V2 p_bc(T x) {
  return V2{x, x};
}
// interior rows are symmetric (c[0] = c[4], c[1] = c[3]): om, os = the M and S filters of the taps
// t0..t4 (pairs), sharing the pair sums
template <typename V2>
__device__ __forceinline__ void sym2(V2 t0, V2 t1, V2 t2, V2 t3, V2 t4, const V2* m, const V2* s, V2& om, V2& os) {
  const V2 q0 = p_add(t0, t4), q1 = p_add(t1, t3);
  om = p_fma(m[2], t2, p_fma(m[1], q1, p_mul(m[0], q0)));
  os = p_fma(s[2], t2, p_fma(s[1], q1, p_mul(s[0], q0)));
}

template <typename T, int MODE, bool EDGE>
__global__ void __launch_bounds__(kThreads) k_op3(const __grid_constant__ CUtensorMap mx,
                                                  const __grid_constant__ CUtensorMap mf,
                                                  const __grid_constant__ CUtensorMap mp, T* out,
                                                  const __grid_constant__ Op3Args<T> A) {
  typedef Geo3<T> G;
  typedef typename Vec2<T>::type V2;
  constexpr int NS = G::NS, BW = G::BW, XOFF = G::XOFF, TXP = G::TXP;
  extern __shared__ __align__(128) unsigned char smem[];
  T(*s_x)[SH][BW] = reinterpret_cast<T(*)[SH][BW]>(smem + G::OFF_X);
  T(*s_f)[TY][TXP] = reinterpret_cast<T(*)[TY][TXP]>(smem + G::OFF_F);
  T(*s_p)[TY][TXP] = reinterpret_cast<T(*)[TY][TXP]>(smem + G::OFF_P);
  T(*s_um)[SH][TXP] = reinterpret_cast<T(*)[SH][TXP]>(smem + G::OFF_UM);
  T(*s_us)[SH][TXP] = reinterpret_cast<T(*)[SH][TXP]>(smem + G::OFF_US);
  T(*s_k)[BW] = reinterpret_cast<T(*)[BW]>(smem + G::OFF_K);
  T* s_dx = reinterpret_cast<T*>(smem + G::OFF_DX);  // [BW][2] then [SH][2]: (m, s) diagonal entries
  T* s_dy = s_dx + 2 * BW;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + G::OFF_BAR);
  int* s_abort = reinterpret_cast<int*>(smem + G::OFF_BAR + NS * 8);
  const LevelView<T>& lv = A.lv;
  const int res = 1 << lv.L;
  const int64_t plane = (int64_t)res * res;
  const int t = threadIdx.x, p = t & 31, ty = t >> 5;
  int bx, by;
  if (EDGE) edge_tile(blockIdx.x, A.nbx, A.nby, A.all, bx, by);
  else {
    bx = blockIdx.x + A.ox;
    by = blockIdx.y + A.oy;
  }
  const int x0 = bx * TXP, y0 = by * TY;
  const int z0 = (blockIdx.z + A.oz) * kZChunk3, z1 = min(z0 + kZChunk3, res);
  const int gx = x0 + 2 * p, gy = y0 + ty;  // res >= 64: every column is inside the grid
  const int nplanes = z1 - z0 + 4;
  const int ngroups = (nplanes + NS - 1) / NS;  // planes past z1 + 1 read zeros and emit nothing
  constexpr bool use_f = MODE == kOpResid || MODE == kOpCheb || MODE == kOpChebPF;
  constexpr bool two = MODE == kOpApplyD;  // second haloed plane, staged in the f/p space
  const bool use_p = MODE == kOpCheb && A.use_p;
  const uint32_t bytes = G::XBYTES + (use_f ? G::OBYTES : 0u) + (use_p ? G::OBYTES : 0u) + (two ? G::XBYTES : 0u);
  T(*s_z)[SH][BW] = reinterpret_cast<T(*)[SH][BW]>(smem + G::OFF_F);
  if (t == 0) {
    for (int s = 0; s < NS; ++s) mbar_init(&bar[s], 1);
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (EDGE && MODE == kOpChebF) {
    for (int i = t; i < BW; i += kThreads) {
      const int X = x0 - 2 - XOFF + i;
      const bool in = X >= 0 && X < res;
      s_dx[2 * i] = in ? lv.tM[5 * X + 2] : T(0);
      s_dx[2 * i + 1] = in ? lv.tS[5 * X + 2] : T(0);
    }
    for (int i = t; i < SH; i += kThreads) {
      const int Y = y0 - 2 + i;
      const bool in = Y >= 0 && Y < res;
      s_dy[2 * i] = in ? lv.tM[5 * Y + 2] : T(0);
      s_dy[2 * i + 1] = in ? lv.tS[5 * Y + 2] : T(0);
    }
  }
  __syncthreads();
  auto issue = [&](int it) {
    const int s = it % NS, zin = z0 - 2 + it;
    mbar_expect_tx(&bar[s], bytes);
    tma_load_3d(&s_x[s][0][0], &mx, x0 - 2 - XOFF, y0 - 2, zin, &bar[s]);
    if (use_f) tma_load_3d(&s_f[s][0][0], &mf, x0, y0, zin - 2, &bar[s]);
    if (use_p) tma_load_3d(&s_p[s][0][0], &mp, x0, y0, zin - 2, &bar[s]);
    if (two) tma_load_3d(&s_z[s][0][0], &mf, x0 - 2 - XOFF, y0 - 2, zin, &bar[s]);
  };
  const int nissue = ngroups * NS;
  if (t == 0)
    for (int it = 0; it < NS; ++it) issue(it);
  // EDGE: x rows of the pair and the y row of this thread
  T cmx[2][5], csx[2][5], cmy[5], csy[5];
  if (EDGE) {
#pragma unroll
    for (int d = 0; d < 5; ++d) {
      cmx[0][d] = lv.tM[5 * gx + d];
      csx[0][d] = lv.tS[5 * gx + d];
      cmx[1][d] = lv.tM[5 * gx + 5 + d];
      csx[1][d] = lv.tS[5 * gx + 5 + d];
      cmy[d] = lv.tM[5 * gy + d];
      csy[d] = lv.tS[5 * gy + d];
    }
  }
  // diagonal dg(z) = H (dA mz + dC sz) + wg of the two outputs, and its inverse on interior planes
  T dA[2], dC[2], invI[2];
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    if (EDGE) {
      dA[j] = csx[j][2] * cmy[2] + cmx[j][2] * csy[2];
      dC[j] = cmx[j][2] * cmy[2];
      invI[j] = T(1) / (lv.H * (dA[j] * A.im[2] + dC[j] * A.is[2]) + lv.wg);
    } else {
      dA[j] = A.is[2] * A.im[2] + A.im[2] * A.is[2];
      dC[j] = A.im[2] * A.im[2];
      invI[j] = A.invd;
    }
  }
  // interior: the symmetric rows as pairs and the epilogue of the interior planes as at most two
  // pair operations on (acc, centre, f, xp), its coefficients folded here:
  //   kOpApply   H acc + wg c                           kOpResid  f - H acc - wg c
  //   kOpCheb    (1 + ca) c - ca xp + cb D^-1 r,  r = f - H acc - wg c
  //   kOpChebPF  (1 + ca) c - ca c0 D^-1 f + cb D^-1 r
  //   kOpChebF   x1 = c0 D^-1 c (c = f): (1 + ca) x1 + cb D^-1 (c - H acc - wg x1)
  V2 pm[3], ps[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    pm[d] = p_bc<V2>(A.im[d]);
    ps[d] = p_bc<V2>(A.is[d]);
  }
  const T cbinv = A.cb * A.invd, c0inv = A.c0 * A.invd;
  T e_acc, e_c, e_f, e_p;  // interior epilogue: res = e_acc acc + e_c c + e_f f + e_p xp (+ cb D^-1 f below)
  if (MODE == kOpApply || MODE == kOpApplyD) { e_acc = lv.H; e_c = lv.wg; e_f = 0; e_p = 0; }
  else if (MODE == kOpResid) { e_acc = -lv.H; e_c = -lv.wg; e_f = 1; e_p = 0; }
  else if (MODE == kOpCheb) { e_acc = -cbinv * lv.H; e_c = (T(1) + A.ca) - cbinv * lv.wg; e_f = cbinv; e_p = -A.ca; }
  else if (MODE == kOpChebPF) {
    e_acc = -cbinv * lv.H; e_c = (T(1) + A.ca) - cbinv * lv.wg; e_f = cbinv - A.ca * c0inv; e_p = 0;
  } else {  // kOpChebF
    e_acc = -cbinv * lv.H; e_c = (T(1) + A.ca) * c0inv + cbinv * (T(1) - lv.wg * c0inv); e_f = 0; e_p = 0;
  }
  const V2 pe_acc = p_bc<V2>(e_acc), pe_c = p_bc<V2>(e_c), pe_f = p_bc<V2>(e_f), pe_p = p_bc<V2>(e_p);
  V2 wa[NS], wb[NS], wc[NS], wo[NS];  // wo: kOpApplyD, the centres of dold
#pragma unroll
  for (int k = 0; k < NS; ++k) wa[k] = wb[k] = wc[k] = wo[k] = V2{T(0), T(0)};
  const V2 pbeta = p_bc<V2>(A.s1);
  T* op = out + (int64_t)gx + (int64_t)res * gy + plane * (z0 - 4);  // output row of plane zo = z0 - 4 + it
  const bool want_dot = A.dot != nullptr;
  double dacc = 0.0;  // A.dot: this thread's share of the product
  int kstate = -1;  // EDGE kOpChebF: s_k holds the scales of: -1 nothing, 0 interior planes, 1 plane kzin
  int kzin = 0;
  int it = 0;
  bool stop = false;
  for (int g = 0; g < ngroups; ++g) {
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      it = g * NS + k;
      // kOpApplyD: the iterate of this step's output plane, loaded before the wait
      V2 xold = V2{T(0), T(0)};
      if (two && A.xmode == 2 && (unsigned)(it - 4) < (unsigned)(z1 - z0))
        xold = *reinterpret_cast<const V2*>(A.xacc + (op - out));
      if (!mbar_wait(&bar[k], (uint32_t)g & 1u)) {
        atomicExch(A.err, 1);
        *s_abort = 1;
      }
      const int b = (g + k) & 1;  // = it & 1 (NS is odd)
      const int zin = z0 - 2 + it;
      const bool zin_int = zin >= A.edge && zin < res - A.edge;
      // kOpChebF: the staged f becomes x1 = c0 D^-1 f
      T kz = T(0);
      if (MODE == kOpChebF) {
        if (EDGE) {
          if (zin_int ? kstate != 0 : (kstate != 1 || kzin != zin)) {
            const bool zok = zin >= 0 && zin < res;
            const int zr = zok ? zin : 0;
            const T mz = zok ? lv.tM[5 * zr + 2] : T(0), sz = zok ? lv.tS[5 * zr + 2] : T(0);
            for (int i = t; i < SH * BW; i += kThreads) {
              const int r = i / BW, c = i % BW;
              const T dxm = s_dx[2 * c], dxs = s_dx[2 * c + 1], dym = s_dy[2 * r], dys = s_dy[2 * r + 1];
              const T dg = lv.H * (dxs * dym * mz + dxm * dys * mz + dxm * dym * sz) + lv.wg;
              s_k[r][c] = (zok && dxm != T(0) && dym != T(0)) ? A.c0 / dg : T(0);
            }
            kstate = zin_int ? 0 : 1;
            kzin = zin;
            __syncthreads();
          }
        } else if (zin_int) {
          kz = c0inv;
        } else if (zin < 0 || zin >= res) {
          kz = T(0);  // a zero-filled plane
        } else {
          const T mz = lv.tM[5 * zin + 2], sz = lv.tS[5 * zin + 2];
          kz = A.c0 / (lv.H * (dA[0] * mz + dC[0] * sz) + lv.wg);
        }
      }
      // x filter: rows ty and ty + 8 of the 12 staged rows, two outputs per thread
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int r = ty + 8 * q;
        if (r < SH) {
          const T* row = &s_x[k][r][2 * p + XOFF];
          V2 v0 = *reinterpret_cast<const V2*>(row), v1 = *reinterpret_cast<const V2*>(row + 2),
             v2 = *reinterpret_cast<const V2*>(row + 4);
          if (two) {  // d = z + beta dold
            const T* zr = &s_z[k][r][2 * p + XOFF];
            v0 = p_fma(pbeta, v0, *reinterpret_cast<const V2*>(zr));
            v1 = p_fma(pbeta, v1, *reinterpret_cast<const V2*>(zr + 2));
            v2 = p_fma(pbeta, v2, *reinterpret_cast<const V2*>(zr + 4));
          }
          V2 um, us;
          if (EDGE) {
            T v[6] = {v0.x, v0.y, v1.x, v1.y, v2.x, v2.y};
            if (MODE == kOpChebF) {
              const T* kr = &s_k[r][2 * p + XOFF];
#pragma unroll
              for (int e = 0; e < 6; ++e) v[e] *= kr[e];
            }
            um = V2{filt(v, cmx[0]), filt(v + 1, cmx[1])};
            us = V2{filt(v, csx[0]), filt(v + 1, csx[1])};
          } else {
            // output 0 taps v0..v4, output 1 taps v1..v5: pairs (v0,v1) (v1,v2) (v2,v3) (v3,v4) (v4,v5)
            const V2 v12 = V2{v0.y, v1.x}, v34 = V2{v1.y, v2.x};
            sym2(v0, v12, v1, v34, v2, pm, ps, um, us);
            if (MODE == kOpChebF) {
              const V2 kp = p_bc<V2>(kz);
              um = p_mul(kp, um);
              us = p_mul(kp, us);
            }
          }
          *reinterpret_cast<V2*>(&s_um[b][r][2 * p]) = um;
          *reinterpret_cast<V2*>(&s_us[b][r][2 * p]) = us;
        }
      }
      // centre values: x (f for kOpChebF; d = z + beta dold for kOpApplyD)
      V2 xc = *reinterpret_cast<const V2*>(&s_x[k][ty + 2][2 * p + 2 + XOFF]);
      if (two) {
        wo[k] = xc;
        xc = p_fma(pbeta, xc, *reinterpret_cast<const V2*>(&s_z[k][ty + 2][2 * p + 2 + XOFF]));
      }
      V2 fo = V2{T(0), T(0)}, po = V2{T(0), T(0)};
      if (use_f) fo = *reinterpret_cast<const V2*>(&s_f[k][ty][2 * p]);
      if (use_p) po = *reinterpret_cast<const V2*>(&s_p[k][ty][2 * p]);
      __syncthreads();  // stage k is read; s_um/s_us[b] are written
      if (*s_abort) {
        stop = true;
        break;
      }
      if (t == 0 && it + NS < nissue) issue(it + NS);
      // y filter into the window slot k
      {
        V2 a[5], c[5];
#pragma unroll
        for (int d = 0; d < 5; ++d) {
          a[d] = *reinterpret_cast<const V2*>(&s_um[b][ty + d][2 * p]);
          c[d] = *reinterpret_cast<const V2*>(&s_us[b][ty + d][2 * p]);
        }
        if (EDGE) {
          T a0[5], a1[5], c0[5], c1[5];
#pragma unroll
          for (int d = 0; d < 5; ++d) {
            a0[d] = a[d].x;
            a1[d] = a[d].y;
            c0[d] = c[d].x;
            c1[d] = c[d].y;
          }
          wa[k] = V2{filt(c0, cmy) + filt(a0, csy), filt(c1, cmy) + filt(a1, csy)};
          wb[k] = V2{filt(a0, cmy), filt(a1, cmy)};
        } else {
          V2 vmm, vms, vsm, unused;
          sym2(a[0], a[1], a[2], a[3], a[4], pm, ps, vmm, vms);
          sym2(c[0], c[1], c[2], c[3], c[4], pm, ps, vsm, unused);
          wa[k] = p_add(vsm, vms);
          wb[k] = vmm;
        }
      }
      wc[k] = xc;
      const int zo = zin - 2;
      if ((unsigned)(zo - z0) < (unsigned)(z1 - z0)) {
        const bool zint = zo >= A.edge && zo < res - A.edge;
        V2 res2;
        if (!EDGE && zint) {
          // the symmetric z filter and the folded epilogue, both lanes at once
          V2 acc, u;
          sym2(wa[(k + 1) % NS], wa[(k + 2) % NS], wa[(k + 3) % NS], wa[(k + 4) % NS], wa[(k + 5) % NS], pm, ps, acc, u);
          V2 um2, us2;
          sym2(wb[(k + 1) % NS], wb[(k + 2) % NS], wb[(k + 3) % NS], wb[(k + 4) % NS], wb[(k + 5) % NS], pm, ps, um2, us2);
          acc = p_add(acc, us2);
          const V2 cc = wc[(k + 3) % NS];
          res2 = p_fma(pe_c, cc, p_mul(pe_acc, acc));
          if (MODE == kOpResid || MODE == kOpCheb || MODE == kOpChebPF) res2 = p_fma(pe_f, fo, res2);
          if (MODE == kOpCheb) res2 = p_fma(pe_p, po, res2);
        } else {
          T acc[2], inv[2];
          if (zint) {
#pragma unroll
            for (int j = 0; j < 2; ++j) {
              T wA[NS], wB[NS];
#pragma unroll
              for (int q = 0; q < NS; ++q) {
                wA[q] = j == 0 ? wa[q].x : wa[q].y;
                wB[q] = j == 0 ? wb[q].x : wb[q].y;
              }
              acc[j] = A.im[0] * (wA[(k + 1) % NS] + wA[(k + 5) % NS]) + A.im[1] * (wA[(k + 2) % NS] + wA[(k + 4) % NS]) +
                       A.im[2] * wA[(k + 3) % NS] + A.is[0] * (wB[(k + 1) % NS] + wB[(k + 5) % NS]) +
                       A.is[1] * (wB[(k + 2) % NS] + wB[(k + 4) % NS]) + A.is[2] * wB[(k + 3) % NS];
              inv[j] = invI[j];
            }
          } else {
            T cz_m[5], cz_s[5];
#pragma unroll
            for (int d = 0; d < 5; ++d) {
              cz_m[d] = lv.tM[5 * zo + d];
              cz_s[d] = lv.tS[5 * zo + d];
            }
#pragma unroll
            for (int j = 0; j < 2; ++j) {
              T sacc = 0;
#pragma unroll
              for (int d = 0; d < 5; ++d) {
                const T wA = j == 0 ? wa[(k + 1 + d) % NS].x : wa[(k + 1 + d) % NS].y;
                const T wB = j == 0 ? wb[(k + 1 + d) % NS].x : wb[(k + 1 + d) % NS].y;
                sacc += cz_m[d] * wA + cz_s[d] * wB;
              }
              acc[j] = sacc;
              inv[j] = T(1) / (lv.H * (dA[j] * cz_m[2] + dC[j] * cz_s[2]) + lv.wg);
            }
          }
          T rr2[2];
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            const T fj = j == 0 ? fo.x : fo.y;
            const T pj = j == 0 ? po.x : po.y;
            const T cj = j == 0 ? wc[(k + 3) % NS].x : wc[(k + 3) % NS].y;  // the centre (f for kOpChebF)
            if (MODE == kOpChebF) {
              const T x1 = A.c0 * inv[j] * cj;
              const T ax = lv.H * acc[j] + lv.wg * x1;
              rr2[j] = (T(1) + A.ca) * x1 + A.cb * (cj - ax) * inv[j];
            } else {
              const T ax = lv.H * acc[j] + lv.wg * cj;
              if (MODE == kOpApply || MODE == kOpApplyD) rr2[j] = ax;
              else if (MODE == kOpResid) rr2[j] = fj - ax;
              else if (MODE == kOpCheb) rr2[j] = cj + A.ca * (cj - pj) + A.cb * (fj - ax) * inv[j];
              else rr2[j] = cj + A.ca * (cj - A.c0 * inv[j] * fj) + A.cb * (fj - ax) * inv[j];  // kOpChebPF
            }
          }
          res2 = V2{rr2[0], rr2[1]};
        }
        *reinterpret_cast<V2*>(op) = res2;
        if (two) {
          *reinterpret_cast<V2*>(A.out2 + (op - out)) = wc[(k + 3) % NS];
          if (A.xmode) *reinterpret_cast<V2*>(A.xacc + (op - out)) = p_fma(p_bc<V2>(A.s2), wo[(k + 3) % NS], xold);
        }
        if ((MODE == kOpApply || MODE == kOpApplyD) && want_dot) {
          const V2 cc = wc[(k + 3) % NS];
          dacc += (double)cc.x * (double)res2.x + (double)cc.y * (double)res2.y;
        }
        if (MODE == kOpCheb && want_dot) dacc += (double)fo.x * (double)res2.x + (double)fo.y * (double)res2.y;
      }
      op += plane;
    }
    if (stop) break;
  }
  if (stop && t == 0) {
    // stopped early: let the loads still in flight land before the CTA's shared memory goes
    for (int q = it; q < min(it + NS, nissue); ++q) mbar_wait(&bar[q % NS], (uint32_t)(q / NS) & 1u);
  }
  if ((MODE == kOpApply || MODE == kOpCheb || MODE == kOpApplyD) && A.dot != nullptr) {
    typedef cub::BlockReduce<double, kThreads> BR;
    __shared__ typename BR::TempStorage tmp;
    const double tot = BR(tmp).Sum(dacc);
    if (t == 0)
      A.dot[A.dot_base + (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = tot;
  }
}

// A level whose every row is the interior row (edge 0: the finest level) with the y and z filters
// in registers: 4 warps on the same 64 x 8 tile and stages as k_op3, each thread two output rows.
// A thread runs the x filter of its six staged rows straight from the TMA stage (no shared
// intermediate, one barrier per plane), the y filter on registers, and scatters each input plane
// into the five output planes it touches (zin - 2 .. zin + 2, register accumulators rotating with
// the stage index). Planes outside the grid are zero-filled and never emitted, so every tap uses
// the interior coefficients and the body has no boundary path (its size bounds the instruction
// cache). Same modes, epilogues and per-CTA dot partials as k_op3<T, MODE, false> at edge 0; for
// kOpChebF the scale x1 = c0 D^-1 f is one constant there and folds into the epilogue.
constexpr int kThreadsR = 128;
template <typename T>
struct Geo3R {
  typedef Geo3<T> G;
  static constexpr size_t OFF_BAR = G::OFF_P + (size_t)G::NS * G::OBYTES;
  static constexpr size_t BYTES = OFF_BAR + G::NS * 8 + 16;
};

template <typename T, int MODE>
__global__ void __launch_bounds__(kThreadsR) k_op3r(const __grid_constant__ CUtensorMap mx,
                                                    const __grid_constant__ CUtensorMap mf,
                                                    const __grid_constant__ CUtensorMap mp, T* out,
                                                    const __grid_constant__ Op3Args<T> A) {
  typedef Geo3<T> G;
  typedef typename Vec2<T>::type V2;
  constexpr int NS = G::NS, BW = G::BW, XOFF = G::XOFF, TXP = G::TXP, RY = 2;
  extern __shared__ __align__(128) unsigned char smem[];
  T(*s_x)[SH][BW] = reinterpret_cast<T(*)[SH][BW]>(smem + G::OFF_X);
  T(*s_f)[TY][TXP] = reinterpret_cast<T(*)[TY][TXP]>(smem + G::OFF_F);
  T(*s_p)[TY][TXP] = reinterpret_cast<T(*)[TY][TXP]>(smem + G::OFF_P);
  T(*s_z)[SH][BW] = reinterpret_cast<T(*)[SH][BW]>(smem + G::OFF_F);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + Geo3R<T>::OFF_BAR);
  int* s_abort = reinterpret_cast<int*>(smem + Geo3R<T>::OFF_BAR + NS * 8);
  const LevelView<T>& lv = A.lv;
  const int res = 1 << lv.L;
  const int64_t plane = (int64_t)res * res;
  const int t = threadIdx.x, p = t & 31, ry = RY * (t >> 5);  // tile rows ry, ry + 1; staged ry .. ry + 5
  const int x0 = (blockIdx.x + A.ox) * TXP, y0 = (blockIdx.y + A.oy) * TY;
  const int z0 = (blockIdx.z + A.oz) * kZChunk3, z1 = min(z0 + kZChunk3, res);
  const int gx = x0 + 2 * p;
  const int nplanes = z1 - z0 + 4;
  const int ngroups = (nplanes + NS - 1) / NS;
  constexpr bool refine = MODE == kOpRefine;
  constexpr bool use_f = MODE == kOpResid || MODE == kOpCheb || MODE == kOpChebPF || refine;
  constexpr bool two = MODE == kOpApplyD;
  const bool use_p = MODE == kOpCheb && A.use_p;
  const bool use_x = !(refine && A.xzero);
  // kOpRefine: e (FP32) staged 72 wide from x0 - 4 (16-byte aligned) in the xp space
  constexpr int EW = 72;
  constexpr uint32_t EBYTES = EW * SH * 4;
  static_assert(!refine || (size_t)NS * EBYTES <= (size_t)NS * G::OBYTES, "e stages fit the xp space");
  float(*s_e)[SH][EW] = reinterpret_cast<float(*)[SH][EW]>(smem + G::OFF_P);
  const uint32_t bytes = (use_x ? G::XBYTES : 0u) + (use_f ? G::OBYTES : 0u) + (use_p ? G::OBYTES : 0u) +
                         (two ? G::XBYTES : 0u) + (refine ? EBYTES : 0u);
  if (t == 0) {
    for (int s = 0; s < NS; ++s) mbar_init(&bar[s], 1);
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto issue = [&](int it) {
    const int s = it % NS, zin = z0 - 2 + it;
    mbar_expect_tx(&bar[s], bytes);
    if (use_x) tma_load_3d(&s_x[s][0][0], &mx, x0 - 2 - XOFF, y0 - 2, zin, &bar[s]);
    if (use_f) tma_load_3d(&s_f[s][0][0], &mf, x0, y0, zin - 2, &bar[s]);
    if (use_p) tma_load_3d(&s_p[s][0][0], &mp, x0, y0, zin - 2, &bar[s]);
    if (two) tma_load_3d(&s_z[s][0][0], &mf, x0 - 2 - XOFF, y0 - 2, zin, &bar[s]);
    if (refine) tma_load_3d(&s_e[s][0][0], &mp, x0 - 4, y0 - 2, zin, &bar[s]);
  };
  const int nissue = ngroups * NS;
  if (t == 0)
    for (int it = 0; it < NS; ++it) issue(it);
  V2 pm[3], ps[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    pm[d] = p_bc<V2>(A.im[d]);
    ps[d] = p_bc<V2>(A.is[d]);
  }
  const T cbinv = A.cb * A.invd, c0inv = A.c0 * A.invd;
  T e_acc, e_c, e_f, e_p;  // interior epilogue, as in k_op3
  if (MODE == kOpApply || MODE == kOpApplyD) { e_acc = lv.H; e_c = lv.wg; e_f = 0; e_p = 0; }
  else if (MODE == kOpResid || refine) { e_acc = -lv.H; e_c = -lv.wg; e_f = 1; e_p = 0; }
  else if (MODE == kOpCheb) { e_acc = -cbinv * lv.H; e_c = (T(1) + A.ca) - cbinv * lv.wg; e_f = cbinv; e_p = -A.ca; }
  else if (MODE == kOpChebPF) {
    e_acc = -cbinv * lv.H; e_c = (T(1) + A.ca) - cbinv * lv.wg; e_f = cbinv - A.ca * c0inv; e_p = 0;
  } else {  // kOpChebF: acc filters f, x1 = c0inv f
    e_acc = -cbinv * lv.H * c0inv; e_c = (T(1) + A.ca) * c0inv + cbinv * (T(1) - lv.wg * c0inv); e_f = 0; e_p = 0;
  }
  const V2 pe_acc = p_bc<V2>(e_acc), pe_c = p_bc<V2>(e_c), pe_f = p_bc<V2>(e_f), pe_p = p_bc<V2>(e_p);
  // acc[j][s]: the output plane of slot s (zo = z0 - 4 + it for it = s mod NS) of row j, partial;
  // wc: centres of the staged planes (x; f for kOpChebF, d for kOpApplyD) by stage
  V2 acc[RY][NS], wc[RY][NS];
#pragma unroll
  for (int j = 0; j < RY; ++j)
#pragma unroll
    for (int k = 0; k < NS; ++k) acc[j][k] = wc[j][k] = V2{T(0), T(0)};
  const V2 pbeta = p_bc<V2>(A.s1);
  T* op = out + (int64_t)gx + (int64_t)res * (y0 + ry) + plane * (z0 - 4);  // row ry of plane z0 - 4 + it
  const bool want_dot = A.dot != nullptr;
  double dacc = 0.0;
  int it = 0;
  bool stop = false;
  // kOpApplyD with xmode 2: the iterate's rows of the staged plane zin = z0 - 2 + it, loaded one
  // plane ahead (issued while the previous plane is filtered) so the load latency stays hidden
  // (the first staged plane that is one of this CTA's comes at it = 2, so nothing is loaded before
  // the loop)
  const bool xread = two && A.xmode == 2;
  V2 xnext[RY];
#pragma unroll
  for (int j = 0; j < RY; ++j) xnext[j] = V2{T(0), T(0)};
  for (int g = 0; g < ngroups; ++g) {
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      it = g * NS + k;
      const bool emit = (unsigned)(it - 4) < (unsigned)(z1 - z0);
      // kOpApplyD: xacc += s2 dold on the staged plane zin = zo + 2 when it is one of this CTA's
      // planes (the iterate of those rows, loaded one plane ahead)
      const bool own = (unsigned)(it - 2) < (unsigned)(z1 - z0);  // staged plane zin is one of this CTA's
      const bool upd = two && A.xmode && own;
      V2 xold[RY];
#pragma unroll
      for (int j = 0; j < RY; ++j) {
        xold[j] = xnext[j];
        xnext[j] = V2{T(0), T(0)};
        if (xread && (unsigned)(it + 1 - 2) < (unsigned)(z1 - z0))
          xnext[j] = *reinterpret_cast<const V2*>(A.xacc + (op - out) + 3 * plane + (int64_t)j * res);
      }
      if (!mbar_wait(&bar[k], (uint32_t)g & 1u)) {
        atomicExch(A.err, 1);
        *s_abort = 1;
      }
      // x filter of the staged rows ry .. ry + 5
      V2 um[RY + 4], us[RY + 4];
#pragma unroll
      for (int r = 0; r < RY + 4; ++r) {
        const T* row = &s_x[k][ry + r][2 * p + XOFF];
        V2 v0 = V2{T(0), T(0)}, v1 = v0, v2 = v0;
        if (use_x) {
          v0 = *reinterpret_cast<const V2*>(row);
          v1 = *reinterpret_cast<const V2*>(row + 2);
          v2 = *reinterpret_cast<const V2*>(row + 4);
        }
        if (refine) {  // xn = x + e (e column c + 2 is x column c)
          const float* er = &s_e[k][ry + r][2 * p + XOFF + 2];
          const float2 e0 = *reinterpret_cast<const float2*>(er), e1 = *reinterpret_cast<const float2*>(er + 2),
                       e2 = *reinterpret_cast<const float2*>(er + 4);
          v0 = p_add(v0, V2{(T)e0.x, (T)e0.y});
          v1 = p_add(v1, V2{(T)e1.x, (T)e1.y});
          v2 = p_add(v2, V2{(T)e2.x, (T)e2.y});
          if (own && (r == 2 || r == 3))
            *reinterpret_cast<V2*>(A.out2 + (op - out) + 2 * plane + (int64_t)(r - 2) * res) = v1;
        }
        if (upd && (r == 2 || r == 3))  // centre columns 2p, 2p + 1 of dold
          *reinterpret_cast<V2*>(A.xacc + (op - out) + 2 * plane + (int64_t)(r - 2) * res) =
              p_fma(p_bc<V2>(A.s2), v1, xold[r - 2]);
        if (two) {
          const T* zr = &s_z[k][ry + r][2 * p + XOFF];
          v0 = p_fma(pbeta, v0, *reinterpret_cast<const V2*>(zr));
          v1 = p_fma(pbeta, v1, *reinterpret_cast<const V2*>(zr + 2));
          v2 = p_fma(pbeta, v2, *reinterpret_cast<const V2*>(zr + 4));
        }
        if (r == 2 || r == 3) wc[r - 2][k] = v1;  // centre: x (f for kOpChebF; d for kOpApplyD)
        const V2 v12 = V2{v0.y, v1.x}, v34 = V2{v1.y, v2.x};
        sym2(v0, v12, v1, v34, v2, pm, ps, um[r], us[r]);
      }
      V2 fo[RY], po[RY];
#pragma unroll
      for (int j = 0; j < RY; ++j) {
        fo[j] = po[j] = V2{T(0), T(0)};
        if (use_f) fo[j] = *reinterpret_cast<const V2*>(&s_f[k][ry + j][2 * p]);
        if (use_p) po[j] = *reinterpret_cast<const V2*>(&s_p[k][ry + j][2 * p]);
      }
      __syncthreads();  // stage k is read
      if (*s_abort) {
        stop = true;
        break;
      }
      if (t == 0 && it + NS < nissue) issue(it + NS);
#pragma unroll
      for (int j = 0; j < RY; ++j) {
        // y filter: wa = M_y us + S_y um, wb = M_y um
        V2 vmm, vms, vsm, unused;
        sym2(um[j], um[j + 1], um[j + 2], um[j + 3], um[j + 4], pm, ps, vmm, vms);
        sym2(us[j], us[j + 1], us[j + 2], us[j + 3], us[j + 4], pm, ps, vsm, unused);
        const V2 wa = p_add(vsm, vms), wb = vmm;
        // z scatter: plane zin is tap 4 - e (= tap e, symmetric rows) of output plane zin - 2 + e,
        // slot (k + e) mod NS
#pragma unroll
        for (int e = 0; e < 5; ++e) {
          const V2 cm = pm[e < 3 ? e : 4 - e], cs = ps[e < 3 ? e : 4 - e];
          V2& a = acc[j][(k + e) % NS];
          a = e == 4 ? p_fma(cs, wb, p_mul(cm, wa)) : p_fma(cs, wb, p_fma(cm, wa, a));
        }
      }
      if (emit) {
#pragma unroll
        for (int j = 0; j < RY; ++j) {
          const V2 a = acc[j][k], cc = wc[j][(k + 3) % NS];
          V2 res2 = p_fma(pe_c, cc, p_mul(pe_acc, a));
          if (use_f) res2 = p_fma(pe_f, fo[j], res2);
          if (MODE == kOpCheb) res2 = p_fma(pe_p, po[j], res2);
          T* oj = op + (int64_t)j * res;
          *reinterpret_cast<V2*>(oj) = res2;
          if (two) *reinterpret_cast<V2*>(A.out2 + (oj - out)) = cc;
          if (refine) *reinterpret_cast<float2*>(A.r32 + (oj - out)) = make_float2((float)res2.x, (float)res2.y);
          if ((MODE == kOpResid || refine) && want_dot)
            dacc += (double)res2.x * (double)res2.x + (double)res2.y * (double)res2.y;
          if ((MODE == kOpApply || MODE == kOpApplyD) && want_dot)
            dacc += (double)cc.x * (double)res2.x + (double)cc.y * (double)res2.y;
          if (MODE == kOpCheb && want_dot) dacc += (double)fo[j].x * (double)res2.x + (double)fo[j].y * (double)res2.y;
        }
      }
      op += plane;
    }
    if (stop) break;
  }
  if (stop && t == 0) {
    for (int q = it; q < min(it + NS, nissue); ++q) mbar_wait(&bar[q % NS], (uint32_t)(q / NS) & 1u);
  }
  if ((MODE == kOpApply || MODE == kOpCheb || MODE == kOpApplyD || MODE == kOpResid || refine) && A.dot != nullptr) {
    typedef cub::BlockReduce<double, kThreadsR> BR;
    __shared__ typename BR::TempStorage tmp;
    const double tot = BR(tmp).Sum(dacc);
    if (t == 0)
      A.dot[A.dot_base + (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = tot;
  }
}

// one warp sums np partials in a fixed order
__global__ void k_sum_parts(const double* __restrict__ part, int np, double* __restrict__ out) {
  double s = 0.0;
  for (int i = threadIdx.x; i < np; i += 32) s += part[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (threadIdx.x == 0) out[0] = s;
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

// Grid transfers with the B2 subdivision P (fine 2c + k <- coarse c, weights 1/4, 3/4, 3/4, 1/4 for
// k = -1..2), separable, two coarse nodes (2c', 2c' + 1) per thread: the prolongation
// (out = xf + P ec) writes the fine 4 x 2 x 2 block 4c' .. 4c' + 3 from the coarse 4 x 3 x 3
// neighbourhood; the restriction reads fine rows 4c' - 1 .. 4c' + 4 (a scalar, four 16-byte
// aligned values, a scalar).
template <typename T>
struct F4 {
  T v[4];
};
template <typename T>
__device__ __forceinline__ F4<T> ld4x(const T* p) {
  typedef typename Vec2<T>::type V2;
  if (sizeof(T) == 4) {
    const float4 a = *reinterpret_cast<const float4*>(p);
    return F4<T>{{(T)a.x, (T)a.y, (T)a.z, (T)a.w}};
  }
  const V2 a = reinterpret_cast<const V2*>(p)[0], b = reinterpret_cast<const V2*>(p)[1];
  return F4<T>{{a.x, a.y, b.x, b.y}};
}
template <typename T>
__device__ __forceinline__ void st4x(T* p, const F4<T>& v) {
  typedef typename Vec2<T>::type V2;
  if (sizeof(T) == 4) {
    *reinterpret_cast<float4*>(p) = make_float4((float)v.v[0], (float)v.v[1], (float)v.v[2], (float)v.v[3]);
    return;
  }
  reinterpret_cast<V2*>(p)[0] = V2{v.v[0], v.v[1]};
  reinterpret_cast<V2*>(p)[1] = V2{v.v[2], v.v[3]};
}

template <typename T>
__global__ void k_prolong4(const T* __restrict__ xf, const T* __restrict__ ec, int Lf, T* __restrict__ out) {
  typedef typename Vec2<T>::type V2;
  const int Lc = Lf - 1, rc = 1 << Lc, rf = 1 << Lf, hc = rc >> 1;
  const uint64_t np = 1ull << (3 * Lc - 1);
  const int64_t pc = (int64_t)rc * rc, pf = (int64_t)rf * rf;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < np; i += (uint64_t)gridDim.x * blockDim.x) {
    const int cp = (int)(i % hc), cy = (int)((i / hc) % rc), cz = (int)(i / ((uint64_t)hc * rc));
    const int c0 = 2 * cp;
    T a[3][3][4];  // x pass: [dz][dy][fine x 4cp .. 4cp + 3]
#pragma unroll
    for (int dz = 0; dz < 3; ++dz)
#pragma unroll
      for (int dy = 0; dy < 3; ++dy) {
        const int Z = cz + dz - 1, Y = cy + dy - 1;
        T em = 0, e0 = 0, e1 = 0, ep = 0;  // coarse c0 - 1, c0, c0 + 1, c0 + 2
        if (Z >= 0 && Z < rc && Y >= 0 && Y < rc) {
          const T* row = ec + Z * pc + (int64_t)Y * rc;
          const V2 e = *reinterpret_cast<const V2*>(row + c0);
          e0 = e.x;
          e1 = e.y;
          if (c0 > 0) em = row[c0 - 1];
          if (c0 + 2 < rc) ep = row[c0 + 2];
        }
        a[dz][dy][0] = T(0.75) * e0 + T(0.25) * em;
        a[dz][dy][1] = T(0.75) * e0 + T(0.25) * e1;
        a[dz][dy][2] = T(0.75) * e1 + T(0.25) * e0;
        a[dz][dy][3] = T(0.75) * e1 + T(0.25) * ep;
      }
#pragma unroll
    for (int zo = 0; zo < 2; ++zo)
#pragma unroll
      for (int yo = 0; yo < 2; ++yo) {
        const int64_t f = (int64_t)(4 * cp) + (int64_t)rf * (2 * cy + yo) + pf * (2 * cz + zo);
        F4<T> v = ld4x(xf + f);
#pragma unroll
        for (int xo = 0; xo < 4; ++xo) {
          T b[3];
#pragma unroll
          for (int dz = 0; dz < 3; ++dz) b[dz] = T(0.75) * a[dz][1][xo] + T(0.25) * a[dz][yo == 0 ? 0 : 2][xo];
          v.v[xo] += T(0.75) * b[1] + T(0.25) * b[zo == 0 ? 0 : 2];
        }
        st4x(out + f, v);
      }
  }
}

template <typename T>
__global__ void k_restrict4(const T* __restrict__ rf, int Lf, T* __restrict__ fc) {
  typedef typename Vec2<T>::type V2;
  const int Lc = Lf - 1, res = 1 << Lf, rc = 1 << Lc, hc = rc >> 1;
  const uint64_t np = 1ull << (3 * Lc - 1);
  const int64_t pf = (int64_t)res * res, pc = (int64_t)rc * rc;
  const T w[4] = {T(0.25), T(0.75), T(0.75), T(0.25)};
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < np; i += (uint64_t)gridDim.x * blockDim.x) {
    const int cp = (int)(i % hc), cy = (int)((i / hc) % rc), cz = (int)(i / ((uint64_t)hc * rc));
    T acc0 = 0, acc1 = 0;
#pragma unroll
    for (int kz = 0; kz < 4; ++kz) {
      const int fz = 2 * cz - 1 + kz;
      if (fz < 0 || fz >= res) continue;
      T az0 = 0, az1 = 0;
#pragma unroll
      for (int ky = 0; ky < 4; ++ky) {
        const int fy = 2 * cy - 1 + ky;
        if (fy < 0 || fy >= res) continue;
        const T* row = rf + fz * pf + (int64_t)fy * res + 4 * cp;
        const F4<T> c = ld4x(row);
        const T lo = cp > 0 ? row[-1] : T(0), hi = 4 * cp + 4 < res ? row[4] : T(0);
        const T ax0 = T(0.25) * (lo + c.v[2]) + T(0.75) * (c.v[0] + c.v[1]);
        const T ax1 = T(0.25) * (c.v[1] + hi) + T(0.75) * (c.v[2] + c.v[3]);
        az0 += w[ky] * ax0;
        az1 += w[ky] * ax1;
      }
      acc0 += w[kz] * az0;
      acc1 += w[kz] * az1;
    }
    *reinterpret_cast<V2*>(fc + cz * pc + (int64_t)cy * rc + 2 * cp) = V2{acc0, acc1};
  }
}

// The restriction on the TMA levels (fine res >= 64), streaming in z: a CTA owns a 64 x 16 fine
// tile (32 x 8 coarse nodes) and kRestrictCZ coarse planes, with the fine planes 2 cz0 - 1 ..
// 2 cz1 staged through a four-deep ring (72 x 18 FP32 / 68 x 18 FP64 boxes: fine rows y0 - 1 ..
// y0 + 16 and the columns 4c' - 1 .. 4c' + 4 of every coarse pair). A thread owns one coarse
// pair in one coarse row: x and y restriction from shared memory as in k_restrict4, z in
// registers with the terms of every coarse plane added in the order kz = 0..3. Planes, rows and
// columns outside the grid read as zeros.
constexpr int kRestrictCZ = 38;  // coarse planes per CTA: 78 staged fine planes
template <typename T>
struct GeoRs {
  static constexpr int NS = 4;
  static constexpr int BW = Geo3<T>::BW, XOFF = Geo3<T>::XOFF;  // stage column of global x0 - 2 is XOFF
  static constexpr int SR = 18;                                   // fine rows y0 - 1 .. y0 + 16
  static constexpr uint32_t SBYTES = BW * SR * sizeof(T);    // one box
  static constexpr uint32_t SSTRIDE = (SBYTES + 127) & ~127u;  // stages 128-byte aligned
  static constexpr size_t OFF_BAR = (size_t)NS * SSTRIDE;
  static constexpr size_t BYTES = OFF_BAR + NS * 8 + 16;
};

template <typename T>
__global__ void __launch_bounds__(kThreadsR) k_restrict3(const __grid_constant__ CUtensorMap mr, int Lf,
                                                         T* __restrict__ fc, int* __restrict__ err) {
  typedef GeoRs<T> G;
  typedef typename Vec2<T>::type V2;
  constexpr int NS = G::NS, BW = G::BW, XOFF = G::XOFF;
  extern __shared__ __align__(128) unsigned char smem[];
  auto stage = [&](int st) { return reinterpret_cast<T*>(smem + (size_t)st * G::SSTRIDE); };  // [SR][BW]
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + G::OFF_BAR);
  int* s_abort = reinterpret_cast<int*>(smem + G::OFF_BAR + NS * 8);
  const int res = 1 << Lf, rc = res >> 1;
  const int64_t pc = (int64_t)rc * rc;
  const int t = threadIdx.x, tx = t & 15, ty = t >> 4;  // coarse pair tx, coarse row ty of the tile
  const int x0 = blockIdx.x * 64, y0 = blockIdx.y * 16;
  const int cz0 = blockIdx.z * kRestrictCZ, cz1 = min(cz0 + kRestrictCZ, rc);
  const int nplanes = 2 * (cz1 - cz0) + 2;  // fine 2 cz0 - 1 .. 2 cz1
  if (t == 0) {
    for (int q = 0; q < NS; ++q) mbar_init(&bar[q], 1);
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto issue = [&](int q) {
    mbar_expect_tx(&bar[q % NS], G::SBYTES);
    tma_load_3d(stage(q % NS), &mr, x0 - 2 - XOFF, y0 - 1, 2 * cz0 - 1 + q, &bar[q % NS]);
  };
  if (t == 0)
    for (int q = 0; q < NS && q < nplanes; ++q) issue(q);
  const T w[4] = {T(0.25), T(0.75), T(0.75), T(0.25)};
  const int c0 = 4 * tx + 2 + XOFF;  // stage column of fine 4c' (c' = x0 / 4 + tx)
  T* out = fc + (int64_t)(x0 / 2 + 2 * tx) + (int64_t)rc * (y0 / 2 + ty);
  T acc[2][2] = {{T(0), T(0)}, {T(0), T(0)}};  // [coarse plane cz, cz + 1][pair]
  int q = 0;
  bool stop = false;
  for (; q < nplanes; ++q) {
    const int st = q % NS;
    if (!mbar_wait(&bar[st], (uint32_t)(q / NS) & 1u)) {
      atomicExch(err, 1);
      *s_abort = 1;
    }
    T az0 = 0, az1 = 0;  // x and y restriction of fine plane 2 cz0 - 1 + q
#pragma unroll
    for (int ky = 0; ky < 4; ++ky) {
      const T* row = stage(st) + (2 * ty + ky) * BW + c0;
      const F4<T> c = ld4x(row);
      const T lo = row[-1], hi = row[4];
      const T ax0 = T(0.25) * (lo + c.v[2]) + T(0.75) * (c.v[0] + c.v[1]);
      const T ax1 = T(0.25) * (c.v[1] + hi) + T(0.75) * (c.v[2] + c.v[3]);
      az0 += w[ky] * ax0;
      az1 += w[ky] * ax1;
    }
    __syncthreads();  // stage st is read
    if (*s_abort) {
      stop = true;
      break;
    }
    if (t == 0 && q + NS < nplanes) issue(q + NS);
    // fine plane 2 cz0 - 1 + q is kz = (q & 1) of coarse cz0 + q / 2 (acc[1], or acc[0] while
    // q < 2) and kz = 2 + (q & 1) of coarse cz0 + q / 2 - 1 (acc[0]), emitted after its kz = 3
    const int kz = q & 1;
    const T wn = kz ? T(0.75) : T(0.25), wc = kz ? T(0.25) : T(0.75);  // w[kz], w[2 + kz]
    if (q < nplanes - 2) {
      if (q >= 2) {
        acc[1][0] += wn * az0;
        acc[1][1] += wn * az1;
      } else {
        acc[0][0] += wn * az0;
        acc[0][1] += wn * az1;
      }
    }
    if (q >= 2) {
      acc[0][0] += wc * az0;
      acc[0][1] += wc * az1;
      if (kz == 1) {
        *reinterpret_cast<V2*>(out + (cz0 + q / 2 - 1) * pc) = V2{acc[0][0], acc[0][1]};
        acc[0][0] = acc[1][0];
        acc[0][1] = acc[1][1];
        acc[1][0] = acc[1][1] = T(0);
      }
    }
  }
  if (stop && t == 0) {
    for (int r = q; r < min(q + NS, nplanes); ++r) mbar_wait(&bar[r % NS], (uint32_t)(r / NS) & 1u);
  }
}

// The prolongation out = xf + P ec on the TMA levels (fine res >= 64), streaming in z: a CTA owns
// a 64 x 16 fine tile and kProlongCZ coarse planes; the coarse planes cz0 - 1 .. cz1 (rows and
// columns with a one-node halo) come through a TMA ring and are read once each, into a rolling
// window of three coarse planes interpolated in x and y. A thread owns the fine 4 x 2 block of one
// coarse pair in one coarse row (as k_prolong4, same arithmetic), and reads and writes its fine
// rows with 16-byte accesses.
constexpr int kProlongCZ = 32;
template <typename T>
struct GeoPr {
  static constexpr int NS = 6;
  static constexpr int XO = sizeof(T) == 4 ? 4 : 2;   // stage column of coarse cx0 (16-byte aligned start)
  static constexpr int CW = sizeof(T) == 4 ? 40 : 36;  // staged coarse columns cx0 - XO ..
  static constexpr int CR = 10;                         // coarse rows cy0 - 1 .. cy0 + 8
  static constexpr uint32_t SBYTES = CW * CR * sizeof(T);
  static constexpr uint32_t SSTRIDE = (SBYTES + 127) & ~127u;
  static constexpr size_t OFF_BAR = (size_t)NS * SSTRIDE;
  static constexpr size_t BYTES = OFF_BAR + NS * 8 + 16;
};

template <typename T>
__global__ void __launch_bounds__(kThreadsR) k_prolong3(const __grid_constant__ CUtensorMap mc, const T* __restrict__ xf,
                                                        int Lf, T* __restrict__ out, int* __restrict__ err) {
  typedef GeoPr<T> G;
  typedef typename Vec2<T>::type V2;
  constexpr int NS = G::NS, XO = G::XO, CW = G::CW;
  extern __shared__ __align__(128) unsigned char smem[];
  auto stage = [&](int st) { return reinterpret_cast<const T*>(smem + (size_t)st * G::SSTRIDE); };  // [CR][CW]
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + G::OFF_BAR);
  int* s_abort = reinterpret_cast<int*>(smem + G::OFF_BAR + NS * 8);
  const int rf = 1 << Lf, rc = rf >> 1;
  const int64_t pf = (int64_t)rf * rf;
  const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
  const int x0 = blockIdx.x * 64, y0 = blockIdx.y * 16, cx0 = x0 / 2, cy0 = y0 / 2;
  const int cz0 = blockIdx.z * kProlongCZ, cz1 = min(cz0 + kProlongCZ, rc);
  const int nplanes = cz1 - cz0 + 2;  // coarse cz0 - 1 .. cz1
  if (t == 0) {
    for (int q = 0; q < NS; ++q) mbar_init(&bar[q], 1);
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto issue = [&](int q) {
    mbar_expect_tx(&bar[q % NS], G::SBYTES);
    tma_load_3d(const_cast<T*>(stage(q % NS)), &mc, cx0 - XO, cy0 - 1, cz0 - 1 + q, &bar[q % NS]);
  };
  if (t == 0)
    for (int q = 0; q < NS && q < nplanes; ++q) issue(q);
  // x and y interpolation of staged coarse plane q: B[yo][xo] for fine rows 2ty + yo, columns 4tx + xo
  auto interp = [&](int q, T B[2][4]) -> bool {
    const int st = q % NS;
    bool ok = true;
    if (!mbar_wait(&bar[st], (uint32_t)(q / NS) & 1u)) {
      atomicExch(err, 1);
      *s_abort = 1;
      ok = false;
    }
    T a[3][4];
#pragma unroll
    for (int dy = 0; dy < 3; ++dy) {
      const T* row = stage(st) + (ty + dy) * CW + 2 * tx + XO;  // coarse row cy - 1 + dy, column 2tx
      const V2 e = *reinterpret_cast<const V2*>(row);
      const T e0 = e.x, e1 = e.y, em = row[-1], ep = row[2];
      a[dy][0] = T(0.75) * e0 + T(0.25) * em;
      a[dy][1] = T(0.75) * e0 + T(0.25) * e1;
      a[dy][2] = T(0.75) * e1 + T(0.25) * e0;
      a[dy][3] = T(0.75) * e1 + T(0.25) * ep;
    }
#pragma unroll
    for (int xo = 0; xo < 4; ++xo) {
      B[0][xo] = T(0.75) * a[1][xo] + T(0.25) * a[0][xo];
      B[1][xo] = T(0.75) * a[1][xo] + T(0.25) * a[2][xo];
    }
    __syncthreads();  // stage st is read
    if (*s_abort) return false;
    if (t == 0 && q + NS < nplanes) issue(q + NS);
    return ok;
  };
  T B0[2][4], B1[2][4], B2[2][4];  // coarse planes cz - 1, cz, cz + 1
  int q = 0;                        // the next staged plane to read
  bool good = interp(q, B1);
  if (good) good = interp(++q, B2);
  if (good) ++q;
  for (int cz = cz0; good && cz < cz1; ++cz, ++q) {
#pragma unroll
    for (int yo = 0; yo < 2; ++yo)
#pragma unroll
      for (int xo = 0; xo < 4; ++xo) {
        B0[yo][xo] = B1[yo][xo];
        B1[yo][xo] = B2[yo][xo];
      }
    good = interp(q, B2);
    if (!good) break;
#pragma unroll
    for (int zo = 0; zo < 2; ++zo)
#pragma unroll
      for (int yo = 0; yo < 2; ++yo) {
        const int64_t f = (int64_t)(x0 + 4 * tx) + (int64_t)rf * (y0 + 2 * ty + yo) + pf * (2 * cz + zo);
        F4<T> v = ld4x(xf + f);
#pragma unroll
        for (int xo = 0; xo < 4; ++xo) v.v[xo] += T(0.75) * B1[yo][xo] + T(0.25) * (zo == 0 ? B0 : B2)[yo][xo];
        st4x(out + f, v);
      }
  }
  if (!good && t == 0) {
    for (int r = q; r < min(q + NS, nplanes); ++r) mbar_wait(&bar[r % NS], (uint32_t)(r / NS) & 1u);
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
// 9 (dz + 1) + 3 (dy + 1) + (dx + 1); basis values (FP64, FP32); count of points with a node.
// One thread per pair (the point's three axis evaluations repeated per pair), so every array is
// written coalesced; a point has a node in the grid iff [c - 1, c + 1] meets [0, res) on every
// axis, counted once per block.
__global__ void k_pair_keys2(const double* __restrict__ upos, uint64_t P, uint32_t D, uint32_t* __restrict__ keys,
                             uint32_t* __restrict__ vals, double* __restrict__ phi64, float* __restrict__ phi32,
                             unsigned long long* __restrict__ nin) {
  const int64_t res = 1ll << D;
  const double h = 1.0 / (double)res;
  const uint32_t sentinel = 1u << (3 * D);
  unsigned long long cnt = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < 27 * P; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t p = i / 27;
    const int k = (int)(i - 27 * p), dx = k % 3, dy = (k / 3) % 3, dz = k / 9;
    int64_t c[3];
    double b[3][3];
    axis2(upos[p], h, c[0], b[0]);
    axis2(upos[P + p], h, c[1], b[1]);
    axis2(upos[2 * P + p], h, c[2], b[2]);
    const int64_t x = c[0] + dx - 1, y = c[1] + dy - 1, z = c[2] + dz - 1;
    const bool ok = x >= 0 && y >= 0 && z >= 0 && x < res && y < res && z < res;
    keys[i] = ok ? (uint32_t)(x + res * (y + res * z)) : sentinel;
    vals[i] = (uint32_t)i;
    const double phi = ok ? xmul(xmul(b[0][dx], b[1][dy]), b[2][dz]) : 0.0;
    phi64[i] = phi;
    phi32[i] = (float)phi;
    if (k == 0)
      cnt += (c[0] + 1 >= 0 && c[0] - 1 < res && c[1] + 1 >= 0 && c[1] - 1 < res && c[2] + 1 >= 0 && c[2] - 1 < res);
  }
  typedef cub::BlockReduce<unsigned long long, kThreads> BR;
  __shared__ typename BR::TempStorage tmp;
  const unsigned long long tot = BR(tmp).Sum(cnt);
  if (threadIdx.x == 0 && tot) atomicAdd(nin, tot);
}

// splat per touched node, points in input order: nf = -(sum phi n) / (sum phi), w = sum phi
__global__ void k_splat2(const uint32_t* __restrict__ run_key, const uint32_t* __restrict__ run_off, uint64_t T,
                         const uint32_t* __restrict__ sval, const double* __restrict__ phi,
                         const double* __restrict__ unrm, uint64_t P, uint64_t n, double* __restrict__ nf,
                         double* __restrict__ w) {  // w: the weights alone (nf == nullptr), for the accessor
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < T; t += (uint64_t)gridDim.x * blockDim.x) {
    double fx = 0.0, fy = 0.0, fz = 0.0, sw = 0.0;
    for (uint32_t e = run_off[t]; e < run_off[t + 1]; ++e) {
      const uint32_t pk = sval[e];
      const uint32_t p = pk / 27;
      const double wgt = phi[pk];
      if (nf) {
        fx = xadd(fx, xmul(unrm[p], wgt));
        fy = xadd(fy, xmul(unrm[P + p], wgt));
        fz = xadd(fz, xmul(unrm[2 * P + p], wgt));
      }
      sw = xadd(sw, wgt);
    }
    const uint32_t node = run_key[t];
    if (!nf) {
      w[node] = sw;
      continue;
    }
    if (sw > 0.0) {
      fx = xdiv(-fx, sw);
      fy = xdiv(-fy, sw);
      fz = xdiv(-fz, sw);
    }
    nf[node] = fx;
    nf[n + node] = fy;
    nf[2 * n + node] = fz;
  }
}

// 1-D integrals of the right-hand side (g: N2' N2, m: N2 N2), h^2, the TMA wait flag
struct RhsCoef {
  double g[5], m[5], h2;
  int* err;
};

// the same per touched node, into a compact field: nfc[t], nfc[T + t], nfc[2 T + t] for run t
__global__ void k_splat2c(const uint32_t* __restrict__ run_off, uint64_t T, const uint32_t* __restrict__ sval,
                          const double* __restrict__ phi, const double* __restrict__ unrm, uint64_t P,
                          double* __restrict__ nfc) {
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
    nfc[t] = fx;
    nfc[T + t] = fy;
    nfc[2 * T + t] = fz;
  }
}
// dense[node] = compact[t] per component (the accessor's and the small levels' dense field)
__global__ void k_nf_scatter(const uint32_t* __restrict__ run_key, uint64_t T, const double* __restrict__ nfc,
                             uint64_t n, double* __restrict__ nf) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < T; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t node = run_key[t];
    nf[node] = nfc[t];
    nf[n + node] = nfc[T + t];
    nf[2 * n + node] = nfc[2 * T + t];
  }
}

// Bricks (8^3 blocks of the natural-order grid) whose right-hand side can be nonzero: those within
// 2 nodes of a touched node.  flag[brick] = 1, brick = bx + nb (by + nb bz).
__global__ void k_rhs_mark_bricks(const uint32_t* __restrict__ run_key, uint64_t T, int D, uint8_t* __restrict__ flag) {
  const int res = 1 << D, nb = res >> 3;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < T; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t node = run_key[t];
    const int c[3] = {(int)(node & (res - 1)), (int)((node >> D) & (res - 1)), (int)(node >> (2 * D))};
    int lo[3], hi[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      lo[a] = max(c[a] - 2, 0) >> 3;
      hi[a] = min(c[a] + 2, res - 1) >> 3;
    }
    for (int z = lo[2]; z <= hi[2]; ++z)
      for (int y = lo[1]; y <= hi[1]; ++y)
        for (int x = lo[0]; x <= hi[0]; ++x) flag[x + nb * (y + nb * z)] = 1;
  }
}

// b = h^2 sum_a (G_a M M) nf_a on the listed bricks (b is zero elsewhere): per brick, the compact
// normal field of the brick and its 2-node halo goes into a shared 12^3 x 3 tile (each of the
// 144 tile rows found by a binary search of the sorted run keys), then z, y and x passes.
constexpr int kRB = 12, kRB3 = kRB * kRB * kRB;
constexpr size_t kRhsBrickSmem = (3 * kRB3 + 8 * kRB * kRB + 8 * 8 * kRB) * sizeof(double);
__global__ void __launch_bounds__(kThreads) k_rhs2_bricks(const uint32_t* __restrict__ bricks, uint64_t NBo, int D,
                                                          const uint32_t* __restrict__ run_key, uint64_t T,
                                                          const double* __restrict__ nfc, RhsCoef k,
                                                          double* __restrict__ b) {
  extern __shared__ double sm2[];
  double* nf = sm2;                 // [3][12][12][12]
  double* tz = nf + 3 * kRB3;       // [8][12][12]
  double* ty = tz + 8 * kRB * kRB;  // [8][8][12]
  const int t = threadIdx.x, res = 1 << D, nb = res >> 3;
  for (uint64_t i = blockIdx.x; i < NBo; i += gridDim.x) {
    const uint32_t bid = bricks[i];
    const int bx = (int)(bid % nb), by = (int)((bid / nb) % nb), bz = (int)(bid / ((uint32_t)nb * nb));
    const int ox = 8 * bx - 2, oy = 8 * by - 2, oz = 8 * bz - 2;
    for (int j = t; j < 3 * kRB3; j += kThreads) nf[j] = 0.0;
    __syncthreads();
    if (t < kRB * kRB) {
      const int gy = oy + t % kRB, gz = oz + t / kRB;
      if (gy >= 0 && gz >= 0 && gy < res && gz < res) {
        const uint64_t row = (uint64_t)res * (gy + (uint64_t)res * gz);
        const uint64_t k0 = row + (uint64_t)max(ox, 0), k1 = row + (uint64_t)min(ox + kRB, res);
        uint64_t a = 0, e = T;
        while (a < e) {
          const uint64_t m = (a + e) >> 1;
          if ((uint64_t)run_key[m] < k0) a = m + 1;
          else e = m;
        }
        for (uint64_t r = a; r < T && (uint64_t)run_key[r] < k1; ++r) {
          const int o = t * kRB + (int)((uint64_t)run_key[r] - row) - ox;
          nf[o] = nfc[r];
          nf[kRB3 + o] = nfc[T + r];
          nf[2 * kRB3 + o] = nfc[2 * T + r];
        }
      }
    }
    __syncthreads();
    double acc[2] = {0.0, 0.0};
    for (int a = 0; a < 3; ++a) {
      const double* fz = a == 2 ? k.g : k.m;
      const double* fy = a == 1 ? k.g : k.m;
      const double* fx = a == 0 ? k.g : k.m;
      const double* src = nf + a * kRB3;
      for (int j = t; j < 8 * kRB * kRB; j += kThreads) {
        const int z = j / (kRB * kRB), yx = j % (kRB * kRB);
        double v = 0.0;
#pragma unroll
        for (int c = 0; c < 5; ++c) v += fz[c] * src[(z + c) * kRB * kRB + yx];
        tz[j] = v;
      }
      __syncthreads();
      for (int j = t; j < 8 * 8 * kRB; j += kThreads) {
        const int z = j / (8 * kRB), y = (j / kRB) % 8, x = j % kRB;
        double v = 0.0;
#pragma unroll
        for (int c = 0; c < 5; ++c) v += fy[c] * tz[(z * kRB + y + c) * kRB + x];
        ty[j] = v;
      }
      __syncthreads();
#pragma unroll
      for (int jj = 0; jj < 2; ++jj) {
        const int o = t + jj * kThreads, z = o >> 6, y = (o >> 3) & 7, x = o & 7;
        double v = 0.0;
#pragma unroll
        for (int c = 0; c < 5; ++c) v += fx[c] * ty[(z * 8 + y) * kRB + x + c];
        acc[jj] += v;
      }
      __syncthreads();
    }
#pragma unroll
    for (int jj = 0; jj < 2; ++jj) {
      const int o = t + jj * kThreads, z = o >> 6, y = (o >> 3) & 7, x = o & 7;
      b[(uint64_t)(8 * bx + x) + (uint64_t)res * ((8 * by + y) + (uint64_t)res * (8 * bz + z))] = k.h2 * acc[jj];
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
// (sq: optional per-block sums of proj^2, so that x . (wh3 Phi Phi^T x) = wh3 sum proj^2)
template <typename T>
__global__ void k_screen_proj2(const uint32_t* __restrict__ key, const T* __restrict__ phi, uint64_t P,
                               uint32_t sentinel, const T* __restrict__ x, T* __restrict__ proj,
                               double* __restrict__ sq) {
  double acc = 0.0;
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < P; p += (uint64_t)gridDim.x * blockDim.x) {
    T s = 0;
    for (int k = 0; k < 27; ++k) {
      const uint32_t kk = key[27 * p + k];
      if (kk != sentinel) s += phi[27 * p + k] * x[kk];
    }
    proj[p] = s;
    acc += (double)s * (double)s;
  }
  if (sq) {
    typedef cub::BlockReduce<double, kThreads> BR;
    __shared__ typename BR::TempStorage tmp;
    const double tot = BR(tmp).Sum(acc);
    if (threadIdx.x == 0) sq[blockIdx.x] = tot;
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
// k_screen_gather2 for the fused refinement: also rounds the updated residual to y32 (if given) and leaves
// per-block sums of (y_new^2 - y_old^2), so that ||y||^2 = (the operator pass's sum of y_old^2)
// + (these), every term in FP64
template <typename T>
__global__ void k_screen_gather2_fix(const uint32_t* __restrict__ snode, const uint32_t* __restrict__ soff, uint64_t S,
                                     const uint32_t* __restrict__ sval, const T* __restrict__ phi,
                                     const T* __restrict__ proj, T wh3s, T* __restrict__ y, float* __restrict__ y32,
                                     double* __restrict__ part) {
  double dsq = 0.0;
  for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < S; u += (uint64_t)gridDim.x * blockDim.x) {
    T acc = 0;
    for (uint32_t e = soff[u]; e < soff[u + 1]; ++e) {
      const uint32_t pk = sval[e];
      acc += phi[pk] * proj[pk / 27];
    }
    const uint32_t i = snode[u];
    const T old = y[i], nw = old + wh3s * acc;
    y[i] = nw;
    if (y32) y32[i] = (float)nw;
    dsq += (double)nw * (double)nw - (double)old * (double)old;
  }
  typedef cub::BlockReduce<double, kThreads> BR;
  __shared__ typename BR::TempStorage tmp;
  const double tot = BR(tmp).Sum(dsq);
  if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

// natural <-> Morton
template <typename T>
__global__ void k_nat_to_morton(const T* __restrict__ in, uint32_t D, T* __restrict__ out) {
  const uint64_t n = 1ull << (3 * D), m = (1ull << D) - 1;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[morton3((uint32_t)(i & m), (uint32_t)((i >> D) & m), (uint32_t)(i >> (2 * D)))] = in[i];
}

// The same permutation by 16^3 bricks (D >= 4): an aligned brick is 4096 consecutive Morton codes,
// so a CTA reads the brick's natural rows (16 contiguous values), reorders them in shared memory
// and writes one contiguous run.
template <typename T>
__global__ void __launch_bounds__(256) k_nat_to_morton_brick(const T* __restrict__ in, uint32_t D, T* __restrict__ out) {
  __shared__ T s[4096];
  const uint64_t res = 1ull << D, nb = 1ull << (3 * (D - 4));
  for (uint64_t b = blockIdx.x; b < nb; b += gridDim.x) {
    uint32_t bx, by, bz;
    unmorton3((uint32_t)b, bx, by, bz);
    const T* src = in + 16 * ((uint64_t)bx + res * ((uint64_t)by + res * (uint64_t)bz));
#pragma unroll 4
    for (int i = 0; i < 16; ++i) {
      const int e = i * 256 + threadIdx.x, lx = e & 15, ly = (e >> 4) & 15, lz = e >> 8;
      s[morton3((uint32_t)lx, (uint32_t)ly, (uint32_t)lz)] = src[(uint64_t)lx + res * ((uint64_t)ly + res * (uint64_t)lz)];
    }
    __syncthreads();
    T* dst = out + (b << 12);
#pragma unroll 4
    for (int i = 0; i < 16; ++i) dst[i * 256 + threadIdx.x] = s[i * 256 + threadIdx.x];
    __syncthreads();
  }
}
template <typename T>
void nat_to_morton(cudaStream_t s, const T* in, uint32_t D, T* out) {
  if (D >= 4)
    k_nat_to_morton_brick<T><<<(unsigned)std::min<uint64_t>(1ull << (3 * (D - 4)), 148 * 32), 256, 0, s>>>(in, D, out);
  else k_nat_to_morton<T><<<grid_for(1ull << (3 * D)), kThreads, 0, s>>>(in, D, out);
  PR_CHECK_LAUNCH();
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

// ------------------------------------------------------------------ host: tensor maps
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    PR_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    PR_REQUIRE(p != nullptr && q == cudaDriverEntryPointSuccess, PR_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}
// 3-D map of a res^3 natural-order grid with a (bx, by, 1) box; outside the grid reads 0
template <typename T>
CUtensorMap plane_map(const T* base, int L, uint32_t bx, uint32_t by) {
  CUtensorMap m;
  const cuuint64_t res = 1ull << L;
  const cuuint64_t dims[3] = {res, res, res};
  const cuuint64_t strides[2] = {res * sizeof(T), res * res * sizeof(T)};
  const cuuint32_t box[3] = {bx, by, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  PR_REQUIRE((reinterpret_cast<uintptr_t>(base) & 15u) == 0 && (bx * sizeof(T)) % 16 == 0, PR_ERR_INTERNAL,
             "tensor map: base or box not 16-byte aligned");
  const CUresult r = encode_tiled()(&m, sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                                    3, const_cast<T*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  PR_REQUIRE(r == CUDA_SUCCESS, PR_ERR_CUDA, "cuTensorMapEncodeTiled failed with " + std::to_string((int)r));
  return m;
}
constexpr int kTmaMinLevel = 6;  // res >= 64: full 64-wide x tiles (k_op3)

// launches the operator pass of a level: k_op3r when every row is the interior row, else k_op3
// over the interior tiles and the face tiles
// returns the number of CTAs (= dot partials written when a.dot is set)
template <typename T, int MODE>
int launch_op3(pr_context* c, cudaStream_t s, const CUtensorMap& mx, const CUtensorMap& mf, const CUtensorMap& mp,
               T* out, const Op3Args<T>& a, int nz) {
  typedef Geo3<T> G;
  typedef Geo3R<T> GR;
  if constexpr (MODE == kOpRefine) {  // a level without boundary rows only
    PR_REQUIRE(a.edge == 0, PR_ERR_INTERNAL, "the fused refinement needs a level without boundary rows");
    allow_smem(k_op3r<T, MODE>, GR::BYTES);
    Op3Args<T> e = a;
    e.ox = e.oy = e.oz = 0;
    e.dot_base = 0;
    k_op3r<T, MODE><<<dim3(a.nbx, a.nby, nz), kThreadsR, GR::BYTES, s>>>(mx, mf, mp, out, e);
    PR_CHECK_LAUNCH();
    return a.nbx * a.nby * nz;
  } else {
    allow_smem(k_op3<T, MODE, false>, G::BYTES);
    allow_smem(k_op3<T, MODE, true>, G::BYTES);
    allow_smem(k_op3r<T, MODE>, GR::BYTES);
    const int nbx = a.nbx, nby = a.nby;
    Op3Args<T> e = a;
    e.ox = e.oy = e.oz = 0;
    e.dot_base = 0;
    if (a.edge == 0) {  // every row acts as the interior row: one launch of the register-window variant
      k_op3r<T, MODE><<<dim3(nbx, nby, nz), kThreadsR, GR::BYTES, s>>>(mx, mf, mp, out, e);
      PR_CHECK_LAUNCH();
      return nbx * nby * nz;
    }
    // interior tiles need every output row at least `edge` from the faces: edge <= 8 (one tile row)
    const bool split = nbx > 2 && nby > 2 && a.edge <= TY;
    e.all = split ? 0 : 1;
    if (split) {
      e.ox = e.oy = 1;
      // z runs of the interior tiles whose staged planes (and, with edge <= 6, the tiles' halo rows
      // and columns) all act as the interior row run k_op3r, the others k_op3; with fewer than five
      // runs the extra launches cost more than they save
      const int res = nbx * G::TXP;
      int zlo = nz, zhi = nz;
      if (a.edge <= 6 && nz >= 5) {
        zlo = 0;
        while (zlo < nz && zlo * kZChunk3 - 2 < a.edge) ++zlo;
        zhi = zlo;
        while (zhi < nz && std::min((zhi + 1) * kZChunk3, res) + 2 <= res - a.edge) ++zhi;
      }
      const int ni = (nbx - 2) * (nby - 2);
      auto run = [&](int z_begin, int z_end, bool regs) {
        if (z_end <= z_begin) return;
        e.oz = z_begin;
        const dim3 g(nbx - 2, nby - 2, z_end - z_begin);
        if (regs) k_op3r<T, MODE><<<g, kThreadsR, GR::BYTES, s>>>(mx, mf, mp, out, e);
        else k_op3<T, MODE, false><<<g, kThreads, G::BYTES, s>>>(mx, mf, mp, out, e);
        PR_CHECK_LAUNCH();
        e.dot_base += ni * (z_end - z_begin);
      };
      // the face tiles (disjoint outputs and partial slots) run beside the interior launches on
      // the side stream, forked from and joined back to s
      Op3Args<T> ef = e;
      ef.oz = 0;
      ef.ox = ef.oy = 0;
      ef.dot_base = ni * nz;
      cudaStream_t s2 = c->side_stream();
      PR_CUDA(cudaEventRecord(c->ev_fork, s));
      PR_CUDA(cudaStreamWaitEvent(s2, c->ev_fork, 0));
      k_op3<T, MODE, true><<<dim3(2 * nbx + 2 * (nby - 2), 1, nz), kThreads, G::BYTES, s2>>>(mx, mf, mp, out, ef);
      PR_CHECK_LAUNCH();
      run(0, zlo, false);
      run(zlo, zhi, true);
      run(zhi, nz, false);
      PR_CUDA(cudaEventRecord(c->ev_join, s2));
      PR_CUDA(cudaStreamWaitEvent(s, c->ev_join, 0));
    } else {
      k_op3<T, MODE, true><<<dim3(nbx * nby, 1, nz), kThreads, G::BYTES, s>>>(mx, mf, mp, out, e);
      PR_CHECK_LAUNCH();
    }
    return nbx * nby * nz;
  }
}

// out = xf + P ec (fine level Lf)
template <typename T>
void launch_prolong(cudaStream_t s, const T* xf, const T* ec, int Lf, T* out, int* err) {
  if (Lf >= kTmaMinLevel) {
    typedef GeoPr<T> G;
    const int rf = 1 << Lf, rc = rf >> 1;
    const CUtensorMap m = plane_map<T>(ec, Lf - 1, G::CW, G::CR);
    const dim3 grid(rf / 64, rf / 16, (rc + kProlongCZ - 1) / kProlongCZ);
    k_prolong3<T><<<grid, kThreadsR, G::BYTES, s>>>(m, xf, Lf, out, err);
  } else {
    k_prolong4<T><<<grid_for(1ull << (3 * (Lf - 1) - 1)), kThreads, 0, s>>>(xf, ec, Lf, out);
  }
  PR_CHECK_LAUNCH();
}

// the restriction of the fine residual rf (level Lf) to the coarse right-hand side fc
template <typename T>
void launch_restrict(cudaStream_t s, const T* rf, int Lf, T* fc, int* err) {
  if (Lf >= kTmaMinLevel) {
    typedef GeoRs<T> G;
    const int res = 1 << Lf, rc = res >> 1;
    const CUtensorMap m = plane_map<T>(rf, Lf, G::BW, G::SR);
    const dim3 grid(res / 64, res / 16, (rc + kRestrictCZ - 1) / kRestrictCZ);
    k_restrict3<T><<<grid, kThreadsR, G::BYTES, s>>>(m, Lf, fc, err);
  } else {
    k_restrict4<T><<<grid_for(1ull << (3 * (Lf - 1) - 1)), kThreads, 0, s>>>(rf, Lf, fc);
  }
  PR_CHECK_LAUNCH();
}

// ------------------------------------------------------------------ host: the system
template <typename T>
struct Level2 {
  int L = 0;
  uint64_t n = 0;
  T* tM = nullptr;
  T* tS = nullptr;
  double H = 0, wg = 0;
  int edge = 0;           // rows [edge, res - edge) of tM, tS equal the interior row
  double im[5], is[5];    // the interior rows
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
  int* err = nullptr;         // set by a TMA wait that ran out

  // levels D (finest) down to the dense 4^3 level; `multigrid` false: the finest level only
  void init(pr_context* ctx, uint32_t depth, double pw, bool multigrid) {
    c = ctx;
    D = depth;
    const double h = 1.0 / (double)(1u << D);
    const double wh3 = pw > 0.0 ? pw * h * h * h / 1.5 : 0.0;
    const double wg = wh3 * 0.005;
    const std::string tn = tn2<T>();
    err = c->buf<int>("d2_err", 1);
    PR_CUDA(cudaMemsetAsync(err, 0, sizeof(int), c->stream));
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
      {
        // a row acts as the interior row when they agree on every column inside the grid: the
        // kernels read zeros outside it (the truncated rows of the finest level are such rows)
        const int res = 1 << l, mid = res / 2;
        auto same = [&](int i) {
          for (int d = 0; d < 5; ++d) {
            const int col = i + d - 2;
            if (col < 0 || col >= res) continue;
            if ((T)M[5 * i + d] != (T)M[5 * mid + d] || (T)S[5 * i + d] != (T)S[5 * mid + d]) return false;
          }
          return true;
        };
        int e = 0;
        while (e < mid && !(same(e) && same(res - 1 - e))) ++e;
        q.edge = e;
        for (int d = 0; d < 5; ++d) {
          q.im[d] = M[5 * mid + d];
          q.is[d] = S[5 * mid + d];
        }
      }
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

  // y += sign wh3 Phi Phi^T x; with sq, per-block sums of (Phi^T x)^2; returns the block count
  int screen(const T* x, T* y, int sign, double* sq = nullptr) {
    if (scr.S == 0) return 0;
    cudaStream_t s = c->stream;
    const unsigned nb = grid_for(scr.P, 1u << 20);
    k_screen_proj2<T><<<nb, kThreads, 0, s>>>(scr.key, scr.phi, scr.P, scr.sentinel, x, scr.proj, sq);
    PR_CHECK_LAUNCH();
    k_screen_gather2<T><<<grid_for(scr.S, 1u << 20), kThreads, 0, s>>>(scr.snode, scr.soff, scr.S, scr.sval, scr.phi,
                                                                        scr.proj, (T)(sign * scr.wh3), y);
    PR_CHECK_LAUNCH();
    bytes += (double)scr.P * 27 * (4 + 2 * sizeof(T)) + (double)scr.P * sizeof(T) +
             (double)scr.pairs * (4 + 2 * sizeof(T)) + (double)scr.S * (8 + 2 * sizeof(T));
    return (int)nb;
  }

  // The FP64 refinement step on the finest level in one operator pass: xn = x + e (x = 0 when
  // xzero), r = b - A xn with the screening term, r32 = (float) r; returns ||r||
  double refine(const T* x, const float* e32, const T* b, T* xn, T* r, float* r32, bool xzero) {
    alloc_parts();
    Fuse fu;
    fu.out2 = xn;
    fu.e32 = e32;
    fu.r32 = r32;
    fu.xzero = xzero;
    const int na = op(0, kOpRefine, x, b, nullptr, r, 0.0, 0.0, 1, 0.0, parts_a, &fu);
    const int nb = screen_fix(xn, r, r32);
    return std::sqrt(std::max(0.0, sum_parts(na, nb, 1.0)));
  }
  // r = b - A x with the screening term on the finest level (TMA operator) and ||r|| from the
  // pass's partials
  double resid_norm(const T* x, const T* b, T* r) {
    alloc_parts();
    const int na = op(0, kOpResid, x, b, nullptr, r, 0.0, 0.0, 1, 0.0, parts_a);
    const int nb = screen_fix(x, r, nullptr);
    return std::sqrt(std::max(0.0, sum_parts(na, nb, 1.0)));
  }
  // r -= wh3 Phi Phi^T x with r32 (if given) updated at the screened nodes and per-block partials
  // of the change of r . r in parts_b; returns the partial count
  int screen_fix(const T* x, T* r, float* r32) {
    if (scr.S == 0) return 0;
    cudaStream_t s = c->stream;
    const unsigned np = grid_for(scr.P, 1u << 20);
    k_screen_proj2<T><<<np, kThreads, 0, s>>>(scr.key, scr.phi, scr.P, scr.sentinel, x, scr.proj, nullptr);
    PR_CHECK_LAUNCH();
    const int nb = (int)grid_for(scr.S, 1u << 20);
    k_screen_gather2_fix<T><<<nb, kThreads, 0, s>>>(scr.snode, scr.soff, scr.S, scr.sval, scr.phi, scr.proj,
                                                     (T)(-scr.wh3), r, r32, parts_b);
    PR_CHECK_LAUNCH();
    bytes += (double)scr.P * 27 * (4 + 2 * sizeof(T)) + (double)scr.P * sizeof(T) +
             (double)scr.pairs * (4 + 2 * sizeof(T)) + (double)scr.S * (8 + 2 * sizeof(T) + (r32 ? 4 : 0));
    return nb;
  }

  // fused dot products (finest level on the TMA operator): per-CTA partials and their sums
  double* parts_a = nullptr;  // operator partials
  double* parts_b = nullptr;  // screening partials
  double* sums = nullptr;     // 2 doubles
  double* rz_parts = nullptr; // set by pcg2: the last post-smoothing step at level 0 writes f . out
  int rz_np = 0;
  bool fused_dots() const { return !lv.empty() && lv[0].L >= kTmaMinLevel; }
  void alloc_parts() {
    const int res = 1 << lv[0].L;
    const size_t tiles = (size_t)(res / Geo3<T>::TXP) * (res / TY) * ((res + kZChunk3 - 1) / kZChunk3);
    parts_a = c->buf<double>(std::string("d2_parts_a_") + tn2<T>(), tiles);
    parts_b = c->buf<double>(std::string("d2_parts_b_") + tn2<T>(), 1u << 20);
    sums = c->buf<double>(std::string("d2_sums_") + tn2<T>(), 2);
  }
  // na partials of parts_a + w * (nb partials of parts_b), summed in a fixed order
  double sum_parts(int na, int nb, double w) {
    cudaStream_t s = c->stream;
    k_sum_parts<<<1, 32, 0, s>>>(parts_a, na, sums);
    PR_CHECK_LAUNCH();
    if (nb > 0) {
      k_sum_parts<<<1, 32, 0, s>>>(parts_b, nb, sums + 1);
      PR_CHECK_LAUNCH();
    }
    PR_CUDA(cudaMemcpyAsync(c->h_scalars, sums, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    c->sync();
    return c->h_scalars[0] + (nb > 0 ? w * c->h_scalars[1] : 0.0);
  }

  // One operator pass on level li (modes k_op2 / k_op3); c0 is the first Chebyshev coefficient of
  // the fused modes.  tma < 0: k_op3 on levels with res >= 64, k_op2 below.
  // the fused CG direction update (kOpApplyD): f is the second staged plane (z)
  struct Fuse {
    T* out2 = nullptr;
    T* xacc = nullptr;
    double s1 = 0.0, s2 = 0.0;
    int xmode = 2;               // see Op3Args::xmode
    const float* e32 = nullptr;  // kOpRefine: the correction
    float* r32 = nullptr;        // kOpRefine: the residual in FP32
    bool xzero = false;          // kOpRefine: x = 0
  };
  int op(int li, int mode, const T* x, const T* f, const T* xp, T* out, double a = 0.0, double b = 0.0,
         int tma = -1, double c0 = 0.0, double* dot = nullptr, const Fuse* fu = nullptr) {
    int nparts = 0;
    const Level2<T>& q = lv[li];
    const int res = 1 << q.L;
    cudaStream_t s = c->stream;
    const LevelView<T> v = q.view();
    if (tma < 0) tma = q.L >= kTmaMinLevel;
    if (tma) {
      PR_REQUIRE(q.L >= kTmaMinLevel, PR_ERR_INTERNAL, "TMA operator below its minimum level");
      typedef Geo3<T> G;
      Op3Args<T> A{};  // every field zero unless set below
      A.lv = v;
      for (int d = 0; d < 5; ++d) {
        A.im[d] = (T)q.im[d];
        A.is[d] = (T)q.is[d];
      }
      A.invd = (T)(1.0 / (q.H * ((q.is[2] * q.im[2] + q.im[2] * q.is[2]) * q.im[2] + q.im[2] * q.im[2] * q.is[2]) + q.wg));
      A.edge = q.edge;
      A.ca = (T)a;
      A.cb = (T)b;
      A.c0 = (T)c0;
      A.use_p = (mode == kOpCheb && xp) ? 1 : 0;
      A.nbx = res / G::TXP;
      A.nby = res / TY;
      A.err = err;
      A.dot = dot;
      A.dot_base = 0;
      const bool two = mode == kOpApplyD, refine = mode == kOpRefine;
      PR_REQUIRE(!two || (fu && fu->out2 && fu->xacc && f), PR_ERR_INTERNAL, "fused CG pass without its operands");
      PR_REQUIRE(!refine || (fu && fu->out2 && fu->e32 && fu->r32 && f && sizeof(T) == 8), PR_ERR_INTERNAL,
                 "fused refinement without its operands");
      A.r32 = refine ? fu->r32 : nullptr;
      A.xzero = refine && fu->xzero ? 1 : 0;
      A.s1 = two ? (T)fu->s1 : T(0);
      A.s2 = two ? (T)fu->s2 : T(0);
      A.out2 = (two || refine) ? fu->out2 : nullptr;
      A.xacc = two ? fu->xacc : nullptr;
      A.xmode = two ? fu->xmode : 0;
      const int nz = (res + kZChunk3 - 1) / kZChunk3;
      const CUtensorMap mx = plane_map<T>(x, q.L, G::BW, SH);
      const CUtensorMap mf = f ? (two ? plane_map<T>(f, q.L, G::BW, SH) : plane_map<T>(f, q.L, G::TXP, TY)) : mx;
      const CUtensorMap mp = refine ? plane_map<float>(fu->e32, q.L, 72, SH)
                                    : (xp ? plane_map<T>(xp, q.L, G::TXP, TY) : mx);
      switch (mode) {
        case kOpApply: nparts = launch_op3<T, kOpApply>(c, s, mx, mf, mp, out, A, nz); break;
        case kOpResid: nparts = launch_op3<T, kOpResid>(c, s, mx, mf, mp, out, A, nz); break;
        case kOpCheb: nparts = launch_op3<T, kOpCheb>(c, s, mx, mf, mp, out, A, nz); break;
        case kOpChebF: nparts = launch_op3<T, kOpChebF>(c, s, mx, mf, mp, out, A, nz); break;
        case kOpChebPF: nparts = launch_op3<T, kOpChebPF>(c, s, mx, mf, mp, out, A, nz); break;
        case kOpRefine:
          if constexpr (sizeof(T) == 8) nparts = launch_op3<T, kOpRefine>(c, s, mx, mf, mp, out, A, nz);
          break;
        default: nparts = launch_op3<T, kOpApplyD>(c, s, mx, mf, mp, out, A, nz); break;
      }
    } else {
      PR_REQUIRE(mode <= kOpCheb, PR_ERR_INTERNAL, "fused Chebyshev modes need the TMA operator");
      PR_REQUIRE(dot == nullptr, PR_ERR_INTERNAL, "fused dot products need the TMA operator");
      dim3 grid((res + TX - 1) / TX, (res + TY - 1) / TY, (res + kZChunk - 1) / kZChunk);
      if (mode == kOpApply) k_op2<T, kOpApply><<<grid, kThreads, 0, s>>>(x, f, xp, out, v, (T)a, (T)b);
      else if (mode == kOpResid) k_op2<T, kOpResid><<<grid, kThreads, 0, s>>>(x, f, xp, out, v, (T)a, (T)b);
      else k_op2<T, kOpCheb><<<grid, kThreads, 0, s>>>(x, f, xp, out, v, (T)a, (T)b);
      PR_CHECK_LAUNCH();
    }
    // vectors moved (reads + writes)
    if (mode == kOpRefine) {  // x (unless zero), b, xn, r in T; e, r32 in FP32
      bytes += (double)q.n * (sizeof(T) * (fu->xzero ? 3 : 4) + 8);
      return nparts;
    }
    const int vecs = mode == kOpApplyD ? 4 + (fu->xmode == 2 ? 2 : fu->xmode)
                                       : (mode == kOpApply || mode == kOpChebF ? 2 : (mode == kOpCheb && xp ? 4 : 3));
    bytes += (double)q.n * sizeof(T) * vecs;
    return nparts;
  }

  // throws if a TMA wait ran out since init()
  void check() {
    int h = 0;
    PR_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    c->sync();
    PR_REQUIRE(h == 0, PR_ERR_CUDA, "degree-2 operator: a TMA pipeline wait timed out");
  }

  // Chebyshev smoothing on level li.  From zero (pre-smoothing): x1 in x, x2 in y, x3 in x (on
  // levels with res >= 64 the first two steps are one fused pass from f, and the third recomputes
  // x1 from f).  From y0 held in y (post-smoothing): y1 in x, y2 in y, y3 in x.
  void chebyshev(int li, const T* f, T* x, T* y, bool from_zero) {
    const Level2<T>& q = lv[li];
    const double hi = kLamMax, lo = kLamMax / kLamRatio;
    const double th = 0.5 * (hi + lo), de = 0.5 * (hi - lo), sig = th / de;
    double ca[kChebSteps], cb[kChebSteps];
    double rho = 1.0 / sig;
    ca[0] = 0.0;
    cb[0] = 1.0 / th;
    for (int k = 1; k < kChebSteps; ++k) {
      const double rn = 1.0 / (2.0 * sig - rho);
      ca[k] = rn * rho;
      cb[k] = 2.0 * rn / de;
      rho = rn;
    }
    static_assert(kChebSteps == 3, "the fused pre-smoothing is written for three steps");
    if (from_zero && q.L >= kTmaMinLevel) {
      op(li, kOpChebF, f, nullptr, nullptr, y, ca[1], cb[1], 1, cb[0]);
      op(li, kOpChebPF, y, f, nullptr, x, ca[2], cb[2], 1, cb[0]);
      return;
    }
    if (from_zero) {
      k_cheb_first2<T><<<grid_for(q.n), kThreads, 0, c->stream>>>(f, x, q.view(), (T)cb[0]);
      PR_CHECK_LAUNCH();
      bytes += 2.0 * q.n * sizeof(T);
    } else {
      op(li, kOpCheb, y, f, nullptr, x, 0.0, cb[0]);
    }
    T* cur = x;
    T* prev = from_zero ? nullptr : y;
    for (int k = 1; k < kChebSteps; ++k) {
      T* dst = (cur == x) ? y : x;
      const bool last_fine = li == 0 && !from_zero && k == kChebSteps - 1 && rz_parts != nullptr;
      const int np = op(li, kOpCheb, cur, f, prev, dst, ca[k], cb[k], -1, 0.0, last_fine ? rz_parts : nullptr);
      if (last_fine) rz_np = np;
      prev = cur;
      cur = dst;
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
    launch_restrict<T>(s, q.y, q.L, qc.f, err);
    bytes += (double)(q.n + qc.n) * sizeof(T);
    vcycle(li + 1, qc.f, qc.x);
    launch_prolong<T>(s, X, qc.x, q.L, q.y, err);
    bytes += (double)(2 * q.n + qc.n) * sizeof(T);
    chebyshev(li, f, X, q.y, false);
  }
};

// preconditioned CG on the finest level from x = 0 to ||r|| <= tol_abs; r holds b on entry and is
// overwritten with the recursively updated residual; rr0 = r . r on entry when the caller knows it
// (else negative).  On the TMA operator (res >= 64) the vector
// updates ride on passes that read the vectors anyway: d = z + beta d, q = A d, d . q and
// x += alpha d (of the previous step) in the operator pass, r . z in the V-cycle's last smoothing
// step; r -= alpha q with r . r is its own pass, so that convergence is known before the next
// V-cycle.
template <typename T>
int pcg2(pr_context* c, System2<T>& sys, T* r, T* x, double tol_abs, int maxit, double rr0 = -1.0) {
  const uint64_t n = sys.lv[0].n;
  cudaStream_t s = c->stream;
  const std::string tn = tn2<T>();
  T* z = c->buf<T>("d2cg_z_" + tn, n);
  T* d = c->buf<T>("d2cg_d_" + tn, n);
  T* q = c->buf<T>("d2cg_q_" + tn, n);
  const bool fused = sys.fused_dots();
  // the fused path defines x in its second direction pass (x = alpha d); the other one adds to it
  if (!fused) PR_CUDA(cudaMemsetAsync(x, 0, n * sizeof(T), s));
  double rr = rr0;
  if (rr < 0.0) {
    rr = dot<T>(c, r, r, n);
    sys.bytes += 2.0 * n * sizeof(T);
  }
  if (!(std::sqrt(rr) > tol_abs)) {
    if (fused) PR_CUDA(cudaMemsetAsync(x, 0, n * sizeof(T), s));
    return 0;
  }
  int it = 0;
  if (!fused) {
    sys.vcycle(0, r, z);
    double rz = dot<T>(c, r, z, n);
    PR_CUDA(cudaMemcpyAsync(d, z, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
    sys.bytes += 4.0 * n * sizeof(T);
    while (it < maxit) {
      sys.op(0, kOpApply, d, nullptr, nullptr, q);
      sys.screen(d, q, +1);
      const double dq = dot<T>(c, d, q, n);
      sys.bytes += 2.0 * n * sizeof(T);
      if (!(dq > 0.0) || !(rz > 0.0)) break;
      const double alpha = rz / dq;
      rr = cg_update<T>(c, n, alpha, d, q, x, r);
      sys.bytes += 6.0 * n * sizeof(T);
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
  sys.alloc_parts();
  T* d2 = c->buf<T>("d2cg_d2_" + tn, n);
  T* dcur = d;
  T* dalt = d2;
  const T* dprev = nullptr;
  // z = M r, r . z
  auto precondition = [&]() {
    sys.rz_parts = sys.parts_a;
    sys.rz_np = 0;
    sys.vcycle(0, r, z);
    sys.rz_parts = nullptr;
    PR_REQUIRE(sys.rz_np > 0, PR_ERR_INTERNAL, "fused r.z was not produced");
    return sys.sum_parts(sys.rz_np, 0, 0.0);
  };
  double rz = precondition();
  double alpha = 0.0, alpha_prev = 0.0, beta = 0.0;
  bool pending = false;  // x += alpha dcur not applied yet
  bool x_def = false;    // x written (until then it is zero and never read)
  while (it < maxit) {
    // d = z + beta dprev (d = z at first), q = A d (+ screening), d . q, x += alpha_prev dprev
    typename System2<T>::Fuse fu;
    fu.out2 = dcur;
    fu.xacc = x;
    fu.s1 = dprev ? beta : 0.0;
    fu.s2 = dprev ? alpha_prev : 0.0;
    fu.xmode = dprev ? (x_def ? 2 : 1) : 0;
    const int na = sys.op(0, kOpApplyD, dprev ? dprev : z, z, nullptr, q, 0.0, 0.0, -1, 0.0, sys.parts_a, &fu);
    if (dprev) x_def = true;
    pending = false;
    const int nb = sys.screen(dcur, q, +1, sys.parts_b);
    const double dq = sys.sum_parts(na, nb, sys.scr.wh3);
    if (!(dq > 0.0) || !(rz > 0.0)) break;
    alpha = rz / dq;
    pending = true;
    ++it;
    rr = r_update<T>(c, n, alpha, q, r);
    sys.bytes += 3.0 * n * sizeof(T);
    if (!std::isfinite(rr) || std::sqrt(rr) <= tol_abs) break;
    const double rz_new = precondition();
    beta = rz_new / rz;
    rz = rz_new;
    alpha_prev = alpha;
    dprev = dcur;
    std::swap(dcur, dalt);
  }
  if (pending && x_def) {
    axpy<T, T>(s, n, alpha, dcur, x);
    sys.bytes += 3.0 * n * sizeof(T);
  } else if (pending) {
    scale_convert<T, T>(s, n, alpha, dcur, x);
    sys.bytes += 2.0 * n * sizeof(T);
  } else if (!x_def) {
    PR_CUDA(cudaMemsetAsync(x, 0, n * sizeof(T), s));
  }
  return it;
}

}  // namespace

namespace {
// b = h^2 sum_a (G_a M M) nf_a from the dense natural-order normal field (3 n)
__global__ void k_rhs_small(const double* __restrict__ nf, int L, RhsCoef k, double* __restrict__ b) {
  const int res = 1 << L;
  const uint64_t n = 1ull << (3 * L);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i & (res - 1)), y = (int)((i >> L) & (res - 1)), z = (int)(i >> (2 * L));
    double acc = 0.0;
    for (int dz = -2; dz <= 2; ++dz) {
      if (z + dz < 0 || z + dz >= res) continue;
      for (int dy = -2; dy <= 2; ++dy) {
        if (y + dy < 0 || y + dy >= res) continue;
        for (int dx = -2; dx <= 2; ++dx) {
          if (x + dx < 0 || x + dx >= res) continue;
          const uint64_t j = (uint64_t)(x + dx) + (uint64_t)res * ((uint64_t)(y + dy) + (uint64_t)res * (z + dz));
          acc += nf[j] * k.g[dx + 2] * k.m[dy + 2] * k.m[dz + 2] + nf[n + j] * k.m[dx + 2] * k.g[dy + 2] * k.m[dz + 2] +
                 nf[2 * n + j] * k.m[dx + 2] * k.m[dy + 2] * k.g[dz + 2];
        }
      }
    }
    b[i] = k.h2 * acc;
  }
}

// b = h^2 sum_a (G_a M M) nf_a from the compact normal field of the T touched nodes: zero, then
// the bricks within 2 nodes of a touched node (the 1-D integrals reach 2 nodes)
void deg2_rhs(pr_context* c, const double* nfc, uint64_t T, double* b, uint32_t D, double h) {
  cudaStream_t s = c->stream;
  RhsCoef k;
  for (int d = 0; d < 5; ++d) {
    k.g[d] = consts().g[d];
    k.m[d] = consts().m[d];
  }
  k.h2 = h * h;
  k.err = nullptr;
  const uint64_t n = 1ull << (3 * D);
  PR_CUDA(cudaMemsetAsync(b, 0, n * sizeof(double), s));
  if (T == 0) return;
  const uint32_t* run_key = c->get<uint32_t>("d2s_runkey");
  if (D < 3) {  // a grid smaller than one brick: the dense field
    double* nf = c->buf<double>("d2_nf_small", 3 * n);
    PR_CUDA(cudaMemsetAsync(nf, 0, 3 * n * sizeof(double), s));
    k_nf_scatter<<<grid_for(T), kThreads, 0, s>>>(run_key, T, nfc, n, nf);
    PR_CHECK_LAUNCH();
    k_rhs_small<<<grid_for(n), kThreads, 0, s>>>(nf, (int)D, k, b);
    PR_CHECK_LAUNCH();
    c->release("d2_nf_small");
    return;
  }
  const uint64_t nb = 1ull << (D - 3), nb3 = nb * nb * nb;
  uint8_t* flag = c->buf<uint8_t>("d2_rflag", nb3);
  uint32_t* list = c->buf<uint32_t>("d2_rlist", nb3);
  uint32_t* nsel = c->buf<uint32_t>("d2_rnsel", 1);
  PR_CUDA(cudaMemsetAsync(flag, 0, nb3, s));
  k_rhs_mark_bricks<<<grid_for(T, 1u << 20), kThreads, 0, s>>>(run_key, T, (int)D, flag);
  PR_CHECK_LAUNCH();
  thrust::counting_iterator<uint32_t> ids(0);
  size_t tb = 0;
  PR_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, ids, flag, list, nsel, (int64_t)nb3, s));
  void* tmp = c->buf<char>("cub_tmp", tb);
  PR_COUNT_PRIMITIVE();
  PR_CUDA(cub::DeviceSelect::Flagged(tmp, tb, ids, flag, list, nsel, (int64_t)nb3, s));
  uint32_t h_n = 0;
  PR_CUDA(cudaMemcpyAsync(&h_n, nsel, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  c->sync();
  if (h_n > 0) {
    allow_smem(k_rhs2_bricks, kRhsBrickSmem);
    const unsigned grid = (unsigned)std::min<uint64_t>(h_n, 148 * 16);
    k_rhs2_bricks<<<grid, kThreads, kRhsBrickSmem, s>>>(list, h_n, (int)D, run_key, T, nfc, k, b);
    PR_CHECK_LAUNCH();
  }
  c->release("d2_rflag");
  c->release("d2_rlist");
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
  k_pair_keys2<<<grid_for(m, 1u << 20), kThreads, 0, s>>>(upos, P, D, kin, vin, phi64, phi32, nin);
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
  // the normal field only at the touched nodes (it is zero elsewhere)
  double* nfc = c->buf<double>("d2_nfc", 3 * std::max<uint64_t>(T, 1));
  if (T > 0) {
    k_splat2c<<<grid_for(T, 1u << 20), kThreads, 0, s>>>(c->get<uint32_t>("d2s_runoff"), T, c->get<uint32_t>("d2s_val"),
                                                         phi64, unrm, P, nfc);
    PR_CHECK_LAUNCH();
  }
  const double h = 1.0 / (double)(1u << D);
  double* b = c->buf<double>("d2_b", n);
  deg2_rhs(c, nfc, T, b, D, h);
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
  solve_deg2(c, p, st, c->get<double>("d2_b"));
}

// A x = b with the degree-2 system of the context (b natural order, any right-hand side); the
// solution is left at c->d2_xnat (one of the solver's buffers)
void solve_deg2(pr_context* c, const pr_params& p, pr_stats& st, const double* b) {
  const uint32_t D = c->D;
  const uint64_t n = c->n;
  cudaStream_t s = c->stream;
  double* x = c->buf<double>("d2_x", n);
  double* r = c->buf<double>("d2_r", n);
  const double target = p.target_rel_residual > 0.0 ? p.target_rel_residual : 1e-6;
  const int max_iters = p.max_iters > 0 ? (int)p.max_iters : 200;
  const bool mixed = p.precision != PR_PRECISION_FP64;
  st.pcg_iterations = 0;
  st.refinement_steps = 0;
  System2<double> sys64;
  sys64.init(c, D, c->pw, !mixed);
  sys64.set_screen(c->get<double>("d2_phi64"));
  // ||b||: mixed, from the conversion of b that starts the FP32 solve; FP64, a dot product
  float* r32 = mixed ? c->buf<float>("d2_r32", n) : nullptr;
  const double bn = mixed ? convert_norm(c, b, r32, n) : std::sqrt(dot<double>(c, b, b, n));
  double bytes = mixed ? 12.0 * n : 8.0 * n;
  double rn = bn;
  int used = 0;
  bool x_zero = true;  // x = 0: the first correction is x itself (no zero fill, no x += e)
  if (bn > 0.0) {
    if (mixed) {
      System2<float> sys32;
      sys32.init(c, D, c->pw, true);
      sys32.set_screen(c->get<float>("d2_phi32"));
      float* e32 = c->buf<float>("d2_e32", n);
      const double inner = p.inner_rel_tol > 0.0 ? p.inner_rel_tol : 1e-4;
      // on the TMA operator the refinement step (x += e, r = b - A x, r32, ||r||) is one pass
      // into a second iterate buffer (the pass reads x with halos, so it cannot write x)
      const bool fused_refine = D >= (uint32_t)kTmaMinLevel;
      double* xn = fused_refine ? c->buf<double>("d2_x2", n) : nullptr;
      while (rn > target * bn && used < max_iters) {
        const double tol = std::max(inner, 0.5 * target * bn / rn);
        // r32 . r32 differs from rn^2 only by the FP32 rounding of r32: good enough for the entry test
        const int it = pcg2<float>(c, sys32, r32, e32, tol * rn, max_iters - used, rn * rn);
        used += it;
        double rn_new;
        if (fused_refine) {
          rn_new = sys64.refine(x, e32, b, xn, r, r32, x_zero);
          std::swap(x, xn);
        } else {
          if (x_zero) {
            scale_convert<float, double>(s, n, 1.0, e32, x);
            bytes += 12.0 * n;
          } else {
            axpy<float, double>(s, n, 1.0, e32, x);
            bytes += 20.0 * n;
          }
          sys64.op(0, kOpResid, x, b, nullptr, r);  // r = b - A x
          sys64.screen(x, r, -1);
          rn_new = convert_norm(c, r, r32, n);
          bytes += 12.0 * n;
        }
        x_zero = false;
        st.refinement_steps++;
        const bool stalled = it == 0 || !(rn_new < rn);
        rn = rn_new;
        if (stalled) break;
      }
      bytes += sys32.bytes;
      sys32.check();
    } else {
      double* e64 = c->buf<double>("d2_e64", n);
      PR_CUDA(cudaMemcpyAsync(r, b, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
      bytes += 16.0 * n;
      while (rn > target * bn && used < max_iters) {
        const int it = pcg2<double>(c, sys64, r, e64, 0.5 * target * bn, max_iters - used, rn * rn);
        used += it;
        if (x_zero) {
          std::swap(x, e64);  // x = 0 + e
        } else {
          axpy<double, double>(s, n, 1.0, e64, x);
          bytes += 24.0 * n;
        }
        x_zero = false;
        double rn_new;
        if (D >= (uint32_t)kTmaMinLevel) {  // the norm from the residual pass's partials
          rn_new = sys64.resid_norm(x, b, r);
        } else {
          sys64.op(0, kOpResid, x, b, nullptr, r);
          sys64.screen(x, r, -1);
          rn_new = std::sqrt(dot<double>(c, r, r, n));
          bytes += 8.0 * n;
        }
        st.refinement_steps++;
        const bool stalled = it == 0 || !(rn_new < rn);
        rn = rn_new;
        if (stalled) break;
      }
    }
  }
  if (x_zero) PR_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), s));
  bytes += sys64.bytes;
  sys64.check();
  st.pcg_iterations = (uint32_t)used;
  st.rel_residual = bn > 0.0 ? rn / bn : 0.0;
  st.converged = st.rel_residual <= target ? 1 : 0;
  st.solve_bytes = bytes;
  // the extraction reads the natural order; the Morton copy is made when an accessor asks for it
  c->d2_xnat = x;
  c->x64_ready = false;
  c->have_coeffs = true;
}

const double* coeffs_morton(pr_context* c) {
  if (c->degree == 2 && !c->x64_ready) {
    PR_REQUIRE(c->d2_xnat != nullptr, PR_ERR_INTERNAL, "degree-2 coefficients missing");
    double* xm = c->buf<double>("x64", c->n);
    nat_to_morton<double>(c->stream, c->d2_xnat, c->D, xm);
    c->x64_ready = true;
  }
  return c->get<double>("x64");
}

namespace {
template <typename T>
__global__ void k_fill2(T* __restrict__ v, uint64_t n, uint32_t seed) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t h = (uint32_t)i * 2654435761u ^ seed * 40503u;
    h ^= h >> 15;
    h *= 2246822519u;
    h ^= h >> 13;
    v[i] = (T)((double)(h & 0xffffff) / 8388608.0 - 1.0);
  }
}

template <typename T>
double bench2(pr_context* c, int kid, uint32_t D, int reps, double* bytes) {
  cudaStream_t s = c->stream;
  const uint64_t n = 1ull << (3 * D), nc = n / 8;
  const std::string tn = tn2<T>();
  T* x = c->buf<T>("kb2_x_" + tn, n);
  T* f = c->buf<T>("kb2_f_" + tn, n);
  T* p = c->buf<T>("kb2_p_" + tn, n);
  T* y = c->buf<T>("kb2_y_" + tn, n);
  T* ec = c->buf<T>("kb2_c_" + tn, nc);
  // the fused passes (ids 10, 11) need two more vectors, and the refinement two FP32 ones
  T* xa = (kid == 10 || kid == 11) ? c->buf<T>("kb2_a_" + tn, n) : nullptr;
  float* e32 = kid == 11 ? c->buf<float>("kb2_e32", n) : nullptr;
  float* r32 = kid == 11 ? c->buf<float>("kb2_r32", n) : nullptr;
  k_fill2<T><<<148 * 16, 256, 0, s>>>(x, n, 1u);
  k_fill2<T><<<148 * 16, 256, 0, s>>>(f, n, 2u);
  k_fill2<T><<<148 * 16, 256, 0, s>>>(p, n, 3u);
  k_fill2<T><<<148 * 16, 256, 0, s>>>(ec, nc, 4u);
  if (xa) k_fill2<T><<<148 * 16, 256, 0, s>>>(xa, n, 5u);
  if (e32) k_fill2<float><<<148 * 16, 256, 0, s>>>(e32, n, 6u);
  PR_CHECK_LAUNCH();
  System2<T> sys;
  sys.init(c, D, 4.0, false);
  const double nb = (double)n * sizeof(T);
  // 10: CG direction pass d = z + beta dold, q = A d, x += alpha dold (6 vectors); 11: FP64
  // refinement step xn = x + e, r = b - A xn, r32 (x, b, xn, r in T; e, r32 in FP32)
  const double algo[] = {4 * nb, 4 * nb, 2 * nb, 2 * nb, 3 * nb, nb + nb / 8, 2 * nb + nb / 8, 2 * nb, 2 * nb, 3 * nb,
                         6 * nb, 4 * nb + 8.0 * (double)n};
  PR_REQUIRE(kid >= 0 && kid < 12, PR_ERR_INVALID_ARGUMENT, "unknown kernel id");
  PR_REQUIRE(kid != 11 || sizeof(T) == 8, PR_ERR_INVALID_ARGUMENT, "the refinement step is FP64");
  PR_REQUIRE(D >= (uint32_t)kTmaMinLevel || (kid != 0 && kid != 2 && kid != 4 && kid < 8), PR_ERR_INVALID_ARGUMENT,
             "the TMA operator needs depth >= 6");
  *bytes = algo[kid];
  typename System2<T>::Fuse fu;
  if (kid == 10) {
    fu.out2 = p;
    fu.xacc = xa;
    fu.s1 = 0.3;
    fu.s2 = 0.2;
    fu.xmode = 2;
  } else if (kid == 11) {
    fu.out2 = xa;
    fu.e32 = e32;
    fu.r32 = r32;
  }
  const LevelView<T> v = sys.lv[0].view();
  auto run = [&]() {
    switch (kid) {
      case 0: sys.op(0, kOpCheb, x, f, p, y, 0.3, 0.5, 1); break;
      case 1: sys.op(0, kOpCheb, x, f, p, y, 0.3, 0.5, 0); break;
      case 2: sys.op(0, kOpApply, x, nullptr, nullptr, y, 0.0, 0.0, 1); break;
      case 3: sys.op(0, kOpApply, x, nullptr, nullptr, y, 0.0, 0.0, 0); break;
      case 4: sys.op(0, kOpResid, x, f, nullptr, y, 0.0, 0.0, 1); break;
      case 5:
        launch_restrict<T>(s, x, (int)D, ec, sys.err);
        break;
      case 6:
        launch_prolong<T>(s, x, ec, (int)D, y, sys.err);
        break;
      case 7:
        k_cheb_first2<T><<<grid_for(n), kThreads, 0, s>>>(f, y, v, (T)0.5);
        PR_CHECK_LAUNCH();
        break;
      case 8: sys.op(0, kOpChebF, f, nullptr, nullptr, y, 0.3, 0.5, 1, 0.6); break;
      case 9: sys.op(0, kOpChebPF, x, f, nullptr, y, 0.3, 0.5, 1, 0.6); break;
      case 10: sys.op(0, kOpApplyD, x, f, nullptr, y, 0.0, 0.0, 1, 0.0, nullptr, &fu); break;
      default: sys.op(0, kOpRefine, x, f, nullptr, y, 0.0, 0.0, 1, 0.0, nullptr, &fu); break;
    }
  };
  run();
  PR_CUDA(cudaStreamSynchronize(s));
  cudaEvent_t e0, e1;
  PR_CUDA(cudaEventCreate(&e0));
  PR_CUDA(cudaEventCreate(&e1));
  PR_CUDA(cudaEventRecord(e0, s));
  for (int r = 0; r < reps; ++r) run();
  PR_CUDA(cudaEventRecord(e1, s));
  PR_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  PR_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  sys.check();
  return (double)ms / reps;
}
}  // namespace

// Kernel bench of the degree-2 kernels on the finest level of depth D (synthetic vectors):
// 0 Chebyshev step (TMA), 1 Chebyshev step (register staging), 2 A x (TMA), 3 A x (register
// staging), 4 f - A x (TMA), 5 restriction, 6 prolongation + add, 7 first Chebyshev step,
// 8 the first two steps fused (from f), 9 the third step with x1 recomputed from f, 10 the fused
// CG direction pass, 11 the fused FP64 refinement step (FP64 only).
double deg2_kernel_bench(pr_context* c, int kid, uint32_t D, int precision, int reps, double* bytes) {
  if (reps < 1) reps = 1;
  return precision == PR_PRECISION_FP64 ? bench2<double>(c, kid, D, reps, bytes) : bench2<float>(c, kid, D, reps, bytes);
}

void deg2_constants(double* m5, double* s5, double* g5) {
  for (int d = 0; d < 5; ++d) {
    m5[d] = consts().m[d];
    s5[d] = consts().s[d];
    g5[d] = consts().g[d];
  }
}

// accessors in Morton order (the order of the degree-1 vectors and of the oracle)
void deg2_rhs_morton(pr_context* c, double* d_out) {
  nat_to_morton<double>(c->stream, c->get<double>("d2_b"), c->D, d_out);
  PR_CHECK_LAUNCH();
}
void deg2_normal_field_morton(pr_context* c, double* d_nf3, double* d_w) {
  // the dense field, scattered from the compact one for the accessor
  double* nf = c->buf<double>("d2_nf_acc", 3 * c->n);
  PR_CUDA(cudaMemsetAsync(nf, 0, 3 * c->n * sizeof(double), c->stream));
  if (c->T > 0) {
    k_nf_scatter<<<grid_for(c->T, 1u << 20), kThreads, 0, c->stream>>>(c->get<uint32_t>("d2s_runkey"), c->T,
                                                                        c->get<double>("d2_nfc"), c->n, nf);
    PR_CHECK_LAUNCH();
  }
  k_nat3_to_morton_aos<<<grid_for(c->n), kThreads, 0, c->stream>>>(nf, c->D, d_nf3);
  PR_CHECK_LAUNCH();
  c->release("d2_nf_acc");
  // the per-node weight sums, rebuilt here from the node-sorted pairs (the reconstruction does not
  // need them): the splat's own loop, so the values are the same
  cudaStream_t s = c->stream;
  double* w = c->buf<double>("d2_w", c->n);
  PR_CUDA(cudaMemsetAsync(w, 0, c->n * sizeof(double), s));
  if (c->T > 0) {
    k_splat2<<<grid_for(c->T, 1u << 20), kThreads, 0, s>>>(
        c->get<uint32_t>("d2s_runkey"), c->get<uint32_t>("d2s_runoff"), c->T, c->get<uint32_t>("d2s_val"),
        c->get<double>("d2_phi64"), c->get<double>("unrm"), c->P, c->n, nullptr, w);
    PR_CHECK_LAUNCH();
  }
  nat_to_morton<double>(s, w, c->D, d_w);
  c->release("d2_w");
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
  sys.check();
  nat_to_morton<T>(c->stream, yn, c->D, d_y);
  PR_CHECK_LAUNCH();
}
template void deg2_apply_morton<double>(pr_context*, const double*, double*);
template void deg2_apply_morton<float>(pr_context*, const float*, float*);

}  // namespace pr

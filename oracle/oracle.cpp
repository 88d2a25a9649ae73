// TEST INFRASTRUCTURE ONLY — the CPU oracle for parity checks and the CPU baseline.
//
// A C++ FP64 restatement of the reference crate's `reconstructor::reconstruct` path
// (Avanatiker/PoissonReconstruction, crate `poisson-recon`).  It follows the Rust
// sources operation by operation (no FMA contraction: build with -ffp-contract=off),
// so that a quantity computed here equals the crate's bit for bit wherever the crate's
// own order is deterministic.  Two places where the crate's order is NOT deterministic
// are restated with a fixed order instead:
//   * rayon `sum()` in dot/square_norm (src/solvers.rs:6-15) and in the iso average
//     (src/reconstructor.rs:56) — here a fixed-chunk pairwise order;
// Nothing here is part of the shipped library; only tests/, bench.py's CPU leg and
// the smoke check load it.
//
// Parity status: the crate cannot be built in this environment (no Rust toolchain),
// so this restatement is pinned by the crate's own unit tests (ported in
// tests/test_oracle.py) and by hand-derived known answers; the fem_tree path has no
// golden vectors in the reference.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PR_MC_TABLE_QUAL static const
#include "../poissonreconstruction_b200/csrc/mc_tri_table.inc"

namespace {

typedef int64_t isize;

// ---------------------------------------------------------------- casts (Rust `as`)
// f64 -> isize / u64 are saturating in Rust (NaN -> 0).
inline isize f64_to_isize(double v) {
  if (std::isnan(v)) return 0;
  if (v >= 9223372036854775807.0) return INT64_MAX;
  if (v <= -9223372036854775808.0) return INT64_MIN;
  return (isize)v;
}
inline uint64_t f64_to_u64(double v) {
  if (std::isnan(v) || v <= 0.0) return 0;
  if (v >= 18446744073709551615.0) return UINT64_MAX;
  return (uint64_t)v;
}

// ---------------------------------------------------------------- Morton index
// The crate's FEM index of a max-depth leaf is its position in the depth-first order
// of `SortedTreeNodes::collect_nodes` (src/octree.rs:235-248) with child i at offset
// (i&1, (i>>1)&1, (i>>2)&1) (src/octree.rs:145-153): the 3-D Morton code, x in bit 0.
// bit b of v moves to bit 3b (21-bit coordinates), by the usual shift-and-mask interleave
inline uint64_t spread3(uint64_t v) {
  v &= 0x1fffffull;
  v = (v | v << 32) & 0x1f00000000ffffull;
  v = (v | v << 16) & 0x1f0000ff0000ffull;
  v = (v | v << 8) & 0x100f00f00f00f00full;
  v = (v | v << 4) & 0x10c30c30c30c30c3ull;
  v = (v | v << 2) & 0x1249249249249249ull;
  return v;
}
// inverse of spread3: bit 3b of v moves to bit b
inline uint64_t compact3(uint64_t v) {
  v &= 0x1249249249249249ull;
  v = (v ^ (v >> 2)) & 0x10c30c30c30c30c3ull;
  v = (v ^ (v >> 4)) & 0x100f00f00f00f00full;
  v = (v ^ (v >> 8)) & 0x1f0000ff0000ffull;
  v = (v ^ (v >> 16)) & 0x1f00000000ffffull;
  v = (v ^ (v >> 32)) & 0x1fffffull;
  return v;
}
inline uint64_t morton(uint64_t x, uint64_t y, uint64_t z) {
  return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}
inline void unmorton(uint64_t m, uint64_t& x, uint64_t& y, uint64_t& z) {
  x = compact3(m);
  y = compact3(m >> 1);
  z = compact3(m >> 2);
}

// The Morton codes of the 27 neighbours of node m: per axis the interleaved bits of the
// coordinate minus one, itself and plus one (p[a][0..2]), and whether that coordinate lies in
// [0, res) (v[a][0..2]); neighbour (dx,dy,dz) = p[0][dx+1] | p[1][dy+1] | p[2][dz+1].  The
// masked increment carries through the gaps of the other axes' bits.
struct MortonNbrs {
  uint64_t p[3][3];
  bool v[3][3];
  uint64_t c[3];  // coordinates
  MortonNbrs(uint64_t m, uint64_t res) {
    const uint64_t X = 0x1249249249249249ull;
    for (int a = 0; a < 3; ++a) {
      const uint64_t mask = X << a, one = 1ull << a;
      const uint64_t part = m & mask;
      c[a] = compact3(m >> a);
      p[a][1] = part;
      p[a][0] = (part - one) & mask;
      p[a][2] = ((part | ~mask) + one) & mask;
      v[a][0] = c[a] > 0;
      v[a][1] = true;
      v[a][2] = c[a] + 1 < res;
    }
  }
};

// Visits the 2^D grid Morton-aligned block by block (blocks of B^3 nodes, B = min(8, res), each
// one contiguous range of the FEM index starting at blk * B^3).  For each block, `tile` holds the
// C components of src at the block's nodes and its H-node halo, in natural order (x fastest,
// row length T = B + 2H), zero outside the grid, and blockfn(blk, tile, T, B, loc, base) is
// called; loc[3l..3l+2] are the local coordinates of the block's l-th node (Morton order) and
// base[3] the block's first grid coordinates.  Gathering the halo once per block keeps the
// per-node work free of index arithmetic.
template <int C, int H, typename BlockFn>
void blocked_tiles(uint32_t D, const double* src, BlockFn&& blockfn) {
  const uint64_t res = 1ull << D;
  const int B = res < 8 ? (int)res : 8;
  const int T = B + 2 * H;
  const uint64_t nb = res / (uint64_t)B, bsz = (uint64_t)B * B * B;
  std::vector<uint64_t> sp(res);
  for (uint64_t g = 0; g < res; ++g) sp[g] = spread3(g);
  std::vector<int> loc(3 * bsz);
  for (uint64_t l = 0; l < bsz; ++l) {
    uint64_t a, b, c;
    unmorton(l, a, b, c);
    loc[3 * l] = (int)a;
    loc[3 * l + 1] = (int)b;
    loc[3 * l + 2] = (int)c;
  }
#pragma omp parallel
  {
    std::vector<double> tile((size_t)T * T * T * C);
#pragma omp for schedule(static)
    for (int64_t blk = 0; blk < (int64_t)(nb * nb * nb); ++blk) {
      uint64_t bx, by, bz;
      unmorton((uint64_t)blk, bx, by, bz);
      const int64_t base[3] = {(int64_t)bx * B, (int64_t)by * B, (int64_t)bz * B};
      for (int z = -H; z < B + H; ++z)
        for (int y = -H; y < B + H; ++y)
          for (int x = -H; x < B + H; ++x) {
            const int64_t gx = base[0] + x, gy = base[1] + y, gz = base[2] + z;
            double* t = &tile[(size_t)(((z + H) * T + (y + H)) * T + (x + H)) * C];
            if (gx < 0 || gy < 0 || gz < 0 || gx >= (int64_t)res || gy >= (int64_t)res || gz >= (int64_t)res) {
              for (int k = 0; k < C; ++k) t[k] = 0.0;
              continue;
            }
            const uint64_t j = sp[gx] | (sp[gy] << 1) | (sp[gz] << 2);
            for (int k = 0; k < C; ++k) t[k] = src[C * j + k];
          }
      blockfn((uint64_t)blk, tile.data(), T, B, loc.data(), base);
    }
  }
}

// blocked_tiles with a per-node callback: row(i, tile, o, T, g) for every node i of the block in
// index order, o its tile offset, g[3] its grid coordinates.
template <int C, int H = 1, typename Row>
void blocked_rows(uint32_t D, const double* src, Row&& row) {
  blocked_tiles<C, H>(D, src, [&](uint64_t blk, const double* tile, int T, int B, const int* loc,
                                  const int64_t* base) {
    const uint64_t bsz = (uint64_t)B * B * B;
    for (uint64_t l = 0; l < bsz; ++l) {
      const int* q = &loc[3 * l];
      const int64_t g[3] = {base[0] + q[0], base[1] + q[1], base[2] + q[2]};
      row(blk * bsz + l, tile, (size_t)((q[2] + H) * T + (q[1] + H)) * T + (q[0] + H), T, g);
    }
  });
}

// ---------------------------------------------------------------- 1-D constants
// src/fem_tree.rs:39-41
inline double mass_1d(isize d) { d = d < 0 ? -d : d; return d == 0 ? 2. / 3. : (d == 1 ? 1. / 6. : 0.0); }
inline double stiff_1d(isize d) { d = d < 0 ? -d : d; return d == 0 ? 2. : (d == 1 ? -1. : 0.0); }
inline double deriv_mass_1d(isize d) { return d == 0 ? 0. : (d == 1 ? -0.5 : (d == -1 ? 0.5 : 0.0)); }
// src/fem_tree.rs:44-48
inline double stiffness_entry(double h, isize dx, isize dy, isize dz) {
  return (stiff_1d(dx) * mass_1d(dy) * mass_1d(dz) + mass_1d(dx) * stiff_1d(dy) * mass_1d(dz) +
          mass_1d(dx) * mass_1d(dy) * stiff_1d(dz)) * h;
}
// src/fem_tree.rs:640-642
inline double bspline1(double t) {
  if (t < 0.0 || t > 2.0) return 0.0;
  if (t <= 1.0) return t;
  return 2.0 - t;
}
// src/fem_tree.rs:645-649
inline void contributing_offsets(double s, isize res, uint32_t& o0, uint32_t& o1) {
  isize f = f64_to_isize(std::floor(s));
  isize a = f - 1, b = f;
  a = a < 0 ? 0 : (a > res - 1 ? res - 1 : a);
  b = b < 0 ? 0 : (b > res - 1 ? res - 1 : b);
  o0 = (uint32_t)a;
  o1 = (uint32_t)b;
}

// deterministic sum (fixed chunking, independent of the thread count)
double det_dot(const double* a, const double* b, uint64_t n) {
  const uint64_t CH = 4096;
  uint64_t nch = (n + CH - 1) / CH;
  std::vector<double> part(nch, 0.0);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < (int64_t)nch; ++c) {
    uint64_t lo = (uint64_t)c * CH, hi = std::min(n, lo + CH);
    double s = 0.0;
    for (uint64_t i = lo; i < hi; ++i) s += a[i] * b[i];
    part[c] = s;
  }
  // pairwise combine
  while (part.size() > 1) {
    std::vector<double> nx((part.size() + 1) / 2);
    for (size_t i = 0; i < nx.size(); ++i)
      nx[i] = part[2 * i] + (2 * i + 1 < part.size() ? part[2 * i + 1] : 0.0);
    part.swap(nx);
  }
  return part.empty() ? 0.0 : part[0];
}

// ---------------------------------------------------------------- CSR (src/sparse.rs)
struct Csr {
  uint64_t rows = 0;
  std::vector<uint64_t> ptr;   // rows+1
  std::vector<uint32_t> col;
  std::vector<double> val;
  // src/sparse.rs:105-117 — row sum in entry order, starting at 0.0
  void spmv(const double* x, double* y) const {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)rows; ++i) {
      double s = 0.0;
      for (uint64_t k = ptr[i]; k < ptr[i + 1]; ++k) s = s + val[k] * x[col[k]];
      y[i] = s;
    }
  }
};

// src/solvers.rs:164-175
void gauss_seidel_sweep(const Csr& a, const double* b, double* x) {
  for (uint64_t i = 0; i < a.rows; ++i) {
    double diag = 0.0, sum = 0.0;
    for (uint64_t k = a.ptr[i]; k < a.ptr[i + 1]; ++k) {
      if (a.col[k] == i) diag = a.val[k];
      else sum += a.val[k] * x[a.col[k]];
    }
    if (diag != 0.0) x[i] = (b[i] - sum) / diag;
  }
}

// src/solvers.rs:20-69
uint64_t solve_cg(const Csr& a, const double* b, double* x, uint64_t max_iters, double accuracy) {
  uint64_t n = a.rows;
  std::vector<double> r(n), d(n), q(n);
  a.spmv(x, q.data());
  for (uint64_t i = 0; i < n; ++i) r[i] = b[i] - q[i];
  d = r;
  double delta_new = det_dot(r.data(), r.data(), n);
  double delta_0 = delta_new;
  if (delta_new == 0.0) return 0;
  for (uint64_t iter = 0; iter < max_iters; ++iter) {
    a.spmv(d.data(), q.data());
    double dq = det_dot(d.data(), q.data(), n);
    if (dq == 0.0) return iter + 1;
    double alpha = delta_new / dq;
    for (uint64_t i = 0; i < n; ++i) x[i] += alpha * d[i];
    if ((iter + 1) % 10 == 0) {
      a.spmv(x, q.data());
      for (uint64_t i = 0; i < n; ++i) r[i] = b[i] - q[i];
    } else {
      for (uint64_t i = 0; i < n; ++i) r[i] -= alpha * q[i];
    }
    double delta_old = delta_new;
    delta_new = det_dot(r.data(), r.data(), n);
    if (delta_new <= delta_0 * accuracy * accuracy) return iter + 1;
    double beta = delta_new / delta_old;
    if (std::isnan(beta) || std::isinf(beta)) break;
    for (uint64_t i = 0; i < n; ++i) d[i] = r[i] + beta * d[i];
  }
  return max_iters;
}

struct P6 { double x, y, z, nx, ny, nz; };

struct KeyHash {
  size_t operator()(const std::array<uint64_t, 3>& k) const {
    uint64_t h = k[0] * 0x9E3779B97F4A7C15ull;
    h ^= k[1] + 0x7F4A7C159E3779B9ull + (h << 6) + (h >> 2);
    h ^= k[2] + 0x94D049BB133111EBull + (h << 6) + (h >> 2);
    return (size_t)h;
  }
};


// Per-row accumulation in push order, then CSR sorted by column (src/fem_tree.rs:229-248).
struct RowBuilder {
  uint32_t D;
  uint64_t res, n;
  std::vector<double> slot;      // n * 27, slot index = (dz+1)*9+(dy+1)*3+(dx+1)
  std::vector<uint32_t> present; // n bitmasks
  RowBuilder(uint32_t depth, bool lexicographic) : D(depth) {
    res = 1ull << D;
    n = res * res * res;
    slot.assign(n * 27, 0.0);
    present.assign(n, 0u);
    lex = lexicographic;
  }
  bool lex;
  uint64_t index(uint64_t x, uint64_t y, uint64_t z) const {
    return lex ? (z * res + y) * res + x : morton(x, y, z);
  }
  void coords(uint64_t i, uint64_t& x, uint64_t& y, uint64_t& z) const {
    if (lex) { x = i % res; y = (i / res) % res; z = i / (res * res); }
    else unmorton(i, x, y, z);
  }
  void push(uint64_t i, isize dx, isize dy, isize dz, double v) {
    int s = (int)((dz + 1) * 9 + (dy + 1) * 3 + (dx + 1));
    slot[i * 27 + s] += v;
    present[i] |= 1u << s;
  }
  Csr finish() {
    Csr a;
    a.rows = n;
    a.ptr.assign(n + 1, 0);
    for (uint64_t i = 0; i < n; ++i) a.ptr[i + 1] = a.ptr[i] + __builtin_popcount(present[i]);
    a.col.resize(a.ptr[n]);
    a.val.resize(a.ptr[n]);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
      uint64_t x, y, z;
      coords(i, x, y, z);
      std::pair<uint64_t, double> e[27];
      int m = 0;
      for (int s = 0; s < 27; ++s) {
        if (!(present[i] >> s & 1u)) continue;
        isize dx = s % 3 - 1, dy = (s / 3) % 3 - 1, dz = s / 9 - 1;
        e[m++] = {index(x + dx, y + dy, z + dz), slot[(uint64_t)i * 27 + s]};
      }
      std::sort(e, e + m, [](const std::pair<uint64_t, double>& a1, const std::pair<uint64_t, double>& b1) {
        return a1.first < b1.first;
      });
      uint64_t p = a.ptr[i];
      for (int k = 0; k < m; ++k) { a.col[p + k] = (uint32_t)e[k].first; a.val[p + k] = e[k].second; }
    }
    std::vector<double>().swap(slot);
    return a;
  }
};

}  // namespace

// ======================================================================= C ABI
extern "C" {

struct orc_tree {
  uint32_t D;
  uint64_t res, n;
  double h;
  std::vector<P6> pts;          // unit-cube points
  std::vector<double> nf;       // 3n normal field (after normalisation)
  std::vector<double> nw;       // n node weights
  Csr A;
  bool have_A = false;
  double pw_A = -1.0;
};

struct orc_mesh {
  double* verts;   // 3*nv
  uint64_t nv;
  uint64_t* tris;  // 3*nt
  uint64_t nt;
};

struct orc_params {
  uint32_t depth;
  double scale;
  double cg_accuracy;
  uint64_t cg_iters;
  double point_weight;
  int32_t solve_mode;        // 0 = reference schedule, 1 = converged
  double target_rel_residual;
  uint64_t max_iters;
};

struct orc_stats {
  double iso_value;
  uint64_t fem_nodes, mesh_vertices, mesh_triangles;
  double rel_residual;
  uint64_t iterations;
  double time_tree, time_solve, time_extract, time_total;
};

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

double orc_bspline1(double t) { return bspline1(t); }
double orc_stiffness_entry(double h, int dx, int dy, int dz) { return stiffness_entry(h, dx, dy, dz); }
uint64_t orc_morton(uint64_t x, uint64_t y, uint64_t z) { return morton(x, y, z); }

// Mesh edge mask of a marching-cubes case: edge e (corners a,b of src/fem_tree.rs:585)
// is cut iff the two corners classify differently.  Equals the crate's EDGE_TABLE.
uint32_t orc_mc_edge_mask(uint32_t mc) {
  static const int ev[12][2] = {{0,1},{1,2},{2,3},{3,0},{4,5},{5,6},{6,7},{7,4},{0,4},{1,5},{2,6},{3,7}};
  uint32_t m = 0;
  for (int e = 0; e < 12; ++e)
    if (((mc >> ev[e][0]) & 1u) != ((mc >> ev[e][1]) & 1u)) m |= 1u << e;
  return m;
}
// Triangle table row as edge indices (-1 terminated, 16 entries)
void orc_mc_tri_row(uint32_t mc, int* out16) {
  for (int i = 0; i < 16; ++i) out16[i] = -1;
  for (int i = 0; i < 3 * PR_MC_NTRI[mc]; ++i) out16[i] = (int)((PR_MC_TRIS[mc] >> (4 * i)) & 15ull);
}

// ---------------------------------------------------------------- geometry
// BBox::extend (src/geometry.rs:356-363): f64::min/max ignore NaN like fmin/fmax.
void orc_bbox(const double* pts6, uint64_t n, double* bmin, double* bmax) {
  for (int k = 0; k < 3; ++k) { bmin[k] = INFINITY; bmax[k] = -INFINITY; }
  for (uint64_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      bmin[k] = std::fmin(bmin[k], pts6[6 * i + k]);
      bmax[k] = std::fmax(bmax[k], pts6[6 * i + k]);
    }
}

// unit_cube_transform (src/geometry.rs:384-402). m is column-major: m[col*4+row].
void orc_unit_cube_transform(const double* bmin, const double* bmax, double scale, double* m) {
  double c[3], s3[3];
  for (int k = 0; k < 3; ++k) { c[k] = (bmin[k] + bmax[k]) * 0.5; s3[k] = bmax[k] - bmin[k]; }
  double max_dim = std::fmax(std::fmax(s3[0], s3[1]), s3[2]);
  double s = max_dim > 0.0 ? scale / max_dim : 1.0;
  for (int i = 0; i < 16; ++i) m[i] = 0.0;
  m[0] = s; m[5] = s; m[10] = s;
  m[12] = -s * c[0] + 0.5; m[13] = -s * c[1] + 0.5; m[14] = -s * c[2] + 0.5; m[15] = 1.0;
}

// Mat4::inverse (src/geometry.rs:274-317)
void orc_mat4_inverse(const double* M, double* out) {
#define MM(col, row) M[(col) * 4 + (row)]
  double a = MM(0,0), b = MM(1,0), c = MM(2,0);
  double d = MM(0,1), e = MM(1,1), f = MM(2,1);
  double g = MM(0,2), h = MM(1,2), i = MM(2,2);
  double det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
  for (int k = 0; k < 16; ++k) out[k] = 0.0;
  if (std::fabs(det) < 1e-30) { out[0] = out[5] = out[10] = out[15] = 1.0; return; }
  double inv_det = 1.0 / det;
  double a_inv = (e * i - f * h) * inv_det, b_inv = (c * h - b * i) * inv_det, c_inv = (b * f - c * e) * inv_det;
  double d_inv = (f * g - d * i) * inv_det, e_inv = (a * i - c * g) * inv_det, f_inv = (c * d - a * f) * inv_det;
  double g_inv = (d * h - e * g) * inv_det, h_inv = (b * g - a * h) * inv_det, i_inv = (a * e - b * d) * inv_det;
  double tx = MM(3,0), ty = MM(3,1), tz = MM(3,2);
  double itx = -(a_inv * tx + b_inv * ty + c_inv * tz);
  double ity = -(d_inv * tx + e_inv * ty + f_inv * tz);
  double itz = -(g_inv * tx + h_inv * ty + i_inv * tz);
  double cols[4][4] = {{a_inv, d_inv, g_inv, 0.0}, {b_inv, e_inv, h_inv, 0.0}, {c_inv, f_inv, i_inv, 0.0}, {itx, ity, itz, 1.0}};
  for (int cc = 0; cc < 4; ++cc) for (int r = 0; r < 4; ++r) out[cc * 4 + r] = cols[cc][r];
#undef MM
}

// Mat4::transform_point / transform_vector (src/geometry.rs:256-270), Vec3::normalize (:49-56)
void orc_transform_point(const double* M, const double* p, double* out) {
  for (int r = 0; r < 3; ++r) out[r] = M[0 * 4 + r] * p[0] + M[1 * 4 + r] * p[1] + M[2 * 4 + r] * p[2] + M[3 * 4 + r];
}
void orc_transform_points(const double* M, const double* pts6, uint64_t n, double* unit6) {
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < (int64_t)n; ++k) {
    const double* p = pts6 + 6 * k;
    double* o = unit6 + 6 * k;
    for (int r = 0; r < 3; ++r) o[r] = M[0 * 4 + r] * p[0] + M[1 * 4 + r] * p[1] + M[2 * 4 + r] * p[2] + M[3 * 4 + r];
    double v[3];
    for (int r = 0; r < 3; ++r) v[r] = M[0 * 4 + r] * p[3] + M[1 * 4 + r] * p[4] + M[2 * 4 + r] * p[5];
    double nn = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (nn > 0.0) { o[3] = v[0] / nn; o[4] = v[1] / nn; o[5] = v[2] / nn; }
    else { o[3] = 0.0; o[4] = 0.0; o[5] = 0.0; }
  }
}

// ---------------------------------------------------------------- tree
// FEMTree::{initialize, finalize, splat_normal_field} (src/fem_tree.rs:83-178).
orc_tree* orc_tree_new(uint32_t depth, const double* unit6, uint64_t npts) {
  orc_tree* t = new orc_tree();
  t->D = depth;
  t->res = 1ull << depth;
  t->n = t->res * t->res * t->res;
  t->h = 1.0 / (double)t->res;
  t->pts.resize(npts);
  std::memcpy(t->pts.data(), unit6, npts * sizeof(P6));
  t->nf.assign(3 * t->n, 0.0);
  t->nw.assign(t->n, 0.0);
  const double h = t->h;
  const uint64_t res = t->res;
  for (const P6& pt : t->pts) {
    isize cx = f64_to_isize(std::floor(pt.x / h));
    isize cy = f64_to_isize(std::floor(pt.y / h));
    isize cz = f64_to_isize(std::floor(pt.z / h));
    double tx = pt.x / h - (double)cx, ty = pt.y / h - (double)cy, tz = pt.z / h - (double)cz;
    double bx0 = 1.0 - tx, bx1 = tx, by0 = 1.0 - ty, by1 = ty, bz0 = 1.0 - tz, bz1 = tz;
    for (isize dz = 0; dz <= 1; ++dz)
      for (isize dy = 0; dy <= 1; ++dy)
        for (isize dx = 0; dx <= 1; ++dx) {
          uint64_t ox = (uint64_t)(cx + dx), oy = (uint64_t)(cy + dy), oz = (uint64_t)(cz + dz);
          if (ox >= res || oy >= res || oz >= res) continue;
          uint64_t idx = morton(ox, oy, oz);
          double bx = dx == 0 ? bx0 : bx1, by = dy == 0 ? by0 : by1, bz = dz == 0 ? bz0 : bz1;
          double w = bx * by * bz;
          t->nf[3 * idx + 0] += pt.nx * w;
          t->nf[3 * idx + 1] += pt.ny * w;
          t->nf[3 * idx + 2] += pt.nz * w;
          t->nw[idx] += w;
        }
  }
  for (uint64_t i = 0; i < t->n; ++i) {
    if (t->nw[i] > 0.0) {
      double inv = 1.0 / t->nw[i];
      t->nf[3 * i + 0] = -t->nf[3 * i + 0] * inv;
      t->nf[3 * i + 1] = -t->nf[3 * i + 1] * inv;
      t->nf[3 * i + 2] = -t->nf[3 * i + 2] * inv;
    }
  }
  return t;
}

void orc_tree_free(orc_tree* t) { delete t; }
uint64_t orc_tree_nodes(const orc_tree* t) { return t->n; }

void orc_tree_normal_field(const orc_tree* t, double* nf3, double* w) {
  std::memcpy(nf3, t->nf.data(), 3 * t->n * sizeof(double));
  std::memcpy(w, t->nw.data(), t->n * sizeof(double));
}

// trunc-cell basis of one point, as in assemble_system / assemble_rhs (src/fem_tree.rs:207-219, :283-295)
static int screening_basis(const orc_tree* t, const P6& pt, uint64_t* idx, double* bx_, double* by_, double* bz_,
                           int* cdx = nullptr, int* cdy = nullptr, int* cdz = nullptr) {
  const double h = t->h;
  isize cx = f64_to_isize(pt.x / h), cy = f64_to_isize(pt.y / h), cz = f64_to_isize(pt.z / h);
  double tx = pt.x / h - (double)cx, ty = pt.y / h - (double)cy, tz = pt.z / h - (double)cz;
  double bx0 = 1. - tx, bx1 = tx, by0 = 1. - ty, by1 = ty, bz0 = 1. - tz, bz1 = tz;
  int m = 0;
  for (isize dz = 0; dz <= 1; ++dz)
    for (isize dy = 0; dy <= 1; ++dy)
      for (isize dx = 0; dx <= 1; ++dx) {
        uint32_t ox = (uint32_t)(uint64_t)(cx + dx), oy = (uint32_t)(uint64_t)(cy + dy), oz = (uint32_t)(uint64_t)(cz + dz);
        if (ox >= (uint32_t)t->res || oy >= (uint32_t)t->res || oz >= (uint32_t)t->res) continue;
        idx[m] = morton(ox, oy, oz);
        bx_[m] = dx == 0 ? bx0 : bx1;
        by_[m] = dy == 0 ? by0 : by1;
        bz_[m] = dz == 0 ? bz0 : bz1;
        if (cdx) { cdx[m] = (int)dx; cdy[m] = (int)dy; cdz[m] = (int)dz; }
        ++m;
      }
  return m;
}

// FEMTree::assemble_rhs (src/fem_tree.rs:251-299)
void orc_tree_rhs(const orc_tree* t, double pw, double* rhs) {
  const isize res = (isize)t->res;
  const double h = t->h;
  blocked_rows<3>(t->D, t->nf.data(), [&](uint64_t i, const double* tile, size_t o, int T, const int64_t* g) {
    double sum = 0.0;
    for (isize dx = -1; dx <= 1; ++dx)
      for (isize dy = -1; dy <= 1; ++dy)
        for (isize dz = -1; dz <= 1; ++dz) {
          isize jx = g[0] + dx, jy = g[1] + dy, jz = g[2] + dz;
          if (jx < 0 || jx >= res || jy < 0 || jy >= res || jz < 0 || jz >= res) continue;
          const double* v = &tile[3 * (o + (dz * T + dy) * T + dx)];
          sum += h * h * (v[0] * deriv_mass_1d(dx) * mass_1d(dy) * mass_1d(dz) +
                          v[1] * mass_1d(dx) * deriv_mass_1d(dy) * mass_1d(dz) +
                          v[2] * mass_1d(dx) * mass_1d(dy) * deriv_mass_1d(dz));
        }
    rhs[i] = sum;
  });
  if (pw > 0.0) {
    double wh3 = pw * (h * h * h) / 1.5;
    double target = 0.5;
    for (const P6& pt : t->pts) {
      uint64_t idx[8];
      double bx[8], by[8], bz[8];
      int m = screening_basis(t, pt, idx, bx, by, bz);
      for (int k = 0; k < m; ++k) rhs[idx[k]] += wh3 * target * bx[k] * by[k] * bz[k];
    }
  }
}

// FEMTree::assemble_system (src/fem_tree.rs:180-249); returns nnz
int64_t orc_tree_assemble(orc_tree* t, double pw) {
  const uint64_t res = t->res;
  const double h = t->h;
  RowBuilder rb(t->D, false);
  for (uint64_t i = 0; i < t->n; ++i) {
    uint64_t ix, iy, iz;
    unmorton(i, ix, iy, iz);
    for (isize dx = -1; dx <= 1; ++dx)
      for (isize dy = -1; dy <= 1; ++dy)
        for (isize dz = -1; dz <= 1; ++dz) {
          isize jx = (isize)ix + dx, jy = (isize)iy + dy, jz = (isize)iz + dz;
          if (jx < 0 || jx >= (isize)res || jy < 0 || jy >= (isize)res || jz < 0 || jz >= (isize)res) continue;
          double val = stiffness_entry(h, dx, dy, dz);
          if (val != 0.0) rb.push(i, dx, dy, dz, val);
        }
  }
  if (pw > 0.0) {
    double wh3 = pw * (h * h * h) / 1.5;
    double wg = wh3 * 0.005;
    for (uint64_t i = 0; i < t->n; ++i) rb.push(i, 0, 0, 0, wg);
    for (const P6& pt : t->pts) {
      uint64_t idx[8];
      double bx[8], by[8], bz[8];
      int cdx[8], cdy[8], cdz[8];
      int m = screening_basis(t, pt, idx, bx, by, bz, cdx, cdy, cdz);
      double phi[8];
      for (int k = 0; k < m; ++k) phi[k] = bx[k] * by[k] * bz[k];
      for (int a = 0; a < m; ++a)
        for (int b = 0; b < m; ++b)
          rb.push(idx[a], (isize)cdx[b] - (isize)cdx[a], (isize)cdy[b] - (isize)cdy[a], (isize)cdz[b] - (isize)cdz[a],
                  wh3 * phi[a] * phi[b]);
    }
  }
  t->A = rb.finish();
  t->have_A = true;
  t->pw_A = pw;
  return (int64_t)t->A.ptr[t->n];
}

void orc_tree_csr(const orc_tree* t, uint64_t* ptr, uint32_t* col, double* val) {
  std::memcpy(ptr, t->A.ptr.data(), (t->n + 1) * sizeof(uint64_t));
  std::memcpy(col, t->A.col.data(), t->A.col.size() * sizeof(uint32_t));
  std::memcpy(val, t->A.val.data(), t->A.val.size() * sizeof(double));
}

int orc_tree_spmv(const orc_tree* t, const double* x, double* y) {
  if (!t->have_A) return -1;
  t->A.spmv(x, y);
  return 0;
}

// FEMTree::build_system_at_depth (src/fem_tree.rs:346-404), lexicographic coarse index.
static void build_system_at_depth(const orc_tree* t, uint32_t depth, double pw, Csr& A, std::vector<double>& rhs) {
  const uint64_t res = 1ull << depth;
  const double h = 1.0 / (double)res;
  const uint64_t n = res * res * res;
  double scale_factor = (double)(1ull << (2 * (t->D - depth)));
  double effective_pw = pw * scale_factor;
  RowBuilder rb(depth, true);
  for (uint64_t z = 0; z < res; ++z)
    for (uint64_t y = 0; y < res; ++y)
      for (uint64_t x = 0; x < res; ++x) {
        uint64_t i = (z * res + y) * res + x;
        for (isize dz = -1; dz <= 1; ++dz)
          for (isize dy = -1; dy <= 1; ++dy)
            for (isize dx = -1; dx <= 1; ++dx) {
              isize jx = (isize)x + dx, jy = (isize)y + dy, jz = (isize)z + dz;
              if (jx < 0 || jx >= (isize)res || jy < 0 || jy >= (isize)res || jz < 0 || jz >= (isize)res) continue;
              double v = stiffness_entry(h, dx, dy, dz);
              if (v != 0.0) rb.push(i, dx, dy, dz, v);
            }
        if (effective_pw > 0.0) {
          double wh3 = effective_pw * (h * h * h) / 1.5;
          rb.push(i, 0, 0, 0, wh3 * 1.005);
        }
      }
  A = rb.finish();
  rhs.assign(n, 0.0);
  for (uint64_t i = 0; i < t->n; ++i) {
    uint64_t fx, fy, fz;
    unmorton(i, fx, fy, fz);
    uint64_t cx = fx >> (t->D - depth), cy = fy >> (t->D - depth), cz = fz >> (t->D - depth);
    uint64_t ci = (cz * res + cy) * res + cx;
    if (ci < n) rhs[ci] += t->nf[3 * i] + t->nf[3 * i + 1] + t->nf[3 * i + 2];
  }
  if (effective_pw > 0.0) {
    double wh3 = effective_pw * (h * h * h) / 1.5;
    for (uint64_t i = 0; i < n; ++i) rhs[i] += wh3 * 0.5;
  }
}

// FEMTree::prolongate (src/fem_tree.rs:310-343): one-level stencil, whatever the gap.
static void prolongate(const orc_tree* t, const std::vector<double>& coarse, uint32_t coarse_depth, std::vector<double>& fine) {
  const isize fine_res = (isize)t->res;
  const uint64_t cres = 1ull << coarse_depth;
  fine.assign(t->n, 0.0);
  const double bw[3] = {0.5, 1.0, 0.5};
  for (uint64_t cz = 0; cz < cres; ++cz)
    for (uint64_t cy = 0; cy < cres; ++cy)
      for (uint64_t cx = 0; cx < cres; ++cx) {
        uint64_t ci = (cz * cres + cy) * cres + cx;
        if (ci >= coarse.size()) continue;
        double v = coarse[ci];
        if (v == 0.0) continue;
        for (isize dz = 0; dz <= 2; ++dz) {
          isize fz = (isize)cz * 2 + dz - 1;
          if (fz < 0 || fz >= fine_res) continue;
          for (isize dy = 0; dy <= 2; ++dy) {
            isize fy = (isize)cy * 2 + dy - 1;
            if (fy < 0 || fy >= fine_res) continue;
            for (isize dx = 0; dx <= 2; ++dx) {
              isize fx = (isize)cx * 2 + dx - 1;
              if (fx < 0 || fx >= fine_res) continue;
              double w = bw[dx] * bw[dy] * bw[dz];
              fine[morton(fx, fy, fz)] += v * w;
            }
          }
        }
      }
}

// FEMTree::solve_cascadic (src/fem_tree.rs:458-487) with gs = 20 and base depth D-2
// (src/reconstructor.rs:51-52).  x receives the fine solution.  info[0] = coarse CG
// iterations, info[1] = fine CG iterations.
int orc_tree_solve_reference(orc_tree* t, double pw, uint64_t cg_iters, double eps, double* x, uint64_t* info) {
  const uint64_t gs = 20;
  if (!t->have_A || t->pw_A != pw) orc_tree_assemble(t, pw);
  std::vector<double> b(t->n);
  orc_tree_rhs(t, pw, b.data());
  uint32_t base_depth = t->D > 2 ? t->D - 2 : 0;
  if (base_depth >= t->D) {
    std::fill(x, x + t->n, 0.0);
    for (uint64_t k = 0; k < gs; ++k) gauss_seidel_sweep(t->A, b.data(), x);
    uint64_t it = solve_cg(t->A, b.data(), x, cg_iters, eps);
    if (info) { info[0] = 0; info[1] = it; }
    return 0;
  }
  Csr B;
  std::vector<double> brhs;
  build_system_at_depth(t, base_depth, pw, B, brhs);
  std::vector<double> csol(brhs.size(), 0.0);
  for (uint64_t k = 0; k < gs; ++k) gauss_seidel_sweep(B, brhs.data(), csol.data());
  uint64_t itc = solve_cg(B, brhs.data(), csol.data(), cg_iters, eps);
  std::vector<double> init;
  prolongate(t, csol, base_depth, init);
  std::memcpy(x, init.data(), t->n * sizeof(double));
  for (uint64_t k = 0; k < gs; ++k) gauss_seidel_sweep(t->A, b.data(), x);
  uint64_t itf = solve_cg(t->A, b.data(), x, cg_iters / 4, eps);
  if (info) { info[0] = itc; info[1] = itf; }
  return 0;
}

// Stage outputs of the reference schedule for diagnostics: coarse system RHS (lexicographic)
// and the prolongated initial guess.
int orc_tree_coarse_rhs(const orc_tree* t, double pw, double* brhs_out) {
  uint32_t base_depth = t->D > 2 ? t->D - 2 : 0;
  if (base_depth >= t->D) return -1;
  Csr B;
  std::vector<double> brhs;
  build_system_at_depth(t, base_depth, pw, B, brhs);
  std::memcpy(brhs_out, brhs.data(), brhs.size() * sizeof(double));
  return 0;
}
int orc_tree_prolongate(const orc_tree* t, const double* coarse_lex, uint32_t coarse_depth, double* fine_out) {
  std::vector<double> c(coarse_lex, coarse_lex + (1ull << (3 * coarse_depth)));
  std::vector<double> f;
  prolongate(t, c, coarse_depth, f);
  std::memcpy(fine_out, f.data(), t->n * sizeof(double));
  return 0;
}

// Converged solve of the same fine system: CG (the crate's loop, without its early exit)
// until ||b - A x|| <= tol ||b||, x holds the initial guess on entry.
uint64_t orc_tree_solve_converged(orc_tree* t, double pw, double tol, uint64_t maxit, double* x, double* relres) {
  if (!t->have_A || t->pw_A != pw) orc_tree_assemble(t, pw);
  const uint64_t n = t->n;
  std::vector<double> b(n), r(n), d(n), q(n);
  orc_tree_rhs(t, pw, b.data());
  double bb = det_dot(b.data(), b.data(), n);
  t->A.spmv(x, q.data());
  for (uint64_t i = 0; i < n; ++i) r[i] = b[i] - q[i];
  d = r;
  double rr = det_dot(r.data(), r.data(), n);
  uint64_t it = 0;
  if (bb == 0.0) { if (relres) *relres = 0.0; return 0; }
  while (it < maxit && rr > tol * tol * bb) {
    t->A.spmv(d.data(), q.data());
    double dq = det_dot(d.data(), q.data(), n);
    if (dq == 0.0) break;
    double alpha = rr / dq;
    for (uint64_t i = 0; i < n; ++i) x[i] += alpha * d[i];
    ++it;
    if (it % 50 == 0) {
      t->A.spmv(x, q.data());
      for (uint64_t i = 0; i < n; ++i) r[i] = b[i] - q[i];
    } else {
      for (uint64_t i = 0; i < n; ++i) r[i] -= alpha * q[i];
    }
    double rr_new = det_dot(r.data(), r.data(), n);
    double beta = rr_new / rr;
    rr = rr_new;
    for (uint64_t i = 0; i < n; ++i) d[i] = r[i] + beta * d[i];
  }
  t->A.spmv(x, q.data());
  for (uint64_t i = 0; i < n; ++i) r[i] = b[i] - q[i];
  if (relres) *relres = std::sqrt(det_dot(r.data(), r.data(), n) / bb);
  return it;
}

// ---------------------------------------------------------------- matrix-free fine operator
// The crate's CSR (src/fem_tree.rs:180-249) needs about 1 TB of host memory at depth 10, so
// the large-depth checks use the same entries computed on the fly.  Row i of A x:
//   stiffness_entry(h, d) x_{i+d} over the 27 neighbours inside the grid (zero entries skipped,
//   src/fem_tree.rs:187-193), then + wg x_i (src/fem_tree.rs:195-200), then the screening rows
//   sum_p wh3 phi_a(p) phi_b(p) x_b of the points whose trunc cell touches node i
//   (src/fem_tree.rs:201-228).
// The CSR product sums a row's entries in column order; here they are grouped by kind, so the
// two agree to rounding (tests/test_oracle.py compares them).
void orc_tree_apply_mf(const orc_tree* t, double pw, const double* x, double* y) {
  const uint64_t n = t->n;
  const isize res = (isize)t->res;
  const double h = t->h;
  const double wh3 = pw > 0.0 ? pw * (h * h * h) / 1.5 : 0.0;
  const double wg = wh3 * 0.005;
  (void)n;
  (void)res;
  // the nonzero entries (21 of 27), in the neighbour order dz, dy, dx
  double st[27];
  int off[27], nz = 0;
  const int T = t->res < 8 ? (int)t->res + 2 : 10;
  for (int k = 0; k < 27; ++k) {
    const double v = stiffness_entry(h, k % 3 - 1, (k / 3) % 3 - 1, k / 9 - 1);
    if (v == 0.0) continue;
    st[nz] = v;
    off[nz++] = ((k / 9 - 1) * T + ((k / 3) % 3 - 1)) * T + (k % 3 - 1);
  }
  // entries to neighbours outside the grid are omitted: their tile values are zero
  blocked_rows<1>(t->D, x, [&](uint64_t i, const double* tile, size_t o, int, const int64_t*) {
    const double* c = tile + o;
    double s = 0.0;
    for (int k = 0; k < nz; ++k) s += st[k] * c[off[k]];
    y[i] = pw > 0.0 ? s + wg * c[0] : s;
  });
  if (pw > 0.0) {
    const uint64_t np = t->pts.size();
    std::vector<double> proj(np);
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < (int64_t)np; ++p) {
      uint64_t idx[8];
      double bx[8], by[8], bz[8];
      const int m = screening_basis(t, t->pts[p], idx, bx, by, bz);
      double v = 0.0;
      for (int k = 0; k < m; ++k) v += bx[k] * by[k] * bz[k] * x[idx[k]];
      proj[p] = v;
    }
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < (int64_t)np; ++p) {
      uint64_t idx[8];
      double bx[8], by[8], bz[8];
      const int m = screening_basis(t, t->pts[p], idx, bx, by, bz);
      for (int k = 0; k < m; ++k) {
        const double v = wh3 * (bx[k] * by[k] * bz[k]) * proj[p];
#pragma omp atomic
        y[idx[k]] += v;
      }
    }
  }
}

// Frees the normal field and node weights (the right-hand side no longer needs them): at
// depth 10 they hold 34 GB that the matrix-free solves below do not use.
void orc_tree_release_field(orc_tree* t) {
  std::vector<double>().swap(t->nf);
  std::vector<double>().swap(t->nw);
}

}  // extern "C"
namespace {
void par_copy(double* dst, const double* src, uint64_t n) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i) dst[i] = src[i];
}
// r = b - q
void par_sub(double* r, const double* b, const double* q, uint64_t n) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i) r[i] = b[i] - q[i];
}
// x += a d
void par_axpy(double* x, double a, const double* d, uint64_t n) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i) x[i] += a * d[i];
}
// d = r + beta d
void par_xpby(double* d, const double* r, double beta, uint64_t n) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i) d[i] = r[i] + beta * d[i];
}
}  // namespace
extern "C" {

// solve_cg (src/solvers.rs:20-69) on the fine system with the matrix-free operator and the
// caller's right-hand side b: from x (initial guess on entry), at most max_iters iterations,
// the residual recomputed as b - A x every 10th iteration, stop when ||r||^2 <= ||r0||^2 acc^2.
// delta (may be NULL) receives ||r||^2 before the first iteration and after each one
// (max_iters + 1 slots; unused slots are left as they were).  Returns the iteration count as
// the crate does.
uint64_t orc_tree_cg_mf(const orc_tree* t, double pw, const double* b, double* x, uint64_t max_iters, double accuracy,
                        double* delta) {
  const uint64_t n = t->n;
  std::vector<double> r(n), d(n), q(n);
  orc_tree_apply_mf(t, pw, x, q.data());
  par_sub(r.data(), b, q.data(), n);
  par_copy(d.data(), r.data(), n);
  double delta_new = det_dot(r.data(), r.data(), n);
  const double delta_0 = delta_new;
  if (delta) delta[0] = delta_new;
  if (delta_new == 0.0) return 0;
  for (uint64_t iter = 0; iter < max_iters; ++iter) {
    orc_tree_apply_mf(t, pw, d.data(), q.data());
    const double dq = det_dot(d.data(), q.data(), n);
    if (dq == 0.0) return iter + 1;
    const double alpha = delta_new / dq;
    par_axpy(x, alpha, d.data(), n);
    if ((iter + 1) % 10 == 0) {
      orc_tree_apply_mf(t, pw, x, q.data());
      par_sub(r.data(), b, q.data(), n);
    } else {
      par_axpy(r.data(), -alpha, q.data(), n);
    }
    const double delta_old = delta_new;
    delta_new = det_dot(r.data(), r.data(), n);
    if (delta) delta[iter + 1] = delta_new;
    if (delta_new <= delta_0 * accuracy * accuracy) return iter + 1;
    const double beta = delta_new / delta_old;
    if (std::isnan(beta) || std::isinf(beta)) break;
    par_xpby(d.data(), r.data(), beta, n);
  }
  return max_iters;
}

// orc_tree_solve_converged with the matrix-free operator and the caller's b: CG from the
// initial guess in x until ||b - A x|| <= tol ||b|| (explicit residual every 50 iterations).
// relres (may be NULL) receives the final explicit relative residual.
uint64_t orc_tree_solve_converged_mf(const orc_tree* t, double pw, const double* b, double tol, uint64_t maxit,
                                     double* x, double* relres) {
  const uint64_t n = t->n;
  std::vector<double> r(n), d(n), q(n);
  const double bb = det_dot(b, b, n);
  if (bb == 0.0) {
    if (relres) *relres = 0.0;
    return 0;
  }
  orc_tree_apply_mf(t, pw, x, q.data());
  par_sub(r.data(), b, q.data(), n);
  par_copy(d.data(), r.data(), n);
  double rr = det_dot(r.data(), r.data(), n);
  uint64_t it = 0;
  while (it < maxit && rr > tol * tol * bb) {
    orc_tree_apply_mf(t, pw, d.data(), q.data());
    const double dq = det_dot(d.data(), q.data(), n);
    if (dq == 0.0) break;
    const double alpha = rr / dq;
    par_axpy(x, alpha, d.data(), n);
    ++it;
    if (it % 50 == 0) {
      orc_tree_apply_mf(t, pw, x, q.data());
      par_sub(r.data(), b, q.data(), n);
    } else {
      par_axpy(r.data(), -alpha, q.data(), n);
    }
    const double rr_new = det_dot(r.data(), r.data(), n);
    const double beta = rr_new / rr;
    rr = rr_new;
    par_xpby(d.data(), r.data(), beta, n);
  }
  orc_tree_apply_mf(t, pw, x, q.data());
  par_sub(r.data(), b, q.data(), n);
  if (relres) *relres = std::sqrt(det_dot(r.data(), r.data(), n) / bb);
  return it;
}

// ---------------------------------------------------------------- evaluate / iso / MC
// FEMTree::evaluate (src/fem_tree.rs:490-513)
double orc_evaluate(uint32_t D, const double* sol, double px, double py, double pz) {
  const isize res = (isize)1 << D;
  const double h = 1.0 / (double)res;
  double sx = px / h, sy = py / h, sz = pz / h;
  uint32_t ox[2], oy[2], oz[2];
  contributing_offsets(sx, res, ox[0], ox[1]);
  contributing_offsets(sy, res, oy[0], oy[1]);
  contributing_offsets(sz, res, oz[0], oz[1]);
  double bx[2] = {bspline1(sx - (double)ox[0]), bspline1(sx - (double)ox[1])};
  double by[2] = {bspline1(sy - (double)oy[0]), bspline1(sy - (double)oy[1])};
  double bz[2] = {bspline1(sz - (double)oz[0]), bspline1(sz - (double)oz[1])};
  double v = 0.0;
  for (int a = 0; a < 2; ++a) {
    if (bx[a] == 0.0) continue;
    for (int b = 0; b < 2; ++b) {
      if (by[b] == 0.0) continue;
      for (int c = 0; c < 2; ++c) {
        if (bz[c] == 0.0) continue;
        v += sol[morton(ox[a], oy[b], oz[c])] * bx[a] * by[b] * bz[c];
      }
    }
  }
  return v;
}

void orc_evaluate_many(uint32_t D, const double* sol, const double* pts, uint64_t stride, uint64_t n, double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i)
    out[i] = orc_evaluate(D, sol, pts[stride * i], pts[stride * i + 1], pts[stride * i + 2]);
}

// iso = mean of evaluate at the unit-cube points (src/reconstructor.rs:56)
double orc_iso(uint32_t D, const double* sol, const double* unit6, uint64_t n) {
  std::vector<double> v(n), one(n, 1.0);
  orc_evaluate_many(D, sol, unit6, 6, n, v.data());
  return det_dot(v.data(), one.data(), n) / (double)n;
}



// FEMTree::extract_surface (src/fem_tree.rs:576-636).  Vertices in unit-cube space.  `eval` is the
// implicit function (evaluate() at degree 1; the degree-2 evaluation for the extension).
}  // extern "C"

template <typename Eval>
static int extract_surface_impl(uint32_t D, const double* sol, double iso, orc_mesh* out, Eval eval) {
  static const uint32_t co[8][3] = {{0,0,0},{1,0,0},{1,1,0},{0,1,0},{0,0,1},{1,0,1},{1,1,1},{0,1,1}};
  static const int ev[12][2] = {{0,1},{1,2},{2,3},{3,0},{4,5},{5,6},{6,7},{7,4},{0,4},{1,5},{2,6},{3,7}};
  const uint64_t max_res = 1ull << D;
  const uint64_t n = max_res * max_res * max_res;
  const double w = 1.0 / (double)max_res;  // (max_res >> D) as f64 / max_res as f64
  std::vector<double> verts;
  std::vector<uint64_t> tris;
  std::unordered_map<std::array<uint64_t, 3>, uint64_t, KeyHash> edge_hash;
  for (uint64_t cell = 0; cell < n; ++cell) {
    uint64_t off[3];
    unmorton(cell, off[0], off[1], off[2]);
    double cv[8];
    uint32_t mc = 0;
    for (int k = 0; k < 8; ++k) {
      double p[3];
      for (int a = 0; a < 3; ++a) p[a] = (double)(off[a] + co[k][a]) * w;
      cv[k] = eval(D, sol, p[0], p[1], p[2]);
      if (cv[k] < iso) mc |= 1u << k;
    }
    uint32_t em = orc_mc_edge_mask(mc);
    if (em == 0) continue;
    uint64_t evi[12];
    for (int e = 0; e < 12; ++e) {
      evi[e] = UINT64_MAX;
      if (!((em >> e) & 1u)) continue;
      int a = ev[e][0], b = ev[e][1];
      double dv = cv[b] - cv[a];
      double t = std::fabs(dv) < 1e-15 ? 0.5 : (iso - cv[a]) / dv;
      double pos[3];
      for (int ax = 0; ax < 3; ++ax) {
        double base = (double)(off[ax] + co[a][ax]) * w;
        pos[ax] = base + t * (double)((int32_t)co[b][ax] - (int32_t)co[a][ax]) * w;
      }
      std::array<uint64_t, 3> key = {f64_to_u64(pos[0] * 1e9), f64_to_u64(pos[1] * 1e9), f64_to_u64(pos[2] * 1e9)};
      auto it = edge_hash.find(key);
      if (it != edge_hash.end()) evi[e] = it->second;
      else {
        uint64_t idx = verts.size() / 3;
        edge_hash.emplace(key, idx);
        verts.insert(verts.end(), pos, pos + 3);
        evi[e] = idx;
      }
    }
    for (int i = 0; i < 3 * PR_MC_NTRI[mc]; i += 3) {
      for (int k = 0; k < 3; ++k) tris.push_back(evi[(PR_MC_TRIS[mc] >> (4 * (i + k))) & 15ull]);
    }
  }
  out->nv = verts.size() / 3;
  out->nt = tris.size() / 3;
  out->verts = (double*)std::malloc(std::max<size_t>(1, verts.size()) * sizeof(double));
  out->tris = (uint64_t*)std::malloc(std::max<size_t>(1, tris.size()) * sizeof(uint64_t));
  if (!verts.empty()) std::memcpy(out->verts, verts.data(), verts.size() * sizeof(double));
  if (!tris.empty()) std::memcpy(out->tris, tris.data(), tris.size() * sizeof(uint64_t));
  return 0;
}

extern "C" {

int orc_extract_surface(uint32_t D, const double* sol, double iso, orc_mesh* out) {
  return extract_surface_impl(D, sol, iso, out, orc_evaluate);
}

void orc_mesh_free(orc_mesh* m) {
  std::free(m->verts);
  std::free(m->tris);
  m->verts = nullptr;
  m->tris = nullptr;
  m->nv = m->nt = 0;
}

// ---------------------------------------------------------------- generic CSR (ported unit tests)
uint64_t orc_csr_cg(uint64_t n, const uint64_t* ptr, const uint32_t* col, const double* val, const double* b,
                    double* x, uint64_t maxit, double acc) {
  Csr a;
  a.rows = n;
  a.ptr.assign(ptr, ptr + n + 1);
  a.col.assign(col, col + ptr[n]);
  a.val.assign(val, val + ptr[n]);
  return solve_cg(a, b, x, maxit, acc);
}
void orc_csr_spmv(uint64_t n, const uint64_t* ptr, const uint32_t* col, const double* val, const double* x, double* y) {
  Csr a;
  a.rows = n;
  a.ptr.assign(ptr, ptr + n + 1);
  a.col.assign(col, col + ptr[n]);
  a.val.assign(val, val + ptr[n]);
  a.spmv(x, y);
}
void orc_csr_gs_sweep(uint64_t n, const uint64_t* ptr, const uint32_t* col, const double* val, const double* b, double* x) {
  Csr a;
  a.rows = n;
  a.ptr.assign(ptr, ptr + n + 1);
  a.col.assign(col, col + ptr[n]);
  a.val.assign(val, val + ptr[n]);
  gauss_seidel_sweep(a, b, x);
}

// ---------------------------------------------------------------- full pipeline
// reconstructor::reconstruct (src/reconstructor.rs:25-70).  solve_mode 0 runs the crate's
// cascadic schedule; solve_mode 1 solves the same fine system to target_rel_residual.
// coeffs (n doubles, Morton order) may be NULL.
int orc_reconstruct(const double* pts6, uint64_t n, const orc_params* p, orc_mesh* mesh, orc_stats* st,
                    double* coeffs) {
  std::memset(st, 0, sizeof(*st));
  mesh->verts = nullptr; mesh->tris = nullptr; mesh->nv = mesh->nt = 0;
  if (n == 0) return 0;
  double bmin[3], bmax[3], M[16], Minv[16];
  orc_bbox(pts6, n, bmin, bmax);
  orc_unit_cube_transform(bmin, bmax, p->scale, M);
  orc_mat4_inverse(M, Minv);
  std::vector<double> unit(6 * n);
  orc_transform_points(M, pts6, n, unit.data());
  orc_tree* t = orc_tree_new(p->depth, unit.data(), n);
  st->fem_nodes = t->n;
  std::vector<double> x(t->n, 0.0);
  if (p->solve_mode == 0) {
    uint64_t info[2];
    orc_tree_solve_reference(t, p->point_weight, p->cg_iters, p->cg_accuracy, x.data(), info);
    st->iterations = info[1];
  } else {
    double rr = 0.0;
    st->iterations = orc_tree_solve_converged(t, p->point_weight, p->target_rel_residual, p->max_iters, x.data(), &rr);
    st->rel_residual = rr;
  }
  double iso = orc_iso(t->D, x.data(), unit.data(), n);
  st->iso_value = iso;
  orc_extract_surface(t->D, x.data(), iso, mesh);
  for (uint64_t v = 0; v < mesh->nv; ++v) {
    double q[3];
    orc_transform_point(Minv, mesh->verts + 3 * v, q);
    std::memcpy(mesh->verts + 3 * v, q, sizeof(q));
  }
  st->mesh_vertices = mesh->nv;
  st->mesh_triangles = mesh->nt;
  if (coeffs) std::memcpy(coeffs, x.data(), t->n * sizeof(double));
  orc_tree_free(t);
  return 0;
}

// ---------------------------------------------------------------- adjoint (no reference counterpart)
// Gradient of a loss on the implicit function at K query points.  chi_k = evaluate(x, M q_k)
// (q_k in model space, M the unit-cube transform of the input, held fixed: the bbox is not
// differentiated).  Upstream g_k = dL/dchi_k; with g = NULL the loss is L = mean_k chi_k^2
// and g_k = 2 chi_k / K.  With A x = b (A symmetric) the adjoint is A lambda = E^T g, and
//   dL/dtheta = lambda . (db/dtheta) - lambda . (dA/dtheta) x.
// b = G nf + screening RHS, nf_j = -(sum_i phi_j(u_i) nu_i) / w_j, w_j = sum_i phi_j(u_i)
// (splat, floor cells, src/fem_tree.rs:130-178; divergence stencil G, :251-274; screening
// RHS and matrix on trunc cells, :276-297 and :220-228).

// CG from x = 0 until ||b - A x|| <= tol ||b|| (explicit residual every 50 iterations).
static uint64_t cg_to_tol(const Csr& A, const double* b, double* x, double tol, uint64_t maxit) {
  const uint64_t n = A.rows;
  std::vector<double> r(b, b + n), d(b, b + n), q(n);
  std::fill(x, x + n, 0.0);
  const double bb = det_dot(b, b, n);
  if (bb == 0.0) return 0;
  double rr = bb;
  uint64_t it = 0;
  while (it < maxit && rr > tol * tol * bb) {
    A.spmv(d.data(), q.data());
    const double dq = det_dot(d.data(), q.data(), n);
    if (dq == 0.0) break;
    const double alpha = rr / dq;
    for (uint64_t i = 0; i < n; ++i) x[i] += alpha * d[i];
    ++it;
    if (it % 50 == 0) {
      A.spmv(x, q.data());
      for (uint64_t i = 0; i < n; ++i) r[i] = b[i] - q[i];
    } else {
      for (uint64_t i = 0; i < n; ++i) r[i] -= alpha * q[i];
    }
    const double rr_new = det_dot(r.data(), r.data(), n);
    const double beta = rr_new / rr;
    rr = rr_new;
    for (uint64_t i = 0; i < n; ++i) d[i] = r[i] + beta * d[i];
  }
  return it;
}

// Trilinear basis of one corner: value and gradient in unit-cube coordinates.  t: in-cell
// coordinates; d: corner offsets; inv_h = 1/h.
static inline void corner_basis(const double t[3], const int d[3], double inv_h, double& phi, double g[3]) {
  double b[3], db[3];
  for (int a = 0; a < 3; ++a) {
    b[a] = d[a] ? t[a] : 1.0 - t[a];
    db[a] = d[a] ? inv_h : -inv_h;
  }
  phi = b[0] * b[1] * b[2];
  g[0] = db[0] * b[1] * b[2];
  g[1] = b[0] * db[1] * b[2];
  g[2] = b[0] * b[1] * db[2];
}

// Shared forward: transform, tree, converged solve of A x = b, chi at the queries.
struct AdjFwd {
  double M[16];
  std::vector<double> unit;
  orc_tree* t = nullptr;
  std::vector<double> x, qu;
  ~AdjFwd() { if (t) orc_tree_free(t); }
};
static void adj_forward(AdjFwd& f, const double* pts6, uint64_t n, uint32_t depth, double pw, double scale,
                        const double* q3, uint64_t k, double tol, double* chi) {
  double bmin[3], bmax[3];
  orc_bbox(pts6, n, bmin, bmax);
  orc_unit_cube_transform(bmin, bmax, scale, f.M);
  f.unit.resize(6 * n);
  orc_transform_points(f.M, pts6, n, f.unit.data());
  f.t = orc_tree_new(depth, f.unit.data(), n);
  orc_tree_assemble(f.t, pw);
  std::vector<double> b(f.t->n);
  orc_tree_rhs(f.t, pw, b.data());
  f.x.assign(f.t->n, 0.0);
  cg_to_tol(f.t->A, b.data(), f.x.data(), tol, 100000);
  f.qu.resize(3 * k);
  for (uint64_t i = 0; i < k; ++i) orc_transform_point(f.M, q3 + 3 * i, &f.qu[3 * i]);
  orc_evaluate_many(depth, f.x.data(), f.qu.data(), 3, k, chi);
}

// Loss only (for finite differences): mean chi^2, or sum g_k chi_k when g is given.
double orc_loss(const double* pts6, uint64_t n, uint32_t depth, double pw, double scale, const double* q3, uint64_t k,
                const double* g, double tol) {
  AdjFwd f;
  std::vector<double> chi(k);
  adj_forward(f, pts6, n, depth, pw, scale, q3, k, tol, chi.data());
  double L = 0.0;
  for (uint64_t i = 0; i < k; ++i) L += g ? g[i] * chi[i] : chi[i] * chi[i];
  return g ? L : L / (double)k;
}

// Gradients w.r.t. the model-space positions and normals of the input (n x 3 each).
int orc_loss_backward(const double* pts6, uint64_t n, uint32_t depth, double pw, double scale, const double* q3,
                      uint64_t k, const double* dl_dchi, double tol, double* chi, double* dpos, double* dnrm,
                      double* loss) {
  if (n == 0 || k == 0) return -1;
  AdjFwd f;
  adj_forward(f, pts6, n, depth, pw, scale, q3, k, tol, chi);
  orc_tree* t = f.t;
  const isize res = (isize)t->res;
  const double h = t->h, inv_h = 1.0 / h;
  std::vector<double> g(k);
  double L = 0.0;
  for (uint64_t i = 0; i < k; ++i) {
    g[i] = dl_dchi ? dl_dchi[i] : 2.0 * chi[i] / (double)k;
    L += dl_dchi ? dl_dchi[i] * chi[i] : chi[i] * chi[i];
  }
  if (loss) *loss = dl_dchi ? L : L / (double)k;
  // E^T g: the transpose of evaluate's shifted trilinear basis (src/fem_tree.rs:490-513)
  std::vector<double> rhs(t->n, 0.0);
  for (uint64_t i = 0; i < k; ++i) {
    const double s[3] = {f.qu[3 * i] / h, f.qu[3 * i + 1] / h, f.qu[3 * i + 2] / h};
    uint32_t o[3][2];
    double bs[3][2];
    for (int a = 0; a < 3; ++a) {
      contributing_offsets(s[a], res, o[a][0], o[a][1]);
      bs[a][0] = bspline1(s[a] - (double)o[a][0]);
      bs[a][1] = bspline1(s[a] - (double)o[a][1]);
    }
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int c = 0; c < 2; ++c)
          rhs[morton(o[0][a], o[1][b], o[2][c])] += g[i] * bs[0][a] * bs[1][b] * bs[2][c];
  }
  std::vector<double> lam(t->n, 0.0);
  cg_to_tol(t->A, rhs.data(), lam.data(), tol, 100000);
  // mu_j = dL/dnf_j = G^T lambda at nodes with a splat weight
  std::vector<double> mu(3 * t->n, 0.0);
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < (int64_t)t->n; ++j) {
    if (!(t->nw[j] > 0.0)) continue;
    uint64_t jx, jy, jz;
    unmorton((uint64_t)j, jx, jy, jz);
    double m0 = 0.0, m1 = 0.0, m2 = 0.0;
    for (isize dx = -1; dx <= 1; ++dx)
      for (isize dy = -1; dy <= 1; ++dy)
        for (isize dz = -1; dz <= 1; ++dz) {
          // row i = j - d sees node j at offset d
          const isize ix = (isize)jx - dx, iy = (isize)jy - dy, iz = (isize)jz - dz;
          if (ix < 0 || iy < 0 || iz < 0 || ix >= res || iy >= res || iz >= res) continue;
          const double l = lam[morton(ix, iy, iz)] * h * h;
          m0 += l * deriv_mass_1d(dx) * mass_1d(dy) * mass_1d(dz);
          m1 += l * mass_1d(dx) * deriv_mass_1d(dy) * mass_1d(dz);
          m2 += l * mass_1d(dx) * mass_1d(dy) * deriv_mass_1d(dz);
        }
    mu[3 * j] = m0;
    mu[3 * j + 1] = m1;
    mu[3 * j + 2] = m2;
  }
  const double wh3 = pw > 0.0 ? pw * (h * h * h) / 1.5 : 0.0;
  const double s_m = f.M[0];
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < (int64_t)n; ++p) {
    const double* u = &f.unit[6 * p];
    const double nu[3] = {u[3], u[4], u[5]};
    double gu[3] = {0, 0, 0}, gn[3] = {0, 0, 0};
    {  // splat (floor cells)
      isize c[3];
      double tt[3];
      for (int a = 0; a < 3; ++a) {
        c[a] = f64_to_isize(std::floor(u[a] / h));
        tt[a] = u[a] / h - (double)c[a];
      }
      for (int kk = 0; kk < 8; ++kk) {
        const int d[3] = {kk & 1, (kk >> 1) & 1, kk >> 2};
        const uint64_t ox = (uint64_t)(c[0] + d[0]), oy = (uint64_t)(c[1] + d[1]), oz = (uint64_t)(c[2] + d[2]);
        if (ox >= t->res || oy >= t->res || oz >= t->res) continue;
        const uint64_t j = morton(ox, oy, oz);
        const double w = t->nw[j];
        if (!(w > 0.0)) continue;
        double phi, gp[3];
        corner_basis(tt, d, inv_h, phi, gp);
        const double* m = &mu[3 * j];
        const double* nf = &t->nf[3 * j];
        const double sdot = m[0] * (nu[0] + nf[0]) + m[1] * (nu[1] + nf[1]) + m[2] * (nu[2] + nf[2]);
        for (int a = 0; a < 3; ++a) {
          gn[a] -= phi / w * m[a];
          gu[a] -= gp[a] / w * sdot;
        }
      }
    }
    if (pw > 0.0) {  // screening RHS and matrix (trunc cells)
      isize c[3];
      double tt[3];
      for (int a = 0; a < 3; ++a) {
        c[a] = f64_to_isize(u[a] / h);
        tt[a] = u[a] / h - (double)c[a];
      }
      double Lv = 0.0, Xv = 0.0, gL[3] = {0, 0, 0}, gX[3] = {0, 0, 0};
      for (int kk = 0; kk < 8; ++kk) {
        const int d[3] = {kk & 1, (kk >> 1) & 1, kk >> 2};
        const uint32_t ox = (uint32_t)(uint64_t)(c[0] + d[0]), oy = (uint32_t)(uint64_t)(c[1] + d[1]),
                       oz = (uint32_t)(uint64_t)(c[2] + d[2]);
        if (ox >= (uint32_t)t->res || oy >= (uint32_t)t->res || oz >= (uint32_t)t->res) continue;
        const uint64_t j = morton(ox, oy, oz);
        double phi, gp[3];
        corner_basis(tt, d, inv_h, phi, gp);
        Lv += phi * lam[j];
        Xv += phi * f.x[j];
        for (int a = 0; a < 3; ++a) {
          gL[a] += gp[a] * lam[j];
          gX[a] += gp[a] * f.x[j];
        }
      }
      for (int a = 0; a < 3; ++a) gu[a] += wh3 * 0.5 * gL[a] - wh3 * (gL[a] * Xv + Lv * gX[a]);
    }
    // model space: u = s p + c (transform held fixed); nu = v/|v|, v = s n
    const double* pm = pts6 + 6 * p;
    const double v[3] = {s_m * pm[3], s_m * pm[4], s_m * pm[5]};
    const double len = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    const double ng = nu[0] * gn[0] + nu[1] * gn[1] + nu[2] * gn[2];
    for (int a = 0; a < 3; ++a) {
      dpos[3 * p + a] = s_m * gu[a];
      dnrm[3 * p + a] = len > 0.0 ? s_m / len * (gn[a] - nu[a] * ng) : 0.0;
    }
  }
  return 0;
}

// ================================================================ degree 2 (extension)
// The crate's degree-2 code (src/bspline.rs:74-123, 322-417) is not on its reconstruction path.
// This restatement defines the degree-2 system the library builds, on the crate's conventions:
// node functions phi_i(x) = N2(x/h - i + 1), i in [0, res) (cell-centred quadratic B-splines,
// src/bspline.rs:334-345), stencil values of the infinite grid on every row with neighbours
// outside the grid omitted (as the crate's degree-1 stiffness, src/fem_tree.rs:180-249),
//   A(d) = h (s m m + m s m + m m s)(d) + wg [d = 0] + wh3 sum_p phi(p) phi(p)^T,
//   b_i  = h^2 sum_j sum_a nf_j^a (g m m)_a(j - i) + (wh3/2) sum_p phi_i(p),
// with m, s, g the 1-D integrals of N2 N2, N2' N2', N2' N2 at offsets -2..2 (exact: 3-point
// Gauss-Legendre per unit cell), nf the normalised splat of the normals with the same basis
// (27 functions per point), wh3 = pw h^3 / 1.5 and wg = wh3 / 200 as at degree 1.  Grid vectors
// are in Morton order like the degree-1 ones.
}  // extern "C"
namespace {
double n2(double x) {
  if (x <= 0.0 || x >= 3.0) return 0.0;
  if (x <= 1.0) return 0.5 * x * x;
  if (x <= 2.0) return 0.5 * (-2.0 * x * x + 6.0 * x - 3.0);
  const double t = 3.0 - x;
  return 0.5 * t * t;
}
double dn2(double x) {
  if (x <= 0.0 || x >= 3.0) return 0.0;
  if (x <= 1.0) return x;
  if (x <= 2.0) return 3.0 - 2.0 * x;
  return x - 3.0;
}
struct Deg2 {
  double m[5], s[5], g[5];  // offset d = -2..2 at index d + 2
  Deg2() {
    const double gx[3] = {-0.7745966692414834, 0.0, 0.7745966692414834};
    const double gw[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
    for (int d = -2; d <= 2; ++d) {
      double am = 0.0, as = 0.0, ag = 0.0;
      for (int c = -1; c < 5; ++c)
        for (int q = 0; q < 3; ++q) {
          const double t = c + 0.5 + 0.5 * gx[q], w = 0.5 * gw[q];
          am += w * n2(t) * n2(t - d);
          as += w * dn2(t) * dn2(t - d);
          ag += w * dn2(t) * n2(t - d);
        }
      m[d + 2] = am;
      s[d + 2] = as;
      g[d + 2] = ag;
    }
  }
};
const Deg2& deg2() {
  static const Deg2 k;
  return k;
}
// basis of one axis at unit coordinate u: nodes o[3] (c-1, c, c+1) and weights b[3], grad db[3]
// (d/du); valid[k] = node in [0, res)
void axis2(double u, double h, isize res, isize* o, double* b, double* db) {
  const double s = u / h;
  const isize c = f64_to_isize(std::floor(s));
  const double t = s - (double)c;
  o[0] = c - 1; o[1] = c; o[2] = c + 1;
  b[0] = 0.5 * (1.0 - t) * (1.0 - t);
  b[1] = 0.5 * (-2.0 * t * t + 2.0 * t + 1.0);
  b[2] = 0.5 * t * t;
  db[0] = -(1.0 - t) / h;
  db[1] = (1.0 - 2.0 * t) / h;
  db[2] = t / h;
  (void)res;
}
inline bool in_range(isize i, isize res) { return i >= 0 && i < res; }
}  // namespace
extern "C" {

void orc_deg2_constants(double* m5, double* s5, double* g5) {
  for (int k = 0; k < 5; ++k) {
    m5[k] = deg2().m[k];
    s5[k] = deg2().s[k];
    g5[k] = deg2().g[k];
  }
}

double orc_evaluate2(uint32_t D, const double* sol, double px, double py, double pz) {
  const isize res = (isize)1 << D;
  const double h = 1.0 / (double)res;
  isize o[3][3];
  double b[3][3], db[3][3];
  axis2(px, h, res, o[0], b[0], db[0]);
  axis2(py, h, res, o[1], b[1], db[1]);
  axis2(pz, h, res, o[2], b[2], db[2]);
  double v = 0.0;
  for (int k = 0; k < 3; ++k) {
    if (!in_range(o[2][k], res)) continue;
    for (int j = 0; j < 3; ++j) {
      if (!in_range(o[1][j], res)) continue;
      for (int i = 0; i < 3; ++i) {
        if (!in_range(o[0][i], res)) continue;
        v += sol[morton(o[0][i], o[1][j], o[2][k])] * b[0][i] * b[1][j] * b[2][k];
      }
    }
  }
  return v;
}

struct orc_tree2 {
  uint32_t D;
  isize res;
  uint64_t n;
  double h, pw;
  std::vector<P6> pts;
  std::vector<double> nf, nw;  // 3n normal field (normalised, negated), n weights
};

orc_tree2* orc_tree2_new(uint32_t depth, const double* unit6, uint64_t npts, double pw) {
  orc_tree2* t = new orc_tree2();
  t->D = depth;
  t->res = (isize)1 << depth;
  t->n = (uint64_t)t->res * t->res * t->res;
  t->h = 1.0 / (double)t->res;
  t->pw = pw;
  t->pts.resize(npts);
  std::memcpy(t->pts.data(), unit6, npts * sizeof(P6));
  t->nf.assign(3 * t->n, 0.0);
  t->nw.assign(t->n, 0.0);
  for (const P6& p : t->pts) {
    isize o[3][3];
    double b[3][3], db[3][3];
    axis2(p.x, t->h, t->res, o[0], b[0], db[0]);
    axis2(p.y, t->h, t->res, o[1], b[1], db[1]);
    axis2(p.z, t->h, t->res, o[2], b[2], db[2]);
    for (int k = 0; k < 3; ++k)
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
          if (!in_range(o[0][i], t->res) || !in_range(o[1][j], t->res) || !in_range(o[2][k], t->res)) continue;
          const uint64_t idx = morton(o[0][i], o[1][j], o[2][k]);
          const double w = b[0][i] * b[1][j] * b[2][k];
          t->nf[3 * idx] += p.nx * w;
          t->nf[3 * idx + 1] += p.ny * w;
          t->nf[3 * idx + 2] += p.nz * w;
          t->nw[idx] += w;
        }
  }
  for (uint64_t i = 0; i < t->n; ++i)
    if (t->nw[i] > 0.0)
      for (int a = 0; a < 3; ++a) t->nf[3 * i + a] = -t->nf[3 * i + a] / t->nw[i];
  return t;
}
void orc_tree2_free(orc_tree2* t) { delete t; }

void orc_tree2_normal_field(const orc_tree2* t, double* nf3, double* w) {
  std::memcpy(nf3, t->nf.data(), 3 * t->n * sizeof(double));
  std::memcpy(w, t->nw.data(), t->n * sizeof(double));
}

void orc_tree2_rhs(const orc_tree2* t, double* b) {
  const Deg2& K = deg2();
  const isize res = t->res;
  const double h2 = t->h * t->h;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)t->n; ++i) {
    uint64_t ix, iy, iz;
    unmorton((uint64_t)i, ix, iy, iz);
    double sum = 0.0;
    for (int dz = -2; dz <= 2; ++dz)
      for (int dy = -2; dy <= 2; ++dy)
        for (int dx = -2; dx <= 2; ++dx) {
          const isize jx = (isize)ix + dx, jy = (isize)iy + dy, jz = (isize)iz + dz;
          if (!in_range(jx, res) || !in_range(jy, res) || !in_range(jz, res)) continue;
          const double* v = &t->nf[3 * morton(jx, jy, jz)];
          sum += v[0] * K.g[dx + 2] * K.m[dy + 2] * K.m[dz + 2] + v[1] * K.m[dx + 2] * K.g[dy + 2] * K.m[dz + 2] +
                 v[2] * K.m[dx + 2] * K.m[dy + 2] * K.g[dz + 2];
        }
    b[i] = h2 * sum;
  }
  if (t->pw > 0.0) {
    const double wh3 = t->pw * t->h * t->h * t->h / 1.5;
    for (const P6& p : t->pts) {
      isize o[3][3];
      double bb[3][3], db[3][3];
      axis2(p.x, t->h, res, o[0], bb[0], db[0]);
      axis2(p.y, t->h, res, o[1], bb[1], db[1]);
      axis2(p.z, t->h, res, o[2], bb[2], db[2]);
      for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 3; ++j)
          for (int i = 0; i < 3; ++i) {
            if (!in_range(o[0][i], res) || !in_range(o[1][j], res) || !in_range(o[2][k], res)) continue;
            b[morton(o[0][i], o[1][j], o[2][k])] += wh3 * 0.5 * bb[0][i] * bb[1][j] * bb[2][k];
          }
    }
  }
}

// y = A x (125-point stencil + wg + screening), matrix-free
void orc_tree2_apply(const orc_tree2* t, const double* x, double* y) {
  const Deg2& K = deg2();
  const isize res = t->res;
  const double h = t->h;
  const double wh3 = t->pw > 0.0 ? t->pw * h * h * h / 1.5 : 0.0;
  const double wg = wh3 * 0.005;
  (void)res;
  // h (S m m + m S m + m m S) x on the zero-extended vector (neighbours outside the grid omitted),
  // as separable passes over each block's tile: z (M, S), then y, then x
  blocked_tiles<1, 2>(t->D, x, [&](uint64_t blk, const double* tile, int T, int B, const int* loc, const int64_t*) {
    const int T2 = T * T;
    thread_local std::vector<double> um, us, w1, w23;  // [z][y][x]: z in the block; y, x in the tile / x in the tile
    um.resize((size_t)B * T2);
    us.resize((size_t)B * T2);
    w1.resize((size_t)B * B * T);
    w23.resize((size_t)B * B * T);
    for (int z = 0; z < B; ++z)
      for (int yx = 0; yx < T2; ++yx) {
        double am = 0.0, as = 0.0;
        for (int c = 0; c < 5; ++c) {
          const double v = tile[(size_t)(z + c) * T2 + yx];
          am += K.m[c] * v;
          as += K.s[c] * v;
        }
        um[(size_t)z * T2 + yx] = am;
        us[(size_t)z * T2 + yx] = as;
      }
    for (int z = 0; z < B; ++z)
      for (int y = 0; y < B; ++y)
        for (int xx = 0; xx < T; ++xx) {
          double a1 = 0.0, a2 = 0.0, a3 = 0.0;
          for (int c = 0; c < 5; ++c) {
            const size_t q = (size_t)z * T2 + (size_t)(y + c) * T + xx;
            a1 += K.m[c] * um[q];
            a2 += K.s[c] * um[q];
            a3 += K.m[c] * us[q];
          }
          w1[((size_t)z * B + y) * T + xx] = a1;
          w23[((size_t)z * B + y) * T + xx] = a2 + a3;
        }
    const uint64_t bsz = (uint64_t)B * B * B;
    for (uint64_t l = 0; l < bsz; ++l) {
      const int* q = &loc[3 * l];
      const size_t r = ((size_t)q[2] * B + q[1]) * T + q[0];
      double acc = 0.0;
      for (int c = 0; c < 5; ++c) acc += K.s[c] * w1[r + c] + K.m[c] * w23[r + c];
      const double xc = tile[(size_t)((q[2] + 2) * T + (q[1] + 2)) * T + (q[0] + 2)];
      y[blk * bsz + l] = h * acc + wg * xc;
    }
  });
  if (wh3 > 0.0) {
#pragma omp parallel for schedule(static)
    for (int64_t pi = 0; pi < (int64_t)t->pts.size(); ++pi) {
      const P6& p = t->pts[pi];
      isize o[3][3];
      double bb[3][3], db[3][3];
      axis2(p.x, h, res, o[0], bb[0], db[0]);
      axis2(p.y, h, res, o[1], bb[1], db[1]);
      axis2(p.z, h, res, o[2], bb[2], db[2]);
      uint64_t idx[27];
      double phi[27];
      int m = 0;
      for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 3; ++j)
          for (int ii = 0; ii < 3; ++ii) {
            if (!in_range(o[0][ii], res) || !in_range(o[1][j], res) || !in_range(o[2][k], res)) continue;
            idx[m] = morton(o[0][ii], o[1][j], o[2][k]);
            phi[m] = bb[0][ii] * bb[1][j] * bb[2][k];
            ++m;
          }
      double proj = 0.0;
      for (int q = 0; q < m; ++q) proj += phi[q] * x[idx[q]];
      for (int q = 0; q < m; ++q) {
        const double v = wh3 * phi[q] * proj;
#pragma omp atomic
        y[idx[q]] += v;
      }
    }
  }
}

// Frees the normal field and weights (the operator needs only the points).
void orc_tree2_release_field(orc_tree2* t) {
  std::vector<double>().swap(t->nf);
  std::vector<double>().swap(t->nw);
}

// A CG run kept between calls, one iteration per orc_cg_step: the loop body of solve_cg
// (src/solvers.rs:20-69; residual recomputed as b - A x every 10th iteration) on a matrix-free
// operator, from x = 0.  The CPU baseline times single iterations of it.
struct orc_cg {
  std::function<void(const double*, double*)> apply;
  uint64_t n = 0;
  std::vector<double> b, x, r, d, q;
  double delta = 0.0;
  uint64_t it = 0;
};
static orc_cg* cg_new(std::function<void(const double*, double*)> apply, uint64_t n, const double* b) {
  orc_cg* s = new orc_cg();
  s->apply = std::move(apply);
  s->n = n;
  s->b.assign(b, b + n);
  s->x.assign(n, 0.0);
  s->r = s->b;
  s->d = s->b;
  s->q.assign(n, 0.0);
  s->delta = det_dot(s->r.data(), s->r.data(), n);
  return s;
}
orc_cg* orc_cg2_new(const orc_tree2* t, const double* b) {
  return cg_new([t](const double* x, double* y) { orc_tree2_apply(t, x, y); }, t->n, b);
}
orc_cg* orc_cg1_new(const orc_tree* t, double pw, const double* b) {
  return cg_new([t, pw](const double* x, double* y) { orc_tree_apply_mf(t, pw, x, y); }, t->n, b);
}
double orc_cg_step(orc_cg* s) {
  const uint64_t n = s->n;
  s->apply(s->d.data(), s->q.data());
  const double dq = det_dot(s->d.data(), s->q.data(), n);
  if (dq == 0.0) return s->delta;
  const double alpha = s->delta / dq;
  par_axpy(s->x.data(), alpha, s->d.data(), n);
  if ((s->it + 1) % 10 == 0) {
    s->apply(s->x.data(), s->q.data());
    par_sub(s->r.data(), s->b.data(), s->q.data(), n);
  } else {
    par_axpy(s->r.data(), -alpha, s->q.data(), n);
  }
  const double delta_old = s->delta;
  s->delta = det_dot(s->r.data(), s->r.data(), n);
  par_xpby(s->d.data(), s->r.data(), s->delta / delta_old, n);
  ++s->it;
  return s->delta;
}
void orc_cg_free(orc_cg* s) { delete s; }

// CG (from x = 0) to ||b - A x|| <= tol ||b||; returns iterations, *relres the final relative residual
uint64_t orc_tree2_solve(const orc_tree2* t, double tol, uint64_t maxit, double* x, double* relres) {
  const uint64_t n = t->n;
  std::vector<double> b(n), r(n), d(n), q(n);
  orc_tree2_rhs(t, b.data());
  std::fill(x, x + n, 0.0);
  const double bb = det_dot(b.data(), b.data(), n);
  if (bb == 0.0) {
    if (relres) *relres = 0.0;
    return 0;
  }
  r = b;
  d = b;
  double rr = bb;
  uint64_t it = 0;
  while (it < maxit && rr > tol * tol * bb) {
    orc_tree2_apply(t, d.data(), q.data());
    const double dq = det_dot(d.data(), q.data(), n);
    if (dq == 0.0) break;
    const double alpha = rr / dq;
    for (uint64_t i = 0; i < n; ++i) x[i] += alpha * d[i];
    ++it;
    if (it % 50 == 0) {
      orc_tree2_apply(t, x, q.data());
      for (uint64_t i = 0; i < n; ++i) r[i] = b[i] - q[i];
    } else {
      for (uint64_t i = 0; i < n; ++i) r[i] -= alpha * q[i];
    }
    const double rr_new = det_dot(r.data(), r.data(), n);
    const double beta = rr_new / rr;
    rr = rr_new;
    for (uint64_t i = 0; i < n; ++i) d[i] = r[i] + beta * d[i];
  }
  orc_tree2_apply(t, x, q.data());
  for (uint64_t i = 0; i < n; ++i) r[i] = b[i] - q[i];
  if (relres) *relres = std::sqrt(det_dot(r.data(), r.data(), n) / bb);
  return it;
}

double orc_evaluate2(uint32_t D, const double* sol, double px, double py, double pz);
int orc_extract_surface2(uint32_t D, const double* sol, double iso, orc_mesh* out) {
  return extract_surface_impl(D, sol, iso, out, orc_evaluate2);
}

// Degree-2 pipeline: transform (as reconstruct), tree2, converged CG, iso (mean of the degree-2
// evaluation over the unit points), marching cubes on the degree-2 function, back-transform.
int orc_reconstruct2(const double* pts6, uint64_t n, uint32_t depth, double scale, double pw, double tol,
                     uint64_t maxit, orc_mesh* mesh, double* iso_out, double* relres, double* coeffs) {
  mesh->verts = nullptr; mesh->tris = nullptr; mesh->nv = mesh->nt = 0;
  if (n == 0) return 0;
  double bmin[3], bmax[3], M[16], Minv[16];
  orc_bbox(pts6, n, bmin, bmax);
  orc_unit_cube_transform(bmin, bmax, scale, M);
  orc_mat4_inverse(M, Minv);
  std::vector<double> unit(6 * n);
  orc_transform_points(M, pts6, n, unit.data());
  orc_tree2* t = orc_tree2_new(depth, unit.data(), n, pw);
  std::vector<double> x(t->n, 0.0);
  orc_tree2_solve(t, tol, maxit, x.data(), relres);
  std::vector<double> v(n), one(n, 1.0);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i) v[i] = orc_evaluate2(depth, x.data(), unit[6 * i], unit[6 * i + 1], unit[6 * i + 2]);
  const double iso = det_dot(v.data(), one.data(), n) / (double)n;
  if (iso_out) *iso_out = iso;
  orc_extract_surface2(depth, x.data(), iso, mesh);
  for (uint64_t k = 0; k < mesh->nv; ++k) {
    double q[3];
    orc_transform_point(Minv, mesh->verts + 3 * k, q);
    std::memcpy(mesh->verts + 3 * k, q, sizeof(q));
  }
  if (coeffs) std::memcpy(coeffs, x.data(), t->n * sizeof(double));
  orc_tree2_free(t);
  return 0;
}

}  // extern "C"

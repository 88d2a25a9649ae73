// Extraction stage: iso value and marching cubes, bit-identical to the crate given the
// same FP64 coefficients.
//
//   iso  = mean of FEMTree::evaluate at the points      src/reconstructor.rs:56, src/fem_tree.rs:490-513
//   mesh = FEMTree::extract_surface                      src/fem_tree.rs:576-636
//
// The crate visits every leaf cell in Morton order, classifies the 8 corner values
// against iso, emits one vertex per cut edge (edge order 0..11), deduplicates vertices
// through a hash map keyed by ((x*1e9) as u64, (y*1e9) as u64, (z*1e9) as u64) and numbers
// them in order of first appearance, then emits TRI_TABLE triangles in row order.  The GPU
// version is a count / scan / emit pipeline:
//   1. per cell: case index; per block of cells: active-cell count      (k_mc_count)
//   2. exclusive scan; active cells written in Morton order             (k_mc_compact)
//   3. per active cell: vertex slots (cell order, then edge order) with position and key
//   4. stable sort of slots by key; the first slot of each key run is its vertex; vertex
//      ids = rank of first slots in slot order (= the crate's first-appearance numbering)
//   5. triangles from the packed table, vertices back-transformed to model space.
// Corner values at integer grid positions reduce to a shifted gather (the evaluation is
// offset by one cell, src/fem_tree.rs:645-649): node k-1 per axis, none at k = 0 and the
// last node counted twice at k = res.
#include <cub/cub.cuh>

#include "pr_internal.cuh"

#define PR_MC_TABLE_QUAL __constant__
#include "mc_tri_table.inc"

namespace pr {

namespace {

constexpr int kThreads = 256;

inline unsigned grid_for(uint64_t n, int threads = kThreads, uint64_t cap = 1u << 22) {
  uint64_t g = (n + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (unsigned)g;
}

__constant__ int c_co[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
__constant__ int c_ev[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};

// edge e is cut iff its corners classify differently (== the crate's EDGE_TABLE)
__device__ __forceinline__ uint32_t edge_mask(uint32_t mc) {
  uint32_t m = 0;
#pragma unroll
  for (int e = 0; e < 12; ++e)
    if (((mc >> c_ev[e][0]) & 1u) != ((mc >> c_ev[e][1]) & 1u)) m |= 1u << e;
  return m;
}

// bspline1 (src/fem_tree.rs:640-642)
__device__ __forceinline__ double bspline1(double t) {
  if (t < 0.0 || t > 2.0) return 0.0;
  if (t <= 1.0) return t;
  return xsub(2.0, t);
}

// FEMTree::evaluate (src/fem_tree.rs:490-513), same operation order
__device__ double eval_fem(const double* __restrict__ x, uint32_t D, double px, double py, double pz) {
  const int64_t res = 1ll << D;
  const double h = 1.0 / (double)res;
  double s[3] = {xdiv(px, h), xdiv(py, h), xdiv(pz, h)};
  uint32_t o[3][2];
  double b[3][2];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    int64_t f = sat_i64(floor(s[a]));
    int64_t lo = f - 1, hi = f;
    lo = lo < 0 ? 0 : (lo > res - 1 ? res - 1 : lo);
    hi = hi < 0 ? 0 : (hi > res - 1 ? res - 1 : hi);
    o[a][0] = (uint32_t)lo;
    o[a][1] = (uint32_t)hi;
    b[a][0] = bspline1(xsub(s[a], (double)o[a][0]));
    b[a][1] = bspline1(xsub(s[a], (double)o[a][1]));
  }
  double v = 0.0;
  for (int i = 0; i < 2; ++i) {
    if (b[0][i] == 0.0) continue;
    for (int j = 0; j < 2; ++j) {
      if (b[1][j] == 0.0) continue;
      for (int k = 0; k < 2; ++k) {
        if (b[2][k] == 0.0) continue;
        v = xadd(v, xmul(xmul(xmul(x[morton3(o[0][i], o[1][j], o[2][k])], b[0][i]), b[1][j]), b[2][k]));
      }
    }
  }
  return v;
}

// evaluate() at the integer grid position (kx,ky,kz) in [0,res]^3: the term of node k-1
// per axis, repeated twice at k = res, absent at k = 0; v accumulates the repeats.
__device__ __forceinline__ double corner_value(const double* __restrict__ x, int res, int kx, int ky, int kz) {
  int mx = kx == 0 ? 0 : (kx == res ? 2 : 1);
  int my = ky == 0 ? 0 : (ky == res ? 2 : 1);
  int mz = kz == 0 ? 0 : (kz == res ? 2 : 1);
  int m = mx * my * mz;
  if (m == 0) return 0.0;
  double s = x[morton3(kx == res ? res - 1 : kx - 1, ky == res ? res - 1 : ky - 1, kz == res ? res - 1 : kz - 1)];
  double v = 0.0;
  for (int i = 0; i < m; ++i) v = xadd(v, s);
  return v;
}

// Degree-2 coefficients come in Morton order (as every grid vector of the API) or, inside the
// reconstruction, in the natural order of the degree-2 solver (x + res (y + res z)). The extraction
// templates take DEG = 1 (the crate's basis), 2 (quadratic, Morton order) or 3 (quadratic, natural
// order); the arithmetic of 2 and 3 is the same.
template <bool NAT>
__device__ __forceinline__ uint64_t node_index(uint32_t x, uint32_t y, uint32_t z, uint32_t D) {
  return NAT ? (uint64_t)x + ((uint64_t)y << D) + ((uint64_t)z << (2 * D)) : (uint64_t)morton3(x, y, z);
}

// Degree-2 evaluation (the extension's quadratic node functions): per axis s = u / h, c = floor(s),
// t = s - c, weights (1-t)^2/2, (-2t^2 + 2t + 1)/2, t^2/2 of nodes c-1, c, c+1; nodes outside the
// grid are skipped; terms summed z-major, then y, then x, as ((x_j b_x) b_y) b_z.
template <bool NAT>
__device__ double eval_fem2(const double* __restrict__ x, uint32_t D, double px, double py, double pz) {
  const int64_t res = 1ll << D;
  const double h = 1.0 / (double)res;
  const double u[3] = {px, py, pz};
  int64_t c[3];
  double b[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double s = xdiv(u[a], h);
    c[a] = sat_i64(floor(s));
    const double t = xsub(s, (double)c[a]);
    const double omt = xsub(1.0, t);
    b[a][0] = xmul(xmul(0.5, omt), omt);
    b[a][1] = xmul(0.5, xadd(xadd(xmul(xmul(-2.0, t), t), xmul(2.0, t)), 1.0));
    b[a][2] = xmul(xmul(0.5, t), t);
  }
  double v = 0.0;
  for (int k = 0; k < 3; ++k) {
    const int64_t z = c[2] + k - 1;
    if (z < 0 || z >= res) continue;
    for (int j = 0; j < 3; ++j) {
      const int64_t y = c[1] + j - 1;
      if (y < 0 || y >= res) continue;
      for (int i = 0; i < 3; ++i) {
        const int64_t xx = c[0] + i - 1;
        if (xx < 0 || xx >= res) continue;
        v = xadd(v, xmul(xmul(xmul(x[node_index<NAT>((uint32_t)xx, (uint32_t)y, (uint32_t)z, D)], b[0][i]), b[1][j]),
                         b[2][k]));
      }
    }
  }
  return v;
}

// eval_fem2 at the integer grid position (kx,ky,kz): t = 0 on every axis, so the weights are
// 1/2, 1/2, 0 for nodes k-1, k, k+1; the zero-weight terms add +-0 and are left out (the sum
// never holds -0), which keeps the result identical.
template <bool NAT>
__device__ __forceinline__ double corner_value2(const double* __restrict__ x, uint32_t D, int kx, int ky, int kz) {
  const int res = 1 << D;
  double v = 0.0;
#pragma unroll
  for (int dz = -1; dz <= 0; ++dz) {
    const int z = kz + dz;
    if (z < 0 || z >= res) continue;
#pragma unroll
    for (int dy = -1; dy <= 0; ++dy) {
      const int y = ky + dy;
      if (y < 0 || y >= res) continue;
#pragma unroll
      for (int dx = -1; dx <= 0; ++dx) {
        const int xx = kx + dx;
        if (xx < 0 || xx >= res) continue;
        v = xadd(v, xmul(xmul(xmul(x[node_index<NAT>((uint32_t)xx, (uint32_t)y, (uint32_t)z, D)], 0.5), 0.5), 0.5));
      }
    }
  }
  return v;
}

template <int DEG>
__device__ __forceinline__ double eval_deg(const double* __restrict__ x, uint32_t D, double px, double py, double pz) {
  return DEG >= 2 ? eval_fem2<DEG == 3>(x, D, px, py, pz) : eval_fem(x, D, px, py, pz);
}

template <int DEG>
__device__ __forceinline__ uint32_t cell_case(const double* __restrict__ x, uint32_t D, uint32_t cell, double iso,
                                              double* cv) {
  const int res = 1 << D;
  uint32_t ox, oy, oz;
  unmorton3(cell, ox, oy, oz);
  uint32_t mc = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int kx = (int)ox + c_co[k][0], ky = (int)oy + c_co[k][1], kz = (int)oz + c_co[k][2];
    cv[k] = DEG >= 2 ? corner_value2<DEG == 3>(x, D, kx, ky, kz) : corner_value(x, res, kx, ky, kz);
    if (cv[k] < iso) mc |= 1u << k;
  }
  return mc;
}

// ------------------------------------------------------------------ iso value
// Per-point evaluate, then a deterministic compensated (Neumaier) sum.
template <int DEG>
__global__ void k_eval_points(const double* __restrict__ x, uint32_t D, const double* __restrict__ pts,
                              uint64_t stride_pt, uint64_t stride_axis, uint64_t n, double* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = eval_deg<DEG>(x, D, pts[i * stride_pt], pts[i * stride_pt + stride_axis],
                           pts[i * stride_pt + 2 * stride_axis]);
}

struct Neu {
  double s, c;
};
__device__ __forceinline__ Neu neu_add(Neu a, double v) {
  double t = a.s + v;
  if (fabs(a.s) >= fabs(v)) a.c += (a.s - t) + v;
  else a.c += (v - t) + a.s;
  a.s = t;
  return a;
}

template <int DEG>
__global__ void k_iso_partial(const double* __restrict__ x, uint32_t D, const double* __restrict__ upos, uint64_t P,
                              double* __restrict__ part) {
  Neu acc{0.0, 0.0};
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < P; i += (uint64_t)gridDim.x * blockDim.x)
    acc = neu_add(acc, eval_deg<DEG>(x, D, upos[i], upos[P + i], upos[2 * P + i]));
  __shared__ double ss[kThreads], sc[kThreads];
  ss[threadIdx.x] = acc.s;
  sc[threadIdx.x] = acc.c;
  __syncthreads();
  if (threadIdx.x == 0) {
    Neu t{0.0, 0.0};
    for (int i = 0; i < kThreads; ++i) {
      t = neu_add(t, ss[i]);
      t = neu_add(t, sc[i]);
    }
    part[2 * blockIdx.x] = t.s;
    part[2 * blockIdx.x + 1] = t.c;
  }
}

__global__ void k_iso_final(const double* __restrict__ part, int nb, double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  Neu t{0.0, 0.0};
  for (int i = 0; i < nb; ++i) {
    t = neu_add(t, part[2 * i]);
    t = neu_add(t, part[2 * i + 1]);
  }
  out[0] = t.s + t.c;
}

// ------------------------------------------------------------------ marching cubes
template <int DEG>
__global__ void k_mc_count(const double* __restrict__ x, uint32_t D, double iso, uint32_t* __restrict__ blockcnt) {
  const uint64_t n = 1ull << (3 * D);
  uint64_t cell = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  int active = 0;
  if (cell < n) {
    double cv[8];
    uint32_t mc = cell_case<DEG>(x, D, (uint32_t)cell, iso, cv);
    active = (mc != 0u && mc != 255u);
  }
  typedef cub::BlockReduce<int, kThreads> BR;
  __shared__ typename BR::TempStorage tmp;
  int tot = BR(tmp).Sum(active);
  if (threadIdx.x == 0) blockcnt[blockIdx.x] = (uint32_t)tot;
}

template <int DEG>
__global__ void k_mc_compact(const double* __restrict__ x, uint32_t D, double iso, const uint32_t* __restrict__ blockoff,
                             uint32_t* __restrict__ acell, uint8_t* __restrict__ acase, uint32_t* __restrict__ nedge,
                             uint32_t* __restrict__ ntri) {
  const uint64_t n = 1ull << (3 * D);
  uint64_t cell = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  uint32_t mc = 0;
  int active = 0;
  if (cell < n) {
    double cv[8];
    mc = cell_case<DEG>(x, D, (uint32_t)cell, iso, cv);
    active = (mc != 0u && mc != 255u);
  }
  typedef cub::BlockScan<int, kThreads> BS;
  __shared__ typename BS::TempStorage tmp;
  int off;
  BS(tmp).ExclusiveSum(active, off);
  if (active) {
    uint32_t a = blockoff[blockIdx.x] + (uint32_t)off;
    acell[a] = (uint32_t)cell;
    acase[a] = (uint8_t)mc;
    nedge[a] = __popc(edge_mask(mc));
    ntri[a] = PR_MC_NTRI[mc];
  }
}

// Vertex slots: position exactly as src/fem_tree.rs:613-624, key as :625
template <int DEG>
__global__ void k_mc_vertices(const double* __restrict__ x, uint32_t D, double iso, const uint32_t* __restrict__ acell,
                              uint64_t A, const uint32_t* __restrict__ eoff, double* __restrict__ pos,
                              uint64_t* __restrict__ k1, uint32_t* __restrict__ k2, uint32_t* __restrict__ slot_id,
                              uint64_t E, int* __restrict__ err) {
  const int res = 1 << D;
  const double w = 1.0 / (double)res;  // (max_res >> d) as f64 / max_res as f64
  for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < A; a += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t cell = acell[a];
    double cv[8];
    uint32_t mc = cell_case<DEG>(x, D, cell, iso, cv);
    uint32_t em = edge_mask(mc);
    uint32_t ox, oy, oz;
    unmorton3(cell, ox, oy, oz);
    const int off[3] = {(int)ox, (int)oy, (int)oz};
    uint32_t sl = eoff[a];
    for (int e = 0; e < 12; ++e) {
      if (!((em >> e) & 1u)) continue;
      int ia = c_ev[e][0], ib = c_ev[e][1];
      double dv = xsub(cv[ib], cv[ia]);
      double t = fabs(dv) < 1e-15 ? 0.5 : xdiv(xsub(iso, cv[ia]), dv);
      uint64_t key[3];
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) {
        double base = xmul((double)(uint64_t)(off[ax] + c_co[ia][ax]), w);
        double d = (double)(c_co[ib][ax] - c_co[ia][ax]);
        double p = xadd(base, xmul(xmul(t, d), w));
        pos[(uint64_t)ax * E + sl] = p;
        key[ax] = sat_u64(xmul(p, 1e9));
      }
      if (key[0] >= (1ull << 30) || key[1] >= (1ull << 30) || key[2] >= (1ull << 30)) atomicOr(err, 1);
      k1[sl] = (key[0] << 30) | (key[1] & ((1ull << 30) - 1));
      k2[sl] = (uint32_t)(key[2] & ((1u << 30) - 1));
      slot_id[sl] = sl;
      ++sl;
    }
  }
}

// head[i] = sorted position i starts a run of equal keys
__global__ void k_mc_heads(const uint64_t* __restrict__ k1s, const uint32_t* __restrict__ k2s,
                           const uint32_t* __restrict__ slots, uint64_t E, uint32_t* __restrict__ repflag,
                           uint32_t* __restrict__ headpos) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < E; i += (uint64_t)gridDim.x * blockDim.x) {
    bool head = (i == 0) || k1s[i] != k1s[i - 1] || k2s[i] != k2s[i - 1];
    repflag[slots[i]] = head ? 1u : 0u;
    headpos[i] = head ? (uint32_t)i : 0u;
  }
}

// after an inclusive max-scan, headpos[i] = start of i's run
__global__ void k_mc_assign(const uint32_t* __restrict__ slots, const uint32_t* __restrict__ headpos, uint64_t E,
                            const uint32_t* __restrict__ vid_rep, uint32_t* __restrict__ vid) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < E; i += (uint64_t)gridDim.x * blockDim.x)
    vid[slots[i]] = vid_rep[slots[headpos[i]]];
}

struct Mat16 {
  double m[16];
};

__global__ void k_mc_emit_vertices(const double* __restrict__ pos, uint64_t E, const uint32_t* __restrict__ repflag,
                                   const uint32_t* __restrict__ vid_rep, int transform, Mat16 Mi,
                                   double* __restrict__ verts) {
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < E; s += (uint64_t)gridDim.x * blockDim.x) {
    if (!repflag[s]) continue;
    double p[3] = {pos[s], pos[E + s], pos[2 * E + s]};
    uint64_t v = vid_rep[s];
    if (transform) {
      // Mat4::transform_point (src/geometry.rs:256-262) with the inverse transform
#pragma unroll
      for (int r = 0; r < 3; ++r)
        verts[3 * v + r] =
            xadd(xadd(xadd(xmul(Mi.m[r], p[0]), xmul(Mi.m[4 + r], p[1])), xmul(Mi.m[8 + r], p[2])), Mi.m[12 + r]);
    } else {
#pragma unroll
      for (int r = 0; r < 3; ++r) verts[3 * v + r] = p[r];
    }
  }
}

__global__ void k_mc_emit_tris(const uint8_t* __restrict__ acase, uint64_t A, const uint32_t* __restrict__ eoff,
                               const uint32_t* __restrict__ toff, const uint32_t* __restrict__ vid,
                               uint64_t* __restrict__ tris) {
  for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < A; a += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t mc = acase[a];
    uint32_t em = edge_mask(mc);
    uint64_t packed = PR_MC_TRIS[mc];
    uint32_t nt = PR_MC_NTRI[mc];
    uint64_t t0 = toff[a];
    uint32_t e0 = eoff[a];
    for (uint32_t i = 0; i < 3 * nt; ++i) {
      uint32_t e = (uint32_t)((packed >> (4 * i)) & 15ull);
      uint32_t rank = __popc(em & ((1u << e) - 1u));
      tris[3 * t0 + i] = vid[e0 + rank];
    }
  }
}

}  // namespace

// ------------------------------------------------------------------ block-tiled classification (depth >= 4)
// A CTA classifies the 16^3 cells of one Morton block.  Cell c has corners at grid
// positions c + co[k]; the corner value is node (position - 1) per axis, so the CTA needs
// nodes [-1, 15]^3 of its block: the block's own 16^3 nodes plus the low layer from the
// neighbour blocks (zeros outside the domain, matching the crate's empty evaluation at 0).
constexpr int MCW = 17;  // node tile width, tile coordinate = node local + 1

__device__ __forceinline__ uint32_t sp4(uint32_t v) {
  return (v & 1u) | ((v & 2u) << 2) | ((v & 4u) << 4) | ((v & 8u) << 6);
}

__device__ void mc_load_tile(double* tile, const double* __restrict__ x, uint32_t blk, int res) {
  const int t = threadIdx.x;
  uint32_t bx, by, bz;
  unmorton3(blk, bx, by, bz);
  const uint64_t base = (uint64_t)blk << 12;
  for (int i = t; i < 4096; i += blockDim.x) {
    uint32_t lx, ly, lz;
    unmorton3((uint32_t)i, lx, ly, lz);
    tile[((lz + 1) * MCW + (ly + 1)) * MCW + (lx + 1)] = __ldg(x + base + i);
  }
  // low layer: positions with a local coordinate -1 (817 of them)
  const int nba = res >> 4;
  for (int i = t; i < 817; i += blockDim.x) {
    int lx, ly, lz;
    if (i < 289) { lx = -1; ly = i % 17 - 1; lz = i / 17 - 1; }
    else if (i < 561) { const int u = i - 289; lx = u % 16; ly = -1; lz = u / 16 - 1; }
    else { const int u = i - 561; lx = u % 16; ly = u / 16; lz = -1; }
    const int nx = (int)bx + (lx < 0 ? -1 : 0), ny = (int)by + (ly < 0 ? -1 : 0), nz = (int)bz + (lz < 0 ? -1 : 0);
    double v = 0.0;
    if (nx >= 0 && ny >= 0 && nz >= 0 && nx < nba && ny < nba && nz < nba) {
      const uint32_t nb = morton3((uint32_t)nx, (uint32_t)ny, (uint32_t)nz) << 12;
      v = __ldg(x + nb + (sp4((uint32_t)(lx & 15)) | (sp4((uint32_t)(ly & 15)) << 1) | (sp4((uint32_t)(lz & 15)) << 2)));
    }
    tile[((lz + 1) * MCW + (ly + 1)) * MCW + (lx + 1)] = v;
  }
}

// Inside/outside bits of the tile's 17^3 corner positions, one 17-bit word per (y, z) row:
// bit tx of row (ty, tz) is (corner value < iso) for grid position (o + t).  The value at a grid
// position equal to res on k axes is the node value added 2^k times in sequence, like the crate's
// evaluate() at the top boundary.  Every cell then reads 4 words instead of 8 doubles.
__device__ __forceinline__ void mc_build_masks(const double* tile, uint32_t* mask, int ox, int oy, int oz, int res,
                                               double iso) {
  for (int r = threadIdx.x; r < MCW * MCW; r += blockDim.x) {
    const int ty = r % MCW, tz = r / MCW;
    const int myz = ((oy + ty == res) ? 2 : 1) * ((oz + tz == res) ? 2 : 1);
    const double* row = tile + (tz * MCW + ty) * MCW;
    uint32_t m = 0;
#pragma unroll
    for (int tx = 0; tx < MCW; ++tx) {
      const double s = row[tx];
      const int mult = myz * ((ox + tx == res) ? 2 : 1);
      double v = s;
      for (int i = 1; i < mult; ++i) v = xadd(v, s);
      m |= (uint32_t)(v < iso) << tx;
    }
    mask[r] = m;
  }
}
// Degree 2: the corner value at grid position p is the sum over the nodes p-1, p per axis of
// ((x 1/2) 1/2) 1/2, z-major, then y, then x (corner_value2).  The CTA stages the terms
// ((x 1/2) 1/2) 1/2 of nodes [-1, 16]^3 of its block (the same products, formed once per node;
// zeros outside the domain, which add +0 like the skipped terms).
constexpr int MCW2 = 18;  // node tile width, tile coordinate = node local + 1

__device__ __forceinline__ double mc_term2(double v) { return xmul(xmul(xmul(v, 0.5), 0.5), 0.5); }

template <bool NAT>
__device__ void mc_load_tile2(double* tile, const double* __restrict__ x, uint32_t blk, int res) {
  uint32_t bx, by, bz;
  unmorton3(blk, bx, by, bz);
  if (NAT) {  // natural order: the tile's rows are contiguous in memory (18 values per row)
    const uint32_t D = 31 - __clz(res);
    for (int i = threadIdx.x; i < MCW2 * MCW2 * MCW2; i += blockDim.x) {
      const int tx = i % MCW2, ty = (i / MCW2) % MCW2, tz = i / (MCW2 * MCW2);
      const int gx = (int)bx * 16 + tx - 1, gy = (int)by * 16 + ty - 1, gz = (int)bz * 16 + tz - 1;
      double v = 0.0;
      if (gx >= 0 && gy >= 0 && gz >= 0 && gx < res && gy < res && gz < res)
        v = mc_term2(__ldg(x + node_index<true>((uint32_t)gx, (uint32_t)gy, (uint32_t)gz, D)));
      tile[i] = v;
    }
    return;
  }
  const uint64_t base = (uint64_t)blk << 12;
  for (int i = threadIdx.x; i < 4096; i += blockDim.x) {
    uint32_t lx, ly, lz;
    unmorton3((uint32_t)i, lx, ly, lz);
    tile[((lz + 1) * MCW2 + (ly + 1)) * MCW2 + (lx + 1)] = mc_term2(__ldg(x + base + i));
  }
  // the shell, 18^3 - 16^3 = 1736 entries: the z faces (2 x 18 x 18), then the y faces of the
  // inner z range (2 x 16 x 18), then the x faces of the inner y and z ranges (2 x 16 x 16)
  for (int i = threadIdx.x; i < 1736; i += blockDim.x) {
    int tx, ty, tz;
    if (i < 648) {
      const int r = i % 324;
      tz = i < 324 ? 0 : 17;
      ty = r / 18;
      tx = r % 18;
    } else if (i < 1224) {
      const int j = i - 648, r = j % 288;
      ty = j < 288 ? 0 : 17;
      tz = 1 + r / 18;
      tx = r % 18;
    } else {
      const int j = i - 1224, r = j % 256;
      tx = j < 256 ? 0 : 17;
      tz = 1 + r / 16;
      ty = 1 + r % 16;
    }
    const int gx = (int)bx * 16 + tx - 1, gy = (int)by * 16 + ty - 1, gz = (int)bz * 16 + tz - 1;
    double v = 0.0;
    if (gx >= 0 && gy >= 0 && gz >= 0 && gx < res && gy < res && gz < res)
      v = mc_term2(__ldg(x + morton3((uint32_t)gx, (uint32_t)gy, (uint32_t)gz)));
    tile[(tz * MCW2 + ty) * MCW2 + tx] = v;
  }
}

__device__ __forceinline__ void mc_build_masks2(const double* tile, uint32_t* mask, double iso) {
  for (int r = threadIdx.x; r < MCW * MCW; r += blockDim.x) {
    const int ty = r % MCW, tz = r / MCW;
    uint32_t m = 0;
    for (int tx = 0; tx < MCW; ++tx) {
      double v = 0.0;
#pragma unroll
      for (int dz = 0; dz < 2; ++dz)
#pragma unroll
        for (int dy = 0; dy < 2; ++dy)
#pragma unroll
          for (int dx = 0; dx < 2; ++dx) v = xadd(v, tile[((tz + dz) * MCW2 + ty + dy) * MCW2 + tx + dx]);
      m |= (uint32_t)(v < iso) << tx;
    }
    mask[r] = m;
  }
}

template <int DEG>
__device__ __forceinline__ void mc_block_masks(double* tile, uint32_t* mask, const double* __restrict__ x,
                                               uint32_t blk, int res, double iso) {
  uint32_t bx, by, bz;
  unmorton3(blk, bx, by, bz);
  if (DEG >= 2) {
    mc_load_tile2<DEG == 3>(tile, x, blk, res);
    __syncthreads();
    mc_build_masks2(tile, mask, iso);
  } else {
    mc_load_tile(tile, x, blk, res);
    __syncthreads();
    mc_build_masks(tile, mask, bx * 16, by * 16, bz * 16, res, iso);
  }
}

// case of local cell (lx, ly, lz) from the row masks (corner order of c_co)
__device__ __forceinline__ uint32_t mc_mask_case(const uint32_t* mask, int lx, int ly, int lz) {
  const uint32_t m00 = mask[lz * MCW + ly] >> lx, m10 = mask[lz * MCW + ly + 1] >> lx;
  const uint32_t m01 = mask[(lz + 1) * MCW + ly] >> lx, m11 = mask[(lz + 1) * MCW + ly + 1] >> lx;
  return (m00 & 1u) | ((m00 >> 1) & 1u) << 1 | ((m10 >> 1) & 1u) << 2 | (m10 & 1u) << 3 | (m01 & 1u) << 4 |
         ((m01 >> 1) & 1u) << 5 | ((m11 >> 1) & 1u) << 6 | (m11 & 1u) << 7;
}

template <int DEG>
__global__ void __launch_bounds__(256) k_mc_block_count(const double* __restrict__ x, uint32_t D, double iso,
                                                        uint32_t* __restrict__ blockcnt) {
  __shared__ double tile[DEG >= 2 ? MCW2 * MCW2 * MCW2 : MCW * MCW * MCW];
  __shared__ uint32_t mask[MCW * MCW];
  const int res = 1 << D;
  const uint32_t blk = blockIdx.x;
  mc_block_masks<DEG>(tile, mask, x, blk, res, iso);
  __syncthreads();
  // thread = one x row of 16 cells
  const int ly = threadIdx.x & 15, lz = threadIdx.x >> 4;
  int cnt = 0;
#pragma unroll 4
  for (int lx = 0; lx < 16; ++lx) {
    const uint32_t mc = mc_mask_case(mask, lx, ly, lz);
    cnt += (mc != 0u && mc != 255u);
  }
  typedef cub::BlockReduce<int, 256> BR;
  __shared__ typename BR::TempStorage tmp;
  const int tot = BR(tmp).Sum(cnt);
  if (threadIdx.x == 0) blockcnt[blk] = (uint32_t)tot;
}

// active blocks only (list from a compaction of blockcnt > 0); cells written in Morton order
template <int DEG>
__global__ void __launch_bounds__(256) k_mc_block_emit(const double* __restrict__ x, uint32_t D, double iso,
                                                       const uint32_t* __restrict__ ablk,
                                                       const uint32_t* __restrict__ blockoff,
                                                       uint32_t* __restrict__ acell, uint8_t* __restrict__ acase,
                                                       uint32_t* __restrict__ nedge, uint32_t* __restrict__ ntri) {
  __shared__ double tile[DEG >= 2 ? MCW2 * MCW2 * MCW2 : MCW * MCW * MCW];
  __shared__ uint32_t mask[MCW * MCW];
  const int res = 1 << D;
  const uint32_t blk = ablk[blockIdx.x];
  mc_block_masks<DEG>(tile, mask, x, blk, res, iso);
  __syncthreads();
  typedef cub::BlockScan<int, 256> BS;
  __shared__ typename BS::TempStorage tmp;
  uint32_t running = blockoff[blk];
  for (int chunk = 0; chunk < 16; ++chunk) {
    const int i = chunk * 256 + threadIdx.x;  // Morton-local cell index
    uint32_t lx, ly, lz;
    unmorton3((uint32_t)i, lx, ly, lz);
    const uint32_t mc = mc_mask_case(mask, (int)lx, (int)ly, (int)lz);
    const int active = (mc != 0u && mc != 255u);
    int off, tot;
    BS(tmp).ExclusiveSum(active, off, tot);
    if (active) {
      const uint32_t a = running + (uint32_t)off;
      acell[a] = (blk << 12) | (uint32_t)i;
      acase[a] = (uint8_t)mc;
      nedge[a] = __popc(edge_mask(mc));
      ntri[a] = PR_MC_NTRI[mc];
    }
    running += (uint32_t)tot;
    __syncthreads();  // temp storage reuse
  }
}

__global__ void k_flags_nonzero(const uint32_t* __restrict__ cnt, uint32_t n, uint32_t* __restrict__ flag) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) flag[i] = cnt[i] != 0;
}
__global__ void k_scatter_ids(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ pos, uint32_t n,
                              uint32_t* __restrict__ ids) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (flag[i]) ids[pos[i]] = i;
}

// ====================================================================== host stages
namespace {
__global__ void k_gather_u64(const uint64_t* __restrict__ v, const uint32_t* __restrict__ perm, uint64_t E,
                             uint64_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < E; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = v[perm[i]];
}
__global__ void k_gather_u32(const uint32_t* __restrict__ v, const uint32_t* __restrict__ perm, uint64_t E,
                             uint32_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < E; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = v[perm[i]];
}
}  // namespace

void mc_gather_u64(cudaStream_t s, const uint64_t* v, const uint32_t* perm, uint64_t E, uint64_t* out) {
  k_gather_u64<<<grid_for(E), kThreads, 0, s>>>(v, perm, E, out);
  PR_CHECK_LAUNCH();
}
void mc_gather_u32(cudaStream_t s, const uint32_t* v, const uint32_t* perm, uint64_t E, uint32_t* out) {
  k_gather_u32<<<grid_for(E), kThreads, 0, s>>>(v, perm, E, out);
  PR_CHECK_LAUNCH();
}

struct MaxOp {
  __device__ __forceinline__ uint32_t operator()(uint32_t a, uint32_t b) const { return a > b ? a : b; }
};
void evaluate_points(pr_context* c, uint32_t D, const double* d_x64, const double* d_pts, uint64_t stride,
                     uint64_t n, double* d_out, int degree) {
  if (n == 0) return;
  if (degree == 3) k_eval_points<3><<<grid_for(n), kThreads, 0, c->stream>>>(d_x64, D, d_pts, stride, 1, n, d_out);
  else if (degree == 2) k_eval_points<2><<<grid_for(n), kThreads, 0, c->stream>>>(d_x64, D, d_pts, stride, 1, n, d_out);
  else k_eval_points<1><<<grid_for(n), kThreads, 0, c->stream>>>(d_x64, D, d_pts, stride, 1, n, d_out);
  PR_CHECK_LAUNCH();
}

double stage_iso(pr_context* c, const double* d_x64, bool natural) {
  const uint64_t P = c->P;
  int nb = (int)std::min<uint64_t>(kDotBlocks, (P + kThreads - 1) / kThreads);
  if (nb < 1) nb = 1;
  double* part = c->buf<double>("iso_part", 2 * (size_t)nb);
  double* out = c->buf<double>("iso_out", 1);
  const double* up = c->get<double>("upos");
  if (c->degree == 2 && natural) k_iso_partial<3><<<nb, kThreads, 0, c->stream>>>(d_x64, c->D, up, P, part);
  else if (c->degree == 2) k_iso_partial<2><<<nb, kThreads, 0, c->stream>>>(d_x64, c->D, up, P, part);
  else k_iso_partial<1><<<nb, kThreads, 0, c->stream>>>(d_x64, c->D, up, P, part);
  PR_CHECK_LAUNCH();
  k_iso_final<<<1, 32, 0, c->stream>>>(part, nb, out);
  PR_CHECK_LAUNCH();
  double sum = 0.0;
  PR_CUDA(cudaMemcpyAsync(&sum, out, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  c->sync();
  return sum / (double)P;
}

void stage_extract(pr_context* c, uint32_t D, const double* x, double iso, bool back_transform, int degree,
                   bool natural) {
  const uint64_t n = 1ull << (3 * D);
  cudaStream_t s = c->stream;
  c->nv = c->nt = 0;
  c->have_mesh = true;
  uint64_t A = 0;
  uint32_t *acell, *nedge, *ntri, *eoff, *toff;
  uint8_t* acase;
  size_t tb = 0;
  void* tmp = nullptr;
  if (D >= 4) {
    // 16^3 cell blocks: count per block, then emit the active blocks only
    const uint32_t nblk = 1u << (3 * (D - 4));
    uint32_t* blockcnt = c->buf<uint32_t>("mc_blockcnt", (size_t)nblk + 1);
    uint32_t* blockoff = c->buf<uint32_t>("mc_blockoff", (size_t)nblk + 1);
    uint32_t* flag = c->buf<uint32_t>("mc_flag", (size_t)nblk + 1);
    uint32_t* fpos = c->buf<uint32_t>("mc_fpos", (size_t)nblk + 1);
    uint32_t* ablk = c->buf<uint32_t>("mc_ablk", (size_t)nblk);
    if (degree == 2 && natural) k_mc_block_count<3><<<nblk, 256, 0, s>>>(x, D, iso, blockcnt);
    else if (degree == 2) k_mc_block_count<2><<<nblk, 256, 0, s>>>(x, D, iso, blockcnt);
    else k_mc_block_count<1><<<nblk, 256, 0, s>>>(x, D, iso, blockcnt);
    PR_CHECK_LAUNCH();
    PR_CUDA(cudaMemsetAsync(blockcnt + nblk, 0, sizeof(uint32_t), s));
    k_flags_nonzero<<<grid_for(nblk + 1), kThreads, 0, s>>>(blockcnt, nblk + 1, flag);
    PR_CHECK_LAUNCH();
    PR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, blockcnt, blockoff, (int64_t)nblk + 1, s));
    tmp = c->buf<char>("cub_tmp", tb);
    PR_COUNT_PRIMITIVE();
    PR_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, blockcnt, blockoff, (int64_t)nblk + 1, s));
    PR_COUNT_PRIMITIVE();
    PR_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, flag, fpos, (int64_t)nblk + 1, s));
    k_scatter_ids<<<grid_for(nblk), kThreads, 0, s>>>(flag, fpos, nblk, ablk);
    PR_CHECK_LAUNCH();
    uint32_t hv[2] = {0, 0};
    PR_CUDA(cudaMemcpyAsync(&hv[0], blockoff + nblk, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    PR_CUDA(cudaMemcpyAsync(&hv[1], fpos + nblk, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    c->sync();
    A = hv[0];
    if (A == 0) return;
    acell = c->buf<uint32_t>("mc_acell", A);
    acase = c->buf<uint8_t>("mc_acase", A);
    nedge = c->buf<uint32_t>("mc_nedge", A + 1);
    ntri = c->buf<uint32_t>("mc_ntri", A + 1);
    if (degree == 2 && natural)
      k_mc_block_emit<3><<<hv[1], 256, 0, s>>>(x, D, iso, ablk, blockoff, acell, acase, nedge, ntri);
    else if (degree == 2)
      k_mc_block_emit<2><<<hv[1], 256, 0, s>>>(x, D, iso, ablk, blockoff, acell, acase, nedge, ntri);
    else k_mc_block_emit<1><<<hv[1], 256, 0, s>>>(x, D, iso, ablk, blockoff, acell, acase, nedge, ntri);
    PR_CHECK_LAUNCH();
  } else {
    const unsigned nblk = (unsigned)((n + kThreads - 1) / kThreads);
    uint32_t* blockcnt = c->buf<uint32_t>("mc_blockcnt", (size_t)nblk + 1);
    uint32_t* blockoff = c->buf<uint32_t>("mc_blockoff", (size_t)nblk + 1);
    if (degree == 2 && natural) k_mc_count<3><<<nblk, kThreads, 0, s>>>(x, D, iso, blockcnt);
    else if (degree == 2) k_mc_count<2><<<nblk, kThreads, 0, s>>>(x, D, iso, blockcnt);
    else k_mc_count<1><<<nblk, kThreads, 0, s>>>(x, D, iso, blockcnt);
    PR_CHECK_LAUNCH();
    PR_CUDA(cudaMemsetAsync(blockcnt + nblk, 0, sizeof(uint32_t), s));
    PR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, blockcnt, blockoff, (int64_t)nblk + 1, s));
    tmp = c->buf<char>("cub_tmp", tb);
    PR_COUNT_PRIMITIVE();
    PR_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, blockcnt, blockoff, (int64_t)nblk + 1, s));
    uint32_t hA = 0;
    PR_CUDA(cudaMemcpyAsync(&hA, blockoff + nblk, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    c->sync();
    A = hA;
    if (A == 0) return;
    acell = c->buf<uint32_t>("mc_acell", A);
    acase = c->buf<uint8_t>("mc_acase", A);
    nedge = c->buf<uint32_t>("mc_nedge", A + 1);
    ntri = c->buf<uint32_t>("mc_ntri", A + 1);
    if (degree == 2 && natural) k_mc_compact<3><<<nblk, kThreads, 0, s>>>(x, D, iso, blockoff, acell, acase, nedge, ntri);
    else if (degree == 2) k_mc_compact<2><<<nblk, kThreads, 0, s>>>(x, D, iso, blockoff, acell, acase, nedge, ntri);
    else k_mc_compact<1><<<nblk, kThreads, 0, s>>>(x, D, iso, blockoff, acell, acase, nedge, ntri);
    PR_CHECK_LAUNCH();
  }
  eoff = c->buf<uint32_t>("mc_eoff", A + 1);
  toff = c->buf<uint32_t>("mc_toff", A + 1);
  PR_CUDA(cudaMemsetAsync(nedge + A, 0, sizeof(uint32_t), s));
  PR_CUDA(cudaMemsetAsync(ntri + A, 0, sizeof(uint32_t), s));
  tb = 0;
  PR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, nedge, eoff, (int64_t)A + 1, s));
  tmp = c->buf<char>("cub_tmp", tb);
  PR_COUNT_PRIMITIVE();
  PR_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, nedge, eoff, (int64_t)A + 1, s));
  PR_COUNT_PRIMITIVE();
  PR_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, ntri, toff, (int64_t)A + 1, s));
  uint32_t hE = 0, hT = 0;
  PR_CUDA(cudaMemcpyAsync(&hE, eoff + A, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  PR_CUDA(cudaMemcpyAsync(&hT, toff + A, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  c->sync();
  const uint64_t E = hE, NT = hT;

  double* pos = c->buf<double>("mc_pos", 3 * E);
  uint64_t* k1 = c->buf<uint64_t>("mc_k1", E);
  uint32_t* k2 = c->buf<uint32_t>("mc_k2", E);
  uint32_t* sid = c->buf<uint32_t>("mc_sid", E);
  uint64_t* k1b = c->buf<uint64_t>("mc_k1b", E);
  uint32_t* k2b = c->buf<uint32_t>("mc_k2b", E);
  uint32_t* sidb = c->buf<uint32_t>("mc_sidb", E);
  int* err = c->buf<int>("mc_err", 1);
  PR_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
  if (degree == 2 && natural)
    k_mc_vertices<3><<<grid_for(A), kThreads, 0, s>>>(x, D, iso, acell, A, eoff, pos, k1, k2, sid, E, err);
  else if (degree == 2)
    k_mc_vertices<2><<<grid_for(A), kThreads, 0, s>>>(x, D, iso, acell, A, eoff, pos, k1, k2, sid, E, err);
  else k_mc_vertices<1><<<grid_for(A), kThreads, 0, s>>>(x, D, iso, acell, A, eoff, pos, k1, k2, sid, E, err);
  PR_CHECK_LAUNCH();

  // stable LSD sort: by k2 (z key), then by k1 (x,y key); ties keep slot order
  size_t b1 = 0, b2 = 0;
  PR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b1, k2, k2b, sid, sidb, (int64_t)E, 0, 30, s));
  PR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b2, k1, k1b, sidb, sid, (int64_t)E, 0, 60, s));
  tb = std::max(b1, b2);
  tmp = c->buf<char>("cub_tmp", tb);
  PR_COUNT_PRIMITIVE();
  PR_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, k2, k2b, sid, sidb, (int64_t)E, 0, 30, s));
  // k1 in the order of the first sort
  uint64_t* k1g = c->buf<uint64_t>("mc_k1g", E);
  mc_gather_u64(s, k1, sidb, E, k1g);
  PR_COUNT_PRIMITIVE();
  PR_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, k1g, k1b, sidb, sid, (int64_t)E, 0, 60, s));
  // sorted: k1b (x,y keys), sid (slots); need the z keys in the same order
  uint32_t* k2s = c->buf<uint32_t>("mc_k2s", E);
  mc_gather_u32(s, k2, sid, E, k2s);

  uint32_t* repflag = c->buf<uint32_t>("mc_rep", E + 1);
  uint32_t* headpos = c->buf<uint32_t>("mc_head", E);
  uint32_t* vid_rep = c->buf<uint32_t>("mc_vidrep", E + 1);
  uint32_t* vid = c->buf<uint32_t>("mc_vid", E);
  k_mc_heads<<<grid_for(E), kThreads, 0, s>>>(k1b, k2s, sid, E, repflag, headpos);
  PR_CHECK_LAUNCH();
  PR_CUDA(cudaMemsetAsync(repflag + E, 0, sizeof(uint32_t), s));
  size_t b3 = 0, b4 = 0;
  PR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, b3, repflag, vid_rep, (int64_t)E + 1, s));
  uint32_t* headrun = c->buf<uint32_t>("mc_headrun", E);
  PR_CUDA(cub::DeviceScan::InclusiveScan(nullptr, b4, headpos, headrun, MaxOp(), (int64_t)E, s));
  tb = std::max(b3, b4);
  tmp = c->buf<char>("cub_tmp", tb);
  PR_COUNT_PRIMITIVE();
  PR_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, repflag, vid_rep, (int64_t)E + 1, s));
  PR_COUNT_PRIMITIVE();
  PR_CUDA(cub::DeviceScan::InclusiveScan(tmp, tb, headpos, headrun, MaxOp(), (int64_t)E, s));
  k_mc_assign<<<grid_for(E), kThreads, 0, s>>>(sid, headrun, E, vid_rep, vid);
  PR_CHECK_LAUNCH();
  uint32_t hNV = 0;
  int herr = 0;
  PR_CUDA(cudaMemcpyAsync(&hNV, vid_rep + E, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  PR_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s));
  c->sync();
  PR_REQUIRE(!herr, PR_ERR_INTERNAL, "marching cubes: vertex key outside [0, 2^30)");
  const uint64_t NV = hNV;
  double* verts = c->buf<double>("mesh_v", 3 * NV);
  uint64_t* tris = c->buf<uint64_t>("mesh_t", 3 * NT);
  Mat16 mi;
  for (int k = 0; k < 16; ++k) mi.m[k] = c->Minv[k];
  k_mc_emit_vertices<<<grid_for(E), kThreads, 0, s>>>(pos, E, repflag, vid_rep, back_transform ? 1 : 0, mi, verts);
  PR_CHECK_LAUNCH();
  k_mc_emit_tris<<<grid_for(A), kThreads, 0, s>>>(acase, A, eoff, toff, vid, tris);
  PR_CHECK_LAUNCH();
  c->nv = NV;
  c->nt = NT;
}


}  // namespace pr

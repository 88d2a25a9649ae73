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

__device__ __forceinline__ uint32_t cell_case(const double* __restrict__ x, int res, uint32_t cell, double iso,
                                              double* cv) {
  uint32_t ox, oy, oz;
  unmorton3(cell, ox, oy, oz);
  uint32_t mc = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    cv[k] = corner_value(x, res, (int)ox + c_co[k][0], (int)oy + c_co[k][1], (int)oz + c_co[k][2]);
    if (cv[k] < iso) mc |= 1u << k;
  }
  return mc;
}

// ------------------------------------------------------------------ iso value
// Per-point evaluate, then a deterministic compensated (Neumaier) sum.
__global__ void k_eval_points(const double* __restrict__ x, uint32_t D, const double* __restrict__ pts,
                              uint64_t stride_pt, uint64_t stride_axis, uint64_t n, double* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = eval_fem(x, D, pts[i * stride_pt], pts[i * stride_pt + stride_axis], pts[i * stride_pt + 2 * stride_axis]);
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

__global__ void k_iso_partial(const double* __restrict__ x, uint32_t D, const double* __restrict__ upos, uint64_t P,
                              double* __restrict__ part) {
  Neu acc{0.0, 0.0};
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < P; i += (uint64_t)gridDim.x * blockDim.x)
    acc = neu_add(acc, eval_fem(x, D, upos[i], upos[P + i], upos[2 * P + i]));
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
__global__ void k_mc_count(const double* __restrict__ x, uint32_t D, double iso, uint32_t* __restrict__ blockcnt) {
  const int res = 1 << D;
  const uint64_t n = 1ull << (3 * D);
  uint64_t cell = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  int active = 0;
  if (cell < n) {
    double cv[8];
    uint32_t mc = cell_case(x, res, (uint32_t)cell, iso, cv);
    active = (mc != 0u && mc != 255u);
  }
  typedef cub::BlockReduce<int, kThreads> BR;
  __shared__ typename BR::TempStorage tmp;
  int tot = BR(tmp).Sum(active);
  if (threadIdx.x == 0) blockcnt[blockIdx.x] = (uint32_t)tot;
}

__global__ void k_mc_compact(const double* __restrict__ x, uint32_t D, double iso, const uint32_t* __restrict__ blockoff,
                             uint32_t* __restrict__ acell, uint8_t* __restrict__ acase, uint32_t* __restrict__ nedge,
                             uint32_t* __restrict__ ntri) {
  const int res = 1 << D;
  const uint64_t n = 1ull << (3 * D);
  uint64_t cell = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  uint32_t mc = 0;
  int active = 0;
  if (cell < n) {
    double cv[8];
    mc = cell_case(x, res, (uint32_t)cell, iso, cv);
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
__global__ void k_mc_vertices(const double* __restrict__ x, uint32_t D, double iso, const uint32_t* __restrict__ acell,
                              uint64_t A, const uint32_t* __restrict__ eoff, double* __restrict__ pos,
                              uint64_t* __restrict__ k1, uint32_t* __restrict__ k2, uint32_t* __restrict__ slot_id,
                              uint64_t E, int* __restrict__ err) {
  const int res = 1 << D;
  const double w = 1.0 / (double)res;  // (max_res >> d) as f64 / max_res as f64
  for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < A; a += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t cell = acell[a];
    double cv[8];
    uint32_t mc = cell_case(x, res, cell, iso, cv);
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
                     uint64_t n, double* d_out) {
  if (n == 0) return;
  k_eval_points<<<grid_for(n), kThreads, 0, c->stream>>>(d_x64, D, d_pts, stride, 1, n, d_out);
  PR_CHECK_LAUNCH();
}

double stage_iso(pr_context* c, const double* d_x64) {
  const uint64_t P = c->P;
  int nb = (int)std::min<uint64_t>(kDotBlocks, (P + kThreads - 1) / kThreads);
  if (nb < 1) nb = 1;
  double* part = c->buf<double>("iso_part", 2 * (size_t)nb);
  double* out = c->buf<double>("iso_out", 1);
  k_iso_partial<<<nb, kThreads, 0, c->stream>>>(d_x64, c->D, c->get<double>("upos"), P, part);
  PR_CHECK_LAUNCH();
  k_iso_final<<<1, 32, 0, c->stream>>>(part, nb, out);
  PR_CHECK_LAUNCH();
  double sum = 0.0;
  PR_CUDA(cudaMemcpyAsync(&sum, out, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  c->sync();
  return sum / (double)P;
}

void stage_extract(pr_context* c, uint32_t D, const double* x, double iso, bool back_transform) {
  const uint64_t n = 1ull << (3 * D);
  const unsigned nblk = (unsigned)((n + kThreads - 1) / kThreads);
  cudaStream_t s = c->stream;
  uint32_t* blockcnt = c->buf<uint32_t>("mc_blockcnt", (size_t)nblk + 1);
  uint32_t* blockoff = c->buf<uint32_t>("mc_blockoff", (size_t)nblk + 1);
  k_mc_count<<<nblk, kThreads, 0, s>>>(x, D, iso, blockcnt);
  PR_CHECK_LAUNCH();
  PR_CUDA(cudaMemsetAsync(blockcnt + nblk, 0, sizeof(uint32_t), s));
  size_t tb = 0;
  PR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, blockcnt, blockoff, (int64_t)nblk + 1, s));
  void* tmp = c->buf<char>("cub_tmp", tb);
  PR_COUNT_PRIMITIVE();
  PR_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, blockcnt, blockoff, (int64_t)nblk + 1, s));
  uint32_t hA = 0;
  PR_CUDA(cudaMemcpyAsync(&hA, blockoff + nblk, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  c->sync();
  const uint64_t A = hA;
  c->nv = c->nt = 0;
  c->have_mesh = true;
  if (A == 0) return;
  uint32_t* acell = c->buf<uint32_t>("mc_acell", A);
  uint8_t* acase = c->buf<uint8_t>("mc_acase", A);
  uint32_t* nedge = c->buf<uint32_t>("mc_nedge", A + 1);
  uint32_t* ntri = c->buf<uint32_t>("mc_ntri", A + 1);
  uint32_t* eoff = c->buf<uint32_t>("mc_eoff", A + 1);
  uint32_t* toff = c->buf<uint32_t>("mc_toff", A + 1);
  k_mc_compact<<<nblk, kThreads, 0, s>>>(x, D, iso, blockoff, acell, acase, nedge, ntri);
  PR_CHECK_LAUNCH();
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
  k_mc_vertices<<<grid_for(A), kThreads, 0, s>>>(x, D, iso, acell, A, eoff, pos, k1, k2, sid, E, err);
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

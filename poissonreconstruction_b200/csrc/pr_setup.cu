// Setup stage: bounding box + unit-cube transform, normal splat, right-hand side and the
// screening payload of the matrix-free operator.
//
// Replaces, in the reference crate:
//   bbox / unit_cube_transform / transform   src/reconstructor.rs:31-40, src/geometry.rs:256-402
//   FEMTree::{initialize, finalize}          src/fem_tree.rs:83-126 (implicit: node = Morton index)
//   FEMTree::splat_normal_field              src/fem_tree.rs:130-178
//   FEMTree::assemble_rhs                    src/fem_tree.rs:251-299
//   screening part of assemble_system        src/fem_tree.rs:199-226 (kept as per-point payload)
//
// Every FP64 quantity here is computed with the crate's operation order and without
// multiply-add contraction, so splat weights, the normal field and b equal the crate's
// values bit for bit.  Per-node sums run in input-point order because the (node, point)
// pairs are ordered by a stable radix sort of keys generated in point order.
#include <cub/cub.cuh>

#include "pr_internal.cuh"

namespace pr {

namespace {

constexpr int kThreads = 256;

inline unsigned grid_for(uint64_t n, int threads = kThreads, uint64_t cap = 1u << 20) {
  uint64_t g = (n + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (unsigned)g;
}

// ------------------------------------------------------------------ bbox
__global__ void k_bbox_partial(const double* __restrict__ pts6, uint64_t n, double* __restrict__ part,
                               int* __restrict__ bad) {
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  int nonfinite = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const double* p = pts6 + 6 * i;
#pragma unroll
    for (int k = 0; k < 6; ++k) nonfinite |= !isfinite(p[k]);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      lo[k] = fmin(lo[k], p[k]);
      hi[k] = fmax(hi[k], p[k]);
    }
  }
  __shared__ double s[6][kThreads];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    s[k][threadIdx.x] = lo[k];
    s[3 + k][threadIdx.x] = hi[k];
  }
  if (nonfinite) atomicOr(bad, 1);
  __syncthreads();
  for (int w = kThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        s[k][threadIdx.x] = fmin(s[k][threadIdx.x], s[k][threadIdx.x + w]);
        s[3 + k][threadIdx.x] = fmax(s[3 + k][threadIdx.x], s[3 + k][threadIdx.x + w]);
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 6; ++k) part[6 * blockIdx.x + k] = s[k][0];
}

// one warp: lane l folds the partials l, l + 32, ..., then the lanes fold by shuffle (min and max
// are exact, so the order does not change the result)
__global__ void k_bbox_final(const double* __restrict__ part, int nparts, double* __restrict__ out) {
  const int l = threadIdx.x;
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int b = l; b < nparts; b += 32)
    for (int k = 0; k < 3; ++k) {
      lo[k] = fmin(lo[k], part[6 * b + k]);
      hi[k] = fmax(hi[k], part[6 * b + 3 + k]);
    }
  for (int o = 16; o > 0; o >>= 1)
    for (int k = 0; k < 3; ++k) {
      lo[k] = fmin(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
      hi[k] = fmax(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
    }
  if (l == 0)
    for (int k = 0; k < 3; ++k) {
      out[k] = lo[k];
      out[3 + k] = hi[k];
    }
}

struct Mat16 {
  double m[16];  // column-major m[col*4+row], as the crate's Mat4 (src/geometry.rs:237-240)
};

// Mat4::transform_point + transform_vector + Vec3::normalize (src/reconstructor.rs:36-40)
__global__ void k_transform(const double* __restrict__ pts6, uint64_t n, Mat16 M, double* __restrict__ upos,
                            double* __restrict__ unrm, double* __restrict__ ulen) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const double* p = pts6 + 6 * i;
    double v[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      double o = xadd(xadd(xadd(xmul(M.m[r], p[0]), xmul(M.m[4 + r], p[1])), xmul(M.m[8 + r], p[2])), M.m[12 + r]);
      upos[r * n + i] = o;
      v[r] = xadd(xadd(xmul(M.m[r], p[3]), xmul(M.m[4 + r], p[4])), xmul(M.m[8 + r], p[5]));
    }
    double nn = __dsqrt_rn(xadd(xadd(xmul(v[0], v[0]), xmul(v[1], v[1])), xmul(v[2], v[2])));
#pragma unroll
    for (int r = 0; r < 3; ++r) unrm[r * n + i] = nn > 0.0 ? xdiv(v[r], nn) : 0.0;
    ulen[i] = nn;  // |M n|, for the derivative of the normalisation
  }
}

// ------------------------------------------------------------------ (node, point) pairs
// Cell and in-cell coordinate of one axis.  kTrunc: `(x / h) as isize` (screening,
// src/fem_tree.rs:207,283); otherwise `(x / h).floor() as isize` (splat, :138).
template <bool kTrunc>
__device__ __forceinline__ void cell_of(double x, double h, int64_t& c, double& t) {
  double s = xdiv(x, h);
  c = kTrunc ? sat_i64(s) : sat_i64(floor(s));
  t = xsub(s, (double)c);
}

// Validity of corner c + d on an axis: splat casts `as usize` (src/fem_tree.rs:150-153),
// screening casts `as u32` (src/fem_tree.rs:212-213) before comparing with res.
template <bool kTrunc>
__device__ __forceinline__ bool corner_ok(int64_t c, int d, uint32_t res, uint32_t& o) {
  uint64_t u = (uint64_t)c + (uint64_t)d;
  if (kTrunc) {
    o = (uint32_t)u;
    return o < res;
  }
  o = (uint32_t)u;
  return u < (uint64_t)res;
}

// keys[8p+k] = Morton index of corner k (k = dz*4 + dy*2 + dx, the crate's loop order) or
// the sentinel res^3; vals[8p+k] = 8p+k.  For the screening pairs also the basis value
// phi = bx*by*bz in FP64 and FP32.
template <bool kTrunc>
__global__ void k_pair_keys(const double* __restrict__ upos, uint64_t P, uint32_t D, uint32_t* __restrict__ keys,
                            uint32_t* __restrict__ vals, double* __restrict__ phi64, float* __restrict__ phi32,
                            unsigned long long* __restrict__ n_inside) {
  const uint32_t res = 1u << D;
  const uint32_t sentinel = 1u << (3 * D);
  const double h = 1.0 / (double)res;
  unsigned inside = 0;
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < P; p += (uint64_t)gridDim.x * blockDim.x) {
    int64_t cx, cy, cz;
    double tx, ty, tz;
    cell_of<kTrunc>(upos[p], h, cx, tx);
    cell_of<kTrunc>(upos[P + p], h, cy, ty);
    cell_of<kTrunc>(upos[2 * P + p], h, cz, tz);
    bool any = false;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      int dx = k & 1, dy = (k >> 1) & 1, dz = k >> 2;
      uint32_t ox, oy, oz;
      bool ok = corner_ok<kTrunc>(cx, dx, res, ox) & corner_ok<kTrunc>(cy, dy, res, oy) &
                corner_ok<kTrunc>(cz, dz, res, oz);
      any |= ok;
      keys[8 * p + k] = ok ? morton3(ox, oy, oz) : sentinel;
      vals[8 * p + k] = (uint32_t)(8 * p + k);
      if (phi64) {
        double bx = dx ? tx : xsub(1.0, tx);
        double by = dy ? ty : xsub(1.0, ty);
        double bz = dz ? tz : xsub(1.0, tz);
        double phi = ok ? xmul(xmul(bx, by), bz) : 0.0;
        phi64[8 * p + k] = phi;
        phi32[8 * p + k] = (float)phi;
      }
    }
    inside += any;
  }
  if (n_inside) {
    typedef cub::BlockReduce<unsigned, kThreads> BR;
    __shared__ typename BR::TempStorage tmp;
    unsigned tot = BR(tmp).Sum(inside);
    if (threadIdx.x == 0 && tot) atomicAdd(n_inside, (unsigned long long)tot);
  }
}

// Splat reduction (src/fem_tree.rs:137-177): per touched node, in point order,
// normal_field += n * w and weight += w; then v = -normal_field / weight where weight > 0.
__global__ void k_splat_reduce(const uint32_t* __restrict__ run_key, const uint32_t* __restrict__ run_off,
                               uint64_t T, const uint32_t* __restrict__ sval, const double* __restrict__ upos,
                               const double* __restrict__ unrm, uint64_t P, uint32_t D, double* __restrict__ v,
                               uint32_t* __restrict__ map) {
  const double h = 1.0 / (double)(1u << D);
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < T; t += (uint64_t)gridDim.x * blockDim.x) {
    double fx = 0.0, fy = 0.0, fz = 0.0, sw = 0.0;
    for (uint32_t e = run_off[t]; e < run_off[t + 1]; ++e) {
      uint32_t pk = sval[e];
      uint32_t p = pk >> 3, k = pk & 7u;
      int64_t c;
      double tx, ty, tz;
      cell_of<false>(upos[p], h, c, tx);
      cell_of<false>(upos[P + p], h, c, ty);
      cell_of<false>(upos[2 * P + p], h, c, tz);
      double bx = (k & 1u) ? tx : xsub(1.0, tx);
      double by = (k & 2u) ? ty : xsub(1.0, ty);
      double bz = (k & 4u) ? tz : xsub(1.0, tz);
      double w = xmul(xmul(bx, by), bz);
      fx = xadd(fx, xmul(unrm[p], w));
      fy = xadd(fy, xmul(unrm[P + p], w));
      fz = xadd(fz, xmul(unrm[2 * P + p], w));
      sw = xadd(sw, w);
    }
    if (sw > 0.0) {
      double inv = xdiv(1.0, sw);
      fx = xmul(-fx, inv);
      fy = xmul(-fy, inv);
      fz = xmul(-fz, inv);
    }
    v[t] = fx;
    v[T + t] = fy;
    v[2 * T + t] = fz;
    v[3 * T + t] = sw;
    map[run_key[t]] = (uint32_t)t;
  }
}

// 1-D constants of src/fem_tree.rs:39-41 (offset d in -1..1)
__device__ __forceinline__ double mass1(int d) { return d == 0 ? 2.0 / 3.0 : 1.0 / 6.0; }
__device__ __forceinline__ double dmass1(int d) { return d == 0 ? 0.0 : (d == 1 ? -0.5 : 0.5); }

constexpr uint32_t kEmpty = 0xffffffffu;

// Laplacian part of assemble_rhs (src/fem_tree.rs:258-274) at node i, exact order dx
// (outer), dy, dz (inner); neighbours without a touched node contribute exactly 0.
__device__ __forceinline__ double rhs_node(uint32_t i, int res, double h2, const uint32_t* __restrict__ map,
                                           const double* __restrict__ v, uint64_t T) {
  uint32_t ix, iy, iz;
  unmorton3(i, ix, iy, iz);
  double sum = 0.0;
  for (int dx = -1; dx <= 1; ++dx) {
    const int jx = (int)ix + dx;
    if (jx < 0 || jx >= res) continue;
    for (int dy = -1; dy <= 1; ++dy) {
      const int jy = (int)iy + dy;
      if (jy < 0 || jy >= res) continue;
      for (int dz = -1; dz <= 1; ++dz) {
        const int jz = (int)iz + dz;
        if (jz < 0 || jz >= res) continue;
        const uint32_t slot = map[morton3(jx, jy, jz)];
        if (slot == kEmpty) continue;
        const double vx = v[slot], vy = v[T + slot], vz = v[2 * T + slot];
        const double a = xmul(xmul(xmul(vx, dmass1(dx)), mass1(dy)), mass1(dz));
        const double bb = xmul(xmul(xmul(vy, mass1(dx)), dmass1(dy)), mass1(dz));
        const double cc = xmul(xmul(xmul(vz, mass1(dx)), mass1(dy)), dmass1(dz));
        sum = xadd(sum, xmul(h2, xadd(xadd(a, bb), cc)));
      }
    }
  }
  return sum;
}

// every node (small grids)
__global__ void k_rhs_dense(uint32_t D, const uint32_t* __restrict__ map, const double* __restrict__ v, uint64_t T,
                            double* __restrict__ b) {
  const int res = 1 << D;
  const double h = 1.0 / (double)res;
  const double h2 = xmul(h, h);
  const uint64_t n = 1ull << (3 * D);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    b[i] = rhs_node((uint32_t)i, res, h2, map, v, T);
}

// Only the 16^3 blocks that hold a touched node or border one; b is zero elsewhere.
__global__ void k_mark_rhs_blocks(const uint32_t* __restrict__ tnode, uint64_t T, uint32_t nba,
                                  uint32_t* __restrict__ flag) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < T; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t node = tnode[t];
    uint32_t bx, by, bz, lx, ly, lz;
    unmorton3(node >> 12, bx, by, bz);
    unmorton3(node & 4095u, lx, ly, lz);
    const int x0 = lx == 0 ? -1 : 0, x1 = lx == 15 ? 1 : 0;
    const int y0 = ly == 0 ? -1 : 0, y1 = ly == 15 ? 1 : 0;
    const int z0 = lz == 0 ? -1 : 0, z1 = lz == 15 ? 1 : 0;
    for (int dz = z0; dz <= z1; ++dz)
      for (int dy = y0; dy <= y1; ++dy)
        for (int dx = x0; dx <= x1; ++dx) {
          const int x = (int)bx + dx, y = (int)by + dy, z = (int)bz + dz;
          if (x < 0 || y < 0 || z < 0 || x >= (int)nba || y >= (int)nba || z >= (int)nba) continue;
          flag[morton3(x, y, z)] = 1u;
        }
  }
}

__global__ void k_list_blocks(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ pos, uint32_t n,
                              uint32_t* __restrict__ ids) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (flag[i]) ids[pos[i]] = i;
}

__global__ void __launch_bounds__(256) k_rhs_blocks(uint32_t D, const uint32_t* __restrict__ blocks,
                                                    const uint32_t* __restrict__ map, const double* __restrict__ v,
                                                    uint64_t T, double* __restrict__ b) {
  const int res = 1 << D;
  const double h = 1.0 / (double)res;
  const double h2 = xmul(h, h);
  const uint32_t base = blocks[blockIdx.x] << 12;
  for (int k = threadIdx.x; k < 4096; k += 256) b[base + k] = rhs_node(base + (uint32_t)k, res, h2, map, v, T);
}

// Screening part of assemble_rhs (src/fem_tree.rs:276-297): b[node] += wh3*0.5*bx*by*bz per
// point in input order.
__global__ void k_rhs_screen(const uint32_t* __restrict__ snode, const uint32_t* __restrict__ soff, uint64_t S,
                             const uint32_t* __restrict__ qval, const double* __restrict__ upos, uint64_t P,
                             uint32_t D, double wh3, double* __restrict__ b) {
  const double h = 1.0 / (double)(1u << D);
  const double wt = xmul(wh3, 0.5);
  for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < S; u += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t node = snode[u];
    double acc = b[node];
    for (uint32_t e = soff[u]; e < soff[u + 1]; ++e) {
      uint32_t pk = qval[e];
      uint32_t p = pk >> 3, k = pk & 7u;
      int64_t c;
      double tx, ty, tz;
      cell_of<true>(upos[p], h, c, tx);
      cell_of<true>(upos[P + p], h, c, ty);
      cell_of<true>(upos[2 * P + p], h, c, tz);
      double bx = (k & 1u) ? tx : xsub(1.0, tx);
      double by = (k & 2u) ? ty : xsub(1.0, ty);
      double bz = (k & 4u) ? tz : xsub(1.0, tz);
      acc = xadd(acc, xmul(xmul(xmul(wt, bx), by), bz));
    }
    b[node] = acc;
  }
}

__global__ void k_scatter_nf(const uint32_t* __restrict__ run_key, uint64_t T, const double* __restrict__ v,
                             double* __restrict__ nf3, double* __restrict__ w) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < T; t += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t node = run_key[t];
    nf3[3ull * node] = v[t];
    nf3[3ull * node + 1] = v[T + t];
    nf3[3ull * node + 2] = v[2 * T + t];
    w[node] = v[3 * T + t];
  }
}

}  // namespace

// Sort 8P (key, pair) entries by key (stable) and run-length encode the keys.  Outputs:
// sorted keys/vals, the distinct valid keys (`run_key`, length R) and their segment offsets
// `run_off` (R+1).  Returns R.
uint64_t sort_and_segment(pr_context* c, const std::string& tag, uint32_t* keys_in, uint32_t* vals_in, uint64_t m,
                          uint32_t D) {
  uint32_t* keys = c->buf<uint32_t>(tag + "_key", m);
  uint32_t* vals = c->buf<uint32_t>(tag + "_val", m);
  uint32_t* run_key = c->buf<uint32_t>(tag + "_runkey", m);
  uint32_t* run_cnt = c->buf<uint32_t>(tag + "_runcnt", m + 1);
  uint32_t* run_off = c->buf<uint32_t>(tag + "_runoff", m + 1);
  uint32_t* nrun = c->buf<uint32_t>("nrun", 2);
  int end_bit = (int)(3 * D + 1);
  size_t b1 = 0, b2 = 0, b3 = 0;
  PR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b1, keys_in, keys, vals_in, vals, (int64_t)m, 0, end_bit, c->stream));
  PR_CUDA(cub::DeviceRunLengthEncode::Encode(nullptr, b2, keys, run_key, run_cnt, nrun, (int64_t)m, c->stream));
  PR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, b3, run_cnt, run_off, (int64_t)(m + 1), c->stream));
  size_t tb = std::max(b1, std::max(b2, b3));
  void* tmp = c->buf<char>("cub_tmp", tb);
  PR_COUNT_PRIMITIVE();
  PR_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, keys_in, keys, vals_in, vals, (int64_t)m, 0, end_bit, c->stream));
  PR_COUNT_PRIMITIVE();
  PR_CUDA(cub::DeviceRunLengthEncode::Encode(tmp, tb, keys, run_key, run_cnt, nrun, (int64_t)m, c->stream));
  uint32_t h_nrun = 0, h_last = 0;
  PR_CUDA(cudaMemcpyAsync(&h_nrun, nrun, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
  c->sync();
  if (h_nrun > 0) {
    PR_CUDA(cudaMemcpyAsync(&h_last, run_key + (h_nrun - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
    c->sync();
  }
  uint64_t R = h_nrun;
  if (R > 0 && h_last == (1u << (3 * D))) --R;  // drop the sentinel run
  // offsets of the R valid runs: exclusive scan over counts with a zero appended
  PR_CUDA(cudaMemsetAsync(run_cnt + R, 0, sizeof(uint32_t), c->stream));
  PR_COUNT_PRIMITIVE();
  PR_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, run_cnt, run_off, (int64_t)(R + 1), c->stream));
  return R;
}

// ------------------------------------------------------------------ stage: transform
void stage_transform(pr_context* c, const double* d_pts6, uint64_t P, double scale) {
  int nb = (int)std::min<uint64_t>(kDotBlocks, (P + kThreads - 1) / kThreads);
  if (nb < 1) nb = 1;
  double* part = c->buf<double>("bbox_part", 6 * (size_t)nb);
  double* bb = c->buf<double>("bbox", 8);
  int* bad = c->buf<int>("bbox_bad", 1);
  PR_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), c->stream));
  k_bbox_partial<<<nb, kThreads, 0, c->stream>>>(d_pts6, P, part, bad);
  PR_CHECK_LAUNCH();
  k_bbox_final<<<1, 32, 0, c->stream>>>(part, nb, bb);
  PR_CHECK_LAUNCH();
  double hb[6];
  int hbad = 0;
  PR_CUDA(cudaMemcpyAsync(hb, bb, 6 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  PR_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  c->sync();
  PR_REQUIRE(!hbad, PR_ERR_INVALID_ARGUMENT, "input contains a non-finite coordinate or normal component");

  // unit_cube_transform (src/geometry.rs:384-402) and Mat4::inverse (:274-317), on the host
  double ctr[3], sz[3];
  for (int k = 0; k < 3; ++k) {
    ctr[k] = (hb[k] + hb[3 + k]) * 0.5;
    sz[k] = hb[3 + k] - hb[k];
  }
  double max_dim = std::fmax(std::fmax(sz[0], sz[1]), sz[2]);
  double s = max_dim > 0.0 ? scale / max_dim : 1.0;
  double* M = c->M;
  for (int i = 0; i < 16; ++i) M[i] = 0.0;
  M[0] = s;
  M[5] = s;
  M[10] = s;
  M[12] = -s * ctr[0] + 0.5;
  M[13] = -s * ctr[1] + 0.5;
  M[14] = -s * ctr[2] + 0.5;
  M[15] = 1.0;
  {
#define MM(col, row) M[(col) * 4 + (row)]
    double a = MM(0, 0), b = MM(1, 0), cc = MM(2, 0);
    double d = MM(0, 1), e = MM(1, 1), f = MM(2, 1);
    double g = MM(0, 2), hh = MM(1, 2), i = MM(2, 2);
    double det = a * (e * i - f * hh) - b * (d * i - f * g) + cc * (d * hh - e * g);
    double* O = c->Minv;
    for (int k = 0; k < 16; ++k) O[k] = 0.0;
    if (std::fabs(det) < 1e-30) {
      O[0] = O[5] = O[10] = O[15] = 1.0;
    } else {
      double inv_det = 1.0 / det;
      double a_inv = (e * i - f * hh) * inv_det, b_inv = (cc * hh - b * i) * inv_det, c_inv = (b * f - cc * e) * inv_det;
      double d_inv = (f * g - d * i) * inv_det, e_inv = (a * i - cc * g) * inv_det, f_inv = (cc * d - a * f) * inv_det;
      double g_inv = (d * hh - e * g) * inv_det, h_inv = (b * g - a * hh) * inv_det, i_inv = (a * e - b * d) * inv_det;
      double tx = MM(3, 0), ty = MM(3, 1), tz = MM(3, 2);
      double cols[4][4] = {{a_inv, d_inv, g_inv, 0.0},
                           {b_inv, e_inv, h_inv, 0.0},
                           {c_inv, f_inv, i_inv, 0.0},
                           {-(a_inv * tx + b_inv * ty + c_inv * tz), -(d_inv * tx + e_inv * ty + f_inv * tz),
                            -(g_inv * tx + h_inv * ty + i_inv * tz), 1.0}};
      for (int cc2 = 0; cc2 < 4; ++cc2)
        for (int r = 0; r < 4; ++r) O[cc2 * 4 + r] = cols[cc2][r];
    }
#undef MM
  }
  Mat16 m16;
  for (int k = 0; k < 16; ++k) m16.m[k] = M[k];
  double* upos = c->buf<double>("upos", 3 * P);
  double* unrm = c->buf<double>("unrm", 3 * P);
  double* ulen = c->buf<double>("ulen", P);
  k_transform<<<grid_for(P), kThreads, 0, c->stream>>>(d_pts6, P, m16, upos, unrm, ulen);
  PR_CHECK_LAUNCH();
  c->P = P;
  c->have_points = true;
}

// ------------------------------------------------------------------ stage: splat + rhs + screening
void stage_splat_rhs(pr_context* c, uint32_t D, double pw) {
  const uint64_t P = c->P;
  const uint64_t n = 1ull << (3 * D);
  const uint64_t m = 8 * P;
  c->D = D;
  c->n = n;
  c->pw = pw;
  const double* upos = c->get<double>("upos");
  const double* unrm = c->get<double>("unrm");

  // --- splat: floor cells
  uint32_t* kin = c->buf<uint32_t>("pair_kin", m);
  uint32_t* vin = c->buf<uint32_t>("pair_vin", m);
  k_pair_keys<false><<<grid_for(P), kThreads, 0, c->stream>>>(upos, P, D, kin, vin, nullptr, nullptr, nullptr);
  PR_CHECK_LAUNCH();
  uint64_t T = sort_and_segment(c, "splat", kin, vin, m, D);
  c->T = T;
  uint32_t* map = c->buf<uint32_t>("map", n);
  PR_CUDA(cudaMemsetAsync(map, 0xff, n * sizeof(uint32_t), c->stream));
  double* v = c->buf<double>("nfield", 4 * std::max<uint64_t>(T, 1));
  if (T > 0) {
    k_splat_reduce<<<grid_for(T), kThreads, 0, c->stream>>>(c->get<uint32_t>("splat_runkey"),
                                                             c->get<uint32_t>("splat_runoff"), T,
                                                             c->get<uint32_t>("splat_val"), upos, unrm, P, D, v, map);
    PR_CHECK_LAUNCH();
  }
  double* b = c->buf<double>("b64", n);
  if (D >= 4 && T > 0) {
    const uint32_t nblk = 1u << (3 * (D - 4));
    uint32_t* flag = c->buf<uint32_t>("rhs_flag", (size_t)nblk + 1);
    uint32_t* fpos = c->buf<uint32_t>("rhs_fpos", (size_t)nblk + 1);
    uint32_t* ids = c->buf<uint32_t>("rhs_blocks", nblk);
    PR_CUDA(cudaMemsetAsync(flag, 0, ((size_t)nblk + 1) * sizeof(uint32_t), c->stream));
    PR_CUDA(cudaMemsetAsync(b, 0, n * sizeof(double), c->stream));
    k_mark_rhs_blocks<<<grid_for(T), kThreads, 0, c->stream>>>(c->get<uint32_t>("splat_runkey"), T, 1u << (D - 4),
                                                               flag);
    PR_CHECK_LAUNCH();
    size_t tb = 0;
    PR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, flag, fpos, (int64_t)nblk + 1, c->stream));
    void* tmp = c->buf<char>("cub_tmp", tb);
    PR_COUNT_PRIMITIVE();
    PR_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, flag, fpos, (int64_t)nblk + 1, c->stream));
    k_list_blocks<<<grid_for(nblk), kThreads, 0, c->stream>>>(flag, fpos, nblk, ids);
    PR_CHECK_LAUNCH();
    uint32_t nact = 0;
    PR_CUDA(cudaMemcpyAsync(&nact, fpos + nblk, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
    c->sync();
    if (nact > 0) {
      k_rhs_blocks<<<nact, 256, 0, c->stream>>>(D, ids, map, v, T, b);
      PR_CHECK_LAUNCH();
    }
  } else {
    k_rhs_dense<<<grid_for(n, kThreads, 1u << 22), kThreads, 0, c->stream>>>(D, map, v, T, b);
    PR_CHECK_LAUNCH();
  }

  // --- screening: trunc cells; kept as per-point payload for the operator
  c->S = 0;
  c->S_pairs = 0;
  c->P_in = 0;
  if (pw > 0.0) {
    uint32_t* qkin = c->buf<uint32_t>("scr_kin", m);  // per (point, corner): node or sentinel
    uint32_t* qvin = c->buf<uint32_t>("scr_vin", m);
    double* phi64 = c->buf<double>("phi64", m);
    float* phi32 = c->buf<float>("phi32", m);
    unsigned long long* nin = c->buf<unsigned long long>("n_inside", 1);
    PR_CUDA(cudaMemsetAsync(nin, 0, sizeof(unsigned long long), c->stream));
    k_pair_keys<true><<<grid_for(P), kThreads, 0, c->stream>>>(upos, P, D, qkin, qvin, phi64, phi32, nin);
    PR_CHECK_LAUNCH();
    uint64_t S = sort_and_segment(c, "scr", qkin, qvin, m, D);
    unsigned long long h_nin = 0;
    uint32_t h_pairs = 0;
    PR_CUDA(cudaMemcpyAsync(&h_nin, nin, sizeof(h_nin), cudaMemcpyDeviceToHost, c->stream));
    PR_CUDA(cudaMemcpyAsync(&h_pairs, c->get<uint32_t>("scr_runoff") + S, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                            c->stream));
    c->sync();
    c->S = S;
    c->S_pairs = h_pairs;
    c->P_in = h_nin;
    const double h = 1.0 / (double)(1u << D);
    const double wh3 = pw * (h * h * h) / 1.5;
    if (S > 0) {
      k_rhs_screen<<<grid_for(S), kThreads, 0, c->stream>>>(c->get<uint32_t>("scr_runkey"),
                                                            c->get<uint32_t>("scr_runoff"), S,
                                                            c->get<uint32_t>("scr_val"), upos, P, D, wh3, b);
      PR_CHECK_LAUNCH();
    }
  }
  c->have_state = true;
}

void scatter_normal_field(pr_context* c, double* d_nf3, double* d_w) {
  PR_CUDA(cudaMemsetAsync(d_nf3, 0, 3 * c->n * sizeof(double), c->stream));
  PR_CUDA(cudaMemsetAsync(d_w, 0, c->n * sizeof(double), c->stream));
  if (c->T > 0) {
    k_scatter_nf<<<grid_for(c->T), kThreads, 0, c->stream>>>(c->get<uint32_t>("splat_runkey"), c->T,
                                                             c->get<double>("nfield"), d_nf3, d_w);
    PR_CHECK_LAUNCH();
  }
}

}  // namespace pr

// Block-tiled multigrid and CG kernels.
//
// Vectors live in Morton order, so a TB^3 block (TB = 8 or 16) is TB^3 consecutive
// entries: a CTA loads its block with coalesced loads, gathers the one-node halo of its
// 26 neighbour blocks, and works in shared memory.  No kernel writes a vector that it
// (or another CTA of the same launch) reads as halo: every halo-reading update writes a
// second buffer, so each launch is deterministic.
//
// Operator of level l (Galerkin, exact for the 1-D linear prolongation):
//   A_l = H (S_l (x) M_l (x) M_l + M_l (x) S_l (x) M_l + M_l (x) M_l (x) S_l) + shift I
// with H the finest spacing and 1-D matrices M_l, S_l that are tridiagonal Toeplitz except
// for the diagonal entry of node 0 (the coarse basis function at 0 is cut at the domain's
// low face: the fine grid has no node -1).  Interior nodes see the crate's constant
// stencil (src/fem_tree.rs:39-48) scaled to their level — centre, 12 edge and 8 corner
// neighbours; nodes on a low face use per-face coefficients from an 8 x 27 table.
//
// Smoother: multicolour Gauss-Seidel inside each block (8 parity colours, exact), blocks
// coupled through their halo values from before the sweep.  Forward sweeps relax colours
// 0..7 and backward sweeps 7..0, each the adjoint of the other, so the V-cycle (forward
// pre-, backward post-smoothing) is a symmetric preconditioner.  The smoother keeps its
// tile in a parity-split layout (8 sub-tiles, one per parity class), in which the nodes
// of one colour are contiguous and a warp's neighbour loads hit distinct banks.
#include <cub/cub.cuh>

#include <mutex>
#include <tuple>
#include <map>
#include <cstdio>
#include <cstdlib>
#include <set>
#include <string>
#include <type_traits>
#include <vector>

#include "pr_mg.cuh"

namespace pr {

namespace {

template <int TB>
struct Geo {
  static constexpr int W = TB + 2;                  // tile width with a one-node halo
  static constexpr int H = W / 2;                   // parity sub-tile width
  static constexpr int H3 = H * H * H;
  static constexpr int N = TB * TB * TB;            // nodes of a block
  static constexpr int C = TB / 2;                  // colour lattice width
  static constexpr int C3 = C * C * C;
  static constexpr int LOGC = TB == 16 ? 3 : 2;
  static constexpr int THREADS = C3;                // one node per colour per thread
  static constexpr int HALO = W * W * W - N;
};

template <typename T>
struct DevCoef {
  T c0, ce, cc;       // interior: centre (+shift), edge, corner (faces are 0 in the interior)
  const T* table;     // [8 low-face masks][27 offsets], offset (dx+1) + 3(dy+1) + 9(dz+1)
  int has_faces;      // level has low-face modifications
};

// parity-split index of tile coordinate u in [0, W)^3
template <int TB>
__device__ __forceinline__ int ps_index(int ux, int uy, int uz) {
  constexpr int H = Geo<TB>::H, H3 = Geo<TB>::H3;
  const int sub = (ux & 1) | ((uy & 1) << 1) | ((uz & 1) << 2);
  return sub * H3 + ((uz >> 1) * H + (uy >> 1)) * H + (ux >> 1);
}

// h-th position of the one-node halo shell of a (TB+2)^3 tile: 6 faces, 12 edges, 8 corners
template <int TB>
__device__ __forceinline__ void halo_u(int h, int& ux, int& uy, int& uz) {
  constexpr int W = TB + 2, F = TB * TB, LT = TB == 16 ? 4 : 3;  // log2 TB
  if (h < 6 * F) {
    const int f = h >> (2 * LT), a = (h & (F - 1)) & (TB - 1), b = (h & (F - 1)) >> LT;
    const int axis = f >> 1, side = (f & 1) ? W - 1 : 0;
    if (axis == 0) { ux = side; uy = a + 1; uz = b + 1; }
    else if (axis == 1) { ux = a + 1; uy = side; uz = b + 1; }
    else { ux = a + 1; uy = b + 1; uz = side; }
    return;
  }
  h -= 6 * F;
  if (h < 12 * TB) {
    const int e = h >> LT, a = (h & (TB - 1)) + 1, axis = e >> 2;
    const int s0 = (e & 1) ? W - 1 : 0, s1 = (e & 2) ? W - 1 : 0;
    if (axis == 0) { ux = a; uy = s0; uz = s1; }
    else if (axis == 1) { ux = s0; uy = a; uz = s1; }
    else { ux = s0; uy = s1; uz = a; }
    return;
  }
  h -= 12 * TB;
  ux = (h & 1) ? W - 1 : 0;
  uy = (h & 2) ? W - 1 : 0;
  uz = (h & 4) ? W - 1 : 0;
}

template <typename T>
__device__ __forceinline__ T ldg_or0(const T* __restrict__ x, int gx, int gy, int gz, int res) {
  if (gx < 0 || gy < 0 || gz < 0 || gx >= res || gy >= res || gz >= res) return (T)0;
  return __ldg(x + morton3(gx, gy, gz));
}

// ------------------------------------------------------------------ smoother
// MODE 0: xo = sweep(xi); MODE 1: xo = sweep(0) (xi unused); MODE 2: xo = sweep(xi + P ec).
// DOT: part[block] = sum_i f_i xo_i over the block.
template <typename T, int TB, int MODE, bool DOT, bool FWD>
__global__ void __launch_bounds__(Geo<TB>::THREADS) k_smooth(uint32_t D, const T* __restrict__ xi, T* __restrict__ xo,
                                                           const T* __restrict__ f, const T* __restrict__ ec,
                                                           DevCoef<T> k, double* __restrict__ part) {
  using G = Geo<TB>;
  constexpr int W = G::W, H = G::H, H3 = G::H3, N = G::N, C = G::C, C3 = G::C3, LOGC = G::LOGC;
  constexpr int CW = TB / 2 + 2;  // coarse tile width (MODE 2): coarse [ox/2 - 1, ox/2 + TB/2]
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* tile = reinterpret_cast<T*>(smem_raw);  // W^3, parity-split
  T* fs = tile + W * W * W;                  // N, colour-major: fs[col * C3 + lattice index]
  T* ctile = fs + N;                         // CW^3 (MODE 2)
  const int res = 1 << D;
  {
    const uint64_t nl = 1ull << (3 * D);
    xi = cloud_slice(xi, nl);
    xo = cloud_slice(xo, nl);
    f = cloud_slice(f, nl);
    ec = cloud_slice(ec, nl / 8);
    part = cloud_slice(part, gridDim.x);
  }
  const uint32_t blk = blockIdx.x;
  const uint64_t base = (uint64_t)blk * N;
  uint32_t bx, by, bz;
  unmorton3(blk, bx, by, bz);
  const int ox = (int)bx * TB, oy = (int)by * TB, oz = (int)bz * TB;
  const int tid = threadIdx.x;
  const int cox = ox / 2 - 1, coy = oy / 2 - 1, coz = oz / 2 - 1;

  if (MODE == 2) {
    const int resc = res >> 1;
    for (int t = tid; t < CW * CW * CW; t += G::THREADS) {
      const int cx = cox + t % CW, cy = coy + (t / CW) % CW, cz = coz + t / (CW * CW);
      T v = 0;
      if (cx >= 0 && cx < resc && cy >= 0 && cy < resc && cz >= 0 && cz < resc) v = __ldg(ec + morton3(cx, cy, cz));
      ctile[t] = v;
    }
    __syncthreads();
  }
  // P ec at global (gx,gy,gz): even -> coarse g/2 (w 1), odd -> (g-1)/2, (g+1)/2 (w 1/2 each)
  auto prolong = [&](int gx, int gy, int gz) -> T {
    const int ax = (gx >> 1) - cox, ay = (gy >> 1) - coy, az = (gz >> 1) - coz;
    const int nx = 1 + (gx & 1), ny = 1 + (gy & 1), nz = 1 + (gz & 1);
    T s = 0;
    for (int a = 0; a < nz; ++a)
      for (int b = 0; b < ny; ++b)
        for (int c = 0; c < nx; ++c) s += ctile[((az + a) * CW + (ay + b)) * CW + (ax + c)];
    const T w = (T)(((gx & 1) ? 0.5 : 1.0) * ((gy & 1) ? 0.5 : 1.0) * ((gz & 1) ? 0.5 : 1.0));
    return w * s;
  };
  // interior + f
  for (int t = tid; t < N; t += G::THREADS) {
    uint32_t lx, ly, lz;
    unmorton3((uint32_t)t, lx, ly, lz);
    const int col = (lx & 1) | ((ly & 1) << 1) | ((lz & 1) << 2);
    const int lat = (lx >> 1) | ((ly >> 1) << LOGC) | ((lz >> 1) << (2 * LOGC));
    fs[col * C3 + lat] = __ldg(f + base + t);
    T v = 0;
    if (MODE != 1) v = __ldg(xi + base + t);
    if (MODE == 2) v += prolong(ox + (int)lx, oy + (int)ly, oz + (int)lz);
    tile[ps_index<TB>(lx + 1, ly + 1, lz + 1)] = v;
  }
  // halo
  for (int h = tid; h < G::HALO; h += G::THREADS) {
    int ux, uy, uz;
    halo_u<TB>(h, ux, uy, uz);
    T v = 0;
    if (MODE != 1) {
      const int gx = ox + ux - 1, gy = oy + uy - 1, gz = oz + uz - 1;
      if (gx >= 0 && gy >= 0 && gz >= 0 && gx < res && gy < res && gz < res) {
        v = __ldg(xi + morton3(gx, gy, gz));
        if (MODE == 2) v += prolong(gx, gy, gz);
      }
    }
    tile[ps_index<TB>(ux, uy, uz)] = v;
  }
  __syncthreads();

  // Gauss-Seidel over the 8 colours
  const int li = tid & (C - 1), lj = (tid >> LOGC) & (C - 1), lk = tid >> (2 * LOGC);
#pragma unroll
  for (int step = 0; step < 8; ++step) {
    const int col = FWD ? step : 7 - step;
    const int cx = col & 1, cy = (col >> 1) & 1, cz = col >> 2;
    const int own = (1 - cx) | ((1 - cy) << 1) | ((1 - cz) << 2);  // sub-tile of tile coordinate l + 1
    const int pos = ((lk + cz) * H + (lj + cy)) * H + (li + cx);
    const int self = own * H3 + pos;
    int mask = 0;
    if (k.has_faces)
      mask = ((ox == 0 && cx == 0 && li == 0) ? 1 : 0) | ((oy == 0 && cy == 0 && lj == 0) ? 2 : 0) |
             ((oz == 0 && cz == 0 && lk == 0) ? 4 : 0);
    T vals[27];
#pragma unroll
    for (int o = 0; o < 27; ++o) {
      const int dx = o % 3 - 1, dy = (o / 3) % 3 - 1, dz = o / 9 - 1;
      const int sub = own ^ ((dx != 0) | ((dy != 0) << 1) | ((dz != 0) << 2));
      const int hx = dx == 0 ? 0 : (dx < 0 ? -cx : 1 - cx);
      const int hy = dy == 0 ? 0 : (dy < 0 ? -cy : 1 - cy);
      const int hz = dz == 0 ? 0 : (dz < 0 ? -cz : 1 - cz);
      const int nzc = (dx != 0) + (dy != 0) + (dz != 0);
      // faces are only read on the (rare) low-face path
      vals[o] = (o == 13 || (nzc == 1 && mask == 0)) ? (T)0 : tile[sub * H3 + pos + (hz * H + hy) * H + hx];
    }
    const T fi = fs[col * C3 + tid];
    T nv;
    if (mask == 0) {
      T se = 0, sc = 0;
#pragma unroll
      for (int o = 0; o < 27; ++o) {
        const int nzc = (o % 3 != 1) + ((o / 3) % 3 != 1) + (o / 9 != 1);
        if (nzc == 2) se += vals[o];
        else if (nzc == 3) sc += vals[o];
      }
      nv = (fi - k.ce * se - k.cc * sc) / k.c0;
    } else {
      const T* cm = k.table + 27 * mask;
      T off = 0;
#pragma unroll
      for (int o = 0; o < 27; ++o)
        if (o != 13) off += cm[o] * vals[o];
      nv = (fi - off) / cm[13];
    }
    tile[self] = nv;
    __syncthreads();
  }

  double acc = 0.0;
  for (int t = tid; t < N; t += G::THREADS) {
    uint32_t lx, ly, lz;
    unmorton3((uint32_t)t, lx, ly, lz);
    const T v = tile[ps_index<TB>(lx + 1, ly + 1, lz + 1)];
    xo[base + t] = v;
    if (DOT) {
      const int col = (lx & 1) | ((ly & 1) << 1) | ((lz & 1) << 2);
      const int lat = (lx >> 1) | ((ly >> 1) << LOGC) | ((lz >> 1) << (2 * LOGC));
      acc += (double)v * (double)fs[col * C3 + lat];
    }
  }
  if (DOT) {
    typedef cub::BlockReduce<double, Geo<TB>::THREADS> BR;
    __shared__ typename BR::TempStorage tmp;
    const double s = BR(tmp).Sum(acc);
    if (tid == 0) part[blk] = s;
  }
}

// ------------------------------------------------------------------ stencil rows on a natural tile
// tile index (ux,uy,uz) -> (uz*W + uy)*W + ux
template <typename T, int W>
__device__ __forceinline__ T row_general(const T* __restrict__ s, int idx, const T* __restrict__ cm) {
  T r = 0;
#pragma unroll
  for (int o = 0; o < 27; ++o) {
    const int dx = o % 3 - 1, dy = (o / 3) % 3 - 1, dz = o / 9 - 1;
    r += cm[o] * s[idx + dx + W * dy + W * W * dz];
  }
  return r;
}

template <typename T, int W>
__device__ __forceinline__ T row_interior(const T* __restrict__ s, int idx, T c0, T ce, T cc) {
  T se = 0, sc = 0;
#pragma unroll
  for (int o = 0; o < 27; ++o) {
    const int dx = o % 3 - 1, dy = (o / 3) % 3 - 1, dz = o / 9 - 1;
    const int nzc = (dx != 0) + (dy != 0) + (dz != 0);
    if (nzc == 2) se += s[idx + dx + W * dy + W * W * dz];
    else if (nzc == 3) sc += s[idx + dx + W * dy + W * W * dz];
  }
  return c0 * s[idx] + ce * se + cc * sc;
}

// Column sweep along z: for the column (ux,uy) of a natural tile, output A x at tile
// z coordinates uz0..uz0+ZL-1 through fn(k, centre value, row value).  Plane partial sums
// are shared by the three outputs that use them.
template <typename T, int W, int ZL, typename Fn>
__device__ __forceinline__ void column_apply(const T* __restrict__ s, int ux, int uy, int uz0, T c0, T ce, T cc,
                                             Fn fn) {
  auto plane = [&](int uz, T& pc, T& pf, T& pe) {
    const int b = (uz * W + uy) * W + ux;
    pc = s[b];
    pf = s[b - 1] + s[b + 1] + s[b - W] + s[b + W];
    pe = s[b - 1 - W] + s[b + 1 - W] + s[b - 1 + W] + s[b + 1 + W];
  };
  T pcm, pfm, pem, pc0, pf0, pe0;
  plane(uz0 - 1, pcm, pfm, pem);
  plane(uz0, pc0, pf0, pe0);
#pragma unroll
  for (int k = 0; k < ZL; ++k) {
    T pcp, pfp, pep;
    plane(uz0 + k + 1, pcp, pfp, pep);
    fn(k, pc0, c0 * pc0 + ce * (pe0 + pfm + pfp) + cc * (pem + pep));
    pcm = pc0;
    pfm = pf0;
    pem = pe0;
    pc0 = pcp;
    pf0 = pfp;
    pe0 = pep;
  }
  (void)pcm;
}

// ------------------------------------------------------------------ fine-level SpMV
// XPBY: dn = z + beta d (tile and halo), dn written; q = A dn (stencil part); part = dn.q
template <typename T, int TB, bool XPBY>
__global__ void __launch_bounds__(Geo<TB>::THREADS) k_spmv(uint32_t D, const T* __restrict__ z,
                                                         const T* __restrict__ d, T* __restrict__ dn, T beta,
                                                         T* __restrict__ q, DevCoef<T> k, double* __restrict__ part) {
  using G = Geo<TB>;
  constexpr int W = G::W, N = G::N;
  constexpr int SEG = G::THREADS / (TB * TB);  // z segments per column
  constexpr int ZL = TB / SEG;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* tile = reinterpret_cast<T*>(smem_raw);  // W^3 natural
  T* out = tile + W * W * W;                 // N, Morton-local
  const int res = 1 << D;
  {
    const uint64_t nl = 1ull << (3 * D);
    z = cloud_slice(z, nl);
    d = cloud_slice(d, nl);
    dn = cloud_slice(dn, nl);
    q = cloud_slice(q, nl);
    part = cloud_slice(part, gridDim.x);
  }
  const uint32_t blk = blockIdx.x;
  const uint64_t base = (uint64_t)blk * N;
  uint32_t bx, by, bz;
  unmorton3(blk, bx, by, bz);
  const int ox = (int)bx * TB, oy = (int)by * TB, oz = (int)bz * TB;
  const int tid = threadIdx.x;
  for (int t = tid; t < N; t += G::THREADS) {
    uint32_t lx, ly, lz;
    unmorton3((uint32_t)t, lx, ly, lz);
    T v = __ldg(d + base + t);
    if (XPBY) {
      v = __ldg(z + base + t) + beta * v;
      out[t] = v;  // staged dn for the coalesced store below
    }
    tile[((lz + 1) * W + (ly + 1)) * W + (lx + 1)] = v;
  }
  for (int h = tid; h < G::HALO; h += G::THREADS) {
    int ux, uy, uz;
    halo_u<TB>(h, ux, uy, uz);
    const int gx = ox + ux - 1, gy = oy + uy - 1, gz = oz + uz - 1;
    T v = 0;
    if (gx >= 0 && gy >= 0 && gz >= 0 && gx < res && gy < res && gz < res) {
      const uint32_t m = morton3(gx, gy, gz);
      v = __ldg(d + m);
      if (XPBY) v = __ldg(z + m) + beta * v;
    }
    tile[(uz * W + uy) * W + ux] = v;
  }
  __syncthreads();
  if (XPBY) {
    for (int t = tid; t < N; t += G::THREADS) dn[base + t] = out[t];
    __syncthreads();
  }
  const int col = tid % (TB * TB), seg = tid / (TB * TB);
  const int ux = col % TB + 1, uy = col / TB + 1;
  double acc = 0.0;
  column_apply<T, W, ZL>(tile, ux, uy, seg * ZL + 1, k.c0, k.ce, k.cc, [&](int kk, T dv, T y) {
    const int lz = seg * ZL + kk;
    out[morton3(ux - 1, uy - 1, lz)] = y;
    acc += (double)dv * (double)y;
  });
  __syncthreads();
  for (int t = tid; t < N; t += G::THREADS) q[base + t] = out[t];
  typedef cub::BlockReduce<double, Geo<TB>::THREADS> BR;
  __shared__ typename BR::TempStorage tmp;
  const double s = BR(tmp).Sum(acc);
  if (tid == 0) part[blk] = s;
}

// ------------------------------------------------------------------ residual + restriction
// fc = P^T (f - A e) for the (TB/2)^3 coarse nodes whose fine centre lies in the block.
// r is needed on local [-1, TB-1]^3: the block interior (z columns) plus its low shell.
template <typename T, int TB>
__global__ void __launch_bounds__(Geo<TB>::THREADS) k_resid_restrict(uint32_t D, const T* __restrict__ e,
                                                                   const T* __restrict__ f, T* __restrict__ fc,
                                                                   DevCoef<T> k) {
  using G = Geo<TB>;
  constexpr int N = G::N;
  constexpr int WE = TB + 3;  // e over local [-2, TB]
  constexpr int WR = TB + 1;  // r over local [-1, TB-1]
  constexpr int TC = TB / 2;
  constexpr int SEG = G::THREADS / (TB * TB);
  constexpr int ZL = TB / SEG;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* et = reinterpret_cast<T*>(smem_raw);  // WE^3 natural, tile coordinate = local + 2
  T* rt = et + WE * WE * WE;               // WR^3 natural, coordinate = local + 1
  const int res = 1 << D;
  {
    const uint64_t nl = 1ull << (3 * D);
    e = cloud_slice(e, nl);
    f = cloud_slice(f, nl);
    fc = cloud_slice(fc, nl / 8);
  }
  const uint32_t blk = blockIdx.x;
  const uint64_t base = (uint64_t)blk * N;
  uint32_t bx, by, bz;
  unmorton3(blk, bx, by, bz);
  const int ox = (int)bx * TB, oy = (int)by * TB, oz = (int)bz * TB;
  const int tid = threadIdx.x;
  for (int t = tid; t < N; t += G::THREADS) {
    uint32_t lx, ly, lz;
    unmorton3((uint32_t)t, lx, ly, lz);
    et[((lz + 2) * WE + (ly + 2)) * WE + (lx + 2)] = __ldg(e + base + t);
    rt[((lz + 1) * WR + (ly + 1)) * WR + (lx + 1)] = __ldg(f + base + t);  // f first, r = f - A e below
  }
  for (int t = tid; t < WE * WE * WE; t += G::THREADS) {
    const int tx = t % WE, ty = (t / WE) % WE, tz = t / (WE * WE);
    if (tx >= 2 && tx < TB + 2 && ty >= 2 && ty < TB + 2 && tz >= 2 && tz < TB + 2) continue;
    et[t] = ldg_or0(e, ox + tx - 2, oy + ty - 2, oz + tz - 2, res);
  }
  __syncthreads();
  // interior: z columns with the interior rows
  {
    const int col = tid % (TB * TB), seg = tid / (TB * TB);
    const int lx = col % TB, ly = col / TB;
    column_apply<T, WE, ZL>(et, lx + 2, ly + 2, seg * ZL + 2, k.c0, k.ce, k.cc, [&](int kk, T, T y) {
      const int lz = seg * ZL + kk;
      rt[((lz + 1) * WR + (ly + 1)) * WR + (lx + 1)] -= y;
    });
  }
  // low shell of r: local coordinate -1 on at least one axis
  {
    constexpr int S1 = WR * WR, S2 = TB * WR, S3 = TB * TB;
    for (int t = tid; t < S1 + S2 + S3; t += G::THREADS) {
      int lx, ly, lz;
      if (t < S1) { lx = -1; ly = t % WR - 1; lz = t / WR - 1; }
      else if (t < S1 + S2) { const int u = t - S1; lx = u % TB; ly = -1; lz = u / TB - 1; }
      else { const int u = t - S1 - S2; lx = u % TB; ly = u / TB; lz = -1; }
      const int gx = ox + lx, gy = oy + ly, gz = oz + lz;
      T r = 0;
      if (gx >= 0 && gy >= 0 && gz >= 0) {
        const int ei = ((lz + 2) * WE + (ly + 2)) * WE + (lx + 2);
        const int mask = k.has_faces ? ((gx == 0) | ((gy == 0) << 1) | ((gz == 0) << 2)) : 0;
        const T y = mask ? row_general<T, WE>(et, ei, k.table + 27 * mask) : row_interior<T, WE>(et, ei, k.c0, k.ce, k.cc);
        r = __ldg(f + morton3(gx, gy, gz)) - y;
      }
      rt[((lz + 1) * WR + (ly + 1)) * WR + (lx + 1)] = r;
    }
  }
  __syncthreads();
  if (k.has_faces && (ox == 0 || oy == 0 || oz == 0)) {
    // interior nodes on a low domain face: replace the interior row by the face row
    for (int t = tid; t < N; t += G::THREADS) {
      uint32_t lx, ly, lz;
      unmorton3((uint32_t)t, lx, ly, lz);
      const int gx = ox + lx, gy = oy + ly, gz = oz + lz;
      const int mask = (gx == 0) | ((gy == 0) << 1) | ((gz == 0) << 2);
      if (!mask) continue;
      const int ei = ((lz + 2) * WE + (ly + 2)) * WE + (lx + 2);
      const T yi = row_interior<T, WE>(et, ei, k.c0, k.ce, k.cc);
      const T yf = row_general<T, WE>(et, ei, k.table + 27 * mask);
      rt[((lz + 1) * WR + (ly + 1)) * WR + (lx + 1)] += yi - yf;
    }
    __syncthreads();
  }
  const uint64_t cbase = (uint64_t)blk * (TC * TC * TC);
  for (int t = tid; t < TC * TC * TC; t += G::THREADS) {
    uint32_t cx, cy, cz;
    unmorton3((uint32_t)t, cx, cy, cz);
    const int fx = 2 * cx + 1, fy = 2 * cy + 1, fz = 2 * cz + 1;  // r tile coordinate of the fine centre
    T s = 0;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
      for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
          const T w = (T)((dx ? 0.5 : 1.0) * (dy ? 0.5 : 1.0) * (dz ? 0.5 : 1.0));
          s += w * rt[((fz + dz) * WR + (fy + dy)) * WR + (fx + dx)];
        }
    fc[cbase + t] = s;
  }
}

// fixed-order sum of two partial arrays: out = sum(part) + scale2 * sum(part2)
__global__ void __launch_bounds__(1024) k_sum_parts(const double* __restrict__ part, int np, double scale2,
                                                    const double* __restrict__ part2, int np2,
                                                    double* __restrict__ out) {
  part += (uint64_t)blockIdx.x * np;  // block k: cloud k's partials (packed launches)
  part2 += (uint64_t)blockIdx.x * np2;
  out += blockIdx.x;
  double s = 0.0, s2 = 0.0;
  for (int i = threadIdx.x; i < np; i += 1024) s += part[i];
  for (int i = threadIdx.x; i < np2; i += 1024) s2 += part2[i];
  typedef cub::BlockReduce<double, 1024> BR;
  __shared__ typename BR::TempStorage tmp;
  const double a = BR(tmp).Sum(s);
  __syncthreads();
  const double b = BR(tmp).Sum(s2);
  if (threadIdx.x == 0) out[0] = a + scale2 * b;
}

// ------------------------------------------------------------------ helpers of the 16^3 block kernels
namespace s16 {
constexpr int CW = 10;  // coarse tile width

// spread the 4 low bits of v to bit positions 0,3,6,9
__device__ __forceinline__ uint32_t sp4(uint32_t v) {
  return (v & 1u) | ((v & 2u) << 2) | ((v & 4u) << 4) | ((v & 8u) << 6);
}
template <typename T>
struct Vec4;
template <>
struct Vec4<float> {
  typedef float4 type;
};
template <>
struct Vec4<double> {
  typedef double4 type;
};

__device__ __forceinline__ float4 ld4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ double4 ld4(const double* p) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(p)), b = __ldg(reinterpret_cast<const double2*>(p) + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ void st4(float* p, const float4& v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ void st4(double* p, const double4& v) {
  reinterpret_cast<double2*>(p)[0] = make_double2(v.x, v.y);
  reinterpret_cast<double2*>(p)[1] = make_double2(v.z, v.w);
}

// local coordinates of element 4q of a 16^3 Morton block (q = quad index), x0 = y0 = 0
__device__ __forceinline__ void quad_coords(int q, int& lx, int& ly, int& lz) {
  lx = ((q >> 1) & 1) << 1 | ((q >> 4) & 1) << 2 | ((q >> 7) & 1) << 3;
  ly = ((q >> 2) & 1) << 1 | ((q >> 5) & 1) << 2 | ((q >> 8) & 1) << 3;
  lz = (q & 1) | ((q >> 3) & 1) << 1 | ((q >> 6) & 1) << 2 | ((q >> 9) & 1) << 3;
}

// Load the one-node halo of the block into a tile (idx: tile index of tile coordinates).
// nb[27]: Morton base of the neighbour block (dx+1)+3(dy+1)+9(dz+1), or ~0u if outside.
// NT: threads of the CTA.
template <int NT, typename T, typename Idx, typename Xf>
__device__ __forceinline__ void load_halo(T* tile, const T* __restrict__ x, const uint32_t* nb, Idx idx, Xf xf) {
#pragma unroll
  for (int i = threadIdx.x; i < 256; i += NT) {  // faces: (a, b) = in-face coordinates of position i
    const int a = i & 15, b = i >> 4;
    const uint32_t sa = sp4(a), sb = sp4(b);
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const int axis = f >> 1, hi = f & 1;
      const int nbi = axis == 0 ? (hi ? 14 : 12) : (axis == 1 ? (hi ? 16 : 10) : (hi ? 22 : 4));
      const uint32_t side = hi ? 0u : 0x249u;  // neighbour-local coordinate 0 or 15, spread
      uint32_t m;
      int ux, uy, uz;
      const int s = hi ? 17 : 0;
      if (axis == 0) { m = side | (sa << 1) | (sb << 2); ux = s; uy = a + 1; uz = b + 1; }
      else if (axis == 1) { m = sa | (side << 1) | (sb << 2); ux = a + 1; uy = s; uz = b + 1; }
      else { m = sa | (sb << 1) | (side << 2); ux = a + 1; uy = b + 1; uz = s; }
      const uint32_t base = nb[nbi];
      tile[idx(ux, uy, uz)] = base != ~0u ? xf(base + m) : (T)0;
    }
  }
#pragma unroll
  for (int i = threadIdx.x; i < 200; i += NT) {
    if (i >= 192) {  // corners
      const int c = i - 192;
      const int sx = c & 1, sy = (c >> 1) & 1, sz = (c >> 2) & 1;
      const uint32_t m = (sx ? 0u : 0x249u) | ((sy ? 0u : 0x249u) << 1) | ((sz ? 0u : 0x249u) << 2);
      const int nbi = (sx ? 2 : 0) + 3 * (sy ? 2 : 0) + 9 * (sz ? 2 : 0);
      const uint32_t base = nb[nbi];
      tile[idx(sx ? 17 : 0, sy ? 17 : 0, sz ? 17 : 0)] = base != ~0u ? xf(base + m) : (T)0;
      continue;
    }
    // edges: 4 per axis, 16 nodes each
    const int e = i >> 4, a = i & 15, axis = e >> 2, s1 = e & 1, s2 = (e >> 1) & 1;
    const uint32_t sa = sp4(a);
    const uint32_t c1 = s1 ? 0u : 0x249u, c2 = s2 ? 0u : 0x249u;
    const int d1 = s1 ? 1 : -1, d2 = s2 ? 1 : -1;
    const int u1 = s1 ? 17 : 0, u2 = s2 ? 17 : 0;
    uint32_t m;
    int ux, uy, uz, nbi;
    if (axis == 0) { m = sa | (c1 << 1) | (c2 << 2); ux = a + 1; uy = u1; uz = u2; nbi = 1 + 3 * (d1 + 1) + 9 * (d2 + 1); }
    else if (axis == 1) { m = c1 | (sa << 1) | (c2 << 2); ux = u1; uy = a + 1; uz = u2; nbi = (d1 + 1) + 3 + 9 * (d2 + 1); }
    else { m = c1 | (c2 << 1) | (sa << 2); ux = u1; uy = u2; uz = a + 1; nbi = (d1 + 1) + 3 * (d2 + 1) + 9; }
    const uint32_t base = nb[nbi];
    tile[idx(ux, uy, uz)] = base != ~0u ? xf(base + m) : (T)0;
  }
}

// The sum over a 16^3 block of one value per (quad column q, plane z), in an order fixed by the
// block whatever the launch shape: each column's planes in z order, then the 64 column sums by a
// fixed tree.  red: 1024 doubles of shared memory holding the value of (q, z) at [z 64 + q] (the
// caller writes it after a barrier that ends every other use of that memory).  Every thread calls
// this (it has barriers); thread 0 returns the sum.
__device__ __forceinline__ double block_sum_fixed(double* red) {
  __syncthreads();
  const int t = threadIdx.x;
  double s = 0.0;
  if (t < 64) {
#pragma unroll
    for (int z = 0; z < 16; ++z) s += red[z * 64 + t];
  }
  __syncthreads();
  if (t < 64) red[t] = s;
  __syncthreads();
  if (t < 32) {
    s = red[t] + red[t + 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  }
  return s;
}

__device__ __forceinline__ void neighbour_bases(uint32_t* nb, uint32_t bx, uint32_t by, uint32_t bz, int nblk_axis) {
  const int t = threadIdx.x;
  if (t < 27) {
    const int dx = t % 3 - 1, dy = (t / 3) % 3 - 1, dz = t / 9 - 1;
    const int x = (int)bx + dx, y = (int)by + dy, z = (int)bz + dz;
    nb[t] = (x < 0 || y < 0 || z < 0 || x >= nblk_axis || y >= nblk_axis || z >= nblk_axis)
                ? ~0u
                : (morton3((uint32_t)x, (uint32_t)y, (uint32_t)z) << 12);
  }
}

// Coarse tile for the prolongation: coarse block (8^3, Morton-contiguous) with a one-node
// halo, natural layout 10^3, coordinate = coarse local + 1.  Ends with a barrier.
template <int NT, typename T>
__device__ __forceinline__ void load_coarse_tile(T* ctile, const T* __restrict__ ec, uint32_t blk, uint32_t bx,
                                                 uint32_t by, uint32_t bz, int nblk_axis, uint32_t* cnb) {
  const int t = threadIdx.x;
  // interior: 512 contiguous coarse values
  for (int i = t; i < 512; i += NT) {
    uint32_t cx, cy, cz;
    unmorton3((uint32_t)i, cx, cy, cz);
    ctile[((cz + 1) * CW + (cy + 1)) * CW + (cx + 1)] = __ldg(ec + (uint64_t)blk * 512 + i);
  }
  // halo (488 positions): faces of 8x8 from the neighbour coarse blocks, then edges, corners
  if (t < 27) {
    const int dx = t % 3 - 1, dy = (t / 3) % 3 - 1, dz = t / 9 - 1;
    const int x = (int)bx + dx, y = (int)by + dy, z = (int)bz + dz;
    cnb[t] = (x < 0 || y < 0 || z < 0 || x >= nblk_axis || y >= nblk_axis || z >= nblk_axis)
                 ? ~0u
                 : (morton3((uint32_t)x, (uint32_t)y, (uint32_t)z) << 9);
  }
  __syncthreads();
  auto sp3 = [](uint32_t v) { return (v & 1u) | ((v & 2u) << 2) | ((v & 4u) << 4); };
  for (int i = t; i < 488; i += NT) {
    int ux, uy, uz;
    uint32_t mloc;
    int nbi;
    if (i < 384) {  // faces: 6 x 64
      const int f = i >> 6, a = i & 7, b = (i >> 3) & 7, axis = f >> 1, hi = f & 1;
      const uint32_t side = hi ? 0u : 0x49u;  // local 0 or 7, spread
      const int s = hi ? 9 : 0;
      if (axis == 0) { mloc = side | (sp3(a) << 1) | (sp3(b) << 2); ux = s; uy = a + 1; uz = b + 1; nbi = (hi ? 2 : 0) + 3 + 9; }
      else if (axis == 1) { mloc = sp3(a) | (side << 1) | (sp3(b) << 2); ux = a + 1; uy = s; uz = b + 1; nbi = 1 + 3 * (hi ? 2 : 0) + 9; }
      else { mloc = sp3(a) | (sp3(b) << 1) | (side << 2); ux = a + 1; uy = b + 1; uz = s; nbi = 1 + 3 + 9 * (hi ? 2 : 0); }
    } else if (i < 480) {  // edges: 12 x 8
      const int e = (i - 384) >> 3, a = (i - 384) & 7, axis = e >> 2, s1 = e & 1, s2 = (e >> 1) & 1;
      const uint32_t c1 = s1 ? 0u : 0x49u, c2 = s2 ? 0u : 0x49u;
      const int u1 = s1 ? 9 : 0, u2 = s2 ? 9 : 0, d1 = s1 ? 2 : 0, d2 = s2 ? 2 : 0;
      if (axis == 0) { mloc = sp3(a) | (c1 << 1) | (c2 << 2); ux = a + 1; uy = u1; uz = u2; nbi = 1 + 3 * d1 + 9 * d2; }
      else if (axis == 1) { mloc = c1 | (sp3(a) << 1) | (c2 << 2); ux = u1; uy = a + 1; uz = u2; nbi = d1 + 3 + 9 * d2; }
      else { mloc = c1 | (c2 << 1) | (sp3(a) << 2); ux = u1; uy = u2; uz = a + 1; nbi = d1 + 3 * d2 + 9; }
    } else {  // corners
      const int c = i - 480, sx = c & 1, sy = (c >> 1) & 1, sz = (c >> 2) & 1;
      mloc = (sx ? 0u : 0x49u) | ((sy ? 0u : 0x49u) << 1) | ((sz ? 0u : 0x49u) << 2);
      ux = sx ? 9 : 0; uy = sy ? 9 : 0; uz = sz ? 9 : 0;
      nbi = (sx ? 2 : 0) + 3 * (sy ? 2 : 0) + 9 * (sz ? 2 : 0);
    }
    const uint32_t b0 = cnb[nbi];
    ctile[(uz * CW + uy) * CW + ux] = b0 != ~0u ? __ldg(ec + b0 + mloc) : (T)0;
  }
  __syncthreads();  // the caller reads halo entries written by other threads
}

// P ec at fine tile coordinate (ux,uy,uz) (fine local + 1); ctile coordinate = coarse local + 1.
// Even fine local coordinate l -> coarse l/2 (w 1); odd -> (l-1)/2, (l+1)/2 (w 1/2 each).
template <typename T>
__device__ __forceinline__ T prolong_at(const T* ctile, int ux, int uy, int uz) {
  const int lx = ux - 1, ly = uy - 1, lz = uz - 1;
  const int ax = (lx >> 1) + 1, ay = (ly >> 1) + 1, az = (lz >> 1) + 1;  // floor(l/2) + 1
  const int ox = lx & 1, oy = ly & 1, oz = lz & 1;
  const T* c = ctile + (az * CW + ay) * CW + ax;
  // the +1 neighbours exist (index <= CW-1) exactly when the coordinate is odd
  T v00 = c[0];
  T v01 = oy ? c[CW] : (T)0;
  T v10 = oz ? c[CW * CW] : (T)0;
  T v11 = (oy && oz) ? c[CW * CW + CW] : (T)0;
  if (ox) {
    v00 = (T)0.5 * (v00 + c[1]);
    if (oy) v01 = (T)0.5 * (v01 + c[CW + 1]);
    if (oz) v10 = (T)0.5 * (v10 + c[CW * CW + 1]);
    if (oy && oz) v11 = (T)0.5 * (v11 + c[CW * CW + CW + 1]);
  }
  const T y0 = oy ? (T)0.5 * (v00 + v01) : v00;
  const T y1 = oy ? (T)0.5 * (v10 + v11) : v10;
  return oz ? (T)0.5 * (y0 + y1) : y0;
}

}  // namespace s16

// ------------------------------------------------------------------ 16^3 stencil SpMV (finest level)
// 256 threads: thread = one 2x2 (x, y) quad column over 4 z planes (64 quads x 4 z segments).
// Natural tile with a one-node halo; local x sits at offset x + 1 so that the pairs (x0-1, x0)
// and (x0+1, x0+2) a quad's row needs are 8-byte (FP32) / 16-byte (FP64) aligned, and the row
// stride of 24 puts the two quad rows of a half-warp on disjoint banks.  The planes are swept
// in z once: each plane's in-plane sums go to the output row of the plane itself (centre,
// in-plane edges) and to the rows above and below (edges and corners), so a thread keeps two
// accumulators per node instead of three planes of sums.
namespace n16 {
// ZT: z planes per thread (2, 4 or 8); the CTA has 1024 / ZT threads (64 quad columns x 16 / ZT
// z segments).  The arithmetic of a node, and every per-block sum, is the same for every ZT.
constexpr int N = 4096;
template <int ZT>
struct Zt {
  static constexpr int NT = 1024 / ZT;
};
constexpr int RS = 24, PS = 18 * RS + 4, TILE = 18 * PS;
__device__ __forceinline__ int nat(int ux, int uy, int uz) { return uz * PS + uy * RS + ux; }  // u = local + 1

template <typename T>
struct Pair;
template <>
struct Pair<float> {
  typedef float2 type;
};
template <>
struct Pair<double> {
  typedef double2 type;
};

// the 4 x 4 patch (rows y0-1..y0+2, columns x0-1..x0+2) of tile plane uz around quad (x0, y0)
template <typename T, int RSX>
__device__ __forceinline__ void patch(const T* tile, int off, T r[4][4]) {
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const typename Pair<T>::type l = *reinterpret_cast<const typename Pair<T>::type*>(tile + off + j * RSX);
    const typename Pair<T>::type h = *reinterpret_cast<const typename Pair<T>::type*>(tile + off + j * RSX + 2);
    r[j][0] = l.x;
    r[j][1] = l.y;
    r[j][2] = h.x;
    r[j][3] = h.y;
  }
}

// in-plane sums of the quad's 4 nodes: tz = ce*faces + cc*diagonals (for the rows z-1, z+1),
// own = c0*centre + ce*diagonals (for row z)
template <typename T>
__device__ __forceinline__ void plane_terms(const T r[4][4], T c0, T ce, T cc, T tz[4], T own[4], T ctr[4]) {
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int e = 2 * j + i, R = j + 1, Cc = i + 1;
      const T pf = r[R][Cc - 1] + r[R][Cc + 1] + r[R - 1][Cc] + r[R + 1][Cc];
      const T pe = r[R - 1][Cc - 1] + r[R - 1][Cc + 1] + r[R + 1][Cc - 1] + r[R + 1][Cc + 1];
      tz[e] = ce * pf + cc * pe;
      own[e] = c0 * r[R][Cc] + ce * pe;
      ctr[e] = r[R][Cc];
    }
}

// KIND 0: q = A a, part = a.q;  1: an = bvec + beta a, q = A an, part = an.q;
// 2: an = a + beta bvec (FP64 solution + correction of type E), q = rhs - A an.
// beta_dev (packed launches): the cloud's beta, in place of the beta argument.
template <typename T, int KIND, typename E, int ZT>
__global__ void __launch_bounds__(Zt<ZT>::NT, (sizeof(T) == 4 ? 5 : 3) * ZT / 4)
    k_spmv16(uint32_t D, const T* __restrict__ a, const E* __restrict__ bvec, T* __restrict__ an, T beta,
             T* __restrict__ q, T c0, T ce, T cc, const T* __restrict__ rhs, double* __restrict__ part,
             const double* __restrict__ beta_dev) {
  constexpr int NT = Zt<ZT>::NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* tile = reinterpret_cast<T*>(smem_raw);
  __shared__ uint32_t nb[27];
  const int res = 1 << D;
  {
    const uint64_t nl = 1ull << (3 * D);
    a = cloud_slice(a, nl);
    bvec = cloud_slice(bvec, nl);
    an = cloud_slice(an, nl);
    q = cloud_slice(q, nl);
    rhs = cloud_slice(rhs, nl);
    part = cloud_slice(part, gridDim.x);
    if (beta_dev) beta = (T)beta_dev[blockIdx.y];
  }
  const uint32_t blk = blockIdx.x;
  const uint64_t base = (uint64_t)blk * N;
  uint32_t bx, by, bz;
  unmorton3(blk, bx, by, bz);
  const int t = threadIdx.x;
  s16::neighbour_bases(nb, bx, by, bz, res >> 4);
  auto val = [&](uint32_t m) -> T {
    if (KIND == 0) return __ldg(a + m);
    if (KIND == 1) return (T)__ldg(bvec + m) + beta * __ldg(a + m);
    // KIND 2 with beta 0: a cloud of a packed launch that has stopped keeps its solution
    return beta == (T)0 ? __ldg(a + m) : __ldg(a + m) + beta * (T)__ldg(bvec + m);
  };
#pragma unroll
  for (int r = 0; r < ZT; ++r) {
    const int qd = t + NT * r;
    int lx, ly, lz;
    s16::quad_coords(qd, lx, ly, lz);
    const uint64_t m = base + 4 * qd;
    typename s16::Vec4<T>::type v = s16::ld4(a + m);
    if (KIND != 0) {
      const typename s16::Vec4<E>::type bv = s16::ld4(bvec + m);
      if (KIND == 1) {
        v.x = (T)bv.x + beta * v.x; v.y = (T)bv.y + beta * v.y; v.z = (T)bv.z + beta * v.z; v.w = (T)bv.w + beta * v.w;
      } else if (beta != (T)0) {
        v.x += beta * (T)bv.x; v.y += beta * (T)bv.y; v.z += beta * (T)bv.z; v.w += beta * (T)bv.w;
      }
      s16::st4(an + m, v);
    }
    T* p0 = tile + nat(lx + 1, ly + 1, lz + 1);
    p0[0] = v.x;
    p0[1] = v.y;
    p0[RS] = v.z;
    p0[RS + 1] = v.w;
  }
  __syncthreads();  // nb
  s16::load_halo<NT>(tile, a, nb, [](int ux, int uy, int uz) { return nat(ux, uy, uz); }, val);
  __syncthreads();
  const int qi = t & 63, zs = t >> 6;
  const int x0 = 2 * (qi & 7), y0 = 2 * (qi >> 3), z0 = ZT * zs;
  const uint32_t mq = s16::sp4(x0) | (s16::sp4(y0) << 1);
  T cur[4] = {0, 0, 0, 0}, nxt[4] = {0, 0, 0, 0}, cprev[4] = {0, 0, 0, 0};
  double pv[ZT];  // per plane: the quad's four products of the dot
#pragma unroll
  for (int p = 0; p < ZT + 2; ++p) {  // tile plane z0 + p = local z0 + p - 1
    T r[4][4], tz[4], own[4], ctr[4];
    patch<T, RS>(tile, nat(x0, y0, z0 + p), r);
    plane_terms<T>(r, c0, ce, cc, tz, own, ctr);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      cur[e] += tz[e];
      nxt[e] += own[e];
    }
    if (p >= 2) {  // row of local z0 + p - 2 is complete
      const uint64_t m = base + (mq | (s16::sp4(z0 + p - 2) << 2));
      typename s16::Vec4<T>::type o;
      if (KIND == 2) {
        const typename s16::Vec4<T>::type rv = s16::ld4(rhs + m);
        o.x = rv.x - cur[0]; o.y = rv.y - cur[1]; o.z = rv.z - cur[2]; o.w = rv.w - cur[3];
      } else {
        o.x = cur[0]; o.y = cur[1]; o.z = cur[2]; o.w = cur[3];
        double a4 = 0.0;
#pragma unroll
        for (int e = 0; e < 4; ++e) a4 += (double)cprev[e] * (double)cur[e];
        pv[p - 2] = a4;
      }
      s16::st4(q + m, o);
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      cur[e] = nxt[e];
      nxt[e] = tz[e];
      cprev[e] = ctr[e];
    }
  }
  if (KIND != 2) {
    __syncthreads();  // the tile's last reads: its memory takes the per-plane sums
    double* red = reinterpret_cast<double*>(smem_raw);
#pragma unroll
    for (int k = 0; k < ZT; ++k) red[(z0 + k) * 64 + qi] = pv[k];
    const double sdot = s16::block_sum_fixed(red);
    if (t == 0) part[blk] = sdot;
  }
}
template <typename T>
constexpr size_t smem_bytes() {
  return sizeof(T) * TILE;
}
}  // namespace n16

// ------------------------------------------------------------------ 16^3 residual + restriction
// Two launches, no redundant work.  k_resid16: r = f - A e on the block's 16^3 nodes (the
// SpMV's tile and quad columns), then (a) the part of the restriction to the block's 8^3 coarse
// nodes that comes from its own fine nodes, and (b) the restriction partials its high faces
// (local 15) owe the coarse nodes of its high neighbours: per face the sum over the face's other
// two axes (8 x 8), per edge over the remaining axis (8), and the corner (1), into a face buffer
// of 224 values per block.  k_restrict_faces adds to the coarse nodes on each block's low faces
// these partials of its low neighbours, scaled by 1/2 per crossed axis.  Restriction: coarse c
// gathers fine 2c-1, 2c, 2c+1 per axis with weights 1/2, 1, 1/2.
namespace r16 {
constexpr int N = 4096, FACE = 224;  // ZT, NT: as n16 (the residual is the same for every ZT)
// face buffer layout: [0,64) x face (cy + 8 cz), [64,128) y face (cx + 8 cz), [128,192) z face
// (cx + 8 cy), [192,200) xy edge (cz), [200,208) xz edge (cy), [208,216) yz edge (cx), 216 corner
constexpr int RSR = 20, PSR = 16 * RSR + 8, RTILE = 16 * PSR;  // half-warps of the restriction on disjoint banks
__device__ __forceinline__ int ridx(int x, int y, int z) { return z * PSR + y * RSR + x; }  // local coordinates

template <typename T, bool FACES, int ZT>
__global__ void __launch_bounds__(n16::Zt<ZT>::NT, (sizeof(T) == 4 ? 4 : 2) * ZT / 4)
    k_resid16(uint32_t D, const T* __restrict__ e, const T* __restrict__ f, T* __restrict__ fc,
              T* __restrict__ face, T c0, T ce, T cc, const T* __restrict__ table) {
  constexpr int NT = n16::Zt<ZT>::NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* et = reinterpret_cast<T*>(smem_raw);  // n16::TILE
  T* rt = et + n16::TILE;                  // RTILE
  __shared__ uint32_t nb[27];
  const int res = 1 << D;
  {
    const uint64_t nl = 1ull << (3 * D);
    e = cloud_slice(e, nl);
    f = cloud_slice(f, nl);
    fc = cloud_slice(fc, nl / 8);
    face = cloud_slice(face, (uint64_t)gridDim.x * FACE);
  }
  const uint32_t blk = blockIdx.x;
  const uint64_t base = (uint64_t)blk * N;
  uint32_t bx, by, bz;
  unmorton3(blk, bx, by, bz);
  const int ox = (int)bx * 16, oy = (int)by * 16, oz = (int)bz * 16;
  const int t = threadIdx.x;
  s16::neighbour_bases(nb, bx, by, bz, res >> 4);
#pragma unroll
  for (int r = 0; r < ZT; ++r) {
    const int qd = t + NT * r;
    int lx, ly, lz;
    s16::quad_coords(qd, lx, ly, lz);
    const typename s16::Vec4<T>::type ev = s16::ld4(e + base + 4 * qd);
    T* p0 = et + n16::nat(lx + 1, ly + 1, lz + 1);
    p0[0] = ev.x;
    p0[1] = ev.y;
    p0[n16::RS] = ev.z;
    p0[n16::RS + 1] = ev.w;
  }
  __syncthreads();  // nb
  s16::load_halo<NT>(et, e, nb, [](int ux, int uy, int uz) { return n16::nat(ux, uy, uz); },
                    [&](uint32_t m) { return __ldg(e + m); });
  __syncthreads();
  {  // r = f - A e on quad columns, z swept once
    const int qi = t & 63, zs = t >> 6;
    const int x0 = 2 * (qi & 7), y0 = 2 * (qi >> 3), z0 = ZT * zs;
    const uint32_t mq = s16::sp4(x0) | (s16::sp4(y0) << 1);
    T cur[4] = {0, 0, 0, 0}, nxt[4] = {0, 0, 0, 0};
#pragma unroll
    for (int p = 0; p < ZT + 2; ++p) {  // local plane z0 + p - 1
      T r[4][4], tz[4], own[4], ctr[4];
      n16::patch<T, n16::RS>(et, n16::nat(x0, y0, z0 + p), r);
      n16::plane_terms<T>(r, c0, ce, cc, tz, own, ctr);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        cur[k] += tz[k];
        nxt[k] += own[k];
      }
      if (p >= 2) {
        const int lz = z0 + p - 2;
        const typename s16::Vec4<T>::type fv = s16::ld4(f + base + (mq | (s16::sp4(lz) << 2)));
        T* q0 = rt + ridx(x0, y0, lz);
        q0[0] = fv.x - cur[0];
        q0[1] = fv.y - cur[1];
        q0[RSR] = fv.z - cur[2];
        q0[RSR + 1] = fv.w - cur[3];
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        cur[k] = nxt[k];
        nxt[k] = tz[k];
      }
    }
  }
  __syncthreads();
  if (FACES && (ox == 0 || oy == 0 || oz == 0)) {
    // nodes on a low domain face: replace the interior row by the face row
    for (int i = t; i < N; i += NT) {
      uint32_t lx, ly, lz;
      unmorton3((uint32_t)i, lx, ly, lz);
      const int mask = ((ox + (int)lx) == 0) | (((oy + (int)ly) == 0) << 1) | (((oz + (int)lz) == 0) << 2);
      if (!mask) continue;
      const int ei = n16::nat(lx + 1, ly + 1, lz + 1);
      T yf = 0, se = 0, sc = 0;
      const T* cm = table + 27 * mask;
#pragma unroll
      for (int o = 0; o < 27; ++o) {
        const int dx = o % 3 - 1, dy = (o / 3) % 3 - 1, dz = o / 9 - 1;
        const int nzc = (dx != 0) + (dy != 0) + (dz != 0);
        const T v = et[ei + dx + n16::RS * dy + n16::PS * dz];
        yf += cm[o] * v;
        if (nzc == 2) se += v;
        else if (nzc == 3) sc += v;
      }
      const T yi = c0 * et[ei] + ce * se + cc * sc;
      rt[ridx(lx, ly, lz)] += yi - yf;
    }
    __syncthreads();
  }
  // own part of the restriction
  const uint64_t cbase = (uint64_t)blk * 512;
#pragma unroll
  for (int ci = t; ci < 512; ci += NT) {
    uint32_t cx, cy, cz;
    unmorton3((uint32_t)ci, cx, cy, cz);
    T s = 0;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz) {
      const int fz = 2 * (int)cz + dz;
      if (fz < 0) continue;
#pragma unroll
      for (int dy = -1; dy <= 1; ++dy) {
        const int fy = 2 * (int)cy + dy;
        if (fy < 0) continue;
        const T wyz = (T)((dy == 0 ? 1.0 : 0.5) * (dz == 0 ? 1.0 : 0.5));
        const T* row = rt + ridx(2 * cx, fy, fz);
        const typename n16::Pair<T>::type pr = *reinterpret_cast<const typename n16::Pair<T>::type*>(row);
        const T left = cx > 0 ? row[-1] : (T)0;
        s += wyz * (pr.x + (T)0.5 * (pr.y + left));
      }
    }
    fc[cbase + ci] = s;
  }
  // restriction partials of the high faces, edges and corner
  {
    T* fb = face + (uint64_t)blk * FACE;
    auto w = [](int d) { return (T)(d == 0 ? 1.0 : 0.5); };
    for (int u = t; u < 217; u += NT) {
      if (u < 192) {  // faces: the two free axes restricted, the face axis at local 15
        const int axis = u >> 6, i = u & 7, j = (u >> 3) & 7;
        T acc = 0;
#pragma unroll
        for (int dj = -1; dj <= 1; ++dj) {
          const int fj = 2 * j + dj;
          if (fj < 0) continue;
#pragma unroll
          for (int di = -1; di <= 1; ++di) {
            const int fi = 2 * i + di;
            if (fi < 0) continue;
            const int x = axis == 0 ? 15 : fi, y = axis == 1 ? 15 : (axis == 0 ? fi : fj), z = axis == 2 ? 15 : fj;
            acc += w(di) * w(dj) * rt[ridx(x, y, z)];
          }
        }
        fb[u] = acc;
      } else if (u < 216) {  // edges: the free axis restricted
        const int e = (u - 192) >> 3, i = (u - 192) & 7;
        T acc = 0;
#pragma unroll
        for (int di = -1; di <= 1; ++di) {
          const int fi = 2 * i + di;
          if (fi < 0) continue;
          const int x = e == 2 ? fi : 15, y = e == 1 ? fi : 15, z = e == 0 ? fi : 15;
          acc += w(di) * rt[ridx(x, y, z)];
        }
        fb[u] = acc;
      } else {
        fb[216] = rt[ridx(15, 15, 15)];
      }
    }
  }
}

// Adds to the coarse nodes on each block's low faces what the fine nodes at local -1 contribute:
// the partials of the low neighbours (k_resid16), 1/2 per axis crossed, fixed order.  Four
// blocks per CTA, 169 boundary coarse nodes per block.
template <typename T>
__global__ void __launch_bounds__(768) k_restrict_faces(uint32_t D, const T* __restrict__ face, T* __restrict__ fc,
                                                       uint32_t nblk) {
  const int nba = 1 << (D - 4);
  face = cloud_slice(face, (uint64_t)nblk * FACE);
  fc = cloud_slice(fc, (uint64_t)nblk * 512);
  const uint32_t blk = blockIdx.x * 4 + threadIdx.x / 192;
  const int j = threadIdx.x % 192;
  if (blk >= nblk || j >= 169) return;
  uint32_t bx, by, bz;
  unmorton3(blk, bx, by, bz);
  int cx, cy, cz;
  if (j < 64) { cx = 0; cy = j & 7; cz = j >> 3; }
  else if (j < 120) { cx = 1 + (j - 64) % 7; cy = 0; cz = (j - 64) / 7; }
  else { cx = 1 + (j - 120) % 7; cy = 1 + (j - 120) / 7; cz = 0; }
  T s = 0;
  bool any = false;
#pragma unroll
  for (int e = 1; e < 8; ++e) {
    const int ex = e & 1, ey = (e >> 1) & 1, ez = e >> 2;
    if ((ex && cx) || (ey && cy) || (ez && cz)) continue;  // only coarse index 0 reaches fine -1
    const int nx = (int)bx - ex, ny = (int)by - ey, nz = (int)bz - ez;
    if (nx < 0 || ny < 0 || nz < 0) continue;  // outside the domain
    (void)nba;
    const T* fb = face + (uint64_t)morton3((uint32_t)nx, (uint32_t)ny, (uint32_t)nz) * FACE;
    T v;
    switch (e) {
      case 1: v = (T)0.5 * fb[cy + 8 * cz]; break;
      case 2: v = (T)0.5 * fb[64 + cx + 8 * cz]; break;
      case 4: v = (T)0.5 * fb[128 + cx + 8 * cy]; break;
      case 3: v = (T)0.25 * fb[192 + cz]; break;
      case 5: v = (T)0.25 * fb[200 + cy]; break;
      case 6: v = (T)0.25 * fb[208 + cx]; break;
      default: v = (T)0.125 * fb[216]; break;
    }
    s += v;
    any = true;
  }
  if (any) fc[(uint64_t)blk * 512 + morton3((uint32_t)cx, (uint32_t)cy, (uint32_t)cz)] += s;
}
template <typename T>
constexpr size_t smem_bytes() {
  return sizeof(T) * (n16::TILE + RTILE);
}
}  // namespace r16

// ------------------------------------------------------------------ 16^3 smoother (levels >= 4)
// Multicolour Gauss-Seidel in the block, blocks coupled through the halo values from before
// the sweep.  Every level's interior stencil has no face couplings, so nodes that share the
// parity of x and y are uncoupled along z: the sweep has 4 phases, one per (x, y) parity class,
// each relaxing whole columns of that class at once (forward order (0,0) (1,0) (0,1) (1,1),
// backward the reverse, each the adjoint of the other).  Thread = one 2x2 quad column over ZT z
// planes of a parity-split tile (below); in phase k it relaxes the class-k column of its quad, sweeping
// the planes once: a plane's ring around the column gives its in-plane edge sum D (diagonals)
// and face-adjacent sum F, and the node at z uses D(z), F(z-1), F(z+1), D(z-1), D(z+1).
// FACES (coarse levels): nodes on the low domain faces use their 27-entry table row, which does
// couple z-neighbours of the same class; those take the values from before the phase (new
// values are written after a barrier), a Jacobi step along the column for those rows only.
namespace g16 {
constexpr int CW = s16::CW;  // ZT, NT: as n16 (a node's relaxation is the same for every ZT)
// Parity-split tile (u = local + 1 in 0..17 per axis): each row holds its even columns (u even)
// first, then its odd ones, HS words each, so the columns of one class that a warp relaxes
// (x0 = 0, 2, .., 14: stride 2 in x) are consecutive words, and its four quad rows (y two apart,
// 2 RS = 40 words = 8 banks apart) fill the 32 banks once: every tile access of a phase is free
// of bank conflicts for FP32, and per half-warp for FP64.
constexpr int HS = 10, RS = 2 * HS, PS = 18 * RS + 4, TILE = 18 * PS;
__device__ __forceinline__ int col(int ux) { return (ux & 1) * HS + (ux >> 1); }
__device__ __forceinline__ int nat(int ux, int uy, int uz) { return uz * PS + uy * RS + col(ux); }

// One phase: new values of the class-CLS column of the thread's quad (planes z0..z0+ZT-1).
// On the thread's own planes the ring members inside its quad come from registers (v), the
// other five from the tile; the two halo planes read all eight.
// ZERO: a forward sweep from zero, in which the classes after CLS are still zero everywhere
// (their loads are skipped; phase 0 needs none).
template <typename T, int CLS, bool ZERO, int ZT>
__device__ __forceinline__ void relax_column(const T* tile, int x0, int y0, int z0, const T (&fv)[ZT][4],
                                             const T (&v)[ZT][4], T ce, T cc, T c0inv, T (&nv)[ZT]) {
  constexpr int CX = CLS & 1, CY = CLS >> 1;
  constexpr int EDX = CX == 0 ? -1 : 1, EDY = CY == 0 ? -1 : 1;  // direction of the external ring side
  constexpr int EFX = (CX ^ 1) | (CY << 1), EFY = CX | ((CY ^ 1) << 1), ED = (CX ^ 1) | ((CY ^ 1) << 1);
  // classes updated before CLS in a forward sweep are 0..CLS-1
  constexpr bool NFX = !ZERO || EFX < CLS, NFY = !ZERO || EFY < CLS, ND = !ZERO || ED < CLS;
  if (ZERO && CLS == 0) {
#pragma unroll
    for (int k = 0; k < ZT; ++k) nv[k] = fv[k][CLS] * c0inv;
    return;
  }
  // the ring's columns x-1, x, x+1 (x = x0 + CX, tile column x + 1; x0 even): their row offsets
  const int xh = x0 >> 1;
  const int cm = CX * HS + xh, cz = (1 - CX) * HS + xh + CX, cp = CX * HS + xh + 1;
  const int cxe = EDX < 0 ? cm : cp;  // the external column x + EDX
  const T* rbase = tile + (y0 + CY) * RS;  // ring row y-1 of tile plane 0
  T Dm = 0, Fm = 0, D0 = 0, F0 = 0;
#pragma unroll
  for (int p = 0; p < ZT + 2; ++p) {  // local plane z0 + p - 1
    const T* r0 = rbase + (z0 + p) * PS;
    T Dp = 0, Fp = 0;
    if (p >= 1 && p <= ZT) {  // own plane: (x', y), (x, y'), (x', y') from registers
      const int k = p - 1;
      const T* rr = r0 + (EDY + 1) * RS;  // external row: columns x-1, x, x+1
      T q0 = 0, q1 = 0, q2 = 0;
      if (ND) {
        q0 = rr[cm];
        q2 = rr[cp];
      }
      if (NFY) q1 = rr[cz];
      // the same pairing as a halo plane's (row y-1 pair + row y+1 pair), so that a node's sums
      // do not depend on which of its planes are a thread's own
      if (ND) Dp = (q0 + q2) + (r0[(1 - EDY) * RS + cxe] + v[k][ED]);
      if (NFY) Fp += q1 + v[k][EFY];
      if (NFX) Fp += r0[RS + cxe] + v[k][EFX];
    } else {  // halo plane: the whole ring from the tile
      const T a0 = r0[cm], a1 = r0[cz], a2 = r0[cp];
      const T c0v = r0[2 * RS + cm], c1 = r0[2 * RS + cz], c2 = r0[2 * RS + cp];
      Dp = (a0 + a2) + (c0v + c2);
      Fp = (a1 + c1) + (r0[RS + cm] + r0[RS + cp]);
    }
    if (p >= 2) {  // node at local z0 + p - 2: edges D0 + Fm + Fp, corners Dm + Dp
      const int k = p - 2;
      nv[k] = (fv[k][CLS] - ce * (D0 + Fm + Fp) - cc * (Dm + Dp)) * c0inv;
    }
    Dm = D0;
    Fm = F0;
    D0 = Dp;
    F0 = Fp;
  }
}

// MODE 0: xo = sweep(xi); 1: xo = sweep(0); 2: xo = sweep(xi + P ec).  DOT: part = f.xo
// MODE 3 (finest level, forward): first the CG update x += alpha d, r -= alpha q in place
// (pointwise), then xo = sweep(0) with f = the new r; part = per-block sums of r^2.  A sweep
// from zero reads no halo, so updating r in place is race-free.
template <typename T, int MODE, bool DOT, bool FWD, bool FACES, int ZT>
__global__ void __launch_bounds__(n16::Zt<ZT>::NT, (sizeof(T) == 4 ? 4 : 2) * ZT / 4)
    k_smooth16(uint32_t D, const T* __restrict__ xi, T* __restrict__ xo, const T* __restrict__ f,
               const T* __restrict__ ec, T c0inv, T ce, T cc, const T* __restrict__ table,
               double* __restrict__ part, CgFuse<T> cg) {
  static_assert(MODE != 3 || (FWD && !FACES), "the fused CG update is a forward sweep on the finest level");
  constexpr int NT = n16::Zt<ZT>::NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* tile = reinterpret_cast<T*>(smem_raw);  // TILE
  T* ctile = tile + TILE;                    // CW^3 (MODE 2)
  __shared__ uint32_t nb[27], cnb[27];
  const int res = 1 << D;
  {
    const uint64_t nl = 1ull << (3 * D);
    xi = cloud_slice(xi, nl);
    xo = cloud_slice(xo, nl);
    f = cloud_slice(f, nl);
    ec = cloud_slice(ec, nl / 8);
    part = cloud_slice(part, gridDim.x);
    if (MODE == 3) {
      cg.x = cloud_slice(cg.x, nl);
      cg.d = cloud_slice(cg.d, nl);
      cg.q = cloud_slice(cg.q, nl);
      cg.r = cloud_slice(cg.r, nl);
      if (cg.alpha_dev) cg.alpha = (T)cg.alpha_dev[blockIdx.y];
    }
  }
  const uint32_t blk = blockIdx.x;
  const uint64_t base = (uint64_t)blk * 4096;
  uint32_t bx, by, bz;
  unmorton3(blk, bx, by, bz);
  const int ox = (int)bx * 16, oy = (int)by * 16, oz = (int)bz * 16;
  const int t = threadIdx.x;
  constexpr bool FROM_ZERO = MODE == 1 || MODE == 3;
  if (!FROM_ZERO) s16::neighbour_bases(nb, bx, by, bz, res >> 4);
  else if (t < 27) nb[t] = ~0u;  // zero halo
  if (MODE == 2) s16::load_coarse_tile<NT>(ctile, ec, blk, bx, by, bz, res >> 4, cnb);  // ends with a barrier
  else __syncthreads();                                                                 // nb
  const int qi = t & 63, zs = t >> 6;
  const int x0 = 2 * (qi & 7), y0 = 2 * (qi >> 3), z0 = ZT * zs;
  const uint32_t mq = s16::sp4(x0) | (s16::sp4(y0) << 1);
  T fv[ZT][4], v[ZT][4];
  double rr[ZT];  // MODE 3: per plane, the quad's r^2
#pragma unroll
  for (int k = 0; k < ZT; ++k) {
    const uint64_t m = base + (mq | (s16::sp4(z0 + k) << 2));
    typename s16::Vec4<T>::type fq;
    if (MODE == 3) {  // the CG update of this quad (plain loads: x and r are written here)
      typedef typename s16::Vec4<T>::type V4;
      fq = *reinterpret_cast<const V4*>(cg.r + m);
      if (cg.alpha != (T)0) {  // alpha 0: a cloud of a packed launch that has stopped keeps x and r
        V4 xq = *reinterpret_cast<const V4*>(cg.x + m);
        const V4 dq = s16::ld4(cg.d + m), qq = s16::ld4(cg.q + m);
        xq.x += cg.alpha * dq.x; xq.y += cg.alpha * dq.y; xq.z += cg.alpha * dq.z; xq.w += cg.alpha * dq.w;
        fq.x -= cg.alpha * qq.x; fq.y -= cg.alpha * qq.y; fq.z -= cg.alpha * qq.z; fq.w -= cg.alpha * qq.w;
        s16::st4(cg.x + m, xq);
        s16::st4(cg.r + m, fq);
      }
      rr[k] = (double)fq.x * fq.x + (double)fq.y * fq.y + (double)fq.z * fq.z + (double)fq.w * fq.w;
    } else {
      fq = s16::ld4(f + m);
    }
    fv[k][0] = fq.x; fv[k][1] = fq.y; fv[k][2] = fq.z; fv[k][3] = fq.w;
    if (FROM_ZERO) {
      v[k][0] = v[k][1] = v[k][2] = v[k][3] = (T)0;
    } else {
      const typename s16::Vec4<T>::type xq = s16::ld4(xi + m);
      v[k][0] = xq.x; v[k][1] = xq.y; v[k][2] = xq.z; v[k][3] = xq.w;
    }
  }
  if (MODE == 2) {
    // P ec on the quad column: coarse (cx, cx+1) x (cy, cy+1) at the coarse planes z0/2 .. z0/2+2
    // (z0 even: planes z0, z0+2 lie on a coarse plane, z0+1, z0+3 halfway between two)
    const int ax = x0 / 2 + 1, ay = y0 / 2 + 1, az = z0 / 2 + 1;
    T pl[ZT / 2 + 1][4];
#pragma unroll
    for (int w = 0; w <= ZT / 2; ++w) {
      const T* c = ctile + ((az + w) * CW + ay) * CW + ax;
      const T c00 = c[0], c10 = c[1], c01 = c[CW], c11 = c[CW + 1];
      pl[w][0] = c00;
      pl[w][1] = (T)0.5 * (c00 + c10);
      pl[w][2] = (T)0.5 * (c00 + c01);
      pl[w][3] = (T)0.25 * ((c00 + c10) + (c01 + c11));
    }
#pragma unroll
    for (int k = 0; k < ZT; ++k)  // even planes on a coarse plane, odd halfway between two
#pragma unroll
      for (int e = 0; e < 4; ++e) v[k][e] += (k & 1) ? (T)0.5 * (pl[k / 2][e] + pl[k / 2 + 1][e]) : pl[k / 2][e];
  }
#pragma unroll
  for (int k = 0; k < ZT; ++k) {
    T* p0 = tile + nat(0, y0 + 1, z0 + k + 1);
    p0[col(x0 + 1)] = v[k][0];
    p0[col(x0 + 2)] = v[k][1];
    p0[RS + col(x0 + 1)] = v[k][2];
    p0[RS + col(x0 + 2)] = v[k][3];
  }
  s16::load_halo<NT>(tile, xi, nb, [](int ux, int uy, int uz) { return nat(ux, uy, uz); },
                    [&](uint32_t m) -> T { return FROM_ZERO ? (T)0 : __ldg(xi + m); });
  __syncthreads();
  if (MODE == 2) {  // add P ec on the halo shell (in-domain positions only)
    for (int i = t; i < 1736; i += NT) {
      int ux, uy, uz;
      halo_u<16>(i, ux, uy, uz);
      const int gx = ox - 1 + ux, gy = oy - 1 + uy, gz = oz - 1 + uz;
      if (gx < 0 || gy < 0 || gz < 0 || gx >= res || gy >= res || gz >= res) continue;
      tile[nat(ux, uy, uz)] += s16::prolong_at<T>(ctile, ux, uy, uz);
    }
    __syncthreads();
  }
  const bool faces = FACES && (ox == 0 || oy == 0 || oz == 0);
#pragma unroll
  for (int ph = 0; ph < 4; ++ph) {
    const int cls = FWD ? ph : 3 - ph;
    const int cx = cls & 1, cy = cls >> 1;
    const int x = x0 + cx, y = y0 + cy;
    T nv[ZT];
    constexpr bool ZERO = FROM_ZERO && FWD;
    switch (cls) {
      case 0: relax_column<T, 0, ZERO, ZT>(tile, x0, y0, z0, fv, v, ce, cc, c0inv, nv); break;
      case 1: relax_column<T, 1, ZERO, ZT>(tile, x0, y0, z0, fv, v, ce, cc, c0inv, nv); break;
      case 2: relax_column<T, 2, ZERO, ZT>(tile, x0, y0, z0, fv, v, ce, cc, c0inv, nv); break;
      default: relax_column<T, 3, ZERO, ZT>(tile, x0, y0, z0, fv, v, ce, cc, c0inv, nv); break;
    }
    if (faces) {  // low-domain-face nodes of this column: their table rows, neighbours from the tile
#pragma unroll 1
      for (int k = 0; k < ZT; ++k) {
        const int z = z0 + k;
        const int mask = ((ox + x) == 0) | (((oy + y) == 0) << 1) | (((oz + z) == 0) << 2);
        if (!mask) continue;
        const T* cm = table + 27 * mask;
        T off = 0;
#pragma unroll 1
        for (int o = 0; o < 27; ++o) {
          if (o == 13) continue;
          off += cm[o] * tile[nat(x + 1 + (o % 3 - 1), y + 1 + ((o / 3) % 3 - 1), z + 1 + (o / 9 - 1))];
        }
        T fk = fv[0][cls];
#pragma unroll
        for (int kk = 1; kk < ZT; ++kk)
          if (kk == k) fk = fv[kk][cls];
        const T nvk = (fk - off) / cm[13];
#pragma unroll
        for (int kk = 0; kk < ZT; ++kk)
          if (kk == k) nv[kk] = nvk;
      }
    }
    if (FACES) __syncthreads();  // same-class column neighbours were read with their old values
#pragma unroll
    for (int k = 0; k < ZT; ++k) {
      v[k][cls] = nv[k];
      tile[nat(x + 1, y + 1, z0 + k + 1)] = nv[k];
    }
    __syncthreads();
  }
  double acc[ZT];  // DOT: per plane, the quad's f.x
#pragma unroll
  for (int k = 0; k < ZT; ++k) {
    const uint64_t m = base + (mq | (s16::sp4(z0 + k) << 2));
    typename s16::Vec4<T>::type o;
    o.x = v[k][0]; o.y = v[k][1]; o.z = v[k][2]; o.w = v[k][3];
    s16::st4(xo + m, o);
    acc[k] = 0.0;
    if (DOT)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[k] += (double)fv[k][e] * (double)v[k][e];
  }
  if (DOT || MODE == 3) {
    // the last phase ended with a barrier: the tile's memory takes the per-plane sums
    double* red = reinterpret_cast<double*>(smem_raw);
#pragma unroll
    for (int k = 0; k < ZT; ++k) red[(z0 + k) * 64 + qi] = MODE == 3 ? rr[k] : acc[k];
    const double sum = s16::block_sum_fixed(red);
    if (t == 0) part[blk] = sum;
  }
}
template <typename T>
constexpr size_t smem_bytes(int mode) {
  return sizeof(T) * (TILE + (mode == 2 ? CW * CW * CW : 0));
}
}  // namespace g16

template <typename T>
DevCoef<T> dev_coef(const LevelCoef& L, const T* table) {
  DevCoef<T> k;
  k.c0 = (T)L.c0;
  k.ce = (T)L.ce;
  k.cc = (T)L.cc;
  k.table = table;
  k.has_faces = L.has_faces ? 1 : 0;
  return k;
}

inline int tile_for(uint32_t D) { return D >= 4 ? 16 : 8; }

template <typename T, int TB, int MODE, bool DOT, bool FWD>
void launch_smooth(cudaStream_t s, uint32_t D, const T* xi, T* xo, const T* f, const T* ec, const DevCoef<T>& k,
                   double* part, uint32_t clouds) {
  using G = Geo<TB>;
  constexpr int CW = TB / 2 + 2;
  const size_t sm = sizeof(T) * (G::W * G::W * G::W + G::N + (MODE == 2 ? CW * CW * CW : 0));
  const unsigned nb = 1u << (3 * (D - (TB == 16 ? 4 : 3)));
  allow_smem(k_smooth<T, TB, MODE, DOT, FWD>, sm);
  k_smooth<T, TB, MODE, DOT, FWD><<<dim3(nb, clouds), G::THREADS, sm, s>>>(D, xi, xo, f, ec, k, part);
}

template <typename T, int TB>
void smooth_dispatch(cudaStream_t s, uint32_t D, const T* xi, T* xo, const T* f, const T* ec, const DevCoef<T>& k,
                     int mode, bool forward, double* part, uint32_t clouds) {
#define PR_SM(M, DT, FW) launch_smooth<T, TB, M, DT, FW>(s, D, xi, xo, f, ec, k, part, clouds)
  if (mode == 1) {
    if (forward) PR_SM(1, false, true);
    else PR_SM(1, false, false);
  } else if (mode == 2) {
    if (part) {
      if (forward) PR_SM(2, true, true);
      else PR_SM(2, true, false);
    } else {
      if (forward) PR_SM(2, false, true);
      else PR_SM(2, false, false);
    }
  } else {
    if (part) {
      if (forward) PR_SM(0, true, true);
      else PR_SM(0, true, false);
    } else {
      if (forward) PR_SM(0, false, true);
      else PR_SM(0, false, false);
    }
  }
#undef PR_SM
}

// ------------------------------------------------------------------ the z-segment autotuner
// The 16^3 block kernels (SpMV, residual + restriction, smoother) run with ZT = 2, 4 or 8 z planes
// per thread, i.e. 512, 256 or 128 threads per 16^3 brick: more planes per thread read fewer halo
// planes from shared memory per node but leave fewer threads to hide latency.  Every ZT computes
// the same values (per-block sums in a fixed order), so the choice is free and made by timing: the
// first FP32 launch of a (kernel family, level, launch size) key times each ZT (one warm-up and
// three timed launches on the launch's own buffers; every candidate writes what the real launch
// then overwrites) and keeps the fastest for the process.  FP64 launches and launches inside a
// stream capture use ZT = 4.  PR_AUTOTUNE=0 fixes ZT = 4; PR_ZT=2|4|8 forces one.
enum TuneFamily { kTuneSpmv = 0, kTuneResid = 1, kTuneSmooth = 2, kTuneSmoothPost = 3 };
struct TuneTable {
  std::mutex mu;
  std::map<std::tuple<int, int, int, int>, int> zt;  // (device, family, level, log2 blocks) -> ZT
  std::string log;
};
TuneTable& tune_table() {
  static TuneTable* t = new TuneTable();  // never destroyed
  return *t;
}
const char* family_name(int f) {
  return f == kTuneSpmv ? "spmv16" : (f == kTuneResid ? "resid16" : (f == kTuneSmooth ? "smooth16" : "smooth16-post"));
}
// PR_ZT_<FAMILY> (e.g. PR_ZT_SPMV16), else PR_ZT, forces a choice; read at every launch, so that a
// process may switch
int forced_zt(int family) {
  auto valid = [](const char* v) { return v && (std::atoi(v) == 2 || std::atoi(v) == 4 || std::atoi(v) == 8); };
  char name[32];
  std::snprintf(name, sizeof(name), "PR_ZT_%s", family == kTuneSpmv ? "SPMV16" : (family == kTuneResid ? "RESID16" : "SMOOTH16"));
  // (both smoother families answer to PR_ZT_SMOOTH16)
  if (valid(std::getenv(name))) return std::atoi(std::getenv(name));
  if (valid(std::getenv("PR_ZT"))) return std::atoi(std::getenv("PR_ZT"));
  const char* a = std::getenv("PR_AUTOTUNE");
  return (a && std::atoi(a) == 0) ? 4 : 0;
}

// Runs launch(zt) with the ZT of the key, timing the candidates first for a new key.
template <typename L>
void tuned_launch(cudaStream_t s, int family, uint32_t level, uint64_t blocks, bool tunable, L launch) {
  if (!tunable) {
    launch(4);
    return;
  }
  if (const int f = forced_zt(family)) {
    launch(f);
    return;
  }
  int dev = 0;
  PR_CUDA(cudaGetDevice(&dev));
  int bin = 0;
  while ((2ull << bin) <= blocks) ++bin;
  const auto key = std::make_tuple(dev, family, (int)level, bin);
  TuneTable& tt = tune_table();
  {
    std::lock_guard<std::mutex> g(tt.mu);
    auto it = tt.zt.find(key);
    if (it != tt.zt.end()) {
      launch(it->second);
      return;
    }
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  PR_CUDA(cudaStreamIsCapturing(s, &cs));
  if (cs != cudaStreamCaptureStatusNone) {
    launch(4);
    return;
  }
  cudaEvent_t e0, e1;
  PR_CUDA(cudaEventCreate(&e0));
  PR_CUDA(cudaEventCreate(&e1));
  const int cand[3] = {2, 4, 8};
  float ms[3];
  for (int k = 0; k < 3; ++k) {
    launch(cand[k]);
    PR_CUDA(cudaEventRecord(e0, s));
    for (int r = 0; r < 3; ++r) launch(cand[k]);
    PR_CUDA(cudaEventRecord(e1, s));
    PR_CUDA(cudaEventSynchronize(e1));
    PR_CUDA(cudaEventElapsedTime(&ms[k], e0, e1));
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  int best = 1;  // ZT = 4 unless another is faster
  for (int k = 0; k < 3; ++k)
    if (ms[k] < ms[best]) best = k;
  {
    std::lock_guard<std::mutex> g(tt.mu);
    tt.zt[key] = cand[best];
    char line[200];
    std::snprintf(line, sizeof(line), "%s level %u blocks 2^%d: ZT 2/4/8 = %.4f/%.4f/%.4f ms -> ZT %d\n",
                  family_name(family), level, bin, ms[0] / 3, ms[1] / 3, ms[2] / 3, cand[best]);
    tt.log += line;
  }
  launch(cand[best]);
}

template <typename T, int MODE, bool DOT, bool FWD, bool FACES>
void launch_s16(cudaStream_t s, uint32_t D, const T* xi, T* xo, const T* f, const T* ec, const LevelCoef& L,
                const T* table, double* part, uint32_t clouds) {
  const size_t sm = g16::smem_bytes<T>(MODE);
  const dim3 grid(1u << (3 * (D - 4)), clouds);
  auto go = [&](auto z) {
    constexpr int ZT = decltype(z)::value;
    allow_smem(g16::k_smooth16<T, MODE, DOT, FWD, FACES, ZT>, sm);
    g16::k_smooth16<T, MODE, DOT, FWD, FACES, ZT><<<grid, n16::Zt<ZT>::NT, sm, s>>>(
        D, xi, xo, f, ec, (T)(1.0 / L.c0), (T)L.ce, (T)L.cc, table, part, CgFuse<T>());
  };
  constexpr bool kTunable = std::is_same<T, float>::value && MODE != 0;
  tuned_launch(s, MODE == 2 ? kTuneSmoothPost : kTuneSmooth, D, (uint64_t)grid.x * grid.y, kTunable, [&](int zt) {
    if constexpr (kTunable) {
      if (zt == 2) return go(std::integral_constant<int, 2>());
      if (zt == 8) return go(std::integral_constant<int, 8>());
    }
    go(std::integral_constant<int, 4>());
  });
}

template <typename T, int MODE, bool DOT, bool FWD>
void launch_s16f(cudaStream_t s, uint32_t D, const T* xi, T* xo, const T* f, const T* ec, const LevelCoef& L,
                 const T* table, double* part, uint32_t clouds) {
  if (L.has_faces) launch_s16<T, MODE, DOT, FWD, true>(s, D, xi, xo, f, ec, L, table, part, clouds);
  else launch_s16<T, MODE, DOT, FWD, false>(s, D, xi, xo, f, ec, L, table, part, clouds);
}

template <typename T>
void smooth16_dispatch(cudaStream_t s, const LevelCoef& L, uint32_t D, const T* xi, T* xo, const T* f, const T* ec,
                       const T* table, int mode, bool forward, double* part, uint32_t clouds) {
#define PR_S16(M, DT, FW) launch_s16f<T, M, DT, FW>(s, D, xi, xo, f, ec, L, table, part, clouds)
  if (mode == 1) {
    if (forward) PR_S16(1, false, true);
    else PR_S16(1, false, false);
  } else if (mode == 2) {
    if (part) {
      if (forward) PR_S16(2, true, true);
      else PR_S16(2, true, false);
    } else {
      if (forward) PR_S16(2, false, true);
      else PR_S16(2, false, false);
    }
  } else {
    if (part) {
      if (forward) PR_S16(0, true, true);
      else PR_S16(0, true, false);
    } else {
      if (forward) PR_S16(0, false, true);
      else PR_S16(0, false, false);
    }
  }
#undef PR_S16
}

}  // namespace

// ====================================================================== host side
LevelCoef level_coef(uint32_t D, uint32_t l, double shift_l) {
  // 1-D Galerkin recurrence (p^T m p for the linear prolongation p), from the fine level:
  //   interior diagonal m0 -> 1.5 m0 + 2 m1, off-diagonal m1 -> m1 + m0/4,
  //   node-0 diagonal  mb -> mb + m1 + m0/4  (the fine node -1 does not exist)
  double m0 = 2.0 / 3.0, m1 = 1.0 / 6.0, mb = 2.0 / 3.0;
  double s0 = 2.0, s1 = -1.0, sb = 2.0;
  for (uint32_t k = D; k > l; --k) {
    const double nm0 = 1.5 * m0 + 2.0 * m1, nm1 = m1 + 0.25 * m0, nmb = mb + m1 + 0.25 * m0;
    const double ns0 = 1.5 * s0 + 2.0 * s1, ns1 = s1 + 0.25 * s0, nsb = sb + s1 + 0.25 * s0;
    m0 = nm0;
    m1 = nm1;
    mb = nmb;
    s0 = ns0;
    s1 = ns1;
    sb = nsb;
  }
  const double H = 1.0 / (double)(1u << D);
  LevelCoef L;
  L.depth = l;
  L.shift = shift_l;
  auto M = [&](int d, bool b) { return d == 0 ? (b ? mb : m0) : m1; };
  auto S = [&](int d, bool b) { return d == 0 ? (b ? sb : s0) : s1; };
  for (int mask = 0; mask < 8; ++mask)
    for (int o = 0; o < 27; ++o) {
      const int dx = o % 3 - 1, dy = (o / 3) % 3 - 1, dz = o / 9 - 1;
      const bool bxm = mask & 1, bym = mask & 2, bzm = mask & 4;
      double v = H * (S(dx, bxm) * M(dy, bym) * M(dz, bzm) + M(dx, bxm) * S(dy, bym) * M(dz, bzm) +
                      M(dx, bxm) * M(dy, bym) * S(dz, bzm));
      if (o == 13) v += shift_l;
      L.table[mask][o] = v;
    }
  // interior values by offset class, o = (dx+1) + 3(dy+1) + 9(dz+1)
  L.c0 = L.table[0][13];
  L.ce = L.table[0][2 + 3 * 2 + 9 * 1];  // (1,1,0)
  L.cc = L.table[0][2 + 3 * 2 + 9 * 2];  // (1,1,1)
  L.cf = L.table[0][2 + 3 * 1 + 9 * 1];  // (1,0,0): 0 in exact arithmetic
  if (std::fabs(L.cf) > 1e-12 * std::fabs(L.c0))
    throw Error(PR_ERR_INTERNAL, "multigrid level has a non-zero interior face coupling");
  L.cf = 0.0;
  for (int mask = 0; mask < 8; ++mask)
    for (int o = 0; o < 27; ++o)
      if (std::fabs(L.table[mask][o]) <= 1e-12 * std::fabs(L.c0)) L.table[mask][o] = 0.0;
  L.has_faces = (l < D);
  return L;
}

template <typename T>
void mg_smooth(cudaStream_t s, const LevelCoef& L, const T* table, const T* xi, T* xo, const T* f, const T* ec,
               int mode, bool forward, double* part, uint32_t clouds) {
  const uint32_t D = L.depth;
  const DevCoef<T> k = dev_coef<T>(L, table);
  if (tile_for(D) == 16) smooth16_dispatch<T>(s, L, D, xi, xo, f, ec, table, mode, forward, part, clouds);
  else smooth_dispatch<T, 8>(s, D, xi, xo, f, ec, k, mode, forward, part, clouds);
  PR_CHECK_LAUNCH();
}

template <typename T>
void mg_cg_update_presmooth(cudaStream_t s, const LevelCoef& L, const T* table, const CgFuse<T>& cg, T* xo,
                            double* part, uint32_t clouds) {
  const uint32_t D = L.depth;
  if (D < 4 || L.has_faces) throw Error(PR_ERR_INTERNAL, "the fused CG update needs the finest level, depth >= 4");
  const size_t sm = g16::smem_bytes<T>(3);
  const dim3 grid(1u << (3 * (D - 4)), clouds);
  auto go = [&](auto z) {
    constexpr int ZT = decltype(z)::value;
    allow_smem(g16::k_smooth16<T, 3, false, true, false, ZT>, sm);
    g16::k_smooth16<T, 3, false, true, false, ZT><<<grid, n16::Zt<ZT>::NT, sm, s>>>(
        D, nullptr, xo, nullptr, nullptr, (T)(1.0 / L.c0), (T)L.ce, (T)L.cc, table, part, cg);
  };
  // in place (x and r), so not timed: ZT = 4 unless forced
  const int zt = std::is_same<T, float>::value && forced_zt(kTuneSmooth) ? forced_zt(kTuneSmooth) : 4;
  if constexpr (std::is_same<T, float>::value) {
    if (zt == 2) go(std::integral_constant<int, 2>());
    else if (zt == 8) go(std::integral_constant<int, 8>());
    else go(std::integral_constant<int, 4>());
  } else {
    go(std::integral_constant<int, 4>());
  }
  PR_CHECK_LAUNCH();
}

template <typename T>
void mg_resid_restrict(cudaStream_t s, const LevelCoef& L, const T* table, const T* e, const T* f, T* fc, T* face,
                       uint32_t clouds) {
  const uint32_t D = L.depth;
  const DevCoef<T> k = dev_coef<T>(L, table);
  if (tile_for(D) == 16) {
    const size_t sm = r16::smem_bytes<T>();
    const unsigned nb = 1u << (3 * (D - 4));
    auto go = [&](auto z, auto fcs) {
      constexpr int ZT = decltype(z)::value;
      constexpr bool FC = decltype(fcs)::value;
      allow_smem(r16::k_resid16<T, FC, ZT>, sm);
      r16::k_resid16<T, FC, ZT><<<dim3(nb, clouds), n16::Zt<ZT>::NT, sm, s>>>(D, e, f, fc, face, (T)L.c0, (T)L.ce,
                                                                              (T)L.cc, table);
    };
    auto go_f = [&](auto z) {
      if (L.has_faces) go(z, std::true_type());
      else go(z, std::false_type());
    };
    constexpr bool kTunable = std::is_same<T, float>::value;
    tuned_launch(s, kTuneResid, D, (uint64_t)nb * clouds, kTunable, [&](int zt) {
      if constexpr (kTunable) {
        if (zt == 2) return go_f(std::integral_constant<int, 2>());
        if (zt == 8) return go_f(std::integral_constant<int, 8>());
      }
      go_f(std::integral_constant<int, 4>());
    });
    PR_CHECK_LAUNCH();
    r16::k_restrict_faces<T><<<dim3((nb + 3) / 4, clouds), 768, 0, s>>>(D, face, fc, nb);
  } else {
    const size_t sm = sizeof(T) * (11 * 11 * 11 + 9 * 9 * 9);
    allow_smem(k_resid_restrict<T, 8>, sm);
    k_resid_restrict<T, 8><<<dim3(1u << (3 * (D - 3)), clouds), Geo<8>::THREADS, sm, s>>>(D, e, f, fc, k);
  }
  PR_CHECK_LAUNCH();
}

size_t mg_face_entries(uint32_t D) { return D >= 4 ? (size_t)r16::FACE << (3 * (D - 4)) : 0; }

template <typename T>
void mg_spmv(cudaStream_t s, const LevelCoef& L, const T* table, const T* z, const T* d, T* dn, double beta,
             bool xpby, T* q, double* part, uint32_t clouds, const double* beta_dev) {
  const uint32_t D = L.depth;
  const DevCoef<T> k = dev_coef<T>(L, table);
  if (L.has_faces) throw Error(PR_ERR_INTERNAL, "mg_spmv is for the finest level");
  if (tile_for(D) == 16) {
    const dim3 g(1u << (3 * (D - 4)), clouds);
    const size_t sm = n16::smem_bytes<T>();
    auto go = [&](auto zc) {
      constexpr int ZT = decltype(zc)::value;
      if (xpby) {
        allow_smem(n16::k_spmv16<T, 1, T, ZT>, sm);
        n16::k_spmv16<T, 1, T, ZT><<<g, n16::Zt<ZT>::NT, sm, s>>>(D, d, z, dn, (T)beta, q, (T)L.c0, (T)L.ce,
                                                                  (T)L.cc, nullptr, part, beta_dev);
      } else {
        allow_smem(n16::k_spmv16<T, 0, T, ZT>, sm);
        n16::k_spmv16<T, 0, T, ZT><<<g, n16::Zt<ZT>::NT, sm, s>>>(D, d, nullptr, nullptr, (T)0, q, (T)L.c0,
                                                                  (T)L.ce, (T)L.cc, nullptr, part, nullptr);
      }
    };
    constexpr bool kTunable = std::is_same<T, float>::value;
    tuned_launch(s, kTuneSpmv, D, (uint64_t)g.x * g.y, kTunable, [&](int zt) {
      if constexpr (kTunable) {
        if (zt == 2) return go(std::integral_constant<int, 2>());
        if (zt == 8) return go(std::integral_constant<int, 8>());
      }
      go(std::integral_constant<int, 4>());
    });
  } else {
    if (clouds != 1 || beta_dev) throw Error(PR_ERR_INTERNAL, "packed SpMV needs depth >= 4");
    const unsigned nb = 1u << (3 * (D - 3));
    const size_t sm = sizeof(T) * (10 * 10 * 10 + 512);
    if (xpby) k_spmv<T, 8, true><<<nb, Geo<8>::THREADS, sm, s>>>(D, z, d, dn, (T)beta, q, k, part);
    else k_spmv<T, 8, false><<<nb, Geo<8>::THREADS, sm, s>>>(D, z, d, dn, (T)beta, q, k, part);
  }
  PR_CHECK_LAUNCH();
}

template <typename E>
void mg_resid_update(cudaStream_t s, const LevelCoef& L, const double* x, const E* e, double scale, double* xn,
                     const double* b, double* r, uint32_t clouds, const double* scale_dev) {
  const uint32_t D = L.depth;
  if (D < 4 || L.has_faces) throw Error(PR_ERR_INTERNAL, "mg_resid_update needs the finest level, depth >= 4");
  const size_t sm = n16::smem_bytes<double>();
  allow_smem(n16::k_spmv16<double, 2, E, 4>, sm);
  n16::k_spmv16<double, 2, E, 4><<<dim3(1u << (3 * (D - 4)), clouds), n16::Zt<4>::NT, sm, s>>>(
      D, x, e, xn, scale, r, L.c0, L.ce, L.cc, b, nullptr, scale_dev);
  PR_CHECK_LAUNCH();
}
template void mg_resid_update<float>(cudaStream_t, const LevelCoef&, const double*, const float*, double, double*,
                                     const double*, double*, uint32_t, const double*);
template void mg_resid_update<double>(cudaStream_t, const LevelCoef&, const double*, const double*, double, double*,
                                      const double*, double*, uint32_t, const double*);

uint32_t mg_blocks(uint32_t D) { return tile_for(D) == 16 ? (1u << (3 * (D - 4))) : (1u << (3 * (D - 3))); }

void sum_parts(cudaStream_t s, const double* part, int np, double scale2, const double* part2, int np2, double* out,
               uint32_t clouds) {
  k_sum_parts<<<clouds, 1024, 0, s>>>(part, np, scale2, part2, np2, out);
  PR_CHECK_LAUNCH();
}

// ------------------------------------------------------------------ kernel micro-benchmark
namespace {
template <typename T>
__global__ void k_fill(T* __restrict__ x, uint64_t n, uint32_t seed) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t h = (uint32_t)i * 2654435761u ^ seed;
    h ^= h >> 15;
    h *= 2246822519u;
    h ^= h >> 13;
    x[i] = (T)((double)(h & 0xffffff) / 16777216.0 - 0.5);
  }
}

template <typename T>
double bench_one(pr_context* c, int kid, uint32_t D, int reps, double* bytes) {
  cudaStream_t s = c->stream;
  const uint64_t n = 1ull << (3 * D), nc = n / 8;
  const std::string tn = std::is_same<T, double>::value ? "f64" : "f32";
  T* x = c->buf<T>("kb_x_" + tn, n);
  T* y = c->buf<T>("kb_y_" + tn, n);
  T* f = c->buf<T>("kb_f_" + tn, n);
  T* w = c->buf<T>("kb_w_" + tn, n);
  T* ec = c->buf<T>("kb_c_" + tn, nc);
  T* face = c->buf<T>("kb_face_" + tn, std::max<size_t>(mg_face_entries(D), 1));
  T* r2 = c->buf<T>("kb_r_" + tn, n);
  double* part = c->buf<double>("kb_part", std::max<uint32_t>(mg_blocks(D), kDotBlocks));
  const unsigned g = 148 * 16;
  k_fill<T><<<g, 256, 0, s>>>(x, n, 1u);
  k_fill<T><<<g, 256, 0, s>>>(f, n, 2u);
  k_fill<T><<<g, 256, 0, s>>>(w, n, 3u);
  k_fill<T><<<g, 256, 0, s>>>(ec, nc, 4u);
  k_fill<T><<<g, 256, 0, s>>>(r2, n, 5u);
  PR_CHECK_LAUNCH();
  // the finest level (no low-face rows: the variants that dominate a solve) and, for ids 7-8,
  // a coarse level (low-face table rows)
  const LevelCoef Lf = level_coef(D, D, 0.0), Lc = level_coef(D + 1, D, 0.0);
  std::vector<T> tab(216);
  for (int m = 0; m < 8; ++m)
    for (int o = 0; o < 27; ++o) tab[27 * m + o] = (T)Lc.table[m][o];
  T* table = c->buf<T>("kb_tab_" + tn, 216);
  PR_CUDA(cudaMemcpyAsync(table, tab.data(), 216 * sizeof(T), cudaMemcpyHostToDevice, s));
  const double es = sizeof(T);
  auto run = [&]() {
    switch (kid) {
      case 0: mg_spmv<T>(s, Lf, table, nullptr, x, nullptr, 0.0, false, y, part); break;
      case 1: mg_spmv<T>(s, Lf, table, f, x, w, 0.5, true, y, part); break;
      case 2: mg_smooth<T>(s, Lf, table, nullptr, y, f, nullptr, 1, true, nullptr); break;
      case 3: mg_smooth<T>(s, Lf, table, x, y, f, nullptr, 0, true, nullptr); break;
      case 4: mg_smooth<T>(s, Lf, table, x, y, f, ec, 2, false, part); break;
      case 5: mg_resid_restrict<T>(s, Lf, table, x, f, ec, face); break;
      case 7: mg_smooth<T>(s, Lc, table, x, y, f, ec, 2, false, part); break;
      case 8: mg_resid_restrict<T>(s, Lc, table, x, f, ec, face); break;
      case 9: {  // CG update fused with the first pre-smoothing sweep: x += a d, r -= a q, y = S(r)
        CgFuse<T> cg;
        cg.x = w;
        cg.d = x;
        cg.q = f;
        cg.r = r2;
        cg.alpha = (T)1e-3;  // small: the reps leave r and the update bounded
        mg_cg_update_presmooth<T>(s, Lf, table, cg, y, part);
        break;
      }
      case 6: stencil_apply<T>(s, D, x, nullptr, y, cast_coef<T>(stencil_coef(D, 0.0)), 0); break;
      default: throw Error(PR_ERR_INVALID_ARGUMENT, "unknown kernel id");
    }
  };
  const double nb = (double)n * es;
  const double algo[] = {2 * nb, 4 * nb, 2 * nb, 3 * nb, 3 * nb + nb / 8, 2 * nb + nb / 8, 2 * nb,
                         3 * nb + nb / 8, 2 * nb + nb / 8, 7 * nb};
  if (kid < 0 || kid > 9) throw Error(PR_ERR_INVALID_ARGUMENT, "unknown kernel id");
  *bytes = algo[kid];
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
  return (double)ms / reps;
}
}  // namespace

std::string autotune_log() {
  TuneTable& tt = tune_table();
  std::lock_guard<std::mutex> g(tt.mu);
  return tt.log;
}

double kernel_bench(pr_context* c, int kid, uint32_t D, int precision, int reps, double* bytes) {
  if (D < 4 || D > kMaxDepth) throw Error(PR_ERR_INVALID_ARGUMENT, "kernel bench depth must be in [4, 10]");
  if (kid >= 20) return deg2_kernel_bench(c, kid - 20, D, precision, reps, bytes);
  if (reps < 1) reps = 1;
  return precision == PR_PRECISION_FP64 ? bench_one<double>(c, kid, D, reps, bytes)
                                        : bench_one<float>(c, kid, D, reps, bytes);
}

#define PR_INST(T)                                                                                                 \
  template void mg_smooth<T>(cudaStream_t, const LevelCoef&, const T*, const T*, T*, const T*, const T*, int, bool, \
                             double*, uint32_t);                                                                  \
  template void mg_resid_restrict<T>(cudaStream_t, const LevelCoef&, const T*, const T*, const T*, T*, T*,        \
                                     uint32_t);                                                                   \
  template void mg_cg_update_presmooth<T>(cudaStream_t, const LevelCoef&, const T*, const CgFuse<T>&, T*, double*, \
                                          uint32_t);                                                              \
  template void mg_spmv<T>(cudaStream_t, const LevelCoef&, const T*, const T*, const T*, T*, double, bool, T*,    \
                           double*, uint32_t, const double*);
PR_INST(float)
PR_INST(double)
#undef PR_INST

}  // namespace pr

// Adaptive (narrow-band) reconstruction: depth up to 12 without a dense fine grid.  An
// extension: the crate refines every leaf to max_depth and ignores the points
// (src/fem_tree.rs:83-93), so its grid is the dense res^3 one (src/fem_tree.rs:96-126), which at
// depth 12 would hold 6.9e10 nodes.  Here the fine level exists only where the points are.
//
//   1. coarse level: the dense degree-2 reconstruction system at depth Dc (the solver of
//      pr_deg2.cu), solved to the requested residual; x_c its coefficients;
//   2. bricks: the fine grid (depth D) is cut into bricks of 8^3 nodes; a brick is active when
//      it holds a node of some point's 27 basis functions (every point's support lies in active
//      bricks), or every brick with PR_BAND_FULL.  B = the nodes of active bricks (the band),
//      H = every other node;
//   3. the fine function is u = sum_{i in B} f_i phi_i + sum_{j in H} g_j phi_j, where g = P^L x_c
//      (L = D - Dc levels of the B2 subdivision, the exact depth-D coefficients of the coarse
//      function): f solves the depth-D system of the dense degree-2 reconstruction restricted to
//      B with g fixed on H,
//            A_BB f = b_B - A_BH g_H,
//      A and b being exactly the dense system's (stiffness, screening of every point, splat of the
//      normals, right-hand side); with every brick active this IS the dense system.  Written as
//      f = g_B + e: A_BB e = r0 = b_B - (A g)_B;
//   4. A_BB e = r0 by Jacobi-preconditioned CG: FP32 inner solves with FP64 residual refinement,
//      or FP64 throughout (the same precision modes as the dense solve);
//   5. iso = mean over the points of the fine function; marching cubes over the cells of the
//      active bricks (corner values from f on B and g on H), vertices deduplicated by grid-edge key.
//
// Layout: band vectors are brick-major, 512 nodes per brick in natural order (x fastest); bricks
// are sorted by their Morton code, so a brick's neighbours are mostly near it in memory.  The
// operator pass gives each CTA one brick: its 12^3 tile (brick and 2-node halo, gathered from the
// 27 neighbouring bricks, zero on H) goes to shared memory and the separable stencil
// h (S M M + M S M + M M S) runs as z, y and x passes there.  The screening term reuses the
// dense path's (node, point) pair lists, keyed by band index.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <cmath>
#include <string>
#include <vector>

#include "pr_internal.cuh"
#include "pr_ops.cuh"

#define PR_MC_TABLE_QUAL static __constant__
#include "mc_tri_table.inc"

namespace pr {

namespace {

constexpr int kThreads = 256;
constexpr uint32_t kSent = 0xffffffffu;  // no brick / no node
constexpr int kBN = 512;                 // nodes per brick
constexpr int kOT = 12;                  // operator tile edge: brick + 2-node halo
constexpr int kOT3 = kOT * kOT * kOT;
constexpr int kMT = 10;                  // marching-cubes node tile edge: brick + 1 node each side
constexpr int kMaxW = 64;                // taps of the composite prolongation (L <= 4: 46)

inline unsigned grid_for(uint64_t n, uint64_t cap = 1u << 22) {
  uint64_t g = (n + kThreads - 1) / kThreads;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (unsigned)g;
}
inline unsigned brick_grid(uint64_t nb) { return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(nb, 148 * 64)); }

// 1-D integrals of N2 N2, N2' N2', N2' N2 (offsets -2..2), the operator's scale and shift
template <typename T>
struct BandCoef {
  T m[5], s[5];
  T H, wg;
};
// g_f = sum_I w[f - 2^L I - kmin] x_c[I] per axis
struct Prolong {
  double w[kMaxW];
  int kmin, kmax, L, resc;
};

// degree-2 basis of one axis at unit coordinate u (the dense setup's expressions, so that the
// basis values of a point are the same bits in both paths)
__device__ __forceinline__ void axis2b(double u, double h, int64_t& c, double* b) {
  const double s = xdiv(u, h);
  c = sat_i64(floor(s));
  const double t = xsub(s, (double)c);
  const double omt = xsub(1.0, t);
  b[0] = xmul(xmul(0.5, omt), omt);
  b[1] = xmul(0.5, xadd(xadd(xmul(xmul(-2.0, t), t), xmul(2.0, t)), 1.0));
  b[2] = xmul(xmul(0.5, t), t);
}

__device__ __forceinline__ int floor_div(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

// The coarse function's depth-D coefficients on a TT^3 tile of fine nodes starting at (ox, oy, oz)
// (zero outside the grid), by the whole CTA: the coarse coefficients that reach the tile (at most
// 9 per axis), then the separable sums over x, y and z, every one in increasing coarse index, so
// a node gets the same bits in any tile.  scratch: 729 + 81 TT + 9 TT^2 doubles.
__host__ __device__ constexpr int kProlongScratch(int tt) { return 729 + 81 * tt + 9 * tt * tt; }
template <int TT>
__device__ void prolong_tile(const double* __restrict__ xc, const Prolong& W, int res, int ox, int oy, int oz,
                             double* scratch, double* out) {
  const int step = 1 << W.L;
  const int o[3] = {ox, oy, oz};
  int lo[3], cnt[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    lo[a] = max(0, -floor_div(W.kmax - o[a], step));  // ceil((o - kmax) / step)
    const int hi = min(W.resc - 1, floor_div(o[a] + TT - 1 - W.kmin, step));
    cnt[a] = max(0, hi - lo[a] + 1);
  }
  double* c = scratch;        // [cz][cy][cx]
  double* ax = c + 729;       // [cz][cy][TT]
  double* ay = ax + 81 * TT;  // [cz][TT][TT]
  const int t = threadIdx.x, nt = blockDim.x;
  for (int i = t; i < cnt[0] * cnt[1] * cnt[2]; i += nt) {
    const int ix = i % cnt[0], iy = (i / cnt[0]) % cnt[1], iz = i / (cnt[0] * cnt[1]);
    c[i] = xc[(int64_t)(lo[0] + ix) + (int64_t)W.resc * ((lo[1] + iy) + (int64_t)W.resc * (lo[2] + iz))];
  }
  __syncthreads();
  for (int i = t; i < cnt[2] * cnt[1] * TT; i += nt) {
    const int tx = i % TT, r = i / TT;  // r = iz cnt1 + iy
    const int f = ox + tx;
    double v = 0.0;
    if (f >= 0 && f < res)
      for (int ix = 0; ix < cnt[0]; ++ix) {
        const int k = f - step * (lo[0] + ix) - W.kmin;
        if (k >= 0 && k <= W.kmax - W.kmin) v += W.w[k] * c[r * cnt[0] + ix];
      }
    ax[i] = v;
  }
  __syncthreads();
  for (int i = t; i < cnt[2] * TT * TT; i += nt) {
    const int tx = i % TT, ty = (i / TT) % TT, iz = i / (TT * TT);
    const int f = oy + ty;
    double v = 0.0;
    if (f >= 0 && f < res)
      for (int iy = 0; iy < cnt[1]; ++iy) {
        const int k = f - step * (lo[1] + iy) - W.kmin;
        if (k >= 0 && k <= W.kmax - W.kmin) v += W.w[k] * ax[(iz * cnt[1] + iy) * TT + tx];
      }
    ay[i] = v;
  }
  __syncthreads();
  for (int i = t; i < TT * TT * TT; i += nt) {
    const int yx = i % (TT * TT), tz = i / (TT * TT);
    const int f = oz + tz;
    double v = 0.0;
    if (f >= 0 && f < res)
      for (int iz = 0; iz < cnt[2]; ++iz) {
        const int k = f - step * (lo[2] + iz) - W.kmin;
        if (k >= 0 && k <= W.kmax - W.kmin) v += W.w[k] * ay[iz * TT * TT + yx];
      }
    out[i] = v;
  }
  __syncthreads();
}

// ------------------------------------------------------------------ bricks
// the bricks holding nodes c-1 .. c+1 of each point (up to 2 per axis), Morton-coded; duplicates
// and points outside the grid give kSent
__global__ void k_ab_brick_keys(const double* __restrict__ upos, uint64_t P, uint32_t D, uint32_t* __restrict__ keys) {
  const int64_t res = 1ll << D;
  const double h = 1.0 / (double)res;
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < P; p += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    bool ok = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const int64_t c = sat_i64(floor(xdiv(upos[(uint64_t)a * P + p], h)));
      const int64_t a0 = c - 1 < 0 ? 0 : c - 1, a1 = c + 1 > res - 1 ? res - 1 : c + 1;
      if (a0 > a1) ok = false;
      else {
        lo[a] = (uint32_t)(a0 >> 3);
        hi[a] = (uint32_t)(a1 >> 3);
      }
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int sx = k & 1, sy = (k >> 1) & 1, sz = k >> 2;
      const bool dup = (sx && hi[0] == lo[0]) || (sy && hi[1] == lo[1]) || (sz && hi[2] == lo[2]);
      keys[8 * p + k] = (!ok || dup) ? kSent : morton3(sx ? hi[0] : lo[0], sy ? hi[1] : lo[1], sz ? hi[2] : lo[2]);
    }
  }
}

__global__ void k_ab_iota(uint32_t* __restrict__ v, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    v[i] = (uint32_t)i;
}

__global__ void k_ab_brick_map(const uint32_t* __restrict__ bkey, uint64_t NB, uint32_t* __restrict__ bmap) {
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < NB; s += (uint64_t)gridDim.x * blockDim.x)
    bmap[bkey[s]] = (uint32_t)s;
}

// 27 neighbour slots per brick, k = 9 (dz + 1) + 3 (dy + 1) + (dx + 1)
__global__ void k_ab_neighbours(const uint32_t* __restrict__ bkey, uint64_t NB, uint32_t nbr_res,
                                const uint32_t* __restrict__ bmap, uint32_t* __restrict__ nbr) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < 27 * NB; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t s = i / 27;
    const int k = (int)(i - 27 * s);
    uint32_t bx, by, bz;
    unmorton3(bkey[s], bx, by, bz);
    const int x = (int)bx + k % 3 - 1, y = (int)by + (k / 3) % 3 - 1, z = (int)bz + k / 9 - 1;
    const bool in = x >= 0 && y >= 0 && z >= 0 && x < (int)nbr_res && y < (int)nbr_res && z < (int)nbr_res;
    nbr[i] = in ? bmap[morton3((uint32_t)x, (uint32_t)y, (uint32_t)z)] : kSent;
  }
}

// (band node, 27 p + k) pairs of the points' basis functions, with the basis values (the dense
// degree-2 setup's pairs with the band index in place of the natural one)
__global__ void k_ab_pair_keys(const double* __restrict__ upos, uint64_t P, uint32_t D, const uint32_t* __restrict__ bmap,
                               uint32_t* __restrict__ keys, uint32_t* __restrict__ vals, double* __restrict__ phi64,
                               float* __restrict__ phi32, unsigned long long* __restrict__ nin) {
  const int64_t res = 1ll << D;
  const double h = 1.0 / (double)res;
  unsigned long long cnt = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < 27 * P; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t p = i / 27;
    const int k = (int)(i - 27 * p), dx = k % 3, dy = (k / 3) % 3, dz = k / 9;
    int64_t c[3];
    double b[3][3];
    axis2b(upos[p], h, c[0], b[0]);
    axis2b(upos[P + p], h, c[1], b[1]);
    axis2b(upos[2 * P + p], h, c[2], b[2]);
    const int64_t x = c[0] + dx - 1, y = c[1] + dy - 1, z = c[2] + dz - 1;
    bool ok = x >= 0 && y >= 0 && z >= 0 && x < res && y < res && z < res;
    uint32_t key = kSent;
    if (ok) {
      const uint32_t slot = bmap[morton3((uint32_t)(x >> 3), (uint32_t)(y >> 3), (uint32_t)(z >> 3))];
      ok = slot != kSent;
      if (ok) key = slot * (uint32_t)kBN + (uint32_t)(((z & 7) << 6) | ((y & 7) << 3) | (x & 7));
    }
    keys[i] = key;
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

// per touched node (points in input order): nf = -(sum phi n) / (sum phi), sum phi, sum phi^2
__global__ void k_ab_splat(const uint32_t* __restrict__ run_off, uint64_t T, const uint32_t* __restrict__ sval,
                           const double* __restrict__ phi, const double* __restrict__ unrm, uint64_t P,
                           double* __restrict__ nfc, double* __restrict__ sphi, double* __restrict__ sphi2) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < T; t += (uint64_t)gridDim.x * blockDim.x) {
    double fx = 0.0, fy = 0.0, fz = 0.0, sw = 0.0, s2 = 0.0;
    for (uint32_t e = run_off[t]; e < run_off[t + 1]; ++e) {
      const uint32_t pk = sval[e];
      const uint32_t p = pk / 27;
      const double wgt = phi[pk];
      fx = xadd(fx, xmul(unrm[p], wgt));
      fy = xadd(fy, xmul(unrm[P + p], wgt));
      fz = xadd(fz, xmul(unrm[2 * P + p], wgt));
      sw = xadd(sw, wgt);
      s2 += wgt * wgt;
    }
    if (sw > 0.0) {
      fx = xdiv(-fx, sw);
      fy = xdiv(-fy, sw);
      fz = xdiv(-fz, sw);
    }
    nfc[3 * t] = fx;
    nfc[3 * t + 1] = fy;
    nfc[3 * t + 2] = fz;
    sphi[t] = sw;
    sphi2[t] = s2;
  }
}

// brun[s] = first run of brick s (runs sorted by band key, key / 512 = brick)
__global__ void k_ab_brick_runs(const uint32_t* __restrict__ run_key, uint64_t T, uint64_t NB,
                                uint32_t* __restrict__ brun) {
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s <= NB; s += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t target = s * kBN;
    uint64_t a = 0, b = T;
    while (a < b) {
      const uint64_t m = (a + b) >> 1;
      if ((uint64_t)run_key[m] < target) a = m + 1;
      else b = m;
    }
    brun[s] = (uint32_t)a;
  }
}

// ------------------------------------------------------------------ right-hand side
// b = h^2 sum_a (G_a M M) nf_a + (wh3 / 2) sum_p phi: per brick, the normal field of the brick
// and its 2-node halo into a shared tile (zero where no point splatted), then z, y and x passes
__global__ void __launch_bounds__(kThreads) k_ab_rhs(const uint32_t* __restrict__ nbr, const uint32_t* __restrict__ run_key,
                                                     const uint32_t* __restrict__ brun, const double* __restrict__ nfc,
                                                     const double* __restrict__ sphi, double wt, BandCoef<double> K,
                                                     double g0, double g1, double g3, double g4, double h2, uint64_t NB,
                                                     double* __restrict__ b) {
  extern __shared__ double sm[];
  double* nf = sm;                  // [3][12][12][12]
  double* tz = nf + 3 * kOT3;       // [8][12][12]
  double* ty = tz + 8 * kOT * kOT;  // [8][8][12]
  double* ob = ty + 8 * 8 * kOT;    // [512]
  __shared__ uint32_t nb[27];
  const int t = threadIdx.x;
  const double gg[5] = {g0, g1, 0.0, g3, g4};
  for (uint64_t slot = blockIdx.x; slot < NB; slot += gridDim.x) {
    if (t < 27) nb[t] = nbr[27 * slot + t];
    for (int i = t; i < 3 * kOT3; i += kThreads) nf[i] = 0.0;
    __syncthreads();
    for (int k = 0; k < 27; ++k) {
      const uint32_t s2 = nb[k];
      if (s2 == kSent) continue;
      const int ox = k % 3 - 1, oy = (k / 3) % 3 - 1, oz = k / 9 - 1;
      for (uint32_t r = brun[s2] + t; r < brun[s2 + 1]; r += kThreads) {
        const uint32_t local = run_key[r] - s2 * (uint32_t)kBN;
        const int tx = (int)(local & 7) + 8 * ox + 2, ty_ = (int)((local >> 3) & 7) + 8 * oy + 2,
                  tz_ = (int)(local >> 6) + 8 * oz + 2;
        if (tx < 0 || ty_ < 0 || tz_ < 0 || tx >= kOT || ty_ >= kOT || tz_ >= kOT) continue;
        const int o = (tz_ * kOT + ty_) * kOT + tx;
        nf[o] = nfc[3 * (uint64_t)r];
        nf[kOT3 + o] = nfc[3 * (uint64_t)r + 1];
        nf[2 * kOT3 + o] = nfc[3 * (uint64_t)r + 2];
      }
    }
    __syncthreads();
    double acc[2] = {0.0, 0.0};
    for (int a = 0; a < 3; ++a) {
      const double* fz = a == 2 ? gg : K.m;
      const double* fy = a == 1 ? gg : K.m;
      const double* fx = a == 0 ? gg : K.m;
      const double* src = nf + a * kOT3;
      for (int i = t; i < 8 * kOT * kOT; i += kThreads) {
        const int z = i / (kOT * kOT), yx = i % (kOT * kOT);
        double v = 0.0;
#pragma unroll
        for (int c = 0; c < 5; ++c) v += fz[c] * src[(z + c) * kOT * kOT + yx];
        tz[i] = v;
      }
      __syncthreads();
      for (int i = t; i < 8 * 8 * kOT; i += kThreads) {
        const int z = i / (8 * kOT), y = (i / kOT) % 8, x = i % kOT;
        double v = 0.0;
#pragma unroll
        for (int c = 0; c < 5; ++c) v += fy[c] * tz[(z * kOT + y + c) * kOT + x];
        ty[i] = v;
      }
      __syncthreads();
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int o = t + j * kThreads, z = o >> 6, y = (o >> 3) & 7, x = o & 7;
        double v = 0.0;
#pragma unroll
        for (int c = 0; c < 5; ++c) v += fx[c] * ty[(z * 8 + y) * kOT + x + c];
        acc[j] += v;
      }
      __syncthreads();
    }
    ob[t] = h2 * acc[0];
    ob[t + kThreads] = h2 * acc[1];
    __syncthreads();
    for (uint32_t r = brun[slot] + t; r < brun[slot + 1]; r += kThreads)
      ob[run_key[r] - (uint32_t)slot * kBN] += wt * sphi[r];
    __syncthreads();
    b[slot * kBN + t] = ob[t];
    b[slot * kBN + t + kThreads] = ob[t + kThreads];
    __syncthreads();
  }
}

// ------------------------------------------------------------------ the band operator
// One brick per CTA iteration, kOpThreads threads.  The brick and its 2-node halo (a 12^3 tile,
// gathered from the 27 neighbouring bricks, zero outside the band) go to shared memory; the
// stencil h (S M M + M S M + M M S) + wg then runs as three register passes: a thread per (x, y)
// column filters z (M and S), a thread per (x, z) column filters y, a thread per (y, z) row filters
// x and writes its 8 outputs as two 16-byte stores.
//   kBandApply: y = A x          kBandResid: y = f - A x
//   kBandDir:   the CG direction step: d = z + beta dold (dold = x, z = f; x unread when beta = 0)
//               formed while gathering, written to dout (a buffer other than x: neighbouring CTAs
//               still gather dold) for the brick, and y = A d with per-CTA partials of d . y
// GSRC (kBandResid, FP64): the tile is the prolonged coarse function on every node (x unused):
// y = f - (K + wg I) g on the band.
constexpr int kOpThreads = 160;
constexpr int kWS = 13;  // row stride of the y-filtered planes (conflict-free x pass)
enum { kBandApply = 0, kBandResid = 1, kBandDir = 2 };

template <typename T>
constexpr size_t band_op_smem(bool gsrc) {
  return (size_t)(kOT3 + 2 * 8 * kOT * kOT + 2 * 8 * 8 * kWS) * sizeof(T) +
         (gsrc ? (size_t)(kProlongScratch(kOT) + kOT3) * sizeof(double) : 0);
}

// 12 values of a tile row from the band vector v: brick sl[0] at x = 6, 7, sl[1] at x = 0..7,
// sl[2] at x = 0, 1 of the row at offset rowoff; zero for kSent
template <typename T>
__device__ __forceinline__ void ab_load_row(const T* __restrict__ v, const uint32_t* sl, int rowoff, T* out) {
#pragma unroll
  for (int k = 0; k < kOT; ++k) out[k] = T(0);
  if (sl[0] != kSent) {
    const T* p = v + (uint64_t)sl[0] * kBN + rowoff + 6;
    out[0] = p[0];
    out[1] = p[1];
  }
  if (sl[1] != kSent) {
    const T* p = v + (uint64_t)sl[1] * kBN + rowoff;
    if (sizeof(T) == 4) {
      const float4 a = *reinterpret_cast<const float4*>(p), b = *reinterpret_cast<const float4*>(p + 4);
      out[2] = (T)a.x; out[3] = (T)a.y; out[4] = (T)a.z; out[5] = (T)a.w;
      out[6] = (T)b.x; out[7] = (T)b.y; out[8] = (T)b.z; out[9] = (T)b.w;
    } else {
#pragma unroll
      for (int k = 0; k < 8; k += 2) {
        const double2 a = *reinterpret_cast<const double2*>(p + k);
        out[2 + k] = (T)a.x;
        out[3 + k] = (T)a.y;
      }
    }
  }
  if (sl[2] != kSent) {
    const T* p = v + (uint64_t)sl[2] * kBN + rowoff;
    out[10] = p[0];
    out[11] = p[1];
  }
}
template <typename T>
__device__ __forceinline__ void ab_store8(T* __restrict__ p, const T* v) {
  if (sizeof(T) == 4) {
    *reinterpret_cast<float4*>(p) = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
    *reinterpret_cast<float4*>(p + 4) = make_float4((float)v[4], (float)v[5], (float)v[6], (float)v[7]);
  } else {
#pragma unroll
    for (int k = 0; k < 8; k += 2) *reinterpret_cast<double2*>(p + k) = make_double2((double)v[k], (double)v[k + 1]);
  }
}
template <typename T>
__device__ __forceinline__ void ab_store_tile_row(T* p, const T* v) {
  if (sizeof(T) == 4) {
#pragma unroll
    for (int k = 0; k < kOT; k += 4)
      *reinterpret_cast<float4*>(p + k) = make_float4((float)v[k], (float)v[k + 1], (float)v[k + 2], (float)v[k + 3]);
  } else {
#pragma unroll
    for (int k = 0; k < kOT; k += 2) *reinterpret_cast<double2*>(p + k) = make_double2((double)v[k], (double)v[k + 1]);
  }
}

template <typename T, int MODE, bool GSRC>
__global__ void __launch_bounds__(kOpThreads) k_ab_op(const T* __restrict__ x, const T* __restrict__ f,
                                                      T* __restrict__ y, T* __restrict__ dout, double beta,
                                                      const uint32_t* __restrict__ nbr,
                                                      const uint32_t* __restrict__ bkey, uint64_t NB, BandCoef<T> K,
                                                      const double* __restrict__ xc, Prolong W, int res,
                                                      double* __restrict__ part) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* tile = reinterpret_cast<T*>(smem_raw);   // [z][y][x], 12^3
  T* um = tile + kOT3;                         // [z 8][y 12][x 12]
  T* us = um + 8 * kOT * kOT;
  T* w1 = us + 8 * kOT * kOT;                  // [z 8][y 8][x kWS]
  T* w23 = w1 + 8 * 8 * kWS;
  double* gs = reinterpret_cast<double*>(w23 + 8 * 8 * kWS);  // GSRC: prolongation scratch, then the tile
  __shared__ uint32_t nb[27];
  __shared__ double red[kOpThreads / 32 + 1];
  const int t = threadIdx.x;
  const T tb = (T)beta;
  double dacc = 0.0;
  for (uint64_t slot = blockIdx.x; slot < NB; slot += gridDim.x) {
    if (t < 27) nb[t] = nbr[27 * slot + t];
    __syncthreads();
    if (GSRC) {
      uint32_t bx, by, bz;
      unmorton3(bkey[slot], bx, by, bz);
      double* gt = gs + kProlongScratch(kOT);
      prolong_tile<kOT>(xc, W, res, 8 * (int)bx - 2, 8 * (int)by - 2, 8 * (int)bz - 2, gs, gt);
      for (int i = t; i < kOT3; i += kOpThreads) tile[i] = (T)gt[i];
    } else if (t < kOT * kOT) {
      // a thread per tile row (y, z): 2 values of the left neighbour brick (its x = 6, 7), 8 of the
      // centre one, 2 of the right one (x = 0, 1), as vector loads
      const int ly = t % kOT - 2, lz = t / kOT - 2;
      const int oy = ly < 0 ? -1 : (ly >= 8 ? 1 : 0), oz = lz < 0 ? -1 : (lz >= 8 ? 1 : 0);
      const int rowoff = ((lz - 8 * oz) << 6) | ((ly - 8 * oy) << 3);
      const int kb = (oz + 1) * 9 + (oy + 1) * 3;
      const uint32_t sl[3] = {nb[kb], nb[kb + 1], nb[kb + 2]};
      T v[kOT];
      ab_load_row<T>(MODE == kBandDir ? f : x, sl, rowoff, v);
      if (MODE == kBandDir) {
        if (beta != 0.0) {
          T w[kOT];
          ab_load_row<T>(x, sl, rowoff, w);
#pragma unroll
          for (int k = 0; k < kOT; ++k) v[k] += tb * w[k];
        }
        if (oy == 0 && oz == 0) ab_store8<T>(dout + slot * kBN + rowoff, v + 2);
      }
      ab_store_tile_row<T>(tile + t * kOT, v);
    }    __syncthreads();
    if (t < kOT * kOT) {  // z filter of column (x, y)
      T v[kOT];
#pragma unroll
      for (int z = 0; z < kOT; ++z) v[z] = tile[z * kOT * kOT + t];
#pragma unroll
      for (int z = 0; z < 8; ++z) {
        T am = T(0), as = T(0);
#pragma unroll
        for (int c = 0; c < 5; ++c) {
          am += K.m[c] * v[z + c];
          as += K.s[c] * v[z + c];
        }
        um[z * kOT * kOT + t] = am;
        us[z * kOT * kOT + t] = as;
      }
    }
    __syncthreads();
    if (t < 8 * kOT) {  // y filter of column (x, z)
      const int xx = t % kOT, z = t / kOT;
      T a[kOT], b[kOT];
#pragma unroll
      for (int yy = 0; yy < kOT; ++yy) {
        a[yy] = um[(z * kOT + yy) * kOT + xx];
        b[yy] = us[(z * kOT + yy) * kOT + xx];
      }
#pragma unroll
      for (int yy = 0; yy < 8; ++yy) {
        T a1 = T(0), a2 = T(0), a3 = T(0);
#pragma unroll
        for (int c = 0; c < 5; ++c) {
          a1 += K.m[c] * a[yy + c];
          a2 += K.s[c] * a[yy + c];
          a3 += K.m[c] * b[yy + c];
        }
        w1[(z * 8 + yy) * kWS + xx] = a1;
        w23[(z * 8 + yy) * kWS + xx] = a2 + a3;
      }
    }
    __syncthreads();
    if (t < 64) {  // x filter of row (y, z), 8 outputs
      const int yy = t % 8, z = t / 8;
      T p[kOT], q[kOT], o[8];
#pragma unroll
      for (int xx = 0; xx < kOT; ++xx) {
        p[xx] = w1[(z * 8 + yy) * kWS + xx];
        q[xx] = w23[(z * 8 + yy) * kWS + xx];
      }
      const uint64_t g0 = slot * kBN + (uint64_t)(z * 64 + yy * 8);
      T dpart = T(0);  // this row's share of d . q (at most 8 terms, then accumulated in FP64)
#pragma unroll
      for (int xx = 0; xx < 8; ++xx) {
        T acc = T(0);
#pragma unroll
        for (int c = 0; c < 5; ++c) acc += K.s[c] * p[xx + c] + K.m[c] * q[xx + c];
        const T ctr = tile[((z + 2) * kOT + yy + 2) * kOT + xx + 2];
        o[xx] = K.H * acc + K.wg * ctr;
        if (MODE == kBandResid) o[xx] = f[g0 + xx] - o[xx];
        if (MODE == kBandDir) dpart += ctr * o[xx];
      }
      if (MODE == kBandDir) dacc += (double)dpart;
      ab_store8<T>(y + g0, o);
    }
    __syncthreads();
  }
  if (MODE == kBandDir && part) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) dacc += __shfl_down_sync(0xffffffffu, dacc, off);
    if ((t & 31) == 0) red[t >> 5] = dacc;
    __syncthreads();
    if (t == 0) {
      double sum = 0.0;
      for (int w = 0; w < kOpThreads / 32; ++w) sum += red[w];
      part[blockIdx.x] = sum;
    }
  }
}

// screening: proj_p = sum_k phi x[key]; y[node] += sgn wh3 sum phi proj over the node's pairs;
// sq (optional): per-block sums of proj^2 (x . wh3 Phi Phi^T x = wh3 sum_p proj_p^2)
template <typename T>
__global__ void k_ab_screen_proj(const uint32_t* __restrict__ key, const T* __restrict__ phi, uint64_t P,
                                 const T* __restrict__ x, T* __restrict__ proj, double* __restrict__ sq) {
  double acc = 0.0;
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < P; p += (uint64_t)gridDim.x * blockDim.x) {
    T s = T(0);
    for (int k = 0; k < 27; ++k) {
      const uint32_t kk = key[27 * p + k];
      if (kk != kSent) s += phi[27 * p + k] * x[kk];
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
__global__ void k_ab_screen_gather(const uint32_t* __restrict__ snode, const uint32_t* __restrict__ soff, uint64_t S,
                                   const uint32_t* __restrict__ sval, const T* __restrict__ phi,
                                   const T* __restrict__ proj, T wh3s, T* __restrict__ y) {
  for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < S; u += (uint64_t)gridDim.x * blockDim.x) {
    T acc = T(0);
    for (uint32_t e = soff[u]; e < soff[u + 1]; ++e) {
      const uint32_t pk = sval[e];
      acc += phi[pk] * proj[pk / 27];
    }
    y[snode[u]] += wh3s * acc;
  }
}

// Jacobi: 1 / (interior diagonal + wh3 sum phi^2)
template <typename T>
__global__ void k_ab_dinv(double diag, uint64_t n, T* __restrict__ dinv) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    dinv[i] = (T)(1.0 / diag);
}
template <typename T>
__global__ void k_ab_dinv_screen(const uint32_t* __restrict__ run_key, const double* __restrict__ sphi2, uint64_t T_runs,
                                 double diag, double wh3, T* __restrict__ dinv) {
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < T_runs; r += (uint64_t)gridDim.x * blockDim.x)
    dinv[run_key[r]] = (T)(1.0 / (diag + wh3 * sphi2[r]));
}
// the CG update with the Jacobi step: x += alpha d, r -= alpha q, z = dinv r; per-block sums of
// r . r (part[2 b]) and r . z (part[2 b + 1]) in FP64
template <typename T>
__global__ void k_ab_update(uint64_t n, double alpha, const T* __restrict__ d, const T* __restrict__ q,
                            T* __restrict__ x, T* __restrict__ r, const T* __restrict__ dinv, T* __restrict__ z,
                            double* __restrict__ part) {
  const T a = (T)alpha;
  double rr = 0.0, rz = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    x[i] += a * d[i];
    const T ri = r[i] - a * q[i];
    r[i] = ri;
    const T zi = dinv[i] * ri;
    z[i] = zi;
    rr += (double)ri * (double)ri;
    rz += (double)ri * (double)zi;
  }
  typedef cub::BlockReduce<double, kThreads> BR;
  __shared__ typename BR::TempStorage tmp;
  const double trr = BR(tmp).Sum(rr);
  __syncthreads();
  const double trz = BR(tmp).Sum(rz);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = trr;
    part[2 * blockIdx.x + 1] = trz;
  }
}
// z = dinv r with per-block sums of r . r and r . z (the first step)
template <typename T>
__global__ void k_ab_precond(uint64_t n, const T* __restrict__ r, const T* __restrict__ dinv, T* __restrict__ z,
                             double* __restrict__ part) {
  double rr = 0.0, rz = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const T ri = r[i], zi = dinv[i] * ri;
    z[i] = zi;
    rr += (double)ri * (double)ri;
    rz += (double)ri * (double)zi;
  }
  typedef cub::BlockReduce<double, kThreads> BR;
  __shared__ typename BR::TempStorage tmp;
  const double trr = BR(tmp).Sum(rr);
  __syncthreads();
  const double trz = BR(tmp).Sum(rz);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = trr;
    part[2 * blockIdx.x + 1] = trz;
  }
}
// out[k] = sum of part[stride i + k] over i < np (k < stride), in a fixed order (one warp per k)
__global__ void k_ab_sum_parts(const double* __restrict__ part, int np, int stride, double scale, double* __restrict__ out) {
  const int k = blockIdx.x;
  double s = 0.0;
  for (int i = threadIdx.x; i < np; i += 32) s += part[(size_t)i * stride + k];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (threadIdx.x == 0) out[k] = scale * s;
}

// g on the band nodes, a brick per CTA iteration
__global__ void __launch_bounds__(kThreads) k_ab_prolong_band(const uint32_t* __restrict__ bkey, uint64_t NB,
                                                              const double* __restrict__ xc, Prolong W, int res,
                                                              double* __restrict__ g) {
  __shared__ double scratch[kProlongScratch(8)], tile[kBN];
  for (uint64_t slot = blockIdx.x; slot < NB; slot += gridDim.x) {
    uint32_t bx, by, bz;
    unmorton3(bkey[slot], bx, by, bz);
    prolong_tile<8>(xc, W, res, 8 * (int)bx, 8 * (int)by, 8 * (int)bz, scratch, tile);
    for (int i = threadIdx.x; i < kBN; i += kThreads) g[slot * kBN + i] = tile[i];
    __syncthreads();
  }
}

// ------------------------------------------------------------------ iso value
struct Neu {
  double s, c;
};
__device__ __forceinline__ Neu neu_add(Neu a, double v) {
  const double t = a.s + v;
  if (fabs(a.s) >= fabs(v)) a.c += (a.s - t) + v;
  else a.c += (v - t) + a.s;
  a.s = t;
  return a;
}
__global__ void k_ab_iso_partial(const double* __restrict__ f, const uint32_t* __restrict__ key,
                                 const double* __restrict__ phi, uint64_t P, double* __restrict__ part) {
  Neu acc{0.0, 0.0};
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < P; p += (uint64_t)gridDim.x * blockDim.x) {
    double v = 0.0;
    for (int k = 0; k < 27; ++k) {
      const uint32_t kk = key[27 * p + k];
      if (kk != kSent) v = xadd(v, xmul(f[kk], phi[27 * p + k]));
    }
    acc = neu_add(acc, v);
  }
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
__global__ void k_ab_iso_final(const double* __restrict__ part, int nb, double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  Neu t{0.0, 0.0};
  for (int i = 0; i < nb; ++i) {
    t = neu_add(t, part[2 * i]);
    t = neu_add(t, part[2 * i + 1]);
  }
  out[0] = t.s + t.c;
}

// ------------------------------------------------------------------ marching cubes
__constant__ int c_abco[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
__constant__ int c_abev[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                  {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
__device__ __forceinline__ uint32_t ab_edge_mask(uint32_t mc) {
  uint32_t m = 0;
#pragma unroll
  for (int e = 0; e < 12; ++e)
    if (((mc >> c_abev[e][0]) & 1u) != ((mc >> c_abev[e][1]) & 1u)) m |= 1u << e;
  return m;
}

// The brick's 9^3 corner values at grid positions 8b + q (q = 0..8 per axis): node tile 10^3
// (nodes 8b - 1 .. 8b + 8; f on the band, g elsewhere), each corner the in-order sum over the
// nodes p - 1, p per axis inside the grid of ((x / 2) / 2) / 2 (the dense path's grid-position
// evaluation).
__device__ void ab_corner_values(uint64_t slot, const uint32_t* nb, const double* __restrict__ f,
                                 const uint32_t* __restrict__ bkey, const double* __restrict__ xc, const Prolong& W,
                                 int res, double* node, double* cv, double* scratch) {
  const int t = threadIdx.x;
  uint32_t bx, by, bz;
  unmorton3(bkey[slot], bx, by, bz);
  const int org[3] = {8 * (int)bx, 8 * (int)by, 8 * (int)bz};
  prolong_tile<kMT>(xc, W, res, org[0] - 1, org[1] - 1, org[2] - 1, scratch, node);
  for (int i = t; i < kMT * kMT * kMT; i += kThreads) {
    const int lz = i / (kMT * kMT) - 1, ly = (i / kMT) % kMT - 1, lx = i % kMT - 1;
    const int ox = lx < 0 ? -1 : (lx >= 8 ? 1 : 0), oy = ly < 0 ? -1 : (ly >= 8 ? 1 : 0),
              oz = lz < 0 ? -1 : (lz >= 8 ? 1 : 0);
    const uint32_t s2 = nb[(oz + 1) * 9 + (oy + 1) * 3 + (ox + 1)];
    if (s2 != kSent) node[i] = f[(uint64_t)s2 * kBN + (((lz - 8 * oz) << 6) | ((ly - 8 * oy) << 3) | (lx - 8 * ox))];
  }
  __syncthreads();
  for (int i = t; i < 9 * 9 * 9; i += kThreads) {
    const int qz = i / 81, qy = (i / 9) % 9, qx = i % 9;
    double v = 0.0;
    for (int dz = -1; dz <= 0; ++dz) {
      const int z = org[2] + qz + dz;
      if (z < 0 || z >= res) continue;
      for (int dy = -1; dy <= 0; ++dy) {
        const int y = org[1] + qy + dy;
        if (y < 0 || y >= res) continue;
        for (int dx = -1; dx <= 0; ++dx) {
          const int x = org[0] + qx + dx;
          if (x < 0 || x >= res) continue;
          const double nv = node[((qz + dz + 1) * kMT + qy + dy + 1) * kMT + qx + dx + 1];
          v = xadd(v, xmul(xmul(xmul(nv, 0.5), 0.5), 0.5));
        }
      }
    }
    cv[i] = v;
  }
  __syncthreads();
}

// key of edge e of a cell: its lower grid position and axis, ((z (res+1) + y) (res+1) + x) 3 + axis
__device__ __forceinline__ uint64_t ab_edge_key(const int* cell, int e, uint64_t R1) {
  const int ia = c_abev[e][0], ib = c_abev[e][1];
  int st[3], axis = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    st[a] = cell[a] + min(c_abco[ia][a], c_abco[ib][a]);
    if (c_abco[ia][a] != c_abco[ib][a]) axis = a;
  }
  return (((uint64_t)st[2] * R1 + (uint64_t)st[1]) * R1 + (uint64_t)st[0]) * 3 + (uint64_t)axis;
}

__device__ __forceinline__ uint32_t ab_cell_case(const double* cv, int o, double iso) {
  const int z = o >> 6, y = (o >> 3) & 7, x = o & 7;
  uint32_t mc = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const double v = cv[((z + c_abco[k][2]) * 9 + y + c_abco[k][1]) * 9 + x + c_abco[k][0]];
    if (v < iso) mc |= 1u << k;
  }
  return mc;
}

__global__ void __launch_bounds__(kThreads) k_ab_mc_count(const double* __restrict__ f, const uint32_t* __restrict__ nbr,
                                                          const uint32_t* __restrict__ bkey, uint64_t NB,
                                                          const double* __restrict__ xc, Prolong W, int res, double iso,
                                                          uint32_t* __restrict__ ntri, uint32_t* __restrict__ nedge) {
  __shared__ double node[kMT * kMT * kMT], cv[729], scratch[kProlongScratch(kMT)];
  __shared__ uint32_t nb[27];
  typedef cub::BlockReduce<uint32_t, kThreads> BR;
  __shared__ typename BR::TempStorage tmp;
  const int t = threadIdx.x;
  for (uint64_t slot = blockIdx.x; slot < NB; slot += gridDim.x) {
    if (t < 27) nb[t] = nbr[27 * slot + t];
    __syncthreads();
    ab_corner_values(slot, nb, f, bkey, xc, W, res, node, cv, scratch);
    uint32_t a = 0, e = 0;
    for (int j = 0; j < 2; ++j) {
      const uint32_t mc = ab_cell_case(cv, 2 * t + j, iso);
      a += PR_MC_NTRI[mc];
      e += __popc(ab_edge_mask(mc));
    }
    const uint32_t ta = BR(tmp).Sum(a);
    __syncthreads();
    const uint32_t te = BR(tmp).Sum(e);
    if (t == 0) {
      ntri[slot] = ta;
      nedge[slot] = te;
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kThreads, 2) k_ab_mc_emit(const double* __restrict__ f, const uint32_t* __restrict__ nbr,
                                                         const uint32_t* __restrict__ bkey, uint64_t NB,
                                                         const double* __restrict__ xc, Prolong W, int res, double iso,
                                                         const uint64_t* __restrict__ toff, const uint64_t* __restrict__ eoff,
                                                         uint64_t* __restrict__ tri_key, uint64_t* __restrict__ edge_key,
                                                         double* __restrict__ epos) {
  __shared__ double node[kMT * kMT * kMT], cv[729], scratch[kProlongScratch(kMT)];
  __shared__ uint32_t nb[27];
  typedef cub::BlockScan<uint32_t, kThreads> BS;
  __shared__ typename BS::TempStorage tmp;
  const int t = threadIdx.x;
  const double w = 1.0 / (double)res;
  const uint64_t R1 = (uint64_t)res + 1;
  for (uint64_t slot = blockIdx.x; slot < NB; slot += gridDim.x) {
    if (t < 27) nb[t] = nbr[27 * slot + t];
    __syncthreads();
    ab_corner_values(slot, nb, f, bkey, xc, W, res, node, cv, scratch);
    uint32_t bx, by, bz;
    unmorton3(bkey[slot], bx, by, bz);
    const int org[3] = {8 * (int)bx, 8 * (int)by, 8 * (int)bz};
    uint32_t mc[2], ct = 0, ce = 0;
    for (int j = 0; j < 2; ++j) {
      mc[j] = ab_cell_case(cv, 2 * t + j, iso);
      ct += PR_MC_NTRI[mc[j]];
      ce += __popc(ab_edge_mask(mc[j]));
    }
    uint32_t pt, pe;
    BS(tmp).ExclusiveSum(ct, pt);
    __syncthreads();
    BS(tmp).ExclusiveSum(ce, pe);
    uint64_t to = toff[slot] + pt, eo = eoff[slot] + pe;
    for (int j = 0; j < 2; ++j) {
      const int o = 2 * t + j, cz = o >> 6, cy = (o >> 3) & 7, cx = o & 7;
      const int cell[3] = {org[0] + cx, org[1] + cy, org[2] + cz};
      const uint32_t em = ab_edge_mask(mc[j]);
      for (int e = 0; e < 12; ++e) {
        if (!((em >> e) & 1u)) continue;
        const int ia = c_abev[e][0], ib = c_abev[e][1];
        const double va = cv[((cz + c_abco[ia][2]) * 9 + cy + c_abco[ia][1]) * 9 + cx + c_abco[ia][0]];
        const double vb = cv[((cz + c_abco[ib][2]) * 9 + cy + c_abco[ib][1]) * 9 + cx + c_abco[ib][0]];
        const double dv = xsub(vb, va);
        const double tt = fabs(dv) < 1e-15 ? 0.5 : xdiv(xsub(iso, va), dv);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const double base = xmul((double)(cell[a] + c_abco[ia][a]), w);
          const double d = (double)(c_abco[ib][a] - c_abco[ia][a]);
          epos[3 * eo + a] = xadd(base, xmul(xmul(tt, d), w));
        }
        edge_key[eo] = ab_edge_key(cell, e, R1);
        ++eo;
      }
      const uint64_t packed = PR_MC_TRIS[mc[j]];
      const uint32_t ntr = PR_MC_NTRI[mc[j]];
      for (uint32_t i = 0; i < 3 * ntr; ++i) tri_key[3 * to + i] = ab_edge_key(cell, (int)((packed >> (4 * i)) & 15u), R1);
      to += ntr;
    }
    __syncthreads();
  }
}

__global__ void k_ab_heads(const uint64_t* __restrict__ skey, uint64_t E, uint32_t* __restrict__ head) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < E; i += (uint64_t)gridDim.x * blockDim.x)
    head[i] = (i == 0 || skey[i] != skey[i - 1]) ? 1u : 0u;
}
struct Mat16 {
  double m[16];  // column-major, as the crate's Mat4
};
__global__ void k_ab_vertices(const uint64_t* __restrict__ skey, const uint32_t* __restrict__ sslot,
                              const uint32_t* __restrict__ head, const uint32_t* __restrict__ vid, uint64_t E,
                              const double* __restrict__ epos, Mat16 Mi, uint64_t* __restrict__ vkey,
                              double* __restrict__ verts) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < E; i += (uint64_t)gridDim.x * blockDim.x) {
    if (!head[i]) continue;
    const uint64_t v = vid[i], s = sslot[i];
    const double p[3] = {epos[3 * s], epos[3 * s + 1], epos[3 * s + 2]};
    // Mat4::transform_point (src/geometry.rs:256-262) with the inverse transform
#pragma unroll
    for (int r = 0; r < 3; ++r)
      verts[3 * v + r] = xadd(xadd(xadd(xmul(Mi.m[r], p[0]), xmul(Mi.m[4 + r], p[1])), xmul(Mi.m[8 + r], p[2])), Mi.m[12 + r]);
    vkey[v] = skey[i];
  }
}
__global__ void k_ab_tris(const uint64_t* __restrict__ tri_key, uint64_t n, const uint64_t* __restrict__ vkey, uint64_t NV,
                          uint64_t* __restrict__ tris) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = tri_key[i];
    uint64_t a = 0, b = NV;
    while (a < b) {
      const uint64_t m = (a + b) >> 1;
      if (vkey[m] < k) a = m + 1;
      else b = m;
    }
    tris[i] = a;
  }
}

// ------------------------------------------------------------------ host side
Prolong make_prolong(int L, int resc) {
  std::vector<double> cur(1, 1.0);
  int lo = 0;
  const double wk[4] = {0.25, 0.75, 0.75, 0.25};  // fine 2i + k <- coarse i, k = -1..2
  for (int l = 0; l < L; ++l) {
    std::vector<double> nxt(2 * cur.size() + 2, 0.0);
    const int nlo = 2 * lo - 1;
    for (size_t i = 0; i < cur.size(); ++i)
      for (int k = -1; k <= 2; ++k) nxt[(size_t)(2 * (lo + (int)i) + k - nlo)] += cur[i] * wk[k + 1];
    cur.swap(nxt);
    lo = nlo;
  }
  PR_REQUIRE(cur.size() <= (size_t)kMaxW, PR_ERR_INTERNAL, "prolongation taps exceed the table");
  Prolong W{};
  for (size_t i = 0; i < cur.size(); ++i) W.w[i] = cur[i];
  W.kmin = lo;
  W.kmax = lo + (int)cur.size() - 1;
  W.L = L;
  W.resc = resc;
  return W;
}

template <typename T>
BandCoef<T> band_coef(uint32_t D, double pw) {
  double m[5], s[5], g[5];
  deg2_constants(m, s, g);
  const double h = 1.0 / (double)(1u << D);
  const double wh3 = pw > 0.0 ? pw * h * h * h / 1.5 : 0.0;
  BandCoef<T> K;
  for (int d = 0; d < 5; ++d) {
    K.m[d] = (T)m[d];
    K.s[d] = (T)s[d];
  }
  K.H = (T)h;
  K.wg = (T)(wh3 * 0.005);
  return K;
}

// the band system of the current adaptive state
struct Band {
  pr_context* c = nullptr;
  uint64_t NB = 0, n = 0, S = 0, P = 0;
  int res = 0;
  double wh3 = 0.0;
  const uint32_t *nbr = nullptr, *bkey = nullptr, *kin = nullptr, *snode = nullptr, *soff = nullptr, *sval = nullptr;
  const double* xc = nullptr;
  Prolong W{};
  double bytes = 0.0;

  void init(pr_context* ctx) {
    c = ctx;
    NB = c->band_nb;
    n = NB * kBN;
    P = c->P;
    S = c->S;
    res = 1 << c->D;
    const double h = 1.0 / (double)res;
    wh3 = c->pw > 0.0 ? c->pw * h * h * h / 1.5 : 0.0;
    nbr = c->get<uint32_t>("ab_nbr");
    bkey = c->get<uint32_t>("ab_bkey");
    xc = c->get<double>("ab_xc");
    W = make_prolong((int)(c->D - c->band_Dc), 1 << c->band_Dc);
    if (S > 0) {
      kin = c->get<uint32_t>("ab_kin");
      snode = c->get<uint32_t>("abs_runkey");
      soff = c->get<uint32_t>("abs_runoff");
      sval = c->get<uint32_t>("abs_val");
    }
  }
  template <typename T>
  const T* phi() {
    return sizeof(T) == 8 ? (const T*)c->get<double>("ab_phi64") : (const T*)c->get<float>("ab_phi32");
  }
  // y = A_BB x (kBandApply) or y = f - A_BB x (kBandResid), screening included
  template <typename T, int MODE>
  void op(const T* x, const T* f, T* y) {
    launch_op<T, MODE, false>(x, f, y, nullptr, 0.0, nullptr);
    bytes += 2.0 * n * sizeof(T) + (MODE == kBandResid ? n * sizeof(T) : 0.0);
    screen<T>(x, y, MODE == kBandApply ? 1.0 : -1.0, nullptr);
  }
  template <typename T, int MODE, bool GSRC>
  void launch_op(const T* x, const T* f, T* y, T* dout, double beta, double* part) {
    const size_t sm = band_op_smem<T>(GSRC);
    allow_smem(k_ab_op<T, MODE, GSRC>, sm);
    k_ab_op<T, MODE, GSRC><<<grid_op(), kOpThreads, sm, c->stream>>>(x, f, y, dout, beta, nbr, bkey, NB,
                                                                     band_coef<T>(c->D, c->pw), xc, W, res, part);
    PR_CHECK_LAUNCH();
  }
  unsigned grid_op() const { return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(NB, 148 * 16)); }
  // y += sign wh3 Phi Phi^T x; sq: per-block sums of proj^2 (returns their count)
  template <typename T>
  int screen(const T* x, T* y, double sign, double* sq) {
    if (S == 0 || !(wh3 > 0.0)) return 0;
    T* proj = c->buf<T>(std::string("ab_proj_") + tname<T>(), P);
    const unsigned np = grid_for(P, 1u << 20);
    k_ab_screen_proj<T><<<np, kThreads, 0, c->stream>>>(kin, phi<T>(), P, x, proj, sq);
    PR_CHECK_LAUNCH();
    k_ab_screen_gather<T><<<grid_for(S, 1u << 20), kThreads, 0, c->stream>>>(snode, soff, S, sval, phi<T>(), proj,
                                                                              (T)(sign * wh3), y);
    PR_CHECK_LAUNCH();
    bytes += (double)P * 27 * (4 + 2 * sizeof(T)) + (double)S * (8 + 2 * sizeof(T));
    return (int)np;
  }
  template <typename T>
  T* dinv() {
    const std::string nm = std::string("ab_dinv_") + tname<T>();
    auto it = c->bufs.find(nm);
    if (it != c->bufs.end() && it->second.ptr) return reinterpret_cast<T*>(it->second.ptr);
    T* d = c->buf<T>(nm, n);
    const BandCoef<double> K = band_coef<double>(c->D, c->pw);
    const double diag = (double)K.H * 3.0 * K.s[2] * K.m[2] * K.m[2] + (double)K.wg;
    k_ab_dinv<T><<<grid_for(n), kThreads, 0, c->stream>>>(diag, n, d);
    PR_CHECK_LAUNCH();
    if (S > 0 && wh3 > 0.0) {
      k_ab_dinv_screen<T><<<grid_for(S, 1u << 20), kThreads, 0, c->stream>>>(snode, c->get<double>("ab_sphi2"), S, diag,
                                                                              wh3, d);
      PR_CHECK_LAUNCH();
    }
    return d;
  }
};

void release_prefix(pr_context* c, const std::string& prefix);

// Jacobi-preconditioned CG on A_BB x = r from x = 0 until ||r|| <= tol; r is overwritten with
// the residual; returns the iterations.  Per iteration: one operator pass that forms the direction
// d = z + beta dold and q = A d with d . q (plus the screening pass), and one update pass x, r, z
// with r . r and r . z; every sum is a fixed-order FP64 sum of per-block partials.
template <typename T>
int band_pcg(Band& B, T* r, T* x, double tol, int maxit) {
  pr_context* c = B.c;
  const uint64_t n = B.n;
  cudaStream_t s = c->stream;
  const std::string tn = tname<T>();
  T* z = c->buf<T>("ab_z_" + tn, n);
  T* d = c->buf<T>("ab_d_" + tn, n);
  T* dn = c->buf<T>("ab_dn_" + tn, n);  // the direction alternates between d and dn
  T* q = c->buf<T>("ab_q_" + tn, n);
  const T* dv = B.dinv<T>();
  const int nbk = kDotBlocks;
  double* part = c->buf<double>("ab_part", 2 * (size_t)std::max<unsigned>(nbk, B.grid_op()));
  double* part2 = c->buf<double>("ab_part2", grid_for(B.P, 1u << 20));
  double* sums = c->buf<double>("ab_sums", 4);
  double* h = c->h_scalars;
  PR_CUDA(cudaMemsetAsync(x, 0, n * sizeof(T), s));
  k_ab_precond<T><<<nbk, kThreads, 0, s>>>(n, r, dv, z, part);
  PR_CHECK_LAUNCH();
  k_ab_sum_parts<<<2, 32, 0, s>>>(part, nbk, 2, 1.0, sums);
  PR_CHECK_LAUNCH();
  PR_CUDA(cudaMemcpyAsync(h, sums, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  c->sync();
  double rr = h[0], rz = h[1], beta = 0.0;
  B.bytes += 3.0 * n * sizeof(T);
  int it = 0;
  while (std::sqrt(rr) > tol && it < maxit) {
    // dn = z + beta d, q = A dn (beta = 0 on the first pass: d is not read)
    const int nop = (int)B.grid_op();
    B.launch_op<T, kBandDir, false>(d, z, q, dn, beta, part);
    std::swap(d, dn);
    const int nsq = B.screen<T>(d, q, 1.0, part2);
    k_ab_sum_parts<<<1, 32, 0, s>>>(part, nop, 1, 1.0, sums);
    PR_CHECK_LAUNCH();
    if (nsq) {
      k_ab_sum_parts<<<1, 32, 0, s>>>(part2, nsq, 1, B.wh3, sums + 2);
      PR_CHECK_LAUNCH();
    }
    PR_CUDA(cudaMemcpyAsync(h, sums, 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
    c->sync();
    const double dq = h[0] + (nsq ? h[2] : 0.0);
    B.bytes += 4.0 * n * sizeof(T);
    if (!(dq > 0.0)) break;
    const double alpha = rz / dq;
    k_ab_update<T><<<nbk, kThreads, 0, s>>>(n, alpha, d, q, x, r, dv, z, part);
    PR_CHECK_LAUNCH();
    k_ab_sum_parts<<<2, 32, 0, s>>>(part, nbk, 2, 1.0, sums);
    PR_CHECK_LAUNCH();
    PR_CUDA(cudaMemcpyAsync(h, sums, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    c->sync();
    B.bytes += 8.0 * n * sizeof(T);
    ++it;
    rr = h[0];
    beta = h[1] / rz;
    rz = h[1];
  }
  return it;
}

// A_BB e = r0 from e = 0 to ||r0 - A_BB e|| <= target ||b|| (bn = ||b||): Jacobi-PCG in FP32 with
// FP64 residual refinement, or in FP64 throughout.  The band solve gets 10 x max_iters PCG
// iterations (Jacobi preconditioning).  Returns the iterations; rn: the final residual norm.
int band_solve(Band& B, const double* r0, double bn, double* e64, const pr_params& p, double& rn, uint32_t& refinements) {
  pr_context* c = B.c;
  const uint64_t n = B.n;
  cudaStream_t s = c->stream;
  double* r64 = c->buf<double>("ab_r64", std::max<uint64_t>(n, 1));
  const double target = p.target_rel_residual > 0.0 ? p.target_rel_residual : 1e-6;
  const int max_iters = 10 * (p.max_iters > 0 ? (int)p.max_iters : 200);
  const bool mixed = p.precision != PR_PRECISION_FP64;
  int used = 0;
  refinements = 0;
  PR_CUDA(cudaMemcpyAsync(r64, r0, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  PR_CUDA(cudaMemsetAsync(e64, 0, n * sizeof(double), s));
  rn = std::sqrt(dot<double>(c, r64, r64, n));
  if (mixed) {
    float* r32 = c->buf<float>("ab_r32", n);
    float* e32 = c->buf<float>("ab_e32", n);
    const double inner = p.inner_rel_tol > 0.0 ? p.inner_rel_tol : 1e-4;
    while (rn > target * bn && used < max_iters) {
      convert_norm(c, r64, r32, n);
      const double tol = std::max(inner, 0.5 * target * bn / rn) * rn;
      const int it = band_pcg<float>(B, r32, e32, tol, max_iters - used);
      used += it;
      axpy<float, double>(s, n, 1.0, e32, e64);
      B.op<double, kBandResid>(e64, r0, r64);
      const double rn_new = std::sqrt(dot<double>(c, r64, r64, n));
      refinements++;
      const bool stalled = it == 0 || !(rn_new < rn);
      rn = rn_new;
      if (stalled) break;
    }
  } else if (rn > target * bn) {
    used = band_pcg<double>(B, r64, e64, 0.5 * target * bn, max_iters);
    B.op<double, kBandResid>(e64, r0, r64);
    rn = std::sqrt(dot<double>(c, r64, r64, n));
  }
  c->release("ab_r64");
  c->release("ab_r32");
  c->release("ab_e32");
  release_prefix(c, "ab_z_");
  release_prefix(c, "ab_d_");
  release_prefix(c, "ab_dn_");
  release_prefix(c, "ab_q_");
  c->release("ab_part");
  c->release("ab_part2");
  return used;
}

void release_prefix(pr_context* c, const std::string& prefix) {
  std::vector<std::string> names;
  for (const auto& kv : c->bufs)
    if (kv.first.compare(0, prefix.size(), prefix) == 0) names.push_back(kv.first);
  for (const auto& nm : names) c->release(nm);
}

// stable sort of m (key, value) pairs by 32-bit key and run-length encoding into "abs_*"; the
// run of kSent is dropped; returns the runs
uint64_t band_sort_segment(pr_context* c, const uint32_t* keys_in, const uint32_t* vals_in, uint64_t m) {
  uint32_t* keys = c->buf<uint32_t>("abs_key", m);
  uint32_t* vals = c->buf<uint32_t>("abs_val", m);
  uint32_t* run_key = c->buf<uint32_t>("abs_runkey", m);
  uint32_t* run_cnt = c->buf<uint32_t>("abs_runcnt", m + 1);
  uint32_t* run_off = c->buf<uint32_t>("abs_runoff", m + 1);
  uint32_t* nrun = c->buf<uint32_t>("ab_nrun", 2);
  size_t b1 = 0, b2 = 0, b3 = 0;
  PR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b1, keys_in, keys, vals_in, vals, (int64_t)m, 0, 32, c->stream));
  PR_CUDA(cub::DeviceRunLengthEncode::Encode(nullptr, b2, keys, run_key, run_cnt, nrun, (int64_t)m, c->stream));
  PR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, b3, run_cnt, run_off, (int64_t)(m + 1), c->stream));
  size_t tb = std::max(b1, std::max(b2, b3));
  void* tmp = c->buf<char>("ab_cub_tmp", tb);
  PR_COUNT_PRIMITIVE();
  PR_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, keys_in, keys, vals_in, vals, (int64_t)m, 0, 32, c->stream));
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
  if (R > 0 && h_last == kSent) --R;
  PR_CUDA(cudaMemsetAsync(run_cnt + R, 0, sizeof(uint32_t), c->stream));
  PR_COUNT_PRIMITIVE();
  PR_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, run_cnt, run_off, (int64_t)(R + 1), c->stream));
  return R;
}

// active bricks: sorted unique Morton codes in "ab_bkey"; returns their number
uint64_t find_bricks(pr_context* c, uint32_t D, bool full) {
  cudaStream_t s = c->stream;
  const uint32_t nres = 1u << (D - 3);
  const uint64_t nall = (uint64_t)nres * nres * nres;
  if (full) {
    uint32_t* bkey = c->buf<uint32_t>("ab_bkey", nall);
    k_ab_iota<<<grid_for(nall), kThreads, 0, s>>>(bkey, nall);
    PR_CHECK_LAUNCH();
    return nall;
  }
  const uint64_t m = 8 * c->P;
  uint32_t* kin = c->buf<uint32_t>("ab_bk_in", m);
  uint32_t* kso = c->buf<uint32_t>("ab_bk_sorted", m);
  uint32_t* kun = c->buf<uint32_t>("ab_bk_unique", m);
  uint32_t* nsel = c->buf<uint32_t>("ab_nsel", 2);
  k_ab_brick_keys<<<grid_for(c->P, 1u << 20), kThreads, 0, s>>>(c->get<double>("upos"), c->P, D, kin);
  PR_CHECK_LAUNCH();
  size_t b1 = 0, b2 = 0;
  PR_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, b1, kin, kso, (int64_t)m, 0, 32, s));
  PR_CUDA(cub::DeviceSelect::Unique(nullptr, b2, kso, kun, nsel, (int64_t)m, s));
  void* tmp = c->buf<char>("ab_cub_tmp", std::max(b1, b2));
  PR_COUNT_PRIMITIVE();
  PR_CUDA(cub::DeviceRadixSort::SortKeys(tmp, b1, kin, kso, (int64_t)m, 0, 32, s));
  PR_COUNT_PRIMITIVE();
  PR_CUDA(cub::DeviceSelect::Unique(tmp, b2, kso, kun, nsel, (int64_t)m, s));
  uint32_t h_n = 0, h_last = 0;
  PR_CUDA(cudaMemcpyAsync(&h_n, nsel, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  c->sync();
  if (h_n > 0) {
    PR_CUDA(cudaMemcpyAsync(&h_last, kun + (h_n - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    c->sync();
  }
  uint64_t NB = h_n;
  if (NB > 0 && h_last == kSent) --NB;
  PR_REQUIRE(NB < (1ull << 32) / kBN, PR_ERR_INVALID_ARGUMENT,
             "adaptive reconstruction: more than 8,388,607 active bricks (" + std::to_string(NB) + ")");
  uint32_t* bkey = c->buf<uint32_t>("ab_bkey", std::max<uint64_t>(NB, 1));
  if (NB) PR_CUDA(cudaMemcpyAsync(bkey, kun, NB * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  c->release("ab_bk_in");
  c->release("ab_bk_sorted");
  c->release("ab_bk_unique");
  return NB;
}

void band_setup(pr_context* c, uint32_t D, uint32_t Dc, double pw, bool full) {
  cudaStream_t s = c->stream;
  const uint64_t P = c->P;
  const uint64_t m = 27 * P;
  PR_REQUIRE(m < (1ull << 31), PR_ERR_INVALID_ARGUMENT, "degree 2 takes at most 79,536,431 points per call");
  const uint64_t NB = find_bricks(c, D, full);
  c->D = D;
  c->band_Dc = Dc;
  c->band_nb = NB;
  c->n = NB * kBN;
  c->pw = pw;
  c->adaptive = true;
  const uint32_t nres = 1u << (D - 3);
  const uint64_t nall = (uint64_t)nres * nres * nres;
  uint32_t* bmap = c->buf<uint32_t>("ab_bmap", nall);
  PR_CUDA(cudaMemsetAsync(bmap, 0xff, nall * sizeof(uint32_t), s));
  const uint32_t* bkey = c->get<uint32_t>("ab_bkey");
  if (NB) {
    k_ab_brick_map<<<grid_for(NB), kThreads, 0, s>>>(bkey, NB, bmap);
    PR_CHECK_LAUNCH();
  }
  uint32_t* nbr = c->buf<uint32_t>("ab_nbr", 27 * std::max<uint64_t>(NB, 1));
  if (NB) {
    k_ab_neighbours<<<grid_for(27 * NB, 1u << 20), kThreads, 0, s>>>(bkey, NB, nres, bmap, nbr);
    PR_CHECK_LAUNCH();
  }
  // (band node, point) pairs, splat, right-hand side
  uint32_t* kin = c->buf<uint32_t>("ab_kin", m);
  uint32_t* vin = c->buf<uint32_t>("ab_vin", m);
  double* phi64 = c->buf<double>("ab_phi64", m);
  float* phi32 = c->buf<float>("ab_phi32", m);
  unsigned long long* nin = c->buf<unsigned long long>("ab_nin", 1);
  PR_CUDA(cudaMemsetAsync(nin, 0, sizeof(unsigned long long), s));
  k_ab_pair_keys<<<grid_for(m, 1u << 20), kThreads, 0, s>>>(c->get<double>("upos"), P, D, bmap, kin, vin, phi64, phi32,
                                                            nin);
  PR_CHECK_LAUNCH();
  const uint64_t T = band_sort_segment(c, kin, vin, m);
  unsigned long long h_nin = 0;
  PR_CUDA(cudaMemcpyAsync(&h_nin, nin, sizeof(h_nin), cudaMemcpyDeviceToHost, s));
  c->sync();
  c->release("ab_vin");
  c->release("abs_key");
  c->release("abs_runcnt");
  c->release("ab_bmap");
  c->T = T;
  c->P_in = h_nin;
  double* nfc = c->buf<double>("ab_nfc", 3 * std::max<uint64_t>(T, 1));
  double* sphi = c->buf<double>("ab_sphi", std::max<uint64_t>(T, 1));
  double* sphi2 = c->buf<double>("ab_sphi2", std::max<uint64_t>(T, 1));
  const uint32_t* run_key = c->get<uint32_t>("abs_runkey");
  if (T) {
    k_ab_splat<<<grid_for(T, 1u << 20), kThreads, 0, s>>>(c->get<uint32_t>("abs_runoff"), T, c->get<uint32_t>("abs_val"),
                                                          phi64, c->get<double>("unrm"), P, nfc, sphi, sphi2);
    PR_CHECK_LAUNCH();
  }
  uint32_t* brun = c->buf<uint32_t>("ab_brun", NB + 1);
  k_ab_brick_runs<<<grid_for(NB + 1), kThreads, 0, s>>>(run_key, T, NB, brun);
  PR_CHECK_LAUNCH();
  const double h = 1.0 / (double)(1u << D);
  const double wh3 = pw > 0.0 ? pw * h * h * h / 1.5 : 0.0;
  double m5[5], s5[5], g5[5];
  deg2_constants(m5, s5, g5);
  BandCoef<double> K = band_coef<double>(D, pw);
  double* b = c->buf<double>("ab_b", std::max<uint64_t>(c->n, 1));
  const size_t smem = (3 * kOT3 + 8 * kOT * kOT + 8 * 8 * kOT + kBN) * sizeof(double);
  allow_smem(k_ab_rhs, smem);
  if (NB) {
    k_ab_rhs<<<brick_grid(NB), kThreads, smem, s>>>(nbr, run_key, brun, nfc, sphi, pw > 0.0 ? 0.5 * wh3 : 0.0, K, g5[0],
                                                    g5[1], g5[3], g5[4], h * h, NB, b);
    PR_CHECK_LAUNCH();
  }
  c->release("ab_nfc");
  c->release("ab_sphi");
  c->S = pw > 0.0 ? T : 0;
  c->S_pairs = 0;
  c->have_state = true;
}

}  // namespace

void stage_adaptive(pr_context* c, const pr_params& p, pr_stats& st, bool extract) {
  const uint32_t D = p.depth, Dc = p.coarse_depth;
  const double pw = p.point_weight;
  cudaStream_t s = c->stream;
  double t0 = now_seconds();
  release_prefix(c, "ab_");  // buffers of an earlier adaptive state (the Jacobi scales are cached)
  // 1. the dense coarse level
  pr_params pc = p;
  pc.depth = Dc;
  pc.coarse_depth = 0;
  c->adaptive = false;
  stage_setup_deg2(c, Dc, pw);
  c->sync();
  const double tc = now_seconds();
  pr_stats sc;
  std::memset(&sc, 0, sizeof(sc));
  stage_solve_deg2(c, pc, sc);
  const uint64_t nc = 1ull << (3 * Dc);
  double* xc = c->buf<double>("ab_xc", nc);
  PR_CUDA(cudaMemcpyAsync(xc, c->d2_xnat, nc * sizeof(double), cudaMemcpyDeviceToDevice, s));
  c->sync();
  c->d2_xnat = nullptr;
  release_prefix(c, "d2");
  release_prefix(c, "cub_tmp");
  double t1 = now_seconds();
  // 2. the band
  band_setup(c, D, Dc, pw, (p.band_flags & PR_BAND_FULL) != 0);
  c->sync();
  double t2 = now_seconds();
  st.time_tree = (tc - t0) + (t2 - t1);
  // 3. solve A_BB e = r0 = b - (A g)_B, f = g_B + e
  Band B;
  B.init(c);
  const uint64_t n = B.n;
  const double* b = c->get<double>("ab_b");
  double* gB = c->buf<double>("ab_g", std::max<uint64_t>(n, 1));
  const double target = p.target_rel_residual > 0.0 ? p.target_rel_residual : 1e-6;
  int used = 0;
  double bn = 0.0, rn = 0.0;
  st.pcg_iterations = sc.pcg_iterations;
  st.refinement_steps = 0;
  if (n > 0) {
    double* r0 = c->buf<double>("ab_r0", n);
    double* e64 = c->buf<double>("ab_e64", n);
    k_ab_prolong_band<<<brick_grid(B.NB), kThreads, 0, s>>>(B.bkey, B.NB, B.xc, B.W, B.res, gB);
    PR_CHECK_LAUNCH();
    B.launch_op<double, kBandResid, true>(nullptr, b, r0, nullptr, 0.0, nullptr);  // r0 = b - (K + wg) g
    B.screen<double>(gB, r0, -1.0, nullptr);
    bn = std::sqrt(dot<double>(c, b, b, n));
    used = band_solve(B, r0, bn, e64, p, rn, st.refinement_steps);
    double* f = c->buf<double>("ab_f", n);
    PR_CUDA(cudaMemcpyAsync(f, gB, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    axpy<double, double>(s, n, 1.0, e64, f);
  }
  c->release("ab_r0");
  c->release("ab_e64");
  c->sync();
  double t3 = now_seconds();
  st.time_solve = (t1 - tc) + (t3 - t2);
  st.rel_residual = bn > 0.0 ? rn / bn : 0.0;
  st.converged = st.rel_residual <= target ? 1 : 0;
  st.pcg_iterations += (uint32_t)used;
  st.solve_bytes = B.bytes + sc.solve_bytes;
  st.fem_nodes = n;
  st.points_in_cube = c->P_in;
  c->have_coeffs = true;
  c->coeffs_converged = true;
  if (!extract) return;
  // 4. iso value and marching cubes over the active bricks
  const uint64_t P = c->P;
  const double* f = c->get<double>("ab_f");
  double iso = 0.0;
  {
    int nb = (int)std::min<uint64_t>(kDotBlocks, (P + kThreads - 1) / kThreads);
    if (nb < 1) nb = 1;
    double* part = c->buf<double>("iso_part", 2 * (size_t)nb);
    double* out = c->buf<double>("iso_out", 1);
    k_ab_iso_partial<<<nb, kThreads, 0, s>>>(f, c->get<uint32_t>("ab_kin"), c->get<double>("ab_phi64"), P, part);
    PR_CHECK_LAUNCH();
    k_ab_iso_final<<<1, 32, 0, s>>>(part, nb, out);
    PR_CHECK_LAUNCH();
    PR_CUDA(cudaMemcpyAsync(&iso, out, sizeof(double), cudaMemcpyDeviceToHost, s));
    c->sync();
    iso /= (double)P;
  }
  const uint64_t NB = B.NB;
  c->nv = c->nt = 0;
  if (NB > 0) {
    uint32_t* bt = c->buf<uint32_t>("ab_mc_nt", NB + 1);
    uint32_t* be = c->buf<uint32_t>("ab_mc_ne", NB + 1);
    uint64_t* toff = c->buf<uint64_t>("ab_mc_toff", NB + 1);
    uint64_t* eoff = c->buf<uint64_t>("ab_mc_eoff", NB + 1);
    k_ab_mc_count<<<brick_grid(NB), kThreads, 0, s>>>(f, B.nbr, B.bkey, NB, B.xc, B.W, B.res, iso, bt, be);
    PR_CHECK_LAUNCH();
    PR_CUDA(cudaMemsetAsync(bt + NB, 0, sizeof(uint32_t), s));
    PR_CUDA(cudaMemsetAsync(be + NB, 0, sizeof(uint32_t), s));
    size_t b1 = 0;
    PR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, b1, bt, toff, (int64_t)(NB + 1), s));
    void* tmp = c->buf<char>("ab_cub_tmp", b1);
    PR_COUNT_PRIMITIVE();
    PR_CUDA(cub::DeviceScan::ExclusiveSum(tmp, b1, bt, toff, (int64_t)(NB + 1), s));
    PR_COUNT_PRIMITIVE();
    PR_CUDA(cub::DeviceScan::ExclusiveSum(tmp, b1, be, eoff, (int64_t)(NB + 1), s));
    uint64_t NT = 0, E = 0;
    PR_CUDA(cudaMemcpyAsync(&NT, toff + NB, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    PR_CUDA(cudaMemcpyAsync(&E, eoff + NB, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    c->sync();
    if (NT > 0 && E > 0) {
      PR_REQUIRE(E < (1ull << 32), PR_ERR_INVALID_ARGUMENT, "adaptive marching cubes: more than 2^32 cut edges");
      uint64_t* tri_key = c->buf<uint64_t>("ab_mc_tkey", 3 * NT);
      uint64_t* ekey = c->buf<uint64_t>("ab_mc_ekey", E);
      double* epos = c->buf<double>("ab_mc_epos", 3 * E);
      k_ab_mc_emit<<<brick_grid(NB), kThreads, 0, s>>>(f, B.nbr, B.bkey, NB, B.xc, B.W, B.res, iso, toff, eoff, tri_key,
                                                       ekey, epos);
      PR_CHECK_LAUNCH();
      uint32_t* eslot = c->buf<uint32_t>("ab_mc_eslot", E);
      k_ab_iota<<<grid_for(E, 1u << 20), kThreads, 0, s>>>(eslot, E);
      PR_CHECK_LAUNCH();
      uint64_t* skey = c->buf<uint64_t>("ab_mc_skey", E);
      uint32_t* sslot = c->buf<uint32_t>("ab_mc_sslot", E);
      uint32_t* head = c->buf<uint32_t>("ab_mc_head", E);
      uint32_t* vid = c->buf<uint32_t>("ab_mc_vid", E);
      size_t b2 = 0, b3 = 0;
      PR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b2, ekey, skey, eslot, sslot, (int64_t)E, 0, 64, s));
      PR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, b3, head, vid, (int64_t)E, s));
      tmp = c->buf<char>("ab_cub_tmp", std::max(b2, b3));
      PR_COUNT_PRIMITIVE();
      PR_CUDA(cub::DeviceRadixSort::SortPairs(tmp, b2, ekey, skey, eslot, sslot, (int64_t)E, 0, 64, s));
      k_ab_heads<<<grid_for(E, 1u << 20), kThreads, 0, s>>>(skey, E, head);
      PR_CHECK_LAUNCH();
      PR_COUNT_PRIMITIVE();
      PR_CUDA(cub::DeviceScan::ExclusiveSum(tmp, b3, head, vid, (int64_t)E, s));
      uint32_t h_vid = 0, h_head = 0;
      PR_CUDA(cudaMemcpyAsync(&h_vid, vid + (E - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      PR_CUDA(cudaMemcpyAsync(&h_head, head + (E - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      c->sync();
      const uint64_t NV = (uint64_t)h_vid + h_head;
      uint64_t* vkey = c->buf<uint64_t>("ab_mc_vkey", NV);
      double* verts = c->buf<double>("mesh_v", 3 * NV);
      uint64_t* tris = c->buf<uint64_t>("mesh_t", 3 * NT);
      Mat16 Mi;
      for (int k = 0; k < 16; ++k) Mi.m[k] = c->Minv[k];
      k_ab_vertices<<<grid_for(E, 1u << 20), kThreads, 0, s>>>(skey, sslot, head, vid, E, epos, Mi, vkey, verts);
      PR_CHECK_LAUNCH();
      k_ab_tris<<<grid_for(3 * NT, 1u << 20), kThreads, 0, s>>>(tri_key, 3 * NT, vkey, NV, tris);
      PR_CHECK_LAUNCH();
      c->sync();
      c->nv = NV;
      c->nt = NT;
      release_prefix(c, "ab_mc_");
    }
  }
  c->have_mesh = true;
  c->sync();
  double t4 = now_seconds();
  st.time_extract = t4 - t3;
  st.iso_value = iso;
  st.mesh_vertices = c->nv;
  st.mesh_triangles = c->nt;
  st.peak_device_bytes = (double)c->peak_bytes;
}

void band_vector(pr_context* c, int which, double* d_out) {
  PR_REQUIRE(c->adaptive, PR_ERR_STATE, "no adaptive reconstruction state");
  const char* nm = which == 0 ? "ab_b" : (which == 1 ? "ab_f" : "ab_g");
  PR_REQUIRE(which >= 0 && which <= 2, PR_ERR_INVALID_ARGUMENT, "band vector: which must be 0, 1 or 2");
  PR_REQUIRE(which != 1 || c->have_coeffs, PR_ERR_STATE, "no solved band coefficients");
  if (c->n) PR_CUDA(cudaMemcpyAsync(d_out, c->get<double>(nm), c->n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
}

void band_apply64(pr_context* c, const double* d_x, double* d_y) {
  PR_REQUIRE(c->adaptive, PR_ERR_STATE, "no adaptive reconstruction state");
  Band B;
  B.init(c);
  if (B.n) B.op<double, kBandApply>(d_x, nullptr, d_y);
}

namespace {

// ------------------------------------------------------------------ adjoint of the band
// L = sum_q g_q chi(q), chi the fine function u = sum_B f_i phi_i + sum_H g_j phi_j (g = P x_c).
// With w = d L / d u (the queries' basis values times g_q), the band equations R_B (A u - b) = 0
// and the coarse system A_c x_c = b_c:
//   A_BB lam = w_B                                   (band adjoint solve)
//   A_c mu_c = P^T (w_H - E_H A_HB lam)              (coarse adjoint solve)
// and every point's gradient is -lam^T (dA u - db) at depth D plus -mu_c^T (dA_c x_c - db_c) at
// the coarse depth (the dense degree-2 adjoint's per-point terms, pr_adjoint.cu).  dL/dg =
// w - A E lam (E: extension by zero), whose band rows w_B - A_BB lam vanish by the band adjoint
// equation: they are dropped rather than formed as a difference (A_c is nearly singular on smooth
// functions, and would amplify the solver's residual).  So only the ring of H nodes next to the
// band (A_HB lam: the stiffness, the screening stays inside the band) and the queries' terms on H
// nodes (w_H) reach the coarse level; with every brick active both are empty.

// band index of the in-grid fine node (x, y, z), kSent when its brick is not active
__device__ __forceinline__ uint32_t abj_index(const uint32_t* __restrict__ bmap, int64_t x, int64_t y, int64_t z) {
  const uint32_t slot = bmap[morton3((uint32_t)(x >> 3), (uint32_t)(y >> 3), (uint32_t)(z >> 3))];
  return slot == kSent ? kSent : slot * (uint32_t)kBN + (uint32_t)(((z & 7) << 6) | ((y & 7) << 3) | (x & 7));
}

// the coarse indices I (and taps k = f - 2^L I - kmin) of fine coordinate f: I in [lo, hi]
__device__ __forceinline__ void abj_coarse_range(const Prolong& W, int64_t f, int& lo, int& hi) {
  const int step = 1 << W.L;
  lo = max(0, -floor_div((int)(W.kmax - f), step));  // ceil((f - kmax) / step)
  hi = min(W.resc - 1, floor_div((int)(f - W.kmin), step));
}

// g at the in-grid fine node (x, y, z): the coarse function's depth-D coefficient
__device__ double abj_prolong_node(const double* __restrict__ xc, const Prolong& W, int64_t x, int64_t y, int64_t z) {
  const int step = 1 << W.L;
  int lo[3], hi[3];
  const int64_t f[3] = {x, y, z};
  for (int a = 0; a < 3; ++a) abj_coarse_range(W, f[a], lo[a], hi[a]);
  double v = 0.0;
  for (int iz = lo[2]; iz <= hi[2]; ++iz) {
    const double wz = W.w[f[2] - (int64_t)step * iz - W.kmin];
    for (int iy = lo[1]; iy <= hi[1]; ++iy) {
      const double wy = W.w[f[1] - (int64_t)step * iy - W.kmin];
      for (int ix = lo[0]; ix <= hi[0]; ++ix)
        v += W.w[f[0] - (int64_t)step * ix - W.kmin] * wy * wz *
             xc[(int64_t)ix + (int64_t)W.resc * (iy + (int64_t)W.resc * iz)];
    }
  }
  return v;
}

// chi at the queries (qu: 3 K, AoS unit coordinates) from f on the band and g elsewhere; missing:
// the queries with a node outside the band
__global__ void k_abj_eval(const double* __restrict__ qu, uint64_t K, uint32_t D, const uint32_t* __restrict__ bmap,
                           const double* __restrict__ f, const double* __restrict__ xc, Prolong W,
                           double* __restrict__ chi, unsigned long long* __restrict__ missing) {
  const int64_t res = 1ll << D;
  const double h = 1.0 / (double)res;
  unsigned long long cnt = 0;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < K; q += (uint64_t)gridDim.x * blockDim.x) {
    int64_t c[3];
    double b[3][3];
    for (int a = 0; a < 3; ++a) axis2b(qu[3 * q + a], h, c[a], b[a]);
    double v = 0.0;
    bool miss = false;
    for (int e = 0; e < 27; ++e) {
      const int64_t x = c[0] + e % 3 - 1, y = c[1] + (e / 3) % 3 - 1, z = c[2] + e / 9 - 1;
      if (x < 0 || y < 0 || z < 0 || x >= res || y >= res || z >= res) continue;
      const double phi = xmul(xmul(b[0][e % 3], b[1][(e / 3) % 3]), b[2][e / 9]);
      const uint32_t j = abj_index(bmap, x, y, z);
      double u;
      if (j != kSent) {
        u = f[j];
      } else {
        u = abj_prolong_node(xc, W, x, y, z);
        miss = true;
      }
      v = xadd(v, xmul(u, phi));
    }
    chi[q] = v;
    cnt += miss;
  }
  typedef cub::BlockReduce<unsigned long long, kThreads> BR;
  __shared__ typename BR::TempStorage tmp;
  const unsigned long long tot = BR(tmp).Sum(cnt);
  if (threadIdx.x == 0 && tot) atomicAdd(missing, tot);
}

// dL/dchi: the upstream gradient, or d mean(chi^2) / d chi
__global__ void k_abj_upstream(const double* __restrict__ chi, const double* __restrict__ dl, uint64_t K,
                               double* __restrict__ g) {
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < K; q += (uint64_t)gridDim.x * blockDim.x)
    g[q] = dl ? dl[q] : 2.0 * chi[q] / (double)K;
}

// (band node, 27 q + e) pairs of the queries' band nodes (kSent for the others) with the basis values
__global__ void k_abj_pairs(const double* __restrict__ qu, uint64_t K, uint32_t D, const uint32_t* __restrict__ bmap,
                            uint32_t* __restrict__ keys, uint32_t* __restrict__ vals, double* __restrict__ phi) {
  const int64_t res = 1ll << D;
  const double h = 1.0 / (double)res;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < 27 * K; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t q = i / 27;
    const int e = (int)(i - 27 * q);
    int64_t c[3];
    double b[3][3];
    for (int a = 0; a < 3; ++a) axis2b(qu[3 * q + a], h, c[a], b[a]);
    const int64_t x = c[0] + e % 3 - 1, y = c[1] + (e / 3) % 3 - 1, z = c[2] + e / 9 - 1;
    uint32_t key = kSent;
    if (x >= 0 && y >= 0 && z >= 0 && x < res && y < res && z < res) key = abj_index(bmap, x, y, z);
    keys[i] = key;
    vals[i] = (uint32_t)i;
    phi[i] = key != kSent ? xmul(xmul(b[0][e % 3], b[1][(e / 3) % 3]), b[2][e / 9]) : 0.0;
  }
}

// w on the band: per run (band node), the pairs' phi g_q in query order
__global__ void k_abj_scatter(const uint32_t* __restrict__ run_key, const uint32_t* __restrict__ run_off, uint64_t R,
                              const uint32_t* __restrict__ sval, const double* __restrict__ phi,
                              const double* __restrict__ g, double* __restrict__ w) {
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < R; r += (uint64_t)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (uint32_t e = run_off[r]; e < run_off[r + 1]; ++e) acc += phi[sval[e]] * g[sval[e] / 27];
    w[run_key[r]] = acc;
  }
}

// P^T of the queries' terms on nodes outside the band (w_H), added to the coarse right-hand side
__global__ void k_abj_missing(const double* __restrict__ qu, uint64_t K, uint32_t D, const uint32_t* __restrict__ bmap,
                              const double* __restrict__ g, Prolong W, double* __restrict__ yc) {
  const int64_t res = 1ll << D;
  const double h = 1.0 / (double)res;
  const int step = 1 << W.L;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < K; q += (uint64_t)gridDim.x * blockDim.x) {
    int64_t c[3];
    double b[3][3];
    for (int a = 0; a < 3; ++a) axis2b(qu[3 * q + a], h, c[a], b[a]);
    for (int e = 0; e < 27; ++e) {
      const int64_t f[3] = {c[0] + e % 3 - 1, c[1] + (e / 3) % 3 - 1, c[2] + e / 9 - 1};
      if (f[0] < 0 || f[1] < 0 || f[2] < 0 || f[0] >= res || f[1] >= res || f[2] >= res) continue;
      if (abj_index(bmap, f[0], f[1], f[2]) != kSent) continue;
      const double v = xmul(xmul(b[0][e % 3], b[1][(e / 3) % 3]), b[2][e / 9]) * g[q];
      int lo[3], hi[3];
      for (int a = 0; a < 3; ++a) abj_coarse_range(W, f[a], lo[a], hi[a]);
      for (int iz = lo[2]; iz <= hi[2]; ++iz)
        for (int iy = lo[1]; iy <= hi[1]; ++iy)
          for (int ix = lo[0]; ix <= hi[0]; ++ix)
            atomicAdd(yc + (int64_t)ix + (int64_t)W.resc * (iy + (int64_t)W.resc * iz),
                      v * W.w[f[0] - (int64_t)step * ix - W.kmin] * W.w[f[1] - (int64_t)step * iy - W.kmin] *
                          W.w[f[2] - (int64_t)step * iz - W.kmin]);
    }
  }
}

// mu = h^2 (G M M, M G M, M M G)^T lam at the band's touched nodes (run keys), lam 0 off the band
__global__ void k_abj_mu(const uint32_t* __restrict__ run_key, uint64_t T, const double* __restrict__ lam,
                         const uint32_t* __restrict__ nbr, uint32_t D, BandCoef<double> K, double g0, double g1,
                         double g3, double g4, double* __restrict__ mu) {
  const double h = 1.0 / (double)(1u << D);
  const double h2 = h * h;
  const double gg[5] = {g0, g1, 0.0, g3, g4};
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < T; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t j = run_key[t];
    const uint32_t slot = j / kBN, loc = j % kBN;
    const int lx = (int)(loc & 7), ly = (int)((loc >> 3) & 7), lz = (int)(loc >> 6);
    double m0 = 0.0, m1 = 0.0, m2 = 0.0;
    for (int dz = -2; dz <= 2; ++dz) {
      const int nz = lz - dz, bz = nz < 0 ? -1 : (nz > 7 ? 1 : 0);
      for (int dy = -2; dy <= 2; ++dy) {
        const int ny = ly - dy, by = ny < 0 ? -1 : (ny > 7 ? 1 : 0);
        for (int dx = -2; dx <= 2; ++dx) {
          const int nx = lx - dx, bx = nx < 0 ? -1 : (nx > 7 ? 1 : 0);
          const uint32_t ns = nbr[27 * (uint64_t)slot + 9 * (bz + 1) + 3 * (by + 1) + (bx + 1)];
          if (ns == kSent) continue;
          const double l = lam[(uint64_t)ns * kBN + (uint32_t)((((nz - 8 * bz)) << 6) | ((ny - 8 * by) << 3) | (nx - 8 * bx))] * h2;
          m0 += l * gg[dx + 2] * K.m[dy + 2] * K.m[dz + 2];
          m1 += l * K.m[dx + 2] * gg[dy + 2] * K.m[dz + 2];
          m2 += l * K.m[dx + 2] * K.m[dy + 2] * gg[dz + 2];
        }
      }
    }
    mu[t] = m0;
    mu[T + t] = m1;
    mu[2 * T + t] = m2;
  }
}

// Per brick: -(K E lam) on the window of the brick and its 2-node ring (12^3) for the brick's own
// lam, kept on the ring's H nodes (in the grid, in an inactive brick), then P^T of those into the
// coarse right-hand side yc (atomic adds: the sums over bricks come in no fixed order).
constexpr int kRW = 12, kRW3 = kRW * kRW * kRW;
constexpr size_t kRestrictSmem = (kBN + 2 * 8 * 8 * kRW + 3 * 8 * kRW * kRW + kRW3 + 9 * kRW * kRW + 81 * kRW) *
                                 sizeof(double);
__global__ void __launch_bounds__(kThreads) k_abj_restrict(const double* __restrict__ lam, const uint32_t* __restrict__ nbr,
                                                           const uint32_t* __restrict__ bkey, uint64_t NB,
                                                           BandCoef<double> K, Prolong W, int res,
                                                           double* __restrict__ yc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* lt = reinterpret_cast<double*>(smem_raw);  // [z][y][x] 8^3
  double* am = lt + kBN;                              // [z][y][ox] 8 x 8 x 12
  double* as = am + 8 * 8 * kRW;
  double* mm = as + 8 * 8 * kRW;                      // [z][oy][ox] 8 x 12 x 12
  double* ms = mm + 8 * kRW * kRW;
  double* sm = ms + 8 * kRW * kRW;
  double* tw = sm + 8 * kRW * kRW;                    // [oz][oy][ox] 12^3
  double* r1 = tw + kRW3;                             // [cz][oy][ox] 9 x 12 x 12
  double* r2 = r1 + 9 * kRW * kRW;                    // [cz][cy][ox] 9 x 9 x 12
  const int t = threadIdx.x;
  const int step = 1 << W.L;
  for (uint64_t sl = blockIdx.x; sl < NB; sl += gridDim.x) {
    uint32_t bx, by, bz;
    unmorton3(bkey[sl], bx, by, bz);
    const int o[3] = {8 * (int)bx - 2, 8 * (int)by - 2, 8 * (int)bz - 2};  // fine coordinate of window index 0
    for (int i = t; i < kBN; i += kThreads) lt[i] = lam[sl * kBN + i];
    __syncthreads();
    for (int i = t; i < 8 * 8 * kRW; i += kThreads) {  // x filters
      const int ox = i % kRW, zy = i / kRW;
      double a = 0.0, b = 0.0;
      for (int ix = max(0, ox - 4); ix <= min(7, ox); ++ix) {
        const int d = ox - 2 - ix + 2;
        a += K.m[d] * lt[zy * 8 + ix];
        b += K.s[d] * lt[zy * 8 + ix];
      }
      am[i] = a;
      as[i] = b;
    }
    __syncthreads();
    for (int i = t; i < 8 * kRW * kRW; i += kThreads) {  // y filters
      const int ox = i % kRW, oy = (i / kRW) % kRW, z = i / (kRW * kRW);
      double a = 0.0, b = 0.0, c = 0.0;
      for (int iy = max(0, oy - 4); iy <= min(7, oy); ++iy) {
        const int d = oy - 2 - iy + 2;
        const double xm = am[(z * 8 + iy) * kRW + ox], xs = as[(z * 8 + iy) * kRW + ox];
        a += K.m[d] * xm;
        b += K.s[d] * xm;
        c += K.m[d] * xs;
      }
      mm[i] = a;
      ms[i] = b;
      sm[i] = c;
    }
    __syncthreads();
    for (int i = t; i < kRW3; i += kThreads) {  // z filters; H nodes of the ring only
      const int ox = i % kRW, oy = (i / kRW) % kRW, oz = i / (kRW * kRW);
      const int bxo = ox < 2 ? -1 : (ox >= 10 ? 1 : 0), byo = oy < 2 ? -1 : (oy >= 10 ? 1 : 0),
                bzo = oz < 2 ? -1 : (oz >= 10 ? 1 : 0);
      const int fx = o[0] + ox, fy = o[1] + oy, fz = o[2] + oz;
      bool h_node = (bxo | byo | bzo) != 0 && fx >= 0 && fy >= 0 && fz >= 0 && fx < res && fy < res && fz < res;
      if (h_node) h_node = nbr[27 * sl + 9 * (bzo + 1) + 3 * (byo + 1) + (bxo + 1)] == kSent;
      double val = 0.0;
      if (h_node) {
        double a = 0.0;
        for (int iz = max(0, oz - 4); iz <= min(7, oz); ++iz) {
          const int d = oz - 2 - iz + 2;
          const int j = (iz * kRW + oy) * kRW + ox;
          a += K.m[d] * (sm[j] + ms[j]) + K.s[d] * mm[j];
        }
        val = -K.H * a;
      }
      tw[i] = val;
    }
    __syncthreads();
    int lo[3], cnt[3];
    for (int a = 0; a < 3; ++a) {
      int l, hh;
      abj_coarse_range(W, o[a], l, hh);
      int l2, h2;
      abj_coarse_range(W, o[a] + kRW - 1, l2, h2);
      lo[a] = l;
      cnt[a] = max(0, h2 - l + 1);
    }
    for (int i = t; i < cnt[2] * kRW * kRW; i += kThreads) {  // z: fine planes -> coarse planes
      const int yx = i % (kRW * kRW), cz = i / (kRW * kRW);
      const int I = lo[2] + cz;
      double a = 0.0;
      for (int oz = 0; oz < kRW; ++oz) {
        const int k = o[2] + oz - step * I - W.kmin;
        if (k >= 0 && k <= W.kmax - W.kmin) a += W.w[k] * tw[oz * kRW * kRW + yx];
      }
      r1[i] = a;
    }
    __syncthreads();
    for (int i = t; i < cnt[2] * cnt[1] * kRW; i += kThreads) {  // y
      const int ox = i % kRW, cy = (i / kRW) % cnt[1], cz = i / (kRW * cnt[1]);
      const int I = lo[1] + cy;
      double a = 0.0;
      for (int oy = 0; oy < kRW; ++oy) {
        const int k = o[1] + oy - step * I - W.kmin;
        if (k >= 0 && k <= W.kmax - W.kmin) a += W.w[k] * r1[(cz * kRW + oy) * kRW + ox];
      }
      r2[i] = a;
    }
    __syncthreads();
    for (int i = t; i < cnt[2] * cnt[1] * cnt[0]; i += kThreads) {  // x, then into the coarse grid
      const int cx = i % cnt[0], cy = (i / cnt[0]) % cnt[1], cz = i / (cnt[0] * cnt[1]);
      const int I = lo[0] + cx;
      double a = 0.0;
      for (int ox = 0; ox < kRW; ++ox) {
        const int k = o[0] + ox - step * I - W.kmin;
        if (k >= 0 && k <= W.kmax - W.kmin) a += W.w[k] * r2[(cz * cnt[1] + cy) * kRW + ox];
      }
      if (a != 0.0)
        atomicAdd(yc + (int64_t)I + (int64_t)W.resc * ((lo[1] + cy) + (int64_t)W.resc * (lo[2] + cz)), a);
    }
    __syncthreads();
  }
}

// Mat4::transform_point (src/geometry.rs:256-262), the forward transform's operation order
__global__ void k_abj_query_unit(const double* __restrict__ q3, uint64_t K, Mat16 M, double* __restrict__ qu) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < K; i += (uint64_t)gridDim.x * blockDim.x) {
    const double* p = q3 + 3 * i;
#pragma unroll
    for (int r = 0; r < 3; ++r)
      qu[3 * i + r] =
          xadd(xadd(xadd(xmul(M.m[r], p[0]), xmul(M.m[4 + r], p[1])), xmul(M.m[8 + r], p[2])), M.m[12 + r]);
  }
}

}  // namespace

void adjoint_backward_band(pr_context* c, const double* d_q3, uint64_t K, const double* d_dl, double* d_chi,
                           double* d_dpos, double* d_dnrm, pr_adjoint_stats& st) {
  cudaStream_t s = c->stream;
  const uint32_t D = c->D, Dc = c->band_Dc;
  const uint64_t NB = c->band_nb, n = c->n, P = c->P, T = c->T, S = c->S, Pin = c->P_in, Spairs = c->S_pairs;
  const double pw = c->pw;
  const pr_params prm = c->params;
  PR_REQUIRE(NB > 0, PR_ERR_STATE, "the adaptive reconstruction has no active bricks");
  Band B;
  B.init(c);
  const uint32_t nres = 1u << (D - 3);
  const uint64_t nall = (uint64_t)nres * nres * nres;
  uint32_t* bmap = c->buf<uint32_t>("ab_bmap", nall);
  PR_CUDA(cudaMemsetAsync(bmap, 0xff, nall * sizeof(uint32_t), s));
  k_ab_brick_map<<<grid_for(NB), kThreads, 0, s>>>(B.bkey, NB, bmap);
  PR_CHECK_LAUNCH();
  // chi and dL/dchi at the queries
  Mat16 M;
  for (int k = 0; k < 16; ++k) M.m[k] = c->M[k];
  double* qu = c->buf<double>("abj_qu", 3 * K);
  k_abj_query_unit<<<grid_for(K), kThreads, 0, s>>>(d_q3, K, M, qu);
  PR_CHECK_LAUNCH();
  const double* f = c->get<double>("ab_f");
  unsigned long long* miss = c->buf<unsigned long long>("abj_miss", 1);
  PR_CUDA(cudaMemsetAsync(miss, 0, sizeof(unsigned long long), s));
  k_abj_eval<<<grid_for(K), kThreads, 0, s>>>(qu, K, D, bmap, f, B.xc, B.W, d_chi, miss);
  PR_CHECK_LAUNCH();
  double* g = c->buf<double>("abj_g", K);
  k_abj_upstream<<<grid_for(K), kThreads, 0, s>>>(d_chi, d_dl, K, g);
  PR_CHECK_LAUNCH();
  st.loss = d_dl ? dot<double>(c, d_dl, d_chi, K) : dot<double>(c, d_chi, d_chi, K) / (double)K;
  unsigned long long h_miss = 0;
  PR_CUDA(cudaMemcpyAsync(&h_miss, miss, sizeof(h_miss), cudaMemcpyDeviceToHost, s));
  // w on the band: the queries' (band node, term) pairs sorted by node, summed in query order
  double* w = c->buf<double>("abj_w", n);
  PR_CUDA(cudaMemsetAsync(w, 0, n * sizeof(double), s));
  {
    uint32_t* kin = c->buf<uint32_t>("abj_kin", 27 * K);
    uint32_t* vin = c->buf<uint32_t>("abj_vin", 27 * K);
    double* qphi = c->buf<double>("abj_phi", 27 * K);
    k_abj_pairs<<<grid_for(27 * K, 1u << 20), kThreads, 0, s>>>(qu, K, D, bmap, kin, vin, qphi);
    PR_CHECK_LAUNCH();
    // the band's own sorted pairs ("abs_*") stay: sort the queries' under other names
    uint32_t* keys = c->buf<uint32_t>("abjs_key", 27 * K);
    uint32_t* vals = c->buf<uint32_t>("abjs_val", 27 * K);
    uint32_t* rkey = c->buf<uint32_t>("abjs_runkey", 27 * K);
    uint32_t* rcnt = c->buf<uint32_t>("abjs_runcnt", 27 * K + 1);
    uint32_t* roff = c->buf<uint32_t>("abjs_runoff", 27 * K + 1);
    uint32_t* nrun = c->buf<uint32_t>("abjs_nrun", 1);
    const int64_t m = (int64_t)(27 * K);
    size_t b1 = 0, b2 = 0, b3 = 0;
    PR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b1, kin, keys, vin, vals, m, 0, 32, s));
    PR_CUDA(cub::DeviceRunLengthEncode::Encode(nullptr, b2, keys, rkey, rcnt, nrun, m, s));
    PR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, b3, rcnt, roff, m + 1, s));
    size_t tb = std::max(b1, std::max(b2, b3));
    void* tmp = c->buf<char>("abj_cub_tmp", tb);
    PR_COUNT_PRIMITIVE();
    PR_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, kin, keys, vin, vals, m, 0, 32, s));
    PR_COUNT_PRIMITIVE();
    PR_CUDA(cub::DeviceRunLengthEncode::Encode(tmp, tb, keys, rkey, rcnt, nrun, m, s));
    uint32_t h_nrun = 0, h_last = 0;
    PR_CUDA(cudaMemcpyAsync(&h_nrun, nrun, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    c->sync();
    if (h_nrun > 0) {
      PR_CUDA(cudaMemcpyAsync(&h_last, rkey + (h_nrun - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      c->sync();
    }
    uint64_t R = h_nrun;
    if (R > 0 && h_last == kSent) --R;
    PR_CUDA(cudaMemsetAsync(rcnt + R, 0, sizeof(uint32_t), s));
    PR_COUNT_PRIMITIVE();
    PR_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, rcnt, roff, (int64_t)(R + 1), s));
    if (R > 0) {
      k_abj_scatter<<<grid_for(R, 1u << 20), kThreads, 0, s>>>(rkey, roff, R, vals, qphi, g, w);
      PR_CHECK_LAUNCH();
    }
    release_prefix(c, "abjs_");
    c->release("abj_kin");
    c->release("abj_vin");
    c->release("abj_phi");
    c->release("abj_cub_tmp");
  }
  // band adjoint solve A_BB lam = w_B
  double* lam = c->buf<double>("abj_lam", n);
  c->sync();
  const double t0 = now_seconds();
  const double wn = std::sqrt(dot<double>(c, w, w, n));
  double rn = 0.0;
  uint32_t refine = 0;
  int used = 0;
  if (wn > 0.0) used = band_solve(B, w, wn, lam, prm, rn, refine);
  else PR_CUDA(cudaMemsetAsync(lam, 0, n * sizeof(double), s));
  c->sync();
  const double t_band = now_seconds() - t0;
  const double target = prm.target_rel_residual > 0.0 ? prm.target_rel_residual : 1e-6;
  const double band_rel = wn > 0.0 ? rn / wn : 0.0;
  // the fine level's per-point terms (the band's pairs, runs, normal field; lam and u = f)
  const double h = 1.0 / (double)(1u << D);
  const double wh3 = pw > 0.0 ? pw * h * h * h / 1.5 : 0.0;
  if (T > 0) {
    double* nfc = c->buf<double>("ab_nfc", 3 * T);
    double* sphi = c->buf<double>("ab_sphi", T);
    double* sphi2 = c->buf<double>("ab_sphi2", T);
    k_ab_splat<<<grid_for(T, 1u << 20), kThreads, 0, s>>>(c->get<uint32_t>("abs_runoff"), T, c->get<uint32_t>("abs_val"),
                                                          c->get<double>("ab_phi64"), c->get<double>("unrm"), P, nfc,
                                                          sphi, sphi2);
    PR_CHECK_LAUNCH();
    double* mu = c->buf<double>("abj_mu", 3 * T);
    double m5[5], s5[5], g5[5];
    deg2_constants(m5, s5, g5);
    k_abj_mu<<<grid_for(T, 1u << 20), kThreads, 0, s>>>(c->get<uint32_t>("abs_runkey"), T, lam, B.nbr, D,
                                                        band_coef<double>(D, pw), g5[0], g5[1], g5[3], g5[4], mu);
    PR_CHECK_LAUNCH();
    double* wt = c->buf<double>("abj_wt", T);
    uint32_t* runidx = c->buf<uint32_t>("abj_runidx", 27 * P);
    run_weights2(c, c->get<uint32_t>("abs_runoff"), T, c->get<uint32_t>("abs_val"), c->get<double>("ab_phi64"), wt,
                 runidx);
    PointGrad2In a;
    a.upos = c->get<double>("upos");
    a.unrm = c->get<double>("unrm");
    a.ulen = c->get<double>("ulen");
    a.P = P;
    a.D = D;
    a.key = c->get<uint32_t>("ab_kin");
    a.sentinel = kSent;
    a.runidx = runidx;
    a.nfc = nfc;
    a.nfc_aos = 1;
    a.w = wt;
    a.mu = mu;
    a.T = T;
    a.lam = lam;
    a.x = f;
    a.wh3 = wh3;
    a.s = c->M[0];
    a.dpos = d_dpos;
    a.dnrm = d_dnrm;
    a.accumulate = 0;
    point_grad2(c, a);
    c->sync();
    c->release("ab_nfc");
    c->release("ab_sphi");
    c->release("abj_mu");
    c->release("abj_wt");
    c->release("abj_runidx");
  } else {
    PR_CUDA(cudaMemsetAsync(d_dpos, 0, 3 * P * sizeof(double), s));
    PR_CUDA(cudaMemsetAsync(d_dnrm, 0, 3 * P * sizeof(double), s));
  }
  // the coarse right-hand side P^T (w_H - E_H A_HB lam)
  const uint64_t ncs = 1ull << (3 * Dc);
  double* yc = c->buf<double>("abj_yc", ncs);
  PR_CUDA(cudaMemsetAsync(yc, 0, ncs * sizeof(double), s));
  allow_smem(k_abj_restrict, kRestrictSmem);
  k_abj_restrict<<<brick_grid(NB), kThreads, kRestrictSmem, s>>>(lam, B.nbr, B.bkey, NB, band_coef<double>(D, pw),
                                                                 B.W, B.res, yc);
  PR_CHECK_LAUNCH();
  if (h_miss > 0) {
    k_abj_missing<<<grid_for(K), kThreads, 0, s>>>(qu, K, D, bmap, g, B.W, yc);
    PR_CHECK_LAUNCH();
  }
  c->sync();
  c->release("abj_w");
  c->release("ab_bmap");
  c->release("abj_qu");
  c->release("abj_g");
  // the coarse adjoint: the dense degree-2 system at the coarse depth (set up again), A_c mu_c = yc,
  // and its per-point terms with mu_c and x_c, added
  double* xc_keep = c->buf<double>("abj_xc", ncs);
  PR_CUDA(cudaMemcpyAsync(xc_keep, B.xc, ncs * sizeof(double), cudaMemcpyDeviceToDevice, s));
  pr_params pc = prm;
  pc.depth = Dc;
  pc.coarse_depth = 0;
  stage_setup_deg2(c, Dc, pw);
  pr_stats sst;
  std::memset(&sst, 0, sizeof(sst));
  c->sync();
  const double t1 = now_seconds();
  solve_deg2(c, pc, sst, yc);
  c->sync();
  const double t_coarse = now_seconds() - t1;
  const uint64_t Tc = c->T;
  if (Tc > 0) {
    double* muc = c->buf<double>("abj_muc", 3 * Tc);
    mu2_dense(c, c->get<uint32_t>("d2s_runkey"), Tc, c->d2_xnat, Dc, muc);
    double* wc = c->buf<double>("abj_wc", Tc);
    uint32_t* runidx = c->buf<uint32_t>("abj_runidx", 27 * P);
    run_weights2(c, c->get<uint32_t>("d2s_runoff"), Tc, c->get<uint32_t>("d2s_val"), c->get<double>("d2_phi64"), wc,
                 runidx);
    const double hc = 1.0 / (double)(1u << Dc);
    PointGrad2In a;
    a.upos = c->get<double>("upos");
    a.unrm = c->get<double>("unrm");
    a.ulen = c->get<double>("ulen");
    a.P = P;
    a.D = Dc;
    a.key = c->get<uint32_t>("d2_kin");
    a.sentinel = 1u << (3 * Dc);
    a.runidx = runidx;
    a.nfc = c->get<double>("d2_nfc");
    a.w = wc;
    a.mu = muc;
    a.T = Tc;
    a.lam = c->d2_xnat;
    a.x = xc_keep;
    a.wh3 = pw > 0.0 ? pw * hc * hc * hc / 1.5 : 0.0;
    a.s = c->M[0];
    a.dpos = d_dpos;
    a.dnrm = d_dnrm;
    a.accumulate = 1;
    point_grad2(c, a);
    c->sync();
    c->release("abj_muc");
    c->release("abj_wc");
    c->release("abj_runidx");
  }
  // back to the band state
  c->d2_xnat = nullptr;
  release_prefix(c, "d2");
  release_prefix(c, "cub_tmp");
  c->release("abj_yc");
  c->release("abj_xc");
  c->release("abj_lam");
  c->D = D;
  c->n = n;
  c->T = T;
  c->S = S;
  c->S_pairs = Spairs;
  c->P_in = Pin;
  c->pw = pw;
  c->band_Dc = Dc;
  c->band_nb = NB;
  c->adaptive = true;
  c->degree = 2;
  c->params = prm;
  c->have_state = true;
  c->have_coeffs = true;
  c->coeffs_converged = true;
  st.time_solve = t_band + t_coarse;
  st.pcg_iterations = (uint32_t)used + sst.pcg_iterations;
  st.refinement_steps = refine + sst.refinement_steps;
  st.rel_residual = std::max(band_rel, sst.rel_residual);
  st.converged = band_rel <= target && sst.converged ? 1 : 0;
  st.queries_off_band = (int32_t)std::min<unsigned long long>(h_miss, 0x7fffffff);
}

}  // namespace pr

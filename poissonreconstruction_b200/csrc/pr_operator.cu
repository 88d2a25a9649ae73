// Matrix-free operator and multigrid kernels on the dense Morton-ordered grid.
//
// The crate assembles a CSR matrix (src/fem_tree.rs:180-249, 16 B per nonzero) and runs
// a row-parallel SpMV over it (src/sparse.rs:105-117).  Here the same operator is applied
// without a matrix: the stiffness is a constant 21-point stencil, the global screening
// mass is a diagonal shift, and the per-point screening blocks are applied as
// y += wh3 * Phi (Phi^T x) from a per-point payload (two small gather kernels).
//
// Vectors are indexed by the crate's FEM index (Morton, x in bit 0), so an 8^k block of
// nodes is contiguous; the smoother works on 8x8x8 bricks (512 contiguous entries).
#include <cub/cub.cuh>

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

// ------------------------------------------------------------------ stencil (one node per thread)
template <typename T, int MODE>
__global__ void k_stencil(uint32_t D, const T* __restrict__ x, const T* __restrict__ f, T* __restrict__ y, T c0, T ce,
                          T cc) {
  const int res = 1 << D;
  const uint64_t n = 1ull << (3 * D);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t ix, iy, iz;
    unmorton3((uint32_t)i, ix, iy, iz);
    uint32_t mx[3], my[3], mz[3];
    bool vx[3], vy[3], vz[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      int a = (int)ix + d - 1, b = (int)iy + d - 1, cz = (int)iz + d - 1;
      vx[d] = a >= 0 && a < res;
      vy[d] = b >= 0 && b < res;
      vz[d] = cz >= 0 && cz < res;
      mx[d] = vx[d] ? spread3(a) : 0u;
      my[d] = vy[d] ? spread3(b) << 1 : 0u;
      mz[d] = vz[d] ? spread3(cz) << 2 : 0u;
    }
    T se = 0, sc = 0;
#pragma unroll
    for (int dz = 0; dz < 3; ++dz)
#pragma unroll
      for (int dy = 0; dy < 3; ++dy)
#pragma unroll
        for (int dx = 0; dx < 3; ++dx) {
          int nz = (dx != 1) + (dy != 1) + (dz != 1);
          if (nz < 2) continue;
          if (!(vx[dx] && vy[dy] && vz[dz])) continue;
          T v = x[mx[dx] | my[dy] | mz[dz]];
          if (nz == 2) se += v;
          else sc += v;
        }
    T r = c0 * x[i] + ce * se + cc * sc;
    y[i] = MODE == 0 ? r : f[i] - r;
  }
}

// ------------------------------------------------------------------ screening
template <typename T>
__global__ void k_screen_project(const uint32_t* __restrict__ key, const T* __restrict__ phi, uint64_t P,
                                 uint32_t sentinel, const T* __restrict__ x, T* __restrict__ proj) {
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < P; p += (uint64_t)gridDim.x * blockDim.x) {
    T s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      uint32_t kk = key[8 * p + k];
      if (kk != sentinel) s += phi[8 * p + k] * x[kk];
    }
    proj[p] = s;
  }
}

template <typename T>
__global__ void k_screen_gather(const uint32_t* __restrict__ snode, const uint32_t* __restrict__ soff, uint64_t S,
                                const uint32_t* __restrict__ sval, const T* __restrict__ phi,
                                const T* __restrict__ proj, T wh3s, T* __restrict__ y) {
  for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < S; u += (uint64_t)gridDim.x * blockDim.x) {
    T acc = 0;
    for (uint32_t e = soff[u]; e < soff[u + 1]; ++e) {
      uint32_t pk = sval[e];
      acc += phi[pk] * proj[pk >> 3];
    }
    uint32_t node = snode[u];
    y[node] += wh3s * acc;
  }
}

// packed screening: cloud blockIdx.y, its descriptor and vector slice (n per cloud); the per-point
// and per-node arithmetic of k_screen_project / k_screen_gather
template <typename T>
__device__ __forceinline__ const T* sd_phi(const ScreenDesc& d);
template <>
__device__ __forceinline__ const float* sd_phi<float>(const ScreenDesc& d) { return d.phi32; }
template <>
__device__ __forceinline__ const double* sd_phi<double>(const ScreenDesc& d) { return d.phi64; }
template <typename T>
__device__ __forceinline__ T* sd_proj(const ScreenDesc& d);
template <>
__device__ __forceinline__ float* sd_proj<float>(const ScreenDesc& d) { return d.proj32; }
template <>
__device__ __forceinline__ double* sd_proj<double>(const ScreenDesc& d) { return d.proj64; }

// proj = Phi^T x; part (nullable): per-block sums of proj^2 (blockDim 256)
template <typename T>
__global__ void k_screen_project_pk(const ScreenDesc* __restrict__ desc, uint32_t sentinel, const T* __restrict__ x,
                                    uint64_t n, double* __restrict__ part) {
  const ScreenDesc d = desc[blockIdx.y];
  x = cloud_slice(x, n);
  const T* __restrict__ phi = sd_phi<T>(d);
  T* __restrict__ proj = sd_proj<T>(d);
  double acc = 0.0;
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < d.P; p += (uint64_t)gridDim.x * blockDim.x) {
    T s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const uint32_t kk = d.key[8 * p + k];
      if (kk != sentinel) s += phi[8 * p + k] * x[kk];
    }
    proj[p] = s;
    acc += (double)s * (double)s;
  }
  if (part) {
    typedef cub::BlockReduce<double, kThreads> BR;
    __shared__ typename BR::TempStorage tmp;
    const double t = BR(tmp).Sum(acc);
    if (threadIdx.x == 0) part[(uint64_t)blockIdx.y * gridDim.x + blockIdx.x] = t;
  }
}

template <typename T>
__global__ void k_screen_gather_pk(const ScreenDesc* __restrict__ desc, T wh3s, T* __restrict__ y, uint64_t n) {
  const ScreenDesc d = desc[blockIdx.y];
  y = cloud_slice(y, n);
  const T* __restrict__ phi = sd_phi<T>(d);
  const T* __restrict__ proj = sd_proj<T>(d);
  for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < d.S; u += (uint64_t)gridDim.x * blockDim.x) {
    T acc = 0;
    for (uint32_t e = d.soff[u]; e < d.soff[u + 1]; ++e) {
      const uint32_t pk = d.sval[e];
      acc += phi[pk] * proj[pk >> 3];
    }
    y[d.snode[u]] += wh3s * acc;
  }
}

// ------------------------------------------------------------------ dots / vector ops
template <typename TA, typename TB>
__global__ void k_dot_partial(const TA* __restrict__ a, const TB* __restrict__ b, uint64_t n, double* __restrict__ part) {
  double s = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    s += (double)a[i] * (double)b[i];
  typedef cub::BlockReduce<double, kThreads> BR;
  __shared__ typename BR::TempStorage tmp;
  double t = BR(tmp).Sum(s);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// 16-byte vector access in chunks of four elements (one float4, or two double2); used when every
// pointer of a call is 16-byte aligned, the scalar kernels otherwise
template <typename T>
struct Q4 {
  T v[4];
};
__device__ __forceinline__ Q4<float> ld4(const float* p, uint64_t i) {
  const float4 a = reinterpret_cast<const float4*>(p)[i];
  return Q4<float>{{a.x, a.y, a.z, a.w}};
}
__device__ __forceinline__ Q4<double> ld4(const double* p, uint64_t i) {
  const double2* q = reinterpret_cast<const double2*>(p) + 2 * i;
  const double2 a = q[0], b = q[1];
  return Q4<double>{{a.x, a.y, b.x, b.y}};
}
__device__ __forceinline__ void st4(float* p, uint64_t i, const Q4<float>& v) {
  reinterpret_cast<float4*>(p)[i] = make_float4(v.v[0], v.v[1], v.v[2], v.v[3]);
}
__device__ __forceinline__ void st4(double* p, uint64_t i, const Q4<double>& v) {
  double2* q = reinterpret_cast<double2*>(p) + 2 * i;
  q[0] = make_double2(v.v[0], v.v[1]);
  q[1] = make_double2(v.v[2], v.v[3]);
}
inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

template <typename T>
__global__ void k_dot_partial4(const T* __restrict__ a, const T* __restrict__ b, uint64_t n, double* __restrict__ part) {
  a = cloud_slice(a, n);  // packed launches: cloud blockIdx.y
  b = cloud_slice(b, n);
  part = cloud_slice(part, gridDim.x);
  double s = 0.0;
  const uint64_t n4 = n / 4, stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n4; i += stride) {
    const Q4<T> x = ld4(a, i), y = ld4(b, i);
#pragma unroll
    for (int k = 0; k < 4; ++k) s += (double)x.v[k] * (double)y.v[k];
  }
  for (uint64_t i = 4 * n4 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride)
    s += (double)a[i] * (double)b[i];
  typedef cub::BlockReduce<double, kThreads> BR;
  __shared__ typename BR::TempStorage tmp;
  const double t = BR(tmp).Sum(s);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

template <typename T>
__global__ void k_cg_update4(uint64_t n, T alpha, const T* __restrict__ d, const T* __restrict__ q, T* __restrict__ x,
                             T* __restrict__ r, double* __restrict__ part) {
  double s = 0.0;
  const uint64_t n4 = n / 4, stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n4; i += stride) {
    const Q4<T> dv = ld4(d, i), qv = ld4(q, i);
    Q4<T> xv = ld4(x, i), rv = ld4(r, i);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      xv.v[k] += alpha * dv.v[k];
      rv.v[k] = rv.v[k] - alpha * qv.v[k];
      s += (double)rv.v[k] * (double)rv.v[k];
    }
    st4(x, i, xv);
    st4(r, i, rv);
  }
  for (uint64_t i = 4 * n4 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    x[i] += alpha * d[i];
    const T ri = r[i] - alpha * q[i];
    r[i] = ri;
    s += (double)ri * (double)ri;
  }
  typedef cub::BlockReduce<double, kThreads> BR;
  __shared__ typename BR::TempStorage tmp;
  const double t = BR(tmp).Sum(s);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// r -= alpha q with per-block sums of r^2 (the CG residual update when x is updated elsewhere)
template <typename T>
__global__ void k_r_update4(uint64_t n, T alpha, const T* __restrict__ q, T* __restrict__ r,
                            double* __restrict__ part) {
  double s = 0.0;
  const uint64_t n4 = n / 4, stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n4; i += stride) {
    const Q4<T> qv = ld4(q, i);
    Q4<T> rv = ld4(r, i);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      rv.v[k] = rv.v[k] - alpha * qv.v[k];
      s += (double)rv.v[k] * (double)rv.v[k];
    }
    st4(r, i, rv);
  }
  for (uint64_t i = 4 * n4 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    const T ri = r[i] - alpha * q[i];
    r[i] = ri;
    s += (double)ri * (double)ri;
  }
  typedef cub::BlockReduce<double, kThreads> BR;
  __shared__ typename BR::TempStorage tmp;
  const double t = BR(tmp).Sum(s);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

template <typename T>
__global__ void k_xpby4(uint64_t n, const T* __restrict__ z, T beta, T* __restrict__ d) {
  const uint64_t n4 = n / 4, stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n4; i += stride) {
    const Q4<T> zv = ld4(z, i);
    Q4<T> dv = ld4(d, i);
#pragma unroll
    for (int k = 0; k < 4; ++k) dv.v[k] = zv.v[k] + beta * dv.v[k];
    st4(d, i, dv);
  }
  for (uint64_t i = 4 * n4 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride)
    d[i] = z[i] + beta * d[i];
}

template <typename Tin, typename Tout>
__global__ void k_axpy4(uint64_t n, double a, const Tin* __restrict__ x, Tout* __restrict__ y) {
  const uint64_t n4 = n / 4, stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n4; i += stride) {
    const Q4<Tin> xv = ld4(x, i);
    Q4<Tout> yv = ld4(y, i);
#pragma unroll
    for (int k = 0; k < 4; ++k) yv.v[k] = (Tout)((double)yv.v[k] + a * (double)xv.v[k]);
    st4(y, i, yv);
  }
  for (uint64_t i = 4 * n4 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride)
    y[i] = (Tout)((double)y[i] + a * (double)x[i]);
}

__global__ void k_convert_norm4(uint64_t n, const double* __restrict__ x, float* __restrict__ y,
                                double* __restrict__ part) {
  x = cloud_slice(x, n);  // packed launches: cloud blockIdx.y
  y = cloud_slice(y, n);
  part = cloud_slice(part, gridDim.x);
  double s = 0.0;
  const uint64_t n4 = n / 4, stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n4; i += stride) {
    const Q4<double> v = ld4(x, i);
    Q4<float> o;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      o.v[k] = (float)v.v[k];
      s += v.v[k] * v.v[k];
    }
    st4(y, i, o);
  }
  for (uint64_t i = 4 * n4 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    const double v = x[i];
    y[i] = (float)v;
    s += v * v;
  }
  typedef cub::BlockReduce<double, kThreads> BR;
  __shared__ typename BR::TempStorage tmp;
  const double t = BR(tmp).Sum(s);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void k_sum_final(const double* __restrict__ part, int np, double* __restrict__ out) {
  // one warp, fixed order: lane-strided partial sums then a fixed shuffle tree; block b sums the
  // partials of cloud b (packed launches)
  part += (uint64_t)blockIdx.x * np;
  out += blockIdx.x;
  double s = 0.0;
  for (int i = threadIdx.x; i < np; i += 32) s += part[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (threadIdx.x == 0) out[0] = s;
}

template <typename T>
__global__ void k_cg_update(uint64_t n, T alpha, const T* __restrict__ d, const T* __restrict__ q, T* __restrict__ x,
                            T* __restrict__ r, double* __restrict__ part) {
  double s = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    x[i] += alpha * d[i];
    T ri = r[i] - alpha * q[i];
    r[i] = ri;
    s += (double)ri * (double)ri;
  }
  typedef cub::BlockReduce<double, kThreads> BR;
  __shared__ typename BR::TempStorage tmp;
  double t = BR(tmp).Sum(s);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

template <typename T>
__global__ void k_xpby(uint64_t n, const T* __restrict__ z, T beta, T* __restrict__ d) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    d[i] = z[i] + beta * d[i];
}

// y = (float)x with per-block sums of x^2 (FP64), one pass
__global__ void k_convert_norm(uint64_t n, const double* __restrict__ x, float* __restrict__ y,
                               double* __restrict__ part) {
  double s = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const double v = x[i];
    y[i] = (float)v;
    s += v * v;
  }
  typedef cub::BlockReduce<double, kThreads> BR;
  __shared__ typename BR::TempStorage tmp;
  const double t = BR(tmp).Sum(s);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

template <typename Tin, typename Tout>
__global__ void k_scale_convert(uint64_t n, double a, const Tin* __restrict__ x, Tout* __restrict__ y) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    y[i] = (Tout)(a * (double)x[i]);
}

template <typename Tin, typename Tout>
__global__ void k_axpy(uint64_t n, double a, const Tin* __restrict__ x, Tout* __restrict__ y) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    y[i] = (Tout)((double)y[i] + a * (double)x[i]);
}

// ------------------------------------------------------------------ multicolour block Gauss-Seidel
// One launch updates every brick of one brick colour (brick Morton index & 7): bricks of a
// colour share no stencil neighbour, so the launch is an exact Gauss-Seidel step over them.
// Inside a brick, nodes are relaxed in 8 node colours (Morton index & 7), each colour
// class being independent.  Forward = colours ascending, backward = descending (its adjoint).
template <typename T>
__global__ void __launch_bounds__(64) k_gs_brick(uint32_t D, T* __restrict__ x, const T* __restrict__ f, T c0, T ce,
                                                 T cc, int colour, int forward) {
  __shared__ T tile[10][10][10];
  __shared__ T fs[512];
  const int res = 1 << D;
  const uint32_t B = (blockIdx.x << 3) | (uint32_t)colour;
  const uint64_t base = (uint64_t)B << 9;
  uint32_t bx, by, bz;
  unmorton3(B, bx, by, bz);
  const int ox = (int)bx * 8 - 1, oy = (int)by * 8 - 1, oz = (int)bz * 8 - 1;
  for (int t = threadIdx.x; t < 1000; t += blockDim.x) {
    int tz = t / 100, ty = (t / 10) % 10, tx = t % 10;
    int gx = ox + tx, gy = oy + ty, gz = oz + tz;
    T v = 0;
    if (gx >= 0 && gx < res && gy >= 0 && gy < res && gz >= 0 && gz < res) v = x[morton3(gx, gy, gz)];
    tile[tz][ty][tx] = v;
  }
  for (int t = threadIdx.x; t < 512; t += blockDim.x) fs[t] = f[base + t];
  __syncthreads();
  const T inv = (T)1 / c0;
  for (int step = 0; step < 8; ++step) {
    const int col = forward ? step : 7 - step;
    const uint32_t li = ((uint32_t)threadIdx.x << 3) | (uint32_t)col;  // local Morton index
    uint32_t lx, ly, lz;
    unmorton3(li, lx, ly, lz);
    const int cx = lx + 1, cy = ly + 1, czz = lz + 1;
    T se = 0, sc = 0;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
      for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
          int nz = (dx != 0) + (dy != 0) + (dz != 0);
          if (nz < 2) continue;
          T v = tile[czz + dz][cy + dy][cx + dx];
          if (nz == 2) se += v;
          else sc += v;
        }
    tile[czz][cy][cx] = (fs[li] - ce * se - cc * sc) * inv;
    __syncthreads();
  }
  for (int t = threadIdx.x; t < 512; t += blockDim.x) {
    uint32_t lx, ly, lz;
    unmorton3((uint32_t)t, lx, ly, lz);
    x[base + t] = tile[lz + 1][ly + 1][lx + 1];
  }
}

// ------------------------------------------------------------------ grid transfer (linear B-spline refinement)
// Prolongation P: fine node f takes coarse f/2 (weight 1) if f is even, (f-1)/2 and (f+1)/2
// (weight 1/2 each) if odd, per axis; restriction is P^T.
template <typename T>
__global__ void k_restrict(uint32_t Dc, const T* __restrict__ rf, T* __restrict__ fc) {
  const int resf = 2 << Dc;
  const uint64_t nc = 1ull << (3 * Dc);
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < nc; c += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t cx, cy, cz;
    unmorton3((uint32_t)c, cx, cy, cz);
    T s = 0;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz) {
      int fz = 2 * (int)cz + dz;
      if (fz < 0 || fz >= resf) continue;
#pragma unroll
      for (int dy = -1; dy <= 1; ++dy) {
        int fy = 2 * (int)cy + dy;
        if (fy < 0 || fy >= resf) continue;
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
          int fx = 2 * (int)cx + dx;
          if (fx < 0 || fx >= resf) continue;
          T w = (T)((dx ? 0.5 : 1.0) * (dy ? 0.5 : 1.0) * (dz ? 0.5 : 1.0));
          s += w * rf[morton3(fx, fy, fz)];
        }
      }
    }
    fc[c] = s;
  }
}

template <typename T>
__global__ void k_prolong_add(uint32_t Df, const T* __restrict__ ec, T* __restrict__ ef) {
  const int resc = 1 << (Df - 1);
  const uint64_t nf = 1ull << (3 * Df);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nf; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t fx, fy, fz;
    unmorton3((uint32_t)i, fx, fy, fz);
    int cxs[2], cys[2], czs[2];
    T wx[2], wy[2], wz[2];
    int nx = 0, ny = 0, nzc = 0;
    if (!(fx & 1)) { cxs[0] = fx >> 1; wx[0] = 1; nx = 1; }
    else { cxs[0] = fx >> 1; wx[0] = 0.5; nx = 1; if ((int)(fx >> 1) + 1 < resc) { cxs[1] = (fx >> 1) + 1; wx[1] = 0.5; nx = 2; } }
    if (!(fy & 1)) { cys[0] = fy >> 1; wy[0] = 1; ny = 1; }
    else { cys[0] = fy >> 1; wy[0] = 0.5; ny = 1; if ((int)(fy >> 1) + 1 < resc) { cys[1] = (fy >> 1) + 1; wy[1] = 0.5; ny = 2; } }
    if (!(fz & 1)) { czs[0] = fz >> 1; wz[0] = 1; nzc = 1; }
    else { czs[0] = fz >> 1; wz[0] = 0.5; nzc = 1; if ((int)(fz >> 1) + 1 < resc) { czs[1] = (fz >> 1) + 1; wz[1] = 0.5; nzc = 2; } }
    T s = 0;
    for (int a = 0; a < nzc; ++a)
      for (int b = 0; b < ny; ++b)
        for (int cI = 0; cI < nx; ++cI) s += wz[a] * wy[b] * wx[cI] * ec[morton3(cxs[cI], cys[b], czs[a])];
    ef[i] += s;
  }
}

template <typename T>
__global__ void k_dense_solve(uint32_t nc, const T* __restrict__ inv, const T* __restrict__ f, T* __restrict__ e) {
  __shared__ T fs[512];
  f = cloud_slice(f, nc);  // packed launches: cloud blockIdx.y
  e = cloud_slice(e, nc);
  for (uint32_t i = threadIdx.x; i < nc; i += blockDim.x) fs[i] = f[i];
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < nc; i += blockDim.x) {
    double s = 0.0;
    for (uint32_t j = 0; j < nc; ++j) s += (double)inv[(uint64_t)i * nc + j] * (double)fs[j];
    e[i] = (T)s;
  }
}

}  // namespace

// ====================================================================== wrappers
Coef<double> stencil_coef(uint32_t depth, double diag_shift) {
  // stiffness_entry (src/fem_tree.rs:44-48) evaluated with the crate's constants
  const double h = 1.0 / (double)(1u << depth);
  const double m0 = 2. / 3., m1 = 1. / 6., s0 = 2., s1 = -1.;
  Coef<double> c;
  c.c0 = (s0 * m0 * m0 + m0 * s0 * m0 + m0 * m0 * s0) * h + diag_shift;
  c.ce = (s1 * m1 * m0 + m1 * s1 * m0 + m1 * m1 * s0) * h;  // offsets (1,1,0)
  c.cc = (s1 * m1 * m1 + m1 * s1 * m1 + m1 * m1 * s1) * h;  // offsets (1,1,1)
  return c;
}

template <typename T>
void stencil_apply(cudaStream_t s, uint32_t D, const T* x, const T* f, T* y, Coef<T> c, int mode) {
  uint64_t n = 1ull << (3 * D);
  if (mode == 0) k_stencil<T, 0><<<grid_for(n), kThreads, 0, s>>>(D, x, f, y, c.c0, c.ce, c.cc);
  else k_stencil<T, 1><<<grid_for(n), kThreads, 0, s>>>(D, x, f, y, c.c0, c.ce, c.cc);
  PR_CHECK_LAUNCH();
}

template <typename T>
void screen_apply(cudaStream_t s, const Screen<T>& scr, const T* x, T* y, int sign) {
  if (!scr.active()) return;
  k_screen_project<T><<<grid_for(scr.P), kThreads, 0, s>>>(scr.key, scr.phi, scr.P, scr.sentinel, x, scr.proj);
  PR_CHECK_LAUNCH();
  k_screen_gather<T><<<grid_for(scr.S), kThreads, 0, s>>>(scr.snode, scr.soff, scr.S, scr.sval, scr.phi, scr.proj,
                                                          (T)sign * scr.wh3, y);
  PR_CHECK_LAUNCH();
}

template <typename T>
void screen_project(cudaStream_t s, const Screen<T>& scr, const T* x) {
  if (!scr.active()) return;
  k_screen_project<T><<<grid_for(scr.P), kThreads, 0, s>>>(scr.key, scr.phi, scr.P, scr.sentinel, x, scr.proj);
  PR_CHECK_LAUNCH();
}

template <typename T>
void screen_gather(cudaStream_t s, const Screen<T>& scr, T* y, int sign) {
  if (!scr.active()) return;
  k_screen_gather<T><<<grid_for(scr.S), kThreads, 0, s>>>(scr.snode, scr.soff, scr.S, scr.sval, scr.phi, scr.proj,
                                                          (T)sign * scr.wh3, y);
  PR_CHECK_LAUNCH();
}

template <typename T>
double dot(pr_context* c, const T* a, const T* b, uint64_t n) {
  double* part = c->buf<double>("dot_part", kDotBlocks);
  double* out = c->buf<double>("dot_out", 1);
  if (aligned16(a) && aligned16(b)) k_dot_partial4<T><<<kDotBlocks, kThreads, 0, c->stream>>>(a, b, n, part);
  else k_dot_partial<T, T><<<kDotBlocks, kThreads, 0, c->stream>>>(a, b, n, part);
  PR_CHECK_LAUNCH();
  k_sum_final<<<1, 32, 0, c->stream>>>(part, kDotBlocks, out);
  PR_CHECK_LAUNCH();
  PR_CUDA(cudaMemcpyAsync(c->h_scalars, out, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  c->sync();
  return c->h_scalars[0];
}

template <typename T>
void screen_project_pk(cudaStream_t s, const ScreenPack& scr, const T* x, uint64_t n, double* part, int nparts) {
  if (!scr.active()) return;
  const unsigned g = part ? (unsigned)nparts : grid_for(scr.maxP);
  k_screen_project_pk<T><<<dim3(g, scr.clouds), kThreads, 0, s>>>(scr.desc, scr.sentinel, x, n, part);
  PR_CHECK_LAUNCH();
}

template <typename T>
void screen_gather_pk(cudaStream_t s, const ScreenPack& scr, T* y, uint64_t n, int sign) {
  if (!scr.active()) return;
  k_screen_gather_pk<T><<<dim3(grid_for(scr.maxS), scr.clouds), kThreads, 0, s>>>(scr.desc, (T)sign * (T)scr.wh3,
                                                                                   y, n);
  PR_CHECK_LAUNCH();
}

template <typename T>
void dots_pk(cudaStream_t s, const T* a, const T* b, uint64_t n, uint32_t clouds, double* part, double* out) {
  PR_REQUIRE(aligned16(a) && aligned16(b), PR_ERR_INTERNAL, "packed dot products need 16-byte aligned vectors");
  k_dot_partial4<T><<<dim3(kDotBlocks, clouds), kThreads, 0, s>>>(a, b, n, part);
  PR_CHECK_LAUNCH();
  k_sum_final<<<clouds, 32, 0, s>>>(part, kDotBlocks, out);
  PR_CHECK_LAUNCH();
}

void convert_sq_pk(cudaStream_t s, const double* x, float* y, uint64_t n, uint32_t clouds, double* part, double* out) {
  PR_REQUIRE(aligned16(x) && aligned16(y), PR_ERR_INTERNAL, "packed conversion needs 16-byte aligned vectors");
  k_convert_norm4<<<dim3(kDotBlocks, clouds), kThreads, 0, s>>>(n, x, y, part);
  PR_CHECK_LAUNCH();
  k_sum_final<<<clouds, 32, 0, s>>>(part, kDotBlocks, out);
  PR_CHECK_LAUNCH();
}

template <typename T>
double cg_update(pr_context* c, uint64_t n, double alpha, const T* d, const T* q, T* x, T* r) {
  double* part = c->buf<double>("dot_part", kDotBlocks);
  double* out = c->buf<double>("dot_out", 1);
  if (aligned16(d) && aligned16(q) && aligned16(x) && aligned16(r))
    k_cg_update4<T><<<kDotBlocks, kThreads, 0, c->stream>>>(n, (T)alpha, d, q, x, r, part);
  else
    k_cg_update<T><<<kDotBlocks, kThreads, 0, c->stream>>>(n, (T)alpha, d, q, x, r, part);
  PR_CHECK_LAUNCH();
  k_sum_final<<<1, 32, 0, c->stream>>>(part, kDotBlocks, out);
  PR_CHECK_LAUNCH();
  PR_CUDA(cudaMemcpyAsync(c->h_scalars, out, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  c->sync();
  return c->h_scalars[0];
}

template <typename T>
double r_update(pr_context* c, uint64_t n, double alpha, const T* q, T* r) {
  PR_REQUIRE(aligned16(q) && aligned16(r), PR_ERR_INTERNAL, "r_update needs 16-byte aligned vectors");
  double* part = c->buf<double>("dot_part", kDotBlocks);
  double* out = c->buf<double>("dot_out", 1);
  k_r_update4<T><<<kDotBlocks, kThreads, 0, c->stream>>>(n, (T)alpha, q, r, part);
  PR_CHECK_LAUNCH();
  k_sum_final<<<1, 32, 0, c->stream>>>(part, kDotBlocks, out);
  PR_CHECK_LAUNCH();
  PR_CUDA(cudaMemcpyAsync(c->h_scalars, out, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  c->sync();
  return c->h_scalars[0];
}

double convert_norm(pr_context* c, const double* x, float* y, uint64_t n) {
  double* part = c->buf<double>("dot_part", kDotBlocks);
  double* out = c->buf<double>("dot_out", 1);
  if (aligned16(x) && aligned16(y)) k_convert_norm4<<<kDotBlocks, kThreads, 0, c->stream>>>(n, x, y, part);
  else k_convert_norm<<<kDotBlocks, kThreads, 0, c->stream>>>(n, x, y, part);
  PR_CHECK_LAUNCH();
  k_sum_final<<<1, 32, 0, c->stream>>>(part, kDotBlocks, out);
  PR_CHECK_LAUNCH();
  PR_CUDA(cudaMemcpyAsync(c->h_scalars, out, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  c->sync();
  return std::sqrt(c->h_scalars[0]);
}

template <typename T>
void xpby(cudaStream_t s, uint64_t n, const T* z, double beta, T* d) {
  if (aligned16(z) && aligned16(d)) k_xpby4<T><<<grid_for((n + 3) / 4), kThreads, 0, s>>>(n, z, (T)beta, d);
  else k_xpby<T><<<grid_for(n), kThreads, 0, s>>>(n, z, (T)beta, d);
  PR_CHECK_LAUNCH();
}

template <typename Tin, typename Tout>
void scale_convert(cudaStream_t s, uint64_t n, double a, const Tin* x, Tout* y) {
  k_scale_convert<Tin, Tout><<<grid_for(n), kThreads, 0, s>>>(n, a, x, y);
  PR_CHECK_LAUNCH();
}

template <typename Tin, typename Tout>
void axpy(cudaStream_t s, uint64_t n, double a, const Tin* x, Tout* y) {
  if (aligned16(x) && aligned16(y)) k_axpy4<Tin, Tout><<<grid_for((n + 3) / 4), kThreads, 0, s>>>(n, a, x, y);
  else k_axpy<Tin, Tout><<<grid_for(n), kThreads, 0, s>>>(n, a, x, y);
  PR_CHECK_LAUNCH();
}

template <typename T>
void gs_sweep(cudaStream_t s, uint32_t D, T* x, const T* f, Coef<T> c, bool forward) {
  if (D < 3) throw Error(PR_ERR_INTERNAL, "gs_sweep needs depth >= 3");
  if (D == 3) {  // a single brick: only brick colour 0 exists
    k_gs_brick<T><<<1, 64, 0, s>>>(D, x, f, c.c0, c.ce, c.cc, 0, forward ? 1 : 0);
    PR_CHECK_LAUNCH();
    return;
  }
  const unsigned per_colour = 1u << (3 * (D - 3) - 3);
  for (int step = 0; step < 8; ++step) {
    int col = forward ? step : 7 - step;
    k_gs_brick<T><<<per_colour, 64, 0, s>>>(D, x, f, c.c0, c.ce, c.cc, col, forward ? 1 : 0);
    PR_CHECK_LAUNCH();
  }
}

template <typename T>
void restrict_to_coarse(cudaStream_t s, uint32_t Df, const T* rf, T* fc) {
  uint64_t nc = 1ull << (3 * (Df - 1));
  k_restrict<T><<<grid_for(nc), kThreads, 0, s>>>(Df - 1, rf, fc);
  PR_CHECK_LAUNCH();
}

template <typename T>
void prolong_add(cudaStream_t s, uint32_t Df, const T* ec, T* ef) {
  uint64_t nf = 1ull << (3 * Df);
  k_prolong_add<T><<<grid_for(nf), kThreads, 0, s>>>(Df, ec, ef);
  PR_CHECK_LAUNCH();
}

template <typename T>
void dense_solve(cudaStream_t s, uint32_t nc, const T* inv, const T* f, T* e, uint32_t clouds) {
  k_dense_solve<T><<<dim3(1, clouds), 512, 0, s>>>(nc, inv, f, e);
  PR_CHECK_LAUNCH();
}

// explicit instantiations
#define PR_INST(T)                                                                                     \
  template void stencil_apply<T>(cudaStream_t, uint32_t, const T*, const T*, T*, Coef<T>, int);       \
  template void screen_apply<T>(cudaStream_t, const Screen<T>&, const T*, T*, int);                   \
  template void screen_project<T>(cudaStream_t, const Screen<T>&, const T*);                          \
  template void screen_gather<T>(cudaStream_t, const Screen<T>&, T*, int);                            \
  template double dot<T>(pr_context*, const T*, const T*, uint64_t);                                  \
  template double cg_update<T>(pr_context*, uint64_t, double, const T*, const T*, T*, T*);            \
  template double r_update<T>(pr_context*, uint64_t, double, const T*, T*);                           \
  template void xpby<T>(cudaStream_t, uint64_t, const T*, double, T*);                                \
  template void gs_sweep<T>(cudaStream_t, uint32_t, T*, const T*, Coef<T>, bool);                     \
  template void restrict_to_coarse<T>(cudaStream_t, uint32_t, const T*, T*);                          \
  template void prolong_add<T>(cudaStream_t, uint32_t, const T*, T*);                                 \
  template void dense_solve<T>(cudaStream_t, uint32_t, const T*, const T*, T*, uint32_t);              \
  template void screen_project_pk<T>(cudaStream_t, const ScreenPack&, const T*, uint64_t, double*, int); \
  template void screen_gather_pk<T>(cudaStream_t, const ScreenPack&, T*, uint64_t, int);                \
  template void dots_pk<T>(cudaStream_t, const T*, const T*, uint64_t, uint32_t, double*, double*);
PR_INST(float)
PR_INST(double)
#undef PR_INST
template void scale_convert<double, float>(cudaStream_t, uint64_t, double, const double*, float*);
template void scale_convert<float, double>(cudaStream_t, uint64_t, double, const float*, double*);
template void scale_convert<float, float>(cudaStream_t, uint64_t, double, const float*, float*);
template void scale_convert<double, double>(cudaStream_t, uint64_t, double, const double*, double*);
template void axpy<float, double>(cudaStream_t, uint64_t, double, const float*, double*);
template void axpy<float, float>(cudaStream_t, uint64_t, double, const float*, float*);
template void axpy<double, double>(cudaStream_t, uint64_t, double, const double*, double*);

double dot64(pr_context* c, const double* a, const double* b, uint64_t n) { return dot<double>(c, a, b, n); }

}  // namespace pr

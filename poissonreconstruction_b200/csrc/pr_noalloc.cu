// Iso value without any device allocation.
//
// pr_reconstruct computes the iso value (the mean of the implicit function over the input
// points, src/reconstructor.rs:56) with per-block partial sums held in a buffer that the
// context allocates.  Some callers cannot allocate device memory at all: a host application
// whose caching allocator already reserves the free device memory (a raw cudaMalloc then
// fails or fragments it), or a latency-bound loop that must not pay for the device-wide
// synchronisation cudaMalloc/cudaFree imply.  pr_iso_value_noalloc serves them: the caller
// passes device pointers for every input and for the output, and the partial sums live in
// a fixed file-scope __device__ array that every GPU loading this library keeps until exit.
//
// Only the crate's linear (degree-1) basis is evaluated, on coefficients in the FEM index
// order (Morton, x in bit 0).  The arithmetic (per-point evaluation, block-level Neumaier sums
// over the same fixed grid of at most 1184 blocks, the final compensated combine, one correctly
// rounded division by n) is the same as the iso value computed inside a degree-1
// pr_reconstruct, so for the same coefficients and points both return the same double.
//
// The device address of the scratch array is resolved once per device and cached; a
// cudaDeviceReset in the calling process invalidates it (the header says so).
#include <mutex>

#include "pr_internal.cuh"

namespace pr {
void set_last_error(const std::string& msg);  // the message pr_last_error() returns
}

namespace {

constexpr int kThreads = 256;
constexpr int kBlocks = 1184;                      // fixed grid: 8 x 148 SMs
constexpr uint64_t kMaxPointsNoAlloc = 1ull << 28;  // accepted input size

// 2 doubles (sum, compensation) per block: 2 * 1184 * 8 B = 18,944 bytes per device.
static __device__ __align__(256) double g_iso_scratch[2 * kBlocks];

__device__ __forceinline__ double bsp1(double t) {
  if (t < 0.0 || t > 2.0) return 0.0;
  if (t <= 1.0) return t;
  return pr::xsub(2.0, t);
}

// FEMTree::evaluate (src/fem_tree.rs:490-513), same operation order as the library's
// evaluation kernel
__device__ double eval_point(const double* __restrict__ x, uint32_t D, double px, double py, double pz) {
  using namespace pr;
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
    b[a][0] = bsp1(xsub(s[a], (double)o[a][0]));
    b[a][1] = bsp1(xsub(s[a], (double)o[a][1]));
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

// points: n x 3 (x y z), unit-cube positions; part: the static scratch (2 per block)
__global__ void k_iso_partial_noalloc(const double* __restrict__ x, uint32_t D, const double* __restrict__ pts,
                                      uint64_t n, double* __restrict__ part) {
  Neu acc{0.0, 0.0};
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    acc = neu_add(acc, eval_point(x, D, pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]));
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

__global__ void k_iso_final_noalloc(const double* __restrict__ part, int nb, uint64_t n, double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  Neu t{0.0, 0.0};
  for (int i = 0; i < nb; ++i) {
    t = neu_add(t, part[2 * i]);
    t = neu_add(t, part[2 * i + 1]);
  }
  out[0] = (t.s + t.c) / (double)n;
}

// Device address of g_iso_scratch for the current device, resolved once per device.
int scratch_address(double** out) {
  static std::mutex mu;
  static double* addr[64] = {nullptr};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    pr::set_last_error(std::string("cudaGetDevice failed: ") + cudaGetErrorString(e));
    return PR_ERR_NO_DEVICE;
  }
  if (dev < 0 || dev >= 64) {
    pr::set_last_error("device index above 63");
    return PR_ERR_INVALID_ARGUMENT;
  }
  std::lock_guard<std::mutex> g(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_iso_scratch);
    if (e != cudaSuccess) {
      pr::set_last_error(std::string("cudaGetSymbolAddress(iso scratch) failed: ") + cudaGetErrorString(e));
      return PR_ERR_CUDA;
    }
    addr[dev] = static_cast<double*>(p);
  }
  *out = addr[dev];
  return PR_OK;
}

}  // namespace

extern "C" {

// Iso value = mean of the implicit function of `d_coefficients` (res^3 FP64 coefficients of the
// degree-1 basis in the FEM index order, res = 2^depth) over n unit-cube points (d_points3: n x 3 doubles), written
// to d_iso[0]; enqueued on `stream` (NULL = the default stream) without synchronising and
// without allocating.  The first call on a device resolves the scratch address on the
// current device; make that first call before any stream capture.  Calls share one scratch
// array per device: calls whose kernels overlap on the GPU (different streams without
// ordering) race.  The cached scratch address is stale after a cudaDeviceReset in this process.
// Accepts 1 <= n <= 2^28 points and depth 1..10.
int pr_iso_value_noalloc(uint32_t depth, const double* d_coefficients, const double* d_points3, uint64_t n,
                         double* d_iso, void* stream) {
  if (!d_coefficients || !d_points3 || !d_iso) {
    pr::set_last_error("pr_iso_value_noalloc: NULL pointer");
    return PR_ERR_INVALID_ARGUMENT;
  }
  if (depth < 1 || depth > 10) {
    pr::set_last_error("pr_iso_value_noalloc: depth must be in [1, 10]");
    return PR_ERR_INVALID_ARGUMENT;
  }
  if (n == 0 || n > kMaxPointsNoAlloc) {
    pr::set_last_error("pr_iso_value_noalloc: n must be in [1, 2^28] points, got " + std::to_string(n));
    return PR_ERR_INVALID_ARGUMENT;
  }
  double* part = nullptr;
  const int rc = scratch_address(&part);
  if (rc != PR_OK) return rc;
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  int nb = (int)((n + kThreads - 1) / kThreads);
  if (nb > kBlocks) nb = kBlocks;
  // every partial slot the final kernel reads is written first: nothing needs zeroing
  k_iso_partial_noalloc<<<nb, kThreads, 0, s>>>(d_coefficients, depth, d_points3, n, part);
  pr::pr_count_launch_(0);
  k_iso_final_noalloc<<<1, 32, 0, s>>>(part, nb, n, d_iso);
  pr::pr_count_launch_(0);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    pr::set_last_error(std::string("pr_iso_value_noalloc launch failed: ") + cudaGetErrorString(e));
    return PR_ERR_CUDA;
  }
  return PR_OK;
}

}  // extern "C"

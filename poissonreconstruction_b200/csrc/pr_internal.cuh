// Internal declarations shared by the CUDA translation units of libpoisson_recon_b200.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <chrono>
#include <map>
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/poisson_recon.h"

namespace pr {

// ------------------------------------------------------------------ errors
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define PR_CUDA(call)                                                                              \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) {                                                                       \
      int code_ = (e_ == cudaErrorMemoryAllocation) ? PR_ERR_OUT_OF_MEMORY : PR_ERR_CUDA;          \
      throw ::pr::Error(code_, std::string(#call) + " failed: " + cudaGetErrorString(e_) + " at " + \
                                   __FILE__ + ":" + std::to_string(__LINE__));                     \
    }                                                                                              \
  } while (0)

// Every kernel launch of the library is followed by PR_CHECK_LAUNCH (error check + count);
// every CUB primitive call by PR_COUNT_PRIMITIVE.
extern "C" void pr_count_launch_(int primitive);
// launches (primitive 0) or primitive calls (1) counted on the calling thread so far
uint64_t thread_launch_count(int primitive);
#define PR_CHECK_LAUNCH()   \
  do {                      \
    pr_count_launch_(0);    \
    PR_CUDA(cudaGetLastError()); \
  } while (0)
#define PR_COUNT_PRIMITIVE() pr_count_launch_(1)

#define PR_REQUIRE(cond, code, msg)         \
  do {                                      \
    if (!(cond)) throw ::pr::Error(code, msg); \
  } while (0)

// ------------------------------------------------------------------ limits
constexpr uint32_t kMinDepth = 1;
constexpr uint32_t kMaxDepth = 10;              // dense grid: 2^30 nodes, 32-bit node index
constexpr uint32_t kMaxBandDepth = 12;          // adaptive band: brick codes of 3 x 9 bits
constexpr uint64_t kMaxPoints = 1ull << 28;     // 8 x points must fit a 31-bit pair index
constexpr uint32_t kCoarsestDepth = 3;          // multigrid direct-solve level (512 nodes)
constexpr int kDotBlocks = 1184;                // 8 x 148 SMs: fixed => deterministic dots

// ------------------------------------------------------------------ Morton (x in bit 0)
__host__ __device__ __forceinline__ uint32_t spread3(uint32_t v) {  // 10 bits -> 30 bits
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}
__host__ __device__ __forceinline__ uint32_t compact3(uint32_t v) {
  v &= 0x09249249u;
  v = (v | (v >> 2)) & 0x030c30c3u;
  v = (v | (v >> 4)) & 0x0300f00fu;
  v = (v | (v >> 8)) & 0x030000ffu;
  v = (v | (v >> 16)) & 0x000003ffu;
  return v;
}
__host__ __device__ __forceinline__ uint32_t morton3(uint32_t x, uint32_t y, uint32_t z) {
  return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}
__host__ __device__ __forceinline__ void unmorton3(uint32_t m, uint32_t& x, uint32_t& y, uint32_t& z) {
  x = compact3(m);
  y = compact3(m >> 1);
  z = compact3(m >> 2);
}

// Packed launches over several clouds of one depth: cloud blockIdx.y owns the slice
// [blockIdx.y * count, (blockIdx.y + 1) * count) of every vector (count = its per-cloud size), so
// a kernel shifts its pointers once and then runs its single-cloud body.  A null pointer stays null.
template <typename P>
__device__ __forceinline__ P* cloud_slice(P* p, uint64_t count) {
  return p ? p + (uint64_t)blockIdx.y * count : p;
}

// ------------------------------------------------------------------ exact FP64 (no contraction)
// The crate (Rust) never fuses multiply-add; kernels that must match it bit for bit use
// these round-to-nearest intrinsics, which the compiler never contracts.
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }

// Rust `f64 as i64` (saturating, NaN -> 0)
__host__ __device__ __forceinline__ int64_t sat_i64(double v) {
  if (v != v) return 0;
  if (v >= 9223372036854775807.0) return INT64_MAX;
  if (v <= -9223372036854775808.0) return INT64_MIN;
  return (int64_t)v;
}
// Rust `f64 as u64` (saturating, NaN -> 0)
__host__ __device__ __forceinline__ uint64_t sat_u64(double v) {
  if (!(v > 0.0)) return 0;
  if (v >= 18446744073709551615.0) return UINT64_MAX;
  return (uint64_t)v;
}

// ------------------------------------------------------------------ device buffers
struct DBuf {
  void* ptr = nullptr;
  size_t cap = 0;
};
// Frees the device memory the batch engine keeps between batches on `device` (pr_abi.cu); false
// if it holds none or is running.  A failed allocation calls it once and retries.
bool release_cached_memory(int device);
// Every context's spare blocks (released, kept for reuse) are guarded by one process-wide lock; a
// failed allocation frees the spare blocks of every context on its device (pr_abi.cu keeps the
// registry of contexts) and retries.
std::mutex& spare_mutex();
void free_all_spare(int device);

}  // namespace pr

// The context: one device, one stream, named device buffers reused across calls.
struct pr_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::map<std::string, pr::DBuf> bufs;
  size_t bytes_held = 0, peak_bytes = 0;
  // pinned scalar staging (dot products, counters)
  double* h_scalars = nullptr;  // 64 doubles
  double* h_pack = nullptr;     // more of them for packed solves (grown on demand)
  size_t h_pack_cap = 0;
  double* pinned_scalars(size_t count) {
    if (count <= 64) return h_scalars;
    if (h_pack_cap < count) {
      if (h_pack) PR_CUDA(cudaFreeHost(h_pack));
      h_pack = nullptr;
      h_pack_cap = 0;
      PR_CUDA(cudaMallocHost(&h_pack, count * sizeof(double)));
      h_pack_cap = count;
    }
    return h_pack;
  }
  // pinned staging for device->host mesh copies (grown on demand)
  unsigned char* h_stage = nullptr;
  size_t h_stage_cap = 0;
  std::vector<cudaEvent_t> copy_events;  // one per staged chunk of a mesh copy
  // --- state of the last reconstruction ---
  bool have_state = false;
  bool have_points = false;
  uint32_t D = 0;
  uint64_t n = 0;        // res^3
  uint64_t P = 0;        // input points
  uint64_t T = 0;        // splat-touched nodes
  uint64_t S = 0;        // screened nodes
  uint64_t S_pairs = 0;  // valid screening (node, point) pairs
  uint64_t P_in = 0;     // points with >= 1 screening node
  double pw = 0.0;
  double M[16], Minv[16];
  bool have_mesh = false;
  uint64_t nv = 0, nt = 0;
  bool have_coeffs = false;
  bool coeffs_converged = false;  // x64 solves A x = b (converged mode), not the reference schedule
  // reference schedule: its coarse right-hand side "ref_brhs" (depth ref_coarse_D, Morton order)
  // belongs to the current state
  bool have_ref_coarse = false;
  uint32_t ref_coarse_D = 0;
  // adaptive state: D = the band depth, band_Dc the coarse depth, band_nb active bricks (their
  // Morton brick codes in "ab_bkey"); band vectors hold 512 band_nb values
  bool adaptive = false;
  uint32_t band_Dc = 0;
  uint64_t band_nb = 0;
  int degree = 1;                 // node functions of the current state: 1 (the crate's) or 2
  // degree 2: the solved coefficients in natural order (one of the solver's buffers) and whether
  // their Morton copy "x64" is up to date (made on demand by coeffs_morton)
  const double* d2_xnat = nullptr;
  bool x64_ready = true;
  // a second stream for independent launches of one pass (made on first use), with the events that
  // fork it from and join it back to `stream`
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaStream_t side_stream() {
    if (!side) {
      PR_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
      PR_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
      PR_CUDA(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
    }
    return side;
  }
  pr_params params{};             // parameters of the last reconstruction
  // Instantiated CUDA graphs of repeated launch sequences on `stream` (the solver's V-cycle),
  // keyed by everything they were captured with (sizes, coefficients, buffer addresses); kept for
  // reuse, with the kernel launches they hold (counted again at every replay).
  struct Graph {
    cudaGraphExec_t exec = nullptr;
    uint64_t launches = 0, primitives = 0;
  };
  std::map<std::string, Graph> graphs;
  // Runs body() through the graph of `key`, capturing it on first use.
  template <typename F>
  void run_graph(const std::string& key, F body) {
    auto it = graphs.find(key);
    if (it == graphs.end()) {
      cudaGraph_t g = nullptr;
      const uint64_t l0 = pr::thread_launch_count(0), p0 = pr::thread_launch_count(1);
      PR_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      try {
        body();
      } catch (...) {
        cudaStreamEndCapture(stream, &g);
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        throw;
      }
      PR_CUDA(cudaStreamEndCapture(stream, &g));
      const uint64_t l1 = pr::thread_launch_count(0), p1 = pr::thread_launch_count(1);
      Graph gr;
      const cudaError_t e = cudaGraphInstantiate(&gr.exec, g, 0);
      cudaGraphDestroy(g);
      PR_CUDA(e);
      gr.launches = l1 - l0;
      gr.primitives = p1 - p0;
      PR_CUDA(cudaGraphLaunch(gr.exec, stream));  // counted by the capture
      graphs.emplace(key, gr);
      return;
    }
    PR_CUDA(cudaGraphLaunch(it->second.exec, stream));
    for (uint64_t k = 0; k < it->second.launches; ++k) pr::pr_count_launch_(0);
    for (uint64_t k = 0; k < it->second.primitives; ++k) pr::pr_count_launch_(1);
  }

  template <typename T>
  T* buf(const std::string& name, size_t count) {
    size_t bytes = count * sizeof(T);
    if (bytes == 0) bytes = 16;
    pr::DBuf& b = bufs[name];
    if (b.cap < bytes) {
      if (b.ptr) PR_CUDA(cudaStreamSynchronize(stream));
      std::unique_lock<std::mutex> lk(pr::spare_mutex());
      if (b.ptr) {  // too small: back to the spare blocks
        spare.insert({b.cap, b.ptr});
        spare_bytes += b.cap;
        b.ptr = nullptr;
        b.cap = 0;
      }
      size_t cap = (bytes + 255) & ~size_t(255);
      auto it = spare.lower_bound(cap);  // the smallest spare block that holds it, if not far larger
      if (it != spare.end() && it->first <= 2 * cap + (size_t(64) << 20)) {
        b.ptr = it->second;
        b.cap = it->first;
        spare_bytes -= it->first;
        spare.erase(it);
      } else {
        lk.unlock();
        cudaError_t e = cudaMalloc(&b.ptr, cap);
        if (e == cudaErrorMemoryAllocation) {  // every context's spare blocks, then the batch engine's
          cudaGetLastError();
          pr::free_all_spare(device);
          e = cudaMalloc(&b.ptr, cap);
          if (e == cudaErrorMemoryAllocation && pr::release_cached_memory(device)) {
            cudaGetLastError();
            e = cudaMalloc(&b.ptr, cap);
          }
        }
        lk.lock();
        if (e != cudaSuccess) {
          cudaGetLastError();
          b.ptr = nullptr;
          throw pr::Error(PR_ERR_OUT_OF_MEMORY, "cudaMalloc(" + std::to_string(cap) + " bytes) for '" + name +
                                                    "' failed: " + cudaGetErrorString(e));
        }
        b.cap = cap;
        bytes_held += cap;
      }
      const size_t live = bytes_held - spare_bytes;
      if (live > peak_bytes) peak_bytes = live;
    }
    return reinterpret_cast<T*>(b.ptr);
  }
  // Released blocks stay allocated and serve later requests of a similar size (cudaMalloc and
  // cudaFree synchronise the device and cost milliseconds per GB at this size); they are freed
  // when an allocation fails or the context is destroyed.  peak_bytes counts live buffers only.
  std::multimap<size_t, void*> spare;
  size_t spare_bytes = 0;
  void free_spare() {
    std::lock_guard<std::mutex> g(pr::spare_mutex());
    free_spare_locked();
  }
  void free_spare_locked() {  // the caller holds spare_mutex (spare blocks are idle: their stream was synchronised)
    for (auto& kv : spare) cudaFree(kv.second);
    bytes_held -= spare_bytes;
    spare.clear();
    spare_bytes = 0;
  }
  template <typename T>
  T* get(const std::string& name) {
    auto it = bufs.find(name);
    if (it == bufs.end() || !it->second.ptr) throw pr::Error(PR_ERR_INTERNAL, "missing device buffer '" + name + "'");
    return reinterpret_cast<T*>(it->second.ptr);
  }
  void release(const std::string& name) {
    auto it = bufs.find(name);
    if (it == bufs.end() || !it->second.ptr) return;
    PR_CUDA(cudaStreamSynchronize(stream));
    std::lock_guard<std::mutex> g(pr::spare_mutex());
    spare.insert({it->second.cap, it->second.ptr});
    spare_bytes += it->second.cap;
    bufs.erase(it);
  }
  void sync() { PR_CUDA(cudaStreamSynchronize(stream)); }
};

namespace pr {

// ------------------------------------------------------------------ stage entry points
// setup (pr_setup.cu)
void stage_transform(pr_context* c, const double* d_pts6, uint64_t n, double scale);
void stage_splat_rhs(pr_context* c, uint32_t depth, double pw);
// Stable sort of m (key, value) pairs by key (keys < 2^(3D+1)) and run-length encoding into
// the buffers tag_key/_val/_runkey/_runoff; the run of key 2^(3D) (sentinel) is dropped.
// Returns the number of valid runs.
uint64_t sort_and_segment(pr_context* c, const std::string& tag, uint32_t* keys_in, uint32_t* vals_in, uint64_t m,
                          uint32_t D);
// solve (pr_solve.cu): fills "x64"; returns rel residual etc. in stats
void stage_solve(pr_context* c, const pr_params& p, pr_stats& st);
// A x = b with the current system's operator (x = 0 initially; b, x: n doubles)
void solve_system(pr_context* c, const pr_params& p, pr_stats& st, const double* b, double* x);
// The degree-1 systems of several contexts (set up, one depth and screening weight, depth >= 5)
// solved together, one launch per step for all of them, on the stream and buffers of `sc`; each
// context's solution goes to its "x64" and its solve figures to st[k].  Bit-identical to
// stage_solve on each context.
void solve_packed(pr_context* sc, const std::vector<pr_context*>& clouds, const pr_params& p,
                  std::vector<pr_stats>& st);
// degree 2 (pr_deg2.cu): natural-order system, solve, accessors in Morton order
void stage_setup_deg2(pr_context* c, uint32_t depth, double pw);
void stage_solve_deg2(pr_context* c, const pr_params& p, pr_stats& st);
// A x = b with the degree-2 system of the context (natural order); the solution at c->d2_xnat
void solve_deg2(pr_context* c, const pr_params& p, pr_stats& st, const double* b);
// Pieces of the degree-2 adjoint (pr_adjoint.cu), shared by the dense grid and the adaptive band.
// Per point p: the gradient of L = lam^T (b - A x) w.r.t. its unit-cube position and normal, b and A
// the degree-2 system's (splat of the normals, screening) at depth D; key: 27 P node indices into
// lam and x (sentinel: no node), runidx: 27 P runs (touched nodes) of the pairs, nfc / w / mu: the
// runs' normal field, basis sums and the divergence stencil applied to lam (3 x T).  Writes (or with
// accumulate adds) s x the gradients into dpos / dnrm (P x 3 each, model space by s = M[0]).
struct PointGrad2In {
  const double* upos = nullptr;
  const double* unrm = nullptr;
  const double* ulen = nullptr;
  uint64_t P = 0;
  uint32_t D = 0;
  const uint32_t* key = nullptr;
  uint32_t sentinel = 0;
  const uint32_t* runidx = nullptr;
  const double* nfc = nullptr;
  int nfc_aos = 0;  // nfc as [T][3] (the band's) rather than [3][T]
  const double* w = nullptr;
  const double* mu = nullptr;
  uint64_t T = 0;
  const double* lam = nullptr;
  const double* x = nullptr;
  double wh3 = 0.0;
  double s = 0.0;
  double* dpos = nullptr;
  double* dnrm = nullptr;
  int accumulate = 0;
};
void point_grad2(pr_context* c, const PointGrad2In& a);
// w[t] = sum of the run's basis values (pair order), runidx[pair] = its run
void run_weights2(pr_context* c, const uint32_t* run_off, uint64_t T, const uint32_t* sval, const double* phi, double* w,
                  uint32_t* runidx);
// mu = h^2 (G M M, M G M, M M G)^T lam at the touched nodes of a dense natural-order grid
void mu2_dense(pr_context* c, const uint32_t* run_key, uint64_t T, const double* lam, uint32_t D, double* mu);
// adjoint of an adaptive reconstruction (pr_adaptive.cu): as adjoint_backward, band state
void adjoint_backward_band(pr_context* c, const double* d_q3, uint64_t K, const double* d_dl, double* d_chi,
                           double* d_dpos, double* d_dnrm, pr_adjoint_stats& st);
// adjoint of a degree-2 reconstruction (pr_adjoint.cu): as adjoint_backward, natural-order state
void adjoint_backward2(pr_context* c, const double* d_q3, uint64_t K, const double* d_dl, double* d_chi,
                       double* d_dpos, double* d_dnrm, pr_adjoint_stats& st);
void deg2_rhs_morton(pr_context* c, double* d_out);
void deg2_normal_field_morton(pr_context* c, double* d_nf3, double* d_w);
template <typename T>
void deg2_apply_morton(pr_context* c, const T* d_x, T* d_y);
double deg2_kernel_bench(pr_context* c, int kid, uint32_t depth, int precision, int reps, double* bytes);
// the 1-D integrals of N2 N2, N2' N2', N2' N2 at offsets -2..2
void deg2_constants(double* m5, double* s5, double* g5);
// adaptive (narrow-band) reconstruction (pr_adaptive.cu): a dense degree-2 coarse level at
// p.coarse_depth and the depth-p.depth system on the 8^3-node bricks around the points
void stage_adaptive(pr_context* c, const pr_params& p, pr_stats& st, bool extract);
// band accessors: which 0 = right-hand side, 1 = solved coefficients, 2 = the prolonged coarse
// function on the band (brick-major, natural order inside a brick); n = 512 band_nb doubles
void band_vector(pr_context* c, int which, double* d_out);
// y = A_BB x on the band (FP64, device vectors of 512 band_nb doubles)
void band_apply64(pr_context* c, const double* d_x, double* d_y);
// the solved coefficients in Morton order ("x64"), permuted from the degree-2 solver's order first
// when needed
const double* coeffs_morton(pr_context* c);
// extract (pr_mc.cu); `degree` selects the node functions (1: the crate's, 2: quadratic)
// natural: degree-2 coefficients in the solver's natural order instead of Morton order
double stage_iso(pr_context* c, const double* d_x64, bool natural = false);
void stage_extract(pr_context* c, uint32_t depth, const double* d_x64, double iso, bool back_transform,
                   int degree = 1, bool natural = false);
// degree 1 (the crate's basis), 2 (quadratic, Morton order) or 3 (quadratic, natural order)
void evaluate_points(pr_context* c, uint32_t depth, const double* d_x64, const double* d_pts, uint64_t stride,
                     uint64_t n, double* d_out, int degree = 1);

// the crate's CG loop (src/solvers.rs:20-69) on the current degree-1 fine system, FP64, from the
// iterate in d_x (n doubles, updated in place); delta (host, may be NULL) receives ||r||^2 before
// the first iteration and after each one (max_iters + 1 slots); returns the iteration count
uint64_t cg_reference_fine(pr_context* c, double* d_x, uint64_t max_iters, double accuracy, double* delta);

// operator helpers (pr_operator.cu), exposed for tests through the ABI
void apply_operator64(pr_context* c, const double* d_x, double* d_y);
void apply_operator32(pr_context* c, const float* d_x, float* d_y);

// dense-scatter helpers for accessors
void scatter_normal_field(pr_context* c, double* d_nf3, double* d_w);

double dot64(pr_context* c, const double* a, const double* b, uint64_t n);

// adjoint (pr_adjoint.cu): gradients of a loss on chi at model-space queries (device arrays)
void adjoint_backward(pr_context* c, const double* d_q3, uint64_t K, const double* d_dl, double* d_chi,
                      double* d_dpos, double* d_dnrm, pr_adjoint_stats& st);

// dynamic shared memory beyond 48 KB needs a per-kernel opt-in on each device: set once per
// (kernel, device), safe from several host threads
template <typename K>
void allow_smem(K kernel, size_t bytes) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  PR_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(mu);
  const auto key = std::make_pair(reinterpret_cast<const void*>(kernel), dev);
  if (done.count(key)) return;
  PR_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  done.insert(key);
}

inline double now_seconds() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace pr

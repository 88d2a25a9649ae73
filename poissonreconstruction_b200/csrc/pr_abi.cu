// C ABI of libpoisson_recon_b200 (declared in include/poisson_recon.h).
//
// pr_reconstruct mirrors reconstructor::reconstruct (src/reconstructor.rs:25-70):
//   bbox + unit-cube transform (stage_transform), tree + splat (stage_splat_rhs: the tree
//   is implicit, the FEM index is the Morton index), solve (stage_solve), iso value and
//   marching cubes (stage_iso / stage_extract), back-transform of the vertices.
// Every entry point converts exceptions into a status code and a thread-local message.
#include <sys/mman.h>
#include <unistd.h>

#include <atomic>
#include <unordered_map>
#include <map>
#include <set>
#include <mutex>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <tuple>
#include <vector>
#include <algorithm>

#include <cmath>

#include "pr_mg.cuh"

namespace pr {
void stage_solve_reference(pr_context* c, const pr_params& p, pr_stats& st);
}

namespace {

thread_local std::string g_last_error;

template <typename F>
int guard(F&& f) {
  try {
    f();
    return PR_OK;
  } catch (const pr::Error& e) {
    g_last_error = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    g_last_error = "host allocation failed";
    return PR_ERR_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return PR_ERR_INTERNAL;
  } catch (...) {
    g_last_error = "unknown error";
    return PR_ERR_INTERNAL;
  }
}

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

void validate(const pr_params* p) {
  PR_REQUIRE(p != nullptr, PR_ERR_INVALID_ARGUMENT, "params is NULL");
  if (p->coarse_depth > 0) {
    PR_REQUIRE(p->depth >= 3 && p->depth <= pr::kMaxBandDepth, PR_ERR_INVALID_ARGUMENT,
               "adaptive reconstruction: depth must be in [3, 12], got " + std::to_string(p->depth));
    PR_REQUIRE(p->coarse_depth < p->depth && p->depth - p->coarse_depth <= 4, PR_ERR_INVALID_ARGUMENT,
               "adaptive reconstruction: depth - coarse_depth must be in [1, 4]");
    PR_REQUIRE(p->degree == 2, PR_ERR_INVALID_ARGUMENT, "adaptive reconstruction is built for degree 2");
    PR_REQUIRE(p->solve_mode == PR_SOLVE_CONVERGED, PR_ERR_INVALID_ARGUMENT,
               "adaptive reconstruction solves in solve_mode PR_SOLVE_CONVERGED");
  } else {
    PR_REQUIRE(p->depth >= pr::kMinDepth && p->depth <= pr::kMaxDepth, PR_ERR_INVALID_ARGUMENT,
               "depth must be in [1, 10] (dense grid of 2^(3 depth) nodes), got " + std::to_string(p->depth));
  }
  PR_REQUIRE(std::isfinite(p->scale) && p->scale > 0.0, PR_ERR_INVALID_ARGUMENT, "scale must be finite and > 0");
  PR_REQUIRE(std::isfinite(p->point_weight) && p->point_weight >= 0.0, PR_ERR_INVALID_ARGUMENT,
             "point_weight must be finite and >= 0");
  PR_REQUIRE(p->solve_mode == PR_SOLVE_CONVERGED || p->solve_mode == PR_SOLVE_REFERENCE_SCHEDULE,
             PR_ERR_INVALID_ARGUMENT, "unknown solve_mode");
  PR_REQUIRE(p->precision == PR_PRECISION_MIXED || p->precision == PR_PRECISION_FP64, PR_ERR_INVALID_ARGUMENT,
             "unknown precision");
  PR_REQUIRE(!(p->target_rel_residual < 0.0) && std::isfinite(p->target_rel_residual), PR_ERR_INVALID_ARGUMENT,
             "target_rel_residual must be finite and >= 0");
  PR_REQUIRE(p->degree <= 2, PR_ERR_INVALID_ARGUMENT, "degree must be 1 or 2, got " + std::to_string(p->degree));
  PR_REQUIRE(p->degree != 2 || p->solve_mode == PR_SOLVE_CONVERGED, PR_ERR_INVALID_ARGUMENT,
             "degree 2 is solved in solve_mode PR_SOLVE_CONVERGED only");
}

int degree_of(const pr_params& p) { return p.degree == 2 ? 2 : 1; }

void set_device(pr_context* c) { PR_CUDA(cudaSetDevice(c->device)); }

// Pool of pinned host blocks for returned meshes.  A mesh copied into pinned memory needs one
// DMA and no host copy; pinning fresh memory is slow, so blocks released by pr_mesh_free /
// pr_host_free are kept (up to PR_HOST_POOL_MB; 0 disables the pool) and handed out again to
// later meshes of a similar size.  Blocks stay pinned until exit.  The default keeps up to an
// eighth of the physical memory, between 4 and 32 GiB: a batch of a few hundred clouds returns
// several GiB of meshes, and a pool smaller than one batch's output re-pins (and unpins, both
// device-synchronising) the difference on every batch.
struct HostPool {
  std::mutex mu;
  std::multimap<size_t, void*> idle;        // capacity -> block
  std::unordered_map<void*, size_t> owned;  // every pool block -> capacity
  size_t idle_bytes = 0;
  size_t limit = 0;
  HostPool() {
    const char* e = std::getenv("PR_HOST_POOL_MB");
    if (e) {
      limit = (size_t)std::strtoull(e, nullptr, 10) << 20;
    } else {
      const long pages = sysconf(_SC_PHYS_PAGES), page = sysconf(_SC_PAGESIZE);
      const size_t phys = pages > 0 && page > 0 ? (size_t)pages * (size_t)page : 0;
      limit = std::min(std::max(phys / 8, size_t(4) << 30), size_t(32) << 30);
    }
  }
};
HostPool& host_pool() {
  static HostPool* p = new HostPool();  // never destroyed: blocks may be freed during exit
  return *p;
}
// A pinned block of >= bytes, or nullptr (pool disabled, or pinning failed).
void* pool_alloc(size_t bytes) {
  HostPool& hp = host_pool();
  if (hp.limit == 0 || bytes == 0) return nullptr;
  {
    std::lock_guard<std::mutex> g(hp.mu);
    auto it = hp.idle.lower_bound(bytes);
    if (it != hp.idle.end() && it->first <= 2 * bytes + (size_t(64) << 20)) {
      void* p = it->second;
      hp.idle_bytes -= it->first;
      hp.idle.erase(it);
      return p;
    }
  }
  const size_t cap = (bytes + (size_t(2) << 20) - 1) & ~((size_t(2) << 20) - 1);
  void* p = nullptr;
  if (cudaHostAlloc(&p, cap, cudaHostAllocPortable) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  std::lock_guard<std::mutex> g(hp.mu);
  hp.owned[p] = cap;
  return p;
}
// Returns false if p is not a pool block.
bool pool_release(void* p) {
  if (!p) return true;
  HostPool& hp = host_pool();
  std::vector<void*> evict;
  {
    std::lock_guard<std::mutex> g(hp.mu);
    auto it = hp.owned.find(p);
    if (it == hp.owned.end()) return false;
    hp.idle.insert({it->second, p});
    hp.idle_bytes += it->second;
    while (hp.idle_bytes > hp.limit && !hp.idle.empty()) {  // drop the largest idle blocks
      auto last = std::prev(hp.idle.end());
      hp.idle_bytes -= last->first;
      hp.owned.erase(last->second);
      evict.push_back(last->second);
      hp.idle.erase(last);
    }
  }
  for (void* q : evict) cudaFreeHost(q);
  return true;
}

// Host output buffer of the mesh: 2 MiB-aligned and advised for transparent huge pages when
// large, so that first-touch page faults (which dominate a copy into fresh memory) are few.
// Freed with free() like any malloc'd block.
void* alloc_host_out(size_t bytes) {
  if (bytes == 0) return nullptr;
  if (bytes < (size_t(4) << 20)) return std::malloc(bytes);
  void* p = nullptr;
  if (posix_memalign(&p, size_t(2) << 20, bytes) != 0) return nullptr;
  madvise(p, bytes & ~((size_t(2) << 20) - 1), MADV_HUGEPAGE);  // advisory; failure is harmless
  return p;
}

// Device mesh -> caller memory: D2H copies of 8 MiB chunks into the context's pinned staging,
// each followed by an event, while host threads copy finished chunks on to the output
// buffers (the DMA of later chunks overlaps the host copies and page faults of earlier ones).
void copy_mesh_to_host(pr_context* c, pr_mesh* out) {
  out->vertices = nullptr;
  out->triangles = nullptr;
  out->n_vertices = c->nv;
  out->n_triangles = c->nt;
  const size_t vb = 3 * c->nv * sizeof(double), tb = 3 * c->nt * sizeof(uint64_t);
  const size_t total = vb + tb;
  if (total == 0) return;
  {  // pinned pool blocks: one DMA each, straight into the caller's arrays
    void* pv = vb ? pool_alloc(vb) : nullptr;
    void* pt = tb ? pool_alloc(tb) : nullptr;
    if ((!vb || pv) && (!tb || pt)) {
      if (vb) PR_CUDA(cudaMemcpyAsync(pv, c->get<double>("mesh_v"), vb, cudaMemcpyDeviceToHost, c->stream));
      if (tb) PR_CUDA(cudaMemcpyAsync(pt, c->get<uint64_t>("mesh_t"), tb, cudaMemcpyDeviceToHost, c->stream));
      const cudaError_t e = cudaStreamSynchronize(c->stream);
      if (e != cudaSuccess) {
        pool_release(pv);
        pool_release(pt);
        throw pr::Error(PR_ERR_CUDA, std::string("mesh copy to host failed: ") + cudaGetErrorString(e));
      }
      out->vertices = static_cast<double*>(pv);
      out->triangles = static_cast<uint64_t*>(pt);
      return;
    }
    pool_release(pv);
    pool_release(pt);
  }
  if (c->h_stage_cap < total) {
    if (c->h_stage) cudaFreeHost(c->h_stage);
    c->h_stage = nullptr;
    c->h_stage_cap = 0;
    const size_t cap = total + (total >> 3);
    PR_CUDA(cudaMallocHost(&c->h_stage, cap));
    c->h_stage_cap = cap;
  }
  const size_t CH = size_t(8) << 20;
  const size_t nch = (total + CH - 1) / CH;
  if (c->copy_events.size() < nch) {
    const size_t have = c->copy_events.size();
    c->copy_events.resize(nch, nullptr);
    for (size_t k = have; k < nch; ++k) PR_CUDA(cudaEventCreateWithFlags(&c->copy_events[k], cudaEventDisableTiming));
  }
  const unsigned char* dv = reinterpret_cast<const unsigned char*>(vb ? c->get<double>("mesh_v") : nullptr);
  const unsigned char* dt = reinterpret_cast<const unsigned char*>(tb ? c->get<uint64_t>("mesh_t") : nullptr);
  for (size_t k = 0; k < nch; ++k) {  // chunk k covers bytes [k CH, min(total, (k+1) CH)) of [vertices | triangles]
    size_t lo = k * CH;
    const size_t hi = std::min(total, lo + CH);
    while (lo < hi) {
      const bool in_v = lo < vb;
      const size_t end = in_v ? std::min(hi, vb) : hi;
      const unsigned char* src = in_v ? dv + lo : dt + (lo - vb);
      PR_CUDA(cudaMemcpyAsync(c->h_stage + lo, src, end - lo, cudaMemcpyDeviceToHost, c->stream));
      lo = end;
    }
    PR_CUDA(cudaEventRecord(c->copy_events[k], c->stream));
  }
  unsigned char* ov = static_cast<unsigned char*>(alloc_host_out(vb));
  unsigned char* ot = static_cast<unsigned char*>(alloc_host_out(tb));
  if ((vb && !ov) || (tb && !ot)) {
    std::free(ov);
    std::free(ot);
    c->sync();
    throw std::bad_alloc();
  }
  const unsigned nt = (unsigned)std::max<size_t>(1, std::min<size_t>({8, nch, std::thread::hardware_concurrency()}));
  std::atomic<int> failed{0};
  auto worker = [&](unsigned id) {
    for (size_t k = id; k < nch; k += nt) {
      if (cudaEventSynchronize(c->copy_events[k]) != cudaSuccess) {
        failed = 1;
        return;
      }
      size_t lo = k * CH;
      const size_t hi = std::min(total, lo + CH);
      while (lo < hi) {
        const bool in_v = lo < vb;
        const size_t end = in_v ? std::min(hi, vb) : hi;
        std::memcpy(in_v ? ov + lo : ot + (lo - vb), c->h_stage + lo, end - lo);
        lo = end;
      }
    }
  };
  std::vector<std::thread> th;
  for (unsigned i = 1; i < nt; ++i) th.emplace_back(worker, i);
  worker(0);
  for (auto& t : th) t.join();
  if (failed) {
    std::free(ov);
    std::free(ot);
    PR_CUDA(cudaStreamSynchronize(c->stream));
    throw pr::Error(PR_ERR_CUDA, "mesh copy to host failed");
  }
  out->vertices = reinterpret_cast<double*>(ov);
  out->triangles = reinterpret_cast<uint64_t*>(ot);
}

void pipeline_setup(pr_context* c, const pr_params& p, pr_stats& st, double t1);
void pipeline_extract(pr_context* c, const pr_params& p, uint64_t n, pr_stats& st, double t3);

void reset_state(pr_context* c) {
  c->have_state = false;
  c->have_mesh = false;
  c->have_coeffs = false;
  c->coeffs_converged = false;
  c->have_ref_coarse = false;
  c->adaptive = false;
  c->nv = c->nt = 0;
}

// The pipeline on device-resident points (c->buf "pts6" or caller memory).
void run_pipeline(pr_context* c, const double* d_pts6, uint64_t n, const pr_params& p, pr_stats& st, double t_start,
                  bool extract = true) {
  double t0 = now_s();
  pr::stage_transform(c, d_pts6, n, p.scale);
  c->sync();
  double t1 = now_s();
  st.time_transform = t1 - t0 + (t0 - t_start);
  c->degree = degree_of(p);
  c->params = p;
  if (p.coarse_depth > 0) {  // adaptive: coarse level, band setup, band solve, extraction
    pr::stage_adaptive(c, p, st, extract);
    st.time_system = 0.0;
    if (p.verbose)
      std::fprintf(stderr,
                   "pr: adaptive depth=%u coarse=%u points=%llu bricks=%llu xform=%.4f tree=%.4f solve=%.4f "
                   "extract=%.4f s; pcg=%u refine=%u relres=%.3e iso=%.6f verts=%llu tris=%llu\n",
                   p.depth, p.coarse_depth, (unsigned long long)n, (unsigned long long)c->band_nb, st.time_transform,
                   st.time_tree, st.time_solve, st.time_extract, st.pcg_iterations, st.refinement_steps,
                   st.rel_residual, st.iso_value, (unsigned long long)c->nv, (unsigned long long)c->nt);
    return;
  }
  pipeline_setup(c, p, st, t1);
  const double t2 = now_s();
  if (c->degree == 2) pr::stage_solve_deg2(c, p, st);
  else if (p.solve_mode == PR_SOLVE_REFERENCE_SCHEDULE) pr::stage_solve_reference(c, p, st);
  else pr::stage_solve(c, p, st);
  c->coeffs_converged = p.solve_mode != PR_SOLVE_REFERENCE_SCHEDULE;
  c->sync();
  double t3 = now_s();
  st.time_solve = t3 - t2;
  st.peak_device_bytes = (double)c->peak_bytes;
  if (!extract) return;
  pipeline_extract(c, p, n, st, t3);
}

// Tree, splat, right-hand side and screening payload of the dense grid (after the transform).
void pipeline_setup(pr_context* c, const pr_params& p, pr_stats& st, double t1) {
  if (c->degree == 2) pr::stage_setup_deg2(c, p.depth, p.point_weight);
  else pr::stage_splat_rhs(c, p.depth, p.point_weight);
  c->sync();
  const double t2 = now_s();
  st.time_tree = t2 - t1;  // tree (implicit) + splat + RHS + screening payload
  st.time_system = 0.0;
  st.fem_nodes = c->n;
  st.points_in_cube = c->P_in;
  c->params = p;
}

// Iso value and marching cubes of the solved dense grid (t3: end of the solve).
void pipeline_extract(pr_context* c, const pr_params& p, uint64_t n, pr_stats& st, double t3) {
  const bool nat = c->degree == 2;  // degree 2: straight from the solver's natural order
  const double* x = nat ? c->d2_xnat : c->get<double>("x64");
  double iso = pr::stage_iso(c, x, nat);
  pr::stage_extract(c, c->D, x, iso, true, c->degree, nat);
  c->sync();
  double t4 = now_s();
  st.time_extract = t4 - t3;
  st.iso_value = iso;
  st.mesh_vertices = c->nv;
  st.mesh_triangles = c->nt;
  st.peak_device_bytes = (double)c->peak_bytes;
  if (p.verbose)
    std::fprintf(stderr,
                 "pr: depth=%u degree=%d points=%llu xform=%.4f tree=%.4f solve=%.4f extract=%.4f s; pcg=%u "
                 "refine=%u relres=%.3e iso=%.6f verts=%llu tris=%llu\n",
                 p.depth, c->degree, (unsigned long long)n, st.time_transform, st.time_tree, st.time_solve, st.time_extract,
                 st.pcg_iterations, st.refinement_steps, st.rel_residual, iso, (unsigned long long)c->nv,
                 (unsigned long long)c->nt);
}

void reconstruct_impl(pr_context* c, const double* points6, uint64_t n, const pr_params* params, bool device_input,
                      pr_mesh* out_mesh, pr_stats* out_stats, bool extract = true) {
  double t_start = now_s();
  validate(params);
  PR_REQUIRE(n == 0 || points6 != nullptr, PR_ERR_INVALID_ARGUMENT, "points is NULL");
  PR_REQUIRE(n <= pr::kMaxPoints, PR_ERR_INVALID_ARGUMENT, "at most 2^28 points per call");
  set_device(c);
  pr_stats st;
  std::memset(&st, 0, sizeof(st));
  reset_state(c);
  if (out_mesh) std::memset(out_mesh, 0, sizeof(*out_mesh));
  if (n == 0) {  // src/reconstructor.rs:28
    c->have_mesh = true;
    if (out_stats) *out_stats = st;
    return;
  }
  const double* d_pts = points6;
  if (!device_input) {
    double* dp = c->buf<double>("pts6", 6 * n);
    PR_CUDA(cudaMemcpyAsync(dp, points6, 6 * n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    d_pts = dp;
  }
  run_pipeline(c, d_pts, n, *params, st, t_start, extract);
  if (out_mesh && extract) {
    const double t_copy = now_s();
    copy_mesh_to_host(c, out_mesh);
    st.time_mesh_copy = now_s() - t_copy;
  }
  st.time_total = now_s() - t_start;
  if (out_stats) *out_stats = st;
}

thread_local std::unique_ptr<pr_context, int (*)(pr_context*)> g_thread_ctx(nullptr, pr_context_destroy);

// ------------------------------------------------------------------ packed batches
// Clouds of a batch that share the solver's parameters and a dense degree-1 grid of depth >= 5
// (converged solve) are reconstructed in packs: each cloud is set up in a context of its own (host
// threads, one stream each), the pack's systems are solved together (pr::solve_packed: one launch
// per solver step for every cloud of the pack) and each cloud is extracted and copied out in its
// context.  A pack takes as many clouds of one depth as the free device memory holds.  The
// contexts are kept for later batches (one engine per device); their memory is given back when an
// allocation elsewhere in the process fails (pr::release_cached_memory).
thread_local bool t_in_batch = false;

struct BatchEngine {
  std::mutex mu;
  int device = 0;
  pr_context* solver = nullptr;
  std::vector<pr_context*> cl;
  pr_context* make() {
    pr_context* c = nullptr;
    const int rc = pr_context_create(device, nullptr, &c);
    if (rc != PR_OK) throw pr::Error(rc, g_last_error);
    return c;
  }
  void ensure(size_t k) {
    if (!solver) solver = make();
    while (cl.size() < k) cl.push_back(make());
  }
  size_t held() const {
    size_t b = solver ? solver->bytes_held : 0;
    for (const pr_context* c : cl) b += c->bytes_held;
    return b;
  }
  // frees every buffer (and graph) of the contexts, keeping the contexts
  void free_buffers() {
    auto drop = [](pr_context* c) {
      PR_CUDA(cudaStreamSynchronize(c->stream));
      for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second.exec);
      c->graphs.clear();
      for (auto& kv : c->bufs)
        if (kv.second.ptr) cudaFree(kv.second.ptr);
      c->bufs.clear();
      c->free_spare();
      c->bytes_held = 0;
    };
    if (solver) drop(solver);
    for (pr_context* c : cl) drop(c);
  }
  void release() {
    if (solver) pr_context_destroy(solver);
    solver = nullptr;
    for (pr_context* c : cl) pr_context_destroy(c);
    cl.clear();
  }
};
BatchEngine& batch_engine(int device) {
  static std::mutex m;
  static std::map<int, BatchEngine*>* engines = new std::map<int, BatchEngine*>();  // never destroyed
  std::lock_guard<std::mutex> g(m);
  BatchEngine*& e = (*engines)[device];
  if (!e) {
    e = new BatchEngine();
    e->device = device;
  }
  return *e;
}

struct PackKey {
  uint32_t depth, precision, max_iters, smooth_sweeps;
  double pw, target, inner;
  bool operator<(const PackKey& o) const {
    return std::tie(depth, precision, max_iters, smooth_sweeps, pw, target, inner) <
           std::tie(o.depth, o.precision, o.max_iters, o.smooth_sweeps, o.pw, o.target, o.inner);
  }
};
PackKey pack_key(const pr_params& p) {
  return PackKey{p.depth, (uint32_t)p.precision, p.max_iters, p.smooth_sweeps, p.point_weight, p.target_rel_residual,
                 p.inner_rel_tol};
}
bool packable(const pr_params& p, const double* pts, uint64_t n) {
  try {
    validate(&p);
  } catch (const pr::Error&) {
    return false;  // reported by the single-cloud path
  }
  return pts != nullptr && n > 0 && n <= pr::kMaxPoints && degree_of(p) == 1 && p.coarse_depth == 0 &&
         p.solve_mode == PR_SOLVE_CONVERGED && p.depth >= 5;
}
// device bytes of one cloud of a pack: its context (input, setup, solution, extraction) and its
// share of the packed solve's vectors
double pack_ctx_bytes(const pr_params& p, uint64_t P) {
  const double nodes = std::ldexp(1.0, 3 * (int)p.depth), res2 = std::ldexp(1.0, 2 * (int)p.depth);
  return 20.0 * nodes + 800.0 * (double)P + 1000.0 * res2 + 64e6;
}
double pack_solver_bytes(const pr_params& p) {
  return (p.precision == PR_PRECISION_FP64 ? 96.0 : 64.0) * std::ldexp(1.0, 3 * (int)p.depth);
}

template <typename F>
void parallel_for(size_t m, unsigned max_threads, F f) {
  std::atomic<size_t> next{0};
  auto w = [&] {
    t_in_batch = true;
    for (;;) {
      const size_t j = next.fetch_add(1);
      if (j >= m) return;
      f(j);
    }
  };
  const unsigned nt = (unsigned)std::max<size_t>(1, std::min<size_t>(m, max_threads));
  std::vector<std::thread> th;
  for (unsigned t = 1; t < nt; ++t) th.emplace_back(w);
  w();
  for (auto& t : th) t.join();
}

void run_pack(BatchEngine& E, const std::vector<uint32_t>& pk, const double* const* points6, const uint64_t* n,
              const pr_params* params, pr_mesh* out_meshes, pr_stats* out_stats, std::vector<int>& status,
              std::vector<std::string>& msgs) {
  const size_t m = pk.size();
  const double tp0 = now_s();
  E.ensure(m);
  std::vector<pr_stats> st(m);
  std::vector<char> ok(m, 1);
  const unsigned hw = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
  parallel_for(m, hw, [&](size_t j) {  // input, transform, tree, splat, right-hand side
    const uint32_t i = pk[j];
    pr_context* c = E.cl[j];
    const int r = guard([&] {
      const double ts = now_s();
      set_device(c);
      std::memset(&st[j], 0, sizeof(pr_stats));
      reset_state(c);
      double* dp = c->buf<double>("pts6", 6 * n[i]);
      PR_CUDA(cudaMemcpyAsync(dp, points6[i], 6 * n[i] * sizeof(double), cudaMemcpyHostToDevice, c->stream));
      pr::stage_transform(c, dp, n[i], params[i].scale);
      c->sync();
      const double t1 = now_s();
      st[j].time_transform = t1 - ts;
      c->degree = 1;
      c->params = params[i];
      pipeline_setup(c, params[i], st[j], t1);
    });
    if (r != PR_OK) {
      status[i] = r;
      msgs[i] = g_last_error;
      ok[j] = 0;
    }
  });
  const double tp1 = now_s();
  std::vector<pr_context*> sc;
  std::vector<size_t> idx;
  for (size_t j = 0; j < m; ++j)
    if (ok[j]) {
      sc.push_back(E.cl[j]);
      idx.push_back(j);
    }
  if (!sc.empty()) {  // the packed solve
    std::vector<pr_stats> sst(sc.size());
    for (size_t k = 0; k < sc.size(); ++k) sst[k] = st[idx[k]];
    const double ts = now_s();
    const int r = guard([&] {
      set_device(E.solver);
      pr::solve_packed(E.solver, sc, params[pk[idx[0]]], sst);
    });
    const double share = (now_s() - ts) / (double)sc.size();
    for (size_t k = 0; k < sc.size(); ++k) {
      const size_t j = idx[k];
      if (r != PR_OK) {
        status[pk[j]] = r;
        msgs[pk[j]] = g_last_error;
        ok[j] = 0;
        continue;
      }
      st[j] = sst[k];
      st[j].time_solve = share;  // the cloud's share of the packed solve
      sc[k]->coeffs_converged = true;
    }
  }
  const double tp2 = now_s();
  parallel_for(m, hw, [&](size_t j) {  // iso value, marching cubes, mesh to host
    if (!ok[j]) return;
    const uint32_t i = pk[j];
    pr_context* c = E.cl[j];
    const int r = guard([&] {
      set_device(c);
      pipeline_extract(c, params[i], n[i], st[j], now_s());
      const double tc = now_s();
      copy_mesh_to_host(c, &out_meshes[i]);
      st[j].time_mesh_copy = now_s() - tc;
      c->have_mesh = true;
      st[j].peak_device_bytes = (double)c->peak_bytes + (double)E.solver->peak_bytes / (double)m;
      st[j].time_total = st[j].time_transform + st[j].time_tree + st[j].time_solve + st[j].time_extract +
                         st[j].time_mesh_copy;
    });
    if (r != PR_OK) {
      status[i] = r;
      msgs[i] = g_last_error;
    } else if (out_stats) {
      out_stats[i] = st[j];
    }
  });
  const char* vb = std::getenv("PR_BATCH_VERBOSE");
  if (vb && std::atoi(vb) != 0)
    std::fprintf(stderr, "pr: pack of %zu: setup %.4f s, solve %.4f s, extract + copy %.4f s\n", m, tp1 - tp0,
                 tp2 - tp1, now_s() - tp2);
}

void run_packed(int device, const std::map<PackKey, std::vector<uint32_t>>& groups, const double* const* points6,
                const uint64_t* n, const pr_params* params, pr_mesh* out_meshes, pr_stats* out_stats,
                std::vector<int>& status, std::vector<std::string>& msgs) {
  BatchEngine& E = batch_engine(device);
  std::lock_guard<std::mutex> g(E.mu);
  struct Flag {
    Flag() { t_in_batch = true; }
    ~Flag() { t_in_batch = false; }
  } flag;
  std::vector<std::vector<uint32_t>> order;
  for (const auto& kv : groups) order.push_back(kv.second);
  // deepest first: later packs reuse the buffers of earlier ones
  std::stable_sort(order.begin(), order.end(), [&](const std::vector<uint32_t>& a, const std::vector<uint32_t>& b) {
    return params[a[0]].depth > params[b[0]].depth;
  });
  const char* lim = std::getenv("PR_PACK_MAX_CLOUDS");  // cap on the clouds of one pack (0: none)
  const size_t max_clouds = lim ? (size_t)std::strtoull(lim, nullptr, 10) : 0;
  const char* vb = std::getenv("PR_BATCH_VERBOSE");
  const bool verbose = vb && std::atoi(vb) != 0;
  // Packs are sized against a fixed share of the device (PR_PACK_MEMORY_FRACTION, default 0.65)
  // rather than against the free memory of the moment, so that every batch of the same clouds forms
  // the same packs and reuses the buffers of the last one: the solver's vectors for the largest
  // pack, and per context the largest cloud it served.  A group is split into packs of even size.
  size_t free_b = 0, total_b = 0;
  PR_CUDA(cudaSetDevice(device));
  PR_CUDA(cudaMemGetInfo(&free_b, &total_b));
  const char* fr = std::getenv("PR_PACK_MEMORY_FRACTION");
  const double frac = fr ? std::min(0.9, std::max(0.05, std::atof(fr))) : 0.65;
  const double cap = frac * (double)total_b;
  for (std::vector<uint32_t> grp : order) {
    std::stable_sort(grp.begin(), grp.end(), [&](uint32_t a, uint32_t b) { return n[a] > n[b]; });
    double sum = 0.0;
    for (uint32_t i : grp) sum += pack_ctx_bytes(params[i], n[i]) + pack_solver_bytes(params[i]);
    size_t packs = (size_t)std::max(1.0, std::ceil(sum / cap));
    if (max_clouds) packs = std::max(packs, (grp.size() + max_clouds - 1) / max_clouds);
    size_t pos = 0;
    for (size_t k = 0; k < packs && pos < grp.size(); ++k) {
      // even split by estimated bytes (the clouds are largest first): the remaining bytes over the
      // remaining packs, at least one cloud
      double rest = 0.0;
      for (size_t j = pos; j < grp.size(); ++j) rest += pack_ctx_bytes(params[grp[j]], n[grp[j]]) + pack_solver_bytes(params[grp[j]]);
      const double share = rest / (double)(packs - k);
      std::vector<uint32_t> pk;
      double acc = 0.0;
      while (pos < grp.size()) {
        const uint32_t i = grp[pos];
        const double b = pack_ctx_bytes(params[i], n[i]) + pack_solver_bytes(params[i]);
        if (!pk.empty() && (acc + 0.5 * b > share || (max_clouds && pk.size() >= max_clouds))) break;
        pk.push_back(i);
        acc += b;
        ++pos;
      }
      if (k + 1 == packs)
        while (pos < grp.size()) pk.push_back(grp[pos++]);  // (rounding) the last pack takes the rest
      const double t0 = now_s();
      run_pack(E, pk, points6, n, params, out_meshes, out_stats, status, msgs);
      bool oom = false;
      for (uint32_t i : pk) oom = oom || status[i] == PR_ERR_OUT_OF_MEMORY;
      if (oom && E.held() > 0) {  // other users took the memory: free the held buffers, try again once
        for (uint32_t i : pk) {
          pr_mesh_free(&out_meshes[i]);
          status[i] = PR_OK;
          msgs[i].clear();
        }
        E.free_buffers();
        run_pack(E, pk, points6, n, params, out_meshes, out_stats, status, msgs);
      }
      if (verbose)
        std::fprintf(stderr, "pr: pack depth=%u clouds=%zu est=%.2f GB held=%.2f GB %.4f s\n", params[pk[0]].depth,
                     pk.size(), acc / 1e9, (double)E.held() / 1e9, now_s() - t0);
    }
  }
}

}  // namespace

namespace pr {
std::mutex& spare_mutex() {
  static std::mutex* m = new std::mutex();  // never destroyed
  return *m;
}
std::set<pr_context*>& context_registry() {  // every live context; guarded by spare_mutex
  static std::set<pr_context*>* r = new std::set<pr_context*>();
  return *r;
}
void free_all_spare(int device) {
  std::lock_guard<std::mutex> g(spare_mutex());
  for (pr_context* c : context_registry())
    if (c->device == device) c->free_spare_locked();
}
bool release_cached_memory(int device) {
  if (t_in_batch) return false;
  BatchEngine& e = batch_engine(device);
  std::unique_lock<std::mutex> g(e.mu, std::try_to_lock);
  if (!g.owns_lock() || e.held() == 0) return false;
  e.release();
  cudaSetDevice(device);
  return true;
}
}  // namespace pr

namespace {


}  // namespace

namespace pr {
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace pr

static std::atomic<uint64_t> g_launches{0}, g_primitives{0};
static thread_local uint64_t t_counts[2] = {0, 0};
namespace pr {
uint64_t thread_launch_count(int primitive) { return t_counts[primitive ? 1 : 0]; }
}  // namespace pr

extern "C" {

void pr_count_launch_(int primitive) {
  ++t_counts[primitive ? 1 : 0];
  if (primitive) g_primitives.fetch_add(1, std::memory_order_relaxed);
  else g_launches.fetch_add(1, std::memory_order_relaxed);
}

uint64_t pr_kernel_launches(uint64_t* primitive_calls) {
  if (primitive_calls) *primitive_calls = g_primitives.load();
  return g_launches.load();
}

int pr_ctx_apply_operator_device(pr_context* c, const void* d_x, void* d_y, int precision) {
  return guard([&] {
    PR_REQUIRE(c != nullptr && d_x != nullptr && d_y != nullptr, PR_ERR_INVALID_ARGUMENT, "NULL argument");
    PR_REQUIRE(c->have_state, PR_ERR_STATE, "no reconstruction state");
    PR_REQUIRE(!c->adaptive, PR_ERR_STATE, "the last reconstruction was adaptive: read it with the band accessors");
    set_device(c);
    if (c->degree == 2) {
      if (precision == PR_PRECISION_FP64) pr::deg2_apply_morton<double>(c, (const double*)d_x, (double*)d_y);
      else pr::deg2_apply_morton<float>(c, (const float*)d_x, (float*)d_y);
    } else if (precision == PR_PRECISION_FP64) {
      pr::apply_operator64(c, (const double*)d_x, (double*)d_y);
    } else {
      pr::apply_operator32(c, (const float*)d_x, (float*)d_y);
    }
  });
}

int pr_ctx_kernel_bench(pr_context* c, int kernel, uint32_t depth, int precision, int reps, double* ms,
                        double* bytes) {
  return guard([&] {
    PR_REQUIRE(c != nullptr && ms != nullptr && bytes != nullptr, PR_ERR_INVALID_ARGUMENT, "NULL argument");
    set_device(c);
    *ms = pr::kernel_bench(c, kernel, depth, precision, reps, bytes);
  });
}

const char* pr_version(void) { return "poisson_recon_b200 0.1 (sm_100a)"; }

const char* pr_autotune_log(void) {
  static thread_local std::string text;
  text = pr::autotune_log();
  return text.c_str();
}

void pr_abi_layout(uint64_t* out4) {
  if (!out4) return;
  out4[0] = sizeof(pr_params);
  out4[1] = sizeof(pr_mesh);
  out4[2] = sizeof(pr_stats);
  out4[3] = sizeof(pr_oriented_point);
}

const char* pr_last_error(void) { return g_last_error.c_str(); }

pr_params pr_params_default(void) {
  pr_params p;
  std::memset(&p, 0, sizeof(p));
  // ReconstructParams::default() (src/reconstructor.rs:14)
  p.depth = 8;
  p.samples_per_node = 1.5;
  p.scale = 1.1;
  p.cg_accuracy = 1e-3;
  p.cg_iters = 500;
  p.point_weight = 0.0;
  p.verbose = 0;
  p.solve_mode = PR_SOLVE_CONVERGED;
  p.precision = PR_PRECISION_MIXED;
  p.target_rel_residual = 1e-6;
  p.degree = 1;
  p.max_iters = 200;
  p.smooth_sweeps = 1;
  p.inner_rel_tol = 1e-4;
  return p;
}

int pr_context_create(int device, void* stream, pr_context** out_ctx) {
  return guard([&] {
    PR_REQUIRE(out_ctx != nullptr, PR_ERR_INVALID_ARGUMENT, "out_ctx is NULL");
    *out_ctx = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
      cudaGetLastError();
      throw pr::Error(PR_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
    }
    PR_REQUIRE(device >= 0 && device < count, PR_ERR_INVALID_ARGUMENT, "device index out of range");
    cudaDeviceProp prop;
    PR_CUDA(cudaGetDeviceProperties(&prop, device));
    PR_REQUIRE(prop.major == 10, PR_ERR_NO_DEVICE,
               std::string("library is built for sm_100a; device is ") + prop.name + " (sm_" +
                   std::to_string(prop.major) + std::to_string(prop.minor) + ")");
    PR_CUDA(cudaSetDevice(device));
    std::unique_ptr<pr_context> c(new pr_context());
    c->device = device;
    if (stream) {
      c->stream = (cudaStream_t)stream;
      c->own_stream = false;
    } else {
      PR_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
      c->own_stream = true;
    }
    PR_CUDA(cudaMallocHost(&c->h_scalars, 64 * sizeof(double)));
    {
      std::lock_guard<std::mutex> g(pr::spare_mutex());
      pr::context_registry().insert(c.get());
    }
    *out_ctx = c.release();
  });
}

int pr_context_destroy(pr_context* c) {
  if (!c) return PR_OK;
  return guard([&] {
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    for (auto& kv : c->bufs)
      if (kv.second.ptr) cudaFree(kv.second.ptr);
    c->bufs.clear();
    {
      std::lock_guard<std::mutex> g(pr::spare_mutex());
      c->free_spare_locked();
      pr::context_registry().erase(c);
    }
    for (cudaEvent_t e : c->copy_events)
      if (e) cudaEventDestroy(e);
    c->copy_events.clear();
    for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second.exec);
    c->graphs.clear();
    if (c->side) {
      cudaStreamSynchronize(c->side);
      cudaStreamDestroy(c->side);
      cudaEventDestroy(c->ev_fork);
      cudaEventDestroy(c->ev_join);
    }
    if (c->h_scalars) cudaFreeHost(c->h_scalars);
    if (c->h_pack) cudaFreeHost(c->h_pack);
    if (c->h_stage) cudaFreeHost(c->h_stage);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
  });
}

int pr_ctx_reconstruct(pr_context* c, const double* points6, uint64_t n, const pr_params* params, pr_mesh* out_mesh,
                       pr_stats* out_stats) {
  return guard([&] {
    PR_REQUIRE(c != nullptr, PR_ERR_INVALID_ARGUMENT, "context is NULL");
    PR_REQUIRE(out_mesh != nullptr, PR_ERR_INVALID_ARGUMENT, "out_mesh is NULL");
    reconstruct_impl(c, points6, n, params, false, out_mesh, out_stats);
  });
}

int pr_ctx_reconstruct_device(pr_context* c, const double* d_points6, uint64_t n, const pr_params* params,
                              pr_stats* out_stats) {
  return guard([&] {
    PR_REQUIRE(c != nullptr, PR_ERR_INVALID_ARGUMENT, "context is NULL");
    reconstruct_impl(c, d_points6, n, params, true, nullptr, out_stats);
  });
}

int pr_reconstruct(const double* points6, uint64_t n, const pr_params* params, pr_mesh* out_mesh,
                   pr_stats* out_stats) {
  return guard([&] {
    PR_REQUIRE(out_mesh != nullptr, PR_ERR_INVALID_ARGUMENT, "out_mesh is NULL");
    validate(params);
    PR_REQUIRE(n == 0 || points6 != nullptr, PR_ERR_INVALID_ARGUMENT, "points is NULL");
    PR_REQUIRE(n <= pr::kMaxPoints, PR_ERR_INVALID_ARGUMENT, "at most 2^28 points per call");
    if (n == 0) {  // src/reconstructor.rs:28: empty mesh, default stats; no device needed
      std::memset(out_mesh, 0, sizeof(*out_mesh));
      if (out_stats) std::memset(out_stats, 0, sizeof(*out_stats));
      return;
    }
    if (!g_thread_ctx) {
      pr_context* c = nullptr;
      int rc = pr_context_create(0, nullptr, &c);
      if (rc != PR_OK) throw pr::Error(rc, g_last_error);
      g_thread_ctx.reset(c);
    }
    reconstruct_impl(g_thread_ctx.get(), points6, n, params, false, out_mesh, out_stats);
  });
}

int pr_ctx_solve(pr_context* c, const double* points6, uint64_t n, const pr_params* params, pr_stats* out_stats) {
  return guard([&] {
    PR_REQUIRE(c != nullptr, PR_ERR_INVALID_ARGUMENT, "context is NULL");
    reconstruct_impl(c, points6, n, params, false, nullptr, out_stats, false);
  });
}

static void loss_backward_impl(pr_context* c, const double* queries3, uint64_t k, const double* dl_dchi, double* chi,
                               double* dl_dpositions, double* dl_dnormals, pr_adjoint_stats* out_stats) {
  const double t_start = now_s();
  PR_REQUIRE(queries3 != nullptr, PR_ERR_INVALID_ARGUMENT, "queries is NULL");
  PR_REQUIRE(k >= 1 && k <= pr::kMaxPoints, PR_ERR_INVALID_ARGUMENT, "k must be in [1, 2^28] query points");
  PR_REQUIRE(c->have_state && c->have_coeffs, PR_ERR_STATE, "no solved reconstruction on this context");
  PR_REQUIRE(c->coeffs_converged, PR_ERR_STATE,
             "the last solve used the reference schedule; the adjoint needs solve_mode PR_SOLVE_CONVERGED");
  for (uint64_t i = 0; i < 3 * k; ++i)
    PR_REQUIRE(std::isfinite(queries3[i]), PR_ERR_INVALID_ARGUMENT, "non-finite query coordinate");
  set_device(c);
  pr_adjoint_stats st;
  std::memset(&st, 0, sizeof(st));
  double* dq = c->buf<double>("adj_q3", 3 * k);
  PR_CUDA(cudaMemcpyAsync(dq, queries3, 3 * k * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  double* ddl = nullptr;
  if (dl_dchi) {
    ddl = c->buf<double>("adj_dl", k);
    PR_CUDA(cudaMemcpyAsync(ddl, dl_dchi, k * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  }
  double* dchi = c->buf<double>("adj_chi", k);
  double* dpos = c->buf<double>("adj_dpos", 3 * c->P);
  double* dnrm = c->buf<double>("adj_dnrm", 3 * c->P);
  if (c->adaptive) pr::adjoint_backward_band(c, dq, k, ddl, dchi, dpos, dnrm, st);
  else if (c->degree == 2) pr::adjoint_backward2(c, dq, k, ddl, dchi, dpos, dnrm, st);
  else pr::adjoint_backward(c, dq, k, ddl, dchi, dpos, dnrm, st);
  if (chi) PR_CUDA(cudaMemcpyAsync(chi, dchi, k * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (dl_dpositions)
    PR_CUDA(cudaMemcpyAsync(dl_dpositions, dpos, 3 * c->P * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (dl_dnormals)
    PR_CUDA(cudaMemcpyAsync(dl_dnormals, dnrm, 3 * c->P * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  c->sync();
  st.time_total = now_s() - t_start;
  if (out_stats) *out_stats = st;
  if (!st.converged)
    throw pr::Error(PR_ERR_NOT_CONVERGED, "adjoint solve stopped at relative residual " +
                                              std::to_string(st.rel_residual) + " (outputs hold the last iterate)");
}

int pr_ctx_loss_backward(pr_context* c, const double* queries3, uint64_t k, const double* dl_dchi, double* chi,
                         double* dl_dpositions, double* dl_dnormals, pr_adjoint_stats* out_stats) {
  return guard([&] {
    PR_REQUIRE(c != nullptr, PR_ERR_INVALID_ARGUMENT, "context is NULL");
    loss_backward_impl(c, queries3, k, dl_dchi, chi, dl_dpositions, dl_dnormals, out_stats);
  });
}

int pr_loss_backward(const double* points6, uint64_t n, const pr_params* params, const double* queries3, uint64_t k,
                     const double* dl_dchi, double* chi, double* dl_dpositions, double* dl_dnormals,
                     pr_adjoint_stats* out_stats) {
  return guard([&] {
    validate(params);
    PR_REQUIRE(n >= 1 && points6 != nullptr, PR_ERR_INVALID_ARGUMENT, "the adjoint needs at least one point");
    PR_REQUIRE(params->solve_mode == PR_SOLVE_CONVERGED, PR_ERR_INVALID_ARGUMENT,
               "the adjoint needs solve_mode PR_SOLVE_CONVERGED");
    if (!g_thread_ctx) {
      pr_context* c = nullptr;
      int rc = pr_context_create(0, nullptr, &c);
      if (rc != PR_OK) throw pr::Error(rc, g_last_error);
      g_thread_ctx.reset(c);
    }
    pr_context* c = g_thread_ctx.get();
    reconstruct_impl(c, points6, n, params, false, nullptr, nullptr, false);
    loss_backward_impl(c, queries3, k, dl_dchi, chi, dl_dpositions, dl_dnormals, out_stats);
  });
}

int pr_ctx_reconstruct_batch(pr_context* const* ctxs, uint32_t n_ctx, const double* const* points6, const uint64_t* n,
                             uint32_t count, const pr_params* params, pr_mesh* out_meshes, pr_stats* out_stats,
                             int* out_status) {
  std::vector<std::string> msgs;
  std::vector<int> status;
  const int rc = guard([&] {
    PR_REQUIRE(count == 0 || (ctxs && n_ctx > 0 && points6 && n && params && out_meshes), PR_ERR_INVALID_ARGUMENT,
               "NULL argument");
    for (uint32_t i = 0; i < n_ctx && count > 0; ++i) PR_REQUIRE(ctxs[i] != nullptr, PR_ERR_INVALID_ARGUMENT, "NULL context");
    for (uint32_t i = 0; i < count; ++i) std::memset(&out_meshes[i], 0, sizeof(pr_mesh));
    if (count == 0) return;
    status.assign(count, PR_OK);
    msgs.assign(count, std::string());
    // packs of clouds that share the solver's parameters; the others one per context
    std::map<PackKey, std::vector<uint32_t>> groups;
    std::vector<uint32_t> rest;
    for (uint32_t i = 0; i < count; ++i) {
      if (packable(params[i], points6[i], n[i])) groups[pack_key(params[i])].push_back(i);
      else rest.push_back(i);
    }
    if (!groups.empty())
      run_packed(ctxs[0]->device, groups, points6, n, params, out_meshes, out_stats, status, msgs);
    // largest clouds first, one host thread per context pulling the next cloud
    std::stable_sort(rest.begin(), rest.end(), [&](uint32_t a, uint32_t b) { return n[a] > n[b]; });
    std::atomic<uint32_t> next{0};
    auto worker = [&](uint32_t w) {
      for (;;) {
        const uint32_t k = next.fetch_add(1);
        if (k >= rest.size()) return;
        const uint32_t i = rest[k];
        pr_stats st;
        const int r = pr_ctx_reconstruct(ctxs[w], points6[i], n[i], &params[i], &out_meshes[i], &st);
        status[i] = r;
        if (r != PR_OK) msgs[i] = g_last_error;
        else if (out_stats) out_stats[i] = st;
      }
    };
    const uint32_t nw = std::min<uint32_t>(n_ctx, (uint32_t)rest.size());
    std::vector<std::thread> th;
    for (uint32_t w = 1; w < nw; ++w) th.emplace_back(worker, w);
    if (nw > 0) worker(0);
    for (auto& t : th) t.join();
  });
  if (out_status)
    for (uint32_t i = 0; i < count; ++i) out_status[i] = i < status.size() ? status[i] : rc;
  if (rc != PR_OK) return rc;
  for (uint32_t i = 0; i < status.size(); ++i)
    if (status[i] != PR_OK) {
      g_last_error = "cloud " + std::to_string(i) + ": " + msgs[i];
      return status[i];
    }
  return PR_OK;
}

int pr_reconstruct_batch(const double* const* points6, const uint64_t* n, uint32_t count, const pr_params* params,
                         uint32_t concurrency, pr_mesh* out_meshes, pr_stats* out_stats, int* out_status) {
  static std::mutex mu;
  static std::vector<pr_context*> pool;  // device 0, kept for later calls
  std::lock_guard<std::mutex> g(mu);
  const uint32_t want = concurrency ? std::min<uint32_t>(concurrency, 64) : 4;
  while (pool.size() < want) {
    pr_context* c = nullptr;
    const int rc = pr_context_create(0, nullptr, &c);
    if (rc != PR_OK) return rc;
    pool.push_back(c);
  }
  return pr_ctx_reconstruct_batch(pool.data(), want, points6, n, count, params, out_meshes, out_stats, out_status);
}

void pr_host_free(void* p) {
  if (!pool_release(p)) std::free(p);
}

void pr_mesh_free(pr_mesh* m) {
  if (!m) return;
  pr_host_free(m->vertices);
  pr_host_free(m->triangles);
  m->vertices = nullptr;
  m->triangles = nullptr;
  m->n_vertices = m->n_triangles = 0;
}

int pr_ctx_mesh_device(pr_context* c, const double** dv, uint64_t* nv, const uint64_t** dt, uint64_t* nt) {
  return guard([&] {
    PR_REQUIRE(c != nullptr, PR_ERR_INVALID_ARGUMENT, "context is NULL");
    PR_REQUIRE(c->have_mesh, PR_ERR_STATE, "no mesh: run a reconstruction first");
    if (dv) *dv = c->nv ? c->get<double>("mesh_v") : nullptr;
    if (nv) *nv = c->nv;
    if (dt) *dt = c->nt ? c->get<uint64_t>("mesh_t") : nullptr;
    if (nt) *nt = c->nt;
  });
}

int pr_ctx_mesh_copy(pr_context* c, pr_mesh* out) {
  return guard([&] {
    PR_REQUIRE(c != nullptr && out != nullptr, PR_ERR_INVALID_ARGUMENT, "NULL argument");
    PR_REQUIRE(c->have_mesh, PR_ERR_STATE, "no mesh: run a reconstruction first");
    set_device(c);
    copy_mesh_to_host(c, out);
  });
}

int pr_ctx_synchronize(pr_context* c) {
  return guard([&] {
    PR_REQUIRE(c != nullptr, PR_ERR_INVALID_ARGUMENT, "context is NULL");
    set_device(c);
    c->sync();
  });
}

int pr_ctx_info(pr_context* c, uint32_t* depth, uint64_t* fem_nodes, double* m16) {
  return guard([&] {
    PR_REQUIRE(c != nullptr, PR_ERR_INVALID_ARGUMENT, "context is NULL");
    PR_REQUIRE(c->have_state, PR_ERR_STATE, "no reconstruction state");
    if (depth) *depth = c->D;
    if (fem_nodes) *fem_nodes = c->n;
    if (m16) std::memcpy(m16, c->M, sizeof(c->M));
  });
}

static void copy_dev_to_host(pr_context* c, const char* name, double* out, uint64_t count) {
  PR_REQUIRE(out != nullptr, PR_ERR_INVALID_ARGUMENT, "output is NULL");
  set_device(c);
  PR_CUDA(cudaMemcpyAsync(out, c->get<double>(name), count * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  c->sync();
}

int pr_ctx_get_coefficients(pr_context* c, double* out) {
  return guard([&] {
    PR_REQUIRE(c != nullptr, PR_ERR_INVALID_ARGUMENT, "context is NULL");
    PR_REQUIRE(c->have_coeffs, PR_ERR_STATE, "no solved coefficients");
    PR_REQUIRE(!c->adaptive, PR_ERR_STATE, "the last reconstruction was adaptive: read it with the band accessors");
    pr::coeffs_morton(c);
    copy_dev_to_host(c, "x64", out, c->n);
  });
}

int pr_ctx_get_rhs(pr_context* c, double* out) {
  return guard([&] {
    PR_REQUIRE(c != nullptr, PR_ERR_INVALID_ARGUMENT, "context is NULL");
    PR_REQUIRE(c->have_state, PR_ERR_STATE, "no reconstruction state");
    PR_REQUIRE(!c->adaptive, PR_ERR_STATE, "the last reconstruction was adaptive: read it with the band accessors");
    if (c->degree == 2) {
      PR_REQUIRE(out != nullptr, PR_ERR_INVALID_ARGUMENT, "output is NULL");
      set_device(c);
      pr::deg2_rhs_morton(c, c->buf<double>("acc_b", c->n));
      copy_dev_to_host(c, "acc_b", out, c->n);
      c->release("acc_b");
      return;
    }
    copy_dev_to_host(c, "b64", out, c->n);
  });
}

int pr_ctx_get_coarse_rhs(pr_context* c, uint32_t* coarse_depth, double* out) {
  return guard([&] {
    PR_REQUIRE(c != nullptr && coarse_depth != nullptr, PR_ERR_INVALID_ARGUMENT, "NULL argument");
    PR_REQUIRE(c->have_ref_coarse, PR_ERR_STATE, "the last reconstruction did not run the reference schedule");
    *coarse_depth = c->ref_coarse_D;
    if (out) copy_dev_to_host(c, "ref_brhs", out, 1ull << (3 * c->ref_coarse_D));
  });
}

int pr_ctx_cg_reference(pr_context* c, const double* x0, uint64_t max_iters, double accuracy, double* x,
                        double* delta, uint64_t* out_iters) {
  return guard([&] {
    PR_REQUIRE(c != nullptr && x != nullptr, PR_ERR_INVALID_ARGUMENT, "NULL argument");
    PR_REQUIRE(c->have_state, PR_ERR_STATE, "no reconstruction state");
    PR_REQUIRE(!c->adaptive, PR_ERR_STATE, "the last reconstruction was adaptive: read it with the band accessors");
    PR_REQUIRE(c->degree == 1, PR_ERR_INVALID_ARGUMENT, "the crate's CG runs on the degree-1 system only");
    set_device(c);
    const uint64_t n = c->n;
    double* dx = c->buf<double>("acc_x", n);
    if (x0) PR_CUDA(cudaMemcpyAsync(dx, x0, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    else PR_CUDA(cudaMemsetAsync(dx, 0, n * sizeof(double), c->stream));
    const uint64_t it = pr::cg_reference_fine(c, dx, max_iters, accuracy, delta);
    PR_CUDA(cudaMemcpyAsync(x, dx, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    c->sync();
    c->release("acc_x");
    if (out_iters) *out_iters = it;
  });
}

int pr_ctx_band_info(pr_context* c, uint32_t* depth, uint32_t* coarse_depth, uint64_t* n_bricks, uint32_t* brick_codes) {
  return guard([&] {
    PR_REQUIRE(c != nullptr, PR_ERR_INVALID_ARGUMENT, "context is NULL");
    PR_REQUIRE(c->have_state && c->adaptive, PR_ERR_STATE, "no adaptive reconstruction state");
    if (depth) *depth = c->D;
    if (coarse_depth) *coarse_depth = c->band_Dc;
    if (n_bricks) *n_bricks = c->band_nb;
    if (brick_codes && c->band_nb) {
      set_device(c);
      PR_CUDA(cudaMemcpyAsync(brick_codes, c->get<uint32_t>("ab_bkey"), c->band_nb * sizeof(uint32_t),
                              cudaMemcpyDeviceToHost, c->stream));
      c->sync();
    }
  });
}

int pr_ctx_band_get(pr_context* c, int which, double* out) {
  return guard([&] {
    PR_REQUIRE(c != nullptr && out != nullptr, PR_ERR_INVALID_ARGUMENT, "NULL argument");
    PR_REQUIRE(c->have_state && c->adaptive, PR_ERR_STATE, "no adaptive reconstruction state");
    set_device(c);
    double* d = c->buf<double>("acc_band", std::max<uint64_t>(c->n, 1));
    pr::band_vector(c, which, d);
    if (c->n) PR_CUDA(cudaMemcpyAsync(out, d, c->n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    c->sync();
    c->release("acc_band");
  });
}

int pr_ctx_band_apply(pr_context* c, const double* x, double* y) {
  return guard([&] {
    PR_REQUIRE(c != nullptr && x != nullptr && y != nullptr, PR_ERR_INVALID_ARGUMENT, "NULL argument");
    PR_REQUIRE(c->have_state && c->adaptive, PR_ERR_STATE, "no adaptive reconstruction state");
    set_device(c);
    const uint64_t n = std::max<uint64_t>(c->n, 1);
    double* dx = c->buf<double>("acc_bx", n);
    double* dy = c->buf<double>("acc_by", n);
    PR_CUDA(cudaMemcpyAsync(dx, x, c->n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    pr::band_apply64(c, dx, dy);
    PR_CUDA(cudaMemcpyAsync(y, dy, c->n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    c->sync();
    c->release("acc_bx");
    c->release("acc_by");
  });
}

int pr_ctx_get_unit_points(pr_context* c, double* out6) {
  return guard([&] {
    PR_REQUIRE(c != nullptr && out6 != nullptr, PR_ERR_INVALID_ARGUMENT, "NULL argument");
    PR_REQUIRE(c->have_points, PR_ERR_STATE, "no points");
    set_device(c);
    std::unique_ptr<double[]> pos(new double[3 * c->P]), nrm(new double[3 * c->P]);
    PR_CUDA(cudaMemcpyAsync(pos.get(), c->get<double>("upos"), 3 * c->P * sizeof(double), cudaMemcpyDeviceToHost,
                            c->stream));
    PR_CUDA(cudaMemcpyAsync(nrm.get(), c->get<double>("unrm"), 3 * c->P * sizeof(double), cudaMemcpyDeviceToHost,
                            c->stream));
    c->sync();
    for (uint64_t i = 0; i < c->P; ++i)
      for (int k = 0; k < 3; ++k) {
        out6[6 * i + k] = pos[k * c->P + i];
        out6[6 * i + 3 + k] = nrm[k * c->P + i];
      }
  });
}

int pr_ctx_get_normal_field(pr_context* c, double* out3, double* outw) {
  return guard([&] {
    PR_REQUIRE(c != nullptr && out3 != nullptr && outw != nullptr, PR_ERR_INVALID_ARGUMENT, "NULL argument");
    PR_REQUIRE(c->have_state, PR_ERR_STATE, "no reconstruction state");
    PR_REQUIRE(!c->adaptive, PR_ERR_STATE, "the last reconstruction was adaptive: read it with the band accessors");
    set_device(c);
    double* nf = c->buf<double>("acc_nf3", 3 * c->n);
    double* w = c->buf<double>("acc_w", c->n);
    if (c->degree == 2) pr::deg2_normal_field_morton(c, nf, w);
    else pr::scatter_normal_field(c, nf, w);
    PR_CUDA(cudaMemcpyAsync(out3, nf, 3 * c->n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    PR_CUDA(cudaMemcpyAsync(outw, w, c->n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    c->sync();
    c->release("acc_nf3");
    c->release("acc_w");
  });
}

int pr_ctx_apply_operator(pr_context* c, const double* x, double* y, int precision) {
  return guard([&] {
    PR_REQUIRE(c != nullptr && x != nullptr && y != nullptr, PR_ERR_INVALID_ARGUMENT, "NULL argument");
    PR_REQUIRE(c->have_state, PR_ERR_STATE, "no reconstruction state");
    PR_REQUIRE(!c->adaptive, PR_ERR_STATE, "the last reconstruction was adaptive: read it with the band accessors");
    set_device(c);
    const uint64_t n = c->n;
    double* dx = c->buf<double>("acc_x", n);
    double* dy = c->buf<double>("acc_y", n);
    PR_CUDA(cudaMemcpyAsync(dx, x, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    if (precision == PR_PRECISION_FP64) {
      if (c->degree == 2) pr::deg2_apply_morton<double>(c, dx, dy);
      else pr::apply_operator64(c, dx, dy);
    } else {
      float* fx = c->buf<float>("acc_fx", n);
      float* fy = c->buf<float>("acc_fy", n);
      pr::scale_convert<double, float>(c->stream, n, 1.0, dx, fx);
      if (c->degree == 2) pr::deg2_apply_morton<float>(c, fx, fy);
      else pr::apply_operator32(c, fx, fy);
      pr::scale_convert<float, double>(c->stream, n, 1.0, fy, dy);
    }
    PR_CUDA(cudaMemcpyAsync(y, dy, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    c->sync();
  });
}

int pr_ctx_evaluate(pr_context* c, const double* coeffs, const double* pts3, uint64_t n, double* out) {
  return guard([&] {
    PR_REQUIRE(c != nullptr && (pts3 != nullptr || n == 0) && (out != nullptr || n == 0), PR_ERR_INVALID_ARGUMENT,
               "NULL argument");
    PR_REQUIRE(c->have_state, PR_ERR_STATE, "no reconstruction state");
    PR_REQUIRE(!c->adaptive, PR_ERR_STATE, "the last reconstruction was adaptive: read it with the band accessors");
    set_device(c);
    if (n == 0) return;
    const double* dx;
    if (coeffs) {
      double* t = c->buf<double>("acc_x", c->n);
      PR_CUDA(cudaMemcpyAsync(t, coeffs, c->n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
      dx = t;
    } else {
      PR_REQUIRE(c->have_coeffs, PR_ERR_STATE, "no solved coefficients");
      dx = pr::coeffs_morton(c);
    }
    double* dp = c->buf<double>("acc_pts", 3 * n);
    double* dout = c->buf<double>("acc_out", n);
    PR_CUDA(cudaMemcpyAsync(dp, pts3, 3 * n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    pr::evaluate_points(c, c->D, dx, dp, 3, n, dout, c->degree);
    PR_CUDA(cudaMemcpyAsync(out, dout, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    c->sync();
  });
}

static void extract_common(pr_context* c, uint32_t depth, const double* coeffs, double iso, pr_mesh* out,
                           int degree) {
  PR_REQUIRE(coeffs != nullptr && out != nullptr, PR_ERR_INVALID_ARGUMENT, "NULL argument");
  PR_REQUIRE(depth >= pr::kMinDepth && depth <= pr::kMaxDepth, PR_ERR_INVALID_ARGUMENT, "depth must be in [1, 10]");
  PR_REQUIRE(std::isfinite(iso), PR_ERR_INVALID_ARGUMENT, "iso must be finite");
  set_device(c);
  std::memset(out, 0, sizeof(*out));
  const uint64_t n = 1ull << (3 * depth);
  double* dx = c->buf<double>("ext_x", n);
  PR_CUDA(cudaMemcpyAsync(dx, coeffs, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  pr::stage_extract(c, depth, dx, iso, false, degree);
  copy_mesh_to_host(c, out);
}

int pr_ctx_extract(pr_context* c, const double* coeffs, double iso, pr_mesh* out) {
  return guard([&] {
    PR_REQUIRE(c != nullptr, PR_ERR_INVALID_ARGUMENT, "context is NULL");
    PR_REQUIRE(c->have_state, PR_ERR_STATE, "no reconstruction state");
    PR_REQUIRE(!c->adaptive, PR_ERR_STATE, "the last reconstruction was adaptive: read it with the band accessors");
    extract_common(c, c->D, coeffs, iso, out, c->degree);
  });
}

int pr_ctx_extract_at_depth(pr_context* c, uint32_t depth, const double* coeffs, double iso, pr_mesh* out) {
  return guard([&] {
    PR_REQUIRE(c != nullptr, PR_ERR_INVALID_ARGUMENT, "context is NULL");
    extract_common(c, depth, coeffs, iso, out, 1);
  });
}

}  // extern "C"

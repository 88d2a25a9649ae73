// Launch wrappers of the solver kernels (pr_operator.cu), templated on the vector type.
#pragma once

#include <string>
#include <type_traits>

#include "pr_internal.cuh"

namespace pr {

// Constant 21-point stencil of the degree-1 FEM stiffness (src/fem_tree.rs:39-48):
// centre c0 (plus a diagonal shift), edge neighbours ce, corner neighbours cc; the six
// face neighbours are exactly 0 and dropped (src/fem_tree.rs:194).
template <typename T>
struct Coef {
  T c0, ce, cc;
};
Coef<double> stencil_coef(uint32_t depth, double diag_shift);
template <typename T>
inline Coef<T> cast_coef(const Coef<double>& c) {
  return Coef<T>{(T)c.c0, (T)c.ce, (T)c.cc};
}

// Screening payload: per (point, corner) node key (or sentinel) and basis value, plus
// the node-sorted pair lists.  (S x)_i = wh3 * sum_p phi_i(p) * (sum_j phi_j(p) x_j).
template <typename T>
struct Screen {
  const uint32_t* key = nullptr;   // 8P, per point in input order
  const T* phi = nullptr;          // 8P
  const uint32_t* snode = nullptr; // S screened nodes (sorted)
  const uint32_t* soff = nullptr;  // S+1
  const uint32_t* sval = nullptr;  // pairs: 8p+k, node-sorted, point order inside a node
  uint64_t P = 0, S = 0;
  uint32_t sentinel = 0;            // res^3: key of a corner outside the grid
  T wh3 = 0;
  T* proj = nullptr;               // P scratch: phi(p) . x
  bool active() const { return S > 0; }
};

// One cloud's screening payload in a packed solve (several clouds of one depth and screening
// weight, vectors concatenated): a device array holds one descriptor per cloud.
struct ScreenDesc {
  const uint32_t* key = nullptr;  // 8P
  const float* phi32 = nullptr;   // 8P
  const double* phi64 = nullptr;  // 8P
  const uint32_t* snode = nullptr, *soff = nullptr, *sval = nullptr;
  float* proj32 = nullptr;        // P scratch
  double* proj64 = nullptr;       // P scratch
  uint64_t P = 0, S = 0;
};
struct ScreenPack {
  const ScreenDesc* desc = nullptr;  // device, one per cloud
  uint32_t clouds = 0;
  uint64_t maxP = 0, maxS = 0;
  uint32_t sentinel = 0;  // res^3
  double wh3 = 0.0;
  bool active() const { return maxS > 0; }
};
// per cloud: proj = Phi^T x; part (nullable, nparts per cloud): per-block sums of proj^2
template <typename T>
void screen_project_pk(cudaStream_t s, const ScreenPack& scr, const T* x, uint64_t n, double* part = nullptr,
                       int nparts = 0);
// per cloud: y += sign * wh3 * Phi proj
template <typename T>
void screen_gather_pk(cudaStream_t s, const ScreenPack& scr, T* y, uint64_t n, int sign);
// per cloud k: out[k] = a_k . b_k (fixed order), part: kDotBlocks per cloud (device results)
template <typename T>
void dots_pk(cudaStream_t s, const T* a, const T* b, uint64_t n, uint32_t clouds, double* part, double* out);
// per cloud k: y_k = (float) x_k, out[k] = x_k . x_k (device results)
void convert_sq_pk(cudaStream_t s, const double* x, float* y, uint64_t n, uint32_t clouds, double* part, double* out);

// y = A' x (mode 0) or y = f - A' x (mode 1), A' = constant stencil at `depth`
template <typename T>
void stencil_apply(cudaStream_t s, uint32_t depth, const T* x, const T* f, T* y, Coef<T> c, int mode);
// y += sign * S x
template <typename T>
void screen_apply(cudaStream_t s, const Screen<T>& scr, const T* x, T* y, int sign);
// scr.proj[p] = phi(p) . x
template <typename T>
void screen_project(cudaStream_t s, const Screen<T>& scr, const T* x);
// y += sign * wh3 * Phi proj  (proj from a previous projection)
template <typename T>
void screen_gather(cudaStream_t s, const Screen<T>& scr, T* y, int sign);

// dot products (deterministic, accumulated in FP64); result returned on the host
template <typename T>
double dot(pr_context* c, const T* a, const T* b, uint64_t n);

// x += alpha d ; r -= alpha q ; returns r.r (host)
template <typename T>
double cg_update(pr_context* c, uint64_t n, double alpha, const T* d, const T* q, T* x, T* r);
// r -= alpha q ; returns r.r (host)
template <typename T>
double r_update(pr_context* c, uint64_t n, double alpha, const T* q, T* r);
// d = z + beta d
template <typename T>
void xpby(cudaStream_t s, uint64_t n, const T* z, double beta, T* d);
// y = a * x  (conversion between types allowed)
// y = (float)x; returns ||x|| (fixed-order FP64 sum)
double convert_norm(pr_context* c, const double* x, float* y, uint64_t n);
template <typename Tin, typename Tout>
void scale_convert(cudaStream_t s, uint64_t n, double a, const Tin* x, Tout* y);
// y += a * x  (conversion allowed)
template <typename Tin, typename Tout>
void axpy(cudaStream_t s, uint64_t n, double a, const Tin* x, Tout* y);

// multigrid pieces
template <typename T>
void gs_sweep(cudaStream_t s, uint32_t depth, T* x, const T* f, Coef<T> c, bool forward);
template <typename T>
void restrict_to_coarse(cudaStream_t s, uint32_t fine_depth, const T* r_fine, T* f_coarse);
template <typename T>
void prolong_add(cudaStream_t s, uint32_t fine_depth, const T* e_coarse, T* e_fine);
// e = inv f per cloud (clouds > 1: packed vectors of nc entries per cloud)
template <typename T>
void dense_solve(cudaStream_t s, uint32_t nc, const T* inv, const T* f, T* e, uint32_t clouds = 1);

// ------------------------------------------------------------------ the fine operator
template <typename T>
const char* tname();
template <>
inline const char* tname<float>() { return "f32"; }
template <>
inline const char* tname<double>() { return "f64"; }

// Fine operator A = K + wg I + S (matrix-free)
template <typename T>
struct FineOp {
  uint32_t D = 0;
  Coef<T> coef{};
  Screen<T> scr;
  void apply(cudaStream_t s, const T* x, T* y) const {
    stencil_apply<T>(s, D, x, nullptr, y, coef, 0);
    screen_apply<T>(s, scr, x, y, +1);
  }
  void residual(cudaStream_t s, const T* x, const T* b, T* r) const {
    stencil_apply<T>(s, D, x, b, r, coef, 1);
    screen_apply<T>(s, scr, x, r, -1);
  }
};

template <typename T>
inline FineOp<T> make_fine_op(pr_context* c, double wg) {
  FineOp<T> op;
  op.D = c->D;
  op.coef = cast_coef<T>(stencil_coef(c->D, wg));
  if (c->pw > 0.0 && c->S > 0) {
    const double h = 1.0 / (double)(1u << c->D);
    op.scr.key = c->get<uint32_t>("scr_kin");
    op.scr.phi = std::is_same<T, double>::value ? (const T*)c->get<double>("phi64") : (const T*)c->get<float>("phi32");
    op.scr.snode = c->get<uint32_t>("scr_runkey");
    op.scr.soff = c->get<uint32_t>("scr_runoff");
    op.scr.sval = c->get<uint32_t>("scr_val");
    op.scr.P = c->P;
    op.scr.S = c->S;
    op.scr.sentinel = 1u << (3 * c->D);
    op.scr.wh3 = (T)(c->pw * (h * h * h) / 1.5);
    op.scr.proj = c->buf<T>(std::string("scr_proj_") + tname<T>(), c->P);
  }
  return op;
}

}  // namespace pr

/*
 * poisson_recon.h — C ABI of the B200-native screened Poisson reconstructor.
 *
 * Drop-in for the reference crate's one public hot path,
 *     pub fn reconstruct(points: &[OrientedPoint], params: &ReconstructParams)
 *         -> (Mesh, ReconstructStats)                      (src/reconstructor.rs:25)
 * with the crate's types mirrored field for field:
 *     OrientedPoint     src/fem_tree.rs:10  (position Point3 + normal Vec3, 6 x f64)
 *     ReconstructParams src/reconstructor.rs:8-15
 *     ReconstructStats  src/reconstructor.rs:17-23
 *     Mesh              src/marching_cubes.rs:8-11 (vertices [f64;3], triangles [usize;3])
 *
 * All entry points return a status (PR_OK = 0, negative on failure) and never abort;
 * the message of the last failure on the calling thread is pr_last_error().
 * Signatures carry plain pointers and sizes only.
 */
#ifndef POISSON_RECON_H
#define POISSON_RECON_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status codes */
#define PR_OK 0
#define PR_ERR_INVALID_ARGUMENT -1 /* bad pointer, depth outside [1,10], non-finite input, ... */
#define PR_ERR_OUT_OF_MEMORY -2    /* device or host allocation failed */
#define PR_ERR_CUDA -3             /* a CUDA call failed (message names it) */
#define PR_ERR_NOT_CONVERGED -4    /* solver hit max_iters before target_rel_residual */
#define PR_ERR_NO_DEVICE -5        /* no usable sm_100 device */
#define PR_ERR_STATE -6            /* accessor called before a reconstruction */
#define PR_ERR_INTERNAL -7

/* solve_mode */
#define PR_SOLVE_CONVERGED 0          /* solve the crate's fine system to target_rel_residual */
#define PR_SOLVE_REFERENCE_SCHEDULE 1 /* the crate's cascade: D-2 system, GS(20)+CG(cg_iters),
                                         one-level prolongation, GS(20)+CG(cg_iters/4); GS is
                                         8-colour (parallel) instead of sequential Morton order */
/* precision (converged mode) */
#define PR_PRECISION_MIXED 0 /* FP32 multigrid-preconditioned CG + FP64 residual refinement */
#define PR_PRECISION_FP64 1  /* FP64 multigrid-preconditioned CG throughout */

/* OrientedPoint (src/fem_tree.rs:10): AoS, 48 bytes. */
typedef struct pr_oriented_point {
  double x, y, z;    /* position (model space) */
  double nx, ny, nz; /* normal; need not be unit length (renormalised, src/reconstructor.rs:38) */
} pr_oriented_point;

/* ReconstructParams (src/reconstructor.rs:8-11): the crate's fields in order, then
 * extensions.  pr_params_default() gives ReconstructParams::default() for the crate's
 * fields (src/reconstructor.rs:14). */
typedef struct pr_params {
  uint32_t depth;          /* octree depth D; grid res = 2^D; 1 <= D <= 10 (12 with coarse_depth) */
  double samples_per_node; /* accepted and ignored, as in the crate */
  double scale;            /* s = scale / max bbox extent (src/geometry.rs:384-388) */
  double cg_accuracy;      /* reference schedule: CG stop ||r||^2 <= ||r0||^2 acc^2 */
  uint64_t cg_iters;       /* reference schedule: coarse CG iterations (fine: /4) */
  double point_weight;     /* screening weight; 0 disables screening */
  int32_t verbose;         /* print stage timings to stderr */
  /* --- extensions --- */
  int32_t solve_mode;         /* PR_SOLVE_* (default PR_SOLVE_CONVERGED) */
  int32_t precision;          /* PR_PRECISION_* (default PR_PRECISION_MIXED) */
  double target_rel_residual; /* ||b - A x||_2 / ||b||_2 in FP64 (default 1e-6) */
  uint32_t max_iters;         /* cap on preconditioned CG iterations, all passes (default 200) */
  uint32_t smooth_sweeps;     /* multigrid pre/post Gauss-Seidel sweeps (default 1) */
  double inner_rel_tol;       /* mixed: relative tolerance of each FP32 inner solve (default 1e-4) */
  uint32_t degree;            /* B-spline degree of the node functions: 1 (the crate's; 0 means 1) or 2
                                 (quadratic B-splines, converged mode only; default 1) */
  uint32_t coarse_depth;      /* 0 (default): one dense grid at `depth`.  Otherwise the adaptive
                                 (narrow-band) reconstruction, degree 2 only: a dense solve at this
                                 depth, then the depth-`depth` system on the 8^3-node bricks that hold
                                 the points' basis functions, with the prolonged coarse solution outside
                                 them (Jacobi-preconditioned CG, capped at 10 max_iters);
                                 3 <= depth <= 12, 1 <= depth - coarse_depth <= 4 */
  uint32_t band_flags;        /* adaptive: PR_BAND_FULL activates every brick (the dense system) */
  uint32_t reserved[5];
} pr_params;
#define PR_BAND_FULL 1u

/* Mesh (src/marching_cubes.rs:8-11).  Vertices are model-space [x,y,z] triples; triangles
 * are vertex-index triples (the crate's usize -> uint64).  Library-owned: free with
 * pr_mesh_free() (or each array with pr_host_free()). */
typedef struct pr_mesh {
  double* vertices;
  uint64_t n_vertices;
  uint64_t* triangles;
  uint64_t n_triangles;
} pr_mesh;

/* ReconstructStats (src/reconstructor.rs:17-23), then extensions. */
typedef struct pr_stats {
  double time_transform, time_tree, time_system, time_solve, time_extract, time_total; /* seconds */
  uint64_t fem_nodes;  /* res^3 */
  uint64_t matrix_nnz; /* 0: the operator is matrix-free (the crate also leaves it 0) */
  uint64_t mesh_vertices, mesh_triangles;
  double iso_value;
  /* --- extensions --- */
  double rel_residual;          /* final ||b - A x|| / ||b|| (FP64) */
  uint32_t pcg_iterations;      /* preconditioned CG iterations, summed over passes */
  uint32_t refinement_steps;    /* FP64 outer residual steps (mixed precision) */
  uint64_t points_in_cube;      /* points with at least one screening node */
  double solve_bytes;           /* algorithmic HBM bytes moved by the solve */
  double peak_device_bytes;     /* peak device memory of the context's live buffers (spare blocks kept for reuse not counted) */
  int32_t converged;            /* converged mode: 1 if rel_residual <= target_rel_residual */
  int32_t reserved_i;
  double time_mesh_copy;        /* seconds copying the mesh to the caller's host memory */
  double reserved[4];
} pr_stats;

/* ------------------------------------------------------------------ one-shot API */
pr_params pr_params_default(void);

/* reconstruct(points, params) -> (mesh, stats)  (src/reconstructor.rs:25-70).
 * points: n AoS records of 6 doubles (host memory; pinned memory is copied faster).
 * An empty input returns PR_OK with an empty mesh and zeroed stats, like the crate.
 * out_stats may be NULL. */
int pr_reconstruct(const double* points6, uint64_t n, const pr_params* params, pr_mesh* out_mesh,
                   pr_stats* out_stats);
/* Frees a mesh returned by this library (both arrays).  Mesh arrays may live in pinned memory
 * from a library pool: release them only through pr_mesh_free / pr_host_free, never free(). */
void pr_mesh_free(pr_mesh* mesh);
/* Frees ONE array of a returned mesh (for bindings that own the two arrays separately). */
void pr_host_free(void* array);
const char* pr_last_error(void);

/* ------------------------------------------------------------------ context API
 * A context owns one device, one CUDA stream (caller-provided or its own) and the
 * device buffers of its last reconstruction (reused by the next call).  Calls on
 * distinct contexts are thread-safe; one context must not be used concurrently. */
typedef struct pr_context pr_context;

/* stream: a cudaStream_t, or NULL for a context-owned stream. */
int pr_context_create(int device, void* stream, pr_context** out_ctx);
int pr_context_destroy(pr_context* ctx);

int pr_ctx_reconstruct(pr_context* ctx, const double* points6, uint64_t n, const pr_params* params,
                       pr_mesh* out_mesh, pr_stats* out_stats);
/* Same, input already in device memory; the mesh stays on the device (read it with
 * pr_ctx_mesh_device / pr_ctx_mesh_copy).  Nothing is copied between host and device
 * except a few scalars. */
int pr_ctx_reconstruct_device(pr_context* ctx, const double* d_points6, uint64_t n, const pr_params* params,
                              pr_stats* out_stats);
int pr_ctx_mesh_device(pr_context* ctx, const double** d_vertices, uint64_t* n_vertices,
                       const uint64_t** d_triangles, uint64_t* n_triangles);
int pr_ctx_mesh_copy(pr_context* ctx, pr_mesh* out_mesh);
int pr_ctx_synchronize(pr_context* ctx);

/* --- accessors of the last reconstruction's state (parity tests, diagnostics) --- */
/* depth, res^3, the model->unit transform (column-major 4x4, src/geometry.rs:384-402) */
int pr_ctx_info(pr_context* ctx, uint32_t* depth, uint64_t* fem_nodes, double* model_to_unit16);
/* FP64 solved coefficients in the crate's FEM index order (Morton, x in bit 0). */
int pr_ctx_get_coefficients(pr_context* ctx, double* out_n);
/* FP64 right-hand side b (src/fem_tree.rs:251-299), FEM index order. */
int pr_ctx_get_rhs(pr_context* ctx, double* out_n);
/* Unit-cube points (AoS x y z nx ny nz) after the transform of src/reconstructor.rs:36-40. */
int pr_ctx_get_unit_points(pr_context* ctx, double* out_6n);
/* Normal field after splat + normalisation (src/fem_tree.rs:130-178), dense (n x 3) and
 * node weights (n). */
int pr_ctx_get_normal_field(pr_context* ctx, double* out_3n, double* out_weight_n);
/* y = A x with the fine operator of src/fem_tree.rs:180-249 (stiffness + screening),
 * matrix-free; precision PR_PRECISION_FP64 or PR_PRECISION_MIXED (FP32 operator, FP64 I/O). */
int pr_ctx_apply_operator(pr_context* ctx, const double* x_n, double* y_n, int precision);
/* Adaptive reconstruction (pr_params.coarse_depth > 0) only.  No counterpart in the crate, which
 * refines every leaf to max_depth (src/fem_tree.rs:83-93); the fine system is the dense one of
 * pr_params.degree = 2 (src/fem_tree.rs:180-299 with quadratic node functions) restricted to the
 * band.  Band vectors hold 512 values per active brick, bricks in the order of brick_codes (Morton
 * codes of the brick coordinates, brick b covering fine nodes 8 b .. 8 b + 7 per axis), nodes in
 * natural order inside a brick (x fastest).  The dense accessors above refuse an adaptive state. */
int pr_ctx_band_info(pr_context* ctx, uint32_t* depth, uint32_t* coarse_depth, uint64_t* n_bricks,
                     uint32_t* brick_codes);
/* which: 0 = right-hand side b on the band, 1 = the solved coefficients f, 2 = the prolonged coarse
 * solution g on the band (the function outside the band is g) */
int pr_ctx_band_get(pr_context* ctx, int which, double* out);
/* y = A_BB x: the band rows and columns of the fine operator (stiffness, shift, screening), FP64 */
int pr_ctx_band_apply(pr_context* ctx, const double* x, double* y);
/* Reference schedule (PR_SOLVE_REFERENCE_SCHEDULE) only: the right-hand side of its coarse
 * system (FEMTree::build_system_at_depth, src/fem_tree.rs:386-402) at *coarse_depth = max(D-2, 0),
 * 8^(*coarse_depth) values in Morton order (out may be NULL to query the depth). */
int pr_ctx_get_coarse_rhs(pr_context* ctx, uint32_t* coarse_depth, double* out);
/* The crate's CG loop (solve_cg, src/solvers.rs:20-69: residual recomputed every 10th iteration,
 * stop at ||r||^2 <= ||r0||^2 accuracy^2) on the fine system of the last degree-1 reconstruction,
 * FP64 on the device, from x0 (n doubles, FEM order; NULL = 0) for at most max_iters
 * iterations.  x receives the iterate; delta (may be NULL) receives ||r||^2 before the first
 * iteration and after each one (max_iters + 1 slots); *out_iters the crate's return value. */
int pr_ctx_cg_reference(pr_context* ctx, const double* x0, uint64_t max_iters, double accuracy, double* x,
                        double* delta, uint64_t* out_iters);
/* Evaluate the implicit function (src/fem_tree.rs:490-513) of `coefficients` (NULL = the
 * solved ones) at unit-cube points (3 doubles each). */
int pr_ctx_evaluate(pr_context* ctx, const double* coefficients, const double* pts3, uint64_t n, double* out);
/* Marching cubes (src/fem_tree.rs:576-636) of given FP64 coefficients at the context's depth
 * and the given iso value; vertices in UNIT-CUBE space (no back-transform). */
int pr_ctx_extract(pr_context* ctx, const double* coefficients, double iso, pr_mesh* out_mesh);
/* Same, at an explicit depth, without a prior reconstruction. */
int pr_ctx_extract_at_depth(pr_context* ctx, uint32_t depth, const double* coefficients, double iso,
                            pr_mesh* out_mesh);

/* y = A x on device-resident vectors (n = res^3 entries, float for PR_PRECISION_MIXED,
 * double for PR_PRECISION_FP64), enqueued on the context's stream without synchronising.
 * For benchmarks of the operator kernel. */
int pr_ctx_apply_operator_device(pr_context* ctx, const void* d_x, void* d_y, int precision);

/* Micro-benchmark of one solver kernel on context-owned buffers at `depth` (4..10):
 * kernel 0 = fine-level stencil SpMV, 1 = SpMV fused with d = z + beta d, 2 = multigrid
 * smoothing sweep from zero, 3 = smoothing sweep, 4 = smoothing sweep fused with the
 * prolongation and a dot product, 5 = residual fused with the restriction, 6 = per-node
 * stencil (ids 0-6 on the finest level's coefficients), 7 and 8 = ids 4 and 5 on a coarse
 * level's (rows on the low domain faces use their own table rows), 9 = the CG update fused
 * with the first pre-smoothing sweep.  Degree 2 (finest level of `depth`): 20 = Chebyshev
 * smoothing step (TMA-fed), 21 = the same with register staging, 22 / 23 = A x (TMA / register
 * staging), 24 = f - A x (TMA), 25 = restriction, 26 = prolongation + add, 27 = first
 * Chebyshev step, 28 = the first two steps fused (from f), 29 = the third step recomputing the
 * first from f, 30 = the fused CG direction pass (d = z + beta d, q = A d, x += alpha d), 31 = the
 * fused FP64 refinement step (x + e, b - A x, FP32 copy; FP64 only) (TMA variants need depth >= 6).  Times `reps` launches
 * with CUDA events on the context's stream; returns the mean ms per launch and the
 * algorithmic HBM bytes per launch. */
int pr_ctx_kernel_bench(pr_context* ctx, int kernel, uint32_t depth, int precision, int reps, double* ms_per_launch,
                        double* bytes_per_launch);

/* ------------------------------------------------------------------ batches
 * Many independent clouds (each with its own params, e.g. its own depth).  Clouds on a dense
 * degree-1 grid of depth >= 5 in solve_mode PR_SOLVE_CONVERGED that share depth, point_weight,
 * precision, target_rel_residual, inner_rel_tol, max_iters and smooth_sweeps are reconstructed in
 * packs: set up and extracted one per context on host threads, their systems solved together
 * with one launch per solver step for every cloud of the pack (a pack holds as many clouds as
 * the free device memory does; PR_PACK_MAX_CLOUDS caps it).  Packed results equal single calls
 * bit for bit; a packed cloud's time_solve is its share of the pack's solve.  The packs use
 * library-owned contexts on ctxs[0]'s device, kept for later batches (their memory is released
 * when an allocation elsewhere in the process fails).  Every other cloud goes through ctxs: one
 * host thread per context drives that context's stream, clouds taken largest first.
 * out_meshes[i] / out_stats[i] / out_status[i] belong to cloud i (out_stats and out_status may
 * be NULL).  Returns PR_OK if every cloud succeeded, else the status of the lowest-numbered
 * failed cloud (its message in pr_last_error); the other clouds' results are still written.  No
 * counterpart in the reference crate, which reconstructs one cloud per call
 * (src/reconstructor.rs:25). */
int pr_ctx_reconstruct_batch(pr_context* const* ctxs, uint32_t n_ctx, const double* const* points6, const uint64_t* n,
                             uint32_t count, const pr_params* params, pr_mesh* out_meshes, pr_stats* out_stats,
                             int* out_status);
/* Same on a library-owned set of `concurrency` contexts on device 0 (0 = 4), kept between calls
 * (calls are serialised). */
int pr_reconstruct_batch(const double* const* points6, const uint64_t* n, uint32_t count, const pr_params* params,
                         uint32_t concurrency, pr_mesh* out_meshes, pr_stats* out_stats, int* out_status);

/* ------------------------------------------------------------------ adjoint (gradients)
 * No counterpart in the reference crate.  The implicit function chi(q) = evaluate(x, M q)
 * (src/fem_tree.rs:490-513) of the solved coefficients x (A x = b, src/fem_tree.rs:180-299)
 * at K query points q (MODEL space, mapped with the reconstruction's unit-cube transform M)
 * is differentiated w.r.t. the input points' model-space positions and normals.  Given the
 * upstream gradient g_k = dL/dchi_k, the adjoint solve A lambda = E^T g (A is symmetric; E =
 * the evaluation matrix) gives dL/dtheta = lambda . db/dtheta - lambda . (dA/dtheta) x through
 * the normalised splat (src/fem_tree.rs:130-178), the divergence RHS and the screening RHS and
 * matrix.  M follows the bounding box of the input and is HELD FIXED (not differentiated).
 * Degree 1 (the crate's piecewise linear basis) and degree 2 (quadratic B-splines, the same
 * formulas with 27 nodes per point), dense grids and the adaptive band.  For the band, chi is the
 * fine function (f on the band, the prolonged coarse solution elsewhere); the adjoint solves the
 * band system (A_BB lambda = E^T g on the band) and then the coarse system with the right-hand side
 * P^T (E^T g - A E lambda), and adds both levels' per-point terms; the brick set is held fixed.
 * At a point exactly on a cell face the one-sided derivative of the cell the point falls in is
 * returned. */
typedef struct pr_adjoint_stats {
  double loss;          /* sum_k g_k chi_k, or mean chi_k^2 when dl_dchi was NULL */
  double rel_residual;  /* adjoint solve ||E^T g - A lambda|| / ||E^T g|| */
  uint32_t pcg_iterations;
  uint32_t refinement_steps;
  int32_t converged;
  int32_t queries_off_band; /* adaptive state: queries with a basis node outside the band (their
                               terms go through the coarse function) */
  double time_solve;  /* seconds in the adjoint solve */
  double time_total;  /* seconds in the whole call */
  double reserved[4];
} pr_adjoint_stats;

/* Forward without marching cubes: transform, splat, RHS and the solve of the crate's fine
 * system (host points; stats as pr_ctx_reconstruct, mesh counts 0).  The state it leaves is
 * what pr_ctx_loss_backward differentiates. */
int pr_ctx_solve(pr_context* ctx, const double* points6, uint64_t n, const pr_params* params, pr_stats* out_stats);
/* Backward of the last pr_ctx_solve / pr_ctx_reconstruct on this context (which must have
 * used solve_mode PR_SOLVE_CONVERGED).  queries3: k model-space points (x y z); dl_dchi: k
 * upstream gradients, or NULL for the loss L = mean_k chi_k^2.  Outputs (host, any may be
 * NULL): chi (k), dl_dpositions and dl_dnormals (n x 3 each, the input's point order).  The
 * adjoint solve uses the last call's precision and target_rel_residual. */
int pr_ctx_loss_backward(pr_context* ctx, const double* queries3, uint64_t k, const double* dl_dchi, double* chi,
                         double* dl_dpositions, double* dl_dnormals, pr_adjoint_stats* out_stats);
/* One-shot: pr_ctx_solve + pr_ctx_loss_backward on the calling thread's default context. */
int pr_loss_backward(const double* points6, uint64_t n, const pr_params* params, const double* queries3, uint64_t k,
                     const double* dl_dchi, double* chi, double* dl_dpositions, double* dl_dnormals,
                     pr_adjoint_stats* out_stats);

/* ------------------------------------------------------------------ PLY files (host)
 * ply::read_oriented_points (src/ply.rs:13-70): ASCII as the crate reads it (header up to
 * "end_header"; "element vertex N"; a header line containing "nx" or "normal_x" is required;
 * every later line with >= 6 tokens gives x y z nx ny nz from its first six tokens, a token
 * that does not parse as f64 reads as 0.0, shorter lines are skipped); extension: files in
 * binary_little_endian, read by property name.  *out_points6 (n AoS records of 6 doubles) is
 * library memory: free it with pr_host_free.  Errors carry the crate's messages. */
int pr_ply_read_points(const char* path, double** out_points6, uint64_t* out_n);
#define PR_PLY_ASCII 0  /* ply::write_mesh (src/ply.rs:73-107), byte for byte */
#define PR_PLY_BINARY 1 /* binary_little_endian, double vertices, uint32 (or uint64) indices */
int pr_ply_write_mesh(const char* path, const pr_mesh* mesh, int format);

/* Number of kernels launched by this library in this process (own kernels; library
 * primitives such as radix sorts and scans are counted in *primitive_calls). */
uint64_t pr_kernel_launches(uint64_t* primitive_calls);

/* The z-segment choices of the degree-1 block kernels made so far in this process: the first
 * FP32 launch of a (kernel family, level, launch size) times 2, 4 and 8 z planes per thread
 * (identical results) and keeps the fastest; one line per choice with its timings.  Library
 * memory, valid until the next call. */
const char* pr_autotune_log(void);

/* Iso value without any device allocation.  No counterpart in the reference crate: it exists
 * for callers that cannot allocate device memory — a host whose caching allocator already
 * holds the free device memory (a raw cudaMalloc would fail or fragment it), or a
 * latency-bound loop that must not pay for the device-wide synchronisation of
 * cudaMalloc/cudaFree.  Every input and the output are caller device pointers:
 * d_coefficients (res^3 FP64 values, res = 2^depth: the coefficients of the crate's linear
 * (degree-1) basis in the FEM index order, i.e. Morton order with x in bit 0, as
 * pr_ctx_get_coefficients returns them for a degree-1 reconstruction; degree-2 coefficients are
 * NOT accepted — the call cannot tell them apart and would return a wrong value), d_points3 (n
 * unit-cube points, x y z each), d_iso (1 double: the mean of the implicit function over the
 * points, as in src/reconstructor.rs:56; the same double as pr_stats.iso_value of a degree-1
 * reconstruction of these points).  Enqueued on `stream` (NULL = default stream), no
 * synchronisation.  Per-block partial sums live in a fixed 18,944-byte __device__ array that
 * each GPU loading the library keeps until exit; the first call on a device (with that
 * device current) resolves its address — make that first call before any stream capture.
 * All calls share the array: calls whose kernels overlap on the GPU race.  The resolved address
 * is cached per device; after cudaDeviceReset in the calling process it is stale, so do not call
 * this function after resetting a device.  Limits:
 * 1 <= n <= 2^28 points, depth 1..10; anything else returns PR_ERR_INVALID_ARGUMENT. */
int pr_iso_value_noalloc(uint32_t depth, const double* d_coefficients, const double* d_points3, uint64_t n,
                         double* d_iso, void* stream);

/* Library build information (static string). */
const char* pr_version(void);
/* sizeof(pr_params), sizeof(pr_mesh), sizeof(pr_stats), sizeof(pr_oriented_point): lets a
 * binding check its struct layouts without a GPU. */
void pr_abi_layout(uint64_t* out4);

#ifdef __cplusplus
}
#endif
#endif /* POISSON_RECON_H */

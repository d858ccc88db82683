/*
 * sdot_b200.h -- the C ABI of the B200-native semi-discrete optimal transport core.
 *
 * Every entry point is `extern "C"`, takes plain pointers, element counts and a `cudaStream_t`-owning
 * context, and reports through an `sdot_status`.  Nothing here names a torch or numpy type.  Each entry
 * point says which interface of the reference (hleclerc/sdot-ffi, package `sdot`) it replaces; the
 * reference binds those through its FFI layer (`loom.ffi_call` with a C++ expression naming a template
 * entry point), and this library is what such a call would bind instead.
 *
 * Conventions
 *   - Positions are row-major `[n, dim]` FP64, `dim` 2 or 3.  Weights are `[n]` FP64 or NULL (Voronoi).
 *   - The power cell of seed i is `{ x : |x - p_i|^2 - w_i <= |x - p_j|^2 - w_j for all j }` intersected
 *     with the axis-aligned domain box (src/sdot/PowerDiagram.py:3-10, 657-713).
 *   - Outputs are in the caller's seed order ("user order"); internally seeds are Morton-ranked.
 *   - `memory` fields say where the caller's arrays live: SDOT_HOST (the library copies them in and out
 *     on its stream, inside the call) or SDOT_DEVICE (pointers on the context's device).
 *   - Calls on one context are serialised by the caller: a context is not thread-safe.  Distinct
 *     contexts may be used from distinct threads.
 */
#ifndef SDOT_B200_H
#define SDOT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SDOT_ABI_VERSION 1

/* ---- status ------------------------------------------------------------------------------------ */
enum sdot_code {
    SDOT_OK = 0,
    SDOT_ERR_ARGS = 1,            /* a null pointer, a bad size, an unknown option                          */
    SDOT_ERR_CUDA = 2,            /* a CUDA call failed: `message` holds cudaGetErrorString                  */
    SDOT_ERR_NO_MEMORY = 3,       /* the device pool refused; nothing was launched past the refusal          */
    SDOT_ERR_CAPACITY = 4,        /* a cell exceeded its vertex / neighbour capacity: `id` is the user seed  */
    SDOT_ERR_UNSUPPORTED = 5,     /* a density / dimension combination this build does not integrate         */
    SDOT_ERR_NOT_CONVERGED = 6,   /* (solve only, informational: `stats[0]` holds the solver status)        */
    SDOT_ERR_TOPOLOGY = 7         /* a cell's clip gave a non-finite measure: `id` is the user seed; the cell
                                     is written empty, never NaN (gpu/Cell2D.cuh:99-102, 1214-1231)           */
};

/* the reference's error buffer records (kind, id, value) (src/sdot/include/sdot/gpu/Cell2D.cuh:99-102);
   `kind` 2 = failure, `id` the failing user seed, `needed` the capacity that would have sufficed */
typedef struct sdot_status {
    int32_t code;
    int32_t kind;
    int64_t id;
    int64_t value;
    int64_t needed;
    char message[160];
} sdot_status;

enum sdot_memory { SDOT_HOST = 0, SDOT_DEVICE = 1 };

/* ---- densities (distributions/Image.py, SumOfGaussians.py, Box.py) --------------------------------- */
enum sdot_density_kind {
    SDOT_DENSITY_UNIFORM = 0,     /* `value` on the domain box                                               */
    SDOT_DENSITY_IMAGE = 1,       /* piecewise constant, axis-aligned pixels; 2D                             */
    SDOT_DENSITY_GAUSSIANS = 2    /* sum of isotropic gaussians, `masses[g]` = mass of gaussian g            */
};

typedef struct sdot_density {
    int32_t kind;
    double value;                 /* UNIFORM: the density                                                    */
    int32_t shape[3];             /* IMAGE: pixels per axis                                                  */
    double origin[3];             /* IMAGE: corner of pixel (0, 0)                                           */
    double step[3];               /* IMAGE: pixel size per axis                                              */
    const double *values;         /* IMAGE: [shape[0], shape[1]] row-major, i along x (Image.py:12-20)       */
    int32_t count;                /* GAUSSIANS: number of gaussians                                          */
    const double *centres;        /* GAUSSIANS: [count, dim]                                                 */
    const double *sigmas;         /* GAUSSIANS: [count]                                                      */
    const double *masses;         /* GAUSSIANS: [count]                                                      */
} sdot_density;

/* ---- a diagram: seeds, weights, domain, density ---------------------------------------------------- */
typedef struct sdot_diagram_desc {
    int32_t dim;
    int64_t n;
    const double *positions;      /* [n, dim]                                                                */
    const double *weights;        /* [n] or NULL                                                             */
    double box_lo[3], box_hi[3];  /* the domain box                                                          */
    sdot_density density;         /* its arrays live where `memory` says                                     */
    int32_t memory;               /* SDOT_HOST or SDOT_DEVICE, for every array of this call                  */
} sdot_diagram_desc;

/* what a cells call writes; every pointer may be NULL (not computed) */
typedef struct sdot_cells_out {
    double *masses;               /* [n]        int_cell rho                                                 */
    double *barycentres;          /* [n, dim]   int x rho / int rho (the seed for an empty cell)             */
    double *costs;                /* [n]        int_cell |x - p_i|^2 rho                                     */
    int32_t cap;                  /* neighbours per cell in the three tables below                           */
    int32_t *nb_count;            /* [n]        facets towards other seeds                                   */
    int32_t *nb_ids;              /* [n, cap]   neighbour user index                                         */
    double *nb_coef;              /* [n, cap]   c_ij = int_facet rho / (2 |p_i - p_j|)  (sdotplan/Laplacian.h:7) */
    double *nb_measure;           /* [n, cap]   int_facet rho (the face length / area for rho = 1)            */
    int32_t precision;            /* 0: FP64 clipping; 1 (2D): FP32 clipping with FP64 re-checks of the vertices */
                                  /* within the FP32 band, every vertex re-solved in FP64 before the integration */
                                  /* (the reference's float kernel, gpu/Cell2D.cuh:56-60, 991-1042); 3D: refused */
} sdot_cells_out;

typedef struct sdot_context_s *sdot_context;

/* ---- context --------------------------------------------------------------------------------------- */
int32_t sdot_abi_version(void);

/* a context owns a CUDA stream and a stream-ordered device pool on `device`; `pool_limit` bytes (0: no
   limit besides the device) bound what the pool hands out at once (see sdot_context_memory).  Replaces the reference's per-call
   `queue` + `allocator` pair (docs/guide/ffi-internals.md:1-126, gpu/Cell2D.cuh:1519-1537). */
int32_t sdot_context_create(int32_t device, uint64_t pool_limit, sdot_context *out, sdot_status *st);
void sdot_context_destroy(sdot_context ctx);
void *sdot_context_stream(sdot_context ctx);                 /* the cudaStream_t every call runs on       */
int32_t sdot_context_synchronize(sdot_context ctx, sdot_status *st);
/* kernels this library launched on the context since its creation (a counter for benchmarks) */
uint64_t sdot_context_kernel_launches(sdot_context ctx);
/* the context's device pool: bytes handed out now, the most handed out at once since the last reset, and the limit
   given at creation (0: none).  A context created with a `pool_limit` refuses, with SDOT_ERR_NO_MEMORY, any allocation
   past it, and a solve whose model (`sdot_solve_bytes`) does not fit in what is left before anything is built -- the
   reference's check of the card's memory (CardMemory.check_card_memory, src/sdot/CardMemory.py:158-190).
   Synchronises the context's stream. */
int32_t sdot_context_memory(sdot_context ctx, uint64_t *in_use, uint64_t *peak, uint64_t *limit, int32_t reset_peak);
/* CUDA-event timing of the kernels by class (the reference's LOOM_KERNEL_TIMING, bench/README.md:112-140);
   also switched on for every context by the environment variable SDOT_KERNEL_TIMING=1 */
enum sdot_kernel_class { SDOT_K_CELLS2D = 0, SDOT_K_CELLS3D, SDOT_K_LAPLACIAN, SDOT_K_CG, SDOT_K_VECTOR, SDOT_K_INDEX, SDOT_K_REPORT,
                         SDOT_K_MULTIGRID,   /* the multigrid hierarchy's build and the CG's start on it */
                         SDOT_NB_KERNEL_CLASSES };
int32_t sdot_context_set_timing(sdot_context ctx, int32_t on);
/* THE GATHER MODEL of the cell kernels' traffic (what the search reads beyond the compulsory bytes, mostly from L2):
   while on, every `sdot_cells` of the context counts, per dimension, the records its neighbour search reads --
   candidate seeds (position + weight, 8 (dim + 1) bytes each), grid cells whose weight majorant it tested (8 bytes),
   grid cells whose seed range it read (8 bytes), pyramid nodes (affine majorant, 8 (dim + 1) bytes) -- in kernel
   instantiations of their own (the uncounted ones are unchanged).  A measurement aid with no counterpart in the
   reference, whose device counters (gpu/Cell2D.cuh:363) hold facets and overflow lists only.  The big-cell passes are
   not counted. */
int32_t sdot_context_set_counters(sdot_context ctx, int32_t on);
/* the counts of `dim` (2 or 3) since the last reset: counts[5] = { cells built, candidate seeds, grid cells tested,
   grid ranges read, pyramid nodes }; synchronises the context's stream */
int32_t sdot_context_gather_counters(sdot_context ctx, int32_t dim, uint64_t *counts, int32_t reset);
/* accumulated device time (ms), launches and units (seeds for the cells, rows x iterations for the CG) of a class
   since the last reset; synchronises the context's stream */
int32_t sdot_context_kernel_stats(sdot_context ctx, int32_t kernel_class, double *ms, uint64_t *launches, double *units, int32_t reset);

/* ---- one diagram -------------------------------------------------------------------------------------
 * Replaces `sdot::gpu2d::measures<V>(queue, pd, res, errors, allocator, rho, max_vertices, overflow_warps)`
 * and `sdot::gpu2d::cells<V,OUT>(queue, pd, res, lap, mom, ...)` (src/sdot/include/sdot/gpu/Cell2D.cuh:
 * 1801-1811; gpu/Cell3D.cuh:1941-2019), bound by PowerDiagram_Bsp._card_call (PowerDiagram_Bsp.py:271-305),
 * and the CPU sweeps behind `PowerDiagram.measures / moments / hessian_rows` (PowerDiagram.py:324-496).
 * Builds the Morton grid index on the device, clips every cell, integrates the density. */
int32_t sdot_cells(sdot_context ctx, const sdot_diagram_desc *desc, sdot_cells_out *out, sdot_status *st);

/* the adjoint of the masses: given `grad_masses` [n], writes `grad_positions` [n, dim] and `grad_weights` [n]
   (either may be NULL).  Replaces `sdot::gpu2d::measures_vjp<V>` (gpu/Cell2D.cuh:1815-1839): per cell
   grad_w_i = sum_j c_ij (g_i - g_j), grad_p_i = sum_j 2 c_ij (g_i - g_j)(x_ij - p_i) with x_ij the facet
   centroid (for rho constant on the facet). */
int32_t sdot_cells_vjp(sdot_context ctx, const sdot_diagram_desc *desc, const double *grad_masses, double *grad_positions,
                       double *grad_weights, sdot_status *st);

/* the adjoint of the masses and of the first moments F_i = int_{cell_i} x rho (world frame: the mass times the
   barycentre that sdot_cells writes): given `grad_masses` [n] and / or `grad_first` [n, dim] (either may be NULL, not both),
   writes `grad_positions` [n, dim] and `grad_weights` [n] (either may be NULL).  Replaces the backward of
   `PowerDiagram.moment(k)` for k < dim (src/sdot/PowerDiagram.py:341-353, "differentiable like measures"), which
   `SdotPlanNd._attach_derivatives` turns into the barycentres' derivative (SdotPlanNd.py:1018-1070).  A facet ij moves
   by dw / 2|p_ij| with a weight and by (x - p_i).dp_i / |p_ij| with a seed, so with G = gF_i - gF_j:
   grad_w_i += G . int_facet x rho / 2|p_ij|, grad_p_i += ((G . p_i) int_facet (x - p_i) rho
   + int_facet (x - p_i)(x - p_i)^T rho G) / |p_ij|.  A constant density only (SDOT_ERR_UNSUPPORTED otherwise). */
int32_t sdot_cells_vjp_moments(sdot_context ctx, const sdot_diagram_desc *desc, const double *grad_masses, const double *grad_first,
                               double *grad_positions, double *grad_weights, sdot_status *st);

/* the Laplacian of the Laguerre graph, CSR in user order, bit-symmetric, `dia` = row sum (1 for an empty row).
   `row_ptr` [n+1], `cols` [cap_nnz], `vals` [cap_nnz] (c_ij > 0: the matrix holds -c_ij), `dia` [n].
   `*nnz` receives the entry count; past `cap_nnz` the call fails with SDOT_ERR_CAPACITY and `needed`.
   Replaces `assemble_laplacian_in` (gpu/Laplacian2D.cuh:139-297) and `PowerDiagram.hessian_rows`. */
int32_t sdot_laplacian(sdot_context ctx, const sdot_diagram_desc *desc, int64_t cap_nnz, int64_t *row_ptr, int32_t *cols,
                       double *vals, double *dia, int64_t *nnz, sdot_status *st);

/* ---- the linear solve alone -------------------------------------------------------------------------
 * `L x_k = rhs_k` for k < nrhs with L = diag(dia) - offdiag(vals) given as CSR (row_ptr int64, cols int32),
 * each rhs of zero sum; x gauge-fixed to `x[0] = 0`.  `method` 0 = preconditioned CG (Jacobi),
 * 1 = CG preconditioned by the aggregation multigrid; 2 and 3 = the same two with the CG in FP32 on FP32
 * copies of the matrix and vectors, refined in FP64 (x and the residual b - L x kept in FP64, the inner CG
 * restarted on each new residual until it meets `tol`).  `iterations[k]` = CG iterations (-1: failed).
 * The reference's options of precision (gpu/Linear2D.cuh:80-102) map onto methods 2 / 3.
 * Replaces `sdot::gpu2d::linear_solves(queue, row, col, val, dia, rhs, options, solution, iterations,
 * allocator)` (gpu/Newton2D.cuh:1916-1960), the test hook `_card_linear_solves` (SdotPlanNd.py:204-236). */
int32_t sdot_linear_solve(sdot_context ctx, int64_t n, const int64_t *row_ptr, const int32_t *cols, const double *vals,
                          const double *dia, int32_t nrhs, const double *rhs, double *x, int32_t method, double tol,
                          int32_t maxit, int32_t memory, int32_t *iterations, sdot_status *st);

/* ---- the linear solve without allocations (no counterpart in the reference) -------------------------------
 * `sdot_linear_solve` with method 0 (Jacobi-PCG), its work vectors held in a static device array of the
 * library instead of memory allocated per call: no cudaMalloc / cudaFree / pool allocation in the call, for a
 * caller that cannot allocate while it solves (its framework holds the GPU's free memory, or it cannot pay the
 * device-wide synchronisation of cudaFree).  Every array is device memory.  At most SDOT_NOALLOC_MAX_ROWS rows
 * (past it: SDOT_ERR_CAPACITY, `needed` = n).  The array is shared by every call on a device: calls that
 * overlap in time race (one context serialises its own calls).  The first call on a device looks the array's
 * address up; make it before any stream capture on that device, and do not reset a device the library has
 * used (the address is kept).  The array (16 MB) is reserved on every device where the library's device code
 * is loaded, whether or not this entry point is called.  Every array must be memory of the context's own
 * device (or managed memory): another GPU's memory is refused with SDOT_ERR_ARGS before any launch. */
#define SDOT_NOALLOC_MAX_ROWS 262144
int32_t sdot_linear_solve_noalloc(sdot_context ctx, int64_t n, const int64_t *row_ptr, const int32_t *cols, const double *vals,
                                  const double *dia, int32_t nrhs, const double *rhs, double *x, double tol, int32_t maxit,
                                  int32_t *iterations, sdot_status *st);

/* ---- the Newton solve -----------------------------------------------------------------------------------
 * Options, in this order (`sdot_solve_desc.options`, `SDOT_NB_OPTIONS` values; SdotPlanNd._CARD_OPTIONS holds
 * the reference's card list, gpu/Newton2D.cuh:98-110): */
enum sdot_option {
    SDOT_OPT_TOL_ABS = 0,         /* stop when max|m - nu| <= tol_abs ...                                    */
    SDOT_OPT_TOL_REL,             /* ... or max|m - nu| / nu <= tol_rel (0: unused)                          */
    SDOT_OPT_MAXIT,
    SDOT_OPT_MAX_BACKTRACKS,
    SDOT_OPT_T_MIN,
    SDOT_OPT_MULT_OK,             /* the next trial starts from mult_ok * last accepted step                 */
    SDOT_OPT_RESIDUAL,            /* 0 lin, 1 log, 2 power                                                    */
    SDOT_OPT_POWER,
    SDOT_OPT_SWITCH,              /* log -> lin once max|m-nu|/nu <= switch                                   */
    SDOT_OPT_LIN_TOL,             /* relative residual of each linear solve                                  */
    SDOT_OPT_LIN_MAXIT,
    SDOT_OPT_KEEP_START,
    SDOT_OPT_CONTINUATION,        /* 0 never, 1 auto, 2 always                                                */
    SDOT_OPT_CONV_THRESHOLD,
    SDOT_OPT_CONV_S0,
    SDOT_OPT_CONV_RATIO,
    SDOT_OPT_CONV_MIN,
    SDOT_OPT_LIN_METHOD,          /* 0 Jacobi-PCG, 1 multigrid-PCG                                            */
    SDOT_OPT_PRECISION,           /* 0 FP64 clipping; 1 FP32 clipping + FP64 re-checks (2D; 3D: UNSUPPORTED) */
    SDOT_OPT_LIN_PRECISION,       /* 0 FP64 CG; 1 FP32 inner CG with FP64 iterative refinement                */
    SDOT_OPT_AGG_MARGIN,          /* aggregation of near-coincident seeds: merge a pair when c_ij ulp(w) margin  */
                                  /* > the tolerance (sdotplan/Aggregation.h); 0: off; the reference uses 4      */
    SDOT_OPT_STEP,                /* 0 trials (KMT backtracking); 1 limits (2D: the step brought under the limits */
                                  /* of the cells below the floor, sdotplan/Newton.h:330-366); 3D takes trials   */
    SDOT_NB_OPTIONS
};
#define SDOT_NB_STATS 31          /* the order of SdotPlanNd._STATS (SdotPlanNd.py:100-103)                  */
#define SDOT_NB_HIST 8            /* the order of SdotPlanNd._HISTORY (SdotPlanNd.py:105)                    */

typedef struct sdot_solve_desc {
    sdot_diagram_desc diagram;    /* positions, domain, density; `diagram.weights` = the start (NULL: zero)  */
    const double *nu;             /* [n] target masses (NULL: 1/n)                                            */
    double options[SDOT_NB_OPTIONS];
} sdot_solve_desc;

typedef struct sdot_solve_out {
    double *weights;              /* [n]                                                                     */
    double *masses;               /* [n]  the masses Newton measured at the fitted weights                   */
    double *barycentres;          /* [n, dim] (may be NULL)                                                  */
    double *cost;                 /* [1]  W2^2 = sum_i int_cell |x - p_i|^2 rho (may be NULL)               */
    double stats[SDOT_NB_STATS];  /* always host                                                             */
    double *history;              /* [cap_history, SDOT_NB_HIST] host (may be NULL)                          */
    int32_t cap_history;
    int32_t nb_history;           /* rows written                                                            */
    int32_t *clusters;            /* [n] (may be NULL, memory as `weights`): the smallest user index of each   */
                                  /* seed's cluster of near-coincident seeds, its own index if none             */
} sdot_solve_out;

/* One damped-Newton SDOT solve.  Replaces `sdot::gpu2d::solve<V,VD>(queue, pd, nu, w0, dups, options,
   weights, history, stats, cell_masses, barycenters, cost, clusters, ...)` (gpu/Newton2D.cuh:846-1888),
   bound by SdotPlanNd._build_card (SdotPlanNd.py:864-890), and the CPU `sdotplan::solve` (Solve.h:111-371). */
int32_t sdot_solve(sdot_context ctx, const sdot_solve_desc *desc, sdot_solve_out *out, sdot_status *st);

/* `count` independent solves advanced together: their cells, Laplacians and CG iterations share launches
   (block-diagonal batching).  Problems of both dimensions may be mixed.  Each `st[k]` reports solve k. */
int32_t sdot_solve_batch(sdot_context ctx, int32_t count, const sdot_solve_desc *descs, sdot_solve_out *outs, sdot_status *st);

/* The backward of the W2 loss of `batch` solved transports of `n` seeds each (device pointers, problem-major):
   grad_positions = g_b * 2 m_i (p_i - b_i) and grad_nu = g_b * (w_i - mean_b(w)) -- the envelope theorem at the fitted
   weights, the gradient in nu projected on sum(d nu) = 0.  `positions` / `grad_positions` / `grad_nu` are FP32 when
   `positions_fp32`, else FP64; either gradient may be NULL.  Enqueued on the context's stream, not waited for.
   Replaces the reference's envelope derivatives (SdotPlanNd.py:1037-1040, 1107-1122, `cost_and_position_grad`). */
int32_t sdot_w2_backward(sdot_context ctx, int32_t batch, int64_t n, int32_t dim, const void *positions, int32_t positions_fp32,
                         const double *masses, const double *barycentres, const double *weights, const double *grad_cost,
                         void *grad_positions, void *grad_nu, sdot_status *st);

/* ---- serving: continuous batching of solves ------------------------------------------------------------
 * A server owns a worker thread that advances every admitted solve one Newton step at a time.  Requests
 * submitted while others run are admitted at the next step boundary when the memory budget allows
 * (admission by the memory model of sdot_solve_bytes); finished solves leave at once.  Host arrays only:
 * the server copies a request's inputs at submission.  No counterpart in the reference (it has no serving
 * layer); `sdot_solve_bytes` restates CardMemory.card_solve_bytes (src/sdot/CardMemory.py:1-190). */
typedef struct sdot_server_s *sdot_server;

typedef struct sdot_server_config {
    int32_t device;
    uint64_t memory_budget;       /* bytes the admitted solves may hold together (0: 60% of free memory)      */
    int32_t max_active;           /* at most this many solves in flight (0: no limit)                         */
} sdot_server_config;

uint64_t sdot_solve_bytes(int32_t dim, int64_t n, const sdot_density *density);
int32_t sdot_server_create(const sdot_server_config *cfg, sdot_server *out, sdot_status *st);
/* copies the request; `*ticket` identifies it; never blocks on the GPU */
int32_t sdot_server_submit(sdot_server srv, const sdot_solve_desc *desc, int64_t *ticket, sdot_status *st);
/* 1 when the ticket's solve has finished (its outputs are then written into `out`, host arrays), 0 if not yet;
   `wait_ms` < 0 waits without limit */
int32_t sdot_server_poll(sdot_server srv, int64_t ticket, sdot_solve_out *out, int32_t wait_ms, sdot_status *st);
/* [0] admitted, [1] finished, [2] active now, [3] max active seen, [4] steps run, [5] kernel launches, [6] refused for memory */
int32_t sdot_server_counters(sdot_server srv, int64_t counters[8]);
void sdot_server_destroy(sdot_server srv);

#ifdef __cplusplus
}
#endif
#endif

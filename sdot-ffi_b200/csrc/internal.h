// Internal types shared by the host engine and the kernels of the B200 SDOT core.
//
// Layout in HBM (one "problem" = one diagram or one solve):
//   - seeds are RANKED in Morton order of the uniform grid cell that holds them (ties: user order), so a
//     rank range is a compact blob of space -- the neighbour search, the candidate loads and the
//     aggregation multigrid (rank >> k packets) all rely on it;
//   - positions are kept ranked, FP64, AoS `[n, dim]`; weights, masses and every Newton/CG vector are
//     FP64 `[n]` in rank order; `user[rank]` / `rank_of[user]` convert at the boundary;
//   - the grid is `g[0] x g[1] (x g[2])` cells of size `gh`, `cell_range[cell] = (first rank, last rank + 1)`
//     with cells numbered row-major (x fastest);
//   - facets are written per cell into a fixed-capacity neighbour table `[n, cap]` (rank ids, c_ij),
//     then mirrored into a bit-symmetric CSR by the "mutual" rule (laplacian kernels).
// Every kernel is batched: it takes an array of ProbDev and a table of chunks (problem, first rank, end rank),
// so one launch serves any mix of problems of one dimension (the serving batch, the batch of 64 gradients).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define SDOT_DEV __device__ __forceinline__

namespace sdot {

constexpr int CHUNK = 64;              // seeds per chunk (one block of the cell kernels)
// seeds per chunk of one problem's diagram: CHUNK for a large problem; for a small one fewer seeds per warp, so that its
// diagram still spreads over the 148 SMs (the warps the main cell kernels keep resident: 24 an SM in 2D, 16 in 3D).  A
// function of the problem alone, so that its report folds its chunks in the same order alone and in any batch
inline int cell_chunk( int dim, long n ) {
    const long resident = dim == 2 ? 148L * 24 : 148L * 16;
    const int warps = dim == 2 ? 8 : 4;                   // warps a block of k_cells2d / k_cells3d
    long per_warp = n / resident;
    per_warp = per_warp < 1 ? 1 : ( per_warp > CHUNK / warps ? CHUNK / warps : per_warp );
    return int( per_warp * warps );
}
constexpr int CAP2 = 32;               // neighbour table capacity per cell, 2D
constexpr int CAP3 = 64;               // ... 3D
constexpr int NB_REPORT = 12;          // doubles of the per-diagram report

enum DensKind : int { D_UNIFORM = 0, D_IMAGE = 1, D_GAUSS = 2 };

// what a diagram computes
enum DiagFlags : unsigned {
    F_MASS = 1u,            // masses (always cheap)
    F_FACETS = 2u,          // neighbour table (ids, c_ij)
    F_MEASURES = 4u,        // int_facet rho in the table
    F_MOMENTS = 8u,         // first moment and int |x - p|^2 rho
    F_REPORT = 16u,         // the Newton report (needs nu)
    F_USER_ORDER = 32u,     // write outputs at user index instead of rank
    F_VJP = 64u,            // adjoint gather (grad of masses)
    F_FP32 = 128u,          // FP32 clipping with FP64 re-check
    F_GATHER = 256u         // count the search's reads into ProbDev.gather (set with it)
};

constexpr int MAX_LEV = 24;      // levels of the weight majorants (grids up to 2^23 cells per side)
__host__ __device__ inline int lev_dim( int g, int l ) { return ( g + ( 1 << l ) - 1 ) >> l; }
// the moments of a node's seeds: n, sum p, sum w, sum p p^T (upper triangle), sum p w
__host__ __device__ inline int wmom_size( int dim ) { return dim == 2 ? 9 : 14; }

struct ProbDev {
    int dim, dkind, cap, n;
    int fp32;                     // 2D: the clip in FP32 with FP64 re-checks (precision "mixed"), the outputs in FP64
    double lo[3], hi[3];
    int g[3];
    double go[3], gh[3], ghmin;
    const int2 *cell_range;
    const double *pos;            // ranked [n, dim]
    const int *user;              // rank -> user
    const int *rank_of;           // user -> rank
    // density
    double rho;
    const double *dval;           // image values [nx * ny] (i along x) | gaussians [ng, dim + 2]
    const double *dpre;           // image: per row prefix of mass, [ny, nx + 1]
    int dn[3];
    double dorg[3], dstep[3];
    // this evaluation
    const double *w;              // ranked weights (NULL: zero)
    const unsigned long long *wmax_slot;   // -> ordered-integer max weight; NULL: 0
    double *mass;                 // [n]
    double *first;                // [n, dim] first moment about the seed, or barycentre if F_USER_ORDER
    double *cost;                 // [n]
    int *nb;                      // [n]
    int *nid;                     // [n, cap]
    double *nc;                   // [n, cap]
    double *nm;                   // [n, cap]
    const double *nu;             // [n] ranked targets (report)
    const double *gm;             // [n] cotangent of masses (vjp), ranked (NULL: none)
    const double *gf;             // [n, dim] cotangent of the first moments int_cell x rho, world frame (vjp; NULL: none)
    unsigned long long *gather;   // [NB_GATHER][32] the search's record reads (NULL: not counted), see count_reads
    double *gpos;                 // [n, dim] (vjp)
    double *gw;                   // [n] (vjp)
    double *report;               // [NB_REPORT] per problem (report)
    double *partials;             // [nchunks_of_problem, NB_REPORT]
    unsigned *counter;            // chunk counter for the last-block finalisation
    int chunk0, nchunk;           // this problem's chunks in the launch's table
    int res;                      // residual kind for the report (0 lin, 1 log, 2 power)
    double power;
    // the facets of the cells past `cap` (rank order only): nb[ row ] > cap, nid[ row * cap ] = offset in the store
    int *ovf_count;
    int ovf_cap;
    int *ovf_ids;
    double *ovf_c;
    // weight majorants w_j <= a . p_j + b of the seeds of each grid cell (level 0), then of each 2^l block of cells
    // (level l, dims lev_dim( g, l )), up to one block: records [ a[ dim ], b as an ordered integer ] at
    // wpyr + ( dim + 1 ) ( poff[ l ] + node ); b = -1e300: no seed.  NULL: the global max bounds the search
    double *wpyr;
    double *wmom;                 // [ nodes, wmom_size( dim ) ] the moments the slopes are fitted from
    double *perr;                 // set to 1 when a cell of this problem exceeds every capacity (NULL: none)
    double *prefuse;              // a trial diagram: set to 1 instead when a cell exceeds the big-cell pass (NULL: not a trial)
    int nlev;
    int poff[ MAX_LEV ];
};

// THE LIMITS STEP (2D; sdotplan/Bounds.h:1-40, gpu/Newton2D.cuh:538-776): for each cell of a trial diagram below the
// mass floor, the first step along the Newton direction where its mass falls below the floor, the cell computed alone
// from the neighbours it has in the accepted and in the trial diagram
struct LimDev {
    ProbDev P;                    // geometry and density; P.w the accepted weights (ranked)
    const double *d;              // the Newton direction (ranked)
    const double *a2;             // the trial's masses (ranked)
    const int *nb0, *nid0;        // the accepted diagram's neighbour table
    const int *nb1, *nid1;        // the trial's
    double eps, t;                // the mass floor, the trial step (the horizon of the search)
    double *out;                  // [0] the cells below the floor, [1] the smallest limit (ordered integer, atomic min)
};

// cells the warp-register kernel could not hold (more than 32 vertices, or more facets than the table's row):
// queued here and rebuilt by the global-memory kernel
struct OvfItem { int prob; int seed; };
struct OvfList {
    int count, cap;
    OvfItem *items;
};
constexpr int VBIG = 4096;       // vertices of a cell in the global-memory pass

struct Chunk {
    int prob;      // index into the launch's ProbDev array
    int begin;     // first rank
    int end;       // end rank
    int index;     // chunk index within its problem
};

// device-side error record (first error wins)
struct ErrRec {
    int code;      // 0 none, 4 capacity
    int kind;
    int prob;
    int seed;      // user index
    int needed;
};

// report layout (per problem, after a diagram with F_REPORT)
enum Report : int {
    R_WORST = 0, R_WORST_REL, R_AMIN, R_ASUM, R_LIN2, R_GCOUNT, R_GMEAN, R_GM2, R_SU, R_SUG, R_NUSUM, R_NEMPTY
};

// per-problem view for the Laplacian, CG and Newton vector kernels
struct VecDev {
    int n, cap, rank0, res;
    double power;
    // the neighbour table of the accepted diagram -> CSR (row_ptr local to the problem)
    const int *nb;
    const int *nid;
    const double *nc;
    const int *ovf_ids;           // the facets of the rows past `cap` (see ProbDev)
    const double *ovf_c;
    int *row_ptr;                 // [n + 1]
    int *col;                     // [n * cap]
    double *val;                  // [n * cap]  c_ij > 0 (the matrix holds -c_ij)
    double *dia;                  // [n]
    int *rowcnt;                  // [n] scratch
    // vectors (ranked)
    double *x, *r, *z, *p, *q, *b;
    const double *nu, *a;
    double *w, *w2, *d;
    double t;                     // the trial step of this launch
    double tol;                   // relative residual of the CG
    int maxit;                    // CG iterations at most
    const double *report;         // the Newton report of the accepted diagram (rhs)
    unsigned long long *wmax_slot;   // ordered-integer max of the trial weights
    double *sc;                   // [NB_SC] scalars of the problem
    double *partials;             // [nchunk * 4]
    unsigned *counter;
    int chunk0, nchunk;
    int active;
    int precond;                  // 0 Jacobi, 1 multigrid (the V-cycle writes z)
    // lin_precision 1: the inner CG on FP32 copies (matrix values, diagonal, e = x32, r32, z32, p32, q32); x, r, b stay FP64
    int mixed;
    float *val32, *dia32, *x32, *r32, *z32, *p32, *q32;
    // the detection of near-coincident pairs on this Laplacian (NULL: off): the pairs (i < j, ranks) whose facet the
    // doubles of the weights cannot place within the tolerance, c_ij ulp( max |w| ) margin > tau
    int2 *agg_pairs;
    int agg_cap;
    double *agg_count;
    double agg_margin, agg_tol_abs, agg_tol_rel;
    double agg_ccond;             // a coupling past this is merged whatever the weights (1e9 times the scale of a facet)
};
// one level of the multigrid preconditioner of one problem (mg.cu)
constexpr int MG_BOTTOM = 32;          // the coarsest level has at most this many rows (dense inverse)
constexpr int MG_MAX_LEVELS = 12;
struct MgLevel {
    int level, vec;                    // level index; the problem's index in the CG batch's VecDev array
    int n, pack, nn;                   // rows of this level, aggregate size, rows of the next level
    const int *rp, *col;               // this level's CSR (level 0: the Newton CSR's)
    float *val, *dia, *dinv;
    float *b, *x, *y;                  // rhs, pre-smoothed x, post-smoothed y (level 0 writes z instead)
    float *bn;                         // the next level's rhs
    const float *xn;                   // the next level's solution (its y)
    int *rcn, *rpn, *coln;             // the next level's CSR, being built
    float *valn, *dian, *dinvn;
    double *part;                      // [nchunk * 2] chunk totals and offsets of the build
    int nchunk;
    int capn;                          // entries the next level's col / val can hold
    float *inv;                        // the coarsest level: dense inverse [n * n]
};

enum Scalar : int { SC_RZ = 0, SC_ALPHA, SC_BETA, SC_BNORM, SC_RNORM, SC_CONV, SC_ITER, SC_MEAN, SC_C, SC_TOL, SC_PQ, SC_FAIL, SC_NNZ,
                    SC_REFINE,      // mixed CG: 1 once the inner FP32 CG has converged (x += e, then the FP64 residual)
                    SC_IN0,         // mixed CG: the inner CG's starting residual norm
                    SC_RPREV,       // mixed CG: the FP64 residual norm of the last refinement
                    SC_NREF,        // mixed CG: refinements so far
                    NB_SC };
constexpr int VCHUNK = 256;      // rows per chunk of the vector kernels (one block each: many blocks keep loads in flight)
// rows per chunk of one problem's vector kernels: VCHUNK for a large problem, fewer for a small one so that its CG still
// spreads over the 148 SMs.  A function of the problem alone: its reductions fold in the same order alone and in any batch
inline int vec_chunk( long n ) { return n >= 148L * 2 * VCHUNK ? VCHUNK : ( n >= 148L * VCHUNK ? VCHUNK / 2 : VCHUNK / 4 ); }
constexpr int MG_FUSE_ROWS = 4096;   // multigrid levels of at most this many rows run in one launch per problem (k_mg_fused)

// ---- the search's reads, counted on request: the gather model of the cell kernels' traffic ------------------------
// candidate seed records (position + weight), grid cells whose weight majorant was read, grid cells whose seed range
// was read, pyramid node records (affine majorant); spread over 32 slots by block so the atomics do not queue on one word
enum { G_CAND = 0, G_GRID, G_RANGE, G_NODE, NB_GATHER };
constexpr int GATHER_SLOTS = 32;
// `n` reads of kind `what` for the current cell: called by every lane of the warp, counted once
SDOT_DEV void count_reads( const ProbDev &P, int lane, int what, unsigned n ) {
    if ( lane == 0 && n ) atomicAdd( P.gather + what * GATHER_SLOTS + ( blockIdx.x & ( GATHER_SLOTS - 1 ) ), ( unsigned long long ) n );
}

// ---- warp helpers ------------------------------------------------------------------------------------
SDOT_DEV double warp_sum( double v ) {
#pragma unroll
    for ( int o = 16; o > 0; o >>= 1 ) v += __shfl_xor_sync( 0xffffffffu, v, o );
    return v;
}
SDOT_DEV double warp_max( double v ) {
#pragma unroll
    for ( int o = 16; o > 0; o >>= 1 ) v = fmax( v, __shfl_xor_sync( 0xffffffffu, v, o ) );
    return v;
}
SDOT_DEV double warp_min( double v ) {
#pragma unroll
    for ( int o = 16; o > 0; o >>= 1 ) v = fmin( v, __shfl_xor_sync( 0xffffffffu, v, o ) );
    return v;
}
SDOT_DEV int lane_id() { return threadIdx.x & 31; }

// ordered-integer image of a double, for exact atomic max
SDOT_DEV unsigned long long dbl_order( double x ) {
    unsigned long long u = __double_as_longlong( x );
    return ( u >> 63 ) ? ~u : ( u | 0x8000000000000000ull );
}
SDOT_DEV double order_dbl( unsigned long long u ) {
    return __longlong_as_double( ( u >> 63 ) ? ( u & 0x7fffffffffffffffull ) : ~u );
}

// accumulators of the Newton report of a warp, a chunk or a problem (Chan's parallel combination for the mean / M2
// of g); combined in a fixed order, so that a report is bitwise reproducible
struct Rep {
    double v[ NB_REPORT ];
    SDOT_DEV void init() {
        v[ R_WORST ] = 0; v[ R_WORST_REL ] = 0; v[ R_AMIN ] = 1e300; v[ R_ASUM ] = 0; v[ R_LIN2 ] = 0;
        v[ R_GCOUNT ] = 0; v[ R_GMEAN ] = 0; v[ R_GM2 ] = 0; v[ R_SU ] = 0; v[ R_SUG ] = 0; v[ R_NUSUM ] = 0; v[ R_NEMPTY ] = 0;
    }
    SDOT_DEV void combine( const double *o ) {   // Chan's parallel combination for the mean / M2 of g
        v[ R_WORST ] = fmax( v[ R_WORST ], o[ R_WORST ] );
        v[ R_WORST_REL ] = fmax( v[ R_WORST_REL ], o[ R_WORST_REL ] );
        v[ R_AMIN ] = fmin( v[ R_AMIN ], o[ R_AMIN ] );
        v[ R_ASUM ] += o[ R_ASUM ];
        v[ R_LIN2 ] += o[ R_LIN2 ];
        double na = v[ R_GCOUNT ], nb = o[ R_GCOUNT ], n = na + nb;
        if ( nb > 0 ) {
            double d = o[ R_GMEAN ] - v[ R_GMEAN ];
            v[ R_GMEAN ] += d * nb / n;
            v[ R_GM2 ] += o[ R_GM2 ] + d * d * na * nb / n;
            v[ R_GCOUNT ] = n;
        }
        v[ R_SU ] += o[ R_SU ];
        v[ R_SUG ] += o[ R_SUG ];
        v[ R_NUSUM ] += o[ R_NUSUM ];
        v[ R_NEMPTY ] += o[ R_NEMPTY ];
    }
};

// the last block of a problem folds its chunks' reports: thread t the chunks t, t + blockDim, ... in order, then the
// lanes of each warp by a shuffle tree, then the warps in order -- a fixed tree, whatever the scheduling. Every thread
// of the block calls it (blockDim a multiple of 32); the result goes to P.report and the problem's counter is reset
// (NW: the warps of the block at most -- the fold's shared memory counts against the cell kernels' occupancy)
template<int NW>
__device__ __forceinline__ void fold_reports_block( const ProbDev &P ) {
    __shared__ double sh_fold[ NW ][ NB_REPORT ];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = int( blockDim.x >> 5 );
    Rep r;
    r.init();
    for ( int c = threadIdx.x; c < P.nchunk; c += blockDim.x ) {
        double o[ NB_REPORT ];
        const volatile double *src = P.partials + ( size_t ) c * NB_REPORT;
        for ( int k = 0; k < NB_REPORT; ++k ) o[ k ] = src[ k ];
        r.combine( o );
    }
    for ( int off = 16; off > 0; off >>= 1 ) {
        double o[ NB_REPORT ];
        for ( int k = 0; k < NB_REPORT; ++k ) o[ k ] = __shfl_down_sync( 0xffffffffu, r.v[ k ], off );
        if ( lane < off ) r.combine( o );
    }
    if ( lane == 0 )
        for ( int k = 0; k < NB_REPORT; ++k ) sh_fold[ warp ][ k ] = r.v[ k ];
    __syncthreads();
    if ( threadIdx.x == 0 ) {
        Rep f;
        f.init();
        for ( int w = 0; w < nw; ++w ) f.combine( sh_fold[ w ] );
        for ( int k = 0; k < NB_REPORT; ++k ) P.report[ k ] = f.v[ k ];
        *P.counter = 0;
    }
}

// ---- weight majorants -------------------------------------------------------------------------------------------------
// b of majorant record `node` (the grid's own cells are nodes 0 .. ncell - 1, with a = 0: b is their max weight)
SDOT_DEV double wmaj_b( const ProbDev &P, size_t node ) {
    return order_dbl( reinterpret_cast<const unsigned long long *>( P.wpyr )[ node * ( P.dim + 1 ) + P.dim ] );
}
// may a seed of a node with majorant w <= a . q + b, q in the box [ lo, hi ], claim the point X = p_i + v of seed i's
// cell?  Its power distance there is at least min_q |X - q|^2 - a . q - b = dist^2( X + a/2, box ) - a . X - |a|^2/4 - b,
// against |v|^2 - w_i for seed i (with a margin of rounding)
// (rel: the margin, relative to the terms; larger for a vertex held in FP32)
SDOT_DEV bool wmaj_claims( const double *a, double b, const double *lo, const double *hi, const double *X, const double *v, int dim, double wi,
                           double rel = 1e-12 ) {
    double d2 = 0, aX = 0, a2 = 0, v2 = 0;
    for ( int q = 0; q < dim; ++q ) {
        double u = X[ q ] + 0.5 * a[ q ];
        double d = fmax( 0.0, fmax( lo[ q ] - u, u - hi[ q ] ) );
        d2 += d * d;
        aX += a[ q ] * X[ q ];
        a2 += a[ q ] * a[ q ];
        v2 += v[ q ] * v[ q ];
    }
    double lhs = d2 - aX - 0.25 * a2 - b, rhs = v2 - wi;
    return lhs < rhs + rel * ( fabs( aX ) + fabs( b ) + fabs( wi ) + v2 + d2 );
}

// ---- launchers (each in the .cu next to its kernels) --------------------------------------------------
// CUDA-event timing per kernel class (off by default; `sdot_context_set_timing`)
enum KClass : int { K_CELLS2D = 0, K_CELLS3D, K_LAPLACIAN, K_CG, K_VECTOR, K_INDEX, K_REPORT, K_MULTIGRID, NB_KCLASS };
struct Timer {
    bool on = false;
    struct Rec { int kind; cudaEvent_t a, b; double units; };
    Rec *pending = nullptr;
    int npending = 0, cap = 0;
    cudaEvent_t *pool = nullptr;
    int npool = 0, cappool = 0;
    double ms[ NB_KCLASS ] = {}, units[ NB_KCLASS ] = {};
    unsigned long long count[ NB_KCLASS ] = {};
    int open_kind = -1;
    double open_units = 0;
    cudaEvent_t open_a = nullptr;
    void begin( cudaStream_t s, int kind, double units );
    void end( cudaStream_t s, unsigned long long launches = 1 );
    void resolve();
    void release();
};

struct Launch {
    cudaStream_t stream;
    unsigned long long *launches;   // incremented per kernel launched
    Timer *timer = nullptr;
};

// index.cu
void launch_bbox( const Launch &L, const double *pos, int n, int dim, unsigned long long *mm /* [2*dim] */ );
void launch_keys( const Launch &L, const double *pos, int n, int dim, const int *g, const double *go, const double *gh, int bits,
                  unsigned long long *keys, int *vals );
void launch_gather( const Launch &L, const double *pos, const int *vals, int n, int dim, double *pos_ranked, int *user, int *rank_of,
                    const double *w_user, double *w_ranked );
void launch_cell_ranges( const Launch &L, const unsigned long long *keys, const double *pos_ranked, int n, int dim, const int *g,
                         const double *go, const double *gh, int2 *cell_range );
size_t radix_temp_bytes( int n, int bits );
void radix_sort( const Launch &L, void *temp, size_t temp_bytes, const unsigned long long *kin, unsigned long long *kout, const int *vin,
                 int *vout, int n, int bits );
void launch_image_prefix( const Launch &L, const double *values, int nx, int ny, double hx, double *pre );
// one axis of the separable gaussian blur of an image [nx, ny] (i along x, j contiguous): taps ker[ 0 .. 2r ],
// renormalised by the taps that fall inside the axis
void launch_blur_axis( const Launch &L, const double *src, double *dst, int nx, int ny, int axis, int r, const double *ker );
void launch_wmax( const Launch &L, const double *w, int n, unsigned long long *slot );
// the levels of the weight majorants of a grid: returns the doubles they take, fills nlev and poff
long wpyr_layout( int dim, const int *g, int &nlev, int *poff );
// (re)builds the weight majorants of every problem of `probs` (those with wpyr) from their current weights
void launch_wpyr( const Launch &L, const ProbDev *probs, int nprob );
void launch_finish_wmax( const Launch &L, unsigned long long *slot, double *wmax, int count );

// linalg.cu
void launch_lap_count( const Launch &L, const VecDev *v, const Chunk *ch, int nch );
void launch_lap_scan( const Launch &L, const VecDev *v, int nprob );
void launch_lap_fill( const Launch &L, const VecDev *v, const Chunk *ch, int nch );
void launch_rhs( const Launch &L, const VecDev *v, const Chunk *ch, int nch );
void launch_cg_init( const Launch &L, const VecDev *v, const Chunk *ch, int nch );
void launch_cg_iter( const Launch &L, const VecDev *v, const Chunk *ch, int nch );
void launch_gauge( const Launch &L, const VecDev *v, const Chunk *ch, int nch );
// the re-splitting's trial weights: w2 = w - shift, then w2[ idx[ t ] ] += val[ t ] (idx distinct)
void launch_polish_weights( const Launch &L, const double *w, double *w2, int n, double shift, const int *idx, const double *val, int k );
// the pairs the aggregation merges (VecDev.agg_*)
void launch_agg_detect( const Launch &L, const VecDev *v, const Chunk *ch, int nch );
// the direction with clusters: their internal couplings capped at `cap` in the CSR the CG solves (the true ones kept in
// `blk`, [ members ][ AGG_KMAX + 1 ]), then after the solve the members tied and the split corrected by the true local
// systems (`y`: [ members ] scratch); `cl` = [ begins (ncl + 1) | members ]
constexpr int AGG_KMAX = 16;
void launch_agg_cap( const Launch &L, const int *row_ptr, const int *col, double *val, double *dia, const int *cl, int ncl, double cap, double *blk );
void launch_agg_direction( const Launch &L, const int *row_ptr, const int *col, const double *val, const int *cl, int ncl, const double *blk,
                           const double *nu, const double *b, double *x, double *y );
// the cluster shares of the masses: ae[ i ] = nu[ i ] a_C / nu_C for the members i of each cluster C (others untouched)
void launch_agg_shares( const Launch &L, const double *a, const double *nu, const int *cl_begin, const int *cl_members, int ncl, double *ae );
// the multigrid-preconditioned CG: init in two halves around the first V-cycle, then per iteration
// spmv -> update -> V-cycle -> r.z -> p
void launch_cg_init0( const Launch &L, const VecDev *v, const Chunk *ch, int nch );
void launch_cg_init1( const Launch &L, const VecDev *v, const Chunk *ch, int nch );
void launch_cg_spmv_update( const Launch &L, const VecDev *v, const Chunk *ch, int nch );
void launch_cg_rz_p( const Launch &L, const VecDev *v, const Chunk *ch, int nch );
// the mixed CG (FP32 inner CG, FP64 iterative refinement): the same sequence of launches as the FP64 CG
void launch_mx_init( const Launch &L, const VecDev *v, const Chunk *ch, int nch );          // (Jacobi) or before the first V-cycle (multigrid)
void launch_mx_init1( const Launch &L, const VecDev *v, const Chunk *ch, int nch );         // (multigrid) after the first V-cycle
void launch_mx_iter( const Launch &L, const VecDev *v, const Chunk *ch, int nch );          // (Jacobi) one iteration
void launch_mx_spmv_update( const Launch &L, const VecDev *v, const Chunk *ch, int nch );   // (multigrid) before the V-cycle
void launch_mx_rz_p( const Launch &L, const VecDev *v, const Chunk *ch, int nch );          // (multigrid) after the V-cycle
// mg.cu
void launch_mg_level0( const Launch &L, const MgLevel *lv, const VecDev *vs, const Chunk *ch, int nch );
void launch_mg_coarsen( const Launch &L, const MgLevel *lv, int nprob, const Chunk *ch, int nch, ErrRec *err );
void launch_mg_bottom_build( const Launch &L, const MgLevel *lv, int nprob );
void launch_mg_down( const Launch &L, const MgLevel *lv, const VecDev *vs, const Chunk *ch, int nch );
void launch_mg_bottom( const Launch &L, const MgLevel *lv, const VecDev *vs, int nprob );
void launch_mg_up( const Launch &L, const MgLevel *lv, const VecDev *vs, const Chunk *ch, int nch );
// the levels of at most MG_FUSE_ROWS rows of each problem, down, bottom and up, one block per problem: chain holds those
// levels of every problem, idx[ p ] = ( first, count )
void launch_mg_fused( const Launch &L, const MgLevel *chain, const int2 *idx, const VecDev *vs, int nprob );
void launch_trial( const Launch &L, const VecDev *v, const Chunk *ch, int nch );

// cells2d.cu / cells3d.cu
// the limits of the cells below the floor (one thread a cell; chunks of CHUNK cells over the LimDev array)
void launch_limits2d( const Launch &L, const LimDev *lims, const Chunk *chunks, int nchunks );
// clips: bit 0 the problems that clip in FP64, bit 1 those that clip in FP32 (ProbDev.fp32): one launch each
void launch_cells2d( const Launch &L, const ProbDev *probs, const Chunk *chunks, int nchunks, unsigned flags, ErrRec *err, OvfList *ovf,
                     int clips = 1 );
// the queued big cells (count known on the host), polygons in `scratch` (VBIG vertices x 2 buffers per warp)
void launch_cells2d_big( const Launch &L, const ProbDev *probs, const OvfList *ovf, int count, unsigned flags, ErrRec *err, char *scratch,
                         int warps );
size_t big_scratch_bytes( int warps );
void launch_report( const Launch &L, const ProbDev *probs, const Chunk *chunks, int nchunks );
void launch_scale( const Launch &L, double *v, int n, double s );
void launch_scatter( const Launch &L, const double *ranked, const int *user, int n, int dim, double *out_user );
void launch_gather_vec( const Launch &L, const double *user_vals, const int *user, int n, double *ranked, double scale );
// the clipped cells of the gaussian problems between the two passes of the 3D main kernel (cells3d.cu)
struct Split3 {
    char *mem;                        // the records
    unsigned long long *used;         // bytes taken (zeroed before pass 1)
    unsigned long long cap;           // bytes of `mem`
    long long *slot;                  // [ chunk of the launch ][ CHUNK ]: a cell's record offset; -1 none (pass 2 does it whole), -2 queued
};
// sp NULL: one pass; else two passes for the gaussian problems (sp->slot holds nchunks * CHUNK entries)
void launch_cells3d( const Launch &L, const ProbDev *probs, const Chunk *chunks, int nchunks, unsigned flags, ErrRec *err, OvfList *ovf,
                     const Split3 *sp = nullptr );
// the queued 3D cells (past the warp cell's capacities) rebuilt one warp a block with larger capacities
void launch_cells3d_big( const Launch &L, const ProbDev *probs, const OvfList *ovf, int count, unsigned flags, ErrRec *err, OvfList *next );
// the 3D cells past the big pass's capacities (queued on its `next`), each warp's cell in a slot of `scratch`
size_t giant3_slot_bytes();
void launch_cells3d_giant( const Launch &L, const ProbDev *probs, const OvfList *list, int count, unsigned flags, ErrRec *err, char *scratch,
                           int slots );

} // namespace sdot

// The Newton Hessian and its solve, batched over problems (block-diagonal).
//
// CSR assembly (the reference: gpu/Laplacian2D.cuh:139-297, sdotplan/Laplacian.h:37-62).  Each cell wrote
// its facets into a fixed-capacity table.  An entry (i, j) enters the CSR when BOTH cells saw the facet
// (the "mutual" rule), with the value measured by the cell of the smaller rank: the matrix is symmetric
// to the bit, a facet seen by one side only (a sliver below rounding) is dropped on both, and the rows
// come out in table order, which is deterministic.  `dia` = the row sum, 1 for an empty row.
//
// CG: preconditioned by the diagonal, FP64, one chunk of VCHUNK rows per block.  Every reduction is a
// fixed tree inside the block, then a fixed-tree fold of the chunk partials by the last block of the problem to
// finish (a counter per problem): bitwise reproducible whatever the scheduling, the reference's requirement too
// (gpu/Reduce.cuh:3-20, gpu/Linear2D.cuh:39-41).
#include "internal.h"
#include <cub/block/block_scan.cuh>

namespace sdot {

constexpr int VT = 256;                       // threads per block of the vector kernels
constexpr int VPT = VCHUNK / VT;              // rows per thread

// deterministic block sum of NV values; thread 0 gets the result
template<int NV>
__device__ __forceinline__ void block_sum( double ( &v )[ NV ] ) {
    __shared__ double sh[ VT / 32 ][ NV ];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for ( int k = 0; k < NV; ++k ) v[ k ] = warp_sum( v[ k ] );
    if ( lane == 0 )
#pragma unroll
        for ( int k = 0; k < NV; ++k ) sh[ warp ][ k ] = v[ k ];
    __syncthreads();
    if ( threadIdx.x == 0 )
#pragma unroll
        for ( int k = 0; k < NV; ++k ) {
            double s = 0;
            for ( int w = 0; w < VT / 32; ++w ) s += sh[ w ][ k ];
            v[ k ] = s;
        }
    __syncthreads();
}

// thread 0 of the chunk writes its partials; the last block of the problem folds them -- thread t the chunks t, t + VT,
// ... in order, then the block's fixed tree -- and returns true in its thread 0, which then holds the sums in `tot`
template<int NV>
__device__ __forceinline__ bool fold_last( const VecDev &V, const Chunk &ch, const double ( &v )[ NV ], double ( &tot )[ NV ] ) {
    __shared__ int last;
    if ( threadIdx.x == 0 ) {
        double *dst = V.partials + ( size_t ) ch.index * 4;
#pragma unroll
        for ( int k = 0; k < NV; ++k ) dst[ k ] = v[ k ];
        __threadfence();
        unsigned prev = atomicAdd( V.counter, 1u );
        last = prev == unsigned( V.nchunk - 1 );
    }
    __syncthreads();
    if ( ! last ) return false;
    __threadfence();
    double acc[ NV ];
#pragma unroll
    for ( int k = 0; k < NV; ++k ) acc[ k ] = 0;
    for ( int c = threadIdx.x; c < V.nchunk; c += VT ) {
        const volatile double *src = V.partials + ( size_t ) c * 4;
#pragma unroll
        for ( int k = 0; k < NV; ++k ) acc[ k ] += src[ k ];
    }
    block_sum<NV>( acc );
    if ( threadIdx.x != 0 ) return false;
#pragma unroll
    for ( int k = 0; k < NV; ++k ) tot[ k ] = acc[ k ];
    *V.counter = 0;
    return true;
}

// ---- CSR -------------------------------------------------------------------------------------------------------
// the facets of a row: its table row, or its slice of the overflow store when it has more than `cap`
__device__ __forceinline__ const int *row_ids( const VecDev &V, int row, int nb ) {
    return nb > V.cap ? V.ovf_ids + V.nid[ ( size_t ) row * V.cap ] : V.nid + ( size_t ) row * V.cap;
}
__device__ __forceinline__ const double *row_cs( const VecDev &V, int row, int nb ) {
    return nb > V.cap ? V.ovf_c + V.nid[ ( size_t ) row * V.cap ] : V.nc + ( size_t ) row * V.cap;
}

__device__ __forceinline__ int find_in_row( const VecDev &V, int row, int key ) {
    const int nb = V.nb[ row ];
    const int *ids = row_ids( V, row, nb );
    for ( int l = 0; l < nb; ++l ) if ( ids[ l ] == key ) return l;
    return -1;
}

__global__ void __launch_bounds__( VT ) k_lap_count( const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks, int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const VecDev &V = vs[ ch.prob ];
    double tot = 0;
    for ( int row = ch.begin + threadIdx.x; row < ch.end; row += VT ) {
        int cnt = 0;
        const int nb = V.nb[ row ];
        const int *ids = row_ids( V, row, nb );
        for ( int k = 0; k < nb; ++k ) cnt += find_in_row( V, ids[ k ], row ) >= 0;
        V.rowcnt[ row ] = cnt;
        tot += cnt;
    }
    double v[ 1 ] = { tot };
    block_sum<1>( v );
    if ( threadIdx.x == 0 ) V.partials[ ( size_t ) ch.index * 4 ] = v[ 0 ];
}

void launch_lap_count( const Launch &L, const VecDev *v, const Chunk *ch, int nch ) {
    if ( nch <= 0 ) return;
    k_lap_count<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    ++*L.launches;
}

// one block per problem: exclusive scan of the chunk totals, in place
__global__ void __launch_bounds__( 1024 ) k_lap_scan( const VecDev *__restrict__ vs ) {
    const VecDev &V = vs[ blockIdx.x ];
    if ( ! V.active ) return;
    typedef cub::BlockScan<long long, 1024> Scan;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ long long carry;
    if ( threadIdx.x == 0 ) carry = 0;
    __syncthreads();
    for ( int base = 0; base < V.nchunk; base += 1024 ) {
        int c = base + threadIdx.x;
        long long x = c < V.nchunk ? ( long long ) V.partials[ ( size_t ) c * 4 ] : 0, ex, agg;
        Scan( tmp ).ExclusiveSum( x, ex, agg );
        if ( c < V.nchunk ) V.partials[ ( size_t ) c * 4 + 1 ] = double( carry + ex );
        __syncthreads();
        if ( threadIdx.x == 0 ) carry += agg;
        __syncthreads();
    }
    if ( threadIdx.x == 0 ) {
        V.sc[ SC_NNZ ] = double( carry );
        V.row_ptr[ V.n ] = carry > ( long long ) V.n * V.cap ? 0 : int( carry );   // past the capacity: empty rows, CG fails
    }
}

void launch_lap_scan( const Launch &L, const VecDev *v, int nprob ) {
    if ( nprob <= 0 ) return;
    k_lap_scan<<<nprob, 1024, 0, L.stream>>>( v );
    ++*L.launches;
}

__global__ void __launch_bounds__( VT ) k_lap_fill( const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks, int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const VecDev &V = vs[ ch.prob ];
    typedef cub::BlockScan<int, VT> Scan;
    __shared__ typename Scan::TempStorage tmp;
    const int r0 = ch.begin + threadIdx.x * VPT;
    int cnt[ VPT ], loc = 0;
#pragma unroll
    for ( int q = 0; q < VPT; ++q ) { int row = r0 + q; cnt[ q ] = row < ch.end ? V.rowcnt[ row ] : 0; loc += cnt[ q ]; }
    int ex;
    Scan( tmp ).ExclusiveSum( loc, ex );
    if ( V.sc[ SC_NNZ ] > double( V.n ) * V.cap ) {                // past the CSR's capacity: empty rows (k_lap_scan)
        for ( int q = 0; q < VPT && r0 + q < ch.end; ++q ) { V.row_ptr[ r0 + q ] = 0; V.dia[ r0 + q ] = 1.0; }
        return;
    }
    int at = int( V.partials[ ( size_t ) ch.index * 4 + 1 ] ) + ex;
#pragma unroll
    for ( int q = 0; q < VPT; ++q ) {
        int row = r0 + q;
        if ( row >= ch.end ) break;
        V.row_ptr[ row ] = at;
        double s = 0;
        const int nb = V.nb[ row ];
        const int *ids = row_ids( V, row, nb );
        const double *cs = row_cs( V, row, nb );
        for ( int k = 0; k < nb; ++k ) {
            int j = ids[ k ];
            int l = find_in_row( V, j, row );
            if ( l < 0 ) continue;
            double c = row < j ? cs[ k ] : row_cs( V, j, V.nb[ j ] )[ l ];
            V.col[ at ] = j;
            V.val[ at ] = c;
            s += c;
            ++at;
        }
        V.dia[ row ] = s > 0 ? s : 1.0;
    }
}

void launch_lap_fill( const Launch &L, const VecDev *v, const Chunk *ch, int nch ) {
    if ( nch <= 0 ) return;
    k_lap_fill<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    ++*L.launches;
}

// ---- Newton right-hand side (sdotplan/Newton.h:178-203), then projected on the range of L ------------------------
__device__ __forceinline__ double g_of( double x, int r, double p ) {
    x = fmax( x, 1e-300 );
    if ( r == 2 ) return p == 0 ? log( x ) : ( pow( x, p ) - 1 ) / p;
    return r == 1 ? log( x ) : x - 1;
}
__device__ __forceinline__ double gp_of( double x, int r, double p ) {
    x = fmax( x, 1e-300 );
    if ( r == 2 ) return pow( x, p - 1 );
    return r == 1 ? 1 / x : 1;
}

__global__ void __launch_bounds__( VT ) k_rhs( const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks, int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const VecDev &V = vs[ ch.prob ];
    if ( ! V.active ) return;
    const double c = V.res == 0 ? 0.0 : V.report[ R_SUG ] / V.report[ R_SU ];
    double s = 0;
    for ( int i = ch.begin + threadIdx.x; i < ch.end; i += VT ) {
        double nu = V.nu[ i ], a = V.a[ i ], b;
        if ( V.res == 0 ) b = nu > 0 ? nu - a : 0.0;
        else {
            double x = a / nu;
            b = nu > 0 ? nu / gp_of( x, V.res, V.power ) * ( c - g_of( x, V.res, V.power ) ) : 0.0;
        }
        V.b[ i ] = b;
        s += b;
    }
    double v[ 1 ] = { s }, tot[ 1 ];
    block_sum<1>( v );
    if ( fold_last<1>( V, ch, v, tot ) ) V.sc[ SC_MEAN ] = tot[ 0 ] / V.n;
}

void launch_rhs( const Launch &L, const VecDev *v, const Chunk *ch, int nch ) {
    if ( nch <= 0 ) return;
    k_rhs<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    ++*L.launches;
}

// ---- CG --------------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__( VT ) k_cg_init( const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks, int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const VecDev &V = vs[ ch.prob ];
    if ( ! V.active ) return;
    const double mean = V.sc[ SC_MEAN ];
    double rz = 0, bb = 0;
    for ( int i = ch.begin + threadIdx.x; i < ch.end; i += VT ) {
        double b = V.b[ i ] - mean;
        V.b[ i ] = b;
        V.x[ i ] = 0;
        V.r[ i ] = b;
        double z = b / V.dia[ i ];
        V.z[ i ] = z;
        V.p[ i ] = z;
        rz += b * z;
        bb += b * b;
    }
    double v[ 2 ] = { rz, bb }, tot[ 2 ];
    block_sum<2>( v );
    if ( fold_last<2>( V, ch, v, tot ) ) {
        V.sc[ SC_RZ ] = tot[ 0 ];
        V.sc[ SC_BNORM ] = sqrt( tot[ 1 ] );
        V.sc[ SC_RNORM ] = sqrt( tot[ 1 ] );
        V.sc[ SC_ITER ] = 0;
        V.sc[ SC_FAIL ] = 0;
        V.sc[ SC_CONV ] = tot[ 1 ] == 0 ? 1.0 : 0.0;
        if ( V.sc[ SC_NNZ ] > double( V.n ) * V.cap ) { V.sc[ SC_FAIL ] = 1; V.sc[ SC_CONV ] = 2; }
    }
}

// q = L p: LPR lanes per row (the reference's `lanes`, gpu/Linear2D.cuh:96), each lane every LPR-th entry of the row,
// the lanes' sums folded by a fixed shuffle tree -- independent loads in flight, deterministic sums
constexpr int LPR = 4;
__device__ __forceinline__ double row_dot_lanes( const VecDev &V, int i, int sub, const double *__restrict__ x ) {
    double t = 0;
    const int e1 = V.row_ptr[ i + 1 ];
    for ( int e = V.row_ptr[ i ] + sub; e < e1; e += LPR ) t += V.val[ e ] * x[ V.col[ e ] ];
#pragma unroll
    for ( int o = 1; o < LPR; o <<= 1 ) t += __shfl_xor_sync( 0xffffffffu, t, o, LPR );
    return t;
}

__global__ void __launch_bounds__( VT ) k_cg_spmv( const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks, int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const VecDev &V = vs[ ch.prob ];
    if ( ! V.active || V.sc[ SC_CONV ] != 0 ) return;
    double pq = 0;
    const int sub = threadIdx.x % LPR;
    // every lane of a warp takes part in the shuffles: the loop runs to the chunk's end rounded up, rows past it idle
    for ( int i0 = ch.begin + int( threadIdx.x ) / LPR; i0 < ch.begin + ( ( ch.end - ch.begin + VT / LPR - 1 ) / ( VT / LPR ) ) * ( VT / LPR );
          i0 += VT / LPR ) {
        const bool in = i0 < ch.end;
        const double t = row_dot_lanes( V, in ? i0 : ch.begin, sub, V.p );
        if ( in && sub == 0 ) {
            const double pi = V.p[ i0 ];
            const double s = V.dia[ i0 ] * pi - t;
            V.q[ i0 ] = s;
            pq += pi * s;
        }
    }
    double v[ 1 ] = { pq }, tot[ 1 ];
    block_sum<1>( v );
    if ( fold_last<1>( V, ch, v, tot ) ) {
        if ( tot[ 0 ] > 0 ) V.sc[ SC_ALPHA ] = V.sc[ SC_RZ ] / tot[ 0 ];
        else { V.sc[ SC_ALPHA ] = 0; V.sc[ SC_FAIL ] = 1; V.sc[ SC_CONV ] = 2; }
    }
}

__global__ void __launch_bounds__( VT ) k_cg_update( const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks, int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const VecDev &V = vs[ ch.prob ];
    if ( ! V.active || V.sc[ SC_CONV ] != 0 ) return;
    const double al = V.sc[ SC_ALPHA ];
    double rz = 0, rr = 0;
    for ( int i = ch.begin + threadIdx.x; i < ch.end; i += VT ) {
        V.x[ i ] += al * V.p[ i ];
        double r = V.r[ i ] - al * V.q[ i ];
        V.r[ i ] = r;
        double z = r / V.dia[ i ];
        V.z[ i ] = z;
        rz += r * z;
        rr += r * r;
    }
    double v[ 2 ] = { rz, rr }, tot[ 2 ];
    block_sum<2>( v );
    if ( fold_last<2>( V, ch, v, tot ) ) {
        double it = V.sc[ SC_ITER ] + 1;
        V.sc[ SC_ITER ] = it;
        V.sc[ SC_BETA ] = tot[ 0 ] / V.sc[ SC_RZ ];
        V.sc[ SC_RZ ] = tot[ 0 ];
        double rn = sqrt( tot[ 1 ] );
        V.sc[ SC_RNORM ] = rn;
        if ( rn <= V.tol * V.sc[ SC_BNORM ] ) V.sc[ SC_CONV ] = 1;
        else if ( it >= V.maxit ) { V.sc[ SC_CONV ] = 2; V.sc[ SC_FAIL ] = 1; }
    }
}

__global__ void __launch_bounds__( VT ) k_cg_p( const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks, int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const VecDev &V = vs[ ch.prob ];
    if ( ! V.active || V.sc[ SC_CONV ] != 0 ) return;
    const double be = V.sc[ SC_BETA ];
    for ( int i = ch.begin + threadIdx.x; i < ch.end; i += VT ) V.p[ i ] = V.z[ i ] + be * V.p[ i ];
}

void launch_cg_init( const Launch &L, const VecDev *v, const Chunk *ch, int nch ) {
    if ( nch <= 0 ) return;
    k_cg_init<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    ++*L.launches;
}

void launch_cg_iter( const Launch &L, const VecDev *v, const Chunk *ch, int nch ) {
    if ( nch <= 0 ) return;
    k_cg_spmv<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    k_cg_update<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    k_cg_p<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    *L.launches += 3;
}

// ---- the multigrid-preconditioned CG -----------------------------------------------------------------------------------
__global__ void __launch_bounds__( VT ) k_cg_init0( const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks, int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const VecDev &V = vs[ ch.prob ];
    if ( ! V.active ) return;
    const double mean = V.sc[ SC_MEAN ];
    double bb = 0;
    for ( int i = ch.begin + threadIdx.x; i < ch.end; i += VT ) {
        double b = V.b[ i ] - mean;
        V.b[ i ] = b;
        V.x[ i ] = 0;
        V.r[ i ] = b;
        bb += b * b;
    }
    double v[ 1 ] = { bb }, tot[ 1 ];
    block_sum<1>( v );
    if ( fold_last<1>( V, ch, v, tot ) ) {
        V.sc[ SC_BNORM ] = sqrt( tot[ 0 ] );
        V.sc[ SC_RNORM ] = sqrt( tot[ 0 ] );
        V.sc[ SC_ITER ] = 0;
        V.sc[ SC_FAIL ] = 0;
        V.sc[ SC_CONV ] = tot[ 0 ] == 0 ? 1.0 : 0.0;
        if ( V.sc[ SC_NNZ ] > double( V.n ) * V.cap ) { V.sc[ SC_FAIL ] = 1; V.sc[ SC_CONV ] = 2; }
    }
}

// after the V-cycle wrote z: p = z, rz = r . z
__global__ void __launch_bounds__( VT ) k_cg_init1( const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks, int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const VecDev &V = vs[ ch.prob ];
    if ( ! V.active || V.sc[ SC_CONV ] != 0 ) return;
    double rz = 0;
    for ( int i = ch.begin + threadIdx.x; i < ch.end; i += VT ) {
        double z = V.z[ i ];
        V.p[ i ] = z;
        rz += V.r[ i ] * z;
    }
    double v[ 1 ] = { rz }, tot[ 1 ];
    block_sum<1>( v );
    if ( fold_last<1>( V, ch, v, tot ) ) V.sc[ SC_RZ ] = tot[ 0 ];
}

// x += alpha p, r -= alpha q, |r| and the convergence test (z comes from the V-cycle)
__global__ void __launch_bounds__( VT ) k_cg_update_mg( const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks, int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const VecDev &V = vs[ ch.prob ];
    if ( ! V.active || V.sc[ SC_CONV ] != 0 ) return;
    const double al = V.sc[ SC_ALPHA ];
    double rr = 0;
    for ( int i = ch.begin + threadIdx.x; i < ch.end; i += VT ) {
        V.x[ i ] += al * V.p[ i ];
        double r = V.r[ i ] - al * V.q[ i ];
        V.r[ i ] = r;
        rr += r * r;
    }
    double v[ 1 ] = { rr }, tot[ 1 ];
    block_sum<1>( v );
    if ( fold_last<1>( V, ch, v, tot ) ) {
        double it = V.sc[ SC_ITER ] + 1;
        V.sc[ SC_ITER ] = it;
        double rn = sqrt( tot[ 0 ] );
        V.sc[ SC_RNORM ] = rn;
        if ( rn <= V.tol * V.sc[ SC_BNORM ] ) V.sc[ SC_CONV ] = 1;
        else if ( it >= V.maxit ) { V.sc[ SC_CONV ] = 2; V.sc[ SC_FAIL ] = 1; }
    }
}

// rz' = r . z, beta = rz' / rz
__global__ void __launch_bounds__( VT ) k_cg_rz( const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks, int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const VecDev &V = vs[ ch.prob ];
    if ( ! V.active || V.sc[ SC_CONV ] != 0 ) return;
    double rz = 0;
    for ( int i = ch.begin + threadIdx.x; i < ch.end; i += VT ) rz += V.r[ i ] * V.z[ i ];
    double v[ 1 ] = { rz }, tot[ 1 ];
    block_sum<1>( v );
    if ( fold_last<1>( V, ch, v, tot ) ) {
        V.sc[ SC_BETA ] = tot[ 0 ] / V.sc[ SC_RZ ];
        V.sc[ SC_RZ ] = tot[ 0 ];
    }
}

void launch_cg_init0( const Launch &L, const VecDev *v, const Chunk *ch, int nch ) {
    if ( nch <= 0 ) return;
    k_cg_init0<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    ++*L.launches;
}
void launch_cg_init1( const Launch &L, const VecDev *v, const Chunk *ch, int nch ) {
    if ( nch <= 0 ) return;
    k_cg_init1<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    ++*L.launches;
}
void launch_cg_spmv_update( const Launch &L, const VecDev *v, const Chunk *ch, int nch ) {
    if ( nch <= 0 ) return;
    k_cg_spmv<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    k_cg_update_mg<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    *L.launches += 2;
}
void launch_cg_rz_p( const Launch &L, const VecDev *v, const Chunk *ch, int nch ) {
    if ( nch <= 0 ) return;
    k_cg_rz<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    k_cg_p<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    *L.launches += 2;
}

// ---- FP32 CG with FP64 iterative refinement (lin_precision 1) ----------------------------------------------------------
// The inner CG runs on FP32 copies of the matrix values, of the diagonal and of its vectors (e, r32, z32, p32, q32): half
// the bytes of every product and update.  x, the residual r and b stay FP64.  When the inner residual has fallen by
// MX_INNER (or under half the outer target), x += e in FP64, the residual r = b - A x is recomputed with the FP64 matrix,
// and the inner CG restarts on it; the outer stop is the FP64 residual's, tol |b|.  A refinement that does not cut the
// FP64 residual by 10 % ends the solve with SC_FAIL = 2: the refinement stalls once the condition number times the FP32
// rounding reaches 1 (the FP32 matrix and products then perturb the system by more than the inner CG gains), as on the
// Laplacians of a million seeds under a density that varies a hundredfold.
// Everything runs inside the ordinary sequence of CG launches (so a burst, and its CUDA graph, is unchanged), steered by
// the problem's scalars: the update's fold sets SC_REFINE; the next p kernel adds e to x instead of updating p; the next
// product computes the FP64 residual instead of q, resets e and p to 0 and sets alpha = 0, rz = 1 -- so that the
// update, the V-cycle and p = z + beta p that follow start a fresh CG.  Dot products are summed in FP64, in fixed trees.
constexpr double MX_INNER = 1e-3;

__device__ __forceinline__ bool mx_idle( const VecDev &V ) { return ! V.active || V.sc[ SC_CONV ] != 0; }

__device__ __forceinline__ float row_dot32( const VecDev &V, int i, int sub, const float *__restrict__ x ) {
    float t = 0;
    const int e1 = V.row_ptr[ i + 1 ];
    for ( int e = V.row_ptr[ i ] + sub; e < e1; e += LPR ) t += V.val32[ e ] * x[ V.col[ e ] ];
#pragma unroll
    for ( int o = 1; o < LPR; o <<= 1 ) t += __shfl_xor_sync( 0xffffffffu, t, o, LPR );
    return t;
}

// b -= mean; x = 0, r = b; the FP32 copies; e = 0, r32 = r; Jacobi: z32 = r32 / dia, p32 = z32; multigrid: p32 = 0 (set by
// init1 after the first V-cycle)
__global__ void __launch_bounds__( VT ) k_mx_init( const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks, int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const VecDev &V = vs[ ch.prob ];
    if ( ! V.active ) return;
    const double mean = V.sc[ SC_MEAN ];
    const bool jac = ! V.precond;
    double bb = 0, ss = 0, rz = 0;
    for ( int i = ch.begin + threadIdx.x; i < ch.end; i += VT ) {
        for ( int e = V.row_ptr[ i ]; e < V.row_ptr[ i + 1 ]; ++e ) V.val32[ e ] = float( V.val[ e ] );
        const float d32 = float( V.dia[ i ] );
        V.dia32[ i ] = d32;
        const double b = V.b[ i ] - mean;
        V.b[ i ] = b;
        V.x[ i ] = 0;
        V.r[ i ] = b;
        const float r32 = float( b ), z32 = jac ? r32 / d32 : 0.0f;
        V.x32[ i ] = 0; V.r32[ i ] = r32; V.q32[ i ] = 0; V.z32[ i ] = z32; V.p32[ i ] = z32;
        bb += b * b;
        ss += double( r32 ) * r32;
        rz += double( r32 ) * z32;
    }
    double v[ 3 ] = { bb, ss, rz }, tot[ 3 ];
    block_sum<3>( v );
    if ( fold_last<3>( V, ch, v, tot ) ) {
        const double bn = sqrt( tot[ 0 ] );
        V.sc[ SC_BNORM ] = bn; V.sc[ SC_RNORM ] = bn; V.sc[ SC_RPREV ] = bn;
        V.sc[ SC_IN0 ] = sqrt( tot[ 1 ] );
        V.sc[ SC_RZ ] = jac ? tot[ 2 ] : 1.0;
        V.sc[ SC_ITER ] = 0; V.sc[ SC_FAIL ] = 0; V.sc[ SC_REFINE ] = 0; V.sc[ SC_NREF ] = 0;
        V.sc[ SC_CONV ] = tot[ 0 ] == 0 ? 1.0 : 0.0;
        if ( V.sc[ SC_NNZ ] > double( V.n ) * V.cap ) { V.sc[ SC_FAIL ] = 1; V.sc[ SC_CONV ] = 2; }
    }
}

// (multigrid) after the first V-cycle: p32 = z32, rz
__global__ void __launch_bounds__( VT ) k_mx_init1( const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks, int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const VecDev &V = vs[ ch.prob ];
    if ( mx_idle( V ) ) return;
    double rz = 0;
    for ( int i = ch.begin + threadIdx.x; i < ch.end; i += VT ) {
        const float z = V.z32[ i ];
        V.p32[ i ] = z;
        rz += double( V.r32[ i ] ) * z;
    }
    double v[ 1 ] = { rz }, tot[ 1 ];
    block_sum<1>( v );
    if ( fold_last<1>( V, ch, v, tot ) ) V.sc[ SC_RZ ] = tot[ 0 ];
}

// q32 = A32 p32 and alpha; or, after an inner convergence, the refinement: r = b - A x (FP64), the inner CG restarted on it
__global__ void __launch_bounds__( VT ) k_mx_spmv( const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks, int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const VecDev &V = vs[ ch.prob ];
    if ( mx_idle( V ) ) return;
    const bool refine = V.sc[ SC_REFINE ] != 0;       // (read by every block before the last one's fold clears it)
    const int sub = threadIdx.x % LPR;
    double a0 = 0, a1 = 0;
    const int end = ch.begin + ( ( ch.end - ch.begin + VT / LPR - 1 ) / ( VT / LPR ) ) * ( VT / LPR );
    for ( int i0 = ch.begin + int( threadIdx.x ) / LPR; i0 < end; i0 += VT / LPR ) {
        const bool in = i0 < ch.end;
        const int row = in ? i0 : ch.begin;
        if ( refine ) {
            const double t = row_dot_lanes( V, row, sub, V.x );
            if ( in && sub == 0 ) {
                const double r = V.b[ i0 ] - ( V.dia[ i0 ] * V.x[ i0 ] - t );
                V.r[ i0 ] = r;
                const float r32 = float( r );
                V.r32[ i0 ] = r32; V.x32[ i0 ] = 0; V.p32[ i0 ] = 0;
                a0 += r * r;
                a1 += double( r32 ) * r32;
            }
        } else {
            const float t = row_dot32( V, row, sub, V.p32 );
            if ( in && sub == 0 ) {
                const float pi = V.p32[ i0 ], q = V.dia32[ i0 ] * pi - t;
                V.q32[ i0 ] = q;
                a0 += double( pi ) * q;
            }
        }
    }
    double v[ 2 ] = { a0, a1 }, tot[ 2 ];
    block_sum<2>( v );
    if ( fold_last<2>( V, ch, v, tot ) ) {
        if ( refine ) {
            const double rn = sqrt( tot[ 0 ] );
            V.sc[ SC_RNORM ] = rn;
            V.sc[ SC_NREF ] += 1;
            V.sc[ SC_REFINE ] = 0;
            if ( rn <= V.tol * V.sc[ SC_BNORM ] ) V.sc[ SC_CONV ] = 1;
            else if ( ! ( rn < 0.9 * V.sc[ SC_RPREV ] ) ) { V.sc[ SC_FAIL ] = 2; V.sc[ SC_CONV ] = 2; }    // (2: the refinement stalls)
            else {
                V.sc[ SC_RPREV ] = rn;
                V.sc[ SC_IN0 ] = sqrt( tot[ 1 ] );
                V.sc[ SC_ALPHA ] = 0;
                V.sc[ SC_RZ ] = 1;
            }
        } else if ( tot[ 0 ] > 0 )
            V.sc[ SC_ALPHA ] = V.sc[ SC_RZ ] / tot[ 0 ];
        else { V.sc[ SC_ALPHA ] = 0; V.sc[ SC_FAIL ] = 1; V.sc[ SC_CONV ] = 2; }
    }
}

// e += alpha p32, r32 -= alpha q32 (Jacobi: z32 = r32 / dia, rz, beta); the inner stop sets SC_REFINE
__global__ void __launch_bounds__( VT ) k_mx_update( const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks, int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const VecDev &V = vs[ ch.prob ];
    if ( mx_idle( V ) ) return;
    const float al = float( V.sc[ SC_ALPHA ] );
    const bool jac = ! V.precond;
    double rz = 0, rr = 0;
    for ( int i = ch.begin + threadIdx.x; i < ch.end; i += VT ) {
        V.x32[ i ] += al * V.p32[ i ];
        const float r = V.r32[ i ] - al * V.q32[ i ];
        V.r32[ i ] = r;
        if ( jac ) {
            const float z = r / V.dia32[ i ];
            V.z32[ i ] = z;
            rz += double( r ) * z;
        }
        rr += double( r ) * r;
    }
    double v[ 2 ] = { rz, rr }, tot[ 2 ];
    block_sum<2>( v );
    if ( fold_last<2>( V, ch, v, tot ) ) {
        const double it = V.sc[ SC_ITER ] + 1;
        V.sc[ SC_ITER ] = it;
        if ( jac ) {
            V.sc[ SC_BETA ] = tot[ 0 ] / V.sc[ SC_RZ ];
            V.sc[ SC_RZ ] = tot[ 0 ];
        }
        const double rn = sqrt( tot[ 1 ] );
        if ( it >= V.maxit ) { V.sc[ SC_CONV ] = 2; V.sc[ SC_FAIL ] = 1; }
        else if ( rn <= MX_INNER * V.sc[ SC_IN0 ] || rn <= 0.5 * V.tol * V.sc[ SC_BNORM ] ) V.sc[ SC_REFINE ] = 1;
    }
}

// (multigrid) rz = r32 . z32 after the V-cycle, beta
__global__ void __launch_bounds__( VT ) k_mx_rz( const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks, int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const VecDev &V = vs[ ch.prob ];
    if ( mx_idle( V ) || V.sc[ SC_REFINE ] != 0 ) return;
    double rz = 0;
    for ( int i = ch.begin + threadIdx.x; i < ch.end; i += VT ) rz += double( V.r32[ i ] ) * V.z32[ i ];
    double v[ 1 ] = { rz }, tot[ 1 ];
    block_sum<1>( v );
    if ( fold_last<1>( V, ch, v, tot ) ) {
        V.sc[ SC_BETA ] = tot[ 0 ] / V.sc[ SC_RZ ];
        V.sc[ SC_RZ ] = tot[ 0 ];
    }
}

// p32 = z32 + beta p32; or, after an inner convergence, x += e (FP64)
__global__ void __launch_bounds__( VT ) k_mx_p( const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks, int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const VecDev &V = vs[ ch.prob ];
    if ( mx_idle( V ) ) return;
    if ( V.sc[ SC_REFINE ] != 0 ) {
        for ( int i = ch.begin + threadIdx.x; i < ch.end; i += VT ) V.x[ i ] += double( V.x32[ i ] );
        return;
    }
    const float be = float( V.sc[ SC_BETA ] );
    for ( int i = ch.begin + threadIdx.x; i < ch.end; i += VT ) V.p32[ i ] = V.z32[ i ] + be * V.p32[ i ];
}

void launch_mx_init( const Launch &L, const VecDev *v, const Chunk *ch, int nch ) {
    if ( nch <= 0 ) return;
    k_mx_init<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    ++*L.launches;
}
void launch_mx_init1( const Launch &L, const VecDev *v, const Chunk *ch, int nch ) {
    if ( nch <= 0 ) return;
    k_mx_init1<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    ++*L.launches;
}
void launch_mx_iter( const Launch &L, const VecDev *v, const Chunk *ch, int nch ) {
    if ( nch <= 0 ) return;
    k_mx_spmv<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    k_mx_update<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    k_mx_p<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    *L.launches += 3;
}
void launch_mx_spmv_update( const Launch &L, const VecDev *v, const Chunk *ch, int nch ) {
    if ( nch <= 0 ) return;
    k_mx_spmv<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    k_mx_update<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    *L.launches += 2;
}
void launch_mx_rz_p( const Launch &L, const VecDev *v, const Chunk *ch, int nch ) {
    if ( nch <= 0 ) return;
    k_mx_rz<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    k_mx_p<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    *L.launches += 2;
}

// d = x - x[ rank of user seed 0 ]: the gauge w_0 = 0 kept by the direction
__global__ void k_gauge( const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks, int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const VecDev &V = vs[ ch.prob ];
    if ( ! V.active ) return;
    const double x0 = V.x[ V.rank0 ];
    for ( int i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x ) V.d[ i ] = V.x[ i ] - x0;
}

void launch_gauge( const Launch &L, const VecDev *v, const Chunk *ch, int nch ) {
    if ( nch <= 0 ) return;
    k_gauge<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    ++*L.launches;
}

// w2 = w + t d, and the max of w2 for the security radius of the next diagram
__global__ void k_trial( const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks, int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const VecDev &V = vs[ ch.prob ];
    if ( ! V.active ) return;
    double m = -1e300;
    for ( int i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x ) {
        double w2 = i == V.rank0 ? 0.0 : V.w[ i ] + V.t * V.d[ i ];
        V.w2[ i ] = w2;
        m = fmax( m, w2 );
    }
    m = warp_max( m );
    if ( ( threadIdx.x & 31 ) == 0 ) atomicMax( V.wmax_slot, dbl_order( m ) );
}

void launch_trial( const Launch &L, const VecDev *v, const Chunk *ch, int nch ) {
    if ( nch <= 0 ) return;
    k_trial<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    ++*L.launches;
}

__global__ void k_scale( double *v, int n, double s ) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if ( i < n ) v[ i ] *= s;
}
void launch_scale( const Launch &L, double *v, int n, double s ) {
    if ( n <= 0 ) return;
    k_scale<<<( n + 255 ) / 256, 256, 0, L.stream>>>( v, n, s );
    ++*L.launches;
}

// out_user[ user[ s ] ] = ranked[ s ]  (dim values per seed)
__global__ void k_scatter( const double *__restrict__ ranked, const int *__restrict__ user, int n, int dim, double *out ) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if ( s >= n ) return;
    int u = user[ s ];
    for ( int a = 0; a < dim; ++a ) out[ ( size_t ) u * dim + a ] = ranked[ ( size_t ) s * dim + a ];
}
void launch_scatter( const Launch &L, const double *ranked, const int *user, int n, int dim, double *out_user ) {
    if ( n <= 0 ) return;
    k_scatter<<<( n + 255 ) / 256, 256, 0, L.stream>>>( ranked, user, n, dim, out_user );
    ++*L.launches;
}

// ranked[ s ] = scale * user_vals[ user[ s ] ]  (user_vals NULL: scale)
__global__ void k_gather_vec( const double *__restrict__ uv, const int *__restrict__ user, int n, double *ranked, double scale ) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if ( s >= n ) return;
    ranked[ s ] = uv ? scale * uv[ user[ s ] ] : scale;
}
void launch_gather_vec( const Launch &L, const double *user_vals, const int *user, int n, double *ranked, double scale ) {
    if ( n <= 0 ) return;
    k_gather_vec<<<( n + 255 ) / 256, 256, 0, L.stream>>>( user_vals, user, n, ranked, scale );
    ++*L.launches;
}

// ---- the re-splitting's weights: w2 = w - shift, then the members' steps added ------------------------------------------
__global__ void k_polish_shift( const double *__restrict__ w, double *__restrict__ w2, int n, double shift ) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if ( i < n ) w2[ i ] = w[ i ] - shift;
}
__global__ void k_polish_add( double *__restrict__ w2, const int *__restrict__ idx, const double *__restrict__ val, int k ) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if ( t < k ) w2[ idx[ t ] ] += val[ t ];
}
void launch_polish_weights( const Launch &L, const double *w, double *w2, int n, double shift, const int *idx, const double *val, int k ) {
    k_polish_shift<<<( n + 255 ) / 256, 256, 0, L.stream>>>( w, w2, n, shift );
    k_polish_add<<<( k + 255 ) / 256, 256, 0, L.stream>>>( w2, idx, val, k );
    *L.launches += 2;
}

// ---- the aggregation of near-coincident seeds (sdotplan/Aggregation.h:1-44, 229-250) ---------------------------------
// A facet's plane moves by ( w_i - w_j ) / ( 2 |p_i - p_j| ): the doubles of the weights place it no better than
// m_ij = c_ij ulp( max( |w_i|, |w_j| ) ) of mass.  The pair is merged when m_ij margin > tau_ij,
// tau_ij = max( tol_abs, tol_rel nu, 1e-12 nu ), nu = min( nu_i, nu_j ).
__global__ void __launch_bounds__( VT ) k_agg_detect( const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks, int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const VecDev &V = vs[ ch.prob ];
    if ( ! V.active || ! V.agg_pairs || ! ( V.agg_margin > 0 ) ) return;
    for ( int i = ch.begin + threadIdx.x; i < ch.end; i += VT ) {
        for ( int e = V.row_ptr[ i ]; e < V.row_ptr[ i + 1 ]; ++e ) {
            const int j = V.col[ e ];
            if ( j <= i ) continue;
            const double wm = fmax( fabs( V.w[ i ] ), fabs( V.w[ j ] ) );
            const double ulp = __longlong_as_double( __double_as_longlong( wm ) + 1 ) - wm;     // the spacing of the doubles at wm
            const double nm = fmin( V.nu[ i ], V.nu[ j ] );
            const double tau = fmax( V.agg_tol_abs, fmax( V.agg_tol_rel * nm, 1e-12 * nm ) );
            // (a coupling past 1e9 times the scale of a facet is merged whatever the weights: gpu/Newton2D.cuh:1287-1313)
            if ( V.val[ e ] * ulp * V.agg_margin > tau || V.val[ e ] > V.agg_ccond ) {
                const int k = int( atomicAdd( V.agg_count, 1.0 ) );
                if ( k < V.agg_cap ) V.agg_pairs[ k ] = make_int2( i, j );
            }
        }
    }
}

void launch_agg_detect( const Launch &L, const VecDev *v, const Chunk *ch, int nch ) {
    if ( nch <= 0 ) return;
    k_agg_detect<<<nch, VT, 0, L.stream>>>( v, ch, nch );
    ++*L.launches;
}

// THE DIRECTION WITH CLUSTERS (the reference card's rule, gpu/Newton2D.cuh:443-478, 1386-1440, 1565-1612): the coupling
// between two members of a cluster (2.5e10 for a pair 1e-12 apart) is capped at `cap` in the system the CG solves -- the
// multigrid's FP32 levels do not hold it -- and the true couplings kept aside for the correction after the solve.  One
// thread per cluster (members sorted by rank): blk[ q * ( AGG_KMAX + 1 ) + p ] the true coupling of member q to member p,
// blk[ q * ( AGG_KMAX + 1 ) + AGG_KMAX ] the true diagonal of member q (kept for clusters of at most AGG_KMAX members)
__device__ __forceinline__ int member_of( const int *clm, int b0, int b1, int j ) {
    int lo = b0, hi = b1;
    while ( lo < hi ) { const int mid = ( lo + hi ) >> 1; if ( clm[ mid ] < j ) lo = mid + 1; else hi = mid; }
    return lo < b1 && clm[ lo ] == j ? lo - b0 : -1;
}

__global__ void k_agg_cap( const int *__restrict__ row_ptr, const int *__restrict__ col, double *val, double *dia, const int *__restrict__ clb,
                           const int *__restrict__ clm, int ncl, double cap, double *blk ) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if ( c >= ncl ) return;
    const int b0 = clb[ c ], b1 = clb[ c + 1 ], k = b1 - b0;
    for ( int q = b0; q < b1; ++q ) {
        const int i = clm[ q ];
        double *T = blk + size_t( q ) * ( AGG_KMAX + 1 );
        if ( k <= AGG_KMAX ) {
            for ( int p = 0; p < k; ++p ) T[ p ] = 0;
            T[ AGG_KMAX ] = dia[ i ];
        }
        bool capped = false;
        for ( int e = row_ptr[ i ]; e < row_ptr[ i + 1 ]; ++e ) {
            const int p = member_of( clm, b0, b1, col[ e ] );
            if ( p < 0 ) continue;
            if ( k <= AGG_KMAX ) T[ p ] = val[ e ];
            if ( val[ e ] > cap ) { val[ e ] = cap; capped = true; }
        }
        if ( capped ) {                  // the diagonal summed again, in row order
            double d = 0;
            for ( int e = row_ptr[ i ]; e < row_ptr[ i + 1 ]; ++e ) d += val[ e ];
            dia[ i ] = d > 0 ? d : 1.0;
        }
    }
}

void launch_agg_cap( const Launch &L, const int *row_ptr, const int *col, double *val, double *dia, const int *cl, int ncl, double cap, double *blk ) {
    if ( ncl <= 0 ) return;
    k_agg_cap<<<( ncl + 127 ) / 128, 128, 0, L.stream>>>( row_ptr, col, val, dia, cl, cl + ncl + 1, ncl, cap, blk );
    ++*L.launches;
}

// ... after the solve of the capped system: each cluster's members tied to their cluster's direction, `x_i = sum nu_j x_j /
// sum nu_j`, then the split inside the cluster corrected by its exact local system, the rest of x fixed: `L_CC y = b_C -
// ( L x )_C` with the TRUE couplings, y's mean over the cluster (weighted by the targets) taken out, x_C += y -- one
// two-level step.  One block: the ties of every cluster, then (reading the tied x) the corrections into `y`, then the sums,
// so that a cluster never reads another's half-updated members
__global__ void __launch_bounds__( 128 ) k_agg_direction( const int *__restrict__ row_ptr, const int *__restrict__ col, const double *__restrict__ val,
                                                         const int *__restrict__ clb, const int *__restrict__ clm, int ncl, const double *__restrict__ blk,
                                                         const double *__restrict__ nu, const double *__restrict__ b, double *x, double *y ) {
    for ( int c = threadIdx.x; c < ncl; c += blockDim.x ) {
        double s = 0, sn = 0;
        for ( int q = clb[ c ]; q < clb[ c + 1 ]; ++q ) { s += nu[ clm[ q ] ] * x[ clm[ q ] ]; sn += nu[ clm[ q ] ]; }
        const double xm = sn > 0 ? s / sn : 0.0;
        for ( int q = clb[ c ]; q < clb[ c + 1 ]; ++q ) x[ clm[ q ] ] = xm;
    }
    __syncthreads();
    for ( int c = threadIdx.x; c < ncl; c += blockDim.x ) {
        const int b0 = clb[ c ], b1 = clb[ c + 1 ], k = b1 - b0;
        for ( int q = b0; q < b1; ++q ) y[ q ] = 0;
        if ( k > AGG_KMAX ) continue;
        double M[ AGG_KMAX * AGG_KMAX ], r[ AGG_KMAX ];
        for ( int q = 0; q < k; ++q ) {
            const int i = clm[ b0 + q ];
            const double *T = blk + size_t( b0 + q ) * ( AGG_KMAX + 1 );
            double ld = T[ AGG_KMAX ] * x[ i ];
            for ( int e = row_ptr[ i ]; e < row_ptr[ i + 1 ]; ++e ) {
                const int p = member_of( clm, b0, b1, col[ e ] );
                ld -= ( p >= 0 ? T[ p ] : val[ e ] ) * x[ col[ e ] ];
            }
            r[ q ] = b[ i ] - ld;
            for ( int p = 0; p < k; ++p ) M[ q * k + p ] = p == q ? T[ AGG_KMAX ] : -T[ p ];
        }
        // Cholesky of the k x k block (positive definite when the cluster has a neighbour outside it), then the solve
        bool ok = true;
        for ( int j = 0; j < k && ok; ++j ) {
            double d = M[ j * k + j ];
            for ( int p = 0; p < j; ++p ) d -= M[ j * k + p ] * M[ j * k + p ];
            if ( ! ( d > 0 ) ) { ok = false; break; }
            const double l = sqrt( d );
            M[ j * k + j ] = l;
            for ( int i = j + 1; i < k; ++i ) {
                double v = M[ i * k + j ];
                for ( int p = 0; p < j; ++p ) v -= M[ i * k + p ] * M[ j * k + p ];
                M[ i * k + j ] = v / l;
            }
        }
        if ( ! ok ) continue;
        for ( int i = 0; i < k; ++i ) {
            double v = r[ i ];
            for ( int p = 0; p < i; ++p ) v -= M[ i * k + p ] * r[ p ];
            r[ i ] = v / M[ i * k + i ];
        }
        for ( int i = k - 1; i >= 0; --i ) {
            double v = r[ i ];
            for ( int p = i + 1; p < k; ++p ) v -= M[ p * k + i ] * r[ p ];
            r[ i ] = v / M[ i * k + i ];
        }
        double s = 0, sn = 0;
        for ( int q = 0; q < k; ++q ) { s += nu[ clm[ b0 + q ] ] * r[ q ]; sn += nu[ clm[ b0 + q ] ]; }
        const double m = sn > 0 ? s / sn : 0.0;
        bool fin = true;
        for ( int q = 0; q < k; ++q ) fin = fin && isfinite( r[ q ] - m );
        if ( fin )
            for ( int q = 0; q < k; ++q ) y[ b0 + q ] = r[ q ] - m;
    }
    __syncthreads();
    for ( int c = threadIdx.x; c < ncl; c += blockDim.x )
        for ( int q = clb[ c ]; q < clb[ c + 1 ]; ++q ) x[ clm[ q ] ] += y[ q ];
}

void launch_agg_direction( const Launch &L, const int *row_ptr, const int *col, const double *val, const int *cl, int ncl, const double *blk,
                           const double *nu, const double *b, double *x, double *y ) {
    if ( ncl <= 0 ) return;
    k_agg_direction<<<1, 128, 0, L.stream>>>( row_ptr, col, val, cl, cl + ncl + 1, ncl, blk, nu, b, x, y );
    ++*L.launches;
}

// one thread per cluster: its members' masses summed in member order, each member's share of it
__global__ void k_agg_shares( const double *__restrict__ a, const double *__restrict__ nu, const int *__restrict__ clb,
                              const int *__restrict__ clm, int ncl, double *ae ) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if ( c >= ncl ) return;
    double sa = 0, sn = 0;
    for ( int k = clb[ c ]; k < clb[ c + 1 ]; ++k ) { sa += a[ clm[ k ] ]; sn += nu[ clm[ k ] ]; }
    const double r = sn > 0 ? sa / sn : 0.0;
    for ( int k = clb[ c ]; k < clb[ c + 1 ]; ++k ) ae[ clm[ k ] ] = nu[ clm[ k ] ] * r;
}

void launch_agg_shares( const Launch &L, const double *a, const double *nu, const int *cl_begin, const int *cl_members, int ncl, double *ae ) {
    if ( ncl <= 0 ) return;
    k_agg_shares<<<( ncl + 127 ) / 128, 128, 0, L.stream>>>( a, nu, cl_begin, cl_members, ncl, ae );
    ++*L.launches;
}

} // namespace sdot

// Aggregation multigrid preconditioner of the Laplacian CG, batched over problems.
//
// Levels: level 0 is the Newton Laplacian (its FP64 CSR copied to FP32); level l+1 aggregates PACK consecutive
// Morton ranks of level l (4 in 2D, 8 in 3D) -- consecutive ranks are neighbours in space, the reference's own
// aggregation by `rank >> shift` (gpu/Linear2D.cuh:15-16, sdotplan/Multigrid.h:10-18) -- with the Galerkin
// operator P^T A P of the piecewise-constant prolongation, which is again a graph Laplacian: off-diagonals
// c_IJ = sum of the c_ij between the two aggregates, dia = the row sum.  The coarsest level (<= MG_BOTTOM rows)
// is solved exactly by the dense inverse of A + mu 1 1^T, which acts as the pseudo-inverse on zero-sum vectors.
// One V(1,1)-cycle with damped Jacobi on both sides and an over-corrected coarse correction (symmetric, so it is a
// valid CG preconditioner), all in FP32:
// the outer CG stays in FP64 and plays the part of the iterative refinement.
//
// Each launch covers one level of every problem that has it; pre-smoothing from zero, the residual and the
// restriction are one kernel (the smoothed x of a neighbour is recomputed from its rhs), prolongation and
// post-smoothing another.  Coarse rows are built by one warp each from the aggregate's fine rows, summing equal
// columns in gather order -- deterministic.
#include "internal.h"
#include <cub/block/block_scan.cuh>

namespace sdot {

constexpr int MGT = 256;                // threads per block
constexpr int MG_PAIRS = 1024;          // (column, value) pairs a warp gathers for one coarse row
constexpr int MG_WARPS = 4;             // warps per block of the coarsening kernels

// ---- build -------------------------------------------------------------------------------------------------------------
// level 0 from the FP64 CSR of the Newton Laplacian.  A coupling far above the rest of both its rows (two seeds 1e-12
// apart: c_ij ~ 1e10 next to couplings ~ 1) would make the FP32 cycle's residuals cancel to noise (a row of
// 1e10 x_i - 1e10 x_j loses everything to rounding) and the preconditioner would stop being positive: in the
// PRECONDITIONER's copy it is capped at MG_CAP times the smaller of the two rows' other couplings (symmetric; the outer
// FP64 CG keeps the exact matrix).  Ordinary diagrams never reach the cap.
constexpr double MG_CAP = 1e3;

// each row's couplings but its largest, summed (the cap's scale), into the level's x (free during the build)
__global__ void k_mg_rest( const MgLevel *__restrict__ lv, const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks, int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const MgLevel &M = lv[ ch.prob ];
    const VecDev &V = vs[ M.vec ];
    for ( int i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x ) {
        double sum = 0, mx = 0;
        for ( int e = V.row_ptr[ i ]; e < V.row_ptr[ i + 1 ]; ++e ) { sum += V.val[ e ]; mx = fmax( mx, V.val[ e ] ); }
        M.x[ i ] = float( sum - mx );
    }
}

__global__ void k_mg_level0( const MgLevel *__restrict__ lv, const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks, int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const MgLevel &M = lv[ ch.prob ];
    const VecDev &V = vs[ M.vec ];
    for ( int i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x ) {
        const int b = V.row_ptr[ i ], e1 = V.row_ptr[ i + 1 ];
        if ( b == e1 ) {                               // an empty row keeps the Newton Laplacian's unit diagonal
            M.dia[ i ] = float( V.dia[ i ] );
            M.dinv[ i ] = float( 1.0 / V.dia[ i ] );
            continue;
        }
        double dia = 0;
        for ( int e = b; e < e1; ++e ) {
            const double rest = fmin( double( M.x[ i ] ), double( M.x[ V.col[ e ] ] ) );
            const double c = rest > 0 ? fmin( V.val[ e ], MG_CAP * rest ) : V.val[ e ];
            M.val[ e ] = float( c );
            dia += c;
        }
        M.dia[ i ] = float( dia );
        M.dinv[ i ] = float( 1.0 / dia );
    }
}

// the (column, value) pairs of coarse row I, gathered by one warp into shared memory as keys ( column << 11 | pair index )
// and values by pair index, then sorted by key (a bitonic sort over the warp, padded to a power of 2): the pairs of
// each coarse column form a run, in pair order.  Returns the pair count (-1: past MG_PAIRS)
constexpr int MG_KEY_SHIFT = 11;                         // pair indices < 2048 (MG_PAIRS is 1024)
__device__ int gather_sorted( const MgLevel &M, int I, long long *key, float *cv, int lane ) {
    const int i0 = I * M.pack, i1 = min( M.n, i0 + M.pack );
    int cnt = 0;
    for ( int i = i0; i < i1; ++i ) {
        const int b = M.rp[ i ], e = M.rp[ i + 1 ];
        for ( int base = b; base < e; base += 32 ) {
            const int k = base + lane, at = cnt + ( k - base );
            if ( k < e && at < MG_PAIRS ) {
                key[ at ] = ( ( long long ) ( M.col[ k ] / M.pack ) << MG_KEY_SHIFT ) | at;
                cv[ at ] = M.val[ k ];
            }
            cnt += min( 32, e - base );
        }
    }
    __syncwarp();
    if ( cnt > MG_PAIRS ) return -1;
    int n2 = 1;
    while ( n2 < cnt ) n2 <<= 1;
    for ( int k = cnt + lane; k < n2; k += 32 ) key[ k ] = 0x7fffffffffffffffll;
    __syncwarp();
    for ( int k = 2; k <= n2; k <<= 1 )
        for ( int j = k >> 1; j > 0; j >>= 1 ) {
            for ( int i = lane; i < n2; i += 32 ) {
                const int l = i ^ j;
                if ( l > i ) {
                    const long long x = key[ i ], y = key[ l ];
                    if ( ( x > y ) == ( ( i & k ) == 0 ) ) { key[ i ] = y; key[ l ] = x; }
                }
            }
            __syncwarp();
        }
    return cnt;
}

// in the sorted pairs: does position p start the run of a coarse column other than the diagonal I?
__device__ __forceinline__ bool run_start( const long long *key, int p, int I ) {
    const long long J = key[ p ] >> MG_KEY_SHIFT;
    return J != I && ( p == 0 || ( key[ p - 1 ] >> MG_KEY_SHIFT ) != J );
}

__global__ void __launch_bounds__( 32 * MG_WARPS ) k_mg_count( const MgLevel *__restrict__ lv, const Chunk *__restrict__ chunks, int nch,
                                                              ErrRec *err ) {
    extern __shared__ long long mg_pairs_smem[];
    long long ( *sk )[ MG_PAIRS ] = reinterpret_cast<long long ( * )[ MG_PAIRS ]>( mg_pairs_smem );
    float ( *sv )[ MG_PAIRS ] = reinterpret_cast<float ( * )[ MG_PAIRS ]>( mg_pairs_smem + MG_WARPS * MG_PAIRS );
    __shared__ double tot_w[ MG_WARPS ];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const Chunk ch = chunks[ blockIdx.x ];
    const MgLevel &M = lv[ ch.prob ];
    double tot = 0;
    for ( int I = ch.begin + warp; I < ch.end; I += MG_WARPS ) {
        int cnt = gather_sorted( M, I, sk[ warp ], sv[ warp ], lane );
        int distinct = 0;
        for ( int k = lane; k < cnt; k += 32 ) distinct += run_start( sk[ warp ], k, I );
        for ( int o = 16; o > 0; o >>= 1 ) distinct += __shfl_xor_sync( 0xffffffffu, distinct, o );
        if ( cnt < 0 ) distinct = M.capn + 1;                           // too many pairs: the level is refused (k_mg_scan)
        if ( lane == 0 ) M.rcn[ I ] = distinct;
        tot += distinct;
        __syncwarp();
    }
    if ( lane == 0 ) tot_w[ warp ] = tot;
    __syncthreads();
    if ( threadIdx.x == 0 ) {
        double s = 0;
        for ( int w = 0; w < MG_WARPS; ++w ) s += tot_w[ w ];
        M.part[ ( size_t ) ch.index * 2 ] = s;
    }
}

// one block per problem: exclusive scan of the chunk totals -> part[ 2 c + 1 ]; the coarse row_ptr end
__global__ void __launch_bounds__( 1024 ) k_mg_scan( const MgLevel *__restrict__ lv ) {
    const MgLevel &M = lv[ blockIdx.x ];
    if ( ! M.rpn ) return;                                              // this job's coarsest level: nothing to build
    typedef cub::BlockScan<long long, 1024> Scan;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ long long carry;
    if ( threadIdx.x == 0 ) carry = 0;
    __syncthreads();
    for ( int base = 0; base < M.nchunk; base += 1024 ) {
        int c = base + threadIdx.x;
        long long x = c < M.nchunk ? ( long long ) M.part[ ( size_t ) c * 2 ] : 0, ex, agg;
        Scan( tmp ).ExclusiveSum( x, ex, agg );
        if ( c < M.nchunk ) M.part[ ( size_t ) c * 2 + 1 ] = double( carry + ex );
        __syncthreads();
        if ( threadIdx.x == 0 ) carry += agg;
        __syncthreads();
    }
    if ( threadIdx.x == 0 ) M.rpn[ M.nn ] = int( carry > M.capn ? 0 : carry );
    if ( threadIdx.x == 0 && carry > M.capn ) M.part[ 0 ] = -1;        // refused: the next level is diagonal
}

__global__ void __launch_bounds__( 32 * MG_WARPS ) k_mg_fill( const MgLevel *__restrict__ lv, const Chunk *__restrict__ chunks, int nch ) {
    extern __shared__ long long mg_pairs_smem[];
    long long ( *sk )[ MG_PAIRS ] = reinterpret_cast<long long ( * )[ MG_PAIRS ]>( mg_pairs_smem );
    float ( *sv )[ MG_PAIRS ] = reinterpret_cast<float ( * )[ MG_PAIRS ]>( mg_pairs_smem + MG_WARPS * MG_PAIRS );
    __shared__ int run[ MG_WARPS ];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const Chunk ch = chunks[ blockIdx.x ];
    const MgLevel &M = lv[ ch.prob ];
    // a refused level (see k_mg_scan) keeps only its diagonal: empty rows, nothing written past the capacity
    const bool refused = M.part[ 0 ] < 0;
    // the chunk's rows in order: each warp needs the offset of its row, i.e. the counts of the rows before it
    int at = refused ? 0 : int( M.part[ ( size_t ) ch.index * 2 + 1 ] );
    for ( int I0 = ch.begin; I0 < ch.end; I0 += MG_WARPS ) {
        const int I = I0 + warp;
        if ( lane == 0 ) run[ warp ] = I < ch.end && ! refused ? M.rcn[ I ] : 0;
        __syncthreads();
        int my = at;
        for ( int w = 0; w < warp; ++w ) my += run[ w ];
        int step = 0;
        for ( int w = 0; w < MG_WARPS; ++w ) step += run[ w ];
        __syncthreads();
        if ( I < ch.end ) {
            int cnt = gather_sorted( M, I, sk[ warp ], sv[ warp ], lane );
            if ( cnt < 0 ) cnt = 0;
            // the distinct columns in increasing order, each with its sum in pair order (its run)
            const long long *key = sk[ warp ];
            int done = 0;
            float dsum = 0;
            for ( int base = 0; base < cnt; base += 32 ) {
                int k = base + lane;
                bool first = k < cnt && run_start( key, k, I );
                float s = 0;
                if ( first ) {
                    const long long J = key[ k ] >> MG_KEY_SHIFT;
                    for ( int q = k; q < cnt && ( key[ q ] >> MG_KEY_SHIFT ) == J; ++q ) s += sv[ warp ][ key[ q ] & ( ( 1 << MG_KEY_SHIFT ) - 1 ) ];
                }
                unsigned m = __ballot_sync( 0xffffffffu, first );
                int slot = done + __popc( m & ( ( 1u << lane ) - 1 ) );
                if ( first && ! refused ) { M.coln[ my + slot ] = int( key[ k ] >> MG_KEY_SHIFT ); M.valn[ my + slot ] = s; }
                float ws = first ? s : 0.f;
                for ( int o = 16; o > 0; o >>= 1 ) ws += __shfl_xor_sync( 0xffffffffu, ws, o );
                dsum += ws;
                done += __popc( m );
            }
            if ( lane == 0 ) {
                M.rpn[ I ] = refused ? 0 : my;
                M.dian[ I ] = dsum > 0 ? dsum : 1.f;
                M.dinvn[ I ] = 1.f / ( dsum > 0 ? dsum : 1.f );
            }
        }
        at += step;
        __syncwarp();
    }
}

// the coarsest level: the dense inverse of A + mu 1 1^T (Gauss-Jordan in FP64), one warp per problem
__global__ void __launch_bounds__( 32 ) k_mg_bottom_build( const MgLevel *__restrict__ lv ) {
    const MgLevel &M = lv[ blockIdx.x ];
    const int n = M.n, lane = threadIdx.x;
    __shared__ double A[ MG_BOTTOM ][ 2 * MG_BOTTOM ];
    double mu = 0;
    for ( int i = 0; i < n; ++i ) mu += M.dia[ i ];
    mu = mu / ( n * n );
    for ( int i = 0; i < n; ++i )
        for ( int j = lane; j < 2 * n; j += 32 ) A[ i ][ j ] = j < n ? ( i == j ? double( M.dia[ i ] ) : 0.0 ) + mu : ( j - n == i ? 1.0 : 0.0 );
    __syncwarp();
    for ( int i = 0; i < n; ++i )
        for ( int e = M.rp[ i ]; e < M.rp[ i + 1 ]; ++e )
            if ( lane == 0 ) A[ i ][ M.col[ e ] ] -= M.val[ e ];
    __syncwarp();
    double dmax = 0;
    for ( int i = 0; i < n; ++i ) dmax = fmax( dmax, double( M.dia[ i ] ) );
    dmax = dmax > 0 ? dmax : 1.0;
    for ( int k = 0; k < n; ++k ) {
        __syncwarp();
        if ( lane == 0 && ! ( A[ k ][ k ] > 1e-12 * dmax ) ) A[ k ][ k ] += dmax;
        __syncwarp();
        double piv = A[ k ][ k ];
        __syncwarp();
        for ( int j = lane; j < 2 * n; j += 32 ) A[ k ][ j ] /= piv;
        __syncwarp();
        for ( int i = 0; i < n; ++i ) {
            if ( i == k ) continue;
            double f = A[ i ][ k ];
            __syncwarp();
            for ( int j = lane; j < 2 * n; j += 32 ) A[ i ][ j ] -= f * A[ k ][ j ];
            __syncwarp();
        }
    }
    for ( int i = 0; i < n; ++i )
        for ( int j = lane; j < n; j += 32 ) M.inv[ i * n + j ] = float( A[ i ][ n + j ] );
}

// ---- apply: one V(1,1) cycle --------------------------------------------------------------------------------------------
constexpr float OMEGA = 0.8f;
// the coarse-grid correction is over-corrected by ALPHA: the Galerkin operator of piecewise-constant aggregates
// underestimates the smooth error's energy, and a scaled correction (still symmetric, still positive for ALPHA < 2)
// cuts the CG iterations by about a quarter on Voronoi Laplacians
constexpr float ALPHA = 1.5f;

// the cycle's kernels give MG_LANES lanes to a row: a coarse row's fine rows are split among them (down), a fine row's
// entries (up); their sums are folded by a fixed shuffle tree (deterministic)
constexpr int MG_LANES = 4;
__device__ __forceinline__ float lanes_sum( float t ) {
#pragma unroll
    for ( int o = 1; o < MG_LANES; o <<= 1 ) t += __shfl_xor_sync( 0xffffffffu, t, o, MG_LANES );
    return t;
}
// the rows a block's lanes walk: the chunk rounded up to whole passes, so that every lane of a warp reaches each shuffle
__device__ __forceinline__ int lane_rows_end( const Chunk &ch ) {
    constexpr int per = MGT / MG_LANES;
    return ch.begin + ( ( ch.end - ch.begin + per - 1 ) / per ) * per;
}

// pre-smoothing from zero (x = w D^-1 b), the residual and its restriction to the next level, for the coarse rows
// [ I0, I1 ) of level M: MG_LANES lanes per coarse row (thread t of nt; nt a multiple of 32), each lane every MG_LANES-th of
// its fine rows; every lane of a warp reaches each shuffle
__device__ __forceinline__ void mg_down_rows( const MgLevel &M, const VecDev *V, int I0, int I1, int t, int nt ) {
    const bool top = M.level == 0;
    const int sub = t % MG_LANES, per = nt / MG_LANES;
    const int end = I0 + ( ( I1 - I0 + per - 1 ) / per ) * per;
    for ( int I = I0 + t / MG_LANES; I < end; I += per ) {
        const bool in = I < I1;
        const int i0 = I * M.pack, i1 = in ? min( M.n, i0 + M.pack ) : i0;
        float acc = 0;
        for ( int i = i0 + sub; i < i1; i += MG_LANES ) {
            float bi = top ? ( V->mixed ? V->r32[ i ] : float( V->r[ i ] ) ) : M.b[ i ];
            if ( top ) M.b[ i ] = bi;
            float xi = OMEGA * M.dinv[ i ] * bi;
            M.x[ i ] = xi;
            float ax = M.dia[ i ] * xi;
            for ( int e = M.rp[ i ]; e < M.rp[ i + 1 ]; ++e ) {
                const int j = M.col[ e ];
                float bj = top ? ( V->mixed ? V->r32[ j ] : float( V->r[ j ] ) ) : M.b[ j ];
                ax -= M.val[ e ] * OMEGA * M.dinv[ j ] * bj;
            }
            acc += bi - ax;
        }
        acc = lanes_sum( acc );
        if ( in && sub == 0 ) M.bn[ I ] = acc;
    }
}

// prolongation of the next level's solution and post-smoothing for the fine rows [ i0, i1 ) of level M; level 0 writes z
// (FP64, or z32 for the mixed CG); MG_LANES lanes per fine row
__device__ __forceinline__ void mg_up_rows( const MgLevel &M, const VecDev &V, int i0, int i1, int t, int nt ) {
    const int sub = t % MG_LANES, per = nt / MG_LANES;
    const int end = i0 + ( ( i1 - i0 + per - 1 ) / per ) * per;
    for ( int i = i0 + t / MG_LANES; i < end; i += per ) {
        const bool in = i < i1;
        const int r = in ? i : i0;
        float s = 0;
        for ( int e = M.rp[ r ] + sub; e < M.rp[ r + 1 ]; e += MG_LANES ) {
            const int j = M.col[ e ];
            s += M.val[ e ] * ( M.x[ j ] + ALPHA * M.xn[ j / M.pack ] );
        }
        s = lanes_sum( s );
        if ( in && sub == 0 ) {
            const float xi = M.x[ i ] + ALPHA * M.xn[ i / M.pack ];
            const float ai = M.dia[ i ] * xi - s;
            const float yi = xi + OMEGA * M.dinv[ i ] * ( M.b[ i ] - ai );
            if ( M.level == 0 ) {
                if ( V.mixed ) V.z32[ i ] = yi;
                else V.z[ i ] = double( yi );
            } else
                M.y[ i ] = yi;
        }
    }
}

// the coarsest level: y = inv b
__device__ __forceinline__ void mg_bottom_rows( const MgLevel &M, int t, int nt ) {
    const int n = M.n;
    for ( int i = t; i < n; i += nt ) {
        float s = 0;
        for ( int j = 0; j < n; ++j ) s += M.inv[ i * n + j ] * M.b[ j ];
        M.y[ i ] = s;
    }
}

__device__ __forceinline__ bool mg_idle( const VecDev &V ) { return V.sc[ SC_CONV ] != 0 || V.sc[ SC_REFINE ] != 0; }

__global__ void __launch_bounds__( MGT ) k_mg_down( const MgLevel *__restrict__ lv, const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks,
                                                   int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const MgLevel &M = lv[ ch.prob ];
    const VecDev *V = vs + M.vec;
    if ( mg_idle( *V ) ) return;
    mg_down_rows( M, V, ch.begin, ch.end, threadIdx.x, MGT );
}

// the coarsest level: x = inv b (one warp per problem)
__global__ void __launch_bounds__( 32 ) k_mg_bottom( const MgLevel *__restrict__ lv, const VecDev *__restrict__ vs ) {
    const MgLevel &M = lv[ blockIdx.x ];
    if ( mg_idle( vs[ M.vec ] ) ) return;
    mg_bottom_rows( M, threadIdx.x, 32 );
}

__global__ void __launch_bounds__( MGT ) k_mg_up( const MgLevel *__restrict__ lv, const VecDev *__restrict__ vs, const Chunk *__restrict__ chunks,
                                                 int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const MgLevel &M = lv[ ch.prob ];
    const VecDev &V = vs[ M.vec ];
    if ( mg_idle( V ) ) return;
    mg_up_rows( M, V, ch.begin, ch.end, threadIdx.x, MGT );
}

// THE SMALL LEVELS OF A CYCLE IN ONE LAUNCH: one block per problem walks its levels from the first one of at most
// MG_FUSE_ROWS rows down to the coarsest and back up (chain[ first .. first + count ), `idx` per problem), the block's
// threads synchronised between levels.  A launch per level and direction there would cost more in launch latency than
// the levels cost in work (a few thousand rows each, most of them a few hundred).
constexpr int MGF = 1024;
__global__ void __launch_bounds__( MGF ) k_mg_fused( const MgLevel *__restrict__ chain, const int2 *__restrict__ idx, const VecDev *__restrict__ vs ) {
    const int2 c = idx[ blockIdx.x ];
    const MgLevel *L = chain + c.x;
    const VecDev &V = vs[ L[ 0 ].vec ];
    if ( mg_idle( V ) ) return;                 // (block-uniform: one problem per block)
    for ( int k = 0; k + 1 < c.y; ++k ) {
        mg_down_rows( L[ k ], &V, 0, L[ k ].nn, threadIdx.x, MGF );
        __syncthreads();
    }
    mg_bottom_rows( L[ c.y - 1 ], threadIdx.x, MGF );
    __syncthreads();
    for ( int k = c.y - 2; k >= 0; --k ) {
        mg_up_rows( L[ k ], V, 0, L[ k ].n, threadIdx.x, MGF );
        __syncthreads();
    }
}

void launch_mg_fused( const Launch &L, const MgLevel *chain, const int2 *idx, const VecDev *vs, int nprob ) {
    if ( nprob <= 0 ) return;
    k_mg_fused<<<nprob, MGF, 0, L.stream>>>( chain, idx, vs );
    ++*L.launches;
}

void launch_mg_level0( const Launch &L, const MgLevel *lv, const VecDev *vs, const Chunk *ch, int nch ) {
    if ( nch <= 0 ) return;
    k_mg_rest<<<nch, MGT, 0, L.stream>>>( lv, vs, ch, nch );
    ++*L.launches;
    k_mg_level0<<<nch, MGT, 0, L.stream>>>( lv, vs, ch, nch );
    ++*L.launches;
}
void launch_mg_coarsen( const Launch &L, const MgLevel *lv, int nprob, const Chunk *ch, int nch, ErrRec *err ) {
    if ( nch <= 0 ) return;
    // the pairs of each warp's coarse row: MG_PAIRS keys (8 bytes) and values (4 bytes)
    constexpr int smem = MG_WARPS * MG_PAIRS * 12;
    static bool configured = false;
    if ( ! configured ) {
        cudaFuncSetAttribute( k_mg_count, cudaFuncAttributeMaxDynamicSharedMemorySize, smem );
        cudaFuncSetAttribute( k_mg_fill, cudaFuncAttributeMaxDynamicSharedMemorySize, smem );
        configured = true;
    }
    k_mg_count<<<nch, 32 * MG_WARPS, smem, L.stream>>>( lv, ch, nch, err );
    k_mg_scan<<<nprob, 1024, 0, L.stream>>>( lv );
    k_mg_fill<<<nch, 32 * MG_WARPS, smem, L.stream>>>( lv, ch, nch );
    *L.launches += 3;
}
void launch_mg_bottom_build( const Launch &L, const MgLevel *lv, int nprob ) {
    if ( nprob <= 0 ) return;
    k_mg_bottom_build<<<nprob, 32, 0, L.stream>>>( lv );
    ++*L.launches;
}
void launch_mg_down( const Launch &L, const MgLevel *lv, const VecDev *vs, const Chunk *ch, int nch ) {
    if ( nch <= 0 ) return;
    k_mg_down<<<nch, MGT, 0, L.stream>>>( lv, vs, ch, nch );
    ++*L.launches;
}
void launch_mg_bottom( const Launch &L, const MgLevel *lv, const VecDev *vs, int nprob ) {
    if ( nprob <= 0 ) return;
    k_mg_bottom<<<nprob, 32, 0, L.stream>>>( lv, vs );
    ++*L.launches;
}
void launch_mg_up( const Launch &L, const MgLevel *lv, const VecDev *vs, const Chunk *ch, int nch ) {
    if ( nch <= 0 ) return;
    k_mg_up<<<nch, MGT, 0, L.stream>>>( lv, vs, ch, nch );
    ++*L.launches;
}

} // namespace sdot

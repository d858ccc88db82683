// The acceleration structure, built on the device: a uniform grid whose cells are ranked in Morton
// order.  It plays the role of the reference's median-cut BSP (src/sdot/AaBsp.py:16-100,
// gpu/Bsp2D.cuh:366-456): consecutive ranks are neighbours in space, and every seed is found by the
// cell it falls in.  Its weight majorants are a pyramid of maxima over the grid (below).
#include "internal.h"

namespace sdot {

__device__ __forceinline__ int grid_coord( double x, double o, double h, int g ) {
    int k = int( floor( ( x - o ) / h ) );
    return k < 0 ? 0 : ( k >= g ? g - 1 : k );
}

__device__ __forceinline__ unsigned long long spread2( unsigned long long v ) {      // 32 bits -> every other bit
    v &= 0xffffffffull;
    v = ( v | ( v << 16 ) ) & 0x0000ffff0000ffffull;
    v = ( v | ( v << 8 ) ) & 0x00ff00ff00ff00ffull;
    v = ( v | ( v << 4 ) ) & 0x0f0f0f0f0f0f0f0full;
    v = ( v | ( v << 2 ) ) & 0x3333333333333333ull;
    v = ( v | ( v << 1 ) ) & 0x5555555555555555ull;
    return v;
}
__device__ __forceinline__ unsigned long long spread3( unsigned long long v ) {      // 21 bits -> every third bit
    v &= 0x1fffffull;
    v = ( v | ( v << 32 ) ) & 0x1f00000000ffffull;
    v = ( v | ( v << 16 ) ) & 0x1f0000ff0000ffull;
    v = ( v | ( v << 8 ) ) & 0x100f00f00f00f00full;
    v = ( v | ( v << 4 ) ) & 0x10c30c30c30c30c3ull;
    v = ( v | ( v << 2 ) ) & 0x1249249249249249ull;
    return v;
}

__global__ void k_bbox( const double *__restrict__ pos, int n, int dim, unsigned long long *mm ) {
    double lo[ 3 ] = { 1e300, 1e300, 1e300 }, hi[ 3 ] = { -1e300, -1e300, -1e300 };
    for ( int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x )
        for ( int a = 0; a < dim; ++a ) {
            double x = pos[ ( size_t ) i * dim + a ];
            lo[ a ] = fmin( lo[ a ], x );
            hi[ a ] = fmax( hi[ a ], x );
        }
    for ( int a = 0; a < dim; ++a ) {
        double l = warp_min( lo[ a ] ), h = warp_max( hi[ a ] );
        if ( lane_id() == 0 ) {
            atomicMin( mm + a, dbl_order( l ) );
            atomicMax( mm + dim + a, dbl_order( h ) );
        }
    }
}

void launch_bbox( const Launch &L, const double *pos, int n, int dim, unsigned long long *mm ) {
    int blocks = n / 256 + 1;
    if ( blocks > 592 ) blocks = 592;
    k_bbox<<<blocks, 256, 0, L.stream>>>( pos, n, dim, mm );
    ++*L.launches;
}

struct GridArgs { int g[ 3 ]; double go[ 3 ], gh[ 3 ]; };

__global__ void k_keys( const double *__restrict__ pos, int n, int dim, GridArgs G, unsigned long long *keys, int *vals ) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if ( i >= n ) return;
    unsigned long long k = 0;
    if ( dim == 2 ) {
        int cx = grid_coord( pos[ 2 * ( size_t ) i ], G.go[ 0 ], G.gh[ 0 ], G.g[ 0 ] );
        int cy = grid_coord( pos[ 2 * ( size_t ) i + 1 ], G.go[ 1 ], G.gh[ 1 ], G.g[ 1 ] );
        k = spread2( cx ) | ( spread2( cy ) << 1 );
    } else {
        int cx = grid_coord( pos[ 3 * ( size_t ) i ], G.go[ 0 ], G.gh[ 0 ], G.g[ 0 ] );
        int cy = grid_coord( pos[ 3 * ( size_t ) i + 1 ], G.go[ 1 ], G.gh[ 1 ], G.g[ 1 ] );
        int cz = grid_coord( pos[ 3 * ( size_t ) i + 2 ], G.go[ 2 ], G.gh[ 2 ], G.g[ 2 ] );
        k = spread3( cx ) | ( spread3( cy ) << 1 ) | ( spread3( cz ) << 2 );
    }
    keys[ i ] = k;
    vals[ i ] = i;
}

void launch_keys( const Launch &L, const double *pos, int n, int dim, const int *g, const double *go, const double *gh, int bits,
                  unsigned long long *keys, int *vals ) {
    (void) bits;
    GridArgs G;
    for ( int a = 0; a < 3; ++a ) { G.g[ a ] = g[ a ]; G.go[ a ] = go[ a ]; G.gh[ a ] = gh[ a ]; }
    k_keys<<<( n + 255 ) / 256, 256, 0, L.stream>>>( pos, n, dim, G, keys, vals );
    ++*L.launches;
}

// ---- THE SORT of the Morton keys (the reference sorts its own keys too, gpu/Bsp2D.cuh:72-186) --------------------------------
// A stable least-significant-digit radix sort of ( key, value ) pairs on the keys' low `bits` bits, 8 bits a pass, three
// launches a pass: the digit histogram of every tile of RS_TILE keys (digit-major: [ digit ][ tile ]), its exclusive scan
// (the place of each tile's keys of each digit), and the scatter, which ranks a tile's keys of one digit in index order --
// 8 rounds of 256 consecutive keys, a warp's equal digits found by __match_any_sync, the warps' counts summed in warp
// order -- so that equal digits keep their order and every pass is stable.
constexpr int RS_T = 256, RS_K = 8, RS_TILE = RS_T * RS_K, RS_BINS = 256;

__global__ void __launch_bounds__( RS_T ) k_rs_hist( const unsigned long long *__restrict__ keys, int n, int shift, int *hist, int tiles ) {
    __shared__ int h[ RS_BINS ];
    h[ threadIdx.x ] = 0;
    __syncthreads();
    const int t0 = blockIdx.x * RS_TILE;
    for ( int k = threadIdx.x; k < RS_TILE; k += RS_T ) {
        const int i = t0 + k;
        if ( i < n ) atomicAdd( &h[ int( ( keys[ i ] >> shift ) & 0xff ) ], 1 );
    }
    __syncthreads();
    hist[ ( size_t ) threadIdx.x * tiles + blockIdx.x ] = h[ threadIdx.x ];
}

// exclusive scan of `count` ints in place, one block of 1024 threads (warp scans, then the warps' totals)
__global__ void __launch_bounds__( 1024 ) k_rs_scan( int *v, long count ) {
    __shared__ int wt[ 32 ];
    __shared__ long long carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if ( threadIdx.x == 0 ) carry = 0;
    __syncthreads();
    for ( long base = 0; base < count; base += 1024 ) {
        const long i = base + threadIdx.x;
        const int x = i < count ? v[ i ] : 0;
        int inc = x;
#pragma unroll
        for ( int o = 1; o < 32; o <<= 1 ) { const int t = __shfl_up_sync( 0xffffffffu, inc, o ); if ( lane >= o ) inc += t; }
        if ( lane == 31 ) wt[ warp ] = inc;
        __syncthreads();
        if ( warp == 0 ) {
            int w = wt[ lane ], wi = w;
#pragma unroll
            for ( int o = 1; o < 32; o <<= 1 ) { const int t = __shfl_up_sync( 0xffffffffu, wi, o ); if ( lane >= o ) wi += t; }
            wt[ lane ] = wi - w;                               // exclusive prefix of the warps' totals
        }
        __syncthreads();
        const long long c = carry;
        if ( i < count ) v[ i ] = int( c + wt[ warp ] + inc - x );
        __syncthreads();
        if ( threadIdx.x == 1023 ) carry = c + wt[ warp ] + inc;
        __syncthreads();
    }
}

__global__ void __launch_bounds__( RS_T ) k_rs_scatter( const unsigned long long *__restrict__ kin, const int *__restrict__ vin,
                                                       unsigned long long *kout, int *vout, int n, int shift, const int *__restrict__ off,
                                                       int tiles ) {
    __shared__ int cnt[ RS_T / 32 ][ RS_BINS ];
    __shared__ int base[ RS_BINS ];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    base[ threadIdx.x ] = off[ ( size_t ) threadIdx.x * tiles + blockIdx.x ];
    const int t0 = blockIdx.x * RS_TILE;
    for ( int r = 0; r < RS_K; ++r ) {
        for ( int w = 0; w < RS_T / 32; ++w ) cnt[ w ][ threadIdx.x ] = 0;
        __syncthreads();
        const int i = t0 + r * RS_T + threadIdx.x;
        const bool in = i < n;
        unsigned long long key = 0;
        int val = 0, d = RS_BINS;                          // (RS_BINS: no key)
        if ( in ) { key = kin[ i ]; val = vin[ i ]; d = int( ( key >> shift ) & 0xff ); }
        const unsigned peers = __match_any_sync( 0xffffffffu, d );
        const int lower = __popc( peers & ( ( 1u << lane ) - 1 ) );
        if ( in && lower == 0 ) cnt[ warp ][ d ] = __popc( peers );
        __syncthreads();
        if ( in ) {
            int rank = base[ d ] + lower;
            for ( int w = 0; w < warp; ++w ) rank += cnt[ w ][ d ];
            kout[ rank ] = key;
            vout[ rank ] = val;
        }
        __syncthreads();
        int add = 0;
        for ( int w = 0; w < RS_T / 32; ++w ) add += cnt[ w ][ threadIdx.x ];
        base[ threadIdx.x ] += add;
        __syncthreads();
    }
}

size_t radix_temp_bytes( int n, int bits ) {
    (void) bits;
    const size_t tiles = ( size_t( n ) + RS_TILE - 1 ) / RS_TILE;
    return ( ( size_t( n ) * 8 + 255 ) & ~size_t( 255 ) ) + ( ( size_t( n ) * 4 + 255 ) & ~size_t( 255 ) ) + tiles * RS_BINS * 4 + 256;
}

void radix_sort( const Launch &L, void *temp, size_t temp_bytes, const unsigned long long *kin, unsigned long long *kout, const int *vin,
                 int *vout, int n, int bits ) {
    (void) temp_bytes;
    if ( n <= 0 ) return;
    const int passes = ( bits + 7 ) / 8;
    if ( passes == 0 ) {
        cudaMemcpyAsync( kout, kin, size_t( n ) * 8, cudaMemcpyDeviceToDevice, L.stream );
        cudaMemcpyAsync( vout, vin, size_t( n ) * 4, cudaMemcpyDeviceToDevice, L.stream );
        return;
    }
    const int tiles = ( n + RS_TILE - 1 ) / RS_TILE;
    char *t = static_cast<char *>( temp );
    unsigned long long *kt = reinterpret_cast<unsigned long long *>( t );
    int *vt = reinterpret_cast<int *>( t + ( ( size_t( n ) * 8 + 255 ) & ~size_t( 255 ) ) );
    int *hist = reinterpret_cast<int *>( reinterpret_cast<char *>( vt ) + ( ( size_t( n ) * 4 + 255 ) & ~size_t( 255 ) ) );
    const unsigned long long *ks = kin;
    const int *vs = vin;
    for ( int p = 0; p < passes; ++p ) {
        // the last pass writes the output; the passes before alternate so that it does
        const bool to_out = ( passes - 1 - p ) % 2 == 0;
        unsigned long long *kd = to_out ? kout : kt;
        int *vd = to_out ? vout : vt;
        k_rs_hist<<<tiles, RS_T, 0, L.stream>>>( ks, n, 8 * p, hist, tiles );
        k_rs_scan<<<1, 1024, 0, L.stream>>>( hist, long( tiles ) * RS_BINS );
        k_rs_scatter<<<tiles, RS_T, 0, L.stream>>>( ks, vs, kd, vd, n, 8 * p, hist, tiles );
        *L.launches += 3;
        ks = kd;
        vs = vd;
    }
}

__global__ void k_gather( const double *__restrict__ pos, const int *__restrict__ vals, int n, int dim, double *pos_ranked, int *user,
                          int *rank_of, const double *__restrict__ w_user, double *w_ranked ) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if ( s >= n ) return;
    int u = vals[ s ];
    user[ s ] = u;
    rank_of[ u ] = s;
    for ( int a = 0; a < dim; ++a ) pos_ranked[ ( size_t ) s * dim + a ] = pos[ ( size_t ) u * dim + a ];
    if ( w_ranked ) w_ranked[ s ] = w_user ? w_user[ u ] : 0.0;
}

void launch_gather( const Launch &L, const double *pos, const int *vals, int n, int dim, double *pos_ranked, int *user, int *rank_of,
                    const double *w_user, double *w_ranked ) {
    k_gather<<<( n + 255 ) / 256, 256, 0, L.stream>>>( pos, vals, n, dim, pos_ranked, user, rank_of, w_user, w_ranked );
    ++*L.launches;
}

__global__ void k_cell_ranges( const unsigned long long *__restrict__ keys, const double *__restrict__ pos, int n, int dim, GridArgs G,
                               int2 *cell_range ) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if ( s >= n ) return;
    bool first = s == 0 || keys[ s ] != keys[ s - 1 ];
    bool last = s == n - 1 || keys[ s ] != keys[ s + 1 ];
    if ( ! first && ! last ) return;
    long c = 0;
    for ( int a = dim - 1; a >= 0; --a ) c = c * G.g[ a ] + grid_coord( pos[ ( size_t ) s * dim + a ], G.go[ a ], G.gh[ a ], G.g[ a ] );
    if ( first ) cell_range[ c ].x = s;
    if ( last ) cell_range[ c ].y = s + 1;
}

void launch_cell_ranges( const Launch &L, const unsigned long long *keys, const double *pos_ranked, int n, int dim, const int *g,
                         const double *go, const double *gh, int2 *cell_range ) {
    GridArgs G;
    for ( int a = 0; a < 3; ++a ) { G.g[ a ] = g[ a ]; G.go[ a ] = go[ a ]; G.gh[ a ] = gh[ a ]; }
    k_cell_ranges<<<( n + 255 ) / 256, 256, 0, L.stream>>>( keys, pos_ranked, n, dim, G, cell_range );
    ++*L.launches;
}

// image row prefix: pre[ j * ( nx + 1 ) + i ] = hx * sum_{i' < i} values[ i' * ny + j ]
__global__ void k_image_prefix( const double *__restrict__ v, int nx, int ny, double hx, double *pre ) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if ( j >= ny ) return;
    double s = 0;
    pre[ ( size_t ) j * ( nx + 1 ) ] = 0;
    for ( int i = 0; i < nx; ++i ) {
        s += v[ ( size_t ) i * ny + j ] * hx;
        pre[ ( size_t ) j * ( nx + 1 ) + i + 1 ] = s;
    }
}

void launch_image_prefix( const Launch &L, const double *values, int nx, int ny, double hx, double *pre ) {
    k_image_prefix<<<( ny + 127 ) / 128, 128, 0, L.stream>>>( values, nx, ny, hx, pre );
    ++*L.launches;
}

// the image continuation's blur along one axis (sdotplan/convolved/Image.h:51-74): dst = sum_k ker src( . + k ) / sum_k ker
// over the taps inside the axis, k ascending, without contraction (the same sums as a plain CPU loop)
__global__ void k_blur_axis( const double *__restrict__ src, double *__restrict__ dst, int nx, int ny, int axis, int r,
                             const double *__restrict__ ker ) {
    const size_t flat = size_t( blockIdx.x ) * blockDim.x + threadIdx.x;
    if ( flat >= size_t( nx ) * ny ) return;
    const int i = int( flat / ny ), j = int( flat % ny );
    const int p = axis ? j : i, len = axis ? ny : nx;
    const long stride = axis ? 1 : ny;
    const int lo = -r > -p ? -r : -p, hi = r < len - 1 - p ? r : len - 1 - p;
    double sum = 0, ws = 0;
    for ( int k = lo; k <= hi; ++k ) {
        const double t = ker[ k + r ];
        sum = __dadd_rn( sum, __dmul_rn( t, src[ long( flat ) + k * stride ] ) );
        ws = __dadd_rn( ws, t );
    }
    dst[ flat ] = sum / ws;
}

void launch_blur_axis( const Launch &L, const double *src, double *dst, int nx, int ny, int axis, int r, const double *ker ) {
    const size_t tot = size_t( nx ) * ny;
    k_blur_axis<<<unsigned( ( tot + 255 ) / 256 ), 256, 0, L.stream>>>( src, dst, nx, ny, axis, r, ker );
    ++*L.launches;
}

__global__ void k_wmax( const double *__restrict__ w, int n, unsigned long long *slot ) {
    double m = -1e300;
    for ( int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x ) m = fmax( m, w[ i ] );
    m = warp_max( m );
    if ( lane_id() == 0 ) atomicMax( slot, dbl_order( m ) );
}
void launch_wmax( const Launch &L, const double *w, int n, unsigned long long *slot ) {
    int blocks = n / 256 + 1;
    if ( blocks > 592 ) blocks = 592;
    k_wmax<<<blocks, 256, 0, L.stream>>>( w, n, slot );
    ++*L.launches;
}
__global__ void k_finish_wmax( unsigned long long *slot, double *wmax, int count ) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if ( i < count ) wmax[ i ] = order_dbl( slot[ i ] );
}
void launch_finish_wmax( const Launch &L, unsigned long long *slot, double *wmax, int count ) {
    k_finish_wmax<<<( count + 127 ) / 128, 128, 0, L.stream>>>( slot, wmax, count );
    ++*L.launches;
}

// ---- weight majorants ------------------------------------------------------------------------------------------------
// Every grid cell, then every 2x2 (2x2x2) block of the level below up to a single block, gets an affine majorant of the
// weights of its seeds: w_j <= a . p_j + b.  a is the least-squares slope of the block's weights (0 on the grid's own
// cells, which hold two seeds or so), b the exact max of w_j - a . p_j; correctness needs only b, the slope only
// sharpens the pruning.  The cell kernels skip a block that cannot claim any vertex of the current cell (wmaj_may_cut):
// the per-node affine majorants of the reference's tree (gpu/Majorant2D.cuh:3-28, 253; Pruning.h:1-30) on the grid's
// pyramid.  Record of a node: a[ dim ], then b as an ordered integer (-1e300: no seed).
long wpyr_layout( int dim, const int *g, int &nlev, int *poff ) {
    long total = 0;
    nlev = 0;
    for ( int l = 0; l < MAX_LEV; ++l ) {
        long sz = 1;
        bool one = true;
        for ( int a = 0; a < dim; ++a ) { int d = lev_dim( g[ a ], l ); sz *= d; one = one && d == 1; }
        poff[ l ] = int( total );
        total += sz;
        nlev = l + 1;
        if ( one ) break;
    }
    return total;
}

// level 0: the moments of each cell's seeds (n, sum p, sum w, sum p p^T (upper), sum p w) and its record (a = 0, b = max w)
__global__ void k_wpyr0( const ProbDev *__restrict__ probs ) {
    const ProbDev &P = probs[ blockIdx.y ];
    if ( ! P.wpyr ) return;
    const int dim = P.dim, RS = dim + 1, MS = wmom_size( dim );
    long ncell = 1;
    for ( int a = 0; a < dim; ++a ) ncell *= P.g[ a ];
    for ( long c = long( blockIdx.x ) * blockDim.x + threadIdx.x; c < ncell; c += long( gridDim.x ) * blockDim.x ) {
        int2 rg = P.cell_range[ c ];
        double m = -1e300, mom[ 14 ];
        for ( int k = 0; k < MS; ++k ) mom[ k ] = 0;
        for ( int j = rg.x; j < rg.y; ++j ) {
            const double w = P.w ? P.w[ j ] : 0.0;
            m = fmax( m, w );
            double x[ 3 ];
            for ( int a = 0; a < dim; ++a ) x[ a ] = P.pos[ ( size_t ) j * dim + a ];
            int k = 0;
            mom[ k++ ] += 1;
            for ( int a = 0; a < dim; ++a ) mom[ k++ ] += x[ a ];
            mom[ k++ ] += w;
            for ( int a = 0; a < dim; ++a )
                for ( int b = a; b < dim; ++b ) mom[ k++ ] += x[ a ] * x[ b ];
            for ( int a = 0; a < dim; ++a ) mom[ k++ ] += x[ a ] * w;
        }
        for ( int k = 0; k < MS; ++k ) P.wmom[ c * MS + k ] = mom[ k ];
        for ( int a = 0; a < dim; ++a ) P.wpyr[ c * RS + a ] = 0;
        reinterpret_cast<unsigned long long *>( P.wpyr )[ c * RS + dim ] = dbl_order( m );
    }
}

// the least-squares slope of the weights from a node's moments (0 when too few or degenerate seeds)
__device__ void fit_slope( const double *mom, int dim, double *a ) {
    for ( int q = 0; q < dim; ++q ) a[ q ] = 0;
    const double n = mom[ 0 ];
    if ( n < dim + 1 ) return;
    double mean[ 3 ], C[ 3 ][ 3 ], r[ 3 ];
    for ( int q = 0; q < dim; ++q ) mean[ q ] = mom[ 1 + q ] / n;
    const double mw = mom[ 1 + dim ] / n;
    int k = 2 + dim;
    for ( int q = 0; q < dim; ++q )
        for ( int t = q; t < dim; ++t ) { C[ q ][ t ] = C[ t ][ q ] = mom[ k++ ] / n - mean[ q ] * mean[ t ]; }
    for ( int q = 0; q < dim; ++q ) r[ q ] = mom[ k++ ] / n - mean[ q ] * mw;
    double tr = 0;
    for ( int q = 0; q < dim; ++q ) tr += C[ q ][ q ];
    if ( ! ( tr > 0 ) ) return;
    if ( dim == 2 ) {
        double det = C[ 0 ][ 0 ] * C[ 1 ][ 1 ] - C[ 0 ][ 1 ] * C[ 0 ][ 1 ];
        if ( ! ( det > 1e-6 * tr * tr ) ) return;
        a[ 0 ] = ( r[ 0 ] * C[ 1 ][ 1 ] - r[ 1 ] * C[ 0 ][ 1 ] ) / det;
        a[ 1 ] = ( r[ 1 ] * C[ 0 ][ 0 ] - r[ 0 ] * C[ 0 ][ 1 ] ) / det;
    } else {
        double c00 = C[ 1 ][ 1 ] * C[ 2 ][ 2 ] - C[ 1 ][ 2 ] * C[ 2 ][ 1 ], c01 = C[ 1 ][ 2 ] * C[ 2 ][ 0 ] - C[ 1 ][ 0 ] * C[ 2 ][ 2 ],
               c02 = C[ 1 ][ 0 ] * C[ 2 ][ 1 ] - C[ 1 ][ 1 ] * C[ 2 ][ 0 ];
        double det = C[ 0 ][ 0 ] * c00 + C[ 0 ][ 1 ] * c01 + C[ 0 ][ 2 ] * c02;
        if ( ! ( det > 1e-9 * tr * tr * tr ) ) return;
        for ( int q = 0; q < 3; ++q ) {
            double M[ 3 ][ 3 ];
            for ( int i = 0; i < 3; ++i )
                for ( int j = 0; j < 3; ++j ) M[ i ][ j ] = j == q ? r[ i ] : C[ i ][ j ];
            double d = M[ 0 ][ 0 ] * ( M[ 1 ][ 1 ] * M[ 2 ][ 2 ] - M[ 1 ][ 2 ] * M[ 2 ][ 1 ] ) - M[ 0 ][ 1 ] * ( M[ 1 ][ 0 ] * M[ 2 ][ 2 ] - M[ 1 ][ 2 ] * M[ 2 ][ 0 ] ) +
                       M[ 0 ][ 2 ] * ( M[ 1 ][ 0 ] * M[ 2 ][ 1 ] - M[ 1 ][ 1 ] * M[ 2 ][ 0 ] );
            a[ q ] = d / det;
        }
    }
    for ( int q = 0; q < dim; ++q ) if ( ! isfinite( a[ q ] ) ) { for ( int t = 0; t < dim; ++t ) a[ t ] = 0; return; }
}

// the levels above: moments summed from the children, the slope fitted, b reset (one block per problem, level by level)
__global__ void __launch_bounds__( 1024 ) k_wpyr_up( const ProbDev *__restrict__ probs ) {
    const ProbDev &P = probs[ blockIdx.x ];
    if ( ! P.wpyr ) return;
    const int dim = P.dim, RS = dim + 1, MS = wmom_size( dim );
    for ( int l = 1; l < P.nlev; ++l ) {
        int d[ 3 ] = { 1, 1, 1 }, e[ 3 ] = { 1, 1, 1 };
        for ( int a = 0; a < dim; ++a ) { d[ a ] = lev_dim( P.g[ a ], l ); e[ a ] = lev_dim( P.g[ a ], l - 1 ); }
        const long src = P.poff[ l - 1 ], dst = P.poff[ l ];
        const long cnt = long( d[ 0 ] ) * d[ 1 ] * d[ 2 ];
        for ( long c = threadIdx.x; c < cnt; c += blockDim.x ) {
            int X = int( c % d[ 0 ] ), Y = int( ( c / d[ 0 ] ) % d[ 1 ] ), Z = int( c / ( long( d[ 0 ] ) * d[ 1 ] ) );
            double mom[ 14 ];
            for ( int k = 0; k < MS; ++k ) mom[ k ] = 0;
            for ( int dz = 0; dz < ( dim == 3 ? 2 : 1 ); ++dz )
                for ( int dy = 0; dy < 2; ++dy )
                    for ( int dx = 0; dx < 2; ++dx ) {
                        int x = 2 * X + dx, y = 2 * Y + dy, z = 2 * Z + dz;
                        if ( x < e[ 0 ] && y < e[ 1 ] && z < e[ 2 ] ) {
                            const double *cm = P.wmom + ( src + ( long( z ) * e[ 1 ] + y ) * e[ 0 ] + x ) * MS;
                            for ( int k = 0; k < MS; ++k ) mom[ k ] += cm[ k ];
                        }
                    }
            for ( int k = 0; k < MS; ++k ) P.wmom[ ( dst + c ) * MS + k ] = mom[ k ];
            double a[ 3 ];
            fit_slope( mom, dim, a );
            for ( int q = 0; q < dim; ++q ) P.wpyr[ ( dst + c ) * RS + q ] = a[ q ];
            reinterpret_cast<unsigned long long *>( P.wpyr )[ ( dst + c ) * RS + dim ] = dbl_order( -1e300 );
        }
        __syncthreads();
    }
}

// b of the levels above the grid: the max of w_j - a . p_j over each node's seeds.  Seeds are in Morton order, so those
// of one node are consecutive: a segmented max across the warp, then one atomic per segment
__global__ void k_wpyr_b( const ProbDev *__restrict__ probs ) {
    const ProbDev &P = probs[ blockIdx.y ];
    if ( ! P.wpyr ) return;
    const int dim = P.dim, RS = dim + 1, lane = threadIdx.x & 31;
    unsigned long long *B = reinterpret_cast<unsigned long long *>( P.wpyr );
    const long gw = ( long( blockIdx.x ) * blockDim.x + threadIdx.x ) >> 5, nw = ( long( gridDim.x ) * blockDim.x ) >> 5;
    for ( long j0 = gw * 32; j0 < P.n; j0 += nw * 32 ) {      // 32 consecutive seeds per warp
        const long j = j0 + lane;
        const bool ok = j < P.n;
        int c[ 3 ] = { 0, 0, 0 };
        double x[ 3 ] = { 0, 0, 0 }, w = 0;
        if ( ok ) {
            w = P.w ? P.w[ j ] : 0.0;
            for ( int a = 0; a < dim; ++a ) {
                x[ a ] = P.pos[ ( size_t ) j * dim + a ];
                int k = int( floor( ( x[ a ] - P.go[ a ] ) / P.gh[ a ] ) );
                c[ a ] = k < 0 ? 0 : ( k >= P.g[ a ] ? P.g[ a ] - 1 : k );
            }
        }
        for ( int l = 1; l < P.nlev; ++l ) {
            long node = -1;
            if ( ok ) {
                long idx = 0;
                for ( int a = dim - 1; a >= 0; --a ) idx = idx * lev_dim( P.g[ a ], l ) + ( c[ a ] >> l );
                node = P.poff[ l ] + idx;
            }
            double v = -1e300;
            if ( ok ) {
                v = w;
                for ( int a = 0; a < dim; ++a ) v -= P.wpyr[ node * RS + a ] * x[ a ];
            }
            for ( int o = 1; o < 32; o <<= 1 ) {
                double vo = __shfl_down_sync( 0xffffffffu, v, o );
                long no = __shfl_down_sync( 0xffffffffu, node, o );
                if ( lane + o < 32 && no == node ) v = fmax( v, vo );
            }
            long prev = __shfl_up_sync( 0xffffffffu, node, 1 );
            if ( ok && ( lane == 0 || prev != node ) ) atomicMax( &B[ node * RS + dim ], dbl_order( v ) );
        }
    }
}

void launch_wpyr( const Launch &L, const ProbDev *probs, int nprob ) {
    if ( nprob <= 0 ) return;
    k_wpyr0<<<dim3( 64, nprob ), 256, 0, L.stream>>>( probs );
    k_wpyr_up<<<nprob, 1024, 0, L.stream>>>( probs );
    k_wpyr_b<<<dim3( 64, nprob ), 256, 0, L.stream>>>( probs );
    *L.launches += 3;
}

} // namespace sdot

// The acceleration structure, built on the device: a uniform grid whose cells are ranked in Morton
// order.  It plays the role of the reference's median-cut BSP (src/sdot/AaBsp.py:16-100,
// gpu/Bsp2D.cuh:366-456): consecutive ranks are neighbours in space, and every seed is found by the
// cell it falls in.  Unlike a tree it has no per-node majorants: the neighbour search is bounded by a
// security radius on the largest weight instead (cells*.cu).
#include "internal.h"
#include <cub/device/device_radix_sort.cuh>

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

size_t radix_temp_bytes( int n, int bits ) {
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs( nullptr, bytes, ( const unsigned long long * ) nullptr, ( unsigned long long * ) nullptr,
                                     ( const int * ) nullptr, ( int * ) nullptr, n, 0, bits );
    return bytes;
}

void radix_sort( const Launch &L, void *temp, size_t temp_bytes, const unsigned long long *kin, unsigned long long *kout, const int *vin,
                 int *vout, int n, int bits ) {
    cub::DeviceRadixSort::SortPairs( temp, temp_bytes, kin, kout, vin, vout, n, 0, bits, L.stream );
    *L.launches += ( bits + 7 ) / 8 + 1;
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

} // namespace sdot

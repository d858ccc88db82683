// `sdot_linear_solve_noalloc`: the Jacobi-preconditioned CG of `sdot_linear_solve` (method 0) with every work
// array in one static device array of this file, so that a call allocates no device memory at all.
//
// Who needs it: a caller that cannot allocate while it solves -- one whose framework has already reserved the
// GPU's free memory for its own caching allocator (a cudaMalloc would fail there), or one in a latency-bound loop
// that must not pay the device-wide synchronisation of cudaFree.  The price is a fixed size: at most
// SDOT_NOALLOC_MAX_ROWS rows, and every call on a device shares the one array, so two calls that overlap in time
// (two host threads, or two contexts on one device) corrupt each other's work vectors.  Calls made through one
// context are serialised by its mutex; across contexts the caller serialises them.
//
// The array's device address is looked up once per device, on the first call made with that device current
// (cudaGetSymbolAddress; host code cannot take the address of a __device__ symbol).  That first call should
// come before any stream capture on the device.  The address is kept for the life of the process, so the library
// must not outlive a reset of a device it has used (cudaDeviceReset, or the primary context destroyed and made
// again): after one, the next call would write through the stale address.
//
// The array is part of the library's device code: every device on which the library's module is loaded holds its
// 16 MB until the process exits, whether or not this entry point is ever called.
//
// The kernels read the caller's matrix and vectors in place (nothing is staged through a copy), so every array
// must be memory of the context's own device, or managed memory; memory of another GPU is refused before any
// launch (SDOT_ERR_ARGS) -- without peer access a kernel reading it would fault.
//
// The kernels are those of `sdot_linear_solve`: only the rhs' mean differs, a deterministic block reduction on
// the device here, a sequential host sum there (the solutions agree to rounding).
#include "engine.h"
#include <cstring>
#include <mutex>

using namespace sdot;

namespace {

constexpr long NA_ROWS = SDOT_NOALLOC_MAX_ROWS;
constexpr long NA_CHUNKS = ( NA_ROWS + VCHUNK - 1 ) / VCHUNK;
constexpr size_t al256( size_t b ) { return ( b + 255 ) & ~size_t( 255 ); }

// the layout of the static array (every part 256-byte aligned)
constexpr size_t OFF_DESC = 0;
constexpr size_t OFF_CHUNKS = OFF_DESC + al256( sizeof( VecDev ) );
constexpr size_t OFF_RP = OFF_CHUNKS + al256( NA_CHUNKS * sizeof( Chunk ) );
constexpr size_t OFF_VEC = OFF_RP + al256( ( NA_ROWS + 1 ) * sizeof( int ) );
constexpr int NA_VECS = 7;                                   // x r z p q b d
constexpr size_t VEC_BYTES = al256( NA_ROWS * sizeof( double ) );
constexpr size_t OFF_PART = OFF_VEC + NA_VECS * VEC_BYTES;
constexpr size_t OFF_SC = OFF_PART + al256( NA_CHUNKS * 4 * sizeof( double ) );
constexpr size_t OFF_COUNTER = OFF_SC + al256( NB_SC * sizeof( double ) );
constexpr size_t NA_BYTES = OFF_COUNTER + 256;

} // namespace

// the work area: about 16 MB for 2^18 rows
static __device__ __align__( 256 ) unsigned char g_noalloc_work[ NA_BYTES ];

namespace {

constexpr int NA_MAX_DEVICES = 64;
std::mutex g_setup_mu;
char *g_work[ NA_MAX_DEVICES ] = {};

// the address of g_noalloc_work on the current device (looked up on the first call per device)
char *work_area( int device ) {
    if ( device < 0 || device >= NA_MAX_DEVICES ) throw Error( SDOT_ERR_ARGS, "sdot_linear_solve_noalloc: device index out of range" );
    std::lock_guard<std::mutex> lock( g_setup_mu );
    if ( ! g_work[ device ] ) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress( &p, g_noalloc_work );
        if ( e != cudaSuccess || ! p )
            throw Error( SDOT_ERR_CUDA, std::string( "sdot_linear_solve_noalloc: cudaGetSymbolAddress failed: " ) + cudaGetErrorString( e ) );
        g_work[ device ] = static_cast<char *>( p );
    }
    return g_work[ device ];
}

void na_status( sdot_status *st, int code, const std::string &msg, long long needed = 0 ) {
    if ( ! st ) return;
    std::memset( st, 0, sizeof( *st ) );
    st->code = code;
    st->kind = code == SDOT_ERR_CAPACITY ? 2 : 0;
    st->id = -1;
    st->needed = needed;
    std::strncpy( st->message, msg.c_str(), sizeof( st->message ) - 1 );
}

// memory that kernels on `device` may read in place: that device's own memory, or managed memory
bool on_device( const void *p, int device ) {
    cudaPointerAttributes a;
    if ( cudaPointerGetAttributes( &a, p ) != cudaSuccess ) { cudaGetLastError(); return false; }
    if ( a.type == cudaMemoryTypeManaged ) return true;
    return a.type == cudaMemoryTypeDevice && a.device == device;
}

// int64 row offsets -> the int32 ones of the CG kernels
__global__ void k_na_row_ptr( const int64_t *__restrict__ src, int *__restrict__ dst, long n1 ) {
    long i = long( blockIdx.x ) * blockDim.x + threadIdx.x;
    if ( i < n1 ) dst[ i ] = int( src[ i ] );
}

// b = rhs, and the rhs' mean in sc[ SC_MEAN ] (one block: fixed-order partial sums, then a fixed tree)
constexpr int NA_T = 1024;
__global__ void __launch_bounds__( NA_T ) k_na_rhs( const double *__restrict__ rhs, double *__restrict__ b, double *__restrict__ sc, int n ) {
    __shared__ double sh[ NA_T ];
    double s = 0;
    for ( int i = threadIdx.x; i < n; i += NA_T ) {
        double v = rhs[ i ];
        b[ i ] = v;
        s += v;
    }
    sh[ threadIdx.x ] = s;
    __syncthreads();
    for ( int w = NA_T / 2; w > 0; w >>= 1 ) {
        if ( threadIdx.x < w ) sh[ threadIdx.x ] += sh[ threadIdx.x + w ];
        __syncthreads();
    }
    if ( threadIdx.x == 0 ) sc[ SC_MEAN ] = sh[ 0 ] / n;
}

} // namespace

extern "C" int32_t sdot_linear_solve_noalloc( sdot_context ctx, int64_t n, const int64_t *row_ptr, const int32_t *cols, const double *vals,
                                              const double *dia, int32_t nrhs, const double *rhs, double *x, double tol, int32_t maxit,
                                              int32_t *iterations, sdot_status *st ) {
    if ( ! ctx || ! row_ptr || ! dia || ! rhs || ! x || n <= 0 || nrhs <= 0 ) {
        na_status( st, SDOT_ERR_ARGS, "sdot_linear_solve_noalloc: bad argument" );
        return SDOT_ERR_ARGS;
    }
    if ( n > NA_ROWS ) {
        na_status( st, SDOT_ERR_CAPACITY,
                   "sdot_linear_solve_noalloc: " + std::to_string( n ) + " rows, past the static work area's " + std::to_string( NA_ROWS ) +
                       " (use sdot_linear_solve)",
                   n );
        return SDOT_ERR_CAPACITY;
    }
    std::lock_guard<std::mutex> lock( ctx->mu );
    try {
        Ctx &c = ctx->c;
        CK( cudaSetDevice( c.device ) );
        for ( const void *p : { ( const void * ) row_ptr, ( const void * ) dia, ( const void * ) rhs, ( const void * ) x } )
            if ( ! on_device( p, c.device ) )
                throw Error( SDOT_ERR_ARGS, "sdot_linear_solve_noalloc: every array must be device memory of the context's device" );
        char *w = work_area( c.device );
        int64_t nnz = 0;
        CK( cudaMemcpyAsync( &nnz, row_ptr + n, sizeof( nnz ), cudaMemcpyDeviceToHost, c.stream ) );
        CK( cudaStreamSynchronize( c.stream ) );
        if ( nnz < 0 || nnz >= ( 1ll << 31 ) ) throw Error( SDOT_ERR_ARGS, "sdot_linear_solve_noalloc: nnz must fit int32" );
        if ( nnz > 0 && ( ! cols || ! vals || ! on_device( cols, c.device ) || ! on_device( vals, c.device ) ) )
            throw Error( SDOT_ERR_ARGS, "sdot_linear_solve_noalloc: cols / vals must be device memory of the context's device" );
        const int nch = int( ( n + VCHUNK - 1 ) / VCHUNK );
        int *rp = reinterpret_cast<int *>( w + OFF_RP );
        double *vec[ NA_VECS ];
        for ( int k = 0; k < NA_VECS; ++k ) vec[ k ] = reinterpret_cast<double *>( w + OFF_VEC + k * VEC_BYTES );
        double *part = reinterpret_cast<double *>( w + OFF_PART ), *sc = reinterpret_cast<double *>( w + OFF_SC );
        unsigned *counter = reinterpret_cast<unsigned *>( w + OFF_COUNTER );
        VecDev V;
        std::memset( &V, 0, sizeof( V ) );
        V.n = int( n ); V.row_ptr = rp; V.col = const_cast<int *>( cols ); V.val = const_cast<double *>( vals );
        V.dia = const_cast<double *>( dia );       // the CG kernels only read the matrix
        V.x = vec[ 0 ]; V.r = vec[ 1 ]; V.z = vec[ 2 ]; V.p = vec[ 3 ]; V.q = vec[ 4 ]; V.b = vec[ 5 ]; V.d = vec[ 6 ];
        V.tol = tol > 0 ? tol : 1e-10;
        V.maxit = maxit > 0 ? maxit : 100000;
        V.sc = sc; V.partials = part; V.counter = counter; V.nchunk = nch; V.active = 1;
        V.rank0 = 0;
        Chunk hch[ NA_CHUNKS ];
        for ( int k = 0; k < nch; ++k ) hch[ k ] = Chunk{ 0, k * VCHUNK, int( std::min<int64_t>( n, int64_t( k + 1 ) * VCHUNK ) ), k };
        VecDev *dv = reinterpret_cast<VecDev *>( w + OFF_DESC );
        Chunk *dch = reinterpret_cast<Chunk *>( w + OFF_CHUNKS );
        // what must start at zero: the fold counter (the kernels leave it at zero after each fold) and the scalars
        CK( cudaMemsetAsync( counter, 0, 8, c.stream ) );
        CK( cudaMemcpyAsync( dv, &V, sizeof( V ), cudaMemcpyHostToDevice, c.stream ) );
        CK( cudaMemcpyAsync( dch, hch, nch * sizeof( Chunk ), cudaMemcpyHostToDevice, c.stream ) );
        k_na_row_ptr<<<int( ( n + 1 + 255 ) / 256 ), 256, 0, c.stream>>>( row_ptr, rp, long( n + 1 ) );
        CK( cudaGetLastError() );
        ++c.launches;
        Launch L = c.L();
        for ( int k = 0; k < nrhs; ++k ) {
            CK( cudaMemsetAsync( sc, 0, NB_SC * sizeof( double ), c.stream ) );
            k_na_rhs<<<1, NA_T, 0, c.stream>>>( rhs + size_t( k ) * n, V.b, sc, int( n ) );
            CK( cudaGetLastError() );
            ++c.launches;
            launch_cg_init( L, dv, dch, nch );
            double hsc[ NB_SC ];
            for ( ;; ) {
                for ( int s = 0; s < 32; ++s ) launch_cg_iter( L, dv, dch, nch );
                CK( cudaMemcpyAsync( hsc, sc, sizeof( hsc ), cudaMemcpyDeviceToHost, c.stream ) );
                CK( cudaStreamSynchronize( c.stream ) );
                if ( hsc[ SC_CONV ] != 0 ) break;
            }
            if ( iterations ) iterations[ k ] = hsc[ SC_FAIL ] != 0 ? -1 : int( hsc[ SC_ITER ] );
            launch_gauge( L, dv, dch, nch );
            CK( cudaMemcpyAsync( x + size_t( k ) * n, V.d, n * 8, cudaMemcpyDeviceToDevice, c.stream ) );
            CK( cudaStreamSynchronize( c.stream ) );
        }
        na_status( st, SDOT_OK, "" );
        return SDOT_OK;
    } catch ( const Error &e ) {
        na_status( st, e.code, e.msg, e.needed );
        return e.code;
    } catch ( const std::exception &e ) {
        na_status( st, SDOT_ERR_ARGS, e.what() );
        return SDOT_ERR_ARGS;
    }
}

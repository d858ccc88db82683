// The host engine: device geometry of a problem, and the batched damped Newton.
//
// A solve is a state machine (start selection, stages of the width continuation, Newton iterations, trial
// steps, final moments).  `job_run` / `jobs_tick` advance many solves together: each TICK launches
//   A. one cell kernel over every solve that needs a diagram (trial weights, start weights, a new stage),
//   B. up to CG_BURST CG iterations over every solve that is solving its Newton system,
// then reads back every solve's scalars in ONE device->host copy and lets each solve take its decisions
// (accept or halve the step, switch the residual, converge), and finally launches
//   D. the Laplacian assembly + rhs + CG start of the solves that begin an iteration, and the trial
//      weights w + t d of the solves that go on trying.
// The semantics of the decisions are those of sdotplan/Newton.h:243-429 and sdotplan/Solve.h:111-371
// (TRIALS step, no aggregation); only the scheduling is batched.
#include "engine.h"
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>

namespace sdot {

void check_cuda( cudaError_t e, const char *what ) {
    if ( e == cudaSuccess ) return;
    if ( e == cudaErrorMemoryAllocation ) {
        cudaGetLastError();
        throw Error( SDOT_ERR_NO_MEMORY, std::string( what ) + ": out of device memory" );
    }
    throw Error( SDOT_ERR_CUDA, std::string( what ) + ": " + cudaGetErrorString( e ) );
}

// the bytes the context's pool hands out now
uint64_t pool_in_use( Ctx &c ) {
    uint64_t used = 0;
    CK( cudaMemPoolGetAttribute( c.pool, cudaMemPoolAttrUsedMemCurrent, &used ) );
    return uint64_t( used );
}

void *dalloc( Ctx &c, size_t bytes ) {
    void *p = nullptr;
    if ( bytes == 0 ) bytes = 256;
    if ( c.pool_limit ) {
        const uint64_t used = pool_in_use( c );
        if ( used + bytes > c.pool_limit )
            throw Error( SDOT_ERR_NO_MEMORY, "device pool refused " + std::to_string( bytes ) + " bytes: the context's limit is " +
                                                 std::to_string( c.pool_limit ) + " and " + std::to_string( used ) + " are in use",
                         -1, ( long long ) bytes );
    }
    cudaError_t e = cudaMallocFromPoolAsync( &p, bytes, c.pool, c.stream );
    if ( e == cudaErrorMemoryAllocation ) {
        cudaGetLastError();
        throw Error( SDOT_ERR_NO_MEMORY, "device pool refused " + std::to_string( bytes ) + " bytes", -1, ( long long ) bytes );
    }
    CK( e );
    return p;
}

void dfree( Ctx &c, void *p ) {
    if ( p ) CK( cudaFreeAsync( p, c.stream ) );
}

void ctx_init( Ctx &c, int device, uint64_t pool_limit ) {
    c.device = device;
    CK( cudaSetDevice( device ) );
    CK( cudaStreamCreateWithFlags( &c.stream, cudaStreamNonBlocking ) );
    cudaMemPoolProps props;
    std::memset( &props, 0, sizeof( props ) );
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    CK( cudaMemPoolCreate( &c.pool, &props ) );
    uint64_t thr = pool_limit ? pool_limit : UINT64_MAX;
    CK( cudaMemPoolSetAttribute( c.pool, cudaMemPoolAttrReleaseThreshold, &thr ) );
    c.pool_limit = pool_limit;
    c.max_slots = 4096;
    c.dscal = ( double * ) dalloc( c, size_t( c.max_slots ) * SLOT_DOUBLES * 8 );
    CK( cudaMemsetAsync( c.dscal, 0, size_t( c.max_slots ) * SLOT_DOUBLES * 8, c.stream ) );
    c.dcount = ( unsigned * ) dalloc( c, size_t( c.max_slots ) * 4 * sizeof( unsigned ) );
    CK( cudaMemsetAsync( c.dcount, 0, size_t( c.max_slots ) * 4 * sizeof( unsigned ), c.stream ) );
    c.derr = ( ErrRec * ) dalloc( c, sizeof( ErrRec ) );
    CK( cudaMemsetAsync( c.derr, 0, sizeof( ErrRec ), c.stream ) );
    c.dgather = ( unsigned long long * ) dalloc( c, GATHER_BYTES );
    CK( cudaMemsetAsync( c.dgather, 0, GATHER_BYTES, c.stream ) );
    CK( cudaMallocHost( &c.hscal, size_t( c.max_slots ) * SLOT_DOUBLES * 8 ) );
    CK( cudaMallocHost( &c.herr, sizeof( ErrRec ) ) );
    std::memset( c.herr, 0, sizeof( ErrRec ) );
    for ( int s = c.max_slots - 1; s >= 0; --s ) c.free_slots.push_back( s );
    // the big-cell queue: OvfList header then its items, in one allocation
    char *q = ( char * ) dalloc( c, 256 + size_t( c.ovf_cap ) * sizeof( OvfItem ) );
    c.dovf = ( OvfList * ) q;
    OvfList hl{ 0, c.ovf_cap, ( OvfItem * ) ( q + 256 ) };
    CK( cudaMemcpyAsync( c.dovf, &hl, sizeof( hl ), cudaMemcpyHostToDevice, c.stream ) );
    CK( cudaMallocHost( &c.hovf, sizeof( int ) ) );
    *c.hovf = 0;
    c.hstage_bytes = size_t( 16 ) << 20;
    CK( cudaMallocHost( &c.hstage, c.hstage_bytes ) );
    char *gq = ( char * ) dalloc( c, 256 + size_t( c.giant_cap ) * sizeof( OvfItem ) );
    c.dgiant = ( OvfList * ) gq;
    OvfList gl{ 0, c.giant_cap, ( OvfItem * ) ( gq + 256 ) };
    CK( cudaMemcpyAsync( c.dgiant, &gl, sizeof( gl ), cudaMemcpyHostToDevice, c.stream ) );
    CK( cudaMallocHost( &c.hgiant, sizeof( int ) ) );
    *c.hgiant = 0;
    c.big_scratch = ( char * ) dalloc( c, big_scratch_bytes( c.big_warps ) );
    const char *t = std::getenv( "SDOT_KERNEL_TIMING" );
    c.timer.on = t && t[ 0 ] == '1';
    CK( cudaStreamSynchronize( c.stream ) );
}

void ctx_release( Ctx &c ) {
    cudaSetDevice( c.device );
    c.timer.release();
    for ( auto &g : c.graphs ) cudaGraphExecDestroy( g.exec );
    c.graphs.clear();
    if ( c.stream ) {
        if ( c.desc ) cudaFreeAsync( c.desc, c.stream );
        if ( c.dscal ) cudaFreeAsync( c.dscal, c.stream );
        if ( c.dcount ) cudaFreeAsync( c.dcount, c.stream );
        if ( c.derr ) cudaFreeAsync( c.derr, c.stream );
        if ( c.dgather ) cudaFreeAsync( c.dgather, c.stream );
        if ( c.dovf ) cudaFreeAsync( c.dovf, c.stream );
        if ( c.big_scratch ) cudaFreeAsync( c.big_scratch, c.stream );
        if ( c.dgiant ) cudaFreeAsync( c.dgiant, c.stream );
        if ( c.giant_scratch ) cudaFreeAsync( c.giant_scratch, c.stream );
        if ( c.split.mem ) cudaFreeAsync( c.split.mem, c.stream );
        if ( c.split.used ) cudaFreeAsync( c.split.used, c.stream );
        if ( c.split.slot ) cudaFreeAsync( c.split.slot, c.stream );
        cudaStreamSynchronize( c.stream );
        cudaStreamDestroy( c.stream );
    }
    if ( c.hscal ) cudaFreeHost( c.hscal );
    if ( c.herr ) cudaFreeHost( c.herr );
    if ( c.hovf ) cudaFreeHost( c.hovf );
    if ( c.hgiant ) cudaFreeHost( c.hgiant );
    if ( c.hstage ) cudaFreeHost( c.hstage );
    if ( c.pool ) cudaMemPoolDestroy( c.pool );
    c = Ctx{};
}

// ---- kernel timing ------------------------------------------------------------------------------------------------------
static cudaEvent_t take_event( Timer &T ) {
    if ( T.npool ) return T.pool[ --T.npool ];
    cudaEvent_t e;
    CK( cudaEventCreate( &e ) );
    return e;
}
void Timer::begin( cudaStream_t s, int kind, double u ) {
    if ( ! on ) return;
    open_kind = kind;
    open_units = u;
    open_a = take_event( *this );
    CK( cudaEventRecord( open_a, s ) );
}
void Timer::end( cudaStream_t s, unsigned long long launches ) {
    if ( ! on || open_kind < 0 ) return;
    cudaEvent_t b = take_event( *this );
    CK( cudaEventRecord( b, s ) );
    if ( npending == cap ) {
        cap = cap ? 2 * cap : 256;
        Rec *p = new Rec[ cap ];
        for ( int k = 0; k < npending; ++k ) p[ k ] = pending[ k ];
        delete[] pending;
        pending = p;
    }
    pending[ npending++ ] = Rec{ open_kind, open_a, b, open_units };
    count[ open_kind ] += launches;
    open_kind = -1;
}
void Timer::resolve() {
    for ( int k = 0; k < npending; ++k ) {
        Rec &r = pending[ k ];
        CK( cudaEventSynchronize( r.b ) );
        float t = 0;
        CK( cudaEventElapsedTime( &t, r.a, r.b ) );
        ms[ r.kind ] += t;
        units[ r.kind ] += r.units;
        for ( cudaEvent_t e : { r.a, r.b } ) {
            if ( npool == cappool ) {
                cappool = cappool ? 2 * cappool : 512;
                cudaEvent_t *p = new cudaEvent_t[ cappool ];
                for ( int q = 0; q < npool; ++q ) p[ q ] = pool[ q ];
                delete[] pool;
                pool = p;
            }
            pool[ npool++ ] = e;
        }
    }
    npending = 0;
}
void Timer::release() {
    for ( int k = 0; k < npending; ++k ) { cudaEventDestroy( pending[ k ].a ); cudaEventDestroy( pending[ k ].b ); }
    for ( int k = 0; k < npool; ++k ) cudaEventDestroy( pool[ k ] );
    delete[] pending;
    delete[] pool;
    pending = nullptr;
    pool = nullptr;
    npending = npool = cap = cappool = 0;
}

int take_slot( Ctx &c ) {
    if ( c.free_slots.empty() ) throw Error( SDOT_ERR_NO_MEMORY, "too many solves in flight on one context" );
    int s = c.free_slots.back();
    c.free_slots.pop_back();
    return s;
}
void give_slot( Ctx &c, int s ) { c.free_slots.push_back( s ); }

static double now_s() {
    return std::chrono::duration<double>( std::chrono::steady_clock::now().time_since_epoch() ).count();
}

// copies `count` elements to the device buffer `dst`, from host or device memory
template<class T>
static void to_device( Ctx &c, T *dst, const T *src, size_t count, int memory ) {
    if ( count == 0 ) return;
    CK( cudaMemcpyAsync( dst, src, count * sizeof( T ), memory == SDOT_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c.stream ) );
}
template<class T>
static void to_host_vec( Ctx &c, std::vector<T> &dst, const T *src, size_t count, int memory ) {
    dst.resize( count );
    if ( count == 0 ) return;
    if ( memory == SDOT_DEVICE ) {
        CK( cudaMemcpyAsync( dst.data(), src, count * sizeof( T ), cudaMemcpyDeviceToHost, c.stream ) );
        CK( cudaStreamSynchronize( c.stream ) );
    } else
        std::memcpy( dst.data(), src, count * sizeof( T ) );
}

// uploads a descriptor block and returns its device address (stream ordered: the area is reused)
// a host block for an asynchronous upload: copied into the pinned ring (so that the copy does not wait for the stream),
// or the block itself when the ring is full (a pageable copy, which the runtime stages)
static const void *stage( Ctx &c, const void *src, size_t bytes ) {
    if ( ! c.hstage || c.hstage_used + bytes > c.hstage_bytes ) return src;
    char *p = c.hstage + c.hstage_used;
    std::memcpy( p, src, bytes );
    c.hstage_used += ( bytes + 255 ) & ~size_t( 255 );
    return p;
}

static char *upload_desc( Ctx &c, const void *src, size_t bytes ) {
    if ( bytes > c.desc_bytes ) {
        for ( auto &g : c.graphs ) cudaGraphExecDestroy( g.exec );
        c.graphs.clear();
        if ( c.desc ) dfree( c, c.desc );
        c.desc_bytes = std::max( bytes, size_t( 1 ) << 20 );
        c.desc = ( char * ) dalloc( c, c.desc_bytes );
    }
    CK( cudaMemcpyAsync( c.desc, stage( c, src, bytes ), bytes, cudaMemcpyHostToDevice, c.stream ) );
    return c.desc;
}

// a second block in the upload area, after `offset` bytes already uploaded by this step (stream ordered)
// (past the area's end: a block of its own, freed in stream order at the end of the tick)
static char *upload_desc_at( Ctx &c, const void *src, size_t bytes, size_t offset ) {
    offset = ( offset + 255 ) & ~size_t( 255 );
    char *dst = c.desc + offset;
    if ( offset + bytes > c.desc_bytes ) {
        dst = ( char * ) dalloc( c, bytes );
        c.desc_spill.push_back( dst );
    }
    CK( cudaMemcpyAsync( dst, stage( c, src, bytes ), bytes, cudaMemcpyHostToDevice, c.stream ) );
    return dst;
}

void check_errors( Ctx &c, const char *where ) {
    if ( c.herr->code == 0 ) return;
    ErrRec e = *c.herr;
    *c.herr = ErrRec{};
    CK( cudaMemsetAsync( c.derr, 0, sizeof( ErrRec ), c.stream ) );
    if ( e.code == SDOT_ERR_CAPACITY )
        throw Error( SDOT_ERR_CAPACITY, std::string( where ) + ": a cell exceeded its capacity (seed " + std::to_string( e.seed ) + ")", e.seed,
                     e.needed );
    if ( e.code == SDOT_ERR_TOPOLOGY )
        throw Error( SDOT_ERR_TOPOLOGY, std::string( where ) + ": a cell's clip lost its topology (seed " + std::to_string( e.seed ) + ")", e.seed );
    throw Error( e.code, std::string( where ) + ": device error", e.seed );
}

// a capacity error of the engine's kernels belongs to its problem (the per-slot flag read in `decide`): not a batch error
int run_giant_cells( Ctx &c, const ProbDev *dprob, unsigned flags ) {
    CK( cudaMemcpyAsync( c.hgiant, &c.dgiant->count, sizeof( int ), cudaMemcpyDeviceToHost, c.stream ) );
    CK( cudaStreamSynchronize( c.stream ) );
    const int count = std::min( *c.hgiant, c.giant_cap );
    if ( count <= 0 ) return 0;
    if ( ! c.giant_scratch ) c.giant_scratch = ( char * ) dalloc( c, giant3_slot_bytes() * c.giant_slots );
    Launch L = c.L();
    launch_cells3d_giant( L, dprob, c.dgiant, count, flags, c.derr, c.giant_scratch, c.giant_slots );
    CK( cudaMemsetAsync( &c.dgiant->count, 0, sizeof( int ), c.stream ) );
    return count;
}

// a capacity or topology error of a solve's cell is its problem's (the per-slot flag read in `decide`), not the batch's
// about 1.5 KB a stored cell (25 vertices, 15 planes); the records never take more than 2 GiB (past it, pass 2 does the
// cells that found no room whole)
const Split3 *split3_for( Ctx &c, int nchunks, long gcells ) {
    if ( gcells <= 0 || nchunks <= 0 ) return nullptr;
    const unsigned long long want = std::min<unsigned long long>( 2ull << 30, std::max<unsigned long long>( 64ull << 20, gcells * 2048ull ) );
    try {
        if ( ! c.split.used ) c.split.used = ( unsigned long long * ) dalloc( c, 256 );
        if ( c.split.cap < want ) {
            if ( c.split.mem ) dfree( c, c.split.mem );
            c.split.mem = nullptr;
            c.split.cap = 0;
            c.split.mem = ( char * ) dalloc( c, want );
            c.split.cap = want;
        }
        const size_t slots = size_t( nchunks ) * CHUNK;
        if ( c.split_slots < slots ) {
            if ( c.split.slot ) dfree( c, c.split.slot );
            c.split.slot = nullptr;
            c.split_slots = 0;
            c.split.slot = ( long long * ) dalloc( c, slots * sizeof( long long ) );
            c.split_slots = slots;
        }
    } catch ( const Error & ) {
        return nullptr;
    }
    return c.split.mem && c.split.slot ? &c.split : nullptr;
}

static void clear_capacity_error( Ctx &c ) {
    if ( c.herr->code != SDOT_ERR_CAPACITY && c.herr->code != SDOT_ERR_TOPOLOGY ) return;
    if ( std::getenv( "SDOT_TRACE" ) )
        std::fprintf( stderr, "sdot: capacity: problem %d of the launch, seed %d, needed %d\n", c.herr->prob, c.herr->seed, c.herr->needed );
    *c.herr = ErrRec{};
    CK( cudaMemsetAsync( c.derr, 0, sizeof( ErrRec ), c.stream ) );
}

// ---- geometry ----------------------------------------------------------------------------------------------------------
void Geometry::fill( ProbDev &P ) const {
    std::memset( &P, 0, sizeof( P ) );
    P.dim = dim;
    P.n = n;
    P.dkind = dkind;
    for ( int a = 0; a < 3; ++a ) {
        P.lo[ a ] = lo[ a ]; P.hi[ a ] = hi[ a ]; P.g[ a ] = g[ a ]; P.go[ a ] = go[ a ]; P.gh[ a ] = gh[ a ];
        P.dn[ a ] = dn[ a ]; P.dorg[ a ] = dorg[ a ]; P.dstep[ a ] = dstep[ a ];
    }
    P.ghmin = ghmin;
    P.cell_range = cell_range;
    P.pos = pos;
    P.user = user;
    P.rank_of = rank_of;
    P.rho = rho;
    P.dval = dval;
    P.dpre = dpre;
    P.cap = dim == 2 ? CAP2 : CAP3;
    P.wpyr = wpyr;
    P.wmom = wmom;
    P.nlev = nlev;
    for ( int l = 0; l < MAX_LEV; ++l ) P.poff[ l ] = poff[ l ];
}

void build_geometry( Ctx &c, Geometry &G, int dim, long n, const double *positions, const double box_lo[ 3 ], const double box_hi[ 3 ],
                     const sdot_density &dens, int memory ) {
    if ( dim != 2 && dim != 3 ) throw Error( SDOT_ERR_ARGS, "dim must be 2 or 3" );
    if ( n <= 0 || n >= ( 1l << 31 ) - 1 ) throw Error( SDOT_ERR_ARGS, "n must be in [1, 2^31)" );
    if ( ! positions ) throw Error( SDOT_ERR_ARGS, "positions is NULL" );
    if ( dens.kind == SDOT_DENSITY_IMAGE && dim != 2 ) throw Error( SDOT_ERR_UNSUPPORTED, "image densities are integrated in 2D only" );
    if ( dens.kind < 0 || dens.kind > 2 ) throw Error( SDOT_ERR_ARGS, "unknown density kind" );
    G.dim = dim;
    G.n = int( n );
    for ( int a = 0; a < dim; ++a ) {
        G.lo[ a ] = box_lo[ a ];
        G.hi[ a ] = box_hi[ a ];
        if ( ! ( G.hi[ a ] > G.lo[ a ] ) ) throw Error( SDOT_ERR_ARGS, "the domain box is empty" );
    }
    to_host_vec( c, G.pos_host, positions, size_t( n ) * dim, memory );
    // the grid covers the domain and every seed, about two seeds per grid cell
    double mn[ 3 ], mx[ 3 ];
    for ( int a = 0; a < dim; ++a ) { mn[ a ] = G.lo[ a ]; mx[ a ] = G.hi[ a ]; }
    for ( long i = 0; i < n; ++i )
        for ( int a = 0; a < dim; ++a ) {
            double x = G.pos_host[ i * dim + a ];
            if ( ! std::isfinite( x ) ) throw Error( SDOT_ERR_ARGS, "a position is not finite", i );
            mn[ a ] = std::min( mn[ a ], x );
            mx[ a ] = std::max( mx[ a ], x );
        }
    double vol = 1;
    for ( int a = 0; a < dim; ++a ) vol *= mx[ a ] - mn[ a ];
    double h = std::pow( vol / std::max( 1.0, n / 2.0 ), 1.0 / dim );
    const int gmax = dim == 2 ? 32768 : 2048;
    G.ncell = 1;
    G.ghmin = 1e300;
    int bits = 1;
    for ( int a = 0; a < 3; ++a ) {
        if ( a >= dim ) { G.g[ a ] = 1; G.go[ a ] = 0; G.gh[ a ] = 1; continue; }
        double ext = mx[ a ] - mn[ a ];
        int ga = int( std::ceil( ext / h ) );
        ga = std::max( 1, std::min( ga, gmax ) );
        G.g[ a ] = ga;
        G.go[ a ] = mn[ a ];
        G.gh[ a ] = ext / ga;
        G.ghmin = std::min( G.ghmin, G.gh[ a ] );
        G.ncell *= ga;
        while ( ( 1 << bits ) < ga ) ++bits;
    }
    int key_bits = dim * bits;
    // one allocation: ranked positions, user, rank_of, cell ranges, density
    size_t dbytes = 0;
    G.dkind = dens.kind;
    G.rho = dens.value;
    long nval = 0, npre = 0;
    if ( dens.kind == SDOT_DENSITY_IMAGE ) {
        if ( ! dens.values || dens.shape[ 0 ] <= 0 || dens.shape[ 1 ] <= 0 ) throw Error( SDOT_ERR_ARGS, "image without values" );
        nval = long( dens.shape[ 0 ] ) * dens.shape[ 1 ];
        npre = long( dens.shape[ 1 ] ) * ( dens.shape[ 0 ] + 1 );
        for ( int a = 0; a < 2; ++a ) { G.dn[ a ] = dens.shape[ a ]; G.dorg[ a ] = dens.origin[ a ]; G.dstep[ a ] = dens.step[ a ]; }
    } else if ( dens.kind == SDOT_DENSITY_GAUSSIANS ) {
        if ( dens.count <= 0 || ! dens.centres || ! dens.sigmas || ! dens.masses ) throw Error( SDOT_ERR_ARGS, "gaussians without parameters" );
        G.dn[ 0 ] = dens.count;
        nval = long( dens.count ) * ( dim + 2 );
        std::vector<double> cc, ss, mm;
        to_host_vec( c, cc, dens.centres, size_t( dens.count ) * dim, memory );
        to_host_vec( c, ss, dens.sigmas, dens.count, memory );
        to_host_vec( c, mm, dens.masses, dens.count, memory );
        G.gauss.resize( nval );
        for ( int k = 0; k < dens.count; ++k ) {
            for ( int a = 0; a < dim; ++a ) G.gauss[ k * ( dim + 2 ) + a ] = cc[ k * dim + a ];
            if ( ! ( ss[ k ] > 0 ) ) throw Error( SDOT_ERR_ARGS, "a gaussian has a non-positive sigma", k );
            G.gauss[ k * ( dim + 2 ) + dim ] = ss[ k ];
            G.gauss[ k * ( dim + 2 ) + dim + 1 ] = mm[ k ];
        }
    }
    // an image also keeps its values as given and room for the continuation's blur (one pass's output, the taps)
    const long nimg = dens.kind == SDOT_DENSITY_IMAGE ? 2 * nval + 2 * long( std::max( G.dn[ 0 ], G.dn[ 1 ] ) ) + 1 : 0;
    dbytes = size_t( nval + npre + nimg ) * 8 + 4 * 256;
    const long npyr = wpyr_layout( dim, G.g, G.nlev, G.poff );
    size_t bytes = size_t( n ) * dim * 8 + size_t( n ) * 8 + size_t( G.ncell ) * 8 + size_t( npyr ) * 8 * ( dim + 1 + wmom_size( dim ) ) + dbytes +
                   10 * 256;
    G.mem = ( char * ) dalloc( c, bytes );
    Arena A{ G.mem, bytes, 0 };
    G.pos = A.take<double>( size_t( n ) * dim );
    G.user = A.take<int>( n );
    G.rank_of = A.take<int>( n );
    G.cell_range = A.take<int2>( G.ncell );
    G.wpyr = A.take<double>( size_t( npyr ) * ( dim + 1 ) );
    G.wmom = A.take<double>( size_t( npyr ) * wmom_size( dim ) );
    if ( nval ) G.dval = A.take<double>( nval );
    if ( npre ) G.dpre = A.take<double>( npre );
    if ( nimg ) {
        G.dorig = A.take<double>( nval );
        G.dtmp = A.take<double>( nval );
        G.dker = A.take<double>( 2 * size_t( std::max( G.dn[ 0 ], G.dn[ 1 ] ) ) + 1 );
    }
    // the sort, in a temporary allocation
    size_t tb = radix_temp_bytes( int( n ), key_bits );
    size_t tbytes = size_t( n ) * ( 8 + 8 + 4 + 4 ) + size_t( n ) * dim * 8 + tb + 6 * 256;
    char *tmp = ( char * ) dalloc( c, tbytes );
    Arena T{ tmp, tbytes, 0 };
    double *pos_user = T.take<double>( size_t( n ) * dim );
    unsigned long long *k0 = T.take<unsigned long long>( n ), *k1 = T.take<unsigned long long>( n );
    int *v0 = T.take<int>( n ), *v1 = T.take<int>( n );
    void *sort_tmp = T.take<char>( tb );
    CK( cudaMemcpyAsync( pos_user, G.pos_host.data(), size_t( n ) * dim * 8, cudaMemcpyHostToDevice, c.stream ) );
    Launch L = c.L();
    launch_keys( L, pos_user, int( n ), dim, G.g, G.go, G.gh, key_bits, k0, v0 );
    radix_sort( L, sort_tmp, tb, k0, k1, v0, v1, int( n ), key_bits );
    launch_gather( L, pos_user, v1, int( n ), dim, G.pos, G.user, G.rank_of, nullptr, nullptr );
    CK( cudaMemsetAsync( G.cell_range, 0, size_t( G.ncell ) * sizeof( int2 ), c.stream ) );
    launch_cell_ranges( L, k1, G.pos, int( n ), dim, G.g, G.go, G.gh, G.cell_range );
    if ( dens.kind == SDOT_DENSITY_IMAGE ) {
        to_device( c, G.dval, dens.values, nval, memory );
        CK( cudaMemcpyAsync( G.dorig, G.dval, size_t( nval ) * 8, cudaMemcpyDeviceToDevice, c.stream ) );
        launch_image_prefix( L, G.dval, G.dn[ 0 ], G.dn[ 1 ], G.dstep[ 0 ], G.dpre );
    } else if ( dens.kind == SDOT_DENSITY_GAUSSIANS ) {
        CK( cudaMemcpyAsync( G.dval, G.gauss.data(), nval * 8, cudaMemcpyHostToDevice, c.stream ) );
    }
    dfree( c, tmp );
}

void free_geometry( Ctx &c, Geometry &G ) {
    dfree( c, G.mem );
    G.mem = nullptr;
}

// ---- the solve ---------------------------------------------------------------------------------------------------------
enum JState { J_START0, J_START_VOR, J_START_SIM, J_STAGE_DIAG, J_REPORT, J_ITER, J_CG, J_TRIAL, J_POLISH, J_FINAL, J_DONE };
enum Pend : unsigned { P_NEWTON = 1, P_GAUGE = 2, P_TRIAL = 4, P_RESCALE = 8, P_SET_W2 = 16, P_ZERO_W2 = 32, P_DENSITY = 64 };
enum NStatus { NS_RUNNING = 0, NS_CONVERGED = 1, NS_MAX_ITER = 2, NS_STAGNATION = 3, NS_LINEAR_FAILURE = 4, NS_CAPACITY = 5, NS_FAILURE = 6,
               NS_CONVERGED_AGG = 7 };
constexpr int AGG_CAP = 4096;        // near-coincident pairs one Laplacian can report
enum StatIdx {
    ST_STATUS = 0, ST_RESIDUAL, ST_RESIDUAL0, ST_NB_ITER, ST_NB_DIAG, ST_NB_BACKTRACKS, ST_T_MAJORANT, ST_T_DIAG, ST_T_ASM, ST_T_LIN, ST_T_LIM, ST_EPS,
    ST_DOMAIN_MASS, ST_NB_OVERFLOWED, ST_NB_CELL_LIM, ST_NB_LIMIT_ROUNDS, ST_LIN_NB_HIERARCHIES, ST_LIN_NB_ITER, ST_LIN_WORST, ST_START, ST_T_TOTAL,
    ST_NB_CONTINUATION_STEPS, ST_MIN_START_MASS, ST_IT_SWITCH, ST_IT_DOUBLE, ST_SCRATCH_BYTES, ST_NB_CLUSTERS, ST_NB_AGGREGATED, ST_NB_DUPLICATES,
    ST_RESIDUAL_FULL, ST_NB_POLISH
};

struct SolveJob {
    Geometry G;
    int slot = -1;
    double opt[ SDOT_NB_OPTIONS ];
    std::vector<double> nu_user;
    double nu_min = 0, nu_sum = 0;
    bool given = false;
    int start = 1;
    char *mem = nullptr;
    size_t mem_bytes = 0;
    double *w, *w2, *a, *a2, *d, *nu, *nu_dev_user, *b, *x, *r, *z, *p, *q, *dia, *val, *tmpw;
    int *nb[ 2 ], *nid[ 2 ];
    double *nc[ 2 ];
    int *ovf_count[ 2 ], *ovf_ids[ 2 ];
    double *ovf_c[ 2 ];
    int ovf_cap = 0;
    int cur = 0;
    // the multigrid hierarchy (sizes fixed by n; values rebuilt every Newton iteration)
    int mg_L = 0, mg_pack = 4;
    int mg_n[ MG_MAX_LEVELS ], mg_cap[ MG_MAX_LEVELS ], mg_nch[ MG_MAX_LEVELS ];
    int *mg_rp[ MG_MAX_LEVELS ], *mg_col[ MG_MAX_LEVELS ], *mg_rc[ MG_MAX_LEVELS ];
    float *mg_val[ MG_MAX_LEVELS ], *mg_dia[ MG_MAX_LEVELS ], *mg_dinv[ MG_MAX_LEVELS ], *mg_b[ MG_MAX_LEVELS ], *mg_x[ MG_MAX_LEVELS ],
        *mg_y[ MG_MAX_LEVELS ];
    double *mg_part[ MG_MAX_LEVELS ];
    float *mg_inv = nullptr;
    char *mg_mem = nullptr;
    int *row_ptr, *col, *rowcnt;
    double *part_cells, *part_vec;
    unsigned long long *wslot;          // [2]
    int wcur = 0;                       // wslot[ wcur ] belongs to w
    double *obary = nullptr, *ocost = nullptr;
    int cap = CAP2, nch_cells = 0, nch_vec = 0;
    int rank0 = 0;                      // rank of user seed 0: the gauge w_0 = 0
    int repA = 0;                       // which report holds the accepted diagram's
    // Newton state
    JState state = J_START0;
    unsigned pend = 0;
    int res_cur = 1;
    double t_last = 1, t = 1, eps = 0, nr = 0, worst = 0, worst_rel = 0;
    int it = 0, trial = 0, nb_evals = 0;
    bool redo = false;
    double h_tprev = 0, h_sprev = 0;
    bool h_has = false;
    // the limits step (2D, sdotplan/Newton.h:330-366): the first trial at `beta`, kept from one iteration to the next;
    // while a probe diagram has cells below the floor, the step is brought under their limits (8 rounds at most)
    bool lim_on = false, lim_probe = false;
    double beta = 0.25, t_done = 0;
    int lim_round = 0;
    std::vector<double> scales;
    int stage = 0;
    double stats[ SDOT_NB_STATS ];
    std::vector<double> hist;
    long steps_before = 0;
    int nstatus = NS_RUNNING;
    double domain_mass = 0, nu_scale = 1;
    double t_begin = 0;
    std::vector<double> wsim;           // similarity weights (user order)
    double amin_best = 0;
    bool first_stage = true;
    int err_code = 0;
    std::string err_msg;
    long long err_id = -1;
    // the aggregation of near-coincident seeds (sdotplan/Aggregation.h): a union-find over the ranks, the clusters
    // (CSR over ranks, members increasing), their device copy [ begins | members ] and the shares the tests read
    double agg_margin = 0;
    int2 *agg_pairs = nullptr;
    std::vector<int> agg_parent, cl_begin, cl_members;
    int *d_cl = nullptr;
    double *ae = nullptr;
    double *cl_true = nullptr;          // the true couplings inside each cluster ([ members ][ AGG_KMAX + 1 ]), then scratch
    double c_scale = 1;                 // the scale of a facet's coupling: rho (or the box's mean density) x (3D) the spacing
    int ncl = 0;
    bool full_set = false;              // stats[ residual_full ] computed on the full problem
    int polish_round = 0;               // the re-splitting after an aggregated convergence: rounds done,
    double polish_before = 0;           // ... and the members' residual before the current one
    // lin_precision 1: the FP32 copies of the inner CG (matrix values [n * cap], diagonal and five vectors [n])
    char *mx_mem = nullptr;
    bool mx_off = false;                // set once a refinement stalled: this solve's later systems take the FP64 CG
    float *val32 = nullptr, *dia32 = nullptr, *x32 = nullptr, *r32 = nullptr, *z32 = nullptr, *p32 = nullptr, *q32 = nullptr;
};

static void alloc_mixed( Ctx &c, SolveJob &J ) {
    const size_t n = size_t( J.G.n );
    const size_t bytes = n * J.cap * 4 + 6 * ( n * 4 + 256 ) + 256;
    J.mx_mem = ( char * ) dalloc( c, bytes );
    Arena A{ J.mx_mem, bytes, 0 };
    J.val32 = A.take<float>( n * J.cap );
    J.dia32 = A.take<float>( n ); J.x32 = A.take<float>( n ); J.r32 = A.take<float>( n );
    J.z32 = A.take<float>( n ); J.p32 = A.take<float>( n ); J.q32 = A.take<float>( n );
}

static size_t mg_bytes( int dim, long n, int cap );

size_t job_bytes( int dim, long n, int dkind, long dcount ) {
    const int cap = dim == 2 ? CAP2 : CAP3;
    const long cs = cell_chunk( dim, n ), nch = ( n + cs - 1 ) / cs, nv = ( n + vec_chunk( n ) - 1 ) / vec_chunk( n );
    size_t b = size_t( n ) * 8 * 18 + 2 * ( size_t( n ) * 4 + size_t( n ) * cap * 12 ) + size_t( n + 1 ) * 4 + size_t( n ) * cap * 12 +
               size_t( n ) * 4 + size_t( nch ) * NB_REPORT * 8 + size_t( nv ) * 4 * 8 + 64 + size_t( n ) * 8 * ( dim + 1 ) + 40 * 256;
    // geometry: ranked positions, user, rank_of, the grid (about n / 2 cells), the density, and the sort's scratch
    b += size_t( n ) * dim * 8 + size_t( n ) * 8 + size_t( n ) * 4 + 1024;
    b += size_t( n ) * ( dim == 2 ? 64 : 84 ) + 1024;    // the weight majorants and their moments (4/3, 8/7 of the grid's cells)
    b += dkind == D_IMAGE ? size_t( dcount ) * 32 + 32768 : size_t( dcount ) * 8 * ( dim + 2 );     // (image: values, prefix, original, blur pass)
    b += size_t( n ) * ( 24 + dim * 8 ) + 4096;
    return b + mg_bytes( dim, n, cap );
}

static void alloc_job( Ctx &c, SolveJob &J ) {
    const long n = J.G.n;
    const int dim = J.G.dim, cap = J.cap;
    J.nch_cells = int( ( n + cell_chunk( dim, n ) - 1 ) / cell_chunk( dim, n ) );
    J.nch_vec = int( ( n + vec_chunk( n ) - 1 ) / vec_chunk( n ) );
    J.ovf_cap = int( n ) + 4096;
    size_t bytes = size_t( n ) * 8 * 18 + 2 * ( size_t( n ) * 4 + size_t( n ) * cap * 12 ) + size_t( n + 1 ) * 4 + size_t( n ) * cap * 12 +
                   size_t( n ) * 4 + size_t( J.nch_cells ) * NB_REPORT * 8 + size_t( J.nch_vec ) * 4 * 8 + 64 + size_t( n ) * 8 * ( dim + 1 ) +
                   2 * ( size_t( J.ovf_cap ) * 12 + 16 ) + ( J.agg_margin > 0 ? AGG_CAP * sizeof( int2 ) : 0 ) + 49 * 256;
    J.mem_bytes = bytes;
    J.mem = ( char * ) dalloc( c, bytes );
    Arena A{ J.mem, bytes, 0 };
    J.w = A.take<double>( n ); J.w2 = A.take<double>( n ); J.a = A.take<double>( n ); J.a2 = A.take<double>( n );
    J.d = A.take<double>( n ); J.nu = A.take<double>( n ); J.nu_dev_user = A.take<double>( n ); J.b = A.take<double>( n );
    J.x = A.take<double>( n ); J.r = A.take<double>( n ); J.z = A.take<double>( n ); J.p = A.take<double>( n );
    J.q = A.take<double>( n ); J.dia = A.take<double>( n ); J.tmpw = A.take<double>( n );
    for ( int k = 0; k < 2; ++k ) {
        J.nb[ k ] = A.take<int>( n ); J.nid[ k ] = A.take<int>( size_t( n ) * cap ); J.nc[ k ] = A.take<double>( size_t( n ) * cap );
        J.ovf_count[ k ] = A.take<int>( 4 ); J.ovf_ids[ k ] = A.take<int>( J.ovf_cap ); J.ovf_c[ k ] = A.take<double>( J.ovf_cap );
    }
    if ( J.agg_margin > 0 ) J.agg_pairs = A.take<int2>( AGG_CAP );
    J.row_ptr = A.take<int>( n + 1 );
    J.col = A.take<int>( size_t( n ) * cap );
    J.val = A.take<double>( size_t( n ) * cap );
    J.rowcnt = A.take<int>( n );
    J.part_cells = A.take<double>( size_t( J.nch_cells ) * NB_REPORT );
    J.part_vec = A.take<double>( size_t( J.nch_vec ) * 4 );
    J.wslot = A.take<unsigned long long>( 2 );
    J.obary = A.take<double>( size_t( n ) * dim );
    J.ocost = A.take<double>( n );
}

constexpr int MG_CCH = 16;           // coarse rows per chunk of the coarsening kernels (4 a warp: a small level still spreads)
constexpr int MG_RCH = 64;           // rows per chunk of the cycle's per-level kernels (one pass of a block)

// the level sizes of the hierarchy of a problem of n seeds; 0 levels when it is too small to need one
static int mg_levels( int dim, long n, int *sizes ) {
    const int pack = dim == 2 ? 4 : 8;
    if ( n <= MG_BOTTOM ) return 0;
    int L = 0;
    long m = n;
    sizes[ L++ ] = int( m );
    while ( m > MG_BOTTOM && L < MG_MAX_LEVELS ) {
        m = ( m + pack - 1 ) / pack;
        sizes[ L++ ] = int( m );
    }
    return sizes[ L - 1 ] <= MG_BOTTOM ? L : 0;
}

static size_t mg_bytes( int dim, long n, int cap ) {
    int sz[ MG_MAX_LEVELS ];
    int L = mg_levels( dim, n, sz );
    if ( ! L ) return 0;
    size_t b = size_t( n ) * cap * 4 + size_t( n ) * 4 * 4;
    const int capc = dim == 2 ? 16 : 64;   // coarse entries a row can take on average (about 8 in 2D, 22 in 3D)
    for ( int l = 1; l < L; ++l ) b += size_t( sz[ l ] + 1 ) * 4 * 2 + size_t( sz[ l ] ) * capc * 8 + size_t( sz[ l ] ) * 5 * 4 +
                                        size_t( sz[ l ] / MG_CCH + 1 ) * 16 + 12 * 256;
    return b + MG_BOTTOM * MG_BOTTOM * 4 + 16 * 256;
}

static void alloc_mg( Ctx &c, SolveJob &J ) {
    const int dim = J.G.dim;
    J.mg_L = mg_levels( dim, J.G.n, J.mg_n );
    if ( ! J.mg_L ) return;
    J.mg_pack = dim == 2 ? 4 : 8;
    const size_t bytes = mg_bytes( dim, J.G.n, J.cap );
    J.mg_mem = ( char * ) dalloc( c, bytes );
    Arena A{ J.mg_mem, bytes, 0 };
    const int capc = dim == 2 ? 16 : 64;   // coarse entries a row can take on average (about 8 in 2D, 22 in 3D)
    for ( int l = 0; l < J.mg_L; ++l ) {
        const int n = J.mg_n[ l ];
        if ( l == 0 ) {
            J.mg_rp[ 0 ] = J.row_ptr;
            J.mg_col[ 0 ] = J.col;
            J.mg_rc[ 0 ] = nullptr;
            J.mg_cap[ 0 ] = n * J.cap;
            J.mg_val[ 0 ] = A.take<float>( size_t( n ) * J.cap );
            J.mg_part[ 0 ] = nullptr;
            J.mg_nch[ 0 ] = 0;
            J.mg_y[ 0 ] = nullptr;
        } else {
            J.mg_rp[ l ] = A.take<int>( n + 1 );
            J.mg_rc[ l ] = A.take<int>( n + 1 );
            J.mg_cap[ l ] = n * capc;
            J.mg_col[ l ] = A.take<int>( size_t( n ) * capc );
            J.mg_val[ l ] = A.take<float>( size_t( n ) * capc );
            J.mg_nch[ l ] = ( n + MG_CCH - 1 ) / MG_CCH;
            J.mg_part[ l ] = A.take<double>( size_t( J.mg_nch[ l ] ) * 2 );
            J.mg_y[ l ] = A.take<float>( n );
        }
        J.mg_dia[ l ] = A.take<float>( n );
        J.mg_dinv[ l ] = A.take<float>( n );
        J.mg_b[ l ] = A.take<float>( n );
        J.mg_x[ l ] = A.take<float>( n );
    }
    J.mg_inv = A.take<float>( MG_BOTTOM * MG_BOTTOM );
}

// the level-l descriptor of a job for a CG batch in which its VecDev sits at `vec`
static MgLevel mg_level( const SolveJob &J, int l, int vec ) {
    MgLevel M;
    std::memset( &M, 0, sizeof( M ) );
    M.level = l;
    M.vec = vec;
    M.n = J.mg_n[ l ];
    M.pack = J.mg_pack;
    M.rp = J.mg_rp[ l ]; M.col = J.mg_col[ l ]; M.val = J.mg_val[ l ]; M.dia = J.mg_dia[ l ]; M.dinv = J.mg_dinv[ l ];
    M.b = J.mg_b[ l ]; M.x = J.mg_x[ l ]; M.y = J.mg_y[ l ];
    if ( l + 1 < J.mg_L ) {
        M.nn = J.mg_n[ l + 1 ];
        M.bn = J.mg_b[ l + 1 ];
        M.xn = J.mg_y[ l + 1 ];
        M.rcn = J.mg_rc[ l + 1 ]; M.rpn = J.mg_rp[ l + 1 ]; M.coln = J.mg_col[ l + 1 ]; M.valn = J.mg_val[ l + 1 ];
        M.dian = J.mg_dia[ l + 1 ]; M.dinvn = J.mg_dinv[ l + 1 ];
        M.part = J.mg_part[ l + 1 ];
        M.nchunk = J.mg_nch[ l + 1 ];
        M.capn = J.mg_cap[ l + 1 ];
    }
    if ( l == J.mg_L - 1 ) M.inv = J.mg_inv;
    return M;
}

static std::vector<double> continuation_scales( const SolveJob &J );
static void set_stage_density( Ctx &c, SolveJob &J );
// the densities the width continuation can widen: gaussians, and 2D images (blurred on their grid)
static bool convolvable( const SolveJob &J ) { return J.G.dkind == D_GAUSS || ( J.G.dkind == D_IMAGE && J.G.dim == 2 ); }

SolveJob *job_create( Ctx &c, const sdot_solve_desc &desc ) {
    const sdot_diagram_desc &D = desc.diagram;
    if ( desc.options[ SDOT_OPT_PRECISION ] != 0 && desc.options[ SDOT_OPT_PRECISION ] != 1 )
        throw Error( SDOT_ERR_ARGS, "option precision: 0 (FP64 clipping) or 1 (FP32 clipping with FP64 re-checks)" );
    if ( desc.options[ SDOT_OPT_PRECISION ] == 1 && desc.diagram.dim != 2 )
        throw Error( SDOT_ERR_UNSUPPORTED, "option precision 1 (FP32 clipping with FP64 re-checks) is built in 2D; 3D clips in FP64 (0)" );
    if ( desc.options[ SDOT_OPT_LIN_PRECISION ] != 0 && desc.options[ SDOT_OPT_LIN_PRECISION ] != 1 )
        throw Error( SDOT_ERR_ARGS, "option lin_precision: 0 (FP64 CG) or 1 (FP32 CG with FP64 iterative refinement)" );
    if ( c.pool_limit ) {
        // THE MEMORY MODEL before anything is built (CardMemory.check_card_memory, src/sdot/CardMemory.py:158-190): a solve
        // that cannot fit in what the pool has left is refused at once, with what it needs
        const uint64_t need = sdot_solve_bytes( D.dim, D.n, &D.density ), used = pool_in_use( c );
        if ( used + need > c.pool_limit )
            throw Error( SDOT_ERR_NO_MEMORY, "the solve of " + std::to_string( D.n ) + " seeds needs about " + std::to_string( need ) +
                                                 " bytes of the device (" + std::to_string( need / std::max<long>( D.n, 1 ) ) +
                                                 " per seed, sdot_solve_bytes) and the context's pool has " +
                                                 std::to_string( c.pool_limit > used ? c.pool_limit - used : 0 ) +
                                                 " left: solve fewer seeds, or give the context a larger pool_limit",
                         -1, ( long long ) need );
    }
    SolveJob *J = new SolveJob;
    try {
        J->t_begin = now_s();
        build_geometry( c, J->G, D.dim, D.n, D.positions, D.box_lo, D.box_hi, D.density, D.memory );
        J->cap = D.dim == 2 ? CAP2 : CAP3;
        std::memcpy( J->opt, desc.options, sizeof( J->opt ) );
        J->agg_margin = J->opt[ SDOT_OPT_AGG_MARGIN ];
        {
            // the scale of a facet's coupling (gpu/Newton2D.cuh:1273): the density (uniform: rho; else the box's mean, 1 /
            // volume) times, in 3D, the seeds' spacing
            double vol = 1;
            for ( int a = 0; a < D.dim; ++a ) vol *= D.box_hi[ a ] - D.box_lo[ a ];
            J->c_scale = ( D.density.kind == SDOT_DENSITY_UNIFORM ? D.density.value : 1.0 / std::max( vol, 1e-300 ) ) *
                         ( D.dim == 3 ? std::cbrt( vol / double( std::max<long>( D.n, 1 ) ) ) : 1.0 );
        }
        J->lim_on = D.dim == 2 && int( J->opt[ SDOT_OPT_STEP ] ) == 1;     // (3D: the trials, as the reference)
        for ( int k = 0; k < SDOT_NB_STATS; ++k ) J->stats[ k ] = 0;
        const long n = D.n;
        if ( desc.nu ) to_host_vec( c, J->nu_user, desc.nu, n, D.memory );
        else J->nu_user.assign( n, 1.0 / n );
        J->nu_min = 1e300;
        J->nu_sum = 0;
        for ( long i = 0; i < n; ++i ) {
            if ( ! ( J->nu_user[ i ] > 0 ) ) throw Error( SDOT_ERR_ARGS, "a target mass is not positive", i );
            J->nu_min = std::min( J->nu_min, J->nu_user[ i ] );
            J->nu_sum += J->nu_user[ i ];
        }
        std::vector<double> w0;
        if ( D.weights ) to_host_vec( c, w0, D.weights, n, D.memory );
        else w0.assign( n, 0.0 );
        J->given = false;
        for ( double v : w0 ) J->given |= v != 0;
        J->start = J->given ? 0 : 1;
        double g0 = w0[ 0 ];
        for ( double &v : w0 ) v -= g0;
        alloc_job( c, *J );
        if ( int( J->opt[ SDOT_OPT_LIN_METHOD ] ) == 1 ) alloc_mg( c, *J );
        if ( int( J->opt[ SDOT_OPT_LIN_PRECISION ] ) == 1 ) alloc_mixed( c, *J );
        J->slot = take_slot( c );
        CK( cudaMemsetAsync( c.dscal + size_t( J->slot ) * SLOT_DOUBLES + SLOT_ERR, 0, 2 * sizeof( double ), c.stream ) );
        CK( cudaMemcpyAsync( &J->rank0, J->G.rank_of, sizeof( int ), cudaMemcpyDeviceToHost, c.stream ) );
        CK( cudaStreamSynchronize( c.stream ) );
        Launch L = c.L();
        // targets and start weights, ranked
        CK( cudaMemcpyAsync( J->nu_dev_user, J->nu_user.data(), n * 8, cudaMemcpyHostToDevice, c.stream ) );
        launch_gather_vec( L, J->nu_dev_user, J->G.user, int( n ), J->nu, 1.0 );
        CK( cudaMemcpyAsync( J->tmpw, w0.data(), n * 8, cudaMemcpyHostToDevice, c.stream ) );
        launch_gather_vec( L, J->tmpw, J->G.user, int( n ), J->w, 1.0 );
        CK( cudaMemsetAsync( J->wslot, 0, 16, c.stream ) );
        launch_wmax( L, J->w, int( n ), J->wslot );
        CK( cudaMemsetAsync( c.dcount + 4 * J->slot, 0, 16, c.stream ) );
        J->res_cur = int( J->opt[ SDOT_OPT_RESIDUAL ] );
        J->stats[ ST_SCRATCH_BYTES ] = double( J->mem_bytes );
        J->stats[ ST_IT_DOUBLE ] = -1;
        J->stats[ ST_IT_SWITCH ] = -1;
        J->state = J_START0;
        J->scales.assign( 1, 0.0 );
        if ( convolvable( *J ) && int( J->opt[ SDOT_OPT_CONTINUATION ] ) == 2 ) {
            // continuation "always": the start is chosen on the first width already (sdotplan/Solve.h:196-199)
            J->scales = continuation_scales( *J );
            J->stage = 0;
            set_stage_density( c, *J );
        }
    } catch ( ... ) {
        job_destroy( c, J );
        throw;
    }
    return J;
}

void job_destroy( Ctx &c, SolveJob *J ) {
    if ( ! J ) return;
    if ( J->mg_mem ) dfree( c, J->mg_mem );
    if ( J->mx_mem ) dfree( c, J->mx_mem );
    if ( J->d_cl ) dfree( c, J->d_cl );
    if ( J->cl_true ) dfree( c, J->cl_true );
    if ( J->ae ) dfree( c, J->ae );
    if ( J->mem ) dfree( c, J->mem );
    if ( J->G.mem ) free_geometry( c, J->G );
    if ( J->slot >= 0 ) give_slot( c, J->slot );
    delete J;
}

bool job_done( const SolveJob *j ) { return j->state == J_DONE; }

static double *rep_dev( Ctx &c, const SolveJob &J, int which ) { return c.dscal + size_t( J.slot ) * SLOT_DOUBLES + which * NB_REPORT; }
static const double *rep_host( Ctx &c, const SolveJob &J, int which ) { return c.hscal + size_t( J.slot ) * SLOT_DOUBLES + which * NB_REPORT; }
static double *sc_dev( Ctx &c, const SolveJob &J ) { return c.dscal + size_t( J.slot ) * SLOT_DOUBLES + 2 * NB_REPORT; }
static const double *sc_host( Ctx &c, const SolveJob &J ) { return c.hscal + size_t( J.slot ) * SLOT_DOUBLES + 2 * NB_REPORT; }

static double merit_of( const double *rep, int res ) { return res == 0 ? std::sqrt( rep[ R_LIN2 ] ) : std::sqrt( rep[ R_GM2 ] ); }

// the diagram a job needs now: weights / outputs / report slot
struct DiagReq {
    SolveJob *job;
    const double *w;
    const unsigned long long *wslot;
    double *mass;
    int table;          // -1: none
    int report;         // -1: none
    bool moments;
    bool report_only;
};

static bool needs_diagram( SolveJob &J, DiagReq &R ) {
    R = DiagReq{ &J, nullptr, nullptr, nullptr, -1, -1, false, false };
    switch ( J.state ) {
    case J_START0:
    case J_STAGE_DIAG:
        R.w = J.w; R.wslot = J.wslot + J.wcur; R.mass = J.a; R.table = J.cur; R.report = J.repA; return true;
    case J_START_VOR:
    case J_START_SIM:
    case J_TRIAL:
    case J_POLISH:
        R.w = J.w2; R.wslot = J.wslot + ( 1 - J.wcur ); R.mass = J.a2; R.table = 1 - J.cur; R.report = 1 - J.repA; return true;
    case J_REPORT:
        R.mass = J.a; R.report = J.repA; R.report_only = true; return true;
    case J_FINAL:
        R.w = J.w; R.wslot = J.wslot + J.wcur; R.moments = true; return true;
    default:
        return false;
    }
}

static void hist_push( SolveJob &J, int it, double t, int nb_evals, const double *rep ) {
    double row[ SDOT_NB_HIST ] = { double( J.steps_before + it ), t, std::sqrt( rep[ R_LIN2 ] ), rep[ R_AMIN ], rep[ R_WORST ],
                                   J.stats[ ST_NB_DIAG ], double( nb_evals ), J.scales[ J.stage ] };
    J.hist.insert( J.hist.end(), row, row + SDOT_NB_HIST );
}

// the stages of the width continuation (sdotplan/Continuation.h:33-40): s0, s0 / r, ... >= s_min, then 0
static std::vector<double> continuation_scales( const SolveJob &J ) {
    const int dim = J.G.dim;
    double s0 = J.opt[ SDOT_OPT_CONV_S0 ];
    if ( s0 <= 0 ) {
        double d2 = 0;
        for ( int a = 0; a < dim; ++a ) d2 += ( J.G.hi[ a ] - J.G.lo[ a ] ) * ( J.G.hi[ a ] - J.G.lo[ a ] );
        s0 = 0.5 * std::sqrt( d2 );
    }
    double smin = J.opt[ SDOT_OPT_CONV_MIN ];
    if ( smin <= 0 && J.G.dkind == D_IMAGE ) smin = std::min( J.G.dstep[ 0 ], J.G.dstep[ 1 ] ) / 4;   // a quarter of a pixel
    if ( smin <= 0 ) {
        double sg = 1e300;
        for ( int k = 0; k < J.G.dn[ 0 ]; ++k ) sg = std::min( sg, J.G.gauss[ k * ( dim + 2 ) + dim ] );
        smin = sg / 4;
    }
    double ratio = J.opt[ SDOT_OPT_CONV_RATIO ] > 1 ? J.opt[ SDOT_OPT_CONV_RATIO ] : std::sqrt( 2.0 );
    std::vector<double> res;
    for ( double s = s0; s >= smin * ( 1 - 1e-12 ) && s > 0 && res.size() < 200; s /= ratio ) res.push_back( s );
    res.push_back( 0 );
    return res;
}

static void set_stage_density( Ctx &c, SolveJob &J ) {
    if ( J.G.dkind == D_IMAGE ) {
        // the image at width s: blurred on its grid by a gaussian of s / step pixels along each axis, truncated at 4 of them
        // and renormalised at the border (sdotplan/convolved/Image.h:37-74), then its prefix sums
        Geometry &G = J.G;
        const int nx = G.dn[ 0 ], ny = G.dn[ 1 ];
        const size_t nval = size_t( nx ) * ny;
        const double s = J.scales[ J.stage ];
        Launch L = c.L();
        CK( cudaMemcpyAsync( G.dval, G.dorig, nval * 8, cudaMemcpyDeviceToDevice, c.stream ) );
        if ( s > 0 ) {
            std::vector<double> ker;
            for ( int a = 0; a < 2; ++a ) {
                const double sp = s / G.dstep[ a ];
                if ( ! ( sp > 1e-3 ) ) continue;
                const int len = G.dn[ a ];
                const int r = int( std::min( std::ceil( 4 * sp ), double( len ) ) );
                ker.resize( 2 * size_t( r ) + 1 );
                for ( int k = -r; k <= r; ++k ) ker[ k + r ] = std::exp( -0.5 * double( k ) * double( k ) / ( sp * sp ) );
                CK( cudaMemcpyAsync( G.dker, ker.data(), ker.size() * 8, cudaMemcpyHostToDevice, c.stream ) );
                launch_blur_axis( L, G.dval, G.dtmp, nx, ny, a, r, G.dker );
                std::swap( G.dval, G.dtmp );
                CK( cudaStreamSynchronize( c.stream ) );       // `ker` is refilled for the next axis
            }
        }
        launch_image_prefix( L, G.dval, nx, ny, G.dstep[ 0 ], G.dpre );
        return;
    }
    if ( J.G.dkind != D_GAUSS ) return;
    const int dim = J.G.dim, st = dim + 2;
    std::vector<double> g = J.G.gauss;
    double s = J.scales[ J.stage ];
    for ( int k = 0; k < J.G.dn[ 0 ]; ++k ) g[ k * st + dim ] = std::sqrt( g[ k * st + dim ] * g[ k * st + dim ] + s * s );
    CK( cudaMemcpyAsync( J.G.dval, g.data(), g.size() * 8, cudaMemcpyHostToDevice, c.stream ) );
    CK( cudaStreamSynchronize( c.stream ) );       // `g` leaves scope
}

static double order_dbl_host( unsigned long long u ) {
    u = ( u >> 63 ) ? ( u & 0x7fffffffffffffffull ) : ~u;
    double x;
    std::memcpy( &x, &u, 8 );
    return x;
}

static void end_stage( Ctx &c, SolveJob &J );
static void full_residual( Ctx &c, SolveJob &J, double &worst, double &worst_rel );
static void final_status( Ctx &c, SolveJob &J );
static bool polish_start( Ctx &c, SolveJob &J );

static void begin_iterations( Ctx &c, SolveJob &J ) {
    // the domain mass of this density and the targets rescaled to it (sdotplan/Solve.h:250-257)
    const double *rep = rep_host( c, J, J.repA );
    J.domain_mass = rep[ R_ASUM ];
    double f = ( J.domain_mass > 0 && J.nu_sum > 0 && J.domain_mass != J.nu_sum ) ? J.domain_mass / J.nu_sum : 1.0;
    J.it = 0;
    J.t_last = 1;
    J.res_cur = int( J.opt[ SDOT_OPT_RESIDUAL ] );
    if ( f != J.nu_scale ) {
        J.nu_scale = f;
        J.pend |= P_RESCALE;
        J.state = J_REPORT;
    } else
        J.state = J_ITER;
}

// one Newton iteration's decision, from the accepted diagram's report (sdotplan/Newton.h:293-343)
static void newton_iter( Ctx &c, SolveJob &J ) {
    const double *rep = rep_host( c, J, J.repA );
    if ( J.it == 0 && ! J.redo ) hist_push( J, 0, 0, 1, rep );
    J.redo = false;
    J.worst = rep[ R_WORST ];
    J.worst_rel = rep[ R_WORST_REL ];
    if ( J.opt[ SDOT_OPT_SWITCH ] > 0 && J.res_cur != 0 && J.worst_rel <= J.opt[ SDOT_OPT_SWITCH ] ) {
        J.res_cur = 0;
        if ( J.first_stage ) J.stats[ ST_IT_SWITCH ] = J.it;
    }
    if ( J.it == 0 ) {
        J.eps = 0.5 * std::min( J.nu_min * J.nu_scale, rep[ R_AMIN ] );
        if ( J.first_stage ) { J.stats[ ST_EPS ] = J.eps; J.stats[ ST_RESIDUAL0 ] = J.worst; }
    }
    J.nr = merit_of( rep, J.res_cur );
    J.stats[ ST_RESIDUAL ] = J.worst;
    if ( J.worst <= J.opt[ SDOT_OPT_TOL_ABS ] || ( J.opt[ SDOT_OPT_TOL_REL ] > 0 && J.worst_rel <= J.opt[ SDOT_OPT_TOL_REL ] ) ) {
        J.nstatus = NS_CONVERGED;
        end_stage( c, J );
        return;
    }
    if ( J.it >= int( J.opt[ SDOT_OPT_MAXIT ] ) ) {
        J.nstatus = NS_MAX_ITER;
        end_stage( c, J );
        return;
    }
    J.stats[ ST_NB_ITER ] += 1;
    J.pend |= P_NEWTON;
    J.state = J_CG;
}

static void end_stage( Ctx &c, SolveJob &J ) {
    J.first_stage = false;
    J.steps_before = J.hist.empty() ? 0 : long( J.hist[ J.hist.size() - SDOT_NB_HIST ] ) + 1;
    if ( J.nstatus != NS_LINEAR_FAILURE && J.stage + 1 < int( J.scales.size() ) ) {
        ++J.stage;
        J.nstatus = NS_RUNNING;
        set_stage_density( c, J );
        J.state = J_STAGE_DIAG;
        return;
    }
    if ( ( J.G.dkind == D_GAUSS || J.G.dkind == D_IMAGE ) && J.scales[ J.stage ] != 0 ) {
        J.stage = int( J.scales.size() ) - 1;
        set_stage_density( c, J );
    }
    if ( J.nstatus == NS_CONVERGED && J.ncl > 0 && polish_start( c, J ) ) return;
    final_status( c, J );
}

// the status of a finished solve: the tests read the clusters' masses, so the full problem's residual is reported, and
// "converged (aggregated)" when only the aggregated problem passes (sdotplan/Solve.h:300-306)
static void final_status( Ctx &c, SolveJob &J ) {
    if ( J.nstatus == NS_CONVERGED && J.ncl > 0 ) {
        double wf, wfr;
        full_residual( c, J, wf, wfr );
        J.stats[ ST_RESIDUAL_FULL ] = wf;
        J.full_set = true;
        if ( ! ( wf <= J.opt[ SDOT_OPT_TOL_ABS ] || ( J.opt[ SDOT_OPT_TOL_REL ] > 0 && wfr <= J.opt[ SDOT_OPT_TOL_REL ] ) ) ) J.nstatus = NS_CONVERGED_AGG;
    }
    J.stats[ ST_STATUS ] = J.nstatus;
    J.state = J_FINAL;
}

// THE RE-SPLITTING (sdotplan/Newton.h:434-471, Aggregation.h:250-276): once the aggregated problem has converged, each
// cluster's members alone take a Newton step on their k x k block of the Laplacian (the rest of the diagram fixed,
// the gauge kept by a shift of everyone), one diagram for all the clusters; kept while the members' residual
// decreases and the aggregated problem stays converged, 4 rounds at most. False when there is nothing to do.
static bool polish_start( Ctx &c, SolveJob &J ) {
    if ( J.polish_round >= 4 ) return false;
    const long n = J.G.n;
    std::vector<double> a( n ), nu( n );
    CK( cudaMemcpyAsync( a.data(), J.a, n * 8, cudaMemcpyDeviceToHost, c.stream ) );
    CK( cudaMemcpyAsync( nu.data(), J.nu, n * 8, cudaMemcpyDeviceToHost, c.stream ) );
    CK( cudaStreamSynchronize( c.stream ) );
    double wf = 0, wfr = 0, before = 0;
    for ( long i = 0; i < n; ++i ) { const double e = std::fabs( a[ i ] - nu[ i ] ); wf = std::max( wf, e ); wfr = std::max( wfr, e / nu[ i ] ); }
    if ( wf <= J.opt[ SDOT_OPT_TOL_ABS ] || ( J.opt[ SDOT_OPT_TOL_REL ] > 0 && wfr <= J.opt[ SDOT_OPT_TOL_REL ] ) ) return false;
    for ( int m : J.cl_members ) before = std::max( before, std::fabs( a[ m ] - nu[ m ] ) );
    const int cap = J.cap;
    std::vector<int> idx;
    std::vector<double> val;
    std::vector<int> rid( cap );
    std::vector<double> rc( cap );
    for ( int k = 0; k < J.ncl; ++k ) {
        const int b = J.cl_begin[ k ], e = J.cl_begin[ k + 1 ], m = e - b;
        if ( m < 2 || m > 64 ) continue;
        const int *mem = J.cl_members.data() + b;                  // increasing ranks
        std::vector<double> M( size_t( m ) * m, 0.0 ), r( m );
        bool ok = true;
        for ( int u = 0; u < m && ok; ++u ) {
            const int i = mem[ u ];
            int nbi = 0;
            CK( cudaMemcpy( &nbi, J.nb[ J.cur ] + i, sizeof( int ), cudaMemcpyDeviceToHost ) );
            if ( nbi > cap ) { ok = false; break; }                 // (a row in the overflow store: this cluster stays)
            if ( nbi > 0 ) {
                CK( cudaMemcpy( rid.data(), J.nid[ J.cur ] + size_t( i ) * cap, nbi * sizeof( int ), cudaMemcpyDeviceToHost ) );
                CK( cudaMemcpy( rc.data(), J.nc[ J.cur ] + size_t( i ) * cap, nbi * sizeof( double ), cudaMemcpyDeviceToHost ) );
            }
            double dia = 0;
            for ( int q = 0; q < nbi; ++q ) {
                dia += rc[ q ];
                const int *at = std::lower_bound( mem, mem + m, rid[ q ] );
                if ( at != mem + m && *at == rid[ q ] ) M[ size_t( u ) * m + ( at - mem ) ] -= rc[ q ];
            }
            M[ size_t( u ) * m + u ] += dia;
            r[ u ] = nu[ i ] - a[ i ];
        }
        if ( ! ok ) continue;
        // Cholesky (M symmetric positive definite unless the cluster has no neighbour)
        for ( int p = 0; p < m && ok; ++p ) {
            double d = M[ size_t( p ) * m + p ];
            for ( int q = 0; q < p; ++q ) d -= M[ size_t( p ) * m + q ] * M[ size_t( p ) * m + q ];
            if ( ! ( d > 0 ) ) { ok = false; break; }
            d = std::sqrt( d );
            M[ size_t( p ) * m + p ] = d;
            for ( int u = p + 1; u < m; ++u ) {
                double t = M[ size_t( u ) * m + p ];
                for ( int q = 0; q < p; ++q ) t -= M[ size_t( u ) * m + q ] * M[ size_t( p ) * m + q ];
                M[ size_t( u ) * m + p ] = t / d;
            }
        }
        if ( ! ok ) continue;
        for ( int u = 0; u < m; ++u ) {
            double t = r[ u ];
            for ( int q = 0; q < u; ++q ) t -= M[ size_t( u ) * m + q ] * r[ q ];
            r[ u ] = t / M[ size_t( u ) * m + u ];
        }
        for ( int u = m - 1; u >= 0; --u ) {
            double t = r[ u ];
            for ( int q = u + 1; q < m; ++q ) t -= M[ size_t( q ) * m + u ] * r[ q ];
            r[ u ] = t / M[ size_t( u ) * m + u ];
        }
        for ( int u = 0; u < m; ++u ) { idx.push_back( mem[ u ] ); val.push_back( r[ u ] ); }
    }
    if ( idx.empty() ) return false;
    double d0 = 0;
    for ( size_t t = 0; t < idx.size(); ++t ) if ( idx[ t ] == J.rank0 ) d0 = val[ t ];
    const size_t k = idx.size();
    char *d = ( char * ) dalloc( c, k * 12 + 256 );
    c.desc_spill.push_back( d );
    double *dv = reinterpret_cast<double *>( d );
    int *di = reinterpret_cast<int *>( d + ( ( k * 8 + 255 ) & ~size_t( 255 ) ) );
    CK( cudaMemcpyAsync( dv, val.data(), k * 8, cudaMemcpyHostToDevice, c.stream ) );
    CK( cudaMemcpyAsync( di, idx.data(), k * 4, cudaMemcpyHostToDevice, c.stream ) );
    Launch L = c.L();
    launch_polish_weights( L, J.w, J.w2, int( n ), d0, di, dv, int( k ) );
    unsigned long long *slot = J.wslot + ( 1 - J.wcur );
    CK( cudaMemsetAsync( slot, 0, 8, c.stream ) );
    launch_wmax( L, J.w2, int( n ), slot );
    CK( cudaStreamSynchronize( c.stream ) );       // `val`, `idx` leave scope
    J.polish_before = before;
    J.state = J_POLISH;
    return true;
}

static void after_start( Ctx &c, SolveJob &J ) {
    // seeds outside the domain leave cells empty: the similarity start (sdotplan/Solve.h:66-97, 212-226)
    const double amin = rep_host( c, J, J.repA )[ R_AMIN ];
    const bool keep = J.opt[ SDOT_OPT_KEEP_START ] != 0;
    if ( J.state != J_START_SIM && amin <= 0 && ! ( J.given && keep ) ) {
        const int dim = J.G.dim;
        const long n = J.G.n;
        double plo[ 3 ], phi[ 3 ], al = 1, bb[ 3 ];
        for ( int a = 0; a < dim; ++a ) { plo[ a ] = 1e300; phi[ a ] = -1e300; }
        for ( long i = 0; i < n; ++i )
            for ( int a = 0; a < dim; ++a ) { plo[ a ] = std::min( plo[ a ], J.G.pos_host[ i * dim + a ] ); phi[ a ] = std::max( phi[ a ], J.G.pos_host[ i * dim + a ] ); }
        for ( int a = 0; a < dim; ++a ) al = std::min( al, ( J.G.hi[ a ] - J.G.lo[ a ] ) * 0.8 / std::max( phi[ a ] - plo[ a ], 1e-300 ) );
        for ( int a = 0; a < dim; ++a ) bb[ a ] = ( J.G.lo[ a ] + J.G.hi[ a ] ) / 2 - al * ( plo[ a ] + phi[ a ] ) / 2;
        J.wsim.assign( n, 0.0 );
        for ( long i = 0; i < n; ++i ) {
            double pp = 0, qq = 0;
            for ( int a = 0; a < dim; ++a ) { double x = J.G.pos_host[ i * dim + a ], y = al * x + bb[ a ]; pp += x * x; qq += y * y; }
            J.wsim[ i ] = pp - qq / al;
        }
        double g0 = J.wsim[ 0 ];
        for ( double &v : J.wsim ) v -= g0;
        J.amin_best = amin;
        J.pend |= P_SET_W2;
        J.state = J_START_SIM;
        return;
    }
    // the continuation, decided on the start (sdotplan/Solve.h:229-235)
    J.stats[ ST_MIN_START_MASS ] = amin;
    J.stats[ ST_START ] = J.start;
    int cont = int( J.opt[ SDOT_OPT_CONTINUATION ] );
    if ( convolvable( J ) && J.scales.size() == 1 && cont == 1 && amin < J.opt[ SDOT_OPT_CONV_THRESHOLD ] * J.nu_min ) {
        J.scales = continuation_scales( J );
        J.stage = 0;
        set_stage_density( c, J );
        J.state = J_STAGE_DIAG;
    } else
        begin_iterations( c, J );
    J.stats[ ST_NB_CONTINUATION_STEPS ] = double( J.scales.size() );
}

static void accept_trial( SolveJob &J ) {
    std::swap( J.w, J.w2 );
    std::swap( J.a, J.a2 );
    J.cur ^= 1;
    J.wcur ^= 1;
    J.repA ^= 1;
}

// after the tick's read-back: the decisions of every job
// ---- the aggregation of near-coincident seeds (sdotplan/Aggregation.h) ------------------------------------------------
static int uf_find( std::vector<int> &p, int i ) {
    while ( p[ i ] != i ) { p[ i ] = p[ p[ i ] ]; i = p[ i ]; }
    return i;
}

// the pairs the last Laplacian showed: merged (latched, a cluster only grows), the clusters rebuilt and uploaded
// (sdotplan/Aggregation.h:109-141, 229-250)
static bool agg_update( Ctx &c, SolveJob &J ) {
    double *cnt = c.hscal + size_t( J.slot ) * SLOT_DOUBLES + SLOT_AGG;
    const int k = std::min( int( *cnt ), AGG_CAP );
    if ( k <= 0 ) return false;
    std::vector<int2> pairs( k );
    CK( cudaMemcpy( pairs.data(), J.agg_pairs, size_t( k ) * sizeof( int2 ), cudaMemcpyDeviceToHost ) );
    CK( cudaMemsetAsync( c.dscal + size_t( J.slot ) * SLOT_DOUBLES + SLOT_AGG, 0, sizeof( double ), c.stream ) );
    *cnt = 0;
    const int n = int( J.G.n );
    if ( J.agg_parent.empty() ) {
        J.agg_parent.resize( n );
        for ( int i = 0; i < n; ++i ) J.agg_parent[ i ] = i;
    }
    bool changed = false;
    for ( const int2 &p : pairs ) {
        int a = uf_find( J.agg_parent, p.x ), b = uf_find( J.agg_parent, p.y );
        if ( a == b ) continue;
        J.agg_parent[ std::max( a, b ) ] = std::min( a, b );
        changed = true;
    }
    if ( ! changed ) return false;
    std::vector<int> size( n, 0 ), id( n, -1 );
    for ( int i = 0; i < n; ++i ) ++size[ uf_find( J.agg_parent, i ) ];
    J.cl_begin.assign( 1, 0 );
    for ( int i = 0; i < n; ++i )
        if ( J.agg_parent[ i ] == i && size[ i ] > 1 ) { id[ i ] = int( J.cl_begin.size() ) - 1; J.cl_begin.push_back( J.cl_begin.back() + size[ i ] ); }
    J.ncl = int( J.cl_begin.size() ) - 1;
    J.cl_members.assign( J.cl_begin.back(), 0 );
    std::vector<int> at( J.cl_begin.begin(), J.cl_begin.end() - 1 );
    for ( int i = 0; i < n; ++i ) {
        const int cidx = id[ uf_find( J.agg_parent, i ) ];
        if ( cidx >= 0 ) J.cl_members[ at[ cidx ]++ ] = i;
    }
    std::vector<int> dev( J.cl_begin );
    dev.insert( dev.end(), J.cl_members.begin(), J.cl_members.end() );
    if ( J.d_cl ) dfree( c, J.d_cl );
    J.d_cl = ( int * ) dalloc( c, dev.size() * sizeof( int ) );
    CK( cudaMemcpyAsync( J.d_cl, dev.data(), dev.size() * sizeof( int ), cudaMemcpyHostToDevice, c.stream ) );
    if ( ! J.ae ) J.ae = ( double * ) dalloc( c, size_t( n ) * 8 );
    if ( J.cl_true ) dfree( c, J.cl_true );
    J.cl_true = ( double * ) dalloc( c, J.cl_members.size() * ( AGG_KMAX + 2 ) * sizeof( double ) );
    CK( cudaStreamSynchronize( c.stream ) );       // `dev` leaves scope
    J.stats[ ST_NB_CLUSTERS ] = J.ncl;
    J.stats[ ST_NB_AGGREGATED ] = double( J.cl_members.size() );
    return true;
}

// the residual of the full problem (every cell its own target), at the accepted masses: max |a - nu| and its relative
// form (sdotplan/Aggregation.h:199-209)
static void full_residual( Ctx &c, SolveJob &J, double &worst, double &worst_rel ) {
    const long n = J.G.n;
    std::vector<double> a( n ), nu( n );
    CK( cudaMemcpyAsync( a.data(), J.a, n * 8, cudaMemcpyDeviceToHost, c.stream ) );
    CK( cudaMemcpyAsync( nu.data(), J.nu, n * 8, cudaMemcpyDeviceToHost, c.stream ) );
    CK( cudaStreamSynchronize( c.stream ) );
    worst = worst_rel = 0;
    for ( long i = 0; i < n; ++i ) {
        const double e = std::fabs( a[ i ] - nu[ i ] );
        worst = std::max( worst, e );
        worst_rel = std::max( worst_rel, e / nu[ i ] );
    }
}

static void decide( Ctx &c, SolveJob &J, bool had_diag, bool had_cg ) {
    if ( J.agg_margin > 0 && agg_update( c, J ) && J.state == J_CG ) {
        // new clusters on the Laplacian the CG is solving: the system again, with their couplings capped and the direction
        // tied and corrected after the solve (the reference card merges before its solve, gpu/Newton2D.cuh:1557-1612)
        J.pend |= P_NEWTON;
        had_cg = false;
    }
    if ( had_diag && c.hscal[ size_t( J.slot ) * SLOT_DOUBLES + SLOT_ERR ] != 0 ) {
        // a cell past every capacity: this solve stops with the reference's "card capacity" status (the others go on);
        // its outputs are the moments at the last accepted weights
        CK( cudaMemsetAsync( c.dscal + size_t( J.slot ) * SLOT_DOUBLES + SLOT_ERR, 0, sizeof( double ), c.stream ) );
        J.nstatus = NS_CAPACITY;
        J.stats[ ST_STATUS ] = NS_CAPACITY;
        J.pend = 0;
        if ( J.state == J_FINAL ) {
            J.stats[ ST_T_TOTAL ] = now_s() - J.t_begin;
            J.state = J_DONE;
        } else
            J.state = J_FINAL;
        return;
    }
    if ( had_diag ) {
        const double *B = nullptr;
        switch ( J.state ) {
        case J_START0:
            J.stats[ ST_NB_DIAG ] += 1;
            {
                const double amin = rep_host( c, J, J.repA )[ R_AMIN ];
                // a warm start that empties a cell: the Voronoi start if it does better (sdotplan/Solve.h:203-210)
                if ( J.given && J.opt[ SDOT_OPT_KEEP_START ] == 0 && amin < 1e-3 * J.nu_min ) {
                    J.amin_best = amin;
                    J.pend |= P_ZERO_W2;
                    J.state = J_START_VOR;
                } else
                    after_start( c, J );
            }
            break;
        case J_START_VOR:
        case J_START_SIM: {
            J.stats[ ST_NB_DIAG ] += 1;
            B = rep_host( c, J, 1 - J.repA );
            bool vor = J.state == J_START_VOR;
            if ( B[ R_AMIN ] > J.amin_best ) {
                accept_trial( J );
                J.start = vor ? 1 : 2;
            }
            if ( vor ) { J.state = J_START0; after_start( c, J ); }
            else { J.state = J_START_SIM; after_start( c, J ); }
            break;
        }
        case J_STAGE_DIAG:
            J.stats[ ST_NB_DIAG ] += 1;
            begin_iterations( c, J );
            break;
        case J_REPORT:
            J.state = J_ITER;
            break;
        case J_TRIAL: {
            J.stats[ ST_NB_DIAG ] += 1;
            ++J.nb_evals;
            ++J.trial;
            B = rep_host( c, J, 1 - J.repA );
            // a cell past the big-cell pass in the trial: the step is refused (the damping halves it)
            const bool giant = c.hscal[ size_t( J.slot ) * SLOT_DOUBLES + SLOT_REFUSE ] != 0;
            if ( giant && J.lim_probe ) { J.lim_probe = false; J.trial = 1; }
            if ( J.lim_probe ) {
                // THE LIMITS (sdotplan/Newton.h:336-366): cells below the floor at this probe bring the step under their
                // limits; none: this diagram is the damping's first trial
                const double *S = c.hscal + size_t( J.slot ) * SLOT_DOUBLES + SLOT_LIM;
                const double nbad = S[ 0 ];
                bool end_probe = true;
                if ( nbad > 0 ) {
                    J.stats[ ST_NB_LIMIT_ROUNDS ] += 1;
                    J.stats[ ST_NB_CELL_LIM ] += nbad;
                    unsigned long long bits;
                    std::memcpy( &bits, S + 1, 8 );
                    const double al = std::min( J.t, order_dbl_host( bits ) );
                    J.t_done = J.t;
                    J.t = 0.9 * al;
                    ++J.lim_round;
                    if ( J.t < J.opt[ SDOT_OPT_T_MIN ] ) J.t = J.t_done / 2;     // no reason to stagnate: the trials, from half
                    else end_probe = J.lim_round >= 8;
                }
                if ( end_probe ) {
                    J.lim_probe = false;
                    if ( J.t >= J.beta ) J.beta = std::min( 1.0, 2 * J.beta );  // a direct pass: the next probe goes further
                    J.trial = 0;
                }
                if ( nbad > 0 ) {
                    J.pend |= P_TRIAL;
                    J.state = J_TRIAL;
                    break;
                }
                J.trial = 1;
            }
            double m2 = B[ R_AMIN ], n2r = merit_of( B, J.res_cur );
            bool ok = ! giant && m2 >= J.eps && std::isfinite( n2r );
            if ( ok && n2r <= ( 1 - J.t / 2 ) * J.nr && n2r < J.nr ) {
                accept_trial( J );
                J.t_last = J.t;
                ++J.it;
                hist_push( J, J.it, J.t, J.nb_evals, rep_host( c, J, J.repA ) );
                J.state = J_ITER;
            } else {
                // the hopeless damping (sdotplan/Report.h:33-57)
                bool hopeless = false;
                if ( ! ok || ! ( J.nr > 0 ) ) J.h_has = false;
                else {
                    double s = ( J.nr - n2r ) / J.t, sp = J.h_sprev, asp = std::fabs( sp );
                    hopeless = J.h_has && J.h_tprev == 2 * J.t && s < J.nr / 4 && sp < J.nr / 4 && s - sp <= 0.25 * asp && sp - s <= 0.25 * asp &&
                               2 * s - sp < J.nr / 4;
                    J.h_tprev = J.t; J.h_sprev = s; J.h_has = true;
                }
                J.t /= 2;
                J.stats[ ST_NB_BACKTRACKS ] += 1;
                if ( J.t < J.opt[ SDOT_OPT_T_MIN ] || hopeless || J.trial >= int( J.opt[ SDOT_OPT_MAX_BACKTRACKS ] ) ) {
                    if ( J.res_cur != 0 ) {
                        // a refused step of the log residual: the iteration again, in LIN (sdotplan/Newton.h:375-389)
                        J.res_cur = 0;
                        if ( J.first_stage ) J.stats[ ST_IT_SWITCH ] = J.it;
                        J.stats[ ST_NB_ITER ] -= 1;
                        J.redo = true;
                        J.state = J_ITER;
                    } else {
                        J.nstatus = NS_STAGNATION;
                        end_stage( c, J );
                    }
                } else {
                    J.pend |= P_TRIAL;
                    J.state = J_TRIAL;
                }
            }
            break;
        }
        case J_POLISH: {
            J.stats[ ST_NB_DIAG ] += 1;
            J.stats[ ST_NB_POLISH ] += 1;
            B = rep_host( c, J, 1 - J.repA );
            const long n = J.G.n;
            std::vector<double> a2( n ), nu( n );
            CK( cudaMemcpyAsync( a2.data(), J.a2, n * 8, cudaMemcpyDeviceToHost, c.stream ) );
            CK( cudaMemcpyAsync( nu.data(), J.nu, n * 8, cudaMemcpyDeviceToHost, c.stream ) );
            CK( cudaStreamSynchronize( c.stream ) );
            double after = 0;
            for ( int m : J.cl_members ) after = std::max( after, std::fabs( a2[ m ] - nu[ m ] ) );
            const bool agg_ok = B[ R_WORST ] <= J.opt[ SDOT_OPT_TOL_ABS ] || ( J.opt[ SDOT_OPT_TOL_REL ] > 0 && B[ R_WORST_REL ] <= J.opt[ SDOT_OPT_TOL_REL ] );
            const bool giant = c.hscal[ size_t( J.slot ) * SLOT_DOUBLES + SLOT_REFUSE ] != 0;
            if ( ! giant && after < J.polish_before && B[ R_AMIN ] > 0 && agg_ok ) {
                accept_trial( J );
                J.stats[ ST_RESIDUAL ] = B[ R_WORST ];
                ++J.polish_round;
                if ( polish_start( c, J ) ) break;
            }
            final_status( c, J );
            break;
        }
        case J_FINAL:
            J.stats[ ST_T_TOTAL ] = now_s() - J.t_begin;
            J.state = J_DONE;
            break;
        default:
            break;
        }
    }
    if ( had_cg && J.state == J_CG ) {
        const double *S = sc_host( c, J );
        if ( S[ SC_CONV ] != 0 ) {
            J.stats[ ST_LIN_NB_ITER ] += S[ SC_ITER ];
            if ( S[ SC_BNORM ] > 0 ) J.stats[ ST_LIN_WORST ] = std::max( J.stats[ ST_LIN_WORST ], S[ SC_RNORM ] / S[ SC_BNORM ] );
            if ( S[ SC_FAIL ] != 0 && J.mx_mem && ! J.mx_off ) {
                // the FP32 CG failed on this system (its refinement stalled, or p . A p lost its sign to FP32 rounding):
                // it is solved again by the FP64 CG (its FP32 multigrid levels inside an FP64 CG), and so are the later
                // systems of this solve
                J.mx_off = true;
                J.pend |= P_NEWTON;
            } else if ( S[ SC_FAIL ] != 0 ) {
                J.nstatus = NS_LINEAR_FAILURE;
                end_stage( c, J );
            } else {
                J.pend |= P_GAUGE | P_TRIAL;
                J.t = std::min( 1.0, J.opt[ SDOT_OPT_MULT_OK ] * J.t_last );
                if ( J.lim_on ) { J.t = J.beta; J.lim_probe = true; J.lim_round = 0; }
                J.trial = 0;
                J.nb_evals = 0;
                J.h_has = false;
                J.state = J_TRIAL;
            }
        }
    }
    if ( J.state == J_ITER ) newton_iter( c, J );
}

static VecDev vec_of( Ctx &c, SolveJob &J ) {
    VecDev V;
    std::memset( &V, 0, sizeof( V ) );
    V.n = J.G.n;
    V.cap = J.cap;
    V.rank0 = J.rank0;
    V.res = J.res_cur;
    V.power = J.opt[ SDOT_OPT_POWER ];
    V.nb = J.nb[ J.cur ];
    V.nid = J.nid[ J.cur ];
    V.nc = J.nc[ J.cur ];
    V.ovf_ids = J.ovf_ids[ J.cur ];
    V.ovf_c = J.ovf_c[ J.cur ];
    V.row_ptr = J.row_ptr;
    V.col = J.col;
    V.val = J.val;
    V.dia = J.dia;
    V.rowcnt = J.rowcnt;
    V.x = J.x; V.r = J.r; V.z = J.z; V.p = J.p; V.q = J.q; V.b = J.b;
    V.nu = J.nu;
    V.a = J.a;
    V.w = J.w; V.w2 = J.w2; V.d = J.d;
    V.t = J.t;
    V.tol = J.opt[ SDOT_OPT_LIN_TOL ] > 0 ? J.opt[ SDOT_OPT_LIN_TOL ] : 1e-6;     // the card's default (gpu/Linear2D.cuh:82)
    V.maxit = J.opt[ SDOT_OPT_LIN_MAXIT ] > 0 ? int( J.opt[ SDOT_OPT_LIN_MAXIT ] ) : 20000;
    V.report = rep_dev( c, J, J.repA );
    V.wmax_slot = J.wslot + ( 1 - J.wcur );
    V.sc = sc_dev( c, J );
    V.partials = J.part_vec;
    V.counter = c.dcount + 4 * J.slot + 1;
    V.nchunk = J.nch_vec;
    V.active = 1;
    V.precond = J.mg_L > 0 ? 1 : 0;
    if ( J.mx_mem && ! J.mx_off ) {
        V.mixed = 1;
        V.val32 = J.val32; V.dia32 = J.dia32; V.x32 = J.x32; V.r32 = J.r32; V.z32 = J.z32; V.p32 = J.p32; V.q32 = J.q32;
    }
    if ( J.agg_margin > 0 ) {
        V.agg_pairs = J.agg_pairs;
        V.agg_cap = AGG_CAP;
        V.agg_count = c.dscal + size_t( J.slot ) * SLOT_DOUBLES + SLOT_AGG;
        V.agg_margin = J.agg_margin;
        V.agg_tol_abs = J.opt[ SDOT_OPT_TOL_ABS ];
        V.agg_tol_rel = J.opt[ SDOT_OPT_TOL_REL ];
        V.agg_ccond = 1e9 * J.c_scale;
    }
    return V;
}

struct VecBatch {
    std::vector<VecDev> v;
    std::vector<Chunk> ch;
    std::vector<const SolveJob *> jobs;
    // the multigrid part: per level the descriptors of the jobs that have it and their chunk tables
    int maxL = 0;
    std::vector<MgLevel> lv[ MG_MAX_LEVELS ];
    std::vector<Chunk> down[ MG_MAX_LEVELS ], up[ MG_MAX_LEVELS ], crs[ MG_MAX_LEVELS ];
    std::vector<MgLevel> bottom;
    // the cycle's small levels (at most MG_FUSE_ROWS rows, down to the coarsest): one fused launch, a block per problem
    std::vector<MgLevel> fchain;
    std::vector<int2> fidx;
    std::vector<Chunk> build0;                     // the level-0 rows of every problem, for the hierarchy's build
    struct MgJob { const SolveJob *J; int q[ MG_MAX_LEVELS ]; };    // a problem's index in lv[ l ], per level
    std::vector<MgJob> mgjobs;
    bool down_up_planned = false;
    // device copies
    VecDev *dv = nullptr;
    Chunk *dch = nullptr;
    MgLevel *dlv[ MG_MAX_LEVELS ], *dbottom = nullptr, *dfchain = nullptr;
    int2 *dfidx = nullptr;
    Chunk *dbuild0 = nullptr;
    Chunk *ddown[ MG_MAX_LEVELS ], *dup[ MG_MAX_LEVELS ], *dcrs[ MG_MAX_LEVELS ];

    void add( const VecDev &d, const SolveJob *J = nullptr ) {
        int p = int( v.size() );
        VecDev x = d;
        x.chunk0 = int( ch.size() );
        v.push_back( x );
        jobs.push_back( J );
        int k = 0;
        const int vc = vec_chunk( d.n );
        for ( int b = 0; b < d.n; b += vc, ++k ) ch.push_back( Chunk{ p, b, std::min( d.n, b + vc ), k } );
        if ( ! J || ! J->mg_L || ! d.precond ) return;
        maxL = std::max( maxL, J->mg_L );
        MgJob mj{ J, {} };
        for ( int l = 0; l < J->mg_L; ++l ) {
            int q = int( lv[ l ].size() );
            mj.q[ l ] = q;
            lv[ l ].push_back( mg_level( *J, l, p ) );
            if ( l == 0 ) {
                int kk = 0;
                for ( int b = 0; b < J->mg_n[ 0 ]; b += vc, ++kk ) build0.push_back( Chunk{ q, b, std::min( J->mg_n[ 0 ], b + vc ), kk } );
            }
            if ( l + 1 < J->mg_L ) {
                const int nn = J->mg_n[ l + 1 ];
                int kk = 0;
                for ( int b = 0; b < nn; b += MG_CCH, ++kk ) crs[ l ].push_back( Chunk{ q, b, std::min( nn, b + MG_CCH ), kk } );
            } else
                bottom.push_back( lv[ l ].back() );
        }
        mgjobs.push_back( mj );
    }
    // the cycle's launches: the levels above the fusion threshold one launch per level and direction, the others of each
    // problem in the fused launch (a block per problem).  A block holds one SM, so the threshold is small when few problems
    // share the batch (their larger levels are better spread over the GPU) and larger when many do
    void plan_cycle() {
        down_up_planned = true;
        const int T = mgjobs.size() >= 32 ? MG_FUSE_ROWS : MG_FUSE_ROWS / 8;
        for ( const MgJob &mj : mgjobs ) {
            const SolveJob *J = mj.J;
            int f = J->mg_L - 1;
            while ( f > 0 && J->mg_n[ f - 1 ] <= T ) --f;
            fidx.push_back( make_int2( int( fchain.size() ), J->mg_L - f ) );
            for ( int l = 0; l < J->mg_L; ++l ) {
                const int q = mj.q[ l ];
                if ( l >= f ) fchain.push_back( lv[ l ][ q ] );
                if ( l >= f || l + 1 >= J->mg_L ) continue;
                const int nn = J->mg_n[ l + 1 ], n = J->mg_n[ l ];
                int kk = 0;
                for ( int b = 0; b < nn; b += MG_RCH, ++kk ) down[ l ].push_back( Chunk{ q, b, std::min( nn, b + MG_RCH ), kk } );
                kk = 0;
                for ( int b = 0; b < n; b += MG_RCH, ++kk ) up[ l ].push_back( Chunk{ q, b, std::min( n, b + MG_RCH ), kk } );
            }
        }
    }
    bool mg() const { return maxL > 0; }
    // what the launches of a CG burst depend on: the upload area, the burst, and every table's size
    std::vector<long long> layout_key( const char *desc, int burst ) {
        if ( ! down_up_planned ) plan_cycle();
        std::vector<long long> k{ ( long long ) ( uintptr_t ) desc, burst, ( long long ) ch.size(), maxL, ( long long ) bottom.size() };
        for ( auto &x : v ) { k.push_back( x.n ); k.push_back( x.precond ); k.push_back( x.mixed ); }
        for ( int l = 0; l < maxL; ++l ) {
            k.push_back( ( long long ) lv[ l ].size() );
            k.push_back( ( long long ) down[ l ].size() );
            k.push_back( ( long long ) up[ l ].size() );
            k.push_back( ( long long ) crs[ l ].size() );
        }
        k.push_back( ( long long ) fchain.size() );
        k.push_back( ( long long ) fidx.size() );
        return k;
    }
    // everything in one copy
    void upload( Ctx &c ) {
        if ( ! down_up_planned ) plan_cycle();
        std::vector<std::pair<const void *, size_t>> parts;
        parts.push_back( { v.data(), v.size() * sizeof( VecDev ) } );
        parts.push_back( { ch.data(), ch.size() * sizeof( Chunk ) } );
        for ( int l = 0; l < maxL; ++l ) {
            parts.push_back( { lv[ l ].data(), lv[ l ].size() * sizeof( MgLevel ) } );
            parts.push_back( { down[ l ].data(), down[ l ].size() * sizeof( Chunk ) } );
            parts.push_back( { up[ l ].data(), up[ l ].size() * sizeof( Chunk ) } );
            parts.push_back( { crs[ l ].data(), crs[ l ].size() * sizeof( Chunk ) } );
        }
        parts.push_back( { bottom.data(), bottom.size() * sizeof( MgLevel ) } );
        parts.push_back( { fchain.data(), fchain.size() * sizeof( MgLevel ) } );
        parts.push_back( { fidx.data(), fidx.size() * sizeof( int2 ) } );
        parts.push_back( { build0.data(), build0.size() * sizeof( Chunk ) } );
        std::vector<size_t> off;
        size_t total = 0;
        for ( auto &p : parts ) { off.push_back( total ); total += ( p.second + 255 ) & ~size_t( 255 ); }
        std::vector<char> buf( total + 256 );
        for ( size_t k = 0; k < parts.size(); ++k ) if ( parts[ k ].second ) std::memcpy( buf.data() + off[ k ], parts[ k ].first, parts[ k ].second );
        char *d = upload_desc( c, buf.data(), total + 256 );
        int k = 0;
        dv = reinterpret_cast<VecDev *>( d + off[ k++ ] );
        dch = reinterpret_cast<Chunk *>( d + off[ k++ ] );
        for ( int l = 0; l < maxL; ++l ) {
            dlv[ l ] = reinterpret_cast<MgLevel *>( d + off[ k++ ] );
            ddown[ l ] = reinterpret_cast<Chunk *>( d + off[ k++ ] );
            dup[ l ] = reinterpret_cast<Chunk *>( d + off[ k++ ] );
            dcrs[ l ] = reinterpret_cast<Chunk *>( d + off[ k++ ] );
        }
        dbottom = reinterpret_cast<MgLevel *>( d + off[ k++ ] );
        dfchain = reinterpret_cast<MgLevel *>( d + off[ k++ ] );
        dfidx = reinterpret_cast<int2 *>( d + off[ k++ ] );
        dbuild0 = reinterpret_cast<Chunk *>( d + off[ k++ ] );
    }
    // the hierarchies of every job, from their fresh Laplacians
    void build( const Launch &L, ErrRec *err ) {
        if ( ! mg() ) return;
        std::vector<Chunk> l0;
        // level 0 rows: the vector chunks, re-indexed to the level-0 array
        launch_mg_level0( L, dlv[ 0 ], dv, dbuild0, int( build0.size() ) );
        for ( int l = 0; l + 1 < maxL; ++l ) launch_mg_coarsen( L, dlv[ l ], int( lv[ l ].size() ), dcrs[ l ], int( crs[ l ].size() ), err );
        launch_mg_bottom_build( L, dbottom, int( bottom.size() ) );
    }
    // z = M^-1 r for every job
    void vcycle( const Launch &L ) {
        for ( int l = 0; l + 1 < maxL; ++l ) launch_mg_down( L, dlv[ l ], dv, ddown[ l ], int( down[ l ].size() ) );
        launch_mg_fused( L, dfchain, dfidx, dv, int( fidx.size() ) );
        for ( int l = maxL - 2; l >= 0; --l ) launch_mg_up( L, dlv[ l ], dv, dup[ l ], int( up[ l ].size() ) );
    }
};

// one Laplacian given as a device CSR (V: matrix, work vectors, scalars; b and SC_MEAN uploaded): its solve by the CG
// preconditioned with the aggregation multigrid of the Newton engine (aggregates of 4 consecutive rows, 8 when the rows
// hold more than 10 entries on average, as in 3D),
// x in V.x, the gauge-fixed direction in V.d.  Returns the CG iterations, -1 if the CG failed.
// a CG burst as a CUDA graph: captured the first time a batch layout is seen, replayed while it stays the same (the
// descriptors it reads are re-uploaded into the same area before every replay); direct launches if capture fails
template<class Issue>
static void run_burst( Ctx &c, const std::vector<long long> &key, Issue issue ) {
    for ( auto &g : c.graphs )
        if ( g.key == key ) {
            CK( cudaGraphLaunch( g.exec, c.stream ) );
            c.launches += g.launches;
            return;
        }
    const unsigned long long l0 = c.launches;
    if ( cudaStreamBeginCapture( c.stream, cudaStreamCaptureModeThreadLocal ) != cudaSuccess ) {
        cudaGetLastError();
        issue();
        return;
    }
    issue();
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const unsigned long long n = c.launches - l0;
    c.launches = l0;
    bool ok = cudaStreamEndCapture( c.stream, &graph ) == cudaSuccess && graph &&
              cudaGraphInstantiate( &exec, graph, 0 ) == cudaSuccess;
    if ( graph ) cudaGraphDestroy( graph );
    if ( ! ok ) {
        cudaGetLastError();
        issue();
        return;
    }
    if ( c.graphs.size() >= 32 ) {
        cudaGraphExecDestroy( c.graphs.front().exec );
        c.graphs.erase( c.graphs.begin() );
    }
    c.graphs.push_back( Ctx::BurstGraph{ key, exec, n } );
    CK( cudaGraphLaunch( exec, c.stream ) );
    c.launches += n;
}

constexpr int MG_BURST_SOLVE = 8;
int mg_linear_solve( Ctx &c, const VecDev &V0, long nnz, double *hsc ) {
    SolveJob J;                                      // only its hierarchy is used
    J.G.dim = nnz > 10 * long( V0.n ) ? 3 : 2;       // the aggregates of a 3D Laplacian (about 15 entries a row) pack 8 rows
    J.G.n = V0.n;
    J.cap = int( ( nnz + V0.n - 1 ) / V0.n ) + 1;
    J.row_ptr = V0.row_ptr;
    J.col = V0.col;
    alloc_mg( c, J );
    struct Free {
        Ctx &c;
        SolveJob &J;
        ~Free() { if ( J.mg_mem ) dfree( c, J.mg_mem ); }
    } fr{ c, J };
    VecDev V = V0;
    V.precond = J.mg_L > 0 ? 1 : 0;
    VecBatch B;
    B.add( V, &J );
    B.upload( c );
    Launch L = c.L();
    const int nch = int( B.ch.size() );
    const bool mixed = V.mixed != 0;
    if ( B.mg() ) {
        B.build( L, c.derr );
        if ( mixed ) launch_mx_init( L, B.dv, B.dch, nch );
        else launch_cg_init0( L, B.dv, B.dch, nch );
        B.vcycle( L );
        if ( mixed ) launch_mx_init1( L, B.dv, B.dch, nch );
        else launch_cg_init1( L, B.dv, B.dch, nch );
    } else if ( mixed )
        launch_mx_init( L, B.dv, B.dch, nch );
    else
        launch_cg_init( L, B.dv, B.dch, nch );
    for ( ;; ) {
        for ( int k = 0; k < MG_BURST_SOLVE; ++k ) {
            if ( B.mg() ) {
                if ( mixed ) launch_mx_spmv_update( L, B.dv, B.dch, nch );
                else launch_cg_spmv_update( L, B.dv, B.dch, nch );
                B.vcycle( L );
                if ( mixed ) launch_mx_rz_p( L, B.dv, B.dch, nch );
                else launch_cg_rz_p( L, B.dv, B.dch, nch );
            } else if ( mixed )
                launch_mx_iter( L, B.dv, B.dch, nch );
            else
                launch_cg_iter( L, B.dv, B.dch, nch );
        }
        CK( cudaMemcpyAsync( hsc, V.sc, NB_SC * sizeof( double ), cudaMemcpyDeviceToHost, c.stream ) );
        CK( cudaMemcpyAsync( c.herr, c.derr, sizeof( ErrRec ), cudaMemcpyDeviceToHost, c.stream ) );
        CK( cudaStreamSynchronize( c.stream ) );
        check_errors( c, "multigrid" );
        if ( hsc[ SC_CONV ] != 0 ) break;
    }
    launch_gauge( L, B.dv, B.dch, nch );
    return hsc[ SC_FAIL ] != 0 ? -1 : int( hsc[ SC_ITER ] );
}

// phase D: the vector work the decisions asked for
static void launch_pending( Ctx &c, std::vector<SolveJob *> &jobs ) {
    Launch L = c.L();
    VecBatch newton, gauge, trial;
    for ( SolveJob *J : jobs ) {
        if ( ! J->pend ) continue;
        if ( J->pend & P_RESCALE ) launch_gather_vec( L, J->nu_dev_user, J->G.user, J->G.n, J->nu, J->nu_scale );
        if ( J->pend & P_ZERO_W2 ) {
            CK( cudaMemsetAsync( J->w2, 0, size_t( J->G.n ) * 8, c.stream ) );
            CK( cudaMemsetAsync( J->wslot + ( 1 - J->wcur ), 0, 8, c.stream ) );
            launch_wmax( L, J->w2, J->G.n, J->wslot + ( 1 - J->wcur ) );
        }
        if ( J->pend & P_SET_W2 ) {
            CK( cudaMemcpyAsync( J->tmpw, J->wsim.data(), size_t( J->G.n ) * 8, cudaMemcpyHostToDevice, c.stream ) );
            launch_gather_vec( L, J->tmpw, J->G.user, J->G.n, J->w2, 1.0 );
            CK( cudaMemsetAsync( J->wslot + ( 1 - J->wcur ), 0, 8, c.stream ) );
            launch_wmax( L, J->w2, J->G.n, J->wslot + ( 1 - J->wcur ) );
        }
        VecDev V = vec_of( c, *J );
        if ( J->pend & P_NEWTON ) newton.add( V, J );
        if ( J->pend & P_GAUGE ) gauge.add( V );
        if ( J->pend & P_TRIAL ) {
            CK( cudaMemsetAsync( J->wslot + ( 1 - J->wcur ), 0, 8, c.stream ) );
            trial.add( V );
        }
    }
    if ( ! newton.v.empty() ) {
        // Jacobi- and multigrid-preconditioned problems, FP64 and mixed CG, go in four batches
        VecBatch jac, mgb, jacx, mgbx;
        for ( size_t k = 0; k < newton.v.size(); ++k ) {
            const VecDev &v = newton.v[ k ];
            ( v.precond ? ( v.mixed ? mgbx : mgb ) : ( v.mixed ? jacx : jac ) ).add( v, newton.jobs[ k ] );
        }
        for ( VecBatch *B : { &jac, &mgb, &jacx, &mgbx } ) {
            if ( B->v.empty() ) continue;
            B->upload( c );
            const int nch = int( B->ch.size() );
            double rows = 0;
            for ( auto &v : B->v ) rows += v.n;
            c.timer.begin( c.stream, K_LAPLACIAN, rows );
            launch_lap_count( L, B->dv, B->dch, nch );
            launch_lap_scan( L, B->dv, int( B->v.size() ) );
            launch_lap_fill( L, B->dv, B->dch, nch );
            bool agg = false;
            for ( auto &v : B->v ) agg |= v.agg_pairs != nullptr;
            if ( agg ) launch_agg_detect( L, B->dv, B->dch, nch );
            for ( const SolveJob *J : B->jobs )
                if ( J && J->ncl > 0 && J->cl_true )
                    launch_agg_cap( L, J->row_ptr, J->col, J->val, J->dia, J->d_cl, J->ncl, 1e6 * J->c_scale, J->cl_true );
            launch_rhs( L, B->dv, B->dch, nch );
            const bool mixed = B == &jacx || B == &mgbx;
            if ( B->mg() ) {
                c.timer.end( c.stream, 5 );
                c.timer.begin( c.stream, K_MULTIGRID, rows );
                B->build( L, c.derr );
                if ( mixed ) launch_mx_init( L, B->dv, B->dch, nch );
                else launch_cg_init0( L, B->dv, B->dch, nch );
                B->vcycle( L );
                if ( mixed ) launch_mx_init1( L, B->dv, B->dch, nch );
                else launch_cg_init1( L, B->dv, B->dch, nch );
            } else if ( mixed )
                launch_mx_init( L, B->dv, B->dch, nch );
            else
                launch_cg_init( L, B->dv, B->dch, nch );
            c.timer.end( c.stream, 5 );
        }
    }
    for ( SolveJob *J : jobs )
        if ( ( J->pend & P_GAUGE ) && J->ncl > 0 && J->cl_true )
            launch_agg_direction( L, J->row_ptr, J->col, J->val, J->d_cl, J->ncl, J->cl_true, J->nu, J->b, J->x,
                                  J->cl_true + J->cl_members.size() * ( AGG_KMAX + 1 ) );
    if ( ! gauge.v.empty() ) {
        gauge.upload( c );
        launch_gauge( L, gauge.dv, gauge.dch, int( gauge.ch.size() ) );
    }
    if ( ! trial.v.empty() ) {
        trial.upload( c );
        launch_trial( L, trial.dv, trial.dch, int( trial.ch.size() ) );
    }
    for ( SolveJob *J : jobs ) J->pend = 0;
}

constexpr int CG_BURST = 32;
constexpr int MG_BURST = 8;

void jobs_tick( Ctx &c, std::vector<SolveJob *> &jobs ) {
    Launch L = c.L();
    // A. the diagrams
    std::vector<ProbDev> P2, P3, PR;
    // the diagrams of solves with clusters: their reports again, from the clusters' shares of the masses
    struct AggDiag { SolveJob *J; ProbDev P; };
    std::vector<AggDiag> AG;
    auto agg_reports = [&]() {
        if ( AG.empty() ) return;
        std::vector<ProbDev> Q;
        std::vector<Chunk> QC;
        for ( auto &e : AG ) {
            SolveJob *J = e.J;
            CK( cudaMemcpyAsync( J->ae, e.P.mass, size_t( J->G.n ) * 8, cudaMemcpyDeviceToDevice, c.stream ) );
            launch_agg_shares( L, e.P.mass, J->nu, J->d_cl, J->d_cl + J->ncl + 1, J->ncl, J->ae );
            ProbDev P = e.P;
            P.mass = J->ae;
            const int qi = int( Q.size() );
            Q.push_back( P );
            int k = 0;
            const int cs = cell_chunk( J->G.dim, J->G.n );
            for ( int b = 0; b < J->G.n; b += cs, ++k ) QC.push_back( Chunk{ qi, b, std::min( J->G.n, b + cs ), k } );
        }
        const size_t oq = ( Q.size() * sizeof( ProbDev ) + 255 ) & ~size_t( 255 );
        std::vector<char> buf( oq + QC.size() * sizeof( Chunk ) );
        std::memcpy( buf.data(), Q.data(), Q.size() * sizeof( ProbDev ) );
        std::memcpy( buf.data() + oq, QC.data(), QC.size() * sizeof( Chunk ) );
        char *d = ( char * ) dalloc( c, buf.size() );
        c.desc_spill.push_back( d );
        CK( cudaMemcpyAsync( d, stage( c, buf.data(), buf.size() ), buf.size(), cudaMemcpyHostToDevice, c.stream ) );
        launch_report( L, reinterpret_cast<ProbDev *>( d ), reinterpret_cast<Chunk *>( d + oq ), int( QC.size() ) );
    };
    // the limits step's probes of this tick: their descriptors (uploaded once), launched after the diagrams, and again after
    // a big-cell pass (which completes the masses the kernel reads)
    struct LimLaunch { char *d = nullptr; size_t off = 0; int nch = 0; std::vector<SolveJob *> js; } LL;
    auto limits_launch = [&]() {
        if ( LL.js.empty() ) return;
        for ( SolveJob *J : LL.js ) {
            double *o = c.dscal + size_t( J->slot ) * SLOT_DOUBLES + SLOT_LIM;
            CK( cudaMemsetAsync( o, 0, 8, c.stream ) );
            CK( cudaMemsetAsync( o + 1, 0xff, 8, c.stream ) );
        }
        launch_limits2d( L, reinterpret_cast<LimDev *>( LL.d ), reinterpret_cast<Chunk *>( LL.d + LL.off ), LL.nch );
    };
    std::vector<Chunk> C2, C3, CR;
    std::vector<SolveJob *> with_diag;
    for ( SolveJob *J : jobs ) {
        DiagReq R;
        if ( J->state == J_DONE || ! needs_diagram( *J, R ) ) continue;
        with_diag.push_back( J );
        ProbDev P;
        J->G.fill( P );
        P.fp32 = int( J->opt[ SDOT_OPT_PRECISION ] ) == 1;
        P.cap = J->cap;
        P.w = R.w;
        P.wmax_slot = R.wslot;
        P.mass = R.mass;
        if ( R.table >= 0 ) {
            P.nb = J->nb[ R.table ]; P.nid = J->nid[ R.table ]; P.nc = J->nc[ R.table ];
            if ( J->ovf_cap ) {
                P.ovf_count = J->ovf_count[ R.table ]; P.ovf_cap = J->ovf_cap; P.ovf_ids = J->ovf_ids[ R.table ]; P.ovf_c = J->ovf_c[ R.table ];
                CK( cudaMemsetAsync( P.ovf_count, 0, sizeof( int ), c.stream ) );
            }
        }
        P.nu = J->nu;
        P.res = J->res_cur;
        P.power = J->opt[ SDOT_OPT_POWER ];
        P.perr = c.dscal + size_t( J->slot ) * SLOT_DOUBLES + SLOT_ERR;
        if ( J->state == J_TRIAL || J->state == J_POLISH ) {
            P.prefuse = c.dscal + size_t( J->slot ) * SLOT_DOUBLES + SLOT_REFUSE;
            CK( cudaMemsetAsync( P.prefuse, 0, 8, c.stream ) );
        }
        if ( R.report >= 0 ) {
            P.report = rep_dev( c, *J, R.report );
            P.partials = J->part_cells;
            P.counter = c.dcount + 4 * J->slot;
            P.nchunk = J->nch_cells;
        }
        if ( R.moments ) { P.first = J->obary; P.cost = J->ocost; }
        if ( J->ncl > 0 && R.report >= 0 ) AG.push_back( { J, P } );
        std::vector<ProbDev> &PP = R.report_only ? PR : ( J->G.dim == 2 ? P2 : P3 );
        std::vector<Chunk> &CC = R.report_only ? CR : ( J->G.dim == 2 ? C2 : C3 );
        int pi = int( PP.size() );
        P.chunk0 = int( CC.size() );
        PP.push_back( P );
        int k = 0;
        const int cs = cell_chunk( J->G.dim, J->G.n );
        for ( int b = 0; b < J->G.n; b += cs, ++k ) CC.push_back( Chunk{ pi, b, std::min( J->G.n, b + cs ), k } );
    }
    // the problems of this tick's diagrams in ONE array (both dimensions), so that the big-cell queue's problem indices mean
    // the same thing to every kernel: [ 2D normal | 2D final (moments) | 3D normal | 3D final ], flags uniform per launch
    std::vector<ProbDev> big_probs;
    std::vector<std::vector<Chunk>> big_chunks;      // per problem of big_probs, its chunks of a normal diagram (report recompute)
    size_t desc_used = 0;                            // bytes of the upload area this tick's cells use
    CK( cudaMemsetAsync( &c.dovf->count, 0, sizeof( int ), c.stream ) );
    {
        std::vector<ProbDev> PX;
        std::vector<Chunk> CX[ 4 ];                     // ( dim 2, 3 ) x ( normal, final )
        for ( int dim = 2; dim <= 3; ++dim ) {
            std::vector<ProbDev> &PP = dim == 2 ? P2 : P3;
            std::vector<Chunk> &CC = dim == 2 ? C2 : C3;
            std::vector<int> idx( PP.size(), -1 );
            for ( int pass = 0; pass < 2; ++pass )
                for ( size_t k = 0; k < PP.size(); ++k )
                    if ( ( PP[ k ].first != nullptr ) == ( pass == 1 ) ) { idx[ k ] = int( PX.size() ); PX.push_back( PP[ k ] ); }
            for ( auto &ch : CC ) {
                Chunk x = ch;
                x.prob = idx[ ch.prob ];
                CX[ 2 * ( dim - 2 ) + ( PP[ ch.prob ].first != nullptr ) ].push_back( x );
            }
        }
        if ( ! PX.empty() ) {
            size_t off[ 5 ];
            size_t total = ( PX.size() * sizeof( ProbDev ) + 255 ) & ~size_t( 255 );
            for ( int q = 0; q < 4; ++q ) { off[ q ] = total; total += ( CX[ q ].size() * sizeof( Chunk ) + 255 ) & ~size_t( 255 ); }
            std::vector<char> buf( total );
            std::memcpy( buf.data(), PX.data(), PX.size() * sizeof( ProbDev ) );
            for ( int q = 0; q < 4; ++q )
                if ( ! CX[ q ].empty() ) std::memcpy( buf.data() + off[ q ], CX[ q ].data(), CX[ q ].size() * sizeof( Chunk ) );
            char *d = upload_desc( c, buf.data(), buf.size() );
            desc_used = total;
            ProbDev *dp = reinterpret_cast<ProbDev *>( d );
            c.timer.begin( c.stream, K_INDEX, double( PX.size() ) );
            launch_wpyr( L, dp, int( PX.size() ) );
            c.timer.end( c.stream );
            for ( int q = 0; q < 4; ++q ) {
                if ( CX[ q ].empty() ) continue;
                const int dim = 2 + q / 2;
                Chunk *dc = reinterpret_cast<Chunk *>( d + off[ q ] );
                double seeds = 0;
                for ( auto &ch : CX[ q ] ) seeds += ch.end - ch.begin;
                unsigned flags = ( q & 1 ) ? ( F_MOMENTS | F_USER_ORDER ) : ( F_MASS | F_FACETS | F_REPORT );
                long gseeds = 0;
                if ( dim == 3 )
                    for ( auto &ch : CX[ q ] ) gseeds += PX[ ch.prob ].dkind == D_GAUSS ? ch.end - ch.begin : 0;
                const Split3 *sp = dim == 3 ? split3_for( c, int( CX[ q ].size() ), gseeds ) : nullptr;
                c.timer.begin( c.stream, dim == 2 ? K_CELLS2D : K_CELLS3D, seeds );
                int clips = 0;
                if ( dim == 2 )
                    for ( auto &ch : CX[ q ] ) clips |= PX[ ch.prob ].fp32 ? 2 : 1;
                if ( dim == 2 ) launch_cells2d( L, dp, dc, int( CX[ q ].size() ), flags, c.derr, c.dovf, clips );
                else launch_cells3d( L, dp, dc, int( CX[ q ].size() ), flags, c.derr, c.dovf, sp );
                c.timer.end( c.stream, sp ? 2 : 1 );
            }
            big_probs = PX;
            big_chunks.assign( PX.size(), {} );
            for ( int q : { 0, 2 } )
                for ( auto &ch : CX[ q ] ) big_chunks[ ch.prob ].push_back( ch );
        }
    }
    // the report-only problems (targets rescaled): their report from the masses in memory
    if ( ! PR.empty() ) {
        size_t b1 = PR.size() * sizeof( ProbDev ), o2 = ( b1 + 255 ) & ~size_t( 255 );
        std::vector<char> buf( o2 + CR.size() * sizeof( Chunk ) );
        std::memcpy( buf.data(), PR.data(), b1 );
        std::memcpy( buf.data() + o2, CR.data(), CR.size() * sizeof( Chunk ) );
        char *d = desc_used ? upload_desc_at( c, buf.data(), buf.size(), desc_used ) : upload_desc( c, buf.data(), buf.size() );
        double seeds = 0;
        for ( auto &ch : CR ) seeds += ch.end - ch.begin;
        c.timer.begin( c.stream, K_REPORT, seeds );
        launch_report( L, reinterpret_cast<ProbDev *>( d ), reinterpret_cast<Chunk *>( d + o2 ), int( CR.size() ) );
        c.timer.end( c.stream );
    }
    agg_reports();
    {
        std::vector<LimDev> LD;
        std::vector<Chunk> LC;
        for ( SolveJob *J : with_diag ) {
            if ( J->state != J_TRIAL || ! J->lim_probe ) continue;
            LimDev D;
            std::memset( &D, 0, sizeof( D ) );
            J->G.fill( D.P );
            D.P.fp32 = 0;
            D.P.cap = J->cap;
            D.P.w = J->w;
            D.d = J->d;
            D.a2 = J->a2;
            D.nb0 = J->nb[ J->cur ]; D.nid0 = J->nid[ J->cur ];
            D.nb1 = J->nb[ 1 - J->cur ]; D.nid1 = J->nid[ 1 - J->cur ];
            D.eps = J->eps;
            D.t = J->t;
            D.out = c.dscal + size_t( J->slot ) * SLOT_DOUBLES + SLOT_LIM;
            const int li = int( LD.size() );
            LD.push_back( D );
            int k = 0;
            for ( int b = 0; b < J->G.n; b += CHUNK, ++k ) LC.push_back( Chunk{ li, b, std::min( J->G.n, b + CHUNK ), k } );
            LL.js.push_back( J );
        }
        if ( ! LD.empty() ) {
            LL.off = ( LD.size() * sizeof( LimDev ) + 255 ) & ~size_t( 255 );
            std::vector<char> buf( LL.off + LC.size() * sizeof( Chunk ) );
            std::memcpy( buf.data(), LD.data(), LD.size() * sizeof( LimDev ) );
            std::memcpy( buf.data() + LL.off, LC.data(), LC.size() * sizeof( Chunk ) );
            LL.d = ( char * ) dalloc( c, buf.size() );
            c.desc_spill.push_back( LL.d );
            LL.nch = int( LC.size() );
            CK( cudaMemcpyAsync( LL.d, stage( c, buf.data(), buf.size() ), buf.size(), cudaMemcpyHostToDevice, c.stream ) );
            c.timer.begin( c.stream, K_CELLS2D, 0.0 );
            limits_launch();
            c.timer.end( c.stream );
        }
    }
    // B. CG iterations
    VecBatch cgj, cgm, cgjx, cgmx;
    std::vector<SolveJob *> with_cg;
    for ( SolveJob *J : jobs )
        if ( J->state == J_CG ) {
            VecDev V = vec_of( c, *J );
            ( V.precond ? ( V.mixed ? cgmx : cgm ) : ( V.mixed ? cgjx : cgj ) ).add( V, J );
            with_cg.push_back( J );
        }
    for ( VecBatch *B : { &cgj, &cgm, &cgjx, &cgmx } ) {
        if ( B->v.empty() ) continue;
        B->upload( c );
        const int nch = int( B->ch.size() );
        int burst = B->mg() ? MG_BURST : CG_BURST;
        if ( with_diag.empty() ) burst *= 4;
        double rows = 0;
        for ( auto &v : B->v ) rows += v.n;
        const bool mixed = B == &cgjx || B == &cgmx;
        auto issue = [&]() {
            for ( int k = 0; k < burst; ++k ) {
                if ( B->mg() ) {
                    if ( mixed ) launch_mx_spmv_update( L, B->dv, B->dch, nch );
                    else launch_cg_spmv_update( L, B->dv, B->dch, nch );
                    B->vcycle( L );
                    if ( mixed ) launch_mx_rz_p( L, B->dv, B->dch, nch );
                    else launch_cg_rz_p( L, B->dv, B->dch, nch );
                } else if ( mixed )
                    launch_mx_iter( L, B->dv, B->dch, nch );
                else
                    launch_cg_iter( L, B->dv, B->dch, nch );
            }
        };
        unsigned long long l0 = c.launches;
        c.timer.begin( c.stream, K_CG, rows * burst );
        run_burst( c, B->layout_key( c.desc, burst ), issue );
        c.timer.end( c.stream, c.launches - l0 );
    }
    // C. one read-back, then the decisions
    int top = 0;
    for ( SolveJob *J : jobs ) top = std::max( top, J->slot + 1 );
    CK( cudaMemcpyAsync( c.hscal, c.dscal, size_t( top ) * SLOT_DOUBLES * 8, cudaMemcpyDeviceToHost, c.stream ) );
    CK( cudaMemcpyAsync( c.herr, c.derr, sizeof( ErrRec ), cudaMemcpyDeviceToHost, c.stream ) );
    CK( cudaMemcpyAsync( c.hovf, &c.dovf->count, sizeof( int ), cudaMemcpyDeviceToHost, c.stream ) );
    CK( cudaStreamSynchronize( c.stream ) );
    c.hstage_used = 0;                   // every upload of the ring has completed
    clear_capacity_error( c );
    check_errors( c, "cells" );
    if ( *c.hovf > 0 ) {
        // the big cells: rebuilt in global memory, then the reports of their problems recomputed from the masses
        const int count = std::min( *c.hovf, c.ovf_cap );
        std::vector<OvfItem> items( count );
        CK( cudaMemcpy( items.data(), ( char * ) c.dovf + 256, count * sizeof( OvfItem ), cudaMemcpyDeviceToHost ) );
        ProbDev *dp = reinterpret_cast<ProbDev *>( upload_desc( c, big_probs.data(), big_probs.size() * sizeof( ProbDev ) ) );
        std::vector<char> touched( big_probs.size(), 0 );
        for ( auto &it : items ) touched[ it.prob ] = 1;
        c.timer.begin( c.stream, K_CELLS2D, double( count ) );
        launch_cells2d_big( L, dp, c.dovf, count, 0, c.derr, c.big_scratch, c.big_warps );     // flags per problem
        launch_cells3d_big( L, dp, c.dovf, count, 0, c.derr, c.dgiant );
        run_giant_cells( c, dp, 0 );
        c.timer.end( c.stream );
        std::vector<Chunk> rc;
        for ( size_t k = 0; k < big_probs.size(); ++k )
            if ( touched[ k ] && big_probs[ k ].report ) rc.insert( rc.end(), big_chunks[ k ].begin(), big_chunks[ k ].end() );
        if ( ! rc.empty() ) {
            Chunk *dc = reinterpret_cast<Chunk *>( upload_desc_at( c, rc.data(), rc.size() * sizeof( Chunk ), big_probs.size() * sizeof( ProbDev ) ) );
            launch_report( L, dp, dc, int( rc.size() ) );
        }
        agg_reports();
        limits_launch();
        CK( cudaMemcpyAsync( c.hscal, c.dscal, size_t( top ) * SLOT_DOUBLES * 8, cudaMemcpyDeviceToHost, c.stream ) );
        CK( cudaMemcpyAsync( c.herr, c.derr, sizeof( ErrRec ), cudaMemcpyDeviceToHost, c.stream ) );
        CK( cudaStreamSynchronize( c.stream ) );
        clear_capacity_error( c );
        check_errors( c, "big cells" );
    }
    for ( SolveJob *J : jobs ) {
        if ( J->state == J_DONE ) continue;
        bool hd = std::find( with_diag.begin(), with_diag.end(), J ) != with_diag.end();
        bool hc = std::find( with_cg.begin(), with_cg.end(), J ) != with_cg.end();
        decide( c, *J, hd, hc );
    }
    // D. the vector work
    launch_pending( c, jobs );
    for ( void *p : c.desc_spill ) dfree( c, p );
    c.desc_spill.clear();
}

void job_run( Ctx &c, std::vector<SolveJob *> &jobs, int max_ticks ) {
    for ( int tick = 0; max_ticks < 0 || tick < max_ticks; ++tick ) {
        bool any = false;
        for ( SolveJob *J : jobs ) any |= J->state != J_DONE;
        if ( ! any ) break;
        jobs_tick( c, jobs );
    }
}

void job_outputs( Ctx &c, SolveJob *J, sdot_solve_out &out, int memory ) {
    const long n = J->G.n;
    const int dim = J->G.dim;
    Launch L = c.L();
    // weights and masses back to user order, in the job's scratch
    double *wu = J->x, *au = J->r;
    launch_scatter( L, J->w, J->G.user, int( n ), 1, wu );
    launch_scatter( L, J->a, J->G.user, int( n ), 1, au );
    auto kind = memory == SDOT_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if ( out.weights ) CK( cudaMemcpyAsync( out.weights, wu, n * 8, kind, c.stream ) );
    if ( out.masses ) CK( cudaMemcpyAsync( out.masses, au, n * 8, kind, c.stream ) );
    if ( out.barycentres ) CK( cudaMemcpyAsync( out.barycentres, J->obary, size_t( n ) * dim * 8, kind, c.stream ) );
    std::vector<double> costs( n );
    CK( cudaMemcpyAsync( costs.data(), J->ocost, n * 8, cudaMemcpyDeviceToHost, c.stream ) );
    CK( cudaStreamSynchronize( c.stream ) );
    double cost = 0;
    for ( double v : costs ) cost += v;
    if ( out.cost ) {
        if ( memory == SDOT_DEVICE ) CK( cudaMemcpyAsync( out.cost, &cost, 8, cudaMemcpyHostToDevice, c.stream ) );
        else *out.cost = cost;
    }
    J->stats[ ST_DOMAIN_MASS ] = J->domain_mass;
    if ( ! J->full_set ) J->stats[ ST_RESIDUAL_FULL ] = J->stats[ ST_RESIDUAL ];
    if ( out.clusters ) {
        // each seed's cluster by its smallest user index
        std::vector<int32_t> cl( n );
        for ( long i = 0; i < n; ++i ) cl[ i ] = int32_t( i );
        std::vector<int> user( n );
        if ( J->ncl > 0 ) {
            CK( cudaMemcpy( user.data(), J->G.user, n * sizeof( int ), cudaMemcpyDeviceToHost ) );
            for ( int k = 0; k < J->ncl; ++k ) {
                int rep = INT32_MAX;
                for ( int q = J->cl_begin[ k ]; q < J->cl_begin[ k + 1 ]; ++q ) rep = std::min( rep, user[ J->cl_members[ q ] ] );
                for ( int q = J->cl_begin[ k ]; q < J->cl_begin[ k + 1 ]; ++q ) cl[ user[ J->cl_members[ q ] ] ] = rep;
            }
        }
        CK( cudaMemcpy( out.clusters, cl.data(), n * sizeof( int32_t ), memory == SDOT_DEVICE ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost ) );
    }
    J->stats[ ST_IT_DOUBLE ] = -1;
    std::memcpy( out.stats, J->stats, sizeof( out.stats ) );
    int rows = int( J->hist.size() / SDOT_NB_HIST );
    if ( out.history && out.cap_history > 0 ) {
        int k = std::min( rows, out.cap_history );
        std::memcpy( out.history, J->hist.data(), size_t( k ) * SDOT_NB_HIST * 8 );
        out.nb_history = k;
    } else
        out.nb_history = rows;
    CK( cudaStreamSynchronize( c.stream ) );
}

} // namespace sdot

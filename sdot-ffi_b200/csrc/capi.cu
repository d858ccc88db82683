// The extern "C" boundary (include/sdot_b200.h): argument checks, host/device staging, errors -> sdot_status.
#include "engine.h"
#include <algorithm>
#include <cstring>
#include <mutex>

using namespace sdot;

namespace {

void set_status( sdot_status *st, int code, const std::string &msg, long long id = -1, long long needed = 0 ) {
    if ( ! st ) return;
    std::memset( st, 0, sizeof( *st ) );
    st->code = code;
    st->kind = code == SDOT_ERR_CAPACITY || code == SDOT_ERR_TOPOLOGY ? 2 : 0;
    st->id = id;
    st->needed = needed;
    std::strncpy( st->message, msg.c_str(), sizeof( st->message ) - 1 );
}

template<class F>
int32_t guard( sdot_status *st, F &&f ) {
    try {
        f();
        set_status( st, SDOT_OK, "" );
        return SDOT_OK;
    } catch ( const Error &e ) {
        set_status( st, e.code, e.msg, e.id, e.needed );
        return e.code;
    } catch ( const std::exception &e ) {
        set_status( st, SDOT_ERR_ARGS, e.what() );
        return SDOT_ERR_ARGS;
    }
}

// reverse Cuthill-McKee order of a symmetric pattern: perm[ new ] = old.  Consecutive rows are then neighbours, which
// the multigrid's aggregates of consecutive rows need (a caller's CSR comes in any order)
std::vector<int> rcm_order( long n, const std::vector<int> &rp, const std::vector<int> &col ) {
    std::vector<int> perm, deg( n );
    perm.reserve( n );
    for ( long i = 0; i < n; ++i ) deg[ i ] = rp[ i + 1 ] - rp[ i ];
    std::vector<char> seen( n, 0 );
    std::vector<int> by_deg( n );
    for ( long i = 0; i < n; ++i ) by_deg[ i ] = int( i );
    std::stable_sort( by_deg.begin(), by_deg.end(), [&]( int a, int b ) { return deg[ a ] < deg[ b ]; } );
    std::vector<int> nb;
    for ( int start : by_deg ) {
        if ( seen[ start ] ) continue;
        seen[ start ] = 1;
        size_t head = perm.size();
        perm.push_back( start );
        while ( head < perm.size() ) {
            const int i = perm[ head++ ];
            nb.clear();
            for ( int e = rp[ i ]; e < rp[ i + 1 ]; ++e ) {
                const int j = col[ e ];
                if ( j >= 0 && j < n && ! seen[ j ] ) { seen[ j ] = 1; nb.push_back( j ); }
            }
            std::stable_sort( nb.begin(), nb.end(), [&]( int a, int b ) { return deg[ a ] < deg[ b ]; } );
            perm.insert( perm.end(), nb.begin(), nb.end() );
        }
    }
    std::reverse( perm.begin(), perm.end() );
    return perm;
}

struct DevVec {
    Ctx &c;
    void *p = nullptr;
    DevVec( Ctx &c, size_t bytes ) : c( c ) { p = dalloc( c, bytes ); }
    ~DevVec() { if ( p ) cudaFreeAsync( p, c.stream ); }
    template<class T> T *as() { return reinterpret_cast<T *>( p ); }
};

// a user array seen on the device: the pointer itself (SDOT_DEVICE) or a staged copy (SDOT_HOST)
struct InArr {
    const double *d = nullptr;
    DevVec *own = nullptr;
    InArr( Ctx &c, const double *src, size_t count, int memory ) {
        if ( ! src ) return;
        if ( memory == SDOT_DEVICE ) { d = src; return; }
        own = new DevVec( c, count * 8 );
        CK( cudaMemcpyAsync( own->p, src, count * 8, cudaMemcpyHostToDevice, c.stream ) );
        d = own->as<double>();
    }
    ~InArr() { delete own; }
};

// after a standalone diagram: the cells queued as too big for a warp's registers, rebuilt in global memory
void run_big_cells( Ctx &c, ProbDev *dprob, unsigned flags ) {
    CK( cudaMemcpyAsync( c.hovf, &c.dovf->count, sizeof( int ), cudaMemcpyDeviceToHost, c.stream ) );
    CK( cudaStreamSynchronize( c.stream ) );
    const int count = *c.hovf;
    if ( count <= 0 ) return;
    Launch L = c.L();
    c.timer.begin( c.stream, K_CELLS2D, double( count ) );
    launch_cells2d_big( L, dprob, c.dovf, std::min( count, c.ovf_cap ), flags, c.derr, c.big_scratch, c.big_warps );
    launch_cells3d_big( L, dprob, c.dovf, std::min( count, c.ovf_cap ), flags, c.derr, c.dgiant );
    run_giant_cells( c, dprob, flags );
    c.timer.end( c.stream );
    CK( cudaMemsetAsync( &c.dovf->count, 0, sizeof( int ), c.stream ) );
}

} // namespace

extern "C" {

int32_t sdot_abi_version( void ) { return SDOT_ABI_VERSION; }

int32_t sdot_context_create( int32_t device, uint64_t pool_limit, sdot_context *out, sdot_status *st ) {
    if ( ! out ) { set_status( st, SDOT_ERR_ARGS, "out is NULL" ); return SDOT_ERR_ARGS; }
    *out = nullptr;
    auto *ctx = new sdot_context_s;
    int32_t r = guard( st, [&] { ctx_init( ctx->c, device, pool_limit ); } );
    if ( r != SDOT_OK ) { sdot_context_destroy( ctx ); return r; }
    *out = ctx;
    return SDOT_OK;
}

void sdot_context_destroy( sdot_context ctx ) {
    if ( ! ctx ) return;
    ctx_release( ctx->c );
    delete ctx;
}

void *sdot_context_stream( sdot_context ctx ) { return ctx ? ( void * ) ctx->c.stream : nullptr; }

uint64_t sdot_context_kernel_launches( sdot_context ctx ) { return ctx ? ctx->c.launches : 0; }

int32_t sdot_context_memory( sdot_context ctx, uint64_t *in_use, uint64_t *peak, uint64_t *limit, int32_t reset_peak ) {
    if ( ! ctx ) return SDOT_ERR_ARGS;
    std::lock_guard<std::mutex> lock( ctx->mu );
    sdot_status st;
    return guard( &st, [&] {
        Ctx &c = ctx->c;
        CK( cudaSetDevice( c.device ) );
        CK( cudaStreamSynchronize( c.stream ) );
        uint64_t high = 0;
        CK( cudaMemPoolGetAttribute( c.pool, cudaMemPoolAttrUsedMemHigh, &high ) );
        if ( in_use ) *in_use = pool_in_use( c );
        if ( peak ) *peak = uint64_t( high );
        if ( limit ) *limit = c.pool_limit;
        if ( reset_peak ) {
            uint64_t zero = 0;
            CK( cudaMemPoolSetAttribute( c.pool, cudaMemPoolAttrUsedMemHigh, &zero ) );
        }
    } );
}

int32_t sdot_context_set_timing( sdot_context ctx, int32_t on ) {
    if ( ! ctx ) return SDOT_ERR_ARGS;
    ctx->c.timer.on = on != 0;
    return SDOT_OK;
}

int32_t sdot_context_kernel_stats( sdot_context ctx, int32_t kernel_class, double *ms, uint64_t *launches, double *units, int32_t reset ) {
    if ( ! ctx || kernel_class < 0 || kernel_class >= NB_KCLASS ) return SDOT_ERR_ARGS;
    std::lock_guard<std::mutex> lock( ctx->mu );
    sdot_status st;
    return guard( &st, [&] {
        Timer &T = ctx->c.timer;
        CK( cudaSetDevice( ctx->c.device ) );
        T.resolve();
        if ( ms ) *ms = T.ms[ kernel_class ];
        if ( launches ) *launches = T.count[ kernel_class ];
        if ( units ) *units = T.units[ kernel_class ];
        if ( reset ) {
            for ( int k = 0; k < NB_KCLASS; ++k ) { T.ms[ k ] = 0; T.units[ k ] = 0; T.count[ k ] = 0; }
        }
    } );
}

int32_t sdot_context_set_counters( sdot_context ctx, int32_t on ) {
    if ( ! ctx ) return SDOT_ERR_ARGS;
    std::lock_guard<std::mutex> lock( ctx->mu );
    ctx->c.gather_on = on != 0;
    return SDOT_OK;
}

int32_t sdot_context_gather_counters( sdot_context ctx, int32_t dim, uint64_t *counts, int32_t reset ) {
    if ( ! ctx || ! counts || ( dim != 2 && dim != 3 ) ) return SDOT_ERR_ARGS;
    std::lock_guard<std::mutex> lock( ctx->mu );
    sdot_status st;
    return guard( &st, [&] {
        Ctx &c = ctx->c;
        CK( cudaSetDevice( c.device ) );
        unsigned long long h[ NB_GATHER * GATHER_SLOTS ];
        unsigned long long *d = c.dgather + size_t( dim - 2 ) * NB_GATHER * GATHER_SLOTS;
        CK( cudaMemcpyAsync( h, d, sizeof( h ), cudaMemcpyDeviceToHost, c.stream ) );
        CK( cudaStreamSynchronize( c.stream ) );
        counts[ 0 ] = c.gather_cells[ dim - 2 ];
        for ( int k = 0; k < NB_GATHER; ++k ) {
            uint64_t sum = 0;
            for ( int q = 0; q < GATHER_SLOTS; ++q ) sum += h[ k * GATHER_SLOTS + q ];
            counts[ 1 + k ] = sum;
        }
        if ( reset ) {
            CK( cudaMemsetAsync( d, 0, sizeof( h ), c.stream ) );
            CK( cudaStreamSynchronize( c.stream ) );
            c.gather_cells[ dim - 2 ] = 0;
        }
    } );
}

int32_t sdot_context_synchronize( sdot_context ctx, sdot_status *st ) {
    if ( ! ctx ) { set_status( st, SDOT_ERR_ARGS, "null context" ); return SDOT_ERR_ARGS; }
    return guard( st, [&] { CK( cudaSetDevice( ctx->c.device ) ); CK( cudaStreamSynchronize( ctx->c.stream ) ); } );
}

int32_t sdot_cells( sdot_context ctx, const sdot_diagram_desc *desc, sdot_cells_out *out, sdot_status *st ) {
    if ( ! ctx || ! desc || ! out ) { set_status( st, SDOT_ERR_ARGS, "null argument" ); return SDOT_ERR_ARGS; }
    std::lock_guard<std::mutex> lock( ctx->mu );
    return guard( st, [&] {
        Ctx &c = ctx->c;
        CK( cudaSetDevice( c.device ) );
        const int dim = desc->dim;
        const long n = desc->n;
        if ( out->precision != 0 && out->precision != 1 ) throw Error( SDOT_ERR_ARGS, "precision: 0 (FP64 clipping) or 1 (FP32 clipping)" );
        if ( out->precision == 1 && dim != 2 )
            throw Error( SDOT_ERR_UNSUPPORTED, "precision 1 (FP32 clipping with FP64 re-checks) is built in 2D; 3D clips in FP64 (precision 0)" );
        const bool facets = out->nb_count || out->nb_ids || out->nb_coef || out->nb_measure;
        if ( facets && ( ! out->nb_count || ! out->nb_ids || ! out->nb_coef || out->cap <= 0 ) )
            throw Error( SDOT_ERR_ARGS, "facets need nb_count, nb_ids, nb_coef and cap > 0" );
        Geometry G;
        build_geometry( c, G, dim, n, desc->positions, desc->box_lo, desc->box_hi, desc->density, desc->memory );
        struct Free { Ctx &c; Geometry &G; ~Free() { free_geometry( c, G ); } } fg{ c, G };
        const int cap = facets ? out->cap : 1;
        const bool host = desc->memory != SDOT_DEVICE;
        // device outputs (the caller's when on the device)
        size_t bytes = size_t( n ) * 8 * ( 3 + dim ) + size_t( n ) * 4 + ( facets ? size_t( n ) * cap * 20 : 0 ) + 16 * 256;
        DevVec mem( c, bytes );
        Arena A{ ( char * ) mem.p, bytes, 0 };
        double *wr = A.take<double>( n );
        unsigned long long *slot = A.take<unsigned long long>( 1 );
        double *dm = host ? A.take<double>( n ) : out->masses;
        double *db = host ? A.take<double>( size_t( n ) * dim ) : out->barycentres;
        double *dc = host ? A.take<double>( n ) : out->costs;
        int *dnb = nullptr, *dnid = nullptr;
        double *dnc = nullptr, *dnm = nullptr;
        if ( facets ) {
            dnb = host ? A.take<int>( n ) : out->nb_count;
            dnid = host ? A.take<int>( size_t( n ) * cap ) : out->nb_ids;
            dnc = host ? A.take<double>( size_t( n ) * cap ) : out->nb_coef;
            dnm = out->nb_measure ? ( host ? A.take<double>( size_t( n ) * cap ) : out->nb_measure ) : nullptr;
        }
        Launch L = c.L();
        InArr w( c, desc->weights, n, desc->memory );
        launch_gather_vec( L, w.d, G.user, int( n ), wr, w.d ? 1.0 : 0.0 );
        CK( cudaMemsetAsync( slot, 0, 8, c.stream ) );
        launch_wmax( L, wr, int( n ), slot );
        if ( facets ) {       // the unused tail of each row reads as (-1, 0, 0)
            CK( cudaMemsetAsync( dnid, 0xff, size_t( n ) * cap * 4, c.stream ) );
            CK( cudaMemsetAsync( dnc, 0, size_t( n ) * cap * 8, c.stream ) );
            if ( dnm ) CK( cudaMemsetAsync( dnm, 0, size_t( n ) * cap * 8, c.stream ) );
        }
        ProbDev P;
        G.fill( P );
        P.fp32 = out->precision == 1;
        P.cap = cap;
        P.w = wr;
        P.wmax_slot = slot;
        P.mass = out->masses ? dm : nullptr;
        P.first = out->barycentres ? db : nullptr;
        P.cost = out->costs ? dc : nullptr;
        if ( facets ) { P.nb = dnb; P.nid = dnid; P.nc = dnc; P.nm = dnm; }
        unsigned flags = F_MASS | F_USER_ORDER | ( facets ? F_FACETS : 0u ) | ( ( out->barycentres || out->costs ) ? F_MOMENTS : 0u );
        if ( c.gather_on ) {
            P.gather = c.dgather + size_t( dim - 2 ) * NB_GATHER * GATHER_SLOTS;
            flags |= F_GATHER;
            c.gather_cells[ dim - 2 ] += uint64_t( n );
        }
        std::vector<Chunk> ch;
        const int cs = cell_chunk( dim, n );
        for ( int b = 0, k = 0; b < n; b += cs, ++k ) ch.push_back( Chunk{ 0, b, int( std::min<long>( n, b + cs ) ), k } );
        size_t o2 = ( sizeof( ProbDev ) + 255 ) & ~size_t( 255 );
        DevVec dd( c, o2 + ch.size() * sizeof( Chunk ) );
        CK( cudaMemcpyAsync( dd.p, &P, sizeof( P ), cudaMemcpyHostToDevice, c.stream ) );
        CK( cudaMemcpyAsync( ( char * ) dd.p + o2, ch.data(), ch.size() * sizeof( Chunk ), cudaMemcpyHostToDevice, c.stream ) );
        CK( cudaMemsetAsync( &c.dovf->count, 0, sizeof( int ), c.stream ) );
        const Split3 *sp = dim == 3 && P.dkind == D_GAUSS ? split3_for( c, int( ch.size() ), n ) : nullptr;
        c.timer.begin( c.stream, dim == 2 ? K_CELLS2D : K_CELLS3D, double( n ) );
        launch_wpyr( L, dd.as<ProbDev>(), 1 );
        if ( dim == 2 ) launch_cells2d( L, dd.as<ProbDev>(), ( Chunk * ) ( ( char * ) dd.p + o2 ), int( ch.size() ), flags, c.derr, c.dovf,
                                        P.fp32 ? 2 : 1 );
        else launch_cells3d( L, dd.as<ProbDev>(), ( Chunk * ) ( ( char * ) dd.p + o2 ), int( ch.size() ), flags, c.derr, c.dovf, sp );
        c.timer.end( c.stream, sp ? 2 : 1 );
        run_big_cells( c, dd.as<ProbDev>(), flags );
        CK( cudaGetLastError() );
        CK( cudaMemcpyAsync( c.herr, c.derr, sizeof( ErrRec ), cudaMemcpyDeviceToHost, c.stream ) );
        if ( host ) {
            if ( out->masses ) CK( cudaMemcpyAsync( out->masses, dm, n * 8, cudaMemcpyDeviceToHost, c.stream ) );
            if ( out->barycentres ) CK( cudaMemcpyAsync( out->barycentres, db, size_t( n ) * dim * 8, cudaMemcpyDeviceToHost, c.stream ) );
            if ( out->costs ) CK( cudaMemcpyAsync( out->costs, dc, n * 8, cudaMemcpyDeviceToHost, c.stream ) );
            if ( facets ) {
                CK( cudaMemcpyAsync( out->nb_count, dnb, n * 4, cudaMemcpyDeviceToHost, c.stream ) );
                CK( cudaMemcpyAsync( out->nb_ids, dnid, size_t( n ) * cap * 4, cudaMemcpyDeviceToHost, c.stream ) );
                CK( cudaMemcpyAsync( out->nb_coef, dnc, size_t( n ) * cap * 8, cudaMemcpyDeviceToHost, c.stream ) );
                if ( out->nb_measure ) CK( cudaMemcpyAsync( out->nb_measure, dnm, size_t( n ) * cap * 8, cudaMemcpyDeviceToHost, c.stream ) );
            }
        }
        CK( cudaStreamSynchronize( c.stream ) );
        check_errors( c, "sdot_cells" );
    } );
}

// the adjoint of the masses and / or of the first moments: one cell pass in user order
static int32_t cells_vjp( sdot_context ctx, const sdot_diagram_desc *desc, const double *grad_masses, const double *grad_first,
                          double *grad_positions, double *grad_weights, sdot_status *st ) {
    if ( ! ctx || ! desc || ( ! grad_masses && ! grad_first ) ) { set_status( st, SDOT_ERR_ARGS, "null argument" ); return SDOT_ERR_ARGS; }
    std::lock_guard<std::mutex> lock( ctx->mu );
    return guard( st, [&] {
        Ctx &c = ctx->c;
        CK( cudaSetDevice( c.device ) );
        const int dim = desc->dim;
        const long n = desc->n;
        if ( dim != 2 && dim != 3 ) throw Error( SDOT_ERR_ARGS, "dim must be 2 or 3" );
        if ( dim == 3 && desc->density.kind != SDOT_DENSITY_UNIFORM )
            throw Error( SDOT_ERR_UNSUPPORTED, "the adjoint of 3D cells is written for a constant density (as the reference's card)" );
        if ( grad_first && desc->density.kind != SDOT_DENSITY_UNIFORM )
            throw Error( SDOT_ERR_UNSUPPORTED, "the adjoint of the first moments is written for a constant density" );
        Geometry G;
        build_geometry( c, G, dim, n, desc->positions, desc->box_lo, desc->box_hi, desc->density, desc->memory );
        struct Free { Ctx &c; Geometry &G; ~Free() { free_geometry( c, G ); } } fg{ c, G };
        const bool host = desc->memory != SDOT_DEVICE;
        size_t bytes = size_t( n ) * 8 * ( 3 + dim ) + 8 * 256;
        DevVec mem( c, bytes );
        Arena A{ ( char * ) mem.p, bytes, 0 };
        double *wr = A.take<double>( n );
        unsigned long long *slot = A.take<unsigned long long>( 1 );
        double *gp = host ? A.take<double>( size_t( n ) * dim ) : grad_positions;
        double *gw = host ? A.take<double>( n ) : grad_weights;
        Launch L = c.L();
        InArr w( c, desc->weights, n, desc->memory );
        InArr gm( c, grad_masses, n, desc->memory );
        InArr gf( c, grad_first, size_t( n ) * dim, desc->memory );
        launch_gather_vec( L, w.d, G.user, int( n ), wr, w.d ? 1.0 : 0.0 );
        CK( cudaMemsetAsync( slot, 0, 8, c.stream ) );
        launch_wmax( L, wr, int( n ), slot );
        ProbDev P;
        G.fill( P );
        P.fp32 = 0;
        P.w = wr;
        P.wmax_slot = slot;
        P.gm = gm.d;
        P.gf = gf.d;
        P.gpos = grad_positions ? gp : nullptr;
        P.gw = grad_weights ? gw : nullptr;
        std::vector<Chunk> ch;
        const int cs = cell_chunk( dim, n );
        for ( int b = 0, k = 0; b < n; b += cs, ++k ) ch.push_back( Chunk{ 0, b, int( std::min<long>( n, b + cs ) ), k } );
        size_t o2 = ( sizeof( ProbDev ) + 255 ) & ~size_t( 255 );
        DevVec dd( c, o2 + ch.size() * sizeof( Chunk ) );
        CK( cudaMemcpyAsync( dd.p, &P, sizeof( P ), cudaMemcpyHostToDevice, c.stream ) );
        CK( cudaMemcpyAsync( ( char * ) dd.p + o2, ch.data(), ch.size() * sizeof( Chunk ), cudaMemcpyHostToDevice, c.stream ) );
        CK( cudaMemsetAsync( &c.dovf->count, 0, sizeof( int ), c.stream ) );
        launch_wpyr( L, dd.as<ProbDev>(), 1 );
        if ( dim == 2 ) launch_cells2d( L, dd.as<ProbDev>(), ( Chunk * ) ( ( char * ) dd.p + o2 ), int( ch.size() ), F_VJP | F_USER_ORDER, c.derr, c.dovf );
        else launch_cells3d( L, dd.as<ProbDev>(), ( Chunk * ) ( ( char * ) dd.p + o2 ), int( ch.size() ), F_VJP | F_USER_ORDER, c.derr, c.dovf );
        run_big_cells( c, dd.as<ProbDev>(), F_VJP | F_USER_ORDER );
        CK( cudaGetLastError() );
        CK( cudaMemcpyAsync( c.herr, c.derr, sizeof( ErrRec ), cudaMemcpyDeviceToHost, c.stream ) );
        if ( host ) {
            if ( grad_positions ) CK( cudaMemcpyAsync( grad_positions, gp, size_t( n ) * dim * 8, cudaMemcpyDeviceToHost, c.stream ) );
            if ( grad_weights ) CK( cudaMemcpyAsync( grad_weights, gw, n * 8, cudaMemcpyDeviceToHost, c.stream ) );
        }
        CK( cudaStreamSynchronize( c.stream ) );
        check_errors( c, "sdot_cells_vjp" );
    } );
}

int32_t sdot_cells_vjp( sdot_context ctx, const sdot_diagram_desc *desc, const double *grad_masses, double *grad_positions, double *grad_weights,
                        sdot_status *st ) {
    if ( ! grad_masses ) { set_status( st, SDOT_ERR_ARGS, "null argument" ); return SDOT_ERR_ARGS; }
    return cells_vjp( ctx, desc, grad_masses, nullptr, grad_positions, grad_weights, st );
}

int32_t sdot_cells_vjp_moments( sdot_context ctx, const sdot_diagram_desc *desc, const double *grad_masses, const double *grad_first,
                                double *grad_positions, double *grad_weights, sdot_status *st ) {
    return cells_vjp( ctx, desc, grad_masses, grad_first, grad_positions, grad_weights, st );
}

int32_t sdot_laplacian( sdot_context ctx, const sdot_diagram_desc *desc, int64_t cap_nnz, int64_t *row_ptr, int32_t *cols, double *vals, double *dia,
                        int64_t *nnz, sdot_status *st ) {
    if ( ! ctx || ! desc || ! row_ptr || ! dia ) { set_status( st, SDOT_ERR_ARGS, "null argument" ); return SDOT_ERR_ARGS; }
    std::lock_guard<std::mutex> lock( ctx->mu );
    return guard( st, [&] {
        Ctx &c = ctx->c;
        CK( cudaSetDevice( c.device ) );
        const int dim = desc->dim;
        const long n = desc->n;
        Geometry G;
        build_geometry( c, G, dim, n, desc->positions, desc->box_lo, desc->box_hi, desc->density, desc->memory );
        struct Free { Ctx &c; Geometry &G; ~Free() { free_geometry( c, G ); } } fg{ c, G };
        const int cap = dim == 2 ? CAP2 : CAP3;
        const long nch = ( n + vec_chunk( n ) - 1 ) / vec_chunk( n );
        size_t bytes = size_t( n ) * 8 * 3 + size_t( n ) * cap * 12 * 2 + size_t( n + 1 ) * 4 + size_t( n ) * 8 + size_t( nch ) * 32 + NB_SC * 8 +
                       64 + 16 * 256;
        DevVec mem( c, bytes );
        Arena A{ ( char * ) mem.p, bytes, 0 };
        double *wr = A.take<double>( n );
        unsigned long long *slot = A.take<unsigned long long>( 1 );
        int *nb = A.take<int>( n ), *nid = A.take<int>( size_t( n ) * cap ), *rp = A.take<int>( n + 1 ), *col = A.take<int>( size_t( n ) * cap );
        int *rowcnt = A.take<int>( n );
        double *nc = A.take<double>( size_t( n ) * cap ), *val = A.take<double>( size_t( n ) * cap ), *ddia = A.take<double>( n );
        double *part = A.take<double>( size_t( nch ) * 4 ), *sc = A.take<double>( NB_SC );
        unsigned *counter = A.take<unsigned>( 2 );
        // the facets of cells past the table's row (2D): an overflow store
        DevVec ovf( c, ( size_t( n ) + 4096 ) * 12 + 512 );
        Arena B{ ( char * ) ovf.p, ( size_t( n ) + 4096 ) * 12 + 512, 0 };
        int *ovf_count = B.take<int>( 4 ), *ovf_ids = B.take<int>( n + 4096 );
        double *ovf_c = B.take<double>( n + 4096 );
        CK( cudaMemsetAsync( counter, 0, 8, c.stream ) );
        CK( cudaMemsetAsync( ovf_count, 0, 16, c.stream ) );
        Launch L = c.L();
        InArr w( c, desc->weights, n, desc->memory );
        launch_gather_vec( L, w.d, G.user, int( n ), wr, w.d ? 1.0 : 0.0 );
        CK( cudaMemsetAsync( slot, 0, 8, c.stream ) );
        launch_wmax( L, wr, int( n ), slot );
        ProbDev P;
        G.fill( P );
        P.fp32 = 0;
        P.cap = cap;
        P.w = wr;
        P.wmax_slot = slot;
        P.nb = nb; P.nid = nid; P.nc = nc;
        P.ovf_count = ovf_count; P.ovf_cap = int( n ) + 4096; P.ovf_ids = ovf_ids; P.ovf_c = ovf_c;
        std::vector<Chunk> ch;
        const int cs = cell_chunk( dim, n );
        for ( int b = 0, k = 0; b < n; b += cs, ++k ) ch.push_back( Chunk{ 0, b, int( std::min<long>( n, b + cs ) ), k } );
        std::vector<Chunk> vch;
        for ( int b = 0, k = 0; b < n; b += vec_chunk( n ), ++k ) vch.push_back( Chunk{ 0, b, int( std::min<long>( n, b + vec_chunk( n ) ) ), k } );
        VecDev V;
        std::memset( &V, 0, sizeof( V ) );
        V.n = int( n ); V.cap = cap; V.nb = nb; V.nid = nid; V.nc = nc; V.row_ptr = rp; V.col = col; V.val = val; V.dia = ddia; V.rowcnt = rowcnt;
        V.sc = sc; V.partials = part; V.counter = counter; V.nchunk = int( vch.size() ); V.active = 1;
        V.ovf_ids = ovf_ids; V.ovf_c = ovf_c;
        size_t o1 = ( sizeof( ProbDev ) + 255 ) & ~size_t( 255 ), o2 = o1 + ( ( ch.size() * sizeof( Chunk ) + 255 ) & ~size_t( 255 ) ),
               o3 = o2 + ( ( sizeof( VecDev ) + 255 ) & ~size_t( 255 ) );
        DevVec dd( c, o3 + vch.size() * sizeof( Chunk ) );
        char *base = ( char * ) dd.p;
        CK( cudaMemcpyAsync( base, &P, sizeof( P ), cudaMemcpyHostToDevice, c.stream ) );
        CK( cudaMemcpyAsync( base + o1, ch.data(), ch.size() * sizeof( Chunk ), cudaMemcpyHostToDevice, c.stream ) );
        CK( cudaMemcpyAsync( base + o2, &V, sizeof( V ), cudaMemcpyHostToDevice, c.stream ) );
        CK( cudaMemcpyAsync( base + o3, vch.data(), vch.size() * sizeof( Chunk ), cudaMemcpyHostToDevice, c.stream ) );
        // the cells in USER order: the table holds user ids, and the CSR comes out in user order
        CK( cudaMemsetAsync( &c.dovf->count, 0, sizeof( int ), c.stream ) );
        launch_wpyr( L, ( ProbDev * ) base, 1 );
        if ( dim == 2 ) launch_cells2d( L, ( ProbDev * ) base, ( Chunk * ) ( base + o1 ), int( ch.size() ), F_FACETS | F_USER_ORDER, c.derr, c.dovf );
        else
            launch_cells3d( L, ( ProbDev * ) base, ( Chunk * ) ( base + o1 ), int( ch.size() ), F_FACETS | F_USER_ORDER, c.derr, c.dovf,
                            P.dkind == D_GAUSS ? split3_for( c, int( ch.size() ), n ) : nullptr );
        run_big_cells( c, ( ProbDev * ) base, F_FACETS | F_USER_ORDER );
        launch_lap_count( L, ( VecDev * ) ( base + o2 ), ( Chunk * ) ( base + o3 ), int( vch.size() ) );
        launch_lap_scan( L, ( VecDev * ) ( base + o2 ), 1 );
        CK( cudaMemcpyAsync( c.herr, c.derr, sizeof( ErrRec ), cudaMemcpyDeviceToHost, c.stream ) );
        double hs[ NB_SC ];
        CK( cudaMemcpyAsync( hs, sc, sizeof( hs ), cudaMemcpyDeviceToHost, c.stream ) );
        CK( cudaStreamSynchronize( c.stream ) );
        check_errors( c, "sdot_laplacian" );
        const long long total = ( long long ) hs[ SC_NNZ ];
        if ( nnz ) *nnz = total;
        if ( total > cap_nnz ) throw Error( SDOT_ERR_CAPACITY, "sdot_laplacian: cap_nnz too small", -1, total );
        if ( total > ( long long ) n * cap ) throw Error( SDOT_ERR_CAPACITY, "sdot_laplacian: more entries than the CSR work area holds", -1, total );
        launch_lap_fill( L, ( VecDev * ) ( base + o2 ), ( Chunk * ) ( base + o3 ), int( vch.size() ) );
        std::vector<int> hrp( n + 1 );
        CK( cudaMemcpyAsync( hrp.data(), rp, ( n + 1 ) * 4, cudaMemcpyDeviceToHost, c.stream ) );
        auto kind = desc->memory == SDOT_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        if ( total > 0 && cols ) CK( cudaMemcpyAsync( cols, col, total * 4, kind, c.stream ) );
        if ( total > 0 && vals ) CK( cudaMemcpyAsync( vals, val, total * 8, kind, c.stream ) );
        CK( cudaMemcpyAsync( dia, ddia, n * 8, kind, c.stream ) );
        CK( cudaStreamSynchronize( c.stream ) );
        std::vector<int64_t> r64( hrp.begin(), hrp.end() );
        CK( cudaMemcpyAsync( row_ptr, r64.data(), ( n + 1 ) * 8, desc->memory == SDOT_DEVICE ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost,
                             c.stream ) );
        CK( cudaStreamSynchronize( c.stream ) );
    } );
}

int32_t sdot_linear_solve( sdot_context ctx, int64_t n, const int64_t *row_ptr, const int32_t *cols, const double *vals, const double *dia,
                           int32_t nrhs, const double *rhs, double *x, int32_t method, double tol, int32_t maxit, int32_t memory, int32_t *iterations,
                           sdot_status *st ) {
    if ( ! ctx || ! row_ptr || ! dia || ! rhs || ! x || n <= 0 || nrhs <= 0 ) { set_status( st, SDOT_ERR_ARGS, "bad argument" ); return SDOT_ERR_ARGS; }
    std::lock_guard<std::mutex> lock( ctx->mu );
    return guard( st, [&] {
        Ctx &c = ctx->c;
        CK( cudaSetDevice( c.device ) );
        if ( method < 0 || method > 3 )
            throw Error( SDOT_ERR_ARGS, "linear method: 0 (Jacobi-PCG), 1 (multigrid-PCG), 2 / 3 (the same, FP32 CG with FP64 iterative refinement)" );
        const bool mg = method & 1, mixed = method >= 2;
        std::vector<int64_t> hrp;
        if ( memory == SDOT_DEVICE ) {
            hrp.resize( n + 1 );
            CK( cudaMemcpy( hrp.data(), row_ptr, ( n + 1 ) * 8, cudaMemcpyDeviceToHost ) );
        } else
            hrp.assign( row_ptr, row_ptr + n + 1 );
        const long long nnz = hrp[ n ];
        if ( nnz >= ( 1ll << 31 ) ) throw Error( SDOT_ERR_ARGS, "nnz must fit int32" );
        std::vector<int> rp32( hrp.begin(), hrp.end() );
        const long nch = ( n + vec_chunk( n ) - 1 ) / vec_chunk( n );
        size_t bytes = size_t( n + 1 ) * 4 + size_t( nnz + 1 ) * 12 + size_t( n ) * 8 * 9 + size_t( nch ) * 32 + NB_SC * 8 + 64 + 16 * 256;
        if ( mixed ) bytes += size_t( nnz + 1 ) * 4 + size_t( n ) * 4 * 6 + 8 * 256;
        DevVec mem( c, bytes );
        Arena A{ ( char * ) mem.p, bytes, 0 };
        int *rp = A.take<int>( n + 1 ), *col = A.take<int>( nnz + 1 );
        double *val = A.take<double>( nnz + 1 ), *ddia = A.take<double>( n );
        double *xx = A.take<double>( n ), *r = A.take<double>( n ), *z = A.take<double>( n ), *p = A.take<double>( n ), *q = A.take<double>( n );
        double *b = A.take<double>( n ), *d = A.take<double>( n ), *part = A.take<double>( size_t( nch ) * 4 ), *sc = A.take<double>( NB_SC );
        unsigned *counter = A.take<unsigned>( 2 );
        float *m32[ 7 ] = {};
        if ( mixed ) {
            m32[ 0 ] = A.take<float>( nnz + 1 );
            for ( int q = 1; q < 7; ++q ) m32[ q ] = A.take<float>( n );
        }
        CK( cudaMemsetAsync( counter, 0, 8, c.stream ) );
        auto kind = memory == SDOT_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        std::vector<int> perm, iperm;                       // multigrid: the system in reverse Cuthill-McKee order
        if ( mg ) {
            std::vector<int> hcol( nnz );
            std::vector<double> hval( nnz ), hdia( n );
            auto to_host = memory == SDOT_DEVICE ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost;
            if ( nnz ) {
                CK( cudaMemcpy( hcol.data(), cols, nnz * 4, to_host ) );
                CK( cudaMemcpy( hval.data(), vals, nnz * 8, to_host ) );
            }
            CK( cudaMemcpy( hdia.data(), dia, n * 8, to_host ) );
            perm = rcm_order( n, rp32, hcol );
            iperm.assign( n, 0 );
            for ( long k = 0; k < n; ++k ) iperm[ perm[ k ] ] = int( k );
            std::vector<int> prp( n + 1, 0 ), pcol( nnz );
            std::vector<double> pval( nnz ), pdia( n );
            for ( long k = 0; k < n; ++k ) {
                const int i = perm[ k ];
                prp[ k + 1 ] = prp[ k ] + ( rp32[ i + 1 ] - rp32[ i ] );
                pdia[ k ] = hdia[ i ];
                for ( int e = rp32[ i ], f = prp[ k ]; e < rp32[ i + 1 ]; ++e, ++f ) { pcol[ f ] = iperm[ hcol[ e ] ]; pval[ f ] = hval[ e ]; }
            }
            CK( cudaMemcpy( rp, prp.data(), ( n + 1 ) * 4, cudaMemcpyHostToDevice ) );
            if ( nnz ) {
                CK( cudaMemcpy( col, pcol.data(), nnz * 4, cudaMemcpyHostToDevice ) );
                CK( cudaMemcpy( val, pval.data(), nnz * 8, cudaMemcpyHostToDevice ) );
            }
            CK( cudaMemcpy( ddia, pdia.data(), n * 8, cudaMemcpyHostToDevice ) );
        } else {
            CK( cudaMemcpyAsync( rp, rp32.data(), ( n + 1 ) * 4, cudaMemcpyHostToDevice, c.stream ) );
            if ( nnz ) {
                CK( cudaMemcpyAsync( col, cols, nnz * 4, kind, c.stream ) );
                CK( cudaMemcpyAsync( val, vals, nnz * 8, kind, c.stream ) );
            }
            CK( cudaMemcpyAsync( ddia, dia, n * 8, kind, c.stream ) );
        }
        std::vector<Chunk> vch;
        for ( int bb = 0, k = 0; bb < n; bb += vec_chunk( n ), ++k ) vch.push_back( Chunk{ 0, bb, int( std::min<long>( n, bb + vec_chunk( n ) ) ), k } );
        VecDev V;
        std::memset( &V, 0, sizeof( V ) );
        V.n = int( n ); V.row_ptr = rp; V.col = col; V.val = val; V.dia = ddia;
        V.x = xx; V.r = r; V.z = z; V.p = p; V.q = q; V.b = b; V.d = d;
        V.tol = tol > 0 ? tol : 1e-10;
        V.maxit = maxit > 0 ? maxit : 100000;
        V.sc = sc; V.partials = part; V.counter = counter; V.nchunk = int( vch.size() ); V.active = 1;
        V.rank0 = mg ? iperm[ 0 ] : 0;                     // the gauge x[ 0 ] = 0, row 0 wherever it went
        if ( mixed ) {
            V.mixed = 1;
            V.val32 = m32[ 0 ]; V.dia32 = m32[ 1 ]; V.x32 = m32[ 2 ]; V.r32 = m32[ 3 ]; V.z32 = m32[ 4 ]; V.p32 = m32[ 5 ]; V.q32 = m32[ 6 ];
        }
        size_t o1 = ( sizeof( VecDev ) + 255 ) & ~size_t( 255 );
        DevVec dd( c, o1 + vch.size() * sizeof( Chunk ) );
        CK( cudaMemcpyAsync( dd.p, &V, sizeof( V ), cudaMemcpyHostToDevice, c.stream ) );
        CK( cudaMemcpyAsync( ( char * ) dd.p + o1, vch.data(), vch.size() * sizeof( Chunk ), cudaMemcpyHostToDevice, c.stream ) );
        VecDev *dv = dd.as<VecDev>();
        Chunk *dch = ( Chunk * ) ( ( char * ) dd.p + o1 );
        Launch L = c.L();
        std::vector<double> hb( n );
        for ( int k = 0; k < nrhs; ++k ) {
            const double *src = rhs + size_t( k ) * n;
            if ( memory == SDOT_DEVICE ) CK( cudaMemcpy( hb.data(), src, n * 8, cudaMemcpyDeviceToHost ) );
            else std::memcpy( hb.data(), src, n * 8 );
            double mean = 0;
            for ( double v : hb ) mean += v;
            mean /= double( n );
            if ( mg ) {
                std::vector<double> hp( n );
                for ( long q = 0; q < n; ++q ) hp[ q ] = hb[ perm[ q ] ];
                hb.swap( hp );
            }
            CK( cudaMemcpyAsync( b, hb.data(), n * 8, cudaMemcpyHostToDevice, c.stream ) );
            double hsc[ NB_SC ] = {};
            hsc[ SC_MEAN ] = mean;
            CK( cudaMemcpyAsync( sc, hsc, sizeof( hsc ), cudaMemcpyHostToDevice, c.stream ) );
            if ( mg ) {
                const int its = mg_linear_solve( c, V, nnz, hsc );
                if ( iterations ) iterations[ k ] = its;
                std::vector<double> hd( n ), hx( n );
                CK( cudaMemcpyAsync( hd.data(), d, n * 8, cudaMemcpyDeviceToHost, c.stream ) );
                CK( cudaStreamSynchronize( c.stream ) );
                for ( long q = 0; q < n; ++q ) hx[ perm[ q ] ] = hd[ q ];
                CK( cudaMemcpy( x + size_t( k ) * n, hx.data(), n * 8, memory == SDOT_DEVICE ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost ) );
                continue;
            }
            if ( mixed ) launch_mx_init( L, dv, dch, int( vch.size() ) );
            else launch_cg_init( L, dv, dch, int( vch.size() ) );
            for ( ;; ) {
                for ( int s = 0; s < 32; ++s ) {
                    if ( mixed ) launch_mx_iter( L, dv, dch, int( vch.size() ) );
                    else launch_cg_iter( L, dv, dch, int( vch.size() ) );
                }
                CK( cudaMemcpyAsync( hsc, sc, sizeof( hsc ), cudaMemcpyDeviceToHost, c.stream ) );
                CK( cudaStreamSynchronize( c.stream ) );
                if ( hsc[ SC_CONV ] != 0 ) break;
            }
            if ( iterations ) iterations[ k ] = hsc[ SC_FAIL ] != 0 ? -1 : int( hsc[ SC_ITER ] );
            launch_gauge( L, dv, dch, int( vch.size() ) );
            CK( cudaMemcpyAsync( x + size_t( k ) * n, d, n * 8, memory == SDOT_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c.stream ) );
            CK( cudaStreamSynchronize( c.stream ) );
        }
    } );
}

int32_t sdot_solve_batch( sdot_context ctx, int32_t count, const sdot_solve_desc *descs, sdot_solve_out *outs, sdot_status *st ) {
    if ( ! ctx || count <= 0 || ! descs || ! outs ) { set_status( st, SDOT_ERR_ARGS, "bad argument" ); return SDOT_ERR_ARGS; }
    std::lock_guard<std::mutex> lock( ctx->mu );
    Ctx &c = ctx->c;
    std::vector<SolveJob *> jobs( count, nullptr );
    int32_t worst = SDOT_OK;
    for ( int k = 0; k < count; ++k ) {
        int32_t r = guard( st ? st + k : nullptr, [&] {
            CK( cudaSetDevice( c.device ) );
            jobs[ k ] = job_create( c, descs[ k ] );
        } );
        if ( r != SDOT_OK ) worst = r;
    }
    std::vector<SolveJob *> live;
    for ( SolveJob *j : jobs ) if ( j ) live.push_back( j );
    sdot_status batch;
    int32_t r = guard( &batch, [&] { job_run( c, live ); } );
    for ( int k = 0; k < count; ++k ) {
        if ( ! jobs[ k ] ) continue;
        int32_t rk = guard( st ? st + k : nullptr, [&] {
            if ( r != SDOT_OK ) throw Error( r, batch.message, batch.id, batch.needed );
            job_outputs( c, jobs[ k ], outs[ k ], descs[ k ].diagram.memory );
        } );
        if ( rk != SDOT_OK ) worst = rk;
        job_destroy( c, jobs[ k ] );
    }
    return worst;
}

int32_t sdot_w2_backward( sdot_context ctx, int32_t batch, int64_t n, int32_t dim, const void *positions, int32_t positions_fp32,
                          const double *masses, const double *barycentres, const double *weights, const double *grad_cost, void *grad_positions,
                          void *grad_nu, sdot_status *st ) {
    if ( ! ctx || batch <= 0 || n <= 0 || ( dim != 2 && dim != 3 ) || ! positions || ! masses || ! barycentres || ! weights || ! grad_cost ) {
        set_status( st, SDOT_ERR_ARGS, "bad argument" );
        return SDOT_ERR_ARGS;
    }
    std::lock_guard<std::mutex> lock( ctx->mu );
    return guard( st, [&] {
        Ctx &c = ctx->c;
        CK( cudaSetDevice( c.device ) );
        launch_w2_backward( c.L(), batch, int( n ), dim, positions, positions_fp32, masses, barycentres, weights, grad_cost, grad_positions,
                            grad_nu );
        CK( cudaGetLastError() );
    } );
}

int32_t sdot_solve( sdot_context ctx, const sdot_solve_desc *desc, sdot_solve_out *out, sdot_status *st ) {
    return sdot_solve_batch( ctx, 1, desc, out, st );
}

} // extern "C"

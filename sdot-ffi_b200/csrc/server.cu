// Serving: continuous batching of SDOT solves (no counterpart in the reference, which solves one problem per
// FFI call).  A worker thread owns a context and advances every admitted solve by one engine TICK at a time
// (jobs_tick: one batched cell launch, one batched CG burst, one read-back, the decisions).  Between two
// ticks it retires the finished solves and admits waiting ones while the memory budget (sdot_solve_bytes,
// the reference's CardMemory idea, CardMemory.py:1-190) and `max_active` allow, so a request that arrives
// while others run joins them at the next step boundary and its work overlaps theirs on the device.
#include "engine.h"
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>

using namespace sdot;

namespace {

struct Req {
    int64_t ticket = 0;
    sdot_solve_desc desc;
    std::vector<double> pos, w0, nu, dv0, dv1, dv2;   // owned copies of the inputs
    size_t bytes = 0;
    SolveJob *job = nullptr;
    bool done = false;
    sdot_status status;
    std::vector<double> weights, masses, bary, history;
    std::vector<int32_t> clusters;
    double cost = 0;
    double stats[ SDOT_NB_STATS ];
    int nb_history = 0;
};

void set_status( sdot_status *st, int code, const std::string &msg, long long id = -1, long long needed = 0 ) {
    if ( ! st ) return;
    std::memset( st, 0, sizeof( *st ) );
    st->code = code;
    st->kind = code == SDOT_ERR_CAPACITY ? 2 : 0;
    st->id = id;
    st->needed = needed;
    std::strncpy( st->message, msg.c_str(), sizeof( st->message ) - 1 );
}

size_t density_count( const sdot_density &d ) {
    if ( d.kind == SDOT_DENSITY_IMAGE ) return size_t( d.shape[ 0 ] ) * d.shape[ 1 ];
    if ( d.kind == SDOT_DENSITY_GAUSSIANS ) return size_t( d.count );
    return 0;
}

} // namespace

struct sdot_server_s {
    Ctx c;
    sdot_server_config cfg;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req *> queue;
    std::vector<Req *> active;
    std::map<int64_t, Req *> all;
    bool stop = false;
    int64_t next_ticket = 1;
    uint64_t budget = 0, used = 0;
    int64_t counters[ 8 ] = { 0, 0, 0, 0, 0, 0, 0, 0 };
    void run();
};

void sdot_server_s::run() {
    cudaSetDevice( c.device );
    std::vector<SolveJob *> jobs;
    for ( ;; ) {
        std::vector<Req *> admit;
        {
            std::unique_lock<std::mutex> lock( mu );
            if ( active.empty() && queue.empty() ) cv_work.wait( lock, [&] { return stop || ! queue.empty(); } );
            if ( stop ) break;
            while ( ! queue.empty() ) {
                Req *r = queue.front();
                bool fits = used + r->bytes <= budget || active.empty();
                bool room = cfg.max_active <= 0 || int( active.size() + admit.size() ) < cfg.max_active;
                if ( ! fits || ! room ) {
                    if ( ! fits ) ++counters[ 6 ];
                    break;
                }
                queue.pop_front();
                used += r->bytes;
                admit.push_back( r );
            }
        }
        for ( Req *r : admit ) {
            try {
                r->job = job_create( c, r->desc );
                std::lock_guard<std::mutex> lock( mu );
                active.push_back( r );
                ++counters[ 0 ];
            } catch ( const std::exception &e ) {
                // (an Error carries the code; anything else, std::bad_alloc included, is the host running out)
                const Error *E = dynamic_cast<const Error *>( &e );
                std::lock_guard<std::mutex> lock( mu );
                set_status( &r->status, E ? E->code : SDOT_ERR_NO_MEMORY, e.what(), E ? E->id : -1, E ? E->needed : 0 );
                r->done = true;
                used -= r->bytes;
                ++counters[ 1 ];
                cv_done.notify_all();
            }
        }
        {
            std::lock_guard<std::mutex> lock( mu );
            counters[ 2 ] = int64_t( active.size() );
            counters[ 3 ] = std::max<int64_t>( counters[ 3 ], int64_t( active.size() ) );
        }
        if ( active.empty() ) continue;
        jobs.clear();
        for ( Req *r : active ) jobs.push_back( r->job );
        std::string fail;
        int fail_code = 0;
        try {
            jobs_tick( c, jobs );
            ++counters[ 4 ];
        } catch ( const std::exception &e ) {
            const Error *E = dynamic_cast<const Error *>( &e );
            fail = e.what();
            fail_code = E ? E->code : SDOT_ERR_NO_MEMORY;
        }
        std::vector<Req *> keep, finished;
        for ( Req *r : active ) {
            if ( fail_code || job_done( r->job ) ) finished.push_back( r );
            else keep.push_back( r );
        }
        for ( Req *r : finished ) {
            const long n = r->desc.diagram.n;
            const int dim = r->desc.diagram.dim;
            if ( fail_code ) set_status( &r->status, fail_code, fail );
            else {
                try {
                    r->weights.resize( n );
                    r->masses.resize( n );
                    r->bary.resize( size_t( n ) * dim );
                    r->history.resize( size_t( 8 ) * 1024 );
                    r->clusters.resize( n );
                    sdot_solve_out o;
                    std::memset( &o, 0, sizeof( o ) );
                    o.weights = r->weights.data();
                    o.masses = r->masses.data();
                    o.barycentres = r->bary.data();
                    o.cost = &r->cost;
                    o.history = r->history.data();
                    o.cap_history = 1024;
                    o.clusters = r->clusters.data();
                    job_outputs( c, r->job, o, SDOT_HOST );
                    std::memcpy( r->stats, o.stats, sizeof( r->stats ) );
                    r->nb_history = o.nb_history;
                    set_status( &r->status, SDOT_OK, "" );
                } catch ( const std::exception &e ) {
                    const Error *E = dynamic_cast<const Error *>( &e );
                    set_status( &r->status, E ? E->code : SDOT_ERR_NO_MEMORY, e.what(), E ? E->id : -1, E ? E->needed : 0 );
                }
            }
            job_destroy( c, r->job );
            r->job = nullptr;
        }
        std::lock_guard<std::mutex> lock( mu );
        active.swap( keep );
        for ( Req *r : finished ) {
            r->done = true;
            used -= r->bytes;
            ++counters[ 1 ];
        }
        counters[ 5 ] = int64_t( c.launches );
        if ( ! finished.empty() ) cv_done.notify_all();
    }
    for ( Req *r : active ) job_destroy( c, r->job );
    active.clear();
}

extern "C" {

uint64_t sdot_solve_bytes( int32_t dim, int64_t n, const sdot_density *density ) {
    sdot_density d;
    std::memset( &d, 0, sizeof( d ) );
    if ( density ) d = *density;
    return job_bytes( dim, long( n ), d.kind, long( density_count( d ) ) );
}

int32_t sdot_server_create( const sdot_server_config *cfg, sdot_server *out, sdot_status *st ) {
    if ( ! cfg || ! out ) { set_status( st, SDOT_ERR_ARGS, "null argument" ); return SDOT_ERR_ARGS; }
    *out = nullptr;
    auto *srv = new sdot_server_s;
    try {
        ctx_init( srv->c, cfg->device, 0 );
    } catch ( const Error &e ) {
        ctx_release( srv->c );
        delete srv;
        set_status( st, e.code, e.msg );
        return e.code;
    }
    srv->cfg = *cfg;
    size_t fr = 0, tot = 0;
    cudaSetDevice( cfg->device );
    cudaMemGetInfo( &fr, &tot );
    srv->budget = cfg->memory_budget ? cfg->memory_budget : uint64_t( 0.6 * double( fr ) );
    srv->worker = std::thread( [srv] { srv->run(); } );
    *out = srv;
    set_status( st, SDOT_OK, "" );
    return SDOT_OK;
}

int32_t sdot_server_submit( sdot_server srv, const sdot_solve_desc *desc, int64_t *ticket, sdot_status *st ) {
    if ( ! srv || ! desc || ! ticket ) { set_status( st, SDOT_ERR_ARGS, "null argument" ); return SDOT_ERR_ARGS; }
    const sdot_diagram_desc &D = desc->diagram;
    if ( D.memory != SDOT_HOST ) { set_status( st, SDOT_ERR_ARGS, "the server takes host arrays" ); return SDOT_ERR_ARGS; }
    if ( ( D.dim != 2 && D.dim != 3 ) || D.n <= 0 || ! D.positions ) { set_status( st, SDOT_ERR_ARGS, "bad problem" ); return SDOT_ERR_ARGS; }
    Req *r = new Req;
    r->desc = *desc;
    const long n = D.n;
    r->pos.assign( D.positions, D.positions + size_t( n ) * D.dim );
    r->desc.diagram.positions = r->pos.data();
    if ( D.weights ) { r->w0.assign( D.weights, D.weights + n ); r->desc.diagram.weights = r->w0.data(); }
    if ( desc->nu ) { r->nu.assign( desc->nu, desc->nu + n ); r->desc.nu = r->nu.data(); }
    const sdot_density &dd = D.density;
    if ( dd.kind == SDOT_DENSITY_IMAGE ) {
        r->dv0.assign( dd.values, dd.values + size_t( dd.shape[ 0 ] ) * dd.shape[ 1 ] );
        r->desc.diagram.density.values = r->dv0.data();
    } else if ( dd.kind == SDOT_DENSITY_GAUSSIANS ) {
        r->dv0.assign( dd.centres, dd.centres + size_t( dd.count ) * D.dim );
        r->dv1.assign( dd.sigmas, dd.sigmas + dd.count );
        r->dv2.assign( dd.masses, dd.masses + dd.count );
        r->desc.diagram.density.centres = r->dv0.data();
        r->desc.diagram.density.sigmas = r->dv1.data();
        r->desc.diagram.density.masses = r->dv2.data();
    }
    r->bytes = sdot_solve_bytes( D.dim, n, &dd );
    if ( desc->options[ SDOT_OPT_LIN_PRECISION ] == 1 )      // the FP32 copies of the mixed CG
        r->bytes += uint64_t( n ) * ( ( D.dim == 2 ? CAP2 : CAP3 ) * 4 + 24 ) + 4096;
    {
        std::lock_guard<std::mutex> lock( srv->mu );
        r->ticket = srv->next_ticket++;
        srv->all[ r->ticket ] = r;
        srv->queue.push_back( r );
    }
    srv->cv_work.notify_one();
    *ticket = r->ticket;
    set_status( st, SDOT_OK, "" );
    return SDOT_OK;
}

int32_t sdot_server_poll( sdot_server srv, int64_t ticket, sdot_solve_out *out, int32_t wait_ms, sdot_status *st ) {
    if ( ! srv ) { set_status( st, SDOT_ERR_ARGS, "null server" ); return -SDOT_ERR_ARGS; }
    std::unique_lock<std::mutex> lock( srv->mu );
    auto it = srv->all.find( ticket );
    if ( it == srv->all.end() ) { set_status( st, SDOT_ERR_ARGS, "unknown ticket" ); return -SDOT_ERR_ARGS; }
    Req *r = it->second;
    if ( ! r->done ) {
        if ( wait_ms < 0 ) srv->cv_done.wait( lock, [&] { return r->done; } );
        else if ( wait_ms > 0 ) srv->cv_done.wait_for( lock, std::chrono::milliseconds( wait_ms ), [&] { return r->done; } );
        if ( ! r->done ) { set_status( st, SDOT_OK, "" ); return 0; }
    }
    if ( st ) *st = r->status;
    if ( out && r->status.code == SDOT_OK ) {
        const long n = r->desc.diagram.n;
        const int dim = r->desc.diagram.dim;
        if ( out->weights ) std::memcpy( out->weights, r->weights.data(), n * 8 );
        if ( out->masses ) std::memcpy( out->masses, r->masses.data(), n * 8 );
        if ( out->barycentres ) std::memcpy( out->barycentres, r->bary.data(), size_t( n ) * dim * 8 );
        if ( out->cost ) *out->cost = r->cost;
        if ( out->clusters ) std::memcpy( out->clusters, r->clusters.data(), n * sizeof( int32_t ) );
        std::memcpy( out->stats, r->stats, sizeof( out->stats ) );
        int k = std::min( r->nb_history, out->cap_history );
        if ( out->history && k > 0 ) std::memcpy( out->history, r->history.data(), size_t( k ) * 8 * 8 );
        out->nb_history = out->history ? k : r->nb_history;
    }
    srv->all.erase( it );
    delete r;
    return 1;
}

int32_t sdot_server_counters( sdot_server srv, int64_t counters[ 8 ] ) {
    if ( ! srv || ! counters ) return SDOT_ERR_ARGS;
    std::lock_guard<std::mutex> lock( srv->mu );
    for ( int k = 0; k < 8; ++k ) counters[ k ] = srv->counters[ k ];
    return SDOT_OK;
}

void sdot_server_destroy( sdot_server srv ) {
    if ( ! srv ) return;
    {
        std::lock_guard<std::mutex> lock( srv->mu );
        srv->stop = true;
    }
    srv->cv_work.notify_all();
    if ( srv->worker.joinable() ) srv->worker.join();
    for ( auto &kv : srv->all ) delete kv.second;
    ctx_release( srv->c );
    delete srv;
}

} // extern "C"

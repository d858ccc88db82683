// Host side of the B200 SDOT core: the context, a problem's device geometry, and the batched Newton engine.
#pragma once
#include "internal.h"
#include "../../include/sdot_b200.h"
#include <exception>
#include <mutex>
#include <string>
#include <vector>

namespace sdot {

struct Error : std::exception {
    int code;
    std::string msg;
    long long id = -1, needed = 0;
    Error( int c, std::string m, long long i = -1, long long nd = 0 ) : code( c ), msg( std::move( m ) ), id( i ), needed( nd ) {}
    const char *what() const noexcept override { return msg.c_str(); }
};

void check_cuda( cudaError_t e, const char *what );
#define CK( x ) ::sdot::check_cuda( ( x ), #x )

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr;
    uint64_t pool_limit = 0;          // bytes the pool may hand out at once (0: no limit but the device's)
    unsigned long long launches = 0;
    // engine-wide per-slot scalars: [slot][ 2 * NB_REPORT + NB_SC ] doubles, and two counters per slot
    int max_slots = 0;
    double *dscal = nullptr;
    double *hscal = nullptr;          // pinned mirror
    unsigned *dcount = nullptr;       // [slot][4]
    std::vector<int> free_slots;
    ErrRec *derr = nullptr;
    ErrRec *herr = nullptr;           // pinned
    // the queue of big cells (device) and its count's host mirror; the global-memory polygons of the big-cell pass
    OvfList *dovf = nullptr;
    int *hovf = nullptr;
    char *big_scratch = nullptr;
    int big_warps = 256;
    int ovf_cap = 1 << 18;
    // 3D cells past the big pass: their queue, its count's host mirror, and the warps' cells (allocated at first use)
    OvfList *dgiant = nullptr;
    int *hgiant = nullptr;
    char *giant_scratch = nullptr;
    int giant_slots = 16;
    int giant_cap = 1 << 14;
    // descriptor upload area, and the pinned staging ring its uploads go through (refilled from the start after each
    // tick's read-back, when every earlier copy has completed)
    char *desc = nullptr;
    size_t desc_bytes = 0;
    char *hstage = nullptr;
    size_t hstage_bytes = 0, hstage_used = 0;
    std::vector<void *> desc_spill;   // descriptor blocks past the area, freed at the end of the tick
    // CUDA graphs of the CG bursts, keyed by the layout of the batch they were captured for
    struct BurstGraph {
        std::vector<long long> key;
        cudaGraphExec_t exec = nullptr;
        unsigned long long launches = 0;
    };
    std::vector<BurstGraph> graphs;
    // the two passes of the gaussian 3D cells: their records and per-cell slots (grown on demand, see `split3_for`)
    Split3 split{};
    size_t split_slots = 0;
    Timer timer;
    // the search's read counters of the standalone diagrams (sdot_cells) of dims 2 and 3, on request: [2][NB_GATHER][32]
    // on the device, and the cells those diagrams built
    unsigned long long *dgather = nullptr;
    bool gather_on = false;
    uint64_t gather_cells[ 2 ] = { 0, 0 };
    Launch L() { return Launch{ stream, &launches, &timer }; }
};
constexpr size_t GATHER_BYTES = size_t( 2 ) * NB_GATHER * GATHER_SLOTS * sizeof( unsigned long long );
constexpr int SLOT_ERR = 2 * NB_REPORT + NB_SC;                 // a problem's capacity-failure flag
constexpr int SLOT_AGG = SLOT_ERR + 1;                           // the near-coincident pairs its last Laplacian showed
constexpr int SLOT_LIM = SLOT_AGG + 1;                           // the limits step: cells below the floor, smallest limit
constexpr int SLOT_REFUSE = SLOT_LIM + 2;                        // a trial diagram with a cell past the big-cell pass
constexpr int SLOT_DOUBLES = 2 * NB_REPORT + NB_SC + 5;

void ctx_init( Ctx &c, int device, uint64_t pool_limit );   // throws Error
void ctx_release( Ctx &c );
// after a big-cell pass that queued 3D cells on `dgiant`: the giant-cell pass over them (synchronises); their number
int run_giant_cells( Ctx &c, const ProbDev *dprob, unsigned flags );
// the scratch of the two-pass gaussian 3D cells for a launch of `nchunks` chunks that holds `gcells` cells of gaussian
// problems: NULL when there are none, or when the pool cannot give it (the kernel then takes one pass)
const Split3 *split3_for( Ctx &c, int nchunks, long gcells );
void *dalloc( Ctx &c, size_t bytes );
uint64_t pool_in_use( Ctx &c );
void dfree( Ctx &c, void *p );

// a bump allocator over one device allocation
struct Arena {
    char *base = nullptr;
    size_t size = 0, off = 0;
    template<class T> T *take( size_t count ) {
        off = ( off + 255 ) & ~size_t( 255 );
        T *p = reinterpret_cast<T *>( base + off );
        off += count * sizeof( T );
        return p;
    }
};

// the seeds of one problem, ranked on the device, with their grid and density
struct Geometry {
    int dim = 2, n = 0;
    double lo[ 3 ] = { 0, 0, 0 }, hi[ 3 ] = { 1, 1, 1 };
    int g[ 3 ] = { 1, 1, 1 };
    double go[ 3 ] = { 0, 0, 0 }, gh[ 3 ] = { 1, 1, 1 }, ghmin = 1;
    long ncell = 0;
    double *pos = nullptr;            // ranked
    int *user = nullptr, *rank_of = nullptr;
    int2 *cell_range = nullptr;
    double *wpyr = nullptr;           // the weight majorants (rebuilt before each diagram) and their moments
    double *wmom = nullptr;
    int nlev = 0;
    int poff[ MAX_LEV ] = {};
    int dkind = D_UNIFORM;
    double rho = 1;
    double *dval = nullptr, *dpre = nullptr;
    double *dorig = nullptr, *dtmp = nullptr, *dker = nullptr;   // image: the values as given, a pass's output, the taps
    int dn[ 3 ] = { 0, 0, 0 };
    double dorg[ 3 ] = { 0, 0, 0 }, dstep[ 3 ] = { 0, 0, 0 };
    std::vector<double> gauss;        // [ng, dim + 2] as given (continuation widens it)
    std::vector<double> pos_host;     // user order (similarity start)
    char *mem = nullptr;
    void fill( ProbDev &P ) const;
};

// builds the geometry (copies `positions` / density arrays from where `memory` says)
void build_geometry( Ctx &c, Geometry &G, int dim, long n, const double *positions, const double box_lo[ 3 ], const double box_hi[ 3 ],
                     const sdot_density &dens, int memory );
void free_geometry( Ctx &c, Geometry &G );

int take_slot( Ctx &c );
void give_slot( Ctx &c, int s );

void check_errors( Ctx &c, const char *where );

// the batched Newton engine: advances `solves` together until all are done
struct SolveJob;
SolveJob *job_create( Ctx &c, const sdot_solve_desc &desc );
void job_run( Ctx &c, std::vector<SolveJob *> &jobs, int max_ticks = -1 );
bool job_done( const SolveJob *j );
void job_outputs( Ctx &c, SolveJob *j, sdot_solve_out &out, int memory );
void job_destroy( Ctx &c, SolveJob *j );
size_t job_bytes( int dim, long n, int dkind, long dcount );
void launch_w2_backward( const Launch &L, int batch, int n, int dim, const void *pos, int fp32, const double *mass, const double *bary,
                         const double *w, const double *gcost, void *gpos, void *gnu );
struct Engine;
// continuous batching: one step of every active job (used by the server)
void jobs_tick( Ctx &c, std::vector<SolveJob *> &jobs );
// one Laplacian (device CSR in V, b and SC_MEAN uploaded) solved by the multigrid-preconditioned CG: iterations, -1 on failure
int mg_linear_solve( Ctx &c, const VecDev &V, long nnz, double *hsc );

} // namespace sdot

// the object behind `sdot_context`: the device state and the mutex that serialises the calls made through it
struct sdot_context_s {
    sdot::Ctx c;
    std::mutex mu;
};

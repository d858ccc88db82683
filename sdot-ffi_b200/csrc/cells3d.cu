// 3D Laguerre cells: ONE WARP PER CELL, the polyhedron in the warp's slice of shared memory.
//
// The cell is kept as its dual: every vertex is a triple of plane ids (a, b, c) -- the three faces meeting there,
// ordered so that the triples form a consistently oriented triangulation of the sphere -- and its position is
// ALWAYS re-solved from those three planes (solve3: FP64, seed frame), so no error accumulates along the
// cuts (the reference re-solves its float vertices for the same reason, gpu/Cell3D.cuh:1093-1147).  A cut by the
// plane P: lanes mark the vertices outside; for each directed edge (e0, e1) of a removed vertex whose twin (e1, e0)
// belongs to a kept vertex, the new vertex (e0, e1, P) is created; kept vertices are compacted in order and the
// new ones appended.  This is the dual-triangulation clipping published by Ray, Sokolov, Lefebvre and Levy
// ("Meshless Voronoi on the GPU", ACM TOG 2018), written here for a warp.
//
// Candidates: the Morton grid, shell by shell around the seed's grid cell, 32 at a time, each candidate pre-tested
// by one lane against every vertex; the walk stops by the same security radius as in 2D.  Integration: signed
// tetrahedra (seed, point of face f, K, T) for every vertex K and directed edge (f, b) of K, T the vertex across
// that edge -- exact for volume, first and second moments; per-face areas summed in plane order (deterministic).
// Sums of gaussians: face integrals only, by Gauss's theorem (integrate_gauss3).
#include "internal.h"

namespace sdot {

constexpr unsigned FULL3 = 0xffffffffu;
constexpr int W3 = 4;            // warps per block (main kernel)

// the cell of one warp: VC vertices, PC planes, I the type of a vertex / plane index
template<int VC_, int PC_, class I_>
struct Cell3T {
    static constexpr int VC = VC_, PC = PC_;
    typedef I_ I;
    static constexpr int NONE = int( I_( ~I_( 0 ) ) );   // "no vertex" / "no new vertex"
    double vx[ VC ], vy[ VC ], vz[ VC ];
    double area[ 3 * VC ];                       // per (vertex, edge): the face-triangle contribution (integration)
    double nx[ PC ], ny[ PC ], nz[ PC ], no[ PC ];
    int pid[ PC ];
    I va[ VC ], vb[ VC ], vc[ VC ];
    // the ADJACENCY: ad[ q ][ k ] is the vertex across edge q of vertex k (edge 0 = (va, vb), 1 = (vb, vc), 2 = (vc, va)),
    // the one holding the reversed directed edge; kept through every cut, so that no cut and no integration searches
    I ad[ 3 ][ VC ];
    unsigned char out[ VC ];
    I nt[ VC ][ 3 ];                             // new triples of a cut; gaussians: the next entry of each face's list
    I nk[ VC ];                                  // a cut: the kept vertex across each new vertex's first edge
    I nidx[ VC ];                                // a cut: the index of each kept vertex after the compaction
    I e0t[ PC ], e1t[ PC ];                      // a cut: the new vertex whose first (second) plane is this one; NONE between cuts
    double fmp[ PC ];                            // gaussians: the winding-angle part of each face's integral
    double par[ PC ];                            // each face's integral (facets pass)
    unsigned char used[ PC ];                    // plane compaction
    I remap[ PC ];
    double L;                                    // the farthest corner of the box from the seed (the tie band)
    int nv, np;
};
using Cell3 = Cell3T<128, 96, unsigned char>;            // the main kernel, in shared memory
using Cell3B = Cell3T<1024, 256, unsigned short>;        // the big-cell pass: one warp a block, about 90 KB
using Cell3G = Cell3T<32768, 8192, unsigned short>;      // the giant-cell pass (the reference's card_max_vertices, PowerDiagram_Bsp.py:122): one warp a block, about 2.8 MB in global memory

// the vertex of planes a, b, c (n . y = o, seed frame), found on the line of the two most transverse of them: from the
// line's point nearest the seed, by the step the third plane's equation asks for.  The vertex then lies on all three
// planes to rounding, however close to parallel the third plane is to one of the others (two seeds 1e-10 apart make two
// bisectors 1e-9 rad apart; Cramer's rule left such vertices off the planes by eps / sin(angle), and the polyhedron
// lost up to 1e-4 of its volume)
template<class C3>
__device__ __forceinline__ void solve3( const C3 &C, int a, int b, int c, double &x, double &y, double &z ) {
    auto cross2 = [&]( int p, int q ) {          // |n_p x n_q|^2
        const double cx = C.ny[ p ] * C.nz[ q ] - C.nz[ p ] * C.ny[ q ], cy = C.nz[ p ] * C.nx[ q ] - C.nx[ p ] * C.nz[ q ],
                     cz = C.nx[ p ] * C.ny[ q ] - C.ny[ p ] * C.nx[ q ];
        return cx * cx + cy * cy + cz * cz;
    };
    auto norm2 = [&]( int p ) { return C.nx[ p ] * C.nx[ p ] + C.ny[ p ] * C.ny[ p ] + C.nz[ p ] * C.nz[ p ]; };
    // the line: the pair with the largest angle (sin^2 = |n_p x n_q|^2 / |n_p|^2 |n_q|^2, compared times the product of
    // the three |n|^2); the plane: the third one
    const double na = norm2( a ), nb = norm2( b ), nc = norm2( c );
    const double sab = cross2( a, b ) * nc, sbc = cross2( b, c ) * na, sca = cross2( c, a ) * nb;
    int p = a, q = b, r = c;
    double pn2 = na, qn2 = nb;
    if ( sbc > sab && sbc >= sca ) { p = b; q = c; r = a; pn2 = nb; qn2 = nc; }
    else if ( sca > sab && sca > sbc ) { p = c; q = a; r = b; pn2 = nc; qn2 = na; }
    const double pq = C.nx[ p ] * C.nx[ q ] + C.ny[ p ] * C.ny[ q ] + C.nz[ p ] * C.nz[ q ];
    const double dx = C.ny[ p ] * C.nz[ q ] - C.nz[ p ] * C.ny[ q ], dy = C.nz[ p ] * C.nx[ q ] - C.nx[ p ] * C.nz[ q ],
                 dz = C.nx[ p ] * C.ny[ q ] - C.ny[ p ] * C.nx[ q ];
    const double G = pn2 * qn2 - pq * pq;                                    // |d|^2
    const double al = ( C.no[ p ] * qn2 - C.no[ q ] * pq ) / G, be = ( C.no[ q ] * pn2 - C.no[ p ] * pq ) / G;
    const double X0 = al * C.nx[ p ] + be * C.nx[ q ], Y0 = al * C.ny[ p ] + be * C.ny[ q ], Z0 = al * C.nz[ p ] + be * C.nz[ q ];
    const double t = ( C.no[ r ] - ( C.nx[ r ] * X0 + C.ny[ r ] * Y0 + C.nz[ r ] * Z0 ) ) / ( C.nx[ r ] * dx + C.ny[ r ] * dy + C.nz[ r ] * dz );
    x = X0 + t * dx;
    y = Y0 + t * dy;
    z = Z0 + t * dz;
}

// THE TIES: how far beyond the plane n . y = off a vertex must lie to count as outside -- what the rounding of
// n . v - off can reach for a vertex of the cell (|v| <= L, off computed from |n|^2 and the weights), 32 doubles' eps.
// A plane through vertices that lie on it in exact arithmetic (a grid: the bisector of a diagonal neighbour passes
// through an edge of the box cell) then leaves them inside, instead of cutting them off at the noise and making new
// vertices from three planes through one line.  The cell moves by tol / |n| at most.
__device__ __forceinline__ double tie_tol3( double nx, double ny, double nz, double off, double L ) {
    const double n = sqrt( nx * nx + ny * ny + nz * nz );
    return 32 * 2.220446049250313e-16 * ( n * ( n + L ) + fabs( off ) );
}

// the vertex holding the directed edge (e0, e1), -1 if none
template<class C3>
__device__ __forceinline__ int twin_of( const C3 &C, int e0, int e1 ) {
    for ( int t = 0; t < C.nv; ++t ) {
        int a = C.va[ t ], b = C.vb[ t ], c = C.vc[ t ];
        if ( ( a == e0 && b == e1 ) || ( b == e0 && c == e1 ) || ( c == e0 && a == e1 ) ) return t;
    }
    return -1;
}

// the adjacency of every vertex by search (the box, a loaded record, a cut whose boundary is not one cycle)
template<class C3>
__device__ void rebuild_adj( C3 &C, int lane ) {
    typedef typename C3::I I;
    for ( int k = lane; k < C.nv; k += 32 ) {
        const int e[ 3 ] = { C.va[ k ], C.vb[ k ], C.vc[ k ] };
        for ( int q = 0; q < 3; ++q ) {
            const int t = twin_of( C, e[ ( q + 1 ) % 3 ], e[ q ] );
            C.ad[ q ][ k ] = t < 0 ? I( C3::NONE ) : I( t );
        }
    }
    __syncwarp();
}

template<class C3>
__device__ void init_box3( C3 &C, int lane, const double *lo, const double *hi, double px, double py, double pz ) {
    // planes: 0 -x, 1 +x, 2 -y, 3 +y, 4 -z, 5 +z ; ids -1 .. -6
    if ( lane < 6 ) {
        int ax = lane >> 1, sg = lane & 1;
        double p = ax == 0 ? px : ( ax == 1 ? py : pz );
        C.nx[ lane ] = ax == 0 ? ( sg ? 1.0 : -1.0 ) : 0.0;
        C.ny[ lane ] = ax == 1 ? ( sg ? 1.0 : -1.0 ) : 0.0;
        C.nz[ lane ] = ax == 2 ? ( sg ? 1.0 : -1.0 ) : 0.0;
        C.no[ lane ] = sg ? hi[ ax ] - p : p - lo[ ax ];
        C.pid[ lane ] = -1 - lane;
    }
    if ( lane < 8 ) {
        int sx = lane & 1, sy = ( lane >> 1 ) & 1, sz = ( lane >> 2 ) & 1;
        int a = sx, b = 2 + sy, c = 4 + sz;
        // orientation: det( n_a, n_b, n_c ) > 0 ; det( +-x, +-y, +-z ) = sx' sy' sz'
        int s = ( sx ? 1 : -1 ) * ( sy ? 1 : -1 ) * ( sz ? 1 : -1 );
        if ( s < 0 ) { int t = b; b = c; c = t; }
        C.va[ lane ] = a; C.vb[ lane ] = b; C.vc[ lane ] = c;
        C.vx[ lane ] = ( sx ? hi[ 0 ] : lo[ 0 ] ) - px;
        C.vy[ lane ] = ( sy ? hi[ 1 ] : lo[ 1 ] ) - py;
        C.vz[ lane ] = ( sz ? hi[ 2 ] : lo[ 2 ] ) - pz;
    }
    if ( lane == 0 ) {
        C.nv = 8; C.np = 6;
        const double ex = fmax( hi[ 0 ] - px, px - lo[ 0 ] ), ey = fmax( hi[ 1 ] - py, py - lo[ 1 ] ), ez = fmax( hi[ 2 ] - pz, pz - lo[ 2 ] );
        C.L = sqrt( ex * ex + ey * ey + ez * ez );
    }
    for ( int p = lane; p < C3::PC; p += 32 ) { C.e0t[ p ] = typename C3::I( C3::NONE ); C.e1t[ p ] = typename C3::I( C3::NONE ); }
    __syncwarp();
    rebuild_adj( C, lane );
}

// drops the planes no vertex uses (when the plane table is full); false if it cannot make room
template<class C3>
__device__ bool compact_planes( C3 &C, int lane ) {
    constexpr int PC = C3::PC;
    unsigned char *used = C.used;
    for ( int p = lane; p < PC; p += 32 ) used[ p ] = 0;
    __syncwarp();
    for ( int k = lane; k < C.nv; k += 32 ) { used[ C.va[ k ] ] = 1; used[ C.vb[ k ] ] = 1; used[ C.vc[ k ] ] = 1; }
    __syncwarp();
    // new index of each used plane: a serial prefix by lane 0 (rare path)
    typename C3::I *remap = C.remap;
    if ( lane == 0 ) {
        int q = 0;
        for ( int p = 0; p < C.np; ++p ) {
            if ( ! used[ p ] ) continue;
            remap[ p ] = ( typename C3::I ) q;
            C.nx[ q ] = C.nx[ p ]; C.ny[ q ] = C.ny[ p ]; C.nz[ q ] = C.nz[ p ]; C.no[ q ] = C.no[ p ]; C.pid[ q ] = C.pid[ p ];
            ++q;
        }
        C.np = q;
    }
    __syncwarp();
    for ( int k = lane; k < C.nv; k += 32 ) { C.va[ k ] = remap[ C.va[ k ] ]; C.vb[ k ] = remap[ C.vb[ k ] ]; C.vc[ k ] = remap[ C.vc[ k ] ]; }
    __syncwarp();
    return C.np < PC;
}

// keep n . y <= off (a vertex within the tie band of the plane stays); false past a capacity
template<class C3>
__device__ bool wclip3( C3 &C, int lane, double nx, double ny, double nz, double off, int id ) {
    const int nv = C.nv;
    const double tol = tie_tol3( nx, ny, nz, off, C.L );
    int nout = 0;
    for ( int base = 0; base < nv; base += 32 ) {
        int k = base + lane;
        bool o = k < nv && nx * C.vx[ k ] + ny * C.vy[ k ] + nz * C.vz[ k ] - off > tol;
        if ( k < nv ) C.out[ k ] = o;
        nout += __popc( __ballot_sync( FULL3, o ) );
    }
    __syncwarp();
    if ( nout == 0 ) return true;
    if ( nout == nv ) {
        if ( lane == 0 ) C.nv = 0;
        __syncwarp();
        return true;
    }
    constexpr int VC = C3::VC, PC = C3::PC;
    typedef typename C3::I I;
    const bool full = C.np >= PC;
    __syncwarp();
    if ( full && ! compact_planes( C, lane ) ) return false;
    const int P = C.np;
    __syncwarp();
    if ( lane == 0 ) { C.nx[ P ] = nx; C.ny[ P ] = ny; C.nz[ P ] = nz; C.no[ P ] = off; C.pid[ P ] = id; C.np = P + 1; }
    __syncwarp();
    // the boundary edges: directed edges of removed vertices whose twin (`ad`) is kept.  Each new vertex (e0, e1, P) is
    // re-solved from its three planes; where that lands off the edge it replaces (three planes nearly through one
    // line: a cut that grazes the edge), it is taken on the edge instead, from its kept end, where n . y = off.  Its
    // position waits in `area` (free until the integration) while the kept vertices are compacted; the new vertex whose
    // first (second) plane is p is recorded in e0t[ p ] (e1t[ p ]), which links the new vertices around the new face.
    int nnew = 0;
    for ( int base = 0; base < nv; base += 32 ) {
        int k = base + lane;
        I tr[ 3 ][ 2 ];
        int tt[ 3 ];
        int cnt = 0;
        if ( k < nv && C.out[ k ] ) {
            int e[ 3 ] = { C.va[ k ], C.vb[ k ], C.vc[ k ] };
            for ( int q = 0; q < 3; ++q ) {
                const int t = C.ad[ q ][ k ];
                if ( t != C3::NONE && ! C.out[ t ] ) { tr[ cnt ][ 0 ] = I( e[ q ] ); tr[ cnt ][ 1 ] = I( e[ ( q + 1 ) % 3 ] ); tt[ cnt ] = t; ++cnt; }
            }
        }
        int inc = cnt;
#pragma unroll
        for ( int o = 1; o < 32; o <<= 1 ) { int t = __shfl_up_sync( FULL3, inc, o ); if ( lane >= o ) inc += t; }
        int total = __shfl_sync( FULL3, inc, 31 );
        int at = nnew + inc - cnt;
        for ( int q = 0; q < cnt; ++q ) {
            const int j = at + q;
            if ( j >= VC ) continue;
            C.nt[ j ][ 0 ] = tr[ q ][ 0 ]; C.nt[ j ][ 1 ] = tr[ q ][ 1 ]; C.nt[ j ][ 2 ] = I( P );
            const int t = tt[ q ];
            C.nk[ j ] = I( t );
            C.e0t[ tr[ q ][ 0 ] ] = I( j );
            C.e1t[ tr[ q ][ 1 ] ] = I( j );
            const double Rx = C.vx[ k ], Ry = C.vy[ k ], Rz = C.vz[ k ], Tx = C.vx[ t ], Ty = C.vy[ t ], Tz = C.vz[ t ];
            double x, y, z;
            solve3( C, tr[ q ][ 0 ], tr[ q ][ 1 ], P, x, y, z );
            const double ex = Rx - Tx, ey = Ry - Ty, ez = Rz - Tz, e2 = ex * ex + ey * ey + ez * ez;
            const double un = ( x - Tx ) * ex + ( y - Ty ) * ey + ( z - Tz ) * ez;     // u e2, u the edge parameter (NaN: no solve)
            if ( ! ( un >= -1e-9 * e2 && un <= ( 1 + 1e-9 ) * e2 ) ) {
                const double dT = nx * Tx + ny * Ty + nz * Tz - off, dR = nx * Rx + ny * Ry + nz * Rz - off;   // dR > tol >= dT
                const double s = fmin( 1.0, fmax( 0.0, -dT / ( dR - dT ) ) );
                x = Tx + s * ex; y = Ty + s * ey; z = Tz + s * ez;
            }
            C.area[ j ] = x; C.area[ VC + j ] = y; C.area[ 2 * VC + j ] = z;
        }
        nnew += total;
    }
    __syncwarp();
    const int nkeep = nv - nout;
    const bool room = ! ( nkeep + nnew > VC || nnew >= VC );
    // the new vertices make one cycle around the new face when every plane of the boundary is the first plane of exactly
    // one new vertex and the second plane of exactly one; otherwise (a removed region that is not a disc, at the limits of
    // rounding) the adjacency is searched again after the cut
    bool cyc = true;
    for ( int j = lane; j < nnew && room; j += 32 )
        cyc = cyc && C.e0t[ C.nt[ j ][ 0 ] ] == j && C.e1t[ C.nt[ j ][ 1 ] ] == j && C.e0t[ C.nt[ j ][ 1 ] ] != C3::NONE &&
              C.e1t[ C.nt[ j ][ 0 ] ] != C3::NONE;
    cyc = __all_sync( FULL3, cyc );
    if ( ! room ) {
        for ( int j = lane; j < nnew && j < VC; j += 32 ) { C.e0t[ C.nt[ j ][ 0 ] ] = I( C3::NONE ); C.e1t[ C.nt[ j ][ 1 ] ] = I( C3::NONE ); }
        __syncwarp();
        return false;
    }
    // compaction of the kept vertices, in order (destinations never pass their sources): first their new indices, then
    // the moves, their adjacency mapped to those indices (an edge to a removed vertex gets its new vertex below)
    int kept_before = 0;
    for ( int base = 0; base < nv; base += 32 ) {
        int k = base + lane;
        bool keep = k < nv && ! C.out[ k ];
        unsigned m = __ballot_sync( FULL3, keep );
        if ( keep ) C.nidx[ k ] = I( kept_before + __popc( m & ( ( 1u << lane ) - 1 ) ) );
        kept_before += __popc( m );
    }
    __syncwarp();
    for ( int base = 0; base < nkeep + nout; base += 32 ) {
        int k = base + lane;
        bool keep = k < nv && ! C.out[ k ];
        int dst = keep ? C.nidx[ k ] : 0;
        double x = 0, y = 0, z = 0;
        I a = 0, b = 0, c = 0, j0 = 0, j1 = 0, j2 = 0;
        if ( keep ) {
            x = C.vx[ k ]; y = C.vy[ k ]; z = C.vz[ k ]; a = C.va[ k ]; b = C.vb[ k ]; c = C.vc[ k ];
            const int t0 = C.ad[ 0 ][ k ], t1 = C.ad[ 1 ][ k ], t2 = C.ad[ 2 ][ k ];
            j0 = t0 == C3::NONE || C.out[ t0 ] ? I( C3::NONE ) : C.nidx[ t0 ];
            j1 = t1 == C3::NONE || C.out[ t1 ] ? I( C3::NONE ) : C.nidx[ t1 ];
            j2 = t2 == C3::NONE || C.out[ t2 ] ? I( C3::NONE ) : C.nidx[ t2 ];
        }
        __syncwarp();
        if ( keep ) {
            C.vx[ dst ] = x; C.vy[ dst ] = y; C.vz[ dst ] = z; C.va[ dst ] = a; C.vb[ dst ] = b; C.vc[ dst ] = c;
            C.ad[ 0 ][ dst ] = j0; C.ad[ 1 ][ dst ] = j1; C.ad[ 2 ][ dst ] = j2;
        }
        __syncwarp();
    }
    // the new vertices, placed above: edge 0 (e0, e1) faces their kept vertex, edge 1 (e1, P) the new vertex that starts
    // at e1, edge 2 (P, e0) the one that ends at e0; the kept vertex's edge (e1, e0) faces the new vertex
    for ( int j = lane; j < nnew; j += 32 ) {
        const int d = nkeep + j, e0 = C.nt[ j ][ 0 ], e1 = C.nt[ j ][ 1 ];
        C.va[ d ] = I( e0 ); C.vb[ d ] = I( e1 ); C.vc[ d ] = I( P );
        C.vx[ d ] = C.area[ j ]; C.vy[ d ] = C.area[ VC + j ]; C.vz[ d ] = C.area[ 2 * VC + j ];
        const int T = C.nidx[ C.nk[ j ] ];
        C.ad[ 0 ][ d ] = I( T );
        C.ad[ 1 ][ d ] = cyc ? I( nkeep + C.e0t[ e1 ] ) : I( C3::NONE );
        C.ad[ 2 ][ d ] = cyc ? I( nkeep + C.e1t[ e0 ] ) : I( C3::NONE );
        const int ta = C.va[ T ], tb = C.vb[ T ], tc = C.vc[ T ];
        const int qT = ( ta == e1 && tb == e0 ) ? 0 : ( ( tb == e1 && tc == e0 ) ? 1 : 2 );
        C.ad[ qT ][ T ] = I( d );
    }
    __syncwarp();
    for ( int j = lane; j < nnew; j += 32 ) { C.e0t[ C.nt[ j ][ 0 ] ] = I( C3::NONE ); C.e1t[ C.nt[ j ][ 1 ] ] = I( C3::NONE ); }
    if ( lane == 0 ) C.nv = nkeep + nnew;
    __syncwarp();
    if ( ! cyc ) rebuild_adj( C, lane );
    return true;
}

// ---- the neighbour search ---------------------------------------------------------------------------------------------
// may a seed of weight at most W, at least sqrt( d2 ) away, cut a cell of squared radius R2 around a seed of weight wi?
// (its bisector reaches the cell's ball only if |q| < R + sqrt( R^2 + wj - wi ); W < -1e299: empty)
__device__ __forceinline__ bool may_cut3( double d2, double W, double R2, double wi ) {
    if ( W < -1e299 ) return false;
    double ex = R2 + W - wi, rb = sqrt( R2 ) + sqrt( ex > 0 ? ex : 0.0 );
    return d2 < rb * rb;
}
// squared distance from p to the grid cells [ a0, a1 ] (inclusive, per axis)
__device__ __forceinline__ double cells_dist2_3( const ProbDev &P, const int *a0, const int *a1, double px, double py, double pz ) {
    const double p[ 3 ] = { px, py, pz };
    double d2 = 0;
    for ( int a = 0; a < 3; ++a ) {
        double lo = P.go[ a ] + a0[ a ] * P.gh[ a ], hi = P.go[ a ] + ( a1[ a ] + 1 ) * P.gh[ a ];
        double d = fmax( 0.0, fmax( lo - p[ a ], p[ a ] - hi ) );
        d2 += d * d;
    }
    return d2;
}
template<class C3>
__device__ __forceinline__ double radius2_3( const C3 &C, int lane ) {
    double R2 = 0;
    for ( int k = lane; k < C.nv; k += 32 ) R2 = fmax( R2, C.vx[ k ] * C.vx[ k ] + C.vy[ k ] * C.vy[ k ] + C.vz[ k ] * C.vz[ k ] );
    return warp_max( R2 );
}

// the seeds of up to 32 grid cells (lane k: the range [ beg, beg + cnt ) of one cell) as candidates, 32 at a time:
// each lane pre-tests one candidate against every vertex, then the cuts run in lane order
template<bool CNT, class C3>
__device__ void cut_by_ranges3( C3 &C, const ProbDev &P, int lane, int s, double px, double py, double pz, double wi, int beg, int cnt,
                                bool &overflow ) {
    int inc = cnt;
#pragma unroll
    for ( int o = 1; o < 32; o <<= 1 ) { int t = __shfl_up_sync( FULL3, inc, o ); if ( lane >= o ) inc += t; }
    const int total = __shfl_sync( FULL3, inc, 31 );
    const int exc = inc - cnt;
    for ( int t0 = 0; t0 < total && C.nv > 0 && ! overflow; t0 += 32 ) {
        const int t = t0 + lane;
        int owner = 0;
#pragma unroll
        for ( int st = 16; st > 0; st >>= 1 ) { int v = __shfl_sync( FULL3, inc, owner + st - 1 ); if ( v <= t ) owner += st; }
        owner = owner > 31 ? 31 : owner;
        int obeg = __shfl_sync( FULL3, beg, owner ), oexc = __shfl_sync( FULL3, exc, owner );
        int j = obeg + ( t - oexc );
        bool valid = t < total && j != s;
        if constexpr ( CNT ) if ( P.gather ) count_reads( P, lane, G_CAND, __popc( __ballot_sync( FULL3, valid ) ) );
        double qx = 0, qy = 0, qz = 0, off = 0;
        if ( valid ) {
            qx = P.pos[ 3 * ( size_t ) j ] - px;
            qy = P.pos[ 3 * ( size_t ) j + 1 ] - py;
            qz = P.pos[ 3 * ( size_t ) j + 2 ] - pz;
            double qw = P.w ? P.w[ j ] : 0.0;
            off = 0.5 * ( ( wi - qw ) + ( qx * qx + qy * qy + qz * qz ) );
        }
        bool cuts = false;
        const double tol = valid ? tie_tol3( qx, qy, qz, off, C.L ) : 0.0;
        for ( int k = 0; k < C.nv && valid; ++k ) cuts |= qx * C.vx[ k ] + qy * C.vy[ k ] + qz * C.vz[ k ] - off > tol;
        unsigned todo = __ballot_sync( FULL3, valid && cuts );
        while ( todo ) {
            int k = __ffs( todo ) - 1;
            todo &= todo - 1;
            double nx = __shfl_sync( FULL3, qx, k ), ny = __shfl_sync( FULL3, qy, k ), nz = __shfl_sync( FULL3, qz, k );
            double no = __shfl_sync( FULL3, off, k );
            int nid = __shfl_sync( FULL3, j, k );
            if ( ! wclip3( C, lane, nx, ny, nz, no, nid ) ) { overflow = true; break; }
            if ( C.nv == 0 ) break;
        }
    }
}

constexpr int WALK_STACK3 = 96;      // at most 7 entries per level stay on the stack (12 levels)
constexpr int SHELLS_FIRST = 2;      // shells walked before the pyramid takes over
constexpr int WALK_LEAF3 = 1;        // the walk's leaves: blocks of 2 x 2 x 2 grid cells, one cell per lane

// the pyramid of weight majorants, depth first, nearest child first, skipping the cells within Chebyshev distance rd of
// c0 (the shells already walked) and the blocks that claim no vertex of the cell (wmaj_claims); a leaf block has
// one cell per lane, each tested by `may_cut3`, clipped together.  A node's children are tested when it is expanded, one
// child per lane for their majorant records (eight loads in flight instead of one per pop), then each against the cell's
// vertices; only the claiming children are pushed
template<bool CNT, class C3>
__device__ void walk_pyramid3( C3 &C, const ProbDev &P, int lane, int s, double px, double py, double pz, double wi, const int *c0, int rd,
                               int2 *stk, bool &overflow ) {
    const int *g = P.g;
    if ( lane == 0 ) stk[ 0 ] = make_int2( ( P.nlev - 1 ) << 22, 0 );
    int sp = 1;
    __syncwarp();
    double R2 = radius2_3( C, lane );
    for ( int guard = 0; sp > 0 && guard < ( 1 << 24 ); ++guard ) {
        const int2 e = stk[ sp - 1 ];
        --sp;
        __syncwarp();
        const int l = e.x >> 22, X[ 3 ] = { ( e.x >> 11 ) & 0x7ff, e.x & 0x7ff, e.y };
        int a0[ 3 ], a1[ 3 ];
        for ( int a = 0; a < 3; ++a ) {
            a0[ a ] = X[ a ] << l;
            a1[ a ] = min( ( X[ a ] + 1 ) << l, g[ a ] ) - 1;
        }
        if ( l <= WALK_LEAF3 ) {
            const int bw[ 3 ] = { a1[ 0 ] - a0[ 0 ] + 1, a1[ 1 ] - a0[ 1 ] + 1, a1[ 2 ] - a0[ 2 ] + 1 };   // at most 2 x 2 x 2
            int beg = 0, cnt = 0;
            bool tested = false, ranged = false;
            if ( lane < bw[ 0 ] * bw[ 1 ] * bw[ 2 ] ) {
                int x[ 3 ] = { a0[ 0 ] + lane % bw[ 0 ], a0[ 1 ] + ( lane / bw[ 0 ] ) % bw[ 1 ], a0[ 2 ] + lane / ( bw[ 0 ] * bw[ 1 ] ) };
                bool walked = true;
                for ( int a = 0; a < 3; ++a ) walked = walked && x[ a ] >= c0[ a ] - rd && x[ a ] <= c0[ a ] + rd;
                const size_t gc = ( ( size_t ) x[ 2 ] * g[ 1 ] + x[ 1 ] ) * g[ 0 ] + x[ 0 ];
                tested = ! walked;
                if ( ! walked && may_cut3( cells_dist2_3( P, x, x, px, py, pz ), wmaj_b( P, gc ), R2, wi ) ) {
                    int2 rg = P.cell_range[ gc ];
                    beg = rg.x;
                    cnt = rg.y - rg.x;
                    ranged = true;
                }
            }
            if constexpr ( CNT ) if ( P.gather ) {
                count_reads( P, lane, G_GRID, __popc( __ballot_sync( FULL3, tested ) ) );
                count_reads( P, lane, G_RANGE, __popc( __ballot_sync( FULL3, ranged ) ) );
            }
            cut_by_ranges3<CNT>( C, P, lane, s, px, py, pz, wi, beg, cnt, overflow );
            if ( overflow || C.nv == 0 ) return;
            R2 = radius2_3( C, lane );
            continue;
        }
        // the (up to 8) children, lane k the child k: in the grid, not all inside the walked shells, not empty
        int Y[ 3 ], b0[ 3 ], b1[ 3 ];
        bool ok = lane < 8, inside = true;
        for ( int a = 0; a < 3; ++a ) {
            Y[ a ] = 2 * X[ a ] + ( ( lane >> a ) & 1 );
            ok = ok && Y[ a ] < lev_dim( g[ a ], l - 1 );
            b0[ a ] = Y[ a ] << ( l - 1 );
            b1[ a ] = min( ( Y[ a ] + 1 ) << ( l - 1 ), g[ a ] ) - 1;
            inside = inside && b0[ a ] >= c0[ a ] - rd && b1[ a ] <= c0[ a ] + rd;
        }
        ok = ok && ! inside;
        double cb = -1e300, ca[ 3 ] = { 0, 0, 0 }, lo[ 3 ] = { 0, 0, 0 }, hi[ 3 ] = { 0, 0, 0 }, dd = 0;
        if constexpr ( CNT ) if ( P.gather ) count_reads( P, lane, G_NODE, __popc( __ballot_sync( FULL3, ok ) ) );
        if ( ok ) {
            const size_t rec = P.poff[ l - 1 ] + ( ( size_t ) Y[ 2 ] * lev_dim( g[ 1 ], l - 1 ) + Y[ 1 ] ) * lev_dim( g[ 0 ], l - 1 ) + Y[ 0 ];
            cb = wmaj_b( P, rec );
            const double *am = P.wpyr + rec * 4;
            ca[ 0 ] = am[ 0 ]; ca[ 1 ] = am[ 1 ]; ca[ 2 ] = am[ 2 ];
            for ( int q = 0; q < 3; ++q ) { lo[ q ] = P.go[ q ] + b0[ q ] * P.gh[ q ]; hi[ q ] = P.go[ q ] + ( b1[ q ] + 1 ) * P.gh[ q ]; }
            dd = cells_dist2_3( P, b0, b1, px, py, pz );
            ok = cb >= -1e299;
        }
        // does each child claim a vertex of the cell?  (lanes over the vertices, the child's record broadcast)
        unsigned todo = __ballot_sync( FULL3, ok ), claim = 0;
        while ( todo ) {
            const int c = __ffs( todo ) - 1;
            todo &= todo - 1;
            const double A[ 3 ] = { __shfl_sync( FULL3, ca[ 0 ], c ), __shfl_sync( FULL3, ca[ 1 ], c ), __shfl_sync( FULL3, ca[ 2 ], c ) };
            const double B = __shfl_sync( FULL3, cb, c );
            const double LO[ 3 ] = { __shfl_sync( FULL3, lo[ 0 ], c ), __shfl_sync( FULL3, lo[ 1 ], c ), __shfl_sync( FULL3, lo[ 2 ], c ) };
            const double HI[ 3 ] = { __shfl_sync( FULL3, hi[ 0 ], c ), __shfl_sync( FULL3, hi[ 1 ], c ), __shfl_sync( FULL3, hi[ 2 ], c ) };
            bool may = false;
            for ( int k = lane; k < C.nv && ! may; k += 32 ) {
                const double v[ 3 ] = { C.vx[ k ], C.vy[ k ], C.vz[ k ] }, Xp[ 3 ] = { px + v[ 0 ], py + v[ 1 ], pz + v[ 2 ] };
                may = wmaj_claims( A, B, LO, HI, Xp, v, 3, wi );
            }
            if ( __any_sync( FULL3, may ) ) claim |= 1u << c;
        }
        // the claiming children pushed farthest first (equal distances in child order), so that the nearest is popped first
        int rank = 0;
#pragma unroll
        for ( int c = 0; c < 8; ++c ) {
            const double dc = __shfl_sync( FULL3, dd, c );
            if ( ( ( claim >> c ) & 1 ) && ( dc > dd || ( dc == dd && c < lane ) ) ) ++rank;
        }
        const int nc = __popc( claim );
        if ( sp + nc > WALK_STACK3 ) return;               // cannot happen below 2^13 cells per side
        if ( ( claim >> lane ) & 1 ) stk[ sp + rank ] = make_int2( ( ( l - 1 ) << 22 ) | ( Y[ 0 ] << 11 ) | Y[ 1 ], Y[ 2 ] );
        sp += nc;
        __syncwarp();
    }
}

// ---- sums of isotropic gaussians over the polyhedron ------------------------------------------------------------------
// rho_g = m / ((2 pi)^{3/2} s^3) exp(-|y - c|^2 / 2 s^2).  Everything reduces to integrals over the faces:
//  * mass (Gauss's theorem with the radial field G(r)/(4 pi r^2), G the gaussian's mass within radius r, minus the
//    point mass m at c, which leaves erfc tails and no cancellation far from c):
//        M = m [c inside] + sum_f h_f/(4 pi) int_face-angle [ Ht( r_out ) - Ht( |h_f| ) ] dtheta,  Ht(r) = m erfc(r/(s sqrt2))/r
//    with h_f = (y - c).n_f on face f and the angle taken about the foot of c on the face;
//  * face integrals: int_face rho = K e^{-h^2/2s^2} s^2 [ Theta_f - int exp(-R(theta)^2/2s^2) dtheta ], Theta_f the
//    winding angle of the face about the foot (2 pi or 0), R(theta) the distance from the foot to the face's edge;
//  * moments from (y - c) rho = -s^2 grad rho and |y - c|^2 rho = s^2 (3 rho - div((y - c) rho)):
//        int (y - c) rho = -s^2 sum_f n_f int_face rho,   int |y - c|^2 rho = s^2 ( 3 M - sum_f h_f int_face rho ).
// The angle integrals run per edge, in u with s = d sinh u along the edge's line (s measured from the foot's
// perpendicular on the line, d the foot's distance to it): R = d cosh u and dtheta = du / cosh u, so every kernel is
// smooth in u (1 / cosh u has its only poles at +-i pi/2).  Gauss-Legendre pieces of 8 points are uniform in
// V(u) = int max( 1 / G3_WU, d |sinh u| / ( G3_FR s ) ) du: at most G3_WU wide in u, and R changes by at most G3_FR s over
// each, the gaussian's own scale.  Against 30-digit quadrature on the edges of real power cells (1e3 to 3e4 seeds in
// the unit cube, 4 gaussians of sigma in [0.05, 0.15]) the rule is within 2e-14 and takes 1.2 pieces per edge on
// average, 12 at most.
// The work is spread over the warp as (gaussian, entry) and (gaussian, face) items, one per lane at a time.
__constant__ double c_g3x[ 8 ] = { -0.9602898564975363, -0.7966664774136267, -0.5255324099163290, -0.1834346424956498,
                                    0.1834346424956498, 0.5255324099163290, 0.7966664774136267, 0.9602898564975363 };
__constant__ double c_g3w[ 8 ] = { 0.1012285362903763, 0.2223810344533745, 0.3137066458778873, 0.3626837833783620,
                                    0.3626837833783620, 0.3137066458778873, 0.2223810344533745, 0.1012285362903763 };
constexpr double G3_WU = 0.7, G3_FR = 0.5;
constexpr int G3_MAX_PIECES = 64;

// the signed angle of the edge K -> T about F, positive counterclockwise about -n (the cell's edges run clockwise
// about the outward normal n, so a foot inside the face gets +2 pi in total)
__device__ __forceinline__ double edge_angle3( double Fx, double Fy, double Fz, double Kx, double Ky, double Kz, double Tx, double Ty,
                                               double Tz, double nx, double ny, double nz ) {
    double ax = Kx - Fx, ay = Ky - Fy, az = Kz - Fz, bx = Tx - Fx, by = Ty - Fy, bz = Tz - Fz;
    double o = -( nx * ( ay * bz - az * by ) + ny * ( az * bx - ax * bz ) + nz * ( ax * by - ay * bx ) );
    return atan2( o, ax * bx + ay * by + az * bz );
}

// A = int erfc( r / s sqrt2 ) / r dtheta and B = int exp( -R^2 / 2 s^2 ) dtheta along the edge K -> T of a face (F the
// foot of the centre on the face's plane, n its unit normal, h the centre's distance to the plane, r^2 = h^2 + R^2),
// signed as `edge_angle3`.  erfc( k r ) = exp( -k^2 h^2 ) exp( -k^2 R^2 ) erfcx( k r ): one exponential serves both.
// An EDGE ITEM holds one such integral between its pieces: `edge_setup3` places the pieces, `edge_piece3` integrates one
// (8 Gauss-Legendre points) -- so that the lanes of a warp can each hold a different edge and take the next one as soon
// as theirs is done, instead of the whole warp waiting for its longest edge
struct EdgeItem3 {
    double d, h2, k2, kr, eh, us, chs, vs, kd, v0, dv, u1, ua, A, B, sgn;
    int np, j;
};

__device__ __forceinline__ void edge_setup3( EdgeItem3 &I, double Fx, double Fy, double Fz, double Kx, double Ky, double Kz, double Tx, double Ty,
                                             double Tz, double nx, double ny, double nz, double h, double sg ) {
    I.A = I.B = 0;
    I.np = I.j = 0;
    const double ax = Kx - Fx, ay = Ky - Fy, az = Kz - Fz, ex = Tx - Kx, ey = Ty - Ky, ez = Tz - Kz;
    const double L = sqrt( ex * ex + ey * ey + ez * ez );
    if ( ! ( L > 0 ) ) return;
    const double iL = 1 / L, ux = ex * iL, uy = ey * iL, uz = ez * iL;
    const double s0 = ax * ux + ay * uy + az * uz, s1 = s0 + L;
    const double qx = ax - s0 * ux, qy = ay - s0 * uy, qz = az - s0 * uz;
    const double d = sqrt( qx * qx + qy * qy + qz * qz );
    if ( ! ( d > 0 ) ) return;
    const double bx = Tx - Fx, by = Ty - Fy, bz = Tz - Fz;
    const double o = -( nx * ( ay * bz - az * by ) + ny * ( az * bx - ax * bz ) + nz * ( ax * by - ay * bx ) );
    I.sgn = o >= 0 ? 1.0 : -1.0;
    // (past |s / d| = 1e17, u = 40.4, the kernel 1 / cosh u is under 1e-17)
    const double id = 1 / d;
    const double x0 = fmax( -1e17, fmin( 1e17, s0 * id ) ), x1 = fmax( -1e17, fmin( 1e17, s1 * id ) );
    const double u0 = asinh( x0 ), u1 = asinh( x1 );
    const double fs = G3_FR * sg, c = fmin( 1e17, fs / ( G3_WU * d ) );      // sinh of the u where the two bounds meet
    I.us = asinh( c ); I.chs = sqrt( 1 + c * c ); I.vs = I.us / G3_WU; I.kd = d / fs;
    auto V = [&]( double u, double x ) {          // (cosh u = sqrt( 1 + x^2 ) at u = asinh x)
        const double a = fabs( u );
        return copysign( a <= I.us ? a / G3_WU : I.vs + I.kd * ( sqrt( 1 + x * x ) - I.chs ), u );
    };
    I.v0 = V( u0, x0 );
    const double v1 = V( u1, x1 );
    I.np = max( 1, min( G3_MAX_PIECES, int( ceil( v1 - I.v0 ) ) ) );
    I.dv = ( v1 - I.v0 ) / I.np;
    I.kr = 0.7071067811865476 / sg; I.k2 = I.kr * I.kr; I.h2 = h * h;
    I.eh = exp( -I.k2 * I.h2 );
    I.d = d; I.u1 = u1; I.ua = u0;
}

__device__ __forceinline__ void edge_piece3( EdgeItem3 &I ) {
    double ub = I.u1;
    if ( I.j + 1 < I.np ) {
        const double a = fabs( I.v0 + ( I.j + 1 ) * I.dv );
        ub = copysign( a <= I.vs ? a * G3_WU : acosh( I.chs + ( a - I.vs ) / I.kd ), I.v0 + ( I.j + 1 ) * I.dv );
    }
    const double hw = 0.5 * ( ub - I.ua ), mid = 0.5 * ( ub + I.ua );
    double A = 0, B = 0;
#pragma unroll 2
    for ( int q = 0; q < 8; ++q ) {
        const double uq = mid + hw * c_g3x[ q ], w = hw * c_g3w[ q ];
        // 1 / cosh u = 2 e^u / ( e^2u + 1 ) and R = d cosh u, from one division
        const double eu = exp( uq ), s1 = eu * eu + 1, iq = 1 / ( eu * s1 );
        const double ich = 2 * eu * eu * iq, R = 0.5 * I.d * s1 * s1 * iq, R2 = R * R;
        const double gw = w * ich * exp( -I.k2 * R2 );
        B += gw;
        if ( I.h2 != 0 ) {
            const double r2 = I.h2 + R2, ir = rsqrt( r2 );
            A += gw * I.eh * erfcx( I.kr * ( r2 * ir ) ) * ir;
        }
    }
    I.A += A;
    I.B += B;
    I.ua = ub;
    ++I.j;
}

// the gaussian sums over the clipped cell: lane parts of the mass, of the first moment about the seed and of
// int |y|^2 rho (seed frame); C.area receives each (vertex, edge) entry's part of its face integral and C.fmp each
// face's winding-angle part (both summed over the gaussians, in gaussian order)
template<class C3>
__device__ __noinline__ void integrate_gauss3( C3 &C, const ProbDev &P, int lane, double px, double py, double pz, double &M, double &Fx,
                                                double &Fy, double &Fz, double &S2 ) {
    const int nv = C.nv, np = C.np;
    for ( int k = lane; k < 3 * nv; k += 32 ) C.area[ k ] = 0;
    for ( int p = lane; p < np; p += 32 ) C.fmp[ p ] = 0;
    __syncwarp();
    if ( nv == 0 ) return;
    // each face's boundary entries (vertex k, edge q with e[ q ] the face), as a list in vertex order, built once for all
    // the gaussians: the head vertex in `remap`, the next vertex after (k, q) in `nt[ k ][ q ]` (both free once the cell
    // is clipped)
    for ( int p = lane; p < np; p += 32 ) {
        int prev = -1, pq = 0;
        for ( int k = 0; k < nv; ++k ) {
            const int e[ 3 ] = { C.va[ k ], C.vb[ k ], C.vc[ k ] };
            for ( int q = 0; q < 3; ++q ) {
                if ( e[ q ] != p || C.ad[ q ][ k ] == C3::NONE ) continue;
                if ( prev < 0 ) C.remap[ p ] = ( typename C3::I ) k;
                else C.nt[ prev ][ pq ] = ( typename C3::I ) k;
                prev = k;
                pq = q;
            }
        }
        if ( prev < 0 ) C.remap[ p ] = ( typename C3::I ) C3::NONE;
        else C.nt[ prev ][ pq ] = ( typename C3::I ) C3::NONE;
    }
    __syncwarp();
    const double INV4PI = 0.07957747154594767, TWO_PI = 6.283185307179586;
    const int ng = P.dn[ 0 ];
    // a gaussian whose centre lies beyond a face of the cell, at distance D from its plane, puts at most
    // B = m erfc( D / sigma sqrt 2 ) / 2 in the cell (its mass in that half-space): one whose B is under 1e-20 of the
    // largest B of the cell's gaussians is left out (its part is below the doubles of the cell's mass and measures)
    auto bound = [&]( int g ) {
        const double *G = P.dval + g * 5;
        const double cx = G[ 0 ] - px, cy = G[ 1 ] - py, cz = G[ 2 ] - pz;
        double D = 0;
        for ( int p = lane; p < np; p += 32 ) {
            const double nn = sqrt( C.nx[ p ] * C.nx[ p ] + C.ny[ p ] * C.ny[ p ] + C.nz[ p ] * C.nz[ p ] );
            D = fmax( D, ( C.nx[ p ] * cx + C.ny[ p ] * cy + C.nz[ p ] * cz - C.no[ p ] ) / nn );
        }
        for ( int o = 16; o > 0; o >>= 1 ) D = fmax( D, __shfl_xor_sync( FULL3, D, o ) );
        return 0.5 * G[ 4 ] * erfc( D * 0.7071067811865476 / G[ 3 ] );
    };
    double bmax = 0;
    for ( int g = 0; g < ng; ++g ) bmax = fmax( bmax, bound( g ) );
    // the parts of one item: dM of the mass, and the face integral b of the face f (unit normal n); with the gaussian's
    // centre c (seed frame) and variance s2 they give the moments' parts (moments about c, moved to the seed)
    auto add = [&]( double dM, double b, double h, double nhx, double nhy, double nhz, double cx, double cy, double cz, double s2g ) {
        const double gx = -s2g * nhx * b, gy = -s2g * nhy * b, gz = -s2g * nhz * b;
        M += dM;
        Fx += gx + cx * dM; Fy += gy + cy * dM; Fz += gz + cz * dM;
        S2 += s2g * ( 3 * dM - h * b ) + 2 * ( cx * gx + cy * gy + cz * gz ) + ( cx * cx + cy * cy + cz * cz ) * dM;
    };
    // the face items are (gaussian of the group's selection, face), lane-consecutive; with at least 32 faces per
    // gaussian, the 32 items of one round hold distinct faces, so their sums into `fmp` never meet, and each face's sum
    // runs in gaussian order
    const int NE = 3 * nv, NPp = np > 32 ? np : 32;
    for ( int g0 = 0; g0 < ng; g0 += 32 ) {
        const int gn = min( 32, ng - g0 );
        unsigned sel = 0;
        for ( int j = 0; j < gn; ++j )
            if ( ng == 1 || ! ( bound( g0 + j ) < 1e-20 * bmax ) ) sel |= 1u << j;      // (warp uniform: the bound is a warp max)
        const int ns = __popc( sel );
        auto nth = [&]( int i ) {          // the i-th selected gaussian
            unsigned m = sel;
            for ( int k = 0; k < i; ++k ) m &= m - 1;
            return g0 + __ffs( m ) - 1;
        };
        // the edge integrals of every (gaussian, entry), as a queue: a lane whose item is done takes the next one (items
        // in gaussian-major order), every lane integrates one piece of its item per step.  An item's part goes to its entry
        // of `area` when it is done; two lanes finishing the same entry in one step add in lane order
        {
            const int total = ns * NE;
            int nxt = 0, item = -1;
            EdgeItem3 I;
            I.np = I.j = 0;
            double h = 0, nhx = 0, nhy = 0, nhz = 0, cx = 0, cy = 0, cz = 0, s2g = 0, mg = 0, KG = 0;
            for ( int guard = 0; guard < 1 << 20; ++guard ) {
                const bool need = item < 0;
                const unsigned nm = __ballot_sync( FULL3, need );
                const int mine = nxt + __popc( nm & ( ( 1u << lane ) - 1 ) );
                nxt = min( total, nxt + __popc( nm ) );
                if ( need && mine < total ) {
                    item = mine;
                    const int gi = mine / NE, e = mine - gi * NE, k = e / 3, q = e - 3 * k, t = C.ad[ q ][ k ];
                    const int g = nth( gi );
                    const double *G = P.dval + g * 5;
                    const double sg = G[ 3 ];
                    cx = G[ 0 ] - px; cy = G[ 1 ] - py; cz = G[ 2 ] - pz; mg = G[ 4 ];
                    s2g = sg * sg; KG = mg / ( 15.749609945722419 * s2g * sg );          // (2 pi)^{3/2}
                    if ( t == C3::NONE ) I.np = I.j = 0;
                    else {
                        const int f = q == 0 ? C.va[ k ] : ( q == 1 ? C.vb[ k ] : C.vc[ k ] );
                        const double nn = sqrt( C.nx[ f ] * C.nx[ f ] + C.ny[ f ] * C.ny[ f ] + C.nz[ f ] * C.nz[ f ] ), inn = 1 / nn;
                        nhx = C.nx[ f ] * inn; nhy = C.ny[ f ] * inn; nhz = C.nz[ f ] * inn;
                        h = ( C.no[ f ] - ( C.nx[ f ] * cx + C.ny[ f ] * cy + C.nz[ f ] * cz ) ) * inn;
                        edge_setup3( I, cx + h * nhx, cy + h * nhy, cz + h * nhz, C.vx[ k ], C.vy[ k ], C.vz[ k ], C.vx[ t ], C.vy[ t ],
                                     C.vz[ t ], nhx, nhy, nhz, h, sg );
                    }
                }
                if ( ! __any_sync( FULL3, item >= 0 ) ) break;
                if ( item >= 0 && I.j < I.np ) edge_piece3( I );
                const bool done = item >= 0 && I.j >= I.np;
                const unsigned dm = __ballot_sync( FULL3, done && I.np > 0 );
                if ( done ) {
                    const int e = item % NE;
                    if ( I.np > 0 ) {
                        const double A = I.sgn * I.A, B = I.sgn * I.B;
                        const double b = -KG * I.eh * s2g * B;             // (eh = exp( -h^2 / 2 s^2 ))
                        const unsigned same = __match_any_sync( dm, e );
                        const int rank = __popc( same & ( ( 1u << lane ) - 1 ) ), nsame = __popc( same );
                        for ( int r = 0; r < nsame; ++r ) {
                            if ( r == rank ) C.area[ e ] += b;
                            __syncwarp( same );
                        }
                        add( h * INV4PI * mg * A, b, h, nhx, nhy, nhz, cx, cy, cz, s2g );
                    }
                    item = -1;
                }
                __syncwarp();
            }
        }
        // per (gaussian, face): the winding angle of the face about the foot of c, its part of the face integral and of
        // the flux of the erfc field's constant part
        for ( int base = 0; base < ns * NPp; base += 32 ) {
            const int idx = base + lane, gi = idx / NPp, p = idx - gi * NPp;
            if ( gi < ns && p < np ) {
                const int g = nth( gi );
                const double *G = P.dval + g * 5;
                const double cx = G[ 0 ] - px, cy = G[ 1 ] - py, cz = G[ 2 ] - pz, sg = G[ 3 ], mg = G[ 4 ];
                const double s2g = sg * sg, KG = mg / ( 15.749609945722419 * s2g * sg ), kr = 0.7071067811865476 / sg;
                const double nn = sqrt( C.nx[ p ] * C.nx[ p ] + C.ny[ p ] * C.ny[ p ] + C.nz[ p ] * C.nz[ p ] );
                const double nhx = C.nx[ p ] / nn, nhy = C.ny[ p ] / nn, nhz = C.nz[ p ] / nn;
                const double h = ( C.no[ p ] - ( C.nx[ p ] * cx + C.ny[ p ] * cy + C.nz[ p ] * cz ) ) / nn;
                const double Fx0 = cx + h * nhx, Fy0 = cy + h * nhy, Fz0 = cz + h * nhz;
                // the face is convex: its winding angle about the foot is 2 pi inside (every edge turns the same way, the
                // signs of `edge_angle3`'s cross products), 0 outside (both signs); a foot within 1e-6 (sine) of an edge's
                // line takes the walk of the angles
                int npos = 0, nneg = 0;
                bool near = false;
                for ( int k = C.remap[ p ]; k != C3::NONE; ) {
                    const int q = C.va[ k ] == p ? 0 : ( C.vb[ k ] == p ? 1 : 2 );
                    const int t = C.ad[ q ][ k ];
                    const double ax = C.vx[ k ] - Fx0, ay = C.vy[ k ] - Fy0, az = C.vz[ k ] - Fz0;
                    const double bx = C.vx[ t ] - Fx0, by = C.vy[ t ] - Fy0, bz = C.vz[ t ] - Fz0;
                    const double o = -( nhx * ( ay * bz - az * by ) + nhy * ( az * bx - ax * bz ) + nhz * ( ax * by - ay * bx ) );
                    const double a2 = ax * ax + ay * ay + az * az, b2 = bx * bx + by * by + bz * bz;
                    if ( ! ( o * o > 1e-12 * a2 * b2 ) ) near = true;
                    else if ( o > 0 ) ++npos;
                    else ++nneg;
                    k = C.nt[ k ][ q ];
                }
                double Th = nneg == 0 ? TWO_PI : ( npos == 0 ? -TWO_PI : 0.0 );
                if ( near ) {
                    double th = 0;
                    for ( int k = C.remap[ p ]; k != C3::NONE; ) {
                        const int q = C.va[ k ] == p ? 0 : ( C.vb[ k ] == p ? 1 : 2 );
                        const int t = C.ad[ q ][ k ];
                        th += edge_angle3( Fx0, Fy0, Fz0, C.vx[ k ], C.vy[ k ], C.vz[ k ], C.vx[ t ], C.vy[ t ], C.vz[ t ], nhx, nhy, nhz );
                        k = C.nt[ k ][ q ];
                    }
                    const double kk = rint( th / TWO_PI );
                    Th = fabs( th - TWO_PI * kk ) < 1e-6 ? TWO_PI * kk : th;
                }
                if ( Th != 0 ) {
                    const double I = KG * exp( -h * h * 0.5 / s2g ) * s2g * Th;
                    C.fmp[ p ] += I;
                    // the flux of the erfc field's constant part; at h = 0 its limit from the inner side
                    const double dM = h != 0 ? -h * INV4PI * mg * erfc( fabs( h ) * kr ) / fabs( h ) * Th : -INV4PI * mg * Th;
                    add( dM, I, h, nhx, nhy, nhz, cx, cy, cz, s2g );
                }
            }
            __syncwarp();
        }
        // the point mass taken out of the field, for a centre on the inner side of every face
        for ( int gi = 0; gi < ns; ++gi ) {
            const int g = nth( gi );
            const double *G = P.dval + g * 5;
            const double cx = G[ 0 ] - px, cy = G[ 1 ] - py, cz = G[ 2 ] - pz;
            bool ok = true;
            for ( int p = lane; p < np; p += 32 ) ok = ok && C.no[ p ] - ( C.nx[ p ] * cx + C.ny[ p ] * cy + C.nz[ p ] * cz ) >= 0;
            if ( __all_sync( FULL3, ok ) && lane == 0 ) add( G[ 4 ], 0.0, 0.0, 0.0, 0.0, 0.0, cx, cy, cz, G[ 3 ] * G[ 3 ] );
        }
        __syncwarp();
    }
}

__device__ __forceinline__ void record_error3( const ProbDev &P, ErrRec *err, int code, int prob, int seed, int needed ) {
    if ( P.perr ) *P.perr = 1.0;
    if ( atomicCAS( &err->code, 0, code ) == 0 ) { err->kind = 2; err->prob = prob; err->seed = seed; err->needed = needed; }
}

__device__ __forceinline__ double g_of3( double x, int r, double p ) {
    x = fmax( x, 1e-300 );
    if ( r == 2 ) return p == 0 ? log( x ) : ( pow( x, p ) - 1 ) / p;
    return r == 1 ? log( x ) : x - 1;
}
__device__ __forceinline__ double gp_of3( double x, int r, double p ) {
    x = fmax( x, 1e-300 );
    if ( r == 2 ) return pow( x, p - 1 );
    return r == 1 ? 1 / x : 1;
}

// a cell for the big-cell pass: queued (prob, seed); past the queue's capacity, an error of its problem
__device__ __forceinline__ void queue3( const ProbDev &P, ErrRec *err, OvfList *ovf, int prob, int s, int user, int lane ) {
    if ( lane == 0 ) {
        int k = atomicAdd( &ovf->count, 1 );
        if ( k < ovf->cap ) ovf->items[ k ] = OvfItem{ prob, s };
        else record_error3( P, err, 4, prob, user, 0 );
    }
    __syncwarp();
}

// THE CELL of seed s (rank) of problem `prob`, first half: the clip.  A cell past the vertex / plane capacities of this
// pass is queued on `ovf` for the next pass (main -> big -> giant; NULL: an error of its problem) and the call returns
// false (nothing written); true: the clipped cell is in C (possibly empty)
template<bool CNT, class C3>
__device__ __noinline__ bool clip3( C3 &C, const ProbDev &P, int prob, int s, int lane, ErrRec *err, OvfList *ovf, int2 *stk, double wmax, bool big ) {
    const double px = P.pos[ 3 * ( size_t ) s ], py = P.pos[ 3 * ( size_t ) s + 1 ], pz = P.pos[ 3 * ( size_t ) s + 2 ];
    const double wi = P.w ? P.w[ s ] : 0.0;
    init_box3( C, lane, P.lo, P.hi, px, py, pz );
    bool overflow = false;
    int c0[ 3 ];
    for ( int a = 0; a < 3; ++a ) {
        double x = a == 0 ? px : ( a == 1 ? py : pz );
        int k = int( floor( ( x - P.go[ a ] ) / P.gh[ a ] ) );
        c0[ a ] = k < 0 ? 0 : ( k >= P.g[ a ] ? P.g[ a ] - 1 : k );
    }
    int rmax = 0;
    for ( int a = 0; a < 3; ++a ) rmax = max( rmax, max( c0[ a ], P.g[ a ] - 1 - c0[ a ] ) );
    int rd = -1;                 // the shells walked, when the pyramid takes over
    for ( int r = 0; r <= rmax && C.nv > 0 && ! overflow; ++r ) {
        const int side = 2 * r + 1, ncube = side * side * side;
        const double R2s = radius2_3( C, lane );
        for ( int cb = 0; cb < ncube && C.nv > 0 && ! overflow; cb += 32 ) {
            int ci = cb + lane, beg = 0, cnt = 0;
            bool tested = false, ranged = false;
            if ( ci < ncube ) {
                int dx = ci % side - r, dy = ( ci / side ) % side - r, dz = ci / ( side * side ) - r;
                bool shell = max( abs( dx ), max( abs( dy ), abs( dz ) ) ) == r;
                int x[ 3 ] = { c0[ 0 ] + dx, c0[ 1 ] + dy, c0[ 2 ] + dz };
                if ( shell && x[ 0 ] >= 0 && x[ 0 ] < P.g[ 0 ] && x[ 1 ] >= 0 && x[ 1 ] < P.g[ 1 ] && x[ 2 ] >= 0 && x[ 2 ] < P.g[ 2 ] ) {
                    const size_t gc = ( ( size_t ) x[ 2 ] * P.g[ 1 ] + x[ 1 ] ) * P.g[ 0 ] + x[ 0 ];
                    tested = P.wpyr != nullptr;
                    if ( may_cut3( cells_dist2_3( P, x, x, px, py, pz ), P.wpyr ? wmaj_b( P, gc ) : wmax, R2s, wi ) ) {
                        int2 rg = P.cell_range[ gc ];
                        beg = rg.x;
                        cnt = rg.y - rg.x;
                        ranged = true;
                    }
                }
            }
            if constexpr ( CNT ) if ( P.gather ) {
                count_reads( P, lane, G_GRID, __popc( __ballot_sync( FULL3, tested ) ) );
                count_reads( P, lane, G_RANGE, __popc( __ballot_sync( FULL3, ranged ) ) );
            }
            cut_by_ranges3<CNT>( C, P, lane, s, px, py, pz, wi, beg, cnt, overflow );
        }
        if ( C.nv == 0 || overflow ) break;
        double R2 = radius2_3( C, lane );
        double ex = R2 + wmax - wi;
        if ( r * P.ghmin >= sqrt( R2 ) + sqrt( ex > 0 ? ex : 0.0 ) ) break;
        if ( P.wpyr && r >= SHELLS_FIRST && r < rmax && sqrt( R2 ) + sqrt( ex > 0 ? ex : 0.0 ) > ( r + 2 ) * P.ghmin ) { rd = r; break; }
    }
    if ( rd >= 0 && C.nv > 0 && ! overflow ) walk_pyramid3<CNT>( C, P, lane, s, px, py, pz, wi, c0, rd, stk, overflow );
    const int user = P.user[ s ];
    if ( overflow ) {
        // past the capacity of this warp's cell: the next pass rebuilds it -- but a trial diagram does not go past the big
        // pass: a cell of more than its 1024 vertices there refuses the step (the damping halves it)
        if ( big && P.prefuse ) {
            if ( lane == 0 ) *P.prefuse = 1.0;
            __syncwarp();
            return false;
        }
        if ( ovf ) { queue3( P, err, ovf, prob, s, user, lane ); return false; }
        if ( lane == 0 ) record_error3( P, err, 4, prob, user, C3::VC );
        if ( lane == 0 ) C.nv = 0;
        __syncwarp();
    }
    return true;
}

// THE CELL, second half: integrate the clipped cell in C, write.  The main kernel (`big` false) queues a cell with more
// facets than the table's row (and returns false, nothing written); the other passes write those to the overflow
// store.  `rep` (lane 0, may be NULL) accumulates the Newton report
template<class C3>
__device__ __noinline__ bool finish3( C3 &C, const ProbDev &P, int prob, int s, int lane, unsigned flags, ErrRec *err, OvfList *ovf, double *rep, bool big ) {
    const bool moments = flags & F_MOMENTS, facets = flags & F_FACETS, user_order = flags & F_USER_ORDER;
    const double px = P.pos[ 3 * ( size_t ) s ], py = P.pos[ 3 * ( size_t ) s + 1 ], pz = P.pos[ 3 * ( size_t ) s + 2 ];
    const int user = P.user[ s ];
    // ---- integration: signed tetrahedra ( 0, c_f, K, T ) -- every (vertex, directed edge) once; gaussians by
    // their face integrals (the sums below are then already density-weighted)
    double vol = 0, fx = 0, fy = 0, fz = 0, s2 = 0;
    const int nv = C.nv;
    const bool gauss = P.dkind == D_GAUSS;
    const double rho = gauss ? 1.0 : P.rho;
    if ( gauss ) integrate_gauss3( C, P, lane, px, py, pz, vol, fx, fy, fz, s2 );
    for ( int k = lane; k < nv && ! gauss; k += 32 ) {
        int e[ 3 ] = { C.va[ k ], C.vb[ k ], C.vc[ k ] };
        double Kx = C.vx[ k ], Ky = C.vy[ k ], Kz = C.vz[ k ];
        for ( int q = 0; q < 3; ++q ) {
            const int f = e[ q ];
            const int t = C.ad[ q ][ k ] == C3::NONE ? -1 : int( C.ad[ q ][ k ] );    // the vertex across edge (f, e[ q + 1 ])
            double a2 = 0;
            if ( t >= 0 ) {
                double Tx = C.vx[ t ], Ty = C.vy[ t ], Tz = C.vz[ t ];
                double nn = C.nx[ f ] * C.nx[ f ] + C.ny[ f ] * C.ny[ f ] + C.nz[ f ] * C.nz[ f ];
                double cf = C.no[ f ] / nn;
                double Cx = C.nx[ f ] * cf, Cy = C.ny[ f ] * cf, Cz = C.nz[ f ] * cf;
                // det( c_f, K, T ) with the sign that makes the box positive
                double det = -( Cx * ( Ky * Tz - Kz * Ty ) - Cy * ( Kx * Tz - Kz * Tx ) + Cz * ( Kx * Ty - Ky * Tx ) );
                double tv = det / 6;
                vol += tv;
                if ( moments ) {
                    fx += tv * ( Cx + Kx + Tx ) / 4;
                    fy += tv * ( Cy + Ky + Ty ) / 4;
                    fz += tv * ( Cz + Kz + Tz ) / 4;
                    s2 += tv / 10 * ( Cx * Cx + Cy * Cy + Cz * Cz + Kx * Kx + Ky * Ky + Kz * Kz + Tx * Tx + Ty * Ty + Tz * Tz +
                                      Cx * Kx + Cy * Ky + Cz * Kz + Cx * Tx + Cy * Ty + Cz * Tz + Kx * Tx + Ky * Ty + Kz * Tz );
                }
                // the area of the face triangle ( c_f, K, T ) along the unit normal
                double ux = Kx - Cx, uy = Ky - Cy, uz = Kz - Cz, vx = Tx - Cx, vy = Ty - Cy, vz = Tz - Cz;
                double cx = uy * vz - uz * vy, cy = uz * vx - ux * vz, cz = ux * vy - uy * vx;
                a2 = -( cx * C.nx[ f ] + cy * C.ny[ f ] + cz * C.nz[ f ] ) / ( 2 * sqrt( nn ) );
            }
            C.area[ 3 * k + q ] = a2;
        }
    }
    __syncwarp();
    double mass = rho * warp_sum( vol );
    if ( ! isfinite( mass ) ) {
        // a clip that lost its topology: never a NaN in the outputs -- an error of the problem (its user seed), an empty
        // cell, no facet (the reference's failure record, gpu/Cell2D.cuh:99-102, 1214-1231)
        if ( lane == 0 ) {
            record_error3( P, err, 7, prob, user, 0 );
            const int row = user_order ? user : s;
            if ( P.mass ) P.mass[ row ] = 0;
            if ( facets ) P.nb[ row ] = 0;
            if ( moments && P.first ) {
                P.first[ 3 * ( size_t ) row ] = user_order ? px : 0.0;
                P.first[ 3 * ( size_t ) row + 1 ] = user_order ? py : 0.0;
                P.first[ 3 * ( size_t ) row + 2 ] = user_order ? pz : 0.0;
            }
            if ( moments && P.cost ) P.cost[ row ] = 0;
        }
        __syncwarp();
        return true;
    }
    // the facets: per plane, its triangles summed in vertex order (first the count, then the writes)
    if ( facets ) {
        const int row = user_order ? user : s;
        int nf = 0;
        for ( int pbase = 0; pbase < C.np; pbase += 32 ) {
            int p = pbase + lane;
            double ar = 0;
            bool seed_plane = p < C.np && C.pid[ p ] >= 0;
            if ( seed_plane ) {
                for ( int k = 0; k < nv; ++k ) {
                    if ( C.va[ k ] == p ) ar += C.area[ 3 * k ];
                    if ( C.vb[ k ] == p ) ar += C.area[ 3 * k + 1 ];
                    if ( C.vc[ k ] == p ) ar += C.area[ 3 * k + 2 ];
                }
                if ( gauss ) ar += C.fmp[ p ];
            }
            if ( p < C.np ) C.par[ p ] = seed_plane && ar > 0 ? ar : 0.0;
            nf += __popc( __ballot_sync( FULL3, seed_plane && ar > 0 ) );
        }
        __syncwarp();
        // more facets than the table's row: the big-cell pass (main kernel), or the overflow store (big-cell pass)
        const bool to_store = nf > P.cap;
        if ( to_store && ! big && ovf ) { queue3( P, err, ovf, prob, s, user, lane ); return false; }
        if ( to_store && ! P.ovf_ids ) {
            if ( lane == 0 ) record_error3( P, err, 4, prob, user, nf );
            return true;
        }
        int base_at = 0;
        if ( to_store ) {
            if ( lane == 0 ) base_at = atomicAdd( P.ovf_count, nf );
            base_at = __shfl_sync( FULL3, base_at, 0 );
            if ( base_at + nf > P.ovf_cap ) {
                if ( lane == 0 ) record_error3( P, err, 4, prob, user, nf );
                return true;
            }
        }
        int written = 0;
        for ( int pbase = 0; pbase < C.np; pbase += 32 ) {
            int p = pbase + lane;
            const double ar = p < C.np ? C.par[ p ] : 0.0;
            const bool fac = ar > 0;
            unsigned fm = __ballot_sync( FULL3, fac );
            int slot = written + __popc( fm & ( ( 1u << lane ) - 1 ) );
            if ( fac ) {
                double dist = sqrt( C.nx[ p ] * C.nx[ p ] + C.ny[ p ] * C.ny[ p ] + C.nz[ p ] * C.nz[ p ] );
                int j = C.pid[ p ];
                const int jid = user_order ? P.user[ j ] : j;
                if ( to_store ) { P.ovf_ids[ base_at + slot ] = jid; P.ovf_c[ base_at + slot ] = rho * ar / ( 2 * dist ); }
                else {
                    size_t at = ( size_t ) row * P.cap + slot;
                    P.nid[ at ] = jid;
                    P.nc[ at ] = rho * ar / ( 2 * dist );
                    if ( P.nm ) P.nm[ at ] = rho * ar;
                }
            }
            written += __popc( fm );
        }
        if ( lane == 0 ) {
            P.nb[ row ] = nf;
            if ( to_store ) P.nid[ ( size_t ) row * P.cap ] = base_at;
        }
    }
    if ( ( flags & F_VJP ) && ! gauss ) {
        // THE ADJOINT of the masses (gpu/Cell3D.cuh:1954-1978), a constant density: grad_w_i = sum_j c_ij ( g_i - g_j ),
        // grad_p_i = sum_j 2 c_ij ( g_i - g_j ) ( x_ij - p_i ), x_ij the facet's centroid -- summed triangle by triangle of
        // the facets, c_f K T, each with its own centroid (no per-facet storage)
        // The first moments F_i = int_cell x rho: with G = gF_i - gF_j, y = x - p_i and the face triangle ( c_f, K, T ) of
        // area a, int y = a ( c_f + K + T ) / 3 and int y y^T = a ( c_f c_f^T + K K^T + T T^T + S S^T ) / 12, S = c_f + K + T:
        // grad_w_i += G . int x rho / 2|p_ij|, grad_p_i += ( ( G . p_i ) int y rho + int y y^T rho G ) / |p_ij|
        const int ui = user_order ? user : s;
        const double gi = P.gm ? P.gm[ ui ] : 0.0;
        const double gfx = P.gf ? P.gf[ 3 * size_t( ui ) ] : 0.0, gfy = P.gf ? P.gf[ 3 * size_t( ui ) + 1 ] : 0.0,
                     gfz = P.gf ? P.gf[ 3 * size_t( ui ) + 2 ] : 0.0;
        double gw = 0, gx = 0, gy = 0, gz = 0;
        for ( int k = lane; k < nv; k += 32 ) {
            const int e[ 3 ] = { C.va[ k ], C.vb[ k ], C.vc[ k ] };
            for ( int q = 0; q < 3; ++q ) {
                const int f = e[ q ], j = C.pid[ f ];
                const double a2 = C.area[ 3 * k + q ];
                if ( j < 0 || a2 == 0 ) continue;
                const int t = C.ad[ q ][ k ];
                if ( t == C3::NONE ) continue;
                const double nn = C.nx[ f ] * C.nx[ f ] + C.ny[ f ] * C.ny[ f ] + C.nz[ f ] * C.nz[ f ];
                const double cf = C.no[ f ] / nn;
                const size_t uj = user_order ? P.user[ j ] : j;
                const double dist = sqrt( nn );
                const double Cx = C.nx[ f ] * cf, Cy = C.ny[ f ] * cf, Cz = C.nz[ f ] * cf;
                const double Sx = Cx + C.vx[ k ] + C.vx[ t ], Sy = Cy + C.vy[ k ] + C.vy[ t ], Sz = Cz + C.vz[ k ] + C.vz[ t ];
                if ( P.gm ) {
                    const double coef = rho * a2 / ( 2 * dist ) * ( gi - P.gm[ uj ] );
                    gw += coef;
                    gx += 2 * coef * Sx / 3;
                    gy += 2 * coef * Sy / 3;
                    gz += 2 * coef * Sz / 3;
                }
                if ( P.gf ) {
                    const double Gx = gfx - P.gf[ 3 * uj ], Gy = gfy - P.gf[ 3 * uj + 1 ], Gz = gfz - P.gf[ 3 * uj + 2 ];
                    const double ra = rho * a2;
                    gw += ( Gx * ( ra * px + ra * Sx / 3 ) + Gy * ( ra * py + ra * Sy / 3 ) + Gz * ( ra * pz + ra * Sz / 3 ) ) / ( 2 * dist );
                    const double Kx = C.vx[ k ], Ky = C.vy[ k ], Kz = C.vz[ k ], Tx = C.vx[ t ], Ty = C.vy[ t ], Tz = C.vz[ t ];
                    const double cg = Cx * Gx + Cy * Gy + Cz * Gz, kg = Kx * Gx + Ky * Gy + Kz * Gz, tg = Tx * Gx + Ty * Gy + Tz * Gz,
                                 sg = Sx * Gx + Sy * Gy + Sz * Gz, pg = px * Gx + py * Gy + pz * Gz;
                    gx += ( pg * ra * Sx / 3 + ra / 12 * ( Cx * cg + Kx * kg + Tx * tg + Sx * sg ) ) / dist;
                    gy += ( pg * ra * Sy / 3 + ra / 12 * ( Cy * cg + Ky * kg + Ty * tg + Sy * sg ) ) / dist;
                    gz += ( pg * ra * Sz / 3 + ra / 12 * ( Cz * cg + Kz * kg + Tz * tg + Sz * sg ) ) / dist;
                }
            }
        }
        gw = warp_sum( gw ); gx = warp_sum( gx ); gy = warp_sum( gy ); gz = warp_sum( gz );
        if ( lane == 0 ) {
            const int row = user_order ? user : s;
            if ( P.gw ) P.gw[ row ] = gw;
            if ( P.gpos ) { P.gpos[ 3 * ( size_t ) row ] = gx; P.gpos[ 3 * ( size_t ) row + 1 ] = gy; P.gpos[ 3 * ( size_t ) row + 2 ] = gz; }
        }
    }
    if ( moments ) {
        double mx = warp_sum( fx ), my = warp_sum( fy ), mz = warp_sum( fz ), ss = warp_sum( s2 );
        double vv = mass / rho;
        if ( lane == 0 ) {
            if ( user_order ) {
                if ( P.first ) {
                    P.first[ 3 * ( size_t ) user ] = vv > 0 ? px + mx / vv : px;
                    P.first[ 3 * ( size_t ) user + 1 ] = vv > 0 ? py + my / vv : py;
                    P.first[ 3 * ( size_t ) user + 2 ] = vv > 0 ? pz + mz / vv : pz;
                }
                if ( P.cost ) P.cost[ user ] = rho * ss;
            } else {
                if ( P.first ) { P.first[ 3 * ( size_t ) s ] = rho * mx; P.first[ 3 * ( size_t ) s + 1 ] = rho * my; P.first[ 3 * ( size_t ) s + 2 ] = rho * mz; }
                if ( P.cost ) P.cost[ s ] = rho * ss;
            }
        }
    }
    if ( lane == 0 && P.mass ) P.mass[ user_order ? user : s ] = mass;
    if ( rep && lane == 0 ) {
        double nu = P.nu[ s ];
        double e2 = fabs( nu - mass );
        rep[ R_WORST ] = fmax( rep[ R_WORST ], e2 );
        rep[ R_WORST_REL ] = fmax( rep[ R_WORST_REL ], e2 / nu );
        rep[ R_AMIN ] = fmin( rep[ R_AMIN ], mass );
        rep[ R_ASUM ] += mass;
        rep[ R_LIN2 ] += ( nu - mass ) * ( nu - mass );
        double x = mass / nu, g = g_of3( x, P.res, P.power );
        double n1 = rep[ R_GCOUNT ] + 1, d = g - rep[ R_GMEAN ];
        rep[ R_GMEAN ] += d / n1;
        rep[ R_GM2 ] += d * ( g - rep[ R_GMEAN ] );
        rep[ R_GCOUNT ] = n1;
        double u = nu / gp_of3( x, P.res, P.power );
        rep[ R_SU ] += u;
        rep[ R_SUG ] += u * g;
        rep[ R_NUSUM ] += nu;
        rep[ R_NEMPTY ] += mass > 0 ? 0.0 : 1.0;
    }
    __syncwarp();
    return true;
}

// THE CELL, both halves
template<bool CNT, class C3>
__device__ bool cell3( C3 &C, const ProbDev &P, int prob, int s, int lane, unsigned flags, ErrRec *err, OvfList *ovf, int2 *stk, double wmax,
                       double *rep, bool big ) {
    if ( ! clip3<CNT>( C, P, prob, s, lane, err, ovf, stk, wmax, big ) ) return false;
    return finish3( C, P, prob, s, lane, flags, err, ovf, rep, big );
}

// ---- the two passes of the gaussian cells -------------------------------------------------------------------------------
// Under a sum of gaussians the integration is most of a cell's work, and one kernel doing both halves keeps the warps of an
// SM in different code (the clip's walk, the quadrature, their math functions) that the instruction cache cannot hold at
// once: the warps then mostly wait for instructions.  So the main kernel runs twice: pass 1 clips every gaussian cell and
// stores it (its used planes and its vertices) in `Split3::mem`; pass 2 loads each one and integrates it.  A cell that
// finds no room in `mem` is done whole by pass 2.  The record of a cell, 16-byte aligned: int nv, np (16 bytes), then
// doubles vx, vy, vz [nv] and nx, ny, nz, no [np], ints pid [np], ushorts va, vb, vc [nv] and the adjacency ad [3][nv].
__device__ __forceinline__ size_t rec3_bytes( int nv, int np ) {
    return ( 16 + size_t( 8 ) * ( 3 * nv + 4 * np ) + size_t( 4 ) * np + size_t( 12 ) * nv + 15 ) & ~size_t( 15 );
}

template<class C3>
__device__ long long store3( C3 &C, const Split3 &sp, int lane ) {
    // only the planes a vertex uses
    compact_planes( C, lane );
    const int nv = C.nv, np = C.np;
    const size_t bytes = rec3_bytes( nv, np );
    unsigned long long at = 0;
    if ( lane == 0 ) at = atomicAdd( sp.used, ( unsigned long long ) bytes );
    at = __shfl_sync( FULL3, at, 0 );
    if ( at + bytes > sp.cap ) return -1;
    char *r = sp.mem + at;
    if ( lane == 0 ) { reinterpret_cast<int *>( r )[ 0 ] = nv; reinterpret_cast<int *>( r )[ 1 ] = np; }
    double *v = reinterpret_cast<double *>( r + 16 ), *pl = v + 3 * nv;
    int *pid = reinterpret_cast<int *>( pl + 4 * np );
    unsigned short *ids = reinterpret_cast<unsigned short *>( pid + np );
    for ( int k = lane; k < nv; k += 32 ) {
        v[ k ] = C.vx[ k ]; v[ nv + k ] = C.vy[ k ]; v[ 2 * nv + k ] = C.vz[ k ];
        ids[ k ] = C.va[ k ]; ids[ nv + k ] = C.vb[ k ]; ids[ 2 * nv + k ] = C.vc[ k ];
        ids[ 3 * nv + k ] = C.ad[ 0 ][ k ] == C3::NONE ? 0xffff : C.ad[ 0 ][ k ];
        ids[ 4 * nv + k ] = C.ad[ 1 ][ k ] == C3::NONE ? 0xffff : C.ad[ 1 ][ k ];
        ids[ 5 * nv + k ] = C.ad[ 2 ][ k ] == C3::NONE ? 0xffff : C.ad[ 2 ][ k ];
    }
    for ( int p = lane; p < np; p += 32 ) {
        pl[ p ] = C.nx[ p ]; pl[ np + p ] = C.ny[ p ]; pl[ 2 * np + p ] = C.nz[ p ]; pl[ 3 * np + p ] = C.no[ p ];
        pid[ p ] = C.pid[ p ];
    }
    return ( long long ) at;
}

template<class C3>
__device__ void load3( C3 &C, const Split3 &sp, long long at, int lane ) {
    const char *r = sp.mem + at;
    const int nv = reinterpret_cast<const int *>( r )[ 0 ], np = reinterpret_cast<const int *>( r )[ 1 ];
    const double *v = reinterpret_cast<const double *>( r + 16 ), *pl = v + 3 * nv;
    const int *pid = reinterpret_cast<const int *>( pl + 4 * np );
    const unsigned short *ids = reinterpret_cast<const unsigned short *>( pid + np );
    typedef typename C3::I I;
    for ( int k = lane; k < nv; k += 32 ) {
        C.vx[ k ] = v[ k ]; C.vy[ k ] = v[ nv + k ]; C.vz[ k ] = v[ 2 * nv + k ];
        C.va[ k ] = I( ids[ k ] ); C.vb[ k ] = I( ids[ nv + k ] ); C.vc[ k ] = I( ids[ 2 * nv + k ] );
        for ( int q = 0; q < 3; ++q ) {
            const unsigned short t = ids[ ( 3 + q ) * nv + k ];
            C.ad[ q ][ k ] = t == 0xffff ? I( C3::NONE ) : I( t );
        }
    }
    for ( int p = lane; p < np; p += 32 ) {
        C.nx[ p ] = pl[ p ]; C.ny[ p ] = pl[ np + p ]; C.nz[ p ] = pl[ 2 * np + p ]; C.no[ p ] = pl[ 3 * np + p ];
        C.pid[ p ] = pid[ p ];
    }
    if ( lane == 0 ) { C.nv = nv; C.np = np; }
    __syncwarp();
}

// the main kernel: one warp per cell, W3 cells of a chunk at a time.  mode 0: every cell whole.  mode 1 (pass 1) and
// mode 2 (pass 2): the cells of a gaussian problem are clipped and stored by pass 1 and integrated by pass 2 (the report
// too); the other problems are done whole by pass 1 and skipped by pass 2.  (The warps' cells, about 55 KB of shared
// memory a block, hold 4 blocks on an SM: the registers are bounded for 4, not more.)
template<bool CNT>
__global__ void __launch_bounds__( 32 * W3, 4 ) k_cells3d( const ProbDev *__restrict__ probs, const Chunk *__restrict__ chunks, int nchunks,
                                                        unsigned flags, ErrRec *err, OvfList *ovf, int mode, Split3 sp ) {
    extern __shared__ char smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    Cell3 &C = reinterpret_cast<Cell3 *>( smem )[ warp ];
    __shared__ double sh_rep[ W3 ][ NB_REPORT ];
    __shared__ int2 sh_stk[ W3 ][ WALK_STACK3 ];
    __shared__ int sh_last;
    for ( int cidx = blockIdx.x; cidx < nchunks; cidx += gridDim.x ) {
        const Chunk ch = chunks[ cidx ];
        const ProbDev &P = probs[ ch.prob ];
        const bool two = mode != 0 && P.dkind == D_GAUSS;       // block-uniform: one problem per chunk
        if ( mode == 2 && ! two ) continue;
        const bool report = ( flags & F_REPORT ) && ! ( mode == 1 && two );
        double rep[ NB_REPORT ];
        rep[ R_WORST ] = 0; rep[ R_WORST_REL ] = 0; rep[ R_AMIN ] = 1e300; rep[ R_ASUM ] = 0; rep[ R_LIN2 ] = 0; rep[ R_GCOUNT ] = 0;
        rep[ R_GMEAN ] = 0; rep[ R_GM2 ] = 0; rep[ R_SU ] = 0; rep[ R_SUG ] = 0; rep[ R_NUSUM ] = 0; rep[ R_NEMPTY ] = 0;
        double *rp = report ? rep : nullptr;
        const double wmax = P.wmax_slot ? order_dbl( *P.wmax_slot ) : 0.0;
        for ( int s = ch.begin + warp; s < ch.end; s += W3 ) {
            if ( ! two ) {
                cell3<CNT>( C, P, ch.prob, s, lane, flags, err, ovf, sh_stk[ warp ], wmax, rp, false );
                continue;
            }
            long long *slot = sp.slot + ( size_t ) cidx * CHUNK + ( s - ch.begin );
            if ( mode == 1 ) {
                long long at = -2;                  // queued for the big-cell pass
                if ( clip3<CNT>( C, P, ch.prob, s, lane, err, ovf, sh_stk[ warp ], wmax, false ) ) at = store3( C, sp, lane );
                if ( lane == 0 ) *slot = at;
                __syncwarp();
            } else {
                const long long at = *slot;
                if ( at >= 0 ) {
                    load3( C, sp, at, lane );
                    finish3( C, P, ch.prob, s, lane, flags, err, ovf, rp, false );
                } else if ( at == -1 )              // no room in pass 1: the whole cell here
                    cell3<CNT>( C, P, ch.prob, s, lane, flags, err, ovf, sh_stk[ warp ], wmax, rp, false );
            }
        }
        if ( report ) {
            // the chunk's report, then the last block of the problem folds them (fixed tree)
            if ( lane == 0 ) for ( int k = 0; k < NB_REPORT; ++k ) sh_rep[ warp ][ k ] = rep[ k ];
            __syncthreads();
            if ( threadIdx.x == 0 ) {
                Rep r;
                for ( int k = 0; k < NB_REPORT; ++k ) r.v[ k ] = sh_rep[ 0 ][ k ];
                for ( int w = 1; w < W3; ++w ) r.combine( sh_rep[ w ] );
                double *dst = P.partials + ( size_t ) ch.index * NB_REPORT;
                for ( int k = 0; k < NB_REPORT; ++k ) dst[ k ] = r.v[ k ];
                __threadfence();
                unsigned prev = atomicAdd( P.counter, 1u );
                sh_last = prev == unsigned( P.nchunk - 1 );
            }
            __syncthreads();
            if ( sh_last ) {
                __threadfence();
                fold_reports_block<W3>( P );
            }
            __syncthreads();
        }
    }
}


// the big-cell pass: one warp a block, the cell in dynamic shared memory (Cell3B), over the queued 3D items (the 2D ones
// are the 2D pass's); flags 0: each problem's own pass (a final-moments diagram has `first`)
__global__ void __launch_bounds__( 32 ) k_cells3d_big( const ProbDev *__restrict__ probs, const OvfList *__restrict__ ovf, int count,
                                                        unsigned flags, ErrRec *err, OvfList *next ) {
    extern __shared__ char smem[];
    __shared__ int2 stk[ WALK_STACK3 ];
    Cell3B &C = *reinterpret_cast<Cell3B *>( smem );
    const int lane = threadIdx.x;
    for ( int it = blockIdx.x; it < count; it += gridDim.x ) {
        const OvfItem item = ovf->items[ it ];
        const ProbDev &P = probs[ item.prob ];
        if ( P.dim != 3 ) continue;
        const unsigned fl = flags ? flags : ( P.first ? ( F_MOMENTS | F_USER_ORDER ) : ( F_MASS | F_FACETS ) );
        const double wmax = P.wmax_slot ? order_dbl( *P.wmax_slot ) : 0.0;
        cell3<false>( C, P, item.prob, item.seed, lane, fl, err, next, stk, wmax, nullptr, true );
    }
}

// the giant-cell pass: the cells past the big pass's capacities (hundreds of faces: a seed in a density desert whose cell
// reaches across a dense cluster), one warp a block, each block's cell in its slot of `scratch` (global memory, L2-backed)
__global__ void __launch_bounds__( 32 ) k_cells3d_giant( const ProbDev *__restrict__ probs, const OvfList *__restrict__ list, int count,
                                                          unsigned flags, ErrRec *err, char *scratch ) {
    __shared__ int2 stk[ WALK_STACK3 ];
    Cell3G &C = *reinterpret_cast<Cell3G *>( scratch + size_t( blockIdx.x ) * sizeof( Cell3G ) );
    const int lane = threadIdx.x;
    for ( int it = blockIdx.x; it < count; it += gridDim.x ) {
        const OvfItem item = list->items[ it ];
        const ProbDev &P = probs[ item.prob ];
        if ( P.dim != 3 ) continue;
        const unsigned fl = flags ? flags : ( P.first ? ( F_MOMENTS | F_USER_ORDER ) : ( F_MASS | F_FACETS ) );
        const double wmax = P.wmax_slot ? order_dbl( *P.wmax_slot ) : 0.0;
        cell3<false>( C, P, item.prob, item.seed, lane, fl, err, nullptr, stk, wmax, nullptr, true );
    }
}

size_t giant3_slot_bytes() { return ( sizeof( Cell3G ) + 255 ) & ~size_t( 255 ); }

void launch_cells3d_giant( const Launch &L, const ProbDev *probs, const OvfList *list, int count, unsigned flags, ErrRec *err, char *scratch,
                           int slots ) {
    if ( count <= 0 ) return;
    static_assert( sizeof( Cell3G ) % 8 == 0, "slots keep the doubles aligned" );
    k_cells3d_giant<<<count < slots ? count : slots, 32, 0, L.stream>>>( probs, list, count, flags, err, scratch );
    ++*L.launches;
}

// four blocks of the main kernel on an SM (its static shared memory is under 4 KB; 1 KB a block is the system's)
static_assert( 4 * ( W3 * sizeof( Cell3 ) + 4096 + 1024 ) <= 228 * 1024, "the main 3D kernel keeps four blocks on an SM" );

void launch_cells3d( const Launch &L, const ProbDev *probs, const Chunk *chunks, int nchunks, unsigned flags, ErrRec *err, OvfList *ovf,
                     const Split3 *sp ) {
    if ( nchunks <= 0 ) return;
    const size_t smem = sizeof( Cell3 ) * W3;
    static bool configured = false;
    if ( ! configured ) {
        for ( auto k : { k_cells3d<false>, k_cells3d<true> } ) {
            cudaFuncSetAttribute( k, cudaFuncAttributeMaxDynamicSharedMemorySize, int( smem ) );
            cudaFuncSetAttribute( k, cudaFuncAttributePreferredSharedMemoryCarveout, 100 );
        }
        configured = true;
    }
    // the counting instantiation only when the search's reads are counted (F_GATHER): the other compiles without them
    auto *kern = ( flags & F_GATHER ) ? k_cells3d<true> : k_cells3d<false>;
    if ( ! sp ) {
        kern<<<nchunks, 32 * W3, smem, L.stream>>>( probs, chunks, nchunks, flags, err, ovf, 0, Split3{} );
        ++*L.launches;
        return;
    }
    cudaMemsetAsync( sp->used, 0, sizeof( unsigned long long ), L.stream );
    kern<<<nchunks, 32 * W3, smem, L.stream>>>( probs, chunks, nchunks, flags, err, ovf, 1, *sp );
    kern<<<nchunks, 32 * W3, smem, L.stream>>>( probs, chunks, nchunks, flags, err, ovf, 2, *sp );
    *L.launches += 2;
}

void launch_cells3d_big( const Launch &L, const ProbDev *probs, const OvfList *ovf, int count, unsigned flags, ErrRec *err, OvfList *next ) {
    if ( count <= 0 ) return;
    const size_t smem = sizeof( Cell3B );
    static bool configured = false;
    if ( ! configured ) {
        cudaFuncSetAttribute( k_cells3d_big, cudaFuncAttributeMaxDynamicSharedMemorySize, int( smem ) );
        configured = true;
    }
    k_cells3d_big<<<count < 296 ? count : 296, 32, smem, L.stream>>>( probs, ovf, count, flags, err, next );
    ++*L.launches;
}

} // namespace sdot

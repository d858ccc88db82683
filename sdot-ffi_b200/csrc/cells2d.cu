// 2D Laguerre cells: ONE WARP PER CELL.
//
// The cell of seed i is the domain box clipped by the power bisectors of its neighbours.  It is held
// across the warp: lane k owns vertex k (FP64, in the frame of the seed) and the line of edge k -> k+1
// (`n . y <= off` with its cut id: a seed rank >= 0, or a box side -1 bottom, -2 right, -3 top,
// -4 left -- the conventions of src/sdot/include/sdot/gpu/Cell2D.cuh:453-463).  A cut is a ballot of
// the vertices outside, two line-line intersections and one shuffle permutation; every vertex is
// always the intersection of its two lines, so no error accumulates along the cuts (the reference
// re-solves its float vertices in FP64 for the same reason, Cell2D.cuh:991-1042).
//
// Candidates come from the Morton grid, ring by ring around the seed's grid cell; 32 candidates are
// loaded at a time and pre-tested in parallel (lane l tests candidate l against every vertex), so only
// the candidates that do cut go through the serial clip.  The walk stops by the SECURITY RADIUS: every
// unvisited seed q is at least `r h` away, and cannot cut the cell once
//     r h >= R + sqrt( max( 0, R^2 + w_max - w_i ) ),    R = max_k |v_k|.
//
// Integration is a warp reduction over the edges: the shoelace terms for a constant density; for an
// image, Green's theorem on rows (mass = closed integral of F dy, F = int rho dx, the edges walked pixel
// by pixel from row prefix sums, cf. gpu/Density2D.cuh:16-26 for the reference's use of the same
// identity); for gaussians the same identity with F in closed form (erf), Gauss-Legendre along the edge.
#include "internal.h"

namespace sdot {

constexpr unsigned FULL = 0xffffffffu;

// ---- the density along one edge (seed frame) ------------------------------------------------------------
struct EdgeInt {
    double m, fx, fy, s2, meas, mx, my;   // mass, first moments, second moment, int_edge rho, int_edge x rho
};

// the point of line 1 ( a1 x + b1 y = c1 ) on line 2, found ALONG line 1: from its foot, by the step that line 2's
// equation asks for.  The result lies on line 1 to rounding and on line 2 to rounding, however close to parallel the
// lines are -- Cramer's rule would leave it off both by eps / sin(angle): seeds 1e-10 apart make two bisectors 1e-8
// rad apart, whose crossing Cramer placed 1e-10 off the lines (1e-12 of a cell's mass)
__device__ __forceinline__ void isect( double a1, double b1, double c1, double a2, double b2, double c2, double &x, double &y, bool &ok ) {
    const double det = a1 * b2 - a2 * b1;
    const double sc = ( fabs( a1 ) + fabs( b1 ) ) * ( fabs( a2 ) + fabs( b2 ) );
    ok = fabs( det ) > 1e-13 * sc;
    const double k = c1 / ( a1 * a1 + b1 * b1 ), fx = k * a1, fy = k * b1;       // the foot of line 1
    const double t = ( c2 - ( a2 * fx + b2 * fy ) ) / det;                       // along ( -b1, a1 )
    x = fx - t * b1;
    y = fy + t * a1;
}

// uniform density: the shoelace terms of the edge (x0,y0)->(x1,y1)
__device__ __forceinline__ void edge_uniform( double x0, double y0, double x1, double y1, double rho, bool moments, EdgeInt &e ) {
    double c = x0 * y1 - x1 * y0;
    e.m = rho * c * 0.5;
    if ( moments ) {
        e.fx = rho * ( x0 + x1 ) * c / 6;
        e.fy = rho * ( y0 + y1 ) * c / 6;
        e.s2 = rho * c * ( x0 * x0 + x0 * x1 + x1 * x1 + y0 * y0 + y0 * y1 + y1 * y1 ) / 12;
    }
    double len = sqrt( ( x1 - x0 ) * ( x1 - x0 ) + ( y1 - y0 ) * ( y1 - y0 ) );
    e.meas = rho * len;
    e.mx = rho * len * 0.5 * ( x0 + x1 );
    e.my = rho * len * 0.5 * ( y0 + y1 );
}

// image: F(x, y) = int_{X_ref}^{x} rho(t, y) dt along each piece of the edge inside one pixel
__device__ __noinline__ void edge_image( const ProbDev &P, double px, double py, int iref, double x0, double y0, double x1, double y1, bool moments,
                            EdgeInt &e ) {
    const int nx = P.dn[ 0 ], ny = P.dn[ 1 ];
    const double hx = P.dstep[ 0 ], hy = P.dstep[ 1 ];
    const double X0 = P.dorg[ 0 ] - px, Y0 = P.dorg[ 1 ] - py;      // pixel (0, 0) corner, seed frame
    double dx = x1 - x0, dy = y1 - y0;
    double len = sqrt( dx * dx + dy * dy );
    e.m = e.fx = e.fy = e.s2 = e.meas = e.mx = e.my = 0;
    if ( len == 0 ) return;
    // next crossing parameters of the vertical / horizontal pixel lines
    double tx = 2, ty = 2, stx = 0, sty = 0;
    int kx = 0, ky = 0, ddx = 0, ddy = 0;
    if ( dx != 0 ) {
        double f = ( x0 - X0 ) / hx;
        kx = dx > 0 ? int( floor( f ) ) + 1 : int( ceil( f ) ) - 1;
        ddx = dx > 0 ? 1 : -1;
        tx = ( X0 + kx * hx - x0 ) / dx;
        stx = hx / fabs( dx );
    }
    if ( dy != 0 ) {
        double f = ( y0 - Y0 ) / hy;
        ky = dy > 0 ? int( floor( f ) ) + 1 : int( ceil( f ) ) - 1;
        ddy = dy > 0 ? 1 : -1;
        ty = ( Y0 + ky * hy - y0 ) / dy;
        sty = hy / fabs( dy );
    }
    const double *pre = P.dpre;
    const int irc = iref < 0 ? 0 : ( iref > nx ? nx : iref );
    double t0 = 0;
    for ( int guard = 0; guard < 4 * ( nx + ny ) + 8; ++guard ) {
        double t1 = fmin( 1.0, fmin( tx, ty ) );
        if ( t1 > t0 ) {
            double tm = 0.5 * ( t0 + t1 );
            int i = int( floor( ( x0 + tm * dx - X0 ) / hx ) ), j = int( floor( ( y0 + tm * dy - Y0 ) / hy ) );
            if ( j >= 0 && j < ny ) {
                double xa = x0 + t0 * dx, ya = y0 + t0 * dy, xb = x0 + t1 * dx, yb = y0 + t1 * dy;
                double v = ( i >= 0 && i < nx ) ? P.dval[ ( size_t ) i * ny + j ] : 0.0;
                int ic = i < 0 ? 0 : ( i > nx ? nx : i );
                const double *row = pre + ( size_t ) j * ( nx + 1 );
                double Xi = X0 + i * hx;
                double C = row[ ic ] - row[ irc ];                   // int_{X_ref}^{X_i} rho
                double Fa = C + v * ( xa - Xi ), Fb = C + v * ( xb - Xi );
                double Dy = yb - ya;
                e.m += Dy * 0.5 * ( Fa + Fb );
                double pl = ( t1 - t0 ) * len;
                e.meas += v * pl;
                e.mx += v * pl * 0.5 * ( xa + xb );
                e.my += v * pl * 0.5 * ( ya + yb );
                if ( moments ) {
                    // G = int_{X_ref}^{x} t rho dt and H = int t^2 rho dt (seed frame), prefixes summed locally
                    double Cg = 0, Ch = 0;
                    int lo = i < iref ? i : iref, hi = i < iref ? iref : i;
                    for ( int k = lo; k < hi; ++k ) {
                        double vk = ( k >= 0 && k < nx ) ? P.dval[ ( size_t ) k * ny + j ] : 0.0;
                        double a = X0 + k * hx, b = a + hx;
                        Cg += vk * ( b * b - a * a ) * 0.5;
                        Ch += vk * ( b * b * b - a * a * a ) / 3;
                    }
                    if ( i < iref ) { Cg = -Cg; Ch = -Ch; }
                    e.fx += Dy * ( Cg - v * Xi * Xi * 0.5 + v * ( xa * xa + xa * xb + xb * xb ) / 6 );
                    e.fy += Dy * ( Fa * ( 2 * ya + yb ) + Fb * ( ya + 2 * yb ) ) / 6;
                    e.s2 += Dy * ( Ch - v * Xi * Xi * Xi / 3 + v * ( xa * xa * xa + xa * xa * xb + xa * xb * xb + xb * xb * xb ) / 12 );
                    e.s2 += Dy * ( Fa * ( 3 * ya * ya + 2 * ya * yb + yb * yb ) + Fb * ( ya * ya + 2 * ya * yb + 3 * yb * yb ) ) / 12;
                }
            }
        }
        if ( t1 >= 1.0 ) break;
        t0 = t1;
        if ( tx <= ty ) { tx += stx; kx += ddx; } else { ty += sty; ky += ddy; }
    }
}

// gaussians: F(x, y) = int_{0}^{x} g(t, y) dt (seed frame, reference at the seed), Gauss-Legendre along the edge
__constant__ double c_glx[ 8 ] = { -0.9602898564975363, -0.7966664774136267, -0.5255324099163290, -0.1834346424956498,
                                    0.1834346424956498, 0.5255324099163290, 0.7966664774136267, 0.9602898564975363 };
__constant__ double c_glw[ 8 ] = { 0.1012285362903763, 0.2223810344533745, 0.3137066458778873, 0.3626837833783620,
                                    0.3626837833783620, 0.3137066458778873, 0.2223810344533745, 0.1012285362903763 };

// erf( u ) - erf( u0 ) without cancellation in the tails, with the u0 terms of an edge computed once:
// c0 = erfc( |u0| ), f0 = erf( |u0| ); one erf or erfc per call
__device__ __forceinline__ double erf_from( double u0, double c0, double f0, double u ) {
    if ( u0 >= 0 && u >= 0 ) return c0 - erfc( u );
    if ( u0 <= 0 && u <= 0 ) return erfc( -u ) - c0;
    return u > 0 ? erf( u ) + f0 : -( erf( -u ) + f0 );
}
__device__ __forceinline__ double erf_diff( double a, double b ) {
    if ( a >= 0 && b >= 0 ) return erfc( a ) - erfc( b );
    if ( a <= 0 && b <= 0 ) return erfc( -b ) - erfc( -a );
    return erf( b ) - erf( a );
}

// gaussian g's part of the edge (x0,y0)->(x1,y1), ADDED to e
__device__ __noinline__ void edge_gauss_one( const ProbDev &P, int g, double px, double py, double x0, double y0, double x1, double y1,
                                             bool moments, bool measures, EdgeInt &e ) {
    double dx = x1 - x0, dy = y1 - y0, len = sqrt( dx * dx + dy * dy );
    if ( len == 0 ) return;
    const double r2 = 1.4142135623730951;
    {
        const double *G = P.dval + g * 4;
        double cx = G[ 0 ] - px, cy = G[ 1 ] - py, sg = G[ 2 ], mg = G[ 3 ];
        double K = mg / ( 2 * M_PI * sg * sg ), s2g = sg * sg, sq = sg * r2;
        double E0 = sg * 1.2533141373155003;              // sigma sqrt( pi / 2 )
        if ( measures ) {
            // the facet measure: closed form
            double ux = dx / len, uy = dy / len;
            double sa = ( x0 - cx ) * ux + ( y0 - cy ) * uy, sb = sa + len;
            double fx = x0 - sa * ux - cx, fy = y0 - sa * uy - cy;
            double h2 = fx * fx + fy * fy;
            double span = erf_diff( sa / sq, sb / sq );
            double mm = K * exp( -h2 / ( 2 * s2g ) ) * E0 * span;
            e.meas += mm;
            // int_edge x rho ds: x = x0 + ux ( s - sa ); int s g ds closed form
            double ea = exp( -sa * sa / ( 2 * s2g ) ), eb = exp( -sb * sb / ( 2 * s2g ) );
            double ms = K * exp( -h2 / ( 2 * s2g ) ) * s2g * ( ea - eb );     // int s g ds
            e.mx += ( x0 - ux * sa ) * mm + ux * ms;
            e.my += ( y0 - uy * sa ) * mm + uy * ms;
        }
        if ( dy == 0 ) return;                             // no part in the closed integral of F dy
        double u0 = ( 0 - cx ) / sq;                       // reference abscissa: the seed
        double e0 = exp( -( cx * cx ) / ( 2 * s2g ) );
        double c0 = erfc( fabs( u0 ) ), f0 = erf( fabs( u0 ) );
        // the closed integral, split so that each piece spans at most one sigma
        int np = int( len / sg ) + 1;
        if ( np > 64 ) np = 64;
        for ( int p = 0; p < np; ++p ) {
            double ta = double( p ) / np, tb = double( p + 1 ) / np;
            double xa = x0 + ta * dx, ya = y0 + ta * dy, xb = x0 + tb * dx, yb = y0 + tb * dy;
            double Dy = yb - ya;
            double am = 0, afx = 0, afy = 0, as2 = 0;
            for ( int q = 0; q < 8; ++q ) {
                double t = 0.5 + 0.5 * c_glx[ q ], wq = 0.5 * c_glw[ q ];
                double x = xa + t * ( xb - xa ), y = ya + t * ( yb - ya );
                double ey = K * exp( -( y - cy ) * ( y - cy ) / ( 2 * s2g ) );
                double u = ( x - cx ) / sq;
                double D = erf_from( u0, c0, f0, u );
                double F = ey * E0 * D;
                am += wq * F;
                if ( moments ) {
                    double ex = exp( -( x - cx ) * ( x - cx ) / ( 2 * s2g ) );
                    // int_0^x t g dt = cx F - sigma^2 ey ( ex - e0 )
                    double F1 = cx * F - s2g * ey * ( ex - e0 );
                    // int_0^x t^2 g dt, with t = ( t - cx ) + cx
                    double A = ey * ( s2g * E0 * D - s2g * ( ( x - cx ) * ex - ( 0 - cx ) * e0 ) );
                    double F2 = A + 2 * cx * ( -s2g * ey * ( ex - e0 ) ) + cx * cx * F;
                    afx += wq * F1;
                    afy += wq * y * F;
                    as2 += wq * ( F2 + y * y * F );
                }
            }
            e.m += Dy * am;
            if ( moments ) { e.fx += Dy * afx; e.fy += Dy * afy; e.s2 += Dy * as2; }
        }
    }
}

// every gaussian's part of the edge, in gaussian order
__device__ void edge_gauss( const ProbDev &P, double px, double py, double x0, double y0, double x1, double y1, bool moments, bool measures,
                            EdgeInt &e ) {
    e.m = e.fx = e.fy = e.s2 = e.meas = e.mx = e.my = 0;
    for ( int g = 0; g < P.dn[ 0 ]; ++g ) edge_gauss_one( P, g, px, py, x0, y0, x1, y1, moments, measures, e );
}

// a warp's polygon (m edges, vertex `lane` in (vx, vy)) under a sum of gaussians: the (edge, gaussian) pairs spread over the
// lanes -- lane t takes the pairs t, t + 32, ..., edge t % m and gaussian t / m -- so that a cell of 6 edges keeps 24
// lanes busy, not 6.  `e` of each lane: its pairs' part of the cell integrals (summed over the warp by the caller), and
// for lane < m the facet measure and moments of edge `lane`, its gaussians summed in order (as edge_gauss does)
__device__ void warp_edges_gauss( const ProbDev &P, int m, int lane, double vx, double vy, double px, double py, bool moments, bool measures,
                                  EdgeInt &e ) {
    e.m = e.fx = e.fy = e.s2 = e.meas = e.mx = e.my = 0;
    const int ng = P.dn[ 0 ], pairs = m * ng;
    for ( int r = 0; r * 32 < pairs; ++r ) {
        const int t = lane + 32 * r;
        const int ed = t < pairs ? t % m : 0, g = t < pairs ? t / m : 0;
        const int nx = ed + 1 >= m ? 0 : ed + 1;
        const double x0 = __shfl_sync( FULL, vx, ed ), y0 = __shfl_sync( FULL, vy, ed );
        const double x1 = __shfl_sync( FULL, vx, nx ), y1 = __shfl_sync( FULL, vy, nx );
        EdgeInt ep;
        ep.m = ep.fx = ep.fy = ep.s2 = ep.meas = ep.mx = ep.my = 0;
        if ( t < pairs ) edge_gauss_one( P, g, px, py, x0, y0, x1, y1, moments, measures, ep );
        e.m += ep.m;
        e.fx += ep.fx; e.fy += ep.fy; e.s2 += ep.s2;
        if ( ! measures ) continue;
        for ( int q = 0; q < ng; ++q ) {
            const int src = lane + m * q - 32 * r;         // the pair ( edge lane, gaussian q ) in this round
            const bool own = lane < m && src >= 0 && src < 32;
            const double a = __shfl_sync( FULL, ep.meas, own ? src : 0 );
            const double b = __shfl_sync( FULL, ep.mx, own ? src : 0 );
            const double c = __shfl_sync( FULL, ep.my, own ? src : 0 );
            if ( own ) { e.meas += a; e.mx += b; e.my += c; }
        }
    }
}

// ---- the warp-held polygon ----------------------------------------------------------------------------------
struct WPoly {
    int m;                     // vertex count (warp uniform)
    double vx, vy;             // vertex `lane`
    double lnx, lny, loff;     // line of edge lane -> lane + 1
    int lid;
    static constexpr double R2_MARGIN = 1, CLAIM_REL = 1e-12;    // (the security tests on the vertices: exact)
};

// keep n . y <= off; false past 32 vertices
__device__ __forceinline__ bool wclip( WPoly &C, int lane, double nx, double ny, double off, int id ) {
    const int m = C.m;
    double s = nx * C.vx + ny * C.vy - off;
    unsigned out = __ballot_sync( FULL, lane < m && s > 0 );
    if ( ! out ) return true;
    unsigned valid = m >= 32 ? FULL : ( ( 1u << m ) - 1 );
    if ( out == valid ) { C.m = 0; return true; }
    unsigned in = valid & ~out;
    unsigned rot_out = ( ( out >> 1 ) | ( out << ( m - 1 ) ) ) & valid;
    unsigned rot_in = ( ( in >> 1 ) | ( in << ( m - 1 ) ) ) & valid;
    unsigned A = in & rot_out, B = out & rot_in;
    int a, b;
    if ( __popc( A ) == 1 ) {
        a = __ffs( A ) - 1;
        b = __ffs( B ) - 1;
    } else {
        // several outside runs: rounding near a vertex where many lines meet.  The run holding the most outside
        // vertex is the real one; the others (noise-level) are kept
        double sv = lane < m ? s : -1e300;
        double smax = warp_max( sv );
        int kstar = __ffs( __ballot_sync( FULL, lane < m && sv == smax ) ) - 1;
        int da = ( A >> lane ) & 1 ? ( ( kstar - lane ) % m + m ) % m : 1 << 20;       // a: the in->out edge before kstar
        int db = ( B >> lane ) & 1 ? ( ( lane - kstar ) % m + m ) % m : 1 << 20;       // b: the out->in edge from kstar on
        for ( int o = 16; o > 0; o >>= 1 ) { da = min( da, __shfl_xor_sync( FULL, da, o ) ); db = min( db, __shfl_xor_sync( FULL, db, o ) ); }
        a = ( ( kstar - da ) % m + m ) % m;
        b = ( kstar + db ) % m;
    }
    int K = ( ( a - b - 1 ) % m + m ) % m + 1;
    if ( K + 2 > 32 ) return false;
    // the new vertices: line[a] ^ L and L ^ line[b]; near-parallel lines fall back on the edge interpolation
    int a1 = a + 1 == m ? 0 : a + 1, b1 = b + 1 == m ? 0 : b + 1;
    double anx = __shfl_sync( FULL, C.lnx, a ), any = __shfl_sync( FULL, C.lny, a ), aoff = __shfl_sync( FULL, C.loff, a );
    double bnx = __shfl_sync( FULL, C.lnx, b ), bny = __shfl_sync( FULL, C.lny, b ), boff = __shfl_sync( FULL, C.loff, b );
    int bid = __shfl_sync( FULL, C.lid, b );
    double Px, Py, Qx, Qy;
    bool okP, okQ;
    isect( anx, any, aoff, nx, ny, off, Px, Py, okP );
    isect( nx, ny, off, bnx, bny, boff, Qx, Qy, okQ );
    // (okP, okQ are warp uniform: the edges' end points are fetched only for the rare near-parallel fallback)
    if ( ! okP ) {
        double xa = __shfl_sync( FULL, C.vx, a ), ya = __shfl_sync( FULL, C.vy, a ), sa = __shfl_sync( FULL, s, a );
        double xa1 = __shfl_sync( FULL, C.vx, a1 ), ya1 = __shfl_sync( FULL, C.vy, a1 ), sa1 = __shfl_sync( FULL, s, a1 );
        double t = sa / ( sa - sa1 );
        Px = xa + t * ( xa1 - xa ); Py = ya + t * ( ya1 - ya );
    }
    if ( ! okQ ) {
        double xb = __shfl_sync( FULL, C.vx, b ), yb = __shfl_sync( FULL, C.vy, b ), sb = __shfl_sync( FULL, s, b );
        double xb1 = __shfl_sync( FULL, C.vx, b1 ), yb1 = __shfl_sync( FULL, C.vy, b1 ), sb1 = __shfl_sync( FULL, s, b1 );
        double t = sb / ( sb - sb1 );
        Qx = xb + t * ( xb1 - xb ); Qy = yb + t * ( yb1 - yb );
    }
    int src = ( b + 1 + lane ) % m;
    double nvx = __shfl_sync( FULL, C.vx, src ), nvy = __shfl_sync( FULL, C.vy, src );
    double nlx = __shfl_sync( FULL, C.lnx, src ), nly = __shfl_sync( FULL, C.lny, src ), nlo = __shfl_sync( FULL, C.loff, src );
    int nli = __shfl_sync( FULL, C.lid, src );
    if ( lane == K ) { nvx = Px; nvy = Py; nlx = nx; nly = ny; nlo = off; nli = id; }
    if ( lane == K + 1 ) { nvx = Qx; nvy = Qy; nlx = bnx; nly = bny; nlo = boff; nli = bid; }
    C.vx = nvx; C.vy = nvy; C.lnx = nlx; C.lny = nly; C.loff = nlo; C.lid = nli;
    C.m = K + 2;
    return true;
}

__device__ __forceinline__ void ring_offset( int r, int ci, int &dx, int &dy ) {
    if ( r == 0 ) { dx = dy = 0; return; }
    int side = ci / ( 2 * r ), t = ci % ( 2 * r );
    if ( side == 0 ) { dx = -r + t; dy = -r; }
    else if ( side == 1 ) { dx = r; dy = -r + t; }
    else if ( side == 2 ) { dx = r - t; dy = r; }
    else { dx = -r; dy = r - t; }
}

// may a seed of weight at most W, whose nearest possible position is sqrt( d2 ) away, cut a cell of squared radius R2
// around a seed of weight wi?  Its bisector is ( |q|^2 + wi - wj ) / ( 2 |q| ) from the seed: it reaches the cell's
// ball only if |q| < R + sqrt( R^2 + wj - wi ).  W < -1e299: an empty cell or block
__device__ __forceinline__ bool may_cut( double d2, double W, double R2, double wi ) {
    if ( W < -1e299 ) return false;
    double ex = R2 + W - wi, rb = sqrt( R2 ) + sqrt( ex > 0 ? ex : 0.0 );
    return d2 < rb * rb;
}

// squared distance from ( px, py ) to the grid cells [ x0, x1 ] x [ y0, y1 ] (inclusive)
__device__ __forceinline__ double cells_dist2( const ProbDev &P, int x0, int x1, int y0, int y1, double px, double py ) {
    double bx0 = P.go[ 0 ] + x0 * P.gh[ 0 ], bx1 = P.go[ 0 ] + ( x1 + 1 ) * P.gh[ 0 ];
    double by0 = P.go[ 1 ] + y0 * P.gh[ 1 ], by1 = P.go[ 1 ] + ( y1 + 1 ) * P.gh[ 1 ];
    double dx = fmax( 0.0, fmax( bx0 - px, px - bx1 ) ), dy = fmax( 0.0, fmax( by0 - py, py - by1 ) );
    return dx * dx + dy * dy;
}

constexpr int WALK_STACK = 64;       // pyramid walk: at most 3 entries per level stay on the stack (16 levels in 2D)
constexpr int RINGS_FIRST = 2;       // rings walked before the pyramid takes over
constexpr int WALK_LEAF = 1;         // the walk's leaves: blocks of 2 x 2 grid cells, one cell per lane (4 x 4 leaves: 8 % slower)

// The pyramid of weight majorants walked depth first, nearest child first, skipping the cells within Chebyshev
// distance rd of ( cx, cy ) (the rings already walked) and every block that claims no vertex of the current cell
// (`claims( lo, hi, a, b )`, warp-uniform).  At a leaf block, lane k holds the seed range of its k-th cell (empty if
// `may_cut` rules it out) and `cut( beg, cnt )` clips by them; it returns false to stop.  `radius2()` is the cell's
// squared radius.  Lane 0 writes the stack.
template<bool CNT, class Cut, class Radius2, class Claims>
__device__ void walk_pyramid2( const ProbDev &P, int lane, double px, double py, double wi, int cx, int cy, int rd, int2 *stk, Cut cut,
                               Radius2 radius2, Claims claims ) {
    const int g0 = P.g[ 0 ], g1 = P.g[ 1 ];
    if ( lane == 0 ) stk[ 0 ] = make_int2( ( P.nlev - 1 ) << 16, 0 );
    int sp = 1;
    __syncwarp();
    double R2 = radius2();
    for ( int guard = 0; sp > 0 && guard < ( 1 << 24 ); ++guard ) {
        const int2 e = stk[ sp - 1 ];
        --sp;
        __syncwarp();
        const int l = e.x >> 16, X = e.x & 0xffff, Y = e.y;
        const int x0 = X << l, y0 = Y << l;
        const int x1 = min( ( X + 1 ) << l, g0 ) - 1, y1 = min( ( Y + 1 ) << l, g1 ) - 1;
        if ( l <= WALK_LEAF ) {
            const int bw = x1 - x0 + 1, bh = y1 - y0 + 1;           // at most 2 x 2
            int beg = 0, cnt = 0;
            bool tested = false, ranged = false;
            if ( lane < bw * bh ) {
                const int x = x0 + lane % bw, y = y0 + lane / bw;
                const bool walked = x >= cx - rd && x <= cx + rd && y >= cy - rd && y <= cy + rd;
                const size_t gc = ( size_t ) y * g0 + x;
                tested = ! walked;
                if ( ! walked && may_cut( cells_dist2( P, x, x, y, y, px, py ), wmaj_b( P, gc ), R2, wi ) ) {
                    int2 rg = P.cell_range[ gc ];
                    beg = rg.x;
                    cnt = rg.y - rg.x;
                    ranged = true;
                }
            }
            if constexpr ( CNT ) if ( P.gather ) {
                count_reads( P, lane, G_GRID, __popc( __ballot_sync( FULL, tested ) ) );
                count_reads( P, lane, G_RANGE, __popc( __ballot_sync( FULL, ranged ) ) );
            }
            if ( ! cut( beg, cnt ) ) return;
            R2 = radius2();
            continue;
        }
        // the (up to 4) children, lane k the child k, tested when their parent is expanded (their majorant records loaded
        // together): in the grid, not all inside the walked rings, not empty, claiming a vertex of the cell
        const int X2 = 2 * X + ( lane & 1 ), Y2 = 2 * Y + ( ( lane >> 1 ) & 1 );
        const int a0 = X2 << ( l - 1 ), b0 = Y2 << ( l - 1 );
        const int a1 = min( ( X2 + 1 ) << ( l - 1 ), g0 ) - 1, b1 = min( ( Y2 + 1 ) << ( l - 1 ), g1 ) - 1;
        bool ok = lane < 4 && X2 < lev_dim( g0, l - 1 ) && Y2 < lev_dim( g1, l - 1 ) &&
                  ! ( a0 >= cx - rd && a1 <= cx + rd && b0 >= cy - rd && b1 <= cy + rd );
        double cb = -1e300, ca0 = 0, ca1 = 0, dd = 0;
        if constexpr ( CNT ) if ( P.gather ) count_reads( P, lane, G_NODE, __popc( __ballot_sync( FULL, ok ) ) );
        if ( ok ) {
            const size_t rec = P.poff[ l - 1 ] + ( size_t ) Y2 * lev_dim( g0, l - 1 ) + X2;
            cb = wmaj_b( P, rec );
            ca0 = P.wpyr[ rec * 3 ];
            ca1 = P.wpyr[ rec * 3 + 1 ];
            dd = cells_dist2( P, a0, a1, b0, b1, px, py );
            ok = cb >= -1e299;
        }
        unsigned todo = __ballot_sync( FULL, ok ), claim = 0;
        while ( todo ) {
            const int c = __ffs( todo ) - 1;
            todo &= todo - 1;
            const double A[ 2 ] = { __shfl_sync( FULL, ca0, c ), __shfl_sync( FULL, ca1, c ) }, B = __shfl_sync( FULL, cb, c );
            const int ca = __shfl_sync( FULL, a0, c ), ca1i = __shfl_sync( FULL, a1, c ), cb0 = __shfl_sync( FULL, b0, c ),
                      cb1 = __shfl_sync( FULL, b1, c );
            const double lo[ 2 ] = { P.go[ 0 ] + ca * P.gh[ 0 ], P.go[ 1 ] + cb0 * P.gh[ 1 ] };
            const double hi[ 2 ] = { P.go[ 0 ] + ( ca1i + 1 ) * P.gh[ 0 ], P.go[ 1 ] + ( cb1 + 1 ) * P.gh[ 1 ] };
            if ( claims( lo, hi, A, B ) ) claim |= 1u << c;
        }
        // the claiming children pushed farthest first (equal distances in child order), so that the nearest is walked first
        int rank = 0;
#pragma unroll
        for ( int c = 0; c < 4; ++c ) {
            const double dc = __shfl_sync( FULL, dd, c );
            if ( ( ( claim >> c ) & 1 ) && ( dc > dd || ( dc == dd && c < lane ) ) ) ++rank;
        }
        const int nc = __popc( claim );
        if ( sp + nc > WALK_STACK ) return;                // cannot happen below 2^21 cells per side
        if ( ( claim >> lane ) & 1 ) stk[ sp + rank ] = make_int2( ( ( l - 1 ) << 16 ) | X2, Y2 );
        sp += nc;
        __syncwarp();
    }
}

// the seeds of up to 32 grid cells (lane k: the range [ beg, beg + cnt ) of one cell) as candidates, 32 at a time:
// a parallel pre-test against the polygon, then the clips of those that cut, in lane order
template<bool CNT>
__device__ __forceinline__ void cut_by_ranges( WPoly &C, const ProbDev &P, int lane, int s, double px, double py, double wi, int beg, int cnt,
                                               bool &overflow ) {
    int inc = cnt;
#pragma unroll
    for ( int o = 1; o < 32; o <<= 1 ) { int t = __shfl_up_sync( FULL, inc, o ); if ( lane >= o ) inc += t; }
    const int total = __shfl_sync( FULL, inc, 31 );
    const int exc = inc - cnt;
    for ( int t0 = 0; t0 < total && C.m > 0 && ! overflow; t0 += 32 ) {
        const int t = t0 + lane;
        int owner = 0;
#pragma unroll
        for ( int st = 16; st > 0; st >>= 1 ) { int v = __shfl_sync( FULL, inc, owner + st - 1 ); if ( v <= t ) owner += st; }
        owner = owner > 31 ? 31 : owner;
        int obeg = __shfl_sync( FULL, beg, owner ), oexc = __shfl_sync( FULL, exc, owner );
        int j = obeg + ( t - oexc );
        bool valid = t < total && j != s;
        if constexpr ( CNT ) if ( P.gather ) count_reads( P, lane, G_CAND, __popc( __ballot_sync( FULL, valid ) ) );
        double qx = 0, qy = 0, off = 0;
        if ( valid ) {
            qx = P.pos[ 2 * ( size_t ) j ] - px;
            qy = P.pos[ 2 * ( size_t ) j + 1 ] - py;
            double qw = P.w ? P.w[ j ] : 0.0;
            // the weights' difference first: added to a weight, the |q|^2 of two seeds 1e-10 apart is lost and the two
            // cells of the pair cut planes |q| apart
            off = 0.5 * ( ( wi - qw ) + ( qx * qx + qy * qy ) );
        }
        // the parallel pre-test: does candidate `lane` cut the current polygon at all?
        bool cuts = false;
        for ( int k = 0; k < C.m; ++k ) {
            double X = __shfl_sync( FULL, C.vx, k ), Y = __shfl_sync( FULL, C.vy, k );
            cuts |= qx * X + qy * Y > off;
        }
        unsigned todo = __ballot_sync( FULL, valid && cuts );
        while ( todo ) {
            int k = __ffs( todo ) - 1;
            todo &= todo - 1;
            double nx = __shfl_sync( FULL, qx, k ), ny = __shfl_sync( FULL, qy, k ), no = __shfl_sync( FULL, off, k );
            int nid = __shfl_sync( FULL, j, k );
            if ( ! wclip( C, lane, nx, ny, no, nid ) ) { overflow = true; break; }
            if ( C.m == 0 ) break;
        }
    }
}

// ---- THE FP32 CLIP (precision "mixed": the reference's float kernel and its FP64 re-solve, gpu/Cell2D.cuh:56-60, 991-1042) ------
// The polygon is held in FP32 (vertices and lines in registers: half the shuffles of a cut) and every decision is the FP64
// kernel's: a vertex is tested in FP32 against a band that bounds the FP32 error of the test, and only a vertex inside the
// band is re-checked in FP64, re-solved from its two lines as the FP64 kernel holds it; a new vertex is computed in FP32
// where its two lines cross at more than 1/20 rad, else in FP64 (then rounded).  At the end every vertex is re-solved in
// FP64 from its two lines (the seeds' positions and weights read again) and the cell is integrated as the FP64 one.
struct WPolyF {
    int m;
    float vx, vy;              // vertex `lane`
    float lnx, lny, loff;      // line of edge lane -> lane + 1
    int lid;
    bool ip;                   // interpolated on its edge (two lines nearly parallel, as the FP64 kernel does): kept as is
    // the security tests on FP32 vertices: the radius inflated, the majorants' claims with a margin of 1e-5
    static constexpr double R2_MARGIN = 1 + 1e-5, CLAIM_REL = 1e-5;
};

// the FP32 band of a test n . v - off at vertices of |v|_1 <= Rs: 64 float eps of the terms (the test's own rounding and
// that of a vertex crossed in FP32 at more than 1/20 rad)
constexpr float F32_BAND = 3.814697265625e-6f;        // 2^-18

// the FP64 line of edge `id` of the cell of seed (px, py, wi): a seed's bisector (as cut_by_ranges makes it) or a box side
// (as the kernel's start makes it)
__device__ __forceinline__ void line64( const ProbDev &P, int id, double px, double py, double wi, double &a, double &b, double &c ) {
    if ( id >= 0 ) {
        a = P.pos[ 2 * ( size_t ) id ] - px;
        b = P.pos[ 2 * ( size_t ) id + 1 ] - py;
        const double qw = P.w ? P.w[ id ] : 0.0;
        c = 0.5 * ( ( wi - qw ) + ( a * a + b * b ) );
    } else {
        const int side = -1 - id;
        a = side == 1 ? 1.0 : ( side == 3 ? -1.0 : 0.0 );
        b = side == 0 ? -1.0 : ( side == 2 ? 1.0 : 0.0 );
        c = side == 0 ? -( P.lo[ 1 ] - py ) : ( side == 1 ? P.hi[ 0 ] - px : ( side == 2 ? P.hi[ 1 ] - py : -( P.lo[ 0 ] - px ) ) );
    }
}

// the FP32 crossing of two lines, along line 1 (as `isect`); good: they cross at more than 1/20 rad
__device__ __forceinline__ void isectf( float a1, float b1, float c1, float a2, float b2, float c2, float &x, float &y, bool &good ) {
    const float det = a1 * b2 - a2 * b1;
    good = det * det > 0.0025f * ( a1 * a1 + b1 * b1 ) * ( a2 * a2 + b2 * b2 );
    const float k = c1 / ( a1 * a1 + b1 * b1 ), fx = k * a1, fy = k * b1;
    const float t = ( c2 - ( a2 * fx + b2 * fy ) ) / det;
    x = fx - t * b1;
    y = fy + t * a1;
}

// the crossing of the lines id1 then id2 in FP64 (as the FP64 kernel computes it), rounded; ok false: nearly parallel
__device__ __forceinline__ void isect64_ids( const ProbDev &P, int id1, int id2, double px, double py, double wi, float &x, float &y, bool &ok ) {
    double a1, b1, c1, a2, b2, c2, X, Y;
    line64( P, id1, px, py, wi, a1, b1, c1 );
    line64( P, id2, px, py, wi, a2, b2, c2 );
    isect( a1, b1, c1, a2, b2, c2, X, Y, ok );
    x = float( X );
    y = float( Y );
}

// keep n . y <= off (n, off: the candidate's FP64 bisector); Rs bounds |v|_1 over the polygon; false past 32 vertices
__device__ __forceinline__ bool wclip( WPolyF &C, int lane, double nx64, double ny64, double off64, int id, float Rs, const ProbDev &P, double px,
                                       double py, double wi ) {
    const int m = C.m;
    const float nx = float( nx64 ), ny = float( ny64 ), off = float( off64 );
    const float band = F32_BAND * ( ( fabsf( nx ) + fabsf( ny ) ) * Rs + fabsf( off ) );
    const float sf = nx * C.vx + ny * C.vy - off;
    double s = sf;
    const int plid = __shfl_sync( FULL, C.lid, lane == 0 ? ( m > 0 ? m - 1 : 0 ) : lane - 1 );
    const bool unc = lane < m && fabsf( sf ) <= band;
    if ( __any_sync( FULL, unc ) && unc ) {
        // the FP64 re-check: the vertex as the FP64 kernel holds it, the crossing of its two lines
        float x = C.vx, y = C.vy;
        bool ok = false;
        double X = C.vx, Y = C.vy;
        if ( ! C.ip ) {
            double a1, b1, c1, a2, b2, c2;
            line64( P, plid, px, py, wi, a1, b1, c1 );
            line64( P, C.lid, px, py, wi, a2, b2, c2 );
            isect( a1, b1, c1, a2, b2, c2, X, Y, ok );
            if ( ! ok ) { X = x; Y = y; }
        }
        s = nx64 * X + ny64 * Y - off64;
    }
    unsigned out = __ballot_sync( FULL, lane < m && s > 0 );
    if ( ! out ) return true;
    unsigned valid = m >= 32 ? FULL : ( ( 1u << m ) - 1 );
    if ( out == valid ) { C.m = 0; return true; }
    unsigned in = valid & ~out;
    unsigned rot_out = ( ( out >> 1 ) | ( out << ( m - 1 ) ) ) & valid;
    unsigned rot_in = ( ( in >> 1 ) | ( in << ( m - 1 ) ) ) & valid;
    unsigned A = in & rot_out, B = out & rot_in;
    int a, b;
    if ( __popc( A ) == 1 ) {
        a = __ffs( A ) - 1;
        b = __ffs( B ) - 1;
    } else {
        double sv = lane < m ? s : -1e300;
        double smax = warp_max( sv );
        int kstar = __ffs( __ballot_sync( FULL, lane < m && sv == smax ) ) - 1;
        int da = ( A >> lane ) & 1 ? ( ( kstar - lane ) % m + m ) % m : 1 << 20;
        int db = ( B >> lane ) & 1 ? ( ( lane - kstar ) % m + m ) % m : 1 << 20;
        for ( int o = 16; o > 0; o >>= 1 ) { da = min( da, __shfl_xor_sync( FULL, da, o ) ); db = min( db, __shfl_xor_sync( FULL, db, o ) ); }
        a = ( ( kstar - da ) % m + m ) % m;
        b = ( kstar + db ) % m;
    }
    int K = ( ( a - b - 1 ) % m + m ) % m + 1;
    if ( K + 2 > 32 ) return false;
    int a1 = a + 1 == m ? 0 : a + 1, b1 = b + 1 == m ? 0 : b + 1;
    const float anx = __shfl_sync( FULL, C.lnx, a ), any = __shfl_sync( FULL, C.lny, a ), aoff = __shfl_sync( FULL, C.loff, a );
    const float bnx = __shfl_sync( FULL, C.lnx, b ), bny = __shfl_sync( FULL, C.lny, b ), boff = __shfl_sync( FULL, C.loff, b );
    const int aid = __shfl_sync( FULL, C.lid, a ), bid = __shfl_sync( FULL, C.lid, b );
    float Px, Py, Qx, Qy;
    bool gP, gQ, ipP = false, ipQ = false;
    isectf( anx, any, aoff, nx, ny, off, Px, Py, gP );
    isectf( nx, ny, off, bnx, bny, boff, Qx, Qy, gQ );
    // (gP, gQ warp uniform) a crossing at less than 1/20 rad: in FP64, from the two FP64 lines; nearly parallel there too:
    // on the edge, as the FP64 kernel
    if ( ! gP ) {
        double a1x, a1y, a1c, X, Y;
        bool ok;
        line64( P, aid, px, py, wi, a1x, a1y, a1c );
        isect( a1x, a1y, a1c, nx64, ny64, off64, X, Y, ok );
        Px = float( X ); Py = float( Y );
        if ( ! ok ) {
            const float xa = __shfl_sync( FULL, C.vx, a ), ya = __shfl_sync( FULL, C.vy, a );
            const double sa = __shfl_sync( FULL, s, a );
            const float xa1 = __shfl_sync( FULL, C.vx, a1 ), ya1 = __shfl_sync( FULL, C.vy, a1 );
            const double sa1 = __shfl_sync( FULL, s, a1 );
            const double t = sa / ( sa - sa1 );
            Px = float( xa + t * ( xa1 - xa ) ); Py = float( ya + t * ( ya1 - ya ) );
            ipP = true;
        }
    }
    if ( ! gQ ) {
        double b1x, b1y, b1c, X, Y;
        bool ok;
        line64( P, bid, px, py, wi, b1x, b1y, b1c );
        isect( nx64, ny64, off64, b1x, b1y, b1c, X, Y, ok );
        Qx = float( X ); Qy = float( Y );
        if ( ! ok ) {
            const float xb = __shfl_sync( FULL, C.vx, b ), yb = __shfl_sync( FULL, C.vy, b );
            const double sb = __shfl_sync( FULL, s, b );
            const float xb1 = __shfl_sync( FULL, C.vx, b1 ), yb1 = __shfl_sync( FULL, C.vy, b1 );
            const double sb1 = __shfl_sync( FULL, s, b1 );
            const double t = sb / ( sb - sb1 );
            Qx = float( xb + t * ( xb1 - xb ) ); Qy = float( yb + t * ( yb1 - yb ) );
            ipQ = true;
        }
    }
    int src = ( b + 1 + lane ) % m;
    float nvx = __shfl_sync( FULL, C.vx, src ), nvy = __shfl_sync( FULL, C.vy, src );
    float nlx = __shfl_sync( FULL, C.lnx, src ), nly = __shfl_sync( FULL, C.lny, src ), nlo = __shfl_sync( FULL, C.loff, src );
    int nli = __shfl_sync( FULL, C.lid, src );
    bool nip = __shfl_sync( FULL, int( C.ip ), src ) != 0;
    if ( lane == K ) { nvx = Px; nvy = Py; nlx = nx; nly = ny; nlo = off; nli = id; nip = ipP; }
    if ( lane == K + 1 ) { nvx = Qx; nvy = Qy; nlx = bnx; nly = bny; nlo = boff; nli = bid; nip = ipQ; }
    C.vx = nvx; C.vy = nvy; C.lnx = nlx; C.lny = nly; C.loff = nlo; C.lid = nli; C.ip = nip;
    C.m = K + 2;
    return true;
}

template<bool CNT>
__device__ __forceinline__ void cut_by_ranges( WPolyF &C, const ProbDev &P, int lane, int s, double px, double py, double wi, int beg, int cnt,
                                               bool &overflow ) {
    int inc = cnt;
#pragma unroll
    for ( int o = 1; o < 32; o <<= 1 ) { int t = __shfl_up_sync( FULL, inc, o ); if ( lane >= o ) inc += t; }
    const int total = __shfl_sync( FULL, inc, 31 );
    const int exc = inc - cnt;
    for ( int t0 = 0; t0 < total && C.m > 0 && ! overflow; t0 += 32 ) {
        const int t = t0 + lane;
        int owner = 0;
#pragma unroll
        for ( int st = 16; st > 0; st >>= 1 ) { int v = __shfl_sync( FULL, inc, owner + st - 1 ); if ( v <= t ) owner += st; }
        owner = owner > 31 ? 31 : owner;
        int obeg = __shfl_sync( FULL, beg, owner ), oexc = __shfl_sync( FULL, exc, owner );
        int j = obeg + ( t - oexc );
        bool valid = t < total && j != s;
        if constexpr ( CNT ) if ( P.gather ) count_reads( P, lane, G_CAND, __popc( __ballot_sync( FULL, valid ) ) );
        double qx = 0, qy = 0, off = 0;
        if ( valid ) {
            qx = P.pos[ 2 * ( size_t ) j ] - px;
            qy = P.pos[ 2 * ( size_t ) j + 1 ] - py;
            double qw = P.w ? P.w[ j ] : 0.0;
            off = 0.5 * ( ( wi - qw ) + ( qx * qx + qy * qy ) );
        }
        // the parallel pre-test in FP32: a candidate within the band of a vertex goes on to the clip, which decides in FP64
        float Rs = lane < C.m ? fabsf( C.vx ) + fabsf( C.vy ) : 0.f;
#pragma unroll
        for ( int o = 16; o > 0; o >>= 1 ) Rs = fmaxf( Rs, __shfl_xor_sync( FULL, Rs, o ) );
        const float fx = float( qx ), fy = float( qy ), fo = float( off );
        const float band = F32_BAND * ( ( fabsf( fx ) + fabsf( fy ) ) * Rs + fabsf( fo ) );
        bool cuts = false;
        for ( int k = 0; k < C.m; ++k ) {
            const float X = __shfl_sync( FULL, C.vx, k ), Y = __shfl_sync( FULL, C.vy, k );
            cuts |= fx * X + fy * Y - fo > -band;
        }
        unsigned todo = __ballot_sync( FULL, valid && cuts );
        while ( todo ) {
            int k = __ffs( todo ) - 1;
            todo &= todo - 1;
            double nx = __shfl_sync( FULL, qx, k ), ny = __shfl_sync( FULL, qy, k ), no = __shfl_sync( FULL, off, k );
            int nid = __shfl_sync( FULL, j, k );
            if ( ! wclip( C, lane, nx, ny, no, nid, Rs, P, px, py, wi ) ) { overflow = true; break; }
            if ( C.m == 0 ) break;
        }
    }
}

// the FP32 polygon in FP64: every vertex re-solved from its two lines (the FP64 kernel's crossing), the lines in FP64
__device__ __forceinline__ void to_fp64( const WPolyF &F, WPoly &C, const ProbDev &P, int lane, double px, double py, double wi ) {
    C.m = F.m;
    C.lid = F.lid;
    double a = 0, b = 0, c = 0;
    if ( lane < F.m ) line64( P, F.lid, px, py, wi, a, b, c );
    C.lnx = a; C.lny = b; C.loff = c;
    const int prv = lane == 0 ? ( F.m > 0 ? F.m - 1 : 0 ) : lane - 1;
    const double pa = __shfl_sync( FULL, a, prv ), pb = __shfl_sync( FULL, b, prv ), pc = __shfl_sync( FULL, c, prv );
    double X = F.vx, Y = F.vy;
    bool ok = false;
    if ( lane < F.m && ! F.ip ) isect( pa, pb, pc, a, b, c, X, Y, ok );
    C.vx = ok ? X : double( F.vx );
    C.vy = ok ? Y : double( F.vy );
}

__device__ __forceinline__ void record_error( const ProbDev &P, ErrRec *err, int code, int prob, int seed, int needed ) {
    if ( P.perr ) *P.perr = 1.0;
    if ( atomicCAS( &err->code, 0, code ) == 0 ) { err->kind = 2; err->prob = prob; err->seed = seed; err->needed = needed; }
}


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

// the report of one problem's chunk, written by its block; the last block of the problem folds them (fixed tree)
__device__ void finish_report( const ProbDev &P, const Chunk &ch, double ( *sh )[ NB_REPORT ] ) {
    __shared__ int am_last;
    __syncthreads();
    if ( threadIdx.x == 0 ) {
        Rep r;
        r.init();
        for ( int w = 0; w < int( blockDim.x >> 5 ); ++w ) r.combine( sh[ w ] );
        double *dst = P.partials + ( size_t ) ch.index * NB_REPORT;
        for ( int k = 0; k < NB_REPORT; ++k ) dst[ k ] = r.v[ k ];
        __threadfence();
        unsigned prev = atomicAdd( P.counter, 1u );
        am_last = prev == unsigned( P.nchunk - 1 );
    }
    __syncthreads();
    if ( am_last ) {
        __threadfence();
        fold_reports_block<8>( P );
    }
    __syncthreads();
}

__device__ __forceinline__ void start_flags( WPoly & ) {}
__device__ __forceinline__ void start_flags( WPolyF &C ) { C.ip = false; }

// THE CLIP of the cell of seed s (rank): the box, then the grid's rings, then the pyramid of weight majorants; `Poly`
// the FP64 polygon (WPoly) or the FP32 one (WPolyF, precision "mixed")
template<bool CNT, class Poly>
__device__ __forceinline__ void clip2( Poly &C, const ProbDev &P, int lane, int s, double px, double py, double wi, double wmax, int2 *stk,
                                       bool &overflow ) {
    C.m = 4;
    start_flags( C );
    {
        double lx = P.lo[ 0 ] - px, ly = P.lo[ 1 ] - py, hx = P.hi[ 0 ] - px, hy = P.hi[ 1 ] - py;
        C.vx = ( lane == 1 || lane == 2 ) ? hx : lx;
        C.vy = ( lane >= 2 ) ? hy : ly;
        C.lnx = lane == 1 ? 1.0 : ( lane == 3 ? -1.0 : 0.0 );
        C.lny = lane == 0 ? -1.0 : ( lane == 2 ? 1.0 : 0.0 );
        C.loff = lane == 0 ? -ly : ( lane == 1 ? hx : ( lane == 2 ? hy : -lx ) );
        C.lid = -1 - lane;
    }
    // ---- the walk over the grid rings
    const int g0 = P.g[ 0 ], g1 = P.g[ 1 ];
    int cx = int( floor( ( px - P.go[ 0 ] ) / P.gh[ 0 ] ) ), cy = int( floor( ( py - P.go[ 1 ] ) / P.gh[ 1 ] ) );
    cx = cx < 0 ? 0 : ( cx >= g0 ? g0 - 1 : cx );
    cy = cy < 0 ? 0 : ( cy >= g1 ? g1 - 1 : cy );
    int rmax = max( max( cx, g0 - 1 - cx ), max( cy, g1 - 1 - cy ) );
    int rd = -1;                 // the rings walked, when the pyramid takes over
    for ( int r = 0; r <= rmax && C.m > 0 && ! overflow; ++r ) {
        const int ncell = r == 0 ? 1 : 8 * r;
        // a grid cell farther than the security radius of its own largest weight holds no cutting seed
        double R2 = Poly::R2_MARGIN * warp_max( lane < C.m ? double( C.vx * C.vx + C.vy * C.vy ) : 0.0 );
        for ( int cb = 0; cb < ncell && C.m > 0 && ! overflow; cb += 32 ) {
            int ci = cb + lane, beg = 0, cnt = 0;
            bool tested = false, ranged = false;
            if ( ci < ncell ) {
                int dx, dy;
                ring_offset( r, ci, dx, dy );
                int x = cx + dx, y = cy + dy;
                if ( x >= 0 && x < g0 && y >= 0 && y < g1 ) {
                    const size_t gc = ( size_t ) y * g0 + x;
                    tested = P.wpyr != nullptr;
                    if ( may_cut( cells_dist2( P, x, x, y, y, px, py ), P.wpyr ? wmaj_b( P, gc ) : wmax, R2, wi ) ) {
                        int2 rg = P.cell_range[ gc ];
                        beg = rg.x;
                        cnt = rg.y - rg.x;
                        ranged = true;
                    }
                }
            }
            if constexpr ( CNT ) if ( P.gather ) {
                count_reads( P, lane, G_GRID, __popc( __ballot_sync( FULL, tested ) ) );
                count_reads( P, lane, G_RANGE, __popc( __ballot_sync( FULL, ranged ) ) );
            }
            cut_by_ranges<CNT>( C, P, lane, s, px, py, wi, beg, cnt, overflow );
        }
        if ( C.m == 0 || overflow ) break;
        R2 = Poly::R2_MARGIN * warp_max( lane < C.m ? double( C.vx * C.vx + C.vy * C.vy ) : 0.0 );
        double ex = R2 + wmax - wi;
        if ( r * P.ghmin >= sqrt( R2 ) + sqrt( ex > 0 ? ex : 0.0 ) ) break;
        // the pyramid once the global bound reaches well past the next rings (non-uniform weights)
        if ( P.wpyr && r >= RINGS_FIRST && r < rmax && sqrt( R2 ) + sqrt( ex > 0 ? ex : 0.0 ) > ( r + 2 ) * P.ghmin ) { rd = r; break; }
    }
    if ( rd >= 0 && C.m > 0 && ! overflow )
        walk_pyramid2<CNT>(
            P, lane, px, py, wi, cx, cy, rd, stk,
            [&]( int beg, int cnt ) {
                cut_by_ranges<CNT>( C, P, lane, s, px, py, wi, beg, cnt, overflow );
                return C.m > 0 && ! overflow;
            },
            [&]() { return Poly::R2_MARGIN * warp_max( lane < C.m ? double( C.vx * C.vx + C.vy * C.vy ) : 0.0 ); },
            [&]( const double *lo, const double *hi, const double *a, double b ) {
                bool may = false;
                if ( lane < C.m ) {
                    const double X[ 2 ] = { px + C.vx, py + C.vy }, v[ 2 ] = { C.vx, C.vy };
                    may = wmaj_claims( a, b, lo, hi, X, v, 2, wi, Poly::CLAIM_REL );
                }
                return __any_sync( FULL, may ) != 0;
            } );
}

// the main kernel, one warp per cell; F32: the launch for the problems that clip in FP32 (the others skip its chunks, and
// the FP64 launch skips theirs -- one kernel each keeps each clip's registers to itself)
// THE ADJOINT of the masses and of the first moments of one cell (its lane's edge), the row `ui` of the outputs: off the
// clip's register allocation (a call, not inlined)
__device__ __noinline__ void vjp2( const ProbDev &P, int lane, bool fac, int ui, int uj, double cij, double dist, const EdgeInt &e, double ax,
                                   double ay, double x1, double y1, double px, double py ) {
    // the masses: grad_w_i = sum_j c_ij ( g_i - g_j ); grad_p_i = sum_j 2 c_ij ( g_i - g_j ) ( x_ij - p_i )
    double gw = 0, gpx = 0, gpy = 0;
    if ( fac && P.gm ) {
        const double dg = P.gm[ ui ] - P.gm[ uj ];
        gw = cij * dg;
        const double cxm = e.mx / e.meas, cym = e.my / e.meas;      // facet centroid, seed frame
        gpx = 2 * cij * dg * cxm;
        gpy = 2 * cij * dg * cym;
    }
    // the first moments F_i = int_cell x rho (a constant density): the facet ij moves by dw_j / 2|p_ij| when a weight
    // changes and by ( x - p_i ) . dp_i / |p_ij| when a seed moves, so with G = gF_i - gF_j and y = x - p_i:
    // grad_w_i += G . int_facet x rho / 2|p_ij|, grad_p_i += ( ( G . p_i ) int_facet y rho + int_facet y y^T rho G ) / |p_ij|
    if ( fac && P.gf ) {
        const double gx = P.gf[ 2 * size_t( ui ) ] - P.gf[ 2 * size_t( uj ) ], gy = P.gf[ 2 * size_t( ui ) + 1 ] - P.gf[ 2 * size_t( uj ) + 1 ];
        gw += ( gx * ( e.meas * px + e.mx ) + gy * ( e.meas * py + e.my ) ) / ( 2 * dist );
        // the segment A -> B (seed frame): int y y^T = rho len ( 2 A A^T + A B^T + B A^T + 2 B B^T ) / 6
        const double sxx = e.meas * ( ax * ax + ax * x1 + x1 * x1 ) / 3, syy = e.meas * ( ay * ay + ay * y1 + y1 * y1 ) / 3;
        const double sxy = e.meas * ( 2 * ax * ay + ax * y1 + x1 * ay + 2 * x1 * y1 ) / 6;
        const double pg = px * gx + py * gy;
        gpx += ( pg * e.mx + sxx * gx + sxy * gy ) / dist;
        gpy += ( pg * e.my + sxy * gx + syy * gy ) / dist;
    }
    gw = warp_sum( gw ); gpx = warp_sum( gpx ); gpy = warp_sum( gpy );
    if ( lane == 0 ) {
        if ( P.gw ) P.gw[ ui ] = gw;
        if ( P.gpos ) { P.gpos[ 2 * ( size_t ) ui ] = gpx; P.gpos[ 2 * ( size_t ) ui + 1 ] = gpy; }
    }
}

template<bool F32, bool CNT>
__global__ void __launch_bounds__( 256, 3 ) k_cells2d( const ProbDev *__restrict__ probs, const Chunk *__restrict__ chunks, int nchunks,
                                                    unsigned flags, ErrRec *err, OvfList *ovf ) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    __shared__ double sh_rep[ 8 ][ NB_REPORT ];
    __shared__ int2 sh_stk[ 8 ][ WALK_STACK ];
    const bool moments = flags & F_MOMENTS, facets = flags & F_FACETS, user_order = flags & F_USER_ORDER;
    for ( int c = blockIdx.x; c < nchunks; c += gridDim.x ) {
        const Chunk ch = chunks[ c ];
        const ProbDev &P = probs[ ch.prob ];
        if ( ( P.fp32 != 0 ) != F32 ) continue;          // (block uniform: the other launch's)
        double *rep = sh_rep[ warp ];          // this warp's report accumulators (lane 0 updates them)
        if ( lane == 0 ) {
            Rep r0;
            r0.init();
            for ( int k = 0; k < NB_REPORT; ++k ) rep[ k ] = r0.v[ k ];
        }
        const double wmax = P.wmax_slot ? order_dbl( *P.wmax_slot ) : 0.0;
        for ( int s = ch.begin + warp; s < ch.end; s += nwarps ) {
            const double px = P.pos[ 2 * ( size_t ) s ], py = P.pos[ 2 * ( size_t ) s + 1 ];
            const double wi = P.w ? P.w[ s ] : 0.0;
            WPoly C;
            bool overflow = false;
            if constexpr ( F32 ) {
                WPolyF F;
                clip2<CNT>( F, P, lane, s, px, py, wi, wmax, sh_stk[ warp ], overflow );
                if ( ! overflow ) to_fp64( F, C, P, lane, px, py, wi );
            } else
                clip2<CNT>( C, P, lane, s, px, py, wi, wmax, sh_stk[ warp ], overflow );
            const int user = P.user[ s ];
            if ( overflow ) {
                // past the 32 vertices a warp holds: the global-memory pass rebuilds it (report included)
                if ( lane == 0 ) {
                    if ( ovf ) {
                        int k = atomicAdd( &ovf->count, 1 );
                        if ( k < ovf->cap ) ovf->items[ k ] = OvfItem{ ch.prob, s };
                        else record_error( P, err, 4, ch.prob, user, 33 );
                    } else
                        record_error( P, err, 4, ch.prob, user, 33 );
                }
                continue;
            }
            // ---- integration over the edges
            const int m = C.m;
            const bool act = lane < m;
            int nxt = lane + 1 >= m ? 0 : lane + 1;
            double x1 = __shfl_sync( FULL, C.vx, nxt ), y1 = __shfl_sync( FULL, C.vy, nxt );
            EdgeInt e;
            e.m = e.fx = e.fy = e.s2 = e.meas = e.mx = e.my = 0;
            if ( P.dkind == D_GAUSS ) warp_edges_gauss( P, m, lane, C.vx, C.vy, px, py, moments, facets || ( flags & F_VJP ), e );
            else if ( act ) {
                if ( P.dkind == D_UNIFORM ) edge_uniform( C.vx, C.vy, x1, y1, P.rho, moments, e );
                else {
                    int iref = int( floor( ( 0 - ( P.dorg[ 0 ] - px ) ) / P.dstep[ 0 ] ) );
                    edge_image( P, px, py, iref, C.vx, C.vy, x1, y1, moments, e );
                }
            }
            double mass = warp_sum( e.m );
            if ( mass < 0 && mass > -1e-300 ) mass = 0;
            // facets
            bool fac = act && C.lid >= 0 && e.meas > 0;
            unsigned fmask = __ballot_sync( FULL, fac );
            int nf = __popc( fmask );
            if ( facets && nf > P.cap ) {
                if ( lane == 0 ) {
                    if ( ovf ) {
                        int k = atomicAdd( &ovf->count, 1 );
                        if ( k < ovf->cap ) ovf->items[ k ] = OvfItem{ ch.prob, s };
                        else record_error( P, err, 4, ch.prob, user, nf );
                    } else
                        record_error( P, err, 4, ch.prob, user, nf );
                }
                continue;
            }
            double dist = sqrt( C.lnx * C.lnx + C.lny * C.lny );
            double cij = fac ? e.meas / ( 2 * dist ) : 0.0;
            if ( facets ) {
                const int row = user_order ? user : s;
                if ( fac && nf ) {
                    int slot = __popc( fmask & ( ( 1u << lane ) - 1 ) );
                    size_t at = ( size_t ) row * P.cap + slot;
                    P.nid[ at ] = user_order ? P.user[ C.lid ] : C.lid;
                    P.nc[ at ] = cij;
                    if ( P.nm ) P.nm[ at ] = e.meas;
                }
                if ( lane == 0 ) P.nb[ row ] = nf;
            }
            if ( flags & F_VJP ) vjp2( P, lane, fac, user_order ? user : s, user_order ? P.user[ C.lid < 0 ? 0 : C.lid ] : C.lid, cij, dist, e, C.vx,
                                       C.vy, x1, y1, px, py );
            if ( moments ) {
                double fx = warp_sum( e.fx ), fy = warp_sum( e.fy ), s2 = warp_sum( e.s2 );
                if ( lane == 0 ) {
                    if ( user_order ) {
                        if ( P.first ) {
                            P.first[ 2 * ( size_t ) user ] = mass > 0 ? px + fx / mass : px;
                            P.first[ 2 * ( size_t ) user + 1 ] = mass > 0 ? py + fy / mass : py;
                        }
                        if ( P.cost ) P.cost[ user ] = s2;
                    } else {
                        if ( P.first ) { P.first[ 2 * ( size_t ) s ] = fx; P.first[ 2 * ( size_t ) s + 1 ] = fy; }
                        if ( P.cost ) P.cost[ s ] = s2;
                    }
                }
            }
            if ( lane == 0 && P.mass ) P.mass[ user_order ? user : s ] = mass;
            if ( ( flags & F_REPORT ) && lane == 0 ) {
                double nu = P.nu[ s ];
                double e2 = fabs( nu - mass );
                rep[ R_WORST ] = fmax( rep[ R_WORST ], e2 );
                rep[ R_WORST_REL ] = fmax( rep[ R_WORST_REL ], e2 / nu );
                rep[ R_AMIN ] = fmin( rep[ R_AMIN ], mass );
                rep[ R_ASUM ] += mass;
                rep[ R_LIN2 ] += ( nu - mass ) * ( nu - mass );
                double x = mass / nu, g = g_of( x, P.res, P.power );
                double n1 = rep[ R_GCOUNT ] + 1, d = g - rep[ R_GMEAN ];
                rep[ R_GMEAN ] += d / n1;
                rep[ R_GM2 ] += d * ( g - rep[ R_GMEAN ] );
                rep[ R_GCOUNT ] = n1;
                double u = nu / gp_of( x, P.res, P.power );
                rep[ R_SU ] += u;
                rep[ R_SUG ] += u * g;
                rep[ R_NUSUM ] += nu;
                rep[ R_NEMPTY ] += mass > 0 ? 0.0 : 1.0;
            }
        }
        if ( flags & F_REPORT ) finish_report( P, ch, sh_rep );
    }
}

// the Newton report alone, from masses and targets already in memory (after a rescale of the targets)
__global__ void __launch_bounds__( 256 ) k_report( const ProbDev *__restrict__ probs, const Chunk *__restrict__ chunks, int nchunks ) {
    __shared__ double sh_rep[ 8 ][ NB_REPORT ];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for ( int c = blockIdx.x; c < nchunks; c += gridDim.x ) {
        const Chunk ch = chunks[ c ];
        const ProbDev &P = probs[ ch.prob ];
        Rep rep;
        rep.init();
        if ( lane == 0 )
            for ( int s = ch.begin + warp; s < ch.end; s += 8 ) {
                double mass = P.mass[ s ], nu = P.nu[ s ];
                double e2 = fabs( nu - mass );
                rep.v[ R_WORST ] = fmax( rep.v[ R_WORST ], e2 );
                rep.v[ R_WORST_REL ] = fmax( rep.v[ R_WORST_REL ], e2 / nu );
                rep.v[ R_AMIN ] = fmin( rep.v[ R_AMIN ], mass );
                rep.v[ R_ASUM ] += mass;
                rep.v[ R_LIN2 ] += ( nu - mass ) * ( nu - mass );
                double x = mass / nu, g = g_of( x, P.res, P.power );
                double n1 = rep.v[ R_GCOUNT ] + 1, d = g - rep.v[ R_GMEAN ];
                rep.v[ R_GMEAN ] += d / n1;
                rep.v[ R_GM2 ] += d * ( g - rep.v[ R_GMEAN ] );
                rep.v[ R_GCOUNT ] = n1;
                double u = nu / gp_of( x, P.res, P.power );
                rep.v[ R_SU ] += u;
                rep.v[ R_SUG ] += u * g;
                rep.v[ R_NUSUM ] += nu;
                rep.v[ R_NEMPTY ] += mass > 0 ? 0.0 : 1.0;
            }
        if ( lane == 0 ) for ( int k = 0; k < NB_REPORT; ++k ) sh_rep[ warp ][ k ] = rep.v[ k ];
        finish_report( P, ch, sh_rep );
    }
}

void launch_report( const Launch &L, const ProbDev *probs, const Chunk *chunks, int nchunks ) {
    if ( nchunks <= 0 ) return;
    k_report<<<nchunks, 256, 0, L.stream>>>( probs, chunks, nchunks );
    ++*L.launches;
}

void launch_cells2d( const Launch &L, const ProbDev *probs, const Chunk *chunks, int nchunks, unsigned flags, ErrRec *err, OvfList *ovf,
                     int clips ) {
    if ( nchunks <= 0 ) return;
    // the counting instantiations only when the search's reads are counted (F_GATHER): the others compile without them
    const bool cnt = flags & F_GATHER;
    if ( clips & 1 ) {
        if ( cnt ) k_cells2d<false, true><<<nchunks, 256, 0, L.stream>>>( probs, chunks, nchunks, flags, err, ovf );
        else k_cells2d<false, false><<<nchunks, 256, 0, L.stream>>>( probs, chunks, nchunks, flags, err, ovf );
        ++*L.launches;
    }
    if ( clips & 2 ) {
        if ( cnt ) k_cells2d<true, true><<<nchunks, 256, 0, L.stream>>>( probs, chunks, nchunks, flags, err, ovf );
        else k_cells2d<true, false><<<nchunks, 256, 0, L.stream>>>( probs, chunks, nchunks, flags, err, ovf );
        ++*L.launches;
    }
}

// ---- the big cells: one warp per cell, the polygon in global memory (two buffers of VBIG vertices) ---------------------------
struct BigPoly {
    double *x, *y, *nx, *ny, *off;
    int *id;
    unsigned char *out;
};

__device__ __forceinline__ BigPoly big_buffer( char *base, int which ) {
    BigPoly B;
    char *p = base + size_t( which ) * VBIG * ( 5 * 8 + 4 + 1 );
    B.x = ( double * ) p; B.y = B.x + VBIG; B.nx = B.y + VBIG; B.ny = B.nx + VBIG; B.off = B.ny + VBIG;
    B.id = ( int * ) ( B.off + VBIG );
    B.out = ( unsigned char * ) ( B.id + VBIG );
    return B;
}

__device__ __forceinline__ int warp_min_int( int v ) {
#pragma unroll
    for ( int o = 16; o > 0; o >>= 1 ) v = min( v, __shfl_xor_sync( FULL, v, o ) );
    return v;
}

// keep n . y <= off; returns the new vertex count, -1 past VBIG; `moved`: the new polygon is in D
__device__ int big_clip( BigPoly &S, BigPoly &D, int m, int lane, double nx, double ny, double off, int id, bool &moved ) {
    moved = false;
    int nout = 0;
    for ( int k = lane; k - lane < m; k += 32 ) {
        bool o = k < m && nx * S.x[ k ] + ny * S.y[ k ] - off > 0;
        if ( k < m ) S.out[ k ] = o;
        nout += __popc( __ballot_sync( FULL, o ) );
    }
    __syncwarp();
    if ( nout == 0 ) return m;
    if ( nout == m ) return 0;
    // the outside run that holds the most outside vertex (other runs are rounding noise, kept)
    double smax = -1e300;
    int kstar = 0;
    for ( int k = lane; k < m; k += 32 ) {
        double sk = nx * S.x[ k ] + ny * S.y[ k ] - off;
        if ( sk > smax ) { smax = sk; kstar = k; }
    }
    double wmaxs = warp_max( smax );
    int kcand = smax == wmaxs ? kstar : 1 << 30;
    kstar = warp_min_int( kcand );
    int da = 1 << 30, db = 1 << 30;
    for ( int k = lane; k < m; k += 32 ) {
        int k1 = k + 1 == m ? 0 : k + 1;
        if ( ! S.out[ k ] && S.out[ k1 ] ) da = min( da, ( ( kstar - k ) % m + m ) % m );
        if ( S.out[ k ] && ! S.out[ k1 ] ) db = min( db, ( ( k - kstar ) % m + m ) % m );
    }
    da = warp_min_int( da );
    db = warp_min_int( db );
    const int a = ( ( kstar - da ) % m + m ) % m;
    const int b = ( kstar + db ) % m;
    const int K = ( ( a - b - 1 ) % m + m ) % m + 1;
    if ( K + 2 > VBIG ) return -1;
    for ( int t = lane; t < K; t += 32 ) {
        int src = ( b + 1 + t ) % m;
        D.x[ t ] = S.x[ src ]; D.y[ t ] = S.y[ src ]; D.nx[ t ] = S.nx[ src ]; D.ny[ t ] = S.ny[ src ]; D.off[ t ] = S.off[ src ];
        D.id[ t ] = S.id[ src ];
    }
    if ( lane == 0 ) {
        int a1 = a + 1 == m ? 0 : a + 1, b1 = b + 1 == m ? 0 : b + 1;
        double Px, Py, Qx, Qy;
        bool okP, okQ;
        isect( S.nx[ a ], S.ny[ a ], S.off[ a ], nx, ny, off, Px, Py, okP );
        isect( nx, ny, off, S.nx[ b ], S.ny[ b ], S.off[ b ], Qx, Qy, okQ );
        if ( ! okP ) {
            double sa = nx * S.x[ a ] + ny * S.y[ a ] - off, sa1 = nx * S.x[ a1 ] + ny * S.y[ a1 ] - off, t = sa / ( sa - sa1 );
            Px = S.x[ a ] + t * ( S.x[ a1 ] - S.x[ a ] ); Py = S.y[ a ] + t * ( S.y[ a1 ] - S.y[ a ] );
        }
        if ( ! okQ ) {
            double sb = nx * S.x[ b ] + ny * S.y[ b ] - off, sb1 = nx * S.x[ b1 ] + ny * S.y[ b1 ] - off, t = sb / ( sb - sb1 );
            Qx = S.x[ b ] + t * ( S.x[ b1 ] - S.x[ b ] ); Qy = S.y[ b ] + t * ( S.y[ b1 ] - S.y[ b ] );
        }
        D.x[ K ] = Px; D.y[ K ] = Py; D.nx[ K ] = nx; D.ny[ K ] = ny; D.off[ K ] = off; D.id[ K ] = id;
        D.x[ K + 1 ] = Qx; D.y[ K + 1 ] = Qy; D.nx[ K + 1 ] = S.nx[ b ]; D.ny[ K + 1 ] = S.ny[ b ]; D.off[ K + 1 ] = S.off[ b ];
        D.id[ K + 1 ] = S.id[ b ];
    }
    __syncwarp();
    moved = true;
    return K + 2;
}

__global__ void __launch_bounds__( 32 ) k_cells2d_big( const ProbDev *__restrict__ probs, const OvfList *__restrict__ ovf, int count,
                                                        unsigned flags, ErrRec *err, char *scratch ) {
    const int lane = threadIdx.x;
    __shared__ int2 stk[ WALK_STACK ];
    char *mine = scratch + size_t( blockIdx.x ) * 2 * VBIG * ( 5 * 8 + 4 + 1 );
    for ( int it = blockIdx.x; it < count; it += gridDim.x ) {
        const OvfItem item = ovf->items[ it ];
        const ProbDev &P = probs[ item.prob ];
        if ( P.dim != 2 ) continue;                      // the 3D items are the 3D pass's
        // flags 0: each problem's own pass (a final-moments diagram has `first`, a Newton diagram has not)
        const unsigned fl = flags ? flags : ( P.first ? ( F_MOMENTS | F_USER_ORDER ) : ( F_MASS | F_FACETS ) );
        const bool moments = fl & F_MOMENTS, facets = fl & F_FACETS, user_order = fl & F_USER_ORDER;
        const int s = item.seed;
        BigPoly A = big_buffer( mine, 0 ), B = big_buffer( mine, 1 );
        BigPoly *S = &A, *D = &B;
        const double px = P.pos[ 2 * ( size_t ) s ], py = P.pos[ 2 * ( size_t ) s + 1 ];
        const double wi = P.w ? P.w[ s ] : 0.0;
        const double wmax = P.wmax_slot ? order_dbl( *P.wmax_slot ) : 0.0;
        if ( lane < 4 ) {
            double lx = P.lo[ 0 ] - px, ly = P.lo[ 1 ] - py, hx = P.hi[ 0 ] - px, hy = P.hi[ 1 ] - py;
            S->x[ lane ] = ( lane == 1 || lane == 2 ) ? hx : lx;
            S->y[ lane ] = ( lane >= 2 ) ? hy : ly;
            S->nx[ lane ] = lane == 1 ? 1.0 : ( lane == 3 ? -1.0 : 0.0 );
            S->ny[ lane ] = lane == 0 ? -1.0 : ( lane == 2 ? 1.0 : 0.0 );
            S->off[ lane ] = lane == 0 ? -ly : ( lane == 1 ? hx : ( lane == 2 ? hy : -lx ) );
            S->id[ lane ] = -1 - lane;
        }
        __syncwarp();
        int m = 4;
        bool overflow = false;
        const int g0 = P.g[ 0 ], g1 = P.g[ 1 ];
        int cx = int( floor( ( px - P.go[ 0 ] ) / P.gh[ 0 ] ) ), cy = int( floor( ( py - P.go[ 1 ] ) / P.gh[ 1 ] ) );
        cx = cx < 0 ? 0 : ( cx >= g0 ? g0 - 1 : cx );
        cy = cy < 0 ? 0 : ( cy >= g1 ? g1 - 1 : cy );
        const int rmax = max( max( cx, g0 - 1 - cx ), max( cy, g1 - 1 - cy ) );
        // the seeds of a range, clipped one by one
        auto cut_range = [&]( int b, int e ) {
            for ( int j = b; j < e && m > 0 && ! overflow; ++j ) {
                if ( j == s ) continue;
                double qx = P.pos[ 2 * ( size_t ) j ] - px, qy = P.pos[ 2 * ( size_t ) j + 1 ] - py;
                double qw = P.w ? P.w[ j ] : 0.0;
                double off = 0.5 * ( ( wi - qw ) + ( qx * qx + qy * qy ) );
                bool moved;
                int nm = big_clip( *S, *D, m, lane, qx, qy, off, j, moved );
                if ( nm < 0 ) { overflow = true; break; }
                if ( moved ) { BigPoly *t = S; S = D; D = t; }
                m = nm;
            }
        };
        // the ranges held by the lanes (a leaf of the pyramid walk), lane by lane
        auto cut_lanes = [&]( int beg, int cnt ) {
            for ( int k = 0; k < 32 && m > 0 && ! overflow; ++k ) {
                int b = __shfl_sync( FULL, beg, k ), c = __shfl_sync( FULL, cnt, k );
                cut_range( b, b + c );
            }
            return m > 0 && ! overflow;
        };
        auto radius2 = [&]() {
            double R2 = 0;
            for ( int k = lane; k < m; k += 32 ) R2 = fmax( R2, S->x[ k ] * S->x[ k ] + S->y[ k ] * S->y[ k ] );
            return warp_max( R2 );
        };
        int rd = -1;
        for ( int r = 0; r <= rmax && m > 0 && ! overflow; ++r ) {
            const double R2 = radius2();
            double ex = R2 + wmax - wi, rb = sqrt( R2 ) + sqrt( ex > 0 ? ex : 0.0 );
            if ( r > 0 && ( r - 1 ) * P.ghmin >= rb ) break;
            if ( P.wpyr && r > RINGS_FIRST && rb > ( r + 1 ) * P.ghmin ) { rd = r - 1; break; }
            const int ncell = r == 0 ? 1 : 8 * r;
            for ( int ci = 0; ci < ncell && m > 0 && ! overflow; ++ci ) {
                int dx, dy;
                ring_offset( r, ci, dx, dy );
                int x = cx + dx, y = cy + dy;
                if ( x < 0 || x >= g0 || y < 0 || y >= g1 ) continue;
                if ( ! may_cut( cells_dist2( P, x, x, y, y, px, py ), P.wpyr ? wmaj_b( P, ( size_t ) y * g0 + x ) : wmax, R2, wi ) ) continue;
                int2 rg = P.cell_range[ ( size_t ) y * g0 + x ];
                cut_range( rg.x, rg.y );
            }
        }
        auto claims = [&]( const double *lo, const double *hi, const double *a, double b ) {
            bool may = false;
            for ( int k = lane; k < m && ! may; k += 32 ) {
                const double X[ 2 ] = { px + S->x[ k ], py + S->y[ k ] }, v[ 2 ] = { S->x[ k ], S->y[ k ] };
                may = wmaj_claims( a, b, lo, hi, X, v, 2, wi );
            }
            return __any_sync( FULL, may ) != 0;
        };
        if ( rd >= 0 && m > 0 && ! overflow ) walk_pyramid2<false>( P, lane, px, py, wi, cx, cy, rd, stk, cut_lanes, radius2, claims );
        const int user = P.user[ s ];
        if ( overflow ) {
            // past the global-memory polygon: an error of its problem -- or, in a trial diagram, a refused step
            if ( lane == 0 ) {
                if ( P.prefuse ) *P.prefuse = 1.0;
                else record_error( P, err, 4, item.prob, user, VBIG );
            }
            continue;
        }
        // integration, edges strided over the lanes
        double em = 0, efx = 0, efy = 0, es2 = 0;
        int nf = 0;
        for ( int base = 0; base < m; base += 32 ) {
            int k = base + lane;
            EdgeInt e;
            e.m = e.fx = e.fy = e.s2 = e.meas = e.mx = e.my = 0;
            if ( k < m ) {
                int k1 = k + 1 == m ? 0 : k + 1;
                double x0 = S->x[ k ], y0 = S->y[ k ], x1 = S->x[ k1 ], y1 = S->y[ k1 ];
                if ( P.dkind == D_UNIFORM ) edge_uniform( x0, y0, x1, y1, P.rho, moments, e );
                else if ( P.dkind == D_IMAGE ) {
                    int iref = int( floor( ( 0 - ( P.dorg[ 0 ] - px ) ) / P.dstep[ 0 ] ) );
                    edge_image( P, px, py, iref, x0, y0, x1, y1, moments, e );
                } else edge_gauss( P, px, py, x0, y0, x1, y1, moments, true, e );
            }
            em += e.m; efx += e.fx; efy += e.fy; es2 += e.s2;
            bool fac = k < m && S->id[ k ] >= 0 && e.meas > 0;
            if ( k < m ) { D->off[ k ] = fac ? e.meas : -1.0; }   // the facet measure of edge k (scratch)
            nf += __popc( __ballot_sync( FULL, fac ) );
        }
        __syncwarp();
        double mass = warp_sum( em );
        const int row = user_order ? user : s;
        if ( facets ) {
            const bool to_store = nf > P.cap;
            if ( to_store && ! P.ovf_ids ) {
                if ( lane == 0 ) record_error( P, err, 4, item.prob, user, nf );
                continue;
            }
            int base_at = 0;
            if ( to_store ) {
                if ( lane == 0 ) base_at = atomicAdd( P.ovf_count, nf );
                base_at = __shfl_sync( FULL, base_at, 0 );
                if ( base_at + nf > P.ovf_cap ) {
                    if ( lane == 0 ) record_error( P, err, 4, item.prob, user, nf );
                    continue;
                }
            }
            int written = 0;
            for ( int base = 0; base < m; base += 32 ) {
                int k = base + lane;
                double meas = k < m ? D->off[ k ] : -1.0;
                bool fac = meas > 0;
                unsigned fm = __ballot_sync( FULL, fac );
                int slot = written + __popc( fm & ( ( 1u << lane ) - 1 ) );
                if ( fac ) {
                    int j = S->id[ k ];
                    double dist = sqrt( S->nx[ k ] * S->nx[ k ] + S->ny[ k ] * S->ny[ k ] );
                    double cij = meas / ( 2 * dist );
                    int jid = user_order ? P.user[ j ] : j;
                    if ( to_store ) { P.ovf_ids[ base_at + slot ] = jid; P.ovf_c[ base_at + slot ] = cij; }
                    else {
                        size_t at = ( size_t ) row * P.cap + slot;
                        P.nid[ at ] = jid;
                        P.nc[ at ] = cij;
                        if ( P.nm ) P.nm[ at ] = meas;
                    }
                }
                written += __popc( fm );
            }
            if ( lane == 0 ) {
                P.nb[ row ] = nf;
                if ( to_store ) P.nid[ ( size_t ) row * P.cap ] = base_at;
            }
        }
        if ( moments ) {
            double fx = warp_sum( efx ), fy = warp_sum( efy ), s2 = warp_sum( es2 );
            if ( lane == 0 ) {
                if ( user_order ) {
                    if ( P.first ) {
                        P.first[ 2 * ( size_t ) user ] = mass > 0 ? px + fx / mass : px;
                        P.first[ 2 * ( size_t ) user + 1 ] = mass > 0 ? py + fy / mass : py;
                    }
                    if ( P.cost ) P.cost[ user ] = s2;
                } else {
                    if ( P.first ) { P.first[ 2 * ( size_t ) s ] = fx; P.first[ 2 * ( size_t ) s + 1 ] = fy; }
                    if ( P.cost ) P.cost[ s ] = s2;
                }
            }
        }
        if ( ( fl & F_VJP ) && lane == 0 ) record_error( P, err, 4, item.prob, user, m );
        if ( lane == 0 && P.mass ) P.mass[ row ] = mass;
        __syncwarp();
    }
}

size_t big_scratch_bytes( int warps ) { return size_t( warps ) * 2 * VBIG * ( 5 * 8 + 4 + 1 ) + 256; }

void launch_cells2d_big( const Launch &L, const ProbDev *probs, const OvfList *ovf, int count, unsigned flags, ErrRec *err, char *scratch,
                         int warps ) {
    if ( count <= 0 ) return;
    int grid = count < warps ? count : warps;
    k_cells2d_big<<<grid, 32, 0, L.stream>>>( probs, ovf, count, flags, err, scratch );
    ++*L.launches;
}

// ---- THE LIMITS STEP (2D) -------------------------------------------------------------------------------------------
// The cell of seed s at the weights w + a d, computed by one thread: the box clipped by the bisectors of the neighbours s
// has in the accepted and in the trial diagram (a superset of the true cell when a neighbour appears in between: the
// limit is then a little late, and the trial diagram at the step it gives says so), integrated edge by edge.
constexpr int LIMV = 4 + 2 * CAP2 + 8;

__device__ double lim_cell_mass( const LimDev &L, int s, double a, double px, double py, bool &ok ) {
    const ProbDev &P = L.P;
    double X[ LIMV ], Y[ LIMV ], U[ LIMV ], V[ LIMV ];
    int m = 4;
    X[ 0 ] = P.lo[ 0 ] - px; Y[ 0 ] = P.lo[ 1 ] - py;
    X[ 1 ] = P.hi[ 0 ] - px; Y[ 1 ] = P.lo[ 1 ] - py;
    X[ 2 ] = P.hi[ 0 ] - px; Y[ 2 ] = P.hi[ 1 ] - py;
    X[ 3 ] = P.lo[ 0 ] - px; Y[ 3 ] = P.hi[ 1 ] - py;
    const double wi = P.w[ s ] + a * L.d[ s ];
    for ( int tab = 0; tab < 2 && m > 0; ++tab ) {
        const int *nb = tab ? L.nb1 : L.nb0, *nid = tab ? L.nid1 : L.nid0;
        const int k = nb[ s ];
        for ( int q = 0; q < k && m > 0; ++q ) {
            const int j = nid[ size_t( s ) * P.cap + q ];
            const double qx = P.pos[ 2 * size_t( j ) ] - px, qy = P.pos[ 2 * size_t( j ) + 1 ] - py;
            const double off = 0.5 * ( ( wi - ( P.w[ j ] + a * L.d[ j ] ) ) + ( qx * qx + qy * qy ) );
            int m2 = 0;
            for ( int v = 0; v < m; ++v ) {
                const int v1 = v + 1 == m ? 0 : v + 1;
                const double s0 = qx * X[ v ] + qy * Y[ v ] - off, s1 = qx * X[ v1 ] + qy * Y[ v1 ] - off;
                if ( m2 + 2 > LIMV ) { ok = false; return 0; }
                if ( s0 <= 0 ) { U[ m2 ] = X[ v ]; V[ m2 ] = Y[ v ]; ++m2; }
                if ( ( s0 <= 0 ) != ( s1 <= 0 ) ) {
                    // from the kept end (the two cells of an edge make the same point)
                    const int ui = s0 <= 0 ? v : v1, vi = s0 <= 0 ? v1 : v;
                    const double su = s0 <= 0 ? s0 : s1, sv = s0 <= 0 ? s1 : s0, tt = su / ( su - sv );
                    U[ m2 ] = X[ ui ] + tt * ( X[ vi ] - X[ ui ] );
                    V[ m2 ] = Y[ ui ] + tt * ( Y[ vi ] - Y[ ui ] );
                    ++m2;
                }
            }
            m = m2;
            for ( int v = 0; v < m; ++v ) { X[ v ] = U[ v ]; Y[ v ] = V[ v ]; }
        }
    }
    double mass = 0;
    const int iref = P.dkind == D_IMAGE ? int( floor( ( 0 - ( P.dorg[ 0 ] - px ) ) / P.dstep[ 0 ] ) ) : 0;
    for ( int v = 0; v < m; ++v ) {
        const int v1 = v + 1 == m ? 0 : v + 1;
        EdgeInt e;
        e.m = e.fx = e.fy = e.s2 = e.meas = e.mx = e.my = 0;
        if ( P.dkind == D_UNIFORM ) edge_uniform( X[ v ], Y[ v ], X[ v1 ], Y[ v1 ], P.rho, false, e );
        else if ( P.dkind == D_IMAGE ) edge_image( P, px, py, iref, X[ v ], Y[ v ], X[ v1 ], Y[ v1 ], false, e );
        else edge_gauss( P, px, py, X[ v ], Y[ v ], X[ v1 ], Y[ v1 ], false, false, e );
        mass += e.m;
    }
    return mass;
}

// the first a in ( 0, t ] where the mass of cell s falls below eps: the first of 8 even samples below it, then 30
// bisections; t when no sample falls below (on these neighbours), 0 when the cell starts below, t / 2 past the capacity
__device__ double lim_alpha( const LimDev &L, int s ) {
    const double px = L.P.pos[ 2 * size_t( s ) ], py = L.P.pos[ 2 * size_t( s ) + 1 ];
    bool ok = true;
    const double m0 = lim_cell_mass( L, s, 0.0, px, py, ok );
    if ( ! ok ) return 0.5 * L.t;
    if ( ! ( m0 >= L.eps ) ) return 0.0;
    double lo = 0, hi = -1;
    for ( int k = 1; k <= 8; ++k ) {
        const double a = L.t * k / 8;
        const double m = lim_cell_mass( L, s, a, px, py, ok );
        if ( ! ok ) return 0.5 * L.t;
        if ( m < L.eps ) { hi = a; break; }
        lo = a;
    }
    if ( hi < 0 ) return L.t;
    for ( int it = 0; it < 30; ++it ) {
        const double mid = 0.5 * ( lo + hi );
        const double m = lim_cell_mass( L, s, mid, px, py, ok );
        if ( ! ok ) break;
        if ( m < L.eps ) hi = mid;
        else lo = mid;
    }
    return lo;
}

__global__ void __launch_bounds__( CHUNK ) k_limits2d( const LimDev *__restrict__ lims, const Chunk *__restrict__ chunks, int nch ) {
    const Chunk ch = chunks[ blockIdx.x ];
    const LimDev &L = lims[ ch.prob ];
    for ( int s = ch.begin + int( threadIdx.x ); s < ch.end; s += blockDim.x ) {
        if ( ! ( L.a2[ s ] < L.eps ) ) continue;
        atomicAdd( L.out, 1.0 );
        const int cap = L.P.cap;
        // a row past the table (its facets in the overflow store): the trials' halving for this cell
        const double alpha = ( L.nb0[ s ] > cap || L.nb1[ s ] > cap ) ? 0.5 * L.t : lim_alpha( L, s );
        atomicMin( reinterpret_cast<unsigned long long *>( L.out + 1 ), dbl_order( alpha ) );
    }
}

void launch_limits2d( const Launch &L, const LimDev *lims, const Chunk *chunks, int nchunks ) {
    if ( nchunks <= 0 ) return;
    k_limits2d<<<nchunks, CHUNK, 0, L.stream>>>( lims, chunks, nchunks );
    ++*L.launches;
}


} // namespace sdot

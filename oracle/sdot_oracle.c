/*
 * ORACLE -- TEST INFRASTRUCTURE, NOT THE PRODUCT.
 *
 * A CPU restatement, in FP64 with OpenMP, of the semi-discrete optimal transport path of hleclerc/sdot-ffi
 * (package `sdot`): power (Laguerre) cells clipped from the domain box, their masses, barycentres, costs
 * and facet measures against a density, the Laplacian of the Laguerre graph, and the damped Newton of
 * Kitagawa-Merigot-Thibert on the dual weights.  Only the tests, `__graft_entry__.smoke()` and the
 * `cpu_baseline` / `--impl reference` legs of `bench.py` may load this library, and only as the checker
 * or as the timed CPU baseline; the product (the CUDA library) never calls it.
 *
 * Parity status: PINNED on the reference's own known-answer tests for this path -- the fixtures under
 * tests/golden/ (tests/test_PowerDiagram.py:35-45, 46-57, 58-76, 217-244, 245-264, 266-284, 374-404),
 * the closed-form gaussian facet and its both-sides symmetry (tests/test_SumOfGaussians.py:20-61), the
 * closed-form moments (tests/test_SdotPlanNd.py:460-498) and the reference's solver tests restated in
 * the oracle's own test file -- and on independent checks that share no code with it (Monte-Carlo argmin
 * partition, lifted convex hull neighbour sets, brute force versus grid search, finite differences).
 * Not pinned against outputs of the reference itself: it cannot be imported or compiled here (its C++
 * needs the third-party `loom-ffi==2026.10.10.1` support headers and loom-generated aggregate headers,
 * absent from the tree; its CPU Cholesky needs Eigen 3.4.0, absent).
 *
 * What is restated, and from where (all paths relative to the reference project):
 *   - the power bisector `|x-p_i|^2 - w_i <= |x-p_j|^2 - w_j`, written in the frame of seed i as
 *     `y.q <= (|q|^2 + w_i - w_j) / 2`, q = p_j - p_i (src/sdot/PowerDiagram.py:3-10, 600-607;
 *     src/sdot/include/sdot/gpu/Cell2D.cuh:135-160);
 *   - the facet coefficient `c_ij = int_facet rho / (2 |p_i - p_j|)` (sdotplan/Laplacian.h:7);
 *   - the Laplacian with the row's own facet measure and `dia = 1` for an empty row
 *     (sdotplan/Laplacian.h:37-62);
 *   - the Newton loop, TRIALS step, LOG->LIN residual switch, eps floor, strict merit decrease and
 *     hopeless-damping stop (sdotplan/Newton.h:135-232, 243-429; sdotplan/Report.h:33-57);
 *   - the driver: start selection (given / Voronoi / similarity), nu rescaled to the domain mass,
 *     width continuation stages, final moments on the true density (sdotplan/Solve.h:66-97, 111-371;
 *     sdotplan/Continuation.h:33-40; sdotplan/convolved/SumOfGaussians.h:38-41);
 *   - cut identifiers: box sides are negative (-1 .. -2d), seeds are their user index
 *     (src/sdot/include/sdot/gpu/Cell2D.cuh:453-463);
 *   - 3D sums of gaussians: the reference integrates them on the CPU only, facets exactly and masses by
 *     adaptive quadrature (src/sdot/.../SumOfGaussians.cxx:120-210, PointwiseDensity.h); here both by
 *     adaptive Gauss product rules over tetrahedra / triangles (gauss_cell3, gauss_face3).
 * The neighbour search is a uniform grid visited ring by ring and stopped by a security radius (or,
 * `brute != 0`, every other seed) -- it changes what a cell costs, never what it is.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OD_CAP2 1024      /* polygon vertices, 2D */
#define OD_MAXF 160       /* faces of a 3D cell */
#define OD_MAXFV 96       /* vertices of one face */

enum { OD_OK = 0, OD_ERR_VERTICES = 1, OD_ERR_NEIGHBOURS = 2, OD_ERR_UNSUPPORTED = 3, OD_ERR_ARGS = 4 };
enum { DENS_UNIFORM = 0, DENS_IMAGE = 1, DENS_GAUSS = 2 };

/* ------------------------------------------------------------------------------------------------ */
/* Gauss-Legendre nodes on [-1, 1], computed once by Newton iteration on P_n                          */
/* ------------------------------------------------------------------------------------------------ */
#define GL_N 12
static double gl_x[ GL_N ], gl_w[ GL_N ];
static int gl_ready = 0;
#define TQ_N 6
static double tq_x[ TQ_N ], tq_w[ TQ_N ];      /* the same construction with 6 points: the tetrahedral rules */
static void gl_init( void ) {
    if ( gl_ready ) return;
    for ( int i = 0; i < GL_N; ++i ) {
        double x = cos( M_PI * ( i + 0.75 ) / ( GL_N + 0.5 ) ), dp = 0;
        for ( int it = 0; it < 100; ++it ) {
            double p0 = 1, p1 = x;
            for ( int k = 2; k <= GL_N; ++k ) { double p2 = ( ( 2 * k - 1 ) * x * p1 - ( k - 1 ) * p0 ) / k; p0 = p1; p1 = p2; }
            dp = GL_N * ( x * p1 - p0 ) / ( x * x - 1 );
            double dx = p1 / dp;
            x -= dx;
            if ( fabs( dx ) < 1e-16 ) break;
        }
        gl_x[ i ] = x;
        gl_w[ i ] = 2 / ( ( 1 - x * x ) * dp * dp );
    }
    for ( int i = 0; i < TQ_N; ++i ) {
        double x = cos( M_PI * ( i + 0.75 ) / ( TQ_N + 0.5 ) ), dp = 0;
        for ( int it = 0; it < 100; ++it ) {
            double p0 = 1, p1 = x;
            for ( int k = 2; k <= TQ_N; ++k ) { double p2 = ( ( 2 * k - 1 ) * x * p1 - ( k - 1 ) * p0 ) / k; p0 = p1; p1 = p2; }
            dp = TQ_N * ( x * p1 - p0 ) / ( x * x - 1 );
            double dx = p1 / dp;
            x -= dx;
            if ( fabs( dx ) < 1e-16 ) break;
        }
        tq_x[ i ] = x;
        tq_w[ i ] = 2 / ( ( 1 - x * x ) * dp * dp );
    }
    gl_ready = 1;
}

/* ------------------------------------------------------------------------------------------------ */
/* the problem: seeds, domain box, density                                                         */
/* ------------------------------------------------------------------------------------------------ */
typedef struct {
    int dim;
    long n;
    const double *pos;      /* [n, dim] */
    const double *w;        /* [n] or NULL */
    double lo[ 3 ], hi[ 3 ];
    int dkind;
    const double *dpar;     /* uniform: [rho]; image: [x0,y0,hx,hy,nx,ny]; gauss: [ng] */
    const double *dval;     /* image: values [nx*ny], i along x; gauss: [ng, dim+2] = centre, sigma, mass */
    /* the search grid */
    int g[ 3 ];
    double go[ 3 ], gh[ 3 ], ghmin;
    long *cstart, *citems;
    double wmax;
} od_pb;

static double wt( const od_pb *pb, long i ) { return pb->w ? pb->w[ i ] : 0.0; }

static void build_grid( od_pb *pb ) {
    int d = pb->dim;
    double lo[ 3 ], hi[ 3 ];
    for ( int a = 0; a < d; ++a ) { lo[ a ] = pb->lo[ a ]; hi[ a ] = pb->hi[ a ]; }
    for ( long i = 0; i < pb->n; ++i )
        for ( int a = 0; a < d; ++a ) {
            double x = pb->pos[ i * d + a ];
            if ( x < lo[ a ] ) lo[ a ] = x;
            if ( x > hi[ a ] ) hi[ a ] = x;
        }
    double vol = 1;
    for ( int a = 0; a < d; ++a ) vol *= ( hi[ a ] - lo[ a ] ) > 0 ? ( hi[ a ] - lo[ a ] ) : 1;
    double target = pb->n / 2.0 > 1 ? pb->n / 2.0 : 1;      /* ~2 seeds per grid cell */
    double h = pow( vol / target, 1.0 / d );
    long total = 1;
    pb->ghmin = 1e300;
    for ( int a = 0; a < d; ++a ) {
        double ext = hi[ a ] - lo[ a ];
        int ga = ext > 0 ? ( int ) ceil( ext / h ) : 1;
        if ( ga < 1 ) ga = 1;
        if ( ga > 4096 ) ga = 4096;
        pb->g[ a ] = ga;
        pb->go[ a ] = lo[ a ];
        pb->gh[ a ] = ext > 0 ? ext / ga : 1;
        if ( pb->gh[ a ] < pb->ghmin ) pb->ghmin = pb->gh[ a ];
        total *= ga;
    }
    for ( int a = d; a < 3; ++a ) { pb->g[ a ] = 1; pb->go[ a ] = 0; pb->gh[ a ] = 1; }
    pb->cstart = ( long * ) calloc( total + 1, sizeof( long ) );
    pb->citems = ( long * ) malloc( ( pb->n > 0 ? pb->n : 1 ) * sizeof( long ) );
    long *cell_of = ( long * ) malloc( ( pb->n > 0 ? pb->n : 1 ) * sizeof( long ) );
    pb->wmax = -1e300;
    for ( long i = 0; i < pb->n; ++i ) {
        long c = 0;
        for ( int a = d - 1; a >= 0; --a ) {
            int k = ( int ) floor( ( pb->pos[ i * d + a ] - pb->go[ a ] ) / pb->gh[ a ] );
            if ( k < 0 ) k = 0;
            if ( k >= pb->g[ a ] ) k = pb->g[ a ] - 1;
            c = c * pb->g[ a ] + k;
        }
        cell_of[ i ] = c;
        pb->cstart[ c + 1 ]++;
        if ( wt( pb, i ) > pb->wmax ) pb->wmax = wt( pb, i );
    }
    for ( long c = 0; c < total; ++c ) pb->cstart[ c + 1 ] += pb->cstart[ c ];
    long *fill = ( long * ) malloc( ( total + 1 ) * sizeof( long ) );
    memcpy( fill, pb->cstart, ( total + 1 ) * sizeof( long ) );
    for ( long i = 0; i < pb->n; ++i ) pb->citems[ fill[ cell_of[ i ] ]++ ] = i;
    free( fill );
    free( cell_of );
}

static void free_grid( od_pb *pb ) { free( pb->cstart ); free( pb->citems ); }

/* ------------------------------------------------------------------------------------------------ */
/* 2D polygon in the frame of its seed: vertex k and the cut id of the edge k -> k+1                */
/* ------------------------------------------------------------------------------------------------ */
typedef struct { int m; double x[ OD_CAP2 ], y[ OD_CAP2 ]; int id[ OD_CAP2 ]; } poly2;

/* keep `nx x + ny y <= off`; returns 0, or -1 past the capacity */
static int clip2( poly2 *P, double nx, double ny, double off, int cid, poly2 *T ) {
    int m = P->m, nout = 0;
    if ( m == 0 ) return 0;
    double s[ OD_CAP2 ];
    for ( int k = 0; k < m; ++k ) { s[ k ] = nx * P->x[ k ] + ny * P->y[ k ] - off; nout += s[ k ] > 0; }
    if ( nout == 0 ) return 0;
    if ( nout == m ) { P->m = 0; return 0; }
    int q = 0;
    for ( int k = 0; k < m; ++k ) {
        int k1 = k + 1 == m ? 0 : k + 1;
        if ( q + 2 >= OD_CAP2 ) return -1;
        if ( s[ k ] <= 0 ) {
            T->x[ q ] = P->x[ k ]; T->y[ q ] = P->y[ k ];
            if ( s[ k1 ] > 0 ) {
                T->id[ q++ ] = P->id[ k ];
                double t = s[ k ] / ( s[ k ] - s[ k1 ] );
                T->x[ q ] = P->x[ k ] + t * ( P->x[ k1 ] - P->x[ k ] );
                T->y[ q ] = P->y[ k ] + t * ( P->y[ k1 ] - P->y[ k ] );
                T->id[ q++ ] = cid;
            } else
                T->id[ q++ ] = P->id[ k ];
        } else if ( s[ k1 ] <= 0 ) {
            double t = s[ k ] / ( s[ k ] - s[ k1 ] );
            T->x[ q ] = P->x[ k ] + t * ( P->x[ k1 ] - P->x[ k ] );
            T->y[ q ] = P->y[ k ] + t * ( P->y[ k1 ] - P->y[ k ] );
            T->id[ q++ ] = P->id[ k ];
        }
    }
    T->m = q;
    memcpy( P->x, T->x, q * sizeof( double ) );
    memcpy( P->y, T->y, q * sizeof( double ) );
    memcpy( P->id, T->id, q * sizeof( int ) );
    P->m = q;
    return 0;
}

/* area, first moment and `int |y|^2` of a polygon (uniform density 1), in its own frame */
static void poly2_integrals( const poly2 *P, double *A, double *Fx, double *Fy, double *S ) {
    double a = 0, fx = 0, fy = 0, s = 0;
    for ( int k = 0; k < P->m; ++k ) {
        int k1 = k + 1 == P->m ? 0 : k + 1;
        double x0 = P->x[ k ], y0 = P->y[ k ], x1 = P->x[ k1 ], y1 = P->y[ k1 ];
        double c = x0 * y1 - x1 * y0;
        a += c;
        fx += ( x0 + x1 ) * c;
        fy += ( y0 + y1 ) * c;
        s += c * ( x0 * x0 + x0 * x1 + x1 * x1 + y0 * y0 + y0 * y1 + y1 * y1 );
    }
    *A = a / 2; *Fx = fx / 6; *Fy = fy / 6; *S = s / 12;
}

/* ---- image density (2D, axis aligned pixels; values[ i * ny + j ], i along x) ------------------ */
static void image_cell2( const od_pb *pb, const poly2 *P, double px, double py, double *M, double *Fx, double *Fy, double *S ) {
    const double x0 = pb->dpar[ 0 ] - px, y0 = pb->dpar[ 1 ] - py, hx = pb->dpar[ 2 ], hy = pb->dpar[ 3 ];
    const int nx = ( int ) pb->dpar[ 4 ], ny = ( int ) pb->dpar[ 5 ];
    double m = 0, fx = 0, fy = 0, s = 0;
    *M = *Fx = *Fy = *S = 0;
    if ( P->m == 0 ) return;
    double ylo = 1e300, yhi = -1e300;
    for ( int k = 0; k < P->m; ++k ) { if ( P->y[ k ] < ylo ) ylo = P->y[ k ]; if ( P->y[ k ] > yhi ) yhi = P->y[ k ]; }
    int j0 = ( int ) floor( ( ylo - y0 ) / hy ), j1 = ( int ) floor( ( yhi - y0 ) / hy );
    if ( j0 < 0 ) j0 = 0;
    if ( j1 > ny - 1 ) j1 = ny - 1;
    poly2 *R = ( poly2 * ) malloc( sizeof( poly2 ) ), *C = ( poly2 * ) malloc( sizeof( poly2 ) ), *T = ( poly2 * ) malloc( sizeof( poly2 ) );
    for ( int j = j0; j <= j1; ++j ) {
        *R = *P;
        clip2( R, 0, 1, y0 + ( j + 1 ) * hy, -100, T );
        clip2( R, 0, -1, -( y0 + j * hy ), -100, T );
        if ( R->m == 0 ) continue;
        double xlo = 1e300, xhi = -1e300;
        for ( int k = 0; k < R->m; ++k ) { if ( R->x[ k ] < xlo ) xlo = R->x[ k ]; if ( R->x[ k ] > xhi ) xhi = R->x[ k ]; }
        int i0 = ( int ) floor( ( xlo - x0 ) / hx ), i1 = ( int ) floor( ( xhi - x0 ) / hx );
        if ( i0 < 0 ) i0 = 0;
        if ( i1 > nx - 1 ) i1 = nx - 1;
        for ( int i = i0; i <= i1; ++i ) {
            double v = pb->dval[ ( long ) i * ny + j ];
            if ( v == 0 ) continue;
            *C = *R;
            clip2( C, 1, 0, x0 + ( i + 1 ) * hx, -100, T );
            clip2( C, -1, 0, -( x0 + i * hx ), -100, T );
            if ( C->m == 0 ) continue;
            double a, gx, gy, g2;
            poly2_integrals( C, &a, &gx, &gy, &g2 );
            m += v * a; fx += v * gx; fy += v * gy; s += v * g2;
        }
    }
    free( R ); free( C ); free( T );
    *M = m; *Fx = fx; *Fy = fy; *S = s;
}

/* `int_segment rho ds` for the image: the segment cut at every pixel line, each piece weighted by its pixel */
static int cmp_dbl( const void *a, const void *b ) { double x = *( const double * ) a, y = *( const double * ) b; return ( x > y ) - ( x < y ); }
static double image_segment2( const od_pb *pb, double ax, double ay, double bx, double by ) {
    const double x0 = pb->dpar[ 0 ], y0 = pb->dpar[ 1 ], hx = pb->dpar[ 2 ], hy = pb->dpar[ 3 ];
    const int nx = ( int ) pb->dpar[ 4 ], ny = ( int ) pb->dpar[ 5 ];
    double len = hypot( bx - ax, by - ay );
    if ( len == 0 ) return 0;
    int cap = 4 + 2 * ( nx + ny + 2 ), nt = 0;
    double *ts = ( double * ) malloc( cap * sizeof( double ) );
    ts[ nt++ ] = 0; ts[ nt++ ] = 1;
    if ( bx != ax ) {
        double lo = ax < bx ? ax : bx, hi = ax < bx ? bx : ax;
        for ( int i = ( int ) ceil( ( lo - x0 ) / hx ); i <= ( int ) floor( ( hi - x0 ) / hx ) && nt < cap; ++i ) {
            if ( i < 0 || i > nx ) continue;
            double t = ( x0 + i * hx - ax ) / ( bx - ax );
            if ( t > 0 && t < 1 ) ts[ nt++ ] = t;
        }
    }
    if ( by != ay ) {
        double lo = ay < by ? ay : by, hi = ay < by ? by : ay;
        for ( int j = ( int ) ceil( ( lo - y0 ) / hy ); j <= ( int ) floor( ( hi - y0 ) / hy ) && nt < cap; ++j ) {
            if ( j < 0 || j > ny ) continue;
            double t = ( y0 + j * hy - ay ) / ( by - ay );
            if ( t > 0 && t < 1 ) ts[ nt++ ] = t;
        }
    }
    qsort( ts, nt, sizeof( double ), cmp_dbl );
    double res = 0;
    for ( int k = 0; k + 1 < nt; ++k ) {
        double tm = 0.5 * ( ts[ k ] + ts[ k + 1 ] );
        double mx = ax + tm * ( bx - ax ), my = ay + tm * ( by - ay );
        int i = ( int ) floor( ( mx - x0 ) / hx ), j = ( int ) floor( ( my - y0 ) / hy );
        if ( i < 0 || j < 0 || i >= nx || j >= ny ) continue;
        res += pb->dval[ ( long ) i * ny + j ] * ( ts[ k + 1 ] - ts[ k ] ) * len;
    }
    free( ts );
    return res;
}

/* ---- sums of isotropic gaussians (2D) ------------------------------------------------------------
 * The mass, first and second moments of a gaussian centred at c over a polygon are sums, over its
 * edges, of the integrals over the signed triangles (c, v_k, v_k+1).  In polar coordinates about c the
 * radial integrals have closed forms (below) and the angle is integrated by adaptive Gauss-Legendre. */
typedef struct { double h, tn, s2; } gtri;      /* distance from c to the edge line, angle of its normal, sigma^2 */
static void g_radial( double R, double sig, double *i1, double *i2, double *i3 ) {
    /* i1 = int_0^R r e^{-r^2/2s^2} dr, i2 = int_0^R r^2 e^..., i3 = int_0^R r^3 e^... */
    double u = R / sig, e = exp( -0.5 * u * u );
    *i1 = sig * sig * ( 1 - e );
    *i2 = sig * sig * sig * ( sqrt( M_PI / 2 ) * erf( u / sqrt( 2.0 ) ) - u * e );
    *i3 = sig * sig * sig * sig * ( 2 - ( 2 + u * u ) * e );
}
static void g_integrand( const gtri *g, double th, double out[ 4 ] ) {
    double c = cos( th - g->tn );
    double R = c > 1e-300 ? g->h / c : 1e300;
    double sig = sqrt( g->s2 ), i1, i2, i3;
    if ( R > 40 * sig ) R = 40 * sig;
    g_radial( R, sig, &i1, &i2, &i3 );
    out[ 0 ] = i1; out[ 1 ] = i2 * cos( th ); out[ 2 ] = i2 * sin( th ); out[ 3 ] = i3;
}
static void g_gl( const gtri *g, double a, double b, double out[ 4 ] ) {
    double v[ 4 ];
    out[ 0 ] = out[ 1 ] = out[ 2 ] = out[ 3 ] = 0;
    for ( int k = 0; k < GL_N; ++k ) {
        g_integrand( g, 0.5 * ( a + b ) + 0.5 * ( b - a ) * gl_x[ k ], v );
        for ( int q = 0; q < 4; ++q ) out[ q ] += gl_w[ k ] * v[ q ];
    }
    for ( int q = 0; q < 4; ++q ) out[ q ] *= 0.5 * ( b - a );
}
static void g_adapt( const gtri *g, double a, double b, const double whole[ 4 ], double tol, int depth, double out[ 4 ] ) {
    double l[ 4 ], r[ 4 ], m = 0.5 * ( a + b );
    g_gl( g, a, m, l );
    g_gl( g, m, b, r );
    double err = 0, mag = 0;
    for ( int q = 0; q < 4; ++q ) { err = fmax( err, fabs( l[ q ] + r[ q ] - whole[ q ] ) ); mag = fmax( mag, fabs( l[ q ] ) + fabs( r[ q ] ) ); }
    /* the tolerance is absolute and the same at every level; the rounding floor and a depth cap end it */
    if ( err <= tol || err <= 1e-15 * mag || depth >= 18 ) { for ( int q = 0; q < 4; ++q ) out[ q ] = l[ q ] + r[ q ]; return; }
    double lo[ 4 ], ro[ 4 ];
    g_adapt( g, a, m, l, tol, depth + 1, lo );
    g_adapt( g, m, b, r, tol, depth + 1, ro );
    for ( int q = 0; q < 4; ++q ) out[ q ] = lo[ q ] + ro[ q ];
}
/* mass, first moment about the seed and `int |y|^2` of the gaussian (c, sig, mass mg) over polygon P (seed frame) */
static void gauss_cell2( const poly2 *P, double cx, double cy, double sig, double mg, double *M, double *Fx, double *Fy, double *S ) {
    double acc[ 4 ] = { 0, 0, 0, 0 };
    for ( int k = 0; k < P->m; ++k ) {
        int k1 = k + 1 == P->m ? 0 : k + 1;
        double ax = P->x[ k ] - cx, ay = P->y[ k ] - cy, bx = P->x[ k1 ] - cx, by = P->y[ k1 ] - cy;
        double cr = ax * by - ay * bx;
        double ex = bx - ax, ey = by - ay, el = hypot( ex, ey );
        if ( el == 0 ) continue;
        double h = fabs( cr ) / el;
        if ( h < 1e-300 ) continue;
        double ta = atan2( ay, ax ), tb = atan2( by, bx );
        double dt = tb - ta;
        while ( dt > M_PI ) dt -= 2 * M_PI;
        while ( dt < -M_PI ) dt += 2 * M_PI;
        /* the foot of the perpendicular from c on the edge line gives the angle of the normal */
        double t = -( ax * ex + ay * ey ) / ( el * el );
        double fx = ax + t * ex, fy = ay + t * ey;
        gtri g = { h, atan2( fy, fx ), sig * sig };
        double whole[ 4 ], r[ 4 ];
        double a = ta, b = ta + dt;
        g_gl( &g, a, b, whole );
        g_adapt( &g, a, b, whole, 1e-16 * sig * sig, 0, r );
        for ( int q = 0; q < 4; ++q ) acc[ q ] += r[ q ];
    }
    double k = mg / ( 2 * M_PI * sig * sig );
    double m0 = k * acc[ 0 ], f0x = k * acc[ 1 ], f0y = k * acc[ 2 ], s0 = k * acc[ 3 ];   /* about c */
    *M = m0;
    *Fx = f0x + cx * m0;
    *Fy = f0y + cy * m0;
    *S = s0 + 2 * ( cx * f0x + cy * f0y ) + ( cx * cx + cy * cy ) * m0;
}
/* `int_segment g ds` for one gaussian: closed form with erf / erfc */
static double gauss_segment( double ax, double ay, double bx, double by, double cx, double cy, double sig, double mg, int dim ) {
    double ex = bx - ax, ey = by - ay, el = hypot( ex, ey );
    if ( el == 0 ) return 0;
    double ux = ex / el, uy = ey / el;
    double s0 = ( ax - cx ) * ux + ( ay - cy ) * uy, s1 = s0 + el;
    double fx = ax - s0 * ux - cx, fy = ay - s0 * uy - cy;
    double h2 = fx * fx + fy * fy;
    double r2 = sqrt( 2.0 ) * sig, span;
    if ( s0 >= 0 ) span = erfc( s0 / r2 ) - erfc( s1 / r2 );
    else if ( s1 <= 0 ) span = erfc( -s1 / r2 ) - erfc( -s0 / r2 );
    else span = erf( s1 / r2 ) - erf( s0 / r2 );
    (void) dim;
    return mg / ( 2 * M_PI * sig * sig ) * exp( -h2 / ( 2 * sig * sig ) ) * sig * sqrt( M_PI / 2 ) * span;
}

/* the mass, first moment (about the seed) and second moment of a cell, and `int_edge rho`, 2D */
static void dens_cell2( const od_pb *pb, const poly2 *P, double px, double py, double *M, double *Fx, double *Fy, double *S ) {
    if ( pb->dkind == DENS_UNIFORM ) {
        double a, fx, fy, s;
        poly2_integrals( P, &a, &fx, &fy, &s );
        double r = pb->dpar[ 0 ];
        *M = r * a; *Fx = r * fx; *Fy = r * fy; *S = r * s;
    } else if ( pb->dkind == DENS_IMAGE ) {
        image_cell2( pb, P, px, py, M, Fx, Fy, S );
    } else {
        int ng = ( int ) pb->dpar[ 0 ];
        double m = 0, fx = 0, fy = 0, s = 0;
        for ( int g = 0; g < ng; ++g ) {
            const double *G = pb->dval + g * 4;
            double a, b, c, e;
            gauss_cell2( P, G[ 0 ] - px, G[ 1 ] - py, G[ 2 ], G[ 3 ], &a, &b, &c, &e );
            m += a; fx += b; fy += c; s += e;
        }
        *M = m; *Fx = fx; *Fy = fy; *S = s;
    }
}
static double dens_edge2( const od_pb *pb, double ax, double ay, double bx, double by ) {
    if ( pb->dkind == DENS_UNIFORM ) return pb->dpar[ 0 ] * hypot( bx - ax, by - ay );
    if ( pb->dkind == DENS_IMAGE ) return image_segment2( pb, ax, ay, bx, by );
    int ng = ( int ) pb->dpar[ 0 ];
    double r = 0;
    for ( int g = 0; g < ng; ++g ) {
        const double *G = pb->dval + g * 4;
        r += gauss_segment( ax, ay, bx, by, G[ 0 ], G[ 1 ], G[ 2 ], G[ 3 ], 2 );
    }
    return r;
}

/* ------------------------------------------------------------------------------------------------ */
/* 2D cells                                                                                        */
/* ------------------------------------------------------------------------------------------------ */
typedef struct {
    double *mass, *bary, *cost;       /* [n], [n, d], [n] -- each may be NULL */
    int cap;                          /* neighbours per cell in the tables below */
    int *nb;                          /* [n] facets towards seeds */
    int *nid;                         /* [n, cap] neighbour (user index) */
    double *nc;                       /* [n, cap] c_ij */
    double *nm;                       /* [n, cap] int_facet rho */
    int *nvert;                       /* [n] vertices of the cell (may be NULL) */
} od_out;

static int cell2( const od_pb *pb, long i, int brute, poly2 *P, poly2 *T ) {
    const double px = pb->pos[ 2 * i ], py = pb->pos[ 2 * i + 1 ], wi = wt( pb, i );
    P->m = 4;
    P->x[ 0 ] = pb->lo[ 0 ] - px; P->y[ 0 ] = pb->lo[ 1 ] - py; P->id[ 0 ] = -1;   /* bottom */
    P->x[ 1 ] = pb->hi[ 0 ] - px; P->y[ 1 ] = pb->lo[ 1 ] - py; P->id[ 1 ] = -2;   /* right */
    P->x[ 2 ] = pb->hi[ 0 ] - px; P->y[ 2 ] = pb->hi[ 1 ] - py; P->id[ 2 ] = -3;   /* top */
    P->x[ 3 ] = pb->lo[ 0 ] - px; P->y[ 3 ] = pb->hi[ 1 ] - py; P->id[ 3 ] = -4;   /* left */
#define CUT2( j ) do { \
        double qx = pb->pos[ 2 * ( j ) ] - px, qy = pb->pos[ 2 * ( j ) + 1 ] - py; \
        double off = 0.5 * ( ( wi - wt( pb, j ) ) + ( qx * qx + qy * qy ) ); \
        if ( clip2( P, qx, qy, off, ( int ) ( j ), T ) ) return OD_ERR_VERTICES; } while ( 0 )
    if ( brute ) {
        for ( long j = 0; j < pb->n && P->m; ++j ) if ( j != i ) CUT2( j );
        return OD_OK;
    }
    int cx = ( int ) floor( ( px - pb->go[ 0 ] ) / pb->gh[ 0 ] ), cy = ( int ) floor( ( py - pb->go[ 1 ] ) / pb->gh[ 1 ] );
    if ( cx < 0 ) cx = 0;
    if ( cx >= pb->g[ 0 ] ) cx = pb->g[ 0 ] - 1;
    if ( cy < 0 ) cy = 0;
    if ( cy >= pb->g[ 1 ] ) cy = pb->g[ 1 ] - 1;
    int rmax = pb->g[ 0 ] > pb->g[ 1 ] ? pb->g[ 0 ] : pb->g[ 1 ];
    for ( int r = 0; r <= rmax && P->m; ++r ) {
        for ( int dy = -r; dy <= r; ++dy ) {
            int y = cy + dy;
            if ( y < 0 || y >= pb->g[ 1 ] ) continue;
            int step = ( dy == -r || dy == r ) ? 1 : 2 * r;
            for ( int dx = -r; dx <= r; dx += step ) {
                int x = cx + dx;
                if ( x < 0 || x >= pb->g[ 0 ] ) { if ( step == 0 ) break; continue; }
                long c = ( long ) y * pb->g[ 0 ] + x;
                for ( long e = pb->cstart[ c ]; e < pb->cstart[ c + 1 ]; ++e ) {
                    long j = pb->citems[ e ];
                    if ( j != i ) CUT2( j );
                }
                if ( step == 0 ) break;
            }
        }
        /* the security radius: every unvisited seed is at least `r h` away */
        double R2 = 0;
        for ( int k = 0; k < P->m; ++k ) { double d2 = P->x[ k ] * P->x[ k ] + P->y[ k ] * P->y[ k ]; if ( d2 > R2 ) R2 = d2; }
        double R = sqrt( R2 ), ex = R2 + pb->wmax - wi;
        if ( r * pb->ghmin >= R + sqrt( ex > 0 ? ex : 0 ) ) break;
    }
#undef CUT2
    return OD_OK;
}

static int write2( const od_pb *pb, long i, long oi, const poly2 *P, const od_out *o ) {
    const double px = pb->pos[ 2 * i ], py = pb->pos[ 2 * i + 1 ];
    double M, Fx, Fy, S;
    dens_cell2( pb, P, px, py, &M, &Fx, &Fy, &S );
    if ( o->mass ) o->mass[ oi ] = M;
    if ( o->bary ) {
        o->bary[ 2 * oi ] = M > 0 ? px + Fx / M : px;
        o->bary[ 2 * oi + 1 ] = M > 0 ? py + Fy / M : py;
    }
    if ( o->cost ) o->cost[ oi ] = S;
    if ( o->nvert ) o->nvert[ oi ] = P->m;
    if ( o->nb ) {
        int c = 0;
        for ( int k = 0; k < P->m; ++k ) {
            int j = P->id[ k ];
            if ( j < 0 ) continue;
            if ( c >= o->cap ) { o->nb[ oi ] = c; return OD_ERR_NEIGHBOURS; }
            int k1 = k + 1 == P->m ? 0 : k + 1;
            double meas = dens_edge2( pb, P->x[ k ] + px, P->y[ k ] + py, P->x[ k1 ] + px, P->y[ k1 ] + py );
            double dx = pb->pos[ 2 * j ] - px, dy = pb->pos[ 2 * j + 1 ] - py;
            o->nid[ ( long ) oi * o->cap + c ] = j;
            o->nm[ ( long ) oi * o->cap + c ] = meas;
            o->nc[ ( long ) oi * o->cap + c ] = meas / ( 2 * sqrt( dx * dx + dy * dy ) );
            ++c;
        }
        o->nb[ oi ] = c;
    }
    return OD_OK;
}

/* ------------------------------------------------------------------------------------------------ */
/* 3D cells: a convex polyhedron as a list of planar faces, each a polygon in outward (CCW) order     */
/* ------------------------------------------------------------------------------------------------ */
typedef struct { double p[ 3 ]; } v3;
typedef struct {
    int nf;
    int id[ OD_MAXF ];
    double nrm[ OD_MAXF ][ 3 ];       /* outward normal direction (not normalised) */
    int nv[ OD_MAXF ];
    v3 v[ OD_MAXF ][ OD_MAXFV ];
} poly3;

static double dot3( const double *a, const double *b ) { return a[ 0 ] * b[ 0 ] + a[ 1 ] * b[ 1 ] + a[ 2 ] * b[ 2 ]; }

static void box3( poly3 *P, const double *lo, const double *hi ) {
    /* ids: -1 x=lo, -2 x=hi, -3 y=lo, -4 y=hi, -5 z=lo, -6 z=hi */
    static const int corner[ 6 ][ 4 ][ 3 ] = {
        { { 0, 0, 0 }, { 0, 0, 1 }, { 0, 1, 1 }, { 0, 1, 0 } },   /* x = lo, outward -x */
        { { 1, 0, 0 }, { 1, 1, 0 }, { 1, 1, 1 }, { 1, 0, 1 } },   /* x = hi */
        { { 0, 0, 0 }, { 1, 0, 0 }, { 1, 0, 1 }, { 0, 0, 1 } },   /* y = lo */
        { { 0, 1, 0 }, { 0, 1, 1 }, { 1, 1, 1 }, { 1, 1, 0 } },   /* y = hi */
        { { 0, 0, 0 }, { 0, 1, 0 }, { 1, 1, 0 }, { 1, 0, 0 } },   /* z = lo */
        { { 0, 0, 1 }, { 1, 0, 1 }, { 1, 1, 1 }, { 0, 1, 1 } },   /* z = hi */
    };
    P->nf = 6;
    for ( int f = 0; f < 6; ++f ) {
        P->id[ f ] = -1 - f;
        for ( int a = 0; a < 3; ++a ) P->nrm[ f ][ a ] = 0;
        P->nrm[ f ][ f / 2 ] = ( f & 1 ) ? 1 : -1;
        P->nv[ f ] = 4;
        for ( int k = 0; k < 4; ++k )
            for ( int a = 0; a < 3; ++a )
                P->v[ f ][ k ].p[ a ] = corner[ f ][ k ][ a ] ? hi[ a ] : lo[ a ];
    }
}

/* keep `n.x <= off`; the crossing points of the faces make the new face. 0, or -1 past a capacity */
static int clip3( poly3 *P, const double *n, double off, int cid ) {
    int nout = 0, ntot = 0;
    for ( int f = 0; f < P->nf; ++f )
        for ( int k = 0; k < P->nv[ f ]; ++k ) { ntot++; nout += dot3( n, P->v[ f ][ k ].p ) - off > 0; }
    if ( nout == 0 ) return 0;
    if ( nout == ntot ) { P->nf = 0; return 0; }
    v3 cross[ 4 * OD_MAXF ];
    int nc = 0, nf = 0;
    for ( int f = 0; f < P->nf; ++f ) {
        int m = P->nv[ f ], q = 0;
        double s[ OD_MAXFV ];
        v3 out[ OD_MAXFV ];
        for ( int k = 0; k < m; ++k ) s[ k ] = dot3( n, P->v[ f ][ k ].p ) - off;
        for ( int k = 0; k < m; ++k ) {
            int k1 = k + 1 == m ? 0 : k + 1;
            if ( q + 2 >= OD_MAXFV ) return -1;
            if ( s[ k ] <= 0 ) out[ q++ ] = P->v[ f ][ k ];
            /* a kept vertex ON the plane (to rounding) belongs to the new face although no edge of it crosses: on a
               grid the planes pass through vertices, and a section made of the crossings alone lost its corners */
            if ( s[ k ] <= 0 && fabs( s[ k ] ) <= 16 * DBL_EPSILON * ( sqrt( dot3( n, n ) * dot3( P->v[ f ][ k ].p, P->v[ f ][ k ].p ) ) + fabs( off ) ) ) {
                if ( nc >= 4 * OD_MAXF ) return -1;
                cross[ nc++ ] = P->v[ f ][ k ];
            }
            if ( ( s[ k ] <= 0 ) != ( s[ k1 ] <= 0 ) ) {
                /* from the kept end, whichever face reports the edge: the two faces of an edge then make the same point
                   to the bit (an edge nearly parallel to the plane would place its two copies far apart) */
                const int ui = s[ k ] <= 0 ? k : k1, vi = s[ k ] <= 0 ? k1 : k;
                double t = s[ ui ] / ( s[ ui ] - s[ vi ] );
                v3 x;
                for ( int a = 0; a < 3; ++a ) x.p[ a ] = P->v[ f ][ ui ].p[ a ] + t * ( P->v[ f ][ vi ].p[ a ] - P->v[ f ][ ui ].p[ a ] );
                out[ q++ ] = x;
                if ( nc >= 4 * OD_MAXF ) return -1;
                cross[ nc++ ] = x;
            }
        }
        if ( q >= 3 ) {
            P->id[ nf ] = P->id[ f ];
            for ( int a = 0; a < 3; ++a ) P->nrm[ nf ][ a ] = P->nrm[ f ][ a ];
            P->nv[ nf ] = q;
            for ( int k = 0; k < q; ++k ) P->v[ nf ][ k ] = out[ k ];
            ++nf;
        }
    }
    P->nf = nf;
    if ( nc < 3 ) return 0;
    /* the new face: the crossing points, each seen twice, without repeats, in angular order about n */
    double ctr[ 3 ] = { 0, 0, 0 }, scale = 0;
    for ( int k = 0; k < nc; ++k ) for ( int a = 0; a < 3; ++a ) ctr[ a ] += cross[ k ].p[ a ] / nc;
    for ( int k = 0; k < nc; ++k ) for ( int a = 0; a < 3; ++a ) scale = fmax( scale, fabs( cross[ k ].p[ a ] - ctr[ a ] ) );
    double e1[ 3 ], e2[ 3 ], nn = sqrt( dot3( n, n ) );
    double un[ 3 ] = { n[ 0 ] / nn, n[ 1 ] / nn, n[ 2 ] / nn };
    double t[ 3 ] = { 1, 0, 0 };
    if ( fabs( un[ 0 ] ) > 0.6 ) { t[ 0 ] = 0; t[ 1 ] = 1; }
    e1[ 0 ] = un[ 1 ] * t[ 2 ] - un[ 2 ] * t[ 1 ]; e1[ 1 ] = un[ 2 ] * t[ 0 ] - un[ 0 ] * t[ 2 ]; e1[ 2 ] = un[ 0 ] * t[ 1 ] - un[ 1 ] * t[ 0 ];
    double l1 = sqrt( dot3( e1, e1 ) );
    for ( int a = 0; a < 3; ++a ) e1[ a ] /= l1;
    e2[ 0 ] = un[ 1 ] * e1[ 2 ] - un[ 2 ] * e1[ 1 ]; e2[ 1 ] = un[ 2 ] * e1[ 0 ] - un[ 0 ] * e1[ 2 ]; e2[ 2 ] = un[ 0 ] * e1[ 1 ] - un[ 1 ] * e1[ 0 ];
    double ang[ 4 * OD_MAXF ];
    int ord[ 4 * OD_MAXF ];
    for ( int k = 0; k < nc; ++k ) {
        double d[ 3 ] = { cross[ k ].p[ 0 ] - ctr[ 0 ], cross[ k ].p[ 1 ] - ctr[ 1 ], cross[ k ].p[ 2 ] - ctr[ 2 ] };
        ang[ k ] = atan2( dot3( d, e2 ), dot3( d, e1 ) );
        ord[ k ] = k;
    }
    for ( int a = 1; a < nc; ++a ) {          /* insertion sort by angle */
        int o = ord[ a ], b = a;
        while ( b > 0 && ang[ ord[ b - 1 ] ] > ang[ o ] ) { ord[ b ] = ord[ b - 1 ]; --b; }
        ord[ b ] = o;
    }
    if ( nf >= OD_MAXF ) return -1;
    int q = 0;
    double tol = 1e-13 * ( scale > 0 ? scale : 1 );
    for ( int a = 0; a < nc; ++a ) {
        const v3 *x = &cross[ ord[ a ] ];
        if ( q > 0 ) {
            const v3 *y = &P->v[ nf ][ q - 1 ];
            if ( fabs( x->p[ 0 ] - y->p[ 0 ] ) <= tol && fabs( x->p[ 1 ] - y->p[ 1 ] ) <= tol && fabs( x->p[ 2 ] - y->p[ 2 ] ) <= tol ) continue;
        }
        if ( q >= OD_MAXFV ) return -1;
        P->v[ nf ][ q++ ] = *x;
    }
    while ( q > 1 ) {
        const v3 *x = &P->v[ nf ][ q - 1 ], *y = &P->v[ nf ][ 0 ];
        if ( fabs( x->p[ 0 ] - y->p[ 0 ] ) <= tol && fabs( x->p[ 1 ] - y->p[ 1 ] ) <= tol && fabs( x->p[ 2 ] - y->p[ 2 ] ) <= tol ) --q;
        else break;
    }
    if ( q >= 3 ) {
        P->id[ nf ] = cid;
        for ( int a = 0; a < 3; ++a ) P->nrm[ nf ][ a ] = n[ a ];
        P->nv[ nf ] = q;
        P->nf = nf + 1;
    }
    return 0;
}

static double face_area3( const poly3 *P, int f ) {
    double s[ 3 ] = { 0, 0, 0 };
    const v3 *V = P->v[ f ];
    for ( int k = 1; k + 1 < P->nv[ f ]; ++k ) {
        double a[ 3 ], b[ 3 ];
        for ( int q = 0; q < 3; ++q ) { a[ q ] = V[ k ].p[ q ] - V[ 0 ].p[ q ]; b[ q ] = V[ k + 1 ].p[ q ] - V[ 0 ].p[ q ]; }
        s[ 0 ] += a[ 1 ] * b[ 2 ] - a[ 2 ] * b[ 1 ]; s[ 1 ] += a[ 2 ] * b[ 0 ] - a[ 0 ] * b[ 2 ]; s[ 2 ] += a[ 0 ] * b[ 1 ] - a[ 1 ] * b[ 0 ];
    }
    double nn = sqrt( dot3( P->nrm[ f ], P->nrm[ f ] ) );
    return fabs( dot3( s, P->nrm[ f ] ) / nn ) / 2;
}

/* volume, first moment and `int |y|^2` of the polyhedron (frame of the seed) by tetrahedra from the origin */
static void poly3_integrals( const poly3 *P, double *V, double F[ 3 ], double *S ) {
    double vol = 0, f[ 3 ] = { 0, 0, 0 }, s = 0;
    for ( int fa = 0; fa < P->nf; ++fa ) {
        const v3 *X = P->v[ fa ];
        /* orient the fan outward: the sign of its normal against the stored outward direction */
        double nrm[ 3 ] = { 0, 0, 0 };
        for ( int k = 1; k + 1 < P->nv[ fa ]; ++k ) {
            double a[ 3 ], b[ 3 ];
            for ( int q = 0; q < 3; ++q ) { a[ q ] = X[ k ].p[ q ] - X[ 0 ].p[ q ]; b[ q ] = X[ k + 1 ].p[ q ] - X[ 0 ].p[ q ]; }
            nrm[ 0 ] += a[ 1 ] * b[ 2 ] - a[ 2 ] * b[ 1 ]; nrm[ 1 ] += a[ 2 ] * b[ 0 ] - a[ 0 ] * b[ 2 ]; nrm[ 2 ] += a[ 0 ] * b[ 1 ] - a[ 1 ] * b[ 0 ];
        }
        double sg = dot3( nrm, P->nrm[ fa ] ) >= 0 ? 1 : -1;
        for ( int k = 1; k + 1 < P->nv[ fa ]; ++k ) {
            const double *a = X[ 0 ].p, *b = X[ k ].p, *c = X[ k + 1 ].p;
            double det = a[ 0 ] * ( b[ 1 ] * c[ 2 ] - b[ 2 ] * c[ 1 ] ) - a[ 1 ] * ( b[ 0 ] * c[ 2 ] - b[ 2 ] * c[ 0 ] ) + a[ 2 ] * ( b[ 0 ] * c[ 1 ] - b[ 1 ] * c[ 0 ] );
            double tv = sg * det / 6;
            vol += tv;
            for ( int q = 0; q < 3; ++q ) f[ q ] += tv * ( a[ q ] + b[ q ] + c[ q ] ) / 4;
            s += tv / 10 * ( dot3( a, a ) + dot3( b, b ) + dot3( c, c ) + dot3( a, b ) + dot3( a, c ) + dot3( b, c ) );
        }
    }
    *V = vol; F[ 0 ] = f[ 0 ]; F[ 1 ] = f[ 1 ]; F[ 2 ] = f[ 2 ]; *S = s;
}

/* ---- sums of isotropic gaussians (3D) ------------------------------------------------------------
 * Volume quadrature, independent of any closed form: the polyhedron is cut into tetrahedra (a fan of each
 * face from the vertex mean), each integrated by the collapsed (Duffy) product of TQ_N-point Gauss-Legendre
 * rules and refined by 8-way subdivision until the children agree with their parent.  Faces likewise by
 * collapsed 2D rules and 4-way subdivision.  rho_g = m / ((2 pi)^{3/2} s^3) exp(-|x - c|^2 / 2 s^2). */
typedef struct { double c[ 3 ], s, m, k; } g3;
static void g3_tet_rule( const g3 *g, const double T[ 4 ][ 3 ], double out[ 5 ] ) {
    double e1[ 3 ], e2[ 3 ], e3[ 3 ];
    for ( int q = 0; q < 3; ++q ) { e1[ q ] = T[ 1 ][ q ] - T[ 0 ][ q ]; e2[ q ] = T[ 2 ][ q ] - T[ 0 ][ q ]; e3[ q ] = T[ 3 ][ q ] - T[ 0 ][ q ]; }
    double vol6 = fabs( e1[ 0 ] * ( e2[ 1 ] * e3[ 2 ] - e2[ 2 ] * e3[ 1 ] ) - e1[ 1 ] * ( e2[ 0 ] * e3[ 2 ] - e2[ 2 ] * e3[ 0 ] ) +
                        e1[ 2 ] * ( e2[ 0 ] * e3[ 1 ] - e2[ 1 ] * e3[ 0 ] ) );
    for ( int q = 0; q < 5; ++q ) out[ q ] = 0;
    for ( int i = 0; i < TQ_N; ++i ) {
        double a = 0.5 * ( tq_x[ i ] + 1 ), wa = 0.5 * tq_w[ i ];
        for ( int j = 0; j < TQ_N; ++j ) {
            double b = 0.5 * ( tq_x[ j ] + 1 ), wb = 0.5 * tq_w[ j ];
            for ( int l = 0; l < TQ_N; ++l ) {
                double t = 0.5 * ( tq_x[ l ] + 1 ), wt_ = 0.5 * tq_w[ l ];
                double u = a, v = b * ( 1 - a ), z = t * ( 1 - a ) * ( 1 - b );
                double J = ( 1 - a ) * ( 1 - a ) * ( 1 - b ) * wa * wb * wt_ * vol6;
                double x[ 3 ], r2 = 0;
                for ( int q = 0; q < 3; ++q ) { x[ q ] = T[ 0 ][ q ] + u * e1[ q ] + v * e2[ q ] + z * e3[ q ]; r2 += ( x[ q ] - g->c[ q ] ) * ( x[ q ] - g->c[ q ] ); }
                double f = J * g->k * exp( -r2 / ( 2 * g->s * g->s ) );
                out[ 0 ] += f;
                out[ 1 ] += f * x[ 0 ]; out[ 2 ] += f * x[ 1 ]; out[ 3 ] += f * x[ 2 ];
                out[ 4 ] += f * ( x[ 0 ] * x[ 0 ] + x[ 1 ] * x[ 1 ] + x[ 2 ] * x[ 2 ] );
            }
        }
    }
}
static void g3_tet_adapt( const g3 *g, const double T[ 4 ][ 3 ], const double whole[ 5 ], int depth, double out[ 5 ] ) {
    double m[ 6 ][ 3 ];
    static const int pr[ 6 ][ 2 ] = { { 0, 1 }, { 0, 2 }, { 0, 3 }, { 1, 2 }, { 1, 3 }, { 2, 3 } };
    for ( int e = 0; e < 6; ++e ) for ( int q = 0; q < 3; ++q ) m[ e ][ q ] = 0.5 * ( T[ pr[ e ][ 0 ] ][ q ] + T[ pr[ e ][ 1 ] ][ q ] );
    /* the 8 children: 4 corners, and the inner octahedron cut along the diagonal m02-m13 */
    const double *C[ 8 ][ 4 ] = {
        { T[ 0 ], m[ 0 ], m[ 1 ], m[ 2 ] }, { m[ 0 ], T[ 1 ], m[ 3 ], m[ 4 ] }, { m[ 1 ], m[ 3 ], T[ 2 ], m[ 5 ] }, { m[ 2 ], m[ 4 ], m[ 5 ], T[ 3 ] },
        { m[ 0 ], m[ 1 ], m[ 2 ], m[ 4 ] }, { m[ 0 ], m[ 1 ], m[ 3 ], m[ 4 ] }, { m[ 1 ], m[ 2 ], m[ 4 ], m[ 5 ] }, { m[ 1 ], m[ 3 ], m[ 4 ], m[ 5 ] } };
    double ch[ 8 ][ 5 ], sum[ 5 ] = { 0, 0, 0, 0, 0 };
    double Tc[ 8 ][ 4 ][ 3 ];
    for ( int c = 0; c < 8; ++c ) {
        for ( int k = 0; k < 4; ++k ) for ( int q = 0; q < 3; ++q ) Tc[ c ][ k ][ q ] = C[ c ][ k ][ q ];
        g3_tet_rule( g, ( const double( * )[ 3 ] ) Tc[ c ], ch[ c ] );
        for ( int q = 0; q < 5; ++q ) sum[ q ] += ch[ c ][ q ];
    }
    double err = 0, mag = 0;
    for ( int q = 0; q < 5; ++q ) { err = fmax( err, fabs( sum[ q ] - whole[ q ] ) ); mag = fmax( mag, fabs( sum[ q ] ) ); }
    if ( err <= 1e-12 * mag + 1e-20 * g->m || depth >= 5 ) { for ( int q = 0; q < 5; ++q ) out[ q ] = sum[ q ]; return; }
    for ( int q = 0; q < 5; ++q ) out[ q ] = 0;
    for ( int c = 0; c < 8; ++c ) {
        double r[ 5 ];
        g3_tet_adapt( g, ( const double( * )[ 3 ] ) Tc[ c ], ch[ c ], depth + 1, r );
        for ( int q = 0; q < 5; ++q ) out[ q ] += r[ q ];
    }
}
static void g3_tri_rule( const g3 *g, const double *A, const double *B, const double *C, double *out ) {
    double e1[ 3 ], e2[ 3 ], cr[ 3 ];
    for ( int q = 0; q < 3; ++q ) { e1[ q ] = B[ q ] - A[ q ]; e2[ q ] = C[ q ] - A[ q ]; }
    cr[ 0 ] = e1[ 1 ] * e2[ 2 ] - e1[ 2 ] * e2[ 1 ]; cr[ 1 ] = e1[ 2 ] * e2[ 0 ] - e1[ 0 ] * e2[ 2 ]; cr[ 2 ] = e1[ 0 ] * e2[ 1 ] - e1[ 1 ] * e2[ 0 ];
    double area2 = sqrt( dot3( cr, cr ) );
    *out = 0;
    for ( int i = 0; i < GL_N; ++i ) {
        double a = 0.5 * ( gl_x[ i ] + 1 ), wa = 0.5 * gl_w[ i ];
        for ( int j = 0; j < GL_N; ++j ) {
            double b = 0.5 * ( gl_x[ j ] + 1 ), wb = 0.5 * gl_w[ j ];
            double u = a, v = b * ( 1 - a ), r2 = 0;
            for ( int q = 0; q < 3; ++q ) { double x = A[ q ] + u * e1[ q ] + v * e2[ q ]; r2 += ( x - g->c[ q ] ) * ( x - g->c[ q ] ); }
            *out += wa * wb * ( 1 - a ) * area2 * g->k * exp( -r2 / ( 2 * g->s * g->s ) );
        }
    }
}
static double g3_tri_adapt( const g3 *g, const double *A, const double *B, const double *C, double whole, int depth ) {
    double ab[ 3 ], bc[ 3 ], ca[ 3 ];
    for ( int q = 0; q < 3; ++q ) { ab[ q ] = 0.5 * ( A[ q ] + B[ q ] ); bc[ q ] = 0.5 * ( B[ q ] + C[ q ] ); ca[ q ] = 0.5 * ( C[ q ] + A[ q ] ); }
    double r[ 4 ];
    g3_tri_rule( g, A, ab, ca, &r[ 0 ] ); g3_tri_rule( g, ab, B, bc, &r[ 1 ] ); g3_tri_rule( g, ca, bc, C, &r[ 2 ] ); g3_tri_rule( g, ab, bc, ca, &r[ 3 ] );
    double sum = r[ 0 ] + r[ 1 ] + r[ 2 ] + r[ 3 ];
    if ( fabs( sum - whole ) <= 1e-13 * fabs( sum ) + 1e-22 * g->m || depth >= 8 ) return sum;
    return g3_tri_adapt( g, A, ab, ca, r[ 0 ], depth + 1 ) + g3_tri_adapt( g, ab, B, bc, r[ 1 ], depth + 1 ) +
           g3_tri_adapt( g, ca, bc, C, r[ 2 ], depth + 1 ) + g3_tri_adapt( g, ab, bc, ca, r[ 3 ], depth + 1 );
}
static void g3_of( const od_pb *pb, int gi, const double *p, g3 *g ) {
    const double *G = pb->dval + gi * 5;
    for ( int q = 0; q < 3; ++q ) g->c[ q ] = G[ q ] - p[ q ];
    g->s = G[ 3 ]; g->m = G[ 4 ];
    g->k = g->m / ( pow( 2 * M_PI, 1.5 ) * g->s * g->s * g->s );
}
/* mass, first moment and `int |y|^2 rho` of the polyhedron (seed frame), summed over the gaussians */
static void gauss_cell3( const od_pb *pb, const poly3 *P, const double *p, double *M, double F[ 3 ], double *S ) {
    double apex[ 3 ] = { 0, 0, 0 };
    int cnt = 0;
    for ( int f = 0; f < P->nf; ++f )
        for ( int k = 0; k < P->nv[ f ]; ++k ) { for ( int q = 0; q < 3; ++q ) apex[ q ] += P->v[ f ][ k ].p[ q ]; ++cnt; }
    for ( int q = 0; q < 3; ++q ) apex[ q ] /= cnt ? cnt : 1;
    double acc[ 5 ] = { 0, 0, 0, 0, 0 };
    const int ng = ( int ) pb->dpar[ 0 ];
    for ( int gi = 0; gi < ng; ++gi ) {
        g3 g;
        g3_of( pb, gi, p, &g );
        for ( int f = 0; f < P->nf; ++f )
            for ( int k = 1; k + 1 < P->nv[ f ]; ++k ) {
                double T[ 4 ][ 3 ];
                for ( int q = 0; q < 3; ++q ) {
                    T[ 0 ][ q ] = apex[ q ]; T[ 1 ][ q ] = P->v[ f ][ 0 ].p[ q ]; T[ 2 ][ q ] = P->v[ f ][ k ].p[ q ]; T[ 3 ][ q ] = P->v[ f ][ k + 1 ].p[ q ];
                }
                double whole[ 5 ], r[ 5 ];
                g3_tet_rule( &g, ( const double( * )[ 3 ] ) T, whole );
                g3_tet_adapt( &g, ( const double( * )[ 3 ] ) T, whole, 0, r );
                for ( int q = 0; q < 5; ++q ) acc[ q ] += r[ q ];
            }
    }
    *M = acc[ 0 ]; F[ 0 ] = acc[ 1 ]; F[ 1 ] = acc[ 2 ]; F[ 2 ] = acc[ 3 ]; *S = acc[ 4 ];
}
/* `int_face rho` of face f (seed frame) */
static double gauss_face3( const od_pb *pb, const poly3 *P, int f, const double *p ) {
    const int ng = ( int ) pb->dpar[ 0 ];
    double r = 0;
    for ( int gi = 0; gi < ng; ++gi ) {
        g3 g;
        g3_of( pb, gi, p, &g );
        for ( int k = 1; k + 1 < P->nv[ f ]; ++k ) {
            const double *A = P->v[ f ][ 0 ].p, *B = P->v[ f ][ k ].p, *C = P->v[ f ][ k + 1 ].p;
            double whole;
            g3_tri_rule( &g, A, B, C, &whole );
            r += g3_tri_adapt( &g, A, B, C, whole, 0 );
        }
    }
    return r;
}

static int cell3( const od_pb *pb, long i, int brute, poly3 *P ) {
    const double *p = pb->pos + 3 * i, wi = wt( pb, i );
    double lo[ 3 ], hi[ 3 ];
    for ( int a = 0; a < 3; ++a ) { lo[ a ] = pb->lo[ a ] - p[ a ]; hi[ a ] = pb->hi[ a ] - p[ a ]; }
    box3( P, lo, hi );
#define CUT3( j ) do { \
        double q[ 3 ] = { pb->pos[ 3 * ( j ) ] - p[ 0 ], pb->pos[ 3 * ( j ) + 1 ] - p[ 1 ], pb->pos[ 3 * ( j ) + 2 ] - p[ 2 ] }; \
        double off = 0.5 * ( ( wi - wt( pb, j ) ) + dot3( q, q ) ); \
        if ( clip3( P, q, off, ( int ) ( j ) ) ) return OD_ERR_VERTICES; } while ( 0 )
    if ( brute ) {
        for ( long j = 0; j < pb->n && P->nf; ++j ) if ( j != i ) CUT3( j );
        return OD_OK;
    }
    int c0[ 3 ];
    for ( int a = 0; a < 3; ++a ) {
        c0[ a ] = ( int ) floor( ( p[ a ] - pb->go[ a ] ) / pb->gh[ a ] );
        if ( c0[ a ] < 0 ) c0[ a ] = 0;
        if ( c0[ a ] >= pb->g[ a ] ) c0[ a ] = pb->g[ a ] - 1;
    }
    int rmax = pb->g[ 0 ];
    if ( pb->g[ 1 ] > rmax ) rmax = pb->g[ 1 ];
    if ( pb->g[ 2 ] > rmax ) rmax = pb->g[ 2 ];
    for ( int r = 0; r <= rmax && P->nf; ++r ) {
        for ( int dz = -r; dz <= r; ++dz ) {
            int z = c0[ 2 ] + dz;
            if ( z < 0 || z >= pb->g[ 2 ] ) continue;
            for ( int dy = -r; dy <= r; ++dy ) {
                int y = c0[ 1 ] + dy;
                if ( y < 0 || y >= pb->g[ 1 ] ) continue;
                int shell = dz == -r || dz == r || dy == -r || dy == r;
                int step = shell ? 1 : 2 * r;
                for ( int dx = -r; dx <= r; dx += ( step ? step : 1 ) ) {
                    int x = c0[ 0 ] + dx;
                    if ( x >= 0 && x < pb->g[ 0 ] ) {
                        long c = ( ( long ) z * pb->g[ 1 ] + y ) * pb->g[ 0 ] + x;
                        for ( long e = pb->cstart[ c ]; e < pb->cstart[ c + 1 ]; ++e ) {
                            long j = pb->citems[ e ];
                            if ( j != i ) CUT3( j );
                        }
                    }
                    if ( step == 0 ) break;
                }
            }
        }
        double R2 = 0;
        for ( int f = 0; f < P->nf; ++f )
            for ( int k = 0; k < P->nv[ f ]; ++k ) { double d2 = dot3( P->v[ f ][ k ].p, P->v[ f ][ k ].p ); if ( d2 > R2 ) R2 = d2; }
        double R = sqrt( R2 ), ex = R2 + pb->wmax - wi;
        if ( r * pb->ghmin >= R + sqrt( ex > 0 ? ex : 0 ) ) break;
    }
#undef CUT3
    return OD_OK;
}

static int write3( const od_pb *pb, long i, long oi, const poly3 *P, const od_out *o ) {
    const double *p = pb->pos + 3 * i;
    double V, F[ 3 ], S, M;
    const int gauss = pb->dkind == DENS_GAUSS;
    double r = gauss ? 1.0 : pb->dpar[ 0 ];
    if ( gauss ) {
        M = S = F[ 0 ] = F[ 1 ] = F[ 2 ] = 0;
        if ( o->mass || o->bary || o->cost ) gauss_cell3( pb, P, p, &M, F, &S );   /* facets only: no volume quadrature */
        V = M;
    } else {
        poly3_integrals( P, &V, F, &S );
        M = r * V;
        S *= r;
    }
    if ( o->mass ) o->mass[ oi ] = M;
    if ( o->bary ) for ( int a = 0; a < 3; ++a ) o->bary[ 3 * oi + a ] = V > 0 ? p[ a ] + F[ a ] / V : p[ a ];
    if ( o->cost ) o->cost[ oi ] = S;
    if ( o->nvert ) {
        int nv = 0;
        for ( int f = 0; f < P->nf; ++f ) nv += P->nv[ f ];
        o->nvert[ oi ] = nv;
    }
    if ( o->nb ) {
        int c = 0;
        for ( int f = 0; f < P->nf; ++f ) {
            int j = P->id[ f ];
            if ( j < 0 ) continue;
            if ( c >= o->cap ) { o->nb[ oi ] = c; return OD_ERR_NEIGHBOURS; }
            double meas = gauss ? gauss_face3( pb, P, f, p ) : r * face_area3( P, f );
            double q[ 3 ] = { pb->pos[ 3 * j ] - p[ 0 ], pb->pos[ 3 * j + 1 ] - p[ 1 ], pb->pos[ 3 * j + 2 ] - p[ 2 ] };
            o->nid[ ( long ) oi * o->cap + c ] = j;
            o->nm[ ( long ) oi * o->cap + c ] = meas;
            o->nc[ ( long ) oi * o->cap + c ] = meas / ( 2 * sqrt( dot3( q, q ) ) );
            ++c;
        }
        o->nb[ oi ] = c;
    }
    return OD_OK;
}

/* ------------------------------------------------------------------------------------------------ */
/* one diagram: every cell, in parallel                                                           */
/* ------------------------------------------------------------------------------------------------ */
/* `rows` (NULL: every cell) the cells to compute, `nrows` of them, output k for cell rows[ k ] */
static int diagram_rows( od_pb *pb, int brute, const od_out *o, long nrows, const long *rows, long *bad ) {
    int status = OD_OK;
    long first_bad = -1;
    if ( pb->dim == 3 && pb->dkind == DENS_IMAGE ) return OD_ERR_UNSUPPORTED;
    gl_init();
    build_grid( pb );
    const long count = rows ? nrows : pb->n;
#pragma omp parallel
    {
        void *buf = malloc( pb->dim == 2 ? 2 * sizeof( poly2 ) : sizeof( poly3 ) );
#pragma omp for schedule( dynamic, 4 )
        for ( long k = 0; k < count; ++k ) {
            const long i = rows ? rows[ k ] : k;
            int st;
            if ( pb->dim == 2 ) {
                poly2 *P = ( poly2 * ) buf, *T = P + 1;
                st = cell2( pb, i, brute, P, T );
                if ( st == OD_OK ) st = write2( pb, i, k, P, o );
            } else {
                poly3 *P = ( poly3 * ) buf;
                st = cell3( pb, i, brute, P );
                if ( st == OD_OK ) st = write3( pb, i, k, P, o );
            }
            if ( st != OD_OK ) {
#pragma omp critical
                { if ( status == OD_OK ) { status = st; first_bad = i; } }
            }
        }
        free( buf );
    }
    free_grid( pb );
    if ( bad ) *bad = first_bad;
    return status;
}

static int diagram( od_pb *pb, int brute, const od_out *o, long *bad ) { return diagram_rows( pb, brute, o, 0, NULL, bad ); }

static void init_pb( od_pb *pb, int dim, long n, const double *pos, const double *w, const double *box, int dkind, const double *dpar, const double *dval ) {
    memset( pb, 0, sizeof( *pb ) );
    pb->dim = dim; pb->n = n; pb->pos = pos; pb->w = w;
    for ( int a = 0; a < dim; ++a ) { pb->lo[ a ] = box[ a ]; pb->hi[ a ] = box[ dim + a ]; }
    pb->dkind = dkind; pb->dpar = dpar; pb->dval = dval;
}

/* THE CELLS: `box` = [lo..., hi...]; outputs may be NULL; returns a status, `bad` the first failing seed */
int od_cells( int dim, long n, const double *pos, const double *w, const double *box, int dkind, const double *dpar, const double *dval,
              int brute, double *mass, double *bary, double *cost, int cap, int *nb, int *nid, double *nc, double *nm, int *nvert, long *bad ) {
    if ( dim != 2 && dim != 3 ) return OD_ERR_ARGS;
    od_pb pb;
    init_pb( &pb, dim, n, pos, w, box, dkind, dpar, dval );
    od_out o = { mass, bary, cost, cap, nb, nid, nc, nm, nvert };
    return diagram( &pb, brute, &o, bad );
}

/* THE CELLS of a subset: the diagram of all the seeds, computed for cells rows[ 0 .. nrows ) only; output k (every output
   array holds nrows rows) is cell rows[ k ]'s; `bad` the first failing seed */
int od_cells_rows( int dim, long n, const double *pos, const double *w, const double *box, int dkind, const double *dpar,
                   const double *dval, long nrows, const long *rows, double *mass, double *bary, double *cost, int cap, int *nb, int *nid,
                   double *nc, double *nm, int *nvert, long *bad ) {
    if ( dim != 2 && dim != 3 ) return OD_ERR_ARGS;
    for ( long k = 0; k < nrows; ++k )
        if ( rows[ k ] < 0 || rows[ k ] >= n ) return OD_ERR_ARGS;
    od_pb pb;
    init_pb( &pb, dim, n, pos, w, box, dkind, dpar, dval );
    od_out o = { mass, bary, cost, cap, nb, nid, nc, nm, nvert };
    return diagram_rows( &pb, 0, &o, nrows, rows, bad );
}

int od_max_threads( void ) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void od_set_threads( int t ) {
#ifdef _OPENMP
    if ( t > 0 ) omp_set_num_threads( t );
#else
    (void) t;
#endif
}

/* ------------------------------------------------------------------------------------------------ */
/* the Laplacian (each row with its own facet measures) and the Jacobi-preconditioned CG           */
/* ------------------------------------------------------------------------------------------------ */
typedef struct { long n; long *row; long *col; double *c; double *dia; } od_lap;

static void lap_build( od_lap *L, long n, int cap, const int *nb, const int *nid, const double *nc ) {
    L->n = n;
    L->row = ( long * ) malloc( ( n + 1 ) * sizeof( long ) );
    L->row[ 0 ] = 0;
    for ( long i = 0; i < n; ++i ) L->row[ i + 1 ] = L->row[ i ] + nb[ i ];
    L->col = ( long * ) malloc( ( L->row[ n ] + 1 ) * sizeof( long ) );
    L->c = ( double * ) malloc( ( L->row[ n ] + 1 ) * sizeof( double ) );
    L->dia = ( double * ) malloc( n * sizeof( double ) );
    for ( long i = 0; i < n; ++i ) {
        double s = 0;
        for ( int k = 0; k < nb[ i ]; ++k ) {
            L->col[ L->row[ i ] + k ] = nid[ i * cap + k ];
            L->c[ L->row[ i ] + k ] = nc[ i * cap + k ];
            s += nc[ i * cap + k ];
        }
        L->dia[ i ] = s > 0 ? s : 1;
    }
}
static void lap_free( od_lap *L ) { free( L->row ); free( L->col ); free( L->c ); free( L->dia ); }

static void lap_mul( const od_lap *L, const double *x, double *y ) {
#pragma omp parallel for schedule( static )
    for ( long i = 0; i < L->n; ++i ) {
        double s = L->dia[ i ] * x[ i ];
        for ( long e = L->row[ i ]; e < L->row[ i + 1 ]; ++e ) s -= L->c[ e ] * x[ L->col[ e ] ];
        y[ i ] = s;
    }
}
static double vdot( long n, const double *a, const double *b ) {
    double s = 0;
#pragma omp parallel for reduction( + : s ) schedule( static )
    for ( long i = 0; i < n; ++i ) s += a[ i ] * b[ i ];
    return s;
}

/* `L x = b` (b of zero sum), relative tolerance `tol`; `x[ 0 ] = 0` on output. Returns the iterations, -1 on failure */
static int lap_cg( const od_lap *L, const double *b, double *x, double tol, int maxit ) {
    long n = L->n;
    double *r = ( double * ) malloc( n * sizeof( double ) ), *z = ( double * ) malloc( n * sizeof( double ) );
    double *p = ( double * ) malloc( n * sizeof( double ) ), *q = ( double * ) malloc( n * sizeof( double ) );
    for ( long i = 0; i < n; ++i ) { x[ i ] = 0; r[ i ] = b[ i ]; z[ i ] = r[ i ] / L->dia[ i ]; p[ i ] = z[ i ]; }
    double bn = sqrt( vdot( n, b, b ) ), rz = vdot( n, r, z );
    int it = 0, ok = bn == 0;
    for ( ; it < maxit && ! ok; ++it ) {
        lap_mul( L, p, q );
        double pq = vdot( n, p, q );
        if ( ! ( pq > 0 ) ) break;
        double al = rz / pq;
#pragma omp parallel for schedule( static )
        for ( long i = 0; i < n; ++i ) { x[ i ] += al * p[ i ]; r[ i ] -= al * q[ i ]; z[ i ] = r[ i ] / L->dia[ i ]; }
        double rn = sqrt( vdot( n, r, r ) );
        if ( rn <= tol * bn ) { ok = 1; ++it; break; }
        double rz2 = vdot( n, r, z ), be = rz2 / rz;
        rz = rz2;
#pragma omp parallel for schedule( static )
        for ( long i = 0; i < n; ++i ) p[ i ] = z[ i ] + be * p[ i ];
    }
    double g = n ? x[ 0 ] : 0;
    for ( long i = 0; i < n; ++i ) x[ i ] -= g;
    free( r ); free( z ); free( p ); free( q );
    return ok ? it : -1;
}

/* the direct solve of small systems, as the reference's CPU path factors its Laplacian (sdotplan/Linear.h:67-68): the rows and
   columns 1..n-1 (x[ 0 ] = 0) by a dense Cholesky. Returns 0, or -1 when the grounded matrix is not positive definite */
static int lap_dense( const od_lap *L, const double *b, double *x ) {
    long m = L->n - 1;
    x[ 0 ] = 0;
    if ( m <= 0 ) return 0;
    double *A = ( double * ) calloc( ( size_t ) m * m, sizeof( double ) );
    for ( long i = 1; i < L->n; ++i ) {
        A[ ( i - 1 ) * m + i - 1 ] += L->dia[ i ];
        for ( long e = L->row[ i ]; e < L->row[ i + 1 ]; ++e )
            if ( L->col[ e ] > 0 ) A[ ( i - 1 ) * m + L->col[ e ] - 1 ] -= L->c[ e ];
    }
    int ok = 1;
    for ( long j = 0; j < m && ok; ++j ) {
        double d = A[ j * m + j ];
        for ( long k = 0; k < j; ++k ) d -= A[ j * m + k ] * A[ j * m + k ];
        if ( ! ( d > 0 ) ) { ok = 0; break; }
        d = sqrt( d );
        A[ j * m + j ] = d;
#pragma omp parallel for schedule( static )
        for ( long i = j + 1; i < m; ++i ) {
            double s = A[ i * m + j ];
            for ( long k = 0; k < j; ++k ) s -= A[ i * m + k ] * A[ j * m + k ];
            A[ i * m + j ] = s / d;
        }
    }
    if ( ok ) {
        double *y = x + 1;
        for ( long i = 0; i < m; ++i ) {
            double s = b[ i + 1 ];
            for ( long k = 0; k < i; ++k ) s -= A[ i * m + k ] * y[ k ];
            y[ i ] = s / A[ i * m + i ];
        }
        for ( long i = m - 1; i >= 0; --i ) {
            double s = y[ i ];
            for ( long k = i + 1; k < m; ++k ) s -= A[ k * m + i ] * y[ k ];
            y[ i ] = s / A[ i * m + i ];
        }
    }
    free( A );
    return ok ? 0 : -1;
}

/* the Laplacian solve alone, for the tests: CSR from a neighbour table, b of zero sum */
int od_laplacian_solve( long n, int cap, const int *nb, const int *nid, const double *nc, const double *b, double *x, double tol, int maxit ) {
    od_lap L;
    lap_build( &L, n, cap, nb, nid, nc );
    int it = lap_cg( &L, b, x, tol, maxit );
    lap_free( &L );
    return it;
}

/* ------------------------------------------------------------------------------------------------ */
/* THE SOLVE                                                                                       */
/* ------------------------------------------------------------------------------------------------ */
enum { O_TOL_ABS = 0, O_TOL_REL, O_MAXIT, O_MAX_BACKTRACKS, O_T_MIN, O_MULT_OK, O_RESIDUAL, O_POWER, O_SWITCH, O_LIN_TOL, O_LIN_MAXIT,
       O_KEEP_START, O_CONTINUATION, O_CONV_THRESHOLD, O_CONV_S0, O_CONV_RATIO, O_CONV_MIN, O_BRUTE, O_CAP, O_AGG_MARGIN, NB_OPTIONS };
enum { S_STATUS = 0, S_RESIDUAL, S_RESIDUAL0, S_NB_ITER, S_NB_DIAG, S_NB_BACKTRACKS, S_T_MAJORANT, S_T_DIAG, S_T_ASM, S_T_LIN, S_T_LIM, S_EPS,
       S_DOMAIN_MASS, S_NB_OVERFLOWED, S_NB_CELL_LIM, S_NB_LIMIT_ROUNDS, S_LIN_NB_HIERARCHIES, S_LIN_NB_ITER, S_LIN_WORST, S_START, S_T_TOTAL,
       S_NB_CONTINUATION_STEPS, S_MIN_START_MASS, S_IT_SWITCH, S_IT_DOUBLE, S_SCRATCH_BYTES, S_NB_CLUSTERS, S_NB_AGGREGATED, S_NB_DUPLICATES,
       S_RESIDUAL_FULL, S_NB_POLISH, NB_STATS };
enum { RES_LIN = 0, RES_LOG = 1, RES_POWER = 2 };
enum { ST_RUNNING = 0, ST_CONVERGED = 1, ST_MAX_ITER = 2, ST_STAGNATION = 3, ST_LINEAR_FAILURE = 4, ST_CAPACITY = 5, ST_FAILURE = 6,
       ST_CONVERGED_AGG = 7 };

static double now_s( void ) {
#ifdef _OPENMP
    return omp_get_wtime();
#else
    return 0;
#endif
}

typedef struct {
    od_pb pb;
    int brute, cap;
    int *nb, *nid;
    double *nc, *nm;
    double *gauss_conv;             /* the gaussians at the width of the stage */
    /* the aggregation of near-coincident seeds (sdotplan/Aggregation.h): margin, tolerance, union-find (NULL: none) */
    double agg_margin, agg_tol_abs, agg_tol_rel;
    int *agg_parent;
    double *img_conv;                 /* image continuation: the blurred values [nx*ny] and a pass's output */
    int agg_changed;
    int nb_diag;
    double t_diag;
    int status;
} od_sweep;

/* measures and facets for the weights w; the facets land in the sweep's tables */
static int sweep( od_sweep *sw, const double *w, double *a ) {
    sw->pb.w = w;
    od_out o = { a, NULL, NULL, sw->cap, sw->nb, sw->nid, sw->nc, sw->nm, NULL };
    double t0 = now_s();
    int st = diagram( &sw->pb, sw->brute, &o, NULL );
    sw->t_diag += now_s() - t0;
    sw->nb_diag++;
    if ( st != OD_OK && sw->status == OD_OK ) sw->status = st;
    return st;
}

static double g_of( double x, int r, double p ) {
    x = x > 1e-300 ? x : 1e-300;
    if ( r == RES_POWER ) return p == 0 ? log( x ) : ( pow( x, p ) - 1 ) / p;
    return r == RES_LOG ? log( x ) : x - 1;
}
static double gp_of( double x, int r, double p ) {
    x = x > 1e-300 ? x : 1e-300;
    if ( r == RES_POWER ) return pow( x, p - 1 );
    return r == RES_LOG ? 1 / x : 1;
}
static void rhs_of( long n, const double *A, const double *N, int res, double p, double *b ) {
    if ( res == RES_LIN ) { for ( long i = 0; i < n; ++i ) b[ i ] = N[ i ] > 0 ? N[ i ] - A[ i ] : 0; return; }
    double su = 0, sug = 0;
    for ( long i = 0; i < n; ++i ) {
        if ( ! ( N[ i ] > 0 ) ) continue;
        double x = A[ i ] / N[ i ], u = N[ i ] / gp_of( x, res, p );
        su += u; sug += u * g_of( x, res, p );
    }
    double c = sug / su;
    for ( long i = 0; i < n; ++i ) {
        b[ i ] = 0;
        if ( ! ( N[ i ] > 0 ) ) continue;
        double x = A[ i ] / N[ i ];
        b[ i ] = N[ i ] / gp_of( x, res, p ) * ( c - g_of( x, res, p ) );
    }
}
static void project_on_range( long n, double *b ) {
    if ( ! n ) return;
    double s = 0;
    for ( long i = 0; i < n; ++i ) s += b[ i ];
    s /= ( double ) n;
    for ( long i = 0; i < n; ++i ) b[ i ] -= s;
}
static double merit( long n, const double *A, const double *nu, int res, double p ) {
    double s = 0;
    if ( res == RES_LIN ) {
        for ( long i = 0; i < n; ++i ) s += ( nu[ i ] - A[ i ] ) * ( nu[ i ] - A[ i ] );
        return sqrt( s );
    }
    double m = 0;
    for ( long i = 0; i < n; ++i ) m += g_of( A[ i ] / nu[ i ], res, p );
    m /= ( double ) n;
    for ( long i = 0; i < n; ++i ) { double e = g_of( A[ i ] / nu[ i ], res, p ) - m; s += e * e; }
    return sqrt( s );
}
static double vmin( long n, const double *v ) { double m = n ? v[ 0 ] : 0; for ( long i = 0; i < n; ++i ) if ( v[ i ] < m ) m = v[ i ]; return m; }

typedef struct { double t_prev, s_prev; int has_prev; } hopeless_t;
static int hopeless_refused( hopeless_t *h, double t, double n2r, double nr, int ok ) {
    if ( ! ok || ! ( nr > 0 ) ) { h->has_prev = 0; return 0; }
    double s = ( nr - n2r ) / t;
    double sp = h->s_prev, asp = sp > 0 ? sp : -sp;
    int hl = h->has_prev && h->t_prev == 2 * t && s < nr / 4 && sp < nr / 4 && s - sp <= 0.25 * asp && sp - s <= 0.25 * asp && 2 * s - sp < nr / 4;
    h->t_prev = t; h->s_prev = s; h->has_prev = 1;
    return hl;
}

typedef struct {
    double *rows;        /* [cap_steps, 8] */
    long cap_steps, nb_steps, steps_before;
    double s_current;
} od_hist;

static void hist_push( od_hist *H, int it, double t, int nb_evals, long n, const double *a, const double *nu, int nb_diag ) {
    if ( ! H->rows || H->nb_steps >= H->cap_steps ) return;
    double mn = n ? a[ 0 ] : 0, mx = 0, l2 = 0;
    for ( long i = 0; i < n; ++i ) {
        if ( a[ i ] < mn ) mn = a[ i ];
        double e = a[ i ] - nu[ i ];
        if ( fabs( e ) > mx ) mx = fabs( e );
        l2 += e * e;
    }
    double *r = H->rows + 8 * H->nb_steps;
    r[ 0 ] = ( double ) ( H->steps_before + it ); r[ 1 ] = t; r[ 2 ] = sqrt( l2 ); r[ 3 ] = mn; r[ 4 ] = mx;
    r[ 5 ] = nb_diag; r[ 6 ] = nb_evals; r[ 7 ] = H->s_current;
    H->nb_steps++;
}

/* one stage of Newton from (w, a, facets of w); the accepted w and a come back in place */
/* ---- the aggregation of near-coincident seeds (restates sdotplan/Aggregation.h:109-168, 229-250) ---- */
static int agg_find( int *p, int i ) {
    while ( p[ i ] != i ) { p[ i ] = p[ p[ i ] ]; i = p[ i ]; }
    return i;
}
/* the pairs whose facet the doubles of the weights cannot place, c_ij ulp( max |w| ) margin > tau, merged */
static void agg_detect( od_sweep *sw, const od_lap *L, const double *w, const double *nu ) {
    if ( ! ( sw->agg_margin > 0 ) ) return;
    const long n = L->n;
    for ( long i = 0; i < n; ++i )
        for ( long e = L->row[ i ]; e < L->row[ i + 1 ]; ++e ) {
            const long j = L->col[ e ];
            if ( j <= i ) continue;
            const double wm = fmax( fabs( w[ i ] ), fabs( w[ j ] ) );
            const double ulp = nextafter( wm, INFINITY ) - wm;
            const double nm = fmin( nu[ i ], nu[ j ] );
            const double tau = fmax( sw->agg_tol_abs, fmax( sw->agg_tol_rel * nm, 1e-12 * nm ) );
            if ( ! ( L->c[ e ] * ulp * sw->agg_margin > tau ) ) continue;
            if ( ! sw->agg_parent ) {
                sw->agg_parent = ( int * ) malloc( n * sizeof( int ) );
                for ( long k = 0; k < n; ++k ) sw->agg_parent[ k ] = ( int ) k;
            }
            int a = agg_find( sw->agg_parent, ( int ) i ), b = agg_find( sw->agg_parent, ( int ) j );
            if ( a != b ) { sw->agg_parent[ a > b ? a : b ] = a < b ? a : b; sw->agg_changed = 1; }
        }
}
/* the masses the tests read: each member of a cluster gets nu_i a_C / nu_C (members summed in index order) */
static const double *agg_shares( od_sweep *sw, long n, const double *a, const double *nu, double *ae ) {
    if ( ! sw->agg_parent ) return a;
    double *sa = calloc( n, sizeof( double ) ), *sn = calloc( n, sizeof( double ) );
    for ( long i = 0; i < n; ++i ) { int r = agg_find( sw->agg_parent, ( int ) i ); sa[ r ] += a[ i ]; sn[ r ] += nu[ i ]; }
    for ( long i = 0; i < n; ++i ) {
        int r = agg_find( sw->agg_parent, ( int ) i );
        ae[ i ] = r == i && sn[ r ] == nu[ i ] ? a[ i ] : nu[ i ] * ( sn[ r ] > 0 ? sa[ r ] / sn[ r ] : 0.0 );
    }
    free( sa ); free( sn );
    return ae;
}

static int newton_stage( od_sweep *sw, const double *o, const double *nu, double *w, double *a, double *stats, od_hist *H, int first_stage ) {
    long n = sw->pb.n;
    double *b = malloc( n * sizeof( double ) ), *d = malloc( n * sizeof( double ) ), *w2 = malloc( n * sizeof( double ) ), *a2 = malloc( n * sizeof( double ) );
    int cap = sw->cap;
    int *nb2 = malloc( n * sizeof( int ) ), *nid2 = malloc( ( size_t ) n * cap * sizeof( int ) );
    double *nc2 = malloc( ( size_t ) n * cap * sizeof( double ) ), *nm2 = malloc( ( size_t ) n * cap * sizeof( double ) );
    int status = ST_RUNNING, res_cur = ( int ) o[ O_RESIDUAL ];
    double t_last = 1, eps = 0;
    int nb_iter = 0, nb_bt = 0, it_switch = -1;
    double t_asm = 0, t_lin = 0;
    double *ae = malloc( n * sizeof( double ) ), *ae2 = malloc( n * sizeof( double ) );
    hist_push( H, 0, 0, 1, n, a, nu, sw->nb_diag );
    const int maxit = ( int ) o[ O_MAXIT ];
    for ( int it = 0; it < maxit; ++it ) {
        const double *A = agg_shares( sw, n, a, nu, ae );      /* the tests read the clusters' masses */
        double worst = 0, worst_rel = 0;
        for ( long i = 0; i < n; ++i ) {
            double e = fabs( nu[ i ] - A[ i ] );
            if ( e > worst ) worst = e;
            if ( e / nu[ i ] > worst_rel ) worst_rel = e / nu[ i ];
        }
        if ( o[ O_SWITCH ] > 0 && res_cur != RES_LIN && worst_rel <= o[ O_SWITCH ] ) { res_cur = RES_LIN; it_switch = it; }
        rhs_of( n, a, nu, res_cur, o[ O_POWER ], b );
        project_on_range( n, b );
        if ( it == 0 ) {
            eps = 0.5 * fmin( vmin( n, nu ), vmin( n, A ) );
            if ( first_stage ) { stats[ S_EPS ] = eps; stats[ S_RESIDUAL0 ] = worst; }
        }
        double nr = merit( n, A, nu, res_cur, o[ O_POWER ] );
        stats[ S_RESIDUAL ] = worst;
        if ( worst <= o[ O_TOL_ABS ] || ( o[ O_TOL_REL ] > 0 && worst_rel <= o[ O_TOL_REL ] ) ) { status = ST_CONVERGED; break; }
        ++nb_iter;
        double t0 = now_s();
        od_lap L;
        lap_build( &L, n, cap, sw->nb, sw->nid, sw->nc );
        agg_detect( sw, &L, w, nu );
        t_asm += now_s() - t0;
        t0 = now_s();
        int lit = lap_cg( &L, b, d, o[ O_LIN_TOL ], ( int ) o[ O_LIN_MAXIT ] );
        if ( lit < 0 && n <= 4096 && lap_dense( &L, b, d ) == 0 ) lit = 0;    /* CG lost to the conditioning: factor */
        t_lin += now_s() - t0;
        lap_free( &L );
        if ( lit < 0 ) { status = ST_LINEAR_FAILURE; break; }
        stats[ S_LIN_NB_ITER ] += lit;
        double t = fmin( 1.0, o[ O_MULT_OK ] * t_last );
        int taken = 0, nb_evals = 0;
        hopeless_t hope = { 0, 0, 0 };
        for ( int trial = 0; trial < ( int ) o[ O_MAX_BACKTRACKS ]; ++trial ) {
            for ( long i = 0; i < n; ++i ) w2[ i ] = w[ i ] + t * d[ i ];
            w2[ 0 ] = 0;
            int *sb = sw->nb, *si = sw->nid;
            double *sc = sw->nc, *sm = sw->nm;
            sw->nb = nb2; sw->nid = nid2; sw->nc = nc2; sw->nm = nm2;
            sweep( sw, w2, a2 );
            sw->nb = sb; sw->nid = si; sw->nc = sc; sw->nm = sm;
            ++nb_evals;
            const double *A2 = agg_shares( sw, n, a2, nu, ae2 );
            double m2 = vmin( n, A2 ), n2r = merit( n, A2, nu, res_cur, o[ O_POWER ] );
            if ( m2 >= eps && isfinite( n2r ) && n2r <= ( 1 - t / 2 ) * nr && n2r < nr ) { taken = 1; break; }
            int hl = hopeless_refused( &hope, t, n2r, nr, m2 >= eps && isfinite( n2r ) );
            t /= 2;
            ++nb_bt;
            if ( t < o[ O_T_MIN ] || hl ) break;
        }
        if ( ! taken && res_cur != RES_LIN ) { res_cur = RES_LIN; it_switch = it; --nb_iter; --it; continue; }
        if ( ! taken ) { status = ST_STAGNATION; break; }
        t_last = t;
        memcpy( w, w2, n * sizeof( double ) );
        memcpy( a, a2, n * sizeof( double ) );
        int *ti = sw->nb; sw->nb = nb2; nb2 = ti;
        ti = sw->nid; sw->nid = nid2; nid2 = ti;
        double *td = sw->nc; sw->nc = nc2; nc2 = td;
        td = sw->nm; sw->nm = nm2; nm2 = td;
        hist_push( H, it + 1, t, nb_evals, n, a, nu, sw->nb_diag );
    }
    if ( status == ST_RUNNING ) {
        const double *A = agg_shares( sw, n, a, nu, ae );
        double worst = 0;
        for ( long i = 0; i < n; ++i ) worst = fmax( worst, fabs( nu[ i ] - A[ i ] ) );
        stats[ S_RESIDUAL ] = worst;
        status = ST_MAX_ITER;
    }
    free( ae ); free( ae2 );
    stats[ S_NB_ITER ] += nb_iter;
    stats[ S_NB_BACKTRACKS ] += nb_bt;
    stats[ S_T_ASM ] += t_asm;
    stats[ S_T_LIN ] += t_lin;
    if ( first_stage ) stats[ S_IT_SWITCH ] = it_switch;
    free( b ); free( d ); free( w2 ); free( a2 ); free( nb2 ); free( nid2 ); free( nc2 ); free( nm2 );
    return status;
}

/* the gaussians at width s: sigma -> sqrt( sigma^2 + s^2 ) */
static void gauss_at( od_sweep *sw, const double *dval, int dim, double s ) {
    int ng = ( int ) sw->pb.dpar[ 0 ], st = dim + 2;
    for ( int g = 0; g < ng; ++g ) {
        for ( int q = 0; q < st; ++q ) sw->gauss_conv[ g * st + q ] = dval[ g * st + q ];
        sw->gauss_conv[ g * st + dim ] = sqrt( dval[ g * st + dim ] * dval[ g * st + dim ] + s * s );
    }
    sw->pb.dval = sw->gauss_conv;
}

/* the image at width s (sdotplan/convolved/Image.h:51-74): along each axis a gaussian of s / step pixels, truncated at
 * ceil( 4 s / step ) pixels (at most the axis), each value renormalised by the taps inside the axis; axis x first */
static void image_at( od_sweep *sw, const double *dval, double s ) {
    const double *P = sw->pb.dpar;
    const int nx = ( int ) P[ 4 ], ny = ( int ) P[ 5 ];
    const long tot = ( long ) nx * ny;
    double *buf = sw->img_conv, *tmp = sw->img_conv + tot;
    memcpy( buf, dval, tot * sizeof( double ) );
    for ( int a = 0; a < 2 && s > 0; ++a ) {
        const double sp = s / P[ 2 + a ];
        if ( ! ( sp > 1e-3 ) ) continue;
        const int len = a ? ny : nx;
        const long stride = a ? 1 : ny;
        int r = ( int ) ceil( 4 * sp );
        if ( r > len ) r = len;
        double *ker = malloc( ( 2 * ( size_t ) r + 1 ) * sizeof( double ) );
        for ( int k = -r; k <= r; ++k ) ker[ k + r ] = exp( -0.5 * ( double ) k * ( double ) k / ( sp * sp ) );
#pragma omp parallel for schedule( static )
        for ( long flat = 0; flat < tot; ++flat ) {
            const int p = a ? ( int ) ( flat % ny ) : ( int ) ( flat / ny );
            const int lo = -r > -p ? -r : -p, hi = r < len - 1 - p ? r : len - 1 - p;
            double sum = 0, ws = 0;
            for ( int k = lo; k <= hi; ++k ) { sum += ker[ k + r ] * buf[ flat + k * stride ]; ws += ker[ k + r ]; }
            tmp[ flat ] = sum / ws;
        }
        free( ker );
        double *t = buf; buf = tmp; tmp = t;
    }
    if ( buf != sw->img_conv ) memcpy( sw->img_conv, buf, tot * sizeof( double ) );
    sw->pb.dval = sw->img_conv;
}

/* THE SOLVE (restates sdotplan/Solve.h::solve with the aggregation of near-coincident seeds, exact duplicates left to the
 * caller, and the TRIALS step).
 * Inputs in user order; `w0` may be NULL; `opts` [NB_OPTIONS]; outputs: weights [n], masses [n], bary [n, d],
 * cost [1], stats [NB_STATS], hist [cap_steps, 8] (may be NULL) and the number of rows written. */
int od_solve( int dim, long n, const double *pos, const double *nu_in, const double *w0, const double *box, int dkind, const double *dpar,
              const double *dval, const double *opts, double *weights, double *masses, double *bary, double *cost, double *stats,
              double *hist, long cap_steps, long *nb_steps, int *clusters ) {
    double t_begin = now_s();
    od_sweep sw;
    memset( &sw, 0, sizeof( sw ) );
    init_pb( &sw.pb, dim, n, pos, NULL, box, dkind, dpar, dval );
    sw.brute = ( int ) opts[ O_BRUTE ];
    sw.cap = ( int ) opts[ O_CAP ];
    sw.agg_margin = opts[ O_AGG_MARGIN ];
    sw.agg_tol_abs = opts[ O_TOL_ABS ];
    sw.agg_tol_rel = opts[ O_TOL_REL ];
    sw.nb = malloc( n * sizeof( int ) );
    sw.nid = malloc( ( size_t ) n * sw.cap * sizeof( int ) );
    sw.nc = malloc( ( size_t ) n * sw.cap * sizeof( double ) );
    sw.nm = malloc( ( size_t ) n * sw.cap * sizeof( double ) );
    int ng = dkind == DENS_GAUSS ? ( int ) dpar[ 0 ] : 0;
    sw.gauss_conv = malloc( ( ng > 0 ? ng : 1 ) * ( dim + 2 ) * sizeof( double ) );
    if ( dkind == DENS_IMAGE ) sw.img_conv = malloc( 2 * ( size_t ) dpar[ 4 ] * ( size_t ) dpar[ 5 ] * sizeof( double ) );
    for ( int k = 0; k < NB_STATS; ++k ) stats[ k ] = 0;
    od_hist H = { hist, hist ? cap_steps : 0, 0, 0, 0 };

    double *nu = malloc( n * sizeof( double ) ), *w = malloc( n * sizeof( double ) ), *a = malloc( n * sizeof( double ) );
    double *wt0 = malloc( n * sizeof( double ) ), *at0 = malloc( n * sizeof( double ) );
    int given = 0;
    for ( long i = 0; i < n; ++i ) { nu[ i ] = nu_in[ i ]; w[ i ] = w0 ? w0[ i ] : 0; given |= w[ i ] != 0; }
    int start = given ? 0 : 1;
    double gauge = n ? w[ 0 ] : 0;
    for ( long i = 0; i < n; ++i ) w[ i ] -= gauge;

    /* the stages of the width continuation */
    int possible = dkind == DENS_GAUSS || ( dkind == DENS_IMAGE && dim == 2 );
    double s0 = opts[ O_CONV_S0 ];
    if ( s0 <= 0 ) {
        double diam2 = 0;
        for ( int q = 0; q < dim; ++q ) diam2 += ( box[ dim + q ] - box[ q ] ) * ( box[ dim + q ] - box[ q ] );
        s0 = 0.5 * sqrt( diam2 );
    }
    double smin = opts[ O_CONV_MIN ];
    if ( smin <= 0 && dkind == DENS_GAUSS ) {
        double sg = 1e300;
        for ( int g = 0; g < ng; ++g ) sg = fmin( sg, dval[ g * ( dim + 2 ) + dim ] );
        smin = sg / 4;
    }
    if ( smin <= 0 && dkind == DENS_IMAGE ) smin = fmin( dpar[ 2 ], dpar[ 3 ] ) / 4;      /* a quarter of a pixel */
    double scales[ 256 ];
    int nsc = 0;
    int cont = ( int ) opts[ O_CONTINUATION ];
    double ratio = opts[ O_CONV_RATIO ] > 1 ? opts[ O_CONV_RATIO ] : sqrt( 2.0 );
#define MAKE_SCALES() do { nsc = 0; if ( s0 > 0 ) for ( double s = s0; s >= smin * ( 1 - 1e-12 ) && s > 0 && nsc < 255; s /= ratio ) scales[ nsc++ ] = s; scales[ nsc++ ] = 0; } while ( 0 )
    if ( cont == 2 && possible ) MAKE_SCALES();
    else { scales[ 0 ] = 0; nsc = 1; }

#define DENS_AT( s ) do { if ( dkind == DENS_GAUSS ) gauss_at( &sw, dval, dim, ( s ) ); else if ( possible ) image_at( &sw, dval, ( s ) ); } while ( 0 )
    DENS_AT( scales[ 0 ] );
    H.s_current = scales[ 0 ];
    int st = sweep( &sw, w, a );
    double nu_min = vmin( n, nu );
    if ( given && ! opts[ O_KEEP_START ] && vmin( n, a ) < 1e-3 * nu_min ) {
        for ( long i = 0; i < n; ++i ) wt0[ i ] = 0;
        sweep( &sw, wt0, at0 );
        if ( vmin( n, at0 ) > vmin( n, a ) ) { memcpy( w, wt0, n * sizeof( double ) ); memcpy( a, at0, n * sizeof( double ) ); start = 1; }
        sweep( &sw, w, a );     /* the facets of the kept start */
        sw.nb_diag--;
    }
    if ( vmin( n, a ) <= 0 && ! ( given && opts[ O_KEEP_START ] ) ) {
        /* the similarity that packs the cloud into the domain box minus a margin of 0.1 (sdotplan/Solve.h:66-97) */
        double plo[ 3 ], phi[ 3 ], al = 1, bb[ 3 ];
        for ( int q = 0; q < dim; ++q ) { plo[ q ] = 1e300; phi[ q ] = -1e300; }
        for ( long i = 0; i < n; ++i ) for ( int q = 0; q < dim; ++q ) { plo[ q ] = fmin( plo[ q ], pos[ i * dim + q ] ); phi[ q ] = fmax( phi[ q ], pos[ i * dim + q ] ); }
        for ( int q = 0; q < dim; ++q ) {
            double sd = ( box[ dim + q ] - box[ q ] ) * 0.8, sp = fmax( phi[ q ] - plo[ q ], 1e-300 );
            al = fmin( al, sd / sp );
        }
        for ( int q = 0; q < dim; ++q ) bb[ q ] = ( box[ q ] + box[ dim + q ] ) / 2 - al * ( plo[ q ] + phi[ q ] ) / 2;
        for ( long i = 0; i < n; ++i ) {
            double pp = 0, qq = 0;
            for ( int q = 0; q < dim; ++q ) { double x = pos[ i * dim + q ], y = al * x + bb[ q ]; pp += x * x; qq += y * y; }
            wt0[ i ] = pp - qq / al;
        }
        double g0 = wt0[ 0 ];
        for ( long i = 0; i < n; ++i ) wt0[ i ] -= g0;
        sweep( &sw, wt0, at0 );
        if ( vmin( n, at0 ) > vmin( n, a ) ) { memcpy( w, wt0, n * sizeof( double ) ); memcpy( a, at0, n * sizeof( double ) ); start = 2; }
        sweep( &sw, w, a );
        sw.nb_diag--;
    }
    double min_start_mass = vmin( n, a );
    if ( cont == 1 && possible && nsc == 1 && min_start_mass < opts[ O_CONV_THRESHOLD ] * nu_min ) {
        MAKE_SCALES();
        DENS_AT( scales[ 0 ] );
        H.s_current = scales[ 0 ];
        sweep( &sw, w, a );
    }
#undef MAKE_SCALES
    int status = st == OD_OK ? ST_RUNNING : ST_CAPACITY;
    double domain_mass = 0;
    double *nu_s = malloc( n * sizeof( double ) );
    for ( int step = 0; step < nsc && status != ST_CAPACITY; ++step ) {
        H.s_current = scales[ step ];
        if ( step > 0 ) {
            DENS_AT( scales[ step ] );
            sweep( &sw, w, a );
        }
        double num = 0;
        domain_mass = 0;
        for ( long i = 0; i < n; ++i ) { domain_mass += a[ i ]; num += nu[ i ]; }
        for ( long i = 0; i < n; ++i ) nu_s[ i ] = ( domain_mass > 0 && num > 0 && domain_mass != num ) ? nu[ i ] * ( domain_mass / num ) : nu[ i ];
        status = newton_stage( &sw, opts, nu_s, w, a, stats, &H, step == 0 );
        H.steps_before = H.nb_steps > 0 ? ( long ) hist[ 8 * ( H.nb_steps - 1 ) ] + 1 : 0;
        if ( status == ST_LINEAR_FAILURE ) break;
        if ( sw.status != OD_OK ) { status = ST_CAPACITY; break; }
    }
    int nb_diag_descent = sw.nb_diag;
    for ( long i = 0; i < n; ++i ) { weights[ i ] = w[ i ]; masses[ i ] = a[ i ]; }
    /* the moments on the true density at the fitted weights */
#undef DENS_AT
    sw.pb.dval = dval;
    {
        double *cst = malloc( n * sizeof( double ) );
        sw.pb.w = w;
        od_out o = { NULL, bary, cst, 0, NULL, NULL, NULL, NULL, NULL };
        diagram( &sw.pb, sw.brute, &o, NULL );
        double c = 0;
        for ( long i = 0; i < n; ++i ) c += cst[ i ];
        *cost = c;
        free( cst );
    }
    stats[ S_STATUS ] = status;
    stats[ S_NB_DIAG ] = nb_diag_descent;
    stats[ S_T_DIAG ] = sw.t_diag;
    stats[ S_DOMAIN_MASS ] = domain_mass;
    stats[ S_START ] = start;
    stats[ S_T_TOTAL ] = now_s() - t_begin;
    stats[ S_NB_CONTINUATION_STEPS ] = nsc;
    stats[ S_MIN_START_MASS ] = min_start_mass;
    stats[ S_RESIDUAL_FULL ] = stats[ S_RESIDUAL ];
    if ( clusters ) for ( long i = 0; i < n; ++i ) clusters[ i ] = sw.agg_parent ? agg_find( sw.agg_parent, ( int ) i ) : ( int ) i;
    if ( sw.agg_parent ) {
        /* the full problem's residual; "converged (aggregated)" when only the clusters' masses pass (sdotplan/Solve.h:300-306) */
        double wf = 0, wfr = 0;
        long ncl = 0, nagg = 0;
        int *size = calloc( n, sizeof( int ) );
        for ( long i = 0; i < n; ++i ) {
            const double e = fabs( a[ i ] - nu_s[ i ] );
            wf = fmax( wf, e );
            wfr = fmax( wfr, e / nu_s[ i ] );
            ++size[ agg_find( sw.agg_parent, ( int ) i ) ];
        }
        for ( long i = 0; i < n; ++i ) if ( size[ i ] > 1 ) { ++ncl; nagg += size[ i ]; }
        free( size );
        stats[ S_RESIDUAL_FULL ] = wf;
        stats[ S_NB_CLUSTERS ] = ( double ) ncl;
        stats[ S_NB_AGGREGATED ] = ( double ) nagg;
        if ( status == ST_CONVERGED && ! ( wf <= opts[ O_TOL_ABS ] || ( opts[ O_TOL_REL ] > 0 && wfr <= opts[ O_TOL_REL ] ) ) )
            stats[ S_STATUS ] = ST_CONVERGED_AGG;
        free( sw.agg_parent );
    }
    if ( nb_steps ) *nb_steps = H.nb_steps;
    free( nu ); free( w ); free( a ); free( wt0 ); free( at0 ); free( nu_s );
    free( sw.nb ); free( sw.nid ); free( sw.nc ); free( sw.nm ); free( sw.gauss_conv ); free( sw.img_conv );
    return st == OD_OK ? OD_OK : st;
}

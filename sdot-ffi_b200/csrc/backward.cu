// The backward of the W2 loss of a batch of transports (the envelope theorem at the fitted weights):
//   d W2 / d p_i  = 2 m_i ( p_i - b_i )                    (SdotPlanNd.py:1107-1122, cost_and_position_grad)
//   d W2 / d nu_i = w_i - mean( w )                         (the dual's envelope, projected on sum( d nu ) = 0,
//                                                            SdotPlanNd.py:1037-1040)
// scaled by the cotangent of each problem's cost.  One block per problem (the mean of its weights is a
// deterministic block reduction), positions in FP32 or FP64.
#include "engine.h"
#include <cstring>

namespace sdot {

template<class TP>
__global__ void __launch_bounds__( 256 ) k_w2_backward( int n, int dim, const TP *__restrict__ pos, const double *__restrict__ mass,
                                                        const double *__restrict__ bary, const double *__restrict__ w,
                                                        const double *__restrict__ gcost, TP *gpos, TP *gnu ) {
    const int b = blockIdx.x;
    const size_t o = size_t( b ) * n;
    __shared__ double sh[ 8 ];
    double s = 0;
    for ( int i = threadIdx.x; i < n; i += blockDim.x ) s += w[ o + i ];
    s = warp_sum( s );
    if ( ( threadIdx.x & 31 ) == 0 ) sh[ threadIdx.x >> 5 ] = s;
    __syncthreads();
    double mean = 0;
    for ( int k = 0; k < int( blockDim.x >> 5 ); ++k ) mean += sh[ k ];
    mean /= n;
    const double g = gcost[ b ];
    for ( int i = threadIdx.x; i < n; i += blockDim.x ) {
        if ( gnu ) gnu[ o + i ] = TP( g * ( w[ o + i ] - mean ) );
        if ( gpos )
            for ( int a = 0; a < dim; ++a ) {
                size_t k = ( o + i ) * dim + a;
                gpos[ k ] = TP( g * 2 * mass[ o + i ] * ( double( pos[ k ] ) - bary[ k ] ) );
            }
    }
}

void launch_w2_backward( const Launch &L, int batch, int n, int dim, const void *pos, int fp32, const double *mass, const double *bary,
                         const double *w, const double *gcost, void *gpos, void *gnu ) {
    if ( fp32 )
        k_w2_backward<float><<<batch, 256, 0, L.stream>>>( n, dim, ( const float * ) pos, mass, bary, w, gcost, ( float * ) gpos, ( float * ) gnu );
    else
        k_w2_backward<double><<<batch, 256, 0, L.stream>>>( n, dim, ( const double * ) pos, mass, bary, w, gcost, ( double * ) gpos,
                                                            ( double * ) gnu );
    ++*L.launches;
}

} // namespace sdot

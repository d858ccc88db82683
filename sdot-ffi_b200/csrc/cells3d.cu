// 3D Laguerre cells (placeholder until the warp-per-cell polyhedron clipper lands): refuses with a status.
#include "internal.h"

namespace sdot {

__global__ void k_cells3d_refuse( ErrRec *err ) {
    if ( atomicCAS( &err->code, 0, 5 ) == 0 ) { err->kind = 2; err->prob = 0; err->seed = -1; err->needed = 0; }
}

void launch_cells3d( const Launch &L, const ProbDev *probs, const Chunk *chunks, int nchunks, unsigned flags, ErrRec *err ) {
    (void) probs; (void) chunks; (void) nchunks; (void) flags;
    k_cells3d_refuse<<<1, 1, 0, L.stream>>>( err );
    ++*L.launches;
}

} // namespace sdot

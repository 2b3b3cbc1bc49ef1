// The single-rank MPI stand-in for the reference's GPU-path sources, alone in
// this directory so that their <cuda.h> resolves to the real CUDA header.
#include "../ref_stub/mpi.h"

// Throughput build of the stage kernels: FMA contraction on, WENO weights with a
// single division per face.  Agrees with the reference-order build to round-off.
#define NUC3D_NS fast
#define NUC3D_FAST 1
#include "kernels.cuh"

// Reference-order build of the stage kernels: compiled with -fmad=false so no
// multiply-add is contracted and every operation rounds exactly where the
// reference's does; results are bit-comparable with the CPU oracle.
#define NUC3D_NS exact
#define NUC3D_FAST 0
#include "kernels.cuh"

// Exact arithmetic build of kernels.cuh: compiled with -fmad=false so every
// multiply and add rounds separately, in the reference's order.
#define KF_FAST 0
#define KF_NS kf_exact
#include "kernels.cuh"

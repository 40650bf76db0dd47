// Fast build of kernels.cuh: fused multiply-add, reciprocals of the constant
// beta and of c^2 hoisted, reciprocal square root for the tangent frame.
#define KF_FAST 1
#define KF_NS kf_fast
#include "kernels.cuh"

/*
 * Test infrastructure only (oracle build).
 *
 * Shadow of the reference's inc/phy.h (inc/phy.h:1-11), placed first on the
 * include path when the reference sources are compiled into
 * oracle/_ref/libkfun3d_ref.so.  It keeps the reference's constants B, P and W
 * and turns the free-stream velocity (U, V), which the reference hard-codes for
 * an angle of attack of 3 degrees, into two run-time variables so one build
 * serves every angle of attack.  The include guard is the reference's own, so
 * the original header is never seen after this one.
 */
#ifndef __FUN3D_INC_PHY_H
#define __FUN3D_INC_PHY_H

#include <math.h>

extern double kf_ref_phy_u;
extern double kf_ref_phy_v;

#define B 15
#define P 1
#define U kf_ref_phy_u
#define V kf_ref_phy_v
#define W 0

#endif /* __FUN3D_INC_PHY_H */

// gx_transport_parity.cu -- the FP64 parity variant of the transport engine.
//
// gx_transport.cu compiled a second time with GX_PARITY defined, built
// without floating-point contraction (-fmad=false), into namespace
// gx::parity and for FP64 only: every table lookup in the reference's spline
// form, the reference's ionisation along-step functions, the general helix
// step with the oracle's sub-step length, and the elementary functions of
// gx_math.h.  The oracle's parity build (oracle/liboracle_gxm.so) runs the same
// operations in the same order on the CPU, so the two agree track by track:
// the same steps for every primary, deposits equal up to the order in which
// the device's atomic additions sum them.  Selected with
// gx_transport_config.fp64_parity = 1.
#define GX_PARITY 1
#include "gx_transport.cu"

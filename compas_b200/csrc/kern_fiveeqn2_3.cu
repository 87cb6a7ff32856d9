// Stage kernels of the FiveEqN<2, 3> model (N-phase five-equation, 2D, NPHASE = 3), plain FP64 form.
#include "kern_impl.cuh"

namespace compas {
using FiveEqN2_3 = FiveEqN<2, 3>;
}

COMPAS_DEFINE_LAUNCHERS(fiveeqn2_3, FiveEqN2_3, 0)

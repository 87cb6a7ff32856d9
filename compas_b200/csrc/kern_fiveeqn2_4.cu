// Stage kernels of the FiveEqN<2, 4> model (N-phase five-equation, 2D, NPHASE = 4), plain FP64 form.
#include "kern_impl.cuh"

namespace compas {
using FiveEqN2_4 = FiveEqN<2, 4>;
}

COMPAS_DEFINE_LAUNCHERS(fiveeqn2_4, FiveEqN2_4, 0)

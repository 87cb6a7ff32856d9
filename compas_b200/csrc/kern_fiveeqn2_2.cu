// Stage kernels of the FiveEqN<2, 2> model (N-phase five-equation, 2D, NPHASE = 2), plain FP64 form.
#include "kern_impl.cuh"

namespace compas {
using FiveEqN2_2 = FiveEqN<2, 2>;
}

COMPAS_DEFINE_LAUNCHERS(fiveeqn2_2, FiveEqN2_2, 0)

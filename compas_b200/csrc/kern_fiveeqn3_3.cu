// Stage kernels of the FiveEqN<3, 3> model (N-phase five-equation, 3D, NPHASE = 3), plain FP64 form.
#include "kern_impl.cuh"

namespace compas {
using FiveEqN3_3 = FiveEqN<3, 3>;
}

COMPAS_DEFINE_LAUNCHERS(fiveeqn3_3, FiveEqN3_3, 0)

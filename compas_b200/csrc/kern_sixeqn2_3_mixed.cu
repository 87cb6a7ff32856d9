// Stage kernels of the SixEqN<2, 3> model (N-phase six-equation in the internal-energy form, 2D,
// NPHASE = 3), mixed-precision form.
#include "kern_impl.cuh"

namespace compas {
using SixEqN2_3 = SixEqN<2, 3>;
}

COMPAS_DEFINE_LAUNCHERS(sixeqn2_3, SixEqN2_3, 1)

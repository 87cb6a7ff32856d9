// Stage kernels of the SixEqN<2, 2> model (N-phase six-equation in the internal-energy form, 2D,
// NPHASE = 2), mixed-precision form.
#include "kern_impl.cuh"

namespace compas {
using SixEqN2_2 = SixEqN<2, 2>;
}

COMPAS_DEFINE_LAUNCHERS(sixeqn2_2, SixEqN2_2, 1)

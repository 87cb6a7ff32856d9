// Stage kernels of the SixEqN<3, 3> model (N-phase six-equation in the internal-energy form, 3D,
// NPHASE = 3), plain FP64 form.
#include "kern_impl.cuh"

namespace compas {
using SixEqN3_3 = SixEqN<3, 3>;
}

COMPAS_DEFINE_LAUNCHERS(sixeqn3_3, SixEqN3_3, 0)

// Stage kernels of the FiveEq<3> model (instantiations and launchers), mixed-precision form.
#include "kern_impl.cuh"

COMPAS_DEFINE_LAUNCHERS(fiveeq3, FiveEq<3>, 1)

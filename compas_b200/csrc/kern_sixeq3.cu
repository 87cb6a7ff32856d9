// Stage kernels of the SixEq<3> model (instantiations and launchers), plain FP64 form.
#include "kern_impl.cuh"

COMPAS_DEFINE_LAUNCHERS(sixeq3, SixEq<3>, 0)

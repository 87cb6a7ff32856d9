// Stage kernels of the SixEq<2> model (instantiations and launchers), plain FP64 form.
#include "kern_impl.cuh"

COMPAS_DEFINE_LAUNCHERS(sixeq2, SixEq<2>, 0)

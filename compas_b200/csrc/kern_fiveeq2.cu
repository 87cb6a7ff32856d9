// Stage kernels of the FiveEq<2> model (instantiations and launchers), plain FP64 form.
#include "kern_impl.cuh"

COMPAS_DEFINE_LAUNCHERS(fiveeq2, FiveEq<2>, 0)

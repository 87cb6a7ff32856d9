// Test infrastructure (oracle): forwards to the shared AMReX-compatible shim.
#include "amrex_shim_core.H"

// Bound-preserving kernels (FiniteVolume.ID_Bound = 1) of FIVEEQS and FIVEEQS_NPHASE: instantiations and
// launchers (one translation unit, built in parallel with the stage-kernel units).
#include <algorithm>

#include "compas_b200.h"
#include "launch.h"
#include "stage_kernel.cuh"
#include "bound.cuh"

namespace compas {

// The model of a launch: FIVEEQS in 2D / 3D, FIVEEQS_NPHASE with the NPHASE values this build has.
template <class F>
static cudaError_t bp_dispatch(int physics, int dim, int nphase, F&& f) {
    if (physics == COMPAS_B200_FIVEEQS) {
        if (dim == 2) return f(FiveEq<2>());
        return f(FiveEq<3>());
    }
    if (physics == COMPAS_B200_FIVEEQS_NPHASE) {
        if (dim == 3) return f(FiveEqN<3, 3>());
        if (nphase == 2) return f(FiveEqN<2, 2>());
        if (nphase == 3) return f(FiveEqN<2, 3>());
        return f(FiveEqN<2, 4>());
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_bp_faces_model(const BpFaceArgs& a, cudaStream_t st) {
    const long long total = a.off[a.D];
    if (total == 0) return cudaSuccess;
    const unsigned blocks = (unsigned)std::min<long long>((total + 127) / 128, 148LL * 16);
    return bp_dispatch(a.physics, a.D, a.nphase, [&](auto m) {
        using M = decltype(m);
        bp_face_kernel<M><<<blocks, 128, 0, st>>>(a);
        return cudaGetLastError();
    });
}

cudaError_t launch_bp_update_model(const BpUpdateArgs& a, cudaStream_t st) {
    const long long cells = (long long)a.g.n[0] * a.g.n[1] * (a.D == 3 ? a.g.n[2] : 1);
    const unsigned blocks = (unsigned)std::max<long long>(1, std::min<long long>((cells + 127) / 128, 148LL * 16));
    return bp_dispatch(a.physics, a.D, a.nphase, [&](auto m) {
        using M = decltype(m);
        bp_update_kernel<M><<<blocks, 128, 0, st>>>(a);
        return cudaGetLastError();
    });
}

cudaError_t launch_bp_min_model(const double* U, const Grid& g, const Eos& e, int dim, int physics, int nphase,
                                unsigned long long* key, unsigned blocks, cudaStream_t st) {
    return bp_dispatch(physics, dim, nphase, [&](auto m) {
        using M = decltype(m);
        bp_min_kernel<M><<<blocks, 128, 0, st>>>(U, g, e, key, nullptr);
        return cudaGetLastError();
    });
}

}  // namespace compas

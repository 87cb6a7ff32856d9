// Launchers of the stage kernels. The kernels are compiled in one translation unit per model and
// dimension (kern_*.cu, built in parallel); the C-ABI translation unit calls them through these
// declarations. Each returns the CUDA error of its launch.
#pragma once

#include <cuda_runtime.h>

namespace compas {

struct StageArgs;
struct ListArgs;
struct TmaMaps;
struct BpFaceArgs;
struct BpUpdateArgs;
struct Grid;
struct Eos;

// Bound-preserving kernels (FiniteVolume.ID_Bound = 1; kern_bound.cu): the face pass, the stage update
// and the smallest energy bound, for the model named by physics / nphase (FIVEEQS, FIVEEQS_NPHASE).
cudaError_t launch_bp_faces_model(const BpFaceArgs& a, cudaStream_t st);
cudaError_t launch_bp_update_model(const BpUpdateArgs& a, cudaStream_t st);
cudaError_t launch_bp_min_model(const double* U, const Grid& g, const Eos& e, int dim, int physics, int nphase,
                                unsigned long long* key, unsigned blocks, cudaStream_t st);

// Variant of the stage kernel: FiniteVolume.Scheme (5 WENO5, 6 WENO5B), precision (0 FP64, 1 mixed),
// FiniteVolume.THINC (single-box kernel only), and the Phase-Field regularisation right-hand side
// instead of the hyperbolic one (FIVEEQS and SIXEQS, single-box kernel only). The N-phase model
// (fiveeqn<dim>_<nphase>) runs WENO5 only.
struct KernelChoice {
    int limiter;
    int precision;
    int thinc;
    int phase_field;
    int shape;  // launch shape (kern_impl.cuh ShapeParams; 0..kShapes-1), chosen by the autotuner
};

// Launch shapes compiled per kernel variant, and tile traversal orders (tile_coords).
constexpr int kShapes = 3;
constexpr int kOrders = 2;

// Tile side of the stage kernels (cells per direction): 16^2 tiles in 2D, 8^3 in 3D.
constexpr int kTile2 = 16;
constexpr int kTile3 = 8;

// Each model's kernels are compiled in two translation units, one per precision form (kern_<name>.cu
// plain FP64, kern_<name>_mixed.cu mixed precision), built in parallel; launch_*_<name> picks the unit
// by KernelChoice::precision.
#define COMPAS_DECLARE_LAUNCHERS(name)                                                               \
    cudaError_t launch_stage_##name##_p0(const KernelChoice& k, const StageArgs& a, cudaStream_t st,   \
                                         const TmaMaps* tm);                                         \
    cudaError_t launch_stage_##name##_p1(const KernelChoice& k, const StageArgs& a, cudaStream_t st,   \
                                         const TmaMaps* tm);                                         \
    cudaError_t launch_list_##name##_p0(const KernelChoice& k, const ListArgs& L, cudaStream_t st);   \
    cudaError_t launch_list_##name##_p1(const KernelChoice& k, const ListArgs& L, cudaStream_t st);   \
    inline cudaError_t launch_stage_##name(const KernelChoice& k, const StageArgs& a, cudaStream_t st, \
                                           const TmaMaps* tm) {                                      \
        return (k.precision == 1) ? launch_stage_##name##_p1(k, a, st, tm)                           \
                                  : launch_stage_##name##_p0(k, a, st, tm);                          \
    }                                                                                                \
    inline cudaError_t launch_list_##name(const KernelChoice& k, const ListArgs& L, cudaStream_t st) { \
        return (k.precision == 1) ? launch_list_##name##_p1(k, L, st) : launch_list_##name##_p0(k, L, st); \
    }
COMPAS_DECLARE_LAUNCHERS(fiveeq2)
COMPAS_DECLARE_LAUNCHERS(fiveeq3)
COMPAS_DECLARE_LAUNCHERS(sixeq2)
COMPAS_DECLARE_LAUNCHERS(sixeq3)
COMPAS_DECLARE_LAUNCHERS(fiveeqn2_2)
COMPAS_DECLARE_LAUNCHERS(fiveeqn2_3)
COMPAS_DECLARE_LAUNCHERS(fiveeqn2_4)
COMPAS_DECLARE_LAUNCHERS(fiveeqn3_3)
// SIXEQS_IE_NPHASE (sixeqn<dim>_<nphase>)
COMPAS_DECLARE_LAUNCHERS(sixeqn2_2)
COMPAS_DECLARE_LAUNCHERS(sixeqn2_3)
COMPAS_DECLARE_LAUNCHERS(sixeqn3_3)
#undef COMPAS_DECLARE_LAUNCHERS


}  // namespace compas

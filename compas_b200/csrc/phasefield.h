// Phase-Field regularisation of the five-equation model on the device: the mechanism's pseudo-time
// evolution of the volume fraction (CAC-Adv or ACDI), the regularisation potential Q (an elliptic
// solve for the implicit approach, a local formula for the explicit one), and its face gradients,
// which the Phase-Field stage kernel (stage_kernel.cuh, kVarPhaseField) turns into fluxes.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "compas_b200.h"

namespace compas {

struct PfLevel;

// Counters of one Phase-Field step (the quantities PhaseField_Evolve prints or derives).
struct PfInfo {
    double max_v;       // max |u| over the valid cells (MaxVelocity)
    double mobility;    // 0.5 eta max|u|
    double eta;
    int mech_steps;     // pseudo-time steps of the mechanism
    int solve_iters;    // conjugate-gradient iterations of the elliptic solve (0 for explicit)
    double solve_res;   // final max-norm residual / max-norm right-hand side
    double gmax;        // max |grad Q| over the faces
};

int pf_create(const compas_b200_parm* p, const compas_b200_geom* g, PfLevel** out, std::string* err);
void pf_destroy(PfLevel* pf);

// Face gradients of Q (pf_gq) for the padded state U (Array4 layout of g) after a hyperbolic step of
// size dt. Synchronises the stream (the reference's host loop reads the same scalars).
int pf_grad_q(PfLevel* pf, const compas_b200_parm* p, const double* U, double dt, cudaStream_t st, PfInfo* info,
              std::string* err);

// The face gradient arrays (direction d nodal in d, x fastest), valid after pf_grad_q.
const double* pf_gq(const PfLevel* pf, int d);
// Device scalar holding the Phase-Field sub-step size for the stage kernels.
double* pf_dt_slot(PfLevel* pf);
// Device bytes held by the Phase-Field work arrays.
long long pf_bytes(const PfLevel* pf);

}  // namespace compas

// Batched advance of many independent single-box cases (uneven sizes, own EOS, own boundaries, own
// time-step control) through one persistent box-list launch per RK stage.
//
// Every array the launches read - the box descriptors, the tile and ghost prefix sums, the number of
// boxes and the per-case step-control blocks - lives in device memory at a fixed address, so the
// launches of one coarse step are captured once into a CUDA graph and replayed while cases are
// admitted and retired between replays (only the contents change). A case whose stop time or step
// budget is reached becomes a no-op until it is removed.
#pragma once

#include <algorithm>
#include <vector>

namespace compas {

struct FillListArgs {
    const BoxDesc* boxes;
    const int* nbox;
    const long long* ghost_off;  // exclusive prefix sums of BoxDesc::ghosts, nbox + 1 entries
    int N, D, m0;                // components, dimension, first momentum component
    int stage;                   // fills BoxDesc::U[stage]
};

__device__ __forceinline__ int find_box_ll(const long long* off, int nb, long long q) {
    int lo = 0, hi = nb - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= q) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void fill_list_kernel(FillListArgs F) {
    const int nb = *F.nbox;
    if (nb <= 0) return;
    const long long total = F.ghost_off[nb];
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int b = find_box_ll(F.ghost_off, nb, q);
        const BoxDesc& B = F.boxes[b];
        if (*B.done) continue;
        fill_ghost_cell(B.U[F.stage], B.g, F.N, F.D, F.m0, B.lo_bc, B.hi_bc, q - F.ghost_off[b]);
    }
}

// Per-case parameters of the device time-step control.
struct CaseStep {
    double cfl;
    double dx[3];
    int D;
    int limiter;
    int max_steps;
    double stop_time;
};

__global__ void step_begin_list_kernel(StepCtl* ctl, const CaseStep* cs, const int* slots, const int* nbox) {
    const int nb = *nbox;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        const int sl = slots[b];
        StepCtl* s = &ctl[sl];
        const CaseStep p = cs[sl];
        if (s->done) continue;
        if (!(s->t < p.stop_time) || s->steps >= p.max_steps) {
            s->done = 1;
            continue;
        }
        const double cmax = __longlong_as_double((long long)s->cmax);
        double dt_est = DBL_MAX;
        for (int d = 0; d < p.D; ++d) dt_est = dmin(dt_est, p.cfl * p.dx[d] / cmax);
        if (s->t == 0.0) s->dt_prev = dt_est;
        if (p.limiter && s->dt_prev > 0.0) dt_est = dmin(dt_est, 1.1 * s->dt_prev);
        double dt0 = dt_est;
        const double eps = 1.0e-3 * dt0;
        if (s->t + dt0 > p.stop_time - eps) dt0 = p.stop_time - s->t;
        if (!(dt0 > 0.0) || !(dt0 <= DBL_MAX)) {
            s->err |= COMPAS_B200_ERR_CFL;
            s->done = 1;
            continue;
        }
        s->dt = dt0;
        s->dt_prev = dt0;
        s->cmax = 0ull;
    }
}

__global__ void step_end_list_kernel(StepCtl* ctl, const int* slots, const int* nbox) {
    const int nb = *nbox;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        StepCtl* s = &ctl[slots[b]];
        if (s->done) continue;
        s->t += s->dt;
        s->steps += 1;
    }
}

static int tile_count(int dim, const Grid& g) {
    const int T = (dim == 2) ? kTile2 : kTile3;
    const long long t = (long long)((g.n[0] + T - 1) / T) * ((g.n[1] + T - 1) / T) * ((g.n[2] + (dim == 2 ? 1 : T) - 1) /
                                                                                     (dim == 2 ? 1 : T));
    return (int)t;
}

struct BatchCase {
    int id = -1;
    int slot = -1;
    compas_b200_parm p;
    compas_b200_geom g;
    double* U[3] = {nullptr, nullptr, nullptr};
    long long bytes = 0;
};

}  // namespace compas

struct compas_b200_batch {
    int physics, dim, nphase, limiter, precision;
    int capacity;
    std::vector<compas::BatchCase> cases;  // active cases, in box-list order
    std::vector<int> free_slots;
    int next_id = 0;
    compas::BoxDesc* d_boxes = nullptr;
    int* d_nbox = nullptr;
    int* d_tile_off = nullptr;
    long long* d_ghost_off = nullptr;
    int* d_slots = nullptr;
    compas::StepCtl* d_ctl = nullptr;
    compas::CaseStep* d_cs = nullptr;
    long long bytes_in_use = 0;
    long long launches = 0;
    cudaGraphExec_t graph = nullptr;
    cudaStream_t graph_stream = nullptr;
    int shape = 0, order = 0;   // box-list kernel launch shape and tile order (autotuner or forced)
    bool tuned = false, forced = false;
};

/* Test infrastructure (oracle): the C interface shared by the two CPU oracles of the finite-volume
 * right-hand side and TVD-RK3 level advance.
 *
 *   oracle/compas_oracle.c        plain-C restatement of the reference's algorithm (liboracle.so)
 *   oracle/ref_driver.cpp         the reference's own include/Physics_* and include/Operators_* headers,
 *                                 compiled against oracle/refshim, driven by a loop that restates
 *                                 source/Class_Compressible_PhaseField.cpp (oracle/_ref/libref_*.so)
 *
 * Both export the same symbols so a test can check one against the other and against the CUDA path.
 * Only tests, smoke() and the CPU-baseline leg of bench.py load these libraries.
 *
 * Array layout (AMReX Array4 with ghosts, one box covering the domain): component n of cell
 * (i,j,k), 0 <= i < n[0] valid, -ng <= i < n[0]+ng with ghosts, sits at
 *   n*S + (k+ng)*PY*PX + (j+ng)*PX + (i+ng),  PX = n[0]+2ng, PY = n[1]+2ng, PZ = n[2]+2ng (1 in 2D),
 *   S = PX*PY*PZ. In 2D there are no z ghosts (PZ = 1, k = 0).
 */
#ifndef COMPAS_ORACLE_API_H_
#define COMPAS_ORACLE_API_H_

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cmp_case {
    int physics;        /* 555 FIVEEQS, 666 SIXEQS, 55501 FIVEEQS_NPHASE, 66601 SIXEQS_IE_NPHASE
                         * (include/Macros.H:56-59; the last in the reference build only) */
    int dim;            /* 2 or 3 */
    int n[3];           /* valid cells per direction (n[2] = 1 in 2D) */
    int ng;             /* ghost cells (3 for WENO5/WENO5B) */
    double dx[3];       /* cell sizes (dx[2] unused in 2D) */
    int lo_bc[3];       /* COMPAS boundary codes: 0 interior/periodic, 2 outflow, 3 symmetry, */
    int hi_bc[3];       /*   4 slip wall, 5 no-slip wall (docs/user-guide/inputs.md:113-120) */
    double A1, A2, B1, B2, C1, C2, D1, D2;  /* EOS coefficients as source/Parm.cpp:101-188 */
    int id_limiter;     /* FiniteVolume.Scheme (FiniteVolume_Parameter.H:51-147): with id_weno 1, 5 WENO5, 6 WENO5B; */
    int id_weno;        /*   with id_weno 0, 0 GODUNOV, 1 MUSCL(-Minmod), 2 -vanLeer, 3 -Superbee, 4 -MC */
    int id_riemann;     /* Physics.RiemannSolver: 0 LLF, 1 HLL, 2 HLLC */
    int source_term;    /* FIVEEQS Physics.source_term (K term): 0 or 1 */
    int relaxation;     /* SIXEQS, SIXEQS_IE_NPHASE Physics.pressure_relaxation: 0 or 1 */
    double relax_trace; /* SIXEQS, SIXEQS_IE_NPHASE Physics.pressure_relaxation_trace */
    int thinc;          /* FiniteVolume.THINC: 0 or 1 */
    int thinc_use_normal;
    double thinc_eps, thinc_beta, thinc_normal_threshold;
    double cfl;         /* run.cfl */
    int change_limiter; /* run.timestep_change_limiter */
    int nphase;         /* FIVEEQS_NPHASE, SIXEQS_IE_NPHASE: phases (the build's NPHASE); 2 otherwise */
    double Ak[4], Bk[4], Ck[4], Dk[4];  /* the N-phase models' EOS coefficients per phase (source/Parm.cpp:185-253) */
    int amr_interp;     /* amr.Interpolater of the multi-level advance: 0 lincc_interp, 1 pc_interp */
    int id_bound;       /* FiniteVolume.ID_Bound (FiniteVolume_Parameter.H:45): 1 the bound-preserving branch and
                         * the energy check of every stage with the step taken again (FIVEEQS) */
    int id_lambda;      /* FiniteVolume_Parm.ID_Lambda of cmp_compute_dudt / cmp_rk3_step (1 default; the
                         * advance switches it to 0 for a step it takes again) */
} cmp_case;

/* Number of conserved components of the case (NSTATE). */
int cmp_nstate(const cmp_case* c);

/* Fill the ghost cells of U (all components) from the valid cells by the boundary codes, direction by
 * direction (x, then y, then z), each over the full extent of the other directions. */
int cmp_fill_ghosts(const cmp_case* c, double* U);

/* dUdt (same layout as U; valid cells written) of the state U whose ghosts are filled, and the largest
 * face wave speed over the low faces of the valid cells (the c_max norm of the reference). */
int cmp_compute_dudt(const cmp_case* c, const double* U, double* dUdt, double* cmax);

/* FiniteVolume.ID_Bound = 1: smallest energy bound over the valid cells of U (MinEnergyBound), and
 * the number of steps the last cmp_advance took again. */
int cmp_energy_bound_min(const cmp_case* c, const double* U, double* out);
int cmp_bound_restarts(void);

/* Pressure relaxation of the valid cells of U in place (SIXEQS, SIXEQS_IE_NPHASE; no-op otherwise). */
int cmp_relax(const cmp_case* c, double* U);

/* One TVD-RK3 step of size dt on U (valid cells in, valid cells out; ghosts are scratch).
 * cmax receives the largest face wave speed over the three stages. */
int cmp_rk3_step(const cmp_case* c, double* U, double dt, double* cmax);

/* nsteps level steps with the reference's time-step control (ComputeDt: cfl, the 1.1x change limiter,
 * the stop-time clamp). *t is the start time on entry and the end time on exit; dts[s] receives the
 * step sizes (may be NULL). Returns the number of steps taken. */
int cmp_advance(const cmp_case* c, double* U, int nsteps, double stop_time, double* t, double* dts);

/* Threads the library uses (OpenMP builds); 1 otherwise. */
int cmp_threads(void);

/* Phase-Field regularisation step (FIVEEQS, SIXEQS; PhaseField_Evolve, source/Class_Compressible_PhaseField.cpp:
 * 424-595). The reference-header build implements it; the plain-C port returns -2. */
typedef struct cmp_pf {
    int mechanism;          /* PhaseField ID_Mechanism: 1 CAC-Adv, 3 ACDI (PhaseField_Parameter.H:66-110) */
    int explicit_rc;        /* PhaseField.ID_ExplicitRC: 0 implicit (elliptic solve), 1 explicit */
    double lambda;          /* PhaseField.Lambda (<= 0: 1) */
    double eta;             /* PhaseField.Eta (<= 0: Eta_Multiplier x the largest cell size) */
    double eta_factor;      /* PhaseField.Eta_Factor */
    double eta_multiplier;  /* PhaseField.Eta_Multiplier */
    double cfl;             /* PhaseField.cfl */
    int max_step;           /* PhaseField.max_step */
    double tol_rel;         /* LinearSystem.tol_rel of the elliptic solve */
    int phase2flux;         /* PhaseField.ID_FluxPhase2Flux: 0 phasic, 1 mixture (PhaseField_Parameter.H:53) */
    int flux;               /* PhaseField.ID_Flux: 0 upwind/downwind, 1 HLL (PhaseField_Parameter.H:52) */
} cmp_pf;

/* One Phase-Field step after a hyperbolic step of size dt: mechanism pseudo-time evolution, the
 * regularisation potential gradient on faces, and the sub-stepped TVD-RK3 advance of U over dt.
 * info (may be NULL) receives {max |u|, mobility, eta, mechanism sub-steps, Phase-Field sub-steps,
 * max |grad Q|}. */
int cmp_pf_step(const cmp_case* c, const cmp_pf* pf, double* U, double dt, double* info);

/* The face gradients grad Q (component d in gq[d], nodal in direction d, (n[d]+1) faces, x fastest)
 * that cmp_pf_step computes for U and dt, without advancing U. */
int cmp_pf_grad_q(const cmp_case* c, const cmp_pf* pf, const double* U, double dt, double* gq0, double* gq1,
                  double* gq2, double* info);

/* cmp_advance with a Phase-Field step after every hyperbolic step (Evolve, source/
 * Class_Compressible_PhaseField.cpp:171-330). */
/* The Phase-Field right-hand side (PhaseField_compute_dUdt_FV) of the padded state U, its ghosts filled
 * here, for given face gradients gq_d of the regularisation potential; dUdt (padded) receives the valid
 * cells. The reference-header build implements it; the plain-C port returns -2. */
int cmp_pf_dudt(const cmp_case* c, const cmp_pf* pf, const double* U, const double* gq0, const double* gq1,
                const double* gq2, double* dUdt);

int cmp_advance_pf(const cmp_case* c, const cmp_pf* pf, double* U, int nsteps, double stop_time, double* t,
                   double* dts);

/* Multi-level (AMR) advance of a fixed box hierarchy, refinement ratio 2, with subcycling, flux
 * registers, reflux and average-down (timeStepWithSubcycling, source/Class_Compressible_PhaseField.cpp:
 * 4359-4451). c describes level 0 (domain cells, cell size, boundary codes, scheme); box b lives on
 * level boxes[b].lev with inclusive corners lo/hi in that level's index space, and U[b] is its
 * padded state (the Array4 layout of a single-box case of the box's size). Level 0 must cover the
 * domain and every level must be properly nested in the one below. The reference-header build
 * implements it; the plain-C port returns -2. Returns the number of level-0 steps. */
typedef struct cmp_amr_box {
    int lev;
    int lo[3];
    int hi[3];
} cmp_amr_box;

int cmp_amr_advance(const cmp_case* c, int nlev, const cmp_amr_box* boxes, int nbox, double** U, int nsteps,
                    double stop_time, double* t, double* dts);

/* Refinement tags of one level (ErrorEst, source/COMPAS.cpp:767-932): for each criterion, the state
 * component (derived 0) or the derived variable (derived 1, compute_derived_var of the model, into a
 * scratch array over the valid cells grown by one) is tested with the reference's Tagging.H functions:
 * kind 0 state_grad (threshold v0), 1 state_value_less (v0), 2 state_value_greater (v0), 3
 * state_value_range (v0, v1). U is padded with its ghosts filled (two layers where a velocity-gradient
 * variable is tagged by gradient); tags (valid cells, x fastest) receive 1 where tagged, 0 elsewhere.
 * cv holds prob.EOS.cv_1, cv_2 (temperature). FIVEEQS and SIXEQS in the reference-header build; the
 * plain-C port returns -2. */
typedef struct cmp_tag_crit {
    int var;
    int derived;
    int kind;
    double v0, v1;
} cmp_tag_crit;

int cmp_tag(const cmp_case* c, const double* cv, const double* U, const cmp_tag_crit* crit, int ncrit,
            unsigned char* tags);

/* Plot variables of the valid cells: variable v is state component vars[v] (derived[v] = 0) or the
 * model's derived variable vars[v] (compute_derived_var, derived[v] = 1); out receives nvars x cells
 * doubles, variable-major, x fastest. U is padded with its ghosts filled. FIVEEQS and SIXEQS in the
 * reference-header build; the plain-C port returns -2. */
int cmp_derive(const cmp_case* c, const double* cv, const double* U, const int* vars, const int* derived, int nvars,
               double* out);

/* The reference's THINC face value (Reconstruction2Face_THINC_D, include/Operators_FV/
 * Reconstruction2Face_THINC_D.H:13-35) for n parameter sets. Reference-header build; the port returns -2. */
int cmp_thinc_face(const double* beta, const double* sigma, const double* abar, const int* side, long long n,
                   double* out);

#ifdef __cplusplus
}
#endif

#endif

/* compas_b200: B200-native (sm_100a) finite-volume right-hand side and TVD-RK3 level advance of the
 * COMPAS five- and six-equation diffuse-interface models, behind a plain C ABI.
 *
 * Data layout. A state array is one AMReX FArrayBox as Array4 sees it: double precision, SoA,
 * component-major, x fastest, covering the valid box plus `ng` ghost cells on every side (no z
 * ghosts in 2D). Component n of cell (i,j,k), 0 <= i < n[0] valid, sits at
 *     n*S + (k+gz)*PY*PX + (j+ng)*PX + (i+ng),
 *     PX = n[0]+2ng, PY = n[1]+2ng, PZ = n[2]+2gz, S = PX*PY*PZ, gz = ng in 3D and 0 in 2D.
 * This is the layout of MultiFab::fabPtr(mfi)->dataPtr() for a box grown by ng, so an AMReX caller
 * passes its device pointers unchanged.
 *
 * Errors. Functions return COMPAS_B200_OK (0) or a negative COMPAS_B200_E* code; the reference
 * aborts the process instead (amrex::Abort). Device kernels never trap: conditions the reference
 * aborts on inside device code (NASG covolume, NaN state) set bits of a device status word
 * (COMPAS_B200_ERR_*), which the host reads after the step.
 *
 * Streams. Every device-side call is asynchronous on the cudaStream_t passed as `stream` (NULL =
 * legacy default stream); calls on one level object must not overlap.
 */
#ifndef COMPAS_B200_H_
#define COMPAS_B200_H_

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes --------------------------------------------------------------------------- */
#define COMPAS_B200_OK 0
#define COMPAS_B200_EARG (-1)      /* invalid argument or unknown inputs key/value */
#define COMPAS_B200_ECUDA (-2)     /* a CUDA runtime call failed */
#define COMPAS_B200_ENOMEM (-3)    /* device allocation failed */
#define COMPAS_B200_ESTATE (-4)    /* the status word reports an error (see compas_b200_level_status) */
#define COMPAS_B200_EUNSUPPORTED (-5)

/* ---- device status word bits (set by kernels, read by the host) ----------------------------- */
#define COMPAS_B200_ERR_NAN 0x1u          /* a NaN in the updated state (reference: SumVar abort) */
#define COMPAS_B200_ERR_COVOLUME 0x2u     /* NASG 1 - b rho <= 0 (include/EquationOfState_NASG.H:26-32) */
#define COMPAS_B200_ERR_RELAX_NOROOT 0x4u /* safeguarded relaxation found no root */
#define COMPAS_B200_ERR_CFL 0x8u          /* non-positive or non-finite time step */
#define COMPAS_B200_ERR_TIMEOUT 0x10u     /* an asynchronous (TMA) copy did not complete within its bounded wait */
#define COMPAS_B200_ERR_BOUND 0x20u       /* FiniteVolume.ID_Bound = 1: the energy bound still failed after the
                                           * step was taken again with the general wave-speed bound */

/* ---- models and schemes (the reference's compile-time PHYSICS and run-time keys) ------------ */
#define COMPAS_B200_FIVEEQS 555 /* include/Macros.H:56 */
#define COMPAS_B200_SIXEQS 666  /* include/Macros.H:57 */
#define COMPAS_B200_FIVEEQS_NPHASE 55501 /* include/Macros.H:58: N-phase five-equation model */
#define COMPAS_B200_SIXEQS_IE_NPHASE 66601 /* include/Macros.H:59: N-phase six-equation model, internal-energy
                                             * form (plain FP64, single-level API; NPHASE 2, 3 in 2D, 3 in 3D) */
#define COMPAS_B200_MAX_PHASES 4         /* largest NPHASE this build instantiates */

/* Parameters of the hot path: the fields of the reference's `struct Parm`
 * (exec/_Tests/Advection/prob/Parm.H:33-117) that the right-hand side reads, plus the run keys of
 * the level advance. Fill with compas_b200_parm_init, then compas_b200_parm_set per inputs key. */
typedef struct compas_b200_parm {
    int physics;          /* COMPAS_B200_FIVEEQS, COMPAS_B200_SIXEQS, COMPAS_B200_FIVEEQS_NPHASE or
                           * COMPAS_B200_SIXEQS_IE_NPHASE */
    int dim;              /* 2 or 3 (AMREX_SPACEDIM) */
    /* prob.EOS.* (source/Parm.cpp:101-188): raw inputs and the derived partial-form coefficients */
    int eos;              /* 0 ideal gas, 1 stiffened gas, 3 NASG */
    double gamma_1, gamma_2, pinf_1, pinf_2, b_1, b_2, q_1, q_2;
    double A1, A2, B1, B2, C1, C2, D1, D2;
    /* FiniteVolume.* (include/Operators_FV/FiniteVolume_Parameter.H:25-202) */
    int id_limiter;       /* with id_weno 1: 3 WENO3, 4 WENO3B, 5 WENO5, 6 WENO5B; with id_weno 0: 0 GODUNOV, 1 MUSCL(-Minmod),
                           * 2 MUSCL-vanLeer, 3 MUSCL-Superbee, 4 MUSCL-MC (the reference's ID_Limiter) */
    int id_weno;          /* the reference's ID_WENO: 1 for WENO5 / WENO5B, 0 for GODUNOV and MUSCL */
    int num_grow;         /* ghost cells the scheme reads (3 for WENO5/WENO5B) */
    int thinc;            /* FiniteVolume.THINC */
    int thinc_use_normal;
    double thinc_eps, thinc_beta, thinc_normal_threshold;
    /* Physics.* */
    int id_riemann;       /* Physics.RiemannSolver: 2 HLLC (source/Class_Compressible_PhaseField.cpp:92-111) */
    int source_term;      /* FIVEEQS Physics.source_term (Kapila K term) */
    int relaxation;       /* SIXEQS Physics.pressure_relaxation */
    double relax_trace;   /* SIXEQS Physics.pressure_relaxation_trace */
    /* run.* (source/COMPAS.cpp:1276-1314) */
    double cfl;
    int change_limiter;   /* run.timestep_change_limiter */
    /* precision of the bulk arithmetic (inputs key compas_b200.precision): 0 plain FP64, bit-compatible
     * with the reference; 1 mixed: FP32 reconstruction, FP64 pressure recovery, Riemann solver,
     * stage accumulation and relaxation */
    int precision;
    /* PhaseField.* (include/Physics_PhaseField/PhaseField_Parameter.H:25-117) and LinearSystem.tol_rel
     * (include/Operators_LinearSystem/LinearSystem_Parameter.H:27): the regularisation step after
     * every hyperbolic step (FIVEEQS, SIXEQS) */
    int phase_field;          /* PhaseField.phase_field */
    int pf_mechanism;         /* PhaseField.Mechanism: 1 CAC-Adv, 3 ACDI (the reference's ID_Mechanism) */
    int pf_explicit_rc;       /* PhaseField.ID_ExplicitRC: 0 elliptic solve, 1 explicit (flux-based only) */
    int pf_flux;              /* PhaseField.ID_Flux: 0 upwind/downwind, 1 HLL phase fluxes */
    int pf_phase2flux;        /* PhaseField.ID_FluxPhase2Flux: 0 phasic, 1 mixture formulation; default 1
                               * for FIVEEQS (PhaseField_Parameter.H:53) and 0 for SIXEQS, whose Parm.H
                               * sets it (exec/_Tests/Advection/prob/Parm.H:48-50) */
    double pf_lambda;         /* PhaseField.Lambda (<= 0: 1) */
    double pf_eta;            /* PhaseField.Eta (<= 0: Eta_Multiplier x the largest cell size) */
    double pf_eta_factor;     /* PhaseField.Eta_Factor */
    double pf_eta_multiplier; /* PhaseField.Eta_Multiplier */
    double pf_cfl;            /* PhaseField.cfl */
    int pf_max_step;          /* PhaseField.max_step */
    double pf_tol_rel;        /* LinearSystem.tol_rel */
    /* FIVEEQS_NPHASE, SIXEQS_IE_NPHASE: the number of phases (the reference's compile-time NPHASE; 2 for
     * the two-phase models) and the per-phase lists prob.EOS.gamma/pinf/b/q with their partial-form
     * coefficients (source/Parm.cpp:185-262, :364-446); the A1..D2 fields above are not used by these
     * models */
    int nphase;
    double gamma_k[COMPAS_B200_MAX_PHASES], pinf_k[COMPAS_B200_MAX_PHASES];
    double b_k[COMPAS_B200_MAX_PHASES], q_k[COMPAS_B200_MAX_PHASES];
    double Ak[COMPAS_B200_MAX_PHASES], Bk[COMPAS_B200_MAX_PHASES];
    double Ck[COMPAS_B200_MAX_PHASES], Dk[COMPAS_B200_MAX_PHASES];
    /* compas_b200.autotune (this engine's key, default 1): levels and batches pick the stage kernel's
     * launch shape and tile traversal order by timing the candidates on their own data the first
     * time they advance (the result is the same for every candidate) */
    int autotune;
    /* compas_b200.tma (this engine's key, default 1): levels of the 3D mixed form may stage the y and z
     * halo slabs of every tile into shared memory by TMA while the previous direction's faces are
     * computed (needs an even padded row length); the autotuner times both forms and keeps the faster,
     * a forced kernel (compas_b200_level_set_kernel) uses TMA; 0 always loads them with ordinary loads.
     * Same results either way. */
    int tma;
    /* prob.EOS.cv_1, prob.EOS.cv_2 (default 1): the phases' heat capacities, used by the derived
     * temperature of the refinement tagging (Conservative2Temperature) */
    double cv_1, cv_2;
    /* amr.Interpolater of the multi-level object's coarse-fine ghost cells and new fine cells
     * (source/COMPAS.cpp:1217-1221, :1611-1618): 0 lincc_interp (default), 1 pc_interp */
    int amr_interp;
    /* FiniteVolume.ID_Bound (include/Operators_FV/FiniteVolume_Parameter.H:45, :56): 1 the bound-preserving
     * right-hand side of FIVEEQS and FIVEEQS_NPHASE (MUSCLBP / WENO5BP face states limited by the energy
     * bound, the HLL solver with bounded wave speeds) and the level advance's energy check of every
     * stage with the step taken again on a violation (source/Class_Compressible_PhaseField.cpp:236-306,
     * :3780-3790); FP64 only. id_lambda is the reference's FiniteVolume_Parm.ID_Lambda (:47, not an inputs key):
     * 1 (default) the wave speeds from the sound speed, 0 the general bound the driver switches to
     * for the step it takes again; the level advance switches it by itself, a host that drives the
     * stage entry points sets it as the reference's Evolve does. */
    int id_bound;
    int id_lambda;
} compas_b200_parm;

/* One box covering a single-level domain (the valid cells), its ghost width and its boundary codes
 * (COMPAS codes, docs/user-guide/inputs.md:113-120: 0 interior/periodic, 2 outflow, 3 symmetry,
 * 4 slip wall, 5 no-slip wall). */
typedef struct compas_b200_geom {
    int n[3];       /* valid cells per direction; n[2] = 1 in 2D */
    int ng;         /* ghost cells of the arrays (>= parm.num_grow) */
    double dx[3];   /* cell sizes */
    int lo_bc[3];
    int hi_bc[3];
} compas_b200_geom;

/* ---- parameters ------------------------------------------------------------------------------- */

/* Reference defaults for the model (Parm, FiniteVolume_Parameter, Physics_Parameter and COMPAS run
 * defaults: WENO5, HLLC, cfl 0.4, change limiter on). FIVEEQS_NPHASE gets NPHASE = 2, the
 * reference's default (include/Macros.H:83-85). */
int compas_b200_parm_init(compas_b200_parm* p, int physics, int dim);

/* The same with the number of phases of FIVEEQS_NPHASE or SIXEQS_IE_NPHASE (2 <= nphase <=
 * COMPAS_B200_MAX_PHASES; this build instantiates the FIVEEQS_NPHASE kernels for nphase 2, 3, 4 in 2D
 * and 3 in 3D, the SIXEQS_IE_NPHASE kernels for nphase 2, 3 in 2D and 3 in 3D). For the two-phase
 * models nphase must be 2. */
int compas_b200_parm_init_nphase(compas_b200_parm* p, int physics, int dim, int nphase);

/* Set one inputs key, reference syntax and value set, e.g. ("FiniteVolume.Scheme", "WENO5B"),
 * ("Physics.RiemannSolver", "HLLC"), ("prob.EOS.gamma_2", "4.4"), ("run.cfl", "0.5"). Unknown keys
 * or values return COMPAS_B200_EARG with the valid values in compas_b200_last_error(), where the
 * reference aborts (e.g. include/Operators_FV/FiniteVolume_Parameter.H:143-146). EOS keys take
 * effect at compas_b200_parm_finalize. FIVEEQS_NPHASE and SIXEQS_IE_NPHASE take the per-phase lists
 * ("prob.EOS.gamma", "1.4 1.5 1.5"), "prob.EOS.pinf", "prob.EOS.b", "prob.EOS.q" with exactly
 * nphase values each (source/Parm.cpp:82-92). */
int compas_b200_parm_set(compas_b200_parm* p, const char* key, const char* value);

/* Derive the EOS coefficients A, B, C, D from prob.EOS.* as Parm::Initialize does
 * (source/Parm.cpp:101-188) and check the combination. */
int compas_b200_parm_finalize(compas_b200_parm* p);

/* Bytes of one state array (all components, with ghosts) of the geometry. */
long long compas_b200_state_bytes(const compas_b200_parm* p, const compas_b200_geom* g);

/* Last error message of the calling thread. */
const char* compas_b200_last_error(void);

/* ---- drop-in kernels on caller-owned device arrays ------------------------------------------- */
/* With compas_b200.autotune = 1 the stage-kernel entry points below run the launch shape and tile
 * order that a level of the same model and box size has tuned in this process (they never time
 * anything themselves); the results do not depend on it. */

/* Ghost cells of U from its valid cells by the boundary codes (single-box domain). Replaces the
 * physical-boundary and periodic part of COMPAS::FillPatch (source/COMPAS.cpp:1629-1732). */
int compas_b200_fill_boundary(const compas_b200_parm* p, const compas_b200_geom* g, double* U, void* stream);

/* dUdt = -div F(U) + non-conservative terms of the valid cells (dUdt has U's layout), from U with
 * its ghosts filled, in one fused launch (no face arrays in HBM). Replaces
 * Compressible_PhaseField::compute_dUdt_FV / ComputeFaceFluxes + FluxDivergence
 * (source/Class_Compressible_PhaseField.cpp:3151-3537; include/Classes_Physics/
 * Class_Compressible_PhaseField.H:116-139). cmax_dev (device double, may be NULL) receives
 * max(*cmax_dev, largest face wave speed over the low faces of the valid cells); err_dev (device
 * unsigned, may be NULL) is OR-ed with status bits. With FiniteVolume.ID_Bound = 1 (FIVEEQS, FIVEEQS_NPHASE) the
 * bound-preserving right-hand side runs instead (a face pass into stream-ordered scratch face arrays,
 * then the divergence), its cmax the flux functor's CFL speed of that branch. */
int compas_b200_compute_dUdt(const compas_b200_parm* p, const compas_b200_geom* g, const double* U, double* dUdt,
                             double* cmax_dev, unsigned int* err_dev, void* stream);

/* Number of non-conservative face terms of the model: 1 for FIVEEQS, FIVEEQS_NPHASE and SIXEQS_IE_NPHASE (the face
 * velocity u*), 3 for SIXEQS (u, u a1p1, u a2p2) - NC_TERMS of include/Macros.H, the component
 * count of the reference's fluxes_nc (source/Class_Compressible_PhaseField.cpp:3127-3143). */
int compas_b200_nc_terms(const compas_b200_parm* p);

#define COMPAS_B200_FACES_ALL 0       /* every face of the box */
#define COMPAS_B200_FACES_BOUNDARY 1  /* the faces on the box boundary: face 0 and face n[d] along d */

/* Face fluxes of one box, for the flux registers of a multi-level host. The fused kernels never
 * write face fluxes; a host that keeps AMReX's FluxRegister gets them here, recomputed from the same
 * ghost-filled stage state Us by the same device arithmetic as the stage kernel (FP64 form: the same
 * bits as the fluxes the stage used). Replaces what ComputeFaceFluxes leaves in `fluxes` and
 * `fluxes_nc` (source/Class_Compressible_PhaseField.cpp:3151-3301) for the flux registers; with
 * area_scaled set the values are multiplied by the face area as ScaleFaceFluxesByArea does
 * (:3433-3466: dy dz, dx dz, dx dy; dz = 1 in 2D), so the host calls CrseInit(flux[d], d, 0, 0, NSTATE,
 * -dt_lev) and FineAdd(flux[d], d, 0, 0, NSTATE, dt_lev) (and the same on flux_nc with NC_TERMS) as
 * compute_dUdt_FV does (:3501-3536).
 *   which: COMPAS_B200_FACES_ALL (CrseInit on a coarse level: coarse-fine faces may lie inside the
 *          box) or COMPAS_B200_FACES_BOUNDARY (FineAdd: only the box's own boundary faces are read),
 *          so the fused path keeps its zero face traffic and the registers cost one face pass.
 *   flux[d]: device face array of direction d, the layout of a face MultiFab with no ghosts
 *          (surroundingNodes(d)): n[e] + (e == d) faces along each e, nstate components, x fastest;
 *          flux_nc[d] likewise with compas_b200_nc_terms components. Either may be NULL (not
 *          written); in BOUNDARY mode only the boundary faces of the arrays are written.
 * The hyperbolic right-hand side without THINC (EUNSUPPORTED otherwise); with FiniteVolume.ID_Bound = 1
 * the fluxes of the bound-preserving branch. */
int compas_b200_face_fluxes(const compas_b200_parm* p, const compas_b200_geom* g, const double* Us, int which,
                            int area_scaled, double* const flux[3], double* const flux_nc[3], unsigned int* err_dev,
                            void* stream);

/* Smallest energy bound over the valid cells of U (FIVEEQS, FIVEEQS_NPHASE): rho E - |rho u|^2 / (2 rho)
 * minus the internal energy of every phase at its p_min (Conservative2EnergyBound), the value the reference's
 * MinEnergyBound (source/Class_Compressible_PhaseField.cpp:3596-3635) returns after every stage when
 * FiniteVolume.ID_Bound = 1; a negative value restarts the step. Written to *min_dev (device double;
 * +inf for a box without finite values). */
int compas_b200_energy_bound_min(const compas_b200_parm* p, const compas_b200_geom* g, const double* U,
                                 double* min_dev, void* stream);

/* One fused TVD-RK3 stage (stage 0, 1, 2) of ThirdOrderSSPRK
 * (source/Class_Compressible_PhaseField.cpp:3937-4107) followed by PostTimeStage (the SIXEQS
 * pressure relaxation, source/Class_Compressible6Eq_PhaseField.cpp:46-59, 437-474):
 *   stage 0: Unew = Us + dt L(Us)
 *   stage 1: Unew = 0.25 Us + 0.75 Uold;  Unew += (0.25 dt) L(Us)
 *   stage 2: Unew = 2/3 Us + 1/3 Uold;    Unew += (2/3 dt) L(Us)
 * Us must have its ghosts filled. dt is read from device memory (dt_dev). Unew may not alias Us. */
int compas_b200_rk3_stage(const compas_b200_parm* p, const compas_b200_geom* g, int stage, const double* Us,
                          const double* Uold, double* Unew, const double* dt_dev, double* cmax_dev,
                          unsigned int* err_dev, void* stream);

/* Pressure relaxation of the valid cells of U in place (SIXEQS). Replaces
 * Compressible6Eq_PhaseField::Relaxation (source/Class_Compressible6Eq_PhaseField.cpp:437-474). */
int compas_b200_relaxation(const compas_b200_parm* p, const compas_b200_geom* g, double* U, unsigned int* err_dev,
                           void* stream);

/* ---- Phase-Field regularisation (FIVEEQS, SIXEQS; PhaseField.phase_field = 1) -------------------
 * The level advance runs the Phase-Field step after every hyperbolic step by itself. The entry
 * points below expose its pieces to a host that keeps the reference's Phase-Field loop. Face arrays
 * gq_d are nodal in direction d: (n[0]+(d==0)) x (n[1]+(d==1)) x (n[2]+(d==2)) doubles, x fastest. */

/* Mechanism pseudo-time evolution over dt and the face gradients of the regularisation potential Q
 * for the padded state U: replaces PhaseFieldMechanism_Evolve + PhaseField_GradQPF
 * (source/Class_Compressible_PhaseField.cpp:596-711, :2132-2401) as PhaseField_Evolve (:424-545) calls
 * them. The implicit approach solves div(beta grad Q) = Div_Jhat with this engine's multigrid-
 * preconditioned conjugate gradients to LinearSystem.tol_rel (the reference uses AMReX MLMG).
 * Synchronous (the reference's loop reads the same scalars on the host); allocates work arrays.
 * info (host, 7 doubles, may be NULL): max|u|, mobility, eta, mechanism sub-steps, solver iterations,
 * max|grad Q|, final relative residual. */
int compas_b200_pf_grad_q(const compas_b200_parm* p, const compas_b200_geom* g, const double* U, double dt,
                          double* gq0, double* gq1, double* gq2, double* info, void* stream);

/* Phase-Field right-hand side of the padded state U (ghosts filled) into dUdt: replaces
 * PhaseField_compute_dUdt_FV (source/Class_Compressible_PhaseField.cpp:950-1004), SIXEQS with the
 * phase-energy exchange of PhaseField_FVM_SurfaceIntegral_NC
 * (include/Operators_Compressible6Eq_PhaseField/FVM_PhaseField_SurfaceIntegralNC_Compressible6Eq_PhaseField.H). */
int compas_b200_pf_compute_dUdt(const compas_b200_parm* p, const compas_b200_geom* g, const double* U, double* dUdt,
                                const double* gq0, const double* gq1, const double* gq2, unsigned int* err_dev,
                                void* stream);

/* One stage of PhaseField_ThirdOrderSSPRK (source/Class_Compressible_PhaseField.cpp:2619-2752): the
 * Phase-Field right-hand side of Us and the stage combination with Uold, dt read from device memory;
 * SIXEQS with Physics.pressure_relaxation relaxes the new state as PhaseField_PostTimeStage does
 * (source/Class_Compressible6Eq_PhaseField.cpp:61-70). */
int compas_b200_pf_rk3_stage(const compas_b200_parm* p, const compas_b200_geom* g, int stage, const double* Us,
                             const double* Uold, double* Unew, const double* dt_dev, const double* gq0,
                             const double* gq1, const double* gq2, unsigned int* err_dev, void* stream);

/* One TVD-RK3 step of size dt (stages 0-2 with their boundary fills and, for SIXEQS, the pressure
 * relaxation) in place on the caller-owned state U, WITHOUT ALLOCATING ANY DEVICE MEMORY. This entry
 * point has no counterpart in the reference. It is for callers that cannot call cudaMalloc - hosts
 * whose device memory is owned by another allocator (an AMReX arena, a framework's caching
 * allocator) that must stay the only allocator, or hosts with a fixed memory reservation that may
 * not grow - which still want a whole step from one call.
 *   - The two intermediate stage states live in a file-scope device array of this library,
 *     2 x 16 MiB plus 256 bytes, created on every GPU that loads the library and held until the
 *     process exits. A state (compas_b200_state_bytes) larger than 16 MiB is rejected with
 *     COMPAS_B200_EARG; use compas_b200_level_* for larger boxes.
 *   - The first call on a device looks up that array's device address (cudaGetSymbolAddress) and
 *     caches it for the life of the process, so make the first call on each device before any
 *     stream capture, and do not use this entry point after a cudaDeviceReset of that device.
 *   - The stage kernels run with the launch shape a level of the same box size has tuned in this
 *     process (as compas_b200_rk3_stage does), else the default shape.
 *   - Every call on a device shares the one array and leaves its contents behind; the call rewrites
 *     everything it reads. Calls that overlap on the GPU (other streams, other host threads) race on
 *     it: serialize them.
 *   - cmax_dev and err_dev as in compas_b200_rk3_stage (device pointers, may be NULL; cmax is
 *     max-accumulated, so clear it first if the step's own maximum is wanted). */
int compas_b200_rk3_step_noalloc(const compas_b200_parm* p, const compas_b200_geom* g, double* U, double dt,
                                 double* cmax_dev, unsigned int* err_dev, void* stream);

/* ---- single-level advance with device-resident state and time-step control -------------------- */

typedef struct compas_b200_level compas_b200_level;

/* Allocate the state (two arrays with ghosts) and the step-control block on the current device. */
int compas_b200_level_create(const compas_b200_parm* p, const compas_b200_geom* g, compas_b200_level** out);
int compas_b200_level_destroy(compas_b200_level* lv);

/* Copy a state (layout above, with ghosts; ghost values are ignored) in or out. `host` may be
 * pageable or pinned host memory, or device memory when is_device != 0. Sets the time to t0. */
int compas_b200_level_upload(compas_b200_level* lv, const double* src, int is_device, double t0, void* stream);
int compas_b200_level_download(compas_b200_level* lv, double* dst, int is_device, void* stream);

/* Replace the state only (host or device source), keeping the time, the step count and the time-step
 * control; for callers that hand the state over every step. */
int compas_b200_level_set_state(compas_b200_level* lv, const double* src, int is_device, void* stream);

/* One coarse step of a host-resident state: replaces ThirdOrderSSPRK on a MultiFab that lives in host
 * memory (source/Class_Compressible_PhaseField.cpp:3937-4107) for a host that hands the state over every
 * step. host_in (the state at the start of the step) and host_out (the state after it), both in the
 * layout above, should be pinned host memory for the copies to run asynchronously; they may be the
 * same array. The state moves in `slabs` slabs of whole tile layers along the slowest direction, copied
 * in and out on two copy streams of the level while the stages of neighbouring slabs run, so the copies
 * in both directions overlap the computation. Bit-identical to set_state + advance(1) + download, which
 * it falls back to for the level's first step, a periodic slowest direction, a Phase-Field level or
 * slabs < 2 (at most 64 slabs are used). Completion is ordered on `stream`. */
int compas_b200_level_step_host(compas_b200_level* lv, const double* host_in, double* host_out, int slabs,
                                void* stream);

/* Device pointer of the current state (layout above) for callers that keep data on the GPU. */
double* compas_b200_level_state(compas_b200_level* lv);

/* Enqueue nsteps coarse steps: ComputeDt (cfl, 1.1x change limiter, stop-time clamp;
 * source/COMPAS.cpp:2249-2303, CalculateInitialcmax at t = 0) then ThirdOrderSSPRK, all on the
 * device with no host synchronisation; steps after the stop time do nothing. With use_graph != 0
 * the launches of one step are captured once into a CUDA graph and replayed. */
int compas_b200_level_advance(compas_b200_level* lv, int nsteps, double stop_time, int use_graph, void* stream);

/* Wait for the level's work; report the time, the number of steps taken since upload and the status
 * word. Returns COMPAS_B200_ESTATE when the status word is non-zero. */
int compas_b200_level_sync(compas_b200_level* lv, double* t, int* steps, unsigned int* status);

/* FiniteVolume.ID_Bound = 1: how many steps of this level were taken again because a stage state
 * violated the energy bound (each restart is logged by the reference's Evolve,
 * source/Class_Compressible_PhaseField.cpp:264-306). Synchronises with the level's last advance. */
long long compas_b200_level_bound_restarts(const compas_b200_level* lv);

/* Step sizes of the steps taken since upload (up to n values). */
int compas_b200_level_dts(compas_b200_level* lv, double* dts, int n);

/* The stage kernel's launch shape (0..2: threads per CTA and CTAs per SM) and tile traversal order
 * (0 x fastest, 1 bricks of tiles) the level runs: the autotuner's choice after the first advance
 * (compas_b200.autotune = 1), else shape 0 / order 0 or what set_kernel forced. */
int compas_b200_level_kernel(const compas_b200_level* lv, int* shape, int* order);
int compas_b200_level_set_kernel(compas_b200_level* lv, int shape, int order);

/* 1 if the level's stage kernel stages the halo slabs by TMA (compas_b200.tma = 1, 3D mixed form, an
 * even padded row length, and after tuning the faster form), 0 if it loads them with ordinary loads. */
int compas_b200_level_tma(const compas_b200_level* lv);

/* Kernel launches the library enqueued on this level since upload. */
long long compas_b200_level_launches(compas_b200_level* lv);

/* Phase-Field sub-steps taken by the level so far (0 without PhaseField.phase_field). */
long long compas_b200_level_pf_substeps(const compas_b200_level* lv);

/* Counters of the level's last Phase-Field step, the quantities PhaseField_Evolve prints
 * (source/Class_Compressible_PhaseField.cpp:424-595) into info (host, 7 doubles) as
 * compas_b200_pf_grad_q returns them. */
int compas_b200_level_pf_info(const compas_b200_level* lv, double* info);

/* ---- batched independent cases ------------------------------------------------------------------
 * Many single-box cases of uneven size (each with its own EOS, boundary codes, stop time, step budget
 * and time-step control) advanced together: every RK stage of every case runs in ONE persistent
 * launch over a device-side box list (the serving/batching form; no reference counterpart - the
 * reference advances one problem per process). The launches of one coarse step are captured once in
 * a CUDA graph; admitting and retiring cases between advances does not invalidate it. A case whose
 * stop time or step budget is reached stays in place as a no-op until it is removed. All cases of a
 * batch share the model, dimension, scheme and precision. */
typedef struct compas_b200_batch compas_b200_batch;

int compas_b200_batch_create(int physics, int dim, int id_limiter, int precision, int capacity,
                             compas_b200_batch** out);
/* The same for FIVEEQS_NPHASE cases with nphase phases (compas_b200_batch_create takes nphase = 2). */
int compas_b200_batch_create_nphase(int physics, int dim, int nphase, int id_limiter, int precision, int capacity,
                                    compas_b200_batch** out);
int compas_b200_batch_destroy(compas_b200_batch* b);

/* Admit a case: allocates its three state arrays, copies the state in (padded layout, time 0) and
 * runs the t = 0 wave-speed pass. *case_id receives its id. */
int compas_b200_batch_add(compas_b200_batch* b, const compas_b200_parm* p, const compas_b200_geom* g,
                          const double* U, int is_device, double stop_time, int max_steps, void* stream,
                          int* case_id);
int compas_b200_batch_remove(compas_b200_batch* b, int case_id, void* stream);

/* The box-list kernel's launch shape and tile order (as compas_b200_level_kernel; a batch is tuned on
 * the cases it holds at its first advance, when the first case's parm has compas_b200.autotune = 1). */
int compas_b200_batch_kernel(const compas_b200_batch* b, int* shape, int* order);
int compas_b200_batch_set_kernel(compas_b200_batch* b, int shape, int order);

/* Enqueue nsteps coarse steps of every active case (no host synchronisation). */
int compas_b200_batch_advance(compas_b200_batch* b, int nsteps, int use_graph, void* stream);

/* Wait for the device and report, for up to `cap` cases in admission order, id, time, steps taken,
 * the no-op flag and the status word. Returns the number of cases in the batch. */
int compas_b200_batch_poll(compas_b200_batch* b, int* ids, double* t, int* steps, int* done, unsigned int* status,
                           int cap);
int compas_b200_batch_download(compas_b200_batch* b, int case_id, double* dst, int is_device, void* stream);

/* Device bytes held by the cases' state arrays. */
long long compas_b200_batch_bytes(compas_b200_batch* b);
long long compas_b200_batch_launches(compas_b200_batch* b);

/* ---- multi-level (AMR) advance of a fixed box hierarchy ------------------------------------------
 * Replaces timeStepWithSubcycling with its per-level ThirdOrderSSPRK, FillPatch / FillPatchStage,
 * flux registers, RefluxLev and AverageDownTo (source/Class_Compressible_PhaseField.cpp:4359-4451,
 * :3937-4107, :3472-3537; source/COMPAS.cpp:1549-1558, 1598-1799, 2249-2303;
 * source/Class_Compressible5Eq_PhaseField.cpp:77-160) for a hierarchy that does not regrid:
 * refinement ratio 2, subcycling, TVD-RK3 (FIVEEQS, WENO5 / WENO5B). Every level's boxes advance
 * together in one persistent box-list launch per RK stage. g0 describes level 0 (domain cells,
 * cell size, ghost width, boundary codes); box b lives on level boxes[b].lev with inclusive corners
 * lo / hi in that level's index space. Level 0 must tile the domain; every finer level must be
 * properly nested (its ghost cells and their interpolation stencil reach valid coarser cells). */
typedef struct compas_b200_amr compas_b200_amr;
typedef struct compas_b200_amr_box {
    int lev;
    int lo[3];
    int hi[3];
} compas_b200_amr_box;

int compas_b200_amr_create(const compas_b200_parm* p, const compas_b200_geom* g0, int nlev,
                           const compas_b200_amr_box* boxes, int nbox, compas_b200_amr** out);
int compas_b200_amr_destroy(compas_b200_amr* A);
/* State of box b (padded Array4 layout of a single box of the box's size and ghost width). */
int compas_b200_amr_upload(compas_b200_amr* A, int box, const double* src, int is_device, void* stream);
int compas_b200_amr_download(compas_b200_amr* A, int box, double* dst, int is_device, void* stream);
/* nsteps level-0 steps (each with its subcycled finer steps); the host computes dt from the levels'
 * wave speeds (ComputeDt), so every step synchronises the stream once. */
int compas_b200_amr_advance(compas_b200_amr* A, int nsteps, double stop_time, void* stream);
int compas_b200_amr_sync(compas_b200_amr* A, double* t, int* steps, unsigned int* status);
/* Level-0 step sizes taken so far (the first n). */
int compas_b200_amr_dts(const compas_b200_amr* A, double* dts, int n);
long long compas_b200_amr_launches(const compas_b200_amr* A);
/* Number of boxes of level lev. */
int compas_b200_amr_nbox(const compas_b200_amr* A, int lev);
/* Ghost cells of every box of level lev at its current time (same-level copies, coarse-fine
 * interpolation, physical boundaries: the FillPatch of a stage), so that compas_b200_amr_download
 * returns ghost-filled arrays (for plot variables that read neighbours). */
int compas_b200_amr_fill(compas_b200_amr* A, int lev, void* stream);
/* New box list for levels 1 .. nlev-1 (the regrid that follows ErrorEst; level 0 must be listed
 * unchanged, every level keeps at least one box, nesting as for compas_b200_amr_create). The state
 * stays on the device: a new box takes its valid cells from the old boxes of its level where they
 * overlap and elsewhere from the cell-conservative linear interpolation of the new coarser level
 * (the same interpolation as the coarse-fine ghost cells); time, step count and step sizes carry
 * over. Call between steps; synchronises the stream; A keeps its handle, box indices are the new
 * list's. */
int compas_b200_amr_regrid(compas_b200_amr* A, const compas_b200_amr_box* boxes, int nbox, void* stream);

/* Step control of a level, for checkpoint and restart: its time, the previous step size (COMPAS
 * dt[lev], the 1.1x change limiter's reference), the largest face wave speed of the last step's
 * stages (the next ComputeDt's input) and the step count. get synchronises the device. After set,
 * the next advance continues exactly as the checkpointed run would have (no initial wave-speed pass):
 * a restart from compas_b200_level_set_state + set_control reproduces the uninterrupted run to the
 * bit. Replaces the time-control part of COMPAS's WriteCheckpointFile / ReadCheckpointFile
 * (source/COMPAS.cpp:2514-2748). */
int compas_b200_level_get_control(compas_b200_level* lv, double* t, double* dt_prev, double* cmax, int* steps);
int compas_b200_level_set_control(compas_b200_level* lv, double t, double dt_prev, double cmax, int steps,
                                  void* stream);

/* ---- refinement tagging (ErrorEst, source/COMPAS.cpp:767-932) ------------------------------------
 * One criterion of one level, as ErrorEst applies it (include/Tagging.H): the variable is state
 * component `var` (derived = 0; the names of the model's vnamesC) or derived variable `var`
 * (derived = 1; the model's vnamesD: FIVEEQS a1rho1 a2rho2 rho_u rho_v rho_w rho_E a1 rho u v w P T c
 * Mach vorticity_mag q_criterion lambda2; SIXEQS a1rho1 a2rho2 rho_u rho_v rho_w a1rho1E1 a2rho2E2 a1
 * rho u v w P a1P1 a2P2 T c Mach vorticity_mag q_criterion lambda2), resolved from a name as the
 * reference's VariableRegistry does (state names first). kind: GRAD (run.refine.<name>.grad of the
 * level, v0), LESS (value_less, v0), GREATER (value_greater, v0), RANGE (value_range, v0 < x < v1). */
#define COMPAS_B200_TAG_GRAD 0
#define COMPAS_B200_TAG_LESS 1
#define COMPAS_B200_TAG_GREATER 2
#define COMPAS_B200_TAG_RANGE 3
#define COMPAS_B200_MAX_TAG_CRITERIA 16
typedef struct compas_b200_tag_criterion {
    int var;
    int derived;
    int kind;
    double v0, v1;
} compas_b200_tag_criterion;

/* Tags of the valid cells of one box: tags (device, n[0] x n[1] x n[2] bytes, x fastest) receive 1
 * where any criterion holds and 0 elsewhere. U is the padded device state with its ghosts filled
 * (two ghost layers where a velocity-gradient variable - vorticity_mag, q_criterion, lambda2 - is
 * tagged by its gradient). criteria is a host array of at most COMPAS_B200_MAX_TAG_CRITERIA entries:
 * the level's criteria (those whose run.refine.<name>.max_level exceeds the level). Replaces the
 * tagging loop of COMPAS::ErrorEst for FIVEEQS and SIXEQS; the AMReX host keeps its TagBoxArray
 * (copy the bytes into it) and its regrid. FIVEEQS_NPHASE: EUNSUPPORTED. */
int compas_b200_tag_cells(const compas_b200_parm* p, const compas_b200_geom* g, const double* U,
                          const compas_b200_tag_criterion* criteria, int ncriteria, unsigned char* tags,
                          void* stream);

/* Refinement tags of level lev at its current time (ErrorEst, source/COMPAS.cpp:767-932): the
 * level's ghost cells are filled as for a stage, then every box is tagged as compas_b200_tag_cells
 * does; tags (device) receives the valid cells of the level's boxes one after the other, in box order,
 * x fastest within a box. */
int compas_b200_amr_tag(compas_b200_amr* A, int lev, const compas_b200_tag_criterion* criteria, int ncriteria,
                        unsigned char* tags, void* stream);

/* Derived variables of the valid cells of one box, for plot files (PlotFileMF with
 * compute_derived_var, source/COMPAS.cpp:2483-2511): variable v is state component vars[v]
 * (derived[v] = 0) or the model's derived variable vars[v] (derived[v] = 1, the vnamesD list above);
 * out (device) receives n[0] x n[1] x n[2] doubles per variable, variable-major, x fastest. U is the
 * padded state with its ghosts filled (velocity-gradient variables read the neighbours). At most 32
 * variables; FIVEEQS and SIXEQS. */
int compas_b200_derive(const compas_b200_parm* p, const compas_b200_geom* g, const double* U, const int* vars,
                       const int* derived, int nvars, double* out, void* stream);

/* (check entry point) The THINC face value of alpha1 the stage kernels use (the tanh profile of
 * include/Operators_FV/Reconstruction2Face_THINC_D.H:13-35: steepness beta, sign sigma, cell mean
 * abar, side 1 the cell's high face, 0 its low face) for n parameter sets in device arrays; it calls
 * CUDA's exp, log and tanh where the reference's host build calls the C library's, so the two can
 * differ in the last bits - this entry point lets a test measure that difference face by face. */
int compas_b200_thinc_face_values(const double* beta, const double* sigma, const double* abar, const int* side,
                                  long long n, double* out, void* stream);

/* ---- measurement -------------------------------------------------------------------------------
 * (no counterpart in the reference) Sustained FMA throughput of the current GPU's FP32 (fp64 = 0)
 * or FP64 (fp64 = 1) pipe, in floating-point operations per second (one FMA = 2): one warm-up and one
 * timed launch of iters x 8 independent FMA chains per thread over every SM; synchronises the stream.
 * The denominators of the stage kernels' compute roofline. */
int compas_b200_fma_peak(int fp64, int iters, double* flops_per_s, void* stream);

#ifdef __cplusplus
}
#endif

#endif

/*
 * libchastegpu -- B200 monodomain tissue behind a plain C ABI.
 *
 * One context holds one monodomain tissue resident on one GPU: the mesh
 * operators (A = Am*Cm/dt*M + K and M), the cell states in
 * structure-of-arrays layout, the voltage, the Iion/Istim caches and the CG
 * workspace.  A PDE step is the operator-split step Chaste takes in
 * AbstractDynamicLinearPdeSolver::Solve (pde/src/solver/AbstractDynamicLinearPdeSolver.hpp:372-469):
 *   1. the ionic ODEs of every node with V clamped
 *      (AbstractCardiacTissue::SolveCellSystems, heart/src/tissue/AbstractCardiacTissue.cpp:464-567),
 *   2. b = M (Am*Cm*V/dt - Am*Iion - Istim)
 *      (MonodomainSolver::SetupLinearSystem, heart/src/solver/electrics/monodomain/MonodomainSolver.cpp:42-131),
 *   3. CG on A V' = b from the guess V (LinearSystem::Solve, linalg/src/LinearSystem.cpp:674-1215),
 * all on the device; host memory is touched only by the set/get calls.
 *
 * Every call returns a cg_status (0 = CG_OK).  No C++ exception crosses the
 * ABI.  A context is bound to one CUDA device and one stream; calls on the
 * same context must not run concurrently.
 */
#ifndef CHASTE_GPU_H
#define CHASTE_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cg_ctx cg_ctx;

/* Status codes.  CG_ERR_CG_MAXIT / CG_ERR_CG_DIVERGED are the KSP failures
 * Chaste turns into an exception (KSPEXCEPT, linalg/src/LinearSystem.cpp:1119-1129);
 * CG_ERR_STATE_RANGE mirrors VerifyStateVariables. */
typedef enum {
    CG_OK = 0,
    CG_ERR_ARG = 1,           /* invalid argument */
    CG_ERR_CUDA = 2,          /* CUDA runtime error (or no device) */
    CG_ERR_CG_MAXIT = 3,      /* KSP_DIVERGED_ITS */
    CG_ERR_CG_DIVERGED = 4,   /* KSP_DIVERGED_DTOL / indefinite matrix */
    CG_ERR_NAN = 5,           /* KSP_DIVERGED_NANORINF */
    CG_ERR_STATE_RANGE = 6,   /* a gate left [0,1] or a concentration became <= 0 */
    CG_ERR_ORDER = 7,         /* calls made in the wrong order */
    CG_ERR_TIMEOUT = 8,       /* a device-side grid barrier gave up (bounded wait) */
    CG_ERR_NOMEM = 9,         /* device allocation failed */
    CG_ERR_UNSUPPORTED = 10
} cg_status;

enum { CG_MODEL_LR91 = 0, CG_MODEL_TT06 = 1 };
/* Forward Euler (EulerIvpOdeSolver), Rush-Larsen (AbstractRushLarsenCardiacCell),
 * backward Euler (AbstractBackwardEulerCardiacCell: implicit steps for the states
 * linear in themselves, Newton for the rest), or the generalised Rush-Larsen
 * solvers GRL1IvpOdeSolver / GRL2IvpOdeSolver (ode/src/solver/GRL{1,2}IvpOdeSolver.cpp). */
enum { CG_ODE_FORWARD_EULER = 0, CG_ODE_RUSH_LARSEN = 1, CG_ODE_BACKWARD_EULER = 2,
       CG_ODE_GRL1 = 3, CG_ODE_GRL2 = 4 };
enum { CG_PC_NONE = 0, CG_PC_JACOBI = 1, CG_PC_BJACOBI = 2 };
/* Inner preconditioner of the mixed-precision solve on the slab stencil: the
 * tridiagonal x-line part of A over each warp's 32 consecutive nodes, or Jacobi.
 * No Chaste counterpart (Chaste has no mixed-precision solve). */
enum { CG_INNER_PC_LINE = 0, CG_INNER_PC_JACOBI = 1 };
enum { CG_PRECISION_FP64 = 0, CG_PRECISION_MIXED = 1 };
enum { CG_STIM_NONE = 0, CG_STIM_SIMPLE = 1, CG_STIM_REGULAR = 2 };
/* MonodomainSolver (heart/src/solver/electrics/monodomain/MonodomainSolver.cpp) or
 * OperatorSplittingMonodomainSolver (OperatorSplittingMonodomainSolver.cpp:40-117,
 * HeartConfig::SetUseReactionDiffusionOperatorSplitting): half a step of the cells
 * including V, the diffusion solve with z = Am*Cm*V/dt, the second half. */
enum { CG_SOLVER_MONODOMAIN = 0, CG_SOLVER_OPERATOR_SPLITTING = 1 };

/* HeartConfig fields used by the path (heart/src/problem/HeartConfig.cpp:1581-1650,
 * 2337-2412; defaults heart/src/problem/HeartConfigDefaults.hpp:53-91). */
typedef struct {
    int model;                 /* CG_MODEL_* */
    int ode_method;            /* CG_ODE_* */
    double ode_time_step;      /* ms */
    double pde_time_step;      /* ms */
    double surface_area_to_volume_ratio;  /* Am, 1/cm (default 1400) */
    double capacitance;        /* Cm, uF/cm^2 (default 1) */
    int ksp_preconditioner;    /* CG_PC_*; bjacobi (PETSc's on one process: ILU(0) of the whole
                                  matrix) in FP64 only, CG_ERR_UNSUPPORTED with mixed precision */
    int use_absolute_tolerance;/* 1: KSPSetTolerances(DBL_EPSILON, tol); 0: (tol, default) */
    double ksp_tolerance;
    int use_mass_lumping;
    int max_iterations;        /* 0 -> PETSc default 10000 */
    int precision;             /* CG_PRECISION_* */
    int device;                /* CUDA device ordinal */
    int check_state_ranges;    /* 1: device-side VerifyStateVariables analogue */
    double activation_threshold; /* mV; activation time = first step with V above it */
    int solver;                /* CG_SOLVER_* (default CG_SOLVER_MONODOMAIN) */
    int use_state_variable_interpolation; /* 1: SVI correction of the RHS
                                  (HeartConfig::SetUseStateVariableInterpolation,
                                  MonodomainCorrectionTermAssembler); default solver only */
    int mixed_inner_preconditioner; /* CG_INNER_PC_*: the FP32 inner solve of the mixed
                                  mode on a slab (default CG_INNER_PC_LINE); the FP64 outer
                                  residual and its stopping test keep ksp_preconditioner */
} cg_config;

/* SimpleStimulus (heart/src/stimulus/SimpleStimulus.cpp:44-76) / RegularStimulus
 * (heart/src/stimulus/RegularStimulus.cpp:43-81), magnitude in uA/cm^3. */
typedef struct {
    int kind;
    double magnitude;
    double duration;
    double start;
    double period;
    double stop;
} cg_stimulus;

typedef struct {
    long long steps;               /* PDE steps taken */
    double time;                   /* current simulation time, ms */
    int last_cg_iterations;
    int max_cg_iterations;
    long long total_cg_iterations;
    int refinement_sweeps;         /* mixed precision: FP64 outer corrections, last step */
    int operator_kind;             /* 0 CSR, 1 structured slab stencil */
    int status_bits;
    double ms_last_call;           /* device time of the last cg_step call */
    int pipelined_nodes_per_thread; /* mixed slab solve: > 0 when the single-reduction (pipelined)
                                       inner solve runs, keeping this many nodes per thread in registers */
    int cg_blocks;                 /* blocks of the persistent CG kernel (512 threads each; 1024 for a
                                      pipelined solve of a slab that fills every SM with them) */
    int inner_preconditioner;      /* mixed precision: CG_INNER_PC_* the inner solve uses
                                      (CG_INNER_PC_JACOBI on CSR meshes); FP64: -1 */
    int inner_line_segment;        /* x-line preconditioner: nodes per segment its x-lines are cut
                                      to (32, a warp's nodes); 0 without it */
    int step_graph;                /* 1: cg_step replays a CUDA graph of the step, 0: plain launches */
    int host_call_graph;           /* 1: the last cg_step_host call was replayed from a graph */
    int capture_error;             /* cudaError_t of the last graph capture that failed (0: none);
                                      the call then ran as plain launches */
} cg_stats;

/* Fill cfg with Chaste's defaults (LR91, FE, dt 0.01, Am 1400, Cm 1, Jacobi, atol 2e-4). */
void cg_default_config(cg_config* cfg);

/* Replaces MonodomainProblem construction + HeartConfig reads
 * (heart/src/problem/MonodomainProblem.cpp:45-77). */
int cg_create(const cg_config* cfg, cg_ctx** out);

/* Mesh + conductivities; assembles A and M on the host once and uploads them
 * (MonodomainSolver::SetupLinearSystem with computeMatrix, MonodomainSolver.cpp:51-76).
 * conn: n_elems x (dim+1) node indices; sigma: n_elems x dim diagonal
 * intracellular conductivities (AbstractCardiacTissue::CreateIntracellularConductivityTensor,
 * heart/src/tissue/AbstractCardiacTissue.cpp:240-349, axis-aligned fibres). */
int cg_set_mesh(cg_ctx* ctx, int n_nodes, int dim, const double* xyz, int n_elems,
                const int* conn, const double* sigma);

/* Regular slab mesh (AbstractTetrahedralMesh::ConstructRegularSlabMesh,
 * mesh/src/common/AbstractTetrahedralMesh.cpp:569-614) with uniform diagonal
 * sigma (dim values); lets the library use the matrix-free slab stencil. */
int cg_set_slab_mesh(cg_ctx* ctx, int dim, double h, double width, double height,
                     double depth, const double* sigma, int* n_nodes_out);

/* Bidomain without a bath (BidomainProblem, heart/src/problem/BidomainProblem.cpp;
 * BidomainSolver, heart/src/solver/electrics/bidomain/BidomainSolver.cpp:63-190;
 * BidomainAssembler.cpp:41-89): instead of cg_set_mesh, the same mesh with intracellular
 * and extracellular conductivities (n_elems x dim each).  The unknowns become the
 * interleaved pairs (V_i, phi_e_i); a step is the cells' ODEs, b = (M z, 0) and CG on
 * B = [Am Cm/dt M + K_i, K_i; K_i, K_i + K_e].  Without fixed nodes B is singular and
 * the solve removes the null space of constant phi_e from every preconditioned vector
 * (AbstractBidomainSolver::GenerateNullBasis, AbstractBidomainSolver.cpp:112-134).
 * FP64, Jacobi or no preconditioner, CG_SOLVER_MONODOMAIN, no SVI or mass lumping
 * (CG_ERR_UNSUPPORTED otherwise); snapshots are not available for it. */
int cg_set_bidomain_mesh(cg_ctx* ctx, int n_nodes, int dim, const double* xyz, int n_elems, const int* conn,
                         const double* sigma_i, const double* sigma_e);
/* SetFixedExtracellularPotentialNodes (AbstractBidomainSolver.cpp:262-290): phi_e = 0 at
 * these nodes (Dirichlet rows and columns), which removes the null space.  Before the
 * first step, once. */
int cg_set_fixed_extracellular_nodes(cg_ctx* ctx, const int* nodes, int n_nodes);
/* phi_e of every node (n_nodes doubles). */
int cg_get_extracellular_potential(cg_ctx* ctx, double* phi_e);

/* Cells: what AbstractCardiacCellFactory::CreateCardiacCellForTissueNode decides per node
 * (heart/src/problem/cell_factories/AbstractCardiacCellFactory.cpp:42-67).
 * init_states: n_nodes x n_states node-major (AoS as Chaste cells hold them) or NULL
 * for the model defaults; param_set: per-node index into param_table
 * (n_param_sets x n_params scale factors, n_param_sets <= 255) or NULL for all-ones. */
int cg_set_cells(cg_ctx* ctx, const double* init_states, const int* param_set,
                 const double* param_table, int n_param_sets);

/* Stimulus per node: stim_id[i] = -1 (ZeroStimulus) or an index into stims (< 255). */
int cg_set_stimulus(cg_ctx* ctx, const int* stim_id, const cg_stimulus* stims, int n_stims);

/* Advance n PDE steps (ODE -> RHS -> CG each), launched as a CUDA graph. */
int cg_step(cg_ctx* ctx, int n_steps);
/* The same with the voltage in host memory, for a caller that keeps V on the host
 * between steps (AbstractDynamicLinearPdeSolver::Solve hands the solution Vec back
 * every step, pde/src/solver/AbstractDynamicLinearPdeSolver.hpp:233-272): v_in
 * (n_nodes, may be NULL) is V before the first step -- page-locked memory is read by
 * the first step's ODE kernel through its device mapping, over the host link while
 * it computes; pageable memory is copied in, in pieces, the first step's ODE starting
 * on each piece as it arrives -- and V after the last step is copied to v_out (may be
 * NULL), with one synchronisation for the whole call.  v_in must not change during
 * the call.
 * keep_history = 1 declares that v_in continues the trajectory (the caller passes
 * back what the previous call returned), so the mixed solve keeps its extrapolated
 * initial guess; 0 treats v_in as new (as cg_set_voltage does).  With page-locked host
 * buffers the copy out is a DMA transfer and, when no printing-step output is configured,
 * the whole call is captured as a CUDA graph on its first use and replayed afterwards
 * (the four most recent (v_in, v_out, n_steps, keep_history) combinations are kept;
 * cg_stats.host_call_graph says whether the last call was a replay). */
int cg_step_host(cg_ctx* ctx, const double* v_in, int n_steps, double* v_out, int keep_history);

/* cg_step with device-side event timing per phase, launched kernel by kernel
 * (no graph): ms_solve_odes accumulates the ODE kernel (HeartEventHandler
 * SOLVE_ODES), ms_linear_solve the fused RHS + CG kernel (ASSEMBLE_RHS +
 * SOLVE_LINEAR_SYSTEM); global/src/timing/HeartEventHandler.hpp:55-71. */
int cg_step_profiled(cg_ctx* ctx, int n_steps, double* ms_solve_odes, double* ms_linear_solve);

int cg_get_voltage(cg_ctx* ctx, double* v);
int cg_set_voltage(cg_ctx* ctx, const double* v);
int cg_get_states(cg_ctx* ctx, double* states /* n_nodes x n_states, node-major */);
int cg_get_cell_state(cg_ctx* ctx, int node, double* state /* n_states */);
/* rGetIionicCacheReplicated / rGetIntracellularStimulusCacheReplicated
 * (heart/src/tissue/AbstractCardiacTissue.hpp:457-460). */
int cg_get_caches(cg_ctx* ctx, double* iionic, double* istim);
int cg_get_activation_times(cg_ctx* ctx, double* t /* -1 where not activated */);
int cg_get_stats(cg_ctx* ctx, cg_stats* stats);
/* Iteration count of each of the last min(n, steps) solves, oldest first. */
int cg_get_iteration_history(cg_ctx* ctx, int n, int* iterations);

/* y = B x for the inner preconditioner of a mixed-precision slab solve (the x-line
 * solve, CG_INNER_PC_LINE), applied on the device in FP32 to a host vector of n
 * values.  A diagnostic of the mixed solve (B must be symmetric positive definite for
 * CG); no Chaste counterpart.  CG_ERR_UNSUPPORTED when the context's solve has no
 * x-line preconditioner (FP64, CSR meshes, CG_INNER_PC_JACOBI). */
int cg_apply_inner_preconditioner(cg_ctx* ctx, const double* x, double* y);

int cg_num_nodes(cg_ctx* ctx, int* n);
/* Host only: the regular slab cg_set_slab_mesh builds (ConstructRegularSlabMesh,
 * mesh/src/common/AbstractTetrahedralMesh.cpp:569-614), for the calls that take a mesh
 * (cg_set_mesh, cg_set_bidomain_mesh).  With xyz and conn NULL only the sizes are
 * returned; xyz: n_nodes x 3, conn: n_elems x (dim + 1). */
int cg_slab_mesh(int dim, double h, double width, double height, double depth, int* n_nodes, int* n_elems,
                 double* xyz, int* conn);
int cg_num_states(int model, int* n);
int cg_num_params(int model, int* n);

/* Device-resident state snapshot: step, V, states, caches, activation times
 * (stands in for CardiacSimulationArchiver, heart/src/problem/CardiacSimulationArchiver.cpp:55-110). */
int cg_snapshot_size(cg_ctx* ctx, size_t* bytes);
int cg_snapshot(cg_ctx* ctx, void* host_buffer, size_t bytes);
int cg_restore(cg_ctx* ctx, const void* host_buffer, size_t bytes);

int cg_destroy(cg_ctx* ctx);
const char* cg_status_string(int status);

/* ------------------------------------------------- single-cell populations --
 * Many independent cells, each run for its own number of beats, integrated by
 * Rush-Larsen (AbstractRushLarsenCardiacCell::Compute,
 * heart/src/odes/AbstractRushLarsenCardiacCell.cpp:57-104) in FP64 and in FP32
 * within one launch per beat, with APD90 of every action potential measured as
 * CellProperties::CalculateActionPotentialDurations does
 * (heart/src/postprocessing/CellProperties.cpp:55-312, threshold -30 mV).
 * params: n_cells x n_params scale factors (or NULL for ones); stim: the
 * stimulus every cell receives (uA/uF; e.g. RegularStimulus(-52, 1, 1000, start)). */
typedef struct cg_batch cg_batch;
int cg_batch_create(int model, int n_cells, const int* beats, const double* params, const cg_stimulus* stim,
                    double dt, double beat_length, int max_aps, int device, cg_batch** out);
/* Times each candidate -- the per-beat kernel's launch shapes, threads per block
 * (32, 64, 128, 256) x cells advanced together by each thread (1, 2), and the
 * persistent engine -- on `steps` steps and keeps the fastest; the population is
 * reset to its initial state afterwards. */
int cg_batch_autotune(cg_batch* b, int steps, int* threads_per_block);
/* Set the per-beat engine's launch shape (threads per block a multiple of 32 up to
 * 1024, cells per thread 1 or 2) without timing, and select that engine; results do
 * not depend on it. */
int cg_batch_set_launch_shape(cg_batch* b, int threads_per_block, int cells_per_thread);
/* The launch shape in use (after cg_batch_autotune, or the default 64 x 1). */
int cg_batch_launch_shape(const cg_batch* b, int* threads_per_block, int* cells_per_thread);
/* Engines: CG_BATCH_PERSISTENT (default) runs the whole population in ONE launch
 * inside a CUDA graph -- blocks of 4 warps draw groups of 32 cells from a work queue
 * ordered by decreasing beat count, and each cell's step is split over a gate thread
 * (the voltage-only gates) and a state thread (currents, V, other states), with the
 * FP64 and FP32 copies in lockstep; CG_BATCH_PER_BEAT replays a graph of one launch
 * per beat.  cg_batch_autotune times both and keeps the faster; the results do not
 * depend on the engine. */
enum { CG_BATCH_PER_BEAT = 0, CG_BATCH_PERSISTENT = 1 };
int cg_batch_set_engine(cg_batch* b, int engine);
int cg_batch_engine(const cg_batch* b, int* engine);
/* Runs every beat of every cell; ms = device time. */
int cg_batch_run(cg_batch* b, double* ms);
/* apd64/apd32: n_cells x max_aps (-1 where no AP), n_ap: APs completed per cell,
 * max_dv: n_cells x max_beats largest |V32 - V64| per beat (0.1 ms samples),
 * states: n_cells x n_states final states.  Any pointer may be NULL. */
int cg_batch_results(cg_batch* b, double* apd64, double* apd32, int* n_ap64, int* n_ap32, float* max_dv,
                     double* states64, double* states32);
int cg_batch_destroy(cg_batch* b);

/* ------------------------------------------ cables for parameter fitting --
 * A 1D monodomain cable (P1 elements, forward Euler ODE step equal to the PDE
 * step, CG + Jacobi with PETSc's stopping test) whose parameters vary over R
 * contiguous regions, with the loss
 *     L = mean over steps n and probes k of (V_{n+1}(probe_k) - target[n][k])^2
 * and its gradient by the discrete adjoint of the operator-split step.  The
 * forward step is the one cg_step takes (MonodomainSolver.cpp:92-101,
 * MonodomainAssembler.cpp:43-66, AbstractCardiacTissue::SolveCellSystems with
 * ComputeExceptVoltage); the adjoint has no counterpart in the reference.
 *
 * Parameters of one set: n_regions rows of (n_params cell scale factors,
 * conductivity scale), so n_regions * (cg_num_params(model) + 1) doubles.
 * Node i lies in region floor(i R / n_nodes), element e (nodes e, e+1) in
 * region floor(e R / (n_nodes - 1)), both capped at R - 1.
 * Device pointers throughout; each call returns once its work on `stream`
 * (NULL: legacy default stream) has finished. */
typedef struct {
    int model;                     /* CG_MODEL_* */
    int n_nodes;                   /* 2 .. 1024 */
    double h;                      /* node spacing, cm */
    double conductivity;           /* mS/cm, before the region scale */
    double surface_area_to_volume_ratio;
    double capacitance;
    double time_step;              /* ms (ODE and PDE) */
    int n_steps;
    int n_regions;                 /* 1 .. 8 */
    int n_stimulated_nodes;        /* nodes 0 .. k-1 */
    double stimulus_magnitude;     /* uA/cm^3, SimpleStimulus from t = 0 */
    double stimulus_duration;      /* ms */
    double ksp_tolerance;          /* relative */
    int max_iterations;
    int checkpoint_every;          /* steps between adjoint checkpoints */
} cg_cable_config;

typedef struct cg_cable cg_cable;
/* 1000 nodes of h = 0.01 cm, LR91, sigma 1.75, Am 1400, Cm 1, dt 0.01 ms,
 * 400 ms, 4 regions, -5e5 uA/cm^3 for 0.5 ms on x < 0.02 cm, rtol 1e-8,
 * checkpoints every 200 steps. */
void cg_cable_default_config(cg_cable_config* cfg);
/* probes: n_probes distinct node indices (host). */
int cg_cable_create(const cg_cable_config* cfg, const int* probes, int n_probes, int device, cg_cable** out);
/* n_sets parameter sets in one launch (one CTA each).  d_targets (n_steps x
 * n_probes) and d_loss (n_sets) may both be NULL; d_traces (n_sets x n_steps x
 * n_probes) may be NULL; d_iterations (n_sets, total CG iterations) may be NULL.
 * keep_checkpoints: store the states every checkpoint_every steps for
 * cg_cable_backward (needs d_targets). */
int cg_cable_forward(cg_cable* c, int n_sets, const double* d_params, const double* d_targets, double* d_loss,
                     double* d_traces, int* d_iterations, int keep_checkpoints, void* stream);
/* dL/dparams (n_sets x R x (n_params + 1)) of the sets of the last forward
 * call made with keep_checkpoints, which must have had the same parameters
 * and targets. */
int cg_cable_backward(cg_cable* c, int n_sets, const double* d_params, const double* d_targets, double* d_grad,
                      void* stream);
int cg_cable_destroy(cg_cable* c);

/* ---------------------------------------------- mixed run populations --
 * Single-cell runs and cable runs of ONE cell model, each with its own length,
 * time step, parameters and stimulus, run together in ONE persistent launch
 * replayed from a CUDA graph: blocks draw jobs -- a group of single cells of about
 * one length, or one whole cable -- from a queue ordered by decreasing estimated
 * cost.  FP64.  A single-cell run is AbstractCardiacCell::Compute(0, t_end, tsamp)
 * with forward Euler (AbstractOneStepIvpOdeSolver::Solve,
 * ode/src/solver/AbstractOneStepIvpOdeSolver.cpp:41-91) or Rush-Larsen
 * (AbstractRushLarsenCardiacCell::Compute, heart/src/odes/AbstractRushLarsenCardiacCell.cpp:57-104),
 * Cm = 1; a cable run takes the cg_cable forward step.  Host pointers throughout. */
typedef struct cg_runs cg_runs;
int cg_runs_create(int model, int device, cg_runs** out);
/* A single-cell run of n_steps steps of dt (method CG_ODE_FORWARD_EULER or
 * CG_ODE_RUSH_LARSEN) sampled every sample_every steps (tsamp = sample_every * dt;
 * n_steps a multiple of sample_every).  params: cg_num_params(model) scale factors
 * (NULL: all 1); stim may be NULL.  *id receives the run's id. */
int cg_runs_add_cell(cg_runs* r, int method, const double* params, const cg_stimulus* stim, double dt, int n_steps,
                     int sample_every, int* id);
/* A cable run: cfg as for cg_cable_create (cfg->model must be the population's;
 * checkpoint_every is ignored), params n_regions x (n_params + 1), V at the probes
 * recorded after every sample_every-th step (cfg->n_steps a multiple of it). */
int cg_runs_add_cable(cg_runs* r, const cg_cable_config* cfg, const double* params, const int* probes, int n_probes,
                      int sample_every, int* id);
/* Times each launch shape -- threads per block (64, 128, 256) x single cells per
 * thread (1, 2); a cable's nodes are spread over the block's threads -- on the first
 * `steps` steps of every run and keeps the fastest.  Results do not depend on it
 * beyond the order of the cables' block sums. */
int cg_runs_autotune(cg_runs* r, int steps, int* threads_per_block, int* cells_per_thread);
int cg_runs_set_shape(cg_runs* r, int threads_per_block, int cells_per_thread);
int cg_runs_shape(const cg_runs* r, int* threads_per_block, int* cells_per_thread);
/* Runs every run from its initial state; ms = device time of the launch. */
int cg_runs_run(cg_runs* r, double* ms);
/* Results of run `id` after cg_runs_run.  Cell: states (n_states), trace
 * (n_samples = n_steps / sample_every + 1 voltages, the first at t = 0).  Cable:
 * states (n_nodes x n_states), trace (n_samples = n_steps / sample_every rows of
 * n_probes voltages), cg_iterations (summed over its steps).  Any pointer may be NULL. */
int cg_runs_result(cg_runs* r, int id, double* states, double* trace, int* n_samples, long long* cg_iterations);
int cg_runs_destroy(cg_runs* r);

/* Self-test of the device-side failure path, no counterpart in the reference:
 * launches a small kernel whose blocks wait, through the same bounded wait the
 * CG kernels' grid reductions use, for an arrival that never comes.  The wait
 * must end after about limit_ms (1 .. 2000) with the barrier-timeout status bit
 * (16) in *status_bits; *waited_ms (may be NULL) receives the longest wait.  No
 * fault, trap or hang is involved, and the device stays usable afterwards. */
int cg_selftest_barrier_timeout(int device, double limit_ms, int* status_bits, double* waited_ms);

/* ---------------------------------------------------------------- output --
 * Printing-step output kept on the device.  Replaces what
 * AbstractCardiacProblem::Solve writes through Hdf5DataWriter at t = 0 and every
 * printing time step (heart/src/problem/AbstractCardiacProblem.cpp:552-565; extra
 * state variables as HeartConfig::SetOutputVariables adds them), and the maps
 * PostProcessingWriter then derives from that file
 * (heart/src/postprocessing/PostProcessingWriter.cpp:226-345).
 *
 * cg_output_configure: a frame of V (and the listed state variables, indices
 * 1..S-1 as in cg_get_cell_state) is stored on the device now and after every
 * printing_steps PDE steps of cg_step / cg_step_profiled, up to max_frames
 * frames (0: no frames, printing-step modifiers only); a cg_step call that would
 * need more returns CG_ERR_NOMEM without stepping.  printing_steps = 0 turns the
 * output off and frees the frames.
 * cg_output_activation: ActivationOutputModifier (heart/src/problem/
 * ActivationOutputModifier.cpp:91-119) on the device at the current time and every
 * printing time from now on; cg_output_get_activation gives its four columns per
 * node (first activation, first recovery, second activation, second recovery;
 * -1 where not reached), n_nodes x 4.
 * cg_output_frames: frames so far and their times (ms).
 * cg_output_fetch: frames [first, first + count) in Hdf5DataWriter's Data
 * layout, count x n_nodes x (1 + n_state_vars) doubles, V first.
 * cg_output_cell_properties: CellProperties (heart/src/postprocessing/
 * CellProperties.cpp:55-330) of every node's stored voltage frames with the
 * given threshold: the APD map of WriteApdMapFile(percentage, threshold), the
 * upstroke-time map of WriteUpstrokeTimeMap and the maximum-upstroke-velocity
 * map of WriteMaxUpstrokeVelocityMap, each n_nodes x max_aps (row i: node i's
 * list, -999 after it; [0] where CellProperties raises) with the list lengths
 * in n_apd / n_upstroke (which may exceed max_aps; lists are then truncated).
 * Any output pointer may be NULL.
 * cg_output_conduction_velocity: WriteConductionVelocityMap(origin, distances)
 * (PropagationPropertiesCalculator::CalculateAllConductionVelocities), same
 * layout, distances[i] from the origin node to node i. */
int cg_output_configure(cg_ctx* ctx, int printing_steps, int max_frames, const int* state_vars, int n_state_vars);
int cg_output_frames(const cg_ctx* ctx, int* n_frames, double* times);
int cg_output_activation(cg_ctx* ctx, double threshold);
int cg_output_get_activation(cg_ctx* ctx, double* times);
int cg_output_fetch(cg_ctx* ctx, int first, int count, double* data);
int cg_output_cell_properties(cg_ctx* ctx, double percentage, double threshold, int max_aps, double* apd,
                              int* n_apd, double* upstroke_time, double* max_upstroke_velocity, int* n_upstroke);
int cg_output_conduction_velocity(cg_ctx* ctx, int origin, const double* distances, double threshold, int max_aps,
                                  double* cv, int* n_cv);

/* ------------------------------------------------------ multi-GPU slabs --
 * One rank's share of a slab tissue, one process per GPU.  Rows are owned in the
 * contiguous ranges PETSc's PETSC_DECIDE split gives Chaste's
 * DistributedVectorFactory (global/src/parallel/DistributedVectorFactory.cpp:44-64):
 * rank r of W owns n/W rows, one more when r < n % W.  With the slab numbering
 * ((k*NY + j)*NX + i) a range is a block of z-planes, and the stencil reaches
 * `halo` = NX*NY + NX + 1 rows on each side.  The ODE step is local
 * (AbstractCardiacTissue::SolveCellSystems over the rank's cells); the diffusion
 * solve is PETSc's CG with Jacobi (KSPSolve_CG, linalg/src/LinearSystem.cpp:1099)
 * split at its two inner-product reductions into phases that the caller
 * sequences, all-reducing each phase's four partial sums across the ranks and
 * exchanging halos before each operator application (chaste_b200/partition.py
 * does both with torch.distributed):
 *   phase 0: b = M z, r = b - A x, z' = B r; sums sum|b|, |B b|^2, |z'|^2, (r, z')
 *            (needs the V and z halos)
 *   phase 1: zero guess for a tiny right-hand side (LinearSystem.cpp:984-994):
 *            x = 0, r = b, z' = B b; sums |z'|^2, (b, z')
 *   phase 2: q = A z' + s0 q, p = z' + s0 p (s1 != 0: first iteration, no old p);
 *            sum (p, q) (needs the z' halo)
 *   phase 3: x += s0 p, r -= s0 q, z' = B r; sums |z'|^2, (z', r)
 * cg_part_halo_pack copies the `halo` rows next to the lower and upper neighbour
 * of vector `which` (0 V, 1 z, 2 z') into lo_out / hi_out; _unpack writes the
 * neighbours' rows into the halos; buffers may be host or device memory.  Global
 * arrays (init_states n x S, param_set, stim_id) are indexed by global row; the
 * rank keeps its own rows.  FP64, Jacobi or no preconditioner, the default solver;
 * a rank of a multi-rank run must own at least `halo` rows.  No counterpart in
 * the reference beyond the distributed PETSc objects it stands in for. */
typedef struct cg_part cg_part;
int cg_part_create(const cg_config* cfg, int dim, double h, double width, double height, double depth,
                   const double* sigma, int rank, int world, cg_part** out);
int cg_part_rows(const cg_part* part, int* lo, int* hi, int* halo, int* n_global);
int cg_part_set_cells(cg_part* part, const double* init_states, const int* param_set, const double* param_table,
                      int n_param_sets);
int cg_part_set_stimulus(cg_part* part, const int* stim_id, const cg_stimulus* stims, int n_stims);
int cg_part_ode(cg_part* part);
int cg_part_halo_pack(cg_part* part, int which, void* lo_out, void* hi_out);
int cg_part_halo_unpack(cg_part* part, int which, const void* lo_in, const void* hi_in);
int cg_part_cg_phase(cg_part* part, int phase, const double* scalars /* 2 */, double* sums /* 4 */);
/* ends the PDE step (the ODE step of the next call is at the next time) */
int cg_part_finish_step(cg_part* part);
int cg_part_get_voltage(cg_part* part, double* v /* the rank's rows */);
int cg_part_config(const cg_part* part, cg_config* cfg);
int cg_part_destroy(cg_part* part);

/* Allocation-free diffusion solve of one PDE step on a regular slab.
 *
 * No counterpart in the reference: Chaste always owns its PETSc vectors.  This
 * entry point is for callers that cannot allocate device memory (an embedding
 * program whose pool owns every device buffer, or code running where
 * cudaMalloc is not permitted): it solves (Am*Cm/dt*M + K) x = M z with the
 * same CG + Jacobi/none preconditioning, tolerance and stopping test as
 * cg_step, reading the caller's device buffers d_z and d_x (n doubles each;
 * d_x holds the initial guess on entry and the solution on return), and uses
 * a fixed device array inside the library for all of its workspace.
 *
 * Limit: slabs of at most 32768 nodes whose x-y plane (NX*NY + NX + 1) also
 * fits in 32768; larger sizes are rejected with CG_ERR_ARG.  The array is
 * reserved on every GPU that loads the library until the process exits and is
 * shared by all calls: calls that overlap on the GPU race, so serialise them.
 * The first call on a device resolves the array's device address and should be
 * made before any stream capture; a cudaDeviceReset after that first call is not
 * supported.  sigma is a HOST array of dim conductivities (mS/cm); d_z and d_x
 * are device pointers on the current device.  stream may be NULL (legacy default
 * stream) and otherwise must be a stream of the current device; the call returns
 * after the solve has completed on it.  cfg supplies pde_time_step, Am, Cm, the
 * KSP tolerance/preconditioner, max_iterations and mass lumping; FP64 only. */
int cg_slab_solve_noalloc(const cg_config* cfg, int dim, double h, double width, double height,
                          double depth, const double* sigma, const double* d_z, double* d_x,
                          void* stream, int* iterations);

#ifdef __cplusplus
}
#endif
#endif /* CHASTE_GPU_H */

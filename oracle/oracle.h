/*
 * CPU oracle for the monodomain operator-split step -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain C++ restatement of Chaste's CPU algorithm for this path.  Only the
 * tests, the smoke check and the CPU-baseline leg of the benchmark load it, as
 * the checker; the product path (libchastegpu.so) never links or calls it.
 *
 * Pinned against Chaste's own golden vectors (tests/golden/, extracted from
 * heart/test/data/ionicmodels/ ValidData files and the hard-coded values of
 * heart/test/monodomain/TestMonodomainProblem.hpp, TestIonicModels.hpp and
 * TestRushLarsen.hpp).  Each function cites the reference it restates.
 */
#ifndef CHASTE_ORACLE_H
#define CHASTE_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_LR91 = 0, ORC_TT06 = 1 };
/* cell ODE methods: forward Euler, Rush-Larsen, backward Euler, and the cell's ODE
 * solver set to GRL1IvpOdeSolver / GRL2IvpOdeSolver */
enum { ORC_FE = 0, ORC_RL = 1, ORC_BE = 2, ORC_GRL1 = 3, ORC_GRL2 = 4 };
enum { ORC_PC_NONE = 0, ORC_PC_JACOBI = 1, ORC_PC_BJACOBI = 2 };
enum { ORC_STIM_NONE = 0, ORC_STIM_SIMPLE = 1, ORC_STIM_REGULAR = 2 };
/* MonodomainSolver (default) or OperatorSplittingMonodomainSolver */
enum { ORC_SOLVER_MONODOMAIN = 0, ORC_SOLVER_OPERATOR_SPLITTING = 1 };

/* SimpleStimulus (heart/src/stimulus/SimpleStimulus.cpp:44-76) and
 * RegularStimulus (heart/src/stimulus/RegularStimulus.cpp:43-81).  The
 * DBL_EPSILON duration padding is applied by the evaluator. */
typedef struct {
    int kind;
    double magnitude;
    double duration;
    double start;
    double period;   /* regular only */
    double stop;     /* regular only (default DBL_MAX) */
} orc_stimulus;

int orc_num_states(int model);
int orc_num_params(int model);
void orc_initial_states(int model, double* y);

/* Evaluate a stimulus at time t. */
double orc_stimulus_value(const orc_stimulus* s, double t);

/* Single-cell Compute(tStart, tEnd, tSamp) with forward Euler
 * (AbstractCardiacCell::Compute -> AbstractOneStepIvpOdeSolver::Solve,
 * ode/src/solver/AbstractOneStepIvpOdeSolver.cpp:41-91) or Rush-Larsen
 * (AbstractRushLarsenCardiacCell::Compute, heart/src/odes/AbstractRushLarsenCardiacCell.cpp:57-104).
 * y (n_states) is updated in place; samples (n_samples x n_states, including
 * the initial state) are written when non-null.  Returns the sample count. */
int orc_cell_compute(int model, int method, double* y, const double* params,
                     const orc_stimulus* stim, double cm, double t0, double t1,
                     double dt, double tsamp, double* samples, int max_samples);

/* ComputeExceptVoltage(t0, t1) of one cell (V clamped), then GetIIonic. */
double orc_cell_compute_except_voltage(int model, int method, double* y, const double* params,
                                       const orc_stimulus* stim, double am_for_tissue, double cm,
                                       double t0, double t1, double dt);

double orc_cell_iionic(int model, const double* y, const double* params, double cm);

/* ---------------------------------------------------------------- mesh -- */
/* AbstractTetrahedralMesh::ConstructRegularSlabMesh
 * (mesh/src/common/AbstractTetrahedralMesh.cpp:569-614; 1D :244-275,
 * 2D staggered :277-381, 3D 6-tet cubes :384-566).  With xyz/conn null only
 * the sizes are returned.  Returns 0, or -1 when h does not divide a side. */
int orc_slab_mesh(int dim, double h, double width, double height, double depth,
                  int* n_nodes, int* n_elems, int* grid /* nx,ny,nz elements */,
                  double* xyz /* n_nodes*3 */, int* conn /* n_elems*(dim+1) */);

/* -------------------------------------------------------------- tissue -- */
typedef struct {
    int model;
    int ode_method;
    double dt_ode;
    double dt_pde;
    double am;            /* surface-area-to-volume ratio, 1/cm */
    double cm;            /* capacitance, uF/cm^2 */
    int pc;               /* ORC_PC_* */
    int use_abs_tol;      /* 1: KSP absolute tolerance, else relative */
    double tol;
    int mass_lumping;
    int max_iterations;   /* PETSc default 10000 */
    int solver;           /* ORC_SOLVER_* */
    int svi;              /* 1: state-variable interpolation (HeartConfig::SetUseStateVariableInterpolation) */
} orc_config;

typedef struct orc_tissue orc_tissue;

/* sigma: n_elems*dim diagonal conductivities (mS/cm).  stim_id: per node,
 * -1 = no stimulus, else index into stims.  param_id: per node index into
 * param_table (n_param_sets x n_params) or null for defaults.  init_states:
 * n_nodes x n_states (node-major) or null for the model defaults. */
orc_tissue* orc_tissue_create(const orc_config* cfg, int dim, int n_nodes, const double* xyz,
                              int n_elems, const int* conn, const double* sigma,
                              const int* stim_id, const orc_stimulus* stims, int n_stims,
                              const int* param_id, const double* param_table, int n_param_sets,
                              const double* init_states);
void orc_tissue_destroy(orc_tissue* t);
/* Advance n PDE steps starting at the tissue's current time.  Returns 0, or a
 * negative code when CG did not converge (-1 max iterations, -2 divergence,
 * -3 NaN).  cg_iters (n) receives the iteration count of each solve. */
int orc_tissue_step(orc_tissue* t, int n, int* cg_iters);
double orc_tissue_time(const orc_tissue* t);
void orc_tissue_get_voltage(const orc_tissue* t, double* v);
void orc_tissue_get_states(const orc_tissue* t, double* states /* n_nodes*n_states */);
void orc_tissue_get_caches(const orc_tissue* t, double* iion, double* istim);
/* Bidomain without a bath (BidomainProblem, BidomainSolver, BidomainAssembler): the
 * tissue's unknowns become the interleaved (V, phi_e) pairs of every node.  Call once,
 * before the first step, with the mesh again and both conductivities (n_elems*dim
 * each); fixed: nodes whose phi_e is held at 0 (SetFixedExtracellularPotentialNodes),
 * none for the singular system with the null space of constant phi_e.  Steps are
 * taken by orc_tissue_step; Jacobi or no preconditioner.  Returns 0 or -4. */
int orc_tissue_set_bidomain(orc_tissue* t, const double* xyz, int n_elems, const int* conn, const double* sigma_i,
                            const double* sigma_e, const int* fixed, int n_fixed);
void orc_tissue_get_extracellular(const orc_tissue* t, double* phi);
/* CSR of A = Am*Cm/dt*M + K and of M (for tests): returns nnz. */
int orc_tissue_matrix(const orc_tissue* t, int which /*0 A, 1 M*/, int* rowptr, int* cols, double* vals);
void orc_set_threads(int n);

/* --------------------------------------------------------------- cable -- */
/* A 1D cable with the ODE step equal to the PDE step, parameters varying over
 * R regions (node i in region floor(i R / n), element e in floor(e R / (n-1)),
 * capped at R-1); params: R rows of (cell scale factors, conductivity scale).
 * Nodes 0..n_stim-1 get SimpleStimulus(stim_mag, stim_dur, 0). */
typedef struct {
    int model;
    int n_nodes;
    double h, sigma, am, cm, dt;
    int n_steps, n_regions, n_stim;
    double stim_mag, stim_dur, rtol;
    int max_iterations;
    int checkpoint_every;   /* adjoint: steps between stored states (0: one segment) */
} orc_cable_config;

/* Loss L = mean over steps and probes of (V_{n+1}(probe) - target)^2, the probe
 * traces (n_steps x n_probes) when traces is non-null, and dL/dparams by the
 * discrete adjoint when grad is non-null (each segment of checkpoint_every
 * steps recomputed from its checkpoint; n_nodes * n_states times both the
 * segment length and the checkpoint count must stay <= 4e7).  Returns 0, -1 when CG reached maxit, -4 on bad arguments. */
int orc_cable_run(const orc_cable_config* c, const double* params, const int* probes, int n_probes,
                  const double* targets, double* loss, double* traces, double* grad);

/* The same gradient by forward mode: one tangent-linear run per parameter
 * (dual numbers through the cell model, A dV' = M dz - dA V' for the voltage),
 * `threads` runs at a time.  Independent of the adjoint's reverse products. */
int orc_cable_tangent_gradient(const orc_cable_config* c, const double* params, const int* probes, int n_probes,
                               const double* targets, double* grad, int threads);

#ifdef __cplusplus
}
#endif
#endif

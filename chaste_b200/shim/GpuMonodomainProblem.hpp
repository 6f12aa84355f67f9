/*
 * GpuMonodomainProblem -- the Chaste-side binding of libchastegpu.so.
 *
 * A Chaste build that wants the monodomain step on a B200 uses
 * GpuMonodomainProblem<DIM> where it used MonodomainProblem<DIM>; nothing else in
 * Chaste changes.  The problem creates its tissue and solver through Chaste's own
 * factory methods (MonodomainProblem::CreateCardiacTissue / CreateSolver,
 * heart/src/problem/MonodomainProblem.cpp:45-77), so AbstractCardiacProblem::Solve
 * (heart/src/problem/AbstractCardiacProblem.cpp:412-620) keeps its printing loop,
 * HDF5 output and checkpointing, and AbstractDynamicLinearPdeSolver::Solve
 * (pde/src/solver/AbstractDynamicLinearPdeSolver.hpp:328-497) keeps its TimeStepper
 * loop.  The device takes the step through the solver hooks that loop calls
 * (pde/src/solver/AbstractLinearPdeSolver.hpp:93-140):
 *
 *   InitialiseForSolve(V0)          -- the device tissue receives V0; the linear system
 *                                      is set to the identity once
 *   PrepareForSetupLinearSystem(V)  -- cg_step_host(ctx, NULL, 1, V_host, 1): the cells' ODEs, b = M z and the
 *                                      CG solve, on the device (MonodomainSolver's
 *                                      SolveCellSystems + SetupLinearSystem + KSPSolve)
 *   SetupLinearSystem(V, ...)       -- the right-hand side becomes the device solution,
 *                                      which the identity system hands back unchanged
 *
 * Set-up transfers, once, what the reference tissue holds:
 *   - the mesh: a regular slab made from HeartConfig goes to cg_set_slab_mesh (the
 *     matrix-free stencil); any other mesh to cg_set_mesh with its node coordinates,
 *     element connectivity and per-element diagonal intracellular conductivities
 *     (AbstractCardiacTissue::rGetIntracellularConductivityTensor);
 *   - the cells: model and ODE method of each node's cell, its state vector
 *     (AoS, as GetStdVecStateVariables returns it) and its modifiable parameters as
 *     scale factors of the generated models' defaults;
 *   - the stimuli: ZeroStimulus, SimpleStimulus and RegularStimulus objects of the
 *     cells, deduplicated into the stimulus table.
 * GetCardiacCell(i) stays a host object; SyncCellsFromDevice() copies the device
 * states into those objects (and the Iion cache into rGetIionicCacheReplicated) when
 * the caller wants them -- at the end of Solve, or at every printing time with
 * SetSyncCellsAtPrintingTimes(true).
 *
 * Every libchastegpu status other than CG_OK becomes an EXCEPTION, as the
 * reference raises KSPEXCEPT (linalg/src/LinearSystem.cpp:1119-1129) or
 * VerifyStateVariables' exception.
 */
#ifndef GPUMONODOMAINPROBLEM_HPP_
#define GPUMONODOMAINPROBLEM_HPP_

#include <cmath>
#include <map>
#include <string>
#include <vector>

#include "AbstractDynamicLinearPdeSolver.hpp"
#include "AbstractRushLarsenCardiacCell.hpp"
#include "EulerIvpOdeSolver.hpp"
#include "Exception.hpp"
#include "GRL1IvpOdeSolver.hpp"
#include "GRL2IvpOdeSolver.hpp"
#include "HeartConfig.hpp"
#include "MonodomainProblem.hpp"
#include "MonodomainTissue.hpp"
#include "RegularStimulus.hpp"
#include "SimpleStimulus.hpp"
#include "ZeroStimulus.hpp"
#include "chaste_gpu.h"

namespace chaste_gpu_shim
{

inline void Check(int status, const std::string& rWhere)
{
    if (status != CG_OK)
    {
        EXCEPTION(rWhere + ": " + cg_status_string(status));
    }
}

/*
 * An archive for a stimulus class's own serialize(): it keeps the doubles the class
 * passes (SimpleStimulus archives mMagnitudeOfStimulus, mDuration, mTimeOfStimulus in
 * that order, heart/src/stimulus/SimpleStimulus.hpp:59-66) and ignores the rest.
 */
struct DoubleCapture
{
    std::vector<double> mValues;
    template <class T>
    DoubleCapture& operator&(T& rValue)
    {
        Take(rValue);
        return *this;
    }
    template <class T>
    DoubleCapture& operator&(const T& rValue)
    {
        return *this;
    }
    void Take(double& rValue)
    {
        mValues.push_back(rValue);
    }
    template <class T>
    void Take(T&)
    {
    }
};

/* The cg_stimulus equivalent of a cell's stimulus function. */
inline cg_stimulus Describe(const boost::shared_ptr<AbstractStimulusFunction>& rpStim)
{
    cg_stimulus s = {CG_STIM_NONE, 0.0, 0.0, 0.0, 0.0, 0.0};
    AbstractStimulusFunction* p = rpStim.get();
    if (p == nullptr || dynamic_cast<ZeroStimulus*>(p) != nullptr)
    {
        return s;
    }
    if (RegularStimulus* p_reg = dynamic_cast<RegularStimulus*>(p))
    {
        s.kind = CG_STIM_REGULAR;
        s.magnitude = p_reg->GetMagnitude();
        s.duration = p_reg->GetDuration();
        s.start = p_reg->GetStartTime();
        s.period = p_reg->GetPeriod();
        s.stop = p_reg->GetStopTime();
        return s;
    }
    if (SimpleStimulus* p_simple = dynamic_cast<SimpleStimulus*>(p))
    {
        DoubleCapture capture;
        boost::serialization::access::serialize(capture, *p_simple, 0u);
        if (capture.mValues.size() != 3u)
        {
            EXCEPTION("SimpleStimulus did not archive its three parameters");
        }
        s.kind = CG_STIM_SIMPLE;
        s.magnitude = capture.mValues[0];
        s.duration = capture.mValues[1];
        s.start = capture.mValues[2];
        return s;
    }
    EXCEPTION("the GPU tissue takes ZeroStimulus, SimpleStimulus and RegularStimulus cells only");
}

/* Model and ODE method of a cell (the two generated models libchastegpu carries).
 * Rush-Larsen cells derive from AbstractRushLarsenCardiacCell; backward-Euler cells
 * (AbstractBackwardEulerCardiacCell) are built without an ODE solver; the others are
 * told apart by theirs. */
inline void ModelOf(AbstractCardiacCellInterface* pCell, int& rModel, int& rMethod)
{
    AbstractUntemplatedParameterisedSystem* p_system = dynamic_cast<AbstractUntemplatedParameterisedSystem*>(pCell);
    if (p_system == nullptr)
    {
        EXCEPTION("cell without a system name");
    }
    const std::string name = p_system->GetSystemName();
    if (name == "luo_rudy_1991")
    {
        rModel = CG_MODEL_LR91;
    }
    else if (name == "tentusscher_model_2006_epi")
    {
        rModel = CG_MODEL_TT06;
    }
    else
    {
        EXCEPTION("no GPU cell model for " + name);
    }
    const AbstractIvpOdeSolver* p_solver = pCell->GetSolver().get();
    if (dynamic_cast<AbstractRushLarsenCardiacCell*>(pCell) != nullptr)
    {
        rMethod = CG_ODE_RUSH_LARSEN;
    }
    else if (p_solver == nullptr)
    {
        rMethod = CG_ODE_BACKWARD_EULER;
    }
    else if (dynamic_cast<const GRL1IvpOdeSolver*>(p_solver) != nullptr)
    {
        rMethod = CG_ODE_GRL1;
    }
    else if (dynamic_cast<const GRL2IvpOdeSolver*>(p_solver) != nullptr)
    {
        rMethod = CG_ODE_GRL2;
    }
    else if (dynamic_cast<const EulerIvpOdeSolver*>(p_solver) != nullptr)
    {
        rMethod = CG_ODE_FORWARD_EULER;
    }
    else
    {
        EXCEPTION("the GPU tissue integrates cells by forward Euler, Rush-Larsen, backward Euler, GRL1 or GRL2");
    }
}

/*
 * The modifiable parameters of the reference's generated cells, as scale factors
 * of the GPU models' parameter vector: (Chaste parameter name, index, value the
 * scale is relative to).  LuoRudy1991.cellml:313, 817, 1118 (annotations
 * :2066-2088); TenTusscher2006Epi.cellml:3697-3705.
 */
struct ParameterLink
{
    const char* mName;
    int mIndex;
    double mReference;
};
inline const std::vector<ParameterLink>& ParameterLinks(int model)
{
    static const std::vector<ParameterLink> lr91 = {
        {"membrane_fast_sodium_current_conductance", 0, 23.0},
        {"membrane_L_type_calcium_current_conductance", 1, 0.09},
        {"membrane_rapid_delayed_rectifier_potassium_current_conductance", 2, 0.282}};
    static const std::vector<ParameterLink> tt06 = {
        {"ScaleFactorGks", 6, 1.0}, {"ScaleFactorGkr", 7, 1.0}, {"ScaleFactorIto", 8, 1.0}};
    return model == CG_MODEL_LR91 ? lr91 : tt06;
}

/* HeartConfig -> cg_config (heart/src/problem/HeartConfig.cpp:1581-1650, 2337-2412). */
inline cg_config ConfigFromHeartConfig(int model, int method)
{
    HeartConfig* p_config = HeartConfig::Instance();
    cg_config cfg;
    cg_default_config(&cfg);
    cfg.model = model;
    cfg.ode_method = method;
    cfg.ode_time_step = p_config->GetOdeTimeStep();
    cfg.pde_time_step = p_config->GetPdeTimeStep();
    cfg.surface_area_to_volume_ratio = p_config->GetSurfaceAreaToVolumeRatio();
    cfg.capacitance = p_config->GetCapacitance();
    cfg.use_absolute_tolerance = p_config->GetUseAbsoluteTolerance() ? 1 : 0;
    cfg.ksp_tolerance = p_config->GetUseAbsoluteTolerance() ? p_config->GetAbsoluteTolerance()
                                                            : p_config->GetRelativeTolerance();
    const std::string pc = p_config->GetKSPPreconditioner();
    if (pc == "bjacobi")
    {
        cfg.ksp_preconditioner = CG_PC_BJACOBI;
    }
    else if (pc == "jacobi")
    {
        cfg.ksp_preconditioner = CG_PC_JACOBI;
    }
    else if (pc == "none")
    {
        cfg.ksp_preconditioner = CG_PC_NONE;
    }
    else
    {
        EXCEPTION("the GPU tissue supports the bjacobi, jacobi and none preconditioners, not " + pc);
    }
    if (std::string(p_config->GetKSPSolver()) != "cg")
    {
        EXCEPTION("the GPU tissue solves with CG (the monodomain matrix is SPD)");
    }
    cfg.use_mass_lumping = p_config->GetUseMassLumping() ? 1 : 0;
    cfg.solver = p_config->GetUseReactionDiffusionOperatorSplitting() ? CG_SOLVER_OPERATOR_SPLITTING
                                                                      : CG_SOLVER_MONODOMAIN;
    cfg.use_state_variable_interpolation = p_config->GetUseStateVariableInterpolation() ? 1 : 0;
    return cfg;
}

}  // namespace chaste_gpu_shim

/*
 * The tissue: Chaste's MonodomainTissue (its cells, conductivity tensors and caches
 * stay the host view) plus the device tissue that steps them.
 */
template <unsigned DIM>
class GpuMonodomainTissue : public MonodomainTissue<DIM>
{
private:
    cg_ctx* mpCtx;
    unsigned mNumStates;

public:
    // MonodomainTissue derives virtually from AbstractCardiacTissue, so the most
    // derived class constructs that base itself
    explicit GpuMonodomainTissue(AbstractCardiacCellFactory<DIM>* pCellFactory)
        : AbstractCardiacTissue<DIM>(pCellFactory),
          MonodomainTissue<DIM>(pCellFactory),
          mpCtx(nullptr),
          mNumStates(0u)
    {
    }

    ~GpuMonodomainTissue()
    {
        if (mpCtx != nullptr)
        {
            cg_destroy(mpCtx);
        }
    }

    cg_ctx* GetContext()
    {
        return mpCtx;
    }

    /* Builds the device tissue from this tissue's mesh, cells and stimuli. */
    void Upload()
    {
        using namespace chaste_gpu_shim;
        AbstractTetrahedralMesh<DIM, DIM>* p_mesh = this->mpMesh;
        const unsigned n = p_mesh->GetNumNodes();
        int model = -1, method = -1;
        ModelOf(this->GetCardiacCell(0), model, method);
        cg_config cfg = ConfigFromHeartConfig(model, method);
        Check(cg_create(&cfg, &mpCtx), "cg_create");

        // mesh and conductivities
        HeartConfig* p_config = HeartConfig::Instance();
        std::vector<double> sigma_elem;
        const unsigned n_elem = p_mesh->GetNumElements();
        sigma_elem.reserve((size_t)n_elem * DIM);
        for (unsigned e = 0; e < n_elem; ++e)
        {
            const c_matrix<double, DIM, DIM>& r_sigma = this->rGetIntracellularConductivityTensor(e);
            for (unsigned a = 0; a < DIM; ++a)
            {
                for (unsigned b = 0; b < DIM; ++b)
                {
                    if (a != b && r_sigma(a, b) != 0.0)
                    {
                        EXCEPTION("the GPU tissue takes axis-aligned (diagonal) conductivity tensors");
                    }
                }
                sigma_elem.push_back(r_sigma(a, a));
            }
        }
        bool uniform = true;
        for (size_t k = DIM; k < sigma_elem.size() && uniform; ++k)
        {
            uniform = sigma_elem[k] == sigma_elem[k % DIM];
        }
        if (p_config->GetCreateSlab() && uniform)
        {
            c_vector<double, 3> dims;
            p_config->GetSlabDimensions(dims);
            int n_nodes = 0;
            Check(cg_set_slab_mesh(mpCtx, (int)DIM, p_config->GetInterNodeSpace(), dims[0], DIM > 1 ? dims[1] : 0.0,
                                   DIM > 2 ? dims[2] : 0.0, sigma_elem.data(), &n_nodes),
                  "cg_set_slab_mesh");
            if ((unsigned)n_nodes != n)
            {
                EXCEPTION("slab node count differs from the mesh");
            }
        }
        else
        {
            std::vector<double> xyz((size_t)n * 3, 0.0);
            for (unsigned i = 0; i < n; ++i)
            {
                const c_vector<double, DIM>& r_x = p_mesh->GetNode(i)->rGetLocation();
                for (unsigned a = 0; a < DIM; ++a)
                {
                    xyz[(size_t)i * 3 + a] = r_x[a];
                }
            }
            std::vector<int> conn;
            conn.reserve((size_t)n_elem * (DIM + 1));
            for (unsigned e = 0; e < n_elem; ++e)
            {
                Element<DIM, DIM>* p_element = p_mesh->GetElement(e);
                for (unsigned j = 0; j < DIM + 1; ++j)
                {
                    conn.push_back((int)p_element->GetNodeGlobalIndex(j));
                }
            }
            Check(cg_set_mesh(mpCtx, (int)n, (int)DIM, xyz.data(), (int)n_elem, conn.data(), sigma_elem.data()),
                  "cg_set_mesh");
        }

        // cells: states (AoS), parameter sets, stimuli
        int n_states = 0, n_params = 0;
        Check(cg_num_states(model, &n_states), "cg_num_states");
        Check(cg_num_params(model, &n_params), "cg_num_params");
        mNumStates = (unsigned)n_states;
        std::vector<double> states((size_t)n * n_states);
        std::vector<int> param_set(n), stim_id(n);
        std::vector<std::vector<double> > sets;
        std::vector<cg_stimulus> stims;
        for (unsigned i = 0; i < n; ++i)
        {
            AbstractCardiacCellInterface* p_cell = this->GetCardiacCell(i);
            int m = -1, meth = -1;
            ModelOf(p_cell, m, meth);
            if (m != model || meth != method)
            {
                EXCEPTION("the GPU tissue runs one cell model and ODE method on every node");
            }
            const std::vector<double> y = p_cell->GetStdVecStateVariables();
            if (y.size() != (size_t)n_states)
            {
                EXCEPTION("cell state vector of unexpected length");
            }
            std::copy(y.begin(), y.end(), states.begin() + (size_t)i * n_states);
            std::vector<double> row(n_params, 1.0);
            for (const ParameterLink& r_link : ParameterLinks(model))
            {
                row[r_link.mIndex] = p_cell->GetParameter(r_link.mName) / r_link.mReference;
            }
            size_t k = 0;
            while (k < sets.size() && sets[k] != row)
            {
                ++k;
            }
            if (k == sets.size())
            {
                sets.push_back(row);
            }
            param_set[i] = (int)k;
            const cg_stimulus s = Describe(p_cell->GetStimulusFunction());
            if (s.kind == CG_STIM_NONE)
            {
                stim_id[i] = -1;
                continue;
            }
            size_t q = 0;
            while (q < stims.size()
                   && !(stims[q].kind == s.kind && stims[q].magnitude == s.magnitude && stims[q].duration == s.duration
                        && stims[q].start == s.start && stims[q].period == s.period && stims[q].stop == s.stop))
            {
                ++q;
            }
            if (q == stims.size())
            {
                stims.push_back(s);
            }
            stim_id[i] = (int)q;
        }
        if (sets.size() > 255u || stims.size() > 255u)
        {
            EXCEPTION("more than 255 distinct parameter sets or stimuli");
        }
        std::vector<double> table;
        for (const std::vector<double>& r_row : sets)
        {
            table.insert(table.end(), r_row.begin(), r_row.end());
        }
        Check(cg_set_cells(mpCtx, states.data(), param_set.data(), table.data(), (int)sets.size()), "cg_set_cells");
        Check(cg_set_stimulus(mpCtx, stim_id.data(), stims.data(), (int)stims.size()), "cg_set_stimulus");
    }

    /* The ODE update runs inside the device step (GpuMonodomainSolver). */
    void SolveCellSystems(Vec existingSolution, double time, double nextTime, bool updateVoltage = false)
    {
    }

    /* GetCardiacCell(i) and the Iion cache from the device (a device -> host copy). */
    void SyncCellsFromDevice()
    {
        using namespace chaste_gpu_shim;
        const unsigned n = this->mpMesh->GetNumNodes();
        std::vector<double> states((size_t)n * mNumStates);
        Check(cg_get_states(mpCtx, states.data()), "cg_get_states");
        for (unsigned i = 0; i < n; ++i)
        {
            std::vector<double> y(states.begin() + (size_t)i * mNumStates,
                                  states.begin() + (size_t)(i + 1) * mNumStates);
            this->GetCardiacCell(i)->SetStateVariables(y);
        }
        std::vector<double> iion(n), istim(n);
        Check(cg_get_caches(mpCtx, iion.data(), istim.data()), "cg_get_caches");
        ReplicatableVector& r_iion = this->rGetIionicCacheReplicated();
        ReplicatableVector& r_istim = this->rGetIntracellularStimulusCacheReplicated();
        for (unsigned i = 0; i < n; ++i)
        {
            r_iion[i] = iion[i];
            r_istim[i] = istim[i];
        }
    }
};

/*
 * The solver: Chaste's dynamic linear PDE loop with the device doing each step.
 */
template <unsigned DIM>
class GpuMonodomainSolver : public AbstractDynamicLinearPdeSolver<DIM, DIM, 1>
{
private:
    GpuMonodomainTissue<DIM>* mpTissue;
    std::vector<double> mHostV;

public:
    GpuMonodomainSolver(AbstractTetrahedralMesh<DIM, DIM>* pMesh, GpuMonodomainTissue<DIM>* pTissue)
        : AbstractDynamicLinearPdeSolver<DIM, DIM, 1>(pMesh),
          mpTissue(pTissue)
    {
        this->mMatrixIsConstant = true;
    }

    /* AbstractLinearPdeSolver::InitialiseForSolve, then an identity system (set once)
     * and the initial condition on the device. */
    void InitialiseForSolve(Vec initialSolution = nullptr)
    {
        using namespace chaste_gpu_shim;
        const bool first = (this->mpLinearSystem == nullptr);
        AbstractDynamicLinearPdeSolver<DIM, DIM, 1>::InitialiseForSolve(initialSolution);
        if (first)
        {
            PetscInt lo, hi;
            this->mpLinearSystem->GetOwnershipRange(lo, hi);
            for (PetscInt i = lo; i < hi; ++i)
            {
                this->mpLinearSystem->SetMatrixElement(i, i, 1.0);
            }
            this->mpLinearSystem->AssembleFinalLhsMatrix();
            this->mpLinearSystem->SetMatrixIsConstant(true);
        }
        if (initialSolution != nullptr)
        {
            ReplicatableVector v0(initialSolution);
            mHostV.assign(v0.GetSize(), 0.0);
            for (unsigned i = 0; i < v0.GetSize(); ++i)
            {
                mHostV[i] = v0[i];
            }
            Check(cg_set_voltage(mpTissue->GetContext(), mHostV.data()), "cg_set_voltage");
        }
    }

    /* The whole monodomain step on the device (ODEs, b = M z, CG) and the new V copied
     * back, one call and one synchronisation. */
    void PrepareForSetupLinearSystem(Vec currentSolution)
    {
        mHostV.resize(this->mpMesh->GetNumNodes());
        chaste_gpu_shim::Check(cg_step_host(mpTissue->GetContext(), nullptr, 1, mHostV.data(), 1), "cg_step_host");
    }

    /* b = the device solution; the identity system returns it as the next solution. */
    void SetupLinearSystem(Vec currentSolution, bool computeMatrix)
    {
        using namespace chaste_gpu_shim;
        PetscInt lo, hi;
        this->mpLinearSystem->GetOwnershipRange(lo, hi);
        for (PetscInt i = lo; i < hi; ++i)
        {
            this->mpLinearSystem->SetRhsVectorElement(i, mHostV[i]);
        }
        this->mpLinearSystem->AssembleRhsVector();
    }
};

template <unsigned DIM>
class GpuMonodomainProblem : public MonodomainProblem<DIM>
{
private:
    GpuMonodomainTissue<DIM>* mpGpuTissue;
    bool mSyncAtPrintingTimes;

protected:
    AbstractCardiacTissue<DIM>* CreateCardiacTissue()
    {
        mpGpuTissue = new GpuMonodomainTissue<DIM>(this->mpCellFactory);
        this->mpMonodomainTissue = mpGpuTissue;
        mpGpuTissue->Upload();
        return mpGpuTissue;
    }

    AbstractDynamicLinearPdeSolver<DIM, DIM, 1>* CreateSolver()
    {
        return new GpuMonodomainSolver<DIM>(this->mpMesh, mpGpuTissue);
    }

    void OnEndOfTimestep(double time)
    {
        if (mSyncAtPrintingTimes)
        {
            mpGpuTissue->SyncCellsFromDevice();
        }
    }

public:
    explicit GpuMonodomainProblem(AbstractCardiacCellFactory<DIM>* pCellFactory)
        : MonodomainProblem<DIM>(pCellFactory),
          mpGpuTissue(nullptr),
          mSyncAtPrintingTimes(false)
    {
    }

    /* Copy the device cells into GetCardiacCell(i) at every printing time (off by default). */
    void SetSyncCellsAtPrintingTimes(bool sync)
    {
        mSyncAtPrintingTimes = sync;
    }

    /* The device cells into GetCardiacCell(i) now (e.g. after Solve()). */
    void SyncCellsFromDevice()
    {
        mpGpuTissue->SyncCellsFromDevice();
    }

    GpuMonodomainTissue<DIM>* GetGpuTissue()
    {
        return mpGpuTissue;
    }
};

#endif  // GPUMONODOMAINPROBLEM_HPP_

// Test stand-ins for the Chaste classes the GPU binding
// (chaste_b200/shim/GpuMonodomainProblem.hpp) uses, with the same names, members
// and call sequence as the reference: AbstractCardiacProblem::Solve's printing loop
// (heart/src/problem/AbstractCardiacProblem.cpp:412-620, reduced to its calls),
// AbstractDynamicLinearPdeSolver::Solve's step loop with its hooks
// (pde/src/solver/AbstractDynamicLinearPdeSolver.hpp:328-497), MonodomainProblem's
// CreateCardiacTissue / CreateSolver (heart/src/problem/MonodomainProblem.cpp:45-77),
// the tissue's cells built by the factory, SimpleStimulus's private members and
// serialize(), RegularStimulus's getters.  Only what the binding touches is here;
// PETSc vectors are plain host arrays and the linear system is diagonal.
#pragma once

#include <cmath>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

class Exception : public std::runtime_error
{
public:
    explicit Exception(const std::string& rMessage) : std::runtime_error(rMessage) {}
    std::string GetMessage() const { return what(); }
};
#define EXCEPTION(message)                \
    do                                    \
    {                                     \
        std::ostringstream msg_;          \
        msg_ << message;                  \
        throw Exception(msg_.str());      \
    } while (false)

namespace boost
{
using std::shared_ptr;
namespace serialization
{
class access
{
public:
    template <class Archive, class T>
    static void serialize(Archive& rArchive, T& rObject, const unsigned int version)
    {
        rObject.serialize(rArchive, version);
    }
};
template <class Base, class Derived>
Base& base_object(Derived& rDerived)
{
    return rDerived;
}
}  // namespace serialization
}  // namespace boost

template <class T, unsigned N>
struct c_vector
{
    T mData[N] = {};
    T& operator[](unsigned i) { return mData[i]; }
    const T& operator[](unsigned i) const { return mData[i]; }
};
template <class T, unsigned R, unsigned C>
struct c_matrix
{
    T mData[R][C] = {};
    T& operator()(unsigned i, unsigned j) { return mData[i][j]; }
    const T& operator()(unsigned i, unsigned j) const { return mData[i][j]; }
};

typedef int PetscInt;
struct StubVec
{
    std::vector<double> mValues;
};
typedef StubVec* Vec;

class ReplicatableVector
{
    std::vector<double> mValues;
public:
    ReplicatableVector() {}
    explicit ReplicatableVector(Vec v) : mValues(v->mValues) {}
    void Resize(unsigned n) { mValues.assign(n, 0.0); }
    unsigned GetSize() const { return (unsigned)mValues.size(); }
    double& operator[](unsigned i) { return mValues[i]; }
};

// Diagonal systems only (the binding's identity); counts its solves.
class LinearSystem
{
    std::vector<double> mDiag, mRhs;
    bool mOffDiagonal = false;
public:
    int mSolves = 0;
    explicit LinearSystem(unsigned n) : mDiag(n, 0.0), mRhs(n, 0.0) {}
    void GetOwnershipRange(PetscInt& lo, PetscInt& hi) { lo = 0; hi = (PetscInt)mDiag.size(); }
    void SetMatrixElement(PetscInt i, PetscInt j, double v) { if (i == j) mDiag[i] = v; else mOffDiagonal = true; }
    void AssembleFinalLhsMatrix() {}
    void SetMatrixIsConstant(bool) {}
    void SetRhsVectorElement(PetscInt i, double v) { mRhs[i] = v; }
    void AssembleRhsVector() {}
    void ResetKspSolver() {}
    Vec Solve(Vec)
    {
        if (mOffDiagonal) EXCEPTION("stub linear system is diagonal only");
        Vec x = new StubVec;
        x->mValues.resize(mDiag.size());
        for (size_t i = 0; i < mDiag.size(); ++i) x->mValues[i] = mRhs[i] / mDiag[i];
        mSolves++;
        return x;
    }
};

class AbstractStimulusFunction
{
public:
    virtual ~AbstractStimulusFunction() {}
    virtual double GetStimulus(double time) = 0;
};
class ZeroStimulus : public AbstractStimulusFunction
{
public:
    double GetStimulus(double) { return 0.0; }
};
class SimpleStimulus : public AbstractStimulusFunction
{
    friend class boost::serialization::access;
    template <class Archive>
    void serialize(Archive& archive, const unsigned int version)
    {
        archive & boost::serialization::base_object<AbstractStimulusFunction>(*this);
        archive & mMagnitudeOfStimulus;
        archive & mDuration;
        archive & mTimeOfStimulus;
    }
private:
    double mMagnitudeOfStimulus;
    double mDuration;
    double mTimeOfStimulus;
public:
    SimpleStimulus(double magnitude, double duration, double start = 0.0)
        : mMagnitudeOfStimulus(magnitude), mDuration(duration), mTimeOfStimulus(start) {}
    double GetStimulus(double t)
    {
        return (mTimeOfStimulus <= t && t <= mDuration + mTimeOfStimulus) ? mMagnitudeOfStimulus : 0.0;
    }
};
class RegularStimulus : public AbstractStimulusFunction
{
    double mMagnitude, mDuration, mPeriod, mStart, mStop;
public:
    RegularStimulus(double magnitude, double duration, double period, double start, double stop = 1e300)
        : mMagnitude(magnitude), mDuration(duration), mPeriod(period), mStart(start), mStop(stop) {}
    double GetStimulus(double) { return 0.0; }
    double GetPeriod() { return mPeriod; }
    double GetMagnitude() { return mMagnitude; }
    double GetDuration() { return mDuration; }
    double GetStartTime() { return mStart; }
    double GetStopTime() { return mStop; }
};

class AbstractIvpOdeSolver
{
public:
    virtual ~AbstractIvpOdeSolver() {}
};
class EulerIvpOdeSolver : public AbstractIvpOdeSolver {};
class GRL1IvpOdeSolver : public AbstractIvpOdeSolver {};
class GRL2IvpOdeSolver : public AbstractIvpOdeSolver {};

class AbstractUntemplatedParameterisedSystem
{
protected:
    std::string mSystemName;
public:
    virtual ~AbstractUntemplatedParameterisedSystem() {}
    std::string GetSystemName() const { return mSystemName; }
};

class AbstractCardiacCellInterface
{
protected:
    boost::shared_ptr<AbstractIvpOdeSolver> mpOdeSolver;
    boost::shared_ptr<AbstractStimulusFunction> mpIntracellularStimulus;
public:
    AbstractCardiacCellInterface(boost::shared_ptr<AbstractIvpOdeSolver> pSolver,
                                 boost::shared_ptr<AbstractStimulusFunction> pStim)
        : mpOdeSolver(pSolver), mpIntracellularStimulus(pStim) {}
    virtual ~AbstractCardiacCellInterface() {}
    virtual std::vector<double> GetStdVecStateVariables() = 0;
    virtual void SetStateVariables(const std::vector<double>& rVariables) = 0;
    virtual double GetParameter(const std::string& rParameterName) = 0;
    boost::shared_ptr<AbstractStimulusFunction> GetStimulusFunction() { return mpIntracellularStimulus; }
    const boost::shared_ptr<AbstractIvpOdeSolver> GetSolver() const { return mpOdeSolver; }
};

class AbstractCardiacCell : public AbstractCardiacCellInterface, public AbstractUntemplatedParameterisedSystem
{
protected:
    std::vector<double> mStateVariables;
    std::map<std::string, double> mParameters;
public:
    AbstractCardiacCell(boost::shared_ptr<AbstractIvpOdeSolver> pSolver, boost::shared_ptr<AbstractStimulusFunction> pStim)
        : AbstractCardiacCellInterface(pSolver, pStim) {}
    std::vector<double> GetStdVecStateVariables() { return mStateVariables; }
    void SetStateVariables(const std::vector<double>& rVariables) { mStateVariables = rVariables; }
    double GetParameter(const std::string& rName)
    {
        std::map<std::string, double>::iterator it = mParameters.find(rName);
        if (it == mParameters.end()) EXCEPTION("no parameter " << rName);
        return it->second;
    }
    void SetParameter(const std::string& rName, double v) { mParameters[rName] = v; }
};
class AbstractRushLarsenCardiacCell : public AbstractCardiacCell
{
public:
    using AbstractCardiacCell::AbstractCardiacCell;
};

template <unsigned DIM>
class Node
{
    c_vector<double, DIM> mLocation;
public:
    explicit Node(const c_vector<double, DIM>& rX) : mLocation(rX) {}
    const c_vector<double, DIM>& rGetLocation() const { return mLocation; }
};
template <unsigned ELEMENT_DIM, unsigned SPACE_DIM>
class Element
{
    unsigned mNodes[ELEMENT_DIM + 1];
public:
    explicit Element(const unsigned* pNodes) { for (unsigned j = 0; j <= ELEMENT_DIM; ++j) mNodes[j] = pNodes[j]; }
    unsigned GetNodeGlobalIndex(unsigned j) const { return mNodes[j]; }
};
template <unsigned ELEMENT_DIM, unsigned SPACE_DIM = ELEMENT_DIM>
class AbstractTetrahedralMesh
{
    std::vector<Node<SPACE_DIM>*> mNodes;
    std::vector<Element<ELEMENT_DIM, SPACE_DIM>*> mElements;
public:
    ~AbstractTetrahedralMesh()
    {
        for (size_t i = 0; i < mNodes.size(); ++i) delete mNodes[i];
        for (size_t i = 0; i < mElements.size(); ++i) delete mElements[i];
    }
    // ConstructRegularSlabMesh in 1D (mesh/src/common/AbstractTetrahedralMesh.cpp:569-614)
    void ConstructRegularSlabMesh(double h, double width)
    {
        const unsigned nx = (unsigned)(width / h + 0.5);
        for (unsigned i = 0; i <= nx; ++i)
        {
            c_vector<double, SPACE_DIM> x;
            x[0] = i * h;
            mNodes.push_back(new Node<SPACE_DIM>(x));
        }
        for (unsigned e = 0; e < nx; ++e)
        {
            const unsigned v[2] = {e, e + 1};
            mElements.push_back(new Element<ELEMENT_DIM, SPACE_DIM>(v));
        }
    }
    unsigned GetNumNodes() const { return (unsigned)mNodes.size(); }
    unsigned GetNumElements() const { return (unsigned)mElements.size(); }
    Node<SPACE_DIM>* GetNode(unsigned i) { return mNodes[i]; }
    Element<ELEMENT_DIM, SPACE_DIM>* GetElement(unsigned e) { return mElements[e]; }
};

template <unsigned ELEMENT_DIM, unsigned SPACE_DIM = ELEMENT_DIM>
class AbstractCardiacCellFactory
{
protected:
    AbstractTetrahedralMesh<ELEMENT_DIM, SPACE_DIM>* mpMesh = nullptr;
public:
    virtual ~AbstractCardiacCellFactory() {}
    virtual AbstractCardiacCellInterface* CreateCardiacCellForTissueNode(Node<SPACE_DIM>* pNode) = 0;
    void SetMesh(AbstractTetrahedralMesh<ELEMENT_DIM, SPACE_DIM>* pMesh) { mpMesh = pMesh; }
    AbstractTetrahedralMesh<ELEMENT_DIM, SPACE_DIM>* GetMesh() { return mpMesh; }
};

class HeartConfig
{
    double mOdeDt = 0.01, mPdeDt = 0.01, mPrintingDt = 0.01, mEnd = 10.0;
    double mAm = 1400.0, mCm = 1.0, mTol = 2e-4;
    bool mAbsolute = true, mLumping = false, mSplitting = false, mSvi = false, mSlab = true;
    std::string mPc = "bjacobi";
    double mH = 0.01;
    c_vector<double, 3> mSlabDims;
    c_vector<double, 3> mSigma;
public:
    static HeartConfig* Instance() { static HeartConfig c; return &c; }
    void SetOdePdeAndPrintingTimeSteps(double o, double p, double pr) { mOdeDt = o; mPdeDt = p; mPrintingDt = pr; }
    void SetSimulationDuration(double t) { mEnd = t; }
    void SetUseAbsoluteTolerance(double t) { mAbsolute = true; mTol = t; }
    void SetUseRelativeTolerance(double t) { mAbsolute = false; mTol = t; }
    void SetKSPPreconditioner(const char* pc) { mPc = pc; }
    void SetIntracellularConductivities(double s) { mSigma[0] = mSigma[1] = mSigma[2] = s; }
    void SetFibreLength(double length, double h) { mSlabDims[0] = length; mH = h; mSlab = true; }
    void SetCreateSlab(bool flag) { mSlab = flag; }
    double GetOdeTimeStep() const { return mOdeDt; }
    double GetPdeTimeStep() const { return mPdeDt; }
    double GetPrintingTimeStep() const { return mPrintingDt; }
    double GetSimulationDuration() const { return mEnd; }
    double GetSurfaceAreaToVolumeRatio() const { return mAm; }
    double GetCapacitance() const { return mCm; }
    bool GetUseAbsoluteTolerance() const { return mAbsolute; }
    double GetAbsoluteTolerance() const { return mTol; }
    double GetRelativeTolerance() const { return mTol; }
    const char* GetKSPSolver() const { return "cg"; }
    const char* GetKSPPreconditioner() const { return mPc.c_str(); }
    bool GetUseMassLumping() { return mLumping; }
    bool GetUseReactionDiffusionOperatorSplitting() { return mSplitting; }
    bool GetUseStateVariableInterpolation() const { return mSvi; }
    bool GetCreateSlab() const { return mSlab; }
    void GetSlabDimensions(c_vector<double, 3>& rDims) const { rDims = mSlabDims; }
    double GetInterNodeSpace() const { return mH; }
    double GetSigma() const { return mSigma[0]; }
};

template <unsigned ELEMENT_DIM, unsigned SPACE_DIM = ELEMENT_DIM>
class AbstractCardiacTissue
{
protected:
    AbstractTetrahedralMesh<ELEMENT_DIM, SPACE_DIM>* mpMesh;
    std::vector<AbstractCardiacCellInterface*> mCellsDistributed;
    ReplicatableVector mIionicCacheReplicated, mIntracellularStimulusCacheReplicated;
    c_matrix<double, SPACE_DIM, SPACE_DIM> mSigma;
public:
    explicit AbstractCardiacTissue(AbstractCardiacCellFactory<ELEMENT_DIM, SPACE_DIM>* pFactory,
                                   bool exchangeHalos = false)
        : mpMesh(pFactory->GetMesh())
    {
        for (unsigned i = 0; i < mpMesh->GetNumNodes(); ++i)
            mCellsDistributed.push_back(pFactory->CreateCardiacCellForTissueNode(mpMesh->GetNode(i)));
        mIionicCacheReplicated.Resize(mpMesh->GetNumNodes());
        mIntracellularStimulusCacheReplicated.Resize(mpMesh->GetNumNodes());
        for (unsigned a = 0; a < SPACE_DIM; ++a) mSigma(a, a) = HeartConfig::Instance()->GetSigma();
    }
    virtual ~AbstractCardiacTissue()
    {
        for (size_t i = 0; i < mCellsDistributed.size(); ++i) delete mCellsDistributed[i];
    }
    AbstractCardiacCellInterface* GetCardiacCell(unsigned globalIndex) { return mCellsDistributed[globalIndex]; }
    const c_matrix<double, SPACE_DIM, SPACE_DIM>& rGetIntracellularConductivityTensor(unsigned) { return mSigma; }
    virtual void SolveCellSystems(Vec existingSolution, double time, double nextTime, bool updateVoltage = false)
    {
        EXCEPTION("the stub tissue integrates no cells on the host");
    }
    ReplicatableVector& rGetIionicCacheReplicated() { return mIionicCacheReplicated; }
    ReplicatableVector& rGetIntracellularStimulusCacheReplicated() { return mIntracellularStimulusCacheReplicated; }
};

template <unsigned ELEMENT_DIM, unsigned SPACE_DIM = ELEMENT_DIM>
class MonodomainTissue : public virtual AbstractCardiacTissue<ELEMENT_DIM, SPACE_DIM>
{
public:
    explicit MonodomainTissue(AbstractCardiacCellFactory<ELEMENT_DIM, SPACE_DIM>* pFactory, bool exchangeHalos = false)
        : AbstractCardiacTissue<ELEMENT_DIM, SPACE_DIM>(pFactory, exchangeHalos) {}
};

template <unsigned ELEMENT_DIM, unsigned SPACE_DIM, unsigned PROBLEM_DIM>
class AbstractDynamicLinearPdeSolver
{
protected:
    AbstractTetrahedralMesh<ELEMENT_DIM, SPACE_DIM>* mpMesh;
    LinearSystem* mpLinearSystem = nullptr;
    bool mMatrixIsConstant = false;
    double mTstart = 0.0, mTend = 0.0, mIdealTimeStep = -1.0;
    Vec mInitialCondition = nullptr;
public:
    explicit AbstractDynamicLinearPdeSolver(AbstractTetrahedralMesh<ELEMENT_DIM, SPACE_DIM>* pMesh) : mpMesh(pMesh) {}
    virtual ~AbstractDynamicLinearPdeSolver() { delete mpLinearSystem; }
    virtual void InitialiseForSolve(Vec initialSolution = nullptr)
    {
        if (mpLinearSystem == nullptr) mpLinearSystem = new LinearSystem(mpMesh->GetNumNodes());
    }
    virtual void PrepareForSetupLinearSystem(Vec currentSolution) {}
    virtual void FinaliseLinearSystem(Vec currentSolution) {}
    virtual void FollowingSolveLinearSystem(Vec currentSolution) {}
    virtual void SetupLinearSystem(Vec currentSolution, bool computeMatrix) = 0;
    LinearSystem* GetLinearSystem() { return mpLinearSystem; }
    void SetTimes(double t0, double t1) { mTstart = t0; mTend = t1; }
    void SetTimeStep(double dt) { mIdealTimeStep = dt; }
    void SetInitialCondition(Vec v) { mInitialCondition = v; }
    // the step loop of AbstractDynamicLinearPdeSolver::Solve with a fixed step
    Vec Solve()
    {
        InitialiseForSolve(mInitialCondition);
        const unsigned n_steps = (unsigned)((mTend - mTstart) / mIdealTimeStep + 0.5);
        Vec solution = mInitialCondition;
        for (unsigned k = 0; k < n_steps; ++k)
        {
            PrepareForSetupLinearSystem(solution);
            SetupLinearSystem(solution, k == 0);
            FinaliseLinearSystem(solution);
            Vec next = mpLinearSystem->Solve(solution);
            FollowingSolveLinearSystem(next);
            if (solution != mInitialCondition) delete solution;
            solution = next;
        }
        return solution;
    }
};

template <unsigned ELEMENT_DIM, unsigned SPACE_DIM = ELEMENT_DIM>
class MonodomainProblem
{
protected:
    AbstractCardiacCellFactory<ELEMENT_DIM, SPACE_DIM>* mpCellFactory;
    AbstractTetrahedralMesh<ELEMENT_DIM, SPACE_DIM>* mpMesh = nullptr;
    MonodomainTissue<ELEMENT_DIM, SPACE_DIM>* mpMonodomainTissue = nullptr;
    AbstractCardiacTissue<ELEMENT_DIM, SPACE_DIM>* mpCardiacTissue = nullptr;
    Vec mSolution = nullptr;
    virtual AbstractCardiacTissue<ELEMENT_DIM, SPACE_DIM>* CreateCardiacTissue()
    {
        mpMonodomainTissue = new MonodomainTissue<ELEMENT_DIM, SPACE_DIM>(mpCellFactory);
        return mpMonodomainTissue;
    }
    virtual AbstractDynamicLinearPdeSolver<ELEMENT_DIM, SPACE_DIM, 1>* CreateSolver() = 0;
    virtual void OnEndOfTimestep(double time) {}
public:
    explicit MonodomainProblem(AbstractCardiacCellFactory<ELEMENT_DIM, SPACE_DIM>* pFactory) : mpCellFactory(pFactory) {}
    virtual ~MonodomainProblem()
    {
        delete mpCardiacTissue;
        delete mpMesh;
        delete mSolution;
    }
    // AbstractCardiacProblem::Initialise: mesh from HeartConfig, then the tissue
    void Initialise()
    {
        HeartConfig* p = HeartConfig::Instance();
        c_vector<double, 3> dims;
        p->GetSlabDimensions(dims);
        mpMesh = new AbstractTetrahedralMesh<ELEMENT_DIM, SPACE_DIM>;
        mpMesh->ConstructRegularSlabMesh(p->GetInterNodeSpace(), dims[0]);
        mpCellFactory->SetMesh(mpMesh);
        mpCardiacTissue = CreateCardiacTissue();
    }
    // AbstractCardiacProblem::Solve: initial condition from the cells' voltages, then
    // one solver Solve per printing interval and OnEndOfTimestep after each
    void Solve()
    {
        HeartConfig* p = HeartConfig::Instance();
        AbstractDynamicLinearPdeSolver<ELEMENT_DIM, SPACE_DIM, 1>* p_solver = CreateSolver();
        Vec current = new StubVec;
        for (unsigned i = 0; i < mpMesh->GetNumNodes(); ++i)
            current->mValues.push_back(mpCardiacTissue->GetCardiacCell(i)->GetStdVecStateVariables()[0]);
        const unsigned n_print = (unsigned)(p->GetSimulationDuration() / p->GetPrintingTimeStep() + 0.5);
        for (unsigned k = 0; k < n_print; ++k)
        {
            p_solver->SetTimes(k * p->GetPrintingTimeStep(), (k + 1) * p->GetPrintingTimeStep());
            p_solver->SetTimeStep(p->GetPdeTimeStep());
            p_solver->SetInitialCondition(current);
            Vec next = p_solver->Solve();
            delete current;
            current = next;
            OnEndOfTimestep((k + 1) * p->GetPrintingTimeStep());
        }
        delete p_solver;
        delete mSolution;
        mSolution = current;
    }
    Vec GetSolution() { return mSolution; }
    MonodomainTissue<ELEMENT_DIM, SPACE_DIM>* GetMonodomainTissue() { return mpMonodomainTissue; }
};

// Runs chaste_b200/shim/GpuMonodomainProblem.hpp against libchastegpu.so with the
// Chaste classes stubbed (tests/cpp/chaste_stubs): the call sequence of a Chaste
// MonodomainProblem solve, through the binding, on a 1D LR91 fibre.
//
//   test_gpu_binding describe   host-only checks of the binding's translations
//   test_gpu_binding run        the solve through the binding, then the same run
//                               directly through the C-ABI; prints both, exit 0
//                               when they agree bit for bit (exit 3 when the
//                               library raises, e.g. without a CUDA device)
#include <cstdio>
#include <cstring>

#include "GpuMonodomainProblem.hpp"
#include "models/lr91.h"

namespace
{

class CellLuoRudy1991FromCellML : public AbstractCardiacCell
{
public:
    CellLuoRudy1991FromCellML(boost::shared_ptr<AbstractStimulusFunction> pStim)
        : AbstractCardiacCell(boost::shared_ptr<AbstractIvpOdeSolver>(new EulerIvpOdeSolver), pStim)
    {
        mSystemName = "luo_rudy_1991";
        mStateVariables.assign(chb::LuoRudy1991::kInitialStates, chb::LuoRudy1991::kInitialStates + 8);
        SetParameter("membrane_fast_sodium_current_conductance", 23.0);
        SetParameter("membrane_L_type_calcium_current_conductance", 0.09);
        SetParameter("membrane_rapid_delayed_rectifier_potassium_current_conductance", 0.282);
    }
};

// PlaneStimulusCellFactory's shape: a SimpleStimulus on the nodes with x < 0.02
class FibreFactory : public AbstractCardiacCellFactory<1>
{
public:
    double mGkScale = 1.0;
    AbstractCardiacCellInterface* CreateCardiacCellForTissueNode(Node<1>* pNode)
    {
        const double x = pNode->rGetLocation()[0];
        boost::shared_ptr<AbstractStimulusFunction> stim;
        if (x < 0.02)
            stim.reset(new SimpleStimulus(-5e5, 0.5, 0.0));
        else
            stim.reset(new ZeroStimulus);
        CellLuoRudy1991FromCellML* p_cell = new CellLuoRudy1991FromCellML(stim);
        if (x > 0.5) p_cell->SetParameter("membrane_rapid_delayed_rectifier_potassium_current_conductance", 0.282 * mGkScale);
        return p_cell;
    }
};

int DescribeChecks()
{
    using namespace chaste_gpu_shim;
    boost::shared_ptr<AbstractStimulusFunction> s1(new SimpleStimulus(-25.5, 2.0, 50.0));
    boost::shared_ptr<AbstractStimulusFunction> s2(new RegularStimulus(-52.0, 1.0, 1000.0, 10.0, 5000.0));
    boost::shared_ptr<AbstractStimulusFunction> s3(new ZeroStimulus);
    const cg_stimulus a = Describe(s1), b = Describe(s2), c = Describe(s3);
    std::printf("simple %d %g %g %g\n", a.kind, a.magnitude, a.duration, a.start);
    std::printf("regular %d %g %g %g %g %g\n", b.kind, b.magnitude, b.duration, b.start, b.period, b.stop);
    std::printf("zero %d\n", c.kind);
    CellLuoRudy1991FromCellML cell(s3);
    int model = -1, method = -1;
    ModelOf(&cell, model, method);
    std::printf("model %d method %d\n", model, method);
    HeartConfig::Instance()->SetKSPPreconditioner("bjacobi");
    HeartConfig::Instance()->SetUseRelativeTolerance(1e-8);
    cg_config cfg = ConfigFromHeartConfig(model, method);
    std::printf("config pc %d abs %d tol %g\n", cfg.ksp_preconditioner, cfg.use_absolute_tolerance, cfg.ksp_tolerance);
    HeartConfig::Instance()->SetKSPPreconditioner("hypre");
    try
    {
        ConfigFromHeartConfig(model, method);
        std::printf("hypre accepted\n");
    }
    catch (const Exception& e)
    {
        std::printf("hypre rejected: %s\n", e.GetMessage().c_str());
    }
    return 0;
}

int Run(bool slab, const char* pc)
{
    HeartConfig* p = HeartConfig::Instance();
    p->SetOdePdeAndPrintingTimeSteps(0.01, 0.01, 0.5);
    p->SetSimulationDuration(4.0);
    p->SetUseRelativeTolerance(1e-8);
    p->SetKSPPreconditioner(pc);
    p->SetIntracellularConductivities(1.75);
    p->SetFibreLength(1.0, 0.01);
    p->SetCreateSlab(slab);
    FibreFactory factory;
    factory.mGkScale = 1.5;
    std::vector<double> v_binding;
    unsigned n = 0;
    try
    {
        GpuMonodomainProblem<1> problem(&factory);
        problem.Initialise();
        problem.SetSyncCellsAtPrintingTimes(true);
        problem.Solve();
        Vec v = problem.GetSolution();
        v_binding = v->mValues;
        n = (unsigned)v_binding.size();
        // the host views: cell 0's voltage and the Iion cache, synchronised at the last printing time
        const double v0 = problem.GetGpuTissue()->GetCardiacCell(0)->GetStdVecStateVariables()[0];
        const double iion0 = problem.GetGpuTissue()->rGetIionicCacheReplicated()[0];
        std::printf("binding V[0] %.17g cell view V %.17g Iion[0] %.17g\n", v_binding[0], v0, iion0);
        if (v0 != v_binding[0])
        {
            std::printf("cell view differs from the solution\n");
            return 1;
        }
    }
    catch (const Exception& e)
    {
        std::printf("EXCEPTION: %s\n", e.GetMessage().c_str());
        return 3;
    }
    // the same run directly through the C-ABI
    cg_config cfg;
    cg_default_config(&cfg);
    cfg.model = CG_MODEL_LR91;
    cfg.ode_method = CG_ODE_FORWARD_EULER;
    cfg.ode_time_step = cfg.pde_time_step = 0.01;
    cfg.use_absolute_tolerance = 0;
    cfg.ksp_tolerance = 1e-8;
    cfg.ksp_preconditioner = std::strcmp(pc, "bjacobi") == 0 ? CG_PC_BJACOBI : CG_PC_JACOBI;
    cg_ctx* ctx = nullptr;
    if (cg_create(&cfg, &ctx) != CG_OK) return 3;
    const double sigma = 1.75;
    int nn = 0;
    std::vector<double> xyz(3 * n, 0.0);
    std::vector<int> conn;
    for (unsigned i = 0; i < n; ++i) xyz[3 * i] = i * 0.01;
    for (unsigned e = 0; e + 1 < n; ++e)
    {
        conn.push_back((int)e);
        conn.push_back((int)e + 1);
    }
    std::vector<double> sig(n - 1, sigma);
    const int rc_mesh = slab ? cg_set_slab_mesh(ctx, 1, 0.01, 1.0, 0.0, 0.0, &sigma, &nn)
                             : cg_set_mesh(ctx, (int)n, 1, xyz.data(), (int)n - 1, conn.data(), sig.data());
    std::vector<int> pset(n), sid(n);
    // the scale the binding derives from the cell's parameter value
    const double gk = (0.282 * factory.mGkScale) / 0.282;
    const double table[12] = {1, 1, 1, 1, 1, 1, 1, 1, gk, 1, 1, 1};
    for (unsigned i = 0; i < n; ++i)
    {
        pset[i] = i * 0.01 > 0.5 ? 1 : 0;
        sid[i] = i * 0.01 < 0.02 ? 0 : -1;
    }
    cg_stimulus st = {CG_STIM_SIMPLE, -5e5, 0.5, 0.0, 0.0, 0.0};
    std::vector<double> v_direct(n);
    if (rc_mesh != CG_OK || cg_set_cells(ctx, nullptr, pset.data(), table, 2) != CG_OK ||
        cg_set_stimulus(ctx, sid.data(), &st, 1) != CG_OK || cg_step(ctx, 400) != CG_OK ||
        cg_get_voltage(ctx, v_direct.data()) != CG_OK)
    {
        cg_destroy(ctx);
        return 3;
    }
    cg_destroy(ctx);
    double diff = 0.0;
    for (unsigned i = 0; i < n; ++i) diff = std::fmax(diff, std::fabs(v_direct[i] - v_binding[i]));
    std::printf("nodes %u direct V[0] %.17g max |binding - direct| %.3g V[50] %.6g\n", n, v_direct[0], diff,
                v_binding[50]);
    return diff == 0.0 ? 0 : 1;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc > 1 && std::strcmp(argv[1], "describe") == 0) return DescribeChecks();
    const bool slab = !(argc > 2 && std::strcmp(argv[2], "mesh") == 0);
    const char* pc = argc > 3 ? argv[3] : "jacobi";
    return Run(slab, pc);
}

// CPU oracle, tissue part -- test infrastructure only (see oracle.h).
//
// Restates, for one process, Chaste's monodomain step:
//   MonodomainProblem -> AbstractDynamicLinearPdeSolver::Solve
//     (pde/src/solver/AbstractDynamicLinearPdeSolver.hpp:328-497)
//   a. MonodomainSolver::PrepareForSetupLinearSystem -> AbstractCardiacTissue::SolveCellSystems
//      (heart/src/tissue/AbstractCardiacTissue.cpp:464-567, caches :730-734)
//   b. MonodomainSolver::SetupLinearSystem (heart/src/solver/electrics/monodomain/MonodomainSolver.cpp:42-131)
//      with A = Am*Cm/dt*M + K (MonodomainAssembler.cpp:43-66) assembled once
//   c. LinearSystem::Solve (linalg/src/LinearSystem.cpp:674-1215) = PETSc KSPCG with
//      jacobi / bjacobi(ILU(0)) and the default convergence test.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <set>
#include <thread>
#include <vector>

#include "oracle.h"
#include "oracle_internal.h"

namespace orc {

// ------------------------------------------------------------ thread pool --
class Pool {
  public:
    explicit Pool(int n) { resize(n); }
    ~Pool() { stop(); }
    int size() const { return (int)workers_.size() + 1; }
    void resize(int n) {
        stop();
        if (n < 1) n = 1;
        quit_ = false;
        for (int i = 1; i < n; ++i) workers_.emplace_back([this, i] { loop(i); });
    }
    // fn(thread_index, n_threads)
    void run(const std::function<void(int, int)>& fn) {
        const int nt = size();
        if (nt == 1) {
            fn(0, 1);
            return;
        }
        {
            std::lock_guard<std::mutex> lk(m_);
            job_ = &fn;
            pending_ = nt - 1;
            gen_++;
        }
        cv_.notify_all();
        fn(0, nt);
        std::unique_lock<std::mutex> lk(m_);
        done_cv_.wait(lk, [this] { return pending_ == 0; });
        job_ = nullptr;
    }

  private:
    void loop(int idx) {
        unsigned long seen = 0;
        for (;;) {
            const std::function<void(int, int)>* job;
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return quit_ || gen_ != seen; });
                if (quit_) return;
                seen = gen_;
                job = job_;
            }
            (*job)(idx, size());
            {
                std::lock_guard<std::mutex> lk(m_);
                if (--pending_ == 0) done_cv_.notify_one();
            }
        }
    }
    void stop() {
        {
            std::lock_guard<std::mutex> lk(m_);
            quit_ = true;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
        workers_.clear();
    }
    std::vector<std::thread> workers_;
    std::mutex m_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(int, int)>* job_ = nullptr;
    int pending_ = 0;
    unsigned long gen_ = 0;
    bool quit_ = false;
};

static Pool& pool() {
    static Pool p(1);
    return p;
}

template <class F>
static void parallel_for(int n, F f) {
    Pool& P = pool();
    P.run([&](int ti, int nt) {
        const int b = (int)((long long)n * ti / nt), e = (int)((long long)n * (ti + 1) / nt);
        f(b, e);
    });
}

// Deterministic sum over [0,n): per-thread partials added in thread order.
template <class F>
static double parallel_sum(int n, F f) {
    Pool& P = pool();
    std::vector<double> part(P.size(), 0.0);
    P.run([&](int ti, int nt) {
        const int b = (int)((long long)n * ti / nt), e = (int)((long long)n * (ti + 1) / nt);
        double s = 0.0;
        for (int i = b; i < e; ++i) s += f(i);
        part[ti] = s;
    });
    double s = 0.0;
    for (double x : part) s += x;
    return s;
}

// ------------------------------------------------------------------- CSR --
struct Csr {
    int n = 0;
    std::vector<int> rp, ci;
    std::vector<double> v;
    void matvec(const double* x, double* y) const {
        parallel_for(n, [&](int b, int e) {
            for (int i = b; i < e; ++i) {
                double s = 0.0;
                for (int k = rp[i]; k < rp[i + 1]; ++k) s += v[k] * x[ci[k]];
                y[i] = s;
            }
        });
    }
    int find(int i, int j) const {
        int lo = rp[i], hi = rp[i + 1] - 1;
        while (lo <= hi) {
            const int mid = (lo + hi) / 2;
            if (ci[mid] == j) return mid;
            if (ci[mid] < j) lo = mid + 1;
            else hi = mid - 1;
        }
        return -1;
    }
};

// ---------------------------------------------------- element matrices --
// P1 simplex in dim dimensions.  The reference integrates with the order-2
// Gauss rule (AbstractFeVolumeIntegralAssembler.hpp:253, GaussianQuadratureRule.cpp),
// which is exact for these integrands, so the closed forms are used:
//   M_e = |J| * vol_ref * (1 + delta_ij) / ((d+1)(d+2))   (MassMatrixAssembler.hpp:76-104)
//   K_e = |J| * vol_ref * gradphi^T sigma gradphi        (MonodomainStiffnessMatrixAssembler.hpp:68-84)
static bool element_matrices(int dim, const double* X /*(dim+1)x3*/, const double* sigma,
                             bool lump, double* Me, double* Ke) {
    const int nb = dim + 1;
    double J[3][3] = {{0}}, Ji[3][3] = {{0}};
    for (int c = 0; c < dim; ++c)
        for (int r = 0; r < dim; ++r) J[r][c] = X[(c + 1) * 3 + r] - X[r];
    double det;
    if (dim == 1) {
        det = J[0][0];
        Ji[0][0] = 1.0 / det;
    } else if (dim == 2) {
        det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
        Ji[0][0] = J[1][1] / det;
        Ji[0][1] = -J[0][1] / det;
        Ji[1][0] = -J[1][0] / det;
        Ji[1][1] = J[0][0] / det;
    } else {
        det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
              J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
              J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
        Ji[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
        Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
        Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
        Ji[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
        Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
        Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
        Ji[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
        Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
        Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
    }
    if (det == 0.0) return false;
    const double adet = std::fabs(det);
    const double vol_ref = dim == 1 ? 1.0 : (dim == 2 ? 0.5 : 1.0 / 6.0);
    // reference gradients: phi_0 = 1 - sum xi, phi_k = xi_k
    double G[3][4] = {{0}};   // G[s][b] = d phi_b / d x_s
    for (int b = 0; b < nb; ++b) {
        double g_ref[3] = {0, 0, 0};
        if (b == 0)
            for (int s = 0; s < dim; ++s) g_ref[s] = -1.0;
        else
            g_ref[b - 1] = 1.0;
        for (int s = 0; s < dim; ++s) {
            double acc = 0.0;
            for (int r = 0; r < dim; ++r) acc += Ji[r][s] * g_ref[r];   // (J^{-T} g)_s
            G[s][b] = acc;
        }
    }
    const double w = adet * vol_ref;
    for (int i = 0; i < nb; ++i)
        for (int j = 0; j < nb; ++j) {
            double k = 0.0;
            for (int s = 0; s < dim; ++s) k += G[s][i] * sigma[s] * G[s][j];
            Ke[i * nb + j] = w * k;
            Me[i * nb + j] = w * (i == j ? 2.0 : 1.0) / ((dim + 1) * (dim + 2));
        }
    if (lump) {
        for (int i = 0; i < nb; ++i) {
            double s = 0.0;
            for (int j = 0; j < nb; ++j) s += Me[i * nb + j];
            for (int j = 0; j < nb; ++j) Me[i * nb + j] = (i == j) ? s : 0.0;
        }
    }
    return true;
}

// ---------------------------------------------------------------- tissue --
struct Tissue {
    orc_config cfg;
    int dim, n, ns, np;
    std::vector<double> V, states /* node-major */, iion, istim;
    std::vector<int> stim_id, param_id;
    std::vector<orc_stimulus> stims;
    std::vector<double> param_table;
    Csr A, M;
    std::vector<double> dinv;                 // Jacobi
    std::vector<double> ilu;                  // ILU(0) factors in A's pattern
    std::vector<int> ilu_diag;
    std::vector<double> b, z, r, p, w, x;
    std::vector<int> conn;                    // kept for state-variable interpolation
    std::vector<double> detj;                 // |det J| per element
    double t = 0.0;
    long long steps = 0;
    // bidomain (orc_tissue_set_bidomain): the interleaved system of (V, phi_e)
    bool bido = false;
    bool nullspace = true;                    // no fixed phi_e: PETSc null space of constant phi_e
    Csr B;                                    // 2n x 2n, row 2i the V equation, 2i+1 the phi_e one
    std::vector<double> bdinv, u, bb, br, bz, bp, bw, bmz;
};

static void ilu0_factor(const Csr& A, std::vector<double>& lu, std::vector<int>& diag) {
    // ILU(0) with natural ordering, no pivoting: PETSc bjacobi on one process
    // applies ILU(0) to the single diagonal block (the whole matrix).
    const int n = A.n;
    lu = A.v;
    diag.assign(n, -1);
    for (int i = 0; i < n; ++i) diag[i] = A.find(i, i);
    for (int i = 1; i < n; ++i) {
        for (int kk = A.rp[i]; kk < A.rp[i + 1] && A.ci[kk] < i; ++kk) {
            const int k = A.ci[kk];
            lu[kk] /= lu[diag[k]];
            const double lik = lu[kk];
            // row i -= lik * row k (only on the pattern of row i, columns > k)
            int jj = kk + 1;
            for (int kj = diag[k] + 1; kj < A.rp[k + 1]; ++kj) {
                const int j = A.ci[kj];
                while (jj < A.rp[i + 1] && A.ci[jj] < j) ++jj;
                if (jj < A.rp[i + 1] && A.ci[jj] == j) lu[jj] -= lik * lu[kj];
            }
        }
    }
}

static void ilu0_apply(const Csr& A, const std::vector<double>& lu, const std::vector<int>& diag,
                       const double* rin, double* zout) {
    const int n = A.n;
    for (int i = 0; i < n; ++i) {
        double s = rin[i];
        for (int k = A.rp[i]; k < diag[i]; ++k) s -= lu[k] * zout[A.ci[k]];
        zout[i] = s;
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = zout[i];
        for (int k = diag[i] + 1; k < A.rp[i + 1]; ++k) s -= lu[k] * zout[A.ci[k]];
        zout[i] = s / lu[diag[i]];
    }
}

static void pc_apply(Tissue& T, const double* rin, double* zout) {
    const int n = T.n;
    if (T.cfg.pc == ORC_PC_JACOBI) {
        const double* d = T.dinv.data();
        parallel_for(n, [&](int b, int e) {
            for (int i = b; i < e; ++i) zout[i] = rin[i] * d[i];
        });
    } else if (T.cfg.pc == ORC_PC_BJACOBI) {
        ilu0_apply(T.A, T.ilu, T.ilu_diag, rin, zout);
    } else {
        std::memcpy(zout, rin, sizeof(double) * n);
    }
}

static double dot(int n, const double* a, const double* b) {
    return parallel_sum(n, [&](int i) { return a[i] * b[i]; });
}

// PETSc KSPSolve_CG (src/ksp/ksp/impls/cg/cg.c, standard variant, left
// preconditioning, KSP_NORM_PRECONDITIONED) with KSPConvergedDefault: with a
// nonzero initial guess rnorm0 = ||B b||, ttol = max(rtol*rnorm0, abstol);
// converged when ||B r_k|| <= ttol (checked from iteration 0), diverged when
// ||B r_k|| >= dtol*rnorm0 (dtol 1e5) or the iteration count reaches max_it.
// `pc` is KSP_PCApply: the preconditioner followed, when the operator has a null
// space, by its removal from the result.
template <class Mv, class Pc>
static int cg_core(const orc_config& cfg, int n, double* xv, const double* bv, double* R, double* Z, double* P,
                   double* W, Mv matvec, Pc pc, int* iters) {
    const double rtol = cfg.use_abs_tol ? DBL_EPSILON : cfg.tol;
    const double abstol = cfg.use_abs_tol ? cfg.tol : 1e-50;
    const double dtol = 1e5;
    const int maxit = cfg.max_iterations > 0 ? cfg.max_iterations : 10000;
    // LinearSystem::Solve: small nonzero RHS -> zero guess (LinearSystem.cpp:984-994)
    double rhs1 = parallel_sum(n, [&](int i) { return std::fabs(bv[i]); });
    bool guess_zero = false;
    if (rhs1 < 1e-15 && rhs1 > 0.0) {
        std::fill(xv, xv + n, 0.0);
        guess_zero = true;
    }
    // r = b - A x
    matvec(xv, R);
    parallel_for(n, [&](int b, int e) {
        for (int i = b; i < e; ++i) R[i] = bv[i] - R[i];
    });
    pc(R, Z);
    double dp = std::sqrt(dot(n, Z, Z));
    double rnorm0;
    if (!guess_zero) {
        pc(bv, W);
        double snorm = std::sqrt(dot(n, W, W));
        rnorm0 = snorm != 0.0 ? snorm : dp;
    } else {
        rnorm0 = dp;
    }
    const double ttol = std::max(rtol * rnorm0, abstol);
    *iters = 0;
    if (std::isnan(dp) || std::isinf(dp)) return -3;
    if (dp <= ttol) return 0;
    if (dp >= dtol * rnorm0) return -2;
    double beta = dot(n, Z, R), betaold = 0.0;
    int i = 0;
    do {
        *iters = i + 1;
        if (beta == 0.0) return 0;
        if (i == 0) {
            std::memcpy(P, Z, sizeof(double) * n);
        } else {
            const double bb = beta / betaold;
            parallel_for(n, [&](int b, int e) {
                for (int k = b; k < e; ++k) P[k] = Z[k] + bb * P[k];
            });
        }
        matvec(P, Z);                           // Z = A p
        const double dpi = dot(n, P, Z);
        if (dpi <= 0.0) return -2;              // indefinite matrix
        const double a = beta / dpi;
        parallel_for(n, [&](int b, int e) {
            for (int k = b; k < e; ++k) {
                xv[k] += a * P[k];
                R[k] -= a * Z[k];
            }
        });
        pc(R, Z);
        dp = std::sqrt(dot(n, Z, Z));
        if (std::isnan(dp) || std::isinf(dp)) return -3;
        if (dp <= ttol) return 0;
        if (dp >= dtol * rnorm0) return -2;
        betaold = beta;
        beta = dot(n, Z, R);
        i++;
    } while (i < maxit);
    return -1;
}

static int cg_solve(Tissue& T, double* xv, const double* bv, int* iters) {
    return cg_core(
        T.cfg, T.n, xv, bv, T.r.data(), T.z.data(), T.p.data(), T.w.data(),
        [&](const double* x, double* y) { T.A.matvec(x, y); },
        [&](const double* r, double* z) { pc_apply(T, r, z); }, iters);
}

template <class Mdl>
static void solve_cells(Tissue& T, double t0, double t1) {
    const int ns = Mdl::kNumStates;
    const int np = Mdl::kNumParams;
    parallel_for(T.n, [&](int b, int e) {
        double y[Mdl::kNumStates];
        double pdef[16];
        for (int k = 0; k < np; ++k) pdef[k] = 1.0;
        for (int i = b; i < e; ++i) {
            double* s = &T.states[(size_t)i * ns];
            for (int k = 0; k < ns; ++k) y[k] = s[k];
            y[0] = T.V[i];                                   // SetVoltage
            const double* p = pdef;
            if (!T.param_id.empty() && T.param_id[i] >= 0)
                p = &T.param_table[(size_t)T.param_id[i] * np];
            const orc_stimulus* st = (!T.stim_id.empty() && T.stim_id[i] >= 0) ? &T.stims[T.stim_id[i]] : nullptr;
            except_voltage<Mdl>(T.cfg.ode_method, y, p, st, T.cfg.am, T.cfg.cm, t0, t1, T.cfg.dt_ode);
            y[0] = T.V[i];                                   // restore V (AbstractCardiacCell.cpp:98)
            for (int k = 0; k < ns; ++k) s[k] = y[k];
            T.iion[i] = Mdl::template iionic<double>(y, T.cfg.cm, p);     // UpdateCaches
            T.istim[i] = stimulus_value(st, t1);
        }
    });
}

// SolveCellSystems(..., updateVoltage = true) for the operator-splitting solver
// (AbstractCardiacTissue.cpp:531-536): every cell's SolveAndUpdateState over
// [t0, t1] including V -- forward Euler through AbstractOneStepIvpOdeSolver's
// InternalSolve (ode/src/solver/AbstractOneStepIvpOdeSolver.cpp:115-153), Rush-Larsen
// (AbstractRushLarsenCardiacCell.cpp:130-147, V by Euler first) or backward Euler
// (AbstractBackwardEulerCardiacCell.hpp SolveAndUpdateState, chb::be_step) --
// then V from the cell and UpdateCaches at t1.
template <class Mdl>
static void solve_cells_with_voltage(Tissue& T, double t0, double t1) {
    const int ns = Mdl::kNumStates;
    const int np = Mdl::kNumParams;
    parallel_for(T.n, [&](int b, int e) {
        double y[Mdl::kNumStates], dy[Mdl::kNumStates];
        double pdef[16];
        for (int k = 0; k < np; ++k) pdef[k] = 1.0;
        for (int i = b; i < e; ++i) {
            double* s = &T.states[(size_t)i * ns];
            for (int k = 0; k < ns; ++k) y[k] = s[k];
            y[0] = T.V[i];
            const double* p = pdef;
            if (!T.param_id.empty() && T.param_id[i] >= 0)
                p = &T.param_table[(size_t)T.param_id[i] * np];
            const orc_stimulus* st = (!T.stim_id.empty() && T.stim_id[i] >= 0) ? &T.stims[T.stim_id[i]] : nullptr;
            TimeStepper ts(t0, t1, T.cfg.dt_ode);
            while (!ts.AtEnd()) {
                const double sv = stimulus_value(st, ts.Time()) / T.cfg.am;   // GetIntracellularAreaStimulus
                if (T.cfg.ode_method == ORC_RL) {
                    chb::rl_step<Mdl, double>(y, sv, T.cfg.cm, p, T.cfg.dt_ode);
                } else if (T.cfg.ode_method == ORC_BE) {
                    chb::be_step<Mdl, double>(y, sv, T.cfg.cm, p, T.cfg.dt_ode, true);
                } else if (T.cfg.ode_method == ORC_GRL1 || T.cfg.ode_method == ORC_GRL2) {
                    grl_next<Mdl>(T.cfg.ode_method, y, sv, T.cfg.cm, p, ts.NextStep(), false);
                } else {
                    const double h = ts.NextStep();
                    Mdl::template rhs<double>(y, sv, T.cfg.cm, p, dy);
                    for (int k = 0; k < ns; ++k) y[k] += h * dy[k];
                }
                ts.Advance();
            }
            T.V[i] = y[0];
            for (int k = 0; k < ns; ++k) s[k] = y[k];
            T.iion[i] = Mdl::template iionic<double>(y, T.cfg.cm, p);
            T.istim[i] = stimulus_value(st, t1);
        }
    });
}

// OperatorSplittingMonodomainSolver (heart/src/solver/electrics/monodomain/
// OperatorSplittingMonodomainSolver.cpp:40-117): half a step of the cells with V,
// the diffusion solve with z = Am*Cm*V/dt (no reaction term), the second half.
static int step_split(Tissue& T, int* iters) {
    const double t0 = T.t;
    const double dt = T.cfg.dt_pde;
    const double t1 = (double)(T.steps + 1) * dt;
    if (T.cfg.model == ORC_TT06) solve_cells_with_voltage<chb::TenTusscher2006Epi>(T, t0, t0 + dt / 2.0);
    else solve_cells_with_voltage<chb::LuoRudy1991>(T, t0, t0 + dt / 2.0);
    const double am = T.cfg.am, cm = T.cfg.cm;
    const double dtinv = 1.0 / dt;
    double* zz = T.w.data();
    parallel_for(T.n, [&](int b, int e) {
        for (int i = b; i < e; ++i) zz[i] = am * cm * T.V[i] * dtinv;
    });
    T.M.matvec(zz, T.b.data());
    T.x = T.V;
    const int rc = cg_solve(T, T.x.data(), T.b.data(), iters);
    if (rc != 0) return rc;
    T.V = T.x;
    if (T.cfg.model == ORC_TT06) solve_cells_with_voltage<chb::TenTusscher2006Epi>(T, t0 + dt / 2.0, t1);
    else solve_cells_with_voltage<chb::LuoRudy1991>(T, t0 + dt / 2.0, t1);
    T.steps++;
    T.t = t1;
    return 0;
}

// State-variable interpolation: MonodomainCorrectionTermAssembler::ComputeVectorTerm
// (heart/src/solver/electrics/monodomain/MonodomainCorrectionTermAssembler.cpp:47-66)
// on the elements AbstractCorrectionTermAssembler::ElementAssemblyCriterion selects
// (heart/src/solver/electrics/AbstractCorrectionTermAssembler.cpp:109-146: largest
// |Iion_a - Iion_b| over the element's nodes above 1), with the order-2 Gaussian rule
// (pde/src/solver/GaussianQuadratureRule.cpp) -- at quadrature point q one node has
// basis value A and the others B -- accumulated element by element onto b.
template <class Mdl>
static void svi_correction(Tissue& T, double* b) {
    constexpr int S = Mdl::kNumStates;
    const int nb = T.dim + 1;
    const int ne = (int)T.detj.size();
    double A, B, wref;
    int big[4];
    if (T.dim == 1) {
        const double r = std::sqrt(1.0 / 3.0);
        A = (r + 1.0) / 2.0;       // basis 1 - xi at xi = (1 - r)/2
        B = (-r + 1.0) / 2.0;
        wref = 0.5;
        big[0] = 0, big[1] = 1;
    } else if (T.dim == 2) {
        A = 2.0 / 3.0, B = 1.0 / 6.0, wref = 1.0 / 6.0;
        big[0] = 1, big[1] = 0, big[2] = 2;
    } else {
        const double sf = 1.0 / std::sqrt(5.0);
        A = (1.0 + 3.0 * sf) / 4.0, B = (1.0 - sf) / 4.0, wref = 1.0 / 24.0;
        big[0] = 1, big[1] = 2, big[2] = 3, big[3] = 0;
    }
    double pdef[16];
    for (int k = 0; k < T.np; ++k) pdef[k] = 1.0;
    for (int e = 0; e < ne; ++e) {
        const int* nd = &T.conn[(size_t)e * nb];
        double di = 0.0;
        for (int x = 0; x < nb; ++x)
            for (int y = x + 1; y < nb; ++y) di = std::max(di, std::fabs(T.iion[nd[x]] - T.iion[nd[y]]));
        if (!(di > 1.0)) continue;
        const double wj = T.detj[e] * wref;
        const double* p = pdef;
        if (!T.param_id.empty() && T.param_id[nd[0]] >= 0) p = &T.param_table[(size_t)T.param_id[nd[0]] * T.np];
        double be[4] = {0, 0, 0, 0};
        for (int q = 0; q < nb; ++q) {
            double phi[4], y[S], iint = 0.0;
            for (int j = 0; j < nb; ++j) phi[j] = j == big[q] ? A : B;
            for (int k = 0; k < S; ++k) y[k] = 0.0;
            for (int j = 0; j < nb; ++j) {
                iint += phi[j] * T.iion[nd[j]];
                const double* sj = &T.states[(size_t)nd[j] * T.ns];
                for (int k = 0; k < S; ++k) y[k] += phi[j] * sj[k];
            }
            const double isv = Mdl::template iionic<double>(y, T.cfg.cm, p);
            for (int i = 0; i < nb; ++i) be[i] += phi[i] * (-T.cfg.am) * (isv - iint) * wj;
        }
        for (int i = 0; i < nb; ++i) b[nd[i]] += be[i];
    }
}

// ------------------------------------------------------------- bidomain --
// BidomainProblem without a bath: BidomainSolver::SetupLinearSystem
// (heart/src/solver/electrics/bidomain/BidomainSolver.cpp:63-190) on the interleaved
// unknowns (V_0, phi_0, V_1, phi_1, ...) with the blocks of BidomainAssembler
// (BidomainAssembler.cpp:41-89) and BidomainMassMatrixAssembler (mass in the V-V block
// only), b = M z with z = (Am Cm V/dt - Am Iion - Istim, 0); then PETSc CG.  With no
// fixed phi_e the system is singular and the solve carries the null space of constant
// phi_e (AbstractBidomainSolver::FinaliseLinearSystem / GenerateNullBasis,
// AbstractBidomainSolver.cpp:112-186): KSP_PCApply removes it from every
// preconditioned vector.  Fixed phi_e nodes are Dirichlet rows and columns
// (BoundaryConditionsContainer::ApplyDirichletToLinearProblem on a symmetric matrix,
// pde/src/common/BoundaryConditionsContainerImplementation.hpp:257-417) with value 0.
static void bido_pc(Tissue& T, const double* r, double* z) {
    const int n2 = 2 * T.n;
    if (T.cfg.pc == ORC_PC_JACOBI) {
        const double* d = T.bdinv.data();
        parallel_for(n2, [&](int b, int e) {
            for (int i = b; i < e; ++i) z[i] = r[i] * d[i];
        });
    } else {
        std::memcpy(z, r, sizeof(double) * n2);
    }
    if (T.nullspace) {
        // MatNullSpaceRemove: z -= (z . e) e, e = (0, 1/sqrt(n), 0, 1/sqrt(n), ...)
        const double inv = 1.0 / std::sqrt((double)T.n);
        const double alpha = parallel_sum(T.n, [&](int i) { return z[2 * i + 1] * inv; });
        parallel_for(T.n, [&](int b, int e) {
            for (int i = b; i < e; ++i) z[2 * i + 1] -= alpha * inv;
        });
    }
}

static int step_bido(Tissue& T, int* iters) {
    const double t0 = T.t;
    const double t1 = (double)(T.steps + 1) * T.cfg.dt_pde;
    if (T.cfg.model == ORC_TT06) solve_cells<chb::TenTusscher2006Epi>(T, t0, t1);
    else solve_cells<chb::LuoRudy1991>(T, t0, t1);
    const double am = T.cfg.am, cm = T.cfg.cm;
    const double dtinv = 1.0 / T.cfg.dt_pde;
    double* zz = T.w.data();
    parallel_for(T.n, [&](int b, int e) {
        for (int i = b; i < e; ++i) zz[i] = am * cm * T.V[i] * dtinv + (-am * T.iion[i] - T.istim[i]);
    });
    T.M.matvec(zz, T.bmz.data());
    for (int i = 0; i < T.n; ++i) {
        T.bb[2 * i] = T.bmz[i];
        T.bb[2 * i + 1] = 0.0;   // phi_e rows of M z are zero; fixed rows hold the value 0
    }
    for (int i = 0; i < T.n; ++i) T.u[2 * i] = T.V[i];
    const int rc = cg_core(
        T.cfg, 2 * T.n, T.u.data(), T.bb.data(), T.br.data(), T.bz.data(), T.bp.data(), T.bw.data(),
        [&](const double* x, double* y) { T.B.matvec(x, y); }, [&](const double* r, double* z) { bido_pc(T, r, z); },
        iters);
    if (rc != 0) return rc;
    for (int i = 0; i < T.n; ++i) T.V[i] = T.u[2 * i];
    T.steps++;
    T.t = t1;
    return 0;
}

static int step_once(Tissue& T, int* iters) {
    if (T.bido) return step_bido(T, iters);
    if (T.cfg.solver == ORC_SOLVER_OPERATOR_SPLITTING) return step_split(T, iters);
    const double t0 = T.t;
    const double t1 = (double)(T.steps + 1) * T.cfg.dt_pde;
    if (T.cfg.model == ORC_TT06) solve_cells<chb::TenTusscher2006Epi>(T, t0, t1);
    else solve_cells<chb::LuoRudy1991>(T, t0, t1);
    // z = Am*Cm*V/dt - Am*Iion - Istim ; b = M z  (MonodomainSolver.cpp:92-107)
    const double am = T.cfg.am, cm = T.cfg.cm;
    const double dtinv = 1.0 / T.cfg.dt_pde;
    double* zz = T.w.data();
    parallel_for(T.n, [&](int b, int e) {
        for (int i = b; i < e; ++i) {
            const double F = -am * T.iion[i] - T.istim[i];
            zz[i] = am * cm * T.V[i] * dtinv + F;
        }
    });
    T.M.matvec(zz, T.b.data());
    if (T.cfg.svi) {
        if (T.cfg.model == ORC_TT06) svi_correction<chb::TenTusscher2006Epi>(T, T.b.data());
        else svi_correction<chb::LuoRudy1991>(T, T.b.data());
    }
    T.x = T.V;
    const int rc = cg_solve(T, T.x.data(), T.b.data(), iters);
    if (rc != 0) return rc;
    T.V = T.x;
    T.steps++;
    T.t = t1;
    return 0;
}

}  // namespace orc

using namespace orc;

struct orc_tissue {
    Tissue T;
};

extern "C" {

void orc_set_threads(int n) { pool().resize(n); }

int orc_slab_mesh(int dim, double h, double width, double height, double depth, int* n_nodes,
                  int* n_elems, int* grid, double* xyz, int* conn) {
    // ConstructRegularSlabMesh (AbstractTetrahedralMesh.cpp:569-614)
    const unsigned nx = (unsigned)((width + 0.5 * h) / h);
    const unsigned ny = dim > 1 ? (unsigned)((height + 0.5 * h) / h) : 0;
    const unsigned nz = dim > 2 ? (unsigned)((depth + 0.5 * h) / h) : 0;
    if (std::fabs(nx * h - width) > DBL_EPSILON * width ||
        (dim > 1 && height != 0.0 && std::fabs(ny * h - height) > DBL_EPSILON * height) ||
        (dim > 2 && depth != 0.0 && std::fabs(nz * h - depth) > DBL_EPSILON * depth))
        return -1;
    const int NX = nx + 1, NY = dim > 1 ? ny + 1 : 1, NZ = dim > 2 ? nz + 1 : 1;
    *n_nodes = NX * NY * NZ;
    *n_elems = dim == 1 ? nx : (dim == 2 ? 2 * nx * ny : 6 * nx * ny * nz);
    if (grid) {
        grid[0] = nx;
        grid[1] = ny;
        grid[2] = nz;
    }
    if (!xyz || !conn) return 0;
    // node index (k*(ny+1)+j)*(nx+1)+i; coordinates scaled by h (Scale, :613)
    for (int k = 0; k < NZ; ++k)
        for (int j = 0; j < NY; ++j)
            for (int i = 0; i < NX; ++i) {
                const long idx = ((long)k * NY + j) * NX + i;
                xyz[idx * 3 + 0] = i * h;
                xyz[idx * 3 + 1] = j * h;
                xyz[idx * 3 + 2] = k * h;
            }
    if (dim == 1) {
        // ConstructLinearMesh (:244-275)
        for (unsigned e = 0; e < nx; ++e) {
            conn[e * 2] = e;
            conn[e * 2 + 1] = e + 1;
        }
    } else if (dim == 2) {
        // ConstructRectangularMesh with stagger (:336-376)
        long el = 0;
        for (unsigned j = 0; j < ny; ++j)
            for (unsigned i = 0; i < nx; ++i) {
                const unsigned parity = (i + (ny - j)) % 2;
                const int nw = (j + 1) * (nx + 1) + i;
                const int sw = j * (nx + 1) + i;
                conn[el * 3 + 0] = nw;
                conn[el * 3 + 1] = nw + 1;
                conn[el * 3 + 2] = parity == 1 ? sw + 1 : sw;
                el++;
                conn[el * 3 + 0] = sw + 1;
                conn[el * 3 + 1] = sw;
                conn[el * 3 + 2] = parity == 1 ? nw : nw + 1;
                el++;
            }
    } else {
        // ConstructCuboid: 6 tetrahedra per cube sharing the diagonal 0-7 (:420-422)
        static const int en[6][4] = {{0, 1, 5, 7}, {0, 1, 3, 7}, {0, 2, 3, 7},
                                     {0, 2, 6, 7}, {0, 4, 6, 7}, {0, 4, 5, 7}};
        long el = 0;
        for (unsigned k = 0; k < nz; ++k)
            for (unsigned j = 0; j < ny; ++j)
                for (unsigned i = 0; i < nx; ++i) {
                    int g[8], l = 0;
                    for (int z = 0; z < 2; ++z)
                        for (int y = 0; y < 2; ++y)
                            for (int x = 0; x < 2; ++x)
                                g[l++] = i + x + (nx + 1) * (j + y + (ny + 1) * (k + z));
                    for (int m = 0; m < 6; ++m) {
                        for (int q = 0; q < 4; ++q) conn[el * 4 + q] = g[en[m][q]];
                        el++;
                    }
                }
    }
    return 0;
}

orc_tissue* orc_tissue_create(const orc_config* cfg, int dim, int n_nodes, const double* xyz,
                              int n_elems, const int* conn, const double* sigma, const int* stim_id,
                              const orc_stimulus* stims, int n_stims, const int* param_id,
                              const double* param_table, int n_param_sets, const double* init_states) {
    orc_tissue* h = new orc_tissue();
    Tissue& T = h->T;
    T.cfg = *cfg;
    T.dim = dim;
    T.n = n_nodes;
    T.ns = orc_num_states(cfg->model);
    T.np = orc_num_params(cfg->model);
    T.states.resize((size_t)T.n * T.ns);
    std::vector<double> y0(T.ns);
    orc_initial_states(cfg->model, y0.data());
    for (int i = 0; i < T.n; ++i)
        for (int k = 0; k < T.ns; ++k)
            T.states[(size_t)i * T.ns + k] = init_states ? init_states[(size_t)i * T.ns + k] : y0[k];
    // initial condition: each cell's voltage (AbstractCardiacProblem.cpp:265-292)
    T.V.resize(T.n);
    for (int i = 0; i < T.n; ++i) T.V[i] = T.states[(size_t)i * T.ns];
    T.iion.assign(T.n, 0.0);
    T.istim.assign(T.n, 0.0);
    if (stim_id) T.stim_id.assign(stim_id, stim_id + T.n);
    if (stims) T.stims.assign(stims, stims + n_stims);
    if (param_id) T.param_id.assign(param_id, param_id + T.n);
    if (param_table) T.param_table.assign(param_table, param_table + (size_t)n_param_sets * T.np);
    // sparsity: node adjacency through elements
    const int nb = dim + 1;
    std::vector<std::vector<int>> adj(T.n);
    for (int e = 0; e < n_elems; ++e)
        for (int a = 0; a < nb; ++a)
            for (int c = 0; c < nb; ++c) adj[conn[e * nb + a]].push_back(conn[e * nb + c]);
    for (Csr* C : {&T.A, &T.M}) {
        C->n = T.n;
        C->rp.assign(T.n + 1, 0);
    }
    for (int i = 0; i < T.n; ++i) {
        std::sort(adj[i].begin(), adj[i].end());
        adj[i].erase(std::unique(adj[i].begin(), adj[i].end()), adj[i].end());
        T.A.rp[i + 1] = T.A.rp[i] + (int)adj[i].size();
    }
    T.A.ci.resize(T.A.rp[T.n]);
    for (int i = 0; i < T.n; ++i) std::copy(adj[i].begin(), adj[i].end(), T.A.ci.begin() + T.A.rp[i]);
    T.A.v.assign(T.A.ci.size(), 0.0);
    T.M.rp = T.A.rp;
    T.M.ci = T.A.ci;
    T.M.v.assign(T.A.ci.size(), 0.0);
    if (cfg->svi) {
        T.conn.assign(conn, conn + (size_t)n_elems * nb);
        T.detj.resize(n_elems);
        for (int e = 0; e < n_elems; ++e) {
            const double* x0 = &xyz[(size_t)conn[e * nb] * 3];
            double d[3][3] = {{0}};
            for (int a = 1; a < nb; ++a)
                for (int s2 = 0; s2 < 3; ++s2) d[a - 1][s2] = xyz[(size_t)conn[e * nb + a] * 3 + s2] - x0[s2];
            double det;
            if (dim == 1) det = d[0][0];
            else if (dim == 2) det = d[0][0] * d[1][1] - d[0][1] * d[1][0];
            else
                det = d[0][0] * (d[1][1] * d[2][2] - d[1][2] * d[2][1]) - d[0][1] * (d[1][0] * d[2][2] - d[1][2] * d[2][0]) +
                      d[0][2] * (d[1][0] * d[2][1] - d[1][1] * d[2][0]);
            T.detj[e] = std::fabs(det);
        }
    }
    // assemble (AbstractFeVolumeIntegralAssembler::DoAssemble, element loop)
    const double mass_scale = cfg->am * cfg->cm / cfg->dt_pde;
    for (int e = 0; e < n_elems; ++e) {
        double X[4 * 3];
        for (int a = 0; a < nb; ++a)
            for (int s = 0; s < 3; ++s) X[a * 3 + s] = xyz[(size_t)conn[e * nb + a] * 3 + s];
        double Me[16], Ke[16];
        if (!element_matrices(dim, X, sigma + (size_t)e * dim, cfg->mass_lumping != 0, Me, Ke)) {
            delete h;
            return nullptr;
        }
        for (int a = 0; a < nb; ++a)
            for (int c = 0; c < nb; ++c) {
                const int k = T.A.find(conn[e * nb + a], conn[e * nb + c]);
                T.A.v[k] += mass_scale * Me[a * nb + c] + Ke[a * nb + c];
                T.M.v[k] += Me[a * nb + c];
            }
    }
    T.dinv.resize(T.n);
    for (int i = 0; i < T.n; ++i) T.dinv[i] = 1.0 / T.A.v[T.A.find(i, i)];
    if (cfg->pc == ORC_PC_BJACOBI) ilu0_factor(T.A, T.ilu, T.ilu_diag);
    T.b.assign(T.n, 0.0);
    T.z.assign(T.n, 0.0);
    T.r.assign(T.n, 0.0);
    T.p.assign(T.n, 0.0);
    T.w.assign(T.n, 0.0);
    T.x.assign(T.n, 0.0);
    return h;
}

int orc_tissue_set_bidomain(orc_tissue* h, const double* xyz, int n_elems, const int* conn, const double* sigma_i,
                            const double* sigma_e, const int* fixed, int n_fixed) {
    Tissue& T = h->T;
    if (T.bido || T.steps != 0 || T.cfg.solver != ORC_SOLVER_MONODOMAIN || T.cfg.svi || T.cfg.mass_lumping ||
        T.cfg.pc == ORC_PC_BJACOBI || n_fixed < 0 || (n_fixed > 0 && !fixed))
        return -4;
    const int n = T.n, dim = T.dim, nb = dim + 1;
    for (int k = 0; k < n_fixed; ++k)
        if (fixed[k] < 0 || fixed[k] >= n) return -4;
    // pattern: rows 2i and 2i+1 both hold columns 2j, 2j+1 for every j of A's row i
    Csr& B = T.B;
    B.n = 2 * n;
    B.rp.assign(2 * n + 1, 0);
    for (int i = 0; i < n; ++i) {
        const int len = 2 * (T.A.rp[i + 1] - T.A.rp[i]);
        B.rp[2 * i + 1] = B.rp[2 * i] + len;
        B.rp[2 * i + 2] = B.rp[2 * i + 1] + len;
    }
    B.ci.resize(B.rp[2 * n]);
    for (int i = 0; i < n; ++i)
        for (int r = 0; r < 2; ++r) {
            int q = B.rp[2 * i + r];
            for (int k = T.A.rp[i]; k < T.A.rp[i + 1]; ++k) {
                B.ci[q++] = 2 * T.A.ci[k];
                B.ci[q++] = 2 * T.A.ci[k] + 1;
            }
        }
    B.v.assign(B.ci.size(), 0.0);
    const double ms = T.cfg.am * T.cfg.cm / T.cfg.dt_pde;
    for (int e = 0; e < n_elems; ++e) {
        double X[4 * 3];
        for (int a = 0; a < nb; ++a)
            for (int c = 0; c < 3; ++c) X[a * 3 + c] = xyz[(size_t)conn[e * nb + a] * 3 + c];
        double Me[16], Ki[16], Me2[16], Ke[16];
        if (!element_matrices(dim, X, sigma_i + (size_t)e * dim, false, Me, Ki) ||
            !element_matrices(dim, X, sigma_e + (size_t)e * dim, false, Me2, Ke))
            return -4;
        for (int a = 0; a < nb; ++a)
            for (int c = 0; c < nb; ++c) {
                const int i = conn[e * nb + a], j = conn[e * nb + c];
                const double ki = Ki[a * nb + c];
                B.v[B.find(2 * i, 2 * j)] += ms * Me[a * nb + c] + ki;
                B.v[B.find(2 * i, 2 * j + 1)] += ki;
                B.v[B.find(2 * i + 1, 2 * j)] += ki;
                B.v[B.find(2 * i + 1, 2 * j + 1)] += ki + Ke[a * nb + c];
            }
    }
    // fixed phi_e = 0: zero the row and the column, 1 on the diagonal
    std::vector<char> is_fixed(2 * n, 0);
    for (int k = 0; k < n_fixed; ++k) is_fixed[2 * fixed[k] + 1] = 1;
    for (int r = 0; r < 2 * n; ++r)
        for (int k = B.rp[r]; k < B.rp[r + 1]; ++k)
            if (is_fixed[r] || is_fixed[B.ci[k]]) B.v[k] = (B.ci[k] == r) ? 1.0 : 0.0;
    T.nullspace = n_fixed == 0;
    T.bdinv.resize(2 * n);
    for (int r = 0; r < 2 * n; ++r) T.bdinv[r] = 1.0 / B.v[B.find(r, r)];
    for (auto* v : {&T.bb, &T.br, &T.bz, &T.bp, &T.bw}) v->assign(2 * n, 0.0);
    T.bmz.assign(n, 0.0);
    T.u.assign(2 * n, 0.0);
    for (int i = 0; i < n; ++i) T.u[2 * i] = T.V[i];
    T.bido = true;
    return 0;
}

void orc_tissue_get_extracellular(const orc_tissue* h, double* phi) {
    for (int i = 0; i < h->T.n; ++i) phi[i] = h->T.bido ? h->T.u[2 * i + 1] : 0.0;
}

void orc_tissue_destroy(orc_tissue* t) { delete t; }

int orc_tissue_step(orc_tissue* h, int n, int* cg_iters) {
    for (int s = 0; s < n; ++s) {
        int it = 0;
        const int rc = step_once(h->T, &it);
        if (cg_iters) cg_iters[s] = it;
        if (rc != 0) return rc;
    }
    return 0;
}

double orc_tissue_time(const orc_tissue* h) { return h->T.t; }

void orc_tissue_get_voltage(const orc_tissue* h, double* v) {
    std::memcpy(v, h->T.V.data(), sizeof(double) * h->T.n);
}

void orc_tissue_get_states(const orc_tissue* h, double* s) {
    std::memcpy(s, h->T.states.data(), sizeof(double) * h->T.states.size());
    for (int i = 0; i < h->T.n; ++i) s[(size_t)i * h->T.ns] = h->T.V[i];
}

void orc_tissue_get_caches(const orc_tissue* h, double* iion, double* istim) {
    std::memcpy(iion, h->T.iion.data(), sizeof(double) * h->T.n);
    std::memcpy(istim, h->T.istim.data(), sizeof(double) * h->T.n);
}

int orc_tissue_matrix(const orc_tissue* h, int which, int* rowptr, int* cols, double* vals) {
    const Csr& C = which == 0 ? h->T.A : h->T.M;
    if (rowptr) std::memcpy(rowptr, C.rp.data(), sizeof(int) * (C.n + 1));
    if (cols) std::memcpy(cols, C.ci.data(), sizeof(int) * C.ci.size());
    if (vals) std::memcpy(vals, C.v.data(), sizeof(double) * C.v.size());
    return (int)C.ci.size();
}

}  // extern "C"

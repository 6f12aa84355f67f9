// CPU oracle, single-cell part -- test infrastructure only (see oracle.h).
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle.h"
#include "oracle_internal.h"

namespace orc {

// TimeStepper (global/src/TimeStepper.cpp:43-135): times are start + k*dt,
// snapped to the end when within epsilon; epsilon = DBL_EPSILON*end if end > 1.
TimeStepper::TimeStepper(double start, double end, double dt)
    : mStart(start), mEnd(end), mDt(dt), mSteps(0), mTime(start), mEps(DBL_EPSILON) {
    if (mEnd > 1.0) mEps = DBL_EPSILON * mEnd;
    mNext = CalcNext();
}

double TimeStepper::CalcNext() const {
    double next = mStart + (mSteps + 1) * mDt;
    if (mEnd - next <= mEps) next = mEnd;
    return next;
}

void TimeStepper::Advance() {
    mSteps++;
    mTime = mNext;
    mNext = CalcNext();
}

double stimulus_value(const orc_stimulus* s, double t) {
    if (!s) return 0.0;
    switch (s->kind) {
        case ORC_STIM_SIMPLE: {
            // SimpleStimulus.cpp:44-51 pads the duration by (dur+start)*eps
            const double dur = s->duration + (s->duration + s->start) * DBL_EPSILON;
            return (s->start <= t && t <= dur + s->start) ? s->magnitude : 0.0;
        }
        case ORC_STIM_REGULAR: {
            // RegularStimulus.cpp:43-81 pads the duration by period*eps
            const double dur = s->duration + s->period * DBL_EPSILON;
            if (t < s->start) return 0.0;
            const double beat = std::fmod(t - s->start, s->period);
            return (beat >= 0 && beat <= dur && t <= s->stop) ? s->magnitude : 0.0;
        }
        default:
            return 0.0;
    }
}

// EvaluateYDerivatives of a cell whose voltage derivative may be forced to zero
// (AbstractCardiacCell::SetVoltageDerivativeToZero).
template <class M>
static void derivs(const std::vector<double>& y, double stim, double cm, const double* p, bool zero_dv,
                   std::vector<double>& dy) {
    M::template rhs<double>(y.data(), stim, cm, p, dy.data());
    if (zero_dv) dy[0] = 0.0;
}

// GRL1IvpOdeSolver::CalculateNextYValue (ode/src/solver/GRL1IvpOdeSolver.cpp:47-93)
// and GRL2IvpOdeSolver::CalculateNextYValue (ode/src/solver/GRL2IvpOdeSolver.cpp:47-119),
// in the order those functions evaluate and perturb the state vector.
template <class M>
void grl_next(int method, double* yio, double stim, double cm, const double* p, double h, bool zero_dv) {
    const double delta = 1.0e-8;
    const int n = M::kNumStates;
    std::vector<double> cur(yio, yio + n), next(n), evalf(n), partial(n), temp(n);
    if (method == ORC_GRL1) {
        derivs<M>(cur, stim, cm, p, zero_dv, evalf);
        for (int i = 0; i < n; ++i) {
            const double t = cur[i];
            cur[i] = t + delta;
            derivs<M>(cur, stim, cm, p, zero_dv, temp);
            partial[i] = (temp[i] - evalf[i]) / delta;
            cur[i] = t;
        }
        for (int i = 0; i < n; ++i)
            next[i] = std::fabs(partial[i]) < delta ? cur[i] + evalf[i] * h
                                                    : cur[i] + (evalf[i] / partial[i]) * (std::exp(partial[i] * h) - 1);
    } else {
        next = cur;
        const std::vector<double> yinit = next;
        derivs<M>(next, stim, cm, p, zero_dv, evalf);
        for (int i = 0; i < n; ++i) {
            next[i] = next[i] + delta;
            derivs<M>(next, stim, cm, p, zero_dv, temp);
            partial[i] = (temp[i] - evalf[i]) / delta;
            next[i] = next[i] - delta;
        }
        for (int i = 0; i < n; ++i)   // midpoint
            next[i] = std::fabs(partial[i]) < delta ? next[i] + 0.5 * evalf[i] * h
                                                    : next[i] + (evalf[i] / partial[i]) * (std::exp(partial[i] * 0.5 * h) - 1);
        for (int i = 0; i < n; ++i) {
            const double ysave = next[i];
            next[i] = yinit[i];
            derivs<M>(next, stim, cm, p, zero_dv, temp);
            evalf[i] = temp[i];
            next[i] = next[i] + delta;
            derivs<M>(next, stim, cm, p, zero_dv, temp);
            partial[i] = (temp[i] - evalf[i]) / delta;
            next[i] = ysave;
        }
        for (int i = 0; i < n; ++i)
            next[i] = std::fabs(partial[i]) < delta ? yinit[i] + evalf[i] * h
                                                    : yinit[i] + (evalf[i] / partial[i]) * (std::exp(partial[i] * h) - 1);
    }
    for (int i = 0; i < n; ++i) yio[i] = next[i];
}

template void grl_next<chb::LuoRudy1991>(int, double*, double, double, const double*, double, bool);
template void grl_next<chb::TenTusscher2006Epi>(int, double*, double, double, const double*, double, bool);

// AbstractCardiacCell::ComputeExceptVoltage (heart/src/odes/AbstractCardiacCell.cpp:90-105)
// with a GRL1/GRL2 ODE solver: AbstractOneStepIvpOdeSolver::InternalSolve over
// TimeStepper steps, dV/dt forced to 0.
template <class M>
static void grl_except_voltage(int method, double* y, const double* p, const orc_stimulus* stim,
                               double am_div, double cm, double t0, double t1, double dt) {
    TimeStepper st(t0, t1, dt);
    while (!st.AtEnd()) {
        const double s = stimulus_value(stim, st.Time()) / am_div;
        grl_next<M>(method, y, s, cm, p, st.NextStep(), true);
        st.Advance();
    }
}

template <class M>
static void fe_except_voltage(double* y, const double* p, const orc_stimulus* stim,
                              double am_div, double cm, double t0, double t1, double dt) {
    // AbstractOneStepIvpOdeSolver::InternalSolve (.cpp:115-153) with Euler
    // (EulerIvpOdeSolver.cpp:38-57); dV/dt forced to 0 (SetVoltageDerivativeToZero).
    TimeStepper st(t0, t1, dt);
    double dy[M::kNumStates];
    while (!st.AtEnd()) {
        const double h = st.NextStep();
        const double s = stimulus_value(stim, st.Time()) / am_div;
        M::template rhs<double>(y, s, cm, p, dy);
        for (int i = 1; i < M::kNumStates; ++i) y[i] += h * dy[i];
        st.Advance();
    }
}

template <class M>
static void rl_except_voltage(double* y, const double* p, const orc_stimulus* stim,
                              double am_div, double cm, double t0, double t1, double dt) {
    // AbstractRushLarsenCardiacCell::ComputeExceptVoltage (.cpp:106-128): the
    // step length is the cell's mDt on every step.
    TimeStepper st(t0, t1, dt);
    while (!st.AtEnd()) {
        const double s = stimulus_value(stim, st.Time()) / am_div;
        chb::rl_step_except_voltage<M, double>(y, s, cm, p, dt);
        st.Advance();
    }
}

// AbstractBackwardEulerCardiacCell::ComputeExceptVoltage (heart/src/odes/
// AbstractBackwardEulerCardiacCell.hpp): n = (t1 - t0)/dt + 0.5 steps at times
// t0 + i dt, each ComputeOneStepExceptVoltage with V fixed.
template <class M>
static void be_except_voltage(double* y, const double* p, const orc_stimulus* stim,
                              double am_div, double cm, double t0, double t1, double dt) {
    const unsigned n_steps = (unsigned)((t1 - t0) / dt + 0.5);
    const double v = y[0];
    for (unsigned i = 0; i < n_steps; ++i) {
        const double s = stimulus_value(stim, t0 + i * dt) / am_div;
        chb::be_step<M, double>(y, s, cm, p, dt, false);
        y[0] = v;
    }
}

template <class M>
void except_voltage(int method, double* y, const double* p, const orc_stimulus* stim,
                    double am_div, double cm, double t0, double t1, double dt) {
    if (method == ORC_RL) rl_except_voltage<M>(y, p, stim, am_div, cm, t0, t1, dt);
    else if (method == ORC_BE) be_except_voltage<M>(y, p, stim, am_div, cm, t0, t1, dt);
    else if (method == ORC_GRL1 || method == ORC_GRL2) grl_except_voltage<M>(method, y, p, stim, am_div, cm, t0, t1, dt);
    else fe_except_voltage<M>(y, p, stim, am_div, cm, t0, t1, dt);
}

template void except_voltage<chb::LuoRudy1991>(int, double*, const double*, const orc_stimulus*,
                                               double, double, double, double, double);
template void except_voltage<chb::TenTusscher2006Epi>(int, double*, const double*,
                                                      const orc_stimulus*, double, double,
                                                      double, double, double);

template <class M>
static int compute(int method, double* y, const double* p, const orc_stimulus* stim,
                   double cm, double t0, double t1, double dt, double tsamp,
                   double* samples, int max_samples) {
    const int n = M::kNumStates;
    if (tsamp < dt) tsamp = dt;
    int ns = 0;
    auto record = [&]() {
        if (samples && ns < max_samples) std::memcpy(samples + (size_t)ns * n, y, n * sizeof(double));
        ns++;
    };
    record();
    double dy[M::kNumStates];
    if (method == ORC_FE || method == ORC_GRL1 || method == ORC_GRL2) {
        // AbstractOneStepIvpOdeSolver::Solve with sampling (.cpp:41-91)
        TimeStepper outer(t0, t1, tsamp);
        while (!outer.AtEnd()) {
            TimeStepper inner(outer.Time(), outer.Next(), dt);
            while (!inner.AtEnd()) {
                const double h = inner.NextStep();
                const double s = stimulus_value(stim, inner.Time());
                if (method == ORC_FE) {
                    M::template rhs<double>(y, s, cm, p, dy);
                    for (int i = 0; i < n; ++i) y[i] += h * dy[i];
                } else {
                    grl_next<M>(method, y, s, cm, p, h, false);
                }
                inner.Advance();
            }
            outer.Advance();
            record();
        }
    } else {
        // AbstractRushLarsenCardiacCell::Compute (.cpp:57-104)
        const unsigned n_steps = (unsigned)std::floor((t1 - t0) / tsamp + 0.5);
        const unsigned n_small = (unsigned)std::floor(tsamp / dt + 0.5);
        for (unsigned i = 0; i < n_steps; ++i) {
            for (unsigned j = 0; j < n_small; ++j) {
                const double t = t0 + i * tsamp + j * dt;
                const double s = stimulus_value(stim, t);
                chb::rl_step<M, double>(y, s, cm, p, dt);
            }
            record();
        }
    }
    return ns;
}

template <class M>
static void defaults(double* p) {
    for (int i = 0; i < M::kNumParams; ++i) p[i] = 1.0;
}

}  // namespace orc

using namespace orc;

extern "C" {

int orc_num_states(int model) {
    return model == ORC_TT06 ? chb::TenTusscher2006Epi::kNumStates : chb::LuoRudy1991::kNumStates;
}

int orc_num_params(int model) {
    return model == ORC_TT06 ? chb::TenTusscher2006Epi::kNumParams : chb::LuoRudy1991::kNumParams;
}

void orc_initial_states(int model, double* y) {
    if (model == ORC_TT06)
        for (int i = 0; i < chb::TenTusscher2006Epi::kNumStates; ++i)
            y[i] = chb::TenTusscher2006Epi::kInitialStates[i];
    else
        for (int i = 0; i < chb::LuoRudy1991::kNumStates; ++i)
            y[i] = chb::LuoRudy1991::kInitialStates[i];
}

double orc_stimulus_value(const orc_stimulus* s, double t) { return stimulus_value(s, t); }

int orc_cell_compute(int model, int method, double* y, const double* params,
                     const orc_stimulus* stim, double cm, double t0, double t1, double dt,
                     double tsamp, double* samples, int max_samples) {
    double p[16];
    if (model == ORC_TT06) {
        defaults<chb::TenTusscher2006Epi>(p);
        if (params) std::memcpy(p, params, sizeof(double) * chb::TenTusscher2006Epi::kNumParams);
        return compute<chb::TenTusscher2006Epi>(method, y, p, stim, cm, t0, t1, dt, tsamp, samples,
                                                max_samples);
    }
    defaults<chb::LuoRudy1991>(p);
    if (params) std::memcpy(p, params, sizeof(double) * chb::LuoRudy1991::kNumParams);
    return compute<chb::LuoRudy1991>(method, y, p, stim, cm, t0, t1, dt, tsamp, samples, max_samples);
}

double orc_cell_iionic(int model, const double* y, const double* params, double cm) {
    double p[16];
    if (model == ORC_TT06) {
        defaults<chb::TenTusscher2006Epi>(p);
        if (params) std::memcpy(p, params, sizeof(double) * chb::TenTusscher2006Epi::kNumParams);
        return chb::TenTusscher2006Epi::iionic<double>(y, cm, p);
    }
    defaults<chb::LuoRudy1991>(p);
    if (params) std::memcpy(p, params, sizeof(double) * chb::LuoRudy1991::kNumParams);
    return chb::LuoRudy1991::iionic<double>(y, cm, p);
}

double orc_cell_compute_except_voltage(int model, int method, double* y, const double* params,
                                       const orc_stimulus* stim, double am_for_tissue, double cm,
                                       double t0, double t1, double dt) {
    double p[16];
    const double am_div = am_for_tissue > 0 ? am_for_tissue : 1.0;
    if (model == ORC_TT06) {
        defaults<chb::TenTusscher2006Epi>(p);
        if (params) std::memcpy(p, params, sizeof(double) * chb::TenTusscher2006Epi::kNumParams);
        except_voltage<chb::TenTusscher2006Epi>(method, y, p, stim, am_div, cm, t0, t1, dt);
        return chb::TenTusscher2006Epi::iionic<double>(y, cm, p);
    }
    defaults<chb::LuoRudy1991>(p);
    if (params) std::memcpy(p, params, sizeof(double) * chb::LuoRudy1991::kNumParams);
    except_voltage<chb::LuoRudy1991>(method, y, p, stim, am_div, cm, t0, t1, dt);
    return chb::LuoRudy1991::iionic<double>(y, cm, p);
}

}  // extern "C"

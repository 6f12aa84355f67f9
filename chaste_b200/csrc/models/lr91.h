// Generated by chaste_b200/codegen/emit.py from heart/src/odes/cellml/LuoRudy1991.cellml.
// Do not edit: re-run `python -m chaste_b200.codegen.emit` instead.
#pragma once
#include "cellmodel_common.h"

namespace chb {

struct LuoRudy1991 {
    static constexpr const char* kName = "luo_rudy_1991";
    static constexpr int kNumStates = 8;
    static constexpr int kNumParams = 6;
    static constexpr bool kCurrentPerCapacitance = false;
    static constexpr double kInitialStates[8] = {-83.853, 0.00187018, 0.9804713, 0.98767124, 0.00316354, 0.99427859, 0.16647703, 0.0002};
    static constexpr const char* kStateNames[8] = {"V", "m", "h", "j", "d", "f", "X", "Cai"};
    static constexpr const char* kParamNames[6] = {"g_Na", "g_si", "g_K", "g_K1", "g_Kp", "g_b"};
    // 1 where the state is advanced by Rush-Larsen (ODE affine in itself)
    static constexpr bool kRushLarsen[8] = {false, true, true, true, true, true, true, false};
    CHB_HD static constexpr bool rush_larsen(int i) { return i == 1 || i == 2 || i == 3 || i == 4 || i == 5 || i == 6; }
    // range class per state: 1 gate in [0,1], 2 concentration > 0, 0 unchecked
    static constexpr int kRangeClass[8] = {0, 1, 1, 1, 1, 1, 1, 2};
    CHB_HD static constexpr int range_class(int i) { return (i == 1 || i == 2 || i == 3 || i == 4 || i == 5 || i == 6) ? 1 : ((i == 7) ? 2 : 0); }

    // dy/dt for every state at (y, stim) where stim is the Chaste area stimulus
    // in uA/cm^2 and cm the Chaste capacitance in uF/cm^2.  y[0] is the voltage.
    template <typename T>
    CHB_HD static void rhs(const T* __restrict__ y, T stim, T cm,
                                  const T* __restrict__ p, T* __restrict__ dy) {
        (void)stim; (void)cm; (void)p;
        const T v_background_current__i_b = ((T(0.03921)*p[5])*(y[0] - (-T(59.87))));
        const T v_fast_sodium_current__i_Na = ((T(23.0)*p[0])*(y[1]*y[1]*y[1])*y[2]*y[3]*(y[0] - T(54.79446393509185)));
        const T v_membrane__I_stim = stim;
        const T v_plateau_potassium_current__Kp = (m_div(T(1.0), (T(1.0) + m_exp((m_divk((T(7.488) - y[0]), T(5.98), T(0.16722408026755853)))))));
        const T v_plateau_potassium_current__i_Kp = ((T(0.0183)*p[4])*v_plateau_potassium_current__Kp*(y[0] - (-T(87.8929017138025))));
        const T v_slow_inward_current__E_si = (T(7.7) - (T(13.0287)*m_log((m_divk(y[7], T(1.0), T(1.0))))));
        const T v_slow_inward_current__i_si = ((T(0.09)*p[1])*y[4]*y[5]*(y[0] - v_slow_inward_current__E_si));
        const T v_time_dependent_potassium_current_Xi_gate__Xi = ((y[0] > (-T(100.0))) ? (((chb::singularity_offset<T>()*T(1.0)) > fabs((y[0] + T(77.0)))) ? ((m_div((T(2.837)*(m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0))), (((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(35.0))))))) + (m_div((y[0] - (-T(77.0) - (chb::singularity_offset<T>()*T(1.0))))*((m_div((T(2.837)*(m_exp((T(0.04)*((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0))), (((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(35.0))))))) - (m_div((T(2.837)*(m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0))), (((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(35.0)))))))), (T(2.0)*(chb::singularity_offset<T>()*T(1.0)))))) : (m_div((T(2.837)*(m_exp((T(0.04)*(y[0] + T(77.0)))) - T(1.0))), ((y[0] + T(77.0))*m_exp((T(0.04)*(y[0] + T(35.0)))))))) : T(1.0));
        const T v_time_dependent_potassium_current__g_K__scaled = (T(0.282)*p[2]);
        const T v_time_dependent_potassium_current__i_K = (v_time_dependent_potassium_current__g_K__scaled*y[6]*v_time_dependent_potassium_current_Xi_gate__Xi*(y[0] - (-T(77.56758438531939))));
        const T v_time_independent_potassium_current_K1_gate__alpha_K1 = (m_div(T(1.02), (T(1.0) + m_exp((T(0.2385)*((y[0] - (-T(87.8929017138025))) - T(59.215)))))));
        const T v_time_independent_potassium_current_K1_gate__beta_K1 = (m_div(((T(0.49124)*m_exp((T(0.08032)*((y[0] + T(5.476)) - (-T(87.8929017138025)))))) + (T(1.0)*m_exp((T(0.06175)*(y[0] - (-T(87.8929017138025) + T(594.31))))))), (T(1.0) + m_exp(((-T(0.5143))*((y[0] - (-T(87.8929017138025))) + T(4.753)))))));
        const T v_time_independent_potassium_current_K1_gate__K1_infinity = (m_div(v_time_independent_potassium_current_K1_gate__alpha_K1, (v_time_independent_potassium_current_K1_gate__alpha_K1 + v_time_independent_potassium_current_K1_gate__beta_K1)));
        const T v_time_independent_potassium_current__g_K1__scaled = (T(0.6047)*p[3]);
        const T v_time_independent_potassium_current__i_K1 = (v_time_independent_potassium_current__g_K1__scaled*v_time_independent_potassium_current_K1_gate__K1_infinity*(y[0] - (-T(87.8929017138025))));
        const T v_fast_sodium_current_m_gate__alpha_m = (((chb::singularity_offset<T>()*T(10.0)) > fabs((y[0] + T(47.13)))) ? ((m_div((T(0.32)*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13))), (T(1.0) - m_exp(((-T(0.1))*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13))))))) + (m_div((y[0] - (-T(47.13) - (chb::singularity_offset<T>()*T(10.0))))*((m_div((T(0.32)*((-T(47.13) + (chb::singularity_offset<T>()*T(10.0))) + T(47.13))), (T(1.0) - m_exp(((-T(0.1))*((-T(47.13) + (chb::singularity_offset<T>()*T(10.0))) + T(47.13))))))) - (m_div((T(0.32)*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13))), (T(1.0) - m_exp(((-T(0.1))*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13)))))))), (T(2.0)*(chb::singularity_offset<T>()*T(10.0)))))) : (m_div((T(0.32)*(y[0] + T(47.13))), (T(1.0) - m_exp(((-T(0.1))*(y[0] + T(47.13))))))));
        const T v_fast_sodium_current_m_gate__beta_m = (T(0.08)*m_exp((m_divk((-y[0]), T(11.0), T(0.09090909090909091)))));
        const T v_fast_sodium_current_h_gate__alpha_h = ((y[0] < (-T(40.0))) ? (T(0.135)*m_exp((m_div((T(80.0) + y[0]), (-T(6.8)))))) : T(0.0));
        const T v_fast_sodium_current_h_gate__beta_h = ((y[0] < (-T(40.0))) ? ((T(3.56)*m_exp((T(0.079)*y[0]))) + (T(310000.0)*m_exp((T(0.35)*y[0])))) : (m_div(T(1.0), (T(0.13)*(T(1.0) + m_exp((m_div((y[0] + T(10.66)), (-T(11.1))))))))));
        const T v_fast_sodium_current_j_gate__alpha_j = ((y[0] < (-T(40.0))) ? (m_div(((((-T(127140.0))*m_exp((T(0.2444)*y[0]))) - (T(3.474e-05)*m_exp(((-T(0.04391))*y[0]))))*(y[0] + T(37.78))), (T(1.0) + m_exp((T(0.311)*(y[0] + T(79.23))))))) : T(0.0));
        const T v_fast_sodium_current_j_gate__beta_j = ((y[0] < (-T(40.0))) ? (m_div((T(0.1212)*m_exp(((-T(0.01052))*y[0]))), (T(1.0) + m_exp(((-T(0.1378))*(y[0] + T(40.14))))))) : (m_div((T(0.3)*m_exp(((-T(2.535e-07))*y[0]))), (T(1.0) + m_exp(((-T(0.1))*(y[0] + T(32.0))))))));
        const T v_slow_inward_current_d_gate__alpha_d = (m_div((T(0.095)*m_exp(((-T(0.01))*(y[0] - T(5.0))))), (T(1.0) + m_exp(((-T(0.072))*(y[0] - T(5.0)))))));
        const T v_slow_inward_current_d_gate__beta_d = (m_div((T(0.07)*m_exp(((-T(0.017))*(y[0] + T(44.0))))), (T(1.0) + m_exp((T(0.05)*(y[0] + T(44.0)))))));
        const T v_slow_inward_current_f_gate__alpha_f = (m_div((T(0.012)*m_exp(((-T(0.008))*(y[0] + T(28.0))))), (T(1.0) + m_exp((T(0.15)*(y[0] + T(28.0)))))));
        const T v_slow_inward_current_f_gate__beta_f = (m_div((T(0.0065)*m_exp(((-T(0.02))*(y[0] + T(30.0))))), (T(1.0) + m_exp(((-T(0.2))*(y[0] + T(30.0)))))));
        const T v_time_dependent_potassium_current_X_gate__alpha_X = (m_div((T(0.0005)*m_exp((T(0.083)*(y[0] + T(50.0))))), (T(1.0) + m_exp((T(0.057)*(y[0] + T(50.0)))))));
        const T v_time_dependent_potassium_current_X_gate__beta_X = (m_div((T(0.0013)*m_exp(((-T(0.06))*(y[0] + T(20.0))))), (T(1.0) + m_exp(((-T(0.04))*(y[0] + T(20.0)))))));
        dy[0] = ((m_divk((-T(1.0)), T(1.0), T(1.0)))*(v_membrane__I_stim + v_fast_sodium_current__i_Na + v_slow_inward_current__i_si + v_time_dependent_potassium_current__i_K + v_time_independent_potassium_current__i_K1 + v_plateau_potassium_current__i_Kp + v_background_current__i_b));
        dy[1] = ((v_fast_sodium_current_m_gate__alpha_m*(T(1.0) - y[1])) - (v_fast_sodium_current_m_gate__beta_m*y[1]));
        dy[2] = ((v_fast_sodium_current_h_gate__alpha_h*(T(1.0) - y[2])) - (v_fast_sodium_current_h_gate__beta_h*y[2]));
        dy[3] = ((v_fast_sodium_current_j_gate__alpha_j*(T(1.0) - y[3])) - (v_fast_sodium_current_j_gate__beta_j*y[3]));
        dy[4] = ((v_slow_inward_current_d_gate__alpha_d*(T(1.0) - y[4])) - (v_slow_inward_current_d_gate__beta_d*y[4]));
        dy[5] = ((v_slow_inward_current_f_gate__alpha_f*(T(1.0) - y[5])) - (v_slow_inward_current_f_gate__beta_f*y[5]));
        dy[6] = ((v_time_dependent_potassium_current_X_gate__alpha_X*(T(1.0) - y[6])) - (v_time_dependent_potassium_current_X_gate__beta_X*y[6]));
        dy[7] = (((m_divk((-T(0.0001)), T(1.0), T(1.0)))*v_slow_inward_current__i_si) + (T(0.07)*(T(0.0001) - y[7])));
    }

    // Rush-Larsen terms: for RL states inf[i] is the fixed point and rate[i]
    // the (negative) affine coefficient h so y' = inf + (y - inf)*exp(h*dt);
    // for the other states rate[i] holds dy/dt.  rate[0] is dV/dt.
    template <typename T>
    CHB_HD static void rl_terms(const T* __restrict__ y, T stim, T cm,
                                       const T* __restrict__ p, T* __restrict__ rate,
                                       T* __restrict__ inf) {
        (void)stim; (void)cm; (void)p; (void)inf;
        const T v_background_current__i_b = ((T(0.03921)*p[5])*(y[0] - (-T(59.87))));
        const T v_fast_sodium_current__i_Na = ((T(23.0)*p[0])*(y[1]*y[1]*y[1])*y[2]*y[3]*(y[0] - T(54.79446393509185)));
        const T v_membrane__I_stim = stim;
        const T v_plateau_potassium_current__Kp = (m_div(T(1.0), (T(1.0) + m_exp((m_divk((T(7.488) - y[0]), T(5.98), T(0.16722408026755853)))))));
        const T v_plateau_potassium_current__i_Kp = ((T(0.0183)*p[4])*v_plateau_potassium_current__Kp*(y[0] - (-T(87.8929017138025))));
        const T v_slow_inward_current__E_si = (T(7.7) - (T(13.0287)*m_log((m_divk(y[7], T(1.0), T(1.0))))));
        const T v_slow_inward_current__i_si = ((T(0.09)*p[1])*y[4]*y[5]*(y[0] - v_slow_inward_current__E_si));
        const T v_time_dependent_potassium_current_Xi_gate__Xi = ((y[0] > (-T(100.0))) ? (((chb::singularity_offset<T>()*T(1.0)) > fabs((y[0] + T(77.0)))) ? ((m_div((T(2.837)*(m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0))), (((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(35.0))))))) + (m_div((y[0] - (-T(77.0) - (chb::singularity_offset<T>()*T(1.0))))*((m_div((T(2.837)*(m_exp((T(0.04)*((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0))), (((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(35.0))))))) - (m_div((T(2.837)*(m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0))), (((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(35.0)))))))), (T(2.0)*(chb::singularity_offset<T>()*T(1.0)))))) : (m_div((T(2.837)*(m_exp((T(0.04)*(y[0] + T(77.0)))) - T(1.0))), ((y[0] + T(77.0))*m_exp((T(0.04)*(y[0] + T(35.0)))))))) : T(1.0));
        const T v_time_dependent_potassium_current__g_K__scaled = (T(0.282)*p[2]);
        const T v_time_dependent_potassium_current__i_K = (v_time_dependent_potassium_current__g_K__scaled*y[6]*v_time_dependent_potassium_current_Xi_gate__Xi*(y[0] - (-T(77.56758438531939))));
        const T v_time_independent_potassium_current_K1_gate__alpha_K1 = (m_div(T(1.02), (T(1.0) + m_exp((T(0.2385)*((y[0] - (-T(87.8929017138025))) - T(59.215)))))));
        const T v_time_independent_potassium_current_K1_gate__beta_K1 = (m_div(((T(0.49124)*m_exp((T(0.08032)*((y[0] + T(5.476)) - (-T(87.8929017138025)))))) + (T(1.0)*m_exp((T(0.06175)*(y[0] - (-T(87.8929017138025) + T(594.31))))))), (T(1.0) + m_exp(((-T(0.5143))*((y[0] - (-T(87.8929017138025))) + T(4.753)))))));
        const T v_time_independent_potassium_current_K1_gate__K1_infinity = (m_div(v_time_independent_potassium_current_K1_gate__alpha_K1, (v_time_independent_potassium_current_K1_gate__alpha_K1 + v_time_independent_potassium_current_K1_gate__beta_K1)));
        const T v_time_independent_potassium_current__g_K1__scaled = (T(0.6047)*p[3]);
        const T v_time_independent_potassium_current__i_K1 = (v_time_independent_potassium_current__g_K1__scaled*v_time_independent_potassium_current_K1_gate__K1_infinity*(y[0] - (-T(87.8929017138025))));
        const T v_fast_sodium_current_m_gate__alpha_m = (((chb::singularity_offset<T>()*T(10.0)) > fabs((y[0] + T(47.13)))) ? ((m_div((T(0.32)*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13))), (T(1.0) - m_exp(((-T(0.1))*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13))))))) + (m_div((y[0] - (-T(47.13) - (chb::singularity_offset<T>()*T(10.0))))*((m_div((T(0.32)*((-T(47.13) + (chb::singularity_offset<T>()*T(10.0))) + T(47.13))), (T(1.0) - m_exp(((-T(0.1))*((-T(47.13) + (chb::singularity_offset<T>()*T(10.0))) + T(47.13))))))) - (m_div((T(0.32)*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13))), (T(1.0) - m_exp(((-T(0.1))*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13)))))))), (T(2.0)*(chb::singularity_offset<T>()*T(10.0)))))) : (m_div((T(0.32)*(y[0] + T(47.13))), (T(1.0) - m_exp(((-T(0.1))*(y[0] + T(47.13))))))));
        const T v_fast_sodium_current_m_gate__beta_m = (T(0.08)*m_exp((m_divk((-y[0]), T(11.0), T(0.09090909090909091)))));
        const T v_fast_sodium_current_h_gate__alpha_h = ((y[0] < (-T(40.0))) ? (T(0.135)*m_exp((m_div((T(80.0) + y[0]), (-T(6.8)))))) : T(0.0));
        const T v_fast_sodium_current_h_gate__beta_h = ((y[0] < (-T(40.0))) ? ((T(3.56)*m_exp((T(0.079)*y[0]))) + (T(310000.0)*m_exp((T(0.35)*y[0])))) : (m_div(T(1.0), (T(0.13)*(T(1.0) + m_exp((m_div((y[0] + T(10.66)), (-T(11.1))))))))));
        const T v_fast_sodium_current_j_gate__alpha_j = ((y[0] < (-T(40.0))) ? (m_div(((((-T(127140.0))*m_exp((T(0.2444)*y[0]))) - (T(3.474e-05)*m_exp(((-T(0.04391))*y[0]))))*(y[0] + T(37.78))), (T(1.0) + m_exp((T(0.311)*(y[0] + T(79.23))))))) : T(0.0));
        const T v_fast_sodium_current_j_gate__beta_j = ((y[0] < (-T(40.0))) ? (m_div((T(0.1212)*m_exp(((-T(0.01052))*y[0]))), (T(1.0) + m_exp(((-T(0.1378))*(y[0] + T(40.14))))))) : (m_div((T(0.3)*m_exp(((-T(2.535e-07))*y[0]))), (T(1.0) + m_exp(((-T(0.1))*(y[0] + T(32.0))))))));
        const T v_slow_inward_current_d_gate__alpha_d = (m_div((T(0.095)*m_exp(((-T(0.01))*(y[0] - T(5.0))))), (T(1.0) + m_exp(((-T(0.072))*(y[0] - T(5.0)))))));
        const T v_slow_inward_current_d_gate__beta_d = (m_div((T(0.07)*m_exp(((-T(0.017))*(y[0] + T(44.0))))), (T(1.0) + m_exp((T(0.05)*(y[0] + T(44.0)))))));
        const T v_slow_inward_current_f_gate__alpha_f = (m_div((T(0.012)*m_exp(((-T(0.008))*(y[0] + T(28.0))))), (T(1.0) + m_exp((T(0.15)*(y[0] + T(28.0)))))));
        const T v_slow_inward_current_f_gate__beta_f = (m_div((T(0.0065)*m_exp(((-T(0.02))*(y[0] + T(30.0))))), (T(1.0) + m_exp(((-T(0.2))*(y[0] + T(30.0)))))));
        const T v_time_dependent_potassium_current_X_gate__alpha_X = (m_div((T(0.0005)*m_exp((T(0.083)*(y[0] + T(50.0))))), (T(1.0) + m_exp((T(0.057)*(y[0] + T(50.0)))))));
        const T v_time_dependent_potassium_current_X_gate__beta_X = (m_div((T(0.0013)*m_exp(((-T(0.06))*(y[0] + T(20.0))))), (T(1.0) + m_exp(((-T(0.04))*(y[0] + T(20.0)))))));
        rate[0] = ((m_divk((-T(1.0)), T(1.0), T(1.0)))*(v_membrane__I_stim + v_fast_sodium_current__i_Na + v_slow_inward_current__i_si + v_time_dependent_potassium_current__i_K + v_time_independent_potassium_current__i_K1 + v_plateau_potassium_current__i_Kp + v_background_current__i_b));
        inf[1] = (-m_div(v_fast_sodium_current_m_gate__alpha_m, (-v_fast_sodium_current_m_gate__alpha_m - v_fast_sodium_current_m_gate__beta_m)));
        rate[1] = (-v_fast_sodium_current_m_gate__alpha_m - v_fast_sodium_current_m_gate__beta_m);
        inf[2] = (-m_div(v_fast_sodium_current_h_gate__alpha_h, (-v_fast_sodium_current_h_gate__alpha_h - v_fast_sodium_current_h_gate__beta_h)));
        rate[2] = (-v_fast_sodium_current_h_gate__alpha_h - v_fast_sodium_current_h_gate__beta_h);
        inf[3] = (-m_div(v_fast_sodium_current_j_gate__alpha_j, (-v_fast_sodium_current_j_gate__alpha_j - v_fast_sodium_current_j_gate__beta_j)));
        rate[3] = (-v_fast_sodium_current_j_gate__alpha_j - v_fast_sodium_current_j_gate__beta_j);
        inf[4] = (-m_div(v_slow_inward_current_d_gate__alpha_d, (-v_slow_inward_current_d_gate__alpha_d - v_slow_inward_current_d_gate__beta_d)));
        rate[4] = (-v_slow_inward_current_d_gate__alpha_d - v_slow_inward_current_d_gate__beta_d);
        inf[5] = (-m_div(v_slow_inward_current_f_gate__alpha_f, (-v_slow_inward_current_f_gate__alpha_f - v_slow_inward_current_f_gate__beta_f)));
        rate[5] = (-v_slow_inward_current_f_gate__alpha_f - v_slow_inward_current_f_gate__beta_f);
        inf[6] = (-m_div(v_time_dependent_potassium_current_X_gate__alpha_X, (-v_time_dependent_potassium_current_X_gate__alpha_X - v_time_dependent_potassium_current_X_gate__beta_X)));
        rate[6] = (-v_time_dependent_potassium_current_X_gate__alpha_X - v_time_dependent_potassium_current_X_gate__beta_X);
        rate[7] = (((m_divk((-T(0.0001)), T(1.0), T(1.0)))*v_slow_inward_current__i_si) + (T(0.07)*(T(0.0001) - y[7])));
    }

    // Rush-Larsen states whose (inf, rate) depend on the voltage alone (and the
    // parameters): with V clamped over a PDE step (ComputeExceptVoltage) their terms,
    // and so exp(rate*dt), are the same in every substep.
    static constexpr bool kRlVoltageOnly[8] = {false, true, true, true, true, true, true, false};
    CHB_HD static constexpr bool rl_voltage_only(int i) { return i == 1 || i == 2 || i == 3 || i == 4 || i == 5 || i == 6; }
    static constexpr int kNumVoltageGates = 6;
    // rl_terms of the voltage-only Rush-Larsen states (reads y[0] and p only).
    template <typename T>
    CHB_HD static void rl_terms_voltage(const T* __restrict__ y, const T* __restrict__ p,
                                       T* __restrict__ rate, T* __restrict__ inf) {
        (void)p;
        const T v_fast_sodium_current_m_gate__alpha_m = (((chb::singularity_offset<T>()*T(10.0)) > fabs((y[0] + T(47.13)))) ? ((m_div((T(0.32)*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13))), (T(1.0) - m_exp(((-T(0.1))*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13))))))) + (m_div((y[0] - (-T(47.13) - (chb::singularity_offset<T>()*T(10.0))))*((m_div((T(0.32)*((-T(47.13) + (chb::singularity_offset<T>()*T(10.0))) + T(47.13))), (T(1.0) - m_exp(((-T(0.1))*((-T(47.13) + (chb::singularity_offset<T>()*T(10.0))) + T(47.13))))))) - (m_div((T(0.32)*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13))), (T(1.0) - m_exp(((-T(0.1))*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13)))))))), (T(2.0)*(chb::singularity_offset<T>()*T(10.0)))))) : (m_div((T(0.32)*(y[0] + T(47.13))), (T(1.0) - m_exp(((-T(0.1))*(y[0] + T(47.13))))))));
        const T v_fast_sodium_current_m_gate__beta_m = (T(0.08)*m_exp((m_divk((-y[0]), T(11.0), T(0.09090909090909091)))));
        const T v_fast_sodium_current_h_gate__alpha_h = ((y[0] < (-T(40.0))) ? (T(0.135)*m_exp((m_div((T(80.0) + y[0]), (-T(6.8)))))) : T(0.0));
        const T v_fast_sodium_current_h_gate__beta_h = ((y[0] < (-T(40.0))) ? ((T(3.56)*m_exp((T(0.079)*y[0]))) + (T(310000.0)*m_exp((T(0.35)*y[0])))) : (m_div(T(1.0), (T(0.13)*(T(1.0) + m_exp((m_div((y[0] + T(10.66)), (-T(11.1))))))))));
        const T v_fast_sodium_current_j_gate__alpha_j = ((y[0] < (-T(40.0))) ? (m_div(((((-T(127140.0))*m_exp((T(0.2444)*y[0]))) - (T(3.474e-05)*m_exp(((-T(0.04391))*y[0]))))*(y[0] + T(37.78))), (T(1.0) + m_exp((T(0.311)*(y[0] + T(79.23))))))) : T(0.0));
        const T v_fast_sodium_current_j_gate__beta_j = ((y[0] < (-T(40.0))) ? (m_div((T(0.1212)*m_exp(((-T(0.01052))*y[0]))), (T(1.0) + m_exp(((-T(0.1378))*(y[0] + T(40.14))))))) : (m_div((T(0.3)*m_exp(((-T(2.535e-07))*y[0]))), (T(1.0) + m_exp(((-T(0.1))*(y[0] + T(32.0))))))));
        const T v_slow_inward_current_d_gate__alpha_d = (m_div((T(0.095)*m_exp(((-T(0.01))*(y[0] - T(5.0))))), (T(1.0) + m_exp(((-T(0.072))*(y[0] - T(5.0)))))));
        const T v_slow_inward_current_d_gate__beta_d = (m_div((T(0.07)*m_exp(((-T(0.017))*(y[0] + T(44.0))))), (T(1.0) + m_exp((T(0.05)*(y[0] + T(44.0)))))));
        const T v_slow_inward_current_f_gate__alpha_f = (m_div((T(0.012)*m_exp(((-T(0.008))*(y[0] + T(28.0))))), (T(1.0) + m_exp((T(0.15)*(y[0] + T(28.0)))))));
        const T v_slow_inward_current_f_gate__beta_f = (m_div((T(0.0065)*m_exp(((-T(0.02))*(y[0] + T(30.0))))), (T(1.0) + m_exp(((-T(0.2))*(y[0] + T(30.0)))))));
        const T v_time_dependent_potassium_current_X_gate__alpha_X = (m_div((T(0.0005)*m_exp((T(0.083)*(y[0] + T(50.0))))), (T(1.0) + m_exp((T(0.057)*(y[0] + T(50.0)))))));
        const T v_time_dependent_potassium_current_X_gate__beta_X = (m_div((T(0.0013)*m_exp(((-T(0.06))*(y[0] + T(20.0))))), (T(1.0) + m_exp(((-T(0.04))*(y[0] + T(20.0)))))));
        inf[1] = (-m_div(v_fast_sodium_current_m_gate__alpha_m, (-v_fast_sodium_current_m_gate__alpha_m - v_fast_sodium_current_m_gate__beta_m)));
        rate[1] = (-v_fast_sodium_current_m_gate__alpha_m - v_fast_sodium_current_m_gate__beta_m);
        inf[2] = (-m_div(v_fast_sodium_current_h_gate__alpha_h, (-v_fast_sodium_current_h_gate__alpha_h - v_fast_sodium_current_h_gate__beta_h)));
        rate[2] = (-v_fast_sodium_current_h_gate__alpha_h - v_fast_sodium_current_h_gate__beta_h);
        inf[3] = (-m_div(v_fast_sodium_current_j_gate__alpha_j, (-v_fast_sodium_current_j_gate__alpha_j - v_fast_sodium_current_j_gate__beta_j)));
        rate[3] = (-v_fast_sodium_current_j_gate__alpha_j - v_fast_sodium_current_j_gate__beta_j);
        inf[4] = (-m_div(v_slow_inward_current_d_gate__alpha_d, (-v_slow_inward_current_d_gate__alpha_d - v_slow_inward_current_d_gate__beta_d)));
        rate[4] = (-v_slow_inward_current_d_gate__alpha_d - v_slow_inward_current_d_gate__beta_d);
        inf[5] = (-m_div(v_slow_inward_current_f_gate__alpha_f, (-v_slow_inward_current_f_gate__alpha_f - v_slow_inward_current_f_gate__beta_f)));
        rate[5] = (-v_slow_inward_current_f_gate__alpha_f - v_slow_inward_current_f_gate__beta_f);
        inf[6] = (-m_div(v_time_dependent_potassium_current_X_gate__alpha_X, (-v_time_dependent_potassium_current_X_gate__alpha_X - v_time_dependent_potassium_current_X_gate__beta_X)));
        rate[6] = (-v_time_dependent_potassium_current_X_gate__alpha_X - v_time_dependent_potassium_current_X_gate__beta_X);
    }
    // rl_terms of every state but the voltage-only gates (dV/dt in rate[0]).
    template <typename T>
    CHB_HD static void rl_terms_states(const T* __restrict__ y, T stim, T cm,
                                       const T* __restrict__ p, T* __restrict__ rate,
                                       T* __restrict__ inf) {
        (void)stim; (void)cm; (void)p; (void)inf;
        const T v_background_current__i_b = ((T(0.03921)*p[5])*(y[0] - (-T(59.87))));
        const T v_fast_sodium_current__i_Na = ((T(23.0)*p[0])*(y[1]*y[1]*y[1])*y[2]*y[3]*(y[0] - T(54.79446393509185)));
        const T v_membrane__I_stim = stim;
        const T v_plateau_potassium_current__Kp = (m_div(T(1.0), (T(1.0) + m_exp((m_divk((T(7.488) - y[0]), T(5.98), T(0.16722408026755853)))))));
        const T v_plateau_potassium_current__i_Kp = ((T(0.0183)*p[4])*v_plateau_potassium_current__Kp*(y[0] - (-T(87.8929017138025))));
        const T v_slow_inward_current__E_si = (T(7.7) - (T(13.0287)*m_log((m_divk(y[7], T(1.0), T(1.0))))));
        const T v_slow_inward_current__i_si = ((T(0.09)*p[1])*y[4]*y[5]*(y[0] - v_slow_inward_current__E_si));
        const T v_time_dependent_potassium_current_Xi_gate__Xi = ((y[0] > (-T(100.0))) ? (((chb::singularity_offset<T>()*T(1.0)) > fabs((y[0] + T(77.0)))) ? ((m_div((T(2.837)*(m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0))), (((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(35.0))))))) + (m_div((y[0] - (-T(77.0) - (chb::singularity_offset<T>()*T(1.0))))*((m_div((T(2.837)*(m_exp((T(0.04)*((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0))), (((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(35.0))))))) - (m_div((T(2.837)*(m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0))), (((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(35.0)))))))), (T(2.0)*(chb::singularity_offset<T>()*T(1.0)))))) : (m_div((T(2.837)*(m_exp((T(0.04)*(y[0] + T(77.0)))) - T(1.0))), ((y[0] + T(77.0))*m_exp((T(0.04)*(y[0] + T(35.0)))))))) : T(1.0));
        const T v_time_dependent_potassium_current__g_K__scaled = (T(0.282)*p[2]);
        const T v_time_dependent_potassium_current__i_K = (v_time_dependent_potassium_current__g_K__scaled*y[6]*v_time_dependent_potassium_current_Xi_gate__Xi*(y[0] - (-T(77.56758438531939))));
        const T v_time_independent_potassium_current_K1_gate__alpha_K1 = (m_div(T(1.02), (T(1.0) + m_exp((T(0.2385)*((y[0] - (-T(87.8929017138025))) - T(59.215)))))));
        const T v_time_independent_potassium_current_K1_gate__beta_K1 = (m_div(((T(0.49124)*m_exp((T(0.08032)*((y[0] + T(5.476)) - (-T(87.8929017138025)))))) + (T(1.0)*m_exp((T(0.06175)*(y[0] - (-T(87.8929017138025) + T(594.31))))))), (T(1.0) + m_exp(((-T(0.5143))*((y[0] - (-T(87.8929017138025))) + T(4.753)))))));
        const T v_time_independent_potassium_current_K1_gate__K1_infinity = (m_div(v_time_independent_potassium_current_K1_gate__alpha_K1, (v_time_independent_potassium_current_K1_gate__alpha_K1 + v_time_independent_potassium_current_K1_gate__beta_K1)));
        const T v_time_independent_potassium_current__g_K1__scaled = (T(0.6047)*p[3]);
        const T v_time_independent_potassium_current__i_K1 = (v_time_independent_potassium_current__g_K1__scaled*v_time_independent_potassium_current_K1_gate__K1_infinity*(y[0] - (-T(87.8929017138025))));
        rate[0] = ((m_divk((-T(1.0)), T(1.0), T(1.0)))*(v_membrane__I_stim + v_fast_sodium_current__i_Na + v_slow_inward_current__i_si + v_time_dependent_potassium_current__i_K + v_time_independent_potassium_current__i_K1 + v_plateau_potassium_current__i_Kp + v_background_current__i_b));
        rate[7] = (((m_divk((-T(0.0001)), T(1.0), T(1.0)))*v_slow_inward_current__i_si) + (T(0.07)*(T(0.0001) - y[7])));
    }
    // The subexpressions of rl_terms_states that depend on the voltage and the
    // parameters alone and hold an exponential, logarithm, power, quotient or branch:
    // with V clamped over a PDE step they are computed once (rl_vterms) and the
    // substeps take them from vt (rl_terms_states_vt, the same terms otherwise).
    static constexpr int kNumVTerms = 3;
    template <typename T>
    CHB_HD static void rl_vterms(const T* __restrict__ y, const T* __restrict__ p, T* __restrict__ vt) {
        (void)y; (void)p; (void)vt;
        const T v_time_independent_potassium_current_K1_gate__alpha_K1 = (m_div(T(1.02), (T(1.0) + m_exp((T(0.2385)*((y[0] - (-T(87.8929017138025))) - T(59.215)))))));
        const T v_time_independent_potassium_current_K1_gate__beta_K1 = (m_div(((T(0.49124)*m_exp((T(0.08032)*((y[0] + T(5.476)) - (-T(87.8929017138025)))))) + (T(1.0)*m_exp((T(0.06175)*(y[0] - (-T(87.8929017138025) + T(594.31))))))), (T(1.0) + m_exp(((-T(0.5143))*((y[0] - (-T(87.8929017138025))) + T(4.753)))))));
        vt[0] = (m_div(T(1.0), (T(1.0) + m_exp((m_divk((T(7.488) - y[0]), T(5.98), T(0.16722408026755853)))))));
        vt[1] = ((y[0] > (-T(100.0))) ? (((chb::singularity_offset<T>()*T(1.0)) > fabs((y[0] + T(77.0)))) ? ((m_div((T(2.837)*(m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0))), (((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(35.0))))))) + (m_div((y[0] - (-T(77.0) - (chb::singularity_offset<T>()*T(1.0))))*((m_div((T(2.837)*(m_exp((T(0.04)*((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0))), (((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(35.0))))))) - (m_div((T(2.837)*(m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0))), (((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(35.0)))))))), (T(2.0)*(chb::singularity_offset<T>()*T(1.0)))))) : (m_div((T(2.837)*(m_exp((T(0.04)*(y[0] + T(77.0)))) - T(1.0))), ((y[0] + T(77.0))*m_exp((T(0.04)*(y[0] + T(35.0)))))))) : T(1.0));
        vt[2] = (m_div(v_time_independent_potassium_current_K1_gate__alpha_K1, (v_time_independent_potassium_current_K1_gate__alpha_K1 + v_time_independent_potassium_current_K1_gate__beta_K1)));
    }
    // vt is anything indexable: the array rl_vterms wrote, or an accessor that
    // reads each term where it is used (a per-thread column of shared memory).
    template <typename T, class VT = const T*>
    CHB_HD static void rl_terms_states_vt(const T* __restrict__ y, T stim, T cm,
                                          const T* __restrict__ p, const VT& vt,
                                          T* __restrict__ rate, T* __restrict__ inf) {
        (void)stim; (void)cm; (void)p; (void)vt; (void)inf;
        const T v_background_current__i_b = ((T(0.03921)*p[5])*(y[0] - (-T(59.87))));
        const T v_fast_sodium_current__i_Na = ((T(23.0)*p[0])*(y[1]*y[1]*y[1])*y[2]*y[3]*(y[0] - T(54.79446393509185)));
        const T v_membrane__I_stim = stim;
        const T v_plateau_potassium_current__i_Kp = ((T(0.0183)*p[4])*vt[0]*(y[0] - (-T(87.8929017138025))));
        const T v_slow_inward_current__E_si = (T(7.7) - (T(13.0287)*m_log((m_divk(y[7], T(1.0), T(1.0))))));
        const T v_slow_inward_current__i_si = ((T(0.09)*p[1])*y[4]*y[5]*(y[0] - v_slow_inward_current__E_si));
        const T v_time_dependent_potassium_current__g_K__scaled = (T(0.282)*p[2]);
        const T v_time_dependent_potassium_current__i_K = (v_time_dependent_potassium_current__g_K__scaled*y[6]*vt[1]*(y[0] - (-T(77.56758438531939))));
        const T v_time_independent_potassium_current__g_K1__scaled = (T(0.6047)*p[3]);
        const T v_time_independent_potassium_current__i_K1 = (v_time_independent_potassium_current__g_K1__scaled*vt[2]*(y[0] - (-T(87.8929017138025))));
        rate[0] = ((m_divk((-T(1.0)), T(1.0), T(1.0)))*(v_membrane__I_stim + v_fast_sodium_current__i_Na + v_slow_inward_current__i_si + v_time_dependent_potassium_current__i_K + v_time_independent_potassium_current__i_K1 + v_plateau_potassium_current__i_Kp + v_background_current__i_b));
        rate[7] = (((m_divk((-T(0.0001)), T(1.0), T(1.0)))*v_slow_inward_current__i_si) + (T(0.07)*(T(0.0001) - y[7])));
    }

    // Total ionic current in uA/cm^2 (GetIIonic): the dV/dt currents without
    // the stimulus.
    template <typename T>
    CHB_HD static T iionic(const T* __restrict__ y, T cm, const T* __restrict__ p) {
        (void)cm; (void)p;
        const T stim = T(0.0); (void)stim;
        const T v_background_current__i_b = ((T(0.03921)*p[5])*(y[0] - (-T(59.87))));
        const T v_fast_sodium_current__i_Na = ((T(23.0)*p[0])*(y[1]*y[1]*y[1])*y[2]*y[3]*(y[0] - T(54.79446393509185)));
        const T v_plateau_potassium_current__Kp = (m_div(T(1.0), (T(1.0) + m_exp((m_divk((T(7.488) - y[0]), T(5.98), T(0.16722408026755853)))))));
        const T v_plateau_potassium_current__i_Kp = ((T(0.0183)*p[4])*v_plateau_potassium_current__Kp*(y[0] - (-T(87.8929017138025))));
        const T v_slow_inward_current__E_si = (T(7.7) - (T(13.0287)*m_log((m_divk(y[7], T(1.0), T(1.0))))));
        const T v_slow_inward_current__i_si = ((T(0.09)*p[1])*y[4]*y[5]*(y[0] - v_slow_inward_current__E_si));
        const T v_time_dependent_potassium_current_Xi_gate__Xi = ((y[0] > (-T(100.0))) ? (((chb::singularity_offset<T>()*T(1.0)) > fabs((y[0] + T(77.0)))) ? ((m_div((T(2.837)*(m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0))), (((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(35.0))))))) + (m_div((y[0] - (-T(77.0) - (chb::singularity_offset<T>()*T(1.0))))*((m_div((T(2.837)*(m_exp((T(0.04)*((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0))), (((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(35.0))))))) - (m_div((T(2.837)*(m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0))), (((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(35.0)))))))), (T(2.0)*(chb::singularity_offset<T>()*T(1.0)))))) : (m_div((T(2.837)*(m_exp((T(0.04)*(y[0] + T(77.0)))) - T(1.0))), ((y[0] + T(77.0))*m_exp((T(0.04)*(y[0] + T(35.0)))))))) : T(1.0));
        const T v_time_dependent_potassium_current__g_K__scaled = (T(0.282)*p[2]);
        const T v_time_dependent_potassium_current__i_K = (v_time_dependent_potassium_current__g_K__scaled*y[6]*v_time_dependent_potassium_current_Xi_gate__Xi*(y[0] - (-T(77.56758438531939))));
        const T v_time_independent_potassium_current_K1_gate__alpha_K1 = (m_div(T(1.02), (T(1.0) + m_exp((T(0.2385)*((y[0] - (-T(87.8929017138025))) - T(59.215)))))));
        const T v_time_independent_potassium_current_K1_gate__beta_K1 = (m_div(((T(0.49124)*m_exp((T(0.08032)*((y[0] + T(5.476)) - (-T(87.8929017138025)))))) + (T(1.0)*m_exp((T(0.06175)*(y[0] - (-T(87.8929017138025) + T(594.31))))))), (T(1.0) + m_exp(((-T(0.5143))*((y[0] - (-T(87.8929017138025))) + T(4.753)))))));
        const T v_time_independent_potassium_current_K1_gate__K1_infinity = (m_div(v_time_independent_potassium_current_K1_gate__alpha_K1, (v_time_independent_potassium_current_K1_gate__alpha_K1 + v_time_independent_potassium_current_K1_gate__beta_K1)));
        const T v_time_independent_potassium_current__g_K1__scaled = (T(0.6047)*p[3]);
        const T v_time_independent_potassium_current__i_K1 = (v_time_independent_potassium_current__g_K1__scaled*v_time_independent_potassium_current_K1_gate__K1_infinity*(y[0] - (-T(87.8929017138025))));
        return (v_background_current__i_b + v_fast_sodium_current__i_Na + v_plateau_potassium_current__i_Kp + v_slow_inward_current__i_si + v_time_dependent_potassium_current__i_K + v_time_independent_potassium_current__i_K1);
    }

    // Reverse-mode product for rhs: gy[j] += sum_i w_i d(out_i)/d(y_j),
    // gp[k] += sum_i w_i d(out_i)/d(p_k)  (w: weights of dy[0..S-1]; y[0] is the voltage).
    template <typename T>
    CHB_HD static void vjp_rhs(const T* __restrict__ y, T stim, T cm, const T* __restrict__ p,
                                const T* __restrict__ w, T* __restrict__ gy, T* __restrict__ gp) {
        (void)stim; (void)cm; (void)p; (void)w; (void)gy; (void)gp;
        const T v_background_current__i_b = ((T(0.03921)*p[5])*(y[0] - (-T(59.87))));
        const T v_fast_sodium_current__i_Na = ((T(23.0)*p[0])*(y[1]*y[1]*y[1])*y[2]*y[3]*(y[0] - T(54.79446393509185)));
        const T v_membrane__I_stim = stim;
        const T v_plateau_potassium_current__Kp = (m_div(T(1.0), (T(1.0) + m_exp((m_divk((T(7.488) - y[0]), T(5.98), T(0.16722408026755853)))))));
        const T v_plateau_potassium_current__i_Kp = ((T(0.0183)*p[4])*v_plateau_potassium_current__Kp*(y[0] - (-T(87.8929017138025))));
        const T v_slow_inward_current__E_si = (T(7.7) - (T(13.0287)*m_log((m_divk(y[7], T(1.0), T(1.0))))));
        const T v_slow_inward_current__i_si = ((T(0.09)*p[1])*y[4]*y[5]*(y[0] - v_slow_inward_current__E_si));
        const T v_time_dependent_potassium_current_Xi_gate__Xi = ((y[0] > (-T(100.0))) ? (((chb::singularity_offset<T>()*T(1.0)) > fabs((y[0] + T(77.0)))) ? ((m_div((T(2.837)*(m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0))), (((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(35.0))))))) + (m_div((y[0] - (-T(77.0) - (chb::singularity_offset<T>()*T(1.0))))*((m_div((T(2.837)*(m_exp((T(0.04)*((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0))), (((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(35.0))))))) - (m_div((T(2.837)*(m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0))), (((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(35.0)))))))), (T(2.0)*(chb::singularity_offset<T>()*T(1.0)))))) : (m_div((T(2.837)*(m_exp((T(0.04)*(y[0] + T(77.0)))) - T(1.0))), ((y[0] + T(77.0))*m_exp((T(0.04)*(y[0] + T(35.0)))))))) : T(1.0));
        const T v_time_dependent_potassium_current__g_K__scaled = (T(0.282)*p[2]);
        const T v_time_dependent_potassium_current__i_K = (v_time_dependent_potassium_current__g_K__scaled*y[6]*v_time_dependent_potassium_current_Xi_gate__Xi*(y[0] - (-T(77.56758438531939))));
        const T v_time_independent_potassium_current_K1_gate__alpha_K1 = (m_div(T(1.02), (T(1.0) + m_exp((T(0.2385)*((y[0] - (-T(87.8929017138025))) - T(59.215)))))));
        const T v_time_independent_potassium_current_K1_gate__beta_K1 = (m_div(((T(0.49124)*m_exp((T(0.08032)*((y[0] + T(5.476)) - (-T(87.8929017138025)))))) + (T(1.0)*m_exp((T(0.06175)*(y[0] - (-T(87.8929017138025) + T(594.31))))))), (T(1.0) + m_exp(((-T(0.5143))*((y[0] - (-T(87.8929017138025))) + T(4.753)))))));
        const T v_time_independent_potassium_current_K1_gate__K1_infinity = (m_div(v_time_independent_potassium_current_K1_gate__alpha_K1, (v_time_independent_potassium_current_K1_gate__alpha_K1 + v_time_independent_potassium_current_K1_gate__beta_K1)));
        const T v_time_independent_potassium_current__g_K1__scaled = (T(0.6047)*p[3]);
        const T v_time_independent_potassium_current__i_K1 = (v_time_independent_potassium_current__g_K1__scaled*v_time_independent_potassium_current_K1_gate__K1_infinity*(y[0] - (-T(87.8929017138025))));
        const T v_fast_sodium_current_m_gate__alpha_m = (((chb::singularity_offset<T>()*T(10.0)) > fabs((y[0] + T(47.13)))) ? ((m_div((T(0.32)*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13))), (T(1.0) - m_exp(((-T(0.1))*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13))))))) + (m_div((y[0] - (-T(47.13) - (chb::singularity_offset<T>()*T(10.0))))*((m_div((T(0.32)*((-T(47.13) + (chb::singularity_offset<T>()*T(10.0))) + T(47.13))), (T(1.0) - m_exp(((-T(0.1))*((-T(47.13) + (chb::singularity_offset<T>()*T(10.0))) + T(47.13))))))) - (m_div((T(0.32)*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13))), (T(1.0) - m_exp(((-T(0.1))*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13)))))))), (T(2.0)*(chb::singularity_offset<T>()*T(10.0)))))) : (m_div((T(0.32)*(y[0] + T(47.13))), (T(1.0) - m_exp(((-T(0.1))*(y[0] + T(47.13))))))));
        const T v_fast_sodium_current_m_gate__beta_m = (T(0.08)*m_exp((m_divk((-y[0]), T(11.0), T(0.09090909090909091)))));
        const T v_fast_sodium_current_h_gate__alpha_h = ((y[0] < (-T(40.0))) ? (T(0.135)*m_exp((m_div((T(80.0) + y[0]), (-T(6.8)))))) : T(0.0));
        const T v_fast_sodium_current_h_gate__beta_h = ((y[0] < (-T(40.0))) ? ((T(3.56)*m_exp((T(0.079)*y[0]))) + (T(310000.0)*m_exp((T(0.35)*y[0])))) : (m_div(T(1.0), (T(0.13)*(T(1.0) + m_exp((m_div((y[0] + T(10.66)), (-T(11.1))))))))));
        const T v_fast_sodium_current_j_gate__alpha_j = ((y[0] < (-T(40.0))) ? (m_div(((((-T(127140.0))*m_exp((T(0.2444)*y[0]))) - (T(3.474e-05)*m_exp(((-T(0.04391))*y[0]))))*(y[0] + T(37.78))), (T(1.0) + m_exp((T(0.311)*(y[0] + T(79.23))))))) : T(0.0));
        const T v_fast_sodium_current_j_gate__beta_j = ((y[0] < (-T(40.0))) ? (m_div((T(0.1212)*m_exp(((-T(0.01052))*y[0]))), (T(1.0) + m_exp(((-T(0.1378))*(y[0] + T(40.14))))))) : (m_div((T(0.3)*m_exp(((-T(2.535e-07))*y[0]))), (T(1.0) + m_exp(((-T(0.1))*(y[0] + T(32.0))))))));
        const T v_slow_inward_current_d_gate__alpha_d = (m_div((T(0.095)*m_exp(((-T(0.01))*(y[0] - T(5.0))))), (T(1.0) + m_exp(((-T(0.072))*(y[0] - T(5.0)))))));
        const T v_slow_inward_current_d_gate__beta_d = (m_div((T(0.07)*m_exp(((-T(0.017))*(y[0] + T(44.0))))), (T(1.0) + m_exp((T(0.05)*(y[0] + T(44.0)))))));
        const T v_slow_inward_current_f_gate__alpha_f = (m_div((T(0.012)*m_exp(((-T(0.008))*(y[0] + T(28.0))))), (T(1.0) + m_exp((T(0.15)*(y[0] + T(28.0)))))));
        const T v_slow_inward_current_f_gate__beta_f = (m_div((T(0.0065)*m_exp(((-T(0.02))*(y[0] + T(30.0))))), (T(1.0) + m_exp(((-T(0.2))*(y[0] + T(30.0)))))));
        const T v_time_dependent_potassium_current_X_gate__alpha_X = (m_div((T(0.0005)*m_exp((T(0.083)*(y[0] + T(50.0))))), (T(1.0) + m_exp((T(0.057)*(y[0] + T(50.0)))))));
        const T v_time_dependent_potassium_current_X_gate__beta_X = (m_div((T(0.0013)*m_exp(((-T(0.06))*(y[0] + T(20.0))))), (T(1.0) + m_exp(((-T(0.04))*(y[0] + T(20.0)))))));
        T a_v_background_current__i_b = T(0.0);
        T a_v_fast_sodium_current__i_Na = T(0.0);
        T a_v_membrane__I_stim = T(0.0);
        T a_v_plateau_potassium_current__i_Kp = T(0.0);
        T a_v_slow_inward_current__i_si = T(0.0);
        T a_v_time_dependent_potassium_current__i_K = T(0.0);
        T a_v_time_independent_potassium_current__i_K1 = T(0.0);
        T a_v_fast_sodium_current_m_gate__alpha_m = T(0.0);
        T a_v_fast_sodium_current_m_gate__beta_m = T(0.0);
        T a_y_1 = T(0.0);
        T a_v_fast_sodium_current_h_gate__alpha_h = T(0.0);
        T a_v_fast_sodium_current_h_gate__beta_h = T(0.0);
        T a_y_2 = T(0.0);
        T a_v_fast_sodium_current_j_gate__alpha_j = T(0.0);
        T a_v_fast_sodium_current_j_gate__beta_j = T(0.0);
        T a_y_3 = T(0.0);
        T a_v_slow_inward_current_d_gate__alpha_d = T(0.0);
        T a_v_slow_inward_current_d_gate__beta_d = T(0.0);
        T a_y_4 = T(0.0);
        T a_v_slow_inward_current_f_gate__alpha_f = T(0.0);
        T a_v_slow_inward_current_f_gate__beta_f = T(0.0);
        T a_y_5 = T(0.0);
        T a_y_6 = T(0.0);
        T a_v_time_dependent_potassium_current_X_gate__alpha_X = T(0.0);
        T a_v_time_dependent_potassium_current_X_gate__beta_X = T(0.0);
        T a_y_7 = T(0.0);
        a_v_background_current__i_b += w[0]*((-T(1.0)));
        a_v_fast_sodium_current__i_Na += w[0]*((-T(1.0)));
        a_v_membrane__I_stim += w[0]*((-T(1.0)));
        a_v_plateau_potassium_current__i_Kp += w[0]*((-T(1.0)));
        a_v_slow_inward_current__i_si += w[0]*((-T(1.0)));
        a_v_time_dependent_potassium_current__i_K += w[0]*((-T(1.0)));
        a_v_time_independent_potassium_current__i_K1 += w[0]*((-T(1.0)));
        a_v_fast_sodium_current_m_gate__alpha_m += w[1]*((T(1.0) - y[1]));
        a_v_fast_sodium_current_m_gate__beta_m += w[1]*((-y[1]));
        a_y_1 += w[1]*((-v_fast_sodium_current_m_gate__alpha_m - v_fast_sodium_current_m_gate__beta_m));
        a_v_fast_sodium_current_h_gate__alpha_h += w[2]*((T(1.0) - y[2]));
        a_v_fast_sodium_current_h_gate__beta_h += w[2]*((-y[2]));
        a_y_2 += w[2]*((-v_fast_sodium_current_h_gate__alpha_h - v_fast_sodium_current_h_gate__beta_h));
        a_v_fast_sodium_current_j_gate__alpha_j += w[3]*((T(1.0) - y[3]));
        a_v_fast_sodium_current_j_gate__beta_j += w[3]*((-y[3]));
        a_y_3 += w[3]*((-v_fast_sodium_current_j_gate__alpha_j - v_fast_sodium_current_j_gate__beta_j));
        a_v_slow_inward_current_d_gate__alpha_d += w[4]*((T(1.0) - y[4]));
        a_v_slow_inward_current_d_gate__beta_d += w[4]*((-y[4]));
        a_y_4 += w[4]*((-v_slow_inward_current_d_gate__alpha_d - v_slow_inward_current_d_gate__beta_d));
        a_v_slow_inward_current_f_gate__alpha_f += w[5]*((T(1.0) - y[5]));
        a_v_slow_inward_current_f_gate__beta_f += w[5]*((-y[5]));
        a_y_5 += w[5]*((-v_slow_inward_current_f_gate__alpha_f - v_slow_inward_current_f_gate__beta_f));
        a_y_6 += w[6]*((-v_time_dependent_potassium_current_X_gate__alpha_X - v_time_dependent_potassium_current_X_gate__beta_X));
        a_v_time_dependent_potassium_current_X_gate__alpha_X += w[6]*((T(1.0) - y[6]));
        a_v_time_dependent_potassium_current_X_gate__beta_X += w[6]*((-y[6]));
        a_y_7 += w[7]*((-T(0.07)));
        a_v_slow_inward_current__i_si += w[7]*((-T(0.0001)));
        T a_y_0 = T(0.0);
        a_y_0 += a_v_time_dependent_potassium_current_X_gate__beta_X*(((m_div(T(7.03743472830386e-06)*m_exp(((-T(0.1))*y[0])), ((T(1.0) + (T(0.44932896411722156)*m_exp(((-T(0.04))*y[0]))))*(T(1.0) + (T(0.44932896411722156)*m_exp(((-T(0.04))*y[0]))))))) - (m_div(T(2.3493148529151763e-05)*m_exp(((-T(0.06))*y[0])), (T(1.0) + (T(0.44932896411722156)*m_exp(((-T(0.04))*y[0]))))))));
        a_y_0 += a_v_time_dependent_potassium_current_X_gate__alpha_X*(((m_div(T(0.0026325110123721187)*m_exp((T(0.083)*y[0])), (T(1.0) + (T(17.28778184056764)*m_exp((T(0.057)*y[0])))))) - (m_div(T(0.031254045015211084)*m_exp((T(0.14)*y[0])), ((T(1.0) + (T(17.28778184056764)*m_exp((T(0.057)*y[0]))))*(T(1.0) + (T(17.28778184056764)*m_exp((T(0.057)*y[0])))))))));
        a_y_0 += a_v_slow_inward_current_f_gate__beta_f*(((m_div(T(1.7684784488122608e-06)*m_exp(((-T(0.22))*y[0])), ((T(1.0) + (T(0.0024787521766663576)*m_exp(((-T(0.2))*y[0]))))*(T(1.0) + (T(0.0024787521766663576)*m_exp(((-T(0.2))*y[0]))))))) - (m_div(T(7.134551269222344e-05)*m_exp(((-T(0.02))*y[0])), (T(1.0) + (T(0.0024787521766663576)*m_exp(((-T(0.2))*y[0]))))))));
        a_y_0 += a_v_slow_inward_current_f_gate__alpha_f*((-(m_div(T(7.673425289945905e-05)*m_exp(((-T(0.008))*y[0])), (T(1.0) + (T(66.68633104092513)*m_exp((T(0.15)*y[0])))))) - (m_div(T(0.09594610858183865)*m_exp((T(0.142)*y[0])), ((T(1.0) + (T(66.68633104092513)*m_exp((T(0.15)*y[0]))))*(T(1.0) + (T(66.68633104092513)*m_exp((T(0.15)*y[0])))))))));
        a_y_0 += a_v_slow_inward_current_d_gate__beta_d*((-(m_div(T(0.0005632415551395898)*m_exp(((-T(0.017))*y[0])), (T(1.0) + (T(9.025013499434122)*m_exp((T(0.05)*y[0])))))) - (m_div(T(0.014950772466403138)*m_exp((T(0.033)*y[0])), ((T(1.0) + (T(9.025013499434122)*m_exp((T(0.05)*y[0]))))*(T(1.0) + (T(9.025013499434122)*m_exp((T(0.05)*y[0])))))))));
        a_y_0 += a_v_slow_inward_current_d_gate__alpha_d*(((m_div(T(0.010306633650171919)*m_exp(((-T(0.08199999999999999))*y[0])), ((T(1.0) + (T(1.4333294145603401)*m_exp(((-T(0.072))*y[0]))))*(T(1.0) + (T(1.4333294145603401)*m_exp(((-T(0.072))*y[0]))))))) - (m_div(T(0.000998707541557223)*m_exp(((-T(0.01))*y[0])), (T(1.0) + (T(1.4333294145603401)*m_exp(((-T(0.072))*y[0]))))))));
        a_y_0 += a_v_fast_sodium_current_j_gate__beta_j*(((y[0] < (-T(40.0))) ? ((m_div(T(6.615188805734336e-05)*m_exp(((-T(0.14832))*y[0])), ((T(1.0) + (T(0.003960868339904256)*m_exp(((-T(0.1378))*y[0]))))*(T(1.0) + (T(0.003960868339904256)*m_exp(((-T(0.1378))*y[0]))))))) - (m_div(T(0.001275024)*m_exp(((-T(0.01052))*y[0])), (T(1.0) + (T(0.003960868339904256)*m_exp(((-T(0.1378))*y[0]))))))) : ((m_div(T(0.001222866119350986)*m_exp(((-T(0.10000025350000001))*y[0])), ((T(1.0) + (T(0.040762203978366204)*m_exp(((-T(0.1))*y[0]))))*(T(1.0) + (T(0.040762203978366204)*m_exp(((-T(0.1))*y[0]))))))) - (m_div(T(7.605e-08)*m_exp(((-T(2.535e-07))*y[0])), (T(1.0) + (T(0.040762203978366204)*m_exp(((-T(0.1))*y[0])))))))));
        a_y_0 += a_v_fast_sodium_current_j_gate__alpha_j*(((y[0] < (-T(40.0))) ? ((m_div((-(T(127140.0)*m_exp((T(0.2444)*y[0]))) - (T(3.474e-05)*m_exp(((-T(0.04391))*y[0])))), (T(1.0) + (T(50262745825.95395)*m_exp((T(0.311)*y[0])))))) + (m_div((T(37.78) + y[0])*((T(1.5254334e-06)*m_exp(((-T(0.04391))*y[0]))) - (T(31073.016)*m_exp((T(0.2444)*y[0])))), (T(1.0) + (T(50262745825.95395)*m_exp((T(0.311)*y[0])))))) - (m_div(T(15631713951.87168)*(T(37.78) + y[0])*(-(T(127140.0)*m_exp((T(0.2444)*y[0]))) - (T(3.474e-05)*m_exp(((-T(0.04391))*y[0]))))*m_exp((T(0.311)*y[0])), ((T(1.0) + (T(50262745825.95395)*m_exp((T(0.311)*y[0]))))*(T(1.0) + (T(50262745825.95395)*m_exp((T(0.311)*y[0])))))))) : T(0.0)));
        a_y_0 += a_v_fast_sodium_current_h_gate__beta_h*(((y[0] < (-T(40.0))) ? ((T(0.28124)*m_exp((T(0.079)*y[0]))) + (T(108500.0)*m_exp((T(0.35)*y[0])))) : (m_div(T(0.00448271541296745)*m_exp(((-T(0.0900900900900901))*y[0])), ((T(0.13) + (T(0.049758141083938695)*m_exp(((-T(0.0900900900900901))*y[0]))))*(T(0.13) + (T(0.049758141083938695)*m_exp(((-T(0.0900900900900901))*y[0])))))))));
        a_y_0 += a_v_fast_sodium_current_h_gate__alpha_h*(((y[0] < (-T(40.0))) ? ((-T(1.5433982726867125e-07))*m_exp(((-T(0.14705882352941177))*y[0]))) : T(0.0)));
        a_y_0 += a_v_fast_sodium_current_m_gate__beta_m*(((-T(0.007272727272727273))*m_exp(((-T(0.09090909090909091))*y[0]))));
        a_y_0 += a_v_fast_sodium_current_m_gate__alpha_m*((((T(10.0)*chb::singularity_offset<T>()) > fabs((T(47.13) + y[0]))) ? (m_div(T(0.05)*((m_div(T(3.2)*chb::singularity_offset<T>(), (T(1.0) - m_exp((T(1.0)*chb::singularity_offset<T>()))))) + (m_div(T(3.2)*chb::singularity_offset<T>(), (T(1.0) - m_exp((-chb::singularity_offset<T>())))))), chb::singularity_offset<T>())) : ((m_div(T(0.32), (T(1.0) - (T(0.008977803730697237)*m_exp(((-T(0.1))*y[0])))))) - (m_div(T(0.0008977803730697238)*(T(15.081600000000002) + (T(0.32)*y[0]))*m_exp(((-T(0.1))*y[0])), ((T(1.0) - (T(0.008977803730697237)*m_exp(((-T(0.1))*y[0]))))*(T(1.0) - (T(0.008977803730697237)*m_exp(((-T(0.1))*y[0]))))))))));
        a_y_0 += a_v_time_independent_potassium_current__i_K1*((v_time_independent_potassium_current_K1_gate__K1_infinity*v_time_independent_potassium_current__g_K1__scaled));
        T a_v_time_independent_potassium_current_K1_gate__K1_infinity = T(0.0);
        a_v_time_independent_potassium_current_K1_gate__K1_infinity += a_v_time_independent_potassium_current__i_K1*((v_time_independent_potassium_current__g_K1__scaled*(T(87.8929017138025) + y[0])));
        T a_v_time_independent_potassium_current__g_K1__scaled = T(0.0);
        a_v_time_independent_potassium_current__g_K1__scaled += a_v_time_independent_potassium_current__i_K1*((v_time_independent_potassium_current_K1_gate__K1_infinity*(T(87.8929017138025) + y[0])));
        T a_p_3 = T(0.0);
        a_p_3 += a_v_time_independent_potassium_current__g_K1__scaled*(T(0.6047));
        T a_v_time_independent_potassium_current_K1_gate__alpha_K1 = T(0.0);
        a_v_time_independent_potassium_current_K1_gate__alpha_K1 += a_v_time_independent_potassium_current_K1_gate__K1_infinity*(((m_div(T(1.0), (v_time_independent_potassium_current_K1_gate__alpha_K1 + v_time_independent_potassium_current_K1_gate__beta_K1))) - (m_div(v_time_independent_potassium_current_K1_gate__alpha_K1, ((v_time_independent_potassium_current_K1_gate__alpha_K1 + v_time_independent_potassium_current_K1_gate__beta_K1)*(v_time_independent_potassium_current_K1_gate__alpha_K1 + v_time_independent_potassium_current_K1_gate__beta_K1))))));
        T a_v_time_independent_potassium_current_K1_gate__beta_K1 = T(0.0);
        a_v_time_independent_potassium_current_K1_gate__beta_K1 += a_v_time_independent_potassium_current_K1_gate__K1_infinity*((-m_div(v_time_independent_potassium_current_K1_gate__alpha_K1, ((v_time_independent_potassium_current_K1_gate__alpha_K1 + v_time_independent_potassium_current_K1_gate__beta_K1)*(v_time_independent_potassium_current_K1_gate__alpha_K1 + v_time_independent_potassium_current_K1_gate__beta_K1)))));
        a_y_0 += a_v_time_independent_potassium_current_K1_gate__beta_K1*(((m_div(((T(71.29534875031702)*m_exp((T(0.08032)*y[0]))) + (T(1.6207018112661692e-15)*m_exp((T(0.06175)*y[0])))), (T(1.0) + (T(2.0268841278228537e-21)*m_exp(((-T(0.5143))*y[0])))))) + (m_div(T(1.0424265069392937e-21)*((T(887.6412942021542)*m_exp((T(0.08032)*y[0]))) + (T(2.6246183178399503e-14)*m_exp((T(0.06175)*y[0]))))*m_exp(((-T(0.5143))*y[0])), ((T(1.0) + (T(2.0268841278228537e-21)*m_exp(((-T(0.5143))*y[0]))))*(T(1.0) + (T(2.0268841278228537e-21)*m_exp(((-T(0.5143))*y[0])))))))));
        a_y_0 += a_v_time_independent_potassium_current_K1_gate__alpha_K1*((m_div((-T(227.26033654832673))*m_exp((T(0.2385)*y[0])), ((T(1.0) + (T(934.1897338279555)*m_exp((T(0.2385)*y[0]))))*(T(1.0) + (T(934.1897338279555)*m_exp((T(0.2385)*y[0]))))))));
        a_y_0 += a_v_time_dependent_potassium_current__i_K*((y[6]*v_time_dependent_potassium_current_Xi_gate__Xi*v_time_dependent_potassium_current__g_K__scaled));
        a_y_6 += a_v_time_dependent_potassium_current__i_K*((v_time_dependent_potassium_current_Xi_gate__Xi*v_time_dependent_potassium_current__g_K__scaled*(T(77.56758438531939) + y[0])));
        T a_v_time_dependent_potassium_current_Xi_gate__Xi = T(0.0);
        a_v_time_dependent_potassium_current_Xi_gate__Xi += a_v_time_dependent_potassium_current__i_K*((y[6]*v_time_dependent_potassium_current__g_K__scaled*(T(77.56758438531939) + y[0])));
        T a_v_time_dependent_potassium_current__g_K__scaled = T(0.0);
        a_v_time_dependent_potassium_current__g_K__scaled += a_v_time_dependent_potassium_current__i_K*((y[6]*v_time_dependent_potassium_current_Xi_gate__Xi*(T(77.56758438531939) + y[0])));
        T a_p_2 = T(0.0);
        a_p_2 += a_v_time_dependent_potassium_current__g_K__scaled*(T(0.282));
        a_y_0 += a_v_time_dependent_potassium_current_Xi_gate__Xi*(((y[0] > (-T(100.0))) ? (((T(1.0)*chb::singularity_offset<T>()) > fabs((T(77.0) + y[0]))) ? (m_div(T(0.5)*((m_div(T(5.365555971121975)*(-T(2.837) + (T(2.837)*m_exp((T(0.04)*chb::singularity_offset<T>()))))*m_exp(((-T(0.04))*chb::singularity_offset<T>())), chb::singularity_offset<T>())) + (m_div(T(5.365555971121975)*(-T(2.837) + (T(2.837)*m_exp(((-T(0.04))*chb::singularity_offset<T>()))))*m_exp((T(0.04)*chb::singularity_offset<T>())), chb::singularity_offset<T>()))), chb::singularity_offset<T>())) : ((m_div(T(0.6088832916029218), (T(77.0) + y[0]))) - (m_div(T(0.00986387855766426)*(-T(2.837) + (T(61.72858759801112)*m_exp((T(0.04)*y[0]))))*m_exp(((-T(0.04))*y[0])), (T(77.0) + y[0]))) - (m_div(T(0.24659696394160646)*(-T(2.837) + (T(61.72858759801112)*m_exp((T(0.04)*y[0]))))*m_exp(((-T(0.04))*y[0])), ((T(77.0) + y[0])*(T(77.0) + y[0])))))) : T(0.0)));
        T a_p_1 = T(0.0);
        a_p_1 += a_v_slow_inward_current__i_si*((T(0.09)*y[4]*y[5]*(y[0] - v_slow_inward_current__E_si)));
        a_y_0 += a_v_slow_inward_current__i_si*((T(0.09)*p[1]*y[4]*y[5]));
        T a_v_slow_inward_current__E_si = T(0.0);
        a_v_slow_inward_current__E_si += a_v_slow_inward_current__i_si*(((-T(0.09))*p[1]*y[4]*y[5]));
        a_y_4 += a_v_slow_inward_current__i_si*((T(0.09)*p[1]*y[5]*(y[0] - v_slow_inward_current__E_si)));
        a_y_5 += a_v_slow_inward_current__i_si*((T(0.09)*p[1]*y[4]*(y[0] - v_slow_inward_current__E_si)));
        a_y_7 += a_v_slow_inward_current__E_si*((m_div((-T(13.0287)), y[7])));
        T a_p_4 = T(0.0);
        a_p_4 += a_v_plateau_potassium_current__i_Kp*((T(0.0183)*v_plateau_potassium_current__Kp*(T(87.8929017138025) + y[0])));
        a_y_0 += a_v_plateau_potassium_current__i_Kp*((T(0.0183)*p[4]*v_plateau_potassium_current__Kp));
        T a_v_plateau_potassium_current__Kp = T(0.0);
        a_v_plateau_potassium_current__Kp += a_v_plateau_potassium_current__i_Kp*((T(0.0183)*p[4]*(T(87.8929017138025) + y[0])));
        a_y_0 += a_v_plateau_potassium_current__Kp*((m_div(T(0.5849396175627496)*m_exp(((-T(0.16722408026755853))*y[0])), ((T(1.0) + (T(3.497938913025243)*m_exp(((-T(0.16722408026755853))*y[0]))))*(T(1.0) + (T(3.497938913025243)*m_exp(((-T(0.16722408026755853))*y[0]))))))));
        T a_p_0 = T(0.0);
        a_p_0 += a_v_fast_sodium_current__i_Na*((T(23.0)*y[2]*y[3]*(y[1]*y[1]*y[1])*(-T(54.79446393509185) + y[0])));
        a_y_2 += a_v_fast_sodium_current__i_Na*((T(23.0)*p[0]*y[3]*(y[1]*y[1]*y[1])*(-T(54.79446393509185) + y[0])));
        a_y_3 += a_v_fast_sodium_current__i_Na*((T(23.0)*p[0]*y[2]*(y[1]*y[1]*y[1])*(-T(54.79446393509185) + y[0])));
        a_y_1 += a_v_fast_sodium_current__i_Na*((T(69.0)*p[0]*y[2]*y[3]*(y[1]*y[1])*(-T(54.79446393509185) + y[0])));
        a_y_0 += a_v_fast_sodium_current__i_Na*((T(23.0)*p[0]*y[2]*y[3]*(y[1]*y[1]*y[1])));
        T a_p_5 = T(0.0);
        a_p_5 += a_v_background_current__i_b*((T(2.3475027) + (T(0.03921)*y[0])));
        a_y_0 += a_v_background_current__i_b*((T(0.03921)*p[5]));
        gy[0] += a_y_0;
        gy[1] += a_y_1;
        gy[2] += a_y_2;
        gy[3] += a_y_3;
        gy[4] += a_y_4;
        gy[5] += a_y_5;
        gy[6] += a_y_6;
        gy[7] += a_y_7;
        gp[0] += a_p_0;
        gp[1] += a_p_1;
        gp[2] += a_p_2;
        gp[3] += a_p_3;
        gp[4] += a_p_4;
        gp[5] += a_p_5;
    }

    // Reverse-mode product for iionic: gy[j] += sum_i w_i d(out_i)/d(y_j),
    // gp[k] += sum_i w_i d(out_i)/d(p_k)  (w[0]: weight of iionic; y[0] is the voltage).
    template <typename T>
    CHB_HD static void vjp_iionic(const T* __restrict__ y, T stim, T cm, const T* __restrict__ p,
                                const T* __restrict__ w, T* __restrict__ gy, T* __restrict__ gp) {
        (void)stim; (void)cm; (void)p; (void)w; (void)gy; (void)gp;
        const T v_background_current__i_b = ((T(0.03921)*p[5])*(y[0] - (-T(59.87))));
        const T v_fast_sodium_current__i_Na = ((T(23.0)*p[0])*(y[1]*y[1]*y[1])*y[2]*y[3]*(y[0] - T(54.79446393509185)));
        const T v_plateau_potassium_current__Kp = (m_div(T(1.0), (T(1.0) + m_exp((m_divk((T(7.488) - y[0]), T(5.98), T(0.16722408026755853)))))));
        const T v_plateau_potassium_current__i_Kp = ((T(0.0183)*p[4])*v_plateau_potassium_current__Kp*(y[0] - (-T(87.8929017138025))));
        const T v_slow_inward_current__E_si = (T(7.7) - (T(13.0287)*m_log((m_divk(y[7], T(1.0), T(1.0))))));
        const T v_slow_inward_current__i_si = ((T(0.09)*p[1])*y[4]*y[5]*(y[0] - v_slow_inward_current__E_si));
        const T v_time_dependent_potassium_current_Xi_gate__Xi = ((y[0] > (-T(100.0))) ? (((chb::singularity_offset<T>()*T(1.0)) > fabs((y[0] + T(77.0)))) ? ((m_div((T(2.837)*(m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0))), (((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(35.0))))))) + (m_div((y[0] - (-T(77.0) - (chb::singularity_offset<T>()*T(1.0))))*((m_div((T(2.837)*(m_exp((T(0.04)*((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0))), (((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(35.0))))))) - (m_div((T(2.837)*(m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0))), (((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(35.0)))))))), (T(2.0)*(chb::singularity_offset<T>()*T(1.0)))))) : (m_div((T(2.837)*(m_exp((T(0.04)*(y[0] + T(77.0)))) - T(1.0))), ((y[0] + T(77.0))*m_exp((T(0.04)*(y[0] + T(35.0)))))))) : T(1.0));
        const T v_time_dependent_potassium_current__g_K__scaled = (T(0.282)*p[2]);
        const T v_time_dependent_potassium_current__i_K = (v_time_dependent_potassium_current__g_K__scaled*y[6]*v_time_dependent_potassium_current_Xi_gate__Xi*(y[0] - (-T(77.56758438531939))));
        const T v_time_independent_potassium_current_K1_gate__alpha_K1 = (m_div(T(1.02), (T(1.0) + m_exp((T(0.2385)*((y[0] - (-T(87.8929017138025))) - T(59.215)))))));
        const T v_time_independent_potassium_current_K1_gate__beta_K1 = (m_div(((T(0.49124)*m_exp((T(0.08032)*((y[0] + T(5.476)) - (-T(87.8929017138025)))))) + (T(1.0)*m_exp((T(0.06175)*(y[0] - (-T(87.8929017138025) + T(594.31))))))), (T(1.0) + m_exp(((-T(0.5143))*((y[0] - (-T(87.8929017138025))) + T(4.753)))))));
        const T v_time_independent_potassium_current_K1_gate__K1_infinity = (m_div(v_time_independent_potassium_current_K1_gate__alpha_K1, (v_time_independent_potassium_current_K1_gate__alpha_K1 + v_time_independent_potassium_current_K1_gate__beta_K1)));
        const T v_time_independent_potassium_current__g_K1__scaled = (T(0.6047)*p[3]);
        const T v_time_independent_potassium_current__i_K1 = (v_time_independent_potassium_current__g_K1__scaled*v_time_independent_potassium_current_K1_gate__K1_infinity*(y[0] - (-T(87.8929017138025))));
        T a_v_background_current__i_b = T(0.0);
        T a_v_fast_sodium_current__i_Na = T(0.0);
        T a_v_plateau_potassium_current__i_Kp = T(0.0);
        T a_v_slow_inward_current__i_si = T(0.0);
        T a_v_time_dependent_potassium_current__i_K = T(0.0);
        T a_v_time_independent_potassium_current__i_K1 = T(0.0);
        a_v_background_current__i_b += w[0]*(T(1.0));
        a_v_fast_sodium_current__i_Na += w[0]*(T(1.0));
        a_v_plateau_potassium_current__i_Kp += w[0]*(T(1.0));
        a_v_slow_inward_current__i_si += w[0]*(T(1.0));
        a_v_time_dependent_potassium_current__i_K += w[0]*(T(1.0));
        a_v_time_independent_potassium_current__i_K1 += w[0]*(T(1.0));
        T a_y_0 = T(0.0);
        a_y_0 += a_v_time_independent_potassium_current__i_K1*((v_time_independent_potassium_current_K1_gate__K1_infinity*v_time_independent_potassium_current__g_K1__scaled));
        T a_v_time_independent_potassium_current_K1_gate__K1_infinity = T(0.0);
        a_v_time_independent_potassium_current_K1_gate__K1_infinity += a_v_time_independent_potassium_current__i_K1*((v_time_independent_potassium_current__g_K1__scaled*(T(87.8929017138025) + y[0])));
        T a_v_time_independent_potassium_current__g_K1__scaled = T(0.0);
        a_v_time_independent_potassium_current__g_K1__scaled += a_v_time_independent_potassium_current__i_K1*((v_time_independent_potassium_current_K1_gate__K1_infinity*(T(87.8929017138025) + y[0])));
        T a_p_3 = T(0.0);
        a_p_3 += a_v_time_independent_potassium_current__g_K1__scaled*(T(0.6047));
        T a_v_time_independent_potassium_current_K1_gate__alpha_K1 = T(0.0);
        a_v_time_independent_potassium_current_K1_gate__alpha_K1 += a_v_time_independent_potassium_current_K1_gate__K1_infinity*(((m_div(T(1.0), (v_time_independent_potassium_current_K1_gate__alpha_K1 + v_time_independent_potassium_current_K1_gate__beta_K1))) - (m_div(v_time_independent_potassium_current_K1_gate__alpha_K1, ((v_time_independent_potassium_current_K1_gate__alpha_K1 + v_time_independent_potassium_current_K1_gate__beta_K1)*(v_time_independent_potassium_current_K1_gate__alpha_K1 + v_time_independent_potassium_current_K1_gate__beta_K1))))));
        T a_v_time_independent_potassium_current_K1_gate__beta_K1 = T(0.0);
        a_v_time_independent_potassium_current_K1_gate__beta_K1 += a_v_time_independent_potassium_current_K1_gate__K1_infinity*((-m_div(v_time_independent_potassium_current_K1_gate__alpha_K1, ((v_time_independent_potassium_current_K1_gate__alpha_K1 + v_time_independent_potassium_current_K1_gate__beta_K1)*(v_time_independent_potassium_current_K1_gate__alpha_K1 + v_time_independent_potassium_current_K1_gate__beta_K1)))));
        a_y_0 += a_v_time_independent_potassium_current_K1_gate__beta_K1*(((m_div(((T(71.29534875031702)*m_exp((T(0.08032)*y[0]))) + (T(1.6207018112661692e-15)*m_exp((T(0.06175)*y[0])))), (T(1.0) + (T(2.0268841278228537e-21)*m_exp(((-T(0.5143))*y[0])))))) + (m_div(T(1.0424265069392937e-21)*((T(887.6412942021542)*m_exp((T(0.08032)*y[0]))) + (T(2.6246183178399503e-14)*m_exp((T(0.06175)*y[0]))))*m_exp(((-T(0.5143))*y[0])), ((T(1.0) + (T(2.0268841278228537e-21)*m_exp(((-T(0.5143))*y[0]))))*(T(1.0) + (T(2.0268841278228537e-21)*m_exp(((-T(0.5143))*y[0])))))))));
        a_y_0 += a_v_time_independent_potassium_current_K1_gate__alpha_K1*((m_div((-T(227.26033654832673))*m_exp((T(0.2385)*y[0])), ((T(1.0) + (T(934.1897338279555)*m_exp((T(0.2385)*y[0]))))*(T(1.0) + (T(934.1897338279555)*m_exp((T(0.2385)*y[0]))))))));
        a_y_0 += a_v_time_dependent_potassium_current__i_K*((y[6]*v_time_dependent_potassium_current_Xi_gate__Xi*v_time_dependent_potassium_current__g_K__scaled));
        T a_y_6 = T(0.0);
        a_y_6 += a_v_time_dependent_potassium_current__i_K*((v_time_dependent_potassium_current_Xi_gate__Xi*v_time_dependent_potassium_current__g_K__scaled*(T(77.56758438531939) + y[0])));
        T a_v_time_dependent_potassium_current_Xi_gate__Xi = T(0.0);
        a_v_time_dependent_potassium_current_Xi_gate__Xi += a_v_time_dependent_potassium_current__i_K*((y[6]*v_time_dependent_potassium_current__g_K__scaled*(T(77.56758438531939) + y[0])));
        T a_v_time_dependent_potassium_current__g_K__scaled = T(0.0);
        a_v_time_dependent_potassium_current__g_K__scaled += a_v_time_dependent_potassium_current__i_K*((y[6]*v_time_dependent_potassium_current_Xi_gate__Xi*(T(77.56758438531939) + y[0])));
        T a_p_2 = T(0.0);
        a_p_2 += a_v_time_dependent_potassium_current__g_K__scaled*(T(0.282));
        a_y_0 += a_v_time_dependent_potassium_current_Xi_gate__Xi*(((y[0] > (-T(100.0))) ? (((T(1.0)*chb::singularity_offset<T>()) > fabs((T(77.0) + y[0]))) ? (m_div(T(0.5)*((m_div(T(5.365555971121975)*(-T(2.837) + (T(2.837)*m_exp((T(0.04)*chb::singularity_offset<T>()))))*m_exp(((-T(0.04))*chb::singularity_offset<T>())), chb::singularity_offset<T>())) + (m_div(T(5.365555971121975)*(-T(2.837) + (T(2.837)*m_exp(((-T(0.04))*chb::singularity_offset<T>()))))*m_exp((T(0.04)*chb::singularity_offset<T>())), chb::singularity_offset<T>()))), chb::singularity_offset<T>())) : ((m_div(T(0.6088832916029218), (T(77.0) + y[0]))) - (m_div(T(0.00986387855766426)*(-T(2.837) + (T(61.72858759801112)*m_exp((T(0.04)*y[0]))))*m_exp(((-T(0.04))*y[0])), (T(77.0) + y[0]))) - (m_div(T(0.24659696394160646)*(-T(2.837) + (T(61.72858759801112)*m_exp((T(0.04)*y[0]))))*m_exp(((-T(0.04))*y[0])), ((T(77.0) + y[0])*(T(77.0) + y[0])))))) : T(0.0)));
        T a_p_1 = T(0.0);
        a_p_1 += a_v_slow_inward_current__i_si*((T(0.09)*y[4]*y[5]*(y[0] - v_slow_inward_current__E_si)));
        a_y_0 += a_v_slow_inward_current__i_si*((T(0.09)*p[1]*y[4]*y[5]));
        T a_v_slow_inward_current__E_si = T(0.0);
        a_v_slow_inward_current__E_si += a_v_slow_inward_current__i_si*(((-T(0.09))*p[1]*y[4]*y[5]));
        T a_y_4 = T(0.0);
        a_y_4 += a_v_slow_inward_current__i_si*((T(0.09)*p[1]*y[5]*(y[0] - v_slow_inward_current__E_si)));
        T a_y_5 = T(0.0);
        a_y_5 += a_v_slow_inward_current__i_si*((T(0.09)*p[1]*y[4]*(y[0] - v_slow_inward_current__E_si)));
        T a_y_7 = T(0.0);
        a_y_7 += a_v_slow_inward_current__E_si*((m_div((-T(13.0287)), y[7])));
        T a_p_4 = T(0.0);
        a_p_4 += a_v_plateau_potassium_current__i_Kp*((T(0.0183)*v_plateau_potassium_current__Kp*(T(87.8929017138025) + y[0])));
        a_y_0 += a_v_plateau_potassium_current__i_Kp*((T(0.0183)*p[4]*v_plateau_potassium_current__Kp));
        T a_v_plateau_potassium_current__Kp = T(0.0);
        a_v_plateau_potassium_current__Kp += a_v_plateau_potassium_current__i_Kp*((T(0.0183)*p[4]*(T(87.8929017138025) + y[0])));
        a_y_0 += a_v_plateau_potassium_current__Kp*((m_div(T(0.5849396175627496)*m_exp(((-T(0.16722408026755853))*y[0])), ((T(1.0) + (T(3.497938913025243)*m_exp(((-T(0.16722408026755853))*y[0]))))*(T(1.0) + (T(3.497938913025243)*m_exp(((-T(0.16722408026755853))*y[0]))))))));
        T a_p_0 = T(0.0);
        a_p_0 += a_v_fast_sodium_current__i_Na*((T(23.0)*y[2]*y[3]*(y[1]*y[1]*y[1])*(-T(54.79446393509185) + y[0])));
        T a_y_2 = T(0.0);
        a_y_2 += a_v_fast_sodium_current__i_Na*((T(23.0)*p[0]*y[3]*(y[1]*y[1]*y[1])*(-T(54.79446393509185) + y[0])));
        T a_y_3 = T(0.0);
        a_y_3 += a_v_fast_sodium_current__i_Na*((T(23.0)*p[0]*y[2]*(y[1]*y[1]*y[1])*(-T(54.79446393509185) + y[0])));
        T a_y_1 = T(0.0);
        a_y_1 += a_v_fast_sodium_current__i_Na*((T(69.0)*p[0]*y[2]*y[3]*(y[1]*y[1])*(-T(54.79446393509185) + y[0])));
        a_y_0 += a_v_fast_sodium_current__i_Na*((T(23.0)*p[0]*y[2]*y[3]*(y[1]*y[1]*y[1])));
        T a_p_5 = T(0.0);
        a_p_5 += a_v_background_current__i_b*((T(2.3475027) + (T(0.03921)*y[0])));
        a_y_0 += a_v_background_current__i_b*((T(0.03921)*p[5]));
        gy[0] += a_y_0;
        gy[1] += a_y_1;
        gy[2] += a_y_2;
        gy[3] += a_y_3;
        gy[4] += a_y_4;
        gy[5] += a_y_5;
        gy[6] += a_y_6;
        gy[7] += a_y_7;
        gp[0] += a_p_0;
        gp[1] += a_p_1;
        gp[2] += a_p_2;
        gp[3] += a_p_3;
        gp[4] += a_p_4;
        gp[5] += a_p_5;
    }
};

}  // namespace chb

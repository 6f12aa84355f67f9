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
        const T v_plateau_potassium_current__Kp = (T(1.0)/(T(1.0) + m_exp(((T(7.488) - y[0])/T(5.98)))));
        const T v_plateau_potassium_current__i_Kp = ((T(0.0183)*p[4])*v_plateau_potassium_current__Kp*(y[0] - (-T(87.8929017138025))));
        const T v_slow_inward_current__E_si = (T(7.7) - (T(13.0287)*m_log((y[7]/T(1.0)))));
        const T v_slow_inward_current__i_si = ((T(0.09)*p[1])*y[4]*y[5]*(y[0] - v_slow_inward_current__E_si));
        const T v_time_dependent_potassium_current_Xi_gate__Xi = ((y[0] > (-T(100.0))) ? (((chb::singularity_offset<T>()*T(1.0)) > fabs((y[0] + T(77.0)))) ? (((T(2.837)*(m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0)))/(((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(35.0)))))) + ((y[0] - (-T(77.0) - (chb::singularity_offset<T>()*T(1.0))))*(((T(2.837)*(m_exp((T(0.04)*((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0)))/(((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(35.0)))))) - ((T(2.837)*(m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0)))/(((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(35.0)))))))/(T(2.0)*(chb::singularity_offset<T>()*T(1.0))))) : ((T(2.837)*(m_exp((T(0.04)*(y[0] + T(77.0)))) - T(1.0)))/((y[0] + T(77.0))*m_exp((T(0.04)*(y[0] + T(35.0))))))) : T(1.0));
        const T v_time_dependent_potassium_current__g_K__scaled = (T(0.282)*p[2]);
        const T v_time_dependent_potassium_current__i_K = (v_time_dependent_potassium_current__g_K__scaled*y[6]*v_time_dependent_potassium_current_Xi_gate__Xi*(y[0] - (-T(77.56758438531939))));
        const T v_time_independent_potassium_current_K1_gate__alpha_K1 = (T(1.02)/(T(1.0) + m_exp((T(0.2385)*((y[0] - (-T(87.8929017138025))) - T(59.215))))));
        const T v_time_independent_potassium_current_K1_gate__beta_K1 = (((T(0.49124)*m_exp((T(0.08032)*((y[0] + T(5.476)) - (-T(87.8929017138025)))))) + (T(1.0)*m_exp((T(0.06175)*(y[0] - (-T(87.8929017138025) + T(594.31)))))))/(T(1.0) + m_exp(((-T(0.5143))*((y[0] - (-T(87.8929017138025))) + T(4.753))))));
        const T v_time_independent_potassium_current_K1_gate__K1_infinity = (v_time_independent_potassium_current_K1_gate__alpha_K1/(v_time_independent_potassium_current_K1_gate__alpha_K1 + v_time_independent_potassium_current_K1_gate__beta_K1));
        const T v_time_independent_potassium_current__g_K1__scaled = (T(0.6047)*p[3]);
        const T v_time_independent_potassium_current__i_K1 = (v_time_independent_potassium_current__g_K1__scaled*v_time_independent_potassium_current_K1_gate__K1_infinity*(y[0] - (-T(87.8929017138025))));
        const T v_fast_sodium_current_m_gate__alpha_m = (((chb::singularity_offset<T>()*T(10.0)) > fabs((y[0] + T(47.13)))) ? (((T(0.32)*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13)))/(T(1.0) - m_exp(((-T(0.1))*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13)))))) + ((y[0] - (-T(47.13) - (chb::singularity_offset<T>()*T(10.0))))*(((T(0.32)*((-T(47.13) + (chb::singularity_offset<T>()*T(10.0))) + T(47.13)))/(T(1.0) - m_exp(((-T(0.1))*((-T(47.13) + (chb::singularity_offset<T>()*T(10.0))) + T(47.13)))))) - ((T(0.32)*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13)))/(T(1.0) - m_exp(((-T(0.1))*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13)))))))/(T(2.0)*(chb::singularity_offset<T>()*T(10.0))))) : ((T(0.32)*(y[0] + T(47.13)))/(T(1.0) - m_exp(((-T(0.1))*(y[0] + T(47.13)))))));
        const T v_fast_sodium_current_m_gate__beta_m = (T(0.08)*m_exp(((-y[0])/T(11.0))));
        const T v_fast_sodium_current_h_gate__alpha_h = ((y[0] < (-T(40.0))) ? (T(0.135)*m_exp(((T(80.0) + y[0])/(-T(6.8))))) : T(0.0));
        const T v_fast_sodium_current_h_gate__beta_h = ((y[0] < (-T(40.0))) ? ((T(3.56)*m_exp((T(0.079)*y[0]))) + (T(310000.0)*m_exp((T(0.35)*y[0])))) : (T(1.0)/(T(0.13)*(T(1.0) + m_exp(((y[0] + T(10.66))/(-T(11.1))))))));
        const T v_fast_sodium_current_j_gate__alpha_j = ((y[0] < (-T(40.0))) ? (((((-T(127140.0))*m_exp((T(0.2444)*y[0]))) - (T(3.474e-05)*m_exp(((-T(0.04391))*y[0]))))*(y[0] + T(37.78)))/(T(1.0) + m_exp((T(0.311)*(y[0] + T(79.23)))))) : T(0.0));
        const T v_fast_sodium_current_j_gate__beta_j = ((y[0] < (-T(40.0))) ? ((T(0.1212)*m_exp(((-T(0.01052))*y[0])))/(T(1.0) + m_exp(((-T(0.1378))*(y[0] + T(40.14)))))) : ((T(0.3)*m_exp(((-T(2.535e-07))*y[0])))/(T(1.0) + m_exp(((-T(0.1))*(y[0] + T(32.0)))))));
        const T v_slow_inward_current_d_gate__alpha_d = ((T(0.095)*m_exp(((-T(0.01))*(y[0] - T(5.0)))))/(T(1.0) + m_exp(((-T(0.072))*(y[0] - T(5.0))))));
        const T v_slow_inward_current_d_gate__beta_d = ((T(0.07)*m_exp(((-T(0.017))*(y[0] + T(44.0)))))/(T(1.0) + m_exp((T(0.05)*(y[0] + T(44.0))))));
        const T v_slow_inward_current_f_gate__alpha_f = ((T(0.012)*m_exp(((-T(0.008))*(y[0] + T(28.0)))))/(T(1.0) + m_exp((T(0.15)*(y[0] + T(28.0))))));
        const T v_slow_inward_current_f_gate__beta_f = ((T(0.0065)*m_exp(((-T(0.02))*(y[0] + T(30.0)))))/(T(1.0) + m_exp(((-T(0.2))*(y[0] + T(30.0))))));
        const T v_time_dependent_potassium_current_X_gate__alpha_X = ((T(0.0005)*m_exp((T(0.083)*(y[0] + T(50.0)))))/(T(1.0) + m_exp((T(0.057)*(y[0] + T(50.0))))));
        const T v_time_dependent_potassium_current_X_gate__beta_X = ((T(0.0013)*m_exp(((-T(0.06))*(y[0] + T(20.0)))))/(T(1.0) + m_exp(((-T(0.04))*(y[0] + T(20.0))))));
        dy[0] = (((-T(1.0))/T(1.0))*(v_membrane__I_stim + v_fast_sodium_current__i_Na + v_slow_inward_current__i_si + v_time_dependent_potassium_current__i_K + v_time_independent_potassium_current__i_K1 + v_plateau_potassium_current__i_Kp + v_background_current__i_b));
        dy[1] = ((v_fast_sodium_current_m_gate__alpha_m*(T(1.0) - y[1])) - (v_fast_sodium_current_m_gate__beta_m*y[1]));
        dy[2] = ((v_fast_sodium_current_h_gate__alpha_h*(T(1.0) - y[2])) - (v_fast_sodium_current_h_gate__beta_h*y[2]));
        dy[3] = ((v_fast_sodium_current_j_gate__alpha_j*(T(1.0) - y[3])) - (v_fast_sodium_current_j_gate__beta_j*y[3]));
        dy[4] = ((v_slow_inward_current_d_gate__alpha_d*(T(1.0) - y[4])) - (v_slow_inward_current_d_gate__beta_d*y[4]));
        dy[5] = ((v_slow_inward_current_f_gate__alpha_f*(T(1.0) - y[5])) - (v_slow_inward_current_f_gate__beta_f*y[5]));
        dy[6] = ((v_time_dependent_potassium_current_X_gate__alpha_X*(T(1.0) - y[6])) - (v_time_dependent_potassium_current_X_gate__beta_X*y[6]));
        dy[7] = ((((-T(0.0001))/T(1.0))*v_slow_inward_current__i_si) + (T(0.07)*(T(0.0001) - y[7])));
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
        const T v_plateau_potassium_current__Kp = (T(1.0)/(T(1.0) + m_exp(((T(7.488) - y[0])/T(5.98)))));
        const T v_plateau_potassium_current__i_Kp = ((T(0.0183)*p[4])*v_plateau_potassium_current__Kp*(y[0] - (-T(87.8929017138025))));
        const T v_slow_inward_current__E_si = (T(7.7) - (T(13.0287)*m_log((y[7]/T(1.0)))));
        const T v_slow_inward_current__i_si = ((T(0.09)*p[1])*y[4]*y[5]*(y[0] - v_slow_inward_current__E_si));
        const T v_time_dependent_potassium_current_Xi_gate__Xi = ((y[0] > (-T(100.0))) ? (((chb::singularity_offset<T>()*T(1.0)) > fabs((y[0] + T(77.0)))) ? (((T(2.837)*(m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0)))/(((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(35.0)))))) + ((y[0] - (-T(77.0) - (chb::singularity_offset<T>()*T(1.0))))*(((T(2.837)*(m_exp((T(0.04)*((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0)))/(((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(35.0)))))) - ((T(2.837)*(m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0)))/(((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(35.0)))))))/(T(2.0)*(chb::singularity_offset<T>()*T(1.0))))) : ((T(2.837)*(m_exp((T(0.04)*(y[0] + T(77.0)))) - T(1.0)))/((y[0] + T(77.0))*m_exp((T(0.04)*(y[0] + T(35.0))))))) : T(1.0));
        const T v_time_dependent_potassium_current__g_K__scaled = (T(0.282)*p[2]);
        const T v_time_dependent_potassium_current__i_K = (v_time_dependent_potassium_current__g_K__scaled*y[6]*v_time_dependent_potassium_current_Xi_gate__Xi*(y[0] - (-T(77.56758438531939))));
        const T v_time_independent_potassium_current_K1_gate__alpha_K1 = (T(1.02)/(T(1.0) + m_exp((T(0.2385)*((y[0] - (-T(87.8929017138025))) - T(59.215))))));
        const T v_time_independent_potassium_current_K1_gate__beta_K1 = (((T(0.49124)*m_exp((T(0.08032)*((y[0] + T(5.476)) - (-T(87.8929017138025)))))) + (T(1.0)*m_exp((T(0.06175)*(y[0] - (-T(87.8929017138025) + T(594.31)))))))/(T(1.0) + m_exp(((-T(0.5143))*((y[0] - (-T(87.8929017138025))) + T(4.753))))));
        const T v_time_independent_potassium_current_K1_gate__K1_infinity = (v_time_independent_potassium_current_K1_gate__alpha_K1/(v_time_independent_potassium_current_K1_gate__alpha_K1 + v_time_independent_potassium_current_K1_gate__beta_K1));
        const T v_time_independent_potassium_current__g_K1__scaled = (T(0.6047)*p[3]);
        const T v_time_independent_potassium_current__i_K1 = (v_time_independent_potassium_current__g_K1__scaled*v_time_independent_potassium_current_K1_gate__K1_infinity*(y[0] - (-T(87.8929017138025))));
        const T v_fast_sodium_current_m_gate__alpha_m = (((chb::singularity_offset<T>()*T(10.0)) > fabs((y[0] + T(47.13)))) ? (((T(0.32)*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13)))/(T(1.0) - m_exp(((-T(0.1))*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13)))))) + ((y[0] - (-T(47.13) - (chb::singularity_offset<T>()*T(10.0))))*(((T(0.32)*((-T(47.13) + (chb::singularity_offset<T>()*T(10.0))) + T(47.13)))/(T(1.0) - m_exp(((-T(0.1))*((-T(47.13) + (chb::singularity_offset<T>()*T(10.0))) + T(47.13)))))) - ((T(0.32)*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13)))/(T(1.0) - m_exp(((-T(0.1))*((-T(47.13) - (chb::singularity_offset<T>()*T(10.0))) + T(47.13)))))))/(T(2.0)*(chb::singularity_offset<T>()*T(10.0))))) : ((T(0.32)*(y[0] + T(47.13)))/(T(1.0) - m_exp(((-T(0.1))*(y[0] + T(47.13)))))));
        const T v_fast_sodium_current_m_gate__beta_m = (T(0.08)*m_exp(((-y[0])/T(11.0))));
        const T v_fast_sodium_current_h_gate__alpha_h = ((y[0] < (-T(40.0))) ? (T(0.135)*m_exp(((T(80.0) + y[0])/(-T(6.8))))) : T(0.0));
        const T v_fast_sodium_current_h_gate__beta_h = ((y[0] < (-T(40.0))) ? ((T(3.56)*m_exp((T(0.079)*y[0]))) + (T(310000.0)*m_exp((T(0.35)*y[0])))) : (T(1.0)/(T(0.13)*(T(1.0) + m_exp(((y[0] + T(10.66))/(-T(11.1))))))));
        const T v_fast_sodium_current_j_gate__alpha_j = ((y[0] < (-T(40.0))) ? (((((-T(127140.0))*m_exp((T(0.2444)*y[0]))) - (T(3.474e-05)*m_exp(((-T(0.04391))*y[0]))))*(y[0] + T(37.78)))/(T(1.0) + m_exp((T(0.311)*(y[0] + T(79.23)))))) : T(0.0));
        const T v_fast_sodium_current_j_gate__beta_j = ((y[0] < (-T(40.0))) ? ((T(0.1212)*m_exp(((-T(0.01052))*y[0])))/(T(1.0) + m_exp(((-T(0.1378))*(y[0] + T(40.14)))))) : ((T(0.3)*m_exp(((-T(2.535e-07))*y[0])))/(T(1.0) + m_exp(((-T(0.1))*(y[0] + T(32.0)))))));
        const T v_slow_inward_current_d_gate__alpha_d = ((T(0.095)*m_exp(((-T(0.01))*(y[0] - T(5.0)))))/(T(1.0) + m_exp(((-T(0.072))*(y[0] - T(5.0))))));
        const T v_slow_inward_current_d_gate__beta_d = ((T(0.07)*m_exp(((-T(0.017))*(y[0] + T(44.0)))))/(T(1.0) + m_exp((T(0.05)*(y[0] + T(44.0))))));
        const T v_slow_inward_current_f_gate__alpha_f = ((T(0.012)*m_exp(((-T(0.008))*(y[0] + T(28.0)))))/(T(1.0) + m_exp((T(0.15)*(y[0] + T(28.0))))));
        const T v_slow_inward_current_f_gate__beta_f = ((T(0.0065)*m_exp(((-T(0.02))*(y[0] + T(30.0)))))/(T(1.0) + m_exp(((-T(0.2))*(y[0] + T(30.0))))));
        const T v_time_dependent_potassium_current_X_gate__alpha_X = ((T(0.0005)*m_exp((T(0.083)*(y[0] + T(50.0)))))/(T(1.0) + m_exp((T(0.057)*(y[0] + T(50.0))))));
        const T v_time_dependent_potassium_current_X_gate__beta_X = ((T(0.0013)*m_exp(((-T(0.06))*(y[0] + T(20.0)))))/(T(1.0) + m_exp(((-T(0.04))*(y[0] + T(20.0))))));
        rate[0] = (((-T(1.0))/T(1.0))*(v_membrane__I_stim + v_fast_sodium_current__i_Na + v_slow_inward_current__i_si + v_time_dependent_potassium_current__i_K + v_time_independent_potassium_current__i_K1 + v_plateau_potassium_current__i_Kp + v_background_current__i_b));
        inf[1] = (-(v_fast_sodium_current_m_gate__alpha_m/(-v_fast_sodium_current_m_gate__alpha_m - v_fast_sodium_current_m_gate__beta_m)));
        rate[1] = (-v_fast_sodium_current_m_gate__alpha_m - v_fast_sodium_current_m_gate__beta_m);
        inf[2] = (-(v_fast_sodium_current_h_gate__alpha_h/(-v_fast_sodium_current_h_gate__alpha_h - v_fast_sodium_current_h_gate__beta_h)));
        rate[2] = (-v_fast_sodium_current_h_gate__alpha_h - v_fast_sodium_current_h_gate__beta_h);
        inf[3] = (-(v_fast_sodium_current_j_gate__alpha_j/(-v_fast_sodium_current_j_gate__alpha_j - v_fast_sodium_current_j_gate__beta_j)));
        rate[3] = (-v_fast_sodium_current_j_gate__alpha_j - v_fast_sodium_current_j_gate__beta_j);
        inf[4] = (-(v_slow_inward_current_d_gate__alpha_d/(-v_slow_inward_current_d_gate__alpha_d - v_slow_inward_current_d_gate__beta_d)));
        rate[4] = (-v_slow_inward_current_d_gate__alpha_d - v_slow_inward_current_d_gate__beta_d);
        inf[5] = (-(v_slow_inward_current_f_gate__alpha_f/(-v_slow_inward_current_f_gate__alpha_f - v_slow_inward_current_f_gate__beta_f)));
        rate[5] = (-v_slow_inward_current_f_gate__alpha_f - v_slow_inward_current_f_gate__beta_f);
        inf[6] = (-(v_time_dependent_potassium_current_X_gate__alpha_X/(-v_time_dependent_potassium_current_X_gate__alpha_X - v_time_dependent_potassium_current_X_gate__beta_X)));
        rate[6] = (-v_time_dependent_potassium_current_X_gate__alpha_X - v_time_dependent_potassium_current_X_gate__beta_X);
        rate[7] = ((((-T(0.0001))/T(1.0))*v_slow_inward_current__i_si) + (T(0.07)*(T(0.0001) - y[7])));
    }

    // Total ionic current in uA/cm^2 (GetIIonic): the dV/dt currents without
    // the stimulus.
    template <typename T>
    CHB_HD static T iionic(const T* __restrict__ y, T cm, const T* __restrict__ p) {
        (void)cm; (void)p;
        const T stim = T(0.0); (void)stim;
        const T v_background_current__i_b = ((T(0.03921)*p[5])*(y[0] - (-T(59.87))));
        const T v_fast_sodium_current__i_Na = ((T(23.0)*p[0])*(y[1]*y[1]*y[1])*y[2]*y[3]*(y[0] - T(54.79446393509185)));
        const T v_plateau_potassium_current__Kp = (T(1.0)/(T(1.0) + m_exp(((T(7.488) - y[0])/T(5.98)))));
        const T v_plateau_potassium_current__i_Kp = ((T(0.0183)*p[4])*v_plateau_potassium_current__Kp*(y[0] - (-T(87.8929017138025))));
        const T v_slow_inward_current__E_si = (T(7.7) - (T(13.0287)*m_log((y[7]/T(1.0)))));
        const T v_slow_inward_current__i_si = ((T(0.09)*p[1])*y[4]*y[5]*(y[0] - v_slow_inward_current__E_si));
        const T v_time_dependent_potassium_current_Xi_gate__Xi = ((y[0] > (-T(100.0))) ? (((chb::singularity_offset<T>()*T(1.0)) > fabs((y[0] + T(77.0)))) ? (((T(2.837)*(m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0)))/(((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(35.0)))))) + ((y[0] - (-T(77.0) - (chb::singularity_offset<T>()*T(1.0))))*(((T(2.837)*(m_exp((T(0.04)*((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0)))/(((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) + (chb::singularity_offset<T>()*T(1.0))) + T(35.0)))))) - ((T(2.837)*(m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0)))) - T(1.0)))/(((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(77.0))*m_exp((T(0.04)*((-T(77.0) - (chb::singularity_offset<T>()*T(1.0))) + T(35.0)))))))/(T(2.0)*(chb::singularity_offset<T>()*T(1.0))))) : ((T(2.837)*(m_exp((T(0.04)*(y[0] + T(77.0)))) - T(1.0)))/((y[0] + T(77.0))*m_exp((T(0.04)*(y[0] + T(35.0))))))) : T(1.0));
        const T v_time_dependent_potassium_current__g_K__scaled = (T(0.282)*p[2]);
        const T v_time_dependent_potassium_current__i_K = (v_time_dependent_potassium_current__g_K__scaled*y[6]*v_time_dependent_potassium_current_Xi_gate__Xi*(y[0] - (-T(77.56758438531939))));
        const T v_time_independent_potassium_current_K1_gate__alpha_K1 = (T(1.02)/(T(1.0) + m_exp((T(0.2385)*((y[0] - (-T(87.8929017138025))) - T(59.215))))));
        const T v_time_independent_potassium_current_K1_gate__beta_K1 = (((T(0.49124)*m_exp((T(0.08032)*((y[0] + T(5.476)) - (-T(87.8929017138025)))))) + (T(1.0)*m_exp((T(0.06175)*(y[0] - (-T(87.8929017138025) + T(594.31)))))))/(T(1.0) + m_exp(((-T(0.5143))*((y[0] - (-T(87.8929017138025))) + T(4.753))))));
        const T v_time_independent_potassium_current_K1_gate__K1_infinity = (v_time_independent_potassium_current_K1_gate__alpha_K1/(v_time_independent_potassium_current_K1_gate__alpha_K1 + v_time_independent_potassium_current_K1_gate__beta_K1));
        const T v_time_independent_potassium_current__g_K1__scaled = (T(0.6047)*p[3]);
        const T v_time_independent_potassium_current__i_K1 = (v_time_independent_potassium_current__g_K1__scaled*v_time_independent_potassium_current_K1_gate__K1_infinity*(y[0] - (-T(87.8929017138025))));
        return (v_background_current__i_b + v_fast_sodium_current__i_Na + v_plateau_potassium_current__i_Kp + v_slow_inward_current__i_si + v_time_dependent_potassium_current__i_K + v_time_independent_potassium_current__i_K1);
    }
};

}  // namespace chb

// Generated by chaste_b200/codegen/emit.py from heart/src/odes/cellml/TenTusscher2006Epi.cellml.
// Do not edit: re-run `python -m chaste_b200.codegen.emit` instead.
#pragma once
#include "cellmodel_common.h"

namespace chb {

struct TenTusscher2006Epi {
    static constexpr const char* kName = "tentusscher_model_2006_epi";
    static constexpr int kNumStates = 19;
    static constexpr int kNumParams = 9;
    static constexpr bool kCurrentPerCapacitance = true;
    static constexpr double kInitialStates[19] = {-85.23, 0.00621, 0.4712, 0.0095, 0.00172, 0.7444, 0.7045, 3.373e-05, 0.7888, 0.9755, 0.9953, 0.999998, 2.42e-08, 0.9073, 0.000126, 3.64, 0.00036, 8.604, 136.89};
    static constexpr const char* kStateNames[19] = {"V", "Xr1", "Xr2", "Xs", "m", "h", "j", "d", "f", "f2", "fCass", "s", "r", "R_prime", "Ca_i", "Ca_SR", "Ca_ss", "Na_i", "K_i"};
    static constexpr const char* kParamNames[9] = {"g_Na", "g_CaL", "g_Kr", "g_Ks", "g_K1", "g_to", "ScaleFactorGks", "ScaleFactorGkr", "ScaleFactorIto"};
    // 1 where the state is advanced by Rush-Larsen (ODE affine in itself)
    static constexpr bool kRushLarsen[19] = {false, true, true, true, true, true, true, true, true, true, true, true, true, true, false, false, false, false, false};
    CHB_HD static constexpr bool rush_larsen(int i) { return i == 1 || i == 2 || i == 3 || i == 4 || i == 5 || i == 6 || i == 7 || i == 8 || i == 9 || i == 10 || i == 11 || i == 12 || i == 13; }
    // range class per state: 1 gate in [0,1], 2 concentration > 0, 0 unchecked
    static constexpr int kRangeClass[19] = {0, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 2, 2, 2, 2, 2};
    CHB_HD static constexpr int range_class(int i) { return (i == 1 || i == 2 || i == 3 || i == 4 || i == 5 || i == 6 || i == 7 || i == 8 || i == 9 || i == 10 || i == 11 || i == 12 || i == 13) ? 1 : ((i == 14 || i == 15 || i == 16 || i == 17 || i == 18) ? 2 : 0); }

    // dy/dt for every state at (y, stim) where stim is the Chaste area stimulus
    // in uA/cm^2 and cm the Chaste capacitance in uF/cm^2.  y[0] is the voltage.
    template <typename T>
    CHB_HD static void rhs(const T* __restrict__ y, T stim, T cm,
                                  const T* __restrict__ p, T* __restrict__ dy) {
        (void)stim; (void)cm; (void)p;
        const T v_L_type_Ca_current__i_CaL = (((chb::singularity_offset<T>()*T(13.356880329847824)) > fabs((y[0] - T(15.0)))) ? ((((((T(3.98e-05)*p[1])*y[7]*y[8]*y[9]*y[10]*T(4.0)*((T(15.0) - (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*(T(96485.3415)*T(96485.3415)))/(T(8314.472)*T(310.0)))*((T(0.25)*y[16]*m_exp(((T(2.0)*((T(15.0) - (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0))))) - T(2.0)))/(m_exp(((T(2.0)*((T(15.0) - (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0)))) - T(1.0))) + ((y[0] - (T(15.0) - (chb::singularity_offset<T>()*T(13.356880329847824))))*((((((T(3.98e-05)*p[1])*y[7]*y[8]*y[9]*y[10]*T(4.0)*((T(15.0) + (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*(T(96485.3415)*T(96485.3415)))/(T(8314.472)*T(310.0)))*((T(0.25)*y[16]*m_exp(((T(2.0)*((T(15.0) + (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0))))) - T(2.0)))/(m_exp(((T(2.0)*((T(15.0) + (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0)))) - T(1.0))) - (((((T(3.98e-05)*p[1])*y[7]*y[8]*y[9]*y[10]*T(4.0)*((T(15.0) - (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*(T(96485.3415)*T(96485.3415)))/(T(8314.472)*T(310.0)))*((T(0.25)*y[16]*m_exp(((T(2.0)*((T(15.0) - (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0))))) - T(2.0)))/(m_exp(((T(2.0)*((T(15.0) - (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0)))) - T(1.0))))/(T(2.0)*(chb::singularity_offset<T>()*T(13.356880329847824))))) : (((((T(3.98e-05)*p[1])*y[7]*y[8]*y[9]*y[10]*T(4.0)*(y[0] - T(15.0))*(T(96485.3415)*T(96485.3415)))/(T(8314.472)*T(310.0)))*((T(0.25)*y[16]*m_exp(((T(2.0)*(y[0] - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0))))) - T(2.0)))/(m_exp(((T(2.0)*(y[0] - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0)))) - T(1.0))));
        const T v_reversal_potentials__E_Ca = (((T(0.5)*T(8314.472)*T(310.0))/T(96485.3415))*m_log((T(2.0)/y[14])));
        const T v_calcium_background_current__i_b_Ca = (T(0.000592)*(y[0] - v_reversal_potentials__E_Ca));
        const T v_calcium_pump_current__i_p_Ca = ((T(0.1238)*y[14])/(y[14] + T(0.0005)));
        const T v_reversal_potentials__E_Na = (((T(8314.472)*T(310.0))/T(96485.3415))*m_log((T(140.0)/y[17])));
        const T v_fast_sodium_current__i_Na = ((T(14.838)*p[0])*(y[4]*y[4]*y[4])*y[5]*y[6]*(y[0] - v_reversal_potentials__E_Na));
        const T v_reversal_potentials__E_K = (((T(8314.472)*T(310.0))/T(96485.3415))*m_log((T(5.4)/y[18])));
        const T v_inward_rectifier_potassium_current__alpha_K1 = (T(0.1)/(T(1.0) + m_exp((T(0.06)*((y[0] - v_reversal_potentials__E_K) - T(200.0))))));
        const T v_inward_rectifier_potassium_current__beta_K1 = (((T(3.0)*m_exp((T(0.0002)*((y[0] - v_reversal_potentials__E_K) + T(100.0))))) + m_exp((T(0.1)*((y[0] - v_reversal_potentials__E_K) - T(10.0)))))/(T(1.0) + m_exp(((-T(0.5))*(y[0] - v_reversal_potentials__E_K)))));
        const T v_inward_rectifier_potassium_current__xK1_inf = (v_inward_rectifier_potassium_current__alpha_K1/(v_inward_rectifier_potassium_current__alpha_K1 + v_inward_rectifier_potassium_current__beta_K1));
        const T v_inward_rectifier_potassium_current__i_K1 = ((T(5.405)*p[4])*v_inward_rectifier_potassium_current__xK1_inf*(y[0] - v_reversal_potentials__E_K));
        const T v_membrane__i_Stim = (stim/cm);
        const T v_potassium_pump_current__i_p_K = ((T(0.0146)*(y[0] - v_reversal_potentials__E_K))/(T(1.0) + m_exp(((T(25.0) - y[0])/T(5.98)))));
        const T v_rapid_time_dependent_potassium_current__i_Kr = (p[7]*(T(0.153)*p[2])*(T(0.4303314829119352)*m_sqrt(T(5.4)))*y[1]*y[2]*(y[0] - v_reversal_potentials__E_K));
        const T v_reversal_potentials__E_Ks = (((T(8314.472)*T(310.0))/T(96485.3415))*m_log(((T(5.4) + (T(0.03)*T(140.0)))/(y[18] + (T(0.03)*y[17])))));
        const T v_slow_time_dependent_potassium_current__i_Ks = (p[6]*(T(0.392)*p[3])*(y[3]*y[3])*(y[0] - v_reversal_potentials__E_Ks));
        const T v_sodium_background_current__i_b_Na = (T(0.00029)*(y[0] - v_reversal_potentials__E_Na));
        const T v_sodium_calcium_exchanger_current__i_NaCa = ((T(1000.0)*((m_exp(((T(0.35)*y[0]*T(96485.3415))/(T(8314.472)*T(310.0))))*(y[17]*y[17]*y[17])*T(2.0)) - (m_exp((((T(0.35) - T(1.0))*y[0]*T(96485.3415))/(T(8314.472)*T(310.0))))*(T(140.0)*T(140.0)*T(140.0))*y[14]*T(2.5))))/(((T(87.5)*T(87.5)*T(87.5)) + (T(140.0)*T(140.0)*T(140.0)))*(T(1.38) + T(2.0))*(T(1.0) + (T(0.1)*m_exp((((T(0.35) - T(1.0))*y[0]*T(96485.3415))/(T(8314.472)*T(310.0))))))));
        const T v_sodium_potassium_pump_current__i_NaK = (((((T(2.724)*T(5.4))/(T(5.4) + T(1.0)))*y[17])/(y[17] + T(40.0)))/(T(1.0) + (T(0.1245)*m_exp((((-T(0.1))*y[0]*T(96485.3415))/(T(8314.472)*T(310.0))))) + (T(0.0353)*m_exp((((-y[0])*T(96485.3415))/(T(8314.472)*T(310.0)))))));
        const T v_transient_outward_current__i_to = (p[8]*(T(0.294)*p[5])*y[12]*y[11]*(y[0] - v_reversal_potentials__E_K));
        const T v_rapid_time_dependent_potassium_current_Xr1_gate__alpha_xr1 = (T(450.0)/(T(1.0) + m_exp(((-T(45.0) - y[0])/T(10.0)))));
        const T v_rapid_time_dependent_potassium_current_Xr1_gate__beta_xr1 = (T(6.0)/(T(1.0) + m_exp(((y[0] + T(30.0))/T(11.5)))));
        const T v_rapid_time_dependent_potassium_current_Xr1_gate__tau_xr1 = (v_rapid_time_dependent_potassium_current_Xr1_gate__alpha_xr1*v_rapid_time_dependent_potassium_current_Xr1_gate__beta_xr1);
        const T v_rapid_time_dependent_potassium_current_Xr1_gate__xr1_inf = (T(1.0)/(T(1.0) + m_exp(((-T(26.0) - y[0])/T(7.0)))));
        const T v_rapid_time_dependent_potassium_current_Xr2_gate__alpha_xr2 = (T(3.0)/(T(1.0) + m_exp(((-T(60.0) - y[0])/T(20.0)))));
        const T v_rapid_time_dependent_potassium_current_Xr2_gate__beta_xr2 = (T(1.12)/(T(1.0) + m_exp(((y[0] - T(60.0))/T(20.0)))));
        const T v_rapid_time_dependent_potassium_current_Xr2_gate__tau_xr2 = (v_rapid_time_dependent_potassium_current_Xr2_gate__alpha_xr2*v_rapid_time_dependent_potassium_current_Xr2_gate__beta_xr2);
        const T v_rapid_time_dependent_potassium_current_Xr2_gate__xr2_inf = (T(1.0)/(T(1.0) + m_exp(((y[0] + T(88.0))/T(24.0)))));
        const T v_slow_time_dependent_potassium_current_Xs_gate__alpha_xs = (T(1400.0)/m_sqrt((T(1.0) + m_exp(((T(5.0) - y[0])/T(6.0))))));
        const T v_slow_time_dependent_potassium_current_Xs_gate__beta_xs = (T(1.0)/(T(1.0) + m_exp(((y[0] - T(35.0))/T(15.0)))));
        const T v_slow_time_dependent_potassium_current_Xs_gate__tau_xs = ((v_slow_time_dependent_potassium_current_Xs_gate__alpha_xs*v_slow_time_dependent_potassium_current_Xs_gate__beta_xs) + T(80.0));
        const T v_slow_time_dependent_potassium_current_Xs_gate__xs_inf = (T(1.0)/(T(1.0) + m_exp(((-T(5.0) - y[0])/T(14.0)))));
        const T v_fast_sodium_current_m_gate__m_inf = (T(1.0)/((T(1.0) + m_exp(((-T(56.86) - y[0])/T(9.03))))*(T(1.0) + m_exp(((-T(56.86) - y[0])/T(9.03))))));
        const T v_fast_sodium_current_m_gate__alpha_m = (T(1.0)/(T(1.0) + m_exp(((-T(60.0) - y[0])/T(5.0)))));
        const T v_fast_sodium_current_m_gate__beta_m = ((T(0.1)/(T(1.0) + m_exp(((y[0] + T(35.0))/T(5.0))))) + (T(0.1)/(T(1.0) + m_exp(((y[0] - T(50.0))/T(200.0))))));
        const T v_fast_sodium_current_m_gate__tau_m = (v_fast_sodium_current_m_gate__alpha_m*v_fast_sodium_current_m_gate__beta_m);
        const T v_fast_sodium_current_h_gate__h_inf = (T(1.0)/((T(1.0) + m_exp(((y[0] + T(71.55))/T(7.43))))*(T(1.0) + m_exp(((y[0] + T(71.55))/T(7.43))))));
        const T v_fast_sodium_current_h_gate__alpha_h = ((y[0] < (-T(40.0))) ? (T(0.057)*m_exp(((-(y[0] + T(80.0)))/T(6.8)))) : T(0.0));
        const T v_fast_sodium_current_h_gate__beta_h = ((y[0] < (-T(40.0))) ? ((T(2.7)*m_exp((T(0.079)*y[0]))) + (T(310000.0)*m_exp((T(0.3485)*y[0])))) : (T(0.77)/(T(0.13)*(T(1.0) + m_exp(((y[0] + T(10.66))/(-T(11.1))))))));
        const T v_fast_sodium_current_h_gate__tau_h = (T(1.0)/(v_fast_sodium_current_h_gate__alpha_h + v_fast_sodium_current_h_gate__beta_h));
        const T v_fast_sodium_current_j_gate__j_inf = (T(1.0)/((T(1.0) + m_exp(((y[0] + T(71.55))/T(7.43))))*(T(1.0) + m_exp(((y[0] + T(71.55))/T(7.43))))));
        const T v_fast_sodium_current_j_gate__alpha_j = ((y[0] < (-T(40.0))) ? (((((-T(25428.0))*m_exp((T(0.2444)*y[0]))) - (T(6.948e-06)*m_exp(((-T(0.04391))*y[0]))))*(y[0] + T(37.78)))/(T(1.0) + m_exp((T(0.311)*(y[0] + T(79.23)))))) : T(0.0));
        const T v_fast_sodium_current_j_gate__beta_j = ((y[0] < (-T(40.0))) ? ((T(0.02424)*m_exp(((-T(0.01052))*y[0])))/(T(1.0) + m_exp(((-T(0.1378))*(y[0] + T(40.14)))))) : ((T(0.6)*m_exp((T(0.057)*y[0])))/(T(1.0) + m_exp(((-T(0.1))*(y[0] + T(32.0)))))));
        const T v_fast_sodium_current_j_gate__tau_j = (T(1.0)/(v_fast_sodium_current_j_gate__alpha_j + v_fast_sodium_current_j_gate__beta_j));
        const T v_L_type_Ca_current_d_gate__d_inf = (T(1.0)/(T(1.0) + m_exp(((-T(8.0) - y[0])/T(7.5)))));
        const T v_L_type_Ca_current_d_gate__alpha_d = ((T(1.4)/(T(1.0) + m_exp(((-T(35.0) - y[0])/T(13.0))))) + T(0.25));
        const T v_L_type_Ca_current_d_gate__beta_d = (T(1.4)/(T(1.0) + m_exp(((y[0] + T(5.0))/T(5.0)))));
        const T v_L_type_Ca_current_d_gate__gamma_d = (T(1.0)/(T(1.0) + m_exp(((T(50.0) - y[0])/T(20.0)))));
        const T v_L_type_Ca_current_d_gate__tau_d = ((v_L_type_Ca_current_d_gate__alpha_d*v_L_type_Ca_current_d_gate__beta_d) + v_L_type_Ca_current_d_gate__gamma_d);
        const T v_L_type_Ca_current_f_gate__f_inf = (T(1.0)/(T(1.0) + m_exp(((y[0] + T(20.0))/T(7.0)))));
        const T v_L_type_Ca_current_f_gate__tau_f = ((T(1102.5)*m_exp(((-((y[0] + T(27.0))*(y[0] + T(27.0))))/T(225.0)))) + (T(200.0)/(T(1.0) + m_exp(((T(13.0) - y[0])/T(10.0))))) + (T(180.0)/(T(1.0) + m_exp(((y[0] + T(30.0))/T(10.0))))) + T(20.0));
        const T v_L_type_Ca_current_f2_gate__f2_inf = ((T(0.67)/(T(1.0) + m_exp(((y[0] + T(35.0))/T(7.0))))) + T(0.33));
        const T v_L_type_Ca_current_f2_gate__tau_f2 = ((T(562.0)*m_exp(((-((y[0] + T(27.0))*(y[0] + T(27.0))))/T(240.0)))) + (T(31.0)/(T(1.0) + m_exp(((T(25.0) - y[0])/T(10.0))))) + (T(80.0)/(T(1.0) + m_exp(((y[0] + T(30.0))/T(10.0))))));
        const T v_L_type_Ca_current_fCass_gate__fCass_inf = ((T(0.6)/(T(1.0) + ((y[16]/T(0.05))*(y[16]/T(0.05))))) + T(0.4));
        const T v_L_type_Ca_current_fCass_gate__tau_fCass = ((T(80.0)/(T(1.0) + ((y[16]/T(0.05))*(y[16]/T(0.05))))) + T(2.0));
        const T v_transient_outward_current_s_gate__s_inf = (T(1.0)/(T(1.0) + m_exp(((y[0] + T(20.0))/T(5.0)))));
        const T v_transient_outward_current_s_gate__tau_s = ((T(85.0)*m_exp(((-((y[0] + T(45.0))*(y[0] + T(45.0))))/T(320.0)))) + (T(5.0)/(T(1.0) + m_exp(((y[0] - T(20.0))/T(5.0))))) + T(3.0));
        const T v_transient_outward_current_r_gate__r_inf = (T(1.0)/(T(1.0) + m_exp(((T(20.0) - y[0])/T(6.0)))));
        const T v_transient_outward_current_r_gate__tau_r = ((T(9.5)*m_exp(((-((y[0] + T(40.0))*(y[0] + T(40.0))))/T(1800.0)))) + T(0.8));
        const T v_calcium_dynamics__kcasr = (T(2.5) - ((T(2.5) - T(1.0))/(T(1.0) + ((T(1.5)/y[15])*(T(1.5)/y[15])))));
        const T v_calcium_dynamics__k2 = (T(0.045)*v_calcium_dynamics__kcasr);
        const T v_calcium_dynamics__Ca_i_bufc = (T(1.0)/(T(1.0) + ((T(0.2)*T(0.001))/((y[14] + T(0.001))*(y[14] + T(0.001))))));
        const T v_calcium_dynamics__i_leak = (T(0.00036)*(y[15] - y[14]));
        const T v_calcium_dynamics__i_up = (T(0.006375)/(T(1.0) + ((T(0.00025)*T(0.00025))/(y[14]*y[14]))));
        const T v_calcium_dynamics__i_xfer = (T(0.0038)*(y[16] - y[14]));
        const T v_calcium_dynamics__Ca_sr_bufsr = (T(1.0)/(T(1.0) + ((T(10.0)*T(0.3))/((y[15] + T(0.3))*(y[15] + T(0.3))))));
        const T v_calcium_dynamics__k1 = (T(0.15)/v_calcium_dynamics__kcasr);
        const T v_calcium_dynamics__O = ((v_calcium_dynamics__k1*(y[16]*y[16])*y[13])/(T(0.06) + (v_calcium_dynamics__k1*(y[16]*y[16]))));
        const T v_calcium_dynamics__i_rel = (T(0.102)*v_calcium_dynamics__O*(y[15] - y[16]));
        const T v_calcium_dynamics__Ca_ss_bufss = (T(1.0)/(T(1.0) + ((T(0.4)*T(0.00025))/((y[16] + T(0.00025))*(y[16] + T(0.00025))))));
        dy[0] = (((-T(1.0))/T(1.0))*(v_inward_rectifier_potassium_current__i_K1 + v_transient_outward_current__i_to + v_rapid_time_dependent_potassium_current__i_Kr + v_slow_time_dependent_potassium_current__i_Ks + v_L_type_Ca_current__i_CaL + v_sodium_potassium_pump_current__i_NaK + v_fast_sodium_current__i_Na + v_sodium_background_current__i_b_Na + v_sodium_calcium_exchanger_current__i_NaCa + v_calcium_background_current__i_b_Ca + v_potassium_pump_current__i_p_K + v_calcium_pump_current__i_p_Ca + v_membrane__i_Stim));
        dy[1] = ((v_rapid_time_dependent_potassium_current_Xr1_gate__xr1_inf - y[1])/v_rapid_time_dependent_potassium_current_Xr1_gate__tau_xr1);
        dy[2] = ((v_rapid_time_dependent_potassium_current_Xr2_gate__xr2_inf - y[2])/v_rapid_time_dependent_potassium_current_Xr2_gate__tau_xr2);
        dy[3] = ((v_slow_time_dependent_potassium_current_Xs_gate__xs_inf - y[3])/v_slow_time_dependent_potassium_current_Xs_gate__tau_xs);
        dy[4] = ((v_fast_sodium_current_m_gate__m_inf - y[4])/v_fast_sodium_current_m_gate__tau_m);
        dy[5] = ((v_fast_sodium_current_h_gate__h_inf - y[5])/v_fast_sodium_current_h_gate__tau_h);
        dy[6] = ((v_fast_sodium_current_j_gate__j_inf - y[6])/v_fast_sodium_current_j_gate__tau_j);
        dy[7] = ((v_L_type_Ca_current_d_gate__d_inf - y[7])/v_L_type_Ca_current_d_gate__tau_d);
        dy[8] = ((v_L_type_Ca_current_f_gate__f_inf - y[8])/v_L_type_Ca_current_f_gate__tau_f);
        dy[9] = ((v_L_type_Ca_current_f2_gate__f2_inf - y[9])/v_L_type_Ca_current_f2_gate__tau_f2);
        dy[10] = ((v_L_type_Ca_current_fCass_gate__fCass_inf - y[10])/v_L_type_Ca_current_fCass_gate__tau_fCass);
        dy[11] = ((v_transient_outward_current_s_gate__s_inf - y[11])/v_transient_outward_current_s_gate__tau_s);
        dy[12] = ((v_transient_outward_current_r_gate__r_inf - y[12])/v_transient_outward_current_r_gate__tau_r);
        dy[13] = (((-v_calcium_dynamics__k2)*y[16]*y[13]) + (T(0.005)*(T(1.0) - y[13])));
        dy[14] = (v_calcium_dynamics__Ca_i_bufc*(((((v_calcium_dynamics__i_leak - v_calcium_dynamics__i_up)*T(0.001094))/T(0.016404)) + v_calcium_dynamics__i_xfer) - ((((v_calcium_background_current__i_b_Ca + v_calcium_pump_current__i_p_Ca) - (T(2.0)*v_sodium_calcium_exchanger_current__i_NaCa))*T(0.185))/(T(2.0)*T(0.016404)*T(96485.3415)))));
        dy[15] = (v_calcium_dynamics__Ca_sr_bufsr*(v_calcium_dynamics__i_up - (v_calcium_dynamics__i_rel + v_calcium_dynamics__i_leak)));
        dy[16] = (v_calcium_dynamics__Ca_ss_bufss*(((((-v_L_type_Ca_current__i_CaL)*T(0.185))/(T(2.0)*T(5.468e-05)*T(96485.3415))) + ((v_calcium_dynamics__i_rel*T(0.001094))/T(5.468e-05))) - ((v_calcium_dynamics__i_xfer*T(0.016404))/T(5.468e-05))));
        dy[17] = (((-(v_fast_sodium_current__i_Na + v_sodium_background_current__i_b_Na + (T(3.0)*v_sodium_potassium_pump_current__i_NaK) + (T(3.0)*v_sodium_calcium_exchanger_current__i_NaCa)))/(T(0.016404)*T(96485.3415)))*T(0.185));
        dy[18] = (((-((v_inward_rectifier_potassium_current__i_K1 + v_transient_outward_current__i_to + v_rapid_time_dependent_potassium_current__i_Kr + v_slow_time_dependent_potassium_current__i_Ks + v_potassium_pump_current__i_p_K + v_membrane__i_Stim) - (T(2.0)*v_sodium_potassium_pump_current__i_NaK)))/(T(0.016404)*T(96485.3415)))*T(0.185));
    }

    // Rush-Larsen terms: for RL states inf[i] is the fixed point and rate[i]
    // the (negative) affine coefficient h so y' = inf + (y - inf)*exp(h*dt);
    // for the other states rate[i] holds dy/dt.  rate[0] is dV/dt.
    template <typename T>
    CHB_HD static void rl_terms(const T* __restrict__ y, T stim, T cm,
                                       const T* __restrict__ p, T* __restrict__ rate,
                                       T* __restrict__ inf) {
        (void)stim; (void)cm; (void)p; (void)inf;
        const T v_L_type_Ca_current__i_CaL = (((chb::singularity_offset<T>()*T(13.356880329847824)) > fabs((y[0] - T(15.0)))) ? ((((((T(3.98e-05)*p[1])*y[7]*y[8]*y[9]*y[10]*T(4.0)*((T(15.0) - (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*(T(96485.3415)*T(96485.3415)))/(T(8314.472)*T(310.0)))*((T(0.25)*y[16]*m_exp(((T(2.0)*((T(15.0) - (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0))))) - T(2.0)))/(m_exp(((T(2.0)*((T(15.0) - (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0)))) - T(1.0))) + ((y[0] - (T(15.0) - (chb::singularity_offset<T>()*T(13.356880329847824))))*((((((T(3.98e-05)*p[1])*y[7]*y[8]*y[9]*y[10]*T(4.0)*((T(15.0) + (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*(T(96485.3415)*T(96485.3415)))/(T(8314.472)*T(310.0)))*((T(0.25)*y[16]*m_exp(((T(2.0)*((T(15.0) + (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0))))) - T(2.0)))/(m_exp(((T(2.0)*((T(15.0) + (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0)))) - T(1.0))) - (((((T(3.98e-05)*p[1])*y[7]*y[8]*y[9]*y[10]*T(4.0)*((T(15.0) - (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*(T(96485.3415)*T(96485.3415)))/(T(8314.472)*T(310.0)))*((T(0.25)*y[16]*m_exp(((T(2.0)*((T(15.0) - (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0))))) - T(2.0)))/(m_exp(((T(2.0)*((T(15.0) - (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0)))) - T(1.0))))/(T(2.0)*(chb::singularity_offset<T>()*T(13.356880329847824))))) : (((((T(3.98e-05)*p[1])*y[7]*y[8]*y[9]*y[10]*T(4.0)*(y[0] - T(15.0))*(T(96485.3415)*T(96485.3415)))/(T(8314.472)*T(310.0)))*((T(0.25)*y[16]*m_exp(((T(2.0)*(y[0] - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0))))) - T(2.0)))/(m_exp(((T(2.0)*(y[0] - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0)))) - T(1.0))));
        const T v_reversal_potentials__E_Ca = (((T(0.5)*T(8314.472)*T(310.0))/T(96485.3415))*m_log((T(2.0)/y[14])));
        const T v_calcium_background_current__i_b_Ca = (T(0.000592)*(y[0] - v_reversal_potentials__E_Ca));
        const T v_calcium_pump_current__i_p_Ca = ((T(0.1238)*y[14])/(y[14] + T(0.0005)));
        const T v_reversal_potentials__E_Na = (((T(8314.472)*T(310.0))/T(96485.3415))*m_log((T(140.0)/y[17])));
        const T v_fast_sodium_current__i_Na = ((T(14.838)*p[0])*(y[4]*y[4]*y[4])*y[5]*y[6]*(y[0] - v_reversal_potentials__E_Na));
        const T v_reversal_potentials__E_K = (((T(8314.472)*T(310.0))/T(96485.3415))*m_log((T(5.4)/y[18])));
        const T v_inward_rectifier_potassium_current__alpha_K1 = (T(0.1)/(T(1.0) + m_exp((T(0.06)*((y[0] - v_reversal_potentials__E_K) - T(200.0))))));
        const T v_inward_rectifier_potassium_current__beta_K1 = (((T(3.0)*m_exp((T(0.0002)*((y[0] - v_reversal_potentials__E_K) + T(100.0))))) + m_exp((T(0.1)*((y[0] - v_reversal_potentials__E_K) - T(10.0)))))/(T(1.0) + m_exp(((-T(0.5))*(y[0] - v_reversal_potentials__E_K)))));
        const T v_inward_rectifier_potassium_current__xK1_inf = (v_inward_rectifier_potassium_current__alpha_K1/(v_inward_rectifier_potassium_current__alpha_K1 + v_inward_rectifier_potassium_current__beta_K1));
        const T v_inward_rectifier_potassium_current__i_K1 = ((T(5.405)*p[4])*v_inward_rectifier_potassium_current__xK1_inf*(y[0] - v_reversal_potentials__E_K));
        const T v_membrane__i_Stim = (stim/cm);
        const T v_potassium_pump_current__i_p_K = ((T(0.0146)*(y[0] - v_reversal_potentials__E_K))/(T(1.0) + m_exp(((T(25.0) - y[0])/T(5.98)))));
        const T v_rapid_time_dependent_potassium_current__i_Kr = (p[7]*(T(0.153)*p[2])*(T(0.4303314829119352)*m_sqrt(T(5.4)))*y[1]*y[2]*(y[0] - v_reversal_potentials__E_K));
        const T v_reversal_potentials__E_Ks = (((T(8314.472)*T(310.0))/T(96485.3415))*m_log(((T(5.4) + (T(0.03)*T(140.0)))/(y[18] + (T(0.03)*y[17])))));
        const T v_slow_time_dependent_potassium_current__i_Ks = (p[6]*(T(0.392)*p[3])*(y[3]*y[3])*(y[0] - v_reversal_potentials__E_Ks));
        const T v_sodium_background_current__i_b_Na = (T(0.00029)*(y[0] - v_reversal_potentials__E_Na));
        const T v_sodium_calcium_exchanger_current__i_NaCa = ((T(1000.0)*((m_exp(((T(0.35)*y[0]*T(96485.3415))/(T(8314.472)*T(310.0))))*(y[17]*y[17]*y[17])*T(2.0)) - (m_exp((((T(0.35) - T(1.0))*y[0]*T(96485.3415))/(T(8314.472)*T(310.0))))*(T(140.0)*T(140.0)*T(140.0))*y[14]*T(2.5))))/(((T(87.5)*T(87.5)*T(87.5)) + (T(140.0)*T(140.0)*T(140.0)))*(T(1.38) + T(2.0))*(T(1.0) + (T(0.1)*m_exp((((T(0.35) - T(1.0))*y[0]*T(96485.3415))/(T(8314.472)*T(310.0))))))));
        const T v_sodium_potassium_pump_current__i_NaK = (((((T(2.724)*T(5.4))/(T(5.4) + T(1.0)))*y[17])/(y[17] + T(40.0)))/(T(1.0) + (T(0.1245)*m_exp((((-T(0.1))*y[0]*T(96485.3415))/(T(8314.472)*T(310.0))))) + (T(0.0353)*m_exp((((-y[0])*T(96485.3415))/(T(8314.472)*T(310.0)))))));
        const T v_transient_outward_current__i_to = (p[8]*(T(0.294)*p[5])*y[12]*y[11]*(y[0] - v_reversal_potentials__E_K));
        const T v_rapid_time_dependent_potassium_current_Xr1_gate__xr1_inf = (T(1.0)/(T(1.0) + m_exp(((-T(26.0) - y[0])/T(7.0)))));
        const T v_rapid_time_dependent_potassium_current_Xr1_gate__alpha_xr1 = (T(450.0)/(T(1.0) + m_exp(((-T(45.0) - y[0])/T(10.0)))));
        const T v_rapid_time_dependent_potassium_current_Xr1_gate__beta_xr1 = (T(6.0)/(T(1.0) + m_exp(((y[0] + T(30.0))/T(11.5)))));
        const T v_rapid_time_dependent_potassium_current_Xr1_gate__tau_xr1 = (v_rapid_time_dependent_potassium_current_Xr1_gate__alpha_xr1*v_rapid_time_dependent_potassium_current_Xr1_gate__beta_xr1);
        const T v_rapid_time_dependent_potassium_current_Xr2_gate__xr2_inf = (T(1.0)/(T(1.0) + m_exp(((y[0] + T(88.0))/T(24.0)))));
        const T v_rapid_time_dependent_potassium_current_Xr2_gate__alpha_xr2 = (T(3.0)/(T(1.0) + m_exp(((-T(60.0) - y[0])/T(20.0)))));
        const T v_rapid_time_dependent_potassium_current_Xr2_gate__beta_xr2 = (T(1.12)/(T(1.0) + m_exp(((y[0] - T(60.0))/T(20.0)))));
        const T v_rapid_time_dependent_potassium_current_Xr2_gate__tau_xr2 = (v_rapid_time_dependent_potassium_current_Xr2_gate__alpha_xr2*v_rapid_time_dependent_potassium_current_Xr2_gate__beta_xr2);
        const T v_slow_time_dependent_potassium_current_Xs_gate__xs_inf = (T(1.0)/(T(1.0) + m_exp(((-T(5.0) - y[0])/T(14.0)))));
        const T v_slow_time_dependent_potassium_current_Xs_gate__alpha_xs = (T(1400.0)/m_sqrt((T(1.0) + m_exp(((T(5.0) - y[0])/T(6.0))))));
        const T v_slow_time_dependent_potassium_current_Xs_gate__beta_xs = (T(1.0)/(T(1.0) + m_exp(((y[0] - T(35.0))/T(15.0)))));
        const T v_slow_time_dependent_potassium_current_Xs_gate__tau_xs = ((v_slow_time_dependent_potassium_current_Xs_gate__alpha_xs*v_slow_time_dependent_potassium_current_Xs_gate__beta_xs) + T(80.0));
        const T v_fast_sodium_current_m_gate__m_inf = (T(1.0)/((T(1.0) + m_exp(((-T(56.86) - y[0])/T(9.03))))*(T(1.0) + m_exp(((-T(56.86) - y[0])/T(9.03))))));
        const T v_fast_sodium_current_m_gate__alpha_m = (T(1.0)/(T(1.0) + m_exp(((-T(60.0) - y[0])/T(5.0)))));
        const T v_fast_sodium_current_m_gate__beta_m = ((T(0.1)/(T(1.0) + m_exp(((y[0] + T(35.0))/T(5.0))))) + (T(0.1)/(T(1.0) + m_exp(((y[0] - T(50.0))/T(200.0))))));
        const T v_fast_sodium_current_m_gate__tau_m = (v_fast_sodium_current_m_gate__alpha_m*v_fast_sodium_current_m_gate__beta_m);
        const T v_fast_sodium_current_h_gate__h_inf = (T(1.0)/((T(1.0) + m_exp(((y[0] + T(71.55))/T(7.43))))*(T(1.0) + m_exp(((y[0] + T(71.55))/T(7.43))))));
        const T v_fast_sodium_current_h_gate__alpha_h = ((y[0] < (-T(40.0))) ? (T(0.057)*m_exp(((-(y[0] + T(80.0)))/T(6.8)))) : T(0.0));
        const T v_fast_sodium_current_h_gate__beta_h = ((y[0] < (-T(40.0))) ? ((T(2.7)*m_exp((T(0.079)*y[0]))) + (T(310000.0)*m_exp((T(0.3485)*y[0])))) : (T(0.77)/(T(0.13)*(T(1.0) + m_exp(((y[0] + T(10.66))/(-T(11.1))))))));
        const T v_fast_sodium_current_h_gate__tau_h = (T(1.0)/(v_fast_sodium_current_h_gate__alpha_h + v_fast_sodium_current_h_gate__beta_h));
        const T v_fast_sodium_current_j_gate__j_inf = (T(1.0)/((T(1.0) + m_exp(((y[0] + T(71.55))/T(7.43))))*(T(1.0) + m_exp(((y[0] + T(71.55))/T(7.43))))));
        const T v_fast_sodium_current_j_gate__alpha_j = ((y[0] < (-T(40.0))) ? (((((-T(25428.0))*m_exp((T(0.2444)*y[0]))) - (T(6.948e-06)*m_exp(((-T(0.04391))*y[0]))))*(y[0] + T(37.78)))/(T(1.0) + m_exp((T(0.311)*(y[0] + T(79.23)))))) : T(0.0));
        const T v_fast_sodium_current_j_gate__beta_j = ((y[0] < (-T(40.0))) ? ((T(0.02424)*m_exp(((-T(0.01052))*y[0])))/(T(1.0) + m_exp(((-T(0.1378))*(y[0] + T(40.14)))))) : ((T(0.6)*m_exp((T(0.057)*y[0])))/(T(1.0) + m_exp(((-T(0.1))*(y[0] + T(32.0)))))));
        const T v_fast_sodium_current_j_gate__tau_j = (T(1.0)/(v_fast_sodium_current_j_gate__alpha_j + v_fast_sodium_current_j_gate__beta_j));
        const T v_L_type_Ca_current_d_gate__d_inf = (T(1.0)/(T(1.0) + m_exp(((-T(8.0) - y[0])/T(7.5)))));
        const T v_L_type_Ca_current_d_gate__alpha_d = ((T(1.4)/(T(1.0) + m_exp(((-T(35.0) - y[0])/T(13.0))))) + T(0.25));
        const T v_L_type_Ca_current_d_gate__beta_d = (T(1.4)/(T(1.0) + m_exp(((y[0] + T(5.0))/T(5.0)))));
        const T v_L_type_Ca_current_d_gate__gamma_d = (T(1.0)/(T(1.0) + m_exp(((T(50.0) - y[0])/T(20.0)))));
        const T v_L_type_Ca_current_d_gate__tau_d = ((v_L_type_Ca_current_d_gate__alpha_d*v_L_type_Ca_current_d_gate__beta_d) + v_L_type_Ca_current_d_gate__gamma_d);
        const T v_L_type_Ca_current_f_gate__f_inf = (T(1.0)/(T(1.0) + m_exp(((y[0] + T(20.0))/T(7.0)))));
        const T v_L_type_Ca_current_f_gate__tau_f = ((T(1102.5)*m_exp(((-((y[0] + T(27.0))*(y[0] + T(27.0))))/T(225.0)))) + (T(200.0)/(T(1.0) + m_exp(((T(13.0) - y[0])/T(10.0))))) + (T(180.0)/(T(1.0) + m_exp(((y[0] + T(30.0))/T(10.0))))) + T(20.0));
        const T v_L_type_Ca_current_f2_gate__f2_inf = ((T(0.67)/(T(1.0) + m_exp(((y[0] + T(35.0))/T(7.0))))) + T(0.33));
        const T v_L_type_Ca_current_f2_gate__tau_f2 = ((T(562.0)*m_exp(((-((y[0] + T(27.0))*(y[0] + T(27.0))))/T(240.0)))) + (T(31.0)/(T(1.0) + m_exp(((T(25.0) - y[0])/T(10.0))))) + (T(80.0)/(T(1.0) + m_exp(((y[0] + T(30.0))/T(10.0))))));
        const T v_L_type_Ca_current_fCass_gate__fCass_inf = ((T(0.6)/(T(1.0) + ((y[16]/T(0.05))*(y[16]/T(0.05))))) + T(0.4));
        const T v_L_type_Ca_current_fCass_gate__tau_fCass = ((T(80.0)/(T(1.0) + ((y[16]/T(0.05))*(y[16]/T(0.05))))) + T(2.0));
        const T v_transient_outward_current_s_gate__s_inf = (T(1.0)/(T(1.0) + m_exp(((y[0] + T(20.0))/T(5.0)))));
        const T v_transient_outward_current_s_gate__tau_s = ((T(85.0)*m_exp(((-((y[0] + T(45.0))*(y[0] + T(45.0))))/T(320.0)))) + (T(5.0)/(T(1.0) + m_exp(((y[0] - T(20.0))/T(5.0))))) + T(3.0));
        const T v_transient_outward_current_r_gate__r_inf = (T(1.0)/(T(1.0) + m_exp(((T(20.0) - y[0])/T(6.0)))));
        const T v_transient_outward_current_r_gate__tau_r = ((T(9.5)*m_exp(((-((y[0] + T(40.0))*(y[0] + T(40.0))))/T(1800.0)))) + T(0.8));
        const T v_calcium_dynamics__kcasr = (T(2.5) - ((T(2.5) - T(1.0))/(T(1.0) + ((T(1.5)/y[15])*(T(1.5)/y[15])))));
        const T v_calcium_dynamics__k2 = (T(0.045)*v_calcium_dynamics__kcasr);
        const T v_calcium_dynamics__Ca_i_bufc = (T(1.0)/(T(1.0) + ((T(0.2)*T(0.001))/((y[14] + T(0.001))*(y[14] + T(0.001))))));
        const T v_calcium_dynamics__i_leak = (T(0.00036)*(y[15] - y[14]));
        const T v_calcium_dynamics__i_up = (T(0.006375)/(T(1.0) + ((T(0.00025)*T(0.00025))/(y[14]*y[14]))));
        const T v_calcium_dynamics__i_xfer = (T(0.0038)*(y[16] - y[14]));
        const T v_calcium_dynamics__Ca_sr_bufsr = (T(1.0)/(T(1.0) + ((T(10.0)*T(0.3))/((y[15] + T(0.3))*(y[15] + T(0.3))))));
        const T v_calcium_dynamics__k1 = (T(0.15)/v_calcium_dynamics__kcasr);
        const T v_calcium_dynamics__O = ((v_calcium_dynamics__k1*(y[16]*y[16])*y[13])/(T(0.06) + (v_calcium_dynamics__k1*(y[16]*y[16]))));
        const T v_calcium_dynamics__i_rel = (T(0.102)*v_calcium_dynamics__O*(y[15] - y[16]));
        const T v_calcium_dynamics__Ca_ss_bufss = (T(1.0)/(T(1.0) + ((T(0.4)*T(0.00025))/((y[16] + T(0.00025))*(y[16] + T(0.00025))))));
        rate[0] = (((-T(1.0))/T(1.0))*(v_inward_rectifier_potassium_current__i_K1 + v_transient_outward_current__i_to + v_rapid_time_dependent_potassium_current__i_Kr + v_slow_time_dependent_potassium_current__i_Ks + v_L_type_Ca_current__i_CaL + v_sodium_potassium_pump_current__i_NaK + v_fast_sodium_current__i_Na + v_sodium_background_current__i_b_Na + v_sodium_calcium_exchanger_current__i_NaCa + v_calcium_background_current__i_b_Ca + v_potassium_pump_current__i_p_K + v_calcium_pump_current__i_p_Ca + v_membrane__i_Stim));
        inf[1] = v_rapid_time_dependent_potassium_current_Xr1_gate__xr1_inf;
        rate[1] = (-(T(1.0)/v_rapid_time_dependent_potassium_current_Xr1_gate__tau_xr1));
        inf[2] = v_rapid_time_dependent_potassium_current_Xr2_gate__xr2_inf;
        rate[2] = (-(T(1.0)/v_rapid_time_dependent_potassium_current_Xr2_gate__tau_xr2));
        inf[3] = v_slow_time_dependent_potassium_current_Xs_gate__xs_inf;
        rate[3] = (-(T(1.0)/v_slow_time_dependent_potassium_current_Xs_gate__tau_xs));
        inf[4] = v_fast_sodium_current_m_gate__m_inf;
        rate[4] = (-(T(1.0)/v_fast_sodium_current_m_gate__tau_m));
        inf[5] = v_fast_sodium_current_h_gate__h_inf;
        rate[5] = (-(T(1.0)/v_fast_sodium_current_h_gate__tau_h));
        inf[6] = v_fast_sodium_current_j_gate__j_inf;
        rate[6] = (-(T(1.0)/v_fast_sodium_current_j_gate__tau_j));
        inf[7] = v_L_type_Ca_current_d_gate__d_inf;
        rate[7] = (-(T(1.0)/v_L_type_Ca_current_d_gate__tau_d));
        inf[8] = v_L_type_Ca_current_f_gate__f_inf;
        rate[8] = (-(T(1.0)/v_L_type_Ca_current_f_gate__tau_f));
        inf[9] = v_L_type_Ca_current_f2_gate__f2_inf;
        rate[9] = (-(T(1.0)/v_L_type_Ca_current_f2_gate__tau_f2));
        inf[10] = v_L_type_Ca_current_fCass_gate__fCass_inf;
        rate[10] = (-(T(1.0)/v_L_type_Ca_current_fCass_gate__tau_fCass));
        inf[11] = v_transient_outward_current_s_gate__s_inf;
        rate[11] = (-(T(1.0)/v_transient_outward_current_s_gate__tau_s));
        inf[12] = v_transient_outward_current_r_gate__r_inf;
        rate[12] = (-(T(1.0)/v_transient_outward_current_r_gate__tau_r));
        inf[13] = (-(T(0.005)/(-T(0.005) - (y[16]*v_calcium_dynamics__k2))));
        rate[13] = (-T(0.005) - (y[16]*v_calcium_dynamics__k2));
        rate[14] = (v_calcium_dynamics__Ca_i_bufc*(((((v_calcium_dynamics__i_leak - v_calcium_dynamics__i_up)*T(0.001094))/T(0.016404)) + v_calcium_dynamics__i_xfer) - ((((v_calcium_background_current__i_b_Ca + v_calcium_pump_current__i_p_Ca) - (T(2.0)*v_sodium_calcium_exchanger_current__i_NaCa))*T(0.185))/(T(2.0)*T(0.016404)*T(96485.3415)))));
        rate[15] = (v_calcium_dynamics__Ca_sr_bufsr*(v_calcium_dynamics__i_up - (v_calcium_dynamics__i_rel + v_calcium_dynamics__i_leak)));
        rate[16] = (v_calcium_dynamics__Ca_ss_bufss*(((((-v_L_type_Ca_current__i_CaL)*T(0.185))/(T(2.0)*T(5.468e-05)*T(96485.3415))) + ((v_calcium_dynamics__i_rel*T(0.001094))/T(5.468e-05))) - ((v_calcium_dynamics__i_xfer*T(0.016404))/T(5.468e-05))));
        rate[17] = (((-(v_fast_sodium_current__i_Na + v_sodium_background_current__i_b_Na + (T(3.0)*v_sodium_potassium_pump_current__i_NaK) + (T(3.0)*v_sodium_calcium_exchanger_current__i_NaCa)))/(T(0.016404)*T(96485.3415)))*T(0.185));
        rate[18] = (((-((v_inward_rectifier_potassium_current__i_K1 + v_transient_outward_current__i_to + v_rapid_time_dependent_potassium_current__i_Kr + v_slow_time_dependent_potassium_current__i_Ks + v_potassium_pump_current__i_p_K + v_membrane__i_Stim) - (T(2.0)*v_sodium_potassium_pump_current__i_NaK)))/(T(0.016404)*T(96485.3415)))*T(0.185));
    }

    // Total ionic current in uA/cm^2 (GetIIonic): the dV/dt currents without
    // the stimulus, times the capacitance cm.
    template <typename T>
    CHB_HD static T iionic(const T* __restrict__ y, T cm, const T* __restrict__ p) {
        (void)cm; (void)p;
        const T stim = T(0.0); (void)stim;
        const T v_L_type_Ca_current__i_CaL = (((chb::singularity_offset<T>()*T(13.356880329847824)) > fabs((y[0] - T(15.0)))) ? ((((((T(3.98e-05)*p[1])*y[7]*y[8]*y[9]*y[10]*T(4.0)*((T(15.0) - (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*(T(96485.3415)*T(96485.3415)))/(T(8314.472)*T(310.0)))*((T(0.25)*y[16]*m_exp(((T(2.0)*((T(15.0) - (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0))))) - T(2.0)))/(m_exp(((T(2.0)*((T(15.0) - (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0)))) - T(1.0))) + ((y[0] - (T(15.0) - (chb::singularity_offset<T>()*T(13.356880329847824))))*((((((T(3.98e-05)*p[1])*y[7]*y[8]*y[9]*y[10]*T(4.0)*((T(15.0) + (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*(T(96485.3415)*T(96485.3415)))/(T(8314.472)*T(310.0)))*((T(0.25)*y[16]*m_exp(((T(2.0)*((T(15.0) + (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0))))) - T(2.0)))/(m_exp(((T(2.0)*((T(15.0) + (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0)))) - T(1.0))) - (((((T(3.98e-05)*p[1])*y[7]*y[8]*y[9]*y[10]*T(4.0)*((T(15.0) - (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*(T(96485.3415)*T(96485.3415)))/(T(8314.472)*T(310.0)))*((T(0.25)*y[16]*m_exp(((T(2.0)*((T(15.0) - (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0))))) - T(2.0)))/(m_exp(((T(2.0)*((T(15.0) - (chb::singularity_offset<T>()*T(13.356880329847824))) - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0)))) - T(1.0))))/(T(2.0)*(chb::singularity_offset<T>()*T(13.356880329847824))))) : (((((T(3.98e-05)*p[1])*y[7]*y[8]*y[9]*y[10]*T(4.0)*(y[0] - T(15.0))*(T(96485.3415)*T(96485.3415)))/(T(8314.472)*T(310.0)))*((T(0.25)*y[16]*m_exp(((T(2.0)*(y[0] - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0))))) - T(2.0)))/(m_exp(((T(2.0)*(y[0] - T(15.0))*T(96485.3415))/(T(8314.472)*T(310.0)))) - T(1.0))));
        const T v_reversal_potentials__E_Ca = (((T(0.5)*T(8314.472)*T(310.0))/T(96485.3415))*m_log((T(2.0)/y[14])));
        const T v_calcium_background_current__i_b_Ca = (T(0.000592)*(y[0] - v_reversal_potentials__E_Ca));
        const T v_calcium_pump_current__i_p_Ca = ((T(0.1238)*y[14])/(y[14] + T(0.0005)));
        const T v_reversal_potentials__E_Na = (((T(8314.472)*T(310.0))/T(96485.3415))*m_log((T(140.0)/y[17])));
        const T v_fast_sodium_current__i_Na = ((T(14.838)*p[0])*(y[4]*y[4]*y[4])*y[5]*y[6]*(y[0] - v_reversal_potentials__E_Na));
        const T v_reversal_potentials__E_K = (((T(8314.472)*T(310.0))/T(96485.3415))*m_log((T(5.4)/y[18])));
        const T v_inward_rectifier_potassium_current__alpha_K1 = (T(0.1)/(T(1.0) + m_exp((T(0.06)*((y[0] - v_reversal_potentials__E_K) - T(200.0))))));
        const T v_inward_rectifier_potassium_current__beta_K1 = (((T(3.0)*m_exp((T(0.0002)*((y[0] - v_reversal_potentials__E_K) + T(100.0))))) + m_exp((T(0.1)*((y[0] - v_reversal_potentials__E_K) - T(10.0)))))/(T(1.0) + m_exp(((-T(0.5))*(y[0] - v_reversal_potentials__E_K)))));
        const T v_inward_rectifier_potassium_current__xK1_inf = (v_inward_rectifier_potassium_current__alpha_K1/(v_inward_rectifier_potassium_current__alpha_K1 + v_inward_rectifier_potassium_current__beta_K1));
        const T v_inward_rectifier_potassium_current__i_K1 = ((T(5.405)*p[4])*v_inward_rectifier_potassium_current__xK1_inf*(y[0] - v_reversal_potentials__E_K));
        const T v_potassium_pump_current__i_p_K = ((T(0.0146)*(y[0] - v_reversal_potentials__E_K))/(T(1.0) + m_exp(((T(25.0) - y[0])/T(5.98)))));
        const T v_rapid_time_dependent_potassium_current__i_Kr = (p[7]*(T(0.153)*p[2])*(T(0.4303314829119352)*m_sqrt(T(5.4)))*y[1]*y[2]*(y[0] - v_reversal_potentials__E_K));
        const T v_reversal_potentials__E_Ks = (((T(8314.472)*T(310.0))/T(96485.3415))*m_log(((T(5.4) + (T(0.03)*T(140.0)))/(y[18] + (T(0.03)*y[17])))));
        const T v_slow_time_dependent_potassium_current__i_Ks = (p[6]*(T(0.392)*p[3])*(y[3]*y[3])*(y[0] - v_reversal_potentials__E_Ks));
        const T v_sodium_background_current__i_b_Na = (T(0.00029)*(y[0] - v_reversal_potentials__E_Na));
        const T v_sodium_calcium_exchanger_current__i_NaCa = ((T(1000.0)*((m_exp(((T(0.35)*y[0]*T(96485.3415))/(T(8314.472)*T(310.0))))*(y[17]*y[17]*y[17])*T(2.0)) - (m_exp((((T(0.35) - T(1.0))*y[0]*T(96485.3415))/(T(8314.472)*T(310.0))))*(T(140.0)*T(140.0)*T(140.0))*y[14]*T(2.5))))/(((T(87.5)*T(87.5)*T(87.5)) + (T(140.0)*T(140.0)*T(140.0)))*(T(1.38) + T(2.0))*(T(1.0) + (T(0.1)*m_exp((((T(0.35) - T(1.0))*y[0]*T(96485.3415))/(T(8314.472)*T(310.0))))))));
        const T v_sodium_potassium_pump_current__i_NaK = (((((T(2.724)*T(5.4))/(T(5.4) + T(1.0)))*y[17])/(y[17] + T(40.0)))/(T(1.0) + (T(0.1245)*m_exp((((-T(0.1))*y[0]*T(96485.3415))/(T(8314.472)*T(310.0))))) + (T(0.0353)*m_exp((((-y[0])*T(96485.3415))/(T(8314.472)*T(310.0)))))));
        const T v_transient_outward_current__i_to = (p[8]*(T(0.294)*p[5])*y[12]*y[11]*(y[0] - v_reversal_potentials__E_K));
        return (v_L_type_Ca_current__i_CaL + v_calcium_background_current__i_b_Ca + v_calcium_pump_current__i_p_Ca + v_fast_sodium_current__i_Na + v_inward_rectifier_potassium_current__i_K1 + v_potassium_pump_current__i_p_K + v_rapid_time_dependent_potassium_current__i_Kr + v_slow_time_dependent_potassium_current__i_Ks + v_sodium_background_current__i_b_Na + v_sodium_calcium_exchanger_current__i_NaCa + v_sodium_potassium_pump_current__i_NaK + v_transient_outward_current__i_to)*cm;
    }
};

}  // namespace chb

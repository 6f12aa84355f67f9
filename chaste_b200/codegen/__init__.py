"""CellML route: reader (cellml.py) and C++/CUDA emitter (emit.py).

PARAM_NAMES lists, per model id, the per-cell scale factors the generated
headers read from p[], and STATE_NAMES the state variables in the headers'
order (kept here so the runtime does not import sympy).
"""
PARAM_NAMES = {
    0: ["g_Na", "g_si", "g_K", "g_K1", "g_Kp", "g_b"],
    1: ["g_Na", "g_CaL", "g_Kr", "g_Ks", "g_K1", "g_to",
        "ScaleFactorGks", "ScaleFactorGkr", "ScaleFactorIto"],
}
STATE_NAMES = {
    0: ["V", "m", "h", "j", "d", "f", "X", "Cai"],
    1: ["V", "Xr1", "Xr2", "Xs", "m", "h", "j", "d", "f", "f2", "fCass", "s", "r", "R_prime", "Ca_i", "Ca_SR",
        "Ca_ss", "Na_i", "K_i"],
}

"""CellML route: reader (cellml.py) and C++/CUDA emitter (emit.py).

PARAM_NAMES lists, per model id, the per-cell scale factors the generated
headers read from p[] (kept here so the runtime does not import sympy).
"""
PARAM_NAMES = {
    0: ["g_Na", "g_si", "g_K", "g_K1", "g_Kp", "g_b"],
    1: ["g_Na", "g_CaL", "g_Kr", "g_Ks", "g_K1", "g_to",
        "ScaleFactorGks", "ScaleFactorGkr", "ScaleFactorIto"],
}

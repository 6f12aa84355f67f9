"""CellML -> C++/CUDA cell-model emitter (the project's CUDA backend of the CellML route).

Chaste turns each ``heart/src/odes/cellml/*.cellml`` into C++ at build time
with chaste_codegen (build rule ``cmake/Modules/ChasteMacros.cmake:65-99``).
This module does the same job for the GPU tissue: it reads the CellML with
:mod:`chaste_b200.codegen.cellml` and writes one header per model holding a
traits struct whose static member templates are ``__host__ __device__`` and
typed on the arithmetic type ``T`` (``double`` for the FP64 path, ``float``
for the mixed path).  The same header is compiled by g++ for the CPU oracle
and by nvcc for the kernels.

Conventions applied (those a Chaste cell class obeys):

* the membrane voltage is state 0 (``AbstractCardiacCell`` voltage index; the
  tissue test ``heart/test/monodomain/TestMonodomainTissue.hpp:199-213`` reads
  ``rGetStateVariables()[0]`` as V); other states keep document order;
* the CellML stimulus is replaced by the Chaste stimulus, given in uA/cm^2
  (``AbstractCardiacCellInterface::GetIntracellularAreaStimulus``,
  ``heart/src/odes/AbstractCardiacCellInterface.cpp:106-119``) and converted to
  the model's current units (divided by the Chaste capacitance ``cm`` when the
  model's currents are per unit capacitance);
* ``iionic`` is the sum of the non-stimulus currents of the dV/dt equation,
  converted to uA/cm^2 (the quantity ``GetIIonic`` caches,
  ``heart/src/tissue/AbstractCardiacTissue.cpp:730-734``);
* Rush-Larsen: every non-voltage state whose ODE is affine in itself,
  dy/dt = g + h*y with g, h independent of y, is advanced exactly over one step
  with g, h frozen: y' = y_inf + (y - y_inf)*exp(h*dt), y_inf = -g/h; the
  others take a forward-Euler step (``AbstractRushLarsenCardiacCell.cpp:106-153``).
  The emitter prints (inf, tau) directly when the ODE is written (inf-y)/tau and
  (alpha, beta) when written alpha*(1-y)-beta*y.
* conductances listed in ``PARAMS`` become multiplicative scale factors p[i]
  (default 1), read from a per-cell parameter vector.

Sub-expressions of constants only are folded to double literals at generation
time so both precisions see the correctly rounded value.
"""
from __future__ import annotations

import argparse
import math
import os
import sys

import sympy as sp

from . import cellml

# Conductance variables exposed as multiplicative scale factors, per model.
# Names are CellML variable names; the scale multiplies every use.
PARAMS = {
    "luo_rudy_1991": [
        ("g_Na", "fast_sodium_current", "g_Na"),
        ("g_si", "slow_inward_current", "P_si"),
        ("g_K", "time_dependent_potassium_current", "g_K"),
        ("g_K1", "time_independent_potassium_current", "g_K1"),
        ("g_Kp", "plateau_potassium_current", "g_Kp"),
        ("g_b", "background_current", "g_b"),
    ],
    "tentusscher_model_2006_epi": [
        ("g_Na", "fast_sodium_current", "g_Na"),
        ("g_CaL", "L_type_Ca_current", "g_CaL"),
        ("g_Kr", "rapid_time_dependent_potassium_current", "g_Kr"),
        ("g_Ks", "slow_time_dependent_potassium_current", "g_Ks"),
        ("g_K1", "inward_rectifier_potassium_current", "g_K1"),
        ("g_to", "transient_outward_current", "g_to"),
        # Chaste's own modifiable parameters (TenTusscher2006Epi.cellml:3697-3705);
        # these are CellML variables with default 1, replaced by p[i].
        ("ScaleFactorGks", "slow_time_dependent_potassium_current", "ScaleFactorGks"),
        ("ScaleFactorGkr", "rapid_time_dependent_potassium_current", "ScaleFactorGkr"),
        ("ScaleFactorIto", "transient_outward_current", "ScaleFactorIto"),
    ],
}

SHORT = {"luo_rudy_1991": "LuoRudy1991", "tentusscher_model_2006_epi": "TenTusscher2006Epi"}

_CURRENT_AREA = None  # dims of A/m^2
_CURRENT_PER_CAP = None  # dims of V/s


def _dims(**kw):
    return tuple(kw.get(k, 0) for k in cellml._DIMS)


_CURRENT_AREA = _dims(A=1, m=-2)
_CURRENT_PER_CAP = _dims(kg=1, m=2, s=-4, A=-1)  # V/s


def _lit(x: float) -> str:
    if not math.isfinite(x):
        raise ValueError("non-finite constant")
    r = repr(float(x))
    if "e" not in r and "." not in r and "inf" not in r:
        r += ".0"
    return r


class Printer:
    """Prints sympy expressions as C++ with literals cast to ``T``."""

    def __init__(self, names):
        self.names = names

    def num(self, x):
        return f"T({_lit(float(x))})"

    def __call__(self, e) -> str:
        return self.p(e)

    def p(self, e):
        if e.is_Symbol:
            return self.names[e]
        if e.is_Number:
            v = float(e)
            if v < 0:
                return f"(-{self.num(-v)})"
            return self.num(v)
        if isinstance(e, sp.Add):
            out = ""
            for i, t in enumerate(e.args):
                neg, body = self._split_neg(t)
                if i == 0:
                    out = ("-" if neg else "") + self._paren_add(body) if neg else self.p(body)
                else:
                    out += (" - " if neg else " + ") + (self._paren_add(body) if neg else self.p(body))
            return f"({out})"
        if isinstance(e, sp.Mul):
            num, den = [], []
            for f in e.args:
                if isinstance(f, sp.Pow) and f.exp.is_Number and float(f.exp) < 0:
                    ex = -f.exp
                    den.append(f.base if ex == 1 else sp.Pow(f.base, ex, evaluate=False))
                else:
                    num.append(f)
            if len(num) >= 1 and num[0].is_Number and float(num[0]) == -1:
                rest = num[1:]
                ns = "T(1.0)" if not rest else "*".join(self._fac(f) for f in rest)
                s = f"-{ns}" if not den else f"-{self._div(ns, den)}"
                return f"({s})"
            ns = "T(1.0)" if not num else "*".join(self._fac(f) for f in num)
            if den:
                return f"({self._div(ns, den)})"
            return f"({ns})" if len(num) > 1 else ns
        if isinstance(e, sp.Pow):
            b, x = e.base, e.exp
            if x.is_Number:
                xv = float(x)
                if xv == 2:
                    bs = self.p(b)
                    return f"({bs}*{bs})"
                if xv == 3:
                    bs = self.p(b)
                    return f"({bs}*{bs}*{bs})"
                if xv == 0.5:
                    return f"m_sqrt({self.p(b)})"
                if xv == -1:
                    return f"({self._div('T(1.0)', [b])})"
                if xv == int(xv) and 4 <= xv <= 8:
                    bs = self.p(b)
                    return "(" + "*".join([bs] * int(xv)) + ")"
            return f"m_pow({self.p(b)}, {self.p(x)})"
        if isinstance(e, sp.exp):
            return f"m_exp({self.p(e.args[0])})"
        if isinstance(e, sp.log):
            if len(e.args) == 2:
                return f"m_div(m_log({self.p(e.args[0])}), m_log({self.p(e.args[1])}))"
            return f"m_log({self.p(e.args[0])})"
        if isinstance(e, sp.floor):
            return f"floor({self.p(e.args[0])})"
        if isinstance(e, sp.Abs):
            return f"fabs({self.p(e.args[0])})"
        if isinstance(e, sp.Piecewise):
            out = None
            for expr, cond in reversed(e.args):
                if cond is sp.true or cond == True:  # noqa: E712
                    out = self.p(expr)
                else:
                    out = f"(({self.cond(cond)}) ? {self.p(expr)} : {out if out is not None else 'T(NAN)'})"
            return out
        raise ValueError(f"cannot print {type(e)}: {e}")

    def _div(self, ns, den):
        """Quotient: m_divk for a numeric denominator (exact in double, multiply by the
        reciprocal in float), m_div otherwise (a / b, or the fast quotient in float)."""
        if len(den) == 1 and den[0].is_Number:
            c = float(den[0])
            return f"m_divk({ns}, {self.p(den[0])}, T({_lit(1.0 / c)}))"
        return f"m_div({ns}, {self._den(den)})"

    def _split_neg(self, t):
        if isinstance(t, sp.Mul) and t.args[0].is_Number and float(t.args[0]) < 0:
            c = -t.args[0]
            rest = t.args[1:]
            if c == 1:
                body = rest[0] if len(rest) == 1 else sp.Mul(*rest, evaluate=False)
            else:
                body = sp.Mul(c, *rest, evaluate=False)
            return True, body
        if t.is_Number and float(t) < 0:
            return True, -t
        return False, t

    def _paren_add(self, body):
        s = self.p(body)
        return s

    def _fac(self, f):
        s = self.p(f)
        return s

    def _den(self, den):
        if len(den) == 1:
            return self.p(den[0])
        return "(" + "*".join(self.p(d) for d in den) + ")"

    def cond(self, c):
        if isinstance(c, sp.And):
            return " && ".join(f"({self.cond(a)})" for a in c.args)
        if isinstance(c, sp.Or):
            return " || ".join(f"({self.cond(a)})" for a in c.args)
        ops = {sp.StrictLessThan: "<", sp.LessThan: "<=", sp.StrictGreaterThan: ">",
               sp.GreaterThan: ">=", sp.Equality: "==", sp.Unequality: "!="}
        for k, op in ops.items():
            if isinstance(c, k):
                return f"{self.p(c.lhs)} {op} {self.p(c.rhs)}"
        raise ValueError(f"cannot print condition {c}")


def _free(e):
    return {s for s in e.free_symbols}


class ModelEmitter:
    def __init__(self, model: cellml.CellModel, struct_name: str):
        self.m = model
        self.struct = struct_name
        m = model
        self.V = m.annotations["membrane_voltage"]
        self.stim_sym = m.annotations["membrane_stimulus_current"]
        self.states = [self.V] + [s for s in m.states if s != self.V]
        self.n = len(self.states)
        self.stim_arg = sp.Symbol("__stim", real=True)
        self.cm_arg = sp.Symbol("__cm", real=True)
        self.pnames = PARAMS[m.name]
        self.psyms = [sp.Symbol(f"__p{i}", real=True) for i in range(len(self.pnames))]
        self._prepare()

    # ------------------------------------------------------------------
    def _key_of(self, sym):
        for k, s in self.m.symbols.items():
            if s == sym:
                return k
        raise KeyError(sym)

    def _prepare(self):
        m = self.m
        defs = dict(m.algebraic)
        # stimulus -> Chaste stimulus argument in model units
        sk = self._key_of(self.stim_sym)
        dims = m.units_dims[sk]
        f = m.units_factor[sk]
        if dims == _CURRENT_AREA:
            conv = 1e-2 / f                         # uA/cm^2 = 1e-2 A/m^2
            stim_expr = sp.Mul(sp.Float(conv, 17), self.stim_arg, evaluate=False) \
                if abs(conv - 1) > 1e-15 else self.stim_arg
            self.current_per_cap = False
        elif dims == _CURRENT_PER_CAP:
            conv = 1.0 / f                          # (uA/cm^2)/(uF/cm^2) = V/s
            stim_expr = sp.Mul(self.stim_arg, sp.Pow(self.cm_arg, -1, evaluate=False),
                               evaluate=False)
            if abs(conv - 1) > 1e-15:
                stim_expr = sp.Mul(sp.Float(conv, 17), stim_expr, evaluate=False)
            self.current_per_cap = True
        else:
            raise ValueError("stimulus current has unsupported units")
        defs[self.stim_sym] = stim_expr
        # scale-factor parameters
        self.scaled = {}
        replace = {}
        for i, (pname, comp, var) in enumerate(self.pnames):
            sym = m.symbol_for(comp, var)
            if sym in m.constants:
                # a CellML constant: the parameter replaces it when its default
                # is 1 (ScaleFactor*), else scales it.
                if m.constants[sym] == 1.0 and pname.startswith("ScaleFactor"):
                    replace[sym] = self.psyms[i]
                else:
                    replace[sym] = sp.Mul(sp.Float(m.constants[sym], 17), self.psyms[i],
                                          evaluate=False)
            else:
                new = sp.Symbol(str(sym) + "__scaled", real=True)
                defs[new] = sp.Mul(sym, self.psyms[i], evaluate=False)
                replace[sym] = new
                self.scaled[new] = sym
        # apply the parameter replacement in every definition except the
        # scaled variable's own product
        newdefs = {}
        with sp.evaluate(False):
            for k, e in defs.items():
                if k in self.scaled:
                    newdefs[k] = e
                else:
                    newdefs[k] = e.xreplace(replace)
            odes = {s: e.xreplace(replace) for s, e in m.odes.items()}
        self.defs = newdefs
        self.odes = odes
        self.consts = {s: v for s, v in m.constants.items() if s not in replace}
        # fold constant-only algebraic variables
        self.folded = dict(self.consts)
        dyn = set(self.states) | {self.stim_arg, self.cm_arg, m.time} | set(self.psyms)
        changed = True
        while changed:
            changed = False
            for k, e in self.defs.items():
                if k in self.folded:
                    continue
                fs = _free(e)
                if fs & dyn:
                    continue
                if all(s in self.folded for s in fs):
                    val = float(e.xreplace({s: sp.Float(v, 30) for s, v in self.folded.items()}).evalf(30))
                    self.folded[k] = val
                    changed = True
        # dependency graph for non-folded algebraic variables
        self.live = {k: e for k, e in self.defs.items() if k not in self.folded}
        # ionic currents: symbols of the dV/dt equation with current units
        dv = self.odes[self.V]
        cur = []
        for s in sorted(_free(dv), key=str):
            if s == self.stim_sym:
                continue
            try:
                k = self._key_of(s)
            except KeyError:
                # a scaled symbol
                k = self._key_of(self.scaled[s]) if s in self.scaled else None
            if k is None:
                continue
            if m.units_dims[k] in (_CURRENT_AREA, _CURRENT_PER_CAP):
                cur.append(s)
        self.currents = cur
        # time must not remain
        for k, e in self.live.items():
            if m.time in _free(e) and k != self.stim_sym:
                raise ValueError(f"{k} depends on time beyond the stimulus")
        self._fix_singularities()
        self._rl_analysis()

    # --------------------------------------------------------------------
    def _inline(self, e, target, depth=0):
        """Inline algebraic definitions that depend (transitively) on target."""
        memo = {}

        def dep(s):
            if s in memo:
                return memo[s]
            if s == target:
                memo[s] = True
                return True
            if s in self.live:
                memo[s] = False
                r = any(dep(x) for x in _free(self.live[s]))
                memo[s] = r
                return r
            memo[s] = False
            return False

        def sub(x):
            reps = {}
            for s in _free(x):
                if s != target and s in self.live and dep(s):
                    reps[s] = sub(self.live[s])
            return x.xreplace(reps) if reps else x

        return sub(e)

    # ------------------------------------------------------------------
    # Removable singularities (GHK-type terms such as (V-V0)/(exp(c(V-V0))-1)).
    # chaste_codegen replaces such an expression f(V), within a small window of
    # the exponent argument U = c(V-V0) around 0, by the straight line through
    # f(V0-eps) and f(V0+eps), eps = U_offset/|c|.  The same is done here; the
    # offset is a per-precision constant (chb::singularity_offset<T>()).
    def _affine_root(self, e):
        """Root V0 and slope c if e (constants folded) is c*V + d, else None."""
        V = self.V
        e = self._fold_expr(e)
        try:
            ev = sp.sympify(str(e), locals={str(x): x for x in _free(e)})
        except Exception:  # noqa: BLE001
            return None
        if _free(ev) != {V}:
            return None
        c = sp.diff(ev, V)
        if not c.is_Number or c == 0:
            return None
        d = ev.xreplace({V: sp.Integer(0)})
        if not d.is_Number:
            return None
        return float(-d / c), float(c)

    def _zero_roots(self, b):
        """Roots in V of b when b is affine in V or of the form +-(exp(E) - 1), E affine."""
        out = []
        r = self._affine_root(b)
        if r is not None:
            out.append(r)
        if isinstance(b, sp.Add) and len(b.args) == 2:
            ex = [a for a in b.args if a.has(sp.exp)]
            cs = [a for a in b.args if a.is_number]
            if len(ex) == 1 and len(cs) == 1 and abs(abs(float(cs[0])) - 1.0) < 1e-15:
                term, sign = ex[0], 1.0
                if isinstance(term, sp.Mul) and term.args[0].is_number and float(term.args[0]) == -1:
                    term = sp.Mul(*term.args[1:], evaluate=False) if len(term.args) > 2 else term.args[1]
                    sign = -1.0
                # exp(E) - 1 or 1 - exp(E) vanish at E = 0; exp(E) + 1 never does
                if isinstance(term, sp.exp) and sign * float(cs[0]) < 0:
                    r = self._affine_root(term.args[0])
                    if r is not None:
                        out.append(r)
        return out

    def _factor_roots(self, e, in_den, num, den):
        """Roots of the factors of a product (through nested products and reciprocals)."""
        if isinstance(e, sp.Pow) and e.exp.is_Number and float(e.exp) < 0:
            self._factor_roots(e.base, not in_den, num, den)
            return
        if isinstance(e, sp.Mul):
            for a in e.args:
                self._factor_roots(a, in_den, num, den)
            return
        for r in self._zero_roots(e):
            (den if in_den else num).append(r)

    def _fix_expr(self, e):
        V = self.V
        if isinstance(e, sp.Piecewise):
            return sp.Piecewise(*[(self._fix_expr(x), c) for x, c in e.args])
        if V not in _free(e):
            return e
        num, den = [], []
        self._factor_roots(e, False, num, den)
        pts = []
        for v0, c in den:
            if any(abs(v0 - w0) <= 1e-9 * max(1.0, abs(v0)) for w0, _ in num):
                if not any(abs(v0 - p[0]) <= 1e-9 * max(1.0, abs(v0)) for p in pts):
                    pts.append((v0, c))
        for v0, c in pts:
            eps = sp.Mul(self.ueps, sp.Float(1.0 / abs(c), 17), evaluate=False)
            lo = sp.Add(sp.Float(v0, 17), sp.Mul(-1, eps, evaluate=False), evaluate=False)
            hi = sp.Add(sp.Float(v0, 17), eps, evaluate=False)
            with sp.evaluate(False):
                fa = e.xreplace({V: lo})
                fb = e.xreplace({V: hi})
                line = sp.Add(fa, sp.Mul(sp.Add(V, sp.Mul(-1, lo)), sp.Add(fb, sp.Mul(-1, fa)),
                                         sp.Pow(sp.Mul(2, eps), -1)))
                cond = sp.StrictLessThan(sp.Abs(sp.Add(V, sp.Float(-v0, 17))), eps)
            e = sp.Piecewise((line, cond), (e, True))
            self.singular_points.append(v0)
        return e

    def _fix_singularities(self):
        self.ueps = sp.Symbol("__ueps", real=True)
        self.singular = {}
        for k in list(self.live):
            self.singular_points = []
            self.live[k] = self._fix_expr(self.live[k])
            if self.singular_points:
                self.singular[k] = list(self.singular_points)

    def _rl_analysis(self):
        self.rl = {}
        for s in self.states[1:]:
            e = self.odes[s]
            full = self._inline(e, s)
            # evaluated copy (structure-preserving trees do not differentiate
            # cleanly); affine in s <=> d/ds no longer contains s.  No
            # simplification pass: it is far too slow on the calcium ODEs.
            ev = sp.sympify(str(full), locals={str(x): x for x in _free(full)})
            h = sp.diff(ev, s)
            if h == 0 or s in _free(h):
                continue
            g = ev.xreplace({s: sp.Integer(0)})
            inf = -g / h
            self.rl[s] = (inf, h)

    def _state_deps(self, exprs):
        """States the expressions depend on, through the live algebraic variables
        (the stimulus and the capacitance count as a state: they change per substep)."""
        seen, out = set(), set()
        stack = [x for e in exprs for x in _free(e)]
        while stack:
            s_ = stack.pop()
            if s_ in seen:
                continue
            seen.add(s_)
            if s_ in self.states or s_ in (self.stim_arg, self.cm_arg, self.m.time):
                out.add(s_)
            elif s_ in self.live:
                stack.extend(_free(self.live[s_]))
        return out

    def _hoist_voltage_terms(self, outs):
        """Split the per-substep terms (the expressions `outs` of the states that are not
        voltage-only gates) for a clamped voltage: every maximal subexpression that
        depends on V and the parameters alone and holds an exponential, logarithm,
        power, quotient or piecewise branch becomes a voltage term vt[k], computed once
        per PDE step.  Returns (terms, live, outs): the hoisted expressions in order, the
        live definitions with the terms substituted, and the substituted outputs."""
        V = self.V
        fixed = set(self.psyms) | {V}
        if getattr(self, "ueps", None) is not None:
            fixed.add(self.ueps)
        needed = self._needed(outs)
        deps = {s_: self._state_deps([self.live[s_]]) for s_ in needed}
        vonly = {s_ for s_ in needed if deps[s_] == {V}}
        fixed |= {s_ for s_ in needed if not deps[s_]}   # constants: no state, no voltage

        def is_vonly(e):
            # depends on V (directly or through a voltage-only variable) and on nothing
            # that changes between substeps; constant subexpressions stay for the compiler
            free = _free(e)
            return all(x in fixed or x in vonly for x in free) and any(x == V or x in vonly for x in free)

        def costly(e):
            if e.has(sp.exp) or e.has(sp.log) or e.has(sp.Piecewise):
                return True
            return any(not (a.exp.is_Integer and a.exp > 0) for a in e.atoms(sp.Pow))

        terms, memo = [], {}

        def term(e):
            if e not in memo:
                memo[e] = sp.Symbol(f"__vt{len(terms)}", real=True)
                terms.append((memo[e], e))
            return memo[e]

        def rec(e):
            if e.is_Atom:
                if e in vonly and costly(self._fold_expr(self.live[e])):
                    return term(self._fold_expr(self.live[e]))
                return e
            if is_vonly(e) and costly(e):
                return term(e)
            args = [rec(a) for a in e.args]
            if all(a is b for a, b in zip(args, e.args)):
                return e
            with sp.evaluate(False):
                return e.func(*args)

        live = {}
        for s_ in needed:
            e = self._fold_expr(self.live[s_])
            live[s_] = e if (s_ in vonly and costly(e)) else rec(e)
        new_outs = [rec(self._fold_expr(e)) for e in outs]
        return terms, live, new_outs

    def _body_from(self, live, outs, pr, indent="        "):
        """Statements for the symbols of `live` (a substituted definition map) that the
        expressions `outs` need, in dependency order."""
        order, seen = [], set()

        def visit(s_):
            if s_ in seen or s_ not in live:
                return
            seen.add(s_)
            for x in sorted(_free(live[s_]), key=str):
                visit(x)
            order.append(s_)

        for e in outs:
            for x in sorted(_free(e), key=str):
                visit(x)
        return [f"{indent}const T {self.cname(s_)} = {pr(live[s_])};" for s_ in order]

    # ------------------------------------------------------------------ emit
    def cname(self, s):
        if s == self.stim_arg:
            return "stim"
        if s == self.cm_arg:
            return "cm"
        if s == getattr(self, "ueps", None):
            return "chb::singularity_offset<T>()"
        if s in self.psyms:
            return f"p[{self.psyms.index(s)}]"
        if s in self.states:
            return f"y[{self.states.index(s)}]"
        return "v_" + str(s)

    def _needed(self, exprs):
        """Topologically ordered live algebraic symbols needed by exprs."""
        order, seen = [], set()

        def visit(s):
            if s in seen or s not in self.live:
                return
            seen.add(s)
            for x in sorted(_free(self.live[s]), key=str):
                visit(x)
            order.append(s)

        for e in exprs:
            for s in sorted(_free(e), key=str):
                visit(s)
        return order

    def _names(self):
        names = {}
        for s in list(self.live) + list(self.states) + [self.stim_arg, self.cm_arg, self.ueps] + self.psyms:
            names[s] = self.cname(s)
        return names

    def _fold_expr(self, e):
        reps = {s: sp.Float(v, 17) for s, v in self.folded.items() if s in _free(e)}
        if not reps:
            return e
        with sp.evaluate(False):
            return e.xreplace(reps)

    def _body(self, outs, pr, indent="        "):
        """Statements computing every live symbol needed by the expressions in outs."""
        lines = []
        for s in self._needed(outs):
            lines.append(f"{indent}const T {self.cname(s)} = {pr(self._fold_expr(self.live[s]))};")
        return lines

    def emit(self, source_name: str) -> str:
        names = self._names()
        pr = Printer(names)
        n = self.n
        st = self.struct
        V = self.V
        # expressions with V replaced by the (clamped) voltage argument handled by
        # loading y[0] = V before the call
        lines = []
        A = lines.append
        A("// Generated by chaste_b200/codegen/emit.py from " + source_name + ".")
        A("// Do not edit: re-run `python -m chaste_b200.codegen.emit` instead.")
        A("#pragma once")
        A('#include "cellmodel_common.h"')
        A("")
        A("namespace chb {")
        A("")
        A(f"struct {st} {{")
        A(f'    static constexpr const char* kName = "{self.m.name}";')
        A(f"    static constexpr int kNumStates = {n};")
        A(f"    static constexpr int kNumParams = {len(self.pnames)};")
        A(f"    static constexpr bool kCurrentPerCapacitance = {'true' if self.current_per_cap else 'false'};")
        inits = []
        for s in self.states:
            k = self._key_of(s)
            inits.append(_lit(self.m.variables[k].initial_value))
        A(f"    static constexpr double kInitialStates[{n}] = {{{', '.join(inits)}}};")
        snames = ", ".join(f'"{self._key_of(s)[1]}"' for s in self.states)
        A(f"    static constexpr const char* kStateNames[{n}] = {{{snames}}};")
        pn = ", ".join(f'"{p[0]}"' for p in self.pnames)
        A(f"    static constexpr const char* kParamNames[{len(self.pnames)}] = {{{pn}}};")
        rl_flags = ", ".join("true" if s in self.rl else "false" for s in self.states)
        A(f"    // 1 where the state is advanced by Rush-Larsen (ODE affine in itself)")
        A(f"    static constexpr bool kRushLarsen[{n}] = {{{rl_flags}}};")
        rl_idx = [str(i) for i, st in enumerate(self.states) if st in self.rl]
        cond = " || ".join(f"i == {k}" for k in rl_idx) or "false"
        A(f"    CHB_HD static constexpr bool rush_larsen(int i) {{ return {cond}; }}")
        # verify ranges: dimensionless RL states with initial value in [0,1] are gates
        kinds = []
        for s in self.states:
            k = self._key_of(s)
            d = self.m.units_dims[k]
            if s == V:
                kinds.append("0")
            elif all(x == 0 for x in d) and s in self.rl:
                kinds.append("1")   # gate: 0 <= y <= 1
            elif d == _dims(mol=1, m=-3):
                kinds.append("2")   # concentration: y > 0
            else:
                kinds.append("0")
        A(f"    // range class per state: 1 gate in [0,1], 2 concentration > 0, 0 unchecked")
        A(f"    static constexpr int kRangeClass[{n}] = {{{', '.join(kinds)}}};")
        g = [str(i) for i, k in enumerate(kinds) if k == "1"]
        cc = [str(i) for i, k in enumerate(kinds) if k == "2"]
        gc = " || ".join(f"i == {k}" for k in g) or "false"
        ccc = " || ".join(f"i == {k}" for k in cc) or "false"
        A(f"    CHB_HD static constexpr int range_class(int i) {{ return ({gc}) ? 1 : (({ccc}) ? 2 : 0); }}")
        A("")
        # ---- rhs (forward Euler derivatives, all states, dV included)
        dy_exprs = [self.odes[s] for s in self.states]
        A("    // dy/dt for every state at (y, stim) where stim is the Chaste area stimulus")
        A("    // in uA/cm^2 and cm the Chaste capacitance in uF/cm^2.  y[0] is the voltage.")
        A("    template <typename T>")
        A("    CHB_HD static void rhs(const T* __restrict__ y, T stim, T cm,")
        A("                                  const T* __restrict__ p, T* __restrict__ dy) {")
        A("        (void)stim; (void)cm; (void)p;")
        lines.extend(self._body(dy_exprs, pr))
        for i, e in enumerate(dy_exprs):
            A(f"        dy[{i}] = {pr(self._fold_expr(e))};")
        A("    }")
        A("")
        # ---- rush-larsen terms
        A("    // Rush-Larsen terms: for RL states inf[i] is the fixed point and rate[i]")
        A("    // the (negative) affine coefficient h so y' = inf + (y - inf)*exp(h*dt);")
        A("    // for the other states rate[i] holds dy/dt.  rate[0] is dV/dt.")
        A("    template <typename T>")
        A("    CHB_HD static void rl_terms(const T* __restrict__ y, T stim, T cm,")
        A("                                       const T* __restrict__ p, T* __restrict__ rate,")
        A("                                       T* __restrict__ inf) {")
        A("        (void)stim; (void)cm; (void)p; (void)inf;")
        rl_exprs = []
        for s in self.states:
            if s in self.rl:
                inf, h = self.rl[s]
                rl_exprs += [inf, h]
            else:
                rl_exprs.append(self.odes[s])
        lines.extend(self._body(rl_exprs, pr))
        for i, s in enumerate(self.states):
            if s in self.rl:
                inf, h = self.rl[s]
                A(f"        inf[{i}] = {pr(self._fold_expr(inf))};")
                A(f"        rate[{i}] = {pr(self._fold_expr(h))};")
            else:
                A(f"        rate[{i}] = {pr(self._fold_expr(self.odes[s]))};")
        A("    }")
        A("")
        # ---- the same terms split by what they depend on (V clamped over a PDE step)
        vonly = [s_ for s_ in self.states[1:] if s_ in self.rl and self._state_deps(self.rl[s_]) <= {V}]
        vflags = ", ".join("true" if s_ in vonly else "false" for s_ in self.states)
        vidx = " || ".join(f"i == {self.states.index(s_)}" for s_ in vonly) or "false"
        A("    // Rush-Larsen states whose (inf, rate) depend on the voltage alone (and the")
        A("    // parameters): with V clamped over a PDE step (ComputeExceptVoltage) their terms,")
        A("    // and so exp(rate*dt), are the same in every substep.")
        A(f"    static constexpr bool kRlVoltageOnly[{n}] = {{{vflags}}};")
        A(f"    CHB_HD static constexpr bool rl_voltage_only(int i) {{ return {vidx}; }}")
        A(f"    static constexpr int kNumVoltageGates = {len(vonly)};")
        A("    // rl_terms of the voltage-only Rush-Larsen states (reads y[0] and p only).")
        A("    template <typename T>")
        A("    CHB_HD static void rl_terms_voltage(const T* __restrict__ y, const T* __restrict__ p,")
        A("                                       T* __restrict__ rate, T* __restrict__ inf) {")
        A("        (void)p;")
        v_exprs = []
        for s_ in vonly:
            v_exprs += list(self.rl[s_])
        lines.extend(self._body(v_exprs, pr))
        for s_ in vonly:
            i = self.states.index(s_)
            inf, h = self.rl[s_]
            A(f"        inf[{i}] = {pr(self._fold_expr(inf))};")
            A(f"        rate[{i}] = {pr(self._fold_expr(h))};")
        A("    }")
        A("    // rl_terms of every state but the voltage-only gates (dV/dt in rate[0]).")
        A("    template <typename T>")
        A("    CHB_HD static void rl_terms_states(const T* __restrict__ y, T stim, T cm,")
        A("                                       const T* __restrict__ p, T* __restrict__ rate,")
        A("                                       T* __restrict__ inf) {")
        A("        (void)stim; (void)cm; (void)p; (void)inf;")
        r_exprs = []
        for s_ in self.states:
            if s_ in vonly:
                continue
            r_exprs += list(self.rl[s_]) if s_ in self.rl else [self.odes[s_]]
        lines.extend(self._body(r_exprs, pr))
        for i, s_ in enumerate(self.states):
            if s_ in vonly:
                continue
            if s_ in self.rl:
                inf, h = self.rl[s_]
                A(f"        inf[{i}] = {pr(self._fold_expr(inf))};")
                A(f"        rate[{i}] = {pr(self._fold_expr(h))};")
            else:
                A(f"        rate[{i}] = {pr(self._fold_expr(self.odes[s_]))};")
        A("    }")
        # ---- the same split once more: the voltage-only parts of those terms, once per PDE step
        r_outs = []
        for s_ in self.states:
            if s_ in vonly:
                continue
            r_outs += list(self.rl[s_]) if s_ in self.rl else [self.odes[s_]]
        terms, live_vt, outs_vt = self._hoist_voltage_terms(r_outs)
        for k, (sym, _) in enumerate(terms):
            names[sym] = f"vt[{k}]"
        A("    // The subexpressions of rl_terms_states that depend on the voltage and the")
        A("    // parameters alone and hold an exponential, logarithm, power, quotient or branch:")
        A("    // with V clamped over a PDE step they are computed once (rl_vterms) and the")
        A("    // substeps take them from vt (rl_terms_states_vt, the same terms otherwise).")
        A(f"    static constexpr int kNumVTerms = {len(terms)};")
        A("    template <typename T>")
        A("    CHB_HD static void rl_vterms(const T* __restrict__ y, const T* __restrict__ p, T* __restrict__ vt) {")
        A("        (void)y; (void)p; (void)vt;")
        lines.extend(self._body([e for _, e in terms], pr))
        for k, (_, e) in enumerate(terms):
            A(f"        vt[{k}] = {pr(e)};")
        A("    }")
        A("    // vt is anything indexable: the array rl_vterms wrote, or an accessor that")
        A("    // reads each term where it is used (a per-thread column of shared memory).")
        A("    template <typename T, class VT = const T*>")
        A("    CHB_HD static void rl_terms_states_vt(const T* __restrict__ y, T stim, T cm,")
        A("                                          const T* __restrict__ p, const VT& vt,")
        A("                                          T* __restrict__ rate, T* __restrict__ inf) {")
        A("        (void)stim; (void)cm; (void)p; (void)vt; (void)inf;")
        lines.extend(self._body_from(live_vt, outs_vt, pr))
        q = iter(outs_vt)
        for i, s_ in enumerate(self.states):
            if s_ in vonly:
                continue
            if s_ in self.rl:
                A(f"        inf[{i}] = {pr(next(q))};")
                A(f"        rate[{i}] = {pr(next(q))};")
            else:
                A(f"        rate[{i}] = {pr(next(q))};")
        A("    }")
        A("")
        # ---- iionic
        conv = "cm" if self.current_per_cap else None
        tot = sp.Add(*self.currents, evaluate=False)
        f_area = None
        if not self.current_per_cap:
            k = self._key_of(self.currents[0]) if self.currents[0] not in self.scaled else self._key_of(self.scaled[self.currents[0]])
            f_area = self.m.units_factor[k] / 1e-2
        A("    // Total ionic current in uA/cm^2 (GetIIonic): the dV/dt currents without")
        A("    // the stimulus" + (", times the capacitance cm." if self.current_per_cap else "."))
        A("    template <typename T>")
        A("    CHB_HD static T iionic(const T* __restrict__ y, T cm, const T* __restrict__ p) {")
        A("        (void)cm; (void)p;")
        A("        const T stim = T(0.0); (void)stim;")
        lines.extend(self._body([tot], pr))
        if self.current_per_cap:
            A(f"        return {pr(tot)}*cm;")
        else:
            if abs(f_area - 1) > 1e-15:
                A(f"        return {pr(tot)}*T({_lit(f_area)});")
            else:
                A(f"        return {pr(tot)};")
        A("    }")
        # ---- reverse-mode products (adjoint of one forward-Euler step and of GetIIonic)
        lines.extend(self._emit_vjp("vjp_rhs", [(self.odes[s_], f"w[{i}]") for i, s_ in enumerate(self.states)],
                                    "w: weights of dy[0..S-1]"))
        tot = sp.Add(*self.currents, evaluate=False)
        scale = None if not self.current_per_cap else self.cm_arg
        if scale is None and f_area is not None and abs(f_area - 1) > 1e-15:
            tot = sp.Mul(sp.Float(f_area, 17), tot, evaluate=False)
        elif scale is not None:
            tot = sp.Mul(tot, scale, evaluate=False)
        lines.extend(self._emit_vjp("vjp_iionic", [(tot, "w[0]")], "w[0]: weight of iionic", stim_zero=True))
        A("};")
        A("")
        A("}  // namespace chb")
        return "\n".join(lines) + "\n"


def _sym_diff(e, x):
    """d e / d x on an evaluated copy of a structure-preserving expression."""
    ev = sp.sympify(str(e), locals={str(s): s for s in _free(e)})
    return sp.diff(ev, x)


def _vjp_body(self, outputs, pr, stim_zero=False):
    """Statements for: forward recompute, then adjoints a_v of every symbol."""
    needed = self._needed([o for o, _ in outputs])
    body = []
    for s_ in needed:
        body.append(f"        const T {self.cname(s_)} = {pr(self._fold_expr(self.live[s_]))};")
    adj = {}

    def aname(s_):
        if s_ not in adj:
            adj[s_] = "a_" + self.cname(s_).replace("[", "_").replace("]", "").replace(".", "_")
            body.append(f"        T {adj[s_]} = T(0.0);")
        return adj[s_]

    targets = set(self.states) | set(self.psyms)
    acc = []
    for expr, w in outputs:
        e = self._fold_expr(expr)
        for x in sorted(_free(e), key=str):
            if x in targets or x in self.live:
                d = _sym_diff(e, x)
                if d != 0:
                    acc.append((aname(x), f"{w}*({pr(d)})"))
    body.extend(f"        {a} += {t};" for a, t in acc)
    for s_ in reversed(needed):
        if s_ not in adj:
            continue
        e = self._fold_expr(self.live[s_])
        for x in sorted(_free(e), key=str):
            if x in targets or x in self.live:
                d = _sym_diff(e, x)
                if d != 0:
                    body.append(f"        {aname(x)} += {adj[s_]}*({pr(d)});")
    return body, adj


def _emit_vjp(self, fname, outputs, wdoc, stim_zero=False):
    pr = Printer(self._names())
    L = []
    L.append("")
    L.append(f"    // Reverse-mode product for {fname[4:]}: gy[j] += sum_i w_i d(out_i)/d(y_j),")
    L.append(f"    // gp[k] += sum_i w_i d(out_i)/d(p_k)  ({wdoc}; y[0] is the voltage).")
    L.append("    template <typename T>")
    L.append(f"    CHB_HD static void {fname}(const T* __restrict__ y, T stim, T cm, const T* __restrict__ p,")
    L.append("                                const T* __restrict__ w, T* __restrict__ gy, T* __restrict__ gp) {")
    L.append("        (void)stim; (void)cm; (void)p; (void)w; (void)gy; (void)gp;")
    body, adj = _vjp_body(self, outputs, pr, stim_zero)
    L.extend(body)
    for i, st in enumerate(self.states):
        if st in adj:
            L.append(f"        gy[{i}] += {adj[st]};")
    for k, ps in enumerate(self.psyms):
        if ps in adj:
            L.append(f"        gp[{k}] += {adj[ps]};")
    L.append("    }")
    return L


ModelEmitter._emit_vjp = _emit_vjp

MODELS = [("LuoRudy1991.cellml", "LuoRudy1991", "lr91"),
          ("TenTusscher2006Epi.cellml", "TenTusscher2006Epi", "tt06")]


def generate(cellml_dir, out_dirs):
    written = []
    for fname, struct, short in MODELS:
        model = cellml.load(os.path.join(cellml_dir, fname))
        em = ModelEmitter(model, struct)
        text = em.emit(f"heart/src/odes/cellml/{fname}")
        for d in out_dirs:
            os.makedirs(d, exist_ok=True)
            p = os.path.join(d, f"{short}.h")
            with open(p, "w") as fh:
                fh.write(text)
            written.append(p)
    return written


def main(argv=None):
    here = os.path.dirname(os.path.abspath(__file__))
    repo = os.path.dirname(os.path.dirname(here))
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    # the Chaste source tree: --cellml-dir, else $CHASTE_SOURCE_DIR/heart/src/odes/cellml
    src = os.environ.get("CHASTE_SOURCE_DIR")
    ap.add_argument("--cellml-dir", default=os.path.join(src, "heart", "src", "odes", "cellml") if src else None,
                    required=src is None)
    ap.add_argument("--out", nargs="*", default=[os.path.join(repo, "chaste_b200", "csrc", "models")])
    a = ap.parse_args(argv)
    for p in generate(a.cellml_dir, a.out):
        print("wrote", p)


if __name__ == "__main__":
    main()

"""CellML 1.0 reader producing a flat sympy model of a cardiac cell.

This is the front half of the project's CellML route (the role chaste_codegen
plays for Chaste, pinned there as ``chaste_codegen>=0.10.0,<0.11.0`` in
``chaste_codegen.txt:1``; it is not vendored in the reference).  It reads the
model sources Chaste ships, ``heart/src/odes/cellml/LuoRudy1991.cellml`` and
``heart/src/odes/cellml/TenTusscher2006Epi.cellml``, and flattens the component
network into one namespace:

* every ``<connection>`` is resolved to the source variable (the end of the
  chain that is not ``in``), with a units-conversion factor where the two ends
  carry different units;
* ``<math>`` blocks become sympy equations, either algebraic ``x = f(...)`` or
  ODEs ``d(y)/d(time) = f(...)``;
* oxford-metadata annotations (``membrane_voltage``, ``time``,
  ``membrane_stimulus_current`` ...) are kept so the emitter can apply the
  Chaste conventions (voltage first, stimulus replaced by the Chaste stimulus).

Only the MathML subset used by those models is accepted; anything else raises.
"""
from __future__ import annotations

import math
import re
import xml.etree.ElementTree as ET
from dataclasses import dataclass, field

import sympy as sp

NS_CELLML = "http://www.cellml.org/cellml/1.0#"
NS_MATHML = "http://www.w3.org/1998/Math/MathML"
NS_CMETA = "http://www.cellml.org/metadata/1.0#"
NS_RDF = "http://www.w3.org/1999/02/22-rdf-syntax-ns#"
NS_BQBIOL = "http://biomodels.net/biology-qualifiers/"
OXMETA = "https://chaste.comlab.ox.ac.uk/cellml/ns/oxford-metadata#"

# ---------------------------------------------------------------- units ----
# Base dimensions: (A, cd, K, kg, m, mol, s)
_DIMS = ("A", "cd", "K", "kg", "m", "mol", "s")


def _d(**kw):
    return tuple(kw.get(k, 0) for k in _DIMS)


_BUILTIN_UNITS = {
    "dimensionless": (1.0, _d()),
    "ampere": (1.0, _d(A=1)),
    "candela": (1.0, _d(cd=1)),
    "kelvin": (1.0, _d(K=1)),
    "celsius": (1.0, _d(K=1)),
    "kilogram": (1.0, _d(kg=1)),
    "gram": (1e-3, _d(kg=1)),
    "metre": (1.0, _d(m=1)),
    "meter": (1.0, _d(m=1)),
    "mole": (1.0, _d(mol=1)),
    "second": (1.0, _d(s=1)),
    "litre": (1e-3, _d(m=3)),
    "liter": (1e-3, _d(m=3)),
    "coulomb": (1.0, _d(A=1, s=1)),
    "volt": (1.0, _d(kg=1, m=2, s=-3, A=-1)),
    "farad": (1.0, _d(A=2, s=4, kg=-1, m=-2)),
    "siemens": (1.0, _d(A=2, s=3, kg=-1, m=-2)),
    "ohm": (1.0, _d(A=-2, s=-3, kg=1, m=2)),
    "joule": (1.0, _d(kg=1, m=2, s=-2)),
    "watt": (1.0, _d(kg=1, m=2, s=-3)),
    "newton": (1.0, _d(kg=1, m=1, s=-2)),
    "pascal": (1.0, _d(kg=1, m=-1, s=-2)),
    "hertz": (1.0, _d(s=-1)),
    "becquerel": (1.0, _d(s=-1)),
    "katal": (1.0, _d(mol=1, s=-1)),
    "radian": (1.0, _d()),
    "steradian": (1.0, _d()),
}

_PREFIX = {
    "yotta": 24, "zetta": 21, "exa": 18, "peta": 15, "tera": 12, "giga": 9,
    "mega": 6, "kilo": 3, "hecto": 2, "deka": 1, "deca": 1, "deci": -1,
    "centi": -2, "milli": -3, "micro": -6, "nano": -9, "pico": -12,
    "femto": -15, "atto": -18, "zepto": -21, "yocto": -24,
}


def _tag(e):
    return e.tag.split("}", 1)[1] if "}" in e.tag else e.tag


@dataclass
class Variable:
    component: str
    name: str
    units: str
    initial_value: float | None
    public: str | None
    private: str | None
    cmeta_id: str | None
    annotations: list = field(default_factory=list)

    @property
    def key(self):
        return (self.component, self.name)


@dataclass
class CellModel:
    """Flattened model: symbols are sympy Symbols named ``component__name``."""

    name: str
    symbols: dict            # key -> sympy Symbol (source variables only)
    variables: dict          # key -> Variable (source variables only)
    units_factor: dict       # key -> SI factor of the variable's units
    units_dims: dict         # key -> SI dims
    algebraic: dict          # Symbol -> expr
    odes: dict               # state Symbol -> expr (document order)
    states: list             # state Symbols, document order
    constants: dict          # Symbol -> float
    time: sp.Symbol
    annotations: dict        # oxmeta term -> Symbol

    def symbol_for(self, component, name):
        return self.symbols[(component, name)]

    def find(self, name):
        """Return the unique source symbol whose variable name is ``name``."""
        hits = [s for k, s in self.symbols.items() if k[1] == name]
        if len(hits) != 1:
            raise KeyError(f"{name!r}: {len(hits)} matches")
        return hits[0]


class CellMLReader:
    def __init__(self, path):
        self.path = path
        self.root = ET.parse(path).getroot()
        if self.root.tag != f"{{{NS_CELLML}}}model":
            raise ValueError("not a CellML 1.0 model")
        self.units = {}          # model-level units
        self.comp_units = {}     # component -> {name: (f, dims)}
        self.vars = {}           # (comp, name) -> Variable
        self.math = {}           # comp -> [math elements]
        self._read()

    # ------------------------------------------------------------ units --
    def _unit_def(self, el, scope):
        factor, dims = 1.0, [0] * len(_DIMS)
        if el.get("base_units") == "yes":
            raise ValueError("new base units are not supported")
        for u in el.findall(f"{{{NS_CELLML}}}unit"):
            f_u, d_u = self._lookup_units(u.get("units"), scope)
            pre = u.get("prefix")
            p = 0
            if pre:
                p = _PREFIX[pre] if pre in _PREFIX else int(pre)
            e = float(u.get("exponent", "1"))
            m = float(u.get("multiplier", "1"))
            factor *= m * (10.0 ** p * f_u) ** e
            for i in range(len(_DIMS)):
                dims[i] += e * d_u[i]
        return factor, tuple(dims)

    def _lookup_units(self, name, scope=None):
        if scope and name in self.comp_units.get(scope, {}):
            return self.comp_units[scope][name]
        if name in self.units:
            return self.units[name]
        if name in _BUILTIN_UNITS:
            return _BUILTIN_UNITS[name]
        raise KeyError(f"unknown units {name!r}")

    # ------------------------------------------------------------- read --
    def _read(self):
        r = self.root
        pending = {u.get("name"): u for u in r.findall(f"{{{NS_CELLML}}}units")}
        # resolve model-level units in dependency order
        while pending:
            progress = False
            for name, el in list(pending.items()):
                try:
                    self.units[name] = self._unit_def(el, None)
                except KeyError:
                    continue
                del pending[name]
                progress = True
            if not progress:
                raise ValueError(f"unresolvable units: {sorted(pending)}")
        for comp in r.findall(f"{{{NS_CELLML}}}component"):
            cname = comp.get("name")
            cu = {}
            self.comp_units[cname] = cu
            for u in comp.findall(f"{{{NS_CELLML}}}units"):
                cu[u.get("name")] = self._unit_def(u, cname)
            for v in comp.findall(f"{{{NS_CELLML}}}variable"):
                iv = v.get("initial_value")
                ann = [res.get(f"{{{NS_RDF}}}resource")
                       for res in v.iter(f"{{{NS_BQBIOL}}}is")]
                var = Variable(cname, v.get("name"), v.get("units"),
                               float(iv) if iv is not None else None,
                               v.get("public_interface"), v.get("private_interface"),
                               v.get(f"{{{NS_CMETA}}}id"), ann)
                self.vars[var.key] = var
            self.math[cname] = comp.findall(f"{{{NS_MATHML}}}math")
        # top-level rdf annotations (rdf:about="#id")
        self.top_annotations = {}
        for desc in r.iter(f"{{{NS_RDF}}}Description"):
            about = desc.get(f"{{{NS_RDF}}}about")
            if not about or not about.startswith("#"):
                continue
            for res in desc.iter(f"{{{NS_BQBIOL}}}is"):
                self.top_annotations.setdefault(about[1:], []).append(
                    res.get(f"{{{NS_RDF}}}resource"))
        self.connections = []
        for c in r.findall(f"{{{NS_CELLML}}}connection"):
            mc = c.find(f"{{{NS_CELLML}}}map_components")
            c1, c2 = mc.get("component_1"), mc.get("component_2")
            for mv in c.findall(f"{{{NS_CELLML}}}map_variables"):
                self.connections.append(((c1, mv.get("variable_1")),
                                         (c2, mv.get("variable_2"))))

    # ------------------------------------------------------- flattening --
    def build(self) -> CellModel:
        # union-find over connected variables
        parent = {k: k for k in self.vars}

        def find(k):
            while parent[k] != k:
                parent[k] = parent[parent[k]]
                k = parent[k]
            return k

        for a, b in self.connections:
            ra, rb = find(a), find(b)
            if ra != rb:
                parent[ra] = rb
        groups = {}
        for k in self.vars:
            groups.setdefault(find(k), []).append(k)

        # which variables are defined by an equation (lhs)
        defined = set()
        for comp, maths in self.math.items():
            for m in maths:
                for eq in m:
                    lhs = eq[1]
                    if _tag(lhs) == "ci":
                        defined.add((comp, lhs.text.strip()))
                    elif _tag(lhs) == "apply" and _tag(lhs[0]) == "diff":
                        defined.add((comp, lhs[-1].text.strip()))

        source_of = {}
        for members in groups.values():
            srcs = [k for k in members
                    if self.vars[k].initial_value is not None or k in defined
                    or (self.vars[k].public != "in" and self.vars[k].private != "in")]
            srcs = [k for k in srcs if self.vars[k].public != "in"
                    and self.vars[k].private != "in"] or srcs
            if len(srcs) != 1:
                raise ValueError(f"cannot find unique source among {members}: {srcs}")
            for k in members:
                source_of[k] = srcs[0]

        symbols, variables, ufac, udims = {}, {}, {}, {}
        for k, v in self.vars.items():
            s = source_of[k]
            if s == k:
                sym = sp.Symbol(f"{k[0]}__{k[1]}", real=True)
                symbols[k] = sym
                variables[k] = v
                f, d = self._lookup_units(v.units, k[0])
                ufac[k], udims[k] = f, d

        def ref(comp, name):
            """Expression for a ci reference inside component ``comp``."""
            k = (comp, name)
            s = source_of[k]
            sym = symbols[s]
            f_local, d_local = self._lookup_units(self.vars[k].units, comp)
            if s != k:
                f_src = ufac[s]
                if d_local != udims[s]:
                    raise ValueError(f"dimension mismatch connecting {k} to {s}")
                conv = f_src / f_local
                if abs(conv - 1.0) > 1e-15:
                    return sp.Mul(sp.Float(conv, 17), sym, evaluate=False)
            return sym

        # time
        time_keys = [k for k, v in variables.items()
                     if any(a == OXMETA + "time" for a in self._ann(v))]
        if not time_keys:
            # no annotation: the free variable is the bvar of the ODEs
            bvars = set()
            for comp, maths in self.math.items():
                for m in maths:
                    for b in m.iter(f"{{{NS_MATHML}}}bvar"):
                        bvars.add(source_of[(comp, b[0].text.strip())])
            time_keys = sorted(bvars)
        if len(time_keys) != 1:
            raise ValueError("model needs exactly one oxmeta:time variable")
        time = symbols[time_keys[0]]

        algebraic, odes = {}, {}
        for comp, maths in self.math.items():
            for m in maths:
                for eq in m:
                    if _tag(eq) != "apply" or _tag(eq[0]) != "eq":
                        raise ValueError("only <apply><eq/> equations are supported")
                    lhs, rhs = eq[1], eq[2]
                    rexpr = self._expr(rhs, comp, ref)
                    if _tag(lhs) == "ci":
                        sym = symbols[source_of[(comp, lhs.text.strip())]]
                        if source_of[(comp, lhs.text.strip())] != (comp, lhs.text.strip()):
                            raise ValueError("equation defines a non-source variable")
                        algebraic[sym] = rexpr
                    else:
                        state_name = lhs[-1].text.strip()
                        bvar = lhs.find(f"{{{NS_MATHML}}}bvar")[0].text.strip()
                        if ref(comp, bvar) != time:
                            raise ValueError("ODE not with respect to time")
                        skey = source_of[(comp, state_name)]
                        if skey != (comp, state_name):
                            raise ValueError("ODE defines a non-source variable")
                        # d(y)/dt in the component's own units; time units may
                        # differ from the source time units
                        f_t_local, _ = self._lookup_units(self.vars[(comp, bvar)].units, comp)
                        f_t_src = ufac[time_keys[0]]
                        scale = f_t_src / f_t_local
                        if abs(scale - 1.0) > 1e-15:
                            rexpr = sp.Mul(sp.Float(scale, 17), rexpr, evaluate=False)
                        odes[symbols[skey]] = rexpr
        states = [s for s in odes]
        constants = {}
        for k, v in variables.items():
            sym = symbols[k]
            if sym in odes:
                if v.initial_value is None:
                    raise ValueError(f"state {k} lacks an initial value")
                continue
            if sym in algebraic or sym == time:
                continue
            if v.initial_value is None:
                raise ValueError(f"variable {k} is neither defined nor initialised")
            constants[sym] = v.initial_value
        annotations = {}
        for k, v in variables.items():
            for a in self._ann(v):
                if a and a.startswith(OXMETA):
                    annotations[a[len(OXMETA):]] = symbols[k]
        name = self.root.get("name")
        return CellModel(name, symbols, variables, ufac, udims, algebraic, odes,
                         states, constants, time, annotations)

    def _ann(self, v):
        out = list(v.annotations)
        if v.cmeta_id and v.cmeta_id in self.top_annotations:
            out += self.top_annotations[v.cmeta_id]
        return out

    # ------------------------------------------------------- expressions --
    def _expr(self, e, comp, ref):
        t = _tag(e)
        if t == "ci":
            return ref(comp, e.text.strip())
        if t == "cn":
            if e.get("type") == "e-notation":
                parts = [p.strip() for p in e.itertext() if p.strip()]
                return sp.Float(float(parts[0]) * 10.0 ** float(parts[1]), 17)
            txt = e.text.strip()
            v = float(txt)
            if re.fullmatch(r"[+-]?\d+", txt):
                return sp.Integer(int(txt))
            return sp.Float(v, 17)
        if t == "piecewise":
            pieces = []
            other = None
            for p in e:
                if _tag(p) == "piece":
                    pieces.append((self._expr(p[0], comp, ref), self._cond(p[1], comp, ref)))
                elif _tag(p) == "otherwise":
                    other = self._expr(p[0], comp, ref)
            if other is None:
                other = sp.nan
            pieces.append((other, True))
            return sp.Piecewise(*pieces)
        if t == "apply":
            op = _tag(e[0])
            args = [self._expr(a, comp, ref) for a in e[1:]
                    if _tag(a) not in ("degree", "bvar", "logbase")]
            # Structure is preserved (evaluate=False) so that the emitted
            # code follows the CellML expression tree term by term.
            if op == "plus":
                return sp.Add(*args, evaluate=False)
            if op == "minus":
                if len(args) == 1:
                    return sp.Mul(sp.Integer(-1), args[0], evaluate=False)
                return sp.Add(args[0], sp.Mul(sp.Integer(-1), args[1], evaluate=False),
                              evaluate=False)
            if op == "times":
                return sp.Mul(*args, evaluate=False)
            if op == "divide":
                return sp.Mul(args[0], sp.Pow(args[1], sp.Integer(-1), evaluate=False),
                              evaluate=False)
            if op == "power":
                return sp.Pow(args[0], args[1], evaluate=False)
            if op == "exp":
                return sp.exp(args[0])
            if op == "ln":
                return sp.log(args[0])
            if op == "log":
                return sp.log(args[0], 10)
            if op == "floor":
                return sp.floor(args[0])
            if op == "abs":
                return sp.Abs(args[0])
            if op == "root":
                deg = e.find(f"{{{NS_MATHML}}}degree")
                if deg is not None:
                    return sp.Pow(args[0], 1 / self._expr(deg[0], comp, ref))
                return sp.sqrt(args[0])
            raise ValueError(f"unsupported MathML operator {op}")
        raise ValueError(f"unsupported MathML element {t}")

    def _cond(self, e, comp, ref):
        op = _tag(e[0])
        if op in ("and", "or"):
            parts = [self._cond(a, comp, ref) for a in e[1:]]
            return sp.And(*parts) if op == "and" else sp.Or(*parts)
        a, b = (self._expr(x, comp, ref) for x in e[1:3])
        return {"lt": sp.StrictLessThan, "leq": sp.LessThan, "gt": sp.StrictGreaterThan,
                "geq": sp.GreaterThan, "eq": sp.Eq, "neq": sp.Ne}[op](a, b, evaluate=False)


def load(path) -> CellModel:
    return CellMLReader(path).build()

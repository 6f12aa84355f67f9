"""Host-side mirror of Chaste's monodomain API over the GPU tissue.

Names and argument meanings follow the reference so a Chaste user finds the
same calls:

* :class:`HeartConfig` -- ``heart/src/problem/HeartConfig.hpp`` (the fields
  this path reads; defaults of ``HeartConfigDefaults.hpp:53-91``);
* :class:`SimpleStimulus`, :class:`RegularStimulus`, :class:`ZeroStimulus` --
  ``heart/src/stimulus``;
* :func:`CellLuoRudy1991FromCellML`, :func:`CellTenTusscher2006EpiFromCellML`
  -- the chaste_codegen cell classes (here: which generated model a node runs);
* :class:`AbstractCardiacCellFactory`, :class:`PlaneStimulusCellFactory` --
  ``heart/src/problem/cell_factories``;
* :class:`MonodomainProblem` -- ``heart/src/problem/MonodomainProblem.hpp`` with
  ``Initialise``/``Solve``/``GetSolution``/``GetTissue``;
* :class:`GpuMonodomainTissue` -- the tissue view (``rGetIionicCacheReplicated``,
  ``GetCardiacCell(i)`` ...), served from device memory.

Everything numeric runs in libchastegpu.so.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .codegen import PARAM_NAMES, STATE_NAMES

DBL_MAX = 1.7976931348623157e308


# ----------------------------------------------------------------- config --
class HeartConfig:
    """Singleton holding the options of the monodomain path."""

    _instance = None

    @classmethod
    def Instance(cls) -> "HeartConfig":
        if cls._instance is None:
            cls._instance = cls()
        return cls._instance

    def __init__(self):
        self.Reset()

    def Reset(self):
        self.simulation_duration = 10.0
        self.ode_dt = 0.01
        self.pde_dt = 0.01
        self.printing_dt = 0.01
        self.am = 1400.0
        self.cm = 1.0
        self.sigma = (1.75, 1.75, 1.75)
        self.use_abs_tol = True
        self.tol = 2e-4
        self.ksp_pc = "bjacobi"       # HeartConfigDefaults.hpp:83
        self.mass_lumping = False
        self.space_dimension = 3
        self.slab = None          # (width, height, depth, h)
        self.precision = "fp64"
        self.activation_threshold = -40.0
        self.check_state_ranges = False
        self.device = 0
        self.operator_splitting = False
        self.state_variable_interpolation = False
        self.output_variables = []
        self.apd_maps = []
        self.upstroke_time_maps = []
        self.max_upstroke_velocity_maps = []
        self.conduction_velocity_maps = []
        self.keep_output = True

    # HeartConfig.cpp:1581-1587, 2337
    def SetOdeTimeStep(self, dt):
        self.ode_dt = dt

    def SetPdeTimeStep(self, dt):
        self.pde_dt = dt

    def SetPrintingTimeStep(self, dt):
        self.printing_dt = dt

    def SetOdePdeAndPrintingTimeSteps(self, ode, pde, printing):
        self.ode_dt, self.pde_dt, self.printing_dt = ode, pde, printing

    def GetOdeTimeStep(self):
        return self.ode_dt

    def GetPdeTimeStep(self):
        return self.pde_dt

    def SetSimulationDuration(self, t):
        self.simulation_duration = t

    def GetSimulationDuration(self):
        return self.simulation_duration

    def SetSurfaceAreaToVolumeRatio(self, am):
        self.am = am

    def GetSurfaceAreaToVolumeRatio(self):
        return self.am

    def SetCapacitance(self, cm):
        self.cm = cm

    def GetCapacitance(self):
        return self.cm

    def SetIntracellularConductivities(self, sigma):
        s = tuple(float(x) for x in np.atleast_1d(sigma))
        self.sigma = s + (s[-1],) * (3 - len(s))

    # HeartConfig.cpp:2404-2412
    def SetUseAbsoluteTolerance(self, tol):
        self.use_abs_tol, self.tol = True, tol

    def SetUseRelativeTolerance(self, tol):
        self.use_abs_tol, self.tol = False, tol

    def GetUseAbsoluteTolerance(self):
        return self.use_abs_tol

    def SetKSPSolver(self, name):
        if name != "cg":
            raise ValueError("the GPU tissue solves with CG (the monodomain matrix is SPD)")

    def SetKSPPreconditioner(self, name):
        if name not in ("bjacobi", "jacobi", "none"):
            raise ValueError(f"unsupported preconditioner {name!r} (bjacobi, jacobi or none)")
        self.ksp_pc = name

    def SetUseMassLumping(self, flag=True):
        self.mass_lumping = bool(flag)

    # HeartConfig::SetUseReactionDiffusionOperatorSplitting (MonodomainProblem.cpp:65-69
    # then builds an OperatorSplittingMonodomainSolver)
    def SetUseReactionDiffusionOperatorSplitting(self, flag=True):
        self.operator_splitting = bool(flag)

    def GetUseReactionDiffusionOperatorSplitting(self):
        return self.operator_splitting

    # HeartConfig::SetUseStateVariableInterpolation (MonodomainSolver.cpp:200-209 then
    # adds MonodomainCorrectionTermAssembler's vector to the RHS at :122-126)
    def SetUseStateVariableInterpolation(self, flag=True):
        self.state_variable_interpolation = bool(flag)

    def GetUseStateVariableInterpolation(self):
        return self.state_variable_interpolation

    # Output at printing steps (HeartConfig::SetOutputVariables) and the post-processing
    # maps PostProcessingWriter writes (HeartConfig::SetApdMaps, SetUpstrokeTimeMaps,
    # SetMaxUpstrokeVelocityMaps, SetConductionVelocityMaps), computed on the device
    def SetOutputVariables(self, names):
        self.output_variables = list(names)

    def SetApdMaps(self, maps):
        self.apd_maps = [(float(p), float(t)) for p, t in maps]

    def SetUpstrokeTimeMaps(self, thresholds):
        self.upstroke_time_maps = [float(t) for t in thresholds]

    def SetMaxUpstrokeVelocityMaps(self, thresholds):
        self.max_upstroke_velocity_maps = [float(t) for t in thresholds]

    def SetConductionVelocityMaps(self, origin_nodes):
        self.conduction_velocity_maps = [int(o) for o in origin_nodes]

    def IsPostProcessingRequested(self):
        return bool(self.apd_maps or self.upstroke_time_maps or self.max_upstroke_velocity_maps
                    or self.conduction_velocity_maps)

    # extension of this library: keep the printing-step frames on the device (default on)
    def SetKeepOutputOnDevice(self, flag=True):
        self.keep_output = bool(flag)

    def SetFibreLength(self, length, h):
        self.space_dimension, self.slab = 1, (length, 0.0, 0.0, h)

    def SetSheetDimensions(self, w, hgt, h):
        self.space_dimension, self.slab = 2, (w, hgt, 0.0, h)

    def SetSlabDimensions(self, w, hgt, d, h):
        self.space_dimension, self.slab = 3, (w, hgt, d, h)

    def SetSpaceDimension(self, d):
        self.space_dimension = d

    # extension of this library: FP32 states + FP32 inner CG with FP64 refinement.  The
    # mixed solve's FP64 residual test is Jacobi-preconditioned: a bjacobi request is
    # served by Jacobi in that mode (the converged solution meets the same tolerance).
    def SetPrecision(self, name):
        if name not in ("fp64", "mixed"):
            raise ValueError(name)
        self.precision = name


# -------------------------------------------------------------- stimulus --
@dataclass
class ZeroStimulus:
    def as_native(self):
        return None

    def GetStimulus(self, t):
        return 0.0


@dataclass
class SimpleStimulus:
    magnitude: float
    duration: float
    start: float = 0.0

    def as_native(self):
        return N.stimulus(N.STIM_SIMPLE, self.magnitude, self.duration, self.start)


@dataclass
class RegularStimulus:
    magnitude: float
    duration: float
    period: float
    start: float
    stop: float = DBL_MAX

    def as_native(self):
        return N.stimulus(N.STIM_REGULAR, self.magnitude, self.duration, self.start, self.period, self.stop)


# ------------------------------------------------------------------ cells --
@dataclass
class CellSpec:
    """What a chaste_codegen cell object fixes for a node: model, solver, stimulus, parameters."""

    model: int
    stimulus: object
    solver: str = "ForwardEuler"
    params: dict = field(default_factory=dict)

    def SetParameter(self, name, value):
        if name not in PARAM_NAMES[self.model]:
            raise KeyError(f"no parameter {name!r}; have {PARAM_NAMES[self.model]}")
        self.params[name] = float(value)


def CellLuoRudy1991FromCellML(stimulus=None, solver="ForwardEuler"):
    return CellSpec(N.MODEL_LR91, stimulus or ZeroStimulus(), solver)


def CellTenTusscher2006EpiFromCellML(stimulus=None, solver="RushLarsen"):
    return CellSpec(N.MODEL_TT06, stimulus or ZeroStimulus(), solver)


def CellLuoRudy1991FromCellMLBackwardEuler(stimulus=None):
    """The backward-Euler variant chaste_codegen generates (CellLuoRudy1991FromCellMLBackwardEuler)."""
    return CellLuoRudy1991FromCellML(stimulus, "BackwardEuler")


def CellTenTusscher2006EpiFromCellMLBackwardEuler(stimulus=None):
    return CellTenTusscher2006EpiFromCellML(stimulus, "BackwardEuler")


def CellLuoRudy1991FromCellMLGRL1(stimulus=None):
    return CellSpec(N.MODEL_LR91, stimulus or ZeroStimulus(), "GRL1")


def CellLuoRudy1991FromCellMLGRL2(stimulus=None):
    return CellSpec(N.MODEL_LR91, stimulus or ZeroStimulus(), "GRL2")


def CellTenTusscher2006EpiFromCellMLGRL1(stimulus=None):
    return CellSpec(N.MODEL_TT06, stimulus or ZeroStimulus(), "GRL1")


def CellTenTusscher2006EpiFromCellMLGRL2(stimulus=None):
    return CellSpec(N.MODEL_TT06, stimulus or ZeroStimulus(), "GRL2")


class AbstractCardiacCellFactory:
    """Per-node cell creation (AbstractCardiacCellFactory.cpp:42-67)."""

    def CreateCardiacCellForTissueNode(self, index, x):
        raise NotImplementedError


class PlaneStimulusCellFactory(AbstractCardiacCellFactory):
    """PlaneStimulusCellFactory.hpp:62-86: stimulate the nodes with x^2 <= 1e-10."""

    def __init__(self, cell=CellLuoRudy1991FromCellML, magnitude=-600.0, duration=0.5, solver=None):
        self.cell = cell
        self.stim = SimpleStimulus(magnitude, duration)
        self.solver = solver

    def CreateCardiacCellForTissueNode(self, index, x):
        stim = self.stim if x[0] * x[0] <= 1e-10 else ZeroStimulus()
        return self.cell(stim) if self.solver is None else self.cell(stim, self.solver)


class CuboidStimulusCellFactory(AbstractCardiacCellFactory):
    """Stimulus on the nodes inside an axis-aligned box (corner-cube protocols)."""

    def __init__(self, cell, magnitude, duration, lo, hi, solver=None):
        self.cell, self.solver = cell, solver
        self.stim = SimpleStimulus(magnitude, duration)
        self.lo, self.hi = np.asarray(lo, float), np.asarray(hi, float)

    def CreateCardiacCellForTissueNode(self, index, x):
        d = len(self.lo)
        inside = bool(np.all(x[:d] >= self.lo) and np.all(x[:d] <= self.hi))
        stim = self.stim if inside else ZeroStimulus()
        return self.cell(stim) if self.solver is None else self.cell(stim, self.solver)


# ----------------------------------------------------------------- tissue --
class GpuMonodomainTissue:
    """Device-resident tissue: the AbstractCardiacTissue view of a N.Tissue."""

    def __init__(self, native: N.Tissue, xyz):
        self.native = native
        self.xyz = xyz

    def rGetIionicCacheReplicated(self):
        return self.native.caches()[0]

    def rGetIntracellularStimulusCacheReplicated(self):
        return self.native.caches()[1]

    def GetCardiacCell(self, index):
        return _CellView(self.native, index)

    def GetNumNodes(self):
        return self.native.n


class _CellView:
    """AbstractCardiacCellInterface view of one node (lazy device->host reads)."""

    def __init__(self, native, index):
        self.native, self.index = native, index

    def rGetStateVariables(self):
        return self.native.cell_state(self.index)

    def GetStdVecStateVariables(self):
        return list(self.rGetStateVariables())

    def GetVoltage(self):
        return float(self.rGetStateVariables()[0])

    def GetIIonic(self):
        return float(self.native.caches()[0][self.index])


def slab_coordinates(dim, h, width, height=0.0, depth=0.0):
    """Node coordinates in ConstructRegularSlabMesh order ((k*NY + j)*NX + i)."""
    nx = int((width + 0.5 * h) / h) + 1
    ny = int((height + 0.5 * h) / h) + 1 if dim > 1 else 1
    nz = int((depth + 0.5 * h) / h) + 1 if dim > 2 else 1
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    return np.stack([i.ravel() * h, j.ravel() * h, k.ravel() * h], axis=1)


# Transmural cell heterogeneity of the ten Tusscher 2006 model: the scale factors
# (ScaleFactorGks, ScaleFactorIto, ScaleFactorGkr) of the three layers as Chaste's
# default parameter file lists them (ChasteParameters.xml:54-92, CellHeterogeneity
# #1 endo, #2 mid-myocardial, #3 epi), which HeartConfigRelatedCellFactory applies
# per node (heart/src/problem/cell_factories/HeartConfigRelatedCellFactory.cpp:355-440,
# layers 0 endo, 1 mid, 2 epi as HeartGeometryInformation::DetermineLayerForEachNode
# numbers them).
TRANSMURAL_SCALE_FACTORS = ((0.462, 0.0, 1.0), (1.154, 0.85, 1.0), (1.154, 1.0, 1.0))


def transmural_layers(z, depth):
    """Layer of each node of a slab of the given depth by thirds of z: 0 endo
    (z < depth/3), 1 mid (z < 2 depth/3), 2 epi."""
    z = np.asarray(z, dtype=np.float64)
    third = depth / 3.0
    return np.where(z < third - 1e-12, 0, np.where(z < 2.0 * third - 1e-12, 1, 2)).astype(np.int32)


def transmural_param_table():
    """Per-layer parameter rows of the TT06 model (cg_set_cells' param_table): the six
    conductance scales at 1 and ScaleFactorGks, ScaleFactorGkr, ScaleFactorIto of the layer."""
    rows = []
    for gks, ito, gkr in TRANSMURAL_SCALE_FACTORS:
        rows.append([1.0] * 6 + [gks, gkr, ito])
    return np.asarray(rows)


# ---------------------------------------------------------------- problem --
class MonodomainProblem:
    """MonodomainProblem<DIM> (heart/src/problem/MonodomainProblem.cpp:45-77)."""

    def __init__(self, cell_factory: AbstractCardiacCellFactory, dim=None):
        self.factory = cell_factory
        self.dim = dim
        self.mesh = None
        self.tissue = None
        self.native = None
        self.output_modifiers = []
        self._initialised = False
        self._output_on = False
        self.post_processing = {}
        self.max_paces = 32        # columns kept per node in the post-processing maps

    def SetMesh(self, xyz, conn):
        self.mesh = (np.asarray(xyz, float), np.asarray(conn, np.int32))

    def GetTissue(self):
        if self.tissue is None:
            raise RuntimeError("Tissue not yet set up, you may need to call Initialise() before GetTissue().")
        return self.tissue

    def _config(self):
        hc = HeartConfig.Instance()
        cfg = N.default_config()
        cfg.ode_time_step = hc.ode_dt
        cfg.pde_time_step = hc.pde_dt
        cfg.surface_area_to_volume_ratio = hc.am
        cfg.capacitance = hc.cm
        cfg.use_absolute_tolerance = 1 if hc.use_abs_tol else 0
        cfg.ksp_tolerance = hc.tol
        pc = hc.ksp_pc
        if pc == "bjacobi" and hc.precision == "mixed":
            pc = "jacobi"
        cfg.ksp_preconditioner = {"bjacobi": N.PC_BJACOBI, "jacobi": N.PC_JACOBI, "none": N.PC_NONE}[pc]
        cfg.use_mass_lumping = 1 if hc.mass_lumping else 0
        cfg.precision = N.PRECISION_MIXED if hc.precision == "mixed" else N.PRECISION_FP64
        cfg.activation_threshold = hc.activation_threshold
        cfg.check_state_ranges = 1 if hc.check_state_ranges else 0
        cfg.device = hc.device
        cfg.solver = N.SOLVER_OPERATOR_SPLITTING if hc.operator_splitting else N.SOLVER_MONODOMAIN
        cfg.use_state_variable_interpolation = int(hc.state_variable_interpolation)
        return cfg

    def Initialise(self):
        """Fix the mesh; the tissue itself is built by the first Solve, after HeartConfig
        changes made between Initialise and Solve (as Chaste's tests make them)."""
        hc = HeartConfig.Instance()
        if self.mesh is None and hc.slab is None:
            raise RuntimeError("no mesh: call SetMesh or HeartConfig.Set{Fibre,Sheet,Slab}Dimensions")
        self._initialised = True

    def _build(self):
        hc = HeartConfig.Instance()
        cfg = self._config()
        if self.mesh is None:
            w, hh, d, h = hc.slab
            dim = self.dim or hc.space_dimension
            xyz = slab_coordinates(dim, h, w, hh, d)
        else:
            xyz, conn = self.mesh
            dim = conn.shape[1] - 1
        specs = [self.factory.CreateCardiacCellForTissueNode(i, xyz[i]) for i in range(xyz.shape[0])]
        models = {s.model for s in specs}
        solvers = {s.solver for s in specs}
        if len(models) != 1 or len(solvers) != 1:
            raise ValueError("a GPU tissue runs one cell model with one ODE solver")
        cfg.model = models.pop()
        cfg.ode_method = {"RushLarsen": N.ODE_RUSH_LARSEN, "BackwardEuler": N.ODE_BACKWARD_EULER,
                          "GRL1": N.ODE_GRL1, "GRL2": N.ODE_GRL2}.get(solvers.pop(), N.ODE_FORWARD_EULER)
        native = N.Tissue(cfg)
        if self.mesh is None:
            native.set_slab_mesh(dim, hc.slab[3], hc.slab[0], hc.slab[1], hc.slab[2], hc.sigma)
        else:
            native.set_mesh(xyz, self.mesh[1], np.asarray(hc.sigma[:dim]))
        names = PARAM_NAMES[cfg.model]
        sets, pset = {}, np.zeros(native.n, np.int32)
        for i, s in enumerate(specs):
            pset[i] = sets.setdefault(tuple(sorted(s.params.items())), len(sets))
        if len(sets) == 1 and not specs[0].params:
            native.set_cells()
        else:
            table = np.ones((len(sets), len(names)))
            for key, k in sets.items():
                for name, val in key:
                    table[k, names.index(name)] = val
            native.set_cells(param_set=pset, param_table=table)
        stims, sid, index = [], np.full(native.n, -1, np.int32), {}
        for i, s in enumerate(specs):
            nat = s.stimulus.as_native()
            if nat is None:
                continue
            key = (nat.kind, nat.magnitude, nat.duration, nat.start, nat.period, nat.stop)
            if key not in index:
                index[key] = len(stims)
                stims.append(nat)
            sid[i] = index[key]
        native.set_stimulus(sid, stims)
        self.native = native
        self.tissue = GpuMonodomainTissue(native, xyz)

    def Solve(self):
        """Advance to the simulation duration (AbstractCardiacProblem::Solve, printing-step loop)."""
        if not self._initialised:
            raise RuntimeError("call Initialise() before Solve()")
        hc = HeartConfig.Instance()
        if self.native is None:
            self._build()
        n_total = int(round(hc.simulation_duration / hc.pde_dt))
        per_print = max(1, int(round(hc.printing_dt / hc.pde_dt)))
        done = self.native.stats().steps
        if (hc.keep_output or hc.IsPostProcessingRequested()) and not self._output_on:
            names = STATE_NAMES[self.native.cfg.model]
            idx = [names.index(v) for v in hc.output_variables]
            self.native.configure_output(per_print, (n_total - done) // per_print + 1, idx)
            self._output_on = True
        while done < n_total:
            k = min(per_print, n_total - done)
            self.native.step(k)
            done += k
            for m in self.output_modifiers:
                m(done * hc.pde_dt, self.native)
        if hc.IsPostProcessingRequested():
            self._post_process(hc)

    @staticmethod
    def _hdf5_friendly(threshold):
        """PostProcessingWriter::ConvertToHdf5FriendlyString (PostProcessingWriter.cpp:394-416)."""
        extra = "_"
        if threshold < 0.0:
            extra += "minus_"
            threshold = -threshold
        if threshold - np.floor(threshold) > 1e-8:
            return f"{extra}{int(np.floor(threshold))}pt{int(np.floor(threshold * 100) - np.floor(threshold) * 100)}"
        return f"{extra}{threshold:g}"

    def _post_process(self, hc):
        """PostProcessingWriter::WritePostProcessingFiles (PostProcessingWriter.cpp:73-125),
        each map as per-node lists under its dataset name."""
        out = {}
        for pct, thr in hc.apd_maps:
            m = self.native.cell_property_maps(pct, thr, max_aps=self.max_paces)
            out[f"Apd_{pct:g}{self._hdf5_friendly(thr)}_Map"] = m["apd"]
        for thr in hc.upstroke_time_maps:
            out[f"UpstrokeTimeMap{self._hdf5_friendly(thr)}"] = self.native.cell_property_maps(
                90.0, thr, max_aps=self.max_paces)["upstroke_time"]
        for thr in hc.max_upstroke_velocity_maps:
            out[f"MaxUpstrokeVelocityMap{self._hdf5_friendly(thr)}"] = self.native.cell_property_maps(
                90.0, thr, max_aps=self.max_paces)["max_upstroke_velocity"]
        xyz = self.tissue.xyz
        for origin in hc.conduction_velocity_maps:
            dist = np.linalg.norm(xyz - xyz[origin], axis=1)
            out[f"ConductionVelocityFromNode{origin}"] = self.native.conduction_velocity_map(
                origin, dist, max_aps=self.max_paces)
        self.post_processing = out

    def GetOutput(self):
        """The printing-step output as Hdf5DataWriter writes it: Time, Data (time x node x
        variable) and the variable names, V first."""
        hc = HeartConfig.Instance()
        return dict(Time=self.native.output_times(), Data=self.native.output_frames(),
                    variables=["V"] + list(hc.output_variables))

    def GetPostProcessingMaps(self):
        return dict(self.post_processing)

    def WriteOutput(self, directory):
        """Time.npy and Data.npy (the HDF5 file's two datasets), and one .npy per
        post-processing map padded with -999 as PostProcessingWriter pads them (no HDF5
        library is linked, so the container is NumPy's)."""
        import os

        os.makedirs(directory, exist_ok=True)
        o = self.GetOutput()
        np.save(os.path.join(directory, "Time.npy"), o["Time"])
        np.save(os.path.join(directory, "Data.npy"), o["Data"])
        for name, rows in self.post_processing.items():
            width = max(len(r) for r in rows)
            arr = np.full((width, len(rows)), -999.0)   # pace x node, as the HDF5 map datasets
            for i, r in enumerate(rows):
                arr[:len(r), i] = r
            np.save(os.path.join(directory, name + ".npy"), arr)

    def GetSolution(self):
        return self.native.voltage()

    def AddOutputModifier(self, fn):
        self.output_modifiers.append(fn)

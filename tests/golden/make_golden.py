"""Extract Chaste's own golden vectors for the monodomain path into chaste_kats.json.

Run where the Chaste source tree is present, passing its root as the first
argument or in $CHASTE_SOURCE_DIR; the GPU tests and the benchmark only read the JSON.
Sources:
  heart/test/data/ionicmodels/Lr91DelayedStimValidData.dat   (TestIonicModels.hpp:406-467)
  heart/test/data/ionicmodels/Lr91RegularStimValidData.dat   (TestIonicModels.hpp:469-500)
  heart/test/data/ionicmodels/TenTusscherValidData.dat       (TestIonicModels.hpp:793-835)
  hard-coded values of heart/test/monodomain/TestMonodomainProblem.hpp
  (:166-218, :226-297, :303-340, :784-974) and TestIonicModels.hpp GetIIonic checks.
It also copies the Niederer et al. 2011 benchmark activation map Chaste checks in
heart/test/monodomain/TestNiederer2011BenchmarkSimulation.hpp:278-290
(heart/test/data/benchmark_data_orig/activation_time_h0.05_dt0.01.dat, one
activation time in ms per node of the h = 0.05 slab) into
niederer_activation_h0.05_dt0.01.txt.
"""
import json
import os
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CHASTE_SOURCE_DIR")
if not REF:
    sys.exit("usage: make_golden.py <chaste source root>  (or set CHASTE_SOURCE_DIR)")


def read_dat(rel):
    with open(os.path.join(REF, rel)) as f:
        header = f.readline().split()
        rows = [[float(x) for x in line.split()] for line in f if line.strip()]
    names = [h.split("(")[0] for h in header]
    return {n: [r[i] for r in rows] for i, n in enumerate(names)}


out = {
    "source": "Chaste heart/test (see make_golden.py docstring)",
    "lr91_delayed_stim": {
        "stimulus": {"kind": "simple", "magnitude": -25.5, "duration": 2.0, "start": 50.0},
        "dt": 0.01, "end": 1000.0, "sample_every_steps": 100, "tolerance": 1e-3,
        "V": read_dat("heart/test/data/ionicmodels/Lr91DelayedStimValidData.dat")["V"],
        "iionic_after_1000_plus_60ms": 1.9411, "iionic_tolerance": 1e-3,
    },
    "lr91_regular_stim": {
        "stimulus": {"kind": "regular", "magnitude": -25.5, "duration": 2.0, "period": 500.0,
                     "start": 50.0},
        "dt": 0.01, "end": 1000.0, "sample_every_steps": 100, "tolerance": 1e-3,
        "states": read_dat("heart/test/data/ionicmodels/Lr91RegularStimValidData.dat"),
    },
    "tt06_simple_stim": {
        "stimulus": {"kind": "simple", "magnitude": -38.0, "duration": 1.0, "start": 5.0},
        "dt": 0.001, "end": 40.0, "sample_every_steps": 1000, "tolerance": 1e-3,
        "states": read_dat("heart/test/data/ionicmodels/TenTusscherValidData.dat"),
        "iionic_at_end": -0.1843, "iionic_initial": 0.0012, "iionic_tolerance": 1e-3,
    },
    "cellprops_lr91_regular": {
        "source": "heart/test/postprocessing/TestCellProperties.hpp:195-245",
        "stimulus": {"kind": "regular", "magnitude": -80.0, "duration": 0.5, "period": 1000.0, "start": 100.0},
        "dt": 0.01, "end": 3450.0, "n_aps": 4,
        "last_complete_apd90": 362.0155, "last_peak": 43.1665, "last_resting": -84.4395,
        "tolerance_apd": 0.01, "tolerance_v": 1e-4,
    },
    "tissue": [
        {"name": "TestMonodomainProblem1D", "dim": 1, "h": 0.01, "size": [0.1, 0, 0],
         "sigma": 0.0005, "am": 1.0, "cm": 1.0, "stim": -600.0, "stim_duration": 0.5,
         "end": 2.0, "abs_tol": 2e-4, "nodes": [1, 3, 5, 7, 9, 10],
         "V": [20.7710232, 21.5319692, 22.9280817, 24.0611303, -0.770330519, -19.2234919],
         "tolerance": 5e-3},
        {"name": "TestMonodomainProblem1DWithRelativeTolerance", "dim": 1, "h": 0.01,
         "size": [0.1, 0, 0], "sigma": 0.0005, "am": 1.0, "cm": 1.0, "stim": -600.0,
         "stim_duration": 0.5, "end": 2.0, "rel_tol": 1e-9, "nodes": [1, 3, 5, 7, 9, 10],
         "V": [20.7710232, 21.5319692, 22.9280817, 24.0611303, -0.770330519, -19.2234919],
         "tolerance": 2e-5},
        {"name": "TestMonodomainProblemSimplestMesh1D", "dim": 1, "h": 1.0, "size": [1.0, 0, 0],
         "sigma": 0.0005, "am": 1.0, "cm": 10.0, "stim": -600.0, "stim_duration": 0.5,
         "end": 2.0, "abs_tol": 2e-4, "nodes": [0, 1], "V": [-52.1698, -83.8381],
         "tolerance": 5e-3},
        {"name": "TestMonodomainProblemCreates1DGeometry", "dim": 1, "h": 0.01,
         "size": [1.0, 0, 0], "sigma": 1.75, "am": 1400.0, "cm": 1.0, "stim": -3.0e6,
         "stim_duration": 0.5, "end": 5.0, "abs_tol": 2e-4, "nodes": [1, 3, 5, 7],
         "V": [13.9682, 13.9149, 13.8216, 13.7275], "tolerance": 5e-3},
        {"name": "TestMonodomainProblemCreates2DGeometry", "dim": 2, "h": 0.01,
         "size": [0.3, 0.3, 0], "sigma": 1.75, "am": 1400.0, "cm": 1.0, "stim": -3.0e6,
         "stim_duration": 0.5, "end": 4.0, "abs_tol": 2e-4, "nodes": [1, 3, 5, 7],
         "V": [17.5728, 17.4562, 17.2559, 17.0440], "tolerance": 5e-3},
        {"name": "TestMonodomainProblemCreates3DGeometry", "dim": 3, "h": 0.01,
         "size": [0.1, 0.1, 0.1], "sigma": 1.75, "am": 1400.0, "cm": 1.0, "stim": -3.0e6,
         "stim_duration": 0.5, "end": 2.0, "abs_tol": 2e-4, "nodes": [1, 3, 5, 7, 0, 665, 1330],
         "V": [31.8958, 32.1109, 32.7315, 33.7011, 31.8730, 32.6531, 34.5152],
         "tolerance": 5e-3,
         "midway": {"end": 1.0, "nodes": [0, 665, 1330], "V": [48.0637, 26.5404, -55.3058],
                    "tolerance": 1e-3}},
    ],
    # BidomainProblem<1> with PlaneStimulusCellFactory<LR91> (SimpleStimulus(-600, 0.5) at x = 0),
    # sigma_i = sigma_e = 0.0005, Am = Cm = 1, dt 0.01 ms, HeartConfig's default KSP tolerance
    # (absolute 2e-4); solution entries interleaved as (V_0, phi_0, V_1, phi_1, ...)
    "bidomain": [
        {"name": "TestSimpleBidomain1D", "source": "heart/test/bidomain/TestBidomainProblem.hpp:1006-1040",
         "h": 0.01, "size": 0.1, "sigma_i": 0.0005, "sigma_e": 0.0005, "am": 1.0, "cm": 1.0, "end": 2.0,
         "abs_tol": 2e-4, "fixed": [], "solution_index": [1, 2, 3, 5, 7, 9, 10],
         "solution": [-16.4861, 22.8117, -16.4893, -16.5617, -16.6761, -16.8344, 25.3148], "tolerance": 5e-3},
        {"name": "TestBidomainDg01DPinned", "source": "heart/test/bidomain/TestBidomainProblem.hpp:240-331",
         "h": 0.01, "size": 1.0, "sigma_i": 0.0005, "sigma_e": 0.0005, "am": 1.0, "cm": 1.0, "end": 1.0,
         "abs_tol": 2e-4, "fixed": [100], "voltage_nodes": [0, 1, 2, 3, 4, 5],
         "voltage": [31.0335, 28.9214, 20.0279, -3.92649, -57.9395, -79.7754], "tolerance": 7e-3,
         "rest_from_node": 51, "rest": -83.85, "rest_tolerance": 0.1},
        {"name": "TestCompareBidomainProblemWithMonodomain",
         "source": "heart/test/bidomain/TestBidomainProblem.hpp:475-556",
         "h": 0.01, "size": 1.0, "sigma_i": 0.0005, "sigma_e": 1.0, "am": 1.0, "cm": 1.0, "end": 1.0,
         "abs_tol": 2e-4, "fixed": [], "max_v_difference_from_monodomain": 0.4, "max_abs_phi_e": 0.06},
    ],
}
here = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(here, "chaste_kats.json"), "w") as f:
    json.dump(out, f, indent=1)
print("wrote chaste_kats.json")

with open(os.path.join(REF, "heart/test/data/benchmark_data_orig/activation_time_h0.05_dt0.01.dat")) as f:
    act = [float(x) for x in f.read().split()]
with open(os.path.join(here, "niederer_activation_h0.05_dt0.01.txt"), "w") as f:
    f.write("".join(f"{a!r}\n" for a in act))
print(f"wrote niederer_activation_h0.05_dt0.01.txt ({len(act)} nodes)")

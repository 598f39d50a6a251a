"""The reference's own GPU unit tests of this path (its tests/unit/*.cu),
compiled unchanged against this library and run on the GPU.

`make -C oracle reftests` builds each test file twice (FP64 and mixed
builds, as the reference builds them) plus its Morse, EAM and cell-list
device tests with the reference's deterministic-reduction switch: the path's GPU
headers come from the include-path shim (tests/dropin/include ->
include/tdmd_b200.hpp), the reference's core headers and CPU classes -- the
tests' expected values -- from its own tree (TDMD_B200_REFERENCE_CORE), and
GoogleTest's macros from tests/dropin/unit.  The binaries read their data directory from
TDMD_TEST_DATA_DIR, filled here from committed fixtures: the reference's
256-atom data file (tests/data/cu_fcc_256.data, from run0_morse_256.json),
its Mishin setfl and the LAMMPS run-0 force dumps of that system
(run0_morse_256.json, run0_eam_256.json).

Expected outcome, per test: OK, except
  * FastPipelineScheduler.KernelLaunchInvariant, which pins the reference's
    own launch count (1 + 2 per step + 1; this library's FastPipelineScheduler
    counts its cell-list and list-build launches too);
  * the determinism tests, skipped unless built with the reference's
    TDMD_DETERMINISTIC_REDUCE switch (mapped here onto the run-time switch);
  * PipelineScheduler.DeterministicMatchesM3, which the reference itself
    skips in its mixed build.
The TD zone PipelineScheduler tests (test_pipeline_scheduler.cu and the
NVT / adaptive-dt ones) run on the C++ layer's PipelineScheduler, which
steps all zones together on the whole-system path; the deterministic one
compares it with the reference's own sequential CPU loop.
"""
from __future__ import annotations

import os
import re
import subprocess

import numpy as np
import pytest

from conftest import golden, golden_file

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")

LAUNCH_INVARIANT = {"FastPipelineScheduler.KernelLaunchInvariant"}
SKIPPED_IN_MIXED = {"PipelineScheduler.DeterministicMatchesM3"}
DETERMINISM = {"DeviceMorseDeterminism.EnergyBitIdentical",
               "DeviceEamDeterminism.EnergyBitIdentical",
               "DeviceCellListDeterminism.TwoBuildsBitIdentical"}

CASES = {
    "test_device_buffer": {"DeviceBuffer.AllocAndCopyRoundTrip", "DeviceBuffer.ZeroFill",
                           "DeviceBuffer.MoveSemantics", "DeviceBuffer.Resize",
                           "DeviceSystemState.UploadDownloadRoundTrip",
                           "DeviceSystemState.ZeroForces"},
    "test_device_cell_list": {"DeviceCellList.EveryAtomInExactlyOneCell",
                              "DeviceCellList.MatchesCPUCellList",
                              "DeviceCellListDeterminism.TwoBuildsBitIdentical"},
    "test_device_neighbor_list": {"DeviceNeighborList.FullListSymmetry",
                                  "DeviceNeighborList.MatchesCPUHalfListPairCount"},
    "test_device_morse": {"DeviceMorse.MatchesCPUForces256Atoms",
                          "DeviceMorseDeterminism.EnergyBitIdentical"},
    "test_device_eam": {"DeviceEam.MatchesCPUForces256Atoms",
                        "DeviceEamDeterminism.EnergyBitIdentical"},
    "test_device_lammps_ab": {"DeviceLammpsAB.MorseRun0ForceMatch",
                              "DeviceLammpsAB.EamRun0ForceMatch"},
    "test_device_nve_drift": {"DeviceNVEDrift.Morse256Atoms50kSteps",
                              "DeviceNVEDrift.ADR0007AcceptanceTest100k",
                              "DeviceVelocityVerlet.FusedKickDriftMatchesUnfused"},
    "test_fast_pipeline": {"FastPipelineScheduler.NVEConservation",
                           "FastPipelineScheduler.LongNVEDrift",
                           "FastPipelineScheduler.KernelLaunchInvariant"},
    "test_fast_pipeline_eam": {"FastPipelineSchedulerEam.EamStepMatchesDirectCompute",
                               "FastPipelineSchedulerEam.EamNve100StepsStable",
                               "FastPipelineSchedulerEam.EamDeterministicReplay"},
    "test_nvt_thermostat": {"NVTThermostat.TemperatureConvergesToTarget",
                            "NVTThermostat.DeviceKEMatchesHost",
                            "NVTThermostat.DeterministicReproducibility",
                            "AdaptiveDt.DeviceVmaxMatchesHost", "AdaptiveDt.StableNVETrajectory"},
    "test_sum_order_sensitivity": {"SumOrderSensitivity.MorseEnergyBounded",
                                   "SumOrderSensitivity.EamEnergyBounded"},
    "test_pipeline_scheduler": {"PipelineScheduler.DeterministicMatchesM3",
                                "PipelineScheduler.PipelineNVEConservation",
                                "PipelineScheduler.ZoneTimeStepsAdvance"},
}

LINE = re.compile(r"^\[\s+(OK|FAILED|SKIPPED)\s+\] (\S+)$", re.M)


@pytest.fixture(scope="module")
def data_dir(tmp_path_factory):
    from tdmd_claude_b200 import io as TIO
    from tdmd_claude_b200 import workloads as W
    d = str(tmp_path_factory.mktemp("ref_unit_data"))
    g = golden("run0_morse_256.json")
    ge = golden("run0_eam_256.json")
    pos = np.array(g["positions"])
    n = len(pos)
    s = W.System(pos, np.zeros_like(pos), np.ones(n, np.int32), np.arange(1, n + 1, dtype=np.int32),
                 np.array(g["masses"]), tuple(g["lo"]), tuple(g["hi"]))
    TIO.write_lammps_data(os.path.join(d, "cu_fcc_256.data"), s)
    setfl = golden_file(ge["potential_file"], d)
    os.replace(setfl, os.path.join(d, "Cu_mishin1.eam.alloy"))
    # the LAMMPS run-0 dumps of the same system (verifylab/cases/run0-force-match)
    os.makedirs(os.path.join(d, "reference"))
    for name, fix in (("forces_morse.dump", g), ("forces_eam.dump", ge)):
        TIO.write_force_dump(os.path.join(d, "reference", name), s,
                             np.array(fix["lammps_forces"]), step=0)
    return d


def _run(binary, data_dir):
    exe = os.path.join(REF_DIR, binary)
    if not os.path.exists(exe):
        pytest.skip(f"{exe} not built (make -C oracle reftests needs the reference tree)")
    env = dict(os.environ, TDMD_TEST_DATA_DIR=data_dir)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=900, env=env)
    results = {name: status for status, name in LINE.findall(out.stdout)}
    return out, results


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", sorted(CASES))
def test_reference_unit_tests_run_unchanged(cuda, data_dir, case, precision):
    out, results = _run(f"reftest_{case}_{precision}", data_dir)
    assert set(results) == CASES[case], out.stdout[-3000:]
    for name, status in results.items():
        if name in LAUNCH_INVARIANT:
            want = "FAILED"
        elif name in DETERMINISM or (precision == "mixed" and name in SKIPPED_IN_MIXED):
            want = "SKIPPED"
        else:
            want = "OK"
        assert status == want, f"{name}: {status}\n{out.stdout[-3000:]}"


@pytest.mark.parametrize("case", ["test_device_morse", "test_device_eam", "test_device_cell_list"])
def test_reference_determinism_tests_in_their_deterministic_build(cuda, data_dir, case):
    """The reference's determinism tests, built with its
    TDMD_DETERMINISTIC_REDUCE switch (the library's ID-ordered mode turned on
    before main): two Morse or EAM compute calls give bit-identical
    energies, two cell-list builds bit-identical cells; the other tests of
    each file still pass in that build."""
    out, results = _run(f"reftest_{case}_fp64_det", data_dir)
    assert set(results) == CASES[case], out.stdout[-3000:]
    assert all(v == "OK" for v in results.values()), out.stdout[-3000:]

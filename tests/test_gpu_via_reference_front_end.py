"""The reference's own front end on the B200 path: its unit-test binary and its
CLI, compiled from the reference sources with nekwave_b200/ref_shim/dg_solver.cpp
in place of src/dg_solver.cpp (nekwave_b200/ref_shim/Makefile -> build/dropin/)."""
import csv
import json
import os
import subprocess

import pytest

from tests.gpu_helpers import record

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "build", "dropin")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(os.path.join(DROPIN, "nekwave-test")),
                                 reason="drop-in binaries not built")]


@pytest.mark.parametrize("name", ["MeshQuadratureTest", "ProbeScalingTest", "MaxwellStabilityTest",
                                  "PeriodicBCTest"])
def test_reference_unit_tests_on_nwb(gpu, name):
    r = subprocess.run([os.path.join(DROPIN, "nekwave-test"), name], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "1 passed, 0 failed" in r.stdout


def test_reference_cli_case_on_nwb(gpu, tmp_path):
    """nekwave <case.json>: PEC unit cube, 4^3 elements, 5 points, upwind, CFL 0.5,
    40 steps through Case::simulate (per-step download, host probes and energy)."""
    case = {"mesh": {"nelx": 4, "nely": 4, "nelz": 4, "xmin": 0.0, "xmax": 1.0, "ymin": 0.0,
                     "ymax": 1.0, "zmin": 0.0, "zmax": 1.0},
            "numerics": {"order": 5, "cfl": 0.5, "flux_type": "upwind"},
            "time": {"num_steps": 40},
            "output": {"output_frequency": 5, "output_dir": str(tmp_path / "out"),
                       "export_fields": False, "export_format": "csv"}}
    p = tmp_path / "case.json"
    p.write_text(json.dumps(case))
    r = subprocess.run([os.path.join(DROPIN, "nekwave"), str(p)], capture_output=True, text=True,
                       timeout=300, cwd=tmp_path)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    hist = tmp_path / "out" / "energy_history.csv"
    assert hist.exists(), r.stdout[-2000:]
    rows = list(csv.reader(open(hist)))
    energies = [float(x[-1]) for x in rows[1:]]
    assert len(energies) >= 8
    assert all(b <= a * (1 + 1e-12) for a, b in zip(energies, energies[1:]))  # upwind decays


REF_CLI = os.path.join(ROOT, "oracle", "_ref", "nekwave-ref")


@pytest.mark.skipif(not os.path.exists(REF_CLI), reason="reference CLI not built")
def test_reference_cli_end_to_end_against_dropin(gpu, tmp_path):
    """The same case through the reference's own CLI and CUDA path (oracle/_ref,
    built from its sources) and through the drop-in CLI on libnwb: the benchmark
    workload (periodic 32^3, 8 points, central), 50 steps of Case::simulate with its
    per-step download, host probes and energy.  The CLI has no way to choose an
    initial wave (the reference ignores wave_type in a case file), so the fields
    start at zero and the run times the full Case::simulate loop; the energy
    histories must agree.  Wall times are recorded (cli_e2e.json in the test output
    directory)."""
    import time
    case = {"mesh": {"nelx": 32, "nely": 32, "nelz": 32, "xmin": 0.0, "xmax": 1.0, "ymin": 0.0,
                     "ymax": 1.0, "zmin": 0.0, "zmax": 1.0, "periodic": "all"},
            "numerics": {"order": 8, "cfl": 0.5, "flux_type": "central"},
            "time": {"num_steps": 50},
            # snapshots every 25 steps: the devdiag Case writes them in the background
            "output": {"output_frequency": 10, "export_fields": True, "export_format": "hdf5",
                       "save_frequency": 25}}
    out = {}
    for name, exe in (("reference", REF_CLI), ("dropin", os.path.join(DROPIN, "nekwave"))):
        d = tmp_path / name
        d.mkdir()
        c = dict(case)
        c["output"] = dict(case["output"], output_dir=str(d / "out"))
        p = d / "case.json"
        p.write_text(json.dumps(c))
        t0 = time.perf_counter()
        r = subprocess.run([exe, str(p)], capture_output=True, text=True, timeout=900, cwd=d)
        wall = time.perf_counter() - t0
        assert r.returncode == 0, name + ": " + r.stdout[-2000:] + r.stderr[-2000:]
        rows = list(csv.reader(open(d / "out" / "energy_history.csv")))
        out[name] = dict(wall_s=wall, energies=[float(x[-1]) for x in rows[1:]])
    a, b = out["reference"]["energies"], out["dropin"]["energies"]
    assert len(a) == len(b) >= 5
    assert all(abs(x - y) <= 1e-10 * abs(x) for x, y in zip(a, b))
    record("cli_e2e.json", {"case": "periodic 32^3, 8 points, central, 50 steps, Case::simulate",
                            "reference_wall_s": out["reference"]["wall_s"],
                            "dropin_wall_s": out["dropin"]["wall_s"]})


PULSE_REF = os.path.join(ROOT, "oracle", "_ref", "pulse-case-ref")


@pytest.mark.skipif(not (os.path.exists(PULSE_REF) and
                         os.path.exists(os.path.join(DROPIN, "pulse-case-devdiag"))),
                    reason="pulse-case drivers not built")
def test_device_diagnostics_front_end_on_a_nonzero_wave(gpu, tmp_path):
    """The reference's Case::simulate on a seeded Gaussian pulse (the benchmark
    workload: periodic 32^3, 8 points, central, CFL 0.5), 50 steps, 4 probes,
    diagnostics every 10 steps, run three ways: the reference's own CUDA build,
    the drop-in on libnwb with the reference's per-step full download and host
    diagnostics, and the drop-in with the device-diagnostics Case (probe elements
    only per step, max|E|, max|H| and energy reduced on the device, full state at
    save steps through the background SnapshotWriter, and at the end).  The energy histories (step, time, max|E|, max|H|,
    energy) and probe histories agree to the 9 significant digits the front end
    prints; the simulate() wall times are recorded (cli_devdiag.json)."""
    from nekwave_b200.workloads import single_mesh
    spec = single_mesh("c2", 32, 0)
    comp, (amp, x0, y0, z0, sig) = 2, spec["pulses"][2]
    case = {"mesh": {"nelx": 32, "nely": 32, "nelz": 32, "xmin": 0.0, "xmax": 1.0, "ymin": 0.0,
                     "ymax": 1.0, "zmin": 0.0, "zmax": 1.0, "periodic": "all"},
            "numerics": {"order": 8, "cfl": 0.5, "flux_type": "central"},
            "time": {"num_steps": 50},
            "probes": [[0.31, 0.52, 0.47], [0.5, 0.5, 0.5], [0.77, 0.13, 0.9], [0.05, 0.95, 0.6]],
            # snapshots every 25 steps: the devdiag Case writes them in the background
            "output": {"output_frequency": 10, "export_fields": True, "export_format": "hdf5",
                       "save_frequency": 25}}
    runs = {"reference": PULSE_REF, "dropin": os.path.join(DROPIN, "pulse-case"),
            "devdiag": os.path.join(DROPIN, "pulse-case-devdiag")}
    out = {}
    for name, exe in runs.items():
        d = tmp_path / name
        d.mkdir()
        c = dict(case)
        c["output"] = dict(case["output"], output_dir=str(d / "out"))
        p = d / "case.json"
        p.write_text(json.dumps(c))
        r = subprocess.run([exe, str(p), str(comp), repr(x0), repr(y0), repr(z0), repr(sig)],
                           capture_output=True, text=True, timeout=240, cwd=d)
        assert r.returncode == 0, name + ": " + r.stdout[-2000:] + r.stderr[-2000:]
        sim = [ln for ln in r.stdout.splitlines() if ln.startswith("[pulse-case] simulate_s")]
        hist = [[float(v) for v in row] for row in list(csv.reader(open(d / "out" / "energy_history.csv")))[1:]]
        probes = [[float(v) for v in row] for row in list(csv.reader(open(d / "out" / "probe_history.csv")))[1:]]
        out[name] = dict(simulate_s=float(sim[0].split()[-1]), hist=hist, probes=probes)
    ref = out["reference"]
    assert len(ref["hist"]) == 6 and len(ref["probes"]) == 51
    assert ref["hist"][-1][2] > 0.1 and ref["hist"][-1][4] > 0  # a nonzero wave throughout
    for name in ("dropin", "devdiag"):
        for key in ("hist", "probes"):
            a, b = ref[key], out[name][key]
            assert len(a) == len(b), (name, key)
            scale = max(abs(v) for row in a for v in row[2:])
            for ra, rb in zip(a, b):
                assert ra[:2] == rb[:2], (name, key, ra[:2], rb[:2])
                for va, vb in zip(ra[2:], rb[2:]):
                    # printed to 9 digits; FP64 paths agree to ~1e-14 of the largest value
                    assert abs(va - vb) <= 2e-8 * abs(va) + 1e-12 * scale, (name, key, va, vb)
    record("cli_devdiag.json", {
        "case": "periodic 32^3, 8 points, central, seeded Gaussian Ez, 50 steps, 4 probes, "
                "diagnostics every 10 steps, Case::simulate",
        **{f"{k}_simulate_s": v["simulate_s"] for k, v in out.items()}})


SNAPSHOT_CHECK = os.path.join(DROPIN, "snapshot-check")


@pytest.mark.skipif(not os.path.exists(SNAPSHOT_CHECK), reason="snapshot-check not built")
@pytest.mark.parametrize("N,nel,steps,every", [(6, 6, 40, 5), (8, 4, 21, 1)])
def test_snapshot_writer_matches_synchronous_downloads(gpu, N, nel, steps, every):
    """The devdiag front end's background writer (nwb_dropin::SnapshotWriter): the
    states its jobs receive, with their steps and times, equal bit for bit the
    synchronous downloads the reference's Case::simulate makes at the same steps,
    also when every step is a save and the jobs lag the loop."""
    r = subprocess.run([SNAPSHOT_CHECK, str(N), str(nel), str(steps), str(every)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert f"saves {steps // every} / {steps // every}" in r.stdout and "equal" in r.stdout

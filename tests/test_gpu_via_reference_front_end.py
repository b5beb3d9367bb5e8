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
            # no field export: without HDF5 the reference's writer adds a text VTU file
            # of every saved state (about 3 GB at this size) to its binary archive
            "output": {"output_frequency": 10, "export_fields": False}}
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
    workload: periodic 32^3, 8 points, central, CFL 0.5), 100 steps, 4 probes,
    diagnostics every 10 steps, run three ways: the reference's own CUDA build,
    the drop-in on libnwb with the reference's per-step full download and host
    diagnostics, and the drop-in with the device-diagnostics Case (probe elements
    only per step, max|E|, max|H| and energy reduced on the device, the full state
    at the end).  The energy histories (step, time, max|E|, max|H|, energy) and probe
    histories agree to the 9 significant digits the front end prints; the simulate()
    wall times are recorded (cli_devdiag.json).  No fields are exported at this size:
    the saves, which the device-diagnostics Case moves onto its background writer,
    run in test_front_ends_write_the_same_snapshots."""
    from nekwave_b200.workloads import single_mesh
    spec = single_mesh("c2", 32, 0)
    comp, (amp, x0, y0, z0, sig) = 2, spec["pulses"][2]
    case = {"mesh": {"nelx": 32, "nely": 32, "nelz": 32, "xmin": 0.0, "xmax": 1.0, "ymin": 0.0,
                     "ymax": 1.0, "zmin": 0.0, "zmax": 1.0, "periodic": "all"},
            "numerics": {"order": 8, "cfl": 0.5, "flux_type": "central"},
            "time": {"num_steps": 100},
            "probes": [[0.31, 0.52, 0.47], [0.5, 0.5, 0.5], [0.77, 0.13, 0.9], [0.05, 0.95, 0.6]],
            # no field export at this size (a text VTU file of about 3 GB per saved
            # state without HDF5); the saves run in test_front_ends_write_the_same_snapshots
            "output": {"output_frequency": 10, "export_fields": False}}
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
    assert len(ref["hist"]) == 11 and len(ref["probes"]) == 101
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
        "case": "periodic 32^3, 8 points, central, seeded Gaussian Ez, 100 steps, 4 probes, "
                "diagnostics every 10 steps, Case::simulate",
        **{f"{k}_simulate_s": v["simulate_s"] for k, v in out.items()}})


def read_archive(path):
    """The binary archive the reference's field writer keeps when it is built without
    HDF5 (src/hdf5_writer.cpp:715-727, 1018-1048): a 16-byte magic, int32 N, nelt,
    npts, 0, the node coordinates, then per saved step int32 step, 0, the time and E
    and H as [npts][3] doubles, an int32 flag and (flag 1) the derived fields.
    Returns [(step, time, state [6*npts] in component-major order)]."""
    import numpy as np
    b = open(path, "rb").read()
    assert b[:14] == b"NEKWAVE_BIN_V2", path
    npts = int(np.frombuffer(b, np.int32, 1, 24)[0])
    off = 32 + 24 * npts
    out = []
    while off < len(b):
        step = int(np.frombuffer(b, np.int32, 1, off)[0])
        t = float(np.frombuffer(b, np.float64, 1, off + 8)[0])
        e = np.frombuffer(b, np.float64, 3 * npts, off + 16).reshape(npts, 3)
        h = np.frombuffer(b, np.float64, 3 * npts, off + 16 + 24 * npts).reshape(npts, 3)
        off += 16 + 48 * npts
        derived = int(np.frombuffer(b, np.int32, 1, off)[0])
        off += 4 + (64 * npts if derived else 0)
        out.append((step, t, np.concatenate([e.T.ravel(), h.T.ravel()])))
    assert off == len(b), path
    return out


@pytest.mark.skipif(not (os.path.exists(PULSE_REF) and
                         os.path.exists(os.path.join(DROPIN, "pulse-case-devdiag"))),
                    reason="pulse-case drivers not built")
def test_front_ends_write_the_same_snapshots(gpu, tmp_path):
    """Field export at the save steps through the three front ends of the test
    above, on a mesh small enough for the reference's text output (6^3 elements,
    5 points, periodic, central, a seeded Gaussian Ez, 30 steps, a save every 10):
    without HDF5 the reference's writer appends every saved state to
    out/fields.bin and writes out/fields_step_<step>.vtu.  The device-diagnostics
    Case, whose save block runs on the background SnapshotWriter with the state
    copied behind the queued steps, writes archives and VTU files equal byte for
    byte to those of the drop-in's synchronous per-step downloads, and both hold
    the reference CUDA build's states to the step-parity tolerance."""
    import filecmp

    from tests.gpu_helpers import rel_l2
    from nekwave_b200.workloads import single_mesh
    spec = single_mesh("c2", 32, 0)
    comp, (amp, x0, y0, z0, sig) = 2, spec["pulses"][2]
    case = {"mesh": {"nelx": 6, "nely": 6, "nelz": 6, "xmin": 0.0, "xmax": 1.0, "ymin": 0.0,
                     "ymax": 1.0, "zmin": 0.0, "zmax": 1.0, "periodic": "all"},
            "numerics": {"order": 5, "cfl": 0.5, "flux_type": "central"},
            "time": {"num_steps": 30},
            "output": {"output_frequency": 10, "export_fields": True, "export_format": "hdf5",
                       "save_frequency": 10}}
    runs = {"reference": PULSE_REF, "dropin": os.path.join(DROPIN, "pulse-case"),
            "devdiag": os.path.join(DROPIN, "pulse-case-devdiag")}
    snaps, outdir = {}, {}
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
        outdir[name] = d / "out"
        snaps[name] = read_archive(d / "out" / "fields.bin")
    saved = [0, 10, 20, 30]
    for name in runs:
        assert [s for s, _, _ in snaps[name]] == saved, (name, [s for s, _, _ in snaps[name]])
    for (sa, ta, ua), (sb, tb, ub) in zip(snaps["dropin"], snaps["devdiag"]):
        assert ta == tb and np_equal(ua, ub), (sa, ta, tb)
    for step in saved:
        vtu = f"fields_step_{step}.vtu"
        assert filecmp.cmp(outdir["dropin"] / vtu, outdir["devdiag"] / vtu, shallow=False), vtu
    assert filecmp.cmp(outdir["dropin"] / "fields.bin", outdir["devdiag"] / "fields.bin", shallow=False)
    for (sa, ta, ua), (sb, tb, ub) in zip(snaps["reference"], snaps["dropin"]):
        assert ta == tb, (sa, ta, tb)
        assert rel_l2(ub, ua) < 1e-10, (sa, rel_l2(ub, ua))
    assert rel_l2(snaps["reference"][-1][2], snaps["reference"][0][2]) > 1e-3  # the wave moved


def np_equal(a, b):
    import numpy as np
    return np.array_equal(a, b)


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

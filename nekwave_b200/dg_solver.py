"""DgSolver: the reference's solver interface (src/dg_solver.hpp:35-102) on libnwb.

    solver = DgSolver()
    solver.initialize(mesh, c0)           # DgSolver::initialize
    solver.uploadState(state, state.size) # DgSolver::uploadState
    solver.step(dt, t)                    # DgSolver::step (blocking, one step)
    solver.downloadState(state, state.size)
    solver.finalize()

Everything runs through the C ABI of include/nwb.h; there is no host fallback.
Beyond the reference interface it exposes ``steps`` (many steps, asynchronous),
``evalRhs`` and ``energy`` (device FP64 diagnostics).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import NWB_FP32_BULK, NWB_FP64, SolverInfo, check, dptr

StateVector = np.ndarray  # [Ex, Ey, Ez, Hx, Hy, Hz], each of length npts (src/dg_solver.hpp:14)

PRECISIONS = {"fp64": NWB_FP64, "fp32": NWB_FP32_BULK, "fp32_bulk": NWB_FP32_BULK}


class DgSolver:
    """GPU-resident DG-SEM Maxwell solver (src/dg_solver.hpp:35)."""

    def __init__(self, precision: str = "fp64"):
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        self._prec = PRECISIONS[precision]
        self._h = None
        self._npts = 0

    def initialize(self, mesh, c0: float, true_pmc: bool = False) -> bool:
        """Analyse the mesh and allocate the device state (DgSolver::initialize).
        true_pmc: PMC faces (bc 2) are PMC mirrors instead of the reference's PEC
        mirror (nwb_solver_create_ex, NWB_SOLVER_TRUE_PMC)."""
        self.finalize()
        L = _lib.lib()
        h = C.c_void_p()
        d = mesh.desc()
        flags = _lib.NWB_SOLVER_TRUE_PMC if true_pmc else 0
        check(L.nwb_solver_create_ex(C.byref(d), float(c0), self._prec, flags, C.byref(h)))
        self._h = h
        self._npts = mesh.getTotalPoints()
        self._mesh = mesh
        return True

    def initializeBox(self, N: int, nel, lo, hi, c0: float, periodic=(False, False, False)) -> bool:
        """Box mesh built inside the library (geometry of Mesh::createBoxMesh per
        element, no per-node host arrays), then as initialize()."""
        self.finalize()
        L = _lib.lib()
        h = C.c_void_p()
        mask = (1 if periodic[0] else 0) | (2 if periodic[1] else 0) | (4 if periodic[2] else 0)
        check(L.nwb_solver_create_box(int(N), int(nel[0]), int(nel[1]), int(nel[2]), float(lo[0]),
                                      float(hi[0]), float(lo[1]), float(hi[1]), float(lo[2]),
                                      float(hi[2]), mask, float(c0), self._prec, C.byref(h)))
        self._h = h
        self._npts = int(nel[0]) * int(nel[1]) * int(nel[2]) * int(N) ** 3
        self._mesh = None
        return True

    def initPulse(self, pulses) -> None:
        """Device-generated Gaussian initial state (box solvers): pulses[c] =
        (amp, x0, y0, z0, sigma) for component c of [Ex,Ey,Ez,Hx,Hy,Hz]."""
        q = np.ascontiguousarray(np.asarray(pulses, dtype=np.float64).reshape(30))
        check(_lib.lib().nwb_solver_init_pulse(self._need(), dptr(q)))

    def _need(self):
        if self._h is None:
            raise RuntimeError("DgSolver not initialized")
        return self._h

    def uploadState(self, hostState: np.ndarray, size: int | None = None) -> None:
        h = self._need()
        a = np.ascontiguousarray(hostState, dtype=np.float64)
        n = a.size if size is None else int(size)
        if n > a.size:
            raise ValueError("size larger than the host buffer")
        check(_lib.lib().nwb_upload_state(h, dptr(a), n))

    def downloadState(self, hostState: np.ndarray | None = None, size: int | None = None):
        h = self._need()
        out = np.empty(6 * self._npts) if hostState is None else hostState
        if out.dtype != np.float64 or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("host buffer must be a contiguous float64 array")
        n = out.size if size is None else int(size)
        if n > out.size:
            raise ValueError("size larger than the host buffer")
        check(_lib.lib().nwb_download_state(h, dptr(out), n))
        return out

    def step(self, dt: float, time: float = 0.0) -> None:
        """One LSRK45 step; returns when it has finished, as the reference does."""
        h = self._need()
        L = _lib.lib()
        check(L.nwb_step(h, float(dt), 1))
        check(L.nwb_sync(h))

    def steps(self, dt: float, nsteps: int, sync: bool = True) -> None:
        """nsteps LSRK45 steps, replayed from a CUDA graph."""
        h = self._need()
        L = _lib.lib()
        check(L.nwb_step(h, float(dt), int(nsteps)))
        if sync:
            check(L.nwb_sync(h))

    def evalRhs(self) -> np.ndarray:
        """M^{-1}(K u + F*) of the current state (the reference's d_rhs_)."""
        h = self._need()
        out = np.empty(6 * self._npts)
        check(_lib.lib().nwb_eval_rhs(h, dptr(out), out.size))
        return out

    def energy(self) -> float:
        """FP64 discrete energy 1/2 sum J w3 (|E|^2+|H|^2) (src/case.cpp:733-766)."""
        h = self._need()
        e = C.c_double()
        check(_lib.lib().nwb_energy(h, C.byref(e)))
        return e.value

    def maxNorms(self):
        """(max |E|, max |H|) over the nodes, on the device (Case::getMaxE/getMaxH,
        src/case.cpp:768-794), equal to the host loop bit for bit."""
        e, h = C.c_double(), C.c_double()
        check(_lib.lib().nwb_max_norms(self._need(), C.byref(e), C.byref(h)))
        return e.value, h.value

    def probeSetup(self, node_offset, weights) -> None:
        """Probes as ProbeManager holds them (src/probe.cpp:33-96): per probe the first
        node of its element (e*N^3) and its N^3 Lagrange weights."""
        off = np.ascontiguousarray(node_offset, dtype=np.int64).reshape(-1)
        w = np.ascontiguousarray(weights, dtype=np.float64).reshape(-1)
        if w.size != off.size * self.info()["N"] ** 3:
            raise ValueError("weights must hold N^3 values per probe")
        check(_lib.lib().nwb_probe_setup(self._need(), off.size,
                                         off.ctypes.data_as(C.POINTER(C.c_longlong)),
                                         w.ctypes.data_as(_lib._D)))
        self._nprobes = off.size

    def probesAt(self, mesh, points) -> None:
        """Probes at physical points of a box mesh, located and weighted as
        ProbeManager::init does (src/probe.cpp:33-96)."""
        from .pool import locate_probes
        pts = [tuple(p) for p in points]
        elems, w1d = locate_probes(mesh, pts)
        N = mesh.getN()
        w1d = w1d.reshape(len(pts), 3, N)
        # full tensor weights w[i + N (j + N k)] = wr[i] ws[j] wt[k]
        wfull = np.einsum("pk,pj,pi->pkji", w1d[:, 2], w1d[:, 1], w1d[:, 0]).reshape(len(pts), -1)
        self.probeSetup(elems.astype(np.int64) * N ** 3, wfull)

    def probeRead(self) -> np.ndarray:
        """ProbeManager::record on the device: [nprobes, 6] (Ex, Ey, Ez, Hx, Hy, Hz)."""
        out = np.empty(6 * getattr(self, "_nprobes", 0))
        check(_lib.lib().nwb_probe_read(self._need(), out.ctypes.data_as(_lib._D)))
        return out.reshape(-1, 6)

    def snapshotBegin(self, host: np.ndarray) -> None:
        """Start an asynchronous copy of the current state into host (6*npts doubles,
        C-contiguous; pinned memory lets it overlap later steps)."""
        if host.dtype != np.float64 or not host.flags["C_CONTIGUOUS"]:
            raise ValueError("host must be a C-contiguous float64 array")
        self._snap = host  # keep it alive until the copy lands
        check(_lib.lib().nwb_snapshot_begin(self._need(), host.ctypes.data_as(_lib._D), host.size))

    def snapshotWait(self) -> None:
        check(_lib.lib().nwb_snapshot_wait(self._need()))
        self._snap = None

    def uploadBegin(self, host: np.ndarray) -> None:
        """Start an asynchronous upload of host (6*npts doubles, C-contiguous; pinned
        memory lets it overlap the steps already queued): steps queued afterwards
        start from it.  host must stay unchanged until uploadWait."""
        if host.dtype != np.float64 or not host.flags["C_CONTIGUOUS"]:
            raise ValueError("host must be a C-contiguous float64 array")
        self._up = host  # keep it alive until the copy lands
        check(_lib.lib().nwb_upload_begin(self._need(), host.ctypes.data_as(_lib._D), host.size))

    def uploadWait(self) -> None:
        check(_lib.lib().nwb_upload_wait(self._need()))
        self._up = None

    def info(self) -> dict:
        h = self._need()
        i = SolverInfo()
        check(_lib.lib().nwb_solver_get_info(h, C.byref(i)))
        out = {k: getattr(i, k) for k, _ in SolverInfo._fields_}
        out["structured"] = tuple(i.structured)
        return out

    def launchCount(self) -> int:
        n = C.c_longlong()
        check(_lib.lib().nwb_solver_launch_count(self._need(), C.byref(n)))
        return n.value

    def setVariant(self, variant: int) -> None:
        check(_lib.lib().nwb_solver_set_variant(self._need(), int(variant)))

    def autotune(self, reps: int = 10):
        """Time every launch shape on this mesh, keep the fastest; returns
        (best variant, per-variant ms)."""
        n = self.info()["variant_count"]
        ms = (C.c_float * n)()
        best = C.c_int()
        check(_lib.lib().nwb_solver_autotune(self._need(), int(reps), C.byref(best), ms, n))
        return best.value, [float(x) for x in ms]

    def timeSteps(self, dt: float, nsteps: int, graph: bool = True) -> float:
        """Device time (ms) of nsteps steps, CUDA events on the solver's stream."""
        ms = C.c_float()
        check(_lib.lib().nwb_time_steps(self._need(), float(dt), int(nsteps), int(graph),
                                        C.byref(ms)))
        return ms.value

    def timeStageKernel(self, dt: float, nstages: int) -> float:
        """Average device time (ms) of one fused stage kernel over nstages launches."""
        ms = C.c_float()
        check(_lib.lib().nwb_time_stage_kernel(self._need(), float(dt), int(nstages),
                                               C.byref(ms)))
        return ms.value

    def deviceState(self):
        """(device pointer of the current state [6][stride], cudaStream_t handle)."""
        p = _lib._D()
        s = C.c_void_p()
        check(_lib.lib().nwb_solver_device_state(self._need(), C.byref(p), C.byref(s)))
        return C.cast(p, C.c_void_p).value, s.value

    def finalize(self) -> None:
        """Release device buffers and the stream (DgSolver::finalize)."""
        if self._h is not None:
            _lib.lib().nwb_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.finalize()
        except Exception:
            pass

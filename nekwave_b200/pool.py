"""CavityPool: many independent cavities resident on one GPU (nwb_pool_* in
include/nwb.h).  Admission by a fixed HBM budget, one persistent launch per LSRK
stage for all resident cavities, device-side energy history and probe traces.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import NWB_EBUSY, NwbError, check, dptr, iptr
from .dg_solver import PRECISIONS

FREE, ADDED, RUNNING, FINISHED = -1, 0, 1, 2


class PoolFull(RuntimeError):
    """nwb_pool_add refused the cavity: over the HBM budget or no free slot."""


def lagrange_weights(z: np.ndarray, xi: float) -> np.ndarray:
    """1-D Lagrange basis on GLL nodes z at xi (ProbeManager's evalLagrange1D,
    src/probe.cpp:11-30), including its exact-node shortcut."""
    N = z.size
    hit = np.nonzero(np.abs(xi - z) < 1e-12)[0]
    if hit.size:
        L = np.zeros(N)
        L[hit[0]] = 1.0
        return L
    L = np.ones(N)
    for i in range(N):
        for j in range(N):
            if i != j:
                L[i] *= (xi - z[j]) / (z[i] - z[j])
    return L


def locate_probes(mesh, points):
    """Element and tensor Lagrange weights of each probe point, following
    ProbeManager::init (src/probe.cpp:33-96): the first element whose
    axis-aligned box is nearest, reference coordinates clamped to [-1,1]."""
    box = getattr(mesh, "box", None)
    if box is None:
        raise ValueError("probes need a box mesh (Mesh.createBoxMesh)")
    nel, lo, hi = np.array(box["nel"]), np.array(box["lo"]), np.array(box["hi"])
    h = (hi - lo) / nel
    ex, ey, ez = np.meshgrid(np.arange(nel[0]), np.arange(nel[1]), np.arange(nel[2]), indexing="ij")
    # element order e = ex + nelx (ey + nely ez)
    ex = ex.transpose(2, 1, 0).ravel()
    ey = ey.transpose(2, 1, 0).ravel()
    ez = ez.transpose(2, 1, 0).ravel()
    x0 = np.stack([lo[0] + ex * h[0], lo[1] + ey * h[1], lo[2] + ez * h[2]], axis=1)
    x1 = x0 + h
    z = mesh.getGllZ()
    N = mesh.getN()
    elems, weights = [], []
    for p in points:
        p = np.asarray(p, dtype=np.float64)
        r = 2.0 * (p - x0) / (x1 - x0) - 1.0
        d = np.maximum(0.0, np.maximum(-1.0 - r, r - 1.0))
        e = int(np.argmin(np.sum(d * d, axis=1)))
        rc = np.clip(r[e], -1.0, 1.0)
        w = np.stack([lagrange_weights(z, rc[a]) for a in range(3)])
        elems.append(e)
        weights.append(w.reshape(3 * N))
    return np.array(elems, dtype=np.int32), np.array(weights, dtype=np.float64).reshape(-1)


def box_probes(N, nel, lo, hi, points):
    """ProbeManager::init (src/probe.cpp:33-96) on a box mesh given by its
    parameters, through libnwb's locator (nwb_box_probes, the one the pool uses):
    (element offsets e*N^3 [P], tensor weights [P, N^3])."""
    pts = np.ascontiguousarray(np.asarray(points, dtype=np.float64).reshape(-1, 3))
    P = pts.shape[0]
    elem = np.zeros(max(P, 1), np.int32)
    w1d = np.zeros(max(P, 1) * 3 * N)
    check(_lib.lib().nwb_box_probes(int(N), int(nel[0]), int(nel[1]), int(nel[2]), float(lo[0]),
                                    float(hi[0]), float(lo[1]), float(hi[1]), float(lo[2]),
                                    float(hi[2]), P, dptr(pts), iptr(elem), dptr(w1d)))
    w1d = w1d[:P * 3 * N].reshape(P, 3, N)
    # tensor weight of node i + N (j + N k): w_r[i] w_s[j] w_t[k] (src/probe.cpp order)
    w = (w1d[:, 0, None, None, :] * w1d[:, 1, None, :, None]) * w1d[:, 2, :, None, None]
    return elem[:P].astype(np.int64) * N ** 3, w.reshape(P, N ** 3)


class CavityPool:
    def __init__(self, hbm_budget_bytes: int, max_slots: int = 256, precision: str = "fp64"):
        self._h = C.c_void_p()
        check(_lib.lib().nwb_pool_create(int(hbm_budget_bytes), int(max_slots),
                                         PRECISIONS[precision], C.byref(self._h)))
        self.max_slots = int(max_slots)
        self._meta = {}

    def add(self, mesh, c0: float, dt: float, nsteps: int, probes=None, energy_every: int = 1) -> int:
        """Admit a cavity; raises PoolFull when the HBM budget or the slots are used up."""
        probes = [] if probes is None else list(probes)
        if probes:
            pe, pw = locate_probes(mesh, probes)
        else:
            pe, pw = np.zeros(1, np.int32), np.zeros(3 * mesh.getN())
        slot = C.c_int()
        d = mesh.desc()
        st = _lib.lib().nwb_pool_add(self._h, C.byref(d), float(c0), float(dt), int(nsteps),
                                     len(probes), iptr(pe), dptr(pw), int(energy_every),
                                     C.byref(slot))
        if st == NWB_EBUSY:
            raise PoolFull(_lib.lib().nwb_last_error().decode())
        check(st)
        self._meta[slot.value] = dict(npts=mesh.getTotalPoints(), nsteps=int(nsteps),
                                      nprobes=len(probes), mesh=mesh)
        return slot.value

    def add_box(self, N: int, nel, lo, hi, c0: float, dt: float, nsteps: int, periodic=(False,) * 3,
                probes=None, energy_every: int = 1) -> int:
        """Admit a box cavity whose geometry the library builds from the box
        parameters (no per-node host arrays); probes are physical points."""
        probes = [] if probes is None else list(probes)
        xyz = np.ascontiguousarray(np.array(probes, dtype=np.float64).reshape(-1)) if probes \
            else np.zeros(3)
        mask = (1 if periodic[0] else 0) | (2 if periodic[1] else 0) | (4 if periodic[2] else 0)
        slot = C.c_int()
        st = _lib.lib().nwb_pool_add_box(self._h, int(N), int(nel[0]), int(nel[1]), int(nel[2]),
                                         float(lo[0]), float(hi[0]), float(lo[1]), float(hi[1]),
                                         float(lo[2]), float(hi[2]), mask, float(c0), float(dt),
                                         int(nsteps), len(probes), dptr(xyz), int(energy_every),
                                         C.byref(slot))
        if st == NWB_EBUSY:
            raise PoolFull(_lib.lib().nwb_last_error().decode())
        check(st)
        npts = int(nel[0]) * int(nel[1]) * int(nel[2]) * int(N) ** 3
        self._meta[slot.value] = dict(npts=npts, nsteps=int(nsteps), nprobes=len(probes), mesh=None)
        return slot.value

    def init_pulse(self, slot: int, pulses) -> None:
        """Device-generated initial state: pulses[c] = (amp, x0, y0, z0, sigma) per
        component c of [Ex,Ey,Ez,Hx,Hy,Hz] (sigma <= 0: zero component)."""
        q = np.ascontiguousarray(np.asarray(pulses, dtype=np.float64).reshape(30))
        check(_lib.lib().nwb_pool_init_pulse(self._h, int(slot), dptr(q)))

    def upload(self, slot: int, state: np.ndarray) -> None:
        a = np.ascontiguousarray(state, dtype=np.float64)
        check(_lib.lib().nwb_pool_upload(self._h, int(slot), dptr(a), a.size))

    def step(self, nsteps: int = 1) -> None:
        check(_lib.lib().nwb_pool_step(self._h, int(nsteps)))

    def sync(self) -> None:
        check(_lib.lib().nwb_pool_sync(self._h))

    def query(self):
        """(status[max_slots], steps done[max_slots]); synchronises the pool."""
        st = np.zeros(self.max_slots, np.int32)
        dn = np.zeros(self.max_slots, np.int32)
        check(_lib.lib().nwb_pool_query(self._h, iptr(st), iptr(dn), self.max_slots))
        return st, dn

    def query_begin(self) -> None:
        """Queue a snapshot of every slot's status behind the work already queued
        (nwb_pool_query_begin); query_end() returns it."""
        check(_lib.lib().nwb_pool_query_begin(self._h))

    def query_end(self):
        """(status, steps done) as of the last query_begin(), waiting only for that
        snapshot: steps queued after it keep running."""
        st = np.zeros(self.max_slots, np.int32)
        dn = np.zeros(self.max_slots, np.int32)
        check(_lib.lib().nwb_pool_query_end(self._h, iptr(st), iptr(dn), self.max_slots))
        return st, dn

    def results_async(self, slot: int) -> dict:
        """Queue the copies of a finished slot's energy history and probe traces into
        pinned host buffers and return them at once; they hold the values once a
        later query_end() (or sync()) has returned.  The slot may be removed
        right away."""
        import torch  # pinned host buffers (plumbing)
        m = self._meta[slot]
        ne = m["nsteps"] + 1
        e = torch.empty(ne, dtype=torch.float64, pin_memory=True).numpy()
        p = torch.empty(ne * max(m["nprobes"], 1) * 6, dtype=torch.float64, pin_memory=True).numpy()
        check(_lib.lib().nwb_pool_results_async(self._h, int(slot), C.cast(None, _lib._D), dptr(e),
                                                dptr(p)))
        return {"energy": e, "probes": p[:ne * m["nprobes"] * 6].reshape(ne, m["nprobes"], 6)}

    def results(self, slot: int, state=True, energy=True, probes=True) -> dict:
        m = self._meta[slot]
        out = {}
        s = np.empty(6 * m["npts"]) if state else None
        e = np.empty(m["nsteps"] + 1) if energy else None
        p = np.empty((m["nsteps"] + 1) * max(m["nprobes"], 1) * 6) if probes else None
        null = C.cast(None, _lib._D)
        check(_lib.lib().nwb_pool_results(self._h, int(slot), dptr(s) if s is not None else null,
                                          dptr(e) if e is not None else null,
                                          dptr(p) if p is not None else null))
        if state:
            out["state"] = s
        if energy:
            out["energy"] = e
        if probes:
            out["probes"] = p[:(m["nsteps"] + 1) * m["nprobes"] * 6].reshape(
                m["nsteps"] + 1, m["nprobes"], 6)
        return out

    def remove(self, slot: int) -> None:
        check(_lib.lib().nwb_pool_remove(self._h, int(slot)))
        self._meta.pop(slot, None)

    def info(self) -> dict:
        used, budget = C.c_size_t(), C.c_size_t()
        n = C.c_int()
        launches = C.c_longlong()
        check(_lib.lib().nwb_pool_info(self._h, C.byref(used), C.byref(budget), C.byref(n),
                                       C.byref(launches)))
        return dict(used_bytes=used.value, budget_bytes=budget.value, slots_used=n.value,
                    launches=launches.value)

    def set_mode(self, mode: int) -> None:
        """0: one persistent launch per stage for all N; 1: one launch per N."""
        check(_lib.lib().nwb_pool_set_mode(self._h, int(mode)))

    def autotune(self, reps: int = 5):
        """Time both launch modes on the resident cavities, keep the faster;
        returns (mode, [ms mode 0, ms mode 1])."""
        best = C.c_int()
        ms = (C.c_float * 2)()
        check(_lib.lib().nwb_pool_autotune(self._h, int(reps), C.byref(best), ms))
        return best.value, [float(ms[0]), float(ms[1])]

    def time_steps(self, nsteps: int) -> float:
        ms = C.c_float()
        check(_lib.lib().nwb_pool_time_steps(self._h, int(nsteps), C.byref(ms)))
        return ms.value

    def close(self) -> None:
        if self._h:
            _lib.lib().nwb_pool_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


__all__ = ["CavityPool", "PoolFull", "locate_probes", "lagrange_weights", "NwbError",
           "FREE", "ADDED", "RUNNING", "FINISHED"]

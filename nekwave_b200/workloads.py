"""Seeded synthetic workloads of the benchmark configurations (no dataset exists
for this path; every input is generated from a seed with numpy PCG64).

  tm110_cube()        PEC unit cube, 4^3 elements, 5 points, TM110 mode
  periodic_pulse()    periodic [0,1]^3, 32^3 elements, 8 points, Gaussian Ez
  pec_cavity_pulse()  PEC [0,2]x[0,2]x[0,1], 64x64x32 elements, 6 points
  batch_instances()   256 PEC cavities, uneven sizes and orders
  serving_requests()  Poisson stream of cavity solves
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

CFL = 0.5


def rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def gll_nodes(N: int) -> np.ndarray:
    """GLL nodes on [-1,1] (the reference's Mesh::setupGLL Newton iteration)."""
    p = N - 1
    z = np.zeros(N)
    z[0], z[-1] = -1.0, 1.0

    def leg(n, x):
        if n == 0:
            return 1.0
        p0, p1 = 1.0, x
        for k in range(1, n):
            p0, p1 = p1, ((2 * k + 1) * x * p1 - k * p0) / (k + 1)
        return p1

    for i in range(1, N - 1):
        x = -math.cos(math.pi * i / p)
        for _ in range(20):
            L = leg(p, x)
            Ld = (p / (x * x - 1.0)) * (x * L - leg(p - 1, x))
            Ldd = (2.0 * x * Ld - p * (p + 1.0) * L) / (1.0 - x * x)
            d = Ld / Ldd
            x -= d
            if abs(d) < 1e-15:
                break
        z[i] = x
    return z


def box_dxmin(N: int, nel, lo, hi) -> float:
    """Smallest GLL node spacing of an axis-aligned box mesh."""
    z = gll_nodes(N)
    gap = float(np.min(np.diff(z))) / 2.0
    h = (np.asarray(hi, float) - np.asarray(lo, float)) / np.asarray(nel, float)
    return gap * float(np.min(h))


@dataclass
class Cavity:
    """One PEC (or periodic) box cavity with a Gaussian initial pulse."""
    N: int                       # GLL points per direction (order N-1)
    nel: tuple
    lo: tuple
    hi: tuple
    c0: float
    nsteps: int
    dt: float
    pulses: list                 # per component (amp, x0, y0, z0, sigma)
    periodic: tuple = (False, False, False)
    probes: list = field(default_factory=list)
    T: float = 0.0               # final time (serving requests)
    arrival: float = 0.0         # seconds after the start of the stream

    @property
    def npts(self):
        return self.nel[0] * self.nel[1] * self.nel[2] * self.N ** 3

    @property
    def dof_stages(self):
        return 6 * self.npts * 5 * self.nsteps


def _pulse_ez(r, lo, hi, sig):
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    c = lo + (hi - lo) * r.uniform(0.25, 0.75, 3)
    return [(0.0, 0, 0, 0, 0.0)] * 2 + [(1.0, c[0], c[1], c[2], sig)] + [(0.0, 0, 0, 0, 0.0)] * 3


def batch_instances(n=256, seed=0, steps=400):
    """256 independent PEC cavities: edges ~ U[0.5,2], elements per direction
    ~ U{2..12}, order ~ U{3..8} (4..9 points), Gaussian Ez centred in the middle
    half with sigma ~ U[0.05,0.15] x the shortest edge, upwind, CFL 0.5."""
    r = rng(seed)
    out = []
    for _ in range(n):
        edges = r.uniform(0.5, 2.0, 3)
        nel = tuple(int(x) for x in r.integers(2, 13, 3))
        N = int(r.integers(3, 9)) + 1
        lo, hi = (0.0, 0.0, 0.0), tuple(float(e) for e in edges)
        sig = float(r.uniform(0.05, 0.15) * edges.min())
        dt = CFL * box_dxmin(N, nel, lo, hi)
        out.append(Cavity(N, nel, lo, hi, 1.0, steps, dt, _pulse_ez(r, lo, hi, sig)))
    return out


def serving_requests(n, rate, seed=0, max_nel=48, max_order=8):
    """Poisson stream (rate requests/s) of PEC cavity solves sized as the batch
    instances but with up to max_nel elements per direction and order <= 8;
    each runs to a final time T ~ U[0.5,2] (dt = T / ceil(T / dt_cfl), so the last
    step lands on T) and returns 8 probe traces and its energy history."""
    r = rng(seed)
    t = 0.0
    out = []
    for _ in range(n):
        t += float(r.exponential(1.0 / rate))
        edges = r.uniform(0.5, 2.0, 3)
        nel = tuple(int(x) for x in r.integers(2, max_nel + 1, 3))
        N = int(r.integers(3, max_order + 1)) + 1
        lo, hi = (0.0, 0.0, 0.0), tuple(float(e) for e in edges)
        sig = float(r.uniform(0.05, 0.15) * edges.min())
        T = float(r.uniform(0.5, 2.0))
        dt_cfl = CFL * box_dxmin(N, nel, lo, hi)
        nsteps = max(1, math.ceil(T / dt_cfl))
        probes = [tuple(float(v) for v in np.asarray(lo) + (np.asarray(hi) - np.asarray(lo)) *
                        r.uniform(0.0, 1.0, 3)) for _ in range(8)]
        out.append(Cavity(N, nel, lo, hi, 1.0, nsteps, T / nsteps, _pulse_ez(r, lo, hi, sig),
                          probes=probes, T=T, arrival=t))
    return out


def cavity_state(c: Cavity, x, y, z):
    """Host initial state of a cavity on given node coordinates."""
    n = x.size
    u = np.zeros(6 * n)
    for comp, (a, x0, y0, z0, s) in enumerate(c.pulses):
        if s > 0:
            u[comp * n:(comp + 1) * n] = a * np.exp(-((x - x0) ** 2 + (y - y0) ** 2 + (z - z0) ** 2) / s ** 2)
    return u

"""Seeded synthetic workloads of the benchmark configurations (no dataset exists
for this path; every input is generated from a seed with numpy PCG64).

  single_mesh("c2")   periodic [0,1]^3, 32^3 elements, 8 points, central, Gaussian Ez
  single_mesh("c3")   PEC [0,2]x[0,2]x[0,1], 64x64x32 elements, 6 points, upwind,
                      Gaussians in Ex, Ey, Ez
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


def single_mesh(name="c2", nel=32, seed=0) -> dict:
    """Single-mesh workloads.  c2: periodic [0,1]^3, nel^3 elements (32: the
    headline), 8 points, central flux, Ez = exp(-|r-r0|^2/0.1^2) with r0 ~
    U[0.3,0.7]^3.  c3: PEC [0,2]x[0,2]x[0,1], 2nel x 2nel x nel elements (nel = 32:
    64x64x32), 6 points, upwind, Gaussians in Ex, Ey, Ez with independent centres
    in the middle half of each axis and sigma ~ U[0.05,0.15].  pulses[c] =
    (amp, x0, y0, z0, sigma) per component, as nwb_solver_init_pulse takes them."""
    r = rng(seed)
    if name == "c3":
        nel3 = (64, 64, 32) if nel == 32 else (2 * nel, 2 * nel, nel)
        lo, hi = (0.0, 0.0, 0.0), (2.0, 2.0, 1.0)
        pulses = []
        for c in range(6):
            if c < 3:
                ctr = np.array(lo) + (np.array(hi) - np.array(lo)) * r.uniform(0.25, 0.75, 3)
                pulses.append((1.0, ctr[0], ctr[1], ctr[2], float(r.uniform(0.05, 0.15))))
            else:
                pulses.append((0.0, 0, 0, 0, 0.0))
        return dict(workload="pec_cavity_64x64x32_N6_upwind" if nel == 32 else
                    f"pec_cavity_{nel3[0]}x{nel3[1]}x{nel3[2]}_N6_upwind", N=6, nel=nel3, lo=lo,
                    hi=hi, periodic=(False, False, False), c0=1.0, flux="upwind", pulses=pulses)
    if name != "c2":
        raise ValueError(f"unknown single-mesh workload {name!r}")
    r0 = r.uniform(0.3, 0.7, 3)
    pulses = [(0.0, 0, 0, 0, 0.0)] * 2 + [(1.0, r0[0], r0[1], r0[2], 0.1)] + [(0.0, 0, 0, 0, 0.0)] * 3
    return dict(workload="periodic_box_32x32x32_N8_central" if nel == 32 else
                f"periodic_box_{nel}^3_N8_central", N=8, nel=(nel,) * 3, lo=(0.0, 0.0, 0.0),
                hi=(1.0, 1.0, 1.0), periodic=(True, True, True), c0=0.0, flux="central",
                pulses=pulses)


def pulse_state(pulses, x, y, z):
    """Host state of per-component Gaussian pulses on given node coordinates (the
    function nwb_solver_init_pulse evaluates on the device)."""
    n = x.size
    u = np.zeros(6 * n)
    for comp, (a, x0, y0, z0, s) in enumerate(pulses):
        if s > 0:
            u[comp * n:(comp + 1) * n] = a * np.exp(-((x - x0) ** 2 + (y - y0) ** 2 + (z - z0) ** 2) / s ** 2)
    return u


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


def serving_requests(n, rate, seed=0, max_nel=48, max_order=8, t_scale=1.0):
    """Poisson stream (rate requests/s) of PEC cavity solves sized as the batch
    instances but with up to max_nel elements per direction and order <= 8;
    each runs to a final time T ~ U[0.5,2] (dt = T / ceil(T / dt_cfl), so the last
    step lands on T) and returns 8 probe traces and its energy history.
    t_scale < 1 shortens every final time by that factor (same sizes, orders,
    pulses and probes; fewer steps), for latency sweeps that must fit a time
    budget."""
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
        T = float(r.uniform(0.5, 2.0)) * t_scale
        dt_cfl = CFL * box_dxmin(N, nel, lo, hi)
        nsteps = max(1, math.ceil(T / dt_cfl))
        probes = [tuple(float(v) for v in np.asarray(lo) + (np.asarray(hi) - np.asarray(lo)) *
                        r.uniform(0.0, 1.0, 3)) for _ in range(8)]
        out.append(Cavity(N, nel, lo, hi, 1.0, nsteps, T / nsteps, _pulse_ez(r, lo, hi, sig),
                          probes=probes, T=T, arrival=t))
    return out


def cavity_state(c: Cavity, x, y, z):
    """Host initial state of a cavity on given node coordinates."""
    return pulse_state(c.pulses, x, y, z)

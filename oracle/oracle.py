"""ctypes front end of the oracle -- TEST INFRASTRUCTURE ONLY.

Loads the plain-C restatement (``oracle/liboracle.so``, built from nw_oracle.c)
and, when it has been built, the reference compiled from its own sources
(``oracle/_ref/libnwref_host.so``: the reference Mesh and its kernel bodies run
on the host; ``oracle/_ref/libnwref_cuda.so``: the reference DgSolver on the
GPU).  Only tests, the smoke check and the benchmark's CPU-baseline leg import
this module; the product never does.

Array conventions follow the reference (see nw_oracle.h): state SoA
``[Ex,Ey,Ez,Hx,Hy,Hz][npts]``, metrics ``met[9][npts]`` in the order
rx,sx,tx,ry,sy,ty,rz,sz,tz, face points flattened (element, face, q, p).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


def _dp(a):
    return a.ctypes.data_as(_D)


def _ip(a):
    return a.ctypes.data_as(_I)


_lib = None
_ref = None
_refgpu = None


def lib():
    """The restatement library; raises if it was not built (``make -C oracle``)."""
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle not built: {path} missing (run make -C oracle)")
        L = C.CDLL(path)
        L.nwo_box_mesh.restype = C.c_int
        L.nwo_box_mesh.argtypes = [C.c_int] * 4 + [C.c_double] * 6 + [C.c_int] * 3 + \
            [_D] * 5 + [_I] * 3 + [_D] * 4
        L.nwo_gll.argtypes = [C.c_int, _D, _D, _D, _D]
        L.nwo_hex_mesh.restype = C.c_int
        L.nwo_hex_mesh.argtypes = [C.c_int, C.c_int, _D, _I, _I, _I] + [_D] * 5 + [_I] * 3 + \
            [_D] * 4
        L.nwo_box_corners.restype = C.c_int
        L.nwo_box_corners.argtypes = [C.c_int] * 3 + [C.c_double] * 6 + [C.c_int] * 3 + \
            [_D, _I, _I, _I]
        L.nwo_dxmin.restype = C.c_double
        L.nwo_dxmin.argtypes = [C.c_int, C.c_int, _D, _D, _D]
        L.nwo_rhs.argtypes = [C.c_int, C.c_int, _D, _D, _D, _D, C.c_int, _I, _I, _I,
                              _D, _D, _D, _D, C.c_double, _D, _D]
        L.nwo_step.argtypes = [C.c_int, C.c_int, _D, _D, _D, _D, C.c_int, _I, _I, _I,
                               _D, _D, _D, _D, C.c_double, C.c_double, C.c_int, _D, _D]
        L.nwo_energy.restype = C.c_double
        L.nwo_energy.argtypes = [C.c_int, C.c_int, _D, _D, _D]
        L.nwo_lsrk45.argtypes = [_D, _D]
        L.nwo_set_true_pmc.argtypes = [C.c_int]
        L.nwo_threads.restype = C.c_int
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libnwref_host.so"))


def ref():
    """The reference's own Mesh + kernel bodies on the host (oracle/_ref)."""
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libnwref_host.so")
        if not os.path.exists(path):
            raise RuntimeError(f"reference host build missing: {path}")
        L = C.CDLL(path)
        _bind_mesh_api(L)
        L.nwref_rhs.argtypes = [C.c_int, C.c_int, _D, _D, _D, _D, C.c_int, _I, _I, _I,
                                _D, _D, _D, _D, C.c_double, _D, _D, C.c_int]
        L.nwref_step.argtypes = [C.c_int, C.c_int, _D, _D, _D, _D, C.c_int, _I, _I, _I,
                                 _D, _D, _D, _D, C.c_double, C.c_double, C.c_int, _D, _D,
                                 C.c_int]
        L.nwref_threads.restype = C.c_int
        L.nwref_set_threads.restype = C.c_int
        L.nwref_set_threads.argtypes = [C.c_int]
        L.nwref_probe_init.argtypes = [C.c_void_p, C.c_int, _D, C.POINTER(C.c_long), _D]
        _ref = L
    return _ref


def ref_probes(N, nel, lo, hi, points):
    """The reference's own ProbeManager::init (src/probe.cpp:33-96) on its own box
    Mesh: (element offsets [P], tensor weights [P, N^3])."""
    L = ref()
    h = L.nwref_mesh_box(N, nel[0], nel[1], nel[2], lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], 0, 0, 0)
    if not h:
        raise ValueError("reference createBoxMesh failed")
    try:
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        off = np.zeros(len(pts), dtype=np.int64)
        w = np.zeros((len(pts), N ** 3))
        L.nwref_probe_init(h, len(pts), _dp(pts), off.ctypes.data_as(C.POINTER(C.c_long)), _dp(w))
    finally:
        L.nwref_mesh_free(h)
    return off, w


def ref_gpu_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libnwref_cuda.so"))


def ref_gpu():
    """The reference's own DgSolver built for sm_100a (oracle/_ref)."""
    global _refgpu
    if _refgpu is None:
        path = os.path.join(HERE, "_ref", "libnwref_cuda.so")
        if not os.path.exists(path):
            raise RuntimeError(f"reference CUDA build missing: {path}")
        L = C.CDLL(path)
        _bind_mesh_api(L)
        L.nwref_gpu_create.restype = C.c_void_p
        L.nwref_gpu_create.argtypes = [C.c_void_p, C.c_double]
        L.nwref_gpu_upload.argtypes = [C.c_void_p, _D, C.c_size_t]
        L.nwref_gpu_download.argtypes = [C.c_void_p, _D, C.c_size_t]
        L.nwref_gpu_steps.restype = C.c_double
        L.nwref_gpu_steps.argtypes = [C.c_void_p, C.c_double, C.c_int]
        L.nwref_gpu_destroy.argtypes = [C.c_void_p]
        _refgpu = L
    return _refgpu


def _bind_mesh_api(L):
    L.nwref_mesh_box.restype = C.c_void_p
    L.nwref_mesh_box.argtypes = [C.c_int] * 4 + [C.c_double] * 6 + [C.c_int] * 3
    L.nwref_mesh_free.argtypes = [C.c_void_p]
    L.nwref_mesh_sizes.argtypes = [C.c_void_p] + [C.POINTER(C.c_long)] * 3
    L.nwref_mesh_dxmin.restype = C.c_double
    L.nwref_mesh_dxmin.argtypes = [C.c_void_p]
    L.nwref_mesh_export.argtypes = [C.c_void_p] + [_D] * 9 + [_I] * 3 + [_D] * 4
    L.nwref_mesh_coords.argtypes = [C.c_void_p, _D, _D, _D]


@dataclass
class MeshArrays:
    """The arrays DgSolver::initialize reads from Mesh (src/dg_solver.cpp:40-241)."""
    N: int
    nelt: int
    z: np.ndarray      # GLL nodes [N]
    w: np.ndarray      # GLL weights [N]
    D: np.ndarray      # [N*N] column-major
    w3: np.ndarray     # [N^3]
    x: np.ndarray
    y: np.ndarray
    zc: np.ndarray
    jac: np.ndarray    # [npts]
    met: np.ndarray    # [9, npts]
    vmin: np.ndarray   # [nfp] int32
    vplus: np.ndarray
    bc: np.ndarray
    nx: np.ndarray
    ny: np.ndarray
    nz: np.ndarray
    dA: np.ndarray

    @property
    def npts(self):
        return self.nelt * self.N ** 3

    @property
    def nfp(self):
        return int(self.vmin.shape[0])

    def geo_args(self):
        return (self.N, self.nelt, _dp(self.D), _dp(self.w3), _dp(self.jac), _dp(self.met),
                self.nfp, _ip(self.vmin), _ip(self.vplus), _ip(self.bc),
                _dp(self.nx), _dp(self.ny), _dp(self.nz), _dp(self.dA))


def gll(N):
    z = np.zeros(N); w = np.zeros(N); D = np.zeros(N * N); w3 = np.zeros(N ** 3)
    lib().nwo_gll(N, _dp(z), _dp(w), _dp(D), _dp(w3))
    return z, w, D, w3


def box_mesh(N, nel, lo=(-1.0, -1.0, -1.0), hi=(1.0, 1.0, 1.0), periodic=(False,) * 3):
    """Restated Mesh::createBoxMesh (+ setupFaceData + flattening)."""
    nelx, nely, nelz = nel
    nelt = nelx * nely * nelz
    npts = nelt * N ** 3
    nfp = 6 * N * N * nelt
    z, w, D, w3 = gll(N)
    x = np.zeros(npts); y = np.zeros(npts); zc = np.zeros(npts); jac = np.zeros(npts)
    met = np.zeros((9, npts))
    vmin = np.zeros(nfp, np.int32); vplus = np.zeros(nfp, np.int32); bc = np.zeros(nfp, np.int32)
    nx = np.zeros(nfp); ny = np.zeros(nfp); nz = np.zeros(nfp); dA = np.zeros(nfp)
    rc = lib().nwo_box_mesh(N, nelx, nely, nelz, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2],
                            int(periodic[0]), int(periodic[1]), int(periodic[2]),
                            _dp(x), _dp(y), _dp(zc), _dp(jac), _dp(met),
                            _ip(vmin), _ip(vplus), _ip(bc), _dp(nx), _dp(ny), _dp(nz), _dp(dA))
    if rc != 0:
        raise ValueError("bad box mesh arguments")
    return MeshArrays(N, nelt, z, w, D, w3, x, y, zc, jac, met, vmin, vplus, bc, nx, ny, nz, dA)


def box_corners(nel, lo=(-1.0, -1.0, -1.0), hi=(1.0, 1.0, 1.0), periodic=(False,) * 3):
    """Element corners [nelt,8,3] and face table (kind, nbr elem, nbr face) [nelt,6]
    of createBoxMesh (src/mesh.cpp:700-830)."""
    nelt = nel[0] * nel[1] * nel[2]
    corners = np.zeros((nelt, 8, 3))
    fk = np.zeros((nelt, 6), np.int32); fb = np.zeros((nelt, 6), np.int32)
    ff = np.zeros((nelt, 6), np.int32)
    lib().nwo_box_corners(nel[0], nel[1], nel[2], lo[0], hi[0], lo[1], hi[1], lo[2], hi[2],
                          int(periodic[0]), int(periodic[1]), int(periodic[2]),
                          _dp(corners), _ip(fk), _ip(fb), _ip(ff))
    return corners, fk, fb, ff


def hex_mesh(N, corners, fkind, fnb, fnf):
    """General hexahedral mesh from corners (restated computeMetricsFromCorners +
    setupFaceData + flattening)."""
    corners = np.ascontiguousarray(corners, dtype=np.float64)
    fkind = np.ascontiguousarray(fkind, dtype=np.int32)
    fnb = np.ascontiguousarray(fnb, dtype=np.int32)
    fnf = np.ascontiguousarray(fnf, dtype=np.int32)
    nelt = corners.shape[0]
    npts = nelt * N ** 3
    nfp = 6 * N * N * nelt
    z, w, D, w3 = gll(N)
    x = np.zeros(npts); y = np.zeros(npts); zc = np.zeros(npts); jac = np.zeros(npts)
    met = np.zeros((9, npts))
    vmin = np.zeros(nfp, np.int32); vplus = np.zeros(nfp, np.int32); bc = np.zeros(nfp, np.int32)
    nx = np.zeros(nfp); ny = np.zeros(nfp); nz = np.zeros(nfp); dA = np.zeros(nfp)
    rc = lib().nwo_hex_mesh(N, nelt, _dp(corners), _ip(fkind), _ip(fnb), _ip(fnf),
                            _dp(x), _dp(y), _dp(zc), _dp(jac), _dp(met),
                            _ip(vmin), _ip(vplus), _ip(bc), _dp(nx), _dp(ny), _dp(nz), _dp(dA))
    if rc != 0:
        raise ValueError("bad hex mesh arguments")
    return MeshArrays(N, nelt, z, w, D, w3, x, y, zc, jac, met, vmin, vplus, bc, nx, ny, nz, dA)


def warped_box_mesh(N, nel, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), periodic=(False,) * 3,
                    linear=None, warp=0.0):
    """Box mesh whose corners are mapped by x -> A x (parallelepiped elements, affine)
    and then moved by a smooth bump of amplitude ``warp`` that vanishes on the box
    boundary (trilinear elements)."""
    corners, fk, fb, ff = box_corners(nel, lo, hi, periodic)
    c = corners.copy()
    if warp:
        lo_a, hi_a = np.array(lo), np.array(hi)
        s = (c - lo_a) / (hi_a - lo_a)
        bump = np.prod(np.sin(np.pi * s), axis=-1)
        c = c + warp * bump[..., None] * np.array([1.0, -0.7, 0.4]) * (hi_a - lo_a)
    if linear is not None:
        c = c @ np.asarray(linear, dtype=np.float64).T
    return hex_mesh(N, c, fk, fb, ff)


def ref_box_mesh(N, nel, lo=(-1.0, -1.0, -1.0), hi=(1.0, 1.0, 1.0), periodic=(False,) * 3,
                 L=None):
    """The reference's own Mesh::createBoxMesh, arrays copied out."""
    L = L or ref()
    h = L.nwref_mesh_box(N, nel[0], nel[1], nel[2], lo[0], hi[0], lo[1], hi[1], lo[2], hi[2],
                         int(periodic[0]), int(periodic[1]), int(periodic[2]))
    if not h:
        raise ValueError("reference createBoxMesh failed")
    try:
        a, b, c = C.c_long(), C.c_long(), C.c_long()
        L.nwref_mesh_sizes(h, C.byref(a), C.byref(b), C.byref(c))
        nelt, npts, nfp = a.value, b.value, c.value
        arr = dict(z=np.zeros(N), w=np.zeros(N), D=np.zeros(N * N), w3=np.zeros(N ** 3),
                   x=np.zeros(npts), y=np.zeros(npts), zc=np.zeros(npts), jac=np.zeros(npts),
                   met=np.zeros((9, npts)), vmin=np.zeros(nfp, np.int32),
                   vplus=np.zeros(nfp, np.int32), bc=np.zeros(nfp, np.int32),
                   nx=np.zeros(nfp), ny=np.zeros(nfp), nz=np.zeros(nfp), dA=np.zeros(nfp))
        L.nwref_mesh_export(h, *[_dp(arr[k]) for k in ("z", "w", "D", "w3", "x", "y", "zc",
                                                        "jac", "met")],
                            _ip(arr["vmin"]), _ip(arr["vplus"]), _ip(arr["bc"]),
                            _dp(arr["nx"]), _dp(arr["ny"]), _dp(arr["nz"]), _dp(arr["dA"]))
        dxmin = L.nwref_mesh_dxmin(h)
    finally:
        L.nwref_mesh_free(h)
    m = MeshArrays(N, nelt, **arr)
    m.dxmin_ref = dxmin
    return m


def dxmin(m: MeshArrays) -> float:
    return lib().nwo_dxmin(m.N, m.nelt, _dp(m.x), _dp(m.y), _dp(m.zc))


def rhs(m: MeshArrays, c0: float, u: np.ndarray, true_pmc: bool = False) -> np.ndarray:
    """true_pmc: bc 2 points are PMC mirrors (not the reference's behaviour, which
    mirrors them as PEC; the checker of libnwb's NWB_SOLVER_TRUE_PMC)."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    out = np.zeros(6 * m.npts)
    lib().nwo_set_true_pmc(int(true_pmc))
    try:
        lib().nwo_rhs(*m.geo_args(), float(c0), _dp(u), _dp(out))
    finally:
        lib().nwo_set_true_pmc(0)
    return out


def step(m: MeshArrays, c0: float, dt: float, nsteps: int, u: np.ndarray, k=None,
         true_pmc: bool = False):
    """nsteps LSRK45 steps; returns (u, k) as new arrays."""
    u = np.array(u, dtype=np.float64, copy=True)
    k = np.zeros_like(u) if k is None else np.array(k, dtype=np.float64, copy=True)
    lib().nwo_set_true_pmc(int(true_pmc))
    try:
        lib().nwo_step(*m.geo_args(), float(c0), float(dt), int(nsteps), _dp(u), _dp(k))
    finally:
        lib().nwo_set_true_pmc(0)
    return u, k


def energy(m: MeshArrays, u: np.ndarray) -> float:
    u = np.ascontiguousarray(u, dtype=np.float64)
    return lib().nwo_energy(m.N, m.nelt, _dp(m.w), _dp(m.jac), _dp(u))


def lsrk45():
    a = np.zeros(5); b = np.zeros(5)
    lib().nwo_lsrk45(_dp(a), _dp(b))
    return a, b


def ref_rhs(m: MeshArrays, c0: float, u: np.ndarray, deterministic=True) -> np.ndarray:
    u = np.ascontiguousarray(u, dtype=np.float64)
    out = np.zeros(6 * m.npts)
    ref().nwref_rhs(*m.geo_args(), float(c0), _dp(u), _dp(out), int(deterministic))
    return out


def ref_step(m: MeshArrays, c0: float, dt: float, nsteps: int, u: np.ndarray, k=None,
             deterministic=True):
    u = np.array(u, dtype=np.float64, copy=True)
    k = np.zeros_like(u) if k is None else np.array(k, dtype=np.float64, copy=True)
    ref().nwref_step(*m.geo_args(), float(c0), float(dt), int(nsteps), _dp(u), _dp(k),
                     int(deterministic))
    return u, k


def threads() -> int:
    return lib().nwo_threads()

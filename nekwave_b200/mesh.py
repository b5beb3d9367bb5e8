"""Mesh input of the hot path, mirroring the reference's Mesh getters
(src/mesh.hpp:51-218) for what DgSolver::initialize consumes.

``Mesh(N).createBoxMesh(...)`` builds a structured box mesh in libnwb
(nwb_box_mesh_create, the counterpart of Mesh::createBoxMesh,
src/mesh.cpp:683-843).  ``Mesh.from_arrays`` wraps arrays produced elsewhere
(for example by the reference's own Mesh) in the same interface.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from ._lib import MeshDesc, check, dptr, iptr


class Mesh:
    """Hexahedral DG-SEM mesh with N GLL points per direction (src/mesh.hpp:51)."""

    def __init__(self, N: int = 3, numElements: int = 1):
        self._N = int(N)
        self._nelt = int(numElements)
        self._arrays = None
        self._dxmin = None

    # ---- construction ------------------------------------------------------------
    def createBoxMesh(self, nelx, nely, nelz, xmin=-1.0, xmax=1.0, ymin=-1.0, ymax=1.0,
                      zmin=-1.0, zmax=1.0, periodicX=False, periodicY=False,
                      periodicZ=False) -> bool:
        """Structured box mesh (Mesh::createBoxMesh, src/mesh.cpp:683-843)."""
        L = _lib.lib()
        h = C.c_void_p()
        mask = (1 if periodicX else 0) | (2 if periodicY else 0) | (4 if periodicZ else 0)
        check(L.nwb_box_mesh_create(self._N, int(nelx), int(nely), int(nelz), float(xmin),
                                    float(xmax), float(ymin), float(ymax), float(zmin),
                                    float(zmax), mask, C.byref(h)))
        try:
            d = MeshDesc()
            check(L.nwb_box_mesh_desc(h, C.byref(d)))
            N = self._N
            nelt = d.nelt
            npts = nelt * N ** 3
            nfp = 6 * N * N * nelt

            def grab(ptr, n, dtype=np.float64):
                return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)

            x, y, z = _lib._D(), _lib._D(), _lib._D()
            check(L.nwb_box_mesh_coords(h, C.byref(x), C.byref(y), C.byref(z)))
            gz, gw = _lib._D(), _lib._D()
            check(L.nwb_box_mesh_gll(h, C.byref(gz), C.byref(gw)))
            dx = C.c_double()
            check(L.nwb_box_mesh_dxmin(h, C.byref(dx)))
            a = dict(
                z=grab(gz, N), w=grab(gw, N), D=grab(d.D, N * N), w3=grab(d.w3, N ** 3),
                x=grab(x, npts), y=grab(y, npts), zc=grab(z, npts), jac=grab(d.jac, npts),
                met=np.stack([grab(d.met[c], npts) for c in range(9)]),
                vmin=grab(d.vol_idx_minus, nfp, np.int32),
                vplus=grab(d.vol_idx_plus, nfp, np.int32),
                bc=grab(d.bc_type, nfp, np.int32),
                nx=grab(d.nx, nfp), ny=grab(d.ny, nfp), nz=grab(d.nz, nfp), dA=grab(d.dA, nfp))
            self._dxmin = dx.value
        finally:
            L.nwb_box_mesh_destroy(h)
        self._nelt = nelt
        self._arrays = a
        self.box = dict(nel=(int(nelx), int(nely), int(nelz)),
                        lo=(float(xmin), float(ymin), float(zmin)),
                        hi=(float(xmax), float(ymax), float(zmax)),
                        periodic=(bool(periodicX), bool(periodicY), bool(periodicZ)))
        return True

    @classmethod
    def from_arrays(cls, N, nelt, *, z, w, D, w3, jac, met, vmin, vplus, bc, nx, ny, nz, dA,
                    x=None, y=None, zc=None, **_ignored):
        """Wrap mesh arrays in the reference's layout (see include/nwb.h)."""
        m = cls(N, nelt)
        f64 = lambda v: np.ascontiguousarray(v, dtype=np.float64)
        i32 = lambda v: np.ascontiguousarray(v, dtype=np.int32)
        m._arrays = dict(z=f64(z), w=f64(w), D=f64(D), w3=f64(w3), jac=f64(jac),
                         met=f64(np.asarray(met).reshape(9, -1)), vmin=i32(vmin),
                         vplus=i32(vplus), bc=i32(bc), nx=f64(nx), ny=f64(ny), nz=f64(nz),
                         dA=f64(dA),
                         x=None if x is None else f64(x), y=None if y is None else f64(y),
                         zc=None if zc is None else f64(zc))
        return m

    # ---- getters (src/mesh.hpp:86-152) -------------------------------------------
    def getN(self):
        return self._N

    def getNumPointsPerElement(self):
        return self._N ** 3

    def getNumElements(self):
        return self._nelt

    def getTotalPoints(self):
        return self._nelt * self._N ** 3

    def _a(self, k):
        if self._arrays is None:
            raise RuntimeError("mesh not built")
        return self._arrays[k]

    def getD(self):
        return self._a("D")

    def getW3(self):
        return self._a("w3")

    def getGllZ(self):
        return self._a("z")

    def getGllW(self):
        return self._a("w")

    def getJac(self):
        return self._a("jac")

    def getMetrics(self):
        """[9, npts]: rx, sx, tx, ry, sy, ty, rz, sz, tz."""
        return self._a("met")

    def getCoordX(self):
        return self._a("x")

    def getCoordY(self):
        return self._a("y")

    def getCoordZ(self):
        return self._a("zc")

    def getFaceArrays(self):
        """Flattened face data as DgSolver::initialize builds it (src/dg_solver.cpp:76-112)."""
        a = self._arrays
        return dict(vmin=a["vmin"], vplus=a["vplus"], bc=a["bc"], nx=a["nx"], ny=a["ny"],
                    nz=a["nz"], dA=a["dA"])

    def computeMinNodeDistance(self):
        """Mesh::computeMinNodeDistance (src/mesh.cpp:883-930)."""
        if self._dxmin is None:
            x, y, z = self.getCoordX(), self.getCoordY(), self.getCoordZ()
            N = self._N
            s = (self._nelt, N, N, N)
            best = math.inf
            xs, ys, zs = x.reshape(s), y.reshape(s), z.reshape(s)
            for ax in (3, 2, 1):  # i, j, k directions
                d2 = (np.diff(xs, axis=ax) ** 2 + np.diff(ys, axis=ax) ** 2 +
                      np.diff(zs, axis=ax) ** 2)
                best = min(best, float(d2.min()))
            self._dxmin = math.sqrt(best)
        return self._dxmin

    def computeAutomaticCFL(self, safetyFactor=0.4):
        """Mesh::computeAutomaticCFL (src/mesh.cpp:937-942)."""
        return (safetyFactor * 1.75) / math.sqrt(3.0)

    def computeAutomaticDt(self, waveSpeed=1.0, safetyFactor=0.4):
        return self.computeAutomaticCFL(safetyFactor) * self.computeMinNodeDistance() / waveSpeed

    # ---- C ABI view ----------------------------------------------------------------
    def desc(self) -> MeshDesc:
        """nwb_mesh_desc pointing at this mesh's arrays (valid while the mesh lives)."""
        a = self._arrays
        d = MeshDesc()
        d.N = self._N
        d.nelt = self._nelt
        d.D = dptr(a["D"])
        d.w3 = dptr(a["w3"])
        d.jac = dptr(a["jac"])
        for c in range(9):
            d.met[c] = dptr(a["met"][c])
        d.vol_idx_minus = iptr(a["vmin"])
        d.vol_idx_plus = iptr(a["vplus"])
        d.bc_type = iptr(a["bc"])
        d.nx = dptr(a["nx"])
        d.ny = dptr(a["ny"])
        d.nz = dptr(a["nz"])
        d.dA = dptr(a["dA"])
        return d

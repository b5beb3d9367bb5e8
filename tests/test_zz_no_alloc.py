"""nwb_energy_noalloc: the energy of a device-resident state for callers that
cannot allocate device memory (a server holding a fixed HBM budget, a host
framework whose allocator owns the device memory, a loop that cannot afford
cudaMalloc's implicit synchronisation).  It keeps its partial sums in a fixed
array in the library instead of allocating.

The GPU test compares it, through the C ABI, with nwb_energy (the allocating
entry point) on the same state, on two calls in a row, within the energy
tolerance of the other GPU tests (1e-13 relative).  This file is collected
last so that a run stopping at its first failure has run every other test."""
import ctypes as C

import numpy as np
import pytest

from nekwave_b200 import DgSolver, Mesh, _lib
from oracle import oracle as O

TOL = 1e-13


def test_noalloc_rejects_meshes_beyond_its_scratch():
    L = _lib.lib()
    dummy = C.cast(C.c_void_p(256), _lib._D)  # never dereferenced: rejected before any launch
    n = _lib.NWB_EINVAL
    too_many = 131072 + 1
    assert L.nwb_energy_noalloc(dummy, too_many * 8, 2, too_many, dummy, 0, dummy, dummy, None) == n
    assert b"NWB_ENERGY_NOALLOC_MAX_ELEMENTS" in L.nwb_last_error()
    assert L.nwb_energy_noalloc(None, 8, 2, 1, dummy, 0, dummy, dummy, None) == n


@pytest.mark.gpu
@pytest.mark.parametrize("N,nel", [(5, (4, 4, 4)), (4, (40, 40, 40))])
def test_noalloc_energy_matches_allocating_entry_point(N, nel):
    import torch
    assert torch.cuda.is_available()
    mesh = Mesh(N)
    mesh.createBoxMesh(*nel, 0.0, 1.0, 0.0, 2.0, 0.0, 1.0)
    s = DgSolver()
    s.initialize(mesh, 1.0)
    rng = np.random.Generator(np.random.PCG64(N))
    s.uploadState(rng.standard_normal(6 * mesh.getTotalPoints()))
    want = s.energy()
    d_state, stream = s.deviceState()
    info = s.info()
    jac = torch.from_numpy(mesh.getJac()).cuda()
    w3 = torch.from_numpy(mesh.getW3()).cuda()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    L = _lib.lib()
    nelt = mesh.getNumElements()
    for call in range(2):  # two calls in a row share the scratch array
        st = L.nwb_energy_noalloc(C.cast(C.c_void_p(d_state), _lib._D), info["stride"], N, nelt,
                                  C.cast(C.c_void_p(jac.data_ptr()), _lib._D), 1,
                                  C.cast(C.c_void_p(w3.data_ptr()), _lib._D),
                                  C.cast(C.c_void_p(out.data_ptr() + 8 * call), _lib._D),
                                  C.c_void_p(stream))
        assert st == _lib.NWB_OK, L.nwb_last_error()
    _lib.check(L.nwb_sync(s._h))
    got = out.cpu().numpy()
    for g in got:
        assert abs(g - want) <= TOL * abs(want), (g, want)
    s.finalize()


def _graded_box(N, nel):
    """Axis-aligned box mesh with graded spacing (x -> x^1.6 per axis): affine
    elements whose J differs from element to element."""
    corners, fk, fb, ff = O.box_corners(nel, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
    return O.hex_mesh(N, corners ** 1.6, fk, fb, ff)


def _call(L, d_state, stride, N, nelt, jac, per_node, w3, out_ptr, stream):
    return L.nwb_energy_noalloc(C.cast(C.c_void_p(d_state), _lib._D), stride, N, nelt,
                                C.cast(C.c_void_p(jac.data_ptr()), _lib._D), per_node,
                                C.cast(C.c_void_p(w3.data_ptr()), _lib._D),
                                C.cast(C.c_void_p(out_ptr), _lib._D), C.c_void_p(stream))


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["graded_per_element", "warped_per_node"])
def test_noalloc_energy_with_non_uniform_jacobians(kind):
    """J varies between elements (graded box, J given per element: jac_per_node = 0)
    or between nodes (trilinear warped box, J per node): a wrong element or node
    index would change the sum.  Checked against nwb_energy and the oracle's
    restatement of Case::computeTotalEnergy, on two calls in a row."""
    import torch
    from tests.gpu_helpers import solver_for
    assert torch.cuda.is_available()
    N = 5
    if kind == "graded_per_element":
        m = _graded_box(N, (5, 4, 3))
        jac_e = m.jac.reshape(m.nelt, -1)
        # constant within an element up to rounding, varying between elements
        assert np.allclose(jac_e, jac_e[:, :1], rtol=1e-12, atol=0)
        assert np.ptp(jac_e[:, 0]) > 0.5 * jac_e[:, 0].max()
        jac_host, per_node = np.ascontiguousarray(jac_e[:, 0]), 0
    else:
        m = O.warped_box_mesh(N, (4, 3, 3), warp=0.08)
        jac_e = m.jac.reshape(m.nelt, -1)
        assert np.max(np.ptp(jac_e, axis=1)) > 1e-3 * np.abs(jac_e).max()
        jac_host, per_node = m.jac, 1
    s = solver_for(m, 1.0)
    u = np.random.Generator(np.random.PCG64(7)).standard_normal(6 * m.npts)
    s.uploadState(u)
    want = s.energy()
    oracle = O.energy(m, u)
    assert abs(want - oracle) <= TOL * abs(oracle)
    d_state, stream = s.deviceState()
    stride = s.info()["stride"]
    jac = torch.from_numpy(jac_host).cuda()
    w3 = torch.from_numpy(m.w3).cuda()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    L = _lib.lib()
    for call in range(2):
        st = _call(L, d_state, stride, N, m.nelt, jac, per_node, w3, out.data_ptr() + 8 * call, stream)
        assert st == _lib.NWB_OK, L.nwb_last_error()
    _lib.check(L.nwb_sync(s._h))
    for g in out.cpu().numpy():
        assert abs(g - want) <= TOL * abs(want), (g, want)
    # a host pointer in place of a device one is refused before any launch
    host_w3 = np.ascontiguousarray(m.w3)
    st = L.nwb_energy_noalloc(C.cast(C.c_void_p(d_state), _lib._D), stride, N, m.nelt,
                              C.cast(C.c_void_p(jac.data_ptr()), _lib._D), per_node,
                              host_w3.ctypes.data_as(_lib._D),
                              C.cast(C.c_void_p(out.data_ptr()), _lib._D), C.c_void_p(stream))
    assert st == _lib.NWB_EINVAL and b"current device" in L.nwb_last_error()
    s.finalize()

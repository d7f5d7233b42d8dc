"""The HIP runtime memory shim: the hipMalloc / hipMemcpy / hipFree /
hipGetDeviceCount / hipSetDevice symbols SELF's Fortran memory layer binds
through hipfort (src/SELF_Memory.f90), served by the CUDA runtime."""
import ctypes

import numpy as np
import pytest

import self_b200 as S

H2D, D2H, D2D = 1, 2, 3


def test_device_count_is_reported_without_a_gpu():
    """GPUAvailable (src/SELF_Memory.f90:336-350) reads a count and a status:
    with no usable GPU the count is 0 and the status is not hipSuccess."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    n = ctypes.c_int(-1)
    rc = S.lib().hipGetDeviceCount(ctypes.byref(n))
    assert n.value == 0 and rc != 0


def test_invalid_arguments_are_rejected_on_the_host():
    L = S.lib()
    assert L.hipMalloc(None, 8) == 1
    assert L.hipGetDeviceCount(None) == 1
    assert L.hipMemcpy(None, None, 8, 7) == 1  # no such hipMemcpyKind


@pytest.mark.gpu
def test_alloc_copy_free_round_trip():
    """UpdateDevice / UpdateHost as SELF does them: hipMalloc, host -> device,
    device -> device, device -> host, hipFree; and the rank's GPU selection."""
    L = S.lib()
    n = ctypes.c_int(0)
    assert L.hipGetDeviceCount(ctypes.byref(n)) == 0 and n.value >= 1
    assert L.hipSetDevice(0) == 0
    assert L.hipSetDevice(n.value + 5) == 101  # hipErrorInvalidDevice
    a = np.arange(1000, dtype=np.float64) * 0.5 - 3.0
    b = np.zeros_like(a)
    d1, d2 = ctypes.c_void_p(), ctypes.c_void_p()
    assert L.hipMalloc(ctypes.byref(d1), a.nbytes) == 0 and d1.value
    assert L.hipMalloc(ctypes.byref(d2), a.nbytes) == 0 and d2.value
    host = lambda x: x.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    assert L.hipMemcpy(d1, host(a), a.nbytes, H2D) == 0
    assert L.hipMemcpy(d2, d1, a.nbytes, D2D) == 0
    assert L.hipMemcpy(host(b), d2, a.nbytes, D2H) == 0
    np.testing.assert_array_equal(a, b)
    z = ctypes.c_void_p(1)
    assert L.hipMalloc(ctypes.byref(z), 0) == 0 and not z.value
    assert L.hipFree(d1) == 0 and L.hipFree(d2) == 0
    assert L.hipFree(None) == 0


@pytest.mark.gpu
def test_engine_runs_on_shim_allocated_buffers():
    """A Fortran caller's sequence: hipMalloc the state, UpdateDevice, fused
    RK3 steps through the C ABI on the engine's default stream, UpdateHost:
    the result equals the same steps on the Python mirror's buffers."""
    import torch
    N, nx = 5, 6
    mesh = S.Mesh2D(nx, nx, periodic=(True, True), perturbation=0.05)
    interp = S.Lagrange(N)
    geo = S.SEMQuad(interp, mesh)
    ref = S.CompressibleIdealGas2D(mesh, geo)
    X, Y = geo.x[..., 0], geo.x[..., 1]
    rho = 1.0 + 0.1 * torch.sin(2 * np.pi * X) * torch.sin(2 * np.pi * Y)
    q = torch.stack([rho * 0.5, rho * 0.3, rho, 2.5 + 0.5 * rho * 0.34], dim=1)[:, :, 0].contiguous()
    ref.SetSolution(q)
    ref.ForwardStep(3, 1e-3)
    ref.Sync()
    L = S.lib()
    h = ctypes.c_void_p()
    S.check(L.selfgpu_model2d_create(ctypes.byref(h), S.MODEL_CIG, N, mesh.nElem, S.FP64, None))
    mats = [np.asfortranarray(m) for m in (interp.dgMatrix, interp.bMatrix, interp.qWeights)]
    S.check(L.selfgpu_model2d_set_interp(h, *[m.ctypes.data_as(ctypes.c_void_p) for m in mats]))
    si = np.asfortranarray(mesh.sideInfo)
    dp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    S.check(L.selfgpu_model2d_set_geometry(h, dp(geo.dsdx), dp(geo.J), dp(geo.nHat), dp(geo.nScale),
                                           dp(mesh.sideInfo_d), si.ctypes.data_as(ctypes.c_void_p)))
    host_q = S.to_host(q).copy(order="F")
    nbytes = host_q.nbytes
    d_q, d_g = ctypes.c_void_p(), ctypes.c_void_p()
    assert L.hipMalloc(ctypes.byref(d_q), nbytes) == 0
    assert L.hipMalloc(ctypes.byref(d_g), nbytes) == 0
    zero = np.zeros_like(host_q)
    assert L.hipMemcpy(d_g, zero.ctypes.data_as(ctypes.c_void_p), nbytes, H2D) == 0
    assert L.hipMemcpy(d_q, host_q.ctypes.data_as(ctypes.c_void_p), nbytes, H2D) == 0
    S.check(L.selfgpu_model2d_set_state(h, d_q, d_g))
    S.check(L.selfgpu_model2d_set_params(h, 1.0, 0.0, 1.4, 1.0))
    S.check(L.selfgpu_model2d_rk3(h, 1e-3, 3))
    out = np.zeros_like(host_q)
    assert L.hipMemcpy(out.ctypes.data_as(ctypes.c_void_p), d_q, nbytes, D2H) == 0
    S.check(L.selfgpu_model2d_sync(h))
    np.testing.assert_array_equal(out, S.to_host(ref.solution))
    S.check(L.selfgpu_model2d_destroy(h))
    assert L.hipFree(d_q) == 0 and L.hipFree(d_g) == 0

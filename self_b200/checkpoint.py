"""Checkpoint / pickup files (Write_Model2D / Read_Model2D,
src/SELF_Model2D.f90:861-1099) over the library's container API.

The reference writes HDF5; these files keep its dataset paths, Fortran-order
shapes and the degree attribute N in a plain binary container
(``selfgpu_ckpt_*``), so a pickup needs no HDF5 on the host.
"""
import ctypes

import numpy as np
import torch

from ._lib import SelfGpuError, check, lib

F64, I32, F32 = 1, 2, 3
_DT = {np.dtype(np.float64): F64, np.dtype(np.int32): I32, np.dtype(np.float32): F32,
       torch.float64: F64, torch.int32: I32, torch.float32: F32}
_NP = {F64: np.float64, I32: np.int32, F32: np.float32}


def time_stamp(t):
    """TimeStamp(t, 's') of src/SELF_SupportRoutines.f90:856-924: DDDDHHMMSSmmm."""
    buf = ctypes.create_string_buffer(14)
    check(lib().selfgpu_time_stamp(float(t), buf))
    return buf.value.decode()


class Checkpoint:
    """A checkpoint file opened for writing (mode "w") or reading (mode "r")."""

    def __init__(self, path, mode="r"):
        self.path, self.mode = str(path), mode
        self._h = ctypes.c_void_p()
        check(lib().selfgpu_ckpt_open(ctypes.byref(self._h), self.path.encode(), 1 if mode == "w" else 0))

    def close(self):
        if self._h:
            h, self._h = self._h, ctypes.c_void_p()
            check(lib().selfgpu_ckpt_close(h))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def put(self, name, value, shape=None):
        """Write an array.  Numpy arrays are written in their Fortran-order
        shape; device tensors (reversed-shape, contiguous) with shape =
        the Fortran-order dims (default: the tensor shape reversed)."""
        if isinstance(value, torch.Tensor):
            t = value.contiguous()
            dims = list(shape) if shape is not None else list(reversed(t.shape))
            ptr, dev, dt = t.data_ptr(), 1 if t.is_cuda else 0, _DT[t.dtype]
            keep = t
        else:
            a = np.asfortranarray(value)
            dims = list(a.shape) if shape is None else list(shape)
            ptr, dev, dt = a.ctypes.data, 0, _DT[a.dtype]
            keep = a
        d = (ctypes.c_longlong * len(dims))(*dims)
        if dev:
            torch.cuda.synchronize()
        check(lib().selfgpu_ckpt_put(self._h, name.encode(), ctypes.c_void_p(ptr), dt, len(dims), d, dev))
        del keep

    def attr(self, name, value=None):
        if value is not None:
            check(lib().selfgpu_ckpt_put_attr(self._h, name.encode(), float(value)))
            return value
        out = ctypes.c_double()
        check(lib().selfgpu_ckpt_get_attr(self._h, name.encode(), ctypes.byref(out)))
        return out.value

    def info(self, name):
        dt, nd = ctypes.c_int(), ctypes.c_int()
        dims = (ctypes.c_longlong * 8)()
        check(lib().selfgpu_ckpt_info(self._h, name.encode(), ctypes.byref(dt), ctypes.byref(nd), dims))
        return dt.value, [dims[k] for k in range(nd.value)]

    def get(self, name, elem_offset=0, n_elem=None):
        """Host numpy array in Fortran order; with n_elem, the element slab
        [elem_offset, elem_offset + n_elem) of the last dimension."""
        dt, dims = self.info(name)
        if n_elem is not None:
            dims = dims[:-1] + [n_elem]
        out = np.zeros(dims, dtype=_NP[dt], order="F")
        check(lib().selfgpu_ckpt_get(self._h, name.encode(), ctypes.c_void_p(out.ctypes.data), out.nbytes,
                                     int(elem_offset), -1 if n_elem is None else int(n_elem), 0))
        return out

    def get_into(self, name, tensor, elem_offset=0, n_elem=None):
        """Read into a contiguous device tensor (element slab as in get)."""
        torch.cuda.synchronize()
        check(lib().selfgpu_ckpt_get(self._h, name.encode(), ctypes.c_void_p(tensor.data_ptr()),
                                     tensor.numel() * tensor.element_size(), int(elem_offset),
                                     -1 if n_elem is None else int(n_elem), 1))
        return tensor


def write_model(model, fileName=None):
    """Write_Model2D: quadrature, solution (interior and boundary), mesh
    coordinates (interior and boundary), attribute N; the fused engine keeps no
    flux or fluxDivergence arrays, so /state/interior/dSdt (the tendency of the
    written state) stands in for them."""
    from . import api as A
    if fileName is None:
        fileName = f"solution.{time_stamp(model.t)}.ckpt"
    L, geo = model.interp, model.geometry
    P, nVar, nEl = model.N + 1, model.nVar, model.nElem
    xb = torch.zeros((nEl, 4, 1, P, 2), device="cuda", dtype=torch.float64)
    lib().VectorBoundaryInterp_2D_gpu_wrapper(A.pp(L.device("bMatrix").data_ptr()), A.pp(geo.x.data_ptr()),
                                              A.pp(xb.data_ptr()), model.N, 1, nEl)
    with Checkpoint(fileName, "w") as c:
        c.attr("N", model.N)
        c.attr("nVar", nVar)
        c.attr("nElem", nEl)
        c.attr("time", model.t)
        c.put("/quadrature/xi", L.controlPoints)
        c.put("/quadrature/weights", L.qWeights)
        c.put("/quadrature/dgmatrix", L.dgMatrix)
        c.put("/quadrature/dmatrix", L.dMatrix)
        c.put("/quadrature/bmatrix", L.bMatrix)
        c.put("/state/interior/solution", model.solution, (P, P, nVar, nEl))
        c.put("/state/boundary/solution", model._bnd_interp(model.solution, nVar), (P, nVar, 4, nEl))
        c.put("/state/interior/dSdt", model.CalculateTendency(), (P, P, nVar, nEl))
        c.put("/mesh/interior/x", geo.x, (2, P, P, 1, nEl))
        c.put("/mesh/boundary/x", xb, (2, P, 1, 4, nEl))
    return fileName


def read_model(model, fileName, firstElem=0):
    """Read_Model2D: check the degree attribute N, read the solution interior
    (the slab of elements firstElem.. of a decomposed run) and upload it."""
    with Checkpoint(fileName, "r") as c:
        N = int(c.attr("N"))
        if N != model.N:
            raise SelfGpuError(1, "Solution polynomial degree does not match input file")
        _, dims = c.info("/state/interior/solution")
        if dims[:3] != [model.N + 1, model.N + 1, model.nVar]:
            raise SelfGpuError(1, "checkpoint solution shape does not match the model")
        c.get_into("/state/interior/solution", model.solution, firstElem, model.nElem)
        try:
            model.t = c.attr("time")
        except SelfGpuError:
            pass
    check(lib().selfgpu_model2d_invalidate(model._h))
    return model

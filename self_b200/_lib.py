"""Loader for libselfgpu.so, the CUDA engine's C ABI.

The library is built in-tree by ``self_b200.build``.  Loading fails loudly when
it is missing: there is no CPU fallback for any operation of this package.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libselfgpu.so")

_lib = None

c_int, c_double, c_void_p, c_char_p, c_longlong = (ctypes.c_int, ctypes.c_double, ctypes.c_void_p,
                                                   ctypes.c_char_p, ctypes.c_longlong)
PP = ctypes.POINTER(ctypes.c_void_p)  # real** / int** of the drop-in wrappers

# Exported symbols and their argument types.  Pointer arguments of the fused
# entry points are plain addresses (c_void_p); the drop-in wrappers take the
# address of a variable holding a device pointer (PP), as SELF's Fortran does.
_SIGS = {
    # host set-up
    "selfgpu_last_error": (c_char_p, []),
    "selfgpu_legendre_quadrature": (c_int, [c_int, c_int, c_void_p, c_void_p]),
    "selfgpu_lagrange_init": (c_int, [c_int, c_int, c_int, c_int] + [c_void_p] * 8),
    "selfgpu_mesh2d_structured": (c_int, [c_int, c_int, c_double, c_double, c_double, c_double, c_int, c_int,
                                          c_double, c_int, c_void_p, c_void_p, c_void_p, c_void_p]),
    "selfgpu_validate_side_info": (c_int, [c_void_p, c_int]),
    "selfgpu_semquad_generate": (c_int, [c_int, c_int] + [c_void_p] * 13),
    # fused engine
    "selfgpu_model2d_create": (c_int, [ctypes.POINTER(c_void_p), c_int, c_int, c_int, c_int, c_void_p]),
    "selfgpu_model2d_destroy": (c_int, [c_void_p]),
    "selfgpu_model2d_set_interp": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "selfgpu_model2d_set_geometry": (c_int, [c_void_p] + [c_void_p] * 6),
    "selfgpu_model2d_set_state": (c_int, [c_void_p, c_void_p, c_void_p]),
    "selfgpu_model2d_set_field": (c_int, [c_void_p, c_char_p, c_void_p]),
    "selfgpu_model2d_set_params": (c_int, [c_void_p, c_double, c_double, c_double, c_double]),
    "selfgpu_model2d_invalidate": (c_int, [c_void_p]),
    "selfgpu_model2d_tendency": (c_int, [c_void_p, c_void_p]),
    "selfgpu_model2d_rk3": (c_int, [c_void_p, c_double, c_int]),
    "selfgpu_model2d_sync": (c_int, [c_void_p]),
    "selfgpu_model2d_check_finite": (c_int, [c_void_p]),
    "selfgpu_model2d_entropy": (c_int, [c_void_p, ctypes.POINTER(c_double)]),
    "selfgpu_integral_mapped_scalar2d": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p, c_int, c_int,
                                                 ctypes.POINTER(c_double), c_void_p]),
    "selfgpu_model2d_launch_count": (c_longlong, [c_void_p]),
    "selfgpu_model2d_persistent_launch_count": (c_longlong, [c_void_p]),
    "selfgpu_model2d_set_kernel": (c_int, [c_void_p, c_int]),
    "selfgpu_model2d_set_multistep": (c_int, [c_void_p, c_int]),
    "selfgpu_model2d_autotune": (c_int, [c_void_p, ctypes.POINTER(c_int), ctypes.POINTER(c_int),
                                         ctypes.POINTER(ctypes.c_float)]),
    "selfgpu_model2d_set_launch": (c_int, [c_void_p, c_int, c_int]),
    "selfgpu_model2d_set_multistage": (c_int, [c_void_p, c_int]),
    "selfgpu_ensemble_create": (c_int, [c_void_p, c_int, c_void_p, c_void_p]),
    "selfgpu_ensemble_rk3": (c_int, [c_void_p, c_double, c_int]),
    "selfgpu_ensemble_destroy": (c_int, [c_void_p]),
    "selfgpu_model2d_set_wait_limit": (c_int, [c_void_p, c_longlong]),
    "selfgpu_model2d_inject_stall": (c_int, [c_void_p, c_int]),
    "selfgpu_cig2d_tendency_noalloc": (c_int, [c_void_p] * 11 + [c_double, c_int, c_int, c_void_p]),
    "selfgpu_model2d_set_closure": (c_int, [c_void_p, c_int, c_double, c_double, c_double, c_void_p]),
    "selfgpu_model2d_set_mlp": (c_int, [c_void_p, c_void_p, c_void_p]),
    "selfgpu_model2d_closure_state": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int]),
    "selfgpu_modal_matrix": (c_int, [c_int, c_void_p, c_void_p, c_void_p]),
    "selfgpu_cig2d_closure_features": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p, c_double, c_double,
                                               c_void_p, c_void_p, c_void_p]),
    "selfgpu_mlp_train": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, ctypes.c_float, ctypes.c_ulonglong,
                                  c_void_p, c_void_p, c_void_p]),
    "selfgpu_mlp_infer": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p]),
    "selfgpu_ckpt_open": (c_int, [ctypes.POINTER(c_void_p), ctypes.c_char_p, c_int]),
    "selfgpu_ckpt_put": (c_int, [c_void_p, ctypes.c_char_p, c_void_p, c_int, c_int, c_void_p, c_int]),
    "selfgpu_ckpt_put_attr": (c_int, [c_void_p, ctypes.c_char_p, c_double]),
    "selfgpu_ckpt_info": (c_int, [c_void_p, ctypes.c_char_p, ctypes.POINTER(c_int), ctypes.POINTER(c_int), c_void_p]),
    "selfgpu_ckpt_get": (c_int, [c_void_p, ctypes.c_char_p, c_void_p, c_longlong, c_longlong, c_longlong, c_int]),
    "selfgpu_ckpt_get_attr": (c_int, [c_void_p, ctypes.c_char_p, ctypes.POINTER(c_double)]),
    "selfgpu_ckpt_close": (c_int, [c_void_p]),
    "selfgpu_time_stamp": (c_int, [c_double, ctypes.c_char_p]),
    "selfgpu_domain_decomp": (c_int, [c_int, c_int, c_void_p]),
    "selfgpu_elem_to_rank": (c_int, [c_int, c_void_p, c_int, ctypes.POINTER(c_int)]),
    "selfgpu_halo_plan": (c_int, [c_void_p, c_int, c_int, c_void_p, c_int, c_void_p, ctypes.POINTER(c_int), c_void_p,
                                  c_void_p, c_void_p]),
    "selfgpu_model2d_set_halo": (c_int, [c_void_p, c_int]),
    "selfgpu_model2d_prologue": (c_int, [c_void_p]),
    "selfgpu_model2d_stage": (c_int, [c_void_p, c_double, c_int]),
    "selfgpu_model2d_caches": (c_int, [c_void_p, ctypes.POINTER(c_void_p), ctypes.POINTER(c_int),
                                       ctypes.POINTER(c_void_p), ctypes.POINTER(c_int)]),
    "selfgpu_pack_blocks": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p]),
    "selfgpu_unpack_blocks": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p]),
    # HIP runtime memory shim (hipfort's bind(c) targets)
    "hipMalloc": (c_int, [ctypes.POINTER(c_void_p), ctypes.c_size_t]),
    "hipFree": (c_int, [c_void_p]),
    "hipMemcpy": (c_int, [c_void_p, c_void_p, ctypes.c_size_t, c_int]),
    "hipGetDeviceCount": (c_int, [ctypes.POINTER(c_int)]),
    "hipSetDevice": (c_int, [c_int]),
    # drop-in wrappers (src/hip/*.cpp, src/models/hip/*.cpp of the reference)
    "ScalarGridInterp_2D_gpu_wrapper": (None, [PP, PP, PP, c_int, c_int, c_int, c_int]),
    "VectorGridInterp_2D_gpu_wrapper": (None, [PP, PP, PP, c_int, c_int, c_int, c_int]),
    "ScalarBoundaryInterp_2D_gpu_wrapper": (None, [PP, PP, PP, c_int, c_int, c_int]),
    "VectorBoundaryInterp_2D_gpu_wrapper": (None, [PP, PP, PP, c_int, c_int, c_int]),
    "TensorBoundaryInterp_2D_gpu_wrapper": (None, [PP, PP, PP, c_int, c_int, c_int]),
    "VectorGradient_2D_gpu_wrapper": (None, [PP, PP, PP, c_int, c_int, c_int]),
    "VectorDGDivergence_2D_gpu_wrapper": (None, [PP] * 6 + [c_int, c_int, c_int]),
    "Determinant_Tensor2D_gpu_wrapper": (None, [PP, PP, c_int, c_int, c_int]),
    "CalculateContravariantBasis_SEMQuad_gpu_wrapper": (None, [PP, PP, c_int, c_int]),
    "AdjustBoundaryContravariantBasis_SEMQuad_gpu_wrapper": (None, [PP, PP, c_int, c_int]),
    "GradientBR_MappedScalar2D_gpu_wrapper": (None, [PP] * 10 + [c_int, c_int, c_int]),
    "GradientSF_MappedScalar2D_gpu_wrapper": (None, [PP] * 5 + [c_int, c_int, c_int]),
    "JacobianWeight_MappedScalar2D_gpu_wrapper": (None, [PP, PP, c_int, c_int, c_int]),
    "JacobianWeight_MappedVector2D_gpu_wrapper": (None, [PP, PP, c_int, c_int, c_int]),
    "ContravariantProjection_MappedVector2D_gpu_wrapper": (None, [PP, PP, c_int, c_int, c_int]),
    "SideExchange_MappedScalar2D_gpu_wrapper": (None, [PP, PP, PP, PP, c_int, c_int, c_int, c_int, c_int]),
    "SideExchange_MappedVector2D_gpu_wrapper": (None, [PP, PP, PP, PP, c_int, c_int, c_int, c_int, c_int]),
    "BassiRebaySides_MappedScalar2D_gpu_wrapper": (None, [PP, PP, PP, c_int, c_int, c_int]),
    "UpdateGRK_Model2D_gpu_wrapper": (None, [PP, PP, PP, c_double, c_double, c_double, c_int, c_int, c_int,
                                             c_int]),
    "UpdateSolution_Model2D_gpu_wrapper": (None, [PP, PP, c_double, c_int, c_int, c_int]),
    "CalculateDSDt_Model2D_gpu_wrapper": (None, [PP, PP, PP, c_int, c_int, c_int]),
    "SetBoundaryCondition_LinearShallowWater_gpu_wrapper": (None, [PP, PP, PP, PP, c_int, c_int, c_int]),
    "Source_LinearShallowWater_gpu_wrapper": (None, [PP, PP, PP, c_int, c_int, c_int]),
    "Flux_LinearShallowWater_gpu_wrapper": (None, [PP, PP, PP, c_double, c_int, c_int, c_int]),
    "RiemannSolver_LinearShallowWater_gpu_wrapper": (None, [PP] * 6 + [c_double, c_int, c_int, c_int]),
    "SetBoundaryCondition_ShallowWater_gpu_wrapper": (None, [PP, PP, PP, PP, PP, c_int, c_int, c_int]),
    "Source_ShallowWater_gpu_wrapper": (None, [PP, PP, PP, c_double, c_double, c_int, c_int, c_int]),
    "Flux_ShallowWater_gpu_wrapper": (None, [PP, PP, PP, c_double, c_int, c_int, c_int]),
    "RiemannSolver_ShallowWater_gpu_wrapper": (None, [PP] * 7 + [c_double, c_int, c_int, c_int]),
    "PreTendency_ShallowWater_gpu_wrapper": (None, [PP, PP, PP, PP, c_int, c_int, c_int]),
    "Source_CompressibleIdealGas2D_gpu_wrapper": (None, [PP, PP, PP, c_int, c_int, c_int]),
    "Flux_CompressibleIdealGas2D_gpu_wrapper": (None, [PP, PP, PP, c_int, c_int, c_int]),
    "NaiveLLF_CompressibleIdealGas2D_gpu_wrapper": (None, [PP] * 9 + [c_int, c_int, c_int, c_int]),
    "SetBoundaryCondition_CompressibleIdealGas2D_gpu_wrapper": (None, [PP] * 11 + [c_int, c_int, c_int, c_int]),
    "CalculateDiagnostics_CompressibleIdealGas2D_gpu_wrapper": (None, [PP, PP, c_double, c_double, c_int, c_int,
                                                                       c_int, c_int]),
    "ConservativeToPrimitive_CompressibleIdealGas2D_gpu_wrapper": (None, [PP, PP, c_double, c_int, c_int,
                                                                          c_int]),
    "ConservativeToEntropy_CompressibleIdealGas2D_gpu_wrapper": (None, [PP, PP, c_double, c_int, c_int, c_int]),
}


class SelfGpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"selfgpu error {code}: {msg}")
        self.code = code


def lib():
    """The loaded library; raises if the CUDA extension has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with `python -m self_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS)


def check(rc):
    if rc != 0:
        raise SelfGpuError(rc, lib().selfgpu_last_error().decode())
    return rc


def pp(ptr):
    """A real** for the drop-in wrappers: address of a variable holding ``ptr``."""
    return ctypes.pointer(ctypes.c_void_p(ptr))

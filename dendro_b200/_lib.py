"""ctypes binding of libdendro_b200.so (include/dendro_b200.h).

The library is the only implementation: there is no CPU fallback.  Loading
fails with an exception when the shared object is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "libdendro_b200.so")

OCT_DTYPE = np.dtype([("x", "<u4"), ("y", "<u4"), ("z", "<u4"), ("lf", "<u4")])

STATUS = {0: "ok", 1: "invalid argument", 2: "out of device memory", 3: "CUDA error", 4: "not converged",
          5: "device wait timed out", 6: "octree not linear/complete/balanced", 7: "unsupported depth",
          8: "not implemented"}


class DendroError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str):
        super().__init__(f"{where}: {STATUS.get(status, status)} ({detail})")
        self.status = status


class SolveReport(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("rel_residual", C.c_double),
                ("solve_ms", C.c_double), ("smoother_fallbacks", C.c_int)]


class DamgConfig(C.Structure):
    _fields_ = [("nlevels", C.c_int), ("nu_pre", C.c_int), ("nu_post", C.c_int), ("omega", C.c_double),
                ("rtol", C.c_double), ("maxit", C.c_int), ("inner_prec", C.c_int), ("use_graph", C.c_int),
                ("coarse_op", C.c_int), ("dof", C.c_int), ("mu", C.c_double), ("lambda_", C.c_double)]


_lib = None


def lib():
    """Load the library (raises when it is missing: no fallback path exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(SO):
        raise ImportError(f"{SO} is missing; build it with `python -m dendro_b200.build` "
                          "(nvcc, sm_100a)")
    L = C.CDLL(SO)
    P, I64, U32, I = C.c_void_p, C.c_int64, C.c_uint32, C.c_int
    PP = C.POINTER(C.c_void_p)
    I64P = C.POINTER(C.c_int64)
    sig = {
        "dg_status_string": ([I], C.c_char_p),
        "dg_last_error": ([C.c_char_p, C.c_size_t], None),
        "dg_device_count": ([], I),
        "dg_points2octree": ([P, I64, I, U32, U32, PP], I),
        "dg_octree_from_octants": ([P, I64, I, U32, PP], I),
        "dg_balance_octree": ([P, PP], I),
        "dg_coarsen_octree": ([P, PP], I),
        "dg_octree_size": ([P], I64),
        "dg_octree_max_depth": ([P], U32),
        "dg_octree_export": ([P, P], I),
        "dg_octree_destroy": ([P], None),
        "dg_da_create": ([P, PP], I),
        "dg_da_create_from_maps": ([I64, I64, U32, P, P, P, P, P, P, PP], I),
        "dg_da_sizes": ([P, I64P, I64P, I64P], I),
        "dg_da_octets": ([P], C.c_int64),
        "dg_da_compress_maps": ([P, I], I),
        "dg_da_load_vector": ([P, P, P, I], I),
        "dg_da_compressed_map_bytes": ([P, I64P], C.c_int64),
        "dg_da_decompress_maps": ([P, P], I),
        "dg_da_max_depth": ([P], U32),
        "dg_da_export": ([P] * 9, I),
        "dg_da_element_centers": ([P, P], I),
        "dg_da_destroy": ([P], None),
        "dg_mat_create_lapmass": ([P, P, PP], I),
        "dg_mat_create_elasticity": ([P, C.c_double, C.c_double, P, PP], I),
        "dg_mat_mult": ([P, P, P, P], I),
        "dg_mat_mult_f32": ([P, P, P, P], I),
        "dg_mat_get_diagonal": ([P, P, P], I),
        "dg_mat_mult_host": ([P, P, P], I),
        "dg_mat_size": ([P], I64),
        "dg_mat_kernel_name": ([P, I], C.c_char_p),
        "dg_mat_kernel_count": ([], I),
        "dg_mat_set_kernel": ([P, I, I], I),
        "dg_mat_mult_multi": ([P, P, P, I, I, P], I),
        "dg_damg_set_tolerances": ([P, C.c_double, I], I),
        "dg_mat_destroy": ([P], None),
        "dg_damg_default_config": ([C.POINTER(DamgConfig)], None),
        "dg_damg_create": ([P, C.POINTER(DamgConfig), PP], I),
        "dg_damg_set_lapmass": ([P, P], I),
        "dg_damg_solve": ([P, P, P, I, C.POINTER(SolveReport)], I),
        "dg_damg_solve_multi": ([P, P, P, I, I, C.POINTER(SolveReport)], I),
        "dg_damg_levels": ([P], I),
        "dg_damg_level_sizes": ([P, P, P], I),
        "dg_damg_level_da": ([P, I], P),
        "dg_damg_prolong": ([P, I, P, P, I], I),
        "dg_damg_restrict": ([P, I, P, P, I], I),
        "dg_damg_destroy": ([P], None),
        "dg_vec_dot": ([P, P, I64, P, P], I),
        "dg_damg_create_batch": ([P, I, C.POINTER(DamgConfig), PP], I),
        "dg_damg_vcycle": ([P, P, P], I),
        "dg_mlp_param_count": ([], I),
        "dg_mlp_create": ([P, PP], I),
        "dg_mlp_get_params": ([P, P], I),
        "dg_mlp_set_params": ([P, P], I),
        "dg_mlp_forward": ([P, P, I64, P, I, P], I),
        "dg_mlp_gradient": ([P, P, P, I64, I, P, C.POINTER(C.c_double)], I),
        "dg_mlp_train_step": ([P, P, P, I64, C.c_float, C.POINTER(C.c_double)], I),
        "dg_mlp_destroy": ([P], None),
        "dg_damg_set_smoother": ([P, P, I, C.c_double], I),
        "dg_damg_features": ([P, P, P, C.POINTER(C.c_float)], I),
        "dg_damg_batch_count": ([P], I),
        "dg_damg_batch_offsets": ([P, I, P, P], I),
        "dg_vec_dot_noalloc": ([P, P, I64, P, P], I),
        "dg_device_check": ([P], I),
        "dg_write_pts": ([C.c_char_p, P, I64], I),
        "dg_read_pts": ([C.c_char_p, P, I64, I64P], I),
        "dg_write_data_pts": ([C.c_char_p, P, P, I64], I),
        "dg_read_data_pts": ([C.c_char_p, P, P, I64, I64P], I),
        "dg_octree_write": ([P, C.c_char_p], I),
        "dg_octree_read": ([C.c_char_p, PP], I),
        "dg_da_dump_mesh": ([P, C.c_char_p], I),
        "dg_damg_level_apply": ([P, I, P, P, I], I),
        "dg_mat_create_dirichlet": ([P, I, P, PP], I),
        "dg_set_device_wait_limit": ([I64], I),
        "dg_partition_weighted": ([I64, P, I, P], I),
        "dg_halo_create": ([I64, I64, U32, P, P, P, P, P, P, P, I, I, PP], I),
        "dg_halo_create_from_da": ([P, P, I, I, PP], I),
        "dg_halo_sizes": ([P, I64P, I64P, I64P, I64P, I64P], I),
        "dg_halo_ranges": ([P, P, P], I),
        "dg_halo_comm": ([P, P, P, P, P], I),
        "dg_halo_part": ([P, I, P, P], I),
        "dg_halo_local_da": ([P, I, PP], I),
        "dg_halo_pack": ([P, P, P, I, P], I),
        "dg_halo_accumulate": ([P, P, P, I, P], I),
        "dg_mat_mult_add": ([P, P, P, P], I),
        "dg_damg_transfer_export": ([P, I, I, I64P, P, P, P], I),
        "dg_damg_level_coef": ([P, I, P], I),
        "dg_damg_coarse_solve": ([P, P, P, P], I),
        "dg_parcsr_create": ([I64, I64, P, P, P, P, P, I, I, PP], I),
        "dg_parcsr_sizes": ([P, I64P, I64P, I64P, I64P], I),
        "dg_parcsr_comm": ([P, P, P, P, P], I),
        "dg_parcsr_pack": ([P, P, P, P], I),
        "dg_parcsr_apply": ([P, P, P, P, I, P], I),
        "dg_parcsr_destroy": ([P], None),
        "dg_vec_jacobi_update": ([P, P, P, P, C.c_double, I64, P], I),
        "dg_vec_jacobi_update_f32": ([P, P, P, P, C.c_float, I64, P], I),
        "dg_mat_mult_add_f32": ([P, P, P, P], I),
        "dg_halo_pack_f32": ([P, P, P, I, P], I),
        "dg_parcsr_pack_f32": ([P, P, P, P], I),
        "dg_parcsr_apply_f32": ([P, P, P, P, I, P], I),
        "dg_halo_destroy": ([P], None),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def exported_symbols():
    """Names declared in include/dendro_b200.h that the loaded library must export."""
    return [
        "dg_status_string", "dg_last_error", "dg_device_count", "dg_points2octree", "dg_octree_from_octants",
        "dg_balance_octree", "dg_coarsen_octree", "dg_octree_size", "dg_octree_max_depth", "dg_octree_export",
        "dg_octree_destroy", "dg_da_create", "dg_da_create_from_maps", "dg_da_sizes", "dg_da_max_depth", "dg_da_octets",
        "dg_da_compress_maps", "dg_da_compressed_map_bytes", "dg_da_decompress_maps", "dg_da_load_vector",
        "dg_da_export", "dg_da_element_centers", "dg_da_destroy", "dg_mat_create_lapmass",
        "dg_mat_create_elasticity", "dg_mat_mult", "dg_mat_mult_f32", "dg_mat_get_diagonal",
        "dg_mat_mult_host", "dg_mat_size", "dg_mat_kernel_name", "dg_mat_destroy", "dg_damg_default_config", "dg_damg_create",
        "dg_damg_set_lapmass", "dg_damg_solve", "dg_damg_solve_multi", "dg_damg_levels", "dg_damg_level_sizes", "dg_damg_level_da",
        "dg_damg_prolong", "dg_damg_restrict", "dg_damg_destroy", "dg_vec_dot",
        "dg_damg_create_batch", "dg_damg_batch_count", "dg_damg_batch_offsets", "dg_damg_vcycle",
        "dg_mlp_param_count", "dg_mlp_create", "dg_mlp_get_params", "dg_mlp_set_params", "dg_mlp_forward",
        "dg_mlp_gradient", "dg_mlp_train_step", "dg_mlp_destroy", "dg_damg_set_smoother", "dg_damg_features",
        "dg_vec_dot_noalloc", "dg_mat_kernel_count", "dg_mat_set_kernel", "dg_device_check",
        "dg_set_device_wait_limit", "dg_write_pts", "dg_read_pts", "dg_write_data_pts", "dg_read_data_pts",
        "dg_octree_write", "dg_octree_read", "dg_da_dump_mesh", "dg_damg_level_apply",
        "dg_mat_create_dirichlet",
        "dg_mat_mult_multi", "dg_damg_set_tolerances",
        "dg_partition_weighted", "dg_halo_create", "dg_halo_create_from_da", "dg_halo_sizes", "dg_halo_ranges",
        "dg_halo_comm", "dg_halo_part", "dg_halo_local_da", "dg_halo_pack", "dg_halo_accumulate",
        "dg_halo_destroy", "dg_mat_mult_add", "dg_damg_transfer_export", "dg_damg_level_coef",
        "dg_damg_coarse_solve", "dg_parcsr_create", "dg_parcsr_sizes", "dg_parcsr_comm", "dg_parcsr_pack",
        "dg_parcsr_apply", "dg_parcsr_destroy", "dg_vec_jacobi_update", "dg_vec_jacobi_update_f32",
        "dg_mat_mult_add_f32", "dg_halo_pack_f32", "dg_parcsr_pack_f32", "dg_parcsr_apply_f32",
    ]


def check(status: int, where: str) -> None:
    if status != 0:
        buf = C.create_string_buffer(512)
        lib().dg_last_error(buf, 512)
        raise DendroError(status, where, buf.value.decode(errors="replace"))


def ptr(a):
    """Pointer of a numpy array or a torch tensor (None passes through)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return C.c_void_p(a.ctypes.data)
    return C.c_void_p(a.data_ptr())

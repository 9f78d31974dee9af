"""ctypes binding of libys_newton.so (the C ABI in include/ys_newton.h).

The library is required: importing the compute entry points without it, or
calling them without a CUDA device, raises.  There is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libys_newton.so")

u8, i32, u32, u64, f64, vp = C.c_uint8, C.c_int32, C.c_uint32, C.c_uint64, C.c_double, C.c_void_p
P = C.POINTER

YS_OK = 0
YS_ERR_CUDA = -1
YS_ERR_INVALID = -2
YS_ERR_CAPACITY = -3
YS_ERR_NOT_CONVERGED = -4
YS_ERR_INVALID_RESIDUAL = -5
YS_ERR_SINGULAR_DOMAIN = -6
YS_PREC_BLOCK_JACOBI = 0
YS_PREC_MAS = 1
YS_STOP_PRECONDITIONED = 0
YS_STOP_RESIDUAL = 1
YS_MAX_UNION = 8
(YS_ENERGY_POINT_POINT, YS_ENERGY_POINT_EDGE, YS_ENERGY_POINT_TRIANGLE, YS_ENERGY_EDGE_EDGE, YS_ENERGY_BENDING,
 YS_ENERGY_BARAFF_WITKIN, YS_ENERGY_STVK_MEMBRANE, YS_ENERGY_FRICTION_PT, YS_ENERGY_FRICTION_PE,
 YS_ENERGY_FRICTION_EE, YS_ENERGY_FRICTION_PP) = range(1, 12)
YS_SPMV_TILE_ROWS = 64
YS_SERVE_EMPTY, YS_SERVE_INIT, YS_SERVE_REFINE, YS_SERVE_START, YS_SERVE_ITER, YS_SERVE_DONE, YS_SERVE_FAILED = range(7)


class PatternOut(C.Structure):
  _fields_ = [("positions", vp), ("block_dims", vp), ("value_offset", vp), ("lookup", vp), ("record", vp),
              ("record_begin", vp), ("record_count", vp), ("num_unique", u32), ("num_categories", u32),
              ("category_dims", C.c_uint16 * 32), ("category_counts", u32 * 16), ("category_starts", u32 * 17),
              ("total_records", u64)]


class Union3(C.Structure):
  _fields_ = [("child", vp * YS_MAX_UNION), ("prefix", u32 * (YS_MAX_UNION + 1)), ("num_children", u32)]


class TermPlan(C.Structure):
  _fields_ = [("codes", vp), ("K", u32), ("slot_stride", u32), ("coord_outer", vp), ("record", vp),
              ("grad_outer", vp), ("grad_record", vp)]


class SnhArgs(C.Structure):
  _fields_ = [("position", Union3), ("rest", Union3), ("tets", vp), ("num_elements", u32), ("mu", vp), ("lam", vp),
              ("mu_value", f64), ("lam_value", f64), ("dt", f64), ("projection_method", i32), ("plan", TermPlan),
              ("block_records", vp), ("grad_records", vp), ("energy", vp), ("work_list", vp), ("work_count", vp)]


class InertiaArgs(C.Structure):
  _fields_ = [("position", vp), ("x_before", vp), ("velocity", vp), ("mass", vp), ("dt", f64), ("gravity", f64 * 3),
              ("num_vertices", u32), ("plan", TermPlan), ("block_records", vp), ("grad_records", vp),
              ("energy", vp)]


class EnergyArgs(C.Structure):
  _fields_ = [("kind", i32), ("position", Union3), ("rest", Union3), ("conn", vp), ("arity", u32),
              ("num_elements", u32), ("params", vp), ("param_stride", u32), ("values", f64 * 8),
              ("projection_method", i32), ("plan", TermPlan), ("block_records", vp), ("grad_records", vp),
              ("energy", vp)]


class AffineArgs(C.Structure):
  _fields_ = [("kind", i32), ("affine", vp), ("translation", vp), ("num_bodies", u32), ("num_elements", u32),
              ("body", vp), ("rest", vp), ("tets", vp), ("num_rest", u32), ("x_before", vp), ("velocity", vp),
              ("mass", vp), ("mu", vp), ("lam", vp), ("mu_value", f64), ("lam_value", f64), ("dt", f64),
              ("gravity", f64 * 3), ("stiffness", f64), ("projection_method", i32), ("plan", TermPlan),
              ("block_records", vp), ("grad_records", vp), ("energy", vp)]


YS_AFFINE_ORTHOGONALITY, YS_AFFINE_INERTIA, YS_AFFINE_SNH = 1, 2, 3


class CoupledArgs(C.Structure):
  _fields_ = [("base", EnergyArgs), ("affine_child", u32), ("vertex_body", vp), ("rest", vp), ("affine", vp),
              ("translation", vp), ("num_bodies", u32), ("status", vp)]


class SpmvStream(C.Structure):
  _fields_ = [("blocks32", vp), ("desc", vp), ("rows", vp), ("words", vp), ("halo", vp), ("block_cap", u32),
              ("entry_cap", u32), ("halo_cap", u32)]


class Matrix3(C.Structure):
  _fields_ = [("num_sets", u32), ("values", vp * 2), ("values32", vp * 2), ("row_ptr", vp * 2),
              ("entry_block", vp * 2), ("entry_col", vp * 2), ("num_vars", u32), ("row_block", vp * 2),
              ("tile_cap", u32 * 2), ("entry_cap", u32 * 2), ("stream", SpmvStream * 2)]


class PcgArgs(C.Structure):
  _fields_ = [("matrix", Matrix3), ("precision", i32), ("preconditioner", i32), ("jacobi_inverse", vp), ("mas", vp),
              ("stop_rule", i32), ("tolerance", f64), ("max_iterations", u32), ("rhs", vp), ("solution", vp),
              ("zero_initial_guess", i32), ("workspace", vp), ("jacobi_group", vp)]


class PcgResult(C.Structure):
  _fields_ = [("status", i32), ("iterations", u32), ("delta0", f64), ("delta", f64), ("residual0", f64),
              ("residual", f64)]


class MasDesc(C.Structure):
  _fields_ = [("num_fine_vars", u32), ("num_levels", u32), ("level_node_offset", P(u32)), ("level_weights", P(f64)),
              ("cmap", vp), ("child_ptr", vp), ("child_fine", vp), ("num_domains", u32), ("dom_node_ptr", vp),
              ("dom_nodes", vp), ("inv_offset", vp), ("dom_entry_ptr", vp), ("dom_entry", vp),
              ("fine_blocks", u32), ("coarse_blocks", u32), ("cb_src_ptr", vp), ("cb_src", vp),
              ("cb_level_begin", P(u32)), ("max_domain_dofs", u32), ("coarse_values", vp), ("inverse", vp),
              ("level_residual", vp), ("level_correction", vp), ("status", vp), ("level_residual64", vp)]



class ServeSlotDesc(C.Structure):
  _fields_ = [("mas", vp), ("matrix", Matrix3), ("rhs", vp), ("solution", vp), ("workspace", vp), ("tolerance", f64),
              ("refinement_tolerance", f64), ("max_iterations", u32)]


class ServeSlotStatus(C.Structure):
  _fields_ = [("phase", i32), ("iterations", u32), ("refinements", u32), ("relative_residual", f64)]

# name: (restype, argtypes)
SIGNATURES = {
    "ys_last_error": (C.c_char_p, []),
    "ys_version": (i32, []),
    "ys_join_union_indices": (i32, [vp, u32, u32, u32, P(u32), P(i32), P(u32), u32, vp, vp, vp]),
    "ys_compress_indices": (i32, [vp, vp, u32, u32, vp, vp, vp, vp]),
    "ys_compress_indices_noalloc": (i32, [vp, vp, u32, u32, vp, vp, vp, vp]),
    "ys_compute_coordinates": (i32, [vp, vp, vp, vp, u32, u32, vp, vp, vp]),
    "ys_pattern_workspace_bytes": (i32, [u32, P(u64)]),
    "ys_pattern_build": (i32, [vp, vp, u32, vp, u64, P(PatternOut), vp]),
    "ys_snh_eval": (i32, [P(SnhArgs), vp]),
    "ys_inertia_eval": (i32, [P(InertiaArgs), vp]),
    "ys_energy_eval": (i32, [P(EnergyArgs), vp]),
    "ys_local_hessians": (i32, [P(EnergyArgs), vp, vp]),
    "ys_rest_local_hessians": (i32, [P(EnergyArgs), vp, vp]),
    "ys_snh_local_hessians": (i32, [P(SnhArgs), vp, vp]),
    "ys_snh_rest_local_hessians": (i32, [P(SnhArgs), vp, vp]),
    "ys_inertia_local_hessians": (i32, [vp, f64, f64, u32, u32, vp, vp]),
    "ys_rect_coordinates": (i32, [vp, vp, u32, u32, u32, u32, vp, vp, vp, vp]),
    "ys_rect_records": (i32, [vp, u32, u32, vp, vp, u32, u32, u32, vp, vp, vp, vp]),
    "ys_rect_plan_workspace_bytes": (i32, [u32, P(u64)]),
    "ys_rect_plan": (i32, [vp, u32, u32, u32, u32, vp, vp, vp, vp, u64, vp]),
    "ys_rect_spmv": (i32, [vp, vp, vp, vp, vp, u32, u32, u32, vp, vp, u32, u32, vp]),
    "ys_snh_param_jacobian": (i32, [P(SnhArgs), u32, vp, vp]),
    "ys_inertia_mass_jacobian": (i32, [P(InertiaArgs), u32, vp, vp]),
    "ys_rect_param_coordinates": (i32, [vp, u32, u32, u32, u32, u32, vp, vp, vp, vp]),
    "ys_rect_param_records": (i32, [vp, u32, vp, u32, u32, u32, vp, vp, vp, vp]),
    "ys_affine_position_jacobian": (i32, [vp, vp, u32, C.c_int64, C.c_int64, vp, vp, vp, vp, vp]),
    "ys_affine_eval": (i32, [P(AffineArgs), vp]),
    "ys_coupled_indices": (i32, [vp, u32, u32, u32, P(u32), P(i32), P(u32), u32, vp, u32, i32, u32, i32, u32, vp, vp,
                                 vp]),
    "ys_coupled_energy_eval": (i32, [P(CoupledArgs), vp]),
    "ys_sum_workspace_doubles": (u64, []),
    "ys_sum": (i32, [vp, u32, vp, vp, vp]),
    "ys_assemble": (i32, [vp, vp, vp, vp, vp, u32, vp, vp, vp]),
    "ys_assemble3": (i32, [vp, vp, vp, vp, u32, vp, vp, vp]),
    "ys_assemble_strided": (i32, [vp, vp, vp, vp, u32, vp, u32, vp, vp]),
    "ys_extract_diagonal": (i32, [vp, vp, vp, vp, u32, u32, P(u32), P(u32), P(u32), vp, vp, i32, vp]),
    "ys_invert_diagonal_blocks": (i32, [vp, vp, u32, P(u32), P(u32), P(u32), vp]),
    "ys_spmv_plan_workspace_bytes": (i32, [u32, u32, P(u64)]),
    "ys_spmv_plan_build": (i32, [vp, u32, u32, vp, u64, vp, vp, vp, vp]),
    "ys_spmv3": (i32, [vp, vp, vp, vp, vp, u32, vp, vp, i32, vp]),
    "ys_mas_inverse_floats": (u64, [u32]),
    "ys_mas_failed_domains": (i32, [vp, vp, P(i32)]),
    "ys_pack_x32": (i32, [vp, u32, vp, vp]),
    "ys_spmv3_x32": (i32, [vp, vp, vp, vp, u32, vp, vp, i32, vp]),
    "ys_spmv_tile_plan": (i32, [vp, u32, vp, vp, u32, vp, P(u32), P(u32), vp]),
    "ys_spmv3_x32_tiled": (i32, [vp, vp, vp, vp, vp, u32, u32, u32, u32, vp, vp, i32, vp, vp]),
    "ys_spmv_stream_words": (i32, [u32, u32, P(u64)]),
    "ys_spmv_stream_plan": (i32, [vp, vp, vp, vp, u32, u64, vp, vp, vp, vp, vp, u32, vp, P(u32), vp]),
    "ys_assemble3_streamed": (i32, [vp, vp, vp, vp, u32, vp, vp, vp, vp, vp]),
    "ys_spmv_stream_fill": (i32, [vp, vp, u64, vp, vp]),
    "ys_spmv3_x32_streamed": (i32, [P(SpmvStream), vp, vp, vp, vp, u32, vp, vp, i32, u32, u32, vp, vp]),
    "ys_pcg_workspace_doubles": (u64, [u32]),
    "ys_pcg_create": (i32, [P(PcgArgs), P(vp)]),
    "ys_pcg_run": (i32, [vp, vp, P(PcgResult)]),
    "ys_pcg_launch": (i32, [vp, vp]),
    "ys_pcg_set_params": (i32, [vp, f64, u32]),
    "ys_pcg_set_barrier_poll_limit": (i32, [vp, u32]),
    "ys_pcg_status": (i32, [vp, vp, P(PcgResult)]),
    "ys_pcg_destroy": (i32, [vp]),
    "ys_mas_create": (i32, [P(MasDesc), P(vp)]),
    "ys_mas_numeric_update": (i32, [vp, vp, vp, P(i32)]),
    "ys_mas_union_values": (i32, [vp, vp, vp, vp, u32, vp, vp]),
    "ys_mas_apply": (i32, [vp, vp, vp, vp]),
    "ys_mas_destroy": (i32, [vp]),
    "ys_mas_gemv": (i32, [vp, vp, P(u64)]),
    "ys_gradient_coordinates": (i32, [vp, vp, u32, u32, vp, vp, vp, vp]),
    "ys_refine_workspace_doubles": (u64, [u32]),
    "ys_refine_residual": (i32, [P(Matrix3), vp, vp, vp, vp, vp, P(f64), vp]),
    "ys_serve_workspace_doubles": (u64, [u32]),
    "ys_serve_create": (i32, [u32, u32, P(vp)]),
    "ys_serve_attach": (i32, [vp, u32, P(ServeSlotDesc)]),
    "ys_serve_detach": (i32, [vp, u32]),
    "ys_serve_launch": (i32, [vp, vp]),
    "ys_serve_status": (i32, [vp, vp, P(ServeSlotStatus)]),
    "ys_serve_destroy": (i32, [vp]),
}

_lib = None


class YsError(RuntimeError):
  def __init__(self, name, code, msg):
    super().__init__(f"{name} failed with status {code}: {msg}")
    self.code = code


def load() -> C.CDLL:
  """Load the library (build it first with ``python -m yasps_b200.build``)."""
  global _lib
  if _lib is None:
    if not os.path.exists(LIB_PATH):
      raise ImportError(f"libys_newton.so not built at {LIB_PATH}; run `python -m yasps_b200.build`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
      fn = getattr(lib, name)
      fn.restype = res
      fn.argtypes = args
    _lib = lib
  return _lib


def call(name, *args, ok=(YS_OK,)):
  """Call an entry point and raise YsError unless its status is in ``ok``."""
  lib = load()
  rc = getattr(lib, name)(*args)
  if rc not in ok:
    raise YsError(name, rc, lib.ys_last_error().decode())
  return rc


def ptr(t) -> int | None:
  """Device (or host) address of a tensor, None for None/empty."""
  if t is None:
    return None
  return t.data_ptr() if t.numel() else None


def stream_ptr(stream=None):
  import torch
  s = torch.cuda.current_stream() if stream is None else stream
  return s.cuda_stream

"""The C-ABI library loads and exports every entry point of include/ys_newton.h."""

import ctypes
import os
import re

from yasps_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
  text = open(os.path.join(ROOT, "include", "ys_newton.h")).read()
  text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
  return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\**\s*(ys_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
  names = declared_functions()
  assert "ys_snh_eval" in names and "ys_pcg_create" in names and "ys_mas_create" in names
  assert len(names) >= 25


def test_library_exports_every_declared_symbol():
  lib = _lib.load()
  for name in declared_functions():
    assert hasattr(lib, name), name
    assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"


def test_version_and_error_string_without_gpu():
  lib = _lib.load()
  assert lib.ys_version() >= 100
  assert isinstance(lib.ys_last_error(), bytes)


def _header_structs():
  text = open(os.path.join(ROOT, "include", "ys_newton.h")).read()
  text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
  out = {}
  for body, name in re.findall(r"typedef struct \w+ \{(.*?)\} (\w+);", text, flags=re.S):
    fields = []
    for decl in body.split(";"):
      decl = decl.strip()
      if not decl:
        continue
      for part in decl.split(","):
        m = re.search(r"(\w+)\s*(\[[^\]]*\])?\s*$", part.strip())
        fields.append(m.group(1))
    out[name] = fields
  return out


def test_ctypes_structs_follow_header_field_order():
  structs = _header_structs()
  pairs = {"ys_pattern_out": _lib.PatternOut, "ys_union3": _lib.Union3, "ys_term_plan": _lib.TermPlan,
           "ys_snh_args": _lib.SnhArgs, "ys_inertia_args": _lib.InertiaArgs, "ys_matrix3": _lib.Matrix3,
           "ys_pcg_args": _lib.PcgArgs, "ys_pcg_result": _lib.PcgResult, "ys_mas_desc": _lib.MasDesc,
           "ys_serve_slot_desc": _lib.ServeSlotDesc, "ys_energy_args": _lib.EnergyArgs, "ys_affine_args": _lib.AffineArgs,
           "ys_coupled_args": _lib.CoupledArgs, "ys_spmv_stream": _lib.SpmvStream,
           "ys_serve_slot_status": _lib.ServeSlotStatus}
  for cname, cls in pairs.items():
    assert structs[cname] == [f[0] for f in cls._fields_], cname


def test_struct_layouts_match_header_sizes():
  # pointers 8 bytes, the union descriptor is 8 pointers + 9 u32 + u32 (+pad)
  assert ctypes.sizeof(_lib.Union3) == 8 * 8 + 10 * 4
  assert ctypes.sizeof(_lib.PcgResult) == 4 + 4 + 4 * 8

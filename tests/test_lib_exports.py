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


def test_struct_layouts_match_header_sizes():
  # pointers 8 bytes, the union descriptor is 8 pointers + 9 u32 + u32 (+pad)
  assert ctypes.sizeof(_lib.Union3) == 8 * 8 + 10 * 4
  assert ctypes.sizeof(_lib.PcgResult) == 4 + 4 + 4 * 8

"""Build libys_newton.so (sm_100a) in-tree with nvcc.

Usage: ``python -m yasps_b200.build [--verbose]``.  Compiles every ``.cu`` in
``yasps_b200/csrc`` to an object with ``-gencode arch=compute_100a,code=sm_100a``
and links one shared library next to this file.  Objects are rebuilt when
their source or any header changed.
"""

from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libys_newton.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=hidden", "-I", INCLUDE, "-I", CSRC]


def _newest_header() -> float:
  paths = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
  return max((os.path.getmtime(p) for p in paths), default=0.0)


def build(verbose: bool = False, force: bool = False) -> str:
  os.makedirs(BUILD, exist_ok=True)
  sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
  headers = _newest_header()
  objects = []
  for src in sources:
    obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
    objects.append(obj)
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), headers):
      continue
    cmd = [NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj]
    if verbose:
      cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or res.returncode != 0:
      sys.stderr.write(res.stdout + res.stderr)
    if res.returncode != 0:
      raise RuntimeError(f"nvcc failed for {src}")
  newest = max(os.path.getmtime(o) for o in objects)
  if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objects, "-lcuda"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
      sys.stderr.write(res.stdout + res.stderr)
      raise RuntimeError("nvcc link failed")
  return LIB


if __name__ == "__main__":
  print(build(verbose="--verbose" in sys.argv, force="--force" in sys.argv))

"""Python access to the checkers (test infrastructure only).

* ``run_oracle`` drives the C restatement (``libmac_oracle.so``).
* ``run_ref`` drives the reference's own code compiled from its headers
  (``_ref/mac_ref``), when that binary was built.

Both exchange states through the file format of ``state_format.h``.
Only the tests, the smoke check and bench.py's CPU-baseline leg use this.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libmac_oracle.so")
REF = os.path.join(HERE, "_ref", "mac_ref")
REF_DEPTH = os.path.join(HERE, "_ref", "mac_ref_depth")
REF_B = os.path.join(HERE, "_ref", "mac_ref_b")
PIPELINE_B = ("bstep", "binit", "bode")

_lib = None
# The reference checkout's sources, read in place by the Makefile's _ref
# targets (MAC_REF_SRC overrides the checkout's location).
REF_SRC = os.environ.get("MAC_REF_SRC", "/root/reference/src")


def build(quiet: bool = True) -> None:
    """Builds the restatement (and the reference runner when the reference
    sources are present)."""
    out = subprocess.run(["make", "-C", HERE, "all", f"REF_SRC={REF_SRC}"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = ctypes.CDLL(LIB)
        _lib.mac_oracle_run.restype = ctypes.c_int
        _lib.mac_oracle_run.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                        ctypes.c_int, ctypes.c_double,
                                        ctypes.POINTER(ctypes.c_double)]
        _lib.mac_oracle_probe.restype = ctypes.c_int
        _lib.mac_oracle_probe.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                          ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_double)]
        _lib.mac_oracle_jitter8.restype = None
        _lib.mac_oracle_jitter8.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_double,
                                            ctypes.POINTER(ctypes.c_double)]
    return _lib


def run_oracle(cmd: str, in_path: str, out_path: str, n: int = 1, rtol: float = 1e-14) -> dict:
    """Runs stage ``cmd`` ``n`` times on the state in ``in_path``."""
    stats = (ctypes.c_double * 8)()
    rc = lib().mac_oracle_run(in_path.encode(), (out_path or "").encode(), cmd.encode(), n, rtol,
                              stats)
    if rc != 0:
        raise RuntimeError(f"oracle {cmd} failed ({rc})")
    return {"invalid_reads": stats[0], "created_cells": stats[1], "cg_iters": stats[2],
            "relres": stats[3], "max_div": stats[4], "fluid_cell_steps": stats[5]}


def probe(in_path: str, what: str, pos=(0.0, 0.0, 0.0), key=(0, 0, 0), i=0, sym=1):
    """One policy evaluation on a state: speed | convection | divergence | gradient."""
    code = {"speed": 0, "convection": 1, "divergence": 2, "gradient": 3}[what]
    p = (ctypes.c_double * 3)(*pos)
    k = (ctypes.c_int * 3)(*key)
    out = (ctypes.c_double * 3)()
    rc = lib().mac_oracle_probe(in_path.encode(), code, p, k, i, sym, out)
    if rc != 0:
        raise RuntimeError(f"probe {what} failed ({rc})")
    return [out[0], out[1], out[2]] if code == 0 else out[0]


def jitter8(seed, k, s, h):
    out = (ctypes.c_double * 3)()
    lib().mac_oracle_jitter8(seed, int(k[0]), int(k[1]), int(k[2]), int(s), h[0], h[1], h[2], out)
    return [out[0], out[1], out[2]]


def material(code: int) -> dict:
    """The oracle's material rules for one material code: the predicates and
    the results of SetAir / SetFluid."""
    out = (ctypes.c_int * 5)()
    lib().mac_oracle_material(int(code), out)
    return {"is_fluid": bool(out[0]), "is_air": bool(out[1]), "in_domain": bool(out[2]),
            "after_set_air": out[3], "after_set_fluid": out[4]}


def have_ref() -> bool:
    return os.path.exists(REF)


def _depth_mode(path: str) -> int:
    """depth_mode of a state file's header (byte offset 128, ``state_format.h``)."""
    with open(path, "rb") as f:
        head = f.read(132)
    return int.from_bytes(head[128:132], "little", signed=True) if len(head) == 132 else 0


def run_ref(cmd: str, in_path: str, out_path: str, arg=None, timeout: float = 600.0) -> str:
    """Runs the reference's own code on a state (``cmd`` as in ``ref_world.cpp``);
    a state in the depth composition goes to the depth build of the runner, the
    pipeline-B commands to the build with three speed buffers."""
    exe = REF_B if cmd in PIPELINE_B else (REF_DEPTH if _depth_mode(in_path) else REF)
    args = [exe, cmd, in_path, out_path]
    if arg is not None:
        args.append(str(arg))
    out = subprocess.run(args, capture_output=True, text=True, timeout=timeout)
    if out.returncode != 0:
        raise RuntimeError(f"mac_ref {cmd} failed: {out.stderr}")
    return out.stdout

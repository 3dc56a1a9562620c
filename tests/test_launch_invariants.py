"""Source invariants of the dependent-launch chain (CPU, reads the CUDA sources).

Every kernel the CG loop launches with programmatic stream serialisation
(`launch_k`) must reach `pdl_entry()` -- the wait on the previous kernel -- on
every path before it may return, or a later kernel could complete before an
earlier one and read stale data; and nothing before the wait may store to
global memory. The tests check that each such kernel's body calls
`pdl_entry()` exactly once, with no `return` and no store through a kernel
parameter pointer before it.
"""
import os
import re

import pytest

CSRC = os.path.join(os.path.dirname(__file__), "..", "mac_b200", "csrc")
FILES = ["mac_mg.cu", "mac_pressure.cu"]


def _sources():
    return {f: open(os.path.join(CSRC, f)).read() for f in FILES}


def _launched_names(srcs):
    names = set()
    for s in srcs.values():
        for m in re.finditer(r"launch_k\(c,\s*([A-Za-z_0-9]+)", s):
            names.add(m.group(1))
    return sorted(names)


def _bodies(srcs, name):
    out = []
    for s in srcs.values():
        for m in re.finditer(r"__global__[^;{]*?\b" + re.escape(name) + r"\(", s):
            i = s.index(") {\n", m.end())
            j = s.index("\n}\n", i)
            params = s[m.end():i]
            out.append((params, s[i + 4:j]))
    return out


def test_launch_k_kernels_found():
    names = _launched_names(_sources())
    assert {"k0_pre", "k0_restrict", "k0_post", "kl_pre", "kl_restrict", "kl_jacobi", "kd_coarse_block",
            "k_update_spmv", "k_fin_alpha", "k_fin_beta", "k_fin_rr"} <= set(names), names


def _violations(name, params, body):
    """The ways a kernel body breaks the wait-first rule (empty: none)."""
    out = []
    if body.count("pdl_entry();") != 1:
        return [f"{name}: pdl_entry() not called exactly once"]
    pro = body[:body.index("pdl_entry();")]
    if re.search(r"\breturn\b", pro):
        out.append(f"{name}: return before the wait")
    # pointer parameters of the kernel: no element store before the wait
    ptrs = re.findall(r"\*\s*(?:__restrict__\s+)?([A-Za-z_][A-Za-z_0-9]*)\s*(?:,|$)", params)
    for p in ptrs:
        if re.search(r"\b" + re.escape(p) + r"\s*\[[^\]]*\]\s*(?:[+\-*/]?=)(?!=)", pro) or \
                re.search(r"\b" + re.escape(p) + r"\s*->\s*[A-Za-z_0-9]+\s*=(?!=)", pro):
            out.append(f"{name}: store through {p} before the wait")
    return out


@pytest.mark.parametrize("name", _launched_names(_sources()))
def test_dependent_launch_kernel_waits_first(name):
    bodies = _bodies(_sources(), name)
    assert bodies, name
    for params, body in bodies:
        assert _violations(name, params, body) == []


def test_checker_flags_planted_mistakes():
    """The checker itself, on kernels written to break the rule."""
    params = "const int* __restrict__ a, double* __restrict__ out, Scalars* ds"
    good = "  const int v = a[threadIdx.x];\n  pdl_entry();\n  out[threadIdx.x] = v;\n"
    assert _violations("good", params, good) == []
    early = "  if (a[0] < 0) return;\n  pdl_entry();\n"
    assert any("return" in v for v in _violations("early", params, early))
    store = "  out[threadIdx.x] = 1.0;\n  pdl_entry();\n"
    assert any("store through out" in v for v in _violations("store", params, store))
    member = "  ds->done = 0;\n  pdl_entry();\n"
    assert any("store through ds" in v for v in _violations("member", params, member))
    twice = "  pdl_entry();\n  pdl_entry();\n"
    assert _violations("twice", params, twice)

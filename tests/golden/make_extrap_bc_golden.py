"""Extracts the known answers of the reference's boundary-extrapolation test
(test/test_Extrapolate_Boundary.h, 7 tests, 18 runs of
Algorithm_Extrapolate_Boundary_Condition, 565 asserts) into
tests/golden/extrap_bc_2d.json.

The test file is a flat sequence of statements; each test builds a 2D world
(h = 0.1, chunk edge 2) and interleaves

    v.Set(d, k);  speed.Set(d, s);
    grid[v].Speed_GetRef().Set(Data_Speed_Data(speed), true);
    grid[v].CellType_GetRef().SetAir();  /  .SetFluid();
    alg.Do();
    TS_ASSERT_DELTA(grid[v].Speed_GetRef().Get(i), value, eps);
    TS_ASSERT(std::isnan(grid[v].Speed_GetRef().Get(i)));   (or !std::isnan)

The script replays the variables v and speed and writes, per test, the list
of operations with concrete keys and values: {"op": "speed", "key", "u"},
{"op": "type", "key", "fluid"}, {"op": "do"}, {"op": "expect", "key", "dim",
"value"} and {"op": "nan", "key", "dim", "isnan"}.

    python tests/golden/make_extrap_bc_golden.py [<reference checkout>]
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
NUM = r"(-?\d+(?:\.\d+)?(?:[eE]-?\d+)?)"


def parse(text):
    tests = []
    cur = None
    v = [0, 0]
    speed = [0.0, 0.0]
    for line in text.splitlines():
        s = line.strip()
        if s.startswith("//"):
            continue
        m = re.match(r"void (test\w+)\(\)", s)
        if m:
            cur = {"name": m.group(1), "h": [None, None], "ops": []}
            tests.append(cur)
            continue
        if cur is None:
            continue
        m = re.match(r"h\.Set\((\d),\s*" + NUM + r"\);", s)
        if m:
            cur["h"][int(m.group(1)) - 1] = float(m.group(2))
            continue
        m = re.match(r"v\.Set\((\d),\s*" + NUM + r"\);", s)
        if m:
            v[int(m.group(1)) - 1] = int(m.group(2))
            continue
        m = re.match(r"speed\.Set\((\d),\s*" + NUM + r"\);", s)
        if m:
            speed[int(m.group(1)) - 1] = float(m.group(2))
            continue
        if re.search(r"\[v\]\.Speed_GetRef\(\)\.Set\(Data_Speed_Data<DIM,type_data_value>\(speed\),true\);", s):
            cur["ops"].append({"op": "speed", "key": list(v), "u": list(speed)})
            continue
        m = re.search(r"\[v\]\.CellType_GetRef\(\)\.Set(Air|Fluid)\(\);", s)
        if m:
            cur["ops"].append({"op": "type", "key": list(v), "fluid": m.group(1) == "Fluid"})
            continue
        if re.match(r"alg\.Do\(\);", s):
            cur["ops"].append({"op": "do"})
            continue
        m = re.match(r"TS_ASSERT_DELTA\(.*\[v\]\.Speed_GetRef\(\)\.Get\((\d)\)," + NUM + r",eps\);", s)
        if m:
            cur["ops"].append({"op": "expect", "key": list(v), "dim": int(m.group(1)), "value": float(m.group(2))})
            continue
        m = re.match(r"TS_ASSERT\((!?)std::isnan\(.*\[v\]\.Speed_GetRef\(\)\.Get\((\d)\)\)\);", s)
        if m:
            cur["ops"].append({"op": "nan", "key": list(v), "dim": int(m.group(2)), "isnan": m.group(1) == ""})
            continue
        if "TS_ASSERT" in s or "Speed_GetRef().Set" in s or "CellType_GetRef().Set" in s:
            raise ValueError(f"unparsed statement: {s}")
    return tests


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MAC_REF_ROOT", "/root/reference")
    with open(os.path.join(ref, "test", "test_Extrapolate_Boundary.h")) as f:
        tests = parse(f.read())
    n_assert = sum(1 for t in tests for o in t["ops"] if o["op"] in ("expect", "nan"))
    n_do = sum(1 for t in tests for o in t["ops"] if o["op"] == "do")
    out = {"source": "test/test_Extrapolate_Boundary.h", "dim": 2, "chunk": 2, "tests": tests,
           "asserts": n_assert, "runs": n_do}
    with open(os.path.join(HERE, "extrap_bc_2d.json"), "w") as f:
        json.dump(out, f, indent=0)
    print(f"{len(tests)} tests, {n_do} runs, {n_assert} asserts")


if __name__ == "__main__":
    main()

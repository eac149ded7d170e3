"""Write ``integrators.json``: the coefficient tables of the reference GPU
backend's symplectic integrators (the ``integrator`` argument of its
gpupass), read from atgpu/SymplecticIntegrator.cpp and evaluated as that
file's C++ does (IEEE double arithmetic, correctly rounded sqrt, the
Forest-Ruth constants of atintegrators/atconstants.h), stored as the hex
patterns of the doubles.

Usage: python tests/golden/make_golden_integrators.py [reference root]
"""
import json
import math
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def _constants(ref):
    src = open(os.path.join(ref, "atintegrators", "atconstants.h")).read()
    env = {"sqrt": math.sqrt}
    m = re.search(r"#define\s+THIRD_ROOT_2\s+([0-9.eE+-]+)", src)
    env["THIRD_ROOT_2"] = float(m.group(1))
    for name in ("DRIFT1", "DRIFT2", "KICK1", "KICK2"):
        m = re.search(r"const double\s+%s\s*=\s*([^;]+);" % name, src)
        env[name] = eval(m.group(1), {"__builtins__": {}}, env)
    return env


def main(ref):
    env = _constants(ref)
    src = open(os.path.join(ref, "atgpu", "SymplecticIntegrator.cpp")).read()
    body = src[src.index("switch (type)"):src.index("default:")]
    out = {}
    for m in re.finditer(r"case\s+(\d+):(.*?)break;", body, re.S):
        k = int(m.group(1))
        code = re.sub(r"//[^\n]*", "", m.group(2))
        n = int(re.search(r"allocate\((\d+)\)", code).group(1))
        c, d = [None] * n, [None] * n
        for arr, i, expr in re.findall(r"\b([cd])\[(\d+)\]\s*=\s*([^;]+);", code):
            v = eval(expr, {"__builtins__": {}}, env)
            (c if arr == "c" else d)[int(i)] = float(v)
        out[str(k)] = {"c": [v.hex() for v in c], "d": [v.hex() for v in d]}
    with open(os.path.join(HERE, "integrators.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", sorted(out))


if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from oracle.build_ref import _ref_root
    main(sys.argv[1] if len(sys.argv) > 1 else _ref_root())

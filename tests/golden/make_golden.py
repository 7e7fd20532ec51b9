"""Extract the reference's own known-answer vectors into small JSON fixtures.

Run in a container that has the reference source tree (read as text only):
    python tests/golden/make_golden.py /path/to/SpeckleSim
Writes tests/golden/hankel2_x2.json, tests/golden/hankel2_x2p2i.json,
tests/golden/gmres_tridiag.json and tests/golden/quadrature_tri.json.
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def fnum(s):
    return float(s.replace("_8", "").replace("d", "e").replace("D", "e"))


def hankel(ref, test="test_lib_math_bessel_spherical_third_kind_2_real"):
    path = os.path.join(ref, "src/lib/libmath/src/math/lib_math_bessel.f90")
    src = open(path).read().splitlines()
    start = next(i for i, l in enumerate(src) if "function " + test in l)
    end = next(i for i in range(start + 1, len(src)) if "end function " + test in src[i])
    vals = {}
    pat = re.compile(r"ground_truth_y\((\d+)\)\s*=\s*cmplx\(([^,]+),\s*([+-]?\s*[^,]+),\s*kind=8\)")
    for i in range(start, end):
        m = pat.search(src[i])
        if m:
            vals[int(m.group(1))] = (fnum(m.group(2).strip()), fnum(m.group(3).replace(" ", "")))
    x = None
    for i in range(start, end):
        m = re.search(r"double precision :: x = ([0-9.]+)", src[i])
        if m:
            x = float(m.group(1))
        m = re.search(r"complex\(kind=8\) :: x = cmplx\(([0-9.]+)_8, ([+-]?[0-9.]+)_8, kind=8\)", src[i])
        if m:
            x = [float(m.group(1)), float(m.group(2))]
    n = max(vals)
    return {
        "source": f"src/lib/libmath/src/math/lib_math_bessel.f90:{start + 1}-{end + 1} "
                  f"({test}; values from sageMath)",
        "x": x, "orders": list(range(n)),
        "re": [vals[i + 1][0] for i in range(n)], "im": [vals[i + 1][1] for i in range(n)],
        "tolerance_log": 1e-13,
    }


def gmres(ref):
    path = os.path.join(ref, "src/lib/libmath/src/math/lib_math_solver_GMRES.f90")
    src = open(path).read()
    assert "a(i,i) = dcmplx(4.d0, 0.d0)" in src and "dcmplx(-2.d0, 1.d0)" in src
    line = src[: src.index("subroutine GMRES_test")].count("\n") + 1
    return {
        "source": f"src/lib/libmath/src/math/lib_math_solver_GMRES.f90:{line} (GMRES_test)",
        "n": 100, "diag": [4.0, 0.0], "offdiag": [-2.0, 1.0], "restart": 60,
        "solution": "all ones", "rhs": "A @ ones",
    }


def quadrature(ref):
    """The triangle rules of Quadrature_tri as written in the source (decimal literals;
    the compiled reference holds them as binary32 values)."""
    path = os.path.join(ref, "src/lib_sie_integration_points.f90")
    lines = open(path).read().splitlines()
    start = next(i for i, l in enumerate(lines) if "subroutine Quadrature_tri" in l)
    end = next(i for i in range(start + 1, len(lines)) if lines[i].strip().startswith("end subroutine"))
    body = "\n".join(lines[start:end + 1])
    parts = re.split(r"if \(ngp == (\d+)\) then", body)
    rules = {}
    for k in range(1, len(parts), 2):
        n = int(parts[k])
        rule = {}
        for name in ("alpha", "beta", "ww"):
            m = re.search(name + r"\(1:ngp\)\s*=\s*&?\s*(?:\(/(.*?)/\)|([0-9.]+))", parts[k + 1], re.S)
            if m.group(1) is not None:
                vals = [float(v.replace("&", "").strip()) for v in m.group(1).split(",")]
            else:
                vals = [float(m.group(2))] * n
            assert len(vals) == n
            rule[name] = vals
        rules[str(n)] = rule
    return {
        "source": f"src/lib_sie_integration_points.f90:{start + 1}-{end + 1} (Quadrature_tri)",
        "rules": rules,
    }


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_golden.py <path of the SpeckleSim source tree>")
    ref = sys.argv[1]
    with open(os.path.join(HERE, "hankel2_x2.json"), "w") as f:
        json.dump(hankel(ref), f, indent=1)
    with open(os.path.join(HERE, "hankel2_x2p2i.json"), "w") as f:
        json.dump(hankel(ref, "test_lib_math_bessel_spherical_third_kind_2_cmplx"), f, indent=1)
    with open(os.path.join(HERE, "gmres_tridiag.json"), "w") as f:
        json.dump(gmres(ref), f, indent=1)
    with open(os.path.join(HERE, "quadrature_tri.json"), "w") as f:
        json.dump(quadrature(ref), f, indent=1)
    print("ok")

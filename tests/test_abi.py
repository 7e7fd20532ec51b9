"""The C-ABI library loads and exports every entry point of include/sie_gpu.h (CPU)."""
import ctypes as C
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "sie_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sie_[a-z0-9_]+)\s*\(", src)))


def test_exports_match_header(gpu_lib):
    from specklesim_b200 import _lib
    names = header_functions()
    assert set(names) == set(_lib.EXPORTS)
    for n in names:
        assert hasattr(gpu_lib, n), n


def test_defaults_and_incidence(gpu_lib):
    from specklesim_b200 import _lib
    cfg = _lib.SieConfig()
    gpu_lib.sie_config_default(C.byref(cfg))
    assert cfg.formulation == _lib.SIE_ICTF and cfg.ngp == 3 and cfg.tree_s_opt == 250
    assert cfg.truncation_number == 19
    k = np.zeros(3)
    e = np.zeros(3)
    # theta = 0, phi = 0, TM, against z: k = (0,0,-1), E = (1,0,0) (main.f90:246-295)
    assert gpu_lib.sie_incidence(0.0, 0.0, 1, 2, _lib.dptr(k), _lib.dptr(e)) == 0
    assert np.allclose(k, [0, 0, -1]) and np.allclose(e, [1, 0, 0])
    # the rotation of field_rotation_matrix keeps E transverse for k against z
    assert gpu_lib.sie_incidence(0.3, 0.7, 2, 2, _lib.dptr(k), _lib.dptr(e)) == 0
    assert abs(np.dot(k, e)) < 1e-15


def test_argument_errors_without_device(gpu_lib):
    from specklesim_b200 import _lib
    cfg = _lib.SieConfig()
    gpu_lib.sie_config_default(C.byref(cfg))
    h = C.c_void_p()
    v = np.zeros((3, 3))
    t = np.array([[0, 1, 5]], np.int32)
    # bad vertex index / too small mesh are rejected before any device work
    assert gpu_lib.sie_init(C.byref(cfg), _lib.dptr(v), 3, _lib.iptr(t), 1, C.byref(h)) == _lib.SIE_ERR_ARG
    cfg.ngp = 5
    t2 = np.array([[0, 1, 2], [0, 2, 1]], np.int32)
    assert gpu_lib.sie_init(C.byref(cfg), _lib.dptr(v), 3, _lib.iptr(t2), 2, C.byref(h)) == _lib.SIE_ERR_ARG
    assert b"ngp" in gpu_lib.sie_last_error()
    assert gpu_lib.sie_matvec(None, None, None, 1, 0) == _lib.SIE_ERR_ARG
    p = np.zeros(3)
    assert gpu_lib.sie_field_interior(None, _lib.dptr(p), _lib.dptr(p), 1, 2.25, 0.0, None, None) == _lib.SIE_ERR_ARG
    assert gpu_lib.sie_solve_direct_mixed(None, None, None, 1, 1e-10, 30, None) == _lib.SIE_ERR_ARG


def test_quadrature_rules_are_the_reference_tables(gpu_lib):
    """The library's triangle rules (host tables that the fill kernels copy) against the
    reference's Quadrature_tri literals, as binary32 values, bit for bit."""
    import json
    from specklesim_b200 import _lib
    g = json.load(open(os.path.join(ROOT, "tests", "golden", "quadrature_tri.json")))["rules"]
    a, b, w = np.zeros(12), np.zeros(12), np.zeros(12)
    n = C.c_int()
    f32 = lambda v: np.asarray(v, np.float32).astype(np.float64)
    for ngp, rule in g.items():
        assert gpu_lib.sie_quadrature_rule(int(ngp), _lib.dptr(a), _lib.dptr(b), _lib.dptr(w),
                                           C.byref(n)) == _lib.SIE_OK
        assert n.value == int(ngp)
        assert np.array_equal(a[:n.value], f32(rule["alpha"]))
        assert np.array_equal(b[:n.value], f32(rule["beta"]))
        assert np.array_equal(w[:n.value], f32(rule["ww"]))
    assert gpu_lib.sie_quadrature_rule(5, _lib.dptr(a), _lib.dptr(b), _lib.dptr(w),
                                       C.byref(n)) == _lib.SIE_ERR_ARG
    assert b"ngp" in gpu_lib.sie_last_error()


def test_incidence_matches_the_reference_rotation(gpu_lib):
    """sie_incidence against kin_and_Ein_calculation and
    field_rotation_conical_illumination (lib_sie_math.f90:228-293), restated here: k_in =
    (sin t cos p, sin t sin p, s cos t) with s = +1 / -1 for k_dir 1 / 2, and E_in = Rm
    (1, 0) for TM, Rm (0, 1) for TE, Rm the 3 x 2 rotation of that routine."""
    from specklesim_b200 import _lib
    k = np.zeros(3)
    e = np.zeros(3)
    for t in np.linspace(0.0, 1.4, 6):
        for p in np.linspace(-3.0, 3.0, 7):
            a, b, c, d = np.sin(t), np.cos(t), np.sin(p), np.cos(p)
            Rm = np.array([[d * d * b + c * c, c * d * (b - 1)],
                           [c * d * (b - 1), c * c * b + d * d],
                           [a * d, a * c]])
            for pol, e_t in ((1, [1.0, 0.0]), (2, [0.0, 1.0])):
                for k_dir, s in ((1, 1.0), (2, -1.0)):
                    assert gpu_lib.sie_incidence(t, p, pol, k_dir, _lib.dptr(k), _lib.dptr(e)) == 0
                    assert np.allclose(k, [a * d, a * c, s * b], rtol=0, atol=1e-15)
                    assert np.allclose(e, Rm @ e_t, rtol=0, atol=1e-15)


def _c_structs(src):
    """{name: [(type, field), ...]} of the header's typedef structs."""
    out = {}
    for body, name in re.findall(r"typedef struct \{(.*?)\}\s*(\w+);", src, re.S):
        fields = []
        for decl in re.sub(r"/\*.*?\*/", "", body, flags=re.S).split(";"):
            m = re.match(r"\s*(int|double)\s+(.+)", decl)
            if m:
                fields += [(m.group(1), f.strip()) for f in m.group(2).split(",")]
        out[name] = fields
    return out


def test_fortran_shim_matches_the_header():
    """The Fortran shim is not compiled here (no Fortran compiler), so check it against
    include/sie_gpu.h as text: every bind(C) type has the C struct's fields in the same
    order with the matching kinds, and every bound procedure names a declared function
    with the same number of arguments."""
    hdr = open(os.path.join(ROOT, "include", "sie_gpu.h")).read()
    shim = open(os.path.join(ROOT, "specklesim_b200", "fortran", "sie_shim.f90")).read()
    kinds = {"integer(c_int)": "int", "real(c_double)": "double"}
    structs = _c_structs(hdr)
    ftypes = re.findall(r"type, bind\(C\) :: (\w+)\n(.*?)end type", shim, re.S)
    assert {n for n, _ in ftypes} == {"sie_config", "sie_solver_cfg", "sie_stats"}
    for name, body in ftypes:
        fields = []
        for line in body.strip().splitlines():
            kind, names = line.split("::")
            fields += [(kinds[kind.strip()], f.strip()) for f in names.split(",")]
        assert fields == structs[name], name
    nocomment = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    bound = re.findall(r"(?:function|subroutine) (\w+)\(([^)]*)\)\s*bind\(C, name=\"(\w+)\"\)", shim)
    assert len(bound) >= 12
    for fname, args, cname in bound:
        assert fname == cname
        m = re.search(r"\b" + cname + r"\s*\(([^)]*)\)\s*;", nocomment)
        assert m, cname
        c_args = [a for a in m.group(1).split(",") if a.strip() and a.strip() != "void"]
        f_args = [a for a in args.split(",") if a.strip()]
        assert len(f_args) == len(c_args), cname


def test_fortran_gmres_shim_exports_the_reference_procedures():
    """sie_gmres_shim.f90 stands in for the reference's lib_sie_solver_gmres_interface: it
    declares the same module and the same public procedures
    (src/lib_sie_solver_gmres_interface.f90:27-29), and every library function it calls is
    bound in sie_shim.f90's interface block."""
    shim2 = open(os.path.join(ROOT, "specklesim_b200", "fortran", "sie_gmres_shim.f90")).read()
    shim = open(os.path.join(ROOT, "specklesim_b200", "fortran", "sie_shim.f90")).read()
    assert re.search(r"^module lib_sie_solver_gmres_interface$", shim2, re.M)
    public = set(re.findall(r"public :: (\w+)", shim2))
    assert public == {"run_ml_fmm_GMRES_tri", "lib_sie_solver_GMRES_run",
                      "prerun_ml_fmm_GMRES_tri_conical_planewaves"}
    for name in public:
        assert re.search(r"subroutine " + name + r"\(\)", shim2, re.I)
    bound = set(re.findall(r"bind\(C, name=\"(\w+)\"\)", shim))
    called = set(re.findall(r"\b(sie_\w+)\(", shim2)) - {"sie_check", "sie_shim_context"}
    assert called and called <= bound, called - bound


def test_fortran_shim_defines_its_public_procedures():
    """Every public procedure of sie_shim.f90's lib_sie_tri_mlfmm_interface is defined in
    the module, the reference's eight (src/lib_sie_tri_mlfmm_interface.f90:18-26) among
    them, and every library function the module calls is bound in the interface block
    (the direct solve's included)."""
    shim = open(os.path.join(ROOT, "specklesim_b200", "fortran", "sie_shim.f90")).read()
    body = shim[shim.index("module lib_sie_tri_mlfmm_interface"):]
    public = set(re.findall(r"public :: (\w+)", body))
    assert {"lib_sie_ml_fmm_calculate_vector_b_tri", "lib_sie_ml_fmm_get_vector_b_tri",
            "lib_sie_ml_fmm_get_init_vector_x_tri", "lib_sie_ml_fmm_precalculation_tri",
            "lib_sie_ml_fmm_run_tri", "lib_sie_ml_fmm_save_vector_x_tri",
            "run_MLFMM_one_forward_tri", "lib_sie_ml_fmm_preconditioner_left",
            "lib_sie_ml_fmm_solve_direct_tri"} <= public
    for name in public:
        assert re.search(r"(subroutine|function) " + name + r"\(", body), name
    bound = set(re.findall(r"bind\(C, name=\"(\w+)\"\)", shim))
    called = set(re.findall(r"\b(sie_\w+)\(", body)) - {"sie_check", "sie_shim_context"}
    assert {"sie_solve_direct", "sie_solve_direct_mixed"} <= called
    assert called <= bound, called - bound


def test_ctypes_structs_match_the_header():
    """The ctypes mirrors in specklesim_b200/_lib.py have the header structs' fields in
    order with matching types (Python's reserved 'lambda' is spelled 'lambda_')."""
    from specklesim_b200 import _lib
    structs = _c_structs(open(os.path.join(ROOT, "include", "sie_gpu.h")).read())
    ctype = {C.c_int: "int", C.c_double: "double"}
    for py, name in ((_lib.SieConfig, "sie_config"), (_lib.SieSolverCfg, "sie_solver_cfg"),
                     (_lib.SieStats, "sie_stats")):
        fields = [(ctype[t], f.rstrip("_")) for f, t in py._fields_]
        assert fields == structs[name], name


def test_missing_library_fails_loudly(tmp_path):
    """There is no CPU fallback: without libsiegpu.so the loader raises."""
    import pytest
    from specklesim_b200 import _lib
    with pytest.raises(_lib.SieError):
        _lib.load(str(tmp_path / "libsiegpu.so"))


def test_python_quadrature_rule(gpu_lib):
    import pytest
    from specklesim_b200 import SieError
    from specklesim_b200.sie import quadrature_rule
    a, b, w = quadrature_rule(12)
    assert len(a) == len(b) == len(w) == 12 and abs(w.sum() - 1.0) < 1e-6
    with pytest.raises(SieError):
        quadrature_rule(2)


def _fortran_blocks_balanced(src):
    """Every module, interface, derived type, procedure, DO and IF-THEN block of a free-form
    Fortran source is closed by the matching END (continuation lines joined, comments
    dropped); returns the first problem or None."""
    lines, buf = [], ""
    for raw in src.splitlines():
        line = raw.split("!")[0].rstrip()
        if buf:
            line, buf = buf + " " + line.strip(), ""
        if line.endswith("&"):
            buf = line[:-1]
            continue
        lines.append(line.strip().lower())
    stack = []
    for line in lines:
        if not line:
            continue
        m = re.match(r"^end\s*(subroutine|function|module|interface|type|do|if|select)?\b", line)
        if m and (line == "end" or m.group(1)):
            if not stack:
                return "unmatched " + line
            top = stack.pop()
            if m.group(1) and m.group(1) != top:
                return f"{top} closed by {line}"
            continue
        if line.startswith("module "):
            stack.append("module")
        elif line == "interface":
            stack.append("interface")
        elif re.match(r"^type\s*,|^type\s+\w", line):
            stack.append("type")
        elif re.search(r"\b(subroutine|function)\s+\w+\s*\(", line):
            stack.append("subroutine" if "subroutine" in line.split("(")[0] else "function")
        elif re.match(r"^do\b", line):
            stack.append("do")
        elif re.match(r"^if\s*\(.*\)\s*then$", line):
            stack.append("if")
    return f"left open: {stack}" if stack else None


def test_fortran_shims_have_balanced_blocks():
    """No Fortran compiler here: a structural check that each shim's blocks are closed."""
    for name in ("sie_shim.f90", "sie_gmres_shim.f90"):
        src = open(os.path.join(ROOT, "specklesim_b200", "fortran", name)).read()
        assert _fortran_blocks_balanced(src) is None, (name, _fortran_blocks_balanced(src))
    assert _fortran_blocks_balanced("module a\ncontains\nsubroutine b()\nend subroutine b\n") is not None

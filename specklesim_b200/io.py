"""Result files in the reference's formats, so downstream scripts read ours unchanged.

- Currents file (Result_SEH_*), written by lib_sie_solver_gmres_run
  (src/lib_sie_solver_gmres_interface.f90:164-170) and read back by
  lib_sie_ml_fmm_get_init_vector_x_tri (src/lib_sie_tri_mlfmm_interface.f90:215-222):
  two list-directed header lines ('n_el,' n_el and 'm_pairs' m_pairs), then the 2M
  coefficients one per line as real and imaginary part, each in Fortran es19.12 followed
  by 5 blanks (format '(201(es19.12, tr5))').
- Iteration log (iteration_error_*), written per GMRES step by zgmres_backward_error
  (:82-93): iteration as i10, 5 blanks, the Arnoldi backward error as es19.12, 5 blanks.
"""
import numpy as np


def fortran_es(v, w=19, d=12):
    """Fortran ESw.d: one nonzero digit before the point, d after, a signed exponent of at
    least two digits; a three-digit exponent drops the letter E, as Fortran does."""
    v = float(v)
    if v == 0.0:
        s = f"{0.0:.{d}f}E+00"
    else:
        m, e = f"{v:.{d}E}".split("E")
        ei = int(e)
        s = f"{m}E{ei:+03d}" if abs(ei) < 100 else f"{m}{ei:+04d}"
    return s.rjust(w)


def write_currents(path, n_el, x):
    """Currents file: x holds the 2M coefficients (J then M) in the reference order."""
    x = np.asarray(x, dtype=np.complex128).ravel()
    with open(path, "w") as f:
        f.write(f" n_el, {int(n_el):12d}\n")
        f.write(f" m_pairs {x.size // 2:12d}\n")
        for v in x:
            f.write(fortran_es(v.real) + "     " + fortran_es(v.imag) + "     \n")


def read_currents(path):
    """(n_el, m_pairs, x) from a currents file (list-directed reading, like the reference)."""
    with open(path) as f:
        n_el = int(f.readline().replace(",", " ").split()[-1])
        m_pairs = int(f.readline().split()[-1])
        vals = []
        for _ in range(2 * m_pairs):
            tok = f.readline().split()
            vals.append(complex(_fortran_float(tok[0]), _fortran_float(tok[1])))
    return n_el, m_pairs, np.array(vals)


def _fortran_float(t):
    t = t.upper()
    if "E" not in t:  # three-digit exponent written without the letter
        for i in range(len(t) - 1, 0, -1):
            if t[i] in "+-":
                t = t[:i] + "E" + t[i:]
                break
    return float(t)


def write_iteration_log(path, backward_errors, start=1):
    """Iteration log: one line per GMRES step with the Arnoldi backward error."""
    with open(path, "w") as f:
        for i, be in enumerate(backward_errors, start=start):
            f.write(f"{i:10d}     {fortran_es(be)}     \n")

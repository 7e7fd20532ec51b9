"""Result files in the reference's formats, so downstream scripts read ours unchanged.

- Currents file (Result_SEH_*), written by lib_sie_solver_gmres_run
  (src/lib_sie_solver_gmres_interface.f90:164-170) and read back by
  lib_sie_ml_fmm_get_init_vector_x_tri (src/lib_sie_tri_mlfmm_interface.f90:215-222):
  two list-directed header lines ('n_el,' n_el and 'm_pairs' m_pairs), then the 2M
  coefficients one per line as real and imaginary part, each in Fortran es19.12 followed
  by 5 blanks (format '(201(es19.12, tr5))').
- Iteration log (iteration_error_*), written per GMRES step by zgmres_backward_error
  (:82-93): iteration as i10, 5 blanks, the Arnoldi backward error as es19.12, 5 blanks.
- Run-parameters file (Calculation_parameters_*), written after the solve by
  lib_sie_solver_gmres_run (:171-197, sphere objects) and output_file_GMRES (:214-241,
  surface objects): one list-directed line per item, the reference's label text then
  the value.  Labels and their order are the reference's.  List-directed number layout
  is compiler-specific, so numbers are written as ES with 16 decimals (exact doubles),
  which every list-directed or float() reader takes; read_parameters splits each line
  at its first '='.
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


# The labels (with their padding) of Calculation_parameters_*, in the reference's order.
PARAMETER_LABELS = {
    # output_file_GMRES (src/lib_sie_solver_gmres_interface.f90:214-241)
    "surface": [
        "object_type =                  ", "formulation_type =             ",
        "illumination_type =            ", "beam_waist(nm) (Gaussian beam) =   ",
        "Wavelength (nm) =            ", "object number =             ",
        "object dimension I (nm) =   ", "object dimension II (nm) =  ",
        "object centroid (m) =       ", "N_el =                    ",
        "eps_r2 =                    ", "evaluation_type =        ",
        "evaluation_parameter%dim_c(nm) =   ", "evaluation_parameter%dim_a(nm) =   ",
        "evaluation_parameter%dim_b(nm) =   ", "illumination_p%theta_in =          ",
        "illumination_p%phi_in =          ", "Sphere sampling point =        ",
        "GMRES_time (min.) =               ", "Iteration procedure =          ",
        "convergence_tolerance =        ", "l_max =                        ",
        "dc at l_max =                  ", "tree_s_opt  =                  ",
        "m_pairs  =                  ",
    ],
    # lib_sie_solver_gmres_run, sphere objects (:171-197)
    "sphere": [
        "object_type =                  ", "formulation_type =             ",
        "illumination_type =            ", "beam_waist(nm) (Gaussian beam) =   ",
        "Wavelength (nm) =          ", "sphere number =            ",
        "Sphere diameter (nm) =     ", "Ndisc =                    ",
        "N_el =                    ", "Sphere centroid (m) =      ",
        "eps_r2 =                   ", "evaluation_type =        ",
        "evaluation_parameter%dim_c(nm) =   ", "evaluation_parameter%dim_a(nm) =   ",
        "evaluation_parameter%dim_b(nm) =   ", "illumination_p%theta_in =          ",
        "illumination_p%phi_in =          ", "m_pairs =                ",
        "Sphere sampling point =        ", "GMRES_time (min.) =               ",
        "Iteration procedure =          ", "convergence_tolerance =        ",
        "l_max =                        ", "dc at l_max =                  ",
        "tree_s_opt  =                  ",
    ],
}


def parameter_keys(object_type="surface"):
    """The item names of a run-parameters file: each label without its '=' and padding."""
    return [lab.split("=")[0].strip() for lab in PARAMETER_LABELS[object_type]]


def _list_directed(v):
    if isinstance(v, str):
        return v
    if isinstance(v, (bool, np.bool_)):
        return "T" if v else "F"
    if isinstance(v, (int, np.integer)):
        return f"{int(v):12d}"
    if isinstance(v, (complex, np.complexfloating)):
        return f" ({fortran_es(v.real, 23, 16).strip()},{fortran_es(v.imag, 23, 16).strip()})"
    if isinstance(v, (float, np.floating)):
        return fortran_es(v, 25, 16)
    return "".join(_list_directed(u) for u in v)


def write_parameters(path, values, object_type="surface"):
    """Run-parameters file.  values maps every name of parameter_keys(object_type) to a
    string, a number, a complex number or a sequence of numbers."""
    keys = parameter_keys(object_type)
    missing = [k for k in keys if k not in values]
    if missing:
        raise KeyError(f"write_parameters: missing {missing}")
    with open(path, "w") as f:
        for lab, k in zip(PARAMETER_LABELS[object_type], keys):
            f.write(" " + lab + _list_directed(values[k]) + "\n")


def read_parameters(path):
    """{name: value text} of a run-parameters file, in file order; parse_parameter turns a
    value text into numbers."""
    out = {}
    with open(path) as f:
        for line in f:
            if "=" in line:
                k, v = line.split("=", 1)
                out[k.strip()] = v.strip()
    return out


def parse_parameter(text):
    """A value text as an int, a float, a complex, a tuple of these, or the text itself."""
    toks = text.split()
    vals = []
    for t in toks:
        try:
            if t.startswith("(") and t.endswith(")"):
                re_, im_ = t[1:-1].split(",")
                vals.append(complex(_fortran_float(re_), _fortran_float(im_)))
            elif t.lstrip("+-").isdigit():
                vals.append(int(t))
            else:
                vals.append(_fortran_float(t))
        except ValueError:
            return text
    if not vals:
        return text
    return vals[0] if len(vals) == 1 else tuple(vals)

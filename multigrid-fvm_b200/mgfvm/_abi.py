"""ctypes mirror of include/mgfvm.h (struct layouts, enums, status codes).

The structs follow the reference's InputData fields one for one
(Version-6-26-04.c:27-39, README.md:6-69).
"""
import ctypes as C

MAX_PORTS = 10

# status codes (enum mgfvm_status)
OK, EINVAL, EIO, EOOB, ENONFINITE, ETIMEOUT, ECUDA, ENOMEM, EUNSUPPORTED = range(9)
STATUS_NAMES = {
    OK: "OK", EINVAL: "EINVAL", EIO: "EIO", EOOB: "EOOB", ENONFINITE: "ENONFINITE",
    ETIMEOUT: "ETIMEOUT", ECUDA: "ECUDA", ENOMEM: "ENOMEM", EUNSUPPORTED: "EUNSUPPORTED",
}

# fields (enum mgfvm_field), in struct SoA order
FIELDS = ["u", "v", "p", "pp", "sc", "su", "rs", "resu", "resv", "ressc", "c",
          "aw", "ae", "as", "an", "ap", "apu", "apv", "spu", "spv", "spsc",
          "cx", "cy", "areax", "areay"]
FIELD = {name: k for k, name in enumerate(FIELDS)}

# single-step ops (enum mgfvm_op)
OPS = ["fluxes", "solve_u", "solve_v", "solve_pp", "pbound", "outflow", "solve_sc",
       "restrict", "prolong", "smooth_u", "smooth_v", "smooth_pp", "smooth_sc"]
OP = {name: k for k, name in enumerate(OPS)}

JACOBI, GAUSS_SEIDEL = 1, 2
PREC_FP64, PREC_MIXED = 0, 1
DIR = {"none": 0, "inlet": 1, "amuf": 2, "prsc": 3}


class Config(C.Structure):
    """struct mgfvm_config: one case, everything InputData + pattern.txt hold."""
    _fields_ = [
        ("nfx", C.c_int), ("nfy", C.c_int), ("ngrid", C.c_int), ("ig_obs", C.c_int),
        ("ibeg_obs", C.c_int), ("ig_inlt", C.c_int), ("ig_outlt", C.c_int),
        ("nvcycle", C.c_int), ("nswpm", C.c_int), ("nswpp", C.c_int), ("isolve", C.c_int),
        ("omega", C.c_double), ("convergence", C.c_double),
        ("xl", C.c_double), ("yl", C.c_double), ("amuf", C.c_double), ("prsc", C.c_double),
        ("relxm", C.c_double), ("relxp", C.c_double),
        ("ibc_xm", C.c_int), ("ibc_xp", C.c_int), ("ibc_ym", C.c_int), ("ibc_yp", C.c_int),
        ("u_xm", C.c_double), ("v_xm", C.c_double), ("p_xm", C.c_double), ("sc_xm", C.c_double),
        ("u_xp", C.c_double), ("v_xp", C.c_double), ("p_xp", C.c_double), ("sc_xp", C.c_double),
        ("u_ym", C.c_double), ("v_ym", C.c_double), ("p_ym", C.c_double), ("sc_ym", C.c_double),
        ("u_yp", C.c_double), ("v_yp", C.c_double), ("p_yp", C.c_double), ("sc_yp", C.c_double),
        ("u_guess", C.c_double), ("v_guess", C.c_double), ("p_guess", C.c_double),
        ("sc_guess", C.c_double),
        ("sc_obs", C.c_double),
        ("ninlt", C.c_int),
        ("jfinlt", C.c_int * MAX_PORTS), ("jlinlt", C.c_int * MAX_PORTS),
        ("uinlt", C.c_double * MAX_PORTS), ("vinlt", C.c_double * MAX_PORTS),
        ("scinlt", C.c_double * MAX_PORTS),
        ("noutlt", C.c_int),
        ("jfoutlt", C.c_int * MAX_PORTS), ("jloutlt", C.c_int * MAX_PORTS),
        ("uoutlt", C.c_double * MAX_PORTS), ("voutlt", C.c_double * MAX_PORTS),
        ("scoutlt", C.c_double * MAX_PORTS),
        ("nobs", C.c_int),
        ("obs", C.POINTER(C.c_int)),
        ("dpdxm", C.c_double), ("dpdym", C.c_double),
    ]


class Options(C.Structure):
    """struct mgfvm_options."""
    _fields_ = [("device", C.c_int), ("precision", C.c_int), ("tail_level", C.c_int),
                ("use_graph", C.c_int), ("sync_every", C.c_int), ("tangent", C.c_int)]


MAX_LEVELS = 16


class Tuning(C.Structure):
    """struct mgfvm_tuning: per-level schedule choices (0 = default)."""
    _fields_ = [("smooth_units", C.c_int * MAX_LEVELS), ("smooth_threads", C.c_int * MAX_LEVELS),
                ("asm_slices", C.c_int * MAX_LEVELS), ("restrict_slices", C.c_int * MAX_LEVELS),
                ("update_pfix", C.c_int * MAX_LEVELS), ("odd_chunks", C.c_int * MAX_LEVELS),
                ("pp_level", C.c_int * MAX_LEVELS), ("smooth_tma", C.c_int * MAX_LEVELS),
                ("coarse_kernel", C.c_int * MAX_LEVELS), ("prol_fused", C.c_int * MAX_LEVELS),
                ("tma_first_wait", C.c_int), ("pdl", C.c_int), ("band_visit", C.c_int * MAX_LEVELS),
                ("coarse_cluster", C.c_int)]

    def as_dict(self):
        return {k: (list(v) if isinstance(v := getattr(self, k), C.Array) else v) for k, _ in self._fields_}

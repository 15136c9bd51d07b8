"""Run the mechanically translated reference -- TEST INFRASTRUCTURE ONLY.

oracle/_ref/libref.so is built from the reference's Fortran sources by
oracle/f2c_ref.py (see `build()`); the reference directory is needed only to
build it.  A run writes the cloud in the reference's own input formats
("3d_input_data": idx status x y z tan1 tan2 nor nbhs conn min_dist, per
point_preprocessor.f90:30-36; "stored-solution.dat": x y z rho u1 u2 u3 p, per
initial_conditions.f90:26) and lets the translated program read them, then
calls its setup routines and fpi_solver(t) like meshfree_solver.f90:20-33.
The library holds one cloud at a time; every run starts from scratch.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# Where the reference's Fortran sources lie; the translation is rebuilt only
# when this is set (elsewhere the prebuilt libraries under _ref/ are used).
REF_DIR_ENV = "MFCFD_REFERENCE_DIR"
_LIBS = {"glibc": os.path.join(_HERE, "_ref", "libref.so"),
         "mfmath": os.path.join(_HERE, "_ref", "libref_mfmath.so"),
         # the reference's alternative module sources (f2c_ref.VARIANTS), glibc
         "explicit": os.path.join(_HERE, "_ref", "libref_explicit.so"),
         "backup": os.path.join(_HERE, "_ref", "libref_backup.so")}
_lib = None
_lib_kind = None


def reference_dir():
    """The reference checkout named by $MFCFD_REFERENCE_DIR, or None."""
    d = os.environ.get(REF_DIR_ENV)
    return d if d and os.path.isdir(d) else None


def build(reference_dir: str = None) -> bool:
    """Translate and compile two builds: with glibc's exp/log/erf (what the
    Fortran reference calls) and with the solver's mfmath.h functions.
    reference_dir defaults to $MFCFD_REFERENCE_DIR.  Returns False when the
    reference is absent and nothing was built before."""
    if reference_dir is None:
        reference_dir = os.environ.get(REF_DIR_ENV, "")
    if not reference_dir or not os.path.isdir(reference_dir):
        return all(os.path.exists(p) for p in _LIBS.values())
    out_c = os.path.join(_HERE, "_ref", "ref_translated.c")
    subprocess.run(["python", os.path.join(_HERE, "f2c_ref.py"), reference_dir, out_c],
                   check=True, stdout=subprocess.DEVNULL)
    common = ["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-w"]
    subprocess.run(common + ["-o", _LIBS["glibc"], out_c, os.path.join(_HERE, "ref_runtime.c"),
                             "-lm"], check=True)
    shim = os.path.join(_HERE, "ref_mfmath_shim.h")
    subprocess.run(common + ["-include", shim, "-o", _LIBS["mfmath"], out_c,
                             os.path.join(_HERE, "ref_runtime.c"), "-lm"], check=True)
    for variant in ("explicit", "backup"):
        out_v = os.path.join(_HERE, "_ref", f"ref_translated_{variant}.c")
        subprocess.run(["python", os.path.join(_HERE, "f2c_ref.py"), reference_dir, out_v, variant],
                       check=True, stdout=subprocess.DEVNULL)
        subprocess.run(common + ["-o", _LIBS[variant], out_v, os.path.join(_HERE, "ref_runtime.c"), "-lm"],
                       check=True)
    return True


def available(kind: str = "glibc") -> bool:
    return os.path.exists(_LIBS[kind])


def lib(kind: str = None):
    """One build per process: the translated program keeps global state.
    kind None means the build already loaded (glibc if none was)."""
    global _lib, _lib_kind
    if kind is None:
        kind = _lib_kind or "glibc"
    if _lib is not None and _lib_kind != kind:
        raise RuntimeError("only one translated-reference build can be used per process")
    if _lib is None:
        _lib_kind = kind
        L = ctypes.CDLL(_LIBS[kind])
        L.ref_register_file.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
        L.ref_set_param.argtypes = [ctypes.c_char_p, ctypes.c_double]
        L.ref_call.argtypes = [ctypes.c_char_p]
        L.ref_fpi_solver.argtypes = [ctypes.c_int]
        L.ref_array.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_long)]
        L.ref_array.restype = ctypes.c_void_p
        L.ref_scalar.argtypes = [ctypes.c_char_p]
        L.ref_scalar.restype = ctypes.c_double
        _lib = L
    return _lib


def input_text(cloud) -> str:
    """The reference's 3d_input_data for a cloud (point_preprocessor.f90:31-35)."""
    lines = []
    for k in range(cloud.n):
        nb = int(cloud.nbhs[k])
        vals = [str(k + 1), str(int(cloud.status[k])),
                repr(float(cloud.x[k])), repr(float(cloud.y[k])), repr(float(cloud.z[k]))]
        vals += [repr(float(v)) for v in cloud.tan1[k]]
        vals += [repr(float(v)) for v in cloud.tan2[k]]
        vals += [repr(float(v)) for v in cloud.nor[k]]
        vals.append(str(nb))
        vals += [str(int(v)) for v in cloud.conn[k, :nb]]
        vals.append(repr(float(cloud.min_dist[k])))
        lines.append(" ".join(vals))
    return "\n".join(lines) + "\n"


def solution_text(cloud, prim) -> str:
    """stored-solution.dat: x y z rho u1 u2 u3 p per point (initial_conditions.f90:26)."""
    rows = []
    for k in range(cloud.n):
        vals = [cloud.x[k], cloud.y[k], cloud.z[k]] + list(prim[k])
        rows.append(" ".join(repr(float(v)) for v in vals))
    return "\n".join(rows) + "\n"


class TranslatedReference:
    FIELDS = {"prim": 5, "u": 5, "q": 5, "qm": 10, "dq": 15, "delt": 1, "flux_res": 5,
              "delup": 5, "delun": 5}

    def __init__(self, cloud, prim0, mach, aoa_deg, libm="glibc", inner_iterations=0, power=0.0):
        L = lib(libm)
        L.ref_free_all()
        L.ref_register_file(b"3d_input_data", input_text(cloud).encode())
        L.ref_register_file(b"stored-solution.dat", solution_text(cloud, prim0).encode())
        L.ref_set_param(b"max_points", float(cloud.n))
        L.ref_set_param(b"mach", float(mach))
        L.ref_set_param(b"aoa", float(aoa_deg))
        # overrides persist in the library: set every one on each construction
        L.ref_set_param(b"inner_iterations", float(inner_iterations))
        L.ref_set_param(b"power", float(power))
        L.ref_init_parameters()
        for name in (b"allocate_size", b"read_input_point_data", b"initial_conditions",
                     b"generate_split_stencils", b"aliasing"):
            L.ref_call(name)
        self.n = cloud.n

    def step(self, t):
        L = lib()
        L.ref_fpi_solver(int(t))
        return L.ref_scalar(b"res_new"), L.ref_scalar(b"residue")

    def array(self, name, dtype=np.float64):
        dims = (ctypes.c_long * 3)()
        p = lib().ref_array(name.encode(), dims)
        if not p:
            raise KeyError(name)
        w = self.FIELDS.get(name, 1)
        ctype = ctypes.c_double if dtype == np.float64 else ctypes.c_int
        buf = (ctype * (w * self.n)).from_address(p)
        a = np.ctypeslib.as_array(buf).copy()
        return a.reshape(self.n, w) if w > 1 else a

    def get(self, name):
        return self.array(name)

    def alias(self):
        return (self.array("alias", np.int32), self.array("point_with_alias", np.int32))

"""ctypes binding of the CPU checker libraries.  TEST INFRASTRUCTURE ONLY.

``Oracle`` wraps liblicom_oracle.so (the FP64 restatement in licom_oracle.cpp);
``Reference`` wraps oracle/_ref/libref_tracer.so, the reference's own
tracer.cpp, convadj.cpp and icesnow.cpp compiled for the CPU (present only
where the reference tree was available at build time).  Field ids are those
of include/licom_tracer.h.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liblicom_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_tracer.so")
REF_READYC_LIB = os.path.join(HERE, "_ref", "libref_readyc.so")

FIELDS = ["AT", "ATB", "UTF", "VTF", "UTL", "VTL", "H0F", "H0L", "AKT", "WS", "NET", "UTF_OUT", "VTF_OUT",
          "H0F_OUT", "SWV", "NSWV", "SST", "SSS", "FRESH", "SEAICE", "TAREA", "TAREA_R", "HTW", "HTS", "HUN", "HUE",
          "DXU", "DYU", "AHF", "DTN", "DTS", "DTE", "DTW", "OHBT", "OHBU", "AU0", "AUS", "AUW", "AUSW", "KMT", "KMU",
          "KMTN", "KMTS", "KMTE", "KMTW", "DZP", "ODZP", "ODZT", "PEN", "TO", "SO", "C", "RESTORE", "AX", "AY", "AZ",
          "DZ", "TEND", "DT_DIFF", "DT_CONV", "PENETRATE", "QICE", "RIT", "RICDTTMS", "S2T", "RICT", "PDENSITY",
          "FZ_TIDE", "BUOYTUR", "BUOYSOL", "FCORT", "WAVE_DIS", "ZKP", "AKMT", "AK_TIDE", "AMLD", "RICHARDSON",
          "FZTIDAL", "WP3_TIDAL", "UP", "VP", "DLU", "DLV", "WKA_DRAG", "DUC", "DUM", "DUN", "DUS", "DUE", "DUW",
          "DMC", "DMN", "DMS", "DME", "DMW", "AMF", "UAREA_R", "DXUR", "DYUR"]
FID = {n: i for i, n in enumerate(FIELDS)}
INT = {"KMT", "KMU", "KMTN", "KMTS", "KMTE", "KMTW"}


def shape_of(name, nx, ny, km):
    imt, jmt = nx + 4, ny + 4
    if name in ("AT", "AKT", "RESTORE", "AX", "AY", "AZ", "DZ", "TEND", "DT_DIFF", "DT_CONV"):
        return (2, km, jmt, imt)
    if name == "ATB":
        return (2, km + 1, jmt, imt)
    if name in ("UTF", "VTF", "UTL", "VTL", "UTF_OUT", "VTF_OUT", "PENETRATE", "FZ_TIDE", "AKMT", "AK_TIDE",
                "RICHARDSON", "FZTIDAL", "WP3_TIDAL", "UP", "VP", "DLU", "DLV", "WKA_DRAG"):
        return (km, jmt, imt)
    if name in ("RIT", "RICDTTMS", "S2T", "RICT"):
        return (km - 1, jmt, imt)
    if name == "ZKP":
        return (km + 1,)
    if name in ("WS", "PDENSITY"):
        return (km + 1, jmt, imt)
    if name == "NET":
        return (2, jmt, imt)
    if name in ("DZP", "ODZP", "ODZT", "PEN", "TO", "SO"):
        return (km,)
    if name == "C":
        return (9, km)
    return (jmt, imt)


def _dtype(name):
    return np.int32 if name in INT else np.float64


class Oracle:
    def __init__(self, nx, ny, km, params, ew_cyclic=1, tripole=1, threads=0):
        self.lib = lib = C.CDLL(ORACLE_LIB)
        lib.or_create.restype = C.c_void_p
        lib.or_create.argtypes = [C.c_int] * 3
        for fn in ("or_destroy", "or_tracer_call", "or_convadj"):
            getattr(lib, fn).argtypes = [C.c_void_p]
        lib.or_set_params.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        lib.or_set_field.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]
        lib.or_get_field.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]
        lib.or_step.argtypes = [C.c_void_p, C.c_int]
        lib.or_fw_norm2.argtypes = [C.c_void_p]
        lib.or_fw_norm2.restype = C.c_double
        lib.or_tracer_content.argtypes = [C.c_void_p, C.c_void_p]
        lib.or_halo.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        lib.or_set_threads.argtypes = [C.c_int]
        lib.or_set_sum_order.argtypes = [C.c_void_p, C.c_int]
        lib.or_icesnow.argtypes = [C.c_void_p, C.c_void_p]
        lib.or_turb.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double]
        lib.or_hdiffu_del4.argtypes = [C.c_void_p, C.c_double, C.c_double]
        self.nx, self.ny, self.km = nx, ny, km
        self.h = C.c_void_p(lib.or_create(nx, ny, km))
        if not self.h:
            raise ValueError("oracle: bad sizes")
        self._params = params
        lib.or_set_params(self.h, C.byref(params), int(ew_cyclic), int(tripole))
        if threads:
            lib.or_set_threads(threads)

    def __del__(self):
        try:
            self.lib.or_destroy(self.h)
        except Exception:
            pass

    def set(self, name, a):
        a = np.ascontiguousarray(a, dtype=_dtype(name))
        assert a.size == int(np.prod(shape_of(name, self.nx, self.ny, self.km))), name
        if self.lib.or_set_field(self.h, FID[name], a.ctypes.data, a.nbytes):
            raise ValueError("oracle set " + name)

    def get(self, name):
        a = np.empty(shape_of(name, self.nx, self.ny, self.km), dtype=_dtype(name))
        if self.lib.or_get_field(self.h, FID[name], a.ctypes.data, a.nbytes):
            raise ValueError("oracle get " + name)
        return a

    def load(self, inputs):
        for n, a in inputs.items():
            self.set(n, a)

    def step(self, nsteps=1):
        self.lib.or_step(self.h, nsteps)

    def tracer_call(self):
        self.lib.or_tracer_call(self.h)

    def convadj(self):
        self.lib.or_convadj(self.h)

    def turb(self, tables, ncc, dfricmx):
        """tables: an lt_turb_tables structure (TurbTablesStruct)."""
        if self.lib.or_turb(self.h, C.byref(tables), int(ncc), float(dfricmx)):
            raise ValueError("oracle turb")

    def hdiffu_del4(self, am, c0f):
        if self.lib.or_hdiffu_del4(self.h, float(am), float(c0f)):
            raise ValueError("oracle hdiffu_del4")

    def icesnow(self, params):
        """params: an object with the lt_icesnow_params layout (IcesnowParams)."""
        if self.lib.or_icesnow(self.h, C.byref(params)):
            raise ValueError("oracle icesnow")

    def fw_norm2(self):
        return self.lib.or_fw_norm2(self.h)

    def tracer_content(self):
        out = (C.c_double * 2)()
        self.lib.or_tracer_content(self.h, out)
        return tuple(out)

    def sum_order(self, tree):
        """0: the reference's sequential SSS-norm sum; 1: the device's fixed tree."""
        self.lib.or_set_sum_order(self.h, int(tree))

    def halo(self, a, ew_cyclic=1, tripole=1):
        a = np.ascontiguousarray(a, dtype=np.float64).copy()
        jmt, imt = a.shape[-2], a.shape[-1]
        nz = a.size // (jmt * imt)
        self.lib.or_halo(a.ctypes.data, nz, imt, jmt, int(ew_cyclic), int(tripole))
        return a


def reference_available():
    return os.path.exists(REF_LIB)


class Reference:
    """The reference's own tracer_/convadj_ compiled for the CPU at its built-in
    block size (imt=40, jmt=44, km=55)."""

    def __init__(self, params, ew_cyclic=1, tripole=1):
        self.lib = lib = C.CDLL(REF_LIB)
        lib.ref_set_field.argtypes = [C.c_int, C.c_void_p, C.c_size_t]
        lib.ref_get_field.argtypes = [C.c_int, C.c_void_p, C.c_size_t]
        lib.ref_set_params.argtypes = [C.c_void_p, C.c_int, C.c_int]
        lib.ref_tracer_call.argtypes = [C.c_int]
        lib.ref_icesnow_call.argtypes = [C.c_double, C.c_double, C.c_int]
        lib.ref_fw_norm2.restype = C.c_double
        imt, jmt, km = C.c_int(), C.c_int(), C.c_int()
        lib.ref_dims(C.byref(imt), C.byref(jmt), C.byref(km))
        self.nx, self.ny, self.km = imt.value - 4, jmt.value - 4, km.value
        self._params = params
        lib.ref_set_params(C.byref(params), int(ew_cyclic), int(tripole))

    def set(self, name, a):
        a = np.ascontiguousarray(a, dtype=_dtype(name))
        if self.lib.ref_set_field(FID[name], a.ctypes.data, a.nbytes):
            raise ValueError("reference set " + name)

    def get(self, name):
        a = np.empty(shape_of(name, self.nx, self.ny, self.km), dtype=_dtype(name))
        if self.lib.ref_get_field(FID[name], a.ctypes.data, a.nbytes):
            raise ValueError("reference get " + name)
        return a

    def load(self, inputs):
        for n, a in inputs.items():
            self.set(n, a)

    def tracer_call(self, ii=0):
        self.lib.ref_tracer_call(ii)

    def convadj(self):
        self.lib.ref_convadj_call()

    def icesnow(self, tbice=-1.8, cp=3996.0, frc_core=1):
        """icesnow_ as the reference is configured (frc_core 1: licomqice
        zeroed first) or its build without FRC_CORE (0)."""
        self.lib.ref_icesnow_call(float(tbice), float(cp), int(frc_core))

    def fw_norm2(self):
        return self.lib.ref_fw_norm2()


def reference_readyc_available():
    return os.path.exists(REF_READYC_LIB)


class ReferenceReadyc:
    """Kernels of the reference's own readyc.cpp (turb_cu and the momentum
    biharmonic friction) compiled for the CPU at its built-in block size
    (imt=40, jmt=44, km=55)."""

    NAMES = ("AT", "AKT", "RIT", "RICDTTMS", "S2T", "RICT", "PDENSITY", "FZ_TIDE", "AKMT", "AK_TIDE", "RICHARDSON",
             "FZTIDAL", "WP3_TIDAL", "BUOYTUR", "BUOYSOL", "FCORT", "WAVE_DIS", "AMLD", "DZP", "ZKP", "KMT", "KMU",
             "UP", "VP", "DLU", "DLV", "WKA_DRAG", "HTW", "HTS", "TAREA_R", "DXU", "DYU", "DXUR", "DYUR", "UAREA_R",
             "DUC", "DUM", "DUN", "DUS", "DUE", "DUW", "DMC", "DMN", "DMS", "DME", "DMW", "AMF")

    def __init__(self):
        self.lib = lib = C.CDLL(REF_READYC_LIB)
        lib.ref_turb_set.argtypes = [C.c_char_p, C.c_void_p, C.c_size_t]
        lib.ref_turb_get.argtypes = [C.c_char_p, C.c_void_p, C.c_size_t]
        lib.ref_turb_set_tables.argtypes = [C.c_void_p]
        lib.ref_turb_call.argtypes = [C.c_int, C.c_double, C.c_double]
        lib.ref_del4u_call.argtypes = [C.c_double, C.c_double]
        imt, jmt, km = C.c_int(), C.c_int(), C.c_int()
        lib.ref_turb_dims(C.byref(imt), C.byref(jmt), C.byref(km))
        self.nx, self.ny, self.km = imt.value - 4, jmt.value - 4, km.value

    def set(self, name, a):
        a = np.ascontiguousarray(a, dtype=_dtype(name))
        if self.lib.ref_turb_set(name.encode(), a.ctypes.data, a.nbytes):
            raise ValueError("reference turb set " + name)

    def get(self, name):
        a = np.empty(shape_of(name, self.nx, self.ny, self.km), dtype=_dtype(name))
        if self.lib.ref_turb_get(name.encode(), a.ctypes.data, a.nbytes):
            raise ValueError("reference turb get " + name)
        return a

    def load(self, inputs):
        for n in self.NAMES:
            if n in inputs:
                self.set(n, inputs[n])

    def set_tables(self, tables):
        self._tables = tables          # the reference reads them where they lie
        self.lib.ref_turb_set_tables(C.byref(tables))

    def call(self, ncc, dfricmx, dwndmix):
        """turb_cu with readyc_'s memsets before it."""
        self.lib.ref_turb_call(int(ncc), float(dfricmx), float(dwndmix))

    def del4u(self, am, c0f):
        """readyc_'s momentum biharmonic friction sequence."""
        self.lib.ref_del4u_call(float(am), float(c0f))

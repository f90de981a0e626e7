"""ctypes binding of the CPU checker libraries.  TEST INFRASTRUCTURE ONLY.

``Oracle`` wraps liblicom_oracle.so (the FP64 restatement in licom_oracle.cpp);
``HostSynth`` wraps liblicom_synth_host.so, the seeded input generator built
for the host alone (the CPU baseline uses it so that it never loads the CUDA
library);
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
SYNTH_HOST_LIB = os.path.join(HERE, "liblicom_synth_host.so")

FIELDS = ["AT", "ATB", "UTF", "VTF", "UTL", "VTL", "H0F", "H0L", "AKT", "WS", "NET", "UTF_OUT", "VTF_OUT",
          "H0F_OUT", "SWV", "NSWV", "SST", "SSS", "FRESH", "SEAICE", "TAREA", "TAREA_R", "HTW", "HTS", "HUN", "HUE",
          "DXU", "DYU", "AHF", "DTN", "DTS", "DTE", "DTW", "OHBT", "OHBU", "AU0", "AUS", "AUW", "AUSW", "KMT", "KMU",
          "KMTN", "KMTS", "KMTE", "KMTW", "DZP", "ODZP", "ODZT", "PEN", "TO", "SO", "C", "RESTORE", "AX", "AY", "AZ",
          "DZ", "TEND", "DT_DIFF", "DT_CONV", "PENETRATE", "QICE", "RIT", "RICDTTMS", "S2T", "RICT", "PDENSITY",
          "FZ_TIDE", "BUOYTUR", "BUOYSOL", "FCORT", "WAVE_DIS", "ZKP", "AKMT", "AK_TIDE", "AMLD", "RICHARDSON",
          "FZTIDAL", "WP3_TIDAL", "UP", "VP", "DLU", "DLV", "WKA_DRAG", "DUC", "DUM", "DUN", "DUS", "DUE", "DUW",
          "DMC", "DMN", "DMS", "DME", "DMW", "AMF", "UAREA_R", "DXUR", "DYUR", "RESTORE_AT", "DT_RESTORE"]
FID = {n: i for i, n in enumerate(FIELDS)}
INT = {"KMT", "KMU", "KMTN", "KMTS", "KMTE", "KMTW"}


def shape_of(name, nx, ny, km):
    imt, jmt = nx + 4, ny + 4
    if name in ("AT", "AKT", "RESTORE", "AX", "AY", "AZ", "DZ", "TEND", "DT_DIFF", "DT_CONV", "RESTORE_AT",
                "DT_RESTORE"):
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


class Params(C.Structure):
    """lt_params (include/licom_tracer.h)."""
    _fields_ = [(n, C.c_double) for n in ("dts", "oncc", "onbc", "dwndmix", "gamma", "od0", "od0cp", "ah", "area_t")] + [
        ("nss", C.c_int), ("boundary_restore", C.c_int), ("adv_tracer", C.c_int), ("simple_assm", C.c_int),
        ("ktv", C.c_int)]


class SynthConfig(C.Structure):
    """lt_synth_config (include/licom_synth.h)."""
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("km", C.c_int), ("lat_s", C.c_double), ("lat_n", C.c_double),
                ("dz_top", C.c_double), ("dz_bot", C.c_double), ("depth", C.c_double), ("umax", C.c_double),
                ("seed", C.c_uint64), ("forced", C.c_int), ("cap_north", C.c_int), ("cap_south", C.c_int),
                ("ew_cyclic", C.c_int), ("tripole", C.c_int), ("land_frac", C.c_double), ("member", C.c_uint32),
                ("tpert", C.c_double), ("ah_bihar", C.c_double), ("hypsometry", C.c_int)]


class HostSynth:
    """The seeded synthetic domain of the benchmark configurations, generated
    on the host (OpenMP) without the CUDA library."""

    def __init__(self, nx, ny, km, **kw):
        self.lib = lib = C.CDLL(SYNTH_HOST_LIB)
        lib.lt_synth_defaults.argtypes = [C.c_void_p]
        lib.lt_synth_build.argtypes = [C.c_void_p, C.c_void_p]
        lib.lt_synth_free.argtypes = [C.c_void_p]
        lib.lt_synth_params.argtypes = [C.c_void_p, C.c_void_p]
        lib.lt_synth_field_rows.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_size_t]
        cfg = SynthConfig()
        lib.lt_synth_defaults(C.byref(cfg))
        cfg.nx, cfg.ny, cfg.km = nx, ny, km
        for k, v in kw.items():
            setattr(cfg, k, v)
        self.cfg = cfg
        self.h = C.c_void_p()
        if lib.lt_synth_build(C.byref(cfg), C.byref(self.h)):
            raise ValueError("lt_synth_build")
        self.params = Params()
        lib.lt_synth_params(self.h, C.byref(self.params))
        self.nx, self.ny, self.km = nx, ny, km

    def __del__(self):
        try:
            self.lib.lt_synth_free(self.h)
        except Exception:
            pass

    def fill(self, oracle, rows=None):
        """Write every input field of the oracle in place: the whole domain,
        or (rows) its northern band of that many rows, halo included, for an
        oracle of ny = rows - 4."""
        rows = rows or self.ny + 4
        assert oracle.nx == self.nx and oracle.km == self.km and oracle.ny + 4 == rows
        for name in INPUTS:
            n = int(np.prod(shape_of(name, oracle.nx, oracle.ny, oracle.km)))
            nbytes = n * (4 if name in INT else 8)
            if self.lib.lt_synth_field_rows(self.h, FID[name], rows, oracle.field_ptr(name), nbytes):
                raise ValueError("lt_synth_field_rows " + name)


# inputs of the tracer step (the generator leaves the others zero)
INPUTS = ["AT", "ATB", "UTF", "VTF", "UTL", "VTL", "H0F", "H0L", "AKT", "SWV", "NSWV", "SST", "SSS", "FRESH",
          "SEAICE", "TAREA", "TAREA_R", "HTW", "HTS", "HUN", "HUE", "DXU", "DYU", "AHF", "DTN", "DTS", "DTE", "DTW",
          "OHBT", "OHBU", "AU0", "AUS", "AUW", "AUSW", "KMT", "KMU", "KMTN", "KMTS", "KMTE", "KMTW", "DZP", "ODZP",
          "ODZT", "PEN", "TO", "SO", "C"]


class Oracle:
    def __init__(self, nx, ny, km, params, ew_cyclic=1, tripole=1, threads=0, diagnostics=1):
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
        lib.or_step_timed.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        lib.or_set_diagnostics.argtypes = [C.c_void_p, C.c_int]
        lib.or_field_ptr.argtypes = [C.c_void_p, C.c_int]
        lib.or_field_ptr.restype = C.c_void_p
        self.nx, self.ny, self.km = nx, ny, km
        self.h = C.c_void_p(lib.or_create(nx, ny, km))
        if not self.h:
            raise ValueError("oracle: bad sizes")
        self._params = params
        self._boundaries = (int(ew_cyclic), int(tripole))
        lib.or_set_params(self.h, C.byref(params), int(ew_cyclic), int(tripole))
        if threads:
            lib.or_set_threads(threads)
        if not diagnostics:
            lib.or_set_diagnostics(self.h, 0)

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

    def set_params(self, params):
        self._params = params
        self.lib.or_set_params(self.h, C.byref(params), *self._boundaries)

    def step(self, nsteps=1):
        self.lib.or_step(self.h, nsteps)

    def tracer_call(self):
        self.lib.or_tracer_call(self.h)

    def step_timed(self, nsteps=1):
        """step(); returns the seconds spent inside the tracer_ calls."""
        t = C.c_double()
        self.lib.or_step_timed(self.h, nsteps, C.byref(t))
        return t.value

    def field_ptr(self, name):
        return self.lib.or_field_ptr(self.h, FID[name])

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


def oracle_tracer7(params, n, tf, vit, atb, restore, restore_at, dt_restore):
    """The oracle's restatement of tracer_7 alone (tf and dt_restore updated in
    place): tf, vit [km][jmt][imt]; atb [2][km+1][jmt][imt]; restore,
    restore_at, dt_restore [2][km][jmt][imt]."""
    lib = C.CDLL(ORACLE_LIB)
    lib.or_tracer7.argtypes = [C.c_void_p] + [C.c_int] * 4 + [C.c_void_p] * 6
    km, jmt, imt = tf.shape
    lib.or_tracer7(C.byref(params), int(n), imt, jmt, km, tf.ctypes.data, vit.ctypes.data, atb.ctypes.data,
                   restore.ctypes.data, restore_at.ctypes.data, dt_restore.ctypes.data)


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

    def tracer7(self, n, tf, vit, atb, restore, restore_at, dt_restore, boundary_restore, simple_assm, ktv):
        """The reference's tracer_7 kernel alone on the given arrays (tf and
        dt_restore updated in place; float64, C order, the block size)."""
        f = self.lib.ref_tracer7_call
        f.argtypes = [C.c_int] + [C.c_void_p] * 6 + [C.c_int] * 3
        f(int(n), tf.ctypes.data, vit.ctypes.data, atb.ctypes.data, restore.ctypes.data, restore_at.ctypes.data,
          dt_restore.ctypes.data, int(boundary_restore), int(simple_assm), int(ktv))


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

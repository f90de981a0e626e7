"""LICOM3 baroclinic tracer step on B200 (sm_100a) - host-side interface.

This package mirrors, in Python, the interface LICOM3-HIP's host code uses
for the tracer path (``tracer_(ii)`` and ``convadj_()`` from stepon.cpp:69,77
acting on device-resident state) on top of the C ABI declared in
``include/licom_tracer.h`` and ``include/licom_synth.h``.  The compute path is
``liblicom_tracer.so`` (hand-written CUDA for sm_100a); nothing here computes a
tracer step on the CPU.  Importing fails loudly when the library is missing.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# LICOM_TRACER_LIB selects another build of the same library (e.g. one
# compiled with different flags); the default is the in-tree build
LIB_PATH = os.environ.get("LICOM_TRACER_LIB") or os.path.join(_HERE, "liblicom_tracer.so")

if not os.path.exists(LIB_PATH):
    raise ImportError("%s is not built; run python licom3-hip_b200/build.py" % LIB_PATH)

lib = C.CDLL(LIB_PATH)

LT_OK, LT_E_INVALID, LT_E_OOM, LT_E_CUDA, LT_E_NUMERIC, LT_E_TIMEOUT, LT_E_STATE, LT_E_NODEVICE = range(8)
PREC_FP64, PREC_MIXED = 0, 1
# lt_adv_scheme: pconst_mod adv_tracer "tspas", "centered", "flux"
ADV_TSPAS, ADV_CENTERED, ADV_FLUX = 0, 1, 2
ADV_SCHEMES = {"tspas": ADV_TSPAS, "centered": ADV_CENTERED, "flux": ADV_FLUX}


class LtError(RuntimeError):
    def __init__(self, code, where):
        msg = lib.lt_last_error().decode(errors="replace")
        super().__init__("%s failed with status %d: %s" % (where, code, msg))
        self.code = code


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("km", C.c_int), ("precision", C.c_int),
                ("diagnostics", C.c_int), ("ew_cyclic", C.c_int), ("tripole", C.c_int)]


class Params(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("dts", "oncc", "onbc", "dwndmix", "gamma", "od0", "od0cp", "ah", "area_t")] + [
        ("nss", C.c_int), ("boundary_restore", C.c_int), ("adv_tracer", C.c_int), ("simple_assm", C.c_int),
        ("ktv", C.c_int)]


class IcesnowParams(C.Structure):
    """lt_icesnow_params; defaults are the reference's (tbice -1.8, cp 3996.0,
    latice 3.337e5, QICE reset before each call as in its FRC_CORE build)."""
    _fields_ = [("tbice", C.c_double), ("cp", C.c_double), ("latice", C.c_double), ("reset_qice", C.c_int)]

    def __init__(self, tbice=-1.8, cp=3996.0, latice=3.337e5, reset_qice=1):
        super().__init__(tbice, cp, latice, reset_qice)


TURB_TABLE_ARRAYS = ("rib", "irimax", "slq2b", "smb", "shb", "ssb", "and2on2a1", "amtaun2a1", "sma1", "sha1", "ssa1",
                     "back_ra_r", "sm_r1", "sh_r1", "ss_r1", "slq2_r1")
TURB_TABLE_SCALARS = ("rri", "rnd2on2", "dri", "deltheta_r", "b1", "theta_rcrp", "theta_rcrn", "dand2on2")


class TurbTablesStruct(C.Structure):
    """lt_turb_tables: host pointers to the closure's tables and its scalars."""
    _fields_ = [(n, C.c_void_p) for n in TURB_TABLE_ARRAYS] + [(n, C.c_double) for n in TURB_TABLE_SCALARS]


def turb_tables_struct(t):
    """lt_turb_tables over a dict of arrays and scalars (tests/turb_synth.py tables()
    layout); the arrays must stay alive while the struct is used."""
    st = TurbTablesStruct()
    for n in TURB_TABLE_ARRAYS:
        a = t[n]
        want = np.int32 if n == "irimax" else np.float64
        assert a.dtype == want and a.flags["C_CONTIGUOUS"], n
        setattr(st, n, a.ctypes.data)
    for n in TURB_TABLE_SCALARS:
        setattr(st, n, float(t[n]))
    return st


class Del4uParams(C.Structure):
    _fields_ = [("am", C.c_double), ("c0f", C.c_double)]


class RestartStruct(C.Structure):
    """lt_restart: host pointers to the restart file's fields."""
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("km", C.c_int)] + [
        (n, C.c_void_p) for n in ("h0", "u", "v", "t", "s", "ws", "su", "sv", "swv", "sshf", "lthf", "fresh")] + [
        ("number_month", C.c_int), ("number_day", C.c_int)]


RESTART_2D = ("h0", "su", "sv", "swv", "sshf", "lthf", "fresh")
RESTART_3D = ("u", "v", "t", "s", "ws")


def _restart_struct(nx, ny, km, arrays, month=0, day=0):
    st = RestartStruct()
    st.nx, st.ny, st.km = nx, ny, km
    keep = []
    for n in RESTART_2D + RESTART_3D:
        a = arrays.get(n)
        if a is not None:
            shape = (ny, nx) if n in RESTART_2D else (km, ny, nx)
            assert a.shape == shape and a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], n
            setattr(st, n, a.ctypes.data)
            keep.append(a)
    st.number_month, st.number_day = month, day
    return st, keep


def restart_write(path, nx, ny, km, arrays, month=0, day=0):
    """Write the reference's restart file (include/licom_restart.h) from a
    dict of host arrays; missing fields are written as zeros."""
    st, _keep = _restart_struct(nx, ny, km, arrays, month, day)
    _check(lib.lt_restart_write(os.fsencode(path), C.byref(st)), "lt_restart_write")


def restart_read(path, nx, ny, km):
    """Read a restart file: (dict of arrays, number_month, number_day)."""
    arrays = {n: np.empty((ny, nx)) for n in RESTART_2D}
    arrays.update({n: np.empty((km, ny, nx)) for n in RESTART_3D})
    st, _keep = _restart_struct(nx, ny, km, arrays)
    _check(lib.lt_restart_read(os.fsencode(path), C.byref(st)), "lt_restart_read")
    return arrays, st.number_month, st.number_day


class TurbParams(C.Structure):
    _fields_ = [("ncc", C.c_int), ("dfricmx", C.c_double)]


class SynthConfig(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("km", C.c_int), ("lat_s", C.c_double), ("lat_n", C.c_double),
                ("dz_top", C.c_double), ("dz_bot", C.c_double), ("depth", C.c_double), ("umax", C.c_double),
                ("seed", C.c_uint64), ("forced", C.c_int), ("cap_north", C.c_int), ("cap_south", C.c_int),
                ("ew_cyclic", C.c_int), ("tripole", C.c_int), ("land_frac", C.c_double), ("member", C.c_uint32),
                ("tpert", C.c_double), ("ah_bihar", C.c_double), ("hypsometry", C.c_int)]


class BatchConfig(C.Structure):
    _fields_ = [("column_ctas_per_sm", C.c_int), ("continuity_tile_y", C.c_int), ("use_graph", C.c_int)]


class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget", C.c_size_t), ("max_active", C.c_int), ("chunk_steps", C.c_int),
                ("precision", C.c_int)]


class Request(C.Structure):
    _fields_ = [("domain", SynthConfig), ("steps", C.c_int), ("arrival", C.c_double), ("keep_state", C.c_int)]


class RequestStatus(C.Structure):
    _fields_ = [("state", C.c_int), ("steps_done", C.c_int), ("arrival", C.c_double), ("admitted", C.c_double),
                ("finished", C.c_double), ("content", C.c_double * 2), ("cells", C.c_longlong),
                ("bytes", C.c_size_t)]


class ServerStats(C.Structure):
    _fields_ = [("requests_done", C.c_longlong), ("requests_refused", C.c_longlong), ("iterations", C.c_longlong),
                ("cell_steps", C.c_double), ("busy_s", C.c_double), ("wall_s", C.c_double),
                ("latency_p50", C.c_double), ("latency_p99", C.c_double), ("latency_max", C.c_double),
                ("max_resident", C.c_int), ("peak_bytes", C.c_size_t)]


_vp, _sz, _i = C.c_void_p, C.c_size_t, C.c_int
_SIGS = {
    "lt_create": ([C.POINTER(Grid), C.POINTER(Params), C.POINTER(_vp)], _i),
    "lt_destroy": ([_vp], _i),
    "lt_set_params": ([_vp, C.POINTER(Params)], _i),
    "lt_domain_bytes": ([C.POINTER(Grid)], _sz),
    "lt_set_field": ([_vp, _i, _vp, _sz], _i),
    "lt_get_field": ([_vp, _i, _vp, _sz], _i),
    "lt_set_field_device": ([_vp, _i, _vp, _sz], _i),
    "lt_get_field_device": ([_vp, _i, _vp, _sz], _i),
    "lt_derive_masks": ([_vp], _i),
    "lt_step": ([_vp, _i], _i),
    "lt_step_host": ([_vp, C.POINTER(_vp), C.POINTER(C.c_double), C.POINTER(C.c_double)], _i),
    "lt_step_host_async": ([_vp, C.POINTER(_vp), _vp, _vp], _i),
    "lt_profile": ([_vp, _i], _i),
    "lt_mark": ([_vp, _i], _i),
    "lt_use_tma": ([_vp, _i], _i),
    "lt_set_wait_limit": ([_vp, C.c_uint], _i),
    "lt_phase_ms": ([_vp, C.POINTER(C.c_float), _i], _i),
    "lt_launch_count": ([], C.c_longlong),
    "lt_set_device": ([_i], _i),
    "lt_convadj": ([_vp], _i),
    "lt_icesnow": ([_vp, C.POINTER(IcesnowParams)], _i),
    "lt_icesnow_defaults": ([C.POINTER(IcesnowParams)], None),
    "lt_turb_tables_create": ([C.POINTER(TurbTablesStruct), C.POINTER(_vp)], _i),
    "lt_turb_tables_destroy": ([_vp], _i),
    "lt_turb": ([_vp, _vp, C.POINTER(TurbParams)], _i),
    "lt_hdiffu_del4": ([_vp, C.POINTER(Del4uParams)], _i),
    "lt_restart_write": ([C.c_char_p, C.POINTER(RestartStruct)], _i),
    "lt_restart_read": ([C.c_char_p, C.POINTER(RestartStruct)], _i),
    "lt_domain_save_restart": ([_vp, C.c_char_p, C.POINTER(RestartStruct)], _i),
    "lt_domain_load_restart": ([_vp, C.c_char_p, C.POINTER(RestartStruct)], _i),
    "lt_tracer_content": ([_vp, C.POINTER(C.c_double)], _i),
    "lt_fw_norm2": ([_vp, C.POINTER(C.c_double)], _i),
    "lt_sync": ([_vp], _i),
    "lt_check_numeric": ([_vp, C.POINTER(C.c_longlong)], _i),
    "lt_last_step_ms": ([_vp, C.POINTER(C.c_float)], _i),
    "lt_shim_bind": ([_vp], _i),
    "tracer_": ([_i], None),
    "convadj_": ([], None),
    "icesnow_": ([], None),
    "lt_last_error": ([], C.c_char_p),
    "lt_device_count": ([C.POINTER(_i)], _i),
    "lt_version": ([], C.c_char_p),
    "lt_field_name": ([_i], C.c_char_p),
    "lt_field_count": ([_i, _i, _i, _i], C.c_long),
    "lt_field_is_int": ([_i], _i),
    "lt_field_on_demand": ([_i], _i),
    "lt_synth_defaults": ([C.POINTER(SynthConfig)], None),
    "lt_synth_build": ([C.POINTER(SynthConfig), C.POINTER(_vp)], _i),
    "lt_synth_free": ([_vp], _i),
    "lt_synth_params": ([_vp, C.POINTER(Params)], _i),
    "lt_synth_grid": ([_vp, C.POINTER(Grid)], _i),
    "lt_synth_field": ([_vp, _i, _vp, _sz], _i),
    "lt_synth_field_count": ([_vp, _i], C.c_long),
    "lt_synth_upload": ([_vp, _vp], _i),
    "lt_tracer_content_noalloc": ([_vp, _vp, _vp, _vp, _i, _i, _i, _vp, _vp], _i),
    "lt_batch_create": ([C.POINTER(_vp), _i, C.POINTER(_vp)], _i),
    "lt_batch_destroy": ([_vp], _i),
    "lt_batch_size": ([_vp, C.POINTER(_i)], _i),
    "lt_batch_get_config": ([_vp, C.POINTER(BatchConfig)], _i),
    "lt_batch_set_config": ([_vp, C.POINTER(BatchConfig)], _i),
    "lt_batch_step": ([_vp, _i], _i),
    "lt_batch_sync": ([_vp], _i),
    "lt_batch_last_ms": ([_vp, C.POINTER(C.c_float)], _i),
    "lt_batch_autotune": ([_vp, _i, C.POINTER(BatchConfig)], _i),
    "lt_server_create": ([C.POINTER(ServerConfig), C.POINTER(_vp)], _i),
    "lt_server_destroy": ([_vp], _i),
    "lt_server_clock": ([_vp], C.c_double),
    "lt_server_submit": ([_vp, C.POINTER(Request), C.POINTER(_i)], _i),
    "lt_server_run_once": ([_vp, C.POINTER(_i)], _i),
    "lt_server_drain": ([_vp], _i),
    "lt_server_status": ([_vp, _i, C.POINTER(RequestStatus)], _i),
    "lt_server_state": ([_vp, _i, _vp, _sz], _i),
    "lt_server_stats_get": ([_vp, C.POINTER(ServerStats)], _i),
}
for _name, (_args, _res) in _SIGS.items():
    _fn = getattr(lib, _name)
    _fn.argtypes = _args
    _fn.restype = _res

FIELDS = []
_f = 0
while True:
    _nm = lib.lt_field_name(_f)
    if _nm is None:
        break
    FIELDS.append(_nm.decode())
    _f += 1
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}
INT_FIELDS = {n for n in FIELDS if lib.lt_field_is_int(FIELD_ID[n])}
# inputs a caller supplies (everything except step outputs and diagnostics)
# (WS, NET and QICE are model state the step or icesnow reads and rewrites;
# they start at zero)
INPUT_FIELDS = [n for n in FIELDS if n not in (
    "UTF_OUT", "VTF_OUT", "H0F_OUT", "RESTORE", "AX", "AY", "AZ", "DZ", "TEND", "DT_DIFF", "DT_CONV", "PENETRATE",
    "RESTORE_AT", "DT_RESTORE")
    and not lib.lt_field_on_demand(FIELD_ID[n])]
# fields a domain allocates on first use: the turbulence closure's and the
# momentum friction's
TURB_FIELDS = FIELDS[FIELD_ID["RIT"]:FIELD_ID["WP3_TIDAL"] + 1]
MOM_FIELDS = FIELDS[FIELD_ID["UP"]:FIELD_ID["DYUR"] + 1]


def _check(rc, where):
    if rc != LT_OK:
        raise LtError(rc, where)


def field_shape(name, nx, ny, km):
    imt, jmt = nx + 4, ny + 4
    n = lib.lt_field_count(FIELD_ID[name], nx, ny, km)
    shapes = {2 * km * jmt * imt: (2, km, jmt, imt), 2 * (km + 1) * jmt * imt: (2, km + 1, jmt, imt),
              km * jmt * imt: (km, jmt, imt), (km + 1) * jmt * imt: (km + 1, jmt, imt),
              jmt * imt: (jmt, imt), 2 * jmt * imt: (2, jmt, imt), km: (km,), 9 * km: (9, km),
              (km - 1) * jmt * imt: (km - 1, jmt, imt), km + 1: (km + 1,)}
    return shapes[n]


def field_dtype(name):
    return np.int32 if name in INT_FIELDS else np.float64


def set_device(dev):
    _check(lib.lt_set_device(int(dev)), "lt_set_device")


def launch_count():
    return lib.lt_launch_count()


def device_count():
    n = C.c_int(0)
    lib.lt_device_count(C.byref(n))
    return n.value


class TracerDomain:
    """One LICOM tracer domain resident on the current CUDA device.

    Replaces the reference's global device state (cuda_data.h, cudainit in
    cuda_init.cpp:372-707) for the tracer path, with explicit lifetime.
    """

    def __init__(self, nx, ny, km, params, precision=PREC_FP64, diagnostics=False, ew_cyclic=True, tripole=True):
        self.nx, self.ny, self.km = nx, ny, km
        self.grid = Grid(nx, ny, km, precision, int(bool(diagnostics)), int(bool(ew_cyclic)), int(bool(tripole)))
        self.params = params
        h = _vp()
        _check(lib.lt_create(C.byref(self.grid), C.byref(params), C.byref(h)), "lt_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib.lt_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def shape(self, name):
        return field_shape(name, self.nx, self.ny, self.km)

    def set(self, name, array):
        a = np.ascontiguousarray(array, dtype=field_dtype(name))
        _check(lib.lt_set_field(self.h, FIELD_ID[name], a.ctypes.data, a.nbytes), "lt_set_field(%s)" % name)

    def set_params(self, params):
        """New scalars (lt_set_params) for the following steps."""
        _check(lib.lt_set_params(self.h, C.byref(params)), "lt_set_params")
        self.params = params

    def get(self, name):
        a = np.empty(self.shape(name), dtype=field_dtype(name))
        _check(lib.lt_get_field(self.h, FIELD_ID[name], a.ctypes.data, a.nbytes), "lt_get_field(%s)" % name)
        return a

    def set_device(self, name, ptr, nbytes):
        _check(lib.lt_set_field_device(self.h, FIELD_ID[name], ptr, nbytes), "lt_set_field_device(%s)" % name)

    def derive_masks(self):
        _check(lib.lt_derive_masks(self.h), "lt_derive_masks")

    def step(self, nsteps=1):
        _check(lib.lt_step(self.h, nsteps), "lt_step")

    def step_host(self, forcing=None):
        """One step with host forcing arrays (dict name->array for SWV, NSWV,
        SST, SSS, FRESH, SEAICE); returns (fw_norm2, T content, S content)."""
        arr = (_vp * 6)()
        keep = []
        for m, nm in enumerate(("SWV", "NSWV", "SST", "SSS", "FRESH", "SEAICE")):
            if forcing is not None and nm in forcing:
                a = np.ascontiguousarray(forcing[nm], dtype=np.float64)
                keep.append(a)
                arr[m] = a.ctypes.data
        fw = C.c_double()
        cont = (C.c_double * 2)()
        _check(lib.lt_step_host(self.h, arr, C.byref(fw), cont), "lt_step_host")
        return fw.value, cont[0], cont[1]

    def step_host_ptrs(self, ptrs, fw_out):
        """Step with forcing at raw host addresses (6 ints, 0 = keep) and the
        fw_norm2 written to a ctypes double; the timed end-to-end path."""
        arr = (_vp * 6)(*ptrs)
        _check(lib.lt_step_host(self.h, arr, C.byref(fw_out), None), "lt_step_host")

    def step_host_async_ptrs(self, ptrs, fw_addr, content_addr=None):
        """lt_step_host_async: forcing at raw host addresses (6 ints, 0 =
        keep), fw_norm2 (and the two integrals) delivered to raw host
        addresses once the step has run; returns at once (see sync())."""
        arr = (_vp * 6)(*ptrs)
        _check(lib.lt_step_host_async(self.h, arr, fw_addr, content_addr), "lt_step_host_async")

    def use_tma(self, on=True):
        _check(lib.lt_use_tma(self.h, int(on)), "lt_use_tma")

    def set_wait_limit(self, polls):
        _check(lib.lt_set_wait_limit(self.h, int(polls)), "lt_set_wait_limit")

    def mark(self, which):
        _check(lib.lt_mark(self.h, int(which)), "lt_mark")

    def profile(self, on=True):
        _check(lib.lt_profile(self.h, int(on)), "lt_profile")

    PHASES = ("surface", "sss_sum", "net_halo", "continuity", "tracer", "state_halo")

    def phase_ms(self):
        ms = (C.c_float * 6)()
        n = lib.lt_phase_ms(self.h, ms, 6)
        if n < 0:
            _check(-n, "lt_phase_ms")
        return n, dict(zip(self.PHASES, list(ms)))

    def convadj(self):
        _check(lib.lt_convadj(self.h), "lt_convadj")

    def turb(self, tab, ncc=1, dfricmx=0.1):
        """Canuto turbulence closure (turb_cu, readyc.cpp:1456-1612) with the
        tables of ``tab`` (a TurbTab on this device): writes AKT, AKMT,
        AK_TIDE, AMLD and the tidal diagnostics."""
        prm = TurbParams(int(ncc), float(dfricmx))
        _check(lib.lt_turb(self.h, tab.h, C.byref(prm)), "lt_turb")

    def hdiffu_del4(self, am, c0f):
        """Momentum biharmonic friction (readyc.cpp:343-577): DLU, DLV += the
        friction of UP, VP; WKA_DRAG = c0f*|u|."""
        prm = Del4uParams(float(am), float(c0f))
        _check(lib.lt_hdiffu_del4(self.h, C.byref(prm)), "lt_hdiffu_del4")

    def save_restart(self, path, extra=None, month=0, day=0):
        """Write the domain's state as the reference's restart file; extra:
        dict of host arrays for u, v, su, sv, sshf, lthf (missing: zeros)."""
        st, _keep = _restart_struct(self.nx, self.ny, self.km, extra or {}, month, day)
        _check(lib.lt_domain_save_restart(self.h, os.fsencode(path), C.byref(st)), "lt_domain_save_restart")

    def load_restart(self, path):
        """Set AT (and ATB, H0F as NEXTSTEP does) from a restart file; returns
        (u, v, number_month, number_day)."""
        u = np.empty((self.km, self.ny, self.nx))
        v = np.empty((self.km, self.ny, self.nx))
        st, _keep = _restart_struct(self.nx, self.ny, self.km, {"u": u, "v": v})
        _check(lib.lt_domain_load_restart(self.h, os.fsencode(path), C.byref(st)), "lt_domain_load_restart")
        return u, v, st.number_month, st.number_day

    def icesnow(self, params=None):
        """Sea-ice adjustment of the current state (icesnow.cpp:15-85);
        params an IcesnowParams, None for the reference's values."""
        _check(lib.lt_icesnow(self.h, C.byref(params) if params is not None else None), "lt_icesnow")

    def tracer_content(self):
        out = (C.c_double * 2)()
        _check(lib.lt_tracer_content(self.h, out), "lt_tracer_content")
        return tuple(out)

    def fw_norm2(self):
        v = C.c_double()
        _check(lib.lt_fw_norm2(self.h, C.byref(v)), "lt_fw_norm2")
        return v.value

    def sync(self):
        _check(lib.lt_sync(self.h), "lt_sync")

    def check_numeric(self):
        bad = C.c_longlong(0)
        rc = lib.lt_check_numeric(self.h, C.byref(bad))
        if rc not in (LT_OK, LT_E_NUMERIC):
            _check(rc, "lt_check_numeric")
        return bad.value

    def last_step_ms(self):
        v = C.c_float()
        _check(lib.lt_last_step_ms(self.h, C.byref(v)), "lt_last_step_ms")
        return v.value

    def bind_shim(self):
        _check(lib.lt_shim_bind(self.h), "lt_shim_bind")


class TurbTab:
    """The closure's tables copied to the current device (lt_turb_tables_create);
    ``tables`` is a dict in the tests/turb_synth.py tables() layout."""

    def __init__(self, tables):
        st = turb_tables_struct(tables)
        h = _vp()
        _check(lib.lt_turb_tables_create(C.byref(st), C.byref(h)), "lt_turb_tables_create")
        self.h = h

    def close(self):
        if self.h:
            lib.lt_turb_tables_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tracer_(ii=0):
    """tracer.cpp:1701 - one tracer step on the domain bound with bind_shim()."""
    lib.tracer_(int(ii))
    err = lib.lt_last_error()
    return err.decode() if err else ""


def convadj_():
    """convadj.cpp:290 - convective adjustment of the bound domain."""
    lib.convadj_()


def icesnow_():
    """icesnow.cpp:70 - sea-ice adjustment of the bound domain with the
    reference's parameters."""
    lib.icesnow_()
    err = lib.lt_last_error()
    return err.decode() if err else ""


class Synth:
    """Seeded synthetic domain (grid, masks, state, velocities, mixing, forcing)."""

    def __init__(self, nx=360, ny=196, km=30, **kw):
        cfg = SynthConfig()
        lib.lt_synth_defaults(C.byref(cfg))
        cfg.nx, cfg.ny, cfg.km = nx, ny, km
        for k, v in kw.items():
            setattr(cfg, k, v)
        self.cfg = cfg
        h = _vp()
        _check(lib.lt_synth_build(C.byref(cfg), C.byref(h)), "lt_synth_build")
        self.h = h
        self.nx, self.ny, self.km = nx, ny, km
        p = Params()
        _check(lib.lt_synth_params(self.h, C.byref(p)), "lt_synth_params")
        self.params = p

    def __del__(self):
        try:
            if self.h:
                lib.lt_synth_free(self.h)
                self.h = None
        except Exception:
            pass

    def field(self, name):
        a = np.empty(field_shape(name, self.nx, self.ny, self.km), dtype=field_dtype(name))
        _check(lib.lt_synth_field(self.h, FIELD_ID[name], a.ctypes.data, a.nbytes), "lt_synth_field(%s)" % name)
        return a

    def inputs(self):
        return {n: self.field(n) for n in INPUT_FIELDS}

    def all_fields(self):
        """Every field of the domain (outputs and diagnostics zero)."""
        return {n: self.field(n) for n in FIELDS}

    def upload(self, dom):
        """Fill a TracerDomain: 2-D/1-D inputs from the host, 3-D inputs
        generated on the device (bit-identical to field())."""
        _check(lib.lt_synth_upload(self.h, dom.h), "lt_synth_upload")

    def domain(self, precision=PREC_FP64, diagnostics=False, device_fill=True):
        dom = TracerDomain(self.nx, self.ny, self.km, self.params, precision=precision, diagnostics=diagnostics,
                           ew_cyclic=bool(self.cfg.ew_cyclic), tripole=bool(self.cfg.tripole))
        if device_fill:
            self.upload(dom)
        else:
            for n, a in self.inputs().items():
                dom.set(n, a)
        return dom


class Batch:
    """Several domains stepped together (include/licom_batch.h): ensemble
    members of one grid or regional domains of different sizes, all of one
    precision, on the current device.  Mixed-precision members share one
    continuity launch and one persistent column launch per step; the steps
    replay captured CUDA graphs."""

    def __init__(self, domains):
        self.domains = list(domains)          # the batch holds the domains' arenas
        arr = (_vp * len(self.domains))(*[d.h for d in self.domains])
        h = _vp()
        _check(lib.lt_batch_create(arr, len(self.domains), C.byref(h)), "lt_batch_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib.lt_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, nsteps=1):
        _check(lib.lt_batch_step(self.h, int(nsteps)), "lt_batch_step")

    def sync(self):
        _check(lib.lt_batch_sync(self.h), "lt_batch_sync")

    def last_ms(self):
        ms = C.c_float()
        _check(lib.lt_batch_last_ms(self.h, C.byref(ms)), "lt_batch_last_ms")
        return ms.value

    def config(self):
        c = BatchConfig()
        _check(lib.lt_batch_get_config(self.h, C.byref(c)), "lt_batch_get_config")
        return {"column_ctas_per_sm": c.column_ctas_per_sm, "continuity_tile_y": c.continuity_tile_y,
                "use_graph": c.use_graph}

    def set_config(self, column_ctas_per_sm=None, continuity_tile_y=None, use_graph=None):
        cur = self.config()
        for k, v in (("column_ctas_per_sm", column_ctas_per_sm), ("continuity_tile_y", continuity_tile_y),
                     ("use_graph", use_graph)):
            if v is not None:
                cur[k] = int(v)
        c = BatchConfig(cur["column_ctas_per_sm"], cur["continuity_tile_y"], cur["use_graph"])
        _check(lib.lt_batch_set_config(self.h, C.byref(c)), "lt_batch_set_config")

    def autotune(self, trial_steps=2):
        c = BatchConfig()
        _check(lib.lt_batch_autotune(self.h, int(trial_steps), C.byref(c)), "lt_batch_autotune")
        return {"column_ctas_per_sm": c.column_ctas_per_sm, "continuity_tile_y": c.continuity_tile_y,
                "use_graph": c.use_graph}


REQ_STATES = {0: "pending", 1: "queued", 2: "resident", 3: "done", -1: "refused"}


class Server:
    """Request server (include/licom_serve.h): admission by free HBM,
    resident state, continuous batching of every resident request."""

    def __init__(self, precision=PREC_MIXED, hbm_budget=0, max_active=0, chunk_steps=0):
        c = ServerConfig(int(hbm_budget), int(max_active), int(chunk_steps), int(precision))
        h = _vp()
        _check(lib.lt_server_create(C.byref(c), C.byref(h)), "lt_server_create")
        self.h = h
        self.precision = precision
        self._shapes = {}

    def close(self):
        if getattr(self, "h", None):
            lib.lt_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def clock(self):
        return lib.lt_server_clock(self.h)

    def submit(self, nx, ny, km, steps, arrival=None, keep_state=False, **synth):
        cfg = SynthConfig()
        lib.lt_synth_defaults(C.byref(cfg))
        cfg.nx, cfg.ny, cfg.km = nx, ny, km
        for k, v in synth.items():
            setattr(cfg, k, v)
        r = Request(cfg, int(steps), self.clock() if arrival is None else float(arrival), int(keep_state))
        rid = C.c_int()
        _check(lib.lt_server_submit(self.h, C.byref(r), C.byref(rid)), "lt_server_submit")
        self._shapes[rid.value] = (nx, ny, km)
        return rid.value

    def run_once(self):
        busy = C.c_int()
        _check(lib.lt_server_run_once(self.h, C.byref(busy)), "lt_server_run_once")
        return bool(busy.value)

    def drain(self):
        _check(lib.lt_server_drain(self.h), "lt_server_drain")

    def status(self, rid):
        st = RequestStatus()
        _check(lib.lt_server_status(self.h, int(rid), C.byref(st)), "lt_server_status")
        return {"state": REQ_STATES.get(st.state, st.state), "steps_done": st.steps_done, "arrival": st.arrival,
                "admitted": st.admitted, "finished": st.finished, "content": tuple(st.content), "cells": st.cells,
                "bytes": st.bytes}

    def state(self, rid):
        nx, ny, km = self._shapes[rid]
        a = np.empty((2, km, ny + 4, nx + 4))
        _check(lib.lt_server_state(self.h, int(rid), a.ctypes.data, a.nbytes), "lt_server_state")
        return a

    def stats(self):
        st = ServerStats()
        _check(lib.lt_server_stats_get(self.h, C.byref(st)), "lt_server_stats_get")
        return {f: getattr(st, f) for f, _ in ServerStats._fields_}

"""Generate tests/golden/reference_digests.json from the reference's own code.

Runs LICOM3-HIP's tracer.cpp, convadj.cpp, icesnow.cpp and readyc.cpp
(turb_cu and the momentum biharmonic friction), compiled for the CPU by oracle/Makefile (target ``ref``) from the
reference tree, on seeded
synthetic inputs (with the restoring branch on in the cases of
tests/restore_case.py, the centred and flux advection schemes in those of
tests/scheme_case.py; tracer_7 alone with its nudging branch on, in the
cases of tests/assm_case.py) at the reference's built-in block size (36 x 40 physical, 55
levels) and records SHA-256 digests of every output field plus fw_norm2.  The
icesnow cases start from the cold states of tests/icesnow_state.py; the
turbulence cases use the closure inputs and stand-in tables of
tests/turb_case.py.

    make -C oracle ref && python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "tests"))
sys.path.insert(0, os.path.join(REPO, "oracle"))

import numpy as np  # noqa: E402
from conftest import load_package  # noqa: E402
import pyoracle  # noqa: E402
from icesnow_state import ICE_CASES, cold_state  # noqa: E402
from turb_case import DFRICMX, NCC, TURB_CASES, case, tables  # noqa: E402
import assm_case  # noqa: E402
import del4u_case  # noqa: E402
import restore_case  # noqa: E402
import scheme_case  # noqa: E402

CASES = [(1, 5, 20240611), (0, 3, 7), (1, 2, 99)]
OUT_FIELDS = ["AT", "ATB", "WS", "NET", "UTF", "VTF", "VTL", "H0F", "AKT", "AX", "AY", "AZ", "DZ", "TEND",
              "DT_DIFF", "DT_CONV", "PENETRATE"]


ICE_OUT = ["AT", "ATB", "QICE", "TEND", "DT_CONV", "WS", "NET"]
TURB_OUT = ["AKT", "AKMT", "AK_TIDE", "AMLD", "RICHARDSON", "FZTIDAL", "WP3_TIDAL"]


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    lt = load_package()
    out = {}
    for forced, nsteps, seed in CASES:
        syn = lt.Synth(36, 40, 55, forced=forced, cap_north=0, cap_south=3, dz_top=5.0, dz_bot=300.0, seed=seed)
        inp = syn.all_fields()
        ref = pyoracle.Reference(syn.params)
        ref.load(inp)
        for s in range(nsteps):
            ref.tracer_call(s)
        ref.convadj()
        key = "forced%d_steps%d_seed%d" % (forced, nsteps, seed)
        out[key] = {
            "inputs": {"AT": digest(inp["AT"]), "UTF": digest(inp["UTF"])},
            "outputs": {n: digest(ref.get(n)) for n in OUT_FIELDS},
            "fw_norm2": ref.fw_norm2(),
            "surface_T_sample": ref.get("AT")[0, 0, 20, 5:15].tolist(),
            # temperature alone: the SSS-norm sum (salinity only) cannot move it
            "outputs_T": {n: digest(ref.get(n)[0]) for n in ("AT", "ATB")},
        }
    for forced, nsteps, seed in restore_case.RESTORE_CASES:
        syn, p, inp = restore_case.case(lt, forced, seed)
        ref = pyoracle.Reference(p)
        ref.load(inp)
        for s in range(nsteps):
            ref.tracer_call(s)
        ref.convadj()
        out["restore_forced%d_steps%d_seed%d" % (forced, nsteps, seed)] = {
            "inputs": {"AT": digest(inp["AT"]), "RESTORE": digest(inp["RESTORE"])},
            "outputs": {n: digest(ref.get(n)) for n in OUT_FIELDS},
            "fw_norm2": ref.fw_norm2(),
        }
    for scheme, forced, nsteps, seed in scheme_case.SCHEME_CASES:
        syn, p, inp = scheme_case.case(lt, scheme, forced, seed)
        ref = pyoracle.Reference(p)
        ref.load(inp)
        for s in range(nsteps):
            ref.tracer_call(s)
        ref.convadj()
        out["scheme_%s_forced%d_steps%d_seed%d" % (scheme, forced, nsteps, seed)] = {
            "inputs": {"AT": digest(inp["AT"])},
            # the centred scheme's racy diagnostic levels left out
            "outputs": {n: digest(scheme_case.comparable(scheme, n, ref.get(n))) for n in OUT_FIELDS},
            "fw_norm2": ref.fw_norm2(),
        }
    for frc_core, nsteps, seed in ICE_CASES:
        syn = lt.Synth(36, 40, 55, forced=1, cap_north=0, cap_south=3, dz_top=5.0, dz_bot=300.0, seed=seed)
        inp = syn.all_fields()
        inp["AT"], inp["QICE"] = cold_state(inp, seed)
        ref = pyoracle.Reference(syn.params)
        ref.load(inp)
        if nsteps == 0:
            ref.icesnow(frc_core=frc_core)
        for s in range(nsteps):
            ref.tracer_call(s)
            ref.icesnow(frc_core=frc_core)
            if s == 0:
                ref.convadj()
        key = "icesnow_frc%d_steps%d_seed%d" % (frc_core, nsteps, seed)
        out[key] = {
            "inputs": {"AT": digest(inp["AT"]), "QICE": digest(inp["QICE"])},
            "outputs": {n: digest(ref.get(n)) for n in ICE_OUT},
        }
    if pyoracle.reference_readyc_available():
        for seed, forced in TURB_CASES:
            syn, f = case(lt, seed, forced)
            ref = pyoracle.ReferenceReadyc()
            ref.load(f)
            ref.set_tables(lt.turb_tables_struct(tables(lt)))
            ref.call(NCC, DFRICMX, syn.params.dwndmix)
            out["turb_seed%d_forced%d" % (seed, forced)] = {
                "inputs": {n: digest(f[n]) for n in ("RIT", "PDENSITY", "AT")},
                "outputs": {n: digest(ref.get(n)) for n in TURB_OUT},
            }
    if pyoracle.reference_readyc_available():
        for seed, cap in del4u_case.DEL4U_CASES:
            syn, f, am = del4u_case.case(lt, seed, cap)
            ref = pyoracle.ReferenceReadyc()
            ref.load(f)
            ref.del4u(am, del4u_case.C0F)
            out["del4u_seed%d_cap%d" % (seed, cap)] = {
                "inputs": {n: digest(f[n]) for n in ("UP", "DUC", "DMS")},
                "outputs": {n: digest(ref.get(n)) for n in ("DLU", "DLV", "WKA_DRAG")},
            }
    # tracer_7 alone, nudging branch included (tests/assm_case.py)
    ref = pyoracle.Reference(lt.Synth(36, 40, 55).params)
    for br, sa, ktv, seed in assm_case.ASSM_CASES:
        tf, vit, atb, restore, restore_at = assm_case.arrays(ref.nx, ref.ny, ref.km, seed)
        res = {}
        for n in (0, 1):
            t, d = tf.copy(), np.zeros_like(restore)
            ref.tracer7(n, t, vit, atb, restore, restore_at, d, br, sa, ktv)
            res["TF%d" % n], res["DT_RESTORE%d" % n] = digest(t), digest(d)
        out[assm_case.key(br, sa, ktv, seed)] = {"inputs": {"ATB": digest(atb), "RESTORE_AT": digest(restore_at)},
                                                 "outputs": res}
    with open(os.path.join(HERE, "reference_digests.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", len(out), "cases")


if __name__ == "__main__":
    main()

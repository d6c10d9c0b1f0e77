#!/usr/bin/env python3
"""Regenerate the golden fixtures under tests/golden/ from the MoCHII source tree.

Run once where a MoCHII checkout exists, with its path as the one required
argument: python make_golden.py <MoCHII checkout>.  The fixtures it writes are small and
committed, so the tests never read the reference tree at run time.

  qmc_golden.npz   Sobol integer codes pinned by the reference's own dumps
                   (tests/qmc/q0_raw.txt, q0_scr_<seed>.txt, q2_raw.txt,
                   q2_scr_<seed>.txt, q2_dif_<seed>.txt written by
                   tests/qmc/q0_dump.f90 and q2_dump.f90).  Scrambled uniforms
                   are stored as the integer code rint(u*2^32 - 0.5), exactly
                   as q0_dump.f90 recovers codes from uniforms.
  rates_golden.npz Recombination, collisional-ionisation, cross-section and
                   free-free Gaunt values from tools/python/mochii_rates.py,
                   which tests/rates/check_python_rates.py pins to the Fortran
                   recomb_mod / photo_xsec / cooling_mod at 1e-10 relative.
  g2a_1d_golden.npz The 1D thermal reference of the G2a gate
                   (tests/g2a_thermal/check_g2a.py reference_1d) on 400
                   shells: its definitions are executed from the checkout's
                   own file (h5py stubbed, since only the run's output needs
                   it) and reference_1d(nr=400) is recorded.
"""
import os
import sys

import numpy as np

if len(sys.argv) != 2:
    sys.exit("usage: make_golden.py <path of a MoCHII checkout>")
REF = sys.argv[1]
HERE = os.path.dirname(os.path.abspath(__file__))


def load_rows(path, nrow):
    rows = []
    with open(path) as fh:
        for line in fh:
            parts = line.split()
            if not parts:
                continue
            rows.append([float(p) for p in parts[1:]])
            if len(rows) >= nrow:
                break
    return np.array(rows)


def codes_from_uniforms(u):
    return np.rint(u * 4294967296.0 - 0.5).astype(np.uint64).astype(np.uint32)


def make_qmc():
    q = os.path.join(REF, "tests", "qmc")
    out = {}
    out["q0_raw"] = load_rows(os.path.join(q, "q0_raw.txt"), 1024).astype(np.uint32)
    out["q2_raw"] = load_rows(os.path.join(q, "q2_raw.txt"), 256).astype(np.uint32)
    for seed in (12345, 777, 2024):
        n = 1024 if seed == 12345 else 256
        out[f"q0_scr_{seed}"] = codes_from_uniforms(load_rows(os.path.join(q, f"q0_scr_{seed}.txt"), n))
    for seed in (12345, 777, 2024, 55555, 999983):
        out[f"q2_scr_{seed}"] = codes_from_uniforms(load_rows(os.path.join(q, f"q2_scr_{seed}.txt"), 256))
        out[f"q2_dif_{seed}"] = codes_from_uniforms(load_rows(os.path.join(q, f"q2_dif_{seed}.txt"), 256))
    np.savez_compressed(os.path.join(HERE, "qmc_golden.npz"), **out)
    print("qmc_golden.npz:", {k: v.shape for k, v in out.items()})


def make_rates():
    sys.path.insert(0, os.path.join(REF, "tools", "python"))
    import mochii_rates as R

    T = np.geomspace(1.0e3, 1.0e5, 61)
    out = {"T": T}
    for name in ("alphaA_HII", "alphaB_HII", "alpha1_HII", "alphaA_HeII", "alphaB_HeII",
                 "alpha1_HeII", "alphaA_HeIII", "alphaB_HeIII", "alpha1_HeIII",
                 "ci_HI", "ci_HeI", "ci_HeII", "betaA_HII", "betaB_HII"):
        out[name] = np.asarray(getattr(R, name)(T), dtype=float)
    out["beta_HeII_A"] = R.beta_HeII(T, caseA=True)
    out["beta_HeII_B"] = R.beta_HeII(T, caseA=False)
    out["beta_HeIII_A"] = R.beta_HeIII(T, caseA=True)
    out["beta_HeIII_B"] = R.beta_HeIII(T, caseA=False)
    # cross sections on a grid that starts on each threshold
    E = np.concatenate([[13.598, 24.587, 54.416], np.geomspace(13.6, 100.0, 57), [5.0, 200.0]])
    out["E"] = E
    for name in ("sigma_HI", "sigma_HeI", "sigma_HeII"):
        out[name] = np.array([float(getattr(R, name)(e)) for e in E])
    out["gff_logT"] = np.asarray(R.GFF_LOGT, dtype=float)
    out["gff_z"] = np.asarray(R.GFF_Z, dtype=float)
    np.savez_compressed(os.path.join(HERE, "rates_golden.npz"), **out)
    print("rates_golden.npz:", sorted(out))


def make_g2a(nr=400):
    import types
    d = os.path.join(REF, "tests", "g2a_thermal")
    path = os.path.join(d, "check_g2a.py")
    src = open(path).read()
    src = src[:src.rindex("\n", 0, src.index(" main --"))]   # the definitions, not the run's check
    sys.modules.setdefault("h5py", types.ModuleType("h5py"))
    cwd = os.getcwd()
    os.chdir(d)
    try:
        ns = {"__file__": path, "__name__": "check_g2a_defs"}
        exec(compile(src, path, "exec"), ns)
        r, xHI, xHeI, xHeII, Te = ns["reference_1d"](nr=nr)
    finally:
        os.chdir(cwd)
    np.savez_compressed(os.path.join(HERE, "g2a_1d_golden.npz"), r=r, xHI=xHI, xHeI=xHeI, xHeII=xHeII, Te=Te)
    print("g2a_1d_golden.npz: nr =", nr, "Te range", Te.min(), Te.max())


if __name__ == "__main__":
    make_qmc()
    make_rates()
    make_g2a()

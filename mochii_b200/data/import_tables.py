#!/usr/bin/env python3
"""Copy the physical data tables this path reads from a MoCHII checkout
(its path is the one required argument) into mochii_b200/data/.

  python import_tables.py <MoCHII checkout>

  atomic/cooling_<el>_<stage>.txt   collisional line-cooling fits (cooling_mod)
  atomic/nlevel_<el>_<stage>.txt    n-level atom data (nlevel_mod)
  atomic/element_<el>.txt           trace-element registry (species_mod)
  kext_albedo_WD_MW_3.1_60_D03.all_2003   MW R_V = 3.1 grain extinction (gas_opacity_mod)
  HeI2phot.dat                      He I 2^1S two-photon shape A(y), Drake, Victor &
                                    Dalgarno 1969 (hei_twophoton_mod)

These are data (CHIANTI / Verner / Weingartner & Draine fits with provenance
headers), not code; the library loads them at set-up.
"""
import glob
import os
import shutil
import sys

if len(sys.argv) != 2:
    sys.exit("usage: import_tables.py <path of a MoCHII checkout>")
SRC = sys.argv[1]
DST = os.path.dirname(os.path.abspath(__file__))

os.makedirs(os.path.join(DST, "atomic"), exist_ok=True)
for pat in ("cooling_*.txt", "nlevel_*.txt", "element_*.txt"):
    for f in sorted(glob.glob(os.path.join(SRC, "data", "atomic", pat))):
        if f.endswith("cooling_fit_parameters.txt"):
            continue
        shutil.copyfile(f, os.path.join(DST, "atomic", os.path.basename(f)))
for name in ("kext_albedo_WD_MW_3.1_60_D03.all_2003", "HeI2phot.dat"):
    shutil.copyfile(os.path.join(SRC, "data", name), os.path.join(DST, name))
print("copied", len(os.listdir(os.path.join(DST, "atomic"))), "atomic tables")

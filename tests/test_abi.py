"""The C-ABI library: it loads, exports every symbol include/*.h declares,
and its host-side parameter reader mirrors read_input (CPU only; no device
compute is called here)."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from conftest import ROOT, gpu_available


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(mochii_[A-Za-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from mochii_b200 import _lib
    from mochii_b200.build import build
    build()
    return _lib.load()


def test_library_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    from mochii_b200._lib import SIGNATURES
    assert set(names) == set(SIGNATURES), set(names) ^ set(SIGNATURES)


def test_params_struct_layout(lib):
    from mochii_b200._lib import Params
    assert lib.mochii_params_size() == C.sizeof(Params)


def test_defaults_follow_define_f90(lib):
    from mochii_b200 import default_params
    p = default_params()
    assert p.nphotons == 100000 and p.qmc_seed == 12345 and p.nnu_ion == 16
    assert p.eion_min == 13.598 and p.eion_max == 100.0 and p.ion_align_edges == 1
    assert p.He_abund == 0.1 and p.te_fixed == 1.0e4 and p.caseA == 0 and p.ion_relax == 1.0
    assert p.te_min == 1.0e3 and p.te_max == 5.0e4 and p.gas_tol == 1.0e-3
    assert p.distance2cm == 3.0856776e21   # kpc


def test_namelist_reader(lib):
    from mochii_b200 import parse_namelist
    text = """&parameters
 ! comment line
 par%no_photons    = 4.0e7      ! a real into an integer field
 par%launch_sequence = 'sobol'
 par%grid_type = 'car', par%nx = 64
 par%distance_unit = 'pc'
 par%case_ab = 'A'
 par%solve_te = .true.
 par%src_tstar(2) = 3.5e4, 4.0e4
 par%out_file = 'ignored.h5'
 par%He_abund = 0.0
/"""
    p = parse_namelist(text)
    assert p.nphotons == 40000000 and p.launch_sobol == 1 and p.nx == 64
    assert p.distance2cm == 3.0856776e18 and p.caseA == 1 and p.solve_te == 1
    assert p.src_tstar[1] == 3.5e4 and p.src_tstar[2] == 4.0e4 and p.src_tstar[0] == -999.0
    assert p.He_abund == 0.0


def test_namelist_errors(lib):
    from mochii_b200 import MochiiError, parse_namelist
    with pytest.raises(MochiiError, match="not a component"):
        parse_namelist("&parameters par%no_such_key = 1 /")
    with pytest.raises(MochiiError, match="'A' or 'B'"):
        parse_namelist("&parameters par%case_ab = 'C' /")
    with pytest.raises(MochiiError, match="not a real"):
        parse_namelist("&parameters par%tstar = hot /")
    with pytest.raises(MochiiError, match=">= 1024"):
        parse_namelist("&parameters par%packet_chunk = 100 /")


def test_execution_keys(lib):
    from mochii_b200 import MochiiError, default_params, parse_namelist
    d = default_params()
    assert d.packet_chunk == 1 << 22 and d.tally64 == 1 and d.metal_rate_table == 1 and d.solver_warp == 3
    p = parse_namelist("&parameters par%packet_chunk = 1048576, par%tally_precision = 'compensated'\n"
                       " par%metal_rates = 'exact', par%cell_layout = 'flow' /")
    assert p.packet_chunk == 1048576 and p.tally64 == 0 and p.metal_rate_table == 0 and p.solver_warp == 2
    assert d.packet_order == 2 and parse_namelist("&parameters par%packet_order = 'direction' /").packet_order == 1
    assert parse_namelist("&parameters par%packet_order = 'launch' /").packet_order == 0
    with pytest.raises(MochiiError, match="'coherent', 'direction' or 'launch'"):
        parse_namelist("&parameters par%packet_order = 'random' /")


def test_reference_style_input_reads_unchanged(lib, tmp_path):
    # a reference-style input file with keys outside this path (output,
    # MPI schedule, observers) must read without error
    text = """&parameters
 par%no_photons = 4.0e7
 par%no_print = 4.0e7
 par%iseed = 1234
 par%grid_type = 'car'
 par%nx = 64
 par%ny = 64
 par%nz = 64
 par%xmax = 4.0
 par%ymax = 4.0
 par%zmax = 4.0
 par%dust_density_law = 'none'
 par%nH_const = 100.0
 par%rmax = 4.0
 par%distance_unit = 'pc'
 par%nnu_ion = 32
 par%tstar = 4.0e4
 par%luminosity = 3.177837e38
 par%xHI_init = 1.0
 par%gas_niter = 100
 par%case_ab = 'B'
 par%source_geometry = 'point'
 par%file_format = 'hdf5'
 par%out_file = 'g1.h5'
 par%use_master_slave = .false.
/
"""
    f = tmp_path / "g1.in"
    f.write_text(text)
    from mochii_b200 import read_input
    p = read_input(str(f))
    assert p.nnu_ion == 32 and p.rmax == 4.0 and p.dust_law == 1 and p.random_seed == 1234


@pytest.mark.skipif(gpu_available(), reason="checks the no-device error path")
def test_init_without_device_reports_status(lib):
    from mochii_b200 import MochiiError, Nebula, parse_namelist
    from mochii_b200 import configs
    p = parse_namelist(configs.stromgren64(nphotons=1000, n=8))
    with pytest.raises(MochiiError) as ei:
        Nebula(p)
    assert ei.value.status == 9   # MOCHII_ERR_NO_DEVICE


def test_unsupported_configurations_are_refused_before_device_use(lib):
    from mochii_b200 import MochiiError, Nebula, parse_namelist
    from mochii_b200 import configs
    for extra in ("par%use_sec_ion = .true.", "par%launch_sequence = 'random'", "par%ion_add_dust = .true."):
        p = parse_namelist(configs.stromgren64(nphotons=1000, n=8).replace("/\n", extra + "\n/\n"))
        with pytest.raises(MochiiError) as ei:
            Nebula(p)
        assert ei.value.status == 8, extra   # MOCHII_ERR_UNSUPPORTED
    # an octree needs its leaf list
    p = parse_namelist(configs.stromgren64(nphotons=1000, n=8).replace("par%grid_type = 'car'", "par%grid_type = 'amr'"))
    with pytest.raises(MochiiError) as ei:
        Nebula(p)
    assert ei.value.status == 1 and "amr_file" in str(ei.value)


def test_bad_grid_is_refused(lib):
    from mochii_b200 import MochiiError, Nebula, parse_namelist
    p = parse_namelist("&parameters par%launch_sequence='sobol' par%nx=8 par%ny=4 par%nz=8 "
                       "par%xmax=1 par%ymax=1 par%zmax=1 par%tstar=4e4 par%luminosity=1e38 /")
    with pytest.raises(MochiiError) as ei:
        Nebula(p)
    assert ei.value.status == 1 and "cubic" in str(ei.value)


def test_strerror_covers_every_status(lib):
    for s in range(10):
        assert lib.mochii_strerror(s)


def test_external_field_keys():
    from mochii_b200 import parse_namelist
    """The external field's keys (define.f90:266-278) and the external-only
    source_geometry shorthand (setup.f90:240-258)."""
    base = "&parameters\n par%no_photons = 1000\n"
    p = parse_namelist(base + " par%source_geometry = 'external_sph'\n par%ext_intensity = 2.5e-3\n"
                              " par%ext_tstar = 3.0e4\n par%rmax = 1.5\n/\n")
    assert p.source_external == 2 and p.ext_intensity == 2.5e-3 and p.ext_tstar == 3.0e4 and p.rmax == 1.5
    p = parse_namelist(base + " par%ext_intensity = 1e-3\n par%ext_geometry = 'sph'\n/\n")
    assert p.source_external == 0 and p.ext_geometry == 1 and p.ext_spectrum_set == 0
    p = parse_namelist(base + " par%ext_spectrum = 'draine'\n/\n")
    assert p.ext_spectrum_set == 1
    d = parse_namelist(base + "/\n")
    assert d.ext_intensity < 0 and d.source_external == 0 and d.ext_geometry == 0

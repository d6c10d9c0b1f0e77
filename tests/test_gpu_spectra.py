"""Tabulated source spectra and the ISRF presets on the device against the
oracle: the library's spectrum chains (ion_band_mod.f90:437-615, the file
readers :1438-1597, the presets :1627-1720, the source normalisation of
setup.f90:374-442) build the same samplers as the oracle's restatement, so
the band luminosity agrees to the last bits and every launched packet's
energy, bin, entry point and direction equal the oracle's -- for shape and
absolute files on point sources (one file column per source), all four
physical column types, external fields from a file and from each preset,
and the slab's spectrum from a file."""
import numpy as np
import pytest

from mochii_b200 import Nebula, configs, parse_namelist
from test_oracle_spectra import EV2ERG, H_CGS, HC_EVANG, box, planck_e, write_table

pytestmark = pytest.mark.gpu


def files(tmp_path):
    E = np.geomspace(13.0, 110.0, 3001)
    two = write_table(tmp_path / "two.txt", [E, planck_e(E, 3.0e4), 0.5 * planck_e(E, 5.0e4)])
    LE = 1.0e37 * planck_e(E, 4.0e4) / planck_e(20.0, 4.0e4)
    per = {"per_ev": write_table(tmp_path / "per_ev.txt", [E, LE]),
           "per_hz": write_table(tmp_path / "per_hz.txt", [E * EV2ERG / H_CGS, LE * H_CGS / EV2ERG]),
           "per_ang": write_table(tmp_path / "per_ang.txt", [HC_EVANG / E, LE * E * E / HC_EVANG]),
           "per_um": write_table(tmp_path / "per_um.txt", [HC_EVANG * 1e-4 / E, LE * E * E / (HC_EVANG * 1e-4)])}
    J = write_table(tmp_path / "ext.txt", [E, 2.0e-5 * planck_e(E, 3.5e4) / planck_e(20.0, 3.5e4)])
    return two, per, J


def case_namelist(tmp_path, case):
    two, per, J = files(tmp_path)
    src2 = (" par%nsource = 2\n par%src_x(1) = -0.5\n par%src_x(2) = 0.5\n"
            " par%src_lum(1) = 1.0e38\n par%src_lum(2) = 2.0e38\n")
    fuv = " par%add_fuv = .true.\n par%efuv_min = 6.0\n"
    if case == "shape_two_sources":
        return box(extra=src2 + f" par%src_spectrum_file = '{two}'\n")
    if case == "absolute_two_sources":   # src_lum unset: derived per column
        return box(extra=(" par%nsource = 2\n par%src_x(1) = -0.5\n par%src_x(2) = 0.5\n"
                          f" par%spectrum_type = 'per_ev'\n par%src_spectrum_file = '{two}'\n"))
    if case.startswith("ion_spectrum_"):
        kind = case[len("ion_spectrum_"):]
        return box(extra=f" par%spectrum_type = '{kind}'\n par%ion_spectrum = '{per[kind]}'\n par%luminosity = -999.0\n" + fuv)
    if case == "ext_file_with_point":
        return box(extra=f" par%ext_spectrum = '{J}'\n par%spectrum_type = 'per_ev'\n par%xs_point = 0.25\n")
    if case.startswith("preset_"):
        return box(extra=f" par%source_geometry = 'external_sph'\n par%rmax = 1.0\n par%ext_spectrum = '{case[7:]}'\n"
                         " par%ext_scale = 2.5\n" + fuv)
    if case == "slab_file":
        return configs.slab(nphotons=20000, mode="isotropic").replace(
            "/\n", f" par%ion_spectrum = '{two}'\n/\n")
    raise ValueError(case)


CASES = ["shape_two_sources", "absolute_two_sources", "ion_spectrum_per_ev", "ion_spectrum_per_hz",
         "ion_spectrum_per_ang", "ion_spectrum_per_um", "ext_file_with_point", "preset_draine", "preset_habing",
         "preset_mathis", "slab_file"]


@pytest.mark.parametrize("case", CASES)
def test_spectrum_launch_matches_oracle(orc, tmp_path, case):
    nl = case_namelist(tmp_path, case)
    neb = Nebula(parse_namelist(nl))
    sim = orc.Sim(nl, nthreads=1)
    assert abs(neb.ion_Ltot / sim.ion_Ltot - 1) < 1e-14, (neb.ion_Ltot, sim.ion_Ltot)
    n = 8192
    rec = neb.launch_records(0, n)
    ref = np.array([sim.photon(i) for i in range(n)])
    assert np.array_equal(rec[:, 6], ref[:, 6]) and np.array_equal(rec[:, 7], ref[:, 7])
    tol = 1e-14 * np.abs(ref[:, :3]).max() if case.startswith("preset_") else 0.0   # the sphere's cos/sin
    np.testing.assert_allclose(rec[:, :3], ref[:, :3], rtol=0, atol=tol)
    np.testing.assert_allclose(rec[:, 3:6], ref[:, 3:6], rtol=0, atol=1.2e-15)
    neb.close()


def test_preset_field_pass_matches_oracle(orc, tmp_path):
    """An FP64 pass of the Draine field alone: the FUV tally (G0) and the
    energy ledger against the oracle."""
    nl = case_namelist(tmp_path, "preset_draine").replace(" par%rmax = 1.0\n", " par%rmax = 1.5\n")
    neb = Nebula(parse_namelist(nl))
    sim = orc.Sim(nl)
    st = neb.ionizing_field_and_rates()
    sim.transport_pass()
    e, _ = sim.energy()
    assert st.closure <= 5e-13 and abs(st.energy_emitted / e[0] - 1) < 1e-12
    g, o = neb.get("g0_fuv"), sim.get("g0_fuv")
    big = o > 1e-3 * o.max()
    assert big.sum() > 100 and np.max(np.abs(g[big] / o[big] - 1)) < 1e-9
    neb.close()

"""Tabulated source spectra and the ISRF presets, CPU part: the oracle's
restatement of the spectrum chains (build_point_source_sampler and
build_external_field_sampler, ion_band_mod.f90:437-615; the spectrum files
of read_shape_table / read_phys_table, :1438-1597; the Draine, Habing and
Mathis fields, :1627-1720; the source normalisation of setup.f90:374-442)
against the properties the reference's spectrum checkers gate on
(tests/multi_src/check_specfile.py and the preset inputs): a file holding a
Planck shape reproduces the Planck source, the four physical column types
of one spectrum give the same packets, an external field's file is honoured
over the decoy tstar, the Draine field carries the canonical FUV energy
density, and absolute files fix the luminosity themselves.  The files are
written here from closed forms."""
import numpy as np
import pytest

from mochii_b200 import configs

H_CGS, EV2ERG, C_CGS = 6.62607015e-27, 1.602176634e-12, 2.99792458e10
HC_EVANG = 12398.42
KB_EV = 8.617333262145e-5


def planck_e(E, T):
    return E ** 3 / np.expm1(E / (KB_EV * T))


def box(nphot=20000, extra=""):
    """A thin uniform H box (16^3 cells, n_H = 1e-3), case A, one pass."""
    nl = configs.hhe128(nphotons=nphot, niter=1, n=16, precision="fp64")
    nl = nl.replace(" par%nH_const = 100.0\n", " par%nH_const = 1.0e-3\n")
    return nl.replace("/\n", extra + "/\n")


def write_table(path, cols, header="# E [eV]  values\n"):
    with open(path, "w") as f:
        f.write(header)
        for row in zip(*cols):
            f.write(" ".join(f"{v:.17e}" for v in row) + "\n")
    return str(path)


def energies(orc, nl, n=4096):
    s = orc.Sim(nl, nthreads=1)
    rec = np.array([s.photon(i) for i in range(n)])
    return s, rec


def test_file_reproduces_planck_sources(orc, tmp_path):
    """G-file-equivalence: two point sources take their 3e4 / 5e4 K shapes from
    the columns of one file instead of src_tstar."""
    E = np.geomspace(13.598, 100.0, 20001)
    path = write_table(tmp_path / "two_temp.txt", [E, planck_e(E, 3.0e4), planck_e(E, 5.0e4)])
    src = (" par%nsource = 2\n par%src_lum(1) = 1.0e38\n par%src_lum(2) = 2.0e38\n"
           " par%src_x(1) = -0.5\n par%src_x(2) = 0.5\n")
    s_pl, r_pl = energies(orc, box(extra=src + " par%src_tstar(1) = 3.0e4\n par%src_tstar(2) = 5.0e4\n"))
    s_f, r_f = energies(orc, box(extra=src + f" par%src_spectrum_file = '{path}'\n"))
    assert abs(s_f.ion_Ltot / s_pl.ion_Ltot - 1) < 1e-12   # shape files: L = src_lum / f_ion, f_ion = 1
    assert np.array_equal(r_f[:, 0], r_pl[:, 0])            # the same source picks
    np.testing.assert_allclose(r_f[:, 6], r_pl[:, 6], rtol=2e-4)   # energies to the table's resolution
    nb = int(max(r_f[:, 7].max(), r_pl[:, 7].max())) + 1
    hf = np.bincount(r_f[:, 7].astype(int), minlength=nb)
    hp = np.bincount(r_pl[:, 7].astype(int), minlength=nb)
    assert np.abs(hf - hp).sum() <= 0.01 * len(r_f)


@pytest.mark.parametrize("kind", ["per_hz", "per_ang", "per_um"])
def test_physical_column_types_agree(orc, tmp_path, kind):
    """G-per_ev-equivalence: the same absolute L_E written per eV, per Hz,
    per Angstrom and per micron gives the same luminosity and packets."""
    E = np.geomspace(13.0, 110.0, 4001)
    LE = 1.0e37 * planck_e(E, 4.0e4) / planck_e(20.0, 4.0e4)   # erg/s/eV
    ref = write_table(tmp_path / "per_ev.txt", [E, LE])
    if kind == "per_hz":
        x, y = E * EV2ERG / H_CGS, LE * H_CGS / EV2ERG
    elif kind == "per_ang":
        x, y = HC_EVANG / E, LE * E * E / HC_EVANG
    else:
        x, y = HC_EVANG * 1e-4 / E, LE * E * E / (HC_EVANG * 1e-4)
    alt = write_table(tmp_path / f"{kind}.txt", [x, y])
    s0, r0 = energies(orc, box(extra=f" par%spectrum_type = 'per_ev'\n par%ion_spectrum = '{ref}'\n"
                                     " par%luminosity = -999.0\n"))
    s1, r1 = energies(orc, box(extra=f" par%spectrum_type = '{kind}'\n par%ion_spectrum = '{alt}'\n"
                                     " par%luminosity = -999.0\n"))
    # absolute: the luminosity is the file's band integral (trapezoids over 13.598-100 eV)
    assert abs(s1.ion_Ltot / s0.ion_Ltot - 1) < 1e-9
    sel = (E > 13.598) & (E < 100.0)
    Eb = np.concatenate([[13.598], E[sel], [100.0]])
    Lb = np.interp(Eb, E, LE)
    assert abs(s0.ion_Ltot / np.trapezoid(Lb, Eb) - 1) < 1e-12
    np.testing.assert_allclose(r1[:, 6], r0[:, 6], rtol=1e-9)


def test_external_file_beats_decoy_tstar(orc, tmp_path):
    """G-ext-spectrum: an external-only field takes its shape from
    ext_spectrum (a tabulated 4e4 K Planck) and matches ext_tstar = 4e4 K,
    not the decoy tstar = 2e4 K."""
    E = np.geomspace(13.598, 100.0, 20001)
    path = write_table(tmp_path / "ext_4e4.txt", [E, planck_e(E, 4.0e4)])
    ext = " par%source_geometry = 'external_rec'\n par%ext_intensity = 1.0e-3\n par%tstar = 2.0e4\n"
    s_f, r_f = energies(orc, box(extra=ext + f" par%ext_spectrum = '{path}'\n"))
    s_t, r_t = energies(orc, box(extra=ext + " par%ext_tstar = 4.0e4\n"))
    s_d, r_d = energies(orc, box(extra=ext))
    assert abs(s_f.ion_Ltot / s_t.ion_Ltot - 1) < 1e-12
    np.testing.assert_allclose(r_f[:, 6], r_t[:, 6], rtol=2e-4)
    assert abs(np.mean(r_f[:, 6]) / np.mean(r_d[:, 6]) - 1) > 0.05   # the decoy is a different spectrum


@pytest.mark.parametrize("preset,ratio", [("draine", 1.0), ("habing", 1.0 / 1.71)])
def test_preset_fuv_energy_density(orc, preset, ratio):
    """G-presets: the Draine (1978) field carries u_FUV = (4 pi / c) int_6^13.6
    J_E dE = 8.94e-14 erg/cm^3 (G0 = 1.69), Habing 1/1.71 of it; the
    entering power is pi A int J_E dE."""
    ext = (" par%source_geometry = 'external_rec'\n par%add_fuv = .true.\n par%efuv_min = 6.0\n"
           f" par%ext_spectrum = '{preset}'\n par%ext_scale = 1.0\n")
    s = orc.Sim(box(extra=ext), nthreads=1)
    L = (2 * configs.stromgren_radius_pc(Q=5.0e49) * configs.PC2CM) ** 2 * 6
    u = 4.0 * np.pi / C_CGS * s.ion_Ltot / (np.pi * L)
    assert abs(u / (8.94e-14 * ratio) - 1) < 5e-3
    rec = np.array([s.photon(i) for i in range(2048)])
    assert rec[:, 6].min() >= 6.0 and rec[:, 6].max() <= 13.6


def test_mathis_preset_and_rescale(orc):
    """The Mathis field's J_E from its UV power laws, and ext_intensity
    rescaling any preset to a band J: L = pi A J exactly."""
    ext = (" par%source_geometry = 'external_rec'\n par%add_fuv = .true.\n par%efuv_min = 6.0\n"
           " par%ext_spectrum = 'mathis'\n")
    s = orc.Sim(box(extra=ext), nthreads=1)
    E = np.linspace(6.0, 13.6, 4096)
    lam = HC_EVANG * 1e-4 / E
    Jl = np.where(lam < 0.110, 3069.0 * lam ** 3.4172, np.where(lam < 0.134, 1.627, 0.0566 * lam ** -1.6678))
    Jl[lam < 0.0912] = 0.0   # nothing beyond the Lyman limit
    JE = Jl * (HC_EVANG * 1e-7) / E ** 2
    A = (2 * configs.stromgren_radius_pc(Q=5.0e49) * configs.PC2CM) ** 2 * 6
    assert abs(s.ion_Ltot / (np.pi * A * np.trapezoid(JE, E)) - 1) < 1e-9
    s2 = orc.Sim(box(extra=ext + " par%ext_intensity = 2.0e-4\n"), nthreads=1)
    assert abs(s2.ion_Ltot / (np.pi * A * 2.0e-4) - 1) < 1e-9   # A from the namelist's 10-decimal side


def test_source_normalisation(orc):
    """setup.f90:374-442: no src_lum splits luminosity equally; a lone source
    composed with a field takes the legacy scalars into slot 1."""
    two = (" par%nsource = 2\n par%src_tstar(1) = 4.0e4\n par%src_tstar(2) = 4.0e4\n"
           " par%src_x(1) = -0.5\n par%src_x(2) = 0.5\n par%luminosity = 3.0e38\n")
    s = orc.Sim(box(extra=two), nthreads=1)
    assert abs(s.ion_Ltot / 3.0e38 - 1) < 1e-14
    mix = " par%xs_point = 0.25\n par%ext_intensity = 1.0e-3\n"
    s = orc.Sim(box(extra=mix), nthreads=1)
    rec = np.array([s.photon(i) for i in range(4096)])
    point = np.abs(rec[:, :3]).max(axis=1) < 0.9 * configs.stromgren_radius_pc(Q=5.0e49)
    assert point.sum() > 100 and np.all(rec[point, 0] == 0.25)

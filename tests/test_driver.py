"""The main.f90-style driver (negftrans_b200/negftrans): INPUT/POTENTIAL
parsing, the reference's validation messages, the G17.8 writer (CPU), and an
end-to-end run against the oracle (GPU)."""
import json
import math
import os
import subprocess

import numpy as np
import pytest

from negftrans_b200 import HARTREE
from negftrans_b200 import build as B
from negftrans_b200 import prepare as P
from negftrans_b200 import workloads as W


@pytest.fixture(scope="module")
def driver(built_lib):
    return B.build_driver()


def _potential(path, V):
    with open(path, "w") as f:
        f.write("%5d%5d%5d\n" % V.shape)
        vals = np.asarray(V).ravel(order="F")
        for i in range(0, len(vals), 5):
            f.write("".join("%17.8G" % x for x in vals[i:i + 5]) + "\n")


def _run(driver, cwd, *args, check=True):
    return subprocess.run([driver, *args], cwd=cwd, capture_output=True, text=True, timeout=600, check=check)


def fortran_g17_8(x):
    """Fortran G17.8 output editing, restated from the standard's rules: F
    editing F13.(8-k) + 4 blanks when 10^(k-1) <= |x| (rounded to 8 digits) <
    10^k with 0 <= k <= 8, E17.8 (0.dddddddd E+xx) otherwise."""
    if x == 0:
        return "%13.7f    " % 0.0
    m = "%.7e" % x
    k = int(m.split("e")[1]) + 1
    if 0 <= k <= 8:
        return "%13.*f    " % (8 - k, x)
    digits = m.split("e")[0].replace("-", "").replace(".", "")
    ex = ("E%+03d" % k) if abs(k) <= 99 else ("%+04d" % k)
    return ("%17s" % (("-" if x < 0 else "") + "0." + digits + ex))


def test_g17_8_writer(driver, tmp_path):
    vals = [21.0, 0.50044916e-7, 19.5931634, -3.25, 0.0, 1e8, 99999999.7, 0.1, 0.09999999999,
            1.234e-120, -7.5e12, 6.02214076e23, -0.000123456789, 1.0, 12345678.4]
    out = _run(driver, tmp_path, "--gfmt", *[repr(v) for v in vals]).stdout.split("\n")
    got = [line[1:-1] for line in out if line]
    assert len(got) == len(vals)
    for v, g in zip(vals, got):
        assert len(g) == 17, (v, g)
        assert g == fortran_g17_8(v), (v, g)
        if "E" in g or g.strip().count("-") == 0 or v > 0:
            txt = g.strip()
            if "E" not in txt and ("+" in txt[1:] or "-" in txt[1:]):   # 3-digit exponent form
                pos = max(txt.rfind("+"), txt.rfind("-"))
                txt = txt[:pos] + "e" + txt[pos:]
            assert math.isclose(float(txt.replace("E", "e")), v, rel_tol=6e-8, abs_tol=0.0), (v, g)


NAMELIST = """! a comment before the group
&input
  IF_TRANSMISSION = .TRUE., if_density = F
  LX=1000.0 , LY = 1000.0   ! inline comment
  lz = 80.0
  ENCUT = 1.2D-3
  NKX = 1  NKY = 2
  TRANSMISSION_GRID = 0.0 2.01E-3 8
  ETA = 2.4622d-9
  LDOS_GRID = -1 2*0
  N_circle = 7
/

"""


def test_namelist_parsing(driver, tmp_path):
    (tmp_path / "INPUT").write_text(NAMELIST)
    _potential(tmp_path / "POTENTIAL", np.full((16, 16, 4), 0.0033))
    r = _run(driver, tmp_path, "--check")
    d = json.loads(r.stdout)
    assert d["if_transmission"] == 1 and d["if_density"] == 0 and d["if_LDOS"] == 0
    assert d["LX"] == 1000.0 and d["LZ"] == 80.0 and d["ENCUT"] == 1.2e-3 and d["ETA"] == 2.4622e-9
    assert d["TRANSMISSION_GRID"] == [0.0, 2.01e-3, 8.0]
    assert d["LDOS_GRID"] == [-1, 0, 0] and d["N_circle"] == 7 and d["N_line_per_eV"] == 500
    assert d["nk"] == 2 and (d["Nx"], d["Ny"], d["Nz"]) == (16, 16, 4)
    deck = P.InputDeck(LX=1000.0, LY=1000.0, LZ=80.0, ENCUT=1.2e-3)
    assert (d["NGX"], d["NGY"]) == P.ngrid(deck)
    from negftrans_b200.grid import PlaneWaveBasis_construction_findsize
    assert d["N"] == PlaneWaveBasis_construction_findsize(1.2e-3 / HARTREE, 1000.0 / 0.529177210903,
                                                          1000.0 / 0.529177210903)
    assert math.isclose(d["min_V"], 0.0033 / HARTREE, rel_tol=1e-7)


@pytest.mark.parametrize("text,msg", [
    ("&INPUT\n NKX=1 NKY=1 if_transmission=.true. TRANSMISSION_GRID = 0 1 4\n/\n", "LX, LY, LZ must be specified"),
    ("&INPUT\n LX=1 LY=1 LZ=1 if_transmission=.true. TRANSMISSION_GRID = 0 1 4\n/\n", "NKX, NKY must be specified"),
    ("&INPUT\n LX=1 LY=1 LZ=1 NKX=1 NKY=1\n/\n", "Nothing to do"),
    ("&INPUT\n LX=1 LY=1 LZ=1 NKX=1 NKY=1 if_transmission=.true.\n/\n", "TRANSMISSION_GRID must be specified"),
    ("&INPUT\n LX=1 LY=1 LZ=1 NKX=1 NKY=1 if_LDOS=.true. LDOS_ENERGY_GRID = 0 1 2\n/\n", "LDOS_GRID must be specified"),
    ("&INPUT\n LX=1 LY=1 LZ=1 NKX=1 NKY=1 if_transmission=.true. TRANSMISSION_GRID = 0 1 4 VDS=0.1\n/\n",
     "VDS must be zero"),
])
def test_validation_messages(driver, tmp_path, text, msg):
    (tmp_path / "INPUT").write_text(text)
    _potential(tmp_path / "POTENTIAL", np.zeros((4, 4, 2)))
    r = _run(driver, tmp_path, "--check", check=False)
    assert r.returncode == 1
    out = (tmp_path / "OUTPUT").read_text()
    assert msg in out and "EXIT" in out


def test_odd_grid_rejected(driver, tmp_path):
    (tmp_path / "INPUT").write_text(NAMELIST)
    _potential(tmp_path / "POTENTIAL", np.zeros((5, 4, 2)))
    r = _run(driver, tmp_path, "--check", check=False)
    assert r.returncode == 1
    assert "must be even number" in (tmp_path / "OUTPUT").read_text()


@pytest.mark.gpu
def test_end_to_end_against_oracle(driver, tmp_path, oracle):
    """TRANSMISSION, DENSITY and LDOS files of a small QPC against the oracle."""
    nz = 6
    V = W.MSTAR * W.qpc_potential(32, 32, nz, 100.0, nz * 1.0, 0.05, 15.0, 1.0, disorder=0.002)
    deck = P.InputDeck(if_transmission=True, if_density=True, if_LDOS=True, LX=1000.0, LY=1000.0,
                       LZ=nz * 10.0, ENCUT=1.2e-3, ETA=2.4622e-9, NKX=1, NKY=2, TEMPERATURE=1.0,
                       MU=1.0e-3, N_circle=5, N_line_per_eV=4000, TRANSMISSION_GRID=(0.0, 2.01e-3, 8),
                       LDOS_ENERGY_GRID=(0.0, 2.0e-3, 3), LDOS_GRID=(-1, -1, 0))
    (tmp_path / "INPUT").write_text(
        "&INPUT\n if_transmission=.true. if_density=.true. if_LDOS=.true.\n"
        f" LX={deck.LX} LY={deck.LY} LZ={deck.LZ} ENCUT={deck.ENCUT} ETA={deck.ETA}\n"
        f" NKX=1 NKY=2 TEMPERATURE={deck.TEMPERATURE} MU={deck.MU} N_circle=5 N_line_per_eV=4000\n"
        " TRANSMISSION_GRID = 0.0 2.01E-3 8\n LDOS_ENERGY_GRID = 0.0 2.0E-3 3\n LDOS_GRID = -1 -1 0\n/\n\n")
    _potential(tmp_path / "POTENTIAL", V)
    r = _run(driver, tmp_path, check=False)
    assert r.returncode == 0, (tmp_path / "OUTPUT").read_text()
    assert "DONE" in (tmp_path / "OUTPUT").read_text()
    # the driver reads POTENTIAL as written (8 significant digits)
    Vf = np.array((tmp_path / "POTENTIAL").read_text().split()[3:], float).reshape(V.shape, order="F")
    pr = P.prepare(deck, Vf)
    a = pr.atomic
    p = oracle.Problem(pr.nx, pr.ny, pr.vhat, a.LX, a.LY, a.LZ, a.V_L, a.V_R, a.ETA, pr.kpoint)

    lines = (tmp_path / "TRANSMISSION").read_text().splitlines()
    assert lines[0] == " #   Energy (eV)    Transmission_coefficient"
    data = np.loadtxt(tmp_path / "TRANSMISSION", skiprows=1)
    E = P.transmission_energies(a, 8)
    tau_ref, _ = oracle.transmission_jobs(p, E)
    np.testing.assert_allclose(data[:, 0], E * HARTREE, rtol=1e-7, atol=1e-12)
    np.testing.assert_allclose(data[:, 1], tau_ref, rtol=1e-7, atol=1e-9)

    dtext = (tmp_path / "DENSITY").read_text().split("\n", 1)
    assert [int(x) for x in dtext[0].split()] == [32, 32, nz]
    dens = np.array(dtext[1].split(), float).reshape((32, 32, nz), order="F")
    nl = P.n_line(a, 4000)
    dm, _ = oracle.density_jobs(p, 5, nl, pr.min_V, a.MU, a.GAP, a.TEMPERATURE)
    dref = oracle.density_from_matrix(dm, pr.nx, pr.ny, 32, 32, deck.LX, deck.LY, deck.LZ)
    assert np.max(np.abs(dens - dref)) <= 1e-7 * np.max(np.abs(dref))

    ltext = (tmp_path / "LDOS").read_text().split("\n", 1)
    assert [int(x) for x in ltext[0].split()] == [1, 1, nz, 3]
    ldos = np.array(ltext[1].split(), float).reshape((1, 1, nz, 3), order="F")
    e_lo, e_hi = a.LDOS_ENERGY_GRID
    for ie in range(3):
        mat = np.zeros((pr.N, pr.N, pr.Nz), np.complex128, order="F")
        for ik in range(len(pr.kpoint)):
            oracle.local_density_of_state(p, ik + 1, ie + 1, 3, e_lo, e_hi, mat)
        ref = oracle.ldos_from_matrix(mat, pr.nx, pr.ny, 32, 32, deck.LX, deck.LY, deck.LZ, (-1, -1, 0))
        assert np.max(np.abs(ldos[..., ie] - ref)) <= 1e-7 * np.max(np.abs(ref))


EMASS_DECK = """&INPUT
 if_transmission=.true. if_density=.true. if_LDOS=.true.
 LX=1000.0 LY=1000.0 LZ=60.0 ENCUT={encut!r} ETA={eta!r} EMASS={m!r}
 NKX=1 NKY=2 TEMPERATURE={t!r} MU={mu!r} N_circle=5 N_line_per_eV={nl}
 TRANSMISSION_GRID = {e1!r} {e2!r} 8
 LDOS_ENERGY_GRID = {l1!r} {l2!r} 3
 LDOS_GRID = -1 -1 0
/

"""
M_EFF = 0.067
PHYS = dict(encut=1.2e-3 / M_EFF, eta=1e-6 / HARTREE, t=1.0 / M_EFF, mu=1.0e-3 / M_EFF, nl=268,
            e1=0.0, e2=2.01e-3 / M_EFF, l1=0.0, l2=2.0e-3 / M_EFF)


def _emass_pair(tmp_path):
    """The same device written with EMASS = m* (physical units) and as the
    m*-scaled deck with m* = 1 (the reference's convention)."""
    m = M_EFF
    V = W.qpc_potential(32, 32, 6, 100.0, 6.0, 0.05, 15.0, 1.0, disorder=0.002)
    scaled = {k: (v * m if k in ("encut", "eta", "t", "mu", "e1", "e2", "l1", "l2") else v) for k, v in PHYS.items()}
    scaled["nl"] = int(math.floor(PHYS["nl"] / m + 0.5))
    a, b = tmp_path / "phys", tmp_path / "scaled"
    a.mkdir()
    b.mkdir()
    (a / "INPUT").write_text(EMASS_DECK.format(m=m, **PHYS))
    (b / "INPUT").write_text(EMASS_DECK.format(m=1.0, **scaled))
    _potential(a / "POTENTIAL", V)
    _potential(b / "POTENTIAL", m * np.array((a / "POTENTIAL").read_text().split()[3:], float).reshape(V.shape, order="F"))
    return a, b


def test_emass_key_equals_scaled_deck(driver, tmp_path):
    """EMASS = m* in the driver is the m*-scaled deck: same basis, grids, V table input."""
    a, b = _emass_pair(tmp_path)
    da = json.loads(_run(driver, a, "--check").stdout)
    db = json.loads(_run(driver, b, "--check").stdout)
    assert da["EMASS"] == M_EFF and db["EMASS"] == 1.0
    for k in ("N", "Nz", "NGX", "NGY", "nk", "N_line_per_eV"):
        assert da[k] == db[k], k
    for k in ("ETA", "ENCUT", "MU", "TEMPERATURE", "min_V", "V_sum"):
        assert math.isclose(da[k], db[k], rel_tol=1e-7), (k, da[k], db[k])
    for x, y in zip(da["TRANSMISSION_GRID"], db["TRANSMISSION_GRID"]):
        assert math.isclose(x, y, rel_tol=1e-12, abs_tol=1e-300)
    (a / "INPUT").write_text(EMASS_DECK.format(m=-1.0, **PHYS))
    r = _run(driver, a, "--check", check=False)
    assert r.returncode == 1 and "EMASS must be positive" in (a / "OUTPUT").read_text()


@pytest.mark.gpu
def test_emass_end_to_end(driver, tmp_path):
    """Driver outputs with EMASS = m*: tau and density equal those of the
    scaled deck, energies are physical (scaled / m*), LDOS is per physical eV
    (scaled x m*)."""
    a, b = _emass_pair(tmp_path)
    for d in (a, b):
        r = _run(driver, d, check=False)
        assert r.returncode == 0, (d / "OUTPUT").read_text()
    ta = np.loadtxt(a / "TRANSMISSION", skiprows=1)
    tb = np.loadtxt(b / "TRANSMISSION", skiprows=1)
    np.testing.assert_allclose(ta[:, 0] * M_EFF, tb[:, 0], rtol=1e-7, atol=1e-15)
    np.testing.assert_allclose(ta[:, 1], tb[:, 1], rtol=1e-6, atol=1e-9)
    da = np.array((a / "DENSITY").read_text().split("\n", 1)[1].split(), float)
    db = np.array((b / "DENSITY").read_text().split("\n", 1)[1].split(), float)
    assert np.max(np.abs(da - db)) <= 1e-6 * np.max(np.abs(db))
    la = np.array((a / "LDOS").read_text().split("\n", 1)[1].split(), float)
    lb = np.array((b / "LDOS").read_text().split("\n", 1)[1].split(), float)
    assert np.max(np.abs(la - M_EFF * lb)) <= 1e-6 * np.max(np.abs(M_EFF * lb))


def test_neq_key_accepts_a_bias(driver, tmp_path):
    """VDS != 0 is the reference's error unless the engine key NEQ is set."""
    (tmp_path / "INPUT").write_text("&INPUT\n LX=1 LY=1 LZ=1 NKX=1 NKY=1 if_density=.true. VDS=0.001 NEQ=.true.\n/\n")
    _potential(tmp_path / "POTENTIAL", np.zeros((4, 4, 2)))
    d = json.loads(_run(driver, tmp_path, "--check").stdout)
    assert d["NEQ"] == 1 and d["VDS"] == 0.001


@pytest.mark.gpu
def test_neq_density_end_to_end(driver, tmp_path, oracle):
    """DENSITY under a bias (NEQ = .true., VDS = 1 mV x m*) against the oracle's
    biased density matrix and PtoR."""
    nz = 6
    V = W.MSTAR * W.qpc_potential(32, 32, nz, 100.0, nz * 1.0, 0.05, 15.0, 1.0, disorder=0.002)
    vds = W.MSTAR * 1e-3
    (tmp_path / "INPUT").write_text(
        "&INPUT\n if_density=.true. NEQ=.true.\n"
        f" LX=1000.0 LY=1000.0 LZ={nz * 10.0} ENCUT=1.2E-3 ETA=2.4622D-9 VDS={vds!r}\n"
        " NKX=1 NKY=2 TEMPERATURE=1.0 MU=1.0E-3 N_circle=5 N_line_per_eV=4000\n/\n\n")
    _potential(tmp_path / "POTENTIAL", V)
    r = _run(driver, tmp_path, check=False)
    assert r.returncode == 0, (tmp_path / "OUTPUT").read_text()
    Vf = np.array((tmp_path / "POTENTIAL").read_text().split()[3:], float).reshape(V.shape, order="F")
    deck = P.InputDeck(if_density=True, LX=1000.0, LY=1000.0, LZ=nz * 10.0, ENCUT=1.2e-3, ETA=2.4622e-9,
                       NKX=1, NKY=2, TEMPERATURE=1.0, MU=1.0e-3, N_circle=5, N_line_per_eV=4000)
    pr = P.prepare(deck, Vf)
    a = pr.atomic
    p = oracle.Problem(pr.nx, pr.ny, pr.vhat, a.LX, a.LY, a.LZ, a.V_L, a.V_R, a.ETA, pr.kpoint)
    avds = vds / HARTREE
    n_window = int(math.floor(4000 * ((2 * a.GAP + abs(avds)) * HARTREE) + 0.5))
    dm, _ = oracle.density_neq(p, 5, n_window, pr.min_V, a.MU + avds / 2, a.MU - avds / 2, a.GAP, a.TEMPERATURE)
    ref = oracle.density_from_matrix(dm, pr.nx, pr.ny, 32, 32, 1000.0, 1000.0, nz * 10.0)
    dtext = (tmp_path / "DENSITY").read_text().split("\n", 1)
    dens = np.array(dtext[1].split(), float).reshape((32, 32, nz), order="F")
    assert np.max(np.abs(dens - ref)) <= 1e-7 * np.max(np.abs(ref))

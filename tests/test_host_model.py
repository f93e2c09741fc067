"""The C++ input readers (libftsp host front end) against the reference.

The golden fixtures hold what the reference's own param / sequence / mode /
ion setup derived for each case (dumped by the reference harness), so the
C++ loader is checked on the same files.  Error cases follow the reference's
messages (errHandle.cu).  Field-file tests cover the .rf format, mesh
inference, trilinear resampling and the legacy A/B column order
(fieldIO.cu, trilinear.cu).  No GPU is used.
"""
import os

import numpy as np
import pytest

import pyoracle as po
from ftspolysol_b200 import cases, derive
from ftspolysol_b200.engine import STRESS_NAMES
from ftspolysol_b200.host import Model, ModelError

GOLDEN = ["pe_small", "copoly_m2", "neutral_m2", "pe_main"]


@pytest.fixture(autouse=True)
def in_tmp(tmp_path, monkeypatch):
    """File names inside param files are relative to the working directory."""
    monkeypatch.chdir(tmp_path)


def write_case(tmp_path, g):
    text = bytes(g["param_text"]).decode()
    seq = bytes(g["sequence_text"]).decode()
    name = next(l.split("=", 1)[1].strip() for l in text.splitlines() if l.strip().startswith("sequence_file"))
    (tmp_path / "param").write_text(text)
    (tmp_path / name).write_text(seq)
    return tmp_path / "param"


def arr(ptr, n):
    return np.array([ptr[i] for i in range(n)], dtype=float)


def check_config(cfg, ref):
    assert (cfg.m1, cfg.m2, cfg.m3) == tuple(ref["m"])
    for k, v in (("L1", ref["L"][0]), ("L2", ref["L"][1]), ("L3", ref["L"][2]), ("dV", ref["dV"]), ("a", ref["a"]),
                 ("lB", ref["lB"]), ("dt", ref["dt"]), ("lambda_psi", ref["lambda_psi"]),
                 ("self_pressure", ref["self_pressure"])):
        assert getattr(cfg, k) == pytest.approx(v, rel=1e-15, abs=1e-300), k
    nm = len(ref["modes"])
    assert cfg.n_modes == nm and cfg.M == ref["M"]
    coeff, lam = arr(cfg.mode_coeff, nm), arr(cfg.mode_lambda, nm)
    gam, O = arr(cfg.mode_gamma, 2 * nm), arr(cfg.mode_O, nm * cfg.M)
    for a, md in enumerate(ref["modes"]):
        assert coeff[a] == pytest.approx(md["coeff"], rel=1e-14)
        assert lam[a] == md["lambda"]
        assert complex(gam[2 * a], gam[2 * a + 1]) == md["gamma"]
        # the same Jacobi sweep order and sign convention: bit-level agreement
        np.testing.assert_allclose(O[a * cfg.M:(a + 1) * cfg.M], md["O"], rtol=0, atol=1e-15)
    S = len(ref["species"])
    assert cfg.n_species == S
    off = 0
    for s, sp in enumerate(ref["species"]):
        N = cfg.N[s]
        assert N == len(sp["types"])
        assert cfg.num_chains[s] == sp["num_chains"]
        assert [cfg.seg_type[off + i] for i in range(N)] == sp["types"]
        np.testing.assert_array_equal(arr(cfg.seg_charge, off + N)[off:], sp["charges"])
        np.testing.assert_array_equal(arr(cfg.seg_bond, off + N)[off:], sp["bonds"])
        off += N
    J = len(ref["ions"])
    assert cfg.n_ions == J
    for j, ion in enumerate(ref["ions"]):
        assert (cfg.ion_valence[j], cfg.ion_count[j], cfg.ion_smear[j]) == (ion["valence"], ion["count"], ion["smear"])
    mask = 0
    for c in ref["stress"]:
        mask |= 1 << STRESS_NAMES.index(c)
    assert cfg.stress_mask == mask
    assert cfg.isotropic_pressure == int(ref["isotropic_pressure"])


@pytest.mark.parametrize("name", GOLDEN[:3] + ["mix_m3", "short_neutral"])
def test_loader_matches_reference_dump(name, golden_dir, tmp_path):
    g = np.load(os.path.join(golden_dir, name + ".npz"))
    m = Model(str(write_case(tmp_path, g)))
    check_config(m.config(), po.derived_from_golden(g))


@pytest.mark.parametrize("idx", [1, 2, 3, 4, 5])
def test_loader_matches_python_derivation(idx, tmp_path):
    """The benchmark workloads (up to 128^3, N = 50) through both setups."""
    case = cases.workload(idx)
    files = case.write(str(tmp_path))
    m = Model(files["param"])
    ref = derive.derive(case)
    check_config(m.config(), ref)
    info = m.info
    assert info.rho0 == pytest.approx(ref["rho0"], rel=1e-15)
    assert info.volume == pytest.approx(ref["volume"], rel=1e-15)


def test_pe_main_run_settings(golden_dir, tmp_path):
    g = np.load(os.path.join(golden_dir, "pe_main.npz"))
    m = Model(str(write_case(tmp_path, g)))
    i = m.info
    assert (i.Nt, i.Nss, i.Ntmp, i.N_stat) == (6, 2, 2, 0)
    assert i.noise == 0 and i.legacy_ab == 0


def test_modes_three_types(tmp_path):
    """M = 3 with a zero eigenvalue: the inactive mode is dropped."""
    (tmp_path / "seq").write_text("[polymer.0]\nmonomers = ABCABC\ncharges = 0 0 0 0 0 0\n")
    (tmp_path / "param").write_text("""
[grid]
m1 = 4
m2 = 4
m3 = 4
a = 1
dL = 1
[monomers]
names = [A, B, C]
[polymer]
species_count = 1
sequence_file = seq
[polymer.0]
name = p
num_chains = 3
N = 6
[interactions]
chi = [0, 1, 1; 1, 0, 1; 1, 1, 0]
xi = 0
[dynamics]
dt = 0.1
lambda = 1
""")
    m = Model(str(tmp_path / "param"))
    eig, O = m.modes()
    K = np.ones((3, 3)) - np.eye(3)
    w, _ = np.linalg.eigh(K)
    np.testing.assert_allclose(eig, sorted(w, reverse=True), atol=1e-13)
    np.testing.assert_allclose(O @ O.T, np.eye(3), atol=1e-13)
    np.testing.assert_allclose(O.T @ np.diag(eig) @ O, K, atol=1e-13)
    assert m.info.n_modes == 3   # eigenvalues 2, -1, -1: all active


BASE = """
[grid]
m1 = 4
m2 = 4
m3 = 4
a = 1
dL = 1
[polymer]
species_count = 1
sequence_file = seq
[polymer.0]
name = p
num_chains = 2
N = 4
[interactions]
chi = [0, 1; 1, 0]
xi = 1
lB = 1
[dynamics]
dt = 0.1
lambda = 1
"""
SEQ = "[polymer.0]\nmonomers = A A B B\ncharges = -1 - 0 0\n"


@pytest.mark.parametrize("extra, seq, message", [
    ("[grid]\nfoo = 1\n", SEQ, "unknown parameter [grid] foo"),
    ("[dynamics]\nNt = x\n", SEQ, "cannot parse [dynamics] Nt"),
    ("[interactions]\nchi = [0, 1; 2, 0]\n", SEQ, "invalid chi matrix must be symmetric"),
    ("[interactions]\nchi = [1, 1; 1, 0]\n", SEQ, "invalid chi diagonal entries must be zero"),
    ("[dynamics]\nlambda = [1, 2, 3]\n", SEQ, "invalid lambda_omega length must be 1 or the number of active interaction modes"),
    ("", "[polymer.0]\nmonomers = A A B\ncharges = 0 0 0\n", "sequence length mismatch for p"),
    ("", "[polymer.0]\nmonomers = A A B C\ncharges = 0 0 0 0\n", "invalid unknown monomer label in sequence: C"),
    ("", "[polymer.0]\nmonomers = AABB\n", "missing charges for polymer.0"),
    ("[ions]\nenabled = true\n[ions.counterions]\nenabled = true\nvalence = 3\n", SEQ, "invalid counterion number"),
    ("", SEQ, "electroneutrality failed"),
    ("[observables]\ncomponent_xx = true\n", SEQ,
     "invalid stress components or isotropic_pressure require [observables] stress = true"),
    ("[output]\nstep_psi_file = a/%d/psi.rf\n", SEQ, "invalid step output template (use exactly one %d in the file name)"),
])
def test_reference_error_messages(tmp_path, extra, seq, message):
    (tmp_path / "seq").write_text(seq)
    (tmp_path / "param").write_text(BASE + extra)
    with pytest.raises(ModelError) as e:
        Model(str(tmp_path / "param"))
    assert str(e.value) == message


def test_parse_conveniences(tmp_path):
    """Comments, quotes, multi-line brackets, compact labels, '+'/'-' charges."""
    (tmp_path / "my seq").write_text("# seq\n[polymer.0]\nmonomers = ABBA\ncharges = +,-, +2 -0.5  # c\n"
                                     "bonds = 1, 1.5\nbonds = 2\n")
    (tmp_path / "param").write_text(BASE.replace("sequence_file = seq", 'sequence_file = "my seq"  # quoted')
                                    .replace("chi = [0, 1; 1, 0]", "chi = [\n  [0, 1],  # row\n  [1, 0]\n]")
                                    + "[ions]\nenabled = yes\n[ions.counterions]\nenabled = on\nvalence = -0.5\n")
    m = Model(str(tmp_path / "param"))
    cfg = m.config()
    assert [cfg.seg_type[i] for i in range(4)] == [0, 1, 1, 0]
    assert arr(cfg.seg_charge, 4).tolist() == [1.0, -1.0, 2.0, -0.5]
    assert arr(cfg.seg_bond, 4).tolist() == [1.0, 1.5, 2.0, 1.0]
    # net chain charge 1.5 on 2 chains: auto_neutralize gives 6 counterions of valence -0.5
    assert cfg.n_ions == 1 and (cfg.ion_valence[0], cfg.ion_count[0]) == (-0.5, 6.0)
    assert cfg.ion_smear[0] == 1.0   # default smearing length = a


def test_field_round_trip_and_formats(tmp_path, golden_dir):
    g = np.load(os.path.join(golden_dir, "copoly_m2.npz"))
    m = Model(str(write_case(tmp_path, g)))
    rng = np.random.default_rng(3)
    om = rng.normal(size=(m.info.n_modes, m.size)) + 1j * rng.normal(size=(m.info.n_modes, m.size))
    ps = rng.normal(size=m.size) + 1j * rng.normal(size=m.size)
    m.write_omega(str(tmp_path / "w.rf"), om)
    m.write_fields(str(tmp_path / "p.rf"), ps)
    lines = (tmp_path / "w.rf").read_text().splitlines()
    assert lines[0] == "8 6 12"
    assert lines[1] == "%.17g %.17g %.17g" % (8 * 0.6, 6 * 0.6, 12 * 0.6)
    assert lines[2] == "%.10f  %.10f  %.10f  %.10f" % (om[0, 0].real, om[0, 0].imag, om[1, 0].real, om[1, 0].imag)
    om2, ps2 = m.read_fields(str(tmp_path / "w.rf"), str(tmp_path / "p.rf"))
    np.testing.assert_allclose(om2, om, atol=5.1e-11)
    np.testing.assert_allclose(ps2, ps, atol=5.1e-11)


def trilinear_np(f, n, m):
    """Periodic trilinear resampling written from the definition."""
    out = np.zeros(m, dtype=complex)
    for x in range(m[0]):
        for y in range(m[1]):
            for z in range(m[2]):
                idx, w = [], []
                for i, (c, nn, mm) in enumerate(zip((x, y, z), n, m)):
                    s = c * nn / mm
                    i0 = int(np.floor(s))
                    idx.append((i0 % nn, (i0 + 1) % nn if nn > 1 else 0))
                    w.append(s - i0 if nn > 1 else 0.0)
                v = 0
                for a in (0, 1):
                    for b in (0, 1):
                        for c in (0, 1):
                            wt = (w[0] if a else 1 - w[0]) * (w[1] if b else 1 - w[1]) * (w[2] if c else 1 - w[2])
                            v += wt * f[idx[0][a], idx[1][b], idx[2][c]]
                out[x, y, z] = v
    return out.ravel()


def test_mesh_inference_and_resize(tmp_path, golden_dir):
    """Header-less files on half the mesh are inferred and upsampled."""
    g = np.load(os.path.join(golden_dir, "copoly_m2.npz"))
    m = Model(str(write_case(tmp_path, g)))
    n = (4, 3, 6)
    rng = np.random.default_rng(5)
    src = rng.normal(size=(2,) + n) + 1j * rng.normal(size=(2,) + n)
    psrc = rng.normal(size=n) + 1j * rng.normal(size=n)
    with open(tmp_path / "w_half.rf", "w") as f:
        for i in range(int(np.prod(n))):
            a, b = src[0].ravel()[i], src[1].ravel()[i]
            f.write("%.12f %.12f %.12f %.12f\n" % (a.real, a.imag, b.real, b.imag))
    with open(tmp_path / "p_half.rf", "w") as f:
        for v in psrc.ravel():
            f.write("%.12f %.12f\n" % (v.real, v.imag))
    om, ps = m.read_fields(str(tmp_path / "w_half.rf"), str(tmp_path / "p_half.rf"))
    for a in range(2):
        np.testing.assert_allclose(om[a], trilinear_np(np.round(src[a].real, 12) + 1j * np.round(src[a].imag, 12), n, m.mesh),
                                   atol=1e-11)
    np.testing.assert_allclose(ps, trilinear_np(np.round(psrc.real, 12) + 1j * np.round(psrc.imag, 12), n, m.mesh), atol=1e-11)


def test_missing_default_omega_gives_zero(tmp_path, golden_dir):
    g = np.load(os.path.join(golden_dir, "pe_small.npz"))
    p = write_case(tmp_path, g)
    m = Model(str(p))
    om, ps = m.read_fields()
    assert not om.any() and not ps.any()
    with pytest.raises(ModelError, match="cannot open nothere.rf: No such file"):
        m.read_fields("nothere.rf")


def test_legacy_ab_order(tmp_path):
    """No [monomers] / chi: two columns map to composition / density modes."""
    (tmp_path / "seq").write_text("[polymer.0]\nmonomers = A A B B\ncharges = 0 0 0 0\n")
    (tmp_path / "param").write_text(BASE.replace("chi = [0, 1; 1, 0]\n", "").replace("lB = 1", "lB = 0"))
    m = Model(str(tmp_path / "param"))
    assert m.info.legacy_ab == 1
    eig, _ = m.modes()
    rng = np.random.default_rng(9)
    f = rng.normal(size=(2, m.size)) + 1j * rng.normal(size=(2, m.size))
    m.write_fields(str(tmp_path / "ab.rf"), f)
    om, _ = m.read_fields(str(tmp_path / "ab.rf"), str(tmp_path / "none.rf"))
    # K = xi everywhere: one positive (density) mode; the composition mode is inactive
    assert m.info.n_modes == 1 and eig[0] > 0
    np.testing.assert_allclose(om[0], f[1], atol=5.1e-11)
    m.write_omega(str(tmp_path / "ab_out.rf"), om)
    back = np.loadtxt(tmp_path / "ab_out.rf", skiprows=2)
    np.testing.assert_allclose(back[:, 0], 0)
    np.testing.assert_allclose(back[:, 2] + 1j * back[:, 3], f[1], atol=1e-10)

"""The reference-style program (ftsp_main) against the reference's own run.

The golden fixture pe_main holds every file the unmodified reference
executable wrote for a noise-free polyelectrolyte case (16 x 12 x 8 mesh,
counterions + salt, Nt = 6, Nss = 2, Ntmp = 2, N_stat = 0, stress and
isotropic pressure): observables.dat with its ensemble average,
drift_max.dat, the tmp checkpoints and the final fields and densities.  The
same command line runs through ftsp_main here and every file is compared:
comment and label lines as text, numbers to the printed precision.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from ftspolysol_b200 import cases

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
EXE = os.path.join(ROOT, "ftspolysol_b200", "ftsp_main")
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

pytestmark = pytest.mark.gpu


def run(args, cwd, check=True):
    if not os.path.exists(EXE):
        pytest.fail("ftsp_main is not built (python -m ftspolysol_b200.build)")
    r = subprocess.run([EXE] + list(args), cwd=cwd, capture_output=True, text=True, timeout=600)
    if check and r.returncode != 0:
        raise AssertionError("ftsp_main failed (%d):\n%s\n%s" % (r.returncode, r.stdout[-2000:], r.stderr[-2000:]))
    return r


def compare_table(mine: str, ref: str, rtol: float, atol: float, what: str):
    a, b = mine.splitlines(), ref.splitlines()
    assert len(a) == len(b), (what, len(a), len(b))
    for la, lb in zip(a, b):
        if lb.startswith("#") or not lb.strip():
            assert la == lb, (what, la, lb)
            continue
        ta, tb = la.split(), lb.split()
        assert len(ta) == len(tb), what
        assert ta[0] == tb[0], what
        np.testing.assert_allclose(np.array(ta[1:], float), np.array(tb[1:], float), rtol=rtol, atol=atol, err_msg=what)


def compare_rf(mine: str, ref: str, atol: float, what: str):
    a, b = mine.splitlines(), ref.splitlines()
    assert a[:2] == b[:2], what          # mesh and box header lines
    assert len(a) == len(b), what
    va = np.array([l.split() for l in a[2:]], float)
    vb = np.array([l.split() for l in b[2:]], float)
    np.testing.assert_allclose(va, vb, rtol=0, atol=atol, err_msg=what)


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(HERE, "golden", "pe_main.npz"))


def write_main_case(tmp_path, g):
    case = make_golden.main_case()
    paths = case.write(str(tmp_path), omega=g["input_omega"], psi=g["input_psi"])
    return [os.path.basename(paths[k]) for k in ("param", "omega", "psi")]


def test_main_reproduces_reference_files(tmp_path, golden):
    param, om, ps = write_main_case(tmp_path, golden)
    run(["-p", param, "--omega", om, "--psi", ps, "--seed", "1"], str(tmp_path))
    names = [k[len("file__"):] for k in golden.files if k.startswith("file__")]
    assert sorted(os.path.basename(n) for n in names) == sorted(names)
    for n in names:
        path = tmp_path / n
        assert path.exists(), n
        ref = bytes(golden["file__" + n]).decode()
        mine = path.read_text()
        if n.endswith(".dat"):
            # values printed with %.10e; the trajectories agree to ~1e-12
            compare_table(mine, ref, rtol=2e-9, atol=1e-13, what=n)
        else:
            # %.10f columns: one unit in the last printed place
            compare_rf(mine, ref, atol=1.5e-10, what=n)


def test_main_fp32_tracks_reference(tmp_path, golden):
    param, om, ps = write_main_case(tmp_path, golden)
    run(["-p", param, "--omega", om, "--psi", ps, "--fp32"], str(tmp_path))
    compare_table((tmp_path / "observables.dat").read_text(), bytes(golden["file__observables.dat"]).decode(),
                  rtol=2e-4, atol=1e-6, what="observables.dat (complex64)")
    compare_rf((tmp_path / "omega.rf").read_text(), bytes(golden["file__omega.rf"]).decode(), atol=2e-5, what="omega.rf")


def test_main_semi_implicit_runs(tmp_path, golden):
    """--si changes the update rule (no reference counterpart): same files,
    same columns, finite values, and the k = 0 behaviour of the explicit step
    (the chain terms vanish there)."""
    param, om, ps = write_main_case(tmp_path, golden)
    run(["-p", param, "--omega", om, "--psi", ps, "--si"], str(tmp_path))
    ref = bytes(golden["file__observables.dat"]).decode().splitlines()
    mine = (tmp_path / "observables.dat").read_text().splitlines()
    assert [l for l in mine if l.startswith("#")] == [l for l in ref if l.startswith("#")]
    rows = [l.split() for l in mine if l.strip() and not l.startswith("#")]
    assert [r[0] for r in rows] == ["2", "4", "6", "average"]
    assert np.isfinite(np.array([r[1:] for r in rows], float)).all()


def small_case(**kw):
    base = dict(name="runner", m=(8, 8, 8), dL=0.5, a=1.0, monomer_names=["A"], chi=[0.0], xi=0.1, lB=1.0,
                species=[cases.homopolymer("P", 4, 8)], counterions={"number": "auto_neutralize", "valence": 1.0},
                dt=0.01, Nt=4, Nss=0, Ns=0, Ntmp=0, N_stat=-1, noise=True, init_seed=3)
    base.update(kw)
    return cases.Case(**base)


def test_run_directory_and_step_outputs(tmp_path):
    case = small_case(Nt=3, Nso=1, extra_output={"step_omega_file": "snap_%d.rf", "step_rhop_file": "rhop_%d.rf",
                                                 "step_ion_density_prefix": "ions_%d"})
    paths = case.write(str(tmp_path))
    text = open(paths["param"]).read()
    run(["-p", os.path.basename(paths["param"]), "--omega", os.path.basename(paths["omega"]), "--psi",
         os.path.basename(paths["psi"]), "-i", "r1", "-s", "out", "--seed", "7"], str(tmp_path))
    rd = tmp_path / "out" / "r1"
    assert (rd / "r1.param").read_text() == text
    assert (rd / "r1.sequence").exists()
    for s in (1, 2, 3):
        assert (rd / "snap" / ("snap_%d.rf" % s)).exists()
        assert (rd / "rhop" / ("rhop_%d.rf" % s)).exists()
        assert (rd / "ions" / ("ions_%d_0_counterion.rf" % s)).exists()
    # the last step output is the state the final files are written from
    compare_rf((rd / "snap" / "snap_3.rf").read_text(), (rd / "omega.rf").read_text(), atol=0, what="omega")
    compare_rf((rd / "rhop" / "rhop_3.rf").read_text(), (rd / "rhop.rf").read_text(), atol=0, what="rhop")
    obs = (rd / "observables.dat").read_text().splitlines()
    assert [l.split()[0] for l in obs if l.strip() and not l.startswith("#")] == ["1", "2", "3", "average"]
    assert "# ensemble_average Nss=0 Ns=3 count=3" in obs


def test_same_seed_same_run(tmp_path):
    case = small_case()
    outs = []
    for k in range(2):
        d = tmp_path / str(k)
        paths = case.write(str(d))
        run(["-p", os.path.basename(paths["param"]), "--omega", os.path.basename(paths["omega"]), "--psi",
             os.path.basename(paths["psi"]), "--seed", "11"], str(d))
        outs.append((d / "observables.dat").read_text())
    assert outs[0] == outs[1]


def test_restarts_from_checkpoint_then_gives_up(tmp_path):
    """A step size that overflows exp(-W) at every attempt: each failure
    rolls back to the step-0 checkpoint, the observable file is reopened with
    the restart note, and after max_nan_restarts the program stops with the
    reference's message (complexLangevin.cu:600-609)."""
    case = small_case(dt=1.0e6, Nt=3, Ntmp=1, N_stat=0, max_nan_restarts=2)
    paths = case.write(str(tmp_path))
    r = run(["-p", os.path.basename(paths["param"]), "--omega", os.path.basename(paths["omega"]), "--psi",
             os.path.basename(paths["psi"])], str(tmp_path), check=False)
    assert r.returncode == 1
    assert "error: maximum non-finite restarts exceeded" in r.stderr
    assert r.stderr.count("error: non-finite value at step 1") == 3
    obs = (tmp_path / "observables.dat").read_text()
    assert "# restarted after non-finite value at step 1 from checkpoint step 0; previous observable records discarded" in obs
    drift = (tmp_path / "drift_max.dat").read_text()
    assert "previous drift statistics discarded" in drift
    # the checkpoint is the input state
    om = np.loadtxt(tmp_path / "tmp_omega.rf", skiprows=2)
    ref_om, _ = case.initial_fields()
    np.testing.assert_allclose(om[:, 0] + 1j * om[:, 1], np.atleast_2d(ref_om)[0], atol=1e-10)


def test_legacy_inputs_run_directory_and_step_outputs_match_reference(tmp_path):
    """A second run of the unmodified reference executable: legacy A/B input
    (no [monomers], no chi: the two omega columns map to the modes), a
    header-less psi file on half the mesh (mesh inference and trilinear
    resampling), unmerged salt ions, a run directory (-i/-s), step outputs
    in template folders, checkpoints every 2 steps and drift statistics
    after step 1.  Every file the reference wrote is compared."""
    g = np.load(os.path.join(HERE, "golden", "legacy_main.npz"))
    args = make_golden.write_legacy(str(tmp_path))
    run(args + ["--seed", "3"], str(tmp_path))
    out = tmp_path / "out"
    names = sorted(k[len("file__"):] for k in g.files)
    mine = sorted(str(p.relative_to(out)) for p in out.rglob("*") if p.is_file())
    assert mine == names
    for n in names:
        ref = bytes(g["file__" + n]).decode()
        text = (out / n).read_text()
        if n.endswith((".param", ".sequence")):
            assert text == ref, n
        elif n.endswith(".dat"):
            compare_table(text, ref, rtol=2e-9, atol=1e-13, what=n)
        else:
            compare_rf(text, ref, atol=1.5e-10, what=n)


def test_adaptive_step_option(tmp_path):
    """--adaptive with a bound never reached reproduces the fixed-step run
    file for file; a tight bound changes the trajectory and still finishes."""
    case = small_case(Nt=5)
    outs = []
    for k, extra in enumerate(([], ["--adaptive", "1e30"], ["--adaptive", "0.05"])):
        d = tmp_path / str(k)
        paths = case.write(str(d))
        run(["-p", os.path.basename(paths["param"]), "--omega", os.path.basename(paths["omega"]), "--psi",
             os.path.basename(paths["psi"]), "--seed", "4"] + extra, str(d))
        outs.append(((d / "observables.dat").read_text(), (d / "omega.rf").read_text()))
    assert outs[0] == outs[1]
    assert outs[2][1] != outs[0][1]

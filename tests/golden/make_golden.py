"""Generate the golden vectors under tests/golden/ from the REFERENCE build.

Runs oracle/_ref/ref_harness (the reference's own sources, built by
oracle/build_ref.sh) on small seeded cases and packs its dumps into one
``<case>.npz`` per case.  It needs a CUDA GPU (the reference is CUDA-only), so
it is run once on a GPU machine:

    python tests/golden/make_golden.py <outdir>

and the resulting .npz files are committed under tests/golden/.  The cases
cover: the polyelectrolyte chemistry of the 32^3 workload on a small ragged
grid with injected noise; a two-type copolymer blend (two species, per-bond
lengths, mixed charges, both mode signatures gamma = i and gamma = 1, salt
with 2:1 stoichiometry, unmerged ion species, partial stress components);
an uncharged two-type melt (electrostatics off); three monomer types with a
one-bead charged species on an odd grid; dimers and monomers without
electrostatics; and a noise-free run of the unmodified reference executable
for the step-loop output files.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from ftspolysol_b200.cases import Case, Species, homopolymer  # noqa: E402


def golden_cases():
    cases = []
    # 1. polyelectrolyte chemistry of the 32^3 workload on a 12x8x16 grid.
    V = (12 * 0.5) * (8 * 0.5) * (16 * 0.5)
    c = Case(name="pe_small", m=(12, 8, 16), dL=0.5, a=1.0, monomer_names=["A"], chi=[0.0],
             xi=0.1, lB=1.0, species=[homopolymer("P", int(round(0.5 * V / 8)), 8)],
             counterions={"number": "auto_neutralize", "valence": 1.0},
             salt={"num_salt": int(round(0.1 * V)), "cation_valence": 1.0, "anion_valence": -1.0},
             dt=0.01, lambda_omega=[1.0], lambda_psi=1.0, Nt=3, noise=True,
             stress=("xx", "yy", "zz", "xy", "xz", "yz"), isotropic_pressure=True, init_seed=11)
    cases.append((c, 3))
    # 2. copolymer blend with everything switched on.
    diblock = Species(name="AB", num_chains=10, monomers=list("AAABBB"),
                      charges=[-1.0, -1.0, 0.0, 0.0, 0.5, 0.5], bonds=[1.0, 1.0, 1.2, 0.8, 1.0])
    homoB = Species(name="Bh", num_chains=6, monomers=list("BBBB"), charges=[1.0, 0.0, 1.0, 0.0])
    c = Case(name="copoly_m2", m=(8, 6, 12), dL=0.6, a=0.9, monomer_names=["A", "B"],
             chi=[0.0, 1.5, 1.5, 0.0], xi=0.2, lB=0.7, species=[diblock, homoB],
             counterions={"number": "auto_neutralize", "valence": -1.0, "smearing_length": 0.8, "name": "ci"},
             salt={"num_salt": 5, "cation_valence": 2.0, "anion_valence": -1.0, "cation_stoich": 1,
                   "anion_stoich": 2, "smearing_length": 0.7, "cation_name": "Mg", "anion_name": "Cl"},
             dt=0.02, lambda_omega=[1.0, 0.5], lambda_psi=0.8, Nt=3, noise=True,
             stress=("xx", "xy", "yz"), isotropic_pressure=True, init_seed=22)
    cases.append((c, 3))
    # 3. uncharged melt, electrostatics off, ions off.
    dib = Species(name="AB", num_chains=20, monomers=list("AAAABBBB"), charges=[0.0] * 8)
    c = Case(name="neutral_m2", m=(12, 9, 8), dL=0.5, a=1.0, monomer_names=["A", "B"],
             chi=[0.0, 0.8, 0.8, 0.0], xi=0.05, lB=0.0, species=[dib], ions_enabled=False,
             dt=0.02, lambda_omega=[1.0], lambda_psi=0.0, Nt=3, noise=True,
             stress=("yy", "zz", "xz"), isotropic_pressure=True, init_seed=33)
    cases.append((c, 3))
    # 4. three monomer types (three active modes of mixed signature), a
    #    triblock with per-bond lengths, a one-bead charged species (N = 1),
    #    counterions and salt, on an odd non-cubic grid.
    tri = Species(name="ABC", num_chains=8, monomers=list("AABBCCC"), charges=[-1.0, 0.0, -1.0, 0.0, 1.0, 0.0, -1.0],
                  bonds=[1.0, 0.9, 1.1, 1.0, 1.3, 0.8])
    ion1 = Species(name="M2", num_chains=12, monomers=["C"], charges=[2.0])
    c = Case(name="mix_m3", m=(10, 12, 9), dL=0.55, a=1.0, monomer_names=["A", "B", "C"],
             chi=[0.0, 1.0, 0.5, 1.0, 0.0, 0.5, 0.5, 0.5, 0.0], xi=0.1, lB=1.2, species=[tri, ion1],
             counterions={"number": "auto_neutralize", "valence": -1.0},
             salt={"num_salt": 6, "cation_valence": 1.0, "anion_valence": -1.0},
             dt=0.01, lambda_omega=[1.0, 0.7, 0.5], lambda_psi=1.0, Nt=3, noise=True,
             stress=("xx", "yy", "zz", "xy", "xz", "yz"), isotropic_pressure=True, init_seed=55)
    cases.append((c, 3))
    # 5. short chains without electrostatics: dimers (N = 2) and monomers
    #    (N = 1) of one type, no ions.
    c = Case(name="short_neutral", m=(8, 8, 8), dL=0.5, a=1.0, monomer_names=["A"], chi=[0.0], xi=0.2, lB=0.0,
             species=[Species(name="D", num_chains=40, monomers=["A", "A"], charges=[0.0, 0.0]),
                      Species(name="S", num_chains=60, monomers=["A"], charges=[0.0])],
             ions_enabled=False, dt=0.01, lambda_omega=[1.0], lambda_psi=0.0, Nt=3, noise=True,
             stress=("xx", "zz", "xy"), isotropic_pressure=True, init_seed=66)
    cases.append((c, 3))
    return cases


def main_case():
    """Noise-free case run through the unmodified reference executable."""
    V = (16 * 0.5) * (12 * 0.5) * (8 * 0.5)
    return Case(name="pe_main", m=(16, 12, 8), dL=0.5, a=1.0, monomer_names=["A"], chi=[0.0],
                xi=0.1, lB=1.0, species=[homopolymer("P", int(round(0.5 * V / 16)), 16)],
                counterions={"number": "auto_neutralize", "valence": 1.0},
                salt={"num_salt": int(round(0.1 * V)), "cation_valence": 1.0, "anion_valence": -1.0},
                dt=0.01, Nt=6, Nss=2, Ns=0, Ntmp=2, N_stat=0, noise=False,
                stress=("xx", "yy", "zz"), isotropic_pressure=True, init_seed=44)


LEGACY_PARAM = """# legacy A/B input: no [monomers] section and no chi matrix
[grid]
m1 = 12
m2 = 10
m3 = 8
a = 1.0
dL = 0.5

[polymer]
species_count = 2
sequence_file = legacy.seq

[polymer.0]
name = AB
num_chains = 6
N = 8

[polymer.1]
name = Bh
num_chains = 4
N = 5

[interactions]
xi = 0.15
lB = 0.8

[dynamics]
dt = 0.01
lambda_omega = 1.0
lambdaPsi = 0.9
Nt = 4
Nss = 0
Ns = 3
Ntmp = 2
Nso = 1
N_stat = 1
noise = false

[ions]
enabled = true
[ions.counterions]
enabled = true
number = auto_neutralize
valence = 1
[ions.salt]
enabled = true
num_salt = 7
cation_valence = 1
anion_valence = -1
combine_identical_species = false

[observables]
stress = true
component_xy = true
component_zz = true
isotropic_pressure = true

[output]
step_omega_file = snap_%d.rf
step_rhoc_file = rhoc_%d.rf
step_ion_density_prefix = ions_%d
"""

LEGACY_SEQ = """[polymer.0]
monomers = A A A A B B B B
charges = -1 0 -1 0 0 -1 0 -1
bonds = 1 1 1.2 1 1 0.9 1
[polymer.1]
monomers = BBBBB
charges = -,0,-,0,-
"""


def legacy_inputs(seed: int = 77):
    """Legacy two-column omega file on the full mesh and a header-less psi
    file on half the mesh (the reference infers the mesh and resamples it)."""
    rng = np.random.default_rng(seed)
    m = (12, 10, 8)
    V = 12 * 10 * 8
    om = 0.1 * rng.standard_normal((2, V))
    ps = 0.1 * rng.standard_normal(6 * 5 * 4)
    return m, om, ps


def write_legacy(work: str):
    m, om, ps = legacy_inputs()
    with open(os.path.join(work, "legacy.param"), "w") as f:
        f.write(LEGACY_PARAM)
    with open(os.path.join(work, "legacy.seq"), "w") as f:
        f.write(LEGACY_SEQ)
    with open(os.path.join(work, "w_ab.rf"), "w") as f:
        f.write("%d %d %d\n" % m)
        f.write("6 5 4\n")
        for i in range(om.shape[1]):
            f.write("%.12f %.12f %.12f %.12f\n" % (om[0, i], 0.0, om[1, i], 0.0))
    with open(os.path.join(work, "psi_half.rf"), "w") as f:
        for v in ps:
            f.write("%.12f %.12f\n" % (v, 0.0))
    return ["-p", "legacy.param", "--omega", "w_ab.rf", "--psi", "psi_half.rf", "-i", "run1", "-s", "out"]


def noise_for(case: Case, steps: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    nm = case.active_mode_count()
    dV = case.dL ** 3
    out = np.zeros((steps, nm + 1, case.size))
    for a in range(nm):
        lam = case.lambda_omega[a] if len(case.lambda_omega) > 1 else case.lambda_omega[0]
        out[:, a, :] = np.sqrt(2.0 * lam * case.dt / dV) * rng.standard_normal((steps, case.size))
    if case.lB > 0.0:
        out[:, nm, :] = np.sqrt(2.0 * case.lambda_psi * case.dt / dV) * rng.standard_normal((steps, case.size))
    return out


def load_dump(directory: str) -> dict:
    out = {}
    with open(os.path.join(directory, "manifest.txt")) as f:
        for line in f:
            name, shape = line.split()
            dims = tuple(int(v) for v in shape.split(","))
            data = np.fromfile(os.path.join(directory, name + ".bin"), dtype="<f8")
            if len(dims) >= 2 and dims[-1] == 2:
                data = data.reshape(dims)
                data = data[..., 0] + 1j * data[..., 1]
            else:
                data = data.reshape(dims)
            out[name] = data
    return out


def run(outdir: str, harness: str, main_exe: str, only=None) -> None:
    os.makedirs(outdir, exist_ok=True)
    for case, steps in golden_cases():
        if only and case.name not in only:
            continue
        work = tempfile.mkdtemp(prefix="golden_" + case.name + "_")
        paths = case.write(work)
        noise = noise_for(case, steps, seed=1000 + case.init_seed)
        noise_path = os.path.join(work, "noise.bin")
        noise.astype("<f8").tofile(noise_path)
        dump = os.path.join(work, "dump")
        os.makedirs(dump)
        subprocess.run([harness, "golden", os.path.basename(paths["param"]), paths["omega"], paths["psi"], dump,
                        str(steps), noise_path], cwd=work, check=True)
        arrays = load_dump(dump)
        arrays["noise"] = noise
        arrays["param_text"] = np.frombuffer(case.param_text().encode(), dtype=np.uint8)
        arrays["sequence_text"] = np.frombuffer(case.sequence_text().encode(), dtype=np.uint8)
        np.savez_compressed(os.path.join(outdir, case.name + ".npz"), **arrays)
        shutil.rmtree(work)
        print("golden case", case.name, "->", len(arrays), "arrays")

    if not only or "legacy_main" in only:
        work = tempfile.mkdtemp(prefix="golden_legacy_")
        args = write_legacy(work)
        subprocess.run([main_exe] + args, cwd=work, check=True, stdout=subprocess.DEVNULL)
        files = {}
        base = os.path.join(work, "out")
        for dirpath, _, names in os.walk(base):
            for name in names:
                full = os.path.join(dirpath, name)
                files["file__" + os.path.relpath(full, base)] = np.frombuffer(open(full, "rb").read(), dtype=np.uint8)
        np.savez_compressed(os.path.join(outdir, "legacy_main.npz"), **files)
        shutil.rmtree(work)
        print("golden legacy run ->", sorted(files))
    if only and "pe_main" not in only:
        return
    case = main_case()
    work = tempfile.mkdtemp(prefix="golden_main_")
    paths = case.write(work)
    subprocess.run([main_exe, "-p", os.path.basename(paths["param"]), "--omega", paths["omega"],
                    "--psi", paths["psi"]], cwd=work, check=True, stdout=subprocess.DEVNULL)
    files = {}
    for name in sorted(os.listdir(work)):
        full = os.path.join(work, name)
        if os.path.isfile(full) and not name.endswith((".param", ".seq")) and name not in (
                os.path.basename(paths["omega"]), os.path.basename(paths["psi"])):
            files["file__" + name] = np.frombuffer(open(full, "rb").read(), dtype=np.uint8)
    omega, psi = case.initial_fields()
    files["input_omega"] = omega
    files["input_psi"] = psi
    files["param_text"] = np.frombuffer(case.param_text().encode(), dtype=np.uint8)
    files["sequence_text"] = np.frombuffer(case.sequence_text().encode(), dtype=np.uint8)
    np.savez_compressed(os.path.join(outdir, case.name + ".npz"), **files)
    shutil.rmtree(work)
    print("golden main run ->", sorted(k for k in files if k.startswith("file__")))


if __name__ == "__main__":
    out = sys.argv[1] if len(sys.argv) > 1 else HERE
    only = set(sys.argv[2].split(",")) if len(sys.argv) > 2 else None   # e.g. mix_m3,short_neutral
    ref = os.path.join(ROOT, "oracle", "_ref")
    run(out, os.path.join(ref, "ref_harness"), os.path.join(ref, "main"), only)

"""Input-case writers: param files, sequence files and seeded ``.rf`` fields.

The files follow the reference's input surface exactly:

* the INI-like param file read by ``param::read`` / ``param::apply``
  (FTSPolySol ``param.cu:165-334``): ``[section]`` headers, ``key = value``,
  ``#`` comments, bracketed lists;
* the block sequence file read by ``polymerSpecies::read_block_sequence_file``
  (``polymer.cu:219-273``): ``[polymer.K]`` blocks with ``monomers=``,
  ``charges=`` and optional ``bonds=`` (N-1 values);
* the ``.rf`` field format of ``fieldIO`` (``common.h:375-472``,
  ``fieldIO.cu:480-511``): an ``m1 m2 m3`` line, an ``L1 L2 L3`` line, then one
  row per grid point (row-major, z fastest) holding ``re im`` pairs, one pair
  per field.  Fields are written with ``%.17g`` so a reader gets the exact
  doubles back.

The five named workloads (``workload(1..5)``) are the polyelectrolyte
solution studied by this engine: flexible discrete Gaussian chains with every
bead charged -1, Gaussian-smeared beads (a = b = 1), bead density 0.5 b^-3,
Edwards excluded volume v = 0.1 b^3, Bjerrum length 1 b, point counterions
that neutralise the chains, and 1:1 salt.  Counts are rounded to integers the
way a param file must state them.
"""
from __future__ import annotations

import dataclasses
import math
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

STRESS_COMPONENTS = ("xx", "yy", "zz", "xy", "xz", "yz")


@dataclass
class Species:
    name: str
    num_chains: int
    monomers: List[str]
    charges: List[float]
    bonds: Optional[List[float]] = None

    @property
    def N(self) -> int:
        return len(self.monomers)


@dataclass
class Case:
    name: str
    m: Sequence[int] = (16, 16, 16)
    dL: float = 0.5
    a: float = 1.0
    monomer_names: List[str] = field(default_factory=lambda: ["A"])
    chi: Optional[List[float]] = None          # M*M row-major, zero diagonal
    xi: float = 0.1
    lB: float = 1.0
    eigen_tol_rel: float = 1.0e-12
    species: List[Species] = field(default_factory=list)
    ions_enabled: bool = True
    default_smearing_length: Optional[float] = None
    counterions: Optional[Dict] = None         # keys: number, valence, smearing_length, name
    salt: Optional[Dict] = None                # keys: num_salt, cation_valence, anion_valence, *_stoich, smearing_length
    dt: float = 0.005
    lambda_omega: List[float] = field(default_factory=lambda: [1.0])
    lambda_psi: float = 1.0
    Nt: int = 10
    Nss: int = 0
    Ns: int = 0
    Ntmp: int = 0
    Nso: int = -1
    N_stat: int = -1
    max_nan_restarts: int = 20
    noise: bool = True
    stress: Sequence[str] = ()                 # subset of STRESS_COMPONENTS
    isotropic_pressure: bool = False
    init_seed: int = 1234
    init_std: float = 0.1
    observable_file: str = "observables.dat"
    drift_max_file: str = "drift_max.dat"
    extra_output: Dict[str, str] = field(default_factory=dict)

    # ---- derived quantities (host restatement of param::derive) ----
    @property
    def M(self) -> int:
        return len(self.monomer_names)

    @property
    def size(self) -> int:
        return int(self.m[0]) * int(self.m[1]) * int(self.m[2])

    @property
    def L(self):
        return tuple(self.dL * mi for mi in self.m)

    @property
    def volume(self) -> float:
        L = self.L
        return L[0] * L[1] * L[2]

    def chi_matrix(self) -> np.ndarray:
        if self.chi is None:
            return np.zeros((self.M, self.M))
        return np.asarray(self.chi, dtype=np.float64).reshape(self.M, self.M)

    def active_mode_count(self) -> int:
        """Number of interaction modes with |d| above the tolerance
        (``interactionMode::diagonalize``, ``interactionMode.cu:253-262``)."""
        chi = self.chi_matrix()
        K = self.xi + chi
        np.fill_diagonal(K, self.xi)
        d = np.linalg.eigvalsh(K)
        tol = self.eigen_tol_rel * max(1.0, float(np.max(np.abs(d))))
        return int(np.sum(np.abs(d) > tol))

    # ---- writers ----
    def param_text(self) -> str:
        L = []
        L.append("# generated by ftspolysol_b200.cases for workload %s" % self.name)
        L.append("[grid]")
        L.append("m1 = %d" % self.m[0])
        L.append("m2 = %d" % self.m[1])
        L.append("m3 = %d" % self.m[2])
        L.append("a = %.17g" % self.a)
        L.append("dL = %.17g" % self.dL)
        L.append("")
        L.append("[monomers]")
        L.append("M = %d" % self.M)
        L.append("names = [%s]" % ", ".join(self.monomer_names))
        L.append("")
        L.append("[polymer]")
        L.append("species_count = %d" % len(self.species))
        L.append("sequence_file = %s.seq" % self.name)
        for k, sp in enumerate(self.species):
            L.append("")
            L.append("[polymer.%d]" % k)
            L.append("name = %s" % sp.name)
            L.append("num_chains = %d" % sp.num_chains)
            L.append("N = %d" % sp.N)
        L.append("")
        L.append("[interactions]")
        chi = self.chi_matrix()
        rows = ["[" + ", ".join("%.17g" % v for v in row) + "]" for row in chi]
        L.append("chi = [" + ",\n       ".join(rows) + "]")
        L.append("xi = %.17g" % self.xi)
        L.append("lB = %.17g" % self.lB)
        L.append("eigen_tol_rel = %.17g" % self.eigen_tol_rel)
        L.append("")
        L.append("[dynamics]")
        L.append("dt = %.17g" % self.dt)
        L.append("lambda_omega = [%s]" % ", ".join("%.17g" % v for v in self.lambda_omega))
        L.append("lambdaPsi = %.17g" % self.lambda_psi)
        L.append("Nt = %d" % self.Nt)
        L.append("Nss = %d" % self.Nss)
        L.append("Ns = %d" % self.Ns)
        L.append("Ntmp = %d" % self.Ntmp)
        L.append("Nso = %d" % self.Nso)
        L.append("N_stat = %d" % self.N_stat)
        L.append("max_nan_restarts = %d" % self.max_nan_restarts)
        L.append("noise = %s" % ("true" if self.noise else "false"))
        L.append("")
        L.append("[ions]")
        L.append("enabled = %s" % ("true" if self.ions_enabled else "false"))
        if self.default_smearing_length is not None:
            L.append("default_smearing_length = %.17g" % self.default_smearing_length)
        if self.counterions is not None:
            c = self.counterions
            L.append("")
            L.append("[ions.counterions]")
            L.append("enabled = true")
            L.append("number = %s" % c.get("number", "auto_neutralize"))
            L.append("valence = %.17g" % c["valence"])
            L.append("name = %s" % c.get("name", "counterion"))
            if c.get("smearing_length") is not None:
                L.append("smearing_length = %.17g" % c["smearing_length"])
        if self.salt is not None:
            s = self.salt
            L.append("")
            L.append("[ions.salt]")
            L.append("enabled = true")
            L.append("num_salt = %d" % s["num_salt"])
            L.append("cation_name = %s" % s.get("cation_name", "salt_cation"))
            L.append("cation_valence = %.17g" % s["cation_valence"])
            L.append("cation_stoich = %d" % s.get("cation_stoich", 1))
            L.append("anion_name = %s" % s.get("anion_name", "salt_anion"))
            L.append("anion_valence = %.17g" % s["anion_valence"])
            L.append("anion_stoich = %d" % s.get("anion_stoich", 1))
            if s.get("smearing_length") is not None:
                L.append("smearing_length = %.17g" % s["smearing_length"])
            if "combine_identical_species" in s:
                L.append("combine_identical_species = %s" % ("true" if s["combine_identical_species"] else "false"))
        L.append("")
        L.append("[observables]")
        on = bool(self.stress) or self.isotropic_pressure
        L.append("stress = %s" % ("true" if on else "false"))
        for c in STRESS_COMPONENTS:
            L.append("component_%s = %s" % (c, "true" if c in self.stress else "false"))
        L.append("isotropic_pressure = %s" % ("true" if self.isotropic_pressure else "false"))
        L.append("")
        L.append("[output]")
        L.append("observable_file = %s" % self.observable_file)
        L.append("drift_max_file = %s" % self.drift_max_file)
        for k, v in self.extra_output.items():
            L.append("%s = %s" % (k, v))
        return "\n".join(L) + "\n"

    def sequence_text(self) -> str:
        out = []
        for k, sp in enumerate(self.species):
            out.append("[polymer.%d]" % k)
            out.append("monomers = " + " ".join(sp.monomers))
            out.append("charges = " + " ".join("%.17g" % q for q in sp.charges))
            if sp.bonds is not None:
                out.append("bonds = " + " ".join("%.17g" % b for b in sp.bonds))
            out.append("")
        return "\n".join(out)

    def initial_fields(self):
        """Seeded initial fields: Re ~ N(0, init_std^2), Im = 0.

        Returns (omega[n_modes, size], psi[size]) as complex128 arrays."""
        rng = np.random.default_rng(self.init_seed)
        nm = self.active_mode_count()
        omega = rng.normal(0.0, self.init_std, size=(nm, self.size)).astype(np.complex128)
        psi = rng.normal(0.0, self.init_std, size=self.size).astype(np.complex128)
        if self.lB <= 0.0:
            psi[:] = 0.0
        return omega, psi

    def write(self, directory: str, omega=None, psi=None) -> Dict[str, str]:
        os.makedirs(directory, exist_ok=True)
        paths = {
            "param": os.path.join(directory, self.name + ".param"),
            "sequence": os.path.join(directory, self.name + ".seq"),
            "omega": os.path.join(directory, self.name + "_omega.rf"),
            "psi": os.path.join(directory, self.name + "_psi.rf"),
        }
        with open(paths["param"], "w") as f:
            f.write(self.param_text())
        with open(paths["sequence"], "w") as f:
            f.write(self.sequence_text())
        if omega is None or psi is None:
            o, p = self.initial_fields()
            omega = o if omega is None else omega
            psi = p if psi is None else psi
        write_rf(paths["omega"], self.m, self.L, np.atleast_2d(omega))
        write_rf(paths["psi"], self.m, self.L, np.atleast_2d(psi))
        return paths


def write_rf(path: str, m, L, fields: np.ndarray, fmt: str = "%.17g") -> None:
    """Write field-major complex fields [nf, size] as an ``.rf`` table."""
    fields = np.atleast_2d(np.asarray(fields, dtype=np.complex128))
    nf, size = fields.shape
    cols = np.empty((size, 2 * nf), dtype=np.float64)
    cols[:, 0::2] = fields.real.T
    cols[:, 1::2] = fields.imag.T
    with open(path, "w") as f:
        f.write("%d %d %d\n" % tuple(int(v) for v in m))
        f.write("%.17g %.17g %.17g\n" % tuple(float(v) for v in L))
        np.savetxt(f, cols, fmt=fmt, delimiter="  ")


def read_rf(path: str):
    """Read an ``.rf`` table.  Returns (mesh or None, fields[nf, rows])."""
    mesh = None
    rows = []
    first = True
    maybe_box = False
    with open(path) as f:
        for line in f:
            line = line.split("#", 1)[0].strip()
            if not line:
                continue
            parts = line.split()
            if first:
                first = False
                if len(parts) == 3:
                    try:
                        vals = [int(p) for p in parts]
                        if all(v > 0 for v in vals):
                            mesh = tuple(vals)
                            maybe_box = True
                            continue
                    except ValueError:
                        pass
            if maybe_box:
                maybe_box = False
                if len(parts) == 3:
                    try:
                        vals = [float(p) for p in parts]
                        if all(v > 0 for v in vals):
                            continue
                    except ValueError:
                        pass
            rows.append([float(p) for p in parts])
    arr = np.asarray(rows, dtype=np.float64)
    if arr.size == 0:
        return mesh, np.zeros((0, 0), dtype=np.complex128)
    fields = (arr[:, 0::2] + 1j * arr[:, 1::2]).T.copy()
    return mesh, fields


def homopolymer(name: str, num_chains: int, N: int, charge: float = -1.0, monomer: str = "A") -> Species:
    return Species(name=name, num_chains=num_chains, monomers=[monomer] * N, charges=[charge] * N)


def polyelectrolyte_case(name: str, m: int, N: int, counter_valence: float, salt_conc: float,
                         dL: float = 0.5, bead_density: float = 0.5, **kw) -> Case:
    """Charged homopolymer solution with auto-neutralising counterions and 1:1 salt."""
    V = (m * dL) ** 3
    total_segments = bead_density * V
    chains = int(round(total_segments / N))
    num_salt = int(round(salt_conc * V))
    c = Case(name=name, m=(m, m, m), dL=dL, a=1.0, monomer_names=["A"], chi=[0.0], xi=0.1, lB=1.0,
             species=[homopolymer("P", chains, N)],
             counterions={"number": "auto_neutralize", "valence": counter_valence, "name": "counterion"},
             salt={"num_salt": num_salt, "cation_valence": 1.0, "anion_valence": -1.0,
                   "cation_name": "Na", "anion_name": "Cl"} if num_salt > 0 else None,
             **kw)
    return c


def workload(idx: int, **kw) -> Case:
    """The five named workloads (1-based).

    1: 32^3, L=16b, N=32, monovalent counterions, salt 0.1 b^-3, FP64, sigma_xx.
    2: 64^3, L=32b, N=50, same chemistry (complex64 propagators).
    3: replica batch member template (grid and N vary per replica).
    4: 128^3, L=64b, N=50, divalent counterions, salt 0.05 b^-3, full stress + Pi.
    5: workload 4 with the learned preconditioner (same physics).
    """
    if idx == 1:
        d = dict(dt=0.005, Nt=2000, Nss=10, stress=("xx",), isotropic_pressure=True)
        d.update(kw)
        return polyelectrolyte_case("w1_32cube_N32", 32, 32, 1.0, 0.1, **d)
    if idx == 2:
        d = dict(dt=0.005, Nt=5000, Nss=10, stress=STRESS_COMPONENTS, isotropic_pressure=True)
        d.update(kw)
        return polyelectrolyte_case("w2_64cube_N50", 64, 50, 1.0, 0.1, **d)
    if idx == 3:
        d = dict(dt=0.005, Nt=2000, Nss=10, stress=STRESS_COMPONENTS, isotropic_pressure=True)
        m = kw.pop("m", 32)
        N = kw.pop("N", 32)
        salt = kw.pop("salt", 0.1)
        d.update(kw)
        return polyelectrolyte_case("w3_replica_%d_N%d" % (m, N), m, N, 1.0, salt, **d)
    if idx in (4, 5):
        d = dict(dt=0.005 if idx == 4 else 0.02, Nt=10000, Nss=10, stress=STRESS_COMPONENTS,
                 isotropic_pressure=True)
        d.update(kw)
        return polyelectrolyte_case("w%d_128cube_N50" % idx, 128, 50, 2.0, 0.05, **d)
    raise ValueError("workload index must be 1..5")

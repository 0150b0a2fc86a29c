"""Shell data model, basis-set library and synthetic molecule generator.

The reference builds its basis through Libint (``libint2::BasisSet(name, atoms)``
followed by ``set_pure(false)``, quax/integrals/libint_interface.cc:47-73) and reads
the geometry from an xyz file in Angstrom (quax/integrals/utils.h:4-9).  This module
plays that role for the B200 path:

* ``Shell`` / ``Basis`` hold what the kernels need: angular momentum, primitive
  exponents, raw contraction coefficients, centre (bohr) and owning atom.
* Normalisation follows the Libint convention: each primitive is normalised for
  the axis-aligned Cartesian component x^l, then the contraction is rescaled so
  that x^l has unit self-overlap.  All Cartesian components of a shell share that
  one factor (so e.g. the d_xy component is not unit-normalised).
* Cartesian components are ordered like Libint's "standard" ordering:
  for lx = l..0, for ly = l-lx..0: (lx, ly, l-lx-ly)  ->  xx, xy, xz, yy, yz, zz.
* Basis sets: STO-3G for H, C, N, O from the published Hehre-Stewart-Pople
  tables (J. Chem. Phys. 51, 2657 (1969)); SP shells are split into an s and a p
  shell like Libint does.  Users can register further bases with
  ``register_basis``.
* ``synthetic_molecule`` draws the seeded synthetic workloads (random atoms,
  random shells) used by the throughput benchmarks and the large parity tests.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Sequence, Tuple

import numpy as np

# Bohr radius in Angstrom (CODATA 2018).  Libint's xyz reader converts Angstrom to
# bohr with its own CODATA constant; callers needing bit-identical geometry should
# pass bohr coordinates directly (``Molecule(..., units="bohr")``).
BOHR_TO_ANGSTROM = 0.529177210903

_SYMBOLS = ["X", "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne"]
SYMBOL_TO_Z = {s.upper(): z for z, s in enumerate(_SYMBOLS)}


def ncart(l: int) -> int:
    return (l + 1) * (l + 2) // 2


def nsph(l: int) -> int:
    return 2 * l + 1


def cart_components(l: int) -> List[Tuple[int, int, int]]:
    """Cartesian exponent triples of AM ``l`` in Libint standard order."""
    out = []
    for lx in range(l, -1, -1):
        for ly in range(l - lx, -1, -1):
            out.append((lx, ly, l - lx - ly))
    return out


def _dfact(n: int) -> float:
    """Double factorial n!! with (-1)!! = 0!! = 1."""
    r = 1.0
    while n > 1:
        r *= n
        n -= 2
    return r


def normalize_contraction(l: int, exps: Sequence[float], coefs: Sequence[float]) -> np.ndarray:
    """Return coefficients with primitive and contraction norms folded in.

    Primitive norm for x^l e^{-a r^2}:  N^2 = 2^l (2a)^{l+3/2} / (pi^{3/2} (2l-1)!!).
    Contraction: rescale so that <x^l|x^l> = 1 for the contracted function.
    """
    a = np.asarray(exps, dtype=np.float64)
    c = np.asarray(coefs, dtype=np.float64).copy()
    df = _dfact(2 * l - 1)
    c *= np.sqrt(2.0**l * (2.0 * a) ** (l + 1.5) / (math.pi**1.5 * df))
    g = a[:, None] + a[None, :]
    s = np.sum(c[:, None] * c[None, :] * df * math.pi**1.5 / (2.0**l * g ** (l + 1.5)))
    return c / math.sqrt(s)


@dataclass
class Shell:
    l: int
    exps: np.ndarray
    coefs: np.ndarray  # raw contraction coefficients, as tabulated
    center: np.ndarray  # bohr, shape (3,)
    atom: int

    @property
    def nprim(self) -> int:
        return len(self.exps)

    def size(self, pure: bool = False) -> int:
        return nsph(self.l) if pure else ncart(self.l)

    def norm_coefs(self) -> np.ndarray:
        return normalize_contraction(self.l, self.exps, self.coefs)


@dataclass
class Molecule:
    Z: np.ndarray  # (natom,) int
    coords: np.ndarray  # (natom, 3) bohr
    charge: int = 0

    @property
    def natom(self) -> int:
        return len(self.Z)

    @property
    def nelectron(self) -> int:
        return int(np.sum(self.Z)) - self.charge

    @staticmethod
    def from_xyz(path: str, units: str = "angstrom") -> "Molecule":
        """Read an xyz file (count line, comment line, then symbol x y z)."""
        with open(path) as f:
            lines = [ln for ln in f.read().splitlines()]
        nat = int(lines[0].split()[0])
        Z, xyz = [], []
        for ln in lines[2 : 2 + nat]:
            tok = ln.split()
            Z.append(SYMBOL_TO_Z[tok[0].upper()])
            xyz.append([float(t) for t in tok[1:4]])
        xyz = np.asarray(xyz, dtype=np.float64)
        if units.lower().startswith("ang"):
            xyz = xyz / BOHR_TO_ANGSTROM
        return Molecule(np.asarray(Z, dtype=np.int64), xyz)

    def to_xyz(self, path: str) -> None:
        """Write an xyz file in Angstrom, as the reference writes geom.xyz."""
        with open(path, "w") as f:
            f.write(f"{self.natom}\n\n")
            for z, r in zip(self.Z, self.coords * BOHR_TO_ANGSTROM):
                f.write(f"{_SYMBOLS[int(z)]} {r[0]:.16f} {r[1]:.16f} {r[2]:.16f}\n")


@dataclass
class Basis:
    shells: List[Shell]
    natom: int
    pure: bool = False
    name: str = "custom"

    @property
    def nshell(self) -> int:
        return len(self.shells)

    def nbf(self) -> int:
        return int(sum(s.size(self.pure) for s in self.shells))

    def shell2bf(self) -> np.ndarray:
        sizes = [s.size(self.pure) for s in self.shells]
        return np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)

    def shell2atom(self) -> np.ndarray:
        return np.asarray([s.atom for s in self.shells], dtype=np.int64)

    def max_l(self) -> int:
        return max(s.l for s in self.shells)

    def max_nprim(self) -> int:
        return max(s.nprim for s in self.shells)

    def atom_coords(self) -> np.ndarray:
        xyz = np.zeros((self.natom, 3))
        for s in self.shells:
            xyz[s.atom] = s.center
        return xyz

    def with_coords(self, coords: np.ndarray) -> "Basis":
        """Same shells, moved to new atom coordinates (natom, 3) in bohr."""
        coords = np.asarray(coords, dtype=np.float64).reshape(self.natom, 3)
        sh = [Shell(s.l, s.exps, s.coefs, coords[s.atom].copy(), s.atom) for s in self.shells]
        return Basis(sh, self.natom, self.pure, self.name)

    def flat(self) -> Dict[str, np.ndarray]:
        """Flat arrays in the layout the C ABI takes (raw coefficients)."""
        l = np.asarray([s.l for s in self.shells], dtype=np.int32)
        nprim = np.asarray([s.nprim for s in self.shells], dtype=np.int32)
        atom = np.asarray([s.atom for s in self.shells], dtype=np.int32)
        off = np.concatenate([[0], np.cumsum(nprim)[:-1]]).astype(np.int32)
        centers = np.ascontiguousarray(np.stack([s.center for s in self.shells]).astype(np.float64))
        exps = np.ascontiguousarray(np.concatenate([s.exps for s in self.shells]).astype(np.float64))
        coefs = np.ascontiguousarray(np.concatenate([s.coefs for s in self.shells]).astype(np.float64))
        return dict(l=l, nprim=nprim, atom=atom, prim_off=off, centers=centers, exps=exps, coefs=coefs)


# --------------------------------------------------------------------------------------
# Basis-set library.  Each entry: Z -> list of (l, exponents, coefficients).
# STO-3G: Hehre, Stewart & Pople, J. Chem. Phys. 51, 2657 (1969).
# --------------------------------------------------------------------------------------
_STO3G_1S = [0.15432897, 0.53532814, 0.44463454]
_STO3G_2S = [-0.09996723, 0.39951283, 0.70011547]
_STO3G_2P = [0.15591627, 0.60768372, 0.39195739]


def _sto3g_heavy(e1s, e2sp):
    return [(0, e1s, _STO3G_1S), (0, e2sp, _STO3G_2S), (1, e2sp, _STO3G_2P)]


_BASIS_LIBRARY: Dict[str, Dict[int, list]] = {
    "sto-3g": {
        1: [(0, [3.42525091, 0.62391373, 0.16885540], _STO3G_1S)],
        6: _sto3g_heavy([71.6168370, 13.0450960, 3.5305122], [2.9412494, 0.6834831, 0.2222899]),
        7: _sto3g_heavy([99.1061690, 18.0523120, 4.8856602], [3.7804559, 0.8784966, 0.2857144]),
        8: _sto3g_heavy([130.7093200, 23.8088610, 6.4436083], [5.0331513, 1.1695961, 0.3803890]),
    }
}


def register_basis(name: str, table: Dict[int, list]) -> None:
    """Register a basis: ``{Z: [(l, exps, coefs), ...]}``."""
    _BASIS_LIBRARY[name.lower()] = table


def available_bases() -> List[str]:
    return sorted(_BASIS_LIBRARY)


def build_basis(mol: Molecule, name: str, pure: bool = False) -> Basis:
    """Shells of basis ``name`` placed on every atom of ``mol`` (atom order)."""
    table = _BASIS_LIBRARY.get(name.lower())
    if table is None:
        raise ValueError(f"basis '{name}' is not in the library ({available_bases()})")
    shells = []
    for a in range(mol.natom):
        z = int(mol.Z[a])
        if z not in table:
            raise ValueError(f"basis '{name}' has no entry for Z={z}")
        for l, e, c in table[z]:
            shells.append(Shell(l, np.asarray(e, float), np.asarray(c, float), mol.coords[a].copy(), a))
    return Basis(shells, mol.natom, pure, name.lower())


# --------------------------------------------------------------------------------------
# Synthetic workloads
# --------------------------------------------------------------------------------------
@dataclass
class SyntheticSpec:
    natom: int = 10
    box: float = 12.0
    min_sep: float = 1.8
    charges: Tuple[int, ...] = (1, 6, 8)
    heavy_ls: Tuple[int, ...] = (0, 0, 0, 1, 1, 2)
    h_ls: Tuple[int, ...] = (0, 0, 1)
    kmin: int = 1
    kmax: int = 8
    exp_lo: float = 0.08
    exp_hi: float = 5.0e3
    f_shell: bool = False
    f_kmax: int = 3
    f_exp_lo: float = 0.2
    f_exp_hi: float = 5.0
    pure: bool = False


def synthetic_molecule(spec: SyntheticSpec, seed: int = 0) -> Tuple[Molecule, Basis]:
    """Seeded synthetic molecule and basis.

    Atoms: rejection-sampled uniform in [0, box]^3 bohr with a minimum separation;
    Z uniform over ``charges``.  Heavy atoms carry ``heavy_ls`` shells, H carries
    ``h_ls``; K ~ U{kmin..kmax}; exponents log-uniform in [exp_lo, exp_hi], sorted
    descending; coefficients U[0.1, 1] (normalised later, Libint convention).
    Optional f shell on heavy atoms with K ~ U{1..f_kmax}, exponents log-uniform
    in [f_exp_lo, f_exp_hi].  Closed shell: charge = sum(Z) mod 2.
    """
    rng = np.random.default_rng(seed)
    coords: List[np.ndarray] = []
    tries = 0
    while len(coords) < spec.natom:
        p = rng.uniform(0.0, spec.box, size=3)
        if all(np.linalg.norm(p - q) >= spec.min_sep for q in coords):
            coords.append(p)
        tries += 1
        if tries > 1_000_000:
            raise RuntimeError("could not place atoms with the requested separation")
    Z = rng.choice(np.asarray(spec.charges), size=spec.natom)
    xyz = np.stack(coords)
    shells = []
    for a in range(spec.natom):
        ls = list(spec.h_ls if Z[a] == 1 else spec.heavy_ls)
        if spec.f_shell and Z[a] != 1:
            ls.append(3)
        for l in ls:
            if l == 3 and spec.f_shell:
                k = int(rng.integers(1, spec.f_kmax + 1))
                e = np.exp(rng.uniform(math.log(spec.f_exp_lo), math.log(spec.f_exp_hi), size=k))
            else:
                k = int(rng.integers(spec.kmin, spec.kmax + 1))
                e = np.exp(rng.uniform(math.log(spec.exp_lo), math.log(spec.exp_hi), size=k))
            e = np.sort(e)[::-1].copy()
            c = rng.uniform(0.1, 1.0, size=k)
            shells.append(Shell(l, e, c, xyz[a].copy(), a))
    charge = int(np.sum(Z)) % 2
    return Molecule(Z.astype(np.int64), xyz, charge), Basis(shells, spec.natom, spec.pure, "synthetic")


def config_spec(name: str) -> SyntheticSpec:
    """Named synthetic workloads (sizes as the benchmark configurations state)."""
    if name == "eri10":  # 10 atoms, l<=2
        return SyntheticSpec(natom=10)
    if name == "grad30":  # 30 atoms, l<=2
        return SyntheticSpec(natom=30)
    if name == "mixed60":  # 60 atoms, with f shells
        return SyntheticSpec(natom=60, f_shell=True)
    raise KeyError(name)


def h2o_config1() -> Molecule:
    """H2O with O(0,0,0), H(0,0,1), H(0,1,0) bohr (the small CPU-runnable case)."""
    return Molecule(np.asarray([8, 1, 1]), np.asarray([[0.0, 0.0, 0.0], [0.0, 0.0, 1.0], [0.0, 1.0, 0.0]]))

"""
Generate the golden fixtures in this directory by running the REFERENCE
implementation (Nathan-W123/Ab-Initio-MD, numba CPU code) on the benchmark
geometries. The reference is importable only where its source tree is
available, so the fixtures are committed and the tests read them.

    NUMBA_CACHE_DIR=<writable dir> python tests/golden/make_golden.py <reference source tree> [--only=case1,case2]

Fixtures (all arrays float64, Hartree atomic units):
  boys.npz            F_0..F_32 at 60 arguments (aimd/qc/boys.py:143)
  basis_arrays.npz    the reference BasisSet's flat shell / primitive /
                      block arrays for several molecules and basis sets
                      (the host layout must match them bitwise)
  <case>.npz          positions, Schwarz bounds, a sample of ERIs, J/K of
                      random densities, one-electron matrices, two- and
                      one-electron gradient contractions at fixed
                      densities, SCF energy / gradient / density / dipole,
                      and the FP64 flop model of one ERI pass.
"""

from __future__ import annotations

import os
import sys
import zlib

import numpy as np

ANG = 1.8897261254578281          # bohr per angstrom

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _flop_model(basis, Q, pr, threshold):
    """Flop model of one ERI pass from the reference's own pair data (see oracle.flop_model)."""
    i, j = pr.pair_blocks.T
    l = basis.blk_l
    Lp = l[i] + l[j]
    nc = (l + 1) * (l + 2) // 2
    nab = nc[i] * nc[j]
    ncon = basis.blk_ncon[i] * basis.blk_ncon[j]
    npp = np.diff(pr.pair_pp).astype(float)

    def NH(L):
        return (L + 1) * (L + 2) * (L + 3) // 6

    rs = np.array([sum(NH(L0 - n) for n in range(L0 + 1)) for L0 in range(9)])
    total = nq = 0.0
    for p1 in range(len(Q)):
        p2 = np.arange(p1 + 1)
        p2 = p2[Q[p1] * Q[p2] >= threshold]
        if p2.size == 0:
            continue
        Lb, Lk = Lp[p1], Lp[p2]
        per = 2 * rs[Lb + Lk] + 2 * NH(Lb) * NH(Lk) * nab[p2] * ncon[p2] + 2 * NH(Lb) * nab[p1] * nab[p2] * ncon[p2]
        w = npp[p1] * npp[p2]
        total += float(np.sum(per * w))
        nq += float(np.sum(w))
    return total, nq


def main() -> None:
    args = [a for a in sys.argv[1:] if not a.startswith("--only=")]
    only = [a.split("=", 1)[1].split(",") for a in sys.argv[1:] if a.startswith("--only=")]
    only = set(only[0]) if only else None
    if not args:
        sys.exit("usage: make_golden.py <reference source tree> [--only=case1,case2]")
    ref = args[0]
    sys.path.insert(0, ref)
    sys.path.insert(0, os.path.join(REPO, "ab-initio-md_b200"))
    from aimd.qc import integrals as I
    from aimd.qc.basis import build_basis
    from aimd.qc.boys import boys
    from aimd.qc.gradients import energy_weighted_density, scf_gradient
    from aimd.qc.scf import run_scf
    from aimd_b200 import geometry as G

    rng = np.random.default_rng(2024)
    xs = np.concatenate([10 ** rng.uniform(-8, np.log10(150.0), 50),
                         [0.0, 0.05, 1.0, 39.999999, 40.0, 40.000001, 100.0, 1e3, 1e6, 1e12]])
    if only is None:
        F = np.array([boys(32, float(x)) for x in xs])
        np.savez_compressed(os.path.join(HERE, "boys.npz"), x=xs, F=F)
    if only is None or "basis_arrays" in only:
        _basis_arrays(build_basis, G)

    cases = {
        "water_631gs": (*G.water(), "6-31g*", 0, 1, {}),
        "water_ccpvdz": (*G.water(), "cc-pvdz", 0, 1, {}),
        "methanol_631gss": (*G.methanol(), "6-31g**", 0, 1, {}),
        "ch3_uhf_631gs": (["C", "H", "H", "H"], np.array(
            [[0.0, 0.0, 0.0], [2.0598, 0.0, 0.0], [-1.0299, 1.7839, 0.0], [-1.0299, -1.7839, 0.3]]),
            "6-31g*", 0, 2, {}),
        "h2o8_ccpvdz": (*G.water_cluster(8, seed=0), "cc-pvdz", 0, 1, {"max_nao": 200}),
        # second-row atoms: more primitives and general contractions of 3 s /
        # 2 p columns per block in cc-pVDZ (split into smaller blocks on the device)
        "h2s_631gs": (["S", "H", "H"], _bent(1.336, 92.1), "6-31g*", 0, 1, {}),
        "hcl_ccpvdz": (["Cl", "H"], np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 1.2746 * ANG]]), "cc-pvdz", 0, 1, {}),
    }
    own_rng = {"h2s_631gs", "hcl_ccpvdz"}     # cases added later draw from their own generator
    for name, (sym, pos, basis, charge, mult, opts) in cases.items():
        if only is not None and name not in only:
            continue
        if name in own_rng:
            rng = np.random.default_rng(zlib.crc32(name.encode()))
        print(name, flush=True)
        b = build_basis(sym, pos, basis)
        pr = I._pairs(b)
        Q = I.schwarz_bounds(b)
        n = b.nao
        out = {"symbols": np.array(sym), "positions": pos, "basis": np.array(basis),
               "charge": charge, "multiplicity": mult, "Q": Q}
        flop, nq = _flop_model(b, Q, pr, I.DEFAULT_SCHWARZ)
        out["flop_model"] = flop
        out["prim_quartets"] = nq
        Dr = rng.normal(size=(n, n))
        Dsym = Dr + Dr.T
        Wr = rng.normal(size=(n, n))
        Wsym = Wr + Wr.T
        if n <= 60:
            out["D_rand"] = Dsym
            out["W_rand"] = Wsym
            eri = I.eri_tensor(b)
            idx = rng.integers(0, n, size=(4000, 4))
            out["eri_idx"] = idx
            out["eri_val"] = eri[idx[:, 0], idx[:, 1], idx[:, 2], idx[:, 3]]
            D2 = rng.normal(size=(2, n, n))
            out["D_nonsym"] = D2
            J, K = I.jk_from_eri(eri, D2)
            out["J_nonsym"], out["K_nonsym"] = J, K
            J, K = I.jk_from_eri(eri, Dsym)
            out["J_sym"], out["K_sym"] = J, K
            S, T, M = I._overlap_type(b, np.array([0.3, -0.2, 0.5]))
            out["S"], out["T"], out["M"] = S, T, M
            out["V"] = I.nuclear_attraction_matrix(b)
            out["g2e_rhf"] = I.two_electron_gradient(b, Dsym, [Dsym], 0.5)
            out["g2e_uhf"] = I.two_electron_gradient(b, Dsym, [Dsym, Wsym], 1.0)
            out["g1e"] = I.one_electron_gradient(b, Dsym, Wsym)
        res = run_scf(sym, pos, basis, charge=charge, multiplicity=mult, **opts)
        g = scf_gradient(res)
        out["energy"] = res.energy
        out["iterations"] = res.iterations
        out["gradient"] = g
        out["density"] = res.density
        if res.unrestricted:
            out["spin_densities"] = res.spin_densities
        out["dipole"] = res.dipole
        out["s2"] = res.s2
        if n <= 60:
            out["W"] = energy_weighted_density(res.spin_densities, res.fock)
        print(f"  nao {n} E {res.energy:.12f} it {res.iterations} flop {flop:.3e}", flush=True)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)


BASIS_ARRAYS = ("shell_atom", "shell_l", "shell_prim", "shell_ao", "prim_exp", "prim_coef", "blk_shell", "blk_atom",
                "blk_l", "blk_ncon", "blk_ao", "blk_prim", "blk_exp", "blk_coef", "ao_lxyz", "atom_ao")


def _basis_arrays(build_basis, G) -> None:
    """The reference BasisSet arrays of several molecules, keyed '<case>/<array>'."""
    mols = {
        "water_sto3g": (*G.water(), "sto-3g"),
        "water_631gs": (*G.water(), "6-31g*"),
        "methanol_631gss": (*G.methanol(), "6-31g**"),
        "water2_ccpvdz": (*G.water_cluster(2, seed=4), "cc-pvdz"),
        "h2s_631gs": (["S", "H", "H"], _bent(1.336, 92.1), "6-31g*"),
        "hcl_ccpvdz": (["Cl", "H"], np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 1.2746 * ANG]]), "cc-pvdz"),
        "ch3no_631g": (["C", "H", "H", "H", "N", "O"], np.arange(18, dtype=float).reshape(6, 3) * 0.7, "6-31g"),
    }
    out = {}
    for name, (sym, pos, basis) in mols.items():
        b = build_basis(sym, pos, basis)
        out[f"{name}/symbols"] = np.array(sym)
        out[f"{name}/positions"] = np.asarray(pos, dtype=float)
        out[f"{name}/basis"] = np.array(basis)
        for a in BASIS_ARRAYS:
            out[f"{name}/{a}"] = np.asarray(getattr(b, a))
    np.savez_compressed(os.path.join(HERE, "basis_arrays.npz"), **out)


def _bent(r_ang: float, angle_deg: float) -> np.ndarray:
    """X-H2 at r (A) and H-X-H angle (deg), X at the origin, bohr."""
    t = np.radians(angle_deg) / 2
    r = r_ang * ANG
    return np.array([[0.0, 0.0, 0.0], [r * np.sin(t), 0.0, r * np.cos(t)], [-r * np.sin(t), 0.0, r * np.cos(t)]])


if __name__ == "__main__":
    main()

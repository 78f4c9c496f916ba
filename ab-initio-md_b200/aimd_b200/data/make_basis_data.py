"""
Regenerate ``basis_sets.json`` (Gaussian basis-set data for H-Ar) from the
reference project's basis library, so that both codes use bitwise the same
exponents and contraction coefficients.

The numbers are published basis-set data (STO-3G, 6-31G, 6-31G*, 6-31G**,
cc-pVDZ; EMSL / Basis Set Exchange, identical to PySCF's copies). The
reference keeps them in ``aimd/qc/basis_data.py`` (``BASIS_SETS``,
``aimd/qc/basis_data.py:1032``) in the PySCF/NWChem row layout
``[l, [exp, c_1, c_2, ...], ...]``; this script writes the same rows as JSON.

Run once, in a checkout that has the reference importable:

    python make_basis_data.py <reference source tree>
"""

from __future__ import annotations

import json
import os
import sys


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit("usage: make_basis_data.py <reference source tree>")
    sys.path.insert(0, sys.argv[1])
    from aimd.qc.basis_data import BASIS_SETS  # noqa: E402  (reference module)

    out = {}
    for name, data in BASIS_SETS.items():
        out[name] = {el: [[int(sh[0])] + [list(map(float, row)) for row in sh[1:]] for sh in shells]
                     for el, shells in data.items()}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "basis_sets.json")
    with open(path, "w") as f:
        json.dump(out, f, separators=(",", ":"))
        f.write("\n")
    print(f"wrote {path}: {', '.join(out)}")


if __name__ == "__main__":
    main()

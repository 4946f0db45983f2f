"""Generate the oracle reference values of the config-1 SCF (Si2 fcc
primitive, a = 10.26 bohr, ecutwfc 20 Ry, shifted 4x4x4 MP grid reduced by
symmetry to 10 k-points, 8 bands, Fixed occupations at the deck's default
width 0.05 eV, plain Anderson beta 0.7 ndim 8, energy threshold 1e-10 Ry,
density-rms threshold 1e-8 e/Å³) with Si_hgh.upf and Si.upf.

    python tests/golden/make_oracle_fixtures.py     (CPU, about 2 minutes)

Writes tests/golden/config1_oracle.json.
"""

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "pwdft-rs_b200"))
sys.path.insert(0, ROOT)

from oracle import pwdft_oracle as O  # noqa: E402
from pwgpu.config1 import SCF_KW, config1_system  # noqa: E402
from pwgpu.upf import load_upf  # noqa: E402


def main():
    out = {}
    for name in ("Si_hgh", "Si"):
        pp = load_upf(os.path.join(HERE, "upf", name + ".upf"))
        s = config1_system(pp)
        kw = dict(SCF_KW)
        r = O.run_scf_unpolarized(s, kw.pop("n_bands"), smearing=kw.pop("smearing"), sigma=kw.pop("sigma"), **kw)
        out[name] = {"total_energy": r.total_energy, "harris_foulkes_energy": r.harris_foulkes_energy,
                     "fermi_energy": r.fermi_energy, "n_iterations": r.n_iterations,
                     "eigenvalues": [list(map(float, e)) for e in r.eigenvalues], "n_pw": s.n_pw,
                     "dims": list(s.dims), "n_k": len(s.kpoints)}
        print(name, r.n_iterations, r.total_energy)
    with open(os.path.join(HERE, "config1_oracle.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()

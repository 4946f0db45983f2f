"""Generate the oracle reference values of the mixed-precision SCF case on
the 8-atom cell: Si cubic conventional cell (a = 10.26 bohr) with seeded
±0.05 bohr displacements, Si.upf, ecutwfc 30 Ry (n_pw 2,945 on 36^3), Γ
only, 20 bands, Gaussian 0.01 Ry, Anderson beta 0.4 + Kerker, converged to
a density rms of 1e-9 e/Å³ and an energy change of 1e-9 eV.

    python tests/golden/make_config3_fixtures.py     (CPU, a few minutes)

Writes tests/golden/config3_si8_oracle.json.
"""

import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "pwdft-rs_b200"))
sys.path.insert(0, ROOT)

from oracle import pwdft_oracle as O  # noqa: E402
from pwgpu.config3 import SI8_SCF_KW, config3_si8_system  # noqa: E402
from pwgpu.upf import load_upf  # noqa: E402


def main():
    t0 = time.time()
    s = config3_si8_system(load_upf(os.path.join(HERE, "upf", "Si.upf")))
    kw = dict(SI8_SCF_KW)
    nb = kw.pop("n_bands")
    r = O.run_scf_unpolarized(s, nb, smearing=kw.pop("smearing"), sigma=kw.pop("sigma"), verbose=True, **kw)
    out = {"total_energy": r.total_energy, "harris_foulkes_energy": r.harris_foulkes_energy,
           "fermi_energy": r.fermi_energy, "entropy_ts": r.entropy_ts, "n_iterations": r.n_iterations,
           "final_delta": r.final_delta, "eigenvalues": [list(map(float, e)) for e in r.eigenvalues],
           "components": {k: float(v) for k, v in r.components.items()},
           "n_pw": s.n_pw, "dims": list(s.dims), "n_atoms": len(s.crystal.atoms),
           "thresholds": {k: SI8_SCF_KW[k] for k in ("conv_threshold", "energy_threshold")}}
    with open(os.path.join(HERE, "config3_si8_oracle.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(r.n_iterations, r.total_energy, f"{time.time() - t0:.0f} s", flush=True)


if __name__ == "__main__":
    main()

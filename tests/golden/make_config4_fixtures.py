"""Generate the oracle reference values of the batched-k LSDA case (the
8-atom cubic Si and C diamond cells at 35 Ry, Gamma-centred 6x6x6 mesh
reduced to 20 IBZ k-points, 24 bands, Fermi-Dirac 0.02 Ry, starting
magnetisation 0 on Si and 0.125 on C), converged far below the case's
own thresholds: density rms 1e-9 e/Å^3 and energy change 1e-9 eV, so that
the plain FP64 form can be held to 1e-8 Ha.  Near convergence the
plain-Anderson magnetisation channel of the C cells contracts by ~7 % per
iteration, hence the long tail of iterations.

    python tests/golden/make_config4_fixtures.py [C C_nonlcc Si]

(CPU; each C cell takes about twenty minutes, the Si cell about an hour).
Writes tests/golden/config4_<cell>_oracle.json per cell.
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
from pwgpu.config4 import SCF_KW, config4_system  # noqa: E402
from pwgpu.upf import load_upf  # noqa: E402

TIGHT = dict(max_iter=400, conv_threshold=1e-9, energy_threshold=1e-9)
CASES = {"C": ("C", "C.upf", True), "C_nonlcc": ("C", "C.upf", False), "Si": ("Si", "Si.upf", True)}


def main(names):
    for name in names:
        species, upf, nlcc = CASES[name]
        t0 = time.time()
        s, m = config4_system(species, load_upf(os.path.join(HERE, "upf", upf)), nlcc=nlcc)
        kw = dict(SCF_KW)
        kw.update(TIGHT)
        nb = kw.pop("n_bands")
        r = O.run_scf_spin(s, nb, starting_magnetization=m, smearing=kw.pop("smearing"), sigma=kw.pop("sigma"),
                           verbose=True, **kw)
        out = {"total_energy": r.total_energy, "harris_foulkes_energy": r.harris_foulkes_energy,
               "fermi_energy": r.fermi_energy, "magnetization": r.magnetization, "n_iterations": r.n_iterations,
               "final_delta": r.final_delta, "eigenvalues": [list(map(float, e)) for e in r.eigenvalues],
               "n_pw": s.n_pw, "dims": list(s.dims), "n_k": len(s.kpoints), "starting_magnetization": m,
               "nlcc": nlcc, "thresholds": TIGHT}
        with open(os.path.join(HERE, f"config4_{name}_oracle.json"), "w") as f:
            json.dump(out, f, indent=1)
        print(name, r.n_iterations, r.total_energy, r.magnetization, f"{time.time() - t0:.0f} s", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or list(CASES))

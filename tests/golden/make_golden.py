"""Generate the golden fixtures in tests/golden/ by running the reference's own CPU solvers.

    python tests/golden/make_golden.py

The reference ships no golden vectors, known-answer tests or result files (its only data are the
homogeneous InputFile/SrcRcv examples), so these fixtures are its outputs on seeded inputs:
oracle/_ref/twref_elastic_{f64,f32} (cuda/src/cpp host solver) and
oracle/_ref/twref_acoustic_{f64,f32} (singlecore solver), built from the reference's sources
(oracle.refrun.REFERENCE_DIR, environment variable TW_REFERENCE_DIR) by `make -C oracle ref`. Each .npz holds the case inputs and, per precision, the final fields, the
receiver traces, the three energy records, the stored coefficients and the energy weights.
The "_if_" fixtures select the reference's SAT interface branch for both x ends (a boundary type
other than 'F', grid_drvt.tpp:575-693), which the reference's own inputs never reach.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from cases import acoustic_periodic_case, elastic_case  # noqa: E402
from oracle import refrun  # noqa: E402

ELASTIC = [  # name, Mx, My, seed, cpst, Nt, acoustic (vs = 0), x boundary type
    ("el_24x20_00", 24, 20, 1, "00", 60, False, "F"),
    ("el_20x16_6R", 20, 16, 2, "6R", 60, False, "F"),
    ("el_16x12_3C", 16, 12, 3, "3C", 60, False, "F"),
    ("el_17x9_6C", 17, 9, 4, "6C", 50, False, "F"),
    ("el_12x10_m3R", 12, 10, 5, "-3R", 50, False, "F"),
    ("el_20x16_vs0", 20, 16, 6, "00", 60, True, "F"),
    # the x ends joined by the SAT interface penalty (secure_bdry with a boundary type other than 'F')
    ("el_24x20_if_00", 24, 20, 21, "00", 80, False, "I"),
    ("el_18x14_if_6R", 18, 14, 22, "6R", 70, False, "I"),
    ("el_20x16_if_vs0", 20, 16, 23, "00", 70, True, "I"),
]
ACOUSTIC = [  # name, Nx, Ny, seed, cpst, Nt
    ("ac_16x16_0", 16, 16, 7, "0", 60),
    ("ac_20x24_6", 20, 24, 8, "6", 60),
    ("ac_18x12_3", 18, 12, 9, "3", 50),
]


def main():
    manifest = {}
    for name, Mx, My, seed, cpst, Nt, ac, bc_x in ELASTIC:
        case = elastic_case(Mx, My, seed=seed, cpst=cpst, Nt=Nt, acoustic=ac)
        case.bc_x = bc_x
        out = {"Mx": Mx, "My": My, "num_dx": case.num_dx, "den_dx": case.den_dx, "dt": case.dt,
               "central_f": case.central_f, "time_delay": case.time_delay, "cpst": cpst, "Nt": Nt, "bc_x": bc_x,
               "rho": case.rho, "vp": case.vp, "vs": case.vs, "src": json.dumps(case.src), "rcvs": json.dumps(case.rcvs)}
        for prec in ("f64", "f32"):
            r = refrun.run_elastic(case, prec)
            for k, v in r.fields.items():
                out[f"{prec}_field_{k}"] = v
            for k, v in r.coefs.items():
                out[f"{prec}_coef_{k}"] = v
            for k, v in r.weights.items():
                out[f"{prec}_weight_{k}"] = v
            out[f"{prec}_traces"] = r.traces
            out[f"{prec}_E_k"], out[f"{prec}_E_p0"], out[f"{prec}_E_p1"] = r.E_k, r.E_p0, r.E_p1
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        manifest[name] = {"kind": "elastic", "Mx": Mx, "My": My, "cpst": cpst, "Nt": Nt, "vs0": ac, "bc_x": bc_x}
    for name, Nx, Ny, seed, cpst, Nt in ACOUSTIC:
        case = acoustic_periodic_case(Nx, Ny, seed=seed, cpst=cpst, Nt=Nt)
        out = {"Nx": Nx, "Ny": Ny, "dx": case.dx, "dt": case.dt, "central_f": case.central_f,
               "time_delay": case.time_delay, "cpst": cpst, "Nt": Nt, "rho_vx": case.rho_vx, "rho_vy": case.rho_vy,
               "coef_p": case.coef_p, "src": np.array(case.src), "rcvs": np.array(case.rcvs)}
        for prec in ("f64", "f32"):
            r = refrun.run_acoustic(case, prec)
            for k, v in r.fields.items():
                out[f"{prec}_field_{k}"] = v
            out[f"{prec}_traces"] = r.traces
            out[f"{prec}_energy"] = r.energy
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        manifest[name] = {"kind": "acoustic_periodic", "Nx": Nx, "Ny": Ny, "cpst": cpst, "Nt": Nt}
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)
    print(f"wrote {len(manifest)} fixtures")


if __name__ == "__main__":
    main()

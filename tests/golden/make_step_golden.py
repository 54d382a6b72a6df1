"""Golden fixture of two CP steps of the 192-atom benchmark system from the FP64
oracle (oracle/step.py), for tests/test_configs_gpu.py.

System: 64 O + 128 H at seeded positions (>= 1.8 bohr apart) in a cubic box
of 23.5 bohr, 128 states, Ecut 70 Ry, grid 128^3, EES non-local (s + p,
B-spline order 8), coefficients Gaussian x exp(-|G|^2/8) Loewdin-normalised
(openatom_b200.system.System, seed 1234, built on the CPU), CP masses
(25 fs, 70 Ry), dt = 5 au, the orthoT constraint with cp_norb_tol 1.0.

Stored per step: the energies, the atom forces, max |S - 2I| of the norb
check, and psi and v at 4096 seeded (state, point) pairs.  The oracle's
pieces are pinned to the reference compiled from source (tests/*_oracle.py);
one step takes about half a minute on 8 cores.

Usage: python tests/golden/make_step_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import density as OD  # noqa: E402
from oracle import fftpath as OF  # noqa: E402
from oracle import layout as OL  # noqa: E402
from oracle import step as OS  # noqa: E402

BOX, ECUT, NST, GRID, DT = 23.5, 70.0, 128, 128, 5.0
ATOMS = {"O": 64, "H": 128}
NSAMPLE = 4096
OUT = os.path.join(HERE, "step_water192.npz")
SLOTS = ("EXC", "MUXC", "EHART", "EEXT", "EWD", "EKE", "ENL", "ETOT", "FICT")


def sample_index(nstates, npts, n=NSAMPLE, seed=99):
    rng = np.random.default_rng(seed)
    return rng.integers(0, nstates, n), rng.integers(0, npts, n)


def main():
    from openatom_b200.system import System
    OF.set_workers(os.cpu_count() or 1)
    sysm = System(BOX, ECUT, NST, ATOMS, nfft=GRID)
    lay = OL.Layout(BOX, ECUT, grid=GRID)
    dlay = OD.density_layout(BOX, ECUT, GRID)
    psi = sysm.psi(device="cpu").numpy()
    cmass = OS.cp_mass(lay, 25.0, ECUT)
    si, pi = sample_index(NST, lay.npts)
    out = dict(sample_state=si, sample_point=pi)
    p, v, dyn = psi, np.zeros_like(psi), None
    for it in (1, 2):
        p, v, en, f, aux = OS.cp_step(p, v, np.ones(NST), sysm, lay, dlay, cmass, DT, it,
                                      nonlocal_on=True, tol_norb=1.0, dyn=dyn)
        dyn = aux["dyn"]
        out["energies_%d" % it] = np.array([en[k] for k in SLOTS])
        out["atom_force_%d" % it] = f
        out["norb_dev_%d" % it] = np.array(dyn["dev"])
        out["psi_%d" % it] = p[si, pi]
        out["v_%d" % it] = v[si, pi]
        print("step", it, "E_tot %.12f" % en["ETOT"], flush=True)
    np.savez_compressed(OUT, slots=np.array(SLOTS), **out)
    print(OUT)


if __name__ == "__main__":
    main()

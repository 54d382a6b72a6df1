"""The oracle's CP dynamics constraint (reference form: gamma = orthoT lambda,
F_c = F.orthoT - W psi.gamma on the non-orthogonal coefficients, the norb
check and the PsiV reset) on the CPU.

* At orthoT = I the constraint is the projection of the minimisation form.
* Both forms keep psi orthonormal (S = 2 I) and conserve E_tot + E_fict to
  second order in dt: the drift over a fixed time falls 4x when dt halves.
  A wrong Gx=0 weight W breaks this; a rotation inside the occupied space
  (gamma against its transpose) leaves the energy invariant and cannot be
  seen by it, so that choice rests on the GEMM arguments of
  ckPairCalculator.C:1372-1420, :1444-1510 (cited in oracle/step.py).
* The reset: max |S - 2I| >= cp_norb_tol is fatal on the first step and
  afterwards replaces psi_no by psi, orthoT by I and v by the finite
  difference of psi.
"""
import numpy as np
import pytest

from oracle import density as OD
from oracle import layout as OL
from oracle import ortho as OO
from oracle import step as OS


@pytest.fixture(scope="module")
def small():
    from openatom_b200.system import System
    sysm = System(9.0, 20.0, 6, {"O": 1, "H": 2}, nfft=28, seed=5)
    lay = OL.Layout(9.0, 20.0, grid=28)
    dlay = OD.density_layout(9.0, 20.0, 28)
    psi = sysm.psi(device="cpu").numpy()
    return dict(sys=sysm, lay=lay, dlay=dlay, psi=psi, occ=np.ones(sysm.nstates),
                cmass=OS.cp_mass(lay, 25.0, 20.0))


def test_identity_orthoT_is_the_projection(small):
    lay = small["lay"]
    rng = np.random.default_rng(3)
    F = rng.standard_normal(small["psi"].shape) + 1j * rng.standard_normal(small["psi"].shape)
    fa, lam_a = OS.constrain(F, small["psi"], lay)
    fb, lam_b, gam = OS.constrain_dyn(F, small["psi"], np.eye(F.shape[0]), lay)
    assert np.max(np.abs(fa - fb)) < 1e-12 * np.max(np.abs(F))
    assert np.array_equal(lam_a, lam_b) and np.allclose(gam, lam_b, rtol=0, atol=1e-14)


def _drift(small, form, dt, t_end=4.0):
    p, v, dyn = small["psi"].copy(), np.zeros_like(small["psi"]), None
    cons = []
    for it in range(1, int(round(t_end / dt)) + 2):
        p, v, en, _, aux = OS.cp_step(p, v, small["occ"], small["sys"], small["lay"],
                                      small["dlay"], small["cmass"], dt, it, form=form, dyn=dyn,
                                      tol_norb=10.0)
        dyn = aux.get("dyn")
        S = OO.pc_overlap(p, p, small["lay"].kx)
        assert np.max(np.abs(S - 2.0 * np.eye(S.shape[0]))) < 1e-12
        if it > 1:
            cons.append(en["ETOT"] + en["FICT"])
    return cons[-1] - cons[0]


@pytest.mark.parametrize("form", ["ortho_t", "lowdin"])
def test_second_order_energy_conservation(small, form):
    d1 = _drift(small, form, 1.0)
    d2 = _drift(small, form, 0.5)
    assert abs(d1) < 2e-2
    assert 3.0 < d1 / d2 < 5.5


def test_norb_check_and_psiv_reset(small):
    s, lay = small, small["lay"]
    args = (s["occ"], s["sys"], lay, s["dlay"], s["cmass"], 5.0)
    with pytest.raises(RuntimeError):
        OS.cp_step(s["psi"], np.zeros_like(s["psi"]), *args, 1, tol_norb=1e-6)
    p1, v1, _, _, a1 = OS.cp_step(s["psi"], np.zeros_like(s["psi"]), *args, 1, tol_norb=1.0)
    d = a1["dyn"]
    assert not d["half_reset"] and d["resets"] == 0 and d["dev"] > 0
    # a tolerance below the second step's deviation resets
    p2, v2, _, _, a2 = OS.cp_step(p1, v1, *args, 2, dyn=d, tol_norb=1e-9)
    d2 = a2["dyn"]
    assert d2["half_reset"] and d2["resets"] == 1
    assert np.array_equal(d2["psi_no"], p2) and np.array_equal(d2["T"], np.eye(p2.shape[0]))
    assert np.allclose(v2, (p2 - p1) / 5.0, rtol=0, atol=1e-15)
    # the next step has no second half kick: the velocity after it is the
    # finite difference plus one half kick of its own force
    p3, v3, en3, _, a3 = OS.cp_step(p2, v2, *args, 3, dyn=d2, tol_norb=1.0)
    assert not a3["dyn"]["half_reset"] and a3["dyn"]["resets"] == 1

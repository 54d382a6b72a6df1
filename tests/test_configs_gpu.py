"""Step parity at the benchmark's own system sizes.

* 24-atom system (8 O, 16 H, L = 12 bohr, 32 states, 30 Ry, grid 48^3, EES
  s + p, B-spline order 8): two steps against the FP64 oracle run here.
  FP64 energies 1e-10 relative, psi 1e-9; mixed energy <= 1e-6 Ha/atom and
  atom forces <= 1e-5 Ha/bohr.
* 192-atom system (64 O, 128 H, L = 23.5, 128 states, 70 Ry, grid 128^3, EES):
  two steps against the committed oracle fixture tests/golden/step_water192.npz
  (tests/golden/make_step_golden.py): FP64 energies 1e-10 relative, atom
  forces 1e-9, psi and v at 4096 sampled points 1e-9 (v relative to its
  largest sample); mixed within the energy and force budget.
* 768-atom system (256 O, 512 H, L = 37.2, 1024 states, 70 Ry, grid 200^3,
  EES): too large for the oracle; two steps mixed against two steps FP64 on
  the GPU, within the same budget.
All use the orthoT constraint with cp_norb_tol 1.0 (these random starts
exceed the default on their first step).
"""
import os

import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu

DT = 5.0
TOL = 1.0
HERE = os.path.dirname(os.path.abspath(__file__))
SLOTS = {"EXC": 0, "MUXC": 1, "EHART": 2, "EEXT": 3, "EWD": 4, "EKE": 6, "ENL": 7, "ETOT": 8,
         "FICT": 9}


def _ctx(sysm, precision, ecut):
    from openatom_b200.context import StepContext
    ctx = StepContext(sysm.layout, sysm.nstates, precision=precision)
    ctx.set_atoms(sysm)
    ctx.set_nonlocal(sysm)
    ctx.set_cp_mass(25.0, ecut)
    ctx.set_constraint("ortho_t", TOL)
    return ctx


def _steps(sysm, psi0, precision, ecut, n=2, keep=None):
    """n steps from a copy of psi0; per step (energies, forces, psi, v) as
    numpy, psi/v only at the (state, point) pairs of keep (or whole)."""
    import torch
    ctx = _ctx(sysm, precision, ecut)
    try:
        psi = psi0.to("cuda", copy=True)
        v = torch.zeros_like(psi)
        occ = torch.ones(sysm.nstates, dtype=torch.float64, device="cuda")
        out = []
        for it in range(1, n + 1):
            e, f = ctx.cp_step(psi, v, occ, DT, it)
            _, ok = ctx.step_status()
            assert ok, (precision, it)
            if keep is None:
                p, vv = psi.cpu().numpy(), v.cpu().numpy()
            else:
                si = torch.from_numpy(keep[0]).cuda()
                pi = torch.from_numpy(keep[1]).cuda()
                p, vv = psi[si, pi].cpu().numpy(), v[si, pi].cpu().numpy()
            out.append((e.cpu().numpy().copy(), f.cpu().numpy().copy(), p, vv))
        assert ctx.device_errors() == 0
        return out
    finally:
        ctx.close()


@pytest.fixture(scope="module")
def config1():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    from oracle import density as OD
    from oracle import layout as OL
    from oracle import step as OS
    from openatom_b200.system import System
    sysm = System(12.0, 30.0, 32, {"O": 8, "H": 16}, nfft=48)
    lay = OL.Layout(12.0, 30.0, grid=48)
    dlay = OD.density_layout(12.0, 30.0, 48)
    psi0 = sysm.psi(device="cpu")
    cmass = OS.cp_mass(lay, 25.0, 30.0)
    p, v, dyn, ref = psi0.numpy(), np.zeros(tuple(psi0.shape), complex), None, []
    for it in (1, 2):
        p, v, en, f, aux = OS.cp_step(p, v, np.ones(sysm.nstates), sysm, lay, dlay, cmass, DT, it,
                                      nonlocal_on=True, tol_norb=TOL, dyn=dyn)
        dyn = aux["dyn"]
        ref.append((en, f, p, v))
    return dict(sys=sysm, psi0=psi0, ref=ref)


def test_config1_fp64_matches_oracle(config1):
    out = _steps(config1["sys"], config1["psi0"], "fp64", 30.0)
    for (e, f, p, v), (er, fr, pr, vr) in zip(out, config1["ref"]):
        for name, slot in SLOTS.items():
            assert abs(e[slot] - er[name]) <= 1e-10 * max(1.0, abs(er[name])), name
        assert np.max(np.abs(f - fr)) <= 1e-9 * max(1.0, np.max(np.abs(fr)))
        assert np.max(np.abs(p - pr)) <= 1e-9
        assert np.max(np.abs(v - vr)) <= 1e-9 * max(1.0, np.max(np.abs(vr)))


def test_config1_mixed_within_budget(config1):
    natm = config1["sys"].natm
    out = _steps(config1["sys"], config1["psi0"], "mixed", 30.0)
    for (e, f, p, v), (er, fr, pr, vr) in zip(out, config1["ref"]):
        assert abs(e[8] - er["ETOT"]) / natm <= 1e-6
        assert np.max(np.abs(f - fr)) <= 1e-5


@pytest.fixture(scope="module")
def config2():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    from openatom_b200.system import System
    g = np.load(os.path.join(HERE, "golden", "step_water192.npz"))
    sysm = System(23.5, 70.0, 128, {"O": 64, "H": 128}, nfft=128)
    return dict(sys=sysm, psi0=sysm.psi(device="cpu"), g=g,
                keep=(g["sample_state"].astype(np.int64), g["sample_point"].astype(np.int64)))


def test_config2_fp64_matches_oracle_fixture(config2):
    g = config2["g"]
    slots = [str(s) for s in g["slots"]]
    out = _steps(config2["sys"], config2["psi0"], "fp64", 70.0, keep=config2["keep"])
    for it, (e, f, p, v) in enumerate(out, start=1):
        er = g["energies_%d" % it]
        for k, name in enumerate(slots):
            assert abs(e[SLOTS[name]] - er[k]) <= 1e-10 * max(1.0, abs(er[k])), (it, name)
        fr = g["atom_force_%d" % it]
        assert np.max(np.abs(f - fr)) <= 1e-9 * max(1.0, np.max(np.abs(fr)))
        assert np.max(np.abs(p - g["psi_%d" % it])) <= 1e-9
        vr = g["v_%d" % it]
        assert np.max(np.abs(v - vr)) <= 1e-9 * max(1.0, np.max(np.abs(vr)))


def test_config2_mixed_within_budget(config2):
    g = config2["g"]
    slots = [str(s) for s in g["slots"]]
    natm = config2["sys"].natm
    out = _steps(config2["sys"], config2["psi0"], "mixed", 70.0, keep=config2["keep"])
    for it, (e, f, p, v) in enumerate(out, start=1):
        er = g["energies_%d" % it]
        assert abs(e[8] - er[slots.index("ETOT")]) / natm <= 1e-6, it
        assert np.max(np.abs(f - g["atom_force_%d" % it])) <= 1e-5, it


def test_config5_mixed_against_fp64():
    """The 768-atom, 1024-state, 200^3 system: two mixed steps against two
    FP64 steps of the same input on the GPU (energy per atom 1e-6, atom force
    1e-5, psi at 2048 sampled points 1e-5)."""
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    from openatom_b200.system import System
    sysm = System(37.2, 70.0, 1024, {"O": 256, "H": 512}, nfft=200)
    psi0 = sysm.psi()  # built on the GPU: 4.2 GB, no oracle needs it
    rng = np.random.default_rng(5)
    keep = (rng.integers(0, 1024, 2048), rng.integers(0, sysm.layout.npts, 2048))
    a = _steps(sysm, psi0, "fp64", 70.0, keep=keep)
    torch.cuda.empty_cache()
    b = _steps(sysm, psi0, "mixed", 70.0, keep=keep)
    for (ea, fa, pa, va), (eb, fb, pb, vb) in zip(a, b):
        assert np.isfinite(eb).all() and np.isfinite(fb).all()
        assert abs(ea[8] - eb[8]) / sysm.natm <= 1e-6
        assert np.max(np.abs(fa - fb)) <= 1e-5
        assert np.max(np.abs(pa - pb)) <= 1e-5

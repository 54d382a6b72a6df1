"""State FFT path on the GPU (through the C ABI) against the FP64 oracle.

Tolerances (relative to the largest magnitude of the oracle result):
FP64 path 1e-11; mixed path (FP32 FFTs, FP64 accumulation) 2e-5.
"""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-11, "mixed": 2e-5}
# (box bohr, ecut Ry, grid) -> grids 28, 42 (reference radixme), 48 (grid override);
# 32, 64, 80, 96 and 128 run the register (shuffle) plane FFTs
CASES = [(9.0, 20.0, None), (12.0, 30.0, None), (12.0, 30.0, 48), (9.0, 20.0, 32),
         (12.0, 30.0, 64), (12.0, 30.0, 80), (12.0, 30.0, 96), (12.0, 30.0, 128)]


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module", params=CASES, ids=lambda c: "L%g_E%g_n%s" % c)
def system(request):
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    from oracle import layout as OL
    from openatom_b200.layout import StateLayout
    from openatom_b200.system import make_psi
    box, ecut, grid = request.param
    lay = StateLayout(box, ecut, nfft=grid)
    olay = OL.Layout(box, ecut, grid=grid)
    assert np.array_equal(lay.kx, olay.kx)
    S = 6
    psi = make_psi(lay, S, seed=5, device="cuda")
    occ = torch.tensor([1.0, 1.0, 0.5, 1.0, 0.25, 1.0], dtype=torch.float64, device="cuda")
    return dict(lay=lay, olay=olay, psi=psi, occ=occ, S=S)


@pytest.fixture(params=["fp64", "mixed"])
def ctx(request, system):
    from openatom_b200.context import StepContext
    c = StepContext(system["lay"], system["S"], precision=request.param)
    yield c
    c.close()


def test_expand_pack_roundtrip(system, ctx):
    from oracle import fftpath as OF
    psi = system["psi"]
    lines = ctx.expand_gspace(psi)
    ref = OF.expand(psi.cpu().numpy(), system["olay"])
    assert np.array_equal(lines.cpu().numpy(), ref)
    back = ctx.pack_gspace(lines)
    assert np.array_equal(back.cpu().numpy(), psi.cpu().numpy())


def test_g_to_r_matches_oracle(system, ctx):
    from oracle import fftpath as OF
    pr = ctx.fft_g_to_r(system["psi"]).cpu().numpy()
    ref = OF.state_g_to_r(system["psi"].cpu().numpy(), system["olay"])
    assert relerr(pr, ref) < TOL[ctx.precision]


def test_r_to_g_matches_oracle(system, ctx):
    import torch
    from oracle import fftpath as OF
    n = system["lay"].n
    g = torch.Generator(device="cpu").manual_seed(3)
    f = torch.randn((system["S"], n, n, n), generator=g, dtype=torch.float64)
    out = ctx.fft_r_to_g(f.cuda()).cpu().numpy()
    ref = OF.state_r_to_g(f.numpy(), system["olay"])
    assert relerr(out, ref) < TOL[ctx.precision]


def test_density_matches_oracle(system, ctx):
    from oracle import fftpath as OF
    rho = ctx.density(system["psi"], system["occ"]).cpu().numpy()
    lay = system["lay"]
    ref = OF.density(system["psi"].cpu().numpy(), system["olay"], system["occ"].cpu().numpy(),
                     lay.vol)
    assert relerr(rho, ref) < TOL[ctx.precision]
    # electron count: states normalised to 2 (S = 2 I)
    nel = rho.sum() * lay.vol / lay.n ** 3
    assert abs(nel - 2.0 * float(system["occ"].sum())) < 1e-9 * nel + (1e-5 if ctx.precision == "mixed" else 0)


def test_vks_psi_and_kinetic_match_oracle(system, ctx):
    import torch
    from oracle import fftpath as OF
    lay = system["lay"]
    n = lay.n
    g = torch.Generator(device="cpu").manual_seed(9)
    vks = torch.randn((n, n, n), generator=g, dtype=torch.float64)
    psi = system["psi"]
    occ = system["occ"]
    force, eke = ctx.vks_psi(psi, vks.cuda(), occ, kinetic=True)
    pn, on = psi.cpu().numpy(), occ.cpu().numpy()
    fv = OF.vpsi_force(pn, vks.numpy(), system["olay"], on)
    f_ref = OF.add_forces(fv, None, system["olay"])
    f_ref, e_ref = OF.eke(f_ref, pn, system["olay"], on, lay.ecut_ry)
    assert relerr(force.cpu().numpy(), f_ref) < TOL[ctx.precision]
    assert relerr(eke.cpu().numpy(), e_ref) < 1e-12


def test_eke_entry_matches_oracle(system, ctx):
    import torch
    from oracle import fftpath as OF
    psi = system["psi"]
    occ = system["occ"]
    f0 = torch.zeros_like(psi)
    e = ctx.eke(f0, psi, occ)
    f_ref, e_ref = OF.eke(np.zeros(psi.shape, complex), psi.cpu().numpy(), system["olay"],
                          occ.cpu().numpy(), system["lay"].ecut_ry)
    assert relerr(f0.cpu().numpy(), f_ref) < 1e-13
    assert relerr(e.cpu().numpy(), e_ref) < 1e-13


def test_adjointness_of_the_two_transforms(system, ctx):
    """<F(psi), f> = sum_r psi(r) f(r) with the double-pack weights (size independent)."""
    import torch
    lay = system["lay"]
    n = lay.n
    psi = system["psi"]
    g = torch.Generator(device="cpu").manual_seed(4)
    f = torch.randn((system["S"], n, n, n), generator=g, dtype=torch.float64).cuda()
    pr = ctx.fft_g_to_r(psi)
    lhs = (pr * f).sum(dim=(1, 2, 3))
    Fg = ctx.fft_r_to_g(f)
    w = torch.from_numpy(np.where(lay.kx == 0, 1.0, 2.0)).cuda()
    rhs = (w[None] * (psi.conj() * Fg).real).sum(dim=1)
    tol = 1e-10 if ctx.precision == "fp64" else 1e-4
    assert float((lhs - rhs).abs().max() / lhs.abs().max()) < tol


@pytest.mark.parametrize("form", [0, 1, 2])
def test_plane_pass_forms_match_oracle(system, form):
    """Density and V.psi in a mixed context with each plane-pass form: 0
    shared-memory Stockham, 1 register shuffles, 2 the two-stage form of
    fft_p16.cuh (grids 32, 64, 128; the others run form 1 there)."""
    import torch
    from oracle import fftpath as OF
    from openatom_b200.context import StepContext
    lay, olay = system["lay"], system["olay"]
    psi, occ = system["psi"], system["occ"]
    ctx = StepContext(lay, system["S"], precision="mixed")
    try:
        ctx.tune_set({"plane_shfl": form})
        pn, on = psi.cpu().numpy(), occ.cpu().numpy()
        rho = ctx.density(psi, occ).cpu().numpy()
        ref = OF.density(pn, olay, on, lay.vol)
        assert relerr(rho, ref) < TOL["mixed"]
        n = lay.n
        g = torch.Generator(device="cpu").manual_seed(9)
        vks = torch.randn((n, n, n), generator=g, dtype=torch.float64)
        force, eke = ctx.vks_psi(psi, vks.cuda(), occ, kinetic=True)
        fv = OF.vpsi_force(pn, vks.numpy(), olay, on)
        f_ref = OF.add_forces(fv, None, olay)
        f_ref, e_ref = OF.eke(f_ref, pn, olay, on, lay.ecut_ry)
        assert relerr(force.cpu().numpy(), f_ref) < TOL["mixed"]
        assert ctx.device_errors() == 0
    finally:
        ctx.close()


@pytest.mark.parametrize("form", [0, 2])
def test_plane_pass_forms_n200(form):
    """The 200^3 grid (the largest benchmark system's): V.psi in a mixed context
    with the shared-memory Stockham form (0) and the two-stage 20 x 10 form of
    fft_t20.cuh (2; the density pass runs form 0 there), against the oracle."""
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    from oracle import fftpath as OF
    from oracle import layout as OL
    from openatom_b200.context import StepContext
    from openatom_b200.layout import StateLayout
    from openatom_b200.system import make_psi
    lay = StateLayout(12.0, 30.0, nfft=200)
    olay = OL.Layout(12.0, 30.0, grid=200)
    S = 6
    psi = make_psi(lay, S, seed=5, device="cuda")
    occ = torch.tensor([1.0, 1.0, 0.5, 1.0, 0.25, 1.0], dtype=torch.float64, device="cuda")
    ctx = StepContext(lay, S, precision="mixed")
    try:
        ctx.tune_set({"plane_shfl": form})
        pn, on = psi.cpu().numpy(), occ.cpu().numpy()
        rho = ctx.density(psi, occ).cpu().numpy()
        assert relerr(rho, OF.density(pn, olay, on, lay.vol)) < TOL["mixed"]
        g = torch.Generator(device="cpu").manual_seed(9)
        vks = torch.randn((200, 200, 200), generator=g, dtype=torch.float64)
        force, eke = ctx.vks_psi(psi, vks.cuda(), occ, kinetic=True)
        fv = OF.vpsi_force(pn, vks.numpy(), olay, on)
        f_ref = OF.add_forces(fv, None, olay)
        f_ref, e_ref = OF.eke(f_ref, pn, olay, on, lay.ecut_ry)
        assert relerr(force.cpu().numpy(), f_ref) < TOL["mixed"]
        assert ctx.device_errors() == 0
    finally:
        ctx.close()

"""Independent systems of different sizes stepped by one batch graph: the
same results as stepping each context alone, one captured graph holding all
of their kernels."""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu

# small enough that the first step passes the default cp_norb_tol (0.003) of the
# orthoT constraint on these random states; later steps may take the PsiV reset
DT = 1.0

SYSTEMS = [  # (box, ecut, states, atoms, grid)
    (9.0, 20.0, 6, {"O": 1, "H": 2}, 28),
    (9.0, 30.0, 12, {"O": 2, "H": 4}, 32),
    (12.0, 30.0, 16, {"O": 4, "H": 8}, 48),
]


def _make(precision):
    import torch
    from openatom_b200.context import StepContext
    from openatom_b200.system import System
    out = []
    for k, (box, ec, S, atoms, grid) in enumerate(SYSTEMS):
        sysm = System(box, ec, S, atoms, nfft=grid, seed=20 + k)
        ctx = StepContext(sysm.layout, S, precision=precision)
        ctx.set_atoms(sysm)
        ctx.set_nonlocal(sysm)
        ctx.set_cp_mass(25.0, ec)
        ctx.set_graph(False)
        psi = sysm.psi()
        out.append(dict(sys=sysm, ctx=ctx, psi=psi, v=torch.zeros_like(psi),
                        occ=torch.ones(S, dtype=torch.float64, device="cuda"),
                        e=torch.zeros(16, dtype=torch.float64, device="cuda"),
                        f=torch.zeros((sysm.natm, 3), dtype=torch.float64, device="cuda")))
    return out


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batch_graph_matches_single_contexts(precision):
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    from openatom_b200 import _lib
    from openatom_b200.batch import StepBatch
    a, b = _make(precision), _make(precision)
    batch = StepBatch([d["ctx"] for d in a])
    try:
        caps = []
        n0 = _lib.lib().cpstep_launch_count()
        for it in range(1, 6):
            batch.step([d["psi"] for d in a], [d["v"] for d in a], [d["occ"] for d in a], DT,
                       it, [d["e"] for d in a], [d["f"] for d in a])
            caps.append(batch.status()[1])
        torch.cuda.synchronize()
        nb = _lib.lib().cpstep_launch_count() - n0
        n0 = _lib.lib().cpstep_launch_count()
        for it in range(1, 6):
            for d in b:
                d["ctx"].cp_step(d["psi"], d["v"], d["occ"], DT, it, d["e"], d["f"])
        torch.cuda.synchronize()
        ns = _lib.lib().cpstep_launch_count() - n0
        assert caps == [False, False, True, True, True]
        assert nb == ns
        for da, db in zip(a, b):
            for k in ("psi", "v", "e", "f"):
                assert bool((da[k] == db[k]).all()), k
            ok = da["ctx"].step_status()[1]
            assert ok
        # a context's setter forces a new capture
        a[1]["ctx"].set_cp_mass(25.0, 30.0)
        batch.step([d["psi"] for d in a], [d["v"] for d in a], [d["occ"] for d in a], DT, 6,
                   [d["e"] for d in a], [d["f"] for d in a])
        assert not batch.status()[1]
        torch.cuda.synchronize()
        assert all(np.isfinite(d["e"].cpu().numpy()).all() for d in a)
    finally:
        batch.close()
        for d in a + b:
            d["ctx"].close()

"""The oracle's builder of the synthetic systems (oracle/synth.py, used by the
timed CPU baseline so that it loads nothing of the product) against the
product's (openatom_b200/system.py): the same layout, atoms, tables and
channels, and the same coefficients to FP64 rounding of the orthonormalisation
(numpy's eigh against torch's on the CPU).  Host only."""
import numpy as np
import pytest


@pytest.mark.parametrize("box,ecut,S,counts,grid", [
    (9.0, 20.0, 6, {"O": 1, "H": 2}, 28),
    (23.5, 70.0, 128, {"O": 64, "H": 128}, 128),
])
def test_oracle_synth_is_the_product_system(box, ecut, S, counts, grid):
    from oracle import synth as OSY
    from openatom_b200.system import System
    a = System(box, ecut, S, counts, nfft=grid)
    b = OSY.System(box, ecut, S, counts, nfft=grid)
    for k in ("kx", "ky", "kz"):
        assert np.array_equal(getattr(a.layout, k), getattr(b.layout, k)), k
    assert np.allclose(a.layout.g2(), b.layout.g2, rtol=1e-15, atol=0)
    assert np.array_equal(a.pos, b.pos) and np.array_equal(a.typ, b.typ)
    for k in ("vps", "gzvps", "q"):
        assert np.array_equal(a.tab[k], b.tab[k]), k
    assert a.tab["gmin"] == b.tab["gmin"] and a.tab["dg"] == b.tab["dg"]
    assert a.alp_ewd == b.alp_ewd
    assert len(a.channels) == len(b.channels)
    for ca, cb in zip(a.channels, b.channels):
        assert {k: ca[k] for k in ("type", "l", "m", "gzvps0", "vnorm")} == \
               {k: cb[k] for k in ("type", "l", "m", "gzvps0", "vnorm")}
        assert np.array_equal(ca["vnl"], cb["vnl"])
    pa = a.psi(device="cpu").numpy()
    pb = b.psi()
    assert np.max(np.abs(pa - pb)) < 1e-12

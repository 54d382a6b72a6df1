"""State files in the reference's format (util.C writeStateFile / readState):
the library's writer against the oracle's byte stream, round trips through the
library's reader, the redundant Gx=0 half, and the error cases.  Host only."""
import gzip

import numpy as np
import pytest

from oracle import statefile as OSF


@pytest.fixture(scope="module")
def lay():
    from openatom_b200.layout import StateLayout
    return StateLayout(12.0, 30.0)


def _coef(lay, seed):
    """Random packed coefficients with the Gx=0 symmetry the layout stores:
    a redundant point holds the conjugate of its partner, G=0 is real."""
    rng = np.random.default_rng(seed)
    c = rng.standard_normal(lay.npts) + 1j * rng.standard_normal(lay.npts)
    c *= np.exp(-0.01 * (lay.kx ** 2 + lay.ky ** 2 + lay.kz ** 2))
    where = {(int(x), int(y), int(z)): p for p, (x, y, z) in enumerate(zip(lay.kx, lay.ky, lay.kz))}
    for p, (x, y, z) in enumerate(zip(lay.kx, lay.ky, lay.kz)):
        if x == 0 and (y < 0 or (y == 0 and z < 0)):
            c[p] = np.conj(c[where[(0, -int(y), -int(z))]])
        if x == 0 and y == 0 and z == 0:
            c[p] = c[p].real
    return c


@pytest.mark.parametrize("fmt", ["text", "binary", "text.gz", "binary.gz"])
def test_writer_matches_oracle_bytes(lay, tmp_path, fmt):
    from openatom_b200.statefile import write_state
    c = _coef(lay, 1)
    path = tmp_path / "state1.out"
    write_state(path, c, lay, fmt, grid=(48, 48, 48))
    binary = fmt.startswith("binary")
    want = OSF.write_bytes(c, lay.kx, lay.ky, lay.kz, (48, 48, 48), binary)
    if fmt.endswith(".gz"):
        got = gzip.open(str(path) + ".gz", "rb").read()
    else:
        got = path.read_bytes()
    assert got == want
    # header: the stored half sphere and G=0
    nhalf = int(np.sum(~((lay.kx == 0) & ((lay.ky < 0) | ((lay.ky == 0) & (lay.kz < 0))))))
    if not binary:
        assert got.split(b"\n")[0] == b"%d 48 48 48" % nhalf
        assert got.rstrip(b"\n").split(b"\n")[-1].split()[2:] == [b"0", b"0", b"0"]


@pytest.mark.parametrize("fmt", ["binary", "binary.gz"])
def test_binary_round_trip_is_exact(lay, tmp_path, fmt):
    from openatom_b200.statefile import read_state, write_state
    c = _coef(lay, 2)
    path = tmp_path / "s.bin"
    write_state(path, c, lay, fmt, grid=(50, 48, 46))
    back, grid = read_state(path, lay, fmt)
    assert grid == (50, 48, 46)
    assert np.array_equal(back, c)


@pytest.mark.parametrize("fmt", ["text", "text.gz"])
def test_text_round_trip_matches_oracle_parse(lay, tmp_path, fmt):
    from openatom_b200.statefile import read_state, write_state
    c = _coef(lay, 3)
    path = tmp_path / "s.txt"
    write_state(path, c, lay, fmt)
    back, _ = read_state(path, lay, fmt)
    data = gzip.open(str(path) + ".gz", "rb").read() if fmt.endswith(".gz") else path.read_bytes()
    recs, _ = OSF.read_records(data, binary=False)
    assert np.array_equal(back, OSF.pack(recs, lay.kx, lay.ky, lay.kz))
    # %g keeps six significant digits
    assert np.max(np.abs(back - c) / np.maximum(np.abs(c), 1e-300)) < 1e-5


def test_reader_fills_redundant_half_from_partners(lay, tmp_path):
    from openatom_b200.statefile import read_state
    c = _coef(lay, 4)
    path = tmp_path / "s.bin"
    # a file written by the oracle (the reference's writer restated)
    path.write_bytes(OSF.write_bytes(c, lay.kx, lay.ky, lay.kz, (48, 48, 48), True))
    back, _ = read_state(path, lay, "binary")
    assert np.array_equal(back, c)
    red = (lay.kx == 0) & ((lay.ky < 0) | ((lay.ky == 0) & (lay.kz < 0)))
    assert red.sum() > 0


def test_multi_state_helpers(lay, tmp_path):
    from openatom_b200.statefile import read_states, write_states
    psi = np.stack([_coef(lay, 10 + s) for s in range(3)])
    pat = str(tmp_path / "state%d.out")
    write_states(pat, psi, lay, "binary")
    assert (tmp_path / "state1.out").exists() and (tmp_path / "state3.out").exists()
    assert np.array_equal(read_states(pat, 3, lay, "binary"), psi)


def test_errors(lay, tmp_path):
    from openatom_b200 import _lib
    from openatom_b200.layout import StateLayout
    from openatom_b200.statefile import read_state, write_state
    with pytest.raises(_lib.CpstepError):
        read_state(tmp_path / "missing.bin", lay, "binary")
    # a smaller sphere's file lacks points of this layout
    small = StateLayout(12.0, 20.0)
    path = tmp_path / "small.bin"
    write_state(path, _coef(small, 5), small, "binary")
    with pytest.raises(_lib.CpstepError) as e:
        read_state(path, lay, "binary")
    assert e.value.code == _lib.CPSTEP_ERR_LAYOUT
    # a truncated file
    full = tmp_path / "full.bin"
    write_state(full, _coef(lay, 6), lay, "binary")
    full.write_bytes(full.read_bytes()[:1000])
    with pytest.raises(_lib.CpstepError):
        read_state(full, lay, "binary")

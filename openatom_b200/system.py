"""Synthetic CP systems of the benchmark shapes (seeded, reproducible).

Coefficients: complex Gaussian x exp(-|G|^2/8) on the packed layout, with the
Gamma-point symmetry of the stored Gx=0 lower half (c(0,-ky,-kz) = conj
c(0,ky,kz), the relation flip_data_set builds, para_grp_parse.C:229-240) and a
real G=0 term, then Loewdin-orthonormalised to S = 2 I, the normalisation the
reference's Ortho expects (doc/orthoStoT.txt:9-20; cp_lowdin.C:197-199 halves S).
S_ij = sum_p wpt_p Re(conj c_i(p) c_j(p)), wpt = 1 on Gx=0 and 2 elsewhere, is
the overlap PairCalculator forms from the Gx=0-rescaled real view
(CP_State_GSpacePlane.C:3120-3123, ckPairCalculator.C:682-751).

The orthonormalisation runs in FP64 on the GPU with torch (input preparation,
not part of any measured path).
"""
import numpy as np
import torch


def kx0_partner(layout):
    """Index of the (0,-ky,-kz) partner of every Gx=0 point (-1 elsewhere)."""
    kx, ky, kz = layout.kx, layout.ky, layout.kz
    idx = np.full(layout.npts, -1, dtype=np.int64)
    sel = np.nonzero(kx == 0)[0]
    key = {(int(ky[i]), int(kz[i])): int(i) for i in sel}
    for i in sel:
        idx[i] = key[(-int(ky[i]), -int(kz[i]))]
    return idx


def overlap_weights(layout):
    return np.where(layout.kx == 0, 1.0, 2.0)


def make_psi(layout, nstates, seed=1234, device="cuda", orthonormalize=True):
    """[nstates, npts] complex128 coefficients on `device`."""
    rng = np.random.default_rng(seed)
    g2 = layout.g2()
    env = np.exp(-g2 / 8.0)
    re = rng.standard_normal((nstates, layout.npts))
    im = rng.standard_normal((nstates, layout.npts))
    c = (re + 1j * im) * env[None, :]
    part = kx0_partner(layout)
    sel = np.nonzero(part >= 0)[0]
    # make the Gx=0 plane Hermitian: keep the ky>0 or (ky=0,kz>=0) member, mirror it
    keep = sel[(layout.ky[sel] > 0) | ((layout.ky[sel] == 0) & (layout.kz[sel] >= 0))]
    c[:, part[keep]] = np.conj(c[:, keep])
    g0 = np.nonzero((layout.kx == 0) & (layout.ky == 0) & (layout.kz == 0))[0]
    c[:, g0] = c[:, g0].real
    psi = torch.from_numpy(c).to(device)
    if orthonormalize:
        psi = loewdin(psi, torch.from_numpy(overlap_weights(layout)).to(device))
    return psi


def overlap(psi, w):
    a = torch.view_as_real(psi)  # [S, npts, 2]
    aw = a * w[None, :, None].to(a.dtype)
    return torch.einsum("spc,tpc->st", aw, a)


def loewdin(psi, w):
    """psi <- (S/2)^(-1/2) psi so that the weighted overlap is 2 I (FP64)."""
    S = overlap(psi, w)
    evals, evecs = torch.linalg.eigh(S / 2.0)
    T = evecs @ torch.diag(evals.rsqrt()) @ evecs.T
    return (T.to(psi.dtype) @ psi).contiguous()

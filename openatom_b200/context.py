"""Python host mirror of the libcpstep context (device memory via torch).

Each method is a thin call through the C ABI of ``include/cpstep.h``; the
docstrings name the OpenAtom routine the call replaces.  Arrays are torch CUDA
tensors: coefficients complex128 [nstates, npts] in the reference's packed
order, real-space grids float64 [nz, ny, nx].
"""
import ctypes

import torch

from . import _lib
from ._lib import ptr


class StepContext:
    def __init__(self, layout, nstates, precision="fp64", ecut_ry=None, device=None):
        if not torch.cuda.is_available():
            raise RuntimeError("StepContext needs a CUDA device (no CPU fallback)")
        self.layout = layout
        self.nstates = int(nstates)
        self.precision = precision
        prec = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED}[precision]
        self.device = torch.device(device or "cuda")
        self.n = layout.n
        kx, pkx = _lib.int_array(layout.kx)
        ky, pky = _lib.int_array(layout.ky)
        kz, pkz = _lib.int_array(layout.kz)
        runs, pruns = _lib.int_array(layout.runs.reshape(-1))
        hm = layout.hmat.astype("float64")
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.call("cpstep_ctx_create", ctypes.byref(h), prec, self.nstates, layout.npts,
                      pkx, pky, pkz, len(layout.runs), pruns, self.n, self.n, self.n,
                      hm.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                      float(ecut_ry if ecut_ry is not None else layout.ecut_ry))
        self._h = h
        self._stream = None
        self._sync_stream()

    # -- plumbing ----------------------------------------------------------
    def _sync_stream(self):
        s = torch.cuda.current_stream(self.device).cuda_stream
        if s != self._stream:
            _lib.call("cpstep_ctx_set_stream", self._h, ctypes.c_void_p(s))
            self._stream = s

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib().cpstep_ctx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk_psi(self, psi, nstates=None):
        S = self.nstates if nstates is None else nstates
        if psi.dtype != torch.complex128 or not psi.is_cuda or not psi.is_contiguous():
            raise ValueError("psi must be a contiguous complex128 CUDA tensor")
        if psi.shape != (S, self.layout.npts):
            raise ValueError("psi shape %s != (%d, %d)" % (tuple(psi.shape), S, self.layout.npts))

    def info(self):
        nl, npx = ctypes.c_int(), ctypes.c_int()
        _lib.call("cpstep_ctx_info", self._h, ctypes.byref(nl), ctypes.byref(npx))
        return nl.value, npx.value

    # -- FFTcache mirrors ----------------------------------------------------
    def expand_gspace(self, psi):
        """FFTcache::expandGSpace (fftCache.C:460-507): packed -> [S, nlines, nz]."""
        self._sync_stream()
        S = psi.shape[0]
        out = torch.empty((S, self.layout.nlines, self.n), dtype=torch.complex128,
                          device=self.device)
        _lib.call("cpstep_expand_gspace", self._h, ptr(psi), ptr(out), S)
        return out

    def pack_gspace(self, lines):
        """FFTcache::packGSpace (fftCache.C:517-553): [S, nlines, nz] -> packed."""
        self._sync_stream()
        S = lines.shape[0]
        out = torch.zeros((S, self.layout.npts), dtype=torch.complex128, device=self.device)
        _lib.call("cpstep_pack_gspace", self._h, ptr(lines), ptr(out), S)
        return out

    def fft_g_to_r(self, psi):
        """doStpFFTGtoR_Gchare + transpose + doStpFFTGtoR_Rchare: psi(r) [S, n, n, n]."""
        self._sync_stream()
        S = psi.shape[0]
        self._chk_psi(psi, S)
        out = torch.empty((S, self.n, self.n, self.n), dtype=torch.float64, device=self.device)
        _lib.call("cpstep_stp_fft_gtor", self._h, ptr(psi), ptr(out), S)
        return out

    def fft_r_to_g(self, f):
        """doStpFFTRtoG_Rchare + transpose + doStpFFTRtoG_Gchare (unscaled)."""
        self._sync_stream()
        S = f.shape[0]
        f = f.contiguous()
        out = torch.empty((S, self.layout.npts), dtype=torch.complex128, device=self.device)
        _lib.call("cpstep_stp_fft_rtog", self._h, ptr(f), ptr(out), S)
        return out

    def density(self, psi, occ):
        """rho(r) = sum occ psi^2 / vol (CP_State_RealSpacePlane.C:349-355 + reduction)."""
        self._sync_stream()
        self._chk_psi(psi)
        rho = torch.empty((self.n, self.n, self.n), dtype=torch.float64, device=self.device)
        _lib.call("cpstep_density", self._h, ptr(psi), ptr(occ), ptr(rho))
        return rho

    def vks_psi(self, psi, vks, occ, kinetic=True):
        """F = addForces(-2/N FFT^-1[occ V psi]) (+ CP_eke_calc when kinetic)."""
        self._sync_stream()
        self._chk_psi(psi)
        force = torch.empty_like(psi)
        eke = torch.empty(self.nstates, dtype=torch.float64, device=self.device) if kinetic else None
        _lib.call("cpstep_vks_psi", self._h, ptr(psi), ptr(vks.contiguous()), ptr(occ),
                  ptr(force), ptr(eke))
        return force, eke

    def eke(self, force, psi, occ):
        """CPNONLOCAL::CP_eke_calc on all states; updates force in place."""
        self._sync_stream()
        e = torch.empty(self.nstates, dtype=torch.float64, device=self.device)
        _lib.call("cpstep_eke", self._h, ptr(force), ptr(psi), ptr(occ), ptr(e))
        return e

    # -- PairCalculator / Ortho ---------------------------------------------
    def pc_overlap(self, a, b, alpha=1.0, beta=0.0, out=None):
        """S or lambda: out(i,j) = alpha sum_p wpt Re(conj a_i b_j) + beta out (col-major)."""
        self._sync_stream()
        na, nb = a.shape[0], b.shape[0]
        if out is None:
            out = torch.zeros((nb, na), dtype=torch.float64, device=self.device)  # col-major (na x nb)
        _lib.call("cpstep_pc_overlap", self._h, ptr(a), ptr(b), na, nb, float(alpha), float(beta),
                  ptr(out), na)
        return out

    def pc_backmultiply(self, m_colmajor, x, nout=None, alpha=1.0, beta=0.0, out=None):
        """out_i = alpha sum_j M(j,i) x_j + beta out_i  (psi.T, psi.gamma, F.T)."""
        self._sync_stream()
        nin = x.shape[0]
        nout = nin if nout is None else nout
        if out is None:
            out = torch.zeros((nout, self.layout.npts), dtype=torch.complex128, device=self.device)
        ldm = m_colmajor.shape[1]  # tensor [ncols][ld] holds a column-major matrix
        _lib.call("cpstep_pc_backmultiply", self._h, ptr(m_colmajor), ldm, ptr(x), nin, ptr(out),
                  nout, float(alpha), float(beta))
        return out

    def ortho_tmat(self, S, mixed=False, scale=False, tol=1e-15, max_iter=10):
        """T = (S/2)^(-1/2) (CPORTHOG::get_iter_Tmat); returns (T, iterations, rms)."""
        self._sync_stream()
        n = S.shape[0]
        T = torch.empty_like(S)
        it, rms = ctypes.c_int(), ctypes.c_double()
        mode = (1 if mixed else 0) | (2 if scale else 0)
        _lib.call("cpstep_ortho_tmat", self._h, ptr(S.contiguous()), ptr(T), n, mode, float(tol),
                  int(max_iter), ctypes.byref(it), ctypes.byref(rms))
        return T, it.value, rms.value

    def dgemm(self, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
        """Column-major DGEMM on device tensors (the myGEMM wrapper)."""
        self._sync_stream()
        _lib.call("cpstep_dgemm", self._h, transa.encode(), transb.encode(), m, n, k,
                  float(alpha), ptr(A), lda, ptr(B), ldb, float(beta), ptr(C), ldc)
        return C

    # -- density side --------------------------------------------------------
    def set_atoms(self, system):
        """Atoms + local pseudopotential tables (the PINY data CP_hart_eext_calc reads)."""
        import numpy as np
        tab = system.tab
        typ, ptyp = _lib.int_array(system.typ)
        pos = np.ascontiguousarray(system.pos, dtype=np.float64)
        q = np.ascontiguousarray(tab["q"], dtype=np.float64)
        vps = np.ascontiguousarray(tab["vps"], dtype=np.float64)
        gz = np.ascontiguousarray(tab["gzvps"], dtype=np.float64)
        dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        self._sync_stream()
        _lib.call("cpstep_set_atoms", self._h, len(system.typ), len(tab["q"]), ptyp, dp(pos),
                  dp(q), int(tab["nspl"]), float(tab["gmin"]), float(tab["dg"]), dp(vps), dp(gz),
                  float(system.alp_ewd))
        self.natm = len(system.typ)

    def set_nonlocal(self, system, nkf=None):
        """EES non-local channels of `system` (cpstep_set_nonlocal); nkf defaults
        to the reference's NL grid rule for the layout's kmax."""
        import numpy as np
        chans = system.channels
        if nkf is None:
            nkf = _lib.lib().cpstep_nl_grid_size(int(self.layout.kmax), 1.2, 8)
        ct, pct = _lib.int_array([c["type"] for c in chans])
        cl, pcl = _lib.int_array([c["l"] for c in chans])
        cm, pcm = _lib.int_array([c["m"] for c in chans])
        vnl = np.ascontiguousarray(np.stack([c["vnl"] for c in chans]), dtype=np.float64)
        gz = np.ascontiguousarray([c["gzvps0"] for c in chans], dtype=np.float64)
        vn = np.ascontiguousarray([c["vnorm"] for c in chans], dtype=np.float64)
        dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        self._sync_stream()
        _lib.call("cpstep_set_nonlocal", self._h, int(nkf), 8, len(chans), pct, pcl, pcm,
                  dp(vnl), dp(gz), dp(vn))
        self.nkf = int(nkf)
        return self.nkf

    def ees_nonlocal(self, psi, occ, fpsi=None, forces=True):
        """EES non-local pass: returns (fpsi accumulated, energies, atom forces)."""
        self._sync_stream()
        if fpsi is None:
            fpsi = torch.zeros_like(psi)
        e = self._energies()
        f = torch.zeros((self.natm, 3), dtype=torch.float64, device=self.device) if forces else None
        _lib.call("cpstep_ees_nonlocal", self._h, ptr(psi), ptr(occ), ptr(fpsi), ptr(e), ptr(f))
        return fpsi, e, f

    def set_nonlocal_sf(self, system):
        """Structure-factor (non-EES) non-local path with the l = 0 channels of
        `system` (cpstep_set_nonlocal_sf); replaces an EES set-up."""
        import numpy as np
        chans = [c for c in system.channels if c["l"] == 0]
        ct, pct = _lib.int_array([c["type"] for c in chans])
        cl, pcl = _lib.int_array([0 for _ in chans])
        cm, pcm = _lib.int_array([0 for _ in chans])
        vnl = np.ascontiguousarray(np.stack([c["vnl"] for c in chans]), dtype=np.float64)
        gz = np.ascontiguousarray([c["gzvps0"] for c in chans], dtype=np.float64)
        vn = np.ascontiguousarray([c["vnorm"] for c in chans], dtype=np.float64)
        dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        self._sync_stream()
        _lib.call("cpstep_set_nonlocal_sf", self._h, len(chans), pct, pcl, pcm, dp(vnl), dp(gz),
                  dp(vn))

    def sf_nonlocal(self, psi, occ, fpsi=None, forces=True):
        """Structure-factor non-local pass: (fpsi accumulated, energies, atom forces)."""
        self._sync_stream()
        if fpsi is None:
            fpsi = torch.zeros_like(psi)
        e = self._energies()
        f = torch.zeros((self.natm, 3), dtype=torch.float64, device=self.device) if forces else None
        _lib.call("cpstep_sf_nonlocal", self._h, ptr(psi), ptr(occ), ptr(fpsi), ptr(e), ptr(f))
        return fpsi, e, f

    def set_positions(self, pos):
        """New atom positions (natm x 3, bohr, host array): cpstep_set_positions."""
        import numpy as np
        p = np.ascontiguousarray(pos, dtype=np.float64)
        self._sync_stream()
        _lib.call("cpstep_set_positions", self._h, p.ctypes.data_as(ctypes.c_void_p))

    def ion_forces(self, forces=None):
        """CP_getionforce: (forces += real-space Ewald forces, energies with
        EWD_RS = pot_ewd_rs + vself + vbgr) at the context's positions."""
        self._sync_stream()
        if forces is None:
            forces = torch.zeros((self.natm, 3), dtype=torch.float64, device=self.device)
        e = self._energies()
        _lib.call("cpstep_ion_forces", self._h, ptr(forces), ptr(e))
        return forces, e

    def atoms_integrate(self, itime, pos, vel, forces, mass, dt):
        """Velocity-Verlet step of the ions (in place on pos, vel [natm, 3]):
        NVE, or the NVT branch with massive Nose-Hoover chains once
        set_atom_thermostat has been called (the chains are applied around the
        kicks on the device).  The context's positions follow.  Returns E_kin
        at the step's start."""
        self._sync_stream()
        ek = torch.zeros(1, dtype=torch.float64, device=self.device)
        _lib.call("cpstep_atoms_integrate", self._h, int(itime), ptr(pos), ptr(vel), ptr(forces),
                  ptr(mass), float(dt), ptr(ek))
        return float(ek)

    def rho_layout(self):
        import numpy as np
        n = ctypes.c_int()
        _lib.call("cpstep_rho_layout", self._h, 0, ctypes.byref(n), None, None, None)
        kx = np.zeros(n.value, np.int32)
        ky = np.zeros(n.value, np.int32)
        kz = np.zeros(n.value, np.int32)
        ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        _lib.call("cpstep_rho_layout", self._h, n.value, ctypes.byref(n), ip(kx), ip(ky), ip(kz))
        return kx, ky, kz

    def _energies(self):
        return torch.zeros(_lib.NENERGY, dtype=torch.float64, device=self.device)

    def exc(self, rho):
        """CP_exc_calc: (v_xc(r), energies with EXC/MUXC)."""
        self._sync_stream()
        v = torch.empty_like(rho)
        e = self._energies()
        _lib.call("cpstep_exc_calc", self._h, ptr(rho), ptr(v), ptr(e))
        return v, e

    def rho_r2g(self, rho):
        self._sync_stream()
        n = self.rho_layout()[0].shape[0]
        out = torch.empty(n, dtype=torch.complex128, device=self.device)
        _lib.call("cpstep_rho_fft_r2g", self._h, ptr(rho), ptr(out))
        return out

    def hart_eext(self, rhog, forces=True):
        """CP_hart_eext_calc: (vks(G), energies HART/EXT/EWD, forces [natm,3])."""
        self._sync_stream()
        v = torch.empty_like(rhog)
        e = self._energies()
        f = torch.zeros((self.natm, 3), dtype=torch.float64, device=self.device) if forces else None
        _lib.call("cpstep_hart_eext", self._h, ptr(rhog), ptr(v), ptr(e), ptr(f))
        return v, e, f

    def set_local_ees(self, on=True, ngrid=None, n_interp=8, scale=1.2):
        """The EES form of the Hartree/local/Ewald pass (cp_eext_ees_opt): the
        atoms' structure factors interpolated by order-n_interp B-splines on
        an ngrid^3 grid (default: init_eext_ees's size for this layout and
        scale).  on=False returns to the explicit structure factors."""
        if on and ngrid is None:
            ngrid = _lib.lib().cpstep_eext_grid_size(int(self.layout.kmax), float(scale),
                                                     int(n_interp))
        _lib.call("cpstep_set_local_ees", self._h, 1 if on else 0, int(ngrid or 0), int(n_interp))
        return ngrid

    def vks_g2r(self, vksg):
        self._sync_stream()
        out = torch.empty((self.n, self.n, self.n), dtype=torch.float64, device=self.device)
        _lib.call("cpstep_vks_fft_g2r", self._h, ptr(vksg), ptr(out))
        return out

    def vks_from_rho(self, rho, forces=True):
        """XC -> rho(G) -> Hartree/local/Ewald -> V_KS(r); returns (vks, energies, forces)."""
        self._sync_stream()
        v = torch.empty_like(rho)
        e = self._energies()
        f = torch.zeros((self.natm, 3), dtype=torch.float64, device=self.device) if forces else None
        _lib.call("cpstep_vks_from_rho", self._h, ptr(rho), ptr(v), ptr(e), ptr(f))
        return v, e, f

    XC = {"pz_lda": 0, "blyp": 1}

    def set_xc(self, functional="pz_lda", gradient_cutoff=5.0e-5):
        """Exchange-correlation functional of the density side and the step:
        "pz_lda" (default) or "blyp" (Slater exchange + Becke 88 + LYP, the
        reference's cp_becke / cp_lyp options) with its density cut-off."""
        _lib.call("cpstep_set_xc", self._h, self.XC[functional], float(gradient_cutoff))

    def gga_functional(self, rho, gx, gy, gz, vks):
        """CP_getGGAFunctional on given density gradients: returns (vks + df/drho,
        ux, uy, uz, E_GGA) with u = unit(grad rho) df/d|grad rho|."""
        self._sync_stream()
        v = vks.clone()
        ux, uy, uz = gx.clone(), gy.clone(), gz.clone()
        e = self._energies()
        _lib.call("cpstep_gga_functional", self._h, ptr(rho), ptr(ux), ptr(uy), ptr(uz), ptr(v),
                  ptr(e))
        return v, ux, uy, uz, e

    # -- electronic step -----------------------------------------------------
    def set_cp_mass(self, tau_fs=25.0, cut_ry=None):
        """set_cpmass: CP coefficient masses (cut defaults to the state cutoff)."""
        cut = self.layout.ecut_ry if cut_ry is None else cut_ry
        _lib.call("cpstep_set_cp_mass", self._h, float(tau_fs), float(cut))

    def set_cp_thermostat(self, te_ext, tau_fs=25.0, num_nhc=2, nck=1, nres=4, nyosh=9):
        """initCPNHC: the isokinetic NHC thermostat of the coefficients
        (te_ext <= 0 switches it off); defaults as the reference's."""
        _lib.call("cpstep_set_cp_thermostat", self._h, float(te_ext), float(tau_fs), int(num_nhc),
                  int(nck), int(nres), int(nyosh))
        self._nhc_shape = (self.nstates, int(nck), int(num_nhc), 2) if te_ext > 0 else None

    def cp_thermostat_state(self, x=None, xp=None, v=None):
        """Set the chain state from the given arrays [S][nck][num][2] (those not
        None), then return (x, xp, v) as numpy arrays."""
        import numpy as np
        shp = getattr(self, "_nhc_shape", None)
        if shp is None:   # the library reports the thermostat as off
            _lib.call("cpstep_cp_thermostat_state", self._h, 0, None, None, None)
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (x, xp, v)]
        for a in arrs:
            if a is not None and a.shape != shp:
                raise ValueError("chain state must have shape %s" % (shp,))
        self._sync_stream()
        if any(a is not None for a in arrs):
            _lib.call("cpstep_cp_thermostat_state", self._h, 1,
                      *[None if a is None else a.ctypes.data for a in arrs])
        out = [np.zeros(shp) for _ in range(3)]
        _lib.call("cpstep_cp_thermostat_state", self._h, 0, *[a.ctypes.data for a in out])
        return tuple(out)

    def set_atom_thermostat(self, len_nhc, kT=None, mnhc=None, nres=1, nyosh=1):
        """Massive NHC of the atoms (len_nhc 0: NVE); kT [natm], mnhc [natm][len_nhc]."""
        import numpy as np
        if len_nhc <= 0:
            _lib.call("cpstep_set_atom_thermostat", self._h, 0, 1, 1, None, None)
            self._atom_nhc = None
            return
        kT = np.ascontiguousarray(kT, dtype=np.float64)
        mnhc = np.ascontiguousarray(mnhc, dtype=np.float64)
        if mnhc.shape != (kT.shape[0], len_nhc):
            raise ValueError("mnhc must have shape (natm, len_nhc)")
        _lib.call("cpstep_set_atom_thermostat", self._h, int(len_nhc), int(nres), int(nyosh),
                  kT.ctypes.data, mnhc.ctypes.data)
        self._atom_nhc = (kT.shape[0], int(len_nhc))

    def atom_thermostat_state(self, vnhc=None, pos_kt=None):
        """Set the atom chains (vnhc [natm][3][len], pos_kt [natm]; those not None),
        then return (vnhc, pos_kt, (E_kin NHC, pot NHC) of the last step)."""
        import numpy as np
        shp = getattr(self, "_atom_nhc", None)
        if shp is None:
            _lib.call("cpstep_atom_thermostat_state", self._h, 0, None, None, None)
        n, L = shp
        self._sync_stream()
        a = None if vnhc is None else np.ascontiguousarray(vnhc, dtype=np.float64).reshape(n, 3, L)
        b = None if pos_kt is None else np.ascontiguousarray(pos_kt, dtype=np.float64).reshape(n)
        if a is not None or b is not None:
            _lib.call("cpstep_atom_thermostat_state", self._h, 1,
                      None if a is None else a.ctypes.data, None if b is None else b.ctypes.data,
                      None)
        vo, po, eo = np.zeros((n, 3, L)), np.zeros(n), np.zeros(2)
        _lib.call("cpstep_atom_thermostat_state", self._h, 0, vo.ctypes.data, po.ctypes.data,
                  eo.ctypes.data)
        return vo, po, eo

    def cp_integrate(self, force, psi, vpsi, dt, iteration):
        self._sync_stream()
        ke = torch.zeros(1, dtype=torch.float64, device=self.device)
        _lib.call("cpstep_cp_integrate", self._h, ptr(force), ptr(psi), ptr(vpsi), float(dt),
                  int(iteration), ptr(ke))
        return ke

    def cp_step(self, psi, vpsi, occ, dt, iteration, energies=None, atom_force=None):
        """One electronic step in place on psi / vpsi; returns (energies, atom forces)."""
        self._sync_stream()
        self._chk_psi(psi)
        e = self._energies() if energies is None else energies
        f = atom_force
        if f is None:
            f = torch.zeros((self.natm, 3), dtype=torch.float64, device=self.device)
        _lib.call("cpstep_cp_step", self._h, ptr(psi), ptr(vpsi), ptr(occ), float(dt),
                  int(iteration), ptr(e), ptr(f))
        return e, f

    def set_constraint(self, form="ortho_t", tol_norb=0.003):
        """The step's orthonormality constraint: "ortho_t" (the reference's CP
        dynamics: non-orthogonal coefficients and orthoT carried between
        steps, PsiV reset when max|S-2I| >= tol_norb) or "lowdin"."""
        f = {"ortho_t": _lib.CONSTRAINT_ORTHO_T, "lowdin": _lib.CONSTRAINT_LOWDIN}[form]
        _lib.call("cpstep_set_constraint", self._h, f, float(tol_norb))

    def dyn_state(self, psi_no=None, tmat=None, half_step=1):
        """Load (psi_no and tmat given) or read the carried state of the orthoT
        form: (psi_no, tmat, half_step) with half_step the reference's
        halfStepEvolve (0 right after a PsiV reset)."""
        self._sync_stream()
        if psi_no is not None or tmat is not None:
            tcm = tmat.t().contiguous()  # column-major for the C ABI
            h = ctypes.c_int(int(half_step))
            _lib.call("cpstep_dyn_state", self._h, 1, ptr(psi_no), ptr(tcm), ctypes.byref(h))
            torch.cuda.synchronize(self.device)
            return psi_no, tmat, int(half_step)
        p = torch.empty((self.nstates, self.layout.npts), dtype=torch.complex128,
                        device=self.device)
        t = torch.empty((self.nstates, self.nstates), dtype=torch.float64, device=self.device)
        h = ctypes.c_int()
        _lib.call("cpstep_dyn_state", self._h, 0, ptr(p), ptr(t), ctypes.byref(h))
        torch.cuda.synchronize(self.device)
        return p, t.t().contiguous(), h.value

    def dyn_status(self):
        """(max |S - 2I| of the last step's check, PsiV resets so far)."""
        d, r = ctypes.c_double(), ctypes.c_int()
        _lib.call("cpstep_dyn_status", self._h, ctypes.byref(d), ctypes.byref(r))
        return d.value, r.value

    def set_gemm_path(self, tensor_cores):
        """Mixed contexts: overlap / back-multiply on the tensor cores (split BF16) or in FP64."""
        _lib.call("cpstep_set_gemm_path", self._h, 1 if tensor_cores else 0)

    TUNE_NAMES = ("plane_shfl", "plane_waves", "nl_blocks", "pc_split", "tensor_cores",
                  "ees_gspace")

    def tune_get(self):
        v = (ctypes.c_int * 6)()
        _lib.call("cpstep_tune_get", self._h, v, 6)
        return dict(zip(self.TUNE_NAMES, list(v)))

    def tune_set(self, choices):
        cur = self.tune_get()
        cur.update(choices)
        v = (ctypes.c_int * 6)(*[int(cur[k]) for k in self.TUNE_NAMES])
        _lib.call("cpstep_tune_set", self._h, v, 6)

    def autotune(self, psi, occ):
        """Time the launch choices on psi/occ and keep the fastest; returns
        (choices, best ms per choice)."""
        self._sync_stream()
        ms = (ctypes.c_double * 6)()
        _lib.call("cpstep_autotune", self._h, ptr(psi), ptr(occ), ms)
        return self.tune_get(), dict(zip(self.TUNE_NAMES, list(ms)))

    def set_graph(self, enable):
        """Capture / replay cp_step as a CUDA graph (iteration > 1; default on)."""
        _lib.call("cpstep_ctx_set_graph", self._h, 1 if enable else 0)

    def graph_status(self):
        """(enabled, captured, kernels per replay)."""
        en, cap, k = ctypes.c_int(), ctypes.c_int(), ctypes.c_ulonglong()
        _lib.call("cpstep_ctx_graph_status", self._h, ctypes.byref(en), ctypes.byref(cap),
                  ctypes.byref(k))
        return bool(en.value), bool(cap.value), int(k.value)

    def device_errors(self):
        """Error bits recorded by kernels since the last call (0: none); clears them."""
        f = ctypes.c_int()
        _lib.call("cpstep_device_errors", self._h, ctypes.byref(f))
        return f.value

    def step_status(self):
        it, ok = ctypes.c_int(), ctypes.c_int()
        _lib.call("cpstep_step_status", self._h, ctypes.byref(it), ctypes.byref(ok))
        return it.value, bool(ok.value)

#!/usr/bin/env python
"""Benchmark: CP electronic steps per second on one B200, mixed precision vs the
plain FP64 path, on the 192-atom water-like system (64 O + 128 H, L = 23.5 bohr,
128 states, Ecut 70 Ry, 128^3 grid).  Synthetic seeded inputs of that shape.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Our arm prints one JSON line: value = mixed-precision steps/s (whole job, all
ranks; ranks are independent replicas), the FP64 path's steps/s beside it,
e2e through the C-ABI host-buffer call (positions in, energies and atom forces
out every step), the roofline of the state FFT / density / V.psi kernels, the
CPU baseline (two whole FP64 oracle steps on the host cores), clocks and the
number of library kernel launches in the timed region.
The reference arm (--impl reference) times whole steps of the FP64 CPU oracle
of the same system on the host cores (the reference itself cannot be built
here: no Charm++, FFTW-2, BLAS or Fortran in the image); it builds its inputs
with the oracle alone and loads nothing of the product.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "CP steps/sec, mixed vs FP64-plain on one GPU, at <=1e-6 Ha/atom energy error"
CONFIGS = {
    # name: box (bohr), Ecut (Ry), states, atoms, grid
    "water192": dict(box=23.5, ecut=70.0, nstates=128, atoms={"O": 64, "H": 128}, grid=128),
    "water24": dict(box=12.0, ecut=30.0, nstates=32, atoms={"O": 8, "H": 16}, grid=48),
    "water768": dict(box=37.2, ecut=70.0, nstates=1024, atoms={"O": 256, "H": 512}, grid=200),
}
DT = 5.0          # a.u.
TAU_FS = 25.0     # CP mass parameter
CP_FICT_KE = 1000.0  # K: isokinetic NHC of the coefficients (cp_fict_KE default; the
                     # reference's CP dynamics always runs it, ISOKIN_OPT = 1)
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
# DRAM bytes (read + write) of the FFT / density / V.psi kernels of one step
# (K1, K2 and its reduction, K3, K4: phases 0 + 2), from one ncu capture of the
# mixed path at the workload's size; filled from the capture summarised in
# profiles/ (name, source)
TRAFFIC = {("water192", "mixed"): (1.383e9, "profiles/state_fft_traffic_water192_128states.md")}


def workload_name(name, cfg):
    return ("CP electronic step, %d atoms (%d O, %d H), L=%g bohr, %d states, Ecut=%g Ry, grid %d^3"
            % (sum(cfg["atoms"].values()), cfg["atoms"]["O"], cfg["atoms"]["H"], cfg["box"],
               cfg["nstates"], cfg["ecut"], cfg["grid"]))


def peaks():
    try:
        with open(PEAKS) as f:
            p = json.load(f)
        return p.get("hbm_gbs", 6650.0), "measured", p
    except Exception:
        return 6650.0, "fallback", {}


# ---------------------------------------------------------------------------
# distributed plumbing (replicas: each rank runs its own system)

def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return 0, 1, None
    import datetime
    import torch
    import torch.distributed as dist
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return rank, ws, dist


def max_over_ranks(x, dist):
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


# ---------------------------------------------------------------------------
# clocks during the timed region

class Clocks:
    def __init__(self):
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + q, "--format=csv,noheader,nounits", "-lms", "50",
                 "-i", os.environ.get("LOCAL_RANK", "0")],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def mark(self):
        """Samples from here on belong to the timed region."""
        try:
            with open(self.path) as f:
                self.skip = max(0, sum(1 for _ in f) - 1)  # keep the latest sample before
        except Exception:
            self.skip = 0

    def ready(self, timeout=5.0):
        """Wait until the sampler has written its first line (it starts slowly)."""
        t0 = time.time()
        while self.proc is not None and time.time() - t0 < timeout:
            try:
                if os.path.getsize(self.path) > 0:
                    return
            except OSError:
                return
            time.sleep(0.05)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for k, line in enumerate(open(self.path)):
                if k < getattr(self, "skip", 0):
                    continue
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    smax = max(smax, float(f[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        except Exception:
            pass
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# traffic / flop models of one step (per launch of each phase group)

def models(cfg, lay, nlines, nlines_d, npts_d, c_bytes):
    S, n = cfg["nstates"], cfg["grid"]
    npw, nl, nr = lay.npts, nlines, n ** 3
    # what this design must move for density (phase 0) + V.psi/kinetic (phase 2):
    # psi read (G->R pass) and re-read (kinetic term), F written: 3 x 16 B per point;
    # z-pencils written, read by the density pass, read again and written by the
    # V.psi pass, read by the inverse z pass: 5 x c per pencil element; rho partials,
    # rho, V in working precision.
    ours = S * (3 * 16 * npw + 5 * nl * n * c_bytes) + nr * (8 * 5 + c_bytes)
    # the survey's model of the reference algorithm (psi(r) stored and re-read)
    survey = S * (2 * npw * c_bytes + 4 * nl * n * c_bytes + 2 * nr * c_bytes // 2) + 2 * nr * 8
    K = 2 * npw
    gemm_flops = 4 * 2.0 * S * S * K  # lambda, psi.lambda, S, psi.T
    return ours, survey, gemm_flops


# ---------------------------------------------------------------------------

def run_ours(args, cfg, name, rank, ws, dist):
    import numpy as np
    import torch
    from openatom_b200 import _lib
    from openatom_b200.context import StepContext
    from openatom_b200.system import System

    dev = torch.device("cuda", torch.cuda.current_device())
    sysm = System(cfg["box"], cfg["ecut"], cfg["nstates"], cfg["atoms"], nfft=cfg["grid"],
                  seed=1234 + rank)
    psi0 = sysm.psi(device=dev)
    occ = torch.ones(sysm.nstates, dtype=torch.float64, device=dev)
    L = _lib.lib()

    def make(prec):
        ctx = StepContext(sysm.layout, sysm.nstates, precision=prec, device=dev)
        ctx.set_atoms(sysm)
        ctx.set_nonlocal(sysm)
        ctx.set_cp_mass(TAU_FS, cfg["ecut"])
        ctx.set_cp_thermostat(CP_FICT_KE)
        ctx.set_constraint("ortho_t", args.norb_tol)
        # launch choices from the project's autotuner (timed on this system);
        # profiler runs keep the defaults (a profiler distorts the timing)
        choice = ctx.autotune(psi0, occ)[0] if not args.no_autotune else ctx.tune_get()
        out.setdefault("tune", {})[prec] = choice
        return ctx

    out = {}
    e_ref = f_ref = None
    for prec in ("fp64", "mixed"):
        ctx = make(prec)
        psi = psi0.clone()
        v = torch.zeros_like(psi)
        energies = torch.zeros(_lib.NENERGY, dtype=torch.float64, device=dev)
        forces = torch.zeros((sysm.natm, 3), dtype=torch.float64, device=dev)
        # accuracy: first step from the same input, mixed vs FP64
        ctx.cp_step(psi, v, occ, DT, 1, energies, forces)
        it, ok = ctx.step_status()
        first = (energies.cpu().numpy().copy(), forces.cpu().numpy().copy(), ok, it,
                 orthonormality(psi, sysm.layout))
        if prec == "fp64":
            e_ref, f_ref = first[0], first[1]
        clk = Clocks()
        if prec == "mixed":
            clk.start()
        for w in range(args.warmup):
            ctx.cp_step(psi, v, occ, DT, 2 + w, energies, forces)
        torch.cuda.synchronize()
        ctx_prof = prec == "mixed"
        clk.ready()
        barrier(dist)
        torch.cuda.synchronize()
        clk.mark()
        n0 = L.cpstep_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for k in range(args.steps):
            ctx.cp_step(psi, v, occ, DT, 2 + args.warmup + k, energies, forces)
        e1.record()
        torch.cuda.synchronize()
        launches = L.cpstep_launch_count() - n0
        # the same number of steps from the same input in both precisions
        last = (energies.cpu().numpy().copy(), forces.cpu().numpy().copy(),
                1 + args.warmup + args.steps, ctx.dyn_status()[1])
        # the local error after those steps: one step of each precision from
        # the FP64 state (psi, v, the carried constraint state, the chains)
        it_n = 2 + args.warmup + args.steps
        if prec == "fp64":
            snap = dict(psi=psi.clone(), v=v.clone(), dyn=ctx.dyn_state(),
                        nhc=ctx.cp_thermostat_state())
            p1, v1 = snap["psi"].clone(), snap["v"].clone()
            ctx.cp_step(p1, v1, occ, DT, it_n, energies, forces)
            local = (energies.cpu().numpy().copy(), forces.cpu().numpy().copy())
            del p1, v1
        else:
            local = None  # after this context's other runs, below
        clocks = clk.stop() if prec == "mixed" else None
        ms = e0.elapsed_time(e1)
        ms = max_over_ranks(ms, dist)
        barrier(dist)
        graph = ctx.graph_status()
        phase = None
        if ctx_prof:
            # phase breakdown: a separate profiled run (profiled steps run without the graph)
            import ctypes
            _lib.call("cpstep_ctx_profile", ctx._h, 1)
            for k in range(max(3, args.steps // 2)):
                ctx.cp_step(psi, v, occ, DT, 2 + args.warmup + args.steps + k, energies, forces)
            arr = (ctypes.c_double * 7)()
            nst = ctypes.c_int()
            _lib.call("cpstep_phase_times", ctx._h, arr, ctypes.byref(nst))
            phase = [arr[i] / max(1, nst.value) for i in range(7)]
            _lib.call("cpstep_ctx_profile", ctx._h, 0)
        it2, ok2 = ctx.step_status()
        norb_dev, resets = ctx.dyn_status()
        out[prec] = dict(ms=ms, launches=launches, clocks=clocks, phase=phase, first=first,
                         ortho_ok=ok2, ortho_iters=it2, graph=graph, last=last, local=local,
                         psiv_resets=resets, norb_dev_last=norb_dev)
        if prec == "mixed":
            # e2e: the reference-facing host-buffer call (positions in, energies/forces out)
            import ctypes
            pos = torch.from_numpy(np.ascontiguousarray(sysm.pos)).pin_memory()
            he = torch.zeros(_lib.NENERGY, dtype=torch.float64).pin_memory()
            hf = torch.zeros((sysm.natm, 3), dtype=torch.float64).pin_memory()
            it0 = 2 + args.warmup + 2 * args.steps + 3
            for k in range(3):  # the host-buffer call's own direct step and graph capture
                _lib.call("cpstep_cp_step_host", ctx._h, _lib.ptr(psi), _lib.ptr(v), _lib.ptr(occ),
                          DT, it0 + k, ctypes.c_void_p(pos.data_ptr()),
                          ctypes.c_void_p(he.data_ptr()), ctypes.c_void_p(hf.data_ptr()))
            it0 += 3
            barrier(dist)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for k in range(args.steps):
                _lib.call("cpstep_cp_step_host", ctx._h, _lib.ptr(psi), _lib.ptr(v), _lib.ptr(occ),
                          DT, it0 + k, ctypes.c_void_p(pos.data_ptr()),
                          ctypes.c_void_p(he.data_ptr()), ctypes.c_void_p(hf.data_ptr()))
            t1 = time.perf_counter()
            e2e_ms = max_over_ranks((t1 - t0) * 1e3, dist)
            out["e2e"] = dict(ms=e2e_ms, h2d=pos.numel() * 8,
                              d2h=he.numel() * 8 + hf.numel() * 8)
            # the same call with the coefficients owned by the host (the reference's
            # state chares keep psi and v in host memory, stateSlab.C:151-161): psi and
            # v copied in from pinned buffers before and out after every step
            it0 += args.steps
        if prec == "mixed" and psi.numel() * 16 <= (1 << 30):  # pinned copies: 1 GiB each at most
            hp = psi.to("cpu").pin_memory()
            hv = v.to("cpu").pin_memory()
            nh = max(2, min(args.steps, 10))
            barrier(dist)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for k in range(nh):
                psi.copy_(hp, non_blocking=True)
                v.copy_(hv, non_blocking=True)
                _lib.call("cpstep_cp_step_host", ctx._h, _lib.ptr(psi), _lib.ptr(v), _lib.ptr(occ),
                          DT, it0 + k, ctypes.c_void_p(pos.data_ptr()),
                          ctypes.c_void_p(he.data_ptr()), ctypes.c_void_p(hf.data_ptr()))
                hp.copy_(psi, non_blocking=True)
                hv.copy_(v, non_blocking=True)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            cb = 2 * psi.numel() * 16
            out["e2e_host_psi"] = dict(ms=max_over_ranks((t1 - t0) * 1e3, dist), steps=nh,
                                       h2d=cb + pos.numel() * 8,
                                       d2h=cb + he.numel() * 8 + hf.numel() * 8)
            del hp, hv
        if prec == "mixed":
            out["pc_us"] = pc_kernel_times(ctx, psi, v)
        if prec == "mixed":  # the mixed half of the local error (it replaces the carried state)
            ctx.dyn_state(*snap["dyn"])
            ctx.cp_thermostat_state(*snap["nhc"])
            p1, v1 = snap["psi"].clone(), snap["v"].clone()
            ctx.cp_step(p1, v1, occ, DT, it_n, energies, forces)
            out[prec]["local"] = (energies.cpu().numpy().copy(), forces.cpu().numpy().copy())
            del p1, v1, snap
        nl, _ = ctx.info()
        out.setdefault("nlines", nl)
        out.setdefault("npts_d", ctx.rho_layout()[0].shape[0])
        ctx.close()
    return sysm, out, e_ref, f_ref


def orthonormality(psi, lay):
    """max |psi^T psi / 2 - I| (the S of the packed half sphere, FP64)."""
    import torch
    w = torch.where(torch.from_numpy(lay.kx).to(psi.device) == 0, 1.0, 2.0).to(torch.float64)
    re, im = psi.real.contiguous(), psi.imag.contiguous()
    S = (re * w) @ re.T + (im * w) @ im.T
    eye = torch.eye(S.shape[0], dtype=torch.float64, device=psi.device)
    return float((S / 2 - eye).abs().max())


def pc_kernel_times(ctx, psi, f, reps=5):
    """Device time (us) of the PairCalc products of the context alone, outside
    the timed step: S = psi^T psi, lambda = psi^T F, psi.T."""
    import torch
    S = psi.shape[0]
    cS = torch.zeros((S, S), dtype=torch.float64, device=psi.device)
    out = torch.empty_like(psi)
    T = torch.eye(S, dtype=torch.float64, device=psi.device) * 1.0001
    res = {}
    for name, fn in (("S", lambda: ctx.pc_overlap(psi, psi, out=cS)),
                     ("lambda", lambda: ctx.pc_overlap(psi, f, out=cS)),
                     ("psiT", lambda: ctx.pc_backmultiply(T, psi, out=out))):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        res[name] = e0.elapsed_time(e1) / reps * 1e3
    return res


def oracle_system(cfg, tol_norb):
    """The benchmark system for the FP64 oracle, built by the oracle alone
    (oracle/synth.py: the product package is not imported and its library is
    not loaded), with the GPU arm's settings: EES non-local (s + p, B-spline
    order 8), the isokinetic NHC of the coefficients (1000 K, 2 chains, nres 4,
    nyosh 9, chains on the isokinetic surface), the orthoT constraint."""
    import numpy as np
    from oracle import density as OD
    from oracle import fftpath as OF
    from oracle import isokin as OK
    from oracle import step as OS
    from oracle import synth as OSY
    OF.set_workers(os.cpu_count() or 1)
    sysm = OSY.System(cfg["box"], cfg["ecut"], cfg["nstates"], cfg["atoms"], nfft=cfg["grid"])
    lay = sysm.layout
    cls, _, _ = OS.point_classes(lay)
    p = OK.init_nhc(int(np.sum(cls != 0)), 1, 2, 1, CP_FICT_KE, TAU_FS)
    psi = sysm.psi()
    return dict(sys=sysm, lay=lay, dlay=OD.density_layout(cfg["box"], cfg["ecut"], cfg["grid"]),
                cmass=OS.cp_mass(lay, TAU_FS, cfg["ecut"]),
                nhc=(p, [OK.default_state(p) for _ in range(sysm.nstates)], 4, 9),
                psi=psi, v=np.zeros_like(psi), dyn=None, occ=np.ones(sysm.nstates),
                tol=tol_norb, it=1)


def oracle_steps(st, n):
    """n whole FP64 oracle steps of the system st (density, V_KS, V.psi, EES,
    lambda, the constraint, the thermostatted Verlet, S, T, psi.T); returns
    the wall seconds of each."""
    from oracle import step as OS
    times = []
    for _ in range(n):
        t0 = time.perf_counter()
        st["psi"], st["v"], _, _, aux = OS.cp_step(
            st["psi"], st["v"], st["occ"], st["sys"], st["lay"], st["dlay"], st["cmass"], DT,
            st["it"], nonlocal_on=True, nhc=st["nhc"], tol_norb=st["tol"], dyn=st["dyn"])
        times.append(time.perf_counter() - t0)
        st["dyn"] = aux["dyn"]
        st["it"] += 1
    return times


def cpu_baseline(cfg, tol_norb):
    """Whole FP64 oracle steps on the host cores: one untimed step, then the
    mean of two (about 10-30 s of CPU work)."""
    st = oracle_system(cfg, tol_norb)
    oracle_steps(st, 1)
    t = oracle_steps(st, 2)
    sample = ("2 whole FP64 oracle steps (iterations 2-3, after 1 untimed) of the same system: "
              "numpy/scipy pocketfft, state chunks on %d host threads" % (os.cpu_count() or 1))
    return sum(t) / len(t), sample


def pc_roofline(us, sysm, hbm, pk, gflops, gemm_ms):
    """S = psi^T psi on the tensor cores: it must read psi once (16 B per
    coefficient); the split products issue 6 BF16 MMAs per FP64 product."""
    S, npw = sysm.nstates, sysm.layout.npts
    t = us["S"] * 1e-6
    byt = 16.0 * S * npw
    bf16 = 6 * 2.0 * S * S * 2 * npw
    peak_tc = pk.get("bf16_tflops") if pk else None
    return {"bound": "hbm", "kernel": "k_pc_tc overlap S = psi^T psi (split BF16, tcgen05)",
            "achieved": byt / t / 1e9, "peak": hbm, "unit": "GB/s", "frac": byt / t / 1e9 / hbm,
            "algorithmic_bytes": byt, "bf16_tflops": bf16 / t / 1e12,
            "bf16_frac": (bf16 / t / 1e12 / peak_tc) if peak_tc else None,
            "kernel_us": us, "phases_tflops_fp64_equiv": gflops / (gemm_ms * 1e-3) / 1e12
            if gemm_ms > 0 else None}


def kernel_case(args):
    """Small single-GPU case of one kernel group, for profiler captures.

    statefft: density + 2 x (V.psi, density) of `--states` states of the
    water192 layout (128^3 grid) in the chosen precision.
    rhoside:  the density-side pass (XC, rho FFT, Hartree/local/Ewald and
    atom forces, V_KS) of the water192 system, run 3 times.
    ees:      the EES non-local pass of `--states` states of the water192
    system (8 s+p channels, 80^3 NL grid), run 2 times.
    paircalc: S = overlap(psi, psi) and psi.T of `--states` states of the
    water192 layout (K = 131,472 reals), run 2 times.
    """
    import torch
    from openatom_b200.context import StepContext
    from openatom_b200.system import System
    cfg = CONFIGS["water192"]
    S = args.states
    sysm = System(cfg["box"], cfg["ecut"], S, cfg["atoms"], nfft=cfg["grid"])
    occ = torch.ones(S, dtype=torch.float64, device="cuda")
    ctx = StepContext(sysm.layout, S, precision=args.precision)
    if args.plane_form is not None:
        ctx.tune_set({"plane_shfl": args.plane_form})
    psi = sysm.psi()
    rho = ctx.density(psi, occ)
    if args.kernel_case == "statefft":
        v = torch.randn(cfg["grid"], cfg["grid"], cfg["grid"], dtype=torch.float64,
                        device="cuda") * 0.1
        for _ in range(2):
            f, e = ctx.vks_psi(psi, v, occ)
            rho = ctx.density(psi, occ)
        chk = float(e.sum())
    elif args.kernel_case == "rhoside":
        ctx.set_atoms(sysm)
        for _ in range(3):
            vks, _, _ = ctx.vks_from_rho(rho)
        chk = float(vks.sum())
    elif args.kernel_case == "ees":
        ctx.set_atoms(sysm)
        ctx.set_nonlocal(sysm)
        for _ in range(2):
            fpsi, e, f = ctx.ees_nonlocal(psi, occ)
        chk = float(e[7])
    else:
        for _ in range(2):
            smat = ctx.pc_overlap(psi, psi)
            out = ctx.pc_backmultiply(smat, psi)
        chk = float(smat.sum()) + float(out.real.sum())
    torch.cuda.synchronize()
    ctx.close()
    print(json.dumps({"kernel_case": args.kernel_case, "states": S,
                      "precision": args.precision, "rho_sum": float(rho.sum()),
                      "check": chk}))


def batch16_systems(seed=4):
    """16 water-like systems: states in [16, 256], grids from {32, 48, 64, 96},
    Ecut in [30, 70] Ry, the box chosen so that the grid rule lands on the
    grid (for 32, which the FFT size table skips, the largest box whose grid is
    smaller, with the grid set to 32), water at liquid density (1 molecule per
    200 bohr^3)."""
    import ctypes
    import numpy as np
    from openatom_b200 import _lib
    L = _lib.lib()

    def nfft(box, ec):
        k, n, nk, npts = (ctypes.c_int() for _ in range(4))
        L.cpstep_layout_sizes(float(box), float(ec), ctypes.byref(k), ctypes.byref(n),
                              ctypes.byref(nk), ctypes.byref(npts))
        return n.value

    rng = np.random.default_rng(seed)
    out = []
    for i in range(16):
        grid = int(rng.choice([32, 48, 64, 96]))
        ec = float(rng.uniform(30.0, 70.0))
        S = int(rng.integers(16, 257))
        box = None
        last_below = None
        for b in np.arange(5.0, 60.0, 0.05):
            n = nfft(b, ec)
            if n == grid:
                box = float(b)
                break
            if n < grid:
                last_below = float(b)
        if box is None:
            box = last_below
        nw = max(1, int(round(box ** 3 / 200.0)))
        out.append(dict(box=round(box, 2), ecut=ec, nstates=S, grid=grid,
                        atoms={"O": nw, "H": 2 * nw}))
    return out


def batch16_measure(args):
    """Config 4: 16 independent systems (seeded states in [16, 256], grids from
    {32, 48, 64, 96}, 30-70 Ry), mixed precision, stepped as one batch graph,
    against looping the single-system path over them in the plain FP64 path
    and in the mixed path, both loops with their own step graphs.  Returns the
    aggregate system-steps/s of the three."""
    import numpy as np
    import torch
    from openatom_b200 import _lib
    from openatom_b200.batch import StepBatch
    from openatom_b200.context import StepContext
    from openatom_b200.system import System
    specs = batch16_systems()
    L = _lib.lib()
    systems = []
    for k, sp in enumerate(specs):
        sysm = System(sp["box"], sp["ecut"], sp["nstates"], sp["atoms"], nfft=sp["grid"],
                      seed=300 + k)
        systems.append(sysm)

    def contexts(prec, graph):
        out = []
        for sysm, sp in zip(systems, specs):
            ctx = StepContext(sysm.layout, sysm.nstates, precision=prec)
            ctx.set_atoms(sysm)
            ctx.set_nonlocal(sysm)
            ctx.set_cp_mass(TAU_FS, sp["ecut"])
            ctx.set_cp_thermostat(CP_FICT_KE)
            ctx.set_constraint("ortho_t", args.norb_tol)
            ctx.set_graph(graph)
            psi = sysm.psi()
            out.append(dict(ctx=ctx, psi=psi, v=torch.zeros_like(psi),
                            occ=torch.ones(sysm.nstates, dtype=torch.float64, device="cuda"),
                            e=torch.zeros(_lib.NENERGY, dtype=torch.float64, device="cuda"),
                            f=torch.zeros((sysm.natm, 3), dtype=torch.float64, device="cuda")))
        return out

    def timed(fn, nsteps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for k in range(nsteps):
            fn(k)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    # batched graph, mixed (the contexts' own graphs off: the batch holds one)
    mix = contexts("mixed", False)
    batch = StepBatch([d["ctx"] for d in mix])
    arg = lambda key: [d[key] for d in mix]
    for w in range(args.warmup):
        batch.step(arg("psi"), arg("v"), arg("occ"), DT, 1 + w, arg("e"), arg("f"))
    n0 = L.cpstep_launch_count()
    ms_batch = timed(lambda k: batch.step(arg("psi"), arg("v"), arg("occ"), DT,
                                          1 + args.warmup + k, arg("e"), arg("f")), args.steps)
    launches = L.cpstep_launch_count() - n0
    status = batch.status()
    e_mix = [d["e"].cpu().numpy().copy() for d in mix]
    batch.close()
    for d in mix:
        d["ctx"].close()

    def looped(prec):
        """the single-system step looped over the systems, each with its graph"""
        pl = contexts(prec, True)

        def loop(k):
            for d in pl:
                d["ctx"].cp_step(d["psi"], d["v"], d["occ"], DT, 1 + args.warmup + k, d["e"],
                                 d["f"])
        for w in range(args.warmup):
            for d in pl:
                d["ctx"].cp_step(d["psi"], d["v"], d["occ"], DT, 1 + w, d["e"], d["f"])
        ms = timed(loop, args.steps)
        graphs = all(d["ctx"].graph_status()[1] for d in pl)
        for d in pl:
            d["ctx"].close()
        return ms, graphs
    ms_loop, g64 = looped("fp64")
    ms_mloop, gmx = looped("mixed")
    nsys = len(specs)
    v_batch = nsys * args.steps / (ms_batch / 1e3)
    v_loop = nsys * args.steps / (ms_loop / 1e3)
    v_mloop = nsys * args.steps / (ms_mloop / 1e3)
    return {
        "metric": "aggregate CP steps/sec of 16 independent systems on one GPU",
        "value": v_batch, "unit": "system-steps/s", "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_batch / args.steps,
        "workload": "16 water-like systems, states %s, grids %s" % (
            [sp["nstates"] for sp in specs], [sp["grid"] for sp in specs]),
        "systems": specs, "parallelism": "one batch graph, a branch per system",
        "plain_fp64_loop_value": v_loop, "batched_over_plain_loop": v_batch / v_loop,
        "mixed_loop_value": v_mloop, "batched_over_mixed_loop": v_batch / v_mloop,
        "loops_graphed": bool(g64 and gmx),
        "gpu_launches": int(launches), "batch_graph": {"enabled": status[0],
                                                      "captured": status[1],
                                                      "kernels_per_step": status[2]},
        "energies_finite": bool(all(np.isfinite(e).all() for e in e_mix)),
    }


def run_batch16(args):
    r = batch16_measure(args)
    line = {"metric": r["metric"], "value": r["value"], "unit": r["unit"], "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "mixed (as the single-system line)", "data": "synthetic",
            "config": {"workload": r["workload"], "systems": r["systems"],
                       "parallelism": r["parallelism"]}}
    line.update({k: r[k] for k in ("plain_fp64_loop_value", "batched_over_plain_loop",
                                   "mixed_loop_value", "batched_over_mixed_loop",
                                   "loops_graphed", "gpu_launches", "batch_graph",
                                   "energies_finite")})
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="water192", choices=sorted(CONFIGS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch16", action="store_true",
                    help="leave out the 16-system batch measurement of the main line")
    ap.add_argument("--norb-tol", type=float, default=0.05,
                    help="cp_norb_tol of the orthoT constraint (reference default 0.003; the "
                         "random, unquenched start needs more on its first step)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default launch choices (for profiler runs)")
    ap.add_argument("--kernel-case", choices=["statefft", "rhoside", "ees", "paircalc"], default=None,
                    help="run a small profiling case instead of the benchmark")
    ap.add_argument("--states", type=int, default=8)
    ap.add_argument("--plane-form", type=int, choices=[0, 1, 2], default=None,
                    help="kernel cases: the plane-pass form (0 Stockham, 1 shuffles, 2 two-stage)")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--batch16", action="store_true",
                    help="16 independent systems of uneven size stepped by one batch graph "
                         "(mixed) against looping the plain FP64 path")
    args = ap.parse_args()
    if args.kernel_case:
        kernel_case(args)
        return
    if args.batch16:
        if args.warmup < 3:
            args.warmup = 3
        run_batch16(args)
        return
    if args.warmup < 3:
        args.warmup = 3
    cfg = CONFIGS[args.config]
    wname = workload_name(args.config, cfg)

    if args.impl == "reference":
        # rank 0 alone times the reference's CPU path (the FP64 oracle port);
        # no process group, no GPU, nothing of the product is loaded
        if int(os.environ.get("RANK", "0")) != 0:
            return
        ncpu = os.cpu_count() or 1
        st = oracle_system(cfg, args.norb_tol)
        oracle_steps(st, args.warmup)
        times = oracle_steps(st, args.steps)
        t = statistics.mean(times)
        line = {
            "impl": "reference", "metric": METRIC, "value": 1.0 / t, "unit": "steps/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wname, "precision": "FP64 CPU oracle (the reference's "
                       "algorithm restated; the reference needs Charm++ and FFTW-2)",
                       "parallelism": "host cores", "dt_au": DT,
                       "cp_thermostat": "isokinetic NHC, %g K, 2 chains, nres 4, nyosh 9"
                       % CP_FICT_KE,
                       "constraint": "orthoT (the reference's CP dynamics), cp_norb_tol %g"
                       % args.norb_tol},
            "step_seconds": times,
            "cpu_baseline": {"value": 1.0 / t, "unit": "steps/s", "cores": ncpu, "kind": "port",
                             "sample": "%d whole FP64 oracle steps after %d untimed, "
                                       "numpy/scipy pocketfft, state chunks on %d host threads"
                                       % (args.steps, args.warmup, ncpu)},
            "e2e": {"value": 1.0 / t, "unit": "steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
        return

    rank, ws, dist = dist_init()
    sysm, out, e_ref, f_ref = run_ours(args, cfg, args.config, rank, ws, dist)
    import numpy as np
    mixed, fp64 = out["mixed"], out["fp64"]
    sps_mixed = ws * args.steps / (mixed["ms"] / 1e3)
    sps_fp64 = ws * args.steps / (fp64["ms"] / 1e3)
    e_mix, f_mix = mixed["first"][0], mixed["first"][1]
    err_e = abs(e_mix[8] - e_ref[8]) / sysm.natm
    err_f = float(np.max(np.abs(f_mix - f_ref)))
    hbm, peak_kind, pk = peaks()
    c_bytes = 8  # FP32 complex in the mixed path
    ours_b, survey_b, gflops = models(cfg, sysm.layout, out["nlines"], None, out["npts_d"], c_bytes)
    ph = mixed["phase"] or [0.0] * 7
    fft_ms = ph[0] + ph[2]
    # algorithmic bytes: the per-step model of the plane-wave FFT / density /
    # V.psi path (psi(r) stored once and re-read, two-pass pencil transforms);
    # this design recomputes psi(r) instead of storing it and moves ours_b
    achieved = survey_b / (fft_ms * 1e-3) / 1e9 if fft_ms > 0 else None
    achieved_ours = ours_b / (fft_ms * 1e-3) / 1e9 if fft_ms > 0 else None
    traffic = TRAFFIC.get((args.config, "mixed"))
    gemm_ms = ph[3] + ph[5]
    if rank != 0:
        return
    line = {
        "metric": METRIC,
        "value": sps_mixed,
        "unit": "steps/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": mixed["ms"] / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 FFT/density/V.psi with f64 rho/energy accumulation; PairCalc split-BF16 "
                 "tensor-core products (FP32 accumulate, FP64 sums); Ortho f32 + f64 correction",
        "data": "synthetic",
        "config": {"workload": wname, "parallelism": "replicas" if ws > 1 else "1 GPU",
                   "inputs_vs_L2": "inputs larger than L2: psi %.1f MB FP64 per replica"
                   % (sysm.nstates * sysm.layout.npts * 16 / 1e6),
                   "precision": "mixed", "dt_au": DT,
                   "cp_thermostat": "isokinetic NHC, %g K, 2 chains, nres 4, nyosh 9" % CP_FICT_KE,
                   "constraint": "orthoT (the reference's CP dynamics), cp_norb_tol %g"
                   % args.norb_tol},
        "psiv_resets": {"mixed": mixed["psiv_resets"], "fp64": fp64["psiv_resets"],
                        "norb_dev_last_mixed": mixed["norb_dev_last"]},
        "fp64_steps_per_sec": sps_fp64,
        "fp64_ms_per_step": fp64["ms"] / args.steps,
        "mixed_over_fp64": sps_mixed / sps_fp64,
        "accuracy_vs_fp64": {"energy_Ha_per_atom": err_e, "local_force_Ha_per_bohr": err_f,
                             "orthonormality_mixed": mixed["first"][4],
                             "orthonormality_fp64": fp64["first"][4],
                             "ortho_converged": bool(mixed["ortho_ok"]),
                             "after_steps": mixed["last"][2],
                             "energy_Ha_per_atom_after": abs(mixed["last"][0][8] -
                                                             fp64["last"][0][8]) / sysm.natm,
                             "local_force_Ha_per_bohr_after": float(np.max(np.abs(
                                 mixed["last"][1] - fp64["last"][1]))),
                             "psiv_resets_mixed_fp64": [mixed["last"][3], fp64["last"][3]],
                             "one_step_from_the_fp64_state_after": mixed["last"][2],
                             "energy_Ha_per_atom_one_step": abs(mixed["local"][0][8] -
                                                                fp64["local"][0][8]) / sysm.natm,
                             "local_force_Ha_per_bohr_one_step": float(np.max(np.abs(
                                 mixed["local"][1] - fp64["local"][1])))},
        "phase_ms_mixed": {"density": ph[0], "vks": ph[1], "vpsi_kinetic": ph[2],
                           "lambda": ph[3], "integrate": ph[4], "ortho_psiT": ph[5],
                           "ees_nonlocal": ph[6]},
        "roofline": {"bound": "hbm", "kernel": "state FFT + density + V.psi (phases 0+2)",
                     "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": (achieved / hbm) if achieved else None,
                     "traffic": traffic[0] if traffic else None,
                     "traffic_source": traffic[1] if traffic else None,
                     "algorithmic_bytes": survey_b, "peak_kind": peak_kind,
                     "this_design_bytes": ours_b, "this_design_achieved": achieved_ours,
                     "this_design_frac": (achieved_ours / hbm) if achieved_ours else None},
        "roofline_paircalc": pc_roofline(out["pc_us"], sysm, hbm, pk, gflops, gemm_ms),
        "gpu_launches": int(mixed["launches"]),
        "autotune": out.get("tune"),
        "cuda_graph": {"mixed": mixed["graph"], "fp64": fp64["graph"],
                       "fields": ["enabled", "captured", "kernels_per_step"]},
        "clocks": mixed["clocks"],
        "e2e": {"value": ws * args.steps / (out["e2e"]["ms"] / 1e3), "unit": "steps/s",
                "h2d_bytes_per_step": out["e2e"]["h2d"], "d2h_bytes_per_step": out["e2e"]["d2h"]},
    }
    if "e2e_host_psi" in out:
        eh = out["e2e_host_psi"]
        line["e2e_host_psi"] = {
            "value": ws * eh["steps"] / (eh["ms"] / 1e3), "unit": "steps/s", "steps": eh["steps"],
            "h2d_bytes_per_step": eh["h2d"], "d2h_bytes_per_step": eh["d2h"],
            "note": "psi and v in host memory: copied in before and out after every step"}
    if ws == 1 and not args.no_batch16:
        b = batch16_measure(args)
        line["batch16"] = {k: b[k] for k in ("value", "unit", "workload", "plain_fp64_loop_value",
                                             "batched_over_plain_loop", "mixed_loop_value",
                                             "batched_over_mixed_loop", "loops_graphed",
                                             "batch_graph", "energies_finite")}
    if ws == 1 and not args.no_cpu_baseline:
        t, sample = cpu_baseline(cfg, args.norb_tol)
        line["cpu_baseline"] = {"value": 1.0 / t, "unit": "steps/s", "cores": os.cpu_count() or 1,
                                "kind": "port", "sample": sample}
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""Benchmark of the B200 ChFSI path (one JSON line on rank 0).

Workload: the 64-atom Kleinman-Bylander cell (a = 20.52 bohr, Ecut 20 Ha,
37,073 plane waves, 72^3 grid, 160 bands, 256 projectors, seed 0) in FP64.
A step is one ChFSI iteration as the reference's diagonalize runs it: a
degree-16 Chebyshev filter (17 H|psi> applies per band incl. the final one
for Rayleigh-Ritz) followed by Rayleigh-Ritz.  Metric: H|psi> band-applies
per second (n_bands x 17 per step).

At N = 1 the line also carries the time-to-SCF of the 216-atom ultrasoft
cell (n_pw 173,925, 576 bands, 1,728 projectors, 108^3 / 144^3 grids):
FP64 + Pulay, mixed precision + Pulay and mixed precision + the learned
mixer, each stopped at |dE| < 1e-6 Ha/atom with the occupied eigenvalues
changing by less than 1e-6 Ha between FP64 iterations, and each compared
with the FP64 run continued (untimed) for further iterations toward tight
convergence (about nine minutes), and the batched pass of 96 members (64
k-points of the 8-atom cell and 32 cells of 8-64 atoms) as one CUDA graph
against member by member.  --no-scf-216 and --no-batch skip those blocks; a
block that fails reports its error in the line instead of losing it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's algorithm on the host CPU (the C++
oracle restatement; the reference crate itself cannot be built here) on the
same step: the degree-16 filter of one band per host thread (scaled by the
per-band cost to all 160 bands) plus the Rayleigh-Ritz of all 160 bands.
It loads only the oracle library (the inputs come from the oracle's copy of
the seeded generator).
For N > 1 (torchrun) every rank runs an independent replica of the workload
(weak scaling, no collective on the data path); the value is the total over
ranks divided by the slowest rank's time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "chemrust-scf_b200"))

NDEG = 16
CONFIG_INDEX = 1
METRIC = "H|psi> band-applies/s (ChFSI iteration: degree-16 Chebyshev filter + Rayleigh-Ritz)"
UNIT = "band-applies/s"
# DRAM bytes (read + write) per band of one local H|psi> launch (the three
# FFT-pass kernels, 160 bands: 1,151,111,424 bytes), from an ncu capture of
# dram__bytes_read.sum + dram__bytes_write.sum of those kernels
TRAFFIC_PER_BAND = 1151111424 / 160


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "fallback": True}


def bench_config(s, world):
    """The workload description shared by both arms (identical dicts)."""
    return {"workload": "64-atom KB-projector cell, a=20.52 bohr, Ecut 20 Ha, n_pw=%d, grid "
                        "72^3, 160 bands, 256 projectors, degree 16, FP64" % s.n_pw,
            "n_pw": s.n_pw, "n_bands": s.n_bands, "ndeg": NDEG, "grid": list(s.ngrid),
            "n_proj": s.n_proj, "parallelism": "replicas" if world > 1 else "single",
            "l2": "working set (psi 95 MB + beta 152 MB + sticks 250 MB) exceeds the 126 MB L2"}


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.3)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        mhz, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                mhz.append(float(f[0]))
                mx = max(mx, float(f[1]))
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(mhz)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def run_ours(args):
    import numpy as np
    import torch
    import chfsi

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    s = chfsi.SyntheticSystem(config_index=CONFIG_INDEX, seed=rank)
    ctx = chfsi.Context(s, device=local)
    # V_eff of the first SCF step: V_loc + V_H + V_xc of the uniform density
    rho0 = np.full(s.ng, s.n_elec / s.omega)
    ctx.build_v_eff(rho0)
    # launch configuration of the FFT passes picked by the library's autotuner
    # (untimed; times the local H|psi> on this context's own psi)
    tune_choice, _ = ctx.autotune()
    psi0 = s.psi0()
    stream = torch.cuda.ExternalStream(ctx.stream(), device=local)
    nb = s.n_bands
    applies_per_step = nb * (NDEG + 1)

    # ---- device-resident timing: inputs already in HBM ---------------------
    eig = ctx.diagonalize(NDEG)  # first step from the random start (untimed)
    for _ in range(args.warmup):
        eig = ctx.diagonalize(NDEG, eig)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = chfsi.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            eig = ctx.diagonalize(NDEG, eig)
        ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    launches = (chfsi.launch_count() - launches0) // max(1, args.steps)
    ms = ev0.elapsed_time(ev1)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    ms_step = ms / args.steps
    value = applies_per_step * args.steps * world / (ms * 1e-3)

    # ---- roofline of the dominant kernel group: local H|psi> (3 FFT passes) -
    x = torch.from_numpy(psi0).to(f"cuda:{local}")
    y = torch.empty_like(x)
    torch.cuda.synchronize()
    for _ in range(3):
        ctx.apply_h_local(x.data_ptr(), y.data_ptr(), nb)
    reps = 10
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        ctx.apply_h_local(x.data_ptr(), y.data_ptr(), nb)
    e1.record(stream)
    e1.synchronize()
    t_loc = e0.elapsed_time(e1) / reps * 1e-3
    ncol, nz = s.info.n_columns, s.ngrid[2]
    n3 = s.ngrid[0] * s.ngrid[1] * s.ngrid[2]
    # algorithmic bytes of one band-apply of local H|psi> for the fused 3-pass
    # FFT: grid written, read+written, read (4 N^3) plus psi_k, psi_{k-1} in
    # and psi_{k+1} out (3 n_pw), complex128
    bytes_per_band = 16 * (4 * n3 + 3 * s.n_pw)
    algo_bytes = bytes_per_band * nb
    # what this pruned design itself moves: only the (x, y) columns that hold
    # plane waves are stored between the passes
    pruned_bytes = 16 * (4 * ncol * nz + 4 * s.n_pw) * nb
    pk = peaks()
    achieved = algo_bytes / t_loc / 1e9
    roofline = {"kernel": "local H|psi> (z-sticks inverse, xy-planes x V, z-sticks forward)",
                "bound": "hbm", "achieved": round(achieved, 1), "peak": pk["hbm_gbs"],
                "unit": "GB/s", "frac": round(achieved / pk["hbm_gbs"], 4),
                "traffic": TRAFFIC_PER_BAND * nb if TRAFFIC_PER_BAND else None,
                "algorithmic_bytes_per_launch": algo_bytes,
                "pruned_design_bytes_per_launch": pruned_bytes,
                "launch_ms": round(t_loc * 1e3, 4),
                "peak_source": "measured" if not pk.get("fallback") else "fallback"}

    # ---- end to end through the C ABI with pinned host buffers -------------
    host_in = torch.from_numpy(psi0.copy()).pin_memory()
    host_out = torch.empty_like(host_in).pin_memory()
    hin, hout = host_in.numpy(), host_out.numpy()
    for _ in range(2):
        ctx.set_psi(hin)
        eig = ctx.diagonalize(NDEG, eig)
        _get_psi_into(ctx, hout)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        ctx.set_psi(hin)
        eig = ctx.diagonalize(NDEG, eig)
        _get_psi_into(ctx, hout)
    t1.record(stream)
    t1.synchronize()
    ms_e2e = t0.elapsed_time(t1)
    if dist:
        t = torch.tensor([ms_e2e], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    e2e_value = applies_per_step * args.steps * world / (ms_e2e * 1e-3)
    psi_bytes = psi0.nbytes
    e2e = {"value": round(e2e_value, 1), "unit": UNIT, "h2d_bytes_per_step": psi_bytes,
           "d2h_bytes_per_step": psi_bytes + 8 * nb,
           "api": "chfsi_set_psi + chfsi_diagonalize + chfsi_get_psi (pinned host buffers)"}

    # ---- mixed precision: FP32 filter (tcgen05 BF16x3 projector GEMMs), FP64 Rayleigh-Ritz
    mixed = None
    if not args.fp64_only:
        mctx = chfsi.Context(s, device=local, precision=chfsi.PREC_MIXED)
        mctx.build_v_eff(rho0)
        mctx.autotune()
        mstream = torch.cuda.ExternalStream(mctx.stream(), device=local)
        meig = mctx.diagonalize(NDEG)
        for _ in range(args.warmup):
            meig = mctx.diagonalize(NDEG, meig)
        torch.cuda.synchronize()
        m0 = torch.cuda.Event(enable_timing=True)
        m1 = torch.cuda.Event(enable_timing=True)
        m0.record(mstream)
        for _ in range(args.steps):
            meig = mctx.diagonalize(NDEG, meig)
        m1.record(mstream)
        m1.synchronize()
        mms = m0.elapsed_time(m1)
        if dist:
            t = torch.tensor([mms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            mms = float(t.item())
        mixed = {"value": round(applies_per_step * args.steps * world / (mms * 1e-3), 1),
                 "unit": UNIT, "ms_per_step": round(mms / args.steps, 3),
                 "dtype": "f32 filter (bf16x3 tcgen05 projector GEMMs, fp32 accumulate), f64 Rayleigh-Ritz"}
        mctx.close()
        if not args.no_scf and world == 1:
            import learned_mixer
            net = learned_mixer.load(device=local)
            mixed["time_to_scf"] = guarded(time_to_scf, chfsi, s, NDEG, local, net, max_iter=100,
                                           tight_max_iter=40, cell="64")

    # ---- headline: time-to-SCF of the 216-atom ultrasoft cell (N = 1 only) ----
    scf216 = None
    if world == 1 and not args.no_scf and not args.no_scf_216:
        import learned_mixer
        s2 = chfsi.SyntheticSystem(config_index=2)
        net = learned_mixer.load(device=local)
        scf216 = guarded(time_to_scf, chfsi, s2, 16, local, net, max_iter=args.scf_216_max_iter,
                         tight_max_iter=20, cell="216")
        scf216["workload"] = ("216-atom ultrasoft cell, a=30.78 bohr, Ecut 25 Ha, n_pw=%d, "
                              "grid 108^3 (density 144^3), %d bands, %d projectors, degree 16"
                              % (s2.n_pw, s2.n_bands, s2.n_proj))
        del s2

    batched = None
    if world == 1 and not args.no_batch:
        batched = guarded(batched_passes, chfsi, local)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = guarded(cpu_baseline, steps=2)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded 64-atom diamond cell; per-rank replica)",
            "config": bench_config(s, world),
            "launch_config": int(tune_choice),
            "clocks": clk.summary(),
            "e2e": e2e,
            "gpu_launches": int(launches),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "mixed_precision": mixed,
            "time_to_scf_216atom": scf216,
            "batched": batched,
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    ctx.close()


def guarded(fn, *a, **kw):
    """Run one of the line's optional blocks (single-process only); a failure
    is reported in the block instead of losing the whole JSON line."""
    try:
        return fn(*a, **kw)
    except Exception as e:  # the headline value and e2e are already measured
        import traceback
        traceback.print_exc()
        return {"error": "%s: %s" % (type(e).__name__, e)}


# time-to-SCF stopping rule of every timed arm, and the tight FP64 reference
SCF_TOL_PER_ATOM = 1e-6   # |dE| per atom (Ha)
# largest change of the occupied eigenvalues between FP64 iterations (Ha);
# the mixed arms switch to FP64 once two mixed iterations change them by less
# than twice this.  Their FP32 passes run the residual form (R-ChFSI), whose
# rounding falls with the Ritz residuals: with the plain FP32 filter the
# 216-atom cell's mixed iterations level off at changes of 1-3e-6 Ha and the
# FP64 iterations then need ~30 iterations to move the density to the FP64
# fixed point.
SCF_TOL_EIG = {"64": 1e-6, "216": 1e-6}
# filter form of each arm: the mixed + Pulay arm's FP32 passes run R-ChFSI;
# the learned arm keeps the plain FP32 filter (with R-ChFSI the Pulay
# continuation after the learned mixer's hand-over stalled at density residuals
# of 2-5e-5 on the 216-atom cell in two runs)
FILTER_FORM = {"fp64": lambda c: c.FILTER_CHEBYSHEV, "mixed": lambda c: c.FILTER_RESIDUAL,
               "mixed_learned": lambda c: c.FILTER_CHEBYSHEV}
TIGHT_TOL_PER_ATOM = 1e-10
TIGHT_TOL_EIG = 1e-9


def time_to_scf(chfsi, s, ndeg, device, net, max_iter, tight_max_iter, cell):
    """FP64 + Pulay, mixed + Pulay and mixed + learned-preconditioned Pulay,
    each from the uniform density to the stopping rule (device seconds of the
    SCF loop, context set-up excluded); the FP64 run is then continued,
    untimed, to tight convergence, and every arm's energy and occupied
    eigenvalues are compared with that reference."""
    import numpy as np
    arms = (("fp64", chfsi.PREC_FP64, chfsi.MIXER_PULAY),
            ("mixed", chfsi.PREC_MIXED, chfsi.MIXER_PULAY),
            ("mixed_learned", chfsi.PREC_MIXED, chfsi.MIXER_LEARNED_PULAY))
    res, setup, tight = {}, {}, None
    for name, prec, mode in arms:
        t0 = time.time()
        ctx = chfsi.Context(s, device=device, precision=prec,
                            filter_form=FILTER_FORM[name](chfsi))
        setup[name] = time.time() - t0
        if mode != chfsi.MIXER_PULAY:
            ctx.set_mixer(net)
        res[name] = ctx.run_scf(ndeg, tol_per_atom=SCF_TOL_PER_ATOM, tol_eig=SCF_TOL_EIG[cell],
                                max_iter=max_iter, kT=0.01, mixer=mode,
                                fp64_switch_per_atom=SCF_TOL_PER_ATOM)
        if name == "fp64":
            tight = ctx.run_scf(ndeg, tol_per_atom=TIGHT_TOL_PER_ATOM, tol_eig=TIGHT_TOL_EIG,
                                max_iter=tight_max_iter, kT=0.01, restart=True)
        ctx.close()
    n_occ = s.n_occ
    out = {"criterion": "|dE| < %g Ha/atom and occupied eigenvalues changing by < %g Ha "
                        "on an FP64 iteration (Fermi-Dirac kT = 0.01 Ha; Pulay alpha 0.3, "
                        "history 6); mixed arms (FP32 filter, BF16x3 projector GEMMs, FP64 "
                        "Rayleigh-Ritz; R-ChFSI form in the mixed + Pulay arm) filter in "
                        "FP64 once two mixed iterations change the eigenvalues by < %g Ha "
                        "or those changes level off"
                        % (SCF_TOL_PER_ATOM, SCF_TOL_EIG[cell], 2 * SCF_TOL_EIG[cell]),
           "reference": "FP64 run continued for up to %d more iterations toward |dE| < %g "
                        "Ha/atom and eigenvalue changes < %g Ha" % (tight_max_iter,
                                                                   TIGHT_TOL_PER_ATOM, TIGHT_TOL_EIG),
           "reference_converged": bool(tight["converged"]),
           "reference_extra_iterations": tight["n_iter"],
           "reference_last_energy_change_per_atom_Ha":
               float(abs(tight["energies"][-1] - tight["energies"][-2]) / s.n_atoms)
               if len(tight["energies"]) > 1 else None,
           "arms": {}}
    f = res["fp64"]
    for name, r in res.items():
        a = {"seconds": round(r["seconds"], 3), "iterations": r["n_iter"],
             "iterations_in_mixed_precision": r["n_iter_mixed"], "converged": bool(r["converged"]),
             "setup_seconds": round(setup[name], 2),
             "energy_error_per_atom_Ha": abs(r["e_total"] - tight["e_total"]) / s.n_atoms,
             "max_occupied_eigenvalue_error_Ha":
                 float(np.abs(r["eigenvalues"][:n_occ] - tight["eigenvalues"][:n_occ]).max()),
             "fp64_retries": r["n_fp64_retries"]}
        if name == "mixed_learned":
            a["learned_steps"] = r["n_iter_learned"]
            a["fell_back_to_pulay"] = bool(r["fell_back"])
        if name != "fp64":
            a["speedup_vs_fp64"] = round(f["seconds"] / r["seconds"], 3) if r["seconds"] > 0 else None
        out["arms"][name] = a
    return out


# batched passes: the 8-atom cell on a 4x4x4 Monkhorst-Pack mesh (64
# k-points) and 32 seeded cells of 8, 16, 27 or 64 atoms at the 8-atom cell's
# density (Z = 4, Ecut 15 Ha, 1.25 x the occupied bands)
BATCH_KINDS = [(0, 1, 8), (2, 2, 2), (1, 3, 1), (0, 2, 8)]  # (lattice, n_rep, atoms per cell)
BATCH_DEG = 12


def batch_systems(chfsi):
    import numpy as np
    out = []
    mp = [(i - 2.5) / 4.0 for i in range(1, 5)]
    for kx in mp:
        for ky in mp:
            for kz in mp:
                out.append(chfsi.SyntheticSystem(config_index=0, kpt=(kx, ky, kz)))
    rng = np.random.default_rng(2024)
    vol = 10.26 ** 3 / 8.0
    for i in range(32):
        lattice, n_rep, per = BATCH_KINDS[int(rng.integers(0, len(BATCH_KINDS)))]
        out.append(chfsi.SyntheticSystem(config_index=0, lattice=lattice, n_rep=n_rep,
                                         a_conv=(per * vol) ** (1.0 / 3.0), seed=100 + i,
                                         ngrid=(0, 0, 0), n_bands=0))
    return out


def batched_passes(chfsi, device, reps=3):
    """One mixed-precision pass (degree-12 FP32 filter + FP64 Rayleigh-Ritz)
    of all 96 members: replayed as one CUDA graph, and context by context;
    host wall time per pass including the eigenvalue read-back."""
    import numpy as np
    systems = batch_systems(chfsi)
    ctxs, eigs = [], []
    for s in systems:
        c = chfsi.Context(s, device=device, precision=chfsi.PREC_MIXED)
        c.build_v_eff(np.full(c.ng_density, s.n_elec / s.omega))
        w = c.diagonalize(BATCH_DEG)
        w = c.diagonalize(BATCH_DEG, w)
        ctxs.append(c)
        eigs.append(w)
    b = chfsi.Batch(ctxs)
    nodes = b.capture(BATCH_DEG)
    b.run()
    t0 = time.perf_counter()
    for _ in range(reps):
        eigs = b.run()
    t_graph = (time.perf_counter() - t0) / reps
    for i, c in enumerate(ctxs):
        eigs[i] = c.diagonalize(BATCH_DEG, eigs[i])
    t0 = time.perf_counter()
    for _ in range(reps):
        for i, c in enumerate(ctxs):
            eigs[i] = c.diagonalize(BATCH_DEG, eigs[i])
    t_seq = (time.perf_counter() - t0) / reps
    n_pw = [s.n_pw for s in systems]
    out = {"workload": "64 k-points of the 8-atom cell (4x4x4 Monkhorst-Pack) + 32 cells of "
                       "8/16/27/64 atoms; one degree-%d mixed-precision pass of each" % BATCH_DEG,
           "members": len(systems), "bands": int(sum(s.n_bands for s in systems)),
           "n_pw_min": int(min(n_pw)), "n_pw_max": int(max(n_pw)),
           "graph_nodes": int(nodes), "graph_ms_per_pass": round(t_graph * 1e3, 2),
           "sequential_ms_per_pass": round(t_seq * 1e3, 2),
           "speedup": round(t_seq / t_graph, 3)}
    b.close()
    for c in ctxs:
        c.close()
    return out


def _get_psi_into(ctx, out):
    import ctypes as C
    import chfsi
    ctx._c(chfsi.lib().chfsi_get_psi(ctx.handle, out.ctypes.data_as(C.c_void_p)))


def reference_steps(steps, warmup):
    """The reference's ChFSI iteration on the host cores (the C++/OpenMP
    oracle restatement of chebyshev.rs:626-816 + rayleigh_ritz.rs:48-245),
    inputs from the oracle's own copy of the seeded generator (the CUDA
    library is not loaded).  Each step runs the degree-16 filter on one band
    per host thread (the oracle parallelises over bands) and the
    Rayleigh-Ritz of all 160 bands; the step time is the filter time scaled
    by the per-band cost to 160 bands plus the Rayleigh-Ritz time.
    Returns (seconds per full-step equivalent list, cores, sample text, system)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle
    import synth
    s = synth.System(config_index=CONFIG_INDEX)
    cores = oracle.lib().oracle_num_threads()
    nb = s.n_bands
    nb_s = max(1, min(nb, cores))
    psi0 = s.psi0()
    rho0 = np.full(s.ng, s.n_elec / s.omega)
    args = (s.ngrid, s.miller(), s.kinetic(), s.beta(), s.proj_offsets(), s.dmat())
    tail = (s.vloc_g(), s.omega, s.gmax, s.e_ewald, s.n_atoms)
    o_f = oracle.Oracle(*args, psi0[:nb_s], s.occupations()[:nb_s], *tail)
    o_rr = oracle.Oracle(*args, psi0, s.occupations(), *tail)
    o_f.build_veff(rho0)
    o_rr.build_veff(rho0)
    o_rr.chebyshev_filter(0)  # H|psi> of all bands for the Rayleigh-Ritz (untimed set-up)
    times = []
    for i in range(warmup + steps):
        o_f.set_psi(psi0[:nb_s])
        t0 = time.perf_counter()
        o_f.chebyshev_filter(NDEG)
        t1 = time.perf_counter()
        o_rr.rayleigh_ritz()
        t2 = time.perf_counter()
        if i >= warmup:
            times.append((t1 - t0) * nb / nb_s + (t2 - t1))
    sample = ("per step: degree-16 filter of %d of the %d bands (one per thread), scaled by "
              "%d/%d, plus Rayleigh-Ritz of all %d bands, same 64-atom cell" % (nb_s, nb, nb, nb_s, nb))
    return times, cores, sample, s


def cpu_baseline(steps=2):
    """The reference arm's measurement (reference_steps) on a short sample."""
    times, cores, sample, s = reference_steps(steps, 1)
    value = s.n_bands * (NDEG + 1) * len(times) / sum(times)
    return {"value": round(value, 2), "unit": UNIT, "cores": cores, "kind": "port",
            "sample": sample + "; %d steps" % len(times)}


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return
    times, cores, sample, s = reference_steps(args.steps, args.warmup)
    tot = sum(times)
    value = s.n_bands * (NDEG + 1) * args.steps / tot
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 2), "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(tot / args.steps * 1e3, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded 64-atom diamond cell; per-rank replica)",
            "config": bench_config(s, world),
            "cpu_baseline": {"value": round(value, 2), "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(value, 2), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_profile(kind):
    """Fixed workloads for profiler captures: the 64-atom cell (local, fp64,
    mixed), or two degree-16 passes of the 216-atom ultrasoft cell
    (fp64-216, mixed-216) after one untraced pass from the random start;
    only those two passes run between cudaProfilerStart / Stop (capture
    them with ncu --profile-from-start off)."""
    import numpy as np
    import torch
    import chfsi
    if kind == "gemm":
        # the FP64 tensor-path op::C GEMM at the 216-atom shapes, on random
        # operands of a few GB: psi^H psi (576 x 576, K = 173,925) and a
        # projector product (1,728 x 576) with K cut to 43,000
        g = torch.Generator(device="cuda").manual_seed(0)
        st = torch.cuda.current_stream().cuda_stream
        for m, n, k in ((576, 576, 173925), (1728, 576, 43000)):
            a = torch.randn((m, k), dtype=torch.complex128, device="cuda", generator=g)
            b = a if m == n else torch.randn((n, k), dtype=torch.complex128, device="cuda",
                                             generator=g)
            c = torch.empty((m, n), dtype=torch.complex128, device="cuda")
            for _ in range(2):
                chfsi.zgemm_cn(a.data_ptr(), k, b.data_ptr(), k, m, n, k, c.data_ptr(), st)
            torch.cuda.synchronize()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record()
            chfsi.zgemm_cn(a.data_ptr(), k, b.data_ptr(), k, m, n, k, c.data_ptr(), st)
            ev1.record()
            ev1.synchronize()
            ms = ev0.elapsed_time(ev1)
            print("profile gemm %d x %d x %d: %.3f ms, %.1f TFLOP/s" % (m, n, k, ms,
                                                                       8.0 * m * n * k / ms / 1e9))
            del a, b, c
        return
    if kind.endswith("-216"):
        s = chfsi.SyntheticSystem(config_index=2)
        prec = chfsi.PREC_MIXED if kind.startswith("mixed") else chfsi.PREC_FP64
        ctx = chfsi.Context(s, precision=prec)
        ctx.build_v_eff(np.full(ctx.ng_density, s.n_elec / s.omega))
        e = ctx.diagonalize(16)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        for _ in range(2):
            e = ctx.diagonalize(16, e)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        print("profile %s: 2 traced diagonalisations, lowest eigenvalue %.8f" % (kind, e[0]))
        return
    s = chfsi.SyntheticSystem(config_index=CONFIG_INDEX)
    prec = chfsi.PREC_MIXED if kind == "mixed" else chfsi.PREC_FP64
    ctx = chfsi.Context(s, precision=prec)
    ctx.build_v_eff(np.full(ctx.ng_density, s.n_elec / s.omega))
    if kind == "local":
        x = torch.from_numpy(s.psi0()).cuda()
        y = torch.empty_like(x)
        torch.cuda.synchronize()
        for _ in range(2):
            ctx.apply_h_local(x.data_ptr(), y.data_ptr(), s.n_bands)
        torch.cuda.synchronize()
        print("profile local: 2 launches of %d bands" % s.n_bands)
        return
    e = ctx.diagonalize(NDEG)
    for _ in range(5):
        e = ctx.diagonalize(NDEG, e)
    print("profile %s: 6 diagonalisations, lowest eigenvalue %.8f" % (kind, e[0]))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fp64-only", action="store_true", help="skip the mixed-precision lines")
    ap.add_argument("--no-scf", action="store_true", help="skip every time-to-SCF comparison")
    ap.add_argument("--no-scf-216", action="store_true",
                    help="skip the 216-atom time-to-SCF comparison (about ten minutes)")
    ap.add_argument("--scf-216-max-iter", type=int, default=150)
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the batched-pass comparison (64 k-points + 32 cells)")
    ap.add_argument("--profile", choices=["local", "fp64", "mixed", "fp64-216", "mixed-216", "gemm"],
                    default=None,
                    help="a short fixed workload for ncu captures (no JSON line): two local "
                         "H|psi> launches, or six diagonalisations in one precision (64-atom "
                         "cell), or two traced passes of the 216-atom ultrasoft cell")
    args = ap.parse_args()
    if args.profile:
        run_profile(args.profile)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

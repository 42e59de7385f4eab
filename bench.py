"""Benchmark of the PFDD Ginzburg-Landau step on B200 (one JSON line on rank 0).

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (default `fcc256`): 256x256x128 grid, 12 FCC {111}<110> slip systems,
8 seeded loops (radii U[8,40] cells), sigma_xz = 300 MPa, sine GSFE
(isf 45 / usf 175 mJ/m^2), CD*dt = 0.5, FP32 step with FP64 set-up and FP64
reductions; synthetic seeded input.  A "step" is one GL iteration over the
whole grid; the metric is site-slip updates per second (S * N per step).

  value     device time of K steps (CUDA events on the stepper's stream,
            inputs resident in HBM; the default workload's working set > L2, no
            flush needed; smaller workloads say in config.l2 that they stay
            L2-resident)
  e2e       the same metric through the C ABI from pinned host memory:
            set_state (H2D) + advance(E steps) + get_state (D2H), E =
            --e2e-steps (default 5000, the run length of this configuration)
  roofline  the dominant kernel's algorithmic bytes per launch / its mean
            event-timed duration inside the timed region, against the
            measured HBM copy bandwidth
  cpu_baseline  the reference sources compiled as a CPU oracle (oracle/_ref),
            timed on a bounded sample on this host (rank 0, N = 1 only)

Before the warm-up the x-pencil tile width of every batched group is chosen
by timing (pfdd_gpu_autotune, outside the timed region, like a planner);
--no-autotune keeps the set-up's rule.

Multi-GPU (torchrun): a multi-instance workload (alloy64) is split over the
ranks, each instance on one GPU (scaling "strong"); a one-grid workload runs
one replica per rank (scaling "weak").  No data-path collective; the time is
the max over ranks, the value every rank's units over it.
--impl reference times the reference's own CPU code on this host's cores on
the same workload (see reference_arm) and prints the same line.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "phase-field-dislocation-dynamics-pfdd-2.x_b200")
sys.path.insert(0, PKG_DIR)

METRIC = "site-slip updates/s per GL step"
UNIT = "site-slip updates/s"
FALLBACK_HBM_GBS = 6650.0


def peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


WORKLOADS = ("fcc256", "loop64", "alloy64", "edge128", "frank512")


def workload_config(name):
    """(workloads, description, default precision) of a named configuration."""
    from pfdd_b200 import configs
    if name == "fcc256":
        ws = [configs.fcc_workload()]
        desc = ("fcc256: 256x256x128 grid, 12 FCC slip systems, 8 seeded loops r~U[8,40], "
                "sigma_xz 300 MPa, sine GSFE 45/175 mJ/m^2")
        prec = "fp32"
    elif name == "loop64":
        ws = [configs.loop_workload()]
        desc = ("loop64: 64^3 grid, 3 systems on one {111} plane, loop r=12 + U(-1e-3,1e-3) noise (seed 576), "
                "sigma_xz 200 MPa, sine GSFE 45/175 mJ/m^2, plain FP64")
        prec = "fp64"
    elif name == "alloy64":
        ws = configs.alloy_batch(64)
        desc = ("alloy64: 64 instances, n^3 with n~U{32,48,64,96,128}, 3 systems, lognormal(0,0.15) per-site "
                "isf/usf multiplier, sigma~U[100,400] MPa, batched groups + CUDA graphs")
        prec = "fp32"
    elif name == "edge128":
        ws = [configs.edge_workload()]
        desc = ("edge128: 128x128x32, 3 basal systems, straight edge + 10-cell seeded perturbation, "
                "sigma_xz 250 MPa; adjoint 500 steps, checkpoint every 50")
        prec = "fp32"
    elif name == "frank512":
        ws = [configs.frank_read_workload()]
        desc = ("frank512: 512x512x64 on a 60-degree skewed grid, 2 BCC systems, 64-cell pinned segment (xo mask), "
                "usf 300 mJ/m^2, sigma_yz ramp 0->600 MPa over 20000 one-step stress states")
        prec = "fp32"
    else:
        raise SystemExit("unknown workload %s (one of %s)" % (name, ", ".join(WORKLOADS)))
    return ws, desc, prec


def sample_clocks(dev_index):
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
    try:
        proc = subprocess.Popen(["nvidia-smi", "-i", str(dev_index), "--query-gpu=" + q,
                                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=f,
                                stderr=subprocess.DEVNULL)
    except Exception:
        proc = None
    return proc, f.name


def parse_clocks(proc, path):
    if proc is None:
        return None
    proc.terminate()
    try:
        proc.wait(5)
    except Exception:
        proc.kill()
    sm, mx, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    try:
        for line in open(path):
            c = [x.strip() for x in line.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1]))
                mx.append(float(c[2]))
            except ValueError:
                continue
            for n, v in zip(names, c[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
    finally:
        os.unlink(path)
    if not sm:
        return None
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
            "samples": len(sm)}


def kernel_bytes(w, F, csize, rsize):
    """Algorithmic HBM bytes per launch of each kernel for one instance (one
    read and one write of what the pass must move): the opening forward pass
    reads xi and writes the half spectrum; the x-pencil pass reads and writes
    it; the fused plane pass reads it plus xi (and the mask or per-site GSFE
    field when present), writes the new xi and the next step's spectrum."""
    N = w.nx * w.ny * w.nz
    spec = F * w.nx * w.ny * (w.nz // 2 + 1) * csize
    field = F * N * rsize
    extra = (w.S * N if w.xo is not None else 0) + (w.S * N * rsize if w.site is not None else 0)
    return {"fwd_planes": field + spec, "xpencil": 2 * spec, "step_planes": 2 * spec + 2 * field + extra}


def fields_carried(w):
    """Real fields through the FFT passes: Re xi, plus Im xi when a mask forces
    the full complex carrier (otherwise Im xi rides on the Nyquist planes)."""
    return 2 * w.S if w.xo is not None else w.S


def traffic_from_profiles(kernel, workload):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            t = json.load(f)
        return t[workload][kernel]
    except Exception:
        return None


def cpu_baseline_reference(K=10, procs=1, nx=64, ny=64, nz=32):
    """Reference sources (oracle/_ref) on a bounded sample: the same FCC
    workload on a nx*ny*nz grid, K GL steps per process, `procs` independent
    processes.  Returns (site-slip updates/s aggregate, sample text)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_runner
    from pfdd_b200 import configs
    if not ref_runner.available():
        return None, "reference oracle not built (make -C oracle/ref_build)"
    w = configs.fcc_workload(nx, ny, nz, n_loops=4)
    import concurrent.futures as cf
    import multiprocessing as mp

    def one(_):
        r = ref_runner.run_reference(w, K, timing=True)
        return r["timing"]

    if procs == 1:
        res = [one(0)]
    else:
        with cf.ThreadPoolExecutor(procs) as ex:
            res = list(ex.map(one, range(procs)))
    rate = sum(r["site_slip_updates_per_s"] for r in res)
    fft = statistics.mean(r["fft_gflops"] for r in res)
    sample = ("reference src/*.cpp built -O3 with a single-rank MPI stub and an FP64 FFTW-2 API stand-in "
              "(%.2f GFLOP/s FFT); a bounded sample of the FCC 12-system deck on %dx%dx%d, %d GL steps x %d "
              "process(es), loop time only (the full 256x256x128 grid is timed by bench.py --impl reference)"
              % (fft, nx, ny, nz, K, procs))
    return rate, sample


def mem_available_gb():
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable"):
                return int(line.split()[1]) / 1e6
    except Exception:
        pass
    return None


def reference_host_bytes(w):
    """Resident host bytes of the reference on workload w (FFTW_Slab::allocate,
    fft_fftw_slab.cpp:140-237, as Bmatrix/Fmatrix and the GL loop touch them):
    BB (S^2 N), FF and DD (9 S N each), data_fftw/data_real/temp_data/data_core
    (complex S N each), xi, dE_core, f, xo, fx/fy/fz and the strain/stress
    fields, in doubles."""
    S, N = w.S, w.N
    doubles = S * S * N + 18 * S * N + 8 * S * N + 2 * S * N + 3 * S * N + 3 * N + 4 * 18 * N
    return 8 * doubles


def reference_arm(args):
    """The reference's own CPU implementation (its sources compiled in
    oracle/_ref) on this host, on the same workload as the GPU arm: the full
    grid for one-instance workloads, K' <= 3 GL iterations timed as the
    reference's loop time (Finish, finish.cpp:42-55), set-up excluded.  Its
    per-wavevector set-up runs on forked one-plane slabs and its FFTW-2
    stand-in on threads, over every host core (bit-identical to one process,
    tests/test_oracle_parallel_cpu.py); the reference's own loops
    (internal_energy, core force, update) run on one core, as on one MPI rank.
    Multi-instance workloads run independent single-thread processes, one per
    instance, up to the core count.  Rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_runner
    ncpu = os.cpu_count() or 1
    ws, w_desc, _ = workload_config(args.workload)
    if not ref_runner.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference oracle not built (make -C oracle/ref_build)"}))
        return 0
    t0 = time.time()
    mem = mem_available_gb()
    iters = max(1, min(args.steps, 3))
    if len(ws) == 1:
        w = ws[0]
        need_gb = reference_host_bytes(w) / 1e9
        if mem is not None and mem < 1.25 * need_gb:
            # not enough host memory for the full grid: a labelled sample of the same deck instead
            from pfdd_b200 import configs
            w = configs.fcc_workload(64, 64, 32, n_loops=4)
            w_desc = ("SAMPLE fcc 64x64x32 (12 FCC systems, 4 loops): the host has %.0f GB available, the "
                      "reference needs ~%.0f GB for %s" % (mem, need_gb, args.workload))
        env_old = {k: os.environ.get(k) for k in ("PFDD_ORACLE_SETUP_PROCS", "PFDD_SHIM_THREADS")}
        os.environ["PFDD_ORACLE_SETUP_PROCS"] = str(ncpu)
        os.environ["PFDD_SHIM_THREADS"] = str(ncpu)
        try:
            r = ref_runner.run_reference(w, iters, timing=True, timeout=3000)
        finally:
            for k, v in env_old.items():
                if v is None:
                    os.environ.pop(k, None)
                else:
                    os.environ[k] = v
        tm = r["timing"]
        rate = tm["site_slip_updates_per_s"]
        cores = ncpu
        sample = ("reference src/*.cpp built -O3 with a single-rank MPI stub and an FP64 FFTW-2 API stand-in "
                  "(transforms on %d threads, %.2f GFLOP/s of FFT work per loop second); %dx%dx%d grid x %d systems, "
                  "%d GL iterations, loop time %.2f s (set-up on %d forked processes, not timed); the reference's "
                  "own loops run on one core as on one MPI rank"
                  % (ncpu, tm["fft_gflops"], w.nx, w.ny, w.nz, w.S, tm["iterations"], tm["loop_s"], ncpu))
        parallelism = "1 process, FFT on %d threads" % ncpu
    else:
        import concurrent.futures as cf
        sub = ws[:max(1, min(len(ws), ncpu))]

        def one(w):
            # the per-site-multiplier sine core has no reference counterpart: the
            # reference's per-site-amplitude core (core_energy_mpea, flag 7) stands in
            import copy
            wr = copy.copy(w)
            mpea = None
            if w.core_flag == 103:
                wr.core_flag = 7
                mpea = w.site * w.material.usf
            return ref_runner.run_reference(wr, iters, mpea=mpea, timing=True)["timing"]

        with cf.ThreadPoolExecutor(len(sub)) as ex:
            res = list(ex.map(one, sub))
        rate = sum(r["site_slip_updates_per_s"] for r in res)
        cores = len(sub)
        sample = ("reference src/*.cpp built -O3 with a single-rank MPI stub and an FP64 FFTW-2 API stand-in; "
                  "%d of the %d instances as concurrent single-thread processes, %d GL iterations each, loop time "
                  "only, aggregate throughput; the per-site GSFE field runs through the reference's per-site "
                  "amplitude core (core_energy_mpea)" % (len(sub), len(ws), iters))
        parallelism = "%d independent CPU processes" % len(sub)
    line = {
        "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": iters, "warmup": args.warmup,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": w_desc, "parallelism": parallelism},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "host_mem_available_gb": mem, "wall_s": time.time() - t0,
    }
    print(json.dumps(line))
    return 0


def max_over_ranks(x, dist, device="cuda"):
    """The largest of each rank's x (every rank calls this at the same point;
    one all-reduce).  Without a process group, x itself."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank, world, ms):
    """Whole-job throughput: the units every rank processed over the slowest
    rank's time (ms)."""
    return units_per_rank * world / (ms / 1e3)


def shard_instances(ws, rank, world):
    """The instances rank `rank` advances: a multi-instance workload is split
    round robin over the ranks (each instance on one GPU, no data-path
    collective; the total work is fixed, so scaling is strong); a one-grid
    workload runs as one replica per rank (weak scaling)."""
    if world > 1 and len(ws) > 1:
        if len(ws) < world:
            raise SystemExit("%d instances cannot be split over %d ranks" % (len(ws), world))
        return ws[rank::world], "strong"
    return ws, "weak"


def sum_over_ranks(x, dist, device="cuda"):
    """Sum of each rank's x (every rank calls it at the same point)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def timed_events(stream, fn):
    import torch
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    out = fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), out


def fp32_vs_fp64(ws, K, stream, local, steps=2000, early=10):
    """FP32 and FP64 speed of the same grid (the same timed profile pass of K
    steps), and the FP32 error against the FP64 GPU path (relative L2 of Re
    xi) after `early` and `steps` steps.  The FP64 path equals the oracle to
    1e-10 per step (tests/test_gpu_config_sizes.py).  An FP64 run started 1e-7
    (seeded normal) away is the control: where it drifts as far as FP32 does,
    the trajectory amplifies perturbations and the long-horizon figure
    measures the dynamics, not the arithmetic."""
    import numpy as np
    from pfdd_b200 import capi
    w = ws[0]
    pert = 1e-7 * np.random.default_rng(1).standard_normal(w.xi0.shape)
    out, states = {}, {}
    for name, prec, x0 in (("fp32", capi.FP32, w.xi0), ("fp64", capi.FP64, w.xi0),
                           ("fp64_perturbed", capi.FP64, w.xi0 + pert)):
        with capi.Stepper.from_workloads([w], precision=prec, device=local) as st:
            st.set_stream(stream.cuda_stream)
            st.set_state(0, w.xi0)
            if name != "fp64_perturbed":
                st.autotune(reps=5)
                st.advance(5)
                ms, _ = timed_events(stream, lambda: st.profile(K))
                out[name + "_ms_per_step"] = ms / K
            st.set_state(0, x0)
            st.advance(early)
            states[(name, early)] = st.get_state(0, imag=False)[0]
            st.advance(steps - early)
            states[(name, steps)] = st.get_state(0, imag=False)[0]
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    for n in (early, steps):
        b = states[("fp64", n)]
        out["rel_l2_fp32_vs_fp64_after_%d" % n] = rel(states[("fp32", n)], b)
        out["rel_l2_fp64_perturbed_1e-7_vs_fp64_after_%d" % n] = rel(states[("fp64_perturbed", n)], b)
    out["max_abs_fp32_vs_fp64_after_%d" % steps] = float(np.abs(states[("fp32", steps)] - states[("fp64", steps)]).max())
    out["steps_compared"] = [early, steps]
    out["fp32_speedup"] = out["fp64_ms_per_step"] / out["fp32_ms_per_step"]
    units = w.S * w.N
    out["fp64_site_slip_updates_per_s"] = units / (out["fp64_ms_per_step"] / 1e3)
    out["fp32_site_slip_updates_per_s"] = units / (out["fp32_ms_per_step"] / 1e3)
    return out


def fp64_plain_batch(ws, K, stream, local):
    """The plain FP64 path on a batch: each instance on its own handle, one
    after the other (no batching, no merged launches), K steps each timed
    with CUDA events; site-slip updates/s over the whole batch."""
    from pfdd_b200 import capi
    total_ms, units = 0.0, 0
    for w in ws:
        with capi.Stepper.from_workloads([w], precision=capi.FP64, device=local) as st:
            st.set_stream(stream.cuda_stream)
            st.set_state(0, w.xi0)
            st.advance(3)
            ms, _ = timed_events(stream, lambda: st.advance(K))
            total_ms += ms / K
            units += w.S * w.N
    return {"fp64_plain_ms_per_step": total_ms, "fp64_plain_site_slip_updates_per_s": units / (total_ms / 1e3),
            "note": "each of the %d instances advanced alone in FP64 (graph replay), %d steps each" % (len(ws), K)}


def cufft_comparison(w, F, prec, stream, reps=10):
    """cuFFT (torch.fft) real-to-complex and complex-to-real 3-D transforms of
    the same F fields on the same grid and precision, timed alone with CUDA
    events (median of `reps` single calls into preallocated outputs): what a
    library FFT pair costs before any contraction or update."""
    import torch
    dt = torch.float32 if prec == "fp32" else torch.float64
    x = torch.randn(F, w.nx, w.ny, w.nz, device="cuda", dtype=dt)
    y = torch.fft.rfftn(x, dim=(1, 2, 3))
    z = torch.empty_like(x)

    def t(fn):
        with torch.cuda.stream(stream):
            for _ in range(3):
                fn()
            ms = [timed_events(stream, fn)[0] for _ in range(reps)]
        return statistics.median(ms)

    r = t(lambda: torch.fft.rfftn(x, dim=(1, 2, 3), out=y))
    i = t(lambda: torch.fft.irfftn(y, s=(w.nx, w.ny, w.nz), dim=(1, 2, 3), out=z))
    del x, y, z
    torch.cuda.empty_cache()
    return {"rfftn_ms": r, "irfftn_ms": i, "pair_ms": r + i,
            "note": "torch.fft (cuFFT) on [%d,%d,%d,%d] %s, transforms only, median of %d calls"
                    % (F, w.nx, w.ny, w.nz, prec, reps)}


def adjoint_ratio(st, w, prec, stream, local, steps=500, ckpt=50):
    """Adjoint call over forward time for `steps` steps, keeping every state
    and with checkpoints: pfdd_gpu_adjoint (forward tape + backward) seeded
    with dJ/dRe xi_N of J = sum (Re xi_N - target)^2, the target state from a
    forward run with isf 40 / usf 160 mJ/m^2 and 250 MPa.  st = None: a
    stepper of w of its own."""
    import copy
    import numpy as np
    from pfdd_b200 import capi, configs
    if st is None:
        with capi.Stepper.from_workloads([w], precision=prec, device=local) as own:
            own.set_stream(stream.cuda_stream)
            own.set_state(0, w.xi0)
            own.autotune(reps=5)
            return adjoint_ratio(own, w, prec, stream, local, steps, ckpt)
    wt = copy.deepcopy(w)
    wt.material.isf, wt.material.usf = 0.040, 0.160
    wt.sigma = configs._sigma("xz", 250e6 / wt.material.mu)
    with capi.Stepper.from_workloads([wt], precision=prec, device=local) as tg:
        tg.set_state(0, wt.xi0)
        tg.advance(steps)
        target = tg.get_state(0)[0]
    st.set_state(0, w.xi0)
    fwd_ms, _ = timed_events(stream, lambda: st.advance(steps))
    # the seed of J = sum (Re xi_N - target)^2 at this run's end state
    xN, _ = st.get_state(0, imag=False)
    seed = 2.0 * (xN - target)
    loss = float(np.sum((xN - target) ** 2))
    out = {"steps": steps, "forward_ms": fwd_ms, "loss": loss}
    # every state of the run kept on the device (no recomputation) when it
    # takes under 16 GB, and checkpoints every `ckpt` steps with one forward
    # re-run per segment but the last
    state_bytes = w.S * w.N * (4 if prec == capi.FP32 else 8)
    modes = [("checkpointed", ckpt)]
    if steps * state_bytes <= 16e9:
        modes.insert(0, ("store_all", steps))
    for name, k in modes:
        # one untimed call of the same length first: its scratch buffers (kept
        # by the instance between calls) and first kernel loads
        st.set_state(0, w.xi0)
        st.adjoint(0, steps, k, seed)
        st.set_state(0, w.xi0)
        adj_ms, res = timed_events(stream, lambda: st.adjoint(0, steps, k, seed))
        dp, ds = res
        out[name] = {"checkpoint_every": k, "adjoint_call_ms": adj_ms, "adjoint_call_over_forward": adj_ms / fwd_ms,
                     "backward_over_forward": (adj_ms - fwd_ms) / fwd_ms,
                     "dL_dparams": [float(x) for x in dp], "dL_dsigma": [float(x) for x in ds]}
    return out


def diagnostic_only(args):
    """pfdd_gpu_strain_stress (averages only, as DiagStress reads them between
    dumps) on the first instance of the workload: one untimed call, then four
    event-timed calls; prints one JSON line (not a bench line)."""
    import statistics
    import torch
    from pfdd_b200 import capi
    ws, w_desc, prec_name = workload_config(args.workload)
    prec = capi.FP32 if (args.precision or prec_name) == "fp32" else capi.FP64
    w = ws[0]
    with capi.Stepper.from_workloads([w], precision=prec) as st:
        stream = torch.cuda.current_stream()
        st.set_stream(stream.cuda_stream)
        st.set_state(0, w.xi0)
        st.advance(2)
        st.strain_stress(0, fields=False)
        ms = [timed_events(stream, lambda: st.strain_stress(0, fields=False))[0] for _ in range(4)]
    print(json.dumps({"diagnostic": "strain_stress (averages)", "workload": w_desc,
                      "ms_median": statistics.median(ms), "ms": ms}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="fcc256", choices=WORKLOADS)
    ap.add_argument("--precision", default=None, choices=["fp32", "fp64"])
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the set-up's x-pencil tile widths instead of timing them (pfdd_gpu_autotune)")
    ap.add_argument("--diagnostic-only", action="store_true",
                    help="time only the strain/stress diagnostic (averages) on the workload's first instance, "
                         "after two steps: a short run for profiling its kernels")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        return reference_arm(args)
    if args.diagnostic_only:
        return diagnostic_only(args)

    import numpy as np
    import torch
    from pfdd_b200 import capi

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        import datetime
        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = dist_mod

    ws_all, w_desc, prec_name = workload_config(args.workload)
    ws, scaling = shard_instances(ws_all, rank, world)
    prec_name = args.precision or prec_name
    prec = capi.FP32 if prec_name == "fp32" else capi.FP64
    ramp = args.workload == "frank512"   # one GL step per stress state
    run_len = {"fcc256": 5000, "loop64": 2000, "alloy64": 1000, "edge128": 500, "frank512": 20000}[args.workload]
    E = args.e2e_steps or run_len
    st = capi.Stepper.from_workloads(ws, precision=prec, device=local)
    stream = torch.cuda.current_stream()
    st.set_stream(stream.cuda_stream)
    for i, w in enumerate(ws):
        st.set_state(i, w.xi0)
    # measured x-pencil tile widths (a planner step before the clock starts)
    tile_widths = None if args.no_autotune else sorted(set(st.autotune(reps=5)))
    st.advance(args.warmup)

    # timed region: K GL iterations with per-kernel events (profile pass)
    clk_proc, clk_path = sample_clocks(local)
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    kms, launches_per_step = st.profile(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = parse_clocks(clk_proc, clk_path)
    ms = max_over_ranks(e0.elapsed_time(e1), dist)
    units_per_step = sum(w.S * w.N for w in ws)
    # units of the whole job: every rank's own (sharded or replicated)
    job_units_per_step = sum_over_ranks(units_per_step, dist)
    value = job_units_per_step * args.steps / (ms / 1e3)

    # roofline of the dominant kernel (bytes summed over the instances of every group)
    n_inst, dev_bytes = st.info()
    csize, rsize = (8, 4) if prec == capi.FP32 else (16, 8)
    kb = {k: 0 for k in ("fwd_planes", "xpencil", "step_planes")}
    for w in ws:
        for k, v in kernel_bytes(w, fields_carried(w), csize, rsize).items():
            kb[k] += v
    # per-iteration kernels (the opening forward pass runs once per run)
    dom = max(("xpencil", "step_planes"), key=lambda k: kms[k])
    peak, peak_kind = peak_hbm()
    achieved = kb[dom] / (kms[dom] / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "algorithmic_bytes_per_launch": kb[dom], "mean_launch_ms": kms[dom],
                "traffic": traffic_from_profiles(dom, args.workload),
                "kernel_ms": kms,
                "step_algorithmic_gbs": (kb["xpencil"] + kb["step_planes"] + kb["fwd_planes"] / args.steps)
                / (ms / args.steps / 1e3) / 1e9}

    # end to end through the C ABI from pinned host memory: every instance's
    # state in (H2D), the run, every state out (D2H)
    e2e = None
    if rank == 0 or world > 1:
        import ctypes
        lib = capi.load()
        DP = capi.DP
        hosts = []
        for w in ws:
            n_el = w.S * w.N
            hin = torch.empty(2 * n_el, dtype=torch.float64, pin_memory=True)
            hout = torch.empty(2 * n_el, dtype=torch.float64, pin_memory=True)
            v = hin.numpy()
            v[0::2] = w.xi0.reshape(-1)
            v[1::2] = 0.0
            hosts.append((hin, hout))

        def run_e2e():
            rc = 0
            for i, (hin, _) in enumerate(hosts):
                rc |= lib.pfdd_gpu_set_state_interleaved(st.h, i, ctypes.cast(hin.data_ptr(), DP))
            stats = (capi.StepStats * len(ws))()
            if ramp:
                rc |= lib.pfdd_gpu_advance(st.h, 1, E, 0.0, stats)
            else:
                rc |= lib.pfdd_gpu_advance(st.h, E, 1, 0.0, stats)
            for i, (_, hout) in enumerate(hosts):
                rc |= lib.pfdd_gpu_get_state_interleaved(st.h, i, ctypes.cast(hout.data_ptr(), DP))
            return rc

        ems, rc = timed_events(stream, run_e2e)
        if rc != 0:
            raise RuntimeError(lib.pfdd_gpu_last_error(st.h))
        ems = max_over_ranks(ems, dist)
        nbytes = sum(16 * w.S * w.N for w in ws)
        e2e = {"value": job_units_per_step * E / (ems / 1e3), "unit": UNIT, "steps": E,
               "h2d_bytes_per_step": nbytes / E, "d2h_bytes_per_step": nbytes / E + 16 * len(ws),
               "note": ("set_state_interleaved + advance(%s) + get_state_interleaved per instance, pinned host "
                        "buffers" % ("1 step x %d stress states" % E if ramp else "%d" % E))}

    extras = {}
    if not args.no_extras and rank == 0 and len(ws) == 1:
        extras["cufft_comparison"] = cufft_comparison(ws[0], fields_carried(ws[0]), prec_name, stream)
        # strain / stress diagnostics of the current state (averages only, no field copy-out)
        st.strain_stress(0, fields=False)
        dms = [timed_events(stream, lambda: st.strain_stress(0, fields=False))[0] for _ in range(3)]
        extras["strain_stress_ms"] = statistics.median(dms)
    if not args.no_extras and rank == 0:
        if args.workload == "alloy64":
            # the FP32 batched path against the plain FP64 path on the same instances
            pl = fp64_plain_batch(ws, 20, stream, local)
            pl["fp32_batched_over_fp64_plain"] = value / pl["fp64_plain_site_slip_updates_per_s"]
            extras["fp64_plain"] = pl
        if args.workload in ("loop64", "fcc256"):
            # the metric's "FP32 vs FP64 at stated err" on the timed grid itself
            extras["fp32_vs_fp64"] = fp32_vs_fp64(ws, args.steps, stream, local)
        if args.workload in ("edge128", "fcc256"):
            # the metric's "adjoint/fwd ratio" on its own configuration: 128x128x32,
            # 500 steps, a checkpoint every 50
            from pfdd_b200 import configs
            if args.workload == "edge128":
                extras["adjoint"] = adjoint_ratio(st, ws[0], prec, stream, local)
            else:
                extras["adjoint"] = dict(adjoint_ratio(None, configs.edge_workload(), capi.FP32, stream, local),
                                         workload="edge128: 128x128x32, 3 systems, FP32")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, sample = cpu_baseline_reference(K=10, procs=1)
        if rate is not None:
            cpu = {"value": rate, "unit": UNIT, "cores": 1, "kind": "reference", "sample": sample}
        else:
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": sample}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": scaling, "vs_baseline": None, "dtype": "f32" if prec == capi.FP32 else "f64",
            "data": "synthetic",
            "config": {"workload": w_desc, "instances": len(ws),
                       "grid": [ws[0].nx, ws[0].ny, ws[0].nz] if len(ws) == 1 else "mixed",
                       "slip_systems": ws[0].S, "precision": prec_name,
                       "imag_part": ("full complex carrier (obstacle mask)" if ws[0].xo is not None else
                                     "Nyquist-plane spectrum carried in the x-pencil pass"),
                       "parallelism": ("%d instances split over %d ranks" % (len(ws_all), world)
                                       if scaling == "strong" else "replicas x%d" % world),
                       "pencil_tile_widths": tile_widths if tile_widths is not None else "set-up rule",
                       "l2": (("working set %.2f GB > 126 MB L2 (no flush)" % (dev_bytes / 1e9))
                              if dev_bytes > 126e6 else
                              ("working set %.3f GB < 126 MB L2: stays L2-resident from step to step (not "
                               "flushed; the default fcc256 line exceeds L2)" % (dev_bytes / 1e9)))},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
            "gpu_launches": launches_per_step * args.steps + 2 * (launches_per_step // 3),
        }
        line.update(extras)
        print(json.dumps(line))
    st.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

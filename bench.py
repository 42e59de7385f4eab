"""Benchmark of the PFDD Ginzburg-Landau step on B200 (one JSON line on rank 0).

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (default `fcc256`): 256x256x128 grid, 12 FCC {111}<110> slip systems,
8 seeded loops (radii U[8,40] cells), sigma_xz = 300 MPa, sine GSFE
(isf 45 / usf 175 mJ/m^2), CD*dt = 0.5, FP32 step with FP64 set-up and FP64
reductions; synthetic seeded input.  A "step" is one GL iteration over the
whole grid; the metric is site-slip updates per second (S * N per step).

  value     device time of K steps (CUDA events on the stepper's stream,
            inputs resident in HBM; working set > L2, no flush needed)
  e2e       the same metric through the C ABI from pinned host memory:
            set_state (H2D) + advance(E steps) + get_state (D2H), E =
            --e2e-steps (default 5000, the run length of this configuration)
  roofline  the dominant kernel's algorithmic bytes per launch / its mean
            event-timed duration inside the timed region, against the
            measured HBM copy bandwidth
  cpu_baseline  the reference sources compiled as a CPU oracle (oracle/_ref),
            timed on a bounded sample on this host (rank 0, N = 1 only)

Multi-GPU (torchrun): every rank advances its own replica (no data-path
collective; scaling "weak"); the time is the max over ranks.
--impl reference times the reference's own CPU code on this host's cores
(independent processes, aggregate throughput) and prints the same line.
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


def workload_config(name):
    from pfdd_b200 import configs
    if name == "fcc256":
        w = configs.fcc_workload()
        desc = ("fcc256: 256x256x128 grid, 12 FCC slip systems, 8 seeded loops r~U[8,40], "
                "sigma_xz 300 MPa, sine GSFE 45/175 mJ/m^2")
    elif name == "loop64":
        w = configs.loop_workload()
        desc = "loop64: 64^3 grid, 3 systems on one plane, loop r=12 + 1e-3 noise, sigma_xz 200 MPa"
    else:
        raise SystemExit("unknown workload %s" % name)
    return w, desc


def sample_clocks(dev_index):
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
    try:
        proc = subprocess.Popen(["nvidia-smi", "-i", str(dev_index), "--query-gpu=" + q,
                                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=f,
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
    """Algorithmic HBM bytes per launch of each kernel (one read and one write
    of what the pass must move): P1 reads xi and writes the half spectrum, P2
    reads and writes it, P3 reads it plus xi and writes xi."""
    N = w.nx * w.ny * w.nz
    spec = F * w.nx * w.ny * (w.nz // 2 + 1) * csize
    field = F * N * rsize
    return {"fwd_planes": field + spec, "xpencil": 2 * spec, "inv_update": spec + 2 * field}


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
              "(%.2f GFLOP/s FFT); FCC 12 systems on %dx%dx%d, %d GL steps x %d process(es), loop time only "
              "(the 256x256x128 grid needs ~20 GB and ~10 min of B(k) set-up in the reference)"
              % (fft, nx, ny, nz, K, procs))
    return rate, sample


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    ncpu = os.cpu_count() or 1
    mem_gb = 8.0
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable"):
                mem_gb = int(line.split()[1]) / 1e6
    except Exception:
        pass
    procs = max(1, min(ncpu, int(mem_gb * 0.5 / 1.0), 64))
    K = max(1, args.steps)
    t0 = time.time()
    rate, sample = cpu_baseline_reference(K=K, procs=procs)
    if rate is None:
        print(json.dumps({"impl": "reference", "unavailable": sample}))
        return 0
    wall = time.time() - t0
    w_desc = workload_config(args.workload)[1]
    line = {
        "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": K, "warmup": args.warmup,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": w_desc, "parallelism": "%d independent CPU processes" % procs},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": procs, "kind": "reference", "sample": sample},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": wall,
    }
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="fcc256")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--e2e-steps", type=int, default=5000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        return reference_arm(args)

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

    w, w_desc = workload_config(args.workload)
    prec = capi.FP32 if args.precision == "fp32" else capi.FP64
    st = capi.Stepper.from_workloads([w], precision=prec, device=local)
    stream = torch.cuda.current_stream()
    st.set_stream(stream.cuda_stream)
    st.set_state(0, w.xi0)
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
    ms = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    S, N = w.S, w.N
    per_gpu_updates = S * N * args.steps
    value = per_gpu_updates * world / (ms / 1e3)

    # roofline of the dominant kernel
    F = st.descs[0].n_slip  # Re xi field; Im xi rides on the Nyquist planes (no mask)
    n_inst, dev_bytes = st.info()
    csize, rsize = (8, 4) if prec == capi.FP32 else (16, 8)
    kb = kernel_bytes(w, F, csize, rsize)
    dom = max(kb, key=lambda k: kms[k])
    peak, peak_kind = peak_hbm()
    achieved = kb[dom] / (kms[dom] / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "algorithmic_bytes_per_launch": kb[dom], "mean_launch_ms": kms[dom],
                "traffic": traffic_from_profiles(dom, args.workload),
                "kernel_ms": kms}

    # end to end through the C ABI from pinned host memory
    e2e = None
    if rank == 0 or world > 1:
        n_el = S * N
        host_in = torch.empty(2 * n_el, dtype=torch.float64, pin_memory=True)
        host_out = torch.empty(2 * n_el, dtype=torch.float64, pin_memory=True)
        hin = host_in.numpy()
        hin[0::2] = w.xi0.reshape(-1)
        hin[1::2] = 0.0
        import ctypes
        lib = capi.load()
        DP = capi.DP
        E = args.e2e_steps
        torch.cuda.synchronize()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        rc = lib.pfdd_gpu_set_state_interleaved(st.h, 0, ctypes.cast(host_in.data_ptr(), DP))
        stats = (capi.StepStats * 1)()
        rc |= lib.pfdd_gpu_advance(st.h, E, 1, 0.0, stats)
        rc |= lib.pfdd_gpu_get_state_interleaved(st.h, 0, ctypes.cast(host_out.data_ptr(), DP))
        a1.record(stream)
        torch.cuda.synchronize()
        if rc != 0:
            raise RuntimeError(lib.pfdd_gpu_last_error(st.h))
        ems = a0.elapsed_time(a1)
        if dist:
            t = torch.tensor([ems], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        e2e = {"value": S * N * E * world / (ems / 1e3), "unit": UNIT, "steps": E,
               "h2d_bytes_per_step": 16 * n_el / E, "d2h_bytes_per_step": 16 * n_el / E + 16,
               "note": "set_state_interleaved + advance(%d) + get_state_interleaved, pinned host buffers" % E}

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
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if prec == capi.FP32 else "f64",
            "data": "synthetic",
            "config": {"workload": w_desc, "grid": [w.nx, w.ny, w.nz], "slip_systems": S,
                       "precision": args.precision, "imag_part": "Nyquist-plane spectrum carried in the x-pencil pass",
                       "parallelism": "replicas x%d" % world,
                       "l2": "working set %.2f GB > 126 MB L2 (no flush)" % (dev_bytes / 1e9)},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
            "gpu_launches": launches_per_step * args.steps + 1,
        }
        print(json.dumps(line))
    st.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

"""Benchmark of the B200 ScatCov engine: S1-S4 forward + VJP evaluations per second.

Workload (one step): forward + exact VJP of the full ScatCov statistics
(mean, var, S1..S4; L = 4, J = 9, 11 354 coefficients) of a batch of B = 4
synthetic lognormal HEALPix maps at nside 1024 (12 582 912 NESTED pixels,
x = exp(g - 1/2), g ~ N(0, 1), seeds 0..3), in FP32 fields with FP64 sums;
the cotangent is that of the loss sum |S - S_t|^2 (S_t: the map of seed 100),
computed on the host from the step's values.  One evaluation = one map.
The same step is timed for one FP64 map (the plain FP64 path) and through
the reference-facing host-buffer API (stlp_forward / stlp_vjp: f64 maps in
and gradients out over PCIe).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun (N > 1) every rank evaluates its own batch (independent
replicas, no collective in the path); the time is the max over ranks.
``--impl reference`` times the CPU oracle (the FP64 restatement of the
reference's CPU engine) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "stl-dev-mpi_b200"))

METRIC = "S1–S4 fwd+VJP evals/s, nside 1024 J=9: FP32-batched vs FP64 plain, err≤1e-6"
UNIT = "evals/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--nside", type=int, default=1024)
    p.add_argument("--J", type=int, default=9)
    p.add_argument("--batch", type=int, default=4)
    p.add_argument("--skip-fp64", action="store_true")
    p.add_argument("--skip-cpu", action="store_true")
    p.add_argument("--profile-step", action="store_true",
                   help="one forward + VJP of the batch and exit (no timing, no line): the launch sequence that "
                        "the kernel profiles in profiles/ capture")
    p.add_argument("--no-autotune", action="store_true",
                   help="default tile heights instead of timing them at prepare (for runs under a profiler, whose "
                        "replays make the timing meaningless)")
    p.add_argument("--workload", default="scatcov", choices=["scatcov", "patches", "synthesis", "cross", "spin"],
                   help="scatcov: the headline metric; patches: 512 ragged disc patches (nside 512, J 5); "
                        "synthesis: 200 L-BFGS iterations at nside 1024, J 9; cross: the cross terms of two "
                        "channels at nside 1024, J 9; spin: two (Q, U) maps through the spin-2 front end")
    return p.parse_args()


def lognormal(seed, npix, sigma=1.0):
    g = np.random.default_rng(seed).standard_normal(npix)
    return np.exp(sigma * g - 0.5 * sigma * sigma)


def sum_pixels(nside, J):
    return sum(12 * (nside >> n) ** 2 for n in range(J))


class Clocks:
    """nvidia-smi samples of the SM clock and throttle reasons during a timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *_):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9 and f[1].replace(".", "").isdigit():
                    rows.append(f)
        finally:
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "samples": len(rows),
                "reasons": reasons}


def max_over_ranks(torch, dist, value, device):
    """The largest of the ranks' values, on every rank (the job's time is that
    of its slowest rank); the value itself on one process.  device: "cuda"
    under NCCL, "cpu" under gloo."""
    if not dist:
        return value
    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_seeds(rank, batch):
    """Seeds of the maps rank `rank` holds: rank * batch .. rank * batch + batch - 1
    (replicas: disjoint maps per rank, no exchange between ranks)."""
    return [rank * batch + s for s in range(batch)]


def job_rate(world, units_per_rank, ms):
    """Whole-job throughput: units of all ranks per second of the slowest rank."""
    return world * units_per_rank / (ms / 1e3)


def evaluation_roofline(nside, J, batch, elem, cells_per_row, plan, ms, hbm_gbs, sms, sm_mhz, fp64):
    """Roofline of one forward + VJP of a batch (the scope contract's formula):
    t_roof = max(bytes_alg / HBM, flops_alg / P), with, over the levels n (N_n
    pixels, D_n cells read per wavelet row, c_n coefficients native at n, s the
    field element size, L = 4),
      bytes_alg = sum_n N_n [2 (2 L D_n s + 12) + B s (4 + L (2 + 5 n))]
      flops_alg = B sum_n N_n [6 (2 L D_n) (1 + (n + 1) L) + 24 c_n]
    and P the CUDA-core FMA peak at the maximum SM clock (128 FP32 or 64 FP64
    FMA per clock and SM); frac = t_roof / the measured time."""
    L = 4
    native = [c["native_dg"] for c in plan]
    b = f = 0.0
    for n in range(J):
        N = 12.0 * (nside >> n) ** 2
        D = cells_per_row[n]
        b += N * (2 * (2 * L * D * elem + 12) + batch * elem * (4 + L * (2 + 5 * n)))
        f += batch * N * (6 * (2 * L * D) * (1 + (n + 1) * L) + 24 * native.count(n))
    peak = sms * (64 if fp64 else 128) * 2 * sm_mhz * 1e6
    t_mem, t_fma = b / (hbm_gbs * 1e9), f / peak
    t_roof = max(t_mem, t_fma)
    return {"t_roof_ms": t_roof * 1e3, "ms": ms, "frac": t_roof * 1e3 / ms, "bound": "hbm" if t_mem >= t_fma else "fma",
            "bytes_alg": b, "flops_alg": f, "fma_peak_tflops": peak / 1e12, "hbm_gbs": hbm_gbs}


def time_steps(torch, step, steps, warmup, dist):
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        step()
    b.record()
    torch.cuda.synchronize()
    return max_over_ranks(torch, dist, a.elapsed_time(b), "cuda")


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d["hbm_gbs"], "source": "measured", "sm_max_mhz": d.get("sm_max_mhz")}
    return {"hbm_gbs": 6650.0, "source": "fallback", "sm_max_mhz": None}


def cpu_baseline(nside=1024, J=9):
    """The FP64 CPU oracle (the restatement of the reference's CPU engine) on all
    host cores: one forward + VJP of one lognormal map at (nside, J) -- by
    default the benchmark's own configuration, nside 1024, J = 9 -- timed
    once (the oracle has no warm-up state: its geometry is rebuilt per call
    above its cache budget, as the reference's CPU engine builds its blocks)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    e = oracle.OracleEngine(nside, J, batch=1)
    x = lognormal(0, 12 * nside * nside)
    t0 = time.perf_counter()
    v = e.forward(x)
    e.vjp(2.0 * v)
    dt = time.perf_counter() - t0
    return {"value": 1.0 / dt, "unit": UNIT, "cores": oracle.threads(), "kind": "port",
            "sample": f"one FP64 forward+VJP of one lognormal map at nside {nside}, J={J} ({dt:.1f} s), "
                      f"the benchmark's configuration, timed once"}


def run_reference(args):
    """The reference arm: the CPU oracle on the host cores, at the benchmark's
    configuration (nside 1024, J 9, one FP64 map per evaluation).  One full
    evaluation takes minutes on a CPU, so the arm times one evaluation per
    run whatever --steps asks (``steps`` in the line is the number timed,
    ``steps_requested`` the flag) and runs no warm-up (the oracle keeps no
    state between evaluations).  Under torchrun rank 0 alone runs it."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    b = cpu_baseline(args.nside, args.J)
    value = b["value"]
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": 1, "warmup": 0, "steps_requested": args.steps, "warmup_requested": args.warmup,
            "ms_per_step": 1e3 / value, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"scatcov fwd+vjp nside{args.nside} J{args.J} L4, 1 FP64 map per step "
                                   f"(CPU oracle, all host threads)",
                       "nside": args.nside, "J": args.J, "L": 4, "batch": 1},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": oracle.threads(), "kind": "port",
                             "sample": b["sample"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def family_errors(plan, values, ref):
    """FP32 against FP64 statistics under the 1e-6 family criterion: the worst
    ratio of |v - r| to 1e-6 (max |r| of the coefficient's (family, level,
    map) + |r|), real and imaginary parts apart, and the plain largest
    relative error over the coefficients whose |r| is at least 1e-3 of their
    family scale."""
    fam = np.array([c["family"] for c in plan])
    lev = np.array([c["native_dg"] for c in plan])
    worst = rel = 0.0
    for f in set(fam):
        for n in set(lev):
            sel = (fam == f) & (lev == n)
            if not sel.any():
                continue
            r, v = ref[:, sel], values[:, sel]
            scale = np.max(np.abs(r), axis=1, keepdims=True)
            for part in (np.real, np.imag):
                err = np.abs(part(v) - part(r))
                worst = max(worst, float(np.max(err / (1e-6 * scale + 1e-6 * np.abs(part(r))))))
                big = np.abs(part(r)) >= 1e-3 * scale
                if big.any():
                    rel = max(rel, float(np.max(err[big] / np.abs(part(r))[big])))
    return worst, rel


def patch_workload(nside=512, n=512, seed=3):
    """Centres uniform on the sphere; pixel counts log-uniform in [1024, 65536]
    through R = acos(1 - n Omega_pix / (2 pi)), Omega_pix = 4 pi / (12 nside^2)."""
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    counts = np.exp(rng.uniform(np.log(1024.0), np.log(65536.0), n))
    omega = 4.0 * np.pi / (12.0 * nside * nside)
    radii = np.degrees(np.arccos(1.0 - counts * omega / (2.0 * np.pi)))
    return v, radii


def run_patches(args, torch, dist, world, rank, dev):
    """Forward + VJP of 512 disc patches (nside 512, J 5, L 4, FP32 fields, values
    N(0, 1)): patches per second, device-resident patches and through the host API."""
    import stl_b200
    nside, J = 512, 5
    centres, radii = patch_workload(nside)
    pe = stl_b200.PatchEngine(nside, J, dtype="float32", device=dev.index, autotune=not args.no_autotune)
    t0 = time.perf_counter()
    ids = pe.select(centres, radii)
    sizes = np.array([i.size for i in ids])
    rng = np.random.default_rng(100 + rank)
    patches = [rng.standard_normal(k) for k in sizes]
    x_host = np.concatenate(patches)
    x_dev = torch.tensor(x_host, dtype=torch.float64, device=dev)
    g_dev = torch.empty_like(x_dev)
    ncoeff = pe.ncoeff
    lib = stl_b200.lib()
    vals = np.empty((len(ids), ncoeff), np.complex128)
    cot = np.ascontiguousarray(np.ones((len(ids), ncoeff), np.complex128))
    gen = iter(range(1, 10 ** 9))
    dptr = stl_b200._ptr

    def step_dev():
        g = next(gen)
        torch.cuda.current_stream().synchronize()
        if lib.stlp_patch_forward_device(pe._handle, x_dev.data_ptr(), x_host.size, g, False,
                                         dptr(vals.view(np.float64)), None):
            raise stl_b200._error()
        if lib.stlp_patch_vjp_device(pe._handle, dptr(cot.view(np.float64)), cot.size, g, g_dev.data_ptr()):
            raise stl_b200._error()

    step_dev()  # builds the discs' engines
    build_s = time.perf_counter() - t0
    for _ in range(args.warmup):
        step_dev()
    with Clocks(dev.index) as clk:
        ms = time_steps(torch, step_dev, args.steps, 0, dist)
    clocks = clk.summary()

    g_host = np.empty(x_host.size)  # the gradients' and the statistics' arrays, kept across calls (out=)
    v_host = np.empty((len(ids), pe.ncoeff), np.complex128)
    ones = np.ones_like(v_host)

    def step_host():
        g = next(gen)
        v, _ = pe.forward(patches, moments=False, generation=g, out=v_host)
        pe.vjp(ones, generation=g, out=g_host)

    ms_e2e = time_steps(torch, step_host, max(2, args.steps // 2), 1, dist)
    e2e_steps = max(2, args.steps // 2)
    # Launch overhead of the per-level launches: an engine with CUDA events
    # around every launch (after the timed steps) gives the device time of
    # one step; the rest of the step's time is the device idle between
    # launches, which one persistent kernel would at most recover.
    split = None
    if rank == 0:
        pp = stl_b200.PatchEngine(nside, J, dtype="float32", device=dev.index, autotune=not args.no_autotune,
                                  profile=True)
        pp.select(centres, radii)
        saved = pe
        pe = pp
        for _ in range(2):
            step_dev()
        before = {k["name"]: k["ms"] for k in pp.info()["kernels"]}
        for _ in range(3):
            step_dev()
        torch.cuda.synchronize()
        after = {k["name"]: k["ms"] for k in pp.info()["kernels"]}
        kms = {k: (after[k] - before.get(k, 0.0)) / 3 for k in after}
        busy = sum(kms.values())
        split = {"kernel_ms_per_step": kms, "device_busy_ms_per_step": busy,
                 "idle_fraction": max(0.0, 1.0 - busy / (ms / args.steps)),
                 "split_from": "3 steps of a second engine with CUDA events around every launch"}
        pe = saved
        pp.close()
    # FP32 patches against an FP64 engine on the same discs and values (the
    # 1e-6 family criterion of the headline), after the timed steps
    accuracy = None
    if rank == 0:
        v32, _ = pe.forward(patches, moments=False, generation=next(gen))
        p64 = stl_b200.PatchEngine(nside, J, dtype="float64", device=dev.index, autotune=False)
        p64.select(centres, radii)
        v64, _ = p64.forward(patches, moments=False, generation=1)
        p64.close()
        ratio, rel = family_errors(pe.plan, v32, v64)
        accuracy = {"max_err_ratio": ratio, "max_rel_err": rel,
                    "criterion": "|v32 - v64| <= 1e-6 (max |v64| of the coefficient's family, level and disc) "
                                 "+ 1e-6 |v64|; max_err_ratio <= 1 passes",
                    "reference": "the FP64 disc engine on the same discs and values"}
    if rank == 0:
        b = len(ids)
        line = {"metric": "disc-patch fwd+VJP patches/s (512 ragged discs, nside 512, J=5)",
                "value": world * b * args.steps / (ms / 1e3), "unit": "patches/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic",
                "config": {"workload": "512 disc patches, nside 512, J 5, L 4, FP32 fields, values N(0,1)",
                           "pixels_min": int(sizes.min()), "pixels_max": int(sizes.max()),
                           "pixels_total": int(sizes.sum()), "build_s": build_s,
                           "parallelism": f"replicas x{world}", "launch_overhead": split,
                           "accuracy": accuracy},
                "e2e": {"value": world * b * e2e_steps / (ms_e2e / 1e3), "unit": "patches/s",
                        "h2d_bytes_per_step": int(x_host.size * 8 + cot.size * 16),
                        "d2h_bytes_per_step": int(vals.size * 16 + x_host.size * 8)},
                "clocks": clocks}
        print(json.dumps(line), flush=True)
    pe.close()


def run_cross(args, torch, dist, world, rank, dev):
    """Cross statistics of two channels (config "cross": the cross-only plan) at
    nside 1024, J 9, L 4, FP32 fields, a batch of 2 channel pairs (4 maps):
    channel c of pair b is exp(0.7 g_b + 0.5 e_bc - 1/2) (g, e ~ N(0, 1), seeds
    per rank), the cotangent that of sum |S - S_t|^2 with S_t the statistics of
    pair 0 shifted by a seed.  Forward + VJP evaluations (pairs) per second,
    device-resident and through the host API."""
    import stl_b200
    nside, J, B = args.nside, args.J, 2
    npix = 12 * nside * nside
    eng = stl_b200.NativeEngine(nside, J, batch=B, dtype="float32", device=dev.index, prepare=True, cross=True,
                                autotune=not args.no_autotune)
    rng = np.random.default_rng(500 + rank)
    g = rng.standard_normal((B, 1, npix))
    x_host = np.exp(0.7 * g + 0.5 * rng.standard_normal((B, 2, npix)) - 0.5)
    x = torch.tensor(x_host, dtype=torch.float32, device=dev)
    xt = torch.tensor(np.roll(x_host, 1, axis=0), dtype=torch.float32, device=dev)
    target, _ = eng.forward_tensor(xt, generation=1)
    grad = torch.empty_like(x)
    gen = iter(range(10, 10 ** 9))

    def step():
        k = next(gen)
        values, _ = eng.forward_tensor(x, generation=k)
        eng.vjp_tensor(2.0 * (values - target), grad, generation=k)

    for _ in range(args.warmup):
        step()
    with Clocks(dev.index) as clk:
        ms = time_steps(torch, step, args.steps, 0, dist)
    clocks = clk.summary()
    eng.profile(on=True, reset=True)
    step()
    torch.cuda.synchronize()
    stats = eng.kernel_stats()
    eng.profile(on=False, reset=False)

    g_host = np.empty(x_host.size)  # the gradients' array, kept across calls (vjp out=)

    def step_host():
        k = next(gen)
        values, _ = eng.forward(x_host, generation=k)
        eng.vjp(2.0 * (values - target), generation=k, out=g_host)

    e2e_steps = max(2, args.steps // 2)
    ms_e2e = time_steps(torch, step_host, e2e_steps, 1, dist)
    if rank == 0:
        line = {"metric": f"cross S1-S4 fwd+VJP evals/s (two channels, nside {nside}, J={J}, FP32)",
                "value": job_rate(world, B * args.steps, ms), "unit": "evals/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": f"cross terms of 2 channels, nside {nside}, J {J}, L 4, 2 pairs (4 maps), FP32 fields",
                           "ncoeff": eng.ncoeff, "parallelism": f"replicas x{world}",
                           "kernels_ms_per_step": {k: v["ms"] for k, v in stats.items()}},
                "e2e": {"value": job_rate(world, B * e2e_steps, ms_e2e), "unit": "evals/s",
                        "h2d_bytes_per_step": int(x_host.nbytes), "d2h_bytes_per_step": int(x_host.nbytes)},
                "clocks": clocks}
        print(json.dumps(line), flush=True)
    eng.close()


def run_spin(args, torch, dist, world, rank, dev):
    """Spin-2 statistics (the (Q, U) front end feeding the engine) at nside 1024,
    J 9, L 4, FP32 fields, a batch of 2 (Q, U) maps (4 engine maps: chi_E, chi_B
    of each), scalar pyramid, stencil kernel 5: Q + iU = (g1 + i g2) exp(0.5 g0)
    (g ~ N(0, 1), seeds per rank), the cotangent that of sum |S - S_t|^2 with S_t
    from other seeds.  Forward + VJP evaluations ((Q, U) maps) per second; the
    front end's share is the step's time minus that of a scalar engine of 4 maps
    on the same device (same statistics work)."""
    import stl_b200
    nside, J, B = args.nside, args.J, 2
    npix = 12 * nside * nside
    pyramid = "scalar"
    eng = stl_b200.NativeEngine(nside, J, batch=B, dtype="float32", device=dev.index, spin=2, spin_pyramid=pyramid,
                                autotune=not args.no_autotune)
    t0 = time.perf_counter()
    eng.prepare()
    build_s = time.perf_counter() - t0

    def maps(seed):
        rng = np.random.default_rng(seed)
        g = rng.standard_normal((B, 3, npix))
        amp = np.exp(0.5 * g[:, 0])
        return np.stack([g[:, 1] * amp, g[:, 2] * amp], 1)

    x_host = maps(700 + rank)
    x = torch.tensor(x_host, dtype=torch.float32, device=dev)
    target, _ = eng.forward_tensor(torch.tensor(maps(900 + rank), dtype=torch.float32, device=dev), generation=1)
    grad = torch.empty_like(x)
    gen = iter(range(10, 10 ** 9))

    def step():
        k = next(gen)
        values, _ = eng.forward_tensor(x, generation=k)
        eng.vjp_tensor(2.0 * (values - target), grad, generation=k)

    for _ in range(args.warmup):
        step()
    with Clocks(dev.index) as clk:
        ms = time_steps(torch, step, args.steps, 0, dist)
    clocks = clk.summary()

    g_host = np.empty(x_host.size)  # the gradients' array, kept across calls (vjp out=)

    def step_host():
        k = next(gen)
        values, _ = eng.forward(x_host, generation=k)
        eng.vjp(2.0 * (values - target), generation=k, out=g_host)

    e2e_steps = max(2, args.steps // 2)
    ms_e2e = time_steps(torch, step_host, e2e_steps, 1, dist)
    info = eng.info()
    eng.close()
    del x, grad
    torch.cuda.empty_cache()
    # the same statistics of 4 scalar maps: the front end's cost is the difference
    sc = stl_b200.NativeEngine(nside, J, batch=2 * B, dtype="float32", device=dev.index, prepare=True,
                               autotune=not args.no_autotune)
    xs = torch.tensor(np.abs(x_host.reshape(2 * B, npix)) + 1.0, dtype=torch.float32, device=dev)
    ts, _ = sc.forward_tensor(xs, generation=1)
    gs = torch.empty_like(xs)

    def step_scalar():
        k = next(gen)
        values, _ = sc.forward_tensor(xs, generation=k)
        sc.vjp_tensor(2.0 * (values - ts), gs, generation=k)

    ms_scalar = time_steps(torch, step_scalar, args.steps, args.warmup, dist)
    sc.close()
    if rank == 0:
        line = {"metric": f"spin-2 S1-S4 fwd+VJP evals/s ((Q, U) maps, nside {nside}, J={J}, FP32)",
                "value": job_rate(world, B * args.steps, ms), "unit": "evals/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": f"spin 2 ({pyramid} pyramid, stencil 5), nside {nside}, J {J}, L 4, "
                                       f"{B} (Q, U) maps (4 engine maps), FP32 fields",
                           "ncoeff": info["plan"].__len__(), "parallelism": f"replicas x{world}",
                           "spin_operator_bytes": info.get("spin_bytes"), "spin_build_s": build_s,
                           "scalar_4_maps_ms_per_step": ms_scalar / args.steps,
                           "front_end_ms_per_step": (ms - ms_scalar) / args.steps},
                "e2e": {"value": job_rate(world, B * e2e_steps, ms_e2e), "unit": "evals/s",
                        "h2d_bytes_per_step": int(x_host.nbytes), "d2h_bytes_per_step": int(x_host.nbytes)},
                "clocks": clocks}
        print(json.dumps(line), flush=True)


def run_synthesis(args, torch, dist, world, rank, dev):
    """L-BFGS synthesis at nside 1024, J 9, L 4, m = 10, FP32 engine: target the
    lognormal map of seed 7, start from N(0, 1) (seed 8) rescaled to the target's
    mean and standard deviation, loss sum_k |S_k - T_k|^2 / var_k with var_k the
    target's variance of coefficient k; the iterate, gradients and curvature pairs
    stay in device memory (stlp_synthesize_device).  A step is one L-BFGS
    iteration; the timed call runs 200 (or --steps, if larger)."""
    import stl_b200
    nside, J, B = 1024, 9, 1
    npix = 12 * nside * nside
    eng = stl_b200.NativeEngine(nside, J, batch=B, dtype="float32", device=dev.index, prepare=True,
                                autotune=not args.no_autotune)
    xt = lognormal(7 + 1000 * rank, npix)[None]
    target, var_t = eng.forward(xt, moments=True)
    v = var_t.reshape(-1)
    w = 1.0 / np.maximum(v, 1e-12 * v.max())
    g0 = np.random.default_rng(8 + 1000 * rank).standard_normal(npix)
    x0 = ((g0 - g0.mean()) / g0.std() * xt.std() + xt.mean())[None]
    iters = max(200, args.steps)
    # warm-up: a short run from the same start (operators, pools, clocks)
    xw = torch.tensor(x0, dtype=torch.float64, device=dev)
    eng.synthesize(xw, target, weights=w, options={"max_iter": max(3, args.warmup), "history_size": 10})
    opts = {"max_iter": iters, "history_size": 10, "max_eval": iters * 2}
    x_dev = torch.tensor(x0, dtype=torch.float64, device=dev)
    res = {}

    def run_dev():
        res["n"], res["losses"] = eng.synthesize(x_dev, target, weights=w, options=opts)

    with Clocks(dev.index) as clk:
        ms = time_steps(torch, run_dev, 1, 0, dist)
    clocks = clk.summary()
    x_pin = torch.tensor(x0, dtype=torch.float64).pin_memory()
    out_pin = torch.empty_like(x_pin).pin_memory()

    def run_e2e():
        xd = x_pin.to(dev, non_blocking=True)
        eng.synthesize(xd, target, weights=w, options=opts)
        out_pin.copy_(xd, non_blocking=True)
        torch.cuda.synchronize(dev)

    ms_e2e = time_steps(torch, run_e2e, 1, 0, dist)
    if rank == 0:
        losses = res["losses"]
        line = {"metric": "L-BFGS synthesis iterations/s (nside 1024, J=9, m=10, FP32 engine, FP64 L-BFGS)",
                "value": world * iters / (ms / 1e3), "unit": "iterations/s", "n_gpus": world, "steps": iters,
                "warmup": max(3, args.warmup), "ms_per_step": ms / iters, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "synthesis nside1024 J9 L4 m10, lognormal target seed 7, start seed 8",
                           "evaluations": res["n"], "loss_first": float(losses[0]),
                           "loss_last": float(losses[-1]), "parallelism": f"replicas x{world}",
                           "graph": "iterations 2 on: one CUDA graph launch each (curvature pair, two-loop "
                                    "recursion, first line-search trial, objective and VJP); the host runs "
                                    "the strong Wolfe test on one copy of scalars"},
                # the maps cross PCIe once per run (start in, result out): per iteration
                "e2e": {"value": world * iters / (ms_e2e / 1e3), "unit": "iterations/s",
                        "h2d_bytes_per_step": int(npix * 8 / iters), "d2h_bytes_per_step": int(npix * 8 / iters)},
                "clocks": clocks}
        print(json.dumps(line), flush=True)
    eng.close()


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    import stl_b200

    if args.workload in ("patches", "synthesis", "cross", "spin"):
        run = {"patches": run_patches, "synthesis": run_synthesis, "cross": run_cross, "spin": run_spin}[args.workload]
        run(args, torch, dist, world, rank, torch.device("cuda", local if world > 1 else 0))
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    nside, J, B = args.nside, args.J, args.batch
    npix = 12 * nside * nside
    dev = torch.device("cuda", local if world > 1 else 0)

    # -- FP32 batched: the headline -------------------------------------------
    eng = stl_b200.NativeEngine(nside, J, batch=B, dtype="float32", device=dev.index, prepare=True,
                                autotune=not args.no_autotune)
    seeds = rank_seeds(rank, B)
    x_host = np.stack([lognormal(s, npix) for s in seeds])
    x = torch.tensor(x_host, dtype=torch.float32, device=dev)
    # target statistics S_t: the FP32 engine on the map of seed 100 (replicated over the batch)
    xt = torch.tensor(np.stack([lognormal(100, npix)] * B), dtype=torch.float32, device=dev)
    target, _ = eng.forward_tensor(xt, generation=1)
    grad = torch.empty_like(x)
    gen = iter(range(10, 10 ** 9))

    def step32():
        g = next(gen)
        values, _ = eng.forward_tensor(x, generation=g)
        eng.vjp_tensor(2.0 * (values - target), grad, generation=g)

    if args.profile_step:
        # one step for a profiler's launch list: its launches are the last ones
        # of the process; the line gives their count and the classes' calls and
        # algorithmic bytes, to match a capture's launches to the classes
        eng.profile(on=False, reset=True)
        step32()
        torch.cuda.synchronize()
        info = eng.info()
        stats = {k["name"]: {"launches": k["launches"], "calls": k["calls"], "bytes": k["bytes"]}
                 for k in info["kernels"]}
        print(json.dumps({"profile_step": {"nside": nside, "J": J, "batch": B,
                                           "launches": sum(v["launches"] for v in stats.values()),
                                           "kernels": stats, "mean_cells_per_row": info["mean_cells_per_row"],
                                           "tile_heights": info["tile_heights"]}}))
        eng.close()
        return
    for _ in range(args.warmup):
        step32()
    eng.profile(on=False, reset=True)
    with Clocks(dev.index) as clk:
        ms32 = time_steps(torch, step32, args.steps, 0, dist)
    clocks = clk.summary()
    # the split per kernel class: CUDA events around every launch, in steps of
    # their own after the timed region (the events are not in the timed steps)
    prof_steps = 3
    eng.profile(on=True, reset=True)
    for _ in range(prof_steps):
        step32()
    torch.cuda.synchronize()
    stats = eng.kernel_stats()
    eng.profile(on=False, reset=False)
    value = job_rate(world, B * args.steps, ms32)
    launches = sum(s["launches"] for s in stats.values()) * args.steps // prof_steps
    peaks = load_peaks()
    props = torch.cuda.get_device_properties(dev)
    sm_max = peaks.get("sm_max_mhz") or 1965.0
    info32 = eng.info()
    eval_roof = {"fp32_batched": evaluation_roofline(nside, J, B, 4, info32["mean_cells_per_row"], eng.plan,
                                                     ms32 / args.steps, peaks["hbm_gbs"], props.multi_processor_count,
                                                     sm_max, False)}

    # roofline of the dominant kernel class, timed live with CUDA events
    dom = max(stats.values(), key=lambda s: s["ms"])
    achieved = dom["bytes"] / (dom["ms"] / 1e3) / 1e9 if dom["ms"] > 0 else 0.0
    # DRAM traffic per call of the class: its measured DRAM / algorithmic ratio
    # (single-launch capture of the level-0 call, profiles/traffic.json) times
    # the class's algorithmic bytes per call here
    calls = dom["calls"] / prof_steps
    traffic, traffic_basis = None, None
    tp = ROOT / "profiles" / "traffic.json"
    if tp.exists() and calls > 0:
        t = json.loads(tp.read_text()).get(dom["name"])
        if t:
            traffic = t["dram_over_algorithmic"] * dom["bytes"] / prof_steps / calls
            traffic_basis = (f"DRAM bytes per call: {t['dram_over_algorithmic']} (DRAM / algorithmic bytes of "
                             f"{t['call']}, profiles/{t['profile']}) x the class's algorithmic bytes per call")
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": traffic, "traffic_basis": traffic_basis,
                "kernel": dom["name"], "calls_per_step": calls, "algorithmic_bytes_per_call":
                    dom["bytes"] / prof_steps / calls if calls else None,
                "launches_per_step": dom["launches"] / prof_steps, "ms_per_step": dom["ms"] / prof_steps,
                "peak_source": peaks["source"],
                "fp32_tflops": dom["flops"] / (dom["ms"] / 1e3) / 1e12 if dom["ms"] > 0 else 0.0,
                "all_kernels_ms_per_step": {k: s["ms"] / prof_steps for k, s in stats.items()},
                "split_from": f"{prof_steps} steps with CUDA events around every launch, after the timed steps"}

    # -- end to end through the reference-facing host API ---------------------
    g_host = np.empty_like(x_host)  # the caller's gradient buffer, reused (vjp's out=)

    def step_e2e():
        g = next(gen)
        values, _ = eng.forward(x_host, generation=g)
        eng.vjp(2.0 * (values - target), generation=g, out=g_host)

    ms_e2e = time_steps(torch, step_e2e, max(2, args.steps // 2), 1, dist)
    e2e_steps = max(2, args.steps // 2)
    ncoeff = eng.ncoeff
    # statistics and gradients of the batch, for the accuracy check against FP64
    g_acc = next(gen)
    v32, _ = eng.forward_tensor(x, generation=g_acc)
    eng.vjp_tensor(2.0 * (v32 - target), grad, generation=g_acc)
    g32 = grad.double().cpu().numpy()
    plan = eng.plan
    e2e = {"value": world * B * e2e_steps / (ms_e2e / 1e3), "unit": UNIT,
           "h2d_bytes_per_step": B * npix * 8 + B * ncoeff * 16, "d2h_bytes_per_step": B * ncoeff * 16 + B * npix * 8,
           "api": "stlp_forward + stlp_vjp (host f64 buffers, the gradient into a reused out= array; the FP32 "
                  "gradient crosses PCIe as floats and is widened by the host threads)"}
    eng.close()
    del x, xt, grad
    torch.cuda.empty_cache()

    # -- FP64 plain single map --------------------------------------------------
    fp64 = None
    fp64_split = None
    accuracy = None
    if not args.skip_fp64:
        e64 = stl_b200.NativeEngine(nside, J, batch=1, dtype="float64", device=dev.index, prepare=True,
                                      autotune=not args.no_autotune)
        x64 = torch.tensor(x_host[:1], dtype=torch.float64, device=dev)
        # the target of the FP32 run, on the same FP32-rounded map
        t64, _ = e64.forward_tensor(torch.tensor(lognormal(100, npix)[None], dtype=torch.float32, device=dev).double(),
                                    generation=1)
        g64 = torch.empty_like(x64)

        def step64():
            g = next(gen)
            values, _ = e64.forward_tensor(x64, generation=g)
            e64.vjp_tensor(2.0 * (values - t64), g64, generation=g)

        ms64 = time_steps(torch, step64, args.steps, args.warmup, dist)
        fp64 = world * args.steps / (ms64 / 1e3)
        # its class split, from 3 profiled steps after the timed ones
        e64.profile(on=True, reset=True)
        for _ in range(3):
            step64()
        torch.cuda.synchronize()
        fp64_split = {k: v["ms"] / 3 for k, v in e64.kernel_stats().items()}
        e64.profile(on=False, reset=False)
        # the FP32 batch against FP64 on the same maps (after the timed steps):
        # every coefficient under the 1e-6 family criterion, and the gradients
        v64 = np.empty_like(v32)
        grad_err = 0.0
        for b in range(B):
            k = next(gen)
            xb = torch.tensor(x_host[b:b + 1], dtype=torch.float32, device=dev).double()
            vb, _ = e64.forward_tensor(xb, generation=k)
            v64[b] = vb[0]
            e64.vjp_tensor(2.0 * (vb - t64), g64, generation=k)
            gb = g64.cpu().numpy()[0]
            grad_err = max(grad_err, float(np.max(np.abs(g32[b] - gb)) / np.max(np.abs(gb))))
        ratio, rel = family_errors(plan, v32, v64)
        accuracy = {"max_err_ratio": ratio, "max_rel_err": rel, "grad_rel_err": grad_err,
                    "criterion": "|v32 - v64| <= 1e-6 (max |v64| of the coefficient's family, level and map) "
                                 "+ 1e-6 |v64|, real and imaginary parts; max_err_ratio <= 1 passes",
                    "reference": "the engine's FP64 path on the same FP32-rounded maps (the FP64 path is pinned "
                                 "to the CPU oracle and the reference's fixtures)"}
        eval_roof["fp64_plain"] = evaluation_roofline(nside, J, 1, 8, e64.info()["mean_cells_per_row"], e64.plan,
                                                      ms64 / args.steps, peaks["hbm_gbs"],
                                                      props.multi_processor_count, sm_max, True)
        e64.close()
        del x64, g64
        torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        cpu = cpu_baseline(nside, J)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms32 / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": f"scatcov fwd+vjp nside{nside} J{J} L4 batch{B} fp32 (sums fp64)",
                           "nside": nside, "J": J, "L": 4, "batch_per_gpu": B, "ncoeff": ncoeff,
                           "maps": "lognormal exp(g-1/2), numpy default_rng seeds rank*B..rank*B+B-1",
                           "l2": "inputs larger than L2 (fields and operators of tens of GB per step)",
                           "parallelism": f"replicas x{world}",
                           "fp64_plain_evals_per_s": fp64,
                           "fp64_plain_kernels_ms_per_step": fp64_split,
                           "fp32_batched_over_fp64_plain": (value / world) / (fp64 / world) if fp64 else None,
                           "evaluation_roofline": eval_roof, "accuracy": accuracy,
                           "max_err_ratio": accuracy["max_err_ratio"] if accuracy else None},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
                "gpu_launches": launches}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

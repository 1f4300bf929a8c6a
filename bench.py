"""Benchmark of the compact-difference hot path on B200.

Workload (one "step"): the cd10 periodic first derivative, the cd10 periodic
second derivative and the cf90 periodic filter along x, y and z -- 9 operator
applications -- on a 512^3 FP64 field (random-phase |k|^-5/3 synthesis, seeded;
synthetic data standing in for solver fields).  Metric: Gpts/s = output points
of all operator applications per second (16 algorithmic bytes per point: read
f, write df).  Inputs (1 GiB) exceed L2 (126 MB), so no flush is needed
between iterations.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU (torchrun): every rank processes its own field (lines and fields are
independent, no data-path collective): weak scaling, value = all ranks' points
/ max-over-ranks time.

The JSON line carries: value (device-resident), e2e (the same metric through
the host-buffer C-ABI call pado_apply_host_terms -- one upload of the field,
the nine results downloaded -- copies included; the per-operator host call
pado_apply_host beside it), roofline of the
line kernels (CUDA events, algorithmic bytes / kernel time, against the
measured HBM copy bandwidth), cpu_baseline (the oracle -- the C restatement of
the reference -- on the host cores), clocks sampled during the timed region,
the number of library kernel launches in the timed region, and "extensions":
the batched launch against the per-field loop on 96 uneven fields, and the
adjoint against the forward operators on 256^3 (see extensions()).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N = 512
OPS = [("cd10", 1), ("cd10", 2), ("cf90", 0)]  # (scheme, kind)
METRIC = "Gpts/s cd06/cd10 dd1-3 @512^3 FP64 (%HBM peak); batched, fwd+adjoint vs plain"
BYTES_PER_PT = 16
CONFIG = {"workload": "cd10 d1 + cd10 d2 + cf90, periodic, x/y/z on 512^3 FP64 (9 operator applications per step)",
          "n": N, "operators_per_step": 9, "l2": "inputs larger than L2 (1 GiB field)"}


def measured_peaks() -> tuple[float, str]:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic() -> float | None:
    """DRAM bytes per 512^3 launch of the streaming kernel from the committed ncu
    summary (profiles/stream_kernel_512cube.md, line 'traffic_bytes_per_launch: X')."""
    p = os.path.join(ROOT, "profiles", "stream_kernel_512cube.md")
    try:
        with open(p) as fh:
            for line in fh:
                if line.strip().startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":", 1)[1].split()[0])
    except Exception:
        pass
    return None


class ClockSampler:
    """Samples the SM clock, its maximum and the clock-event (throttle) reasons
    while running: NVML read directly every 10 ms (so that a timed region of
    tens of milliseconds still gets samples), else nvidia-smi every 100 ms.
    Reads only; changes no setting of the GPU."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.nvml = None
        self.stop = threading.Event()
        self.lines: list[str] = []
        self.samples: list[tuple[float, float, set]] = []

    def _nvml_handle(self):
        """NVML handle of CUDA device `index`, found by its PCI bus id; returns
        (module, handle, bus id).  Without the bus id the NVML index is used
        only when CUDA_VISIBLE_DEVICES does not renumber the devices."""
        import pynvml
        import torch

        pynvml.nvmlInit()
        bus = None
        try:
            prop = torch.cuda.get_device_properties(self.index)
            bus = f"{prop.pci_domain_id:08x}:{prop.pci_bus_id:02x}:{prop.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus), bus
        except Exception:
            if os.environ.get("CUDA_VISIBLE_DEVICES"):
                raise
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index), bus

    def _poll(self, nv, h, mx):
        bits = [getattr(nv, "nvmlClocksEventReason" + k, getattr(nv, "nvmlClocksThrottleReason" + k, 0))
                for k in ("HwSlowdown", "HwThermalSlowdown", "SwThermalSlowdown", "SwPowerCap")]
        reasons_fn = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons",
                             getattr(nv, "nvmlDeviceGetCurrentClocksThrottleReasons", None))
        while not self.stop.is_set():
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                act = int(reasons_fn(h)) if reasons_fn else 0
                self.samples.append((sm, mx, {n for n, b in zip(self.NAMES, bits) if b and act & b}))
            except Exception:
                pass
            time.sleep(0.01)

    def __enter__(self):
        self.bus = None
        try:
            nv, h, self.bus = self._nvml_handle()
            mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))  # fails here, not in the thread
            self.nvml = nv
            self.t = threading.Thread(target=self._poll, args=(nv, h, mx), daemon=True)
            self.t.start()
            return self
        except Exception:
            if self.nvml is None:
                try:
                    import pynvml

                    pynvml.nvmlShutdown()
                except Exception:
                    pass
            self.nvml = None
        try:
            dev = self.bus if self.bus else str(self.index)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", dev, f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # nvidia-smi takes a moment to start: wait for its first sample
            t0 = time.perf_counter()
            while not self.lines and time.perf_counter() - t0 < 5.0:
                time.sleep(0.02)
            self.lines.clear()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        self.stop.set()
        if self.nvml:
            self.t.join(timeout=1.0)
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        for a, b, r in self.samples:
            sm.append(a)
            mx.append(b)
            reasons |= r
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(self.NAMES, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvml" if self.samples else "nvidia-smi",
                "pci_bus_id": self.bus}


def make_field(seed: int) -> np.ndarray:
    from tests.fields import spectrum53

    return spectrum53((N, N, N), seed)


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def _cpu_rate(f: np.ndarray, threads: int, budget_s: float, max_ops: int = 9) -> tuple[float, int]:
    """Gpts/s of the oracle (the reference's Release flags) over the step's
    operator applications, as many as fit the budget (at least one)."""
    import oracle

    dx = 2 * np.pi / N
    ops = [oracle.OracleOp({"cd10": oracle.CD10, "cf90": oracle.CF90}[s], N, dx, True, fast=True) for s, _ in OPS]
    out = np.empty_like(f)
    t0 = time.perf_counter()
    done = []
    while len(done) < max_ops and (not done or time.perf_counter() - t0 < budget_s):
        i = len(done)
        op, (s, kind) = ops[i % 3], OPS[i % 3]
        axis = i // 3 + 1
        ts = time.perf_counter()
        op.apply(kind, axis, f, N, N, 0, 0, nthreads=threads, out=out)
        done.append(time.perf_counter() - ts)
    return len(done) * N ** 3 / sum(done) / 1e9, len(done)


def cpu_baseline(f: np.ndarray, threads: int, budget_s: float = 20.0) -> dict:
    """The oracle built with the reference's Release flags on the host cores:
    all cores (OpenMP over independent lines, a stand-in for the reference's
    MPI ranks) and one thread (the reference's per-rank behaviour: its
    compact-scheme modules have no OpenMP)."""
    v_all, n_all = _cpu_rate(f, threads, budget_s)
    v_one, n_one = _cpu_rate(f, 1, budget_s / 2, max_ops=1)
    return {"value": v_all, "unit": "Gpts/s", "cores": threads, "kind": "port", "cpu_model": cpu_model(),
            "threads_all": {"value": v_all, "threads": threads, "applications": n_all},
            "threads_1": {"value": v_one, "threads": 1, "applications": n_one},
            "sample": f"{n_all} of the 9 operator applications on the 512^3 field with {threads} threads, "
                      f"{n_one} with 1 thread (oracle, -O3 -ffast-math -march=x86-64-v3, OpenMP)"}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    f = make_field(7)
    per_step = []
    for s in range(args.warmup + args.steps):
        cb = cpu_baseline(f, threads, budget_s=1e9 if s >= args.warmup else 30.0)
        if s >= args.warmup:
            per_step.append(cb["value"])
    v = statistics.median(per_step)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Gpts/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 9 * N ** 3 / (v * 1e9) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(CONFIG),
            "cpu_baseline": {"value": v, "unit": "Gpts/s", "cores": threads, "kind": "port",
                             "sample": "the full 9-operator step on the 512^3 field per timed step "
                                       "(oracle = C restatement of the reference; the Fortran reference "
                                       "cannot be built: no Fortran compiler in the image)"},
            "e2e": {"value": v, "unit": "Gpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def extensions() -> dict:
    """The two extensions' own comparisons, each timed with CUDA events after
    warm-up (inputs larger than L2):

    * batched: 96 FP64 fields with dimensions drawn (seeded) from {32, ..., 384},
      total <= 4 GiB, each cd06 or cd10, periodic or bounded, along a random
      axis; one persistent launch replayed from a CUDA graph (tiles autotuned)
      against the per-field loop of launches;
    * adjoint: L = 0.5 ||D_x^cd10 u + D_z^cd06,bounded u - g||^2 on 256^3: the
      two forward operators against their two adjoints (the backward pass).
    """
    import torch

    import padeops_b200 as pb
    from padeops_b200.batch import Batch
    from padeops_b200.tune import tune_batch

    def ev_ms(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    rng = np.random.default_rng(4)
    dims = (32, 48, 64, 96, 128, 192, 256, 384)
    while True:
        shapes = [tuple(int(v) for v in rng.choice(dims, 3)) for _ in range(96)]
        if sum(a * b * c for a, b, c in shapes) * 8 <= 4 * 2 ** 30:
            break
    items, pts = [], 0
    gen = torch.Generator(device="cuda").manual_seed(4)
    for sh in shapes:
        scheme, periodic, axis = int(rng.integers(2)), bool(rng.integers(2)), int(rng.integers(1, 4))
        n = sh[3 - axis]
        op = (pb.cd06 if scheme == 0 else pb.cd10)()
        assert op.init(n, 2 * np.pi / n if periodic else 1.0 / (n - 1), periodic, 0, 0) == 0
        fb = torch.randn(sh, dtype=torch.float64, device="cuda", generator=gen)
        items.append((op, 1, axis, fb, torch.empty_like(fb), 0, 0))
        pts += fb.numel()
    batch = Batch(items)
    lines, per_sm, branches, _ = tune_batch(batch, reps=3)
    loop_ms = ev_ms(batch.run_loop)
    graph_ms = ev_ms(batch.run_graph)
    batched = {"fields": len(items), "points": pts, "graph_ms": round(graph_ms, 3), "loop_ms": round(loop_ms, 3),
               "speedup_vs_loop": round(loop_ms / graph_ms, 3), "graph_gpts": round(pts / graph_ms / 1e6, 1),
               "tuned": {"lines": lines, "ctas_per_sm": per_sm, "graph_branches": branches},
               "data": "seeded normal fields (timing only)"}
    batch.destroy()
    del items

    n = 256
    u = torch.randn(n ** 3, dtype=torch.float64, device="cuda", generator=gen)
    o1, o2 = torch.empty_like(u), torch.empty_like(u)
    dx_op, dz_op = pb.cd10(), pb.cd06()
    assert dx_op.init(n, 2 * np.pi / n, True, 0, 0) == 0 and dz_op.init(n, 1.0 / (n - 1), False, 0, 0) == 0
    fwd_ms = ev_ms(lambda: (dx_op.apply(1, 1, u, o1, n, n), dz_op.apply(1, 3, u, o2, n, n)))
    adj_ms = ev_ms(lambda: (dx_op.apply(1, 1, u, o1, n, n, adjoint=True), dz_op.apply(1, 3, u, o2, n, n, adjoint=True)))
    adjoint = {"workload": "D_x^cd10 (periodic) + D_z^cd06 (bounded) on 256^3", "fwd_ms": round(fwd_ms, 4),
               "adjoint_ms": round(adj_ms, 4), "adjoint_over_forward": round(adj_ms / fwd_ms, 3)}
    del u, o1, o2
    torch.cuda.empty_cache()
    return {"batched": batched, "adjoint": adjoint, "field_ops": field_operators(ev_ms, gen)}


def field_operators(ev_ms, gen) -> dict:
    """The field operators of operators.F90 / cgrid%laplacian on 512^3 (cd10
    periodic x, y; cd10 bounded z), each term summed into its output inside
    the kernels.  Algorithmic bytes per output point: a stored term 16 (read
    f, write df), an accumulated term 24 (read f, read and write df), so
    gradient 3 x 16 (three outputs), laplacian and divergence 16 + 24 + 24,
    curl 3 x (16 + 24).  Plus the laplacian of a pinned host field through
    pado_apply_host_terms (one upload, one download)."""
    import torch

    import padeops_b200 as pb
    from padeops_b200 import field_ops

    n = N
    dx, dz = 2 * np.pi / n, 1.0 / (n - 1)
    der = pb.Derivatives()
    der.init(n, n, n, dx, dx, dz, True, True, False, "cd10", "cd10", "cd10")
    u, v, w = (torch.randn((n, n, n), dtype=torch.float64, device="cuda", generator=gen) for _ in range(3))
    o = [torch.empty_like(u) for _ in range(3)]
    cu = torch.stack(o)  # (3, n, n, n)
    del o
    pts = n ** 3
    cases = {
        "gradient": (lambda: field_ops.gradient(der, u, cu[0], cu[1], cu[2]), 3 * pts, 48),
        "laplacian": (lambda: field_ops.laplacian(der, u, cu[0]), pts, 64),
        "divergence": (lambda: field_ops.divergence(der, u, v, w, cu[0]), pts, 64),
        "curl": (lambda: field_ops.curl(der, u, v, w, cu), 3 * pts, 120),
    }
    out = {"workload": "cd10 periodic x/y, cd10 bounded z, 512^3 FP64"}
    for name, (fn, out_pts, bpt) in cases.items():
        ms = ev_ms(fn)
        out[name] = {"ms": round(ms, 3), "bytes_per_point": bpt, "gbs": round(pts * bpt / (ms / 1e3) / 1e9, 1),
                     "gpts_out": round(out_pts / ms / 1e6, 1)}
    hf = u.cpu().pin_memory()
    hl = torch.empty_like(hf).pin_memory()
    field_ops.laplacian_host(der, hf, hl)
    t0 = time.perf_counter()
    reps = 2
    for _ in range(reps):
        field_ops.laplacian_host(der, hf, hl)
    el = (time.perf_counter() - t0) / reps
    out["laplacian_host"] = {"ms": round(el * 1e3, 2), "gpts": round(pts / el / 1e9, 2),
                             "h2d_bytes": pts * 8, "d2h_bytes": pts * 8,
                             "path": "pado_apply_host_terms (pinned): one upload, 3 terms, one download"}
    del u, v, w, cu, hf, hl
    der.destroy()
    torch.cuda.empty_cache()
    return out


def run_gpu(args) -> None:
    import torch

    import padeops_b200 as pb

    from padeops_b200 import dist as pdist

    rank, world, local = pdist.world()
    torch.cuda.set_device(local)
    dist = pdist.init("nccl")

    dx = 2 * np.pi / N
    f_host = make_field(7 + rank)
    f = torch.from_numpy(f_host).cuda()
    df = torch.empty_like(f)
    ops = {}
    for s, _ in OPS:
        op = pb.cd10() if s == "cd10" else pb.cf90()
        assert (op.init(N, dx, True, 0, 0) if s == "cd10" else op.init(N, True)) == 0
        ops[s] = op
    plan = [(ops[s], kind, axis) for axis in (1, 2, 3) for s, kind in OPS]
    stream = torch.cuda.current_stream()

    def step(events=None):
        for i, (op, kind, axis) in enumerate(plan):
            if events is not None:
                events[i][0].record(stream)
            op.apply(kind, axis, f, df, N, N, 0, 0)
            if events is not None:
                events[i][1].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ev = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in plan]
          for _ in range(args.steps)]
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = pb.launch_count()
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        start.record(stream)
        for k in range(args.steps):
            step(ev[k])
        stop.record(stream)
        torch.cuda.synchronize()
    launches = pb.launch_count() - launches0
    ms = pdist.max_over_ranks(start.elapsed_time(stop), dist, "cuda")
    value = pdist.weak_scaling_rate(9 * N ** 3 * args.steps, world, ms / 1e3) / 1e9
    kern_ms = [a.elapsed_time(b) for row in ev for a, b in row]
    per_op = {}
    for i, (op, kind, axis) in enumerate(plan):
        name = f"{type(op).__name__}_{'d1' if kind == 1 else ('d2' if kind == 2 else 'filter')}_axis{axis}"
        t_op = statistics.mean(ev[k][i][0].elapsed_time(ev[k][i][1]) for k in range(args.steps))
        per_op[name] = round(N ** 3 * BYTES_PER_PT / (t_op / 1e3) / 1e9, 1)
    avg_launch_ms = statistics.mean(kern_ms)
    peak, peak_kind = measured_peaks()
    achieved = N ** 3 * BYTES_PER_PT / (avg_launch_ms / 1e3) / 1e9

    # end to end: host buffers through the C ABI host calls, copies included.
    # The step's nine operators all read the same field, so the step is one
    # pado_apply_host_terms call: f uploaded once, the nine results computed
    # on the device and each downloaded to its own host buffer while the next
    # is computed.  The per-operator host call (pado_apply_host, f uploaded
    # for every operator) is reported beside it.
    e2e = None
    if rank == 0 or world > 1:
        from padeops_b200.field_ops import apply_host_terms

        field_bytes = N ** 3 * 8
        e2e_steps = max(1, min(args.steps, 3))
        hf = torch.from_numpy(f_host).pin_memory()
        # nine pinned result buffers per rank (all ranks of a node pin theirs
        # at once): only when they fit in half the host's available memory,
        # else the per-operator host call alone, with one result buffer
        try:
            import psutil

            avail = psutil.virtual_memory().available
        except Exception:  # noqa: BLE001 -- no psutil: assume room for one rank's buffers
            avail = 4 * len(plan) * field_bytes
        local = int(os.environ.get("LOCAL_WORLD_SIZE", world))
        terms_path = len(plan) * field_bytes * local <= avail // 2
        hdf = torch.empty_like(hf).pin_memory()

        def per_operator():
            for op, kind, axis in plan:
                op.apply_host(kind, axis, hf, hdf, N, N)

        per_operator()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        for _ in range(e2e_steps):
            per_operator()
        torch.cuda.synchronize()
        el_op = (time.perf_counter() - t1) / e2e_steps
        per_op = {"value": round(9 * N ** 3 / el_op / 1e9 * world, 3), "unit": "Gpts/s",
                  "h2d_bytes_per_step": 9 * field_bytes, "d2h_bytes_per_step": 9 * field_bytes,
                  "path": "pado_apply_host per operator (pinned host buffers)"}
        if terms_path:
            houts = [hdf] + [torch.empty_like(hf).pin_memory() for _ in plan[1:]]
            terms = [(op, kind, axis, 0, 0, 1.0, 0.0, i) for i, (op, kind, axis) in enumerate(plan)]
            apply_host_terms(hf, (N, N, N), terms, houts)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(e2e_steps):
                apply_host_terms(hf, (N, N, N), terms, houts)
            torch.cuda.synchronize()
            el = (time.perf_counter() - t0) / e2e_steps
            e2e = {"value": 9 * N ** 3 / el / 1e9 * world, "unit": "Gpts/s",
                   "h2d_bytes_per_step": field_bytes, "d2h_bytes_per_step": 9 * field_bytes,
                   "path": "pado_apply_host_terms: one upload of f, nine results downloaded (pinned host buffers)",
                   "per_operator_host_calls": per_op}
            del houts
        else:
            e2e = dict(per_op)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(f_host, os.cpu_count() or 1)
    ext = None
    if rank == 0 and world == 1 and not args.no_ext:
        del f, df
        torch.cuda.empty_cache()
        ext = extensions()

    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 3), "unit": "Gpts/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": dict(CONFIG, per_operator_gbs=per_op),
                "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                             "frac": round(achieved / peak, 4), "traffic": profiled_traffic(),
                             "kernel": "pado::stream_kernel (the 9 launches of a step, averaged)",
                             "peak_source": peak_kind},
                "cpu_baseline": cpu, "e2e": e2e, "clocks": clk.summary(), "gpu_launches": launches,
                "extensions": ext}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_configs(args) -> None:
    """The per-config table of the benchmark's configurations on one GPU and
    the host cores: C1 (cd06 periodic d1 on 64^3, 8 seeded sinusoids), C2
    (cd10 d1, cd10 d2, cf90 periodic on 512^3), C3 (1024x512x256: cd06 and
    cd10 d1 bounded along z, cd06 and cd10 d1 periodic along x and y).  GPU:
    CUDA events over 20 applications after warm-up, per operator; CPU: the
    oracle with the reference's Release flags, 1 thread and all host threads,
    one application per operator.  Prints one JSON line."""
    import torch

    import oracle
    import padeops_b200 as pb
    from tests.fields import poly_z, sinusoids, spectrum53

    threads = os.cpu_count() or 1
    peak, _ = measured_peaks()
    cls = {"cd06": (pb.cd06, oracle.CD06), "cd10": (pb.cd10, oracle.CD10), "cf90": (pb.cf90, oracle.CF90)}
    rows = []

    def measure(cfg, f_host, scheme, kind, axis, periodic, d):
        shape = f_host.shape
        n = shape[3 - axis]
        na, nb = {1: (shape[1], shape[0]), 2: (shape[2], shape[0]), 3: (shape[2], shape[1])}[axis]
        pcls, oscheme = cls[scheme]
        op = pcls()
        assert (op.init(n, periodic) if scheme == "cf90" else op.init(n, d, periodic, 0, 0)) == 0
        f = torch.from_numpy(f_host).cuda()
        df = torch.empty_like(f)
        for _ in range(3):
            op.apply(kind, axis, f, df, na, nb)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(20):
            op.apply(kind, axis, f, df, na, nb)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / 20
        got = df.cpu().numpy()
        o = oracle.OracleOp(oscheme, n, d if scheme != "cf90" else 1.0, periodic, fast=True)
        cpu = {}
        for t in (1, threads):
            ts = time.perf_counter()
            ref = o.apply(kind, axis, f_host, na, nb, nthreads=t)
            cpu[t] = f_host.size / (time.perf_counter() - ts) / 1e9
        strict = oracle.OracleOp(oscheme, n, d if scheme != "cf90" else 1.0, periodic).apply(
            kind, axis, f_host, na, nb, nthreads=threads).reshape(shape)
        err = float(np.abs(got - strict).max() / np.abs(strict).max())
        gpts = f_host.size / ms / 1e6
        rows.append({"config": cfg, "op": f"{scheme} {'d1' if kind == 1 else 'd2' if kind == 2 else 'filter'}",
                     "axis": axis, "periodic": periodic, "shape": list(shape)[::-1], "gpu_us": round(ms * 1e3, 1),
                     "gpu_gpts": round(gpts, 1), "hbm_frac": round(gpts * 16 / peak, 3),
                     "cpu_1thr_gpts": round(cpu[1], 3), "cpu_all_gpts": round(cpu[threads], 3),
                     "max_rel_err_vs_oracle": err})
        del f, df

    f1 = sinusoids(64, seed=1)
    for axis in (1, 2, 3):
        measure("C1", f1, "cd06", 1, axis, True, 2 * np.pi / 64)
    f2 = spectrum53((N, N, N), seed=7)
    for scheme, kind in OPS:
        for axis in (1, 2, 3):
            measure("C2", f2, scheme, kind, axis, True, 2 * np.pi / N)
    del f2
    f3 = poly_z((256, 512, 1024), seed=3)
    for scheme in ("cd06", "cd10"):
        measure("C3", f3, scheme, 1, 3, False, 1.0 / 255)
        measure("C3", f3, scheme, 1, 1, True, 2 * np.pi / 1024)
        measure("C3", f3, scheme, 1, 2, True, 2 * np.pi / 512)
    print(json.dumps({"configs": rows, "cpu_model": cpu_model(), "cpu_threads": threads, "hbm_peak_gbs": peak}),
          flush=True)


def run_single_op(args) -> None:
    """One operator on one field, a few times: the small cases the ncu summaries
    under profiles/ are captured on (prints the launch plan)."""
    import torch

    import padeops_b200 as pb

    if args.op == "batch":
        run_batch_profile(args)
        return
    scheme, kind, axis = args.op.split(":")
    kind, axis = int(kind), int(axis)
    n3, n2, n1 = (int(v) for v in args.shape.split(","))
    n = {1: n1, 2: n2, 3: n3}[axis]
    na, nb = {1: (n2, n3), 2: (n1, n3), 3: (n1, n2)}[axis]
    periodic = not args.bounded
    op = {"cd06": pb.cd06, "cd10": pb.cd10, "cf90": pb.cf90}[scheme]()
    ierr = op.init(n, periodic) if scheme == "cf90" else op.init(n, 2 * np.pi / n, periodic, 0, 0)
    assert ierr == 0, ierr
    op.set_variant(args.variant)
    g = torch.Generator(device="cuda").manual_seed(7)
    f = torch.randn(n1 * n2 * n3, dtype=torch.float64, device="cuda", generator=g)
    df = torch.empty_like(f)
    print(json.dumps({"op": args.op, "shape": [n3, n2, n1], "periodic": periodic,
                      "plan": op.launch_plan(kind, axis, f, df, na, nb)}), flush=True)
    for _ in range(args.repeat):
        op.apply(kind, axis, f, df, na, nb, adjoint=args.adjoint)
    torch.cuda.synchronize()
    assert op.device_status() == 0


def run_batch_profile(args) -> None:
    """The batched launch on a seeded uneven batch of about 1 GiB of inputs
    (cd06 / cd10 first derivatives, dimensions from {32, ..., 256}, periodic or
    bounded, random axis): the small case of the batch kernel's ncu summary."""
    import torch

    import padeops_b200 as pb
    from padeops_b200.batch import Batch

    rng = np.random.default_rng(4)
    dims = (32, 48, 64, 96, 128, 192, 256)
    items, total = [], 0
    gen = torch.Generator(device="cuda").manual_seed(4)
    while total < 2 ** 30:
        sh = tuple(int(v) for v in rng.choice(dims, 3))
        scheme, periodic, axis = int(rng.integers(2)), bool(rng.integers(2)), int(rng.integers(1, 4))
        n = sh[3 - axis]
        op = (pb.cd06 if scheme == 0 else pb.cd10)()
        assert op.init(n, 0.1, periodic, 0, 0) == 0
        f = torch.randn(sh, dtype=torch.float64, device="cuda", generator=gen)
        items.append((op, 1, axis, f, torch.empty_like(f), 0, 0))
        total += f.numel() * 8
    b = Batch(items)
    print(json.dumps({"op": "batch", "fields": len(items), "input_bytes": total, "info": b.info()}), flush=True)
    for _ in range(args.repeat):
        b.run()
    torch.cuda.synchronize()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=150)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="pado", choices=["pado", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-ext", action="store_true", help="skip the batched / adjoint comparisons")
    ap.add_argument("--op", default=None,
                    help="profiling: run only scheme:kind:axis (e.g. cf90:0:3), or 'batch' (an uneven 1 GiB batch)")
    ap.add_argument("--shape", default="512,128,512", help="profiling: field shape n3,n2,n1")
    ap.add_argument("--bounded", action="store_true", help="profiling: bounded instead of periodic lines")
    ap.add_argument("--repeat", type=int, default=3, help="profiling: applications of the operator")
    ap.add_argument("--adjoint", action="store_true", help="profiling: the adjoint operator")
    ap.add_argument("--variant", type=int, default=0, help="profiling: kernel variant (pado_set_kernel_variant)")
    ap.add_argument("--configs", action="store_true", help="the per-config table (C1-C3, GPU and CPU)")
    args = ap.parse_args()
    if args.configs:
        run_configs(args)
    elif args.op:
        run_single_op(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()

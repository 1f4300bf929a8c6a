"""Autotuner for the line kernels and the batched kernel.

For one operator (scheme, kind, n, periodic) along one axis the tuner times
every legal (m, lines) tiling -- m = rows one thread sweeps serially (the
Thomas part), n/m = segments joined by the inter-segment chain (the
reduced/parallel part), lines = lines per CTA -- on a synthetic field of the
caller's shape with CUDA events, and keeps the fastest.  For a batch it times
the persistent kernel's lines-per-tile / CTAs-per-SM choices.  Results are
cached in a JSON file keyed by GPU name and problem signature
(``$PADO_TUNE_CACHE`` or ``~/.cache/padeops_b200/tune.json``).
"""
from __future__ import annotations

import json
import os
import threading

import torch

from . import _lib as L

_CACHE_LOCK = threading.Lock()
M_CHOICES = (16, 32, 64)
LINE_CHOICES = (8, 16, 32)
VARIANTS = (4, 6, 5, 1, 2, 3)  # 4, 6, 5: streaming kernel's resident tiles (they pick their own lines per tile)


def cache_path() -> str:
    return os.environ.get("PADO_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "padeops_b200",
                                                          "tune.json"))


def _load() -> dict:
    try:
        with open(cache_path()) as fh:
            return json.load(fh)
    except Exception:
        return {}


def _store(d: dict) -> None:
    p = cache_path()
    try:
        os.makedirs(os.path.dirname(p), exist_ok=True)
        tmp = p + ".tmp"
        with open(tmp, "w") as fh:
            json.dump(d, fh, indent=1, sort_keys=True)
        os.replace(tmp, p)
    except OSError:
        pass  # a read-only home is not an error: tuning still applies to this process


def _key(op, kind: int, axis: int, shape: tuple[int, int, int]) -> str:
    gpu = torch.cuda.get_device_name()
    return f"{gpu}|scheme={op._scheme}|kind={kind}|n={op.n}|per={int(op.periodic)}|axis={axis}|shape={shape}"


def time_op(op, kind: int, axis: int, f: torch.Tensor, df: torch.Tensor, na: int, nb: int, reps: int = 5,
            bc1: int = 0, bcn: int = 0) -> float:
    """Mean device time (ms) of one application, after one warm-up."""
    op.apply(kind, axis, f, df, na, nb, bc1, bcn)
    st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st.record()
    for _ in range(reps):
        op.apply(kind, axis, f, df, na, nb, bc1, bcn)
    en.record()
    torch.cuda.synchronize()
    return st.elapsed_time(en) / reps


def tune_op(op, kind: int, axis: int, shape: tuple[int, int, int], reps: int = 5, use_cache: bool = True,
            verbose: bool = False) -> tuple[int, int, float]:
    """Pick the fastest (m, lines, kernel variant) for `op` applied along `axis`
    of a field of shape (n3, n2, n1) and set it on the handle.
    Returns (m, lines, variant, ms)."""
    key = _key(op, kind, axis, tuple(shape))
    if use_cache:
        with _CACHE_LOCK:
            hit = _load().get(key)
        if hit:
            op.set_variant(hit.get("variant", 1))
            op.set_tiling(hit["m"], hit["lines"])
            return hit["m"], hit["lines"], hit.get("variant", 1), hit["ms"]
    n3, n2, n1 = shape
    na, nb = {1: (n2, n3), 2: (n1, n3), 3: (n1, n2)}[axis]
    g = torch.Generator(device="cuda").manual_seed(0)
    f = torch.randn(n3 * n2 * n1, dtype=torch.float64, device="cuda", generator=g)
    df = torch.empty_like(f)
    best = None
    for variant in VARIANTS:
        op.set_variant(variant)
        for m in M_CHOICES:
            for lines in ((0,) if variant in (4, 5, 6) else LINE_CHOICES):
                try:
                    op.set_tiling(m, lines)
                    ms = time_op(op, kind, axis, f, df, na, nb, reps)
                except L.PadoError:
                    continue
                if verbose:
                    print(f"  variant={variant} m={m:2d} lines={lines:2d}: {ms * 1e3:9.1f} us  "
                          f"{16 * f.numel() / (ms * 1e-3) / 1e9:8.1f} GB/s")
                if best is None or ms < best[3]:
                    best = (m, lines, variant, ms)
    if best is None:
        raise L.PadoError(L.E_SIZE, "no legal tiling")
    op.set_variant(best[2])
    op.set_tiling(best[0], best[1])
    if use_cache:
        with _CACHE_LOCK:
            d = _load()
            d[key] = {"m": best[0], "lines": best[1], "variant": best[2], "ms": best[3]}
            _store(d)
    return best


def _time(fn, reps: int) -> float:
    fn()
    st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st.record()
    for _ in range(reps):
        fn()
    en.record()
    torch.cuda.synchronize()
    return st.elapsed_time(en) / reps


def tune_batch(batch, reps: int = 5, verbose: bool = False, branches=(0, 2, 4, 8)) -> tuple[int, int, int, float]:
    """Autotune a batch: the persistent kernel's (lines per tile, CTAs per SM),
    then what its CUDA graph holds -- the persistent launch (0) or one
    streaming-kernel launch per item on k concurrent branches -- by timing the
    graph replay.  Returns (lines, ctas_per_sm, branches, ms); 0 means
    automatic / no cap / the persistent launch."""
    best = None
    for lines in (0, 8, 16, 32):
        for per_sm in (0, 1, 2):
            if batch.set_config(lines, per_sm) != 0:
                continue
            ms = _time(batch.run, reps)
            if verbose:
                print(f"  persistent lines={lines or 'auto'} ctas/SM={per_sm or 'max'}: {ms:.3f} ms")
            if best is None or ms < best[2]:
                best = (lines, per_sm, ms)
    batch.set_config(best[0], best[1])
    choice = None
    for k in branches:
        if batch.set_graph_branches(k) != 0:
            continue
        ms = _time(batch.run_graph, reps)
        if verbose:
            print(f"  graph {'persistent launch' if k == 0 else f'{k} branches of per-item launches'}: {ms:.3f} ms")
        if choice is None or ms < choice[1]:
            choice = (k, ms)
    batch.set_graph_branches(choice[0])
    return best[0], best[1], choice[0], choice[1]

"""Project-written autotuner of the step's launch shapes.

The column and point kernels of the step take their threads per block at run
time (``nc_set_block``); the right size depends on the grid (columns per
region, regions and ensemble members), on the precision form (registers per
thread) and on the device.  ``tune`` picks each kernel's block size by
measurement: coordinate-wise, one kernel at a time, it times one eager
profiled step per candidate size (``nc_profile`` events, the kernel's own
time) and keeps the fastest, then writes the choice to a JSON cache keyed by
the device name, the state shape, the precision and the ensemble members, so
a later handle of the same case applies it without measuring.

The tiled stencil kernels keep their compile-time tile shapes (32 x 8 cells of
one region, chosen by measurement on B200) and their resident-block targets
(``NC_F32_*`` / launch bounds in csrc/nc_common.cuh): those are template
constants of the kernels, not launch parameters.

Tuning advances the handle's state by the profiled steps: upload the state
again afterwards (the ensemble driver does).
"""
from __future__ import annotations

import json
import os

TUNABLE = {"diag": 128, "vi_solve": 128, "vi_energy": 128, "vp0_c": 256, "gtend": 1024, "hdiff1": 1024,
           "post": 1024, "split_init": 1024, "trc_vflux": 1024, "trc_vadv": 1024, "trc_remap": 1024,
           "trc_qout": 1024, "trc_apply": 1024, "trc_rhog": 1024}
CANDIDATES = (64, 128, 256, 512)


def _device_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name(torch.cuda.current_device())
    except Exception:
        return "cuda"


def cache_key(core, members: int = 1) -> str:
    return "|".join([_device_name(), "x".join(str(x) for x in core.shape), core.precision, f"members={members}"])


def tune(core, members: int = 1, candidates=CANDIDATES, cache: str | None = None, repeats: int = 1) -> dict:
    """Choose the block size of every tunable kernel on ``core`` (a
    NicamCuda with a state uploaded); returns {kernel: threads}.  With
    ``cache`` (a JSON file), a stored choice for the same key is applied
    without measuring, and a new one is stored."""
    key = cache_key(core, members)
    table = {}
    if cache and os.path.exists(cache):
        with open(cache) as f:
            table = json.load(f)
        if key in table:
            for k, t in table[key].items():
                core.set_block(k, t)
            return dict(table[key])

    def kernel_ms(name: str) -> float:
        core.profile(True)
        core.step(repeats)
        st = core.kernel_stats()
        core.profile(False)
        return st.get(name, (float("inf"), 0))[0] / repeats

    choice = {}
    for name, top in TUNABLE.items():
        sizes = [c for c in candidates if c <= top]
        timing = {}
        for c in sizes:
            core.set_block(name, c)
            timing[c] = kernel_ms(name)
        if not timing or min(timing.values()) == float("inf"):
            core.set_block(name, min(top, 128))   # not launched in this configuration
            choice[name] = min(top, 128)
            continue
        best = min(timing, key=timing.get)
        core.set_block(name, best)
        choice[name] = best
    if cache:
        table[key] = choice
        os.makedirs(os.path.dirname(os.path.abspath(cache)), exist_ok=True)
        with open(cache, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
    return choice

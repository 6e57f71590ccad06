"""Autotuner: picks launch shapes for a context by timing them on the model's own state.

The knob is the tile shape of the tiled 3D right-hand side (sf_ctx_set_tile: 32 x 8, 32 x 4,
64 x 4, 32 x 16 rho points per block), which trades halo re-reads (smaller tiles stage relatively more
halo) against blocks per SM and, for ensembles, against the ragged edges of small members.
Results do not depend on the choice; only the time does.
"""
import ctypes

import torch

from ._lib import check, lib
from .model import stream_handle

TILES = {0: (32, 8), 1: (32, 4), 2: (64, 4), 3: (32, 16)}


def _time(fn, reps):
    s = torch.cuda.current_stream()
    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s)
    for _ in range(reps):
        fn()
    b.record(s)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def tune_rhs3d(model, reps=5, variants=tuple(TILES)):
    """Times sf_rhs3d on `model` (a Model or Ensemble) for each tile variant, leaves the fastest
    set on its context and returns {variant: ms}."""
    c, p = model.ctx.ptr, model._p
    st = stream_handle()

    def run():
        check(lib.sf_rhs3d(c, p(model.u), p(model.v), p(model.Huon), p(model.Hvom), p(model.W),
                           p(model.Hz), p(model.ru), p(model.rv), st), "sf_rhs3d")

    times = {}
    for v in variants:
        check(lib.sf_ctx_set_tile(c, v), "sf_ctx_set_tile")
        times[v] = _time(run, reps)
    best = min(times, key=times.get)
    check(lib.sf_ctx_set_tile(c, best), "sf_ctx_set_tile")
    model.rhs_tile = best
    return times

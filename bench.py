"""Benchmark: 3D cell-steps/s of the reference's baroclinic time step on one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config basin4] [--precision fp32|fp64]

Workload (default): basin4 = Lm=2048, Mm=1024, N=50 (104,857,600 interior cells), dx=1 km,
tanh shelf + two seamounts, dt=120 s, ndtfast=40 (nfast+1 barotropic substeps per step),
closed walls, the reference's step semantics (main3d.py:118-324), starting from rest, plus
vertical mixing every step: the learned closure (FP32 form; plain GLS on its fallback
columns) under wind tau_x = 0.15 cos(pi y/Ly) and T = 4 + 20 exp(z/500).  plain_fp64 is the
same workload in FP64 (bit-identical to the reference kernels) with plain GLS.
One "step" is one baroclinic step including its barotropic loop.  Inputs are larger than
L2 (each 3D field is ~0.43 GB in FP32), so no L2 flush is needed between steps.

Multi-GPU (torchrun): the basin does not shard in the reference, so every rank runs an
independent replica (weak scaling); value = all ranks' cell-steps / max-over-ranks time.

--impl reference times the reference's own kernels (host-compiled, oracle/_ref) driven in
its main3d order with OpenMP over the host cores, on a bounded sample of the same basin.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
MEASURED = os.path.join(ROOT, "MEASURED_PEAKS.json")
METRIC = "3D cell-steps/s"


class _StdoutToStderr:
    """Sends the process's C-level stdout to stderr for the duration (the reference's host
    kernels print from C), so that stdout carries the JSON line alone."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)

    def __exit__(self, *a):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


def phase_pass(m, steps, hook, phases):
    """Per-phase CUDA-event times from a separate pass with the phases run one after another
    (Model.overlap off), so that a kernel's time is its own and not stretched by the phases
    that overlap it in the timed run; the headline value comes from the overlapped run.  The
    pass is queued behind a device-side wait, so that a phase's first event is not stamped
    while the host is still submitting the phase's kernels."""
    import torch
    prev = getattr(m, "overlap", False)
    m.overlap = False
    torch.cuda.synchronize()
    torch.cuda._sleep(int(4e7))   # ~20 ms at the B200's clock: the host queues the pass
    m.step(min(steps, 5), timer=hook)
    m.overlap = prev
    torch.cuda.synchronize()
    return {k: float(np.mean([a.elapsed_time(b) for a, b in v])) for k, v in phases.items()}


def time_pred2d(m, n):
    """Device time (ms) of one launch of the fused barotropic predictor (k_pred2d), which runs
    once per barotropic substep inside the loop's graph, from n launches through
    sf_step2d_predictor on the model's own slots: (back_to_back, isolated).  back_to_back: the
    n launches between one pair of CUDA events on the launching stream, divided by n (the
    loop's own mode: each launch starts as the previous one's last wave drains, programmatic
    dependent launch as the context has it).  isolated: each launch between its own pair of
    events (each then also carries the event and its ramp-up and tail; about 5 us more on
    basin4).  Both are queued behind a device-side wait, so that no event is stamped while the
    host is still submitting a kernel.  None where the context has no fused predictor.  The
    model's fields are overwritten (run it after the timed region)."""
    import ctypes
    import torch
    from sailfish_b200._lib import lib, check
    if not lib.sf_ctx_fused_available(m.ctx.ptr):
        return None
    s = m.state2d()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    stream = torch.cuda.current_stream()

    def launch():
        for name in m.NAMES2:                      # cycleTimes2D on the local slot copy
            a = getattr(s, name)
            a[0], a[1], a[2] = a[1], a[2], a[0]
        check(lib.sf_step2d_predictor(m.ctx.ptr, ctypes.byref(s), m.dtfast, 0.0, 0, st),
              "sf_step2d_predictor")

    evs = []
    torch.cuda.synchronize()
    torch.cuda._sleep(int(2e7))   # ~10 ms at the B200's clock: the host queues all n launches
    for k in range(n):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        launch()
        e1.record(stream)
        evs.append((e0, e1))
    torch.cuda.synchronize()
    isolated = float(np.mean([a.elapsed_time(b) for a, b in evs[1:]]))
    launch()                      # warm the back-to-back run's first launch
    torch.cuda.synchronize()
    torch.cuda._sleep(int(2e7))
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for k in range(n):
        launch()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / n, isolated


def launches_per_step(m, mixing):
    """This package's kernel launches in one baroclinic step of Model.step: set_maxflux/omega,
    rhs3d, set_depth, step3d_uv; per barotropic substep the fused predictor (or its four
    launches), the corrector's zeta kernel, its point update and the zeta boundary program,
    plus the closing momentum RHS and the boundary-value upload of the loop; the mixing's
    launches (plain GLS 1; closure rows, network, GLS on the fallback list 3).  The ROMS form
    (ensembles) as counted below.  Memsets are not kernels of this package and are not
    counted."""
    from sailfish_b200._lib import lib
    mix = {"none": 0, "gls": 1, "mlp": 3}[mixing]
    if getattr(m, "semantics", "reference") == "roms":
        # maxflux/omega, rhs3d, stress3d, set_depth, step3d_uv, lateral BC, walls; per substep
        # the predictor's and the corrector's free surface and momentum (the last substep:
        # the predictor's averages only)
        return 7 + 4 * m.nfast + 1 + mix
    fused = bool(lib.sf_ctx_fused_available(m.ctx.ptr))
    sub = 4 if fused else 7
    return 4 + sub * (m.nfast + 1) + 2 + mix


def traffic_per_launch(kernel, grid):
    """DRAM bytes per launch of `kernel` from the committed ncu summaries (profiles/*.md), with
    the summary's name: a 'traffic <kernel> <read> <write> <s2> <N>' line (a 3D kernel,
    scaled to this grid by the number of 3D points) or 'traffic2d <kernel> <read> <write> <s2>'
    (a 2D kernel, scaled by the 2D points); (None, None) if not recorded."""
    import glob
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        try:
            with open(path) as f:
                for line in f:
                    t = line.split()
                    if len(t) == 6 and t[0] == "traffic" and t[1] == kernel:
                        rd, wr, s2, n = (float(x) for x in t[2:])
                        return (rd + wr) * (grid.s2 * grid.N) / (s2 * n), os.path.basename(path)
                    if len(t) == 5 and t[0] == "traffic2d" and t[1] == kernel:
                        rd, wr, s2 = (float(x) for x in t[2:])
                        return (rd + wr) * grid.s2 / s2, os.path.basename(path)
        except OSError:
            pass
    return None, None


def config_of(args):
    """The workload's configuration (with --levels, the same basin with that many levels)."""
    from sailfish_b200 import configs
    if getattr(args, "levels", None):
        return configs.named(args.config, args.levels)
    return configs.CONFIGS[args.config]()


def peaks():
    try:
        with open(MEASURED) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# -------------------------------------------------------------------------------------------
# CPU (reference) measurement
# -------------------------------------------------------------------------------------------
def reference_cpu(config, steps, warmup, omp, shrink=1):
    """The reference's own CPU path of the step: its kernel sources host-compiled for this
    machine (oracle/_ref, g++ -O3 -march=native, OpenMP over the flat thread index) driven in
    its main3d order (main3d.py:118-324), on the basin set up by the oracle's restatement of
    the reference's host routines (nothing from the package).  shrink > 1 runs the same recipe
    on a (Lm/shrink) x (Mm/shrink) sub-basin (same N, dx, dt, ndtfast) as a bounded sample.
    Returns (cell-steps/s, cores, sample text, config dict)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import build_ref
    import oracle as orc
    import ref_driver
    import ref_setup
    if config not in ref_setup.BASINS:
        raise RuntimeError("no reference set-up for workload %s" % config)
    how = build_ref.build_native()
    b = ref_setup.basin(config, shrink)
    og = orc.Grid(b["L"], b["M"], b["N"], b["h"], b["pm"], b["pn"], b["on_u"], b["om_v"],
                  b["fomn"], b["sc_r"], b["sc_w"], b["Cs_r"], b["Cs_w"], b["hc"], b["Vtransform"])
    O = orc.Ocean(og)
    nfast, w1, w2 = ref_setup.weights(b["ndtfast"])
    ct = orc.CompTimes(b["dt"], b["ndtfast"], nfast, w1, w2)
    K = ref_driver.RefKernels(omp, "_native")
    marks = []
    with _StdoutToStderr():
        ref_driver.main3d(og, orc.Boundary(b["lists"]), O, ct, warmup + steps, kernels=K,
                          step_marks=marks)
    dt = marks[warmup + steps - 1] - marks[warmup - 1] if warmup > 0 else marks[-1] - marks[0]
    n_timed = steps if warmup > 0 else steps - 1
    cells = (b["L"] - 1) * (b["M"] - 1) * b["N"]
    sample = ("the reference's kernels (%s) in main3d order on %s%s, %d timed baroclinic steps "
              "after %d warm-up, %d OpenMP threads"
              % (how, config, "" if shrink == 1 else " shrunk to %dx%dx%d (same recipe, dx, dt, "
                 "ndtfast)" % (b["L"] - 1, b["M"] - 1, b["N"]), n_timed, warmup, omp))
    cfg = {"workload": config, "Lm": b["L"] - 1, "Mm": b["M"] - 1, "N": b["N"], "cells": cells,
           "dt": b["dt"], "ndtfast": b["ndtfast"], "barotropic_substeps": nfast + 1,
           "semantics": "reference main3d", "initial_state": "rest, closed walls",
           "vertical_mixing": "AKv constant (the reference's step has no mixing update)"}
    return cells * n_timed / dt, omp, sample, cfg


def cpu_sample(args):
    """The CPU baseline beside the GPU line: the reference arm on a quarter-by-quarter
    sub-basin, run in a child process of its own (the host-compiled reference kernels and
    their OpenMP runtime stay out of this process, which holds torch's)."""
    cmd = [sys.executable, os.path.abspath(__file__), "--impl", "reference", "--config",
           args.config, "--steps", str(args.cpu_steps), "--warmup", "1", "--shrink", "4"]
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    try:
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True,
                           env=env, timeout=600)
        line = json.loads(r.stdout.strip().splitlines()[-1])
        if "unavailable" in line:
            return {"value": None, "unavailable": line["unavailable"]}
        return dict(line["cpu_baseline"])
    except Exception as e:
        return {"value": None, "unavailable": "CPU sample failed: %s" % e}


# -------------------------------------------------------------------------------------------
# clocks during the timed region
# -------------------------------------------------------------------------------------------
def gpu_id(index):
    """An nvidia-smi -i identifier for torch's CUDA device `index` (nvidia-smi numbers GPUs in
    PCI order and ignores CUDA_VISIBLE_DEVICES, so the ordinal can name another GPU): the first
    of its UUID and its PCI bus id that nvidia-smi recognises, else None (no sampling)."""
    import torch
    p = torch.cuda.get_device_properties(index)
    cands = []
    uuid = str(getattr(p, "uuid", "") or "")
    if uuid:
        cands.append(uuid if uuid.startswith(("GPU-", "MIG-")) else "GPU-" + uuid)
    bus = getattr(p, "pci_bus_id", None)
    if bus is not None:
        cands.append("%08x:%02x:%02x.0" % (getattr(p, "pci_domain_id", 0), bus,
                                           getattr(p, "pci_device_id", 0)))
    for c in cands:
        try:
            r = subprocess.run(["nvidia-smi", "-i", c, "--query-gpu=pci.bus_id",
                                "--format=csv,noheader"], stdout=subprocess.PIPE,
                               stderr=subprocess.DEVNULL, text=True, timeout=20)
            if r.returncode == 0 and r.stdout.strip():
                return c
        except Exception:
            pass
    return None


class Clocks:
    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.rows, self.proc = gpu_id(index), [], None

    def __enter__(self):
        if self.index is None:
            return self
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.index, "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm = [float(r[0]) for r in self.rows if len(r) >= 6 and r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if len(r) >= 6 and r[1].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[k] for r in self.rows if len(r) >= 6 for k in range(4)
                          if r[2 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(sm)}


# -------------------------------------------------------------------------------------------
def algorithmic_bytes(grid, esize, semantics="reference"):
    """Compulsory DRAM bytes per launch of each single-kernel phase: every distinct array read
    once and written once at its stored precision (levels x rho points).  The ROMS form's
    rhs3d (with its surface/bottom stress) and column solve (Adams-Bashforth over three
    right-hand sides, W for the implicit vertical advection) move what their comments say."""
    s2, N = grid.s2, grid.N
    if semantics == "roms":
        return {
            "k_rhs3d": esize * (5 * N + 2 * (N + 1)) * s2,     # u,v,Huon,Hvom,Hz -> ru,rv
            # u,v,ru x3,rv x3,Hz,Akv,z_r,W -> u,v; DU,DV -> ubar,vbar (two slots)
            "k_step3d_uv": esize * (14 * N + 4) * s2 + 16 * s2,
            "k_maxflux_omega": esize * (4 * N + 3 * (N + 1)) * s2,
            "k_set_depth": esize * (3 * N + 1) * s2 + 16 * s2,
        }
    return {
        "k_rhs3d": esize * (6 * N + 2 * (N + 1)) * s2,          # u,v,Huon,Hvom,W,Hz -> ru,rv
        "k_step3d_uv": esize * (9 * N) * s2 + 16 * s2,          # u,v,ru,rv,Hz,Akv,z_r -> u,v; DU,DV
        "k_maxflux_omega": esize * (4 * N + 3 * (N + 1)) * s2,  # u,v,Hz,z_w -> Huon,Hvom,W
        "k_set_depth": esize * (3 * N + 1) * s2 + 16 * s2,      # Zt,h -> z_w,z_r,Hz
        # fused barotropic predictor, per launch: zeta_t0, zeta_t1, ubar_t1, vbar_t1, h, pm,
        # pn, on_u, om_v -> zeta_t2, rzeta_t1, rubar_t1, rvbar_t1, ubar_t2, vbar_t2
        "k_pred2d": esize * 15 * s2,
        # the learned closure (k_closure + GLS on its fallback columns), per interior column:
        # u, v, z_r (N levels), bvf (N-1 interior W levels), sustr, svstr, h -> Akv, Akt (N-1)
        "closure": (esize * (4 * N - 1) + 3 * esize + 2 * esize * (N - 1)) * (grid.L - 1) * (grid.M - 1),
    }


def time_steps(m, steps, warmup):
    """Device time (ms) of `steps` baroclinic steps after `warmup` untimed ones."""
    import torch
    stream = torch.cuda.current_stream()
    m.step(warmup)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    m.step(steps)
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b)


def plain_fp64(args):
    """The same workload through this package's FP64 path, whose results are bit-identical to
    the reference's own kernels: how much of the speed-up over the reference's FP64 kernels
    comes from precision and the learned closure, and how much from the kernels' design."""
    import torch
    from sailfish_b200 import configs
    from sailfish_b200.model import Model
    cfg = configs.CONFIGS[args.config]()
    g = cfg["grid"]
    m = Model(g, cfg["boundary"], cfg["dt"], cfg["ndtfast"], precision="fp64")
    mixing = "none" if args.closure == "none" else "gls"
    install_mixing(m, mixing, args.config)
    steps = max(1, min(args.steps, 3))
    ms = time_steps(m, steps, 3)
    cells = (g.L - 1) * (g.M - 1) * g.N
    del m
    torch.cuda.empty_cache()
    return {"value": cells * steps / (ms * 1e-3), "unit": "cell-steps/s",
            "ms_per_step": ms / steps, "steps": steps, "warmup": 3, "dtype": "f64",
            "semantics": "bit-identical to the reference kernels",
            "vertical_mixing": "plain GLS %s every step, FP64" % gls_model_for(args.config)
                               if mixing == "gls" else "AKv constant (the reference's step)"}


def _ref_basin(cfg):
    """The basin dict the reference's GPU kernels take (baseline/ref_gpu.py) for a package
    config: the same grid, tables and boundary lists."""
    g, B = cfg["grid"], cfg["boundary"]
    lists = {}
    for name in ("zetaBC", "ubarBC", "vbarBC", "uvelBC", "vvelBC"):
        for f in ("bcIdx", "bcIdx1", "bcIdx2", "bcIdxFieldIdx2", "bcIdxFieldType", "LBC"):
            lists["%s_%s" % (name, f)] = getattr(getattr(B, name), f)
    for f in ("zetaClosedOrGradientBCIdx1", "zetaClosedOrGradientBCIdx2", "zetaClampedBCIdx1",
              "ubarClosedBCIdx1", "vbarClosedBCIdx1", "ubarClampedBCIdx1", "vbarClampedBCIdx1",
              "ubarGradientBCIdx1", "ubarGradientBCIdx2", "vbarGradientBCIdx1", "vbarGradientBCIdx2"):
        lists[f] = getattr(B, f)
    b = dict(L=g.L, M=g.M, N=g.N, hc=g.hc, Vtransform=g.Vtransform, dt=cfg["dt"],
             ndtfast=cfg["ndtfast"], lists=lists)
    for k in ("h", "pm", "pn", "on_u", "om_v", "fomn", "sc_r", "sc_w", "Cs_r", "Cs_w"):
        b[k] = getattr(g, k)
    return b


def reference_gpu_fp64(args, gls_ms):
    """The plain FP64 GPU step: the reference's own kernels (NVRTC with its options, for
    sm_100a) launched in its main3d order on this GPU (baseline/ref_gpu.py), plus plain GLS in
    FP64 for the vertical mixing the reference lacks (this package's GLS kernel, its time
    `gls_ms` per step measured on the same basin)."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "baseline"))
    import ref_gpu
    from sailfish_b200 import configs, host
    if not ref_gpu.available():
        return {"value": None, "unavailable": "baseline/_ref/src not generated"}
    cfg = configs.CONFIGS[args.config]()
    g = cfg["grid"]
    nf, w1, w2 = host.set_weights(cfg["ndtfast"])
    with _StdoutToStderr():            # the reference's initialize kernels printf
        r = ref_gpu.RefGPU(_ref_basin(cfg), nf, w1, w2, fmad=True)
        r.step(2)
        torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    steps = max(1, min(args.steps, 3))
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    r.step(steps)
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / steps
    launches = r.launches_per_step()
    del r
    torch.cuda.empty_cache()
    cells = (g.L - 1) * (g.M - 1) * g.N
    tot = ms + (gls_ms or 0.0)
    return {"value": cells / (tot * 1e-3), "unit": "cell-steps/s", "ms_per_step": tot,
            "reference_kernels_ms_per_step": ms, "gls_fp64_ms_per_step": gls_ms,
            "steps": steps, "warmup": 2, "dtype": "f64",
            "kernels": "the reference's own (modules/mod_cppkernels.cpp, nonlinear/rhs_kernels.cpp, "
                       "nonlinear/step3D_uv.kernels.cpp, modules/mod_BC.c), NVRTC for sm_100a with "
                       "-default-device --restrict --std=c++17, launched in main3d order",
            "launches_per_step": launches,
            "vertical_mixing": "plain GLS %s every step, FP64 (this package's kernel; the "
                               "reference has no runnable GLS)" % gls_model_for(args.config)}


def gls_fp64_ms(args):
    """Device time of one plain-GLS update in FP64 on the bench's basin."""
    import torch
    from sailfish_b200 import configs
    from sailfish_b200.model import Model
    cfg = configs.CONFIGS[args.config]()
    m = Model(cfg["grid"], cfg["boundary"], cfg["dt"], cfg["ndtfast"], precision="fp64")
    install_mixing(m, "gls", args.config)
    m.start()
    m.mixing()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(3):
        m.mixing()
    b.record(stream)
    torch.cuda.synchronize()
    del m
    torch.cuda.empty_cache()
    return a.elapsed_time(b) / 3


def error_vs_fp64():
    """One baroclinic step of a 512x512x32 basin (basin1's recipe, square so that the
    reference's flat-index guards stay inside the fields) from a 1 mm Gaussian surface bump,
    FP32 form against the FP64 path from identical inputs: RMS and max absolute error."""
    import torch
    from sailfish_b200 import configs
    from sailfish_b200.model import Model
    cfg = configs.basin(512, 512, 32, 2.0e3, [(0.5, 0.6)], dt=240.0, ndtfast=30)
    g = cfg["grid"]
    x, y = g.x, g.y
    bump = 1e-3 * np.exp(-((x - x.max() / 2) ** 2 + (y - y.max() / 3) ** 2) / (50e3) ** 2)
    res = {}
    for prec in ("fp64", "fp32"):
        m = Model(g, cfg["boundary"], cfg["dt"], cfg["ndtfast"], precision=prec)
        m.Zt_avg1.copy_(torch.from_numpy(bump.ravel()))
        m.step(1)
        torch.cuda.synchronize()
        res[prec] = {"zeta": m._slot("zeta", 2).double().cpu().numpy(),
                     "ubar": m._slot("ubar", 2).double().cpu().numpy(),
                     "u": m.u.double().cpu().numpy(), "v": m.v.double().cpu().numpy()}
        del m
    out = {"case": "512x512x32 basin, dx 2 km, dt 240 s, ndtfast 30, 1 mm bump, 1 step",
           "units": {"zeta": "m", "ubar": "m/s", "u": "m/s", "v": "m/s"}}
    for k in ("zeta", "ubar", "u", "v"):
        a, b = res["fp64"][k], res["fp32"][k]
        d = b - a
        out[k] = {"rms": float(np.sqrt(np.mean(d * d))), "max": float(np.abs(d).max()),
                  "rms_fp64_field": float(np.sqrt(np.mean(a * a))),
                  "finite": bool(np.isfinite(b).all() and np.isfinite(a).all())}
    torch.cuda.empty_cache()
    return out


ROMS_STATE = ("zeta", "ubar", "vbar", "rzeta", "rubar", "rvbar", "Zt_avg1", "DU_avg1", "DV_avg1",
              "DU_avg2", "DV_avg2", "u", "v", "AKv", "W", "Huon", "Hvom")
GLS_STATE = ("tke", "gls", "Akt", "Akk", "Akp", "Lscale")


def _snapshot(m, c):
    """A ROMS-form model's state and its mixing's GLS state, as FP64 copies."""
    snap = {n: getattr(m, n).double().clone() for n in ROMS_STATE}
    snap["ru3"] = [t.double().clone() for t in m._ru3]
    snap["rv3"] = [t.double().clone() for t in m._rv3]
    snap.update({"gls_" + n: getattr(c.cols, n).double().clone() for n in GLS_STATE})
    snap["slots"] = list(m.slots)
    snap["counters"] = (m.iic, m.time, m.time2D)
    return snap


def _restore(m, c, snap):
    """Start model m (any precision) and its mixing c from a snapshot of another run."""
    for n in ROMS_STATE:
        getattr(m, n).copy_(snap[n])
    for dst, srcs in ((m._ru3, snap["ru3"]), (m._rv3, snap["rv3"])):
        for t, s in zip(dst, srcs):
            t.copy_(s)
    for n in GLS_STATE:
        getattr(c.cols, n).copy_(snap["gls_" + n])
    m.slots = list(snap["slots"])
    m.iic, m.time, m.time2D = snap["counters"]


def roms_day(args, hours=24.0, tau0=0.15, rdrag2=3e-3, runs_of=(("fp32", "mlp"), ("fp64", "gls")),
             spinup_hours=0.0):
    """The configuration's physics for `hours` simulated in the ROMS-form step (wind
    tau_x = tau0 cos(pi y/Ly) N/m2, quadratic bottom drag rdrag2, Coriolis, T = 4 + 20 exp(z/500)
    for the mixing, from rest), run twice from identical initial states as `runs_of` says
    ((precision, mixing) pairs: by default the FP32 form with the learned closure against FP64
    with plain GLS every step).  Returns the RMS / max differences of the free surface
    (Zt_avg1, the surface the 3D step uses), ubar, u and v over the interior at the end, with
    the RMS of the second run's fields, and each run's device time per step.  With
    spinup_hours > 0 every run starts instead from the state (flow, averages, right-hand-side
    history, GLS turbulence) of an FP64 + plain-GLS run of that many hours from rest."""
    import torch
    from sailfish_b200 import configs
    from sailfish_b200.model import Model
    cfg = configs.CONFIGS[args.config]()
    g = cfg["grid"]
    nsteps = int(round(hours * 3600.0 / cfg["dt"]))
    # the ROMS-form barotropic step is stable for c dtfast / dx < 0.757 (von Neumann, 2D); a
    # configuration beyond it (basin1: 0.80 at h = 4000 m) runs with more substeps
    ndtfast, courant = configs.roms_ndtfast(cfg)
    stream = torch.cuda.current_stream()
    runs, times = {}, {}
    keys = []

    def make(prec, mode):
        m = Model(g, cfg["boundary"], cfg["dt"], ndtfast, precision=prec, semantics="roms")
        c = install_mixing(m, mode, args.config)
        m.set_forcing(c.cols.sustr.double().cpu().numpy(), c.cols.svstr.double().cpu().numpy(),
                      rdrag2)
        m.check_every = 60
        return m, c

    snap = None
    if spinup_hours > 0:
        m, c = make("fp64", "gls")
        m.step(int(round(spinup_hours * 3600.0 / cfg["dt"])))
        torch.cuda.synchronize()
        snap = _snapshot(m, c)
        del m, c
        torch.cuda.empty_cache()
    for prec, mode in runs_of:
        key = "%s_%s" % (prec, mode)
        keys.append(key)
        m, c = make(prec, mode)
        if snap is not None:
            _restore(m, c, snap)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        m.step(nsteps)
        b.record(stream)
        torch.cuda.synchronize()
        times[key] = a.elapsed_time(b) / nsteps
        runs[key] = {"zeta": m.Zt_avg1.clone(), "ubar": m._slot("ubar", 1).clone(),
                     "u": m.u.clone(), "v": m.v.clone(),
                     "fallback_columns": int(c.mask.sum()) if mode == "mlp" else None}
        del m, c
        torch.cuda.empty_cache()
    J, I, N = g.J, g.I, g.N
    start = ("from rest" if spinup_hours <= 0 else
             "after %g h of FP64 + plain GLS from rest" % spinup_hours)
    out = {"case": "%s, ROMS-form step, %d steps of %g s (%g h) %s, wind %g cos(pi y/Ly) "
                   "N/m2, quadratic drag %g; %s against %s" % (
                       args.config, nsteps, cfg["dt"], hours, start, tau0, rdrag2, keys[0],
                       keys[1]),
           "units": {"zeta": "m", "ubar": "m/s", "u": "m/s", "v": "m/s"},
           "ndtfast": ndtfast, "barotropic_courant_of_config": courant,
           "ms_per_step": times, "fallback_columns": runs[keys[0]]["fallback_columns"]}
    def diff(ka, kb):
        res = {}
        for k in ("zeta", "ubar", "u", "v"):
            a64 = runs[kb][k].double()
            a32 = runs[ka][k].double()
            if k in ("u", "v"):
                a64 = a64.reshape(N + 1, J, I)[:N, 1:-1, 1:-1]
                a32 = a32.reshape(N + 1, J, I)[:N, 1:-1, 1:-1]
            else:
                a64, a32 = a64.reshape(J, I)[1:-1, 1:-1], a32.reshape(J, I)[1:-1, 1:-1]
            d = a32 - a64
            res[k] = {"rms": float(d.pow(2).mean().sqrt()), "max": float(d.abs().max()),
                      "rms_fp64_field": float(a64.pow(2).mean().sqrt()),
                      "finite": bool(torch.isfinite(a32).all() and torch.isfinite(a64).all())}
        return res

    out.update(diff(keys[0], keys[1]))
    out["targets"] = {"zeta_rms_m": 1e-4, "uv_rms_m_per_s": 1e-3,
                      "met": bool(out["zeta"]["rms"] <= 1e-4 and out["u"]["rms"] <= 1e-3 and
                                  out["v"]["rms"] <= 1e-3)}
    if len(keys) > 2:   # the same difference split into its two causes, via the third run
        out["decomposition"] = {"%s_vs_%s" % (keys[2], keys[1]): diff(keys[2], keys[1]),
                                "%s_vs_%s" % (keys[0], keys[2]): diff(keys[0], keys[2])}
    del runs
    torch.cuda.empty_cache()
    return out


WEIGHTS_FOR = {"basin4q": "basin4"}   # basins sharing a recipe (and N) share the closure


def closure_weights(config):
    name = WEIGHTS_FOR.get(config, config)
    path = os.path.join(ROOT, "sailfish_b200", "weights", "closure_%s.npz" % name)
    return path if os.path.exists(path) else None


def install_mixing(m, mode, config):
    """Vertical mixing for the step: 'mlp' (the learned closure with plain GLS on fallback
    columns), 'gls' (plain GLS) or 'none' (AKv constant, the reference's step)."""
    from sailfish_b200 import closure
    if mode == "none":
        return None
    net = None
    path = closure_weights(config)
    if mode == "mlp":
        if path is None:
            raise SystemExit("no trained closure weights for %s (sailfish_b200/weights/); "
                             "train them with python -m sailfish_b200.train_closure" % config)
        net = closure.Network.load(path)
    # plain GLS runs the GLS model the configuration's network learned (its training data)
    gls_model = gls_model_for(config)
    return closure.mixing_for(m, mode, net, gls_model=gls_model)


def closure_act(config):
    path = closure_weights(config)
    if path is None:
        return None
    d = np.load(path)
    return str(d["act"]) if "act" in d else "gelu"


def gls_model_for(config):
    """The GLS model of a configuration: the one its closure weights were trained on (k-psi for
    config 1's basin, as its specification asks), else k-epsilon."""
    path = closure_weights(config)
    if path is not None:
        d = np.load(path)
        if "gls_model" in d:
            return str(d["gls_model"])
    return "k-epsilon"


def closure_variants(m, config, reps=5):
    """Device time (ms) of one closure update on the bench's state for every trained network of
    the configuration (closure_<config>*.npz: the GELU network of the specification and its
    ReLU variant, where present), keyed by activation."""
    import glob
    import torch
    from sailfish_b200 import closure
    name = WEIGHTS_FOR.get(config, config)
    out = {}
    prev = m.mixing
    stream = torch.cuda.current_stream()
    for path in sorted(glob.glob(os.path.join(ROOT, "sailfish_b200", "weights",
                                              "closure_%s*.npz" % name))):
        net = closure.Network.load(path)
        if net.N != m.grid.N:
            continue
        c = closure.mixing_for(m, "mlp", net, gls_model=net.gls_model)
        c()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            c()
        b.record(stream)
        torch.cuda.synchronize()
        out[net.act] = {"ms": a.elapsed_time(b) / reps, "weights": os.path.basename(path),
                        "fallback_columns": int(c.mask.sum())}
    m.mixing = prev
    return out


def closure_error(m, steps=300):
    """Learned closure against plain GLS at the bench state: GLS spun up for `steps`
    iterations on the same columns, then the network's Akv/Akt (in-range columns) against
    GLS's, log10 RMS over the interior columns and levels 1..N-1."""
    import torch
    from sailfish_b200 import closure
    c = m.mixing
    g = m.grid
    ref = closure.Closure(m, "gls")
    closure.basin_forcing(m, ref.cols)
    for _ in range(steps):
        ref()
    akv_g, akt_g = m.AKv.clone(), ref.cols.Akt.clone()
    c()
    torch.cuda.synchronize()
    N, s2 = g.N, g.s2
    cols = closure.interior_columns(g, m.u.device)
    inr = cols[c.mask[cols] == 0]
    lg = lambda a: torch.log10(a.reshape(N + 1, s2)[1:N][:, inr].double().clamp(1e-6, 1e-1))
    ev = (lg(m.AKv) - lg(akv_g)).pow(2).mean().sqrt()
    et = (lg(c.cols.Akt) - lg(akt_g)).pow(2).mean().sqrt()
    cv = (lg(akv_g) + 3.0).pow(2).mean().sqrt()
    return {"akv_log10_rms_vs_gls": float(ev), "akt_log10_rms_vs_gls": float(et),
            "constant_akv_log10_rms_vs_gls": float(cv),
            "fallback_columns": int(c.mask.sum()), "columns": int(cols.numel()),
            "gls_spinup_iterations": steps}


def max_over_ranks(ms, world, device):
    """The slowest rank's time: replicas and ensemble shards run without any collective on
    the data path; only this timing reduction crosses ranks."""
    if world <= 1:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def run_ensemble(args, rank, world):
    """Config 2: 256 basins of uneven size (seeded), FP32 with FP64 accumulators, stepped
    together by the pooled, block-mapped kernels; the barotropic loop replays as one CUDA graph
    and the 3D right-hand side's tile shape is autotuned."""
    import torch
    from sailfish_b200 import autotune, ensemble
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    # weak scaling: args.members per GPU, rank r taking members r, r + world, ... of the
    # world * args.members drawn from the seed
    members = ensemble.ensemble_members(seed=args.seed, n=args.members * world)[rank::world]
    sem = args.semantics or "roms"
    ndtfast = ensemble_ndtfast(members) if sem == "roms" else 30
    m = ensemble.make(members, precision=args.precision, ndtfast=ndtfast, semantics=sem)
    if sem == "roms":
        ensemble.roms_forcing(m, tau0=0.1, rdrag2=3e-3)
    stream = torch.cuda.current_stream()
    m.step(1)
    # the tiled rhs3d's shapes (the reference semantics; the ROMS form has its own kernel)
    tune = autotune.tune_rhs3d(m, reps=3) if sem == "reference" else {}
    phases = {}

    def hook(name):
        ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        phases.setdefault(name, []).append(ev)
        return ev

    m.step(max(args.warmup - 1, 0))
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(torch.cuda.current_device()) as clk:
        start.record(stream)
        m.step(args.steps)
        stop.record(stream)
        torch.cuda.synchronize()
    ms = max_over_ranks(start.elapsed_time(stop), world, dev)
    if world > 1:
        torch.distributed.barrier()
    per_phase = phase_pass(m, args.steps, hook, phases)
    grids = m.members_grids
    esize = 4 if args.precision == "fp32" else 8
    ab = {}
    for g in grids:
        for k, v in algorithmic_bytes(g, esize, sem).items():
            if k != "closure":
                ab[k] = ab.get(k, 0) + v
    dom = max((k for k in per_phase if k in ab), key=lambda k: per_phase[k])
    peak, kind = peaks()
    achieved = ab[dom] / (per_phase[dom] * 1e-3) / 1e9
    cells = m.cells
    all_cells = cells
    if world > 1:   # every rank's own members (host-side count, no data on the path)
        all_cells = sum((g.L - 1) * (g.M - 1) * g.N for g, _, _ in
                        ensemble.ensemble_members(seed=args.seed, n=args.members * world))
    # end to end: u, v pools in from pinned host memory, the zeta pool out, every step
    hu = torch.empty_like(m.u, device="cpu").pin_memory()
    hv = torch.empty_like(m.v, device="cpu").pin_memory()
    hz = torch.empty_like(m.zeta[0], device="cpu").pin_memory()
    hu.copy_(m.u)
    hv.copy_(m.v)
    e_steps = max(1, min(args.steps, 3))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e_steps):
        m.u.copy_(hu, non_blocking=True)
        m.v.copy_(hv, non_blocking=True)
        m.step(1)
        hz.copy_(m._slot("zeta", 2), non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e_ms = e0.elapsed_time(e1) / e_steps
    per_step = launches_per_step(m, "none")
    out = {
        "metric": METRIC, "value": all_cells * args.steps / (ms * 1e-3), "unit": "cell-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if args.precision == "fp32" else "f64",
        "data": "synthetic",
        "config": {"workload": "ensemble%d" % args.members, "members": args.members,
                   "seed": args.seed, "cells": cells,
                   "Lm": [g.L - 1 for g in grids][:8] + ["..."],
                   "N": {"16": sum(g.N == 16 for g in grids), "32": sum(g.N == 32 for g in grids)},
                   "dt": m.dt, "ndtfast": m.ndtfast, "barotropic_substeps": m.nfast + 1,
                   "semantics": "reference main3d per member" if sem == "reference" else
                   "ROMS form per member (wind tau_x = 0.1 cos(pi y/Ly) N/m2, quadratic drag "
                   "3e-3, Coriolis, closed walls)",
                   "initial_state": "Gaussian surface bump per member (seeded), closed walls",
                   "vertical_mixing": "AKv constant (the reference's step; the closure and GLS "
                                      "run single grids)",
                   "l2": "inputs larger than L2 (3D pools %.2f GB each)" % (m.u.numel() * esize / 1e9),
                   "parallelism": "replicas" if world > 1 else "single",
                   "rhs3d_tile_autotune_ms": {str(autotune.TILES[k]): v for k, v in tune.items()},
                   "rhs3d_tile": str(autotune.TILES[m.rhs_tile]) if tune else None},
        "phases_ms": per_phase,
        "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": kind,
                     "algorithmic_bytes": ab[dom], "traffic": None},
        "e2e": {"value": cells / (e_ms * 1e-3), "unit": "cell-steps/s",
                "h2d_bytes_per_step": (hu.numel() + hv.numel()) * hu.element_size(),
                "d2h_bytes_per_step": hz.numel() * hz.element_size()},
        "gpu_launches": args.steps * per_step + 1,
        "clocks": clk.summary(),
    }
    del m
    torch.cuda.empty_cache()
    if not args.no_error and rank == 0:
        out["error_vs_fp64"] = ensemble_error(members, sem, ndtfast, args.error_hours)
    return out


def ensemble_ndtfast(members):
    """Barotropic substeps for the ROMS form on every member (configs.roms_ndtfast, the most
    any member needs)."""
    from sailfish_b200 import configs
    return max(configs.roms_ndtfast({"grid": g, "dt": 240.0, "ndtfast": 30})[0]
               for g, _, _ in members)


def ensemble_error(members, semantics="roms", ndtfast=30, hours=6.0):
    """Every member from its bump for `hours` (the reference semantics: one step), FP32 form
    against FP64 from identical inputs: per-member RMS differences of zeta (the surface the
    3D step uses), u and v over the member's interior, with the members' field RMS; members
    whose FP64 run is not finite (the reference's semantics on non-square grids) are counted
    and left out."""
    import torch
    from sailfish_b200 import ensemble
    nsteps = 1 if semantics == "reference" else max(1, int(round(hours * 3600.0 / 240.0)))
    res = {}
    for prec in ("fp64", "fp32"):
        m = ensemble.make(members, precision=prec, ndtfast=ndtfast, semantics=semantics)
        if semantics == "roms":
            ensemble.roms_forcing(m, tau0=0.1, rdrag2=3e-3)
        m.step(nsteps)
        torch.cuda.synchronize()
        res[prec] = [{k: (m.member("Zt_avg1", i) if k == "zeta" else m.member(k, i))
                      .double().cpu().numpy()[..., 1:-1, 1:-1] for k in ("zeta", "u", "v")}
                     for i in range(len(members))]
        del m
        torch.cuda.empty_cache()
    rms = {"zeta": [], "u": [], "v": []}
    field = {"zeta": [], "u": [], "v": []}
    finite = 0
    for a, b in zip(res["fp64"], res["fp32"]):
        if not all(np.isfinite(a[k]).all() for k in a):
            continue
        finite += 1
        for k in rms:
            d = b[k] - a[k]
            rms[k].append(float(np.sqrt(np.mean(d * d))))
            field[k].append(float(np.sqrt(np.mean(a[k] * a[k]))))
    out = {"case": ("1 step from each member's bump" if semantics == "reference" else
                    "%d steps of 240 s (%.1f h) from each member's bump, ROMS form with wind "
                    "and drag, ndtfast %d" % (nsteps, nsteps * 240.0 / 3600.0, ndtfast)),
           "members_finite": finite, "members": len(members)}
    for k, v in rms.items():
        out[k] = {"rms_max": max(v) if v else None,
                  "rms_median": float(np.median(v)) if v else None,
                  "field_rms_median": float(np.median(field[k])) if v else None}
    return out


def run_ours(args, rank, world):
    import torch
    from sailfish_b200 import autotune, configs
    from sailfish_b200.model import Model
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    cfg = config_of(args)
    grid = cfg["grid"]
    m = Model(grid, cfg["boundary"], cfg["dt"], cfg["ndtfast"], precision=args.precision)
    mixing = args.closure or ("mlp" if args.precision == "fp32" else "gls")
    install_mixing(m, mixing, args.config)
    esize = 4 if args.precision == "fp32" else 8
    cells = (grid.L - 1) * (grid.M - 1) * grid.N
    stream = torch.cuda.current_stream()

    phases = {}

    def hook(name):
        ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        phases.setdefault(name, []).append(ev)
        return ev

    m.step(args.warmup)
    # the tile shape of the 3D right-hand side, timed on this state (ru/rv kept as they were)
    ru0, rv0 = m.ru.clone(), m.rv.clone()
    tune = autotune.tune_rhs3d(m, reps=3)
    m.ru.copy_(ru0)
    m.rv.copy_(rv0)
    del ru0, rv0
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(torch.cuda.current_device()) as clk:
        start.record(stream)
        m.step(args.steps)
        stop.record(stream)
        torch.cuda.synchronize()
    ms = max_over_ranks(start.elapsed_time(stop), world, dev)
    if world > 1:
        torch.distributed.barrier()
    per_phase = phase_pass(m, args.steps, hook, phases)

    # end to end: host state in pinned memory, H2D of the step's prognostic 3D inputs (u, v)
    # and D2H of its surface elevation result, through the same public Model API
    hu = torch.empty_like(m.u, device="cpu").pin_memory()
    hv = torch.empty_like(m.v, device="cpu").pin_memory()
    hz = torch.empty_like(m.zeta[0], device="cpu").pin_memory()
    hu.copy_(m.u)
    hv.copy_(m.v)
    e_start, e_stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_steps = max(1, min(args.steps, 3))
    torch.cuda.synchronize()
    e_start.record(stream)
    for _ in range(e_steps):
        m.u.copy_(hu, non_blocking=True)
        m.v.copy_(hv, non_blocking=True)
        m.step(1)
        hz.copy_(m._slot("zeta", 2), non_blocking=True)
    e_stop.record(stream)
    torch.cuda.synchronize()
    e_ms = e_start.elapsed_time(e_stop) / e_steps
    bi = (hu.numel() + hv.numel()) * hu.element_size()
    bo = hz.numel() * hz.element_size()

    # per-launch times and launches per step of the kernels with algorithmic byte counts; the
    # roofline is reported for the kernel that takes the most time per step
    ab = algorithmic_bytes(grid, esize)
    per_launch = {k: (per_phase[k], 1) for k in per_phase if k in ab}
    t_pred = time_pred2d(m, m.nfast + 1)
    if t_pred is not None:
        per_launch["k_pred2d"] = (t_pred[0], m.nfast + 1)
    dom = max(per_launch, key=lambda k: per_launch[k][0] * per_launch[k][1])
    peak, kind = peaks()
    achieved = ab[dom] / (per_launch[dom][0] * 1e-3) / 1e9
    value = cells * args.steps * world / (ms * 1e-3)
    # launches per baroclinic step, plus one omega at the end of the timed call
    per_step = launches_per_step(m, mixing)
    traffic = traffic_per_launch(dom, grid) if args.precision == "fp32" else (None, None)
    out = {
        "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if args.precision == "fp32" else "f64", "data": "synthetic",
        "config": {"workload": args.config + ("" if not args.levels else " with %d levels" % args.levels),
                   "Lm": grid.L - 1, "Mm": grid.M - 1, "N": grid.N,
                   "cells": cells, "dt": m.dt, "ndtfast": m.ndtfast,
                   "barotropic_substeps": m.nfast + 1, "semantics": "reference main3d",
                   "initial_state": "rest, closed walls",
                   "vertical_mixing": {"none": "AKv constant (the reference's step)",
                                       "gls": "plain GLS %s every step" % gls_model_for(args.config),
                                       "mlp": "learned closure (%s network), plain GLS %s on "
                                              "fallback columns" % (
                                                  closure_act(args.config), gls_model_for(args.config))
                                       }[mixing],
                   "forcing": "closure: wind tau_x = 0.15 cos(pi y/Ly) N/m2, T = 4 + 20 exp(z/500)"
                              if mixing != "none" else None,
                   "l2": "inputs larger than L2 (each 3D field %.2f GB)" % (m.u.numel() * esize / 1e9),
                   "parallelism": "replicas" if world > 1 else "single",
                   "rhs3d_form": autotune.variant_name(
                       "march%d" % m.rhs_march if m.rhs_march else m.rhs_tile),
                   "rhs3d_autotune_ms": {autotune.variant_name(k): v for k, v in tune.items()}},
        "phases_ms": per_phase,
        "kernel_ms_per_step": {k: t * n for k, (t, n) in per_launch.items()},
        "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": kind,
                     "launch_ms": per_launch[dom][0], "launches_per_step": per_launch[dom][1],
                     "launch_timing": "back to back: %d launches between one pair of CUDA events "
                                      "on the launching stream" % per_launch[dom][1]
                     if dom == "k_pred2d" else "the phase between its own pair of CUDA events",
                     "launch_ms_isolated": t_pred[1] if dom == "k_pred2d" else None,
                     "algorithmic_bytes": ab[dom],
                     "traffic": traffic[0],
                     "traffic_source": None if traffic[0] is None else
                     "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch "
                     "(profiles/%s), scaled to this grid" % traffic[1]},
        "e2e": {"value": cells / (e_ms * 1e-3), "unit": "cell-steps/s",
                "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo},
        "gpu_launches": args.steps * per_step + 1,
        "clocks": clk.summary(),
    }
    if mixing == "mlp":
        out["closure_ms_by_network"] = closure_variants(m, args.config)
    if mixing == "mlp" and not args.no_error:
        out["closure_error"] = closure_error(m)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="basin4")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--cpu-steps", type=int, default=10)
    ap.add_argument("--shrink", type=int, default=1,
                    help="reference arm: run the basin's recipe at Lm/shrink x Mm/shrink")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 timing")
    ap.add_argument("--members", type=int, default=256, help="ensemble members (config ensemble)")
    ap.add_argument("--seed", type=int, default=0, help="ensemble seed (config ensemble)")
    ap.add_argument("--closure", choices=["mlp", "gls", "none"], default=None,
                    help="vertical mixing in the step (default: mlp for fp32, gls for fp64)")
    ap.add_argument("--no-error", action="store_true", help="skip the FP32-vs-FP64 error case")
    ap.add_argument("--semantics", choices=["reference", "roms"], default=None,
                    help="ensemble step semantics (default: the ROMS form)")
    ap.add_argument("--error-hours", type=float, default=6.0,
                    help="simulated hours of the ensemble's FP32-vs-FP64 error run (ROMS form)")
    ap.add_argument("--levels", type=int, default=None,
                    help="run the basin with this many levels (profiling cases)")
    ap.add_argument("--day-hours", type=float, default=None,
                    help="simulated hours of the ROMS-form error runs (default 24 on basin4, "
                         "48 = 720 steps on basin1; 0: skip)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    omp = len(os.sched_getaffinity(0))

    if args.impl == "reference":
        if rank != 0:
            return
        try:
            v, cores, sample, cfg = reference_cpu(args.config, max(args.steps, 1), args.warmup,
                                                  omp, shrink=args.shrink)
        except Exception as e:
            print(json.dumps({"impl": "reference", "unavailable": str(e)}))
            return
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": v, "unit": "cell-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": cfg["cells"] / v * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": cores,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}))
        return

    import torch
    if world > 1:
        torch.distributed.init_process_group(
            "nccl", timeout=__import__("datetime").timedelta(seconds=120))
    if args.config == "ensemble":
        out = run_ensemble(args, rank, world)
        if rank == 0:
            print(json.dumps(out))
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    out = run_ours(args, rank, world)
    if rank == 0:
        if args.precision == "fp32" and not args.no_fp64:
            torch.cuda.empty_cache()
            gms = gls_fp64_ms(args) if args.closure != "none" else None
            try:
                out["plain_fp64"] = reference_gpu_fp64(args, gms)
            except Exception as e:
                out["plain_fp64"] = {"value": None, "unavailable": "reference kernels: %s" % e}
            if out["plain_fp64"].get("value"):
                out["plain_fp64"]["speedup_of_value"] = out["value"] / world / out["plain_fp64"]["value"]
            torch.cuda.empty_cache()
            out["opt_fp64"] = plain_fp64(args)
            out["opt_fp64"]["speedup_of_value"] = out["value"] / world / out["opt_fp64"]["value"]
        if not args.no_error:
            out["error_vs_fp64"] = error_vs_fp64()
        # basin4: one simulated day; basin1: its 720 steps of 240 s
        hours = args.day_hours if args.day_hours is not None else (
            48.0 if args.config == "basin1" else 24.0)
        if hours > 0 and args.config in ("basin4", "basin4q", "basin1"):
            try:
                out["day_error_vs_fp64"] = roms_day(args, hours=hours)
            except Exception as e:   # a blow-up check that fired, for instance
                out["day_error_vs_fp64"] = {"failed": str(e)}
                torch.cuda.empty_cache()
            # the same day after a day of spin-up (GLS turbulence developed), with the
            # difference split into precision and closure through a third run
            try:
                out["spun_up_day_error_vs_fp64"] = roms_day(
                    args, hours=hours, spinup_hours=hours,
                    runs_of=(("fp32", "mlp"), ("fp64", "gls"), ("fp32", "gls")))
            except Exception as e:
                out["spun_up_day_error_vs_fp64"] = {"failed": str(e)}
                torch.cuda.empty_cache()
        if not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_sample(args)
        print(json.dumps(out))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()

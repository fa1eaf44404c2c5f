#!/usr/bin/env python
"""Benchmark: ms per OSEM iteration, 128^3 / 120 views, on one B200.

Workload (full128, seed 2000): 128^3 float32 volume, 0.3125 cm voxels,
120 views on an elliptical 22 x 18 cm orbit, 8 subsets, attenuation, a
33x33-tap DRF at every depth and ESSE scatter (collapse 2, two Taylor
terms), Poisson data at 5e6 counts.  One step = one OSEM iteration (all
8 subsets, 120 projections + 120 backprojections with scatter).

  value      device time per iteration with everything resident in HBM,
             CUDA events on the library's stream (IrlOsemIterate)
  e2e        the public call IrlOsem (host buffers in, result out, set-up,
             normalisation images and a per-iteration callback included),
             wall time / iterations
  roofline   the stage with the largest device time (ESSE) against its bound,
             the other stages beside it
  cpu_baseline  the reference C (compiled here) on a bounded sample

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

For N > 1 (torchrun) every rank runs an independent replica (a reconstruction
is one device's work: its subsets depend on one another) and rank 0 prints
the job line.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

# one GPU per rank: pin the visible device before any CUDA initialisation
_LOCAL_RANK = int(os.environ.get("LOCAL_RANK", "0"))
_WORLD = int(os.environ.get("WORLD_SIZE", "1"))
if _WORLD > 1 and "CUDA_VISIBLE_DEVICES" not in os.environ:
    os.environ["CUDA_VISIBLE_DEVICES"] = str(_LOCAL_RANK)

import numpy as np  # noqa: E402

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ms per OSEM iteration, 128³/120 views, 1 B200: ESSE vs learned scatter at ≤1% NRMSE"
WORKLOAD = ("full128: 128^3 x 120 views, 8 subsets x 15 views, attenuation + 33x33 DRF + ESSE scatter "
            "(collapse 2, 2 Taylor terms), 5e6 counts, seed 2000")


def bench_config(world=1):
    """The workload description both arms print."""
    return {"workload": WORKLOAD, "parallelism": "replicas" if world > 1 else "single",
            "l2": "inputs larger than L2: per-view attenuation tables 2.8 GB streamed every iteration",
            "scatter": "ESSE recomputed in every iteration (iNumSrfIterations = iterations)"}


def _dup(s):
    libc = C.CDLL(None)
    libc.strdup.restype = C.c_void_p
    libc.strdup.argtypes = [C.c_char_p]
    return C.cast(libc.strdup(s.encode()), C.c_char_p) if s else None


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi samples every 200 ms while active."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ------------------------------------------------------------ ranks

def max_over_ranks(value, dist, failed=False):
    """(the maximum of value over all ranks, whether any rank failed).
    Every rank calls this at the same point, failed or not, so that the
    ranks' collectives match; without a process group it returns its
    arguments."""
    if not dist:
        return value, failed
    import torch
    dist.barrier()
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value), 1.0 if failed else 0.0], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t[0].item()), bool(t[1].item() > 0.0)


# --------------------------------------------------------------- workload

def make_workload(lib, tmpdir, nviews=120, subsets=8):
    from libirl_b200 import api, workloads as W
    case = W.full128(seed=2000, nviews=nviews, subsets=subsets)
    files = case.write_tables(tmpdir)
    p, o, v = case.parms(), case.options(), case.views()
    act, atn = case.act.copy(), case.atn.copy()
    prj = np.zeros((case.nviews, case.nz, case.n), np.float32)
    rc = lib.IrlGenprj(C.byref(p), C.byref(o), v, _dup(files["drf"]), _dup(files["krnl"]), None, None,
                       api.fptr(act), api.fptr(atn), api.fptr(prj), 1.0, None, None)
    if rc:
        raise RuntimeError(lib.pchIrlErrorString().decode())
    meas = W.poisson_counts(prj, case.counts, 2000)
    return case, files, meas


def run_b200(args):
    import torch
    import libirl_b200 as L
    from libirl_b200 import api

    rank, world = int(os.environ.get("RANK", "0")), _WORLD
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(0)
    L.build()
    lib = L.load()
    tmp = tempfile.mkdtemp(prefix="irlbench_")
    case, files, meas = make_workload(lib, tmp, args.nviews, args.subsets)
    K, Wm, P = args.steps, args.warmup, 1
    n3 = case.n * case.nz * case.n

    # --- device-resident timing through the session API
    p, o, v = case.parms(), case.options(), case.views()
    p.NumIterations = Wm + K + P
    # every iteration recomputes the ESSE source, as all 10 iterations of the
    # workload do (iNumSrfIterations = NumIterations)
    p.iNumSrfIterations = p.NumIterations
    atn = case.atn.copy()
    rec = np.zeros_like(case.act)
    m = meas.copy()
    rc = lib.IrlOsemBegin(C.byref(p), C.byref(o), v, _dup(files["drf"]), _dup(files["krnl"]),
                          api.ITER_CB(), None, api.fptr(atn), api.fptr(m), api.fptr(rec), None, None)
    if rc:
        raise RuntimeError(lib.pchIrlErrorString().decode())
    grids = (C.c_int * 5)()
    lib.irlcu_grids(grids)
    tune = (C.c_float * 2)()
    lib.irlcu_drf_tuning(tune)
    stream = torch.cuda.ExternalStream(lib.irlcu_stream())
    if lib.IrlOsemIterate(Wm):
        raise RuntimeError(lib.pchIrlErrorString().decode())
    gpu_index = int(os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0] or 0)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = lib.irlcu_launch_count()
    with ClockSampler(gpu_index) as clk:
        ev0.record(stream)
        rc = lib.IrlOsemIterate(K)
        ev1.record(stream)
        torch.cuda.synchronize()
    launches = lib.irlcu_launch_count() - l0
    ms_total, failed = max_over_ranks(ev0.elapsed_time(ev1), dist, failed=bool(rc))
    if rc:
        raise RuntimeError(lib.pchIrlErrorString().decode())
    if failed:
        raise RuntimeError("another rank's timed iterations failed")
    ms_step = ms_total / K

    # the shape autotuner decided during the warm-up iterations
    shear_ms, shear_form = (C.c_float * 4)(), (C.c_int * 2)()
    lib.irlcu_shear_tuning(shear_ms, shear_form)

    # --- stage profile over one more iteration (separate from the timing)
    lib.irlcu_profile_enable(1)
    lib.IrlOsemIterate(P)
    prof = L.IrlcuProfile()
    lib.irlcu_profile_read(C.byref(prof))
    lib.irlcu_profile_enable(0)
    lib.IrlOsemEnd(api.fptr(rec))

    # --- end to end: the public call with host buffers, E_IT iterations
    e2e = None
    if not args.no_e2e:
        E_IT = 10
        msgs = os.path.join(tmp, "e2e_messages.txt")
        for it in (1, E_IT):  # a short warm-up call, then the timed one
            p, o, v = case.parms(), case.options(), case.views()
            p.NumIterations = it
            o.iMsgLevel = 5  # the library's own phase timings, to a file
            atn = case.atn.copy()
            rec = np.zeros_like(case.act)
            m = meas.copy()
            cb = api.ITER_CB(lambda i, q: None)
            t0 = time.perf_counter()
            rc = lib.IrlOsem(C.byref(p), C.byref(o), v, _dup(files["drf"]), _dup(files["krnl"]), cb, None,
                             api.fptr(atn), api.fptr(m), api.fptr(rec), None, msgs.encode())
            wall = time.perf_counter() - t0
            if rc:
                raise RuntimeError(lib.pchIrlErrorString().decode())
        phases = _message_phases(msgs)
        # diagnostic split of the same call (not the reported number)
        p, o, v = case.parms(), case.options(), case.views()
        p.NumIterations = E_IT
        atn, rec, m = case.atn.copy(), np.zeros_like(case.act), meas.copy()
        t0 = time.perf_counter()
        lib.IrlOsemBegin(C.byref(p), C.byref(o), v, _dup(files["drf"]), _dup(files["krnl"]), cb, None,
                         api.fptr(atn), api.fptr(m), api.fptr(rec), None, None)
        t1 = time.perf_counter()
        lib.IrlOsemIterate(E_IT)
        t2 = time.perf_counter()
        lib.IrlOsemEnd(api.fptr(rec))
        t3 = time.perf_counter()
        phases["split_begin_iterate_end_s"] = [round(t1 - t0, 4), round(t2 - t1, 4), round(t3 - t2, 4)]
        h2d = (meas.nbytes + case.atn.nbytes + case.act.nbytes) / E_IT
        d2h = (case.act.nbytes * E_IT + case.act.nbytes) / E_IT
        e2e = {"value": round(1000.0 * wall / E_IT, 3), "unit": "ms", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "iterations": E_IT,
               "includes": "set-up (tables, ESSE kernel spectra, attenuation tables, 8 norm images), "
                           "host<->device copies from pageable memory, per-iteration callback",
               "phases_s": phases}

    learned = None
    if not args.no_surrogate and case.n == 128:
        learned = measure_learned_scatter(lib, case, files, meas, K, Wm, ms_step, torch)
    extra = {}
    if rank == 0 and world == 1 and not args.no_extra:
        for name, fn in (("batch32", run_batch32), ("large256", run_large256)):
            try:
                extra[name] = fn(args)
            except Exception as e:  # reported beside the line, never instead of it
                extra[name] = {"error": str(e)[:300]}

    clocks = clk.summary()
    roofline = make_roofline(prof, case, list(grids))
    stages = {L.STAGES[i]: {"ms": round(prof.ms[i], 3), "launches": int(prof.launches[i]),
                            "gflop": round(prof.flops[i] / 1e9, 2), "gbyte": round(prof.bytes[i] / 1e9, 3)}
              for i in range(6)}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(case, files, views=args.cpu_views)
        except Exception as e:  # the baseline is reported, never the product
            cpu = {"value": None, "error": str(e)[:200]}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": round(ms_step / world, 3), "unit": "ms", "n_gpus": world, "steps": K,
        "warmup": Wm, "ms_per_step": round(ms_step, 3), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded phantom, Poisson data)",
        "config": bench_config(world),
        "tuning": {"drf_engine": ("fourier-domain %dx%d grid" % (grids[0], grids[1])) if grids[0] else "direct",
                   "drf_autotune_ms": {"direct": round(tune[0], 3), "fourier": round(tune[1], 3)},
                   "shear_autotune_ms": {
                       src: {"one_slice": round(shear_ms[2 * k], 4), "two_slice": round(shear_ms[2 * k + 1], 4),
                             "kept": "two_slice" if shear_form[k] == 1 else "one_slice"}
                       for k, src in enumerate(("shared_source_rotation", "per_view_source_unrotation"))}},
        "e2e": e2e, "gpu_launches": int(launches), "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
        "stages_ms_per_iteration": {k: {**s, "ms": round(s["ms"] / P, 3)} for k, s in stages.items()},
        "learned_scatter": learned,
    }
    line.update(extra)
    print(json.dumps(line))


def _osem_image(lib, case, files, meas, iterations, srf_iters=None):
    from libirl_b200 import api
    p, o, v = case.parms(), case.options(), case.views()
    p.NumIterations = iterations
    if srf_iters is not None:
        p.iNumSrfIterations = srf_iters
    atn, rec, m = case.atn.copy(), np.zeros_like(case.act), meas.copy()
    rc = lib.IrlOsem(C.byref(p), C.byref(o), v, _dup(files["drf"]), _dup(files["krnl"]), api.ITER_CB(), None,
                     api.fptr(atn), api.fptr(m), api.fptr(rec), None, None)
    if rc:
        raise RuntimeError(lib.pchIrlErrorString().decode())
    return rec


def measure_learned_scatter(lib, case, files, meas, K, Wm, esse_ms, torch):
    """The same OSEM iteration with the learned scatter surrogate in place of
    ESSE (IrlSetScatterSurrogate with the committed weights): device time per
    iteration after the first iteration (ESSE on every view + the per-view
    NRMSE check), the per-view NRMSE against ESSE, and the image NRMSE of a
    10-iteration reconstruction against the ESSE one; the ablation is the
    reconstruction without scatter modelling."""
    from libirl_b200 import api
    from libirl_b200 import surrogate as SU
    wfile = SU.DEFAULT_WEIGHTS
    if not os.path.exists(wfile):
        return {"unavailable": "no trained weights (libirl_b200/surrogate/sur128.bin)"}
    lib.IrlSetScatterSurrogate(wfile.encode(), 0.02)
    try:
        p, o, v = case.parms(), case.options(), case.views()
        p.NumIterations = 1 + Wm + K
        p.iNumSrfIterations = p.NumIterations
        atn, rec, m = case.atn.copy(), np.zeros_like(case.act), meas.copy()
        rc = lib.IrlOsemBegin(C.byref(p), C.byref(o), v, _dup(files["drf"]), _dup(files["krnl"]), api.ITER_CB(),
                              None, api.fptr(atn), api.fptr(m), api.fptr(rec), None, None)
        if rc:
            raise RuntimeError(lib.pchIrlErrorString().decode())
        try:
            lib.IrlOsemIterate(1 + Wm)
            nr = np.zeros(case.nviews, np.float32)
            lib.IrlGetScatterSurrogateNrmse(api.fptr(nr), case.nviews)
            stream = torch.cuda.ExternalStream(lib.irlcu_stream())
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            rc = lib.IrlOsemIterate(K)
            e1.record(stream)
            torch.cuda.synchronize()
            if rc:
                raise RuntimeError(lib.pchIrlErrorString().decode())
            ms = e0.elapsed_time(e1) / K
        finally:
            lib.IrlOsemEnd(None)
        sur_img = _osem_image(lib, case, files, meas, 10)
    finally:
        lib.IrlSetScatterSurrogate(None, 0.0)
    esse_img = _osem_image(lib, case, files, meas, 10)
    none_img = _osem_image(lib, case, files, meas, 10, srf_iters=0)
    ref = np.linalg.norm(esse_img)
    return {
        "ms_per_iteration": round(ms, 3), "esse_ms_per_iteration": round(esse_ms, 3),
        "speedup_vs_esse": round(esse_ms / ms, 3) if ms > 0 else None,
        "image_nrmse_vs_esse": round(float(np.linalg.norm(sur_img - esse_img) / ref), 5),
        "image_nrmse_no_scatter_vs_esse": round(float(np.linalg.norm(none_img - esse_img) / ref), 5),
        "views_on_esse": int((nr > 0.02).sum()),
        "view_nrmse": {"mean": round(float(nr.mean()), 5), "median": round(float(np.median(nr)), 5),
                       "max": round(float(nr.max()), 5)},
        "nrmse": "||x - x_ESSE|| / ||x_ESSE||; per view on the scatter projection after iteration 1",
        "reconstruction": "config-2 data, 10 iterations, scatter model in all of them",
    }


def _message_phases(path):
    """Set-up and per-iteration wall times the library itself logged."""
    out = {"setup": None, "norms": None, "iterations": []}
    try:
        for line in open(path):
            if line.startswith("Done Initialization"):
                out["setup"] = float(line.split("(")[1].split()[0])
            elif line.startswith(("Done scatter kernel", "Done DRF tables", "Done host set-up",
                                  "Done device set-up")):
                key = line.split("(")[0].replace("Done", "").strip().replace(" ", "_").replace("-", "_")
                out.setdefault("setup_marks", {})[key] = float(line.split("(")[1].split()[0])
            elif line.startswith("Done Computing Norm Matrix"):
                out["norms"] = float(line.split("(")[1].split()[0])
            elif "Done iteration" in line:
                out["iterations"].append(float(line.split("(")[1].split()[0]))
    except (OSError, ValueError, IndexError):
        pass
    return out


def _traffic_from_profiles(name, key):
    """DRAM bytes (ncu dram__bytes_read + write) recorded in a committed
    profile summary under profiles/, or None."""
    try:
        for line in open(os.path.join(ROOT, "profiles", name)):
            if line.startswith(key + ":"):
                return float(line.split(":")[1])
    except (OSError, ValueError):
        pass
    return None


def _hbm_peak():
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(peaks["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def make_roofline(prof, case, grids):
    """Roofline of the stage with the largest device time in an OSEM
    iteration, with the other stages beside it.  Algorithmic bytes per view
    follow the per-unit figures of the hot-path scope table (b = 4 bytes,
    V = N^2 Nz voxels, P = N Nz bins):

      ESSE: 3 3D transforms x 3 passes of >= 2 b G (G = Kx Ky Kz), plus
        3 b V for the depth/density combination;
      DRF, Fourier domain (projector + backprojector): per plane 3 2D
        transforms (one forward, forward + inverse backward) x 2 passes of
        >= 2 b Mz Mx; also 5 n log2 n FP32 FLOP per complex transform of
        n = Mz Mx points, against the nominal FP32 peak (the one-CTA-per-
        plane kernels keep the passes in shared memory, so their DRAM
        traffic is far below those bytes);
      rotate: 2 b V per view;
      unrotate + accumulate: 2 b V per view (unrotation) + b V per view
        (accumulation read) + 2 b V per subset (accumulator).

    achieved = those bytes per subset / the stage's device time per subset
    (CUDA events around the stage on the library stream); peak = the
    measured HBM copy bandwidth.  `traffic` = ncu DRAM read + write bytes
    per subset from profiles/osem_subset_full128_traffic.md."""
    peak, src = _hbm_peak()
    n, nz = case.n, case.nz
    vox = n * nz * n
    mz, mx, kx, ky, kz = grids
    subsets = case.subsets
    per = case.nviews // subsets
    b = 4
    stages = []
    if kx:
        stages.append(("esse", (1,), per * (3 * 3 * (2 * b * kx * ky * kz) + 3 * b * vox),
                       "k_esse_row_fwd_reg / k_esse_yz_reg / k_esse_row_inv_reg / k_expand_y / k_smooth_z / "
                       "k_smooth_x_combine (ESSE)"))
    if mz and mx:
        stages.append(("drf", (2, 4), per * n * 3 * 2 * (2 * b * mz * mx),
                       "k_dplane_fwd / k_dplane_fwd_finish / k_dplane_bck (Fourier-domain DRF, one CTA per plane)"))
    # with ESSE at collapse 2 the rotation also writes the collapsed volume
    col = b * vox // 8 if (kx and case.collapse == 2) else 0
    stages.append(("rotate", (0,), per * (2 * b * vox + col),
                   "k_shear_cw2 (three-shear rotation, two slices per CTA; with ESSE it also writes the 2x2x2 "
                   "collapse, b*V/8 per view)"))
    stages.append(("unrotate", (5,), per * 3 * b * vox + 2 * b * vox, "k_shear_cw + k_accumulate"))
    fp32_peak = 148 * 128 * 2 * 1.965e9 / 1e12  # nominal SIMT FP32 TFLOP/s (not measured)
    out = []
    for k, idx, bytes_subset, kern in stages:
        ms = sum(prof.ms[i] for i in idx) / subsets
        if ms <= 0:
            continue
        gbs = bytes_subset / (ms * 1e-3) / 1e9
        tr = _traffic_from_profiles("osem_subset_full128_traffic.md", "traffic_bytes_per_subset_" + k)
        r = {"stage": k, "kernel": kern, "bound": "hbm", "achieved": round(gbs, 1), "peak": peak, "unit": "GB/s",
             "frac": round(gbs / peak, 3), "peak_source": src, "traffic": tr,
             "algorithmic_bytes_per_launch": int(bytes_subset), "launch_ms": round(ms, 4),
             "launch": f"one subset ({per} views)"}
        if k == "drf":
            flop = per * n * 3 * 5 * (mz * mx) * math.log2(mz * mx)
            tf = flop / (ms * 1e-3) / 1e12
            r["fp32"] = {"achieved_tflops": round(tf, 2), "peak_tflops": round(fp32_peak, 1),
                         "frac": round(tf / fp32_peak, 3), "peak_source": "nominal (148 SMs x 128 lanes x 2 x 1.965 GHz)"}
        out.append(r)
    if not out:
        return None
    out.sort(key=lambda r: -r["launch_ms"])
    top = dict(out[0])
    top["other_stages"] = out[1:]
    return top


# ------------------------------------------------------------- CPU baseline

def _ref_view_timer(case, files):
    """Returns f(view) -> seconds of one view of an OSEM iteration
    (Project with ESSE + DRF + attenuation, BackProject with DRF +
    attenuation) run by the reference compiled here, and the kind."""
    from libirl_b200 import api
    from oracle import oracle as O
    atn_i = O.to_internal(case.atn * np.float32(case.atn_scale))
    est_i = O.to_internal(case.act)
    n, nz = case.n, case.nz
    if O.have_ref():
        ref = O.ref()
        F, I, FL = api.FLOAT_P, C.c_int, C.c_float

        class Srf(C.Structure):
            _fields_ = [("c", C.c_int), ("line", C.c_int), ("data", C.c_void_p)]

        ref.pvInitESSEScatterModel.restype = C.c_void_p
        ref.pvInitESSEScatterModel.argtypes = [C.c_char_p, C.c_char_p, FL, I, I, I, I]
        ref.Project.restype = None
        ref.Project.argtypes = [I, I, I, I, FL, I, FL, FL, C.POINTER(api.DrfTab), C.POINTER(Srf), F, F, F, FL, FL,
                                I, I, I, I, I]
        ref.BackProject.restype = None
        ref.BackProject.argtypes = [I, I, I, I, FL, I, FL, FL, C.POINTER(api.DrfTab), C.POINTER(Srf), F, F, F, FL,
                                    FL, I, I, I, I]
        title, col = C.c_char_p(), C.c_char_p()
        tab = ref.sReadDrfTab(files["drf"].encode(), C.byref(title), C.byref(col))
        tab.psBckDrfTab = None
        # sReadDrfTab leaves the convolution switch unset (IrlSetup.c:577
        # sets it from the options); this workload's tables are spatial
        tab.bFFTconvolve = 0
        srf = Srf(case.collapse, 0, ref.pvInitESSEScatterModel(files["krnl"].encode(), b"2 2 2 3", case.pix, n, nz,
                                                                case.collapse, 0))
        ref.InitPrj(nz, n, n, 7)
        calc = np.zeros((nz, n), np.float32)
        img = np.zeros_like(est_i)

        def one(view):
            a, r = float(case.angles[view]), float(case.cfcr[view])
            t0 = time.perf_counter()
            ref.Project(nz, n, n, 7, case.pix, view, a, r, C.byref(tab), C.byref(srf), api.fptr(atn_i),
                        api.fptr(est_i), api.fptr(calc), 1.0, 1.0, 0, 0, 0, 0, 1)
            ratio = np.where(calc > 1e-20, 1.0 / np.maximum(calc, 1e-20), 0).astype(np.float32)
            ref.BackProject(nz, n, n, 3, case.pix, view, a, r, C.byref(tab), C.byref(srf), api.fptr(atn_i),
                            api.fptr(ratio), api.fptr(img), 1.0, 1.0, 0, 0, 1, 1)
            return time.perf_counter() - t0
        return one, "reference"
    pr = O.Problem(case)
    calc = np.zeros((nz, n), np.float32)
    img = np.zeros_like(est_i)

    def one_port(view):
        t0 = time.perf_counter()
        O.orc().or_project(C.byref(pr.P), 7, view, api.fptr(est_i), api.fptr(pr.atn), 1.0, api.fptr(calc))
        ratio = np.where(calc > 1e-20, 1.0 / np.maximum(calc, 1e-20), 0).astype(np.float32)
        O.orc().or_backproject(C.byref(pr.P), 3, view, api.fptr(pr.atn), api.fptr(ratio), api.fptr(img))
        return time.perf_counter() - t0
    return one_port, "port"


def cpu_baseline(case, files, views=2):
    one, kind = _ref_view_timer(case, files)
    sel = [0, case.nviews // 3, 2 * case.nviews // 3][:max(1, views)]
    secs = [one(v) for v in sel]
    per_view = statistics.mean(secs)
    return {"value": round(1000.0 * per_view * case.nviews, 1), "unit": "ms", "cores": 1, "kind": kind,
            "sample": f"{len(sel)} of {case.nviews} views of one OSEM iteration (projection with ESSE + DRF + "
                      f"attenuation and DRF + attenuation backprojection), single-threaded reference C, "
                      f"mean {per_view:.2f} s/view, extrapolated x{case.nviews}",
            "threads_available": os.cpu_count()}


# ---------------------------------------------------------- reference arm
#
# libirl keeps global state and has no threads, so the reference arm gives
# every host core its own spawned process holding the compiled reference
# (oracle/_ref; the restatement where it was not built).  One step is one
# OSEM sub-iteration of the workload as vOsemRecon runs it
# (osemrecon.c:687-852), the subsets taken in order: the subset's 15 views
# run at once, one per process -- Project with ESSE + DRF + attenuation,
# the time scaling, the non-measured-bin mask, the ratio, BackProject with
# DRF + attenuation of the ratio -- and the parent adds their
# backprojections in view order with the clamp of prjbck.c:418-426 and
# applies the EM update x *= U * Ninv (osemrecon.c:850-852).  The metric
# (ms per iteration) is the sum over the 8 subsets of each subset's median
# step, so every subset of the iteration is measured once K >= 8; a whole
# iteration per step would take about half a minute here, too long for K
# steps to end within a few minutes.  The estimate, the measured data and
# the per-view backprojections live in shared memory.

_REF = None  # per worker process


def _ref_worker_init(seed, files, shm_names, procs):
    from multiprocessing import shared_memory
    global _REF
    import libirl_b200.workloads as W
    from libirl_b200 import api
    from oracle import oracle as O
    case = W.full128(seed=seed)
    n, nz, nv = case.n, case.nz, case.nviews
    vox, pl = n * nz * n, nz * n
    shms = [shared_memory.SharedMemory(name=nm) for nm in shm_names]
    est = np.ndarray((vox,), np.float32, buffer=shms[0].buf)
    meas = np.ndarray((nv, pl), np.float32, buffer=shms[1].buf)
    slots = np.ndarray((procs, vox), np.float32, buffer=shms[2].buf)
    atn = O.to_internal(case.atn * np.float32(case.atn_scale))
    calc = np.zeros((pl,), np.float32)
    F, I, FL = api.FLOAT_P, C.c_int, C.c_float
    st = {"case": case, "shms": shms, "est": est, "meas": meas, "slots": slots, "atn": atn, "calc": calc}
    if O.have_ref():
        ref = O.ref()

        class Srf(C.Structure):
            _fields_ = [("c", C.c_int), ("line", C.c_int), ("data", C.c_void_p)]

        ref.pvInitESSEScatterModel.restype = C.c_void_p
        ref.pvInitESSEScatterModel.argtypes = [C.c_char_p, C.c_char_p, FL, I, I, I, I]
        ref.Project.restype = None
        ref.Project.argtypes = [I, I, I, I, FL, I, FL, FL, C.POINTER(api.DrfTab), C.POINTER(Srf), F, F, F, FL, FL,
                                I, I, I, I, I]
        ref.BackProject.restype = None
        ref.BackProject.argtypes = [I, I, I, I, FL, I, FL, FL, C.POINTER(api.DrfTab), C.POINTER(Srf), F, F, F, FL,
                                    FL, I, I, I, I]
        title, col = C.c_char_p(), C.c_char_p()
        tab = ref.sReadDrfTab(files["drf"].encode(), C.byref(title), C.byref(col))
        tab.psBckDrfTab = None
        # sReadDrfTab leaves the convolution switch unset (IrlSetup.c:577
        # sets it from the options); this workload's tables are spatial
        tab.bFFTconvolve = 0
        srf = Srf(case.collapse, 0, ref.pvInitESSEScatterModel(files["krnl"].encode(), b"2 2 2 3", case.pix, n, nz,
                                                                case.collapse, 0))
        ref.InitPrj(nz, n, n, 7)

        def project(view, model, out):
            ref.Project(nz, n, n, model, case.pix, view, float(case.angles[view]), float(case.cfcr[view]),
                        C.byref(tab), C.byref(srf), api.fptr(atn), api.fptr(est), api.fptr(out), 1.0, 1.0,
                        0, 0, 0, 0, 1)

        def backproject(view, ratio, image, atn_rotated):
            ref.BackProject(nz, n, n, 3, case.pix, view, float(case.angles[view]), float(case.cfcr[view]),
                            C.byref(tab), C.byref(srf), api.fptr(atn), api.fptr(ratio), api.fptr(image), 1.0,
                            1.0, 0, 0, int(atn_rotated), 1)
        st["kind"] = "reference"
    else:
        pr = O.Problem(case)
        st["pr"] = pr

        def project(view, model, out):
            O.orc().or_project(C.byref(pr.P), model, view, api.fptr(est), api.fptr(pr.atn), 1.0, api.fptr(out))

        def backproject(view, ratio, image, atn_rotated):
            O.orc().or_backproject(C.byref(pr.P), 3, view, api.fptr(pr.atn), api.fptr(ratio), api.fptr(image))
        st["kind"] = "port"
    st["project"], st["backproject"] = project, backproject
    _REF = st


def _ref_genprj_view(view):
    """Set-up: the noise-free projection of the phantom (in the shared
    estimate) for one view, as IrlGenprj computes it (irlgenprj.c:225-264)."""
    st = _REF
    out = np.zeros_like(st["calc"])
    st["project"](view, 7, out)
    return view, out * np.float32(1.0 / st["case"].nviews)


def _ref_norm_view(args):
    """Set-up: one view's share of its subset's norm image
    (osemrecon.c:223-343): the measured-bin mask times ViewTime, backprojected."""
    view, slot = args
    st = _REF
    ratio = np.where(st["meas"][view] >= 0.0, np.float32(1.0), np.float32(0.0)).astype(np.float32)
    image = st["slots"][slot]
    image[:] = 0.0
    st["backproject"](view, ratio, image, False)
    return 0.0


def _ref_member(args):
    """One view of an OSEM sub-iteration (osemrecon.c:712-830), its
    backprojection left in its shared slot."""
    view, slot = args
    st = _REF
    t0 = time.perf_counter()
    calc = st["calc"]
    st["project"](view, 7, calc)
    calc *= np.float32(1.0)  # ViewTime * Sensitivity
    calc[st["meas"][0] < 0.0] = 0.0  # SetNonMeasuredBinsToZero (view 0's data, osemrecon.c:802-803)
    meas = st["meas"][view]
    ratio = np.zeros_like(calc)
    np.divide(meas, calc, out=ratio, where=calc > 1e-20)
    ratio *= np.float32(1.0)  # ViewTime
    image = st["slots"][slot]
    image[:] = 0.0
    st["backproject"](view, ratio, image, True)
    return time.perf_counter() - t0


def run_reference(args):
    """Reference arm (see the block comment above).  Warm-up steps and the K
    timed steps each run one sub-iteration, the subsets in order;
    ms_per_step = the mean timed step (so steps x ms_per_step is the timed
    region) and value = ms per iteration = the sum over the subsets of each
    subset's median step (the mean step x the subset count while K < the
    subset count).  Under torchrun rank 0 alone runs."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import multiprocessing as mp
    from multiprocessing import shared_memory
    import libirl_b200.workloads as W
    from oracle import oracle as O
    seed = 2000
    case = W.full128(seed=seed)
    n, nz, nv = case.n, case.nz, case.nviews
    vox, pl = n * nz * n, nz * n
    per = nv // case.subsets
    ns = case.subsets
    try:
        procs = len(os.sched_getaffinity(0))
    except AttributeError:
        procs = os.cpu_count() or 1
    procs = max(1, min(procs, per))
    tmp = tempfile.mkdtemp(prefix="irlbench_ref_")
    files = case.write_tables(tmp)
    shms = []
    pool = acc_pool = None
    try:
        for size in (vox * 4, nv * pl * 4, per * vox * 4):
            shms.append(shared_memory.SharedMemory(create=True, size=size))
        est = np.ndarray((vox,), np.float32, buffer=shms[0].buf)
        meas = np.ndarray((nv, pl), np.float32, buffer=shms[1].buf)
        slots = np.ndarray((per, vox), np.float32, buffer=shms[2].buf)
        kind = "reference" if O.have_ref() else "port"
        pool = mp.get_context("spawn").Pool(procs, initializer=_ref_worker_init,
                                             initargs=(seed, files, [m.name for m in shms], per))
        subset_views = [[s // 2 + (s % 2) * ns // 2 + m * ns for m in range(per)] for s in range(ns)]
        # set-up (untimed): Poisson data from the reference's own projections,
        # the norm images, the uniform initial estimate (initial_est.c:29-153)
        est[:] = O.to_internal(case.act).ravel()
        clean = np.zeros((nv, pl), np.float32)
        for view, prj in pool.imap_unordered(_ref_genprj_view, range(nv)):
            clean[view] = prj
        meas[:] = W.poisson_counts(clean, case.counts, seed)
        norms = np.zeros((ns, vox), np.float32)
        for s in range(ns):
            pool.map(_ref_norm_view, [(v, m) for m, v in enumerate(subset_views[s])], chunksize=1)
            for m in range(per):
                norms[s] += slots[m]
                norms[s][norms[s] < 1e-5] = 0.0
            nz_ = norms[s] >= 1e-6
            norms[s][~nz_] = 0.0
            norms[s][nz_] = np.float32(1.0) / norms[s][nz_]
        avg = np.float32(meas.sum(dtype=np.float32) / np.float32(np.pi / 4 * n * n * nz * nv))
        yy, xx = np.meshgrid(np.arange(n, dtype=np.float32) - n / 2, np.arange(n, dtype=np.float32) - n / 2,
                             indexing="ij")
        yy[yy > 0] += 1
        xx[xx > 0] += 1
        inside = np.hypot(xx, yy) <= n / 2
        est.reshape(n, nz, n)[:] = np.where(inside[:, None, :], avg, np.float32(0.0))
        upd = np.zeros((vox,), np.float32)
        from concurrent.futures import ThreadPoolExecutor
        acc_pool = ThreadPoolExecutor(max_workers=procs)
        chunks = [(vox * i // 16, vox * (i + 1) // 16) for i in range(16)]

        def accumulate(s, lo, hi):
            # the worker processes are idle meanwhile, so the ordered clamped
            # accumulation and the EM update run on host threads, a slab each
            u = upd[lo:hi]
            u[:] = 0.0
            for m in range(per):
                np.add(u, slots[m, lo:hi], out=u)
                np.copyto(u, 0.0, where=u < 1e-5)
            est[lo:hi] *= u * norms[s, lo:hi]

        def sub_iteration(s):
            pool.map(_ref_member, [(v, m) for m, v in enumerate(subset_views[s])], chunksize=1)
            list(acc_pool.map(lambda c: accumulate(s, *c), chunks))

        for i in range(args.warmup):
            sub_iteration(i % ns)
        walls, by_subset = [], {}
        for i in range(args.steps):
            s = (args.warmup + i) % ns
            t0 = time.perf_counter()
            sub_iteration(s)
            w = time.perf_counter() - t0
            walls.append(w)
            by_subset.setdefault(s, []).append(w)
    except Exception as e:
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU path failed: {e}"[:300]}))
        return
    finally:
        if pool is not None:
            pool.close()
            pool.join()
        if acc_pool is not None:
            acc_pool.shutdown()
        for m in shms:
            m.close()
            m.unlink()
    step_ms = round(1000.0 * statistics.mean(walls), 1)
    whole = len(by_subset) == ns
    if whole:
        val = round(1000.0 * sum(statistics.median(w) for w in by_subset.values()), 1)
        how = f"sum over the {ns} subsets of each subset's median step"
    else:
        val = round(1000.0 * statistics.mean(walls) * ns, 1)
        how = f"mean step x {ns} (fewer steps than subsets)"
    line = {
        "metric": METRIC, "value": val, "unit": "ms", "n_gpus": _WORLD, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded phantom, Poisson data)",
        "config": bench_config(_WORLD), "impl": "reference",
        "cpu_baseline": {"value": val, "unit": "ms", "cores": procs, "kind": kind,
                         "sample": f"each step one OSEM sub-iteration ({per} views, ESSE in the projector, "
                                   f"spatial 33x33 DRF), the {ns} subsets in order; a subset's views run at "
                                   f"once in {procs} processes of the compiled reference, the parent adds their "
                                   f"backprojections in view order with the clamp and applies the EM update; "
                                   f"ms per iteration = {how}; {len(walls)} steps, "
                                   f"min {1000 * min(walls):.0f} ms, max {1000 * max(walls):.0f} ms per step",
                         "threads_available": os.cpu_count()},
        "e2e": {"value": val, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ------------------------------------------------- further workloads (manual)

def _genprj(lib, case, files, primary=1.0, fft=False):
    from libirl_b200 import api
    p, o, v = case.parms(), case.options(), case.views()
    if fft:
        o.bFFTConvolve = 1
    act, atn = case.act.copy(), case.atn.copy()
    prj = np.zeros((case.nviews, case.nz, case.n), np.float32)
    rc = lib.IrlGenprj(C.byref(p), C.byref(o), v, _dup(files["drf"]), _dup(files["krnl"]), None, None,
                       api.fptr(act), api.fptr(atn), api.fptr(prj), primary, None, None)
    if rc:
        raise RuntimeError(lib.pchIrlErrorString().decode())
    return prj


def run_batch32(args):
    """Config 3: 32 seeded problems of uneven size (N 64..128, 60..120
    views, 4..12 subsets, DRF + ESSE), 5 iterations each: IrlOsemBatch
    against the same 32 IrlOsem calls one after another, wall time, after
    one untimed batch pass (table autotuning and module loading); medians
    of three alternating repeats."""
    import torch  # noqa: F401  (CUDA context for the library)
    import libirl_b200 as L
    from libirl_b200 import api, workloads as W
    lib = L.load()
    tmp = tempfile.mkdtemp(prefix="irlbatch_")
    cases = W.batch32(iterations=5)
    data = []
    for j, case in enumerate(cases):
        files = case.write_tables(os.path.join(tmp, f"c{j}"))
        meas = W.poisson_counts(_genprj(lib, case, files), case.counts, 3000 + j)
        data.append((case, files, meas))

    def batch(iters=None):
        probs = (api.OsemProblem * len(data))()
        keep = []
        for q, (case, files, meas) in zip(probs, data):
            p, o, v = case.parms(), case.options(), case.views()
            if iters is not None:
                p.NumIterations = iters
            atn, prj, rec = case.atn.copy(), meas.copy(), np.zeros_like(case.act)
            keep.append((p, o, v, atn, prj, rec))
            q.psIrlParms, q.psOptions = C.pointer(p), C.pointer(o)
            q.psViews = C.cast(v, C.POINTER(api.PrjView))
            q.pchDrfTabFname = C.cast(_dup(files["drf"]), C.c_void_p)
            q.pchScatKrnlFname = C.cast(_dup(files["krnl"]), C.c_void_p)
            q.pfAtnMap, q.pfPrjImage, q.pfReconImage = api.fptr(atn), api.fptr(prj), api.fptr(rec)
        t0 = time.perf_counter()
        rc = lib.IrlOsemBatch(len(data), probs)
        wall = time.perf_counter() - t0
        if rc:
            raise RuntimeError(lib.pchIrlErrorString().decode())
        return wall, [k[5] for k in keep]

    def sequential(iters=None):
        out = []
        t0 = time.perf_counter()
        for case, files, meas in data:
            out.append(_osem_image(lib, case, files, meas, iters or case.iterations))
        return time.perf_counter() - t0, out

    batch()
    # the small problems make both forms sensitive to host load on a shared
    # machine, so each is timed in three alternating repeats and the medians
    # are reported (every sample beside them)
    samples = {"sequential": [], "batched": [], "sequential_1it": [], "batched_1it": []}
    same = True
    for _ in range(3):
        seq_s, seq_imgs = sequential()
        bat_s, bat_imgs = batch()
        same = same and all(np.array_equal(a, b) for a, b in zip(seq_imgs, bat_imgs))
        # the iteration phase alone: 5 iterations minus 1 (set-up and the
        # first iteration cancel)
        seq1, _ = sequential(1)
        bat1, _ = batch(1)
        for k, t in (("sequential", seq_s), ("batched", bat_s), ("sequential_1it", seq1), ("batched_1it", bat1)):
            samples[k].append(round(t, 3))
    seq_s, bat_s = float(np.median(samples["sequential"])), float(np.median(samples["batched"]))
    seq1, bat1 = float(np.median(samples["sequential_1it"])), float(np.median(samples["batched_1it"]))
    iters = sum(c.iterations for c, _, _ in data)
    it_seq, it_bat = seq_s - seq1, bat_s - bat1
    return {
        "metric": "wall s for 32 uneven OSEM reconstructions (5 iterations each), 1 B200", "value": round(bat_s, 3),
        "unit": "s", "n_gpus": 1, "higher_is_better": False, "impl": "b200 IrlOsemBatch",
        "sequential_s": round(seq_s, 3), "speedup_vs_sequential": round(seq_s / bat_s, 3),
        "ms_per_problem_iteration": round(1000 * bat_s / iters, 3), "identical_to_sequential": bool(same),
        "iterations_2_to_5_s": {"batched": round(it_bat, 3), "sequential": round(it_seq, 3),
                                "speedup": round(it_seq / it_bat, 3) if it_bat > 0 else None},
        "samples_s": samples, "timing": "median of 3 alternating repeats",
        "config": {"workload": "batch32: " + ", ".join(f"{c.n}^3/{c.nviews}v/{c.subsets}s" for c, _, _ in data),
                   "includes": "set-up (tables, norm images) and result copies of every problem"},
        "data": "synthetic (seeded phantoms, Poisson data)"}


def _recon256(lib, case, files, meas, iterations, srf_iters=None):
    from libirl_b200 import api
    p, o, v = case.parms(), case.options(), case.views()
    o.bFFTConvolve = 1
    p.NumIterations = iterations
    p.iNumSrfIterations = iterations if srf_iters is None else srf_iters
    atn, rec, m = case.atn.copy(), np.zeros_like(case.act), meas.copy()
    rc = lib.IrlOsem(C.byref(p), C.byref(o), v, _dup(files["drf"]), _dup(files["krnl"]), api.ITER_CB(), None,
                     api.fptr(atn), api.fptr(m), api.fptr(rec), None, None)
    if rc:
        raise RuntimeError(lib.pchIrlErrorString().decode())
    return rec


def large256_learned(lib, case, files, meas, K, Wm, esse_ms, torch):
    """The 256^3 photopeak window with the learned scatter surrogate trained
    on 256^3 phantoms (libirl_b200/surrogate/sur256.bin): device time per
    iteration after the first (ESSE) iteration, and the image NRMSE of the
    8-iteration reconstruction against the ESSE one and without scatter."""
    from libirl_b200 import api
    from libirl_b200 import surrogate as SU
    if not os.path.exists(SU.WEIGHTS_256):
        return {"unavailable": "no trained 256^3 weights (libirl_b200/surrogate/sur256.bin)"}
    lib.IrlSetScatterSurrogate(SU.WEIGHTS_256.encode(), 0.02)
    try:
        p, o, v = case.parms(), case.options(), case.views()
        o.bFFTConvolve = 1
        p.NumIterations = 1 + Wm + K
        p.iNumSrfIterations = p.NumIterations
        atn, rec, m = case.atn.copy(), np.zeros_like(case.act), meas.copy()
        rc = lib.IrlOsemBegin(C.byref(p), C.byref(o), v, _dup(files["drf"]), _dup(files["krnl"]), api.ITER_CB(),
                              None, api.fptr(atn), api.fptr(m), api.fptr(rec), None, None)
        if rc:
            raise RuntimeError(lib.pchIrlErrorString().decode())
        try:
            lib.IrlOsemIterate(1 + Wm)
            nr = np.zeros(case.nviews, np.float32)
            lib.IrlGetScatterSurrogateNrmse(api.fptr(nr), case.nviews)
            stream = torch.cuda.ExternalStream(lib.irlcu_stream())
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            rc = lib.IrlOsemIterate(K)
            e1.record(stream)
            torch.cuda.synchronize()
            if rc:
                raise RuntimeError(lib.pchIrlErrorString().decode())
            ms = e0.elapsed_time(e1) / K
        finally:
            lib.IrlOsemEnd(None)
        sur_img = _recon256(lib, case, files, meas, case.iterations)
    finally:
        lib.IrlSetScatterSurrogate(None, 0.0)
    esse_img = _recon256(lib, case, files, meas, case.iterations)
    none_img = _recon256(lib, case, files, meas, case.iterations, srf_iters=0)
    ref = np.linalg.norm(esse_img)
    return {
        "ms_per_iteration": round(ms, 2), "esse_ms_per_iteration": round(esse_ms, 2),
        "speedup_vs_esse": round(esse_ms / ms, 3) if ms > 0 else None,
        "image_nrmse_vs_esse": round(float(np.linalg.norm(sur_img - esse_img) / ref), 5),
        "image_nrmse_no_scatter_vs_esse": round(float(np.linalg.norm(none_img - esse_img) / ref), 5),
        "views_on_esse": int((nr > 0.02).sum()),
        "view_nrmse": {"mean": round(float(nr.mean()), 5), "max": round(float(nr.max()), 5)},
        "reconstruction": f"{case.iterations} iterations of {case.subsets} subsets, scatter model in all",
    }


def run_large256(args):
    """Config 5: 256^3, 128 views, 16 subsets, 65 x 65 DRF on libirl's FFT
    convolution path, ESSE; IrlGenprj of the photopeak and the lower
    (scatter-only, fPrimaryFac = 0) window, and OSEM iterations of the
    photopeak window timed with CUDA events on the library stream."""
    import torch
    import libirl_b200 as L
    from libirl_b200 import api, workloads as W
    lib = L.load()
    tmp = tempfile.mkdtemp(prefix="irl256_")
    pp, lw = W.large256(window="photopeak"), W.large256(window="lower")
    fpp, flw = pp.write_tables(os.path.join(tmp, "pp")), lw.write_tables(os.path.join(tmp, "lw"))
    # the process's first device work (context creation, module loading) in
    # a small untimed IrlGenprj, so that the timed calls measure projection
    warm = W.full128(seed=1, n=32, nviews=8, subsets=2, iterations=1, drf_max_offs=6, name="warm")
    _genprj(lib, warm, warm.write_tables(os.path.join(tmp, "warm")), 1.0)
    t0 = time.perf_counter()
    prj = _genprj(lib, pp, fpp, 1.0, fft=True)
    g_pp = time.perf_counter() - t0
    t0 = time.perf_counter()
    _genprj(lib, lw, flw, 0.0, fft=True)
    g_lw = time.perf_counter() - t0
    meas = W.poisson_counts(prj, pp.counts, 5000)
    K, Wm = max(1, min(args.steps, 5)), 3
    p, o, v = pp.parms(), pp.options(), pp.views()
    o.bFFTConvolve = 1
    p.NumIterations = Wm + K
    p.iNumSrfIterations = p.NumIterations
    atn, rec, m = pp.atn.copy(), np.zeros_like(pp.act), meas.copy()
    rc = lib.IrlOsemBegin(C.byref(p), C.byref(o), v, _dup(fpp["drf"]), _dup(fpp["krnl"]), api.ITER_CB(), None,
                          api.fptr(atn), api.fptr(m), api.fptr(rec), None, None)
    if rc:
        raise RuntimeError(lib.pchIrlErrorString().decode())
    try:
        grids = (C.c_int * 5)()
        lib.irlcu_grids(grids)
        lib.IrlOsemIterate(Wm)
        stream = torch.cuda.ExternalStream(lib.irlcu_stream())
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rc = lib.IrlOsemIterate(K)
        e1.record(stream)
        torch.cuda.synchronize()
        if rc:
            raise RuntimeError(lib.pchIrlErrorString().decode())
        ms = e0.elapsed_time(e1) / K
    finally:
        lib.IrlOsemEnd(api.fptr(rec))
    learned = large256_learned(lib, pp, fpp, meas, K, Wm, ms, torch)
    return {
        "metric": "ms per OSEM iteration, 256^3/128 views/16 subsets, 65x65 FFT DRF + ESSE, 1 B200",
        "learned_scatter": learned,
        "value": round(ms, 2), "unit": "ms", "n_gpus": 1, "steps": K, "warmup": Wm, "higher_is_better": False,
        "genprj_s": {"photopeak": round(g_pp, 3), "lower_window": round(g_lw, 3)},
        "image_finite": bool(np.all(np.isfinite(rec))),
        "config": {"workload": "large256: 0.2 cm voxels, 28 cm circular orbit, 2e7 counts, collapse 2",
                   "drf_grid": [grids[0], grids[1]], "esse_grid": [grids[2], grids[3], grids[4]]},
        "data": "synthetic (seeded phantom, Poisson data)"}


def run_kernel_times(args):
    """Warm device time of every kernel of the full128 iteration: `--warmup`
    iterations, then `--steps` iterations (CUDA-graph replay, ESSE in every
    one) with CUPTI kernel records through torch.profiler, summed per kernel
    and divided by the iteration count.  A diagnostic table, not a bench
    line."""
    import collections
    import torch
    from torch.profiler import ProfilerActivity, profile
    import libirl_b200 as L
    from libirl_b200 import api
    torch.cuda.set_device(0)
    L.build()
    lib = L.load()
    tmp = tempfile.mkdtemp(prefix="irlkt_")
    case, files, meas = make_workload(lib, tmp, args.nviews, args.subsets)
    K, Wm = args.steps, args.warmup
    p, o, v = case.parms(), case.options(), case.views()
    p.NumIterations = p.iNumSrfIterations = K + Wm
    atn, rec, m = case.atn.copy(), np.zeros_like(case.act), meas.copy()
    if lib.IrlOsemBegin(C.byref(p), C.byref(o), v, _dup(files["drf"]), _dup(files["krnl"]), api.ITER_CB(), None,
                        api.fptr(atn), api.fptr(m), api.fptr(rec), None, None):
        raise RuntimeError(lib.pchIrlErrorString().decode())
    lib.IrlOsemIterate(Wm)
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        lib.IrlOsemIterate(K)
        torch.cuda.synchronize()
    lib.IrlOsemEnd(api.fptr(rec))
    tot, cnt = collections.defaultdict(float), collections.Counter()
    for e in prof.events():
        if e.device_type == torch.autograd.DeviceType.CUDA:
            name = e.name.split("(")[0].replace("void ", "").replace("irlcu::", "")
            tot[name] += getattr(e, "device_time_total", 0.0)
            cnt[name] += 1
    s = sum(tot.values())
    print("total us per iteration: %.1f" % (s / K))
    for k, t in sorted(tot.items(), key=lambda x: -x[1]):
        print("%-45s %5d launches %9.1f us/iter %5.1f%%" % (k[:45], cnt[k] // K, t / K, 100 * t / s))


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-surrogate", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the batch32 and large256 workloads reported beside the bench line")
    # reduced variants for profiling captures (the bench line uses the defaults)
    ap.add_argument("--nviews", type=int, default=120)
    ap.add_argument("--subsets", type=int, default=8)
    ap.add_argument("--cpu-views", type=int, default=2)
    ap.add_argument("--workload", default="full128", choices=["full128", "batch32", "large256"],
                    help="full128 is the bench line (which also reports the others unless --no-extra)")
    ap.add_argument("--kernel-times", action="store_true",
                    help="print the warm device time of every kernel of the full128 iteration instead")
    args = ap.parse_args()
    if args.kernel_times:
        run_kernel_times(args)
        return
    if args.workload == "batch32":
        print(json.dumps(run_batch32(args)))
        return
    if args.workload == "large256":
        print(json.dumps(run_large256(args)))
        return
    if args.warmup < 3 and args.impl == "b200":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()

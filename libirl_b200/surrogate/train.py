"""Train the learned scatter surrogate on the GPU.

    python -m libirl_b200.surrogate.train --phantoms 200 --val 16 --steps 6000 \
        --out libirl_b200/surrogate/sur128.bin --summary sur128.json

At the learned-scatter configuration's scale (3600 / 200 / 200 phantoms,
training pairs generated in streamed chunks):

    python -m libirl_b200.surrogate.train --phantoms 3600 --val 200 --test 200 \
        --chunk 400 --steps 24000 --init libirl_b200/surrogate/sur128.bin \
        --out libirl_b200/surrogate/sur128.bin --summary libirl_b200/surrogate/sur128_train.json

Training pairs come from the library's GPU ESSE path (irlcu_sur_pairs): for
every seeded full128 phantom (the 128^3 config-2 generator of
libirl_b200.workloads, a different seed per phantom) and each of its 120
views, the pooled rotated activity / attenuation / depth and the ESSE
scatter projection (projection with the scatter model minus without),
divided by the view's mean activity.  The network is trained with the
library's own forward, backward and Adam kernels (irlcu_sur_train_step);
torch only holds the device arrays and draws the batches.  Held-out
phantoms give the per-view NRMSE = ||y - t|| / ||t||.

Phantoms are generated on the host in a pool of processes started with
"spawn" while the GPU turns earlier ones into pairs.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import multiprocessing as mp
import os
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from libirl_b200 import api, workloads as W  # noqa: E402
from libirl_b200 import surrogate as SU  # noqa: E402

_libc = C.CDLL(None)
_libc.strdup.restype = C.c_void_p
_libc.strdup.argtypes = [C.c_char_p]


def _dup(s):
    return C.cast(_libc.strdup(s.encode()), C.c_char_p)


def _phantom(seed):
    return W.full128(seed=seed)


def _phantom256(seed):
    return W.large256(seed=seed)


# workload -> (phantom maker, views per phantom)
WORKLOADS = {"full128": (_phantom, 120), "large256": (_phantom256, 128)}


def generate(lib, seeds, workers=8, workload="full128"):
    """Network inputs X, normalised targets T and scales S of every view of
    every phantom, on the device (targets of 256^3 phantoms as 2 x 2 means
    of their 256 x 256 scatter projections)."""
    import torch
    maker, nv = WORKLOADS[workload]
    N = len(seeds) * nv
    X = torch.empty((N,) + SU.INPUT_SHAPE, dtype=torch.bfloat16, device="cuda")
    T = torch.empty((N, SU.OUTPUT_SIZE), dtype=torch.float32, device="cuda")
    S = torch.empty((N,), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    tmp = tempfile.mkdtemp(prefix="irlsur_")
    k = 0
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        for case in pool.imap(maker, seeds):
            assert case.nviews == nv and case.n in (128, 256)
            batch = case.nviews // case.subsets
            files = case.write_tables(tmp)
            p, o, v = case.parms(), case.options(), case.views()
            o.bReconIsInitEst = 1  # the phantom is the estimate
            rec, atn = case.act.copy(), case.atn.copy()
            prj = np.zeros((case.nviews, case.nz, case.n), np.float32)
            rc = lib.IrlOsemBegin(C.byref(p), C.byref(o), v, _dup(files["drf"]), _dup(files["krnl"]), api.ITER_CB(),
                                  None, api.fptr(atn), api.fptr(prj), api.fptr(rec), None, None)
            if rc:
                raise RuntimeError(lib.pchIrlErrorString().decode())
            try:
                for v0 in range(0, nv, batch):
                    nb = min(batch, nv - v0)
                    views = (C.c_int * nb)(*range(v0, v0 + nb))
                    rc = lib.irlcu_sur_pairs(nb, views, SU.MODEL_SRF, X[k].data_ptr(), T[k].data_ptr(),
                                             S[k].data_ptr())
                    if rc:
                        raise RuntimeError(lib.irlcu_error_string().decode())
                    k += nb
            finally:
                lib.IrlOsemEnd(None)
    return X, T, S


def nrmse(net, X, T, idx, batch):
    """Per-view ||y - t|| / ||t|| of the network on the views idx."""
    import torch
    out = []
    y = torch.empty((batch, SU.OUTPUT_SIZE), dtype=torch.float32, device="cuda")
    for i0 in range(0, len(idx), batch):
        sel = idx[i0:i0 + batch]
        xb = X.index_select(0, sel).contiguous()
        tb = T.index_select(0, sel)
        torch.cuda.synchronize()
        net.forward(len(sel), xb.data_ptr(), y.data_ptr())
        d = (y[:len(sel)] - tb).norm(dim=1) / tb.norm(dim=1).clamp_min(1e-30)
        out.append(d.cpu().numpy())
    return np.concatenate(out)


def _stats(e):
    return {"mean": float(e.mean()), "median": float(np.median(e)), "p90": float(np.percentile(e, 90)),
            "max": float(e.max()), "frac_le_1pct": float((e <= 0.01).mean()),
            "frac_le_2pct": float((e <= 0.02).mean())}


def train_streaming(args, lib):
    """Training at the scale of the learned-scatter configuration: 3600
    training, 200 validation and 200 test phantoms (seeds seed0 + i, split
    by seed), 120 views each.  The training phantoms' pairs are generated
    in chunks of --chunk phantoms and each chunk gets its share of the
    steps (the phantoms are independent draws, so this is streaming SGD
    over every training phantom without holding all 432,000 views);
    validation and test pairs stay resident."""
    import torch
    ntr, nval, nte = args.phantoms, args.val, args.test
    val_seeds = [args.seed0 + ntr + i for i in range(nval)]
    te_seeds = [args.seed0 + ntr + nval + i for i in range(nte)]
    t0 = time.time()
    Xv, Tv, _ = generate(lib, val_seeds, workers=args.workers, workload=args.workload)
    Xt, Tt, _ = generate(lib, te_seeds, workers=args.workers, workload=args.workload)
    t_gen = time.time() - t0
    g = torch.Generator(device="cuda")
    g.manual_seed(1234)
    net = SU.Network(lib, args.batch, seed=17)
    if args.init:
        net.set_weights(SU.load_weights(args.init))
    curve, val_curve = [], []
    step, t_train = 0, 0.0
    nchunks = (ntr + args.chunk - 1) // args.chunk
    for ci in range(nchunks):
        seeds = [args.seed0 + i for i in range(ci * args.chunk, min(ntr, (ci + 1) * args.chunk))]
        t = time.time()
        X, T, _ = generate(lib, seeds, workers=args.workers, workload=args.workload)
        t_gen += time.time() - t
        n = X.shape[0]
        stop = args.steps * (ci + 1) // nchunks
        t = time.time()
        while step < stop:
            warm = min(1.0, (step + 1) / 200.0)
            lr = args.lr * warm * (0.02 + 0.98 * 0.5 * (1.0 + math.cos(math.pi * step / args.steps)))
            idx = torch.randint(0, n, (args.batch,), device="cuda", generator=g)
            xb = X.index_select(0, idx).contiguous()
            tb = T.index_select(0, idx).contiguous()
            torch.cuda.synchronize()
            loss = net.train_step(args.batch, xb.data_ptr(), tb.data_ptr(), lr)
            if step % 200 == 0 or step == args.steps - 1:
                curve.append((step, loss))
                print(f"chunk {ci} step {step} loss {loss:.4e} lr {lr:.2e}", flush=True)
            step += 1
        t_train += time.time() - t
        del X, T
        torch.cuda.empty_cache()
        ev = nrmse(net, Xv, Tv, torch.arange(0, min(Xv.shape[0], 2400), device="cuda"), args.batch)
        val_curve.append((step, float(ev.mean())))
        print(f"chunk {ci}: validation NRMSE mean {ev.mean():.4f}", flush=True)
    ev = nrmse(net, Xv, Tv, torch.arange(0, Xv.shape[0], device="cuda"), args.batch)
    et = nrmse(net, Xt, Tt, torch.arange(0, Xt.shape[0], device="cuda"), args.batch)
    SU.save_weights(args.out, net.get_weights())
    summ = {
        "workload": args.workload, "phantoms": ntr, "val_phantoms": nval, "test_phantoms": nte,
        "views_per_phantom": WORKLOADS[args.workload][1], "training_views": ntr * WORKLOADS[args.workload][1],
        "chunk_phantoms": args.chunk, "steps": args.steps, "batch": args.batch,
        "lr": args.lr, "init": args.init and os.path.basename(args.init), "seed0": args.seed0,
        "generate_s": round(t_gen, 1), "train_s": round(t_train, 1),
        "ms_per_step": round(1000 * t_train / max(1, args.steps), 2),
        "loss_curve": [(s_, float(f"{l_:.4e}")) for s_, l_ in curve],
        "val_nrmse_curve": [(s_, round(v_, 5)) for s_, v_ in val_curve],
        "val_nrmse": _stats(ev), "test_nrmse": _stats(et),
        "weights": os.path.relpath(args.out, ROOT) if args.out.startswith(ROOT) else args.out,
    }
    print(json.dumps(summ))
    if args.summary:
        with open(args.summary, "w") as f:
            json.dump(summ, f, indent=1)
    net.close()


def time_steps(args, lib):
    """Wall time of training steps (forward, loss, backward, Adam; each
    step ends with a stream synchronisation) at --batch on seeded random
    inputs and targets, after 3 untimed steps; no pairs are generated and
    no weights are written."""
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(99)
    B = args.batch
    x = torch.rand((B,) + SU.INPUT_SHAPE, device="cuda", generator=g).to(torch.bfloat16)
    t = torch.rand((B, SU.OUTPUT_SIZE), device="cuda", generator=g)
    torch.cuda.synchronize()
    net = SU.Network(lib, B, seed=17)
    try:
        for _ in range(3):
            net.train_step(B, x.data_ptr(), t.data_ptr(), 1e-4)
        t0 = time.perf_counter()
        for _ in range(args.time_steps):
            loss = net.train_step(B, x.data_ptr(), t.data_ptr(), 1e-4)
        ms = 1000.0 * (time.perf_counter() - t0) / args.time_steps
    finally:
        net.close()
    print(json.dumps({"batch": B, "steps": args.time_steps, "ms_per_step": round(ms, 3), "loss": loss}))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--phantoms", type=int, default=200, help="training phantoms")
    ap.add_argument("--val", type=int, default=16, help="held-out phantoms")
    ap.add_argument("--test", type=int, default=0, help="test phantoms (with --chunk)")
    ap.add_argument("--workload", default="full128", choices=sorted(WORKLOADS),
                    help="phantom generator: full128 (128^3, 120 views) or large256 (256^3, 128 views)")
    ap.add_argument("--chunk", type=int, default=0,
                    help="generate the training pairs in chunks of this many phantoms (streaming)")
    ap.add_argument("--seed0", type=int, default=40000)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--workers", type=int, default=8)
    ap.add_argument("--init", default=None, help="start from this weights file")
    ap.add_argument("--out", default=SU.DEFAULT_WEIGHTS)
    ap.add_argument("--summary", default=None)
    ap.add_argument("--time-steps", type=int, default=0,
                    help="only time this many training steps on seeded random data (no pairs, no weights written)")
    args = ap.parse_args(argv)

    import torch
    import libirl_b200 as L
    lib = L.load()
    if args.time_steps > 0:
        return time_steps(args, lib)
    if args.chunk > 0:
        return train_streaming(args, lib)
    t0 = time.time()
    seeds = [args.seed0 + i for i in range(args.phantoms + args.val)]
    X, T, _ = generate(lib, seeds, workers=args.workers)
    t_gen = time.time() - t0
    ntrain = args.phantoms * 120
    g = torch.Generator(device="cuda")
    g.manual_seed(1234)
    net = SU.Network(lib, args.batch, seed=17)
    if args.init:
        net.set_weights(SU.load_weights(args.init))
    curve = []
    t1 = time.time()
    for step in range(args.steps):
        # linear warm-up over 200 steps, then cosine decay to 2% of lr
        warm = min(1.0, (step + 1) / 200.0)
        lr = args.lr * warm * (0.02 + 0.98 * 0.5 * (1.0 + math.cos(math.pi * step / args.steps)))
        idx = torch.randint(0, ntrain, (args.batch,), device="cuda", generator=g)
        xb = X.index_select(0, idx).contiguous()
        tb = T.index_select(0, idx).contiguous()
        torch.cuda.synchronize()
        loss = net.train_step(args.batch, xb.data_ptr(), tb.data_ptr(), lr)
        if step % 100 == 0 or step == args.steps - 1:
            curve.append((step, loss))
            print(f"step {step} loss {loss:.4e} lr {lr:.2e} ({time.time() - t1:.0f} s)", flush=True)
    t_train = time.time() - t1
    val_idx = torch.arange(ntrain, X.shape[0], device="cuda")
    e = nrmse(net, X, T, val_idx, args.batch)
    tr_idx = torch.arange(0, min(ntrain, 16 * 120), device="cuda")
    etr = nrmse(net, X, T, tr_idx, args.batch)
    SU.save_weights(args.out, net.get_weights())
    summ = {
        "phantoms": args.phantoms, "val_phantoms": args.val, "views": int(X.shape[0]), "steps": args.steps,
        "batch": args.batch, "lr": args.lr, "generate_s": round(t_gen, 1), "train_s": round(t_train, 1),
        "ms_per_step": round(1000 * t_train / max(1, args.steps), 2),
        "loss_curve": [(s, float(f"{l_:.4e}")) for s, l_ in curve],
        "val_nrmse": {"mean": float(e.mean()), "median": float(np.median(e)), "p90": float(np.percentile(e, 90)),
                      "max": float(e.max()), "frac_le_1pct": float((e <= 0.01).mean()),
                      "frac_le_2pct": float((e <= 0.02).mean())},
        "train_nrmse_mean": float(etr.mean()),
        "weights": os.path.relpath(args.out, ROOT) if args.out.startswith(ROOT) else args.out,
    }
    print(json.dumps(summ))
    if args.summary:
        with open(args.summary, "w") as f:
            json.dump(summ, f, indent=1)
    net.close()


if __name__ == "__main__":
    main()

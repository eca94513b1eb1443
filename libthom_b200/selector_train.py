"""Trains and evaluates the learned Ozaki slice-count selector on the GPU.

Data: seeded matrices with shapes from the library's three DGEMM families, capped at 2048 per
dimension — square (M = N = K), tall-skinny (large M, small N) and long-K — with exponent spread
phi ~ U{0..64} and, for the last two families, rows of A / columns of B scaled by 2^s with
s ~ U{-smax..smax}. Each matrix is run through the Ozaki kernels; its componentwise error max |C_s - C_64| / (|alpha||A||B|) against the native FP64 result C_64 is measured for
s = 3..12; for each tolerance in {1e-12, 1e-14, 1e-15} the label is the smallest s meeting it,
as class min(s, 10) - 3 (class 7 = "10 or more slices, or none": the library falls back to the
analytic count there). Features come from lt_ozaki_features; training runs lt_mlp_train_step
(hand-written forward, backward and Adam kernels). The held-out set reports the tolerance-miss rate
of the analytic count, of the learned choice alone and of the library's final choice (learned, or
analytic on fallback), the mean slice counts, and end-to-end throughput (selection included)
against fixed-slice Ozaki and native FP64.

    python -m libthom_b200.selector_train [--train 20000] [--test 2000] [--out PATH]
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import time
from pathlib import Path

import numpy as np

import libthom_b200 as lt

TOLS = (1e-12, 1e-14, 1e-15)
SLICES = list(range(3, 13))   # slice counts whose error is measured
CLASS_TOP = 10                 # classes 3..10, the last one meaning ">= 10 or unreachable"
WEIGHTS = Path(__file__).resolve().parent / "selector_weights.bin"


def draw_shape(rng):
    fam = int(rng.integers(0, 3))
    lu = lambda lo, hi: int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
    if fam == 0:
        n = lu(64, 2048)
        M = N = K = n
        smax = 0
    elif fam == 1:
        M, N, K = lu(256, 2048), lu(16, 128), lu(256, 2048)
        smax = int(rng.integers(0, 65))
    else:
        M = N = lu(64, 512)
        K = lu(1024, 2048)
        smax = int(rng.integers(0, 65))
    return fam, M, N, K, int(rng.integers(0, 65)), smax, int(rng.integers(1, 2**62))


class Generator:
    """Device buffers reused across problems (sized for the largest shape)."""

    def __init__(self, torch, cap=2048):
        self.torch = torch
        n2 = cap * cap
        f = dict(dtype=torch.float64, device="cuda")
        self.A = torch.empty(n2, **f)
        self.B = torch.empty(n2, **f)
        self.C64 = torch.empty(n2, **f)
        self.C = torch.empty(n2, **f)
        self.den = torch.empty(n2, **f)
        self.feat = torch.empty(lt.LT_SEL_FEATURES, dtype=torch.float32, device="cuda")

    def problem(self, M, N, K, phi, smax, seed):
        L = lt.lib()
        lt.check(L.lt_fill(self.A.data_ptr(), M * K, seed, 1, phi, None))
        lt.check(L.lt_fill(self.B.data_ptr(), K * N, seed, 2, phi, None))
        if smax > 0:
            lt.check(L.lt_scale_rows(self.A.data_ptr(), M, K, seed, 4, smax, None))
            lt.check(L.lt_scale_cols(self.B.data_ptr(), K, N, seed, 5, smax, None))

    def errors(self, M, N, K):
        """Componentwise error of the Ozaki result for every s in SLICES against the FP64 result."""
        L = lt.lib()
        A, B = self.A.data_ptr(), self.B.data_ptr()
        lt.check(L.lt_dgemm_fp64(A, B, self.C64.data_ptr(), M, N, K, 1.0, 0.0, None))
        lt.check(L.lt_abs_denominator(A, B, None, self.den.data_ptr(), M, N, K, 1.0, 0.0, None))
        out = []
        for s in SLICES:
            lt.check(L.lt_dgemm_ozaki(A, B, self.C.data_ptr(), M, N, K, 1.0, 0.0, s, None))
            e, _ = lt.componentwise_error(self.C, self.C64, self.den, M * N)
            out.append(e)
        return out

    def features(self, M, N, K):
        lt.check(lt.lib().lt_ozaki_features(self.A.data_ptr(), self.B.data_ptr(), M, N, K, 1.0,
                                            self.feat.data_ptr(), None))
        return self.feat.cpu().numpy().copy()

    def analytic(self, M, N, K, tol):
        """(analytic slice count, gap_bits) — independent of any installed weights."""
        gap = ctypes.c_int()
        lt.check(lt.lib().lt_ozaki_gap_bits(self.A.data_ptr(), self.B.data_ptr(), M, N, K, ctypes.byref(gap), None))
        return int(lt.lib().lt_ozaki_analytic_slices(tol, gap.value)), gap.value


def label_of(errs, tol):
    for s, e in zip(SLICES, errs):
        if e <= tol:
            return min(s, CLASS_TOP) - 3
    return CLASS_TOP - 3


def build_dataset(torch, gen, n, seed, log_every=0):
    rng = np.random.default_rng(seed)
    rows = []
    t0 = time.time()
    for i in range(n):
        fam, M, N, K, phi, smax, pseed = draw_shape(rng)
        gen.problem(M, N, K, phi, smax, pseed)
        errs = gen.errors(M, N, K)
        f = gen.features(M, N, K)
        rows.append(dict(fam=fam, M=M, N=N, K=K, phi=phi, smax=smax, seed=pseed, errs=errs, feat=f))
        if log_every and (i + 1) % log_every == 0:
            print(f"  {i + 1}/{n} problems ({time.time() - t0:.0f} s)", flush=True)
    return rows


def expand(rows):
    X, Y = [], []
    for r in rows:
        for tol in TOLS:
            f = r["feat"].copy()
            f[33] = np.float32(-math.log10(tol) / 16.0)
            X.append(f)
            Y.append(label_of(r["errs"], tol))
    return np.stack(X).astype(np.float32), np.array(Y, dtype=np.int32)


def init_params(seed):
    rng = np.random.default_rng(seed)
    F, H, C = lt.LT_SEL_FEATURES, lt.LT_SEL_HIDDEN, lt.LT_SEL_CLASSES
    parts = [rng.standard_normal(H * F) * math.sqrt(2.0 / F), np.zeros(H),
             rng.standard_normal(H * H) * math.sqrt(2.0 / H), np.zeros(H),
             rng.standard_normal(C * H) * math.sqrt(1.0 / H), np.zeros(C)]
    return np.concatenate(parts).astype(np.float32)


def train(torch, X, Y, epochs=40, batch=256, lr=2e-3, seed=0):
    L = lt.lib()
    dev = dict(device="cuda")
    params = torch.from_numpy(init_params(seed)).to(**dev)
    m = torch.zeros_like(params)
    v = torch.zeros_like(params)
    g = torch.zeros_like(params)
    loss = torch.zeros(1, dtype=torch.float32, **dev)
    Xd = torch.from_numpy(X).to(**dev)
    Yd = torch.from_numpy(Y).to(**dev)
    rng = np.random.default_rng(seed)
    step = 0
    hist = []
    for ep in range(epochs):
        perm = torch.from_numpy(rng.permutation(len(Y))).to(**dev)
        tot = 0.0
        nb = 0
        for b0 in range(0, len(Y) - batch + 1, batch):
            idx = perm[b0:b0 + batch]
            xb = Xd[idx].contiguous()
            yb = Yd[idx].contiguous()
            step += 1
            lt.check(L.lt_mlp_train_step(params.data_ptr(), m.data_ptr(), v.data_ptr(), g.data_ptr(), xb.data_ptr(),
                                         yb.data_ptr(), batch, lr, step, loss.data_ptr(), None))
            tot += float(loss.item()) if (nb % 20 == 0) else 0.0
            nb += 1
        hist.append(tot / max(1, (nb + 19) // 20))
    return params.cpu().numpy(), hist


def predict(torch, params, X):
    L = lt.lib()
    p = torch.from_numpy(params).cuda()
    x = torch.from_numpy(X).cuda()
    out = torch.empty(len(X), lt.LT_SEL_CLASSES, dtype=torch.float32, device="cuda")
    lt.check(L.lt_mlp_forward(p.data_ptr(), x.data_ptr(), len(X), out.data_ptr(), None))
    return out.cpu().numpy()


def learned_only(probs):
    """The network's own answer: smallest s whose cumulative probability reaches 0.9."""
    return 3 + int(np.argmax(np.cumsum(probs) >= 0.9))


QUANTILE = 0.999  # the library's kQuantile (selector.cu)


def decide(probs, s_analytic):
    """The library's rule (selector.cu, decide): the learned count if the top class has >= 0.5 and
    neither it nor the 0.999-quantile is the last class; the analytic count otherwise.
    Returns (slices, learned?)."""
    top = int(np.argmax(probs))
    if probs[top] < 0.5 or top == len(probs) - 1:
        return s_analytic, False
    c = int(np.argmax(np.cumsum(np.asarray(probs, dtype=np.float32), dtype=np.float32) >= np.float32(QUANTILE)))
    if c == len(probs) - 1:
        return s_analytic, False
    return 3 + c, True


def evaluate(torch, gen, params, rows):
    X, Y = expand(rows)
    P = predict(torch, params, X)
    n = len(Y)
    miss = dict(analytic=0, learned_only=0, final=0)
    slices = dict(analytic=[], learned_only=[], final=[])
    used_learned = 0
    per_tol = {}
    chosen = []
    k = 0

    def err(r, s):
        return r["errs"][s - 3] if 3 <= s <= 12 else float("inf")

    for r in rows:
        gen.problem(r["M"], r["N"], r["K"], r["phi"], r["smax"], r["seed"])
        for tol in TOLS:
            s_a, gap = gen.analytic(r["M"], r["N"], r["K"], tol)
            s_l = learned_only(P[k])
            s_f, learned = decide(P[k], s_a)
            for name, sv in (("analytic", s_a), ("learned_only", s_l), ("final", s_f)):
                miss[name] += err(r, sv) > tol
                slices[name].append(sv)
            used_learned += learned
            d = per_tol.setdefault(str(tol), dict(n=0, miss_analytic=0, miss_final=0, analytic=0.0, final=0.0,
                                                 reachable=0))
            d["n"] += 1
            d["miss_analytic"] += err(r, s_a) > tol
            d["miss_final"] += err(r, s_f) > tol
            d["analytic"] += s_a
            d["final"] += s_f
            d["reachable"] += min(r["errs"]) <= tol
            chosen.append((r, tol, s_f, s_a))
            k += 1
    out = dict(samples=n, accuracy_top1=float(np.mean(np.argmax(P, axis=1) == Y)),
               learned_used_fraction=used_learned / n,
               miss_rate={kk: v / n for kk, v in miss.items()},
               mean_slices={kk: float(np.mean(v)) for kk, v in slices.items()},
               mean_slices_saved_vs_analytic=float(np.mean(np.array(slices["analytic"]) - np.array(slices["final"]))),
               per_tolerance={t: {kk: (vv / d["n"] if kk != "n" else vv) for kk, vv in d.items()}
                              for t, d in per_tol.items()})
    return out, chosen


def throughput(torch, gen, chosen, limit=150):
    """End-to-end time over held-out problems, selection included: the library's selector
    (lt_ozaki_select_slices, then Ozaki), the same selection inside a plan's CUDA graph (plan built
    beforehand, as plans are for repeated calls; one graph launch per call), the plan that may also
    pick native FP64 (auto_plan) and its host-side counterpart lt_dgemm_auto, the analytic count (gap
    pass, then Ozaki), fixed s = 8, 10 and 12 (12: the count that meets 1e-12 on every reachable
    problem of this distribution), and native FP64."""
    L = lt.lib()
    A, B, C = gen.A.data_ptr(), gen.B.data_ptr(), gen.C.data_ptr()
    tot = dict(selector=0.0, selector_plan=0.0, auto_plan=0.0, auto=0.0, analytic=0.0, fixed8=0.0, fixed10=0.0,
               fixed12=0.0, fp64=0.0)
    flops = 0.0
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    sel = ctypes.c_int()
    gap = ctypes.c_int()

    def via_selector(M, N, K, tol):
        lt.check(L.lt_ozaki_select_slices(A, B, M, N, K, tol, ctypes.byref(sel), None))
        lt.check(L.lt_dgemm_ozaki(A, B, C, M, N, K, 1.0, 0.0, sel.value, None))

    def via_analytic(M, N, K, tol):
        lt.check(L.lt_ozaki_gap_bits(A, B, M, N, K, ctypes.byref(gap), None))
        s = int(L.lt_ozaki_analytic_slices(tol, gap.value))
        lt.check(L.lt_dgemm_ozaki(A, B, C, M, N, K, 1.0, 0.0, s, None))

    for r, tol, s_final, s_a in chosen[:limit]:
        M, N, K = r["M"], r["N"], r["K"]
        gen.problem(M, N, K, r["phi"], r["smax"], r["seed"])
        flops += 2.0 * M * N * K
        plan = lt.OzakiAutoPlan(gen.A, gen.B, gen.C, M, N, K, 1.0, 0.0, tol)
        aplan = lt.OzakiAutoPlan(gen.A, gen.B, gen.C, M, N, K, 1.0, 0.0, tol, forms=lt.LT_AUTO_PLAN_ANY_FORM)
        runs = {
            "selector": lambda: via_selector(M, N, K, tol),
            "selector_plan": lambda: plan.run(),
            "auto_plan": lambda: aplan.run(),
            "auto": lambda: lt.check(L.lt_dgemm_auto(A, B, C, M, N, K, 1.0, 0.0, None, None, None)),
            "analytic": lambda: via_analytic(M, N, K, tol),
            "fixed8": lambda: lt.check(L.lt_dgemm_ozaki(A, B, C, M, N, K, 1.0, 0.0, 8, None)),
            "fixed10": lambda: lt.check(L.lt_dgemm_ozaki(A, B, C, M, N, K, 1.0, 0.0, 10, None)),
            "fixed12": lambda: lt.check(L.lt_dgemm_ozaki(A, B, C, M, N, K, 1.0, 0.0, 12, None)),
            "fp64": lambda: lt.check(L.lt_dgemm_fp64(A, B, C, M, N, K, 1.0, 0.0, None)),
        }
        for name, fn in runs.items():
            fn()
            torch.cuda.synchronize()
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            tot[name] += e0.elapsed_time(e1)
        plan.close()
        aplan.close()
    return {k: flops / (v * 1e-3) / 1e12 for k, v in tot.items()}, tot


def main():
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=20000)
    ap.add_argument("--test", type=int, default=2000)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--out", default=str(WEIGHTS))
    ap.add_argument("--report", default="")
    ap.add_argument("--eval-only", action="store_true",
                    help="evaluate the weights in --out on the held-out set without training")
    args = ap.parse_args()
    torch.cuda.set_device(0)
    gen = Generator(torch)
    t0 = time.time()
    if args.eval_only:
        train_rows = []
        test_rows = build_dataset(torch, gen, args.test, seed=98765)
        t_data = time.time() - t0
        params = np.fromfile(args.out, dtype=np.float32)
        assert params.size == lt.LT_SEL_PARAMS, params.size
        X, Y, hist, t_train = np.zeros((0, lt.LT_SEL_FEATURES)), np.zeros(0, dtype=np.int64), [], 0.0
    else:
        train_rows = build_dataset(torch, gen, args.train, seed=1234, log_every=2000)
        test_rows = build_dataset(torch, gen, args.test, seed=98765)
        t_data = time.time() - t0
        X, Y = expand(train_rows)
        t1 = time.time()
        params, hist = train(torch, X, Y, epochs=args.epochs)
        t_train = time.time() - t1
        params.astype(np.float32).tofile(args.out)
    lt.check(lt.lib().lt_selector_set_params(params.ctypes.data))
    ev, chosen = evaluate(torch, gen, params, test_rows)
    tput, ms = throughput(torch, gen, chosen)
    report = dict(train_matrices=0 if args.eval_only else args.train, test_matrices=args.test, train_samples=len(Y),
                  label_histogram=np.bincount(Y, minlength=8).tolist(), data_seconds=t_data, train_seconds=t_train,
                  loss_by_epoch=hist, evaluation=ev, throughput_tflops=tput, throughput_ms=ms, weights=args.out)
    text = json.dumps(report, indent=1)
    print(text)
    if args.report:
        Path(args.report).write_text(text)


if __name__ == "__main__":
    main()

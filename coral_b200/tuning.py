"""Autotuning database and the learned configuration selector.

The split-BF16 SGEMM has ten configurations per shape: N tile width
{256, 128} x split-K {1, 2, 4, 8, 16}.  This module

* draws seeded shapes (dims log-uniform in [32, 16384], plus the tall-skinny
  65536 x 64 x 4096 and split-K-heavy 256 x 256 x 65536 shapes),
* times every configuration of every shape on the GPU with the library's
  exhaustive autotuner (``coral_autotune_sgemm``) into a timing database,
* trains the selector network -- 13 features -> 128 -> 128 -> 1 (ReLU),
  predicting log(ms) -- with the library's own CUDA forward/backward/Adam
  kernels (``coral_mlp_*``),
* and measures, on held-out shapes, the runtime regret
  t(selected) / t(exhaustive best) - 1 of the selector and of the default
  configuration rule it replaces.

CLI (runs on a B200):
    python -m coral_b200.tuning collect --count 20000 --seed 1 --out train.npz
    python -m coral_b200.tuning collect --count 2000 --seed 2 --out heldout.npz
    python -m coral_b200.tuning train --db train.npz --out selector.npz
    python -m coral_b200.tuning evaluate --db heldout.npz --weights selector.npz
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import time

import numpy as np

from . import _lib
from .blas import handle

CANDIDATES = [(bn, sp) for bn in (256, 128) for sp in (1, 2, 4, 8, 16)]
N_FEATURES = 13
HIDDEN = 128
DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


# ------------------------------------------------------------------- shapes --
def generate_shapes(count: int, seed: int, lo: int = 32, hi: int = 16384) -> np.ndarray:
    """[count, 5] int64: m, n, k, op_a, op_b.  The first two rows are the
    tall-skinny and split-K-heavy shapes when count >= 2."""
    rng = np.random.default_rng(seed)
    dims = np.exp(rng.uniform(np.log(lo), np.log(hi), (count, 3))).astype(np.int64)
    ops = rng.integers(0, 2, (count, 2))
    shapes = np.concatenate([dims, ops], axis=1)
    if count >= 2:
        shapes[0] = (65536, 64, 4096, 0, 0)
        shapes[1] = (256, 256, 65536, 0, 0)
    return shapes


def features(shape, bn: int, sp: int, products: int = 3) -> np.ndarray:
    """The selector's 13 features for (shape, configuration), computed by the library."""
    m, n, k, op_a, op_b = (int(v) for v in shape)
    out = (C.c_float * N_FEATURES)()
    st = _lib.load().coral_selector_features(products, op_a, op_b, m, n, k, bn, sp, out)
    if st != 0:
        raise RuntimeError(f"coral_selector_features: {st}")
    return np.frombuffer(out, dtype=np.float32).copy()


def feature_matrix(shapes: np.ndarray) -> np.ndarray:
    """[len(shapes) * 10, 13] in shape-major, candidate-minor order."""
    return np.stack([features(s, bn, sp) for s in shapes for (bn, sp) in CANDIDATES])


def default_choice(shape, sm_count: int = 148) -> int:
    """Index in CANDIDATES of the library's default rule (no selector)."""
    m, n, k = (int(v) for v in shape[:3])
    tiles = -(-m // 128) * -(-n // 256)
    sp = 1
    if tiles * 2 <= sm_count and -(-k // 64) >= 16:
        sp = min(16, max(1, sm_count // tiles))
    sp = min(sp, max(1, -(-k // 64)))
    best = max([s for s in (1, 2, 4, 8, 16) if s <= sp])
    return CANDIDATES.index((256, best))


# ------------------------------------------------------------ autotune DB --
def collect(shapes: np.ndarray, reps_small: int = 3, log_every: int = 500) -> np.ndarray:
    """Exhaustively times every candidate of every shape: [len(shapes), 10] ms."""
    import torch
    lib = _lib.load()
    h = handle()
    h.bind_current_stream()
    need_a = int(max(s[0] * s[2] for s in shapes))
    need_b = int(max(s[2] * s[1] for s in shapes))
    need_c = int(max(s[0] * s[1] for s in shapes))
    A = torch.empty(need_a, dtype=torch.float32, device="cuda").uniform_(-1, 1)
    B = torch.empty(need_b, dtype=torch.float32, device="cuda").uniform_(-1, 1)
    Cm = torch.empty(need_c, dtype=torch.float32, device="cuda")
    times = np.zeros((len(shapes), len(CANDIDATES)), np.float32)
    ms = (C.c_float * len(CANDIDATES))()
    best = C.c_int()
    t0 = time.time()
    for i, (m, n, k, op_a, op_b) in enumerate(shapes):
        m, n, k, op_a, op_b = int(m), int(n), int(k), int(op_a), int(op_b)
        lda = m if op_a == 0 else k
        ldb = k if op_b == 0 else n
        reps = reps_small if 2.0 * m * n * k < 2e10 else 1
        st = lib.coral_autotune_sgemm(h.h, 3, op_a, op_b, m, n, k, C.c_void_p(A.data_ptr()), lda,
                                      C.c_void_p(B.data_ptr()), ldb, C.c_void_p(Cm.data_ptr()), m,
                                      reps, ms, C.byref(best))
        if st != 0:
            raise RuntimeError(f"coral_autotune_sgemm failed on {m}x{n}x{k}: {st}")
        times[i] = np.frombuffer(ms, dtype=np.float32)
        if log_every and (i + 1) % log_every == 0:
            print(f"  {i + 1}/{len(shapes)} shapes, {time.time() - t0:.0f} s", flush=True)
    return times


# --------------------------------------------------------------------- MLP --
class Mlp:
    """The library's MLP (coral_mlp_*): parameters on the device."""

    def __init__(self, in_dim=N_FEATURES, hidden=HIDDEN, out_dim=1, seed=0):
        self.lib = _lib.load()
        self.h = handle()
        p = C.c_void_p()
        st = self.lib.coral_mlp_create(self.h.h, in_dim, hidden, out_dim, seed, C.byref(p))
        if st != 0:
            raise RuntimeError(f"coral_mlp_create: {st}")
        self.p = p
        self.shape = (in_dim, hidden, out_dim)

    def close(self):
        if self.p:
            self.lib.coral_mlp_destroy(self.p)
            self.p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nparams(self) -> int:
        return int(self.lib.coral_mlp_param_count(self.p))

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.nparams, np.float32)
        st = self.lib.coral_mlp_get_params(self.p, out.ctypes.data_as(C.POINTER(C.c_float)), out.size)
        if st != 0:
            raise RuntimeError(f"coral_mlp_get_params: {st}")
        return out

    def set_params(self, params: np.ndarray) -> None:
        params = np.ascontiguousarray(params, np.float32)
        st = self.lib.coral_mlp_set_params(self.p, params.ctypes.data_as(C.POINTER(C.c_float)), params.size)
        if st != 0:
            raise RuntimeError(f"coral_mlp_set_params: {st}")

    def forward(self, x):
        """x: CUDA float32 tensor [batch, in] -> [batch, out]."""
        import torch
        self.h.bind_current_stream()
        y = torch.empty((x.shape[0], self.shape[2]), dtype=torch.float32, device=x.device)
        st = self.lib.coral_mlp_forward(self.p, C.c_void_p(x.data_ptr()), x.shape[0], C.c_void_p(y.data_ptr()))
        if st != 0:
            raise RuntimeError(f"coral_mlp_forward: {st}")
        return y

    def gradients(self, x, t):
        import torch
        self.h.bind_current_stream()
        g = torch.empty(self.nparams, dtype=torch.float32, device=x.device)
        loss = C.c_float()
        st = self.lib.coral_mlp_gradients(self.p, C.c_void_p(x.data_ptr()), C.c_void_p(t.data_ptr()),
                                          x.shape[0], C.c_void_p(g.data_ptr()), C.byref(loss))
        if st != 0:
            raise RuntimeError(f"coral_mlp_gradients: {st}")
        return g, loss.value

    def train_step(self, x, t, lr) -> float:
        self.h.bind_current_stream()
        loss = C.c_float()
        st = self.lib.coral_mlp_train_step(self.p, C.c_void_p(x.data_ptr()), C.c_void_p(t.data_ptr()),
                                           x.shape[0], lr, C.byref(loss))
        if st != 0:
            raise RuntimeError(f"coral_mlp_train_step: {st}")
        return loss.value

    def attach(self, h=None) -> None:
        """Make this network the configuration selector of a handle."""
        h = h or self.h
        st = self.lib.coral_set_selector(h.h, self.p)
        if st != 0:
            raise RuntimeError(f"coral_set_selector: {st}")

    def save(self, path: str, meta: dict | None = None) -> None:
        np.savez_compressed(path, params=self.get_params(), shape=np.array(self.shape),
                            meta=json.dumps(meta or {}))

    @classmethod
    def load(cls, path: str) -> "Mlp":
        d = np.load(path)
        net = cls(*[int(v) for v in d["shape"]])
        net.set_params(d["params"])
        return net


def train(db_shapes: np.ndarray, db_times: np.ndarray, epochs: int = 300, batch: int = 4096,
          lr: float = 2e-3, seed: int = 0, log_every: int = 50) -> tuple[Mlp, list]:
    """Fits log(ms) of every (shape, configuration) pair on the GPU."""
    import torch
    X = torch.from_numpy(feature_matrix(db_shapes)).cuda()
    y = torch.from_numpy(np.log(np.maximum(db_times.reshape(-1, 1), 1e-4)).astype(np.float32)).cuda()
    net = Mlp(seed=seed)
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    history = []
    n = X.shape[0]
    for ep in range(epochs):
        perm = torch.randperm(n, device="cuda", generator=g)
        tot = 0.0
        steps = 0
        lr_ep = lr * (0.5 * (1 + np.cos(np.pi * ep / epochs)) * 0.95 + 0.05)
        for s in range(0, n, batch):
            idx = perm[s:s + batch]
            xb = X[idx].contiguous()
            yb = y[idx].contiguous()
            tot += net.train_step(xb, yb, float(lr_ep))
            steps += 1
        history.append(tot / max(steps, 1))
        if log_every and (ep + 1) % log_every == 0:
            print(f"  epoch {ep + 1}: mse(log ms) = {history[-1]:.4f}", flush=True)
    return net, history


def predict_choice(net: Mlp, shapes: np.ndarray) -> np.ndarray:
    import torch
    X = torch.from_numpy(feature_matrix(shapes)).cuda()
    pred = net.forward(X).cpu().numpy().reshape(len(shapes), len(CANDIDATES))
    return pred.argmin(axis=1)


def regret(times: np.ndarray, choice: np.ndarray) -> np.ndarray:
    best = times.min(axis=1)
    return times[np.arange(len(times)), choice] / best - 1.0


def summarize(r: np.ndarray) -> dict:
    return {"mean": float(r.mean()), "p50": float(np.median(r)), "p95": float(np.quantile(r, 0.95)),
            "max": float(r.max()), "frac_optimal": float((r <= 1e-9).mean())}


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m coral_b200.tuning")
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("collect")
    c.add_argument("--count", type=int, default=20000)
    c.add_argument("--seed", type=int, default=1)
    c.add_argument("--out", required=True)
    t = sub.add_parser("train")
    t.add_argument("--db", required=True)
    t.add_argument("--out", required=True)
    t.add_argument("--epochs", type=int, default=300)
    e = sub.add_parser("evaluate")
    e.add_argument("--db", required=True)
    e.add_argument("--weights", required=True)
    args = ap.parse_args(argv)
    if args.cmd == "collect":
        shapes = generate_shapes(args.count, args.seed)
        t0 = time.time()
        times = collect(shapes)
        np.savez_compressed(args.out, shapes=shapes, times=times, candidates=np.array(CANDIDATES),
                            seed=args.seed)
        print(json.dumps({"collected": len(shapes), "seconds": time.time() - t0, "out": args.out}))
    elif args.cmd == "train":
        d = np.load(args.db)
        t0 = time.time()
        net, hist = train(d["shapes"], d["times"], epochs=args.epochs)
        net.save(args.out, {"db": os.path.basename(args.db), "epochs": args.epochs,
                            "final_mse": hist[-1], "seconds": time.time() - t0})
        choice = predict_choice(net, d["shapes"])
        print(json.dumps({"train_mse": hist[-1], "train_regret": summarize(regret(d["times"], choice)),
                          "seconds": time.time() - t0}))
    elif args.cmd == "evaluate":
        d = np.load(args.db)
        net = Mlp.load(args.weights)
        choice = predict_choice(net, d["shapes"])
        dflt = np.array([default_choice(s) for s in d["shapes"]])
        fixed = np.full(len(d["shapes"]), CANDIDATES.index((256, 1)))
        print(json.dumps({"shapes": int(len(d["shapes"])),
                          "selector": summarize(regret(d["times"], choice)),
                          "default_rule": summarize(regret(d["times"], dflt)),
                          "fixed_256x1": summarize(regret(d["times"], fixed))}))


if __name__ == "__main__":
    main()

"""Autotuning database and the learned configuration selector.

The split-BF16 SGEMM has fifteen configurations per shape: tile
{256 x 256 on a CTA pair (tcgen05 cta_group::2, cluster of 2), 128 x 256,
128 x 128} x split-K {1, 2, 4, 8, 16}; the 3-piece (x6) mode has no 128 x 256
tile.  This module

* draws seeded shapes (dims log-uniform in [32, 16384], plus the tall-skinny
  65536 x 64 x 4096 and split-K-heavy 256 x 256 x 65536 shapes; a quarter of
  them in the 3-piece mode, so the data-type feature varies),
* times every configuration of every shape on the GPU with the library's
  exhaustive autotuner (``coral_autotune_sgemm_tiles``) into a timing database
  (configurations a mode does not have are stored as +inf),
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
    python -m coral_b200.tuning evaluate-live --db heldout.npz --weights selector.npz --count 300

The tensor-core grouped GEMM's tile-width policy has its own network and
pipeline (uniform batches of varied data type and instance count; live
regret on held-out uneven batches against all 36 policies):
    python -m coral_b200.tuning grouped-collect --count 6000 --out grouped_train.npz
    python -m coral_b200.tuning grouped-train --db grouped_train.npz --out grouped_selector.npz
    python -m coral_b200.tuning grouped-evaluate --weights grouped_selector.npz
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

TILES = ((256, 256), (128, 256), (128, 128))
CANDIDATES = [(tm, tn, sp) for (tm, tn) in TILES for sp in (1, 2, 4, 8, 16)]
X6_FRACTION = 0.25
N_FEATURES = 13
HIDDEN = 128
DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


# ------------------------------------------------------------------- shapes --
def generate_shapes(count: int, seed: int, lo: int = 32, hi: int = 16384,
                    x6_fraction: float = X6_FRACTION) -> np.ndarray:
    """[count, 6] int64: m, n, k, op_a, op_b, products (3 or 6).  The first two
    rows are the tall-skinny and split-K-heavy shapes when count >= 2."""
    rng = np.random.default_rng(seed)
    dims = np.exp(rng.uniform(np.log(lo), np.log(hi), (count, 3))).astype(np.int64)
    ops = rng.integers(0, 2, (count, 2))
    products = np.where(rng.uniform(size=(count, 1)) < x6_fraction, 6, 3)
    shapes = np.concatenate([dims, ops, products], axis=1)
    if count >= 2:
        shapes[0] = (65536, 64, 4096, 0, 0, 3)
        shapes[1] = (256, 256, 65536, 0, 0, 3)
    return shapes


def shape_products(shape) -> int:
    return int(shape[5]) if len(shape) > 5 else 3


def valid(shape, cand) -> bool:
    """Whether the shape's mode has this configuration (x6: no 128 x 256 tile)."""
    return not (shape_products(shape) == 6 and cand[:2] == (128, 256))


def features(shape, tm: int, tn: int, sp: int) -> np.ndarray:
    """The selector's 13 features for (shape, configuration), computed by the library."""
    m, n, k, op_a, op_b = (int(v) for v in shape[:5])
    out = (C.c_float * N_FEATURES)()
    st = _lib.load().coral_selector_features_tile(shape_products(shape), op_a, op_b, m, n, k, tm, tn, sp, out)
    if st != 0:
        raise RuntimeError(f"coral_selector_features_tile: {st}")
    return np.frombuffer(out, dtype=np.float32).copy()


def feature_matrix(shapes: np.ndarray) -> np.ndarray:
    """[len(shapes) * 15, 13] in shape-major, candidate-minor order."""
    return np.stack([features(s, *c) for s in shapes for c in CANDIDATES])


def valid_mask(shapes: np.ndarray) -> np.ndarray:
    """[len(shapes), 15] bool."""
    return np.array([[valid(s, c) for c in CANDIDATES] for s in shapes])


def default_choice(shape, sm_count: int = 148) -> int:
    """Index in CANDIDATES of the library's default rule (no selector)."""
    m, n, k = (int(v) for v in shape[:3])
    if -(-m // 256) * -(-n // 256) >= sm_count:
        return CANDIDATES.index((256, 256, 1))
    tn = 256 if shape_products(shape) == 3 else 128
    tiles = -(-m // 128) * -(-n // 256)
    sp = 1
    if tiles * 2 <= sm_count and -(-k // 64) >= 16:
        sp = min(16, max(1, sm_count // tiles))
    sp = min(sp, max(1, -(-k // 64)))
    best = max([s for s in (1, 2, 4, 8, 16) if s <= sp])
    return CANDIDATES.index((128, tn, best))


# ------------------------------------------------------------ autotune DB --
def collect(shapes: np.ndarray, reps_small: int = 3, log_every: int = 500) -> np.ndarray:
    """Exhaustively times every candidate of every shape: [len(shapes), 15] ms
    (+inf where the shape's mode has no such configuration)."""
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
    times = np.full((len(shapes), len(CANDIDATES)), np.inf, np.float32)
    t0 = time.time()
    for i, s in enumerate(shapes):
        times[i] = time_all(lib, h, s, A, B, Cm, reps_small)
        if log_every and (i + 1) % log_every == 0:
            print(f"  {i + 1}/{len(shapes)} shapes, {time.time() - t0:.0f} s", flush=True)
    return times


def time_all(lib, h, shape, A, B, Cm, reps_small: int = 3) -> np.ndarray:
    """[15] ms of every configuration of one shape (coral_autotune_sgemm_tiles),
    +inf where the mode has none."""
    m, n, k, op_a, op_b = (int(v) for v in shape[:5])
    prod = shape_products(shape)
    lda = m if op_a == 0 else k
    ldb = k if op_b == 0 else n
    reps = reps_small if 2.0 * m * n * k * prod / 3 < 2e10 else 1
    ms = (C.c_float * len(CANDIDATES))()
    count, best = C.c_int(), C.c_int()
    st = lib.coral_autotune_sgemm_tiles(h.h, prod, op_a, op_b, m, n, k, C.c_void_p(A.data_ptr()), lda,
                                        C.c_void_p(B.data_ptr()), ldb, C.c_void_p(Cm.data_ptr()), m, reps, ms,
                                        len(CANDIDATES), C.byref(count), C.byref(best))
    if st != 0:
        raise RuntimeError(f"coral_autotune_sgemm_tiles failed on {m}x{n}x{k}: {st}")
    got = np.frombuffer(ms, dtype=np.float32)[:count.value]
    out = np.full(len(CANDIDATES), np.inf, np.float32)
    out[[j for j, c in enumerate(CANDIDATES) if valid(shape, c)]] = got
    return out


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
    ok = np.isfinite(db_times.reshape(-1))
    X = torch.from_numpy(feature_matrix(db_shapes)[ok]).cuda()
    y = torch.from_numpy(np.log(np.maximum(db_times.reshape(-1, 1)[ok], 1e-4)).astype(np.float32)).cuda()
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


def choose(pred: np.ndarray, shapes: np.ndarray) -> np.ndarray:
    """Argmin of predicted log ms over each shape's valid configurations."""
    pred = np.asarray(pred, np.float64).reshape(len(shapes), len(CANDIDATES))
    return np.where(valid_mask(shapes), pred, np.inf).argmin(axis=1)


def predict_choice(net: Mlp, shapes: np.ndarray) -> np.ndarray:
    import torch
    X = torch.from_numpy(feature_matrix(shapes)).cuda()
    return choose(net.forward(X).cpu().numpy(), shapes)


def regret(times: np.ndarray, choice: np.ndarray) -> np.ndarray:
    best = times.min(axis=1)
    return times[np.arange(len(times)), choice] / best - 1.0


def evaluate_live(net: Mlp, shapes: np.ndarray, reps_small: int = 3) -> dict:
    """Regret measured on the GPU, not read from a table: for each shape, every
    configuration is timed (exhaustive autotune), then coral_sgemm is timed
    with the configuration the library itself picks -- once with the network
    attached to the handle as its selector, once with the default rule."""
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

    def time_policy(s, reps, trials=3):
        """Median over `trials` of the per-call time of `reps` back-to-back calls."""
        m, n, k, op_a, op_b = (int(v) for v in s[:5])
        lda, ldb = (m if op_a == 0 else k), (k if op_b == 0 else n)
        h.set_gemm_mode(3 if shape_products(s) == 6 else 1)  # SPLIT_BF16X6 / SPLIT_BF16X3
        h.set_gemm_tile(0, 0, 0)
        args = (h.h, op_a, op_b, m, n, k, C.c_float(1.0), C.c_void_p(A.data_ptr()), lda,
                C.c_void_p(B.data_ptr()), ldb, C.c_float(0.0), C.c_void_p(Cm.data_ptr()), m)
        h.check(lib.coral_sgemm(*args), "coral_sgemm")
        out = []
        for _ in range(trials):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                lib.coral_sgemm(*args)
            e1.record()
            torch.cuda.synchronize()
            out.append(e0.elapsed_time(e1) / reps)
        return float(np.median(out))

    rows = []
    for s in shapes:
        m, n, k = (int(v) for v in s[:3])
        reps = reps_small if 2.0 * m * n * k * shape_products(s) / 3 < 2e10 else 1
        t_all = time_all(lib, h, s, A, B, Cm, reps_small)
        net.attach(h)
        t_sel = time_policy(s, reps)
        tm, tn, sk = h.gemm_tile(shape_products(s), int(s[3]), int(s[4]), m, n, k)
        lib.coral_set_selector(h.h, None)
        t_def = time_policy(s, reps)
        rows.append({"shape": [int(v) for v in s], "best_ms": float(t_all.min()),
                     "best": list(CANDIDATES[int(t_all.argmin())]), "selector_ms": t_sel,
                     "selector_choice": [tm, tn, sk], "default_ms": t_def,
                     "selector_table_ms": float(t_all[CANDIDATES.index((tm, tn, sk))])
                     if (tm, tn, sk) in CANDIDATES else None})
    h.set_gemm_mode(0)
    r_sel = np.array([x["selector_ms"] / x["best_ms"] - 1 for x in rows])
    r_def = np.array([x["default_ms"] / x["best_ms"] - 1 for x in rows])
    return {"shapes": len(rows), "selector": summarize(r_sel), "default_rule": summarize(r_def),
            "pair_chosen": float(np.mean([x["selector_choice"][0] == 256 for x in rows])),
            "pair_best": float(np.mean([x["best"][0] == 256 for x in rows])), "rows": rows}


def summarize(r: np.ndarray) -> dict:
    return {"mean": float(r.mean()), "p50": float(np.median(r)), "p95": float(np.quantile(r, 0.95)),
            "max": float(r.max()), "frac_optimal": float((r <= 1e-9).mean())}


# ----------------------------------------------- grouped GEMM tile policy --
# The tensor-core grouped GEMM takes one N tile width per instance class
# (n <= 64, <= 128, <= 256, > 256).  A second network of the same shape
# predicts the log time of a uniform batch (one shape, `batch` instances) under
# each width, from features whose data type (fp32 split / bf16 inputs) and
# batch count vary over the training set; coral_select_grouped_config applies
# it per class of a real batch.
GROUPED_WIDTHS = (64, 128, 256)
GROUPED_CLASS_WIDTHS = ((64, 128), (64, 128), (64, 128, 256), (64, 128, 256))


def grouped_policies() -> list:
    """The 36 policies in coral_autotune_sgemm_grouped's order (class 0 slowest)."""
    return [(a, b, c, d) for a in GROUPED_CLASS_WIDTHS[0] for b in GROUPED_CLASS_WIDTHS[1]
            for c in GROUPED_CLASS_WIDTHS[2] for d in GROUPED_CLASS_WIDTHS[3]]


def grouped_samples(count: int, seed: int) -> np.ndarray:
    """[count, 7] int64: input_type, op_a, op_b, m, n, k, batch.  m, n, k
    log-uniform in [16, 1024]; batch log-uniform in [1, 4096], capped so the
    batch holds at most 2^25 output elements and 2^34 multiply-adds."""
    rng = np.random.default_rng(seed)
    dims = np.exp(rng.uniform(np.log(16), np.log(1024), (count, 3))).astype(np.int64)
    batch = np.exp(rng.uniform(0, np.log(4096), count)).astype(np.int64)
    mn = dims[:, 0] * dims[:, 1]
    batch = np.minimum(batch, np.maximum(1, (1 << 25) // mn))
    batch = np.minimum(batch, np.maximum(1, (1 << 34) // (mn * dims[:, 2])))
    it = rng.integers(0, 2, count)
    op_a = rng.integers(0, 2, count)
    op_b = (rng.uniform(size=count) < 0.25).astype(np.int64)
    return np.stack([it, op_a, op_b, dims[:, 0], dims[:, 1], dims[:, 2], batch], axis=1)


def grouped_feature(sample, bn: int) -> np.ndarray:
    it, op_a, op_b, m, n, k, b = (int(v) for v in sample)
    out = (C.c_float * N_FEATURES)()
    st = _lib.load().coral_grouped_features(it, op_a, op_b, m, n, k, b, bn, out)
    if st != 0:
        raise RuntimeError(f"coral_grouped_features: {st}")
    return np.frombuffer(out, dtype=np.float32).copy()


def grouped_feature_matrix(samples: np.ndarray) -> np.ndarray:
    """[len(samples) * 3, 13], sample-major, width-minor."""
    return np.stack([grouped_feature(s, bn) for s in samples for bn in GROUPED_WIDTHS])


def uniform_records(b, op_a, op_b, m, n, k, ptr_a, ptr_b, ptr_c):
    """Descriptor records of b instances of one shape sharing A and B, each
    with its own m x n block of C."""
    from .blas import sgemm_problem_dtype
    rec = np.zeros(b, dtype=sgemm_problem_dtype())
    for f, v in (("op_a", op_a), ("op_b", op_b), ("m", m), ("n", n), ("k", k), ("alpha", 1.0), ("a", ptr_a),
                 ("b", ptr_b), ("lda", m if op_a == 0 else k), ("ldb", k if op_b == 0 else n), ("ldc", m)):
        rec[f] = v
    rec["c"] = ptr_c + 4 * m * n * np.arange(b, dtype=np.uint64)
    return rec


def collect_grouped(samples: np.ndarray, reps: int = 3, log_every: int = 1000) -> np.ndarray:
    """Times each uniform batch under every width: [len(samples), 3] ms."""
    import torch
    h = handle()
    h.bind_current_stream()
    lib = _lib.load()
    need_ab = int(max(max(s[3] * s[5], s[5] * s[4]) for s in samples))
    need_c = int(max(s[3] * s[4] * s[6] for s in samples))
    A32 = torch.empty(need_ab, dtype=torch.float32, device="cuda").uniform_(-1, 1)
    B32 = torch.empty(need_ab, dtype=torch.float32, device="cuda").uniform_(-1, 1)
    A16, B16 = A32.to(torch.bfloat16), B32.to(torch.bfloat16)
    Cd = torch.zeros(need_c, dtype=torch.float32, device="cuda")
    times = np.zeros((len(samples), len(GROUPED_WIDTHS)), np.float32)
    saved_mode = h.gemm_mode()
    h.set_gemm_mode(1)   # SPLIT_BF16X3: fp32 inputs on the tensor cores
    t0 = time.time()
    try:
        for i, (it, op_a, op_b, m, n, k, b) in enumerate(samples):
            it, op_a, op_b, m, n, k, b = (int(v) for v in (it, op_a, op_b, m, n, k, b))
            A, B = (A16, B16) if it == 1 else (A32, B32)
            rec = uniform_records(b, op_a, op_b, m, n, k, A.data_ptr(), B.data_ptr(), Cd.data_ptr())
            desc = torch.from_numpy(rec.view(np.uint8)).cuda()
            evs = []
            for bn in GROUPED_WIDTHS:
                lib.coral_set_grouped_config(h.h, (C.c_int * 4)(bn, bn, bn, bn))
                h.check(lib.coral_sgemm_grouped(h.h, it, b, C.c_void_p(desc.data_ptr())), "grouped")
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(reps):
                    h.check(lib.coral_sgemm_grouped(h.h, it, b, C.c_void_p(desc.data_ptr())), "grouped")
                e1.record()
                evs.append((e0, e1))
            torch.cuda.synchronize()
            times[i] = [e0.elapsed_time(e1) / reps for e0, e1 in evs]
            if log_every and (i + 1) % log_every == 0:
                print(f"  {i + 1}/{len(samples)} batches, {time.time() - t0:.0f} s", flush=True)
    finally:
        lib.coral_set_grouped_config(h.h, None)
        h.set_gemm_mode(saved_mode)
    return times


def train_grouped(samples: np.ndarray, times: np.ndarray, epochs: int = 400, batch: int = 2048,
                  lr: float = 2e-3, seed: int = 0) -> tuple[Mlp, list]:
    """Fits log(ms) of every (uniform batch, width) pair with the library's kernels."""
    import torch
    X = torch.from_numpy(grouped_feature_matrix(samples)).cuda()
    y = torch.from_numpy(np.log(np.maximum(times.reshape(-1, 1), 1e-4)).astype(np.float32)).cuda()
    net = Mlp(seed=seed)
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    history = []
    n = X.shape[0]
    for ep in range(epochs):
        perm = torch.randperm(n, device="cuda", generator=g)
        tot, steps = 0.0, 0
        lr_ep = lr * (0.5 * (1 + np.cos(np.pi * ep / epochs)) * 0.95 + 0.05)
        for s0 in range(0, n, batch):
            idx = perm[s0:s0 + batch]
            tot += net.train_step(X[idx].contiguous(), y[idx].contiguous(), float(lr_ep))
            steps += 1
        history.append(tot / max(steps, 1))
    return net, history


def predict_grouped_choice(predict, samples: np.ndarray) -> np.ndarray:
    """Index into GROUPED_WIDTHS of the predicted fastest width per sample;
    `predict` maps a feature matrix to predicted log times."""
    pred = np.asarray(predict(grouped_feature_matrix(samples))).reshape(len(samples), len(GROUPED_WIDTHS))
    return pred.argmin(1)


def uneven_batches(count: int, seed: int, max_elems: int = 1 << 27) -> list:
    """Held-out uneven batches: [(input_type, [(op_a, op_b, m, n, k), ...])].
    Each batch draws its instance count log-uniform in [64, 4096], one of
    several dimension ranges and an operation mix, up to max_elems operand
    elements in total."""
    rng = np.random.default_rng(seed)
    ranges = [(16, 512), (16, 128), (32, 256), (64, 1024), (128, 2048), (16, 2048)]
    out = []
    for _ in range(count):
        it = int(rng.integers(0, 2))
        lo, hi = ranges[int(rng.integers(0, len(ranges)))]
        want = int(np.exp(rng.uniform(np.log(64), np.log(4096))))
        p_t = float(rng.uniform(0, 1))
        insts, elems = [], 0
        for _ in range(want):
            m, n, k = (int(v) for v in np.exp(rng.uniform(np.log(lo), np.log(hi), 3)))
            e = m * k + k * n + m * n
            if elems + e > max_elems:
                break
            elems += e
            insts.append((int(rng.uniform() < p_t), int(rng.uniform() < 0.25), m, n, k))
        out.append((it, insts))
    return out


def _default_policy(h, lib):
    lib.coral_set_grouped_config(h.h, None)
    tn = (C.c_int * 4)()
    lib.coral_get_grouped_config(h.h, tn)
    return tuple(int(v) for v in tn)


def evaluate_grouped_live(net: Mlp, batches: list, reps: int = 3) -> dict:
    """For every held-out batch, on this GPU: all 36 policies timed by
    coral_autotune_sgemm_grouped, the network's choice
    (coral_select_grouped_config) and the exhaustive best re-timed on their
    own, and the default policy.  Returns per-batch records and the regret
    summaries t(choice) / t(exhaustive best) - 1."""
    import torch
    from .blas import sgemm_problem_dtype
    h = handle()
    h.bind_current_stream()
    lib = _lib.load()
    pols = grouped_policies()
    default = _default_policy(h, lib)
    rows = []
    saved_mode = h.gemm_mode()
    h.set_gemm_mode(1)
    try:
        for it, insts in batches:
            dt = torch.bfloat16 if it == 1 else torch.float32
            na = sum(m * k for _, _, m, n, k in insts)
            nb = sum(k * n for _, _, m, n, k in insts)
            nc = sum(m * n for _, _, m, n, k in insts)
            A = torch.empty(na, dtype=torch.float32, device="cuda").uniform_(-1, 1).to(dt)
            B = torch.empty(nb, dtype=torch.float32, device="cuda").uniform_(-1, 1).to(dt)
            Cd = torch.zeros(nc, dtype=torch.float32, device="cuda")
            es = A.element_size()
            rec = np.zeros(len(insts), dtype=sgemm_problem_dtype())
            oa = ob = oc = 0
            for i, (op_a, op_b, m, n, k) in enumerate(insts):
                rec[i] = (op_a, op_b, m, n, k, 1.0, 0.0, 0, A.data_ptr() + oa * es, B.data_ptr() + ob * es,
                          Cd.data_ptr() + oc * 4, m if op_a == 0 else k, k if op_b == 0 else n, m)
                oa += m * k
                ob += k * n
                oc += m * n
            desc = torch.from_numpy(rec.view(np.uint8)).cuda()
            ms = (C.c_float * 36)()
            best = C.c_int()
            tn = (C.c_int * 4)()
            h.check(lib.coral_autotune_sgemm_grouped(h.h, it, len(insts), C.c_void_p(desc.data_ptr()), reps, ms,
                                                     C.byref(best), tn), "autotune grouped")
            table = np.frombuffer(ms, dtype=np.float32).copy()
            sel = (C.c_int * 4)()
            h.check(lib.coral_select_grouped_config(h.h, net.p, it, len(insts), rec.ctypes.data_as(C.c_void_p),
                                                    sel), "select grouped")
            choice = tuple(int(v) for v in sel)

            def time_policy(pol):
                lib.coral_set_grouped_config(h.h, (C.c_int * 4)(*pol))
                h.check(lib.coral_sgemm_grouped(h.h, it, len(insts), C.c_void_p(desc.data_ptr())), "grouped")
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(reps):
                    lib.coral_sgemm_grouped(h.h, it, len(insts), C.c_void_p(desc.data_ptr()))
                e1.record()
                torch.cuda.synchronize()
                return e0.elapsed_time(e1) / reps
            t_sel = time_policy(choice)
            t_best = time_policy(pols[int(best.value)])
            rows.append({"input": "bf16" if it == 1 else "fp32", "instances": len(insts),
                         "best_ms": float(table.min()), "choice_ms": float(table[pols.index(choice)]),
                         "default_ms": float(table[pols.index(default)]),
                         "choice_ms_retimed": t_sel, "best_ms_retimed": t_best,
                         "choice": list(choice), "best": list(pols[int(best.value)])})
            del A, B, Cd, desc
    finally:
        lib.coral_set_grouped_config(h.h, None)
        h.set_gemm_mode(saved_mode)
    r_sel = np.array([x["choice_ms"] / x["best_ms"] - 1 for x in rows])
    r_def = np.array([x["default_ms"] / x["best_ms"] - 1 for x in rows])
    r_live = np.array([x["choice_ms_retimed"] / x["best_ms_retimed"] - 1 for x in rows])
    return {"batches": rows, "selector": summarize(r_sel), "default_policy": summarize(r_def),
            "selector_retimed": summarize(r_live)}


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
    el = sub.add_parser("evaluate-live")
    el.add_argument("--db", required=True)
    el.add_argument("--weights", required=True)
    el.add_argument("--count", type=int, default=300)
    el.add_argument("--out", default="")
    gc = sub.add_parser("grouped-collect")
    gc.add_argument("--count", type=int, default=6000)
    gc.add_argument("--seed", type=int, default=11)
    gc.add_argument("--out", required=True)
    gt = sub.add_parser("grouped-train")
    gt.add_argument("--db", required=True)
    gt.add_argument("--out", required=True)
    gt.add_argument("--epochs", type=int, default=400)
    ge = sub.add_parser("grouped-evaluate")
    ge.add_argument("--weights", required=True)
    ge.add_argument("--batches", type=int, default=40)
    ge.add_argument("--seed", type=int, default=12)
    ge.add_argument("--out", default="")
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
        fixed = np.array([CANDIDATES.index((128, 256 if shape_products(s) == 3 else 128, 1))
                          for s in d["shapes"]])
        print(json.dumps({"shapes": int(len(d["shapes"])),
                          "selector": summarize(regret(d["times"], choice)),
                          "default_rule": summarize(regret(d["times"], dflt)),
                          "fixed_single_cta_no_split": summarize(regret(d["times"], fixed))}))
    elif args.cmd == "evaluate-live":
        d = np.load(args.db)
        net = Mlp.load(args.weights)
        res = evaluate_live(net, d["shapes"][:args.count])
        if args.out:
            with open(args.out, "w") as f:
                json.dump(res, f)
        print(json.dumps({k: v for k, v in res.items() if k != "rows"}))
    elif args.cmd == "grouped-collect":
        samples = grouped_samples(args.count, args.seed)
        t0 = time.time()
        times = collect_grouped(samples)
        np.savez_compressed(args.out, samples=samples, times=times, widths=np.array(GROUPED_WIDTHS),
                            seed=args.seed)
        print(json.dumps({"collected": len(samples), "seconds": time.time() - t0, "out": args.out}))
    elif args.cmd == "grouped-train":
        import torch
        d = np.load(args.db)
        t0 = time.time()
        net, hist = train_grouped(d["samples"], d["times"], epochs=args.epochs)
        net.save(args.out, {"db": os.path.basename(args.db), "epochs": args.epochs,
                            "final_mse": hist[-1], "seconds": time.time() - t0})
        choice = predict_grouped_choice(lambda X: net.forward(torch.from_numpy(X).cuda()).cpu().numpy(),
                                        d["samples"])
        print(json.dumps({"train_mse": hist[-1], "train_regret": summarize(regret(d["times"], choice)),
                          "seconds": time.time() - t0}))
    elif args.cmd == "grouped-evaluate":
        net = Mlp.load(args.weights)
        res = evaluate_grouped_live(net, uneven_batches(args.batches, args.seed))
        if args.out:
            with open(args.out, "w") as f:
                json.dump(res, f)
        print(json.dumps({k: v for k, v in res.items() if k != "batches"}))


if __name__ == "__main__":
    main()

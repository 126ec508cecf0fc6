"""The learned planner: a cost model trained on the measuring planner's timings.

The measuring planner (CRDFFT_PLANNER_MEASURE) times every candidate launch shape of every pass of a plan on the
device; its log carries, per candidate, the measured time and the feature vector of (pass, shape). This module

* generates seeded planning problems (1-D C2C and R2C, 2-D C2C; 7-smooth sizes; batch log-uniform in 1..65536 with
  the input capped at 2 GiB; unit or padded (+8) distances; FP32 or split-BF16),
* collects the exhaustive planner's timings for each (`collect`),
* trains a 3-layer MLP (FP32, 64 hidden units) to predict log(ms) with the library's own device kernels
  (crdfft_mlp_gradients / crdfft_mlp_adam, `train`),
* evaluates it on held-out problems (`evaluate`): the runtime of the shapes the model picks against the best measured
  ones (achieved / optimal) and the planning time of both planners.

The reference has no counterpart: its planner reads a board of per-level winners measured offline
(include/crd/hesap/fft/detail/level_plans_gen.hpp:33-148) and picks by size alone.

    python -m crd_b200.learned_planner --train 2000 --heldout 500 --model crd_b200/data/planner_mlp_b200.txt \
        --report profiles/learned_planner_b200.json
"""

from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import time
from dataclasses import dataclass, field

import numpy as np

from . import hesap as F
from ._lib import C2C, R2C, PREC_FP32, PREC_SPLIT_BF16, check, lib

FEATURES = 32
HIDDEN = 64
TRAIN_SEED = 0x5EED0005
HELDOUT_SEED = 0x5EED0105
MAX_INPUT_BYTES = 2 << 30


def smooth7(lo: int, hi: int) -> list[int]:
    """The 7-smooth integers in [lo, hi]."""
    out = []
    p2 = 1
    while p2 <= hi:
        p3 = p2
        while p3 <= hi:
            p5 = p3
            while p5 <= hi:
                p7 = p5
                while p7 <= hi:
                    if p7 >= lo:
                        out.append(p7)
                    p7 *= 7
                p5 *= 5
            p3 *= 3
        p2 *= 2
    return sorted(out)


@dataclass
class Problem:
    dims: tuple
    batch: int
    kind: int
    padded: bool
    precision: int

    def desc_kwargs(self) -> dict:
        pts = int(np.prod(self.dims))
        kw = {"batch": self.batch, "kind": self.kind, "precision": self.precision}
        if self.padded:
            if self.kind == R2C:
                kw.update(idist=pts + 8, odist=pts // 2 + 1 + 8)
            else:
                kw.update(idist=pts + 8, odist=pts + 8)
        return kw

    def label(self) -> str:
        k = "r2c" if self.kind == R2C else "c2c"
        p = "bf16x3" if self.precision == PREC_SPLIT_BF16 else "fp32"
        return f"{k} {'x'.join(map(str, self.dims))} b{self.batch}{' pad' if self.padded else ''} {p}"


def problems(count: int, seed: int) -> list[Problem]:
    """Seeded problems: a quarter each 1-D C2C, 1-D R2C, 2-D C2C and 2-D R2C. 1-D sizes log-uniform over the 7-smooth
    integers in [64, 2^22] (R2C: the even ones); 2-D sides over those in [16, 4096] with at least 64 points (R2C: an
    even last side); batch log-uniform in [1, 65536], capped so the input stays within 2 GiB; half padded (+8 elements
    between transforms; 2-D R2C plans take packed batches only); half split-BF16."""
    rng = np.random.default_rng(seed)
    s1 = np.array(smooth7(64, 1 << 22))
    s1e = s1[s1 % 2 == 0]
    s2 = np.array(smooth7(16, 4096))

    def pick(cands, lo, hi):
        x = math.exp(rng.uniform(math.log(lo), math.log(hi)))
        i = int(np.searchsorted(cands, x))
        return int(cands[min(i, len(cands) - 1)])

    out = []
    s2e = s2[s2 % 2 == 0]
    for _ in range(count):
        shape = int(rng.integers(0, 4))
        if shape == 0:
            dims, kind = (pick(s1, 64, 1 << 22),), C2C
        elif shape == 1:
            dims, kind = (pick(s1e, 64, 1 << 22),), R2C
        else:
            while True:
                dims = (pick(s2, 16, 4096), pick(s2e if shape == 3 else s2, 16, 4096))
                if dims[0] * dims[1] >= 64:
                    break
            kind = R2C if shape == 3 else C2C
        pts = int(np.prod(dims))
        elem = 4 if kind == R2C else 8
        batch = int(round(math.exp(rng.uniform(0.0, math.log(65536)))))
        batch = max(1, min(batch, MAX_INPUT_BYTES // ((pts + 8) * elem)))
        padded = bool(rng.integers(0, 2)) and not (kind == R2C and len(dims) == 2)
        precision = PREC_SPLIT_BF16 if rng.integers(0, 2) else PREC_FP32
        out.append(Problem(dims, batch, kind, padded, precision))
    return out


@dataclass
class PassGroup:
    key: str
    feats: np.ndarray            # candidates x FEATURES
    ms: np.ndarray               # measured time of the whole pass per candidate
    best: int
    heur: int                    # the heuristic planner's choice, or -1


@dataclass
class Measured:
    problem: Problem
    groups: list = field(default_factory=list)    # pass launch-shape candidates
    dgroups: list = field(default_factory=list)   # decomposition candidates of the plan's 1-D lengths
    plan_ms: float = 0.0         # wall time of plan creation in measure mode (exhaustive planning)
    wisdom: str = ""             # the wisdom the exhaustive planner left (its plan, re-created for the evaluation)
    error: str = ""


def parse_log(text: str, decomp: bool = False) -> list[PassGroup]:
    """Group the planner log's candidate lines by pass (consecutive lines with one key); drop failed candidates.
    decomp: the decomposition lines (" decomp " entries) instead of the launch-shape lines."""
    groups: list[PassGroup] = []
    cur_key, rows = None, []

    def flush():
        if cur_key is None or not rows:
            return
        ok = [r for r in rows if r[1] > 0]
        if not ok:
            return
        feats = np.array([r[0] for r in ok], dtype=np.float32)
        ms = np.array([r[1] for r in ok], dtype=np.float64)
        heur = next((i for i, r in enumerate(ok) if r[2]), -1)
        groups.append(PassGroup(cur_key, feats, ms, int(np.argmin(ms)), heur))

    for line in text.splitlines():
        parts = line.split()
        if not parts or (len(parts) > 1 and parts[1] == "decomp") != decomp:
            continue
        key = parts[0]
        kv = dict(p.split("=", 1) for p in parts[1:] if "=" in p)
        feat = [float(v) for v in kv["feat"].split(",")]
        row = (feat, float(kv["ms"]), "heur" in parts[1:])
        if key != cur_key:
            flush()
            cur_key, rows = key, []
        rows.append(row)
    flush()
    return groups


def collect(probs: list[Problem], progress: bool = False) -> list[Measured]:
    """Plan each problem with the measuring planner from empty wisdom and keep its timings."""
    import torch  # noqa: F401  (initialises the CUDA context the library uses)

    out = []
    F.set_planner("measure")
    for i, pr in enumerate(probs):
        F.wisdom_forget()
        m = Measured(pr)
        t0 = time.perf_counter()
        try:
            plan = F.Plan(list(pr.dims), **pr.desc_kwargs())
            m.plan_ms = (time.perf_counter() - t0) * 1e3
            del plan
            log = F.planner_log()
            m.groups = parse_log(log)
            m.dgroups = parse_log(log, decomp=True)
            m.wisdom = F.wisdom_export()
        except F.CrdFftError as exc:
            m.error = str(exc)
        out.append(m)
        if progress and i % 100 == 0:
            print(f"  {i}/{len(probs)} {pr.label()}: {len(m.groups)} passes, plan {m.plan_ms:.1f} ms", flush=True)
    F.wisdom_forget()
    F.set_planner("estimate")
    return out


def dataset(measured: list[Measured], decomp: bool = False):
    """Feature rows and targets: log(ms) of the launch-shape candidates; for the decompositions (decomp), log(ms)
    relative to the mean over the same transform's candidates, because the planner only ranks the decompositions
    of one transform against each other and their times differ far less than across transforms."""
    xs, ys = [], []
    for m in measured:
        for g in (m.dgroups if decomp else m.groups):
            xs.append(g.feats)
            lg = np.log(g.ms)
            ys.append(lg - lg.mean() if decomp else lg)
    if not xs:
        return np.zeros((0, FEATURES), dtype=np.float32), np.zeros(0, dtype=np.float32)
    return np.concatenate(xs).astype(np.float32), np.concatenate(ys).astype(np.float32)


PASS_TAG = "crdfft-mlp"
DECOMP_TAG = "crdfft-mlp-decomp"


@dataclass
class Model:
    mean: np.ndarray
    std: np.ndarray
    t_mean: float
    t_std: float
    params: np.ndarray
    hidden: int = HIDDEN
    tag: str = PASS_TAG          # which ranking the model serves: launch shapes or decompositions

    def text(self) -> str:
        f = lambda v: f"{float(v):.9g}"  # noqa: E731
        lines = [f"{self.tag} 1", f"dims {FEATURES} {self.hidden}",
                 "mean " + " ".join(map(f, self.mean)), "std " + " ".join(map(f, self.std)),
                 f"target {f(self.t_mean)} {f(self.t_std)}", f"params {len(self.params)}"]
        for i in range(0, len(self.params), 8):
            lines.append(" ".join(map(f, self.params[i:i + 8])))
        return "\n".join(lines) + "\n"

    @staticmethod
    def parse(text: str) -> "Model":
        """The first model of a model text."""
        return Model.parse_all(text)[0]

    @staticmethod
    def parse_all(text: str) -> list:
        """Every model of a model text, in order."""
        tok = text.split()
        out = []
        while tok:
            m, used = Model._parse_tokens(tok)
            out.append(m)
            tok = tok[used:]
        return out

    @staticmethod
    def _parse_tokens(tok: list) -> tuple:
        assert tok[0] in (PASS_TAG, DECOMP_TAG) and tok[1] == "1" and tok[2] == "dims"
        tag = tok[0]
        d, h = int(tok[3]), int(tok[4])
        i = 5
        assert tok[i] == "mean"
        mean = np.array(tok[i + 1:i + 1 + d], dtype=np.float32)
        i += 1 + d
        assert tok[i] == "std"
        std = np.array(tok[i + 1:i + 1 + d], dtype=np.float32)
        i += 1 + d
        assert tok[i] == "target"
        tm, ts = float(tok[i + 1]), float(tok[i + 2])
        i += 3
        assert tok[i] == "params"
        n = int(tok[i + 1])
        params = np.array(tok[i + 2:i + 2 + n], dtype=np.float32)
        return Model(mean, std, tm, ts, params, h, tag), i + 2 + n


def init_params(d: int, h: int, seed: int) -> np.ndarray:
    """He-uniform weights, zero biases, in the flat layout of crdfft_mlp_param_count."""
    rng = np.random.default_rng(seed)
    parts = []
    for fan_in, fan_out in ((d, h), (h, h), (h, 1)):
        lim = math.sqrt(6.0 / fan_in)
        parts.append(rng.uniform(-lim, lim, size=fan_out * fan_in).astype(np.float32))
        parts.append(np.zeros(fan_out, dtype=np.float32))
    return np.concatenate(parts)


def train(x: np.ndarray, y: np.ndarray, steps: int = 4000, lr: float = 3e-3, seed: int = 1,
          hidden: int = HIDDEN, log_every: int = 0, tag: str = PASS_TAG) -> tuple[Model, list]:
    """Full-batch Adam on mean-squared error of normalised log(ms), on the device with the library's kernels."""
    import torch

    L = lib()
    mean = x.mean(axis=0)
    std = x.std(axis=0)
    std = np.where(std < 1e-6, 1.0, std).astype(np.float32)
    t_mean, t_std = float(y.mean()), float(max(y.std(), 1e-6))
    xn = ((x - mean) / std).astype(np.float32)
    yn = ((y - t_mean) / t_std).astype(np.float32)
    rows = xn.shape[0]
    dev = torch.device("cuda")
    X = torch.from_numpy(xn).to(dev).contiguous()
    Y = torch.from_numpy(yn).to(dev).contiguous()
    npar = L.crdfft_mlp_param_count(FEATURES, hidden)
    P = torch.from_numpy(init_params(FEATURES, hidden, seed)).to(dev)
    assert P.numel() == npar
    G = torch.zeros_like(P)
    M = torch.zeros_like(P)
    V = torch.zeros_like(P)
    W = torch.empty(L.crdfft_mlp_workspace_floats(FEATURES, hidden, rows), dtype=torch.float32, device=dev)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    st = torch.cuda.current_stream().cuda_stream
    history = []
    for s in range(1, steps + 1):
        check(L.crdfft_mlp_gradients(FEATURES, hidden, P.data_ptr(), X.data_ptr(), Y.data_ptr(), rows, G.data_ptr(),
                                     loss.data_ptr(), W.data_ptr(), st), "mlp_gradients")
        # cosine decay to a tenth of the rate
        rate = lr * (0.1 + 0.9 * 0.5 * (1.0 + math.cos(math.pi * (s - 1) / steps)))
        check(L.crdfft_mlp_adam(P.data_ptr(), G.data_ptr(), M.data_ptr(), V.data_ptr(), npar, s, rate, 0.9, 0.999,
                                1e-8, st), "mlp_adam")
        if log_every and (s % log_every == 0 or s == 1):
            history.append((s, float(loss.item())))
    torch.cuda.synchronize()
    history.append((steps, float(loss.item())))
    return Model(mean.astype(np.float32), std, t_mean, t_std, P.cpu().numpy(), hidden, tag), history


def predict_device(model: Model, x: np.ndarray) -> np.ndarray:
    """The model's log(ms) for each row of x with the device forward kernel (crdfft_mlp_forward)."""
    import torch

    L = lib()
    dev = torch.device("cuda")
    xn = torch.from_numpy(((x - model.mean) / model.std).astype(np.float32)).to(dev).contiguous()
    P = torch.from_numpy(model.params).to(dev)
    rows = xn.shape[0]
    out = torch.empty(rows, dtype=torch.float32, device=dev)
    W = torch.empty(L.crdfft_mlp_workspace_floats(FEATURES, model.hidden, rows), dtype=torch.float32, device=dev)
    check(L.crdfft_mlp_forward(FEATURES, model.hidden, P.data_ptr(), xn.data_ptr(), rows, out.data_ptr(),
                               W.data_ptr(), torch.cuda.current_stream().cuda_stream), "mlp_forward")
    torch.cuda.synchronize()
    return model.t_mean + model.t_std * out.cpu().numpy()


def _exec_ms(plan, pr: Problem, bufs: dict) -> float:
    """Cold-L2 device time of one forward execute of `plan` (min of 3 after a warm-up, CUDA events; a 256 MiB write
    between runs evicts the inputs from L2)."""
    import torch

    pts = int(np.prod(pr.dims))
    kw = pr.desc_kwargs()
    half = pts // pr.dims[-1] * (pr.dims[-1] // 2 + 1)
    idist = kw.get("idist", pts)
    odist = kw.get("odist", pts if pr.kind != R2C else half)
    in_dt = torch.float32 if pr.kind == R2C else torch.complex64
    in_n = idist * (pr.batch - 1) + pts
    out_n = odist * (pr.batch - 1) + (pts if pr.kind != R2C else half)
    key = (in_n, in_dt, out_n)
    if bufs.get("key") != key:
        bufs.clear()
        bufs["key"] = key
        bufs["in"] = torch.zeros(in_n, dtype=in_dt, device="cuda")
        bufs["out"] = torch.empty(out_n, dtype=torch.complex64, device="cuda")
        bufs["flush"] = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
    best = None
    for r in range(4):
        bufs["flush"].zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        plan.execute(bufs["in"], bufs["out"], F.FORWARD)
        e1.record()
        torch.cuda.synchronize()
        if r > 0:
            t = e0.elapsed_time(e1)
            best = t if best is None else min(best, t)
    return float(best)


def evaluate(models: list, measured: list[Measured], replan: bool = True) -> dict:
    """On held-out problems, each planner's plan is built and executed on the device at the problem's full size:
    * exhaustive: the measuring planner's plan (its wisdom from the collection, re-created without timing);
    * learned: the models rank the candidates (decompositions and launch shapes) and the measuring planner times
      only their top proposals (planning time measured here, from empty wisdom);
    * heuristic: the fixed rule, nothing timed.
    achieved / optimal is the exhaustive plan's execute time over the learned plan's, per problem; every problem
    whose plans could be built is scored (failures are counted and named)."""
    for m in models:
        F.learned_model_import(m.text())
    ratios, heur_ratios, optimal = [], [], 0
    learned_ms, exhaustive_ms, failed = [], [], []
    bufs: dict = {}
    for m in measured:
        if m.error:
            failed.append(f"{m.problem.label()}: {m.error}")
            continue
        pr = m.problem
        try:
            F.wisdom_forget()
            F.wisdom_import(m.wisdom)
            F.set_planner("estimate")
            t_ex = _exec_ms(F.Plan(list(pr.dims), **pr.desc_kwargs()), pr, bufs)
            F.wisdom_forget()
            F.set_planner("learned")
            t0 = time.perf_counter()
            lp = F.Plan(list(pr.dims), **pr.desc_kwargs())
            learned_ms.append((time.perf_counter() - t0) * 1e3)
            F.set_planner("estimate")
            t_le = _exec_ms(lp, pr, bufs)
            del lp
            F.wisdom_forget()
            t_he = _exec_ms(F.Plan(list(pr.dims), **pr.desc_kwargs()), pr, bufs)
        except F.CrdFftError as exc:
            F.set_planner("estimate")
            failed.append(f"{pr.label()}: {exc}")
            continue
        exhaustive_ms.append(m.plan_ms)
        ratios.append(t_ex / t_le)
        heur_ratios.append(t_ex / t_he)
        optimal += int(t_le <= t_ex * 1.02)
    F.wisdom_forget()
    F.set_planner("estimate")
    bufs.clear()

    def summ(v):
        v = sorted(v)
        return {"mean": float(np.mean(v)), "geomean": float(np.exp(np.mean(np.log(v)))),
                "median": float(statistics.median(v)), "p10": float(v[max(0, len(v) // 10 - 1)]),
                "min": float(v[0])} if v else None

    return {
        "problems": len(ratios),
        "problems_failed": failed,
        "achieved_over_optimal": summ(ratios),
        "heuristic_achieved_over_optimal": summ(heur_ratios),
        "problems_within_2pct_of_exhaustive": optimal,
        "planning_ms_exhaustive": summ(exhaustive_ms),
        "planning_ms_learned": summ(learned_ms),
        "how": "each plan executed once warm then 3 times cold (CUDA events, min) at the problem's full size",
    }


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--heldout", type=int, default=500)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--model", default=os.path.join(os.path.dirname(__file__), "data", "planner_mlp_b200.txt"))
    ap.add_argument("--report", default=None)
    args = ap.parse_args()

    t0 = time.perf_counter()
    tr = collect(problems(args.train, TRAIN_SEED), progress=True)
    t1 = time.perf_counter()
    ho = collect(problems(args.heldout, HELDOUT_SEED), progress=True)
    t2 = time.perf_counter()
    x, y = dataset(tr)
    model, hist = train(x, y, steps=args.steps, log_every=500)
    xd, yd = dataset(tr, decomp=True)
    dmodel, dhist = train(xd, yd, steps=args.steps, log_every=500, tag=DECOMP_TAG)
    t3 = time.perf_counter()
    xh, yh = dataset(ho)
    pred_h = predict_device(model, xh)
    xdh, ydh = dataset(ho, decomp=True)
    pred_dh = predict_device(dmodel, xdh) if xdh.shape[0] else np.zeros(0)
    rep = evaluate([model, dmodel], ho)
    rep.update({
        "train_problems": args.train, "heldout_problems": args.heldout,
        "train_rows": int(x.shape[0]), "heldout_rows": int(xh.shape[0]),
        "train_decomp_rows": int(xd.shape[0]), "heldout_decomp_rows": int(xdh.shape[0]),
        "train_failed": sum(1 for m in tr if m.error), "heldout_failed": sum(1 for m in ho if m.error),
        "loss_history": hist, "decomp_loss_history": dhist,
        "heldout_rmse_log_ms": float(np.sqrt(np.mean((pred_h - yh) ** 2))),
        "heldout_decomp_rmse_log_ms": float(np.sqrt(np.mean((pred_dh - ydh) ** 2))) if xdh.shape[0] else None,
        "seconds": {"collect_train": t1 - t0, "collect_heldout": t2 - t1, "train": t3 - t2},
        "hidden": HIDDEN, "features": FEATURES, "train_seed": hex(TRAIN_SEED), "heldout_seed": hex(HELDOUT_SEED),
    })
    os.makedirs(os.path.dirname(os.path.abspath(args.model)), exist_ok=True)
    with open(args.model, "w") as f:
        f.write(model.text() + dmodel.text())
    if args.report:
        with open(args.report, "w") as f:
            json.dump(rep, f, indent=1)
    print(json.dumps({k: v for k, v in rep.items() if not k.endswith("loss_history")}, indent=1))


if __name__ == "__main__":
    main()

"""The learned warm start (an addition beside the drop-in; the reference has
none).

A small MLP maps the two marginals of an OT instance on the 32 x 32 grid to
its optimal dual potentials; the predicted duals, with a plan recovered from
them by a few rounds of log-domain balancing on the GPU, start plain PDHG,
which finishes the solve and is the judge of its error. Without a network (or
when it is not trusted) the solve starts cold.

    instances   a, b = 32 x 32 histograms (mixtures of 1-5 isotropic Gaussians
                with sigma in [1, 6] px plus a 1e-4 floor, normalised), C the
                squared grid distance / max, computed on the fly from the grid
                coordinates (the solver's "sqeuclid" cost)
    network     2048 -> 1024 -> 1024 -> 2048, GELU, BF16 weights and
                activations, FP32 accumulation on the tensor cores
                (pdot_mlp_* in include/pdot.h, csrc/pdot_mlp.cu)
    features    log(1024 h) / 2 of the concatenated histograms
    targets     the solver's duals (u, v) made tight by a double c-transform
                (rows and columns of tiny mass leave PDHG's duals loose),
                shifted so that mean(u) = mean(v), then standardised with one
                mean and one scale
    data        solver-generated: batched PDHG solves to relative KKT 1e-4;
                every solved instance also gives the exact solutions of its
                15 images under the symmetries of the grid cost (the 8
                isometries of the square, each with or without exchanging
                source and target), which carry the duals along

Device memory for the network's inputs and targets is held by torch (the
plumbing); every network computation is a pdot_mlp_* kernel.
"""
from __future__ import annotations

import ctypes as ct
import math
import time
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _abi, api, instances

SIDE = 32
BINS = SIDE * SIDE
FEATURE_SHIFT = math.log(BINS)
FEATURE_SCALE = 0.5
RECOVER_PLAN = (3e-4, 100)  # (eps, rounds) of the plan recovered from predicted duals
# Where the network's warm starts begin their restart information: at the zero
# point, as a cold start's. Started at the warm point instead (the solver's
# default), the adaptive restart test compares against the warm point's small
# KKT error, which these warm starts first exceed, so they restart late: alone
# they took a median of 65k iterations on 128 held-out instances (15k cold),
# against a median of 8k on the 1024 held-out ones with the zero point.
WARM_RESTART = "zero"


def grid_points(side: int = SIDE) -> np.ndarray:
    yy, xx = np.mgrid[0:side, 0:side]
    return np.stack([xx.ravel(), yy.ravel()], axis=1).astype(np.float32)


def grid_pair(seed: int, side: int = SIDE):
    """The marginals of instance `seed` (source, target)."""
    rng = np.random.default_rng(seed)
    return instances.grid_histogram(rng, side), instances.grid_histogram(rng, side)


def canonical_duals(u: np.ndarray, v: np.ndarray):
    """Shift (u + t, v - t) so that mean(u) = mean(v); the shift keeps u_i + v_j."""
    t = 0.5 * (np.mean(v) - np.mean(u))
    return u + t, v - t


_GRID_COST = {}


def grid_cost(side: int = SIDE) -> np.ndarray:
    if side not in _GRID_COST:
        _GRID_COST[side] = instances.grid_cost(side)
    return _GRID_COST[side]


def tight_duals(u: np.ndarray, v: np.ndarray, C: np.ndarray):
    """The double c-transform u' = min_j (C_ij - v_j), v' = min_i (C_ij - u'_i):
    a feasible dual pair, each the c-transform of the other, in which the
    values PDHG leaves loose (rows and columns of tiny mass, whose constraints
    never bind) are made tight; then the canonical shift."""
    u1 = np.min(C - np.asarray(v, dtype=np.float64)[None, :], axis=1)
    v1 = np.min(C - u1[:, None], axis=0)
    return canonical_duals(u1, v1)


def grid_symmetries(side: int = SIDE):
    """Index maps p of the 8 isometries of the square grid: (h o p) is the
    image of histogram h. The squared grid distance is invariant under each."""
    idx = np.arange(side * side).reshape(side, side)
    maps = []
    for k in range(4):
        r = np.rot90(idx, k)
        maps.append(r.ravel().copy())
        maps.append(r.T.ravel().copy())
    return maps


def augment(a, b, u, v, side: int = SIDE):
    """The 16 images of a solved instance: (a[p], b[p]) has duals (u[p], v[p])
    for every isometry p, and (b, a) has duals (v, u) since C is symmetric."""
    out = []
    for p in grid_symmetries(side):
        out.append((a[p], b[p], u[p], v[p]))
        out.append((b[p], a[p], v[p], u[p]))
    return out


def solve_grid_batch(seeds, params: api.PdhgParameters, *, device: int = 0, warm_starts=None,
                     recover_plan=None, race_groups=None, warm_restart: str = WARM_RESTART):
    """Solve the grid instances of `seeds` in one batched launch with the
    on-the-fly squared-Euclidean cost. Returns (outputs, device seconds)."""
    pts = grid_points()
    probs = []
    for s in seeds:
        a, b = grid_pair(int(s))
        probs.append(api.OptimalTransportProblem(None, a, b))
    return api.optimize_batched(params, probs, cost="sqeuclid", points=[(pts, pts)] * len(probs), device=device,
                                warm_starts=warm_starts, return_primal=False, recover_plan=recover_plan,
                                race_groups=race_groups, warm_restart=warm_restart)


def generate(seeds, params: api.PdhgParameters, *, batch: int = 256, device: int = 0, log=print,
             starter: Optional["WarmStarter"] = None):
    """Solver-generated training pairs: for each seed its canonical duals,
    iteration count and termination reason. With `starter`, every instance is
    solved by a race of the starter's warm start against a cold start (the
    duals of whichever ends optimal first: both are solutions to the same
    tolerance), which costs about a third of the cold solves' device time."""
    seeds = list(seeds)
    U = np.zeros((len(seeds), BINS))
    V = np.zeros((len(seeds), BINS))
    its = np.zeros(len(seeds), dtype=np.int64)
    reasons = np.zeros(len(seeds), dtype=np.int64)
    total = 0.0
    for k0 in range(0, len(seeds), batch):
        chunk = seeds[k0 : k0 + batch]
        if starter is None:
            outs, sec = solve_grid_batch(chunk, params, device=device)
        else:
            pairs = [grid_pair(int(s)) for s in chunk]
            outs, sec, _ = starter.solve(np.asarray([p[0] for p in pairs]), np.asarray([p[1] for p in pairs]),
                                         params, race=True)
        total += sec
        for k, o in enumerate(outs):
            U[k0 + k], V[k0 + k] = canonical_duals(o.dual_source_solution, o.dual_target_solution)
            its[k0 + k] = o.iteration_count
            reasons[k0 + k] = int(o.termination_reason)
        if log:
            log(f"generate: {k0 + len(chunk)}/{len(seeds)} solved, {sec:.1f} s device, "
                f"mean iterations {its[k0:k0 + len(chunk)].mean():.0f}")
    return {"seeds": np.asarray(seeds), "u": U, "v": V, "iterations": its, "reasons": reasons,
            "seconds": total}


class MLP:
    """pdot_mlp: the network on one GPU (weights, moments, activations)."""

    def __init__(self, input_dim: int = 2 * BINS, hidden_dim: int = 1024, output_dim: int = 2 * BINS,
                 max_batch: int = 256, seed: int = 0, device: int = 0):
        self._lib = _abi.load()
        h = ct.c_void_p()
        rc = self._lib.pdot_mlp_create(device, input_dim, hidden_dim, output_dim, max_batch, seed, ct.byref(h))
        _abi.check(self._lib, rc, "pdot_mlp_create")
        self._h = h
        self.dims = (input_dim, hidden_dim, output_dim)
        self.max_batch = max_batch
        self.device = device
        self.num_parameters = int(self._lib.pdot_mlp_num_parameters(h))

    def close(self):
        if self._h:
            self._lib.pdot_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream_handle(self) -> int:
        return int(self._lib.pdot_mlp_stream(self._h) or 0)

    def get_parameters(self) -> np.ndarray:
        p = np.zeros(self.num_parameters, dtype=np.float32)
        _abi.check(self._lib, self._lib.pdot_mlp_get_parameters(self._h, p.ctypes.data, p.size), "get_parameters")
        return p

    def set_parameters(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.num_parameters:
            raise ValueError(f"{p.size} parameters given, {self.num_parameters} expected")
        _abi.check(self._lib, self._lib.pdot_mlp_set_parameters(self._h, p.ctypes.data, p.size), "set_parameters")

    def gradients(self) -> np.ndarray:
        g = np.zeros(self.num_parameters, dtype=np.float32)
        _abi.check(self._lib, self._lib.pdot_mlp_get_gradients(self._h, g.ctypes.data, g.size), "get_gradients")
        return g

    def set_input(self, hist_ptr: int, batch: int, shift: float = FEATURE_SHIFT, scale: float = FEATURE_SCALE):
        """hist_ptr: device FP64 [batch x input_dim] (row-major)."""
        _abi.check(self._lib, self._lib.pdot_mlp_set_input(self._h, batch, hist_ptr, shift, scale), "set_input")

    def forward(self, out_ptr: Optional[int] = None):
        _abi.check(self._lib, self._lib.pdot_mlp_forward(self._h, out_ptr), "forward")

    def backward(self, target_ptr: int) -> float:
        loss = ct.c_double(0.0)
        _abi.check(self._lib, self._lib.pdot_mlp_backward(self._h, target_ptr, ct.byref(loss)), "backward")
        return loss.value

    def adamw(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8,
              weight_decay: float = 0.0):
        _abi.check(self._lib, self._lib.pdot_mlp_adamw(self._h, lr, beta1, beta2, eps, weight_decay), "adamw")

    def train_step(self, target_ptr: int, lr: float, weight_decay: float, want_loss: bool) -> float:
        loss = ct.c_double(float("nan"))
        rc = self._lib.pdot_mlp_train_step(self._h, target_ptr, lr, weight_decay,
                                           ct.byref(loss) if want_loss else None)
        _abi.check(self._lib, rc, "train_step")
        return loss.value


@dataclass
class WarmStartModel:
    """A trained network with the target standardisation."""

    parameters: np.ndarray  # FP32 (the BF16 weights and FP32 biases widened)
    target_mean: float
    target_scale: float
    hidden_dim: int = 1024

    def save(self, path: str):
        I, H, O = 2 * BINS, self.hidden_dim, 2 * BINS
        p = self.parameters
        sizes = [H * I, H, H * H, H, O * H, O]
        parts, off = [], 0
        for s in sizes:
            parts.append(p[off : off + s])
            off += s
        w = [parts[0], parts[2], parts[4]]
        wbits = [np.ascontiguousarray(x, dtype=np.float32).view(np.uint32) for x in w]
        # the weights are stored as their BF16 bits (what the kernels use)
        np.savez(path, W1=_bf16_bits(wbits[0]), W2=_bf16_bits(wbits[1]), W3=_bf16_bits(wbits[2]), b1=parts[1],
                 b2=parts[3], b3=parts[5], target_mean=self.target_mean, target_scale=self.target_scale,
                 hidden_dim=self.hidden_dim)

    @staticmethod
    def load(path: str) -> "WarmStartModel":
        z = np.load(path)
        f = [_bf16_to_f32(z["W1"]), z["b1"], _bf16_to_f32(z["W2"]), z["b2"], _bf16_to_f32(z["W3"]), z["b3"]]
        return WarmStartModel(np.concatenate([np.asarray(x, dtype=np.float32).ravel() for x in f]),
                              float(z["target_mean"]), float(z["target_scale"]), int(z["hidden_dim"]))


MODEL_PATH = __import__("os").path.join(__import__("os").path.dirname(__file__), "models", "grid32_warmstart.npz")


class WarmStarter:
    """The packaged (or a given) trained network, ready to warm-start solves
    of 32 x 32 grid instances."""

    def __init__(self, model_path: Optional[str] = None, *, device: int = 0, max_batch: int = 512):
        self.model = WarmStartModel.load(model_path or MODEL_PATH)
        self.mlp = MLP(hidden_dim=self.model.hidden_dim, max_batch=max_batch, device=device)
        self.mlp.set_parameters(self.model.parameters)
        self.device = device

    def predict(self, sources: np.ndarray, targets: np.ndarray):
        return predict(self.mlp, self.model, np.atleast_2d(sources), np.atleast_2d(targets))

    def solve(self, sources: np.ndarray, targets: np.ndarray, params: api.PdhgParameters, *, race: bool = True,
              recover_plan=RECOVER_PLAN):
        """Solve the grid instances (rows of `sources`, `targets`) in one
        batched launch from the network's warm starts; with `race`, each next
        to a cold start of itself in one race group, keeping whichever ends
        optimal first. Returns (outputs, device seconds, warm_won flags)."""
        sources, targets = np.atleast_2d(sources), np.atleast_2d(targets)
        n = sources.shape[0]
        u, v = self.predict(sources, targets)
        pts = grid_points()
        probs = [api.OptimalTransportProblem(None, sources[k], targets[k]) for k in range(n)]
        warm = [(u[k], v[k]) for k in range(n)]
        if not race:
            outs, sec = api.optimize_batched(params, probs, cost="sqeuclid", points=[(pts, pts)] * n,
                                             device=self.device, warm_starts=warm, return_primal=False,
                                             recover_plan=recover_plan, warm_restart=WARM_RESTART)
            return outs, sec, [True] * n
        outs, sec = api.optimize_batched(params, probs + probs, cost="sqeuclid", points=[(pts, pts)] * (2 * n),
                                         device=self.device, warm_starts=warm + [None] * n, return_primal=False,
                                         recover_plan=recover_plan, race_groups=list(range(n)) * 2,
                                         warm_restart=WARM_RESTART)
        opt = api.TerminationReason.TERMINATION_REASON_OPTIMAL
        won, best = [], []
        for k in range(n):
            w, c = outs[k], outs[n + k]
            take_w = w.termination_reason == opt or c.termination_reason != opt
            best.append(w if take_w else c)
            won.append(bool(take_w))
        return best, sec, won


def _bf16_bits(u32: np.ndarray) -> np.ndarray:
    u = u32.astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return u.astype(np.uint16)


def _bf16_to_f32(b: np.ndarray) -> np.ndarray:
    return (np.asarray(b, dtype=np.uint32) << 16).view(np.float32)


def _torch():
    import torch

    return torch


def forward_rows(mlp: MLP, hist: np.ndarray) -> np.ndarray:
    """The network's outputs for the rows of hist [N x input_dim] (FP64)."""
    torch = _torch()
    dev = torch.device("cuda", mlp.device)
    n = hist.shape[0]
    out = np.zeros((n, mlp.dims[2]), dtype=np.float32)
    Y = torch.zeros((mlp.max_batch, mlp.dims[2]), dtype=torch.float32, device=dev)
    for k0 in range(0, n, mlp.max_batch):
        h = torch.from_numpy(np.ascontiguousarray(hist[k0 : k0 + mlp.max_batch], dtype=np.float64)).to(dev)
        torch.cuda.synchronize(dev)
        mlp.set_input(h.data_ptr(), h.shape[0])
        mlp.forward(Y.data_ptr())
        out[k0 : k0 + h.shape[0]] = Y[: h.shape[0]].cpu().numpy()
    return out


def train(mlp: MLP, hist: np.ndarray, targets: np.ndarray, *, epochs: int = 60, batch: int = 256,
          lr: float = 1e-3, weight_decay: float = 1e-4, seed: int = 0, validation=None, log=print):
    """Train on (hist [N x 2048] FP64, targets [N x 2048] standardised) with
    AdamW and a cosine learning-rate schedule; batches are drawn without
    replacement each epoch (the last partial batch is dropped). `validation`
    = (hist, targets) of instances kept out of training, scored after every
    epoch. Returns (training losses (epoch, step, loss), validation losses)."""
    torch = _torch()
    dev = torch.device("cuda", mlp.device)
    H = torch.from_numpy(np.ascontiguousarray(hist, dtype=np.float64)).to(dev)
    T = torch.from_numpy(np.ascontiguousarray(targets, dtype=np.float32)).to(dev)
    n = H.shape[0]
    steps_per_epoch = n // batch
    total = epochs * steps_per_epoch
    g = torch.Generator(device="cpu").manual_seed(seed)
    losses, val = [], []
    step = 0
    for ep in range(epochs):
        perm = torch.randperm(n, generator=g).to(dev)
        Hs = H.index_select(0, perm).contiguous()
        Ts = T.index_select(0, perm).contiguous()
        torch.cuda.synchronize(dev)
        acc = 0.0
        for k in range(steps_per_epoch):
            lr_k = lr * 0.5 * (1.0 + math.cos(math.pi * step / max(total, 1)))
            mlp.set_input(Hs[k * batch:(k + 1) * batch].data_ptr(), batch)
            want = (k == steps_per_epoch - 1) or (k % 16 == 0)
            loss = mlp.train_step(Ts[k * batch:(k + 1) * batch].data_ptr(), lr_k, weight_decay, want)
            if want:
                acc = loss if k == 0 else acc
                losses.append((ep, k, loss))
            step += 1
        if validation is not None:
            pred = forward_rows(mlp, validation[0])
            val.append(float(np.mean((pred.astype(np.float64) - validation[1]) ** 2)))
        if log:
            log(f"train: epoch {ep + 1}/{epochs} loss {losses[-1][2]:.5f}"
                + (f" validation {val[-1]:.5f}" if val else ""))
    return losses, val


def predict(mlp: MLP, model: WarmStartModel, a_rows: np.ndarray, b_rows: np.ndarray, symmetrize: bool = False):
    """Predicted canonical duals (u, v) for instances given row-wise. With
    `symmetrize`, the prediction is the mean over the 16 images of each
    instance under the grid cost's symmetries, each mapped back (the exact
    duals map exactly, so this only averages the network's error)."""
    if not symmetrize:
        out = forward_rows(mlp, np.concatenate([a_rows, b_rows], axis=1))
        duals = out.astype(np.float64) * model.target_scale + model.target_mean
        return duals[:, :BINS], duals[:, BINS:]
    n = a_rows.shape[0]
    U = np.zeros((n, BINS))
    V = np.zeros((n, BINS))
    maps = grid_symmetries()
    rows = []
    for p in maps:
        rows.append(np.concatenate([a_rows[:, p], b_rows[:, p]], axis=1))
        rows.append(np.concatenate([b_rows[:, p], a_rows[:, p]], axis=1))
    out = forward_rows(mlp, np.concatenate(rows, axis=0)).astype(np.float64) * model.target_scale + model.target_mean
    for k, p in enumerate(maps):
        d = out[(2 * k) * n:(2 * k + 1) * n]
        U[:, p] += d[:, :BINS]
        V[:, p] += d[:, BINS:]
        d = out[(2 * k + 1) * n:(2 * k + 2) * n]   # the exchanged image: its source duals are v
        V[:, p] += d[:, :BINS]
        U[:, p] += d[:, BINS:]
    return U / (2 * len(maps)), V / (2 * len(maps))


def dataset(data: dict, augment_symmetries: bool = True):
    """(hist [N x 2048], duals [N x 2048]) of generated data, with the 16
    images of every instance when `augment_symmetries`."""
    A, D = [], []
    C = grid_cost()
    for k, s in enumerate(data["seeds"]):
        if data["reasons"][k] != int(api.TerminationReason.TERMINATION_REASON_OPTIMAL):
            continue
        a, b = grid_pair(int(s))
        u, v = tight_duals(data["u"][k], data["v"][k], C)
        imgs = augment(a, b, u, v) if augment_symmetries else [(a, b, u, v)]
        for (aa, bb, uu, vv) in imgs:
            A.append(np.concatenate([aa, bb]))
            D.append(np.concatenate([uu, vv]))
    return np.asarray(A), np.asarray(D)


def evaluate(mlp: MLP, model: WarmStartModel, seeds, params: api.PdhgParameters, *, batch: int = 256,
             device: int = 0, cold: Optional[dict] = None, recover_plan=RECOVER_PLAN, tighten: bool = False,
             symmetrize: bool = False, race: bool = False, log=print):
    """Cold and learned-warm batched solves of the held-out `seeds`:
    iterations, device seconds, and the network's time (inference). `cold`,
    when given, holds the cold solves already made (generate()'s output for
    the same seeds, solved in chunks of the same `batch`). `tighten` replaces
    the predicted duals by their double c-transform (on the host) before the
    warm start; `symmetrize` averages the prediction over the symmetries;
    `race` solves a cold copy of every instance beside its warm start in the
    same batch, the two in one race group, and takes whichever ends optimal
    first (the warm iteration counts are then the winner's, and
    warm_work_iterations adds both copies' iterations)."""
    seeds = list(seeds)
    C = grid_cost()
    res = {"cold_iterations": [], "warm_iterations": [], "cold_seconds": 0.0, "warm_seconds": 0.0,
           "predict_seconds": 0.0, "cold_reasons": [], "warm_reasons": [], "dual_rel_error": [],
           "warm_work_iterations": [], "race_winner_warm": []}
    for k0 in range(0, len(seeds), batch):
        chunk = seeds[k0 : k0 + batch]
        ab = [grid_pair(int(s)) for s in chunk]
        t0 = time.perf_counter()
        u, v = predict(mlp, model, np.asarray([x[0] for x in ab]), np.asarray([x[1] for x in ab]),
                       symmetrize=symmetrize)
        res["predict_seconds"] += time.perf_counter() - t0
        if tighten:
            for k in range(len(chunk)):
                u[k], v[k] = tight_duals(u[k], v[k], C)
        warm = [(u[k], v[k]) for k in range(len(chunk))]
        if race:
            n = len(chunk)
            outs, sec_w = solve_grid_batch(list(chunk) + list(chunk), params, device=device,
                                           warm_starts=warm + [None] * n, recover_plan=recover_plan,
                                           race_groups=list(range(n)) * 2)
            opt = int(api.TerminationReason.TERMINATION_REASON_OPTIMAL)
            for k in range(n):
                w, c = outs[k], outs[n + k]
                win = w if (int(w.termination_reason) == opt or int(c.termination_reason) != opt) else c
                res["warm_iterations"].append(win.iteration_count)
                res["warm_reasons"].append(int(win.termination_reason))
                res["warm_work_iterations"].append(w.iteration_count + c.iteration_count)
                res["race_winner_warm"].append(win is w)
        else:
            outs_w, sec_w = solve_grid_batch(chunk, params, device=device, warm_starts=warm,
                                             recover_plan=recover_plan)
            res["warm_iterations"] += [o.iteration_count for o in outs_w]
            res["warm_work_iterations"] += [o.iteration_count for o in outs_w]
            res["warm_reasons"] += [int(o.termination_reason) for o in outs_w]
        res["warm_seconds"] += sec_w
        if cold is None:
            outs_c, sec_c = solve_grid_batch(chunk, params, device=device)
            res["cold_seconds"] += sec_c
            res["cold_iterations"] += [o.iteration_count for o in outs_c]
            res["cold_reasons"] += [int(o.termination_reason) for o in outs_c]
            cold_duals = [(o.dual_source_solution, o.dual_target_solution) for o in outs_c]
        else:
            sel = slice(k0, k0 + len(chunk))
            res["cold_iterations"] += [int(x) for x in cold["iterations"][sel]]
            res["cold_reasons"] += [int(x) for x in cold["reasons"][sel]]
            cold_duals = list(zip(np.asarray(cold["u"][sel], dtype=np.float64),
                                  np.asarray(cold["v"][sel], dtype=np.float64)))
        for k, (uc, vc) in enumerate(cold_duals):
            ref = np.concatenate(tight_duals(uc, vc, C))
            res["dual_rel_error"].append(float(np.linalg.norm(np.concatenate([u[k], v[k]]) - ref)
                                               / np.linalg.norm(ref - ref.mean())))
        if log:
            log(f"evaluate: {k0 + len(chunk)}/{len(seeds)}: warm {np.mean(res['warm_iterations']):.0f} it, "
                f"cold {np.mean(res['cold_iterations']):.0f} it")
    return res


def summarize(res: dict) -> dict:
    cold = np.asarray(res["cold_iterations"], dtype=float)
    warm = np.asarray(res["warm_iterations"], dtype=float)
    return {
        "instances": int(cold.size),
        "cold_mean_iterations": float(cold.mean()), "warm_mean_iterations": float(warm.mean()),
        "cold_median_iterations": float(np.median(cold)), "warm_median_iterations": float(np.median(warm)),
        "cold_p90_iterations": float(np.percentile(cold, 90)), "warm_p90_iterations": float(np.percentile(warm, 90)),
        "warm_better_fraction": float(np.mean(warm < cold)),
        "warm_work_mean_iterations": float(np.mean(res["warm_work_iterations"])),
        "race_warm_wins": int(sum(res["race_winner_warm"])),
        "cold_seconds": float(res["cold_seconds"]), "warm_seconds": float(res["warm_seconds"]),
        "predict_seconds": float(res["predict_seconds"]),
        "cold_optimal": int(sum(1 for r in res["cold_reasons"] if r == 1)),
        "warm_optimal": int(sum(1 for r in res["warm_reasons"] if r == 1)),
        "dual_rel_error_median": float(np.median(res["dual_rel_error"])),
    }


# ------------------------------------------------------------------ command line
# python -m pdot.learned generate --first SEED --count N --out data.npz
# python -m pdot.learned train --data a.npz [b.npz ...] --model model.npz
# python -m pdot.learned evaluate --model model.npz --first SEED --count N --out eval.json
TRAIN_SEED0 = 1_000_000   # training instances: seeds TRAIN_SEED0 + k
HELDOUT_SEED0 = 9_000_000  # held-out instances: seeds HELDOUT_SEED0 + k


def _params(tol: float = 1e-4, iteration_limit: int = 400_000):
    from .solve import default_parameters

    return default_parameters(tol, iteration_limit=iteration_limit)


def _cmd_generate(args):
    seeds = list(range(args.first, args.first + args.count))
    starter = WarmStarter(args.race_with, max_batch=args.batch) if args.race_with else None
    data = generate(seeds, _params(iteration_limit=args.iteration_limit), batch=args.batch, starter=starter)
    np.savez(args.out, seeds=data["seeds"], u=data["u"].astype(np.float32), v=data["v"].astype(np.float32),
             iterations=data["iterations"], reasons=data["reasons"], seconds=data["seconds"])
    print(f"generate: {len(seeds)} instances in {data['seconds']:.1f} s device; "
          f"optimal {int(np.sum(data['reasons'] == 1))}; mean iterations {data['iterations'].mean():.0f}")


def _load_data(paths):
    parts = [np.load(p) for p in paths]
    return {k: np.concatenate([z[k] for z in parts]) if np.ndim(parts[0][k]) else float(sum(z[k] for z in parts))
            for k in ("seeds", "u", "v", "iterations", "reasons", "seconds")}


def _cmd_train(args):
    import json

    data = _load_data(args.data)
    data["u"] = data["u"].astype(np.float64)
    data["v"] = data["v"].astype(np.float64)
    nval = int(args.val_instances)
    keep = len(data["seeds"]) - nval
    tr = {k: (v[:keep] if np.ndim(v) else v) for k, v in data.items()}
    va = {k: (v[keep:] if np.ndim(v) else v) for k, v in data.items()}
    hist, duals = dataset(tr, augment_symmetries=not args.no_augment)
    mean, scale = float(duals.mean()), float(duals.std())
    targets = ((duals - mean) / scale).astype(np.float32)
    validation = None
    if nval > 0:
        vh, vd = dataset(va, augment_symmetries=False)
        validation = (vh, (vd - mean) / scale)
    print(f"train: {hist.shape[0]} pairs from {keep} solved instances ({nval} kept for validation); "
          f"target mean {mean:.4f} scale {scale:.4f}")
    mlp = MLP(max_batch=args.batch, seed=args.seed)
    t0 = time.perf_counter()
    losses, val = train(mlp, hist, targets, epochs=args.epochs, batch=args.batch, lr=args.lr,
                        weight_decay=args.weight_decay, seed=args.seed, validation=validation)
    secs = time.perf_counter() - t0
    model = WarmStartModel(mlp.get_parameters(), mean, scale, hidden_dim=mlp.dims[1])
    model.save(args.model)
    print(f"train: {args.epochs} epochs in {secs:.1f} s; final loss {losses[-1][2]:.5f}"
          + (f", validation {val[-1]:.5f}" if val else ""))
    if args.log:
        with open(args.log, "w") as f:
            json.dump({"pairs": int(hist.shape[0]), "instances": keep, "validation_instances": nval,
                       "epochs": args.epochs, "batch": args.batch, "lr": args.lr, "weight_decay": args.weight_decay,
                       "seconds": secs, "target_mean": mean, "target_scale": scale, "losses": losses,
                       "validation": val}, f)


def _cmd_evaluate(args):
    import json

    model = WarmStartModel.load(args.model)
    mlp = MLP(hidden_dim=model.hidden_dim, max_batch=min(args.batch, 1024))
    mlp.set_parameters(model.parameters)
    seeds = list(range(args.first, args.first + args.count))
    cold = None
    if args.cold:
        cold = _load_data([args.cold])
        if [int(x) for x in cold["seeds"][: len(seeds)]] != seeds:
            raise SystemExit("the cold data does not hold these seeds")
    res = evaluate(mlp, model, seeds, _params(iteration_limit=args.iteration_limit), batch=args.batch, cold=cold,
                   recover_plan=(args.recover_eps, args.recover_rounds), tighten=args.tight,
                   symmetrize=args.symmetrize, race=args.race)
    if cold is not None:
        res["cold_seconds"] = float(cold["seconds"])
    summary = summarize(res)
    summary.update({"recover_eps": args.recover_eps, "recover_rounds": args.recover_rounds, "tight": args.tight,
                    "symmetrize": args.symmetrize, "race": args.race})
    print(json.dumps(summary, indent=1))
    if args.out:
        with open(args.out, "w") as f:
            json.dump({"summary": summary, "per_instance": res}, f)


def main(argv=None):
    import argparse

    ap = argparse.ArgumentParser(prog="python -m pdot.learned")
    sub = ap.add_subparsers(dest="cmd", required=True)
    g = sub.add_parser("generate")
    g.add_argument("--first", type=int, default=TRAIN_SEED0)
    g.add_argument("--count", type=int, default=256)
    g.add_argument("--batch", type=int, default=512)
    g.add_argument("--iteration-limit", type=int, default=400_000)
    g.add_argument("--race-with", help="a trained network: solve each instance as a race of its warm start "
                   "against a cold start")
    g.add_argument("--out", required=True)
    t = sub.add_parser("train")
    t.add_argument("--data", nargs="+", required=True)
    t.add_argument("--model", required=True)
    t.add_argument("--epochs", type=int, default=60)
    t.add_argument("--batch", type=int, default=256)
    t.add_argument("--lr", type=float, default=1e-3)
    t.add_argument("--weight-decay", type=float, default=1e-4)
    t.add_argument("--seed", type=int, default=0)
    t.add_argument("--no-augment", action="store_true")
    t.add_argument("--val-instances", type=int, default=256, help="last instances of --data kept for validation")
    t.add_argument("--log")
    e = sub.add_parser("evaluate")
    e.add_argument("--model", required=True)
    e.add_argument("--first", type=int, default=HELDOUT_SEED0)
    e.add_argument("--count", type=int, default=1024)
    e.add_argument("--batch", type=int, default=512)
    e.add_argument("--iteration-limit", type=int, default=400_000)
    e.add_argument("--cold", help="generate's output for the same seeds (solved with the same --batch)")
    e.add_argument("--recover-eps", type=float, default=RECOVER_PLAN[0])
    e.add_argument("--recover-rounds", type=int, default=RECOVER_PLAN[1])
    e.add_argument("--tight", action="store_true", help="c-transform the predicted duals first")
    e.add_argument("--symmetrize", action="store_true", help="average the prediction over the 16 symmetries")
    e.add_argument("--race", action="store_true", help="race a cold copy beside every warm start")
    e.add_argument("--out")
    args = ap.parse_args(argv)
    {"generate": _cmd_generate, "train": _cmd_train, "evaluate": _cmd_evaluate}[args.cmd](args)


if __name__ == "__main__":
    main()

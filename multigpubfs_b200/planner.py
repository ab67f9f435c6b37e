"""Learned planner: a small MLP that predicts the next BFS layer from the last
layers and the generators, trained and evaluated by libmgbfs2's own kernels
(csrc/mlp.cu); the plain worst-case planner stays the exact fallback.

Features of instance i at depth d (16, all O(1)):
    log1p |L_d|, log1p |L_{d-1}|, log1p |L_{d-2}|, log1p |L_{d-3}|,
    log1p visited, log orbit (exact group order by Schreier-Sims for distinct
    labels, else the multinomial bound), n/16, g/8, inverse-closed,
    mean and max log generator order, mean fixed-point fraction,
    mean cycle count / n, d/64, visited/orbit, log1p(g |L_d|)
Targets: log1p |L_{d+1}| - log1p |L_d| (log growth) and the duplicate ratio
1 - |L_{d+1}| / (g |L_d|).

A rollout from |L_0| = 1 gives each instance's predicted layer profile; its
peak times a margin sizes the instance's frontier in the batched sweep (a
layer that outgrows it is redone in a larger segment), and for a single run
the prediction (with |G| exact where the labels are distinct) chooses the
bitmap or the hash and sizes the table and buffers through mgbfs2_plan.
Results never depend on the prediction.  There is no counterpart in the reference, which sizes
buffers from worst-case bounds and timed pilot runs
(crates/mgbfs-runtime/src/generic_memory.rs:36-49, multigpubfs/autotune.py:276).
"""
from __future__ import annotations

import functools
import json
import math
from dataclasses import dataclass

import numpy as np

from . import native

INPUTS = 16


# ---------------------------------------------------------------------------
# Features.

def _cycles(perm):
    seen = [False] * len(perm)
    lengths = []
    for i in range(len(perm)):
        if not seen[i]:
            j, length = i, 0
            while not seen[j]:
                seen[j] = True
                j = perm[j]
                length += 1
            lengths.append(length)
    return lengths


@dataclass
class GraphStatics:
    n: int
    gens: int
    inverse_closed: bool
    log_orbit: float
    mean_log_order: float
    max_log_order: float
    fixed_fraction: float
    cycle_fraction: float

    @property
    def orbit(self):
        return math.exp(self.log_orbit)


@functools.lru_cache(maxsize=4096)
def _group_order(generators: tuple) -> int:
    return native.group_order(generators)


def group_order(generators) -> int:
    """|<generators>| (host Schreier-Sims), memoised per generator set."""
    return _group_order(tuple(tuple(int(x) for x in g) for g in generators))


def graph_statics(generators, start) -> GraphStatics:
    n = len(start)
    orders, fixed, cycles = [], [], []
    for g in generators:
        c = _cycles(g)
        order = 1
        for length in c:
            order = order * length // math.gcd(order, length)
        orders.append(math.log(order))
        fixed.append(sum(1 for length in c if length == 1) / n)
        cycles.append(len(c) / n)
    gens = {tuple(g) for g in generators}

    def inverse(g):
        inv = [0] * len(g)
        for i, x in enumerate(g):
            inv[x] = i
        return tuple(inv)
    closed = all(inverse(g) in gens for g in generators)
    counts = {}
    for v in start:
        counts[v] = counts.get(v, 0) + 1
    if len(counts) == n and n <= 20:
        # Distinct labels: the BFS settles exactly |<generators>| states.
        log_orbit = math.log(group_order(generators))
    else:
        log_orbit = math.lgamma(n + 1) - sum(math.lgamma(c + 1) for c in counts.values())
    k = len(generators)
    return GraphStatics(n, k, closed, log_orbit, sum(orders) / k, max(orders), sum(fixed) / k, sum(cycles) / k)


def features(st: GraphStatics, layers, d) -> list:
    last = [math.log1p(layers[d - k]) if d - k >= 0 else 0.0 for k in range(4)]
    visited = float(sum(layers[:d + 1]))
    return last + [math.log1p(visited), st.log_orbit, st.n / 16.0, st.gens / 8.0, float(st.inverse_closed),
                   st.mean_log_order, st.max_log_order, st.fixed_fraction, st.cycle_fraction, d / 64.0,
                   visited / st.orbit, math.log1p(st.gens * layers[d])]


def training_set(graphs, tables):
    """(X, T) from complete layer tables: one row per (instance, depth),
    including the final depth whose next layer is empty."""
    X, T = [], []
    for g, layers in zip(graphs, tables):
        st = graph_statics(g["action"]["generators"], g["start"])
        for d in range(len(layers)):
            nxt = layers[d + 1] if d + 1 < len(layers) else 0
            X.append(features(st, layers, d))
            T.append([math.log1p(nxt) - math.log1p(layers[d]), 1.0 - nxt / (st.gens * layers[d])])
    return np.asarray(X, dtype=np.float32), np.asarray(T, dtype=np.float32)


# ---------------------------------------------------------------------------
# The network, on the device.

class PlannerNet:
    def __init__(self, device: int = 0, seed: int = 0, params=None):
        import torch
        self.lib = native.require_device()
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.count = int(self.lib.mgbfs2_mlp_param_count(INPUTS))
        if params is None:
            rng = np.random.default_rng(seed)
            p = np.zeros(self.count, dtype=np.float32)
            o = 0
            for rows, cols in ((64, INPUTS), (64, 64), (2, 64)):
                p[o:o + rows * cols] = rng.normal(0.0, math.sqrt(2.0 / cols), rows * cols)
                o += rows * cols + rows
            params = p
        self.params = torch.tensor(np.asarray(params, dtype=np.float32), device=self.dev)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.grad = torch.zeros_like(self.params)
        self.step = 0
        self.x_mean = np.zeros(INPUTS, dtype=np.float32)
        self.x_scale = np.ones(INPUTS, dtype=np.float32)

    def _stream(self):
        return native.stream_handle()

    def _x(self, X):
        X = (np.asarray(X, dtype=np.float32) - self.x_mean) / self.x_scale
        return self.torch.tensor(X, device=self.dev).contiguous()

    def loss_and_grad(self, X, T, weights=(1.0, 1.0)):
        """One fused forward/backward over (X, T); returns (loss, grad) as numpy."""
        x = self._x(X)
        t = self.torch.tensor(np.asarray(T, dtype=np.float32), device=self.dev).contiguous()
        self.grad.zero_()
        loss = self.torch.zeros(1, dtype=self.torch.float32, device=self.dev)
        native.check(self.lib.mgbfs2_mlp_loss_grad(INPUTS, self.params.data_ptr(), x.data_ptr(), t.data_ptr(),
                                                   float(weights[0]), float(weights[1]), x.shape[0],
                                                   self.grad.data_ptr(), loss.data_ptr(), self._stream()),
                     "mgbfs2_mlp_loss_grad")
        return float(loss.item()), self.grad.cpu().numpy()

    def fit(self, X, T, steps=1500, lr=3e-3, weights=(1.0, 1.0), batch=4096, seed=0):
        """Adam on minibatches; normalisation statistics come from X.  Returns
        the loss history (every 50 steps)."""
        X = np.asarray(X, dtype=np.float32)
        T = np.asarray(T, dtype=np.float32)
        self.x_mean = X.mean(0)
        self.x_scale = X.std(0) + 1e-3
        x_all = self._x(X)
        t_all = self.torch.tensor(T, device=self.dev).contiguous()
        rng = np.random.default_rng(seed)
        history = []
        loss = self.torch.zeros(1, dtype=self.torch.float32, device=self.dev)
        for step in range(steps):
            if len(X) > batch:
                idx = self.torch.tensor(rng.integers(0, len(X), batch), device=self.dev)
                xb, tb = x_all[idx].contiguous(), t_all[idx].contiguous()
            else:
                xb, tb = x_all, t_all
            self.grad.zero_()
            loss.zero_()
            native.check(self.lib.mgbfs2_mlp_loss_grad(INPUTS, self.params.data_ptr(), xb.data_ptr(), tb.data_ptr(),
                                                       float(weights[0]), float(weights[1]), xb.shape[0],
                                                       self.grad.data_ptr(), loss.data_ptr(), self._stream()),
                         "mgbfs2_mlp_loss_grad")
            self.step += 1
            native.check(self.lib.mgbfs2_mlp_adam(self.count, self.params.data_ptr(), self.grad.data_ptr(),
                                                  self.m.data_ptr(), self.v.data_ptr(), lr, 0.9, 0.999, 1e-8,
                                                  self.step, self._stream()), "mgbfs2_mlp_adam")
            if step % 50 == 0 or step == steps - 1:
                history.append(float(loss.item()))
        return history

    def predict_fp32(self, X):
        x = self._x(X)
        y = self.torch.empty((x.shape[0], 2), dtype=self.torch.float32, device=self.dev)
        native.check(self.lib.mgbfs2_mlp_forward(INPUTS, self.params.data_ptr(), x.data_ptr(), x.shape[0],
                                                 y.data_ptr(), self._stream()), "mgbfs2_mlp_forward")
        return y.cpu().numpy()

    def predict(self, X):
        """bf16 inference kernel."""
        x = self._x(X)
        q = self.torch.empty(self.count, dtype=self.torch.bfloat16, device=self.dev)
        native.check(self.lib.mgbfs2_mlp_to_bf16(self.count, self.params.data_ptr(), q.data_ptr(), self._stream()),
                     "mgbfs2_mlp_to_bf16")
        y = self.torch.empty((x.shape[0], 2), dtype=self.torch.float32, device=self.dev)
        native.check(self.lib.mgbfs2_mlp_infer_bf16(INPUTS, q.data_ptr(), x.data_ptr(), x.shape[0], y.data_ptr(),
                                                    self._stream()), "mgbfs2_mlp_infer_bf16")
        return y.cpu().numpy()

    def to_json(self):
        return json.dumps({"inputs": INPUTS, "params": self.params.cpu().numpy().tolist(),
                           "x_mean": self.x_mean.tolist(), "x_scale": self.x_scale.tolist()})

    @classmethod
    def from_json(cls, text, device=0):
        d = json.loads(text)
        net = cls(device, params=np.asarray(d["params"], dtype=np.float32))
        net.x_mean = np.asarray(d["x_mean"], dtype=np.float32)
        net.x_scale = np.asarray(d["x_scale"], dtype=np.float32)
        return net


# ---------------------------------------------------------------------------
# Using the prediction.

def rollout(net: PlannerNet, graphs, max_depth=512):
    """Predicted layer profiles of all graphs, stepped together (one bf16
    inference launch per depth)."""
    stats = [graph_statics(g["action"]["generators"], g["start"]) for g in graphs]
    # The columns of `features`, built for all active instances at once.
    static = np.array([[st.log_orbit, st.n / 16.0, st.gens / 8.0, float(st.inverse_closed), st.mean_log_order,
                        st.max_log_order, st.fixed_fraction, st.cycle_fraction] for st in stats], dtype=np.float64)
    static = static.reshape(len(graphs), 8)
    gens = np.array([st.gens for st in stats], dtype=np.float64)
    orbit = np.exp(static[:, 0])
    last = np.zeros((len(graphs), 4))  # |L_d|, |L_d-1|, |L_d-2|, |L_d-3| (0 before depth 0)
    last[:, 0] = 1.0
    visited = np.ones(len(graphs))
    layers = [[1.0] for _ in graphs]
    active = np.arange(len(graphs))
    for d in range(max_depth):
        if active.size == 0:
            break
        h, v = last[active], visited[active]
        X = np.column_stack([np.log1p(h), np.log1p(v), static[active], np.full(active.size, d / 64.0),
                             v / orbit[active], np.log1p(gens[active] * h[:, 0])])
        y = net.predict(X)
        nxt = np.expm1(y[:, 0].astype(np.float64) + np.log1p(h[:, 0]))
        nxt = np.minimum(np.minimum(nxt, orbit[active] - v), gens[active] * h[:, 0])
        keep = nxt >= 0.5
        for i, size in zip(active[keep], nxt[keep]):
            layers[i].append(float(size))
        last[active[keep]] = np.column_stack([nxt[keep], h[keep, :3]])
        visited[active[keep]] += nxt[keep]
        active = active[keep]
    return layers


def batch_statics(graphs):
    """(statics, states) of many graphs in one native call
    (mgbfs2_graph_statics, host threads): statics is a (count, 8) float32
    array in the device rollout's layout, equal to `graph_statics` row by row,
    and states the settled-state count of each graph (|G| for distinct labels,
    else the multinomial bound)."""
    return native.graph_statics([(g["action"]["generators"], g["start"]) for g in graphs])


def rollout_device(net: PlannerNet, graphs, max_depth=512, statics=None):
    """(peak, total, depth) of every graph's predicted profile, from one
    launch of the device rollout kernel (mgbfs2_mlp_rollout_bf16): the same
    features and bf16 network as `rollout`, with the depth loop on the GPU, so
    predicting a whole sweep costs one launch instead of one per depth.
    `statics` is `batch_statics(graphs)[0]` when the caller has it."""
    t = net.torch
    if statics is None:
        statics = batch_statics(graphs)[0]
    m = len(statics)
    static = t.from_numpy(statics).to(net.dev).contiguous()
    gens = (static[:, 2] * 8.0).contiguous()
    mean = t.tensor(net.x_mean, dtype=t.float32, device=net.dev)
    scale = t.tensor(net.x_scale, dtype=t.float32, device=net.dev)
    q = t.empty(net.count, dtype=t.bfloat16, device=net.dev)
    native.check(net.lib.mgbfs2_mlp_to_bf16(net.count, net.params.data_ptr(), q.data_ptr(), net._stream()),
                 "mgbfs2_mlp_to_bf16")
    peak = t.empty(m, dtype=t.float64, device=net.dev)
    total = t.empty(m, dtype=t.float64, device=net.dev)
    depth = t.empty(m, dtype=t.int32, device=net.dev)
    native.check(net.lib.mgbfs2_mlp_rollout_bf16(q.data_ptr(), mean.data_ptr(), scale.data_ptr(), static.data_ptr(),
                                                 gens.data_ptr(), m, max_depth, peak.data_ptr(), total.data_ptr(),
                                                 depth.data_ptr(), net._stream()), "mgbfs2_mlp_rollout_bf16")
    return peak.cpu().numpy(), total.cpu().numpy(), depth.cpu().numpy()


def predicted_capacities(net: PlannerNet, graphs, margin=1.5, floor=4096):
    """Per-instance frontier capacity for the batched sweep (predicted peak x
    margin + floor, from the device rollout), never above the exact state count
    |G| (the sweep's instances have distinct labels), which no layer can
    exceed."""
    statics, states = batch_statics(graphs)
    peaks, _, _ = rollout_device(net, graphs, statics=statics)
    return [int(min(int(s), peak * margin + floor)) for s, peak in zip(states, peaks)]


def calibrate_margin(net: PlannerNet, graphs, tables, quantile=0.97, slack=1.1) -> float:
    """Capacity margin from complete layer tables the network was not fitted
    on: the `quantile` of (true peak / predicted peak), at least 1, times
    `slack`.  A larger margin trades memory for fewer exact reruns."""
    peaks, _, _ = rollout_device(net, graphs)
    ratios = sorted(max(t) / max(1.0, p) for t, p in zip(tables, peaks))
    q = ratios[min(len(ratios) - 1, int(quantile * (len(ratios) - 1) + 0.5))]
    return max(1.0, q) * slack


_DEFAULT = {}


def default_planner(device: int = 0):
    """(network, margin) trained by the library's kernels on layer tables the
    batched engine computes for the 512-instance sweep (4/5 fitted, 1/5
    calibrating the margin); made once per process and device, about two
    seconds on a B200."""
    if device not in _DEFAULT:
        from . import workloads
        from .batch import BatchSweep
        graphs = workloads.sweep(512)
        with BatchSweep(graphs, device) as sweep:
            sweep.run()
            tables = sweep.layer_tables()
        fit = [i for i in range(len(graphs)) if i % 5]
        cal = [i for i in range(len(graphs)) if i % 5 == 0]
        net = PlannerNet(device, seed=0)
        net.fit(*training_set([graphs[i] for i in fit], [tables[i] for i in fit]), steps=1500, lr=3e-3)
        margin = calibrate_margin(net, [graphs[i] for i in cal], [tables[i] for i in cal])
        _DEFAULT[device] = (net, margin)
    return _DEFAULT[device]


def predict_graph(graph: dict, net: PlannerNet | None = None, margin: float | None = None, device: int = 0) -> dict:
    """The learned planner's prediction for one permutation graph, as the
    keywords of NativeGraph.plan (mgbfs2_plan with MGBFS2_PLANNER_LEARNED):
    the states the BFS settles -- exactly |<generators>| (host Schreier-Sims)
    when the start's labels are distinct, else the network's predicted total
    times the margin, capped by the multinomial bound -- and the predicted
    peak layer times the margin.  The C planner chooses the bitmap or the hash
    and sizes the hash table and frontier buffers from them; results never
    depend on them.  Graphs outside the planner's features (matrix actions,
    more than 20 points) raise ValueError("LEARNED_PLANNER_UNSUPPORTED")."""
    a = graph["action"]
    if a["kind"] != "permutation" or len(graph["start"]) > 20:
        raise ValueError("LEARNED_PLANNER_UNSUPPORTED")
    if net is None:
        net, default_margin = default_planner(device)
        margin = default_margin if margin is None else margin
    margin = 1.5 if margin is None else margin
    statics, states = batch_statics([graph])
    peak, total, _ = rollout_device(net, [graph], statics=statics)
    bound = int(states[0])
    exact = len(set(graph["start"])) == len(graph["start"])
    predicted = bound if exact else int(min(bound, max(1.0, float(total[0]) * margin)))
    return {"planner": "learned", "predicted_states": max(1, predicted),
            "predicted_peak": int(max(1, min(predicted, float(peak[0]) * margin + 1024))),
            "exact_states": exact}


def choose_path(graph: dict, net: PlannerNet | None = None, margin: float | None = None, device: int = 0) -> dict:
    """The plan keywords of the learned planner for a single run: the
    prediction of `predict_graph`, with which mgbfs2_plan takes the exact
    bitmap when the predicted states fill at least 1/128 of the rank domain
    (and the bitmap fits), else the hash (three layer banks when
    inverse-closed), and sizes the table and buffers."""
    kw = predict_graph(graph, net, margin, device)
    kw.pop("exact_states")
    return kw

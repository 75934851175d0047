"""Continuous-batching server for encrypted Spike-LSTM requests.

A request is one encrypted sequence (T_i timesteps of RLWE inputs).  The
server keeps a pool of slots on the device; each slot holds a request's
encrypted inputs and its per-layer (H, C) state across timesteps.  Every
tick:
  1. admits waiting requests into free slots (their inputs are copied to
     the device once; admission stops when the slot pool, sized from free
     HBM, is full),
  2. runs ONE batched step of every layer over all live requests: layer l
     takes each request's timestep pos - l (a wavefront), its input being
     layer l - 1's state from the previous tick, and the bootstraps of all
     layers and requests share one launch per phase,
  3. retires requests whose sequence ended: one batched head over them and
     a device -> host copy of their logits.
Requests therefore join and leave between ticks while others are on the
GPU, and a request's result does not depend on what it was batched with
(every operator acts on each ciphertext independently and exactly).

The model is anything with the `StepModel` interface; `DeviceStepModel`
adapts the engine's layers (spike_model.DeviceModel).
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field

import numpy as np
import torch


@dataclass
class Request:
    rid: int
    xs: torch.Tensor                 # (T, 2, N) int32, host (pinned) or device
    arrival: float = 0.0             # seconds on the server clock
    done: float = None
    logits: tuple = None             # (a (1, N), b (1,)) int32 host tensors
    slot: int = None
    pos: int = 0

    @property
    def length(self) -> int:
        return self.xs.shape[0]


class StepModel:
    """What the server drives.  States are per-layer tensors with a leading
    slot axis."""
    N: int
    n_layers: int

    def state_shape(self):                 # per layer, per slot: e.g. (2, 2, N) for (H, C)
        raise NotImplementedError

    def layer_input(self, layer, prev_states):
        """Input of `layer` (> 0) from the states of layer - 1."""
        raise NotImplementedError

    def step_layers(self, xs, states):
        """One timestep of every layer on its own slots: xs[l] (S_l, 2, N),
        states[l] (S_l, ...) with any S_l (0 allowed) -> new states[l]."""
        raise NotImplementedError

    def head(self, states):                # last layer's states of finished slots -> (a (S, 1, N), b (S, 1))
        raise NotImplementedError


class _TickGraph:
    """step_merged of one combination of per-layer request counts, captured
    in a CUDA graph on fixed input buffers: a tick then costs a few copies
    and one graph launch instead of its several dozen kernel launches and
    their host work.  The outputs are the graph's, valid until its next
    replay."""

    def __init__(self, model, xs, states):
        self.xs = [x.clone() for x in xs]
        self.states = [st.clone() for st in states]
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.out = model._step_layers(self.xs, self.states)

    def run(self, xs, states):
        for dst, src in zip(self.xs, xs):
            dst.copy_(src)
        for dst, src in zip(self.states, states):
            dst.copy_(src)
        self.graph.replay()
        return self.out


class DeviceStepModel(StepModel):
    """The engine's encrypted layers and head (spike_model.DeviceModel); the
    layers' bootstraps of one tick run as one launch per phase.  With
    graphs (the default on the 2^32 torus) a tick whose per-layer request
    counts were seen before replays a CUDA graph of the step: the first
    tick of a combination runs directly (its launches fill the engine's
    per-shape caches), the second captures the graph, later ones replay it.
    Results are identical either way (the same kernels on the same data).
    The 2^64 torus runs direct launches unless graphs=True is asked for.
    Only ticks of at most graph_max requests per layer are graphed (each
    graph keeps its own working memory; larger ticks have launch work to
    spare anyway), so the cache stays at (graph_max + 1)^layers graphs."""

    def __init__(self, dm, graphs=None, graph_max: int = 8):
        self.dm = dm
        self.N = dm.keys.galois.N
        self.n_layers = len(dm.layers)
        self.dtype = torch.int64 if dm.keys.torus_bits == 64 else torch.int32
        if graphs is None:
            graphs = dm.keys.torus_bits == 32
        self.graphs = {} if graphs else None
        self.graph_max = graph_max
        self._seen = set()

    def state_shape(self):
        return (2, 2, self.N)

    def layer_input(self, layer, prev_states):
        from .lstm import rlwe_rotate_add
        return rlwe_rotate_add(prev_states[:, 0].contiguous(), -self.dm.layers[layer - 1].input_dim)

    def step_layers(self, xs, states):
        if self.graphs is None:
            return self._step_layers(xs, states)
        key = tuple(int(x.shape[0]) for x in xs)
        if max(key) > self.graph_max:
            return self._step_layers(xs, states)
        g = self.graphs.get(key)
        if g is None:
            if key not in self._seen:
                self._seen.add(key)
                return self._step_layers(xs, states)
            g = self.graphs[key] = _TickGraph(self, xs, states)
        return g.run(xs, states)

    def warm_graphs(self, max_count: int):
        """Run and capture ahead of time the tick of every combination of
        per-layer request counts up to max_count (on zero ciphertexts), so a
        serving run meets no capture on its latency path for them."""
        import itertools
        if self.graphs is None:
            return
        dev = self.dm.layers[0].device
        for key in itertools.product(range(min(max_count, self.graph_max) + 1), repeat=self.n_layers):
            if not any(key) or key in self.graphs:
                continue
            xs = [torch.zeros((c, 2, self.N), dtype=self.dtype, device=dev) for c in key]
            states = [torch.zeros((c,) + tuple(self.state_shape()), dtype=self.dtype, device=dev) for c in key]
            self._seen.add(key)
            self._step_layers(xs, states)
            self.graphs[key] = _TickGraph(self, xs, states)
        torch.cuda.synchronize()

    def _step_layers(self, xs, states):
        from .lstm import step_merged
        items, which = [], []
        for li, (x, st) in enumerate(zip(xs, states)):
            if x.shape[0]:
                items.append((self.dm.layers[li], x, st[:, 0].contiguous(), st[:, 1].contiguous()))
                which.append(li)
        out = [None] * len(xs)
        for li, (H, C) in zip(which, step_merged(items)):
            out[li] = torch.stack([H, C], dim=1)
        return out

    def head(self, states):
        return self.dm.head(states[-1][:, 0].contiguous())
def slots_for_memory(model: StepModel, t_max: int, free_bytes: int, reserve_bytes: int, cap: int) -> int:
    """Slots the pool can hold: inputs (t_max, 2, N) plus every layer's
    state per slot, within free device memory minus a reserve for the
    working buffers of one tick."""
    word = 8 if getattr(model, "dtype", torch.int32) == torch.int64 else 4
    per_slot = (t_max * 2 * model.N + model.n_layers * int(np.prod(model.state_shape()))) * word
    return int(max(0, min(cap, (free_bytes - reserve_bytes) // max(per_slot, 1))))


class SpikeLstmServer:
    def __init__(self, model: StepModel, max_slots: int, t_max: int, device=None):
        self.model = model
        self.t_max = t_max
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.max_slots = max_slots
        N = model.N
        dt = getattr(model, "dtype", torch.int32)        # torus words: int32 (q = 2^32) or int64 (q = 2^64)
        self.inputs = torch.zeros((max_slots, t_max, 2, N), dtype=dt, device=self.device)
        self.states = [torch.zeros((max_slots,) + tuple(model.state_shape()), dtype=dt, device=self.device)
                       for _ in range(model.n_layers)]
        self.free = list(range(max_slots))
        self.live = {}                     # slot -> Request
        self.waiting = collections.deque()
        self.finished = []
        self.ticks = 0
        self.batch_sizes = []

    def submit(self, req: Request):
        if req.length < 1 or req.length > self.t_max:
            raise ValueError(f"request {req.rid}: length {req.length} outside [1, {self.t_max}]")
        self.waiting.append(req)

    def _admit(self):
        while self.waiting and self.free:
            req = self.waiting.popleft()
            slot = self.free.pop(0)
            self.inputs[slot, : req.length].copy_(req.xs, non_blocking=True)
            for st in self.states:
                st[slot].zero_()
            req.slot, req.pos = slot, 0
            self.live[slot] = req

    def tick(self, now=None):
        """One batched tick: layer l of every live request takes that
        request's timestep pos - l (a wavefront, so the layers' bootstraps
        share launches); returns the requests retired in this tick."""
        self._admit()
        if not self.live:
            return []
        L = self.model.n_layers
        slots = sorted(self.live)
        xs, idxs = [], []
        for l in range(L):
            sel = [s for s in slots if 0 <= self.live[s].pos - l < self.live[s].length]
            idx = torch.tensor(sel, dtype=torch.long, device=self.device)
            idxs.append(idx)
            if not sel:
                xs.append(torch.zeros((0, 2, self.model.N), dtype=self.inputs.dtype, device=self.device))
            elif l == 0:
                pos = torch.tensor([self.live[s].pos for s in sel], dtype=torch.long, device=self.device)
                xs.append(self.inputs[idx, pos].contiguous())
            else:
                xs.append(self.model.layer_input(l, self.states[l - 1].index_select(0, idx)))
        states = [st.index_select(0, idx) for st, idx in zip(self.states, idxs)]
        new = self.model.step_layers(xs, states)
        for st, idx, nw in zip(self.states, idxs, new):
            if nw is not None and idx.numel():
                st.index_copy_(0, idx, nw)
        self.ticks += 1
        self.batch_sizes.append(len(slots))
        done = []
        for s in slots:
            self.live[s].pos += 1
            if self.live[s].pos == self.live[s].length + L - 1:
                done.append(s)
        out = []
        if done:
            didx = torch.tensor(done, dtype=torch.long, device=self.device)
            a, b = self.model.head([st.index_select(0, didx) for st in self.states])
            a_h, b_h = a.cpu(), b.cpu()
            t_done = time.perf_counter() if now is None else now()
            for i, s in enumerate(done):
                req = self.live.pop(s)
                req.logits = (a_h[i].clone(), b_h[i].clone())
                req.done = t_done
                req.slot = None
                self.free.append(s)
                out.append(req)
            self.free.sort()
            self.finished.extend(out)
        return out

    def idle(self) -> bool:
        return not self.live and not self.waiting


def run_arrivals(server: SpikeLstmServer, requests, clock=time.perf_counter, sleep=time.sleep):
    """Feed `requests` (sorted by .arrival, seconds from start) in real time
    and tick until all are done.  Sets every request's .arrival to the
    server clock; returns the finished requests."""
    t0 = clock()
    pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
    offsets = {r.rid: r.arrival for r in pending}
    while pending or not server.idle():
        now = clock() - t0
        while pending and pending[0].arrival <= now:
            r = pending.popleft()
            r.arrival = t0 + offsets[r.rid]
            server.submit(r)
        if server.idle():
            if pending:
                sleep(max(0.0, min(0.01, pending[0].arrival - (clock() - t0))))
            continue
        server.tick(now=clock)
    return server.finished


def latency_summary(finished):
    lat = np.array([r.done - r.arrival for r in finished])
    if lat.size == 0:
        return {"p50_s": None, "p99_s": None, "mean_s": None, "count": 0}
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "count": int(lat.size)}

"""Continuous-batching server for encrypted Spike-LSTM requests.

A request is one encrypted sequence (T_i timesteps of RLWE inputs).  The
server keeps a pool of slots on the device; each slot holds a request's
encrypted inputs and its per-layer (H, C) state across timesteps.  Every
tick:
  1. admits waiting requests into free slots (their inputs are copied to
     the device once; admission stops when the slot pool, sized from free
     HBM, is full),
  2. gathers the current timestep of every live request and runs ONE
     batched step of every layer over all of them (one bootstrap launch per
     stage for the whole mix),
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
    """What the server drives.  States are lists of per-layer tensors with a
    leading slot axis."""
    N: int
    n_layers: int

    def state_shape(self):                 # per layer, per slot: e.g. (2, 2, N) for (H, C)
        raise NotImplementedError

    def step(self, x, states):             # x (S, 2, N), states [ (S, ...) ] -> new states
        raise NotImplementedError

    def head(self, states):                # states of finished slots -> (a (S, 1, N), b (S, 1))
        raise NotImplementedError


class DeviceStepModel(StepModel):
    """The engine's encrypted layers and head (spike_model.DeviceModel)."""

    def __init__(self, dm):
        self.dm = dm
        self.N = dm.keys.galois.N
        self.n_layers = len(dm.layers)

    def state_shape(self):
        return (2, 2, self.N)

    def step(self, x, states):
        from .lstm import rlwe_rotate_add
        out = []
        for layer, st in zip(self.dm.layers, states):
            H, C = layer.step(x, st[:, 0].contiguous(), st[:, 1].contiguous())
            out.append(torch.stack([H, C], dim=1))
            x = rlwe_rotate_add(H, -layer.input_dim)
        return out

    def head(self, states):
        return self.dm.head(states[-1][:, 0].contiguous())


def slots_for_memory(model: StepModel, t_max: int, free_bytes: int, reserve_bytes: int, cap: int) -> int:
    """Slots the pool can hold: inputs (t_max, 2, N) plus every layer's
    state per slot, within free device memory minus a reserve for the
    working buffers of one tick."""
    per_slot = t_max * 2 * model.N * 4 + model.n_layers * int(np.prod(model.state_shape())) * 4
    return int(max(0, min(cap, (free_bytes - reserve_bytes) // max(per_slot, 1))))


class SpikeLstmServer:
    def __init__(self, model: StepModel, max_slots: int, t_max: int, device=None):
        self.model = model
        self.t_max = t_max
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.max_slots = max_slots
        N = model.N
        self.inputs = torch.zeros((max_slots, t_max, 2, N), dtype=torch.int32, device=self.device)
        self.states = [torch.zeros((max_slots,) + tuple(model.state_shape()), dtype=torch.int32, device=self.device)
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
        """One batched timestep of every live request; returns the requests
        retired in this tick."""
        self._admit()
        if not self.live:
            return []
        slots = sorted(self.live)
        idx = torch.tensor(slots, dtype=torch.long, device=self.device)
        pos = torch.tensor([self.live[s].pos for s in slots], dtype=torch.long, device=self.device)
        x = self.inputs[idx, pos].contiguous()
        states = [st.index_select(0, idx) for st in self.states]
        new = self.model.step(x, states)
        for st, nw in zip(self.states, new):
            st.index_copy_(0, idx, nw)
        self.ticks += 1
        self.batch_sizes.append(len(slots))
        done = []
        for s in slots:
            self.live[s].pos += 1
            if self.live[s].pos == self.live[s].length:
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

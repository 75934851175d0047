"""Scheduling of the continuous-batching server, on CPU with a stand-in
model: admission into free slots, one batched step per tick over every live
request, retirement, slot reuse, and results independent of the mix."""
import numpy as np
import pytest
import torch

from tfhe_b200.serving import Request, SpikeLstmServer, StepModel, latency_summary, run_arrivals, slots_for_memory


class SumModel(StepModel):
    """H += x (wrapping int32), C counts steps; head returns H's mask row and
    C's body word."""

    def __init__(self, N=8, layers=2):
        self.N, self.n_layers = N, layers
        self.steps_seen = []

    def state_shape(self):
        return (2, 2, self.N)

    def layer_input(self, layer, prev_states):
        return prev_states[:, 0]

    def step_layers(self, xs, states):
        self.steps_seen.append(max(x.shape[0] for x in xs))
        out = []
        for x, st in zip(xs, states):
            H = st[:, 0] + x
            C = st[:, 1] + 1
            out.append(torch.stack([H, C], dim=1))
        return out

    def head(self, states):
        st = states[-1]
        return st[:, 0, 0:1].clone(), st[:, 1, 1, 0:1].clone()


def req(rid, T, N=8, seed=0):
    g = torch.Generator().manual_seed(seed + rid)
    return Request(rid, torch.randint(-1000, 1000, (T, 2, N), generator=g, dtype=torch.int32))


def expected(r, layers=2):
    x = r.xs.to(torch.int64)
    H = [torch.zeros((2, r.xs.shape[-1]), dtype=torch.int64) for _ in range(layers)]
    for t in range(r.length):
        xt = x[t]
        for li in range(layers):
            H[li] = H[li] + xt
            xt = H[li]
    return H[-1][0].to(torch.int32), r.length


def test_every_request_gets_its_own_result_in_any_mix():
    model = SumModel()
    srv = SpikeLstmServer(model, max_slots=3, t_max=10, device=torch.device("cpu"))
    reqs = [req(i, T) for i, T in enumerate([3, 7, 1, 5, 10, 2, 4])]
    for r in reqs:
        srv.submit(r)
    while not srv.idle():
        srv.tick()
    assert sorted(r.rid for r in srv.finished) == list(range(len(reqs)))
    for r in reqs:
        want_h, want_c = expected(r)
        assert torch.equal(r.logits[0][0], want_h)
        assert int(r.logits[1][0]) == want_c
    assert max(model.steps_seen) <= 3                       # never more live requests than slots


def test_slots_are_reused_and_admission_waits():
    model = SumModel(layers=1)
    srv = SpikeLstmServer(model, max_slots=2, t_max=8, device=torch.device("cpu"))
    a, b, c = req(0, 2), req(1, 5), req(2, 3)
    for r in (a, b, c):
        srv.submit(r)
    srv.tick()
    assert len(srv.live) == 2 and len(srv.waiting) == 1
    srv.tick()                                               # a (1 layer) retires after its 2nd step
    assert a.done is not None and a.slot is None
    srv.tick()                                               # c admitted into a's slot
    assert c.slot == 0 and len(srv.live) == 2
    while not srv.idle():
        srv.tick()
    assert srv.batch_sizes[:3] == [2, 2, 2]


def test_lengths_outside_the_pool_are_refused():
    srv = SpikeLstmServer(SumModel(), max_slots=1, t_max=4, device=torch.device("cpu"))
    with pytest.raises(ValueError):
        srv.submit(req(0, 5))


def test_slot_count_follows_free_memory():
    m = SumModel(N=1024, layers=2)
    per = 64 * 2 * 1024 * 4 + 2 * 2 * 2 * 1024 * 4
    assert slots_for_memory(m, 64, 100 * per + 10, 10, 1000) == 100
    assert slots_for_memory(m, 64, 100 * per, 0, 7) == 7
    assert slots_for_memory(m, 64, 10, 100, 7) == 0


def test_real_time_arrivals_and_latency():
    model = SumModel(layers=1)
    srv = SpikeLstmServer(model, max_slots=4, t_max=6, device=torch.device("cpu"))
    reqs = [req(i, 1 + i % 5) for i in range(6)]
    for i, r in enumerate(reqs):
        r.arrival = 0.002 * i
    done = run_arrivals(srv, reqs)
    assert len(done) == 6
    s = latency_summary(done)
    assert s["count"] == 6 and 0 <= s["p50_s"] <= s["p99_s"]
    for r in reqs:
        assert torch.equal(r.logits[0][0], expected(r, 1)[0])


def test_wavefront_takes_length_plus_depth_minus_one_ticks():
    model = SumModel(layers=3)
    srv = SpikeLstmServer(model, max_slots=2, t_max=8, device=torch.device("cpu"))
    r = req(0, 5)
    srv.submit(r)
    ticks = 0
    while not srv.idle():
        srv.tick()
        ticks += 1
    assert ticks == 5 + 3 - 1
    assert torch.equal(r.logits[0][0], expected(r, 3)[0])

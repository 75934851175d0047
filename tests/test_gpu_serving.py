"""The server on the GPU with a small encrypted model: every request's
encrypted logits are bit-identical whether it runs alone, in a mix of
requests of other lengths, or straight through the layers and head; the
ticks replayed from CUDA graphs give the same results as direct launches."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_results_alone_equal_results_in_the_mix():
    from tfhe_b200 import spike_model as SM
    from tfhe_b200.params import TINY_C3
    from tfhe_b200.serving import DeviceStepModel, Request, SpikeLstmServer
    cfg = SM.SpikeModelConfig(vocab=64, emb_dim=4, hidden=8, layers=2, n_lut=2, pbs=TINY_C3)
    model = SM.build_model(cfg, 3)
    dm = SM.to_device(model)
    rng = np.random.default_rng(4)
    lengths = [3, 1, 4, 2, 3]
    reqs = []
    for i, T in enumerate(lengths):
        tok = SM.sample_tokens(rng, 1, T, cfg.vocab, cfg.zipf)
        xs = torch.from_numpy(SM.encrypt_tokens(model, tok, rng).view(np.int32))[:, 0].contiguous()
        reqs.append(xs)
    sm = DeviceStepModel(dm)

    def serve(indices, slots):
        srv = SpikeLstmServer(sm, max_slots=slots, t_max=4)
        rs = [Request(i, reqs[i]) for i in indices]
        for r in rs:
            srv.submit(r)
        while not srv.idle():
            srv.tick()
        return {r.rid: r.logits for r in rs}

    mixed = serve(range(len(reqs)), 3)
    for i in range(len(reqs)):
        alone = serve([i], 1)[i]
        assert torch.equal(alone[0], mixed[i][0]) and torch.equal(alone[1], mixed[i][1]), i
        H, _ = SM.run_layers(dm, reqs[i].cuda()[:, None])
        a, b = dm.head(H)
        assert torch.equal(a[0].cpu(), mixed[i][0]) and torch.equal(b[0].cpu(), mixed[i][1]), i
    # repeated request-count combinations were replayed from captured graphs
    assert len(sm.graphs) > 0
    # graphs captured ahead of time give the same logits as well
    sm2 = DeviceStepModel(dm)
    sm2.warm_graphs(2)
    assert (1, 0) in sm2.graphs and (2, 2) in sm2.graphs
    sm = sm2
    again = serve(range(len(reqs)), 3)
    for i in range(len(reqs)):
        assert torch.equal(again[i][0], mixed[i][0]) and torch.equal(again[i][1], mixed[i][1]), i

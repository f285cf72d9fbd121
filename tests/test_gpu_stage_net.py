"""The staged early stop's acceptance network (openems_b200/stage_net.py) on
the tensor-core kernels: causal dilated im2col against the CPU restatement,
forward output and every gradient against the float64 oracle, training
reduces the loss, and the committed trained network against the residual
check alone on held-out patches generated by the batched engine."""
import numpy as np
import pytest
import torch

from openems_b200 import _native as N
from openems_b200 import stage_net as SN

pytestmark = pytest.mark.gpu


def _p(t):
    return t.data_ptr()


def test_causal_im2col_col2im_match_oracle():
    from oracle.tailnet_ref import col2im_causal, im2col_causal, round_bf16
    g = torch.Generator(device="cpu").manual_seed(0)
    B, T, C, ks, dil = 3, 37, 8, 5, 4
    x = torch.randn(B, T, C, generator=g)
    cols = torch.empty(B * T, ks * C, dtype=torch.bfloat16, device="cuda")
    N.check(N.lib().oems_pk_im2col_causal(_p(x.cuda()), _p(cols), B, T, C, ks, dil, ks * C, None))
    want = round_bf16(im2col_causal(x.numpy().astype(np.float64), ks, dil))
    assert np.array_equal(cols.float().cpu().numpy().astype(np.float64), want)
    d = torch.randn(B * T, ks * C, generator=g)
    dx = torch.empty(B, T, C, device="cuda")
    N.check(N.lib().oems_pk_col2im_causal(_p(d.cuda()), ks * C, _p(dx), B, T, C, ks, dil, None))
    ref = col2im_causal(d.numpy().astype(np.float64), B, T, C, ks, dil)
    assert np.allclose(dx.cpu().numpy(), ref, rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("rounded,fwd_tol,grad_tol", [(True, 1e-4, 1e-2), (False, 5e-2, 0.2)])
def test_stage_net_matches_cpu_oracle(rounded, fwd_tol, grad_tol):
    """With bf16 rounding of the GEMM operands in the oracle the kernels
    agree to f32 accumulation order; without, within the bf16 error."""
    from oracle.tailnet_ref import StageNetRef
    net = SN.StageNet(SN.StageNetConfig(channels=32, hidden=64))
    g = torch.Generator(device="cpu").manual_seed(1)
    x = torch.zeros(8, SN.T_WIN, SN.C_IN)
    x[:, :, :2] = torch.randn(8, SN.T_WIN, 2, generator=g)
    s = torch.randn(8, SN.N_SCALAR, generator=g)
    out = net.forward(x.cuda(), s.cuda())
    ref = StageNetRef.from_net(net)
    ro = ref.forward(x.numpy(), s.numpy(), bf16=rounded)
    rel = np.abs(out.detach().cpu().numpy() - ro).max() / np.abs(ro).max()
    assert rel < fwd_tol, rel
    G = torch.randn(8, 8, generator=g)
    net.backward(G.cuda().contiguous())
    grads = ref.backward(G.numpy().astype(np.float64))
    mine = [(l.gw, l.gb) for l in net.dense_layers()]
    for (gw, gb), (rw, rb) in zip(mine, grads):
        for m, r in ((gw, rw), (gb, rb)):
            m = m.cpu().numpy()
            rel = np.linalg.norm(m - r) / max(np.linalg.norm(r), 1e-30)
            assert rel < grad_tol, rel


def test_stage_net_training_reduces_loss():
    net_cfg = SN.StageNetConfig(channels=32, hidden=64, batch=64, epochs=1, lr=3e-3)
    net = SN.StageNet(net_cfg)
    g = torch.Generator(device="cpu").manual_seed(2)
    x = torch.zeros(64, SN.T_WIN, SN.C_IN)
    x[:, :, :2] = torch.randn(64, SN.T_WIN, 2, generator=g)
    s = torch.randn(64, SN.N_SCALAR, generator=g)
    # a learnable target: a function of the scalars and the last samples
    y = (0.5 * s[:, 0] - 0.3 * s[:, 2] + 0.2 * x[:, -1, 0]).cuda()
    xs, ss = x.cuda(), s.cuda()
    losses = [SN.train_step(net, xs, ss, y.contiguous()) for _ in range(150)]
    N.check(N.lib().oems_tc_check(None))
    assert losses[-1] < 0.2 * losses[0], (losses[0], losses[-1])


def test_committed_network_beats_residual_check_on_held_out_patches():
    """Held-out small patch antennas (a seed no training run used), recorded
    with the batched engine through every stage of the dense plan: at equal
    violation budgets (no instance, and 1% and 2% of them, above 0.5 dB) the
    committed network's first-accept rule stops the sweep earlier than the
    residual check alone, and its deployed threshold keeps the worst
    accepted error near the limit."""
    import time
    from openems_b200 import early_stop as ES
    net = SN.load_default()
    assert net is not None, "no committed network"
    plan = ES.StagePlan.dense()
    rec = SN.records("small", 240, 77, plan, 16, None, time.perf_counter())
    x, s, e, sg, it = SN.rows(rec)
    stages, sf = list(plan.stages), rec["steps_full"]
    score_net = net.predict(x, s)
    score_chk = np.log10(rec["check_db"][it, sg] + SN.LOG_FLOOR)
    budgets = (0, 0.01, 0.02)
    tn = SN.tradeoff(score_net, e, sg, it, stages, sf, budgets)
    tc = SN.tradeoff(score_chk, e, sg, it, stages, sf, budgets)
    print("network", [round(r["step_ratio"], 3) for r in tn], "residual check",
          [round(r["step_ratio"], 3) for r in tc])
    assert tn[0]["step_ratio"] > tc[0]["step_ratio"]
    assert sum(r["step_ratio"] for r in tn) > sum(r["step_ratio"] for r in tc)
    dep = SN.evaluate(score_net, net.threshold, e, sg, it, stages, sf)
    print("deployed", dep)
    assert dep["step_ratio"] > 1.0 and dep["over_limit"] <= 0.02 * len(sf)

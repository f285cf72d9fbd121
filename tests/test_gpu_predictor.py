"""Tensor-core BF16 GEMM (tcgen05) and the network kernels against plain
PyTorch fp32/fp64 references of the same ops and the CPU restatement of the
network (oracle/tailnet_ref.py); training on the kernels against truncation
on a synthetic ringdown family."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from openems_b200 import _native as N  # noqa: E402


def gemm(a, b, bias=None, beta=0.0, c=None):
    M, K = a.shape
    n = b.shape[0]
    if c is None:
        c = torch.zeros(M, n, device="cuda", dtype=torch.float32)
    N.check(N.lib().oems_tc_gemm_bf16(a.data_ptr(), a.stride(0), b.data_ptr(), b.stride(0), c.data_ptr(),
                                      c.stride(0), M, n, K, float(beta),
                                      bias.data_ptr() if bias is not None else None, None))
    N.check(N.lib().oems_tc_check(None))
    return c


@pytest.mark.parametrize("M,n,K", [(128, 64, 64), (128, 128, 64), (256, 192, 128), (300, 200, 136),
                                   (1000, 70, 520), (5, 3, 8), (4096, 256, 1024)])
def test_gemm_matches_reference(M, n, K):
    g = torch.Generator(device="cpu").manual_seed(M * 7 + n * 3 + K)
    a = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    b = torch.randn(n, K, generator=g).to(torch.bfloat16).cuda()
    c = gemm(a, b)
    ref = (a.double() @ b.double().T).float()
    err = (c - ref).abs().max().item() / max(ref.abs().max().item(), 1e-30)
    assert err < 1e-5, err


def test_gemm_bias_beta_and_pitch():
    g = torch.Generator(device="cpu").manual_seed(3)
    a_full = torch.randn(200, 96, generator=g).to(torch.bfloat16).cuda()
    a = a_full[:, :72]                       # pitch 96, K 72
    b = torch.randn(130, 72, generator=g).to(torch.bfloat16).cuda()
    bias = torch.randn(130, generator=g).cuda()
    c0 = torch.randn(200, 140, generator=g).cuda()
    c = c0.clone()
    c_view = c[:, :130]
    gemm(a, b, bias=bias, beta=0.5, c=c_view)
    ref = (a.double() @ b.double().T).float() + bias + 0.5 * c0[:, :130]
    assert (c_view - ref).abs().max().item() < 1e-4 * ref.abs().max().item()
    assert torch.equal(c[:, 130:], c0[:, 130:])  # columns beyond N untouched


def test_bounded_wait_runs_out_and_the_context_stays_usable():
    """A wait on an mbarrier nothing arrives at gives up after its limit
    (about a second), the host reads OEMS_ERR_TIMEOUT, and a GEMM on the same
    stream afterwards is correct."""
    import time
    t0 = time.perf_counter()
    N.check(N.lib().oems_tc_wait_probe(None))
    with pytest.raises(N.DeviceTimeoutError):
        N.check(N.lib().oems_tc_check(None))
    assert time.perf_counter() - t0 < 30.0
    N.check(N.lib().oems_tc_check(None))  # the error word was cleared
    g = torch.Generator(device="cpu").manual_seed(9)
    a = torch.randn(256, 64, generator=g).to(torch.bfloat16).cuda()
    b = torch.randn(128, 64, generator=g).to(torch.bfloat16).cuda()
    c = gemm(a, b)
    ref = (a.double() @ b.double().T).float()
    assert (c - ref).abs().max().item() < 1e-5 * ref.abs().max().item()


def test_gemm_rejects_bad_shapes():
    a = torch.zeros(16, 12, dtype=torch.bfloat16, device="cuda")
    b = torch.zeros(16, 12, dtype=torch.bfloat16, device="cuda")
    c = torch.zeros(16, 16, device="cuda")
    with pytest.raises(N.ConfigError):
        N.check(N.lib().oems_tc_gemm_bf16(a.data_ptr(), 12, b.data_ptr(), 12, c.data_ptr(), 16, 16, 16, 12,
                                          0.0, None, None))


def test_elementwise_kernels():
    g = torch.Generator(device="cpu").manual_seed(5)
    B, T, C, ks, s = 3, 37, 5, 8, 4
    x = torch.randn(B, T, C, generator=g).cuda()
    Tout = (T - ks) // s + 1
    ld = 48
    cols = torch.zeros(B * Tout, ld, dtype=torch.bfloat16, device="cuda")
    N.check(N.lib().oems_pk_im2col(x.data_ptr(), cols.data_ptr(), B, T, C, ks, s, ld, None))
    ref = torch.stack([x[:, t * s:t * s + ks, :].reshape(B, ks * C) for t in range(Tout)], 1).reshape(B * Tout, -1)
    assert torch.equal(cols[:, :ks * C], ref.to(torch.bfloat16))
    # col2im is the adjoint of im2col: <im2col(x), d> == <x, col2im(d)>
    d = torch.randn(B * Tout, ld, generator=g).cuda()
    dx = torch.zeros_like(x)
    N.check(N.lib().oems_pk_col2im(d.data_ptr(), ld, dx.data_ptr(), B, T, C, ks, s, None))
    lhs = (ref.double() * d[:, :ks * C].double()).sum()
    rhs = (x.double() * dx.double()).sum()
    assert abs(lhs.item() - rhs.item()) < 1e-6 * max(1.0, abs(lhs.item()))  # f32 accumulation in col2im
    # transpose
    tb = torch.randn(70, 33, generator=g).to(torch.bfloat16).cuda()
    out = torch.zeros(33, 80, dtype=torch.bfloat16, device="cuda")
    N.check(N.lib().oems_pk_transpose_bf16(tb.data_ptr(), 33, out.data_ptr(), 80, 70, 33, None))
    assert torch.equal(out[:, :70], tb.T)
    # relu, relu backward, column sums
    y = torch.randn(40, 24, generator=g).cuda()
    y0 = y.clone()
    yb = torch.zeros(40, 32, dtype=torch.bfloat16, device="cuda")
    N.check(N.lib().oems_pk_relu(y.data_ptr(), yb.data_ptr(), 40, 24, 32, None))
    assert torch.equal(y, y0.clamp_min(0)) and torch.equal(yb[:, :24], y.to(torch.bfloat16))
    dy = torch.randn(40, 24, generator=g).cuda()
    dy0 = dy.clone()
    N.check(N.lib().oems_pk_relu_bwd(dy.data_ptr(), y.data_ptr(), dy.numel(), None))
    assert torch.equal(dy, dy0 * (y > 0))
    db = torch.zeros(24, device="cuda")
    N.check(N.lib().oems_pk_colsum(dy.data_ptr(), 40, 24, db.data_ptr(), None))
    assert torch.allclose(db, dy.sum(0), rtol=1e-5, atol=1e-6)
    torch.cuda.synchronize()


def _round_bf16():
    class RB(torch.autograd.Function):
        """bf16 rounding in forward and backward: the operands the
        tensor-core GEMMs see."""

        @staticmethod
        def forward(ctx, t):
            return t.to(torch.bfloat16).to(torch.float32)

        @staticmethod
        def backward(ctx, g):
            return g.to(torch.bfloat16).to(torch.float32)
    return RB.apply


def _torch_reference(net, x, rounded):
    """The same network in plain PyTorch fp32 (weights from the tensor-core
    network); rounded=True rounds every GEMM operand (and its gradient) to
    bf16 like the kernels do.  Returns the output and the parameters."""
    import torch.nn.functional as Fn
    R = _round_bf16() if rounded else (lambda t: t)
    h = x.clone()
    params = []
    for c in net.convs:
        w = c.fc.w.clone().requires_grad_(True)
        b = c.fc.b.clone().requires_grad_(True)
        params += [w, b]
        B, T, C = h.shape
        To = c.tout(T)
        cols = torch.stack([h[:, t * c.s:t * c.s + c.ks, :].reshape(B, -1) for t in range(To)], 1)
        h = Fn.relu(R(cols) @ R(w).T + b)
    z = h.reshape(h.shape[0], -1)
    w1 = net.fc1.w.clone().requires_grad_(True)
    b1 = net.fc1.b.clone().requires_grad_(True)
    w2 = net.fc2.w.clone().requires_grad_(True)
    b2 = net.fc2.b.clone().requires_grad_(True)
    params += [w1, b1, w2, b2]
    z = Fn.relu(R(z) @ R(w1).T + b1)
    coef = R(z) @ R(w2).T + b2
    out = R(coef) @ R(net.spec.w).T
    return out, params


@pytest.mark.parametrize("rounded,fwd_tol,grad_tol", [(True, 1e-5, 1e-2), (False, 3e-2, 0.15)])
def test_network_forward_backward_matches_torch(rounded, fwd_tol, grad_tol):
    """Against the torch fp32 network with bf16-rounded GEMM operands the
    kernels agree to f32 accumulation order; against plain fp32 the bf16
    rounding (compounded through the ReLU masks) stays within a few %."""
    from openems_b200 import predictor as P
    from openems_b200.predictor_net import NetConfig, TailNet
    cfg = NetConfig(K=512, channels=(16, 32, 32), hidden=64, modes=64, batch=16)
    net = TailNet(cfg, P.FREQS[:61], horizon=4000)
    g = torch.Generator(device="cpu").manual_seed(0)
    x = torch.randn(16, 512, 2, generator=g).cuda()
    out = net.forward(x)
    ref, params = _torch_reference(net, x, rounded)
    rel = (out - ref).abs().max().item() / ref.abs().max().item()
    assert rel < fwd_tol, rel
    net.backward((2 * out.detach() / out.numel()).contiguous())
    (ref.pow(2).sum() / ref.numel()).backward()
    mine = []
    for layer in net.convs:
        mine += [layer.fc.gw, layer.fc.gb]
    mine += [net.fc1.gw, net.fc1.gb, net.fc2.gw, net.fc2.gb]
    for m, p in zip(mine, params):
        rel = (m - p.grad).norm().item() / max(p.grad.norm().item(), 1e-30)
        assert rel < grad_tol, rel


def test_training_reduces_loss():
    from openems_b200 import predictor as P
    from openems_b200.predictor_net import NetConfig, TailNet
    cfg = NetConfig(K=512, channels=(16, 32, 32), hidden=64, batch=32, lr=3e-3)
    net = TailNet(cfg, P.FREQS[:61], horizon=4000)
    g = torch.Generator(device="cpu").manual_seed(1)
    x = torch.randn(32, 512, 2, generator=g).cuda()
    # a learnable target inside the fixed spectral layer's range: modal
    # coefficients that are a linear map of the input's first samples
    A = torch.randn(4 * cfg.modes, 16, generator=g).cuda() * 0.1
    y = ((x[:, :8, :].reshape(32, 16) @ A.T) @ net.spec.w.T).contiguous()
    losses = [net.train_step(x, y) for _ in range(120)]
    N.check(N.lib().oems_tc_check(None))
    assert losses[-1] < 0.5 * losses[0], (losses[0], losses[-1])


@pytest.mark.parametrize("rounded,fwd_tol,grad_tol", [(True, 1e-5, 1e-2), (False, 3e-2, 0.15)])
def test_network_matches_cpu_oracle(rounded, fwd_tol, grad_tol):
    """Forward output and every weight and bias gradient of the tensor-core
    network against the float64 CPU restatement (with bf16 rounding of the
    GEMM operands: agreement to f32 accumulation; without: the bf16 error)."""
    from oracle.tailnet_ref import TailNetRef
    from openems_b200 import predictor as P
    from openems_b200.predictor_net import NetConfig, TailNet
    cfg = NetConfig(K=512, channels=(16, 32, 32), hidden=64, modes=64, batch=16)
    net = TailNet(cfg, P.FREQS[:61], horizon=4000)
    g = torch.Generator(device="cpu").manual_seed(4)
    x = torch.randn(16, 512, 2, generator=g).cuda()
    out = net.forward(x)
    ref = TailNetRef.from_net(net)
    ro = ref.forward(x.cpu().numpy(), bf16=rounded)
    rel = np.abs(out.cpu().numpy() - ro).max() / np.abs(ro).max()
    assert rel < fwd_tol, rel
    dout = (2 * out.detach() / out.numel()).contiguous()
    net.backward(dout)
    N.check(N.lib().oems_tc_check(None))
    grads = ref.backward(dout.cpu().numpy().astype(np.float64))
    mine = [(c.fc.gw, c.fc.gb) for c in net.convs] + [(net.fc1.gw, net.fc1.gb), (net.fc2.gw, net.fc2.gb)]
    for (mw, mb), (rw, rb) in zip(mine, grads):
        for m, r in ((mw, rw), (mb, rb)):
            rel = np.linalg.norm(m.cpu().numpy() - r) / max(np.linalg.norm(r), 1e-30)
            assert rel < grad_tol, rel


def _ringdowns(n, rng, net, K, dt, allowed):
    """Port traces that are one damped sinusoid per channel on a pole of the
    spectral layer's grid, and their exact scaled tail DFTs (the spectral
    layer applied to the modal coefficients at K)."""
    from openems_b200 import predictor as P
    poles = P.PoleGrid().poles()[:net.cfg.modes]
    m = len(poles)
    E = np.exp(np.outer(np.arange(K) * dt, poles))
    C = np.zeros((n, 2, m), complex)
    for ch in range(2):
        j = allowed[rng.integers(0, len(allowed), n)]
        C[np.arange(n), ch, j] = rng.normal(size=n) + 1j * rng.normal(size=n)
    x = np.einsum("km,ncm->nkc", E, C).real.astype(np.float32)
    ck = C * np.exp(poles * K * dt)
    coef = np.concatenate([ck[:, 0].real, ck[:, 0].imag, ck[:, 1].real, ck[:, 1].imag], 1)
    y = coef @ net.spec.w.cpu().numpy().astype(np.float64).T
    return torch.tensor(x).cuda(), torch.tensor(y, dtype=torch.float32).cuda()


def test_trained_network_beats_truncation_on_synthetic_ringdowns():
    """What training on the tensor-core kernels gains over stopping at K
    without a prediction (a zero tail, relative error 1): on ringdowns whose
    modes the first K steps resolve (>= 4 GHz, two periods or more in K), the
    trained network predicts the tail DFT to well under half that error."""
    from openems_b200 import predictor as P
    from openems_b200.predictor_net import NetConfig, TailNet
    K = 512
    cfg = NetConfig(K=K, channels=(16, 32, 32), hidden=256, modes=64, batch=64, lr=1e-3)
    net = TailNet(cfg, P.FREQS[::4], horizon=4000)
    dt = P.grid_dt()
    poles = P.PoleGrid().poles()
    allowed = np.where(np.abs(poles.imag) / (2 * np.pi) >= 4e9)[0]
    rng = np.random.default_rng(1)
    xt, yt = _ringdowns(512, np.random.default_rng(2), net, K, dt, allowed)

    def test_error():
        out = torch.cat([net.forward(xt[i:i + 64].contiguous()) for i in range(0, 512, 64)])
        return ((out - yt).norm() / yt.norm()).item()

    before = test_error()
    for _ in range(1500):
        x, y = _ringdowns(64, rng, net, K, dt, allowed)
        net.train_step(x, y)
    N.check(N.lib().oems_tc_check(None))
    after = test_error()
    print(f"tail DFT relative error: untrained {before:.3f}, trained {after:.3f}, truncation 1.000")
    assert after < 0.5, (before, after)

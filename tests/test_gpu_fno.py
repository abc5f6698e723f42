"""The FNO of libsacfno.so (tcgen05 forward and backward kernels) against the
float64 CPU oracle (oracle/fno_ref.py) on the same BF16-rounded weights and
inputs.  The GPU keeps activations in BF16 and its DFT tables in BF16, so the
bar is a relative L2 of 2e-2 on the output and 5e-2 per gradient group.

Three shapes: CFG, where every layer runs as separate GEMMs; WIDE (F a multiple
of 128, hidden 128), where each Fourier layer's channel-mixing GEMM accumulates
the spectral term as its second product and inference runs the projection in one
kernel that keeps the hidden channels on chip; DUAL, the same layers at width 48
(a 48-column tile)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import fno_ref  # noqa: E402
from sac_b200 import build, fno_abi  # noqa: E402

pytestmark = pytest.mark.gpu

CFG = dict(S=64, F=64, width=32, layers=2, hidden=32, cin=16, cout=6)
WIDE = dict(S=64, F=128, width=32, layers=2, hidden=128, cin=16, cout=6)
DUAL = dict(S=64, F=128, width=48, layers=2, hidden=32, cin=16, cout=6)
SHAPES = pytest.mark.parametrize("cfg", [CFG, WIDE, DUAL], ids=["separate", "fused", "dual"])


@pytest.fixture(scope="module", autouse=True)
def _lib():
    build.build_fno()


def _net(B=2, seed=3, cfg=CFG):
    return fno_abi.Net(max_batch=B, seed=seed, **cfg)


def _layout(cfg=CFG):
    return fno_ref.Layout(width=cfg["width"], layers=cfg["layers"], cin=cfg["cin"], cout=cfg["cout"],
                          hidden=cfg["hidden"])


def _oracle_theta(net, lay):
    th = net.get_params().astype(np.float64)
    # the GEMMs read BF16 copies of the weight matrices; biases stay FP32
    out = fno_ref.bf16_round(th)
    for name in ["Pb", "Q1b", "Q2b"] + [f"Wb{l}" for l in range(lay.layers)]:
        o, n = lay.segs[name]
        out[o:o + n] = th[o:o + n]
    return out


def _rel(a, b):
    return np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-30)


def _inputs(B, seed, cfg=CFG):
    g = torch.Generator().manual_seed(seed)
    x = torch.randn(B, cfg["cin"], cfg["S"], cfg["F"], generator=g).to(torch.bfloat16)
    return x


def test_layout_matches_the_oracle():
    net, lay = _net(), _layout()
    L = net.layout()
    names = ["P", "Pb"] + sum([[f"W{l}", f"Wb{l}", f"Rr{l}", f"Ri{l}"] for l in range(lay.layers)], []) + \
        ["Q1", "Q1b", "Q2", "Q2b"]
    for (off, n), name in zip(L, names):
        assert (off, n) == lay.segs[name], name
    assert net.nparam == lay.n


@SHAPES
def test_forward_matches_oracle(cfg):
    B = 2
    net, lay = _net(B, cfg=cfg), _layout(cfg)
    x = _inputs(B, 1, cfg)
    xd = x.cuda()
    y = torch.zeros(B, cfg["cout"], cfg["S"], cfg["F"], device="cuda")
    torch.cuda.synchronize()
    net.forward(xd.data_ptr(), y.data_ptr(), B)
    net.check()
    yo, _ = fno_ref.forward(lay, _oracle_theta(net, lay), x.double().numpy())
    err = _rel(y.cpu().double().numpy(), yo)
    assert err < 2e-2, err


@SHAPES
def test_gradients_match_oracle(cfg):
    B = 2
    net, lay = _net(B, cfg=cfg), _layout(cfg)
    x = _inputs(B, 2, cfg)
    g = torch.Generator().manual_seed(5)
    dy = torch.zeros(B, net.cpad, cfg["S"], cfg["F"])
    dy[:, :cfg["cout"]] = torch.randn(B, cfg["cout"], cfg["S"], cfg["F"], generator=g)
    dy = dy.to(torch.bfloat16)
    xd, dyd = x.cuda(), dy.cuda()
    y = torch.zeros(B, cfg["cout"], cfg["S"], cfg["F"], device="cuda")
    torch.cuda.synchronize()
    net.zero_grad()
    net.forward(xd.data_ptr(), y.data_ptr(), B)
    net.backward(dyd.data_ptr())
    net.check()
    ggpu = net.get_grads().astype(np.float64)
    th = _oracle_theta(net, lay)
    _, tape = fno_ref.forward(lay, th, x.double().numpy())
    go = fno_ref.backward(lay, th, tape, dy[:, :cfg["cout"]].double().numpy())
    for name, (o, n) in lay.segs.items():
        if name in ("Q2", "Q2b"):
            n = cfg["cout"] * (cfg["hidden"] if name == "Q2" else 1)
        err = _rel(ggpu[o:o + n], go[o:o + n])
        assert err < 5e-2, (name, err)


def test_adam_training_reduces_the_loss():
    B = 2
    net = _net(B, seed=7)
    x = _inputs(B, 3).cuda()
    S, F = CFG["S"], CFG["F"]
    s = torch.linspace(0, 1, S)[:, None]
    f = torch.linspace(0, 1, F)[None, :]
    tgt = torch.stack([torch.sin(2 * np.pi * (c + 1) * s) * torch.cos(2 * np.pi * f) for c in range(6)])
    tgt = tgt[None].repeat(B, 1, 1, 1).to(torch.bfloat16).cuda()
    y = torch.zeros(B, 6, S, F, device="cuda")
    dy = torch.zeros(B, net.cpad, S, F, dtype=torch.bfloat16, device="cuda")
    loss = torch.zeros(1, device="cuda")
    torch.cuda.synchronize()
    losses = []
    for step in range(1, 61):
        loss.zero_()
        torch.cuda.synchronize()
        net.zero_grad()
        net.forward(x.data_ptr(), y.data_ptr(), B)
        net.mse(y.data_ptr(), tgt.data_ptr(), dy.data_ptr(), loss.data_ptr(), B)
        net.backward(dy.data_ptr())
        net.adam(2e-3, step, wd=0.0)
        net.check()
        losses.append(loss.item())
    assert losses[-1] < 0.2 * losses[0], losses[::10]


@SHAPES
def test_inference_pass_equals_training_forward(cfg):
    # WIDE: the fused projection rounds the hidden channels to BF16 and sums them
    # in the same order as the two GEMMs of the training forward
    B = 2
    net = _net(B, cfg=cfg)
    xd = _inputs(B, 4, cfg).cuda()
    y1 = torch.zeros(B, cfg["cout"], cfg["S"], cfg["F"], device="cuda")
    y2 = torch.zeros_like(y1)
    dy = torch.zeros(B, net.cpad, cfg["S"], cfg["F"], dtype=torch.bfloat16, device="cuda")
    torch.cuda.synchronize()
    net.forward(xd.data_ptr(), y1.data_ptr(), B)
    net.infer(xd.data_ptr(), y2.data_ptr(), B)
    net.check()
    assert torch.equal(y1, y2)
    with pytest.raises(fno_abi.FnoError):
        net.backward(dy.data_ptr())  # nothing recorded for a backward pass

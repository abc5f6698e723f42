"""The tcgen05 BF16 GEMM of libsacfno.so against a float64 product of the same
BF16 inputs (FP32 accumulation: relative error a few 1e-6 of sum |a||b|)."""
import pytest

torch = pytest.importorskip("torch")

from sac_b200 import build, fno_abi  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib():
    build.build_fno()
    fno_abi.load()


def _bf(shape, seed):
    g = torch.Generator(device="cpu").manual_seed(seed)
    return torch.randn(*shape, generator=g).to(torch.bfloat16).cuda()


def _close(got, ref, scale):
    err = (got.double() - ref).abs().max().item()
    assert err <= 2e-5 * scale.max().item() + 1e-6, err


def _ref(a, b):  # a: M x K, b: N x K
    return a.double() @ b.double().T


def _scale(a, b):
    return a.double().abs() @ b.double().abs().T


@pytest.mark.parametrize("M,N,K", [(128, 16, 64), (256, 32, 128), (200, 48, 72), (384, 96, 256),
                                   (130, 128, 40), (512, 256, 96), (64, 6 + 10, 16)])
def test_k_major(M, N, K):
    a, b = _bf((M, K), 1), _bf((N, K), 2)
    c = torch.zeros(M, N, dtype=torch.float32, device="cuda")
    fno_abi.gemm(M, N, K, a.data_ptr(), b.data_ptr(), c.data_ptr())
    torch.cuda.synchronize()
    _close(c, _ref(a, b), _scale(a, b))


@pytest.mark.parametrize("amn,bmn", [(True, False), (False, True), (True, True)])
def test_mn_major_operands(amn, bmn):
    M, N, K = 256, 96, 136
    a, b = _bf((M, K), 3), _bf((N, K), 4)
    at, bt = a.T.contiguous(), b.T.contiguous()  # K x M, K x N storage
    c = torch.zeros(M, N, dtype=torch.float32, device="cuda")
    kw = {}
    if amn:
        kw.update(a_mn_major=True, a_m0=1, a_k=M)
    if bmn:
        kw.update(b_mn_major=True, b_n=1, b_k=N)
    fno_abi.gemm(M, N, K, (at if amn else a).data_ptr(), (bt if bmn else b).data_ptr(), c.data_ptr(), **kw)
    torch.cuda.synchronize()
    _close(c, _ref(a, b), _scale(a, b))


def test_split_rows_batches_and_transposed_store():
    # A rows m = (g, s): A[g][k][s] (MN-major per group), C stored as C[g][n][s]
    G, S, K, N, nb = 3, 64, 32, 48, 2
    a = _bf((nb, G, K, S), 5)
    b = _bf((nb, N, K), 6)
    c = torch.zeros(nb, G, N, S, dtype=torch.float32, device="cuda")
    fno_abi.gemm(G * S, N, K, a.data_ptr(), b.data_ptr(), c.data_ptr(), batch=nb,
                 a_mn_major=True, a_m0=1, a_m1=K * S, a_k=S, a_b=G * K * S, a_msplit=S,
                 b_n=K, b_b=N * K, c_m0=1, c_m1=N * S, c_n=S, c_b=G * N * S, c_msplit=S)
    torch.cuda.synchronize()
    for z in range(nb):
        A = a[z].permute(0, 2, 1).reshape(G * S, K)
        ref = _ref(A, b[z]).reshape(G, S, N).permute(0, 2, 1)
        _close(c[z], ref, _scale(A, b[z]).reshape(G, S, N).permute(0, 2, 1))


@pytest.mark.parametrize("K,K2,amn", [(32, 48, True), (64, 40, False), (16, 136, True)])
def test_second_product_accumulates_into_the_tile(K, K2, amn):
    # C[z][n][p] = sum_k A[z][k][p] B[n][k] + sum_j A2[p % F][j] B2[z][n][p // F][j]: the
    # fused spectral term of a Fourier layer, B2's block chosen by the tile's row
    nb, F, S, N = 2, 256, 3, 32
    M = S * F
    a = _bf((nb, K, M), 11) if amn else _bf((nb, M, K), 11)
    b = _bf((N, K), 12)
    a2 = _bf((F, K2), 13)
    b2 = _bf((nb, N, S, K2), 14)
    c = torch.zeros(nb, N, M, dtype=torch.float32, device="cuda")
    kw = dict(a_mn_major=True, a_m0=1, a_k=M, a_b=K * M) if amn else dict(a_m0=K, a_b=M * K)
    fno_abi.gemm(M, N, K, a.data_ptr(), b.data_ptr(), c.data_ptr(), batch=nb, b_n=K, c_m0=1, c_n=M, c_b=N * M,
                 second=dict(K2=K2, a2=a2.data_ptr(), a2_msplit=F, a2_m0=K2, a2_k=1, b2=b2.data_ptr(),
                             b2_n=S * K2, b2_k=1, b2_b=N * S * K2, b2_m=K2, b2_mdiv=F), **kw)
    torch.cuda.synchronize()
    for z in range(nb):
        A = a[z].T if amn else a[z]  # M x K
        A2 = a2.repeat(S, 1)  # row p -> A2[p % F]
        B2 = b2[z].permute(1, 0, 2)  # S x N x K2
        ref = _ref(A, b) + torch.cat([_ref(A2[s * F:(s + 1) * F], B2[s]) for s in range(S)])
        sc = _scale(A, b) + torch.cat([_scale(A2[s * F:(s + 1) * F], B2[s]) for s in range(S)])
        _close(c[z].T, ref, sc)


def test_second_product_argument_checks():
    a, b = _bf((256, 32), 1), _bf((32, 32), 2)
    a2, b2 = _bf((256, 48), 3), _bf((32, 48), 4)
    c = torch.zeros(256, 32, dtype=torch.float32, device="cuda")
    base = dict(K2=48, a2=a2.data_ptr(), a2_m0=48, a2_k=1, b2=b2.data_ptr(), b2_n=48, b2_k=1, b2_mdiv=256)
    for bad in (dict(b2_mdiv=200), dict(K2=44), dict(b2=0), dict(a2_k=2)):
        with pytest.raises(fno_abi.FnoError):
            fno_abi.gemm(256, 32, 32, a.data_ptr(), b.data_ptr(), c.data_ptr(), second={**base, **bad})
    with pytest.raises(fno_abi.FnoError):  # no split K with a second product
        fno_abi.gemm(256, 32, 32, a.data_ptr(), b.data_ptr(), c.data_ptr(), ksplit=2, c_mode=2, second=base)


def test_epilogue_bias_add_gelu_and_grad():
    M, N, K = 256, 32, 64
    a, b = _bf((M, K), 7), _bf((N, K), 8)
    bias = torch.randn(N, device="cuda")
    add = torch.randn(M, N, device="cuda")
    out = torch.zeros(M, N, dtype=torch.bfloat16, device="cuda")
    pre = torch.zeros(M, N, dtype=torch.bfloat16, device="cuda")
    fno_abi.gemm(M, N, K, a.data_ptr(), b.data_ptr(), out.data_ptr(), c_bf16=True, bias_n=bias.data_ptr(),
                 add=add.data_ptr(), act=1, pre=pre.data_ptr())
    torch.cuda.synchronize()
    # GELU is the tanh form, evaluated with the SFU's tanh (relative error ~5e-4)
    z = _ref(a, b) + bias.double() + add.double()
    torch.testing.assert_close(pre.double(), z, rtol=1e-2, atol=1e-2)
    ref = torch.nn.functional.gelu(z, approximate="tanh")
    torch.testing.assert_close(out.double(), ref, rtol=1e-2, atol=1e-2)
    g = torch.zeros(M, N, dtype=torch.float32, device="cuda")
    fno_abi.gemm(M, N, K, a.data_ptr(), b.data_ptr(), g.data_ptr(), act=2, pre=pre.data_ptr())
    torch.cuda.synchronize()
    x = pre.double().requires_grad_(True)
    torch.nn.functional.gelu(x, approximate="tanh").sum().backward()
    acc = _ref(a, b)
    err = (g.double() - acc * x.grad).abs()
    assert (err <= 5e-3 * acc.abs() + 1e-4).all(), err.max().item()  # GELU' moves up to ~5x the tanh error


def test_split_k_atomic_and_accumulate():
    M, N, K = 128, 32, 4096
    a, b = _bf((M, K), 9), _bf((N, K), 10)
    c = torch.ones(M, N, dtype=torch.float32, device="cuda")
    fno_abi.gemm(M, N, K, a.data_ptr(), b.data_ptr(), c.data_ptr(), ksplit=16, c_mode=2)
    fno_abi.gemm(M, N, K, a.data_ptr(), b.data_ptr(), c.data_ptr(), c_mode=1, alpha=-0.5)
    torch.cuda.synchronize()
    _close(c, 1.0 + 0.5 * _ref(a, b), _scale(a, b))


def test_bad_arguments_are_refused():
    a = _bf((128, 12), 11)
    c = torch.zeros(128, 16, device="cuda")
    with pytest.raises(fno_abi.FnoError):
        fno_abi.gemm(128, 16, 12, a.data_ptr(), a.data_ptr(), c.data_ptr())  # K % 8


def test_b_rows_split_mn_major():
    # B(n = (g, s), k) = b[g][k][s] (MN-major within each group), C stored C[g][s][m]
    G, S, K, M = 3, 64, 48, 256
    a = _bf((M, K), 12)
    b = _bf((G, K, S), 13)
    c = torch.zeros(G, S, M, dtype=torch.float32, device="cuda")
    fno_abi.gemm(M, G * S, K, a.data_ptr(), b.data_ptr(), c.data_ptr(), b_mn_major=True, b_n=1, b_k=S,
                 b_n1=K * S, b_nsplit=S, c_m0=1, c_n=M)
    torch.cuda.synchronize()
    Bm = b.permute(0, 2, 1).reshape(G * S, K)
    ref = _ref(a, Bm).T.reshape(G, S, M)
    _close(c, ref, _scale(a, Bm).T.reshape(G, S, M))


def test_wait_time_out_sets_the_error_word_and_returns():
    """wait_tries = -1: the first pipeline wait gives up at once.  The kernel
    raises bit 0 of the error word, drains the MMAs it issued, releases its TMEM
    and returns; the next call with the default bound computes normally."""
    M, N, K = 256, 64, 512  # 8 k tiles: the wait for a free stage comes at k tile 2
    a, b = _bf((M, K), 11), _bf((N, K), 12)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    c = torch.zeros(M, N, dtype=torch.float32, device="cuda")
    fno_abi.gemm(M, N, K, a.data_ptr(), b.data_ptr(), c.data_ptr(), err=err.data_ptr(), wait_tries=-1)
    torch.cuda.synchronize()
    assert int(err.item()) & 1
    err.zero_()
    fno_abi.gemm(M, N, K, a.data_ptr(), b.data_ptr(), c.data_ptr(), err=err.data_ptr())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    _close(c, _ref(a, b), _scale(a, b))


def test_network_reports_the_time_out():
    """The network's GEMMs with the test bound: sac_fno_check returns 7 (a
    tensor-core wait timed out) and the network still runs once the default
    bound is back."""
    net = fno_abi.Net(S=64, F=64, width=32, layers=2, hidden=32, cin=16, cout=6, max_batch=2, seed=1)
    x = torch.randn(2, 16, 64, 64).to(torch.bfloat16).cuda()
    y = torch.zeros(2, 6, 64, 64, dtype=torch.float32, device="cuda")
    net.set_wait_tries(-1)
    net.infer(x.data_ptr(), y.data_ptr(), 2)
    with pytest.raises(fno_abi.FnoError) as e:
        net.check(reset=True)
    assert "status 7" in str(e.value)
    net.set_wait_tries(0)
    net.infer(x.data_ptr(), y.data_ptr(), 2)
    net.check(reset=True)
    assert torch.isfinite(y).all()
    net.close()

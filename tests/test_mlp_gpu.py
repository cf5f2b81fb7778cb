"""The surrogate MLP's tensor-core kernels on the GPU, through the C ABI.

GEMM: every epilogue of ww_mlp_gemm against a PyTorch FP32 matmul of the same bf16 operands
(tolerance: FP32 accumulation order, 1e-5 of the products' magnitude; bf16 outputs within one
bf16 rounding plus the tanh approximation). Gradients: one backward pass against the float64
CPU reference in oracle/mlp_oracle.py, with and without bf16 emulation. AdamW: one update
against the same formula in float64. Training: the loss of a small regression falls.
"""

import numpy as np
import pytest

from conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


@pytest.fixture(scope="module")
def sur(pkg):
    import importlib

    pkg.init()
    return importlib.import_module("ww3_gpu_b200.surrogate")


@pytest.fixture(scope="module")
def mlp_oracle():
    from oracle import mlp_oracle

    return mlp_oracle


def _operands(M, N, K, seed):
    import torch

    g = torch.Generator(device="cpu").manual_seed(seed)
    a = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    b = (torch.randn(N, K, generator=g) / K ** 0.5).to(torch.bfloat16).cuda()
    bias = torch.randn(N, generator=g).cuda()
    return a, b, bias


def _ref(a, b):
    return a.float() @ b.float().T


def _gelu(z):
    import torch

    return 0.5 * z * (1.0 + torch.tanh(0.7978845608028654 * (z + 0.044715 * z ** 3)))


def _dgelu(z):
    import torch

    t = torch.tanh(0.7978845608028654 * (z + 0.044715 * z ** 3))
    return 0.5 * (1 + t) + 0.5 * z * (1 - t * t) * 0.7978845608028654 * (1 + 3 * 0.044715 * z * z)


@pytest.mark.parametrize("M,N,K,bn", [(128, 64, 64, 64), (300, 256, 192, 256),
                                      (1000, 384, 1344, 192), (8256, 1024, 1024, 256),
                                      (257, 1344, 1024, 192), (640, 512, 128, 128)])
def test_gemm_f32_epilogue_matches_torch(sur, M, N, K, bn):
    import torch

    a, b, bias = _operands(M, N, K, seed=M + N + K)
    out = torch.full((M, N), float("nan"), device="cuda")
    sur.gemm(sur.EPI_F32, a, b, bias=bias, out_f32=out, bn=bn)
    torch.cuda.synchronize()
    ref = _ref(a, b) + bias
    scale = (a.float().abs() @ b.float().abs().T) + bias.abs()
    err = ((out - ref).abs() / scale).max().item()
    assert err < 1e-5, f"max relative error {err:.3e} (tile {bn})"


@pytest.mark.parametrize("M,N,K,bn", [(256, 256, 64, 256), (1000, 1344, 1024, 192),
                                      (4096, 1024, 1344, 256), (8320, 1024, 1024, 256),
                                      (300, 512, 128, 128), (520, 192, 256, 64)])
def test_gemm_paired_tiles_match_torch(sur, M, N, K, bn):
    """Two CTAs of a cluster per 256-row tile (tcgen05.mma.cta_group::2, each CTA holding half
    of B's tile): the f32 and GELU inference epilogues against FP32 torch; ragged M."""
    import torch

    a, b, bias = _operands(M, N, K, seed=M + 3 * N + K)
    out = torch.full((M, N), float("nan"), device="cuda")
    sur.gemm(sur.EPI_F32 | sur.PAIRED, a, b, bias=bias, out_f32=out, bn=bn)
    torch.cuda.synchronize()
    ref = _ref(a, b) + bias
    scale = (a.float().abs() @ b.float().abs().T) + bias.abs()
    err = ((out - ref).abs() / scale).max().item()
    assert err < 1e-5, f"max relative error {err:.3e} (paired, tile {bn})"
    g = torch.zeros(M, N, dtype=torch.bfloat16, device="cuda")
    sur.gemm(sur.EPI_GELU_INFER | sur.PAIRED, a, b, bias=bias, out=g, bn=bn)
    torch.cuda.synchronize()
    assert torch.allclose(g.float(), _gelu(ref), rtol=2 ** -7, atol=2e-3)


def test_gemm_gelu_train_epilogue(sur):
    import torch

    M, N, K = 384, 512, 256
    a, b, bias = _operands(M, N, K, seed=11)
    out = torch.zeros(M, N, dtype=torch.bfloat16, device="cuda")
    aux = torch.zeros_like(out)
    out_t = torch.zeros(N, 512, dtype=torch.bfloat16, device="cuda")  # ldt > M
    sur.gemm(sur.EPI_GELU_TRAIN, a, b, bias=bias, out=out, out_t=out_t, aux=aux)
    torch.cuda.synchronize()
    z = _ref(a, b) + bias
    assert torch.allclose(aux.float(), z, rtol=2 ** -7, atol=1e-5)
    g = _gelu(z)
    assert torch.allclose(out.float(), g, rtol=2 ** -7, atol=2e-3)
    assert torch.equal(out_t[:, :M], out.T)


def test_gemm_gelu_infer_epilogue(sur):
    import torch

    M, N, K = 200, 256, 128
    a, b, bias = _operands(M, N, K, seed=12)
    out = torch.zeros(M, N, dtype=torch.bfloat16, device="cuda")
    sur.gemm(sur.EPI_GELU_INFER, a, b, bias=bias, out=out)
    torch.cuda.synchronize()
    assert torch.allclose(out.float(), _gelu(_ref(a, b) + bias), rtol=2 ** -7, atol=2e-3)


def test_gemm_dgelu_epilogue(sur):
    import torch

    M, N, K = 256, 384, 192
    a, b, _ = _operands(M, N, K, seed=13)
    z = torch.randn(M, N, device="cuda").to(torch.bfloat16)
    out = torch.zeros(M, N, dtype=torch.bfloat16, device="cuda")
    out_t = torch.zeros(N, M, dtype=torch.bfloat16, device="cuda")
    sur.gemm(sur.EPI_DGELU, a, b, out=out, out_t=out_t, aux=z)
    torch.cuda.synchronize()
    ref = _ref(a, b) * _dgelu(z.float())
    assert torch.allclose(out.float(), ref, rtol=2 ** -7, atol=2e-3 * ref.abs().max().item())
    assert torch.equal(out_t, out.T)


@pytest.mark.parametrize("splits", [1, 2, 4])
def test_gemm_split_reduction_accumulates(sur, splits):
    import torch

    M, N, K = 1024, 1024, 2048
    a, b, _ = _operands(M, N, K, seed=14)
    out = torch.ones(M, N, device="cuda")
    sur.gemm(sur.EPI_ATOMIC, a, b, out_f32=out, splits=splits)
    torch.cuda.synchronize()
    ref = _ref(a, b) + 1.0
    scale = a.float().abs() @ b.float().abs().T + 1.0
    assert ((out - ref).abs() / scale).max().item() < 1e-5


def test_gemm_refuses_bad_shapes(pkg, sur):
    import torch

    a, b, bias = _operands(128, 100, 64, seed=1)  # N not a multiple of any tile width
    out = torch.zeros(128, 100, device="cuda")
    with pytest.raises(pkg.WwError) as e:
        sur.gemm(sur.EPI_F32, a, b, bias=bias, out_f32=out, bn=64)
    assert e.value.code == pkg.ERR_BAD_SHAPE


def _small_net(sur, seed=0, din=128, dh=128, dout=128):
    rng = np.random.default_rng(seed)
    net = sur.Mlp(din, dh, dout, cap=256, seed=seed + 1)
    layers = [(rng.normal(0, 1 / np.sqrt(k), (n, k)).astype(np.float32),
               rng.normal(0, 0.1, n).astype(np.float32)) for n, k in net.shapes()]
    net.set_params(layers)
    return net, layers, rng


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_gradients_match_cpu_oracle(sur, mlp_oracle):
    import torch

    net, layers, rng = _small_net(sur)
    m = 256
    x = mlp_oracle.bf16(rng.normal(0, 1, (m, 128)).astype(np.float32))
    t = rng.normal(0, 1, (m, 128)).astype(np.float32)
    loss = net.train_step(torch.tensor(x, dtype=torch.bfloat16, device="cuda"),
                          torch.tensor(t, device="cuda"), apply=False)
    grads = net.get_grads()
    loss_e, ref_e = mlp_oracle.forward_backward(layers, x, t, emulate_bf16=True)
    loss_x, ref_x = mlp_oracle.forward_backward(layers, x, t, emulate_bf16=False)
    assert abs(loss[0] - loss_e) < 1e-3 * loss_e
    for l in range(4):
        assert _rel(grads[l][0], ref_e[l][0]) < 1e-2, f"dW{l + 1} vs bf16-emulating oracle"
        assert _rel(grads[l][1], ref_e[l][1]) < 1e-2, f"db{l + 1} vs bf16-emulating oracle"
        assert _rel(grads[l][0], ref_x[l][0]) < 5e-2, f"dW{l + 1} vs float64 oracle"
        assert _rel(grads[l][1], ref_x[l][1]) < 5e-2, f"db{l + 1} vs float64 oracle"


def test_adamw_update_matches_formula(sur, mlp_oracle):
    import torch

    net, layers, rng = _small_net(sur, seed=3)
    m = 128
    x = torch.tensor(mlp_oracle.bf16(rng.normal(0, 1, (m, 128)).astype(np.float32)),
                     dtype=torch.bfloat16, device="cuda")
    t = torch.tensor(rng.normal(0, 1, (m, 128)).astype(np.float32), device="cuda")
    net.train_step(x, t, apply=False)
    grads = net.get_grads()
    lr, wd = 1e-3, 0.01
    net.train_step(x, t, lr=lr, wd=wd, apply=True)
    after = net.get_params()
    for l in range(4):
        w_ref, _, _ = mlp_oracle.adamw_step(layers[l][0], grads[l][0], lr, wd)
        b_ref, _, _ = mlp_oracle.adamw_step(layers[l][1], grads[l][1], lr, wd)
        assert np.allclose(after[l][0], w_ref, rtol=1e-5, atol=1e-6)
        assert np.allclose(after[l][1], b_ref, rtol=1e-5, atol=1e-6)


def test_training_reduces_loss(sur):
    import torch

    net, _, rng = _small_net(sur, seed=5)
    m = 256
    proj = rng.normal(0, 1 / np.sqrt(128), (128, 128))
    xs = rng.normal(0, 1, (m, 128)).astype(np.float32)
    ts = np.sin(xs @ proj).astype(np.float32)
    x = torch.tensor(xs, dtype=torch.bfloat16, device="cuda")
    t = torch.tensor(ts, device="cuda")
    first = net.train_step(x, t, lr=2e-3)[0]
    for _ in range(300):
        last = net.train_step(x, t, lr=2e-3)[0]
    assert last < 0.1 * first, f"loss {first:.4f} -> {last:.4f}"

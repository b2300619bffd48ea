"""The surrogate's device kernels (libdem_b200 through its C ABI) against plain
PyTorch fp32 references of the same ops.

The GEMM takes bf16 operands and accumulates in fp32: its reference is the
fp32 product of the same bf16 values, so the only difference is the fp32
summation order (tolerance 1e-5 relative to the output's scale; bf16 outputs
within one bf16 rounding).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

DEV = torch.device("cuda", 0)


def _ops():
    from mbd_icenav_b200 import sg_ops
    return sg_ops


def _bf(shape, g, scale=1.0):
    return (torch.randn(shape, generator=g, device="cpu") * scale).to(torch.bfloat16).to(DEV)


def _ref_gemm(A, B, bias=None, relu=False, mask=None):
    r = A.float() @ B.float().T
    if bias is not None:
        r = r + bias
    if relu:
        r = torch.clamp(r, min=0.0)
    if mask is not None:
        r = r * (mask.float() > 0)
    return r


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (256, 128, 128), (300, 200, 200), (1000, 64, 576),
                                   (4096, 512, 2240), (130, 3, 512), (77, 96, 8), (2048, 128, 1152),
                                   (8192, 512, 2304), (16000, 600, 200)])
def test_gemm_matches_fp32_reference(M, N, K):
    """Every tile width: 64 (N <= 64), 128, and 256 (N >= 512 with at least 128
    tiles of 128 x 256: the last two shapes, one with ragged M and N edges)."""
    ops = _ops()
    g = torch.Generator().manual_seed(M * 7 + N * 3 + K)
    A, B = _bf((M, K), g), _bf((N, K), g)
    out = ops.gemm(A, B)
    torch.cuda.synchronize()
    ops.error_flag(DEV).check()
    ref = _ref_gemm(A, B)
    scale = ref.abs().max().item() + 1e-30
    err = (out - ref).abs().max().item() / scale
    assert err < 1e-5, (M, N, K, err)


def test_gemm_epilogue_bias_relu_mask_bf16_out_and_strides():
    ops = _ops()
    g = torch.Generator().manual_seed(5)
    M, N, K = 333, 150, 264
    Abig = _bf((M, K + 40), g)  # row stride 304 (a multiple of 8), view of the first K columns
    A = Abig[:, :K]
    B = _bf((N, K), g)
    bias = torch.randn(N, generator=g).to(DEV)
    mask = _bf((M, N), g)
    out = torch.zeros((M, N + 14), dtype=torch.bfloat16, device=DEV)[:, :N]  # row stride 164 (not a multiple of 8)
    ops.gemm(A, B, out=out, bias=bias, relu=True, mask=mask)
    ref = _ref_gemm(A, B, bias, True, mask)
    torch.cuda.synchronize()
    ops.error_flag(DEV).check()
    np.testing.assert_allclose(out.float().cpu().numpy(), ref.to(torch.bfloat16).float().cpu().numpy(),
                               rtol=1.0 / 128, atol=1e-5 * ref.abs().max().item())
    out32 = ops.gemm(A, B, bias=bias, relu=True)
    ref32 = _ref_gemm(A, B, bias, True)
    assert (out32 - ref32).abs().max().item() <= 1e-5 * ref32.abs().max().item()


def test_gemm_repeated_calls_are_bit_identical():
    ops = _ops()
    g = torch.Generator().manual_seed(11)
    A, B = _bf((640, 512), g), _bf((192, 512), g)
    a = ops.gemm(A, B)
    b = ops.gemm(A, B)
    torch.cuda.synchronize()
    assert torch.equal(a, b)


@pytest.mark.parametrize("C", [1, 32])
def test_im2col_gemm_is_conv2d_and_col2im_is_its_adjoint(C):
    """3x3 stride-2 padding-1 convolution as im2col + GEMM equals torch's conv2d
    (fp32, same bf16 values); col2im is the adjoint of im2col: it equals the
    gradient autograd takes through the same patches (then rounded to bf16)."""
    ops = _ops()
    g = torch.Generator().manual_seed(C)
    Bn, H, W, Co = 3, 16, 12, 24
    kpad = ((9 * C + 63) // 64) * 64
    X = _bf((Bn, H, W, C), g)
    Wt = _bf((Co, 3, 3, C), g)  # (out, ky, kx, c) = the patch order of im2col
    Wk = torch.zeros((Co, kpad), dtype=torch.bfloat16, device=DEV)
    Wk[:, :9 * C] = Wt.reshape(Co, 9 * C)
    cols = ops.im2col(X, kpad)
    Y = ops.gemm(cols, Wk).reshape(Bn, H // 2, W // 2, Co)
    ref = torch.nn.functional.conv2d(X.float().permute(0, 3, 1, 2), Wt.float().permute(0, 3, 1, 2), stride=2,
                                     padding=1).permute(0, 2, 3, 1)
    assert (Y - ref).abs().max().item() <= 1e-5 * ref.abs().max().item()
    # adjoint
    dcols = torch.randn(cols.shape, generator=g).to(DEV)
    dcols[:, 9 * C:] = 0
    dX = ops.col2im(dcols, (Bn, H, W, C), kpad)
    # dX is rounded to bf16: compare against the fp32 adjoint computed by autograd
    Xr = X.float().clone().requires_grad_(True)
    cols_t = torch.nn.functional.unfold(Xr.permute(0, 3, 1, 2), 3, padding=1, stride=2)  # (B, C*9, L) in (c, ky, kx)
    Bn_, CK, L = cols_t.shape
    perm = cols_t.reshape(Bn_, C, 9, L).permute(0, 3, 2, 1).reshape(Bn_ * L, 9 * C)  # (ky, kx, c) order
    (perm * dcols[:, :9 * C]).sum().backward()
    np.testing.assert_allclose(dX.float().cpu().numpy(), Xr.grad.to(torch.bfloat16).float().cpu().numpy(),
                               rtol=1.0 / 128, atol=1e-6)


def test_col2im_applies_relu_mask():
    ops = _ops()
    g = torch.Generator().manual_seed(3)
    Bn, H, W, C = 2, 8, 8, 32
    kpad = 320
    dcols = torch.randn((Bn * 16, kpad), generator=g).to(DEV)
    act = _bf((Bn, H, W, C), g)
    a = ops.col2im(dcols, (Bn, H, W, C), kpad, act=act)
    b = ops.col2im(dcols, (Bn, H, W, C), kpad)
    assert torch.equal(a, torch.where(act.float() > 0, b.float(), torch.zeros_like(b.float())).to(torch.bfloat16))


def test_transpose_colsum_to_bf16():
    ops = _ops()
    g = torch.Generator().manual_seed(4)
    X = _bf((1000, 70), g)
    assert torch.equal(ops.transpose(X), X.T.contiguous())
    Xf = torch.randn((5000, 33), generator=g).to(DEV)
    assert torch.allclose(ops.colsum(Xf), Xf.sum(0), rtol=1e-5, atol=1e-4)
    assert torch.allclose(ops.colsum(X), X.float().sum(0), rtol=1e-5, atol=1e-4)
    assert torch.equal(ops.to_bf16(Xf), Xf.to(torch.bfloat16))


def test_adam_matches_torch_adam():
    ops = _ops()
    g = torch.Generator().manual_seed(8)
    R, Cc = 40, 24
    p0 = torch.randn((R, Cc), generator=g).to(DEV)
    p = p0.clone()
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    w = torch.empty((R, Cc), dtype=torch.bfloat16, device=DEV)
    wt = torch.empty((Cc, R), dtype=torch.bfloat16, device=DEV)
    ref = p0.clone().requires_grad_(True)
    opt = torch.optim.Adam([ref], lr=1e-2, betas=(0.9, 0.999), eps=1e-8)
    for t in range(1, 6):
        grad = torch.randn((R, Cc), generator=g).to(DEV)
        ops.adam(p, grad, m, v, 1e-2, t, w, wt)
        ref.grad = grad.clone()
        opt.step()
    assert torch.allclose(p, ref.detach(), rtol=1e-5, atol=1e-6)
    assert torch.equal(w, p.to(torch.bfloat16))
    assert torch.equal(wt, p.to(torch.bfloat16).T.contiguous())


def test_mse_and_row_packing():
    ops = _ops()
    g = torch.Generator().manual_seed(9)
    R = 700
    pred = torch.randn((R, 64), generator=g).to(DEV)
    tgt = torch.randn((R, 3), generator=g).to(DEV)
    grad = torch.empty((R, 64), dtype=torch.bfloat16, device=DEV)
    loss = torch.empty(1, device=DEV)
    ops.mse(pred, tgt, 3, grad, loss)
    d = pred[:, :3] - tgt
    assert abs(loss.item() - (d * d).mean().item()) <= 1e-5 * (d * d).mean().item()
    assert torch.equal(grad[:, :3], (2 * d / (R * 3)).to(torch.bfloat16))
    assert torch.count_nonzero(grad[:, 3:]) == 0
    enc = _bf((5, 40), g)
    rows = torch.tensor([4, 0, 0, 2], dtype=torch.int32, device=DEV)
    extra = torch.randn((4, 6), generator=g).to(DEV)
    x = torch.full((4, 64), 7.0, dtype=torch.bfloat16, device=DEV)
    ops.pack_rows(enc, extra, x, enc_row=rows)
    assert torch.equal(x[:, :40], enc[rows.long()])
    assert torch.equal(x[:, 40:46], extra.to(torch.bfloat16))
    assert torch.count_nonzero(x[:, 46:]) == 0
    act = _bf((4, 40), g)
    de = torch.empty((4, 40), dtype=torch.bfloat16, device=DEV)
    ops.unpack_grad(x, 40, act, de)
    assert torch.equal(de, torch.where(act.float() > 0, x[:, :40].float(), torch.zeros_like(de.float()))
                       .to(torch.bfloat16))


class _RoundBF16(torch.autograd.Function):
    """Identity rounded to bf16 in both directions: the network's kernels store
    every activation and every activation gradient as bf16."""

    @staticmethod
    def forward(ctx, x):
        return x.to(torch.bfloat16).float()

    @staticmethod
    def backward(ctx, g):
        return g.to(torch.bfloat16).float()


class _GradBF16(torch.autograd.Function):
    """Identity forward, gradient rounded to bf16 (the loss gradient the MSE kernel stores)."""

    @staticmethod
    def forward(ctx, x):
        return x.clone()

    @staticmethod
    def backward(ctx, g):
        return g.to(torch.bfloat16).float()


def _torch_reference(net, patches, extra):
    """The same network in plain fp32 PyTorch (autograd, no TF32) on the kernels'
    bf16 weights, rounding activations and their gradients to bf16 where the
    kernels store them."""
    from mbd_icenav_b200 import surrogate as S
    params = []
    x = patches.float().permute(0, 3, 1, 2)
    for layer, (cin, cout) in zip(net.conv, S.CONV):
        w = layer.w.float()[:, :9 * cin].reshape(cout, 3, 3, cin).permute(0, 3, 1, 2).clone().requires_grad_(True)
        b = layer.b.clone().requires_grad_(True)
        params.append((w, b))
        x = _RoundBF16.apply(torch.relu(torch.nn.functional.conv2d(x, w, b, stride=2, padding=1)))
    enc = x.permute(0, 2, 3, 1).reshape(x.shape[0], -1)
    h = torch.cat([enc, extra, torch.zeros((enc.shape[0], net.xdim - enc.shape[1] - extra.shape[1]), device=DEV)], 1)
    for li, layer in enumerate(net.fc):
        w = layer.w.float().clone().requires_grad_(True)
        b = layer.b.clone().requires_grad_(True)
        params.append((w, b))
        h = h @ w.T + b
        if li < len(net.fc) - 1:
            h = _RoundBF16.apply(torch.relu(h))
    return _GradBF16.apply(h), params


def test_network_forward_and_gradients_match_torch_autograd():
    """Forward outputs and every layer's weight / bias gradients of the bf16
    tensor-core network against fp32 autograd on the same bf16 weights and
    inputs, rounding where the kernels round.  What remains is the fp32
    summation order and the bf16 roundings it can flip: relative norms within
    2 % (4 % for the convolutions and the first fully connected layer, whose
    gradients pass through the bf16 rounding of three or more layers above
    them) and direction (cosine) above 0.999 for every layer."""
    from mbd_icenav_b200 import surrogate as S
    ops = _ops()
    R, H = 64, 64
    net = S.SurrogateNet(horizon=H, device=DEV, seed=1)
    g = torch.Generator().manual_seed(2)
    patches = _bf((R, 64, 64, 1), g)
    extra = torch.randn((R, net.n_extra), generator=g).to(DEV) * 0.5
    tgt = torch.randn((R, S.N_OUT), generator=g).to(DEV)
    out = net.forward(patches, extra, keep=True)
    grad = torch.empty((R, S.OUT_ROWS), dtype=torch.bfloat16, device=DEV)
    loss = torch.empty(1, device=DEV)
    ops.mse(out, tgt, S.N_OUT, grad, loss)
    net.backward(grad)
    torch.cuda.synchronize()
    ops.error_flag(DEV).check()
    tf32 = (torch.backends.cudnn.allow_tf32, torch.backends.cuda.matmul.allow_tf32)
    torch.backends.cudnn.allow_tf32 = torch.backends.cuda.matmul.allow_tf32 = False
    try:
        ref_out, params = _torch_reference(net, patches, extra.to(torch.bfloat16).float())
    finally:
        torch.backends.cudnn.allow_tf32, torch.backends.cuda.matmul.allow_tf32 = tf32
    rl = ((ref_out[:, :S.N_OUT] - tgt) ** 2).mean()
    rl.backward()
    o = out[:, :S.N_OUT]
    assert (o - ref_out[:, :S.N_OUT]).norm() <= 2e-2 * ref_out[:, :S.N_OUT].norm()
    assert abs(loss.item() - rl.item()) <= 2e-2 * rl.item()
    layers = net.conv + net.fc
    for i, (layer, (w, b)) in enumerate(zip(layers, params)):
        gw = layer.g
        if i < len(net.conv):
            cin = S.CONV[i][0]
            rw = w.grad.permute(0, 2, 3, 1).reshape(w.shape[0], 9 * cin)
            assert torch.count_nonzero(gw[:, 9 * cin:]) == 0, i  # padded columns get no gradient
            gw = gw[:, :9 * cin]
        else:
            rw = w.grad
        for name, a, r in (("w", gw, rw), ("b", layer.gb, b.grad)):
            rel = ((a - r).norm() / (r.norm() + 1e-30)).item()
            cos = torch.nn.functional.cosine_similarity(a.reshape(1, -1), r.reshape(1, -1)).item()
            assert rel < (4e-2 if i <= len(net.conv) else 2e-2) and cos > 0.999, (i, name, rel, cos)


def test_adam_training_reduces_the_loss():
    """A few Adam steps through the kernels fit a fixed batch."""
    from mbd_icenav_b200 import surrogate as S
    ops = _ops()
    R = 128
    net = S.SurrogateNet(horizon=64, device=DEV, seed=3)
    g = torch.Generator().manual_seed(4)
    patches = _bf((R, 64, 64, 1), g)
    extra = torch.randn((R, net.n_extra), generator=g).to(DEV)
    tgt = torch.randn((R, S.N_OUT), generator=g).to(DEV)
    grad = torch.empty((R, S.OUT_ROWS), dtype=torch.bfloat16, device=DEV)
    loss = torch.empty(1, device=DEV)
    losses = []
    for it in range(30):
        out = net.forward(patches, extra, keep=True)
        ops.mse(out, tgt, S.N_OUT, grad, loss)
        losses.append(loss.item())
        net.backward(grad)
        net.adam_step(1e-3)
    ops.error_flag(DEV).check()
    assert losses[-1] < 0.5 * losses[0], losses

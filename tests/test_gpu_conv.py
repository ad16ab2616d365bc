"""tcgen05 3x3x3 convolutions against a plain PyTorch FP32 reference of the
same operation (BF16-rounded operands)."""
import itertools

import pytest

pytestmark = pytest.mark.gpu


def reference_conv(x, w, bias, relu):
    """x: [B, Z, Y, X, Cin] float; w: [27, Cout, Cin]; NDHWC out."""
    import torch
    cin, cout = x.shape[-1], w.shape[1]
    wt = w.reshape(3, 3, 3, cout, cin).permute(3, 4, 0, 1, 2).contiguous()  # [co, ci, dz, dy, dx]
    y = torch.nn.functional.conv3d(x.permute(0, 4, 1, 2, 3), wt, bias=bias, padding=1)
    y = y.permute(0, 2, 3, 4, 1)
    return torch.relu(y) if relu else y


@pytest.mark.parametrize("cin,cout,shape", [(c, d, s) for (c, d), s in itertools.product(
    [(16, 16), (16, 32), (32, 64), (64, 64), (64, 16), (32, 32)], [(16, 16, 6), (128, 2, 3), (8, 8, 6), (4, 8, 8)])])
def test_conv_matches_torch(cuda, cin, cout, shape):
    import torch
    from diff_solver_b200 import _native as N
    nx, ny, nz = shape
    batch = 2
    g = torch.Generator(device="cpu").manual_seed(cin * 100 + cout)
    x = torch.randn(batch, nz, ny, nx, cin, generator=g).to(torch.bfloat16)
    w = (torch.randn(27, cout, cin, generator=g) / (27 * cin) ** 0.5).to(torch.bfloat16)
    bias = torch.randn(cout, generator=g).float()
    xd, wd, bd = x.cuda(), w.cuda(), bias.cuda()
    out = torch.zeros(batch, nz, ny, nx, cout, dtype=torch.bfloat16, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    for relu in (0, 1):
        N.check("conv", N.lib().xs_conv3d_bf16(None, batch, nx, ny, nz, cin, cout, xd.data_ptr(), wd.data_ptr(), bd.data_ptr(),
                                               out.data_ptr(), relu, err.data_ptr()))
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        want = reference_conv(x.float(), w.float(), bias, relu)
        got = out.float().cpu()
        rel = (got - want).norm() / want.norm()
        assert rel < 1e-2, (cin, cout, shape, relu, float(rel))


@pytest.mark.parametrize("cin,cout,shape,batch", [
    (16, 16, (16, 16, 6), 2), (16, 32, (128, 2, 3), 1), (32, 64, (16, 16, 4), 2), (64, 64, (32, 8, 5), 1),
    (64, 16, (16, 8, 7), 2), (32, 32, (64, 4, 3), 3), (64, 32, (16, 16, 16), 1),
    # volumes whose x-y planes hold fewer than 128 voxels: tiles span several z planes
    (16, 16, (8, 8, 6), 2), (32, 64, (4, 8, 8), 1), (64, 64, (8, 8, 4), 2)])
def test_conv_gradients_match_torch(cuda, cin, cout, shape, batch):
    """Weight gradient (tcgen05, MN-major operands) and input gradient (the
    forward kernel with flipped, transposed weights) against autograd."""
    import torch
    from diff_solver_b200 import _native as N
    L = N.lib()
    nx, ny, nz = shape
    g = torch.Generator(device="cpu").manual_seed(7 * cin + cout + nz)
    x = torch.randn(batch, nz, ny, nx, cin, generator=g).to(torch.bfloat16)
    w = (torch.randn(27, cout, cin, generator=g) / (27 * cin) ** 0.5).to(torch.bfloat16)
    dy = torch.randn(batch, nz, ny, nx, cout, generator=g).to(torch.bfloat16)

    xf = x.float().requires_grad_(True)
    wf = w.float().requires_grad_(True)
    y = reference_conv(xf, wf, None, False)
    y.backward(dy.float())

    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    scratch = torch.empty(L.xs_conv3d_weight_grad_scratch_floats(batch, nx, ny, nz, cin, cout), dtype=torch.float32, device="cuda")
    dw = torch.full((27, cout, cin), 3.0, dtype=torch.float32, device="cuda")
    xd, dyd = x.cuda(), dy.cuda()
    for accumulate in (0, 1):
        N.check("wgrad", L.xs_conv3d_weight_grad_bf16(None, batch, nx, ny, nz, cin, cout, xd.data_ptr(), dyd.data_ptr(),
                                                       scratch.data_ptr(), dw.data_ptr(), accumulate, err.data_ptr()))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    got = dw.cpu() / 2.0  # accumulated twice
    rel = (got - wf.grad).norm() / wf.grad.norm()
    assert rel < 1e-4, (cin, cout, shape, float(rel))

    # input gradient: conv(dY, W') with W'[t][ci][co] = W[26 - t][co][ci]
    wt = w.flip(0).transpose(1, 2).contiguous().cuda()
    dx = torch.zeros(batch, nz, ny, nx, cin, dtype=torch.bfloat16, device="cuda")
    N.check("dgrad", L.xs_conv3d_bf16(None, batch, nx, ny, nz, cout, cin, dyd.data_ptr(), wt.data_ptr(), None, dx.data_ptr(), 0,
                                      err.data_ptr()))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    rel = (dx.float().cpu() - xf.grad).norm() / xf.grad.norm()
    assert rel < 1e-2, (cin, cout, shape, float(rel))

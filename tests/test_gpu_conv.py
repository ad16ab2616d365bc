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
    [(16, 16), (16, 32), (32, 64), (64, 64), (64, 16), (32, 32)], [(16, 16, 6), (128, 2, 3)])])
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

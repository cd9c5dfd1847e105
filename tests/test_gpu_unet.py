"""The learned warm start's kernels: BF16 implicit-GEMM convolutions (every
form the U-Net uses) against torch FP64 on the same BF16 values, weight
gradients, Adam, and the whole network's forward and backward against the
FP64 oracle (oracle/unet_ref.py)."""
import ctypes as C

import numpy as np
import pytest
import torch
import torch.nn.functional as F

from fluxfx_b200 import _native as N
from oracle import unet_ref as U

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def lib():
    return N.load()


def bf(x):
    return x.to(torch.bfloat16)


def rel_l2(a, b):
    a = a.detach().double().cpu()
    b = b.detach().double().cpu()
    return float((a - b).norm() / max(float(b.norm()), 1e-30))


def rel_err(a, b):
    a = a.detach().double().cpu()
    b = b.detach().double().cpu()
    return float((a - b).abs().max() / max(float(b.abs().max()), 1e-30))


def conv_struct(batch, ind, outd, c1, c2, cout, ks, stride, pad, transposed, in1, p1, o1, in2, p2, o2, w, bias,
                relu, out, op, oo, out32, p32, accumulate=0):
    c = N.FfxConv()
    c.batch = batch
    c.in_dims = (N.i32 * 3)(*ind)
    c.out_dims = (N.i32 * 3)(*outd)
    c.c1, c.c2, c.cout = c1, c2, cout
    c.ksize, c.stride, c.pad, c.transposed = ks, stride, pad, transposed
    c.in1 = N.FfxTensorView(in1.data_ptr(), p1, o1)
    c.in2 = N.FfxTensorView(in2.data_ptr() if in2 is not None else None, p2, o2)
    c.weight = w.data_ptr()
    c.bias = bias.data_ptr() if bias is not None else None
    c.relu, c.accumulate = relu, accumulate
    c.out = out.data_ptr() if out is not None else None
    c.out_pitch, c.out_offset = op, oo
    c.out_f32 = out32.data_ptr() if out32 is not None else None
    c.out_f32_pitch = p32
    return c


@pytest.mark.parametrize('kind', ['conv3', 'conv3_concat', 'down', 'up', 'head'])
def test_convolution_forms_match_torch(lib, kind):
    g = torch.Generator().manual_seed(1)
    B, D, H, W = 2, 12, 8, 16
    c1, c2, cout = {'conv3': (16, 0, 32), 'conv3_concat': (16, 24, 40), 'down': (16, 0, 32), 'up': (32, 0, 16),
                    'head': (16, 0, 8)}[kind]
    cin = c1 + c2
    ind = (D // 2, H // 2, W // 2) if kind == 'up' else (D, H, W)
    outd = {'down': (D // 2, H // 2, W // 2), 'up': (D, H, W)}.get(kind, (D, H, W))
    taps = {'down': 8, 'up': 8, 'head': 1}.get(kind, 27)
    x1 = bf(torch.randn((B, *ind, c1 + 8), generator=g))        # pitch c1 + 8, offset 8 (a view)
    x2 = bf(torch.randn((B, *ind, c2), generator=g)) if c2 else None
    w = bf(torch.randn((taps, cin, cout), generator=g) / (taps * cin) ** 0.5)
    bias = torch.randn(cout, generator=g)
    dx1, dx2, dw, db = x1.cuda(), (x2.cuda() if x2 is not None else None), w.cuda(), bias.cuda()
    out32 = torch.zeros((B, *outd, cout), device='cuda')
    out16 = torch.zeros((B, *outd, cout + 16), dtype=torch.bfloat16, device='cuda')
    ks, stride, pad = {'conv3': (3, 1, 1), 'conv3_concat': (3, 1, 1), 'down': (2, 2, 0), 'up': (2, 2, 0),
                       'head': (1, 1, 0)}[kind]
    c = conv_struct(B, ind, outd, c1, c2, cout, ks, stride, pad, int(kind == 'up'), dx1, c1 + 8, 8, dx2, c2, 0, dw,
                    db, 1, out16, cout + 16, 8, out32, cout)
    N.check(lib.ffx_conv_forward(C.byref(c), None))
    torch.cuda.synchronize()
    # torch FP64 on the same BF16 values
    xin = x1[..., 8:].double()
    if x2 is not None:
        xin = torch.cat([xin, x2.double()], -1)
    xt = xin.permute(0, 4, 1, 2, 3)
    wt = U.torch_weight('up' if kind == 'up' else {'head': 'head', 'down': 'down'}.get(kind, 'conv3'), w.double())
    if kind == 'up':
        ref = F.conv_transpose3d(xt, wt, bias.double(), stride=2)
    else:
        ref = F.conv3d(xt, wt, bias.double(), stride=stride, padding=pad)
    ref = torch.relu(ref).permute(0, 2, 3, 4, 1)
    assert rel_err(out32, ref) < 1e-5, rel_err(out32, ref)
    assert rel_err(out16[..., 8:8 + cout].float(), ref) < 8e-3
    assert float(out16[..., :8].abs().max()) == 0 and float(out16[..., 8 + cout:].abs().max()) == 0


@pytest.mark.parametrize('entry', ['ffx_conv_forward', 'ffx_conv_forward_tc'])
@pytest.mark.parametrize('kind', ['conv3', 'conv3_concat', 'down', 'up', 'head', 'wide'])
def test_forward_entries_match_torch(lib, kind, entry):
    """Both forward implementations (mma.sync and tcgen05 with the accumulator
    in tensor memory) against torch FP64 on the same BF16 values, for every
    form and each output tile width (16, 32, 64 channels; 'wide' spans two
    column tiles), with a ragged voxel count."""
    g = torch.Generator().manual_seed(11)
    B, D, H, W = 1, 6, 10, 12          # 720 voxels: not a multiple of the 128-row tile
    c1, c2, cout = {'conv3': (16, 0, 16), 'conv3_concat': (16, 16, 32), 'down': (32, 0, 64), 'up': (64, 0, 32),
                    'head': (16, 0, 8), 'wide': (24, 0, 72)}[kind]
    cin = c1 + c2
    ind = (D // 2, H // 2, W // 2) if kind == 'up' else (D, H, W)
    outd = {'down': (D // 2, H // 2, W // 2), 'up': (D, H, W)}.get(kind, (D, H, W))
    taps = {'down': 8, 'up': 8, 'head': 1}.get(kind, 27)
    x1 = bf(torch.randn((B, *ind, c1), generator=g))
    x2 = bf(torch.randn((B, *ind, c2), generator=g)) if c2 else None
    w = bf(torch.randn((taps, cin, cout), generator=g) / (taps * cin) ** 0.5)
    bias = torch.randn(cout, generator=g)
    dx1, dx2, dw, db = x1.cuda(), (x2.cuda() if x2 is not None else None), w.cuda(), bias.cuda()
    out32 = torch.zeros((B, *outd, cout), device='cuda')
    ks, stride, pad = {'down': (2, 2, 0), 'up': (2, 2, 0), 'head': (1, 1, 0)}.get(kind, (3, 1, 1))
    c = conv_struct(B, ind, outd, c1, c2, cout, ks, stride, pad, int(kind == 'up'), dx1, c1, 0, dx2, c2, 0, dw,
                    db, 0, None, 0, 0, out32, cout)
    N.check(getattr(lib, entry)(C.byref(c), None))
    torch.cuda.synchronize()
    count = C.c_int32(0)
    N.check(lib.ffx_conv_timeouts(C.byref(count), 1))
    assert count.value == 0
    xin = x1.double()
    if x2 is not None:
        xin = torch.cat([xin, x2.double()], -1)
    xt = xin.permute(0, 4, 1, 2, 3)
    wt = U.torch_weight('up' if kind == 'up' else {'head': 'head', 'down': 'down'}.get(kind, 'conv3'), w.double())
    if kind == 'up':
        ref = F.conv_transpose3d(xt, wt, bias.double(), stride=2)
    else:
        ref = F.conv3d(xt, wt, bias.double(), stride=stride, padding=pad)
    ref = ref.permute(0, 2, 3, 4, 1)
    assert rel_err(out32, ref) < 1e-5, rel_err(out32, ref)


@pytest.mark.parametrize('case', [
    # (batch, (D, H, W), cin, cout, view, bf16 output, accumulate)
    (1, (5, 20, 12), 8, 16, False, False, 0),      # cin 8: one plane, ragged tiles in every axis
    (2, (6, 10, 12), 16, 16, True, True, 1),       # input and output views, ReLU, accumulate
    (1, (8, 16, 16), 32, 32, False, True, 0),
    (1, (4, 16, 8), 64, 64, False, False, 0),      # four channel groups through the stage ring
    (1, (8, 8, 8), 128, 128, True, True, 0),       # two 64-channel column blocks, eight groups
    (2, (3, 7, 9), 32, 48, False, False, 0),       # 16-channel columns, grid smaller than one tile
])
def test_tma_convolution_matches_torch(lib, case):
    """The 3x3x3 TMA-staged tcgen05 convolution against torch FP64 on the
    same BF16 values: every channel width it tiles, ragged grids smaller and
    larger than the 8 x 16 x bz tile, channel views, and the BF16 epilogue
    (bias, ReLU, accumulation into the existing output)."""
    B, (D, H, W), cin, cout, view, out_bf16, acc = case
    g = torch.Generator().manual_seed(cin * 7 + cout)
    pitch, off = (cin + 16, 8) if view else (cin, 0)
    x = bf(torch.randn((B, D, H, W, pitch), generator=g))
    w = bf(torch.randn((27, cin, cout), generator=g) / (27 * cin) ** 0.5)
    bias = torch.randn(cout, generator=g)
    dx, dw, db = x.cuda(), w.cuda(), bias.cuda()
    opitch, ooff = (cout + 16, 8) if view else (cout, 0)
    prior = bf(torch.randn((B, D, H, W, opitch), generator=g))
    out16 = prior.clone().cuda()
    out32 = torch.zeros((B, D, H, W, cout), device='cuda')
    relu = int(out_bf16)
    c = conv_struct(B, (D, H, W), (D, H, W), cin, 0, cout, 3, 1, 1, 0, dx, pitch, off, None, 0, 0, dw, db, relu,
                    out16 if out_bf16 else None, opitch, ooff, None if out_bf16 else out32, cout, accumulate=acc)
    nbytes = N.i64(0)
    N.check(lib.ffx_conv_packed_bytes(C.byref(c), C.byref(nbytes)))
    assert nbytes.value == ((cin + 15) // 16) * 27 * 16 * cout * 2
    packed = torch.zeros(nbytes.value // 2, dtype=torch.bfloat16, device='cuda')
    N.check(lib.ffx_conv_pack_weights(C.byref(c), C.c_void_p(packed.data_ptr()), None))
    N.check(lib.ffx_conv_forward_tma(C.byref(c), C.c_void_p(packed.data_ptr()), None))
    torch.cuda.synchronize()
    count = C.c_int32(0)
    N.check(lib.ffx_conv_timeouts(C.byref(count), 1))
    assert count.value == 0
    xt = x[..., off:off + cin].double().permute(0, 4, 1, 2, 3)
    ref = F.conv3d(xt, U.torch_weight('conv3', w.double()), bias.double(), padding=1).permute(0, 2, 3, 4, 1)
    if relu:
        ref = torch.relu(ref)
    if not out_bf16:
        assert rel_err(out32, ref) < 1e-5, rel_err(out32, ref)
        return
    if acc:
        ref = ref + prior[..., ooff:ooff + cout].double()
    got = out16.cpu()
    assert rel_err(got[..., ooff:ooff + cout].float(), ref) < 8e-3, rel_err(got[..., ooff:ooff + cout].float(), ref)
    # channels outside the output view are untouched
    assert torch.equal(got[..., :ooff], prior[..., :ooff]) and torch.equal(got[..., ooff + cout:],
                                                                            prior[..., ooff + cout:])


def test_tma_convolution_other_shapes_use_the_gather_kernel(lib):
    """Shapes the TMA kernel does not tile report no packed size and run the
    mma.sync kernel through the same entry (packed pointer ignored)."""
    g = torch.Generator().manual_seed(3)
    x = bf(torch.randn((1, 8, 8, 8, 16), generator=g)).cuda()
    w = bf(torch.randn((8, 16, 32), generator=g) / 11.0).cuda()
    out32 = torch.zeros((1, 4, 4, 4, 32), device='cuda')
    c = conv_struct(1, (8, 8, 8), (4, 4, 4), 16, 0, 32, 2, 2, 0, 0, x, 16, 0, None, 0, 0, w, None, 0, None, 0, 0,
                    out32, 32)
    nbytes = N.i64(-1)
    N.check(lib.ffx_conv_packed_bytes(C.byref(c), C.byref(nbytes)))
    assert nbytes.value == 0
    assert lib.ffx_conv_pack_weights(C.byref(c), None, None) != 0
    N.check(lib.ffx_conv_forward_tma(C.byref(c), None, None))
    torch.cuda.synchronize()
    ref = F.conv3d(x.double().cpu().permute(0, 4, 1, 2, 3), U.torch_weight('down', w.double().cpu()), stride=2)
    assert rel_err(out32, ref.permute(0, 2, 3, 4, 1)) < 1e-5


@pytest.mark.parametrize('case', [
    # (kind, cin, cout, bf16 output, relu, accumulate)
    ('head', 16, 8, False, 0, 0),      # the network's head: FP32 output
    ('head', 8, 16, True, 0, 1),       # the head's data gradient form, accumulated into a view
    ('up', 32, 16, True, 1, 0),        # up-sampling to the finest level
    ('up', 32, 16, True, 0, 1),        # the down-sampling's data gradient (accumulated)
])
def test_narrow_convolutions_match_torch(lib, case):
    """1^3 and transposed 2^3 convolutions with 8 or 16 output channels run the
    per-voxel kernel through the TMA entry point: against torch FP64 on the
    same BF16 values, with ragged grids, channel views, bias, ReLU and
    accumulation into the existing output."""
    kind, cin, cout, out_bf16, relu, acc = case
    g = torch.Generator().manual_seed(cin + 3 * cout + acc)
    B, D, H, W = 2, 6, 10, 14
    ind = (D // 2, H // 2, W // 2) if kind == 'up' else (D, H, W)
    outd = (D, H, W)
    taps = 8 if kind == 'up' else 1
    pitch, off = cin + 8, 8
    x = bf(torch.randn((B, *ind, pitch), generator=g))
    w = bf(torch.randn((taps, cin, cout), generator=g) / (taps * cin) ** 0.5)
    bias = torch.randn(cout, generator=g)
    opitch, ooff = cout + 16, 8
    prior = bf(torch.randn((B, *outd, opitch), generator=g))
    out16 = prior.clone().cuda()
    out32 = torch.zeros((B, *outd, cout), device='cuda')
    dx, dw, db = x.cuda(), w.cuda(), bias.cuda()
    ks, stride = (2, 2) if kind == 'up' else (1, 1)
    c = conv_struct(B, ind, outd, cin, 0, cout, ks, stride, 0, int(kind == 'up'), dx, pitch, off, None, 0, 0, dw, db,
                    relu, out16 if out_bf16 else None, opitch, ooff, None if out_bf16 else out32, cout,
                    accumulate=acc)
    nbytes = N.i64(-1)
    N.check(lib.ffx_conv_packed_bytes(C.byref(c), C.byref(nbytes)))
    assert nbytes.value == 0
    N.check(lib.ffx_conv_forward_tma(C.byref(c), None, None))
    torch.cuda.synchronize()
    xt = x[..., off:off + cin].double().permute(0, 4, 1, 2, 3)
    wt = U.torch_weight('up' if kind == 'up' else 'head', w.double())
    if kind == 'up':
        ref = F.conv_transpose3d(xt, wt, bias.double(), stride=2)
    else:
        ref = F.conv3d(xt, wt, bias.double())
    ref = ref.permute(0, 2, 3, 4, 1)
    if relu:
        ref = torch.relu(ref)
    if not out_bf16:
        assert rel_err(out32, ref) < 1e-5, rel_err(out32, ref)
        return
    if acc:
        ref = ref + prior[..., ooff:ooff + cout].double()
    got = out16.cpu()
    assert rel_err(got[..., ooff:ooff + cout].float(), ref) < 8e-3
    assert torch.equal(got[..., :ooff], prior[..., :ooff]) and torch.equal(got[..., ooff + cout:],
                                                                            prior[..., ooff + cout:])


@pytest.mark.parametrize('kind', ['conv3', 'down', 'up'])
def test_weight_gradients_match_torch(lib, kind):
    g = torch.Generator().manual_seed(2)
    B, D, H, W = 2, 8, 12, 8
    cin, cout = (16, 32) if kind != 'up' else (32, 16)
    ind = (D // 2, H // 2, W // 2) if kind == 'up' else (D, H, W)
    outd = (D // 2, H // 2, W // 2) if kind == 'down' else (D, H, W)
    taps = 27 if kind == 'conv3' else 8
    x = bf(torch.randn((B, *ind, cin), generator=g))
    gy = bf(torch.randn((B, *outd, cout), generator=g))
    w = bf(torch.randn((taps, cin, cout), generator=g))
    dw = torch.zeros((taps, cin, cout), device='cuda')
    ks, stride, pad = (3, 1, 1) if kind == 'conv3' else (2, 2, 0)
    xcu, wcu, gcu = x.cuda(), w.cuda(), gy.cuda()     # kept alive until the kernels have run
    c = conv_struct(B, ind, outd, cin, 0, cout, ks, stride, pad, int(kind == 'up'), xcu, cin, 0, None, 0, 0,
                    wcu, None, 0, None, 0, 0, None, 0)
    N.check(lib.ffx_conv_weight_grad(C.byref(c), C.c_void_p(gcu.data_ptr()), cout, C.c_void_p(dw.data_ptr()), None))
    db = torch.zeros(cout, device='cuda')
    N.check(lib.ffx_bias_grad(B * outd[0] * outd[1] * outd[2], cout, C.c_void_p(gcu.data_ptr()), cout,
                              C.c_void_p(db.data_ptr()), None))
    torch.cuda.synchronize()
    wl = w.double().requires_grad_(True)
    bl = torch.zeros(cout, dtype=torch.float64, requires_grad=True)
    xt = x.double().permute(0, 4, 1, 2, 3)
    wt = U.torch_weight('up' if kind == 'up' else ('down' if kind == 'down' else 'conv3'), wl)
    y = F.conv_transpose3d(xt, wt, bl, stride=2) if kind == 'up' else F.conv3d(xt, wt, bl, stride=stride, padding=pad)
    (y * gy.double().permute(0, 4, 1, 2, 3)).sum().backward()
    assert rel_err(dw, wl.grad) < 1e-4, rel_err(dw, wl.grad)
    assert rel_err(db, bl.grad) < 1e-4


@pytest.mark.parametrize('zero', [False, True])
def test_device_scaled_input_and_output_match_host_scaling(lib, zero):
    """The network's input packing and output unpacking with the scale read on
    the device from max|div| give the host-scaled results bit for bit (and a
    zero guess for a zero divergence)."""
    g = torch.Generator().manual_seed(9)
    n = 4096
    div = torch.zeros(n) if zero else torch.randn(n, generator=g) * 3.0
    mask = (torch.rand(n, generator=g) < 0.2).to(torch.uint8)
    ddiv, dmask = div.cuda(), mask.cuda()
    mx = torch.zeros(1, device='cuda')
    N.check(lib.ffx_max_abs(n, N.FFX_F32, C.c_void_p(ddiv.data_ptr()), C.c_void_p(mx.data_ptr()), None))
    torch.cuda.synchronize()
    m = float(mx.item())
    a = torch.zeros((n, 8), dtype=torch.bfloat16, device='cuda')
    b = torch.zeros_like(a)
    N.check(lib.ffx_pack_input(n, C.c_void_p(ddiv.data_ptr()), C.c_void_p(dmask.data_ptr()),
                               (1.0 / m) if m else 0.0, C.c_void_p(a.data_ptr()), None))
    N.check(lib.ffx_pack_input_scaled(n, C.c_void_p(ddiv.data_ptr()), C.c_void_p(dmask.data_ptr()),
                                      C.c_void_p(mx.data_ptr()), C.c_void_p(b.data_ptr()), None))
    src = torch.randn((n, 8), generator=g).cuda()
    weight = 16384.0
    u1, u2 = torch.full((n,), 7.0, device='cuda'), torch.full((n,), 7.0, device='cuda')
    N.check(lib.ffx_unpack_channel(n, C.c_void_p(src.data_ptr()), 8, (1.0 / ((1.0 / m) * weight)) if m else 0.0,
                                   C.c_void_p(u1.data_ptr()), None))
    N.check(lib.ffx_unpack_channel_scaled(n, C.c_void_p(src.data_ptr()), 8, C.c_void_p(mx.data_ptr()), weight,
                                          C.c_void_p(u2.data_ptr()), None))
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    assert torch.equal(u1, u2)
    if zero:
        assert float(u2.abs().max()) == 0.0


def test_adam_matches_formula(lib):
    n = 1000
    g = torch.Generator().manual_seed(3)
    w, m, v, gr = (torch.randn(n, generator=g) for _ in range(4))
    v = v.abs()
    dw, dm, dv, dg = w.cuda(), m.cuda(), v.cuda(), gr.cuda()
    w16 = torch.zeros(n, dtype=torch.bfloat16, device='cuda')
    ptr = lambda t: C.c_void_p(t.data_ptr())
    N.check(lib.ffx_adam(n, ptr(dw), ptr(dm), ptr(dv), ptr(dg), ptr(w16), 1e-3, 0.9, 0.999, 1e-8, 3, None))
    torch.cuda.synchronize()
    m2 = 0.9 * m + 0.1 * gr
    v2 = 0.999 * v + 0.001 * gr * gr
    w2 = w - 1e-3 * (m2 / (1 - 0.9 ** 3)) / ((v2 / (1 - 0.999 ** 3)).sqrt() + 1e-8)
    assert rel_err(dw, w2) < 1e-6 and rel_err(dm, m2) < 1e-6 and rel_err(dv, v2) < 1e-6
    assert rel_err(w16.float(), w2) < 1e-2


@pytest.mark.parametrize('entry', ['ffx_conv_forward', 'ffx_conv_forward_tc', 'ffx_conv_forward_tma'])
def test_unet_forward_and_gradients_match_oracle(entry):
    from fluxfx_b200.learned.unet import UNet
    dev = torch.device('cuda')
    net = UNet(dev, seed=4)
    net.conv_entry = entry
    g = torch.Generator().manual_seed(5)
    B, D = 2, 16
    div = torch.randn((B, D, D, D), generator=g)
    mask = (torch.rand((B, D, D, D), generator=g) < 0.1).to(torch.uint8)
    target = torch.randn((B, D, D, D), generator=g)
    stream = torch.cuda.current_stream().cuda_stream
    pred = net.forward(div.cuda(), mask.cuda(), 0.5, stream)
    loss = net.loss_backward(target.cuda(), mask.cuda(), stream)
    torch.cuda.synchronize()
    x = torch.zeros((B, 8, D, D, D), dtype=torch.float64)
    x[:, 0] = (0.5 * div).to(torch.bfloat16).double()
    x[:, 1] = mask.double()
    rpred, rloss, _ = U.loss_and_grads(net.layers, x, target.double(), mask.bool())
    # BF16 activations: the device and the oracle round the same values, but
    # FP32-vs-FP64 accumulation can flip a rounding, which then propagates.
    assert rel_err(pred, rpred) < 3e-2, rel_err(pred, rpred)
    assert float(loss[0]) == pytest.approx(rloss, rel=5e-2)
    # A rounding flip next to zero also flips a ReLU, which zeroes or keeps a
    # whole gradient element; with a fraction f of flipped voxels the L2 error
    # of every gradient upstream grows like sqrt(f). So the gradients are
    # checked with the device's own ReLU pattern, leaving only the BF16
    # rounding of activations and of their gradients (both modelled).
    masks = {l.name: (net.activation(l.name) > 0).permute(0, 4, 1, 2, 3).cpu() for l in net.layers if l.relu}
    _, _, grads = U.loss_and_grads(net.layers, x, target.double(), mask.bool(), relu_masks=masks)
    errs = {l.name: (rel_l2(l.gw, grads[l.name][0]), rel_l2(l.gb, grads[l.name][1])) for l in net.layers}
    for name, (ew, eb) in errs.items():
        assert ew < 2e-2 and eb < 2e-2, (name, errs)


@pytest.mark.parametrize('kind', ['conv3', 'down', 'up', 'head'])
def test_data_gradients_match_torch(lib, kind):
    """The backward-data convolutions as the network issues them: the flipped
    transpose of a 3^3 kernel, the transposed 2^3 stride-2 form for a
    down-sampling, the 2^3 stride-2 form for an up-sampling, and the head."""
    from fluxfx_b200.learned.unet import Layer
    g = torch.Generator().manual_seed(8)
    B, D, H, W = 2, 8, 8, 16
    cin, cout = {'conv3': (16, 32), 'down': (16, 32), 'up': (32, 16), 'head': (16, 8)}[kind]
    layer = Layer('t', kind, cin, cout, True, 'cuda', g)
    ind = (D // 2, H // 2, W // 2) if kind == 'up' else (D, H, W)
    outd = (D // 2, H // 2, W // 2) if kind == 'down' else (D, H, W)
    gy = bf(torch.randn((B, *outd, cout), generator=g))
    gcu = gy.cuda()
    gin = torch.zeros((B, *ind, cin + 8), dtype=torch.bfloat16, device='cuda')   # a view at offset 8
    flip = int(kind == 'conv3')
    N.check(lib.ffx_weight_transpose(layer.taps, cin, cout, flip, C.c_void_p(layer.w16.data_ptr()),
                                     C.c_void_p(layer.wt16.data_ptr()), None))
    ks, stride, pad, tr = {'conv3': (3, 1, 1, 0), 'down': (2, 2, 0, 1), 'up': (2, 2, 0, 0), 'head': (1, 1, 0, 0)}[kind]
    c = conv_struct(B, outd, ind, cout, 0, cin, ks, stride, pad, tr, gcu, cout, 0, None, 0, 0, layer.wt16, None, 0,
                    gin, cin + 8, 8, None, 0)
    N.check(lib.ffx_conv_forward(C.byref(c), None))
    torch.cuda.synchronize()
    x = torch.zeros((B, cin, *ind), dtype=torch.float64, requires_grad=True)
    wt = U.torch_weight(kind, layer.w16.double().cpu())
    if kind == 'up':
        y = F.conv_transpose3d(x, wt, stride=2)
    else:
        y = F.conv3d(x, wt, stride=stride, padding=pad)
    (y * gy.double().permute(0, 4, 1, 2, 3)).sum().backward()
    ref = x.grad.permute(0, 2, 3, 4, 1)
    assert rel_err(gin[..., 8:].float(), ref) < 8e-3, rel_err(gin[..., 8:].float(), ref)
    assert float(gin[..., :8].abs().max()) == 0


def test_training_steps_reduce_the_loss():
    from fluxfx_b200.learned.unet import UNet
    dev = torch.device('cuda')
    net = UNet(dev, seed=6)
    g = torch.Generator().manual_seed(7)
    B, D = 2, 16
    div = torch.randn((B, D, D, D), generator=g).cuda()
    target = (0.3 * div).contiguous()
    stream = torch.cuda.current_stream().cuda_stream
    losses = []
    for _ in range(30):
        net.forward(div, None, 1.0, stream)
        losses.append(float(net.loss_backward(target, None, stream)[0]))
        net.adam_step(3e-3, stream)
    assert losses[-1] < 0.5 * losses[0], losses


def test_trained_network_saves_v_cycles():
    """The packaged network (trained on the GPU by fluxfx_b200.learned.train)
    as the plain solver's initial guess on a held-out 128^3 collider scene:
    the same tolerance is reached in fewer V-cycles than from zero."""
    from dataclasses import replace

    from fluxfx_b200.backend.device import CudaDevice
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    from fluxfx_b200.learned import attach
    from fluxfx_b200.learned.train import scene
    results = {}
    for learned in (False, True):
        grid, settings, colliders, emitters, noise = scene(128, 777)   # seed outside training and evaluation
        s = DenseProjectedSmoke(grid, replace(settings, learned_warm_start=learned), CudaDevice(),
                                colliders=colliders)
        if learned:
            attach(s, colliders)
        s.upload(torch.zeros(grid.cells))
        s.upload_temperature(torch.zeros(grid.cells))
        s.upload_velocity([torch.as_tensor(v) for v in noise])
        dt, cycles = 0.02, []
        for _ in range(12):
            s.step(dt, sources=emitters)
            cycles.append(s.projector.last_cycles)
            umax = max(s.projector.velocity_maxima())
            dt = min(0.02, 0.5 / 128 / umax) if umax > 0 else 0.02
        assert s.projector.metrics()['rel_div_inf'] <= 1e-4
        results[learned] = cycles
        s.close()
    plain, warm = sum(results[False][4:]), sum(results[True][4:])
    assert warm <= 0.8 * plain, results

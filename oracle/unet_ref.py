"""CPU oracle of the learned warm start -- TEST INFRASTRUCTURE ONLY.

The U-Net of ``fluxfx_b200/learned/unet.py`` restated with torch CPU autograd
in FP64 (``conv3d`` / ``conv_transpose3d``, channels-first), from the same
BF16-rounded weights. With ``round_activations`` every layer output is rounded
to bfloat16 as the device stores it, so forward results agree to the
accumulation-order level. The reference has no learned component, so this
oracle is pinned to torch's own convolution definitions, not to the reference.
"""
import torch
import torch.nn.functional as F

LAYERS = ('e0a', 'e0b', 'd0', 'e1a', 'e1b', 'd1', 'e2a', 'e2b', 'd2', 'e3a', 'e3b', 'u2', 'c2a', 'c2b', 'u1', 'c1a',
          'c1b', 'u0', 'c0a', 'c0b', 'head')


def _round(x):
    return x.to(torch.bfloat16).to(torch.float64)


class _RoundBoth(torch.autograd.Function):
    """BF16 rounding of an activation and of the gradient that flows back into
    it (the device stores both in bfloat16)."""

    @staticmethod
    def forward(ctx, x):
        return _round(x)

    @staticmethod
    def backward(ctx, g):
        return _round(g)


class _RoundGrad(torch.autograd.Function):
    """Identity whose backward rounds the gradient to BF16."""

    @staticmethod
    def forward(ctx, x):
        return x.clone()

    @staticmethod
    def backward(ctx, g):
        return _round(g)


def forward(params, x, round_activations=True, relu_masks=None):
    """params: {name: (kind, w [taps][cin][cout], b [cout])} as leaf tensors
    (float64, requires_grad as wanted); x: (B, 8, D, H, W) float64. Returns the
    prediction (B, D, H, W). With `relu_masks` ({layer: bool (B, C, D, H, W)})
    the ReLUs keep exactly the given voxels instead of the positive ones, so a
    comparison with the device can share its activation pattern."""
    r = _RoundBoth.apply if round_activations else (lambda t: t)

    def conv(name, t):
        kind, w, b = params[name]
        wt = torch_weight(kind, w)
        if kind == 'up':
            y = F.conv_transpose3d(t, wt, b, stride=2)
        elif kind == 'down':
            y = F.conv3d(t, wt, b, stride=2)
        elif kind == 'head':
            y = F.conv3d(t, wt, b)
        else:
            y = F.conv3d(t, wt, b, padding=1)
        if kind == 'head':
            return y
        y = torch.relu(y) if relu_masks is None else y * relu_masks[name]
        return r(y)

    e0 = conv('e0b', conv('e0a', x))
    e1 = conv('e1b', conv('e1a', conv('d0', e0)))
    e2 = conv('e2b', conv('e2a', conv('d1', e1)))
    e3 = conv('e3b', conv('e3a', conv('d2', e2)))
    c2 = conv('c2b', conv('c2a', torch.cat([conv('u2', e3), e2], 1)))
    c1 = conv('c1b', conv('c1a', torch.cat([conv('u1', c2), e1], 1)))
    c0 = conv('c0b', conv('c0a', torch.cat([conv('u0', c1), e0], 1)))
    return conv('head', c0)[:, 0]


def torch_weight(kind, w):
    """[taps][cin][cout] -> the torch convolution layout (differentiable)."""
    taps, cin, cout = w.shape
    if kind == 'up':
        return w.permute(1, 2, 0).reshape(cin, cout, 2, 2, 2)
    k = {27: 3, 8: 2, 1: 1}[taps]
    return w.permute(2, 1, 0).reshape(cout, cin, k, k, k)


def loss_and_grads(net_layers, x, target, mask, relu_masks=None):
    """MSE over fluid voxels and the gradients of every weight and bias. The
    gradient of the prediction is rounded to BF16 as the device stores it."""
    params = {}
    for l in net_layers:
        w = l.w.detach().cpu().to(torch.bfloat16).to(torch.float64).requires_grad_(True)
        b = l.b.detach().cpu().to(torch.float64).requires_grad_(True)
        params[l.name] = (l.kind, w, b)
    pred = forward(params, x, relu_masks=relu_masks)
    fluid = torch.ones_like(target, dtype=torch.bool) if mask is None else ~mask
    count = int(fluid.sum())
    loss = (((_RoundGrad.apply(pred) - target) ** 2) * fluid).sum() / count
    loss.backward()
    return pred.detach(), float(loss.detach()), {n: (p[1].grad, p[2].grad) for n, p in params.items()}

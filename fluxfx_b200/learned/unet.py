"""3D U-Net pressure warm start on the library's BF16 tensor-core convolutions.

No counterpart in the reference: the network maps (divergence, solid mask)
to a pressure that replaces the zero initial guess of the multigrid solve;
the solver still iterates to the same tolerance, so the plain method stays
both the fallback and the arbiter of the prediction.

Architecture (4 levels, channels 16/32/64/128): per level two 3^3 convolutions
with ReLU; 2^3 stride-2 convolutions (+ReLU) down; 2^3 stride-2 transposed
convolutions (+ReLU) up, concatenated with the skip connection of the level;
a 1^3 head to one channel. Activations are NDHWC bfloat16; weights are kept
as FP32 masters (Adam) with BF16 copies for the kernels; biases are FP32.
The decoder's concatenation buffers are written in place by both producers
(up-sampling into channels [0, C), the encoder's second convolution into
[C, 2C)), and their gradients likewise, so no copies are made.

All work runs through ``libffx_core`` (``ffx_conv_forward_tma`` with
``ffx_conv_pack_weights``, ``ffx_conv_forward``, ``ffx_conv_weight_grad``,
``ffx_relu_backward``, ``ffx_bias_grad``, ``ffx_weight_transpose``,
``ffx_adam``, ``ffx_pack_input``, ``ffx_mse_grad``); torch only allocates.
The 3^3 layers (forward and data gradient) run on the TMA-staged tcgen05
convolution by default; the stride-2, transposed and 1^3 layers on the
mma.sync implicit GEMM.
"""
import ctypes as C

import torch

from .. import _native as N

CHANNELS = (16, 32, 64, 128)
IN_CHANNELS = 8          # divergence, mask, six zero channels (the kernels read channels in groups of 8)
HEAD_CHANNELS = 8        # output channel 0 is the pressure; 1..7 stay zero


def _p(t):
    return C.c_void_p(0 if t is None else t.data_ptr())


def _view(t, pitch, offset=0):
    return N.FfxTensorView(t.data_ptr() if t is not None else None, pitch, offset)


class Layer:
    """One convolution: kind 'conv3' (3^3, pad 1), 'down' (2^3 stride 2),
    'up' (transposed 2^3 stride 2) or 'head' (1^3); weight [taps][cin][cout]."""

    def __init__(self, name, kind, cin, cout, relu, device, gen):
        self.name, self.kind, self.cin, self.cout, self.relu = name, kind, cin, cout, relu
        self.taps = {'conv3': 27, 'down': 8, 'up': 8, 'head': 1}[kind]
        fan_in = self.taps * cin if kind != 'up' else cin
        w = torch.randn((self.taps, cin, cout), generator=gen, dtype=torch.float32) * (2.0 / fan_in) ** 0.5
        if kind == 'head':
            w[:, :, 1:] = 0.0
        self.w = w.to(device)
        self.b = torch.zeros(cout, dtype=torch.float32, device=device)
        self.w16 = self.w.to(torch.bfloat16)
        self.wt16 = torch.empty((self.taps, cout, cin), dtype=torch.bfloat16, device=device)   # data-gradient weights
        self.gw = torch.zeros_like(self.w)
        self.gb = torch.zeros_like(self.b)
        self.mw, self.vw = torch.zeros_like(self.w), torch.zeros_like(self.w)
        self.mb, self.vb = torch.zeros_like(self.b), torch.zeros_like(self.b)

    def params(self):
        return [(self.w, self.mw, self.vw, self.gw, self.w16), (self.b, self.mb, self.vb, self.gb, None)]


class UNet:
    """Parameters, activation buffers for one (batch, D, H, W), forward,
    backward and Adam. D, H, W must be divisible by 8."""

    def __init__(self, device, seed=0, lib=None):
        self.device = device
        self.lib = lib or N.load()
        gen = torch.Generator().manual_seed(seed)
        c0, c1, c2, c3 = CHANNELS
        spec = [('e0a', 'conv3', IN_CHANNELS, c0, True), ('e0b', 'conv3', c0, c0, True), ('d0', 'down', c0, c1, True),
                ('e1a', 'conv3', c1, c1, True), ('e1b', 'conv3', c1, c1, True), ('d1', 'down', c1, c2, True),
                ('e2a', 'conv3', c2, c2, True), ('e2b', 'conv3', c2, c2, True), ('d2', 'down', c2, c3, True),
                ('e3a', 'conv3', c3, c3, True), ('e3b', 'conv3', c3, c3, True),
                ('u2', 'up', c3, c2, True), ('c2a', 'conv3', 2 * c2, c2, True), ('c2b', 'conv3', c2, c2, True),
                ('u1', 'up', c2, c1, True), ('c1a', 'conv3', 2 * c1, c1, True), ('c1b', 'conv3', c1, c1, True),
                ('u0', 'up', c1, c0, True), ('c0a', 'conv3', 2 * c0, c0, True), ('c0b', 'conv3', c0, c0, True),
                ('head', 'head', c0, HEAD_CHANNELS, False)]
        self.layers = [Layer(*s, device=device, gen=gen) for s in spec]
        self.by_name = {l.name: l for l in self.layers}
        self.shape = None
        self.step_count = 0
        # forward and data-gradient convolutions: 'ffx_conv_forward' (mma.sync,
        # gathered operands), 'ffx_conv_forward_tc' (tcgen05, gathered operands)
        # or 'ffx_conv_forward_tma' (3x3x3 layers as TMA halo tiles + tcgen05 on
        # pre-packed weights, the other shapes on the mma.sync kernel; the default)
        self.conv_entry = 'ffx_conv_forward_tma'
        self.weight_version = 0      # bumped when the weights change (repacks the TMA weights)
        self.calls = 0               # library calls issued (each launches one kernel)
        self._packs = {}

    # ------------------------------------------------------------- buffers
    def _buffers(self, batch, dims):
        if self.shape == (batch, dims):
            return
        D, H, W = dims
        if D % 8 or H % 8 or W % 8:
            raise ValueError('U-Net grid dimensions must be divisible by 8')
        c = CHANNELS
        dev = self.device

        def act(level, ch):
            s = 2 ** level
            return torch.zeros((batch, D // s, H // s, W // s, ch), dtype=torch.bfloat16, device=dev)

        self.dims = [(D // 2 ** k, H // 2 ** k, W // 2 ** k) for k in range(4)]
        self.x = act(0, IN_CHANNELS)
        a = {}
        a['e0a'] = act(0, c[0])
        a['cat0'] = act(0, 2 * c[0])        # [u0 | e0b]
        a['d0'] = act(1, c[1])
        a['e1a'] = act(1, c[1])
        a['cat1'] = act(1, 2 * c[1])
        a['d1'] = act(2, c[2])
        a['e2a'] = act(2, c[2])
        a['cat2'] = act(2, 2 * c[2])
        a['d2'] = act(3, c[3])
        a['e3a'] = act(3, c[3])
        a['e3b'] = act(3, c[3])
        a['c2a'] = act(2, c[2])
        a['c2b'] = act(2, c[2])
        a['c1a'] = act(1, c[1])
        a['c1b'] = act(1, c[1])
        a['c0a'] = act(0, c[0])
        a['c0b'] = act(0, c[0])
        self.act = a
        self.grad = {k: torch.zeros_like(v) for k, v in a.items()}
        self.pred = torch.zeros((batch, D, H, W, HEAD_CHANNELS), dtype=torch.float32, device=dev)
        self.dpred = torch.zeros((batch, D, H, W, HEAD_CHANNELS), dtype=torch.bfloat16, device=dev)
        self.loss_acc = torch.zeros(1, dtype=torch.float64, device=dev)
        self.shape = (batch, dims)
        self.batch = batch
        # (layer, level_in, input views, level_out, output tensor, out pitch, out offset)
        c0, c1, c2, c3 = c
        A = a
        self.graph = [
            ('e0a', 0, [(self.x, IN_CHANNELS, 0, IN_CHANNELS)], 0, A['e0a'], c0, 0),
            ('e0b', 0, [(A['e0a'], c0, 0, c0)], 0, A['cat0'], 2 * c0, c0),
            ('d0', 0, [(A['cat0'], 2 * c0, c0, c0)], 1, A['d0'], c1, 0),
            ('e1a', 1, [(A['d0'], c1, 0, c1)], 1, A['e1a'], c1, 0),
            ('e1b', 1, [(A['e1a'], c1, 0, c1)], 1, A['cat1'], 2 * c1, c1),
            ('d1', 1, [(A['cat1'], 2 * c1, c1, c1)], 2, A['d1'], c2, 0),
            ('e2a', 2, [(A['d1'], c2, 0, c2)], 2, A['e2a'], c2, 0),
            ('e2b', 2, [(A['e2a'], c2, 0, c2)], 2, A['cat2'], 2 * c2, c2),
            ('d2', 2, [(A['cat2'], 2 * c2, c2, c2)], 3, A['d2'], c3, 0),
            ('e3a', 3, [(A['d2'], c3, 0, c3)], 3, A['e3a'], c3, 0),
            ('e3b', 3, [(A['e3a'], c3, 0, c3)], 3, A['e3b'], c3, 0),
            ('u2', 3, [(A['e3b'], c3, 0, c3)], 2, A['cat2'], 2 * c2, 0),
            ('c2a', 2, [(A['cat2'], 2 * c2, 0, 2 * c2)], 2, A['c2a'], c2, 0),
            ('c2b', 2, [(A['c2a'], c2, 0, c2)], 2, A['c2b'], c2, 0),
            ('u1', 2, [(A['c2b'], c2, 0, c2)], 1, A['cat1'], 2 * c1, 0),
            ('c1a', 1, [(A['cat1'], 2 * c1, 0, 2 * c1)], 1, A['c1a'], c1, 0),
            ('c1b', 1, [(A['c1a'], c1, 0, c1)], 1, A['c1b'], c1, 0),
            ('u0', 1, [(A['c1b'], c1, 0, c1)], 0, A['cat0'], 2 * c0, 0),
            ('c0a', 0, [(A['cat0'], 2 * c0, 0, 2 * c0)], 0, A['c0a'], c0, 0),
            ('c0b', 0, [(A['c0a'], c0, 0, c0)], 0, A['c0b'], c0, 0),
            ('head', 0, [(A['c0b'], c0, 0, c0)], 0, None, 0, 0),
        ]
        # gradient tensor of every activation tensor (same layout)
        self.grad_of = {id(v): self.grad[k] for k, v in A.items()}

    def _conv(self, layer, lin, inp, lout, out, out_pitch, out_offset, *, weight=None, transposed=None, ks=None,
              stride=None, pad=None, cout=None, bias=True, relu=None, accumulate=0, out_f32=None, f32_pitch=0):
        (t, pitch, offset, ch) = inp
        c = N.FfxConv()
        c.batch = self.batch
        c.in_dims = (N.i32 * 3)(*self.dims[lin])
        c.out_dims = (N.i32 * 3)(*self.dims[lout])
        c.c1, c.c2, c.cout = ch, 0, cout if cout is not None else layer.cout
        kind = layer.kind
        c.ksize = ks if ks is not None else {'conv3': 3, 'down': 2, 'up': 2, 'head': 1}[kind]
        c.stride = stride if stride is not None else (2 if kind in ('down', 'up') else 1)
        c.pad = pad if pad is not None else (1 if kind == 'conv3' else 0)
        c.transposed = transposed if transposed is not None else int(kind == 'up')
        c.in1 = _view(t, pitch, offset)
        c.in2 = N.FfxTensorView(None, 0, 0)
        c.weight = (weight if weight is not None else layer.w16).data_ptr()
        c.bias = layer.b.data_ptr() if bias else None
        c.relu = int(layer.relu if relu is None else relu)
        c.accumulate = accumulate
        c.out = out.data_ptr() if out is not None else None
        c.out_pitch, c.out_offset = out_pitch, out_offset
        c.out_f32 = out_f32.data_ptr() if out_f32 is not None else None
        c.out_f32_pitch = f32_pitch
        return c

    def _call(self, name, *args):
        N.check(getattr(self.lib, name)(*args))
        self.calls += 1

    def _run_conv(self, key, c, s):
        """One convolution through the selected entry; the TMA entry gets the
        weights packed once per weight version (and per role: forward weights
        or the transposed data-gradient weights)."""
        if self.conv_entry != 'ffx_conv_forward_tma':
            self._call(self.conv_entry, C.byref(c), s)
            return
        n = N.i64(0)
        N.check(self.lib.ffx_conv_packed_bytes(C.byref(c), C.byref(n)))    # a host query, no launch
        packed = None
        if n.value:
            entry = self._packs.get(key)
            if entry is None or entry[0].numel() * 2 < n.value:
                entry = [torch.empty(n.value // 2, dtype=torch.bfloat16, device=self.device), -1]
                self._packs[key] = entry
            if entry[1] != self.weight_version:
                self._call('ffx_conv_pack_weights', C.byref(c), _p(entry[0]), s)
                entry[1] = self.weight_version
            packed = entry[0]
        self._call('ffx_conv_forward_tma', C.byref(c), _p(packed), s)

    # ------------------------------------------------------------ forward
    def forward(self, div, mask, scale, stream, max_abs=None):
        """div: (B, D, H, W) float32, mask: uint8 or None; returns the FP32
        prediction view (B, D, H, W) (channel 0 of the head output). The input
        is div * scale, or div / max|div| read on the device from `max_abs` (a
        one-element FP32 tensor) when it is given."""
        batch, D, H, W = div.shape
        self._buffers(batch, (D, H, W))
        s = C.c_void_p(stream)
        if max_abs is not None:
            self._call('ffx_pack_input_scaled', div.numel(), _p(div), _p(mask), _p(max_abs), _p(self.x), s)
        else:
            self._call('ffx_pack_input', div.numel(), _p(div), _p(mask), float(scale), _p(self.x), s)
        for name, lin, ins, lout, out, pitch, offset in self.graph:
            layer = self.by_name[name]
            if name == 'head':
                c = self._conv(layer, lin, ins[0], lout, None, 0, 0, out_f32=self.pred, f32_pitch=HEAD_CHANNELS)
            else:
                c = self._conv(layer, lin, ins[0], lout, out, pitch, offset)
            self._run_conv((name, 'forward'), c, s)
        return self.pred[..., 0]

    def activation(self, name):
        """The stored output of layer `name` as a (B, D, H, W, C) bfloat16 view
        (the head's FP32 output for 'head')."""
        if name == 'head':
            return self.pred
        for n, _, _, _, out, pitch, offset in self.graph:
            if n == name:
                return out[..., offset:offset + self.by_name[name].cout]
        raise KeyError(name)

    # ------------------------------------------------------------ backward
    def loss_backward(self, target, mask, stream):
        """MSE against `target` over fluid voxels, then gradients of every
        parameter (accumulated into layer.gw / layer.gb, zeroed here first)."""
        s = C.c_void_p(stream)
        count = target.numel() if mask is None else int(target.numel() - int(mask.sum()))
        self.loss_acc.zero_()
        self._call('ffx_mse_grad', target.numel(), _p(self.pred), HEAD_CHANNELS, _p(target), _p(mask),
                   1.0 / max(count, 1), _p(self.dpred), _p(self.loss_acc), s)
        for l in self.layers:
            l.gw.zero_()
            l.gb.zero_()
        for g in self.grad.values():
            g.zero_()
        for name, lin, ins, lout, out, pitch, offset in reversed(self.graph):
            layer = self.by_name[name]
            if name == 'head':
                gout, gpitch = self.dpred, HEAD_CHANNELS
            else:
                gfull = self.grad_of[id(out)]
                gout = gfull.view(-1)[offset:]     # channel offset inside the (concatenated) buffer
                gpitch = pitch
                if layer.relu:
                    self._call('ffx_relu_backward', self._voxels(lout), layer.cout, _p(gout), gpitch, _p(out), pitch,
                               offset, s)
            # weight and bias gradients
            c = self._conv(layer, lin, ins[0], lout, None, 0, 0)
            self._call('ffx_conv_weight_grad', C.byref(c), _p(gout), gpitch, _p(layer.gw), s)
            self._call('ffx_bias_grad', self._voxels(lout), layer.cout, _p(gout), gpitch, _p(layer.gb), s)
            if name == 'e0a':
                continue
            # data gradient into the input's gradient view
            (tin, ipitch, ioff, ich) = ins[0]
            gin = self.grad_of[id(tin)]
            flip = int(layer.kind == 'conv3')
            self._call('ffx_weight_transpose', layer.taps, layer.cin, layer.cout, flip, _p(layer.w16),
                       _p(layer.wt16), s)
            g_view = (gout, gpitch, 0, layer.cout)
            # the input of the down-samplings is a skip half that already holds the decoder's gradient
            accumulate = int(layer.kind == 'down')
            if layer.kind == 'conv3':
                c = self._conv(layer, lout, g_view, lin, gin, ipitch, ioff, weight=layer.wt16, cout=layer.cin,
                               bias=False, relu=False, accumulate=accumulate)
            elif layer.kind == 'head':
                c = self._conv(layer, lout, g_view, lin, gin, ipitch, ioff, weight=layer.wt16, cout=layer.cin,
                               bias=False, relu=False)
            elif layer.kind == 'down':
                c = self._conv(layer, lout, g_view, lin, gin, ipitch, ioff, weight=layer.wt16, transposed=1,
                               ks=2, stride=2, pad=0, cout=layer.cin, bias=False, relu=False, accumulate=1)
            else:   # up: its data gradient is a 2^3 stride-2 convolution of the fine gradient
                c = self._conv(layer, lout, g_view, lin, gin, ipitch, ioff, weight=layer.wt16, transposed=0,
                               ks=2, stride=2, pad=0, cout=layer.cin, bias=False, relu=False)
            self._run_conv((name, 'data'), c, s)
        return self.loss_acc

    def _voxels(self, level):
        d = self.dims[level]
        return self.batch * d[0] * d[1] * d[2]

    def adam_step(self, lr, stream, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step_count += 1
        self.weight_version += 1
        s = C.c_void_p(stream)
        for l in self.layers:
            for w, m, v, g, w16 in l.params():
                self._call('ffx_adam', w.numel(), _p(w), _p(m), _p(v), _p(g), _p(w16), lr, beta1, beta2, eps,
                           self.step_count, s)

    # ------------------------------------------------------------- state
    def state_dict(self):
        return {l.name: (l.w.detach().cpu(), l.b.detach().cpu()) for l in self.layers}

    def load_state_dict(self, state):
        for l in self.layers:
            w, b = state[l.name]
            l.w.copy_(w.to(l.w.device))
            l.b.copy_(b.to(l.b.device))
            l.w16.copy_(l.w.to(torch.bfloat16))
        self.weight_version += 1

    def forward_flops(self, batch, dims):
        """Multiply-add FLOPs (2 per MAC) of one forward pass."""
        D, H, W = dims
        total = 0
        level_of = {'e0a': 0, 'e0b': 0, 'd0': 1, 'e1a': 1, 'e1b': 1, 'd1': 2, 'e2a': 2, 'e2b': 2, 'd2': 3, 'e3a': 3,
                    'e3b': 3, 'u2': 2, 'c2a': 2, 'c2b': 2, 'u1': 1, 'c1a': 1, 'c1b': 1, 'u0': 0, 'c0a': 0, 'c0b': 0,
                    'head': 0}
        for l in self.layers:
            out_vox = batch * (D >> level_of[l.name]) * (H >> level_of[l.name]) * (W >> level_of[l.name])
            per = l.cin * l.cout * (l.taps if l.kind != 'up' else 1)   # a transposed 2^3 tap feeds one output
            total += 2 * per * out_vox
        return total


def main():
    """Time the forward pass and a training step on synthetic input:
    python -m fluxfx_b200.learned.unet --size 128 --batch 1 --repeat 5"""
    import argparse
    import json
    ap = argparse.ArgumentParser(description='U-Net timing on synthetic input')
    ap.add_argument('--size', type=int, default=128)
    ap.add_argument('--batch', type=int, default=1)
    ap.add_argument('--repeat', type=int, default=5)
    ap.add_argument('--train', action='store_true', help='also time forward + backward + Adam')
    ap.add_argument('--tcgen05', action='store_true', help='the gathered-operand tcgen05 convolutions')
    ap.add_argument('--mma-sync', action='store_true', help='the gathered-operand mma.sync convolutions')
    ap.add_argument('--tma', action='store_true', help='3x3x3 layers as TMA halo tiles on tcgen05 (default)')
    args = ap.parse_args()
    dev = torch.device('cuda')
    net = UNet(dev, seed=0)
    if args.tcgen05:
        net.conv_entry = 'ffx_conv_forward_tc'
    if args.mma_sync:
        net.conv_entry = 'ffx_conv_forward'
    g = torch.Generator(device='cuda').manual_seed(0)
    n = args.size
    div = torch.randn((args.batch, n, n, n), device=dev, generator=g)
    mask = (torch.rand((args.batch, n, n, n), device=dev, generator=g) < 0.05).to(torch.uint8)
    target = torch.randn((args.batch, n, n, n), device=dev, generator=g)
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        net.forward(div, mask, 1.0, stream)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(args.repeat):
        net.forward(div, mask, 1.0, stream)
    end.record()
    end.synchronize()
    fwd = start.elapsed_time(end) / args.repeat
    flops = net.forward_flops(args.batch, (n, n, n))
    out = {'size': n, 'batch': args.batch, 'forward_ms': fwd, 'forward_gflop': flops / 1e9,
           'forward_tflops': flops / (fwd * 1e-3) / 1e12}
    if args.train:
        start.record()
        for _ in range(args.repeat):
            net.forward(div, mask, 1.0, stream)
            net.loss_backward(target, mask, stream)
            net.adam_step(1e-4, stream)
        end.record()
        end.synchronize()
        step = start.elapsed_time(end) / args.repeat
        out.update(train_step_ms=step, train_tflops=3 * flops / (step * 1e-3) / 1e12)
    print(json.dumps(out))


if __name__ == '__main__':
    main()

"""Learned surrogate of the (2+1)D viscous evolution: a U-Net that maps the
initial energy density of an event (a 128 x 128 slice) to
(e, u^x, u^y, pi^xx, pi^xy, pi^yy) a fixed proper time later.

The network is trained and run by this library's own kernels (clv_unet_*):
3x3 convolutions as implicit GEMMs on the tensor cores (BF16 weights and
activations, FP32 accumulation), a CUDA-core first layer (one input channel)
and 1x1 head, 2x2 average pooling, nearest upsampling, GELU, a weighted
squared-error loss and Adam on FP32 master weights. Architecture: 4 levels of
two 3x3 convolutions with 32, 64, 128, 256 channels, skip connections by
concatenation, a 1x1 head to 6 channels.

The solver is the yardstick and the fallback: training and test events come from
the batched solver (CLViscBatch) on seeded initial conditions, the error of the
network is measured against solver results, and an event is run by the solver
instead when its prediction fails the energy balance (its transverse energy
strays from the value the training events relate to their initial profile) or
when the predictions for the event and its mirror images disagree by more than
a threshold calibrated on held-out training events.
"""
import ctypes
import math
import time

import numpy as np
import torch

from . import _lib

C1, C2, C3, C4 = 32, 64, 128, 256
K_OUT = 6
FIELDS = ('e', 'ux', 'uy', 'pixx', 'pixy', 'piyy')


class UnetConv(ctypes.Structure):  # clv_unet_conv
    _fields_ = [('in_', ctypes.c_void_p), ('in_cs', ctypes.c_int), ('in_co', ctypes.c_int), ('w', ctypes.c_void_p),
                ('bias', ctypes.c_void_p), ('out', ctypes.c_void_p), ('out_cs', ctypes.c_int),
                ('out_co', ctypes.c_int), ('pre', ctypes.c_void_p), ('gate', ctypes.c_void_p),
                ('gate_cs', ctypes.c_int), ('gate_co', ctypes.c_int), ('N', ctypes.c_int), ('H', ctypes.c_int),
                ('W', ctypes.c_int), ('Cin', ctypes.c_int), ('Cout', ctypes.c_int), ('gelu', ctypes.c_int)]


# (name, Cin, Cout, level) of the 3x3 tensor-core layers; level l has size H / 2^l
LAYERS = [('e1b', C1, C1, 0), ('e2a', C1, C2, 1), ('e2b', C2, C2, 1), ('e3a', C2, C3, 2), ('e3b', C3, C3, 2),
          ('e4a', C3, C4, 3), ('e4b', C4, C4, 3), ('d3a', C4 + C3, C3, 2), ('d3b', C3, C3, 2),
          ('d2a', C3 + C2, C2, 1), ('d2b', C2, C2, 1), ('d1a', C2 + C1, C1, 0), ('d1b', C1, C1, 0)]


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


class UNet(object):
    """Parameters, buffers and the forward / backward passes for batches of
    N images of H x W (H, W divisible by 8)."""

    def __init__(self, N, H=128, W=128, device=None, seed=0):
        if not torch.cuda.is_available():
            raise RuntimeError('the surrogate needs a CUDA device; there is no CPU path')
        self.lib = _lib.load()
        self.dev = torch.device('cuda', 0) if device is None else torch.device(device)
        self.N, self.H, self.W = N, H, W
        # parameter layout in one flat FP32 vector (for one Adam launch)
        self.shapes = {'first.w': (9, C1), 'first.b': (C1,)}
        for name, cin, cout, _ in LAYERS:
            self.shapes[name + '.w'] = (9, cin, cout)
            self.shapes[name + '.b'] = (cout,)
        self.shapes['head.w'] = (C1, K_OUT)
        self.shapes['head.b'] = (K_OUT,)
        self.offsets, n = {}, 0
        for k, s in self.shapes.items():
            self.offsets[k] = n
            n += int(np.prod(s))
        self.nparam = n
        g = torch.Generator().manual_seed(seed)
        flat = torch.zeros(n)
        for k, s in self.shapes.items():
            if k.endswith('.w'):
                fan_in = 9 * (1 if k == 'first.w' else s[1]) if k != 'head.w' else C1
                std = math.sqrt(2.0 / fan_in) * (0.1 if k == 'head.w' else 1.0)
                flat[self.offsets[k]:self.offsets[k] + int(np.prod(s))] = torch.randn(int(np.prod(s)), generator=g) * std
        self.params = flat.to(self.dev)
        self.grads = torch.zeros(n, device=self.dev)
        self.m = torch.zeros(n, device=self.dev)
        self.v = torch.zeros(n, device=self.dev)
        self.step_count = 0
        self.bf = {}
        for name, cin, cout, _ in LAYERS:
            self.bf[name] = (torch.empty(9 * cin * cout, dtype=torch.bfloat16, device=self.dev),
                             torch.empty(9 * cin * cout, dtype=torch.bfloat16, device=self.dev))
        self._alloc(N)
        self.pack()

    def P(self, k):
        return self.params[self.offsets[k]:self.offsets[k] + int(np.prod(self.shapes[k]))]

    def G(self, k):
        return self.grads[self.offsets[k]:self.offsets[k] + int(np.prod(self.shapes[k]))]

    def _alloc(self, N):
        H, W, d = self.H, self.W, self.dev
        bf = lambda h, w, c: torch.zeros((N, h, w, c), dtype=torch.bfloat16, device=d)
        s = [(H >> l, W >> l) for l in range(4)]
        self.buf = {
            'x': torch.zeros((N, H, W), dtype=torch.float32, device=d),
            'z_first': bf(*s[0], C1), 'y_first': bf(*s[0], C1),
            'cat1': bf(*s[0], C2 + C1), 'cat2': bf(*s[1], C3 + C2), 'cat3': bf(*s[2], C4 + C3),
            'p1': bf(*s[1], C1), 'p2': bf(*s[2], C2), 'p3': bf(*s[3], C3),
            'out': torch.zeros((N * H * W, K_OUT), dtype=torch.float32, device=d),
            'gout': torch.zeros((N * H * W, K_OUT), dtype=torch.float32, device=d),
        }
        for name, cin, cout, l in LAYERS:
            self.buf['z_' + name] = bf(*s[l], cout)
            if name not in ('e1b', 'e2b', 'e3b'):  # those write into the concatenations
                self.buf['y_' + name] = bf(*s[l], cout)
            self.buf['g_' + name] = bf(*s[l], cout)  # gradient wrt the pre-activation
        self.buf['gcat1'] = bf(*s[0], C2 + C1)
        self.buf['gcat2'] = bf(*s[1], C3 + C2)
        self.buf['gcat3'] = bf(*s[2], C4 + C3)
        self.buf['gp1'], self.buf['gp2'], self.buf['gp3'] = bf(*s[1], C1), bf(*s[2], C2), bf(*s[3], C3)
        self.buf['g_first'] = bf(*s[0], C1)
        wmax = max(int(self.lib.clv_unet_wgrad_scratch_bytes(N, H >> l, W >> l, cin, cout)) for _, cin, cout, l in LAYERS)
        rmax = int(self.lib.clv_unet_rows_scratch_bytes(9 * C4 + 64))
        self.scratch = torch.empty(max(wmax, rmax) // 4 + 64, dtype=torch.float32, device=d)
        self.loss_part = torch.zeros(256, dtype=torch.float32, device=d)
        self.N = N

    @property
    def stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)

    def _chk(self, rc, what):
        _lib.check(rc, what)

    def check_timeouts(self, what):
        """Raise if a tensor-core kernel's bounded wait ran out since the last
        check (clv_unet_timeouts; such a kernel skips its epilogue and leaves
        output tiles unwritten, so its results cannot be used)."""
        n = ctypes.c_int(0)
        self._chk(self.lib.clv_unet_timeouts(ctypes.byref(n), 1), 'clv_unet_timeouts')
        if n.value:
            raise RuntimeError('%s: %d tensor-core waits timed out; results discarded' % (what, n.value))
        return 0

    def pack(self):
        """BF16 copies of the 3x3 weights for the forward and input-gradient convolutions."""
        for name, cin, cout, _ in LAYERS:
            w, wt = self.bf[name]
            self._chk(self.lib.clv_unet_pack(_p(self.P(name + '.w')), cin, cout, _p(w), _p(wt), self.stream),
                      'clv_unet_pack')

    # --------------------------------------------------------------- views
    def _src(self, name):
        """(tensor, channel stride, offset) of a 3x3 layer's input and output."""
        b = self.buf
        ins = {'e1b': (b['y_first'], C1, 0), 'e2a': (b['p1'], C1, 0), 'e2b': (b['y_e2a'], C2, 0),
               'e3a': (b['p2'], C2, 0), 'e3b': (b['y_e3a'], C3, 0), 'e4a': (b['p3'], C3, 0),
               'e4b': (b['y_e4a'], C4, 0), 'd3a': (b['cat3'], C4 + C3, 0), 'd3b': (b['y_d3a'], C3, 0),
               'd2a': (b['cat2'], C3 + C2, 0), 'd2b': (b['y_d2a'], C2, 0), 'd1a': (b['cat1'], C2 + C1, 0),
               'd1b': (b['y_d1a'], C1, 0)}
        outs = {'e1b': (b['cat1'], C2 + C1, C2), 'e2b': (b['cat2'], C3 + C2, C3), 'e3b': (b['cat3'], C4 + C3, C4)}
        return ins[name], outs.get(name, (b.get('y_' + name), None, 0))

    def _conv(self, name, cin, cout, l, x, out, gelu=True, pre=None, gate=None, w=None):
        a = UnetConv()
        a.in_, a.in_cs, a.in_co = _p(x[0]), x[1], x[2]
        a.w = _p(w if w is not None else self.bf[name][0])
        a.bias = None if w is not None else _p(self.P(name + '.b'))
        a.out, a.out_cs, a.out_co = _p(out[0]), out[1], out[2]
        a.pre = _p(pre)
        if gate is not None:
            a.gate, a.gate_cs, a.gate_co = _p(gate[0]), gate[1], gate[2]
        a.N, a.H, a.W, a.Cin, a.Cout, a.gelu = self.N, self.H >> l, self.W >> l, cin, cout, int(gelu)
        self._chk(self.lib.clv_unet_conv3x3(ctypes.byref(a), self.stream), 'clv_unet_conv3x3 ' + name)

    # ------------------------------------------------------------- forward
    def forward(self, x=None):
        """x: (N, H, W) FP32 images (or the contents of buf['x']); returns the
        (N*H*W, 6) FP32 output."""
        b, N, H, W, lib, s = self.buf, self.N, self.H, self.W, self.lib, self.stream
        if x is not None:
            b['x'].copy_(x.reshape(N, H, W))
        self._chk(lib.clv_unet_first_fwd(_p(b['x']), _p(self.P('first.w')), _p(self.P('first.b')), N, H, W, C1,
                                         _p(b['z_first']), _p(b['y_first']), C1, 0, s), 'first')
        for name, cin, cout, l in LAYERS:
            if name == 'e2a':
                self._chk(lib.clv_unet_pool(_p(b['cat1']), C2 + C1, C2, N, H, W, C1, _p(b['p1']), s), 'pool1')
            if name == 'e3a':
                self._chk(lib.clv_unet_pool(_p(b['cat2']), C3 + C2, C3, N, H >> 1, W >> 1, C2, _p(b['p2']), s),
                          'pool2')
            if name == 'e4a':
                self._chk(lib.clv_unet_pool(_p(b['cat3']), C4 + C3, C4, N, H >> 2, W >> 2, C3, _p(b['p3']), s),
                          'pool3')
            if name == 'd3a':
                self._chk(lib.clv_unet_up(_p(b['y_e4b']), N, H >> 3, W >> 3, C4, _p(b['cat3']), C4 + C3, 0, s), 'up3')
            if name == 'd2a':
                self._chk(lib.clv_unet_up(_p(b['y_d3b']), N, H >> 2, W >> 2, C3, _p(b['cat2']), C3 + C2, 0, s), 'up2')
            if name == 'd1a':
                self._chk(lib.clv_unet_up(_p(b['y_d2b']), N, H >> 1, W >> 1, C2, _p(b['cat1']), C2 + C1, 0, s), 'up1')
            x_in, (o, ocs, oco) = self._src(name)
            self._conv(name, cin, cout, l, x_in, (o, ocs or cout, oco), pre=b['z_' + name])
        self._chk(lib.clv_unet_head_fwd(_p(b['y_d1b']), C1, 0, _p(self.P('head.w')), _p(self.P('head.b')),
                                        N * H * W, C1, K_OUT, _p(b['out']), s), 'head')
        return b['out']

    # ------------------------------------------------------------ backward
    def backward(self):
        """Gradients of every parameter into self.grads from buf['gout']
        (dL/d output), after forward()."""
        b, N, H, W, lib, s = self.buf, self.N, self.H, self.W, self.lib, self.stream
        sc, scb = _p(self.scratch), self.scratch.numel() * 4
        P0 = N * H * W
        self._chk(lib.clv_unet_head_bwd(_p(b['y_d1b']), C1, 0, _p(b['z_d1b']), _p(b['gout']), _p(self.P('head.w')),
                                        P0, C1, K_OUT, _p(b['g_d1b']), _p(self.grads[self.offsets['head.w']:]), sc,
                                        scb, s), 'head_bwd')
        # gradient wrt each layer's pre-activation is in g_<name> when its turn comes
        plain_next = {'d1b': 'd1a', 'd2b': 'd2a', 'd3b': 'd3a', 'e4b': 'e4a', 'e3b': 'e3a', 'e2b': 'e2a',
                      'e1b': None}
        for name, cin, cout, l in reversed(LAYERS):
            h, w = H >> l, W >> l
            x_in, _ = self._src(name)
            g = b['g_' + name]
            self._chk(lib.clv_unet_wgrad3x3(_p(x_in[0]), x_in[1], x_in[2], _p(g), N, h, w, cin, cout,
                                            _p(self.G(name + '.w')), 0, sc, scb, s), 'wgrad ' + name)
            self._chk(lib.clv_unet_bias_grad(_p(g), cout, N * h * w, cout, _p(self.G(name + '.b')), sc, scb, s),
                      'bias ' + name)
            wt = self.bf[name][1]
            if name in plain_next and plain_next[name] is not None:
                prev = plain_next[name]
                # input is GELU(z_prev): fuse gelu'(z_prev) into the input-gradient epilogue
                self._conv(name, cout, cin, l, (g, cout, 0), (b['g_' + prev], cin, 0), gelu=False,
                           gate=(b['z_' + prev], cin, 0), w=wt)
            elif name == 'e1b':
                self._conv(name, cout, cin, l, (g, cout, 0), (b['g_first'], cin, 0), gelu=False,
                           gate=(b['z_first'], cin, 0), w=wt)
            elif name in ('d1a', 'd2a', 'd3a'):
                gcat = {'d1a': 'gcat1', 'd2a': 'gcat2', 'd3a': 'gcat3'}[name]
                self._conv(name, cout, cin, l, (g, cout, 0), (b[gcat], cin, 0), gelu=False, w=wt)
                if name == 'd1a':
                    self._chk(lib.clv_unet_up_grad(_p(b['gcat1']), C2 + C1, 0, _p(b['z_d2b']), N, H >> 1, W >> 1, C2,
                                                   _p(b['g_d2b']), s), 'up_grad1')
                elif name == 'd2a':
                    self._chk(lib.clv_unet_up_grad(_p(b['gcat2']), C3 + C2, 0, _p(b['z_d3b']), N, H >> 2, W >> 2, C3,
                                                   _p(b['g_d3b']), s), 'up_grad2')
                else:
                    self._chk(lib.clv_unet_up_grad(_p(b['gcat3']), C4 + C3, 0, _p(b['z_e4b']), N, H >> 3, W >> 3, C4,
                                                   _p(b['g_e4b']), s), 'up_grad3')
            elif name in ('e2a', 'e3a', 'e4a'):
                # input is the pooled skip output: its gradient joins the skip slice's
                gp = {'e2a': 'gp1', 'e3a': 'gp2', 'e4a': 'gp3'}[name]
                self._conv(name, cout, cin, l, (g, cout, 0), (b[gp], cin, 0), gelu=False, w=wt)
                skip, gcat, cs, co = {'e2a': ('e1b', 'gcat1', C2 + C1, C2), 'e3a': ('e2b', 'gcat2', C3 + C2, C3),
                                      'e4a': ('e3b', 'gcat3', C4 + C3, C4)}[name]
                self._chk(lib.clv_unet_skip_grad(_p(b[gcat]), cs, co, _p(b[gp]), _p(b['z_' + skip]), N, H >> (l - 1),
                                                 W >> (l - 1), cin, _p(b['g_' + skip]), s), 'skip_grad ' + skip)
        self._chk(lib.clv_unet_first_wgrad(_p(b['x']), _p(b['g_first']), N, H, W, C1, _p(self.G('first.w')), sc, scb,
                                           s), 'first_wgrad')
        self._chk(lib.clv_unet_bias_grad(_p(b['g_first']), C1, P0, C1, _p(self.G('first.b')), sc, scb, s),
                  'first_bias')

    def loss(self, target, wch, scale=None):
        """Weighted squared error of buf['out'] against target (N*H*W, 6);
        fills buf['gout']; returns the loss as a device scalar."""
        b = self.buf
        P0 = self.N * self.H * self.W
        scale = 1.0 / (P0 * K_OUT) if scale is None else scale
        self._chk(self.lib.clv_unet_mse(_p(b['out']), _p(target), _p(wch), P0, K_OUT, float(scale), _p(b['gout']),
                                        _p(self.loss_part), self.loss_part.numel(), self.stream), 'mse')
        return self.loss_part.sum()

    def adam(self, lr, b1=0.9, b2=0.999, eps=1e-8):
        self.step_count += 1
        t = self.step_count
        lr_t = lr * math.sqrt(1.0 - b2 ** t) / (1.0 - b1 ** t)
        self._chk(self.lib.clv_unet_adam(_p(self.params), _p(self.grads), _p(self.m), _p(self.v), self.nparam,
                                         float(lr_t), float(b1), float(b2), float(eps), self.stream), 'adam')
        self.pack()

    def state_dict(self):
        return {'params': self.params.detach().cpu(), 'm': self.m.cpu(), 'v': self.v.cpu(), 'step': self.step_count}


# ---------------------------------------------------------------- data
def event_spec(seed, bmax=12.0):
    """Impact parameter of a training / test event, from its seed."""
    rng = np.random.default_rng(seed)
    return float(rng.uniform(0.0, bmax))


def surrogate_cfg(n=128, steps=320):
    """The (2+1)D configuration of the batched workload on an n x n grid."""
    from .config import read_config, set_real
    cfg = read_config([])
    cfg.NX = cfg.NY = n
    cfg.NZ = 1
    cfg.DX = cfg.DY = 0.16
    cfg.DZ = 0.15
    cfg.DT = 0.02
    cfg.TAU0 = 0.6
    cfg.eos_type = 'lattice_pce165'
    cfg.use_float32 = True
    cfg.ETAOS_XMIN, cfg.ETAOS_YMIN, cfg.ETAOS_LEFT_SLOP, cfg.ETAOS_RIGHT_SLOP = 0.18, 0.16, 0.0, 0.0
    cfg.ZETAOS_MAX, cfg.ZETAOS_T0, cfg.ZETAOS_WIDTH, cfg.ZETAOS_SKEW = 0.05, 0.18, 0.02, 0.0
    cfg.TFRZ = 0.137
    cfg.ntskip = 20
    cfg.fPathOut = '/tmp/clv_surrogate'
    return set_real(cfg)


def generate_events(seeds, n=128, steps=320, batch=512, edmax=50.0):
    """Initial energy density (E, n, n), the solver's fields (E, n, n, 6)
    after `steps` steps, from the batched solver, on the device in FP32, and a
    mask of the events whose input and fields are all finite."""
    from .batch import CLViscBatch
    cfg = surrogate_cfg(n, steps)
    xs, ys = [], []
    for i0 in range(0, len(seeds), batch):
        chunk = seeds[i0:i0 + batch]
        # the launch shape the batch autotuner picks for (2+1)D events: 256
        # threads, one cell per thread, the 128-register kernel
        cells = n * n * len(chunk)
        bt = CLViscBatch(cfg, [(n, n, 1)] * len(chunk), max_loops=steps, stop_at_freezeout=False, block_size=256,
                         grid_blocks=(cells + 255) // 256, max_registers=128)
        for e, sd in enumerate(chunk):
            bt.load_hotspot_event(e, b=event_spec(sd), seed=int(sd), edmax=edmax)
        ld = bt.layout[0][0]
        ev0 = bt.d_ev[1].view(len(chunk), 4, ld)[:, 0, :n * n].reshape(-1, n, n).clone()
        bt.evolve()
        ev = bt.d_ev[1].view(len(chunk), 4, ld)[:, :, :n * n]
        pi = bt.d_pi[1].view(len(chunk), bt.npi, ld)[:, :, :n * n]
        vx, vy = ev[:, 1], ev[:, 2]
        g = 1.0 / torch.sqrt(torch.clamp(1.0 - vx * vx - vy * vy - ev[:, 3] * ev[:, 3], min=1e-7))
        y = torch.stack([ev[:, 0], g * vx, g * vy, pi[:, 4], pi[:, 5], pi[:, 7]], dim=-1)
        xs.append(ev0)
        ys.append(y.reshape(len(chunk), n, n, K_OUT).clone())
        del bt
    x, y = torch.cat(xs), torch.cat(ys)
    # events whose state ran away: a non-finite value, or |value| above 50
    # (GeV/fm^3 for e and pi, units of c for u; the initial peak is edmax)
    lim = max(50.0, edmax)
    fin = torch.isfinite(x).reshape(x.shape[0], -1).all(1) & torch.isfinite(y).reshape(y.shape[0], -1).all(1)
    small = (torch.nan_to_num(y, nan=0.0).abs().reshape(y.shape[0], -1).amax(1) <= lim)
    return x, y, fin & small


def rel_l2(pred, true):
    """Per-event relative L2 error ||pred - true|| / ||true|| over the grid."""
    d = (pred - true).reshape(pred.shape[0], -1)
    t = true.reshape(true.shape[0], -1)
    return torch.linalg.vector_norm(d, dim=1) / torch.linalg.vector_norm(t, dim=1)


class Surrogate(object):
    """Training, inference and the solver fallback around UNet."""

    def __init__(self, batch=32, n=128, seed=0):
        self.net = UNet(batch, n, n, seed=seed)
        self.n = n
        self.batch = batch
        self.in_scale = 1.0 / 50.0
        self.out_scale = None
        self.wch = None

    def fit_scales(self, y):
        s = y[:min(y.shape[0], 2048)].reshape(-1, K_OUT).double().std(dim=0).float()
        self.out_scale = torch.clamp(s, min=1e-6)
        # the error that matters is on e: weigh it most
        self.wch = torch.tensor([4.0, 1.0, 1.0, 1.0, 1.0, 1.0], device=y.device)

    def train(self, x, y, epochs=8, lr=1e-3, log=None, max_norm=1.0):
        """Train on (E, n, n) inputs and (E, n, n, 6) targets on the device."""
        if self.out_scale is None:
            self.fit_scales(y)
        net, B = self.net, self.batch
        E = x.shape[0]
        steps_per_epoch = E // B
        total = epochs * steps_per_epoch
        g = torch.Generator(device=x.device).manual_seed(1234)
        step = 0
        history = []
        for ep in range(epochs):
            perm = torch.randperm(E, generator=g, device=x.device)
            ep_loss = torch.zeros((), device=x.device)
            for it in range(steps_per_epoch):
                idx = perm[it * B:(it + 1) * B]
                net.buf['x'].copy_(x[idx] * self.in_scale)
                target = (y[idx].reshape(-1, K_OUT) / self.out_scale).contiguous()
                net.forward()
                ep_loss += net.loss(target, self.wch)
                net.backward()
                # global gradient-norm clipping, on the device
                gn = torch.linalg.vector_norm(net.grads)
                net.grads.mul_(torch.clamp(max_norm / (gn + 1e-6), max=1.0))
                lr_s = lr * 0.5 * (1.0 + math.cos(math.pi * step / total))
                net.adam(lr_s)
                step += 1
            history.append(float(ep_loss) / steps_per_epoch)
            self.net.check_timeouts('training epoch %d' % ep)
            if log:
                log('epoch %d loss %.5f' % (ep, history[-1]))
        return history

    def predict(self, x):
        """(E, n, n) initial energy densities -> (E, n, n, 6) fields."""
        net, B, n = self.net, self.batch, self.n
        out = torch.empty((x.shape[0], n, n, K_OUT), device=x.device)
        for i0 in range(0, x.shape[0], B):
            xb = x[i0:i0 + B]
            m = xb.shape[0]
            net.buf['x'].zero_()
            net.buf['x'][:m].copy_(xb * self.in_scale)
            o = net.forward()
            out[i0:i0 + m] = (o.view(B, n, n, K_OUT)[:m] * self.out_scale)
        net.check_timeouts('inference')
        return out


# The evolution commutes with the reflections of the grid's x and y axes
# (the stencil, the limiters and the initial-condition construction, whose
# impact parameter lies along x, are all mirror symmetric): the fields of a
# mirrored initial condition are the mirrored fields, with u^x (x mirror),
# u^y (y mirror) and pi^xy (either) changing sign.
_FLIPS = ((), (1,), (2,), (1, 2))  # axes of (E, n, n) inputs to reverse
_SIGN = {(): (1, 1, 1, 1, 1, 1), (1,): (1, -1, 1, 1, -1, 1), (2,): (1, 1, -1, 1, -1, 1),
         (1, 2): (1, -1, -1, 1, 1, 1)}


def predict_mirrored(sur, x):
    """The network on x and its three mirror images, each prediction mapped
    back: returns (mean over the four (E, n, n, 6), per-event spread of the
    energy density: the largest relative L2 distance of one of the four from
    their mean)."""
    preds = []
    for ax in _FLIPS:
        xin = torch.flip(x, dims=ax) if ax else x
        out = sur.predict(xin.contiguous())
        if ax:
            out = torch.flip(out, dims=ax)
        sign = torch.tensor(_SIGN[ax], dtype=out.dtype, device=out.device)
        preds.append(out * sign)
    stack = torch.stack(preds)
    mean = stack.mean(0)
    spread = torch.stack([rel_l2(q[..., 0], mean[..., 0]) for q in preds]).amax(0)
    return mean, spread


def calibrate_threshold(score, err, bad=0.02, keep_frac=0.005):
    """The largest threshold on `score` for which, on calibration events,
    at most keep_frac of the events would be kept (score <= threshold) with an
    error above `bad`; events above the threshold go to the solver."""
    order = torch.argsort(score)
    s_sorted, bad_sorted = score[order], (err[order] > bad).double()
    kept_bad = torch.cumsum(bad_sorted, 0)  # bad events among those at or below each score
    ok = kept_bad <= keep_frac * score.numel()
    idx = int(torch.nonzero(ok)[-1]) if bool(ok.any()) else -1
    return float(s_sorted[idx]) if idx >= 0 else float('-inf')


def transverse_energy(fields, eos_p, tau, dx):
    """tau * sum over the slice of T^{tau tau} = (e + P) u0^2 - P, u0^2 = 1 + ux^2 + uy^2."""
    e = fields[..., 0]
    P = eos_p(e)
    u02 = 1.0 + fields[..., 1] ** 2 + fields[..., 2] ** 2
    return tau * dx * dx * ((e + P) * u02 - P).reshape(e.shape[0], -1).sum(dim=1)


def ic_features(x, tau0, dx, P):
    """Integrals of the initial energy-density slices x (N, n, n) that the
    final transverse energy depends on: the initial transverse energy, the
    entropy-like sum of e^(3/4), the sum of e^(1/2), the second radial
    moment and the sum of e^2, and a constant; (N, 6), float64."""
    n = x.shape[-1]
    c = (torch.arange(n, device=x.device, dtype=torch.float32) - (n - 1) / 2.0) * dx
    r2 = c[:, None] ** 2 + c[None, :] ** 2
    e = torch.clamp(torch.nan_to_num(x, nan=0.0), min=0.0)
    zeros = torch.zeros_like(e)
    et0 = transverse_energy(torch.stack([e, zeros, zeros], -1), P, tau0, dx)
    flat = lambda t: t.reshape(e.shape[0], -1).sum(dim=1)
    cols = [et0, flat(e ** 0.75) * dx * dx, flat(e ** 0.5) * dx * dx, flat(e * r2) * dx * dx,
            flat(e * e) * dx * dx, torch.ones_like(et0)]
    return torch.stack(cols, 1).double()


def table_pressure(device):
    """P(e) of the lattice EOS table, linear interpolation on the device."""
    from .eos import Eos, TABLE_SHAPE
    table, meta = Eos('lattice_pce165').create_table(*TABLE_SHAPE['lattice_pce165'])
    p = torch.from_numpy(table.reshape(-1, 4)[:, 1].astype(np.float32)).to(device)
    e0, de = float(meta['ed_start']), float(meta['ed_step'])

    def P(e):
        x = torch.nan_to_num((e.double() - e0) / de, nan=0.0, posinf=0.0, neginf=0.0)
        i = torch.clamp(x.floor(), 0, p.numel() - 2).long()
        r = torch.clamp(x - i, 0.0, 1.0).float()
        return (1.0 - r) * p[i] + r * p[i + 1]
    return P


def run_experiment(n_train=20000, n_test=1000, epochs=12, batch=32, n=128, steps=320, gen_batch=1024, lr=1e-3,
                   residual_max=0.01, log=print):
    """Generate events with the solver, train the surrogate, and compare it
    with the solver on held-out events (seeds 10^5 + i for training,
    9 10^5 + i for testing). Returns a dict of the measured numbers."""
    dev = torch.device('cuda', 0)
    res = {'n_train': n_train, 'n_test': n_test, 'grid': n, 'steps': steps, 'epochs': epochs, 'batch': batch}
    t = time.perf_counter()
    xtr, ytr, ok = generate_events([100000 + i for i in range(n_train)], n, steps, gen_batch)
    torch.cuda.synchronize()
    res['generate_train_s'] = time.perf_counter() - t
    res['train_events_ran_away'] = int((~ok).sum())
    xtr, ytr = xtr[ok], ytr[ok]
    log('generated %d training events in %.1f s (%d ran away, left out)'
        % (n_train, res['generate_train_s'], res['train_events_ran_away']))
    # the solver on the test events, timed: initial condition to fields
    torch.cuda.synchronize()
    t = time.perf_counter()
    xte, yte, okte = generate_events([900000 + i for i in range(n_test)], n, steps, gen_batch)
    torch.cuda.synchronize()
    t_solver = time.perf_counter() - t
    res['test_events_ran_away'] = int((~okte).sum())
    test_seeds = torch.arange(n_test, device=dev)[okte]
    xte, yte = xte[okte], yte[okte]
    res['solver_s'] = t_solver
    res['solver_events_per_h'] = n_test / t_solver * 3600.0
    log('solver: %d test events in %.2f s' % (n_test, t_solver))
    # the last 5 % of the training events calibrate the fallback threshold
    # and are not trained on
    n_cal = max(32, xtr.shape[0] // 20)
    xcal, ycal = xtr[-n_cal:], ytr[-n_cal:]
    xtr, ytr = xtr[:-n_cal], ytr[:-n_cal]
    res['calibration_events'] = int(n_cal)
    sur = Surrogate(batch, n)
    t = time.perf_counter()
    hist = sur.train(xtr, ytr, epochs=epochs, lr=lr, log=log)
    torch.cuda.synchronize()
    res['train_s'] = time.perf_counter() - t
    log('trained %d epochs in %.1f s' % (epochs, res['train_s']))
    res['loss_history'] = [round(h, 6) for h in hist]
    # inference, timed: the network on each event and its three mirror
    # images, averaged; their spread is the network's own error estimate
    torch.cuda.synchronize()
    t = time.perf_counter()
    pred, spread = predict_mirrored(sur, xte)
    torch.cuda.synchronize()
    t_inf = time.perf_counter() - t
    pred_single = sur.predict(xte)
    err = rel_l2(pred[..., 0], yte[..., 0])
    # the method without the network: Bjorken cooling of the initial profile
    tau0, tau1 = 0.6, 0.6 + steps * 0.02
    base = rel_l2(xte * (tau0 / tau1) ** (4.0 / 3.0), yte[..., 0])
    # fallback: transverse energy of the prediction against the value a linear
    # fit on the training events predicts from integrals of the initial
    # profile (ic_features); the fit's own scatter on the true test fields is
    # reported beside it
    Pf = table_pressure(dev)
    et1_tr = transverse_energy(ytr, Pf, tau1, 0.16).double()
    Ftr = ic_features(xtr, tau0, 0.16, Pf)
    scale = Ftr.abs().mean(0).clamp(min=1e-30)
    coef = torch.linalg.lstsq(Ftr / scale, et1_tr[:, None]).solution[:, 0]
    et_expect = ((ic_features(xte, tau0, 0.16, Pf) / scale) @ coef).float()
    resid = (transverse_energy(pred, Pf, tau1, 0.16) - et_expect).abs() / et_expect.abs()
    resid_true = (transverse_energy(yte, Pf, tau1, 0.16) - et_expect).abs() / et_expect.abs()
    res['fallback_fit_scatter'] = {'median': float(resid_true.median()), 'p90': float(resid_true.quantile(0.9))}
    # the same test with the initial transverse energy as the only feature
    c1 = torch.linalg.lstsq(Ftr[:, [0, 5]] / scale[[0, 5]], et1_tr[:, None]).solution[:, 0]
    e1 = ((ic_features(xte, tau0, 0.16, Pf)[:, [0, 5]] / scale[[0, 5]]) @ c1).float()
    res['fallback_events_one_feature'] = int(((transverse_energy(pred, Pf, tau1, 0.16) - e1).abs() / e1.abs()
                                              > residual_max).sum())
    # the fallback: an event goes to the solver when the energy-balance
    # residual of its prediction exceeds residual_max, or the spread of its
    # mirrored predictions exceeds a threshold calibrated on held-out training
    # events (at most 0.5 % of them kept with an error above 2 %, the balance
    # test applied first)
    pcal, scal = predict_mirrored(sur, xcal)
    ecal = rel_l2(pcal[..., 0], ycal[..., 0])
    et_cal = ((ic_features(xcal, tau0, 0.16, Pf) / scale) @ coef).float()
    rcal = (transverse_energy(pcal, Pf, tau1, 0.16) - et_cal).abs() / et_cal.abs()
    keep_cal = rcal <= residual_max
    spread_max = calibrate_threshold(torch.where(keep_cal, scal, torch.full_like(scal, float('inf'))), ecal)
    res['spread_threshold'] = spread_max
    res['calibration'] = {'events': int(n_cal), 'err_mean': float(ecal.mean()),
                          'rerun_frac': float(((~keep_cal) | (scal > spread_max)).float().mean())}
    res['fallback_balance_only'] = int((resid > residual_max).sum())
    res['kept_events_above_2pct_balance_only'] = int(((rel_l2(pred[..., 0], yte[..., 0]) > 0.02) &
                                                      (resid <= residual_max)).sum())
    rerun = (resid > residual_max) | (spread > spread_max)
    net_err = rel_l2(pred[..., 0], yte[..., 0])
    res['kept_events_above_2pct'] = int(((net_err > 0.02) & ~rerun).sum())
    n_rerun = int(rerun.sum())
    t_fb = 0.0
    if n_rerun:
        idx = torch.nonzero(rerun)[:, 0].cpu().numpy()
        seeds = test_seeds[torch.from_numpy(idx).to(dev)].cpu().numpy()
        # the solver of a service is loaded: one untimed run at the fallback's
        # batch size first (module loads and graph set-up of that size, which
        # otherwise fell into the timed region and varied 0.25-0.96 s)
        generate_events([900000 + int(i) for i in seeds], n, 1, gen_batch)
        torch.cuda.synchronize()
        t = time.perf_counter()
        _, yfb, _ = generate_events([900000 + int(i) for i in seeds], n, steps, gen_batch)
        torch.cuda.synchronize()
        t_fb = time.perf_counter() - t
        err = err.clone()
        err[torch.from_numpy(idx).to(dev)] = rel_l2(yfb[..., 0], yte[torch.from_numpy(idx).to(dev)][..., 0])
    res['pred_not_finite'] = int((~torch.isfinite(pred)).reshape(pred.shape[0], -1).any(1).sum())
    res['tensor_core_timeouts'] = sur.net.check_timeouts('evaluation')  # training and inference raised on any
    res.update({
        'inference_s': t_inf, 'fallback_events': n_rerun, 'fallback_s': t_fb,
        'surrogate_events_per_h': xte.shape[0] / (t_inf + t_fb) * 3600.0,
        'speedup_vs_solver': t_solver / (t_inf + t_fb),
        'rel_l2_e': {'mean': float(err.mean()), 'median': float(err.median()), 'p90': float(err.quantile(0.9)),
                     'max': float(err.max()), 'frac_le_2pct': float((err <= 0.02).float().mean())},
        'rel_l2_e_network_only': {'mean': float(rel_l2(pred[..., 0], yte[..., 0]).mean()),
                                  'single_pass_mean': float(rel_l2(pred_single[..., 0], yte[..., 0]).mean())},
        'spread_vs_error_corr': float(torch.corrcoef(torch.stack([spread, net_err]))[0, 1]),
        'rel_l2_e_without_network': {'mean': float(base.mean()), 'median': float(base.median())},
        'rel_l2_other_fields_mean': {f: float(rel_l2(pred[..., k], yte[..., k]).mean())
                                     for k, f in enumerate(FIELDS) if k > 0},
    })
    log('surrogate: mean rel L2 on e %.4f (without network %.4f), %d fallbacks, %.0fx the solver'
        % (res['rel_l2_e']['mean'], res['rel_l2_e_without_network']['mean'], n_rerun, res['speedup_vs_solver']))
    return res

"""CLViscBatch: many viscous events on grids of different sizes, advanced
together on one GPU.

The reference runs one event per CLVisc object (its event-by-event scripts
loop over events); this runner keeps every event's fields in shared device
arenas and advances all running events with one persistent kernel launch per
Runge-Kutta stage. Per event it reproduces CLVisc exactly: the construction
sequence (pi initialised from the empty state, one ideal stage on it,
visc.py:101-102), load_ini, and evolve's loop (visc.py:473-560) with the
fused stages, the maximum energy density recorded with tau every ntskip steps
and the stop when it falls below the freeze-out energy density, so each
event's fields are bit-identical to a CLVisc run of that event alone. The stop
test runs on the device; evolve() captures ntskip steps in a CUDA graph and
replays it until every event has stopped.

    b = CLViscBatch(cfg, [(121, 121, 1), (301, 301, 1), ...])
    for e, ic in enumerate(ics):
        b.load_ini(e, ic)
    b.evolve()
    b.ev_to_host(e), b.pi_to_host(e), b.bulk_to_host(e), b.history(e), b.loops()

The stage kernel is either one thread per cell for any grids
(clv_batch_stage) or, for batches of (2+1)D events, the tiled kernel
(clv_batch_stage_tiled: y strips of rows-4 cells marching along x); both give
the same bits. autotune() times both families over their launch shapes.

Only the viscous path is batched (no Gubser, coupling or Riemann test flags);
freeze-out surfaces are not extracted.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .config import set_real
from .ideal import add_visc_params, load_eos, make_params, plane_stride

MAX_EVENTS = 1024


class _Event(ctypes.Structure):  # clv_batch_event
    _fields_ = [('nx', ctypes.c_int), ('ny', ctypes.c_int), ('nz', ctypes.c_int), ('reserved', ctypes.c_int),
                ('ld', ctypes.c_longlong), ('off_ev', ctypes.c_longlong), ('off_pi', ctypes.c_longlong),
                ('off_src', ctypes.c_longlong), ('off_cell', ctypes.c_longlong)]


class _Ctl(ctypes.Structure):  # clv_batch_ctl
    _fields_ = [('loop', ctypes.c_int), ('n_active', ctypes.c_int), ('active_cells', ctypes.c_longlong),
                ('done', ctypes.c_int), ('hist_len', ctypes.c_int)]


class _Batch(ctypes.Structure):  # clv_batch
    _fields_ = [('events', ctypes.c_void_p), ('n_events', ctypes.c_int),
                ('ev', ctypes.c_void_p * 3), ('pi', ctypes.c_void_p * 3),
                ('src', ctypes.c_void_p), ('udiff', ctypes.c_void_p), ('goodcell', ctypes.c_void_p),
                ('keys', ctypes.c_void_p), ('ctl', ctypes.c_void_p), ('active', ctypes.c_void_p),
                ('prefix', ctypes.c_void_p), ('loops', ctypes.c_void_p), ('history', ctypes.c_void_p),
                ('hist_cap', ctypes.c_int), ('tau0', ctypes.c_double), ('dt', ctypes.c_double),
                ('efrz', ctypes.c_double), ('ntskip', ctypes.c_int), ('max_loops', ctypes.c_int)]


def arena_layout(grids, npi):
    """Plane strides and element offsets of each event's blocks in the arenas:
    (ld, off_ev, off_pi, off_src, off_cell) per event and the arena lengths."""
    ld = [plane_stride(nx * ny * nz) for nx, ny, nz in grids]
    off = {'ev': [0], 'pi': [0], 'src': [0], 'cell': [0]}
    for l in ld:
        off['ev'].append(off['ev'][-1] + 4 * l)
        off['pi'].append(off['pi'][-1] + npi * l)
        off['src'].append(off['src'][-1] + (4 + npi) * l)
        off['cell'].append(off['cell'][-1] + l)
    rows = [(l, off['ev'][e], off['pi'][e], off['src'][e], off['cell'][e]) for e, l in enumerate(ld)]
    sizes = {k: v[-1] for k, v in off.items()}
    return rows, sizes


class CLViscBatch(object):
    """Batched viscous hydro: events of one configuration on their own grids."""

    def __init__(self, configs, grids, handcrafted_eos=None, gpu_id=0, max_loops=-1, block_size=None,
                 grid_blocks=None, max_registers=0, stop_at_freezeout=True, tile=None, launch=None):
        """launch: a shape from autotune(), ('cell', block, grid, max_registers)
        or ('tile', rows, chunk, grid), in place of block_size, grid_blocks,
        max_registers (one thread per cell) or tile = (rows, chunk)."""
        self.cfg = set_real(configs)
        if not torch.cuda.is_available():
            raise RuntimeError('CLViscBatch needs a CUDA device; there is no CPU path')
        if not 1 <= len(grids) <= MAX_EVENTS:
            raise ValueError('a batch holds 1..%d events' % MAX_EVENTS)
        c = self.cfg
        if getattr(c, 'gubser_visc_test', False) or getattr(c, 'pimn_omega_coupling', False) or \
                getattr(c, 'omega_omega_coupling', False) or getattr(c, 'riemann_test', False):
            raise ValueError('test flags (Gubser, couplings, Riemann) are not batched')
        self.lib = _lib.load()
        self.device = torch.device('cuda', gpu_id)
        torch.cuda.set_device(self.device)
        self.dtype = torch.float32 if c.use_float32 else torch.float64
        self.grids = [tuple(int(v) for v in g) for g in grids]
        self.n = len(self.grids)
        self.sizes = [nx * ny * nz for nx, ny, nz in self.grids]
        self.eos, self.eos_table, meta, self.efrz = load_eos(c, handcrafted_eos, self.device)
        big = [max(g[k] for g in self.grids) for k in range(3)]
        self.params = make_params(c, meta, self.eos_table, self.efrz, big[0], big[1], big[2],
                                  plane_stride(big[0] * big[1] * big[2]))
        self.bulk = add_visc_params(c, self.params)
        if not self.bulk and c.ETAOS_YMIN < 1.0E-6 and c.ETAOS_LEFT_SLOP < 1.0E-6 and c.ETAOS_RIGHT_SLOP < 1.0E-6:
            raise ValueError('eta/s = 0 without bulk viscosity: CLVisc runs such events with the ideal '
                             'solver (visc.py:483-489), which is not batched')
        self.npi = 11 if self.bulk else 10
        self.layout, sizes = arena_layout(self.grids, self.npi)
        self.event_params = []
        for (nx, ny, nz), (ld, _, _, _, _) in zip(self.grids, self.layout):
            p = make_params(c, meta, self.eos_table, self.efrz, nx, ny, nz, ld)
            add_visc_params(c, p)
            self.event_params.append(p)

        dev, dt = self.device, self.dtype
        self.d_ev = [torch.zeros(sizes['ev'], dtype=dt, device=dev) for _ in range(3)]
        self.d_pi = [torch.zeros(sizes['pi'], dtype=dt, device=dev) for _ in range(3)]
        self.d_src = torch.zeros(sizes['src'], dtype=dt, device=dev)
        self.d_udiff = torch.zeros(sizes['ev'], dtype=dt, device=dev)
        self.d_goodcell = torch.ones(sizes['cell'], dtype=torch.uint8, device=dev)
        ev_tab = (_Event * self.n)()
        for e, ((nx, ny, nz), (ld, oe, op, os_, oc)) in enumerate(zip(self.grids, self.layout)):
            ev_tab[e] = _Event(nx, ny, nz, 0, ld, oe, op, os_, oc)
        self.d_events = torch.frombuffer(bytearray(bytes(ev_tab)), dtype=torch.uint8).to(dev)
        ktype = torch.int32 if c.use_float32 else torch.int64
        self.d_keys = torch.zeros(self.n, dtype=ktype, device=dev)
        self.d_ctl = torch.zeros(ctypes.sizeof(_Ctl), dtype=torch.uint8, device=dev)
        self.d_active = torch.zeros(self.n, dtype=torch.int32, device=dev)
        self.d_prefix = torch.zeros(self.n + 1, dtype=torch.int64, device=dev)
        self.d_loops = torch.full((self.n,), -1, dtype=torch.int32, device=dev)
        self.max_loops = int(max_loops)
        # without the freeze-out stop every event runs max_loops steps
        self.stop_at_freezeout = bool(stop_at_freezeout)
        if not self.stop_at_freezeout and self.max_loops < 0:
            raise ValueError('stop_at_freezeout=False needs max_loops >= 0')
        self.hist_cap = 0
        self.d_history = torch.zeros(1, dtype=torch.float64, device=dev)
        self.block_size = block_size
        self.grid_blocks = grid_blocks
        self.max_registers = int(max_registers)
        self.tile = None if tile is None else (int(tile[0]), int(tile[1]))
        if launch is not None:
            self._set_launch(tuple(launch))
        if self.tile is not None and not self.all_2d:
            raise ValueError('the tiled batch kernel takes (2+1)D events (nz = 1) only')
        self.tuning = None
        self._graph = None
        self._h_ctl = torch.zeros(ctypes.sizeof(_Ctl), dtype=torch.uint8).pin_memory()
        # CLVisc construction on the still empty state (visc.py:101-102)
        self.IS_initialize()
        self._ideal_predict_for_first_step()

    # ----------------------------------------------------------- helpers
    @property
    def stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _ptr(self, t, elem_off=0):
        return ctypes.c_void_p(t.data_ptr() + elem_off * t.element_size())

    def _call(self, name, p, *args):
        _lib.check(getattr(self.lib, name)(ctypes.byref(p), *args), name)

    def _view(self, arena, e, kind):
        """Event e's planes of an arena as a (w, ld_e) tensor view; kind is
        'ev' (ev slots, udiff: 4 planes), 'pi' (npi planes) or 'src'."""
        ld, oe, op, os_, _ = self.layout[e]
        off, w = {'ev': (oe, 4), 'pi': (op, self.npi), 'src': (os_, 4 + self.npi)}[kind]
        return arena[off:off + w * ld].view(w, ld)

    def IS_initialize(self):
        """Navier-Stokes pi (and Pi) of every event from its d_ev[1] (visc.py:143-149)."""
        for e in range(self.n):
            p = self.event_params[e]
            self._call('clv_visc_initialize', p, _lib.ptr(self._view(self.d_pi[1], e, 'pi')),
                       self._ptr(self.d_goodcell, self.layout[e][4]), _lib.ptr(self._view(self.d_udiff, e, 'ev')),
                       _lib.ptr(self._view(self.d_ev[1], e, 'ev')), float(self.cfg.real(self.cfg.TAU0)), self.stream)

    def _ideal_predict_for_first_step(self):
        """One ideal stage per event into d_ev[2] (visc.py:468-470); the event's
        source block serves as the ideal stage's d_Src."""
        for e in range(self.n):
            p = self.event_params[e]
            ev1 = self._view(self.d_ev[1], e, 'ev')
            self._call('clv_ideal_stage', p, 1, float(self.cfg.real(self.cfg.TAU0)), _lib.ptr(ev1), _lib.ptr(ev1),
                       _lib.ptr(self._view(self.d_ev[2], e, 'ev')), _lib.ptr(self._view(self.d_src, e, 'src')),
                       1, None, self.stream)

    def load_ini(self, e, dat):
        """Event e's (cells, 4) array of (ed, vx, vy, veta) into its d_ev[1]
        (ideal.py:138-144)."""
        n = self.sizes[e]
        if isinstance(dat, torch.Tensor):
            src = dat.to(self.device, self.dtype).reshape(n, 4).contiguous()
        else:
            host = torch.from_numpy(np.ascontiguousarray(dat, dtype=self.cfg.real).reshape(n, 4))
            src = host.pin_memory().to(self.device, non_blocking=True)
        self._call('clv_aos_to_soa', self.event_params[e], _lib.ptr(src), _lib.ptr(self._view(self.d_ev[1], e, 'ev')),
                   n, 4, self.stream)
        if not isinstance(dat, torch.Tensor):
            torch.cuda.current_stream(self.device).synchronize()

    def load_hotspot_event(self, e, b=8.0, seed=5, edmax=50.0):
        """Event e's d_ev[1] = initial.glauber_event(nx, ny, nz, DX, DY, DZ, b,
        seed, edmax), summed on the device from host-sampled participants."""
        from .initial import hotspot_ini, hotspot_table
        c = self.cfg
        keep = hotspot_ini(self.lib, self.event_params[e], self._view(self.d_ev[1], e, 'ev'), hotspot_table(b, seed),
                           c.DX, c.DY, c.DZ, edmax=edmax, stream=self.stream)
        self._keep = keep  # released by the next call, after the stream has used it

    def _batch(self):
        b = _Batch()
        b.events = self.d_events.data_ptr()
        b.n_events = self.n
        for k in range(3):
            b.ev[k] = self.d_ev[k].data_ptr()
            b.pi[k] = self.d_pi[k].data_ptr()
        b.src = self.d_src.data_ptr()
        b.udiff = self.d_udiff.data_ptr()
        b.goodcell = self.d_goodcell.data_ptr()
        b.keys = self.d_keys.data_ptr()
        b.ctl = self.d_ctl.data_ptr()
        b.active = self.d_active.data_ptr()
        b.prefix = self.d_prefix.data_ptr()
        b.loops = self.d_loops.data_ptr()
        b.history = self.d_history.data_ptr()
        b.hist_cap = self.hist_cap
        b.tau0 = float(self.cfg.TAU0)
        b.dt = float(self.cfg.DT)
        b.efrz = float(self.efrz) if self.stop_at_freezeout else -1.0e300
        b.ntskip = int(self.cfg.ntskip)
        b.max_loops = self.max_loops
        return b

    @property
    def all_2d(self):
        return all(g[2] == 1 for g in self.grids)

    def _launch_step(self, b, shape):
        """One fused step (both stages and the stop test) with a launch shape."""
        for step in (1, 2):
            if shape[0] == 'tile':
                _, rows, chunk, grid = shape
                _lib.check(self.lib.clv_batch_stage_tiled(ctypes.byref(self.params), step, ctypes.byref(b), int(rows),
                                                          int(chunk), int(grid), self.stream), 'clv_batch_stage_tiled')
            else:
                _, bs, grid, regs = shape
                _lib.check(self.lib.clv_batch_stage(ctypes.byref(self.params), step, ctypes.byref(b), int(bs),
                                                    int(grid), int(regs), self.stream), 'clv_batch_stage')
        _lib.check(self.lib.clv_batch_advance(ctypes.byref(self.params), ctypes.byref(b), 0, self.stream),
                   'clv_batch_advance')

    def occupancy(self, bs, regs=0):
        """Resident stage-kernel blocks per SM at bs threads (regs: 0, or 128
        for the register-capped FP32 variant)."""
        n = ctypes.c_int()
        _lib.check(self.lib.clv_batch_occupancy(ctypes.byref(self.params), int(bs), int(regs), ctypes.byref(n)),
                   'clv_batch_occupancy')
        return n.value

    def occupancy_tiled(self, rows):
        """Resident tiled stage-kernel blocks per SM at `rows` threads a block."""
        n = ctypes.c_int()
        _lib.check(self.lib.clv_batch_occupancy_tiled(ctypes.byref(self.params), int(rows), ctypes.byref(n)),
                   'clv_batch_occupancy_tiled')
        return n.value

    def tiles(self, rows, chunk):
        """Work items of the tiled kernel at a (rows, chunk) shape."""
        ti = rows - 4
        return sum(((ny + ti - 1) // ti) * ((nx + chunk - 1) // chunk) for nx, ny, _ in self.grids)

    def _set_launch(self, shape):
        if shape[0] == 'tile':
            self.tile = (int(shape[1]), int(shape[2]))
            self.grid_blocks = shape[3]
        else:
            self.tile = None
            self.block_size, self.grid_blocks, self.max_registers = shape[1], shape[2], int(shape[3])

    @property
    def launch(self):
        """The launch shape evolve() uses: ('tile', rows, chunk, grid) or
        ('cell', block, grid, max_registers)."""
        sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        if self.tile is not None:
            if self.grid_blocks is None:
                self.grid_blocks = sms * max(1, self.occupancy_tiled(self.tile[0]))
            return ('tile', self.tile[0], self.tile[1], int(self.grid_blocks))
        if self.block_size is None:
            self.block_size = 128
        if self.grid_blocks is None:
            self.grid_blocks = sms * max(1, self.occupancy(self.block_size, self.max_registers))
        return ('cell', int(self.block_size), int(self.grid_blocks), int(self.max_registers))

    # ------------------------------------------------------------- evolve
    def _start(self, hist_cap):
        """Initial maxima (ideal.py:257-262 per event), control block reset and
        the stop test at step 0."""
        self.hist_cap = int(hist_cap)
        need = max(1, self.hist_cap * self.n * 2)
        if self.d_history.numel() != need:
            self.d_history = torch.zeros(need, dtype=torch.float64, device=self.device)
        else:
            self.d_history.zero_()
        self.d_keys.zero_()
        for e in range(self.n):
            self._call('clv_max_ed', self.event_params[e], _lib.ptr(self._view(self.d_ev[1], e, 'ev')),
                       self._ptr(self.d_keys, e), self.stream)
        self.d_ctl.zero_()
        self.d_loops.fill_(-1)
        b = self._batch()
        _lib.check(self.lib.clv_batch_advance(ctypes.byref(self.params), ctypes.byref(b), 1, self.stream),
                   'clv_batch_advance')
        return b

    def _ctl(self):
        self._h_ctl.copy_(self.d_ctl, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        return _Ctl.from_buffer_copy(bytes(self._h_ctl.numpy().tobytes()))

    def evolve(self, hist_cap=None, use_graph=True, steps_per_check=None):
        """Advance every event until it freezes out (or max_loops); returns the
        number of steps the batch took."""
        c = self.cfg
        if hist_cap is None:
            hist_cap = (self.max_loops // c.ntskip + 2) if self.max_loops >= 0 else 4096
        b = self._start(hist_cap)
        shape = self.launch
        k = int(steps_per_check or c.ntskip)
        if use_graph:
            key = (shape, k, self.hist_cap, self.d_history.data_ptr())
            if self._graph is None or self._graph_key != key:
                self._graph = None
                # loads the stage kernel (and sets its shared-memory size) before the capture
                if shape[0] == 'tile':
                    self.occupancy_tiled(shape[1])
                else:
                    self.occupancy(shape[1], shape[3])
                s = torch.cuda.Stream(self.device)
                s.wait_stream(torch.cuda.current_stream(self.device))
                g = torch.cuda.CUDAGraph()
                with torch.cuda.stream(s):
                    with torch.cuda.graph(g, stream=s):
                        for _ in range(k):
                            self._launch_step(b, shape)
                torch.cuda.current_stream(self.device).wait_stream(s)
                self._graph, self._graph_key = g, key
            while not self._ctl().done:
                self._graph.replay()
        else:
            while not self._ctl().done:
                for _ in range(k):
                    self._launch_step(b, shape)
        return self._ctl().loop

    # ------------------------------------------------------------ results
    def loops(self):
        """Steps each event took before it stopped."""
        return self.d_loops.cpu().numpy()

    def history(self, e):
        """Event e's [tau, max energy density] at every stop test (CLVisc.ideal.history)."""
        n = self._ctl().hist_len
        h = self.d_history[:n * self.n * 2].view(n, self.n, 2)[:, e].cpu().numpy()
        return h[h[:, 0] > 0].astype(self.cfg.real)  # rows after the event stopped stay zero

    def field_to_host(self, arena, e, kind):
        t = self._view(arena, e, kind)
        w = t.shape[0]
        n = self.sizes[e]
        aos = torch.empty((n, w), dtype=self.dtype, device=self.device)
        self._call('clv_soa_to_aos', self.event_params[e], _lib.ptr(t), _lib.ptr(aos), n, w, self.stream)
        return aos.cpu().numpy()

    def ev_to_host(self, e, slot=1):
        return self.field_to_host(self.d_ev[slot], e, 'ev')

    def pi_to_host(self, e, slot=1):
        return self.field_to_host(self.d_pi[slot], e, 'pi')[:, :10]

    def bulk_to_host(self, e, slot=1):
        if not self.bulk:
            return np.zeros(self.sizes[e], self.cfg.real)
        return self.field_to_host(self.d_pi[slot], e, 'pi')[:, 10]

    # ------------------------------------------------------------ tuning
    def _snapshot(self):
        names = ('d_src', 'd_udiff', 'd_goodcell', 'd_keys', 'd_ctl', 'd_active', 'd_prefix', 'd_loops', 'd_history')
        snap = {n: getattr(self, n).clone() for n in names}
        snap['d_ev'] = [t.clone() for t in self.d_ev]
        snap['d_pi'] = [t.clone() for t in self.d_pi]
        return snap

    def _restore(self, snap):
        for n, v in snap.items():
            if isinstance(v, list):
                for dst, src in zip(getattr(self, n), v):
                    dst.copy_(src)
            else:
                getattr(self, n).copy_(v)

    def candidates(self, block_sizes=(64, 128, 256), rows=(64, 128), chunks=(4, 8, 16, 32)):
        """Launch shapes autotune() times. One thread per cell: every block
        size with persistent grids of 1..occupancy blocks per SM and the
        one-cell-per-thread grid, without and (FP32) with a 128-register cap
        (and a 168-register cap below 256 threads). Tiled ((2+1)D batches only): rows x chunks, each with the grid
        that fills the GPU once and the one-tile-per-block grid."""
        sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        out = []
        total = sum(self.sizes)
        caps = (0, 128, 168) if self.cfg.use_float32 else (0,)
        for regs in caps:
            for bs in block_sizes:
                if regs == 168 and bs == 256:
                    continue
                occ = max(1, self.occupancy(bs, regs))
                for grid in sorted({sms * k for k in range(1, occ + 1)} | {(total + bs - 1) // bs}):
                    out.append(('cell', bs, grid, regs))
        if self.all_2d:
            for r in rows:
                fill = sms * max(1, self.occupancy_tiled(r))
                for ch in chunks:
                    for grid in sorted({fill, self.tiles(r, ch)}):
                        out.append(('tile', r, ch, grid))
        return out

    def autotune(self, steps=4, cands=None):
        """Choose the stage kernel and its launch shape by timing `steps`
        steps of this batch for each candidate of candidates() (state
        restored after each); call after load_ini. Returns {shape: ms per
        step}; the fastest becomes self.launch."""
        hist = self.hist_cap
        b = self._start(max(hist, steps // self.cfg.ntskip + 2))
        snap = self._snapshot()
        results = {}
        for shape in (cands or self.candidates()):
            self._launch_step(b, shape)  # warm-up
            torch.cuda.synchronize(self.device)
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            t0.record()
            for _ in range(steps):
                self._launch_step(b, shape)
            t1.record()
            torch.cuda.synchronize(self.device)
            results[shape] = t0.elapsed_time(t1) / steps
            self._restore(snap)
        self._set_launch(min(results, key=results.get))
        self.tuning = results
        self._graph = None
        return results

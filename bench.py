"""Benchmark: viscous (3+1)D hydro step, cell-updates per second.

Workload (the large single event): 385 x 385 x 115 cells, dx = dy = 0.08 fm,
deta = 0.15, dtau = 0.01 fm, tau0 = 0.6 fm, eta/s = 0.08, s95p-PCE165 EOS,
FP32, seeded Pb+Pb initial condition (seed 5, b = 8 fm, peak 50 GeV/fm^3).
One step = one full Runge-Kutta time step (both stages, Israel-Stewart and
Kurganov-Tadmor parts), i.e. one cell-update per cell.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

value: cell-updates/s over the K timed steps with the state resident in HBM
(CUDA events on the launch stream, max over ranks). e2e: the same metric
through the public API with host buffers: load_ini from pinned host memory,
CLVisc.evolve for K steps, ev_to_host. With N > 1 every rank advances its own
replica of the event (weak scaling; the path has no exchange step).
--impl reference times the oracle (the C++/OpenMP restatement of the
reference kernels, all host threads) on the same whole workload, the same
warm-up and timed step counts.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX, NY, NZ = 385, 385, 115
DX, DZ, DT = 0.08, 0.15, 0.01
METRIC = 'viscous cell-updates/s (385x385x115)'
UNIT = 'cell-updates/s'
# bytes per cell-update the step must move, FP32: 78 reals (5S + 2U with
# S = 14 state reals, U = 4 udiff reals; the stencil halo and EOS table
# counted as cache hits)
ALG_BYTES_PER_CELL_UPDATE = 312


def make_cfg(nz=NZ, out='/tmp/clv_bench', nx=NX, ny=NY, fp64=False, arithmetic='fast'):
    from clvisc_b200.config import read_config, set_real
    cfg = read_config([])
    cfg.arithmetic = arithmetic
    cfg.NX, cfg.NY, cfg.NZ = nx, ny, nz
    cfg.DX = cfg.DY = DX
    cfg.DZ = DZ
    cfg.DT = DT
    cfg.TAU0 = 0.6
    cfg.eos_type = 'lattice_pce165'
    cfg.use_float32 = not fp64
    cfg.ETAOS_XMIN, cfg.ETAOS_YMIN, cfg.ETAOS_LEFT_SLOP, cfg.ETAOS_RIGHT_SLOP = 0.18, 0.08, 0.0, 0.0
    cfg.TFRZ = 0.137
    cfg.ntskip = 20
    cfg.nxskip = cfg.nyskip = 2
    cfg.nzskip = 1
    cfg.fPathOut = out
    return set_real(cfg)


def initial_condition(seed=5, nx=NX, ny=NY, nz=NZ):
    from clvisc_b200.initial import glauber_event
    return glauber_event(nx, ny, nz, DX, DX, DZ, b=8.0, seed=seed, edmax=50.0)


class ClockSampler(object):
    """SM clock and throttle reasons sampled during the timed region: NVML
    (read-only queries) every 20 ms from a thread, so that a timed region of a
    fraction of a second still holds several samples; nvidia-smi every 200 ms
    where NVML cannot be loaded."""

    Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
         'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
         'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')
    REASONS = (('hw_slowdown', 0x8), ('hw_thermal_slowdown', 0x40), ('sw_thermal_slowdown', 0x20),
               ('sw_power_cap', 0x4))

    def __init__(self, gpu_index):
        self.gpu = int(gpu_index)
        self.proc = None
        self.lines = []
        self.samples = []  # (sm MHz, max sm MHz, reason bits)
        self.stop = threading.Event()
        self.nvml = None

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            # the CUDA ordinal may differ from NVML's index when
            # CUDA_VISIBLE_DEVICES is set: find the device by its UUID
            h = None
            try:
                import torch
                u = str(torch.cuda.get_device_properties(self.gpu).uuid)
                h = pynvml.nvmlDeviceGetHandleByUUID(u if u.startswith('GPU-') else 'GPU-' + u)
            except Exception:
                h = None
            self.h = h if h is not None else pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.gpu), '--query-gpu=' + self.Q,
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def sample_now(self):
        n = self.nvml
        if n is None:
            return
        try:
            sm = n.nvmlDeviceGetClockInfo(self.h, n.NVML_CLOCK_SM)
            smax = n.nvmlDeviceGetMaxClockInfo(self.h, n.NVML_CLOCK_SM)
            r = n.nvmlDeviceGetCurrentClocksEventReasons(self.h)
            self.samples.append((float(sm), float(smax), int(r)))
        except Exception:
            pass

    def _poll(self):
        while not self.stop.is_set():
            self.sample_now()
            self.stop.wait(0.02)

    def wait_for(self, event, every=0.01):
        """Wait for a CUDA event, sampling the clocks from this thread every
        `every` seconds meanwhile (the queued work is running): the polling
        thread alone can be starved while the launching thread holds the
        interpreter."""
        while not event.query():
            self.sample_now()
            time.sleep(every)

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        self.stop.set()
        if self.nvml is not None:
            self.t.join(timeout=2)
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        sm, smax, reasons = [], [], set()
        for f, fm, r in self.samples:
            sm.append(f)
            smax.append(fm)
            for name, bit in self.REASONS:
                if r & bit:
                    reasons.add(name)
        names = [n for n, _ in self.REASONS]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(',')]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == 'active':
                    reasons.add(n)
        if not sm:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': [], 'samples': 0}
        return {'sm_mhz': statistics.median(sm), 'sm_max_mhz': max(smax), 'reasons': sorted(reasons),
                'samples': len(sm), 'source': 'nvml' if self.samples else 'nvidia-smi'}


def read_peaks():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as f:
            p = json.load(f)
        return float(p['hbm_gbs']), 'measured'
    except (OSError, KeyError, ValueError):
        return 6650.0, 'fallback'


def read_profile_value(key, arithmetic='fast', precision='fp32'):
    """A per-cell-update figure of the stage kernel from the committed ncu
    summary of that arithmetic and precision
    (profiles/visc_stage_tiled_<arithmetic>_*_<precision>.txt, a line
    'key: X'), or None."""
    d = os.path.join(ROOT, 'profiles')
    try:
        for fn in sorted(os.listdir(d)):
            if fn.startswith('visc_stage_tiled_%s_' % arithmetic) and fn.endswith('_%s.txt' % precision):
                for ln in open(os.path.join(d, fn)):
                    if ln.startswith(key + ':'):
                        return float(ln.split(':')[1])
    except OSError:
        pass
    return None


def read_traffic(arithmetic='fast', precision='fp32'):
    """DRAM bytes per cell-update of the stage kernel (committed ncu summary)."""
    return read_profile_value('dram_bytes_per_cell_update', arithmetic, precision)


def issue_roofline(cell_updates_per_s, sm_mhz, arithmetic='fast', precision='fp32'):
    """Warp instructions issued per second by the stage kernel (instructions
    per cell-update from the committed ncu summary, divided by 32, times
    cell-updates/s) against the SMs' issue peak: 4 schedulers x 1 warp
    instruction per cycle x the SM count x the SM clock sampled in the timed
    region."""
    import torch
    inst = read_profile_value('instructions_per_cell_update', arithmetic, precision)
    if inst is None or not sm_mhz:
        return None
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    achieved = inst / 32.0 * cell_updates_per_s
    peak = 4.0 * sms * sm_mhz * 1e6
    return {'achieved': achieved, 'peak': peak, 'unit': 'warp instructions/s', 'frac': achieved / peak,
            'instructions_per_cell_update': inst, 'sm_mhz': sm_mhz}


def time_steps(v, warmup, steps, first=0):
    """ms per fused step of the CLVisc v over `steps` steps after `warmup`
    (CUDA events on the launch stream)."""
    import torch
    stream = torch.cuda.current_stream()
    for n in range(first, first + warmup):
        v.step(n)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for n in range(first + warmup, first + warmup + steps):
        v.step(n)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def fp64_leg(nx, ny, nz, ic, peak, steps=5, warmup=2):
    """The same workload in FP64, both arithmetics: ms per step, cell-updates/s
    and the HBM fraction at 624 B per cell-update."""
    import torch
    from clvisc_b200.visc import CLVisc
    out = {}
    for arith in ('exact', 'fast'):
        cfg = make_cfg(nz=nz, nx=nx, ny=ny, out='/tmp/clv_bench_fp64', fp64=True, arithmetic=arith)
        v = CLVisc(cfg)
        v.load_ini(ic)
        ms = time_steps(v, warmup, steps)
        rate = nx * ny * nz / (ms * 1e-3)
        ach = rate * 2 * ALG_BYTES_PER_CELL_UPDATE / 1e9
        t = read_traffic(arith, 'fp64')
        out[arith] = {'ms_per_step': ms, 'cell_updates_per_s': rate, 'steps': steps, 'warmup': warmup,
                      'roofline': {'achieved': ach, 'peak': peak, 'unit': 'GB/s', 'frac': ach / peak,
                                   'alg_bytes_per_cell_update': 2 * ALG_BYTES_PER_CELL_UPDATE,
                                   'traffic_bytes_per_cell_update': t}}
        del v
        torch.cuda.synchronize()
    out['default'] = 'fast (cfg.arithmetic)'
    return out


def cpu_baseline(steps=5, warmup=0, nx=NX, ny=NY, nz=NZ, ic=None):
    """The oracle (the C++/OpenMP restatement of the reference kernels and
    its orchestration, all host threads) on the whole workload: the same grid,
    initial condition and step as the GPU arm, `warmup` untimed steps, then
    `steps` timed steps."""
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import oracle as O
    cfg = make_cfg(nz=nz, nx=nx, ny=ny, arithmetic='exact')
    if ic is None:
        ic = initial_condition(nx=nx, ny=ny, nz=nz)
    o = O.OracleVisc(cfg)
    o.load_ini(ic)
    for n in range(warmup):
        o.step(n)
    t = time.perf_counter()
    for n in range(warmup, warmup + steps):
        o.step(n)
    dt = time.perf_counter() - t
    cores = int(os.environ.get('OMP_NUM_THREADS', os.cpu_count() or 1))
    cells = nx * ny * nz
    return {'value': cells * steps / dt, 'unit': UNIT, 'cores': cores, 'kind': 'port',
            'sample': '%d steps (after %d untimed) of the whole %dx%dx%d event (oracle, OpenMP, %d threads)'
                      % (steps, warmup, nx, ny, nz, cores),
            'seconds': dt}


def workload_config(nx, ny, nz, fp64, world):
    """The `config` object of both arms' lines."""
    return {'workload': 'viscous %dx%dx%d Pb+Pb b=8 fm seed 5, %s, lattice EOS, dtau=0.01'
                        % (nx, ny, nz, 'FP64' if fp64 else 'FP32'),
            'cells': nx * ny * nz, 'l2': 'inputs larger than L2 (state 0.95 GB per stage)',
            'parallelism': 'replicas x%d' % world}


def max_over_ranks(x, dist):
    """The maximum of a per-rank float over all ranks (x itself with one rank)."""
    if dist is None:
        return x
    import torch
    dev = 'cuda' if dist.get_backend() == 'nccl' else 'cpu'
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(cells, steps, ms, world):
    """Whole-job cell-updates/s: every rank advances its own replica of
    `cells` cells for `steps` steps; `ms` is the slowest rank's time."""
    return world * cells * steps / (ms * 1e-3)


def run_reference(args, rank, world):
    if rank != 0:
        return
    nx, ny, nz = args.grid
    cb = cpu_baseline(steps=max(1, args.steps), warmup=args.warmup, nx=nx, ny=ny, nz=nz)
    line = {'impl': 'reference', 'metric': METRIC, 'value': cb['value'], 'unit': UNIT, 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': 1e3 * cb['seconds'] / max(1, args.steps),
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
            'config': workload_config(nx, ny, nz, False, world),
            'arithmetic': 'the reference\'s (oracle)',
            'cpu_baseline': {k: cb[k] for k in ('value', 'unit', 'cores', 'kind', 'sample')},
            'e2e': {'value': cb['value'], 'unit': UNIT, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)


# The batched workload: 64 seeded (2+1)D Pb+Pb events, NX = NY odd in
# [121, 301], b uniform in [0, 12] fm (both drawn from default_rng(seed)),
# seeds 1000..1063, dx = 0.16 fm, dtau = 0.02 fm, eta/s = 0.16, zeta/s a
# skewed-Cauchy peak of 0.05 at T = 0.18 GeV (width 0.02 GeV), lattice EOS,
# FP32, every event run to freeze-out (T < 137 MeV).
BATCH_EVENTS = 64


def batch_event_spec(e):
    import numpy as np
    rng = np.random.default_rng(1000 + e)
    n = 2 * int(rng.integers(60, 151)) + 1
    return n, float(rng.uniform(0.0, 12.0)), 1000 + e


def batch_cfg(n=121):
    from clvisc_b200.config import read_config, set_real
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
    cfg.fPathOut = '/tmp/clv_bench_batch'
    return set_real(cfg)


def launch_name(shape):
    """'tile<rows-4>x<chunk>/g<grid>' (tiled (2+1)D kernel) or
    '<block>x<grid>/r<max_registers>' (one thread per cell)."""
    if shape[0] == 'tile':
        return 'tile%dx%d/g%d' % (shape[1] - 4, shape[2], shape[3])
    return '%dx%d/r%d' % shape[1:]


def run_batch(n_events=BATCH_EVENTS, one_at_a_time=True, launch=None):
    """events/h of the batched runner against CLVisc one event at a time;
    launch: a fixed launch shape (('tile', rows, chunk, grid) or ('cell',
    block, grid, max_registers)) in place of the autotuner's choice."""
    import numpy as np
    import torch
    from clvisc_b200.batch import CLViscBatch
    from clvisc_b200.initial import glauber_event
    from clvisc_b200.visc import CLVisc
    specs = [batch_event_spec(e) for e in range(n_events)]
    t = time.perf_counter()
    ics = [glauber_event(n, n, 1, 0.16, 0.16, 0.15, b=bb, seed=sd, edmax=50.0) for n, bb, sd in specs]
    ic_s = time.perf_counter() - t
    grids = [(n, n, 1) for n, _, _ in specs]
    cfg = batch_cfg()
    out = {'metric': 'events/h (%d seeded (2+1)D events, 121^2..301^2, to freeze-out)' % n_events,
           'unit': 'events/h', 'events': n_events, 'cells': int(sum(n * n for n, _, _ in specs)),
           'arithmetic': 'exact' if cfg.arithmetic == 'exact' else 'fast',
           'ic_host_s': ic_s}
    # autotuned launch shape (timed separately), then the timed batch from host arrays
    if launch is None:
        bt = CLViscBatch(cfg, grids)
        for e, ic in enumerate(ics):
            bt.load_ini(e, ic)
        t = time.perf_counter()
        tuning = bt.autotune(steps=3)
        out['autotune_s'] = time.perf_counter() - t
        shape = bt.launch
        out['launch'] = {'shape': launch_name(shape),
                         'candidates_ms_per_step': {launch_name(k): round(v, 4) for k, v in sorted(tuning.items())}}
        del bt
    else:
        shape = launch
        out['launch'] = {'shape': launch_name(shape), 'given': True}
    torch.cuda.synchronize()
    t = time.perf_counter()
    bt = CLViscBatch(cfg, grids, launch=shape)
    for e, ic in enumerate(ics):
        bt.load_ini(e, ic)
    t_solve = time.perf_counter()
    steps = bt.evolve()
    torch.cuda.synchronize()
    t_solved = time.perf_counter()
    finals = [bt.ev_to_host(e) for e in range(n_events)]
    t_end = time.perf_counter()
    loops = bt.loops()
    out.update({'value': n_events / (t_solved - t_solve) * 3600.0, 'solve_s': t_solved - t_solve,
                'e2e': {'value': n_events / (t_end - t) * 3600.0, 'unit': 'events/h', 'seconds': t_end - t,
                        'h2d_bytes': int(sum(ic.nbytes for ic in ics)),
                        'd2h_bytes': int(sum(f.nbytes for f in finals))},
                'batch_steps': int(steps), 'event_steps': [int(x) for x in loops],
                'cell_updates_per_s': float(sum(n * n * int(l) for (n, _, _), l in zip(specs, loops)) /
                                            (t_solved - t_solve))})
    out['nan_values'] = int(sum(np.count_nonzero(np.isnan(g)) for g in finals))
    # end to end from the seeds: participants sampled on the host, the energy
    # density summed on the device (clv_hotspot_ini), evolve, results to host
    del bt
    torch.cuda.synchronize()
    t = time.perf_counter()
    bt = CLViscBatch(cfg, grids, launch=shape)
    for e, (n, bb, sd) in enumerate(specs):
        bt.load_hotspot_event(e, b=bb, seed=sd, edmax=50.0)
    bt.evolve()
    finals2 = [bt.ev_to_host(e) for e in range(n_events)]
    t2 = time.perf_counter() - t
    out['e2e_from_seeds'] = {'value': n_events / t2 * 3600.0, 'unit': 'events/h', 'seconds': t2,
                             'initial_condition': 'participants on the host, energy density on the device',
                             'nan_values': int(sum(np.count_nonzero(np.isnan(g)) for g in finals2))}
    del bt
    if one_at_a_time:
        torch.cuda.synchronize()
        t = time.perf_counter()
        differ = 0
        singles = []
        for e, ic in enumerate(ics):
            v = CLVisc(batch_cfg(specs[e][0]))
            v.load_ini(ic)
            v.evolve(save_hypersf=False)
            singles.append(v.ideal.ev_to_host())
        t1 = time.perf_counter() - t
        worst = 0.0
        for f, g in zip(singles, finals):  # bit patterns, so that NaN equals NaN
            differ += int(np.count_nonzero(f.view(np.uint32) != g.view(np.uint32)))
            worst = max(worst, float(np.abs(f[:, 0].astype(np.float64) - g[:, 0]).max() / max(np.abs(g[:, 0]).max(),
                                                                                                  1e-30)))
        out['one_at_a_time'] = {'value': n_events / t1 * 3600.0, 'unit': 'events/h', 'seconds': t1,
                                'api': 'CLVisc(cfg); load_ini; evolve(save_hypersf=False); ev_to_host per event',
                                'bitwise_equal_to_batch': differ == 0, 'values_differing': differ,
                                'max_scaled_energy_density_difference': worst}
        out['speedup_e2e'] = out['e2e']['value'] / out['one_at_a_time']['value']
    return out


def evolve_to_freezeout(args, nx, ny, nz):
    """The whole event: CLVisc.evolve from the initial condition until the
    maximum energy density is below freeze-out, with the T = 0.137 GeV
    hypersurface extracted every ntskip steps and written (visc.py:473-560);
    wall time around construction, load_ini and evolve."""
    import torch
    from clvisc_b200.visc import CLVisc
    cfg = make_cfg(nz=nz, nx=nx, ny=ny, out='/tmp/clv_bench_evolve', fp64=args.fp64)
    ic = initial_condition(seed=5, nx=nx, ny=ny, nz=nz)
    torch.cuda.synchronize()
    t = time.perf_counter()
    # this event's surface (about 1.6 M elements) exceeds the reference's
    # capacity of 1.5 M, which this library reports instead of truncating
    v = CLVisc(cfg, hypersf_capacity=4000000)
    v.load_ini(ic)
    v.evolve(max_loops=4000, save_hypersf=True, save_bulk=False)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t
    steps = int(round((float(v.ideal.tau) - cfg.TAU0) / cfg.DT))
    return {'wall_s': wall, 'steps': steps, 'tau_end': float(v.ideal.tau),
            'hypersurface_elements': int(v.ideal.num_of_sf),
            'cell_updates_per_s': nx * ny * nz * steps / wall}


def run_gpu(args, rank, world, dist):
    import numpy as np
    import torch
    from clvisc_b200.visc import CLVisc
    dev = int(os.environ.get('LOCAL_RANK', 0))
    torch.cuda.set_device(dev)
    nx, ny, nz = args.grid
    cfg = make_cfg(nz=nz, nx=nx, ny=ny, out='/tmp/clv_bench_r%d' % rank, fp64=args.fp64, arithmetic=args.arithmetic)
    ic = initial_condition(seed=5, nx=nx, ny=ny, nz=nz)
    v = CLVisc(cfg, gpu_id=dev)
    v.load_ini(ic)
    stream = torch.cuda.current_stream()
    cells = nx * ny * nz

    def barrier():
        if dist is not None:
            dist.barrier()

    # device-resident timing: K fused steps
    for n in range(args.warmup):
        v.step(n)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clocks:
        e0.record(stream)
        for n in range(args.warmup, args.warmup + args.steps):
            v.step(n)
        e1.record(stream)
        clocks.wait_for(e1)
        torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), dist)
    barrier()
    value = aggregate_rate(cells, args.steps, ms, world)

    if args.no_e2e:
        if rank == 0:
            print(json.dumps({'metric': METRIC, 'value': value, 'unit': UNIT, 'ms_per_step': ms / args.steps,
                              'config': {'grid': [nx, ny, nz]}, 'gpu_launches': 2 * args.steps}), flush=True)
        return
    # end to end through the public API with host buffers
    host_ic = torch.from_numpy(np.ascontiguousarray(ic, dtype=cfg.real)).pin_memory()
    host_out = torch.empty((cells, 4), dtype=v.dtype, pin_memory=True)  # the result's pinned destination
    v2 = CLVisc(cfg, gpu_id=dev)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    v2.load_ini(host_ic)
    v2.evolve(max_loops=args.steps, force_run_to_maxloop=True, save_hypersf=False, save_pi=False)
    out = v2.ideal.ev_to_host(out=host_out)
    f1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(f0.elapsed_time(f1), dist)
    e2e_wall = time.perf_counter() - t0
    e2e = aggregate_rate(cells, args.steps, e2e_ms, world)
    h2d = ic.nbytes / args.steps
    d2h = out.nbytes / args.steps

    peak, peak_kind = read_peaks()
    # FP64 moves twice the bytes
    alg = ALG_BYTES_PER_CELL_UPDATE * (2 if args.fp64 else 1)
    achieved = value / world * alg / 1e9
    arith = 'fast' if v.params.flags & 32 else 'exact'
    precision = 'fp64' if args.fp64 else 'fp32'
    traffic = read_traffic(arith, precision)
    real = 'double' if args.fp64 else 'float'
    if rank == 0:
        line = {
            'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': ms / args.steps, 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'f64' if args.fp64 else 'f32', 'data': 'synthetic',
            'config': workload_config(nx, ny, nz, args.fp64, world),
            'arithmetic': 'fast' if v.params.flags & 32 else 'exact',
            'e2e': {'value': e2e, 'unit': UNIT, 'h2d_bytes_per_step': h2d, 'd2h_bytes_per_step': d2h,
                    'wall_s': e2e_wall},
            'gpu_launches': 2 * args.steps,
            'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                         'frac': achieved / peak, 'peak_kind': peak_kind,
                         'traffic': None if traffic is None else traffic * cells / 2,
                         'alg_bytes_per_launch': alg * cells / 2,
                         'kernel': 'clv::%s::visc_stage_tiled_kernel<%s,IS,KT> (2 launches per step)' % (arith, real)},
            'clocks': clocks.summary(),
        }
        line['roofline']['issue'] = issue_roofline(value / world, line['clocks'].get('sm_mhz'), arith, precision)
        if not args.fp64 and not args.no_fp64 and world == 1:
            line['fp64'] = fp64_leg(nx, ny, nz, ic, peak)
        if args.evolve and world == 1:
            line['evolve'] = evolve_to_freezeout(args, nx, ny, nz)
        if not args.no_cpu_baseline and not args.fp64:
            cb = cpu_baseline(steps=5, nx=nx, ny=ny, nz=nz, ic=ic)
            line['cpu_baseline'] = {k: cb[k] for k in ('value', 'unit', 'cores', 'kind', 'sample')}
        if args.batch_events > 0 and world == 1:
            line['batch'] = run_batch(args.batch_events, one_at_a_time=not args.no_one_at_a_time)
        if args.surrogate_train > 0 and world == 1:
            from clvisc_b200.surrogate import run_experiment
            line['surrogate'] = run_experiment(args.surrogate_train, args.surrogate_test, args.surrogate_epochs,
                                               log=lambda m: print(m, file=sys.stderr, flush=True))
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=50)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-e2e', action='store_true', help='device-timed steps only (profiling runs)')
    ap.add_argument('--batch-events', type=int, default=BATCH_EVENTS,
                    help='events of the batched workload reported under "batch" (0: skip)')
    ap.add_argument('--no-one-at-a-time', action='store_true', help='skip the one-event-at-a-time comparison')
    ap.add_argument('--batch-only', action='store_true', help='print only the batched workload line')
    ap.add_argument('--batch-launch', default=None,
                    help="fixed batch launch shape instead of the autotuner's: tile,ROWS,CHUNK,GRID or "
                         "cell,BLOCK,GRID,MAXREGS")
    ap.add_argument('--surrogate-train', type=int, default=20000,
                    help='training events of the learned-surrogate experiment reported under "surrogate" '
                         '(the 20000 / 1000 configuration by default; 0: skip)')
    ap.add_argument('--surrogate-test', type=int, default=1000)
    ap.add_argument('--surrogate-epochs', type=int, default=12)
    ap.add_argument('--surrogate-only', action='store_true', help='print only the surrogate experiment line')
    ap.add_argument('--fp64', action='store_true', help='the same workload in double precision')
    ap.add_argument('--no-fp64', action='store_true', help='skip the FP64 object of the default line')
    ap.add_argument('--arithmetic', default='fast', choices=['fast', 'exact'],
                    help='fused-stage arithmetic (fast: the default tolerance build; exact: the reference\'s bits)')
    ap.add_argument('--evolve', action='store_true',
                    help='also evolve the whole event to freeze-out with the hypersurface (reported under "evolve")')
    ap.add_argument('--grid', type=lambda s: tuple(int(x) for x in s.split(',')), default=(NX, NY, NZ),
                    help='nx,ny,nz (default: the 385,385,115 workload)')
    args = ap.parse_args()
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    if args.surrogate_only:
        import torch
        from clvisc_b200.surrogate import run_experiment
        torch.cuda.set_device(int(os.environ.get('LOCAL_RANK', 0)))
        out = run_experiment(args.surrogate_train, args.surrogate_test, args.surrogate_epochs,
                             log=lambda m: print(m, file=sys.stderr, flush=True))
        out['metric'] = 'surrogate events/h at rel. L2 error on e (128x128 (2+1)D events, tau0 + 6.4 fm)'
        print(json.dumps(out), flush=True)
        return
    if args.batch_only:
        import torch
        torch.cuda.set_device(int(os.environ.get('LOCAL_RANK', 0)))
        launch = None
        if args.batch_launch:
            f = args.batch_launch.split(',')
            launch = (f[0],) + tuple(int(x) for x in f[1:])
        print(json.dumps(run_batch(args.batch_events, one_at_a_time=not args.no_one_at_a_time, launch=launch)),
              flush=True)
        return
    if args.impl == 'reference':
        # rank 0 alone times the CPU path; the other ranks exit without work
        # and without joining a process group
        run_reference(args, rank, world)
        return
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get('LOCAL_RANK', 0)))
        tdist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))
        dist = tdist
    try:
        run_gpu(args, rank, world, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == '__main__':
    main()

// Batched event-by-event hydro: many independent (2+1)D or (3+1)D events on
// grids of different sizes advanced together, one persistent launch per
// Runge-Kutta stage for all of them.
//
// The fields of every event live in shared arenas: event e's w-plane field
// starts at element off * w-plane block of the arena, with its own plane stride
// ld_e. A persistent kernel walks the flattened cells of the events that are
// still running (a compacted list and a prefix of their cell counts, rebuilt on
// the device after each step) and applies to each cell the same fused stage as
// the single-event kernel (visc_stage_cell), so every event evolves bit for bit
// as it would alone. tau, the step counter, the stop test and the per-event
// history live in device memory, so a block of steps can be captured in one CUDA
// graph and replayed without host work between steps.
//
// Stop rule per event, as CLVisc.evolve (visc.py:473-560) applies it to one
// event: at every step count that is a multiple of ntskip the maximum energy
// density (folded into a per-event key during the preceding step's second
// stage, or measured on the initial state at step 0) is recorded with tau, and
// the event stops when it is below the freeze-out energy density.
#pragma once
#include "clv_stage.cuh"
#include "clv_stage_tiled2d.cuh"

namespace clv {

constexpr int BATCH_MAX_EVENTS = 1024;

struct BatchEvent {  // layout of clv_batch_event
  int nx, ny, nz, reserved;
  long long ld;        // plane stride of this event's fields
  long long off_ev;    // element offset of its 4-plane blocks (ev slots, udiff)
  long long off_pi;    // element offset of its npi-plane blocks (pi slots)
  long long off_src;   // element offset of its (4 + npi)-plane source block
  long long off_cell;  // byte offset of its goodcell block
};

struct BatchCtl {  // layout of clv_batch_ctl
  int loop;                // steps taken by the batch
  int n_active;            // events still running
  long long active_cells;  // cells of those events
  int done;                // no event left
  int hist_len;            // checks recorded
};

template <class real> struct BatchArgs {
  const BatchEvent* events;
  int n_events;
  real* ev[3];
  real* pi[3];
  real* src;
  real* udiff;
  uint8_t* goodcell;
  typename KeyT<real>::type* keys;  // per event
  BatchCtl* ctl;
  int* active;           // compacted running events
  long long* prefix;     // cell prefix over `active`, n_active + 1 entries
  int* loops;            // per event: step count at which it stopped, -1 while running
  double* history;       // [hist_cap][n_events][2]: (tau, max energy density) per check
  int hist_cap;
  double tau0, dt, efrz;  // the host's double values of TAU0, DT and the freeze-out energy density
  int ntskip, max_loops;
};

inline namespace CLV_ARITH {

// tau in the run precision after `n` steps: real(TAU0 + n*DT) as the host
// forms it (ideal.py:317-320; n = 0 gives real(TAU0))
template <class real> __device__ __forceinline__ real batch_tau(double tau0, double dt, int n) {
  return (real)(tau0 + (double)n * dt);
}

// the stage buffers of event e (its slots of every arena) at stage `step`
template <class real>
__device__ __forceinline__ ViscBuffers<real> batch_buffers(const BatchArgs<real>& a, const BatchEvent& E, int e, int step,
                                                           bool fold) {
  // slots chosen without indexing the parameter arrays at run time (which
  // would copy them to local memory)
  real* const ev_st = step == 1 ? a.ev[1] : a.ev[2];
  real* const ev_nw = step == 1 ? a.ev[2] : a.ev[1];
  real* const pi_st = step == 1 ? a.pi[1] : a.pi[2];
  real* const pi_nw = step == 1 ? a.pi[2] : a.pi[1];
  ViscBuffers<real> b;
  b.ev_st = ev_st + E.off_ev;
  b.pi_st = pi_st + E.off_pi;
  b.ev1 = a.ev[1] + E.off_ev;
  b.ev2e = a.ev[2] + E.off_ev;
  b.pi1 = a.pi[1] + E.off_pi;
  b.pin = a.pi[1] + E.off_pi;  // fused step: pi at the start of the step is d_pi[1]
  b.pi2in = pi_nw + E.off_pi;
  b.evnew = ev_nw + E.off_ev;
  b.pinew = pi_nw + E.off_pi;
  b.src = a.src + E.off_src;
  b.udiff = a.udiff + E.off_ev;
  b.goodcell = a.goodcell + E.off_cell;
  b.edmax_key = fold ? a.keys + e : nullptr;
  b.write_src = step == 1;
  b.write_udiff = step == 2;
  return b;
}

template <class real> __device__ __forceinline__ TauConst<real> batch_tau_const(const Params& p, const BatchArgs<real>& a,
                                                                               int loop, int step) {
  TauConst<real> tc;
  tc.tau = batch_tau<real>(a.tau0, a.dt, step == 1 ? loop : loop + 1);
  tc.rtau = (real)1 / tc.tau;
  tc.dzt = (real)p.DZ * tc.tau;
  tc.rdzt = (real)1 / tc.dzt;
  return tc;
}

// MINB > 1 caps the registers so that MINB blocks stay resident per SM
// (MINB = 512 / BS: at most 128 registers a thread, as the single-event
// per-cell kernel); MINB = 1 leaves the count to the compiler.
template <class real, bool BULK, int BS, int MINB>
__global__ void __launch_bounds__(BS, MINB) batch_stage_kernel(Params p, BatchArgs<real> a, int step) {
  __shared__ long long s_prefix[BATCH_MAX_EVENTS + 1];
  __shared__ int s_active[BATCH_MAX_EVENTS];
  const BatchCtl ctl = *a.ctl;
  if (ctl.done) return;
  const int n = ctl.n_active;
  for (int t = threadIdx.x; t <= n; t += BS) {
    s_prefix[t] = a.prefix[t];
    if (t < n) s_active[t] = a.active[t];
  }
  __syncthreads();
  const int loop = ctl.loop;
  const TauConst<real> tc = batch_tau_const<real>(p, a, loop, step);
  const bool fold = (step == 2) && ((loop + 1) % a.ntskip == 0);
  const long long total = s_prefix[n];
  for (long long g = (long long)blockIdx.x * BS + threadIdx.x; g < total; g += (long long)gridDim.x * BS) {
    int lo = 0, hi = n;  // largest slot with prefix <= g
    while (hi - lo > 1) {
      int mid = (lo + hi) >> 1;
      if (s_prefix[mid] <= g) lo = mid;
      else hi = mid;
    }
    const int e = s_active[lo];
    const BatchEvent E = a.events[e];
    const GridDims gd{E.nx, E.ny, E.nz, E.ld};
    const ViscBuffers<real> b = batch_buffers<real>(a, E, e, step, fold);
    visc_stage_cell<real, true, true, false, BULK>(p, gd, b, step, tc, g - s_prefix[lo]);
  }
}

// The same stage for batches of (2+1)D events (every event NZ = 1) with the
// tiled kernel of clv_stage_tiled2d.cuh: the work items are tiles of TB-4 rows
// by `chunk` x planes; a persistent block takes tiles g = blockIdx.x,
// blockIdx.x + gridDim.x, ... of the running events in order.
template <class real, bool BULK, int TB, int MINB>
__global__ void __launch_bounds__(TB, MINB) batch_tiled2d_kernel(Params p, BatchArgs<real> a, int step, int chunk) {
  __shared__ int s_tprefix[BATCH_MAX_EVENTS + 1];  // the only static shared memory: 4 KB
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Tile2Smem<real, BULK, TB>& sm = *reinterpret_cast<Tile2Smem<real, BULK, TB>*>(smem_raw);
  const BatchCtl ctl = *a.ctl;
  if (ctl.done) return;
  const int n = ctl.n_active;
  constexpr int TI = TB - 4;  // rows of a tile
  for (int q = threadIdx.x; q < n; q += TB) {
    const BatchEvent E = a.events[a.active[q]];
    s_tprefix[q + 1] = E.nz == 1 ? ((E.ny + TI - 1) / TI) * ((E.nx + chunk - 1) / chunk) : 0;  // its tiles
  }
  __syncthreads();
  if (threadIdx.x == 0) {  // prefix of the tile counts (n <= 1024)
    s_tprefix[0] = 0;
    for (int q = 0; q < n; q++) s_tprefix[q + 1] += s_tprefix[q];
  }
  __syncthreads();
  const int loop = ctl.loop;
  const TauConst<real> tc = batch_tau_const<real>(p, a, loop, step);
  const bool fold = (step == 2) && ((loop + 1) % a.ntskip == 0);
  const int total = s_tprefix[n];
  for (int g = blockIdx.x; g < total; g += gridDim.x) {  // block-uniform
    int lo = 0, hi = n;  // largest slot with prefix <= g
    while (hi - lo > 1) {
      int mid = (lo + hi) >> 1;
      if (s_tprefix[mid] <= g) lo = mid;
      else hi = mid;
    }
    const int e = a.active[lo];
    const BatchEvent E = a.events[e];
    const GridDims gd{E.nx, E.ny, E.nz, E.ld};
    const ViscBuffers<real> b = batch_buffers<real>(a, E, e, step, fold);
    const int local = g - s_tprefix[lo];
    const int nty = (E.ny + TI - 1) / TI;
    const int ty = local % nty, tx = local / nty;
    const int i0 = tx * chunk;
    tile2d<real, BULK, TB>(p, gd, b, step, tc, ty * TI, i0, min(i0 + chunk, E.nx), sm);
    __syncthreads();
  }
}

template <class real> __device__ __forceinline__ real decode_key(typename KeyT<real>::type k);
template <> __device__ __forceinline__ float decode_key<float>(unsigned int k) {
  if (k == 0) return -3.402823466e+38f;  // no value seen: -FLT_MAX, as clv_max_ed_read
  unsigned int b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  return __uint_as_float(b);
}
template <> __device__ __forceinline__ double decode_key<double>(unsigned long long k) {
  if (k == 0) return -3.402823466e+38;
  unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double((long long)b);
}

// After a step (first = 0) or before the first one (first = 1): advance the
// step count, apply the stop test at multiples of ntskip, record the history,
// and rebuild the list of running events. One block of 1024 threads.
template <class real> __global__ void __launch_bounds__(1024) batch_advance_kernel(BatchArgs<real> a, int first) {
  __shared__ long long s_scan[1024];
  __shared__ int s_flag[1024];
  BatchCtl* c = a.ctl;
  if (c->done) return;
  int loop = c->loop + (first ? 0 : 1);
  const bool stop_all = a.max_loops >= 0 && loop >= a.max_loops;
  const bool check = !stop_all && (loop % a.ntskip == 0);
  const int row = c->hist_len;
  const int tid = threadIdx.x;
  // each thread owns events tid, tid + 1024, ... (at most BATCH_MAX_EVENTS = 1024: one)
  long long cells = 0;
  int running = 0;
  const int e = tid;
  if (e < a.n_events && a.loops[e] < 0) {
    if (stop_all) {
      a.loops[e] = loop;
    } else if (check) {
      real edmax = decode_key<real>(a.keys[e]);
      a.keys[e] = 0;
      if (row < a.hist_cap) {
        a.history[((long long)row * a.n_events + e) * 2 + 0] = (double)batch_tau<real>(a.tau0, a.dt, loop);
        a.history[((long long)row * a.n_events + e) * 2 + 1] = (double)edmax;
      }
      if ((double)edmax < a.efrz) a.loops[e] = loop;
    }
    if (a.loops[e] < 0) {
      running = 1;
      const BatchEvent E = a.events[e];
      cells = (long long)E.nx * E.ny * E.nz;
    }
  }
  // block-wide exclusive scans of running flags and cell counts (Hillis-Steele)
  s_flag[tid] = running;
  s_scan[tid] = cells;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    int f = tid >= o ? s_flag[tid - o] : 0;
    long long v = tid >= o ? s_scan[tid - o] : 0;
    __syncthreads();
    s_flag[tid] += f;
    s_scan[tid] += v;
    __syncthreads();
  }
  if (running) {
    const int slot = s_flag[tid] - 1;
    a.active[slot] = e;
    a.prefix[slot] = s_scan[tid] - cells;
  }
  if (tid == 1023) {
    const int n = s_flag[1023];
    a.prefix[n] = s_scan[1023];
    c->loop = loop;
    c->n_active = n;
    c->active_cells = s_scan[1023];
    if (check) c->hist_len = row + 1;
    c->done = (n == 0);
  }
}

}  // namespace CLV_ARITH
}  // namespace clv

/* clvisc_b200 -- C ABI of the B200 (sm_100a) backend for the CLVisc hydro step.
 *
 * This ABI replaces the OpenCL programs that CLVisc builds and launches from
 * Python (pyvisc/backend_opencl.py and pyvisc/kernel/*.cl, driven by
 * pyvisc/ideal.py and pyvisc/visc.py). Every entry point below names the
 * reference kernel(s) it stands in for.
 *
 * Conventions
 *   - Plain pointers and sizes only. Field pointers are DEVICE pointers to
 *     structure-of-arrays planes: a field with w components occupies w planes
 *     of `ld` elements each (plane c starts at ptr + c*ld), and cell
 *     I = i*NY*NZ + j*NZ + k, the reference's order (kernel_visc.cl:145).
 *     ev has 4 planes (ed, vx, vy, veta); pi has 10 planes in the reference's
 *     packed order 00 01 02 03 11 12 13 22 23 33 (helper.h:31), and an
 *     eleventh, the bulk pressure Pi, when CLV_FLAG_BULK is set.
 *   - The element type is float when clv_params.precision == 4 and double
 *     when it is 8 (the reference's use_float32 flag, config.py:200).
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy stream).
 *   - Every function returns 0 (CLV_OK) or a negative CLV_ERR_* code; no
 *     exception crosses the ABI and nothing is printed. clv_last_error()
 *     gives a one-line message for the last failure of the calling thread.
 *   - Launches are asynchronous on `stream` unless stated otherwise.
 */
#ifndef CLVISC_B200_H
#define CLVISC_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CLV_OK 0
#define CLV_ERR_INVALID (-1)  /* bad argument (null pointer, size, precision) */
#define CLV_ERR_CUDA (-2)     /* CUDA runtime error (launch, copy)            */
#define CLV_ERR_CAPACITY (-3) /* output buffer too small                      */

/* flags: the reference's optional -D defines (ideal.py:164-165, visc.py:111-121) */
#define CLV_FLAG_RIEMANN_TEST 1
#define CLV_FLAG_GUBSER_VISC_TEST 2
#define CLV_FLAG_PIMN_OMEGA_COUPLING 4
#define CLV_FLAG_OMEGA_OMEGA_COUPLING 8
/* Bulk viscosity, an extension with no counterpart in the reference (its
 * kernel_visc.cl:31-33 keeps a zero placeholder for the bulk pressure): pi
 * fields carry an eleventh plane Pi and the stage sources a fifteenth.
 * zeta/s(T) = zetaos_max w^2 / (w^2 + (T - zetaos_t0)^2) with
 * w = zetaos_width (1 + zetaos_skew sign(T - zetaos_t0)); Pi relaxes by
 * tau_Pi D Pi + Pi = -zeta theta - 2/3 tau_Pi Pi theta with the 14-moment
 * tau_Pi = zeta / (14.55 (1/3 - cs2)^2 (e+P)), is held within |Pi| <= P and
 * at zero in cells colder than zetaos_tmin, and P + Pi replaces P in T^{mu nu}. */
#define CLV_FLAG_BULK 16
/* Tolerance arithmetic for the fused viscous stage (both parts in one
 * launch), an option with no counterpart in the reference: the kernels are
 * compiled with fused multiply-add contraction and approximate division and
 * square root, divide by run constants through their reciprocals, evaluate
 * the minmod limiters in sign-test form and
 * take the KT speed max(lambda, 1) as 1 (lambda <= 1 for |v| < 1). Results
 * differ from the reference's arithmetic by rounding: within 1e-5 of each
 * field's largest magnitude in FP32 after the tested step counts. Without the
 * flag every kernel reproduces the reference's arithmetic bit for bit. The
 * split stages (one part per launch) always use the exact arithmetic. */
#define CLV_FLAG_FAST 32

/* parts of a viscous stage (visc.py:287 IS_stepUpdate, visc.py:232 visc_stepUpdate) */
#define CLV_PART_IS 1
#define CLV_PART_KT 2

/* Run constants: the reference's compile-time defines (ideal.py:146-171,
 * eos.py:194-201, ideal.py:190-194). Floating constants are the float values
 * of the "%sf" literals the reference host emits, in FP64 mode too. */
typedef struct clv_params {
  int nx, ny, nz;
  long long ld; /* plane stride in elements, >= nx*ny*nz */
  int precision; /* 4 = float32, 8 = float64 */
  float dt, dx, dy, dz, tau0;
  float etaos_xmin, etaos_ymin, etaos_left_slop, etaos_right_slop, lam1;
  float efrz;
  int nxskip, nyskip, nzskip;
  float eos_ed_start, eos_ed_step;
  int eos_num_ed, eos_nrow, eos_ncol;
  const float *eos_table; /* device, 16-byte aligned, eos_nrow*eos_ncol texels of (cs2, p, T, s) */
  int flags;              /* CLV_FLAG_* */
  float zetaos_max, zetaos_t0, zetaos_width, zetaos_skew; /* bulk sector (CLV_FLAG_BULK) */
  float zetaos_tmin;      /* bulk sector: Pi = 0 in cells colder than this */
  /* Kernel choices of this run (see clv_set_option); 0 = the process-wide
   * setting. opt_stage_kernel = 1 + CLV_OPT_STAGE_KERNEL value, opt_chunk =
   * x planes per tiled CTA, opt_tiled_blocks = 1 or 2, opt_tile = 1 +
   * CLV_OPT_TILE value. */
  int opt_stage_kernel, opt_chunk, opt_tiled_blocks, opt_tile;
  /* Optional (nullable), read by the tolerance build (CLV_FLAG_FAST) only:
   * device, 8-byte aligned, eos_nrow*eos_ncol pairs (p[t], p[t+1]) of the
   * table's pressure column (the last pair repeats p[last]), so that a
   * pressure lookup is one 8-byte read. */
  const float *eos_p2;
} clv_params;

/* Buffers of one viscous Runge-Kutta stage. `step` is 1 or 2 as in
 * visc.py:536-543; d_ev[], d_pi[] are the reference's three-slot buffers. */
typedef struct clv_visc_buffers {
  const void *ev_st;     /* d_ev[step]: stencil input, 4 planes                */
  const void *pi_st;     /* d_pi[step]: stencil input, 10 planes (11: bulk)    */
  const void *ev1;       /* d_ev[1]                                            */
  const void *ev2_ed;    /* plane 0 of d_ev[2] (read by step 1's pi update)    */
  const void *pi1;       /* d_pi[1]: start point of the pi update              */
  const void *pi_n;      /* pi at the start of the time step (d_pi[0])         */
  const void *pi_new_in; /* d_pi[3-step]: read when CLV_PART_IS is not fused   */
  void *ev_new;          /* d_ev[3-step]                                       */
  void *pi_new;          /* d_pi[3-step]                                       */
  void *src;             /* 14 planes: d_Src (4) then d_IS_src (10); 15: bulk  */
  void *udiff;           /* 4 planes                                           */
  unsigned char *goodcell; /* 1 byte per cell (the reference's d_goodcell)     */
  void *edmax_key;       /* optional: running max of ev_new energy density     */
  int write_src;         /* keep the accumulated sources (needed by step 2)    */
  int write_udiff;       /* step 2 only: udiff = u(ev_new) - u(ev1)            */
} clv_visc_buffers;

/* Tuning options (process-wide defaults; a run's own opt_* fields in
 * clv_params take precedence): the viscous-stage kernel variant
 * (0 = automatic, the default: on grids with at least 24 cells along eta and
 * no bulk sector the tiled (3+1)D kernel, else one thread per cell; 1 = one
 * thread per cell without shared memory; 2 = tiled (3+1)D wherever it
 * applies; 3 = the tiled (2+1)D kernel for the fused stage without coupling
 * terms on (2+1)D grids (NZ = 1, NX and NY >= 4), else as 0), the number of x planes a tiled (3+1)D thread block
 * marches through, and the number of tiled blocks kept resident per SM in
 * FP32 (1 or 2; FP64 uses 1). Every variant computes the same values bit for
 * bit. */
#define CLV_OPT_STAGE_KERNEL 1
#define CLV_OPT_CHUNK 2
#define CLV_OPT_TILED_BLOCKS 3
/* (y, eta) tile of the fused tiled stage: 0 = 8 x 32 (default), 1 = 16 x 16,
 * 2 = 8 x 16 (128-thread CTAs, four an SM in FP32), 3 = 16 x 32 (one
 * 512-thread CTA an SM; FP32 tolerance arithmetic only, else as 0) */
#define CLV_OPT_TILE 4
/* (2+1)D tiles: threads of a block (64, the default, or 128; a tile is that
 * many rows minus 4) and x planes per tile (default 8) */
#define CLV_OPT_TILE2D_ROWS 5
#define CLV_OPT_CHUNK2D 6
int clv_set_option(int option, int value);

/* Library version; the low 8 bits bump on any ABI change. */
int clv_version(void);
/* One-line description of the last error on this thread ("" if none). */
const char *clv_last_error(void);
/* Required alignment (bytes) of every field pointer and of ld*elem_size. */
int clv_alignment(void);

/* Health of a state after a step (replaces reading d_goodcell and scanning
 * the fields on the host; the reference reports neither, kernel_IS.cl:697-708
 * only flags bad cells in d_goodcell). Into counts_dev (3 device int64, the
 * caller's memory) it writes, on `stream`: [0] the non-finite values in the 4
 * planes of ev and the npi planes of pi (pi nullable), [1] the cells whose
 * goodcell flag is 0 (goodcell nullable: 0), [2] the surface elements beyond
 * sf_capacity given the device count sf_total (nullable: 0). With counts_host
 * non-null it also copies the three counts there and synchronizes the
 * stream. */
int clv_status(const clv_params *p, const void *ev, const void *pi, int npi, const unsigned char *goodcell,
               const long long *sf_total, long long sf_capacity, long long *counts_dev, long long *counts_host,
               void *stream);
/* sizeof(clv_params) as compiled into the library, for bindings that mirror
 * the struct (a ctypes or cgo binding checks its own size against it). */
size_t clv_params_size(void);

/* One ideal Runge-Kutta stage: kt_src_christoffel + kt_src_alongx/y/z +
 * update_ev (kernel_ideal.cl:3-231, driven by ideal.py:211-255).
 * ev_st = d_ev[step], ev1 = d_ev[1], ev_new = d_ev[3-step], src = d_Src (4
 * planes; zeroed by step 1, accumulated by step 2). ev_new may equal ev1.
 * edmax_key (nullable) receives the max of ev_new's energy density. */
int clv_ideal_stage(const clv_params *p, int step, double tau, const void *ev_st, const void *ev1,
                    void *ev_new, void *src, int write_src, void *edmax_key, void *stream);

/* One viscous Runge-Kutta stage, any of CLV_PART_IS (visc_src_christoffel,
 * visc_src_alongx/y/z, update_pimn: kernel_IS.cl:41-709) and CLV_PART_KT
 * (kt_src_christoffel, kt_src_alongx/y/z, update_ev: kernel_visc.cl:11-393).
 * With both parts the new pi feeds update_ev from registers. */
int clv_visc_stage(const clv_params *p, int step, double tau, int parts, const clv_visc_buffers *b, void *stream);

/* visc_initialize (kernel_IS.cl:10-36): Navier-Stokes pi from ev, udiff = 0,
 * goodcell = 1. Components of pi1 other than 11, 22, 33 are left as they are.
 * With CLV_FLAG_BULK also Pi = -zeta / tau (Navier-Stokes, Bjorken flow). */
int clv_visc_initialize(const clv_params *p, void *pi1, unsigned char *goodcell, void *udiff, const void *ev,
                        double tau, void *stream);

/* get_udiff (kernel_IS.cl:714-724): udiff = u(ev1) - u(ev0). */
int clv_get_udiff(const clv_params *p, void *udiff, const void *ev0, const void *ev1, void *stream);

/* reduction_stage1 + host max (kernel_reduction.cl:7-39, ideal.py:257-262):
 * folds max(ed) over the first plane of ev into *key (device, an ordered
 * integer of precision-sized width; set it to 0 first with clv_max_ed_reset).
 * NaN values are ignored. */
int clv_max_ed_reset(const clv_params *p, void *key, void *stream);
int clv_max_ed(const clv_params *p, const void *ev, void *key, void *stream);
/* Synchronous: decode *key into a double (-FLT_MAX if no value was seen). */
int clv_max_ed_read(const clv_params *p, const void *key, double *out, void *stream);

/* get_hypersf / visc_hypersf (kernel_hypersf.cl:404-660): append the freeze-out
 * surface elements between (ev_old, tau_old) and (ev_new, tau_new) to the
 * output arrays, in coarse-cube (i, j, k) order, after the *total elements
 * already there (total: device long long, updated on the stream).
 *   sf   : capacity x 8 reals (dSigma_0..3, vx, vy, veta, etas)  [real8]
 *   txyz : capacity x 4 reals (tau cosh eta, x, y, tau sinh eta) [real4]
 *   pisf : capacity x 10 reals (visc != 0 only; may be NULL)
 * Elements beyond capacity are counted but not written; compare *total with
 * capacity after the stream completes.
 * scratch: device memory of clv_hypersf_scratch_bytes(p) bytes. */
size_t clv_hypersf_scratch_bytes(const clv_params *p);
int clv_hypersf_append(const clv_params *p, int visc, double tau_old, double tau_new, const void *ev_old,
                       const void *ev_new, const void *pi_old, const void *pi_new, void *sf, void *txyz, void *pisf,
                       long long capacity, long long *total, void *scratch, size_t scratch_bytes, void *stream);

/* clv_hypersf_append without the scratch argument, for callers that cannot
 * allocate device memory: an application whose memory pool owns the device
 * and lets no library allocate, or a time-critical loop where a cudaMalloc
 * (which may synchronise the device) is not acceptable. It has no counterpart
 * in the reference. Its scratch is a fixed array inside the library (about
 * 1 MB, held on every GPU that loads the library until the process exits),
 * which limits a call to 2^26 coarse cubes, ((NX-1)/nxskip+1) *
 * ((NY-1)/nyskip+1) * ((NZ-1)/nzskip+1); larger grids return
 * CLV_ERR_INVALID. It appends the same elements, in the same order, as
 * clv_hypersf_append. All calls share that array: calls whose launches overlap
 * on the GPU race, so serialise them. A call made outside stream capture looks
 * up the array's device address on the current device (so it stays right
 * after a device reset); a call during capture reuses the address of the last
 * call outside capture on that device, so make one call on each device before
 * any stream capture. Nothing is allocated or freed. */
int clv_hypersf_append_noalloc(const clv_params *p, int visc, double tau_old, double tau_new, const void *ev_old,
                               const void *ev_new, const void *pi_old, const void *pi_new, void *sf, void *txyz,
                               void *pisf, long long capacity, long long *total, void *stream);

/* ------------------------------------------------------------------------
 * Batched events: many independent events on grids of different sizes
 * advanced together. No counterpart in the reference, which runs one event
 * per process (its event-by-event scripts loop over CLVisc objects).
 *
 * Event e's fields live in arenas shared by all events: its w-plane field
 * starts at element off * (w planes of ld_e elements) of the arena -- ev
 * slots and udiff at off_ev (4 planes), pi slots at off_pi (10 planes, 11
 * with CLV_FLAG_BULK), the sources at off_src (14, or 15), goodcell at byte
 * off_cell. The clv_params of a batch carry the shared constants; its nx, ny,
 * nz, ld describe no event (set them to the largest event). Each event evolves
 * bit for bit as CLVisc.evolve would evolve it alone (visc.py:473-560):
 * both Runge-Kutta stages fused, the maximum energy density recorded with tau
 * at every multiple of ntskip steps, the event stopping when that maximum is
 * below efrz. Gubser, coupling and Riemann test flags are not batched. */
typedef struct clv_batch_event {
  int nx, ny, nz, reserved;
  long long ld, off_ev, off_pi, off_src, off_cell;
} clv_batch_event;

/* device control block of a batch */
typedef struct clv_batch_ctl {
  int loop;                /* steps taken                     */
  int n_active;            /* events still running            */
  long long active_cells;  /* their cells                     */
  int done;                /* 1 when no event is left         */
  int hist_len;            /* stop tests recorded in history  */
} clv_batch_ctl;

typedef struct clv_batch {
  const clv_batch_event *events; /* device, n_events entries (at most 1024)          */
  int n_events;
  void *ev[3], *pi[3];           /* arenas of d_ev[0..2], d_pi[0..2]                   */
  void *src, *udiff;             /* arenas of the stage sources and udiff              */
  unsigned char *goodcell;       /* arena of goodcell                                  */
  void *keys;                    /* n_events max-energy-density keys (precision bytes) */
  clv_batch_ctl *ctl;            /* device control block                               */
  int *active;                   /* n_events: running events, compacted                */
  long long *prefix;             /* n_events + 1: cell prefix over active              */
  int *loops;                    /* n_events: steps at which each stopped (-1: running) */
  double *history;               /* hist_cap x n_events x (tau, max ed)                */
  int hist_cap;
  double tau0, dt, efrz;         /* the host's double TAU0, DT, freeze-out energy density */
  int ntskip;                    /* stop-test cadence                                  */
  int max_loops;                 /* stop every event after this many steps (-1: never) */
} clv_batch;

/* One fused Runge-Kutta stage (step 1 or 2) of every running event: one
 * persistent launch of grid_blocks blocks of block_size (64, 128 or 256)
 * threads; grid_blocks <= 0 sizes the grid to fill the GPU once.
 * max_registers: 0 lets the compiler choose; 128 (FP32 only) caps the
 * registers a thread so that 512 threads stay resident per SM; 168 (FP32,
 * 64- or 128-thread blocks) so that 384 do. Reads tau and
 * the running list from the device, so it can be captured in a CUDA graph. */
int clv_batch_stage(const clv_params *p, int step, const clv_batch *b, int block_size, int grid_blocks,
                    int max_registers, void *stream);
/* After a step (first = 0) or once before the first step (first = 1, with
 * keys holding each event's initial maximum energy density): count the step,
 * apply the stop test at multiples of ntskip, record the history, rebuild the
 * running list. ctl must start as {0, 0, 0, 0, 0}, loops as -1, keys as 0
 * except for the first call. */
int clv_batch_advance(const clv_params *p, const clv_batch *b, int first, void *stream);
/* Resident blocks per SM of the batch stage kernel at block_size threads. */
int clv_batch_occupancy(const clv_params *p, int block_size, int max_registers, int *blocks_per_sm);
/* The same stage for batches of (2+1)D events with the tiled kernel: work
 * items are tiles of (rows - 4) y rows by `chunk` x planes (rows = 64 or 128
 * threads a block), taken in order by grid_blocks persistent blocks
 * (grid_blocks <= 0: fill the GPU once). Every event must have nz = 1: the
 * kernel gives events with nz != 1 no tiles. Same bits as clv_batch_stage. */
int clv_batch_stage_tiled(const clv_params *p, int step, const clv_batch *b, int rows, int chunk, int grid_blocks,
                          void *stream);
/* Resident blocks per SM of the tiled batch stage kernel. */
int clv_batch_occupancy_tiled(const clv_params *p, int rows, int *blocks_per_sm);

/* ------------------------------------------------------------------------
 * Initial conditions on the device. */

/* The optical Glauber model's constants: the float values of the
 * -D KEY=%ff literals glauber.py:79-90 emits from the configuration. */
typedef struct clv_glauber {
  float num_of_nucleons, sqrts, ro0, r, eta, si0, impact_parameter, edmax, hwn, eta_flat, eta_gw;
} clv_glauber;

/* glauber_ini (kernel_glauber.cl:86-102, called by CLVisc.optical_glauber_ini,
 * visc.py:151-172): ev (4 planes) = (Edmax-scaled two-component energy density
 * of Woods-Saxon thickness functions times the eta plateau profile, 0, 0, 0). */
int clv_glauber_ini(const clv_params *p, const clv_glauber *g, void *ev, void *stream);
/* num_of_binary_collisions (kernel_glauber.cl:104-121, glauber.py:94-103):
 * out[i*ny + j] = Si0 Ta Tb at (xlow + i dx, ylow + j dy); out has p's precision. */
int clv_glauber_nbinary(const clv_params *p, const clv_glauber *g, void *out, double xlow, double ylow, double dx,
                        double dy, int nx, int ny, void *stream);

/* Seeded Monte Carlo Glauber (hotspot) profile, no counterpart in the
 * reference: parts holds n_parts (x, y, weight) triples in double (device),
 * sampled on the host. ev (4 planes) = (e, 0, 0, 0) with
 * e(i, j, k) = sum_p w_p exp(-((x_i - x_p)^2 + (y_j - y_p)^2) / (2 width^2)) h(eta_k)
 * scaled to a maximum of edmax, x_i = (i - nx/2) dx, eta_k = (k - nz/2) dz,
 * h = 1 for |eta| <= plateau, exp(-(|eta| - plateau)^2 / (2 sigma_eta^2))
 * beyond; evaluated in double in participant order (the host construction's
 * arithmetic). scratch: clv_hotspot_scratch_bytes(p, n_parts) bytes, 256-byte
 * aligned. */
size_t clv_hotspot_scratch_bytes(const clv_params *p, int n_parts);
int clv_hotspot_ini(const clv_params *p, void *ev, const double *parts, int n_parts, double dx, double dy, double dz,
                    double width, double plateau, double sigma_eta, double edmax, void *scratch,
                    size_t scratch_bytes, void *stream);

/* ------------------------------------------------------------------------
 * Bulk-evolution diagnostics (pyvisc/bulkinfo.py, bulkinfo_h5.py,
 * kernel_bulkinfo.cl), computed where the state lives. */

/* Elements of the clv_bulk_slices output: ev lines through the grid centre
 * along x, y, eta (4 NX, 4 NY, 4 NZ), the planes k = NZ/2, j = NY/2, i = NX/2
 * (4 NX NY, 4 NX NZ, 4 NY NZ), then pi^xx, pi^yy, pi^tx in the transverse
 * plane (NX NY each), in that order, (w)-interleaved as the reference's real4
 * buffers. */
long long clv_bulk_slices_size(const clv_params *p);
/* get_ed and get_pimn (bulkinfo.py:62-117); pi may be NULL (ideal runs), then
 * the pi part is not written. The pi index is the reference's
 * i*NY*(NZ/2) + j*(NZ/2) + NZ/2. out has the precision of p. */
int clv_bulk_slices(const clv_params *p, const void *ev, const void *pi, void *out, void *stream);
/* Sums behind the reference's host-side diagnostics (bulkinfo.py:184-271),
 * in double, reduced per slice in a fixed order: out[3k + 0..2] =
 * sum over the eta slice k of T^xx, T^yy, T^tx (with veta); out[3 NZ + 0..7]
 * in the plane k = NZ/2 with veta = 0: T^xx, T^yy, T^tx, u0 e v_r, u0 e,
 * u0 s, pi^xx + pi^yy, pi^xx - pi^yy (the last two 0 when pi is NULL); with
 * the reference's floors e >= 1e-10 and v^2 > 1 -> 0.999999. */
int clv_bulk_sums(const clv_params *p, const void *ev, const void *pi, double *out, void *stream);
/* total_energy_and_entropy (kernel_bulkinfo.cl:18-45) summed over all cells
 * and times `volume` (tau DX DY DZ, bulkinfo_h5.py:264-277): out[0] = lab-frame
 * energy, out[1] = entropy. scratch: clv_bulk_lab_scratch_bytes() bytes. */
size_t clv_bulk_lab_scratch_bytes(void);
int clv_bulk_lab_totals(const clv_params *p, const void *ev, double tau, double volume, double *out, void *scratch,
                        size_t scratch_bytes, void *stream);

/* ------------------------------------------------------------------------
 * Cooper-Frye smooth spectra of one hadron species on the freeze-out surface:
 * get_sub_dNdYPtdPtdPhi + get_dNdYPtdPtdPhi (CLSmoothSpec/src/kernel_spec.cl:4-141)
 * for an ideal surface, kernel_spec_csc.cl:4-101 with the viscous delta f when
 * pisf is given. All pointers are device pointers in the given precision:
 * sf = n x 8 (dSigma_0..3, vx, vy, veta, eta_s; the hypersurface buffer of
 * clv_hypersf_append), pisf = n x 10 or NULL, y/pt/cphi/sphi the grids;
 * out = ny x npt x nphi spectra, (y, pt, phi) row-major, in GeV fm^3 units as
 * the reference. Sums are in double in a fixed order. */
typedef struct clv_spectra_args {
  int precision;                         /* 4 or 8 */
  const void *sf, *pisf;                 /* surface elements and their pi^{mu nu} */
  long long n;                           /* elements */
  double mass, gspin, fermi_boson, mu;   /* the hadron: +1 baryon (Fermi), -1 (Bose); chemical potential */
  double tfrz;                           /* freeze-out temperature [GeV] */
  double tcoeff;                         /* 1 / (2 T^2 (e + P)) on the surface (viscous only) */
  const void *y, *pt, *cphi, *sphi;      /* rapidities, transverse momenta, cos/sin of the azimuths */
  int ny, npt, nphi;                     /* npt * nphi <= 1024 */
} clv_spectra_args;
size_t clv_spectra_scratch_bytes(long long n, int ny, int npt, int nphi);
int clv_spectra(const clv_spectra_args *args, void *out, void *scratch, size_t scratch_bytes, void *stream);

/* ------------------------------------------------------------------------
 * Learned surrogate (no counterpart in the reference): kernels of a U-Net on
 * (N, H, W, C) BF16 activations, FP32 accumulation, tensor cores for the 3x3
 * convolutions. Activations may be channel slices of a wider buffer: element
 * (p, c) of a slice is ptr[p * stride + offset + c]. */

/* 3x3 convolution with zero padding as an implicit GEMM (mma.sync BF16,
 * FP32 accumulate): out = act(sum + bias), optionally times gelu'(gate), with
 * the pre-activation stored in pre ([P][Cout]) when given; act is GELU when
 * gelu != 0. w: [9][Cin][Cout] BF16 (tap = 3 (dy + 1) + (dx + 1)). The input
 * gradient of a layer is this call on the output gradient with the weights
 * clv_unet_pack writes to wt. Cin, Cout multiples of 32. */
typedef struct clv_unet_conv {
  const void *in;
  int in_cs, in_co;
  const void *w;
  const float *bias;
  void *out;
  int out_cs, out_co;
  void *pre;
  const void *gate;
  int gate_cs, gate_co;
  int N, H, W, Cin, Cout;
  int gelu;
} clv_unet_conv;
int clv_unet_conv3x3(const clv_unet_conv *args, void *stream);
/* Tensor-core paths (process-wide). 1 (the default): clv_unet_conv3x3 on
 * tcgen05.mma with the accumulator in tensor memory (operands by TMA in the
 * 64-byte swizzled layout when the image tiles into 128-pixel blocks, else by
 * cp.async) and clv_unet_wgrad3x3 on tcgen05 with TMA operands where the
 * pixels tile into 64-pixel blocks (else mma.sync); 3 = the same convolution
 * with the weight gradient on mma.sync; 2 = as 3 with no-swizzle TMA
 * operands; 0 = mma.sync for both. */
int clv_unet_set_conv_path(int path);
/* Bounded waits of the tcgen05 convolutions that ran out since the last
 * reset (0 in a healthy run; a tile whose wait ran out writes no output).
 * Reads device memory: synchronises with the device. */
int clv_unet_timeouts(int *count, int reset);
/* dw ([9][Cin][Cout] FP32) (+)= sum over pixels of x[p + tap][ci] g[p][co]
 * (g: gradient wrt the pre-activation, [P][Cout] BF16). */
size_t clv_unet_wgrad_scratch_bytes(int N, int H, int W, int Cin, int Cout);
int clv_unet_wgrad3x3(const void *x, int x_cs, int x_co, const void *g, int N, int H, int W, int Cin, int Cout,
                      float *dw, int accumulate, void *scratch, size_t scratch_bytes, void *stream);
/* scratch of the row-reduction entry points below for `width` sums */
size_t clv_unet_rows_scratch_bytes(int width);
int clv_unet_bias_grad(const void *g, int g_cs, long long P, int C, float *db, void *scratch, size_t scratch_bytes,
                       void *stream);
/* first layer: FP32 single-channel image -> C channels (w [9][C], GELU) and its weight gradient */
int clv_unet_first_fwd(const float *x, const float *w, const float *bias, int N, int H, int W, int C, void *pre,
                       void *out, int out_cs, int out_co, void *stream);
int clv_unet_first_wgrad(const float *x, const void *g, int N, int H, int W, int C, float *dw, void *scratch,
                         size_t scratch_bytes, void *stream);
/* head: 1x1 convolution C -> K (w [C][K], FP32 output); backward gives the
 * gradient wrt the input's pre-activation z (times gelu'(z)) and
 * dwb = [dW (C x K), db (K)] */
int clv_unet_head_fwd(const void *y, int y_cs, int y_co, const float *w, const float *b, long long P, int C, int K,
                      float *out, void *stream);
int clv_unet_head_bwd(const void *y, int y_cs, int y_co, const void *z, const float *g, const float *w, long long P,
                      int C, int K, void *gz, float *dwb, void *scratch, size_t scratch_bytes, void *stream);
/* 2x2 average pooling, nearest 2x upsampling, and their gradients through
 * the GELU that produced the pooled / upsampled activation */
int clv_unet_pool(const void *x, int x_cs, int x_co, int N, int H, int W, int C, void *out, void *stream);
int clv_unet_up(const void *x, int N, int H, int W, int C, void *out, int out_cs, int out_co, void *stream);
int clv_unet_skip_grad(const void *gcat, int gcat_cs, int gcat_co, const void *gpool, const void *z, int N, int H,
                       int W, int C, void *gz, void *stream);
int clv_unet_up_grad(const void *gcat, int gcat_cs, int gcat_co, const void *z, int N, int H, int W, int C, void *gz,
                     void *stream);
/* weighted squared error: grad = 2 w_k (out - target) scale, part[b] = block sums of w_k (out - target)^2 scale */
int clv_unet_mse(const float *out, const float *target, const float *wch, long long P, int K, float scale,
                 float *grad, float *part, int nparts, void *stream);
/* Adam step on FP32 master weights with the bias-corrected step lr_t */
int clv_unet_adam(float *w, const float *g, float *m, float *v, long long n, float lr_t, float b1, float b2, float eps,
                  void *stream);
/* BF16 weights of a 3x3 layer for the forward (w) and input-gradient (wt) convolutions */
int clv_unet_pack(const float *wf, int Cin, int Cout, void *w, void *wt, void *stream);

/* Host-boundary layout transposes: (n, w) row-major <-> w planes of ld. */
int clv_aos_to_soa(const clv_params *p, const void *aos, void *soa, long long n, int w, void *stream);
int clv_soa_to_aos(const clv_params *p, const void *soa, void *aos, long long n, int w, void *stream);

/* ------------------------------------------------------------------------
 * Output tables. The text files of the reference (hypersf.dat, sf_txyz.dat,
 * pimnsf.dat, written by numpy.savetxt(fmt='%.6e', header=...),
 * ideal.py:304-312, visc.py:413-419), written from a host array of rows x
 * cols reals (precision 4 or 8) with the same bytes: '# ' + header + '\n'
 * (no header line if header is null), then each row's values as %.6e
 * separated by one space and ended by '\n'; NaN as "nan". Host code only:
 * the rows are formatted by parallel host threads. */
int clv_write_table(const char *path, const char *header, const void *data, int precision, long long rows, int cols);

#ifdef __cplusplus
}
#endif
#endif /* CLVISC_B200_H */

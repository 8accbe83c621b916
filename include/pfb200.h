/*
 * pfb200.h - C ABI of the B200 FDTD stepping engine (libpfb200.so).
 *
 * This is the boundary a photonfdtd backend binds to (ctypes in
 * photonfdtd_b200/_native.py). It replaces the reference's PyO3 stepper
 * surface: rust/src/lib.rs:68-133 (step_range_f32/f64) and
 * rust/src/cuda.rs:512-564 (CudaStepper new_f32/new_f64, run_steps,
 * read_field), driven by src/photonfdtd/rustbackend.py:237-304 (_CudaEngine).
 *
 * Conventions
 *  - Every field array is C-order (nx, ny, nz), z fastest, in the engine's
 *    real type (real_bytes 4 = float, 8 = double). Component codes are
 *    0..5 = Ex, Ey, Ez, Hx, Hy, Hz (rust/src/lib.rs:41-47,
 *    src/photonfdtd/rustbackend.py:40).
 *  - Host arrays passed to pf_set_* are borrowed for the duration of the call
 *    only; the engine copies what it needs. The engine owns all device memory.
 *  - Every call returns PF_OK (0) or a negative PF_ERR_* code; the message is
 *    in pf_last_error(). This mirrors the reference mapping CUDA failures to
 *    RuntimeError("CUDA error: ...") (rust/src/cuda.rs:267-269).
 *  - One engine = one CUDA stream on the device current at pf_create. Calls on
 *    one engine must not overlap; different engines are independent.
 *    pf_advance returns after the stream has synchronised, like run_steps
 *    (rust/src/cuda.rs:298-341).
 */
#ifndef PFB200_H
#define PFB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PF_OK 0
#define PF_ERR_INVALID (-1)     /* bad argument or call order           */
#define PF_ERR_CUDA (-2)        /* a CUDA runtime call failed           */
#define PF_ERR_OOM (-3)         /* device allocation failed             */
#define PF_ERR_NONFINITE (-4)   /* non-finite field found by pf_check   */
#define PF_ERR_TIMEOUT (-5)     /* a bounded device wait ran out        */
#define PF_ERR_UNSUPPORTED (-6) /* feature combination not implemented  */
#define PF_ERR_STATE (-7)       /* engine not finalised / finalised     */

/* E-update coefficient encodings (pf_set_ce). */
#define PF_CE_CELL1 0 /* one per-cell array dt/(eps*eps0) for Ex, Ey, Ez  */
#define PF_CE_CELL3 1 /* three per-cell arrays (diagonal subpixel tensor)  */
#define PF_CE_TABLE 2 /* per-cell uint32 word indexing a coefficient table */

/* Stepping kernels (pf_set_kernel). */
#define PF_KERNEL_AUTO 0  /* the faster path for the grid (split on B200) */
#define PF_KERNEL_SPLIT 1 /* separate H and E passes, one thread per cell  */
#define PF_KERNEL_FUSED 2 /* require the fused H+E pass (3D only)          */

typedef struct pf_engine pf_engine;

/* Library version string, e.g. "pfb200 0.1.0 sm_100a". */
const char *pf_version(void);

/* Last error message of an engine (or of the last failed pf_create when
 * eng is NULL). Never NULL. */
const char *pf_last_error(const pf_engine *eng);

/* New engine on the current CUDA device.
 * dx, dy, dz: derivative spacing per axis (1.0 on a collapsed axis, as
 * src/photonfdtd/simulation.py:912). ch: H-update coefficient dt/mu0 already
 * rounded to the real type (simulation.py:954). n_steps: length of the run,
 * bounds the source-waveform and DFT-phase tables.
 * Replaces CudaStepper::new_f32/new_f64 (rust/src/cuda.rs:512-540). */
int pf_create(int nx, int ny, int nz, int real_bytes, double dx, double dy,
              double dz, double ch, int64_t n_steps, pf_engine **out);

/* E-update coefficients (rust/src/cuda.rs:140-247 takes one scalar field;
 * simulation.py:956-969 adds the three-component subpixel form).
 *  PF_CE_CELL1: ce0 = nx*ny*nz reals, ce1 = ce2 = NULL.
 *  PF_CE_CELL3: ce0/ce1/ce2 = per-component arrays for Ex/Ey/Ez.
 *  PF_CE_TABLE: word = nx*ny*nz uint32; word w < 2^31 selects table[w] (the
 *    word must be < n_table); w >= 2^31 marks a dispersive cell whose
 *    coefficient comes from its medium (pf_set_ade). table = n_table reals
 *    given as doubles (each exactly representable in the real type). The
 *    word is checked and copied to device memory during the call (one pass
 *    over it, no host copy); its dispersive words are checked against the
 *    media's cell counts at pf_finalize. */
int pf_set_ce(pf_engine *eng, int mode, const void *ce0, const void *ce1,
              const void *ce2, const uint32_t *word, int n_table,
              const double *table);

/* CPML along one axis (0, 1, 2): b/c on the E and H staggers, n reals each,
 * in the real type (src/photonfdtd/boundaries.py:31-97 builds them in f64;
 * simulation.py:1226-1227 casts them). psi is stored only where c != 0,
 * compacted along the axis as rustbackend._pml_map does (rustbackend.py:126-132).
 * NULL arrays mean no PML on that axis. */
int pf_set_cpml(pf_engine *eng, int axis, const void *b_e, const void *c_e,
                const void *b_h, const void *c_h);

/* Dispersive (ADE) media (simulation.py:572-669). n_media <= 16.
 *  A dispersive cell's word is 0x80000000 | (m << 27) | loc: medium m, and
 *  loc = its rank among medium m's cells in C order (loc < count[m] <= 2^27).
 *  cell_word: PF_CE_TABLE mode: NULL (the ce word carries it); PF_CE_CELL1
 *    mode: nx*ny*nz uint32, 0 for a plain cell.
 *  npole[m] <= 8; coef holds, per medium, per pole, (a, b, c) as doubles;
 *  inv_eps[m] = 1/(eps0*eps_inf); ce_m[m] = the medium's coefficient in table
 *  mode (ignored otherwise). */
int pf_set_ade(pf_engine *eng, int n_media, const int64_t *count,
               const int32_t *npole, const double *coef, const double *inv_eps,
               const double *ce_m, const uint32_t *cell_word);

/* Host-side helper for the ADE cell words, no engine needed: `word` holds,
 * per cell in C order, either a plain entry (bit 31 clear: a table index, or
 * anything when clear_plain != 0) or a dispersive entry bit 31 | m << 27
 * with its low 27 bits zero (m < n_media). Each dispersive entry receives
 * its rank among medium m's cells in C order (the record index
 * pf_set_ade's words carry), counts[m] the number of medium m's cells;
 * clear_plain != 0 zeroes every plain entry (the cell_word of the per-cell
 * coefficient modes). One pass, in place. This is the compact dispersive
 * cell numbering of src/photonfdtd/simulation.py:592-636. Errors go to
 * pf_last_error(NULL). */
int pf_rank_dispersive_words(uint32_t *word, int64_t n, int n_media, int64_t *counts,
                             int clear_plain);

/* Soft point sources (simulation.py:1367-1390; rustbackend.py:151-166).
 * n_src entries in the reference's source order: comp (0..5), flat cell
 * index i*ny*nz + j*nz + k, waveform row, amplitude. wave = n_wave rows of
 * n_steps doubles: row w, column s is the waveform at that source family's
 * Yee time of step s ((s+1/2)dt for H, (s+1)dt for E). The value added at
 * step s is amp * wave[w][s], computed in double and added in double before
 * rounding to the field type, as the reference does. */
int pf_set_sources(pf_engine *eng, int n_src, const int32_t *comp,
                   const int64_t *cell, const int32_t *wave_row,
                   const double *amp, int n_wave, const double *wave);

/* Running DFT monitor (simulation.py:1116-1133; rustbackend.py:384-397).
 * Region: start/stop/stride per axis (a plane is start = i, stop = i+1).
 * comp_mask: bit c set = record component c. Sampled at steps
 * s = 0, interval, 2*interval, ... < n_steps. phase_e / phase_h: one row per
 * sample, n_freq complex values as (re, im) doubles, = exp(i*omega*t) at the E
 * and H time of that sample (computed by the host exactly as the reference
 * does). dt: the Riemann-sum weight. Output id in *mon. */
int pf_add_dft(pf_engine *eng, const int32_t start[3], const int32_t stop[3],
               const int32_t stride[3], int comp_mask, int n_freq,
               int interval, const double *phase_e, const double *phase_h,
               double dt, int *mon);

/* Poynting flux through the full plane normal to axis at index idx
 * (simulation.py:1440-1459, accumulated every step as :1403-1406):
 * flux += real(sum(S) * dA) * dt, S = E_t1*H_t2 - E_t2*H_t1 at the same cell.
 * The plane sum is taken in double; the product with dA is rounded to the
 * real type as the reference's float32 run does. */
int pf_add_flux(pf_engine *eng, int axis, int idx, double dA, double dt,
                int *mon);

/* Kernel choice (PF_KERNEL_*); default PF_KERNEL_AUTO. */
int pf_set_kernel(pf_engine *eng, int kernel);

/* Allocate the device state, upload the tables, zero the fields. */
int pf_finalize(pf_engine *eng);

/* Advance global steps [step0, step0 + n_sub) (rust/src/cuda.rs:298-341,
 * rustbackend.py:222-231 / 297-299). step0 must equal the engine's step
 * counter (steps are not skipped or repeated). */
int pf_advance(pf_engine *eng, int64_t step0, int64_t n_sub);

/* Current value of one field component into host memory, nx*ny*nz reals
 * (rust/src/cuda.rs:552-564, read_field). */
int pf_read_field(pf_engine *eng, int comp, void *host_dst);

/* A strided sub-block of one current field component into host memory:
 * cells start[a], start[a] + stride[a], ... < stop[a] on each axis, C order
 * (the FieldMonitor snapshot of simulation.py:1062-1067: every downsample-th
 * cell, or one plane_z plane). The gather runs on the device, so only the
 * snapshot crosses to the host (the reference copies whole fields). The
 * engine keeps a device staging buffer of the largest region read. */
int pf_read_region(pf_engine *eng, int comp, const int32_t start[3],
                   const int32_t stop[3], const int32_t stride[3], void *host_dst);

/* DFT accumulator of monitor mon, component comp: n_freq x region cells
 * complex128 as interleaved (re, im) doubles (simulation.py:1124-1133). */
int pf_read_dft(pf_engine *eng, int mon, int comp, double *host_dst);

/* Time-integrated flux of flux monitor mon (simulation.py:1403-1406). */
int pf_read_flux(pf_engine *eng, int mon, double *host_dst);

/* Overwrite one field component of the current time level from host memory
 * (nx*ny*nz reals): the inverse of pf_read_field. The reference's engines
 * expose no such call; with pf_read_field it lets a caller start from a
 * state of its own (the reference's out-of-core stepper reloads fields the
 * same way, src/photonfdtd/outofcore.py:12-22). */
int pf_write_field(pf_engine *eng, int comp, const void *host_src);

/* The whole stepping state as one blob, for checkpoints: the six current
 * field components, the E and current H CPML psi arrays, and the
 * polarisation levels P^n then P^(n-1) of dispersive cells, all in the real
 * type. Monitor accumulators are not part of it. pf_state_bytes gives its
 * size; pf_get_state copies it out (dst_on_device != 0: dst is a device
 * pointer); pf_set_state copies it in and sets the step counter to `step`
 * (the state is taken to be the one reached after `step` steps; pending
 * monitor samples are folded first). This is the checkpoint pair of a
 * time-reversed pass: the reference's gradient path keeps the same quantities
 * between remat segments (src/photonfdtd/jaxbackend.py:511-570). */
int pf_state_bytes(const pf_engine *eng, int64_t *bytes);
int pf_get_state(pf_engine *eng, void *dst, int64_t bytes, int dst_on_device);
int pf_set_state(pf_engine *eng, int64_t step, const void *src, int64_t bytes,
                 int src_on_device);

/* Adjoint of the stepping: the gradient of a loss J of the monitor outputs
 * with respect to the per-cell E coefficient K = dt / (eps0 eps_r), i.e. the
 * time-domain adjoint behind value_and_grad_eps
 * (src/photonfdtd/jaxbackend.py:666-722, which differentiates the same step
 * with jax.grad; like it, no dispersive media: PF_ERR_UNSUPPORTED;
 * per-component coefficients, PF_CE_CELL3, are differentiated component by
 * component). Protocol, after a forward run that saved pf_get_state
 * checkpoints at the segment starts:
 *   pf_adj_init(ring_steps)     adjoint state + a replay ring of ring_steps
 *                               steps (the longest segment); zeroes the
 *                               adjoint and the gradient
 *   pf_adj_set_dft_cotangent(mon, cot)
 *                               dJ/d(DFT accumulator) of monitor mon as
 *                               (components in mask order, n_freq, region
 *                               cells) complex128 interleaved, G = dJ/dRe +
 *                               i dJ/dIm
 *   pf_adj_add_field_source(step, comp, region, vals)
 *                               dJ/d(field snapshot taken after step `step`,
 *                               the FieldMonitor frame) over a strided region
 *   pf_adj_set_flux_cotangent(mon, cot)
 *                               dJ/d(flux integral) of flux monitor mon
 *   pf_adj_segment(step0, n, state)
 *                               for segments from the last to the first
 *                               (step0 + n must be where the reverse pass
 *                               stands: n_steps, then the previous step0):
 *                               restores the checkpoint of step0, replays n
 *                               steps recording H and psi_E (monitors not
 *                               sampled), then runs their n reverse steps
 *   pf_adj_read_grad(dst)       dJ/dK per cell, summed over Ex, Ey, Ez
 *                               (ncell doubles); dJ/deps_r = -K/eps_r dJ/dK.
 *                               With one coefficient per cell (PF_CE_TABLE,
 *                               PF_CE_CELL1) the reverse pass accumulates
 *                               only this sum; with PF_CE_CELL3 it keeps
 *                               the three components
 *                               (pf_adj_read_grad_components).
 * The engine's current state afterwards is the end of the last replay. */
int pf_adj_init(pf_engine *eng, int64_t ring_steps);
int pf_adj_set_dft_cotangent(pf_engine *eng, int mon, const double *cot);
/* dJ/d(flux integral) of flux monitor mon: its plane's E and H enter the
 * reverse pass as sources (the replay records the plane's tangential E per
 * step for it). */
int pf_adj_set_flux_cotangent(pf_engine *eng, int mon, double cot);
int pf_adj_add_field_source(pf_engine *eng, int64_t step, int comp, const int32_t start[3],
                            const int32_t stop[3], const int32_t stride[3],
                            const double *vals);
int pf_adj_segment(pf_engine *eng, int64_t step0, int64_t n, const void *state,
                   int64_t bytes, int state_on_device);
int pf_adj_read_grad(pf_engine *eng, double *dst);
/* dJ/dK_c per component and cell (3 * ncell doubles: Ex cells, then Ey,
 * then Ez): the gradient for per-component coefficients (PF_CE_CELL3, e.g.
 * a density mapped to an anisotropic permittivity; jaxbackend.py:725-775
 * value_and_grad_params differentiates the same quantities). */
int pf_adj_read_grad_components(pf_engine *eng, double *dst);

/* Steps advanced so far. */
int pf_step(const pf_engine *eng, int64_t *step);

/* Scan all six fields for non-finite values: PF_OK or PF_ERR_NONFINITE. */
int pf_check_finite(pf_engine *eng);

/* Failure detection while stepping: with k > 0, pf_advance scans the fields
 * after every step whose count is a multiple of k and stops there with
 * PF_ERR_NONFINITE (the engine stays at that step) once a value is inf or
 * nan, e.g. a run past its Courant limit. 0 (the default) turns it off. The
 * reference has no such check. */
int pf_set_check_every(pf_engine *eng, int64_t k);

/* Test hook of the TMA-staged fused step (PF_KERNEL_FUSED where the grid
 * allows TMA): with on != 0, block (0, 0, 0) of every step waits once on a
 * barrier that nothing arrives on, with a short limit, so the wait runs out
 * and the block takes its timeout path (it lets its issued copies land, sets
 * the error flag and leaves); pf_advance then returns PF_ERR_TIMEOUT and the
 * fields are invalid. No counterpart in the reference. */
int pf_set_wait_test(pf_engine *eng, int on);

/* The CUDA stream (a cudaStream_t) the engine launches on, so a caller can
 * time its work with events on that stream. */
int pf_stream(const pf_engine *eng, void **stream);

/* Launch accounting. Kinds: 0 = step passes (H/E or fused), 1 = source
 * injection, 2 = monitor sampling, 3 = monitor flush. launches[k] counts
 * every launch; with profiling on (pf_set_profiling), ms[k] sums the device
 * time of those launches from events recorded around each one. reset != 0
 * zeroes both after reading. Profiling adds event records between launches,
 * so time work with it off. */
int pf_set_profiling(pf_engine *eng, int on);
int pf_read_profile(pf_engine *eng, int64_t launches[4], double ms[4], int reset);

/* Engine configuration as "key=value" pairs separated by spaces (kernel
 * path, tile shape, x chunks, reciprocal-division axes, coefficient mode,
 * media), written NUL-terminated into buf (at most len bytes). */
int pf_info(const pf_engine *eng, char *buf, int len);

/* Device bytes held by the engine. */
int pf_device_bytes(const pf_engine *eng, int64_t *bytes);

/* Release everything. NULL is a no-op. */
void pf_destroy(pf_engine *eng);

/* Poynting flux of one plane of one time level, allocating no device memory.
 * No counterpart in the reference: it is this library's flux reduction for
 * callers that cannot allocate device memory on their call path - a process
 * whose device memory belongs to another allocator (a framework's caching
 * pool, a server that reserved its whole budget up front), code that only
 * borrows field buffers and holds no allocator, or a time loop that must not
 * pay cudaMalloc's device-wide synchronisation.
 * fields: six device pointers Ex, Ey, Ez, Hx, Hy, Hz, C-order (nx, ny, nz) in
 * the real type. Writes, on `stream` (a cudaStream_t, NULL = default stream),
 * *out = double(T(sum S) * T(dA)) * dt into the caller's device double - the
 * quantity the engine's flux monitor adds per step. Asynchronous: read *out
 * after the stream has done.
 * Scratch: the per-block partial sums live in one fixed device array of
 * 65,536 doubles (512 KB) per GPU that loads the library, kept until the
 * process exits; planes of more than 16,777,216 cells are rejected with
 * PF_ERR_INVALID. Every call made outside a stream capture looks up that
 * array's device address with the device current (a lookup, no allocation),
 * so the address stays right after cudaDeviceReset reloads the module; a
 * call inside a capture reuses the last address found on that device, so
 * make the first call on a device before any stream capture (a first call
 * inside one returns PF_ERR_STATE).
 * Every call shares the array and each call writes all partials it reads, so
 * no state carries between calls; calls that overlap on the GPU (other
 * streams or threads) race on it. Error text: pf_noalloc_last_error(). */
int pf_flux_plane_noalloc(int real_bytes, int nx, int ny, int nz,
                          const void *const fields[6], int axis, int idx,
                          double dA, double dt, double *out, void *stream);
const char *pf_noalloc_last_error(void);

/* ----------------------------------------------------------------------
 * Subpixel permittivity on the GPU (replaces the host precompute of
 * src/photonfdtd/smoothing.py:87-172 for scenes made of boxes).
 * Grid nx x ny x nz, `factor` sub-cells per resolved axis; the scene is the
 * background permittivity overwritten, in order, by n_box boxes, box s
 * covering the fine sub-cells [spans[6s], spans[6s+1]) x [spans[6s+2],
 * spans[6s+3]) x [spans[6s+4], spans[6s+5]) with eps_box[s] (fine index i
 * is native cell i / factor on a resolved axis; a collapsed axis has one
 * fine cell). hx, hy, hz: the gradient spacing (the cell size) of each
 * resolved axis. Writes eps_xx, eps_yy, eps_zz (nx*ny*nz each, C order, 4- or
 * 8-byte reals per out_bytes) to host memory, bit for bit the reference's
 * numpy result. Allocates and frees its own device scratch; synchronous.
 * Error text: pf_smooth_last_error(). */
int pf_smooth_boxes(int nx, int ny, int nz, int factor, double background, int n_box,
                    const int32_t *spans, const double *eps_box, double hx, double hy,
                    double hz, int out_bytes, void *out_xx, void *out_yy, void *out_zz);
const char *pf_smooth_last_error(void);

/* ------------------------------------------------------------------------
 * Batched 2D TE engine with a discrete adjoint (pf_batch).
 *
 * Many 2D instances (xy plane, nz = 1) of uneven size, stepped together on
 * one stream: Hz, Ex, Ey with CPML on x and y, per-cell E coefficient
 * K = dt/(eps*eps0), soft sources and one output-line DFT of Ey per instance.
 * It replaces the reference's per-simulation gradient path for this problem:
 * jax_value_and_grad_eps / value_and_grad_eps (src/photonfdtd/
 * jaxbackend.py:666-722, remat checkpointing :511-570) and its reversible
 * variants (src/photonfdtd/reversible_pml.py:100-209), whose stepping is
 * simulation.py:1252-1309 restricted to TE with nz = 1. The forward fields
 * and DFT match the reference's NumPy run of each instance to the bit.
 *
 * Sequence: pfb_create, pfb_set_instance (each k), pfb_set_sources,
 * pfb_set_dft, pfb_finalize; then per design iteration pfb_set_design_ce,
 * pfb_forward, pfb_read_dft, pfb_adjoint(cotangent), pfb_read_grad.
 * Packed layouts: line cells in instance order, ny_k per instance (the x
 * index line_i, every y); design cells in instance order, dn_k * dn_k each,
 * C order (i, j) inside the window.
 * ---------------------------------------------------------------------- */
typedef struct pf_batch pf_batch;

/* n_inst instances sharing dx, dy, ch = dt/mu0 (real type), dt and n_steps. */
int pfb_create(int n_inst, int real_bytes, double dx, double dy, double ch, double dt,
               int64_t n_steps, pf_batch **out);

/* Instance k: grid nx x ny, ce (nx*ny reals, C order), CPML coefficient
 * arrays coef = {b_e_x, c_e_x, b_h_x, c_h_x (nx each), b_e_y, c_e_y, b_h_y,
 * c_h_y (ny each)} (simulation.py:794-808), the design window
 * [di0, di0+dn) x [dj0, dj0+dn) whose coefficient gradient is returned, and
 * the x index of the output line. */
int pfb_set_instance(pf_batch *b, int k, int nx, int ny, const void *ce,
                     const void *const coef[8], int di0, int dj0, int dn, int line_i);

/* Soft sources (simulation.py:1367-1390): source q adds amp[q] *
 * wave[wave_row[q]][n] to component comp[q] (0 Ex, 1 Ey, 2 Hz) of instance
 * inst[q] at (i[q], j[q]) in step n; wave is (n_wave, n_steps) doubles,
 * already evaluated at the family's times. Sources on one cell are added in
 * list order. */
int pfb_set_sources(pf_batch *b, int n_src, const int32_t *inst, const int32_t *comp,
                    const int32_t *i, const int32_t *j, const int32_t *wave_row,
                    const double *amp, int n_wave, const double *wave);

/* DFT phases: phase[n][f] = exp(i w_f (n+1) dt) as (re, im) doubles,
 * n_steps x n_freq (simulation.py:1116-1133). */
int pfb_set_dft(pf_batch *b, int n_freq, const double *phase);

/* Lays out the pooled arrays and uploads everything. checkpoint_every = K:
 * the state is stored every K steps (ceil(n_steps/K) - 1 states), and the
 * adjoint replays K steps at a time; K >= n_steps stores no state and needs
 * no replay. K = 0 makes a forward-only batch: no adjoint state is allocated
 * and pfb_adjoint / pfb_read_grad return PF_ERR_STATE. tile_rows: x rows per 32-wide tile (8, 16 or 32; a thread
 * updates tile_rows / 8 consecutive rows). */
int pfb_finalize(pf_batch *b, int checkpoint_every, int tile_rows);

/* Re-lays the work list at another tile height (8, 16 or 32 x rows) after
 * pfb_finalize; allocates nothing (the tile buffer is sized for 8). Results
 * do not depend on the tile height. No counterpart in the reference (its
 * GPU path launches one thread per cell, rust/src/cuda.rs:298-341). */
int pfb_set_tile_rows(pf_batch *b, int tile_rows);
/* The tile-height autotuner: for 8, 16 and 32 rows, runs trial_steps forward
 * steps (clamped to the checkpoint spacing and n_steps) once to capture
 * their graph and once timed by CUDA events on the batch stream; writes the
 * three ms per step to ms_per_step[3], keeps the fastest height (*best_rows)
 * and resets the state (fields, ring, DFT sums): call it before pfb_forward.
 * No counterpart in the reference. */
int pfb_tune_tiles(pf_batch *b, int trial_steps, float *ms_per_step, int *best_rows);

/* Replaces the design-window coefficients of every instance from a packed
 * host array (n_design reals). */
int pfb_set_design_ce(pf_batch *b, const void *ce_design);

/* Runs all n_steps from zero fields; the DFT accumulators hold the result. */
int pfb_forward(pf_batch *b);

/* Reverse pass for the loss whose DFT cotangent is `cotangent`: packed line
 * cells x n_freq complex (re, im) doubles, G = dL/dRe F + i dL/dIm F.
 * Afterwards pfb_read_grad gives dL/dK of every design cell. May be called
 * again after the same forward with another cotangent. Leaves the forward
 * fields overwritten (pfb_read_field then shows a replayed state). */
int pfb_adjoint(pf_batch *b, const double *cotangent);

/* Packed DFT accumulators (line cells x n_freq complex doubles). */
int pfb_read_dft(pf_batch *b, double *dst);
/* Packed dL/dK of the design cells (doubles). */
int pfb_read_grad(pf_batch *b, double *dst);
/* Component comp (0 Ex, 1 Ey, 2 Hz) of instance k, nx*ny reals. */
int pfb_read_field(pf_batch *b, int k, int comp, void *dst);
/* out[0..n_out): cells, line cells, design cells, tiles, K, segments,
 * reals per stored state, kernel launches issued so far, and 1 when the
 * forward and reverse steps run as one fused launch each on double-buffered
 * state (every batch without Hz sources), 0 for the split passes. */
int pfb_info(const pf_batch *b, int64_t *out, int n_out);
/* The batch's cudaStream_t. */
void *pfb_stream(pf_batch *b);
const char *pfb_last_error(const pf_batch *b);
void pfb_destroy(pf_batch *b);

/* ------------------------------------------------------------------------
 * The density chain of topology optimisation (pfd_*), replacing the
 * reference's JAX conic_filter + tanh_projection (src/photonfdtd/design.py:
 * 40-72) and the density end of value_and_grad_density (:164-175). A batch of
 * n_inst windows of n x n raw densities (float64, device pointers, window k
 * at k * n * n, row-major), n <= 96, filter radius R (cells) <= 32:
 *   rho_phys = tanh_projection(conic_filter(rho, R), beta, eta), where the
 *   filter is the normalised same-size convolution with the cone
 *   max(0, 1 - |d| / R) (R < 1: none) and the projection
 *   (tanh(beta eta) + tanh(beta (y - eta))) / (tanh(beta eta) +
 *   tanh(beta (1 - eta))) (beta = 0: none).
 * pfd_density_backward: grad_rho = (d rho_phys / d rho)^T grad_phys.
 * Asynchronous on `stream`; allocate nothing. Error text: pfd_last_error(). */
const char *pfd_last_error(void);
int pfd_density_forward(int n_inst, int n, const double *rho, double radius, double beta,
                        double eta, double *rho_phys, void *stream);
int pfd_density_backward(int n_inst, int n, const double *rho, double radius, double beta,
                         double eta, const double *grad_phys, double *grad_rho, void *stream);

/* ------------------------------------------------------------------------
 * Surrogate network kernels (pfs_*). The reference has no learned surrogate:
 * these are the training and inference routines of this library's
 * convolutional encoder-decoder (photonfdtd_b200/surrogate.py), which maps
 * a design density to its transmission spectrum. All pointers are device
 * pointers owned by the caller; BF16 buffers are passed as void*; `stream`
 * is a cudaStream_t (NULL = default stream). Calls are asynchronous and
 * allocate nothing. Error text: pfs_last_error() (per host thread).
 * ---------------------------------------------------------------------- */
const char *pfs_last_error(void);
/* C (M x N, FP32, ld ldc) = alpha * A B^T + beta * C; A M x K and B N x K
 * row-major BF16, K a multiple of 32, lda / ldb multiples of 8, A and B
 * 16-byte aligned. Tensor cores (BF16 in, FP32 accumulate). */
int pfs_gemm_bf16(int M, int N, int K, const void *A, int lda, const void *B, int ldb,
                  float *C, int ldc, float alpha, float beta, void *stream);
/* pfs_gemm_bf16 with the K range split over `splits` blocks along z, for
 * small M x N and long K (weight gradients): partial products go to `work`
 * (at least splits * M * N floats) and are added in a fixed order. */
int pfs_gemm_bf16_splitk(int M, int N, int K, const void *A, int lda, const void *B, int ldb,
                         float *C, int ldc, float alpha, float beta, int splits, float *work,
                         int64_t work_floats, void *stream);
/* pfs_gemm_bf16_splitk with either operand stored MN-major: a_mn = 1 means A
 * is held as its transpose, K x M row-major (lda >= M), b_mn = 1 that B is
 * held as K x N row-major (ldb >= N). The tensor cores read such an operand
 * as it lies (no transposed copy): C = alpha * op(A) op(B)^T + beta * C with
 * the same products in the same order. The backward pass of the surrogate's
 * layers uses it for dW = dY^T X and dX = dY W. tcgen05 engine only. */
int pfs_gemm_bf16_ex(int M, int N, int K, const void *A, int lda, int a_mn, const void *B,
                     int ldb, int b_mn, float *C, int ldc, float alpha, float beta, int splits,
                     float *work, int64_t work_floats, void *stream);
/* A layer's forward GEMM with pfs_bias_act fused into its epilogue (the
 * surrogate network's forward pass uses it):
 * y32 = act(A B^T + bias) (FP32, ld ldy) and, when y16 is not NULL, the
 * same values in BF16 (ld ldy); bias may be NULL, relu != 0 applies ReLU.
 * Equal bit for bit to pfs_gemm_bf16 (alpha 1, beta 0) then pfs_bias_act.
 * tcgen05 engine only. */
int pfs_gemm_bf16_bias_act(int M, int N, int K, const void *A, int lda, const void *B, int ldb,
                           const float *bias, int relu, float *y32, void *y16, int ldy,
                           void *stream);
/* Selects the tensor-core engine of the two GEMM entry points for the
 * process: 1 = tcgen05.mma with the accumulator in tensor memory (default),
 * 0 = mma.sync m16n8k16 with register accumulators. Other values only query.
 * Returns the previous engine. */
int pfs_gemm_engine(int engine);
/* Number of tcgen05 GEMM blocks whose bounded wait for their MMAs ran out
 * (their output tile is then not written); reset = 1 clears it. Synchronous. */
int pfs_gemm_timeouts(int *count, int reset);
/* Test hook of the tcgen05 GEMM for the process: with on = 1, the MMA warp of
 * block (0, 0, 0) first waits 100 us on a barrier nothing arrives on, so the
 * wait runs out and the block takes its timeout path (it drains its loads,
 * counts a timeout, leaves its tile unwritten and frees its tensor memory).
 * 0 turns it off; other values only query. Returns the previous setting. */
int pfs_gemm_wait_test(int on);
/* Lowering of a 2D convolution (kernel kh x kw, stride, zero padding ph
 * rows / pw columns) over NHWC BF16 input x (nb, H, W, C): col rows
 * (b, oy, ox), columns (ky * kw + kx) * C + c, zero-padded to Kp. */
int pfs_im2col(int nb, int H, int W, int C, int kh, int kw, int stride, int ph, int pw,
               const void *x, void *col, int Kp, void *stream);
/* Adjoint of pfs_im2col: FP32 dcol -> FP32 dx (nb, H, W, C), overwritten. */
int pfs_col2im(int nb, int H, int W, int C, int kh, int kw, int stride, int ph, int pw,
               const float *dcol, int Kp, float *dx, void *stream);
/* y = act(x + bias) on an M x N matrix (bias may be NULL; relu 0/1); FP32
 * and / or BF16 outputs. */
int pfs_bias_act(int64_t M, int N, const float *x, const float *bias, int relu, float *y32,
                 void *y16, void *stream);
/* Backward of pfs_bias_act: d = dy * (y > 0) (or dy) into d32 / d16 (either
 * may be NULL) and dbias[n] = sum_m d (if dbias; part holds row_blocks * N
 * floats of scratch, row_blocks in [1, 65535]). */
int pfs_act_bwd(int64_t M, int N, const float *dy, const float *y, int relu, float *d32,
                void *d16, float *dbias, float *part, int row_blocks, void *stream);
/* out (Cc x ldo) = transpose of in (R x Cc, ld ldi), columns R..ldo-1 zero. */
int pfs_transpose_bf16(int R, int Cc, const void *in, int ldi, void *out, int ldo,
                       void *stream);
int pfs_to_bf16(int64_t n, const float *x, void *y, void *stream);
/* Nearest 2x upsampling along W of a (nb, W, C) BF16 tensor, and its adjoint
 * (FP32, (nb, 2W, C) -> (nb, W, C)). */
int pfs_upsample2(int64_t nb, int W, int C, const void *x, void *y, void *stream);
int pfs_upsample2_bwd(int64_t nb, int W, int C, const float *dy, float *dx, void *stream);
/* Mean squared error of the first `used` columns of y (rows x ld) against t
 * (rows x used): grad (rows x ld) = 2 (y - t) / (rows * used) in those
 * columns, 0 elsewhere, and nparts partial losses (their sum is the loss). */
int pfs_mse(int64_t rows, int used, int ld, const float *y, const float *t, float *grad,
            float *loss_parts, int nparts, void *stream);
/* One Adam step (bias-corrected, step >= 1; decoupled weight decay:
 * w -= lr * (m_hat / (sqrt(v_hat) + eps) + wd * w)) on FP32 master weights
 * w, refreshing the BF16 copy w16 if given. */
int pfs_adam(int64_t n, float *w, const float *g, float *m, float *v, float lr, float b1,
             float b2, float eps, int step, float wd, void *w16, void *stream);

/* ------------------------------------------------------------------------
 * Waveguide mode operator (pfm_*), for the GPU mode solver
 * (photonfdtd_b200/mode.py), replacing the reference's scipy assembly of the
 * full-vectorial transverse-E operator (src/photonfdtd/mode.py:256-286) and
 * the operator products of its ARPACK eigensolve (:294-297). All pointers
 * are device pointers, doubles; calls are asynchronous on `stream` and
 * allocate nothing. Cross-section ny x nz, flat index iy * nz + iz; a block
 * holds nvec vectors of 2 * ny * nz values each, [E_z; E_y] as the
 * reference orders its unknowns; eps: ny * nz relative permittivities;
 * k2 = (2 pi / wavelength)^2. Error text: pfm_last_error().
 * ---------------------------------------------------------------------- */
const char *pfm_last_error(void);
/* y = P x for the block (x != y). work: 6 * ny * nz * nvec doubles. */
int pfm_apply(int ny, int nz, double dy, double dz, double k2, const double *eps,
              const double *x, double *y, int nvec, double *work, void *stream);
/* x <- T_degree((P - c) / e) x in place, the Chebyshev polynomial of the
 * first kind mapped so that [lo, hi] goes to [-1, 1] (c, e its centre and
 * half width): it damps the part of the spectrum in [lo, hi] and amplifies
 * what lies above hi. work: 10 * ny * nz * nvec doubles. */
int pfm_chebyshev(int ny, int nz, double dy, double dz, double k2, const double *eps,
                  double *x, int nvec, int degree, double lo, double hi, double *work,
                  void *stream);

#ifdef __cplusplus
}
#endif

#endif /* PFB200_H */

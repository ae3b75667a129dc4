/*
 * steam_b200.h -- C ABI of the B200 (sm_100a) STEAM field-generation path.
 *
 * Conventions shared by every entry point:
 *   - Fields are C-order (nx, ny, nz) arrays, z fastest, in device memory the
 *     caller owns (e.g. torch CUDA tensors).  `dtype` selects float32
 *     (STEAM_F32) or float64 (STEAM_F64) element type for every field
 *     argument of the call.
 *   - Per-level vectors (length nz) and small parameter tables are HOST
 *     pointers unless the name ends in `_dev`.
 *   - `stream` is a cudaStream_t; all work is enqueued on it.  Entry points
 *     that return host scalars synchronise that stream before returning.
 *   - Entries that need scratch device memory take (workspace,
 *     workspace_bytes); the matching *_workspace_bytes() query gives the size.
 *   - Every entry returns 0 (STEAM_OK) or a STEAM_ERR_* code; the message is
 *     available from steam_last_error() on the calling thread.
 *   - A `window` (x0, x1, y0, y1) restricts every realized mean to a nest's
 *     own extent; NULL means the whole array (a root run).
 *
 * Each declaration names the reference (thomasdewitt/STEAM) interface it
 * replaces, by file:line.
 */
#ifndef STEAM_B200_H
#define STEAM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* steam_stream_t;

enum { STEAM_F32 = 0, STEAM_F64 = 1 };

enum {
  STEAM_OK = 0,
  STEAM_ERR_ARG = 1,          /* bad argument (maps to ValueError)         */
  STEAM_ERR_CUDA = 2,         /* CUDA runtime error (maps to RuntimeError) */
  STEAM_ERR_WORKSPACE = 3,    /* workspace too small (maps to MemoryError) */
  STEAM_ERR_UNSUPPORTED = 4   /* shape/option outside the kernels' range   */
};

/* Where a working array sits in the world (steam/simulate.py:520-551,
 * NoiseRegion): array shape, world index of cell (0,0,0) on this class's
 * world grid, the world grid's shape (x and y wrap, z never does), the
 * sparsity factors and the class's 96-bit Philox key (steam/noise.py:133). */
typedef struct {
  int64_t shape[3];
  int64_t origin[3];
  int64_t world[3];
  int32_t sparsity[3];
  uint32_t key[3];
} steam_region_t;

/* Domain window (steam/simulate.py:2049, _inner_view). */
typedef struct {
  int64_t x0, x1, y0, y1;
} steam_window_t;

const char* steam_last_error(void);
int steam_version(void);
/* Number of kernels this library has enqueued since it was loaded. */
unsigned long long steam_launch_count(void);

/* ---- a1-a3: world-keyed uniforms --------------------------------------
 * Replaces keyed_uniforms (steam/noise.py:103-130).  world_i* are DEVICE
 * int64 index vectors (already wrapped by the caller; iy must lie in
 * [0, 2^32)); lane0/lane1 are DEVICE float32 outputs of length nx*ny*nz in
 * C order over (ix, iy, iz). */
int steam_keyed_uniforms(const int64_t* world_ix, int64_t nx,
                         const int64_t* world_iy, int64_t ny,
                         const int64_t* world_iz, int64_t nz,
                         uint32_t key0, uint32_t key1, uint32_t key2,
                         float* lane0, float* lane1, steam_stream_t stream);

/* ---- a5-a6: sparse world-keyed extremal Levy field --------------------
 * Replaces _keyed_sparse_levy (steam/simulate.py:554-598) with its CMS
 * transform (_levy_from_uniforms, steam/simulate.py:441-479).  Writes the
 * generator gamma (zero off the turbulon-centre sub-lattice) to `out`. */
int steam_levy_field(int dtype, const steam_region_t* region, double alpha,
                     void* out, steam_stream_t stream);

/* ---- a7 + a11 measure: multiplier noise fused with the entering sums ----
 * Replaces the first half of _advance_flux (steam/simulate.py:2128-2188):
 * gamma -> zero bottom/top n_zero levels -> eps = expm1(scale*gamma - shift)
 * (0 off-centre) -> product = eps * flux.  sums_out (HOST, 4 doubles) gets
 * { sum(flux) over window, count of window cells, sum|eps| over window,
 *   count of nonzero eps over window }. */
size_t steam_flux_noise_workspace_bytes(void);
int steam_flux_noise(int dtype, const steam_region_t* region, double alpha,
                     double per_class_scale, double shift, int32_t n_zero,
                     int32_t zero_bottom, int32_t zero_top, const void* flux,
                     void* product, const steam_window_t* window,
                     double* sums_out, void* workspace, size_t workspace_bytes,
                     steam_stream_t stream);

/* ---- a9/a10/a13: convolution, circular x/y and linear z ----------------
 * Replaces convolve_fft_xy_oa_z (steam/utils.py:293-427) and the CONVOLVE
 * hook (steam/simulate.py:41).  The kernel is given as a separable network
 * (exactly what the turbulon kernels are, up to float32 rounding):
 *   u_c   = f  (*)_z  Z_c                     c < n_z
 *   v_p   = u_{pair_z[p]} (*)_y Y_{pair_y[p]} p < n_pairs
 *   w_a   = sum_p mix[a * n_pairs + p] v_p    a < n_x
 *   out   = epilogue( sum_a w_a (*)_x X_a )
 * with x and y circular over the array period and z linear (zero padded);
 * each axis' filter of length k has its centre at index c (out[i] =
 * sum_j F[j] in[i - j + c]).  Taps are HOST doubles: z_taps[n_z*kz],
 * y_taps[n_y*ky], x_taps[n_x*kx].
 * `pre_div`/`pre_mul` (HOST per-level, may be NULL) scale the input on the
 * fly: f' = (f / pre_div[z]) * pre_mul[z] (the pattern normalisation of
 * steam/simulate.py:1989-1992).
 * Epilogues: STEAM_EPI_STORE writes out; STEAM_EPI_FLUX treats `out` as the
 * flux F and applies F = max(F + conv, 0) (steam/simulate.py:2192-2203),
 * writing to sums_out (HOST, 3 doubles) { sum(F) over window, window cells,
 * count of F+conv < 0 over the whole array }.  STEAM_EPI_STORE_WIDE stores
 * like STEAM_EPI_STORE with the flux convolution's float64 accumulation (the
 * fused separable form; the FFT form computes in float32 and the direct sum
 * in float64 either way): the tiled flux advance stores its convolution and
 * applies the epilogue per tile (steam_flux_clip_async). */
enum { STEAM_EPI_STORE = 0, STEAM_EPI_FLUX = 1, STEAM_EPI_STORE_WIDE = 2 };
typedef struct {
  int32_t kz, ky, kx;
  int32_t cz, cy, cx;
  int32_t n_z, n_y, n_x, n_pairs;
  int32_t pair_z[16];
  int32_t pair_y[16];
  double mix[64];
} steam_sepconv_t;
size_t steam_conv_workspace_bytes(int dtype, int64_t nx, int64_t ny, int64_t nz,
                                  const steam_sepconv_t* spec);
int steam_conv_separable(int dtype, int64_t nx, int64_t ny, int64_t nz,
                         const steam_sepconv_t* spec, const double* z_taps,
                         const double* y_taps, const double* x_taps,
                         const void* in, const double* pre_div,
                         const double* pre_mul, void* out, int32_t epilogue,
                         const steam_window_t* window, double* sums_out,
                         void* workspace, size_t workspace_bytes,
                         steam_stream_t stream);
/* Tuning of the fused separable kernels, which have no counterpart in the
 * reference (its FFT block length is fixed, steam/utils.py:341): x planes
 * per CTA for fields of shape (nx, ny, nz), chosen by the host autotuner
 * (steam_b200/ensemble.py); 0 restores the default (256 for the scalar fused
 * kernel; for the packed float32 kernel the chunk that fills whole waves of
 * CTAs).  The chunk changes which CTA computes an output, never the order of
 * its sums, so results are identical for every chunk.  The workspace query
 * already covers any chunk. */
int steam_conv_set_xchunk(int64_t nx, int64_t ny, int64_t nz, int32_t chunk);
int steam_conv_get_xchunk(int64_t nx, int64_t ny, int64_t nz);
/* The packed float32 kernel's CTA tile height for fields of shape (nx, ny,
 * nz): 32 rows (256 threads, two CTAs per SM) or 64 rows (512 threads, one
 * per SM, 1.19 instead of 1.375 staged rows per output row); 0 restores 32.
 * Every output voxel's arithmetic is the same at either height, so results
 * are identical. */
int steam_conv_set_tile_rows(int64_t nx, int64_t ny, int64_t nz, int32_t rows);
int steam_conv_get_tile_rows(int64_t nx, int64_t ny, int64_t nz);

/* Grouped convolutions (no counterpart in the reference): n float32 fields
 * convolved with the same separable filters (a spec steam_conv_separable
 * runs on the packed kernel) as ONE launch, every field its own range of
 * blocks.  A field's output is the same bits as a launch of its own.  When
 * the group's tiles give every SM at least 4 CTAs, each field's CTAs take its
 * whole x extent (no repeated halo planes) and its flux sums equal its own
 * launch's to rounding; otherwise each keeps its own launch's x chunk and its
 * sums are the same bits too.  Every field: the packed
 * kernel's layout (nz % 4 == 0, ny even, 16-byte aligned in and out), nx, ny
 * >= 13, 32-row tiles; all fields or none take the input scaling.
 * prepare (synchronous, outside stream capture) lays the group out in
 * `workspace` (DEVICE, steam_conv_group_workspace_bytes) and records it under
 * that address; async enqueues the convolutions (capturable, repeatable on
 * the same buffers); release forgets the group.  sums: DEVICE, 2 doubles per
 * field for STEAM_EPI_FLUX ({sum F over the window, clip count}), or NULL. */
typedef struct {
  int64_t nx, ny, nz;
  const void* in;        /* DEVICE float32 (nx, ny, nz) */
  void* out;             /* DEVICE float32 (nx, ny, nz); F for STEAM_EPI_FLUX */
  const void* pre;       /* DEVICE float32 [2][nz] {div, mul}, or NULL */
  int32_t has_window;    /* 0: the whole array */
  steam_window_t window;
  double* sums;
} steam_conv_problem_t;
size_t steam_conv_group_workspace_bytes(int32_t n, const steam_conv_problem_t* problems);
int steam_conv_group_prepare(const steam_sepconv_t* spec, const double* z_taps,
                             const double* y_taps, const double* x_taps, int32_t n,
                             const steam_conv_problem_t* problems, int32_t epilogue,
                             void* workspace, size_t workspace_bytes);
int steam_conv_group_async(void* workspace, steam_stream_t stream);
int steam_conv_group_release(void* workspace);

/* Float32 flux convolutions (STEAM_EPI_FLUX on float32 fields) run on the
 * packed float32 kernel by default (wide = 0); wide = 1 runs them with
 * float64 taps and accumulators instead.  Process-wide. */
int steam_conv_set_flux_wide(int32_t wide);

/* The packed kernel's slab copies complete on mbarriers whose waits are
 * bounded: a block that waits past the limit waits (bounded again) for its
 * copies in flight, counts itself here and leaves without finishing its
 * tile.  Reads the count of such blocks since the last call into *count and
 * resets it (synchronises the current device). */
int steam_take_wait_errors(int32_t* count);
/* The packed kernel's slab-wait limit in polls (0: the default, seconds of
 * waiting) and a test hook: withhold = 1 issues no slab copy at all, so that
 * every wait runs out with nothing in flight -- the blocks give up and count
 * themselves -- without any fault.  Read when a launch is enqueued (a group:
 * when it is prepared); 0, 0 restores the defaults. */
int steam_set_copy_wait(int64_t polls, int32_t withhold);

/* Launches of the packed float32 kernel so far in this process. */
int64_t steam_conv_packed_launches(void);

/* ---- a9/a10 for kernels without a separable form -----------------------
 * The Morlet turbulon (steam/turbulons.py:40-48) and any kernel whose Tucker
 * factorisation is not exact to the dtype's tolerance.  Same semantics as
 * convolve_fft_xy_oa_z (steam/utils.py:293-427): x and y circular over the
 * field's period, z linear with zero padding; the kernel is NOT folded onto
 * the period: (cx, cy) are the centres the fold implies (k//2 - (1 if n even)
 * for an axis longer than its period n, (k-1)//2 otherwise) and cz =
 * (kz-1)//2.  Prologue and epilogues as steam_conv_separable: pre_div /
 * pre_mul (HOST, per level, may be NULL) or pre_dev (DEVICE [2][nz] of the
 * call's dtype) scale the input by pre[1][z] / pre[0][z]; STEAM_EPI_FLUX
 * makes out = max(out + conv, 0) with { sum out over the window, cells,
 * clip count } in sums_out (HOST, 3 doubles) or { sum, clip count } in
 * sums_dev (DEVICE, 2 doubles).
 *
 * Kernel spectrum (replaces steam/utils.py:367-375): the kernel (DEVICE
 * float64, C order (kx, ky, kz), each extent <= 25) zero-padded to 32^3 and
 * transformed in float64 on the device, stored as complex float32
 * [17][32][32] in the order the FFT kernel reads it. */
size_t steam_conv_fft_spectrum_bytes(void);
int steam_conv_fft_spectrum(const double* kernel_dev, int32_t kx, int32_t ky, int32_t kz,
                            void* spectrum_dev, steam_stream_t stream);

/* Float32 overlap-save FFT convolution on 32^3 cubes (kernel extents <= 25):
 * forward transforms, the spectrum product and the inverse transforms of a
 * cube in one CTA's shared memory, prologue and epilogue fused. */
size_t steam_conv_fft_workspace_bytes(int64_t nx, int64_t ny, int64_t nz);
int steam_conv_fft(int64_t nx, int64_t ny, int64_t nz, int32_t kx, int32_t ky, int32_t kz,
                   int32_t cx, int32_t cy, const void* spectrum_dev, const void* in,
                   const double* pre_div, const double* pre_mul, void* out, int32_t epilogue,
                   const steam_window_t* window, double* sums_out, void* workspace,
                   size_t workspace_bytes, steam_stream_t stream);
int steam_conv_fft_async(int64_t nx, int64_t ny, int64_t nz, int32_t kx, int32_t ky,
                         int32_t kz, int32_t cx, int32_t cy, const void* spectrum_dev,
                         const void* in, const void* pre_dev, void* out, int32_t epilogue,
                         const steam_window_t* window, double* sums_dev, void* workspace,
                         size_t workspace_bytes, steam_stream_t stream);

/* Direct summation over the kernel's taps (float64 fields, where the FFT's
 * float32 arithmetic is not wanted, or kernels longer than 25 taps).
 * kernel_dev is a DEVICE array (kx, ky, kz) of the call's dtype; float64
 * accumulation. */
size_t steam_conv_direct_workspace_bytes(int64_t nx, int64_t ny, int64_t nz);
int steam_conv_direct(int dtype, int64_t nx, int64_t ny, int64_t nz, const void* kernel_dev,
                      int32_t kx, int32_t ky, int32_t kz, int32_t cx, int32_t cy,
                      const void* in, const double* pre_div, const double* pre_mul, void* out,
                      int32_t epilogue, const steam_window_t* window, double* sums_out,
                      void* workspace, size_t workspace_bytes, steam_stream_t stream);
int steam_conv_direct_async(int dtype, int64_t nx, int64_t ny, int64_t nz,
                            const void* kernel_dev, int32_t kx, int32_t ky, int32_t kz,
                            int32_t cx, int32_t cy, const void* in, const void* pre_dev,
                            void* out, int32_t epilogue, const steam_window_t* window,
                            double* sums_dev, void* workspace, size_t workspace_bytes,
                            steam_stream_t stream);

/* ---- a11 apply: scalar rescale ----------------------------------------
 * field *= scale (the volume-mean restore of steam/simulate.py:2208-2215;
 * scale is rounded to the dtype first) or, with fill != 0, field = scale. */
int steam_scale(int dtype, int64_t n, void* field, double scale, int32_t fill,
                steam_stream_t stream);

/* ---- a11 apply on a served tile ------------------------------------------
 * out[i][j][k] = box[x0+i][y0+j][z0+k] * scale (fill != 0: = scale) for the
 * (ox, oy, oz) window of an (nx, ny, nz) box (z fastest); out is contiguous.
 * The volume-mean restore of steam/simulate.py:2208-2215 (scale rounded to the
 * dtype first, as steam_scale) applied only to the cells a tile returns, so a
 * tile server needs no whole-box pass and no strided copy. */
int steam_tile_extract(int dtype, int64_t nx, int64_t ny, int64_t nz, const void* box,
                       int64_t x0, int64_t y0, int64_t z0, int64_t ox, int64_t oy,
                       int64_t oz, double scale, int32_t fill, void* out,
                       steam_stream_t stream);

/* ---- output composition ---------------------------------------------------
 * field = clamp(field + add[z], lo, hi): the mean-profile add and bound clamp
 * of _compose_output (steam/simulate.py:3586-3598).  add is a HOST per-level
 * vector. */
int steam_add_levels_clamp(int dtype, int64_t nx, int64_t ny, int64_t nz, void* field,
                           const double* add, double lo, double hi, steam_stream_t stream);

/* ---- z-major slab ---------------------------------------------------------
 * out[z][x][y] = field[x][y][z0 + z] for z < dz: the level-major layout the
 * streamed output writes (steam/streaming.py:1462-1692), on the device. */
int steam_slab_zmajor(int dtype, int64_t nx, int64_t ny, int64_t nz, const void* field,
                      int64_t z0, int64_t dz, void* out, steam_stream_t stream);

/* ---- the flux epilogue on its own, over a tile's columns --------------------
 * F = max(F + conv, 0) with sums_dev (DEVICE, 2 doubles) = { sum F over the
 * window, count of F + conv < 0 over the window }: the tiled driver's
 * per-tile measure of the realized flux and the clip count of the tile's own
 * columns (steam/streaming.py:1225-1236), for a convolution run with
 * STEAM_EPI_STORE on the tile's box. */
int steam_flux_clip_async(int dtype, int64_t nx, int64_t ny, int64_t nz, void* flux,
                          const void* conv, const steam_window_t* window, double* sums_dev,
                          void* workspace, size_t workspace_bytes, steam_stream_t stream);
size_t steam_flux_clip_workspace_bytes(int64_t nx, int64_t ny, int64_t nz);

/* ---- out-of-core transfers (steam/streaming.py:1139-1280 tile passes) -------
 * steam_box_h2d: the box of bx x by columns at (x0, y0) of a HOST field
 * (nx, ny, nz), wrapping in x and y, levels [z0, z0 + bz), into a contiguous
 * DEVICE box (bx, by, bz).  steam_box_d2h: the window (ox, oy, oz) + (bx, by,
 * bz) of a DEVICE box (bx_full, by_full, bz_full) into the HOST field at
 * (x0, y0, z0), wrapping.  Asynchronous on the stream (page-locked host
 * memory for overlap); elem_bytes 4 or 8. */
int steam_box_h2d(int32_t elem_bytes, const void* host, int64_t nx, int64_t ny, int64_t nz,
                  int64_t x0, int64_t y0, int64_t z0, int64_t bx, int64_t by, int64_t bz,
                  void* dev, steam_stream_t stream);
int steam_box_d2h(int32_t elem_bytes, const void* dev, int64_t bx_full, int64_t by_full,
                  int64_t bz_full, int64_t ox, int64_t oy, int64_t oz, int64_t bx, int64_t by,
                  int64_t bz, void* host, int64_t nx, int64_t ny, int64_t nz, int64_t x0,
                  int64_t y0, int64_t z0, steam_stream_t stream);

/* ---- level-weighted accumulate ------------------------------------------
 * acc += coef[z] * (a - b), or coef[z] * a when b is NULL: the compensation
 * deficit update of cascade_loop (steam/simulate.py:1917, 2024).  coef is a
 * HOST per-level vector. */
int steam_accumulate_levels(int dtype, int64_t nx, int64_t ny, int64_t nz,
                            void* acc, const void* a, const void* b,
                            const double* coef, steam_stream_t stream);

/* ---- per-level reductions (steam/simulate.py:2933-2947) ---------------
 * For each level z: sums_out[4*z + {0,1,2,3}] = { sum f, sum |f|, count of
 * nonzero f, count of cells } over the window (HOST output, 4*nz doubles). */
size_t steam_level_sums_workspace_bytes(int64_t nz);
int steam_level_sums(int dtype, int64_t nx, int64_t ny, int64_t nz,
                     const void* field, const steam_window_t* window,
                     double* sums_out, void* workspace, size_t workspace_bytes,
                     steam_stream_t stream);

/* Allocation-free form of steam_level_sums, for callers that cannot allocate
 * device memory (an application whose own allocator owns the device budget,
 * a C FFI with no device allocator, a loop that must not allocate).  It has no
 * counterpart in the reference.  Same arguments and results as
 * steam_level_sums without (workspace, workspace_bytes): the scratch is one
 * static device array of steam_level_sums_noalloc_scratch_bytes() (4 MiB) that
 * every GPU loading this library holds until exit.  Limit: nz <= 1024
 * (STEAM_ERR_UNSUPPORTED above that); any nx, ny.  The array's address is per
 * CUDA context (the context that loaded this library's module); every call
 * looks it up in the calling thread's current context.  All calls share the
 * one array: calls whose work overlaps on the GPU (other streams, other host
 * threads) race on it; serialise them.  sums_out is written before return:
 * the call copies into host memory and synchronises its stream, so it must
 * never be called while a stream is being captured. */
size_t steam_level_sums_noalloc_scratch_bytes(void);
int steam_level_sums_noalloc(int dtype, int64_t nx, int64_t ny, int64_t nz,
                             const void* field, const steam_window_t* window,
                             double* sums_out, steam_stream_t stream);

/* ---- a12: scalar pattern ----------------------------------------------
 * Replaces the per-scalar pattern of cascade_loop (steam/simulate.py:
 * 1928-1983): running = pert + mean_1d; W = advective weight (periodic
 * x/y, np.gradient z, steam/simulate.py:2787-2868); W *= product * s_scale
 * (the signed amplitude S_k); W *= bound taper (steam/simulate.py:2905-2930).
 * Writes W and level_sums_out (HOST, 2*nz doubles) { sum|W|, count W != 0 }
 * per level over the window.  z_coords (HOST, nz doubles) are the level
 * heights (np.gradient semantics), aspect and buffer_b are HOST per-level.
 * product == NULL leaves out the amplitude and buffer_b == NULL the taper,
 * which gives the advective weight alone (steam/simulate.py:2843-2868). */
size_t steam_scalar_pattern_workspace_bytes(int64_t nx, int64_t ny, int64_t nz);
int steam_scalar_pattern(int dtype, int64_t nx, int64_t ny, int64_t nz,
                         const void* pert, const double* mean_1d,
                         const void* product, double s_scale, double dx,
                         double dy, const double* z_coords,
                         const double* aspect, const double* buffer_b,
                         double phi_min, double phi_max, void* w_out,
                         const steam_window_t* window, double* level_sums_out,
                         void* workspace, size_t workspace_bytes,
                         steam_stream_t stream);

/* ---- a14: bounded amplitude-preserving add -----------------------------
 * Replaces _bounded_amplitude_add (steam/simulate.py:3114-3283): per level,
 * the demean / clip / rescale-to-A0 loop (at most n_rescale steps), a final
 * demean and clip, then the zero-mean shift mu, solved exactly (bracketed
 * Newton on the piecewise-linear level mean) instead of by 60 bisection
 * sweeps.  pert += delta; with record_applied the increment buffer is left
 * holding pert_after - pert_before, otherwise it is scratch (the sweeps store
 * the chain's running state there; its contents on return are unspecified).
 * ledger_out (HOST, may be NULL) receives per level a record of
 * steam_bounded_add_ledger_doubles(n_rescale) doubles: { a0, n_loop,
 * final_demean, mu (NaN if none), n_sweeps, chain steps, final clip set,
 * demean[n_rescale], scale[n_rescale] } -- the last four the per-level chain
 * that steam_bounded_add_replay applies. */
size_t steam_bounded_add_ledger_doubles(int32_t n_rescale);
size_t steam_bounded_add_workspace_bytes(int64_t nz, int32_t n_rescale);
int steam_bounded_add(int dtype, int64_t nx, int64_t ny, int64_t nz,
                      void* pert, const double* mean_1d, void* increment,
                      double phi_min, double phi_max,
                      const steam_window_t* window, int32_t n_rescale,
                      int32_t record_applied, double* ledger_out,
                      void* workspace, size_t workspace_bytes,
                      steam_stream_t stream);

/* ---- a16: mean-preserving projection onto bounds -----------------------
 * Replaces _project_onto_bounds (steam/simulate.py:3417-3489) for levels
 * with a violation; float64 level arithmetic.  mu_out (HOST, nz doubles,
 * may be NULL) is NaN for untouched levels. */
int steam_project_bounds(int dtype, int64_t nx, int64_t ny, int64_t nz,
                         void* pert, const double* mean_1d, double phi_min,
                         double phi_max, const steam_window_t* window,
                         double* mu_out, void* workspace,
                         size_t workspace_bytes, steam_stream_t stream);

/* ---- a15: periodic trilinear regrid -------------------------------------
 * Replaces zoom_trilinear (steam/utils.py:507-534): align_corners=False,
 * x/y wrap when periodic_x/periodic_y, z clamps.  Upsampling or identity on
 * periodic axes. */
int steam_regrid(int dtype, const void* in, int64_t nx, int64_t ny, int64_t nz,
                 void* out, int64_t mx, int64_t my, int64_t mz,
                 int32_t periodic_x, int32_t periodic_y, steam_stream_t stream);

/* ---- a17: thermodynamic column solve ------------------------------------
 * Replaces recover_diagnostics (steam/thermodynamics.py:25-123): dry
 * temperature, Bolton saturation, 5 Newton steps, ice/liquid partition and a
 * float64 hypsometric pressure march.  z_values (HOST, nz doubles); surface
 * pressure is a scalar unless ps_field_dev (DEVICE float64 nx*ny) is given.
 * With h_mean/qt_mean (HOST per-level, both or neither) the inputs are
 * perturbations and the output composition of a deficit-free run is fused in
 * front (steam/simulate.py:3586-3598): h = clamp(h' + h_mean, bounds[0..1]),
 * qt = clamp(qt' + qt_mean, bounds[2..3]).
 * Outputs T, qv, qc, qi, p are DEVICE arrays of the call's dtype. */
int steam_thermo(int dtype, int64_t nx, int64_t ny, int64_t nz, const void* h,
                 const void* qt, const double* z_values, const double* h_mean,
                 const double* qt_mean, const double* bounds,
                 double surface_pressure, const double* ps_field_dev,
                 void* T, void* qv, void* qc, void* qi, void* p,
                 steam_stream_t stream);

/* ---- a8: turbulon kernel build ------------------------------------------
 * Replaces _turbulon_envelope (steam/simulate.py:2503-2556) with the shapes
 * of steam/turbulons.py:23-48 (shape 0 mexican_hat, 1 morlet_omega0_6):
 * box +-ceil(support*k/d) per axis, Gaussian-weighted zero-sum correction
 * with its two sums taken in float64 on the device.  `out` is a DEVICE
 * array of shape dims_out (HOST, 3 int64, filled by a NULL-out call). */
int steam_kernel_build(int dtype, double k, double dx, double dy, double dz,
                       double support_factor, int32_t shape, void* out,
                       int64_t* dims_out, steam_stream_t stream);

/* ---- Resident (asynchronous) forms of the class step ---------------------
 * The entries above return their scalars to the host and synchronise their
 * stream, as the reference's stage functions do.  The *_async entries below
 * keep every scalar in DEVICE memory and never synchronise or allocate: a
 * class step built from them enqueues all of its work at once, with each
 * data-dependent decision (the flux restore factor, the product norm, the
 * pattern's level means, the bounded add's demean/rescale/shift solve) taken
 * by small device kernels between the field sweeps.  Per-level vectors whose
 * names end in _dev are device arrays; z_coords stays a host array (only
 * scalars are derived from it).  Workspaces are the same as the synchronous
 * forms'. */

/* Multiplier noise fused with the entering sums (steam/simulate.py:
 * 2128-2188).  sums_dev (DEVICE, 3 doubles) = { sum F over the window,
 * sum |eps| over the window, count of nonzero eps over the window }. */
int steam_flux_noise_async(int dtype, const steam_region_t* region, double alpha,
                           double per_class_scale, double shift, int32_t n_zero,
                           int32_t zero_bottom, int32_t zero_top, const void* flux,
                           void* product, const steam_window_t* window,
                           double* sums_dev, void* workspace, size_t workspace_bytes,
                           steam_stream_t stream);

/* Separable convolution (steam/utils.py:293-427).  pre_dev (DEVICE, [2][nz]
 * of the call's dtype, may be NULL) scales the input: f' = (f / pre[0][z]) *
 * pre[1][z].  With STEAM_EPI_FLUX, sums_dev (DEVICE, 2 doubles) = { sum F
 * over the window after the clip, count of F + conv < 0 }. */
int steam_conv_separable_async(int dtype, int64_t nx, int64_t ny, int64_t nz,
                               const steam_sepconv_t* spec, const double* z_taps,
                               const double* y_taps, const double* x_taps, const void* in,
                               const void* pre_dev, void* out, int32_t epilogue,
                               const steam_window_t* window, double* sums_dev,
                               void* workspace, size_t workspace_bytes,
                               steam_stream_t stream);

/* The flux advance's volume-mean restore (steam/simulate.py:2204-2218) from
 * the device sums of the two calls above: F *= T(entering / realized), or
 * F = T(entering) when the realized mean is not positive.  cells = window
 * cells x nz.  ledger_dev (DEVICE, 10 doubles, may be NULL) = { entering sum,
 * cells, sum |eps|, nonzero eps, realized sum, cells, clipped count,
 * S scale 1/mean|eps| rounded to the dtype, restore factor, fill flag }. */
int steam_flux_finish_async(int dtype, int64_t n, void* flux, const double* noise_sums_dev,
                            const double* conv_sums_dev, double cells, double* ledger_dev,
                            steam_stream_t stream);

/* The scalar pattern's per-level vectors (steam/simulate.py:2787-2930),
 * built once per class: vecs_dev (DEVICE, [6][nz] of the dtype) = mean,
 * np.gradient's three z coefficients, aspect, taper buffer (1 when buffer_b
 * is NULL).  Synchronises (set-up, not the step). */
int steam_scalar_pattern_vectors(int dtype, int64_t nz, const double* mean_1d,
                                 const double* z_coords, const double* aspect,
                                 const double* buffer_b, void* vecs_dev,
                                 steam_stream_t stream);

/* steam_scalar_pattern with its per-level vectors and the S scale on the
 * device (s_scale_dev: one double, e.g. the flux ledger's entry 7).
 * level_sums_dev (DEVICE, [2][nz]) = { sum |W|, count W != 0 } per level
 * over the window. */
int steam_scalar_pattern_async(int dtype, int64_t nx, int64_t ny, int64_t nz,
                               const void* pert, const void* vecs_dev, const void* product,
                               const double* s_scale_dev, double dx, double dy,
                               const double* z_coords, int32_t has_taper, double phi_min,
                               double phi_max, void* w_out, const steam_window_t* window,
                               double* level_sums_dev, void* workspace,
                               size_t workspace_bytes, steam_stream_t stream);

/* The second convolution's input scaling from the pattern's level sums
 * (steam/simulate.py:1989-1992): pre_dev[0][z] = level mean |W| rounded to
 * the dtype (1 where not positive), pre_dev[1][z] = mul_dev[z] (C_k). */
int steam_pattern_norm_async(int dtype, int64_t nz, const double* level_sums_dev,
                             const double* mul_dev, void* pre_dev, steam_stream_t stream);

/* steam_bounded_add with the level means on the device (mean_dev, nz
 * doubles) and its ledger written to ledger_dev (DEVICE, [nz][5], may be
 * NULL).  With nz % 4 == 0 and 16-byte aligned fields the rescale loop and
 * the shift solve each run as ONE cooperative launch that sweeps while any
 * level needs another sweep; its grid barriers wait a bounded time, and a
 * barrier that gives up ends the launch and marks the ledger's sweep count
 * -1 (the host raises).  Otherwise the launch sequence is fixed (one stats
 * sweep, n_rescale rescale sweeps, 48 shift sweeps, one apply sweep) and
 * sweeps whose phase has ended exit at once. */
/* Apply-only replay of a recorded projection (the replay branch of
 * _project_onto_bounds, steam/simulate.py:3462-3488): levels whose recorded
 * mu (HOST, nz doubles) is not NaN become clip(pert + mean - mu, lo, hi) -
 * mean; the others are left bit-identical.  Workspace as steam_project_bounds. */
int steam_project_bounds_replay(int dtype, int64_t nx, int64_t ny, int64_t nz, void* pert,
                                const double* mean_1d, double phi_min, double phi_max,
                                const double* mu, void* workspace, size_t workspace_bytes,
                                steam_stream_t stream);

/* Apply-only replay of a recorded bounded add (the APPLY-ONLY branch of
 * _bounded_amplitude_add, steam/simulate.py:3196-3213, and
 * _bounded_amplitude_add_cuda's replay): per level, the recorded demeans,
 * clips, scales, final demean and shift are applied to the increment with no
 * reduction, then pert += delta (with record_applied the increment is left
 * holding pert_after - pert_before).  Any subset of the columns of the field
 * that recorded the ledger -- a tile of the world -- replays to the same
 * values there, bit for bit.  ledger (HOST [nz][ledger_doubles]) and mean_1d
 * (HOST) in the synchronous form, both DEVICE in the async one. */
size_t steam_bounded_add_replay_workspace_bytes(int64_t nz, int32_t n_rescale);
int steam_bounded_add_replay(int dtype, int64_t nx, int64_t ny, int64_t nz, void* pert,
                             const double* mean_1d, void* increment, double phi_min,
                             double phi_max, int32_t n_rescale, int32_t record_applied,
                             const double* ledger, void* workspace, size_t workspace_bytes,
                             steam_stream_t stream);
int steam_bounded_add_replay_async(int dtype, int64_t nx, int64_t ny, int64_t nz, void* pert,
                                   const double* mean_dev, void* increment, double phi_min,
                                   double phi_max, int32_t n_rescale, int32_t record_applied,
                                   const double* ledger_dev, void* workspace,
                                   size_t workspace_bytes, steam_stream_t stream);

/* The persistent phases' grid barrier: how many polls (with a short sleep
 * each) a block waits for the others before it gives up, records the error
 * and leaves (the ledger's sweep count becomes -1; the synchronous entry
 * returns STEAM_ERR_CUDA).  0 restores the default (2^26 polls, seconds).
 * Applies to calls enqueued after it, process-wide.  No counterpart in the
 * reference, whose bounded add has no device-side wait. */
int steam_set_barrier_spin_limit(int64_t polls);

/* Grouped bounded adds (no counterpart in the reference, which runs one
 * field at a time): n independent fields' steam_bounded_add_async solves
 * (record_applied = 0) as one launch per stage -- the first and apply sweeps
 * over a flat grid; each persistent phase's first iterations as flat
 * launches (a sweep over the fields still in the loop, their sums, their
 * per-level steps), the rest as one cooperative launch whose blocks split
 * into per-field teams with their own grid barriers, a team's size the
 * field's share of the co-resident capacity.  A field's result is
 * the single call's to rounding (another block partition of its sums); the
 * same group gives the same bits every time.  At most 65535 fields; every
 * field: nz % 4 == 0 (4 .. 1024), 16-byte aligned pert and increment.
 *
 * prepare (synchronous, outside stream capture) lays the group's state out
 * in `workspace` (DEVICE, steam_bounded_add_group_workspace_bytes) and
 * records it under that address; async enqueues the solves (capturable,
 * repeatable: the same fields each time); release forgets the group.
 * ledger: DEVICE, nz * (7 + 2 n_rescale) doubles per field (the record of
 * steam_bounded_add_async), or NULL. */
typedef struct {
  int64_t nx, ny, nz;
  void* pert;            /* DEVICE (nx, ny, nz), updated in place */
  void* increment;       /* DEVICE (nx, ny, nz), consumed */
  const double* mean;    /* DEVICE, nz */
  double phi_min, phi_max;
  int32_t has_window;    /* 0: the whole array */
  steam_window_t window;
  double* ledger;
} steam_ba_problem_t;
size_t steam_bounded_add_group_workspace_bytes(int dtype, int32_t n,
                                               const steam_ba_problem_t* problems,
                                               int32_t n_rescale);
int steam_bounded_add_group_prepare(int dtype, int32_t n, const steam_ba_problem_t* problems,
                                    int32_t n_rescale, void* workspace, size_t workspace_bytes);
int steam_bounded_add_group_async(void* workspace, steam_stream_t stream);
int steam_bounded_add_group_release(void* workspace);

int steam_bounded_add_async(int dtype, int64_t nx, int64_t ny, int64_t nz, void* pert,
                            const double* mean_dev, void* increment, double phi_min,
                            double phi_max, const steam_window_t* window, int32_t n_rescale,
                            int32_t record_applied, double* ledger_dev, void* workspace,
                            size_t workspace_bytes, steam_stream_t stream);

/* steam_thermo with its level profiles on the device: prof_dev (DEVICE,
 * [4][nz] doubles) = z, dz (z[k+1] - z[k], last 0), h mean, qt mean; compose
 * != 0 adds and clamps the means as steam_thermo does with h_mean/qt_mean. */
int steam_thermo_async(int dtype, int64_t nx, int64_t ny, int64_t nz, const void* h,
                       const void* qt, const double* prof_dev, int32_t compose,
                       const double* bounds, double surface_pressure,
                       const double* ps_field_dev, void* T, void* qv, void* qc, void* qi,
                       void* p, steam_stream_t stream);

/* Grouped thermodynamics (no counterpart in the reference, which maps one
 * field at a time): n independent fields' steam_thermo_async as ONE launch,
 * each field's blocks a contiguous range of the grid; every field's result
 * is the same bits as its own call.  prepare (synchronous, outside stream
 * capture) writes the fields' descriptors and a block -> field table to
 * `workspace` (DEVICE, steam_thermo_group_workspace_bytes) and records the
 * group under that address; async enqueues the launch (capturable,
 * repeatable); release forgets the group.  All fields of one group have the
 * dtype given. */
typedef struct {
  int64_t nx, ny, nz;
  const void* h;          /* DEVICE (nx, ny, nz) */
  const void* qt;         /* DEVICE (nx, ny, nz) */
  const double* prof;     /* DEVICE [4][nz]: as steam_thermo_async's prof_dev */
  int32_t compose;
  double bounds[4];       /* used when compose != 0 */
  double surface_pressure;
  const double* ps_field; /* DEVICE (nx, ny) or NULL */
  void* T;                /* DEVICE outputs (nx, ny, nz) */
  void* qv;
  void* qc;
  void* qi;
  void* p;
} steam_thermo_problem_t;
size_t steam_thermo_group_workspace_bytes(int32_t n, const steam_thermo_problem_t* problems);
int steam_thermo_group_prepare(int dtype, int32_t n, const steam_thermo_problem_t* problems,
                               void* workspace, size_t workspace_bytes);
int steam_thermo_group_async(void* workspace, steam_stream_t stream);
int steam_thermo_group_release(void* workspace);

#ifdef __cplusplus
}
#endif

#endif /* STEAM_B200_H */

/* C ABI of the B200 ScatCov engine (libstl_b200.so).
 *
 * Drop-in for the reference's stl-bridge C ABI (jmdelouis/STL-Dev-MPI,
 * crates/stl-bridge/src/lib.rs), bound by its Python module
 * python/stl_ensemble/stl_port/native.py (signature table at
 * native.py:56-110) when STL_NATIVE_LIBRARY points at this library.
 *
 * Conventions (as the reference): maps are f64 NESTED [batch, 12 nside^2];
 * values and cotangents complex128 interleaved (re, im) [batch, ncoeff];
 * the gradient is that of Re sum(conj(cotangent) * values); every forward
 * state has an identity (handle, generation, member, objective) that
 * stlp_vjp / stlp_restore check.  Failures return -1 (int), NULL
 * (pointers) and set stlp_last_error().  One caller thread per handle.
 */
#ifndef STL_B200_H
#define STL_B200_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct StlpHandle StlpHandle;
typedef struct StlpSnapshot StlpSnapshot;
typedef struct StlpPatchHandle StlpPatchHandle;

/* Message of the last failure on the calling thread; library-owned, valid
 * until the next failure on that thread.  (stl-bridge lib.rs:260-263) */
const char* stlp_last_error(void);

/* Frees a string returned by stlp_info / stlp_patch_info.  (lib.rs:266-271) */
void stlp_string_free(char* p);

/* New handle from a JSON config: nside (128), j (7), batch (1), kernel (5),
 * orientations (4), backend ("gpu"; "cpu" is refused: no CPU fallback),
 * device (0), dtype ("float64" | "float32": field precision; sums stay
 * FP64), cross (false), spin (0 | 2), spin_kernel (5: 3, 5, 7 or 9),
 * spin_pyramid ("scalar" | "transported"), spin_a (2 | 0, with cross).
 * Spin 2: maps are (Q, U) [batch, 2, 12 nside^2] (cross: the first fields
 * [batch, 1 or 2, npix] then the second [batch, 2, npix]); values
 * [batch, 2 (chi_E, chi_B), K, ncoeff]; cotangents of the maps' shape.
 * Unknown keys are ignored.  The device operators are built on first use
 * (or by stlp_prepare).  NULL on failure.  (lib.rs:280-351) */
StlpHandle* stlp_new(const char* config);

/* Frees a handle (NULL ignored).  (lib.rs:354-359) */
void stlp_free(StlpHandle* h);

/* JSON: version, sizes, dtype, the plan [{index, family, native_dg, c1, c2,
 * j1, j2, j3, l1, l2, l3}], device memory, timers.  Free with
 * stlp_string_free.  (lib.rs:364-391) */
char* stlp_info(StlpHandle* h);

/* Masked averages: k masks [k, 12 nside^2] (k = 0: whole sky).
 * (lib.rs:396-422) */
int stlp_set_masks(StlpHandle* h, const double* weights, size_t k);

/* Pixels each coefficient averages, [K, ncoeff].  (lib.rs:459-472) */
int stlp_native_pixels(StlpHandle* h, size_t* out);

/* Forward sweep of host maps x (n = batch * 12 nside^2): values to out
 * (2 batch ncoeff), with moments the spatial variances to var (batch
 * ncoeff).  (lib.rs:478-530) */
int stlp_forward(StlpHandle* h, const double* x, size_t n, uint64_t generation, uint64_t member, uint64_t objective,
                 bool moments, double* out, double* var);

/* Map cotangent out (batch * 12 nside^2) of the cotangents cot (n = batch
 * ncoeff complex) after the forward of the same identity.  (lib.rs:535-581) */
int stlp_vjp(StlpHandle* h, const double* cot, size_t n, uint64_t generation, uint64_t member, uint64_t objective,
             double* out);

/* Forward on maps already on the device (x: device pointer to f32 if f32,
 * else f64; same layout as stlp_forward).  Values go to host memory.
 * Runs on the handle's stream (stlp_set_stream) and returns once done.
 * No reference counterpart for full-sky maps; the pattern of
 * stlp_patch_forward_device (lib.rs:1153). */
int stlp_forward_device(StlpHandle* h, uint64_t x, size_t n, int f32, uint64_t generation, uint64_t member,
                        uint64_t objective, bool moments, double* out, double* var);

/* Map cotangent written to device memory out (f32 if f32, else f64) after
 * the forward of the same identity; cotangents on the host.  Returns once
 * the stream has finished.  (pattern of stlp_patch_vjp_device, lib.rs:1171) */
int stlp_vjp_device(StlpHandle* h, const double* cot, size_t n, uint64_t generation, uint64_t member,
                    uint64_t objective, uint64_t out, int f32);

/* CUDA stream (cudaStream_t as an integer, 0: default stream) the handle
 * launches on.  No reference counterpart. */
int stlp_set_stream(StlpHandle* h, uint64_t stream);

/* Mean and var coefficients (<x>, <x^2> per map, FP64, as the MEAN and VAR
 * families of stlp_forward) of batch device maps x [batch][n_pix] (f32 if
 * f32, else f64) into device memory out [batch][2], launched on stream
 * (cudaStream_t as an integer); returns after the launches, without waiting.
 * Allocates nothing: the partial sums sit in a fixed device array of at most
 * 64 maps (296 KiB); a larger batch is refused.  Calls in flight together on
 * one device race on that array.  The first call on a device, and the
 * first after a reset of the device (a new context), looks up the array's
 * address (make it before any stream capture).  The stream must belong to
 * the current device (refused otherwise).  No reference counterpart. */
int stlp_mean_var_noalloc(uint64_t x, size_t n_pix, size_t batch, int f32, uint64_t out, uint64_t stream);

/* Builds the device operators now instead of at the first forward.  No
 * reference counterpart (the reference builds in stlp_new). */
int stlp_prepare(StlpHandle* h);

/* Kernel statistics: reset != 0 clears the per-class launch counts, device
 * times and algorithmic bytes/flops reported by stlp_info ("kernels");
 * on != 0 times every launch with CUDA events on the handle's stream.  The
 * reference's counterpart is its per-phase wall timers (crates/stl-gpu/src/
 * engine.rs:811-818, reported by stlp_info). */
int stlp_profile(StlpHandle* h, int on, int reset);

/* Copy of the current forward state (the loaded maps; the fields are
 * recomputed by stlp_restore); NULL on failure.  (lib.rs:647-659) */
StlpSnapshot* stlp_checkpoint(StlpHandle* h);
void stlp_checkpoint_free(StlpSnapshot* s);                /* (lib.rs:662-667) */
size_t stlp_checkpoint_bytes(const StlpSnapshot* s);       /* (lib.rs:670-680) */
/* Makes a checkpoint of this handle the current state.  (lib.rs:684-709) */
int stlp_restore(StlpHandle* h, const StlpSnapshot* s, uint64_t generation, uint64_t member, uint64_t objective);

/* Statistics of maps given at every level (validation).  (lib.rs:588-623) */
int stlp_forward_levels(StlpHandle* h, const double* x, size_t n, double* out);

/* L-BFGS with strong Wolfe line search of the callback from x (updated in
 * place); options JSON: lr (1), max_iter (20), max_eval, tolerance_grad
 * (1e-12), tolerance_change (1e-15), history_size (10).  Returns the number
 * of evaluations, -1 on failure (non-finite loss or gradient included).
 * (lib.rs:711-741) */
typedef double (*stlp_callback)(const double* x, size_t n, double* grad, void* ctx);
int64_t stlp_lbfgs(double* x, size_t n, const char* options, stlp_callback callback, void* ctx);

/* Synthesis with every vector on the device: L-BFGS (the steps and options
 * of stlp_lbfgs) of the loss sum_i w_(i mod ncoeff) |S_i(x) - T_i|^2 over the
 * maps x (device pointer, float64 [batch][12 nside^2], updated in place), the
 * statistics and their VJP from this handle's engine.  target: the values T
 * (complex interleaved, n_target = batch x masks x ncoeff complex values);
 * weights: ncoeff values or NULL (all 1).  losses (NULL allowed) receives the
 * loss of each evaluation, at most n_losses of them.  Returns the number of
 * evaluations, -1 on failure; the handle's forward state is cleared.  The
 * loop of crates/stl-mpi/src/synthesis.rs:207-316 with the optimiser of
 * stlp_lbfgs (lib.rs:711-741); no reference entry point holds the vectors
 * on the device. */
int64_t stlp_synthesize_device(StlpHandle* h, uint64_t x, size_t n, const double* target, size_t n_target,
                               const double* weights, const char* options, double* losses, size_t n_losses);

/* Disc patches (lib.rs:743-1176). */
StlpPatchHandle* stlp_patch_new(const char* config);
void stlp_patch_free(StlpPatchHandle* h);
char* stlp_patch_info(StlpPatchHandle* h);
int stlp_pixel_vectors(size_t nside, const int64_t* ids, size_t n, double* out);
int stlp_patch_select(StlpPatchHandle* h, const double* centres, size_t b, double radius, double core, size_t* counts);
/* stlp_patch_select with a radius and a core radius per disc (radii, cores:
 * b values in radians; cores NULL or a value <= 0: average the whole disc).
 * No reference counterpart: the reference takes one radius per call. */
int stlp_patch_select_radii(StlpPatchHandle* h, const double* centres, size_t b, const double* radii,
                            const double* cores, size_t* counts);
int stlp_patch_ids(StlpPatchHandle* h, size_t patch, int64_t* out);
int stlp_patch_core_pixels(StlpPatchHandle* h, size_t* out);
int stlp_patch_forward(StlpPatchHandle* h, const double* x, size_t n, uint64_t generation, bool moments, double* out,
                       double* var);
int stlp_patch_vjp(StlpPatchHandle* h, const double* cot, size_t n, uint64_t generation, double* out);
int stlp_patch_forward_device(StlpPatchHandle* h, uint64_t x, size_t n, uint64_t generation, bool moments,
                              double* out, double* var);
int stlp_patch_vjp_device(StlpPatchHandle* h, const double* cot, size_t n, uint64_t generation, uint64_t out);

/* Device memory the library holds for all handles of the process: the live
 * bytes and their high-water mark; reset_peak != 0 first restarts the mark
 * at the live bytes.  No reference counterpart (the reference reports its
 * engine's memory in stlp_info, lib.rs:365-391, as stlp_info does here). */
int stlp_memory(size_t* live, size_t* peak, int reset_peak);

/* Map files, the formats on either side of the statistics: NESTED .npy
 * arrays ('<f8' '>f8' '<f4' '>f4' '<i8' '>i8' '<i4' '>i4', C order) and
 * HEALPix FITS binary tables (the map in the first column, 'E' or 'D', a
 * repeat count allowed; RING maps reordered to NESTED on reading).  A path
 * ending in .fits or .fit is FITS, any other .npy.  The reference's
 * synthesis tools call these in-process (crates/stl-mpi/src/io.rs:18-569:
 * map_len, read_map, read_npy_shape, read_map_range, write_npy_shape,
 * write_healpix_fits, SlicedMap::create / write); no C entry to mirror.
 *   stlp_map_len: *n = the pixels of the map;
 *   stlp_npy_shape: *ndim and shape[0 .. ndim) of a .npy array (an error
 *     when it has more than max_dims axes);
 *   stlp_map_read: the whole map (NESTED float64) into out[n], n its length;
 *   stlp_map_read_range: pixels [start, end) into out[end - start] (read at
 *     their offset; a RING map is read whole);
 *   stlp_npy_write: little-endian float64 .npy of shape[ndim];
 *   stlp_fits_write: a full-sky NESTED map of n pixels as a binary table of
 *     one column named `column`, float64 ('D') when dbl, else float32 ('E');
 *   stlp_map_create / stlp_map_write: a file written in pieces (each
 *     process its own range): the headers and the size for n pixels (.npy
 *     float64, or FITS as stlp_fits_write), then pixels [start, start +
 *     count) at their offset. */
int stlp_map_len(const char* path, size_t* n);
int stlp_npy_shape(const char* path, size_t* shape, size_t max_dims, size_t* ndim);
int stlp_map_read(const char* path, double* out, size_t n);
int stlp_map_read_range(const char* path, size_t start, size_t end, double* out);
int stlp_npy_write(const char* path, const double* values, const size_t* shape, size_t ndim);
int stlp_fits_write(const char* path, const double* values, size_t n, const char* column, int dbl);
int stlp_map_create(const char* path, size_t n, const char* column, int dbl);
int stlp_map_write(const char* path, size_t start, const double* values, size_t count, int dbl);

/* The integer tables of the engine's operators, for exact checks: kind 0
 * the sorted distinct input cells (full-sky NESTED ids) each output pixel
 * of level `level` reads in its wavelet (weight: the cell's largest
 * |coefficient|), kind 1 the sorted fine cells of nonzero weight each
 * coarse pixel of level + 1 reads in the decimation (weight: |w|).
 * *needed = the widest row; when out is not NULL and width >= *needed,
 * out [pixels][width] gets the rows in pixel order, padded with -1, and
 * weight (or NULL) the weights, padded with 0.  No reference counterpart
 * (the reference's tests read its Rust tables). */
int stlp_operator_rows(StlpHandle* h, size_t level, int kind, int64_t* out, double* weight, size_t width,
                       size_t* needed);

/* Objective terms of the synthesis on the device (the loss terms stl-synth
 * adds after the statistics).  The reference has no C entry points for
 * them: its CLI calls crates/stl-gpu/src/terms.rs in-process (DeviceTable,
 * Pyramid, RadixSort, marginal_row, add_product; kernels.cu:1454-1707);
 * these expose the same operations to C and Python callers.  Device
 * addresses are uint64_t (f64 arrays unless noted), every launch goes to
 * the handle's stream; calls that return host values wait for it.
 * Configuration JSON: rows (1), len (cells per row, a multiple of
 * 4^depth), depth (pyramid levels above the maps), sort (most values one
 * sort takes), device (0).  Element-wise results equal the host
 * expressions bit for bit; sums over pixels are fixed-order chunk trees. */
typedef struct StlpTerms StlpTerms;
StlpTerms* stlp_terms_new(const char* json);
void stlp_terms_free(StlpTerms* h);
int stlp_terms_set_stream(StlpTerms* h, uint64_t stream);
/* knots x (increasing), values y and slopes d of the monotone cubic (terms.rs:20-35) */
int stlp_terms_kappa_table(StlpTerms* h, const double* x, const double* y, const double* d, size_t n);
/* k = (f(x gs + gm) - km) / ks and its derivative dk, n values (terms.rs:37-58) */
int stlp_terms_kappa(StlpTerms* h, uint64_t x, size_t n, double gm, double gs, double km, double ks, uint64_t k,
                     uint64_t dk);
/* levels 1..depth of the 4-children pyramid of the rows x [rows][len] (terms.rs:78-102) */
int stlp_terms_pyramid(StlpTerms* h, uint64_t x);
/* out [rows][depth][2] = (sum d^2, sum d^4) of the details of every level (terms.rs:117-138) */
int stlp_terms_moments(StlpTerms* h, uint64_t x, double* out);
/* g [rows][len] += sum_{n < L} coef[r L + n] d_n (host coef [rows][L]) (terms.rs:148-163) */
int stlp_terms_level_power_grad(StlpTerms* h, uint64_t x, const double* coef, size_t L, uint64_t g);
/* g += (dk) sum_k cf0 (d^3 - c - cf1 cf2 d) over the levels (host levels [T], cf [rows][T][3];
 * dk 0: none) (terms.rs:165-184) */
int stlp_terms_kurtosis_grad(StlpTerms* h, uint64_t x, const int* levels, size_t T, const double* cf, uint64_t dk,
                             uint64_t g);
/* perm (u32) = positions of the n values x in increasing f64 total order, ties in position
 * order (terms.rs:187-258) */
int stlp_terms_sort(StlpTerms* h, uint64_t x, size_t n, uint64_t perm);
/* g[perm[q]] += coef (x[perm[q]] - t[q]) and *sum_sq = sum of the squares (terms.rs:260-269) */
int stlp_terms_marginal(StlpTerms* h, uint64_t x, uint64_t perm, uint64_t t_sorted, size_t n, double coef,
                        uint64_t g, double* sum_sq);
/* g += a b (b 0: g += a), n values (terms.rs:271-275) */
int stlp_terms_add_product(StlpTerms* h, uint64_t g, uint64_t a, uint64_t b, size_t n);

/* Spin 2: the (Q, U) of `level` (means of the children turned into the
 * parents' frames) and its (chi_E, chi_B), each [batch, 2, 12 (nside /
 * 2^level)^2], of the maps x [batch, 2, 12 nside^2]; level 0 only with the
 * scalar pyramid; not for cross handles.  (lib.rs:625-643) */
int stlp_spin_fields(StlpHandle* h, const double* x, size_t n, size_t level, double* qu, double* chi);

/* Spin 2: the device-built operator rows of `level` for exact checks:
 * kind 0 the stencil -(d_x - i d_y)^2 (cells and complex weights of every
 * pixel), kind 1 the transported means (the 4 children of every coarse
 * pixel of level + 1); cells [rows][width] (-1 past a row's end), weights
 * [rows][width][2]; *needed = the rows' width (cells / weights may be NULL
 * to ask for it).  No reference counterpart (the reference's operators are
 * host structures, crates/stl-core/src/spin.rs:88-157). */
int stlp_spin_rows(StlpHandle* h, size_t level, int kind, int64_t* cells, double* weights, size_t width,
                   size_t* needed);

/* Entry points of subsystems outside this engine (spectrum, U-Net
 * training).  They exist so that native.py's signature table binds; each
 * returns failure with stlp_last_error() naming the subsystem as not
 * built.  (lib.rs:1178-1492; unet.rs) */
void* stlp_spec_new(const char* config);
void stlp_spec_free(void* h);
char* stlp_spec_info(void* h);
int stlp_spec_set_masks(void* h, const double* w, size_t k);
int stlp_spec_forward(void* h, const double* x, size_t n, uint64_t g, uint64_t m, uint64_t o, double* out);
int stlp_spec_vjp(void* h, const double* cot, size_t n, uint64_t g, uint64_t m, uint64_t o, double* out);
void* stlp_unet_new(const char* config);
void stlp_unet_free(void* h);
char* stlp_unet_info(void* h);
int stlp_unet_get_params(void* h, float* out);
int stlp_unet_set_params(void* h, const float* p, size_t n);
int stlp_unet_get_grads(void* h, float* out);
int stlp_unet_zero_grad(void* h);
int stlp_unet_adam(void* h, double lr);
int stlp_unet_set_cond(void* h, const float* c, size_t n);
int stlp_unet_apply(void* h, const double* x, size_t n, double* a, double* b, double* c);
int stlp_train_set_masks(void* h, const double* w, size_t k);
int stlp_train_set_common(void* h, const double* w);
int stlp_train_set_field(void* h, uint32_t f, const double* a, const double* b, const double* c, const double* d,
                         const double* e, const double* g, size_t n, double s);
int stlp_train_bias(void* h, uint32_t f, const uint64_t* a, const double* b, size_t n);
int stlp_train_loss(void* h, uint32_t f, bool a, double* out);
int stlp_train_step(void* h, uint32_t f, double lr, double* out);
int stlp_train_live(void* h, uint32_t f, const uint64_t* a, const double* b, size_t n, const uint64_t* c,
                    const double* d, size_t m, bool e, double s, double* out);
void* stlp_train_lbfgs(void* h, const uint32_t* f, size_t n, const char* opts);
int stlp_train_set_joint(void* h, const double* a, const double* b, uint32_t c, uint32_t d, const char* e, double s);
int stlp_train_front(void* h, const double* x, size_t n, bool a, double* out);

#ifdef __cplusplus
}
#endif

#endif /* STL_B200_H */

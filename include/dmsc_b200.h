/*
 * dmsc_b200.h -- C ABI of the B200 (sm_100a) discrete Morse-Smale complex path.
 *
 * These entry points replace the reference's CUDA-side native entry
 *   dmsc_gpu.extract_dmsc(scalar_field, persistence_threshold, return_gradient,
 *                         is_dual, trace_max_arcs, trace_min_arcs,
 *                         trace_max_groups, trace_min_groups)
 * (dmsc/csrc/dmsc_gpu.cpp:128-180, bound at dmsc/csrc/dmsc_gpu.cpp:249-253),
 * which returns the 19-field DMSComplex (dmsc/csrc/dmsc_struct.hxx:5-30).
 * Every pointer below is a device pointer unless stated otherwise; the stream
 * argument is a cudaStream_t passed as void*.
 *
 * A call is two phases because most output sizes depend on the data:
 *   1. dmsc_b200_extract() runs the whole pipeline on the device, writes the
 *      fixed-size outputs (grad_indices, peaks, basins) into caller buffers and
 *      returns every variable output size (one device->host read of sizes);
 *   2. dmsc_b200_fetch() writes the variable-size outputs into caller buffers
 *      sized from phase 1.
 * A context keeps the device workspace between the two phases and across
 * calls; a context is not thread-safe, use one per host thread.
 */
#ifndef DMSC_B200_H
#define DMSC_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Return codes. */
#define DMSC_B200_OK 0
#define DMSC_B200_ERR_INVALID_ARGUMENT 1 /* bad pointer, size or flag */
#define DMSC_B200_ERR_TOO_LARGE 2        /* 4*(H+1)*(W+1) exceeds int32 cell ids (input_validation.hxx:24-26) */
#define DMSC_B200_ERR_CUDA 3             /* a CUDA runtime call failed */
#define DMSC_B200_ERR_ITERATION_CAP 4    /* a bounded device loop hit its cap */
#define DMSC_B200_ERR_OVERFLOW 5         /* an output exceeds int32 offsets or a work queue */
#define DMSC_B200_ERR_INTERNAL 6

/* Flags (the reference keyword arguments, dmsc/dmsc.py:230-239, 262-271). */
#define DMSC_B200_DUAL 1u           /* is_dual */
#define DMSC_B200_RETURN_GRADIENT 2u /* return_gradient */
#define DMSC_B200_TRACE_RIDGES 4u   /* trace_ridges  (native trace_max_arcs) */
#define DMSC_B200_TRACE_VALLEYS 8u  /* trace_valleys (native trace_min_arcs) */
#define DMSC_B200_TRACE_PEAKS 16u   /* trace_peaks   (native trace_max_groups) */
#define DMSC_B200_TRACE_BASINS 32u  /* trace_basins  (native trace_min_groups) */

typedef struct dmsc_b200_context dmsc_b200_context;

/* Element counts of the 19 outputs of one image (DMSComplex field order).
   2-D outputs give rows and columns. A field that was not requested has
   count 0 (the reference returns an empty tensor for it). */
typedef struct {
  int64_t max_pts, min_pts, sad_pts;
  int64_t e_max_rows, e_min_rows; /* e_max / e_min are [rows, 2] int32 */
  int64_t p_max, p_min, ppairs_max, ppairs_min;
  int64_t grad_indices;
  int64_t peaks_h, peaks_w;
  int64_t ridges, ridge_offsets, ridge_arc_offsets;
  int64_t basins_h, basins_w;
  int64_t valleys, valley_offsets, valley_arc_offsets;
} dmsc_b200_sizes;

/* Variable-size outputs of phase 2 (device pointers; NULL when the size is 0).
   int32 everywhere except p_max / p_min (float32). */
typedef struct {
  int32_t* max_pts;
  int32_t* min_pts;
  int32_t* sad_pts;
  int32_t* e_max;
  int32_t* e_min;
  float* p_max;
  float* p_min;
  int32_t* ppairs_max;
  int32_t* ppairs_min;
  int32_t* ridges;
  int32_t* ridge_offsets;
  int32_t* ridge_arc_offsets;
  int32_t* valleys;
  int32_t* valley_offsets;
  int32_t* valley_arc_offsets;
} dmsc_b200_outputs;

/* Creates a context bound to CUDA device `device`. Replaces the per-call
   gpu::Workspace of the reference (dmsc/csrc/dmsc_gpu.cpp:141-148). */
int dmsc_b200_create(dmsc_b200_context** ctx, int device);

/* Frees the context and its device workspace. */
void dmsc_b200_destroy(dmsc_b200_context* ctx);

/* Phase 1 for one H x W float32 image in device memory (row-major,
   contiguous). Replaces extract_single_dmsc_gpu_t up to output assembly
   (dmsc/csrc/dmsc_gpu.cpp:53-82) and the size part of gpu::Workspace::complex
   (dmsc/csrc/gpu/workspace.hxx:91-397).
   `grad_out`   : int32[4*(H+1)*(W+1)], 16-byte aligned, when DMSC_B200_RETURN_GRADIENT,
                  else NULL.
   `peaks_out`  : int32[(H+1)*(W+1)] in the primal, int32[H*W] in the dual,
                  when DMSC_B200_TRACE_PEAKS, else NULL.
   `basins_out` : int32[H*W] in the primal, int32[(H+1)*(W+1)] in the dual,
                  when DMSC_B200_TRACE_BASINS, else NULL.
   `persistence_threshold` is compared as float32, as the reference's C++
   `float` parameter is. Writes `sizes` (host pointer). */
int dmsc_b200_extract(dmsc_b200_context* ctx, const float* image, int H, int W, float persistence_threshold,
                      unsigned flags, int32_t* grad_out, int32_t* peaks_out, int32_t* basins_out,
                      dmsc_b200_sizes* sizes, void* stream);

/* Phase 2: writes the variable-size outputs of the last extract() or
   extract_batch() on this context. `out` is a host pointer to a struct of
   device pointers. After extract_batch(), every array holds the images'
   parts back to back in image order, each part sized by that image's sizes
   entry (offset arrays too: ridge_offsets holds ridge_offsets[b] + 1 entries
   of image b, and so on); all values are image-local. */
int dmsc_b200_fetch(dmsc_b200_context* ctx, const dmsc_b200_outputs* out, void* stream);

/* Optional host destinations for the fixed-size outputs of the next
   extract() / extract_batch() on this context (no counterpart in the
   reference, whose CPU callers get host tensors only after the whole call).
   Pinned host buffers laid out like grad_out / peaks_out / basins_out (any
   may be NULL). Each output is copied on an internal stream as soon as it
   is produced (the gradient right after the first kernel, the labels after
   the label stage), overlapping the transfer with the rest of the pipeline.
   The caller's stream waits for these copies at the end of the following
   dmsc_b200_fetch(): read the host buffers only after that fetch's work on
   the stream has completed. The registration covers one extract call. */
int dmsc_b200_set_host_outputs(dmsc_b200_context* ctx, int32_t* grad_host, int32_t* peaks_host,
                               int32_t* basins_host);

/* The same for the variable-size outputs of the next dmsc_b200_fetch():
   `host` (host pointer) holds pinned host buffers laid out like that fetch's
   device outputs (NULL fields are skipped). The lists and per-saddle outputs
   are copied as soon as they are written, while the arc geometry is built;
   the geometry when it is done. They are complete once the caller's stream
   has passed that fetch. The registration covers one fetch call. */
int dmsc_b200_set_host_fetch_outputs(dmsc_b200_context* ctx, const dmsc_b200_outputs* host);

/* Optional host source of the image of the next dmsc_b200_extract() on this
   context (no counterpart in the reference, whose CUDA path takes a device
   tensor): `host_image` is a pinned host buffer of H x W float32 values. The
   extract copies it into its `image` argument, which is then a device
   buffer of H x W floats that the call only writes, in bands of rows on an
   internal stream, and starts each band's gradient tiles (and, with
   dmsc_b200_set_host_outputs, the copy of their gradient back to the host)
   as soon as the rows they read have arrived, so the upload overlaps the
   downloads. `host_image` must stay unchanged until the caller's stream has
   passed the extract. NULL clears it; the registration covers one extract
   call and is not allowed before dmsc_b200_extract_batch (returns
   DMSC_B200_ERR_INVALID_ARGUMENT there). */
int dmsc_b200_set_host_input(dmsc_b200_context* ctx, const float* host_image);

/* Phase 1 for a batch of B images of independent sizes, thresholds and
   orientations, computed together (one pass of every stage over the union
   of the images). Replaces the reference's per-image loop over a 3-D batch
   (dmsc/csrc/dmsc_gpu.cpp:84-126, dmsc/csrc/dmsc_cpu.cpp:80-106), which only
   takes images of one size and one threshold; each image's outputs are
   exactly those of dmsc_b200_extract() on it alone.
   `images`     : device float32, the images back to back, image b H[b] x W[b]
                  row-major, starting at element sum_{c<b} H[c]*W[c].
   `H`, `W`, `thresholds`, `is_dual` : host arrays of B entries (is_dual 0/1);
                  DMSC_B200_DUAL in `flags` is ignored, the other flags apply
                  to every image.
   `grad_out`, `peaks_out`, `basins_out` : the per-image arrays of
                  dmsc_b200_extract() back to back in image order.
   `sizes`      : host array of B entries, written per image.
   The cell ids of the whole batch must fit int32 (sum over images of
   4*(H+1)*(W+1)), else DMSC_B200_ERR_TOO_LARGE: split the batch. */
int dmsc_b200_extract_batch(dmsc_b200_context* ctx, const float* images, int B, const int* H, const int* W,
                            const float* thresholds, const unsigned char* is_dual, unsigned flags,
                            int32_t* grad_out, int32_t* peaks_out, int32_t* basins_out, dmsc_b200_sizes* sizes,
                            void* stream);

/* Differentiation support (no counterpart in the reference, whose outputs
   carry no gradient). A persistence value p (p_max / p_min, computed as the
   float32 difference of two input pixels, dmsc/csrc/cpu/persistence.hxx:82-104,
   139-161) has d p / d image = +1 at one pixel and -1 at another on a field
   without ties.
   dmsc_b200_fetch_pair_pixels() writes, for the last extract() or
   extract_batch() on this context, those two image-local pixel ids
   (y * W + x) of every entry of p_max and p_min: `plus_*` and `minus_*` are
   device int32 arrays laid out exactly like p_max / p_min (per image, back
   to back for a batch); -1 in both for a cycle (persistence -1, constant).
   Any pointer may be NULL. It reads the input image again: the image passed
   to extract must be unchanged. */
int dmsc_b200_fetch_pair_pixels(dmsc_b200_context* ctx, int32_t* plus_max, int32_t* minus_max, int32_t* plus_min,
                                int32_t* minus_min, void* stream);

/* Backward scatter: grad_img[0 .. npx) = 0, then for every i < n,
   grad_img[plus[i]] += grad[i] and grad_img[minus[i]] -= grad[i] (ends
   outside [0, npx), such as -1, are skipped). Deterministic: the terms of
   each pixel are summed in ascending order of i, + end before - end, by a
   stable sort and a segmented sum; no float atomics. Device pointers; `plus`
   and `minus` are pixel ids in the caller's flat pixel array. */
int dmsc_b200_scatter_pair_grads(dmsc_b200_context* ctx, const int32_t* plus, const int32_t* minus,
                                 const float* grad, int64_t n, float* grad_img, int64_t npx, void* stream);

/* Static description of a return code. */
const char* dmsc_b200_error_string(int code);

/* Message of the last failure on this context (empty when none). */
const char* dmsc_b200_last_error(const dmsc_b200_context* ctx);

/* Instrumentation (no reference counterpart; the reference exposes its stage
   timings only as RECORD_FUNCTION ranges, e.g. cpu/gradient.hxx:24).
   When enabled, extract() and fetch() record a CUDA event on the call's stream
   at every stage boundary. dmsc_b200_stage_times() writes up to `n` stage
   durations in milliseconds of the last extract()+fetch() pair (host pointer)
   and returns the number of stages: 0 set-up (workspace clears, table
   upload), 1 gradient (the kernel alone), 2 compaction, 3 saddle walks,
   4 pairing (both sides), 5 persistence, cancellation and output ranks,
   6 survivors (flags and counts), 7 replay (both sides), 8 final arcs, 9 label
   set-up (per-extremum labels, bases), 10 labels (the label kernels alone),
   11 sizes, 12 fetch lists, 13 geometry (the chain expansion, which runs at
   the end of extract() while the caller allocates the outputs, plus the
   writer in fetch()). The survivors' sweep order
   and records are computed on a second stream while the replay and the
   labels run (the labels run before the final arcs); the final-arcs stage
   includes the wait for them. */
int dmsc_b200_set_profiling(dmsc_b200_context* ctx, int enable);
int dmsc_b200_stage_times(dmsc_b200_context* ctx, float* ms, int n);

/* Kernel launches issued by the last extract()+fetch() pair (each CUB scan or
   sort call counts once). */
long long dmsc_b200_launch_count(const dmsc_b200_context* ctx);

/* Device loop counts of the last call (host pointer, up to `n` values):
   pairing rounds (faces, vertices), replay rounds (faces, vertices), geometry
   expansion levels (faces, vertices). Returns the number written or -1. */
int dmsc_b200_loop_counts(dmsc_b200_context* ctx, int* out, int n);

/* Device loop timelines of the last call (ns, device global timer), six
   blocks of 64 slots: pairing round starts (faces, vertices), geometry
   expansion level starts (faces, vertices), then replay round starts (faces,
   vertices); then six more blocks in the same order with each round's item
   count (active saddles, queued chain tasks, pending cancellations); then
   the pairing's phase-B start times (faces, vertices). Unused slots are 0.
   Writes up to `n` (at most 896) values to `out` (host pointer), returns the
   number written. */
int dmsc_b200_pairing_timeline(dmsc_b200_context* ctx, long long* out, int n);

/* Failure handling (no counterpart in the reference). Every device loop of
   the pipeline has a bound that no input reaches: pairing rounds (extrema of
   a side + 2), replay rounds (saddles + 2), geometry expansion levels
   (saddles + 4), union-find searches and retries (extrema + 2), V-path walks
   (cells) and chain walks (saddles + 1). A loop that reaches its bound stops,
   leaves the device state consistent (undecided saddles become cycles,
   pending cancellations are dropped), sets a bit of a device status word,
   and the call returns DMSC_B200_ERR_ITERATION_CAP at its next readback;
   nothing traps. dmsc_b200_set_loop_caps() lowers the pairing-round,
   replay-round and expansion-level bounds of the following calls to the given
   values (0 = the normal bound) so that tests can make them run out; the
   context stays usable after such an error. */
int dmsc_b200_set_loop_caps(dmsc_b200_context* ctx, int pair_rounds, int replay_rounds, int emit_levels);

/* Launch shapes (no counterpart in the reference, whose CPU path fixes its
   blocking at compile time, cpu/gradient.hxx:15 DEFAULT_GRADIENT_BLOCK_SIZE
   and cpu/cell_groups.hxx:9 CACHE_DEPTH). They change speed only, never an
   output bit. The Python tuner (dmsc_b200.tuning) sweeps them on the
   caller's data and sets the fastest per image-size class.
   grad_shape   : gradient tile of 32 index columns x {31, 63, 127, 63, 127}
                  rows (threads {256, 256, 512, 256, 512}), 0..4; shapes 3
                  and 4 stage the value windows with tensor-memory copies in a
                  persistent kernel (one image whose width is a multiple of 4
                  in a 16-byte aligned buffer; others run shapes 1 and 2);
                  default 3.
   label_shape  : 64 x 64 label tiles with {1024, 512} threads, 0..1; default 1.
   *_blocks_per_sm : resident blocks per SM of the pairing, replay and
                  geometry-expansion persistent kernels; 0 = as many as fit
                  (the default); larger values are clamped to what fits.
   seg_cursors  : raw-arc walks each lane of the segment writer drives at
                  once, 1..2; default 1.
   pair_shape   : pairing items each thread advances together, {2, 4}
                  (with {5, 4} resident blocks per SM), 0..1; default 0.
   replay_shape : replay cancellations each thread advances together, {1, 2}
                  (with {4, 3} resident blocks per SM), 0..1; default 0.
   emit_shape   : geometry-expansion chain tasks each thread advances
                  together, {1, 2} (with {5, 3} resident blocks per SM),
                  0..1; default 0. */
typedef struct {
  int grad_shape;
  int label_shape;
  int pair_blocks_per_sm;
  int replay_blocks_per_sm;
  int emit_blocks_per_sm;
  int seg_cursors;
  int pair_shape;
  int replay_shape;
  int emit_shape;
} dmsc_b200_tuning;

int dmsc_b200_set_tuning(dmsc_b200_context* ctx, const dmsc_b200_tuning* tuning);
int dmsc_b200_get_tuning(const dmsc_b200_context* ctx, dmsc_b200_tuning* tuning);

/* Choices of the tunables on this context's device (host pointer, up to `n`
   values): number of gradient tile shapes, number of label tile shapes, the
   most blocks per SM of the pairing and replay (in their current shapes)
   and expansion kernels, the most segment-writer cursors per lane, and the
   numbers of pairing, replay and expansion shapes. Returns the number
   written or -1. */
int dmsc_b200_tuning_limits(dmsc_b200_context* ctx, int* out, int n);

/* Host waits inside a call poll an event; after `seconds` (default 600) they
   give up with DMSC_B200_ERR_CUDA. Work may still be running on the device
   then: destroy the context instead of reusing it. */
int dmsc_b200_set_wait_timeout(dmsc_b200_context* ctx, double seconds);

/* No counterpart in the reference. For callers that cannot allocate device
   memory at call time -- code running while a stream is captured into a CUDA
   graph, fixed-memory real-time hosts, or plugins whose framework hands out
   only input and output buffers -- this computes the discrete gradient
   (grad_indices) and the ascending lists of critical vertices, edges and
   faces of one H x W image without allocating. In the primal the critical
   vertices are the minima and the critical faces the maxima; with
   DMSC_B200_DUAL the roles swap (vertices are the maxima, faces the minima),
   as in the reference's dual outputs. Its scratch is a fixed 8 MiB static
   device array of the library: 2 bytes per index (H+1)*(W+1) plus 24 bytes
   per 32-index row segment, each of its 8 parts rounded up to 256 bytes --
   about 2.75 bytes per index, so square images up to 1743 x 1743 fit
   (1744 x 1744 does not). Larger images return DMSC_B200_ERR_TOO_LARGE
   before any buffer is touched.
   `grad_out`    : int32[4*(H+1)*(W+1)], 16-byte aligned.
   `mins_out`    : critical vertices, int32[H*W] capacity;
   `saddles_out` : critical edges, int32[H*(W+1)+(H+1)*W];
   `maxes_out`   : critical faces, int32[(H+1)*(W+1)];
   `counts_out`  : int32[3] = (#vertices, #edges, #faces). All device
                   pointers; only DMSC_B200_DUAL is read from `flags`.
   The first call on a device looks up the static array's device address,
   uploads a table and waits for the device to finish (so any stream may make
   it); make it before any stream capture. Every call shares the one scratch
   array (which keeps the last call's contents), so calls that overlap on the
   GPU race: serialise them. */
int dmsc_b200_critical_cells_static(const float* image, int H, int W, unsigned flags, int32_t* grad_out,
                                    int32_t* mins_out, int32_t* saddles_out, int32_t* maxes_out,
                                    int32_t* counts_out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DMSC_B200_H */

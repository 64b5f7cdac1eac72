/*
 * cusmic_b200 extensions to the reference C ABI (cusmic.h).
 *
 * The reference batch call (src/cusmic.h:80-85) accepts only same-shaped
 * frames with batch-wide scalar calibration, allocates scratch on every call
 * and synchronises the host once per iteration (src/cleaner.cuh:128-142).
 * These entry points add what a B200 deployment needs on top of it:
 *
 *   - ragged batches with per-frame scalar gain / read noise / background,
 *     run as one persistent launch over a tile work list;
 *   - plans: a workspace, tile list and captured CUDA graph of the whole
 *     maxiter loop (with its early exit as a device-side while node), reused
 *     across executions;
 *   - the adjoint of the cleaned pixels with the detection mask frozen.
 *
 * All pointers of a call belong to the caller's current device.  Status codes
 * and message conventions are those of cusmic.h.
 */
#ifndef CUSMIC_B200_H
#define CUSMIC_B200_H

#include "cusmic.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Per-frame scalar calibration of a ragged batch.  A NaN gain or read noise
 * falls back to the options' value; a NaN background means none for that
 * frame.  Maps in the frame's cusmic_image still override these scalars.
 * No counterpart in the reference, whose scalars are batch-wide
 * (src/cusmic.h:45-51). */
struct cusmic_frame_scalars {
	double gain, readnoise, background;
};

/* Ragged batch of 1..65535 device frames of any shapes.  Frame f's outputs
 * start at offset sum_{g<f} width_g * height_g of clean and mask.  scalars
 * may be NULL.  Synchronises before returning, like remove_cosmics_device.
 * Generalises remove_cosmics_batch_device (reference src/api.cu:184-192). */
int
cusmic_ragged_batch_device(const struct cusmic_image *ims, size_t nf,
	const struct cusmic_options *options, const struct cusmic_frame_scalars *scalars,
	double *clean, uint8_t *mask, void *stream, char *msg, size_t message_size);

/* Ragged batch of 1..65535 frames in HOST memory, results into host memory
 * (frame f's outputs at offset sum_{g<f} width_g * height_g of clean and
 * mask).  Frames are cleaned on the current device in chunks of whole frames;
 * the inbound copies of later chunks run while earlier chunks are cleaned
 * (every chunk's inputs are queued at once when they fit a quarter of the
 * free device memory).  A map pointer that several frames share is uploaded
 * and checked once.  A chunk whose frames have no background returns only its
 * flagged pixels (16 bytes each): the other output pixels equal the inputs bit
 * for bit, and host threads copy them.  Map contents are checked like
 * remove_cosmics's (same messages).  Page-locked buffers are copied by DMA
 * directly; pageable ones through pinned staging (correct, with less overlap).
 * On failure, frames of the chunks before the failing one hold their results
 * and the other outputs are unspecified.  Returns after the last result has
 * landed.  No counterpart in the reference, whose host entry point takes one
 * frame (src/api.cu:155-175); this is that call for a batch, with
 * remove_cosmics's status and message rules. */
int
cusmic_batch_host(const struct cusmic_image *ims, size_t nf, const struct cusmic_options *options,
	const struct cusmic_frame_scalars *scalars, double *clean, uint8_t *mask, char *msg,
	size_t message_size);

typedef struct cusmic_plan cusmic_plan;

/* Plan flags. */
enum cusmic_plan_flags {
	CUSMIC_PLAN_GRAPH = 1, /* capture the maxiter loop into one CUDA graph */
	CUSMIC_PLAN_KEEP = 2   /* reserved: plans always keep their last mask for the adjoint */
};

/* Create a plan for a fixed batch (shapes, maps present or absent, options)
 * bound to the given device buffers.  Allocates the workspace once.  No
 * counterpart in the reference (its scratch is per call, src/cleaner.cuh:39-61). */
int
cusmic_plan_create(cusmic_plan **plan, const struct cusmic_image *ims, size_t nf,
	const struct cusmic_options *options, const struct cusmic_frame_scalars *scalars,
	double *clean, uint8_t *mask, int flags, char *msg, size_t message_size);

/* Rebind the plan to new device buffers of the same shapes and map layout
 * (pointers only; the next execution reads the new descriptors). */
int
cusmic_plan_bind(cusmic_plan *plan, const struct cusmic_image *ims, double *clean,
	uint8_t *mask, char *msg, size_t message_size);

/* Enqueue one cleaning of the bound batch on stream; does not synchronise. */
int
cusmic_plan_execute(cusmic_plan *plan, void *stream, char *msg, size_t message_size);

/* Wait for the plan's last execution and report its status ("no finite
 * replacement donors" is CUSMIC_INVALID, as in the reference). */
int
cusmic_plan_wait(cusmic_plan *plan, char *msg, size_t message_size);

/* Detection passes run per frame by the last execution (nf ints, host). */
int
cusmic_plan_passes(cusmic_plan *plan, int *passes);

/* Execute the plan once without its graph, with a CUDA event recorded on
 * stream after every kernel, then synchronise.  ms[k] and launches[k] receive
 * the summed duration and launch count of kernel kind k for k in 0..15:
 * init (with the zeroing of the bit planes), prepare, hole fill, sig_raw
 * (dense detection), candidates (5 x 5 medians), seeds (fine structure),
 * grow/update, control, replace, restore, zero-iteration copy, low
 * candidates, classification of the dense pass's list, block floors, and of
 * the incremental passes the reclassification with work-list gather and the
 * dirty-row scan.  A batch whose frames all have an error map and no
 * background, widths that are multiples of 16 and 16-byte aligned buffers
 * runs prepare and the first pass's dense detection as one kernel, reported
 * under prepare (no sig_raw launch).  A timing aid; no counterpart in the
 * reference. */
int
cusmic_plan_profile(cusmic_plan *plan, void *stream, double *ms, int *launches, int kinds,
	char *msg, size_t message_size);

/* Adjoint of the last execution with its detection mask frozen: given
 * grad_clean = dL/d(clean) (device, laid out like the outputs) writes
 * grad_data = dL/d(data), and, when not NULL, grad_background = dL/d(background):
 * one value per frame when no frame has a background map (zero for frames
 * without background), else a per-pixel map laid out like the outputs.  Each
 * replaced pixel sends its gradient to the donor its replacement median
 * selected (half to each of the two central donors for an even donor count;
 * donors ordered by value, ties by lowest linear index); unflagged and
 * non-finite pixels pass it straight through.  The selection is recomputed
 * from the plan's kept mask, not stored.  Runs on stream; synchronises.
 * No counterpart in the reference. */
int
cusmic_plan_backward(cusmic_plan *plan, const double *grad_clean, double *grad_data,
	double *grad_background, void *stream, char *msg, size_t message_size);

void
cusmic_plan_destroy(cusmic_plan *plan);

/* Launch parameters of the detection pass, chosen per batch size by the
 * project's autotuner (cusmic_b200/autotune.py; results in
 * cusmic_b200/tuning.json).  An entry applies to batches of at most
 * max_pixels pixels; the first matching entry of the table wins. */
struct cusmic_tuning {
	size_t max_pixels;
	int dense_rows;           /* rows per item of the dense detection kernel: 4, 8, 16
	                             or 32; 0 = automatic (shrink from 32 while the batch
	                             has fewer items than the kernel has resident blocks) */
	int dense_blocks_per_sm;  /* dense detection blocks launched per SM: 1..6 */
	int sparse_blocks_per_sm; /* 256-thread blocks per SM of the candidate, seed,
	                             low-candidate, classification and replacement
	                             kernels: 1..8 */
	int row_blocks_per_sm;    /* 256-thread blocks per SM of the row kernels (prepare,
	                             hole fill, growth, restore): 1..8 */
};

/* Replace the process-wide tuning table (n entries, copied; n = 0 restores the
 * built-in defaults).  Plans keep the parameters they were created with.
 * CUSMIC_INVALID for out-of-range fields.  No counterpart in the reference. */
int
cusmic_set_tuning(const struct cusmic_tuning *table, size_t n, char *msg, size_t message_size);

/* The entry that applies to a batch of total_pixels pixels.  No counterpart in
 * the reference. */
int
cusmic_get_tuning(size_t total_pixels, struct cusmic_tuning *out);

/* remove_cosmics_device for callers that cannot allocate device memory when
 * they clean a frame: real-time acquisition loops that allow allocation only
 * at start-up (cudaMalloc can block for milliseconds and cudaFree synchronises
 * the whole device), and processes whose own caching allocator has already
 * reserved the GPU's memory, so that a cudaMalloc of this library's scratch
 * would fail.  Same arguments and results as remove_cosmics_device, for one
 * frame of at most 262144 pixels and 16384 rows (larger frames are rejected
 * with CUSMIC_INVALID).  All scratch lives in a 12 MiB static device array
 * that every GPU loading this library holds until the process exits; the call
 * allocates nothing.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress), so make that first call before any stream
 * capture.  Calls share the array, which keeps the last call's contents:
 * calls whose work overlaps on the GPU race, so serialise them (one stream,
 * or the caller's own ordering).  Synchronises before returning.  No
 * counterpart in the reference. */
int
remove_cosmics_device_noalloc(const struct cusmic_image *image, const struct cusmic_options *options,
	double *clean, uint8_t *mask, void *stream, char *msg, size_t message_size);

/* Failures injected for tests of the error paths; none is in force unless a
 * caller sets it.  No counterpart in the reference, whose tests inject none.
 *
 *   CUSMIC_FAULT_PREPARE_WAIT, CUSMIC_FAULT_DETECT_WAIT: value > 0 makes one
 *     warp of the bulk-staged prepare kernel, or of the dense detection
 *     kernel, wait up to `value` SM cycles on a barrier that nothing
 *     completes, in calls (and plans) laid out after this call.  The wait
 *     runs out like a wait whose copies never land: the kernel drains its
 *     copies in flight, the loop control stops every frame and the call
 *     returns CUSMIC_CUDA_ERROR.  value <= 0 removes the injection.
 *   CUSMIC_FAULT_NO_MEMORY: the next `value` workspace reservations fail as
 *     an exhausted cudaMalloc would (CUSMIC_NO_MEMORY; the host entry point
 *     leaves its outputs unchanged).
 *
 * Returns CUSMIC_INVALID for an unknown kind. */
enum cusmic_fault {
	CUSMIC_FAULT_PREPARE_WAIT = 1,
	CUSMIC_FAULT_DETECT_WAIT = 2,
	CUSMIC_FAULT_NO_MEMORY = 3
};

int
cusmic_inject_fault(int what, long long value);

#ifdef __cplusplus
}
#endif
#endif

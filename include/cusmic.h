/*
 * cusmic_b200 — drop-in C ABI of the rndsrc/cusmic L.A.Cosmic cleaner.
 *
 * Every declaration here mirrors the reference interface src/cusmic.h of
 * rndsrc/cusmic (same names, struct layouts, enum values, argument meaning,
 * status codes and error behaviour), so a program or FFI binding written
 * against the reference links against libcusmic_b200.so unchanged.  The
 * B200-specific extensions live in cusmic_b200.h.
 */
#ifndef CUSMIC_H
#define CUSMIC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Border modes follow scipy.ndimage (reference src/cusmic.h:26). */
enum cusmic_border { CUSMIC_REFLECT, CUSMIC_CONSTANT, CUSMIC_NEAREST, CUSMIC_MIRROR, CUSMIC_WRAP };
/* Status codes (reference src/cusmic.h:27). */
enum cusmic_status { CUSMIC_OK, CUSMIC_INVALID, CUSMIC_CUDA_ERROR, CUSMIC_NO_MEMORY };

/* One frame: contiguous row-major float64 pixels and optional maps of
 * width * height elements (reference src/cusmic.h:29-43).  An error map (1-sigma,
 * image units) overrides gain (electrons per image unit) and read noise
 * (electrons).  Background is added before cleaning and subtracted afterwards.
 * Mask bytes exclude seeds and donors; detections may still grow into masked
 * pixels.  Non-finite input pixels are returned unchanged and never flagged. */
struct cusmic_image {
	const double *data, *error;
	const double *gain;
	const double *readnoise, *background;
	const uint8_t *mask;
	size_t width, height;
};

/* Detection settings (reference src/cusmic.h:45-51).  NaN gain means unset;
 * NaN background means none.  maxiter 0 disables detection but keeps the
 * background arithmetic. */
struct cusmic_options {
	double contrast, cr_threshold, neighbor_threshold;
	double gain;
	double readnoise, background;
	int maxiter;
	int border;
};

/* Library version string (reference src/cusmic.h:53-54, src/api.cu:28-32). */
const char *
cusmic_version(void);

/* CUDA runtime version the library was built with (reference src/cusmic.h:56-57). */
int
cusmic_cuda_version(void);

/* Defaults {contrast 3, cr 5, neighbor 3, gain NaN, readnoise 0, background NaN,
 * maxiter 4, MIRROR} (reference src/cusmic.h:59-63, src/api.cu:40-45). */
void
cusmic_default_options(struct cusmic_options *options);

/* Host arrays in, host arrays out (reference src/cusmic.h:65-70,
 * src/api.cu:155-175).  Map contents are validated on the host; outputs must
 * not overlap inputs or each other; failures leave outputs unchanged; msg is
 * NUL-terminated when message_size > 0. */
int
remove_cosmics(const struct cusmic_image *image, const struct cusmic_options *options,
	double *clean, uint8_t *mask, char *msg, size_t message_size);

/* Device arrays on the caller's current GPU and stream (cudaStream_t cast to
 * void*, NULL allowed); returns after the work completes; the caller validates
 * map contents; outputs are unspecified on failure (reference src/cusmic.h:72-78,
 * src/api.cu:177-182). */
int
remove_cosmics_device(const struct cusmic_image *image, const struct cusmic_options *options,
	double *clean, uint8_t *mask, void *stream, char *msg, size_t message_size);

/* 1..65535 same-sized device frames; calibration pointers may be shared;
 * outputs are contiguous in descriptor order (reference src/cusmic.h:80-85,
 * src/api.cu:184-192). */
int
remove_cosmics_batch_device(const struct cusmic_image *ims, size_t nf,
	const struct cusmic_options *options, double *clean, uint8_t *mask, void *stream, char *msg,
	size_t message_size);

#ifdef __cplusplus
}
#endif
#endif

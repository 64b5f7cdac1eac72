/*
 * CPU oracle for the L.A.Cosmic detect/replace path of rndsrc/cusmic.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, operation by operation and
 * in plain C, what the reference CUDA library computes, so that the CUDA
 * kernels of cusmic_b200 can be checked bit for bit.  Only tests/, the smoke
 * check and the CPU-baseline leg of bench.py may load it.  The product never
 * links it and never falls back to it.
 *
 * Parity is pinned by the reference's own golden fixture
 * (test/data/{input,error,reference}.fits.gz, lacosmic 1.4.0 output, stored
 * as tests/golden/fixture_512.npz) and, on a GPU, by the reference library
 * itself compiled from src/api.cu (see oracle/build.py).
 *
 * Every function cites the reference file:line it follows (paths relative to
 * the reference project root).  Arithmetic must be compiled with
 * -ffp-contract=off, exactly like the reference (Makefile:92-105).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum { O_REFLECT, O_CONSTANT, O_NEAREST, O_MIRROR, O_WRAP };

/* Same field layout as struct cusmic_image (src/cusmic.h:37-43). */
typedef struct {
	const double *data, *error, *gain, *readnoise, *background;
	const uint8_t *mask;
	size_t width, height;
} oracle_image;

/* Detection settings; gain/readnoise/background are this frame's scalars. */
typedef struct {
	double contrast, cr_threshold, neighbor_threshold;
	double gain, readnoise, background;
	int maxiter, border;
} oracle_options;

static const double FINE_FLOOR = 0.01;   /* src/filters.cuh:21 */
static const double SIGNAL_FLOOR = 1e-5; /* src/filters.cuh:22 */

/* src/filters.cuh:24-44 (scipy.ndimage border conventions). */
int
oracle_border_index(int x, int n, int mode)
{
	if (x >= 0 && x < n)
		return x;
	if (mode == O_CONSTANT)
		return -1;
	if (mode == O_NEAREST)
		return x < 0 ? 0 : n - 1;
	if (n == 1)
		return 0;
	int period = mode == O_REFLECT ? 2 * n : mode == O_MIRROR ? 2 * (n - 1) : n;
	x %= period;
	if (x < 0)
		x += period;
	if (mode == O_REFLECT && x >= n)
		return period - x - 1;
	if (mode == O_MIRROR && x >= n)
		return period - x;
	return x;
}

/*
 * Literal odd-even transposition sort, src/sort.cuh:18-36: (n+1)/2 passes of
 * an even and an odd phase, exchanging a neighbour pair when b < a.  Kept for
 * the unit test that pins oracle_window_median() against it.
 */
void
oracle_oets(double *v, int n)
{
	for (int pass = 0; pass < (n + 1) / 2; ++pass)
		for (int start = 0; start < 2; ++start)
			for (int i = start; i + 1 < n; i += 2) {
				double a = v[i], b = v[i + 1];
				int swap = b < a;
				v[i] = swap ? b : a;
				v[i + 1] = swap ? a : b;
			}
}

/*
 * Middle element after oracle_oets(v, n), computed faster.  The exchange never
 * moves a NaN (both comparisons with it are false), so NaNs stay in place and
 * split the window into segments that are sorted independently; n phases sort
 * any segment of at most n elements, and the exchange is stable.  Hence: a NaN
 * at the middle is returned as is; otherwise the segment around the middle is
 * stably sorted (insertion sort, strict <) and its middle slot read.
 */
double
oracle_window_median(double *v, int n)
{
	int mid = n / 2, a = mid, b = mid;
	if (isnan(v[mid]))
		return v[mid];
	while (a > 0 && !isnan(v[a - 1]))
		--a;
	while (b < n - 1 && !isnan(v[b + 1]))
		++b;
	for (int i = a + 1; i <= b; ++i) {
		double x = v[i];
		int j = i;
		while (j > a && x < v[j - 1]) {
			v[j] = v[j - 1];
			--j;
		}
		v[j] = x;
	}
	return v[mid];
}

/* src/filters.cuh:46-70: k x k median, row-major gather, constant pads 0. */
static void
median_filter(const double *a, double *out, int w, int h, int mode, int size)
{
	int r = size / 2;
#pragma omp parallel for schedule(static)
	for (int y = 0; y < h; ++y) {
		double values[49];
		int xs[7], ys[7];
		for (int k = 0; k < size; ++k)
			ys[k] = oracle_border_index(y + k - r, h, mode);
		for (int x = 0; x < w; ++x) {
			for (int k = 0; k < size; ++k)
				xs[k] = oracle_border_index(x + k - r, w, mode);
			for (int yy = 0; yy < size; ++yy)
				for (int xx = 0; xx < size; ++xx)
					values[yy * size + xx] = xs[xx] < 0 || ys[yy] < 0
						? 0 : a[(size_t)ys[yy] * w + xs[xx]];
			out[(size_t)y * w + x] = oracle_window_median(values, size * size);
		}
	}
}

static double
sample(const double *clean, int x, int y, int w, int h, int mode)
{
	x = oracle_border_index(x, w, mode);
	y = oracle_border_index(y, h, mode);
	return x < 0 || y < 0 ? 0 : clean[(size_t)y * w + x];
}

static double
positive(double v)
{
	return v < 0 ? 0 : v;
}

/* src/filters.cuh:86-105: collapsed 2x replicate, Laplacian, clip, 2x2 sum. */
static void
laplacian(const double *clean, double *lap, int w, int h, int mode)
{
	if (mode == O_MIRROR || mode == O_REFLECT)
		mode = O_NEAREST;
#pragma omp parallel for schedule(static)
	for (int y = 0; y < h; ++y)
		for (int x = 0; x < w; ++x) {
			size_t i = (size_t)y * w + x;
			double c = clean[i] / 4;
			double up = c - sample(clean, x, y - 1, w, h, mode) / 4;
			double down = c - sample(clean, x, y + 1, w, h, mode) / 4;
			double left = c - sample(clean, x - 1, y, w, h, mode) / 4;
			double right = c - sample(clean, x + 1, y, w, h, mode) / 4;
			lap[i] = (positive(up + left) + positive(up + right)) +
				(positive(down + left) + positive(down + right));
		}
}

/* src/replace.cuh:19-23 */
static int
is_donor(const double *clean, const uint8_t *crmask, const uint8_t *excluded, size_t i)
{
	return !crmask[i] && !excluded[i] && isfinite(clean[i]);
}

/* src/replace.cuh:37-48: IEEE bits mapped to an unsigned total order. */
static uint64_t
order_key(double v)
{
	uint64_t bits;
	memcpy(&bits, &v, sizeof(bits));
	return bits >> 63 ? ~bits : bits ^ (UINT64_C(1) << 63);
}

static double
order_value(uint64_t k)
{
	uint64_t bits = k >> 63 ? k ^ (UINT64_C(1) << 63) : ~k;
	double v;
	memcpy(&v, &bits, sizeof(v));
	return v;
}

/* src/replace.cuh:50-56 */
static double
midpoint(double lo, double hi)
{
	if (fabs(lo) < 1 && fabs(hi) < 1)
		return (lo + hi) / 2;
	return lo / 2 + hi / 2;
}

/*
 * src/replace.cuh:68-83: ascending bitonic network over 32 lanes, restated on
 * an array.  Lane l compares with lane l ^ step and keeps the smaller value
 * when its (span, step) bits agree, else the larger one.
 */
void
oracle_bitonic32(double v[32])
{
	for (int span = 2; span <= 32; span *= 2)
		for (int step = span / 2; step; step /= 2) {
			double next[32];
			for (int lane = 0; lane < 32; ++lane) {
				double a = v[lane], peer = v[lane ^ step];
				int lower = ((lane & span) == 0) == ((lane & step) == 0);
				next[lane] = lower ? (peer < a ? peer : a) : (a < peer ? peer : a);
			}
			memcpy(v, next, sizeof(next));
		}
}

static int
cmp_u64(const void *a, const void *b)
{
	uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
	return x < y ? -1 : x > y;
}

/*
 * src/replace.cuh:111-153: for every target, the median of the donors in a
 * clipped (2r+1)^2 window, r = 2, 3, ... until a donor exists.  Windows of at
 * most 32 cells use the 32-lane bitonic network (+inf padding, lane = cell in
 * row-major order); larger ones select by ordered key (src/replace.cuh:85-109
 * selects the same ranks bit by bit).  Odd counts give 0.0 + lo, even counts
 * midpoint(lo, hi).  Donors never change inside one call, so targets can be
 * processed in any order.
 */
static void
replace(double *clean, const uint8_t *crmask, const uint8_t *excluded, int w, int h)
{
	int limit = w > h ? w : h;
	size_t n = (size_t)w * h;
#pragma omp parallel
	{
		uint64_t *keys = NULL;
		size_t cap = 0;
#pragma omp for schedule(dynamic, 64)
		for (size_t i = 0; i < n; ++i) {
			if (!crmask[i])
				continue;
			int x = (int)(i % w), y = (int)(i / w);
			for (int r = 2; r <= limit; ++r) {
				int x0 = x - r < 0 ? 0 : x - r, x1 = x + r > w - 1 ? w - 1 : x + r;
				int y0 = y - r < 0 ? 0 : y - r, y1 = y + r > h - 1 ? h - 1 : y + r;
				int ww = x1 - x0 + 1, area = ww * (y1 - y0 + 1), count = 0;
				double lo, hi;
				if (area <= 32) {
					double lanes[32];
					for (int l = 0; l < 32; ++l)
						lanes[l] = INFINITY;
					for (int pos = 0; pos < area; ++pos) {
						size_t j = (size_t)(y0 + pos / ww) * w + x0 + pos % ww;
						if (is_donor(clean, crmask, excluded, j)) {
							lanes[pos] = clean[j];
							++count;
						}
					}
					if (!count)
						continue;
					oracle_bitonic32(lanes);
					lo = lanes[(count - 1) / 2];
					hi = lanes[count / 2];
				} else {
					if ((size_t)area > cap) {
						cap = (size_t)area;
						keys = realloc(keys, cap * sizeof(*keys));
					}
					for (int pos = 0; pos < area; ++pos) {
						size_t j = (size_t)(y0 + pos / ww) * w + x0 + pos % ww;
						if (is_donor(clean, crmask, excluded, j))
							keys[count++] = order_key(clean[j]);
					}
					if (!count)
						continue;
					qsort(keys, (size_t)count, sizeof(*keys), cmp_u64);
					lo = order_value(keys[(count - 1) / 2]);
					hi = order_value(keys[count / 2]);
				}
				clean[i] = count % 2 ? 0.0 + lo : midpoint(lo, hi);
				break;
			}
		}
		free(keys);
	}
}

/*
 * One frame through src/cleaner.cuh:144-187 (with src/image.cuh:24-92,
 * src/filters.cuh:107-193 and src/cleaner.cuh:22-37,78-142).  Frames of a
 * reference batch are independent: a frame whose update flags no new pixel
 * would repeat the same pass forever, so stopping it early (instead of when
 * all frames stop) changes no output, and the "no donors" error of a frame
 * is raised in the same pass either way.
 *
 * Returns 0, or 1 with msg set when a target has no finite donor.  Writes the
 * number of detection passes run to *passes when not NULL.
 */
int
oracle_clean_frame(const oracle_image *im, const oracle_options *o, double *out,
	uint8_t *mask, int *passes, char *msg, size_t msg_size)
{
	int w = (int)im->width, h = (int)im->height;
	size_t n = (size_t)w * h;
	const double *data = im->data;
	int has_bg = im->background || !isnan(o->background);
	if (passes)
		*passes = 0;
	if (msg && msg_size)
		msg[0] = 0;

	if (!o->maxiter) { /* src/image.cuh:72-92 */
		for (size_t i = 0; i < n; ++i) {
			double v = isfinite(data[i]) ? data[i] : 0;
			if (has_bg) {
				double bg = im->background ? im->background[i] : o->background;
				v += 1 * bg;
				v += -1 * bg;
			}
			out[i] = isfinite(data[i]) ? v : data[i];
			mask[i] = 0;
		}
		return 0;
	}

	double *clean = malloc(n * sizeof(double) * 8);
	uint8_t *bytes = calloc(n, 5);
	if (!clean || !bytes) {
		free(clean);
		free(bytes);
		if (msg && msg_size)
			snprintf(msg, msg_size, "out of memory");
		return 3;
	}
	double *lap = clean + n, *noise = lap + n, *med5 = noise + n, *sig = med5 + n;
	double *med3 = sig + n, *med7 = med3 + n, *fine = med7 + n;
	uint8_t *crmask = bytes, *excluded = crmask + n, *cand = excluded + n;
	uint8_t *grown = cand + n, *hole = grown + n;
	int status = 0;

	/* src/image.cuh:24-48 */
	size_t holes = 0, allowed = 0, donors = 0;
	for (size_t i = 0; i < n; ++i) {
		hole[i] = !isfinite(data[i]);
		int ok = !hole[i] && !(im->mask && im->mask[i]);
		excluded[i] = !ok;
		clean[i] = hole[i] ? 0 : data[i];
		if (has_bg)
			clean[i] += 1 * (im->background ? im->background[i] : o->background);
		holes += hole[i];
		allowed += ok;
	}
	/* src/cleaner.cuh:78-100: fill holes from finite, unmasked donors. */
	for (size_t i = 0; i < n; ++i)
		donors += is_donor(clean, crmask, excluded, i);
	if (holes && allowed && !donors) {
		status = 1;
		goto done;
	}
	if (holes && donors)
		replace(clean, hole, excluded, w, h);

	for (int it = 0; it < o->maxiter; ++it) {
		if (passes)
			*passes = it + 1;
		/* src/cleaner.cuh:102-126 */
		laplacian(clean, lap, w, h, o->border);
		const double *nz = im->error;
		if (!nz) { /* src/filters.cuh:107-123 */
			median_filter(clean, med5, w, h, o->border, 5);
			for (size_t i = 0; i < n; ++i) {
				double g = im->gain ? im->gain[i] : o->gain;
				double rn = im->readnoise ? im->readnoise[i] : o->readnoise;
				double m = med5[i] < SIGNAL_FLOOR ? SIGNAL_FLOOR : med5[i];
				noise[i] = sqrt(rn * rn + g * m) / g;
			}
			nz = noise;
		}
		for (size_t i = 0; i < n; ++i) /* src/filters.cuh:125-135 */
			sig[i] = lap[i] / (2 * nz[i]);
		median_filter(sig, med5, w, h, o->border, 5);
		for (size_t i = 0; i < n; ++i) /* src/filters.cuh:137-146 */
			sig[i] = isfinite(data[i]) ? sig[i] - med5[i] : 0;
		median_filter(clean, med3, w, h, o->border, 3);
		median_filter(med3, med7, w, h, o->border, 7);
		for (size_t i = 0; i < n; ++i) { /* src/filters.cuh:148-162 */
			double v = (med3[i] - med7[i]) / nz[i];
			fine[i] = v < FINE_FLOOR ? FINE_FLOOR : v;
		}
		for (size_t i = 0; i < n; ++i) /* src/filters.cuh:164-175 */
			cand[i] = !excluded[i] && sig[i] > o->cr_threshold &&
				sig[i] / fine[i] > o->contrast;
		/* src/filters.cuh:177-193, twice (src/cleaner.cuh:123-125) */
		for (int pass = 0; pass < 2; ++pass) {
			const uint8_t *in = pass ? grown : cand;
			uint8_t *dst = pass ? cand : grown;
			double thr = pass ? o->neighbor_threshold : o->cr_threshold;
			for (int y = 0; y < h; ++y)
				for (int x = 0; x < w; ++x) {
					size_t i = (size_t)y * w + x;
					uint8_t v = 0;
					if (sig[i] > thr)
						for (int yy = y > 0 ? y - 1 : 0; yy <= (y + 1 < h ? y + 1 : h - 1); ++yy)
							for (int xx = x > 0 ? x - 1 : 0; xx <= (x + 1 < w ? x + 1 : w - 1); ++xx)
								v |= in[(size_t)yy * w + xx] != 0;
					dst[i] = v;
				}
		}
		/* src/cleaner.cuh:22-37,128-142 */
		size_t todo = 0;
		donors = 0;
		for (size_t i = 0; i < n; ++i) {
			todo += cand[i] && !crmask[i];
			crmask[i] |= cand[i];
			donors += is_donor(clean, crmask, excluded, i);
		}
		if (todo && !donors) {
			status = 1;
			goto done;
		}
		if (!todo)
			break;
		replace(clean, crmask, excluded, w, h);
	}

	/* src/image.cuh:50-70 */
	for (size_t i = 0; i < n; ++i) {
		double v = clean[i];
		if (has_bg)
			v += -1 * (im->background ? im->background[i] : o->background);
		out[i] = isfinite(data[i]) ? v : data[i];
		mask[i] = crmask[i];
	}
done:
	if (status && msg && msg_size)
		snprintf(msg, msg_size, "no finite replacement donors");
	free(clean);
	free(bytes);
	return status;
}

/* Exposed for tests that restate the reference building blocks. */
void
oracle_median_filter(const double *a, double *out, int w, int h, int mode, int size)
{
	median_filter(a, out, w, h, mode, size);
}

void
oracle_laplacian(const double *clean, double *lap, int w, int h, int mode)
{
	laplacian(clean, lap, w, h, mode);
}

void
oracle_replace(double *clean, const uint8_t *crmask, const uint8_t *excluded, int w, int h)
{
	replace(clean, crmask, excluded, w, h);
}

/*
 * Reference gradient of the cleaned pixels with a frozen mask, from CPU
 * selection indices (the adjoint has no counterpart in the reference; this
 * is its definition).  For the final mask `crmask` of a forward run:
 *   - unflagged pixels pass grad straight through (non-finite ones too);
 *   - a flagged pixel sends grad to the donor its final replacement median
 *     selected (odd count), or half to each of the two central donors (even
 *     count); donors are finite, unmasked, unflagged pixels of data + bg,
 *     ordered by IEEE total order (src/replace.cuh:37-48), ties by lowest
 *     linear index;
 *   - with background, flagged pixels add -grad to their own background and
 *     the donor weights to the donors' backgrounds (scalar background: the
 *     per-target sum, which is zero).
 * grad_bg_map may be NULL; *grad_bg_scalar accumulates the scalar case.
 */
void
oracle_backward(const oracle_image *im, const oracle_options *o, const uint8_t *crmask,
	const double *grad, double *grad_data, double *grad_bg_map, double *grad_bg_scalar)
{
	int w = (int)im->width, h = (int)im->height;
	size_t n = (size_t)w * h;
	int has_bg = im->background || !isnan(o->background);
	double *pre = malloc(n * sizeof(double));
	uint8_t *donor = malloc(n);
	uint64_t *keys = malloc(n * sizeof(uint64_t));
	int *idx = malloc(n * sizeof(int));
	for (size_t i = 0; i < n; ++i) {
		double d = im->data[i];
		double c = isfinite(d) ? d : 0;
		if (has_bg)
			c += 1 * (im->background ? im->background[i] : o->background);
		pre[i] = c;
		int excluded = !isfinite(d) || (im->mask && im->mask[i]);
		donor[i] = !crmask[i] && !excluded && isfinite(c);
		grad_data[i] = crmask[i] ? 0.0 : grad[i];
		if (grad_bg_map)
			grad_bg_map[i] = crmask[i] ? -grad[i] : 0.0;
	}
	double scalar = 0;
	int limit = w > h ? w : h;
	for (size_t i = 0; i < n; ++i) {
		if (!crmask[i])
			continue;
		int x = (int)(i % w), y = (int)(i / w);
		for (int r = 2; r <= limit; ++r) {
			int x0 = x - r < 0 ? 0 : x - r, x1 = x + r > w - 1 ? w - 1 : x + r;
			int y0 = y - r < 0 ? 0 : y - r, y1 = y + r > h - 1 ? h - 1 : y + r;
			int count = 0;
			for (int yy = y0; yy <= y1; ++yy)
				for (int xx = x0; xx <= x1; ++xx) {
					size_t j = (size_t)yy * w + xx;
					if (!donor[j])
						continue;
					/* insertion by (key, linear index); cells arrive in
					 * increasing linear index, so a strict key test is stable */
					uint64_t k = order_key(pre[j]);
					int p = count++;
					while (p > 0 && k < keys[p - 1]) {
						keys[p] = keys[p - 1];
						idx[p] = idx[p - 1];
						--p;
					}
					keys[p] = k;
					idx[p] = (int)j;
				}
			if (!count)
				continue;
			double g = grad[i];
			int lo = idx[(count - 1) / 2], hi = idx[count / 2];
			double wl = count % 2 ? g : g / 2, wh = count % 2 ? 0.0 : g / 2;
			grad_data[lo] += wl;
			if (!(count % 2))
				grad_data[hi] += wh;
			if (grad_bg_map) {
				grad_bg_map[lo] += wl;
				if (!(count % 2))
					grad_bg_map[hi] += wh;
			}
			if (has_bg)
				scalar += (wl + wh) - g;
			break;
		}
	}
	if (grad_bg_scalar)
		*grad_bg_scalar = scalar;
	free(pre);
	free(donor);
	free(keys);
	free(idx);
}

/* Host threads of the OpenMP loops above (n <= 0: leave as is); returns the
 * count in effect.  The CPU baseline times the restatement both on one thread
 * and on every host core. */
int
oracle_set_threads(int n)
{
#ifdef _OPENMP
	if (n > 0)
		omp_set_num_threads(n);
	return omp_get_max_threads();
#else
	(void)n;
	return 1;
#endif
}

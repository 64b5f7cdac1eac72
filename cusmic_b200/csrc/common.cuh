// Shared definitions of the cusmic_b200 kernels: border mapping, frame
// descriptors, per-frame state, bit-plane layout and small device helpers.
//
// HBM layout of one call (all per frame, frames back to back):
//   clean      float64 [h][w]      working pixels; the caller's output buffer
//   bit planes uint32  [N_PLANES][frames][h][words], words = ceil(w / 32); bit b of
//              word (y, k) is pixel (y, 32 k + b); padding bits are zero
//   targets    uint2   {frame, pixel} list of replacement targets
#pragma once
#include <cstdint>
#include <cmath>
#include <cuda_runtime.h>

#if defined(__CUDACC__)
#define CB_HD __host__ __device__ __forceinline__
#else
#define CB_HD inline
#endif

namespace cb {

using std::fabs;
using std::fmax;
using std::fmin;
using std::isfinite;
using std::isnan;
using std::sqrt;

enum Border { REFLECT = 0, CONSTANT = 1, NEAREST = 2, MIRROR = 3, WRAP = 4 };

// Bit planes of a frame.
enum Plane {
	P_HOLE,   // non-finite input pixel
	P_EXCL,   // excluded from seeds and donors: hole or masked
	P_DONOR,  // static donor: not excluded and finite after background
	P_CRMASK, // cumulative cosmic-ray mask
	P_HIGH,   // holds every pixel with sig_raw > cr_threshold (or NaN) on the
	          // current clean pixels (a superset after the first pass)
	P_LOW,    // with HIGH, holds every pixel with sig_raw > neighbor_threshold
	P_S1,     // significance > cr_threshold
	P_S2,     // significance > neighbor_threshold
	P_CAND,   // seed: S1, not excluded, contrast test passed
	P_FRESH,  // pixels the last growth step added to the mask
	P_CHG,    // pixels whose value the last replacement changed
	P_ROWMIN, // noise-model frames: per row and bit word, the smallest high word of
	          // the ordered keys of its finite input pixels (all ones: none)
	N_PLANES
};

static_assert(P_S2 == P_S1 + 1 && P_CAND == P_S1 + 2 && P_FRESH == P_S1 + 3,
	"S1, S2, CAND and FRESH are zeroed as one range before a full pass");

constexpr double FINE_FLOOR = 0.01;   // reference src/filters.cuh:21
constexpr double SIGNAL_FLOOR = 1e-5; // reference src/filters.cuh:22

// scipy.ndimage border conventions, reference src/filters.cuh:24-44: returns
// the in-range index a coordinate reads, or -1 for a constant (zero) pad.
CB_HD int border_index(int x, int n, int mode)
{
	if (x >= 0 && x < n)
		return x;
	if (mode == CONSTANT)
		return -1;
	if (mode == NEAREST)
		return x < 0 ? 0 : n - 1;
	if (n == 1)
		return 0;
	int period = mode == REFLECT ? 2 * n : mode == MIRROR ? 2 * (n - 1) : n;
	x %= period;
	if (x < 0)
		x += period;
	if (mode == REFLECT && x >= n)
		return period - x - 1;
	if (mode == MIRROR && x >= n)
		return period - x;
	return x;
}

CB_HD int clampi(int x, int lo, int hi)
{
	return x < lo ? lo : x > hi ? hi : x;
}

// Noise floor of a 32 x 32 block of a frame (see bulk.cuh): the detection
// threshold of an error-map block, or for a noise-model block lower bounds
// kept as ordered keys (a smaller key is a smaller value): of its clean values
// (lowered by every replacement inside the block), of -gain and of the read
// noise over the block (gain and read-noise maps only).  All-ones keys: no
// value seen yet.
struct BlockFloor {
	double thr;
	unsigned long long key, gkey, rkey;
};

// One frame of a (possibly ragged) batch, as the kernels see it.
struct FrameDesc {
	const double *data, *error, *gain_map, *rn_map, *bg_map;
	const uint8_t *mask;
	double *clean;     // working pixels, restored in place into the output
	double *out;       // output pixels: clean itself (null means the same), or for a frame
	                   // with a background the caller's buffer while clean is a
	                   // workspace buffer: prepare then writes every output pixel
	                   // except the flagged ones, which restore writes
	uint8_t *mask_out; // uint8 output mask
	uint32_t *bits;    // N_PLANES planes of `plane` words
	BlockFloor *floors; // the frame's block floors, row-major by block (null: none)
	uint32_t *rowcand;  // per row: nonzero when growth must visit the row this pass (null: all)
	uint32_t *rowchg;   // per row: nonzero when the row has a CHG pixel (null: no tracking)
	// Noise-model frames, first pass: sig_raw and the noise at every pixel
	// within two of a HIGH pixel (region_sig_kernel), which the high-list
	// candidates read instead of recomputing their windows (null: none).
	double *sig_raw, *noise;
	double gain, rn, bg;
	long long plane;   // words per plane of this frame = h * words
	long long pstride; // words from one plane to the next (planes of all frames of a
	                   // batch are interleaved plane by plane, so pstride >= plane)
	int w, h, words, has_bg;
};

// Device-side control state of a frame.
struct FrameState {
	unsigned int active;  // the next detection pass runs for this frame
	unsigned int replace; // this pass flagged new pixels: re-replace targets
	unsigned int error;   // a target had no finite donor
	unsigned int passes;  // detection passes run
	unsigned int fault;   // a bounded wait inside a kernel ran out (the frame stopped)
	// Nonzero-only facts (set to 1 by many warps, never counted):
	unsigned long long todo;                  // this pass: any new pixel
	long long donors_left;                    // static donors not in the mask (counted)
	unsigned long long holes, allowed, finite; // any hole, any allowed pixel, any finite donor
};

// Loop control shared by the per-pass kernels.
struct Control {
	unsigned long long n_targets; // length of the target list
	unsigned long long n_holes;   // length of the hole list prepare_kernel writes
	unsigned long long n_cand;    // this pass: pixels whose sig_raw can exceed cr_threshold
	unsigned long long n_low;     // this pass: pixels whose sig_raw can only exceed neighbor
	unsigned long long cand_cap;  // capacity of the candidate buffer (high from the front,
	                              // low from the back)
	int iter;                     // detection passes issued so far
	int maxiter;
	int any_active;
	int ticket;                   // next item of the bulk detection kernel (reset every pass)
	int fault;                    // a bounded wait ran out in this pass
	int n_dirty;                  // this pass: length of the dirty-row list
	unsigned n_sel;               // this pass: targets the replacement visits
	unsigned pad;
	unsigned long long n_region;  // first pass: pixels of the noise-model sig_raw map (listed)
	// Injected failures (0: none): the bound, in SM cycles, of one extra wait
	// on a barrier that nothing completes, made by one warp of the first block
	// of the bulk-staged prepare ([0]) and of the dense detection kernel ([1]).
	long long poison_wait[2];
};

CB_HD uint32_t *plane_ptr(const FrameDesc &f, int p)
{
	return f.bits + (long long)p * f.pstride;
}

CB_HD bool test_bit(const uint32_t *plane, int words, int x, int y)
{
	return (plane[(long long)y * words + (x >> 5)] >> (x & 31)) & 1u;
}

#ifdef __CUDACC__
// Sets or clears bit `bit` of *word, for a caller that is the only writer of
// that bit (other bits of the word may change concurrently): an atomic only
// when the bit changes.  `fresh`: the plane was zeroed for this pass, so only
// a set needs an atomic and nothing is read.
__device__ __forceinline__ void write_bit(uint32_t *word, uint32_t bit, bool value, bool fresh = false)
{
	if (fresh) {
		if (value)
			atomicOr(word, bit);
		return;
	}
	const bool now = (*(volatile uint32_t *)word & bit) != 0;
	if (value && !now)
		atomicOr(word, bit);
	else if (!value && now)
		atomicAnd(word, ~bit);
}
#endif

} // namespace cb

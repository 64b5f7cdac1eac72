// Per-pass kernels around the detection kernel: preparation, bit-packed growth
// and mask update, loop control, replacement, restoration.
//
// Row kernels give one warp a frame row at a time (a row-item list of
// {frame, y} covers ragged batches), so each warp instruction reads 32
// consecutive float64 pixels and the bit planes fall out of __ballot_sync.
#pragma once
#include "common.cuh"
#include "select.cuh"

namespace cb {

__device__ __forceinline__ int warp_sum_int(int v)
{
#pragma unroll
	for (int o = 16; o; o >>= 1)
		v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v)
{
#pragma unroll
	for (int o = 16; o; o >>= 1)
		v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}

__device__ __forceinline__ int warp_inclusive_count(int cnt)
{
	const int lane = threadIdx.x & 31;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		int v = __shfl_up_sync(0xffffffffu, cnt, o);
		if (lane >= o)
			cnt += v;
	}
	return cnt;
}

__device__ __forceinline__ int warp_exclusive_count(int cnt)
{
	return warp_inclusive_count(cnt) - cnt;
}

// Append `cnt` entries per lane to a global list; returns this lane's first slot.
__device__ __forceinline__ unsigned long long warp_append(unsigned long long *counter, int cnt)
{
	const int lane = threadIdx.x & 31;
	int incl = cnt;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		int v = __shfl_up_sync(0xffffffffu, incl, o);
		if (lane >= o)
			incl += v;
	}
	int total = __shfl_sync(0xffffffffu, incl, 31);
	unsigned long long base = 0;
	if (lane == 31 && total)
		base = atomicAdd(counter, (unsigned long long)total);
	base = __shfl_sync(0xffffffffu, base, 31);
	return base + (unsigned long long)(incl - cnt);
}

// Per-frame facts that the loop control only tests for zero (any hole, any
// allowed pixel, any new pixel, any donor left): many warps set the same flag
// with a plain store instead of contending on an atomic counter.
__device__ __forceinline__ void set_flag(unsigned long long *flag)
{
	if (!*(volatile unsigned long long *)flag)
		*(volatile unsigned long long *)flag = 1;
}

// Map validation of the host entry point on the device (reference
// src/api.cu:107-114 runs it on the host): sets `bit` in *flags if any of the
// n values is not finite, or (minimum 1) not positive, or (minimum 0)
// negative.
__global__ void __launch_bounds__(256)
validate_kernel(const double *__restrict__ v, long long n, int minimum, unsigned *flags, unsigned bit)
{
	bool bad = false;
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
	     i += (long long)gridDim.x * blockDim.x) {
		const double x = v[i];
		bad |= !isfinite(x) || (minimum == 1 && x <= 0) || (minimum == 0 && x < 0);
	}
	if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0)
		atomicOr(flags, bit);
}

// Per-frame state and loop control of a call; with `zero`, also zeroes the n16
// 16-byte words at zero (the bit planes that nothing writes before the first
// pass, and the row marks) with a grid-stride loop of 16-byte stores.
__device__ __forceinline__ void init_state(FrameState *state, int nf, Control *ctl, int maxiter,
	unsigned long long cand_cap, long long poison_prepare, long long poison_detect, uint4 *zero,
	long long n16, uint4 *zero2, long long n16b)
{
	const long long stride = (long long)gridDim.x * blockDim.x;
	for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n16; j += stride)
		zero[j] = make_uint4(0u, 0u, 0u, 0u);
	for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n16b; j += stride)
		zero2[j] = make_uint4(0u, 0u, 0u, 0u);
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < nf) {
		FrameState s = {};
		s.active = maxiter > 0;
		state[i] = s;
	}
	if (i == 0) {
		Control c = {};
		c.maxiter = maxiter;
		c.cand_cap = cand_cap;
		c.any_active = maxiter > 0;
		c.poison_wait[0] = poison_prepare;
		c.poison_wait[1] = poison_detect;
		*ctl = c;
	}
}

__global__ void init_kernel(FrameState *state, int nf, Control *ctl, int maxiter,
	unsigned long long cand_cap, long long poison_prepare = 0, long long poison_detect = 0,
	uint4 *zero = nullptr, long long n16 = 0, uint4 *zero2 = nullptr, long long n16b = 0)
{
	init_state(state, nf, ctl, maxiter, cand_cap, poison_prepare, poison_detect, zero, n16, zero2, n16b);
}

// IEEE bits mapped to an unsigned total order (reference src/replace.cuh:37-48).
__device__ __forceinline__ unsigned long long order_key(double v)
{
	unsigned long long b = (unsigned long long)__double_as_longlong(v);
	return (b >> 63) ? ~b : b ^ (1ull << 63);
}

__device__ __forceinline__ double order_value(unsigned long long k)
{
	return __longlong_as_double((long long)((k >> 63) ? k ^ (1ull << 63) : ~k));
}

// Reference src/image.cuh:24-48: holes, exclusions, clean = data (+ bg), the
// static donor plane (the reference's is_donor with an empty mask) and the
// per-frame facts the initial fill needs (src/cleaner.cuh:78-100).  A warp
// loads ROW_UNROLL chunks of 32 pixels before using them, so enough bytes are
// in flight per SM to approach the HBM bandwidth.
constexpr int ROW_UNROLL = 4;

// Frame kinds of prepare_row: the input maps it reads and whether it writes
// noise-model row minima.  A batch whose frames are all of one kind gets a
// prepare_kernel compiled for that kind (PREP_ANY decides per row).
enum PrepKind { PREP_ANY, PREP_PLAIN, PREP_MASK, PREP_MAPS, PREP_MODEL, PREP_MODEL_MAPS };

CB_HD int prep_kind(const FrameDesc &fd)
{
	const bool mask = fd.mask, bgmap = fd.bg_map;
	if (fd.floors && !fd.error) // noise-model frame: row minima for the floors
		return mask || bgmap ? PREP_MODEL_MAPS : PREP_MODEL;
	return bgmap ? PREP_MAPS : mask ? PREP_MASK : PREP_PLAIN;
}


// One row of prepare_kernel for the frame kinds that occur: MASK = input
// mask, BGMAP = background map.  Descriptor fields are held in registers (the
// stores below go through pointers the compiler cannot prove distinct from
// them).
template <bool MASK, bool BGMAP, bool ROWMIN, int U = ROW_UNROLL, bool OUT = false>
__device__ __forceinline__ void prepare_row(const FrameDesc &fd, FrameState &st, int f, int y,
	Control *ctl, uint2 *holes)
{
	const int lane = threadIdx.x & 31;
	const int w = fd.w, words = fd.words;
	const long long rowpix = (long long)y * w, roww = (long long)y * words;
	const double *__restrict__ data = fd.data + rowpix;
	// MASK / BGMAP false: the frame has none; true: it may have one.
	const uint8_t *__restrict__ mask = MASK && fd.mask ? fd.mask + rowpix : nullptr;
	const double *__restrict__ bgmap = BGMAP && fd.bg_map ? fd.bg_map + rowpix : nullptr;
	double *__restrict__ clean = fd.clean + rowpix;
	// A separate output buffer (a frame with a background): its pixels now,
	// (x + bg) - bg as the reference's restore computes them, the input at a
	// hole; restore writes only the flagged ones.
	double *__restrict__ out = OUT && fd.out && fd.out != fd.clean ? fd.out + rowpix : nullptr;
	const double bgv = fd.bg;
	const bool has_bg = fd.has_bg;
	uint32_t *hole_plane = plane_ptr(fd, P_HOLE) + roww, *excl_plane = plane_ptr(fd, P_EXCL) + roww;
	uint32_t *donor_plane = plane_ptr(fd, P_DONOR) + roww;
	uint32_t any_hole = 0, any_allowed = 0, any_finite = 0;
	int ndonor = 0;
	// Noise-model frames with floors: per bit word the smallest high word of
	// the ordered keys of the non-hole clean values (a lower bound for the
	// block floors, which the hole fill then lowers with the values it writes).
	uint32_t *rowmin = ROWMIN ? plane_ptr(fd, P_ROWMIN) + roww : nullptr;
	for (int seg = 0; seg * 1024 < w; ++seg) {
		uint32_t my_h = 0, my_e = 0, my_d = 0, my_m = 0xffffffffu;
		for (int c0 = 0; c0 < 32; c0 += U) {
			const int xb = seg * 1024 + c0 * 32;
			if (xb >= w)
				break; // warp-uniform
			double d[U], bg[U];
			bool m[U];
#pragma unroll
			for (int u = 0; u < U; ++u) {
				const int x = xb + 32 * u + lane;
				d[u] = 0;
				bg[u] = bgv;
				m[u] = false;
				if (x < w) {
					d[u] = data[x];
					if (MASK && mask)
						m[u] = mask[x] != 0;
					if (BGMAP && bgmap)
						bg[u] = bgmap[x];
				}
			}
#pragma unroll
			for (int u = 0; u < U; ++u) {
				const int x0 = xb + 32 * u;
				const int x = x0 + lane;
				const bool valid = x < w;
				bool hole = false, ok = false, donor = false;
				double c = 0;
				if (valid) {
					hole = !isfinite(d[u]);
					ok = !hole && !m[u];
					c = hole ? 0 : d[u];
					if (has_bg)
						c += 1 * bg[u];
					clean[x] = c;
					if (out)
						out[x] = hole ? d[u] : c + -1 * bg[u];
					donor = ok && isfinite(c);
				}
				const uint32_t hw = __ballot_sync(0xffffffffu, hole);
				uint32_t mw = 0xffffffffu;
				if (ROWMIN)
					mw = __reduce_min_sync(0xffffffffu,
						valid && !hole ? (uint32_t)(order_key(c) >> 32) : 0xffffffffu);
				const uint32_t ew = __ballot_sync(0xffffffffu, valid && !ok);
				const uint32_t dw = __ballot_sync(0xffffffffu, donor);
				any_allowed |= __ballot_sync(0xffffffffu, ok);
				any_finite |= dw;
				any_hole |= hw;
				ndonor += __popc(dw);
				if (lane == c0 + u) {
					my_h = hw;
					my_e = ew;
					my_d = dw;
					my_m = mw;
				}
			}
		}
		const int k = seg * 32 + lane;
		if (k < words) {
			hole_plane[k] = my_h;
			excl_plane[k] = my_e;
			donor_plane[k] = my_d;
			if (ROWMIN)
				rowmin[k] = my_m;
		}
		if (holes && __any_sync(0xffffffffu, my_h != 0)) { // list the segment's holes for the fill
			unsigned long long slot = warp_append(&ctl->n_holes, __popc(my_h));
			for (uint32_t b = my_h; b; b &= b - 1)
				holes[slot++] = make_uint2((unsigned)f, (unsigned)(rowpix + 32 * k + __ffs(b) - 1));
		}
	}
	if (lane == 0) {
		if (any_hole)
			set_flag(&st.holes);
		if (any_allowed)
			set_flag(&st.allowed);
		if (any_finite)
			set_flag(&st.finite);
		if (ndonor)
			atomicAdd((unsigned long long *)&st.donors_left, (unsigned long long)ndonor);
	}
}

// One warp per row (grid-stride over the row list), in segments of 32 words
// (1024 pixels): lane j keeps the HOLE, EXCL and DONOR words of the
// segment's word j, so each plane gets one coalesced store per segment.  The
// other planes were zeroed before the kernel.  With `holes`, each segment's
// holes are appended to that list (count in ctl->n_holes) for the hole fill.
// KIND: the frame kind every row has (PREP_ANY: decided per row); UL: the
// unroll of the kinds without maps.
// OUT: some frame of the batch has a separate output buffer.
template <int KIND = PREP_ANY, int UL = ROW_UNROLL, bool OUT = false>
__global__ void __launch_bounds__(256, 4)
prepare_kernel(const FrameDesc *__restrict__ frames, FrameState *state, const int2 *__restrict__ rows,
	int nrows, Control *ctl = nullptr, uint2 *holes = nullptr)
{
	const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
	for (int r = gw; r < nrows; r += nw) {
		const int2 item = rows[r];
		const FrameDesc &fd = frames[item.x];
		FrameState &st = state[item.x];
		switch (KIND == PREP_ANY ? prep_kind(fd) : KIND) {
		case PREP_MODEL:
			prepare_row<false, false, true, UL, OUT>(fd, st, item.x, item.y, ctl, holes);
			break;
		case PREP_MODEL_MAPS:
			prepare_row<true, true, true, ROW_UNROLL, OUT>(fd, st, item.x, item.y, ctl, holes);
			break;
		case PREP_MASK:
			prepare_row<true, false, false, UL, OUT>(fd, st, item.x, item.y, ctl, holes);
			break;
		case PREP_PLAIN:
			prepare_row<false, false, false, UL, OUT>(fd, st, item.x, item.y, ctl, holes);
			break;
		default:
			prepare_row<true, true, false, ROW_UNROLL, OUT>(fd, st, item.x, item.y, ctl, holes);
		}
	}
}

// 36-bit window of a bit-plane row around word k: bits 0..35 are pixels
// 32k-2 .. 32k+33 (zero outside the frame).
__device__ __forceinline__ unsigned long long bit_window(const uint32_t *plane, int words, int h,
	int y, int k)
{
	if (y < 0 || y >= h)
		return 0;
	const uint32_t *row = plane + (long long)y * words;
	unsigned long long c = row[k];
	unsigned long long l = k > 0 ? row[k - 1] : 0u;
	unsigned long long r = k + 1 < words ? row[k + 1] : 0u;
	return (l >> 30) | (c << 2) | ((r & 3ull) << 34);
}

__device__ __forceinline__ unsigned long long dilate_row(unsigned long long e)
{
	return e | (e << 1) | (e >> 1);
}

// Rows of a growth item (grow_kernel).
constexpr int GROW_ROWS = 16;

// 36-bit window of a bit-plane row (bit_window) for a lane whose word is past
// the row: zero.
__device__ __forceinline__ unsigned long long lane_window(const uint32_t *plane, int words, int h,
	int y, int k)
{
	return k < words ? bit_window(plane, words, h, y, k) : 0ull;
}

// Reference src/filters.cuh:177-193 twice (src/cleaner.cuh:123-125) and
// src/cleaner.cuh:22-37: grown = dilate3x3(dilate3x3(cand) & S1) & S2 on bit
// planes (clipped to the frame), fresh = grown & ~crmask, crmask |= grown,
// the FRESH plane, the per-frame facts (any fresh pixel; the count of static
// donors left, which the reference recounts in accumulate), and fresh pixels
// appended to the target list.
//
// One warp per item of GROW_ROWS rows x 32 bit words (a lane per word), from
// `items` {frame, first row, first word, end row}, or with items null from
// frame 0 in row-major item order.  The warp sweeps down its rows keeping the
// horizontal dilations of the CAND rows y .. y + 1 and of the S1-masked rows
// y - 1 .. y in registers, so each row step reads one CAND window, an S1
// window only where a dilated CAND pixel is near, S2 and CRMASK only where
// something can grow, and DONOR only where pixels are flagged; the item
// appends its fresh pixels with one atomic.  (Issuing the loads of four rows
// together, unconditionally, measured slower.)
//
// With row marks (fd.rowcand) an item none of whose rows is marked is
// skipped: a full pass marks the rows within two of a CAND pixel (nothing
// grows elsewhere), an incremental pass the rows within six of a pixel whose
// value the last replacement changed (elsewhere grown repeats the last pass
// and is already in the mask).  A visited item computes all its rows (an
// unmarked row adds nothing) and clears the CHG bits of its rows with a CHG
// mark (every such row is marked; replace_select_kernel then clears the
// marks).  FRESH is written on every visited row (the pass starts with it
// zeroed where it skips).
__global__ void __launch_bounds__(256)
grow_kernel(const FrameDesc *__restrict__ frames, FrameState *state, const int4 *__restrict__ items,
	int nitems, uint2 *targets, Control *ctl)
{
	const int lane = threadIdx.x & 31;
	const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
	for (int i = gw; i < nitems; i += nw) {
		int4 it;
		if (items) {
			it = items[i];
		} else {
			const int strips = (frames[0].words + 31) / 32, y0 = (i / strips) * GROW_ROWS;
			it = make_int4(0, y0, (i % strips) * 32, min(y0 + GROW_ROWS, frames[0].h));
		}
		const int f = it.x;
		if (!state[f].active)
			continue; // warp-uniform
		const FrameDesc &fd = frames[f];
		const int w = fd.w, h = fd.h, words = fd.words, y0 = it.y, n = it.w - it.y, k = it.z + lane;
		const bool row_lane = lane < n;
		const unsigned visit = __ballot_sync(0xffffffffu,
			row_lane && (!fd.rowcand || fd.rowcand[y0 + lane]));
		if (!visit)
			continue; // warp-uniform
		const unsigned chg = fd.rowchg
			? __ballot_sync(0xffffffffu, row_lane && fd.rowchg[y0 + lane]) : 0u;
		const uint32_t *cand = plane_ptr(fd, P_CAND), *s1 = plane_ptr(fd, P_S1);
		const uint32_t *s2 = plane_ptr(fd, P_S2), *donor = plane_ptr(fd, P_DONOR);
		uint32_t *crm = plane_ptr(fd, P_CRMASK), *fr = plane_ptr(fd, P_FRESH);
		uint32_t *cg = plane_ptr(fd, P_CHG);
		// Dilated CAND rows y0 - 2 .. y0 + 1, then the dilated S1-masked rows
		// y0 - 1 and y0 (h0, h1); c0, c1: dilated CAND rows y and y + 1.
		unsigned long long c0, c1, h0, h1;
		{
			const unsigned long long d0 = dilate_row(lane_window(cand, words, h, y0 - 2, k));
			const unsigned long long d1 = dilate_row(lane_window(cand, words, h, y0 - 1, k));
			c0 = dilate_row(lane_window(cand, words, h, y0, k));
			c1 = dilate_row(lane_window(cand, words, h, y0 + 1, k));
			const unsigned long long a = d0 | d1 | c0, b = d1 | c0 | c1;
			h0 = a ? dilate_row(a & lane_window(s1, words, h, y0 - 1, k)) : 0ull;
			h1 = b ? dilate_row(b & lane_window(s1, words, h, y0, k)) : 0ull;
		}
		int cnt = 0, lost = 0;
		unsigned rows_fresh = 0; // bit j: this lane flagged pixels in row y0 + j
#pragma unroll 4
		for (int j = 0; j < n; ++j) {
			const int y = y0 + j;
			const unsigned long long c2 = dilate_row(lane_window(cand, words, h, y + 2, k));
			const unsigned long long cc = c0 | c1 | c2;
			const unsigned long long h2 = cc ? dilate_row(cc & lane_window(s1, words, h, y + 1, k)) : 0ull;
			const uint32_t near = (uint32_t)((h0 | h1 | h2) >> 2); // bits 2..33: the word's pixels
			if (k < words) {
				const long long o = (long long)y * words + k;
				uint32_t fresh = 0;
				if (near) {
					const uint32_t grown = near & s2[o], old = crm[o];
					fresh = grown & ~old;
					if (fresh) {
						crm[o] = old | fresh;
						cnt += __popc(fresh);
						lost += __popc(fresh & donor[o]);
						rows_fresh |= 1u << j;
					}
				}
				fr[o] = fresh;
				if ((chg >> j) & 1u)
					cg[o] = 0u;
			}
			c0 = c1;
			c1 = c2;
			h0 = h1;
			h1 = h2;
		}
		const bool any = __any_sync(0xffffffffu, cnt != 0);
		if (any) {
			unsigned long long slot = warp_append(&ctl->n_targets, cnt);
			for (unsigned m = rows_fresh; m; m &= m - 1) {
				const int y = y0 + __ffs(m) - 1;
				uint32_t fresh = fr[(long long)y * words + k]; // this lane's own store
				const unsigned base = (unsigned)((long long)y * w + 32 * k);
				while (fresh) {
					const int b = __ffs(fresh) - 1;
					fresh &= fresh - 1;
					targets[slot++] = make_uint2((unsigned)f, base + b);
				}
			}
		}
		lost = __reduce_add_sync(0xffffffffu, (unsigned)lost);
		if (lane == 0) {
			if (any)
				set_flag(&state[f].todo);
			if (lost)
				atomicAdd((unsigned long long *)&state[f].donors_left,
					(unsigned long long)(-(long long)lost));
		}
	}
}

// Per-frame loop control after a pass (reference src/cleaner.cuh:128-142,
// 175-181): a frame with new pixels but no donors fails, a frame without new
// pixels stops (its later passes would repeat this one), the others replace
// and continue.  With a graph handle, sets the while-node condition.
__global__ void __launch_bounds__(1024)
control_kernel(FrameState *state, int nf, Control *ctl, cudaGraphConditionalHandle handle,
	int use_handle)
{
	int any = 0;
	const int fault = ctl->fault;
	for (int f = threadIdx.x; f < nf; f += blockDim.x) {
		FrameState s = state[f];
		s.replace = 0;
		if (s.active) {
			++s.passes;
			if (fault) { // this pass's detection is incomplete: stop, report
				s.fault = 1;
				s.active = 0;
			} else if (s.todo && s.donors_left <= 0) {
				s.error = 1;
				s.active = 0;
			} else if (s.todo) {
				s.replace = 1;
				any = 1;
			} else {
				s.active = 0;
			}
		}
		s.todo = 0;
		state[f] = s;
	}
	any = __syncthreads_or(any);
	if (threadIdx.x == 0) {
		int it = ++ctl->iter;
		ctl->any_active = any;
		ctl->n_cand = 0;
		ctl->n_low = 0;
		ctl->ticket = 0;
		ctl->n_dirty = 0;
		ctl->n_sel = 0;
		if (use_handle)
			cudaGraphSetConditional(handle, (any && it < ctl->maxiter) ? 1u : 0u);
	}
}

// Reference src/replace.cuh:50-56.
__device__ __forceinline__ double midpoint(double lo, double hi)
{
	if (fabs(lo) < 1 && fabs(hi) < 1)
		return (lo + hi) / 2;
	return lo / 2 + hi / 2;
}

// Ascending bitonic network over the 32 lanes with the reference's exchange
// (src/replace.cuh:68-83): strict < comparisons, so equal values (such as -0
// and +0) end in the same lanes as in the reference.
__device__ __forceinline__ double bitonic32(double v)
{
	const int lane = threadIdx.x & 31;
#pragma unroll
	for (int span = 2; span <= 32; span *= 2) {
#pragma unroll
		for (int step = span / 2; step; step /= 2) {
			double peer = __shfl_xor_sync(0xffffffffu, v, step);
			bool lower = ((lane & span) == 0) == ((lane & step) == 0);
			v = lower ? (peer < v ? peer : v) : (v < peer ? peer : v);
		}
	}
	return v;
}

struct Window {
	int x0, x1, y0, y1;
};

__device__ __forceinline__ bool donor_at(const uint32_t *don, const uint32_t *crm, int words,
	int x, int y)
{
	long long o = (long long)y * words + (x >> 5);
	return ((don[o] & ~crm[o]) >> (x & 31)) & 1u;
}

// The donor of rank `rank` in key order inside a window larger than 32 cells:
// an MSB-first radix select over ordered 64-bit keys (same ranks as reference
// src/replace.cuh:85-109).  Up to 8 cells per lane are kept in registers.
__device__ double select_rank(const FrameDesc &fd, const uint32_t *don, const uint32_t *crm, Window win,
	int rank)
{
	const int lane = threadIdx.x & 31;
	const int ww = win.x1 - win.x0 + 1, area = ww * (win.y1 - win.y0 + 1);
	unsigned long long prefix = 0, used = 0;
	if (area <= 256) {
		unsigned long long keys[8];
		unsigned valid = 0;
#pragma unroll
		for (int s = 0; s < 8; ++s) {
			int pos = lane + 32 * s;
			keys[s] = 0;
			if (pos < area) {
				int x = win.x0 + pos % ww, y = win.y0 + pos / ww;
				if (donor_at(don, crm, fd.words, x, y)) {
					keys[s] = order_key(fd.clean[(long long)y * fd.w + x]);
					valid |= 1u << s;
				}
			}
		}
		for (int bit = 63; bit >= 0; --bit) {
			const unsigned long long flag = 1ull << bit;
			int below = 0;
#pragma unroll
			for (int s = 0; s < 8; ++s)
				below += ((valid >> s) & 1u) && (keys[s] & used) == prefix && !(keys[s] & flag);
			below = warp_sum_int(below);
			used |= flag;
			if (rank >= below) {
				prefix |= flag;
				rank -= below;
			}
		}
		return order_value(prefix);
	}
	for (int bit = 63; bit >= 0; --bit) {
		const unsigned long long flag = 1ull << bit;
		int below = 0;
		for (int pos = lane; pos < area; pos += 32) {
			int x = win.x0 + pos % ww, y = win.y0 + pos / ww;
			if (!donor_at(don, crm, fd.words, x, y))
				continue;
			unsigned long long k = order_key(fd.clean[(long long)y * fd.w + x]);
			below += (k & used) == prefix && !(k & flag);
		}
		below = warp_sum_int(below);
		used |= flag;
		if (rank >= below) {
			prefix |= flag;
			rank -= below;
		}
	}
	return order_value(prefix);
}

// The donors of a window of 33 .. 32 S cells in key order, for the median:
// lane l holds the keys of cells l + 32 s (all ones for a non-donor or a cell
// past the window, which sort last), a bitonic network sorts the warp's 32 S
// keys in unsigned order (the order select_rank's radix select ranks by),
// and the keys of ranks (nd - 1) / 2 and nd / 2 come back as lo and hi.
// Returns nd, the number of donors (0: lo and hi unset).  About 20 to 30
// dependent exchange steps instead of select_rank's 64 warp reductions per
// rank, so a replacement whose window grew past 5 x 5 no longer holds its
// launch for tens of microseconds.
template <int S>
__device__ __noinline__ int sorted_window_median(const FrameDesc &fd, const uint32_t *don,
	const uint32_t *crm, Window win, double &lo, double &hi)
{
	const int lane = threadIdx.x & 31;
	const int ww = win.x1 - win.x0 + 1, area = ww * (win.y1 - win.y0 + 1);
	unsigned long long k[S];
	int nd = 0;
#pragma unroll
	for (int s = 0; s < S; ++s) {
		const int pos = lane + 32 * s;
		k[s] = ~0ull;
		if (pos < area) {
			const int x = win.x0 + pos % ww, y = win.y0 + pos / ww;
			if (donor_at(don, crm, fd.words, x, y))
				k[s] = order_key(fd.clean[(long long)y * fd.w + x]);
		}
		nd += __popc(__ballot_sync(0xffffffffu, k[s] != ~0ull));
	}
	if (!nd)
		return 0;
	// Element i = 32 s + lane; ascending where bit `size` of i is clear.
#pragma unroll
	for (int size = 2; size <= 32 * S; size <<= 1) {
#pragma unroll
		for (int j = size >> 1; j > 0; j >>= 1) {
			if (j >= 32) { // partner in the same lane, slot s ^ (j / 32)
#pragma unroll
				for (int s = 0; s < S; ++s) {
					const int t = s ^ (j >> 5);
					if (t < s)
						continue;
					const bool asc = ((32 * s + lane) & size) == 0;
					const unsigned long long a = k[s], b = k[t];
					const bool swap = asc ? b < a : a < b;
					k[s] = swap ? b : a;
					k[t] = swap ? a : b;
				}
			} else { // partner lane ^ j, same slot
#pragma unroll
				for (int s = 0; s < S; ++s) {
					const unsigned long long p = __shfl_xor_sync(0xffffffffu, k[s], j);
					const bool keep_min = ((lane & j) == 0) == (((32 * s + lane) & size) == 0);
					k[s] = keep_min ? (p < k[s] ? p : k[s]) : (k[s] < p ? p : k[s]);
				}
			}
		}
	}
	const int rl = (nd - 1) / 2, rh = nd / 2;
	unsigned long long vl = 0, vh = 0;
#pragma unroll
	for (int s = 0; s < S; ++s) { // register slots chosen by unrolled tests, not indexed
		if (s == rl >> 5)
			vl = k[s];
		if (s == rh >> 5)
			vh = k[s];
	}
	lo = order_value(__shfl_sync(0xffffffffu, vl, rl & 31));
	hi = order_value(__shfl_sync(0xffffffffu, vh, rh & 31));
	return nd;
}

// Reference src/replace.cuh:111-153 for one pixel, by the whole warp: the
// median of the donors in the clipped (2r+1)^2 window, r = 2, 3, ... until a
// donor exists; lane 0 writes it.  Returns r (0: the frame has no donor).
__device__ __forceinline__ int replace_one(const FrameDesc &fd, int x, int y, bool *changed = nullptr)
{
	const int lane = threadIdx.x & 31;
	const int w = fd.w, h = fd.h, words = fd.words;
	const uint32_t *don = plane_ptr(fd, P_DONOR), *crm = plane_ptr(fd, P_CRMASK);
	const int limit = max(w, h);
	for (int r = 2; r <= limit; ++r) {
		Window win = {max(0, x - r), min(w - 1, x + r), max(0, y - r), min(h - 1, y + r)};
		const int ww = win.x1 - win.x0 + 1, area = ww * (win.y1 - win.y0 + 1);
		double lo, hi;
		int nd;
		if (area <= 32) {
			bool d = false;
			double v = INFINITY;
			if (lane < area) {
				// The value loads with the donor bits and is dropped for a
				// non-donor (whose pixel another warp may be writing).
				int cx = win.x0 + lane % ww, cy = win.y0 + lane / ww;
				const double c = fd.clean[(long long)cy * w + cx];
				d = donor_at(don, crm, words, cx, cy);
				if (d)
					v = c;
			}
			nd = __popc(__ballot_sync(0xffffffffu, d));
			if (!nd)
				continue;
			v = bitonic32(v);
			lo = __shfl_sync(0xffffffffu, v, (nd - 1) / 2);
			hi = __shfl_sync(0xffffffffu, v, nd / 2);
		} else if (area <= 64) {
			nd = sorted_window_median<2>(fd, don, crm, win, lo, hi);
			if (!nd)
				continue;
		} else if (area <= 128) {
			nd = sorted_window_median<4>(fd, don, crm, win, lo, hi);
			if (!nd)
				continue;
		} else {
			int cnt = 0;
			for (int pos = lane; pos < area; pos += 32)
				cnt += donor_at(don, crm, words, win.x0 + pos % ww, win.y0 + pos / ww);
			nd = warp_sum_int(cnt);
			if (!nd)
				continue;
			lo = select_rank(fd, don, crm, win, (nd - 1) / 2);
			hi = nd % 2 ? lo : select_rank(fd, don, crm, win, nd / 2);
		}
		if (lane == 0) {
			const double v = nd % 2 ? 0.0 + lo : midpoint(lo, hi);
			double &dst = fd.clean[(long long)y * w + x];
			if (changed)
				*changed = __double_as_longlong(dst) != __double_as_longlong(v);
			dst = v;
			// Keep the block's floor a lower bound of its clean values.
			if (fd.floors && !fd.error)
				atomicMin(&fd.floors[(y >> 5) * ((w + 31) >> 5) + (x >> 5)].key, order_key(v));
		}
		return r;
	}
	return 0;
}

// Largest window radius whose FRESH neighbourhood replace_kernel inspects.
constexpr int KEEP_RADIUS_MAX = 15;

// Any FRESH pixel in the (2r + 1)^2 window of (x, y) clipped to the frame
// (r <= KEEP_RADIUS_MAX: a window row spans at most two bit words).
__device__ __forceinline__ bool fresh_in_window(const FrameDesc &fd, int x, int y, int r)
{
	const uint32_t *fr = plane_ptr(fd, P_FRESH);
	const int x0 = max(0, x - r), x1 = min(fd.w - 1, x + r);
	const int k0 = x0 >> 5, k1 = x1 >> 5;
	const unsigned long long span = ((1ull << (x1 - x0 + 1)) - 1ull) << (x0 & 31);
	const int ya = max(0, y - r), yb = min(fd.h - 1, y + r);
	const uint32_t *c0 = fr + (long long)ya * fd.words + k0;
	const int dk = k1 - k0; // 0 or 1
	unsigned long long any = 0;
#pragma unroll 4
	for (int i = 0; i <= yb - ya; ++i) { // independent loads, no early exit
		const uint32_t *c = c0 + (long long)i * fd.words;
		any |= (c[0] | (unsigned long long)c[dk] << 32) & span;
	}
	return any != 0;
}

// Which targets the replacement after a pass must visit, for frames whose
// pass flagged new pixels: a lane per target; the indices of those to visit
// are appended to `sel` (count in ctl->n_sel).  The same threads first zero
// `clear` (n16 16-byte words: the CHG row marks, which this pass has read
// and the replacement that follows sets).
//
// radius keeps, per target, the window radius of its last replacement.  A
// target whose last window (radius r <= KEEP_RADIUS_MAX) holds no pixel the
// last growth step flagged keeps its value: donors are never added (the mask
// only grows) and keep their values, so the smaller windows still hold none,
// the same window holds the same donors, and the same median would come out.
// A new target is itself a flagged pixel.
__global__ void __launch_bounds__(256)
replace_select_kernel(const FrameDesc *__restrict__ frames, const FrameState *__restrict__ state,
	const uint2 *__restrict__ list, const unsigned long long *count,
	const uint8_t *__restrict__ radius, Control *ctl, unsigned *sel, uint4 *clear, long long n16)
{
	const int lane = threadIdx.x & 31;
	const long long n = (long long)*count;
	const long long stride = (long long)gridDim.x * blockDim.x;
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n16; i += stride)
		clear[i] = make_uint4(0u, 0u, 0u, 0u);
	for (long long base = blockIdx.x * (long long)blockDim.x + (threadIdx.x & ~31); base < n;
	     base += stride) {
		const long long e = base + lane;
		bool todo = false;
		if (e < n) {
			const uint2 t = list[e];
			if (state[t.x].replace) {
				todo = true;
				const int r = radius[e];
				if (r <= KEEP_RADIUS_MAX) {
					const FrameDesc &fd = frames[t.x];
					todo = fresh_in_window(fd, (int)(t.y % (unsigned)fd.w), (int)(t.y / (unsigned)fd.w), r);
				}
			}
		}
		const unsigned b = __ballot_sync(0xffffffffu, todo);
		unsigned at = 0;
		if (lane == 0 && b)
			at = atomicAdd(&ctl->n_sel, (unsigned)__popc(b));
		at = __shfl_sync(0xffffffffu, at, 0);
		if (todo)
			sel[at + __popc(b & ((1u << lane) - 1u))] = (unsigned)e;
	}
}

// Bits of columns x - 2 .. x + 2 of row y of a bit plane (bit i: column
// x - 2 + i; columns outside the frame read as zero: the words' padding bits
// are zero, and words before the row's first or after its last read as zero).
__device__ __forceinline__ uint32_t bits5(const uint32_t *plane, int words, int x, int y)
{
	const int a = x - 2, k = a >> 5; // k >= -1
	const uint32_t *row = plane + (long long)y * words;
	const uint32_t lo = k >= 0 ? row[k] : 0u, hi = k + 1 < words ? row[k + 1] : 0u;
	return (uint32_t)((((unsigned long long)hi << 32) | lo) >> (a - 32 * k)) & 0x1fu;
}

// replace_one's first window (radius 2, clipped to the frame: at most 25
// cells) evaluated by one thread: the donor bits of its five rows, the
// donors' values, a sorting network over the 25 cells (non-donors as +inf)
// and the same median (rank (nd - 1) / 2, or the midpoint of ranks
// (nd - 1) / 2 and nd / 2).  Equal nonzero donors are the same bits, and an
// odd count's 0.0 + lo drops a zero's sign, so any sort gives the bits of
// replace_one's exchange network except when an even count's two middle
// values are zeros and the window holds zeros of both signs.  Returns false
// for that window and for one without a donor: the caller's warp then runs
// replace_one (the exchange network, expanding windows).
__device__ __forceinline__ bool first_window_value(const FrameDesc &fd, int x, int y, double &out)
{
	const int w = fd.w, h = fd.h, words = fd.words;
	const uint32_t *don = plane_ptr(fd, P_DONOR), *crm = plane_ptr(fd, P_CRMASK);
	uint32_t rb[5];
	int nd = 0;
#pragma unroll
	for (int dy = 0; dy < 5; ++dy) {
		const int yy = y - 2 + dy;
		rb[dy] = yy >= 0 && yy < h ? bits5(don, words, x, yy) & ~bits5(crm, words, x, yy) : 0u;
		nd += __popc(rb[dy]);
	}
	if (nd == 0)
		return false;
	double v[25];
	bool pz = false, nz = false; // donors of +0 and of -0
#pragma unroll
	for (int c = 0; c < 25; ++c) {
		const int dy = c / 5, dx = c % 5;
		v[c] = INFINITY;
		if ((rb[dy] >> dx) & 1u) {
			v[c] = fd.clean[(long long)(y - 2 + dy) * w + (x - 2 + dx)];
			pz |= v[c] == 0 && !signbit(v[c]);
			nz |= v[c] == 0 && signbit(v[c]);
		}
	}
	sort_network(v);
	const int k1 = (nd - 1) / 2, k2 = nd / 2;
	double lo = 0, hi = 0;
#pragma unroll
	for (int c = 0; c < 25; ++c) {
		lo = c == k1 ? v[c] : lo;
		hi = c == k2 ? v[c] : hi;
	}
	if (!(nd % 2) && lo == 0 && hi == 0 && pz && nz)
		return false;
	out = nd % 2 ? 0.0 + lo : midpoint(lo, hi);
	return true;
}

// The bookkeeping of a target's replacement: its window radius, and with
// fd.rowchg, when its value changed (bit for bit), its CHG bit and its row
// mark (the next incremental pass starts from those pixels).
__device__ __forceinline__ void replaced(const FrameDesc &fd, int x, int y, long long e, int r, bool changed,
	uint8_t *radius)
{
	if (radius)
		radius[e] = (uint8_t)(r < 255 ? r : 255);
	if (changed && fd.rowchg) {
		atomicOr(plane_ptr(fd, P_CHG) + (long long)y * fd.words + (x >> 5), 1u << (x & 31));
		fd.rowchg[y] = 1u;
	}
}

// Items the thread path of a block leaves, replaced by all of its warps.
struct WindowQueue {
	long long e[256];
	int n;
};

// Replacement after a pass (src/replace.cuh:111-153): the targets listed in
// sel (with radius: each replacement's window radius is kept), or with sel
// null every target of the frames whose pass flagged new pixels.  A thread
// per target evaluates its first window (first_window_value); the targets it
// leaves (windows inside a cluster of flagged pixels) are queued in shared
// memory and the block's warps replace them with replace_one, spread over all
// eight warps so that a cluster does not hold one warp for many targets.
// Targets are in the mask, so never donors: no target reads another's value.
__global__ void __launch_bounds__(256)
replace_kernel(const FrameDesc *__restrict__ frames, const FrameState *__restrict__ state,
	const uint2 *__restrict__ list, const unsigned long long *count, const unsigned *sel,
	const unsigned *nsel, uint8_t *radius)
{
	__shared__ WindowQueue Q;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
	const long long n = sel ? (long long)*nsel : (long long)*count;
	const long long stride = (long long)gridDim.x * blockDim.x;
	if (threadIdx.x == 0)
		Q.n = 0;
	__syncthreads();
	for (long long base = blockIdx.x * (long long)blockDim.x; base < n; base += stride) { // block-uniform
		const long long s = base + threadIdx.x;
		if (s < n) {
			const long long e = sel ? (long long)sel[s] : s;
			const uint2 t = list[e];
			if (sel || state[t.x].replace) {
				const FrameDesc &fd = frames[t.x];
				const int x = (int)(t.y % (unsigned)fd.w), y = (int)(t.y / (unsigned)fd.w);
				double v;
				if (first_window_value(fd, x, y, v)) {
					double &dst = fd.clean[(long long)y * fd.w + x];
					const bool ch = __double_as_longlong(dst) != __double_as_longlong(v);
					dst = v;
					// Keep the block's floor a lower bound of its clean values.
					if (fd.floors && !fd.error)
						atomicMin(&fd.floors[(y >> 5) * ((fd.w + 31) >> 5) + (x >> 5)].key, order_key(v));
					replaced(fd, x, y, e, 2, ch, radius);
				} else {
					Q.e[atomicAdd(&Q.n, 1)] = e;
				}
			}
		}
		__syncthreads();
		const int nq = Q.n;
		for (int q = warp; q < nq; q += nwarps) {
			const long long e = Q.e[q];
			const uint2 t = list[e];
			const FrameDesc &fd = frames[t.x];
			const int x = (int)(t.y % (unsigned)fd.w), y = (int)(t.y / (unsigned)fd.w);
			bool ch = false;
			const int r = replace_one(fd, x, y, &ch);
			if (lane == 0)
				replaced(fd, x, y, e, r, ch, radius);
		}
		__syncthreads();
		if (threadIdx.x == 0)
			Q.n = 0;
		__syncthreads();
	}
}

// Initial fill of non-finite pixels (src/cleaner.cuh:78-100) for frames with
// a finite donor, from the hole list prepare wrote (holes are never donors, so
// the order does not matter): a thread per hole (first_window_value), the
// block's warps for the holes it leaves (replace_kernel's queue).
__global__ void __launch_bounds__(256)
fill_list_kernel(const FrameDesc *__restrict__ frames, const FrameState *__restrict__ state,
	const uint2 *__restrict__ holes, const unsigned long long *count)
{
	__shared__ WindowQueue Q;
	const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
	const long long n = (long long)*count;
	const long long stride = (long long)gridDim.x * blockDim.x;
	if (threadIdx.x == 0)
		Q.n = 0;
	__syncthreads();
	for (long long base = blockIdx.x * (long long)blockDim.x; base < n; base += stride) { // block-uniform
		const long long e = base + threadIdx.x;
		if (e < n) {
			const uint2 t = holes[e];
			if (state[t.x].finite) {
				const FrameDesc &fd = frames[t.x];
				const int x = (int)(t.y % (unsigned)fd.w), y = (int)(t.y / (unsigned)fd.w);
				double r;
				if (first_window_value(fd, x, y, r)) {
					fd.clean[(long long)y * fd.w + x] = r;
					// Keep the block's floor a lower bound of its clean values.
					if (fd.floors && !fd.error)
						atomicMin(&fd.floors[(y >> 5) * ((fd.w + 31) >> 5) + (x >> 5)].key, order_key(r));
				} else {
					Q.e[atomicAdd(&Q.n, 1)] = e;
				}
			}
		}
		__syncthreads();
		const int nq = Q.n;
		for (int q = warp; q < nq; q += nwarps) {
			const uint2 t = holes[Q.e[q]];
			const FrameDesc &fd = frames[t.x];
			replace_one(fd, (int)(t.y % (unsigned)fd.w), (int)(t.y / (unsigned)fd.w));
		}
		__syncthreads();
		if (threadIdx.x == 0)
			Q.n = 0;
		__syncthreads();
	}
}

// The same fill without a hole list: one warp per row scans the row's HOLE
// words.
__global__ void __launch_bounds__(256)
fill_kernel(const FrameDesc *__restrict__ frames, const FrameState *__restrict__ state,
	const int2 *__restrict__ rows, int nrows)
{
	const int lane = threadIdx.x & 31;
	const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
	for (int ri = gw; ri < nrows; ri += nw) {
		const int2 item = rows[ri];
		const FrameState &st = state[item.x];
		if (!st.holes || !st.finite)
			continue; // warp-uniform
		const FrameDesc &fd = frames[item.x];
		const uint32_t *hp = plane_ptr(fd, P_HOLE) + (long long)item.y * fd.words;
		for (int k0 = 0; k0 < fd.words; k0 += 32) {
			const uint32_t hw = k0 + lane < fd.words ? hp[k0 + lane] : 0u;
			for (unsigned m = __ballot_sync(0xffffffffu, hw != 0); m; m &= m - 1) {
				const int j = __ffs(m) - 1;
				for (uint32_t bits = __shfl_sync(0xffffffffu, hw, j); bits; bits &= bits - 1)
					replace_one(fd, 32 * (k0 + j) + __ffs(bits) - 1, item.y);
			}
		}
	}
}

// Reference src/image.cuh:50-70, in place: clean -= bg, non-finite inputs
// restored bit for bit, uint8 mask from the bit plane.  Without a background
// the clean pixels are already the output and are not rewritten.
__global__ void __launch_bounds__(256)
restore_kernel(const FrameDesc *__restrict__ frames, const int2 *__restrict__ rows, int nrows)
{
	const int lane = threadIdx.x & 31;
	const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
	for (int r = gw; r < nrows; r += nw) {
		const int2 item = rows[r];
		const FrameDesc &fd = frames[item.x];
		// Descriptor fields in registers (the stores below could alias it).
		const int w = fd.w, y = item.y, words = fd.words;
		const uint32_t *hole = plane_ptr(fd, P_HOLE) + (long long)y * words;
		const uint32_t *crm = plane_ptr(fd, P_CRMASK) + (long long)y * words;
		const long long rowpix = (long long)y * w;
		double *clean = fd.clean + rowpix;
		const double *data = fd.data + rowpix, *bgmap = fd.bg_map ? fd.bg_map + rowpix : nullptr;
		uint8_t *mask_out = fd.mask_out + rowpix;
		const double bgv = fd.bg;
		const bool has_bg = fd.has_bg;
		// A separate output buffer: prepare wrote every output pixel but the
		// flagged ones (and restored the holes).
		double *out = fd.out && fd.out != fd.clean ? fd.out + rowpix : nullptr;
		if (!has_bg || out) { // warp-uniform
			// clean (or out) already holds the output but for the flagged
			// pixels of a separate output: only the mask, those pixels and
			// the non-finite inputs are written.  Groups of 32 bit words (1024
			// pixels), two groups' words loaded before either is used; a
			// full group of an aligned row goes out as two contiguous
			// 512-byte warp stores (lane j: the 16 pixels of half (j & 1) of
			// word 16 q + j / 2), the rest byte by byte.
			const bool vec = ((uintptr_t)mask_out & 15u) == 0;
			for (int k0 = 0; k0 < words; k0 += 64) {
				uint32_t cw[2], hw[2];
#pragma unroll
				for (int g = 0; g < 2; ++g) {
					const int k = k0 + 32 * g + lane;
					cw[g] = k < words ? crm[k] : 0u;
					hw[g] = k < words ? hole[k] : 0u;
				}
#pragma unroll
				for (int g = 0; g < 2; ++g) {
					const int kb = k0 + 32 * g, k = kb + lane;
					if (kb >= words)
						break; // warp-uniform
					if (vec && 32 * (kb + 32) <= w) { // warp-uniform
#pragma unroll
						for (int q = 0; q < 2; ++q) {
							const uint32_t word = __shfl_sync(0xffffffffu, cw[g], 16 * q + (lane >> 1));
							const uint32_t half = word >> (16 * (lane & 1));
							uint32_t v[4];
#pragma unroll
							for (int b = 0; b < 4; ++b) {
								const uint32_t nib = half >> (4 * b);
								v[b] = (nib & 1u) | ((nib >> 1) & 1u) << 8 | ((nib >> 2) & 1u) << 16 |
								       ((nib >> 3) & 1u) << 24;
							}
							*reinterpret_cast<uint4 *>(mask_out + 32 * kb + 512 * q + 16 * lane) =
								make_uint4(v[0], v[1], v[2], v[3]);
						}
					} else {
						// Unaligned rows: the group's words one after
						// another, a lane per pixel (coalesced byte stores).
						const int nk = min(32, words - kb);
						for (int j = 0; j < nk; ++j) {
							const uint32_t word = __shfl_sync(0xffffffffu, cw[g], j);
							const int x = 32 * (kb + j) + lane;
							if (x < w)
								mask_out[x] = (word >> lane) & 1u;
						}
					}
					if (out) {
						for (uint32_t fb = cw[g]; fb; fb &= fb - 1) {
							const int x = 32 * k + __ffs(fb) - 1;
							out[x] = clean[x] + -1 * (bgmap ? bgmap[x] : bgv);
						}
					} else {
						for (uint32_t hb = hw[g]; hb; hb &= hb - 1) {
							const int x = 32 * k + __ffs(hb) - 1;
							clean[x] = data[x];
						}
					}
				}
			}
			continue;
		}
		for (int xb = 0; xb < w; xb += 32 * ROW_UNROLL) {
			double v[ROW_UNROLL], bg[ROW_UNROLL];
			uint32_t hb[ROW_UNROLL], cb[ROW_UNROLL];
#pragma unroll
			for (int u = 0; u < ROW_UNROLL; ++u) {
				const int x = xb + 32 * u + lane;
				v[u] = 0;
				bg[u] = bgv;
				hb[u] = cb[u] = 0;
				if (x < w) {
					v[u] = clean[x];
					hb[u] = hole[x >> 5];
					cb[u] = crm[x >> 5];
					if (bgmap)
						bg[u] = bgmap[x];
				}
			}
#pragma unroll
			for (int u = 0; u < ROW_UNROLL; ++u) {
				const int x = xb + 32 * u + lane;
				if (x < w) {
					double o = v[u];
					if (has_bg)
						o += -1 * bg[u];
					if ((hb[u] >> (x & 31)) & 1u)
						o = data[x];
					clean[x] = o;
					mask_out[x] = (cb[u] >> (x & 31)) & 1u;
				}
			}
		}
	}
}

// maxiter == 0 (reference src/image.cuh:72-92): background round trip only.
__global__ void __launch_bounds__(256)
copy_kernel(const FrameDesc *__restrict__ frames, const int2 *__restrict__ rows, int nrows)
{
	const int lane = threadIdx.x & 31;
	const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
	for (int r = gw; r < nrows; r += nw) {
		const int2 item = rows[r];
		const FrameDesc &fd = frames[item.x];
		const long long rowpix = (long long)item.y * fd.w;
		for (int x = lane; x < fd.w; x += 32) {
			const long long i = rowpix + x;
			const double d = fd.data[i];
			double v = isfinite(d) ? d : 0;
			if (fd.has_bg) {
				double bg = fd.bg_map ? fd.bg_map[i] : fd.bg;
				v += 1 * bg;
				v += -1 * bg;
			}
			fd.clean[i] = isfinite(d) ? v : d;
			fd.mask_out[i] = 0;
		}
	}
}

// Up to four copies of 8-byte words between any memory the device can
// address, page-locked host memory included (read or written over the bus by
// the kernel itself, so no copy engine is involved).
struct WordCopy {
	const unsigned long long *src;
	unsigned long long *dst;
	long long n8;
};

struct WordCopies {
	WordCopy part[6];
	int n;
};

__global__ void __launch_bounds__(256)
word_copy_kernel(WordCopies c)
{
	const long long stride = (long long)gridDim.x * blockDim.x;
	for (int k = 0; k < c.n; ++k)
		for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < c.part[k].n8; i += stride)
			c.part[k].dst[i] = c.part[k].src[i];
}

// The cleaned values of the listed targets (the cumulative mask as
// {frame, pixel}): vals[i] = clean of target i.  Without a background every
// other output pixel equals its input bit for bit, so these values and the
// list are all of a frame's result that differs from its input.
__global__ void __launch_bounds__(256)
gather_targets_kernel(const FrameDesc *__restrict__ frames, const uint2 *__restrict__ list,
	const unsigned long long *count, double *vals)
{
	const unsigned long long n = *count, stride = (unsigned long long)gridDim.x * blockDim.x;
	for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
	     i += stride) {
		const uint2 t = list[i];
		vals[i] = frames[t.x].clean[t.y];
	}
}

} // namespace cb

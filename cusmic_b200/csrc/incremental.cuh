// Incremental detection passes (every pass after the first).
//
// A pass of the reference (src/cleaner.cuh:102-142) recomputes the whole
// detection chain on the current clean pixels, and between two passes only
// the pixels that the replacement wrote change.  Every quantity of the chain
// at a pixel p reads clean pixels within a fixed Chebyshev distance of p,
// measured in the frame (mirror, reflect and nearest map a window position
// onto an in-frame pixel no farther from p; constant reads a zero) or on the
// torus (wrap):
//
//   sig_raw = lap / (2 noise)       distance 2 (lap 1, noise-model median 2)
//   sig = sig_raw - med5(sig_raw)   distance 4
//   fine = med3 -> med7             distance 4
//   S1, S2, CAND                    distance 4
//   grown pixel (two dilations)     distance 6 (S2, S1 and CAND within 2)
//
// So with D the pixels whose value the last replacement changed (the CHG
// plane and the per-row marks fd.rowchg, written by replace_kernel), pass
// k + 1 differs from pass k only near D.  An incremental pass keeps the bit
// planes of the previous one and re-evaluates that neighbourhood:
//
//  * dirty_rows_kernel: the rows within 6 of D (the dirty rows), listed;
//  * incremental_rows_kernel, per dirty row: sig_raw of every pixel within 2
//    of D, which updates the HIGH / LOW class planes (exact classes: sig_raw
//    > cr_threshold or NaN, else > neighbor_threshold; classify_kernel's
//    first-pass classes are supersets, from the Laplacian upper bound); a
//    pixel leaving HIGH loses its S1 and CAND bits (sig <= sig_raw <=
//    cr_threshold), a pixel leaving both classes its S2 bit; then the HIGH
//    pixels within 4 of D into the high list, the LOW pixels within 6 of D
//    into the low list.
//
// The row kernel dilates CHG with bit windows (one warp per row, a lane per
// bit word), so every pixel is visited once without atomics.  The candidate
// and seed kernels then run on those lists exactly as in a full pass,
// setting or clearing each bit they evaluate, and growth visits the items
// holding dirty rows (fresh pixels lie within 6 of D), clearing their CHG
// bits (replace_select_kernel clears the CHG row marks) before the
// replacement writes the next D.  What stays exact: S1 and CAND
// everywhere, S2 of every HIGH pixel and of every LOW pixel with a CAND pixel
// within 2 (the only S2 bits growth reads): a LOW pixel whose CAND
// neighbourhood changed is within 6 of D.  Outside HIGH sig <= cr_threshold,
// and a pixel outside both classes has sig <= neighbor_threshold, so its bits
// are zero.
#pragma once

#include "bulk.cuh"
#include "common.cuh"
#include "detect.cuh"
#include "kernels.cuh"

namespace cb {

static_assert(FLOOR_BLOCK == 32, "a bit word of a row lies in one floor block");

// model_threshold of block (bx, by) of a noise-model frame; outside wrap mode
// only the 3 x 3 neighbouring blocks count, read directly.
__device__ __forceinline__ double block_threshold(const FrameDesc &fd, int bx, int by, int mode,
	double tmin2)
{
	if (mode == WRAP)
		return model_threshold(fd, bx, by, mode, tmin2);
	const BlockFloor *bf = fd.floors;
	const int bw = (fd.w + FLOOR_BLOCK - 1) / FLOOR_BLOCK, bh = (fd.h + FLOOR_BLOCK - 1) / FLOOR_BLOCK;
	unsigned long long key = ~0ull;
#pragma unroll
	for (int i = -1; i <= 1; ++i)
#pragma unroll
		for (int j = -1; j <= 1; ++j) {
			const int yy = by + i, xx = bx + j;
			if (yy >= 0 && yy < bh && xx >= 0 && xx < bw)
				key = min(key, bf[yy * bw + xx].key);
		}
	if (mode == CONSTANT && (bx == 0 || by == 0 || (bx + 1) * FLOOR_BLOCK + 2 > fd.w ||
		(by + 1) * FLOOR_BLOCK + 2 > fd.h))
		key = min(key, order_key(0.0));
	double m = order_value(key);
	m = m < SIGNAL_FLOOR ? SIGNAL_FLOOR : m;
	const BlockFloor &own = bf[by * bw + bx];
	const double g = fd.gain_map ? -order_value(own.gkey) : fd.gain;
	const double rn = fd.rn_map ? order_value(own.rkey) : fd.rn;
	return tmin2 * (sqrt(rn * rn + g * m) / g);
}

__device__ __forceinline__ int wrap_index(int i, int n)
{
	i %= n;
	return i < 0 ? i + n : i;
}

// Any changed pixel in rows y - r .. y + r (on the torus for wrap).
__device__ __forceinline__ bool rows_changed(const FrameDesc &fd, int y, int r, bool wrap)
{
	bool any = false;
	for (int d = -r; d <= r; ++d) {
		const int yy = y + d;
		if (wrap)
			any |= fd.rowchg[wrap_index(yy, fd.h)] != 0;
		else if (yy >= 0 && yy < fd.h)
			any |= fd.rowchg[yy] != 0;
	}
	return any;
}

// The rows of active frames with a changed pixel within six rows, appended
// to `out` (count in ctl->n_dirty); every row of an active frame gets its
// growth mark (set on those rows, cleared on the others).  A thread per row.
// The same threads first zero `clear` (n16 16-byte words: the FRESH plane,
// which this pass's growth writes on the rows it visits and the previous
// pass's replacement has read).
__global__ void __launch_bounds__(256)
dirty_rows_kernel(const FrameDesc *__restrict__ frames, const FrameState *__restrict__ state,
	const int2 *__restrict__ rows, int nrows, int mode, Control *ctl, int2 *out, uint4 *clear,
	long long n16)
{
	const int lane = threadIdx.x & 31;
	const bool wrap = mode == WRAP;
	const int stride = gridDim.x * blockDim.x;
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n16; i += stride)
		clear[i] = make_uint4(0u, 0u, 0u, 0u);
	for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < nrows; base += stride) {
		const int i = base + lane;
		int2 item = make_int2(0, 0);
		bool keep = false;
		if (i < nrows) {
			item = rows[i];
			if (state[item.x].active) {
				const FrameDesc &fd = frames[item.x];
				keep = rows_changed(fd, item.y, 6, wrap);
				fd.rowcand[item.y] = keep; // replaces the last pass's marks
			}
		}
		const unsigned b = __ballot_sync(0xffffffffu, keep);
		int at = 0;
		if (lane == 0 && b)
			at = atomicAdd(&ctl->n_dirty, __popc(b));
		at = __shfl_sync(0xffffffffu, at, 0);
		if (keep)
			out[at + __popc(b & ((1u << lane) - 1u))] = item;
	}
}

// Pixels of a bit word of a row within Chebyshev distance 2, 4 and 6 of a
// changed pixel, restricted to the frame.
struct NearMasks {
	uint32_t r2, r4, r6;
};

__device__ __forceinline__ uint32_t dilate_window(unsigned long long win, int r)
{
	// win bit i: column 32k - 6 + i; result bit j: column 32k + j.
	unsigned long long m = 0;
	for (int s = -r; s <= r; ++s)
		m |= win >> (6 + s);
	return (uint32_t)m;
}

// Called by the whole warp for the words k0 + lane of row y (zero past the
// row): vertical ORs of CHG over rows within 2, 4 and 6 (on the torus for
// wrap, clipped otherwise) per word, the neighbouring words' ORs by shuffle
// (the words left and right of the segment loaded one row per lane), then
// horizontal dilation of 44-bit windows.
__device__ __forceinline__ NearMasks near_changed(const FrameDesc &fd, int y, int k0, bool wrap)
{
	const int lane = threadIdx.x & 31;
	const int w = fd.w, h = fd.h, words = fd.words, k = k0 + lane, x0 = 32 * k;
	const uint32_t *chg = plane_ptr(fd, P_CHG);
	auto row_of = [&](int d) {
		int yy = y + d;
		if (wrap)
			yy = wrap_index(yy, h);
		return yy >= 0 && yy < h ? yy : -1;
	};
	uint32_t a = 0, b = 0, c = 0; // rows within 2, 3..4 and 5..6 of y
	if (k < words) {
#pragma unroll
		for (int d = -6; d <= 6; ++d) {
			const int yy = row_of(d);
			const uint32_t v = yy >= 0 ? chg[(long long)yy * words + k] : 0u;
			const int t = d < 0 ? -d : d;
			if (t <= 2)
				a |= v;
			else if (t <= 4)
				b |= v;
			else
				c |= v;
		}
	}
	// Halo words k0 - 1 (lanes 0..12, row y - 6 + lane) and k0 + 32 (lanes
	// 16..28); zero outside the row.
	uint32_t hv = 0;
	int ht = 7;
	{
		const int side = lane >> 4, d = (lane & 15) - 6;
		const int hk = side ? k0 + 32 : k0 - 1;
		if (d <= 6 && hk >= 0 && hk < words) {
			const int yy = row_of(d);
			hv = yy >= 0 ? chg[(long long)yy * words + hk] : 0u;
			ht = d < 0 ? -d : d;
		}
	}
	const uint32_t la2 = __reduce_or_sync(0xffffffffu, lane < 16 && ht <= 2 ? hv : 0u);
	const uint32_t la4 = __reduce_or_sync(0xffffffffu, lane < 16 && ht > 2 && ht <= 4 ? hv : 0u);
	const uint32_t la6 = __reduce_or_sync(0xffffffffu, lane < 16 && ht > 4 && ht <= 6 ? hv : 0u);
	const uint32_t ra2 = __reduce_or_sync(0xffffffffu, lane >= 16 && ht <= 2 ? hv : 0u);
	const uint32_t ra4 = __reduce_or_sync(0xffffffffu, lane >= 16 && ht > 2 && ht <= 4 ? hv : 0u);
	const uint32_t ra6 = __reduce_or_sync(0xffffffffu, lane >= 16 && ht > 4 && ht <= 6 ? hv : 0u);
	uint32_t l[3] = {__shfl_up_sync(0xffffffffu, a, 1), __shfl_up_sync(0xffffffffu, b, 1),
		__shfl_up_sync(0xffffffffu, c, 1)};
	uint32_t r[3] = {__shfl_down_sync(0xffffffffu, a, 1), __shfl_down_sync(0xffffffffu, b, 1),
		__shfl_down_sync(0xffffffffu, c, 1)};
	if (lane == 0) {
		l[0] = la2;
		l[1] = la4;
		l[2] = la6;
	}
	if (lane == 31) {
		r[0] = ra2;
		r[1] = ra4;
		r[2] = ra6;
	}
	if (k >= words)
		return NearMasks{0u, 0u, 0u};
	auto window = [](uint32_t lv, uint32_t mv, uint32_t rv) {
		return ((unsigned long long)lv >> 26) | ((unsigned long long)mv << 6) |
		       (((unsigned long long)rv & 0x3full) << 38);
	};
	unsigned long long w2 = window(l[0], a, r[0]);            // bit i: column x0 - 6 + i
	unsigned long long w4 = w2 | window(l[1], b, r[1]);
	unsigned long long w6 = w4 | window(l[2], c, r[2]);
	if (wrap && !(k > 0 && x0 + 38 <= w)) {
		// Window across the frame's edge on the torus: column by column.
		w2 = w4 = w6 = 0;
		for (int i = 0; i < 44; ++i) {
			const int x = wrap_index(x0 - 6 + i, w);
			int best = 7;
			for (int d = -6; d <= 6; ++d) {
				const int t = d < 0 ? -d : d;
				if (t < best &&
				    ((chg[(long long)wrap_index(y + d, h) * words + (x >> 5)] >> (x & 31)) & 1u))
					best = t;
			}
			w2 |= (unsigned long long)(best <= 2) << i;
			w4 |= (unsigned long long)(best <= 4) << i;
			w6 |= (unsigned long long)(best <= 6) << i;
		}
	}
	const uint32_t clip = x0 + 32 > w ? (1u << (w - x0)) - 1u : 0xffffffffu;
	return NearMasks{dilate_window(w2, 2) & clip, dilate_window(w4, 4) & clip,
		dilate_window(w6, 6) & clip};
}

// Reclassification and work-list gather of one incremental pass, one warp per
// row of the dirty list (rows within six of a changed pixel) whose frame has
// an error map (MODEL false) or uses the noise model (MODEL true).  Per
// segment of 32 words:
//  * the pixels within 2 of a changed pixel are queued in shared memory and
//    their sig_raw evaluated 32 at a time (on noise-model frames only those
//    that pass the block's noise-floor bound); the lane owning each word
//    writes its HIGH / LOW words and clears S1, CAND (left HIGH) and S2 (left
//    both);
//  * HIGH pixels within 4 go to the high list (front of `cands`), LOW pixels
//    within 6 to the low list (back).
// A row's classes are all this needs from the pass, so no other row waits.
template <bool MODEL>
__global__ void __launch_bounds__(256, 4)
incremental_rows_kernel(const FrameDesc *__restrict__ frames, const int2 *__restrict__ rows,
	const int *nrows, DetectParams prm, Control *ctl, uint2 *cands)
{
	constexpr int STG = 128; // staged list entries per warp and list
	__shared__ uint16_t queue[8][1024];
	__shared__ uint32_t hmask[8][32], lmask[8][32];
	__shared__ double thr[MODEL ? 8 : 1][32];
	__shared__ uint2 staged[8][2][STG];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
	const int mode = prm.mode, lm = lap_mode(mode);
	const bool wrap = mode == WRAP;
	const double tmin2 = fmin(prm.thi2, prm.tlo2);
	const unsigned long long cap = ctl->cand_cap;
	const int n = *nrows;
	uint16_t *Q = queue[warp];
	// List entries are staged per warp and written out with one atomic per
	// flush (list 0: high, from the front; list 1: low, from the back).
	int nst[2] = {0, 0};
	auto flush = [&](int li) {
		__syncwarp();
		unsigned long long b0 = 0;
		if (lane == 0)
			b0 = atomicAdd(li ? &ctl->n_low : &ctl->n_cand, (unsigned long long)nst[li]);
		b0 = __shfl_sync(0xffffffffu, b0, 0);
		for (int i = lane; i < nst[li]; i += 32)
			cands[li ? cap - 1 - (b0 + i) : b0 + i] = staged[warp][li][i];
		nst[li] = 0;
		__syncwarp();
	};
	auto emit = [&](int li, uint32_t bits, unsigned f, unsigned base) {
		const int c = __popc(bits), o = warp_exclusive_count(c);
		const int t = __shfl_sync(0xffffffffu, o + c, 31);
		if (!t)
			return;
		if (nst[li] + t > STG)
			flush(li);
		if (t > STG) { // a segment with more entries than the stage holds
			unsigned long long slot = warp_append(li ? &ctl->n_low : &ctl->n_cand, c);
			for (; bits; bits &= bits - 1, ++slot)
				cands[li ? cap - 1 - slot : slot] = make_uint2(f, base + __ffs(bits) - 1);
			return;
		}
		int at = nst[li] + o;
		for (; bits; bits &= bits - 1)
			staged[warp][li][at++] = make_uint2(f, base + __ffs(bits) - 1);
		nst[li] += t;
	};
	for (int ri = gw; ri < n; ri += nw) {
		const int2 item = rows[ri];
		const FrameDesc &fd = frames[item.x];
		if ((fd.error == nullptr) != MODEL)
			continue; // warp-uniform
		const int w = fd.w, y = item.y, words = fd.words;
		for (int k0 = 0; k0 < words; k0 += 32) {
			const int k = k0 + lane;
			const long long o = (long long)y * words + k;
			uint32_t *H = plane_ptr(fd, P_HIGH) + o, *L = plane_ptr(fd, P_LOW) + o;
			uint32_t nh = 0, nl = 0;
			if (k < words) { // loaded with the CHG words, before they are needed
				nh = *H;
				nl = *L;
			}
			const NearMasks nm = near_changed(fd, y, k0, wrap);
			const int cnt = __popc(nm.r2), off = warp_exclusive_count(cnt);
			const int total = __shfl_sync(0xffffffffu, off + cnt, 31);
			if (total) { // warp-uniform
				int pos = off;
				for (uint32_t b = nm.r2; b; b &= b - 1)
					Q[pos++] = (uint16_t)((lane << 5) | (__ffs(b) - 1));
				hmask[warp][lane] = lmask[warp][lane] = 0u;
				int todo = total;
				if (MODEL) {
					// Noise-model bound of each word's 32 x 32 block (the dense
					// kernel's superset test): lap <= T gives sig_raw below both
					// thresholds without the pixel's 5 x 5 median.  The pixels
					// that pass are compacted to the front of the queue.
					thr[warp][lane] = nm.r2 ? block_threshold(fd, k, y / FLOOR_BLOCK, mode, tmin2) : 0.0;
					__syncwarp();
					todo = 0;
					for (int q0 = 0; q0 < total; q0 += 32) {
						int e = 0;
						bool keep = false;
						if (q0 + lane < total) {
							e = Q[q0 + lane];
							const int px = 32 * (k0 + (e >> 5)) + (e & 31);
							const double lap = lap_at(fd, px, y, lm);
							const double T = thr[warp][e >> 5];
							keep = !(T >= 0 && lap <= T);
						}
						const unsigned kb = __ballot_sync(0xffffffffu, keep);
						if (keep)
							Q[todo + __popc(kb & ((1u << lane) - 1u))] = (uint16_t)e;
						todo += __popc(kb);
					}
				}
				__syncwarp();
				if (MODEL) {
					// Exact sig_raw of each pixel that passed, one at a time: its
					// 5 x 5 window of clean one cell per lane, sorted across the
					// warp (+inf padding), the median at rank 12.  The next
					// pixel's window loads before this one's sort (one memory
					// round trip per pixel hidden behind the previous sort), and
					// an interior pixel's Laplacian comes from the window.
					auto window_cell = [&](int q) {
						double c = INFINITY;
						if (q < todo && lane < 25) {
							const int e = Q[q], px = 32 * (k0 + (e >> 5)) + (e & 31);
							const int cx = px + lane % 5 - 2, cy = y + lane / 5 - 2;
							c = cx >= 0 && cy >= 0 && cx < w && cy < fd.h
								? fd.clean[(long long)cy * w + cx] : clean_at(fd, cx, cy, mode);
						}
						return c;
					};
					double cur = window_cell(0);
					for (int q = 0; q < todo; ++q) {
						const double next = window_cell(q + 1);
						const int e = Q[q], kk = e >> 5, bit = e & 31;
						const int px = 32 * (k0 + kk) + bit;
						const double ce = __shfl_sync(0xffffffffu, cur, 12);
						const double up = __shfl_sync(0xffffffffu, cur, 7);
						const double dn = __shfl_sync(0xffffffffu, cur, 17);
						const double lf = __shfl_sync(0xffffffffu, cur, 11);
						const double rt = __shfl_sync(0xffffffffu, cur, 13);
						const double m = __shfl_sync(0xffffffffu, warp_sort32(cur), 12);
						if (lane == 0) {
							const long long i = (long long)y * w + px;
							// Interior: the four neighbours are in the frame, so
							// the window holds the values lap_at reads.
							const double lap = px >= 1 && y >= 1 && px + 1 < w && y + 1 < fd.h
								? lap_formula(ce, up, dn, lf, rt) : lap_at(fd, px, y, lm);
							const double v = lap / (2 * noise_from_median(fd, i, m));
							if (v > prm.cr || v != v)
								hmask[warp][kk] |= 1u << bit;
							else if (v > prm.nb)
								lmask[warp][kk] |= 1u << bit;
						}
						cur = next;
					}
				} else {
					for (int q0 = 0; q0 < todo; q0 += 32) {
						if (q0 + lane < todo) {
							const int e = Q[q0 + lane], kk = e >> 5, bit = e & 31;
							const int px = 32 * (k0 + kk) + bit;
							const long long i = (long long)y * w + px;
							const double v = lap_at(fd, px, y, lm) / (2 * fd.error[i]);
							if (v > prm.cr || v != v)
								atomicOr(&hmask[warp][kk], 1u << bit);
							else if (v > prm.nb)
								atomicOr(&lmask[warp][kk], 1u << bit);
						}
					}
				}
				__syncwarp();
			}
			uint32_t hi = 0, lo = 0;
			if (nm.r6) {
				if (const uint32_t m = nm.r2) {
					const uint32_t oh = nh;
					nh = (oh & ~m) | hmask[warp][lane];
					nl = (nl & ~m) | lmask[warp][lane];
					*H = nh;
					*L = nl;
					if (const uint32_t left = oh & ~nh) {
						plane_ptr(fd, P_S1)[o] &= ~left;
						plane_ptr(fd, P_CAND)[o] &= ~left;
					}
					if (const uint32_t none = m & ~(nh | nl))
						plane_ptr(fd, P_S2)[o] &= ~none;
				}
				hi = nh & nm.r4;
				lo = nl & nm.r6;
			}
			__syncwarp(); // the queue and masks are free for the next segment
			const unsigned base = (unsigned)((long long)y * w + 32 * k);
			emit(0, hi, (unsigned)item.x, base);
			emit(1, lo, (unsigned)item.x, base);
		}
	}
	if (nst[0])
		flush(0);
	if (nst[1])
		flush(1);
}

} // namespace cb

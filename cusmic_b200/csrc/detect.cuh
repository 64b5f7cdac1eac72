// Detection pass of one L.A.Cosmic iteration.
//
// Reference chain (src/cleaner.cuh:102-126): laplacian -> [median5 ->
// noise_model] -> snr -> median5 -> significance -> median3 -> median7 ->
// fine_structure -> detect, every stage a full-frame float64 pass with 25 to
// 49 gathers per pixel.  Two exact facts about that chain let this pass read
// each pixel once and evaluate medians only where a threshold can pass:
//
//  * the Laplacian is a sum of clipped terms, so lap >= 0 and sig_raw =
//    lap / (2 noise) >= 0; hence med5(sig_raw) >= 0 and sig = sig_raw -
//    med5(sig_raw) <= sig_raw.  A pixel whose sig_raw does not exceed
//    min(cr, neighbor) (both >= 0) can set neither `sig > cr` nor
//    `sig > neighbor`, so its 5 x 5 median is never needed (NaN compares
//    false either way);
//  * fine structure (med3 -> med7) is only read by detect behind
//    `sig > cr_threshold` on a non-excluded pixel (src/filters.cuh:164-175).
//
// So a pass is three kernels:
//   A  dense and HBM-bound: a division-free, median-free test that keeps a
//      superset of the pixels whose sig_raw exceeds min(cr, neighbor), appended
//      to a candidate list, and clearing of the S1/S2/CAND bit words.  With an
//      error map (sig_stream_kernel) each warp walks a strip of 32 columns down
//      the frame with a rolling 3-row register window; with the noise model
//      (sig_model_kernel) a tile kernel bounds the noise from below by the
//      tile's minimum;
//   B  one warp per candidate: exact sig_raw over the 5 x 5 window (with the
//      exact noise model where there is no error map), its median, sig, the
//      S1/S2 bits and the candidate's seed slot;
//   C  one warp per seed: 49 3 x 3 medians, their 7 x 7 median, the contrast
//      test and the CAND bit.
// Every value that feeds a threshold is computed in the reference's operation
// order (no FMA), so the bits equal the reference's.
//
// Borders: the chained filters read intermediates at border-mapped positions
// (med7 reads med3 at border_index(x), med5 reads sig_raw there).  B and C
// fold each window position with the median's border map before evaluating
// the intermediate, except that a 3 x 3 median under mirror, reflect or wrap
// is evaluated directly on border-extended clean pixels: those border maps
// are invariant under a group of isometries that folds any coordinate onto
// its image, so both give the same multiset.  The Laplacian itself reads its
// neighbours with nearest semantics for mirror and reflect
// (src/filters.cuh:95-97).
#pragma once
#include "common.cuh"
#include "kernels.cuh"
#include "select.cuh"

namespace cb {

struct DetectParams {
	double contrast, cr, nb;
	double tmin;   // min(cr, nb): sig_raw above it can pass a threshold
	double tloose; // tmin (1 - 1e-12): division-free superset test of kernel A
	int mode;
};

// Seed slot of candidate e (frame NO_SEED when the candidate is not a seed).
struct Seed {
	unsigned frame, pixel;
	double sig, noise;
};
constexpr unsigned NO_SEED = 0xffffffffu;

constexpr int STREAM_ROWS = 32; // rows per strip item of sig_stream_kernel
constexpr int MTILE = 32;       // square tile of sig_model_kernel
constexpr int MHALO = MTILE + 4;

__device__ __forceinline__ double positive(double v)
{
	return v < 0 ? 0 : v;
}

// Reference src/filters.cuh:98-104, same operation order.
__device__ __forceinline__ double lap_formula(double c0, double u0, double d0, double l0, double r0)
{
	double c = c0 / 4;
	double up = c - u0 / 4;
	double down = c - d0 / 4;
	double left = c - l0 / 4;
	double right = c - r0 / 4;
	return (positive(up + left) + positive(up + right)) + (positive(down + left) + positive(down + right));
}

__device__ __forceinline__ int lap_mode(int mode)
{
	return mode == MIRROR || mode == REFLECT ? NEAREST : mode;
}

// clean at (x, y) under a border mode (0 outside for constant).
__device__ __forceinline__ double clean_at(const FrameDesc &fd, int x, int y, int mode)
{
	int mx = border_index(x, fd.w, mode), my = border_index(y, fd.h, mode);
	return mx < 0 || my < 0 ? 0.0 : fd.clean[(long long)my * fd.w + mx];
}

// Noise model at an in-frame pixel from its 5 x 5 median of clean
// (src/filters.cuh:107-123).
__device__ __forceinline__ double noise_from_median(const FrameDesc &fd, long long i, double m)
{
	double g = fd.gain_map ? fd.gain_map[i] : fd.gain;
	double rn = fd.rn_map ? fd.rn_map[i] : fd.rn;
	m = m < SIGNAL_FLOOR ? SIGNAL_FLOOR : m;
	return sqrt(rn * rn + g * m) / g;
}

__device__ __forceinline__ void clear_detect_words(const FrameDesc &fd, long long word, int lane)
{
	if (lane < 3)
		plane_ptr(fd, P_S1 + lane)[word] = 0u;
}

// A, error-map frames: one warp per item {frame, x0, y0}: 32 columns from x0,
// rows y0 .. y0 + STREAM_ROWS - 1, in sub-blocks of STREAM_SUB rows whose
// loads are all issued before any is used (enough bytes in flight per SM to
// approach HBM bandwidth).  The rows above and below stay in registers and
// the left and right neighbours come from adjacent lanes.
//
// This kernel only has to find a superset of {sig_raw > tmin}: B evaluates
// sig_raw exactly for every candidate and drops the others.  So instead of
// dividing it tests lap > thr * (2 noise) with thr = tmin (1 - 1e-12) (prm.
// tloose): the product is rounded by at most 2^-53 relative, so every pixel
// with fl(lap / (2 noise)) > tmin passes (and NaN, infinite or zero noise
// give the same outcome as the division).
constexpr int STREAM_SUB = 8;

// Append the candidates of one strip item (lane = column, bit k of `rows` =
// row y0 + k) with a single atomic per item.
__device__ __forceinline__ void stream_flush(int f, int w, int x, int y0, uint32_t rows,
	Control *ctl, uint2 *cands)
{
	if (!__any_sync(0xffffffffu, rows != 0))
		return;
	unsigned long long slot = warp_append(&ctl->n_cand, __popc(rows));
	while (rows) {
		const int k = __ffs(rows) - 1;
		rows &= rows - 1;
		cands[slot++] = make_uint2((unsigned)f, (unsigned)((long long)(y0 + k) * w + x));
	}
}

__global__ void __launch_bounds__(256, 2)
sig_stream_kernel(const FrameDesc *__restrict__ frames, const FrameState *__restrict__ state,
	const int4 *__restrict__ items, int nitems, DetectParams prm, Control *ctl, uint2 *cands)
{
	const int lane = threadIdx.x & 31;
	const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
	const int lm = lap_mode(prm.mode);
	const double thr = prm.tloose;
	for (int it = gw; it < nitems; it += nw) {
		const int4 item = items[it];
		if (!state[item.x].active)
			continue; // warp-uniform
		const FrameDesc &fd = frames[item.x];
		const int w = fd.w, h = fd.h, words = fd.words;
		const int x0 = item.y, y0 = item.z, y1 = min(y0 + STREAM_ROWS, h);
		const int x = x0 + lane, xc = min(x, w - 1);
		const bool valid = x < w;
		// Strips away from the left/right frame edges take their halo column
		// with a plain load (lane 0: x0 - 1, lane 31: x0 + 32).
		const bool inner = x0 >= 1 && x0 + 32 < w;
		const int hx = lane == 0 ? x0 - 1 : x0 + 32;
		const double *__restrict__ clean = fd.clean, *__restrict__ err = fd.error;
		const uint32_t *holes = plane_ptr(fd, P_HOLE) + (x0 >> 5);
		double up = clean_at(fd, xc, y0 - 1, lm);
		double cur = clean[(long long)y0 * w + xc];
		uint32_t found = 0; // bit k: row y0 + k is a candidate in this lane's column
		int ys = y0;
		if (inner) {
			// Full sub-blocks with a next row inside the frame: no border logic.
			for (; ys + STREAM_SUB <= y1 && ys + STREAM_SUB < h; ys += STREAM_SUB) {
				double nxt[STREAM_SUB], nz[STREAM_SUB], halo[STREAM_SUB];
				uint32_t hw[STREAM_SUB];
				const double *crow = clean + (long long)ys * w;
				const double *erow = err + (long long)ys * w;
#pragma unroll
				for (int k = 0; k < STREAM_SUB; ++k) {
					nxt[k] = crow[(long long)(k + 1) * w + xc];
					nz[k] = erow[(long long)k * w + xc];
					hw[k] = holes[(long long)(ys + k) * words];
					halo[k] = (lane == 0 || lane == 31) ? crow[(long long)k * w + hx] : 0.0;
				}
#pragma unroll
				for (int k = 0; k < STREAM_SUB; ++k) {
					double left = __shfl_up_sync(0xffffffffu, cur, 1);
					double right = __shfl_down_sync(0xffffffffu, cur, 1);
					if (lane == 0)
						left = halo[k];
					if (lane == 31)
						right = halo[k];
					const double lap = lap_formula(cur, up, nxt[k], left, right);
					const bool c = valid && !((hw[k] >> lane) & 1u) && lap > thr * (2 * nz[k]);
					found |= (uint32_t)c << (ys + k - y0);
					clear_detect_words(fd, (long long)(ys + k) * words + (x0 >> 5), lane);
					up = cur;
					cur = nxt[k];
				}
			}
		}
		// Remaining rows, frame edges: one row at a time with border handling.
#pragma unroll 1
		for (int y = ys; y < y1; ++y) {
			const long long row = (long long)y * w;
			const double down = y + 1 < h ? clean[row + w + xc] : clean_at(fd, xc, y + 1, lm);
			const double nz = err[row + xc];
			const uint32_t hw = holes[(long long)y * words];
			double left = __shfl_up_sync(0xffffffffu, cur, 1);
			double right = __shfl_down_sync(0xffffffffu, cur, 1);
			if (lane == 0)
				left = clean_at(fd, x - 1, y, lm);
			if (lane == 31 || x + 1 >= w)
				right = clean_at(fd, x + 1, y, lm);
			const double lap = lap_formula(cur, up, down, left, right);
			const bool c = valid && !((hw >> lane) & 1u) && lap > thr * (2 * nz);
			found |= (uint32_t)c << (y - y0);
			clear_detect_words(fd, (long long)y * words + (x0 >> 5), lane);
			up = cur;
			cur = down;
		}
		stream_flush(item.x, w, x, y0, found, ctl, cands);
	}
}

// A, noise-model frames: one block per MTILE x MTILE tile with its clean
// pixels (halo 2, border-extended) in shared memory.  The noise model is
// monotone non-decreasing in the 5 x 5 median in floating point (max, g * m,
// rn^2 + ., sqrt and / g are each monotone for g > 0), and the median of a
// window is at least the minimum m_lo of the tile and its halo, so
// noise(m_lo) <= noise(med5) and lap / (2 noise(m_lo)) >= sig_raw.  The tile
// therefore tests lap > thr * (2 noise(m_lo)) with thr = tmin (1 - 1e-12): a
// superset of {sig_raw > tmin} without any median.  Scalar gain and read
// noise make noise(m_lo) one value per tile; maps evaluate it per pixel.
__global__ void __launch_bounds__(256)
sig_model_kernel(const FrameDesc *__restrict__ frames, const FrameState *__restrict__ state,
	const int4 *__restrict__ tiles, int ntiles, DetectParams prm, Control *ctl, uint2 *cands)
{
	__shared__ double C[MHALO * MHALO];
	__shared__ double wmin[8];
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int mode = prm.mode, lm = lap_mode(mode);
	const double thr = prm.tloose;
	for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
		const int4 tile = tiles[t];
		if (!state[tile.x].active)
			continue; // block-uniform
		const FrameDesc &fd = frames[tile.x];
		const int w = fd.w, h = fd.h, words = fd.words, x0 = tile.y, y0 = tile.z;
		double lo = INFINITY;
		for (int k = tid; k < MHALO * MHALO; k += 256) {
			const double v = clean_at(fd, x0 - 2 + k % MHALO, y0 - 2 + k / MHALO, mode);
			C[k] = v;
			lo = dmin(lo, v);
		}
#pragma unroll
		for (int o = 16; o; o >>= 1)
			lo = dmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
		if (lane == 0)
			wmin[warp] = lo;
		__syncthreads();
		double m_lo = wmin[0];
#pragma unroll
		for (int i = 1; i < 8; ++i)
			m_lo = dmin(m_lo, wmin[i]);
		const bool scalar_noise = !fd.gain_map && !fd.rn_map;
		const double nz_tile = scalar_noise ? noise_from_median(fd, 0, m_lo) : 0.0;
		const uint32_t *holes = plane_ptr(fd, P_HOLE);
		uint32_t found = 0; // bit j: row warp + 8 j of this lane's column
#pragma unroll 1
		for (int oy = warp; oy < MTILE; oy += 8) {
			const int x = x0 + lane, y = y0 + oy;
			if (y >= h)
				break; // warp-uniform
			bool c = false;
			if (x < w) {
				const int cx = lane + 2, cy = oy + 2;
				double l, r, u, d;
				if (lm == WRAP || lm == CONSTANT) {
					l = C[cy * MHALO + cx - 1];
					r = C[cy * MHALO + cx + 1];
					u = C[(cy - 1) * MHALO + cx];
					d = C[(cy + 1) * MHALO + cx];
				} else {
					l = C[cy * MHALO + clampi(x - 1, 0, w - 1) - x0 + 2];
					r = C[cy * MHALO + clampi(x + 1, 0, w - 1) - x0 + 2];
					u = C[(clampi(y - 1, 0, h - 1) - y0 + 2) * MHALO + cx];
					d = C[(clampi(y + 1, 0, h - 1) - y0 + 2) * MHALO + cx];
				}
				const double lap = lap_formula(C[cy * MHALO + cx], u, d, l, r);
				const double nz = scalar_noise ? nz_tile
					: noise_from_median(fd, (long long)y * w + x, m_lo);
				const uint32_t hw = holes[(long long)y * words + (x0 >> 5)];
				c = !((hw >> lane) & 1u) && lap > thr * (2 * nz);
			}
			found |= (uint32_t)c << (oy >> 3);
			clear_detect_words(fd, (long long)y * words + (x0 >> 5), lane);
		}
		if (__any_sync(0xffffffffu, found != 0)) {
			unsigned long long slot = warp_append(&ctl->n_cand, __popc(found));
			while (found) {
				const int j = __ffs(found) - 1;
				found &= found - 1;
				cands[slot++] = make_uint2((unsigned)tile.x,
					(unsigned)((long long)(y0 + warp + 8 * j) * w + x0 + lane));
			}
		}
		__syncthreads();
	}
}

// Noise model at an in-frame pixel (exact: its own 5 x 5 median of clean
// under the border mode).
__device__ __forceinline__ double noise_model_at(const FrameDesc &fd, int x, int y, int mode)
{
	double v[25];
#pragma unroll
	for (int dy = 0; dy < 5; ++dy)
#pragma unroll
		for (int dx = 0; dx < 5; ++dx)
			v[dy * 5 + dx] = clean_at(fd, x + dx - 2, y + dy - 2, mode);
	return noise_from_median(fd, (long long)y * fd.w + x, median_network(v));
}

// Ascending bitonic network over the 32 lanes (compare-exchange form).
__device__ __forceinline__ double warp_sort32(double v)
{
	const int lane = threadIdx.x & 31;
#pragma unroll
	for (int span = 2; span <= 32; span *= 2) {
#pragma unroll
		for (int step = span / 2; step; step /= 2) {
			double peer = __shfl_xor_sync(0xffffffffu, v, step);
			bool lower = ((lane & span) == 0) == ((lane & step) == 0);
			v = lower ? dmin(v, peer) : dmax(v, peer);
		}
	}
	return v;
}

// B: one warp per candidate.  Lane l < 25 evaluates sig_raw at window cell l
// (row-major, folded by the median's border map; zero outside for constant),
// a 32-lane bitonic network (+inf padding) gives the 5 x 5 median, and
// sig = sig_raw(center) - median decides the S1/S2 bits and the seed list.  A
// window holding a NaN takes the reference's exact rule in lane 0.
__global__ void __launch_bounds__(256)
candidate_kernel(const FrameDesc *__restrict__ frames, const uint2 *__restrict__ cands,
	DetectParams prm, Control *ctl, Seed *seeds)
{
	const int lane = threadIdx.x & 31;
	const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
	const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
	const long long n = (long long)ctl->n_cand;
	const int mode = prm.mode, lm = lap_mode(mode);
	for (long long e = gw; e < n; e += nw) {
		const uint2 t = cands[e];
		const FrameDesc &fd = frames[t.x];
		const int w = fd.w, h = fd.h;
		const int x = (int)(t.y % (unsigned)w), y = (int)(t.y / (unsigned)w);
		double v = INFINITY, nz = 0;
		if (lane < 25) {
			const int mx = border_index(x + lane % 5 - 2, w, mode);
			const int my = border_index(y + lane / 5 - 2, h, mode);
			v = 0;
			if (mx >= 0 && my >= 0) {
				const long long i = (long long)my * w + mx;
				nz = fd.error ? fd.error[i] : noise_model_at(fd, mx, my, mode);
				const double lap = lap_formula(fd.clean[i], clean_at(fd, mx, my - 1, lm),
					clean_at(fd, mx, my + 1, lm), clean_at(fd, mx - 1, my, lm),
					clean_at(fd, mx + 1, my, lm));
				v = lap / (2 * nz);
			}
		}
		const double center = __shfl_sync(0xffffffffu, v, 12);
		const double nz_center = __shfl_sync(0xffffffffu, nz, 12);
		double med;
		if (__any_sync(0xffffffffu, isnan(v))) {
			double win[25];
#pragma unroll
			for (int i = 0; i < 25; ++i)
				win[i] = __shfl_sync(0xffffffffu, v, i);
			med = lane == 0 ? window_median_exact(win, 25) : 0.0;
			med = __shfl_sync(0xffffffffu, med, 0);
		} else {
			med = __shfl_sync(0xffffffffu, warp_sort32(v), 12);
		}
		const double sig = center - med;
		bool seed = false;
		if (lane == 0) {
			const long long word = (long long)y * fd.words + (x >> 5);
			const uint32_t bit = 1u << (x & 31);
			if (sig > prm.cr)
				atomicOr(plane_ptr(fd, P_S1) + word, bit);
			if (sig > prm.nb)
				atomicOr(plane_ptr(fd, P_S2) + word, bit);
			seed = sig > prm.cr && !(plane_ptr(fd, P_EXCL)[word] & bit);
		}
		if (lane == 0)
			seeds[e] = seed ? Seed{t.x, t.y, sig, nz_center} : Seed{NO_SEED, 0, 0.0, 0.0};
	}
}

// Element `rank` of the 64 values held as (a, b) = slots (lane, 32 + lane) of a
// warp, by an ascending bitonic network.  NaN-free inputs.
__device__ __forceinline__ double warp_rank64(double a, double b, int rank)
{
	const int lane = threadIdx.x & 31;
#pragma unroll
	for (int k = 2; k <= 64; k <<= 1) {
#pragma unroll
		for (int j = k >> 1; j > 0; j >>= 1) {
			if (j == 32) {
				cas(a, b);
			} else {
				double pa = __shfl_xor_sync(0xffffffffu, a, j);
				double pb = __shfl_xor_sync(0xffffffffu, b, j);
				int ea = lane, eb = lane + 32;
				bool mina = ((ea & j) == 0) == ((ea & k) == 0);
				bool minb = ((eb & j) == 0) == ((eb & k) == 0);
				a = mina ? dmin(a, pa) : dmax(a, pa);
				b = minb ? dmin(b, pb) : dmax(b, pb);
			}
		}
	}
	double ra = __shfl_sync(0xffffffffu, a, rank & 31);
	double rb = __shfl_sync(0xffffffffu, b, rank & 31);
	return rank < 32 ? ra : rb;
}

// C: one warp per seed: 49 3 x 3 medians (two per lane), their 7 x 7 median,
// fine structure and the contrast test (src/filters.cuh:148-175).
__global__ void __launch_bounds__(256)
seed_kernel(const FrameDesc *__restrict__ frames, const Seed *__restrict__ seeds, DetectParams prm,
	const Control *ctl)
{
	const int lane = threadIdx.x & 31;
	const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
	const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
	const long long n = (long long)ctl->n_cand;
	const int mode = prm.mode;
	for (long long e = gw; e < n; e += nw) {
		const Seed sd = seeds[e];
		if (sd.frame == NO_SEED)
			continue; // warp-uniform
		const FrameDesc &fd = frames[sd.frame];
		const int w = fd.w, h = fd.h;
		const int x = (int)(sd.pixel % (unsigned)w), y = (int)(sd.pixel / (unsigned)w);
		double m3[2] = {INFINITY, INFINITY};
#pragma unroll
		for (int s = 0; s < 2; ++s) {
			const int j = lane + 32 * s;
			if (j < 49) {
				int qx = x + j % 7 - 3, qy = y + j / 7 - 3;
				double m = 0;
				if (!(mode == CONSTANT && (qx < 0 || qx >= w || qy < 0 || qy >= h))) {
					if (mode == NEAREST) {
						qx = clampi(qx, 0, w - 1);
						qy = clampi(qy, 0, h - 1);
					}
					m = median9(clean_at(fd, qx - 1, qy - 1, mode), clean_at(fd, qx, qy - 1, mode),
						clean_at(fd, qx + 1, qy - 1, mode), clean_at(fd, qx - 1, qy, mode),
						clean_at(fd, qx, qy, mode), clean_at(fd, qx + 1, qy, mode),
						clean_at(fd, qx - 1, qy + 1, mode), clean_at(fd, qx, qy + 1, mode),
						clean_at(fd, qx + 1, qy + 1, mode));
				}
				m3[s] = m;
			}
		}
		const double med3c = __shfl_sync(0xffffffffu, m3[0], 24);
		const double med7 = warp_rank64(m3[0], m3[1], 24);
		if (lane == 0) {
			double fine = (med3c - med7) / sd.noise;
			fine = fine < FINE_FLOOR ? FINE_FLOOR : fine;
			if (sd.sig / fine > prm.contrast)
				atomicOr(plane_ptr(fd, P_CAND) + (long long)y * fd.words + (x >> 5), 1u << (x & 31));
		}
	}
}

} // namespace cb

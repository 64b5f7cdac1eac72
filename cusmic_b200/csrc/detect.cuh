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
	double tmin;  // min(cr, nb): sig_raw above it can pass a threshold
	double thi2;  // 2 cr (1 - 1e-12): division-free superset test for sig_raw > cr
	double tlo2;  // 2 nb (1 - 1e-12): the same for sig_raw > neighbor
	int mode;
};

// Kernel A's two superset tests (see sig_stream_kernel): bit 0 = can exceed
// cr_threshold, bit 1 = can only exceed neighbor_threshold.
__device__ __forceinline__ uint32_t candidate_class(double lap, double nz, const DetectParams &p)
{
	if (lap > p.thi2 * nz)
		return 1u;
	return lap > p.tlo2 * nz ? 2u : 0u;
}

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

// The same Laplacian from quarter values q = x / 4 (exact: a power-of-two
// scaling), so a streaming kernel can scale each pixel once.
__device__ __forceinline__ double lap_quarters(double qc, double qu, double qd, double ql, double qr)
{
	double up = qc - qu;
	double down = qc - qd;
	double left = qc - ql;
	double right = qc - qr;
	return (positive(up + left) + positive(up + right)) + (positive(down + left) + positive(down + right));
}

// clean at (x, y) under a border mode (0 outside for constant).
__device__ __forceinline__ double clean_at(const FrameDesc &fd, int x, int y, int mode)
{
	int mx = border_index(x, fd.w, mode), my = border_index(y, fd.h, mode);
	return mx < 0 || my < 0 ? 0.0 : fd.clean[(long long)my * fd.w + mx];
}

// The Laplacian at an in-frame pixel (reference src/filters.cuh:98-104).
__device__ __forceinline__ double lap_at(const FrameDesc &fd, int x, int y, int lm)
{
	return lap_formula(fd.clean[(long long)y * fd.w + x], clean_at(fd, x, y - 1, lm),
		clean_at(fd, x, y + 1, lm), clean_at(fd, x - 1, y, lm), clean_at(fd, x + 1, y, lm));
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

// Append the candidates of one strip item (lane = column, bit k of `rows` =
// row y0 + k) with a single atomic per item; the high list grows from the
// front of the buffer, the low list from its back.
__device__ __forceinline__ void stream_flush(int f, int w, int x, int y0, uint32_t hi, uint32_t lo,
	Control *ctl, uint2 *cands)
{
	if (__any_sync(0xffffffffu, hi != 0)) {
		unsigned long long slot = warp_append(&ctl->n_cand, __popc(hi));
		while (hi) {
			const int k = __ffs(hi) - 1;
			hi &= hi - 1;
			cands[slot++] = make_uint2((unsigned)f, (unsigned)((long long)(y0 + k) * w + x));
		}
	}
	if (__any_sync(0xffffffffu, lo != 0)) {
		unsigned long long slot = warp_append(&ctl->n_low, __popc(lo));
		while (lo) {
			const int k = __ffs(lo) - 1;
			lo &= lo - 1;
			cands[ctl->cand_cap - 1 - slot++] =
				make_uint2((unsigned)f, (unsigned)((long long)(y0 + k) * w + x));
		}
	}
}

// A, error-map frames: one warp per item {frame, x0, y0}: 32 columns from x0,
// rows y0 .. y0 + STREAM_ROWS - 1.  Each warp streams its rows through a
// shared-memory ring filled with cp.async, SR_LEAD rows ahead of the row it
// evaluates, so many row loads are in flight per warp without holding
// registers.  A ring row holds the row's 32 columns plus one halo column on
// each side, each cell already border-mapped with the Laplacian's border mode
// (zero outside for constant), so the evaluation has no border cases.
//
// The kernel only has to find supersets of {sig_raw > cr} and {sig_raw >
// neighbor}: B evaluates sig_raw exactly for every candidate and drops the
// others.  So instead of dividing it tests lap > (2 t (1 - 1e-12)) noise: the
// product is rounded by at most 2^-53 relative and 2 t scales exactly, so
// every pixel with fl(lap / (2 noise)) > t passes (NaN, infinite or zero noise
// give the same outcome as the division, or a larger superset).
constexpr int SR_DEPTH = 8; // ring rows per warp (power of two)
constexpr int SR_LEAD = 5;  // rows issued ahead of the row being evaluated

struct StreamRing {
	double c[SR_DEPTH][34]; // clean, columns x0 - 1 .. x0 + 32
	double e[SR_DEPTH][32]; // error map, columns x0 .. x0 + 31
	uint32_t hole[SR_DEPTH];
};

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem)
{
	unsigned s = (unsigned)__cvta_generic_to_shared(smem);
	asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}

__device__ __forceinline__ void cp_async4(void *smem, const void *gmem)
{
	unsigned s = (unsigned)__cvta_generic_to_shared(smem);
	asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}

__device__ __forceinline__ void cp_async_commit()
{
	asm volatile("cp.async.commit_group;\n" ::);
}

template <int N> __device__ __forceinline__ void cp_async_wait()
{
	asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Every lane issues its cells of ring row r (one commit group per row, empty
// past the last needed row so group counting stays uniform).
__device__ __forceinline__ void stream_issue(StreamRing &R, const FrameDesc &fd, int r, int r_end,
	int y0, int y1, int x0, int lane, int lm, int mx, int mx_halo, int xc)
{
	if (r <= r_end) {
		const int slot = r & (SR_DEPTH - 1);
		const int my = border_index(r, fd.h, lm);
		const double *row = fd.clean + (long long)(my < 0 ? 0 : my) * fd.w;
		if (my >= 0 && mx >= 0)
			cp_async8(&R.c[slot][1 + lane], row + mx);
		else
			R.c[slot][1 + lane] = 0.0;
		if (lane == 0 || lane == 31) {
			const int hi = lane == 0 ? 0 : 33;
			if (my >= 0 && mx_halo >= 0)
				cp_async8(&R.c[slot][hi], row + mx_halo);
			else
				R.c[slot][hi] = 0.0;
		}
		if (r >= y0 && r < y1) {
			cp_async8(&R.e[slot][lane], fd.error + (long long)r * fd.w + xc);
			if (lane == 0)
				cp_async4(&R.hole[slot], plane_ptr(fd, P_HOLE) + (long long)r * fd.words + (x0 >> 5));
		}
	}
	cp_async_commit();
}

__global__ void __launch_bounds__(256)
sig_stream_kernel(const FrameDesc *__restrict__ frames, const FrameState *__restrict__ state,
	const int4 *__restrict__ items, int nitems, DetectParams prm, Control *ctl, uint2 *cands)
{
	__shared__ StreamRing rings[8];
	const int lane = threadIdx.x & 31;
	StreamRing &R = rings[threadIdx.x >> 5];
	const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
	const int lm = lap_mode(prm.mode);
	for (int it = gw; it < nitems; it += nw) {
		const int4 item = items[it];
		if (!state[item.x].active)
			continue; // warp-uniform
		const FrameDesc &fd = frames[item.x];
		const int w = fd.w, h = fd.h, words = fd.words;
		const int x0 = item.y, y0 = item.z, y1 = min(y0 + STREAM_ROWS, h);
		const int x = x0 + lane, xc = min(x, w - 1);
		const bool valid = x < w;
		const int mx = border_index(x, w, lm);
		const int mx_halo = border_index(lane == 0 ? x0 - 1 : x0 + 32, w, lm);
		const int r_end = y1; // the row below the last output row
		for (int r = y0 - 1; r < y0 - 1 + SR_LEAD + 1; ++r)
			stream_issue(R, fd, r, r_end, y0, y1, x0, lane, lm, mx, mx_halo, xc);
		uint32_t hi = 0, lo = 0; // bit k: row y0 + k of this lane's column is a candidate
		double qu = 0, qc = 0;   // quarter values of the rows above and at y
		for (int y = y0; y < y1; ++y) {
			// Groups issued: rows y0 - 1 .. y + SR_LEAD - 1; row y + 1 is done
			// once at most SR_LEAD - 2 newer groups are pending.
			cp_async_wait<SR_LEAD - 2>();
			__syncwarp();
			const int s = y & (SR_DEPTH - 1), sd = (y + 1) & (SR_DEPTH - 1);
			if (y == y0) {
				qu = R.c[(y - 1) & (SR_DEPTH - 1)][1 + lane] * 0.25;
				qc = R.c[s][1 + lane] * 0.25;
			}
			const double qd = R.c[sd][1 + lane] * 0.25;
			const double lap = lap_quarters(qc, qu, qd, R.c[s][lane] * 0.25, R.c[s][lane + 2] * 0.25);
			const uint32_t cls = valid && !((R.hole[s] >> lane) & 1u)
				? candidate_class(lap, R.e[s][lane], prm) : 0u;
			hi |= (cls & 1u) << (y - y0);
			lo |= (cls >> 1) << (y - y0);
			qu = qc;
			qc = qd;
			clear_detect_words(fd, (long long)y * words + (x0 >> 5), lane);
			__syncwarp();
			stream_issue(R, fd, y + SR_LEAD, r_end, y0, y1, x0, lane, lm, mx, mx_halo, xc);
		}
		cp_async_wait<0>();
		__syncwarp();
		stream_flush(item.x, w, x, y0, hi, lo, ctl, cands);
	}
}

__device__ __forceinline__ void tile_flush(int f, int w, int x, int ybase, uint32_t hi, uint32_t lo,
	Control *ctl, uint2 *cands)
{
	if (__any_sync(0xffffffffu, hi != 0)) {
		unsigned long long slot = warp_append(&ctl->n_cand, __popc(hi));
		while (hi) {
			const int j = __ffs(hi) - 1;
			hi &= hi - 1;
			cands[slot++] = make_uint2((unsigned)f, (unsigned)((long long)(ybase + 8 * j) * w + x));
		}
	}
	if (__any_sync(0xffffffffu, lo != 0)) {
		unsigned long long slot = warp_append(&ctl->n_low, __popc(lo));
		while (lo) {
			const int j = __ffs(lo) - 1;
			lo &= lo - 1;
			cands[ctl->cand_cap - 1 - slot++] =
				make_uint2((unsigned)f, (unsigned)((long long)(ybase + 8 * j) * w + x));
		}
	}
}

// A, noise-model frames: one block per MTILE x MTILE tile with its clean
// pixels (halo 2, border-extended) in shared memory.  The noise model is
// monotone non-decreasing in the 5 x 5 median in floating point (max, g * m,
// rn^2 + ., sqrt and / g are each monotone for g > 0), and the median of a
// window is at least the minimum m_lo of the tile and its halo, so
// noise(m_lo) <= noise(med5) and lap / (2 noise(m_lo)) >= sig_raw.  The tile
// therefore applies the superset tests of sig_stream_kernel with noise(m_lo)
// in place of the noise, without any median.  Scalar gain and read
// noise make noise(m_lo) one value per tile; maps evaluate it per pixel.
__global__ void __launch_bounds__(256)
sig_model_kernel(const FrameDesc *__restrict__ frames, const FrameState *__restrict__ state,
	const int4 *__restrict__ tiles, int ntiles, DetectParams prm, Control *ctl, uint2 *cands)
{
	__shared__ double C[MHALO * MHALO];
	__shared__ double wmin[8];
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int mode = prm.mode, lm = lap_mode(mode);
	for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
		const int4 tile = tiles[t];
		if (!state[tile.x].active)
			continue; // block-uniform
		const FrameDesc &fd = frames[tile.x];
		const int w = fd.w, h = fd.h, words = fd.words, x0 = tile.y, y0 = tile.z;
		double vmin = INFINITY;
		for (int k = tid; k < MHALO * MHALO; k += 256) {
			const double v = clean_at(fd, x0 - 2 + k % MHALO, y0 - 2 + k / MHALO, mode);
			C[k] = v;
			vmin = dmin(vmin, v);
		}
#pragma unroll
		for (int o = 16; o; o >>= 1)
			vmin = dmin(vmin, __shfl_xor_sync(0xffffffffu, vmin, o));
		if (lane == 0)
			wmin[warp] = vmin;
		__syncthreads();
		double m_lo = wmin[0];
#pragma unroll
		for (int i = 1; i < 8; ++i)
			m_lo = dmin(m_lo, wmin[i]);
		const bool scalar_noise = !fd.gain_map && !fd.rn_map;
		const double nz_tile = scalar_noise ? noise_from_median(fd, 0, m_lo) : 0.0;
		const uint32_t *holes = plane_ptr(fd, P_HOLE);
		uint32_t hi = 0, lo = 0; // bit j: row warp + 8 j of this lane's column
#pragma unroll 1
		for (int oy = warp; oy < MTILE; oy += 8) {
			const int x = x0 + lane, y = y0 + oy;
			if (y >= h)
				break; // warp-uniform
			uint32_t cls = 0;
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
				cls = (hw >> lane) & 1u ? 0u : candidate_class(lap, nz, prm);
			}
			hi |= (cls & 1u) << (oy >> 3);
			lo |= (cls >> 1) << (oy >> 3);
			clear_detect_words(fd, (long long)y * words + (x0 >> 5), lane);
		}
		// Bits j of this lane are rows y0 + warp + 8 j: append as rows of a
		// strip starting at y0 + warp with stride 8.
		tile_flush(tile.x, w, x0 + lane, y0 + warp, hi, lo, ctl, cands);
		__syncthreads();
	}
}

// Noise model at an in-frame pixel (exact: its own 5 x 5 median of clean
// under the border mode).
__device__ __noinline__ double noise_model_at(const FrameDesc &fd, int x, int y, int mode)
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
			const double peer = __shfl_xor_sync(0xffffffffu, v, step);
			const bool lower = ((lane & span) == 0) == ((lane & step) == 0);
			// The lower lane keeps the smaller value, the upper the larger;
			// on equal values either choice is the same value.
			v = (peer < v) == lower ? peer : v;
		}
	}
	return v;
}

// B: one warp per candidate.  Lane l < 25 evaluates sig_raw at window cell l
// (row-major, folded by the median's border map; zero outside for constant),
// a 32-lane bitonic network (+inf padding) gives the 5 x 5 median, and
// sig = sig_raw(center) - median decides the S1/S2 bits and the seed list.  A
// window holding a NaN takes the reference's exact rule in lane 0.
//
// LOW: the low list (sig_raw can exceed only neighbor_threshold), run after
// the seed kernel.  Only the S2 bit can be set there, and S2 is read only by
// the second growth step, i.e. within distance 2 of a CAND pixel; candidates
// with no CAND bit in their clipped 5 x 5 neighbourhood are skipped.
//
// A candidate at least 4 pixels from every edge stages the 9 x 9 patch of
// clean around it in the warp's shared memory (every position it touches is
// in the frame, so no border mapping is needed) and takes its Laplacians and,
// on noise-model frames, its 25 noise windows from it; the others read
// border-mapped values from global memory.  The patch stays for a seed test
// of the same pixel.
// The warp's evaluation of the candidate at (x, y): sig over its 5 x 5
// window, the S2 bit (and S1 unless LOW) unless `skip`; `fresh`: the bit
// planes were zeroed for this pass; returns sig (every lane) and the
// noise at the pixel (nz_center).  P is the warp's 9 x 9 patch buffer.
// Which frames a kernel variant serves: any (decided per frame), error-map
// frames only, or noise-model frames only (a variant compiles one path and
// needs fewer registers).
enum FramePath { PATH_ANY = 0, PATH_ERROR = 1, PATH_MODEL = 2 };

template <int PATH>
__device__ __forceinline__ bool has_error_map(const FrameDesc &fd)
{
	return PATH == PATH_ERROR ? true : PATH == PATH_MODEL ? false : fd.error != nullptr;
}

template <int PATH>
__device__ __forceinline__ bool serves(const FrameDesc &fd)
{
	return PATH == PATH_ANY || (fd.error != nullptr) == (PATH == PATH_ERROR);
}

// Scratch doubles per warp that candidate_sig needs: the sorted vertical runs
// of the 9 x 9 patch on noise-model frames (CS_RUNS), else only the 25 window
// values of the NaN rule.
constexpr int CS_RUNS = 225;

// The 25 noise medians of a staged candidate (src/filters.cuh:46-70, the
// median<5> that noise_model reads), lane l < 25 returning the median of the
// 5 x 5 block of the 9 x 9 patch P at rows l / 5 .. + 4, columns l % 5 .. + 4
// (the window of window cell l).  Clean pixels are never NaN, so the middle
// order statistic is the reference's value (its sign of a zero aside, which
// max(m, 1e-5) removes).
//
// The 25 blocks share their columns: the 45 vertical runs of five (9 columns
// x 5 row offsets) are sorted once per warp into S (S[(r * 5 + i) * 9 + c] =
// i-th smallest of rows r .. r + 4 of column c).  A block of five sorted
// columns whose rows are then sorted is sorted both ways, and its median is the
// median of the 13 cells (i, j) with (i + 1)(j + 1) <= 13 and
// (5 - i)(5 - j) <= 13: every other cell has at least 13 cells known to be no
// larger (or no smaller) than it, six on each side.  So a lane sorts only the
// rank rows of its five columns and takes a median of 13.
__device__ __forceinline__ double patch_window_median(const double *P, double *S)
{
	const int lane = threadIdx.x & 31;
	for (int k = lane; k < 45; k += 32) {
		const int r = k / 9, c = k % 9;
		const double *p = P + r * 9 + c;
		double a = p[0], b = p[9], d = p[18], e = p[27], f = p[36];
		sort5(a, b, d, e, f);
		double *s = S + r * 45 + c;
		s[0] = a;
		s[9] = b;
		s[18] = d;
		s[27] = e;
		s[36] = f;
	}
	__syncwarp();
	double med = 0;
	if (lane < 25) {
		const double *R = S + (lane / 5) * 45 + lane % 5; // rank row i at R + 9 i, columns 0..4
		double band[13];
		int nb = 0;
#pragma unroll
		for (int i = 0; i < 5; ++i) {
			double a = R[9 * i], b = R[9 * i + 1], c = R[9 * i + 2], d = R[9 * i + 3], e = R[9 * i + 4];
			sort5(a, b, c, d, e);
			const double row[5] = {a, b, c, d, e};
#pragma unroll
			for (int j = 0; j < 5; ++j)
				if ((i + 1) * (j + 1) <= 13 && (5 - i) * (5 - j) <= 13)
					band[nb++] = row[j];
		}
		med = median_network(band);
	}
	__syncwarp();
	return med;
}

// S: the warp's scratch of at least CS_RUNS doubles on noise-model frames
// (25 otherwise).
template <bool LOW, int PATH = PATH_ANY>
__device__ __forceinline__ double candidate_sig(const FrameDesc &fd, int x, int y, double *P,
	double *S, const DetectParams &prm, double &nz_center_out, bool fresh, bool skip = false)
{
	const int lane = threadIdx.x & 31;
	const int w = fd.w, h = fd.h, mode = prm.mode, lm = lap_mode(mode);
	const bool err = has_error_map<PATH>(fd);
	double v = INFINITY, nz = 0;
	if (x >= 4 && y >= 4 && x + 4 < w && y + 4 < h) { // warp-uniform
		__syncwarp();
		const double *src = fd.clean + (long long)(y - 4) * w + (x - 4);
		for (int k = lane; k < 81; k += 32)
			P[k] = src[(long long)(k / 9) * w + k % 9];
		if (lane < 25 && err) // loads with the patch
			nz = fd.error[(long long)(y + lane / 5 - 2) * w + x + lane % 5 - 2];
		__syncwarp();
		const int dy = lane / 5, dx = lane % 5;
		if (!err) { // warp-uniform
			const double m = patch_window_median(P, S);
			if (lane < 25)
				nz = noise_from_median(fd, (long long)(y + dy - 2) * w + x + dx - 2, m);
		}
		if (lane < 25) {
			const double *q = P + (dy + 2) * 9 + dx + 2; // the window cell
			v = lap_formula(q[0], q[-9], q[9], q[-1], q[1]) / (2 * nz);
		}
	} else if (lane < 25) {
		const int mx = border_index(x + lane % 5 - 2, w, mode);
		const int my = border_index(y + lane / 5 - 2, h, mode);
		v = 0;
		if (mx >= 0 && my >= 0) {
			const long long i = (long long)my * w + mx;
			nz = err ? fd.error[i] : noise_model_at(fd, mx, my, mode);
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
		// The reference's NaN rule on the 25 values, in the warp's scratch
		// (a register array indexed at run time would live in local memory).
		__syncwarp();
		if (lane < 25)
			S[lane] = v;
		__syncwarp();
		med = lane == 0 ? window_median_exact(S, 25) : 0.0;
		med = __shfl_sync(0xffffffffu, med, 0);
		__syncwarp();
	} else {
		med = __shfl_sync(0xffffffffu, warp_sort32(v), 12);
	}
	const double sig = center - med;
	if (lane == 0 && !skip) {
		// Set or clear: an incremental pass keeps the bits of the previous
		// pass and re-evaluates some pixels.
		const long long word = (long long)y * fd.words + (x >> 5);
		const uint32_t bit = 1u << (x & 31);
		write_bit(plane_ptr(fd, P_S2) + word, bit, sig > prm.nb, fresh);
		if (!LOW)
			write_bit(plane_ptr(fd, P_S1) + word, bit, sig > prm.cr, fresh);
	}
	nz_center_out = nz_center;
	return sig;
}

// candidate_sig plus the seed slot of candidate e (list-based kernels).  A
// hole (src/filters.cuh:137-146: sig = 0) gets no bit and no seed; its flag
// is loaded before the evaluation and only read after it.
template <bool LOW, int PATH = PATH_ANY>
__device__ __forceinline__ void candidate_eval(const FrameDesc &fd, uint2 t, long long e, int x, int y,
	double *P, double *S, const DetectParams &prm, Seed *seeds, bool fresh, bool hole = false)
{
	double nz;
	const long long word = (long long)y * fd.words + (x >> 5);
	const uint32_t bit = 1u << (x & 31);
	const uint32_t excl = LOW ? 0u : plane_ptr(fd, P_EXCL)[word];
	const double sig = candidate_sig<LOW, PATH>(fd, x, y, P, S, prm, nz, fresh, hole);
	if (!LOW && (threadIdx.x & 31) == 0) {
		const bool seed = !hole && sig > prm.cr && !(excl & bit);
		seeds[e] = seed ? Seed{t.x, t.y, sig, nz} : Seed{NO_SEED, 0, 0.0, 0.0};
		if (!seed) // the seed kernel decides the CAND bit of a seed
			write_bit(plane_ptr(fd, P_CAND) + word, bit, false, fresh);
	}
}

// The first pass's evaluation of a noise-model candidate at least two pixels
// from every edge by one thread: its 25 window values from the sig_raw map
// (region_sig_kernel), their median by a sorting network (NaN-free windows:
// any network gives the median's value, a zero's sign aside, which no
// threshold sees), the S1 / S2 bits and the seed slot, as candidate_eval.
// Returns false for a window holding a NaN (the warp's NaN rule decides it).
__device__ __forceinline__ bool map_candidate(const FrameDesc &fd, uint2 t, long long e, int x, int y,
	const DetectParams &prm, Seed *seeds)
{
	const int w = fd.w;
	double v[25];
	bool nan = false;
#pragma unroll
	for (int c = 0; c < 25; ++c) {
		v[c] = fd.sig_raw[(long long)(y + c / 5 - 2) * w + x + c % 5 - 2];
		nan |= isnan(v[c]);
	}
	if (nan)
		return false;
	const long long word = (long long)y * fd.words + (x >> 5);
	const uint32_t bit = 1u << (x & 31);
	const bool hole = (plane_ptr(fd, P_HOLE)[word] & bit) != 0;
	const uint32_t excl = plane_ptr(fd, P_EXCL)[word];
	const double nz = fd.noise[(long long)y * w + x];
	const double center = v[12];
	const double sig = center - median_network(v);
	if (!hole) { // a hole's significance is zero: no bit (the planes start zeroed)
		write_bit(plane_ptr(fd, P_S2) + word, bit, sig > prm.nb, true);
		write_bit(plane_ptr(fd, P_S1) + word, bit, sig > prm.cr, true);
	}
	const bool seed = !hole && sig > prm.cr && !(excl & bit);
	seeds[e] = seed ? Seed{t.x, t.y, sig, nz} : Seed{NO_SEED, 0, 0.0, 0.0};
	return true;
}

// B, high list: one warp per candidate.  Holes have sig = 0
// (src/filters.cuh:137-146): no bit, no seed; the dense kernel does not test
// the hole plane itself.
// PATH: the frames this launch serves (FramePath); the other launch of a
// mixed batch takes the rest of the list.
template <int PATH>
__global__ void __launch_bounds__(256, 4)
candidate_high_kernel(const FrameDesc *__restrict__ frames, const uint2 *__restrict__ cands,
	DetectParams prm, Control *ctl, Seed *seeds, int fresh)
{
	__shared__ double patches[8][81];
	__shared__ double scratch[8][CS_RUNS];
	double *P = patches[threadIdx.x >> 5], *S = scratch[threadIdx.x >> 5];
	const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
	const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
	const long long n = (long long)ctl->n_cand;
	uint2 next = gw < n ? cands[gw] : make_uint2(0u, 0u);
	for (long long e = gw; e < n; e += nw) {
		const uint2 t = next;
		if (e + nw < n) // the next entry loads during this evaluation
			next = cands[e + nw];
		const FrameDesc &fd = frames[t.x];
		if (!serves<PATH>(fd))
			continue; // warp-uniform
		const int x = (int)(t.y % (unsigned)fd.w), y = (int)(t.y / (unsigned)fd.w);
		const bool hole = test_bit(plane_ptr(fd, P_HOLE), fd.words, x, y);
		candidate_eval<false, PATH>(fd, t, e, x, y, P, S, prm, seeds, fresh != 0, hole);
	}
}

// B, high list, first pass on noise-model frames: a thread per candidate
// whose window the sig_raw map holds (map_candidate); the warp evaluates the
// others (frame edges, windows with a NaN) one after another with
// candidate_eval.  Its own launch bounds: the thread path holds 25 window
// values, the warp path (candidate_high_kernel) runs at four blocks per SM.
__global__ void __launch_bounds__(256, 2)
candidate_map_kernel(const FrameDesc *__restrict__ frames, const uint2 *__restrict__ cands,
	DetectParams prm, Control *ctl, Seed *seeds)
{
	constexpr int PATH = PATH_MODEL;
	__shared__ double patches[8][81];
	__shared__ double scratch[8][CS_RUNS];
	double *P = patches[threadIdx.x >> 5], *S = scratch[threadIdx.x >> 5];
	const long long n = (long long)ctl->n_cand;
	const int lane = threadIdx.x & 31;
	const long long stride = (long long)gridDim.x * blockDim.x;
	for (long long base = blockIdx.x * (long long)blockDim.x + (threadIdx.x & ~31); base < n;
	     base += stride) { // warp-uniform
		const long long e = base + lane;
		uint2 t = make_uint2(0u, 0u);
		bool defer = false;
		if (e < n) {
			t = cands[e];
			const FrameDesc &fd = frames[t.x];
			if (serves<PATH>(fd)) {
				const int x = (int)(t.y % (unsigned)fd.w), y = (int)(t.y / (unsigned)fd.w);
				defer = !(fd.sig_raw && x >= 2 && y >= 2 && x + 2 < fd.w && y + 2 < fd.h &&
					map_candidate(fd, t, e, x, y, prm, seeds));
			}
		}
		for (unsigned m = __ballot_sync(0xffffffffu, defer); m; m &= m - 1) {
			const int j = __ffs(m) - 1;
			const uint2 tj = make_uint2(__shfl_sync(0xffffffffu, t.x, j),
				__shfl_sync(0xffffffffu, t.y, j));
			const FrameDesc &fd = frames[tj.x];
			const int x = (int)(tj.y % (unsigned)fd.w), y = (int)(tj.y / (unsigned)fd.w);
			const bool hole = test_bit(plane_ptr(fd, P_HOLE), fd.words, x, y);
			candidate_eval<false, PATH>(fd, tj, base + j, x, y, P, S, prm, seeds, true, hole);
		}
	}
}

// B, low list (run after the seed kernel): a lane per candidate first tests
// its clipped 5 x 5 neighbourhood of the CAND plane with five 36-bit row
// windows (S2 is read only by the second growth step, within distance 2 of a
// CAND pixel) and its hole bit; the warp then evaluates the survivors.
template <int PATH>
__global__ void __launch_bounds__(256, PATH == PATH_ERROR ? 4 : 3)
candidate_low_kernel(const FrameDesc *__restrict__ frames, const uint2 *__restrict__ cands,
	DetectParams prm, Control *ctl, int fresh)
{
	__shared__ double patches[8][81];
	__shared__ double scratch[8][PATH == PATH_ERROR ? 25 : CS_RUNS];
	const int lane = threadIdx.x & 31;
	double *P = patches[threadIdx.x >> 5], *S = scratch[threadIdx.x >> 5];
	const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
	const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
	const long long n = (long long)ctl->n_low;
	const unsigned long long cap = ctl->cand_cap;
	// Entries per warp and sweep: 32 for a long list; a short list (the late
	// passes) is spread thinner so that its survivors, which a warp
	// evaluates one after another, land on different warps.
	const int chunk = n >= nw * 32 ? 32 : n > nw ? (int)((n + nw - 1) / nw) : 1;
	for (long long base = gw * chunk; base < n; base += nw * chunk) {
		const long long e = base + lane;
		uint2 t = make_uint2(0, 0);
		bool near = false;
		if (lane < chunk && e < n) {
			t = cands[cap - 1 - e];
			const FrameDesc &fd = frames[t.x];
			const int x = (int)(t.y % (unsigned)fd.w), y = (int)(t.y / (unsigned)fd.w);
			const uint32_t *cand = plane_ptr(fd, P_CAND);
			unsigned long long any = 0;
#pragma unroll
			for (int d = -2; d <= 2; ++d)
				any |= bit_window(cand, fd.words, fd.h, y + d, x >> 5);
			near = serves<PATH>(fd) && ((any >> (x & 31)) & 0x1full) &&
				!test_bit(plane_ptr(fd, P_HOLE), fd.words, x, y);
		}
		for (unsigned m = __ballot_sync(0xffffffffu, near); m; m &= m - 1) {
			const int j = __ffs(m) - 1;
			const uint2 tj = make_uint2(__shfl_sync(0xffffffffu, t.x, j), __shfl_sync(0xffffffffu, t.y, j));
			const FrameDesc &fd = frames[tj.x];
			candidate_eval<true, PATH>(fd, tj, base + j, (int)(tj.y % (unsigned)fd.w),
				(int)(tj.y / (unsigned)fd.w), P, S, prm, nullptr, fresh != 0);
		}
	}
}

// Element RANK < 32 of the 64 values held as (a, b) = slots (lane, 32 + lane)
// of a warp, by an ascending bitonic network: a sorts ascending and b
// descending, the half-cleaner keeps the 32 smallest in a, and only a is
// merged further.  NaN-free inputs; on equal values either choice of a
// compare-exchange is the same value.
template <int RANK>
__device__ __forceinline__ double warp_rank64(double a, double b)
{
	static_assert(RANK >= 0 && RANK < 32, "the lower half holds the rank");
	const int lane = threadIdx.x & 31;
#pragma unroll
	for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
		for (int j = k >> 1; j > 0; j >>= 1) {
			const double pa = __shfl_xor_sync(0xffffffffu, a, j);
			const double pb = __shfl_xor_sync(0xffffffffu, b, j);
			const bool mina = ((lane & j) == 0) == ((lane & k) == 0);
			const bool minb = ((lane & j) == 0) == (((lane + 32) & k) == 0);
			a = (pa < a) == mina ? pa : a;
			b = (pb < b) == minb ? pb : b;
		}
	}
	a = dmin(a, b);
#pragma unroll
	for (int j = 16; j > 0; j >>= 1) {
		const double pa = __shfl_xor_sync(0xffffffffu, a, j);
		a = (pa < a) == ((lane & j) == 0) ? pa : a;
	}
	return __shfl_sync(0xffffffffu, a, RANK);
}

// The warp's fine-structure test of a seed at (x, y) (src/filters.cuh:148-175):
// 49 3 x 3 medians (two per lane), their 7 x 7 median, fine structure and the
// contrast test, setting the CAND bit.  A seed at least 4 pixels from every
// edge stages its 9 x 9 patch of clean in the warp's shared memory (P), sorts
// the 63 vertical triples of the patch once (T) and takes each 3 x 3 median
// from three sorted triples (median9's rule).
__device__ __forceinline__ void seed_eval(const FrameDesc &fd, int x, int y, double sig, double noise,
	const DetectParams &prm, double *P, double (*T)[63], bool fresh, bool staged = false)
{
	const int lane = threadIdx.x & 31;
	const int w = fd.w, h = fd.h, mode = prm.mode;
	double m3[2] = {INFINITY, INFINITY};
	if (x >= 4 && y >= 4 && x + 4 < w && y + 4 < h) { // warp-uniform
		__syncwarp();
		if (!staged) { // else the candidate evaluation left this patch in P
			const double *src = fd.clean + (long long)(y - 4) * w + (x - 4);
			for (int k = lane; k < 81; k += 32)
				P[k] = src[(long long)(k / 9) * w + k % 9];
			__syncwarp();
		}
		for (int k = lane; k < 63; k += 32) {
			double a = P[k], b = P[k + 9], c = P[k + 18];
			cas(a, b);
			cas(b, c);
			cas(a, b);
			T[0][k] = a;
			T[1][k] = b;
			T[2][k] = c;
		}
		__syncwarp();
#pragma unroll
		for (int s = 0; s < 2; ++s) {
			const int j = lane + 32 * s;
			if (j < 49) {
				const int k = (j / 7) * 9 + j % 7; // window rows j/7 .. +2, columns j%7 .. +2
				const double *lo = &T[0][k], *mid = &T[1][k], *hi = &T[2][k];
				m3[s] = med3(dmax(dmax(lo[0], lo[1]), lo[2]), med3(mid[0], mid[1], mid[2]),
					dmin(dmin(hi[0], hi[1]), hi[2]));
			}
		}
	} else {
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
	}
	const double med3c = __shfl_sync(0xffffffffu, m3[0], 24);
	const double med7 = warp_rank64<24>(m3[0], m3[1]);
	double fine = (med3c - med7) / noise;
	fine = fine < FINE_FLOOR ? FINE_FLOOR : fine;
	const bool cand = sig / fine > prm.contrast;
	if (lane == 0)
		write_bit(plane_ptr(fd, P_CAND) + (long long)y * fd.words + (x >> 5), 1u << (x & 31), cand,
			fresh);
	// Growth can flag pixels within two rows of a CAND pixel.
	if (cand && fd.rowcand && lane < 5 && y + lane - 2 >= 0 && y + lane - 2 < h)
		fd.rowcand[y + lane - 2] = 1u;
}

// C (list-based): one warp per seed slot.
__global__ void __launch_bounds__(256)
seed_kernel(const FrameDesc *__restrict__ frames, const Seed *__restrict__ seeds, DetectParams prm,
	const Control *ctl, int fresh)
{
	__shared__ double patches[8][81];
	__shared__ double triples[8][3][63];
	const int warp = threadIdx.x >> 5;
	const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
	const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
	const long long n = (long long)ctl->n_cand;
	Seed next = gw < n ? seeds[gw] : Seed{NO_SEED, 0, 0.0, 0.0};
	for (long long e = gw; e < n; e += nw) {
		const Seed sd = next;
		if (e + nw < n) // the next slot loads during this evaluation
			next = seeds[e + nw];
		if (sd.frame == NO_SEED)
			continue; // warp-uniform
		const FrameDesc &fd = frames[sd.frame];
		seed_eval(fd, (int)(sd.pixel % (unsigned)fd.w), (int)(sd.pixel / (unsigned)fd.w), sd.sig,
			sd.noise, prm, patches[warp], triples[warp], fresh != 0);
	}
}

// B and C fused, high list: one warp per candidate, and a candidate that is
// a seed gets its fine-structure test from the same warp at once (it needs
// only its own sig and noise and the clean pixels within 4), so no seed list
// is walked.  PATH as for candidate_high_kernel (error-map frames use it;
// noise-model candidates cost more and balance better as two kernels).  With
// `seeds` (a batch that also runs seed_kernel) each served entry's slot is
// marked empty.
template <int PATH>
__global__ void __launch_bounds__(256, PATH == PATH_ERROR ? 4 : 3)
candidate_seed_kernel(const FrameDesc *__restrict__ frames, const uint2 *__restrict__ cands,
	DetectParams prm, Control *ctl, Seed *seeds, int fresh)
{
	// Error-map frames only: the scratch of candidate_sig holds just the 25
	// values of the NaN rule, and the triples of the seed test serve as it.
	static_assert(PATH == PATH_ERROR, "noise-model candidates run candidate_high_kernel");
	__shared__ double patches[8][81];
	__shared__ double triples[8][3][63];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	double *P = patches[warp];
	const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
	const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
	const long long n = (long long)ctl->n_cand;
	uint2 next = gw < n ? cands[gw] : make_uint2(0u, 0u);
	for (long long e = gw; e < n; e += nw) {
		const uint2 t = next;
		if (e + nw < n) // the next entry loads during this evaluation
			next = cands[e + nw];
		const FrameDesc &fd = frames[t.x];
		if (!serves<PATH>(fd))
			continue; // warp-uniform
		const int x = (int)(t.y % (unsigned)fd.w), y = (int)(t.y / (unsigned)fd.w);
		const long long word = (long long)y * fd.words + (x >> 5);
		const uint32_t bit = 1u << (x & 31);
		const bool hole = (plane_ptr(fd, P_HOLE)[word] & bit) != 0;
		const uint32_t excl = plane_ptr(fd, P_EXCL)[word];
		if (seeds && lane == 0)
			seeds[e] = Seed{NO_SEED, 0, 0.0, 0.0};
		double nz;
		const double sig = candidate_sig<false, PATH>(fd, x, y, P, &triples[warp][0][0], prm, nz,
			fresh != 0, hole);
		// Every lane holds the same sig, so the branch is warp-uniform.
		if (!hole && sig > prm.cr && !(excl & bit))
			seed_eval(fd, x, y, sig, nz, prm, P, triples[warp], fresh != 0, true);
		else if (lane == 0)
			write_bit(plane_ptr(fd, P_CAND) + word, bit, false, fresh != 0);
	}
}

} // namespace cb

// Detection pass of one L.A.Cosmic iteration as one tiled, persistent kernel.
//
// Reference chain (src/cleaner.cuh:102-126): laplacian -> [median5 ->
// noise_model] -> snr -> median5 -> significance -> median3 -> median7 ->
// fine_structure -> detect, every stage a full-frame float64 pass.  Here one
// block owns a TW x TH output tile, stages its clean pixels (halo 4) in shared
// memory, and produces three bit planes: S1 = sig > cr_threshold,
// S2 = sig > neighbor_threshold and CAND (seeds).  Two exact facts make most
// of the median work unnecessary:
//
//  * the Laplacian is a sum of clipped terms, so lap >= 0 and sig_raw =
//    lap / (2 noise) >= 0; hence med5(sig_raw) >= 0 and sig = sig_raw -
//    med5(sig_raw) <= sig_raw.  A pixel whose sig_raw does not exceed
//    min(cr, neighbor) (both >= 0) can set neither S1 nor S2, so its 5 x 5
//    median is never needed (NaN compares false either way);
//  * fine structure (med3 -> med7) is only read by detect behind
//    `sig > cr_threshold` on a non-excluded pixel (src/filters.cuh:164-175),
//    so it is evaluated only at those seeds.
//
// Both sparse steps run from shared-memory work queues so warps stay full:
// threads take 5 x 5 medians, whole warps take seeds (49 3 x 3 medians, then a
// 64-wide warp bitonic select for the 7 x 7 median).  Every value that feeds a
// threshold is computed with the reference's operation order (no FMA), so the
// bits equal the reference's.
//
// Borders: for out-of-frame positions the reference's chained filters read
// the border-mapped value of the intermediate (e.g. med7 reads med3 at
// border_index(x)).  For mirror, reflect and wrap the border map is invariant
// under a group of isometries that folds any coordinate onto its image, so a
// median evaluated on the border-extended clean tile equals the median at the
// folded position.  Nearest folds by clamping; constant pads intermediates with
// zero.  The Laplacian reads neighbours with nearest semantics for mirror and
// reflect (src/filters.cuh:95-97), so it is evaluated at the folded position.
#pragma once
#include "common.cuh"
#include "select.cuh"

namespace cb {

struct DetectParams {
	double contrast, cr, nb, tmin;
	int mode;
};

template <int TW, int TH> struct DetectTile {
	static constexpr int CW = TW + 8, CH = TH + 8; // clean, halo 4
	static constexpr int SW = TW + 4, SH = TH + 4; // noise and sig_raw, halo 2
	static constexpr int WPR = TW / 32;             // bit words per tile row
	static constexpr int NPIX = TW * TH;
	double C[CH * CW];
	double NZ[SH * SW];
	double S[SH * SW];
	double qsig[NPIX];
	int q5[NPIX];
	int qs[NPIX];
	uint32_t hole[TH * WPR], excl[TH * WPR], s1[TH * WPR], s2[TH * WPR], cand[TH * WPR];
	int n5, nseed;
};

__device__ __forceinline__ double positive(double v)
{
	return v < 0 ? 0 : v;
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

template <int TW, int TH, int NT>
__global__ void __launch_bounds__(NT)
detect_kernel(const FrameDesc *__restrict__ frames, const FrameState *__restrict__ state,
	const int4 *__restrict__ tiles, int ntiles, DetectParams prm)
{
	using T = DetectTile<TW, TH>;
	constexpr int CW = T::CW, CH = T::CH, SW = T::SW, SH = T::SH, WPR = T::WPR;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	T &sm = *reinterpret_cast<T *>(smem_raw);
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int mode = prm.mode;

	for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
		const int4 tile = tiles[t];
		if (!state[tile.x].active)
			continue; // block-uniform
		const FrameDesc &fd = frames[tile.x];
		const int w = fd.w, h = fd.h, words = fd.words;
		const int x0 = tile.y, y0 = tile.z;
		const int xe = min(x0 + TW, w), ye = min(y0 + TH, h);
		const uint32_t *hole_p = plane_ptr(fd, P_HOLE), *excl_p = plane_ptr(fd, P_EXCL);
		const double *clean = fd.clean;

		if (tid == 0) {
			sm.n5 = 0;
			sm.nseed = 0;
		}
		for (int k = tid; k < TH * WPR; k += NT) {
			int gy = y0 + k / WPR, gw = (x0 >> 5) + k % WPR;
			uint32_t hb = 0, eb = 0;
			if (gy < h && gw < words) {
				long long o = (long long)gy * words + gw;
				hb = hole_p[o];
				eb = excl_p[o];
			}
			sm.hole[k] = hb;
			sm.excl[k] = eb;
			sm.s1[k] = 0;
			sm.s2[k] = 0;
			sm.cand[k] = 0;
		}
		// Stage 1: border-extended clean pixels, halo 4.
		for (int k = tid; k < CH * CW; k += NT) {
			int gx = x0 - 4 + k % CW, gy = y0 - 4 + k / CW;
			double v = 0;
			if (gx < xe + 4 && gy < ye + 4) {
				int mx = border_index(gx, w, mode), my = border_index(gy, h, mode);
				if (mx >= 0 && my >= 0)
					v = clean[(long long)my * w + mx];
			}
			sm.C[k] = v;
		}
		__syncthreads();

		// Stage 2: noise and sig_raw = lap / (2 noise), halo 2
		// (src/filters.cuh:86-135).
		for (int k = tid; k < SH * SW; k += NT) {
			const int lx = k % SW, ly = k / SW;
			const int gx = x0 - 2 + lx, gy = y0 - 2 + ly;
			double nz = 1, s = 0;
			if (gx < xe + 2 && gy < ye + 2) {
				const int mx = border_index(gx, w, mode), my = border_index(gy, h, mode);
				if (mx >= 0 && my >= 0) {
					const long long mi = (long long)my * w + mx;
					if (fd.error) {
						nz = fd.error[mi];
					} else {
						int cx = (mode == NEAREST ? mx : gx) - x0 + 4;
						int cy = (mode == NEAREST ? my : gy) - y0 + 4;
						double v[25];
#pragma unroll
						for (int dy = 0; dy < 5; ++dy)
#pragma unroll
							for (int dx = 0; dx < 5; ++dx)
								v[dy * 5 + dx] = sm.C[(cy - 2 + dy) * CW + cx - 2 + dx];
						double m = median_network(v);
						double g = fd.gain_map ? fd.gain_map[mi] : fd.gain;
						double rn = fd.rn_map ? fd.rn_map[mi] : fd.rn;
						m = m < SIGNAL_FLOOR ? SIGNAL_FLOOR : m;
						nz = sqrt(rn * rn + g * m) / g;
					}
					// Laplacian at the folded position (nearest neighbours
					// for mirror/reflect/nearest), or on the extended tile.
					int cx, cy, xl, xr, yu, yd;
					if (mode == WRAP || mode == CONSTANT) {
						cx = gx - x0 + 4;
						cy = gy - y0 + 4;
						xl = cx - 1;
						xr = cx + 1;
						yu = cy - 1;
						yd = cy + 1;
					} else {
						cx = mx - x0 + 4;
						cy = my - y0 + 4;
						xl = clampi(mx - 1, 0, w - 1) - x0 + 4;
						xr = clampi(mx + 1, 0, w - 1) - x0 + 4;
						yu = clampi(my - 1, 0, h - 1) - y0 + 4;
						yd = clampi(my + 1, 0, h - 1) - y0 + 4;
					}
					double c = sm.C[cy * CW + cx] / 4;
					double up = c - sm.C[yu * CW + cx] / 4;
					double down = c - sm.C[yd * CW + cx] / 4;
					double left = c - sm.C[cy * CW + xl] / 4;
					double right = c - sm.C[cy * CW + xr] / 4;
					double lap = (positive(up + left) + positive(up + right)) +
						(positive(down + left) + positive(down + right));
					s = lap / (2 * nz);
				}
			}
			sm.NZ[k] = nz;
			sm.S[k] = s;
			const int ox = lx - 2, oy = ly - 2;
			if (ox >= 0 && oy >= 0 && ox < TW && oy < TH && gx < xe && gy < ye &&
				!((sm.hole[oy * WPR + (ox >> 5)] >> (ox & 31)) & 1u) && s > prm.tmin) {
				int slot = atomicAdd(&sm.n5, 1);
				sm.q5[slot] = oy * TW + ox;
			}
		}
		__syncthreads();

		// Stage 3: significance where it can pass a threshold
		// (src/filters.cuh:137-146), S1/S2 bits and the seed queue.
		const int n5 = sm.n5;
		for (int q = tid; q < n5; q += NT) {
			const int pos = sm.q5[q], ox = pos % TW, oy = pos / TW;
			double v[25];
			bool nan = false;
#pragma unroll
			for (int dy = 0; dy < 5; ++dy)
#pragma unroll
				for (int dx = 0; dx < 5; ++dx) {
					double x = sm.S[(oy + dy) * SW + ox + dx];
					nan |= isnan(x);
					v[dy * 5 + dx] = x;
				}
			const double center = v[12];
			double med;
			if (nan) {
				double copy[25];
#pragma unroll
				for (int i = 0; i < 25; ++i)
					copy[i] = v[i];
				med = window_median_exact(copy, 25);
			} else {
				med = median_network(v);
			}
			const double sig = center - med;
			const uint32_t bit = 1u << (ox & 31);
			const int word = oy * WPR + (ox >> 5);
			if (sig > prm.cr)
				atomicOr(&sm.s1[word], bit);
			if (sig > prm.nb)
				atomicOr(&sm.s2[word], bit);
			if (sig > prm.cr && !(sm.excl[word] & bit)) {
				int slot = atomicAdd(&sm.nseed, 1);
				sm.qs[slot] = pos;
				sm.qsig[slot] = sig;
			}
		}
		__syncthreads();

		// Stage 4: fine structure at seeds, one warp per seed
		// (src/filters.cuh:148-175).
		const int nseed = sm.nseed;
		for (int q = warp; q < nseed; q += NT / 32) {
			const int pos = sm.qs[q], ox = pos % TW, oy = pos / TW;
			double m3[2] = {INFINITY, INFINITY};
#pragma unroll
			for (int s = 0; s < 2; ++s) {
				const int j = lane + 32 * s;
				if (j < 49) {
					int qx = x0 + ox + j % 7 - 3, qy = y0 + oy + j / 7 - 3;
					double m;
					if (mode == CONSTANT && (qx < 0 || qx >= w || qy < 0 || qy >= h)) {
						m = 0;
					} else {
						if (mode == NEAREST) {
							qx = clampi(qx, 0, w - 1);
							qy = clampi(qy, 0, h - 1);
						}
						const double *c = &sm.C[(qy - y0 + 4) * CW + qx - x0 + 4];
						m = median9(c[-CW - 1], c[-CW], c[-CW + 1], c[-1], c[0], c[1],
							c[CW - 1], c[CW], c[CW + 1]);
					}
					m3[s] = m;
				}
			}
			const double med3c = __shfl_sync(0xffffffffu, m3[0], 24);
			const double med7 = warp_rank64(m3[0], m3[1], 24);
			if (lane == 0) {
				double fine = (med3c - med7) / sm.NZ[(oy + 2) * SW + ox + 2];
				fine = fine < FINE_FLOOR ? FINE_FLOOR : fine;
				if (sm.qsig[q] / fine > prm.contrast)
					atomicOr(&sm.cand[oy * WPR + (ox >> 5)], 1u << (ox & 31));
			}
		}
		__syncthreads();

		uint32_t *s1_p = plane_ptr(fd, P_S1), *s2_p = plane_ptr(fd, P_S2);
		uint32_t *cand_p = plane_ptr(fd, P_CAND);
		for (int k = tid; k < TH * WPR; k += NT) {
			int gy = y0 + k / WPR, gw = (x0 >> 5) + k % WPR;
			if (gy < h && gw < words) {
				long long o = (long long)gy * words + gw;
				s1_p[o] = sm.s1[k];
				s2_p[o] = sm.s2[k];
				cand_p[o] = sm.cand[k];
			}
		}
		__syncthreads();
	}
}

} // namespace cb

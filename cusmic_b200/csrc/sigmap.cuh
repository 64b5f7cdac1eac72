// The first pass's sig_raw map of noise-model frames.
//
// A high-list candidate's significance needs sig_raw at the 25 cells of its
// 5 x 5 window (src/filters.cuh:125-146), and on a noise-model frame each of
// those needs its own 5 x 5 median of clean (src/filters.cuh:107-123).
// Candidates cluster (a cosmic ray, a star core), so their windows overlap:
// the union of the windows is about 8 cells per candidate, against 25 cells
// each evaluated separately.  region_sig_kernel therefore evaluates sig_raw
// and the noise once at every pixel within two of a HIGH pixel (the union of
// the windows of every high-list candidate, whose classes classify_kernel
// wrote into the HIGH plane) and stores both; candidate_high_kernel then
// reads its window from the map.  The values are computed by the same
// functions the candidate kernel uses on its border path (noise_model_at,
// lap_at), so they are the same bits.
//
// Two launches: region_list_kernel lists the map's pixels (one warp per
// growth item of GROW_ROWS rows x 32 bit words, a lane per word: a 5 x 5
// dilation of the HIGH plane on bit words, one list append per item), then
// region_sig_kernel evaluates one listed pixel per thread.  Within an item the
// list runs row by row, so neighbouring threads hold neighbouring pixels and
// their window loads coalesce.  The list lives in the target list's buffer,
// which the first pass fills only later, in its growth step.
#pragma once

#include "common.cuh"
#include "detect.cuh"
#include "incremental.cuh"
#include "kernels.cuh"

namespace cb {

// Horizontal dilation by two of a 36-bit row window (bit_window): bits
// 2 .. 33 of the result (the word's pixels) are exact.
__device__ __forceinline__ unsigned long long dilate_row2(unsigned long long e)
{
	return e | (e << 1) | (e >> 1) | (e << 2) | (e >> 2);
}

// The 36-bit window of row y of a plane read by the non-coherent path (the
// plane is not written while the kernel runs); zero past the row or frame.
__device__ __forceinline__ unsigned long long nc_window(const uint32_t *plane, int words, int h, int y,
	int k)
{
	if (k >= words || y < 0 || y >= h)
		return 0ull;
	const uint32_t *row = plane + (long long)y * words;
	const unsigned long long c = __ldg(row + k);
	const unsigned long long l = k > 0 ? __ldg(row + k - 1) : 0u;
	const unsigned long long r = k + 1 < words ? __ldg(row + k + 1) : 0u;
	return (l >> 30) | (c << 2) | ((r & 3ull) << 34);
}

__global__ void __launch_bounds__(256)
region_list_kernel(const FrameDesc *__restrict__ frames, const FrameState *__restrict__ state,
	const int4 *__restrict__ items, int nitems, Control *ctl, uint2 *list)
{
	const int lane = threadIdx.x & 31;
	const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
	for (int i = gw; i < nitems; i += nw) {
		const int4 it = items[i];
		const int f = it.x;
		if (!state[f].active)
			continue; // warp-uniform
		const FrameDesc &fd = frames[f];
		if (!fd.sig_raw)
			continue; // warp-uniform: an error-map frame
		const int w = fd.w, h = fd.h, words = fd.words, y0 = it.y, n = it.w - it.y, k = it.z + lane;
		const uint32_t *hp = plane_ptr(fd, P_HIGH);
		// The word's valid pixel bits (the dilation spreads past the row end).
		const uint32_t clip = k >= words ? 0u : 32 * k + 32 <= w ? 0xffffffffu : (1u << (w - 32 * k)) - 1u;
		unsigned long long d[GROW_ROWS + 4];
#pragma unroll
		for (int r = 0; r < GROW_ROWS + 4; ++r) // loads only: one round trip
			d[r] = r < n + 4 ? nc_window(hp, words, h, y0 - 2 + r, k) : 0ull;
#pragma unroll
		for (int r = 0; r < GROW_ROWS + 4; ++r)
			d[r] = dilate_row2(d[r]);
		uint32_t need[GROW_ROWS];
		int cnt = 0;
#pragma unroll
		for (int j = 0; j < GROW_ROWS; ++j) {
			need[j] = j < n ? (uint32_t)((d[j] | d[j + 1] | d[j + 2] | d[j + 3] | d[j + 4]) >> 2) & clip : 0u;
			cnt += __popc(need[j]);
		}
		if (!__any_sync(0xffffffffu, cnt != 0))
			continue;
		// Row-major order within the item: row j's pixels of every lane, then
		// row j + 1's.
		int row_off[GROW_ROWS], total = 0;
#pragma unroll
		for (int j = 0; j < GROW_ROWS; ++j) {
			const int c = __popc(need[j]), o = warp_exclusive_count(c);
			row_off[j] = total + o;
			total += __shfl_sync(0xffffffffu, o + c, 31);
		}
		unsigned long long base = 0;
		if (lane == 0)
			base = atomicAdd(&ctl->n_region, (unsigned long long)total);
		base = __shfl_sync(0xffffffffu, base, 0);
#pragma unroll
		for (int j = 0; j < GROW_ROWS; ++j) {
			unsigned long long at = base + row_off[j];
			const unsigned rowpix = (unsigned)((long long)(y0 + j) * w + 32 * k);
			for (uint32_t b = need[j]; b; b &= b - 1)
				list[at++] = make_uint2((unsigned)f, rowpix + __ffs(b) - 1);
		}
	}
}

// sig_raw and the noise of each listed pixel, one per thread.
__global__ void __launch_bounds__(256, 3)
region_sig_kernel(const FrameDesc *__restrict__ frames, const uint2 *__restrict__ list,
	const Control *ctl, DetectParams prm)
{
	const long long n = (long long)ctl->n_region;
	const int mode = prm.mode, lm = lap_mode(mode);
	for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
	     e += (long long)gridDim.x * blockDim.x) {
		const uint2 t = list[e];
		const FrameDesc &fd = frames[t.x];
		const int w = fd.w, x = (int)(t.y % (unsigned)w), y = (int)(t.y / (unsigned)w);
		double nz, lap;
		if (x >= 2 && y >= 2 && x + 2 < w && y + 2 < fd.h) {
			// No border mapping: the window straight from clean (the same
			// 25 values, so the same median).
			double v[25];
			const double *src = fd.clean + t.y - 2 * (long long)w - 2;
#pragma unroll
			for (int a = 0; a < 5; ++a)
#pragma unroll
				for (int b = 0; b < 5; ++b)
					v[a * 5 + b] = src[(long long)a * w + b];
			lap = lap_formula(v[12], v[7], v[17], v[11], v[13]);
			nz = noise_from_median(fd, t.y, median_network(v));
		} else {
			nz = noise_model_at(fd, x, y, mode);
			lap = lap_at(fd, x, y, lm);
		}
		fd.noise[t.y] = nz;
		fd.sig_raw[t.y] = lap / (2 * nz);
	}
}

} // namespace cb

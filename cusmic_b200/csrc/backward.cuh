// Adjoint of the cleaned pixels with the detection mask frozen.
//
// With the final mask fixed, the forward is piecewise linear in (data, bg):
//   unflagged finite pixel p: out_p = (x_p + bg_p) - bg_p     -> d/dx_p = 1
//   non-finite pixel p:       out_p = x_p (returned as is)     -> identity
//   flagged pixel p:          out_p = sel(x_d + bg_d) - bg_p, where sel is the
//     replacement median over the final donors: one donor d (odd count) or
//     the two central donors with weight 1/2 each (even count).
// So dL/dx_d += w_d g_p, dL/dbg_d += w_d g_p and dL/dbg_p -= g_p.  The donor
// selected at a rank is recomputed (not stored): donors are ordered by their
// IEEE total-order key, ties by lowest linear index.
#pragma once
#include "common.cuh"
#include "kernels.cuh"

namespace cb {

// Pass-through part: grad_data = g off the mask, 0 on it; with background
// maps, grad_bg = -g on the mask and 0 elsewhere.
__global__ void __launch_bounds__(256)
bwd_dense_kernel(const FrameDesc *__restrict__ frames, const int2 *__restrict__ rows, int nrows,
	const double *__restrict__ g, double *__restrict__ gx, double *__restrict__ gbg_map,
	const long long *__restrict__ offsets)
{
	const int lane = threadIdx.x & 31;
	const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
	for (int r = gw; r < nrows; r += nw) {
		const int2 item = rows[r];
		const FrameDesc &fd = frames[item.x];
		const uint32_t *crm = plane_ptr(fd, P_CRMASK) + (long long)item.y * fd.words;
		const long long base = offsets[item.x] + (long long)item.y * fd.w;
		for (int x = lane; x < fd.w; x += 32) {
			const bool flagged = (crm[x >> 5] >> (x & 31)) & 1u;
			const double gi = g[base + x];
			gx[base + x] = flagged ? 0.0 : gi;
			if (gbg_map)
				gbg_map[base + x] = flagged ? -gi : 0.0;
		}
	}
}

// data + bg of an in-frame pixel: the value the forward's replacement compared
// (donors are finite inputs).
__device__ __forceinline__ double donor_value(const FrameDesc &fd, long long i)
{
	double c = fd.data[i];
	if (fd.has_bg)
		c += 1 * (fd.bg_map ? fd.bg_map[i] : fd.bg);
	return c;
}

// Linear index of the donor at `rank` in (key, linear index) order, for a
// window of at most 32 cells held one per lane (key = ~0 for non-donors).
__device__ __forceinline__ int donor_at_rank32(unsigned long long key, int idx, int rank)
{
	const int lane = threadIdx.x & 31;
	unsigned long long v = key;
#pragma unroll
	for (int span = 2; span <= 32; span *= 2) {
#pragma unroll
		for (int step = span / 2; step; step /= 2) {
			unsigned long long peer = __shfl_xor_sync(0xffffffffu, v, step);
			bool lower = ((lane & span) == 0) == ((lane & step) == 0);
			v = lower ? (peer < v ? peer : v) : (v < peer ? peer : v);
		}
	}
	const unsigned long long k = __shfl_sync(0xffffffffu, v, rank);
	const int less = __popc(__ballot_sync(0xffffffffu, key < k));
	unsigned same = __ballot_sync(0xffffffffu, key == k);
	for (int t = rank - less; t > 0; --t)
		same &= same - 1;
	return __shfl_sync(0xffffffffu, idx, __ffs(same) - 1);
}

// Same for windows larger than 32 cells: radix select of the key, then the
// (rank - less)-th donor with that key in row-major (= linear index) order.
__device__ long long donor_at_rank_large(const FrameDesc &fd, const uint32_t *don,
	const uint32_t *crm, Window win, int rank)
{
	const int lane = threadIdx.x & 31;
	const int ww = win.x1 - win.x0 + 1, area = ww * (win.y1 - win.y0 + 1);
	unsigned long long prefix = 0, used = 0;
	int r = rank;
	for (int bit = 63; bit >= 0; --bit) {
		const unsigned long long flag = 1ull << bit;
		int below = 0;
		for (int pos = lane; pos < area; pos += 32) {
			int x = win.x0 + pos % ww, y = win.y0 + pos / ww;
			if (!donor_at(don, crm, fd.words, x, y))
				continue;
			unsigned long long k = order_key(donor_value(fd, (long long)y * fd.w + x));
			below += (k & used) == prefix && !(k & flag);
		}
		below = warp_sum_int(below);
		used |= flag;
		if (r >= below) {
			prefix |= flag;
			r -= below;
		}
	}
	// r is now the number of equal keys to skip in row-major order.
	for (int pos0 = 0; pos0 < area; pos0 += 32) {
		const int pos = pos0 + lane;
		bool match = false;
		int x = 0, y = 0;
		if (pos < area) {
			x = win.x0 + pos % ww;
			y = win.y0 + pos / ww;
			match = donor_at(don, crm, fd.words, x, y) &&
				order_key(donor_value(fd, (long long)y * fd.w + x)) == prefix;
		}
		unsigned m = __ballot_sync(0xffffffffu, match);
		int c = __popc(m);
		if (r < c) {
			for (int t = r; t > 0; --t)
				m &= m - 1;
			int src = __ffs(m) - 1;
			int sx = __shfl_sync(0xffffffffu, x, src), sy = __shfl_sync(0xffffffffu, y, src);
			return (long long)sy * fd.w + sx;
		}
		r -= c;
	}
	return -1; // unreachable when rank < donor count
}

// One warp per flagged pixel: recompute its final replacement window and
// donors, scatter w * g to the selected donor(s).
__global__ void __launch_bounds__(256)
bwd_scatter_kernel(const FrameDesc *__restrict__ frames, const uint2 *__restrict__ list,
	const unsigned long long *count, const long long *__restrict__ offsets,
	const double *__restrict__ g, double *gx, double *gbg_map, double *gbg_scalar)
{
	const int lane = threadIdx.x & 31;
	const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
	const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
	const long long n = (long long)*count;
	for (long long e = gw; e < n; e += nw) {
		const uint2 t = list[e];
		const FrameDesc &fd = frames[t.x];
		const int w = fd.w, h = fd.h;
		const int x = (int)(t.y % (unsigned)w), y = (int)(t.y / (unsigned)w);
		const uint32_t *don = plane_ptr(fd, P_DONOR), *crm = plane_ptr(fd, P_CRMASK);
		const long long off = offsets[t.x];
		const double gp = g[off + t.y];
		const int limit = max(w, h);
		for (int r = 2; r <= limit; ++r) {
			Window win = {max(0, x - r), min(w - 1, x + r), max(0, y - r), min(h - 1, y + r)};
			const int ww = win.x1 - win.x0 + 1, area = ww * (win.y1 - win.y0 + 1);
			long long d_lo, d_hi;
			int nd;
			if (area <= 32) {
				unsigned long long key = ~0ull;
				int idx = 0;
				bool d = false;
				if (lane < area) {
					int cx = win.x0 + lane % ww, cy = win.y0 + lane / ww;
					d = donor_at(don, crm, fd.words, cx, cy);
					idx = cy * w + cx;
					if (d)
						key = order_key(donor_value(fd, idx));
				}
				nd = __popc(__ballot_sync(0xffffffffu, d));
				if (!nd)
					continue;
				d_lo = donor_at_rank32(key, idx, (nd - 1) / 2);
				d_hi = nd % 2 ? d_lo : donor_at_rank32(key, idx, nd / 2);
			} else {
				int cnt = 0;
				for (int pos = lane; pos < area; pos += 32)
					cnt += donor_at(don, crm, fd.words, win.x0 + pos % ww, win.y0 + pos / ww);
				nd = warp_sum_int(cnt);
				if (!nd)
					continue;
				d_lo = donor_at_rank_large(fd, don, crm, win, (nd - 1) / 2);
				d_hi = nd % 2 ? d_lo : donor_at_rank_large(fd, don, crm, win, nd / 2);
			}
			if (lane == 0) {
				// Odd count: the middle donor, weight 1.  Even: the two central
				// donors, weight 1/2 each (midpoint either form).
				const double wl = nd % 2 ? gp : gp / 2, wh = nd % 2 ? 0.0 : gp / 2;
				atomicAdd(&gx[off + d_lo], wl);
				if (!(nd % 2))
					atomicAdd(&gx[off + d_hi], wh);
				if (gbg_map) {
					atomicAdd(&gbg_map[off + d_lo], wl);
					if (!(nd % 2))
						atomicAdd(&gbg_map[off + d_hi], wh);
				}
				if (gbg_scalar && fd.has_bg)
					atomicAdd(&gbg_scalar[t.x], (wl + wh) - gp);
			}
			break;
		}
	}
}

} // namespace cb

// prepare (reference src/image.cuh:24-48) and the first pass's dense
// detection in one streaming kernel, for batches whose frames all have an
// error map, no background, widths that are multiples of 16 and 16-byte
// aligned data, mask and output buffers (the stacked-exposure workloads).
//
// Without a background the working pixels are the input pixels, except at
// holes (non-finite inputs), which prepare zeroes and the hole fill then
// replaces.  So sig_bulk_kernel's Laplacian bound can be evaluated on the
// input rows themselves, in the same pass that writes the working pixels, the
// HOLE / EXCL / DONOR words and the hole list, instead of writing the working
// pixels and streaming them back in: 17.4 instead of 25.4 bytes per pixel for
// the two steps.  Only the pixels whose Laplacian reads a hole depend on the
// fill.  A hole enters the Laplacian as -inf, so such a pixel (its own value
// finite) has a difference of +inf to that neighbour and a bound of +inf,
// which passes every threshold; classify_kernel recomputes the Laplacian of an
// entry listed with +inf from the filled working pixels.  A pixel whose own
// value is finite has finite or +inf differences to its neighbours, so no NaN
// can reach its bound.  Holes themselves are not listed: their significance is
// zero (src/filters.cuh:137-146) and the candidate kernels drop them anyway.
// Every other pixel gets exactly the bound sig_bulk_kernel computes from the
// working pixels (the same values, the same operations), so the lists, and
// everything after them, are those of the two-kernel path.
//
// The block layout is sig_bulk_kernel's: one producer thread streams the
// item's rows (BK_COLS columns plus halo columns, border-mapped rows and
// columns for the Laplacian) of the input into the ring by bulk copies, and
// for the item's own rows the mask bytes of its columns into a second ring;
// four consumer warps evaluate four columns per lane.  A consumer lane handles
// the prepare step of each own row (holes, exclusions, donors, the working
// pixels as two 16-byte stores) when the row arrives in the ring; the bit
// words of the warp's 128 columns are assembled from the lanes' 4-bit groups
// by shuffles.  Per-frame facts are set once per item and warp.
//
// The block floors of error maps depend on the maps only, so they are computed
// before this kernel (prep_init_kernel, with the call's state and zeroing);
// the hole fill runs after it.
//
// Every wait is bounded as in sig_bulk_kernel.  The frames' layout is checked
// again on the device: a frame that does not satisfy it stops the kernel as a
// fault instead of issuing a copy it cannot make.
#pragma once
#include "bulk.cuh"
#include "kernels.cuh"

namespace cb {

constexpr int PD_BLOCKS_PER_SM = 4; // registers: at 5 blocks the kernel spills (measured slower)

// The frames prep_detect_kernel serves (besides an error map and maxiter > 0,
// which the caller checks).
CB_HD bool prep_detect_ok(const FrameDesc &fd)
{
	return fd.error && !fd.bg_map && !fd.has_bg && fd.w % 16 == 0 &&
		(((uintptr_t)fd.data | (uintptr_t)fd.mask | (uintptr_t)fd.clean) & 15u) == 0 &&
		(!fd.out || fd.out == fd.clean);
}

// Issue one ring row: the input row's copies (as bulk_issue) and, for an own
// row of a frame with a mask, the mask bytes of the item's columns.
__device__ __forceinline__ void pd_issue(BulkRing &R, uint8_t (*M)[BK_COLS], int slot, const BulkRow &b,
	const double *data, const uint8_t *mrow, unsigned mbytes)
{
	double *row = R.c[slot];
	R.shift[slot] = b.shift;
	// The consumers' reads of this slot (generic proxy) before the copies'
	// writes (async proxy).
	asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
	mbar_expect_tx(&R.full[slot], b.bytes + (mrow ? mbytes : 0u));
	if (b.n)
		bulk_copy(row + b.cell, b.src < 0 ? bulk_zero_row : data + b.src, 8u * b.n, &R.full[slot]);
	if (mrow)
		bulk_copy(M[slot], mrow, mbytes, &R.full[slot]);
	if (b.hsrc != NO_COPY)
		cp_async8(row + b.hcell, data + b.hsrc);
	if (b.tsrc != NO_COPY)
		cp_async8(row + b.tcell, data + b.tsrc);
	if (b.lsrc != NO_COPY)
		cp_async8(row + b.lcell, b.lsrc < 0 ? bulk_zero_row : data + b.lsrc);
	if (b.rsrc != NO_COPY)
		cp_async8(row + b.rcell, b.rsrc < 0 ? bulk_zero_row : data + b.rsrc);
	mbar_arrive_cp_async(&R.full[slot]);
}

// Producer (one thread): bulk_producer over the input rows, plus the mask
// rows.  Returns false after a fault.
__device__ __forceinline__ bool pd_producer(BulkRing &R, uint8_t (*M)[BK_COLS],
	const FrameDesc *__restrict__ frames, const FrameState *state, const int4 *__restrict__ items,
	int nitems, int lm, Control *ctl, int &g, BulkRow (&base)[2])
{
	int next = atomicAdd(&ctl->ticket, 1);
	for (;;) {
		int t = -1;
		while (next < nitems) {
			const int cand = next;
			next = atomicAdd(&ctl->ticket, 1);
			const int4 it = items[cand];
			if (!state[it.x].active)
				continue;
			if (!prep_detect_ok(frames[it.x])) // the host never lays such a frame out here
				return false;
			t = cand;
			break;
		}
		if (t < 0) { // end of the list: an end marker in the next ring row
			const int slot = g & (BK_SLOTS - 1);
			if (g >= BK_SLOTS && !mbar_wait(&R.empty[slot], ((g / BK_SLOTS) - 1) & 1, &R.abort))
				return false;
			R.meta[slot] = make_int2(-1, 0);
			mbar_arrive(&R.full[slot]);
			mbar_arrive(&R.full[slot]);
			++g;
			return true;
		}
		const int4 it = items[t];
		const FrameDesc &fd = frames[it.x];
		const int w = fd.w, h = fd.h, x0 = it.y, y0 = it.z, y1 = it.w;
		const double *data = fd.data;
		const uint8_t *mask = fd.mask;
		// Mask bytes of an own row: the item's columns, a multiple of 16.
		const unsigned mbytes = (unsigned)(w - x0 < BK_COLS ? w - x0 : BK_COLS);
		const int ra = y0 - 1 < 0 ? 0 : y0 - 1; // first in-frame row of the item
		base[0] = bulk_row(w, h, lm, 0, x0, ra);
		base[1] = bulk_row(w, h, lm, 0, x0, ra + 1 < h ? ra + 1 : ra);
		for (int r = y0 - 1; r <= y1; ++r) {
			const int slot = g & (BK_SLOTS - 1);
			const int d = r - ra;
			const BulkRow b = r < 0 || r >= h ? bulk_row(w, h, lm, 0, x0, r)
				: shift_row(base[d & 1], (long long)(d & ~1) * w);
			if (g >= BK_SLOTS && !mbar_wait(&R.empty[slot], ((g / BK_SLOTS) - 1) & 1, &R.abort))
				return false;
			if (r == y0 - 1)
				R.meta[slot] = make_int2(t, y1);
			const uint8_t *mrow = mask && r >= y0 && r < y1 ? mask + (long long)r * w + x0 : nullptr;
			pd_issue(R, M, slot, b, data, mrow, mbytes);
			++g;
		}
	}
}

// A ring value as the Laplacian reads it: a quarter of the pixel, or -inf
// for a hole.
__device__ __forceinline__ double pd_quarter(double v)
{
	return isfinite(v) ? v * 0.25 : -INFINITY;
}

// The quarters of a lane's six ring values of a row.  `bad` (warp-uniform):
// some value the warp reads from the row may be a hole, so each is checked;
// otherwise every value a lane in the frame reads is finite.
__device__ __forceinline__ void pd_quarters(const double (&v)[6], bool bad, double (&s)[6])
{
	if (bad) {
#pragma unroll
		for (int i = 0; i < 6; ++i)
			s[i] = pd_quarter(v[i]);
	} else {
#pragma unroll
		for (int i = 0; i < 6; ++i)
			s[i] = v[i] * 0.25;
	}
}

// Whether a row read only for its vertical neighbours (values 1..4 of a lane)
// holds a hole under any lane in the frame (warp-uniform).
__device__ __forceinline__ bool pd_row_bad(const double (&v)[6], bool valid)
{
	return __any_sync(0xffffffffu,
		valid && (!isfinite(v[1]) || !isfinite(v[2]) || !isfinite(v[3]) || !isfinite(v[4])));
}

// Bits 0..3: the nonzero bytes of a word of four mask bytes.
__device__ __forceinline__ uint32_t mask_nibble(uint32_t m)
{
	uint32_t t = m | (m >> 4);
	t |= t >> 2;
	t |= t >> 1;
	return ((t & 0x01010101u) * 0x01020408u) >> 24;
}

// What a consumer warp gathers over an item for the frame's state.
struct PdFacts {
	uint32_t hole, allowed; // any hole, any allowed (without a background: any donor)
	int donors;             // donors among the words this lane stored
};

// The prepare step of one own row for a lane's four columns x .. x + 3 (all
// in the frame or none: w is a multiple of 16): the working pixels, the bit
// words (lane 8j stores word j of the warp's 128 columns, from the lanes'
// 4-bit groups OR-ed across the eight lanes by shuffles; DONOR is the
// complement of EXCL within the frame) and the hole list.  Returns the lane's
// hole bits (bit i = column x + i); `any_hole`: some lane has one; `bad`:
// some value the warp reads from the row, halo columns included, is a hole.
__device__ __forceinline__ uint32_t pd_prepare_row(const FrameDesc &fd, int f, int y, int x, bool valid,
	bool has_mask, const double (&v)[6], uint32_t mbytes, Control *ctl, uint2 *holes, PdFacts &acc,
	bool &any_hole, bool &bad)
{
	const int lane = threadIdx.x & 31;
	uint32_t hn = 0;
#pragma unroll
	for (int i = 0; i < 4; ++i)
		hn |= (uint32_t)!isfinite(v[i + 1]) << i;
	if (!valid)
		hn = 0;
	any_hole = __any_sync(0xffffffffu, hn != 0);
	bad = any_hole || __any_sync(0xffffffffu, valid && (!isfinite(v[0]) || !isfinite(v[5])));
	const long long rowpix = (long long)y * fd.w;
	if (valid) {
		double c[4] = {v[1], v[2], v[3], v[4]};
		if (hn) {
#pragma unroll
			for (int i = 0; i < 4; ++i)
				c[i] = (hn >> i) & 1u ? 0.0 : c[i];
		}
		double2 *dst = reinterpret_cast<double2 *>(fd.clean + rowpix + x);
		dst[0] = make_double2(c[0], c[1]);
		dst[1] = make_double2(c[2], c[3]);
	}
	const int sh = 4 * (lane & 7);
	uint32_t ew = 0, hw = 0;
	if (has_mask || any_hole) { // warp-uniform
		ew = (hn | (has_mask && valid ? mask_nibble(mbytes) : 0u)) << sh;
#pragma unroll
		for (int o = 1; o < 8; o <<= 1)
			ew |= __shfl_xor_sync(0xffffffffu, ew, o);
	}
	if (any_hole) {
		hw = hn << sh;
#pragma unroll
		for (int o = 1; o < 8; o <<= 1)
			hw |= __shfl_xor_sync(0xffffffffu, hw, o);
	}
	if ((lane & 7) == 0 && valid) {
		const uint32_t dw = ~ew & (fd.w - x >= 32 ? 0xffffffffu : 0x0000ffffu);
		const long long at = (long long)y * fd.words + (x >> 5);
		plane_ptr(fd, P_HOLE)[at] = hw;
		plane_ptr(fd, P_EXCL)[at] = ew;
		plane_ptr(fd, P_DONOR)[at] = dw;
		acc.donors += __popc(dw);
		acc.allowed |= dw;
	}
	acc.hole |= hn;
	if (any_hole) { // the row's holes for the fill
		unsigned long long slot = warp_append(&ctl->n_holes, __popc(hn));
		for (uint32_t b = hn; b; b &= b - 1)
			holes[slot++] = make_uint2((unsigned)f, (unsigned)(rowpix + x + __ffs(b) - 1));
	}
	return hn;
}

// Consumer warps: bulk_consumer over the input rows, with the prepare step of
// each own row.  Returns false after a fault.
__device__ __forceinline__ bool pd_consumer(BulkRing &R, const uint8_t (*M)[BK_COLS],
	const FrameDesc *__restrict__ frames, FrameState *state, const int4 *__restrict__ items,
	Control *ctl, uint2 *holes, PreCand *pre, int *pre_counts)
{
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const int ct = warp * 32 + lane; // 0 .. 127
	const int c0 = 2 + 4 * ct;       // cell of the lane's first column (before the row's shift)
	const unsigned below = (1u << lane) - 1u;
	int g = 0;
	bool ok = true;
	for (;;) {
		ok = __all_sync(0xffffffffu, mbar_wait(&R.full[g & (BK_SLOTS - 1)], (g / BK_SLOTS) & 1, &R.abort));
		if (!ok)
			break;
		const int2 meta = R.meta[g & (BK_SLOTS - 1)];
		if (meta.x < 0)
			break;
		const int t = meta.x, y1 = meta.y;
		const int4 it = items[t];
		const int f = it.x, x0 = it.y, y0 = it.z;
		const FrameDesc &fd = frames[f];
		const int w = fd.w, x = x0 + 4 * ct;
		const bool valid = x < w;
		const bool has_mask = fd.mask != nullptr;
		// High word of the block threshold (all ones: not a pixel).
		unsigned thr = 0xffffffffu;
		if (valid) {
			const double T = fd.floors[(y0 / FLOOR_BLOCK) * ((w + FLOOR_BLOCK - 1) / FLOOR_BLOCK) +
				x / FLOOR_BLOCK].thr;
			thr = hi_word(T >= 0 ? T : 0.0); // NaN lists everything
		}
		PdFacts acc{0u, 0u, 0};
		ok = __all_sync(0xffffffffu,
			mbar_wait(&R.full[(g + 1) & (BK_SLOTS - 1)], ((g + 1) / BK_SLOTS) & 1, &R.abort));
		if (!ok)
			break;
		// Row y0 - 1 (values) and row y0 (values and neighbours), as quarters;
		// row y0 is an own row.
		double q[4], up[4], ql, qr;
		uint32_t hcur;
		bool hrow; // row y has a hole
		{
			const int s0 = g & (BK_SLOTS - 1), s1 = (g + 1) & (BK_SLOTS - 1);
			double u[6], c[6];
			load_six(R.c[s0], c0, R.shift[s0], u);
			load_six(R.c[s1], c0, R.shift[s1], c);
			const uint32_t mb = has_mask && valid ? *reinterpret_cast<const uint32_t *>(&M[s1][4 * ct]) : 0u;
			__syncwarp();
			if (lane == 0) { // both rows are in registers now
				mbar_arrive(&R.empty[s0]);
				mbar_arrive(&R.empty[s1]);
			}
			bool bad_c;
			hcur = pd_prepare_row(fd, f, y0, x, valid, has_mask, c, mb, ctl, holes, acc, hrow, bad_c);
			double su[6], sc[6];
			pd_quarters(u, pd_row_bad(u, valid), su);
			pd_quarters(c, bad_c, sc);
			ql = sc[0];
			qr = sc[5];
#pragma unroll
			for (int i = 0; i < 4; ++i) {
				q[i] = sc[i + 1];
				up[i] = q[i] - su[i + 1];
			}
		}
		PreCand *region = pre + ((long long)t * BK_CWARPS + warp) * BK_REGION;
		int cnt = 0;
#pragma unroll 2
		for (int y = y0; y < y1; ++y) {
			const int gd = g + 2 + (y - y0); // ring row of y + 1
			const int sd = gd & (BK_SLOTS - 1);
			ok = __all_sync(0xffffffffu, mbar_wait(&R.full[sd], (gd / BK_SLOTS) & 1, &R.abort));
			if (!ok)
				break;
			double n[6];
			load_six(R.c[sd], c0, R.shift[sd], n);
			const bool own = y + 1 < y1;
			const uint32_t mb = own && has_mask && valid ? *reinterpret_cast<const uint32_t *>(&M[sd][4 * ct])
				: 0u;
			__syncwarp();
			if (lane == 0)
				mbar_arrive(&R.empty[sd]); // row y + 1 is in registers
			uint32_t hnext = 0;
			bool hrow_next = false, bad_n;
			if (own) // warp-uniform
				hnext = pd_prepare_row(fd, f, y + 1, x, valid, has_mask, n, mb, ctl, holes, acc,
					hrow_next, bad_n);
			else
				bad_n = pd_row_bad(n, valid);
			double s[6];
			pd_quarters(n, bad_n, s);
			// Horizontal differences: left(x+i) = h[i], right(x+i) = -h[i+1].
			double hd[5];
			hd[0] = q[0] - ql;
#pragma unroll
			for (int i = 0; i < 3; ++i)
				hd[i + 1] = q[i] - q[i + 1];
			hd[4] = q[3] - qr;
			const long long pix0 = (long long)y * w + x;
			double lap[4];
#pragma unroll
			for (int i = 0; i < 4; ++i) {
				const double qd = s[i + 1];
				const double d = q[i] - qd;
				const double lft = i == 0 ? hd[0] : -hd[i], rgt = i == 3 ? hd[4] : hd[i + 1];
				lap[i] = (pos_ub(up[i] + lft) + pos_ub(up[i] + rgt)) + (pos_ub(d + lft) + pos_ub(d + rgt));
				up[i] = -d;
				q[i] = qd;
			}
			ql = s[0];
			qr = s[5];
			bool pass[4];
#pragma unroll
			for (int i = 0; i < 4; ++i)
				pass[i] = valid && hi_word(lap[i]) >= thr;
			if (hrow) { // warp-uniform: holes are not listed
#pragma unroll
				for (int i = 0; i < 4; ++i)
					pass[i] = pass[i] && !((hcur >> i) & 1u);
			}
			hcur = hnext;
			hrow = hrow_next;
			if (__any_sync(0xffffffffu, pass[0] | pass[1] | pass[2] | pass[3])) {
#pragma unroll
				for (int i = 0; i < 4; ++i) {
					const unsigned bal = __ballot_sync(0xffffffffu, pass[i]);
					if (pass[i])
						region[cnt + __popc(bal & below)] = PreCand{(unsigned)(pix0 + i), (unsigned)f, lap[i]};
					cnt += __popc(bal);
				}
			}
		}
		if (!ok)
			break;
		// The item's facts for the frame's state.
		const bool any_hole = __any_sync(0xffffffffu, acc.hole != 0);
		const bool any_allowed = __any_sync(0xffffffffu, acc.allowed != 0);
		const int donors = __reduce_add_sync(0xffffffffu, acc.donors);
		if (lane == 0) {
			pre_counts[t * BK_CWARPS + warp] = cnt;
			FrameState &st = state[f];
			if (any_hole)
				set_flag(&st.holes);
			if (any_allowed) {
				set_flag(&st.allowed);
				set_flag(&st.finite);
			}
			if (donors)
				atomicAdd((unsigned long long *)&st.donors_left, (unsigned long long)donors);
		}
		g += y1 - y0 + 2;
	}
	return ok;
}

// The call's first launch on a batch prep_detect_kernel serves: init_kernel's
// state, control and plane zeroing, and in the same grid the error maps'
// block floors (floor_kernel's jobs, which read the maps only), so the floors
// need no launch of their own and overlap the zeroing.
__global__ void __launch_bounds__(256)
prep_init_kernel(FrameState *state, int nf, Control *ctl, int maxiter, unsigned long long cand_cap,
	long long poison_prepare, long long poison_detect, uint4 *zero, long long n16, uint4 *zero2,
	long long n16b, const FrameDesc *__restrict__ frames, const FloorJob *__restrict__ jobs, int njobs,
	DetectParams prm, BlockFloor *floors)
{
	init_state(state, nf, ctl, maxiter, cand_cap, poison_prepare, poison_detect, zero, n16, zero2, n16b);
	floor_jobs(frames, jobs, njobs, prm, floors);
}

__global__ void __launch_bounds__(BK_THREADS, PD_BLOCKS_PER_SM)
prep_detect_kernel(const FrameDesc *__restrict__ frames, FrameState *state, const int4 *__restrict__ items,
	int nitems, DetectParams prm, Control *ctl, uint2 *holes, PreCand *pre, int *pre_counts)
{
	__shared__ BulkRing R;
	__shared__ __align__(128) uint8_t M[BK_SLOTS][BK_COLS]; // mask bytes of own rows
	__shared__ BulkRow base[2]; // the producer's row copies of the current item
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	if (tid == 0) {
		for (int i = 0; i < BK_SLOTS; ++i) {
			mbar_init(&R.full[i], 2); // the producer's transaction bytes and cp.async arrive
			mbar_init(&R.empty[i], BK_CWARPS);
		}
		mbar_init(&R.poison, 1);
		R.abort = 0;
		asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
	}
	__syncthreads();
	// An injected failure of either step (prepare or detection) makes one
	// consumer warp wait on the barrier nothing completes.
	const long long poison = ctl->poison_wait[0] > ctl->poison_wait[1] ? ctl->poison_wait[0]
		: ctl->poison_wait[1];
	bool ok;
	int issued = 0; // ring rows issued (producer warp)
	if (warp == BK_CWARPS)
		ok = lane || pd_producer(R, M, frames, state, items, nitems, lap_mode(prm.mode), ctl, issued, base);
	else if (warp == 0 && blockIdx.x == 0 && poison > 0)
		ok = __all_sync(0xffffffffu, poisoned_wait(&R.poison, &R.abort, poison));
	else
		ok = pd_consumer(R, M, frames, state, items, ctl, holes, pre, pre_counts);
	if (!ok && lane == 0) {
		R.abort = 1;
		atomicOr(&ctl->fault, 1);
	}
	__syncthreads();
	// After a fault: wait (bounded) for the copies still in flight into this
	// block's shared memory.
	if (warp == BK_CWARPS && lane == 0 && R.abort)
		for (int q = issued - BK_SLOTS < 0 ? 0 : issued - BK_SLOTS; q < issued; ++q) {
			const long long t0 = clock64();
			while (!mbar_test(&R.full[q & (BK_SLOTS - 1)], (q / BK_SLOTS) & 1) &&
				clock64() - t0 < BK_WAIT_CYCLES) {
			}
		}
}

} // namespace cb

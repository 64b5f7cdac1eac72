// prepare_kernel for batches of aligned frames, with its inputs staged by
// bulk copies.
//
// prepare_kernel keeps its loads in registers, so the bytes a warp has in
// flight are bounded by the 64 registers of four blocks per SM.  Here every
// warp streams its rows in segments of PB_SEG pixels into two shared-memory
// buffers of its own: lane 0 issues one `cp.async.bulk` for the segment's
// float64 pixels and one for its mask bytes, completing on the buffer's
// mbarrier, while the warp works on the other buffer.  The arithmetic, the
// bit words and the hole list are prepare_row's (reference
// src/image.cuh:24-48): per 32-pixel chunk the same ballots, with the clean
// pixels stored straight from registers.
//
// It serves a batch when every frame is of a kind without a background map
// and satisfies the bulk copies' alignment: width a multiple of 16 (segment
// byte counts multiples of 16) and data and mask 16-byte aligned (every
// segment starts on a 16-byte boundary).  Other batches use prepare_kernel.
//
// Every wait is bounded.  A wait that runs out sets Control::fault and the
// block's abort word (the loop control then stops the frames and the host
// reports a CUDA error); before the warp exits it waits, again bounded, for
// the copies it still has in flight into its buffers.
#pragma once
#include "bulk.cuh"
#include "kernels.cuh"

namespace cb {

constexpr int PB_SEG = 512;   // pixels per segment (16 bit words)
constexpr int PB_WARPS = 8;   // warps per block
constexpr int PB_BLOCKS = 3;  // blocks per SM (shared memory: 3 x 74 KB)
static_assert(PB_SEG % 32 == 0 && PB_SEG / 32 <= 32, "a segment is whole bit words, one per lane");

struct __align__(128) PrepStage {
	double d[2][PB_SEG];        // pixels of the two buffers
	uint8_t m[2][PB_SEG];       // mask bytes
	unsigned long long full[2]; // completion of each buffer's copies
};

// The warps' stages, then the block's abort word and (8 bytes further) the
// barrier of an injected failure.
constexpr size_t PB_SMEM = PB_WARPS * sizeof(PrepStage) + 16;

// The frames prepare_bulk_kernel serves.
CB_HD bool prep_bulk_ok(const FrameDesc &fd)
{
	return !fd.bg_map && fd.w % 16 == 0 && ((uintptr_t)fd.data & 15u) == 0 &&
		((uintptr_t)fd.mask & 15u) == 0;
}

// A warp's walk over its segments: rows r = gw, gw + nw, ..., and segments
// 0 .. ceil(w / PB_SEG) - 1 of each.
struct SegCursor {
	int r, s;
};

__device__ __forceinline__ bool seg_valid(const SegCursor &c, int nrows)
{
	return c.r < nrows;
}

__device__ __forceinline__ void seg_next(SegCursor &c, const FrameDesc *__restrict__ frames,
	const int2 *__restrict__ rows, int nw)
{
	const FrameDesc &fd = frames[rows[c.r].x];
	if (++c.s * PB_SEG >= fd.w) {
		c.s = 0;
		c.r += nw;
	}
}

// Lane 0: the copies of segment c into buffer b.
__device__ __forceinline__ void seg_issue(PrepStage &S, int b, const SegCursor &c,
	const FrameDesc *__restrict__ frames, const int2 *__restrict__ rows)
{
	const int2 item = rows[c.r];
	const FrameDesc &fd = frames[item.x];
	const long long px = (long long)item.y * fd.w + (long long)c.s * PB_SEG;
	const int n = min(PB_SEG, fd.w - c.s * PB_SEG);
	const unsigned bytes = 8u * n + (fd.mask ? (unsigned)n : 0u);
	// The warp's earlier reads of this buffer (generic proxy) before the
	// copy's writes (async proxy).
	asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
	mbar_expect_tx(&S.full[b], bytes);
	bulk_copy(S.d[b], fd.data + px, 8u * n, &S.full[b]);
	if (fd.mask)
		bulk_copy(S.m[b], fd.mask + px, (unsigned)n, &S.full[b]);
}

// ROWMIN: some frames are noise-model frames, whose row minima are written.
// OUT: some frame has a separate output buffer (a background).
template <bool ROWMIN, bool OUT = false>
__global__ void __launch_bounds__(32 * PB_WARPS, PB_BLOCKS)
prepare_bulk_kernel(const FrameDesc *__restrict__ frames, FrameState *state, const int2 *__restrict__ rows,
	int nrows, Control *ctl, uint2 *holes)
{
	extern __shared__ __align__(128) unsigned char pb_smem[];
	PrepStage *stages = reinterpret_cast<PrepStage *>(pb_smem);
	int *abort = reinterpret_cast<int *>(pb_smem + PB_WARPS * sizeof(PrepStage));
	unsigned long long *poison =
		reinterpret_cast<unsigned long long *>(pb_smem + PB_WARPS * sizeof(PrepStage) + 8);
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	PrepStage &S = stages[warp];
	if (threadIdx.x == 0) {
		*abort = 0;
		mbar_init(poison, 1);
	}
	if (lane == 0) {
		mbar_init(&S.full[0], 1);
		mbar_init(&S.full[1], 1);
		asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
	}
	__syncthreads();
	const int gw = blockIdx.x * PB_WARPS + warp, nw = gridDim.x * PB_WARPS;
	SegCursor proc{gw, 0}, iss{gw, 0};
	int issued = 0; // segments issued by this warp
	// Fill both buffers.
	for (int b = 0; b < 2 && seg_valid(iss, nrows); ++b) {
		if (lane == 0)
			seg_issue(S, b, iss, frames, rows);
		seg_next(iss, frames, rows, nw);
		++issued;
	}
	uint32_t any_hole = 0, any_allowed = 0, any_finite = 0;
	int ndonor = 0;
	bool ok = true;
	if (warp == 0 && blockIdx.x == 0 && ctl->poison_wait[0] > 0) // injected failure
		ok = __all_sync(0xffffffffu, poisoned_wait(poison, abort, ctl->poison_wait[0]));
	for (int i = 0; ok && seg_valid(proc, nrows); ++i) {
		const int b = i & 1;
		ok = __all_sync(0xffffffffu, mbar_wait(&S.full[b], (i >> 1) & 1, abort));
		if (!ok)
			break;
		const int2 item = rows[proc.r];
		const int f = item.x, y = item.y;
		const FrameDesc &fd = frames[f];
		const int w = fd.w, words = fd.words;
		const long long rowpix = (long long)y * w, roww = (long long)y * words;
		const int x0 = proc.s * PB_SEG, n = min(PB_SEG, w - x0);
		const bool has_mask = fd.mask != nullptr, has_bg = fd.has_bg;
		const bool rowmin = ROWMIN && fd.floors && !fd.error; // noise-model row minima
		const double bgv = fd.bg;
		double *__restrict__ clean = fd.clean + rowpix + x0;
		// A separate output buffer (a frame with a background): as prepare_row.
		double *__restrict__ out = OUT && fd.out && fd.out != fd.clean ? fd.out + rowpix + x0 : nullptr;
		uint32_t my_h = 0, my_e = 0, my_d = 0, my_m = 0xffffffffu;
#pragma unroll 4
		for (int c = 0; c < PB_SEG / 32; ++c) {
			const int xr = 32 * c + lane;
			if (32 * c >= n)
				break; // warp-uniform
			const bool valid = xr < n;
			bool hole = false, ok_px = false, donor = false;
			double v = 0;
			if (valid) {
				const double d = S.d[b][xr];
				const bool m = has_mask && S.m[b][xr] != 0;
				hole = !isfinite(d);
				ok_px = !hole && !m;
				v = hole ? 0 : d;
				if (has_bg)
					v += 1 * bgv;
				clean[xr] = v;
				if (out)
					out[xr] = hole ? d : v + -1 * bgv;
				donor = ok_px && isfinite(v);
			}
			const uint32_t hw = __ballot_sync(0xffffffffu, hole);
			uint32_t mw = 0xffffffffu;
			if (rowmin)
				mw = __reduce_min_sync(0xffffffffu,
					valid && !hole ? (uint32_t)(order_key(v) >> 32) : 0xffffffffu);
			const uint32_t ew = __ballot_sync(0xffffffffu, valid && !ok_px);
			const uint32_t dw = __ballot_sync(0xffffffffu, donor);
			any_allowed |= __ballot_sync(0xffffffffu, ok_px);
			any_finite |= dw;
			any_hole |= hw;
			ndonor += __popc(dw);
			if (lane == c) {
				my_h = hw;
				my_e = ew;
				my_d = dw;
				my_m = mw;
			}
		}
		// The buffer is read: refill it with the segment after the next.
		__syncwarp();
		if (seg_valid(iss, nrows)) {
			if (lane == 0)
				seg_issue(S, b, iss, frames, rows);
			seg_next(iss, frames, rows, nw);
			++issued;
		}
		const int k = x0 / 32 + lane;
		if (lane < PB_SEG / 32 && 32 * lane < n) {
			plane_ptr(fd, P_HOLE)[roww + k] = my_h;
			plane_ptr(fd, P_EXCL)[roww + k] = my_e;
			plane_ptr(fd, P_DONOR)[roww + k] = my_d;
			if (rowmin)
				plane_ptr(fd, P_ROWMIN)[roww + k] = my_m;
		}
		if (holes && __any_sync(0xffffffffu, my_h != 0)) { // the segment's holes for the fill
			unsigned long long slot = warp_append(&ctl->n_holes, __popc(my_h));
			for (uint32_t hb = my_h; hb; hb &= hb - 1)
				holes[slot++] = make_uint2((unsigned)f, (unsigned)(rowpix + 32 * k + __ffs(hb) - 1));
		}
		seg_next(proc, frames, rows, nw);
		if (proc.s == 0) { // the row is done: its per-frame facts
			if (lane == 0) {
				FrameState &st = state[f];
				if (any_hole)
					set_flag(&st.holes);
				if (any_allowed)
					set_flag(&st.allowed);
				if (any_finite)
					set_flag(&st.finite);
				if (ndonor)
					atomicAdd((unsigned long long *)&st.donors_left, (unsigned long long)ndonor);
			}
			any_hole = any_allowed = any_finite = 0;
			ndonor = 0;
		}
	}
	if (!ok) {
		if (lane == 0) {
			*(volatile int *)abort = 1;
			atomicOr(&ctl->fault, 1);
			// The copies still in flight into this warp's buffers (at most
			// the last two issued) land before the block's shared memory
			// is released.
			for (int q = issued - 2 < 0 ? 0 : issued - 2; q < issued; ++q) {
				const long long t0 = clock64();
				while (!mbar_test(&S.full[q & 1], (q >> 1) & 1) && clock64() - t0 < BK_WAIT_CYCLES) {
				}
			}
		}
		__syncwarp();
	}
}

} // namespace cb

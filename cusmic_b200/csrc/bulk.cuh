// Dense detection pass: one streaming kernel for every frame of a batch,
// whatever its width, alignment or noise model.
//
// What the pass needs from every pixel is only whether its sig_raw =
// lap / (2 noise) can exceed min(cr_threshold, neighbor_threshold); the exact
// value matters for the ~1% of pixels where it can.  So the work is split:
//
//  * block floors (once per call): a lower bound of the noise over every
//    32 x 32 block, turned into a threshold T = 2 min(cr, nb) (1 - 1e-12) x
//    floor.  With an error map floor_kernel takes min(max(error, 0)) over the
//    block (NaN counts as 0), once for each distinct map.  With the noise
//    model (src/filters.cuh:107-123) it stores a lower bound of the block's
//    clean values as an ordered key (from the row minima prepare_kernel keeps
//    of the non-hole pixels; the hole fill lowers it with the values it
//    writes) and the block's largest gain and smallest read noise when they
//    are maps.  Between passes
//    only replacement changes clean,
//    and replace_kernel lowers the key of the block it writes into, so the key
//    stays a lower bound of the block's values.  Every 5 x 5 median window of
//    a block lies in the block's 3 x 3 neighbourhood of blocks (border-mapped
//    positions included; wrap adds the blocks at the opposite edges, constant
//    adds zero), so the smallest key there bounds every window's median from
//    below, and the model evaluated at it with the block's gain and read noise
//    bounds the noise from below: the model is non-decreasing in the median
//    and in the read noise and non-increasing in the gain;
//  * sig_bulk_kernel (the full first pass): the Laplacian of every pixel against T of
//    its block.  Every pixel whose sig_raw exceeds min(cr, nb) passes (the
//    product is rounded by at most 2^-53 relative, the margin is 1e-12 and
//    the upper bound of the Laplacian used here is never below the
//    reference's value).  Passing pixels are written with that bound to a
//    per-warp region of the `pre` list (no atomics);
//  * classify_kernel: sig_raw of each listed pixel, lap / (2 noise), with the
//    exact noise (error map, or the noise model from the pixel's own 5 x 5
//    median); above cr_threshold -> high candidate list, else above
//    neighbor_threshold -> low list (src/filters.cuh:125-135), and the same
//    classes into the HIGH / LOW planes that incremental passes update.  The
//    candidate kernels recompute every value they threshold exactly.
//
// sig_bulk_kernel is warp-specialised.  One producer thread copies clean row
// segments (BK_COLS columns plus halo columns) into a ring of BK_SLOTS rows in
// shared memory: one `cp.async.bulk` for the 16-byte aligned body of a row
// and up to four single elements with 8-byte `cp.async` (an unaligned first
// or last element, the border columns -1 and w), so rows of any width and
// alignment stream the same way.  A row whose aligned body starts on an odd
// cell is stored one cell to the right (its shift).  Each ring row has a
// "full" mbarrier (the body's transaction bytes plus the producer's cp.async
// arrive) and an "empty" mbarrier on which each of the four consumer warps
// arrives when it is done with the row.  The producer computes the copies of
// an item's rows once per item (they differ by row offsets only), so its
// per-row work is a wait on the row's empty barrier and the issue.  (The S1, S2 and
// CAND planes were zeroed by the call's prologue memset.)  A block takes items
// of BK_COLS x BK_ROWS pixels from a ticket counter (items of frames that
// stopped are skipped there) and the ring runs straight through from one item
// into the next.
//
// The Laplacian (src/filters.cuh:86-105): each consumer thread evaluates four
// consecutive columns x .. x + 3 (lane ct of the four warps: x = x0 + 4 ct)
// and keeps the quarter values of the rows above and at the current row, and
// the current row's left and right neighbours, in registers.  Differences the reference computes twice
// are computed once: down(y) = q(y) - q(y+1) and up(y+1) = q(y+1) - q(y) are
// exact negatives of each other in round-to-nearest, and so are right(x) and
// left(x+1); negation changes at most the sign of a zero difference.
// positive(v) is replaced by an upper bound: v with its high word cleared when
// the sign bit is set (0 or a subnormal instead of the reference's 0 for a
// negative v).  Floating-point addition is monotone, so the sum is never below
// the reference's Laplacian for finite inputs; where a term is NaN the
// reference's sig_raw is NaN and its pixel is never a candidate, and a value
// here only lists a pixel that the candidate kernel drops.
//
// Non-finite input pixels (holes, sig = 0 in the reference) are not tested
// here; the candidate kernel drops candidates that are holes.
//
// Borders (Laplacian border mode: nearest for mirror and reflect): rows
// outside the frame are copied from their border-mapped row, or from a zero
// row in constant mode; columns -1 and w are copied from their border-mapped
// columns (zeros in constant mode), so the evaluation has no border cases.
//
// Every wait is bounded (about one second of SM clock).  A wait that runs out
// sets Control::fault (the loop-control kernel then stops every active frame
// and marks it faulted; the host reports CUSMIC_CUDA_ERROR) and the ring's
// abort word, which ends the block's other waits early; before the block
// exits, its producer waits (again bounded) for the copies it still has in
// flight into shared memory.
#pragma once
#include "detect.cuh"

namespace cb {

constexpr int BK_CWARPS = 4;                     // consumer warps
constexpr int BK_THREADS = 32 * (BK_CWARPS + 1); // plus one producer warp
constexpr int BK_HALF = 64 * BK_CWARPS;          // columns of one pair set (256)
constexpr int BK_COLS = 2 * BK_HALF;             // columns per item (512)
constexpr int BK_ROWS = 32;                      // most rows per item
constexpr int BK_SLOTS = 8;                      // ring rows (power of two)
constexpr int BK_CELLS = BK_COLS + 4;            // cells of a row: columns x0 - 2 .. x0 + BK_COLS + 1
constexpr int BK_STRIDE = BK_CELLS + 2;          // ring row length: room for a shift of one cell
constexpr int BK_BLOCKS_PER_SM = 6;
constexpr int BK_REGION = 4 * 32 * BK_ROWS;      // pre-list entries one consumer warp can write per item
constexpr int FLOOR_BLOCK = 32;                  // noise-floor granularity (square)
constexpr long long BK_WAIT_CYCLES = 1LL << 31;
static_assert((BK_SLOTS & (BK_SLOTS - 1)) == 0, "ring depth must be a power of two");
static_assert(BK_ROWS == FLOOR_BLOCK, "an item spans one row of floor blocks");
static_assert(BK_HALF % FLOOR_BLOCK == 0, "pair sets start on a floor block");
static_assert((BK_STRIDE * 8) % 16 == 0, "ring rows must stay 16-byte aligned");

struct __align__(128) BulkRing {
	double c[BK_SLOTS][BK_STRIDE]; // clean; column x0 - 2 + c at cell c + shift
	int2 meta[BK_SLOTS];           // first ring row of an item: {item index, y1}; index < 0: end
	int shift[BK_SLOTS];           // 0 or 1
	unsigned long long full[BK_SLOTS], empty[BK_SLOTS];
	unsigned long long poison; // never completes (injected failures only)
	int abort;
};

// A pixel that passed the floor test, with its Laplacian bound.
struct PreCand {
	unsigned pixel, frame;
	double lap;
};

// One 32 x 32 block whose floor floor_kernel computes: kind 0 = an error map
// (frames that share a map share its thresholds), 1 = a noise-model frame.
struct FloorJob {
	int frame, x0, y0, kind;
	long long out; // index into the threshold array
};

// Zeros for constant-mode rows and columns outside the frame.
__device__ __align__(16) double bulk_zero_row[BK_CELLS];

__device__ __forceinline__ unsigned smem_u32(const void *p)
{
	return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long *b, unsigned count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long *b, unsigned bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(b)),
		"r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long *b)
{
	asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(b)) : "memory");
}

// Arrive on b once every cp.async this thread issued so far has landed.
__device__ __forceinline__ void mbar_arrive_cp_async(unsigned long long *b)
{
	asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(smem_u32(b)) : "memory");
}

__device__ __forceinline__ bool mbar_test(unsigned long long *b, unsigned parity)
{
	unsigned done;
	asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
		     " selp.u32 %0, 1, 0, p;\n}\n"
		: "=r"(done)
		: "r"(smem_u32(b)), "r"(parity)
		: "memory");
	return done != 0;
}

// Wait until the phase of parity `parity` of barrier b has completed; false
// after about `limit` SM cycles, or as soon as the block aborted.
__device__ __forceinline__ bool mbar_wait(unsigned long long *b, unsigned parity, const int *abort,
	long long limit = BK_WAIT_CYCLES)
{
	if (mbar_test(b, parity))
		return true;
	const long long t0 = clock64();
	for (unsigned i = 1;; ++i) {
		if (mbar_test(b, parity))
			return true;
		if ((i & 15) == 0 && (*(const volatile int *)abort || clock64() - t0 > limit))
			return false;
	}
}

// An injected failure (Control::poison_wait): a wait, bounded by `limit`
// cycles, on barrier b, which was initialised for one arrival that never
// comes.  It runs out and returns false, like a wait whose copies never land.
__device__ __forceinline__ bool poisoned_wait(unsigned long long *b, const int *abort, long long limit)
{
	return mbar_wait(b, 0, abort, limit);
}

// Global -> shared bulk copy completing on barrier bar (16-byte aligned
// addresses, size a multiple of 16).
__device__ __forceinline__ void bulk_copy(void *dst, const void *src, unsigned bytes,
	unsigned long long *bar)
{
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
		::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
		: "memory");
}

// The copies of ring row r of an item starting at column x0 of a w x h frame
// whose clean buffer starts `mis` elements past a 16-byte boundary (0 or 1).
// Cells are relative to the row's shift.
struct BulkRow {
	int shift;         // 0 or 1
	long long src;     // body: element offset into clean (-1: the zero row)
	int cell, n;       // body: destination cell and element count (even, maybe 0)
	// Single-element copies: an unaligned first element (head), an odd last
	// element (tail), columns -1 (left) and w (right).  Source: element
	// offset into clean, -1 for a zero, NO_COPY when there is none.
	long long hsrc, tsrc, lsrc, rsrc;
	int hcell, tcell, lcell, rcell;
	unsigned bytes; // transaction bytes of the body
};
constexpr long long NO_COPY = -2;

CB_HD BulkRow bulk_row(int w, int h, int lm, int mis, int x0, int r)
{
	BulkRow b;
	b.hsrc = b.tsrc = b.lsrc = b.rsrc = NO_COPY;
	b.hcell = b.tcell = b.lcell = b.rcell = 0;
	const int my = border_index(r, h, lm);
	if (my < 0) { // constant mode, row outside the frame
		b.shift = 0;
		b.src = -1;
		b.cell = 0;
		b.n = BK_CELLS;
		b.bytes = 8u * BK_CELLS;
		return b;
	}
	const long long ro = (long long)my * w;
	const int a = x0 - 2 < 0 ? 0 : x0 - 2;
	const int e = x0 + BK_COLS + 2 < w ? x0 + BK_COLS + 2 : w;
	const int head = (int)((mis + ro + a) & 1); // element a is 8 bytes off a 16-byte boundary
	const int a1 = a + head;
	b.shift = a1 & 1; // cell of a1 (x0 is even) made even
	const int len = e - a1 > 0 ? e - a1 : 0;
	b.src = ro + a1;
	b.cell = a1 - x0 + 2 + b.shift;
	b.n = len & ~1;
	b.bytes = 8u * (unsigned)b.n;
	if (head) {
		b.hsrc = ro + a;
		b.hcell = a - x0 + 2 + b.shift;
	}
	if (len & 1) {
		b.tsrc = ro + e - 1;
		b.tcell = e - 1 - x0 + 2 + b.shift;
	}
	if (x0 == 0) { // column -1
		const int mx = border_index(-1, w, lm);
		b.lsrc = mx < 0 ? -1 : ro + mx;
		b.lcell = 1 + b.shift;
	}
	if (w <= x0 + BK_COLS) { // column w
		const int mx = border_index(w, w, lm);
		b.rsrc = mx < 0 ? -1 : ro + mx;
		b.rcell = w - x0 + 2 + b.shift;
	}
	return b;
}

// Floors of 32 x 32 blocks (see the head of this file): of each distinct
// error map (one lane per column, all 32 rows in flight), and of each
// noise-model frame (from prepare_kernel's row minima, one lane per row).
// One warp per block.
//
// Noise-model blocks of frames without gain or read-noise maps are left to
// model_floor_kernel.
__device__ __forceinline__ bool thread_floor_job(const FloorJob &jb, const FrameDesc &fd)
{
	return jb.kind && !fd.gain_map && !fd.rn_map;
}

__device__ __forceinline__ void floor_jobs(const FrameDesc *__restrict__ frames,
	const FloorJob *__restrict__ jobs, int njobs, const DetectParams &prm, BlockFloor *floors)
{
	const int lane = threadIdx.x & 31;
	const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
	const double tmin2 = fmin(prm.thi2, prm.tlo2);
	for (int j = gw; j < njobs; j += nw) {
		const FloorJob jb = jobs[j];
		const FrameDesc &fd = frames[jb.frame];
		if (thread_floor_job(jb, fd))
			continue; // warp-uniform
		const int w = fd.w, x = jb.x0 + lane;
		const int n = (jb.y0 + FLOOR_BLOCK < fd.h ? jb.y0 + FLOOR_BLOCK : fd.h) - jb.y0;
		if (jb.kind) { // noise model: ordered keys of clean, -gain, read noise
			const long long at = (long long)jb.y0 * w + x;
			unsigned long long key = ~0ull, gkey = ~0ull, rkey = ~0ull;
			// Clean: the smallest of the block rows' high words (prepare_kernel;
			// lane = row), as a key with its low word cleared: no larger than
			// the smallest key of the block's non-hole values.
			{
				const uint32_t m = lane < n ? plane_ptr(fd, P_ROWMIN)[(long long)(jb.y0 + lane) * fd.words +
					jb.x0 / 32] : 0xffffffffu;
				const uint32_t hi = __reduce_min_sync(0xffffffffu, m);
				if (hi != 0xffffffffu)
					key = (unsigned long long)hi << 32;
			}
			if (x < w && (fd.gain_map || fd.rn_map))
				for (int k = 0; k < n; ++k) {
					if (fd.gain_map)
						gkey = min(gkey, order_key(-fd.gain_map[at + (long long)k * w]));
					if (fd.rn_map)
						rkey = min(rkey, order_key(fd.rn_map[at + (long long)k * w]));
				}
#pragma unroll
			for (int o = 16; o; o >>= 1) {
				key = min(key, __shfl_xor_sync(0xffffffffu, key, o));
				gkey = min(gkey, __shfl_xor_sync(0xffffffffu, gkey, o));
				rkey = min(rkey, __shfl_xor_sync(0xffffffffu, rkey, o));
			}
			if (lane == 0)
				floors[jb.out] = BlockFloor{0.0, key, gkey, rkey};
			continue;
		}
		const double *col = fd.error + (long long)jb.y0 * w + x;
		double v[FLOOR_BLOCK];
#pragma unroll
		for (int k = 0; k < FLOOR_BLOCK; ++k)
			v[k] = x < w && k < n ? col[(long long)k * w] : INFINITY;
		double m = INFINITY;
#pragma unroll
		for (int k = 0; k < FLOOR_BLOCK; ++k)
			m = dmin(m, v[k] > 0 ? v[k] : 0.0);
#pragma unroll
		for (int o = 16; o; o >>= 1)
			m = dmin(m, __shfl_xor_sync(0xffffffffu, m, o));
		const double T = tmin2 * m;
		if (lane == 0)
			floors[jb.out].thr = T >= 0 ? T : 0.0; // NaN lists everything
	}
}

__global__ void __launch_bounds__(256)
floor_kernel(const FrameDesc *__restrict__ frames, const FloorJob *__restrict__ jobs, int njobs,
	DetectParams prm, BlockFloor *floors)
{
	floor_jobs(frames, jobs, njobs, prm, floors);
}

// Floors of the noise-model blocks of frames without gain or read-noise maps,
// one thread per block: the smallest of the block rows' high words
// (prepare_kernel's row minima) as a key with its low word cleared.
__global__ void __launch_bounds__(256)
model_floor_kernel(const FrameDesc *__restrict__ frames, const FloorJob *__restrict__ jobs, int njobs,
	BlockFloor *floors)
{
	for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < njobs; j += gridDim.x * blockDim.x) {
		const FloorJob jb = jobs[j];
		const FrameDesc &fd = frames[jb.frame];
		if (!thread_floor_job(jb, fd))
			continue;
		const int n = min(FLOOR_BLOCK, fd.h - jb.y0);
		const uint32_t *m = plane_ptr(fd, P_ROWMIN) + (long long)jb.y0 * fd.words + jb.x0 / 32;
		uint32_t hi = 0xffffffffu;
#pragma unroll 8
		for (int k = 0; k < n; ++k)
			hi = min(hi, m[(long long)k * fd.words]);
		floors[jb.out] = BlockFloor{0.0, hi != 0xffffffffu ? (unsigned long long)hi << 32 : ~0ull,
			~0ull, ~0ull};
	}
}

__device__ __forceinline__ int nbr_block(int b, int n, int i, bool wrap)
{
	// i = 0..2: b - 1 .. b + 1; i = 3..6 (wrap mode near an edge only): the two
	// blocks at each edge.  -1: none.
	if (i < 3)
		return b - 1 + i >= 0 && b - 1 + i < n ? b - 1 + i : -1;
	if (!wrap || (b > 1 && b < n - 2))
		return -1;
	const int v = i == 3 ? 0 : i == 4 ? 1 : i == 5 ? n - 2 : n - 1;
	return v >= 0 && v < n ? v : -1;
}

__device__ __forceinline__ double model_threshold(const FrameDesc &fd, int bx, int by, int mode,
	double tmin2)
{
	const BlockFloor *bf = fd.floors;
	const int w = fd.w, h = fd.h;
	const int bw = (w + FLOOR_BLOCK - 1) / FLOOR_BLOCK, bh = (h + FLOOR_BLOCK - 1) / FLOOR_BLOCK;
	const bool wrap = mode == WRAP;
	unsigned long long key = ~0ull;
	for (int i = 0; i < 7; ++i) {
		const int yy = nbr_block(by, bh, i, wrap);
		if (yy < 0)
			continue;
		for (int j = 0; j < 7; ++j) {
			const int xx = nbr_block(bx, bw, j, wrap);
			if (xx >= 0)
				key = min(key, bf[yy * bw + xx].key);
		}
	}
	// In constant mode a window reaching past the frame holds zeros.
	if (mode == CONSTANT && (bx == 0 || by == 0 || (bx + 1) * FLOOR_BLOCK + 2 > w ||
		(by + 1) * FLOOR_BLOCK + 2 > h))
		key = min(key, order_key(0.0));
	double m = order_value(key);
	m = m < SIGNAL_FLOOR ? SIGNAL_FLOOR : m;
	const BlockFloor &own = bf[by * bw + bx];
	const double g = fd.gain_map ? -order_value(own.gkey) : fd.gain;
	const double rn = fd.rn_map ? order_value(own.rkey) : fd.rn;
	return tmin2 * (sqrt(rn * rn + g * m) / g);
}

// Upper bound of positive(v): v when its sign bit is clear; otherwise the
// high word cleared (0 or a subnormal).
__device__ __forceinline__ double pos_ub(double v)
{
	const int hi = __double2hiint(v);
	return __hiloint2double(hi & ~(hi >> 31), __double2loint(v));
}

__device__ __forceinline__ unsigned hi_word(double v)
{
	return (unsigned)__double2hiint(v);
}

// The copies of an in-frame row `by` elements (a whole number of row pairs)
// away from the row b describes: only the element offsets into clean change
// (-1, a zero, stays).
__device__ __forceinline__ BulkRow shift_row(BulkRow b, long long by)
{
	b.src += by;
	if (b.hsrc >= 0)
		b.hsrc += by;
	if (b.tsrc >= 0)
		b.tsrc += by;
	if (b.lsrc >= 0)
		b.lsrc += by;
	if (b.rsrc >= 0)
		b.rsrc += by;
	return b;
}

// Issue the copies of one ring row (one thread: the bulk copy completes on
// the row's full barrier by its transaction bytes, the single-element copies
// by the thread's cp.async arrival).
__device__ __forceinline__ void bulk_issue(BulkRing &R, int slot, const BulkRow &b, const double *clean)
{
	double *row = R.c[slot];
	R.shift[slot] = b.shift;
	mbar_expect_tx(&R.full[slot], b.bytes);
	if (b.n)
		bulk_copy(row + b.cell, b.src < 0 ? bulk_zero_row : clean + b.src, 8u * b.n, &R.full[slot]);
	if (b.hsrc != NO_COPY)
		cp_async8(row + b.hcell, clean + b.hsrc);
	if (b.tsrc != NO_COPY)
		cp_async8(row + b.tcell, clean + b.tsrc);
	if (b.lsrc != NO_COPY)
		cp_async8(row + b.lcell, b.lsrc < 0 ? bulk_zero_row : clean + b.lsrc);
	if (b.rsrc != NO_COPY)
		cp_async8(row + b.rcell, b.rsrc < 0 ? bulk_zero_row : clean + b.rsrc);
	mbar_arrive_cp_async(&R.full[slot]);
}

// Producer of sig_bulk_kernel: one thread (lane 0 of the producer warp); g
// counts the ring rows issued.  Returns false after a fault.  The copies of
// an item's in-frame rows differ only by their row offsets, in two classes
// by row parity (the 16-byte phase of a row start alternates when w is odd),
// so they are computed once per item (kept in `base`, shared memory); rows
// outside the frame (border-mapped or zero) are computed on their own.
__device__ __forceinline__ bool bulk_producer(BulkRing &R, const FrameDesc *__restrict__ frames,
	const FrameState *__restrict__ state, const int4 *__restrict__ items, int nitems, int lm,
	Control *ctl, int &g, BulkRow (&base)[2])
{
	int next = atomicAdd(&ctl->ticket, 1);
	for (;;) {
		// Next active item.
		int t = -1;
		while (next < nitems) {
			const int cand = next;
			next = atomicAdd(&ctl->ticket, 1);
			const int4 it = items[cand];
			if (!state[it.x].active)
				continue;
			if ((uintptr_t)frames[it.x].clean & 7) // the host rejects such buffers
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
		const int w = fd.w, h = fd.h, x0 = it.y, y0 = it.z;
		const int y1 = it.w; // items never cross a 32-row floor block
		const double *clean = fd.clean;
		const int mis = (int)(((uintptr_t)clean >> 3) & 1);
		const int ra = y0 - 1 < 0 ? 0 : y0 - 1; // first in-frame row of the item
		base[0] = bulk_row(w, h, lm, mis, x0, ra);
		base[1] = bulk_row(w, h, lm, mis, x0, ra + 1 < h ? ra + 1 : ra);
		for (int r = y0 - 1; r <= y1; ++r) {
			const int slot = g & (BK_SLOTS - 1);
			const int d = r - ra;
			const BulkRow b = r < 0 || r >= h ? bulk_row(w, h, lm, mis, x0, r)
				: shift_row(base[d & 1], (long long)(d & ~1) * w);
			if (g >= BK_SLOTS && !mbar_wait(&R.empty[slot], ((g / BK_SLOTS) - 1) & 1, &R.abort))
				return false;
			if (r == y0 - 1)
				R.meta[slot] = make_int2(t, y1);
			bulk_issue(R, slot, b, clean);
			++g;
		}
	}
}

// Columns x - 1 .. x + 2 of a ring row (x = the pair's first column, at cell
// c + shift; c even, so every 16-byte load is aligned).
__device__ __forceinline__ void load_quad(const double *row, int c, int shift, double &l, double &a,
	double &b, double &r)
{
	if (shift == 0) {
		const double2 v = *reinterpret_cast<const double2 *>(row + c);
		l = row[c - 1];
		a = v.x;
		b = v.y;
		r = row[c + 2];
	} else {
		const double2 v0 = *reinterpret_cast<const double2 *>(row + c);
		const double2 v1 = *reinterpret_cast<const double2 *>(row + c + 2);
		l = v0.x;
		a = v0.y;
		b = v1.x;
		r = v1.y;
	}
}

// Columns x - 1 .. x + 4 of a ring row (x = the lane's first column, at cell
// c + shift; c even, so every 16-byte load is aligned).
__device__ __forceinline__ void load_six(const double *row, int c, int shift, double (&v)[6])
{
	if (shift == 0) {
		const double2 a = *reinterpret_cast<const double2 *>(row + c);
		const double2 b = *reinterpret_cast<const double2 *>(row + c + 2);
		v[0] = row[c - 1];
		v[1] = a.x;
		v[2] = a.y;
		v[3] = b.x;
		v[4] = b.y;
		v[5] = row[c + 4];
	} else {
		const double2 a = *reinterpret_cast<const double2 *>(row + c);
		const double2 b = *reinterpret_cast<const double2 *>(row + c + 2);
		const double2 d = *reinterpret_cast<const double2 *>(row + c + 4);
		v[0] = a.x;
		v[1] = a.y;
		v[2] = b.x;
		v[3] = b.y;
		v[4] = d.x;
		v[5] = d.y;
	}
}

// Consumer warps of sig_bulk_kernel: lane ct of the four warps evaluates
// columns x0 + 4 ct .. x0 + 4 ct + 3.  Returns false after a fault.
__device__ __forceinline__ bool bulk_consumer(BulkRing &R, const FrameDesc *__restrict__ frames,
	const int4 *__restrict__ items, const DetectParams &prm, PreCand *pre, int *pre_counts)
{
	const double tmin2 = fmin(prm.thi2, prm.tlo2);
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
		// High word of the block threshold per column (all ones: not a pixel).
		unsigned thr[4];
		{
			unsigned tv = 0xffffffffu;
			if (x < w) {
				const int bx = x / FLOOR_BLOCK, by = y0 / FLOOR_BLOCK;
				const double T = fd.error ? fd.floors[by * ((w + FLOOR_BLOCK - 1) / FLOOR_BLOCK) + bx].thr
					: model_threshold(fd, bx, by, prm.mode, tmin2);
				tv = hi_word(T >= 0 ? T : 0.0); // NaN lists everything
			}
#pragma unroll
			for (int i = 0; i < 4; ++i)
				thr[i] = x + i < w ? tv : 0xffffffffu;
		}
		ok = __all_sync(0xffffffffu,
			mbar_wait(&R.full[(g + 1) & (BK_SLOTS - 1)], ((g + 1) / BK_SLOTS) & 1, &R.abort));
		if (!ok)
			break;
		// Row y0 - 1 (values) and row y0 (values and neighbours), as quarters.
		double q[4], up[4], ql, qr;
		{
			double u[6], c[6];
			load_six(R.c[g & (BK_SLOTS - 1)], c0, R.shift[g & (BK_SLOTS - 1)], u);
			load_six(R.c[(g + 1) & (BK_SLOTS - 1)], c0, R.shift[(g + 1) & (BK_SLOTS - 1)], c);
			ql = c[0] * 0.25;
			qr = c[5] * 0.25;
#pragma unroll
			for (int i = 0; i < 4; ++i) {
				q[i] = c[i + 1] * 0.25;
				up[i] = q[i] - u[i + 1] * 0.25;
			}
		}
		__syncwarp();
		if (lane == 0) { // both rows are in registers now
			mbar_arrive(&R.empty[g & (BK_SLOTS - 1)]);
			mbar_arrive(&R.empty[(g + 1) & (BK_SLOTS - 1)]);
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
			__syncwarp();
			if (lane == 0)
				mbar_arrive(&R.empty[sd]); // row y + 1 is in registers
			// Horizontal differences: left(x+i) = h[i], right(x+i) = -h[i+1].
			double h[5];
			h[0] = q[0] - ql;
#pragma unroll
			for (int i = 0; i < 3; ++i)
				h[i + 1] = q[i] - q[i + 1];
			h[4] = q[3] - qr;
			const long long pix0 = (long long)y * w + x;
			// The four columns' Laplacians first (independent chains), then
			// the list appends.
			double lap[4];
#pragma unroll
			for (int i = 0; i < 4; ++i) {
				const double qd = n[i + 1] * 0.25;
				const double d = q[i] - qd;
				const double lft = i == 0 ? h[0] : -h[i], rgt = i == 3 ? h[4] : h[i + 1];
				lap[i] = (pos_ub(up[i] + lft) + pos_ub(up[i] + rgt)) +
					(pos_ub(d + lft) + pos_ub(d + rgt));
				up[i] = -d;
				q[i] = qd;
			}
			ql = n[0] * 0.25;
			qr = n[5] * 0.25;
			bool pass[4];
#pragma unroll
			for (int i = 0; i < 4; ++i)
				pass[i] = hi_word(lap[i]) >= thr[i];
			if (__any_sync(0xffffffffu, pass[0] | pass[1] | pass[2] | pass[3])) {
#pragma unroll
				for (int i = 0; i < 4; ++i) {
					const unsigned bal = __ballot_sync(0xffffffffu, pass[i]);
					if (pass[i])
						region[cnt + __popc(bal & below)] =
							PreCand{(unsigned)(pix0 + i), (unsigned)f, lap[i]};
					cnt += __popc(bal);
				}
			}
		}
		if (!ok)
			break;
		if (lane == 0)
			pre_counts[t * BK_CWARPS + warp] = cnt;
		g += y1 - y0 + 2;
	}
	return ok;
}

__global__ void __launch_bounds__(BK_THREADS, BK_BLOCKS_PER_SM)
sig_bulk_kernel(const FrameDesc *__restrict__ frames, const FrameState *__restrict__ state,
	const int4 *__restrict__ items, int nitems, DetectParams prm, Control *ctl, PreCand *pre,
	int *pre_counts)
{
	__shared__ BulkRing R;
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
	bool ok;
	int issued = 0; // ring rows issued (producer warp)
	if (warp == BK_CWARPS)
		ok = lane || bulk_producer(R, frames, state, items, nitems, lap_mode(prm.mode), ctl, issued,
			base);
	else if (warp == 0 && blockIdx.x == 0 && ctl->poison_wait[1] > 0)
		ok = __all_sync(0xffffffffu, poisoned_wait(&R.poison, &R.abort, ctl->poison_wait[1]));
	else
		ok = bulk_consumer(R, frames, items, prm, pre, pre_counts);
	if (!ok && lane == 0) {
		R.abort = 1;
		atomicOr(&ctl->fault, 1);
	}
	__syncthreads();
	// After a fault: wait (bounded) for the copies still in flight into this
	// block's shared memory (on the normal path the consumers waited for every
	// issued row).
	if (warp == BK_CWARPS && lane == 0 && R.abort)
		for (int q = issued - BK_SLOTS < 0 ? 0 : issued - BK_SLOTS; q < issued; ++q) {
			const long long t0 = clock64();
			while (!mbar_test(&R.full[q & (BK_SLOTS - 1)], (q / BK_SLOTS) & 1) &&
				clock64() - t0 < BK_WAIT_CYCLES) {
			}
		}
}

// Candidates staged in shared memory by classify_kernel before one global
// append per block and list.
constexpr int CL_CAP = 1024;

struct ClassifyStage {
	uint2 buf[CL_CAP];
	int n;    // slots reserved
	int fail; // first reservation that did not fit (entries from there went straight out)
};

// Stage the lanes whose `pred` holds (entry e); a reservation that does not
// fit appends those entries to the global list directly.
__device__ __forceinline__ void classify_stage(ClassifyStage &S, bool pred, uint2 e,
	unsigned long long *counter, uint2 *cands, bool from_back, unsigned long long cap)
{
	const int lane = threadIdx.x & 31;
	const unsigned b = __ballot_sync(0xffffffffu, pred);
	if (!b)
		return;
	const int k = __popc(b), rank = __popc(b & ((1u << lane) - 1u));
	int old = 0;
	if (lane == 0)
		old = atomicAdd(&S.n, k);
	old = __shfl_sync(0xffffffffu, old, 0);
	if (old + k <= CL_CAP) {
		if (pred)
			S.buf[old + rank] = e;
		return;
	}
	unsigned long long base = 0;
	if (lane == 0) {
		atomicMin(&S.fail, old);
		base = atomicAdd(counter, (unsigned long long)k);
	}
	base = __shfl_sync(0xffffffffu, base, 0);
	if (pred)
		cands[from_back ? cap - 1 - (base + rank) : base + rank] = e;
}

// Write a stage out with one atomic per list (block-uniform call).
__device__ __forceinline__ void classify_flush(ClassifyStage &H, ClassifyStage &L, Control *ctl,
	uint2 *cands, unsigned long long *bases)
{
	__syncthreads();
	const int nh = min(H.n, H.fail), nl = min(L.n, L.fail);
	if (threadIdx.x == 0) {
		bases[0] = nh ? atomicAdd(&ctl->n_cand, (unsigned long long)nh) : 0ull;
		bases[1] = nl ? atomicAdd(&ctl->n_low, (unsigned long long)nl) : 0ull;
	}
	__syncthreads();
	const unsigned long long cap = ctl->cand_cap;
	for (int i = threadIdx.x; i < nh; i += blockDim.x)
		cands[bases[0] + i] = H.buf[i];
	for (int i = threadIdx.x; i < nl; i += blockDim.x)
		cands[cap - 1 - (bases[1] + i)] = L.buf[i];
	__syncthreads();
	if (threadIdx.x == 0) {
		H.n = L.n = 0;
		H.fail = L.fail = CL_CAP;
	}
	__syncthreads();
}

// sig_raw of the listed pixels, lap / (2 noise) (src/filters.cuh:125-135),
// with the error map or the exact noise model at the pixel: one warp per
// consumer-warp region of an item, one lane per entry.  The high list grows
// from the front of the candidate buffer, the low list from its back; a NaN
// goes to the high list (the candidate kernel decides).  Error-map entries
// listed with a bound of +inf get their exact Laplacian first.
__global__ void __launch_bounds__(256, 4)
classify_kernel(const FrameDesc *__restrict__ frames, const FrameState *__restrict__ state,
	const int4 *__restrict__ items, int nitems, const PreCand *__restrict__ pre,
	const int *__restrict__ pre_counts, DetectParams prm, Control *ctl, uint2 *cands)
{
	__shared__ ClassifyStage H, L;
	__shared__ unsigned long long bases[2];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	// After a bounded wait of the dense kernel ran out, the counts of the
	// items it left are stale: list nothing (the loop control then stops
	// every frame and the call reports the fault).
	if (*(const volatile int *)&ctl->fault)
		return;
	if (threadIdx.x == 0) {
		H.n = L.n = 0;
		H.fail = L.fail = CL_CAP;
	}
	__syncthreads();
	const unsigned long long cap = ctl->cand_cap;
	const int nreg = nitems * BK_CWARPS;
	for (int base = blockIdx.x * 8; base < nreg; base += gridDim.x * 8) { // block-uniform
		const int rg = base + warp;
		const int f = rg < nreg ? items[rg / BK_CWARPS].x : 0;
		if (rg < nreg && state[f].active) { // warp-uniform
			const int n = pre_counts[rg];
			const FrameDesc &fd = frames[f];
			const PreCand *e = pre + (long long)rg * BK_REGION;
			for (int k0 = 0; k0 < n; k0 += 32) {
				int cls = 0;
				unsigned pix = 0;
				if (k0 + lane < n) {
					const PreCand pc = e[k0 + lane];
					pix = pc.pixel;
					if (fd.error) {
						// A bound of +inf marks a pixel whose Laplacian reads a hole
						// (prep_detect_kernel) or overflowed: the exact Laplacian of
						// the filled working pixels.
						const double lap = pc.lap != INFINITY ? pc.lap
							: lap_at(fd, (int)(pix % (unsigned)fd.w), (int)(pix / (unsigned)fd.w),
								lap_mode(prm.mode));
						const double v = lap / (2 * fd.error[pix]);
						cls = v > prm.cr || v != v ? 1 : v > prm.nb ? 2 : 0;
					} else {
						const int px = (int)(pix % (unsigned)fd.w), py = (int)(pix / (unsigned)fd.w);
						double nz;
						if (px >= 2 && py >= 2 && px + 2 < fd.w && py + 2 < fd.h) {
							double win[25];
							const double *src = fd.clean + pix - 2 * (long long)fd.w - 2;
#pragma unroll
							for (int a = 0; a < 5; ++a)
#pragma unroll
								for (int b = 0; b < 5; ++b)
									win[a * 5 + b] = src[(long long)a * fd.w + b];
							nz = noise_from_median(fd, pix, median_network(win));
						} else {
							nz = noise_model_at(fd, px, py, prm.mode);
						}
						const double v = pc.lap / (2 * nz);
						cls = v > prm.cr || v != v ? 1 : v > prm.nb ? 2 : 0;
					}
					// The class planes that incremental passes keep up to date.
					if (cls) {
						const unsigned px = pix % (unsigned)fd.w, py = pix / (unsigned)fd.w;
						atomicOr(plane_ptr(fd, cls == 1 ? P_HIGH : P_LOW) +
							(long long)py * fd.words + (px >> 5), 1u << (px & 31));
					}
				}
				const uint2 entry = make_uint2((unsigned)f, pix);
				classify_stage(H, cls == 1, entry, &ctl->n_cand, cands, false, cap);
				classify_stage(L, cls == 2, entry, &ctl->n_low, cands, true, cap);
			}
		}
		__syncthreads();
		const bool full = H.n >= CL_CAP / 2 || L.n >= CL_CAP / 2;
		__syncthreads(); // every thread has read the counts before any stages again
		if (full)
			classify_flush(H, L, ctl, cands, bases);
	}
	classify_flush(H, L, ctl, cands, bases);
}

} // namespace cb

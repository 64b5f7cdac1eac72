// Dense detection for error-map frames whose rows can be moved by the bulk
// copy engine: clean 16-byte aligned and an even width (so every row starts on
// a 16-byte boundary).
//
// What the pass needs from every pixel is only whether its sig_raw =
// lap / (2 error) can exceed min(cr_threshold, neighbor_threshold); the exact
// value matters for the ~1% of pixels where it can.  So the work is split:
//
//  * errfloor_kernel (once per call): the floor of every 32 x 32 block of each
//    distinct error map, floor = min(max(error, 0)) (NaN counts as 0);
//  * sig_bulk_kernel (every pass): the Laplacian of every pixel, compared with
//    2 min(cr, nb) (1 - 1e-12) x floor of its block.  Since error >= floor,
//    every pixel whose sig_raw exceeds min(cr, nb) passes (the product is
//    rounded by at most 2^-53 relative, the margin is 1e-12); the error map
//    itself is not read.  Passing pixels are written with their Laplacian to
//    a per-warp region of the `pre` list;
//  * classify_kernel: sig_raw = lap / (2 error) in the reference's operation
//    order for each listed pixel; above cr_threshold -> high candidate list,
//    else above neighbor_threshold -> low list (src/filters.cuh:125-135).
//
// sig_bulk_kernel is warp-specialised.  One producer warp issues
// `cp.async.bulk` copies of whole clean row segments (BK_COLS columns plus a
// 2-column halo on each side) into a ring of BK_SLOTS rows in shared memory,
// one "full" mbarrier per ring row (transaction bytes); it also clears the
// S1/S2/CAND bit words of the rows it issues.  Four consumer warps evaluate
// the rows; each of them arrives on the ring row's "empty" mbarrier when it
// is done with it, which lets the producer reuse the row.  A block takes
// items of BK_COLS x BK_ROWS pixels from a ticket counter (items of frames
// that stopped are skipped there) and the ring runs straight through from one
// item into the next.
//
// The Laplacian (src/filters.cuh:86-105): each consumer thread evaluates two
// column pairs (x, x + 1) and (x + 256, x + 257) and keeps the quarter values
// of the rows above and at the current row in registers.  Differences the
// reference computes twice are computed once: down(y) = q(y) - q(y+1) and
// up(y+1) = q(y+1) - q(y) are exact negatives of each other in
// round-to-nearest, and so are right(x) and left(x+1).  Negation changes at
// most the sign of a zero difference.  positive(v) keeps v when its sign bit
// is clear and gives +0 otherwise (integer operations): equal to the
// reference's `v < 0 ? 0 : v` for every non-NaN v up to the sign of a zero.
// No zero sign reaches a strict comparison with a threshold, so for finite
// inputs the listed Laplacian is the reference's value; where a term is NaN
// the reference's sig_raw is NaN and its pixel is never a candidate, and a
// finite value here only lists a pixel that the candidate kernel drops.
//
// Non-finite input pixels (holes, sig = 0 in the reference) are not tested
// here; the candidate kernel drops candidates that are holes.
//
// Borders (Laplacian border mode: nearest for mirror and reflect): rows
// outside the frame are copied from their border-mapped row, or from a zero
// row in constant mode.  Columns -1 and w come from 16-byte copies of columns
// w-2..w-1 and 0..1 (wrap) or of zeros (constant); in nearest mode the thread
// at the frame edge uses its own column instead.
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
constexpr int BK_ROWS = 32;                      // rows per item
constexpr int BK_SLOTS = 8;                      // ring rows (power of two)
constexpr int BK_CELLS = BK_COLS + 4;            // cells of a ring row: columns x0 - 2 .. x0 + BK_COLS + 1
constexpr int BK_BLOCKS_PER_SM = 6;
constexpr int BK_REGION = 4 * 32 * BK_ROWS;      // pre-list entries one consumer warp can write per item
constexpr int FLOOR_BLOCK = 32;                  // error-map floor granularity (square)
constexpr long long BK_WAIT_CYCLES = 1LL << 31;
static_assert((BK_SLOTS & (BK_SLOTS - 1)) == 0, "ring depth must be a power of two");
static_assert(BK_ROWS == FLOOR_BLOCK, "an item spans one row of floor blocks");
static_assert(BK_HALF % FLOOR_BLOCK == 0, "pair sets start on a floor block");

struct __align__(128) BulkRing {
	double c[BK_SLOTS][BK_CELLS]; // clean (4128 B per row: a multiple of 16)
	int2 meta[BK_SLOTS];          // first ring row of an item: {item index, y1}; index < 0: end
	unsigned long long full[BK_SLOTS], empty[BK_SLOTS];
	int abort;
};

// A pixel that passed the floor test, with its Laplacian.
struct PreCand {
	unsigned pixel, frame;
	double lap;
};

// One 32 x 32 block of a frame's error map whose floor errfloor_kernel
// computes (frames sharing a map share its floors: one job per block of each
// distinct map).
struct FloorJob {
	int frame, x0, y0, pad;
	long long out; // index into the floor array
};

// Zeros for constant-mode rows outside the frame and constant-mode halos.
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
// after about BK_WAIT_CYCLES SM cycles, or as soon as the block aborted.
__device__ __forceinline__ bool mbar_wait(unsigned long long *b, unsigned parity, const int *abort)
{
	if (mbar_test(b, parity))
		return true;
	const long long t0 = clock64();
	for (unsigned i = 1;; ++i) {
		if (mbar_test(b, parity))
			return true;
		if ((i & 15) == 0 && (*(const volatile int *)abort || clock64() - t0 > BK_WAIT_CYCLES))
			return false;
	}
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

// What ring row r of an item starting at column x0 needs copied: the clean
// cells [cell, cell + n) from clean + src (elements) and up to two 16-byte
// halo chunks.
struct BulkRow {
	long long src;  // element offset into clean of the main copy (-1: zero row)
	int cell, n;    // destination cell and element count of the main copy
	long long lsrc; // halo chunk at cells 0..1: -1 none, -2 zeros, else clean offset
	long long rsrc; // halo chunk at cells rcell..rcell+1: -1 none, -2 zeros, else clean offset
	int rcell;
	unsigned bytes; // transaction bytes of the row
};

CB_HD BulkRow bulk_row(int w, int h, int lm, int x0, int r)
{
	BulkRow b;
	const int my = border_index(r, h, lm);
	b.lsrc = b.rsrc = -1;
	b.rcell = 0;
	if (my < 0) { // constant mode, row outside the frame
		b.src = -1;
		b.cell = 0;
		b.n = BK_CELLS;
	} else {
		const int a = x0 - 2 < 0 ? 0 : x0 - 2;
		const int e = x0 + BK_COLS + 2 < w ? x0 + BK_COLS + 2 : w;
		b.src = (long long)my * w + a;
		b.cell = a - (x0 - 2);
		b.n = e - a;
		if (lm != NEAREST) {
			if (x0 == 0)
				b.lsrc = lm == WRAP ? (long long)my * w + w - 2 : -2;
			if (w <= x0 + BK_COLS) {
				b.rsrc = lm == WRAP ? (long long)my * w : -2;
				b.rcell = w - x0 + 2;
			}
		}
	}
	b.bytes = 8u * (unsigned)b.n + (b.lsrc != -1 ? 16u : 0u) + (b.rsrc != -1 ? 16u : 0u);
	return b;
}

// One warp per 32 x 32 block: floor = min over the block of max(error, 0),
// with NaN counted as 0.
__global__ void __launch_bounds__(256)
errfloor_kernel(const FrameDesc *__restrict__ frames, const FloorJob *__restrict__ jobs, int njobs,
	double *floors)
{
	const int lane = threadIdx.x & 31;
	const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
	for (int j = gw; j < njobs; j += nw) {
		const FloorJob jb = jobs[j];
		const FrameDesc &fd = frames[jb.frame];
		const int w = fd.w, x = jb.x0 + lane;
		const int y1 = jb.y0 + FLOOR_BLOCK < fd.h ? jb.y0 + FLOOR_BLOCK : fd.h;
		double m = INFINITY;
		if (x < w)
			for (int y = jb.y0; y < y1; ++y) {
				const double v = fd.error[(long long)y * w + x];
				m = dmin(m, v > 0 ? v : 0.0);
			}
#pragma unroll
		for (int o = 16; o; o >>= 1)
			m = dmin(m, __shfl_xor_sync(0xffffffffu, m, o));
		if (lane == 0)
			floors[jb.out] = m;
	}
}

// positive(v) on the sign bit: v if it is clear, +0 otherwise.
__device__ __forceinline__ double pos_bits(double v)
{
	const long long b = __double_as_longlong(v);
	return __longlong_as_double(b & ~(b >> 63));
}

__device__ __forceinline__ unsigned hi_word(double v)
{
	return (unsigned)((unsigned long long)__double_as_longlong(v) >> 32);
}

// Producer warp of sig_bulk_kernel: returns false after a fault.
__device__ __forceinline__ bool bulk_producer(BulkRing &R, const FrameDesc *__restrict__ frames,
	const FrameState *__restrict__ state, const int4 *__restrict__ items, int nitems, int lm,
	Control *ctl, int &g)
{
	const int lane = threadIdx.x & 31;
	int next = 0;
	bool ok = true;
	if (lane == 0)
		next = atomicAdd(&ctl->ticket, 1);
	for (;;) {
		// Next active item (lane 0 decides, the warp follows).
		int t = -1;
		if (lane == 0) {
			while (next < nitems) {
				const int cand = next;
				next = atomicAdd(&ctl->ticket, 1);
				const int4 it = items[cand];
				if (!state[it.x].active)
					continue;
				const FrameDesc &fd = frames[it.x];
				// The host lists only frames whose rows are 16-byte aligned;
				// a descriptor that breaks this is reported, never copied.
				if ((fd.w & 1) || ((uintptr_t)fd.clean & 15))
					ok = false;
				else
					t = cand;
				break;
			}
		}
		if (!__shfl_sync(0xffffffffu, ok, 0))
			return false;
		t = __shfl_sync(0xffffffffu, t, 0);
		if (t < 0) { // end of the list: an end marker in the next ring row
			if (lane == 0) {
				const int slot = g & (BK_SLOTS - 1);
				ok = g < BK_SLOTS || mbar_wait(&R.empty[slot], ((g / BK_SLOTS) - 1) & 1, &R.abort);
				if (ok) {
					R.meta[slot] = make_int2(-1, 0);
					mbar_arrive(&R.full[slot]);
					++g;
				}
			}
			return __shfl_sync(0xffffffffu, ok, 0);
		}
		const int4 it = items[t];
		const FrameDesc &fd = frames[it.x];
		const int w = fd.w, h = fd.h, words = fd.words, x0 = it.y, y0 = it.z;
		const int y1 = y0 + BK_ROWS < h ? y0 + BK_ROWS : h;
		const double *clean = fd.clean;
		uint32_t *s1 = plane_ptr(fd, P_S1);
		const long long plane = fd.plane;
		for (int r = y0 - 1; r <= y1; ++r) {
			if (lane == 0) {
				const int slot = g & (BK_SLOTS - 1);
				ok = g < BK_SLOTS || mbar_wait(&R.empty[slot], ((g / BK_SLOTS) - 1) & 1, &R.abort);
				if (ok) {
					if (r == y0 - 1)
						R.meta[slot] = make_int2(t, y1);
					const BulkRow b = bulk_row(w, h, lm, x0, r);
					unsigned long long *bar = &R.full[slot];
					mbar_expect_tx(bar, b.bytes);
					bulk_copy(&R.c[slot][b.cell], b.src < 0 ? bulk_zero_row : clean + b.src,
						8u * b.n, bar);
					if (b.lsrc != -1)
						bulk_copy(&R.c[slot][0], b.lsrc < 0 ? bulk_zero_row : clean + b.lsrc, 16u,
							bar);
					if (b.rsrc != -1)
						bulk_copy(&R.c[slot][b.rcell], b.rsrc < 0 ? bulk_zero_row : clean + b.rsrc,
							16u, bar);
					++g;
				}
			}
			if (!__shfl_sync(0xffffffffu, ok, 0))
				return false;
			// Clear the S1, S2 and CAND words of the item's rows (16 words per
			// plane per row).
			if (r >= y0 && r < y1)
				for (int q = lane; q < 48; q += 32) {
					const int word = (x0 >> 5) + (q & 15);
					if (word < words)
						s1[(q >> 4) * plane + (long long)r * words + word] = 0u;
				}
		}
	}
}

// Consumer warps of sig_bulk_kernel: returns false after a fault.
__device__ __forceinline__ bool bulk_consumer(BulkRing &R, const FrameDesc *__restrict__ frames,
	const int4 *__restrict__ items, const double *__restrict__ floors, const DetectParams &prm,
	int lm, PreCand *pre, int *pre_counts)
{
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const int ct = warp * 32 + lane; // 0 .. 127
	const unsigned below = (1u << lane) - 1u;
	const double tmin2 = fmin(prm.thi2, prm.tlo2);
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
		const int w = frames[f].w;
		const int bw = (w + FLOOR_BLOCK - 1) / FLOOR_BLOCK;
		const double *frow = floors + it.w + (long long)(y0 / FLOOR_BLOCK) * bw;
		// Pair sets p = 0, 1: columns xs[p] = x0 + 256 p + 2 ct and xs[p] + 1.
		int xs[2];
		bool nl[2], nr[2];
		unsigned thr[2];
#pragma unroll
		for (int p = 0; p < 2; ++p) {
			xs[p] = x0 + BK_HALF * p + 2 * ct;
			const bool valid = xs[p] < w;
			nl[p] = lm == NEAREST && xs[p] == 0;
			nr[p] = lm == NEAREST && xs[p] + 2 == w;
			double T = valid ? tmin2 * frow[xs[p] / FLOOR_BLOCK] : 0.0;
			T = T >= 0 ? T : 0.0; // NaN (0 x inf) lists everything
			thr[p] = valid ? hi_word(T) : 0xffffffffu;
		}
		ok = __all_sync(0xffffffffu,
			mbar_wait(&R.full[(g + 1) & (BK_SLOTS - 1)], ((g + 1) / BK_SLOTS) & 1, &R.abort));
		if (!ok)
			break;
		double qa[2], qb[2], upa[2], upb[2];
#pragma unroll
		for (int p = 0; p < 2; ++p) {
			const int cell = 2 + BK_HALF * p + 2 * ct;
			const double2 u = *reinterpret_cast<const double2 *>(&R.c[g & (BK_SLOTS - 1)][cell]);
			const double2 c = *reinterpret_cast<const double2 *>(&R.c[(g + 1) & (BK_SLOTS - 1)][cell]);
			qa[p] = c.x * 0.25;
			qb[p] = c.y * 0.25;
			upa[p] = qa[p] - u.x * 0.25;
			upb[p] = qb[p] - u.y * 0.25;
		}
		__syncwarp();
		if (lane == 0)
			mbar_arrive(&R.empty[g & (BK_SLOTS - 1)]); // row y0 - 1
		PreCand *region = pre + ((long long)t * BK_CWARPS + warp) * BK_REGION;
		int cnt = 0;
		for (int y = y0; y < y1; ++y) {
			const int gd = g + 2 + (y - y0); // ring rows of y + 1 (gd) and y (gd - 1)
			const int sd = gd & (BK_SLOTS - 1), sc = (gd - 1) & (BK_SLOTS - 1);
			ok = __all_sync(0xffffffffu, mbar_wait(&R.full[sd], (gd / BK_SLOTS) & 1, &R.abort));
			if (!ok)
				break;
			const long long rowpix = (long long)y * w;
#pragma unroll
			for (int p = 0; p < 2; ++p) {
				const int cell = 2 + BK_HALF * p + 2 * ct;
				const double2 dn = *reinterpret_cast<const double2 *>(&R.c[sd][cell]);
				double ql = R.c[sc][cell - 1] * 0.25, qr = R.c[sc][cell + 2] * 0.25;
				ql = nl[p] ? qa[p] : ql;
				qr = nr[p] ? qb[p] : qr;
				const double qda = dn.x * 0.25, qdb = dn.y * 0.25;
				const double da = qa[p] - qda, db = qb[p] - qdb;
				const double hl = qa[p] - ql, hab = qa[p] - qb[p], hr = qb[p] - qr;
				const double lap_a = (pos_bits(upa[p] + hl) + pos_bits(upa[p] + hab)) +
					(pos_bits(da + hl) + pos_bits(da + hab));
				const double lap_b = (pos_bits(upb[p] - hab) + pos_bits(upb[p] + hr)) +
					(pos_bits(db - hab) + pos_bits(db + hr));
				const bool pa = hi_word(lap_a) >= thr[p], pb = hi_word(lap_b) >= thr[p];
				const unsigned ba = __ballot_sync(0xffffffffu, pa);
				if (ba) {
					if (pa)
						region[cnt + __popc(ba & below)] =
							PreCand{(unsigned)(rowpix + xs[p]), (unsigned)f, lap_a};
					cnt += __popc(ba);
				}
				const unsigned bb = __ballot_sync(0xffffffffu, pb);
				if (bb) {
					if (pb)
						region[cnt + __popc(bb & below)] =
							PreCand{(unsigned)(rowpix + xs[p] + 1), (unsigned)f, lap_b};
					cnt += __popc(bb);
				}
				upa[p] = -da;
				upb[p] = -db;
				qa[p] = qda;
				qb[p] = qdb;
			}
			__syncwarp();
			if (lane == 0)
				mbar_arrive(&R.empty[sc]); // row y
		}
		if (!ok)
			break;
		__syncwarp();
		if (lane == 0) {
			mbar_arrive(&R.empty[(g + y1 - y0 + 1) & (BK_SLOTS - 1)]); // row y1
			pre_counts[t * BK_CWARPS + warp] = cnt;
		}
		g += y1 - y0 + 2;
	}
	return ok;
}

__global__ void __launch_bounds__(BK_THREADS, BK_BLOCKS_PER_SM)
sig_bulk_kernel(const FrameDesc *__restrict__ frames, const FrameState *__restrict__ state,
	const int4 *__restrict__ items, int nitems, const double *__restrict__ floors,
	DetectParams prm, Control *ctl, PreCand *pre, int *pre_counts)
{
	__shared__ BulkRing R;
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int lm = lap_mode(prm.mode);
	if (tid == 0) {
		for (int i = 0; i < BK_SLOTS; ++i) {
			mbar_init(&R.full[i], 1);
			mbar_init(&R.empty[i], BK_CWARPS);
		}
		R.abort = 0;
		asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
	}
	__syncthreads();

	bool ok = true;
	int issued = 0; // ring rows issued (producer lane 0)
	if (warp == BK_CWARPS)
		ok = bulk_producer(R, frames, state, items, nitems, lm, ctl, issued);
	else
		ok = bulk_consumer(R, frames, items, floors, prm, lm, pre, pre_counts);
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

// Exact sig_raw of the listed pixels (src/filters.cuh:125-135, lap / (2 *
// noise)): one warp per consumer-warp region of an item, one lane per entry;
// the high list grows from the front of the candidate buffer, the low list
// from its back.
__global__ void __launch_bounds__(256)
classify_kernel(const FrameDesc *__restrict__ frames, const FrameState *__restrict__ state,
	const int4 *__restrict__ items, int nitems, const PreCand *__restrict__ pre,
	const int *__restrict__ pre_counts, DetectParams prm, Control *ctl, uint2 *cands)
{
	const int lane = threadIdx.x & 31;
	const unsigned below = (1u << lane) - 1u;
	const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
	const int nreg = nitems * BK_CWARPS;
	for (int rg = gw; rg < nreg; rg += nw) {
		const int f = items[rg / BK_CWARPS].x;
		if (!state[f].active)
			continue; // warp-uniform: the region was not written this pass
		const int n = pre_counts[rg];
		const double *error = frames[f].error;
		const PreCand *e = pre + (long long)rg * BK_REGION;
		for (int k0 = 0; k0 < n; k0 += 32) {
			int cls = 0;
			unsigned pix = 0;
			if (k0 + lane < n) {
				const PreCand pc = e[k0 + lane];
				pix = pc.pixel;
				const double v = pc.lap / (2 * error[pc.pixel]);
				cls = v > prm.cr ? 1 : v > prm.nb ? 2 : 0;
			}
			const unsigned bh = __ballot_sync(0xffffffffu, cls == 1);
			const unsigned bl = __ballot_sync(0xffffffffu, cls == 2);
			if (bh) {
				unsigned long long base = 0;
				if (lane == 0)
					base = atomicAdd(&ctl->n_cand, (unsigned long long)__popc(bh));
				base = __shfl_sync(0xffffffffu, base, 0);
				if (cls == 1)
					cands[base + __popc(bh & below)] = make_uint2((unsigned)f, pix);
			}
			if (bl) {
				unsigned long long base = 0;
				if (lane == 0)
					base = atomicAdd(&ctl->n_low, (unsigned long long)__popc(bl));
				base = __shfl_sync(0xffffffffu, base, 0);
				if (cls == 2)
					cands[ctl->cand_cap - 1 - (base + __popc(bl & below))] = make_uint2((unsigned)f, pix);
			}
		}
	}
}

} // namespace cb
